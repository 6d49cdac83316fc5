/* Stand-in for src/nemo/FiringBuffer.hpp: one cycle's fired neurons. */
#ifndef NEMO_FIRING_BUFFER_HPP
#define NEMO_FIRING_BUFFER_HPP
#include <vector>
#include <nemo/config.h>
#include <nemo/types.h>
namespace nemo {
struct NEMO_BASE_DLL_PUBLIC FiredList
{
	cycle_t cycle;
	std::vector<unsigned>& neurons;
	FiredList(cycle_t cycle, std::vector<unsigned>& neurons) : cycle(cycle), neurons(neurons) { }
};
}
#endif
