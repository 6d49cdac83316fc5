/* Stand-in for src/nemo/SimulationBackend.hpp: the interface a backend
 * implements (the step() overloads are implemented once, for every
 * backend, in terms of the others). */
#ifndef NEMO_SIMULATION_BACKEND_HPP
#define NEMO_SIMULATION_BACKEND_HPP
#include "Simulation.hpp"
#include "internal_types.h"
#include "FiringBuffer.hpp"
namespace nemo {
class NEMO_BASE_DLL_PUBLIC SimulationBackend : public Simulation
{
	public :
		virtual ~SimulationBackend() { }
		virtual unsigned getFractionalBits() const = 0;
		virtual void setFiringStimulus(const std::vector<unsigned>& nidx) = 0;
		virtual void initCurrentStimulus(size_t count) = 0;
		virtual void addCurrentStimulus(unsigned, float) = 0;
		virtual void finalizeCurrentStimulus(size_t count) = 0;
		virtual void setCurrentStimulus(const std::vector<float>& current) = 0;
		virtual void prefire() = 0;
		virtual void fire() = 0;
		virtual void postfire() = 0;
		const firing_output& step();
		const firing_output& step(const firing_stimulus&);
		const firing_output& step(const current_stimulus&);
		const firing_output& step(const firing_stimulus&, const current_stimulus&);
		virtual void applyStdp(float reward) = 0;
		virtual FiredList readFiring() = 0;
	protected :
		SimulationBackend() { }
};
}
#endif
