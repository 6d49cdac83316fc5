/* Stand-in for src/nemo/Neuron.hpp: a neuron's parameters and state. */
#ifndef NEMO_NEURON_HPP
#define NEMO_NEURON_HPP
#include <cstddef>
#include <vector>
#include <nemo/config.h>
#include "NeuronType.hpp"
namespace nemo {
class NEMO_BASE_DLL_PUBLIC Neuron
{
	public :
		Neuron() { }
		Neuron(const std::vector<float>& param, const std::vector<float>& state) : m_param(param), m_state(state) {}
		const float* getParameters() const { return m_param.empty() ? NULL : &m_param[0]; }
		const float* getState() const { return m_state.empty() ? NULL : &m_state[0]; }
	private :
		std::vector<float> m_param;
		std::vector<float> m_state;
};
}
#endif
