/* Stand-in for src/nemo/NeuronType.hpp: the accessors the backend adapter
 * uses.  The reference reads the counts from the type's .ini descriptor;
 * the stand-in takes them from its constructor. */
#ifndef NEMO_NEURON_TYPE_HPP
#define NEMO_NEURON_TYPE_HPP
#include <stddef.h>
#include <string>
#include <nemo/config.h>
namespace nemo {
class NEMO_BASE_DLL_PUBLIC NeuronType
{
	public :
		NeuronType(const std::string& name, size_t nParam, size_t nState) :
			m_nParam(nParam), m_nState(nState), m_name(name) {}
		size_t parameterCount() const { return m_nParam; }
		size_t stateVarCount() const { return m_nState; }
		std::string name() const { return m_name; }
	private :
		size_t m_nParam;
		size_t m_nState;
		std::string m_name;
};
}
#endif
