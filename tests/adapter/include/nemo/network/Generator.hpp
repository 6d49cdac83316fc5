/* Stand-in for src/nemo/network/Generator.hpp: the read-only network
 * interface a backend is built from. */
#ifndef NEMO_NETWORK_GENERATOR_HPP
#define NEMO_NETWORK_GENERATOR_HPP
#include <nemo/config.h>
#include <nemo/types.hpp>
#include <nemo/network/iterator.hpp>
#include <nemo/NeuronType.hpp>
namespace nemo {
	namespace network {
class NEMO_BASE_DLL_PUBLIC Generator
{
	public :
		virtual ~Generator() { }
		typedef std::pair<nidx_t, Neuron> neuron;
		typedef Synapse synapse;
		virtual neuron_iterator neuron_begin(unsigned i) const = 0;
		virtual neuron_iterator neuron_end(unsigned i) const = 0;
		virtual synapse_iterator synapse_begin() const = 0;
		virtual synapse_iterator synapse_end() const = 0;
		virtual unsigned neuronCount() const = 0;
		virtual unsigned neuronCount(unsigned type) const = 0;
		virtual unsigned maxDelay() const = 0;
		virtual unsigned minNeuronIndex() const = 0;
		virtual unsigned maxNeuronIndex() const = 0;
		virtual unsigned neuronTypeCount() const = 0;
		virtual const class NeuronType& neuronType(unsigned i) const = 0;
};
	}
}
#endif
