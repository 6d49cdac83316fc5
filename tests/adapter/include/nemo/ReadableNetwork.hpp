/* Stand-in for src/nemo/ReadableNetwork.hpp */
#ifndef NEMO_READABLE_NETWORK_HPP
#define NEMO_READABLE_NETWORK_HPP
#include <vector>
#include <nemo/config.h>
#include <nemo/types.h>
namespace nemo {
class NEMO_BASE_DLL_PUBLIC ReadableNetwork
{
	public :
		virtual ~ReadableNetwork() { }
		unsigned getSynapseSource(const synapse_id& id) const;
		virtual unsigned getSynapseTarget(const synapse_id&) const = 0;
		virtual unsigned getSynapseDelay(const synapse_id&) const = 0;
		virtual float getSynapseWeight(const synapse_id&) const = 0;
		virtual unsigned char getSynapsePlastic(const synapse_id&) const = 0;
		virtual const std::vector<synapse_id>& getSynapsesFrom(unsigned neuron) = 0;
};
}
#endif
