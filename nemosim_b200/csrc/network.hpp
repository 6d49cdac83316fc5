// network.hpp -- host-side network and configuration objects behind the
// C API (the roles of nemo::NetworkImpl, src/nemo/NetworkImpl.hpp, and
// nemo::ConfigurationImpl, src/nemo/ConfigurationImpl.hpp).
#pragma once

#include <stdint.h>

#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "common.hpp"
#include "hugevec.hpp"

namespace nemo_b200 {

struct NeuronCollection {
	std::shared_ptr<const NeuronTypeDesc> desc;
	std::vector<unsigned> gidx;  // insertion order
	std::vector<float> args;     // row-major: size() x (nparam + nstate)
	unsigned nargs() const { return desc->nparam + desc->nstate; }
	size_t size() const { return gidx.size(); }
};

class Network {
public:
	unsigned addNeuronType(const std::string& name);
	void addNeurons(unsigned type, size_t n, const unsigned* idx, unsigned nargs, const float* args);
	void addSynapses(size_t n, const unsigned* src, const unsigned* tgt, const unsigned* delay,
			const float* weight, const unsigned char* plastic, uint64_t* ids);
	unsigned neuronCount() const;

	/* neuron queries and updates (src/nemo/NetworkImpl.cpp:96-166) */
	void setNeuron(unsigned idx, unsigned nargs, const float* args);
	float getNeuronState(unsigned idx, unsigned var) const;
	float getNeuronParameter(unsigned idx, unsigned param) const;
	void setNeuronState(unsigned idx, unsigned var, float val);
	void setNeuronParameter(unsigned idx, unsigned param, float val);

	/* synapse queries (src/nemo/NetworkImpl.cpp:184-226) */
	const std::vector<uint64_t>& getSynapsesFrom(unsigned source);
	unsigned getSynapseTarget(uint64_t id);
	unsigned getSynapseDelay(uint64_t id);
	float getSynapseWeight(uint64_t id);
	unsigned char getSynapsePlastic(uint64_t id);

	std::vector<NeuronCollection> types;
	std::unordered_map<unsigned, uint64_t> neurons;  // gidx -> (type << 32) | index
	std::unordered_map<unsigned, uint32_t> axonCount; // source gidx -> number of synapses
	// synapses in insertion order
	hvector<unsigned> src, tgt, delay;
	hvector<float> weight;
	hvector<uint8_t> plastic;
	hvector<uint32_t> sid;  // per-source synapse index
	unsigned maxDelay = 0;
	bool duplicate = false;
	unsigned duplicateIdx = 0;

private:
	size_t synapsePos(uint64_t id);
	void buildSynapseIndex();
	// lazily built: source gidx -> positions of its synapses, by synapse index
	std::unordered_map<unsigned, std::vector<size_t>> m_synIndex;
	bool m_synIndexValid = false;
	float& neuronArg(unsigned idx, unsigned k, bool state);
	std::vector<uint64_t> m_queried;
};

struct Configuration {
	bool stdp = false;
	std::vector<float> prefire, postfire;
	float minE = 0, maxE = 0, minI = 0, maxI = 0;
	bool writeOnlySynapses = false;
	// build the connectivity on the device where the network allows it
	bool deviceConstruction = true;
	bool logging = false;
	backend_t backend = NEMO_BACKEND_CUDA;
	int device = -1;
	std::string description;

	/* StdpFunction ctor checks, src/nemo/StdpFunction.cpp:12-47 */
	void setStdpFunction(const float* pre, size_t npre, const float* post, size_t npost,
			float minE, float maxE, float minI, float maxI);
};

} // namespace nemo_b200
