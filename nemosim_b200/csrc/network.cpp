// network.cpp -- host-side network and configuration objects.
#include "network.hpp"
#include "plugins.hpp"

#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>

#include <algorithm>

namespace nemo_b200 {

std::string format(const char* fmt, ...)
{
	char buf[1024];
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(buf, sizeof buf, fmt, ap);
	va_end(ap);
	return std::string(buf);
}

/* src/nemo/fixedpoint.cpp:17-28 */
int32_t fx_toFix(float f)
{
	int i = (int) f;
	if(abs(i) >= (1 << (31 - FRACTIONAL_BITS))) {
		throw std::runtime_error(format("Fixed-point overflow. Value %g does not fit into fixed-point format Q%u.%u",
				(double) f, 31 - FRACTIONAL_BITS, FRACTIONAL_BITS));
	}
	return (int32_t) (f * (float) (1 << FRACTIONAL_BITS));
}

/* NetworkImpl::addNeuronType, src/nemo/NetworkImpl.cpp:37-48: a type seen
 * before in this network keeps its id; a new one is read from its .ini
 * descriptor (parseNeuronType) */
unsigned Network::addNeuronType(const std::string& name)
{
	for(unsigned t = 0; t < types.size(); ++t) {
		if(name == types[t].desc->name) return t;
	}
	NeuronCollection c;
	c.desc = std::make_shared<const NeuronTypeDesc>(parseNeuronType(name));
	types.push_back(c);
	return (unsigned) types.size() - 1;
}

/* NetworkImpl::addNeuron (src/nemo/NetworkImpl.cpp:84-92) and Neurons::add
 * (src/nemo/Neurons.cpp:29-48): the neuron is appended before the
 * duplicate-index check, so a duplicate also makes simulation creation fail,
 * as in the reference. */
void Network::addNeurons(unsigned type, size_t n, const unsigned* idx, unsigned nargs, const float* args)
{
	if(type >= types.size()) NB_THROW(NEMO_INVALID_INPUT, "Invalid neuron type id %u", type);
	NeuronCollection& c = types[type];
	unsigned na = c.nargs();
	if(nargs != na) {
		NB_THROW(NEMO_INVALID_INPUT,
				"Unexpected number of parameters/state variables when adding neuron. Expected %u, found %u", na, nargs);
	}
	if(c.gidx.size() + n > c.gidx.capacity()) {
		c.gidx.reserve(std::max(c.gidx.size() + n, 2 * c.gidx.capacity()));
		c.args.reserve(std::max(c.args.size() + n * na, 2 * c.args.capacity()));
	}
	for(size_t i = 0; i < n; ++i) {
		c.gidx.push_back(idx[i]);
		c.args.insert(c.args.end(), args + i * na, args + (i + 1) * na);
		uint64_t v = ((uint64_t) type << 32) | (uint64_t) (c.gidx.size() - 1);
		if(!neurons.emplace(idx[i], v).second) {
			duplicate = true;
			duplicateIdx = idx[i];
			NB_THROW(NEMO_INVALID_INPUT, "Duplicate neuron index %u", idx[i]);
		}
	}
}

/* NetworkImpl::addSynapse, src/nemo/NetworkImpl.cpp:105-130 */
void Network::addSynapses(size_t n, const unsigned* s, const unsigned* t, const unsigned* d,
		const float* w, const unsigned char* p, uint64_t* ids)
{
	m_synIndexValid = false;
	const size_t base = src.size();
	const size_t need = base + n;
	if(need > src.capacity()) {
		size_t cap = std::max(need, src.capacity() * 2);
		src.reserve(cap); tgt.reserve(cap); delay.reserve(cap);
		weight.reserve(cap); plastic.reserve(cap); sid.reserve(cap);
	}
	src.resize(need); tgt.resize(need); delay.resize(need);
	weight.resize(need); plastic.resize(need); sid.resize(need);
	unsigned lastSrc = 0;
	uint32_t* lastCount = nullptr;
	for(size_t i = 0; i < n; ++i) {
		if(d[i] < 1) {
			// roll back this call's partial additions
			for(size_t j = 0; j < i; ++j) axonCount[s[j]]--;
			src.resize(base); tgt.resize(base); delay.resize(base);
			weight.resize(base); plastic.resize(base); sid.resize(base);
			NB_THROW(NEMO_INVALID_INPUT, "Invalid delay (%u) for synapse between %u and %u", d[i], s[i], t[i]);
		}
		if(!lastCount || s[i] != lastSrc) {
			lastSrc = s[i];
			lastCount = &axonCount[s[i]];
		}
		uint32_t id = (*lastCount)++;
		const size_t k = base + i;
		src[k] = s[i];
		tgt[k] = t[i];
		delay[k] = d[i];
		weight[k] = w[i];
		plastic[k] = p[i] != 0;
		sid[k] = id;
		if(d[i] > maxDelay) maxDelay = d[i];
		if(ids) ids[i] = ((uint64_t) s[i] << 32) | id;
	}
}

unsigned Network::neuronCount() const
{
	size_t total = 0;
	for(const NeuronCollection& c : types) total += c.size();
	return (unsigned) total;
}

float& Network::neuronArg(unsigned idx, unsigned k, bool state)
{
	auto it = neurons.find(idx);
	if(it == neurons.end()) NB_THROW(NEMO_INVALID_INPUT, "Non-existing neuron index %u", idx);
	NeuronCollection& c = types[it->second >> 32];
	size_t i = it->second & 0xffffffffu;
	if(state) {
		if(k >= c.desc->nstate) NB_THROW(NEMO_INVALID_INPUT, "Invalid state variable index %u", k);
		return c.args[i * c.nargs() + c.desc->nparam + k];
	}
	if(k >= c.desc->nparam) NB_THROW(NEMO_INVALID_INPUT, "Invalid parameter index %u", k);
	return c.args[i * c.nargs() + k];
}

/* src/nemo/Neurons.cpp:78-95 */
void Network::setNeuron(unsigned idx, unsigned nargs, const float* args)
{
	auto it = neurons.find(idx);
	if(it == neurons.end()) NB_THROW(NEMO_INVALID_INPUT, "Non-existing neuron index %u", idx);
	NeuronCollection& c = types[it->second >> 32];
	size_t i = it->second & 0xffffffffu;
	if(nargs != c.nargs()) {
		NB_THROW(NEMO_INVALID_INPUT,
				"Unexpected number of parameters/state variables when modifying neuron. Expected %u, found %u", c.nargs(), nargs);
	}
	for(unsigned k = 0; k < nargs; ++k) c.args[i * nargs + k] = args[k];
}

float Network::getNeuronState(unsigned idx, unsigned var) const
{
	return const_cast<Network*>(this)->neuronArg(idx, var, true);
}

float Network::getNeuronParameter(unsigned idx, unsigned param) const
{
	return const_cast<Network*>(this)->neuronArg(idx, param, false);
}

void Network::setNeuronState(unsigned idx, unsigned var, float val) { neuronArg(idx, var, true) = val; }
void Network::setNeuronParameter(unsigned idx, unsigned param, float val) { neuronArg(idx, param, false) = val; }

void Network::buildSynapseIndex()
{
	if(m_synIndexValid) return;
	m_synIndex.clear();
	for(auto& kv : axonCount) m_synIndex[kv.first].resize(kv.second);
	for(size_t k = 0; k < src.size(); ++k) m_synIndex[src[k]][sid[k]] = k;
	m_synIndexValid = true;
}

/* NetworkImpl::axon + Axon::getSynapse (src/nemo/NetworkImpl.cpp:170-180, Axon.cpp:22-30) */
size_t Network::synapsePos(uint64_t id)
{
	buildSynapseIndex();
	unsigned source = (unsigned) (id >> 32);
	uint32_t s = (uint32_t) (id & 0xffffffffu);
	auto it = m_synIndex.find(source);
	if(it == m_synIndex.end()) NB_THROW(NEMO_INVALID_INPUT, "synapses of non-existing neuron (%u) requested", source);
	if(s >= it->second.size()) NB_THROW(NEMO_INVALID_INPUT, "synapse id out or range");
	return it->second[s];
}

const std::vector<uint64_t>& Network::getSynapsesFrom(unsigned source)
{
	m_queried.clear();
	auto it = axonCount.find(source);
	if(it != axonCount.end()) {
		m_queried.resize(it->second);
		for(uint32_t i = 0; i < it->second; ++i) m_queried[i] = ((uint64_t) source << 32) | i;
	}
	return m_queried;
}

unsigned Network::getSynapseTarget(uint64_t id) { return tgt[synapsePos(id)]; }
unsigned Network::getSynapseDelay(uint64_t id) { return delay[synapsePos(id)]; }
float Network::getSynapseWeight(uint64_t id) { return weight[synapsePos(id)]; }
unsigned char Network::getSynapsePlastic(uint64_t id) { return plastic[synapsePos(id)]; }

/* src/nemo/StdpFunction.cpp:12-47 */
void Configuration::setStdpFunction(const float* pre, size_t npre, const float* post, size_t npost,
		float minE_, float maxE_, float minI_, float maxI_)
{
	if(maxI_ > 0.0f || minI_ > 0.0f)
		NB_THROW(NEMO_INVALID_INPUT, "STDP function should not have positive limits for inhibitory synapses");
	if(maxE_ < 0.0f || minE_ < 0.0f)
		NB_THROW(NEMO_INVALID_INPUT, "STDP function should not have negative limits for inhibitory synapses");
	if(maxE_ < minE_)
		NB_THROW(NEMO_INVALID_INPUT, "STDP should have maximum excitatory weight >= minimum excitatory weight");
	if(maxI_ > minI_)
		NB_THROW(NEMO_INVALID_INPUT, "STDP should have abs(maximum inhibitory weight) >= abs(minimum inhibitory weight)");
	if(npre + npost > MAX_HISTORY) NB_THROW(NEMO_INVALID_INPUT, "size of STDP window too large");
	prefire.assign(pre, pre + npre);
	postfire.assign(post, post + npost);
	minE = minE_; maxE = maxE_; minI = minI_; maxI = maxI_;
	stdp = true;
}

} // namespace nemo_b200
