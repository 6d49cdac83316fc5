// driver.cpp -- test driver of the backend adapter (test infrastructure).
//
// Builds networks as a reference network::Generator (a vector-backed
// stand-in), creates the backend through the adapter's cuda_simulation, and
// drives it only through the nemo::SimulationBackend interface, as libnemo
// does: step() (prefire / stimulus / fire / postfire / readFiring),
// applyStdp and the queries.  The checks are the reference's own
// known-answer tests (src/test/test.cpp ring and current stimulus,
// src/test/stdp.cpp testStdp) and the comparison of the C++ and C paths
// (src/test/c_api.cpp compareWithCpp).
//
//   driver nodevice   without a GPU: configuration and creation fail with
//                     the reference's status codes
//   driver gpu        on a GPU: the known-answer tests
//
// Prints "ok" and exits 0 on success; prints the failure and exits 1.
#include <nemo/ConfigurationImpl.hpp>
#include <nemo/SimulationBackend.hpp>
#include <nemo/exception.hpp>
#include <nemo/network/Generator.hpp>

#include "nemo_b200.h"

#include <math.h>
#include <stdio.h>
#include <string.h>

#include <memory>
#include <random>
#include <string>
#include <unordered_map>
#include <vector>

extern "C" nemo::SimulationBackend* cuda_simulation(const nemo::network::Generator*, const nemo::ConfigurationImpl*);
extern "C" void cuda_set_configuration(nemo::ConfigurationImpl*, int);

#define REQUIRE(cond)                                                                 \
	do {                                                                              \
		if(!(cond)) {                                                                 \
			fprintf(stderr, "%s:%d: requirement failed: %s\n", __FILE__, __LINE__, #cond); \
			exit(1);                                                                  \
		}                                                                             \
	} while(0)

namespace {

template<class T>
class VectorIterator : public nemo::network::abstract_iterator<T>
{
public:
	VectorIterator(const std::vector<T>* v, size_t i) : m_v(v), m_i(i) {}
	const T& operator*() const { return (*m_v)[m_i]; }
	const T* operator->() const { return &(*m_v)[m_i]; }
	nemo::network::abstract_iterator<T>* clone() const { return new VectorIterator(m_v, m_i); }
	nemo::network::abstract_iterator<T>& operator++() { ++m_i; return *this; }
	bool operator==(const nemo::network::abstract_iterator<T>& o) const
	{
		const VectorIterator* x = dynamic_cast<const VectorIterator*>(&o);
		return x && x->m_v == m_v && x->m_i == m_i;
	}
	bool operator!=(const nemo::network::abstract_iterator<T>& o) const { return !(*this == o); }
private:
	const std::vector<T>* m_v;
	size_t m_i;
};

// a network held in vectors, in insertion order
class VectorGenerator : public nemo::network::Generator
{
public:
	unsigned addType(const std::string& name, size_t np, size_t ns)
	{
		m_types.emplace_back(name, np, ns);
		m_neurons.emplace_back();
		return (unsigned) m_types.size() - 1;
	}
	void addNeuron(unsigned type, unsigned idx, const std::vector<float>& param, const std::vector<float>& state)
	{
		m_neurons[type].emplace_back(idx, nemo::Neuron(param, state));
	}
	void addSynapse(unsigned src, unsigned tgt, unsigned delay, float w, bool plastic)
	{
		const unsigned id = m_outCount[src]++;  // the per-source synapse index
		m_synapses.emplace_back(src, delay, nemo::AxonTerminal(id, tgt, w, plastic));
		if(delay > m_maxDelay) m_maxDelay = delay;
	}

	nemo::network::neuron_iterator neuron_begin(unsigned t) const
	{
		return nemo::network::neuron_iterator(new VectorIterator<neuron>(&m_neurons[t], 0));
	}
	nemo::network::neuron_iterator neuron_end(unsigned t) const
	{
		return nemo::network::neuron_iterator(new VectorIterator<neuron>(&m_neurons[t], m_neurons[t].size()));
	}
	nemo::network::synapse_iterator synapse_begin() const
	{
		return nemo::network::synapse_iterator(new VectorIterator<nemo::Synapse>(&m_synapses, 0));
	}
	nemo::network::synapse_iterator synapse_end() const
	{
		return nemo::network::synapse_iterator(new VectorIterator<nemo::Synapse>(&m_synapses, m_synapses.size()));
	}
	unsigned neuronCount() const
	{
		size_t n = 0;
		for(const auto& v : m_neurons) n += v.size();
		return (unsigned) n;
	}
	unsigned neuronCount(unsigned t) const { return (unsigned) m_neurons[t].size(); }
	unsigned maxDelay() const { return m_maxDelay; }
	unsigned minNeuronIndex() const { return 0; }
	unsigned maxNeuronIndex() const { return neuronCount() - 1; }
	unsigned neuronTypeCount() const { return (unsigned) m_types.size(); }
	const nemo::NeuronType& neuronType(unsigned i) const { return m_types[i]; }

private:
	std::vector<nemo::NeuronType> m_types;
	std::vector<std::vector<neuron>> m_neurons;
	std::vector<nemo::Synapse> m_synapses;
	std::unordered_map<unsigned, unsigned> m_outCount;
	unsigned m_maxDelay = 0;
};

// createRing (src/test/utils.cpp:132-145): neuron i -> i + 1, weight 1000
void ring(VectorGenerator& net, unsigned n, unsigned delay)
{
	const unsigned iz = net.addType("Izhikevich", 5, 2);
	const float v = -65.0f, b = 0.2f, r = 0.5f;
	for(unsigned i = 0; i < n; ++i) {
		net.addNeuron(iz, i, { 0.02f, b, v + 15.0f * r * r, 8.0f - 6.0f * r * r, 0.0f }, { b * v, v });
	}
	for(unsigned i = 0; i < n; ++i) net.addSynapse(i, (i + 1) % n, delay, 1000.0f, false);
}

void testConfiguration()
{
	nemo::ConfigurationImpl conf;
	cuda_set_configuration(&conf, -1);
	REQUIRE(conf.backend() == NEMO_BACKEND_CUDA);
	REQUIRE(conf.cudaDevice() == 0);
	REQUIRE(conf.cudaPartitionSize() == 1024);
	REQUIRE(strlen(conf.backendDescription()) > 0);
	bool threw = false;
	try {
		cuda_set_configuration(&conf, 1 << 20);
	} catch(nemo::exception& e) {
		threw = e.errorNumber() == NEMO_CUDA_ERROR;
	}
	REQUIRE(threw);
}

// runRing (src/test/test.cpp:300-325) through step(fstim) and step()
void testRing()
{
	const unsigned n = 1000;
	VectorGenerator net;
	ring(net, n, 1);
	nemo::ConfigurationImpl conf;
	std::unique_ptr<nemo::SimulationBackend> sim(cuda_simulation(&net, &conf));
	const std::vector<unsigned>& f0 = sim->step(std::vector<unsigned>{ 0 });
	REQUIRE(f0.size() == 1 && f0[0] == 0);
	for(unsigned ms = 1; ms < 2 * n; ++ms) {
		const std::vector<unsigned>& f = sim->step();
		REQUIRE(f.size() == 1 && f[0] == ms % n);
	}
	REQUIRE(sim->elapsedSimulation() == 2 * n);
	sim->resetTimer();
	REQUIRE(sim->elapsedSimulation() == 0);
	// queries through the interface
	const std::vector<synapse_id>& ids = sim->getSynapsesFrom(7);
	REQUIRE(ids.size() == 1);
	REQUIRE(sim->getSynapseSource(ids[0]) == 7);
	REQUIRE(sim->getSynapseTarget(ids[0]) == 8);
	REQUIRE(sim->getSynapseDelay(ids[0]) == 1);
	REQUIRE(sim->getSynapseWeight(ids[0]) == 1000.0f);
	REQUIRE(sim->getSynapsePlastic(ids[0]) == 0);
	REQUIRE(sim->getNeuronParameter(3, 0) == 0.02f);
	REQUIRE(sim->getMembranePotential(3) == sim->getNeuronState(3, 1));
	sim->setNeuronState(3, 1, -70.0f);
	REQUIRE(sim->getNeuronState(3, 1) == -70.0f);
	bool threw = false;
	try {
		sim->getNeuronState(n + 5, 0);
	} catch(nemo::exception& e) {
		threw = e.errorNumber() == NEMO_INVALID_INPUT;
	}
	REQUIRE(threw);
}

// testCurrentStimulus (src/test/test.cpp:244-268) through step(istim)
void testCurrentStimulus()
{
	const unsigned n = 1500;
	VectorGenerator net;
	ring(net, n, 1);
	nemo::ConfigurationImpl conf;
	std::unique_ptr<nemo::SimulationBackend> sim(cuda_simulation(&net, &conf));
	nemo::Simulation::current_stimulus istim = { { 5, 0.001f }, { 8, 0.001f }, { 0, 1000.0f }, { 100, 0.001f } };
	sim->step(istim);
	for(unsigned ms = 1; ms < n; ++ms) {
		const std::vector<unsigned>& f = sim->step();
		REQUIRE(f.size() == 1 && f[0] == ms % n);
	}
}

// testStdp (src/test/stdp.cpp:197-265) through step(fstim), applyStdp and
// getSynapseWeight, with reward 1.0
void testStdp()
{
	const unsigned group = 2 * 768;
	const float initW = 5.0f;
	VectorGenerator net;
	const unsigned iz = net.addType("Izhikevich", 5, 2);
	const float r = 0.5f, b = 0.25f - 0.05f * r, v = -65.0f;
	for(unsigned g = 0; g < 2; ++g) {
		for(unsigned l = 0; l < group; ++l) {
			net.addNeuron(iz, g * group + l, { 0.02f + 0.08f * r, b, v, 2.0f, 0.0f }, { b * v, v });
		}
	}
	for(unsigned l = 0; l < group; ++l) net.addSynapse(l, group + l, 1 + l % 20, initW, true);
	std::vector<float> pre(20), post(20);
	for(unsigned dt = 0; dt < 20; ++dt) {
		pre[dt] = 1.0f * expf(-(float) dt / 20.0f);
		post[dt] = -0.8f * expf(-(float) dt / 20.0f);
	}
	nemo::ConfigurationImpl conf;
	conf.setStdpFunction(pre, post, 0.0f, 10.0f, 0.0f, -0.5f);
	std::unique_ptr<nemo::SimulationBackend> sim(cuda_simulation(&net, &conf));
	REQUIRE(sim->getFractionalBits() == 20);
	std::vector<unsigned> g0, g1;
	for(unsigned l = 0; l < group; ++l) {
		g0.push_back(l);
		g1.push_back(group + l);
	}
	for(unsigned epoch = 1; epoch <= 4; ++epoch) {
		for(unsigned ms = 0; ms < 100; ++ms) {
			if(ms == 10) sim->step(g0);
			else if(ms == 20) sim->step(g1);
			else sim->step();
		}
		sim->applyStdp(1.0f);
		for(unsigned l = 0; l < group; ++l) {
			const synapse_id id = sim->getSynapsesFrom(l)[0];
			const unsigned d = sim->getSynapseDelay(id);
			REQUIRE(d == 1 + l % 20);
			REQUIRE(sim->getSynapsePlastic(id));
			const int dt = -(10 - (int) d);
			const double dw = dt > 0 ? -0.8 * exp(-(dt - 1) / 20.0) : 1.0 * exp(dt / 20.0);
			const double expect = initW + epoch * dw;
			const double got = sim->getSynapseWeight(id);
			REQUIRE(fabs(got - expect) <= 1e-5 * fabs(expect));
		}
	}
}

// compareWithCpp (src/test/c_api.cpp:236-330): the same partially random
// network of 1000 Izhikevich neurons x 1000 synapses (80% excitatory,
// sigma 5 and 2), built once through the reference's C++ network
// interface and run through the adapter's backend, and once through the C
// API, for 2000 steps with an optional firing and current stimulus at
// cycle 0: the fire streams are identical.  The C run reads a synapse back
// every 100 steps, as the reference's does.
void testCompareWithC(bool useFstim, bool useIstim)
{
	const unsigned ncount = 1000, scount = 1000, steps = 2000;
	std::mt19937 rng(5489u);
	auto param = [&]() { return (float) ((double) rng() / 4294967296.0); };
	auto target = [&]() { return (unsigned) (rng() % ncount); };
	VectorGenerator net;
	const unsigned iz = net.addType("Izhikevich", 5, 2);
	nemo_network_t cnet = nemo_new_network();
	REQUIRE(cnet);
	unsigned ciz = 0;
	REQUIRE(nemo_add_neuron_type(cnet, "Izhikevich", &ciz) == NEMO_OK);
	for(unsigned n = 0; n < ncount; ++n) {
		const bool exc = n < ncount * 4 / 5;
		const float v = -65.0f;
		float a, b, c, d, sigma;
		if(exc) {
			const float r1 = param(), r2 = param();
			a = 0.02f;
			b = 0.2f;
			c = v + 15.0f * r1 * r1;
			d = 8.0f - 6.0f * r2 * r2;
			sigma = 5.0f;
		} else {
			const float r1 = param();
			a = 0.02f + 0.08f * r1;
			const float r2 = param();
			b = 0.25f - 0.05f * r2;
			c = v;
			d = 2.0f;
			sigma = 2.0f;
		}
		const float u = b * v;
		net.addNeuron(iz, n, { a, b, c, d, sigma }, { u, v });
		float args[7] = { a, b, c, d, sigma, u, v };
		REQUIRE(nemo_add_neuron(cnet, ciz, n, 7, args) == NEMO_OK);
		for(unsigned k = 0; k < scount; ++k) {
			const unsigned t = target();
			const float w = exc ? 0.5f * param() : -param();
			net.addSynapse(n, t, 1, w, false);
			REQUIRE(nemo_add_synapse(cnet, n, t, 1, w, 0, nullptr) == NEMO_OK);
		}
	}
	std::vector<unsigned> fstim;
	if(useFstim) fstim.push_back(100);
	nemo::Simulation::current_stimulus istim;
	std::vector<unsigned> inidx;
	std::vector<float> icur;
	if(useIstim) {
		for(unsigned i : { 20u, 40u, 60u }) {
			istim.push_back(std::make_pair(i, 20.0f));
			inidx.push_back(i);
			icur.push_back(20.0f);
		}
	}
	std::vector<std::pair<unsigned, unsigned>> cpp, c;
	{
		nemo::ConfigurationImpl conf;
		std::unique_ptr<nemo::SimulationBackend> sim(cuda_simulation(&net, &conf));
		for(unsigned ms = 0; ms < steps; ++ms) {
			const std::vector<unsigned>& f = ms == 0 ? sim->step(fstim, istim) : sim->step();
			for(unsigned id : f) cpp.emplace_back(ms, id);
		}
	}
	{
		nemo_configuration_t conf = nemo_new_configuration();
		nemo_simulation_t sim = nemo_new_simulation(cnet, conf);
		REQUIRE(sim);
		for(unsigned ms = 0; ms < steps; ++ms) {
			unsigned* fired = nullptr;
			size_t nfired = 0;
			if(ms == 0) {
				REQUIRE(nemo_step(sim, fstim.empty() ? nullptr : fstim.data(), fstim.size(),
						inidx.empty() ? nullptr : inidx.data(), icur.empty() ? nullptr : icur.data(), inidx.size(),
						&fired, &nfired) == NEMO_OK);
			} else {
				REQUIRE(nemo_step(sim, nullptr, 0, nullptr, nullptr, 0, &fired, &nfired) == NEMO_OK);
			}
			for(size_t i = 0; i < nfired; ++i) c.emplace_back(ms, fired[i]);
			if(ms % 100 == 0) {
				synapse_id* ids = nullptr;
				size_t len = 0;
				REQUIRE(nemo_get_synapses_from_s(sim, 1, &ids, &len) == NEMO_OK && len == scount);
				float w = 0;
				REQUIRE(nemo_get_synapse_weight_s(sim, ids[0], &w) == NEMO_OK && w >= 0.0f && w <= 0.5f);
			}
		}
		nemo_delete_simulation(sim);
		nemo_delete_configuration(conf);
	}
	nemo_delete_network(cnet);
	REQUIRE(!cpp.empty());
	REQUIRE(cpp == c);
}

// without a device: the configuration fails as DeviceMap::setConfiguration
// does, and creating the backend fails with a status, not a crash
void testNoDevice()
{
	REQUIRE(cuda_device_count() == 0);
	nemo::ConfigurationImpl conf;
	bool threw = false;
	try {
		cuda_set_configuration(&conf, -1);
	} catch(nemo::exception& e) {
		threw = e.errorNumber() == NEMO_CUDA_ERROR;
	}
	REQUIRE(threw);
	VectorGenerator net;
	ring(net, 100, 1);
	threw = false;
	try {
		delete cuda_simulation(&net, &conf);
	} catch(nemo::exception& e) {
		threw = e.errorNumber() != NEMO_OK;
	}
	REQUIRE(threw);
	// a fixed-point format other than Q11.20 is refused before anything else
	conf.setFractionalBits(16);
	threw = false;
	try {
		delete cuda_simulation(&net, &conf);
	} catch(nemo::exception& e) {
		threw = e.errorNumber() == NEMO_API_UNSUPPORTED;
	}
	REQUIRE(threw);
}

} // namespace

int main(int argc, char** argv)
{
	const std::string mode = argc > 1 ? argv[1] : "";
	try {
		if(mode == "nodevice") {
			testNoDevice();
		} else if(mode == "gpu") {
			testConfiguration();
			testRing();
			testCurrentStimulus();
			testStdp();
			for(int k = 0; k < 4; ++k) testCompareWithC(k & 1, k & 2);
		} else {
			fprintf(stderr, "usage: driver nodevice|gpu\n");
			return 2;
		}
	} catch(std::exception& e) {
		fprintf(stderr, "unexpected exception: %s\n", e.what());
		return 1;
	}
	printf("ok\n");
	return 0;
}
