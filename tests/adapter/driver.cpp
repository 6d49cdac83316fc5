// driver.cpp -- test driver of the backend adapter (test infrastructure).
//
// Builds networks as a reference network::Generator (a vector-backed
// stand-in), creates the backend through the adapter's cuda_simulation, and
// drives it only through the nemo::SimulationBackend interface, as libnemo
// does: step() (prefire / stimulus / fire / postfire / readFiring),
// applyStdp and the queries.  The checks are the reference's own
// known-answer tests (src/test/test.cpp ring and current stimulus,
// src/test/stdp.cpp testStdp).
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
#include <string>
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
		unsigned id = 0;
		for(const nemo::Synapse& s : m_synapses) if(s.source == src) ++id;
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
