/*
 * b200_backend.cpp -- the B200 library as NeMo's dynamically loaded CUDA
 * backend.
 *
 * libnemo loads its CUDA backend with dlopen("nemo_cuda")
 * (src/nemo/nemo.cpp:31-42) and resolves four symbols from it:
 * cuda_device_count and cuda_device_description, which libnemo_b200.so
 * exports itself, and the two below, which take the reference's C++ classes
 * (src/nemo/cuda/create_simulation.hpp:16-20, src/nemo/cuda/devices.hpp).
 * This file is compiled on the reference side, against its headers (before
 * nemo_b200.h, which then takes the status codes from <nemo/types.h>), into
 * libnemo_cuda.so linked against libnemo_b200.so; dlsym on that handle also
 * finds the two symbols of its dependency.
 *
 * B200Backend implements nemo::SimulationBackend (src/nemo/SimulationBackend
 * .hpp:34-154, with nemo::Simulation and nemo::ReadableNetwork) by
 * forwarding every virtual to the C ABI of include/nemo_b200.h, and turns a
 * status other than NEMO_OK into nemo::exception(status, nemo_strerror()),
 * as the reference backends throw.
 */
#include <nemo/ConfigurationImpl.hpp>
#include <nemo/NeuronType.hpp>
#include <nemo/SimulationBackend.hpp>
#include <nemo/exception.hpp>
#include <nemo/network/Generator.hpp>

#include "nemo_b200.h"

#include <algorithm>
#include <string>
#include <vector>

namespace {

void check(nemo_status_t s)
{
	if(s != NEMO_OK) throw nemo::exception(s, nemo_strerror());
}

// the backend's only fixed-point format: Q11.20 (src/nemo/ConfigurationImpl.cpp:22)
const unsigned B200_FRACTIONAL_BITS = 20;

// synapses are added in batches through the bulk entry point
const size_t SYNAPSE_BATCH = 1 << 20;

class B200Backend : public nemo::SimulationBackend
{
public:
	B200Backend(const nemo::network::Generator& net, const nemo::ConfigurationImpl& conf) :
		m_sim(NULL), m_cycle(0)
	{
		if(conf.fractionalBitsSet() && conf.fractionalBits() != B200_FRACTIONAL_BITS) {
			throw nemo::exception(NEMO_API_UNSUPPORTED,
					"the B200 backend computes in Q11.20 fixed point only (20 fractional bits)");
		}
		nemo_network_t n = nemo_new_network();
		if(!n) throw nemo::exception(nemo_b200_last_status(), nemo_strerror());
		try {
			copyNeurons(net, n);
			copySynapses(net, n);
			nemo_configuration_t c = nemo_new_configuration();
			if(!c) throw nemo::exception(nemo_b200_last_status(), nemo_strerror());
			try {
				copyConfiguration(conf, c);
				m_sim = nemo_new_simulation(n, c);
				if(!m_sim) throw nemo::exception(nemo_b200_last_status(), nemo_strerror());
			} catch(...) {
				nemo_delete_configuration(c);
				throw;
			}
			nemo_delete_configuration(c);
		} catch(...) {
			nemo_delete_network(n);
			throw;
		}
		// the simulation holds its own copy (src/nemo/Simulation.hpp ownership)
		nemo_delete_network(n);
	}

	~B200Backend()
	{
		nemo_delete_simulation(m_sim);
	}

	/* SimulationBackend */

	unsigned getFractionalBits() const { return B200_FRACTIONAL_BITS; }

	void setFiringStimulus(const std::vector<unsigned>& nidx) { m_fstim = nidx; }

	void initCurrentStimulus(size_t count)
	{
		m_inidx.clear();
		m_icur.clear();
		m_inidx.reserve(count);
		m_icur.reserve(count);
	}

	// the last current given for a neuron wins, as in the reference
	// (src/nemo/cpu/Simulation.cpp:160-163); nemo_step resolves duplicates
	void addCurrentStimulus(unsigned neuron, float current)
	{
		m_inidx.push_back(neuron);
		m_icur.push_back(current);
	}

	void finalizeCurrentStimulus(size_t) {}

	// a dense current vector by backend-internal index serves only the MPI
	// worker; the reference CPU backend rejects it the same way
	// (src/nemo/cpu/Simulation.cpp:177-196)
	void setCurrentStimulus(const std::vector<float>& current)
	{
		if(current.empty()) return;
		throw nemo::exception(NEMO_API_UNSUPPORTED, "setting current stimulus vector not supported for the B200 backend");
	}

	void prefire() {}

	void fire()
	{
		unsigned* fired = NULL;
		size_t nfired = 0;
		const nemo_status_t s = nemo_step(m_sim, m_fstim.empty() ? NULL : &m_fstim[0], m_fstim.size(),
				m_inidx.empty() ? NULL : &m_inidx[0], m_icur.empty() ? NULL : &m_icur[0], m_inidx.size(),
				&fired, &nfired);
		m_fstim.clear();
		m_inidx.clear();
		m_icur.clear();
		check(s);
		m_fired.assign(fired, fired + nfired);
	}

	void postfire() {}

	// the neurons fired in the last cycle, valid until the next step
	// (src/nemo/FiringBuffer.hpp:16-23)
	nemo::FiredList readFiring() { return nemo::FiredList(m_cycle++, m_fired); }

	void applyStdp(float reward) { check(nemo_apply_stdp(m_sim, reward)); }

	/* Simulation */

	void setNeuron(unsigned idx, unsigned nargs, const float args[])
	{
		std::vector<float> a(args, args + nargs);
		check(nemo_set_neuron_s(m_sim, idx, nargs, a.empty() ? NULL : &a[0]));
	}

	void setNeuronState(unsigned neuron, unsigned var, float value)
	{
		check(nemo_set_neuron_state_s(m_sim, neuron, var, value));
	}

	void setNeuronParameter(unsigned neuron, unsigned parameter, float value)
	{
		check(nemo_set_neuron_parameter_s(m_sim, neuron, parameter, value));
	}

	float getNeuronState(unsigned neuron, unsigned var) const
	{
		float v;
		check(nemo_get_neuron_state_s(m_sim, neuron, var, &v));
		return v;
	}

	float getNeuronParameter(unsigned neuron, unsigned parameter) const
	{
		float v;
		check(nemo_get_neuron_parameter_s(m_sim, neuron, parameter, &v));
		return v;
	}

	float getMembranePotential(unsigned neuron) const
	{
		float v;
		check(nemo_get_membrane_potential(m_sim, neuron, &v));
		return v;
	}

	const std::vector<synapse_id>& getSynapsesFrom(unsigned neuron)
	{
		synapse_id* ids = NULL;
		size_t len = 0;
		check(nemo_get_synapses_from_s(m_sim, neuron, &ids, &len));
		m_synapses.assign(ids, ids + len);
		return m_synapses;
	}

	unsigned long elapsedWallclock() const
	{
		unsigned long t;
		check(nemo_elapsed_wallclock(m_sim, &t));
		return t;
	}

	unsigned long elapsedSimulation() const
	{
		unsigned long t;
		check(nemo_elapsed_simulation(m_sim, &t));
		return t;
	}

	void resetTimer() { check(nemo_reset_timer(m_sim)); }

	/* ReadableNetwork */

	unsigned getSynapseTarget(const synapse_id& id) const
	{
		unsigned t;
		check(nemo_get_synapse_target_s(m_sim, id, &t));
		return t;
	}

	unsigned getSynapseDelay(const synapse_id& id) const
	{
		unsigned d;
		check(nemo_get_synapse_delay_s(m_sim, id, &d));
		return d;
	}

	float getSynapseWeight(const synapse_id& id) const
	{
		float w;
		check(nemo_get_synapse_weight_s(m_sim, id, &w));
		return w;
	}

	unsigned char getSynapsePlastic(const synapse_id& id) const
	{
		unsigned char p;
		check(nemo_get_synapse_plastic_s(m_sim, id, &p));
		return p;
	}

private:
	nemo_simulation_t m_sim;
	cycle_t m_cycle;
	std::vector<unsigned> m_fstim, m_inidx, m_fired;
	std::vector<float> m_icur;
	std::vector<synapse_id> m_synapses;

	// every neuron type and neuron, in the generator's order (the backend's
	// local order, which orders the fire stream of a cycle)
	static void copyNeurons(const nemo::network::Generator& net, nemo_network_t n)
	{
		std::vector<unsigned> idx;
		std::vector<float> args;
		for(unsigned t = 0; t < net.neuronTypeCount(); ++t) {
			const nemo::NeuronType& type = net.neuronType(t);
			unsigned id;
			check(nemo_add_neuron_type(n, type.name().c_str(), &id));
			const size_t np = type.parameterCount(), ns = type.stateVarCount();
			idx.clear();
			args.clear();
			for(nemo::network::neuron_iterator i = net.neuron_begin(t); i != net.neuron_end(t); ++i) {
				const nemo::network::Generator::neuron& nr = *i;
				idx.push_back(nr.first);
				const float* p = nr.second.getParameters();
				const float* s = nr.second.getState();
				args.insert(args.end(), p, p + np);
				args.insert(args.end(), s, s + ns);
			}
			if(!idx.empty()) {
				check(nemo_b200_add_neurons(n, id, idx.size(), &idx[0], (unsigned) (np + ns),
						args.empty() ? NULL : &args[0]));
			}
		}
	}

	// every synapse, each source's in the order of its synapse ids, so that
	// the backend numbers them as the generator does (source << 32 | index)
	static void copySynapses(const nemo::network::Generator& net, nemo_network_t n)
	{
		std::vector<nemo::Synapse> all;
		for(nemo::network::synapse_iterator i = net.synapse_begin(); i != net.synapse_end(); ++i) all.push_back(*i);
		std::stable_sort(all.begin(), all.end(), [](const nemo::Synapse& a, const nemo::Synapse& b) {
			return a.source != b.source ? a.source < b.source : a.id() < b.id();
		});
		std::vector<unsigned> src, tgt, dly;
		std::vector<float> w;
		std::vector<unsigned char> pl;
		for(size_t b = 0; b < all.size(); b += SYNAPSE_BATCH) {
			const size_t e = std::min(all.size(), b + SYNAPSE_BATCH);
			src.clear(); tgt.clear(); dly.clear(); w.clear(); pl.clear();
			for(size_t k = b; k < e; ++k) {
				src.push_back(all[k].source);
				tgt.push_back(all[k].target());
				dly.push_back(all[k].delay);
				w.push_back(all[k].weight());
				pl.push_back(all[k].plastic());
			}
			check(nemo_b200_add_synapses(n, e - b, &src[0], &tgt[0], &dly[0], &w[0], &pl[0], NULL));
		}
	}

	static void copyConfiguration(const nemo::ConfigurationImpl& conf, nemo_configuration_t c)
	{
		const auto& fn = conf.stdpFunction();
		if(fn) {
			std::vector<float> pre = fn->prefire(), post = fn->postfire();
			check(nemo_set_stdp_function(c, pre.empty() ? NULL : &pre[0], pre.size(),
					post.empty() ? NULL : &post[0], post.size(), fn->minExcitatoryWeight(),
					fn->maxExcitatoryWeight(), fn->minInhibitoryWeight(), fn->maxInhibitoryWeight()));
		}
		if(conf.writeOnlySynapses()) check(nemo_set_write_only_synapses(c));
		check(nemo_set_cuda_backend(c, (int) conf.cudaDevice()));
	}
};

} // namespace

extern "C" {

/* src/nemo/cuda/create_simulation.hpp:16-20 */
nemo::SimulationBackend* cuda_simulation(const nemo::network::Generator* net, const nemo::ConfigurationImpl* conf)
{
	return new B200Backend(*net, *conf);
}

/* DeviceMap::setConfiguration (src/nemo/cuda/devices.cpp:225-246): the
 * default device is device 0; the partition size is the reference CUDA
 * backend's largest, 1024 (the B200 backend chooses its own launch shape) */
void cuda_set_configuration(nemo::ConfigurationImpl* conf, int device)
{
	const unsigned n = cuda_device_count();
	if(n == 0) throw nemo::exception(NEMO_CUDA_ERROR, "No CUDA devices available");
	conf->setBackend(NEMO_BACKEND_CUDA);
	if(device < 0) {
		conf->setCudaDevice(0);
	} else {
		if((unsigned) device >= n) {
			throw nemo::exception(NEMO_CUDA_ERROR, "Invalid device: " + std::to_string(device));
		}
		conf->setCudaDevice((unsigned) device);
	}
	conf->setCudaPartitionSize(1024);
	conf->setBackendDescription(cuda_device_description(conf->cudaDevice()));
}

}
