// nemo_c.cpp -- the C ABI (include/nemo_b200.h).
//
// Exceptions never cross the ABI: every call catches them and converts them
// to a status code plus a process-global message, as the reference C API
// does (src/nemo/nemo_c.cpp:21-65).  Like the reference, the message is not
// thread-safe.
#include <cuda_runtime.h>
#include <string.h>
#include <sys/stat.h>

#include <memory>
#include <string>
#include <vector>

#include "../../include/nemo_b200.h"
#include "libm_calib.hpp"
#include "bptt.hpp"
#include "handles.hpp"
#include "network.hpp"
#include "plugins.hpp"
#include "probe.hpp"
#include "simulation.hpp"

using namespace nemo_b200;


static std::string g_lastError;
static nemo_status_t g_lastStatus = NEMO_OK;

static void setResult(const char* msg, nemo_status_t status)
{
	g_lastError = msg;
	g_lastStatus = status;
}

#define CALL(...)                                                               \
	do {                                                                        \
		g_lastStatus = NEMO_OK;                                                 \
		try {                                                                   \
			__VA_ARGS__;                                                             \
		} catch(const Error& e) {                                               \
			setResult(e.what(), e.code());                                      \
		} catch(const std::bad_alloc&) {                                        \
			setResult("host memory allocation failed", NEMO_ALLOCATION_ERROR);  \
		} catch(const std::exception& e) {                                      \
			setResult(e.what(), NEMO_UNKNOWN_ERROR);                            \
		} catch(...) {                                                          \
			setResult("unknown exception", NEMO_UNKNOWN_ERROR);                 \
		}                                                                       \
		return g_lastStatus;                                                    \
	} while(0)

#define NULLCHECK(p)                                                            \
	do {                                                                        \
		if(!(p)) {                                                              \
			setResult("NULL handle or output pointer", NEMO_INVALID_INPUT);     \
			return NEMO_INVALID_INPUT;                                          \
		}                                                                       \
	} while(0)

static Simulation& S(nemo_simulation_t s) { return *s->sim; }

extern "C" {

const char* nemo_version(void) { return "0.7.2-b200"; }

const char* nemo_strerror(void) { return g_lastError.c_str(); }

/* src/nemo/nemo_c.cpp:77-80, Plugin::addPath */
nemo_status_t nemo_add_plugin_path(const char* dir)
{
	NULLCHECK(dir);
	CALL(addPluginPath(dir));
}

nemo_status_t nemo_cuda_device_count(unsigned* count)
{
	NULLCHECK(count);
	*count = 0;
	CALL({
		int n = 0;
		cudaError_t e = cudaGetDeviceCount(&n);
		if(e != cudaSuccess) NB_THROW(NEMO_CUDA_ERROR, "%s", cudaGetErrorString(e));
		*count = (unsigned) n;
	});
}

static std::vector<std::string> g_descr;

nemo_status_t nemo_cuda_device_description(unsigned device, const char** descr)
{
	NULLCHECK(descr);
	CALL({
		cudaDeviceProp p;
		cudaError_t e = cudaGetDeviceProperties(&p, (int) device);
		if(e != cudaSuccess) NB_THROW(NEMO_CUDA_ERROR, "%s", cudaGetErrorString(e));
		if(g_descr.size() <= device) g_descr.resize(device + 1);
		g_descr[device] = format("%s (sm_%d%d, %d SMs, %.0f GB)", p.name, p.major, p.minor,
				p.multiProcessorCount, p.totalGlobalMem / 1e9);
		*descr = g_descr[device].c_str();
	});
}

unsigned cuda_device_count(void)
{
	unsigned n = 0;
	return nemo_cuda_device_count(&n) == NEMO_OK ? n : 0;
}

const char* cuda_device_description(unsigned device)
{
	const char* d = nullptr;
	return nemo_cuda_device_description(device, &d) == NEMO_OK ? d : "";
}

/* --- configuration --- */

nemo_configuration_t nemo_new_configuration(void)
{
	try {
		auto* c = new nemo_configuration_class();
		c->conf.description = "B200 (sm_100a) backend";
		return c;
	} catch(...) {
		setResult("failed to allocate configuration", NEMO_ALLOCATION_ERROR);
		return nullptr;
	}
}

void nemo_delete_configuration(nemo_configuration_t c) { delete c; }

nemo_status_t nemo_log_stdout(nemo_configuration_t c)
{
	NULLCHECK(c);
	CALL(c->conf.logging = true);
}

nemo_status_t nemo_set_stdp_function(nemo_configuration_t c, float pre[], size_t npre,
		float post[], size_t npost, float minE, float maxE, float minI, float maxI)
{
	NULLCHECK(c);
	CALL(c->conf.setStdpFunction(pre, npre, post, npost, minE, maxE, minI, maxI));
}

nemo_status_t nemo_set_cpu_backend(nemo_configuration_t c)
{
	NULLCHECK(c);
	CALL({
		c->conf.backend = NEMO_BACKEND_CPU;
		c->conf.description = "CPU backend (not provided by this library)";
	});
}

nemo_status_t nemo_set_cuda_backend(nemo_configuration_t c, int dev)
{
	NULLCHECK(c);
	CALL({
		int n = 0;
		cudaError_t e = cudaGetDeviceCount(&n);
		if(e != cudaSuccess || n == 0) NB_THROW(NEMO_CUDA_ERROR, "No CUDA device available");
		if(dev >= n) NB_THROW(NEMO_INVALID_INPUT, "Invalid CUDA device %d", dev);
		c->conf.backend = NEMO_BACKEND_CUDA;
		c->conf.device = dev;
		c->conf.description = "B200 (sm_100a) backend";
	});
}

nemo_status_t nemo_cuda_device(nemo_configuration_t c, int* dev)
{
	NULLCHECK(c);
	NULLCHECK(dev);
	CALL(*dev = c->conf.device);
}

nemo_status_t nemo_backend(nemo_configuration_t c, backend_t* b)
{
	NULLCHECK(c);
	NULLCHECK(b);
	CALL(*b = c->conf.backend);
}

nemo_status_t nemo_backend_description(nemo_configuration_t c, const char** d)
{
	NULLCHECK(c);
	NULLCHECK(d);
	CALL(*d = c->conf.description.c_str());
}

nemo_status_t nemo_set_write_only_synapses(nemo_configuration_t c)
{
	NULLCHECK(c);
	CALL(c->conf.writeOnlySynapses = true);
}

/* --- network --- */

nemo_network_t nemo_new_network(void)
{
	try {
		return new nemo_network_class();
	} catch(...) {
		setResult("failed to allocate network", NEMO_ALLOCATION_ERROR);
		return nullptr;
	}
}

void nemo_delete_network(nemo_network_t n) { delete n; }

nemo_status_t nemo_add_neuron_type(nemo_network_t n, const char* name, unsigned* type)
{
	NULLCHECK(n);
	NULLCHECK(name);
	NULLCHECK(type);
	CALL(*type = n->net.addNeuronType(name));
}

/* Network::addNeuron(idx, a, b, c, d, u, v, sigma) (src/nemo/Network.cpp:45-55) */
nemo_status_t nemo_add_neuron_iz(nemo_network_t n, unsigned idx, float a, float b, float c,
		float d, float u, float v, float sigma)
{
	NULLCHECK(n);
	CALL({
		unsigned t = n->net.addNeuronType("Izhikevich");
		float args[7] = { a, b, c, d, sigma, u, v };
		n->net.addNeurons(t, 1, &idx, 7, args);
	});
}

nemo_status_t nemo_add_neuron(nemo_network_t n, unsigned type, unsigned idx, unsigned nargs, float args[])
{
	NULLCHECK(n);
	CALL(n->net.addNeurons(type, 1, &idx, nargs, args));
}

nemo_status_t nemo_b200_add_neurons(nemo_network_t n, unsigned type, size_t count,
		const unsigned idx[], unsigned nargs, const float args[])
{
	NULLCHECK(n);
	CALL(n->net.addNeurons(type, count, idx, nargs, args));
}

nemo_status_t nemo_add_synapse(nemo_network_t n, unsigned source, unsigned target, unsigned delay,
		float weight, unsigned char plastic, synapse_id* id)
{
	NULLCHECK(n);
	CALL(n->net.addSynapses(1, &source, &target, &delay, &weight, &plastic, id));
}

nemo_status_t nemo_b200_add_synapses(nemo_network_t n, size_t count, const unsigned source[],
		const unsigned target[], const unsigned delay[], const float weight[],
		const unsigned char plastic[], synapse_id ids[])
{
	NULLCHECK(n);
	CALL(n->net.addSynapses(count, source, target, delay, weight, plastic, ids));
}

nemo_status_t nemo_neuron_count(nemo_network_t n, unsigned* count)
{
	NULLCHECK(n);
	NULLCHECK(count);
	CALL(*count = n->net.neuronCount());
}

nemo_status_t nemo_get_neuron_state_n(nemo_network_t n, unsigned neuron, unsigned var, float* val)
{
	NULLCHECK(n);
	NULLCHECK(val);
	CALL(*val = n->net.getNeuronState(neuron, var));
}

nemo_status_t nemo_get_neuron_parameter_n(nemo_network_t n, unsigned neuron, unsigned param, float* val)
{
	NULLCHECK(n);
	NULLCHECK(val);
	CALL(*val = n->net.getNeuronParameter(neuron, param));
}

nemo_status_t nemo_set_neuron_n(nemo_network_t n, unsigned idx, unsigned nargs, float args[])
{
	NULLCHECK(n);
	CALL(n->net.setNeuron(idx, nargs, args));
}

nemo_status_t nemo_set_neuron_iz_n(nemo_network_t n, unsigned idx, float a, float b, float c,
		float d, float u, float v, float sigma)
{
	NULLCHECK(n);
	float args[7] = { a, b, c, d, sigma, u, v };
	CALL(n->net.setNeuron(idx, 7, args));
}

nemo_status_t nemo_set_neuron_state_n(nemo_network_t n, unsigned neuron, unsigned var, float val)
{
	NULLCHECK(n);
	CALL(n->net.setNeuronState(neuron, var, val));
}

nemo_status_t nemo_set_neuron_parameter_n(nemo_network_t n, unsigned neuron, unsigned param, float val)
{
	NULLCHECK(n);
	CALL(n->net.setNeuronParameter(neuron, param, val));
}

nemo_status_t nemo_get_synapse_source_n(nemo_network_t n, synapse_id s, unsigned* source)
{
	NULLCHECK(n);
	NULLCHECK(source);
	CALL({
		(void) n->net.getSynapseTarget(s); // validates the id
		*source = (unsigned) (s >> 32);
	});
}

nemo_status_t nemo_get_synapse_target_n(nemo_network_t n, synapse_id s, unsigned* target)
{
	NULLCHECK(n);
	NULLCHECK(target);
	CALL(*target = n->net.getSynapseTarget(s));
}

nemo_status_t nemo_get_synapse_delay_n(nemo_network_t n, synapse_id s, unsigned* delay)
{
	NULLCHECK(n);
	NULLCHECK(delay);
	CALL(*delay = n->net.getSynapseDelay(s));
}

nemo_status_t nemo_get_synapse_weight_n(nemo_network_t n, synapse_id s, float* weight)
{
	NULLCHECK(n);
	NULLCHECK(weight);
	CALL(*weight = n->net.getSynapseWeight(s));
}

nemo_status_t nemo_get_synapse_plastic_n(nemo_network_t n, synapse_id s, unsigned char* plastic)
{
	NULLCHECK(n);
	NULLCHECK(plastic);
	CALL(*plastic = n->net.getSynapsePlastic(s));
}

nemo_status_t nemo_get_synapses_from_n(nemo_network_t n, unsigned source, synapse_id* synapses[], size_t* len)
{
	NULLCHECK(n);
	NULLCHECK(synapses);
	NULLCHECK(len);
	CALL({
		const std::vector<uint64_t>& ids = n->net.getSynapsesFrom(source);
		*synapses = ids.empty() ? nullptr : const_cast<synapse_id*>(ids.data());
		*len = ids.size();
	});
}

/* --- simulation --- */

nemo_simulation_t nemo_new_simulation(nemo_network_t n, nemo_configuration_t c)
{
	if(!n || !c) {
		setResult("NULL network or configuration", NEMO_INVALID_INPUT);
		return nullptr;
	}
	g_lastStatus = NEMO_OK;
	try {
		auto* s = new nemo_simulation_class();
		try {
			s->sim.reset(new Simulation(n->net, c->conf));
		} catch(...) {
			delete s;
			throw;
		}
		return s;
	} catch(const Error& e) {
		setResult(e.what(), e.code());
	} catch(const std::bad_alloc&) {
		setResult("host memory allocation failed", NEMO_ALLOCATION_ERROR);
	} catch(const std::exception& e) {
		setResult(e.what(), NEMO_UNKNOWN_ERROR);
	}
	return nullptr;
}

void nemo_delete_simulation(nemo_simulation_t s) { delete s; }

nemo_simulation_t nemo_b200_new_batch(nemo_network_t nets[], unsigned count, nemo_configuration_t c)
{
	if(!nets || !c || count == 0) {
		setResult("NULL networks or configuration", NEMO_INVALID_INPUT);
		return nullptr;
	}
	g_lastStatus = NEMO_OK;
	try {
		std::vector<const Network*> v;
		for(unsigned i = 0; i < count; ++i) {
			if(!nets[i]) NB_THROW(NEMO_INVALID_INPUT, "NULL network %u", i);
			v.push_back(&nets[i]->net);
		}
		auto* s = new nemo_simulation_class();
		try {
			s->sim.reset(new Simulation(v, c->conf));
		} catch(...) {
			delete s;
			throw;
		}
		return s;
	} catch(const Error& e) {
		setResult(e.what(), e.code());
	} catch(const std::bad_alloc&) {
		setResult("host memory allocation failed", NEMO_ALLOCATION_ERROR);
	} catch(const std::exception& e) {
		setResult(e.what(), NEMO_UNKNOWN_ERROR);
	}
	return nullptr;
}

nemo_status_t nemo_b200_network_count(nemo_simulation_t s, unsigned* count)
{
	NULLCHECK(s);
	NULLCHECK(count);
	CALL(*count = S(s).networkCount());
}

nemo_status_t nemo_b200_batch_get_type_state(nemo_simulation_t s, unsigned net, unsigned type, float out[],
		size_t cap, size_t* len)
{
	NULLCHECK(s);
	NULLCHECK(len);
	CALL(S(s).getNetTypeState(net, type, out, cap, len));
}

/* nemo_c.cpp:440-477 */
nemo_status_t nemo_step(nemo_simulation_t s, unsigned fstim[], size_t nf, unsigned inidx[],
		float icur[], size_t ni, unsigned* fired[], size_t* nfired)
{
	NULLCHECK(s);
	CALL({
		const std::vector<unsigned>& f = S(s).step(fstim, nf, inidx, icur, ni);
		if(fired) *fired = f.empty() ? nullptr : const_cast<unsigned*>(f.data());
		if(nfired) *nfired = f.size();
	});
}

// Allocation-free: no CALL wrapper (its error path formats a message) and
// no exception may escape (stepNoAlloc throws nothing).
nemo_status_t nemo_b200_step_no_alloc(nemo_simulation_t s, const unsigned fstim[], size_t nf, const unsigned inidx[],
		const float icur[], size_t ni, unsigned fired[], size_t cap, size_t* nfired)
{
	if(!s || !nfired || (nf && !fstim) || (ni && (!inidx || !icur)) || (cap && !fired)) {
		g_lastStatus = NEMO_INVALID_INPUT;
		return NEMO_INVALID_INPUT;
	}
	g_lastStatus = S(s).stepNoAlloc(fstim, nf, inidx, icur, ni, fired, cap, nfired);
	return g_lastStatus;
}

nemo_status_t nemo_apply_stdp(nemo_simulation_t s, float reward)
{
	NULLCHECK(s);
	CALL(S(s).applyStdp(reward));
}

nemo_status_t nemo_b200_run(nemo_simulation_t s, unsigned steps, unsigned stdpPeriod, float reward,
		unsigned counts[], uint64_t events[], unsigned ids[], size_t cap, size_t* len)
{
	NULLCHECK(s);
	CALL(S(s).run(steps, stdpPeriod, reward, counts, events, ids, cap, len));
}

nemo_status_t nemo_get_membrane_potential(nemo_simulation_t s, unsigned neuron, float* v)
{
	NULLCHECK(s);
	NULLCHECK(v);
	CALL(*v = S(s).getMembranePotential(neuron));
}

nemo_status_t nemo_get_neuron_state_s(nemo_simulation_t s, unsigned neuron, unsigned var, float* val)
{
	NULLCHECK(s);
	NULLCHECK(val);
	CALL(*val = S(s).getNeuronState(neuron, var));
}

nemo_status_t nemo_get_neuron_parameter_s(nemo_simulation_t s, unsigned neuron, unsigned p, float* val)
{
	NULLCHECK(s);
	NULLCHECK(val);
	CALL(*val = S(s).getNeuronParameter(neuron, p));
}

nemo_status_t nemo_set_neuron_s(nemo_simulation_t s, unsigned idx, unsigned nargs, float args[])
{
	NULLCHECK(s);
	CALL(S(s).setNeuron(idx, nargs, args));
}

nemo_status_t nemo_set_neuron_iz_s(nemo_simulation_t s, unsigned idx, float a, float b, float c,
		float d, float u, float v, float sigma)
{
	NULLCHECK(s);
	float args[7] = { a, b, c, d, sigma, u, v };
	CALL(S(s).setNeuron(idx, 7, args));
}

nemo_status_t nemo_set_neuron_state_s(nemo_simulation_t s, unsigned neuron, unsigned var, float val)
{
	NULLCHECK(s);
	CALL(S(s).setNeuronState(neuron, var, val));
}

nemo_status_t nemo_set_neuron_parameter_s(nemo_simulation_t s, unsigned neuron, unsigned p, float val)
{
	NULLCHECK(s);
	CALL(S(s).setNeuronParameter(neuron, p, val));
}

nemo_status_t nemo_get_synapse_source_s(nemo_simulation_t s, synapse_id id, unsigned* source)
{
	NULLCHECK(s);
	NULLCHECK(source);
	CALL({
		(void) S(s).getSynapseTarget(id);
		*source = (unsigned) (id >> 32);
	});
}

nemo_status_t nemo_get_synapse_target_s(nemo_simulation_t s, synapse_id id, unsigned* target)
{
	NULLCHECK(s);
	NULLCHECK(target);
	CALL(*target = S(s).getSynapseTarget(id));
}

nemo_status_t nemo_get_synapse_delay_s(nemo_simulation_t s, synapse_id id, unsigned* delay)
{
	NULLCHECK(s);
	NULLCHECK(delay);
	CALL(*delay = S(s).getSynapseDelay(id));
}

nemo_status_t nemo_get_synapse_weight_s(nemo_simulation_t s, synapse_id id, float* weight)
{
	NULLCHECK(s);
	NULLCHECK(weight);
	CALL(*weight = S(s).getSynapseWeight(id));
}

nemo_status_t nemo_get_synapse_plastic_s(nemo_simulation_t s, synapse_id id, unsigned char* plastic)
{
	NULLCHECK(s);
	NULLCHECK(plastic);
	CALL(*plastic = S(s).getSynapsePlastic(id));
}

nemo_status_t nemo_get_synapses_from_s(nemo_simulation_t s, unsigned source, synapse_id* synapses[], size_t* len)
{
	NULLCHECK(s);
	NULLCHECK(synapses);
	NULLCHECK(len);
	CALL({
		const std::vector<uint64_t>& ids = S(s).getSynapsesFrom(source);
		*synapses = ids.empty() ? nullptr : const_cast<synapse_id*>(ids.data());
		*len = ids.size();
	});
}

nemo_status_t nemo_elapsed_wallclock(nemo_simulation_t s, unsigned long* ms)
{
	NULLCHECK(s);
	NULLCHECK(ms);
	CALL(*ms = S(s).elapsedWallclock());
}

nemo_status_t nemo_elapsed_simulation(nemo_simulation_t s, unsigned long* ms)
{
	NULLCHECK(s);
	NULLCHECK(ms);
	CALL(*ms = S(s).elapsedSimulation());
}

nemo_status_t nemo_reset_timer(nemo_simulation_t s)
{
	NULLCHECK(s);
	CALL(S(s).resetTimer());
}

nemo_status_t nemo_b200_get_weights_fx(nemo_simulation_t s, int32_t out[], size_t cap, size_t* len)
{
	NULLCHECK(s);
	NULLCHECK(len);
	CALL(S(s).getWeightsFx(out, cap, len));
}

nemo_status_t nemo_b200_get_type_state(nemo_simulation_t s, unsigned type, float out[], size_t cap, size_t* len)
{
	NULLCHECK(s);
	NULLCHECK(len);
	CALL(S(s).getTypeState(type, out, cap, len));
}

nemo_status_t nemo_b200_synapse_count(nemo_simulation_t s, uint64_t* count)
{
	NULLCHECK(s);
	NULLCHECK(count);
	CALL(*count = S(s).synapseCount());
}

nemo_status_t nemo_b200_set_profiling(nemo_simulation_t s, int on)
{
	NULLCHECK(s);
	CALL(S(s).profiling = on != 0);
}

nemo_status_t nemo_b200_set_graphs(nemo_simulation_t s, int on)
{
	NULLCHECK(s);
	CALL(S(s).useGraphs = on != 0);
}

nemo_status_t nemo_b200_set_persistent(nemo_simulation_t s, int on)
{
	NULLCHECK(s);
	CALL(S(s).usePersistent = on != 0);
}

nemo_status_t nemo_b200_set_resident_step(nemo_simulation_t s, unsigned idle_us)
{
	NULLCHECK(s);
	CALL(S(s).setResidentIdle(idle_us));
}

nemo_status_t nemo_b200_trace_phases(nemo_simulation_t s, unsigned steps, uint64_t* out, size_t cap,
		unsigned* ctas)
{
	NULLCHECK(s);
	NULLCHECK(out);
	CALL({
		const unsigned g = S(s).tracePhases(steps, out, cap);
		if(ctas) *ctas = g;
	});
}

nemo_status_t nemo_b200_set_wait_limit(nemo_simulation_t s, unsigned polls)
{
	NULLCHECK(s);
	CALL(S(s).setWaitLimit(polls));
}

nemo_status_t nemo_b200_set_device_construction(nemo_configuration_t c, int on)
{
	NULLCHECK(c);
	CALL(c->conf.deviceConstruction = on != 0);
}

nemo_status_t nemo_b200_connectivity_digest(nemo_simulation_t s, uint64_t out[10])
{
	NULLCHECK(s);
	NULLCHECK(out);
	CALL(S(s).connectivityDigest(out));
}

nemo_status_t nemo_b200_run_stats(nemo_simulation_t s, float* runMs, float kernelMs[4], unsigned launches[4],
		uint64_t* fired, uint64_t* events, uint64_t* stdpEntries, uint64_t* plastic)
{
	NULLCHECK(s);
	CALL({
		Simulation& sim = S(s);
		if(runMs) *runMs = sim.lastRunMs;
		for(int k = 0; k < Simulation::K_KINDS; ++k) {
			if(kernelMs) kernelMs[k] = sim.kernelMs[k];
			if(launches) launches[k] = sim.kernelLaunches[k];
		}
		if(fired) *fired = sim.lastFired;
		if(events) *events = sim.lastEvents;
		if(stdpEntries) *stdpEntries = sim.lastStdpEntries;
		if(plastic) *plastic = sim.lastPlastic;
	});
}

nemo_status_t nemo_b200_set_launch(nemo_simulation_t s, unsigned partition, unsigned threads)
{
	NULLCHECK(s);
	CALL(S(s).setLaunch(partition, threads));
}

nemo_status_t nemo_b200_get_launch(nemo_simulation_t s, unsigned* partition, unsigned* threads)
{
	NULLCHECK(s);
	CALL({
		if(partition) *partition = S(s).partition();
		if(threads) *threads = S(s).threads();
	});
}

nemo_status_t nemo_b200_autotune(nemo_simulation_t s, unsigned trial_steps, float* us_per_step)
{
	NULLCHECK(s);
	CALL({
		float us = S(s).autotune(trial_steps);
		if(us_per_step) *us_per_step = us;
	});
}

nemo_status_t nemo_b200_step_events(nemo_simulation_t s, uint64_t* events)
{
	NULLCHECK(s);
	NULLCHECK(events);
	CALL(*events = S(s).stepEvents);
}

unsigned nemo_b200_neuron_type_count(void) { return KIND_COUNT; }

const char* nemo_b200_neuron_type_name(unsigned i) { return i < KIND_COUNT ? KERNELS[i].name : ""; }

nemo_status_t nemo_b200_libm_calibration(uint64_t* logFlips, uint64_t* sinFlips, uint64_t* exceptions)
{
	CALL({
		const CalibTables& t = libm_calibration();
		if(logFlips) *logFlips = t.logFlips;
		if(sinFlips) *sinFlips = t.sinFlips;
		if(exceptions) *exceptions = t.excKey.size();
	});
}

nemo_status_t nemo_b200_libm_verify(uint64_t* mismatches)
{
	NULLCHECK(mismatches);
	CALL(*mismatches = libm_verify());
}

nemo_status_t nemo_b200_last_status(void) { return g_lastStatus; }

nemo_status_t nemo_b200_scatter_probe(unsigned ops, unsigned elements, int kind, unsigned ctas, int device,
		unsigned reps, float* us)
{
	NULLCHECK(us);
	CALL(*us = scatter_probe(ops, elements, kind, ctas, device, reps));
}

nemo_b200_bptt_t nemo_b200_bptt_new(unsigned neurons, unsigned trials, unsigned ms, unsigned readout,
		unsigned checkpoint_ms, size_t synapses, const unsigned source[], const unsigned target[],
		const unsigned delay[], int options, int device)
{
	g_lastStatus = NEMO_OK;
	try {
		auto* h = new nemo_b200_bptt_class();
		try {
			if(options & ~(NEMO_B200_BPTT_SMOOTH | NEMO_B200_BPTT_FP64_STATE)) {
				NB_THROW(NEMO_INVALID_INPUT, "unknown differentiable-mode option bits 0x%x", (unsigned) options);
			}
			h->impl.reset(new Bptt(neurons, trials, ms, readout, checkpoint_ms, synapses, source, target, delay,
					(options & NEMO_B200_BPTT_SMOOTH) != 0, (options & NEMO_B200_BPTT_FP64_STATE) != 0, device));
		} catch(...) {
			delete h;
			throw;
		}
		return h;
	} catch(const Error& e) {
		setResult(e.what(), e.code());
	} catch(const std::exception& e) {
		setResult(e.what(), NEMO_UNKNOWN_ERROR);
	}
	return nullptr;
}

void nemo_b200_bptt_delete(nemo_b200_bptt_t h) { delete h; }

nemo_status_t nemo_b200_bptt_forward(nemo_b200_bptt_t h, const float* w, const float* a, const float* b,
		const float* c, const float* d, const float* noise, const float* target, float* loss, void* stream)
{
	NULLCHECK(h);
	CALL(h->impl->forward(BpttParams{ w, a, b, c, d, noise, target }, loss, stream));
}

nemo_status_t nemo_b200_bptt_readout(nemo_b200_bptt_t h, float* out, void* stream)
{
	NULLCHECK(h);
	NULLCHECK(out);
	CALL(h->impl->readout(out, stream));
}

nemo_status_t nemo_b200_bptt_backward(nemo_b200_bptt_t h, const float* w, const float* a, const float* b,
		const float* c, const float* d, const float* noise, const float* target, float* dw, float* da, float* db,
		void* stream)
{
	NULLCHECK(h);
	CALL(h->impl->backward(BpttParams{ w, a, b, c, d, noise, target }, dw, da, db, stream));
}

float nemo_b200_host_nrand(unsigned state[4])
{
	LibmCalib c = host_calib_view();
	return nb_nrand<true>(c, state[0], state[1], state[2], state[3]);
}

} // extern "C"
