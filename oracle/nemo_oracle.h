/*
 * nemo_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the NeMo 0.7.2 reference CPU backend (src/nemo/cpu/...,
 * src/nemo/cpu/plugins/..., and the shared model code in src/nemo/...) used as
 * the parity checker for the B200 backend.  Nothing in the product links,
 * loads or calls this code; only tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py do.
 *
 * The reference cannot be compiled in this environment (it needs Boost,
 * libltdl and a cmake-generated config.h), so this is a from-the-source
 * restatement.  Parity of the restatement is pinned by the reference's own
 * known-answer tests (ring networks, firing/current stimulus identities,
 * fixed-point saturation, the STDP analytic test, non-contiguous indices),
 * which tests/test_oracle_kat.py replays against this library.
 *
 * The API mirrors the reference C API (src/nemo.h) with a nemo_oracle_
 * prefix, so a test can drive the oracle and the product through identical
 * call sequences.  Status codes are the reference's (src/nemo/types.h:31-61).
 */
#ifndef NEMO_ORACLE_H
#define NEMO_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nemo_oracle_network nemo_oracle_network;
typedef struct nemo_oracle_configuration nemo_oracle_configuration;
typedef struct nemo_oracle_simulation nemo_oracle_simulation;

const char* nemo_oracle_strerror(void);

/* Configuration (src/nemo/ConfigurationImpl.cpp:19-106) */
nemo_oracle_configuration* nemo_oracle_new_configuration(void);
void nemo_oracle_delete_configuration(nemo_oracle_configuration*);
int nemo_oracle_set_stdp_function(nemo_oracle_configuration*,
		const float* prefire, size_t prefire_len,
		const float* postfire, size_t postfire_len,
		float minE, float maxE, float minI, float maxI);
int nemo_oracle_set_write_only_synapses(nemo_oracle_configuration*);

/* Network (src/nemo/NetworkImpl.cpp:25-338) */
nemo_oracle_network* nemo_oracle_new_network(void);
void nemo_oracle_delete_network(nemo_oracle_network*);
int nemo_oracle_add_neuron_type(nemo_oracle_network*, const char* name, unsigned* type);
int nemo_oracle_add_neuron(nemo_oracle_network*, unsigned type, unsigned idx,
		unsigned nargs, const float* args);
/* n neurons; args is row-major n x nargs */
int nemo_oracle_add_neurons(nemo_oracle_network*, unsigned type, size_t n,
		const unsigned* idx, unsigned nargs, const float* args);
int nemo_oracle_add_synapse(nemo_oracle_network*, unsigned source, unsigned target,
		unsigned delay, float weight, unsigned char plastic, uint64_t* id);
int nemo_oracle_add_synapses(nemo_oracle_network*, size_t n,
		const unsigned* source, const unsigned* target, const unsigned* delay,
		const float* weight, const unsigned char* plastic, uint64_t* ids);
int nemo_oracle_neuron_count(nemo_oracle_network*, unsigned* count);

/* Simulation (src/nemo/cpu/Simulation.cpp) */
nemo_oracle_simulation* nemo_oracle_new_simulation(nemo_oracle_network*, nemo_oracle_configuration*);
void nemo_oracle_delete_simulation(nemo_oracle_simulation*);
int nemo_oracle_step(nemo_oracle_simulation*,
		const unsigned* fstim, size_t fstim_count,
		const unsigned* istim_nidx, const float* istim_current, size_t istim_count,
		const unsigned** fired, size_t* fired_count);
/* Run `steps` steps without stimulus, writing the per-step fired counts to
 * counts[steps] and appending fired ids to ids (capacity ids_cap, total
 * written to *ids_len; returns NEMO_BUFFER_OVERFLOW if it does not fit).
 * If stdp_period != 0, applyStdp(reward) is called after every step whose
 * 1-based index is a multiple of stdp_period. */
int nemo_oracle_run(nemo_oracle_simulation*, unsigned steps,
		unsigned stdp_period, float reward,
		unsigned* counts, unsigned* ids, size_t ids_cap, size_t* ids_len);
int nemo_oracle_apply_stdp(nemo_oracle_simulation*, float reward);
int nemo_oracle_get_neuron_state(nemo_oracle_simulation*, unsigned neuron, unsigned var, float* val);
int nemo_oracle_get_neuron_parameter(nemo_oracle_simulation*, unsigned neuron, unsigned param, float* val);
int nemo_oracle_get_membrane_potential(nemo_oracle_simulation*, unsigned neuron, float* val);
int nemo_oracle_set_neuron_state(nemo_oracle_simulation*, unsigned neuron, unsigned var, float val);
int nemo_oracle_set_neuron_parameter(nemo_oracle_simulation*, unsigned neuron, unsigned param, float val);
int nemo_oracle_set_neuron(nemo_oracle_simulation*, unsigned neuron, unsigned nargs, const float* args);
int nemo_oracle_get_synapses_from(nemo_oracle_simulation*, unsigned source,
		const uint64_t** ids, size_t* len);
int nemo_oracle_get_synapse_target(nemo_oracle_simulation*, uint64_t id, unsigned* target);
int nemo_oracle_get_synapse_delay(nemo_oracle_simulation*, uint64_t id, unsigned* delay);
int nemo_oracle_get_synapse_weight(nemo_oracle_simulation*, uint64_t id, float* weight);
int nemo_oracle_get_synapse_plastic(nemo_oracle_simulation*, uint64_t id, unsigned char* plastic);
/* Bulk read-back of every synapse weight, in network iteration order (source
 * neurons ascending, each source's synapses in insertion order) as raw Q11.20. */
int nemo_oracle_get_all_weights_fx(nemo_oracle_simulation*, int32_t* out, size_t cap, size_t* len);
/* Bulk read-back of all neuron state (global order of the network's local
 * index: type order then insertion order). out has nstate*n floats for `type`. */
int nemo_oracle_get_type_state(nemo_oracle_simulation*, unsigned type, float* out, size_t cap, size_t* len);
int nemo_oracle_elapsed_simulation(nemo_oracle_simulation*, unsigned long* elapsed);
int nemo_oracle_reset_timer(nemo_oracle_simulation*);

/* The reference's example network (src/examples/random.cpp:63-88) */
int nemo_oracle_example_random(nemo_oracle_network** out, unsigned ncount, unsigned scount,
		unsigned dmax, int stdp);
int nemo_oracle_example_random_ex(nemo_oracle_network** out, unsigned ncount, unsigned scount,
		unsigned dmax, int stdp, unsigned seed, float sigma_exc, float sigma_inh);
size_t nemo_oracle_network_synapse_count(nemo_oracle_network*);
int nemo_oracle_network_synapses(nemo_oracle_network*, size_t cap,
		unsigned* source, unsigned* target, unsigned* delay, float* weight,
		unsigned char* plastic, size_t* len);

/* The restated RNG (src/nemo/RNG.cpp:9-33), exposed for unit tests */
unsigned nemo_oracle_urand(unsigned state[4]);
float nemo_oracle_nrand(unsigned state[4]);
void nemo_oracle_seed_states(unsigned first, unsigned count, unsigned* out /* count x 4 */);

#ifdef __cplusplus
}
#endif

#endif
