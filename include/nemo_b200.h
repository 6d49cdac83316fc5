/*
 * nemo_b200.h -- C ABI of the B200 (sm_100a) NeMo simulation backend.
 *
 * Part 1 is a drop-in for the reference C API (src/nemo.h).  Every function
 * keeps the reference's name, signature, argument meaning, status codes
 * (src/nemo/types.h:31-61) and error reporting (status return plus the
 * process-global message of nemo_strerror, src/nemo/nemo_c.cpp:21-65).
 * The comment above each declaration cites the reference declaration it
 * replaces.  Handles are opaque pointers; there are no C++ or torch types.
 *
 * Part 2 replaces the backend plugin ABI that libnemo dlopens for the CUDA
 * backend (src/nemo/cuda/devices.hpp:21-52,
 * src/nemo/cuda/create_simulation.hpp:16-20).  The two functions whose
 * reference signatures carry only C types are exported under their reference
 * names.  The two that take reference C++ objects
 * (cuda_simulation(const network::Generator*, const ConfigurationImpl*) and
 * cuda_set_configuration(ConfigurationImpl*, int)) are provided by the
 * C++ adapter nemosim_b200/adapter/b200_backend.cpp, compiled on the
 * reference side against its headers, which forwards to Part 1.
 *
 * Part 3 is extensions with no counterpart in the reference: bulk
 * construction, device-resident multi-step runs and bulk read-back.
 */
#ifndef NEMO_B200_H
#define NEMO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define NEMO_B200_API __attribute__((visibility("default")))
#else
#define NEMO_B200_API
#endif

/* The status codes, backend ids and basic types of src/nemo/types.h.  A
 * translation unit that includes the reference's <nemo/types.h> before this
 * header (the backend adapter does) takes them from there: the values are
 * the same. */
#ifndef NEMO_TYPES_H
/* src/nemo/types.h:31-61 */
#define NEMO_OK 0
#define NEMO_CUDA_INVOCATION_ERROR 1
#define NEMO_CUDA_ASSERTION_FAILURE 2
#define NEMO_CUDA_MEMORY_ERROR 3
#define NEMO_CUDA_ERROR 4
#define NEMO_API_UNSUPPORTED 5
#define NEMO_INVALID_INPUT 6
#define NEMO_BUFFER_OVERFLOW 7
#define NEMO_BUFFER_UNDERFLOW 8
#define NEMO_LOGIC_ERROR 9
#define NEMO_ALLOCATION_ERROR 10
#define NEMO_MPI_ERROR 11
#define NEMO_DL_ERROR 12
#define NEMO_IO_ERROR 13
#define NEMO_UNKNOWN_ERROR 14

/* src/nemo/types.h:63-66 */
enum { NEMO_BACKEND_CUDA = 0, NEMO_BACKEND_CPU = 1 };
typedef unsigned backend_t;
typedef uint64_t synapse_id;
#endif

/* src/nemo.h:42-52 */
struct nemo_network_class;
struct nemo_simulation_class;
struct nemo_configuration_class;
typedef struct nemo_network_class* nemo_network_t;
typedef struct nemo_simulation_class* nemo_simulation_t;
typedef struct nemo_configuration_class* nemo_configuration_t;
typedef int nemo_status_t;

/* ===================================================================== */
/* Part 1: the reference C API (src/nemo.h)                              */
/* ===================================================================== */

/* src/nemo.h:56-57 */
NEMO_B200_API const char* nemo_version(void);
/* src/nemo.h:72-74.  The four in-scope neuron types are linked in; a
 * directory that exists is accepted and recorded. */
NEMO_B200_API nemo_status_t nemo_add_plugin_path(const char* dir);
/* src/nemo.h:88-90 */
NEMO_B200_API nemo_status_t nemo_cuda_device_count(unsigned* count);
/* src/nemo.h:93-95 */
NEMO_B200_API nemo_status_t nemo_cuda_device_description(unsigned device, const char** descr);

/* --- configuration, src/nemo.h:104-191 --- */
/* src/nemo.h:105-106 */
NEMO_B200_API nemo_configuration_t nemo_new_configuration(void);
/* src/nemo.h:109-110 */
NEMO_B200_API void nemo_delete_configuration(nemo_configuration_t);
/* src/nemo.h:114-115 */
NEMO_B200_API nemo_status_t nemo_log_stdout(nemo_configuration_t);
/* src/nemo.h:148-157 */
NEMO_B200_API nemo_status_t nemo_set_stdp_function(nemo_configuration_t,
		float prefire_fn[], size_t prefire_len,
		float postfire_fn[], size_t postfire_len,
		float min_excitatory_weight, float max_excitatory_weight,
		float min_inhibitory_weight, float max_inhibitory_weight);
/* src/nemo.h:160-162.  Recorded; creating a simulation with it fails with
 * NEMO_API_UNSUPPORTED because this library has no CPU backend. */
NEMO_B200_API nemo_status_t nemo_set_cpu_backend(nemo_configuration_t);
/* src/nemo.h:166-168 */
NEMO_B200_API nemo_status_t nemo_set_cuda_backend(nemo_configuration_t conf, int dev);
/* src/nemo.h:171-173 */
NEMO_B200_API nemo_status_t nemo_cuda_device(nemo_configuration_t conf, int* dev);
/* src/nemo.h:177-179 */
NEMO_B200_API nemo_status_t nemo_backend(nemo_configuration_t conf, backend_t* backend);
/* src/nemo.h:183-185 */
NEMO_B200_API nemo_status_t nemo_backend_description(nemo_configuration_t conf, const char** descr);
/* src/nemo.h:189-191 */
NEMO_B200_API nemo_status_t nemo_set_write_only_synapses(nemo_configuration_t conf);

/* --- construction, src/nemo.h:199-292 --- */
/* src/nemo.h:215-216 */
NEMO_B200_API nemo_network_t nemo_new_network(void);
/* src/nemo.h:220-221 */
NEMO_B200_API void nemo_delete_network(nemo_network_t);
/* src/nemo.h:235-239 */
NEMO_B200_API nemo_status_t nemo_add_neuron_type(nemo_network_t, const char* name, unsigned* neuron_type);
/* src/nemo.h:245-250 */
NEMO_B200_API nemo_status_t nemo_add_neuron_iz(nemo_network_t, unsigned idx,
		float a, float b, float c, float d, float u, float v, float sigma);
/* src/nemo.h:265-268 */
NEMO_B200_API nemo_status_t nemo_add_neuron(nemo_network_t, unsigned type, unsigned idx,
		unsigned nargs, float args[]);
/* src/nemo.h:278-286 */
NEMO_B200_API nemo_status_t nemo_add_synapse(nemo_network_t, unsigned source, unsigned target,
		unsigned delay, float weight, unsigned char is_plastic, synapse_id* id);
/* src/nemo.h:290-292 */
NEMO_B200_API nemo_status_t nemo_neuron_count(nemo_network_t net, unsigned* ncount);

/* --- simulation, src/nemo.h:307-762 --- */
/* src/nemo.h:311-312 */
NEMO_B200_API nemo_simulation_t nemo_new_simulation(nemo_network_t, nemo_configuration_t);
/* src/nemo.h:316-317 */
NEMO_B200_API void nemo_delete_simulation(nemo_simulation_t);
/* src/nemo.h:347-352.  *fired points into a buffer owned by the simulation,
 * valid until the next step (src/nemo/nemo_c.cpp:454-460). */
NEMO_B200_API nemo_status_t nemo_step(nemo_simulation_t,
		unsigned fstim_nidx[], size_t fstim_count,
		unsigned istim_nidx[], float istim_current[], size_t istim_count,
		unsigned* fired[], size_t* fired_count);
/* src/nemo.h:356-358 */
NEMO_B200_API nemo_status_t nemo_apply_stdp(nemo_simulation_t, float reward);
/* src/nemo.h:380-382 */
NEMO_B200_API nemo_status_t nemo_get_membrane_potential(nemo_simulation_t sim, unsigned neuron, float* v);
/* src/nemo.h:399-401 */
NEMO_B200_API nemo_status_t nemo_get_neuron_state_n(nemo_network_t net, unsigned neuron, unsigned var, float* val);
/* src/nemo.h:418-420 */
NEMO_B200_API nemo_status_t nemo_get_neuron_parameter_n(nemo_network_t net, unsigned neuron, unsigned param, float* val);
/* src/nemo.h:437-439 */
NEMO_B200_API nemo_status_t nemo_get_neuron_state_s(nemo_simulation_t sim, unsigned neuron, unsigned var, float* val);
/* src/nemo.h:456-458 */
NEMO_B200_API nemo_status_t nemo_get_neuron_parameter_s(nemo_simulation_t sim, unsigned neuron, unsigned param, float* val);
/* src/nemo.h:467-469 */
NEMO_B200_API nemo_status_t nemo_get_synapse_source_n(nemo_network_t, synapse_id synapse, unsigned* source);
/* src/nemo.h:478-480 */
NEMO_B200_API nemo_status_t nemo_get_synapse_source_s(nemo_simulation_t, synapse_id synapse, unsigned* source);
/* src/nemo.h:489-491 */
NEMO_B200_API nemo_status_t nemo_get_synapse_target_n(nemo_network_t, synapse_id synapse, unsigned* target);
/* src/nemo.h:499-501 */
NEMO_B200_API nemo_status_t nemo_get_synapse_target_s(nemo_simulation_t, synapse_id synapse, unsigned* target);
/* src/nemo.h:509-511 */
NEMO_B200_API nemo_status_t nemo_get_synapse_delay_n(nemo_network_t, synapse_id synapse, unsigned* delay);
/* src/nemo.h:519-521 */
NEMO_B200_API nemo_status_t nemo_get_synapse_delay_s(nemo_simulation_t, synapse_id synapse, unsigned* delay);
/* src/nemo.h:529-531 */
NEMO_B200_API nemo_status_t nemo_get_synapse_weight_n(nemo_network_t, synapse_id synapse, float* weight);
/* src/nemo.h:539-541 */
NEMO_B200_API nemo_status_t nemo_get_synapse_weight_s(nemo_simulation_t, synapse_id synapse, float* weight);
/* src/nemo.h:549-551 */
NEMO_B200_API nemo_status_t nemo_get_synapse_plastic_n(nemo_network_t, synapse_id synapse, unsigned char* plastic);
/* src/nemo.h:559-561 */
NEMO_B200_API nemo_status_t nemo_get_synapse_plastic_s(nemo_simulation_t, synapse_id synapse, unsigned char* plastic);
/* src/nemo.h:565-567.  *synapses points into a buffer owned by the network,
 * valid until the next query. */
NEMO_B200_API nemo_status_t nemo_get_synapses_from_n(nemo_network_t, unsigned source, synapse_id* synapses[], size_t* len);
/* src/nemo.h:579-581 */
NEMO_B200_API nemo_status_t nemo_get_synapses_from_s(nemo_simulation_t, unsigned source, synapse_id* synapses[], size_t* len);
/* src/nemo.h:613-615 */
NEMO_B200_API nemo_status_t nemo_set_neuron_n(nemo_network_t, unsigned idx, unsigned nargs, float args[]);
/* src/nemo.h:627-629 */
NEMO_B200_API nemo_status_t nemo_set_neuron_s(nemo_simulation_t, unsigned idx, unsigned nargs, float args[]);
/* src/nemo.h:639-645 */
NEMO_B200_API nemo_status_t nemo_set_neuron_iz_n(nemo_network_t net, unsigned idx,
		float a, float b, float c, float d, float u, float v, float sigma);
/* src/nemo.h:654-660 */
NEMO_B200_API nemo_status_t nemo_set_neuron_iz_s(nemo_simulation_t sim, unsigned idx,
		float a, float b, float c, float d, float u, float v, float sigma);
/* src/nemo.h:675-677 */
NEMO_B200_API nemo_status_t nemo_set_neuron_state_n(nemo_network_t net, unsigned neuron, unsigned var, float val);
/* src/nemo.h:693-695 */
NEMO_B200_API nemo_status_t nemo_set_neuron_parameter_n(nemo_network_t net, unsigned neuron, unsigned param, float val);
/* src/nemo.h:711-713 */
NEMO_B200_API nemo_status_t nemo_set_neuron_state_s(nemo_simulation_t sim, unsigned neuron, unsigned var, float val);
/* src/nemo.h:729-731 */
NEMO_B200_API nemo_status_t nemo_set_neuron_parameter_s(nemo_simulation_t sim, unsigned neuron, unsigned param, float val);
/* src/nemo.h:753-754 */
NEMO_B200_API nemo_status_t nemo_elapsed_wallclock(nemo_simulation_t, unsigned long*);
/* src/nemo.h:757-758 */
NEMO_B200_API nemo_status_t nemo_elapsed_simulation(nemo_simulation_t, unsigned long*);
/* src/nemo.h:761-762 */
NEMO_B200_API nemo_status_t nemo_reset_timer(nemo_simulation_t);
/* src/nemo.h:786-787 */
NEMO_B200_API const char* nemo_strerror(void);

/* ===================================================================== */
/* Part 2: backend plugin ABI                                             */
/* ===================================================================== */

/* src/nemo/cuda/devices.hpp:21-52 (exported at src/nemo/cuda/devices.cpp:282-300) */
NEMO_B200_API unsigned cuda_device_count(void);
NEMO_B200_API const char* cuda_device_description(unsigned device);

/* ===================================================================== */
/* Part 3: extensions (no counterpart in the reference)                   */
/* ===================================================================== */

/* Bulk form of nemo_add_neuron: n neurons of one type, args row-major
 * (n x nargs). */
NEMO_B200_API nemo_status_t nemo_b200_add_neurons(nemo_network_t, unsigned type, size_t n,
		const unsigned idx[], unsigned nargs, const float args[]);
/* Bulk form of nemo_add_synapse.  ids may be NULL. */
NEMO_B200_API nemo_status_t nemo_b200_add_synapses(nemo_network_t, size_t n,
		const unsigned source[], const unsigned target[], const unsigned delay[],
		const float weight[], const unsigned char plastic[], synapse_id ids[]);
/* The reference's example network random::construct
 * (src/examples/random.cpp:63-88), generated in native code. */
NEMO_B200_API nemo_status_t nemo_b200_example_random(nemo_network_t* net,
		unsigned ncount, unsigned scount, unsigned dmax, int stdp);
/* The same generator with its mt19937 seeded by `seed` (the reference uses
 * the default seed 5489) and the input-noise sigma of the excitatory and
 * inhibitory neurons as parameters (the reference uses 5 and 2): one member
 * of a parameter sweep. */
NEMO_B200_API nemo_status_t nemo_b200_example_random_ex(nemo_network_t* net,
		unsigned ncount, unsigned scount, unsigned dmax, int stdp,
		unsigned seed, float sigma_exc, float sigma_inh);

/* Run `steps` unstimulated steps on the device without returning to the
 * host in between.  If stdp_period != 0, applyStdp(reward) is applied after
 * every step whose 1-based index is a multiple of stdp_period.  Per-step
 * fired counts and synaptic events (sum of the out-degrees of the neurons
 * that fired) are written to fired_counts/events when non-NULL; fired ids of
 * each step, in the order nemo_step returns them, are appended to fired_ids
 * (capacity fired_cap, total in *fired_len) when fired_ids is non-NULL. */
NEMO_B200_API nemo_status_t nemo_b200_run(nemo_simulation_t, unsigned steps,
		unsigned stdp_period, float reward,
		unsigned fired_counts[], uint64_t events[],
		unsigned fired_ids[], size_t fired_cap, size_t* fired_len);

/* A batch: `count` independent networks advanced together, one launch per
 * step for all of them, under one configuration.  Each network's fire
 * stream and state are exactly those of its own nemo_new_simulation run.
 * The batch handle accepts nemo_b200_run (fired_counts then holds steps x
 * count entries, [step][network], and fired_ids each step's ids network
 * by network), nemo_apply_stdp, the launch-shape calls and
 * nemo_b200_batch_get_type_state; per-neuron and per-synapse queries are not
 * available on it (synapses are write-only).  Networks whose maximum delay
 * is exactly 64 ms are rejected (NEMO_API_UNSUPPORTED). */
NEMO_B200_API nemo_simulation_t nemo_b200_new_batch(nemo_network_t nets[], unsigned count, nemo_configuration_t conf);
NEMO_B200_API nemo_status_t nemo_b200_network_count(nemo_simulation_t, unsigned* count);
NEMO_B200_API nemo_status_t nemo_b200_batch_get_type_state(nemo_simulation_t, unsigned net, unsigned type,
		float out[], size_t cap, size_t* len);
/* Read every synapse weight (raw Q11.20) in network iteration order: source
 * neurons ascending, each source's synapses in insertion order. */
NEMO_B200_API nemo_status_t nemo_b200_get_weights_fx(nemo_simulation_t, int32_t out[], size_t cap, size_t* len);
/* Read all state variables of the neurons of network type `type`, as
 * [var][neuron] in insertion order. */
NEMO_B200_API nemo_status_t nemo_b200_get_type_state(nemo_simulation_t, unsigned type,
		float out[], size_t cap, size_t* len);
/* Number of synapses in the simulation and the out-degree of each neuron in
 * the order of nemo_b200_get_type_state's neurons (type order, then
 * insertion order). */
NEMO_B200_API nemo_status_t nemo_b200_synapse_count(nemo_simulation_t, uint64_t* count);
/* Turn per-launch CUDA-event timing of nemo_b200_run's kernels on or off. */
NEMO_B200_API nemo_status_t nemo_b200_set_profiling(nemo_simulation_t, int on);
/* Turn the CUDA-graph replay of nemo_b200_run's two-launch step loop
 * (blocks of 100 steps, captured once per launch shape) on (the default) or
 * off. */
NEMO_B200_API nemo_status_t nemo_b200_set_graphs(nemo_simulation_t, int on);
/* Choose how nemo_b200_run advances the steps between applyStdp calls: one
 * persistent cooperative launch per segment, its update and delivery phases
 * separated by grid barriers (on), or two launches per step (off).  The
 * default is on, except for networks with more than two neurons per thread
 * of the persistent loop's co-resident CTAs (large batches), where one
 * launch per phase over the whole network is faster.  With it off, nemo_step
 * uses two launches per call.  Results are identical. */
NEMO_B200_API nemo_status_t nemo_b200_set_persistent(nemo_simulation_t, int on);
/* nemo_step's resident step loop (no counterpart in the reference, whose
 * step runs on the host, src/nemo/cpu/Simulation.cpp:94-111): when the
 * persistent loop is in use (nemo_b200_set_persistent), nemo_step hands
 * each step to a cooperative launch that stays on the GPU between calls,
 * polling a flag in mapped host memory, instead of launching kernels and
 * synchronising a stream per call.  The loop ends after idle_us
 * microseconds without a nemo_step call (at most 100000; the next call
 * launches it again), and before any other call on the simulation does
 * GPU work.  While it is resident it occupies every SM, so other work on
 * the GPU waits up to idle_us for it.  0 turns it off (two launches per
 * nemo_step).  Default 200.  Results are identical either way. */
NEMO_B200_API nemo_status_t nemo_b200_set_resident_step(nemo_simulation_t, unsigned idle_us);
/* Phase trace: runs `steps` steps (then their STDP accumulation, as
 * nemo_b200_run does before an applyStdp) in one launch of the persistent
 * step loop with %globaltimer read by every CTA at 5 points of each step:
 * its start, its arrival at the barrier after the pre-phase (the
 * deliveries arriving at that step and the last step's STDP accumulation),
 * that barrier's release, the end of its neuron update, and the release of
 * the step's final barrier.  out[(step x ctas + cta) x 5 + point] in ns;
 * *ctas receives the launch's CTAs.  The simulation advances by `steps`
 * steps, as nemo_b200_run would.  Needs the persistent loop
 * (NEMO_API_UNSUPPORTED otherwise) and allocates the device buffer for the
 * call. */
NEMO_B200_API nemo_status_t nemo_b200_trace_phases(nemo_simulation_t, unsigned steps, uint64_t* out, size_t cap,
		unsigned* ctas);
/* Bounded waits of the persistent and resident step loops: every wait of a
 * CTA on the others (a grid barrier, the resident loop's request broadcast)
 * gives up after `polls` unsuccessful polls, sets the loop's error word and
 * ends the launch; the call that ran it returns NEMO_CUDA_ERROR and the
 * simulation's state is undefined from then on (delete it).  Default
 * 16,777,216 polls (seconds); 0 gives up at the first unsuccessful poll,
 * which lets a test exercise the error path without waiting.  A resident
 * loop that is running keeps the limit it was launched with; this call
 * ends it first. */
NEMO_B200_API nemo_status_t nemo_b200_set_wait_limit(nemo_simulation_t, unsigned polls);
/* Where a simulation created with this configuration builds its
 * connectivity (the forward matrix sorted by source and delay, its delay
 * groups, the reverse matrix of plastic synapses): on = 1 (the default)
 * builds it on the device when the networks allow it -- one network, or a
 * batch whose networks have one neuron type each; per network global
 * neuron ids below 4 per neuron plus 2^20, fewer than 2^31 - 1 synapses
 * and neurons x maximum delay; no neuron type that reads the reverse
 * matrix of all synapses -- and on the host otherwise; on = 0 always builds
 * it on the host.  Both builds give the same bytes, the same errors and the
 * same results. */
NEMO_B200_API nemo_status_t nemo_b200_set_device_construction(nemo_configuration_t, int on);
/* Digests of the simulation's connectivity as it sits in device memory:
 * out[0..7] hash the forward matrix (targets and weights), its row starts,
 * the delay-group ends, the per-source delay masks, the reverse matrix of
 * plastic synapses (row starts, sources, forward indices) and applyStdp's
 * table of each target's runs per slice; out[8] is the number of
 * delay groups and out[9] is 1 when the device built it.  Two simulations
 * with equal out[0..8] hold the same bytes. */
NEMO_B200_API nemo_status_t nemo_b200_connectivity_digest(nemo_simulation_t, uint64_t out[10]);
/* Statistics of the last nemo_b200_run: its device time in ms (CUDA events
 * on the simulation's stream), and per kernel kind (0 = update kernel and
 * 1 = deliver kernel of the two-launch step, 2 = applyStdp, 3 = persistent
 * step loop) the summed device time and launch count when profiling is on;
 * the spikes, synaptic events and STDP reverse-matrix entries walked in the
 * run; and the number of plastic synapses.  Any output pointer may be NULL. */
NEMO_B200_API nemo_status_t nemo_b200_run_stats(nemo_simulation_t, float* run_ms,
		float kernel_ms[4], unsigned kernel_launches[4],
		uint64_t* fired, uint64_t* events, uint64_t* stdp_entries, uint64_t* plastic_synapses);
/* Launch shape of the active step loop: neurons per partition (rounded up
 * to a multiple of 32; at most 2048 for the two-launch step, where a CTA
 * owns one partition; a CTA of the persistent loop owns one or more) and
 * threads per CTA (a multiple of 32, at most 1024; 64 to 768 for the
 * persistent loop).  Results are identical for every shape. */
NEMO_B200_API nemo_status_t nemo_b200_set_launch(nemo_simulation_t, unsigned partition, unsigned threads);
NEMO_B200_API nemo_status_t nemo_b200_get_launch(nemo_simulation_t, unsigned* partition, unsigned* threads);
/* Autotuner: times candidate launch shapes on `trial_steps` steps each,
 * starting every trial from a device-side snapshot of the simulation state
 * and restoring it afterwards (the simulation is left exactly as it was),
 * then keeps the fastest shape.  *us_per_step receives its time. */
NEMO_B200_API nemo_status_t nemo_b200_autotune(nemo_simulation_t, unsigned trial_steps, float* us_per_step);
/* Synaptic events (sum of the out-degrees of the fired neurons) of all
 * nemo_step calls on this simulation so far. */
NEMO_B200_API nemo_status_t nemo_b200_step_events(nemo_simulation_t, uint64_t* events);
/* Names of the compiled-in neuron types, one per call (index < count). */
NEMO_B200_API unsigned nemo_b200_neuron_type_count(void);
NEMO_B200_API const char* nemo_b200_neuron_type_name(unsigned i);
/* The host-libm calibration used to reproduce glibc logf/sinf bit for bit on
 * the device: the number of inputs at which the device's own double-precision
 * evaluation rounds differently from the host libm, for logf and sinf. */
NEMO_B200_API nemo_status_t nemo_b200_libm_calibration(uint64_t* log_flips, uint64_t* sin_flips,
		uint64_t* exceptions);
/* Test helper: evaluates the host build of the device's logf/sinf (flip
 * table, exception list and the midpoint-distance skip included; the flip
 * word read on demand and fetched up front), and reads the result tables
 * the two-launch update uses, at every reachable argument, 100,663,298 of
 * them, against the host libm on all host threads;
 * *mismatches receives how many differ (0 when the emulation is exact).  A
 * few seconds. */
NEMO_B200_API nemo_status_t nemo_b200_libm_verify(uint64_t* mismatches);
/* Status of the most recent call, including the constructors
 * (nemo_new_simulation and the like) that report failure only by returning
 * NULL. */
NEMO_B200_API nemo_status_t nemo_b200_last_status(void);
/* Measures the scattered-update floor of the step's pre-phase: `ops`
 * operations at pseudo-random indices into `elements` 16-byte slots --
 * kind 0: 64-bit reductions (as delivery issues them), 1: 32-bit
 * reductions, 2: 8-byte loads -- from `ctas` CTAs of 256 threads (0: 8
 * per SM) on `device`.  *us receives the mean CUDA-event time of `reps`
 * launches (1..1000) after one warm-up launch, in microseconds.  ops is at
 * most 2^30.  Allocates and frees its own device memory. */
/* The end-to-end benchmark loop of a C program (the role of the
 * reference's benchmark(), src/examples/common.cpp:13-122): `steps` calls
 * of nemo_step, each with fstim_per_step firing-stimulus indices from
 * fstim (host memory, consecutive per step) and the fired ids returned in
 * host memory, and nemo_apply_stdp(reward) after every `period` steps (0:
 * never).  It uses the public calls above only.  *fired_total receives the
 * number of fired ids returned, *seconds the loop's host wall time. */
NEMO_B200_API nemo_status_t nemo_b200_bench_step_loop(nemo_simulation_t, const unsigned* fstim,
		size_t fstim_per_step, unsigned steps, unsigned period, float reward, uint64_t* fired_total,
		double* seconds);
NEMO_B200_API nemo_status_t nemo_b200_scatter_probe(unsigned ops, unsigned elements, int kind, unsigned ctas,
		int device, unsigned reps, float* us);
/* Differentiable float32 mode.  A network of `neurons` Izhikevich neurons
 * with `synapses` delayed synapses (source[], target[], delay[] in 1..;
 * ordered by source; synapse e has weight w[e]) run for `ms` milliseconds of
 * 4 Euler sub-steps on `trials` independent noise inputs.  The loss is the
 * mean squared error between the exp(-t/20 ms)-filtered spike trains of
 * neurons 0..readout-1 and target rates; the backward pass is a hand-written
 * BPTT adjoint with a fast-sigmoid surrogate (slope 10) for the threshold,
 * replaying `checkpoint_ms`-long segments from state checkpoints.
 * `options` is a bit set: NEMO_B200_BPTT_SMOOTH replaces the threshold by the
 * fast sigmoid itself in the forward pass; NEMO_B200_BPTT_FP64_STATE keeps
 * the neuron state, the stored trajectories and the adjoints in float64
 * (inputs and gradients stay float32), which reproduces a float64
 * evaluation of the gradient; without it they are float32, and the
 * gradient's rounding error is that of a float32 evaluation (about 1e-2
 * relative on chaotic spiking networks).
 * The float arrays of forward/backward are DEVICE pointers: w[synapses],
 * a, b, c, d [neurons], noise [ms][trials][neurons] (the input current noise
 * itself), target [ms][trials][readout], loss a device scalar, gradients
 * dw[synapses], da, db [neurons]; `stream` is a cudaStream_t (NULL = default).
 * backward differentiates the most recent forward call. */
struct nemo_b200_bptt_class;
typedef struct nemo_b200_bptt_class* nemo_b200_bptt_t;
#define NEMO_B200_BPTT_SMOOTH 1
#define NEMO_B200_BPTT_FP64_STATE 2
NEMO_B200_API nemo_b200_bptt_t nemo_b200_bptt_new(unsigned neurons, unsigned trials, unsigned ms, unsigned readout,
		unsigned checkpoint_ms, size_t synapses, const unsigned source[], const unsigned target[],
		const unsigned delay[], int options, int device);
NEMO_B200_API void nemo_b200_bptt_delete(nemo_b200_bptt_t);
NEMO_B200_API nemo_status_t nemo_b200_bptt_forward(nemo_b200_bptt_t, const float* w, const float* a, const float* b,
		const float* c, const float* d, const float* noise, const float* target, float* loss, void* stream);
/* The filtered readout spike trains of the most recent forward call, as a
 * device array [ms][trials][readout] (e.g. the targets made by a teacher). */
NEMO_B200_API nemo_status_t nemo_b200_bptt_readout(nemo_b200_bptt_t, float* out, void* stream);
NEMO_B200_API nemo_status_t nemo_b200_bptt_backward(nemo_b200_bptt_t, const float* w, const float* a, const float* b,
		const float* c, const float* d, const float* noise, const float* target, float* dw, float* da, float* db,
		void* stream);
/* Extension with no counterpart in the reference: nemo_step (same stimulus
 * arguments and results) that allocates no memory of any kind -- no device
 * or pinned allocation, no host heap, no allocating library call -- for
 * callers that must not allocate: a closed-loop controller stepping the
 * simulation every millisecond from a real-time thread, where a device
 * allocation or free would synchronise the device and stall the loop, or a
 * host application whose memory is budgeted up front.  The stimulus is
 * staged in a fixed static buffer of NEMO_B200_NO_ALLOC_STIMULUS_MAX 32-bit
 * words on each device; fstim_count + 2 x istim_count above that returns
 * NEMO_BUFFER_OVERFLOW without stepping.  The fired neurons' ids (in
 * nemo_step's order) are written to fired[0 .. fired_capacity); *fired_count
 * receives their number, and NEMO_BUFFER_OVERFLOW is returned (after the
 * step) when it exceeds fired_capacity.  An invalid neuron index returns
 * NEMO_INVALID_INPUT without stepping; a batch of networks returns
 * NEMO_API_UNSUPPORTED.  Errors are reported by the status code only
 * (formatting a message would allocate): nemo_strerror is not updated.  The
 * first call on a device looks up the static buffer's device address and
 * should come before any stream capture.  Every call takes the two-launch
 * step and first ends the resident step loop of nemo_step if it runs, so a
 * call costs about one two-launch step, more than a resident nemo_step.
 * The static buffers are shared:
 * calls that overlap in time, from several threads or on several
 * simulations, race and must be serialised by the caller. */
#define NEMO_B200_NO_ALLOC_STIMULUS_MAX 65536
NEMO_B200_API nemo_status_t nemo_b200_step_no_alloc(nemo_simulation_t,
		const unsigned fstim_nidx[], size_t fstim_count,
		const unsigned istim_nidx[], const float istim_current[], size_t istim_count,
		unsigned fired[], size_t fired_capacity, size_t* fired_count);
/* Host build of the device's glibc-exact nrand (for tests): advances the
 * xorshift state in place and returns the normal deviate. */
NEMO_B200_API float nemo_b200_host_nrand(unsigned state[4]);

#ifdef __cplusplus
}
#endif

#endif
