// simulation.hpp -- the B200 simulation backend (replaces the reference's
// cuda::Simulation, src/nemo/cuda/Simulation.cpp, and reproduces the
// results of its CPU backend, src/nemo/cpu/Simulation.cpp, bit for bit).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <chrono>
#include <unordered_map>
#include <vector>

#include "network.hpp"
#include "nemo_libm.cuh"

namespace nemo_b200 {

constexpr unsigned MAX_TYPES = 8;
constexpr unsigned STEP_THREADS = 256;   // block size of the apply/stimulus kernels
constexpr unsigned MAX_PARTITION = 2048; // neurons per CTA of the step kernel
constexpr unsigned RUN_THREADS = 768;    // largest block of the persistent step loop (registers for 768 x 1 or 384 x 2 per SM)

// Grid barrier of the persistent step loop (device memory; the counter is
// zeroed before each launch, the error word when the host has read it).
struct GridBarrier {
	uint32_t count;  // arrivals so far: barrier b of the launch is complete at (b + 1) x CTAs
	uint32_t cmd;    // resident step loop: the request being run (| stop flag: end)
	uint32_t error;  // set when a wait gave up
	uint32_t nf, ni; // resident step loop: the request's stimulus sizes
	uint32_t pad[3];
};
static_assert(offsetof(GridBarrier, cmd) == 4, "one memset restarts count and cmd");

// go | SERVE_STOP asks the resident step loop to end; sequence numbers run
// from 1 to 2^31 - 1 and wrap to 1.
constexpr uint32_t SERVE_STOP = 0x80000000u;
__host__ __device__ inline uint32_t serve_next(uint32_t seq) { return seq == 0x7fffffffu ? 1u : seq + 1u; }
constexpr unsigned RESIDENT_IDLE_MAX_US = 100000;  // the grid barrier's wait limit is far longer
// polls of a grid-barrier or request wait before it gives up (seconds)
constexpr uint32_t BARRIER_SPIN_LIMIT = 1u << 24;
constexpr unsigned RESIDENT_REPLY_LIMIT_S = 20;

// Requests to the resident step loop of nemo_step (mapped host memory):
// the host writes the stimulus sizes and then go; the device writes done.
// A request is two 8-byte words, each written and read whole: the
// sequence number in the high half of both, the stimulus sizes (nf firing
// indices, ni (index, current) pairs) in the low halves; it is complete
// when both carry the same sequence number.  req[0] = (seq | stop flag)
// << 32 ends the loop.  A firing stimulus of at most SERVE_INLINE neurons
// without currents travels in the request's own 64-byte line, so that the
// poll that finds the request also reads it: inl[i] = seq << 32 | local
// index, each word checked by its sequence number as the request words
// are, and req[0]'s low half is then SERVE_INLINE_FLAG | count.
constexpr uint32_t SERVE_INLINE = 6;
constexpr uint32_t SERVE_INLINE_FLAG = 0x80000000u;
struct ServeCtl {
	unsigned long long req[2];
	unsigned long long inl[SERVE_INLINE];
	uint32_t pad0[16];
	uint32_t done;     // sequence number of the last completed step
	uint32_t fired;    // its fired neurons (global ids in the fired-id buffer)
	unsigned long long events;  // its synaptic events
	uint32_t pad1[28];
};
static_assert(offsetof(ServeCtl, inl) + 8 * SERVE_INLINE <= 64, "the request and its inline stimulus share one 64-byte line");
static_assert(offsetof(ServeCtl, done) == 128, "the reply starts a line of its own");

// STDP accumulation first tests a source against a shared-memory copy of the
// "fired in the last 64 steps" bit-vector (W words), when it fits in this
// many bytes; else it reads every source's history.
constexpr unsigned RECENT_FILTER_MAX_BYTES = 48 * 1024;

struct TypeRange {
	int kind;
	uint32_t base, n;
	const float* param;  // [nparam][n]
	float* state;        // [history][nstate][n]; slot cycle % history is the current one
	uint32_t history;
};

// STDP process in fixed point (src/nemo/StdpProcess.cpp:20-46)
struct StdpParams {
	int32_t fnPre[MAX_HISTORY];
	int32_t fnPost[MAX_HISTORY];
	uint64_t potBits, depBits, prePostBits, postPreBits, postFireMask;
	uint32_t npre, npost;
	int32_t minE, maxE, minI, maxI;
};

// A list of ranges ("groups") published by one phase for the next, which
// spreads their entries evenly over all warps of the GPU: group i is
// {start lo, start hi, length, first entry}, its entries numbered
// consecutively after those of groups 0..i-1, and bucket[b] is the group
// that holds entry 32 b.
struct WorkList {
	uint4* group;
	unsigned long long* count;  // [2] by the parity of the publishing step: groups << 32 | entries
	uint32_t* bucket;
};

// Everything a kernel needs, passed by value.  Neuron arrays use the
// backend-local index: type order, then insertion order
// (src/nemo/cpu/Simulation.cpp:58-73).
struct DevSim {
	uint32_t N;       // neurons
	uint32_t W;       // 32-bit words per neuron bit-vector
	uint32_t ntypes;
	uint32_t dStride; // entries per source in the delay-group tables (the maximum delay)
	uint32_t R;       // firing ring length (steps)
	TypeRange types[MAX_TYPES];
	uint32_t* rng;            // [4][N] xorshift words
	float* noise;             // [N] next step's nrand, precomputed inside the persistent loop
	uint64_t* hist;           // [2][N] firing history, double-buffered by step parity
	uint32_t* recent;         // [2][recentWords] bit-vectors: history nonzero (fired in the last 64 steps), by parity
	uint32_t recentWords;     // W rounded up to a multiple of 4
	uint32_t recentBytes;     // bytes of shared memory for the copy of one recent bit-vector (0 = none)
	uint32_t* fstim;          // [W] pending firing stimulus
	float* curExt;            // [N] pending current stimulus
	ulonglong2* slot;         // [N] int64 E and I fixed-point sums (two's complement) of this step's arrivals
	const unsigned long long* outPtr; // [N+1] outgoing synapses per source, sorted by delay
	uint32_t* synTgt;         // [S] target | (delay - 1) << 26
	uint32_t* synW;           // [S] weight (Q11.20), apart from the targets: applyStdp moves 4 bytes a synapse
	// delay groups: bit d - 1 of delayMask[n] is set when source n has
	// synapses of delay d that deliverSpikes delivers; dEnd[n][d - 1] is the
	// end of its delay-d group within its row (uint16 when every row is
	// shorter than 65536, else uint32; the other pointer is null)
	const uint64_t* delayMask;
	const uint16_t* dEnd16;
	const uint32_t* dEnd32;
	uint32_t* firedRing;      // [R][W] fired bit-vector per step
	uint32_t* l2g;            // [N] global id of each neuron
	uint32_t* firedIds;       // [N] staging of a step's fired global ids
	uint32_t l2gIdentity;     // l2g[i] == i for every neuron
	uint32_t* firedCount;     // [R]
	unsigned long long* eventCount; // [R] synaptic events (out-degree of fired neurons)
	unsigned long long* stdpCount;  // [R] incoming plastic synapses walked by STDP
	int stdp;
	// reverse matrix of plastic synapses: per target, sorted by forward index
	const unsigned long long* rcmPtr; // [N+1] incoming plastic synapses per target
	const uint32_t* rcmSrc;   // source | (delay - 1) << 26
	const uint32_t* rcmFwd;   // index into the forward matrix (synTgt, synW)
	int32_t* rcmAcc;          // STDP accumulator per incoming plastic synapse
	// applyStdp's slices of the forward matrix: rcmSlice[k][t] is the offset
	// within target t's entries of the first one whose forward index is at
	// least k x sliceLen ([applySlices + 1][N]; the last row is the in-degree)
	const uint32_t* rcmSlice;
	uint32_t applySlices, sliceLen;
	// reverse matrix of all synapses into the targets of a type that reads
	// its sources (Kuramoto): per target, source | (delay - 1) << 26 and the
	// weight as given
	const unsigned long long* allPtr;
	const uint32_t* allSrc;
	const float* allW;
	// work published by a step's update for the next pre-phase: the delay
	// groups arriving next step (ranges of the forward matrix) and the incoming plastic
	// synapses of its STDP targets (ranges of the reverse matrix)
	WorkList dlvWork, stdpWork;
	uint32_t* touchedBits;    // [W] STDP targets since the last applyStdp
	unsigned long long* cycleDev; // step counter read by kernels replayed from a CUDA graph
	StdpParams sp;
	LibmCalib calib;
	uint32_t waitLimit;       // polls of a grid-barrier or request wait before it gives up
	// phase trace of the persistent loop (null: off): %globaltimer of each
	// CTA at TRACE_MARKS points of each of the first traceSteps steps of a
	// launch, [step][CTA][mark]
	unsigned long long* trace;
	uint32_t traceSteps;
};

// the trace points of a step: its start, the CTA's arrival after the
// pre-phase, the release of the barrier after it, the end of the CTA's
// update, and the release of the step's final barrier
constexpr uint32_t TRACE_MARKS = 5;

class Simulation {
public:
	Simulation(const Network& net, const Configuration& conf);
	// a batch of independent networks advanced together (each network's
	// results are those of its own single-network simulation)
	Simulation(const std::vector<const Network*>& nets, const Configuration& conf);
	~Simulation();
	unsigned networkCount() const { return m_nets; }

	const std::vector<unsigned>& step(const unsigned* fstim, size_t nf,
			const unsigned* inidx, const float* icur, size_t ni);
	void applyStdp(float reward);
	// step() that allocates nothing and throws nothing (nemo_b200_step_no_alloc)
	nemo_status_t stepNoAlloc(const unsigned* fstim, size_t nf, const unsigned* inidx, const float* icur, size_t ni,
			unsigned* fired, size_t cap, size_t* nfired) noexcept;
	void run(unsigned steps, unsigned stdpPeriod, float reward, unsigned* counts,
			uint64_t* events, unsigned* ids, size_t cap, size_t* len);

	float getNeuronState(unsigned g, unsigned var);
	float getNeuronParameter(unsigned g, unsigned p);
	float getMembranePotential(unsigned g);
	void setNeuron(unsigned g, unsigned nargs, const float* args);
	void setNeuronState(unsigned g, unsigned var, float v);
	void setNeuronParameter(unsigned g, unsigned p, float v);

	const std::vector<uint64_t>& getSynapsesFrom(unsigned source);
	unsigned getSynapseTarget(uint64_t id);
	unsigned getSynapseDelay(uint64_t id);
	float getSynapseWeight(uint64_t id);
	unsigned char getSynapsePlastic(uint64_t id);

	void getWeightsFx(int32_t* out, size_t cap, size_t* len);
	void getTypeState(unsigned netType, float* out, size_t cap, size_t* len);
	void getNetTypeState(unsigned net, unsigned netType, float* out, size_t cap, size_t* len);
	uint64_t synapseCount() const { return m_nsyn; }

	unsigned long elapsedWallclock() const;
	unsigned long elapsedSimulation() const { return m_timerSteps; }
	void resetTimer();

	// timing of the last run(): whole run and, when profiling is on, each
	// kernel kind (CUDA events around every launch): update and deliver
	// kernels of the two-launch step, applyStdp, persistent step loop
	enum { K_STEP = 0, K_STDP = 1, K_APPLY = 2, K_RUN = 3, K_KINDS = 4 };
	float lastRunMs = 0;
	float kernelMs[K_KINDS] = {0, 0, 0, 0};
	unsigned kernelLaunches[K_KINDS] = {0, 0, 0, 0};
	uint64_t lastFired = 0, lastEvents = 0, lastStdpEntries = 0, lastPlastic = 0;
	bool profiling = false;
	bool useGraphs = true;  // replay the two-launch step loop from CUDA graphs in run()
	// run() advances its step loop with one persistent cooperative launch per
	// segment between applyStdp calls (else with the two-launch step); on by
	// default unless the network has more than two neurons per thread of the
	// persistent loop's co-resident CTAs
	bool usePersistent = true;

	// launch shape of the active step loop (persistent or two-launch):
	// partition size (neurons per partition; a CTA owns one or more) and
	// threads per CTA; results do not depend on them
	uint32_t partition() const { return persistentActive() ? m_runP : m_P; }
	uint32_t threads() const { return persistentActive() ? m_runT : m_T; }
	void setLaunch(uint32_t P, uint32_t T);
	bool persistentActive() const { return usePersistent && m_runGrid != 0; }
	// step() keeps the persistent loop resident on the GPU between calls
	// (serve_kernel) and ends it after this many microseconds without a
	// call (at most RESIDENT_IDLE_MAX_US); 0: two kernel launches per step
	unsigned residentIdleUs = 200;
	bool residentAvailable() const;
	void setResidentIdle(unsigned us);
	// polls of each grid-barrier or request wait of the persistent and
	// resident loops before it gives up and the call reports
	// NEMO_CUDA_ERROR (BARRIER_SPIN_LIMIT by default; 0: give up at the
	// first unsuccessful poll); lets a test make the waits run out
	void setWaitLimit(uint32_t polls);
	// time candidate launch shapes on trial steps from a saved copy of the
	// simulation state, restore it, and keep the fastest; returns its time
	// per step in microseconds
	float autotune(unsigned trialSteps);
	// one launch of the persistent loop over `steps` steps (then its STDP
	// accumulation, as in run()) with the phase trace on: out receives
	// steps x CTAs x TRACE_MARKS %globaltimer values (ns); returns the CTAs
	unsigned tracePhases(unsigned steps, uint64_t* out, size_t cap);
	// digests of the device connectivity (forward matrix, delay-group ends,
	// delay masks, reverse matrix of plastic synapses), its delay-group
	// count, and whether it was built on the device
	enum { DIGESTS = 10 };
	void connectivityDigest(uint64_t out[DIGESTS]);
	uint64_t stepEvents = 0;  // synaptic events of all step() calls so far

private:
	struct HostType {
		NeuronTypeDesc desc;  // copied from the network
		unsigned netType;
		unsigned base, n;
		float* dParam = nullptr;
		float* dState = nullptr;
	};

	void init(const std::vector<const Network*>& nets, const Configuration& conf);
	void releaseAll() noexcept;  // every device and host resource made so far
	float* currentState(const HostType& t) const;
	unsigned localIdx(unsigned g) const;
	bool findLocal(unsigned g, unsigned* l) const;  // localIdx without throwing (one network)
	void locate(unsigned g, const HostType** t, unsigned* i) const;
	size_t synapseKey(uint64_t id);
	// the connectivity built on the device, one network at a time: each
	// network's neurons contiguous in the simulation's local order (one
	// network, or a batch of networks of one neuron type each), its global
	// ids within a dense table of at most 4 entries per neuron plus 2^20,
	// fewer than 2^31 - 1 synapses and delay-group rows per network, and
	// no type that reads the reverse matrix of all synapses
	struct DevicePart {
		uint32_t srcBase = 0, nLocal = 0;
		std::vector<uint32_t> g2l;  // global id -> local index
		uint64_t synOff = 0, plOff = 0, plastic = 0;
	};
	bool planDeviceBuild(const std::vector<const Network*>& nets, bool stdp, std::vector<DevicePart>& parts) const;
	void buildOnDevice(const std::vector<const Network*>& nets, std::vector<DevicePart>& parts, bool deliver,
			std::vector<unsigned long long>& outPtr, std::vector<unsigned long long>& rcmPtr, uint64_t& dlvGroups);
	bool m_builtOnDevice = false;
	uint64_t m_dlvGroups = 0;
	// the device build keeps, per synapse in insertion order, its local
	// source, position in the forward matrix, global target, delay and
	// plasticity on the device until the first synapse query builds the
	// host query tables from them
	struct KeptSynapses {
		uint32_t* src = nullptr;
		uint32_t* pos = nullptr;
		uint32_t* tgt = nullptr;
		uint8_t* delay = nullptr;
		uint8_t* plastic = nullptr;
	} m_kept;
	void ensureQueryTables();
	void freeKept() noexcept;
	void launchStep(bool fullRecord);
	void launchSteps(unsigned n);
	void launchRun(unsigned n, bool finalStdp = true, const uint32_t* stim = nullptr, uint32_t nf = 0, uint32_t ni = 0,
			uint32_t* hostFired = nullptr);
	uint64_t m_barrierBase = 0;  // the barrier counter's value after the launches so far
	void flushStdp();
	// resident step loop
	void launchServe();
	void stopServe() noexcept;
	void stepResident(uint32_t nf, uint32_t ni);
	const std::vector<unsigned>& collectFired();
	ServeCtl* m_hServe = nullptr;   // mapped pinned
	ServeCtl* m_dServe = nullptr;
	cudaEvent_t m_serveEnd = nullptr;  // recorded after each launch of the loop
	bool m_serving = false;            // a launch of the loop may still be running
	uint32_t m_serveSeq = 1;           // sequence number of the next request
	bool m_barrierStale = false;       // the barrier counter must restart from zero
	bool m_stdpPending = false;  // the last step's STDP accumulation has not run yet
	void checkBarrier();
	GridBarrier* m_barrier = nullptr;
	uint32_t* m_hBarrierError = nullptr;  // pinned copy of m_barrier->error
	bool m_barrierUsed = false;           // a persistent launch ran since the last checkBarrier
	unsigned m_runGrid = 0;  // co-resident CTAs of run_kernel at m_runT threads (0: no cooperative launch)
	uint32_t m_runP = 0;     // neurons per partition of run_kernel
	uint32_t m_runT = 384;
	unsigned runGridFor(uint32_t T) const;
	void buildGraph();
	static constexpr unsigned GRAPH_STEPS = 100;
	cudaGraphExec_t m_graph = nullptr;
	uint32_t m_graphP = 0, m_graphT = 0;
	unsigned long long* m_hCycle = nullptr;
	size_t decodeBatchStep(uint32_t r, unsigned step, unsigned* counts, unsigned* ids, size_t pos, size_t cap);
	std::vector<std::vector<uint32_t>> m_batchScratch;
	unsigned m_deliverGrid = 1184;  // CTAs of deliver_kernel
	unsigned m_applyGrid = 1184;    // CTAs of apply_kernel
	uint32_t m_P = 256, m_T = 256;
	uint32_t m_maxOutDeg = 0, m_maxPlasticInDeg = 0;
	int m_sms = 148;
	void applyStdpDevice(int32_t fxReward);
	void sync();

	int m_device = 0;
	cudaStream_t m_stream = nullptr;
	DevSim m_dev;
	unsigned m_N = 0;
	uint64_t m_nsyn = 0;
	unsigned m_maxDelay = 0;
	std::vector<HostType> m_types;
	std::vector<unsigned> m_l2g;
	std::vector<uint8_t> m_ltype;
	std::vector<unsigned> m_netLocal;  // index within its own network's local order
	std::vector<uint32_t> m_netOf;     // network of each neuron (batches only)
	std::vector<std::unordered_map<unsigned, unsigned>> m_g2l;  // per network: global id -> index
	struct NetTypeRange { unsigned hostType, offset, count; };
	std::vector<std::vector<NetTypeRange>> m_netTypes;  // per network and type id
	unsigned m_nets = 1;

	// synapse bookkeeping for queries: for local source l, the synapse with
	// per-source index i is m_srcOrder[m_srcStart[l] + i] (an insertion-order
	// position k); its device slot is m_pos[k]
	bool m_writeOnly = false;
	std::vector<uint64_t> m_srcStart;
	std::vector<uint64_t> m_srcOrder;
	std::vector<uint64_t> m_pos;
	std::vector<unsigned> m_synDelay;  // by insertion order
	std::vector<uint8_t> m_synPlastic; // by insertion order
	std::vector<unsigned> m_synTarget; // global target, by insertion order
	std::vector<uint64_t> m_queried;

	// step state
	uint64_t m_cycle = 0;        // steps since creation (never reset)
	bool m_weightsClamped = false; // every plastic weight within its STDP limits
	unsigned long m_timerSteps = 0;
	std::chrono::steady_clock::time_point m_timerStart;

	// host staging
	uint32_t* m_hFired = nullptr;  // pinned, [R][W]
	uint32_t* m_hStim = nullptr;   // mapped pinned stimulus staging of step()
	uint32_t* m_dStimMapped = nullptr;
	size_t m_stimCap = 0;
	uint32_t* m_hFiredMapped = nullptr;  // mapped pinned [W]: step()'s fired words
	uint32_t* m_hFiredIds = nullptr;     // mapped pinned [N]: the resident loop's fired ids
	uint32_t* m_dFiredIdsMapped = nullptr;
	uint32_t* m_dFiredMapped = nullptr;
	std::vector<uint32_t> m_stepScratch;
	std::vector<std::pair<uint32_t, float>> m_stepCurrents;
	std::vector<unsigned> m_fired;
	std::vector<uint32_t> m_outDegree;

	cudaEvent_t m_ev0 = nullptr, m_ev1 = nullptr;
	std::vector<cudaEvent_t> m_evPool;
	std::vector<std::pair<int, size_t>> m_evUse;  // (kernel kind, first event index)
	size_t m_evNext = 0;
	bool m_inRun = false;
	void timedBegin(int kind);
	void timedEnd();
	std::vector<void*> m_allocs;
	template<typename T> T* dalloc(size_t n);
};

// Device copies of the libm calibration tables (one per device, kept for
// the life of the process).
LibmCalib device_calibration(int device);

} // namespace nemo_b200
