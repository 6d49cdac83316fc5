// simulation.cu -- kernels and host orchestration of the B200 backend.
#include "simulation.hpp"

#include <string.h>

#include <algorithm>
#include <atomic>
#include <mutex>

#include "kernels.cuh"
#include "hugevec.hpp"
#include "libm_calib.hpp"
#include "construction.hpp"
#include "plugins.hpp"

namespace nemo_b200 {

#define NB_CUDA(call)                                                              \
	do {                                                                           \
		cudaError_t err_ = (call);                                                 \
		if(err_ != cudaSuccess) {                                                  \
			NB_THROW(NEMO_CUDA_ERROR, "CUDA error %s at %s:%d (%s)",               \
					cudaGetErrorString(err_), __FILE__, __LINE__, #call);          \
		}                                                                          \
	} while(0)

// ---------------------------------------------------------------------------
// kernels

// A step has two phases, in the reference's order (src/nemo/cpu/
// Simulation.cpp:94-111, deliverSpikes at :259-288):
//
//  - the pre-phase of step t delivers the spikes that arrive at t: every
//    (source, delay d) group whose source fired at t - d, published by the
//    update of step t - 1, adds its weights -- read now, at arrival, as the
//    reference does -- into each target's accumulator; it also runs the
//    STDP accumulation of step t - 1;
//  - the update of step t advances every neuron and publishes, as ranges in
//    two work lists (WorkList), the delay groups that arrive at t + 1 and
//    the incoming plastic synapses of this step's STDP targets.
//
// A pre-phase spreads each list's entries evenly over its warps, so its
// work is balanced however the spikes fall.  The phases run as two kernels
// per step (deliver_kernel, update_kernel) or inside the persistent step
// loop (run_kernel), one cooperative launch for many steps.  The STDP
// accumulation of the last step runs before applyStdp (flushStdp);
// deliveries stay pending until the next step, so they read the weights
// applyStdp leaves.  applyStdp itself walks the forward matrix one slice
// at a time (below).

// applyStdp writes each changed weight into the forward matrix, at an index
// scattered over all of it.  To keep those writes in L2, it processes the
// forward matrix in slices of APPLY_SLICE_ENTRIES entries (16 MB of
// weights; 8 MB slices took 9% longer at 100k x 1000, 32 MB 6%): item
// (slice k, 32 targets) covers the targets' incoming plastic synapses whose
// forward index lies in slice k.  Each target's reverse-matrix entries are
// sorted by forward index, so they form one run per slice, found in a
// table built with the matrix; the items run slice-major, so the warps in
// flight write into about three slices at a time.
constexpr uint32_t APPLY_SLICE_ENTRIES = 4u << 20;
constexpr uint32_t APPLY_MAX_SLICES = 64;
constexpr uint32_t APPLY_ILP = 4;  // entries per lane per round

// Chained launches (programmatic dependent launch): deliver_kernel and
// update_kernel alternate on one stream, each launched while its
// predecessor still runs.  A chained kernel's CTAs first wait until the
// previous grid has completed and its writes are visible (a no-op when the
// kernel was launched without the chaining attribute), then allow the next
// kernel's launch to begin, so only that launch's latency overlaps, never
// the work of two steps.
__device__ __forceinline__ void chain_wait_then_release()
{
	asm volatile("griddepcontrol.wait;" ::: "memory");
	asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Launches `kernel` on `st` chained to the stream's previous kernel.  A
// launch error is reported as for <<<...>>> (cudaGetLastError), not thrown.
template<typename... KArgs, typename... Args>
cudaError_t launch_chained(void (*kernel)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t st,
		Args... args)
{
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = dim3(grid);
	cfg.blockDim = dim3(block);
	cfg.dynamicSmemBytes = smem;
	cfg.stream = st;
	cudaLaunchAttribute attr;
	attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
	attr.val.programmaticStreamSerializationAllowed = 1;
	cfg.attrs = &attr;
	cfg.numAttrs = 1;
	return cudaLaunchKernelEx(&cfg, kernel, ((KArgs) args)...);
}

__device__ __forceinline__ unsigned long long global_ns()
{
	unsigned long long t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

// phase trace point `mark` of trace row `row` (~0u: not traced), by thread 0
__device__ __forceinline__ void trace_mark(const DevSim& S, uint32_t row, uint32_t mark)
{
	if(row != ~0u && threadIdx.x == 0) {
		S.trace[((size_t) row * gridDim.x + blockIdx.x) * TRACE_MARKS + mark] = global_ns();
	}
}

// Inside a CUDA graph the step's cycle comes from a device counter (the
// graph is replayed at different cycles): cycle = *cycleDev + offset.
__device__ __forceinline__ void step_indices(const DevSim& S, uint32_t offset, uint32_t& cur, uint32_t& ring,
		uint32_t& cycleLo)
{
	const unsigned long long c = *S.cycleDev + offset;
	cur = (uint32_t) (c & 1);
	ring = (uint32_t) (c % S.R);
	cycleLo = (uint32_t) c;
}

__global__ void advance_cycle_kernel(unsigned long long* cycle, uint32_t by)
{
	*cycle += by;
}

__device__ __forceinline__ uint32_t warp_inclusive_scan(uint32_t x)
{
	const uint32_t lane = threadIdx.x & 31;
#pragma unroll
	for(int o = 1; o < 32; o <<= 1) {
		uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
		if(lane >= (uint32_t) o) x += y;
	}
	return x;
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long x)
{
#pragma unroll
	for(int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
	return x;
}

constexpr uint32_t BUCKET = 32;  // entries per bucket of a work list

// group g = entries [e, e + len) = [start, start + len) of the list's array
__device__ __forceinline__ void write_group(const WorkList& L, uint32_t g, uint32_t e, unsigned long long start,
		uint32_t len)
{
	L.group[g] = make_uint4((uint32_t) start, (uint32_t) (start >> 32), len, e);
	for(uint32_t b = (e + BUCKET - 1) / BUCKET; b * BUCKET < e + len; ++b) L.bucket[b] = g;
}

// End of source n's delay-d group (its synapses of delay <= d) within its
// row, which holds the synapses sorted by delay.
__device__ __forceinline__ uint32_t delay_end(const DevSim& S, uint32_t n, uint32_t d)
{
	if(d == 0) return 0;
	const size_t i = (size_t) n * S.dStride + (d - 1);
	return S.dEnd16 ? (uint32_t) S.dEnd16[i] : S.dEnd32[i];
}

// CTA-level counters of one step, added to the per-step ring counters once
// per CTA, and the CTA's work-list reservations (groups << 32 | entries)
struct CtaCounters {
	uint32_t fired;
	unsigned long long events, stdp;
	unsigned long long resD, resS;    // the warps' reservations, summed
	unsigned long long baseD, baseS;  // the CTA's place in the delivery / STDP lists
};

// Neuron update of step t (src/nemo/cpu/Simulation.cpp:94-111 minus the
// delivery and STDP loops) for the neurons [first, last) of one CTA (first a
// multiple of 32, so warps cover whole bit-vector words); the CTA's
// blockDim.x threads loop over them.  Every thread of the CTA calls it.
// cur = t & 1.
// hostFired: also write the fired bit-vector words there (host memory)
// cycleLo: the low 32 bits of t (the state slot of a type with history)
__device__ __forceinline__ void update_range(const DevSim& S, uint32_t first, uint32_t last, uint32_t cur,
		uint32_t ring, uint32_t cycleLo, CtaCounters& C, bool preNoise = false, uint32_t* hostFired = nullptr)
{
	const uint32_t tid = threadIdx.x, lane = tid & 31;
	const uint64_t* histPrev = S.hist + (size_t) (cur ^ 1u) * S.N;
	uint64_t* histCur = S.hist + (size_t) cur * S.N;

	for(uint32_t base = first; base < last; base += blockDim.x) {
		const uint32_t n = base + tid;
		bool fired = false, target = false;
		uint32_t fw = 0, outdeg = 0, indeg = 0;
		unsigned long long ob = 0, rb = 0;
		uint64_t pend = 0;
		bool hist_nonzero = false;
		uint32_t g1End = 0, gpD = 0, gpBeg = 0, gpEnd = 0;
		if(n < last) {
			uint32_t k = 0;
			while(k + 1 < S.ntypes && n >= S.types[k + 1].base) ++k;
			const TypeRange& T = S.types[k];
			const uint32_t nl = n - T.base;
			// every load of this neuron before its first store: this step's
			// synaptic input, stimulus, history, CSR spans, delay groups,
			// parameters, state and RNG words
			const ulonglong2 acc = S.slot[n];
			const float ext = S.curExt[n];
			fw = S.fstim[n >> 5];
			const uint64_t hp = histPrev[n];
			const unsigned long long o0 = S.outPtr[n], o1 = S.outPtr[n + 1];
			const uint64_t dm = S.delayMask[n];
			unsigned long long r0 = 0, r1 = 0;
			if(S.stdp) {
				r0 = S.rcmPtr[n];
				r1 = S.rcmPtr[n + 1];
			}
			NeuronRegs R;
			load_neuron(S, T, nl, n, R, preNoise);
			// the delay-group ends this neuron will most likely publish, loaded
			// before the arithmetic: its delay-1 group (if it fires now) and
			// the first group pending from its earlier spikes
			const uint64_t pendPrev = (hp << 1) & dm;
			if(dm & 1ull) g1End = delay_end(S, n, 1);
			if(pendPrev) {
				gpD = (uint32_t) __ffsll((long long) pendPrev);
				gpBeg = delay_end(S, n, gpD - 1);
				gpEnd = delay_end(S, n, gpD);
			}

			if(acc.x | acc.y) S.slot[n] = make_ulonglong2(0, 0);
			if(__float_as_uint(ext) != 0u) S.curExt[n] = 0.0f;
			// wfx_toFloat of the int64 sums (src/nemo/fixedpoint.cpp:40-49)
			const float cE = wfx_to_float((long long) acc.x);
			const float cI = wfx_to_float((long long) acc.y);
			const bool fs = (fw >> lane) & 1u;
			// a Kuramoto oscillator never fires; its phase is updated by the
			// pass after this loop
			if(T.kind != KIND_KURAMOTO) {
				fired = update_neuron(S, T, R, cE, cI, ext, fs);
				store_neuron(S, T, nl, n, R);
			}
			const uint64_t h = (hp << 1) | (uint64_t) fired;
			histCur[n] = h;
			hist_nonzero = h != 0;
			ob = o0;
			if(fired) outdeg = (uint32_t) (o1 - o0);
			// groups arriving next step: delay d of a source that fired d - 1
			// steps ago (bit d - 1 of the history; dm holds only the delays
			// the source has and deliverSpikes accepts)
			pend = h & dm;
			// STDP target: fired |post| steps ago (ConnectivityMatrix.cpp:206)
			if(S.stdp && (h & S.sp.postFireMask)) {
				rb = r0;
				indeg = (uint32_t) (r1 - r0);
				target = indeg > 0;
			}
		}
		const uint32_t fb = __ballot_sync(0xffffffffu, fired);
		const uint32_t rbits = __ballot_sync(0xffffffffu, hist_nonzero);
		if(lane == 0 && n < last) {
			S.firedRing[(size_t) ring * S.W + (n >> 5)] = fb;
			if(hostFired) hostFired[n >> 5] = fb;
			S.recent[(size_t) cur * S.recentWords + (n >> 5)] = rbits;
			if(fw) S.fstim[n >> 5] = 0u;
		}
		// the delay groups that arrive next step and the incoming plastic
		// synapses of this step's STDP targets, both reserved at once
		// range [e0, e1) of this neuron's delay-d group in its row
		auto group = [&](uint32_t d, uint32_t& e0, uint32_t& e1) {
			if(d == 1) { e0 = 0; e1 = g1End; }
			else if(d == gpD) { e0 = gpBeg; e1 = gpEnd; }
			else { e0 = delay_end(S, n, d - 1); e1 = delay_end(S, n, d); }
		};
		uint32_t ngD = 0, neD = 0;
		for(uint64_t b = pend; b; b &= b - 1) {
			uint32_t e0, e1;
			group((uint32_t) __ffsll((long long) b), e0, e1);
			neD += e1 - e0;
			++ngD;
		}
		const uint32_t ngS = target ? 1u : 0u, neS = target ? indeg : 0u;
		// reserve both lists for the whole CTA: warps add their totals to
		// shared counters, one thread reserves the CTA's share of each
		// global list (so that warps do not queue on two global addresses)
		const uint32_t igD = warp_inclusive_scan(ngD), ieD = warp_inclusive_scan(neD);
		const uint32_t igS = warp_inclusive_scan(ngS), ieS = warp_inclusive_scan(neS);
		unsigned long long wD = 0, wS = 0;
		if(lane == 31) {
			if(igD | ieD) wD = atomicAdd(&C.resD, ((unsigned long long) igD << 32) | ieD);
			if(igS | ieS) wS = atomicAdd(&C.resS, ((unsigned long long) igS << 32) | ieS);
		}
		__syncthreads();
		if(tid == 0) {
			C.baseD = C.resD ? atomicAdd(&S.dlvWork.count[cur], C.resD) : 0ull;
			C.baseS = C.resS ? atomicAdd(&S.stdpWork.count[cur], C.resS) : 0ull;
			C.resD = 0;
			C.resS = 0;
		}
		__syncthreads();
		wD = __shfl_sync(0xffffffffu, wD, 31);
		wS = __shfl_sync(0xffffffffu, wS, 31);
		if(ngD) {
			uint32_t gD = (uint32_t) (C.baseD >> 32) + (uint32_t) (wD >> 32) + igD - ngD;
			uint32_t eD = (uint32_t) C.baseD + (uint32_t) wD + ieD - neD;
			for(uint64_t b = pend; b; b &= b - 1) {
				uint32_t e0, e1;
				group((uint32_t) __ffsll((long long) b), e0, e1);
				write_group(S.dlvWork, gD++, eD, ob + e0, e1 - e0);
				eD += e1 - e0;
			}
		}
		if(ngS) {
			write_group(S.stdpWork, (uint32_t) (C.baseS >> 32) + (uint32_t) (wS >> 32) + igS - ngS,
					(uint32_t) C.baseS + (uint32_t) wS + ieS - neS, rb, indeg);
		}
		// targets touched in this STDP period, for applyStdp
		const uint32_t tb = __ballot_sync(0xffffffffu, target);
		if(tb && lane == 0) atomicOr(&S.touchedBits[n >> 5], tb);
		if(fb) {
			const unsigned long long ev = warp_sum(fired ? outdeg : 0);
			if(lane == 0) {
				atomicAdd(&C.fired, (uint32_t) __popc(fb));
				atomicAdd(&C.events, ev);
			}
		}
		if(tb) {
			const unsigned long long se = warp_sum(target ? indeg : 0);
			if(lane == 0) atomicAdd(&C.stdp, se);
		}
	}
	// the phases of the Kuramoto oscillators among [first, last), apart from
	// the loop above so that no register of it stays live across the sums
	if(S.allSrc) {
		for(uint32_t n = first + tid; n < last; n += blockDim.x) {
			uint32_t k = 0;
			while(k + 1 < S.ntypes && n >= S.types[k + 1].base) ++k;
			const TypeRange& T = S.types[k];
			if(T.kind == KIND_KURAMOTO) {
				update_kuramoto(T.param, T.state, T.base, T.n, n - T.base, S.allSrc, S.allW, S.allPtr[n], S.allPtr[n + 1],
						cycleLo);
			}
		}
	}
}

// Adds the CTA's counters to those of ring position `ring` and clears them
// (after a __syncthreads that follows the last update_range of the step).
__device__ __forceinline__ void flush_counters(const DevSim& S, uint32_t ring, CtaCounters& C)
{
	if(threadIdx.x == 0) {
		if(C.fired) atomicAdd(&S.firedCount[ring], C.fired);
		if(C.events) atomicAdd(&S.eventCount[ring], C.events);
		if(C.stdp) atomicAdd(&S.stdpCount[ring], C.stdp);
		C.fired = 0;
		C.events = 0;
		C.stdp = 0;
	}
}

// One step's neuron update: CTA c owns the partition of P consecutive
// neurons starting at c * P (P a multiple of 32).
// Two instances: up to 1024 threads per CTA (64 registers), and up to 256
// threads with at least 5 CTAs per SM (48 registers, 40 warps per SM) for
// the shapes a large network's update takes, where more resident warps hide
// more of each neuron's chain of loads.
template<unsigned MAXT, unsigned MINB>
__global__ void __launch_bounds__(MAXT, MINB)
update_kernel(const DevSim S, uint32_t P, uint32_t cur, uint32_t ring, uint32_t cycleLo, uint32_t offset,
		int fromDev, uint32_t* hostFired = nullptr)
{
	chain_wait_then_release();
	if(fromDev) step_indices(S, offset, cur, ring, cycleLo);
	__shared__ CtaCounters sC;
	if(threadIdx.x == 0) sC = CtaCounters{ 0, 0, 0, 0, 0, 0, 0 };
	__syncthreads();
	const uint32_t first = blockIdx.x * P;
	update_range(S, first, min(S.N, first + P), cur, ring, cycleLo, sC, false, hostFired);
	__syncthreads();
	flush_counters(S, ring, sC);
}

// the update_kernel instance for the two-launch step's threads per CTA
using UpdateKernel = void (*)(const DevSim, uint32_t, uint32_t, uint32_t, uint32_t, uint32_t, int, uint32_t*);
static UpdateKernel update_kernel_for(uint32_t threads)
{
	return threads <= 256 ? update_kernel<256, 5> : update_kernel<1024, 1>;
}

// 64-bit integer reduction into an accumulator word (its result unused)
__device__ __forceinline__ void red_add_u64(unsigned long long* p, unsigned long long v)
{
	asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" :: "l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void red_add_s32(int32_t* p, int32_t v)
{
	asm volatile("red.relaxed.gpu.global.add.s32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}

// One warp's share of a work list: the entries [E0, E1) of the list's
// ne entries, in rounds of 32 x K, each lane finding the group of its entry
// by a binary search over 32 consecutive group descriptors (one per lane).
//  KIND 0 (delivery): add each synapse's weight into its target's
//          accumulator: the E (w >= 0) or I (w < 0) int64 sum, as
//          deliverSpikesOne (src/nemo/cpu/Simulation.cpp:293-307); integer
//          addition is associative, so the sums do not depend on the order
//          of the reductions
//  KIND 1 (STDP): accumulation over the incoming plastic synapses of a
//          target (ConnectivityMatrix::accumulateStdp,
//          ConnectivityMatrix.cpp:193-227) with the history `hist` of the
//          step that published the list
template<int KIND, int K>
__device__ __forceinline__ void process_list(const DevSim& S, const WorkList& L, uint32_t ng, uint32_t ne,
		const uint64_t* hist, const uint32_t* recent, uint32_t warp, uint32_t nwarps)
{
	if(ne == 0) return;
	const uint32_t lane = threadIdx.x & 31;
	const uint32_t per = (ne + nwarps - 1) / nwarps;
	const uint32_t E0 = warp * per;
	if(E0 >= ne) return;
	const uint32_t E1 = min(ne, E0 + per);
	uint32_t g = L.bucket[E0 / BUCKET];
	for(;;) {
		// descriptors g .. g + 31; lanes past the last group hold an offset
		// above every entry
		const bool valid = g + lane < ng;
		const uint4 d = valid ? L.group[g + lane] : make_uint4(0, 0, 0, 0xffffffffu);
		const uint32_t lastLane = min(31u, ng - 1 - g);
		const uint32_t coverEnd = __shfl_sync(0xffffffffu, d.w + d.z, lastLane);
		const uint32_t lo = max(E0, __shfl_sync(0xffffffffu, d.w, 0)), hi = min(E1, coverEnd);
		for(uint32_t base = lo; base < hi; base += 32 * K) {
			// entry indices into the forward / the reverse matrix, both shorter than
			// 2^32 entries (checked when the simulation is built)
			uint32_t idx[K];
#pragma unroll
			for(int j = 0; j < K; ++j) {
				const uint32_t e = base + lane + 32 * j;
				uint32_t q = 0;
#pragma unroll
				for(uint32_t step = 16; step > 0; step >>= 1) {
					if(__shfl_sync(0xffffffffu, d.w, q + step) <= e) q += step;
				}
				idx[j] = __shfl_sync(0xffffffffu, d.x, q) + (e - __shfl_sync(0xffffffffu, d.w, q));
			}
			if(KIND == 0) {
				uint32_t tg[K], wt[K];
#pragma unroll
				for(int j = 0; j < K; ++j) {
					if(base + lane + 32 * j < hi) {
						tg[j] = __ldcs(S.synTgt + idx[j]);
						wt[j] = __ldcs(S.synW + idx[j]);
					}
				}
#pragma unroll
				for(int j = 0; j < K; ++j) {
					if(base + lane + 32 * j < hi) {
						const int32_t w = (int32_t) wt[j];
						unsigned long long* a = reinterpret_cast<unsigned long long*>(S.slot + (tg[j] & (MAX_NEURONS - 1)));
						red_add_u64(a + (w >= 0 ? 0 : 1), (unsigned long long) (long long) w);
					}
				}
			} else {
				uint32_t sd[K];
				uint64_t h[K];
#pragma unroll
				for(int j = 0; j < K; ++j) if(base + lane + 32 * j < hi) sd[j] = __ldcs(S.rcmSrc + idx[j]);
#pragma unroll
				for(int j = 0; j < K; ++j) {
					// a source that fired in none of the last 64 steps has history 0
					const uint32_t src = sd[j] & (MAX_NEURONS - 1);
					h[j] = 0;
					if(base + lane + 32 * j < hi && (!recent || ((recent[src >> 5] >> (src & 31)) & 1u))) h[j] = hist[src];
				}
#pragma unroll
				for(int j = 0; j < K; ++j) {
					if(base + lane + 32 * j < hi) {
						const uint32_t delay = (sd[j] >> 26) + 1;
						const int32_t dw = stdp_weight_change(S.sp, h[j] >> (delay & 63));
						// one lane owns each accumulator in a step: an int32
						// reduction (wrapping) needs no load of the old value
						if(dw != 0) red_add_s32(S.rcmAcc + idx[j], dw);
					}
				}
			}
		}
		if(hi >= E1) break;
		g += 32;
	}
}

// what a pre-phase does
constexpr uint32_t PHASE_DELIVER = 1;  // the published delay groups
constexpr uint32_t PHASE_STDP = 2;     // the published STDP groups
constexpr uint32_t PHASE_RESET = 4;    // empty the lists the next update publishes into

// Pre-phase of a step over the lists published by the update of the step
// with parity `pub`.  When there are both deliveries and STDP entries, the
// warps of every CTA split into two groups in proportion to the work, so
// that the two lists' chains of dependent loads run at the same time on
// every SM; each list's entries are spread evenly over its group's warps
// across the grid.  Every thread of the grid calls this.
__device__ __forceinline__ void deliver_range(const DevSim& S, uint32_t pub, uint32_t what)
{
	const unsigned long long cd = (what & PHASE_DELIVER) ? S.dlvWork.count[pub] : 0ull;
	const unsigned long long cs = (what & PHASE_STDP) ? S.stdpWork.count[pub] : 0ull;
	const uint32_t nd = (uint32_t) cd, ns = (uint32_t) cs;
	const uint32_t wpc = blockDim.x >> 5, lw = threadIdx.x >> 5;
	if((what & PHASE_RESET) && blockIdx.x == 0 && threadIdx.x == 0) {
		S.dlvWork.count[pub ^ 1u] = 0;
		S.stdpWork.count[pub ^ 1u] = 0;
	}
	const uint64_t* hist = S.hist + (size_t) pub * S.N;
	// In every CTA, warps [0, ws) take the STDP list and [ws, wpc) the
	// deliveries, in proportion to their work, so that every SM runs the
	// same mix: an STDP entry (a load, a dependent history load for a
	// recently active source, a reduction where its change is nonzero)
	// costs about 3.5 deliveries.  At 100k x 1000 (352 x 512) a launch of
	// 100 steps took 2098 us, against 2134 us with 2.5, 2185 with 4.5 and
	// 2172 us when whole CTAs took one list or the other.
	constexpr unsigned long long STDP_ENTRY_COST_X2 = 7;  // twice the cost, for half steps
	uint32_t ws = ns ? wpc : 0u;
	if(nd && ns) {
		ws = (uint32_t) (((unsigned long long) wpc * STDP_ENTRY_COST_X2 * ns + (2ull * nd + STDP_ENTRY_COST_X2 * ns) / 2)
				/ (2ull * nd + STDP_ENTRY_COST_X2 * ns));
		ws = max(1u, min(wpc - 1u, ws));
		if(wpc == 1) ws = 0;  // one warp: it does both, deliveries first
	}
	const bool stdpWarp = ns && (lw < ws || wpc == 1);
	const bool dlvWarp = nd && (lw >= ws || wpc == 1);
	if(dlvWarp) {
		const uint32_t dw = wpc == 1 ? 1u : wpc - ws, first = wpc == 1 ? 0u : ws;
		// four entries a lane per round: eight loads (target and weight)
		// in flight, and no spills in the 64-register instance of the
		// persistent loop, which at eight entries spilled inside this loop
		process_list<0, 4>(S, S.dlvWork, (uint32_t) (cd >> 32), nd, hist, nullptr, blockIdx.x * dw + (lw - first),
				gridDim.x * dw);
	}
	// the sources' "fired in the last 64 steps" bits, copied to shared
	// memory by the STDP warps with asynchronous 16-byte copies; they then
	// wait for each other only (named barrier 1)
	extern __shared__ __align__(16) uint32_t sRecent[];
	if(stdpWarp) {
		const uint32_t sw = wpc == 1 ? 1u : ws;
		const bool filter = S.recentBytes != 0;
		if(filter) {
			const uint32_t* g = S.recent + (size_t) pub * S.recentWords;
			for(uint32_t q = threadIdx.x; q < S.recentWords / 4; q += sw * 32) {
				const uint32_t dst = (uint32_t) __cvta_generic_to_shared(sRecent + 4 * q);
				asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(dst), "l"(g + 4 * q) : "memory");
			}
			asm volatile("cp.async.commit_group;" ::: "memory");
			asm volatile("cp.async.wait_all;" ::: "memory");
			asm volatile("bar.sync 1, %0;" :: "r"(sw * 32) : "memory");
		}
		process_list<1, 4>(S, S.stdpWork, (uint32_t) (cs >> 32), ns, hist, filter ? sRecent : nullptr,
				blockIdx.x * sw + lw, gridDim.x * sw);
	}
	__syncthreads();  // the shared copy is rewritten by the next call
}

// A step's stimulus (src/nemo/cpu/Simulation.cpp:141-171) read from host
// memory: nf firing-stimulus indices, then ni current-stimulus indices and
// ni values (distinct indices), for the update that follows.
__device__ __forceinline__ void apply_stimulus(const DevSim& S, const uint32_t* stim, uint32_t nf, uint32_t ni)
{
	// stim is host memory that the resident step loop re-reads each step:
	// load it past the caches
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < max(nf, ni); i += gridDim.x * blockDim.x) {
		if(i < nf) {
			const uint32_t l = __ldcv(stim + i);
			atomicOr(&S.fstim[l >> 5], 1u << (l & 31));
		}
		if(i < ni) S.curExt[__ldcv(stim + nf + i)] = __uint_as_float(__ldcv(stim + nf + ni + i));
	}
}

// Pre-phase of step t (pub = (t - 1) & 1), or with what = PHASE_STDP the
// STDP accumulation of the last step before applyStdp.  With stim, it also
// applies the step's stimulus (apply_stimulus).
__global__ void __launch_bounds__(STEP_THREADS)
deliver_kernel(const DevSim S, uint32_t pub, uint32_t what, uint32_t offset, int fromDev,
		const uint32_t* stim = nullptr, uint32_t nf = 0, uint32_t ni = 0)
{
	chain_wait_then_release();
	if(fromDev) {
		uint32_t cur, ring;
		uint32_t cycleLo;
		step_indices(S, offset, cur, ring, cycleLo);
		pub = cur ^ 1u;
	}
	if(stim) apply_stimulus(S, stim, nf, ni);
	deliver_range(S, pub, what);
}

// Grid-wide barrier of the persistent kernel (all CTAs co-resident: it is
// launched cooperatively).  After a CTA barrier, thread 0 of each CTA
// arrives on a launch-wide counter with a release reduction (which makes
// the writes the CTA made before its barrier visible with it) and polls the
// counter with acquire loads until every CTA has arrived at this barrier;
// a CTA barrier then passes the acquire on to the CTA's other threads.
// Barrier b is complete when the counter reaches (b + 1) x gridDim.x.  A wait
// gives up after S.waitLimit unsuccessful polls (BARRIER_SPIN_LIMIT, seconds,
// unless nemo_b200_set_wait_limit lowered it; a phase takes microseconds): it
// sets the error word, which makes every CTA leave the step loop at its next
// barrier, and the host reports the error.

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p)
{
	uint32_t v;
	asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
	return v;
}

__device__ __forceinline__ void red_release_add(uint32_t* p, uint32_t v)
{
	asm volatile("red.release.gpu.global.add.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}

// Whether a wait gives up: after `limit` unsuccessful polls, or once another
// CTA has given up (the error word, read at every 32nd poll only, so that a
// poll costs one round trip to L2)
__device__ __forceinline__ bool give_up(GridBarrier* gb, uint32_t& polls, uint32_t limit)
{
	++polls;
	return polls > limit || ((polls & 31u) == 0 && ld_acquire(&gb->error));
}

// The barrier in two halves: grid_arrive, then work that needs nothing from
// the other CTAs, then grid_wait.  target: this CTA's count of completed
// barriers x gridDim.x (shared).
__device__ __forceinline__ void grid_arrive(GridBarrier* gb, uint32_t& target)
{
	__syncthreads();
	if(threadIdx.x == 0) {
		target += gridDim.x;
		red_release_add(&gb->count, 1u);
	}
}

// The counter is compared with its target by signed difference, so that it
// may wrap: a resident step loop runs for as long as it is used (at 285 CTAs
// and two barriers a step, 2^32 arrivals are 7.5M steps).
__device__ __forceinline__ bool reached(uint32_t value, uint32_t target) { return (int32_t) (value - target) >= 0; }

__device__ __forceinline__ bool grid_wait(GridBarrier* gb, uint32_t& target, uint32_t& ok, uint32_t limit)
{
	if(threadIdx.x == 0) {
		uint32_t polls = 0;
		while(!reached(ld_acquire(&gb->count), target)) {
			if(give_up(gb, polls, limit)) {
				atomicExch(&gb->error, 1u);
				ok = 0;
				break;
			}
			__nanosleep(20);
		}
	}
	__syncthreads();
	return ok != 0;
}

__device__ __forceinline__ bool grid_barrier(GridBarrier* gb, uint32_t& target, uint32_t& ok, uint32_t limit)
{
	__syncthreads();
	if(threadIdx.x == 0) {
		target += gridDim.x;
		red_release_add(&gb->count, 1u);
		uint32_t polls = 0;
		while(!reached(ld_acquire(&gb->count), target)) {
			if(give_up(gb, polls, limit)) {
				atomicExch(&gb->error, 1u);
				ok = 0;
				break;
			}
			__nanosleep(20);
		}
	}
	__syncthreads();
	return ok != 0;
}

// Persistent step loop: `steps` consecutive steps from cycle `cycle0` in one
// cooperative launch, each step's pre-phase and update separated by grid
// barriers, then the STDP accumulation of the last step (so applyStdp may
// follow directly; its deliveries stay pending for the next step).  CTA c
// owns the partitions c, c + gridDim.x, ... of P neurons; the pre-phases
// spread the work lists over all CTAs of the grid.  After each pre-phase
// the CTAs compute the step's noise while the barrier completes.
// Identical results to deliver_kernel + update_kernel per step.
// base: the barrier counter's value when the launch starts.  Without
// finalStdp the last step's STDP accumulation is left to the next
// pre-phase, as after a two-launch step.  stim (the first step's stimulus,
// apply_stimulus) and hostFired (the last step's fired words) serve
// nemo_step.
// One step of the persistent loop at cycle c (the pre-phase, the noise in
// the shadow of its barrier, the update), ending at a grid barrier; false
// when a barrier wait gave up.
__device__ __forceinline__ bool persistent_step(const DevSim& S, uint32_t P, unsigned long long c, GridBarrier* gb,
		uint32_t& sTarget, uint32_t& sOk, CtaCounters& sC, const uint32_t* stim, uint32_t nf, uint32_t ni,
		uint32_t* hostFired, uint32_t row = ~0u)
{
	trace_mark(S, row, 0);
	__shared__ uint32_t sRng[4 * NOISE_STAGE];
	__shared__ float sSigma[NOISE_STAGE];
	const uint32_t nparts = (S.N + P - 1) / P;
	const uint32_t cur = (uint32_t) (c & 1);
	const uint32_t ring = (uint32_t) (c % S.R);
	// one partition of at most one neuron per thread: its noise inputs are
	// copied to shared memory while the pre-phase runs
	const bool staged = nparts <= gridDim.x && P <= blockDim.x && P <= NOISE_STAGE;
	if(staged && blockIdx.x < nparts) {
		stage_noise_inputs(S, blockIdx.x * P, min(S.N, blockIdx.x * P + P), sRng, sSigma);
	}
	if(stim) apply_stimulus(S, stim, nf, ni);
	deliver_range(S, cur ^ 1u, PHASE_DELIVER | PHASE_STDP | PHASE_RESET);
	if(staged) asm volatile("cp.async.wait_all;" ::: "memory");
	// while the other CTAs finish the pre-phase: this step's noise of this
	// CTA's neurons (it depends on their RNG words only)
	grid_arrive(gb, sTarget);
	trace_mark(S, row, 1);
	if(staged) {
		if(blockIdx.x < nparts) {
			precompute_noise_staged(S, blockIdx.x * P, min(S.N, blockIdx.x * P + P), sRng, sSigma);
		}
	} else {
		for(uint32_t p = blockIdx.x; p < nparts; p += gridDim.x) precompute_noise(S, p * P, min(S.N, p * P + P));
	}
	if(!grid_wait(gb, sTarget, sOk, S.waitLimit)) return false;
	trace_mark(S, row, 2);
	for(uint32_t p = blockIdx.x; p < nparts; p += gridDim.x) {
		update_range(S, p * P, min(S.N, p * P + P), cur, ring, (uint32_t) c, sC, true, hostFired);
	}
	__syncthreads();
	flush_counters(S, ring, sC);
	trace_mark(S, row, 3);
	const bool ok = grid_barrier(gb, sTarget, sOk, S.waitLimit);
	trace_mark(S, row, 4);
	return ok;
}

// TRACE: the instance with the phase trace (tracePhases).  MAXT, MINB: up
// to 768 threads, one CTA per SM (80 registers), or up to 512 threads, two
// CTAs per SM (64 registers).
template<bool TRACE, unsigned MAXT, unsigned MINB>
__global__ void __launch_bounds__(MAXT, MINB)
run_kernel(const DevSim S, uint32_t P, uint32_t steps, unsigned long long cycle0, GridBarrier* gb, uint32_t base,
		int finalStdp, const uint32_t* stim, uint32_t nf, uint32_t ni, uint32_t* hostFired)
{
	__shared__ CtaCounters sC;
	__shared__ uint32_t sTarget, sOk;
	if(threadIdx.x == 0) {
		sC = CtaCounters{ 0, 0, 0, 0, 0, 0, 0 };
		sTarget = base;
		sOk = 1;
	}
	__syncthreads();
	for(uint32_t k = 0; k < steps; ++k) {
		if(!persistent_step(S, P, cycle0 + k, gb, sTarget, sOk, sC, k == 0 ? stim : nullptr, nf, ni,
				k + 1 == steps ? hostFired : nullptr, TRACE && k < S.traceSteps ? k : ~0u)) {
			return;
		}
	}
	if(steps && finalStdp) {
		const uint32_t last = (uint32_t) ((cycle0 + steps - 1) & 1);
		deliver_range(S, last, PHASE_STDP);
		if(!grid_barrier(gb, sTarget, sOk, S.waitLimit)) return;
		if(blockIdx.x == 0 && threadIdx.x == 0) S.stdpWork.count[last] = 0;
	}
}

// The resident step loop of nemo_step: one cooperative launch that stays on
// the GPU between nemo_step calls and runs one step per request, so that a
// call costs a step and a round trip through host memory instead of kernel
// launches and a stream synchronisation.
//
// The host writes the step's stimulus (stim, mapped host memory), its sizes
// and then the request's sequence number to ctl->go.  Thread 0 of CTA 0
// polls ctl->go and broadcasts the request (its sequence number) through
// gb->cmd, which the other CTAs poll.  After the step's final barrier CTA 0
// writes the step's fired neurons as global ids to hostIds (mapped), their
// number and the step's synaptic events to ctl, and then the sequence
// number to ctl->done.  The loop ends when the host asks it to stop
// (go = the next sequence number | SERVE_STOP) or after idleNs nanoseconds
// without a request (the host then launches it again for the next call);
// a wait that gives up ends it with the barrier's error word set.  Step k
// runs cycle cycle0 + k, exactly as run_kernel's step.
constexpr uint32_t SERVE_POLL_LIMIT = 1u << 26;  // bounds the idle wait even without the timer



__device__ __forceinline__ unsigned long long ld_relaxed_sys_u64(const unsigned long long* p)
{
	unsigned long long v;
	asm volatile("ld.relaxed.sys.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
	return v;
}

__device__ __forceinline__ void st_release_sys(uint32_t* p, uint32_t v)
{
	asm volatile("st.release.sys.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}

// n words from device memory (just written by other CTAs: read from L2)
// to host memory by the threads of one CTA, 16 bytes a thread where both
// ends are 16-byte aligned
__device__ __forceinline__ void copy_words_to_host(const uint32_t* src, uint32_t* dst, uint32_t n)
{
	uint32_t i0 = 0;
	if((((uintptr_t) src | (uintptr_t) dst) & 15u) == 0) {
		const uint4* s4 = reinterpret_cast<const uint4*>(src);
		uint4* d4 = reinterpret_cast<uint4*>(dst);
		for(uint32_t i = threadIdx.x; i < n / 4; i += blockDim.x) d4[i] = __ldcg(s4 + i);
		i0 = n & ~3u;
	}
	for(uint32_t i = i0 + threadIdx.x; i < n; i += blockDim.x) dst[i] = __ldcg(src + i);
}

__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v)
{
	asm volatile("st.release.gpu.global.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}

// The fired neurons of a step (words: its fired bit-vector) as global ids in
// ascending local index (setFiring, src/nemo/cpu/Simulation.cpp:200-208),
// by the threads of one CTA: each thread takes a run of words, a CTA-wide
// scan of their counts places its ids, which are staged in shared memory
// (or, beyond SERVE_IDS_SMEM of them, in S.firedIds) and then stored to host
// memory in consecutive words per warp.  Returns the count.
constexpr uint32_t SERVE_IDS_SMEM = 4096;

__device__ uint32_t fired_ids_to_host(const DevSim& S, const uint32_t* words, uint32_t* host)
{
	__shared__ uint32_t sIds[SERVE_IDS_SMEM];
	__shared__ uint32_t sWarp[32];
	__shared__ uint32_t sTotal;
	const uint32_t T = blockDim.x, t = threadIdx.x, lane = t & 31, warp = t >> 5;
	const uint32_t per = (S.W + T - 1) / T;
	const uint32_t w0 = min(S.W, t * per), w1 = min(S.W, w0 + per);
	// up to WREG words per thread stay in registers for the second pass
	constexpr uint32_t WREG = 8;
	uint32_t wr[WREG];
	uint32_t n = 0;
#pragma unroll
	for(uint32_t j = 0; j < WREG; ++j) {
		wr[j] = w0 + j < w1 ? __ldcg(words + w0 + j) : 0u;
		n += __popc(wr[j]);
	}
	for(uint32_t w = w0 + WREG; w < w1; ++w) n += __popc(__ldcg(words + w));
	const uint32_t incl = warp_inclusive_scan(n);
	if(lane == 31) sWarp[warp] = incl;
	__syncthreads();
	if(warp == 0) {
		const uint32_t x = lane < T / 32 ? sWarp[lane] : 0u;
		const uint32_t xi = warp_inclusive_scan(x);
		if(lane < T / 32) sWarp[lane] = xi - x;
		if(lane == 31) sTotal = xi;
	}
	__syncthreads();
	const uint32_t total = sTotal;
	uint32_t pos = sWarp[warp] + incl - n;
	if(total <= SERVE_IDS_SMEM) {
#pragma unroll
		for(uint32_t j = 0; j < WREG; ++j) {
			uint32_t bits = wr[j];
			while(bits) {
				const uint32_t b = __ffs(bits) - 1;
				bits &= bits - 1;
				sIds[pos++] = (w0 + j) * 32 + b;
			}
		}
		for(uint32_t w = w0 + WREG; w < w1; ++w) {
			uint32_t bits = __ldcg(words + w);
			while(bits) {
				const uint32_t b = __ffs(bits) - 1;
				bits &= bits - 1;
				sIds[pos++] = w * 32 + b;
			}
		}
		__syncthreads();
		if(S.l2gIdentity) {
			for(uint32_t i = t; i < total; i += T) host[i] = sIds[i];
		} else {
			for(uint32_t i = t; i < total; i += T) host[i] = __ldg(S.l2g + sIds[i]);
		}
		return total;
	}
	for(uint32_t w = w0; w < w1; ++w) {
		uint32_t bits = __ldcg(words + w);
		while(bits) {
			const uint32_t b = __ffs(bits) - 1;
			bits &= bits - 1;
			S.firedIds[pos++] = S.l2g[w * 32 + b];
		}
	}
	__syncthreads();
	copy_words_to_host(S.firedIds, host, total);
	return total;
}

// A CTA other than 0 waits for CTA 0's broadcast of request `want` (1) or
// of the end of the loop (0); gives up like a grid barrier.
__device__ __forceinline__ uint32_t wait_request(GridBarrier* gb, uint32_t want, uint32_t& ok, uint32_t limit)
{
	__shared__ uint32_t sCmd;
	if(threadIdx.x == 0) {
		uint32_t r = 0, polls = 0;
		for(;;) {
			const uint32_t v = ld_acquire(&gb->cmd);
			if(v == want) {
				r = 1;
				break;
			}
			if(v == (want | SERVE_STOP)) break;
			if(give_up(gb, polls, limit)) {
				atomicExch(&gb->error, 1u);
				ok = 0;
				break;
			}
			__nanosleep(20);
		}
		sCmd = r;
	}
	__syncthreads();
	return sCmd;
}

template<unsigned MAXT, unsigned MINB>
__global__ void __launch_bounds__(MAXT, MINB)
serve_kernel(const DevSim S, uint32_t P, unsigned long long cycle0, GridBarrier* gb, ServeCtl* ctl, uint32_t seq0,
		const uint32_t* stim, uint32_t* hostIds, unsigned long long idleNs)
{
	__shared__ CtaCounters sC;
	__shared__ uint32_t sTarget, sOk;
	if(threadIdx.x == 0) {
		sC = CtaCounters{ 0, 0, 0, 0, 0, 0, 0 };
		sTarget = 0;
		sOk = 1;
	}
	__syncthreads();
	__shared__ uint32_t sOp;
	uint32_t want = seq0;
	for(unsigned long long k = 0;; ++k, want = serve_next(want)) {
		const unsigned long long c = cycle0 + k;
		const uint32_t ring = (uint32_t) (c % S.R);
		// CTA 0 takes the request from the host and broadcasts it (the
		// other CTAs finished the last step at its final barrier)
		uint32_t op;
		if(blockIdx.x == 0) {
			if(threadIdx.x < 32) {
				// warp 0 reads the request line -- the two request words and
				// the inline stimulus -- in one 64-byte read per poll
				const uint32_t FULL = 0xffffffffu, lane = threadIdx.x;
				const unsigned long long* line = &ctl->req[0];
				op = 0;
				const unsigned long long t0 = global_ns();
				for(uint32_t polls = 0; polls < SERVE_POLL_LIMIT; ++polls) {
					const unsigned long long w = lane < 2 + SERVE_INLINE ? ld_relaxed_sys_u64(line + lane) : 0ull;
					const unsigned long long a = __shfl_sync(FULL, w, 0);
					const unsigned long long b = __shfl_sync(FULL, w, 1);
					bool got = (uint32_t) (a >> 32) == want && (uint32_t) (b >> 32) == want;
					const bool inl = got && ((uint32_t) a & SERVE_INLINE_FLAG) != 0u;
					const uint32_t count = (uint32_t) a & ~SERVE_INLINE_FLAG;
					const bool mine = inl && lane >= 2 && lane - 2 < count;
					if(inl) got = __all_sync(FULL, !mine || (uint32_t) (w >> 32) == want);
					if(got) {
						// the stimulus the host wrote before the request
						asm volatile("fence.acq_rel.sys;" ::: "memory");
						// an inline firing stimulus is applied here; the step's
						// first grid barrier orders it before the update reads it
						if(mine) {
							const uint32_t l = (uint32_t) w;
							atomicOr(&S.fstim[l >> 5], 1u << (l & 31));
						}
						if(lane == 0) {
							gb->nf = inl ? 0u : (uint32_t) a;
							gb->ni = (uint32_t) b;
							S.eventCount[ring] = 0;
						}
						op = 1;
						break;
					}
					uint32_t stop = 0;
					if(lane == 0) {
						stop = (uint32_t) (a >> 32) == (want | SERVE_STOP) || global_ns() - t0 > idleNs
								|| ((polls & 1023u) == 1023u && ld_acquire(&gb->error));
					}
					if(__shfl_sync(FULL, stop, 0)) break;
					__nanosleep(32);
				}
				__syncwarp();
				if(lane == 0) {
					st_release(&gb->cmd, op ? want : want | SERVE_STOP);
					sOp = op;
				}
			}
			__syncthreads();
			op = sOp;
		} else {
			op = wait_request(gb, want, sOk, S.waitLimit);
		}
		if(!op) return;
		const uint32_t nf = *(volatile uint32_t*) &gb->nf;
		const uint32_t ni = *(volatile uint32_t*) &gb->ni;
		if(!persistent_step(S, P, c, gb, sTarget, sOk, sC, nf + ni ? stim : nullptr, nf, ni, nullptr)) return;
		// CTA 0 answers: the step's fired ids and events (after the step's
		// final barrier every CTA's words and counts are in place)
		if(blockIdx.x == 0) {
			const uint32_t n = fired_ids_to_host(S, S.firedRing + (size_t) ring * S.W, hostIds);
			__syncthreads();
			if(threadIdx.x == 0) {
				ctl->fired = n;
				ctl->events = *(volatile unsigned long long*) &S.eventCount[ring];
				// a release at system scope: the host that sees done sees
				// every store the CTA made before the __syncthreads
				st_release_sys(&ctl->done, want);
			}
		}
	}
}

// The instances of the persistent loops for a block size
constexpr uint32_t RUN_THREADS_PAIR = 512;
static const void* run_kernel_for(uint32_t threads, bool trace)
{
	if(threads <= RUN_THREADS_PAIR) {
		return trace ? (const void*) run_kernel<true, RUN_THREADS_PAIR, 2> : (const void*) run_kernel<false, RUN_THREADS_PAIR, 2>;
	}
	return trace ? (const void*) run_kernel<true, RUN_THREADS, 1> : (const void*) run_kernel<false, RUN_THREADS, 1>;
}
static const void* serve_kernel_for(uint32_t threads)
{
	return threads <= RUN_THREADS_PAIR ? (const void*) serve_kernel<RUN_THREADS_PAIR, 2>
			: (const void*) serve_kernel<RUN_THREADS, 1>;
}

// applyStdp (src/nemo/ConnectivityMatrix.cpp:241-294): w' =
// updatedWeight(w, reward x acc) for every incoming plastic synapse of the
// touched targets (the only ones whose accumulator can be nonzero), written
// back to the forward matrix when it changed, and the accumulator cleared.
// ALL: every target, whatever its accumulator -- the first call, which also
// clamps weights that start outside their range.  Work items are (slice,
// 32 consecutive targets: one word of the touched bit-vector), slice-major;
// lanes whose target is untouched take an empty run (walking the word
// directly costs less than compacting the touched targets into a list
// first).  A warp flattens its 32 runs with a scan and
// finds each entry's run with a 5-step shuffle search.  The targets of the
// warp's item after next and the runs of its next item are loaded while an
// item is processed (at 5 CTAs of 256 threads per SM: 48 registers, no
// spills), so an item's two dependent prologue loads are off its path.
template<bool ALL>
__global__ void __launch_bounds__(STEP_THREADS, 5)
apply_kernel(const DevSim S, int32_t reward)
{
	const uint32_t FULL = 0xffffffffu;
	const uint32_t lane = threadIdx.x & 31;
	const uint32_t batches = S.W;  // words of 32 targets
	const unsigned long long items = (unsigned long long) batches * S.applySlices;
	const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
	// lane's target of item ii (N: none)
	auto target_of = [&](unsigned long long ii) -> uint32_t {
		if(ii >= items) return S.N;
		const uint32_t kk = (uint32_t) (ii / batches);
		const uint32_t w = (uint32_t) (ii - (unsigned long long) kk * batches);
		const uint32_t t = w * 32 + lane;
		if(t >= S.N) return S.N;
		if(ALL) return t;
		return (S.touchedBits[w] >> lane) & 1u ? t : S.N;
	};
	// lane's run of item ii for target t
	auto run_of = [&](unsigned long long ii, uint32_t t, unsigned long long& lo, uint32_t& len) {
		lo = 0;
		len = 0;
		if(ii < items && t < S.N) {
			const uint32_t kk = (uint32_t) (ii / batches);
			const uint32_t* run = S.rcmSlice + (size_t) kk * S.N + t;
			const uint32_t a = run[0];
			lo = S.rcmPtr[t] + a;
			len = run[S.N] - a;
		}
	};
	unsigned long long i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	unsigned long long nlo;
	uint32_t nlen;
	run_of(i, target_of(i), nlo, nlen);
	uint32_t tn = target_of(i + nw);
	for(; i < items; i += nw) {
		const unsigned long long lo = nlo;
		const uint32_t len = nlen;
		const uint32_t incl = warp_inclusive_scan(len);
		const uint32_t total = __shfl_sync(FULL, incl, 31);
		// the next items' targets and runs, loaded while this one is processed
		const uint32_t tnn = target_of(i + 2ull * nw);
		run_of(i + nw, tn, nlo, nlen);
		tn = tnn;
		for(uint32_t off = 0; off < total; off += 32 * APPLY_ILP) {
			unsigned long long e[APPLY_ILP];
			int32_t acc[APPLY_ILP];
			uint32_t fwd[APPLY_ILP];
			bool live[APPLY_ILP];
#pragma unroll
			for(uint32_t q = 0; q < APPLY_ILP; ++q) {
				const uint32_t x = off + lane + 32 * q;
				// the run holding flattened entry x: the first lane whose
				// inclusive sum exceeds x
				uint32_t r = 0;
#pragma unroll
				for(uint32_t step = 16; step; step >>= 1) {
					if(__shfl_sync(FULL, incl, r + step - 1) <= x) r += step;
				}
				const uint32_t before = __shfl_sync(FULL, incl - len, r);
				const unsigned long long rlo = __shfl_sync(FULL, lo, r);
				e[q] = rlo + (x - before);
				// the accumulator and the forward index load together
				acc[q] = x < total ? __ldcs(S.rcmAcc + e[q]) : 0;
				fwd[q] = x < total ? __ldcs(S.rcmFwd + e[q]) : 0u;
			}
#pragma unroll
			for(uint32_t q = 0; q < APPLY_ILP; ++q) live[q] = off + lane + 32 * q < total && (ALL || acc[q] != 0);
			int32_t w[APPLY_ILP];
#pragma unroll
			for(uint32_t q = 0; q < APPLY_ILP; ++q) w[q] = live[q] ? (int32_t) S.synW[fwd[q]] : 0;
#pragma unroll
			for(uint32_t q = 0; q < APPLY_ILP; ++q) {
				if(!live[q]) continue;
				const int32_t nw2 = stdp_updated_weight(S.sp, w[q], fx_mul_dev(reward, acc[q]));
				if(nw2 != w[q]) S.synW[fwd[q]] = (uint32_t) nw2;
				if(acc[q]) S.rcmAcc[e[q]] = 0;
			}
		}
	}
}

// The run table of applyStdp: rcmSlice[k][t] is the offset, within target
// t's incoming plastic synapses (sorted by forward index), of the first one
// whose forward index is at least k x sliceLen; row K is t's in-degree.
// One warp per target, one lane per slice boundary (a binary search).
__global__ void slice_table_kernel(uint32_t N, const unsigned long long* rcmPtr, const uint32_t* rcmFwd, uint32_t K,
		uint32_t sliceLen, uint32_t* table)
{
	const uint32_t lane = threadIdx.x & 31;
	const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
	for(uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < N; t += warps) {
		const unsigned long long b = rcmPtr[t];
		const uint32_t n = (uint32_t) (rcmPtr[t + 1] - b);
		for(uint32_t k = lane; k <= K; k += 32) {
			uint32_t v = n;
			if(k < K) {
				const unsigned long long bound = (unsigned long long) k * sliceLen;
				uint32_t l = 0, h = n;
				while(l < h) {
					const uint32_t m = (l + h) >> 1;
					if(rcmFwd[b + m] < bound) l = m + 1;
					else h = m;
				}
				v = l;
			}
			table[(size_t) k * N + t] = v;
		}
	}
}

// Firing and current stimulus (src/nemo/cpu/Simulation.cpp:141-171)
__global__ void stimulus_kernel(const DevSim S, const uint32_t* fidx, uint32_t nf,
		const uint32_t* iidx, const float* ival, uint32_t ni)
{
	uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i < nf) {
		uint32_t l = fidx[i];
		atomicOr(&S.fstim[l >> 5], 1u << (l & 31));
	}
	if(i < ni) S.curExt[iidx[i]] = ival[i];
}

// ---------------------------------------------------------------------------
// nemo_step without allocation (nemo_b200_step_no_alloc)
//
// For callers that must not allocate (a real-time loop that steps every
// millisecond, where a device allocation or free would synchronise the
// device; an application with a fixed memory budget), the stimulus is
// staged through fixed static buffers instead of the simulation's growable
// staging buffers: g_stimStage on the host and g_noAllocStim on each device,
// NEMO_B200_NO_ALLOC_STIMULUS_MAX words (256 KiB) each.  Nothing in them is
// read before this call writes it, so nothing needs clearing.  The buffers
// are shared by every simulation of the process: overlapping calls race.

static __device__ __align__(256) uint32_t g_noAllocStim[NEMO_B200_NO_ALLOC_STIMULUS_MAX];

namespace {
constexpr int NO_ALLOC_MAX_DEVICES = 64;
uint32_t* g_noAllocStimAddr[NO_ALLOC_MAX_DEVICES];  // device address of g_noAllocStim per device
uint32_t g_stimStage[NEMO_B200_NO_ALLOC_STIMULUS_MAX];
// current stimulus before deduplication: local index, value, order
uint32_t g_curIdx[NEMO_B200_NO_ALLOC_STIMULUS_MAX / 2];
float g_curVal[NEMO_B200_NO_ALLOC_STIMULUS_MAX / 2];
uint32_t g_curOrder[NEMO_B200_NO_ALLOC_STIMULUS_MAX / 2];
} // namespace

bool Simulation::findLocal(unsigned g, unsigned* l) const
{
	auto it = m_g2l[0].find(g);
	if(it == m_g2l[0].end()) return false;
	*l = it->second;
	return true;
}

nemo_status_t Simulation::stepNoAlloc(const unsigned* fstim, size_t nf, const unsigned* inidx, const float* icur,
		size_t ni, unsigned* fired, size_t cap, size_t* nfired) noexcept
{
	if(m_nets > 1) return NEMO_API_UNSUPPORTED;
	if(nf > NEMO_B200_NO_ALLOC_STIMULUS_MAX || ni > NEMO_B200_NO_ALLOC_STIMULUS_MAX / 2
			|| nf + 2 * ni > NEMO_B200_NO_ALLOC_STIMULUS_MAX) {
		return NEMO_BUFFER_OVERFLOW;
	}
	if(cudaSetDevice(m_device) != cudaSuccess) return NEMO_CUDA_ERROR;
	if(m_device < 0 || m_device >= NO_ALLOC_MAX_DEVICES) return NEMO_API_UNSUPPORTED;
	stopServe();
	uint32_t*& stim = g_noAllocStimAddr[m_device];
	if(!stim) {
		// once per device, with the device current
		void* p = nullptr;
		if(cudaGetSymbolAddress(&p, g_noAllocStim) != cudaSuccess || !p) return NEMO_CUDA_ERROR;
		stim = static_cast<uint32_t*>(p);
	}
	// validate and map the stimulus before touching any state
	// (src/nemo/cpu/Simulation.cpp:141-163)
	for(size_t i = 0; i < nf; ++i) {
		unsigned l;
		if(!findLocal(fstim[i], &l)) return NEMO_INVALID_INPUT;
		g_stimStage[i] = l;
	}
	for(size_t i = 0; i < ni; ++i) {
		unsigned l;
		if(!findLocal(inidx[i], &l)) return NEMO_INVALID_INPUT;
		g_curIdx[i] = l;
		g_curVal[i] = icur[i];
		g_curOrder[i] = (uint32_t) i;
	}
	// the last current given for a neuron wins: order by (neuron, position)
	// in place and keep the last of each neuron's run
	std::sort(g_curOrder, g_curOrder + ni, [](uint32_t a, uint32_t b) {
		return g_curIdx[a] != g_curIdx[b] ? g_curIdx[a] < g_curIdx[b] : a < b;
	});
	size_t nu = 0;
	for(size_t k = 0; k < ni; ++k) {
		if(k + 1 < ni && g_curIdx[g_curOrder[k + 1]] == g_curIdx[g_curOrder[k]]) continue;
		g_curOrder[nu++] = g_curOrder[k];
	}
	for(size_t k = 0; k < nu; ++k) {
		g_stimStage[nf + k] = g_curIdx[g_curOrder[k]];
		memcpy(&g_stimStage[nf + nu + k], &g_curVal[g_curOrder[k]], 4);
	}
	const size_t words = nf + 2 * nu;
	if(words) {
		// the previous call's kernels read the device buffer: it finished
		// before that call returned (it synchronised the stream)
		if(cudaMemcpyAsync(stim, g_stimStage, words * 4, cudaMemcpyHostToDevice, m_stream) != cudaSuccess) {
			return NEMO_CUDA_ERROR;
		}
		const uint32_t nmax = (uint32_t) std::max(nf, nu);
		stimulus_kernel<<<(nmax + 255) / 256, 256, 0, m_stream>>>(m_dev, stim, (uint32_t) nf, stim + nf,
				reinterpret_cast<const float*>(stim + nf + nu), (uint32_t) nu);
	}
	const uint32_t ring = (uint32_t) (m_cycle % m_dev.R);
	launchStep(true);
	if(cudaMemcpyAsync(m_hFired, m_dev.firedRing + (size_t) ring * m_dev.W, (size_t) m_dev.W * 4,
			cudaMemcpyDeviceToHost, m_stream) != cudaSuccess) {
		return NEMO_CUDA_ERROR;
	}
	if(cudaStreamSynchronize(m_stream) != cudaSuccess || cudaGetLastError() != cudaSuccess) return NEMO_CUDA_ERROR;
	// a persistent or resident loop that ran before this call (the stream
	// synchronisation waited for it) and gave up at a wait has left the
	// simulation state undefined: report it as checkBarrier does, without
	// throwing or allocating (the word is read into pinned host memory)
	if(m_barrierUsed) {
		m_barrierUsed = false;
		if(cudaMemcpyAsync(m_hBarrierError, &m_barrier->error, 4, cudaMemcpyDeviceToHost, m_stream) != cudaSuccess
				|| cudaStreamSynchronize(m_stream) != cudaSuccess) {
			return NEMO_CUDA_ERROR;
		}
		if(*m_hBarrierError) {
			*m_hBarrierError = 0;
			cudaMemsetAsync(m_barrier, 0, sizeof(GridBarrier), m_stream);
			cudaStreamSynchronize(m_stream);
			m_barrierBase = 0;
			m_barrierStale = false;
			return NEMO_CUDA_ERROR;
		}
	}
	// fired neurons in ascending local index, as global ids
	// (setFiring, src/nemo/cpu/Simulation.cpp:200-208)
	size_t count = 0;
	for(uint32_t w = 0; w < m_dev.W; ++w) {
		uint32_t bits = m_hFired[w];
		while(bits) {
			const uint32_t l = w * 32 + (uint32_t) __builtin_ctz(bits);
			bits &= bits - 1;
			if(count < cap) fired[count] = m_l2g[l];
			++count;
			stepEvents += m_outDegree[l];
		}
	}
	*nfired = count;
	return count > cap ? NEMO_BUFFER_OVERFLOW : NEMO_OK;
}

// ---------------------------------------------------------------------------
// libm calibration tables on the device

LibmCalib device_calibration(int device)
{
	static std::mutex mtx;
	static std::unordered_map<int, LibmCalib> cache;
	std::lock_guard<std::mutex> lock(mtx);
	auto it = cache.find(device);
	if(it != cache.end()) return it->second;
	const CalibTables& t = libm_calibration();
	uint32_t *dLog, *dSin, *dKey, *dVal;
	size_t nexc = t.excKey.size();
	NB_CUDA(cudaMalloc(&dLog, t.logFlip.size() * 4));
	NB_CUDA(cudaMalloc(&dSin, t.sinFlip.size() * 4));
	NB_CUDA(cudaMalloc(&dKey, (nexc + 1) * 4));
	NB_CUDA(cudaMalloc(&dVal, (nexc + 1) * 4));
	NB_CUDA(cudaMemcpy(dLog, t.logFlip.data(), t.logFlip.size() * 4, cudaMemcpyHostToDevice));
	NB_CUDA(cudaMemcpy(dSin, t.sinFlip.data(), t.sinFlip.size() * 4, cudaMemcpyHostToDevice));
	if(nexc) {
		NB_CUDA(cudaMemcpy(dKey, t.excKey.data(), nexc * 4, cudaMemcpyHostToDevice));
		NB_CUDA(cudaMemcpy(dVal, t.excVal.data(), nexc * 4, cudaMemcpyHostToDevice));
	}
	// the host libm's results at every reachable argument (67 MB + 336 MB)
	float *dLogVal, *dSinVal;
	NB_CUDA(cudaMalloc(&dLogVal, t.logVal.size() * 4));
	NB_CUDA(cudaMalloc(&dSinVal, t.sinVal.size() * 4));
	NB_CUDA(cudaMemcpy(dLogVal, t.logVal.data(), t.logVal.size() * 4, cudaMemcpyHostToDevice));
	NB_CUDA(cudaMemcpy(dSinVal, t.sinVal.data(), t.sinVal.size() * 4, cudaMemcpyHostToDevice));
	LibmCalib c;
	c.logFlip = dLog;
	c.sinFlip = dSin;
	c.excKey = dKey;
	c.excVal = dVal;
	c.nexc = (uint32_t) nexc;
	c.logNear = t.logNear;
	c.sinNear = t.sinNear;
	c.logVal = dLogVal;
	c.sinVal = dSinVal;
	cache[device] = c;
	return c;
}

// ---------------------------------------------------------------------------
// host side

template<typename T>
T* Simulation::dalloc(size_t n)
{
	void* p = nullptr;
	cudaError_t err = cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T));
	if(err != cudaSuccess) {
		NB_THROW(NEMO_CUDA_MEMORY_ERROR, "failed to allocate %zu bytes of device memory: %s",
				n * sizeof(T), cudaGetErrorString(err));
	}
	m_allocs.push_back(p);
	NB_CUDA(cudaMemsetAsync(p, 0, std::max<size_t>(n, 1) * sizeof(T), m_stream));
	return static_cast<T*>(p);
}

static void seed_rng(std::vector<uint32_t>& planes, unsigned N)
{
	// src/nemo/RNG.cpp:38-63: the neuron with local index l takes draws
	// [4l, 4l + 4) of one default-seeded mt19937 stream, each mapped by
	// uniform_int<unsigned long>(0, 0x7fffffff), i.e. x >> 1.
	planes.assign(4 * (size_t) N, 0);
	uint32_t mt[624];
	mt[0] = 5489u;
	for(int i = 1; i < 624; ++i) mt[i] = 1812433253u * (mt[i - 1] ^ (mt[i - 1] >> 30)) + (uint32_t) i;
	int idx = 624;
	auto next = [&]() {
		if(idx >= 624) {
			for(int k = 0; k < 624; ++k) {
				uint32_t y = (mt[k] & 0x80000000u) | (mt[(k + 1) % 624] & 0x7fffffffu);
				mt[k] = mt[(k + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
			}
			idx = 0;
		}
		uint32_t y = mt[idx++];
		y ^= (y >> 11);
		y ^= (y << 7) & 0x9d2c5680u;
		y ^= (y << 15) & 0xefc60000u;
		y ^= (y >> 18);
		return y;
	};
	for(unsigned l = 0; l < N; ++l) {
		for(unsigned p = 0; p < 4; ++p) planes[(size_t) p * N + l] = next() >> 1;
	}
	// planes[p * N + l] is word p of the neuron with local index l
}

static inline uint64_t shl64(uint64_t x, unsigned s) { return x << (s & 63); }

// cpu_init_neurons of the Kuramoto plugin (src/nemo/cpu/plugins/
// Kuramoto.cpp:131-151): the 31 phases before cycle 0, run backwards without
// coupling, into the slots (0 - k) % 32 of state [32][n] (frequency [n]);
// the host's float arithmetic is the plugin's (no contraction).
static void init_kuramoto_history(const float* frequency, float* state, unsigned n)
{
	const unsigned H = 32;
	for(unsigned k = 0; k < H - 1; k++) {
		const unsigned current = 0U - k, previous = 0U - (k + 1U);
		const float* phase0 = state + (size_t) (current % H) * n;
		float* phase1 = state + (size_t) (previous % H) * n;
		for(unsigned i = 0; i < n; i++) {
			const float phase = phase0[i] - frequency[i];
			phase1[i] = (float) ((double) fmodf(phase, (float) (2.0f * M_PI)) + (phase < 0.0f ? 2.0f * M_PI : 0.0f));
		}
	}
}

Simulation::Simulation(const Network& net, const Configuration& conf) :
	Simulation(std::vector<const Network*>{ &net }, conf)
{
}

// Builds the device layout of one network or, for a batch, of several
// independent networks simulated as one: their neurons share the neuron
// arrays (grouped by neuron kind, so that the step kernel sees at most one
// range per kind), their synapses never cross networks, and each network's
// RNG streams and fire stream are those of its own single-network run.
Simulation::Simulation(const std::vector<const Network*>& nets, const Configuration& conf)
{
	// a constructor that throws runs no destructor: free what was made
	try {
		init(nets, conf);
	} catch(...) {
		releaseAll();
		throw;
	}
}

void Simulation::init(const std::vector<const Network*>& nets, const Configuration& conf)
{
	if(nets.empty()) NB_THROW(NEMO_INVALID_INPUT, "no network");
	const bool batch = nets.size() > 1;
	// checks in the order of nemo::simulationBackend (src/nemo/nemo.cpp:109-134)
	// and the backend constructor (src/nemo/cpu/Simulation.cpp:36-82)
	size_t totalN = 0;
	unsigned maxDelay = 0;
	for(const Network* np : nets) {
		const Network& net = *np;
		unsigned n = net.neuronCount();
		if(n == 0) NB_THROW(NEMO_INVALID_INPUT, "Cannot create simulation from empty network");
		if(conf.stdp && net.maxDelay + conf.postfire.size() > MAX_HISTORY) {
			NB_THROW(NEMO_INVALID_INPUT, "Max delay + postfire part of STDP function must be <= %u", MAX_HISTORY);
		}
		if(conf.backend != NEMO_BACKEND_CUDA) {
			NB_THROW(NEMO_API_UNSUPPORTED, "This library provides only the B200 CUDA backend; the CPU backend is not part of it");
		}
		if(net.maxDelay > 64) {
			NB_THROW(NEMO_INVALID_INPUT, "The network has synapses with delay %ums. The B200 backend supports a maximum of 64 ms", net.maxDelay);
		}
		if(batch && net.maxDelay == 64) {
			NB_THROW(NEMO_API_UNSUPPORTED, "A batched network may not have a maximum delay of exactly 64 ms");
		}
		if(net.duplicate) NB_THROW(NEMO_INVALID_INPUT, "Duplicate neuron index %u", net.duplicateIdx);
		// each type's kernel (where the reference loads the type's CUDA
		// plugin, src/nemo/cuda/Neurons.cpp:43)
		for(const NeuronCollection& c : net.types) {
			if(c.size()) checkKernelBinding(*c.desc);
		}
		totalN += n;
		maxDelay = std::max(maxDelay, net.maxDelay);
	}
	if(totalN >= MAX_NEURONS) NB_THROW(NEMO_API_UNSUPPORTED, "The B200 backend supports at most %u neurons", MAX_NEURONS - 1);
	const unsigned N = (unsigned) totalN;

	int ndev = 0;
	NB_CUDA(cudaGetDeviceCount(&ndev));
	if(ndev == 0) NB_THROW(NEMO_CUDA_ERROR, "No CUDA device available");
	if(conf.device >= 0) {
		if(conf.device >= ndev) NB_THROW(NEMO_INVALID_INPUT, "Invalid CUDA device %d", conf.device);
		m_device = conf.device;
	} else {
		NB_CUDA(cudaGetDevice(&m_device));
	}
	NB_CUDA(cudaSetDevice(m_device));
	NB_CUDA(cudaStreamCreateWithFlags(&m_stream, cudaStreamNonBlocking));
	NB_CUDA(cudaEventCreate(&m_ev0));
	NB_CUDA(cudaEventCreate(&m_ev1));

	m_N = N;
	m_nets = (unsigned) nets.size();
	m_maxDelay = maxDelay;
	m_writeOnly = conf.writeOnlySynapses || batch;
	memset(&m_dev, 0, sizeof m_dev);
	DevSim& S = m_dev;
	S.N = N;
	S.W = (N + 31) / 32;
	S.waitLimit = BARRIER_SPIN_LIMIT;

	// neuron layout: kinds in order of first appearance (for one network this
	// is its type order, src/nemo/cpu/Simulation.cpp:58-73), then network
	// order, then insertion order
	std::vector<NeuronKind> kinds;
	for(const Network* np : nets) {
		for(const NeuronCollection& c : np->types) {
			if(c.size() && std::find(kinds.begin(), kinds.end(), c.desc->kind) == kinds.end()) kinds.push_back(c.desc->kind);
		}
	}
	if(kinds.size() > MAX_TYPES) NB_THROW(NEMO_API_UNSUPPORTED, "At most %u neuron types", MAX_TYPES);
	m_l2g.resize(N);
	m_ltype.resize(N);
	m_netLocal.resize(N);
	if(batch) m_netOf.resize(N);
	m_g2l.assign(nets.size(), std::unordered_map<unsigned, unsigned>());
	for(size_t i = 0; i < nets.size(); ++i) m_g2l[i].reserve(nets[i]->neuronCount() * 2);
	m_netTypes.assign(nets.size(), std::vector<NetTypeRange>());
	// network-local index of the first neuron of each type, per network
	std::vector<std::vector<unsigned>> localBase(nets.size());
	for(size_t i = 0; i < nets.size(); ++i) {
		unsigned b = 0;
		for(const NeuronCollection& c : nets[i]->types) {
			localBase[i].push_back(b);
			b += (unsigned) c.size();
		}
		m_netTypes[i].resize(nets[i]->types.size());
	}
	unsigned l = 0;
	bool needCalib = false;
	for(NeuronKind kind : kinds) {
		HostType ht;
		for(const Network* np : nets) {
			for(const NeuronCollection& c : np->types) {
				if(c.size() && c.desc->kind == kind) {
					ht.desc = *c.desc;
					break;
				}
			}
			if(ht.desc.kind == kind) break;
		}
		ht.netType = 0;
		ht.base = l;
		ht.n = 0;
		for(size_t i = 0; i < nets.size(); ++i) {
			for(size_t t = 0; t < nets[i]->types.size(); ++t) {
				if(nets[i]->types[t].desc->kind == kind) ht.n += (unsigned) nets[i]->types[t].size();
			}
		}
		const unsigned np = ht.desc.nparam, ns = ht.desc.nstate, na = np + ns;
		// state [history][nstate][n]: the given state in slot 0, the slot of cycle 0
		std::vector<float> param((size_t) np * ht.n), state((size_t) ht.desc.history * ns * ht.n);
		unsigned i0 = 0;
		for(size_t i = 0; i < nets.size(); ++i) {
			for(size_t t = 0; t < nets[i]->types.size(); ++t) {
				const NeuronCollection& c = nets[i]->types[t];
				if(c.desc->kind != kind || c.size() == 0) continue;
				if(!batch) ht.netType = (unsigned) t;
				m_netTypes[i][t] = NetTypeRange{ (unsigned) m_types.size(), i0, (unsigned) c.size() };
				for(size_t j = 0; j < c.size(); ++j) {
					const unsigned li = i0 + (unsigned) j;
					for(unsigned p = 0; p < np; ++p) param[(size_t) p * ht.n + li] = c.args[j * na + p];
					for(unsigned v = 0; v < ns; ++v) state[(size_t) v * ht.n + li] = c.args[j * na + np + v];
					const unsigned u = l + li;
					m_l2g[u] = c.gidx[j];
					m_ltype[u] = (uint8_t) m_types.size();
					m_netLocal[u] = localBase[i][t] + (unsigned) j;
					if(batch) m_netOf[u] = (uint32_t) i;
					if(!m_g2l[i].emplace(c.gidx[j], u).second) {
						NB_THROW(NEMO_INVALID_INPUT, "Duplicate neuron index %u", c.gidx[j]);
					}
				}
				i0 += (unsigned) c.size();
			}
		}
		if(kind == KIND_KURAMOTO) init_kuramoto_history(param.data(), state.data(), ht.n);
		ht.dParam = dalloc<float>(param.size());
		ht.dState = dalloc<float>(state.size());
		NB_CUDA(cudaMemcpyAsync(ht.dParam, param.data(), param.size() * 4, cudaMemcpyHostToDevice, m_stream));
		NB_CUDA(cudaMemcpyAsync(ht.dState, state.data(), state.size() * 4, cudaMemcpyHostToDevice, m_stream));
		if(kind == KIND_IZHIKEVICH) needCalib = true;
		TypeRange& tr = S.types[m_types.size()];
		tr.kind = kind;
		tr.base = ht.base;
		tr.n = ht.n;
		tr.param = ht.dParam;
		tr.state = ht.dState;
		tr.history = ht.desc.history;
		m_types.push_back(ht);
		l += ht.n;
		NB_CUDA(cudaStreamSynchronize(m_stream)); // host vectors go out of scope
	}
	S.ntypes = (uint32_t) m_types.size();

	// synapses: the forward matrix, its delay groups and, with STDP, the
	// reverse matrix of plastic synapses, built on the device where the
	// network allows it and on the host otherwise (both give the same bytes)
	size_t Sn = 0;
	for(const Network* np : nets) Sn += np->src.size();
	m_nsyn = Sn;
	const unsigned D = std::max(1u, m_maxDelay);
	S.dStride = D;
	// deliverSpikes' validSpikes = ~(~0 << maxDelay) with x86 shift
	// semantics (src/nemo/cpu/Simulation.cpp:263): nothing is delivered when
	// the maximum delay is 0 or 64
	const bool deliver = m_maxDelay >= 1 && m_maxDelay <= 63;
	std::vector<unsigned long long> outPtr(N + 1), rcmPtr(N + 1, 0);
	uint64_t dlvGroups = 0;  // delay groups of all sources (all pending at once, at most)
	bool needAll = false;  // a type reads the reverse matrix of all synapses
	for(const HostType& t : m_types) {
		needAll |= t.desc.rcmSources || t.desc.rcmDelays || t.desc.rcmForward || t.desc.rcmWeights;
	}
	S.stdp = conf.stdp ? 1 : 0;

	std::vector<DevicePart> parts;
	if(conf.deviceConstruction && !needAll && planDeviceBuild(nets, conf.stdp, parts)) {
		buildOnDevice(nets, parts, deliver, outPtr, rcmPtr, dlvGroups);
	} else {
		// synapses of all networks, each mapped through its own network's ids
		hvector<unsigned> lsrc(Sn), ltgt(Sn), sdelay(Sn);
		hvector<int32_t> fxw(Sn);
		hvector<uint8_t> splastic(Sn);
		{
			size_t k = 0;
			for(size_t i = 0; i < nets.size(); ++i) {
				const Network& net = *nets[i];
				const auto& g2l = m_g2l[i];
				for(size_t q = 0; q < net.src.size(); ++q, ++k) {
					auto is = g2l.find(net.src[q]);
					if(is == g2l.end()) NB_THROW(NEMO_INVALID_INPUT, "Non-existing neuron index %u", net.src[q]);
					auto it = g2l.find(net.tgt[q]);
					if(it == g2l.end()) NB_THROW(NEMO_INVALID_INPUT, "Non-existing neuron index %u", net.tgt[q]);
					lsrc[k] = is->second;
					ltgt[k] = it->second;
					fxw[k] = fx_toFix(net.weight[q]);
					sdelay[k] = net.delay[q];
					splastic[k] = net.plastic[q];
				}
			}
		}

		// the reverse matrix of all synapses, for a type that reads its sources
		// (construction/RCM.cpp:58-99 and 150-172 with STDP off); it cannot
		// coexist with STDP's (:90-98)
		{
			if(needAll && conf.stdp) {
				NB_THROW(NEMO_API_UNSUPPORTED, "The current version does not support a mix of STDP with neuron types "
						"which require reverse connectivity for other purposes");
			}
			std::vector<unsigned long long> allPtr(N + 1, 0);
			if(needAll) {
				for(size_t k = 0; k < Sn; ++k) allPtr[ltgt[k] + 1]++;
				for(unsigned t = 0; t < N; ++t) allPtr[t + 1] += allPtr[t];
				hvector<uint32_t> asrc(Sn);
				hvector<float> aw(Sn);
				std::vector<unsigned long long> fill(allPtr.begin(), allPtr.end() - 1);
				size_t k = 0;
				for(const Network* np : nets) {
					for(size_t q = 0; q < np->src.size(); ++q, ++k) {
						// a Kuramoto neuron reads its sources' phases from its own
						// type's history of 32 steps
						const HostType& tt = m_types[m_ltype[ltgt[k]]];
						if(tt.desc.kind == KIND_KURAMOTO) {
							if(m_ltype[lsrc[k]] != m_ltype[ltgt[k]]) {
								NB_THROW(NEMO_INVALID_INPUT, "Synapse %u -> %u: a Kuramoto oscillator's sources must be "
										"Kuramoto oscillators", np->src[q], np->tgt[q]);
							}
							if(sdelay[k] > 31) {
								NB_THROW(NEMO_INVALID_INPUT, "Synapse %u -> %u: delay %u beyond the 31 steps of phase "
										"history a Kuramoto oscillator reads", np->src[q], np->tgt[q], sdelay[k]);
							}
						}
						const unsigned long long p = fill[ltgt[k]]++;
						asrc[p] = lsrc[k] | ((sdelay[k] - 1) << 26);
						aw[p] = np->weight[q];
					}
				}
				auto* dSrc = dalloc<uint32_t>(Sn);
				auto* dW = dalloc<float>(Sn);
				NB_CUDA(cudaMemcpyAsync(dSrc, asrc.data(), Sn * 4, cudaMemcpyHostToDevice, m_stream));
				NB_CUDA(cudaMemcpyAsync(dW, aw.data(), Sn * 4, cudaMemcpyHostToDevice, m_stream));
				S.allSrc = dSrc;
				S.allW = dW;
			}
			auto* dPtr = dalloc<unsigned long long>(N + 1);
			NB_CUDA(cudaMemcpyAsync(dPtr, allPtr.data(), (N + 1) * 8, cudaMemcpyHostToDevice, m_stream));
			S.allPtr = dPtr;
			NB_CUDA(cudaStreamSynchronize(m_stream));
		}

		// forward matrix (src/nemo/ConnectivityMatrix.cpp:65-162): outgoing
		// synapses per local source, sorted by delay, insertion order within a
		// delay -- the reference's row order
		hvector<uint64_t> pos(Sn);
		std::vector<uint64_t> delayMask(N, 0);
		{
			hvector<uint64_t> rowStart((size_t) N * D + 1, 0);
			for(size_t k = 0; k < Sn; ++k) rowStart[(size_t) lsrc[k] * D + sdelay[k]]++;
			for(size_t r = 0; r < (size_t) N * D; ++r) rowStart[r + 1] += rowStart[r];
			for(unsigned s = 0; s <= N; ++s) outPtr[s] = rowStart[(size_t) s * D];
			m_outDegree.resize(N);
			for(unsigned s = 0; s < N; ++s) {
				m_outDegree[s] = (uint32_t) (outPtr[s + 1] - outPtr[s]);
				m_maxOutDeg = std::max(m_maxOutDeg, m_outDegree[s]);
			}
			// delay groups: the end of each source's delay-d group within its row
			const bool narrow = m_maxOutDeg < 65536;
			hvector<uint16_t> end16(narrow ? (size_t) N * D : 0);
			hvector<uint32_t> end32(narrow ? 0 : (size_t) N * D);
			for(unsigned s = 0; s < N; ++s) {
				const uint64_t base = rowStart[(size_t) s * D];
				uint64_t prev = 0;
				for(unsigned d = 1; d <= D; ++d) {
					const uint64_t e = rowStart[(size_t) s * D + d] - base;
					if(narrow) end16[(size_t) s * D + d - 1] = (uint16_t) e;
					else end32[(size_t) s * D + d - 1] = (uint32_t) e;
					if(deliver && e > prev) {
						delayMask[s] |= 1ull << (d - 1);
						++dlvGroups;
					}
					prev = e;
				}
			}
			if(narrow) {
				auto* p = dalloc<uint16_t>(end16.size());
				NB_CUDA(cudaMemcpyAsync(p, end16.data(), end16.size() * 2, cudaMemcpyHostToDevice, m_stream));
				S.dEnd16 = p;
				S.dEnd32 = nullptr;
			} else {
				auto* p = dalloc<uint32_t>(end32.size());
				NB_CUDA(cudaMemcpyAsync(p, end32.data(), end32.size() * 4, cudaMemcpyHostToDevice, m_stream));
				S.dEnd16 = nullptr;
				S.dEnd32 = p;
			}
			auto* dm = dalloc<uint64_t>(N);
			NB_CUDA(cudaMemcpyAsync(dm, delayMask.data(), (size_t) N * 8, cudaMemcpyHostToDevice, m_stream));
			S.delayMask = dm;
			NB_CUDA(cudaStreamSynchronize(m_stream)); // the host tables go out of scope
			for(size_t k = 0; k < Sn; ++k) pos[k] = rowStart[(size_t) lsrc[k] * D + sdelay[k] - 1]++;
		}
		{
			hvector<uint32_t> synTgt(Sn), synW(Sn);
			for(size_t k = 0; k < Sn; ++k) {
				synTgt[pos[k]] = ltgt[k] | ((sdelay[k] - 1) << 26);
				synW[pos[k]] = (uint32_t) fxw[k];
			}
			auto* dOut = dalloc<unsigned long long>(N + 1);
			auto* dTgt = dalloc<uint32_t>(Sn);
			auto* dW = dalloc<uint32_t>(Sn);
			NB_CUDA(cudaMemcpyAsync(dOut, outPtr.data(), (N + 1) * 8, cudaMemcpyHostToDevice, m_stream));
			NB_CUDA(cudaMemcpyAsync(dTgt, synTgt.data(), Sn * 4, cudaMemcpyHostToDevice, m_stream));
			NB_CUDA(cudaMemcpyAsync(dW, synW.data(), Sn * 4, cudaMemcpyHostToDevice, m_stream));
			S.outPtr = dOut;
			S.synTgt = dTgt;
			S.synW = dW;
			NB_CUDA(cudaStreamSynchronize(m_stream));
		}

		// query tables of one network: per local source, its synapses by
		// per-source index
		if(!m_writeOnly) {
			const Network& net = *nets[0];
			m_srcStart.assign(N + 1, 0);
			for(size_t k = 0; k < Sn; ++k) m_srcStart[lsrc[k] + 1]++;
			for(unsigned s = 0; s < N; ++s) m_srcStart[s + 1] += m_srcStart[s];
			m_srcOrder.resize(Sn);
			for(size_t k = 0; k < Sn; ++k) m_srcOrder[m_srcStart[lsrc[k]] + net.sid[k]] = k;
			m_pos.assign(pos.begin(), pos.end());
			m_synDelay.assign(net.delay.begin(), net.delay.end());
			m_synPlastic.assign(net.plastic.begin(), net.plastic.end());
			m_synTarget.assign(net.tgt.begin(), net.tgt.end());
		}

		// the reverse matrix of plastic synapses (src/nemo/construction/RCM.cpp:150-172),
		// each target's synapses in forward-matrix order
		if(conf.stdp) {
			if(Sn > 0xffffffffull) NB_THROW(NEMO_API_UNSUPPORTED, "too many synapses for STDP");
			for(size_t k = 0; k < Sn; ++k) if(splastic[k]) rcmPtr[ltgt[k] + 1]++;
			for(unsigned t = 0; t < N; ++t) {
				m_maxPlasticInDeg = std::max(m_maxPlasticInDeg, (uint32_t) rcmPtr[t + 1]);
				rcmPtr[t + 1] += rcmPtr[t];
			}
			size_t P = rcmPtr[N];
			hvector<uint32_t> rsrc(P), rfwd(P), kAt(Sn);
			for(size_t k = 0; k < Sn; ++k) kAt[pos[k]] = (uint32_t) k;
			std::vector<unsigned long long> fill(rcmPtr.begin(), rcmPtr.end() - 1);
			for(size_t p = 0; p < Sn; ++p) {
				const uint32_t k = kAt[p];
				if(!splastic[k]) continue;
				const size_t q = fill[ltgt[k]]++;
				rsrc[q] = lsrc[k] | ((sdelay[k] - 1) << 26);
				rfwd[q] = (uint32_t) p;
			}
			auto* dRsrc = dalloc<uint32_t>(P);
			auto* dRfwd = dalloc<uint32_t>(P);
			S.rcmAcc = dalloc<int32_t>(P);
			NB_CUDA(cudaMemcpyAsync(dRsrc, rsrc.data(), P * 4, cudaMemcpyHostToDevice, m_stream));
			NB_CUDA(cudaMemcpyAsync(dRfwd, rfwd.data(), P * 4, cudaMemcpyHostToDevice, m_stream));
			S.rcmSrc = dRsrc;
			S.rcmFwd = dRfwd;
			lastPlastic = P;
			NB_CUDA(cudaStreamSynchronize(m_stream));
		}
	}
	// the STDP function (src/nemo/StdpProcess.cpp:20-46)
	if(conf.stdp) {
		StdpParams& sp = S.sp;
		sp.npre = (uint32_t) conf.prefire.size();
		sp.npost = (uint32_t) conf.postfire.size();
		for(unsigned i = 0; i < sp.npre; ++i) sp.fnPre[i] = fx_toFix(conf.prefire[i]);
		for(unsigned i = 0; i < sp.npost; ++i) sp.fnPost[i] = fx_toFix(conf.postfire[i]);
		sp.minE = fx_toFix(conf.minE);
		sp.maxE = fx_toFix(conf.maxE);
		sp.minI = fx_toFix(conf.minI);
		sp.maxI = fx_toFix(conf.maxI);
		// StdpFunction::getBits (src/nemo/StdpFunction.cpp:72-90)
		uint64_t pot = 0, dep = 0;
		unsigned b = 0;
		for(unsigned i = sp.npost; i-- > 0; ++b) {
			if(conf.postfire[i] > 0.0f) pot |= 1ull << b;
			if(conf.postfire[i] < 0.0f) dep |= 1ull << b;
		}
		for(unsigned i = 0; i < sp.npre; ++i, ++b) {
			if(conf.prefire[i] > 0.0f) pot |= 1ull << b;
			if(conf.prefire[i] < 0.0f) dep |= 1ull << b;
		}
		sp.potBits = pot;
		sp.depBits = dep;
		sp.prePostBits = shl64(~shl64(~0ull, sp.npre), sp.npost);
		sp.postPreBits = ~shl64(~0ull, sp.npost);
		sp.postFireMask = shl64(1ull, sp.npost);
	}

	auto* dRcmPtr = dalloc<unsigned long long>(N + 1);
	NB_CUDA(cudaMemcpyAsync(dRcmPtr, rcmPtr.data(), (N + 1) * 8, cudaMemcpyHostToDevice, m_stream));
	S.rcmPtr = dRcmPtr;
	// work lists: room for every delay group of every source pending and
	// every neuron being an STDP target in the same step (entries are
	// counted in 32 bits)
	{
		const uint64_t plastic = rcmPtr[N];
		if(Sn >= (1ull << 32) || plastic >= (1ull << 32) || dlvGroups >= (1ull << 32)) {
			NB_THROW(NEMO_API_UNSUPPORTED, "network too large for the work lists");
		}
		auto makeList = [&](WorkList& L, uint64_t groups, uint64_t entries) {
			L.group = dalloc<uint4>(groups);
			L.count = dalloc<unsigned long long>(2);
			L.bucket = dalloc<uint32_t>(entries / BUCKET + 1);
		};
		makeList(S.dlvWork, dlvGroups, Sn);
		m_dlvGroups = dlvGroups;
		makeList(S.stdpWork, N, plastic);
	}
	// applyStdp's slices of the forward matrix and each target's run in each
	if(conf.stdp) {
		const uint32_t K = (uint32_t) std::min<uint64_t>(APPLY_MAX_SLICES,
				std::max<uint64_t>(1, (Sn + APPLY_SLICE_ENTRIES - 1) / APPLY_SLICE_ENTRIES));
		S.applySlices = K;
		S.sliceLen = (uint32_t) std::max<uint64_t>(1, (Sn + K - 1) / K);
		auto* table = dalloc<uint32_t>((size_t) (K + 1) * N);
		const unsigned grid = std::max(1u, std::min<unsigned>((N + 7) / 8, 148u * 16u));
		slice_table_kernel<<<grid, 256, 0, m_stream>>>(N, S.rcmPtr, S.rcmFwd, K, S.sliceLen, table);
		NB_CUDA(cudaGetLastError());
		S.rcmSlice = table;
		NB_CUDA(cudaStreamSynchronize(m_stream));
	}

	// per-neuron RNG, keyed by the network-local index
	// (src/nemo/cpu/Neurons.cpp:41)
	{
		unsigned maxLocal = 0;
		for(const Network* np : nets) maxLocal = std::max(maxLocal, np->neuronCount());
		std::vector<uint32_t> stream;
		seed_rng(stream, maxLocal);
		std::vector<uint32_t> planes(4 * (size_t) N);
		for(unsigned u = 0; u < N; ++u) {
			for(unsigned p = 0; p < 4; ++p) planes[(size_t) p * N + u] = stream[(size_t) p * maxLocal + m_netLocal[u]];
		}
		S.rng = dalloc<uint32_t>(4 * (size_t) N);
		NB_CUDA(cudaMemcpyAsync(S.rng, planes.data(), planes.size() * 4, cudaMemcpyHostToDevice, m_stream));
		NB_CUDA(cudaStreamSynchronize(m_stream));
	}

	S.hist = dalloc<uint64_t>(2 * (size_t) N);
	S.noise = dalloc<float>(N);
	S.recentWords = (S.W + 3) & ~3u;  // 16-byte rows for the asynchronous copy
	S.recent = dalloc<uint32_t>(2 * (size_t) S.recentWords);
	S.recentBytes = (S.stdp && (size_t) S.recentWords * 4 <= RECENT_FILTER_MAX_BYTES) ? S.recentWords * 4 : 0u;
	S.fstim = dalloc<uint32_t>(S.W);
	S.touchedBits = dalloc<uint32_t>(S.W);
	S.curExt = dalloc<float>(N);
	S.slot = dalloc<ulonglong2>(N);
	S.l2g = dalloc<uint32_t>(N);
	NB_CUDA(cudaMemcpy(S.l2g, m_l2g.data(), (size_t) N * 4, cudaMemcpyHostToDevice));
	S.l2gIdentity = 1;
	for(size_t i = 0; i < N; ++i) {
		if(m_l2g[i] != i) {
			S.l2gIdentity = 0;
			break;
		}
	}
	S.firedIds = dalloc<uint32_t>(N);
	S.cycleDev = dalloc<unsigned long long>(1);
	NB_CUDA(cudaMallocHost(&m_hCycle, 8));
	S.R = (uint32_t) std::max<size_t>(16, std::min<size_t>(1024, (64u << 20) / ((size_t) S.W * 4)));
	S.firedRing = dalloc<uint32_t>((size_t) S.R * S.W);
	S.firedCount = dalloc<uint32_t>(S.R);
	S.eventCount = dalloc<unsigned long long>(S.R);
	S.stdpCount = dalloc<unsigned long long>(S.R);
	NB_CUDA(cudaMallocHost(&m_hFired, (size_t) S.R * S.W * 4));
	NB_CUDA(cudaHostAlloc(&m_hFiredMapped, (size_t) S.W * 4, cudaHostAllocMapped));
	NB_CUDA(cudaHostGetDevicePointer(&m_dFiredMapped, m_hFiredMapped, 0));
	NB_CUDA(cudaHostAlloc(&m_hServe, sizeof(ServeCtl), cudaHostAllocMapped));
	memset(m_hServe, 0, sizeof(ServeCtl));
	NB_CUDA(cudaHostGetDevicePointer(&m_dServe, m_hServe, 0));
	NB_CUDA(cudaEventCreateWithFlags(&m_serveEnd, cudaEventDisableTiming));

	if(needCalib) S.calib = device_calibration(m_device);
	NB_CUDA(cudaDeviceGetAttribute(&m_sms, cudaDevAttrMultiProcessorCount, m_device));
	// the two-launch pre-phase: as many CTAs as fit on the GPU at once
	{
		int perSm = 0;
		NB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, deliver_kernel, STEP_THREADS, S.recentBytes));
		m_deliverGrid = (unsigned) std::max(1, perSm) * (unsigned) m_sms;
	}
	// applyStdp: as many CTAs as fit at once, so that the slice-major work
	// order holds across the whole grid
	{
		int perSm = 0;
		NB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, apply_kernel<false>, STEP_THREADS, 0));
		m_applyGrid = (unsigned) std::max(1, perSm) * (unsigned) m_sms;
	}
	// default shape of the two-launch step (set while the persistent loop is
	// not yet configured): two partitions per SM
	{
		uint32_t P = (uint32_t) ((N + 2 * m_sms - 1) / (2 * m_sms));
		setLaunch(P, std::min<uint32_t>(1024, std::max<uint32_t>(128, (P + 31) & ~31u)));
	}
	// the persistent step loop needs every CTA resident at once: a
	// cooperative launch of at most the occupancy limit
	{
		int coop = 0;
		NB_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, m_device));
		m_runT = 384;  // the default shape: two CTAs of 384 threads per SM
		m_runGrid = coop ? runGridFor(m_runT) : 0;
		if(m_runGrid) {
			const size_t per = (N + m_runGrid - 1) / m_runGrid;
			m_runP = (uint32_t) std::max<size_t>(32, (per + 31) & ~(size_t) 31);
			m_barrier = dalloc<GridBarrier>(1);
			NB_CUDA(cudaMallocHost(&m_hBarrierError, 4));
			*m_hBarrierError = 0;
		}
		// the persistent loop's CTAs are those that fit at once; when each
		// thread would update more than two neurons in turn, the update is
		// faster as one launch over the whole network (a large batch)
		if((uint64_t) N > 2ull * m_runGrid * m_runT) usePersistent = false;
	}
	NB_CUDA(cudaStreamSynchronize(m_stream));
	resetTimer();
}

Simulation::~Simulation()
{
	releaseAll();
}

void Simulation::releaseAll() noexcept
{
	cudaSetDevice(m_device);
	stopServe();
	freeKept();
	if(m_stream) cudaStreamSynchronize(m_stream);
	for(void* p : m_allocs) cudaFree(p);
	m_allocs.clear();
	if(m_graph) cudaGraphExecDestroy(m_graph);
	if(m_hCycle) cudaFreeHost(m_hCycle);
	if(m_hBarrierError) cudaFreeHost(m_hBarrierError);
	if(m_hFired) cudaFreeHost(m_hFired);
	if(m_hFiredMapped) cudaFreeHost(m_hFiredMapped);
	if(m_hStim) cudaFreeHost(m_hStim);
	if(m_hServe) cudaFreeHost(m_hServe);
	if(m_hFiredIds) cudaFreeHost(m_hFiredIds);
	if(m_serveEnd) cudaEventDestroy(m_serveEnd);
	if(m_ev0) cudaEventDestroy(m_ev0);
	if(m_ev1) cudaEventDestroy(m_ev1);
	for(cudaEvent_t e : m_evPool) cudaEventDestroy(e);
	m_evPool.clear();
	if(m_stream) cudaStreamDestroy(m_stream);
	m_graph = nullptr;
	m_hCycle = nullptr;
	m_hBarrierError = nullptr;
	m_hFired = nullptr;
	m_hFiredMapped = nullptr;
	m_hStim = nullptr;
	m_hServe = nullptr;
	m_hFiredIds = nullptr;
	m_serveEnd = m_ev0 = m_ev1 = nullptr;
	m_stream = nullptr;
}

void Simulation::sync()
{
	stopServe();
	NB_CUDA(cudaStreamSynchronize(m_stream));
}

unsigned Simulation::localIdx(unsigned g) const
{
	if(m_nets > 1) NB_THROW(NEMO_API_UNSUPPORTED, "per-neuron access is not available on a batch of networks");
	auto it = m_g2l[0].find(g);
	if(it == m_g2l[0].end()) NB_THROW(NEMO_INVALID_INPUT, "Non-existing neuron index %u", g);
	return it->second;
}

void Simulation::locate(unsigned g, const HostType** t, unsigned* i) const
{
	unsigned l = localIdx(g);
	*t = &m_types[m_ltype[l]];
	*i = l - (*t)->base;
}

void Simulation::timedBegin(int kind)
{
	if(!profiling || !m_inRun) return;
	if(m_evNext + 2 > m_evPool.size()) {
		size_t old = m_evPool.size();
		m_evPool.resize(std::max<size_t>(64, old * 2));
		for(size_t i = old; i < m_evPool.size(); ++i) NB_CUDA(cudaEventCreate(&m_evPool[i]));
	}
	m_evUse.emplace_back(kind, m_evNext);
	NB_CUDA(cudaEventRecord(m_evPool[m_evNext], m_stream));
	m_evNext += 2;
}

void Simulation::timedEnd()
{
	if(!profiling || !m_inRun) return;
	NB_CUDA(cudaEventRecord(m_evPool[m_evUse.back().second + 1], m_stream));
}

unsigned Simulation::runGridFor(uint32_t T) const
{
	// run_kernel and serve_kernel (the resident loop of nemo_step) share
	// the launch shape
	int perSm = 0, perSmServe = 0;
	NB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, run_kernel_for(T, false), (int) T,
			m_dev.recentBytes));
	NB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSmServe, serve_kernel_for(T), (int) T,
			m_dev.recentBytes));
	perSm = std::min(perSm, perSmServe);
	return perSm > 0 ? (unsigned) perSm * (unsigned) m_sms : 0u;
}

void Simulation::setLaunch(uint32_t P, uint32_t T)
{
	stopServe();
	if(persistentActive()) {
		// any multiple of 32 neurons per partition; 64 to RUN_THREADS threads
		m_runP = std::max<uint32_t>(32, (std::min<uint32_t>(P, 1u << 30) + 31) & ~31u);
		T = std::max<uint32_t>(64, std::min<uint32_t>(RUN_THREADS, (T + 31) & ~31u));
		const unsigned g = runGridFor(T);
		if(g) {
			m_runT = T;
			m_runGrid = g;
		}
		return;
	}
	P = std::max<uint32_t>(32, std::min<uint32_t>(MAX_PARTITION, (P + 31) & ~31u));
	T = std::max<uint32_t>(32, std::min<uint32_t>(1024, (T + 31) & ~31u));
	// the per-CTA work offsets are 32-bit
	while(P > 32 && ((uint64_t) P * std::max(m_maxOutDeg, m_maxPlasticInDeg) >= (1ull << 31))) P -= 32;
	m_P = P;
	m_T = T;
}

void Simulation::launchStep(bool /*fullRecord*/)
{
	stopServe();
	const uint32_t cur = (uint32_t) (m_cycle & 1);
	const uint32_t ring = (uint32_t) (m_cycle % m_dev.R);
	const unsigned grid = (m_N + m_P - 1) / m_P;
	timedBegin(K_STDP);
	launch_chained(deliver_kernel, m_deliverGrid, STEP_THREADS, m_dev.recentBytes, m_stream, m_dev, cur ^ 1u,
			(uint32_t) (PHASE_DELIVER | PHASE_STDP | PHASE_RESET), 0u, 0, nullptr, 0u, 0u);
	timedEnd();
	timedBegin(K_STEP);
	launch_chained(update_kernel_for(m_T), grid, m_T, 0, m_stream, m_dev, m_P, cur, ring, (uint32_t) m_cycle, 0u, 0,
			nullptr);
	timedEnd();
	m_cycle++;
	m_timerSteps++;
	m_stdpPending = true;
}

// the STDP accumulation of the last step, which the next step's pre-phase
// would otherwise run (before applyStdp, that must be now)
void Simulation::flushStdp()
{
	stopServe();
	if(!m_stdpPending) return;
	m_stdpPending = false;
	if(!m_dev.stdp || m_cycle == 0) return;
	const uint32_t last = (uint32_t) ((m_cycle - 1) & 1);
	timedBegin(K_STDP);
	deliver_kernel<<<m_deliverGrid, STEP_THREADS, m_dev.recentBytes, m_stream>>>(m_dev, last, PHASE_STDP, 0, 0);
	timedEnd();
	NB_CUDA(cudaMemsetAsync(m_dev.stdpWork.count + last, 0, 8, m_stream));
}

// n consecutive steps in one cooperative launch of the persistent step loop
// (finalStdp, stim, nf, ni, hostFired: see run_kernel)
void Simulation::launchRun(unsigned n, bool finalStdp, const uint32_t* stim, uint32_t nf, uint32_t ni,
		uint32_t* hostFired)
{
	DevSim dev = m_dev;
	uint32_t P = m_runP, steps = n;
	unsigned long long c0 = m_cycle;
	GridBarrier* gb = m_barrier;
	// no more CTAs than partitions (a CTA without one only takes part in the
	// delivery phase, which the other CTAs' warps cover as well)
	const unsigned grid = (unsigned) std::min<uint64_t>(m_runGrid, std::max<uint64_t>(1, (m_N + P - 1) / P));
	// the barrier counter runs on across launches; restart it well before
	// it could wrap
	const uint64_t arrivals = (uint64_t) grid * (2ull * n + (finalStdp ? 1 : 0));
	stopServe();
	if(m_barrierStale || m_barrierBase + arrivals >= (1ull << 31)) {
		NB_CUDA(cudaMemsetAsync(&m_barrier->count, 0, 4, m_stream));
		m_barrierBase = 0;
		m_barrierStale = false;
	}
	uint32_t base = (uint32_t) m_barrierBase;
	int fin = finalStdp ? 1 : 0;
	void* args[] = { &dev, &P, &steps, &c0, &gb, &base, &fin, &stim, &nf, &ni, &hostFired };
	timedBegin(K_RUN);
	NB_CUDA(cudaLaunchCooperativeKernel(run_kernel_for(m_runT, m_dev.trace != nullptr), dim3(grid), dim3(m_runT), args,
			m_dev.recentBytes, m_stream));
	timedEnd();
	m_barrierBase += arrivals;
	m_cycle += n;
	m_timerSteps += n;
	m_stdpPending = !finalStdp;
	m_barrierUsed = true;
}

// after a stream synchronisation: a grid-barrier wait of the persistent step
// loop that gave up (in any launch since the last check) leaves the
// simulation state undefined
void Simulation::checkBarrier()
{
	if(!m_barrierUsed) return;
	m_barrierUsed = false;
	NB_CUDA(cudaMemcpy(m_hBarrierError, &m_barrier->error, 4, cudaMemcpyDeviceToHost));
	if(*m_hBarrierError) {
		*m_hBarrierError = 0;
		NB_CUDA(cudaMemset(m_barrier, 0, sizeof(GridBarrier)));
		m_barrierBase = 0;
		m_barrierStale = false;
		NB_THROW(NEMO_CUDA_ERROR, "persistent step loop: a grid barrier wait timed out");
	}
}

// n consecutive steps: the persistent step loop, or whole CUDA graphs of
// GRAPH_STEPS two-launch steps (captured once per launch shape and replayed
// from a device cycle counter) and single launches for the rest
void Simulation::launchSteps(unsigned n)
{
	stopServe();
	if(usePersistent && m_runGrid && n > 1) {
		launchRun(n);
		return;
	}
	if(!useGraphs || profiling || n < GRAPH_STEPS) {
		for(unsigned i = 0; i < n; ++i) launchStep(false);
		return;
	}
	if(!m_graph || m_graphP != m_P || m_graphT != m_T) buildGraph();
	*m_hCycle = m_cycle;
	NB_CUDA(cudaMemcpyAsync(m_dev.cycleDev, m_hCycle, 8, cudaMemcpyHostToDevice, m_stream));
	while(n >= GRAPH_STEPS) {
		NB_CUDA(cudaGraphLaunch(m_graph, m_stream));
		m_cycle += GRAPH_STEPS;
		m_timerSteps += GRAPH_STEPS;
		m_stdpPending = true;
		n -= GRAPH_STEPS;
	}
	// the pinned cycle value must not change before the copy above ran
	NB_CUDA(cudaStreamSynchronize(m_stream));
	for(unsigned i = 0; i < n; ++i) launchStep(false);
}

void Simulation::buildGraph()
{
	if(m_graph) {
		cudaGraphExecDestroy(m_graph);
		m_graph = nullptr;
	}
	sync();
	const unsigned grid = (m_N + m_P - 1) / m_P;
	cudaGraph_t g;
	NB_CUDA(cudaStreamBeginCapture(m_stream, cudaStreamCaptureModeThreadLocal));
	for(unsigned k = 0; k < GRAPH_STEPS; ++k) {
		launch_chained(deliver_kernel, m_deliverGrid, STEP_THREADS, m_dev.recentBytes, m_stream, m_dev, 0u,
				(uint32_t) (PHASE_DELIVER | PHASE_STDP | PHASE_RESET), k, 1, nullptr, 0u, 0u);
		launch_chained(update_kernel_for(m_T), grid, m_T, 0, m_stream, m_dev, m_P, 0u, 0u, 0u, k, 1, nullptr);
	}
	advance_cycle_kernel<<<1, 1, 0, m_stream>>>(m_dev.cycleDev, GRAPH_STEPS);
	NB_CUDA(cudaStreamEndCapture(m_stream, &g));
	cudaError_t err = cudaGraphInstantiate(&m_graph, g, 0);
	cudaGraphDestroy(g);
	if(err != cudaSuccess) {
		m_graph = nullptr;
		NB_THROW(NEMO_CUDA_ERROR, "CUDA graph instantiation failed: %s", cudaGetErrorString(err));
	}
	m_graphP = m_P;
	m_graphT = m_T;
}

// ---------------------------------------------------------------------------
// the resident step loop of nemo_step (serve_kernel)

void Simulation::setResidentIdle(unsigned us)
{
	if(us > RESIDENT_IDLE_MAX_US) {
		NB_THROW(NEMO_INVALID_INPUT, "resident step loop idle time %u us is above the limit of %u us", us,
				RESIDENT_IDLE_MAX_US);
	}
	// a running loop keeps the idle time it was launched with
	stopServe();
	residentIdleUs = us;
}

void Simulation::setWaitLimit(uint32_t polls)
{
	// a running loop keeps the limit it was launched with
	stopServe();
	m_dev.waitLimit = polls;
}

bool Simulation::residentAvailable() const
{
	return residentIdleUs != 0 && persistentActive() && m_barrier != nullptr;
}

// Launches the loop at the current cycle for the next request; its barrier
// counter starts from zero and is left at a value the host does not track.
void Simulation::launchServe()
{
	if(!m_hFiredIds) {
		NB_CUDA(cudaHostAlloc(&m_hFiredIds, (size_t) m_N * 4, cudaHostAllocMapped));
		NB_CUDA(cudaHostGetDevicePointer(&m_dFiredIdsMapped, m_hFiredIds, 0));
	}
	// the barrier counter and the request word (count and cmd, adjacent)
	NB_CUDA(cudaMemsetAsync(&m_barrier->count, 0, 8, m_stream));
	m_barrierBase = 0;
	DevSim dev = m_dev;
	uint32_t P = m_runP;
	unsigned long long c0 = m_cycle;
	GridBarrier* gb = m_barrier;
	ServeCtl* ctl = m_dServe;
	uint32_t seq0 = m_serveSeq;
	const uint32_t* stim = m_dStimMapped;
	uint32_t* hf = m_dFiredIdsMapped;
	unsigned long long idleNs = (unsigned long long) residentIdleUs * 1000ull;
	const unsigned grid = (unsigned) std::min<uint64_t>(m_runGrid, std::max<uint64_t>(1, (m_N + P - 1) / P));
	void* args[] = { &dev, &P, &c0, &gb, &ctl, &seq0, &stim, &hf, &idleNs };
	NB_CUDA(cudaLaunchCooperativeKernel(serve_kernel_for(m_runT), dim3(grid), dim3(m_runT), args, m_dev.recentBytes,
			m_stream));
	NB_CUDA(cudaEventRecord(m_serveEnd, m_stream));
	m_serving = true;
	m_barrierUsed = true;
	m_barrierStale = true;
}

// Asks a running loop to end; work queued on the stream afterwards runs
// once it has.  The request consumes a sequence number, so that a loop
// still polling when the next request is written (to a new launch, queued
// behind it) matches neither and only waits out its idle time.  Neither
// allocates nor throws.
void Simulation::stopServe() noexcept
{
	if(!m_serving) return;
	m_serving = false;
	std::atomic_thread_fence(std::memory_order_seq_cst);
	reinterpret_cast<volatile ServeCtl*>(m_hServe)->req[0] = (unsigned long long) (m_serveSeq | SERVE_STOP) << 32;
	std::atomic_thread_fence(std::memory_order_seq_cst);
	m_serveSeq = serve_next(m_serveSeq);
}

// One step through the resident loop: the stimulus is already in m_hStim.
void Simulation::stepResident(uint32_t nf, uint32_t ni)
{
	volatile ServeCtl* c = reinterpret_cast<volatile ServeCtl*>(m_hServe);
	const uint32_t want = m_serveSeq;
	// a small firing stimulus goes in the request line itself
	const bool inl = ni == 0 && nf <= SERVE_INLINE;
	if(inl) {
		for(uint32_t i = 0; i < nf; ++i) c->inl[i] = (unsigned long long) want << 32 | m_hStim[i];
	}
	// the stimulus (m_hStim or inline) is in place before the request
	std::atomic_thread_fence(std::memory_order_seq_cst);
	c->req[1] = (unsigned long long) want << 32 | ni;
	c->req[0] = (unsigned long long) want << 32 | (inl ? SERVE_INLINE_FLAG | nf : nf);
	std::atomic_thread_fence(std::memory_order_seq_cst);
	if(!m_serving) launchServe();
	const auto t0 = std::chrono::steady_clock::now();
	for(uint32_t polls = 1;; ++polls) {
		if(c->done == want) break;
		if((polls & 63u) == 0) {
			const cudaError_t q = cudaEventQuery(m_serveEnd);
			if(q == cudaSuccess) {
				if(c->done == want) break;
				// the loop ended before this request: it was idle for too
				// long (launch it again), or a grid barrier gave up
				// (checkBarrier throws)
				m_serving = false;
				checkBarrier();
				launchServe();
			} else if(q != cudaErrorNotReady) {
				NB_CUDA(q);
			}
			if(std::chrono::steady_clock::now() - t0 > std::chrono::seconds(RESIDENT_REPLY_LIMIT_S)) {
				NB_THROW(NEMO_CUDA_ERROR, "resident step loop: no reply within %u s", RESIDENT_REPLY_LIMIT_S);
			}
		}
#if defined(__x86_64__)
		__builtin_ia32_pause();
#endif
	}
	std::atomic_thread_fence(std::memory_order_seq_cst);
	m_fired.assign(m_hFiredIds, m_hFiredIds + c->fired);
	stepEvents += c->events;
	m_serveSeq = serve_next(m_serveSeq);
	m_cycle++;
	m_timerSteps++;
	m_stdpPending = true;
}

// One step with host buffers: the stimulus is staged in mapped host memory
// that the pre-phase kernel reads, and the update writes the fired
// bit-vector words to mapped host memory, so no copy is queued.
const std::vector<unsigned>& Simulation::step(const unsigned* fstim, size_t nf,
		const unsigned* inidx, const float* icur, size_t ni)
{
	NB_CUDA(cudaSetDevice(m_device));
	// validate and map the stimulus before touching any state
	// (src/nemo/cpu/Simulation.cpp:141-163; the last current for a neuron wins)
	std::vector<uint32_t>& fl = m_stepScratch;
	fl.resize(nf);
	for(size_t i = 0; i < nf; ++i) fl[i] = localIdx(fstim[i]);
	std::vector<std::pair<uint32_t, float>>& cur = m_stepCurrents;
	cur.clear();
	if(ni) {
		std::unordered_map<uint32_t, size_t> at;
		for(size_t i = 0; i < ni; ++i) {
			const uint32_t l = localIdx(inidx[i]);
			auto it = at.find(l);
			if(it == at.end()) {
				at.emplace(l, cur.size());
				cur.emplace_back(l, icur[i]);
			} else {
				cur[it->second].second = icur[i];
			}
		}
	}
	const size_t need = nf + 2 * cur.size();
	if(need > m_stimCap) {
		// the resident step loop holds the old buffer's address: end it
		sync();
		if(m_hStim) cudaFreeHost(m_hStim);
		m_hStim = nullptr;
		m_stimCap = std::max<size_t>(need, 1024);
		NB_CUDA(cudaHostAlloc(&m_hStim, m_stimCap * 4, cudaHostAllocMapped));
		NB_CUDA(cudaHostGetDevicePointer(&m_dStimMapped, m_hStim, 0));
	}
	if(need) {
		memcpy(m_hStim, fl.data(), nf * 4);
		for(size_t i = 0; i < cur.size(); ++i) {
			m_hStim[nf + i] = cur[i].first;
			memcpy(&m_hStim[nf + cur.size() + i], &cur[i].second, 4);
		}
	}
	if(residentAvailable()) {
		stepResident((uint32_t) nf, (uint32_t) cur.size());
		return m_fired;
	}
	// two launches (a one-step cooperative launch of the persistent loop is
	// slower here: its launch and grid barriers cost more than a second
	// kernel)
	stopServe();
	const uint32_t c = (uint32_t) (m_cycle & 1);
	const uint32_t ring = (uint32_t) (m_cycle % m_dev.R);
	launch_chained(deliver_kernel, m_deliverGrid, STEP_THREADS, m_dev.recentBytes, m_stream, m_dev, c ^ 1u,
			(uint32_t) (PHASE_DELIVER | PHASE_STDP | PHASE_RESET), 0u, 0,
			need ? (const uint32_t*) m_dStimMapped : nullptr, (uint32_t) nf, (uint32_t) cur.size());
	launch_chained(update_kernel_for(m_T), (m_N + m_P - 1) / m_P, m_T, 0, m_stream, m_dev, m_P, c, ring,
			(uint32_t) m_cycle, 0u, 0,
			m_dFiredMapped);
	m_cycle++;
	m_timerSteps++;
	m_stdpPending = true;
	sync();
	NB_CUDA(cudaGetLastError());
	return collectFired();
}

// the fired words of the last step() (mapped host memory) as global ids in
// ascending local index (setFiring, src/nemo/cpu/Simulation.cpp:200-208)
const std::vector<unsigned>& Simulation::collectFired()
{
	m_fired.clear();
	for(uint32_t w = 0; w < m_dev.W; ++w) {
		uint32_t bits = m_hFiredMapped[w];
		while(bits) {
			uint32_t b = __builtin_ctz(bits);
			bits &= bits - 1;
			const uint32_t l = w * 32 + b;
			m_fired.push_back(m_l2g[l]);
			stepEvents += m_outDegree[l];
		}
	}
	return m_fired;
}

void Simulation::applyStdpDevice(int32_t R)
{
	stopServe();
	flushStdp();
	timedBegin(K_APPLY);
	if(!m_weightsClamped) {
		apply_kernel<true><<<m_applyGrid, STEP_THREADS, 0, m_stream>>>(m_dev, R);
	} else {
		apply_kernel<false><<<m_applyGrid, STEP_THREADS, 0, m_stream>>>(m_dev, R);
	}
	timedEnd();
	// updatedWeight's result always lies within the clamp range of its sign
	// class, so after one full pass every plastic weight does, and only the
	// synapses of touched targets can change
	m_weightsClamped = true;
	NB_CUDA(cudaMemsetAsync(m_dev.touchedBits, 0, (size_t) m_dev.W * 4, m_stream));
}

/* ConnectivityMatrix::applyStdp argument checks (src/nemo/ConnectivityMatrix.cpp:241-259) */
void Simulation::applyStdp(float reward)
{
	if(!m_dev.stdp) NB_THROW(NEMO_LOGIC_ERROR, "applyStdp called, but no STDP model specified");
	int32_t R = fx_toFix(reward);
	if(R == 0 && reward != 0) {
		NB_THROW(NEMO_INVALID_INPUT, "STDP reward rounded down to zero. The smallest valid reward is %f",
				(double) fx_toFloat(1));
	}
	NB_CUDA(cudaSetDevice(m_device));
	applyStdpDevice(R);
	sync();
	NB_CUDA(cudaGetLastError());
}

void Simulation::run(unsigned steps, unsigned stdpPeriod, float reward, unsigned* counts,
		uint64_t* events, unsigned* ids, size_t cap, size_t* len)
{
	NB_CUDA(cudaSetDevice(m_device));
	int32_t R = 0;
	if(stdpPeriod) {
		if(!m_dev.stdp) NB_THROW(NEMO_LOGIC_ERROR, "applyStdp called, but no STDP model specified");
		R = fx_toFix(reward);
		if(R == 0 && reward != 0) NB_THROW(NEMO_INVALID_INPUT, "STDP reward rounded down to zero");
	}
	// the two-launch loop's CUDA graph is instantiated (once per launch
	// shape) before the run's timing events, which time the simulation only
	const unsigned longest = stdpPeriod ? std::min(stdpPeriod, steps) : steps;
	if(!persistentActive() && useGraphs && !profiling && longest >= GRAPH_STEPS
			&& (!m_graph || m_graphP != m_P || m_graphT != m_T)) {
		buildGraph();
	}
	size_t total = 0;
	float runMs = 0;
	for(int k = 0; k < K_KINDS; ++k) { kernelMs[k] = 0; kernelLaunches[k] = 0; }
	lastFired = lastEvents = lastStdpEntries = 0;
	unsigned done = 0;
	struct InRun {
		bool& f;
		explicit InRun(bool& x) : f(x) { f = true; }
		~InRun() { f = false; }
	} inRun(m_inRun);
	while(done < steps) {
		const uint64_t first = m_cycle;
		const unsigned chunk = std::min<unsigned>(steps - done, m_dev.R);
		// the ring positions this chunk uses start at first % R and may wrap
		NB_CUDA(cudaMemsetAsync(m_dev.firedCount, 0, m_dev.R * 4, m_stream));
		NB_CUDA(cudaMemsetAsync(m_dev.eventCount, 0, m_dev.R * 8, m_stream));
		NB_CUDA(cudaMemsetAsync(m_dev.stdpCount, 0, m_dev.R * 8, m_stream));
		m_evUse.clear();
		m_evNext = 0;
		NB_CUDA(cudaEventRecord(m_ev0, m_stream));
		for(unsigned i = 0; i < chunk;) {
			const unsigned untilApply = stdpPeriod ? stdpPeriod - (done + i) % stdpPeriod : chunk - i;
			const unsigned seg = std::min(chunk - i, untilApply);
			launchSteps(seg);
			i += seg;
			if(stdpPeriod && (done + i) % stdpPeriod == 0) applyStdpDevice(R);
		}
		NB_CUDA(cudaEventRecord(m_ev1, m_stream));
		std::vector<uint32_t> hc(m_dev.R);
		std::vector<unsigned long long> he(m_dev.R), hs(m_dev.R);
		NB_CUDA(cudaMemcpyAsync(hc.data(), m_dev.firedCount, m_dev.R * 4, cudaMemcpyDeviceToHost, m_stream));
		NB_CUDA(cudaMemcpyAsync(he.data(), m_dev.eventCount, m_dev.R * 8, cudaMemcpyDeviceToHost, m_stream));
		NB_CUDA(cudaMemcpyAsync(hs.data(), m_dev.stdpCount, m_dev.R * 8, cudaMemcpyDeviceToHost, m_stream));
		if(ids || (m_nets > 1 && counts)) {
			NB_CUDA(cudaMemcpyAsync(m_hFired, m_dev.firedRing, (size_t) m_dev.R * m_dev.W * 4,
					cudaMemcpyDeviceToHost, m_stream));
		}
		sync();
		NB_CUDA(cudaGetLastError());
		checkBarrier();
		float ms = 0;
		NB_CUDA(cudaEventElapsedTime(&ms, m_ev0, m_ev1));
		runMs += ms;
		for(const auto& u : m_evUse) {
			float km = 0;
			NB_CUDA(cudaEventElapsedTime(&km, m_evPool[u.second], m_evPool[u.second + 1]));
			kernelMs[u.first] += km;
			kernelLaunches[u.first]++;
		}
		m_evUse.clear();
		m_evNext = 0;
		for(uint32_t r = 0; r < m_dev.R; ++r) lastStdpEntries += hs[r];
		for(unsigned i = 0; i < chunk; ++i) {
			uint32_t r = (uint32_t) ((first + i) % m_dev.R);
			if(events) events[done + i] = he[r];
			lastFired += hc[r];
			lastEvents += he[r];
			if(m_nets == 1) {
				if(counts) counts[done + i] = hc[r];
				if(ids) {
					const uint32_t* words = m_hFired + (size_t) r * m_dev.W;
					for(uint32_t w = 0; w < m_dev.W; ++w) {
						uint32_t bits = words[w];
						while(bits) {
							uint32_t b = __builtin_ctz(bits);
							bits &= bits - 1;
							if(total >= cap) NB_THROW(NEMO_BUFFER_OVERFLOW, "fired id buffer too small");
							ids[total++] = m_l2g[w * 32 + b];
						}
					}
				} else {
					total += hc[r];
				}
			} else {
				total += decodeBatchStep(r, done + i, counts, ids, total, cap);
			}
		}
		done += chunk;
	}
	if(len) *len = total;
	lastRunMs = runMs;
}

// Fired neurons of ring position r, split by network: per network in its
// own local order (as its single-network run reports them), networks in
// order.  Writes counts[step * nets + net] and appends to ids when given.
size_t Simulation::decodeBatchStep(uint32_t r, unsigned step, unsigned* counts, unsigned* ids, size_t pos, size_t cap)
{
	std::vector<std::vector<uint32_t>>& per = m_batchScratch;
	per.resize(m_nets);
	for(auto& v : per) v.clear();
	const uint32_t* words = m_hFired + (size_t) r * m_dev.W;
	for(uint32_t w = 0; w < m_dev.W; ++w) {
		uint32_t bits = words[w];
		while(bits) {
			uint32_t b = __builtin_ctz(bits);
			bits &= bits - 1;
			const uint32_t u = w * 32 + b;
			per[m_netOf[u]].push_back(u);
		}
	}
	size_t n = 0;
	for(unsigned k = 0; k < m_nets; ++k) {
		auto& v = per[k];
		if(!std::is_sorted(v.begin(), v.end(), [&](uint32_t a, uint32_t b) { return m_netLocal[a] < m_netLocal[b]; })) {
			std::sort(v.begin(), v.end(), [&](uint32_t a, uint32_t b) { return m_netLocal[a] < m_netLocal[b]; });
		}
		if(counts) counts[(size_t) step * m_nets + k] = (unsigned) v.size();
		if(ids) {
			if(pos + n + v.size() > cap) NB_THROW(NEMO_BUFFER_OVERFLOW, "fired id buffer too small");
			for(uint32_t u : v) ids[pos + n++] = m_l2g[u];
		} else {
			n += v.size();
		}
	}
	return n;
}

float Simulation::autotune(unsigned trialSteps)
{
	NB_CUDA(cudaSetDevice(m_device));
	sync();
	trialSteps = std::max(1u, trialSteps);
	// the state that trial steps modify
	std::vector<std::pair<void*, size_t>> regions;
	for(const HostType& t : m_types) regions.emplace_back(t.dState, (size_t) t.n * t.desc.nstate * t.desc.history * 4);
	regions.emplace_back(m_dev.rng, (size_t) 4 * m_N * 4);
	regions.emplace_back(m_dev.hist, (size_t) 2 * m_N * 8);
	regions.emplace_back(m_dev.recent, (size_t) 2 * m_dev.recentWords * 4);
	regions.emplace_back(m_dev.fstim, (size_t) m_dev.W * 4);
	regions.emplace_back(m_dev.curExt, (size_t) m_N * 4);
	regions.emplace_back(m_dev.slot, (size_t) m_N * 16);
	// the work lists published by the last step (pending for the next)
	for(const WorkList* L : { &m_dev.dlvWork, &m_dev.stdpWork }) {
		unsigned long long c[2];
		NB_CUDA(cudaMemcpy(c, L->count, 16, cudaMemcpyDeviceToHost));
		const uint64_t groups = std::max(c[0] >> 32, c[1] >> 32);
		const uint64_t entries = std::max(c[0] & 0xffffffffull, c[1] & 0xffffffffull);
		regions.emplace_back(L->group, (size_t) groups * 16);
		regions.emplace_back(L->bucket, (size_t) (entries / BUCKET + 1) * 4);
		regions.emplace_back(L->count, 16);
	}
	if(m_dev.stdp) regions.emplace_back(m_dev.rcmAcc, (size_t) lastPlastic * 4);
	regions.emplace_back(m_dev.touchedBits, (size_t) m_dev.W * 4);
	std::vector<void*> backup;
	for(auto& r : regions) {
		void* p = nullptr;
		if(r.second == 0) { backup.push_back(nullptr); continue; }
		cudaError_t err = cudaMalloc(&p, r.second);
		if(err != cudaSuccess) {
			for(void* b : backup) if(b) cudaFree(b);
			NB_THROW(NEMO_CUDA_MEMORY_ERROR, "autotune: no device memory for the state snapshot");
		}
		NB_CUDA(cudaMemcpyAsync(p, r.first, r.second, cudaMemcpyDeviceToDevice, m_stream));
		backup.push_back(p);
	}
	const uint64_t cycle = m_cycle;
	const unsigned long timerSteps = m_timerSteps;
	const bool stdpPending = m_stdpPending;
	const bool prof = profiling;
	profiling = false;
	auto restore = [&]() {
		for(size_t i = 0; i < regions.size(); ++i) {
			if(backup[i]) {
				NB_CUDA(cudaMemcpyAsync(regions[i].first, backup[i], regions[i].second, cudaMemcpyDeviceToDevice, m_stream));
			}
		}
		m_cycle = cycle;
		m_timerSteps = timerSteps;
		m_stdpPending = stdpPending;
	};

	std::vector<std::pair<uint32_t, uint32_t>> cands;
	const bool pers = persistentActive();
	if(pers) {
		// persistent loop: 256 to RUN_THREADS threads per CTA, 1 to 4 partitions per CTA
		for(uint32_t T : {256u, 384u, RUN_THREADS_PAIR, RUN_THREADS}) {
			const unsigned g = runGridFor(T);
			if(!g) continue;
			for(unsigned k : {1u, 2u, 4u}) {
				uint32_t P = (uint32_t) ((m_N + (size_t) k * g - 1) / ((size_t) k * g));
				P = std::max<uint32_t>(32, (P + 31) & ~31u);
				if(std::find(cands.begin(), cands.end(), std::make_pair(P, T)) == cands.end()) cands.emplace_back(P, T);
			}
		}
	} else {
		// two-launch step: 1 to 16 partitions per SM, 128 to 1024 threads per CTA
		for(unsigned k : {1u, 2u, 3u, 4u, 6u, 8u, 12u, 16u}) {
			uint32_t P = (uint32_t) ((m_N + (size_t) k * m_sms - 1) / ((size_t) k * m_sms));
			P = std::max<uint32_t>(32, std::min<uint32_t>(MAX_PARTITION, (P + 31) & ~31u));
			for(uint32_t T : {128u, 256u, 512u, 1024u}) {
				if(T > std::max<uint32_t>(128, P)) continue;
				if(std::find(cands.begin(), cands.end(), std::make_pair(P, T)) == cands.end()) cands.emplace_back(P, T);
			}
		}
	}
	const uint32_t P0 = partition(), T0 = threads();
	float best = -1;
	uint32_t bestP = P0, bestT = T0;
	try {
		for(auto& c : cands) {
			setLaunch(c.first, c.second);
			// untimed warm-up of this shape
			if(pers) launchRun(1);
			else launchStep(false);
			NB_CUDA(cudaEventRecord(m_ev0, m_stream));
			if(pers) {
				launchRun(trialSteps);
			} else {
				for(unsigned i = 0; i < trialSteps; ++i) launchStep(false);
			}
			NB_CUDA(cudaEventRecord(m_ev1, m_stream));
			sync();
			NB_CUDA(cudaGetLastError());
			checkBarrier();
			float ms = 0;
			NB_CUDA(cudaEventElapsedTime(&ms, m_ev0, m_ev1));
			if(best < 0 || ms < best) {
				best = ms;
				bestP = partition();
				bestT = threads();
			}
			restore();
		}
	} catch(...) {
		restore();
		sync();
		for(void* b : backup) if(b) cudaFree(b);
		setLaunch(P0, T0);
		profiling = prof;
		throw;
	}
	sync();
	for(void* b : backup) if(b) cudaFree(b);
	profiling = prof;
	setLaunch(bestP, bestT);
	return best * 1e3f / trialSteps;
}

unsigned Simulation::tracePhases(unsigned steps, uint64_t* out, size_t cap)
{
	NB_CUDA(cudaSetDevice(m_device));
	if(!persistentActive()) NB_THROW(NEMO_API_UNSUPPORTED, "the phase trace needs the persistent step loop");
	const unsigned grid = (unsigned) std::min<uint64_t>(m_runGrid, std::max<uint64_t>(1, (m_N + m_runP - 1) / m_runP));
	const size_t n = (size_t) steps * grid * TRACE_MARKS;
	if(cap < n) NB_THROW(NEMO_BUFFER_OVERFLOW, "trace buffer too small: %zu values needed", n);
	sync();
	unsigned long long* d = nullptr;
	NB_CUDA(cudaMalloc(&d, std::max<size_t>(n, 1) * 8));
	m_dev.trace = d;
	m_dev.traceSteps = steps;
	cudaError_t err = cudaSuccess;
	try {
		launchRun(steps);
		sync();
		err = cudaGetLastError();
		checkBarrier();
	} catch(...) {
		m_dev.trace = nullptr;
		m_dev.traceSteps = 0;
		cudaFree(d);
		throw;
	}
	m_dev.trace = nullptr;
	m_dev.traceSteps = 0;
	if(err == cudaSuccess) err = cudaMemcpy(out, d, n * 8, cudaMemcpyDeviceToHost);
	cudaFree(d);
	NB_CUDA(err);
	return grid;
}

// the state of the current cycle of a type (slot cycle % history;
// src/nemo/cpu/Neurons.cpp:80-92, :123)
float* Simulation::currentState(const HostType& t) const
{
	return t.dState + (size_t) (m_cycle % t.desc.history) * t.desc.nstate * t.n;
}

float Simulation::getNeuronState(unsigned g, unsigned var)
{
	const HostType* t; unsigned i;
	locate(g, &t, &i);
	if(var >= t->desc.nstate) NB_THROW(NEMO_INVALID_INPUT, "Invalid state variable index %u", var);
	float v;
	NB_CUDA(cudaSetDevice(m_device));
	NB_CUDA(cudaMemcpyAsync(&v, currentState(*t) + (size_t) var * t->n + i, 4, cudaMemcpyDeviceToHost, m_stream));
	sync();
	return v;
}

float Simulation::getNeuronParameter(unsigned g, unsigned p)
{
	const HostType* t; unsigned i;
	locate(g, &t, &i);
	if(p >= t->desc.nparam) NB_THROW(NEMO_INVALID_INPUT, "Invalid parameter index %u", p);
	float v;
	NB_CUDA(cudaSetDevice(m_device));
	NB_CUDA(cudaMemcpyAsync(&v, t->dParam + (size_t) p * t->n + i, 4, cudaMemcpyDeviceToHost, m_stream));
	sync();
	return v;
}

float Simulation::getMembranePotential(unsigned g)
{
	const HostType* t; unsigned i;
	locate(g, &t, &i);
	return getNeuronState(g, t->desc.mpot);
}

void Simulation::setNeuron(unsigned g, unsigned nargs, const float* args)
{
	const HostType* t; unsigned i;
	locate(g, &t, &i);
	unsigned np = t->desc.nparam, ns = t->desc.nstate;
	if(nargs != np + ns) {
		NB_THROW(NEMO_INVALID_INPUT,
				"Unexpected number of parameters/state variables when modifying neuron. Expected %u, found %u", np + ns, nargs);
	}
	NB_CUDA(cudaSetDevice(m_device));
	for(unsigned p = 0; p < np; ++p) {
		NB_CUDA(cudaMemcpyAsync(t->dParam + (size_t) p * t->n + i, args + p, 4, cudaMemcpyHostToDevice, m_stream));
	}
	for(unsigned v = 0; v < ns; ++v) {
		NB_CUDA(cudaMemcpyAsync(currentState(*t) + (size_t) v * t->n + i, args + np + v, 4, cudaMemcpyHostToDevice,
				m_stream));
	}
	sync();
}

void Simulation::setNeuronState(unsigned g, unsigned var, float v)
{
	const HostType* t; unsigned i;
	locate(g, &t, &i);
	if(var >= t->desc.nstate) NB_THROW(NEMO_INVALID_INPUT, "Invalid state variable index %u", var);
	NB_CUDA(cudaSetDevice(m_device));
	NB_CUDA(cudaMemcpyAsync(currentState(*t) + (size_t) var * t->n + i, &v, 4, cudaMemcpyHostToDevice, m_stream));
	sync();
}

void Simulation::setNeuronParameter(unsigned g, unsigned p, float v)
{
	const HostType* t; unsigned i;
	locate(g, &t, &i);
	if(p >= t->desc.nparam) NB_THROW(NEMO_INVALID_INPUT, "Invalid parameter index %u", p);
	NB_CUDA(cudaSetDevice(m_device));
	NB_CUDA(cudaMemcpyAsync(t->dParam + (size_t) p * t->n + i, &v, 4, cudaMemcpyHostToDevice, m_stream));
	sync();
}

bool Simulation::planDeviceBuild(const std::vector<const Network*>& nets, bool stdp,
		std::vector<DevicePart>& parts) const
{
	const uint32_t D = m_dev.dStride;
	parts.assign(nets.size(), DevicePart());
	uint64_t total = 0;
	for(size_t i = 0; i < nets.size(); ++i) {
		const Network& net = *nets[i];
		DevicePart& part = parts[i];
		if(nets.size() == 1) {
			part.srcBase = 0;
			part.nLocal = m_N;
		} else {
			// one neuron type: the network's neurons are one contiguous run
			int only = -1;
			for(size_t t = 0; t < net.types.size(); ++t) {
				if(net.types[t].size() == 0) continue;
				if(only >= 0) return false;
				only = (int) t;
			}
			if(only < 0) return false;
			const NetTypeRange& r = m_netTypes[i][only];
			part.srcBase = m_types[r.hostType].base + r.offset;
			part.nLocal = r.count;
		}
		const size_t Si = net.src.size();
		if(Si >= (1ull << 31) - 1 || (uint64_t) part.nLocal * D >= (1ull << 31) - 1) return false;
		uint32_t maxGid = 0;
		for(const auto& kv : m_g2l[i]) maxGid = std::max(maxGid, kv.first);
		if((uint64_t) maxGid + 1 > 4ull * part.nLocal + (1u << 20)) return false;
		part.g2l.assign((size_t) maxGid + 1, ~0u);
		for(const auto& kv : m_g2l[i]) part.g2l[kv.first] = kv.second;
		if(stdp) {
			uint64_t p = 0;
			for(size_t k = 0; k < Si; ++k) p += net.plastic[k] != 0;
			part.plastic = p;
		}
		total += Si;
	}
	if(stdp && total > 0xffffffffull) return false;
	// each network's rows and reverse rows follow the order of its neurons
	std::vector<size_t> order(nets.size());
	for(size_t i = 0; i < order.size(); ++i) order[i] = i;
	std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return parts[a].srcBase < parts[b].srcBase; });
	uint64_t so = 0, po = 0;
	for(size_t i : order) {
		parts[i].synOff = so;
		parts[i].plOff = po;
		so += nets[i]->src.size();
		po += parts[i].plastic;
	}
	return true;
}

// The device build of the connectivity (construction.cu), network by
// network into the union arrays: the same forward matrix, delay groups and
// reverse matrix as the host build, and the same errors, in the same order,
// for synapses between non-existing neurons and weights outside the
// fixed-point range.
void Simulation::buildOnDevice(const std::vector<const Network*>& nets, std::vector<DevicePart>& parts, bool deliver,
		std::vector<unsigned long long>& outPtr, std::vector<unsigned long long>& rcmPtr, uint64_t& dlvGroups)
{
	DevSim& S = m_dev;
	const unsigned N = m_N;
	const uint32_t D = S.dStride;
	// the wide delay-group table when some row has 65,536 synapses or more
	uint32_t maxOut = 0;
	uint64_t P = 0;
	for(size_t i = 0; i < nets.size(); ++i) {
		for(const auto& kv : nets[i]->axonCount) maxOut = std::max(maxOut, kv.second);
		P += parts[i].plastic;
	}
	uint32_t* synTgt = dalloc<uint32_t>(m_nsyn);
	uint32_t* synW = dalloc<uint32_t>(m_nsyn);
	auto* dOut = dalloc<unsigned long long>((size_t) N + 1);
	uint16_t* end16 = maxOut < 65536 ? dalloc<uint16_t>((size_t) N * D) : nullptr;
	uint32_t* end32 = maxOut < 65536 ? nullptr : dalloc<uint32_t>((size_t) N * D);
	auto* mask = dalloc<uint64_t>(N);
	uint32_t* rsrc = S.stdp ? dalloc<uint32_t>(P) : nullptr;
	uint32_t* rfwd = S.stdp ? dalloc<uint32_t>(P) : nullptr;
	outPtr.assign((size_t) N + 1, 0);
	rcmPtr.assign((size_t) N + 1, 0);
	dlvGroups = 0;
	for(size_t i = 0; i < nets.size(); ++i) {
		const Network& net = *nets[i];
		DevicePart& part = parts[i];
		DeviceConstruction c;
		c.S = net.src.size();
		c.src = net.src.data();
		c.tgt = net.tgt.data();
		c.delay = net.delay.data();
		c.weight = net.weight.data();
		c.plastic = net.plastic.data();
		c.g2l = part.g2l.data();
		c.maxGid = (uint32_t) (part.g2l.size() - 1);
		c.srcBase = part.srcBase;
		c.nLocal = part.nLocal;
		c.D = D;
		c.deliver = deliver;
		c.stdp = S.stdp != 0;
		c.keepQueries = !m_writeOnly && nets.size() == 1;
		c.synOff = part.synOff;
		c.plOff = part.plOff;
		c.synTgt = synTgt;
		c.synW = synW;
		c.outPtr = dOut;
		c.dEnd16 = end16;
		c.dEnd32 = end32;
		c.delayMask = mask;
		c.rcmSrc = rsrc;
		c.rcmFwd = rfwd;
		try {
			construct_on_device(c, m_stream);
		} catch(...) {
			m_kept = KeptSynapses{ c.keptSrc, c.keptPos, c.keptTgt, c.keptDelay, c.keptPlastic };
			freeKept();
			throw;
		}
		if(c.keepQueries) m_kept = KeptSynapses{ c.keptSrc, c.keptPos, c.keptTgt, c.keptDelay, c.keptPlastic };
		for(uint32_t s = 0; s < part.nLocal; ++s) {
			outPtr[part.srcBase + s] = c.hostOutPtr[s];
			rcmPtr[part.srcBase + s] = c.hostRcmPtr[s];
		}
		dlvGroups += c.dlvGroups;
		part.g2l.clear();
		part.g2l.shrink_to_fit();
	}
	outPtr[N] = m_nsyn;
	rcmPtr[N] = P;
	NB_CUDA(cudaMemcpyAsync(dOut + N, &outPtr[N], 8, cudaMemcpyHostToDevice, m_stream));
	S.synTgt = synTgt;
	S.synW = synW;
	S.outPtr = dOut;
	S.dEnd16 = end16;
	S.dEnd32 = end32;
	S.delayMask = mask;
	S.allPtr = dalloc<unsigned long long>((size_t) N + 1);  // no reverse matrix of all synapses
	m_outDegree.resize(N);
	for(unsigned s = 0; s < N; ++s) {
		m_outDegree[s] = (uint32_t) (outPtr[s + 1] - outPtr[s]);
		m_maxOutDeg = std::max(m_maxOutDeg, m_outDegree[s]);
	}
	if(S.stdp) {
		for(unsigned t = 0; t < N; ++t) {
			m_maxPlasticInDeg = std::max(m_maxPlasticInDeg, (uint32_t) (rcmPtr[t + 1] - rcmPtr[t]));
		}
		S.rcmSrc = rsrc;
		S.rcmFwd = rfwd;
		S.rcmAcc = dalloc<int32_t>(P);
		lastPlastic = P;
	}
	m_builtOnDevice = true;
	NB_CUDA(cudaStreamSynchronize(m_stream));
}

void Simulation::freeKept() noexcept
{
	cudaFree(m_kept.src);
	cudaFree(m_kept.pos);
	cudaFree(m_kept.tgt);
	cudaFree(m_kept.delay);
	cudaFree(m_kept.plastic);
	m_kept = KeptSynapses{};
}

// The query tables of a device-built network, from the arrays it kept: a
// synapse's per-source index is its rank among its source's synapses in
// insertion order (Network::addSynapses), so a stable counting sort by
// source gives each source's synapses in per-source-index order.
void Simulation::ensureQueryTables()
{
	if(!m_kept.src) return;
	const size_t Sn = m_nsyn;
	NB_CUDA(cudaSetDevice(m_device));
	hvector<uint32_t> src(Sn), pos(Sn), tgt(Sn);
	hvector<uint8_t> delay(Sn), plastic(Sn);
	NB_CUDA(cudaMemcpyAsync(src.data(), m_kept.src, Sn * 4, cudaMemcpyDeviceToHost, m_stream));
	NB_CUDA(cudaMemcpyAsync(pos.data(), m_kept.pos, Sn * 4, cudaMemcpyDeviceToHost, m_stream));
	NB_CUDA(cudaMemcpyAsync(tgt.data(), m_kept.tgt, Sn * 4, cudaMemcpyDeviceToHost, m_stream));
	NB_CUDA(cudaMemcpyAsync(delay.data(), m_kept.delay, Sn, cudaMemcpyDeviceToHost, m_stream));
	NB_CUDA(cudaMemcpyAsync(plastic.data(), m_kept.plastic, Sn, cudaMemcpyDeviceToHost, m_stream));
	sync();
	m_srcStart.assign(m_N + 1, 0);
	for(size_t k = 0; k < Sn; ++k) m_srcStart[src[k] + 1]++;
	for(unsigned s = 0; s < m_N; ++s) m_srcStart[s + 1] += m_srcStart[s];
	std::vector<uint64_t> fill(m_srcStart.begin(), m_srcStart.end() - 1);
	m_srcOrder.resize(Sn);
	for(size_t k = 0; k < Sn; ++k) m_srcOrder[fill[src[k]]++] = k;
	m_pos.assign(pos.begin(), pos.end());
	m_synDelay.assign(delay.begin(), delay.end());
	m_synPlastic.assign(plastic.begin(), plastic.end());
	m_synTarget.assign(tgt.begin(), tgt.end());
	freeKept();
}

void Simulation::connectivityDigest(uint64_t out[DIGESTS])
{
	NB_CUDA(cudaSetDevice(m_device));
	const DevSim& S = m_dev;
	const size_t N = m_N, P = lastPlastic;
	const size_t rows = N * S.dStride;
	out[0] = device_digest(S.synTgt, m_nsyn * 4, m_stream)
			+ 0x9E3779B97F4A7C15ull * device_digest(S.synW, m_nsyn * 4, m_stream);
	out[1] = device_digest(S.outPtr, (N + 1) * 8, m_stream);
	out[2] = S.dEnd16 ? device_digest(S.dEnd16, rows * 2, m_stream) : device_digest(S.dEnd32, rows * 4, m_stream) ^ 1;
	out[3] = device_digest(S.delayMask, N * 8, m_stream);
	out[4] = device_digest(S.rcmPtr, (N + 1) * 8, m_stream);
	out[5] = S.stdp ? device_digest(S.rcmSrc, P * 4, m_stream) : 0;
	out[6] = S.stdp ? device_digest(S.rcmFwd, P * 4, m_stream) : 0;
	out[7] = S.stdp ? device_digest(S.rcmSlice, (size_t) (S.applySlices + 1) * N * 4, m_stream) : 0;
	out[8] = m_dlvGroups;
	out[9] = m_builtOnDevice ? 1 : 0;
}

/* src/nemo/ConnectivityMatrix.cpp:298-331 */
const std::vector<uint64_t>& Simulation::getSynapsesFrom(unsigned source)
{
	if(m_writeOnly) NB_THROW(NEMO_INVALID_INPUT, "Cannot read synapse state if simulation configured with write-only synapses");
	auto it = m_g2l[0].find(source);
	if(it == m_g2l[0].end()) NB_THROW(NEMO_INVALID_INPUT, "Non-existing source neuron id (%u) in synapse id query", source);
	ensureQueryTables();
	uint64_t n = m_srcStart[it->second + 1] - m_srcStart[it->second];
	m_queried.resize(n);
	for(uint64_t i = 0; i < n; ++i) m_queried[i] = ((uint64_t) source << 32) | i;
	return m_queried;
}

/* ConnectivityMatrix::axonTerminalAux (src/nemo/ConnectivityMatrix.cpp:343-360) */
size_t Simulation::synapseKey(uint64_t id)
{
	if(m_writeOnly) NB_THROW(NEMO_INVALID_INPUT, "Cannot read synapse state if simulation configured with write-only synapses");
	ensureQueryTables();
	unsigned source = (unsigned) (id >> 32);
	uint32_t s = (uint32_t) (id & 0xffffffffu);
	auto it = m_g2l[0].find(source);
	if(it == m_g2l[0].end() || m_srcStart[it->second + 1] == m_srcStart[it->second]) {
		NB_THROW(NEMO_INVALID_INPUT, "Non-existing neuron id (%u) in synapse query", source);
	}
	uint64_t n = m_srcStart[it->second + 1] - m_srcStart[it->second];
	if(s >= n) NB_THROW(NEMO_UNKNOWN_ERROR, "synapse index %u out of range for neuron %u", s, source);
	return m_srcOrder[m_srcStart[it->second] + s];
}

unsigned Simulation::getSynapseTarget(uint64_t id) { return m_synTarget[synapseKey(id)]; }
unsigned Simulation::getSynapseDelay(uint64_t id) { return m_synDelay[synapseKey(id)]; }
unsigned char Simulation::getSynapsePlastic(uint64_t id) { return m_synPlastic[synapseKey(id)]; }

float Simulation::getSynapseWeight(uint64_t id)
{
	size_t k = synapseKey(id);
	uint32_t w = 0;
	NB_CUDA(cudaSetDevice(m_device));
	NB_CUDA(cudaMemcpyAsync(&w, m_dev.synW + m_pos[k], 4, cudaMemcpyDeviceToHost, m_stream));
	sync();
	return fx_toFloat((int32_t) w);
}

void Simulation::getWeightsFx(int32_t* out, size_t cap, size_t* len)
{
	if(m_writeOnly) NB_THROW(NEMO_INVALID_INPUT, "Cannot read synapse state if simulation configured with write-only synapses");
	if(cap < m_nsyn) NB_THROW(NEMO_BUFFER_OVERFLOW, "weight buffer too small");
	ensureQueryTables();
	std::vector<uint32_t> w(m_nsyn);
	NB_CUDA(cudaSetDevice(m_device));
	NB_CUDA(cudaMemcpyAsync(w.data(), m_dev.synW, m_nsyn * 4, cudaMemcpyDeviceToHost, m_stream));
	sync();
	// network iteration order: sources by ascending global id
	std::vector<unsigned> sources(m_N);
	for(unsigned l = 0; l < m_N; ++l) sources[l] = l;
	std::sort(sources.begin(), sources.end(), [&](unsigned a, unsigned b) { return m_l2g[a] < m_l2g[b]; });
	size_t o = 0;
	for(unsigned l : sources) {
		for(uint64_t j = m_srcStart[l]; j < m_srcStart[l + 1]; ++j) {
			out[o++] = (int32_t) w[m_pos[m_srcOrder[j]]];
		}
	}
	*len = o;
}

void Simulation::getTypeState(unsigned netType, float* out, size_t cap, size_t* len)
{
	getNetTypeState(0, netType, out, cap, len);
}

void Simulation::getNetTypeState(unsigned net, unsigned netType, float* out, size_t cap, size_t* len)
{
	if(net >= m_nets) NB_THROW(NEMO_INVALID_INPUT, "Invalid network index %u", net);
	*len = 0;
	if(netType >= m_netTypes[net].size()) return;
	const NetTypeRange& r = m_netTypes[net][netType];
	if(r.count == 0) return;
	const HostType& t = m_types[r.hostType];
	size_t n = (size_t) r.count * t.desc.nstate;
	if(cap < n) NB_THROW(NEMO_BUFFER_OVERFLOW, "state buffer too small");
	NB_CUDA(cudaSetDevice(m_device));
	for(unsigned v = 0; v < t.desc.nstate; ++v) {
		NB_CUDA(cudaMemcpyAsync(out + (size_t) v * r.count, currentState(t) + (size_t) v * t.n + r.offset,
				(size_t) r.count * 4, cudaMemcpyDeviceToHost, m_stream));
	}
	sync();
	*len = n;
}

unsigned long Simulation::elapsedWallclock() const
{
	auto d = std::chrono::steady_clock::now() - m_timerStart;
	return (unsigned long) std::chrono::duration_cast<std::chrono::milliseconds>(d).count();
}

void Simulation::resetTimer()
{
	m_timerStart = std::chrono::steady_clock::now();
	m_timerSteps = 0;
}

} // namespace nemo_b200
