// kernels.cuh -- sm_100a kernels of the simulation step.
//
// One launch of step_kernel advances the whole network by one millisecond.
// It fuses what the reference does in four passes
// (src/nemo/cpu/Simulation.cpp:94-111 on the CPU; gather, update, scatter and
// updateStdp kernels on the reference CUDA backend):
//
//   1. current read-out: each neuron reads its (E, I) 64-bit fixed-point sums
//      for this step from the accumulator slot ring and clears them;
//   2. neuron update: the type's plugin arithmetic, in the reference's
//      operation order with IEEE-rounded intrinsics (no contraction);
//   3. firing bookkeeping: the history word, the fired bit-vector, and a
//      ballot/popc compaction of the CTA's fired neurons into shared memory;
//   4. spike scatter: the CTA's warps stream the fired neurons' outgoing
//      synapses (pre-sorted by delay, 8 bytes each) and add every weight into
//      the accumulator slot of the step at which it arrives, with 64-bit
//      integer atomics (order-independent, hence bit-exact);
//   5. STDP accumulation for the previous step (the reference does it at the
//      end of the same step; it only needs the previous step's history, which
//      the double-buffered history keeps intact).
//
// Scattering at firing time instead of gathering at arrival time makes one
// kernel boundary per step sufficient.  It delivers the weight a synapse has
// when the spike is emitted; applyStdp compensates in-flight spikes of every
// synapse whose weight it changes, so the arrival-time weight is what is
// delivered, as in the reference.
#pragma once

#include "simulation.hpp"

namespace nemo_b200 {

// wfx_toFloat with saturation (src/nemo/fixedpoint.cpp:40-49)
__device__ __forceinline__ float wfx_to_float(long long v)
{
	v = v > (long long) INT32_MAX ? (long long) INT32_MAX : v;
	v = v < (long long) INT32_MIN ? (long long) INT32_MIN : v;
	return __fdiv_rn(__ll2float_rn(v), 1048576.0f);
}

// x86-64 float -> unsigned conversion (via a truncating 64-bit convert)
__device__ __forceinline__ uint32_t x86_f2u32(float x)
{
	if(!(x > -9.2233720368547758e18f && x < 9.2233720368547758e18f)) return 0u;
	return (uint32_t) (unsigned long long) __float2ll_rz(x);
}

// StdpProcess::updateRegion / weightChange (src/nemo/StdpProcess.cpp:68-124)
__device__ __forceinline__ int32_t stdp_region(const StdpParams& sp, uint64_t x)
{
	if(!x) return 0;
	const uint32_t NONE = ~0u;
	uint64_t vpre = x & sp.prePostBits;
	uint32_t dtPre = vpre ? (uint32_t) (__ffsll((long long) (vpre >> (sp.npost & 63))) - 1) : NONE;
	uint64_t vpost = x & sp.postPreBits;
	uint32_t dtPost = vpost ? (uint32_t) __clzll((long long) (vpost << ((64 - sp.npost) & 63))) : NONE;
	if(dtPre < dtPost) return sp.fnPre[dtPre];
	if(dtPost < dtPre) return sp.fnPost[dtPost];
	return 0;
}

__device__ __forceinline__ int32_t stdp_weight_change(const StdpParams& sp, uint64_t pre)
{
	return (int32_t) ((uint32_t) stdp_region(sp, pre & sp.potBits) + (uint32_t) stdp_region(sp, pre & sp.depBits));
}

// StdpProcess::updatedWeight (src/nemo/StdpProcess.cpp:128-138)
__device__ __forceinline__ int32_t stdp_updated_weight(const StdpParams& sp, int32_t w, int32_t dw)
{
	int32_t sum = (int32_t) ((uint32_t) w + (uint32_t) dw);
	if(w > 0) return min(sp.maxE, max(sum, sp.minE));
	if(w < 0) return min(sp.minI, max(sum, sp.maxI));
	return 0;
}

// fx_mul (src/nemo/fixedpoint.hpp:41-46)
__device__ __forceinline__ int32_t fx_mul_dev(int32_t a, int32_t b)
{
	return (int32_t) (((long long) a * (long long) b) >> FRACTIONAL_BITS);
}

// Fixed-point input sums.  The reference sums E (w >= 0) and I (w < 0)
// contributions in int64 and clamps once (src/nemo/cpu/Simulation.cpp:297-300,
// src/nemo/fixedpoint.cpp:40-49).  Here each (step slot, neuron) keeps the
// low 32 bits of E and of -I in an 8-byte word pair, so the accumulator ring
// fits in L2; a carry out of (or borrow into) a low word, detected from the
// value the atomic returns, is added to a signed high-word counter of the
// same (slot, neuron), and the slot is flagged.  The exact int64 sum is
// high * 2^32 + low, independent of the order of the atomics.
__device__ __forceinline__ void acc_add(const DevSim& S, uint32_t sl, uint32_t n, uint32_t cls, int64_t delta)
{
	const size_t i = (size_t) sl * S.N + n;
	uint32_t* lo = reinterpret_cast<uint32_t*>(S.slots + i) + cls;
	const uint32_t d = (uint32_t) delta;
	const uint32_t old = atomicAdd(lo, d);
	const uint32_t now = old + d;
	const bool wrap = delta >= 0 ? now < old : now > old;
	if(wrap) {
		atomicAdd(reinterpret_cast<int*>(S.slotHigh + i) + cls, delta >= 0 ? 1 : -1);
		S.slotFlag[sl] = 1u;
	}
}

// one synaptic weight arriving in slot sl at neuron n
__device__ __forceinline__ void add_current(const DevSim& S, uint32_t sl, uint32_t n, int32_t w)
{
	if(w >= 0) acc_add(S, sl, n, 0, (int64_t) w);
	else acc_add(S, sl, n, 1, -(int64_t) w);
}

// Izhikevich, src/nemo/cpu/plugins/Izhikevich.cpp:53-94: the v update is
// evaluated in double (0.04, 5.0 and 140.0 are double literals there), u in
// float; both round exactly as the x86-64 SSE build does.
__device__ __forceinline__ bool update_izhikevich(const DevSim& S, const TypeRange& T, uint32_t nl, uint32_t n,
		float cE, float cI, float ext, bool fs)
{
	const float* P = T.param;
	float* X = T.state;
	const uint32_t nn = T.n;
	float I = __fadd_rn(__fadd_rn(cE, cI), ext);
	float sigma = P[4 * nn + nl];
	if(sigma != 0.0f) {
		uint32_t s0 = S.rng[n], s1 = S.rng[S.N + n], s2 = S.rng[2 * S.N + n], s3 = S.rng[3 * S.N + n];
		I = __fadd_rn(I, __fmul_rn(sigma, nb_nrand(S.calib, s0, s1, s2, s3)));
		S.rng[n] = s0; S.rng[S.N + n] = s1; S.rng[2 * S.N + n] = s2; S.rng[3 * S.N + n] = s3;
	}
	float a = P[nl], b = P[nn + nl];
	float u = X[nl], v = X[nn + nl];
	const double dI = (double) I;
	bool fired = false;
#pragma unroll
	for(int k = 0; k < 4; ++k) {
		if(!fired) {
			double vd = (double) v;
			double t = __dadd_rn(__dmul_rn(0.04, vd), 5.0);
			t = __dadd_rn(__dmul_rn(t, vd), 140.0);
			t = __dsub_rn(t, (double) u);
			t = __dadd_rn(t, dI);
			v = __double2float_rn(__dadd_rn(vd, __dmul_rn(0.25, t)));
			u = __fadd_rn(u, __fmul_rn(0.25f, __fmul_rn(a, __fsub_rn(__fmul_rn(b, v), u))));
			fired = v >= 30.0f;
		}
	}
	fired = fired || fs;
	if(fired) {
		v = P[2 * nn + nl];
		u = __fadd_rn(u, P[3 * nn + nl]);
	}
	X[nl] = u;
	X[nn + nl] = v;
	return fired;
}

// IF_curr_exp, src/nemo/cpu/plugins/IF_curr_exp.cpp:74-121 with the header
// parameter order (src/nemo/plugins/IF_curr_exp.h:4-20).
__device__ __forceinline__ bool update_if_curr_exp(const TypeRange& T, uint32_t nl,
		float cE, float cI, float ext, bool fs)
{
	const float* P = T.param;
	float* X = T.state;
	const uint32_t nn = T.n;
	float v_rest = P[nl], v_reset = P[nn + nl], c_m = P[2 * nn + nl], tau_m = P[3 * nn + nl];
	float tau_refrac = P[4 * nn + nl], tau_E = P[5 * nn + nl], tau_I = P[6 * nn + nl];
	float v_thresh = P[7 * nn + nl], i_offset = P[8 * nn + nl];
	float Ie = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, __fdiv_rn(1.0f, tau_E)), X[nn + nl]), cE);
	float Ii = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, __fdiv_rn(1.0f, tau_I)), X[2 * nn + nl]), cI);
	float I = __fadd_rn(__fadd_rn(__fadd_rn(Ie, Ii), ext), i_offset);
	X[nn + nl] = Ie;
	X[2 * nn + nl] = Ii;
	float v = X[nl];
	float lastfired = X[3 * nn + nl];
	bool refractory = lastfired <= tau_refrac;
	if(!refractory) {
		v = __fadd_rn(v, __fadd_rn(__fdiv_rn(I, c_m), __fdiv_rn(__fsub_rn(v_rest, v), tau_m)));
	}
	bool fired = (!refractory && v > v_thresh) || fs;
	if(fired) {
		X[3 * nn + nl] = 1.0f;
		X[nl] = v_reset;
	} else {
		X[3 * nn + nl] = __fadd_rn(lastfired, 1.0f);
		X[nl] = v;
	}
	return fired;
}

// PoissonSource, src/nemo/cpu/plugins/PoissonSource.cpp:6-30
__device__ __forceinline__ bool update_poisson(const DevSim& S, const TypeRange& T, uint32_t nl, uint32_t n, bool fs)
{
	uint32_t p0 = x86_f2u32(__fmul_rn(T.param[nl], 65536.0f));
	uint32_t s0 = S.rng[n], s1 = S.rng[S.N + n], s2 = S.rng[2 * S.N + n], s3 = S.rng[3 * S.N + n];
	uint32_t p1 = nb_urand(s0, s1, s2, s3) & 0xffffu;
	S.rng[n] = s0; S.rng[S.N + n] = s1; S.rng[2 * S.N + n] = s2; S.rng[3 * S.N + n] = s3;
	return p1 < p0 || fs;
}

// A weight that applyStdp changes was already scattered, with its old value,
// for the spikes its source emitted k < delay steps before the last step and
// that have not arrived yet.  The reference reads the weight on arrival
// (deliverSpikesOne, src/nemo/cpu/Simulation.cpp:293-307), so move each such
// contribution from the old weight's class (E if >= 0, else I) to the new
// weight's class with the new value.
__device__ __forceinline__ void compensate_inflight(const DevSim& S, const uint64_t* hist, uint32_t sd,
		uint32_t tgt, uint32_t slot, int32_t w, int32_t nw)
{
	const uint32_t src = sd & (MAX_NEURONS - 1);
	const uint32_t delay = (sd >> 26) + 1;
	uint64_t inflight = hist[src] & ((delay >= 64) ? ~0ull : ((1ull << delay) - 1ull));
	while(inflight) {
		const uint32_t k = __ffsll((long long) inflight) - 1;
		inflight &= inflight - 1;
		// emitted k steps before the last step, arrives delay - k steps after it
		const uint32_t sl = (slot + delay - k) % S.D;
		if(w >= 0) acc_add(S, sl, tgt, 0, -(int64_t) w);
		else acc_add(S, sl, tgt, 1, (int64_t) w);
		add_current(S, sl, tgt, nw);
	}
}

} // namespace nemo_b200
