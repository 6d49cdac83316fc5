// kernels.cuh -- device functions of the simulation step (sm_100a): the
// fixed-point and STDP arithmetic of the reference and the neuron-type
// plugins.  The step's phases (delivery at arrival, neuron update, STDP
// accumulation) are the kernels of simulation.cu.
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

// The neuron-type plugins, each split into a load of the neuron's
// parameters, state and RNG words into registers, the update arithmetic on
// those registers, and the store of what changed.  The step issues every
// load of a neuron before its first store, so that none of them waits for
// another.
struct NeuronRegs {
	float p[9];     // parameters
	float x[4];     // state
	uint32_t r[4];  // xorshift words
	float noise;    // this step's nrand, when precomputed (pre)
	bool pre;
};

__device__ __forceinline__ void load_rng(const DevSim& S, uint32_t n, NeuronRegs& R)
{
	R.r[0] = S.rng[n];
	R.r[1] = S.rng[S.N + n];
	R.r[2] = S.rng[2 * S.N + n];
	R.r[3] = S.rng[3 * S.N + n];
}

__device__ __forceinline__ void store_rng(const DevSim& S, uint32_t n, const NeuronRegs& R)
{
	S.rng[n] = R.r[0];
	S.rng[S.N + n] = R.r[1];
	S.rng[2 * S.N + n] = R.r[2];
	S.rng[3 * S.N + n] = R.r[3];
}

// parameters and state of neuron nl of type T (the plugin layouts of
// src/nemo/plugins/Izhikevich.h, IF_curr_exp.h, PoissonSource.h)
// With pre, an Izhikevich neuron's nrand for this step was computed (and its
// RNG words advanced) by precompute_noise before the update.
__device__ __forceinline__ void load_neuron(const DevSim& S, const TypeRange& T, uint32_t nl, uint32_t n, NeuronRegs& R,
		bool pre)
{
	const float* P = T.param;
	const float* X = T.state;
	const uint32_t nn = T.n;
	R.pre = pre;
	switch(T.kind) {
		case KIND_IZHIKEVICH:
#pragma unroll
			for(int k = 0; k < 5; ++k) R.p[k] = P[k * nn + nl];  // a, b, c, d, sigma
			R.x[0] = X[nl];       // u
			R.x[1] = X[nn + nl];  // v
			if(pre) R.noise = S.noise[n];
			else load_rng(S, n, R);
			break;
		case KIND_IF_CURR_EXP:
#pragma unroll
			for(int k = 0; k < 9; ++k) R.p[k] = P[k * nn + nl];
#pragma unroll
			for(int k = 0; k < 4; ++k) R.x[k] = X[k * nn + nl];  // v, Ie, Ii, lastfired
			break;
		case KIND_POISSON:
			R.p[0] = P[nl];  // rate
			load_rng(S, n, R);
			break;
		case KIND_IZHIKEVICH_RS:
			R.x[0] = X[nl];       // u
			R.x[1] = X[nn + nl];  // v
			break;
		default:
			break;
	}
}

// Izhikevich, src/nemo/cpu/plugins/Izhikevich.cpp:53-94: the v update is
// evaluated in double (0.04, 5.0 and 140.0 are double literals there), u in
// float; both round exactly as the x86-64 SSE build does.
__device__ __forceinline__ bool update_izhikevich(const LibmCalib& calib, NeuronRegs& R, float cE, float cI, float ext,
		bool fs)
{
	const float a = R.p[0], b = R.p[1], sigma = R.p[4];
	float I = __fadd_rn(__fadd_rn(cE, cI), ext);
	if(sigma != 0.0f) {
		// the update's own draw (two-launch step: many neurons per thread,
		// bound by instruction issue) reads the libm results from the
		// tables; precompute_noise (one neuron per thread in the shadow of a
		// barrier, bound by latency) evaluates them, which is faster there
		// and keeps the tables out of L2.  Both give the same bits.
		const float z = R.pre ? R.noise : nb_nrand_table(calib, R.r[0], R.r[1], R.r[2], R.r[3]);
		I = __fadd_rn(I, __fmul_rn(sigma, z));
	}
	float u = R.x[0], v = R.x[1];
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
		v = R.p[2];
		u = __fadd_rn(u, R.p[3]);
	}
	R.x[0] = u;
	R.x[1] = v;
	return fired;
}

// IF_curr_exp, src/nemo/cpu/plugins/IF_curr_exp.cpp:74-121 with the header
// parameter order (src/nemo/plugins/IF_curr_exp.h:4-20).
__device__ __forceinline__ bool update_if_curr_exp(NeuronRegs& R, float cE, float cI, float ext, bool fs)
{
	const float v_rest = R.p[0], v_reset = R.p[1], c_m = R.p[2], tau_m = R.p[3];
	const float tau_refrac = R.p[4], tau_E = R.p[5], tau_I = R.p[6];
	const float v_thresh = R.p[7], i_offset = R.p[8];
	const float Ie = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, __fdiv_rn(1.0f, tau_E)), R.x[1]), cE);
	const float Ii = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, __fdiv_rn(1.0f, tau_I)), R.x[2]), cI);
	const float I = __fadd_rn(__fadd_rn(__fadd_rn(Ie, Ii), ext), i_offset);
	R.x[1] = Ie;
	R.x[2] = Ii;
	float v = R.x[0];
	const float lastfired = R.x[3];
	const bool refractory = lastfired <= tau_refrac;
	if(!refractory) {
		v = __fadd_rn(v, __fadd_rn(__fdiv_rn(I, c_m), __fdiv_rn(__fsub_rn(v_rest, v), tau_m)));
	}
	const bool fired = (!refractory && v > v_thresh) || fs;
	if(fired) {
		R.x[3] = 1.0f;
		R.x[0] = v_reset;
	} else {
		R.x[3] = __fadd_rn(lastfired, 1.0f);
		R.x[0] = v;
	}
	return fired;
}

// IzhikevichRS, the reference's CUDA plugin (it has no CPU plugin),
// src/nemo/cuda/plugins/IzhikevichRS.cu:76-116: the Izhikevich update in
// float with a = 0.02, b = 0.2, c = -65, d = 8 built in and no input noise,
// in source order without contraction.
__device__ __forceinline__ bool update_izhikevich_rs(NeuronRegs& R, float cE, float cI, float ext, bool fs)
{
	const float a = 0.02f, b = 0.2f;
	const float I = __fadd_rn(__fadd_rn(cE, cI), ext);
	float u = R.x[0], v = R.x[1];
	bool fired = false;
#pragma unroll
	for(int k = 0; k < 4; ++k) {
		if(!fired) {
			float t = __fadd_rn(__fmul_rn(0.04f, v), 5.0f);
			t = __fadd_rn(__fmul_rn(t, v), 140.0f);
			t = __fadd_rn(__fsub_rn(t, u), I);
			v = __fadd_rn(v, __fmul_rn(0.25f, t));
			u = __fadd_rn(u, __fmul_rn(0.25f, __fmul_rn(a, __fsub_rn(__fmul_rn(b, v), u))));
			fired = v >= 30.0f;
		}
	}
	fired = fired || fs;
	if(fired) {
		v = -65.0f;
		u = __fadd_rn(u, 8.0f);
	}
	R.x[0] = u;
	R.x[1] = v;
	return fired;
}

// PoissonSource, src/nemo/cpu/plugins/PoissonSource.cpp:6-30
__device__ __forceinline__ bool update_poisson(NeuronRegs& R, bool fs)
{
	const uint32_t p0 = x86_f2u32(__fmul_rn(R.p[0], 65536.0f));
	const uint32_t p1 = nb_urand(R.r[0], R.r[1], R.r[2], R.r[3]) & 0xffffu;
	return p1 < p0 || fs;
}

// Kuramoto oscillators, src/nemo/cpu/plugins/Kuramoto.cpp:78-124
// (src/nemo/plugins/Kuramoto.h): parameter the frequency, state the phase,
// kept for the last 32 cycles (T.state is [32][n]).  One fourth-order
// Runge-Kutta step of the phase; each stage sums, over the target's
// incoming synapses, weight x sin(source phase at emission - target phase),
// the source phase being the one at cycle - (delay - 1).  The neuron never
// fires and ignores stimulus and synaptic current.  sinf is CUDA's, which
// is within an ulp or two of the host libm's but not equal to it, so the
// phases agree with the CPU plugin to a tolerance, not bit for bit.
// b, e: the neuron's range of the all-synapse reverse matrix (sources as
// source | (delay - 1) << 26, weights); base, nn: the type's first local
// index and size; cycle: this step's.
__device__ __forceinline__ bool update_kuramoto(const float* param, float* state, uint32_t base, uint32_t nn,
		uint32_t nl, const uint32_t* allSrc, const float* allW, unsigned long long b, unsigned long long e,
		uint32_t cycle)
{
	constexpr uint32_t H = 32;
	const float f = param[nl];
	const float phase0 = state[(size_t) (cycle % H) * nn + nl];
	auto coupling = [&](float targetPhase) {
		float sum = 0.0f;
		for(unsigned long long p = b; p < e; ++p) {
			const uint32_t sd = allSrc[p];
			const uint32_t delay = (sd >> 26) + 1;
			const uint32_t src = (sd & (MAX_NEURONS - 1)) - base;
			const float sp = state[(size_t) ((cycle - (delay - 1)) % H) * nn + src];
			sum = __fadd_rn(sum, __fmul_rn(allW[p], sinf(__fsub_rn(sp, targetPhase))));
		}
		return sum;
	};
	const float k0 = __fadd_rn(f, coupling(phase0));
	const float k1 = __fadd_rn(f, coupling(__fadd_rn(phase0, __fmul_rn(k0, 0.5f))));
	const float k2 = __fadd_rn(f, coupling(__fadd_rn(phase0, __fmul_rn(k1, 0.5f))));
	const float k3 = __fadd_rn(f, coupling(__fadd_rn(phase0, k2)));
	const float sum = __fadd_rn(__fadd_rn(__fadd_rn(k0, __fmul_rn(2.0f, k1)), __fmul_rn(2.0f, k2)), k3);
	const float phase = __fadd_rn(phase0, __fdiv_rn(sum, 6.0f));
	// fmodf by 2 pi rounded to float, plus 2 pi in double for a negative
	// phase, rounded once to float (the plugin's C expression)
	const double wrapped = (double) fmodf(phase, 6.2831855f) + (phase < 0.0f ? 6.283185307179586 : 0.0);
	state[(size_t) ((cycle + 1) % H) * nn + nl] = __double2float_rn(wrapped);
	return false;
}

// One step of neuron nl (local index n) of type T; returns whether it fired.
__device__ __forceinline__ bool update_neuron(const DevSim& S, const TypeRange& T, NeuronRegs& R, float cE, float cI,
		float ext, bool fs)
{
	switch(T.kind) {
		case KIND_IZHIKEVICH: return update_izhikevich(S.calib, R, cE, cI, ext, fs);
		case KIND_IF_CURR_EXP: return update_if_curr_exp(R, cE, cI, ext, fs);
		case KIND_POISSON: return update_poisson(R, fs);
		case KIND_IZHIKEVICH_RS: return update_izhikevich_rs(R, cE, cI, ext, fs);
		default: return fs;  // Input, src/nemo/cpu/plugins/Input.cpp:17-22
	}
}

// the state and RNG words that update_neuron changed
__device__ __forceinline__ void store_neuron(const DevSim& S, const TypeRange& T, uint32_t nl, uint32_t n,
		const NeuronRegs& R)
{
	float* X = T.state;
	const uint32_t nn = T.n;
	switch(T.kind) {
		case KIND_IZHIKEVICH:
			X[nl] = R.x[0];
			X[nn + nl] = R.x[1];
			if(R.p[4] != 0.0f && !R.pre) store_rng(S, n, R);
			break;
		case KIND_IF_CURR_EXP:
#pragma unroll
			for(int k = 0; k < 4; ++k) X[k * nn + nl] = R.x[k];
			break;
		case KIND_POISSON:
			store_rng(S, n, R);
			break;
		case KIND_IZHIKEVICH_RS:
			X[nl] = R.x[0];
			X[nn + nl] = R.x[1];
			break;
		default:
			break;
	}
}

// Staging of precompute_noise's inputs in shared memory: each thread copies
// the RNG words and sigma of neuron first + threadIdx.x (an Izhikevich
// neuron) with asynchronous copies that complete while the pre-phase runs
// (a CTA with at most NOISE_STAGE neurons of one partition).
constexpr uint32_t NOISE_STAGE = RUN_THREADS;

__device__ __forceinline__ void cp_async4(void* dst, const void* src)
{
	const uint32_t d = (uint32_t) __cvta_generic_to_shared(dst);
	asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" :: "r"(d), "l"(src) : "memory");
}

__device__ __forceinline__ void stage_noise_inputs(const DevSim& S, uint32_t first, uint32_t last, uint32_t* sRng,
		float* sSigma)
{
	const uint32_t n = first + threadIdx.x;
	if(n < last) {
		uint32_t k = 0;
		while(k + 1 < S.ntypes && n >= S.types[k + 1].base) ++k;
		const TypeRange& T = S.types[k];
		if(T.kind == KIND_IZHIKEVICH) {
			cp_async4(sSigma + threadIdx.x, T.param + 4 * T.n + (n - T.base));
#pragma unroll
			for(uint32_t j = 0; j < 4; ++j) cp_async4(sRng + j * NOISE_STAGE + threadIdx.x, S.rng + j * S.N + n);
		}
	}
	asm volatile("cp.async.commit_group;" ::: "memory");
}

// precompute_noise from the staged inputs (after cp.async.wait_all and a
// CTA barrier)
__device__ __forceinline__ void precompute_noise_staged(const DevSim& S, uint32_t first, uint32_t last,
		const uint32_t* sRng, const float* sSigma)
{
	const uint32_t n = first + threadIdx.x;
	if(n >= last) return;
	uint32_t k = 0;
	while(k + 1 < S.ntypes && n >= S.types[k + 1].base) ++k;
	if(S.types[k].kind != KIND_IZHIKEVICH || sSigma[threadIdx.x] == 0.0f) return;
	NeuronRegs R;
#pragma unroll
	for(uint32_t j = 0; j < 4; ++j) R.r[j] = sRng[j * NOISE_STAGE + threadIdx.x];
	S.noise[n] = nb_nrand<true>(S.calib, R.r[0], R.r[1], R.r[2], R.r[3]);
	store_rng(S, n, R);
}

// nrand of the coming update for the Izhikevich neurons [first, last) of a
// CTA with sigma != 0 (the same draws the update would make, in the same
// order), for the update's pre flag.
__device__ __forceinline__ void precompute_noise(const DevSim& S, uint32_t first, uint32_t last)
{
	for(uint32_t n = first + threadIdx.x; n < last; n += blockDim.x) {
		uint32_t k = 0;
		while(k + 1 < S.ntypes && n >= S.types[k + 1].base) ++k;
		const TypeRange& T = S.types[k];
		if(T.kind != KIND_IZHIKEVICH) continue;
		const uint32_t nl = n - T.base;
		// the RNG words load alongside sigma
		NeuronRegs R;
		load_rng(S, n, R);
		if(T.param[4 * T.n + nl] == 0.0f) continue;
		S.noise[n] = nb_nrand<true>(S.calib, R.r[0], R.r[1], R.r[2], R.r[3]);
		store_rng(S, n, R);
	}
}

} // namespace nemo_b200
