// bptt.cu -- differentiable mode: a network of Izhikevich neurons with
// delayed synapses, run forward with checkpoints and differentiated by a
// hand-written backpropagation-through-time adjoint.
//
// Model (per trial b, neuron n, millisecond t; 4 Euler sub-steps per ms as
// in src/nemo/cpu/plugins/Izhikevich.cpp, with a reset after every sub-step
// so that the sub-step chain is differentiable):
//   I(t)  = sum over in-synapses (j, w, d) of w * S_j(t - d)  +  noise(t)
//   sub-step k = 0..3:
//     v1 = v + 1/4 (0.04 v^2 + 5 v + 140 - u + I)
//     u1 = u + 1/4 a (b v1 - u)
//     s  = H(v1 - 30)             (hard)   or  f(v1 - 30)  (smooth)
//     v  = v1 + s (c - v1);  u = u1 + s d;  S(t) += s
//   r(t) = alpha r(t-1) + S(t) for the R readout neurons, alpha = exp(-1/20)
//   loss = sum_t,b,n<R (r - target)^2 / (T R B)
// f(x) = 1/2 (1 + kx / (1 + k|x|)) is the fast sigmoid with slope k = 10,
// and g(x) = f'(x) = k / (2 (1 + k|x|)^2) is the surrogate derivative used
// for H in the backward pass.  Initial state v = -65, u = b v.
//
// Every kernel is a template over the state type Real (float or double):
// the caller's weights, parameters, noise, targets, loss and gradients are
// float32 either way; Real is the type of the neuron state, the stored
// trajectories and the adjoints.  Gradients of this model are sensitive to
// rounding (the spike upstroke amplifies a state perturbation many times
// over), so float32 state gives gradients within about 1e-2 of the exact
// ones, while float64 state reproduces a float64 evaluation.
//
// Layouts: spikes S and input adjoints lambda_I as [n][t][b]; states [n][b];
// noise and targets as PyTorch tensors [T][B][N] and [T][B][R].  One thread
// per (neuron, trial); the 16 trials of one neuron are contiguous.
// Checkpoints of (v, u) every `ckpt` ms; the backward pass replays each
// segment from its checkpoint and keeps the per-ms start states and synaptic
// inputs of that segment.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/nemo_b200.h"
#include "bptt.hpp"
#include "common.hpp"

namespace nemo_b200 {

#define BP_CUDA(call)                                                              \
	do {                                                                           \
		cudaError_t err_ = (call);                                                 \
		if(err_ != cudaSuccess) {                                                  \
			NB_THROW(NEMO_CUDA_ERROR, "CUDA error %s at %s:%d", cudaGetErrorString(err_), __FILE__, __LINE__); \
		}                                                                          \
	} while(0)

template<typename Real>
__device__ __forceinline__ Real spike_fn(Real x, int smooth)
{
	const Real k = Real(10);
	if(smooth) return Real(0.5) * (Real(1) + k * x / (Real(1) + k * fabs(x)));
	return x >= Real(0) ? Real(1) : Real(0);
}

template<typename Real>
__device__ __forceinline__ Real spike_grad(Real x)
{
	const Real q = Real(1) + Real(10) * fabs(x);
	return Real(0.5) * Real(10) / (q * q);
}

// Sum over the range [beg, end) of one neuron's synapses of w * x, with x
// the value term(e) returns (0 when the term does not apply), in G
// interleaved partial sums so that G terms' loads are in flight at once.
// The forward pass and the replay call it with the same arguments, so they
// agree bit for bit.
constexpr int GATHER = 4;

template<typename Real, typename Term>
__device__ __forceinline__ Real gather(int beg, int end, Term term)
{
	Real sum[GATHER], w[GATHER], x[GATHER];
#pragma unroll
	for(int j = 0; j < GATHER; ++j) sum[j] = Real(0);
	int e = beg;
	for(; e + GATHER <= end; e += GATHER) {
#pragma unroll
		for(int j = 0; j < GATHER; ++j) term(e + j, w[j], x[j]);
#pragma unroll
		for(int j = 0; j < GATHER; ++j) sum[j] = fma(w[j], x[j], sum[j]);
	}
	for(; e < end; ++e) {
		term(e, w[0], x[0]);
		sum[0] = fma(w[0], x[0], sum[0]);
	}
#pragma unroll
	for(int h = GATHER / 2; h > 0; h /= 2) {
#pragma unroll
		for(int j = 0; j < h; ++j) sum[j] += sum[j + h];
	}
	return sum[0];
}

// synaptic input of (n, b) at ms t from the stored spikes
template<typename Real>
__device__ __forceinline__ Real syn_input(const BpttDev& D, const BpttState<Real>& X, const float* W, int n, int b, int t)
{
	return gather<Real>(D.inStart[n], D.inStart[n + 1], [&](int e, Real& w, Real& x) {
		const int dl = D.inDelay[e];
		w = (Real) W[D.inSyn[e]];
		x = t >= dl ? X.S[((size_t) D.inSrc[e] * D.T + (t - dl)) * D.B + b] : Real(0);
	});
}

// one Euler sub-step and its reset; returns s
template<typename Real>
__device__ __forceinline__ Real substep(Real& v, Real& u, Real& v1, Real I, Real a, Real b, Real c, Real d, int smooth)
{
	v1 = v + Real(0.25) * (Real(0.04) * v * v + Real(5) * v + Real(140) - u + I);
	const Real u1 = u + Real(0.25) * a * (b * v1 - u);
	const Real s = spike_fn(v1 - Real(30), smooth);
	v = v1 + s * (c - v1);
	u = u1 + s * d;
	return s;
}

// the four sub-steps of one ms; returns S(t)
template<typename Real>
__device__ __forceinline__ Real substeps(Real& v, Real& u, Real I, Real a, Real b, Real c, Real d, int smooth)
{
	Real St = Real(0), v1;
#pragma unroll
	for(int k = 0; k < 4; ++k) St += substep(v, u, v1, I, a, b, c, d, smooth);
	return St;
}

template<typename Real>
__global__ void bptt_init_kernel(BpttDev D, BpttState<Real> X, BpttParams P)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= D.N * D.B) return;
	const int n = i / D.B, b = i % D.B;
	X.v[i] = Real(-65);
	X.u[i] = (Real) P.b[n] * Real(-65);
	X.lossPart[i] = Real(0);
	if(n < D.R) X.r[n * D.B + b] = Real(0);
}

// forward: one ms for every (neuron, trial)
template<typename Real>
__global__ void bptt_forward_kernel(BpttDev D, BpttState<Real> X, BpttParams P, int t)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= D.N * D.B) return;
	const int n = i / D.B, b = i % D.B;
	Real v = X.v[i], u = X.u[i];
	if(t % D.ckpt == 0) {
		const size_t k = (size_t) (t / D.ckpt) * D.N * D.B + i;
		X.ckV[k] = v;
		X.ckU[k] = u;
	}
	const Real I = syn_input(D, X, P.W, n, b, t) + (Real) P.noise[((size_t) t * D.B + b) * D.N + n];
	const Real St = substeps(v, u, I, (Real) P.a[n], (Real) P.b[n], (Real) P.c[n], (Real) P.d[n], D.smooth);
	X.S[((size_t) n * D.T + t) * D.B + b] = St;
	X.v[i] = v;
	X.u[i] = u;
	if(n < D.R) {
		const Real r = X.alpha * X.r[n * D.B + b] + St;
		X.r[n * D.B + b] = r;
		X.rHist[((size_t) n * D.T + t) * D.B + b] = r;
		const Real diff = r - (Real) P.target[((size_t) t * D.B + b) * D.R + n];
		X.lossPart[i] += diff * diff;
	}
}

// deterministic final reduction of the loss (one block of 1024 threads)
template<typename Real>
__global__ void bptt_loss_kernel(BpttDev D, BpttState<Real> X, float* loss)
{
	__shared__ Real part[1024];
	Real s = Real(0);
	for(int i = threadIdx.x; i < D.R * D.B; i += blockDim.x) s += X.lossPart[i];
	part[threadIdx.x] = s;
	__syncthreads();
	for(int o = blockDim.x / 2; o > 0; o >>= 1) {
		if((int) threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
		__syncthreads();
	}
	if(threadIdx.x == 0) *loss = (float) (part[0] * X.lossScale);
}

// backward, segment replay: ms t of the segment starting at t0 (identical
// arithmetic to the forward pass), keeping its start state and input
template<typename Real>
__global__ void bptt_replay_kernel(BpttDev D, BpttState<Real> X, BpttParams P, int t, int t0)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= D.N * D.B) return;
	const int n = i / D.B, b = i % D.B;
	Real v, u;
	if(t == t0) {
		const size_t k = (size_t) (t0 / D.ckpt) * D.N * D.B + i;
		v = X.ckV[k];
		u = X.ckU[k];
	} else {
		v = X.v[i];
		u = X.u[i];
	}
	const Real syn = syn_input(D, X, P.W, n, b, t);
	const size_t s = (size_t) (t - t0) * D.N * D.B + i;
	X.segV[s] = v;
	X.segU[s] = u;
	X.segSyn[s] = syn;
	substeps(v, u, syn + (Real) P.noise[((size_t) t * D.B + b) * D.N + n], (Real) P.a[n], (Real) P.b[n],
			(Real) P.c[n], (Real) P.d[n], D.smooth);
	X.v[i] = v;
	X.u[i] = u;
}

// backward: adjoint of ms t for every (neuron, trial)
template<typename Real>
__global__ void bptt_backward_kernel(BpttDev D, BpttState<Real> X, BpttParams P, int t, int t0)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= D.N * D.B) return;
	const int n = i / D.B, b = i % D.B;

	// dL/dS(t): readout trace and the inputs S(t) drives d ms later
	Real lamS = Real(0);
	if(n < D.R) {
		const Real r = X.rHist[((size_t) n * D.T + t) * D.B + b];
		const Real diff = r - (Real) P.target[((size_t) t * D.B + b) * D.R + n];
		const Real lr = Real(2) * X.lossScale * diff + X.alpha * X.lamR[n * D.B + b];
		X.lamR[n * D.B + b] = lr;
		lamS = lr;
	}
	lamS += gather<Real>(D.outStart[n], D.outStart[n + 1], [&](int e, Real& w, Real& x) {
		const int tt = t + D.outDelay[e];
		w = (Real) P.W[e];
		x = tt < D.T ? X.lamI[((size_t) D.outTgt[e] * D.T + tt) * D.B + b] : Real(0);
	});

	// replay the sub-steps of ms t
	const Real a = P.a[n], bb = P.b[n], c = P.c[n], d = P.d[n];
	const size_t s = (size_t) (t - t0) * D.N * D.B + i;
	const Real I = X.segSyn[s] + (Real) P.noise[((size_t) t * D.B + b) * D.N + n];
	Real vk[4], uk[4], v1k[4], sk[4];
	{
		Real v = X.segV[s], u = X.segU[s];
#pragma unroll
		for(int k = 0; k < 4; ++k) {
			vk[k] = v;
			uk[k] = u;
			sk[k] = substep(v, u, v1k[k], I, a, bb, c, d, D.smooth);
		}
	}

	// reverse through the sub-steps
	Real lamV = X.lamV[i], lamU = X.lamU[i];
	Real lamI = Real(0), ga = X.gA[i], gb = X.gB[i];
#pragma unroll
	for(int k = 3; k >= 0; --k) {
		const Real v = vk[k], u = uk[k], v1 = v1k[k], sp = sk[k];
		// v' = v1 + s (c - v1), u' = u1 + s d
		const Real lams = lamS + lamV * (c - v1) + lamU * d;
		Real lamV1 = lamV * (Real(1) - sp) + lams * spike_grad(v1 - Real(30));
		const Real lamU1 = lamU;
		// u1 = u + a/4 (b v1 - u)
		lamV1 += lamU1 * Real(0.25) * a * bb;
		const Real lamUin = lamU1 * (Real(1) - Real(0.25) * a);
		ga += lamU1 * Real(0.25) * (bb * v1 - u);
		gb += lamU1 * Real(0.25) * a * v1;
		// v1 = v + 1/4 (0.04 v^2 + 5 v + 140 - u + I)
		lamV = lamV1 * (Real(1) + Real(0.25) * (Real(0.08) * v + Real(5)));
		lamU = lamUin - Real(0.25) * lamV1;
		lamI += Real(0.25) * lamV1;
	}
	X.lamV[i] = lamV;
	X.lamU[i] = lamU;
	X.gA[i] = ga;
	X.gB[i] = gb;
	X.lamI[((size_t) n * D.T + t) * D.B + b] = lamI;
}

// readout traces of the last forward pass as [T][B][R]
template<typename Real>
__global__ void bptt_readout_kernel(BpttDev D, BpttState<Real> X, float* out)
{
	const size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
	const size_t total = (size_t) D.T * D.B * D.R;
	if(i >= total) return;
	const int n = (int) (i % D.R), b = (int) ((i / D.R) % D.B), t = (int) (i / ((size_t) D.R * D.B));
	out[i] = (float) X.rHist[((size_t) n * D.T + t) * D.B + b];
}

// parameter gradients: sum over trials, plus u(0) = b v(0) with v(0) = -65
template<typename Real>
__global__ void bptt_param_grad_kernel(BpttDev D, BpttState<Real> X, float* da, float* db)
{
	const int n = blockIdx.x * blockDim.x + threadIdx.x;
	if(n >= D.N) return;
	Real sa = Real(0), sb = Real(0);
	for(int b = 0; b < D.B; ++b) {
		sa += X.gA[n * D.B + b];
		sb += X.gB[n * D.B + b] + X.lamU[n * D.B + b] * Real(-65);
	}
	da[n] = (float) sa;
	db[n] = (float) sb;
}

// dL/dW[e] = sum_t,b S_src(t - d) lambda_I,tgt(t): one CTA per source, its
// spike train in shared memory, one warp per outgoing synapse
template<typename Real>
__global__ void bptt_weight_grad_kernel(BpttDev D, BpttState<Real> X, float* dW)
{
	extern __shared__ __align__(16) unsigned char sRaw[];
	Real* sS = reinterpret_cast<Real*>(sRaw);
	const int j = blockIdx.x;
	const int TB = D.T * D.B;
	for(int k = threadIdx.x; k < TB; k += blockDim.x) sS[k] = X.S[(size_t) j * TB + k];
	__syncthreads();
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
	for(int e = D.outStart[j] + warp; e < D.outStart[j + 1]; e += nw) {
		const int dl = D.outDelay[e];
		const Real* lam = X.lamI + (size_t) D.outTgt[e] * TB + (size_t) dl * D.B;
		const int len = (D.T - dl) * D.B;
		Real acc = Real(0);
		for(int k = lane; k < len; k += 32) acc = fma(sS[k], lam[k], acc);
#pragma unroll
		for(int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
		if(lane == 0) dW[e] = (float) acc;
	}
}

Bptt::Bptt(unsigned N, unsigned B, unsigned T, unsigned R, unsigned ckpt, size_t M, const unsigned* src,
		const unsigned* tgt, const unsigned* delay, bool smooth, bool fp64, int device)
{
	if(N == 0 || B == 0 || T == 0 || ckpt == 0) NB_THROW(NEMO_INVALID_INPUT, "empty differentiable network");
	if(R > N) NB_THROW(NEMO_INVALID_INPUT, "more readout neurons than neurons");
	const size_t realSize = fp64 ? 8 : 4;
	if((size_t) T * B * realSize > 227 * 1024) {
		NB_THROW(NEMO_API_UNSUPPORTED, "ms x trials too large for the weight-gradient kernel (%zu bytes of shared memory)",
				(size_t) T * B * realSize);
	}
	if((size_t) N * B > (size_t) INT32_MAX) NB_THROW(NEMO_API_UNSUPPORTED, "neurons x trials too large");
	m_device = device;
	if(device >= 0) BP_CUDA(cudaSetDevice(device));
	else BP_CUDA(cudaGetDevice(&m_device));
	D.N = (int) N; D.B = (int) B; D.T = (int) T; D.R = (int) R; D.ckpt = (int) ckpt; D.smooth = smooth ? 1 : 0;
	m_fp64 = fp64;
	m_M = M;
	// synapses are given source-major: synapse e's weight is W[e]
	std::vector<int> outStart(N + 1, 0), inStart(N + 1, 0);
	for(size_t e = 0; e < M; ++e) {
		if(src[e] >= N || tgt[e] >= N) NB_THROW(NEMO_INVALID_INPUT, "synapse %zu has an invalid neuron", e);
		if(delay[e] < 1) NB_THROW(NEMO_INVALID_INPUT, "synapse %zu has delay 0", e);
		if(e && src[e] < src[e - 1]) NB_THROW(NEMO_INVALID_INPUT, "synapses must be ordered by source");
		outStart[src[e] + 1]++;
		inStart[tgt[e] + 1]++;
	}
	for(unsigned n = 0; n < N; ++n) {
		outStart[n + 1] += outStart[n];
		inStart[n + 1] += inStart[n];
	}
	std::vector<int> outTgt(M), outDelay(M), inSrc(M), inDelay(M), inSyn(M);
	std::vector<int> fill(inStart.begin(), inStart.end() - 1);
	for(size_t e = 0; e < M; ++e) {
		outTgt[e] = (int) tgt[e];
		outDelay[e] = (int) delay[e];
		const int p = fill[tgt[e]]++;
		inSrc[p] = (int) src[e];
		inDelay[p] = (int) delay[e];
		inSyn[p] = (int) e;
	}
	D.inStart = upload(inStart);
	D.inSrc = upload(inSrc);
	D.inDelay = upload(inDelay);
	D.inSyn = upload(inSyn);
	D.outStart = upload(outStart);
	D.outTgt = upload(outTgt);
	D.outDelay = upload(outDelay);
	if(fp64) {
		allocState(X64);
		BP_CUDA(cudaFuncSetAttribute(bptt_weight_grad_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
				(int) ((size_t) T * B * 8)));
	} else {
		allocState(X32);
		BP_CUDA(cudaFuncSetAttribute(bptt_weight_grad_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
				(int) ((size_t) T * B * 4)));
	}
}

template<typename Real>
void Bptt::allocState(BpttState<Real>& X)
{
	const size_t NB = (size_t) D.N * D.B, R = (size_t) std::max(1, D.R), B = D.B, T = D.T;
	const size_t nck = (T + D.ckpt - 1) / D.ckpt, seg = (size_t) std::min(D.ckpt, D.T);
	auto a = [&](size_t n) { return static_cast<Real*>(alloc(n * sizeof(Real))); };
	X.alpha = (Real) std::exp(-1.0 / 20.0);
	X.lossScale = Real(1) / ((Real) T * (Real) D.R * (Real) B);
	X.S = a(NB * T);
	X.v = a(NB);
	X.u = a(NB);
	X.ckV = a(NB * nck);
	X.ckU = a(NB * nck);
	X.r = a(R * B);
	X.rHist = a(R * T * B);
	X.lossPart = a(NB);
	X.segV = a(NB * seg);
	X.segU = a(NB * seg);
	X.segSyn = a(NB * seg);
	X.lamV = a(NB);
	X.lamU = a(NB);
	X.lamR = a(R * B);
	X.lamI = a(NB * T);
	X.gA = a(NB);
	X.gB = a(NB);
}

Bptt::~Bptt()
{
	for(void* p : m_allocs) cudaFree(p);
}

template<typename Real>
void Bptt::forwardT(BpttState<Real>& X, const BpttParams& P, float* loss, void* stream)
{
	cudaStream_t st = static_cast<cudaStream_t>(stream);
	const int threads = 256, blocks = (D.N * D.B + threads - 1) / threads;
	bptt_init_kernel<Real><<<blocks, threads, 0, st>>>(D, X, P);
	for(int t = 0; t < D.T; ++t) bptt_forward_kernel<Real><<<blocks, threads, 0, st>>>(D, X, P, t);
	bptt_loss_kernel<Real><<<1, 1024, 0, st>>>(D, X, loss);
	BP_CUDA(cudaGetLastError());
}

template<typename Real>
void Bptt::backwardT(BpttState<Real>& X, const BpttParams& P, float* dW, float* da, float* db, void* stream)
{
	cudaStream_t st = static_cast<cudaStream_t>(stream);
	const int threads = 256, blocks = (D.N * D.B + threads - 1) / threads;
	const size_t NB = (size_t) D.N * D.B * sizeof(Real);
	// lamV, lamU, lamR, gA, gB start at zero
	BP_CUDA(cudaMemsetAsync(X.lamV, 0, NB, st));
	BP_CUDA(cudaMemsetAsync(X.lamU, 0, NB, st));
	BP_CUDA(cudaMemsetAsync(X.lamR, 0, (size_t) std::max(1, D.R) * D.B * sizeof(Real), st));
	BP_CUDA(cudaMemsetAsync(X.gA, 0, NB, st));
	BP_CUDA(cudaMemsetAsync(X.gB, 0, NB, st));
	const int nseg = (D.T + D.ckpt - 1) / D.ckpt;
	for(int seg = nseg - 1; seg >= 0; --seg) {
		const int t0 = seg * D.ckpt, t1 = std::min(D.T, t0 + D.ckpt);
		for(int t = t0; t < t1; ++t) bptt_replay_kernel<Real><<<blocks, threads, 0, st>>>(D, X, P, t, t0);
		for(int t = t1 - 1; t >= t0; --t) bptt_backward_kernel<Real><<<blocks, threads, 0, st>>>(D, X, P, t, t0);
	}
	bptt_param_grad_kernel<Real><<<(D.N + 255) / 256, 256, 0, st>>>(D, X, da, db);
	bptt_weight_grad_kernel<Real><<<D.N, 256, (size_t) D.T * D.B * sizeof(Real), st>>>(D, X, dW);
	BP_CUDA(cudaGetLastError());
}

template<typename Real>
void Bptt::readoutT(BpttState<Real>& X, float* out, void* stream)
{
	const size_t total = (size_t) D.T * D.B * D.R;
	if(total) {
		bptt_readout_kernel<Real><<<(unsigned) ((total + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(D,
				X, out);
	}
	BP_CUDA(cudaGetLastError());
}

void Bptt::forward(const BpttParams& P, float* loss, void* stream)
{
	BP_CUDA(cudaSetDevice(m_device));
	if(m_fp64) forwardT(X64, P, loss, stream);
	else forwardT(X32, P, loss, stream);
}

void Bptt::backward(const BpttParams& P, float* dW, float* da, float* db, void* stream)
{
	BP_CUDA(cudaSetDevice(m_device));
	if(m_fp64) backwardT(X64, P, dW, da, db, stream);
	else backwardT(X32, P, dW, da, db, stream);
}

void Bptt::readout(float* out, void* stream)
{
	BP_CUDA(cudaSetDevice(m_device));
	if(m_fp64) readoutT(X64, out, stream);
	else readoutT(X32, out, stream);
}

void* Bptt::alloc(size_t bytes)
{
	void* p = nullptr;
	bytes = std::max<size_t>(bytes, 4);
	if(cudaMalloc(&p, bytes) != cudaSuccess) {
		NB_THROW(NEMO_CUDA_MEMORY_ERROR, "failed to allocate %zu bytes of device memory", bytes);
	}
	m_allocs.push_back(p);
	BP_CUDA(cudaMemset(p, 0, bytes));
	return p;
}

const int* Bptt::upload(const std::vector<int>& v)
{
	void* p = nullptr;
	if(cudaMalloc(&p, std::max<size_t>(v.size(), 1) * 4) != cudaSuccess) {
		NB_THROW(NEMO_CUDA_MEMORY_ERROR, "failed to allocate device memory");
	}
	m_allocs.push_back(p);
	if(!v.empty()) BP_CUDA(cudaMemcpy(p, v.data(), v.size() * 4, cudaMemcpyHostToDevice));
	return static_cast<const int*>(p);
}

} // namespace nemo_b200
