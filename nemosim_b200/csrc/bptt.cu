// bptt.cu -- differentiable float32 mode: a network of Izhikevich neurons
// with delayed synapses, run forward with checkpoints and differentiated by
// a hand-written backpropagation-through-time adjoint.
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
// Layouts (float32): spikes S and input adjoints lambda_I as [n][t][b];
// states [n][b]; noise and targets as PyTorch tensors [T][B][N] and [T][B][R].
// One thread per (neuron, trial); 16 trials of one neuron are 64 contiguous
// bytes.  Checkpoints of (v, u) every `ckpt` ms; the backward pass replays
// each segment from its checkpoint and keeps the per-ms start states and
// synaptic inputs of that segment.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
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

constexpr float BP_K = 10.0f;

__device__ __forceinline__ float spike_fn(float x, int smooth)
{
	if(smooth) return 0.5f * (1.0f + BP_K * x / (1.0f + BP_K * fabsf(x)));
	return x >= 0.0f ? 1.0f : 0.0f;
}

__device__ __forceinline__ float spike_grad(float x)
{
	const float q = 1.0f + BP_K * fabsf(x);
	return 0.5f * BP_K / (q * q);
}

// synaptic input of (n, b) at ms t from the stored spikes
__device__ __forceinline__ float syn_input(const BpttDev& D, const float* W, int n, int b, int t)
{
	float syn = 0.0f;
	for(int e = D.inStart[n]; e < D.inStart[n + 1]; ++e) {
		const int dl = D.inDelay[e];
		if(t >= dl) syn = fmaf(W[D.inSyn[e]], D.S[((size_t) D.inSrc[e] * D.T + (t - dl)) * D.B + b], syn);
	}
	return syn;
}

// the four sub-steps of one ms; returns S(t)
__device__ __forceinline__ float substeps(float& v, float& u, float I, float a, float b, float c, float d, int smooth)
{
	float St = 0.0f;
#pragma unroll
	for(int k = 0; k < 4; ++k) {
		const float v1 = v + 0.25f * (0.04f * v * v + 5.0f * v + 140.0f - u + I);
		const float u1 = u + 0.25f * a * (b * v1 - u);
		const float s = spike_fn(v1 - 30.0f, smooth);
		v = v1 + s * (c - v1);
		u = u1 + s * d;
		St += s;
	}
	return St;
}

__global__ void bptt_init_kernel(BpttDev D, BpttParams P)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= D.N * D.B) return;
	const int n = i / D.B, b = i % D.B;
	D.v[i] = -65.0f;
	D.u[i] = P.b[n] * -65.0f;
	D.lossPart[i] = 0.0f;
	D.lamV[i] = 0.0f;
	D.lamU[i] = 0.0f;
	D.gA[i] = 0.0f;
	D.gB[i] = 0.0f;
	if(n < D.R) {
		D.r[n * D.B + b] = 0.0f;
		D.lamR[n * D.B + b] = 0.0f;
	}
}

// forward: one ms for every (neuron, trial)
__global__ void bptt_forward_kernel(BpttDev D, BpttParams P, int t)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= D.N * D.B) return;
	const int n = i / D.B, b = i % D.B;
	float v = D.v[i], u = D.u[i];
	if(t % D.ckpt == 0) {
		const size_t k = (size_t) (t / D.ckpt) * D.N * D.B + i;
		D.ckV[k] = v;
		D.ckU[k] = u;
	}
	const float I = syn_input(D, P.W, n, b, t) + P.noise[((size_t) t * D.B + b) * D.N + n];
	const float St = substeps(v, u, I, P.a[n], P.b[n], P.c[n], P.d[n], D.smooth);
	D.S[((size_t) n * D.T + t) * D.B + b] = St;
	D.v[i] = v;
	D.u[i] = u;
	if(n < D.R) {
		const float r = D.alpha * D.r[n * D.B + b] + St;
		D.r[n * D.B + b] = r;
		D.rHist[((size_t) n * D.T + t) * D.B + b] = r;
		const float diff = r - P.target[((size_t) t * D.B + b) * D.R + n];
		D.lossPart[i] += diff * diff;
	}
}

// deterministic final reduction of the loss (one block)
__global__ void bptt_loss_kernel(BpttDev D, float* loss)
{
	__shared__ float part[1024];
	float s = 0.0f;
	for(int i = threadIdx.x; i < D.R * D.B; i += blockDim.x) s += D.lossPart[i];
	part[threadIdx.x] = s;
	__syncthreads();
	for(int o = blockDim.x / 2; o > 0; o >>= 1) {
		if((int) threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
		__syncthreads();
	}
	if(threadIdx.x == 0) *loss = part[0] * D.lossScale;
}

// backward, segment replay: ms t of the segment starting at t0 (identical
// arithmetic to the forward pass), keeping its start state and input
__global__ void bptt_replay_kernel(BpttDev D, BpttParams P, int t, int t0)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= D.N * D.B) return;
	const int n = i / D.B, b = i % D.B;
	float v, u;
	if(t == t0) {
		const size_t k = (size_t) (t0 / D.ckpt) * D.N * D.B + i;
		v = D.ckV[k];
		u = D.ckU[k];
	} else {
		v = D.v[i];
		u = D.u[i];
	}
	const float syn = syn_input(D, P.W, n, b, t);
	const size_t s = (size_t) (t - t0) * D.N * D.B + i;
	D.segV[s] = v;
	D.segU[s] = u;
	D.segSyn[s] = syn;
	substeps(v, u, syn + P.noise[((size_t) t * D.B + b) * D.N + n], P.a[n], P.b[n], P.c[n], P.d[n], D.smooth);
	D.v[i] = v;
	D.u[i] = u;
}

// backward: adjoint of ms t for every (neuron, trial)
__global__ void bptt_backward_kernel(BpttDev D, BpttParams P, int t, int t0)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= D.N * D.B) return;
	const int n = i / D.B, b = i % D.B;

	// dL/dS(t): readout trace and the inputs S(t) drives d ms later
	float lamS = 0.0f;
	if(n < D.R) {
		const float r = D.rHist[((size_t) n * D.T + t) * D.B + b];
		const float diff = r - P.target[((size_t) t * D.B + b) * D.R + n];
		const float lr = 2.0f * D.lossScale * diff + D.alpha * D.lamR[n * D.B + b];
		D.lamR[n * D.B + b] = lr;
		lamS = lr;
	}
	for(int e = D.outStart[n]; e < D.outStart[n + 1]; ++e) {
		const int tt = t + D.outDelay[e];
		if(tt < D.T) lamS = fmaf(P.W[e], D.lamI[((size_t) D.outTgt[e] * D.T + tt) * D.B + b], lamS);
	}

	// replay the sub-steps of ms t
	const float a = P.a[n], bb = P.b[n], c = P.c[n], d = P.d[n];
	const size_t s = (size_t) (t - t0) * D.N * D.B + i;
	const float I = D.segSyn[s] + P.noise[((size_t) t * D.B + b) * D.N + n];
	float vk[4], uk[4], v1k[4], sk[4];
	{
		float v = D.segV[s], u = D.segU[s];
#pragma unroll
		for(int k = 0; k < 4; ++k) {
			vk[k] = v;
			uk[k] = u;
			const float v1 = v + 0.25f * (0.04f * v * v + 5.0f * v + 140.0f - u + I);
			const float u1 = u + 0.25f * a * (bb * v1 - u);
			const float sp = spike_fn(v1 - 30.0f, D.smooth);
			v1k[k] = v1;
			sk[k] = sp;
			v = v1 + sp * (c - v1);
			u = u1 + sp * d;
		}
	}

	// reverse through the sub-steps
	float lamV = D.lamV[i], lamU = D.lamU[i];
	float lamI = 0.0f, ga = D.gA[i], gb = D.gB[i];
#pragma unroll
	for(int k = 3; k >= 0; --k) {
		const float v = vk[k], u = uk[k], v1 = v1k[k], sp = sk[k];
		// v' = v1 + s (c - v1), u' = u1 + s d
		const float lams = lamS + lamV * (c - v1) + lamU * d;
		float lamV1 = lamV * (1.0f - sp) + lams * spike_grad(v1 - 30.0f);
		const float lamU1 = lamU;
		// u1 = u + a/4 (b v1 - u)
		lamV1 += lamU1 * 0.25f * a * bb;
		float lamUin = lamU1 * (1.0f - 0.25f * a);
		ga += lamU1 * 0.25f * (bb * v1 - u);
		gb += lamU1 * 0.25f * a * v1;
		// v1 = v + 1/4 (0.04 v^2 + 5 v + 140 - u + I)
		lamV = lamV1 * (1.0f + 0.25f * (0.08f * v + 5.0f));
		lamU = lamUin - 0.25f * lamV1;
		lamI += 0.25f * lamV1;
	}
	D.lamV[i] = lamV;
	D.lamU[i] = lamU;
	D.gA[i] = ga;
	D.gB[i] = gb;
	D.lamI[((size_t) n * D.T + t) * D.B + b] = lamI;
}

// readout traces of the last forward pass as [T][B][R]
__global__ void bptt_readout_kernel(BpttDev D, float* out)
{
	const size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
	const size_t total = (size_t) D.T * D.B * D.R;
	if(i >= total) return;
	const int n = (int) (i % D.R), b = (int) ((i / D.R) % D.B), t = (int) (i / ((size_t) D.R * D.B));
	out[i] = D.rHist[((size_t) n * D.T + t) * D.B + b];
}

// parameter gradients: sum over trials, plus u(0) = b v(0) with v(0) = -65
__global__ void bptt_param_grad_kernel(BpttDev D, float* da, float* db)
{
	const int n = blockIdx.x * blockDim.x + threadIdx.x;
	if(n >= D.N) return;
	float sa = 0.0f, sb = 0.0f;
	for(int b = 0; b < D.B; ++b) {
		sa += D.gA[n * D.B + b];
		sb += D.gB[n * D.B + b] + D.lamU[n * D.B + b] * -65.0f;
	}
	da[n] = sa;
	db[n] = sb;
}

// dL/dW[e] = sum_t,b S_src(t - d) lambda_I,tgt(t): one CTA per source, its
// spike train in shared memory, one warp per outgoing synapse
__global__ void bptt_weight_grad_kernel(BpttDev D, float* dW)
{
	extern __shared__ float sS[];
	const int j = blockIdx.x;
	const int TB = D.T * D.B;
	for(int k = threadIdx.x; k < TB; k += blockDim.x) sS[k] = D.S[(size_t) j * TB + k];
	__syncthreads();
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
	for(int e = D.outStart[j] + warp; e < D.outStart[j + 1]; e += nw) {
		const int dl = D.outDelay[e];
		const float* lam = D.lamI + (size_t) D.outTgt[e] * TB + (size_t) dl * D.B;
		const int len = (D.T - dl) * D.B;
		float acc = 0.0f;
		for(int k = lane; k < len; k += 32) acc = fmaf(sS[k], lam[k], acc);
#pragma unroll
		for(int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
		if(lane == 0) dW[e] = acc;
	}
}

Bptt::Bptt(unsigned N, unsigned B, unsigned T, unsigned R, unsigned ckpt, size_t M, const unsigned* src,
		const unsigned* tgt, const unsigned* delay, int smooth, int device)
{
	if(N == 0 || B == 0 || T == 0 || ckpt == 0) NB_THROW(NEMO_INVALID_INPUT, "empty differentiable network");
	if(R > N) NB_THROW(NEMO_INVALID_INPUT, "more readout neurons than neurons");
	m_device = device;
	if(device >= 0) BP_CUDA(cudaSetDevice(device));
	else BP_CUDA(cudaGetDevice(&m_device));
	D.N = (int) N; D.B = (int) B; D.T = (int) T; D.R = (int) R; D.ckpt = (int) ckpt; D.smooth = smooth;
	D.alpha = expf(-1.0f / 20.0f);
	D.lossScale = 1.0f / ((float) T * (float) R * (float) B);
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
	const size_t NB = (size_t) N * B;
	const size_t nck = (T + ckpt - 1) / ckpt;
	D.S = alloc(NB * T);
	D.v = alloc(NB);
	D.u = alloc(NB);
	D.ckV = alloc(NB * nck);
	D.ckU = alloc(NB * nck);
	D.r = alloc((size_t) std::max(1u, R) * B);
	D.rHist = alloc((size_t) std::max(1u, R) * T * B);
	D.lossPart = alloc(NB);
	D.segV = alloc(NB * ckpt);
	D.segU = alloc(NB * ckpt);
	D.segSyn = alloc(NB * ckpt);
	D.lamV = alloc(NB);
	D.lamU = alloc(NB);
	D.lamR = alloc((size_t) std::max(1u, R) * B);
	D.lamI = alloc(NB * T);
	D.gA = alloc(NB);
	D.gB = alloc(NB);
	BP_CUDA(cudaFuncSetAttribute(bptt_weight_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
			(int) std::min<size_t>(227 * 1024, (size_t) T * B * 4)));
	if((size_t) T * B * 4 > 227 * 1024) NB_THROW(NEMO_API_UNSUPPORTED, "T x trials too large for the weight-gradient kernel");
}


Bptt::~Bptt()
{
	for(void* p : m_allocs) cudaFree(p);
}

void Bptt::forward(const BpttParams& P, float* loss, void* stream)
{
	cudaStream_t st = static_cast<cudaStream_t>(stream);
BP_CUDA(cudaSetDevice(m_device));
	const int threads = 256, blocks = (D.N * D.B + threads - 1) / threads;
	bptt_init_kernel<<<blocks, threads, 0, st>>>(D, P);
	for(int t = 0; t < D.T; ++t) bptt_forward_kernel<<<blocks, threads, 0, st>>>(D, P, t);
	bptt_loss_kernel<<<1, 1024, 0, st>>>(D, loss);
	BP_CUDA(cudaGetLastError());
}

void Bptt::backward(const BpttParams& P, float* dW, float* da, float* db, void* stream)
{
	cudaStream_t st = static_cast<cudaStream_t>(stream);
BP_CUDA(cudaSetDevice(m_device));
	const int threads = 256, blocks = (D.N * D.B + threads - 1) / threads;
	// lamV, lamU, lamR, gA, gB start at zero
	BP_CUDA(cudaMemsetAsync(D.lamV, 0, (size_t) D.N * D.B * 4, st));
	BP_CUDA(cudaMemsetAsync(D.lamU, 0, (size_t) D.N * D.B * 4, st));
	BP_CUDA(cudaMemsetAsync(D.lamR, 0, (size_t) std::max(1, D.R) * D.B * 4, st));
	BP_CUDA(cudaMemsetAsync(D.gA, 0, (size_t) D.N * D.B * 4, st));
	BP_CUDA(cudaMemsetAsync(D.gB, 0, (size_t) D.N * D.B * 4, st));
	const int nseg = (D.T + D.ckpt - 1) / D.ckpt;
	for(int seg = nseg - 1; seg >= 0; --seg) {
		const int t0 = seg * D.ckpt, t1 = std::min(D.T, t0 + D.ckpt);
		for(int t = t0; t < t1; ++t) bptt_replay_kernel<<<blocks, threads, 0, st>>>(D, P, t, t0);
		for(int t = t1 - 1; t >= t0; --t) bptt_backward_kernel<<<blocks, threads, 0, st>>>(D, P, t, t0);
	}
	bptt_param_grad_kernel<<<(D.N + 255) / 256, 256, 0, st>>>(D, da, db);
	bptt_weight_grad_kernel<<<D.N, 256, (size_t) D.T * D.B * 4, st>>>(D, dW);
	BP_CUDA(cudaGetLastError());
}

void Bptt::readout(float* out, void* stream)
{
	BP_CUDA(cudaSetDevice(m_device));
	const size_t total = (size_t) D.T * D.B * D.R;
	if(total) bptt_readout_kernel<<<(unsigned) ((total + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(D, out);
	BP_CUDA(cudaGetLastError());
}

float* Bptt::alloc(size_t n)
{
	void* p = nullptr;
	if(cudaMalloc(&p, std::max<size_t>(n, 1) * 4) != cudaSuccess) {
		NB_THROW(NEMO_CUDA_MEMORY_ERROR, "failed to allocate %zu bytes of device memory", n * 4);
	}
	m_allocs.push_back(p);
	BP_CUDA(cudaMemset(p, 0, std::max<size_t>(n, 1) * 4));
	return static_cast<float*>(p);
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

