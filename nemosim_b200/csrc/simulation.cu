// simulation.cu -- kernels and host orchestration of the B200 backend.
#include "simulation.hpp"

#include <string.h>

#include <algorithm>
#include <mutex>

#include "kernels.cuh"
#include "libm_calib.hpp"

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

// Shared-memory work list of one CTA: the items (fired neurons or STDP
// targets) it collected, each with a span of consecutive entries of a CSR
// array (outgoing synapses or incoming plastic synapses).  off[] is the
// exclusive prefix sum of the span lengths and adj[i] = start(i) - off[i],
// so flat work item k of the CTA is entry adj[i] + k for the i whose span
// contains k.  Spreading all spans over all threads of the CTA keeps every
// thread's loads independent of the item sizes.
struct WorkList {
	uint32_t* item;               // [cap]
	uint32_t* off;                // [cap + 1]
	unsigned long long* adj;      // [cap]
};

__device__ __forceinline__ WorkList carve_list(unsigned char*& p, uint32_t cap)
{
	WorkList w;
	w.adj = reinterpret_cast<unsigned long long*>(p);
	p += 8 * (size_t) cap;
	w.item = reinterpret_cast<uint32_t*>(p);
	p += 4 * (size_t) cap;
	w.off = reinterpret_cast<uint32_t*>(p);
	p += 4 * (size_t) (cap + 1);
	p = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(p) + 15) & ~uintptr_t(15));
	return w;
}

// Block-wide exclusive scan of the span lengths ptr[item+1] - ptr[item] of
// the n collected items; returns the total.  All threads must call it.
__device__ uint32_t build_offsets(const WorkList& L, uint32_t n, const unsigned long long* ptr, uint32_t* warpTmp)
{
	const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
	uint32_t carry = 0;
	for(uint32_t base = 0; base < n; base += blockDim.x) {
		const uint32_t i = base + tid;
		unsigned long long b = 0;
		uint32_t c = 0;
		if(i < n) {
			const uint32_t it = L.item[i];
			b = ptr[it];
			c = (uint32_t) (ptr[it + 1] - b);
		}
		uint32_t x = c;
#pragma unroll
		for(int o = 1; o < 32; o <<= 1) {
			uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
			if(lane >= (uint32_t) o) x += y;
		}
		if(lane == 31) warpTmp[warp] = x;
		__syncthreads();
		if(warp == 0) {
			uint32_t s = lane < nwarps ? warpTmp[lane] : 0;
#pragma unroll
			for(int o = 1; o < 32; o <<= 1) {
				uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
				if(lane >= (uint32_t) o) s += y;
			}
			warpTmp[lane] = s;
		}
		__syncthreads();
		const uint32_t o = carry + (warp ? warpTmp[warp - 1] : 0) + x - c;
		if(i < n) {
			L.off[i] = o;
			L.adj[i] = b - o;
		}
		carry += warpTmp[nwarps - 1];
		__syncthreads();
	}
	if(threadIdx.x == 0) L.off[n] = carry;
	__syncthreads();
	return carry;
}

// the item whose span holds flat work item k: largest i < n with off[i] <= k
__device__ __forceinline__ uint32_t find_item(const uint32_t* off, uint32_t n, uint32_t k)
{
	uint32_t lo = 0, hi = n;
	while(hi - lo > 1) {
		uint32_t mid = (lo + hi) >> 1;
		if(off[mid] <= k) lo = mid; else hi = mid;
	}
	return lo;
}

constexpr uint32_t ILP = 4;

// scatter: add every outgoing synapse of the CTA's fired neurons into the
// accumulator slot of its arrival step (64-bit integer atomics)
__device__ __forceinline__ void scatter_phase(const DevSim& S, const WorkList& L, uint32_t n, uint32_t total, uint32_t slot)
{
	const uint32_t T = blockDim.x;
	for(uint32_t k0 = threadIdx.x; k0 < total; k0 += ILP * T) {
		uint2 s[ILP];
#pragma unroll
		for(uint32_t j = 0; j < ILP; ++j) {
			const uint32_t k = k0 + j * T;
			if(k < total) {
				const uint32_t i = find_item(L.off, n, k);
				s[j] = S.syn[L.adj[i] + k];
			}
		}
#pragma unroll
		for(uint32_t j = 0; j < ILP; ++j) {
			if(k0 + j * T < total) {
				uint32_t d = (s[j].x >> 26) + 1;
				uint32_t sl = slot + d;
				sl = sl >= S.D ? sl - S.D : sl;
				add_current(S.slots + (size_t) sl * S.N + (s[j].x & (MAX_NEURONS - 1)), (int32_t) s[j].y);
			}
		}
	}
}

// STDP accumulation over the incoming plastic synapses of the CTA's targets
// (ConnectivityMatrix::accumulateStdp, src/nemo/ConnectivityMatrix.cpp:193-227)
__device__ __forceinline__ void stdp_phase(const DevSim& S, const WorkList& L, uint32_t n, uint32_t total,
		const uint64_t* hist)
{
	const uint32_t T = blockDim.x;
	for(uint32_t k0 = threadIdx.x; k0 < total; k0 += ILP * T) {
		unsigned long long p[ILP];
		uint32_t sd[ILP];
		int32_t acc[ILP];
		uint64_t h[ILP];
#pragma unroll
		for(uint32_t j = 0; j < ILP; ++j) {
			const uint32_t k = k0 + j * T;
			if(k < total) {
				const uint32_t i = find_item(L.off, n, k);
				p[j] = L.adj[i] + k;
				sd[j] = S.rcmSrc[p[j]];
				acc[j] = S.rcmAcc[p[j]];
			}
		}
#pragma unroll
		for(uint32_t j = 0; j < ILP; ++j) {
			if(k0 + j * T < total) h[j] = hist[sd[j] & (MAX_NEURONS - 1)];
		}
#pragma unroll
		for(uint32_t j = 0; j < ILP; ++j) {
			if(k0 + j * T < total) {
				const uint32_t delay = (sd[j] >> 26) + 1;
				int32_t dw = stdp_weight_change(S.sp, h[j] >> (delay & 63));
				if(dw != 0) S.rcmAcc[p[j]] = (int32_t) ((uint32_t) acc[j] + (uint32_t) dw);
			}
		}
	}
}

// warp-aggregated append of the lanes whose flag is set
__device__ __forceinline__ void append(uint32_t* list, uint32_t* count, bool flag, uint32_t value)
{
	const uint32_t lane = threadIdx.x & 31;
	const uint32_t b = __ballot_sync(0xffffffffu, flag);
	if(!b) return;
	uint32_t base = 0;
	if(lane == 0) base = atomicAdd(count, (uint32_t) __popc(b));
	base = __shfl_sync(0xffffffffu, base, 0);
	if(flag) list[base + __popc(b & ((1u << lane) - 1u))] = value;
}

// One simulation step (see kernels.cuh).  CTA c owns the partition of P
// consecutive neurons starting at c * P (P a multiple of 32, so warps cover
// whole bit-vector words); its blockDim.x threads loop over them.
__global__ void __launch_bounds__(1024)
step_kernel(const DevSim S, uint32_t P, uint32_t cur, uint32_t slot, uint32_t ring, int stdpPrev)
{
	extern __shared__ __align__(16) unsigned char smem[];
	__shared__ uint32_t sNF, sNS, warpTmp[32];

	const uint32_t tid = threadIdx.x, lane = tid & 31;
	const uint32_t first = blockIdx.x * P;
	const uint32_t last = min(S.N, first + P);
	const uint64_t* histPrev = S.hist + (size_t) (cur ^ 1u) * S.N;
	uint64_t* histCur = S.hist + (size_t) cur * S.N;
	unsigned char* sp = smem;
	WorkList LF = carve_list(sp, P);
	WorkList LS = carve_list(sp, P);

	if(tid == 0) { sNF = 0; sNS = 0; }
	__syncthreads();

	// 1-3: read-out, update, history, fired bit-vector, compaction
	for(uint32_t base = first; base < last; base += blockDim.x) {
		const uint32_t n = base + tid;
		bool fired = false, stdpTarget = false;
		uint32_t fw = 0;
		if(n < last) {
			uint32_t k = 0;
			while(k + 1 < S.ntypes && n >= S.types[k + 1].base) ++k;
			const TypeRange& T = S.types[k];
			const uint32_t nl = n - T.base;
			float cE = 0.0f, cI = 0.0f;
			if(S.D) {
				longlong2* a = S.slots + (size_t) slot * S.N + n;
				longlong2 acc = *a;
				if(acc.x | acc.y) *a = make_longlong2(0, 0);
				cE = wfx_to_float(acc.x);
				cI = wfx_to_float(acc.y);
			}
			float ext = S.curExt[n];
			if(__float_as_uint(ext) != 0u) S.curExt[n] = 0.0f;
			fw = S.fstim[n >> 5];
			const bool fs = (fw >> lane) & 1u;
			switch(T.kind) {
				case KIND_IZHIKEVICH: fired = update_izhikevich(S, T, nl, n, cE, cI, ext, fs); break;
				case KIND_IF_CURR_EXP: fired = update_if_curr_exp(T, nl, cE, cI, ext, fs); break;
				case KIND_POISSON: fired = update_poisson(S, T, nl, n, fs); break;
				default: fired = fs; break; // Input, src/nemo/cpu/plugins/Input.cpp:17-22
			}
			const uint64_t h = histPrev[n];
			histCur[n] = (h << 1) | (uint64_t) fired;
			stdpTarget = stdpPrev && (h & S.sp.postFireMask) && S.rcmPtr[n + 1] > S.rcmPtr[n];
		}
		const uint32_t fb = __ballot_sync(0xffffffffu, fired);
		if(lane == 0 && n < last) {
			S.firedRing[(size_t) ring * S.W + (n >> 5)] = fb;
			if(fw) S.fstim[n >> 5] = 0u;
		}
		append(LF.item, &sNF, fired, n);
		append(LS.item, &sNS, stdpTarget, n);
	}
	__syncthreads();
	const uint32_t nf = sNF, ns = sNS;

	// 4. scatter, 5. STDP of the previous step
	const uint32_t wf = nf ? build_offsets(LF, nf, S.outPtr, warpTmp) : 0;
	const uint32_t ws = ns ? build_offsets(LS, ns, S.rcmPtr, warpTmp) : 0;
	if(S.D && wf) scatter_phase(S, LF, nf, wf, slot);
	if(ws) stdp_phase(S, LS, ns, ws, histPrev);

	if(tid == 0) {
		if(nf) atomicAdd(&S.firedCount[ring], nf);
		if(wf) atomicAdd(&S.eventCount[ring], (unsigned long long) wf);
		if(ws) atomicAdd(&S.stdpCount[ring], (unsigned long long) ws);
	}
}

// Pending STDP accumulation of the last completed step (history buffer `par`)
__global__ void __launch_bounds__(1024)
stdp_kernel(const DevSim S, uint32_t P, uint32_t par, uint32_t ring)
{
	extern __shared__ __align__(16) unsigned char smem[];
	__shared__ uint32_t sNS, warpTmp[32];
	const uint32_t tid = threadIdx.x;
	const uint32_t first = blockIdx.x * P;
	const uint32_t last = min(S.N, first + P);
	const uint64_t* hist = S.hist + (size_t) par * S.N;
	unsigned char* sp = smem;
	WorkList LS = carve_list(sp, P);
	if(tid == 0) sNS = 0;
	__syncthreads();
	for(uint32_t base = first; base < last; base += blockDim.x) {
		const uint32_t n = base + tid;
		bool target = n < last && (hist[n] & S.sp.postFireMask) && S.rcmPtr[n + 1] > S.rcmPtr[n];
		append(LS.item, &sNS, target, n);
	}
	__syncthreads();
	const uint32_t ns = sNS;
	const uint32_t ws = ns ? build_offsets(LS, ns, S.rcmPtr, warpTmp) : 0;
	if(ws) stdp_phase(S, LS, ns, ws, hist);
	if(tid == 0 && ws) atomicAdd(&S.stdpCount[ring], (unsigned long long) ws);
}

// applyStdp (src/nemo/ConnectivityMatrix.cpp:241-294): one warp per target,
// lanes over its incoming plastic synapses.  A weight that changes is
// written back to the forward matrix, and the spikes already scattered with
// the old weight but not yet arrived (source fired k < delay steps ago) are
// corrected in their accumulator slots.
__global__ void __launch_bounds__(STEP_THREADS)
apply_stdp_kernel(const DevSim S, int32_t reward, uint32_t par, uint32_t slot, int fullPass)
{
	const uint32_t lane = threadIdx.x & 31;
	const uint32_t warpsTotal = gridDim.x * (STEP_THREADS / 32);
	const uint64_t* hist = S.hist + (size_t) par * S.N;
	for(uint32_t tgt = blockIdx.x * (STEP_THREADS / 32) + (threadIdx.x >> 5); tgt < S.N; tgt += warpsTotal) {
		unsigned long long b = S.rcmPtr[tgt], e = S.rcmPtr[tgt + 1];
		for(unsigned long long p = b + lane; p < e; p += 32) {
			int32_t acc = S.rcmAcc[p];
			// Once every plastic weight lies within its clamp range (after the
			// first pass), a zero accumulator leaves the weight unchanged:
			// updatedWeight(w, 0) == w.
			if(acc == 0 && !fullPass) continue;
			uint32_t fwd = S.rcmFwd[p];
			int32_t w = (int32_t) S.syn[fwd].y;
			int32_t nw = stdp_updated_weight(S.sp, w, fx_mul_dev(reward, acc));
			if(nw != w) {
				S.syn[fwd].y = (uint32_t) nw;
				if(S.D) {
					uint32_t sd = S.rcmSrc[p];
					uint32_t src = sd & (MAX_NEURONS - 1);
					uint32_t delay = (sd >> 26) + 1;
					uint64_t inflight = hist[src] & ((delay >= 64) ? ~0ull : ((1ull << delay) - 1ull));
					while(inflight) {
						uint32_t k = __ffsll((long long) inflight) - 1;
						inflight &= inflight - 1;
						// fired k steps before the last step, arrives delay - k steps after it
						uint32_t sl = (slot + delay - k) % S.D;
						unsigned long long* a = reinterpret_cast<unsigned long long*>(S.slots + (size_t) sl * S.N + tgt);
						// remove the old weight from its class (E if >= 0, else I) and
						// add the new one to its class (deliverSpikesOne,
						// src/nemo/cpu/Simulation.cpp:297-300)
						atomicAdd(a + (w < 0 ? 1 : 0), (unsigned long long) (-(long long) w));
						atomicAdd(a + (nw < 0 ? 1 : 0), (unsigned long long) (long long) nw);
					}
				}
			}
			if(acc) S.rcmAcc[p] = 0;
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
	LibmCalib c;
	c.logFlip = dLog;
	c.sinFlip = dSin;
	c.excKey = dKey;
	c.excVal = dVal;
	c.nexc = (uint32_t) nexc;
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
}

static inline uint64_t shl64(uint64_t x, unsigned s) { return x << (s & 63); }

Simulation::Simulation(const Network& net, const Configuration& conf)
{
	// checks in the order of nemo::simulationBackend (src/nemo/nemo.cpp:109-134)
	// and the backend constructor (src/nemo/cpu/Simulation.cpp:36-82)
	unsigned N = net.neuronCount();
	if(N == 0) NB_THROW(NEMO_INVALID_INPUT, "Cannot create simulation from empty network");
	if(conf.stdp && net.maxDelay + conf.postfire.size() > MAX_HISTORY) {
		NB_THROW(NEMO_INVALID_INPUT, "Max delay + postfire part of STDP function must be <= %u", MAX_HISTORY);
	}
	if(conf.backend != NEMO_BACKEND_CUDA) {
		NB_THROW(NEMO_API_UNSUPPORTED, "This library provides only the B200 CUDA backend; the CPU backend is not part of it");
	}
	if(net.maxDelay > 64) {
		NB_THROW(NEMO_INVALID_INPUT, "The network has synapses with delay %ums. The B200 backend supports a maximum of 64 ms", net.maxDelay);
	}
	if(net.duplicate) NB_THROW(NEMO_INVALID_INPUT, "Duplicate neuron index %u", net.duplicateIdx);
	if(N >= MAX_NEURONS) NB_THROW(NEMO_API_UNSUPPORTED, "The B200 backend supports at most %u neurons", MAX_NEURONS - 1);

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
	m_maxDelay = net.maxDelay;
	m_writeOnly = conf.writeOnlySynapses;
	memset(&m_dev, 0, sizeof m_dev);
	DevSim& S = m_dev;
	S.N = N;
	S.W = (N + 31) / 32;

	// local indices: type order, then insertion order
	m_l2g.resize(N);
	m_ltype.resize(N);
	m_g2l.reserve(N * 2);
	unsigned l = 0;
	bool needCalib = false;
	for(unsigned t = 0; t < net.types.size(); ++t) {
		const NeuronCollection& c = net.types[t];
		if(c.size() == 0) continue;
		if(m_types.size() >= MAX_TYPES) NB_THROW(NEMO_API_UNSUPPORTED, "At most %u neuron types", MAX_TYPES);
		HostType ht;
		ht.desc = c.desc;
		ht.netType = t;
		ht.base = l;
		ht.n = (unsigned) c.size();
		unsigned np = c.desc->nparam, ns = c.desc->nstate, na = np + ns;
		std::vector<float> param((size_t) np * ht.n), state((size_t) ns * ht.n);
		for(size_t i = 0; i < c.size(); ++i) {
			for(unsigned p = 0; p < np; ++p) param[(size_t) p * ht.n + i] = c.args[i * na + p];
			for(unsigned v = 0; v < ns; ++v) state[(size_t) v * ht.n + i] = c.args[i * na + np + v];
			m_l2g[l + i] = c.gidx[i];
			m_ltype[l + i] = (uint8_t) m_types.size();
			if(!m_g2l.emplace(c.gidx[i], l + (unsigned) i).second) {
				NB_THROW(NEMO_INVALID_INPUT, "Duplicate neuron index %u", c.gidx[i]);
			}
		}
		ht.dParam = dalloc<float>(param.size());
		ht.dState = dalloc<float>(state.size());
		NB_CUDA(cudaMemcpyAsync(ht.dParam, param.data(), param.size() * 4, cudaMemcpyHostToDevice, m_stream));
		NB_CUDA(cudaMemcpyAsync(ht.dState, state.data(), state.size() * 4, cudaMemcpyHostToDevice, m_stream));
		if(c.desc->kind == KIND_IZHIKEVICH) needCalib = true;
		TypeRange& tr = S.types[m_types.size()];
		tr.kind = c.desc->kind;
		tr.base = ht.base;
		tr.n = ht.n;
		tr.param = ht.dParam;
		tr.state = ht.dState;
		m_types.push_back(ht);
		l += ht.n;
		NB_CUDA(cudaStreamSynchronize(m_stream)); // host vectors go out of scope
	}
	S.ntypes = (uint32_t) m_types.size();

	// forward matrix (src/nemo/ConnectivityMatrix.cpp:65-162): outgoing
	// synapses per local source, sorted by delay, insertion order within a
	// delay -- the reference's row order
	const size_t Sn = net.src.size();
	m_nsyn = Sn;
	std::vector<unsigned> lsrc(Sn), ltgt(Sn);
	std::vector<int32_t> fxw(Sn);
	for(size_t k = 0; k < Sn; ++k) {
		auto is = m_g2l.find(net.src[k]);
		if(is == m_g2l.end()) NB_THROW(NEMO_INVALID_INPUT, "Non-existing neuron index %u", net.src[k]);
		auto it = m_g2l.find(net.tgt[k]);
		if(it == m_g2l.end()) NB_THROW(NEMO_INVALID_INPUT, "Non-existing neuron index %u", net.tgt[k]);
		lsrc[k] = is->second;
		ltgt[k] = it->second;
		fxw[k] = fx_toFix(net.weight[k]);
	}
	// stable counting sort by (local source, delay)
	const unsigned D = std::max(1u, m_maxDelay);
	std::vector<uint64_t> rowStart((size_t) N * D + 1, 0);
	for(size_t k = 0; k < Sn; ++k) rowStart[(size_t) lsrc[k] * D + net.delay[k]]++;
	for(size_t r = 0; r < (size_t) N * D; ++r) rowStart[r + 1] += rowStart[r];
	m_pos.resize(Sn);
	{
		std::vector<uint64_t> fill(rowStart.begin(), rowStart.end() - 1);
		for(size_t k = 0; k < Sn; ++k) m_pos[k] = fill[(size_t) lsrc[k] * D + net.delay[k] - 1]++;
	}
	std::vector<unsigned long long> outPtr(N + 1);
	for(unsigned s = 0; s <= N; ++s) outPtr[s] = rowStart[(size_t) s * D];
	m_outDegree.resize(N);
	for(unsigned s = 0; s < N; ++s) {
		m_outDegree[s] = (uint32_t) (outPtr[s + 1] - outPtr[s]);
		m_maxOutDeg = std::max(m_maxOutDeg, m_outDegree[s]);
	}
	std::vector<uint2> syn(Sn);
	for(size_t k = 0; k < Sn; ++k) {
		syn[m_pos[k]] = make_uint2(ltgt[k] | ((net.delay[k] - 1) << 26), (uint32_t) fxw[k]);
	}
	rowStart.clear();
	rowStart.shrink_to_fit();
	auto* dOut = dalloc<unsigned long long>(N + 1);
	auto* dSyn = dalloc<uint2>(Sn);
	NB_CUDA(cudaMemcpyAsync(dOut, outPtr.data(), (N + 1) * 8, cudaMemcpyHostToDevice, m_stream));
	NB_CUDA(cudaMemcpyAsync(dSyn, syn.data(), Sn * 8, cudaMemcpyHostToDevice, m_stream));
	S.outPtr = dOut;
	S.syn = dSyn;

	// query tables: per local source, its synapses by per-source index
	if(!m_writeOnly) {
		m_srcStart.assign(N + 1, 0);
		for(size_t k = 0; k < Sn; ++k) m_srcStart[lsrc[k] + 1]++;
		for(unsigned s = 0; s < N; ++s) m_srcStart[s + 1] += m_srcStart[s];
		m_srcOrder.resize(Sn);
		for(size_t k = 0; k < Sn; ++k) m_srcOrder[m_srcStart[lsrc[k]] + net.sid[k]] = k;
		m_synDelay.assign(net.delay.begin(), net.delay.end());
		m_synPlastic.assign(net.plastic.begin(), net.plastic.end());
		m_synTarget.assign(net.tgt.begin(), net.tgt.end());
	}

	// STDP (src/nemo/StdpProcess.cpp:20-46) and the reverse matrix of plastic
	// synapses (src/nemo/construction/RCM.cpp:150-172)
	S.stdp = conf.stdp ? 1 : 0;
	std::vector<unsigned long long> rcmPtr(N + 1, 0);
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

		for(size_t k = 0; k < Sn; ++k) if(net.plastic[k]) rcmPtr[ltgt[k] + 1]++;
		for(unsigned t = 0; t < N; ++t) {
			m_maxPlasticInDeg = std::max(m_maxPlasticInDeg, (uint32_t) rcmPtr[t + 1]);
			rcmPtr[t + 1] += rcmPtr[t];
		}
		size_t P = rcmPtr[N];
		std::vector<uint32_t> rsrc(P), rfwd(P);
		std::vector<unsigned long long> fill(rcmPtr.begin(), rcmPtr.end() - 1);
		for(size_t k = 0; k < Sn; ++k) {
			if(!net.plastic[k]) continue;
			size_t p = fill[ltgt[k]]++;
			rsrc[p] = lsrc[k] | ((net.delay[k] - 1) << 26);
			if(m_pos[k] > 0xffffffffull) NB_THROW(NEMO_API_UNSUPPORTED, "too many synapses for STDP");
			rfwd[p] = (uint32_t) m_pos[k];
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
	auto* dRcmPtr = dalloc<unsigned long long>(N + 1);
	NB_CUDA(cudaMemcpyAsync(dRcmPtr, rcmPtr.data(), (N + 1) * 8, cudaMemcpyHostToDevice, m_stream));
	S.rcmPtr = dRcmPtr;

	// per-neuron RNG, keyed by local index (src/nemo/cpu/Neurons.cpp:41)
	std::vector<uint32_t> planes;
	seed_rng(planes, N);
	S.rng = dalloc<uint32_t>(4 * (size_t) N);
	NB_CUDA(cudaMemcpyAsync(S.rng, planes.data(), planes.size() * 4, cudaMemcpyHostToDevice, m_stream));

	S.hist = dalloc<uint64_t>(2 * (size_t) N);
	S.fstim = dalloc<uint32_t>(S.W);
	S.curExt = dalloc<float>(N);
	// validSpikes = ~(~0 << maxDelay) with x86 shift semantics
	// (src/nemo/cpu/Simulation.cpp:263): nothing is delivered when the
	// maximum delay is 0 or 64
	S.D = (m_maxDelay >= 1 && m_maxDelay <= 63) ? m_maxDelay + 1 : 0;
	S.slots = S.D ? dalloc<longlong2>((size_t) S.D * N) : nullptr;
	S.R = (uint32_t) std::max<size_t>(16, std::min<size_t>(1024, (64u << 20) / ((size_t) S.W * 4)));
	S.firedRing = dalloc<uint32_t>((size_t) S.R * S.W);
	S.firedCount = dalloc<uint32_t>(S.R);
	S.eventCount = dalloc<unsigned long long>(S.R);
	S.stdpCount = dalloc<unsigned long long>(S.R);
	NB_CUDA(cudaMallocHost(&m_hFired, (size_t) S.R * S.W * 4));

	if(needCalib) S.calib = device_calibration(m_device);
	NB_CUDA(cudaDeviceGetAttribute(&m_sms, cudaDevAttrMultiProcessorCount, m_device));
	NB_CUDA(cudaFuncSetAttribute(step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) stepSmem(MAX_PARTITION)));
	NB_CUDA(cudaFuncSetAttribute(stdp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) stepSmem(MAX_PARTITION)));
	// default launch shape: two partitions per SM
	{
		uint32_t P = (uint32_t) ((N + 2 * m_sms - 1) / (2 * m_sms));
		setLaunch(P, std::min<uint32_t>(1024, std::max<uint32_t>(128, (P + 31) & ~31u)));
	}
	NB_CUDA(cudaStreamSynchronize(m_stream));
	resetTimer();
}

Simulation::~Simulation()
{
	cudaSetDevice(m_device);
	if(m_stream) cudaStreamSynchronize(m_stream);
	for(void* p : m_allocs) cudaFree(p);
	if(m_hFired) cudaFreeHost(m_hFired);
	if(m_hStim) cudaFreeHost(m_hStim);
	if(m_dStim) cudaFree(m_dStim);
	if(m_ev0) cudaEventDestroy(m_ev0);
	if(m_ev1) cudaEventDestroy(m_ev1);
	for(cudaEvent_t e : m_evPool) cudaEventDestroy(e);
	if(m_stream) cudaStreamDestroy(m_stream);
}

void Simulation::sync()
{
	NB_CUDA(cudaStreamSynchronize(m_stream));
}

unsigned Simulation::localIdx(unsigned g) const
{
	auto it = m_g2l.find(g);
	if(it == m_g2l.end()) NB_THROW(NEMO_INVALID_INPUT, "Non-existing neuron index %u", g);
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

size_t Simulation::stepSmem(uint32_t P) const
{
	size_t list = ((size_t) 8 * P + 4 * P + 4 * (P + 1) + 15) & ~(size_t) 15;
	return 2 * list;
}

void Simulation::setLaunch(uint32_t P, uint32_t T)
{
	P = std::max<uint32_t>(32, std::min<uint32_t>(MAX_PARTITION, (P + 31) & ~31u));
	T = std::max<uint32_t>(32, std::min<uint32_t>(1024, (T + 31) & ~31u));
	// the per-CTA work offsets are 32-bit
	while(P > 32 && ((uint64_t) P * std::max(m_maxOutDeg, m_maxPlasticInDeg) >= (1ull << 31))) P -= 32;
	m_P = P;
	m_T = T;
}

void Simulation::launchStep(bool /*fullRecord*/)
{
	const uint32_t cur = (uint32_t) (m_cycle & 1);
	const uint32_t slot = m_dev.D ? (uint32_t) (m_cycle % m_dev.D) : 0;
	const uint32_t ring = (uint32_t) (m_cycle % m_dev.R);
	const unsigned grid = (m_N + m_P - 1) / m_P;
	timedBegin(K_STEP);
	step_kernel<<<grid, m_T, stepSmem(m_P), m_stream>>>(m_dev, m_P, cur, slot, ring, m_stdpPending ? 1 : 0);
	timedEnd();
	m_stdpPending = m_dev.stdp != 0;
	m_cycle++;
	m_timerSteps++;
}

const std::vector<unsigned>& Simulation::step(const unsigned* fstim, size_t nf,
		const unsigned* inidx, const float* icur, size_t ni)
{
	NB_CUDA(cudaSetDevice(m_device));
	// validate and map the stimulus before touching any state
	// (src/nemo/cpu/Simulation.cpp:141-163; the last current for a neuron wins)
	size_t nstim = nf + 2 * ni;
	if(nstim) {
		std::vector<uint32_t> fl(nf);
		for(size_t i = 0; i < nf; ++i) fl[i] = localIdx(fstim[i]);
		std::unordered_map<uint32_t, float> cur;
		std::vector<uint32_t> corder;
		for(size_t i = 0; i < ni; ++i) {
			uint32_t l = localIdx(inidx[i]);
			if(cur.find(l) == cur.end()) corder.push_back(l);
			cur[l] = icur[i];
		}
		size_t need = nf + 2 * corder.size();
		if(need > m_stimCap) {
			if(m_hStim) cudaFreeHost(m_hStim);
			if(m_dStim) cudaFree(m_dStim);
			m_stimCap = std::max<size_t>(need, 1024);
			NB_CUDA(cudaMallocHost(&m_hStim, m_stimCap * 4));
			NB_CUDA(cudaMalloc(&m_dStim, m_stimCap * 4));
		}
		else {
			sync(); // the staging buffer may still be in flight
		}
		memcpy(m_hStim, fl.data(), nf * 4);
		for(size_t i = 0; i < corder.size(); ++i) {
			m_hStim[nf + i] = corder[i];
			float v = cur[corder[i]];
			memcpy(&m_hStim[nf + corder.size() + i], &v, 4);
		}
		NB_CUDA(cudaMemcpyAsync(m_dStim, m_hStim, need * 4, cudaMemcpyHostToDevice, m_stream));
		uint32_t nmax = (uint32_t) std::max(nf, corder.size());
		stimulus_kernel<<<(nmax + 255) / 256, 256, 0, m_stream>>>(m_dev, m_dStim, (uint32_t) nf,
				m_dStim + nf, reinterpret_cast<const float*>(m_dStim + nf + corder.size()), (uint32_t) corder.size());
	}
	const uint32_t ring = (uint32_t) (m_cycle % m_dev.R);
	launchStep(true);
	NB_CUDA(cudaMemcpyAsync(m_hFired, m_dev.firedRing + (size_t) ring * m_dev.W, (size_t) m_dev.W * 4,
			cudaMemcpyDeviceToHost, m_stream));
	sync();
	NB_CUDA(cudaGetLastError());
	// fired neurons in ascending local index, as global ids
	// (setFiring, src/nemo/cpu/Simulation.cpp:200-208)
	m_fired.clear();
	for(uint32_t w = 0; w < m_dev.W; ++w) {
		uint32_t bits = m_hFired[w];
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

void Simulation::flushStdp()
{
	if(!m_stdpPending) return;
	const uint32_t par = (uint32_t) ((m_cycle - 1) & 1);
	const unsigned grid = (m_N + m_P - 1) / m_P;
	timedBegin(K_STDP);
	stdp_kernel<<<grid, m_T, stepSmem(m_P) / 2, m_stream>>>(m_dev, m_P, par, (uint32_t) ((m_cycle - 1) % m_dev.R));
	timedEnd();
	m_stdpPending = false;
}

void Simulation::applyStdpDevice(int32_t R)
{
	flushStdp();
	// the last completed step's history and slot; before the first step
	// the history is all zero, so nothing is in flight
	const uint64_t last = m_cycle ? m_cycle - 1 : 0;
	const uint32_t par = (uint32_t) (last & 1);
	const uint32_t slot = m_dev.D ? (uint32_t) (last % m_dev.D) : 0;
	int sms = 148;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m_device);
	unsigned grid = std::min<unsigned>((m_N + 7) / 8, (unsigned) sms * 8);
	timedBegin(K_APPLY);
	apply_stdp_kernel<<<grid, STEP_THREADS, 0, m_stream>>>(m_dev, R, par, slot, m_weightsClamped ? 0 : 1);
	timedEnd();
	// updatedWeight's result always lies within the clamp range of its sign
	// class, so after one full pass every plastic weight does
	m_weightsClamped = true;
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
		for(unsigned i = 0; i < chunk; ++i) {
			launchStep(false);
			if(stdpPeriod && (done + i + 1) % stdpPeriod == 0) applyStdpDevice(R);
		}
		NB_CUDA(cudaEventRecord(m_ev1, m_stream));
		std::vector<uint32_t> hc(m_dev.R);
		std::vector<unsigned long long> he(m_dev.R), hs(m_dev.R);
		NB_CUDA(cudaMemcpyAsync(hc.data(), m_dev.firedCount, m_dev.R * 4, cudaMemcpyDeviceToHost, m_stream));
		NB_CUDA(cudaMemcpyAsync(he.data(), m_dev.eventCount, m_dev.R * 8, cudaMemcpyDeviceToHost, m_stream));
		NB_CUDA(cudaMemcpyAsync(hs.data(), m_dev.stdpCount, m_dev.R * 8, cudaMemcpyDeviceToHost, m_stream));
		if(ids) {
			NB_CUDA(cudaMemcpyAsync(m_hFired, m_dev.firedRing, (size_t) m_dev.R * m_dev.W * 4,
					cudaMemcpyDeviceToHost, m_stream));
		}
		sync();
		NB_CUDA(cudaGetLastError());
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
			if(counts) counts[done + i] = hc[r];
			if(events) events[done + i] = he[r];
			lastFired += hc[r];
			lastEvents += he[r];
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
		}
		done += chunk;
	}
	if(len) *len = total;
	lastRunMs = runMs;
}

float Simulation::autotune(unsigned trialSteps)
{
	NB_CUDA(cudaSetDevice(m_device));
	sync();
	trialSteps = std::max(1u, trialSteps);
	// the state that trial steps modify
	std::vector<std::pair<void*, size_t>> regions;
	for(const HostType& t : m_types) regions.emplace_back(t.dState, (size_t) t.n * t.desc->nstate * 4);
	regions.emplace_back(m_dev.rng, (size_t) 4 * m_N * 4);
	regions.emplace_back(m_dev.hist, (size_t) 2 * m_N * 8);
	regions.emplace_back(m_dev.fstim, (size_t) m_dev.W * 4);
	regions.emplace_back(m_dev.curExt, (size_t) m_N * 4);
	if(m_dev.D) regions.emplace_back(m_dev.slots, (size_t) m_dev.D * m_N * 16);
	if(m_dev.stdp) regions.emplace_back(m_dev.rcmAcc, (size_t) lastPlastic * 4);
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
	const bool pending = m_stdpPending;
	const unsigned long timerSteps = m_timerSteps;
	const bool prof = profiling;
	profiling = false;
	auto restore = [&]() {
		for(size_t i = 0; i < regions.size(); ++i) {
			if(backup[i]) {
				NB_CUDA(cudaMemcpyAsync(regions[i].first, backup[i], regions[i].second, cudaMemcpyDeviceToDevice, m_stream));
			}
		}
		m_cycle = cycle;
		m_stdpPending = pending;
		m_timerSteps = timerSteps;
	};

	// candidates: 1 to 16 partitions per SM, 128 to 1024 threads per CTA
	std::vector<std::pair<uint32_t, uint32_t>> cands;
	for(unsigned k : {1u, 2u, 3u, 4u, 6u, 8u, 12u, 16u}) {
		uint32_t P = (uint32_t) ((m_N + (size_t) k * m_sms - 1) / ((size_t) k * m_sms));
		P = std::max<uint32_t>(32, std::min<uint32_t>(MAX_PARTITION, (P + 31) & ~31u));
		for(uint32_t T : {128u, 256u, 512u, 1024u}) {
			if(T > std::max<uint32_t>(128, P)) continue;
			if(std::find(cands.begin(), cands.end(), std::make_pair(P, T)) == cands.end()) cands.emplace_back(P, T);
		}
	}
	const uint32_t P0 = m_P, T0 = m_T;
	float best = -1;
	uint32_t bestP = P0, bestT = T0;
	try {
		for(auto& c : cands) {
			setLaunch(c.first, c.second);
			launchStep(false); // untimed warm-up of this shape
			NB_CUDA(cudaEventRecord(m_ev0, m_stream));
			for(unsigned i = 0; i < trialSteps; ++i) launchStep(false);
			NB_CUDA(cudaEventRecord(m_ev1, m_stream));
			sync();
			NB_CUDA(cudaGetLastError());
			float ms = 0;
			NB_CUDA(cudaEventElapsedTime(&ms, m_ev0, m_ev1));
			if(best < 0 || ms < best) {
				best = ms;
				bestP = m_P;
				bestT = m_T;
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

float Simulation::getNeuronState(unsigned g, unsigned var)
{
	const HostType* t; unsigned i;
	locate(g, &t, &i);
	if(var >= t->desc->nstate) NB_THROW(NEMO_INVALID_INPUT, "Invalid state variable index %u", var);
	float v;
	NB_CUDA(cudaSetDevice(m_device));
	NB_CUDA(cudaMemcpyAsync(&v, t->dState + (size_t) var * t->n + i, 4, cudaMemcpyDeviceToHost, m_stream));
	sync();
	return v;
}

float Simulation::getNeuronParameter(unsigned g, unsigned p)
{
	const HostType* t; unsigned i;
	locate(g, &t, &i);
	if(p >= t->desc->nparam) NB_THROW(NEMO_INVALID_INPUT, "Invalid parameter index %u", p);
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
	return getNeuronState(g, t->desc->mpot);
}

void Simulation::setNeuron(unsigned g, unsigned nargs, const float* args)
{
	const HostType* t; unsigned i;
	locate(g, &t, &i);
	unsigned np = t->desc->nparam, ns = t->desc->nstate;
	if(nargs != np + ns) {
		NB_THROW(NEMO_INVALID_INPUT,
				"Unexpected number of parameters/state variables when modifying neuron. Expected %u, found %u", np + ns, nargs);
	}
	NB_CUDA(cudaSetDevice(m_device));
	for(unsigned p = 0; p < np; ++p) {
		NB_CUDA(cudaMemcpyAsync(t->dParam + (size_t) p * t->n + i, args + p, 4, cudaMemcpyHostToDevice, m_stream));
	}
	for(unsigned v = 0; v < ns; ++v) {
		NB_CUDA(cudaMemcpyAsync(t->dState + (size_t) v * t->n + i, args + np + v, 4, cudaMemcpyHostToDevice, m_stream));
	}
	sync();
}

void Simulation::setNeuronState(unsigned g, unsigned var, float v)
{
	const HostType* t; unsigned i;
	locate(g, &t, &i);
	if(var >= t->desc->nstate) NB_THROW(NEMO_INVALID_INPUT, "Invalid state variable index %u", var);
	NB_CUDA(cudaSetDevice(m_device));
	NB_CUDA(cudaMemcpyAsync(t->dState + (size_t) var * t->n + i, &v, 4, cudaMemcpyHostToDevice, m_stream));
	sync();
}

void Simulation::setNeuronParameter(unsigned g, unsigned p, float v)
{
	const HostType* t; unsigned i;
	locate(g, &t, &i);
	if(p >= t->desc->nparam) NB_THROW(NEMO_INVALID_INPUT, "Invalid parameter index %u", p);
	NB_CUDA(cudaSetDevice(m_device));
	NB_CUDA(cudaMemcpyAsync(t->dParam + (size_t) p * t->n + i, &v, 4, cudaMemcpyHostToDevice, m_stream));
	sync();
}

/* src/nemo/ConnectivityMatrix.cpp:298-331 */
const std::vector<uint64_t>& Simulation::getSynapsesFrom(unsigned source)
{
	if(m_writeOnly) NB_THROW(NEMO_INVALID_INPUT, "Cannot read synapse state if simulation configured with write-only synapses");
	auto it = m_g2l.find(source);
	if(it == m_g2l.end()) NB_THROW(NEMO_INVALID_INPUT, "Non-existing source neuron id (%u) in synapse id query", source);
	uint64_t n = m_srcStart[it->second + 1] - m_srcStart[it->second];
	m_queried.resize(n);
	for(uint64_t i = 0; i < n; ++i) m_queried[i] = ((uint64_t) source << 32) | i;
	return m_queried;
}

/* ConnectivityMatrix::axonTerminalAux (src/nemo/ConnectivityMatrix.cpp:343-360) */
size_t Simulation::synapseKey(uint64_t id) const
{
	if(m_writeOnly) NB_THROW(NEMO_INVALID_INPUT, "Cannot read synapse state if simulation configured with write-only synapses");
	unsigned source = (unsigned) (id >> 32);
	uint32_t s = (uint32_t) (id & 0xffffffffu);
	auto it = m_g2l.find(source);
	if(it == m_g2l.end() || m_srcStart[it->second + 1] == m_srcStart[it->second]) {
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
	uint2 s;
	NB_CUDA(cudaSetDevice(m_device));
	NB_CUDA(cudaMemcpyAsync(&s, m_dev.syn + m_pos[k], 8, cudaMemcpyDeviceToHost, m_stream));
	sync();
	return fx_toFloat((int32_t) s.y);
}

void Simulation::getWeightsFx(int32_t* out, size_t cap, size_t* len)
{
	if(m_writeOnly) NB_THROW(NEMO_INVALID_INPUT, "Cannot read synapse state if simulation configured with write-only synapses");
	if(cap < m_nsyn) NB_THROW(NEMO_BUFFER_OVERFLOW, "weight buffer too small");
	std::vector<uint2> syn(m_nsyn);
	NB_CUDA(cudaSetDevice(m_device));
	NB_CUDA(cudaMemcpyAsync(syn.data(), m_dev.syn, m_nsyn * 8, cudaMemcpyDeviceToHost, m_stream));
	sync();
	// network iteration order: sources by ascending global id
	std::vector<unsigned> sources(m_N);
	for(unsigned l = 0; l < m_N; ++l) sources[l] = l;
	std::sort(sources.begin(), sources.end(), [&](unsigned a, unsigned b) { return m_l2g[a] < m_l2g[b]; });
	size_t o = 0;
	for(unsigned l : sources) {
		for(uint64_t j = m_srcStart[l]; j < m_srcStart[l + 1]; ++j) {
			out[o++] = (int32_t) syn[m_pos[m_srcOrder[j]]].y;
		}
	}
	*len = o;
}

void Simulation::getTypeState(unsigned netType, float* out, size_t cap, size_t* len)
{
	for(const HostType& t : m_types) {
		if(t.netType != netType) continue;
		size_t n = (size_t) t.n * t.desc->nstate;
		if(cap < n) NB_THROW(NEMO_BUFFER_OVERFLOW, "state buffer too small");
		NB_CUDA(cudaSetDevice(m_device));
		NB_CUDA(cudaMemcpyAsync(out, t.dState, n * 4, cudaMemcpyDeviceToHost, m_stream));
		sync();
		*len = n;
		return;
	}
	*len = 0;
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
