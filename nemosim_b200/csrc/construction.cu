// construction.cu -- the connectivity of one network built on the device
// (construction.hpp).  The synapse arrays are uploaded once; the global ids
// are mapped to local indices through a dense table; a stable radix sort by
// (local source, delay) gives every synapse its place in the forward matrix
// -- the host build's counting sort, which keeps insertion order within a
// row -- and a stable radix sort of the plastic synapses, taken in forward
// order, by target gives the reverse matrix in forward order within a
// target.  The sorts are CUB's (construction is not the step loop).
#include "construction.hpp"

#include <cub/cub.cuh>

#include <algorithm>
#include <stdexcept>

#include "common.hpp"

namespace nemo_b200 {

namespace {

#define CC_CUDA(call)                                                                    \
	do {                                                                                 \
		cudaError_t err_ = (call);                                                       \
		if(err_ != cudaSuccess) {                                                        \
			NB_THROW(NEMO_CUDA_ERROR, "CUDA error %s in network construction (%s)",      \
					cudaGetErrorString(err_), #call);                                    \
		}                                                                                \
	} while(0)

// temporary device buffers, freed at the end of the build
struct Scratch {
	std::vector<void*> ptrs;
	~Scratch() { for(void* p : ptrs) cudaFree(p); }
	template<typename T> T* get(size_t n)
	{
		void* p = nullptr;
		CC_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
		ptrs.push_back(p);
		return static_cast<T*>(p);
	}
	// hands one buffer over to the caller (no longer freed here)
	template<typename T> T* release(T* p)
	{
		ptrs.erase(std::find(ptrs.begin(), ptrs.end(), (void*) p));
		return p;
	}
};

constexpr unsigned THREADS = 256;
constexpr uint32_t TARGET_MASK = (1u << 26) - 1;  // a forward entry's target bits

unsigned blocks(size_t n)
{
	return (unsigned) std::max<size_t>(1, std::min<size_t>((n + THREADS - 1) / THREADS, 148u * 64u));
}

// the first error in insertion order, as the host build meets it: synapse
// index << 2 | code (1: source, 2: target, 3: weight)
__device__ void report(unsigned long long* err, unsigned code, size_t k)
{
	atomicMin(err, ((unsigned long long) k << 2) | code);
}

// fx_toFix (src/nemo/fixedpoint.cpp:17-28) as the x86-64 host evaluates it:
// the truncating conversions give INT32_MIN for NaN and out-of-range values
__device__ __forceinline__ bool fx_to_fix(float f, int32_t& out)
{
	const bool inRange = fabsf(f) < 2147483648.0f;
	const int i = inRange ? __float2int_rz(f) : INT32_MIN;
	if(i != INT32_MIN && abs(i) >= (1 << (31 - FRACTIONAL_BITS))) return false;
	const float s = __fmul_rn(f, (float) (1 << FRACTIONAL_BITS));
	out = fabsf(s) < 2147483648.0f ? __float2int_rz(s) : INT32_MIN;
	return true;
}

__global__ void map_kernel(size_t S, const unsigned* src, const unsigned* tgt, const unsigned* delay,
		const float* weight, const uint32_t* g2l, uint32_t maxGid, uint32_t srcBase, uint32_t D, uint32_t* ls,
		uint32_t* lt, int32_t* fx, uint32_t* key, uint32_t* idx, uint32_t* rowCount, unsigned long long* err)
{
	for(size_t k = blockIdx.x * (size_t) blockDim.x + threadIdx.x; k < S; k += (size_t) gridDim.x * blockDim.x) {
		const unsigned s = src[k], t = tgt[k];
		const uint32_t a = s <= maxGid ? g2l[s] : ~0u;
		const uint32_t b = t <= maxGid ? g2l[t] : ~0u;
		int32_t w = 0;
		if(a == ~0u) report(err, 1, k);
		if(b == ~0u) report(err, 2, k);
		if(!fx_to_fix(weight[k], w)) report(err, 3, k);
		if(a == ~0u || b == ~0u) continue;
		const uint32_t r = (a - srcBase) * D + (delay[k] - 1);
		ls[k] = a;
		lt[k] = b;
		fx[k] = w;
		key[k] = r;
		idx[k] = (uint32_t) k;
		atomicAdd(rowCount + r, 1u);
	}
}

// synTgt, synW: the network's part of the union forward matrix; pos: each synapse's
// place in it
__global__ void fill_forward_kernel(size_t S, const uint32_t* sortedIdx, const uint32_t* lt, const unsigned* delay,
		const int32_t* fx, uint32_t* synTgt, uint32_t* synW, uint32_t* pos)
{
	for(size_t p = blockIdx.x * (size_t) blockDim.x + threadIdx.x; p < S; p += (size_t) gridDim.x * blockDim.x) {
		const uint32_t k = sortedIdx[p];
		synTgt[p] = lt[k] | ((delay[k] - 1) << 26);
		synW[p] = (uint32_t) fx[k];
		pos[k] = (uint32_t) p;
	}
}

// per source s of the network (union index srcBase + s): its row start, the
// end of each delay's group within the row, and the delays deliverSpikes
// delivers (OutgoingDelays.cpp:70-80)
__global__ void groups_kernel(uint32_t n, uint32_t srcBase, uint64_t synOff, uint32_t D, bool deliver,
		const uint32_t* rowStart, unsigned long long* outPtr, uint16_t* end16, uint32_t* end32, uint64_t* delayMask,
		unsigned long long* groups)
{
	for(uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
		const uint32_t base = rowStart[(size_t) s * D];
		const size_t u = (size_t) srcBase + s;
		uint32_t prev = 0;
		uint64_t mask = 0;
		unsigned long long g = 0;
		for(uint32_t d = 1; d <= D; ++d) {
			const uint32_t e = rowStart[(size_t) s * D + d] - base;
			if(end16) end16[u * D + d - 1] = (uint16_t) e;
			else end32[u * D + d - 1] = e;
			if(deliver && e > prev) {
				mask |= 1ull << (d - 1);
				++g;
			}
			prev = e;
		}
		outPtr[u] = synOff + base;
		delayMask[u] = mask;
		if(g) atomicAdd(groups, g);
	}
}

// flag[p]: forward entry p is plastic (sortedIdx[p] is its insertion index)
__global__ void flag_kernel(size_t S, const uint32_t* sortedIdx, const uint8_t* plastic, uint32_t* flag)
{
	for(size_t p = blockIdx.x * (size_t) blockDim.x + threadIdx.x; p <= S; p += (size_t) gridDim.x * blockDim.x) {
		flag[p] = p < S && plastic[sortedIdx[p]] ? 1u : 0u;
	}
}

// the plastic forward entries in forward order (at their exclusive-scan
// positions)
__global__ void compact_kernel(size_t S, const uint32_t* flag, const uint32_t* at, uint32_t* plf)
{
	for(size_t p = blockIdx.x * (size_t) blockDim.x + threadIdx.x; p < S; p += (size_t) gridDim.x * blockDim.x) {
		if(flag[p]) plf[at[p]] = (uint32_t) p;
	}
}

// key2: the plastic entry's target relative to the network's first neuron
__global__ void plastic_keys_kernel(size_t P, const uint32_t* plf, const uint32_t* synTgt, uint32_t srcBase,
		uint32_t* key2, uint32_t* tgtCount)
{
	for(size_t q = blockIdx.x * (size_t) blockDim.x + threadIdx.x; q < P; q += (size_t) gridDim.x * blockDim.x) {
		const uint32_t t = (synTgt[plf[q]] & TARGET_MASK) - srcBase;
		key2[q] = t;
		atomicAdd(tgtCount + t, 1u);
	}
}

// rsrc, rfwd: the network's part of the union reverse matrix
__global__ void fill_reverse_kernel(size_t P, const uint32_t* sortedPlf, const uint32_t* sortedIdx,
		const uint32_t* ls, const uint32_t* synTgt, uint64_t synOff, uint32_t* rsrc, uint32_t* rfwd)
{
	for(size_t q = blockIdx.x * (size_t) blockDim.x + threadIdx.x; q < P; q += (size_t) gridDim.x * blockDim.x) {
		const uint32_t p = sortedPlf[q];
		rsrc[q] = ls[sortedIdx[p]] | (synTgt[p] & ~TARGET_MASK);
		rfwd[q] = (uint32_t) (synOff + p);
	}
}

__global__ void narrow_kernel(size_t S, const unsigned* delay, uint8_t* d8)
{
	for(size_t k = blockIdx.x * (size_t) blockDim.x + threadIdx.x; k < S; k += (size_t) gridDim.x * blockDim.x) {
		d8[k] = (uint8_t) delay[k];
	}
}

// splitmix64 finaliser
__device__ __forceinline__ uint64_t mix64(uint64_t x)
{
	x += 0x9e3779b97f4a7c15ull;
	x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
	x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
	return x ^ (x >> 31);
}

__global__ void digest_kernel(const uint8_t* p, size_t bytes, unsigned long long* out)
{
	unsigned long long acc = 0;
	const size_t words = bytes / 4;
	const uint32_t* w = reinterpret_cast<const uint32_t*>(p);
	for(size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < words; i += (size_t) gridDim.x * blockDim.x) {
		acc += mix64(((uint64_t) i << 32) ^ w[i]);
	}
	if(blockIdx.x == 0 && threadIdx.x == 0) {
		for(size_t i = words * 4; i < bytes; ++i) acc += mix64(((uint64_t) i << 40) ^ p[i]);
	}
	atomicAdd(out, acc);
}

template<typename T>
T* upload(Scratch& scratch, const T* host, size_t n, cudaStream_t st)
{
	T* d = scratch.get<T>(n);
	if(n) CC_CUDA(cudaMemcpyAsync(d, host, n * sizeof(T), cudaMemcpyHostToDevice, st));
	return d;
}

} // namespace

void construct_on_device(DeviceConstruction& c, cudaStream_t st)
{
	Scratch scratch;
	const size_t S = c.S;
	const uint32_t N = c.nLocal, D = c.D;
	const size_t rows = (size_t) N * D;
	if(S >= (1ull << 31) - 1 || rows >= (1ull << 31) - 1) {
		NB_THROW(NEMO_API_UNSUPPORTED, "network too large for the device build");
	}
	unsigned* src = upload(scratch, c.src, S, st);
	unsigned* tgt = upload(scratch, c.tgt, S, st);
	unsigned* dly = upload(scratch, c.delay, S, st);
	float* wgt = upload(scratch, c.weight, S, st);
	uint8_t* pl = upload(scratch, reinterpret_cast<const uint8_t*>(c.plastic), S, st);
	uint32_t* g2l = upload(scratch, c.g2l, (size_t) c.maxGid + 1, st);

	uint32_t* ls = scratch.get<uint32_t>(S);
	uint32_t* lt = scratch.get<uint32_t>(S);
	int32_t* fx = scratch.get<int32_t>(S);
	uint32_t* key = scratch.get<uint32_t>(S);
	uint32_t* idx = scratch.get<uint32_t>(S);
	uint32_t* rowCount = scratch.get<uint32_t>(rows + 1);
	uint32_t* rowStart = scratch.get<uint32_t>(rows + 1);
	unsigned long long* err = scratch.get<unsigned long long>(2);
	CC_CUDA(cudaMemsetAsync(rowCount, 0, (rows + 1) * 4, st));
	CC_CUDA(cudaMemsetAsync(err, 0xff, 8, st));
	CC_CUDA(cudaMemsetAsync(err + 1, 0, 8, st));
	map_kernel<<<blocks(S), THREADS, 0, st>>>(S, src, tgt, dly, wgt, g2l, c.maxGid, c.srcBase, D, ls, lt, fx, key,
			idx, rowCount, err);
	CC_CUDA(cudaGetLastError());
	unsigned long long herr = 0;
	CC_CUDA(cudaMemcpyAsync(&herr, err, 8, cudaMemcpyDeviceToHost, st));
	CC_CUDA(cudaStreamSynchronize(st));
	if(herr != ~0ull) {
		const unsigned code = (unsigned) (herr & 3);
		const size_t k = (size_t) (herr >> 2);
		if(code == 1) NB_THROW(NEMO_INVALID_INPUT, "Non-existing neuron index %u", c.src[k]);
		if(code == 2) NB_THROW(NEMO_INVALID_INPUT, "Non-existing neuron index %u", c.tgt[k]);
		throw std::runtime_error(format("Fixed-point overflow. Value %g does not fit into fixed-point format Q%u.%u",
				(double) c.weight[k], 31 - FRACTIONAL_BITS, FRACTIONAL_BITS));
	}

	// row starts (exclusive scan of the counts; the last entry is S)
	size_t tmpBytes = 0;
	CC_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmpBytes, rowCount, rowStart, (int) (rows + 1), st));
	void* tmp = scratch.get<uint8_t>(tmpBytes);
	CC_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmpBytes, rowCount, rowStart, (int) (rows + 1), st));

	// stable sort by row: insertion order within a row
	int keyBits = 1;
	while(keyBits < 32 && (1ull << keyBits) < rows) ++keyBits;
	uint32_t* keySorted = scratch.get<uint32_t>(S);
	uint32_t* idxSorted = scratch.get<uint32_t>(S);
	tmpBytes = 0;
	CC_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmpBytes, key, keySorted, idx, idxSorted, (int) S, 0, keyBits,
			st));
	tmp = scratch.get<uint8_t>(tmpBytes);
	CC_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tmpBytes, key, keySorted, idx, idxSorted, (int) S, 0, keyBits, st));

	uint32_t* synTgt = c.synTgt + c.synOff;
	uint32_t* synW = c.synW + c.synOff;
	uint32_t* pos = scratch.get<uint32_t>(S);
	fill_forward_kernel<<<blocks(S), THREADS, 0, st>>>(S, idxSorted, lt, dly, fx, synTgt, synW, pos);
	CC_CUDA(cudaGetLastError());

	// delay groups
	unsigned long long* groups = err + 1;
	groups_kernel<<<blocks(N), THREADS, 0, st>>>(N, c.srcBase, c.synOff, D, c.deliver, rowStart, c.outPtr, c.dEnd16,
			c.dEnd32, c.delayMask, groups);
	CC_CUDA(cudaGetLastError());
	std::vector<uint32_t> hostRowStart(rows + 1);
	CC_CUDA(cudaMemcpyAsync(hostRowStart.data(), rowStart, (rows + 1) * 4, cudaMemcpyDeviceToHost, st));
	unsigned long long hg = 0;
	CC_CUDA(cudaMemcpyAsync(&hg, groups, 8, cudaMemcpyDeviceToHost, st));
	CC_CUDA(cudaStreamSynchronize(st));
	c.hostOutPtr.resize(N);
	for(uint32_t s = 0; s < N; ++s) c.hostOutPtr[s] = c.synOff + hostRowStart[(size_t) s * D];

	// the reverse matrix of plastic synapses, in forward order within a
	// target
	c.hostRcmPtr.assign(N, c.plOff);
	c.plastic_count = 0;
	if(c.stdp) {
		uint32_t* flag = scratch.get<uint32_t>(S + 1);
		uint32_t* at = scratch.get<uint32_t>(S + 1);
		flag_kernel<<<blocks(S + 1), THREADS, 0, st>>>(S, idxSorted, pl, flag);
		CC_CUDA(cudaGetLastError());
		tmpBytes = 0;
		CC_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmpBytes, flag, at, (int) (S + 1), st));
		tmp = scratch.get<uint8_t>(tmpBytes);
		CC_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmpBytes, flag, at, (int) (S + 1), st));
		uint32_t hsel = 0;
		CC_CUDA(cudaMemcpyAsync(&hsel, at + S, 4, cudaMemcpyDeviceToHost, st));
		CC_CUDA(cudaStreamSynchronize(st));
		const size_t P = hsel;
		uint32_t* plk = scratch.get<uint32_t>(P);
		compact_kernel<<<blocks(S), THREADS, 0, st>>>(S, flag, at, plk);
		CC_CUDA(cudaGetLastError());
		uint32_t* key2 = scratch.get<uint32_t>(P);
		uint32_t* tgtCount = scratch.get<uint32_t>((size_t) N + 1);
		uint32_t* tgtStart = scratch.get<uint32_t>((size_t) N + 1);
		CC_CUDA(cudaMemsetAsync(tgtCount, 0, ((size_t) N + 1) * 4, st));
		plastic_keys_kernel<<<blocks(P), THREADS, 0, st>>>(P, plk, synTgt, c.srcBase, key2, tgtCount);
		CC_CUDA(cudaGetLastError());
		tmpBytes = 0;
		CC_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmpBytes, tgtCount, tgtStart, (int) N + 1, st));
		tmp = scratch.get<uint8_t>(tmpBytes);
		CC_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmpBytes, tgtCount, tgtStart, (int) N + 1, st));
		int tBits = 1;
		while(tBits < 32 && (1ull << tBits) < N) ++tBits;
		uint32_t* key2Sorted = scratch.get<uint32_t>(P);
		uint32_t* plkSorted = scratch.get<uint32_t>(P);
		tmpBytes = 0;
		CC_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmpBytes, key2, key2Sorted, plk, plkSorted, (int) P, 0,
				tBits, st));
		tmp = scratch.get<uint8_t>(tmpBytes);
		CC_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tmpBytes, key2, key2Sorted, plk, plkSorted, (int) P, 0, tBits,
				st));
		fill_reverse_kernel<<<blocks(P), THREADS, 0, st>>>(P, plkSorted, idxSorted, ls, synTgt, c.synOff,
				c.rcmSrc + c.plOff, c.rcmFwd + c.plOff);
		CC_CUDA(cudaGetLastError());
		std::vector<uint32_t> hs((size_t) N + 1);
		CC_CUDA(cudaMemcpyAsync(hs.data(), tgtStart, ((size_t) N + 1) * 4, cudaMemcpyDeviceToHost, st));
		CC_CUDA(cudaStreamSynchronize(st));
		for(size_t i = 0; i < N; ++i) c.hostRcmPtr[i] = c.plOff + hs[i];
		c.plastic_count = P;
	}

	// what the synapse queries need, kept on the device until first used
	// (the scratch arrays themselves, handed over to the caller)
	if(c.keepQueries) {
		c.keptDelay = scratch.get<uint8_t>(S);
		narrow_kernel<<<blocks(S), THREADS, 0, st>>>(S, dly, c.keptDelay);
		CC_CUDA(cudaGetLastError());
		c.keptSrc = scratch.release(ls);
		c.keptPos = scratch.release(pos);
		c.keptTgt = scratch.release(tgt);
		c.keptDelay = scratch.release(c.keptDelay);
		c.keptPlastic = scratch.release(pl);
	}
	CC_CUDA(cudaStreamSynchronize(st));
	c.dlvGroups = hg;
}

uint64_t device_digest(const void* p, size_t bytes, cudaStream_t st)
{
	if(!p || !bytes) return 0;
	Scratch scratch;
	unsigned long long* out = scratch.get<unsigned long long>(1);
	CC_CUDA(cudaMemsetAsync(out, 0, 8, st));
	digest_kernel<<<148 * 8, THREADS, 0, st>>>(static_cast<const uint8_t*>(p), bytes, out);
	CC_CUDA(cudaGetLastError());
	unsigned long long h = 0;
	CC_CUDA(cudaMemcpyAsync(&h, out, 8, cudaMemcpyDeviceToHost, st));
	CC_CUDA(cudaStreamSynchronize(st));
	return h;
}

} // namespace nemo_b200
