// probe.cu -- a measurement of the scattered-update floor that bounds the
// step's pre-phase: each delivered spike adds its weight into one 16-byte
// accumulator slot of its target, at an index that is effectively random.
// The probe issues `ops` such operations into `elements` slots (64-bit
// reductions, 32-bit reductions, or 8-byte loads for comparison) from a
// grid of `ctas` CTAs of 256 threads and times the launches with CUDA
// events on its own stream.
#include "probe.hpp"

#include <cuda_runtime.h>

#include <algorithm>

#include "common.hpp"

namespace nemo_b200 {

namespace {

__device__ __forceinline__ uint32_t scatter_index(uint32_t i, uint32_t elements)
{
	// a multiplicative hash, then a range reduction by multiply-high
	const uint32_t h = (i + 0x9e3779b9u) * 0x85ebca6bu;
	const uint32_t g = (h ^ (h >> 13)) * 0xc2b2ae35u;
	return __umulhi(g ^ (g >> 16), elements);
}

__global__ void scatter_probe_kernel(ulonglong2* slot, uint32_t elements, uint32_t ops, int kind,
		unsigned long long* sink)
{
	unsigned long long acc = 0;
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ops; i += gridDim.x * blockDim.x) {
		ulonglong2* s = slot + scatter_index(i, elements);
		if(kind == 0) {
			asm volatile("red.global.add.u64 [%0], %1;" :: "l"(&s->x), "l"((unsigned long long) i) : "memory");
		} else if(kind == 1) {
			asm volatile("red.global.add.u32 [%0], %1;" :: "l"(&s->x), "r"(i) : "memory");
		} else {
			acc += *reinterpret_cast<volatile unsigned long long*>(&s->x);
		}
	}
	if(kind == 2 && acc == 0x5bd1e995ull) *sink = acc;  // keeps the loads
}

} // namespace

float scatter_probe(unsigned ops, unsigned elements, int kind, unsigned ctas, int device, unsigned reps)
{
	if(elements == 0 || ops > (1u << 30) || kind < 0 || kind > 2 || reps == 0 || reps > 1000) {
		NB_THROW(NEMO_INVALID_INPUT, "scatter probe: elements > 0, ops <= 2^30, kind 0..2 and reps 1..1000 expected");
	}
	int sms = 148;
	cudaError_t err = cudaSetDevice(device);
	if(err == cudaSuccess) err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
	if(err != cudaSuccess) NB_THROW(NEMO_CUDA_ERROR, "scatter probe: %s", cudaGetErrorString(err));
	if(ctas == 0) ctas = (unsigned) sms * 8;
	cudaStream_t st = nullptr;
	ulonglong2* slot = nullptr;
	unsigned long long* sink = nullptr;
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	float ms = 0;
	err = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
	if(err == cudaSuccess) err = cudaMalloc(&slot, (size_t) elements * sizeof(ulonglong2));
	if(err == cudaSuccess) err = cudaMalloc(&sink, 8);
	if(err == cudaSuccess) err = cudaEventCreate(&e0);
	if(err == cudaSuccess) err = cudaEventCreate(&e1);
	if(err == cudaSuccess) err = cudaMemsetAsync(slot, 0, (size_t) elements * sizeof(ulonglong2), st);
	if(err == cudaSuccess) {
		scatter_probe_kernel<<<ctas, 256, 0, st>>>(slot, elements, ops, kind, sink);  // warm-up
		cudaEventRecord(e0, st);
		for(unsigned r = 0; r < reps; ++r) scatter_probe_kernel<<<ctas, 256, 0, st>>>(slot, elements, ops, kind, sink);
		cudaEventRecord(e1, st);
		err = cudaEventSynchronize(e1);
		if(err == cudaSuccess) err = cudaGetLastError();
		if(err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
	}
	if(e0) cudaEventDestroy(e0);
	if(e1) cudaEventDestroy(e1);
	if(sink) cudaFree(sink);
	if(slot) cudaFree(slot);
	if(st) cudaStreamDestroy(st);
	if(err != cudaSuccess) NB_THROW(NEMO_CUDA_ERROR, "scatter probe: %s", cudaGetErrorString(err));
	return ms * 1e3f / (float) reps;
}

} // namespace nemo_b200
