// construction.hpp -- the forward matrix, its delay groups and the reverse
// matrix of plastic synapses built on the device from the network's synapse
// arrays (the role of ConnectivityMatrix::addSynapse / finalizeForward,
// src/nemo/ConnectivityMatrix.cpp:65-162, and construction/RCM.cpp:109-172).
// The result is byte for byte the host build's: rows keep the reference's
// order (sources, then delays, insertion order within a delay), and the
// reverse matrix holds each target's synapses in forward-matrix order.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <functional>
#include <vector>

namespace nemo_b200 {

struct DeviceConstruction {
	// inputs: the synapses in insertion order (host arrays), and the dense
	// map from global neuron id to local index (~0u: no such neuron)
	size_t S = 0;
	const unsigned* src = nullptr;
	const unsigned* tgt = nullptr;
	const unsigned* delay = nullptr;
	const float* weight = nullptr;
	const unsigned char* plastic = nullptr;
	const uint32_t* g2l = nullptr;  // [maxGid + 1]
	uint32_t maxGid = 0;
	uint32_t N = 0;        // neurons
	uint32_t D = 1;        // maximum delay (at least 1): entries per source in the delay tables
	bool deliver = true;   // deliverSpikes delivers at all (maximum delay 1..63)
	bool stdp = false;     // build the reverse matrix of plastic synapses
	bool keepQueries = true;  // keep what the synapse queries need (below)

	// outputs, allocated with `alloc` (device memory the simulation owns)
	uint2* syn = nullptr;                  // [S] {target | (delay - 1) << 26, weight}
	unsigned long long* outPtr = nullptr;  // [N + 1]
	uint16_t* dEnd16 = nullptr;            // [N][D] when every row is shorter than 65536
	uint32_t* dEnd32 = nullptr;            // [N][D] otherwise
	uint64_t* delayMask = nullptr;         // [N]
	uint32_t* rcmSrc = nullptr;            // [P] source | (delay - 1) << 26
	uint32_t* rcmFwd = nullptr;            // [P] index into syn
	// host copies of the row starts of both matrices ([N + 1] each)
	std::vector<unsigned long long> hostOutPtr, hostRcmPtr;
	uint64_t dlvGroups = 0;
	uint64_t plastic_count = 0;
	// kept on the device for the synapse queries, which build their host
	// tables from them on first use (cudaMalloc'd, freed by the caller):
	// local source, position in syn, global target, delay and plasticity
	// per synapse in insertion order
	uint32_t* keptSrc = nullptr;
	uint32_t* keptPos = nullptr;
	uint32_t* keptTgt = nullptr;
	uint8_t* keptDelay = nullptr;
	uint8_t* keptPlastic = nullptr;
};

// Builds everything on `stream` (synchronised on return).  Throws
// NEMO_INVALID_INPUT for a synapse between non-existing neurons, and a
// plain runtime error for a weight outside the fixed-point range, as the
// host build does.
void construct_on_device(DeviceConstruction& c, cudaStream_t stream, const std::function<void*(size_t)>& alloc);

// A digest of a device array (position-dependent hash of its bytes, summed)
uint64_t device_digest(const void* p, size_t bytes, cudaStream_t stream);

} // namespace nemo_b200
