// construction.hpp -- the forward matrix, its delay groups and the reverse
// matrix of plastic synapses built on the device from the network's synapse
// arrays (the role of ConnectivityMatrix::addSynapse / finalizeForward,
// src/nemo/ConnectivityMatrix.cpp:65-162, and construction/RCM.cpp:109-172).
// The result is byte for byte the host build's: rows keep the reference's
// order (sources, then delays, insertion order within a delay), and the
// reverse matrix holds each target's synapses in forward-matrix order.
//
// One call builds the part of one network: its neurons are the union local
// indices [srcBase, srcBase + nLocal) of the simulation (a batch of
// independent networks is built one network at a time), its forward entries
// go to the union forward matrix from synOff, its reverse entries to the
// union reverse matrix from plOff.  The caller allocates the union arrays.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <vector>

namespace nemo_b200 {

struct DeviceConstruction {
	// inputs: the network's synapses in insertion order (host arrays), and
	// the dense map from its global neuron ids to union local indices
	// (~0u: no such neuron)
	size_t S = 0;
	const unsigned* src = nullptr;
	const unsigned* tgt = nullptr;
	const unsigned* delay = nullptr;
	const float* weight = nullptr;
	const unsigned char* plastic = nullptr;
	const uint32_t* g2l = nullptr;  // [maxGid + 1]
	uint32_t maxGid = 0;
	uint32_t srcBase = 0;  // the network's first union local index
	uint32_t nLocal = 0;   // its neurons
	uint32_t D = 1;        // the union's maximum delay (at least 1): entries per source in the delay tables
	bool deliver = true;   // deliverSpikes delivers at all (maximum delay 1..63)
	bool stdp = false;     // build the reverse matrix of plastic synapses
	bool keepQueries = true;  // keep what the synapse queries need (below)
	uint64_t synOff = 0;   // the network's first entry in the union forward matrix
	uint64_t plOff = 0;    // its first entry in the union reverse matrix

	// the union arrays (device memory, allocated by the caller)
	uint32_t* synTgt = nullptr;            // target | (delay - 1) << 26
	uint32_t* synW = nullptr;              // weight
	unsigned long long* outPtr = nullptr;  // [N + 1] (the caller sets entry N)
	uint16_t* dEnd16 = nullptr;            // [N][D] when every row is shorter than 65536
	uint32_t* dEnd32 = nullptr;            // [N][D] otherwise
	uint64_t* delayMask = nullptr;         // [N]
	uint32_t* rcmSrc = nullptr;            // source | (delay - 1) << 26
	uint32_t* rcmFwd = nullptr;            // index into the forward matrix

	// outputs: the network's row starts in the union arrays ([nLocal] each),
	// its delay groups and plastic synapses
	std::vector<unsigned long long> hostOutPtr, hostRcmPtr;
	uint64_t dlvGroups = 0;
	uint64_t plastic_count = 0;
	// kept on the device for the synapse queries, which build their host
	// tables from them on first use (cudaMalloc'd, freed by the caller):
	// local source, position in the forward matrix, global target, delay and plasticity
	// per synapse in insertion order
	uint32_t* keptSrc = nullptr;
	uint32_t* keptPos = nullptr;
	uint32_t* keptTgt = nullptr;
	uint8_t* keptDelay = nullptr;
	uint8_t* keptPlastic = nullptr;
};

// Builds one network's part on `stream` (synchronised on return).  Throws
// NEMO_INVALID_INPUT for a synapse between non-existing neurons, and a
// plain runtime error for a weight outside the fixed-point range, as the
// host build does, for the first such synapse in insertion order.
void construct_on_device(DeviceConstruction& c, cudaStream_t stream);

// A digest of a device array (position-dependent hash of its bytes, summed)
uint64_t device_digest(const void* p, size_t bytes, cudaStream_t stream);

} // namespace nemo_b200
