// examples.cpp -- the reference's example network generator
// random::construct (src/examples/random.cpp:29-88), in native code so the
// 100M-synapse benchmark network builds in seconds.
//
// The Boost distributions it uses are restated over a 32-bit mt19937 with the
// default seed 5489: uniform_real<double>(0, 1) is x / 2^32, and
// uniform_int<>(lo, hi) divides by a bucket size and rejects out-of-range
// results (Boost >= 1.47), taking no draw when lo == hi.  The arguments of
// Network::addSynapse (random.cpp:78 and :83) are evaluated right to left, as
// GCC does on x86-64.
#include <stdint.h>

#include <vector>

#include "../../include/nemo_b200.h"
#include "handles.hpp"
#include "network.hpp"


namespace {

struct Mt19937 {
	uint32_t mt[624];
	int idx;
	explicit Mt19937(uint32_t seed) {
		mt[0] = seed;
		for(int i = 1; i < 624; ++i) mt[i] = 1812433253u * (mt[i - 1] ^ (mt[i - 1] >> 30)) + (uint32_t) i;
		idx = 624;
	}
	uint32_t operator()() {
		if(idx >= 624) twist();
		uint32_t y = mt[idx++];
		y ^= (y >> 11);
		y ^= (y << 7) & 0x9d2c5680u;
		y ^= (y << 15) & 0xefc60000u;
		y ^= (y >> 18);
		return y;
	}
	void twist() {
		auto mix = [](uint32_t a, uint32_t b, uint32_t c) {
			uint32_t y = (a & 0x80000000u) | (b & 0x7fffffffu);
			return c ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
		};
		int k = 0;
		for(; k < 624 - 397; ++k) mt[k] = mix(mt[k], mt[k + 1], mt[k + 397]);
		for(; k < 623; ++k) mt[k] = mix(mt[k], mt[k + 1], mt[k + 397 - 624]);
		mt[623] = mix(mt[623], mt[0], mt[396]);
		idx = 0;
	}
};

double uniform01(Mt19937& g) { return (double) g() / 4294967296.0; }

unsigned uniformInt(Mt19937& g, unsigned lo, unsigned hi)
{
	uint32_t range = hi - lo;
	if(range == 0) return lo;
	if(range == 0xffffffffu) return lo + g();
	uint32_t bucket = 0xffffffffu / (range + 1u);
	if(0xffffffffu % (range + 1u) == range) bucket++;
	for(;;) {
		uint32_t r = g() / bucket;
		if(r <= range) return lo + r;
	}
}

} // namespace

extern "C" nemo_status_t nemo_b200_example_random(nemo_network_t* out, unsigned ncount, unsigned scount,
		unsigned dmax, int stdp)
{
	return nemo_b200_example_random_ex(out, ncount, scount, dmax, stdp, 5489u, 5.0f, 2.0f);
}

extern "C" nemo_status_t nemo_b200_example_random_ex(nemo_network_t* out, unsigned ncount, unsigned scount,
		unsigned dmax, int stdp, unsigned seed, float sigmaExc, float sigmaInh)
{
	if(!out) return NEMO_INVALID_INPUT;
	nemo_network_t net = nemo_new_network();
	if(!net) return NEMO_ALLOCATION_ERROR;
	unsigned iz = 0;
	nemo_status_t r = nemo_add_neuron_type(net, "Izhikevich", &iz);
	Mt19937 g(seed);
	std::vector<unsigned> src(scount), tgt(scount), dly(scount);
	std::vector<float> w(scount);
	std::vector<unsigned char> pl(scount);
	const size_t total = (size_t) ncount * scount;
	net->net.src.reserve(total);
	net->net.tgt.reserve(total);
	net->net.delay.reserve(total);
	net->net.weight.reserve(total);
	net->net.plastic.reserve(total);
	net->net.sid.reserve(total);
	for(unsigned nidx = 0; nidx < ncount && r == NEMO_OK; ++nidx) {
		const float v = -65.0f;
		const bool exc = nidx < (ncount * 4) / 5;
		float args[7];
		if(exc) {
			// addExcitatoryNeuron, random.cpp:29-42
			float a = 0.02f, b = 0.2f;
			float r1 = (float) uniform01(g);
			float r2 = (float) uniform01(g);
			float c = v + 15.0f * r1 * r1;
			float d = 8.0f - 6.0f * r2 * r2;
			float u = b * v;
			float x[7] = { a, b, c, d, sigmaExc, u, v };
			for(int i = 0; i < 7; ++i) args[i] = x[i];
		} else {
			// addInhibitoryNeuron, random.cpp:46-59
			float r1 = (float) uniform01(g);
			float a = 0.02f + 0.08f * r1;
			float r2 = (float) uniform01(g);
			float b = 0.25f - 0.05f * r2;
			float u = b * v;
			float x[7] = { a, b, v, 2.0f, sigmaInh, u, v };
			for(int i = 0; i < 7; ++i) args[i] = x[i];
		}
		r = nemo_b200_add_neurons(net, iz, 1, &nidx, 7, args);
		for(unsigned s = 0; s < scount; ++s) {
			src[s] = nidx;
			if(exc) {
				w[s] = 0.5f * (float) uniform01(g);
				dly[s] = uniformInt(g, 1, dmax);
				tgt[s] = uniformInt(g, 0, ncount - 1);
				pl[s] = (unsigned char) (stdp != 0);
			} else {
				w[s] = (float) (-uniform01(g));
				tgt[s] = uniformInt(g, 0, ncount - 1);
				dly[s] = 1;
				pl[s] = 0;
			}
		}
		if(r == NEMO_OK && scount) {
			r = nemo_b200_add_synapses(net, scount, src.data(), tgt.data(), dly.data(), w.data(), pl.data(), nullptr);
		}
	}
	if(r != NEMO_OK) {
		nemo_delete_network(net);
		return r;
	}
	*out = net;
	return NEMO_OK;
}
