// bench_loop.cpp -- the end-to-end benchmark loop as a C program runs it,
// the role of the reference's benchmark() (src/examples/common.cpp:13-122):
// nemo_step once per millisecond with a firing stimulus from host memory and
// the fired ids returned in host memory, nemo_apply_stdp every `period`
// steps, through the public C API only, timed on the host clock.
#include <stdint.h>

#include <chrono>

#include "../../include/nemo_b200.h"

extern "C" nemo_status_t nemo_b200_bench_step_loop(nemo_simulation_t sim, const unsigned* fstim,
		size_t fstim_per_step, unsigned steps, unsigned period, float reward, uint64_t* fired_total,
		double* seconds)
{
	if(!sim || (fstim_per_step && !fstim) || !fired_total || !seconds) return NEMO_INVALID_INPUT;
	uint64_t total = 0;
	const auto t0 = std::chrono::steady_clock::now();
	for(unsigned k = 0; k < steps; ++k) {
		unsigned* fired = nullptr;
		size_t nfired = 0;
		nemo_status_t r = nemo_step(sim, const_cast<unsigned*>(fstim) + (size_t) k * fstim_per_step, fstim_per_step,
				nullptr, nullptr, 0, &fired, &nfired);
		if(r != NEMO_OK) return r;
		total += nfired;
		if(period && (k + 1) % period == 0) {
			r = nemo_apply_stdp(sim, reward);
			if(r != NEMO_OK) return r;
		}
	}
	*seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
	*fired_total = total;
	return NEMO_OK;
}
