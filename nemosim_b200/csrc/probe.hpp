// probe.hpp -- the scattered-update floor measurement (probe.cu)
#pragma once

namespace nemo_b200 {

// Microseconds per launch of `ops` scattered operations into `elements`
// 16-byte slots: kind 0 = 64-bit reductions, 1 = 32-bit reductions,
// 2 = 8-byte loads; `ctas` CTAs of 256 threads (0: 8 per SM); the mean of
// `reps` launches after one warm-up launch.
float scatter_probe(unsigned ops, unsigned elements, int kind, unsigned ctas, int device, unsigned reps);

} // namespace nemo_b200
