// libm_calib.hpp -- calibration tables that let the device reproduce the
// host libm's logf/sinf at every argument nrand can produce.
#pragma once

#include <stdint.h>

#include <vector>

#include "nemo_libm.cuh"

namespace nemo_b200 {

struct CalibTables {
	std::vector<uint32_t> logFlip, sinFlip;  // one bit per reachable argument
	std::vector<uint32_t> excKey, excVal;    // arguments a one-ulp step cannot fix
	uint64_t logFlips = 0, sinFlips = 0;
	double logNear = 0.5, sinNear = 0.5;     // see LibmCalib
	std::vector<float> logVal, sinVal;       // the host libm's result at every reachable argument
};

// Computed once per process against the host libm (thread-safe).
const CalibTables& libm_calibration();

// Every reachable argument through the host build of nb_libm_logf and
// nb_libm_sinf against the host libm: the number that differ (0 when exact).
uint64_t libm_verify();

// A LibmCalib whose pointers refer to the host tables.
LibmCalib host_calib_view();

} // namespace nemo_b200
