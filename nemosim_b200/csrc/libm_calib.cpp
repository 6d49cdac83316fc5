// libm_calib.cpp -- host calibration of the device's logf/sinf against the
// host C library (see nemo_libm.cuh for the method).
//
// The reference CPU backend takes its input noise from the host libm
// (src/nemo/RNG.cpp:30-32), so the calibration is made against the libm of
// the process that runs the simulation: every reachable argument is
// evaluated with both the libm and the device's own double-precision
// routine, once per process, on all host threads (about a second).
#include "libm_calib.hpp"

#include <math.h>

#include <algorithm>
#include <mutex>
#include <thread>
#include <vector>

namespace nemo_b200 {

namespace {

struct Exc { uint32_t key, val; };

void calibrate_range(bool isLog, uint32_t wbegin, uint32_t wend, uint32_t count,
		std::vector<uint32_t>& bits, uint64_t& flips, double& near, std::vector<Exc>& exc, float* vals)
{
	for(uint32_t w = wbegin; w < wend; ++w) {
		uint32_t word = 0;
		for(uint32_t b = 0; b < 32; ++b) {
			uint32_t idx = w * 32 + b;
			if(idx >= count) break;
			float libm, mine;
			double d;
			if(isLog) {
				float x = (float) idx * 0x1p-24f;
				libm = logf(x);
				vals[idx] = libm;
				if(x == 0.0f) continue; // special-cased by the emulation
				d = nb_log_d((double) x);
			} else {
				float fu = nb_sin_value(idx);
				float a = fu * NB_NRAND_A;
				libm = sinf(a);
				vals[idx] = libm;
				d = nb_sin_d((double) a);
			}
			mine = (float) d;
			if(nb_fbits(libm) != nb_fbits(mine)) {
				word |= 1u << b;
				flips++;
				near = std::max(near, nb_mid_gaps(mine, d));
				float stepped = nb_step_toward(mine, d);
				if(nb_fbits(stepped) != nb_fbits(libm)) {
					exc.push_back(Exc{ (isLog ? 0u : (1u << 31)) | idx, nb_fbits(libm) });
				}
			}
		}
		bits[w] = word;
	}
}

void calibrate(bool isLog, uint32_t count, std::vector<uint32_t>& bits, uint64_t& flips,
		double& near, std::vector<Exc>& exc, std::vector<float>& vals)
{
	uint32_t nwords = (count + 31) / 32;
	bits.assign(nwords, 0);
	vals.assign(count, 0.0f);
	unsigned nt = std::max(1u, std::thread::hardware_concurrency());
	std::vector<std::thread> threads;
	std::vector<uint64_t> tflips(nt, 0);
	std::vector<double> tnear(nt, 0.0);
	std::vector<std::vector<Exc>> texc(nt);
	uint32_t chunk = (nwords + nt - 1) / nt;
	for(unsigned t = 0; t < nt; ++t) {
		uint32_t b = std::min(nwords, t * chunk), e = std::min(nwords, (t + 1) * chunk);
		threads.emplace_back([&, t, b, e] { calibrate_range(isLog, b, e, count, bits, tflips[t], tnear[t], texc[t], vals.data()); });
	}
	for(auto& th : threads) th.join();
	flips = 0;
	near = 0.0;
	for(unsigned t = 0; t < nt; ++t) {
		flips += tflips[t];
		near = std::max(near, tnear[t]);
		exc.insert(exc.end(), texc[t].begin(), texc[t].end());
	}
}

} // namespace

const CalibTables& libm_calibration()
{
	static CalibTables tables;
	static std::once_flag once;
	std::call_once(once, [] {
		std::vector<Exc> exc;
		calibrate(true, NB_LOG_COUNT, tables.logFlip, tables.logFlips, tables.logNear, exc, tables.logVal);
		calibrate(false, NB_SIN_COUNT, tables.sinFlip, tables.sinFlips, tables.sinNear, exc, tables.sinVal);
		std::sort(exc.begin(), exc.end(), [](const Exc& a, const Exc& b) { return a.key < b.key; });
		for(const Exc& e : exc) {
			tables.excKey.push_back(e.key);
			tables.excVal.push_back(e.val);
		}
	});
	return tables;
}

uint64_t libm_verify()
{
	const LibmCalib c = host_calib_view();
	unsigned nt = std::max(1u, std::thread::hardware_concurrency());
	std::vector<uint64_t> bad(nt, 0);
	std::vector<std::thread> threads;
	const uint64_t total = (uint64_t) NB_LOG_COUNT + NB_SIN_COUNT;
	for(unsigned t = 0; t < nt; ++t) {
		threads.emplace_back([&, t] {
			for(uint64_t i = t; i < total; i += nt) {
				// both forms: the flip word read lazily and fetched up front;
				// and the result table at the index nb_nrand_table uses
				float libm, mine, early, table;
				if(i < NB_LOG_COUNT) {
					float x = (float) i * 0x1p-24f;
					libm = logf(x);
					mine = nb_libm_logf(c, x);
					early = nb_libm_logf_w(c, x, c.logFlip[nb_log_index(x) >> 5]);
					table = c.logVal[nb_log_index(x)];
				} else {
					float fu = nb_sin_value((uint32_t) (i - NB_LOG_COUNT));
					float a = fu * NB_NRAND_A;
					libm = sinf(a);
					mine = nb_libm_sinf(c, fu, a);
					early = nb_libm_sinf_w(c, fu, a, c.sinFlip[nb_sin_index(fu) >> 5]);
					table = c.sinVal[nb_sin_index(fu)];
				}
				bad[t] += nb_fbits(libm) != nb_fbits(mine) || nb_fbits(libm) != nb_fbits(early)
						|| nb_fbits(libm) != nb_fbits(table);
			}
		});
	}
	for(auto& th : threads) th.join();
	uint64_t n = 0;
	for(uint64_t b : bad) n += b;
	return n;
}

LibmCalib host_calib_view()
{
	const CalibTables& t = libm_calibration();
	LibmCalib c;
	c.logFlip = t.logFlip.data();
	c.sinFlip = t.sinFlip.data();
	c.excKey = t.excKey.data();
	c.excVal = t.excVal.data();
	c.nexc = (uint32_t) t.excKey.size();
	c.logNear = t.logNear;
	c.sinNear = t.sinNear;
	c.logVal = t.logVal.data();
	c.sinVal = t.sinVal.data();
	return c;
}

} // namespace nemo_b200
