// nemo_libm.cuh -- glibc-exact logf/sinf for the per-neuron Gaussian RNG.
//
// The reference draws input noise with nrand (src/nemo/RNG.cpp:25-33):
//     a = float(urand) * 1.4629180792671596810513378043098e-9f
//     b = float(urand) * 2^-32
//     r = sqrtf(-2 * logf(1 - b));   return sinf(a) * r
// calling the HOST libm's logf and sinf.  Those are not correctly rounded
// (glibc 2.39 misrounds roughly 3% of the reachable logf arguments and 1% of
// the reachable sinf arguments), so a device that must reproduce the
// reference bit for bit cannot just call a correctly rounded function.
//
// The reachable arguments form two small finite sets:
//   * 1 - b is always a multiple of 2^-24 in [0, 1]   -> 2^24 + 1 values
//   * a is a function of float(u), and float(u) for u < 2^32 takes
//     2^24 + 8 * 2^23 + 1 distinct values               -> 83,886,081 values
// For each set, this header evaluates its own double-precision log/sin with
// textbook methods (the atanh series for log after reduction to
// [sqrt(1/2), sqrt(2)), Cody-Waite reduction by pi/2 and Taylor series for
// sin/cos), using only IEEE +, -, *, / in a fixed order, so the host build
// and the device build produce identical bits.  A calibration pass on the
// host (libm_calib.cpp) compares the rounded result with the host libm over
// every reachable argument and records a one-bit "flip" per argument where
// they differ; the device then steps one ulp toward the unrounded double at
// flipped arguments.  Any argument where that single step would not give the
// libm value is kept in a short exception list.
//
// A libm result can only differ from the rounded double when the double lies
// close to the midpoint between two floats.  The calibration also records,
// per function, the largest midpoint distance (in float gaps) of any flipped
// argument; arguments farther from the midpoint than that skip the table.
// The distance is computed with the same IEEE operations on host and device
// and the bound is compared exactly (the gap is a power of two), so the skip
// changes no result: it only saves the table reads (about 88% of them for
// sinf and 43% for logf with glibc 2.39).
#pragma once

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define NB_HD __host__ __device__ __forceinline__
#else
#define NB_HD inline
#endif

namespace nemo_b200 {

#ifdef __CUDA_ARCH__
#define NB_DADD(a, b) __dadd_rn((a), (b))
#define NB_DSUB(a, b) __dsub_rn((a), (b))
#define NB_DMUL(a, b) __dmul_rn((a), (b))
#define NB_DDIV(a, b) __ddiv_rn((a), (b))
#define NB_FMUL(a, b) __fmul_rn((a), (b))
#define NB_FSUB(a, b) __fsub_rn((a), (b))
#define NB_D2F(x) __double2float_rn(x)
#define NB_U2F(x) __uint2float_rn(x)
#else
// host code is compiled with -ffp-contract=off -fno-fast-math
#define NB_DADD(a, b) ((a) + (b))
#define NB_DSUB(a, b) ((a) - (b))
#define NB_DMUL(a, b) ((a) * (b))
#define NB_DDIV(a, b) ((a) / (b))
#define NB_FMUL(a, b) ((a) * (b))
#define NB_FSUB(a, b) ((a) - (b))
#define NB_D2F(x) ((float) (x))
#define NB_U2F(x) ((float) (x))
#endif

NB_HD uint64_t nb_dbits(double x) { uint64_t u; memcpy(&u, &x, 8); return u; }
NB_HD double nb_bitsd(uint64_t u) { double x; memcpy(&x, &u, 8); return x; }
NB_HD uint32_t nb_fbits(float x) { uint32_t u; memcpy(&u, &x, 4); return u; }
NB_HD float nb_bitsf(uint32_t u) { float x; memcpy(&x, &u, 4); return x; }

// ln 2 = LN2_HI + LN2_LO with LN2_HI rounded to 32 significant bits
#define NB_LN2_HI 0x1.62e42ff000000p-1
#define NB_LN2_LO (-0x1.718432a1b0e26p-35)
#define NB_SQRT2 0x1.6a09e667f3bcdp+0
// pi/2 = P1 + P2 + P3, P1 and P2 rounded to 33 significant bits
#define NB_PIO2_1 0x1.921fb54400000p+0
#define NB_PIO2_2 0x1.0b4611a600000p-34
#define NB_PIO2_3 0x1.3198a2e037073p-69
#define NB_TWO_OVER_PI 0x1.45f306dc9c883p-1

// log(x) for finite x > 0 (normal doubles).  x = m * 2^e with m in
// [sqrt(1/2), sqrt(2)); log(m) = 2 atanh(s) = 2 (s + s^3/3 + ... + s^23/23)
// with s = (m - 1) / (m + 1), |s| <= 0.1716, truncation error < 1e-19.
NB_HD double nb_log_d(double x)
{
	uint64_t bits = nb_dbits(x);
	int e = (int) ((bits >> 52) & 0x7ff) - 1023;
	double m = nb_bitsd((bits & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
	if(m > NB_SQRT2) {
		m = NB_DMUL(m, 0.5);
		e += 1;
	}
	double s = NB_DDIV(NB_DSUB(m, 1.0), NB_DADD(m, 1.0));
	double z = NB_DMUL(s, s);
	double p = 1.0 / 23.0;
	p = NB_DADD(NB_DMUL(p, z), 1.0 / 21.0);
	p = NB_DADD(NB_DMUL(p, z), 1.0 / 19.0);
	p = NB_DADD(NB_DMUL(p, z), 1.0 / 17.0);
	p = NB_DADD(NB_DMUL(p, z), 1.0 / 15.0);
	p = NB_DADD(NB_DMUL(p, z), 1.0 / 13.0);
	p = NB_DADD(NB_DMUL(p, z), 1.0 / 11.0);
	p = NB_DADD(NB_DMUL(p, z), 1.0 / 9.0);
	p = NB_DADD(NB_DMUL(p, z), 1.0 / 7.0);
	p = NB_DADD(NB_DMUL(p, z), 1.0 / 5.0);
	p = NB_DADD(NB_DMUL(p, z), 1.0 / 3.0);
	// log(m) = 2s + 2s * z * p  (keeps the leading term exact)
	double s2 = NB_DMUL(2.0, s);
	double lm = NB_DADD(s2, NB_DMUL(NB_DMUL(s2, z), p));
	double de = (double) e;
	return NB_DADD(NB_DMUL(de, NB_LN2_HI), NB_DADD(NB_DMUL(de, NB_LN2_LO), lm));
}

// sin(a) for 0 <= a <= 8: Cody-Waite reduction by pi/2, then the Taylor
// series of sin or cos on |r| <= pi/4 (truncation error < 1e-19).
NB_HD double nb_sin_d(double a)
{
	// nearest integer multiple of pi/2; a >= 0 so truncation of a+0.5 works
	int k = (int) NB_DADD(NB_DMUL(a, NB_TWO_OVER_PI), 0.5);
	double kd = (double) k;
	double r = NB_DSUB(a, NB_DMUL(kd, NB_PIO2_1));
	r = NB_DSUB(r, NB_DMUL(kd, NB_PIO2_2));
	r = NB_DSUB(r, NB_DMUL(kd, NB_PIO2_3));
	double z = NB_DMUL(r, r);
	double y;
	if(k & 1) {
		// cos r = 1 - z/2! + z^2/4! - ... + z^9/18!
		double p = -1.0 / 6402373705728000.0;          // -1/18!
		p = NB_DADD(NB_DMUL(p, z), 1.0 / 20922789888000.0); // 1/16!
		p = NB_DADD(NB_DMUL(p, z), -1.0 / 87178291200.0);   // -1/14!
		p = NB_DADD(NB_DMUL(p, z), 1.0 / 479001600.0);      // 1/12!
		p = NB_DADD(NB_DMUL(p, z), -1.0 / 3628800.0);       // -1/10!
		p = NB_DADD(NB_DMUL(p, z), 1.0 / 40320.0);          // 1/8!
		p = NB_DADD(NB_DMUL(p, z), -1.0 / 720.0);           // -1/6!
		p = NB_DADD(NB_DMUL(p, z), 1.0 / 24.0);             // 1/4!
		// 1 - z/2 + z^2 * p
		double hz = NB_DMUL(0.5, z);
		double w = NB_DSUB(1.0, hz);
		y = NB_DADD(w, NB_DADD(NB_DSUB(NB_DSUB(1.0, w), hz), NB_DMUL(NB_DMUL(z, z), p)));
	} else {
		// sin r = r - r^3/3! + ... + r^19/19!
		double p = 1.0 / 121645100408832000.0;             // 1/19!
		p = NB_DADD(NB_DMUL(p, z), -1.0 / 355687428096000.0); // -1/17!
		p = NB_DADD(NB_DMUL(p, z), 1.0 / 1307674368000.0);    // 1/15!
		p = NB_DADD(NB_DMUL(p, z), -1.0 / 6227020800.0);      // -1/13!
		p = NB_DADD(NB_DMUL(p, z), 1.0 / 39916800.0);         // 1/11!
		p = NB_DADD(NB_DMUL(p, z), -1.0 / 362880.0);          // -1/9!
		p = NB_DADD(NB_DMUL(p, z), 1.0 / 5040.0);             // 1/7!
		p = NB_DADD(NB_DMUL(p, z), -1.0 / 120.0);             // -1/5!
		p = NB_DADD(NB_DMUL(p, z), 1.0 / 6.0);                // 1/3!, sign below
		// r - r^3 * (1/6 - z/120 + ...)
		y = NB_DSUB(r, NB_DMUL(NB_DMUL(r, z), p));
	}
	return (k & 2) ? -y : y;
}

// one ulp from f toward d
NB_HD float nb_step_toward(float f, double d)
{
	uint32_t u = nb_fbits(f);
	bool up = d > (double) f;
	if((u & 0x7fffffffu) == 0) return nb_bitsf(up ? 1u : 0x80000001u);
	bool pos = (u >> 31) == 0;
	return nb_bitsf(pos == up ? u + 1u : u - 1u);
}

// the constants of nrand (src/nemo/RNG.cpp:27-28) as float literals
#define NB_NRAND_A 1.4629180792671596810513378043098e-9f
#define NB_NRAND_B 0.00000000023283064365386962890625f

// index sets of the two calibrated arguments
#define NB_LOG_COUNT ((1u << 24) + 1u)
#define NB_SIN_COUNT ((1u << 24) + (8u << 23) + 1u)

// float(u) -> dense index of the distinct value
NB_HD uint32_t nb_sin_index(float fu)
{
	if(fu < 16777216.0f) return (uint32_t) fu;
	uint32_t fb = nb_fbits(fu);
	uint32_t e = ((fb >> 23) & 0xffu) - 127u - 24u;
	return (1u << 24) + (e << 23) + (fb & 0x7fffffu);
}

// inverse of nb_sin_index
NB_HD float nb_sin_value(uint32_t idx)
{
	if(idx < (1u << 24)) return (float) idx;
	uint32_t r = idx - (1u << 24);
	uint32_t e = r >> 23;
	return nb_bitsf(((e + 127u + 24u) << 23) | (r & 0x7fffffu));
}

struct LibmCalib {
	const uint32_t* logFlip;   // NB_LOG_COUNT bits
	const uint32_t* sinFlip;   // NB_SIN_COUNT bits
	const uint32_t* excKey;    // sorted: (table << 31) | index
	const uint32_t* excVal;    // float bits of the libm result
	uint32_t nexc;
	// largest nb_mid_gaps of any flipped argument (0.5 reads every argument)
	double logNear, sinNear;
	// the host libm's logf and sinf at every reachable argument, by index
	// (NB_LOG_COUNT and NB_SIN_COUNT floats)
	const float* logVal;
	const float* sinVal;
};

// f = float(d) and its neighbour toward d bound the interval holding d;
// returns |midpoint - d| and stores the interval's width (a power of two).
NB_HD double nb_mid_dist(float f, double d, double* gap)
{
	double a = (double) f, b = (double) nb_step_toward(f, d);
	*gap = a < b ? NB_DSUB(b, a) : NB_DSUB(a, b);
	double m = NB_DMUL(NB_DADD(a, b), 0.5);
	return m < d ? NB_DSUB(d, m) : NB_DSUB(m, d);
}

// the distance of d from the midpoint in gaps (exact: the gap is 2^k)
NB_HD double nb_mid_gaps(float f, double d)
{
	double gap;
	double r = nb_mid_dist(f, d, &gap);
	return NB_DDIV(r, gap);
}

// whether the argument may be flipped: within `near` gaps of the midpoint
NB_HD bool nb_near_mid(float f, double d, double near)
{
	double gap;
	double r = nb_mid_dist(f, d, &gap);
	return r <= NB_DMUL(near, gap);
}

NB_HD bool nb_bit(const uint32_t* bits, uint32_t i) { return (bits[i >> 5] >> (i & 31)) & 1u; }

NB_HD bool nb_exception(const LibmCalib& c, uint32_t key, float* out)
{
	uint32_t lo = 0, hi = c.nexc;
	while(lo < hi) {
		uint32_t mid = (lo + hi) >> 1;
		uint32_t k = c.excKey[mid];
		if(k == key) { *out = nb_bitsf(c.excVal[mid]); return true; }
		if(k < key) lo = mid + 1; else hi = mid;
	}
	return false;
}

// the flip-table index of logf's argument x = 1 - b
NB_HD uint32_t nb_log_index(float x) { return (uint32_t) NB_FMUL(x, 16777216.0f); }

// logf(x) for x = 1 - b as produced by nrand (a multiple of 2^-24 in [0, 1]);
// word: the flip-table word holding the argument's bit (fetched by the
// caller, so that the load overlaps the evaluation)
NB_HD float nb_libm_logf_w(const LibmCalib& c, float x, uint32_t word)
{
	if(x == 0.0f) return nb_bitsf(0xff800000u); // -inf
	uint32_t idx = nb_log_index(x);
	double d = nb_log_d((double) x);
	float f = NB_D2F(d);
	if(nb_near_mid(f, d, c.logNear) && ((word >> (idx & 31)) & 1u)) {
		float e;
		if(c.nexc && nb_exception(c, idx, &e)) return e;
		f = nb_step_toward(f, d);
	}
	return f;
}

// as nb_libm_logf_w, reading the flip table only where the bit may be set
NB_HD float nb_libm_logf(const LibmCalib& c, float x)
{
	if(x == 0.0f) return nb_bitsf(0xff800000u); // -inf
	uint32_t idx = nb_log_index(x);
	double d = nb_log_d((double) x);
	float f = NB_D2F(d);
	if(nb_near_mid(f, d, c.logNear) && nb_bit(c.logFlip, idx)) {
		float e;
		if(c.nexc && nb_exception(c, idx, &e)) return e;
		f = nb_step_toward(f, d);
	}
	return f;
}

// sinf(a) for a = float(u) * NB_NRAND_A; fu = float(u); word as for logf
NB_HD float nb_libm_sinf_w(const LibmCalib& c, float fu, float a, uint32_t word)
{
	uint32_t idx = nb_sin_index(fu);
	double d = nb_sin_d((double) a);
	float f = NB_D2F(d);
	if(nb_near_mid(f, d, c.sinNear) && ((word >> (idx & 31)) & 1u)) {
		float e;
		if(c.nexc && nb_exception(c, (1u << 31) | idx, &e)) return e;
		f = nb_step_toward(f, d);
	}
	return f;
}

// as nb_libm_sinf_w, reading the flip table only where the bit may be set
NB_HD float nb_libm_sinf(const LibmCalib& c, float fu, float a)
{
	uint32_t idx = nb_sin_index(fu);
	double d = nb_sin_d((double) a);
	float f = NB_D2F(d);
	if(nb_near_mid(f, d, c.sinNear) && nb_bit(c.sinFlip, idx)) {
		float e;
		if(c.nexc && nb_exception(c, (1u << 31) | idx, &e)) return e;
		f = nb_step_toward(f, d);
	}
	return f;
}

// xorshift128 of src/nemo/RNG.cpp:9-18
NB_HD uint32_t nb_urand(uint32_t& s0, uint32_t& s1, uint32_t& s2, uint32_t& s3)
{
	uint32_t t = s0 ^ (s0 << 11);
	s0 = s1;
	s1 = s2;
	s2 = s3;
	s3 = (s3 ^ (s3 >> 19)) ^ (t ^ (t >> 8));
	return s3;
}

// nrand of src/nemo/RNG.cpp:25-33 with the host libm reproduced.  EARLY
// fetches both flip-table words before the evaluations (shorter latency,
// more registers); the result is the same.
template<bool EARLY = false>
NB_HD float nb_nrand(const LibmCalib& c, uint32_t& s0, uint32_t& s1, uint32_t& s2, uint32_t& s3)
{
	float fu1 = NB_U2F(nb_urand(s0, s1, s2, s3));
	float a = NB_FMUL(fu1, NB_NRAND_A);
	float fu2 = NB_U2F(nb_urand(s0, s1, s2, s3));
	float b = NB_FMUL(fu2, NB_NRAND_B);
	float x = NB_FSUB(1.0f, b);
	float l, s;
	if(EARLY) {
		// both flip-table words depend only on the draws
		const uint32_t lw = c.logFlip[nb_log_index(x) >> 5];
		const uint32_t sw = c.sinFlip[nb_sin_index(fu1) >> 5];
		l = nb_libm_logf_w(c, x, lw);
		s = nb_libm_sinf_w(c, fu1, a, sw);
	} else {
		l = nb_libm_logf(c, x);
		s = nb_libm_sinf(c, fu1, a);
	}
#ifdef __CUDA_ARCH__
	float r = __fsqrt_rn(__fmul_rn(-2.0f, l));
	return __fmul_rn(s, r);
#else
	float r = __builtin_sqrtf(-2.0f * l);
	return s * r;
#endif
}

// nrand of src/nemo/RNG.cpp:25-33 reading the host libm's logf and sinf
// results from the calibration tables (both arguments come from finite
// sets, indexed as for the flip tables): two loads instead of the
// evaluations, the same bits as nb_nrand.
NB_HD float nb_nrand_table(const LibmCalib& c, uint32_t& s0, uint32_t& s1, uint32_t& s2, uint32_t& s3)
{
	float fu1 = NB_U2F(nb_urand(s0, s1, s2, s3));
	float fu2 = NB_U2F(nb_urand(s0, s1, s2, s3));
	float b = NB_FMUL(fu2, NB_NRAND_B);
	float x = NB_FSUB(1.0f, b);
	const float l = c.logVal[nb_log_index(x)];
	const float s = c.sinVal[nb_sin_index(fu1)];
#ifdef __CUDA_ARCH__
	float r = __fsqrt_rn(__fmul_rn(-2.0f, l));
	return __fmul_rn(s, r);
#else
	float r = __builtin_sqrtf(-2.0f * l);
	return s * r;
#endif
}

} // namespace nemo_b200
