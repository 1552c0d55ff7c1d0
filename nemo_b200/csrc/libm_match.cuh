#ifndef NEMO_B200_LIBM_MATCH_CUH
#define NEMO_B200_LIBM_MATCH_CUH

/* Bit-exact reproduction of the host glibc sinf/logf results that the
 * reference's thalamic-noise generator consumes (src/nemo/RNG.cpp:26-34).
 *
 * glibc's sinf and logf are not correctly rounded (on this image they differ
 * from the correctly rounded value for about 1.2% / 3.5% of the inputs the RNG
 * can produce). The device therefore computes a *candidate* with the code in
 * this header, which is compiled identically for host and device (double
 * arithmetic through explicit round-to-nearest operations, no contraction, no
 * library calls), and applies a 2-bit correction taken from a table that the
 * host builds once by comparing the candidate with glibc for every reachable
 * input (libm_tables.cpp). Because the candidate is bit-identical on both
 * sides, the corrected device result equals glibc's for every input.
 *
 * Reachable inputs. nrand draws two 32-bit words u1, u2 and forms
 * a = float(u1) * 1.4629180792671596810513378043098e-9f and
 * 1 - float(u2) * 2^-32. Both depend only on float(u), which takes
 * 2^24 + 8*2^23 + 1 = 83886081 distinct values; they are numbered by
 * libm_index() and the tables hold one 2-bit code per index:
 *   0: glibc == candidate, 1: glibc bits == candidate bits + 1,
 *   2: glibc bits == candidate bits - 1.
 *
 * Methods (named, restated from their published descriptions):
 * sin: Cody-Waite reduction by pi/2 with the two-part pi/2 of fdlibm
 *      (e_rem_pio2.c: pio2_1, pio2_1t), then the Taylor series of sin/cos on
 *      |r| <= pi/4 to degree 23/22.
 * log: y = m * 2^e with m in [sqrt(2)/2, sqrt(2)), log m = 2 atanh(s),
 *      s = (m-1)/(m+1), atanh series to degree 25, ln 2 split as in fdlibm
 *      e_log.c (ln2_hi, ln2_lo). */

#include <cstdint>

#ifdef __CUDACC__
#define LIBM_HD __host__ __device__ __forceinline__
#else
#define LIBM_HD inline
#endif

#ifdef __CUDA_ARCH__
#define D_ADD(a, b) __dadd_rn((a), (b))
#define D_SUB(a, b) __dsub_rn((a), (b))
#define D_MUL(a, b) __dmul_rn((a), (b))
#define D_DIV(a, b) __ddiv_rn((a), (b))
#define D_FMA(a, b, c) __fma_rn((a), (b), (c))
#else
/* Host builds of this header must use -ffp-contract=off. */
#define D_ADD(a, b) ((a) + (b))
#define D_SUB(a, b) ((a) - (b))
#define D_MUL(a, b) ((a) * (b))
#define D_DIV(a, b) ((a) / (b))
#define D_FMA(a, b, c) __builtin_fma((a), (b), (c))
#endif

/* On the device, host-only names are not available; keep the header free of
 * <cmath>/<cstring> so that both compilers see the same operations. */
namespace nemo_b200 {
namespace libm {

const uint32_t TABLE_ENTRIES = 83886081u;     /* distinct float(u), u < 2^32 */
const uint32_t TABLE_WORDS = (TABLE_ENTRIES + 15u) / 16u;

LIBM_HD uint32_t f2u(float f) {
#ifdef __CUDA_ARCH__
	return __float_as_uint(f);
#else
	union { float f; uint32_t u; } x; x.f = f; return x.u;
#endif
}

LIBM_HD float u2f(uint32_t u) {
#ifdef __CUDA_ARCH__
	return __uint_as_float(u);
#else
	union { float f; uint32_t u; } x; x.u = u; return x.f;
#endif
}

LIBM_HD uint64_t d2u(double d) {
#ifdef __CUDA_ARCH__
	return (uint64_t) __double_as_longlong(d);
#else
	union { double d; uint64_t u; } x; x.d = d; return x.u;
#endif
}

LIBM_HD double u2d(uint64_t u) {
#ifdef __CUDA_ARCH__
	return __longlong_as_double((long long) u);
#else
	union { double d; uint64_t u; } x; x.u = u; return x.d;
#endif
}

/* Index of fu = float(u): integers below 2^24 are exact; above, floats are
 * consecutive in their bit patterns from 2^24 (0x4B800000) to 2^32. */
LIBM_HD uint32_t libm_index(float fu) {
	return fu < 16777216.0f ? uint32_t(fu) : f2u(fu) - 0x4B800000u + 16777216u;
}

LIBM_HD float libm_value(uint32_t idx) {
	return idx < 16777216u ? float(idx) : u2f(idx - 16777216u + 0x4B800000u);
}

/* sin(x) for 0 <= x < 8 (a <= 2^32 * 1.46e-9 < 6.3). Returns double. */
LIBM_HD double sin_candidate_d(double x) {
	const double invpio2 = 0.6366197723675814;
	const double pio2_1 = 1.5707963267341256;        /* 0x3FF921FB54400000 */
	const double pio2_1t = 6.07710050650619224932e-11;
	double kf = D_ADD(D_MUL(x, invpio2), 0.5);
	int k = int(kf);                                  /* x >= 0: floor */
	double kd = double(k);
	double r = D_SUB(D_SUB(x, D_MUL(kd, pio2_1)), D_MUL(kd, pio2_1t));
	double r2 = D_MUL(r, r);
	/* sin r = r + r^3 * (s1 + r^2 (s2 + ...)) */
	double ps = -3.868170170630684e-23;
	ps = D_ADD(D_MUL(ps, r2), 1.9572941063391263e-20);
	ps = D_ADD(D_MUL(ps, r2), -8.22063524662433e-18);
	ps = D_ADD(D_MUL(ps, r2), 2.8114572543455206e-15);
	ps = D_ADD(D_MUL(ps, r2), -7.647163731819816e-13);
	ps = D_ADD(D_MUL(ps, r2), 1.6059043836821613e-10);
	ps = D_ADD(D_MUL(ps, r2), -2.505210838544172e-08);
	ps = D_ADD(D_MUL(ps, r2), 2.7557319223985893e-06);
	ps = D_ADD(D_MUL(ps, r2), -0.0001984126984126984);
	ps = D_ADD(D_MUL(ps, r2), 0.008333333333333333);
	ps = D_ADD(D_MUL(ps, r2), -0.16666666666666666);
	double s = D_ADD(r, D_MUL(D_MUL(r, r2), ps));
	/* cos r = 1 + r^2 * (c1 + r^2 (c2 + ...)) */
	double pc = -8.896791392450574e-22;
	pc = D_ADD(D_MUL(pc, r2), 4.110317623312165e-19);
	pc = D_ADD(D_MUL(pc, r2), -1.5619206968586225e-16);
	pc = D_ADD(D_MUL(pc, r2), 4.779477332387385e-14);
	pc = D_ADD(D_MUL(pc, r2), -1.1470745597729725e-11);
	pc = D_ADD(D_MUL(pc, r2), 2.08767569878681e-09);
	pc = D_ADD(D_MUL(pc, r2), -2.755731922398589e-07);
	pc = D_ADD(D_MUL(pc, r2), 2.48015873015873e-05);
	pc = D_ADD(D_MUL(pc, r2), -0.001388888888888889);
	pc = D_ADD(D_MUL(pc, r2), 0.041666666666666664);
	pc = D_ADD(D_MUL(pc, r2), -0.5);
	double c = D_ADD(1.0, D_MUL(r2, pc));
	switch(k & 3) {
		case 0: return s;
		case 1: return c;
		case 2: return -s;
		default: return -c;
	}
}

/* log(y) for a positive normal float y; y == 0 gives -infinity. */
LIBM_HD double log_candidate_d(float y) {
	if(y == 0.0f) {
		return -u2d(0x7FF0000000000000ull);
	}
	const double ln2_hi = 6.93147180369123816490e-01;  /* 0x3FE62E42FEE00000 */
	const double ln2_lo = 1.90821492927058770002e-10;
	uint32_t bits = f2u(y);
	int e = int((bits >> 23) & 0xff) - 127;
	/* m in [1, 2) as a double with the float's mantissa */
	double m = u2d((uint64_t(1023) << 52) | (uint64_t(bits & 0x7fffff) << 29));
	if(m > 1.4142135623730951) {
		m = D_MUL(m, 0.5);
		e += 1;
	}
	double s = D_DIV(D_SUB(m, 1.0), D_ADD(m, 1.0));
	double s2 = D_MUL(s, s);
	double p = 0.04;
	p = D_ADD(D_MUL(p, s2), 0.043478260869565216);
	p = D_ADD(D_MUL(p, s2), 0.047619047619047616);
	p = D_ADD(D_MUL(p, s2), 0.05263157894736842);
	p = D_ADD(D_MUL(p, s2), 0.058823529411764705);
	p = D_ADD(D_MUL(p, s2), 0.06666666666666667);
	p = D_ADD(D_MUL(p, s2), 0.07692307692307693);
	p = D_ADD(D_MUL(p, s2), 0.09090909090909091);
	p = D_ADD(D_MUL(p, s2), 0.1111111111111111);
	p = D_ADD(D_MUL(p, s2), 0.14285714285714285);
	p = D_ADD(D_MUL(p, s2), 0.2);
	p = D_ADD(D_MUL(p, s2), 0.3333333333333333);
	/* log m = 2s + 2 s^3 p */
	double logm = D_ADD(D_MUL(2.0, s), D_MUL(D_MUL(2.0, D_MUL(s, s2)), p));
	double ed = double(e);
	return D_ADD(D_MUL(ed, ln2_hi), D_ADD(D_MUL(ed, ln2_lo), logm));
}

/* The float arguments of nrand for a given float(u) (src/nemo/RNG.cpp:29-31) */
LIBM_HD float sin_argument(float fu) {
#ifdef __CUDA_ARCH__
	return __fmul_rn(fu, 1.4629180792671596810513378043098e-9f);
#else
	return fu * 1.4629180792671596810513378043098e-9f;
#endif
}

LIBM_HD float log_argument(float fu) {
#ifdef __CUDA_ARCH__
	return __fsub_rn(1.0f, __fmul_rn(fu, 0.00000000023283064365386962890625f));
#else
	return 1.0f - fu * 0.00000000023283064365386962890625f;
#endif
}

LIBM_HD float sin_candidate(float a) { return float(sin_candidate_d(double(a))); }
LIBM_HD float log_candidate(float y) { return float(log_candidate_d(y)); }

/* exp(x) of a float x, evaluated in double with explicitly rounded
 * operations, fused multiply-adds included (identical on host and device):
 * k = round(x / ln2) by adding 1.5 * 2^52 (the fused x * (1/ln2) + 1.5 * 2^52
 * rounds once, to a double whose last place is 1), r = x - k ln2 with the
 * Cody-Waite split of ln2 (|r| <= 0.3466), e^r by its Taylor series to degree
 * 11 (truncation below 7e-15 relative) in Estrin's scheme, scaled by 2^k.
 * Beyond the float range: 0 below -104, infinity above 89; NaN stays NaN.
 * The result is branch-free, so that several evaluations interleave. */
LIBM_HD double exp_candidate_d(float xf) {
	const double ln2_hi = 6.93147180369123816490e-01;  /* 0x3FE62E42FEE00000 */
	const double ln2_lo = 1.90821492927058770002e-10;
	const double shift = 6755399441055744.0;            /* 1.5 * 2^52 */
	const double x = double(xf);
	const double t = D_FMA(x, 1.4426950408889634, shift);
	const double kd = D_SUB(t, shift);
	const uint32_t k = uint32_t(d2u(t));                /* k mod 2^32 */
	const double r = D_FMA(-kd, ln2_lo, D_FMA(-kd, ln2_hi, x));
	/* 1/n! for n = 0..11, rounded to double */
	const double r2 = D_MUL(r, r);
	const double a0 = D_FMA(r, 1.0, 1.0);
	const double a1 = D_FMA(r, 0.16666666666666666, 0.5);
	const double a2 = D_FMA(r, 0.008333333333333333, 0.041666666666666664);
	const double a3 = D_FMA(r, 0.0001984126984126984, 0.001388888888888889);
	const double a4 = D_FMA(r, 2.7557319223985893e-06, 2.48015873015873e-05);
	const double a5 = D_FMA(r, 2.505210838544172e-08, 2.755731922398589e-07);
	const double r4 = D_MUL(r2, r2);
	const double b0 = D_FMA(r2, a1, a0);
	const double b1 = D_FMA(r2, a3, a2);
	const double b2 = D_FMA(r2, a5, a4);
	const double r8 = D_MUL(r4, r4);
	const double p = D_FMA(r8, b2, D_FMA(r4, b1, b0));
	/* 2^k is a normal double for every k the range [-104, 89] gives */
	double res = D_MUL(p, u2d(uint64_t((1023u + k) & 0x7FFu) << 52));
	res = xf > 89.0f ? u2d(0x7FF0000000000000ull) : res;
	res = xf < -104.0f ? 0.0 : res;
	return xf == xf ? res : x;
}

/* How close the double candidate c lies to a float rounding midpoint: the
 * distance in units of 2^-29 of the float spacing, read from the low 29 bits
 * of the double's significand (the part of c below the float spacing; the
 * midpoint is 2^28). Exact integer arithmetic, for c in the float normal
 * range [2^-126, 2^128); 0 outside it, so that such candidates always count
 * as near. */
LIBM_HD uint32_t exp_midpoint_units(double c) {
	const uint64_t b = d2u(c);
	const uint32_t e = uint32_t(b >> 52) & 0x7FFu;
	if(e < 897u || e > 1150u) return 0u;
	const int32_t d = int32_t(uint32_t(b) & 0x1FFFFFFFu) - 0x10000000;
	return uint32_t(d < 0 ? -d : d);
}

/* The exception table as an open-addressing hash: 2^bits slots of
 * (glibc result bits << 32 | input bits), linear probing from exp_hash(key);
 * empty slots hold EXP_EMPTY_KEY, which is no float in [-104, 89]. A probe
 * sequence never runs longer than `probe` slots (the longest run of occupied
 * slots plus one), so an absent key meets an empty slot within the bound. */
#define LIBM_EXP_EMPTY_KEY 0xFFFFFFFFu

LIBM_HD uint32_t exp_hash(uint32_t key, uint32_t bits) {
	return (key * 0x9E3779B1u) >> (32u - bits);
}

LIBM_HD uint64_t exp_slot_load(const uint64_t* p) {
#ifdef __CUDA_ARCH__
	return __ldg((const unsigned long long*) p);
#else
	return *p;
#endif
}

/* glibc's result for an input on which glibc rounds the other way from the
 * candidate; `fallback` (the rounded candidate) when the input is not in the
 * table. */
LIBM_HD float exp_lookup(float x, float fallback, const uint64_t* slots, uint32_t bits, uint32_t probe) {
	const uint32_t key = f2u(x);
	const uint32_t mask = (1u << bits) - 1u;
	uint32_t h = exp_hash(key, bits);
	for(uint32_t k = 0; k < probe; ++k) {
		const uint64_t e = exp_slot_load(slots + h);
		const uint32_t ek = uint32_t(e);
		if(ek == key) return u2f(uint32_t(e >> 32));
		if(ek == LIBM_EXP_EMPTY_KEY) break;
		h = (h + 1u) & mask;
	}
	return fallback;
}

/* glibc expf: the rounded candidate, or the exception table's value for an
 * input on which glibc rounds the other way (only candidates within
 * `nearUnits` of a midpoint can be such inputs) */
LIBM_HD float expf_match(float x, const uint64_t* slots, uint32_t bits, uint32_t probe, uint32_t nearUnits) {
	const double c = exp_candidate_d(x);
	const float r = float(c);
	if(probe && exp_midpoint_units(c) <= nearUnits) return exp_lookup(x, r, slots, bits, probe);
	return r;
}

LIBM_HD float apply_code(float cand, uint32_t code) {
	uint32_t b = f2u(cand);
	b += (code == 1u) ? 1u : 0u;
	b -= (code == 2u) ? 1u : 0u;
	return u2f(b);
}

LIBM_HD uint32_t table_code(const uint32_t* table, uint32_t idx) {
	return (table[idx >> 4] >> ((idx & 15u) * 2u)) & 3u;
}

} // namespace libm
} // namespace nemo_b200

#endif
