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
#else
/* Host builds of this header must use -ffp-contract=off. */
#define D_ADD(a, b) ((a) + (b))
#define D_SUB(a, b) ((a) - (b))
#define D_MUL(a, b) ((a) * (b))
#define D_DIV(a, b) ((a) / (b))
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
 * operations (identical on host and device): x = k ln2 + r with the
 * Cody-Waite split of ln2 (|r| <= ln2/2), e^r by its Taylor series to degree
 * 13 in Horner form, scaled by 2^k. Beyond the float range: 0 below -104,
 * infinity above 89; NaN stays NaN. */
LIBM_HD double exp_candidate_d(float xf) {
	if(!(xf == xf)) return double(xf);
	if(xf > 89.0f) return u2d(0x7FF0000000000000ull);
	if(xf < -104.0f) return 0.0;
	const double invln2 = 1.4426950408889634;
	const double ln2_hi = 6.93147180369123816490e-01;  /* 0x3FE62E42FEE00000 */
	const double ln2_lo = 1.90821492927058770002e-10;
	const double x = double(xf);
	const double t = D_MUL(x, invln2);
#ifdef __CUDA_ARCH__
	const int k = __double2int_rn(t);
#else
	const int k = int(nearbyint(t));
#endif
	const double kd = double(k);
	const double r = D_SUB(D_SUB(x, D_MUL(kd, ln2_hi)), D_MUL(kd, ln2_lo));
	double p = 1.6059043836821613e-10;           /* 1/13! */
	p = D_ADD(D_MUL(p, r), 2.08767569878681e-09);   /* 1/12! */
	p = D_ADD(D_MUL(p, r), 2.505210838544172e-08);  /* 1/11! */
	p = D_ADD(D_MUL(p, r), 2.755731922398589e-07);  /* 1/10! */
	p = D_ADD(D_MUL(p, r), 2.7557319223985893e-06); /* 1/9! */
	p = D_ADD(D_MUL(p, r), 2.48015873015873e-05);   /* 1/8! */
	p = D_ADD(D_MUL(p, r), 0.0001984126984126984);  /* 1/7! */
	p = D_ADD(D_MUL(p, r), 0.001388888888888889);   /* 1/6! */
	p = D_ADD(D_MUL(p, r), 0.008333333333333333);   /* 1/5! */
	p = D_ADD(D_MUL(p, r), 0.041666666666666664);   /* 1/4! */
	p = D_ADD(D_MUL(p, r), 0.16666666666666666);    /* 1/3! */
	p = D_ADD(D_MUL(p, r), 0.5);
	p = D_ADD(D_MUL(p, r), 1.0);
	p = D_ADD(D_MUL(p, r), 1.0);
	return D_MUL(p, u2d(uint64_t(1023 + k) << 52));
}

/* How far the double candidate c lies from the float rounding boundary, in
 * units of the float spacing at float(c): 0.5 - |c - float(c)| / spacing,
 * i.e. 0 on a midpoint and 0.5 on a float. Infinity and NaN give 1. */
LIBM_HD double exp_boundary(double c) {
	const float r = float(c);
	const uint32_t rb = f2u(r);
	if((rb & 0x7F800000u) == 0x7F800000u) return 1.0;
	const float nb = u2f(double(r) < c ? rb + 1u : (rb == 0u ? 1u : rb - 1u));
	const double spacing = double(nb) > double(r) ? D_SUB(double(nb), double(r)) : D_SUB(double(r), double(nb));
	const double off = c > double(r) ? D_SUB(c, double(r)) : D_SUB(double(r), c);
	return D_SUB(0.5, D_DIV(off, spacing));
}

/* Whether the candidate c lies within (0.5 - kfac) spacings of the float
 * rounding boundary (kfac = 0.5 - tau, tau from the exception table); the
 * division-free form of exp_boundary(c) <= tau. */
LIBM_HD bool exp_near_boundary(double c, double kfac) {
	const float r = float(c);
	const uint32_t rb = f2u(r);
	if((rb & 0x7F800000u) == 0x7F800000u) return false;
	const float nb = u2f(double(r) < c ? rb + 1u : (rb == 0u ? 1u : rb - 1u));
	const double spacing = double(nb) > double(r) ? D_SUB(double(nb), double(r)) : D_SUB(double(r), double(nb));
	const double off = c > double(r) ? D_SUB(c, double(r)) : D_SUB(double(r), c);
	return off >= D_MUL(kfac, spacing);
}

/* glibc expf: the rounded candidate, or the exception table's value for an
 * input on which glibc rounds the other way (keys sorted) */
LIBM_HD float expf_match(float x, const uint32_t* keys, const uint32_t* values, uint32_t count, double kfac) {
	const double c = exp_candidate_d(x);
	float r = float(c);
	if(count && exp_near_boundary(c, kfac)) {
		const uint32_t key = f2u(x);
		uint32_t lo = 0, hi = count;
		while(lo < hi) {
			const uint32_t mid = (lo + hi) >> 1;
			if(keys[mid] < key) lo = mid + 1;
			else hi = mid;
		}
		if(lo < count && keys[lo] == key) r = u2f(values[lo]);
	}
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
