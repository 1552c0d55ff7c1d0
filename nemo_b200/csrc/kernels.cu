/* sm_100a kernels of the per-cycle step path (interface: kernels.hpp).
 *
 * Compiled with -fmad=false; in addition every floating-point operation whose
 * rounding is observable goes through an explicit round-to-nearest intrinsic
 * (__fadd_rn, __dmul_rn, ...) so that neither contraction nor reassociation can
 * change the operation order of the reference CPU plugins
 * (src/nemo/cpu/plugins/<Model>.cpp). Integer current accumulation is exact
 * and order-independent, which is what makes the atomics bit-exact here. */

#include <cuda/atomic>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "kernels.hpp"
#include "libm_match.cuh"

namespace nemo_b200 {

namespace {

const unsigned FULL = 0xffffffffu;
/* words per block and cycle of the optional phase trace (kernels.hpp) */
const unsigned TRACE_WORDS = 20;

/* 64-bit shifts by a count that may reach 64, evaluated like the x86-64
 * shift the reference runs on (count modulo 64). */
__device__ __forceinline__ uint64_t shl64(uint64_t x, unsigned n) { return x << (n & 63u); }
__device__ __forceinline__ uint64_t shr64(uint64_t x, unsigned n) { return x >> (n & 63u); }

__device__ __forceinline__ unsigned long long globalTimer()
{
	unsigned long long t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

/* wfx_toFloat: saturate the int64 sum to int32, convert, scale
 * (src/nemo/fixedpoint.cpp:40-49). The reference divides by 2^f; the
 * product with 2^-f is the same float (both are exact: the quotient of an
 * integer-valued float of magnitude >= 1 by a power of two <= 2^31 is a
 * normal float), and a multiplication has no slow path. */
__device__ __forceinline__ float wfxToFloat(long long v, uint32_t fbits)
{
	v = v > 2147483647LL ? 2147483647LL : v;
	v = v < -2147483648LL ? -2147483648LL : v;
	return __fmul_rn(__ll2float_rn(v), __int_as_float(int((127u - fbits) << 23)));
}

/* Bring the bytes [lo, hi) of global memory into L2 ahead of their use: one
 * bulk prefetch through the copy engine (cp.async.bulk.prefetch.L2; a hint,
 * nothing waits for it), over the range rounded out to 16-byte boundaries.
 * The arrays it is used on start on a 256-byte boundary and carry 256 bytes
 * of padding, so the rounded range stays inside the allocation. */
__device__ __forceinline__ void prefetchL2(const void* lo, const void* hi)
{
	const size_t a = __cvta_generic_to_global(lo) & ~size_t(15);
	const size_t e = (__cvta_generic_to_global(hi) + 15u) & ~size_t(15);
	if(e > a) {
		asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" :: "l"(a), "r"(uint32_t(e - a)) : "memory");
	}
}

/* xorshift128 (src/nemo/RNG.cpp:10-18) */
__device__ __forceinline__ uint32_t urand(uint4& s)
{
	uint32_t t = s.x ^ (s.x << 11);
	s.x = s.y;
	s.y = s.z;
	s.z = s.w;
	s.w = (s.w ^ (s.w >> 19)) ^ (t ^ (t >> 8));
	return s.w;
}

/* Box-Muller sine branch (src/nemo/RNG.cpp:26-34) with glibc-matching
 * sinf/logf (libm_match.cuh) and IEEE sqrtf. */
__device__ __forceinline__ float nrandWords(uint32_t u1, uint32_t u2, const uint32_t* sinTab, const uint32_t* logTab)
{
	using namespace libm;
	float f1 = __uint2float_rn(u1);
	float f2 = __uint2float_rn(u2);
	float a = sin_argument(f1);
	float y = log_argument(f2);
	float L = apply_code(log_candidate(y), table_code(logTab, libm_index(f2)));
	float r = __fsqrt_rn(__fmul_rn(-2.0f, L));
	float S = apply_code(sin_candidate(a), table_code(sinTab, libm_index(f1)));
	return __fmul_rn(S, r);
}

__device__ __forceinline__ float nrand(uint4& s, const uint32_t* sinTab, const uint32_t* logTab)
{
	uint32_t u1 = urand(s);
	uint32_t u2 = urand(s);
	return nrandWords(u1, u2, sinTab, logTab);
}

/* Add a weight into the E (w >= 0) or I half of a current slot */
__device__ __forceinline__ void addCurrent(const NetDev& net, uint32_t slot, uint32_t target, int half, long long w)
{
	size_t idx = (size_t(slot) * net.nDev + target) * 2 + half;
	if(net.acc32) {
		atomicAdd(reinterpret_cast<unsigned*>(net.acc) + idx, (unsigned) (int) w);
	} else {
		atomicAdd(reinterpret_cast<unsigned long long*>(net.acc) + idx, (unsigned long long) w);
	}
}

/* Read and clear the raw E/I sums of neuron n in current slot `slot` */
__device__ __forceinline__ void takeSlot(const NetDev& net, uint32_t slot, uint32_t n, long long& e, long long& i)
{
	if(net.acc32) {
		int2* acc = reinterpret_cast<int2*>(net.acc) + size_t(slot) * net.nDev;
		const int2 a = acc[n];
		if(a.x | a.y) acc[n] = make_int2(0, 0);
		e = a.x;
		i = a.y;
	} else {
		longlong2* acc = reinterpret_cast<longlong2*>(net.acc) + size_t(slot) * net.nDev;
		const longlong2 a = acc[n];
		if(a.x | a.y) acc[n] = make_longlong2(0, 0);
		e = a.x;
		i = a.y;
	}
}

/* Add raw E/I sums into neuron n's slot (single writer) */
__device__ __forceinline__ void addSlot(const NetDev& net, uint32_t slot, uint32_t n, long long e, long long i)
{
	if(net.acc32) {
		int2* acc = reinterpret_cast<int2*>(net.acc) + size_t(slot) * net.nDev;
		const int2 a = acc[n];
		acc[n] = make_int2(a.x + int(e), a.y + int(i));
	} else {
		longlong2* acc = reinterpret_cast<longlong2*>(net.acc) + size_t(slot) * net.nDev;
		const longlong2 a = acc[n];
		acc[n] = make_longlong2(a.x + e, a.y + i);
	}
}

/* Read and clear neuron n's delay-1 inbox of cycle parity p */
__device__ __forceinline__ void takeInbox(const NetDev& net, uint32_t p, uint32_t n, long long& e, long long& i)
{
	if(net.acc32) {
		int2* box = reinterpret_cast<int2*>(net.inbox) + size_t(p) * net.nDev;
		const int2 a = box[n];
		if(a.x | a.y) box[n] = make_int2(0, 0);
		e = a.x;
		i = a.y;
	} else {
		longlong2* box = reinterpret_cast<longlong2*>(net.inbox) + size_t(p) * net.nDev;
		const longlong2 a = box[n];
		if(a.x | a.y) box[n] = make_longlong2(0, 0);
		e = a.x;
		i = a.y;
	}
}

/* Delay-1 synapses of the warp's fired neurons (lane ranges d1 of the
 * delay-1 part of the forward matrix, empty for lanes that did not fire) into
 * their targets' inbox of parity p, by fire-and-forget reductions: the
 * arrivals for the next cycle. The ranges are concatenated over the lanes
 * and worked off two records per lane at a time. Returns the number of
 * synapses added (warp total, on every lane). */
__device__ __forceinline__ uint32_t pushDelayOne(const NetDev& net, uint32_t firedMask, uint2 d1, uint32_t p,
		uint32_t lane)
{
	const uint32_t cnt = d1.y - d1.x;
	uint32_t incl = cnt;
#pragma unroll
	for(int d = 1; d < 32; d <<= 1) {
		const uint32_t x = __shfl_up_sync(FULL, incl, d);
		if(lane >= uint32_t(d)) incl += x;
	}
	const uint32_t total = __shfl_sync(FULL, incl, 31);
	const uint32_t excl = incl - cnt;
	const uint2* recs = net.fcm + net.d1Base;
	for(uint32_t base = 0; base < total; base += 64u) {
		uint32_t pos[2] = {0u, 0u};
		/* the record of each index: in the range of the fired lane that
		 * holds it */
		for(uint32_t m = firedMask; m; m &= m - 1) {
			const uint32_t L = uint32_t(__ffs(int(m)) - 1);
			const uint32_t eL = __shfl_sync(FULL, excl, L);
			const uint32_t cL = __shfl_sync(FULL, cnt, L);
			const uint32_t sL = __shfl_sync(FULL, d1.x, L);
#pragma unroll
			for(int h = 0; h < 2; ++h) {
				const uint32_t idx = base + uint32_t(h) * 32u + lane;
				if(idx >= eL && idx < eL + cL) pos[h] = sL + (idx - eL);
			}
		}
		uint2 r[2];
#pragma unroll
		for(int h = 0; h < 2; ++h) {
			r[h] = base + uint32_t(h) * 32u + lane < total ? __ldg(&recs[pos[h]]) : make_uint2(0u, 0u);
		}
#pragma unroll
		for(int h = 0; h < 2; ++h) {
			if(base + uint32_t(h) * 32u + lane < total) {
				const int32_t w = int32_t(r[h].y);
				const size_t idx = (size_t(p) * net.nDev + (r[h].x >> 6)) * 2 + (w < 0 ? 1 : 0);
				if(net.acc32) {
					atomicAdd(reinterpret_cast<unsigned*>(net.inbox) + idx, (unsigned) w);
				} else {
					atomicAdd(reinterpret_cast<unsigned long long*>(net.inbox) + idx, (unsigned long long) (long long) w);
				}
			}
		}
	}
	return total;
}

__device__ __forceinline__ float takeExternal(const NetDev& net, uint32_t n)
{
	float x = net.ext[n];
	if(x != 0.0f) {
		net.ext[n] = 0.0f;
	}
	return x;
}

/* ---------------- neuron models (one neuron per thread) ---------------- */

/* The models take the cycle's E and I currents from the caller (which drains
 * the neuron's slot) and load every other operand before their first store,
 * so that all loads of a neuron are in flight together. */

/* Izhikevich (src/nemo/cpu/plugins/Izhikevich.cpp:53-97). Parameters a, b, c,
 * d, sigma; state u, v. The v update evaluates its bracket in double (double
 * literals in the reference), the u update in float. `noise` is the cycle's
 * normal deviate (drawNoise), used when sigma is not 0. */
__device__ __forceinline__ bool modelIzhikevich(const NetDev& net, const GroupDev& g, uint32_t i, uint32_t n,
		float E, float I, bool stim, float noise)
{
	const size_t c = g.count;
	const float X = net.ext[n];
	/* parameters do not change during a launch: read-only loads */
	const float sigma = __ldg(&g.param[4 * c + i]);
	const float a = __ldg(&g.param[0 * c + i]);
	const float b = __ldg(&g.param[1 * c + i]);
	const float pc = __ldg(&g.param[2 * c + i]);
	const float pd = __ldg(&g.param[3 * c + i]);
	float u = g.state[0 * c + i];
	float v = g.state[1 * c + i];
	if(X != 0.0f) {
		net.ext[n] = 0.0f;
	}
	float In = __fadd_rn(__fadd_rn(E, I), X);
	if(sigma != 0.0f) {
		In = __fadd_rn(In, __fmul_rn(sigma, noise));
	}
	bool fired = false;
	for(int k = 0; k < 4; ++k) {
		if(!fired) {
			double vd = double(v);
			double br = __dadd_rn(__dsub_rn(__dadd_rn(__dmul_rn(__dadd_rn(__dmul_rn(0.04, vd), 5.0), vd), 140.0),
						double(u)), double(In));
			v = __double2float_rn(__dadd_rn(vd, __dmul_rn(0.25, br)));
			u = __fadd_rn(u, __fmul_rn(0.25f, __fmul_rn(a, __fsub_rn(__fmul_rn(b, v), u))));
			fired = v >= 30.0f;
		}
	}
	fired = fired || stim;
	if(fired) {
		v = pc;
		u = __fadd_rn(u, pd);
	}
	g.state[0 * c + i] = u;
	g.state[1 * c + i] = v;
	return fired;
}

/* The Izhikevich thalamic noise of one cycle (Izhikevich.cpp:62-64): a
 * normal deviate drawn from the neuron's generator when its sigma is not 0
 * (the generator advances only then); 0 otherwise. */
__device__ __forceinline__ float drawNoise(const NetDev& net, const GroupDev& g, uint32_t i)
{
	const float sigma = __ldg(&g.param[4 * size_t(g.count) + i]);
	float nz = 0.0f;
	if(sigma != 0.0f) {
		uint4 s = g.rng[i];
		nz = nrand(s, net.sinTab, net.logTab);
		g.rng[i] = s;
	}
	return nz;
}

/* drawNoise for the next cycle of resident stepping, without advancing the
 * neuron's generator: from state `from`, the deviate into noise[pNext] and
 * the state after it into rngAhead[pNext] (the state unchanged when sigma is
 * 0), where the next cycle's update takes both. */
__device__ __forceinline__ void drawNoiseAhead(const NetDev& net, const GroupDev& g, uint32_t i, uint32_t n, uint4 from,
		uint32_t pNext)
{
	const float sigma = __ldg(&g.param[4 * size_t(g.count) + i]);
	float nz = 0.0f;
	if(sigma != 0.0f) nz = nrand(from, net.sinTab, net.logTab);
	net.rngAhead[size_t(pNext) * net.nDev + n] = from;
	net.noise[size_t(pNext) * net.nDev + n] = nz;
}

/* IF_curr_exp (src/nemo/cpu/plugins/IF_curr_exp.cpp:74-121). Parameters in
 * IF_curr_exp.h order; state v, ie, ii, lastfire. Fires on v > v_thresh. */
__device__ __forceinline__ bool modelIfCurrExp(const NetDev& net, const GroupDev& g, uint32_t i, uint32_t n,
		float E, float I, bool stim)
{
	const size_t c = g.count;
	const float* P = g.param;
	float* S = g.state;
	const float X = net.ext[n];
	const float v_rest = P[0 * c + i], v_reset = P[1 * c + i], c_m = P[2 * c + i], tau_m = P[3 * c + i];
	const float tau_refrac = P[4 * c + i], tau_e = P[5 * c + i], tau_i = P[6 * c + i];
	const float v_thresh = P[7 * c + i], i_offset = P[8 * c + i];
	const float ie0 = S[1 * c + i], ii0 = S[2 * c + i];
	float v = S[0 * c + i];
	const float lastfire = S[3 * c + i];
	if(X != 0.0f) {
		net.ext[n] = 0.0f;
	}
	const float ie = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, __fdiv_rn(1.0f, tau_e)), ie0), E);
	const float ii = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, __fdiv_rn(1.0f, tau_i)), ii0), I);
	const float In = __fadd_rn(__fadd_rn(__fadd_rn(ie, ii), X), i_offset);
	S[1 * c + i] = ie;
	S[2 * c + i] = ii;
	const bool refractory = lastfire <= tau_refrac;
	if(!refractory) {
		v = __fadd_rn(v, __fadd_rn(__fdiv_rn(In, c_m), __fdiv_rn(__fsub_rn(v_rest, v), tau_m)));
	}
	const bool fired = (!refractory && v > v_thresh) || stim;
	if(fired) {
		S[3 * c + i] = 1.0f;
		S[0 * c + i] = v_reset;
	} else {
		S[3 * c + i] = __fadd_rn(lastfire, 1.0f);
		S[0 * c + i] = v;
	}
	return fired;
}

/* QIF (src/nemo/cpu/plugins/QIF.cpp:45-106): 10 RK4 substeps of 0.1 ms,
 * threshold 1, reset 0. */
__device__ __forceinline__ bool modelQif(const NetDev& net, const GroupDev& g, uint32_t i, uint32_t n,
		float E, float I, bool stim)
{
	const float dt = 0.1f;
	const float a1 = __fmul_rn(0.5f, dt);
	const float a2 = dt;
	const float bb1 = __fdiv_rn(dt, 6.0f);
	const float X = net.ext[n];
	float v = g.state[i];
	const float a = g.param[i];
	if(X != 0.0f) {
		net.ext[n] = 0.0f;
	}
	bool fired = false;
	for(int k = 0; k < 10; ++k) {
		if(!fired) {
			float In = __fmul_rn(__fadd_rn(__fadd_rn(E, I), X), 0.015f);
			float k1 = __fadd_rn(__fmul_rn(__fmul_rn(a, v), __fsub_rn(v, 1.0f)), In);
			float x2 = __fadd_rn(v, __fmul_rn(a1, k1));
			float k2 = __fadd_rn(__fmul_rn(__fmul_rn(a, x2), __fsub_rn(x2, 1.0f)), In);
			float x3 = __fadd_rn(v, __fmul_rn(a1, k2));
			float k3 = __fadd_rn(__fmul_rn(__fmul_rn(a, x3), __fsub_rn(x3, 1.0f)), In);
			float x4 = __fadd_rn(v, __fmul_rn(a2, k3));
			float k4 = __fadd_rn(__fmul_rn(__fmul_rn(a, x4), __fsub_rn(x4, 1.0f)), In);
			float sum = __fadd_rn(__fadd_rn(__fadd_rn(k1, __fmul_rn(2.0f, k2)), __fmul_rn(2.0f, k3)), k4);
			v = __fadd_rn(v, __fmul_rn(bb1, sum));
			fired = v >= 1.0f;
		}
	}
	fired = fired || stim;
	if(fired) {
		v = 0.0f;
	}
	g.state[i] = v;
	return fired;
}

__device__ __forceinline__ float expfMatch(const NetDev& net, float x)
{
	return libm::expf_match(x, net.expSlots, net.expBits, net.expProbe, net.expNear);
}

/* -a / d rounded to nearest for the constant divisors d of the HH rates,
 * from y = RN(1/d): q0 = RN(a y), the exact residual a - q0 d by FMA, and
 * one correction q0 + r y (Markstein's division step). Equal to __fdiv_rn(a,
 * d) for every a with |a| >= 2^-100, zero or infinite (checked over all such
 * floats by nemo_b200_hh_division_check); the HH argument v + 65 is zero or
 * at least 2^-17 in magnitude, the spacing of floats near -65. */
__device__ __forceinline__ float hhDivConst(float a, float d, float y)
{
	const float q0 = __fmul_rn(a, y);
	const float r = __fmaf_rn(-q0, d, a);
	const float q1 = __fmaf_rn(r, y, q0);
	return (r == 0.0f || !isfinite(q0)) ? q0 : q1;
}

/* Hodgkin-Huxley (src/nemo/cpu/plugins/HH.cpp:14-137): state v, n, m, h, dir;
 * no parameters. The currents act as conductances towards the reversal
 * potentials 0 and -70 mV. 999 Euler substeps of 0.001 ms ((int)(1/0.001f)
 * in float), six glibc-matching expf per substep; fires on the first
 * substep whose voltage change turns negative above -45 mV, from the 10th
 * cycle after the timer reset on.
 *
 * Each neuron has eight lanes (device indices devBase + 8 i .. + 7; only the
 * first is a neuron to the rest of the kernel). In a substep lane s of the
 * eight evaluates the rate that needs exponential s (alpha_n, alpha_m,
 * alpha_h, beta_n, beta_m, beta_h) and the six rates are exchanged by
 * shuffles; every lane then advances the same state with the same
 * operations. Called by all 32 lanes of a warp; `E`, `I` and the stimulus
 * are taken from the neuron's first lane. Returns the neuron's firing on all
 * its lanes. */
__device__ __forceinline__ bool modelHH(const NetDev& net, const GroupDev& g, uint32_t i, float E, float I,
		uint32_t stimWord, uint32_t cycle, uint32_t lane)
{
	const uint32_t lead = lane & ~7u, s = lane & 7u;
	const bool member = i < g.count;
	const size_t c = g.count;
	float* S = g.state;
	const float Excit = __shfl_sync(FULL, E, lead);
	const float Inhib = __shfl_sync(FULL, I, lead);
	const bool stim = (stimWord >> lead) & 1u;
	const uint32_t nLead = g.devBase + (i << 3);
	const float Exter = member ? net.ext[nLead] : 0.0f;
	float v = member ? S[0 * c + i] : -65.0f;
	float nn = member ? S[1 * c + i] : 0.0f;
	float m = member ? S[2 * c + i] : 0.0f;
	float h = member ? S[3 * c + i] : 0.0f;
	float dir = member ? S[4 * c + i] : 0.0f;
	__syncwarp();
	if(member && s == 0u && Exter != 0.0f) {
		net.ext[nLead] = 0.0f;
	}
	const float dt = 0.001f;
	const float gNa = 120.0f, gK = 36.0f, gL = 0.3f;
	const float ENa = __fsub_rn(115.0f, 65.0f);
	const float EK = __fsub_rn(-12.0f, 65.0f);
	const float EL = __fsub_rn(10.6f, 65.0f);
	const float RevE = 0.0f, RevI = -70.0f;
	const int incMax = int(__fdiv_rn(1.0f, dt));
	/* this lane's exponent: a - 0.1 (v + 65) for s = 0, 1, 5 (a = 1, 2.5,
	 * 3), -(v + 65) / d for s = 2, 3, 4 (d = 20, 80, 18), none for 6, 7 */
	const bool argDiv = s >= 2u && s <= 4u;
	const float argA = s == 0u ? 1.0f : (s == 1u ? 2.5f : 3.0f);
	const float argD = s == 2u ? 20.0f : (s == 3u ? 80.0f : 18.0f);
	const float argY = __fdiv_rn(1.0f, argD);
	/* this lane's rate: num / (e -+ 1) for s = 0, 1, 5, coef * e for 2, 3, 4 */
	const bool rateDiv = s <= 1u || s == 5u;
	const float rateCoef = s == 2u ? 0.07f : (s == 3u ? 0.125f : 4.0f);
	const bool lookup = net.expProbe != 0u;
	bool fired = false;
	for(int t = 0; t < incMax; ++t) {
		const float vr = __fadd_rn(v, 65.0f);
		/* (RevI - v) / -1 is the exact negation */
		const float I = __fadd_rn(__fadd_rn(__fmul_rn(Excit, __fsub_rn(RevE, v)),
					__fmul_rn(Inhib, -__fsub_rn(RevI, v))), Exter);
		const float tenth = __fmul_rn(0.1f, vr);
		float x = argDiv ? hhDivConst(-vr, argD, argY) : __fsub_rn(argA, tenth);
		x = s < 6u ? x : 0.0f;
		const double cand = libm::exp_candidate_d(x);
		float e = float(cand);
		if(lookup && libm::exp_midpoint_units(cand) <= net.expNear) {
			e = libm::exp_lookup(x, e, net.expSlots, net.expBits, net.expProbe);
		}
		const float num = s == 0u ? __fsub_rn(0.1f, __fmul_rn(0.01f, vr)) : (s == 1u ? __fsub_rn(2.5f, tenth) : 1.0f);
		const float den = s == 5u ? __fadd_rn(e, 1.0f) : __fsub_rn(e, 1.0f);
		const float rate = rateDiv ? __fdiv_rn(num, den) : __fmul_rn(rateCoef, e);
		const float alphan = __shfl_sync(FULL, rate, lead + 0u);
		const float alpham = __shfl_sync(FULL, rate, lead + 1u);
		const float alphah = __shfl_sync(FULL, rate, lead + 2u);
		const float betan = __shfl_sync(FULL, rate, lead + 3u);
		const float betam = __shfl_sync(FULL, rate, lead + 4u);
		const float betah = __shfl_sync(FULL, rate, lead + 5u);
		m = __fadd_rn(m, __fmul_rn(dt, __fsub_rn(__fmul_rn(alpham, __fsub_rn(1.0f, m)), __fmul_rn(betam, m))));
		nn = __fadd_rn(nn, __fmul_rn(dt, __fsub_rn(__fmul_rn(alphan, __fsub_rn(1.0f, nn)), __fmul_rn(betan, nn))));
		h = __fadd_rn(h, __fmul_rn(dt, __fsub_rn(__fmul_rn(alphah, __fsub_rn(1.0f, h)), __fmul_rn(betah, h))));
		const float m3 = __fmul_rn(__fmul_rn(m, m), m);
		const float n4 = __fmul_rn(__fmul_rn(__fmul_rn(nn, nn), nn), nn);
		const float Ik = __fadd_rn(__fadd_rn(
					__fmul_rn(__fmul_rn(__fmul_rn(gNa, m3), h), __fsub_rn(v, ENa)),
					__fmul_rn(__fmul_rn(gK, n4), __fsub_rn(v, EK))),
				__fmul_rn(gL, __fsub_rn(v, EL)));
		/* division by C = 1 is exact */
		const float newv = __fadd_rn(v, __fmul_rn(dt, __fadd_rn(-Ik, I)));
		const float newDir = __fsub_rn(newv, v);
		const float change = ((dir < 0.0f) | (newv < -45.0f)) ? 0.0f : newDir;
		dir = newDir;
		if(!fired && cycle >= 10u) {
			fired = double(change) < -0.000000001;
		}
		v = newv;
	}
	fired = fired || stim;
	if(member && s == 0u) {
		S[0 * c + i] = v;
		S[1 * c + i] = nn;
		S[2 * c + i] = m;
		S[3 * c + i] = h;
		S[4 * c + i] = dir;
	}
	return fired;
}

/* PoissonSource (src/nemo/cpu/plugins/PoissonSource.cpp:21-29). The
 * currents (drained by the caller, as every neuron's slot must be) and the
 * external current (cleared) are unused. */
__device__ __forceinline__ bool modelPoisson(const NetDev& net, const GroupDev& g, uint32_t i, uint32_t n,
		float, float, bool stim)
{
	(void) takeExternal(net, n);
	uint32_t p0 = uint32_t(__fmul_rn(g.param[i], 65536.0f));
	uint4 s = g.rng[i];
	uint32_t p1 = urand(s) & 0xffffu;
	g.rng[i] = s;
	return p1 < p0 || stim;
}

/* Input (src/nemo/cpu/plugins/Input.cpp:56-60) */
__device__ __forceinline__ bool modelInput(const NetDev& net, const GroupDev&, uint32_t, uint32_t n,
		float, float, bool stim)
{
	(void) takeExternal(net, n);
	return stim;
}

/* ---------------- STDP rule (src/nemo/StdpProcess.cpp:68-138) ---------------- */

__device__ __forceinline__ int32_t updateRegion(uint64_t arrivals, const StdpRule& R)
{
	if(!arrivals) return 0;
	const uint32_t NONE = 0xffffffffu;
	uint64_t vpre = arrivals & R.prePostBits;
	uint32_t dtPre = vpre ? uint32_t(__ffsll((long long) shr64(vpre, R.postPreWindow)) - 1) : NONE;
	uint64_t vpost = arrivals & R.postPreBits;
	uint32_t dtPost = vpost ? uint32_t(__clzll((long long) shl64(vpost, 64u - R.postPreWindow))) : NONE;
	if(dtPre < dtPost) return R.fnPre[dtPre];
	if(dtPost < dtPre) return R.fnPost[dtPost];
	return 0;
}

__device__ __forceinline__ int32_t weightChange(uint64_t pre, const StdpRule& R)
{
	return int32_t(uint32_t(updateRegion(pre & R.potentiation, R)) + uint32_t(updateRegion(pre & R.depression, R)));
}

__device__ __forceinline__ int32_t updatedWeight(int32_t wOld, int32_t wDiff, const StdpRule& R)
{
	int32_t sum = int32_t(uint32_t(wOld) + uint32_t(wDiff));
	if(wOld > 0) return min(R.maxE, max(sum, R.minE));
	if(wOld < 0) return min(R.minI, max(sum, R.maxI));
	return 0;
}

/* ---------------- grid barrier with a bounded wait ---------------- */

/* Barrier over all blocks of the cooperative launch. bar[0] counts arrivals
 * and never goes back: the i-th barrier of a launch that started at count
 * `base` (bar[1], read by every block before its first arrival) is passed
 * once the count reaches base + i * gridDim.x. Arriving is one release
 * reduction, so the last block's arrival is visible to the waiting blocks
 * after a single trip through L2. A block that waits longer than timeoutNs
 * sets the error word and returns false; every waiting block also gives up
 * as soon as it sees the error word, so the kernel always terminates. */
__device__ __forceinline__ bool gridSync(unsigned* bar, unsigned target, unsigned long long timeoutNs)
{
	__shared__ int ok;
	__syncthreads();
	if(threadIdx.x == 0) {
		int good = 1;
		/* the block's writes are ordered before this thread's by the
		 * __syncthreads above; the release makes them visible with the
		 * arrival */
		const size_t gbar = __cvta_generic_to_global(bar);
		asm volatile("red.release.gpu.global.add.u32 [%0], 1;" :: "l"(gbar) : "memory");
		unsigned long long start = 0;
		unsigned spins = 0;
		for(;;) {
			unsigned v;
			asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(gbar) : "memory");
			if(int(v - target) >= 0) break;
			if((++spins & 255u) == 0) {
				if(start == 0) start = globalTimer();
				if(*(volatile unsigned*) &bar[2]) {
					good = 0;
					break;
				}
				if(globalTimer() - start > timeoutNs) {
					*(volatile unsigned*) &bar[2] = 1u;
					good = 0;
					break;
				}
			}
		}
		ok = good;
	}
	__syncthreads();
	return ok != 0;
}

/* ---------------- the persistent step kernel ---------------- */

/* Exclusive prefix of cnt[0, n) into pre[0, n], by one warp */
__device__ __forceinline__ void warpPrefix(const uint32_t* cnt, uint32_t n, uint32_t* pre, uint32_t lane)
{
	const uint32_t per = (n + 31u) / 32u;
	const uint32_t lo = min(n, lane * per), hi = min(n, lo + per);
	uint32_t sum = 0;
	for(uint32_t i = lo; i < hi; ++i) sum += cnt[i];
	uint32_t incl = sum;
#pragma unroll
	for(int d = 1; d < 32; d <<= 1) {
		uint32_t x = __shfl_up_sync(FULL, incl, d);
		if(lane >= uint32_t(d)) incl += x;
	}
	uint32_t run = incl - sum;
	for(uint32_t i = lo; i < hi; ++i) {
		pre[i] = run;
		run += cnt[i];
	}
	if(lane == 31) pre[n] = incl;
}

/* The list (block) holding entry j of a concatenation with prefix pre[0, n]:
 * the last b with pre[b] <= j (j < pre[n]) */
__device__ __forceinline__ uint32_t findList(const uint32_t* pre, uint32_t n, uint32_t j)
{
	uint32_t lo = 0, hi = n;
	while(hi - lo > 1) {
		uint32_t mid = (lo + hi) >> 1;
		if(pre[mid] <= j) lo = mid;
		else hi = mid;
	}
	return lo;
}

/* Block 0 of a resident launch, after its phase for command seq: wait (first
 * warp, at most idleNs) for command seq + 1 in host memory (ResidentHostCmd:
 * every lane reads one chunk per try, and the command is taken when each
 * chunk its payload needs carries seq + 1) and copy it into the broadcast
 * buffer of the next phase (parity (k + 1) & 1: the buffer of this phase's
 * command stays as it is), its number last; an exit command or the idle limit
 * copies an exit. Called by all threads of block 0. */
__device__ __forceinline__ void residentNext(const CycleArgs& A, uint32_t seq, uint32_t k, uint32_t warp, uint32_t lane)
{
	if(warp == 0) {
		const size_t chunkAddr = __cvta_generic_to_global(&A.cmd->c[lane]);
		const unsigned long long start = globalTimer();
		uint4 ch = make_uint4(0u, 0u, 0u, 0u);
		bool got = false;
		for(;;) {
			asm volatile("ld.volatile.global.v4.u32 {%0, %1, %2, %3}, [%4];"
					: "=r"(ch.x), "=r"(ch.y), "=r"(ch.z), "=r"(ch.w) : "l"(chunkAddr) : "memory");
			/* chunk 0: {seq, op, nf, ni}; the payload needs ceil((3 + nf +
			 * 2 ni) / 3) chunks */
			const uint32_t nf = min(__shfl_sync(FULL, ch.z, 0), INLINE_STIM_MAX);
			const uint32_t ni = min(__shfl_sync(FULL, ch.w, 0), INLINE_STIM_MAX);
			const uint32_t need = min((3u + nf + 2u * ni + 2u) / 3u, RESIDENT_CHUNKS);
			const uint32_t fresh = __ballot_sync(FULL, ch.x == seq + 1u);
			const uint32_t want = need >= 32u ? FULL : ((1u << need) - 1u);
			if((fresh & want) == want) {
				got = true;
				break;
			}
			/* lane 0's clock decides for the warp, so that every lane leaves
			 * the loop on the same try */
			if(__shfl_sync(FULL, globalTimer() - start > A.idleNs ? 1u : 0u, 0)) break;
		}
		/* the payload words, in lane order: word 3 l + j is chunk l's w[j] */
		ResidentCmd* c = A.bcast + ((k + 1u) & 1u);
		const uint32_t op = got ? __shfl_sync(FULL, ch.y, 0) : RESIDENT_EXIT;
		const bool step = op == RESIDENT_STEP;
		const uint32_t nf = step ? min(__shfl_sync(FULL, ch.z, 0), INLINE_STIM_MAX) : 0u;
		const uint32_t ni = step ? min(__shfl_sync(FULL, ch.w, 0), INLINE_STIM_MAX) : 0u;
		/* payload word p (p >= 3) is chunk p / 3's word p % 3; every lane
		 * takes part in each round's shuffles */
		for(uint32_t base = 3u; base < 3u + nf + 2u * ni; base += 32u) {
			const uint32_t p = base + lane;
			const uint32_t l = min(p / 3u, 31u), j = p - 3u * (p / 3u);
			const uint32_t y = __shfl_sync(FULL, ch.y, l);
			const uint32_t z = __shfl_sync(FULL, ch.z, l);
			const uint32_t w = __shfl_sync(FULL, ch.w, l);
			const uint32_t v = j == 0u ? y : (j == 1u ? z : w);
			const uint32_t q = p - 3u;
			if(p < 3u + nf + 2u * ni) {
				if(q < nf) c->f[q] = v;
				else if(q < nf + ni) c->i[q - nf] = v;
				else c->cur[q - nf - ni] = __uint_as_float(v);
			}
		}
		if(lane == 0) {
			c->nf = nf;
			c->ni = ni;
			c->op = step ? RESIDENT_STEP : RESIDENT_EXIT;
		}
		__syncwarp();
		if(lane == 0) {
			/* the command's fields, then its number, for the other blocks */
			const size_t seqAddr = __cvta_generic_to_global(&c->seq);
			asm volatile("st.release.gpu.global.u32 [%0], %1;" :: "l"(seqAddr), "r"(seq + 1u) : "memory");
		}
	}
	__syncthreads();
}

/* The other blocks of a resident launch, after their phase for command seq:
 * wait (thread 0) for block 0's copy of command seq + 1. Block 0 forwards a
 * command only after the host has seen every block's phase done, so nothing
 * else orders the phases. Returns false when the wait gives up (limit
 * timeoutNs; the launch is then in error). */
__device__ __forceinline__ bool residentWait(const CycleArgs& A, uint32_t seq, uint32_t k)
{
	__shared__ int ok;
	if(threadIdx.x == 0) {
		const size_t seqAddr = __cvta_generic_to_global(&A.bcast[(k + 1u) & 1u].seq);
		const unsigned long long start = globalTimer();
		int good = 1;
		for(uint32_t spins = 0;; ++spins) {
			uint32_t v;
			asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(seqAddr) : "memory");
			if(v == seq + 1u) break;
			if((spins & 255u) == 255u && globalTimer() - start > A.timeoutNs) {
				good = 0;
				break;
			}
		}
		ok = good;
	}
	__syncthreads();
	return ok != 0;
}

/* Add one forward-matrix record into current slot `slot` of its target
 * (E for w >= 0, else I), in shared memory or in net.acc */
template<bool SMEM>
__device__ __forceinline__ void gatherAdd(const NetDev& net, int2* sAcc, uint32_t ownN, uint32_t ownBase, uint32_t slot,
		uint2 r)
{
	const int32_t w = int32_t(r.y);
	const uint32_t target = r.x >> 6;
	if(SMEM) {
		int* cell = reinterpret_cast<int*>(&sAcc[slot * ownN + (target - ownBase)]);
		atomicAdd(cell + (w < 0 ? 1 : 0), w);
	} else {
		addCurrent(net, slot, target, w < 0 ? 1 : 0, w);
	}
}

/* The fired words of cycle t (its row of the firing ring) of the
 * simulation's warps into host memory as CycleArgs::hostWords describes: the
 * words that are not 0 with their warps, in warp order. Called by every
 * thread of one block, after every block has written its words and fenced;
 * the words are read from L2. Four words per thread are loaded at once. */
__device__ __forceinline__ void writeStepList(const NetDev& net, uint32_t* hostWords, uint32_t t, uint32_t warp, uint32_t lane)
{
	__shared__ uint32_t sCnt[33];
	const uint32_t T = blockDim.x;
	const uint32_t warps = T >> 5;
	const uint32_t lt = (1u << lane) - 1u;
	const uint32_t w0 = net.warpBase;
	const uint32_t nw = net.ownStart[gridDim.x];
	const uint32_t* row = net.firedRing + size_t(t & net.ringMask) * net.nWords + w0;
	uint2* out = reinterpret_cast<uint2*>(hostWords + 2);
	uint32_t done = 0;
	for(uint32_t r0 = 0; r0 < nw; r0 += 4u * T) {
		uint32_t word[4];
#pragma unroll
		for(int q = 0; q < 4; ++q) {
			const uint32_t w = r0 + uint32_t(q) * T + threadIdx.x;
			word[q] = w < nw ? __ldcg(&row[w]) : 0u;
		}
#pragma unroll
		for(int q = 0; q < 4; ++q) {
			if(r0 + uint32_t(q) * T >= nw) break;   /* the same for the whole block */
			const uint32_t w = r0 + uint32_t(q) * T + threadIdx.x;
			const uint32_t m = __ballot_sync(0xffffffffu, word[q] != 0u);
			if(lane == 0) sCnt[warp] = uint32_t(__popc(m));
			__syncthreads();
			if(warp == 0) {
				const uint32_t v = lane < warps ? sCnt[lane] : 0u;
				uint32_t incl = v;
#pragma unroll
				for(int d = 1; d < 32; d <<= 1) {
					const uint32_t x = __shfl_up_sync(0xffffffffu, incl, d);
					if(lane >= uint32_t(d)) incl += x;
				}
				sCnt[lane] = incl - v;
				if(lane == 31) sCnt[32] = incl;
			}
			__syncthreads();
			if(word[q]) out[done + sCnt[warp] + uint32_t(__popc(m & lt))] = make_uint2(word[q], w0 + w);
			done += sCnt[32];
			__syncthreads();
		}
	}
	if(threadIdx.x == 0) hostWords[1] = done;
}

/* k_cycles: see kernels.hpp for the phase structure. HOST: the launch may
 * write a step list to host memory or stay resident (CycleArgs::hostWords,
 * cmd); launches that do neither use the instantiation without that code,
 * which leaves the rest more registers. The forward regions and
 * the reverse-matrix arrays are streamed with evict-first loads and stores
 * (__ldcs / __stcs), so that they do not push the randomly read firing
 * history, segment offsets and noise tables out of L2. SMEM: the owned current
 * slots live in dynamic shared memory as int32 E/I pairs,
 * sAcc[slot * ownN + local]; otherwise every access goes to net.acc. */
template<bool SMEM, unsigned T, bool HOST>
__global__ void __launch_bounds__(T, 1)
k_cycles(const __grid_constant__ CycleArgs A)
{
	extern __shared__ int2 sAcc[];
	__shared__ uint32_t sPreF[MAX_BLOCKS + 2];    /* + the remote list of a shard */
	__shared__ uint32_t sPreP[MAX_BLOCKS + 1];
	__shared__ uint32_t sNFired, sNPost, sWork, sLast;
	__shared__ unsigned long long sEvents, sPushed, sVisits;

	const NetDev& net = A.net;
	const uint32_t tid = threadIdx.x;
	const uint32_t lane = tid & 31u;
	const uint32_t warp = tid >> 5;
	const uint32_t lt = (1u << lane) - 1u;
	const uint32_t warpsPerBlock = blockDim.x >> 5;
	const uint32_t B = gridDim.x;
	const uint32_t b = blockIdx.x;
	const size_t nDev = net.nDev;
	const uint32_t ownN = net.ownWarps * 32u;       /* list and slot stride per block */
	const uint32_t firstWarp = net.warpBase + net.ownStart[b];
	const uint32_t myWarps = net.ownStart[b + 1] - net.ownStart[b];
	const uint32_t myN = myWarps * 32u;
	const uint32_t ownBase = firstWarp * 32u;
	const uint32_t updWarps = min(myWarps, warpsPerBlock);
	const size_t listStride = size_t(B) * ownN;  /* one parity of the fired lists */
	const size_t postParity = size_t(B) * net.postStride;   /* one parity of the STDP entries */
	int2* acc32 = reinterpret_cast<int2*>(net.acc);
	/* this block's buckets of the forward matrix: bucket of source s =
	 * segKey0 + s * segStride */
	const uint32_t grp = net.groupOf[b];
	const uint32_t grpFirst = net.groupFirst[grp];
	const uint32_t segStride = net.groupFirst[grp + 1] - grpFirst;
	const size_t segKey0 = size_t(grpFirst) * nDev + (b - grpFirst);

	/* the first cycle: a kernel parameter, or (for launches replayed from a
	 * CUDA graph) a device counter that block 0 advances at the end */
	const uint64_t first = A.cycleCounter ? *A.cycleCounter : A.firstCycle;
	/* arrivals at the grid barrier when the launch started */
	const unsigned barBase = *(volatile unsigned*) &net.barrier[1];

	if(SMEM) {
		const uint32_t total = net.slots * ownN;
		for(uint32_t x = tid; x < total; x += blockDim.x) {
			const uint32_t s = x / ownN, l = x - s * ownN;
			const size_t n = size_t(ownBase) + l;
			sAcc[x] = l < myN ? acc32[size_t(s) * nDev + n] : make_int2(0, 0);
		}
	}

	/* carry bit 1: the launch ends with its last update phase; the cycle's
	 * gathering waits for the next launch, and nothing follows that phase,
	 * so it needs no grid barrier after it (a one-cycle step has none at
	 * all and runs as an ordinary launch) */
	/* resident stepping (CycleArgs::cmd): one update phase per command until
	 * an exit command or the idle limit; the last cycle stays pending */
	const bool resident = HOST && A.cmd != nullptr;
	const bool lastPending = resident || (A.carry & 2u) != 0u;
	const uint32_t phases = resident ? 0xffffffffu : A.cycles + (lastPending ? 0u : 1u);
	const uint32_t barriers = lastPending && A.cycles ? A.cycles - 1u : A.cycles;
	uint32_t passed = 0;   /* grid barriers passed */
	uint32_t k = 0;
	for(; k < phases; ++k) {
		const uint64_t t64 = first + k;
		const uint32_t t = uint32_t(t64);
		const bool doUpdate = resident || k < A.cycles;
		/* this phase's stimulus: the launch's own (first phase), or the
		 * command block 0 copied before the last grid barrier */
		uint32_t stNf = 0u, stNi = 0u;
		const uint32_t* stF = nullptr;
		const uint32_t* stI = nullptr;
		const float* stC = nullptr;
		if(k == 0) {
			stNf = A.inlineNf;
			stNi = A.inlineNi;
			stF = A.inlineF;
			stI = A.inlineI;
			stC = A.inlineCur;
		} else if(resident) {
			const ResidentCmd* c = A.bcast + (k & 1u);
			stNf = c->nf;
			stNi = c->ni;
			stF = c->f;
			stI = c->i;
			stC = c->cur;
		}
		const bool doPrev = k > 0 || (A.carry & 1u);     /* gather and learn for cycle t-1 */
		const uint32_t slotT = uint32_t(t64 % net.slots);

		if(tid == 0) {
			sNFired = 0;
			sNPost = 0;
			sWork = 0;
			sEvents = 0;
			sPushed = 0;
			sVisits = 0;
			if(doUpdate && b == 0) {
				net.firedCountRing[(t + 1) & net.ringMask] = 0;
				net.eventsRing[(t + 1) & net.ringMask] = 0;
			}
		}
		if(doPrev) {
			const uint32_t par = (t - 1u) & 1u;
			if(warp == 0) {
				warpPrefix(net.firedCnt + par * B, B, sPreF, lane);
				/* a shard's remote fired sources: list B */
				if(lane == 31 && net.remoteList) sPreF[B + 1] = sPreF[B] + net.remoteCnt[par];
			}
			if(warp == 1 && net.stdp) warpPrefix(net.postCnt + par * B, B, sPreP, lane);
		}
		__syncthreads();
		unsigned long long* trace = A.trace ? A.trace + (size_t(k) * B + b) * TRACE_WORDS : nullptr;
		if(trace && tid == 0) trace[0] = globalTimer();

		/* ---- neuron update of cycle t for the owned neurons, by the first
		 * updWarps warps; the other warps start on the deferred work below
		 * at once. The current of cycle t is its slot plus the delay-1
		 * inbox filled when the sources fired ---- */
		if(warp < updWarps && doUpdate) {
			const uint32_t par = t & 1u;
			const uint64_t* rfIn = net.rf + (t & 1u) * nDev;
			uint64_t* rfOut = net.rf + ((t + 1u) & 1u) * nDev;
			uint32_t* firedOut = net.firedList + par * listStride + size_t(b) * ownN;
			uint2* postOut = net.postList + par * postParity + size_t(b) * net.postStride;
			uint32_t pushed = 0;
			for(uint32_t lw = warp; lw < myWarps; lw += warpsPerBlock) {
				const uint32_t w0 = trace ? uint32_t(globalTimer()) : 0u;   /* low words: differences of a few µs */
				const uint32_t dw = firstWarp + lw;
				int gi = 0;
				while(dw >= A.groupWarp[gi + 1]) ++gi;
				const GroupDev& G = A.groups[gi];
				const uint32_t n = dw * 32u + lane;
				const uint32_t rel = n - G.devBase;
				const uint32_t i = rel >> G.shift;
				/* a neuron at this device index (not one of an HH neuron's
				 * seven helper lanes) */
				const bool valid = (rel & ((1u << G.shift) - 1u)) == 0u && i < G.count;
				/* the firing-stimulus word (every lane loads it: one
				 * transaction, and nothing waits for it before the model
				 * needs it); cleared after the model has issued its loads,
				 * so that nothing orders them behind it */
				uint32_t stimWord = net.fstim[dw];
				if(stNf | stNi) {
					/* a step's short stimulus, from the parameters or the
					 * resident command: this warp's firing bits, and the
					 * currents of its own neurons (read by the model below,
					 * by every lane of an HH neuron) */
					for(uint32_t q = 0; q < stNf; ++q) {
						const uint32_t x = stF[q];
						if((x >> 5) == dw) stimWord |= 1u << (x & 31u);
					}
					for(uint32_t q = 0; q < stNi; ++q) {
						if(stI[q] == n) net.ext[n] = stC[q];
					}
					__syncwarp();
				}
				/* operands needed after the update, loaded with its own */
				const uint64_t rfPrev = valid ? rfIn[n] : 0ull;
				const uint32_t deg = valid ? __ldg(&net.outDegree[n]) : 0u;
				uint2 rcm = make_uint2(0u, 0u);
				if(valid && net.stdp) rcm = make_uint2(__ldg(&net.rcmStart[n]), __ldg(&net.rcmStart[n + 1]));
				uint2 d1 = make_uint2(0u, 0u);
				if(valid && net.deliver) d1 = make_uint2(__ldg(&net.d1Start[n]), __ldg(&net.d1Start[n + 1]));
				long long e, in;
				takeInbox(net, par, n, e, in);
				if(SMEM) {
					int2* cell = &sAcc[slotT * ownN + lw * 32u + lane];
					const int2 a = *cell;
					*cell = make_int2(0, 0);
					e += a.x;
					in += a.y;
				} else {
					long long se, si;
					takeSlot(net, slotT, n, se, si);
					e += se;
					in += si;
				}
				const float E = wfxToFloat(e, net.fbits);
				const float I = wfxToFloat(in, net.fbits);
				bool fired = false;
				if(G.kind == 3) {   /* MODEL_HH */
					/* all lanes: eight per neuron */
					fired = modelHH(net, G, i, E, I, stimWord, t - G.timerBase, lane) && valid;
				} else if(valid) {
					const bool stim = (stimWord >> lane) & 1u;
					switch(G.kind) {
						case 0: {
							/* the first cycle of a launch draws its noise here;
							 * later ones use the draw made in the phase before.
							 * A resident launch cannot know whether a next cycle
							 * comes, and a draw advances the generator: there the
							 * draw ahead leaves the generator alone, and the
							 * cycle that uses it advances it here */
							float nz;
							uint4 ahead = make_uint4(0u, 0u, 0u, 0u);
							if(k == 0) {
								nz = drawNoise(net, G, i);
							} else {
								nz = net.noise[par * nDev + n];
								if(resident) ahead = net.rngAhead[size_t(par) * nDev + n];
							}
							fired = modelIzhikevich(net, G, i, n, E, I, stim, nz);
							/* stored after the model has issued its loads */
							if(k > 0 && resident) G.rng[i] = ahead;
							break;
						}
						case 1: fired = modelIfCurrExp(net, G, i, n, E, I, stim); break;
						case 2: fired = modelQif(net, G, i, n, E, I, stim); break;
						case 4: fired = modelPoisson(net, G, i, n, E, I, stim); break;
						case 6:
							/* a plugin model: its firing, stimulus included,
							 * from the bits its update wrote for this cycle */
							fired = (__ldg(&G.extFired[i >> 5]) >> (i & 31u)) & 1u;
							break;
						default: fired = modelInput(net, G, i, n, E, I, stim); break;
					}
				}
				if(lane == 0 && stimWord) net.fstim[dw] = 0u;
				const uint64_t rfNew = (rfPrev << 1) | uint64_t(fired);
				if(valid) {
					rfOut[n] = rfNew;
				}
				const uint32_t word = __ballot_sync(FULL, fired);
				const uint32_t w1 = trace ? uint32_t(globalTimer()) : 0u;
				if(lane == 0) net.firedRing[size_t(t & net.ringMask) * net.nWords + dw] = word;
				if(net.stdp) {
					/* post-synaptic firing P cycles ago (ConnectivityMatrix.cpp:237):
					 * the target's plastic synapses as runs of at most
					 * stdpRun, one list entry each */
					const bool post = valid && ((rfNew >> net.postShift) & 1ull);
					const uint32_t len = post ? rcm.y - rcm.x : 0u;
					const uint32_t run = net.stdpRun;
					const uint32_t runs = (len + run - 1u) / run;
					if(__ballot_sync(FULL, runs != 0u)) {
						uint32_t incl = runs;
#pragma unroll
						for(int d = 1; d < 32; d <<= 1) {
							const uint32_t x = __shfl_up_sync(FULL, incl, d);
							if(lane >= uint32_t(d)) incl += x;
						}
						uint32_t base = 0;
						if(lane == 31) base = atomicAdd(&sNPost, incl);
						base = __shfl_sync(FULL, base, 31) + incl - runs;
						for(uint32_t r = 0; r < runs; ++r) {
							const uint32_t off = r * run;
							postOut[base + r] = make_uint2(rcm.x + off, min(run, len - off));
						}
						if(runs) {
							/* the next phase's STDP accumulation walks this
							 * target's reverse range: into L2 now */
							prefetchL2(net.rcmSrcDelay + rcm.x, net.rcmSrcDelay + rcm.y);
							prefetchL2(net.rcmAcc + rcm.x, net.rcmAcc + rcm.y);
						}
					}
				}
				const uint32_t w2 = trace ? uint32_t(globalTimer()) : 0u;
				if(word) {
					uint32_t base = 0;
					if(lane == 0) base = atomicAdd(&sNFired, uint32_t(__popc(word)));
					base = __shfl_sync(FULL, base, 0);
					if(fired) {
						firedOut[base + __popc(word & lt)] = n;
					}
					const uint32_t ev = __reduce_add_sync(FULL, fired ? deg : 0u);
					if(lane == 0) atomicAdd(&sEvents, (unsigned long long) ev);
					if(net.deliver) {
						/* every block gathers these sources next phase: their
						 * chunk of each block group, and the bucket starts of
						 * the chunk, go into L2 now; one (source, group) pair
						 * per lane. The chunk bounds are loaded before the
						 * delay-1 push, so that the two loads' latencies
						 * overlap */
						const uint32_t G = net.groups;
						const uint32_t pairs = uint32_t(__popc(word)) * G;
						uint32_t c0 = 0u, c1 = 0u;
						size_t k0 = 0;
						uint32_t bg = 0u;
						if(lane < pairs) {
							const uint32_t f = lane / G, g = lane - f * G;
							const uint32_t src = dw * 32u + uint32_t(__fns(word, 0u, int(f) + 1));
							const uint32_t g0 = __ldg(&net.groupFirst[g]);
							bg = __ldg(&net.groupFirst[g + 1]) - g0;
							k0 = size_t(g0) * nDev + size_t(src) * bg;
							prefetchL2(net.segOff + k0, net.segOff + k0 + bg + 1u);
							c0 = __ldg(&net.srcChunk[size_t(src) * G + g]);
							c1 = __ldg(&net.srcChunk[size_t(src + 1u) * G + g]);
						}
						const uint32_t np = pushDelayOne(net, word, fired ? d1 : make_uint2(0u, 0u), (t + 1u) & 1u, lane);
						pushed += lane == 0 ? np : 0u;   /* warp total, counted once */
						if(lane < pairs) prefetchL2(net.fcm + c0, net.fcm + c1);
						/* more than 32 pairs (several sources firing in a
						 * warp of a network with many groups): the rest */
						for(uint32_t q = lane + 32u; q < pairs; q += 32u) {
							const uint32_t f = q / G, g = q - f * G;
							const uint32_t src = dw * 32u + uint32_t(__fns(word, 0u, int(f) + 1));
							const uint32_t g0 = __ldg(&net.groupFirst[g]);
							const uint32_t b2 = __ldg(&net.groupFirst[g + 1]) - g0;
							const size_t k2 = size_t(g0) * nDev + size_t(src) * b2;
							prefetchL2(net.segOff + k2, net.segOff + k2 + b2 + 1u);
							prefetchL2(net.fcm + __ldg(&net.srcChunk[size_t(src) * G + g]),
									net.fcm + __ldg(&net.srcChunk[size_t(src + 1u) * G + g]));
						}
					}
				}
				/* in the first phase the noise of the next cycle is drawn by
				 * the warp that just advanced the generator (later phases
				 * draw it in work units below) */
				if(k == 0 && G.kind == 0 && valid) {
					if(k + 1 < A.cycles) {
						net.noise[(par ^ 1u) * nDev + n] = drawNoise(net, G, i);
					} else if(resident) {
						drawNoiseAhead(net, G, i, n, G.rng[i], par ^ 1u);
					}
				}
				if(trace) {
					/* the warp's loads and model, its whole update, and for
					 * a warp with fired neurons the part after its lists */
					__syncwarp();
					const uint32_t w3 = uint32_t(globalTimer());
					if(lane == 0) {
						atomicAdd(&trace[9], (unsigned long long) (w1 - w0));
						atomicAdd(&trace[10], (unsigned long long) (w3 - w0));
						atomicAdd(&trace[11], 1ull);
						if(word) {
							atomicAdd(&trace[12], (unsigned long long) (w3 - w2));
							atomicAdd(&trace[13], 1ull);
						}
					}
				}
			}
			pushed = __reduce_add_sync(FULL, pushed);
			if(lane == 0 && pushed) atomicAdd(&sPushed, (unsigned long long) pushed);
			if(trace && lane == 0) atomicMax(&trace[2], globalTimer());
		}

		/* ---- overlapped with the update: the gather of cycle t-1 (the
		 * regions hold delays >= 2 only, which go into slots of cycles > t;
		 * delay 1 went to the inbox when the sources fired) and the STDP accumulation of cycle t-1, as units
		 * handed out by a block counter so that warps without neurons to
		 * update start at once. Units [0, G): 32 fired
		 * sources each; units [G + NW, G + NW + S): this block's share of the
		 * grid's STDP entries ---- */
		if(doPrev) {
			const uint32_t par = (t - 1u) & 1u;
			const uint32_t nLists = B + (net.remoteList ? 1u : 0u);
			const uint32_t F = net.deliver ? sPreF[nLists] : 0u;
			const uint32_t G = (F + 31u) / 32u;
			/* STDP entries of cycle t-1 over all blocks; this block takes
			 * entries u * B + b */
			const uint32_t P = net.stdp ? sPreP[B] : 0u;
			const uint32_t Sb = P > b ? (P - b + B - 1u) / B : 0u;
			/* units [G, G + NW): the next cycle's noise of one owned neuron
			 * warp each (from the second phase of a launch on) */
			const uint32_t NW = (k + 1u < A.cycles || (resident && k > 0u)) ? myWarps : 0u;
			const uint32_t units = G + NW + Sb;
			const uint32_t* flist = net.firedList + par * listStride;
			const uint2* plist = net.postList + par * postParity;
			const uint64_t* rfAfter = net.rf + (t & 1u) * nDev;   /* history after update(t-1) */
			const uint32_t slotPrev = uint32_t((t64 - 1u) % net.slots);
			uint32_t pushed = 0;
			uint64_t visited = 0;
			/* Each unit's dependent loads are issued one stage ahead, so that a
			 * unit's chain starts from its last load: its first load (`lead`)
			 * when the unit before it starts, its second (`second`) once the
			 * unit before it has issued its own last loads.
			 * lead: a gather unit's fired source of each lane {s, 1} ({0, 0}
			 * past the end), an STDP unit's entry {first, count}.
			 * second: a gather unit's bucket {first record, end} of each lane,
			 * an STDP unit's source words. */
			auto lead = [&](uint32_t u) -> uint2 {
				uint2 v = make_uint2(0u, 0u);
				if(u < G) {
					const uint32_t j = u * 32u + lane;
					if(j < F) {
						const uint32_t bb = findList(sPreF, nLists, j);
						v.x = bb < B ? flist[size_t(bb) * ownN + (j - sPreF[bb])]
							: net.remoteList[size_t(par) * nDev + (j - sPreF[B])];
						v.y = 1u;
					}
				} else if(u >= G + NW && u < units) {
					const uint32_t it = (u - G - NW) * B + b;
					const uint32_t bb = findList(sPreP, B, it);
					v = plist[size_t(bb) * net.postStride + (it - sPreP[bb])];
				}
				return v;
			};
			auto second = [&](uint32_t u, uint2 h, uint2& row, uint32_t* sd) {
				if(u < G) {
					row = make_uint2(0u, 0u);
					if(h.y) {
						const uint32_t* r = net.segOff + segKey0 + size_t(h.x) * segStride;
						row = make_uint2(r[0], r[1]);
					}
				} else if(u >= G + NW && u < units) {
#pragma unroll
					for(int x = 0; x < int(STDP_PER_LANE); ++x) {
						const uint32_t jj = lane + 32u * x;
						sd[x] = jj < h.y ? __ldcs(&net.rcmSrcDelay[h.x + jj]) : 0u;
					}
				}
			};
			uint32_t u = 0;
			if(lane == 0) u = atomicAdd(&sWork, 1u);
			u = __shfl_sync(FULL, u, 0);
			uint2 head = lead(u);
			uint2 row = make_uint2(0u, 0u);
			uint32_t sd[STDP_PER_LANE];
			second(u, head, row, sd);
			while(u < units) {
				uint32_t un = 0;
				if(lane == 0) un = atomicAdd(&sWork, 1u);
				un = __shfl_sync(FULL, un, 0);
				if(trace && lane == 0 && un < units) atomicMax(&trace[16], globalTimer());
				const uint2 headNext = lead(un);
				uint2 rowNext = make_uint2(0u, 0u);
				uint32_t sdNext[STDP_PER_LANE];
				const unsigned long long u0 = trace ? globalTimer() : 0ull;
				if(u < G) {
					/* 32 fired sources, one per lane; their segments of this
					 * block's region are worked off as one concatenation so
					 * that a warp's loads fall on few lines */
					const uint32_t beg = row.x, cnt = row.y - row.x;
					uint32_t incl = cnt;
#pragma unroll
					for(int d = 1; d < 32; d <<= 1) {
						const uint32_t x = __shfl_up_sync(FULL, incl, d);
						if(lane >= uint32_t(d)) incl += x;
					}
					const uint32_t total = __shfl_sync(FULL, incl, 31);
					const uint32_t excl = incl - cnt;
					pushed += lane == 0 ? total : 0u;
					bool issued = false;   /* the next unit's second loads */
					for(uint32_t base = 0; base < total; base += 32u * GATHER_PER_LANE) {
						uint2 r[GATHER_PER_LANE];
#pragma unroll
						for(int x = 0; x < GATHER_PER_LANE; ++x) {
							const uint32_t idx = base + uint32_t(x) * 32u + lane;
							/* the lane whose range holds idx: the last with excl <= idx */
							uint32_t lo = 0;
#pragma unroll
							for(uint32_t step = 16; step; step >>= 1) {
								const uint32_t e = __shfl_sync(FULL, excl, lo + step);
								if(e <= idx) lo += step;
							}
							const uint32_t eL = __shfl_sync(FULL, excl, lo);
							const uint32_t bL = __shfl_sync(FULL, beg, lo);
							r[x] = idx < total ? __ldcs(&net.fcm[bL + (idx - eL)]) : make_uint2(0u, 0u);
						}
						if(!issued) {
							second(un, headNext, rowNext, sdNext);
							issued = true;
						}
#pragma unroll
						for(int x = 0; x < GATHER_PER_LANE; ++x) {
							if(base + uint32_t(x) * 32u + lane < total) {
								uint32_t slot = slotPrev + (r[x].x & 63u) + 1u;
								slot = slot >= net.slots ? slot - net.slots : slot;
								gatherAdd<SMEM>(net, sAcc, ownN, ownBase, slot, r[x]);
							}
						}
					}
					if(!issued) second(un, headNext, rowNext, sdNext);
				} else if(u < G + NW) {
					second(un, headNext, rowNext, sdNext);
					const uint32_t lw = u - G;
					const uint32_t dw = firstWarp + lw;
					int gi = 0;
					while(dw >= A.groupWarp[gi + 1]) ++gi;
					const GroupDev& Gr = A.groups[gi];
					const uint32_t n = dw * 32u + lane;
					const uint32_t i = n - Gr.devBase;
					if(Gr.kind == 0 && i < Gr.count) {
						if(resident) {
							/* from the state this cycle's update advances the
							 * generator to */
							drawNoiseAhead(net, Gr, i, n, net.rngAhead[size_t(t & 1u) * nDev + n], (t + 1u) & 1u);
						} else {
							net.noise[((t + 1u) & 1u) * nDev + n] = drawNoise(net, Gr, i);
						}
					}
				} else {
					/* STDP (ConnectivityMatrix.cpp:224-258): a run of the
					 * plastic synapses of a target that fired P cycles before
					 * cycle t-1; every accumulator has one writer in a phase
					 * (a plain load and store: a reduction into L2 measured
					 * slower). The source words came with the unit before;
					 * the accumulators and the sources' histories are loaded
					 * together */
					const uint32_t b0 = head.x;
					const uint32_t cnt = head.y;
					visited += cnt;
					int32_t old[STDP_PER_LANE];
					uint64_t pre[STDP_PER_LANE];
#pragma unroll
					for(int x = 0; x < int(STDP_PER_LANE); ++x) {
						const uint32_t jj = lane + 32u * x;
						old[x] = jj < cnt ? __ldcs(&net.rcmAcc[b0 + jj]) : 0;
						pre[x] = jj < cnt ? rfAfter[sd[x] >> 6] : 0ull;
					}
					second(un, headNext, rowNext, sdNext);
#pragma unroll
					for(int x = 0; x < int(STDP_PER_LANE); ++x) {
						const uint32_t jj = lane + 32u * x;
						if(jj < cnt) {
							const int32_t dw = weightChange(shr64(pre[x], (sd[x] & 63u) + 1u), A.rule);
							if(dw != 0) {
								__stcs(&net.rcmAcc[b0 + jj], int32_t(uint32_t(old[x]) + uint32_t(dw)));
							}
						}
					}
				}
				if(trace) {
					__syncwarp();
					if(lane == 0) {
						/* gather units [5] and [7], STDP units [6] and [8],
						 * noise units [14] and [15] */
						const unsigned q = u < G ? 5u : (u < G + NW ? 14u : 6u);
						const unsigned long long u1 = globalTimer();
						atomicAdd(&trace[q], u1 - u0);
						atomicAdd(&trace[q == 14u ? 15u : q + 2u], 1ull);
						atomicMax(&trace[19], u1);
					}
				}
				u = un;
				head = headNext;
				row = rowNext;
#pragma unroll
				for(int x = 0; x < int(STDP_PER_LANE); ++x) sd[x] = sdNext[x];
			}
			if(trace && lane == 0) {
				atomicAdd(&trace[17], globalTimer() - trace[0]);
				atomicAdd(&trace[18], 1ull);
			}
			pushed = __reduce_add_sync(FULL, pushed);
			if(lane == 0) {
				if(pushed) atomicAdd(&sPushed, (unsigned long long) pushed);
				if(visited) atomicAdd(&sVisits, (unsigned long long) visited);
			}
		}
		__syncthreads();
		if(tid == 0) {
			if(doUpdate) {
				const uint32_t par = t & 1u;
				net.firedCnt[par * B + b] = sNFired;
				net.postCnt[par * B + b] = sNPost;
				if(sNFired) {
					atomicAdd(&net.firedCountRing[t & net.ringMask], sNFired);
					atomicAdd(&net.eventsRing[t & net.ringMask], sEvents);
					atomicAdd(&net.stats[2], (unsigned long long) sNFired);
					atomicAdd(&net.stats[3], sEvents);
				}
			}
			if(sPushed) atomicAdd(&net.stats[0], sPushed);
			if(sVisits) atomicAdd(&net.stats[1], sVisits);
		}
		if(trace && tid == 0) trace[3] = globalTimer();
		if(HOST && A.hostWords && doUpdate) {
			/* the step's list, by the block whose update arrives last */
			if(tid == 0) {
				__threadfence();
				sLast = atomicAdd(&net.barrier[3], 1u) == B - 1u;
				if(sLast) {
					/* every block has arrived: the count starts again for
					 * the next step, which the host starts after this one's
					 * list */
					*(volatile unsigned*) &net.barrier[3] = 0u;
					__threadfence();
				}
			}
			__syncthreads();
			if(sLast) {
				writeStepList(net, A.hostWords, t, warp, lane);
				if(resident && tid == 0) {
					__threadfence_system();
					*(volatile uint32_t*) &A.doneWords[0] = A.firstSeq + k;
				}
			}
		}
		if(resident) {
			/* block 0 waits for the next command and hands it to every
			 * block */
			const uint32_t seqK = A.firstSeq + k;
			if(b == 0) {
				residentNext(A, seqK, k, warp, lane);
			} else if(!residentWait(A, seqK, k)) {
				if(HOST && A.hostWords && tid == 0) A.hostWords[0] = 1u;
				return;
			}
			if(*(volatile const uint32_t*) &A.bcast[(k + 1u) & 1u].op != RESIDENT_STEP) break;
		} else if(k < barriers) {
			if(!gridSync(net.barrier, barBase + (k + 1u) * B, A.timeoutNs)) {
				if(HOST && A.hostWords && tid == 0) A.hostWords[0] = 1u;
				return;
			}
			passed++;
		}
		if(trace && tid == 0) trace[4] = globalTimer();
	}

	/* the delay-1 arrivals for the cycle after the launch go into its slot,
	 * so that between launches every spike fired is in the current slots
	 * (a launch that leaves its last cycle pending leaves them in the inbox,
	 * which every reader of the cycle's currents adds: the update, the
	 * plugin current export and applyStdp's arrival-slot correction) */
	if(!lastPending) {
		__syncthreads();
		const uint64_t tEnd = first + A.cycles;
		const uint32_t slotEnd = uint32_t(tEnd % net.slots);
		for(uint32_t l = tid; l < myN; l += blockDim.x) {
			const uint32_t n = ownBase + l;
			long long e, in;
			takeInbox(net, uint32_t(tEnd) & 1u, n, e, in);
			if(e | in) {
				if(SMEM) {
					int2* cell = &sAcc[slotEnd * ownN + l];
					*cell = make_int2(cell->x + int(e), cell->y + int(in));
				} else {
					addSlot(net, slotEnd, n, e, in);
				}
			}
		}
	}
	if(SMEM) {
		__syncthreads();
		const uint32_t total = net.slots * ownN;
		for(uint32_t x = tid; x < total; x += blockDim.x) {
			const uint32_t s = x / ownN, l = x - s * ownN;
			const size_t n = size_t(ownBase) + l;
			if(l < myN) acc32[size_t(s) * nDev + n] = sAcc[x];
		}
	}
	if(b == 0 && tid == 0) {
		if(A.cycleCounter) *A.cycleCounter = first + A.cycles;
		/* every block has read barBase: they all arrived at this launch's
		 * barriers, which block 0 has passed (a launch without barriers
		 * leaves the count as it found it) */
		if(passed) *(volatile unsigned*) &net.barrier[1] = barBase + passed * B;
		if(resident) {
			/* the commands up to firstSeq + k ran; the host waits for the
			 * stream before anything else */
			__threadfence_system();
			*(volatile uint32_t*) A.exitInfo = ((A.firstSeq + k) << 1) | 1u;
		}
	}
}

/* The currents of one cycle of a plugin model's neurons: slot plus inbox,
 * summed as the update sums them, saturated and converted (wfxToFloat). */
__global__ void
k_export_currents(NetDev net, uint32_t devBase, uint32_t count, uint32_t slot, uint32_t par, float* E, float* I)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= count) return;
	const size_t n = size_t(devBase) + i;
	long long e, in;
	if(net.acc32) {
		const int2 a = reinterpret_cast<const int2*>(net.acc)[size_t(slot) * net.nDev + n];
		const int2 b = reinterpret_cast<const int2*>(net.inbox)[size_t(par) * net.nDev + n];
		e = (long long) b.x + a.x;
		in = (long long) b.y + a.y;
	} else {
		const longlong2 a = reinterpret_cast<const longlong2*>(net.acc)[size_t(slot) * net.nDev + n];
		const longlong2 b = reinterpret_cast<const longlong2*>(net.inbox)[size_t(par) * net.nDev + n];
		e = b.x + a.x;
		in = b.y + a.y;
	}
	E[i] = wfxToFloat(e, net.fbits);
	I[i] = wfxToFloat(in, net.fbits);
}

/* Firing and current stimulus of this cycle (src/nemo/cpu/Simulation.cpp:
 * 140-163): set fstim bits, write external currents (last write wins; the
 * host removes duplicates). */
__global__ void
k_stimulus(NetDev net, StimDev s)
{
	uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i < s.nf) {
		uint32_t n = s.fstim[i];
		atomicOr(&net.fstim[n >> 5], 1u << (n & 31u));
	}
	if(i < s.ni) {
		net.ext[s.inidx[i]] = s.icur[i];
	}
}

/* Stimulus of the allocation-free step, read from the per-device scratch
 * below: [0, nf) firing-stimulus device indices, [NOALLOC_STIM_MAX,
 * +ni) current-stimulus device indices, [2 NOALLOC_STIM_MAX, +ni) their
 * currents (float bits). The firing stimulus is one entry per thread of the
 * grid (bit sets commute). The current stimulus is walked in order by the
 * first warp of block 0, 32 entries at a time; of equal indices within a
 * group the highest lane writes, and __syncwarp orders the groups, so the
 * last entry for a neuron wins as in the reference (cpu/Simulation.cpp:
 * 140-163). */
__global__ void
k_stimulus_scratch(NetDev net, const uint32_t* scratch, uint32_t nf, uint32_t ni)
{
	const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
	if(g < nf) {
		const uint32_t n = scratch[g];
		atomicOr(&net.fstim[n >> 5], 1u << (n & 31u));
	}
	if(blockIdx.x != 0 || threadIdx.x >= 32u) return;
	const uint32_t lane = threadIdx.x;
	const uint32_t* idx = scratch + NOALLOC_STIM_MAX;
	const float* cur = reinterpret_cast<const float*>(scratch + 2 * NOALLOC_STIM_MAX);
	for(uint32_t base = 0; base < ni; base += 32) {
		const uint32_t i = base + lane;
		const bool valid = i < ni;
		const uint32_t n = valid ? idx[i] : 0xffffffffu;
		const uint32_t same = __match_any_sync(FULL, n);
		if(valid && 31u - uint32_t(__clz(same)) == lane) {
			net.ext[n] = cur[i];
		}
		__syncwarp();
	}
}

/* applyStdp (src/nemo/ConnectivityMatrix.cpp:272-325): every plastic synapse
 * gets w = clamp(w + (reward * acc) >> f) and its accumulator cleared.
 *
 * The reference reads a synapse's weight when the spike arrives
 * (deliverSpikes at cycle t0 + d), whereas the step kernel adds it one cycle
 * after the source fires. For a spike still in flight when its synapse's
 * weight changes, the arrival slot therefore holds the old weight; it is
 * corrected here by w_new - w_old, into the same E/I half (the sign of a
 * weight never changes, and a weight that reaches 0 contributes 0 to E). The
 * in-flight spikes of a synapse with delay d are the set bits 0..d-1 of its
 * source's firing history after the last completed cycle (cycleNow - 1):
 * bit k fired at cycleNow-1-k and arrives at cycleNow-1-k+d. */
__device__ __forceinline__ void applyOne(const NetDev& net, const StdpRule& rule, int32_t reward, uint64_t cycleNow,
		const uint64_t* rfNow, uint32_t j, uint32_t f, int32_t acc, int32_t wOld, uint32_t target, uint32_t sd)
{
	const int32_t diff = int32_t((int64_t(reward) * int64_t(acc)) >> net.fbits);
	const int32_t wNew = updatedWeight(wOld, diff, rule);
	if(wNew != wOld) {
		net.fcm[f].y = uint32_t(wNew);
		__stcs(&net.rcmWeight[j], wNew);
		if(net.deliver) {
			const uint32_t d = (sd & 63u) + 1u;
			uint64_t pending = rfNow[sd >> 6] & ((uint64_t(1) << d) - 1u);
			if(pending) {
				const long long delta = (long long) wNew - (long long) wOld;
				const int half = wOld >= 0 ? 0 : 1;
				while(pending) {
					const uint32_t k = uint32_t(__ffsll((long long) pending) - 1);
					pending &= pending - 1;
					/* fired at cycleNow-1-k >= 0, arrives at cycleNow-1-k+d */
					const uint32_t slot = uint32_t((cycleNow - 1u - k + d) % net.slots);
					addCurrent(net, slot, target, half, delta);
				}
			}
		}
	}
	if(acc) {
		__stcs(&net.rcmAcc[j], 0);
	}
}

/* Items (target, chunk of 32 x APPLY_PER_LANE of its plastic synapses) of
 * the targets [t0, t1) over a grid-stride loop. The host launches one such
 * kernel per group of consecutive owner blocks whose forward regions together
 * fit comfortably in L2 (APPLY_GROUP_SYNAPSES): a target's plastic synapses
 * all lie in its owner's region (or the delay-1 part), so every forward
 * record a launch rewrites is loaded from DRAM once and reused from L2 by the
 * other targets that share its sector.
 *
 * skipZero: every plastic weight lies within its bounds, so a synapse whose
 * accumulator is 0 keeps its weight (updatedWeight only clamps) and its
 * accumulator: its forward index and record are not loaded. Without it (the
 * first apply of weights set out of bounds) every synapse is clamped, as in
 * ConnectivityMatrix.cpp:295-318. */
__global__ void __launch_bounds__(256)
k_apply_stdp(NetDev net, StdpRule rule, int32_t reward, uint64_t cycleNow, uint32_t t0, uint32_t t1, int skipZero)
{
	const uint64_t* rfNow = net.rf + size_t(cycleNow & 1u) * net.nDev;
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
	const uint32_t chunks = net.applyChunks;
	const uint64_t items = uint64_t(t1 - t0) * chunks;
	for(uint64_t it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < items; it += nwarps) {
		const uint32_t t = t0 + uint32_t(it / chunks);
		const uint32_t c = uint32_t(it % chunks);
		const uint32_t b0 = net.rcmStart[t] + c * (32u * APPLY_PER_LANE);
		const uint32_t e = net.rcmStart[t + 1];
		if(b0 >= e) continue;
		const uint32_t j = b0 + lane;
		/* the accumulators first; a synapse that changes (live) then loads
		 * its forward index, its weight (the reverse-order copy) and its
		 * source word together, all coalesced: no forward record is read */
		int32_t a[APPLY_PER_LANE];
		bool live[APPLY_PER_LANE];
#pragma unroll
		for(int u = 0; u < int(APPLY_PER_LANE); ++u) {
			const uint32_t jj = j + 32u * u;
			a[u] = jj < e ? __ldcs(&net.rcmAcc[jj]) : 0;
			live[u] = jj < e && (a[u] != 0 || !skipZero);
		}
		uint32_t f[APPLY_PER_LANE];
		int32_t w[APPLY_PER_LANE];
		uint32_t sd[APPLY_PER_LANE];
#pragma unroll
		for(int u = 0; u < int(APPLY_PER_LANE); ++u) {
			const uint32_t jj = j + 32u * u;
			f[u] = live[u] ? __ldcs(&net.rcmForward[jj]) : 0u;
			w[u] = live[u] ? __ldcs(&net.rcmWeight[jj]) : 0;
			sd[u] = live[u] && net.deliver ? __ldcs(&net.rcmSrcDelay[jj]) : 0u;
		}
#pragma unroll
		for(int u = 0; u < int(APPLY_PER_LANE); ++u) {
			if(live[u]) applyOne(net, rule, reward, cycleNow, rfNow, j + 32u * u, f[u], a[u], w[u], t, sd[u]);
		}
	}
}

__global__ void
k_nrand_probe(const uint32_t* u1, const uint32_t* u2, float* out, size_t n, const uint32_t* sinTab, const uint32_t* logTab)
{
	size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
	if(i < n) {
		out[i] = nrandWords(u1[i], u2[i], sinTab, logTab);
	}
}

/* The device sinf/logf of every reachable noise input (for the exhaustive
 * comparison with host glibc) */
__global__ void
k_libm_eval(float* sinOut, float* logOut, const uint32_t* sinTab, const uint32_t* logTab)
{
	using namespace libm;
	uint32_t stride = gridDim.x * blockDim.x;
	for(uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < TABLE_ENTRIES; idx += stride) {
		float fu = libm_value(idx);
		sinOut[idx] = apply_code(sin_candidate(sin_argument(fu)), table_code(sinTab, idx));
		logOut[idx] = apply_code(log_candidate(log_argument(fu)), table_code(logTab, idx));
	}
}

/* the device expf of the floats with bits [first, first + n) (diagnostics) */
__global__ void
k_exp_eval(uint32_t first, uint32_t n, float* out, NetDev net)
{
	const uint32_t stride = gridDim.x * blockDim.x;
	for(uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
		out[k] = expfMatch(net, libm::u2f(first + k));
	}
}

/* A sharded simulation: the firing of cycle t of the neurons other shards
 * own (allWords holds every device warp's word; this shard's own warps
 * [ownLo, ownHi) are skipped) enters this shard as its own update would have
 * entered it: the history shift, the fired-ring word, the delay-1 pushes
 * into the inbox of cycle t + 1, the list of remote fired sources that the
 * next launch gathers from (its count zeroed before the launch), and the
 * synaptic events they generate here. One warp per device warp. */
__global__ void
k_shard_inject(NetDev net, uint64_t t64, const uint32_t* allWords, uint32_t ownLo, uint32_t ownHi)
{
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t firstW = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const uint32_t strideW = (gridDim.x * blockDim.x) >> 5;
	const uint32_t t = uint32_t(t64);
	const uint32_t par = t & 1u;
	const size_t nDev = net.nDev;
	const uint64_t* rfIn = net.rf + par * nDev;
	uint64_t* rfOut = net.rf + (par ^ 1u) * nDev;
	unsigned long long events = 0;
	unsigned long long pushed = 0;
	for(uint32_t w = firstW; w < net.nWords; w += strideW) {
		if(w >= ownLo && w < ownHi) continue;
		const uint32_t word = allWords[w];
		const uint32_t n = w * 32u + lane;
		const bool fired = (word >> lane) & 1u;
		const uint64_t rfNew = (rfIn[n] << 1) | uint64_t(fired);
		rfOut[n] = rfNew;
		if(lane == 0) net.firedRing[size_t(t & net.ringMask) * net.nWords + w] = word;
		if(word) {
			uint32_t base = 0;
			if(lane == 0) base = atomicAdd(&net.remoteCnt[par], uint32_t(__popc(word)));
			base = __shfl_sync(FULL, base, 0);
			if(fired) net.remoteList[size_t(par) * nDev + base + __popc(word & ((1u << lane) - 1u))] = n;
			events += __reduce_add_sync(FULL, fired ? __ldg(&net.outDegree[n]) : 0u);
			if(net.deliver) {
				const uint2 d1 = fired ? make_uint2(__ldg(&net.d1Start[n]), __ldg(&net.d1Start[n + 1]))
					: make_uint2(0u, 0u);
				pushed += pushDelayOne(net, word, d1, (t + 1u) & 1u, lane);
			}
		}
	}
	if(lane == 0) {
		if(events) atomicAdd(&net.stats[3], events);
		if(pushed) atomicAdd(&net.stats[0], pushed);
	}
}

/* net.srcChunk from net.segOff: entry s * groups + g is the bucket start of
 * (source s, the first block of group g), the start of source s's chunk in
 * the group; s = nDev gives the group's end */
__global__ void
k_source_chunks(NetDev net, uint32_t* out)
{
	const size_t G = net.groups;
	const size_t total = (size_t(net.nDev) + 1) * G;
	for(size_t x = blockIdx.x * size_t(blockDim.x) + threadIdx.x; x < total; x += size_t(gridDim.x) * blockDim.x) {
		const size_t src = x / G;
		const uint32_t g = uint32_t(x - src * G);
		const uint32_t g0 = net.groupFirst[g], bg = net.groupFirst[g + 1] - g0;
		out[x] = net.segOff[size_t(g0) * net.nDev + src * bg];
	}
}

/* hhDivConst against __fdiv_rn, divisors 20, 80 and 18, on every float with
 * magnitude at least 2^-100 (infinities included) and on both zeros */
__global__ void
k_hh_div_check(unsigned long long* bad)
{
	const float ds[3] = {20.0f, 80.0f, 18.0f};
	unsigned long long nb[3] = {0, 0, 0};
	const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for(uint64_t u = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; u < (uint64_t(1) << 32); u += stride) {
		const float a = libm::u2f(uint32_t(u));
		if(!(fabsf(a) >= 0x1p-100f) && a != 0.0f) continue;   /* NaN and tiny magnitudes */
#pragma unroll
		for(int q = 0; q < 3; ++q) {
			const float y = __fdiv_rn(1.0f, ds[q]);
			if(libm::f2u(hhDivConst(a, ds[q], y)) != libm::f2u(__fdiv_rn(a, ds[q]))) nb[q]++;
		}
	}
	for(int q = 0; q < 3; ++q) {
		if(nb[q]) atomicAdd(&bad[q], nb[q]);
	}
}

int g_smCount = 0;

} // namespace

/* Scratch of the allocation-free step (one copy per device, module-static so
 * that no call allocates): 3 x NOALLOC_STIM_MAX words = 192 KB. Nothing in it
 * has to start at zero: every call writes the entries it then reads. */
static __device__ __align__(256) uint32_t g_noallocStim[3 * NOALLOC_STIM_MAX];

namespace {
std::mutex g_noallocMutex;
uint32_t* g_noallocPtr[NOALLOC_MAX_DEVICES] = {};
}

int
noallocScratch(int device, uint32_t** ptr)
{
	if(device < 0 || device >= NOALLOC_MAX_DEVICES) {
		return int(cudaErrorInvalidDevice);
	}
	std::lock_guard<std::mutex> lock(g_noallocMutex);
	if(g_noallocPtr[device] == nullptr) {
		void* p = nullptr;
		cudaError_t e = cudaGetSymbolAddress(&p, g_noallocStim);
		if(e != cudaSuccess) {
			return int(e);
		}
		g_noallocPtr[device] = static_cast<uint32_t*>(p);
	}
	*ptr = g_noallocPtr[device];
	return int(cudaSuccess);
}

int
smCount()
{
	if(g_smCount == 0) {
		int dev = 0;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&g_smCount, cudaDevAttrMultiProcessorCount, dev);
		if(g_smCount <= 0) g_smCount = 148;
	}
	return g_smCount;
}

static inline cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }

void
launchStimulus(const NetDev& net, const StimDev& stim, void* stream)
{
	uint32_t n = stim.nf > stim.ni ? stim.nf : stim.ni;
	if(n == 0) return;
	k_stimulus<<<(n + 255) / 256, 256, 0, S(stream)>>>(net, stim);
}

void
launchStimulusScratch(const NetDev& net, const uint32_t* scratch, uint32_t nf, uint32_t ni, void* stream)
{
	if(nf + ni == 0) return;
	const uint32_t blocks = std::max<uint32_t>(1u, (nf + 255u) / 256u);
	k_stimulus_scratch<<<blocks, 256, 0, S(stream)>>>(net, scratch, nf, ni);
}

/* The step kernel's plan: one 1024-thread block per SM (its registers allow
 * no more) and no block without neurons; the neuron warps split into
 * contiguous ranges of about equal summed update cost (block b starts at the
 * first warp whose cost prefix reaches b / B of the total); the owned
 * current slots go to shared memory when they are int32 and fit. */
void
cyclesPlan(const std::vector<uint32_t>& warpCost, uint32_t slots, bool acc32, uint32_t* blocks,
		std::vector<uint32_t>* ownStart, uint32_t* ownWarps, bool* smemAcc)
{
	const uint32_t totalWarps = uint32_t(warpCost.size());
	uint32_t B = uint32_t(smCount());
	if(B > MAX_BLOCKS) B = MAX_BLOCKS;
	/* no block without neurons (a small network's extra blocks would only
	 * wait at the grid barrier) */
	if(B > totalWarps) B = totalWarps > 0 ? totalWarps : 1u;
	std::vector<uint64_t> prefix(size_t(totalWarps) + 1, 0);
	for(uint32_t w = 0; w < totalWarps; ++w) prefix[w + 1] = prefix[w] + warpCost[w];
	ownStart->assign(size_t(B) + 1, totalWarps);
	uint32_t most = 0;
	for(uint32_t b = 0; b < B; ++b) {
		const uint64_t target = prefix[totalWarps] * b / B;
		(*ownStart)[b] = uint32_t(std::lower_bound(prefix.begin(), prefix.end(), target) - prefix.begin());
		if((*ownStart)[b] > totalWarps) (*ownStart)[b] = totalWarps;
	}
	(*ownStart)[0] = 0;
	for(uint32_t b = 0; b < B; ++b) most = std::max(most, (*ownStart)[b + 1] - (*ownStart)[b]);
	const uint64_t bytes = uint64_t(slots) * most * 32u * 8u;
	const bool smem = acc32 && bytes <= SMEM_ACC_LIMIT;
	/* the attribute is per device and shared by all simulations: set it to
	 * the largest size any of them uses */
	cudaFuncSetAttribute(k_cycles<true, 1024, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM_ACC_LIMIT));
	cudaFuncSetAttribute(k_cycles<true, 512, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM_ACC_LIMIT));
	cudaFuncSetAttribute(k_cycles<true, 256, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM_ACC_LIMIT));
	cudaFuncSetAttribute(k_cycles<true, 1024, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM_ACC_LIMIT));
	cudaFuncSetAttribute(k_cycles<true, 512, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM_ACC_LIMIT));
	cudaFuncSetAttribute(k_cycles<true, 256, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM_ACC_LIMIT));
	int perSm = 0, perSmHost = 0;
	if(smem) {
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_cycles<true, 1024, false>, 1024, size_t(bytes));
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSmHost, k_cycles<true, 1024, true>, 1024, size_t(bytes));
	} else {
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_cycles<false, 1024, false>, 1024, 0);
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSmHost, k_cycles<false, 1024, true>, 1024, 0);
	}
	perSm = std::min(perSm, perSmHost);
	*blocks = perSm >= 1 ? B : 0u;
	*ownWarps = most;
	*smemAcc = smem;
}

template<bool SMEM, bool HOST>
static cudaError_t
launchCyclesH(const CycleArgs& args, void** params, size_t bytes, cudaStream_t stream)
{
	const NetDev& net = args.net;
	if(args.cycles <= 1u && (args.carry & 2u) && args.cmd == nullptr) {
		/* one update phase and no grid barrier: the blocks never wait for one
		 * another, so they need not be co-resident */
		switch(net.threads) {
			case 256:
				return cudaLaunchKernel((const void*) k_cycles<SMEM, 256, HOST>, dim3(net.blocks), dim3(256), params,
						bytes, stream);
			case 512:
				return cudaLaunchKernel((const void*) k_cycles<SMEM, 512, HOST>, dim3(net.blocks), dim3(512), params,
						bytes, stream);
			default:
				return cudaLaunchKernel((const void*) k_cycles<SMEM, 1024, HOST>, dim3(net.blocks), dim3(1024), params,
						bytes, stream);
		}
	}
	switch(net.threads) {
		case 256:
			return cudaLaunchCooperativeKernel((const void*) k_cycles<SMEM, 256, HOST>, dim3(net.blocks), dim3(256),
					params, bytes, stream);
		case 512:
			return cudaLaunchCooperativeKernel((const void*) k_cycles<SMEM, 512, HOST>, dim3(net.blocks), dim3(512),
					params, bytes, stream);
		default:
			return cudaLaunchCooperativeKernel((const void*) k_cycles<SMEM, 1024, HOST>, dim3(net.blocks), dim3(1024),
					params, bytes, stream);
	}
}

template<bool SMEM>
static cudaError_t
launchCyclesT(const CycleArgs& args, void** params, size_t bytes, cudaStream_t stream)
{
	if(args.hostWords || args.cmd) return launchCyclesH<SMEM, true>(args, params, bytes, stream);
	return launchCyclesH<SMEM, false>(args, params, bytes, stream);
}

void
launchCycles(const CycleArgs& args, void* stream)
{
	void* params[] = {const_cast<CycleArgs*>(&args)};
	const NetDev& net = args.net;
	if(net.smemAcc && !args.globalAcc) {
		const size_t bytes = size_t(net.slots) * net.ownWarps * 32u * 8u;
		launchCyclesT<true>(args, params, bytes, S(stream));
	} else {
		launchCyclesT<false>(args, params, 0, S(stream));
	}
}

/* resident 256-thread blocks of k_apply_stdp per SM (one wave of the grid) */
static uint32_t
applyBlocksPerSm()
{
	static int perSm = 0;
	if(perSm == 0) {
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_apply_stdp, 256, 0);
		if(perSm <= 0) perSm = 1;
	}
	return uint32_t(perSm);
}

void
launchApplyStdp(const NetDev& net, const StdpRule& rule, int32_t reward, uint64_t cycleNow,
		const uint32_t* groupTargets, uint32_t groups, bool skipZero, void* stream)
{
	for(uint32_t g = 0; g < groups; ++g) {
		const uint32_t t0 = groupTargets[g], t1 = groupTargets[g + 1];
		if(t1 <= t0) continue;
		/* one item (32 x APPLY_PER_LANE synapses) per warp at a time */
		const uint64_t items = uint64_t(t1 - t0) * net.applyChunks;
		uint64_t blocks = (items * 32 + 255) / 256;
		const uint64_t cap = uint64_t(smCount()) * applyBlocksPerSm();
		if(blocks > cap) blocks = cap;
		k_apply_stdp<<<uint32_t(blocks), 256, 0, S(stream)>>>(net, rule, reward, cycleNow, t0, t1, skipZero ? 1 : 0);
	}
}

void
launchNrandProbe(const uint32_t* u1, const uint32_t* u2, float* out, size_t n,
		const uint32_t* sinTab, const uint32_t* logTab, void* stream)
{
	if(n == 0) return;
	k_nrand_probe<<<uint32_t((n + 255) / 256), 256, 0, S(stream)>>>(u1, u2, out, n, sinTab, logTab);
}

void
launchExpEval(uint32_t first, uint32_t n, float* out, const NetDev& net, void* stream)
{
	if(n == 0) return;
	k_exp_eval<<<smCount() * 8, 256, 0, S(stream)>>>(first, n, out, net);
}

void
launchSourceChunks(const NetDev& net, uint32_t* srcChunk, void* stream)
{
	const size_t total = (size_t(net.nDev) + 1) * net.groups;
	const uint32_t blocks = uint32_t(std::min<size_t>((total + 255) / 256, size_t(smCount()) * 16));
	k_source_chunks<<<std::max<uint32_t>(blocks, 1u), 256, 0, S(stream)>>>(net, srcChunk);
}

void
launchShardInject(const NetDev& net, uint64_t t, const uint32_t* allWords, uint32_t ownLo, uint32_t ownHi,
		void* stream)
{
	const uint32_t warps = net.nWords;
	const uint32_t blocks = std::max<uint32_t>(1u, std::min<uint32_t>((warps + 7u) / 8u, uint32_t(smCount()) * 8u));
	k_shard_inject<<<blocks, 256, 0, S(stream)>>>(net, t, allWords, ownLo, ownHi);
}

void
launchExportCurrents(const NetDev& net, uint32_t devBase, uint32_t count, uint64_t cycle, float* E, float* I,
		void* stream)
{
	if(count == 0) return;
	k_export_currents<<<(count + 255) / 256, 256, 0, S(stream)>>>(net, devBase, count,
			uint32_t(cycle % net.slots), uint32_t(cycle) & 1u, E, I);
}

void
launchHhDivCheck(unsigned long long* bad, void* stream)
{
	k_hh_div_check<<<smCount() * 8, 256, 0, S(stream)>>>(bad);
}

void
launchLibmEval(float* sinOut, float* logOut, const uint32_t* sinTab, const uint32_t* logTab, void* stream)
{
	k_libm_eval<<<smCount() * 8, 256, 0, S(stream)>>>(sinOut, logOut, sinTab, logTab);
}

} // namespace nemo_b200
