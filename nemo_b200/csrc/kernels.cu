/* sm_100a kernels of the per-cycle step path (interface: kernels.hpp).
 *
 * Compiled with -fmad=false; in addition every floating-point operation whose
 * rounding is observable goes through an explicit round-to-nearest intrinsic
 * (__fadd_rn, __dmul_rn, ...) so that neither contraction nor reassociation can
 * change the operation order of the reference CPU plugins
 * (src/nemo/cpu/plugins/*.cpp). Integer current accumulation is exact and
 * order-independent, which is what makes atomics bit-exact here. */

#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.hpp"
#include "libm_match.cuh"

namespace nemo_b200 {

namespace {

const unsigned FULL = 0xffffffffu;

/* 64-bit shifts by a count that may reach 64, evaluated like the x86-64
 * shift the reference runs on (count modulo 64). */
__device__ __forceinline__ uint64_t shl64(uint64_t x, unsigned n) { return x << (n & 63u); }
__device__ __forceinline__ uint64_t shr64(uint64_t x, unsigned n) { return x >> (n & 63u); }

__device__ __forceinline__ uint32_t cycleOf(const NetDev& net, uint32_t offset)
{
	return *net.cycleBase + offset;
}

/* wfx_toFloat: saturate the int64 sum to int32, convert, scale
 * (src/nemo/fixedpoint.cpp:40-49) */
__device__ __forceinline__ float wfxToFloat(long long v, uint32_t fbits)
{
	v = v > 2147483647LL ? 2147483647LL : v;
	v = v < -2147483648LL ? -2147483648LL : v;
	return __fdiv_rn(__ll2float_rn(v), float(1u << fbits));
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
__device__ __forceinline__ float nrand(uint4& s, const uint32_t* sinTab, const uint32_t* logTab)
{
	using namespace libm;
	float f1 = __uint2float_rn(urand(s));
	float f2 = __uint2float_rn(urand(s));
	float a = sin_argument(f1);
	float y = log_argument(f2);
	float L = apply_code(log_candidate(y), table_code(logTab, libm_index(f2)));
	float r = __fsqrt_rn(__fmul_rn(-2.0f, L));
	float S = apply_code(sin_candidate(a), table_code(sinTab, libm_index(f1)));
	return __fmul_rn(S, r);
}

/* Read and clear this cycle's E/I sums of neuron n */
__device__ __forceinline__ void takeCurrents(const NetDev& net, uint32_t n, float& E, float& I)
{
	longlong2* acc = reinterpret_cast<longlong2*>(net.acc);
	longlong2 a = acc[n];
	if(a.x | a.y) {
		acc[n] = make_longlong2(0, 0);
	}
	E = wfxToFloat(a.x, net.fbits);
	I = wfxToFloat(a.y, net.fbits);
}

__device__ __forceinline__ float takeExternal(const NetDev& net, uint32_t n)
{
	float x = net.ext[n];
	if(x != 0.0f) {
		net.ext[n] = 0.0f;
	}
	return x;
}

/* Per-warp firing-stimulus word of this warp's 32 neurons, cleared after use */
__device__ __forceinline__ uint32_t takeStimWord(const NetDev& net, uint32_t n, uint32_t lane)
{
	uint32_t w = 0;
	if(lane == 0) {
		w = net.fstim[n >> 5];
		if(w) {
			net.fstim[n >> 5] = 0;
		}
	}
	return __shfl_sync(FULL, w, 0);
}

/* Epilogue shared by all models, run by every lane of a warp that owns the
 * 32 neurons starting at n - lane:
 *  - history shift and firing bitmap of cycle t,
 *  - scatter: every fired neuron enqueues its non-empty rows (one per outgoing
 *    delay d) into spike-queue slot t+d; one atomicAdd per (warp, delay),
 *  - the STDP post-spike list (neurons whose history bit P is set),
 *  - per-cycle counters of fired neurons and synaptic events. */
__device__ __forceinline__ void fireEpilogue(const NetDev& net, uint32_t t, uint32_t n, uint32_t lane,
		bool valid, bool fired)
{
	uint64_t rf = 0;
	if(valid) {
		rf = (net.recentFiring[n] << 1) | uint64_t(fired);
		net.recentFiring[n] = rf;
	}
	uint32_t word = __ballot_sync(FULL, fired);
	uint32_t slotR = t & net.ringMask;
	if(lane == 0) {
		net.firedRing[size_t(slotR) * net.nWords + (n >> 5)] = word;
	}

	/* scatter into the delay-bucketed spike queue */
	uint64_t delays = fired ? net.delayBits[n] : 0ull;
	uint32_t anyLo = __reduce_or_sync(FULL, uint32_t(delays));
	uint32_t anyHi = __reduce_or_sync(FULL, uint32_t(delays >> 32));
	uint64_t any = (uint64_t(anyHi) << 32) | anyLo;
	const uint32_t lt = (1u << lane) - 1u;
	while(any) {
		uint32_t k = uint32_t(__ffsll((long long) any) - 1);
		any &= any - 1;
		bool has = (delays >> k) & 1ull;
		uint32_t mask = __ballot_sync(FULL, has);
		uint32_t slot = (t + k + 1) & net.qMask;
		uint32_t leader = __ffs(mask) - 1;
		uint32_t base = 0;
		if(lane == leader) {
			base = atomicAdd(&net.queueFill[slot], __popc(mask));
		}
		base = __shfl_sync(FULL, base, leader);
		if(has) {
			net.queue[size_t(slot) * net.qCap + base + __popc(mask & lt)] = n * net.rowStride + k;
		}
	}

	/* counters */
	if(word) {
		uint32_t deg = fired ? net.outDegree[n] : 0u;
		unsigned long long ev = __reduce_add_sync(FULL, deg);
		if(lane == 0) {
			atomicAdd(&net.eventsRing[slotR], ev);
			atomicAdd(&net.firedCountRing[slotR], uint32_t(__popc(word)));
			atomicAdd(&net.stats[2], (unsigned long long) __popc(word));
			atomicAdd(&net.stats[3], ev);
		}
	}

	/* STDP: targets that fired P cycles ago (src/nemo/ConnectivityMatrix.cpp:237) */
	if(net.stdp) {
		bool post = valid && ((rf >> net.postShift) & 1ull);
		uint32_t pm = __ballot_sync(FULL, post);
		if(pm) {
			uint32_t par = t & 1u;
			uint32_t leader = __ffs(pm) - 1;
			uint32_t base = 0;
			if(lane == leader) {
				base = atomicAdd(&net.postCount[par], __popc(pm));
			}
			base = __shfl_sync(FULL, base, leader);
			if(post) {
				net.postList[size_t(par) * net.nDev + base + __popc(pm & lt)] = n;
			}
		}
	}
}

/* Common prologue: cycle, warp-level bounds. Returns false for warps past
 * the group's padded range (they must not touch the next group's words). */
__device__ __forceinline__ bool groupThread(const NetDev& net, const GroupDev& g, uint32_t offset, bool resetSlot,
		uint32_t& t, uint32_t& i, uint32_t& n, uint32_t& lane, bool& valid)
{
	t = cycleOf(net, offset);
	i = blockIdx.x * blockDim.x + threadIdx.x;
	lane = threadIdx.x & 31u;
	if(resetSlot && i == 0) {
		/* slot t was drained by this cycle's gather; nothing writes it during
		 * cycle t because slots > maxDelay */
		net.queueFill[t & net.qMask] = 0;
	}
	if((i & ~31u) >= g.count) {
		return false;
	}
	n = g.devBase + i;
	valid = i < g.count;
	return true;
}

/* ---------------- neuron models ---------------- */

/* Izhikevich (src/nemo/cpu/plugins/Izhikevich.cpp:53-97). Parameters a, b, c,
 * d, sigma; state u, v. The v update evaluates its bracket in double (double
 * literals in the reference), the u update in float. */
__global__ void __launch_bounds__(256)
k_update_izhikevich(NetDev net, GroupDev g, uint32_t offset, int resetSlot)
{
	uint32_t t, i, n, lane;
	bool valid;
	if(!groupThread(net, g, offset, resetSlot, t, i, n, lane, valid)) return;
	uint32_t stim = takeStimWord(net, n, lane);
	bool fired = false;
	if(valid) {
		const size_t c = g.count;
		float E, I;
		takeCurrents(net, n, E, I);
		float In = __fadd_rn(__fadd_rn(E, I), takeExternal(net, n));
		float sigma = g.param[4 * c + i];
		if(sigma != 0.0f) {
			uint4 s = g.rng[i];
			In = __fadd_rn(In, __fmul_rn(sigma, nrand(s, net.sinTab, net.logTab)));
			g.rng[i] = s;
		}
		float a = g.param[0 * c + i];
		float b = g.param[1 * c + i];
		float u = g.state[0 * c + i];
		float v = g.state[1 * c + i];
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
		fired = fired || ((stim >> lane) & 1u);
		if(fired) {
			v = g.param[2 * c + i];
			u = __fadd_rn(u, g.param[3 * c + i]);
		}
		g.state[0 * c + i] = u;
		g.state[1 * c + i] = v;
	}
	fireEpilogue(net, t, n, lane, valid, fired);
}

/* IF_curr_exp (src/nemo/cpu/plugins/IF_curr_exp.cpp:74-121). Parameters in
 * IF_curr_exp.h order; state v, ie, ii, lastfire. Fires on v > v_thresh. */
__global__ void __launch_bounds__(256)
k_update_if_curr_exp(NetDev net, GroupDev g, uint32_t offset, int resetSlot)
{
	uint32_t t, i, n, lane;
	bool valid;
	if(!groupThread(net, g, offset, resetSlot, t, i, n, lane, valid)) return;
	uint32_t stim = takeStimWord(net, n, lane);
	bool fired = false;
	if(valid) {
		const size_t c = g.count;
		const float* P = g.param;
		float* S = g.state;
		float E, I;
		takeCurrents(net, n, E, I);
		float v_rest = P[0 * c + i], v_reset = P[1 * c + i], c_m = P[2 * c + i], tau_m = P[3 * c + i];
		float tau_refrac = P[4 * c + i], tau_e = P[5 * c + i], tau_i = P[6 * c + i];
		float v_thresh = P[7 * c + i], i_offset = P[8 * c + i];
		float ie = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, __fdiv_rn(1.0f, tau_e)), S[1 * c + i]), E);
		float ii = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, __fdiv_rn(1.0f, tau_i)), S[2 * c + i]), I);
		float In = __fadd_rn(__fadd_rn(__fadd_rn(ie, ii), takeExternal(net, n)), i_offset);
		S[1 * c + i] = ie;
		S[2 * c + i] = ii;
		float v = S[0 * c + i];
		float lastfire = S[3 * c + i];
		bool refractory = lastfire <= tau_refrac;
		if(!refractory) {
			v = __fadd_rn(v, __fadd_rn(__fdiv_rn(In, c_m), __fdiv_rn(__fsub_rn(v_rest, v), tau_m)));
		}
		fired = (!refractory && v > v_thresh) || ((stim >> lane) & 1u);
		if(fired) {
			S[3 * c + i] = 1.0f;
			S[0 * c + i] = v_reset;
		} else {
			S[3 * c + i] = __fadd_rn(lastfire, 1.0f);
			S[0 * c + i] = v;
		}
	}
	fireEpilogue(net, t, n, lane, valid, fired);
}

/* QIF (src/nemo/cpu/plugins/QIF.cpp:45-106): 10 RK4 substeps of 0.1 ms,
 * threshold 1, reset 0. */
__global__ void __launch_bounds__(256)
k_update_qif(NetDev net, GroupDev g, uint32_t offset, int resetSlot)
{
	uint32_t t, i, n, lane;
	bool valid;
	if(!groupThread(net, g, offset, resetSlot, t, i, n, lane, valid)) return;
	uint32_t stim = takeStimWord(net, n, lane);
	bool fired = false;
	if(valid) {
		const float dt = 0.1f;
		const float a1 = __fmul_rn(0.5f, dt);
		const float a2 = dt;
		const float bb1 = __fdiv_rn(dt, 6.0f);
		float E, I;
		takeCurrents(net, n, E, I);
		float X = takeExternal(net, n);
		float v = g.state[i];
		float a = g.param[i];
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
		fired = fired || ((stim >> lane) & 1u);
		if(fired) {
			v = 0.0f;
		}
		g.state[i] = v;
	}
	fireEpilogue(net, t, n, lane, valid, fired);
}

/* PoissonSource (src/nemo/cpu/plugins/PoissonSource.cpp:21-29) */
__global__ void __launch_bounds__(256)
k_update_poisson(NetDev net, GroupDev g, uint32_t offset, int resetSlot)
{
	uint32_t t, i, n, lane;
	bool valid;
	if(!groupThread(net, g, offset, resetSlot, t, i, n, lane, valid)) return;
	uint32_t stim = takeStimWord(net, n, lane);
	bool fired = false;
	if(valid) {
		float E, I;
		takeCurrents(net, n, E, I); /* currents are cleared but unused */
		(void) takeExternal(net, n);
		uint32_t p0 = uint32_t(__fmul_rn(g.param[i], 65536.0f));
		uint4 s = g.rng[i];
		uint32_t p1 = urand(s) & 0xffffu;
		g.rng[i] = s;
		fired = p1 < p0 || ((stim >> lane) & 1u);
	}
	fireEpilogue(net, t, n, lane, valid, fired);
}

/* Input (src/nemo/cpu/plugins/Input.cpp:56-60) */
__global__ void __launch_bounds__(256)
k_update_input(NetDev net, GroupDev g, uint32_t offset, int resetSlot)
{
	uint32_t t, i, n, lane;
	bool valid;
	if(!groupThread(net, g, offset, resetSlot, t, i, n, lane, valid)) return;
	uint32_t stim = takeStimWord(net, n, lane);
	bool fired = false;
	if(valid) {
		float E, I;
		takeCurrents(net, n, E, I);
		(void) takeExternal(net, n);
		fired = (stim >> lane) & 1u;
	}
	fireEpilogue(net, t, n, lane, valid, fired);
}

/* ---------------- gather ---------------- */

/* Drain spike-queue slot t: each warp takes a row (source, delay) and adds
 * its weights into the target accumulators, excitatory (w >= 0) into E and
 * inhibitory into I (src/nemo/cpu/Simulation.cpp:293-308). 64-bit integer
 * reductions in L2 are exact in any order. */
__global__ void __launch_bounds__(256)
k_gather(NetDev net, uint32_t offset)
{
	uint32_t t = cycleOf(net, offset);
	if(blockIdx.x == 0 && threadIdx.x == 0) {
		net.eventsRing[t & net.ringMask] = 0;
		net.firedCountRing[t & net.ringMask] = 0;
	}
	uint32_t slot = t & net.qMask;
	uint32_t nrows = net.queueFill[slot];
	const uint32_t* rows = net.queue + size_t(slot) * net.qCap;
	uint32_t lane = threadIdx.x & 31u;
	uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
	unsigned long long* acc = reinterpret_cast<unsigned long long*>(net.acc);
	uint64_t delivered = 0;
	for(uint32_t r = warp; r < nrows; r += nwarps) {
		uint32_t row = rows[r];
		uint64_t b = net.rowStart[row];
		uint64_t e = net.rowStart[row + 1];
		delivered += e - b;
		for(uint64_t j = b + lane; j < e; j += 32) {
			uint2 syn = net.fcm[j];
			int32_t w = int32_t(syn.y);
			atomicAdd(&acc[2 * size_t(syn.x) + (w < 0 ? 1 : 0)], (unsigned long long) (long long) w);
		}
	}
	if(lane == 0 && delivered) {
		atomicAdd(&net.stats[0], (unsigned long long) delivered);
	}
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

/* ---------------- STDP ---------------- */

/* src/nemo/StdpProcess.cpp:68-113 */
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

/* src/nemo/StdpProcess.cpp:116-124 */
__device__ __forceinline__ int32_t weightChange(uint64_t pre, const StdpRule& R)
{
	return int32_t(uint32_t(updateRegion(pre & R.potentiation, R)) + uint32_t(updateRegion(pre & R.depression, R)));
}

/* Accumulate (src/nemo/ConnectivityMatrix.cpp:224-258): one warp per target
 * that fired P cycles ago walks its plastic in-synapses. Each accumulator has
 * a single writer, so plain read-modify-write is exact. */
__global__ void __launch_bounds__(256)
k_stdp(NetDev net, StdpRule rule, uint32_t offset)
{
	uint32_t t = cycleOf(net, offset);
	uint32_t par = t & 1u;
	if(blockIdx.x == 0 && threadIdx.x == 0) {
		net.postCount[par ^ 1u] = 0; /* consumed by the next cycle's update */
	}
	uint32_t count = net.postCount[par];
	const uint32_t* list = net.postList + size_t(par) * net.nDev;
	uint32_t lane = threadIdx.x & 31u;
	uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
	uint64_t visited = 0;
	for(uint32_t w = warp; w < count; w += nwarps) {
		uint32_t target = list[w];
		uint64_t b = net.rcmStart[target], e = net.rcmStart[target + 1];
		visited += e - b;
		for(uint64_t j = b + lane; j < e; j += 32) {
			uint32_t sd = net.rcmSrcDelay[j];
			uint64_t pre = shr64(net.recentFiring[sd >> 6], (sd & 63u) + 1u);
			int32_t dw = weightChange(pre, rule);
			if(dw != 0) {
				net.rcmAcc[j] = int32_t(uint32_t(net.rcmAcc[j]) + uint32_t(dw));
			}
		}
	}
	if(lane == 0 && visited) {
		atomicAdd(&net.stats[1], (unsigned long long) visited);
	}
}

/* src/nemo/StdpProcess.cpp:128-138 */
__device__ __forceinline__ int32_t updatedWeight(int32_t wOld, int32_t wDiff, const StdpRule& R)
{
	int32_t sum = int32_t(uint32_t(wOld) + uint32_t(wDiff));
	if(wOld > 0) return min(R.maxE, max(sum, R.minE));
	if(wOld < 0) return min(R.minI, max(sum, R.maxI));
	return 0;
}

/* applyStdp (src/nemo/ConnectivityMatrix.cpp:272-325): every plastic synapse
 * gets w = clamp(w + (reward * acc) >> f) and its accumulator cleared. */
__global__ void __launch_bounds__(256)
k_apply_stdp(NetDev net, StdpRule rule, int32_t reward, uint64_t nrcm)
{
	uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
	for(uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < nrcm; j += stride) {
		uint32_t f = net.rcmForward[j];
		int32_t acc = net.rcmAcc[j];
		int32_t wOld = int32_t(net.fcm[f].y);
		int32_t diff = int32_t((int64_t(reward) * int64_t(acc)) >> net.fbits);
		int32_t wNew = updatedWeight(wOld, diff, rule);
		if(wNew != wOld) {
			net.fcm[f].y = uint32_t(wNew);
		}
		if(acc) {
			net.rcmAcc[j] = 0;
		}
	}
}

__global__ void
k_advance_cycle(uint32_t* counter, uint32_t by)
{
	*counter += by;
}

__global__ void
k_nrand_probe(const uint32_t* u1, const uint32_t* u2, float* out, size_t n, const uint32_t* sinTab, const uint32_t* logTab)
{
	size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
	if(i < n) {
		/* a state whose next two outputs are u1[i], u2[i]: with x=y=z=0 and
		 * w chosen, xorshift returns w ^ (w >> 19) ^ 0 ... instead evaluate
		 * the transform directly on the given words */
		using namespace libm;
		float f1 = __uint2float_rn(u1[i]);
		float f2 = __uint2float_rn(u2[i]);
		float a = sin_argument(f1);
		float y = log_argument(f2);
		float L = apply_code(log_candidate(y), table_code(logTab, libm_index(f2)));
		float r = __fsqrt_rn(__fmul_rn(-2.0f, L));
		float S = apply_code(sin_candidate(a), table_code(sinTab, libm_index(f1)));
		out[i] = __fmul_rn(S, r);
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

int g_smCount = 0;

} // namespace

void
launchLibmEval(float* sinOut, float* logOut, const uint32_t* sinTab, const uint32_t* logTab, void* stream)
{
	k_libm_eval<<<smCount() * 8, 256, 0, static_cast<cudaStream_t>(stream)>>>(sinOut, logOut, sinTab, logTab);
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
launchGather(const NetDev& net, uint32_t offset, void* stream)
{
	k_gather<<<smCount() * 4, 256, 0, S(stream)>>>(net, offset);
}

void
launchUpdate(int model, const NetDev& net, const GroupDev& g, uint32_t offset, bool resetSlot, void* stream)
{
	uint32_t blocks = (g.count + 255) / 256;
	if(blocks == 0) blocks = 1;
	int rs = resetSlot ? 1 : 0;
	switch(model) {
		case 0: k_update_izhikevich<<<blocks, 256, 0, S(stream)>>>(net, g, offset, rs); break;
		case 1: k_update_if_curr_exp<<<blocks, 256, 0, S(stream)>>>(net, g, offset, rs); break;
		case 2: k_update_qif<<<blocks, 256, 0, S(stream)>>>(net, g, offset, rs); break;
		case 4: k_update_poisson<<<blocks, 256, 0, S(stream)>>>(net, g, offset, rs); break;
		case 5: k_update_input<<<blocks, 256, 0, S(stream)>>>(net, g, offset, rs); break;
		default: break;
	}
}

void
launchStdp(const NetDev& net, const StdpRule& rule, uint32_t offset, void* stream)
{
	k_stdp<<<smCount() * 4, 256, 0, S(stream)>>>(net, rule, offset);
}

void
launchApplyStdp(const NetDev& net, const StdpRule& rule, int32_t reward, uint64_t nrcm, void* stream)
{
	uint64_t blocks = (nrcm + 255) / 256;
	uint64_t cap = uint64_t(smCount()) * 8;
	if(blocks > cap) blocks = cap;
	if(blocks == 0) blocks = 1;
	k_apply_stdp<<<uint32_t(blocks), 256, 0, S(stream)>>>(net, rule, reward, nrcm);
}

void
launchAdvanceCycle(uint32_t* counter, uint32_t by, void* stream)
{
	k_advance_cycle<<<1, 1, 0, S(stream)>>>(counter, by);
}

void
launchNrandProbe(const uint32_t* u1, const uint32_t* u2, float* out, size_t n,
		const uint32_t* sinTab, const uint32_t* logTab, void* stream)
{
	if(n == 0) return;
	k_nrand_probe<<<uint32_t((n + 255) / 256), 256, 0, S(stream)>>>(u1, u2, out, n, sinTab, logTab);
}

} // namespace nemo_b200
