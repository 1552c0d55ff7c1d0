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

#include <cstdint>
#include <mutex>

#include "kernels.hpp"
#include "libm_match.cuh"

namespace nemo_b200 {

namespace {

const unsigned FULL = 0xffffffffu;
const unsigned BLOCK = 1024;

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

/* Read and clear neuron n's E/I sums for the current cycle's slot. With
 * int32 accumulators the host has proven that no sum can leave the int32
 * range, so the value equals the int64 sum and needs no saturation. */
__device__ __forceinline__ void takeCurrents(const NetDev& net, uint32_t slot, uint32_t n, float& E, float& I)
{
	if(net.acc32) {
		int2* acc = reinterpret_cast<int2*>(net.acc) + size_t(slot) * net.nDev;
		int2 a = acc[n];
		if(a.x | a.y) {
			acc[n] = make_int2(0, 0);
		}
		E = wfxToFloat(a.x, net.fbits);
		I = wfxToFloat(a.y, net.fbits);
	} else {
		longlong2* acc = reinterpret_cast<longlong2*>(net.acc) + size_t(slot) * net.nDev;
		longlong2 a = acc[n];
		if(a.x | a.y) {
			acc[n] = make_longlong2(0, 0);
		}
		E = wfxToFloat(a.x, net.fbits);
		I = wfxToFloat(a.y, net.fbits);
	}
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

/* ---------------- neuron models (one neuron per thread) ---------------- */

/* Izhikevich (src/nemo/cpu/plugins/Izhikevich.cpp:53-97). Parameters a, b, c,
 * d, sigma; state u, v. The v update evaluates its bracket in double (double
 * literals in the reference), the u update in float. */
__device__ __forceinline__ bool modelIzhikevich(const NetDev& net, const GroupDev& g, uint32_t i, uint32_t n,
		uint32_t slot, bool stim)
{
	const size_t c = g.count;
	float E, I;
	takeCurrents(net, slot, n, E, I);
	float In = __fadd_rn(__fadd_rn(E, I), takeExternal(net, n));
	float sigma = g.param[4 * c + i];
	uint4 s = g.rng[i]; /* loaded with the other operands; used only with noise */
	if(sigma != 0.0f) {
		In = __fadd_rn(In, __fmul_rn(sigma, nrand(s, net.sinTab, net.logTab)));
		g.rng[i] = s;
	}
	float a = g.param[0 * c + i];
	float b = g.param[1 * c + i];
	float u = g.state[0 * c + i];
	float v = g.state[1 * c + i];
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
		v = g.param[2 * c + i];
		u = __fadd_rn(u, g.param[3 * c + i]);
	}
	g.state[0 * c + i] = u;
	g.state[1 * c + i] = v;
	return fired;
}

/* IF_curr_exp (src/nemo/cpu/plugins/IF_curr_exp.cpp:74-121). Parameters in
 * IF_curr_exp.h order; state v, ie, ii, lastfire. Fires on v > v_thresh. */
__device__ __forceinline__ bool modelIfCurrExp(const NetDev& net, const GroupDev& g, uint32_t i, uint32_t n,
		uint32_t slot, bool stim)
{
	const size_t c = g.count;
	const float* P = g.param;
	float* S = g.state;
	float E, I;
	takeCurrents(net, slot, n, E, I);
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
	bool fired = (!refractory && v > v_thresh) || stim;
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
		uint32_t slot, bool stim)
{
	const float dt = 0.1f;
	const float a1 = __fmul_rn(0.5f, dt);
	const float a2 = dt;
	const float bb1 = __fdiv_rn(dt, 6.0f);
	float E, I;
	takeCurrents(net, slot, n, E, I);
	float X = takeExternal(net, n);
	float v = g.state[i];
	float a = g.param[i];
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

/* PoissonSource (src/nemo/cpu/plugins/PoissonSource.cpp:21-29). Currents are
 * cleared (every neuron's slot must be) but unused. */
__device__ __forceinline__ bool modelPoisson(const NetDev& net, const GroupDev& g, uint32_t i, uint32_t n,
		uint32_t slot, bool stim)
{
	float E, I;
	takeCurrents(net, slot, n, E, I);
	(void) takeExternal(net, n);
	uint32_t p0 = uint32_t(__fmul_rn(g.param[i], 65536.0f));
	uint4 s = g.rng[i];
	uint32_t p1 = urand(s) & 0xffffu;
	g.rng[i] = s;
	return p1 < p0 || stim;
}

/* Input (src/nemo/cpu/plugins/Input.cpp:56-60) */
__device__ __forceinline__ bool modelInput(const NetDev& net, const GroupDev& g, uint32_t i, uint32_t n,
		uint32_t slot, bool stim)
{
	float E, I;
	takeCurrents(net, slot, n, E, I);
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

/* Sense-reversal barrier over all blocks of the cooperative launch. A block
 * that waits longer than timeoutNs sets the error word and returns false;
 * every waiting block also gives up as soon as it sees the error word, so the
 * kernel always terminates. */
__device__ __forceinline__ bool gridSync(unsigned* bar, unsigned long long timeoutNs)
{
	__shared__ int ok;
	__syncthreads();
	if(threadIdx.x == 0) {
		cuda::atomic_ref<unsigned, cuda::thread_scope_device> count(bar[0]);
		cuda::atomic_ref<unsigned, cuda::thread_scope_device> gen(bar[1]);
		cuda::atomic_ref<unsigned, cuda::thread_scope_device> err(bar[2]);
		int good = 1;
		unsigned g = gen.load(cuda::memory_order_relaxed);
		/* publish the block's writes (ordered before this thread by the
		 * __syncthreads above) to the whole device */
		cuda::atomic_thread_fence(cuda::memory_order_acq_rel, cuda::thread_scope_device);
		unsigned arrived = count.fetch_add(1u, cuda::memory_order_acq_rel);
		if(arrived == gridDim.x - 1) {
			count.store(0u, cuda::memory_order_relaxed);
			gen.fetch_add(1u, cuda::memory_order_release);
		} else {
			unsigned long long start = globalTimer();
			unsigned spins = 0;
			while(gen.load(cuda::memory_order_acquire) == g) {
				if((++spins & 1023u) == 0) {
					if(err.load(cuda::memory_order_relaxed)) {
						good = 0;
						break;
					}
					if(globalTimer() - start > timeoutNs) {
						err.store(1u, cuda::memory_order_relaxed);
						good = 0;
						break;
					}
				}
			}
		}
		ok = good;
	}
	__syncthreads();
	return ok != 0;
}

/* ---------------- the persistent step kernel ---------------- */

/* Work lists of a block, in global memory (per-block regions of listCap
 * entries of {neuron, first synapse, synapse count}):
 *   fired[listCap]   sources fired by this block's neurons in this cycle,
 *   post[2][listCap] this block's post-spiking targets of the last two cycles.
 * Push and STDP work is split into 128-synapse items, one per warp, four
 * independent synapses per lane. */
__global__ void __launch_bounds__(BLOCK, 1)
k_cycles(const __grid_constant__ CycleArgs A)
{
	__shared__ uint32_t sNFired;
	__shared__ uint32_t sNPost[2];
	__shared__ unsigned long long sEvents;

	const NetDev& net = A.net;
	const uint32_t tid = threadIdx.x;
	const uint32_t lane = tid & 31u;
	const uint32_t warp = tid >> 5;
	const uint32_t lt = (1u << lane) - 1u;
	const uint32_t warpsPerBlock = blockDim.x >> 5;
	const uint32_t gridWarps = gridDim.x * warpsPerBlock;
	/* 32-neuron warps are dealt to blocks round-robin, so that every block
	 * updates (and then pushes and learns for) a similar share */
	const uint32_t myWarp = warp * gridDim.x + blockIdx.x;
	const uint32_t totalWarps = A.groupWarp[A.ngroups];
	const size_t nDev = net.nDev;
	const uint32_t cap = A.listCap;
	uint32_t* firedList = net.lists + size_t(blockIdx.x) * cap * 9u;
	uint32_t* postLists = firedList + size_t(cap) * 3u;

	if(tid == 0) {
		sNPost[0] = 0;
		sNPost[1] = 0;
	}

	for(uint32_t k = 0; k <= A.cycles; ++k) {
		const uint64_t t64 = A.firstCycle + k;
		const uint32_t t = uint32_t(t64);
		const uint32_t slotT = uint32_t(t64 % net.slots);   /* current slot of cycle t */
		const bool doUpdate = k < A.cycles;
		const uint32_t pb = t & 1u;

		if(tid == 0) {
			sNFired = 0;
			sEvents = 0;
			if(doUpdate) {
				sNPost[pb] = 0;
				if(blockIdx.x == 0) {
					net.firedCountRing[(t + 1) & net.ringMask] = 0;
					net.eventsRing[(t + 1) & net.ringMask] = 0;
				}
			}
		}
		__syncthreads();
		unsigned long long* trace = A.trace ? A.trace + (size_t(k) * gridDim.x + blockIdx.x) * 4u : nullptr;
		if(trace && tid == 0) trace[0] = globalTimer();

		/* ---- neuron update of cycle t ---- */
		if(doUpdate) {
			const uint32_t slot = slotT;
			const uint64_t* rfIn = net.rf + (t & 1u) * nDev;
			uint64_t* rfOut = net.rf + ((t + 1) & 1u) * nDev;
			uint32_t* postOut = postLists + size_t(pb) * cap * 3u;
			for(uint32_t gw = myWarp; gw < totalWarps; gw += gridWarps) {
				int gi = 0;
				while(gw >= A.groupWarp[gi + 1]) ++gi;
				const GroupDev& G = A.groups[gi];
				const uint32_t i = (gw - A.groupWarp[gi]) * 32u + lane;
				const uint32_t n = G.devBase + i;
				const bool valid = i < G.count;
				const uint32_t stimWord = takeStimWord(net, n, lane);
				uint64_t rfPrev = valid ? rfIn[n] : 0ull;
				bool fired = false;
				if(valid) {
					const bool stim = (stimWord >> lane) & 1u;
					switch(G.kind) {
						case 0: fired = modelIzhikevich(net, G, i, n, slot, stim); break;
						case 1: fired = modelIfCurrExp(net, G, i, n, slot, stim); break;
						case 2: fired = modelQif(net, G, i, n, slot, stim); break;
						case 4: fired = modelPoisson(net, G, i, n, slot, stim); break;
						default: fired = modelInput(net, G, i, n, slot, stim); break;
					}
				}
				const uint64_t rfNew = (rfPrev << 1) | uint64_t(fired);
				if(valid) {
					rfOut[n] = rfNew;
				}
				const uint32_t word = __ballot_sync(FULL, fired);
				if(lane == 0) {
					net.firedRing[size_t(t & net.ringMask) * net.nWords + (n >> 5)] = word;
				}
				if(word) {
					uint32_t base = 0;
					if(lane == 0) base = atomicAdd(&sNFired, uint32_t(__popc(word)));
					base = __shfl_sync(FULL, base, 0);
					uint32_t deg = 0;
					if(fired) {
						uint64_t b = net.rowStart[size_t(n) * net.rowStride];
						uint64_t e = net.rowStart[size_t(n + 1) * net.rowStride];
						deg = uint32_t(e - b);
						uint32_t* entry = firedList + size_t(base + __popc(word & lt)) * 3u;
						entry[0] = n;
						entry[1] = uint32_t(b);
						entry[2] = deg;
					}
					uint32_t ev = __reduce_add_sync(FULL, deg);
					if(lane == 0) atomicAdd(&sEvents, (unsigned long long) ev);
				}
				if(net.stdp) {
					/* post-synaptic firing P cycles ago (ConnectivityMatrix.cpp:237) */
					const bool post = valid && ((rfNew >> net.postShift) & 1ull);
					const uint32_t pm = __ballot_sync(FULL, post);
					if(pm) {
						uint32_t base = 0;
						if(lane == 0) base = atomicAdd(&sNPost[pb], uint32_t(__popc(pm)));
						base = __shfl_sync(FULL, base, 0);
						if(post) {
							uint64_t b = net.rcmStart[n];
							uint64_t e = net.rcmStart[n + 1];
							uint32_t* entry = postOut + size_t(base + __popc(pm & lt)) * 3u;
							entry[0] = n;
							entry[1] = uint32_t(b);
							entry[2] = uint32_t(e - b);
						}
					}
				}
			}
		}
		/* ---- STDP accumulation of cycle t-1 (ConnectivityMatrix.cpp:224-258)
		 * for this block's targets that fired P cycles before it; every
		 * accumulator has a single writer. It only reads the history after
		 * cycle t-1, so warps start on it as soon as their own update of
		 * cycle t is done ---- */
		if(net.stdp && k > 0) {
			const uint32_t* postIn = postLists + size_t(pb ^ 1u) * cap * 3u;
			const uint64_t* rfAfter = net.rf + (t & 1u) * nDev;   /* history after update(t-1) */
			const uint32_t items = sNPost[pb ^ 1u] * net.stdpChunks;
			uint64_t visited = 0;
			for(uint32_t it = warp; it < items; it += warpsPerBlock) {
				const uint32_t* entry = postIn + size_t(it / net.stdpChunks) * 3u;
				const uint32_t off = (it % net.stdpChunks) * 128u;
				const uint32_t len = entry[2];
				if(off >= len) continue;
				const uint64_t b = uint64_t(entry[1]) + off;
				const uint32_t cnt = len - off < 128u ? len - off : 128u;
				visited += cnt;
				uint32_t sd[4];
#pragma unroll
				for(int u = 0; u < 4; ++u) {
					uint32_t j = lane + 32u * u;
					sd[u] = j < cnt ? net.rcmSrcDelay[b + j] : 0u;
				}
				uint64_t pre[4];
				int32_t old[4];
#pragma unroll
				for(int u = 0; u < 4; ++u) {
					uint32_t j = lane + 32u * u;
					pre[u] = j < cnt ? shr64(rfAfter[sd[u] >> 6], (sd[u] & 63u) + 1u) : 0ull;
					old[u] = j < cnt ? net.rcmAcc[b + j] : 0;
				}
#pragma unroll
				for(int u = 0; u < 4; ++u) {
					uint32_t j = lane + 32u * u;
					if(j < cnt) {
						int32_t dw = weightChange(pre[u], A.rule);
						if(dw != 0) {
							net.rcmAcc[b + j] = int32_t(uint32_t(old[u]) + uint32_t(dw));
						}
					}
				}
			}
			if(lane == 0 && visited) {
				atomicAdd(&net.stats[1], (unsigned long long) visited);
			}
		}

		__syncthreads();
		if(trace && tid == 0) trace[1] = globalTimer();

		if(doUpdate) {
			if(tid == 0 && sNFired) {
				atomicAdd(&net.firedCountRing[t & net.ringMask], sNFired);
				atomicAdd(&net.eventsRing[t & net.ringMask], sEvents);
				atomicAdd(&net.stats[2], (unsigned long long) sNFired);
				atomicAdd(&net.stats[3], sEvents);
				if(net.deliver) atomicAdd(&net.stats[0], sEvents);
			}

			/* ---- spike push: the synapses of this block's fired sources go
			 * into the current slots of cycles t + delay ---- */
			if(net.deliver) {
				const uint32_t items = sNFired * net.fireChunks;
				for(uint32_t it = warp; it < items; it += warpsPerBlock) {
					const uint32_t* entry = firedList + size_t(it / net.fireChunks) * 3u;
					const uint32_t off = (it % net.fireChunks) * 128u;
					const uint32_t len = entry[2];
					if(off >= len) continue;
					const uint64_t b = uint64_t(entry[1]) + off;
					const uint32_t cnt = len - off < 128u ? len - off : 128u;
					uint2 syn[4];
#pragma unroll
					for(int u = 0; u < 4; ++u) {
						uint32_t j = lane + 32u * u;
						syn[u] = j < cnt ? net.fcm[b + j] : make_uint2(0u, 0u);
					}
#pragma unroll
					for(int u = 0; u < 4; ++u) {
						if(lane + 32u * u < cnt) {
							/* slot of cycle t + d, d <= maxDelay < slots */
							uint32_t s = slotT + (syn[u].x & 63u) + 1u;
							s = s >= net.slots ? s - net.slots : s;
							const int32_t w = int32_t(syn[u].y);
							addCurrent(net, s, syn[u].x >> 6, w < 0 ? 1 : 0, w);
						}
					}
				}
			}
		}

		if(trace) {
			__syncthreads();
			if(tid == 0) trace[2] = globalTimer();
		}
		if(k < A.cycles) {
			if(!gridSync(net.barrier, A.timeoutNs)) {
				return;
			}
		}
		if(trace && tid == 0) trace[3] = globalTimer();
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

/* Stimulus of the allocation-free step, read from the per-device scratch
 * below: [0, nf) firing-stimulus device indices, [NOALLOC_STIM_MAX,
 * +ni) current-stimulus device indices, [2 NOALLOC_STIM_MAX, +ni) their
 * currents (float bits). One warp walks the current stimulus in order, 32
 * entries at a time; of equal indices within a group the highest lane writes,
 * and __syncwarp orders the groups, so the last entry for a neuron wins as in
 * the reference (cpu/Simulation.cpp:140-163). */
__global__ void
k_stimulus_scratch(NetDev net, const uint32_t* scratch, uint32_t nf, uint32_t ni)
{
	const uint32_t lane = threadIdx.x;
	for(uint32_t i = lane; i < nf; i += 32) {
		uint32_t n = scratch[i];
		atomicOr(&net.fstim[n >> 5], 1u << (n & 31u));
	}
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
 * (deliverSpikes at cycle t0 + d), whereas the step kernel adds it when the
 * source fires (cycle t0). For a spike still in flight when its synapse's
 * weight changes, the arrival slot therefore holds the old weight; it is
 * corrected here by w_new - w_old, into the same E/I half (the sign of a
 * weight never changes, and a weight that reaches 0 contributes 0 to E). The
 * in-flight spikes of a synapse with delay d are the set bits 0..d-1 of its
 * source's firing history after the last completed cycle (cycleNow - 1):
 * bit k fired at cycleNow-1-k and arrives at cycleNow-1-k+d.
 *
 * The synapses are processed in APPLY_WINDOW-sized windows of the forward
 * matrix, one launch per window, so that the weights a launch rewrites stay
 * in L2 (each target's plastic synapses are sorted by forward position, and
 * rcmWindow locates the range of each target in each window). One warp per
 * target. */
__global__ void __launch_bounds__(256)
k_apply_stdp(NetDev net, StdpRule rule, int32_t reward, uint64_t cycleNow, uint32_t window)
{
	const uint64_t* rfNow = net.rf + size_t(cycleNow & 1u) * net.nDev;
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
	for(uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < net.nDev; t += nwarps) {
	const uint64_t base = net.rcmStart[t];
	const uint32_t* win = net.rcmWindow + size_t(t) * (net.windows + 1) + window;
	const uint64_t e = base + win[1];
	for(uint64_t j = base + win[0] + lane; j < e; j += 32) {
		uint32_t f = net.rcmForward[j];
		int32_t acc = net.rcmAcc[j];
		uint2 syn = net.fcm[f];
		int32_t wOld = int32_t(syn.y);
		int32_t diff = int32_t((int64_t(reward) * int64_t(acc)) >> net.fbits);
		int32_t wNew = updatedWeight(wOld, diff, rule);
		if(wNew != wOld) {
			net.fcm[f].y = uint32_t(wNew);
			if(net.deliver) {
				uint32_t sd = net.rcmSrcDelay[j];
				uint32_t d = (sd & 63u) + 1u;
				uint64_t pending = rfNow[sd >> 6] & ((uint64_t(1) << d) - 1u);
				if(pending) {
					size_t target = syn.x >> 6;
					long long delta = (long long) wNew - (long long) wOld;
					int half = wOld >= 0 ? 0 : 1;
					while(pending) {
						uint32_t k = uint32_t(__ffsll((long long) pending) - 1);
						pending &= pending - 1;
						/* fired at cycleNow-1-k >= 0, arrives at cycleNow-1-k+d */
						uint32_t slot = uint32_t((cycleNow - 1u - k + d) % net.slots);
						addCurrent(net, slot, uint32_t(target), half, delta);
					}
				}
			}
		}
		if(acc) {
			net.rcmAcc[j] = 0;
		}
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

int g_smCount = 0;
int g_blocksPerSm = 0;

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
	k_stimulus_scratch<<<1, 32, 0, S(stream)>>>(net, scratch, nf, ni);
}

/* Co-resident grid for the cooperative launch: as many 1024-thread blocks per
 * SM as the registers allow (one), times the SM count. */
void
cyclesGrid(uint32_t totalWarps, unsigned* blocks, uint32_t* listCap)
{
	const uint32_t warpsPerBlock = BLOCK / 32;
	if(g_blocksPerSm == 0) {
		int perSm = 0;
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_cycles, BLOCK, 0);
		g_blocksPerSm = perSm > 0 ? perSm : 1;
	}
	unsigned b = unsigned(smCount() * g_blocksPerSm);
	uint32_t gridWarps = b * warpsPerBlock;
	uint32_t perWarp = (totalWarps + gridWarps - 1) / gridWarps;
	if(perWarp == 0) perWarp = 1;
	*blocks = b;
	*listCap = perWarp * warpsPerBlock * 32;
}

void
launchCycles(const CycleArgs& args, unsigned blocks, void* stream)
{
	void* params[] = {const_cast<CycleArgs*>(&args)};
	cudaLaunchCooperativeKernel((const void*) k_cycles, dim3(blocks), dim3(BLOCK), params, 0, S(stream));
}

void
launchApplyStdp(const NetDev& net, const StdpRule& rule, int32_t reward, uint64_t nrcm, uint64_t cycleNow, void* stream)
{
	if(nrcm == 0) return;
	/* one warp per target per window */
	uint64_t blocks = (uint64_t(net.nDev) * 32 + 255) / 256;
	uint64_t cap = uint64_t(smCount()) * 8;
	if(blocks > cap) blocks = cap;
	for(uint32_t w = 0; w < net.windows; ++w) {
		k_apply_stdp<<<uint32_t(blocks), 256, 0, S(stream)>>>(net, rule, reward, cycleNow, w);
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
launchLibmEval(float* sinOut, float* logOut, const uint32_t* sinTab, const uint32_t* logTab, void* stream)
{
	k_libm_eval<<<smCount() * 8, 256, 0, S(stream)>>>(sinOut, logOut, sinTab, logTab);
}

} // namespace nemo_b200
