#ifndef NEMO_B200_KERNELS_HPP
#define NEMO_B200_KERNELS_HPP

/* Interface between the host orchestration (simulation.cpp) and the sm_100a
 * kernels (kernels.cu). Plain structs of device pointers passed by value.
 *
 * Device index space: neuron types occupy consecutive ranges in registration
 * order, like the reference's simulation indices (src/nemo/cpu/
 * Simulation.cpp:58-73), but each range starts on a multiple of 32 so that one
 * warp owns whole 32-bit words of every per-neuron bitmap. Padding slots
 * never fire and have no synapses.
 *
 * Per-cycle data flow (cycle t):
 *   gather  : drain spike-queue slot t into the int64 E/I accumulators
 *   update  : per type; currents -> state, firing bitmap for t, and the
 *             scatter epilogue that enqueues each fired neuron's rows into
 *             slots t+d, plus the STDP post-spike list
 *   stdp    : accumulate weight changes for targets that fired at t-P
 */

#include <cstdint>

#include <vector_types.h>

namespace nemo_b200 {

struct NetDev {
	uint32_t nDev;          /* device neurons, multiple of 32 */
	uint32_t nWords;        /* nDev / 32 */
	uint32_t rowStride;     /* rows per source: max(maxDelay, 1) */
	uint32_t qMask;         /* spike-queue slots - 1 (power of two > maxDelay) */
	uint64_t qCap;          /* rows per slot: number of non-empty rows */
	uint32_t ringMask;      /* firing-ring cycles - 1 */
	uint32_t fbits;         /* fractional bits of the Q(31-f).f weights */

	const uint32_t* cycleBase;     /* device cycle counter (advanced by graph runs) */

	/* forward connectivity: row r = source * rowStride + delay - 1 */
	const uint64_t* rowStart;      /* [nDev * rowStride + 1] */
	uint2* fcm;                    /* {target device index, int32 weight} */
	const uint64_t* delayBits;     /* [nDev] deliverable delays, bit d-1 */
	const uint32_t* outDegree;     /* [nDev] synapses per source */

	/* spike queue: slot s holds row ids to deliver at cycles = s (mod slots) */
	uint32_t* queue;               /* [slots * qCap] */
	uint32_t* queueFill;           /* [slots] */

	long long* acc;                /* [2 * nDev] int64 E at 2n, I at 2n+1 */
	uint64_t* recentFiring;        /* [nDev] firing history, bit 0 = last cycle */
	uint32_t* firedRing;           /* [ring * nWords] firing bitmaps by cycle */
	unsigned long long* eventsRing;/* [ring] synaptic events (fired x out-degree) */
	uint32_t* firedCountRing;      /* [ring] */
	float* ext;                    /* [nDev] external current, cleared after use */
	uint32_t* fstim;               /* [nWords] firing stimulus, cleared after use */

	/* STDP (reverse connectivity of plastic synapses, grouped by target) */
	int stdp;
	uint32_t postShift;            /* bit of the history that triggers STDP */
	uint32_t* postList;            /* [2 * nDev] */
	uint32_t* postCount;           /* [2] */
	const uint64_t* rcmStart;      /* [nDev + 1] */
	const uint32_t* rcmSrcDelay;   /* source << 6 | (delay - 1) */
	const uint32_t* rcmForward;    /* index into fcm */
	int32_t* rcmAcc;

	/* glibc-matching correction tables (libm_match.cuh) */
	const uint32_t* sinTab;
	const uint32_t* logTab;

	/* cumulative counters: [0] synapses delivered by gather, [1] synapses
	 * visited by STDP accumulation, [2] neurons fired, [3] synaptic events
	 * generated (fired x out-degree) */
	unsigned long long* stats;
};

struct GroupDev {
	uint32_t devBase;       /* first device index (multiple of 32) */
	uint32_t count;
	uint32_t timerBase;     /* cycle at the last timer reset (HH counts from it) */
	float* param;           /* [nParam][count] */
	float* state;           /* [nState][count] */
	uint4* rng;             /* [count] xorshift128 state */
};

/* The STDP rule in fixed point (src/nemo/StdpProcess.cpp:20-46) */
struct StdpRule {
	uint64_t potentiation;
	uint64_t depression;
	uint64_t prePostBits;
	uint64_t postPreBits;
	uint32_t postPreWindow;
	int32_t minE, maxE, minI, maxI;
	int32_t fnPre[64];
	int32_t fnPost[64];
};

struct StimDev {
	const uint32_t* fstim;  /* device indices */
	uint32_t nf;
	const uint32_t* inidx;  /* device indices, unique */
	const float* icur;
	uint32_t ni;
};

/* Launchers (kernels.cu). All launch on `stream`; `offset` is added to the
 * device cycle counter to obtain the cycle. */
void launchStimulus(const NetDev& net, const StimDev& stim, void* stream);
void launchGather(const NetDev& net, uint32_t offset, void* stream);
void launchUpdate(int model, const NetDev& net, const GroupDev& g, uint32_t offset, bool resetSlot, void* stream);
void launchStdp(const NetDev& net, const StdpRule& rule, uint32_t offset, void* stream);
void launchApplyStdp(const NetDev& net, const StdpRule& rule, int32_t reward, uint64_t nrcm, void* stream);
void launchAdvanceCycle(uint32_t* counter, uint32_t by, void* stream);
void launchNrandProbe(const uint32_t* u1, const uint32_t* u2, float* out, size_t n,
		const uint32_t* sinTab, const uint32_t* logTab, void* stream);
void launchLibmEval(float* sinOut, float* logOut, const uint32_t* sinTab, const uint32_t* logTab, void* stream);
int smCount();

} // namespace nemo_b200

#endif
