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
 * The step path is one persistent cooperative kernel (k_cycles) that runs a
 * block of cycles with one grid barrier per cycle. Phase t:
 *   - neuron update of cycle t: read and clear the cycle's current slot
 *     acc[t mod Q], integrate, fire, shift the firing history
 *     (rf[t&1] -> rf[(t+1)&1]), record the firing bitmap and the STDP
 *     post-spike list of cycle t;
 *   - spike push: every neuron fired at t streams its outgoing synapses (one
 *     contiguous range per source, sorted by delay) and adds each weight into
 *     acc[(t+d) mod Q][target] (E or I by sign) with fire-and-forget 64-bit
 *     reductions in L2 — the reference's deliverSpikes at cycle t+d
 *     (src/nemo/cpu/Simulation.cpp:259-308) moved to fire time;
 *   - STDP accumulation of cycle t-1 (targets that fired P cycles before it),
 *     which only reads rf[t&1] and so overlaps the update of cycle t;
 *   - grid barrier.
 * A final half phase accumulates STDP for the last cycle. Integer sums are
 * exact in any order, so the result is bit-identical to the CPU reference. */

#include <cstdint>

#include <vector_types.h>

namespace nemo_b200 {

const int MAX_GROUPS = 8;

/* applyStdp window: 4M synapses = 32 MB of the forward matrix, small enough
 * to stay resident in the 126 MB L2 while its weights are updated */
const uint64_t APPLY_WINDOW = uint64_t(1) << 22;

struct NetDev {
	uint32_t nDev;          /* device neurons, multiple of 32 */
	uint32_t nWords;        /* nDev / 32 */
	uint32_t rowStride;     /* rows per source: max(maxDelay, 1) */
	uint32_t slots;         /* current slots: maxDelay + 1 (cycle t uses slot t mod slots) */
	int acc32;              /* int32 accumulators (proven not to overflow), else int64 */
	uint32_t ringMask;      /* firing-ring cycles - 1 */
	uint32_t fbits;         /* fractional bits of the Q(31-f).f weights */
	int deliver;            /* 0 when no delay is deliverable (max delay 64) */

	/* forward connectivity: row r = source * rowStride + delay - 1; the rows
	 * of one source are contiguous, so [rowStart[s*rowStride],
	 * rowStart[(s+1)*rowStride]) is all of its synapses in delay order */
	const uint64_t* rowStart;      /* [nDev * rowStride + 1] */
	uint2* fcm;                    /* {target << 6 | (delay - 1), int32 weight} */
	const uint32_t* outDegree;     /* [nDev] synapses per source */

	void* acc;                     /* [slots][nDev][2] E, I current of a future cycle (int32 or int64) */
	uint64_t* rf;                  /* [2][nDev] firing history, bit 0 = last cycle */
	uint32_t* firedRing;           /* [ring][nWords] firing bitmaps by cycle */
	unsigned long long* eventsRing;/* [ring] synaptic events (fired x out-degree) */
	uint32_t* firedCountRing;      /* [ring] */
	float* ext;                    /* [nDev] external current, cleared after use */
	uint32_t* fstim;               /* [nWords] firing stimulus, cleared after use */

	/* per-block work lists of the step kernel: [blocks][9 * listCap] */
	uint32_t* lists;
	uint32_t fireChunks;           /* 128-synapse chunks per source (max out-degree) */

	/* STDP (reverse connectivity of plastic synapses, grouped by target) */
	int stdp;
	uint32_t postShift;            /* bit of the history that triggers STDP */
	uint32_t stdpChunks;           /* 128-synapse chunks per target (max in-degree) */
	const uint64_t* rcmStart;      /* [nDev + 1] */
	const uint32_t* rcmSrcDelay;   /* source << 6 | (delay - 1) */
	const uint32_t* rcmForward;    /* index into fcm, ascending within a target */
	int32_t* rcmAcc;
	/* [nDev][windows + 1]: first synapse of each target in each forward
	 * window of APPLY_WINDOW synapses (applyStdp works window by window) */
	const uint32_t* rcmWindow;
	uint32_t windows;

	/* glibc-matching correction tables (libm_match.cuh) */
	const uint32_t* sinTab;
	const uint32_t* logTab;

	/* cumulative counters: [0] synapses pushed, [1] STDP synapse visits,
	 * [2] neurons fired, [3] synaptic events (fired x out-degree) */
	unsigned long long* stats;

	/* grid barrier: [0] arrivals, [1] generation, [2] error (timeout) */
	unsigned* barrier;
};

struct GroupDev {
	uint32_t devBase;       /* first device index (multiple of 32) */
	uint32_t count;
	uint32_t timerBase;     /* cycle at the last timer reset (HH counts from it) */
	int kind;               /* ModelKind */
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

struct CycleArgs {
	NetDev net;
	StdpRule rule;
	GroupDev groups[MAX_GROUPS];
	uint32_t groupWarp[MAX_GROUPS + 1];  /* prefix of 32-neuron warps per group */
	int ngroups;
	uint64_t firstCycle;
	uint32_t cycles;
	uint32_t listCap;                    /* entries per per-block work list */
	unsigned long long timeoutNs;        /* grid-barrier wait limit */
	/* optional phase timestamps (%globaltimer ns), [cycle][block][4]: phase
	 * start, update done, push and STDP done, barrier passed */
	unsigned long long* trace;
};

struct StimDev {
	const uint32_t* fstim;  /* device indices */
	uint32_t nf;
	const uint32_t* inidx;  /* device indices, unique */
	const float* icur;
	uint32_t ni;
};

/* Allocation-free step: at most this many firing-stimulus and this many
 * current-stimulus entries per call, staged in a module-static scratch array
 * (one per device, shared by all simulations on it). */
const uint32_t NOALLOC_STIM_MAX = 16384;
const int NOALLOC_MAX_DEVICES = 64;

/* Device address of the allocation-free scratch on `device`, which must be
 * the current device. Looked up with cudaGetSymbolAddress on the first call
 * per device, then cached. Returns a cudaError_t value. */
int noallocScratch(int device, uint32_t** ptr);

/* Launchers (kernels.cu), all on `stream`. */
void launchStimulus(const NetDev& net, const StimDev& stim, void* stream);
/* Stimulus from the allocation-free scratch (layout in kernels.cu). */
void launchStimulusScratch(const NetDev& net, const uint32_t* scratch, uint32_t nf, uint32_t ni, void* stream);
/* Cooperative launch of k_cycles over `blocks` blocks (from cyclesGrid). */
void launchCycles(const CycleArgs& args, unsigned blocks, void* stream);
/* The co-resident grid (one block per SM) and the per-block list capacity
 * (the most neurons one block updates in a cycle). */
void cyclesGrid(uint32_t totalWarps, unsigned* blocks, uint32_t* listCap);
void launchApplyStdp(const NetDev& net, const StdpRule& rule, int32_t reward, uint64_t nrcm, uint64_t cycleNow,
		void* stream);
void launchNrandProbe(const uint32_t* u1, const uint32_t* u2, float* out, size_t n,
		const uint32_t* sinTab, const uint32_t* logTab, void* stream);
void launchLibmEval(float* sinOut, float* logOut, const uint32_t* sinTab, const uint32_t* logTab, void* stream);
int smCount();

} // namespace nemo_b200

#endif
