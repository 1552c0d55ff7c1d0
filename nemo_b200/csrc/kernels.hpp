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
 * The step path is one persistent cooperative kernel (k_cycles) over one
 * block per SM, with one grid barrier per cycle. Block b owns a contiguous
 * range of 32-neuron warps (NetDev::ownStart): it updates them, and it alone adds spikes
 * into their current slots, which it keeps in shared memory for the whole
 * launch (or in global memory when they do not fit). The forward matrix is
 * partitioned to match: region b holds, source by source, the synapses of
 * delay >= 2 whose target block b owns; the delay-1 synapses follow, grouped
 * by source. Phase t:
 *   - neuron update of cycle t from slot t mod Q plus the delay-1 inbox of
 *     cycle t: firing history, bitmap, the fired and post-spiking lists of
 *     cycle t; each fired neuron's delay-1 synapses are added at once into
 *     the inbox of cycle t+1 (global reductions; 5% of the synapses for
 *     delays U{1..20}); overlapped with
 *   - the gather of cycle t-1: every block reads the fired sources of cycle
 *     t-1 (all blocks' lists) and, for each, its segment of region b, adding
 *     each weight of delay d >= 2 into slot (t-1+d) mod Q of the target (E or
 *     I by sign), and the STDP accumulation of cycle t-1 over all blocks'
 *     post-spiking targets, dealt out over the grid as entries of at most
 *     STDP_ITEM synapses (a target's plastic synapses in consecutive runs).
 *     Together the inbox and the gather are the reference's deliverSpikes at
 *     cycle t0+d (src/nemo/cpu/Simulation.cpp:259-308);
 *   - grid barrier.
 * A final phase gathers and learns for the last cycle, so that between
 * launches every spike fired is in the current slots. Integer sums are exact
 * in any order, so the result is bit-identical to the CPU reference. */

#include <cstdint>
#include <vector>

#include <vector_types.h>

namespace nemo_b200 {

const int MAX_GROUPS = 8;

/* most blocks of the step kernel (static shared prefix arrays) */
const uint32_t MAX_BLOCKS = 256;
/* forward synapses per applyStdp launch: consecutive owner blocks are grouped
 * until their regions hold this many (128 MB of records) */
const uint64_t APPLY_GROUP_SYNAPSES = uint64_t(1) << 24;
/* plastic synapses per lane in one applyStdp work item */
const uint32_t APPLY_PER_LANE = 4;
/* forward records a gather lane loads per round (a unit of 32 sources of
 * about 7 records each in a block's region takes one or two rounds) */
const int GATHER_PER_LANE = 4;
/* plastic synapses a lane visits in one STDP accumulation entry (an entry is
 * a run of at most STDP_ITEM synapses of one post-spiking target) */
const uint32_t STDP_PER_LANE = 4;
const uint32_t STDP_ITEM = 32 * STDP_PER_LANE;
/* the shortest run an STDP entry may be given (NetDev::stdpRun, chosen by
 * the autotuner from STDP_ITEM and this); the lists are sized for it */
const uint32_t STDP_RUN_MIN = 64;
/* stimulus entries of each kind a one-cycle step carries in its kernel
 * parameters (CycleArgs::inlineF / inlineI) */
const uint32_t INLINE_STIM_MAX = 32;
/* shared memory the step kernel may use for current slots */
const uint32_t SMEM_ACC_LIMIT = 200 * 1024;

struct NetDev {
	uint32_t nDev;          /* device neurons, multiple of 32 */
	uint32_t nWords;        /* nDev / 32 */
	uint32_t slots;         /* current slots: maxDelay + 1 (cycle t uses slot t mod slots) */
	int acc32;              /* int32 accumulators (proven not to overflow), else int64 */
	uint32_t ringMask;      /* firing-ring cycles - 1 */
	uint32_t fbits;         /* fractional bits of the Q(31-f).f weights */
	int deliver;            /* 0 when no delay is deliverable (max delay 64) */

	/* ownership: block b owns the neuron warps [ownStart[b], ownStart[b+1])
	 * (relative to warpBase; contiguous, split by the warps' update cost,
	 * cyclesPlan); ownWarps is the most any block owns */
	uint32_t blocks;
	uint32_t threads;       /* threads per block of the step kernel: 1024, 512 or 256 */
	uint32_t ownWarps;
	const uint32_t* ownStart;   /* [blocks + 1] */
	/* first warp of the owned range: 0, or in a sharded simulation the
	 * shard's first warp (block b owns warps warpBase + ownStart[b]...) */
	uint32_t warpBase;
	int smemAcc;            /* current slots of the owned neurons in shared memory */

	/* forward connectivity. Delays >= 2: the owner blocks form `groups`
	 * consecutive block groups (group g: blocks [groupFirst[g],
	 * groupFirst[g + 1])); the synapses whose target a block of group g
	 * owns follow one another in group order, inside a group by source, for
	 * a source by owner block, for a (source, block) pair in insertion order.
	 * The segment of (source s, block b) is bucket
	 *   k = groupFirst[g] * nDev + s * (blocks of g) + (b - groupFirst[g])
	 * = [segOff[k], segOff[k + 1]) (absolute positions): the buckets of one
	 * source in one group are consecutive, so a fired source's synapses in a
	 * group are one contiguous chunk, and its bucket starts for all the
	 * group's blocks share a line. segOff has blocks * nDev + 1 entries.
	 * Delay 1, by source: [d1Base + d1Start[s], d1Base + d1Start[s+1]) */
	uint2* fcm;                    /* {target << 6 | (delay - 1), int32 weight} */
	const uint32_t* segOff;        /* [blocks * nDev + 1] */
	uint32_t groups;
	const uint32_t* groupFirst;    /* [groups + 1] */
	const uint32_t* groupOf;       /* [blocks] the group of each block */
	/* the chunk of source s in group g: [srcChunk[s * groups + g],
	 * srcChunk[(s + 1) * groups + g]) ((nDev + 1) * groups entries, derived
	 * from segOff by launchSourceChunks) */
	const uint32_t* srcChunk;
	const uint32_t* outDegree;     /* [nDev] synapses per source */
	const uint32_t* d1Start;       /* [nDev + 1] */
	uint64_t d1Base;
	void* inbox;                   /* [2][nDev][2] delay-1 arrivals by cycle parity (as acc) */

	void* acc;                     /* [slots][nDev][2] E, I current of a future cycle (int32 or int64) */
	uint64_t* rf;                  /* [2][nDev] firing history, bit 0 = last cycle */
	uint32_t* firedRing;           /* [ring][nWords] firing bitmaps by cycle */
	unsigned long long* eventsRing;/* [ring] synaptic events (fired x out-degree) */
	uint32_t* firedCountRing;      /* [ring] */
	float* ext;                    /* [nDev] external current, cleared after use */
	float* noise;                  /* [2][nDev] Izhikevich noise of the next cycle, by cycle parity */
	/* resident stepping: [2][nDev] the generator state after the next cycle's draw, by cycle
	 * parity, drawn ahead without advancing the neuron's generator (which the next cycle's
	 * update advances to it, if that cycle comes) */
	uint4* rngAhead;
	uint32_t* fstim;               /* [nWords] firing stimulus, cleared after use */

	/* per-cycle lists by cycle parity and block, with their lengths
	 * [2][blocks]: fired sources (device indices), [2][blocks][ownWarps * 32],
	 * and the STDP entries of post-spiking targets, [2][blocks][postStride]:
	 * reverse-matrix runs {first, count}, count in [1, stdpRun] */
	uint32_t* firedList;
	uint32_t* firedCnt;
	uint2* postList;
	uint32_t* postCnt;
	uint32_t postStride;           /* entries of a block's list: the most its neurons can make */
	uint32_t stdpRun;              /* synapses of a full STDP entry: STDP_RUN_MIN .. STDP_ITEM, multiple of 32 */

	/* STDP (reverse connectivity of plastic synapses, grouped by target) */
	int stdp;
	uint32_t postShift;            /* bit of the history that triggers STDP */
	uint32_t applyChunks;          /* (32 x APPLY_PER_LANE)-synapse chunks per target */
	const uint32_t* rcmStart;      /* [nDev + 1] (fewer than 2^32 synapses) */
	const uint32_t* rcmSrcDelay;   /* source << 6 | (delay - 1) */
	const uint32_t* rcmForward;    /* index into fcm, ascending within a target */
	int32_t* rcmAcc;
	/* the plastic weights in reverse order, a copy of the forward records'
	 * weights that applyStdp reads (coalesced) and writes with them */
	int32_t* rcmWeight;

	/* glibc-matching correction tables (libm_match.cuh) */
	const uint32_t* sinTab;
	const uint32_t* logTab;
	/* expf exceptions (libm_tables.hpp ExpExceptions) as the hash of
	 * libm::exp_lookup: slots, log2 of their count, probe bound (0: no
	 * table), and the largest libm::exp_midpoint_units of an exception */
	const uint64_t* expSlots;
	uint32_t expBits;
	uint32_t expProbe;
	uint32_t expNear;

	/* sharded simulation: the fired sources other shards own, by cycle
	 * parity ([2][nDev], counts [2]), gathered like a block's fired list;
	 * null when the simulation owns every neuron */
	uint32_t* remoteList;
	uint32_t* remoteCnt;

	/* cumulative counters: [0] synapses pushed, [1] STDP synapse visits,
	 * [2] neurons fired, [3] synaptic events (fired x out-degree) */
	unsigned long long* stats;

	/* grid barrier: [0] arrivals since the simulation was created (every
	 * block adds 1 at every barrier), [1] the arrival count when the current
	 * launch started (written by block 0 at the end of each launch), [2]
	 * error (timeout) */
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
	uint32_t shift;         /* neuron i at device index devBase + (i << shift):
	                         * HH neurons take 8 lanes each (shift 3), the
	                         * other models one */
	const uint32_t* extFired;  /* a plugin model's firing bits of the cycle
	                            * (bit i % 32 of word i / 32), written by the
	                            * plugin before the update; null otherwise */
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

/* A resident step kernel's command (resident stepping, CycleArgs::cmd).
 *
 * In host memory mapped into the device, as 16-byte chunks {seq, three
 * payload words}: the host writes each chunk's payload, then its seq. Block
 * 0's first warp reads all chunks at once (one read across the bus per try)
 * and takes the command when every chunk it needs carries the command's
 * number; a 16-byte read of one cache line sees the line at one instant, so a
 * chunk with the new number has the new payload. Payload: op, nf, ni, then
 * nf firing-stimulus device indices, ni current-stimulus device indices
 * (unique) and ni currents (float bits); at most RESIDENT_CHUNKS chunks.
 *
 * In device memory (ResidentCmd), block 0's copy for the other blocks, its
 * number written last. */
const uint32_t RESIDENT_STEP = 1;
const uint32_t RESIDENT_EXIT = 2;
const uint32_t RESIDENT_CHUNKS = 32;
struct ResidentChunk {
	uint32_t seq;
	uint32_t w[3];
};
struct ResidentHostCmd {
	ResidentChunk c[RESIDENT_CHUNKS];
};
struct ResidentCmd {
	uint32_t seq;           /* command number, written last */
	uint32_t op;            /* RESIDENT_STEP or RESIDENT_EXIT */
	uint32_t nf, ni;        /* stimulus entries (<= INLINE_STIM_MAX each) */
	uint32_t f[INLINE_STIM_MAX];    /* firing stimulus, device indices */
	uint32_t i[INLINE_STIM_MAX];    /* current stimulus, device indices (unique) */
	float cur[INLINE_STIM_MAX];
};

struct CycleArgs {
	NetDev net;
	StdpRule rule;
	GroupDev groups[MAX_GROUPS];
	uint32_t groupWarp[MAX_GROUPS + 1];  /* prefix of 32-neuron warps per group */
	int ngroups;
	uint64_t firstCycle;
	uint32_t cycles;
	/* bit 0: the first phase also gathers and learns for cycle
	 * firstCycle - 1 (left pending by the previous launch); bit 1: no
	 * trailing gather phase (the launch leaves its last cycle pending).
	 * 0 for the unsharded simulation; a sharded step is one update phase,
	 * its flush one gather phase (cycles 0, carry 1). */
	uint32_t carry;
	/* run on the current slots in global memory even when the simulation
	 * keeps them in shared memory across a launch (the same [slots][nDev]
	 * array the shared copy is loaded from and spilled to): a launch of one
	 * phase saves the copy in and out */
	int globalAcc;
	/* a step's output in mapped host memory, null otherwise: word 0 is set to
	 * 1 when a grid barrier timed out (the host zeroes it first); word 1 the
	 * count of the simulation's warps that fired in the cycle, then that many
	 * {fired word, device warp} pairs in warp order (only the words that are
	 * not 0 cross to the host). The block that finishes the cycle's update
	 * last (arrivals counted in NetDev::barrier[3]) writes the list from the
	 * cycle's row of the firing ring */
	uint32_t* hostWords;
	/* a one-cycle step's stimulus when it is short (device indices; the
	 * owner warp of each neuron applies it before the update), in place of
	 * k_stimulus: firing stimulus inlineF[inlineNf], current stimulus
	 * inlineI[inlineNi] with inlineCur (unique indices) */
	uint32_t inlineNf;
	uint32_t inlineNi;
	uint32_t inlineF[INLINE_STIM_MAX];
	uint32_t inlineI[INLINE_STIM_MAX];
	float inlineCur[INLINE_STIM_MAX];
	unsigned long long timeoutNs;        /* grid-barrier wait limit */
	/* when set, the first cycle is read from here instead of firstCycle and
	 * advanced by the launch (launches replayed from a CUDA graph) */
	uint64_t* cycleCounter;
	/* resident stepping: when cmd is set, the launch runs one update phase
	 * per command instead of `cycles` phases. The first command (seq
	 * firstSeq) is this launch's inline stimulus; after each phase the block
	 * that writes the step list writes the command's seq into doneWords[0]
	 * (mapped host memory) after it, and block 0 waits for command seq + 1 in
	 * *cmd (mapped host memory) for at most idleNs and copies it to
	 * bcast[(phase + 1) & 1] (device), where the other blocks wait for it.
	 * The host issues a command only after the done word has come, which
	 * follows every block's phase, so no grid barrier separates the phases. An exit
	 * command, or no command within idleNs, ends the launch, which leaves its
	 * last cycle pending (as carry bit 1) and writes exitInfo = (last seq done
	 * << 1) | 1 (mapped host memory). */
	const ResidentHostCmd* cmd;
	ResidentCmd* bcast;
	uint32_t* doneWords;
	uint32_t* exitInfo;
	uint32_t firstSeq;
	unsigned long long idleNs;
	/* optional phase trace (%globaltimer ns), [cycles + 1][block][20]: phase
	 * start, (unused), last update warp done (0 when the block updates
	 * nothing), all work done, barrier passed; the summed durations of the
	 * block's gather units and STDP units, and their counts; over the update
	 * warps the summed time to their model's result, their summed update
	 * time and their count, the summed time of the fired warps' part after
	 * their lists (delay-1 push, prefetches) and their count; the summed
	 * durations of the noise units and their count; the time the block's
	 * last unit was taken, the summed times from the phase start at which its
	 * warps left the unit loop and their count, the time its last unit ended */
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
#ifdef __CUDACC__
#define NEMO_HD __host__ __device__
#else
#define NEMO_HD
#endif

/* First neuron warp owned by block b, and the block owning neuron warp w */

/* Cooperative launch of k_cycles (grid, block size and shared memory from
 * args.net). */
void launchCycles(const CycleArgs& args, void* stream);
/* The step kernel's grid (one block per SM, at most MAX_BLOCKS and at most
 * one per neuron warp; 0 when the kernel cannot be resident) and the split of
 * the neuron warps over its blocks: contiguous ranges of about equal summed
 * cost (warpCost[w]: the update cost of warp w), ownStart[blocks + 1]; the
 * most warps a block owns, and whether the owned current slots fit in shared
 * memory. */
void cyclesPlan(const std::vector<uint32_t>& warpCost, uint32_t slots, bool acc32, uint32_t* blocks,
		std::vector<uint32_t>* ownStart, uint32_t* ownWarps, bool* smemAcc);
/* applyStdp over target groups [groupTargets[g], groupTargets[g+1]), one
 * launch per group (groups of owner blocks, see APPLY_GROUP_SYNAPSES);
 * skipZero when every plastic weight is within its bounds (k_apply_stdp) */
void launchApplyStdp(const NetDev& net, const StdpRule& rule, int32_t reward, uint64_t cycleNow,
		const uint32_t* groupTargets, uint32_t groups, bool skipZero, void* stream);
void launchNrandProbe(const uint32_t* u1, const uint32_t* u2, float* out, size_t n,
		const uint32_t* sinTab, const uint32_t* logTab, void* stream);
void launchLibmEval(float* sinOut, float* logOut, const uint32_t* sinTab, const uint32_t* logTab, void* stream);
/* device expf (glibc-matching) of the floats with bits [first, first + n) */
void launchExpEval(uint32_t first, uint32_t n, float* out, const NetDev& net, void* stream);
/* fill net.srcChunk from net.segOff (construction) */
void launchSourceChunks(const NetDev& net, uint32_t* srcChunk, void* stream);
/* sharded simulation: the remote firing of cycle t (k_shard_inject) */
void launchShardInject(const NetDev& net, uint64_t t, const uint32_t* allWords, uint32_t ownLo, uint32_t ownHi,
		void* stream);
/* The currents of cycle `cycle` of device neurons devBase .. devBase +
 * count - 1 (their current slot plus their delay-1 inbox, saturated and
 * converted), into E[count] and I[count], for a plugin model; not cleared
 * (the cycle's update clears them). */
void launchExportCurrents(const NetDev& net, uint32_t devBase, uint32_t count, uint64_t cycle, float* E, float* I,
		void* stream);

/* counts of mismatches [3] (zeroed by the caller) of the HH constant divisions */
void launchHhDivCheck(unsigned long long* bad, void* stream);
int smCount();

} // namespace nemo_b200

#endif
