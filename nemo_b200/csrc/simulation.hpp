#ifndef NEMO_B200_SIMULATION_HPP
#define NEMO_B200_SIMULATION_HPP

/* The B200 simulation backend: the role of the reference's
 * nemo::SimulationBackend implementations (src/nemo/SimulationBackend.hpp:
 * 45-147, cpu/Simulation.cpp, cuda/Simulation.cpp), with the per-cycle work
 * done by the persistent kernel of kernels.cu. */

#include <chrono>
#include <cstdint>
#include <unordered_map>
#include <vector>

#include "kernels.hpp"
#include "network.hpp"
#include "plugin.hpp"

namespace nemo_b200 {

/* One shard of a sharded simulation: shard `rank` of `world` owns the
 * device warps [warpLo, warpHi) (contiguous, equal counts of warps) and
 * holds the synapses whose target it owns; maxDelay is the whole network's. */
/* the step kernel's shape chosen by the autotuner */
struct AutotuneShape {
	unsigned threads;     /* threads per block */
	unsigned stdpRun;     /* synapses of a full STDP work entry */
};

struct ShardSpec {
	unsigned rank = 0;
	unsigned world = 1;
	uint32_t warpLo = 0;
	uint32_t warpHi = 0;
	uint32_t totalWarps = 0;
	unsigned maxDelay = 0;
};

/* Shard `rank` of `world` of a whole network: its owned warp range and the
 * network it builds (every neuron, the synapses to its own neurons). The
 * device layout is the simulation's: types in registration order, each
 * padded to whole warps, Hodgkin-Huxley neurons eight lanes apart. */
Network shardNetwork(const Network& net, unsigned rank, unsigned world, ShardSpec* spec);

/* The warps shard `rank` of `world` owns out of `totalWarps`: sizes differ by
 * at most one, lower ranks take the extra ones. */
void shardWarps(uint32_t totalWarps, unsigned rank, unsigned world, uint32_t* lo, uint32_t* hi);

class Simulation {
public:
	Simulation(const Network& net, const Configuration& conf, const ShardSpec* shard = nullptr);
	~Simulation();

	/* End this simulation's resident step launch, if any (every call but
	 * step() does it first; a resident launch of another simulation on the
	 * same device does it too) */
	void stopResident();

	/* One cycle with stimulus; returns the fired neurons (user indices) in
	 * ascending simulation order (src/nemo/nemo_c.cpp:439-461). */
	const std::vector<unsigned>& step(const unsigned* fstim, size_t nf,
			const unsigned* inidx, const float* icur, size_t ni);

	/* The same cycle as step(), without allocating host or device memory:
	 * stimulus staged through the module-static scratch (at most
	 * NOALLOC_STIM_MAX entries of each kind), fired neurons written to the
	 * caller's array, which must hold neuronCount() entries. The first call
	 * on a device looks up the scratch address. Calls on the same device must
	 * not overlap. */
	size_t stepNoAlloc(const unsigned* fstim, size_t nf, const unsigned* inidx, const float* icur, size_t ni,
			unsigned* firedOut, size_t firedCapacity);

	/* Device-resident run of `cycles` cycles without stimulus in one
	 * persistent launch (for a network with plugin models, one launch
	 * sequence per cycle, queued without waiting); per-cycle fired counts
	 * and synaptic events (fired x out-degree) are returned when the
	 * pointers are non-null. */
	void run(unsigned cycles, uint32_t* firedCounts, uint64_t* events);

	/* Fired neurons of one of the last cycles run (device firing ring). */
	const std::vector<unsigned>& firedAt(uint64_t cycle);

	void applyStdp(float reward);

	/* A shard's cycle, in two calls. shardStep: stimulus for the neurons this
	 * shard owns (entries for other shards' neurons are skipped), the update
	 * of its neurons, and the gathering and learning of the previous cycle;
	 * the fired words of its own warps are written to localWords (host).
	 * shardDeliver: every warp's fired words of that cycle (host, from all
	 * shards) bring the other shards' firing in; returns all fired neurons
	 * (user indices). The cycle's own gathering waits for the next step,
	 * or for applyStdp. */
	void shardStep(const unsigned* fstim, size_t nf, const unsigned* inidx, const float* icur, size_t ni,
			uint32_t* localWords);
	const std::vector<unsigned>& shardDeliver(const uint32_t* allWords);
	/* The same cycle with the fired words kept in device memory and nothing
	 * waited for on the host: shardStepAsync queues the step and a copy of
	 * the shard's own words into localDev (device, shard().warpHi -
	 * warpLo words), then makes `stream` (a cudaStream_t, NULL: the legacy
	 * default stream; e.g. the stream a collective is queued on) wait for
	 * that copy. shardDeliverAsync makes the simulation's stream wait for
	 * `stream`'s work queued so far and then reads allDev (device, every
	 * warp's words). The cycle's fired neurons are read with firedAt. */
	void shardStepAsync(const unsigned* fstim, size_t nf, const unsigned* inidx, const float* icur, size_t ni,
			uint32_t* localDev, void* stream);
	void shardDeliverAsync(const uint32_t* allDev, void* stream);
	/* make `stream` wait for the work queued on the simulation's stream */
	void streamWait(void* stream);
	const ShardSpec& shard() const { return m_shard; }

	float getNeuronState(unsigned gidx, unsigned var);
	float getNeuronParameter(unsigned gidx, unsigned param) const;
	float getMembranePotential(unsigned gidx);
	void setNeuron(unsigned gidx, unsigned nargs, const float* args);
	void setNeuronState(unsigned gidx, unsigned var, float val);
	void setNeuronParameter(unsigned gidx, unsigned param, float val);

	const std::vector<synapse_id>& getSynapsesFrom(unsigned source);
	unsigned getSynapseTarget(synapse_id id) const;
	unsigned getSynapseDelay(synapse_id id) const;
	float getSynapseWeight(synapse_id id);
	void getWeights(const synapse_id* ids, size_t n, float* out);
	unsigned char getSynapsePlastic(synapse_id id) const;

	unsigned long elapsedWallclock() const;
	unsigned long elapsedSimulation() const { return (unsigned long) (m_cycle - m_timerBase); }
	void resetTimer();

	uint64_t cycle() const { return m_cycle; }
	size_t synapseCount() const { return m_nsyn; }
	unsigned neuronCount() const { return m_nNeurons; }
	void synchronize();

	/* device-side probe of the noise generator (tests) */
	void nrandProbe(const uint32_t* u1, const uint32_t* u2, float* out, size_t n);

	/* Evaluate the device sinf/logf on all reachable noise inputs and count
	 * the results that differ from host glibc (tests; expected 0). */
	uint64_t libmCheck();

	/* Evaluate the device expf of the HH model on every float in [-104, 89]
	 * and count the results that differ from host glibc (tests; expected 0). */
	uint64_t expfCheck();

	/* Device-timed throughput loop: `steps` x (one persistent launch of
	 * `cyclesPerStep` cycles, then applyStdp(reward) if apply), bracketed by
	 * CUDA events on the simulation's stream. out: [0] device ms, [1] neurons
	 * fired, [2] synaptic events generated, [3] synapses pushed. */
	void timedSteps(unsigned steps, unsigned cyclesPerStep, bool apply, float reward, double out[4]);

	/* Device times of one persistent launch of `cycles` cycles and of one
	 * applyStdp, with the work they did. out: [0] step-kernel ms, [1] grid
	 * blocks, [2] 0, [3] synapses pushed, [4] neurons fired, [5] STDP synapse
	 * visits, [6] neuron updates, [7] applyStdp ms, [8] plastic synapses,
	 * [9] synaptic events generated. */
	void profile(unsigned cycles, float reward, double out[10]);

	void readStats(uint64_t out[4]);
	unsigned applyLaunches() const { return m_stdpOn && m_nrcm ? unsigned(m_applyGroups.size() - 1) : 0u; }

	/* ---- batches of independent networks (Network::merge) ---- */
	void setBatch(std::vector<uint32_t> base) { m_batchBase = std::move(base); }
	size_t instances() const { return m_batchBase.empty() ? 1 : m_batchBase.size() - 1; }
	/* Fired neurons of every instance at `cycle` (one of the last cycles):
	 * instance-local user indices, instance after instance, each in its own
	 * simulation order, and the offsets of the instances [instances + 1]. */
	void batchFiredAt(uint64_t cycle, const std::vector<unsigned>** fired, const std::vector<size_t>** offsets);

	/* `cycles` cycles (<= the firing ring) as a CUDA graph of launches of
	 * at most `cyclesPerLaunch` cycles each, the first cycle of each launch
	 * read from a device counter; the graph is captured once per (cycles,
	 * cyclesPerLaunch, block size, timer base) and replayed. *usedGraph = 0
	 * when the device refused the capture and the launches ran directly. */
	void runGraph(unsigned cycles, unsigned cyclesPerLaunch, int* usedGraph);

	/* Time `trialCycles` cycles with each shape of the step kernel's work:
	 * block size (1024, 512, 256 threads over the same partitions) and, with
	 * STDP, the synapses of a full STDP work entry (128, 64); the results
	 * are the same. Twice each, interleaved, and keep the fastest. The
	 * cycles are simulated (2 x candidates x trialCycles in all).
	 * autotuneShape: ms[3 r + k] the better device ms per cycle of size k
	 * and run length r. autotune: ms[k] the best of size k; returns the
	 * size. */
	unsigned autotune(unsigned trialCycles, double ms[3]);
	AutotuneShape autotuneShape(unsigned trialCycles, double ms[6]);

	/* bytes that crossed between host and device for nemo_step calls since
	 * the simulation was made: [0] to the device (stimulus), [1] to the
	 * host (the fired lists and their counts and flags) */
	void hostBytes(unsigned long long out[2]) const
	{
		out[0] = m_bytesIn;
		out[1] = m_bytesOut;
	}

	/* Phase timing of one traced persistent launch of `cycles` cycles, means
	 * over cycles in ns: [0] phase, [1] max / [2] mean block update with the
	 * delay-1 push, [3] max / [4] mean block work, [5] first start to last
	 * block done, [6] last arrival to mean barrier exit, [7] spread of block
	 * arrivals, [8] max / [9] mean block work after its update, [10] / [11]
	 * mean duration of a gather / STDP unit, [12] / [13] such units per block
	 * and cycle. */
	void trace(unsigned cycles, double out[24]);

private:
	struct Group {
		NeuronType type;
		uint32_t localBase;   /* contiguous simulation index of the first neuron */
		uint32_t devBase;     /* device index (multiple of 32) */
		uint32_t count;
		uint32_t shift = 0;   /* neuron i at devBase + (i << shift) (GroupDev) */
		std::vector<float> param;   /* host copy, [nParam][count] */
		std::vector<float> state;   /* host copy, [nState][count] */
		float* dParam = nullptr;
		float* dState = nullptr;
		uint4* dRng = nullptr;
		/* a plugin model (MODEL_EXTERNAL): its update, the currents it is
		 * given and the firing bits it writes, per cycle */
		const B200Plugin* plugin = nullptr;
		float* dExtE = nullptr;
		float* dExtI = nullptr;
		uint32_t* dExtFired = nullptr;
	};

	struct Aux {            /* per synapse, in per-source id order */
		uint32_t fcmPos;
		uint32_t target;    /* user index */
		uint8_t delay;
		uint8_t plastic;
	};

	uint32_t devIndex(unsigned gidx) const;
	Group& groupOfDev(uint32_t dev, uint32_t* i);
	const Group& groupOfDev(uint32_t dev, uint32_t* i) const;
	const Aux& aux(synapse_id id) const;
	/* a step's short stimulus, staged by stageStimulus for the next launchStep */
	struct InlineStim {
		uint32_t nf = 0, ni = 0;
		uint32_t f[INLINE_STIM_MAX];
		uint32_t i[INLINE_STIM_MAX];
		float cur[INLINE_STIM_MAX];
	};
	void launchBlock(uint64_t first, unsigned cycles, uint32_t carry = 0, bool globalAcc = false,
			uint32_t* hostWords = nullptr, const InlineStim* inl = nullptr);
	void launchStep();
	void stageStimulus(const unsigned* fstim, size_t nf, const unsigned* inidx, const float* icur, size_t ni,
			bool ownedOnly);
	void construct(const Network& net, const Configuration& conf, const ShardSpec* shard);
	void release();
	void notShard(const char* what) const;
	void notExternal(const char* what) const;
	void runPlugins();
	void pluginBatch(const Group& g, b200_neuron_batch* b) const;
	void launchApply(int32_t reward);
	bool owns(uint32_t dev) const { return dev / 32 >= m_shard.warpLo && dev / 32 < m_shard.warpHi; }
	void flushPending();
	void checkDeviceError();
	void syncStateToHost();
	void* alloc(size_t bytes);
	void decodeFired(const uint32_t* words, std::vector<unsigned>& out) const;
	/* the fired neurons of the last step from the kernel's per-block lists in
	 * mapped memory (CycleArgs::hostWords), in simulation order */
	template<class Emit> void decodeStepList(Emit emit);
	void decodeStepList(std::vector<unsigned>& out);

	unsigned m_nNeurons;
	uint32_t m_nDev;
	uint32_t m_maxDelay;
	uint32_t m_fbits;
	size_t m_nsyn;
	uint64_t m_nrcm;
	std::vector<Group> m_groups;
	std::unordered_map<uint32_t, uint32_t> m_g2d;  /* user index -> device index */
	/* the same as a table from user index m_g2dLo on, when the indices are
	 * compact enough (empty otherwise) */
	uint32_t m_g2dLo = 0;
	std::vector<uint32_t> m_g2dDense;
	/* device index of a user index, ~0u for none */
	uint32_t toDev(uint32_t gidx) const
	{
		if(!m_g2dDense.empty()) {
			const uint32_t k = gidx - m_g2dLo;
			return gidx >= m_g2dLo && k < m_g2dDense.size() ? m_g2dDense[k] : ~0u;
		}
		auto it = m_g2d.find(gidx);
		return it == m_g2d.end() ? ~0u : it->second;
	}
	/* repeated current-stimulus neurons within one call (stageStimulus) */
	std::vector<uint32_t> m_stimEpoch, m_stimEntry;
	uint32_t m_epoch = 0;
	std::vector<uint32_t> m_d2g;                   /* device index -> user index (~0: padding) */
	std::vector<int32_t> m_d2group;                /* device index -> group (-1: padding) */

	NetDev m_net;
	CycleArgs m_args;
	unsigned m_blocks;          /* grid of the persistent step kernel */
	std::vector<uint32_t> m_applyGroups;  /* applyStdp launch target ranges (prefix) */
	bool m_stdpOn;
	StdpRule m_rule;
	/* every plastic weight within its STDP bounds (then applyStdp leaves
	 * synapses with a zero accumulator alone); true after any applyStdp */
	bool m_weightsInRange = false;
	StdpFunction m_stdpFn;
	uint32_t m_ring;

	/* synapse queries */
	bool m_writeOnly;
	std::unordered_map<uint32_t, std::pair<size_t, uint32_t>> m_auxRange;
	std::vector<Aux> m_aux;
	std::vector<uint32_t> m_auxSid;   /* a shard's: each entry's per-source index (ascending per source) */
	std::vector<synapse_id> m_queried;
	std::vector<uint2> m_fcmHost;
	bool m_fcmHostValid;

	/* state */
	uint64_t m_cycle;          /* cycles simulated */
	uint64_t m_timerBase;
	bool m_stateDirty;
	std::chrono::steady_clock::time_point m_wallStart;

	void* m_stream;
	std::vector<void*> m_allocs;

	/* pinned staging */
	uint32_t* m_hWords;        /* one firing bitmap, then the barrier error word */
	uint32_t* m_stepWords = nullptr;    /* mapped: a step's error word and fired-word lists (CycleArgs::hostWords) */
	InlineStim m_inline;
	uint32_t* m_dStepWords = nullptr;   /* its device address */
	uint32_t* m_hStim;         /* fstim + istim indices */
	float* m_hCur;
	uint32_t* m_dStim;
	float* m_dCur;
	size_t m_stimCap;

	std::vector<unsigned> m_fired;

	int m_noallocDevice = -1;  /* device of the simulation, found on the first stepNoAlloc */
	int m_device = 0;          /* the device the simulation was built on */

	/* batch */
	std::vector<uint32_t> m_batchBase;
	std::vector<unsigned> m_batchFired;
	std::vector<size_t> m_batchOffsets;

	/* the last cycle's gathering and learning wait for the next step or a
	 * flush (one-cycle steps and shard steps) */
	bool m_pendingGather = false;
	/* one-cycle steps run on the global current slots (CycleArgs::globalAcc) */
	bool m_stepGlobalAcc = true;

	/* the network has plugin models: every cycle runs their updates
	 * between the current export and the step launch */
	bool m_external = false;

	/* sharded simulation */
	bool m_shardMode = false;
	ShardSpec m_shard;
	bool m_awaitDeliver = false;    /* the last cycle's remote firing has not come in */
	uint32_t* m_dAllWords = nullptr;

	/* resident stepping: nemo_step's cycles go to a step kernel that stays on
	 * the device and takes them from a command in mapped host memory
	 * (CycleArgs::cmd), instead of one launch and one synchronisation per
	 * call. Any other call first ends the resident launch (stopResident). */
	bool stepResident(const unsigned* fstim, size_t nf, const unsigned* inidx, const float* icur, size_t ni);
	bool mapInline(const unsigned* fstim, size_t nf, const unsigned* inidx, const float* icur, size_t ni);
	bool fitsCommand() const { return 3u + m_inline.nf + 2u * m_inline.ni <= 3u * RESIDENT_CHUNKS; }
	void launchResident(uint32_t seq);
	void claimResidentDevice();
	void releaseResidentDevice();
	bool m_resident = false;            /* a resident launch is on the stream */
	bool m_residentOn = true;           /* nemo_step may use resident stepping */
	uint32_t m_rseq = 0;                /* the last command number */
	/* bytes of the per-cycle steps' inputs and outputs across the bus:
	 * stimulus (resident command chunks, or the staged copies and kernel
	 * parameters) and the step lists read back (hostBytes) */
	uint64_t m_bytesIn = 0;
	uint64_t m_bytesOut = 0;
	ResidentHostCmd* m_rcmd = nullptr;  /* mapped host memory */
	ResidentHostCmd* m_dRcmd = nullptr; /* its device address */
	/* write command `seq` (op, and m_inline's stimulus for a step) into
	 * m_rcmd: each chunk's payload, then its number */
	void postCommand(uint32_t seq, uint32_t op);
	ResidentCmd* m_rbcast = nullptr;    /* device, [2] */
	uint32_t* m_rdone = nullptr;        /* mapped host memory: [blocks] done words, then the exit word */
	uint32_t* m_dRdone = nullptr;

	/* events ordering the simulation's stream with a caller's stream, and
	 * the end of the last staged stimulus copy (its pinned source is
	 * rewritten only after it) */
	void* m_evOut = nullptr;
	void* m_evIn = nullptr;
	void* m_evStaged = nullptr;
	bool m_stagedPending = false;
	void* event(void** ev);

	/* graph run */
	void destroyGraph();
	void* m_graphExec = nullptr;
	uint64_t* m_dCycleCounter = nullptr;
	uint64_t m_graphKey[4] = {0, 0, 0, 0};
	bool m_graphUsable = true;
};

/* The HH model's constant divisions against correctly rounded division on
 * the current device (kernels.cu k_hh_div_check): mismatches per divisor. */
void hhDivisionCheck(uint64_t mismatches[3]);

} // namespace nemo_b200

#endif
