/* Host orchestration of the B200 backend (see simulation.hpp).
 *
 * Construction compiles the network into the device layout of kernels.hpp
 * with linear-time counting sorts; error precedence follows the reference
 * (src/nemo/nemo.cpp:110-134, cpu/Simulation.cpp:36-82,
 * ConnectivityMatrix.cpp:65-93): empty network, STDP window vs. max delay,
 * max delay > 64, duplicate neurons, STDP constants, then the first invalid
 * synapse in synapse-iteration order (ascending source, then id). */

#include "simulation.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <random>
#include <sstream>
#include <thread>

#include "compile.hpp"
#include "libm_match.cuh"
#include "libm_tables.hpp"

namespace nemo_b200 {

static inline uint64_t shl64(uint64_t x, unsigned n) { return x << (n & 63); }

static inline cudaStream_t STREAM(void* s) { return static_cast<cudaStream_t>(s); }

/* src/nemo/fixedpoint.cpp:17-29 */
static int32_t
toFix(float f, unsigned fbits)
{
	if(std::abs(int(f)) >= 1 << (31 - fbits)) {
		std::ostringstream msg;
		msg << "Fixed-point overflow. Value " << f << " does not fit into fixed-point format Q"
			<< 31 - fbits << "." << fbits;
		throw std::runtime_error(msg.str());
	}
	return static_cast<int32_t>(f * (1 << fbits));
}

static bool
fitsFix(float f, unsigned fbits)
{
	return !(std::abs(int(f)) >= 1 << (31 - fbits));
}

/* networks of at least this many synapses build their matrices on the
 * device (NEMO_B200_DEVICE_BUILD_MIN overrides it; 0 builds every network
 * there) */
static size_t
deviceBuildMinSynapses()
{
	if(const char* env = getenv("NEMO_B200_DEVICE_BUILD_MIN")) {
		char* end = nullptr;
		const unsigned long long v = strtoull(env, &end, 10);
		if(end != env) return size_t(v);
	}
	return size_t(1) << 22;
}

static float
fixToFloat(int32_t v, unsigned fbits)
{
	return float(v) / float(1 << fbits);
}

void*
Simulation::alloc(size_t bytes)
{
	void* p = nullptr;
	/* 256 bytes of padding: the step kernel's L2 prefetches round ranges
	 * out to 16-byte boundaries */
	bytes += 256;
	NEMO_CUDA(cudaMalloc(&p, bytes));
	m_allocs.push_back(p);
	NEMO_CUDA(cudaMemsetAsync(p, 0, bytes, STREAM(m_stream)));
	return p;
}

Simulation::Simulation(const Network& net, const Configuration& conf, const ShardSpec* shard) :
	m_nNeurons(net.neuronCount()),
	m_nDev(0),
	m_maxDelay(shard ? shard->maxDelay : net.maxDelay()),
	m_fbits(conf.fractionalBits),
	m_nsyn(net.synapseCount()),
	m_nrcm(0),
	m_stdpOn(conf.hasStdp),
	m_stdpFn(conf.stdp),
	m_ring(1024),
	m_writeOnly(conf.writeOnlySynapses),
	m_fcmHostValid(false),
	m_cycle(0),
	m_timerBase(0),
	m_stateDirty(false),
	m_stream(nullptr),
	m_hWords(nullptr),
	m_hStim(nullptr),
	m_hCur(nullptr),
	m_dStim(nullptr),
	m_dCur(nullptr),
	m_stimCap(0)
{
	/* the destructor does not run for a constructor that throws: release
	 * what the construction allocated before passing the error on */
	try {
		construct(net, conf, shard);
	} catch(...) {
		release();
		throw;
	}
}

void
Simulation::construct(const Network& net, const Configuration& conf, const ShardSpec* shard)
{
	std::memset(&m_net, 0, sizeof(m_net));
	std::memset(&m_rule, 0, sizeof(m_rule));
	std::memset(&m_args, 0, sizeof(m_args));

	if(m_nNeurons == 0) {
		fail(NEMO_INVALID_INPUT, "Cannot create simulation from empty network");
	}
	if(m_stdpOn) {
		m_stdpFn.verifyDynamicWindowLength(m_maxDelay);
	}
	if(m_maxDelay > 64) {
		fail(NEMO_INVALID_INPUT, "The network has synapses with delay " + std::to_string(m_maxDelay)
				+ "ms. The B200 backend supports a maximum of 64 ms");
	}

	/* ---- neurons: simulation order = type registration order ---- */
	uint32_t local = 0, devPos = 0;
	std::vector<const std::vector<uint32_t>*> groupGidx;
	std::vector<const std::vector<uint64_t>*> groupSeedKey;
	for(size_t ngi = 0; ngi < net.groups.size(); ++ngi) {
		const NeuronGroup& ng = net.groups[ngi];
		uint32_t n = uint32_t(ng.gidx.size());
		if(n == 0) continue;
		if(ng.type.kind == MODEL_COUNT) {
			fail(NEMO_API_UNSUPPORTED, "The B200 backend has no kernel for neuron model " + ng.type.name
					+ " (a plugin model needs b200/lib" + ng.type.name + ".so beside its .ini)");
		}
		Group g;
		g.type = ng.type;
		if(ng.type.kind == MODEL_EXTERNAL) {
			if(shard) {
				fail(NEMO_API_UNSUPPORTED, "Shard: neuron model " + ng.type.name
						+ " is a plugin model; sharded simulations run built-in models only");
			}
			g.plugin = &loadB200Plugin(ng.type.b200Plugin);
			m_external = true;
		}
		g.localBase = local;
		g.devBase = devPos;
		g.count = n;
		/* an HH neuron's six exponentials per substep run on six lanes of
		 * its own eight (kernels.cu modelHH) */
		g.shift = ng.type.kind == MODEL_HH ? 3u : 0u;
		g.param.resize(size_t(ng.type.nParam) * n);
		g.state.resize(size_t(ng.type.nState) * n);
		for(unsigned p = 0; p < ng.type.nParam; ++p)
			std::copy(ng.param[p].begin(), ng.param[p].end(), g.param.begin() + size_t(p) * n);
		for(unsigned s = 0; s < ng.type.nState; ++s)
			std::copy(ng.state[s].begin(), ng.state[s].end(), g.state.begin() + size_t(s) * n);
		for(uint32_t i = 0; i < n; ++i) {
			if(!m_g2d.emplace(ng.gidx[i], devPos + (i << g.shift)).second) {
				fail(NEMO_INVALID_INPUT, "Duplicate neuron index " + std::to_string(ng.gidx[i]));
			}
		}
		m_groups.push_back(std::move(g));
		groupGidx.push_back(&ng.gidx);
		groupSeedKey.push_back(ngi < net.seedKey.size() ? &net.seedKey[ngi] : nullptr);
		local += n;
		devPos = uint32_t(roundUp(uint64_t(devPos) + (uint64_t(n) << m_groups.back().shift), 32));
	}
	m_nDev = std::max<uint32_t>(devPos, 32);
	if(shard) {
		/* the shard's synapses were chosen with this same layout */
		if(shard->totalWarps != m_nDev / 32 || shard->warpLo > shard->warpHi || shard->warpHi > m_nDev / 32
				|| shard->world == 0 || shard->rank >= shard->world) {
			fail(NEMO_LOGIC_ERROR, "Shard: the warp range does not match the network's device layout");
		}
		m_shardMode = true;
		m_shard = *shard;
	} else {
		m_shard.warpLo = 0;
		m_shard.warpHi = m_nDev / 32;
		m_shard.totalWarps = m_nDev / 32;
		m_shard.maxDelay = m_maxDelay;
	}
	const uint32_t warpLo = m_shard.warpLo;
	if(uint64_t(m_nDev) >= (uint64_t(1) << 26)) {
		fail(NEMO_API_UNSUPPORTED, "The B200 backend supports at most 2^26 neurons per simulation");
	}
	m_d2g.assign(m_nDev, ~0u);
	m_d2group.assign(m_nDev, -1);
	for(size_t gi = 0; gi < m_groups.size(); ++gi) {
		const Group& g = m_groups[gi];
		for(uint32_t i = 0; i < g.count; ++i) {
			m_d2g[g.devBase + (i << g.shift)] = (*groupGidx[gi])[i];
			m_d2group[g.devBase + (i << g.shift)] = int32_t(gi);
		}
	}
	/* dense user -> device table when the user indices are compact (kept:
	 * every step maps its stimulus through it) */
	uint32_t lo = ~0u, hi = 0;
	for(const auto& kv : m_g2d) { lo = std::min(lo, kv.first); hi = std::max(hi, kv.first); }
	if(uint64_t(hi) - lo + 1 <= std::max<uint64_t>(uint64_t(m_nNeurons) * 4, 1u << 20)) {
		m_g2dLo = lo;
		m_g2dDense.assign(size_t(hi) - lo + 1, ~0u);
		for(const auto& kv : m_g2d) m_g2dDense[kv.first - lo] = kv.second;
	}
	auto map = [&](uint32_t gidx) -> uint32_t { return toDev(gidx); };

	/* ---- STDP constants (src/nemo/StdpProcess.cpp:20-46) ---- */
	if(m_stdpOn) {
		m_rule.minE = toFix(m_stdpFn.minE, m_fbits);
		m_rule.maxE = toFix(m_stdpFn.maxE, m_fbits);
		m_rule.minI = toFix(m_stdpFn.minI, m_fbits);
		m_rule.maxI = toFix(m_stdpFn.maxI, m_fbits);
		for(size_t i = 0; i < m_stdpFn.prefire.size(); ++i) m_rule.fnPre[i] = toFix(m_stdpFn.prefire[i], m_fbits);
		for(size_t i = 0; i < m_stdpFn.postfire.size(); ++i) m_rule.fnPost[i] = toFix(m_stdpFn.postfire[i], m_fbits);
		unsigned nPre = unsigned(m_stdpFn.prefire.size());
		unsigned nPost = unsigned(m_stdpFn.postfire.size());
		m_rule.potentiation = m_stdpFn.potentiationBits();
		m_rule.depression = m_stdpFn.depressionBits();
		m_rule.prePostBits = shl64(~shl64(~uint64_t(0), nPre), nPost);
		m_rule.postPreBits = ~shl64(~uint64_t(0), nPost);
		m_rule.postPreWindow = nPost;
	}

	/* ---- synapse validation: first failure in iteration order ---- */
	const size_t S = m_nsyn;
	{
		size_t bad = S;
		int badKind = 0;
		for(size_t s = 0; s < S; ++s) {
			int kind = 0;
			if(map(net.src[s]) == ~0u) kind = 1;
			else if(map(net.tgt[s]) == ~0u) kind = 2;
			else if(!fitsFix(net.wgt[s], m_fbits)) kind = 3;
			if(kind && (bad == S || net.src[s] < net.src[bad]
						|| (net.src[s] == net.src[bad] && net.sid[s] < net.sid[bad]))) {
				bad = s;
				badKind = kind;
			}
		}
		if(bad != S) {
			if(badKind == 1) fail(NEMO_INVALID_INPUT, "Non-existing neuron index " + std::to_string(net.src[bad]));
			if(badKind == 2) fail(NEMO_INVALID_INPUT, "Non-existing neuron index " + std::to_string(net.tgt[bad]));
			toFix(net.wgt[bad], m_fbits); /* throws the overflow error */
		}
	}
	if(S >= (uint64_t(1) << 32)) {
		fail(NEMO_API_UNSUPPORTED, "The B200 backend supports at most 2^32 synapses per simulation");
	}

	/* ---- device: the step kernel's plan decides the forward layout ---- */
	if(conf.cudaDevice >= 0) {
		NEMO_CUDA(cudaSetDevice(conf.cudaDevice));
	}
	NEMO_CUDA(cudaGetDevice(&m_device));
	std::vector<uint32_t> dsrc(S), dtgt(S);
	std::vector<int32_t> wfx(S);
	std::vector<uint32_t> outDegree(m_nDev, 0);
	for(size_t s = 0; s < S; ++s) {
		dsrc[s] = map(net.src[s]);
		dtgt[s] = map(net.tgt[s]);
		wfx[s] = toFix(net.wgt[s], m_fbits);
		outDegree[dsrc[s]]++;
	}
	/* deliverable delays: the reference masks the history with
	 * ~(~0 << maxDelay), a shift evaluated modulo 64 on x86-64
	 * (src/nemo/cpu/Simulation.cpp:264): every delay up to 63 ms is
	 * delivered, and with a 64 ms synapse present none is */
	const bool deliver = S > 0 && m_maxDelay < 64;
	/* current slots: arrivals for cycle c go to slot c mod (maxDelay + 1);
	 * a slot is drained at its cycle before any spike for the cycle one
	 * revolution later can be added */
	const uint32_t slots = deliver ? m_maxDelay + 1 : 1;

	/* src/nemo/StdpProcess.cpp:129-137: a weight updatedWeight leaves alone
	 * when the change is 0 */
	if(m_stdpOn) {
		m_weightsInRange = true;
		for(size_t s = 0; s < S && m_weightsInRange; ++s) {
			if(!net.plastic[s]) continue;
			const int64_t w = wfx[s];
			if(w > 0) m_weightsInRange = w >= m_rule.minE && w <= m_rule.maxE;
			else if(w < 0) m_weightsInRange = w >= m_rule.maxI && w <= m_rule.minI;
		}
	}
	/* int32 accumulators are exact when no slot can leave the int32 range:
	 * a slot of target t only ever holds at most one arrival per incoming
	 * synapse, so it is bounded by the sum of its in-weights, taking each
	 * plastic weight at its STDP limit if that is larger */
	bool acc32 = true;
	{
		std::vector<int64_t> pos(m_nDev, 0), neg(m_nDev, 0);
		for(size_t s = 0; s < S; ++s) {
			int64_t w = wfx[s];
			if(m_stdpOn && net.plastic[s]) {
				if(w > 0) w = std::max<int64_t>(w, m_rule.maxE);
				else if(w < 0) w = std::min<int64_t>(w, m_rule.maxI);
			}
			if(w >= 0) pos[dtgt[s]] += w;
			else neg[dtgt[s]] += w;
		}
		for(uint32_t n = 0; n < m_nDev && acc32; ++n) {
			acc32 = pos[n] <= INT32_MAX && neg[n] >= INT32_MIN;
		}
	}

	/* update cost per owned warp: an HH warp (999 substeps of six exponentials
	 * over eight lanes per neuron) counts 2.5 times another model's, so that
	 * HH warps spread over more blocks while no block owns more warps than it
	 * has update warps in a mixed network of a few HH neurons per ten others */
	std::vector<uint32_t> warpCost(m_shard.warpHi - warpLo, 2u);
	for(const Group& g : m_groups) {
		if(g.type.kind != MODEL_HH) continue;
		const uint32_t w0 = g.devBase / 32, w1 = uint32_t((uint64_t(g.devBase) + (uint64_t(g.count) << g.shift) + 31) / 32);
		for(uint32_t w = std::max(w0, warpLo); w < std::min(w1, m_shard.warpHi); ++w) warpCost[w - warpLo] = 5u;
	}
	std::vector<uint32_t> ownStart;
	uint32_t ownWarps = 0;
	bool smemAcc = false;
	cyclesPlan(warpCost, slots, acc32, &m_blocks, &ownStart, &ownWarps, &smemAcc);
	/* owner block of each owned warp */
	std::vector<uint32_t> ownerOfWarp(warpCost.size(), 0);
	for(uint32_t b = 0; b + 1 < ownStart.size(); ++b) {
		for(uint32_t w = ownStart[b]; w < ownStart[b + 1]; ++w) ownerOfWarp[w] = b;
	}
	NEMO_CUDA(cudaGetLastError());
	if(m_blocks == 0) {
		fail(NEMO_CUDA_INVOCATION_ERROR, "The step kernel cannot be resident on this device");
	}
	const uint32_t B = m_blocks;
	const uint32_t ownN = ownWarps * 32;
	if(uint64_t(B) * m_nDev + m_nDev + 1 >= (uint64_t(1) << 32)) {
		fail(NEMO_API_UNSUPPORTED, "The B200 backend supports at most " + std::to_string((uint64_t(1) << 32) / (B + 1))
				+ " neurons per simulation on this device");
	}

	/* block groups of the forward matrix: consecutive owner blocks whose
	 * delay >= 2 synapses together stay within APPLY_GROUP_SYNAPSES (the
	 * records one applyStdp launch rewrites, kept in L2) */
	std::vector<uint32_t> groupFirst(1, 0), groupOf(B, 0);
	{
		std::vector<uint64_t> perBlock(size_t(B) + 1, 0);
		for(size_t s = 0; s < S; ++s) {
			if(net.dly[s] != 1) perBlock[size_t(ownerOfWarp[dtgt[s] / 32 - warpLo]) + 1]++;
		}
		for(uint32_t b = 0; b < B; ++b) perBlock[b + 1] += perBlock[b];
		for(uint32_t b = 0; b < B;) {
			uint32_t e = b + 1;
			while(e < B && perBlock[e + 1] - perBlock[b] <= APPLY_GROUP_SYNAPSES) ++e;
			for(uint32_t x = b; x < e; ++x) groupOf[x] = uint32_t(groupFirst.size() - 1);
			groupFirst.push_back(e);
			b = e;
		}
	}
	const uint32_t G = uint32_t(groupFirst.size() - 1);

	/* the simulation's stream; the device build of the layout runs on it */
	cudaStream_t stream;
	NEMO_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
	m_stream = stream;

	/* a large network builds its forward and reverse matrices on the
	 * device (compile.cu), a small one on the host below; the two builds
	 * are equal element for element */
	const bool onDevice = S >= deviceBuildMinSynapses() && layoutOnDevice(S, m_nDev, B);
	LayoutOut dev;
	if(onDevice) {
		LayoutIn li;
		li.S = S;
		li.nDev = m_nDev;
		li.blocks = B;
		li.warpLo = warpLo;
		li.ownedWarps = uint32_t(ownerOfWarp.size());
		li.stdp = m_stdpOn;
		li.wantFcmPos = !m_writeOnly;
		li.src = dsrc.data();
		li.tgt = dtgt.data();
		li.wfx = wfx.data();
		li.dly = net.dly.data();
		li.plastic = net.plastic.data();
		li.ownerOfWarp = ownerOfWarp.data();
		li.groupFirst = groupFirst.data();
		li.groupOf = groupOf.data();
		li.groups = G;
		buildLayoutOnDevice(li, [this](size_t bytes) { return alloc(bytes); }, &dev, m_stream);
	}

	/* ---- forward matrix: the synapses of delay >= 2 by block group, in a
	 * group by source, for a source by owner block of the target (bucket
	 * groupFirst[g] * nDev + source * blocks(g) + (b - groupFirst[g])), in
	 * insertion order within a bucket; then the delay-1 synapses grouped by
	 * source (pushed at firing) ---- */
	std::vector<uint32_t> segOff, d1Start;
	std::vector<uint2> fcm;
	std::vector<uint32_t> fcmPos;
	std::vector<uint32_t> synAt;   /* synapse at each forward position */
	uint64_t d1Base = 0;
	if(onDevice) {
		d1Base = dev.d1Base;
		fcmPos.swap(dev.fcmPos);
	} else {
		const size_t buckets = size_t(B) * m_nDev;
		auto bucket = [&](size_t s) -> size_t {
			const uint32_t b = ownerOfWarp[dtgt[s] / 32 - warpLo];
			const uint32_t g0 = groupFirst[groupOf[b]], bg = groupFirst[groupOf[b] + 1] - g0;
			return size_t(g0) * m_nDev + size_t(dsrc[s]) * bg + (b - g0);
		};
		segOff.assign(buckets + 1, 0);
		d1Start.assign(size_t(m_nDev) + 1, 0);
		fcm.resize(S);
		fcmPos.resize(S);
		synAt.resize(S);
		for(size_t s = 0; s < S; ++s) {
			if(net.dly[s] == 1) d1Start[dsrc[s] + 1]++;
			else segOff[bucket(s) + 1]++;
		}
		for(size_t k = 0; k < buckets; ++k) segOff[k + 1] += segOff[k];
		d1Base = segOff[buckets];
		for(uint32_t n = 0; n < m_nDev; ++n) d1Start[n + 1] += d1Start[n];
		std::vector<uint32_t> cursor(segOff.begin(), segOff.end() - 1);
		std::vector<uint32_t> d1Fill(d1Start.begin(), d1Start.end() - 1);
		for(size_t s = 0; s < S; ++s) {
			uint64_t pos;
			if(net.dly[s] == 1) {
				pos = d1Base + d1Fill[dsrc[s]]++;
			} else {
				pos = cursor[bucket(s)]++;
			}
			fcm[pos] = make_uint2((dtgt[s] << 6) | (net.dly[s] - 1), uint32_t(wfx[s]));
			fcmPos[s] = uint32_t(pos);
			synAt[pos] = uint32_t(s);
		}
	}

	/* applyStdp launches: one per block group, as target ranges (a
	 * target's plastic synapses of delay >= 2 all lie in its group's part
	 * of the forward matrix) */
	m_applyGroups.assign(1, warpLo * 32u);
	for(uint32_t g = 0; g < G; ++g) {
		m_applyGroups.push_back(std::min((warpLo + ownStart[groupFirst[g + 1]]) * 32u, m_nDev));
	}

	/* ---- reverse matrix of plastic synapses, grouped by target ---- */
	std::vector<uint32_t> rcmStart;
	std::vector<uint32_t> rcmSrcDelay, rcmForward;
	std::vector<int32_t> rcmWeight;
	uint64_t maxIn = 0;
	if(m_stdpOn && onDevice) {
		m_nrcm = dev.nrcm;
		maxIn = dev.maxIn;
	} else if(m_stdpOn) {
		rcmStart.assign(size_t(m_nDev) + 1, 0);
		for(size_t s = 0; s < S; ++s) if(net.plastic[s]) rcmStart[dtgt[s] + 1]++;
		for(uint32_t n = 0; n < m_nDev; ++n) {
			maxIn = std::max<uint64_t>(maxIn, rcmStart[n + 1]);
			rcmStart[n + 1] += rcmStart[n];
		}
		m_nrcm = rcmStart[m_nDev];
		rcmSrcDelay.resize(m_nrcm);
		rcmForward.resize(m_nrcm);
		rcmWeight.resize(m_nrcm);
		/* filled in forward order, so each target's synapses are sorted by
		 * their position in the forward matrix */
		std::vector<uint32_t> fill(rcmStart.begin(), rcmStart.end() - 1);
		for(size_t pos = 0; pos < S; ++pos) {
			size_t s = synAt[pos];
			if(!net.plastic[s]) continue;
			uint32_t j = fill[dtgt[s]]++;
			rcmSrcDelay[j] = (dsrc[s] << 6) | (net.dly[s] - 1);
			rcmForward[j] = uint32_t(pos);
			rcmWeight[j] = wfx[s];
		}
	}
	/* STDP entries: a post-spiking target's plastic synapses in runs of at
	 * most stdpRun; a block's list of one cycle holds at most the sum of its
	 * neurons' runs at the shortest run length */
	uint64_t postStride = 1;
	if(m_stdpOn) {
		std::vector<uint32_t> hostStart;
		const uint32_t* rs = rcmStart.data();
		if(onDevice) {
			hostStart.resize(size_t(m_nDev) + 1);
			NEMO_CUDA(cudaMemcpyAsync(hostStart.data(), dev.rcmStart, hostStart.size() * 4, cudaMemcpyDeviceToHost,
					STREAM(m_stream)));
			NEMO_CUDA(cudaStreamSynchronize(STREAM(m_stream)));
			rs = hostStart.data();
		}
		for(uint32_t b = 0; b < m_blocks; ++b) {
			uint64_t runs = 0;
			const uint32_t n0 = (warpLo + ownStart[b]) * 32u, n1 = (warpLo + ownStart[b + 1]) * 32u;
			for(uint32_t n = n0; n < n1; ++n) runs += (uint64_t(rs[n + 1] - rs[n]) + STDP_RUN_MIN - 1) / STDP_RUN_MIN;
			postStride = std::max(postStride, runs);
		}
	}
	if(uint64_t(m_blocks) * postStride >= (uint64_t(1) << 32)) {
		fail(NEMO_API_UNSUPPORTED, "The B200 backend supports at most 2^32 STDP entries in one cycle");
	}

	/* ---- synapse query data (src/nemo/ConnectivityMatrix.cpp:128-149) ---- */
	if(!m_writeOnly) {
		net.indexBySource();
		m_auxRange = net.m_srcRange;
		m_aux.resize(S);
		for(size_t k = 0; k < S; ++k) {
			size_t s = net.m_bySource[k];
			m_aux[k] = Aux{fcmPos[s], net.tgt[s], uint8_t(net.dly[s]), net.plastic[s]};
		}
		/* a shard holds some of a source's synapses: their ids keep the
		 * per-source index of the whole network */
		if(m_shardMode) {
			m_auxSid.resize(S);
			for(size_t k = 0; k < S; ++k) m_auxSid[k] = net.sid[net.m_bySource[k]];
		}
	}

	/* ---- device ---- */
	auto put = [&](const void* host, size_t bytes) -> void* {
		void* d = alloc(bytes);
		if(bytes) NEMO_CUDA(cudaMemcpyAsync(d, host, bytes, cudaMemcpyHostToDevice, stream));
		return d;
	};

	m_net.nDev = m_nDev;
	m_net.nWords = m_nDev / 32;
	m_net.slots = slots;
	m_net.acc32 = acc32 ? 1 : 0;
	m_net.ringMask = m_ring - 1;
	m_net.fbits = m_fbits;
	m_net.deliver = deliver ? 1 : 0;
	m_net.blocks = B;
	m_net.threads = 1024;
	m_net.ownWarps = ownWarps;
	m_net.ownStart = (const uint32_t*) put(ownStart.data(), ownStart.size() * 4);
	m_net.warpBase = warpLo;
	m_net.smemAcc = smemAcc ? 1 : 0;
	m_net.fcm = onDevice ? dev.fcm : (uint2*) put(fcm.data(), fcm.size() * 8);
	m_net.segOff = onDevice ? dev.segOff : (const uint32_t*) put(segOff.data(), segOff.size() * 4);
	m_net.groups = G;
	m_net.groupFirst = (const uint32_t*) put(groupFirst.data(), groupFirst.size() * 4);
	m_net.groupOf = (const uint32_t*) put(groupOf.data(), groupOf.size() * 4);
	{
		uint32_t* chunks = (uint32_t*) alloc((size_t(m_nDev) + 1) * G * 4);
		launchSourceChunks(m_net, chunks, m_stream);
		NEMO_CUDA(cudaGetLastError());
		m_net.srcChunk = chunks;
	}
	m_net.outDegree = (const uint32_t*) put(outDegree.data(), outDegree.size() * 4);
	m_net.d1Start = onDevice ? dev.d1Start : (const uint32_t*) put(d1Start.data(), d1Start.size() * 4);
	m_net.d1Base = d1Base;
	m_net.inbox = alloc(size_t(2) * m_nDev * (acc32 ? 8 : 16));
	m_net.acc = alloc(size_t(slots) * m_nDev * (acc32 ? 8 : 16));
	m_net.rf = (uint64_t*) alloc(size_t(2) * m_nDev * 8);
	m_net.firedRing = (uint32_t*) alloc(size_t(m_ring) * m_net.nWords * 4);
	m_net.eventsRing = (unsigned long long*) alloc(size_t(m_ring) * 8);
	m_net.firedCountRing = (uint32_t*) alloc(size_t(m_ring) * 4);
	m_net.ext = (float*) alloc(size_t(m_nDev) * 4);
	m_net.noise = (float*) alloc(size_t(2) * m_nDev * 4);
	m_net.rngAhead = (uint4*) alloc(size_t(2) * m_nDev * 16);
	m_net.fstim = (uint32_t*) alloc(size_t(m_net.nWords) * 4);
	m_net.stats = (unsigned long long*) alloc(4 * 8);
	m_net.barrier = (unsigned*) alloc(4 * 4);
	m_net.firedList = (uint32_t*) alloc(size_t(2) * B * ownN * 4);
	m_net.firedCnt = (uint32_t*) alloc(size_t(2) * B * 4);
	m_net.postList = (uint2*) alloc(size_t(2) * B * postStride * 8);
	m_net.postStride = uint32_t(postStride);
	m_net.stdpRun = STDP_ITEM;
	m_net.postCnt = (uint32_t*) alloc(size_t(2) * B * 4);
	if(m_shard.world > 1) {
		m_net.remoteList = (uint32_t*) alloc(size_t(2) * m_nDev * 4);
		m_net.remoteCnt = (uint32_t*) alloc(2 * 4);
	}
	m_net.stdp = m_stdpOn ? 1 : 0;
	m_net.applyChunks = uint32_t(std::max<uint64_t>(1, (maxIn + 32 * APPLY_PER_LANE - 1) / (32 * APPLY_PER_LANE)));
	if(m_stdpOn) {
		m_net.postShift = unsigned(m_stdpFn.postfire.size()) & 63u;
		if(onDevice) {
			m_net.rcmStart = dev.rcmStart;
			m_net.rcmSrcDelay = dev.rcmSrcDelay;
			m_net.rcmForward = dev.rcmForward;
			m_net.rcmWeight = dev.rcmWeight;
		} else {
			m_net.rcmStart = (const uint32_t*) put(rcmStart.data(), rcmStart.size() * 4);
			m_net.rcmSrcDelay = (const uint32_t*) put(rcmSrcDelay.data(), rcmSrcDelay.size() * 4);
			m_net.rcmForward = (const uint32_t*) put(rcmForward.data(), rcmForward.size() * 4);
			m_net.rcmWeight = (int32_t*) put(rcmWeight.data(), rcmWeight.size() * 4);
		}
		m_net.rcmAcc = (int32_t*) alloc(size_t(m_nrcm) * 4);
	}

	/* per-neuron RNG seeds by simulation index (src/nemo/RNG.cpp:39-62):
	 * outputs 4i..4i+3 of a default-seeded mt19937, reduced to [0, 2^31) by
	 * Boost's uniform_int (bucket size 2, i.e. >> 1) */
	std::mt19937 mt;
	/* a batch seeds each instance as if it were alone: a fresh generator per
	 * instance, outputs 4i..4i+3 for its simulation index i */
	std::vector<std::vector<uint4>> instanceSeeds;
	if(!net.seedKey.empty()) {
		std::vector<uint32_t> count;
		for(const auto& keys : net.seedKey) {
			for(uint64_t key : keys) {
				const uint32_t j = uint32_t(key >> 32), i = uint32_t(key);
				if(count.size() <= j) count.resize(j + 1, 0u);
				count[j] = std::max(count[j], i + 1);
			}
		}
		instanceSeeds.resize(count.size());
		for(size_t j = 0; j < count.size(); ++j) {
			std::mt19937 mi;
			instanceSeeds[j].resize(count[j]);
			for(uint32_t i = 0; i < count[j]; ++i) {
				uint32_t a = mi() >> 1, b = mi() >> 1, c = mi() >> 1, d = mi() >> 1;
				instanceSeeds[j][i] = make_uint4(a, b, c, d);
			}
		}
	}
	bool needTables = false;
	for(size_t gi = 0; gi < m_groups.size(); ++gi) {
		Group& g = m_groups[gi];
		g.dParam = (float*) put(g.param.data(), g.param.size() * 4);
		g.dState = (float*) put(g.state.data(), g.state.size() * 4);
		std::vector<uint4> seeds(g.count);
		const std::vector<uint64_t>* keys = groupSeedKey[gi];
		for(uint32_t i = 0; i < g.count; ++i) {
			if(keys) {
				const uint64_t key = (*keys)[i];
				seeds[i] = instanceSeeds[key >> 32][uint32_t(key)];
			} else {
				uint32_t a = mt() >> 1, b = mt() >> 1, c = mt() >> 1, d = mt() >> 1;
				seeds[i] = make_uint4(a, b, c, d);
			}
		}
		g.dRng = (uint4*) put(seeds.data(), seeds.size() * 16);
		needTables = needTables || g.type.kind == MODEL_IZHIKEVICH;
		if(g.plugin) {
			g.dExtE = (float*) alloc(size_t(g.count) * 4);
			g.dExtI = (float*) alloc(size_t(g.count) * 4);
			g.dExtFired = (uint32_t*) alloc(size_t((g.count + 31) / 32) * 4);
		}
	}
	bool needExp = false;
	for(const Group& g : m_groups) needExp = needExp || g.type.kind == MODEL_HH;
	if(needExp) {
		const ExpExceptions& e = expExceptions();
		m_net.expSlots = (const uint64_t*) put(e.slots.data(), e.slots.size() * 8);
		m_net.expBits = e.slotBits;
		m_net.expProbe = e.slotProbe;
		m_net.expNear = e.nearUnits;
	}
	if(needTables) {
		const LibmTables& t = libmTables();
		m_net.sinTab = (const uint32_t*) put(t.sinCodes.data(), t.sinCodes.size() * 4);
		m_net.logTab = (const uint32_t*) put(t.logCodes.data(), t.logCodes.size() * 4);
	}

	/* the persistent kernel's arguments, except the cycle range */
	if(m_groups.size() > size_t(MAX_GROUPS)) {
		fail(NEMO_API_UNSUPPORTED, "The B200 backend supports at most " + std::to_string(MAX_GROUPS)
				+ " neuron types per simulation");
	}
	m_args.net = m_net;
	m_args.rule = m_rule;
	m_args.ngroups = int(m_groups.size());
	m_args.groupWarp[0] = 0;
	for(size_t gi = 0; gi < m_groups.size(); ++gi) {
		const Group& g = m_groups[gi];
		m_args.groups[gi] = GroupDev{g.devBase, g.count, 0u, int(g.type.kind), g.dParam, g.dState, g.dRng, g.shift,
			g.dExtFired};
		m_args.groupWarp[gi + 1] = m_args.groupWarp[gi] + uint32_t(((uint64_t(g.count) << g.shift) + 31) / 32);
	}
	/* a grid barrier that waits this long has lost a block: give up */
	m_args.timeoutNs = 10ull * 1000 * 1000 * 1000;

	NEMO_CUDA(cudaMallocHost((void**) &m_hWords, size_t(m_net.nWords + 1) * 4));
	/* error word, count, at most one {word, warp} pair per warp */
	NEMO_CUDA(cudaHostAlloc((void**) &m_stepWords, (2 + 2 * size_t(m_net.nWords)) * 4, cudaHostAllocMapped));
	NEMO_CUDA(cudaHostGetDevicePointer((void**) &m_dStepWords, m_stepWords, 0));
	/* plugin models derive their initial state (b200_init_neurons) */
	for(const Group& g : m_groups) {
		if(g.plugin && g.plugin->init) {
			b200_neuron_batch b;
			pluginBatch(g, &b);
			b.cycle = 0;
			b.current_epsp = b.current_ipsp = nullptr;
			b.fstim = nullptr;
			b.fired = nullptr;
			const int rc = g.plugin->init(&b, m_stream);
			if(rc != 0) {
				fail(NEMO_CUDA_INVOCATION_ERROR, "Neuron model plugin " + g.plugin->path + ": b200_init_neurons: "
						+ cudaGetErrorString(cudaError_t(rc)));
			}
			/* the device state is ahead of the host copy */
			m_stateDirty = true;
		}
	}
	NEMO_CUDA(cudaStreamSynchronize(stream));
	m_wallStart = std::chrono::steady_clock::now();
}

Simulation::~Simulation()
{
	release();
}

void
Simulation::release()
{
	if(m_resident && m_rcmd) {
		/* end the resident launch without raising (destructor) */
		postCommand(++m_rseq, RESIDENT_EXIT);
		m_resident = false;
	}
	releaseResidentDevice();
	if(m_stream) cudaStreamSynchronize(STREAM(m_stream));
	destroyGraph();
	for(void** ev : {&m_evOut, &m_evIn, &m_evStaged}) {
		if(*ev) cudaEventDestroy(static_cast<cudaEvent_t>(*ev));
		*ev = nullptr;
	}
	m_stagedPending = false;
	for(void* p : m_allocs) cudaFree(p);
	m_allocs.clear();
	if(m_hWords) cudaFreeHost(m_hWords);
	if(m_stepWords) cudaFreeHost(m_stepWords);
	if(m_rcmd) cudaFreeHost(m_rcmd);
	if(m_rdone) cudaFreeHost(m_rdone);
	m_rcmd = m_dRcmd = nullptr;
	m_rdone = m_dRdone = nullptr;
	m_rbcast = nullptr;
	if(m_hStim) cudaFreeHost(m_hStim);
	if(m_hCur) cudaFreeHost(m_hCur);
	if(m_dStim) cudaFree(m_dStim);
	if(m_dCur) cudaFree(m_dCur);
	if(m_stream) cudaStreamDestroy(STREAM(m_stream));
	m_hWords = nullptr;
	m_stepWords = nullptr;
	m_dStepWords = nullptr;
	m_hStim = nullptr;
	m_hCur = nullptr;
	m_dStim = nullptr;
	m_dCur = nullptr;
	m_stream = nullptr;
}

uint32_t
Simulation::devIndex(unsigned gidx) const
{
	const uint32_t d = toDev(gidx);
	if(d == ~0u) {
		fail(NEMO_INVALID_INPUT, "Non-existing neuron index " + std::to_string(gidx));
	}
	return d;
}

Simulation::Group&
Simulation::groupOfDev(uint32_t dev, uint32_t* i)
{
	Group& g = m_groups.at(size_t(m_d2group.at(dev)));
	*i = (dev - g.devBase) >> g.shift;
	return g;
}

const Simulation::Group&
Simulation::groupOfDev(uint32_t dev, uint32_t* i) const
{
	const Group& g = m_groups.at(size_t(m_d2group.at(dev)));
	*i = (dev - g.devBase) >> g.shift;
	return g;
}

/* One persistent launch for cycles [first, first + cycles) */
void
Simulation::launchBlock(uint64_t first, unsigned cycles, uint32_t carry, bool globalAcc, uint32_t* hostWords,
		const InlineStim* inl)
{
	CycleArgs a = m_args;
	a.firstCycle = first;
	a.cycles = cycles;
	a.carry = carry;
	a.globalAcc = globalAcc ? 1 : 0;
	a.hostWords = hostWords;
	if(inl) {
		a.inlineNf = inl->nf;
		a.inlineNi = inl->ni;
		std::copy(inl->f, inl->f + inl->nf, a.inlineF);
		std::copy(inl->i, inl->i + inl->ni, a.inlineI);
		std::copy(inl->cur, inl->cur + inl->ni, a.inlineCur);
	}
	for(int gi = 0; gi < a.ngroups; ++gi) {
		a.groups[gi].timerBase = uint32_t(m_timerBase);
	}
	launchCycles(a, m_stream);
	NEMO_CUDA(cudaGetLastError());
}

/* The grid barrier gives up after its time limit and leaves an error word
 * instead of hanging the GPU; report it. */
void
Simulation::checkDeviceError()
{
	if(m_hWords[m_net.nWords] != 0) {
		fail(NEMO_CUDA_ASSERTION_FAILURE, "step kernel: a grid barrier timed out; the simulation state is invalid");
	}
}

void
Simulation::decodeFired(const uint32_t* words, std::vector<unsigned>& out) const
{
	/* two words at a time: nearly all are 0 at ordinary firing rates */
	out.resize(0);
	const uint32_t nw = m_net.nWords;
	uint32_t w = 0;
	for(; w + 1 < nw; w += 2) {
		uint64_t bits = uint64_t(words[w]) | (uint64_t(words[w + 1]) << 32);
		while(bits) {
			const uint32_t b = uint32_t(__builtin_ctzll(bits));
			bits &= bits - 1;
			out.push_back(m_d2g[size_t(w) * 32 + b]);
		}
	}
	for(; w < nw; ++w) {
		uint32_t bits = words[w];
		while(bits) {
			const uint32_t b = uint32_t(__builtin_ctz(bits));
			bits &= bits - 1;
			out.push_back(m_d2g[size_t(w) * 32 + b]);
		}
	}
}

/* The fired neurons of the last step from the list the kernel wrote into
 * mapped memory (CycleArgs::hostWords): {fired word, warp} pairs in warp
 * order, one contiguous run for the host to read. */
template<class Emit>
void
Simulation::decodeStepList(Emit emit)
{
	const uint32_t n = m_stepWords[1];
	const uint32_t* e = m_stepWords + 2;
	for(uint32_t k = 0; k < n; ++k) {
		const size_t w = e[2 * k + 1];
		uint32_t bits = e[2 * k];
		while(bits) {
			const uint32_t bit = uint32_t(__builtin_ctz(bits));
			bits &= bits - 1;
			emit(m_d2g[w * 32 + bit]);
		}
	}
}

void
Simulation::decodeStepList(std::vector<unsigned>& out)
{
	out.resize(0);
	decodeStepList([&out](unsigned g) { out.push_back(g); });
}

/* src/nemo/nemo_c.cpp:439-461 and cpu/Simulation.cpp:140-163: firing
 * stimulus, then current stimulus; an invalid index raises after the entries
 * before it have been applied. */
void
Simulation::stageStimulus(const unsigned* fstim, size_t nf, const unsigned* inidx, const float* icur, size_t ni,
		bool ownedOnly)
{
	cudaStream_t stream = STREAM(m_stream);
	/* the pinned buffers are the source of the last staged copy, which a
	 * call that did not wait for its step may still have queued */
	if(m_stagedPending) {
		NEMO_CUDA(cudaEventSynchronize(static_cast<cudaEvent_t>(m_evStaged)));
		m_stagedPending = false;
	}
	size_t need = nf + ni;
	if(need > m_stimCap) {
		/* the old buffers go first; a failed allocation leaves the ones
		 * not yet made null and the capacity 0, so that the next call
		 * allocates again and release() frees only what exists */
		cudaStreamSynchronize(stream);
		if(m_hStim) cudaFreeHost(m_hStim);
		if(m_hCur) cudaFreeHost(m_hCur);
		if(m_dStim) cudaFree(m_dStim);
		if(m_dCur) cudaFree(m_dCur);
		m_hStim = nullptr;
		m_hCur = nullptr;
		m_dStim = nullptr;
		m_dCur = nullptr;
		m_stimCap = 0;
		const size_t cap = std::max<size_t>(need, 1024);
		NEMO_CUDA(cudaMallocHost((void**) &m_hStim, cap * 4));
		NEMO_CUDA(cudaMallocHost((void**) &m_hCur, cap * 4));
		NEMO_CUDA(cudaMalloc((void**) &m_dStim, cap * 4));
		NEMO_CUDA(cudaMalloc((void**) &m_dCur, cap * 4));
		m_stimCap = cap;
	}
	uint32_t nfOk = 0, niOk = 0;
	int err = 0;
	unsigned badIdx = 0;
	for(size_t k = 0; k < nf; ++k) {
		const uint32_t d = toDev(fstim[k]);
		if(d == ~0u) { err = 1; badIdx = fstim[k]; break; }
		if(ownedOnly && !owns(d)) continue;
		m_hStim[nfOk++] = d;
	}
	if(!err && ni) {
		/* last write wins for repeated neurons: the entry of a neuron seen
		 * before in this call (m_stimEntry[d], valid when m_stimEpoch[d] is
		 * this call's epoch) is overwritten */
		if(m_stimEpoch.empty()) {
			m_stimEpoch.assign(m_nDev, 0u);
			m_stimEntry.assign(m_nDev, 0u);
		}
		if(++m_epoch == 0u) {
			std::fill(m_stimEpoch.begin(), m_stimEpoch.end(), 0u);
			m_epoch = 1u;
		}
		uint32_t* idx = m_hStim + nfOk;
		for(size_t k = 0; k < ni; ++k) {
			const uint32_t d = toDev(inidx[k]);
			if(d == ~0u) { err = 1; badIdx = inidx[k]; break; }
			if(ownedOnly && !owns(d)) continue;
			if(m_stimEpoch[d] == m_epoch) {
				m_hCur[m_stimEntry[d]] = icur[k];
			} else {
				m_stimEpoch[d] = m_epoch;
				m_stimEntry[d] = niOk;
				idx[niOk] = d;
				m_hCur[niOk] = icur[k];
				niOk++;
			}
		}
	}
	m_inline.nf = m_inline.ni = 0;
	if(!err && !m_external && nfOk <= INLINE_STIM_MAX && niOk <= INLINE_STIM_MAX) {
		/* short: carried in the step kernel's parameters */
		m_inline.nf = nfOk;
		m_inline.ni = niOk;
		std::copy(m_hStim, m_hStim + nfOk, m_inline.f);
		std::copy(m_hStim + nfOk, m_hStim + nfOk + niOk, m_inline.i);
		std::copy(m_hCur, m_hCur + niOk, m_inline.cur);
	} else if(nfOk + niOk) {
		NEMO_CUDA(cudaMemcpyAsync(m_dStim, m_hStim, size_t(nfOk + niOk) * 4, cudaMemcpyHostToDevice, stream));
		if(niOk) NEMO_CUDA(cudaMemcpyAsync(m_dCur, m_hCur, size_t(niOk) * 4, cudaMemcpyHostToDevice, stream));
		NEMO_CUDA(cudaEventRecord(static_cast<cudaEvent_t>(event(&m_evStaged)), stream));
		m_stagedPending = true;
		StimDev sd{m_dStim, nfOk, m_dStim + nfOk, m_dCur, niOk};
		launchStimulus(m_net, sd, m_stream);
	}
	if(err) {
		NEMO_CUDA(cudaStreamSynchronize(stream));
		fail(NEMO_INVALID_INPUT, "Non-existing neuron index " + std::to_string(badIdx));
	}
}

const std::vector<unsigned>&
Simulation::step(const unsigned* fstim, size_t nf, const unsigned* inidx, const float* icur, size_t ni)
{
	notShard("step");
	if(m_residentOn && !m_external && stepResident(fstim, nf, inidx, icur, ni)) {
		return m_fired;
	}
	stopResident();
	stageStimulus(fstim, nf, inidx, icur, ni, false);
	if(m_external) runPlugins();
	cudaStream_t stream = STREAM(m_stream);
	/* the kernel writes the firing bitmap and the error word into mapped
	 * host memory: no copy after it */
	launchStep();
	NEMO_CUDA(cudaStreamSynchronize(stream));
	NEMO_CUDA(cudaGetLastError());
	if(m_stepWords[0] != 0) {
		fail(NEMO_CUDA_ASSERTION_FAILURE, "step kernel: a grid barrier timed out; the simulation state is invalid");
	}
	m_cycle++;
	m_stateDirty = true;
	decodeStepList(m_fired);
	m_bytesIn += 4 * uint64_t(nf) + 8 * uint64_t(ni);
	m_bytesOut += 8 + 8 * uint64_t(m_stepWords[1]);
	return m_fired;
}

/* A step's stimulus mapped to device indices into m_inline, when it fits in
 * the kernel's inline arrays and every index exists (repeated current
 * stimulus: the last entry wins); false otherwise, with nothing applied. */
bool
Simulation::mapInline(const unsigned* fstim, size_t nf, const unsigned* inidx, const float* icur, size_t ni)
{
	if(nf > INLINE_STIM_MAX || ni > INLINE_STIM_MAX) return false;
	InlineStim st;
	for(size_t k = 0; k < nf; ++k) {
		const uint32_t d = toDev(fstim[k]);
		if(d == ~0u) return false;
		st.f[st.nf++] = d;
	}
	for(size_t k = 0; k < ni; ++k) {
		const uint32_t d = toDev(inidx[k]);
		if(d == ~0u) return false;
		uint32_t e = 0;
		while(e < st.ni && st.i[e] != d) ++e;
		if(e == st.ni) st.i[st.ni++] = d;
		st.cur[e] = icur[k];
	}
	m_inline = st;
	return true;
}

/* The simulation whose resident launch is on each device, if any. Two
 * resident launches must not share a device: each occupies an SM with every
 * block, and when both are partly resident, each one's blocks can wait for
 * its first block, which cannot start while the other's hold the SMs. */
static std::mutex g_residentLock;
static std::map<int, Simulation*> g_residentOwner;

void
Simulation::claimResidentDevice()
{
	Simulation* other = nullptr;
	{
		std::lock_guard<std::mutex> lock(g_residentLock);
		auto it = g_residentOwner.find(m_device);
		if(it != g_residentOwner.end() && it->second != this) other = it->second;
		g_residentOwner[m_device] = this;
	}
	if(other) {
		/* its error, if any, is its own: that simulation reports it on its
		 * next call */
		try {
			other->stopResident();
		} catch(...) {
		}
	}
}

void
Simulation::releaseResidentDevice()
{
	std::lock_guard<std::mutex> lock(g_residentLock);
	auto it = g_residentOwner.find(m_device);
	if(it != g_residentOwner.end() && it->second == this) g_residentOwner.erase(it);
}

/* The resident step kernel's launch for command `seq`, whose stimulus is
 * m_inline; the pending gathering of the last cycle, if any, is its first
 * phase's. The launch keeps the current slots in shared memory while it
 * stays. */
void
Simulation::launchResident(uint32_t seq)
{
	claimResidentDevice();
	if(m_rcmd == nullptr) {
		NEMO_CUDA(cudaHostAlloc((void**) &m_rcmd, sizeof(ResidentHostCmd), cudaHostAllocMapped));
		NEMO_CUDA(cudaHostGetDevicePointer((void**) &m_dRcmd, m_rcmd, 0));
		/* the done word and the exit word */
		NEMO_CUDA(cudaHostAlloc((void**) &m_rdone, 64, cudaHostAllocMapped));
		NEMO_CUDA(cudaHostGetDevicePointer((void**) &m_dRdone, m_rdone, 0));
		m_rbcast = (ResidentCmd*) alloc(2 * sizeof(ResidentCmd));
		std::memset(m_rcmd, 0, sizeof(ResidentHostCmd));
	}
	/* no command of this launch has run yet: done word, exit word */
	reinterpret_cast<volatile uint32_t*>(m_rdone)[0] = 0u;
	reinterpret_cast<volatile uint32_t*>(m_rdone)[1] = 0u;
	m_stepWords[0] = 0u;
	CycleArgs a = m_args;
	a.firstCycle = m_cycle;
	a.cycles = 1;
	a.carry = (m_pendingGather ? 1u : 0u) | 2u;
	a.globalAcc = 0;
	a.hostWords = m_dStepWords;
	a.inlineNf = m_inline.nf;
	a.inlineNi = m_inline.ni;
	std::copy(m_inline.f, m_inline.f + m_inline.nf, a.inlineF);
	std::copy(m_inline.i, m_inline.i + m_inline.ni, a.inlineI);
	std::copy(m_inline.cur, m_inline.cur + m_inline.ni, a.inlineCur);
	for(int gi = 0; gi < a.ngroups; ++gi) a.groups[gi].timerBase = uint32_t(m_timerBase);
	a.cmd = m_dRcmd;
	a.bcast = m_rbcast;
	a.doneWords = m_dRdone;
	a.exitInfo = m_dRdone + 1;
	a.firstSeq = seq;
	/* a caller that stops stepping releases the device after this long */
	a.idleNs = 1000ull * 1000;
	launchCycles(a, m_stream);
	NEMO_CUDA(cudaGetLastError());
	m_inline.nf = m_inline.ni = 0;
	m_pendingGather = true;
	m_resident = true;
}

void
Simulation::postCommand(uint32_t seq, uint32_t op)
{
	const bool step = op == RESIDENT_STEP;
	const uint32_t nf = step ? m_inline.nf : 0u, ni = step ? m_inline.ni : 0u;
	uint32_t payload[3 * RESIDENT_CHUNKS];
	uint32_t n = 0;
	payload[n++] = op;
	payload[n++] = nf;
	payload[n++] = ni;
	for(uint32_t k = 0; k < nf; ++k) payload[n++] = m_inline.f[k];
	for(uint32_t k = 0; k < ni; ++k) payload[n++] = m_inline.i[k];
	for(uint32_t k = 0; k < ni; ++k) std::memcpy(&payload[n++], &m_inline.cur[k], 4);
	const uint32_t chunks = (n + 2) / 3;
	m_bytesIn += 16u * chunks;
	volatile uint32_t* c = reinterpret_cast<volatile uint32_t*>(m_rcmd->c);
	for(uint32_t k = 0; k < chunks; ++k) {
		/* the chunk's payload, then its number (x86 keeps the store order) */
		for(uint32_t j = 0; j < 3; ++j) c[4 * k + 1 + j] = 3 * k + j < n ? payload[3 * k + j] : 0u;
		std::atomic_thread_fence(std::memory_order_release);
		c[4 * k] = seq;
	}
}

/* One cycle through the resident kernel; false when the stimulus does not
 * fit the command (nothing done: the caller takes the ordinary path). */
bool
Simulation::stepResident(const unsigned* fstim, size_t nf, const unsigned* inidx, const float* icur, size_t ni)
{
	if(!mapInline(fstim, nf, inidx, icur, ni)) return false;
	if(!fitsCommand()) {
		m_inline.nf = m_inline.ni = 0;
		return false;
	}
	const uint32_t seq = ++m_rseq;
	if(!m_resident) {
		launchResident(seq);
	} else {
		postCommand(seq, RESIDENT_STEP);
		m_inline.nf = m_inline.ni = 0;
	}
	volatile const uint32_t* done = m_rdone;
	const auto start = std::chrono::steady_clock::now();
	for(uint64_t spin = 0;; ++spin) {
		if(done[0] == seq) break;
		const uint32_t exitInfo = done[1];
		if(exitInfo != 0u && (exitInfo >> 1) < seq) {
			/* the launch ended (idle) before this command: run it in a new one */
			NEMO_CUDA(cudaStreamSynchronize(STREAM(m_stream)));
			m_resident = false;
			if(m_stepWords[0] != 0) {
				fail(NEMO_CUDA_ASSERTION_FAILURE, "step kernel: a grid barrier timed out; the simulation state is invalid");
			}
			mapInline(fstim, nf, inidx, icur, ni);
			launchResident(seq);
			continue;
		}
		if((spin & 4095u) == 4095u) {
			const cudaError_t e = cudaStreamQuery(STREAM(m_stream));
			if(e != cudaErrorNotReady) {
				/* the launch is over without this command done: a fault or a
				 * barrier timeout */
				m_resident = false;
				NEMO_CUDA(e);
				fail(NEMO_CUDA_ASSERTION_FAILURE, "resident step kernel ended without completing the cycle");
			}
			if(std::chrono::steady_clock::now() - start > std::chrono::seconds(20)) {
				fail(NEMO_CUDA_ASSERTION_FAILURE, "resident step kernel: no answer within 20 s");
			}
		}
	}
	std::atomic_thread_fence(std::memory_order_acquire);
	m_cycle++;
	m_stateDirty = true;
	decodeStepList(m_fired);
	/* the done word, the error and count words, the pairs */
	m_bytesOut += 4 + 8 + 8 * uint64_t(m_stepWords[1]);
	return true;
}

/* End the resident launch, if any: an exit command, then the stream drains.
 * The last cycle's gathering stays pending. */
void
Simulation::stopResident()
{
	if(!m_resident) return;
	postCommand(++m_rseq, RESIDENT_EXIT);
	m_resident = false;
	releaseResidentDevice();
	NEMO_CUDA(cudaStreamSynchronize(STREAM(m_stream)));
	NEMO_CUDA(cudaGetLastError());
	if(m_stepWords[0] != 0) {
		fail(NEMO_CUDA_ASSERTION_FAILURE, "step kernel: a grid barrier timed out; the simulation state is invalid");
	}
}

/* One applyStdp on the simulation's stream. Every plastic weight is within
 * its bounds afterwards (updatedWeight clamps each one). */
void
Simulation::launchApply(int32_t reward)
{
	launchApplyStdp(m_net, m_rule, reward, m_cycle, m_applyGroups.data(), uint32_t(m_applyGroups.size() - 1),
			m_weightsInRange, m_stream);
	m_weightsInRange = true;
}

/* The batch of a plugin population for the cycle about to run
 * (nemo_b200_plugin.h): the current of the cycle, the stimulus staged for
 * it, the firing history before it. */
void
Simulation::pluginBatch(const Group& g, b200_neuron_batch* b) const
{
	b->count = g.count;
	b->cycle = (unsigned long long) (m_cycle - m_timerBase);
	b->param = g.dParam;
	b->param_stride = g.count;
	b->state = g.dState;
	b->state_stride = g.count;
	b->current_epsp = g.dExtE;
	b->current_ipsp = g.dExtI;
	b->current_external = m_net.ext + g.devBase;
	b->fstim = m_net.fstim + g.devBase / 32;
	b->recent_firing = m_net.rf + size_t(m_cycle & 1u) * m_nDev + g.devBase;
	b->fired = g.dExtFired;
	b->rng = reinterpret_cast<uint32_t*>(g.dRng);
}

/* Each plugin population's update for the cycle about to run, on the
 * simulation's stream: its currents of the cycle are complete once the
 * previous step has run (its delay-1 arrivals are in the slot; the pending
 * gathering only reaches later cycles), so they are exported, the plugin
 * writes the firing bits, and the step launch that follows reads them. */
void
Simulation::runPlugins()
{
	for(const Group& g : m_groups) {
		if(!g.plugin) continue;
		launchExportCurrents(m_net, g.devBase, g.count, m_cycle, g.dExtE, g.dExtI, m_stream);
		NEMO_CUDA(cudaGetLastError());
		b200_neuron_batch b;
		pluginBatch(g, &b);
		const int rc = g.plugin->update(&b, m_stream);
		if(rc != 0) {
			fail(NEMO_CUDA_INVOCATION_ERROR, "Neuron model plugin " + g.plugin->path + ": b200_update_neurons: "
					+ cudaGetErrorString(cudaError_t(rc)));
		}
	}
}

void
Simulation::notExternal(const char* what) const
{
	if(m_external) {
		fail(NEMO_API_UNSUPPORTED, std::string(what) + ": the network has plugin neuron models, whose updates "
				"run cycle by cycle; step the simulation with nemo_step");
	}
}

void
Simulation::notShard(const char* what) const
{
	if(m_shardMode) {
		fail(NEMO_LOGIC_ERROR, std::string(what) + ": this simulation is one shard of a sharded simulation; "
				"its cycles run through the shard step and deliver calls");
	}
}

/* A shard's update launch: one phase that updates the owned neurons for this
 * cycle and gathers and learns for the previous one when that is pending
 * (carry bit 0), with no trailing gather (carry bit 1): the cycle's firing of
 * the other shards is not known yet. */
void
Simulation::shardStep(const unsigned* fstim, size_t nf, const unsigned* inidx, const float* icur, size_t ni,
		uint32_t* localWords)
{
	if(!m_shardMode) {
		fail(NEMO_LOGIC_ERROR, "shard step: the simulation is not a shard");
	}
	if(m_awaitDeliver) {
		fail(NEMO_LOGIC_ERROR, "shard step: the previous cycle's firing has not been delivered");
	}
	stageStimulus(fstim, nf, inidx, icur, ni, true);
	cudaStream_t stream = STREAM(m_stream);
	launchStep();
	const uint32_t slot = uint32_t(m_cycle) & m_net.ringMask;
	const uint32_t words = m_shard.warpHi - m_shard.warpLo;
	NEMO_CUDA(cudaMemcpyAsync(m_hWords, m_net.firedRing + size_t(slot) * m_net.nWords + m_shard.warpLo,
				size_t(words) * 4, cudaMemcpyDeviceToHost, stream));
	NEMO_CUDA(cudaMemcpyAsync(m_hWords + m_net.nWords, m_net.barrier + 2, 4, cudaMemcpyDeviceToHost, stream));
	NEMO_CUDA(cudaStreamSynchronize(stream));
	NEMO_CUDA(cudaGetLastError());
	checkDeviceError();
	std::memcpy(localWords, m_hWords, size_t(words) * 4);
	m_cycle++;
	m_stateDirty = true;
	m_awaitDeliver = true;
}

const std::vector<unsigned>&
Simulation::shardDeliver(const uint32_t* allWords)
{
	if(!m_awaitDeliver) {
		fail(NEMO_LOGIC_ERROR, "shard deliver: no shard step is waiting for its cycle's firing");
	}
	cudaStream_t stream = STREAM(m_stream);
	const uint64_t t = m_cycle - 1;
	if(!m_dAllWords) m_dAllWords = (uint32_t*) alloc(size_t(m_net.nWords) * 4);
	std::memcpy(m_hWords, allWords, size_t(m_net.nWords) * 4);
	NEMO_CUDA(cudaMemcpyAsync(m_dAllWords, m_hWords, size_t(m_net.nWords) * 4, cudaMemcpyHostToDevice, stream));
	if(m_net.remoteCnt) {
		NEMO_CUDA(cudaMemsetAsync(m_net.remoteCnt + (t & 1u), 0, 4, stream));
		launchShardInject(m_net, t, m_dAllWords, m_shard.warpLo, m_shard.warpHi, m_stream);
		NEMO_CUDA(cudaGetLastError());
	}
	NEMO_CUDA(cudaStreamSynchronize(stream));
	m_awaitDeliver = false;
	decodeFired(allWords, m_fired);
	return m_fired;
}

void*
Simulation::event(void** ev)
{
	if(*ev == nullptr) {
		cudaEvent_t e;
		NEMO_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
		*ev = e;
	}
	return *ev;
}

void
Simulation::streamWait(void* stream)
{
	stopResident();
	cudaEvent_t e = static_cast<cudaEvent_t>(event(&m_evOut));
	NEMO_CUDA(cudaEventRecord(e, STREAM(m_stream)));
	NEMO_CUDA(cudaStreamWaitEvent(STREAM(stream), e, 0));
}

void
Simulation::shardStepAsync(const unsigned* fstim, size_t nf, const unsigned* inidx, const float* icur, size_t ni,
		uint32_t* localDev, void* stream)
{
	if(!m_shardMode) {
		fail(NEMO_LOGIC_ERROR, "shard step: the simulation is not a shard");
	}
	if(m_awaitDeliver) {
		fail(NEMO_LOGIC_ERROR, "shard step: the previous cycle's firing has not been delivered");
	}
	stageStimulus(fstim, nf, inidx, icur, ni, true);
	launchStep();
	const uint32_t slot = uint32_t(m_cycle) & m_net.ringMask;
	const uint32_t words = m_shard.warpHi - m_shard.warpLo;
	NEMO_CUDA(cudaMemcpyAsync(localDev, m_net.firedRing + size_t(slot) * m_net.nWords + m_shard.warpLo,
				size_t(words) * 4, cudaMemcpyDeviceToDevice, STREAM(m_stream)));
	streamWait(stream);
	m_cycle++;
	m_stateDirty = true;
	m_awaitDeliver = true;
}

void
Simulation::shardDeliverAsync(const uint32_t* allDev, void* stream)
{
	if(!m_awaitDeliver) {
		fail(NEMO_LOGIC_ERROR, "shard deliver: no shard step is waiting for its cycle's firing");
	}
	cudaEvent_t e = static_cast<cudaEvent_t>(event(&m_evIn));
	NEMO_CUDA(cudaEventRecord(e, STREAM(stream)));
	NEMO_CUDA(cudaStreamWaitEvent(STREAM(m_stream), e, 0));
	const uint64_t t = m_cycle - 1;
	if(m_net.remoteCnt) {
		NEMO_CUDA(cudaMemsetAsync(m_net.remoteCnt + (t & 1u), 0, 4, STREAM(m_stream)));
		launchShardInject(m_net, t, allDev, m_shard.warpLo, m_shard.warpHi, m_stream);
		NEMO_CUDA(cudaGetLastError());
	}
	m_awaitDeliver = false;
}

/* One cycle as a single phase: the update of cycle m_cycle, overlapped with
 * the gathering and learning of the cycle before when that is pending (carry
 * bit 0); this cycle's own gathering waits (carry bit 1) for the next step or
 * flushPending. Reading the firing never needs it: delivery only affects
 * later cycles' currents and the STDP accumulators. */
void
Simulation::launchStep()
{
	m_stepWords[0] = 0u;
	launchBlock(m_cycle, 1, (m_pendingGather ? 1u : 0u) | 2u, m_stepGlobalAcc, m_dStepWords, &m_inline);
	m_inline.nf = m_inline.ni = 0;
	m_pendingGather = true;
}

/* The pending gathering and learning of the last cycle: one gather phase
 * (carry bit 0, no cycles). Before anything that reads the accumulators or
 * launches the multi-cycle kernel. */
void
Simulation::flushPending()
{
	stopResident();
	if(m_awaitDeliver) {
		fail(NEMO_LOGIC_ERROR, "the last shard step's firing has not been delivered");
	}
	if(m_pendingGather) {
		launchBlock(m_cycle, 0, 1u, m_stepGlobalAcc);
		m_pendingGather = false;
	}
}

/* step() without allocation. Indices are mapped on the host into a small
 * stack buffer and copied chunk by chunk into the module-static scratch
 * (a pageable-source cudaMemcpyAsync returns once the source has been
 * staged, so the buffer can be reused at once); duplicates of the current
 * stimulus are resolved on the device in call order. An invalid index raises
 * after the entries before it have been applied, as step() does. */
size_t
Simulation::stepNoAlloc(const unsigned* fstim, size_t nf, const unsigned* inidx, const float* icur, size_t ni,
		unsigned* firedOut, size_t firedCapacity)
{
	stopResident();
	notShard("stepNoAlloc");
	if(nf > NOALLOC_STIM_MAX || ni > NOALLOC_STIM_MAX) {
		fail(NEMO_INVALID_INPUT, "nemo_b200_step_noalloc: at most " + std::to_string(NOALLOC_STIM_MAX)
				+ " firing-stimulus and " + std::to_string(NOALLOC_STIM_MAX)
				+ " current-stimulus entries per call (got " + std::to_string(nf) + " and "
				+ std::to_string(ni) + ")");
	}
	if(firedOut == nullptr || firedCapacity < m_nNeurons) {
		fail(NEMO_INVALID_INPUT, "nemo_b200_step_noalloc: the fired array must hold the network's "
				+ std::to_string(m_nNeurons) + " neurons");
	}
	if(m_noallocDevice < 0) {
		cudaPointerAttributes attr;
		NEMO_CUDA(cudaPointerGetAttributes(&attr, m_net.rf));
		m_noallocDevice = attr.device;
	}
	int current = -1;
	NEMO_CUDA(cudaGetDevice(&current));
	if(current != m_noallocDevice) {
		fail(NEMO_INVALID_INPUT, "nemo_b200_step_noalloc: device " + std::to_string(m_noallocDevice)
				+ " of the simulation must be the current device (current: " + std::to_string(current) + ")");
	}
	uint32_t* scratch = nullptr;
	NEMO_CUDA(noallocScratch(m_noallocDevice, &scratch));

	cudaStream_t stream = STREAM(m_stream);
	const size_t CHUNK = 1024;
	uint32_t stage[CHUNK];
	int err = 0;
	unsigned badIdx = 0;
	uint32_t nfOk = 0, niOk = 0;
	for(size_t k0 = 0; k0 < nf && !err; k0 += CHUNK) {
		size_t cnt = 0;
		for(size_t k = k0; k < nf && k < k0 + CHUNK; ++k) {
			const uint32_t d = toDev(fstim[k]);
			if(d == ~0u) { err = 1; badIdx = fstim[k]; break; }
			stage[cnt++] = d;
		}
		if(cnt) NEMO_CUDA(cudaMemcpyAsync(scratch + nfOk, stage, cnt * 4, cudaMemcpyHostToDevice, stream));
		nfOk += uint32_t(cnt);
	}
	for(size_t k0 = 0; k0 < ni && !err; k0 += CHUNK) {
		size_t cnt = 0;
		for(size_t k = k0; k < ni && k < k0 + CHUNK; ++k) {
			const uint32_t d = toDev(inidx[k]);
			if(d == ~0u) { err = 1; badIdx = inidx[k]; break; }
			stage[cnt++] = d;
		}
		if(cnt) {
			NEMO_CUDA(cudaMemcpyAsync(scratch + NOALLOC_STIM_MAX + niOk, stage, cnt * 4,
						cudaMemcpyHostToDevice, stream));
			NEMO_CUDA(cudaMemcpyAsync(scratch + 2 * NOALLOC_STIM_MAX + niOk, icur + k0, cnt * 4,
						cudaMemcpyHostToDevice, stream));
		}
		niOk += uint32_t(cnt);
	}
	launchStimulusScratch(m_net, scratch, nfOk, niOk, m_stream);
	if(err) {
		NEMO_CUDA(cudaStreamSynchronize(stream));
		fail(NEMO_INVALID_INPUT, "Non-existing neuron index " + std::to_string(badIdx));
	}
	if(m_external) runPlugins();

	launchStep();
	NEMO_CUDA(cudaStreamSynchronize(stream));
	NEMO_CUDA(cudaGetLastError());
	if(m_stepWords[0] != 0) {
		fail(NEMO_CUDA_ASSERTION_FAILURE, "step kernel: a grid barrier timed out; the simulation state is invalid");
	}
	m_cycle++;
	m_stateDirty = true;
	size_t count = 0;
	decodeStepList([&](unsigned g) { firedOut[count++] = g; });
	return count;
}

void
Simulation::run(unsigned cycles, uint32_t* firedCounts, uint64_t* events)
{
	notShard("run");
	flushPending();
	if(cycles == 0) return;
	if(cycles > m_ring) {
		fail(NEMO_INVALID_INPUT, "run: at most " + std::to_string(m_ring) + " cycles per call");
	}
	cudaStream_t stream = STREAM(m_stream);
	uint64_t first = m_cycle;
	if(m_external) {
		/* plugin models update between the kernel's phases: every cycle's
		 * current export, plugin updates and one-phase step launch are
		 * queued on the stream without waiting, as nemo_step runs them; a
		 * barrier timeout in any of them stays in the barrier's error word */
		for(unsigned k = 0; k < cycles; ++k) {
			runPlugins();
			launchBlock(m_cycle, 1, (m_pendingGather ? 1u : 0u) | 2u, m_stepGlobalAcc);
			m_pendingGather = true;
			m_cycle++;
		}
		flushPending();
	} else {
		launchBlock(m_cycle, cycles);
		m_cycle += cycles;
	}
	m_stateDirty = true;
	std::vector<uint32_t> fc(m_ring);
	std::vector<uint64_t> ev(m_ring);
	if(firedCounts || events) {
		NEMO_CUDA(cudaMemcpyAsync(fc.data(), m_net.firedCountRing, m_ring * 4, cudaMemcpyDeviceToHost, stream));
		NEMO_CUDA(cudaMemcpyAsync(ev.data(), m_net.eventsRing, m_ring * 8, cudaMemcpyDeviceToHost, stream));
	}
	NEMO_CUDA(cudaMemcpyAsync(m_hWords + m_net.nWords, m_net.barrier + 2, 4, cudaMemcpyDeviceToHost, stream));
	NEMO_CUDA(cudaStreamSynchronize(stream));
	checkDeviceError();
	for(unsigned k = 0; k < cycles && (firedCounts || events); ++k) {
		uint32_t slot = uint32_t(first + k) & m_net.ringMask;
		if(firedCounts) firedCounts[k] = fc[slot];
		if(events) events[k] = ev[slot];
	}
}

void
Simulation::batchFiredAt(uint64_t cycle, const std::vector<unsigned>** fired, const std::vector<size_t>** offsets)
{
	const std::vector<unsigned>& all = firedAt(cycle);
	const size_t J = instances();
	m_batchOffsets.assign(J + 1, 0);
	m_batchFired.resize(all.size());
	if(m_batchBase.empty()) {
		std::copy(all.begin(), all.end(), m_batchFired.begin());
		m_batchOffsets[1] = all.size();
	} else {
		/* stable bucketing by instance keeps each instance's order */
		std::vector<uint32_t> inst(all.size());
		for(size_t k = 0; k < all.size(); ++k) {
			inst[k] = uint32_t(std::upper_bound(m_batchBase.begin(), m_batchBase.end(), all[k]) - m_batchBase.begin() - 1);
			m_batchOffsets[inst[k] + 1]++;
		}
		for(size_t j = 0; j < J; ++j) m_batchOffsets[j + 1] += m_batchOffsets[j];
		std::vector<size_t> fill(m_batchOffsets.begin(), m_batchOffsets.end() - 1);
		for(size_t k = 0; k < all.size(); ++k) {
			m_batchFired[fill[inst[k]]++] = all[k] - m_batchBase[inst[k]];
		}
	}
	*fired = &m_batchFired;
	*offsets = &m_batchOffsets;
}

void
Simulation::destroyGraph()
{
	if(m_graphExec) {
		cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(m_graphExec));
		m_graphExec = nullptr;
	}
}

void
Simulation::runGraph(unsigned cycles, unsigned cyclesPerLaunch, int* usedGraph)
{
	notShard("runGraph");
	notExternal("runGraph");
	flushPending();
	if(cycles == 0) return;
	if(cycles > m_ring) {
		fail(NEMO_INVALID_INPUT, "run: at most " + std::to_string(m_ring) + " cycles per call");
	}
	if(cyclesPerLaunch == 0) cyclesPerLaunch = cycles;
	cudaStream_t stream = STREAM(m_stream);
	if(!m_dCycleCounter) {
		m_dCycleCounter = (uint64_t*) alloc(8);
	}
	CycleArgs a = m_args;
	a.cycleCounter = m_dCycleCounter;
	for(int gi = 0; gi < a.ngroups; ++gi) a.groups[gi].timerBase = uint32_t(m_timerBase);
	const uint64_t key[4] = {cycles, cyclesPerLaunch, m_net.threads, m_timerBase};
	if(m_graphUsable && (!m_graphExec || !std::equal(key, key + 4, m_graphKey))) {
		destroyGraph();
		cudaGraph_t graph = nullptr;
		cudaError_t e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
		if(e == cudaSuccess) {
			for(unsigned done = 0; done < cycles; done += cyclesPerLaunch) {
				a.cycles = std::min(cyclesPerLaunch, cycles - done);
				launchCycles(a, m_stream);
			}
			e = cudaStreamEndCapture(stream, &graph);
		}
		cudaGraphExec_t exec = nullptr;
		if(e == cudaSuccess) {
			e = cudaGraphInstantiate(&exec, graph, 0);
		}
		if(graph) cudaGraphDestroy(graph);
		if(e == cudaSuccess) {
			m_graphExec = exec;
			std::copy(key, key + 4, m_graphKey);
		} else {
			(void) cudaGetLastError();   /* the capture failed: launch directly from now on */
			m_graphUsable = false;
		}
	}
	uint64_t counter = m_cycle;
	NEMO_CUDA(cudaMemcpyAsync(m_dCycleCounter, &counter, 8, cudaMemcpyHostToDevice, stream));
	if(m_graphUsable && m_graphExec) {
		NEMO_CUDA(cudaGraphLaunch(static_cast<cudaGraphExec_t>(m_graphExec), stream));
		if(usedGraph) *usedGraph = 1;
	} else {
		for(unsigned done = 0; done < cycles; done += cyclesPerLaunch) {
			a.cycles = std::min(cyclesPerLaunch, cycles - done);
			launchCycles(a, m_stream);
			NEMO_CUDA(cudaGetLastError());
		}
		if(usedGraph) *usedGraph = 0;
	}
	m_cycle += cycles;
	m_stateDirty = true;
	NEMO_CUDA(cudaMemcpyAsync(m_hWords + m_net.nWords, m_net.barrier + 2, 4, cudaMemcpyDeviceToHost, stream));
	NEMO_CUDA(cudaStreamSynchronize(stream));
	checkDeviceError();
}

/* The step kernel's shape by trial: threads per block (1024, 512, 256) and,
 * for a network with STDP, the synapses of a full STDP work entry (128, 64),
 * each candidate timed over trialCycles ordinary cycles (simulated: the
 * network advances), twice, interleaved, the better trial kept (the
 * network's activity drifts between trials); the fastest is kept for the
 * following launches. Results do not depend on the shape. ms[3 * r + k]:
 * ms per cycle with thread size k and run length r (r = 1 only with STDP,
 * else 0). */
AutotuneShape
Simulation::autotuneShape(unsigned trialCycles, double ms[6])
{
	notShard("autotune");
	notExternal("autotune");
	flushPending();
	if(trialCycles == 0 || trialCycles > m_ring) {
		fail(NEMO_INVALID_INPUT, "autotune: trial cycles must be in 1.." + std::to_string(m_ring));
	}
	cudaStream_t stream = STREAM(m_stream);
	const unsigned sizes[3] = {1024, 512, 256};
	const unsigned runs[2] = {STDP_ITEM, STDP_RUN_MIN};
	const int nRuns = m_stdpOn ? 2 : 1;
	AutotuneShape best{sizes[0], runs[0]};
	double bestMs = 1e300;
	cudaEvent_t e0, e1;
	NEMO_CUDA(cudaEventCreate(&e0));
	NEMO_CUDA(cudaEventCreate(&e1));
	for(int k = 0; k < 6; ++k) ms[k] = k < 3 * nRuns ? 1e300 : 0.0;
	for(int round = 0; round < 2; ++round) {
		for(int r = 0; r < nRuns; ++r) {
			for(int k = 0; k < 3; ++k) {
				m_net.threads = sizes[k];
				m_net.stdpRun = runs[r];
				m_args.net.threads = sizes[k];
				m_args.net.stdpRun = runs[r];
				NEMO_CUDA(cudaEventRecord(e0, stream));
				launchBlock(m_cycle, trialCycles);
				NEMO_CUDA(cudaEventRecord(e1, stream));
				NEMO_CUDA(cudaEventSynchronize(e1));
				m_cycle += trialCycles;
				float t = 0;
				NEMO_CUDA(cudaEventElapsedTime(&t, e0, e1));
				ms[3 * r + k] = std::min(ms[3 * r + k], double(t) / trialCycles);
			}
		}
	}
	for(int r = 0; r < nRuns; ++r) {
		for(int k = 0; k < 3; ++k) {
			if(ms[3 * r + k] < bestMs) {
				bestMs = ms[3 * r + k];
				best = AutotuneShape{sizes[k], runs[r]};
			}
		}
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	m_net.threads = best.threads;
	m_net.stdpRun = best.stdpRun;
	m_args.net.threads = best.threads;
	m_args.net.stdpRun = best.stdpRun;
	m_stateDirty = true;
	NEMO_CUDA(cudaMemcpyAsync(m_hWords + m_net.nWords, m_net.barrier + 2, 4, cudaMemcpyDeviceToHost, stream));
	NEMO_CUDA(cudaStreamSynchronize(stream));
	checkDeviceError();
	return best;
}

/* autotuneShape, reported by thread size: ms[k] the best over run lengths */
unsigned
Simulation::autotune(unsigned trialCycles, double ms[3])
{
	double all[6];
	const AutotuneShape best = autotuneShape(trialCycles, all);
	for(int k = 0; k < 3; ++k) ms[k] = m_stdpOn ? std::min(all[k], all[3 + k]) : all[k];
	return best.threads;
}

void
Simulation::synchronize()
{
	stopResident();
	NEMO_CUDA(cudaStreamSynchronize(STREAM(m_stream)));
	NEMO_CUDA(cudaGetLastError());
}

const std::vector<unsigned>&
Simulation::firedAt(uint64_t cycle)
{
	stopResident();
	if(cycle >= m_cycle || m_cycle - cycle > m_ring) {
		fail(NEMO_INVALID_INPUT, "firing of cycle " + std::to_string(cycle) + " is no longer (or not yet) available");
	}
	uint32_t slot = uint32_t(cycle) & m_net.ringMask;
	NEMO_CUDA(cudaMemcpyAsync(m_hWords, m_net.firedRing + size_t(slot) * m_net.nWords,
				size_t(m_net.nWords) * 4, cudaMemcpyDeviceToHost, STREAM(m_stream)));
	NEMO_CUDA(cudaStreamSynchronize(STREAM(m_stream)));
	decodeFired(m_hWords, m_fired);
	return m_fired;
}

/* src/nemo/ConnectivityMatrix.cpp:272-325 */
void
Simulation::applyStdp(float reward)
{
	if(!m_stdpOn) {
		fail(NEMO_LOGIC_ERROR, "applyStdp called, but no STDP model specified");
	}
	int32_t fx = toFix(reward, m_fbits);
	if(fx == 0 && reward != 0) {
		std::ostringstream msg;
		msg << "STDP reward rounded down to zero. The smallest valid reward is " << fixToFloat(1, m_fbits);
		fail(NEMO_INVALID_INPUT, msg.str());
	}
	flushPending();
	if(m_nrcm) {
		launchApply(fx);
	}
	m_fcmHostValid = false;
}

void
Simulation::syncStateToHost()
{
	stopResident();
	if(!m_stateDirty) return;
	cudaStream_t stream = STREAM(m_stream);
	for(Group& g : m_groups) {
		if(!g.state.empty()) {
			NEMO_CUDA(cudaMemcpyAsync(g.state.data(), g.dState, g.state.size() * 4, cudaMemcpyDeviceToHost, stream));
		}
	}
	NEMO_CUDA(cudaStreamSynchronize(stream));
	m_stateDirty = false;
}

static void
checkVar(unsigned i, unsigned n, const char* what)
{
	if(i >= n) {
		fail(NEMO_INVALID_INPUT, std::string("Invalid ") + what + " index " + std::to_string(i));
	}
}

float
Simulation::getNeuronState(unsigned gidx, unsigned var)
{
	uint32_t i;
	Group& g = groupOfDev(devIndex(gidx), &i);
	checkVar(var, g.type.nState, "state variable");
	syncStateToHost();
	return g.state[size_t(var) * g.count + i];
}

float
Simulation::getNeuronParameter(unsigned gidx, unsigned param) const
{
	uint32_t i;
	const Group& g = groupOfDev(devIndex(gidx), &i);
	checkVar(param, g.type.nParam, "parameter");
	return g.param[size_t(param) * g.count + i];
}

float
Simulation::getMembranePotential(unsigned gidx)
{
	uint32_t i;
	Group& g = groupOfDev(devIndex(gidx), &i);
	return getNeuronState(gidx, g.type.membranePotential);
}

void
Simulation::setNeuron(unsigned gidx, unsigned nargs, const float* args)
{
	stopResident();
	uint32_t i;
	Group& g = groupOfDev(devIndex(gidx), &i);
	if(nargs != g.type.nParam + g.type.nState) {
		std::ostringstream msg;
		msg << "Unexpected number of parameters/state variables when modifying neuron. Expected "
			<< g.type.nParam + g.type.nState << ", found " << nargs;
		fail(NEMO_INVALID_INPUT, msg.str());
	}
	syncStateToHost();
	cudaStream_t stream = STREAM(m_stream);
	for(unsigned p = 0; p < g.type.nParam; ++p) {
		float* h = &g.param[size_t(p) * g.count + i];
		*h = args[p];
		NEMO_CUDA(cudaMemcpyAsync(g.dParam + size_t(p) * g.count + i, h, 4, cudaMemcpyHostToDevice, stream));
	}
	for(unsigned s = 0; s < g.type.nState; ++s) {
		float* h = &g.state[size_t(s) * g.count + i];
		*h = args[g.type.nParam + s];
		NEMO_CUDA(cudaMemcpyAsync(g.dState + size_t(s) * g.count + i, h, 4, cudaMemcpyHostToDevice, stream));
	}
	NEMO_CUDA(cudaStreamSynchronize(stream));
}

void
Simulation::setNeuronState(unsigned gidx, unsigned var, float val)
{
	stopResident();
	uint32_t i;
	Group& g = groupOfDev(devIndex(gidx), &i);
	checkVar(var, g.type.nState, "state variable");
	syncStateToHost();
	float* h = &g.state[size_t(var) * g.count + i];
	*h = val;
	NEMO_CUDA(cudaMemcpyAsync(g.dState + size_t(var) * g.count + i, h, 4, cudaMemcpyHostToDevice, STREAM(m_stream)));
	NEMO_CUDA(cudaStreamSynchronize(STREAM(m_stream)));
}

void
Simulation::setNeuronParameter(unsigned gidx, unsigned param, float val)
{
	stopResident();
	uint32_t i;
	Group& g = groupOfDev(devIndex(gidx), &i);
	checkVar(param, g.type.nParam, "parameter");
	float* h = &g.param[size_t(param) * g.count + i];
	*h = val;
	NEMO_CUDA(cudaMemcpyAsync(g.dParam + size_t(param) * g.count + i, h, 4, cudaMemcpyHostToDevice, STREAM(m_stream)));
	NEMO_CUDA(cudaStreamSynchronize(STREAM(m_stream)));
}

/* src/nemo/ConnectivityMatrix.cpp:329-362 */
const std::vector<synapse_id>&
Simulation::getSynapsesFrom(unsigned source)
{
	if(m_writeOnly) {
		fail(NEMO_INVALID_INPUT, "Cannot read synapse state if simulation configured with write-only synapses");
	}
	uint32_t n = 0;
	auto it = m_auxRange.find(source);
	if(it == m_auxRange.end()) {
		if(m_g2d.find(source) == m_g2d.end()) {
			fail(NEMO_INVALID_INPUT, "Non-existing source neuron id (" + std::to_string(source) + ") in synapse id query");
		}
	} else {
		n = it->second.second;
	}
	m_queried.resize(n);
	for(uint32_t i = 0; i < n; ++i) {
		const uint32_t sid = m_auxSid.empty() ? i : m_auxSid[it->second.first + i];
		m_queried[i] = (uint64_t(source) << 32) | sid;
	}
	return m_queried;
}

/* src/nemo/ConnectivityMatrix.cpp:374-391 */
const Simulation::Aux&
Simulation::aux(synapse_id id) const
{
	if(m_writeOnly) {
		fail(NEMO_INVALID_INPUT, "Cannot read synapse state if simulation configured with write-only synapses");
	}
	uint32_t neuron = uint32_t(id >> 32);
	auto it = m_auxRange.find(neuron);
	if(it == m_auxRange.end()) {
		fail(NEMO_INVALID_INPUT, "Non-existing neuron id (" + std::to_string(neuron) + ") in synapse query");
	}
	uint32_t idx = uint32_t(id & 0xffffffffu);
	if(!m_auxSid.empty()) {
		/* a shard: the entry with this per-source index, if the shard holds it */
		const auto b = m_auxSid.begin() + ptrdiff_t(it->second.first);
		const auto e = b + ptrdiff_t(it->second.second);
		const auto p = std::lower_bound(b, e, idx);
		if(p == e || *p != idx) {
			throw std::out_of_range("synapse index out of range (the synapse's target is another shard's)");
		}
		return m_aux[size_t(p - m_auxSid.begin())];
	}
	if(idx >= it->second.second) {
		throw std::out_of_range("synapse index out of range");
	}
	return m_aux[it->second.first + idx];
}

unsigned Simulation::getSynapseTarget(synapse_id id) const { return aux(id).target; }
unsigned Simulation::getSynapseDelay(synapse_id id) const { return aux(id).delay; }
unsigned char Simulation::getSynapsePlastic(synapse_id id) const { return aux(id).plastic; }

float
Simulation::getSynapseWeight(synapse_id id)
{
	stopResident();
	const Aux& a = aux(id);
	if(!m_fcmHostValid) {
		m_fcmHost.resize(m_nsyn);
		if(m_nsyn) {
			NEMO_CUDA(cudaMemcpyAsync(m_fcmHost.data(), m_net.fcm, m_nsyn * 8, cudaMemcpyDeviceToHost, STREAM(m_stream)));
			NEMO_CUDA(cudaStreamSynchronize(STREAM(m_stream)));
		}
		m_fcmHostValid = true;
	}
	return fixToFloat(int32_t(m_fcmHost[a.fcmPos].y), m_fbits);
}

/* getSynapseWeight over many ids: the per-source lookup is made once per run
 * of ids from the same source */
void
Simulation::getWeights(const synapse_id* ids, size_t n, float* out)
{
	if(m_writeOnly) {
		fail(NEMO_INVALID_INPUT, "Cannot read synapse state if simulation configured with write-only synapses");
	}
	if(!m_auxSid.empty()) {
		for(size_t k = 0; k < n; ++k) out[k] = getSynapseWeight(ids[k]);
		return;
	}
	if(n) (void) getSynapseWeight(ids[0]);   /* the host copy of the forward matrix */
	bool have = false;
	uint32_t last = 0;
	size_t first = 0, count = 0;
	for(size_t k = 0; k < n; ++k) {
		const uint32_t neuron = uint32_t(ids[k] >> 32);
		if(!have || neuron != last) {
			auto it = m_auxRange.find(neuron);
			if(it == m_auxRange.end()) {
				fail(NEMO_INVALID_INPUT, "Non-existing neuron id (" + std::to_string(neuron) + ") in synapse query");
			}
			first = it->second.first;
			count = it->second.second;
			last = neuron;
			have = true;
		}
		const uint32_t idx = uint32_t(ids[k] & 0xffffffffu);
		if(idx >= count) {
			throw std::out_of_range("synapse index out of range");
		}
		out[k] = fixToFloat(int32_t(m_fcmHost[m_aux[first + idx].fcmPos].y), m_fbits);
	}
}

unsigned long
Simulation::elapsedWallclock() const
{
	return (unsigned long) std::chrono::duration_cast<std::chrono::milliseconds>(
			std::chrono::steady_clock::now() - m_wallStart).count();
}

void
Simulation::resetTimer()
{
	stopResident();
	m_wallStart = std::chrono::steady_clock::now();
	m_timerBase = m_cycle;
}

void
Simulation::nrandProbe(const uint32_t* u1, const uint32_t* u2, float* out, size_t n)
{
	stopResident();
	const LibmTables& t = libmTables();
	cudaStream_t stream = STREAM(m_stream);
	uint32_t *d1, *d2, *ds, *dl;
	float* dout;
	NEMO_CUDA(cudaMalloc(&d1, n * 4 + 4));
	NEMO_CUDA(cudaMalloc(&d2, n * 4 + 4));
	NEMO_CUDA(cudaMalloc(&dout, n * 4 + 4));
	NEMO_CUDA(cudaMalloc(&ds, t.sinCodes.size() * 4));
	NEMO_CUDA(cudaMalloc(&dl, t.logCodes.size() * 4));
	NEMO_CUDA(cudaMemcpyAsync(d1, u1, n * 4, cudaMemcpyHostToDevice, stream));
	NEMO_CUDA(cudaMemcpyAsync(d2, u2, n * 4, cudaMemcpyHostToDevice, stream));
	NEMO_CUDA(cudaMemcpyAsync(ds, t.sinCodes.data(), t.sinCodes.size() * 4, cudaMemcpyHostToDevice, stream));
	NEMO_CUDA(cudaMemcpyAsync(dl, t.logCodes.data(), t.logCodes.size() * 4, cudaMemcpyHostToDevice, stream));
	launchNrandProbe(d1, d2, dout, n, ds, dl, m_stream);
	NEMO_CUDA(cudaMemcpyAsync(out, dout, n * 4, cudaMemcpyDeviceToHost, stream));
	NEMO_CUDA(cudaStreamSynchronize(stream));
	cudaFree(d1);
	cudaFree(d2);
	cudaFree(dout);
	cudaFree(ds);
	cudaFree(dl);
}

void
Simulation::readStats(uint64_t out[4])
{
	stopResident();
	NEMO_CUDA(cudaMemcpyAsync(out, m_net.stats, 4 * 8, cudaMemcpyDeviceToHost, STREAM(m_stream)));
	NEMO_CUDA(cudaStreamSynchronize(STREAM(m_stream)));
}

void
Simulation::timedSteps(unsigned steps, unsigned cyclesPerStep, bool apply, float reward, double out[4])
{
	notShard("timedSteps");
	notExternal("timedSteps");
	flushPending();
	if(cyclesPerStep == 0 || cyclesPerStep > m_ring) {
		fail(NEMO_INVALID_INPUT, "timed steps: cycles per step must be in 1.." + std::to_string(m_ring));
	}
	if(apply && !m_stdpOn) {
		fail(NEMO_LOGIC_ERROR, "applyStdp called, but no STDP model specified");
	}
	int32_t fx = apply ? toFix(reward, m_fbits) : 0;
	cudaStream_t stream = STREAM(m_stream);
	uint64_t before[4], after[4];
	readStats(before);
	cudaEvent_t e0, e1;
	NEMO_CUDA(cudaEventCreate(&e0));
	NEMO_CUDA(cudaEventCreate(&e1));
	NEMO_CUDA(cudaEventRecord(e0, stream));
	for(unsigned s = 0; s < steps; ++s) {
		launchBlock(m_cycle, cyclesPerStep);
		m_cycle += cyclesPerStep;
		if(apply && m_nrcm) {
			launchApply(fx);
		}
	}
	NEMO_CUDA(cudaEventRecord(e1, stream));
	NEMO_CUDA(cudaEventSynchronize(e1));
	float ms = 0;
	NEMO_CUDA(cudaEventElapsedTime(&ms, e0, e1));
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	NEMO_CUDA(cudaGetLastError());
	m_stateDirty = true;
	m_fcmHostValid = false;
	NEMO_CUDA(cudaMemcpyAsync(m_hWords + m_net.nWords, m_net.barrier + 2, 4, cudaMemcpyDeviceToHost, stream));
	readStats(after);
	checkDeviceError();
	out[0] = ms;
	out[1] = double(after[2] - before[2]);
	out[2] = double(after[3] - before[3]);
	out[3] = double(after[0] - before[0]);
}

void
Simulation::profile(unsigned cycles, float reward, double out[10])
{
	notShard("profile");
	notExternal("profile");
	flushPending();
	cudaStream_t stream = STREAM(m_stream);
	cudaEvent_t e0, e1, e2;
	NEMO_CUDA(cudaEventCreate(&e0));
	NEMO_CUDA(cudaEventCreate(&e1));
	NEMO_CUDA(cudaEventCreate(&e2));
	uint64_t before[4], after[4];
	readStats(before);
	NEMO_CUDA(cudaEventRecord(e0, stream));
	launchBlock(m_cycle, cycles);
	m_cycle += cycles;
	NEMO_CUDA(cudaEventRecord(e1, stream));
	if(m_stdpOn && m_nrcm) {
		launchApply(toFix(reward, m_fbits));
		m_fcmHostValid = false;
	}
	NEMO_CUDA(cudaEventRecord(e2, stream));
	NEMO_CUDA(cudaEventSynchronize(e2));
	float tc = 0, ta = 0;
	NEMO_CUDA(cudaEventElapsedTime(&tc, e0, e1));
	NEMO_CUDA(cudaEventElapsedTime(&ta, e1, e2));
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	cudaEventDestroy(e2);
	NEMO_CUDA(cudaMemcpyAsync(m_hWords + m_net.nWords, m_net.barrier + 2, 4, cudaMemcpyDeviceToHost, stream));
	readStats(after);
	checkDeviceError();
	m_stateDirty = true;
	out[0] = tc;
	out[1] = m_blocks;
	out[2] = 0;
	out[3] = double(after[0] - before[0]);
	out[4] = double(after[2] - before[2]);
	out[5] = double(after[1] - before[1]);
	out[6] = double(m_nNeurons) * cycles;
	out[7] = (m_stdpOn && m_nrcm) ? ta : 0.0;
	out[8] = double(m_nrcm);
	out[9] = double(after[3] - before[3]);
}

void
Simulation::trace(unsigned cycles, double out[24])
{
	notShard("trace");
	notExternal("trace");
	flushPending();
	if(cycles == 0) {
		fail(NEMO_INVALID_INPUT, "trace: no cycles");
	}
	cudaStream_t stream = STREAM(m_stream);
	const unsigned S = 20;
	size_t words = size_t(cycles + 1) * m_blocks * S;
	unsigned long long* dTrace;
	NEMO_CUDA(cudaMalloc(&dTrace, words * 8));
	NEMO_CUDA(cudaMemsetAsync(dTrace, 0, words * 8, stream));
	CycleArgs a = m_args;
	a.firstCycle = m_cycle;
	a.cycles = cycles;
	a.trace = dTrace;
	for(int gi = 0; gi < a.ngroups; ++gi) a.groups[gi].timerBase = uint32_t(m_timerBase);
	launchCycles(a, m_stream);
	NEMO_CUDA(cudaGetLastError());
	m_cycle += cycles;
	m_stateDirty = true;
	std::vector<unsigned long long> h(words);
	NEMO_CUDA(cudaMemcpyAsync(h.data(), dTrace, words * 8, cudaMemcpyDeviceToHost, stream));
	NEMO_CUDA(cudaMemcpyAsync(m_hWords + m_net.nWords, m_net.barrier + 2, 4, cudaMemcpyDeviceToHost, stream));
	NEMO_CUDA(cudaStreamSynchronize(stream));
	cudaFree(dTrace);
	checkDeviceError();
	double acc[14] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
	double gNs = 0, gN = 0, sNs = 0, sN = 0, mNs = 0, uNs = 0, uN = 0, fNs = 0, fN = 0, nNs = 0, nN = 0;
	double lastClaim = 0, exitMean = 0, lastToEnd = 0, lastUnitEnd = 0, blocksClaiming = 0;
	for(unsigned k = 0; k < cycles; ++k) {
		double minT0 = 1e300, maxT4 = 0, maxU = 0, sumU = 0, maxA = 0, sumA = 0, maxR = 0, sumR = 0,
				maxT3 = 0, minT3 = 1e300, sumT4 = 0;
		for(unsigned b = 0; b < m_blocks; ++b) {
			const unsigned long long* r = &h[(size_t(k) * m_blocks + b) * S];
			double t0 = double(r[0]), t2 = double(r[2]), t3 = double(r[3]), t4 = double(r[4]);
			if(r[2] == 0) t2 = t0;   /* the block updates nothing */
			minT0 = std::min(minT0, t0);
			maxT4 = std::max(maxT4, t4);
			maxU = std::max(maxU, t2 - t0);
			sumU += t2 - t0;
			maxA = std::max(maxA, t3 - t0);
			sumA += t3 - t0;
			maxR = std::max(maxR, t3 - t2);
			sumR += t3 - t2;
			maxT3 = std::max(maxT3, t3);
			minT3 = std::min(minT3, t3);
			sumT4 += t4;
			gNs += double(r[5]);
			sNs += double(r[6]);
			gN += double(r[7]);
			sN += double(r[8]);
			mNs += double(r[9]);
			uNs += double(r[10]);
			uN += double(r[11]);
			fNs += double(r[12]);
			fN += double(r[13]);
			nNs += double(r[14]);
			nN += double(r[15]);
			if(r[16] != 0 && r[18] != 0) {
				lastClaim += double(r[16]) - t0;
				exitMean += double(r[17]) / double(r[18]);
				lastUnitEnd += double(r[19]) - t0;
				lastToEnd += t3 - double(r[16]);
				blocksClaiming += 1;
			}
		}
		acc[0] += maxT4 - minT0;
		acc[1] += maxU;
		acc[2] += sumU / m_blocks;
		acc[3] += maxA;
		acc[4] += sumA / m_blocks;
		acc[5] += maxT3 - minT0;
		acc[6] += sumT4 / m_blocks - maxT3;
		acc[7] += maxT3 - minT3;
		acc[8] += maxR;
		acc[9] += sumR / m_blocks;
	}
	for(int i = 0; i < 10; ++i) out[i] = acc[i] / cycles;
	out[10] = gN ? gNs / gN : 0.0;
	out[11] = sN ? sNs / sN : 0.0;
	out[12] = gN / (double(cycles) * m_blocks);
	out[13] = sN / (double(cycles) * m_blocks);
	out[14] = uN ? mNs / uN : 0.0;
	out[15] = uN ? uNs / uN : 0.0;
	out[16] = fN ? fNs / fN : 0.0;
	out[17] = fN / (double(cycles) * m_blocks);
	out[18] = nN ? nNs / nN : 0.0;
	out[19] = nN / (double(cycles) * m_blocks);
	out[20] = blocksClaiming ? lastClaim / blocksClaiming : 0.0;
	out[21] = blocksClaiming ? exitMean / blocksClaiming : 0.0;
	out[22] = blocksClaiming ? lastToEnd / blocksClaiming : 0.0;
	out[23] = blocksClaiming ? lastUnitEnd / blocksClaiming : 0.0;
}

/* Every float in [-104, 89] through the device expf, compared with host
 * glibc expf, in chunks of 2^26 inputs. */
uint64_t
Simulation::expfCheck()
{
	stopResident();
	const ExpExceptions& e = expExceptions();
	cudaStream_t stream = STREAM(m_stream);
	NetDev net = m_net;
	uint64_t* slots = nullptr;
	float* dout = nullptr;
	const uint32_t CHUNK = 1u << 26;
	NEMO_CUDA(cudaMalloc(&slots, e.slots.size() * 8));
	NEMO_CUDA(cudaMalloc(&dout, size_t(CHUNK) * 4));
	NEMO_CUDA(cudaMemcpyAsync(slots, e.slots.data(), e.slots.size() * 8, cudaMemcpyHostToDevice, stream));
	net.expSlots = slots;
	net.expBits = e.slotBits;
	net.expProbe = e.slotProbe;
	net.expNear = e.nearUnits;
	std::vector<float> h(CHUNK);
	uint64_t bad = 0;
	const uint32_t ranges[2][2] = {{0u, libm::f2u(89.0f)}, {0x80000000u, libm::f2u(-104.0f)}};
	unsigned nth = std::max(1u, std::thread::hardware_concurrency());
	for(const auto& rg : ranges) {
		for(uint64_t first = rg[0]; first <= rg[1]; first += CHUNK) {
			const uint32_t n = uint32_t(std::min<uint64_t>(CHUNK, uint64_t(rg[1]) - first + 1));
			launchExpEval(uint32_t(first), n, dout, net, m_stream);
			NEMO_CUDA(cudaMemcpyAsync(h.data(), dout, size_t(n) * 4, cudaMemcpyDeviceToHost, stream));
			NEMO_CUDA(cudaStreamSynchronize(stream));
			std::vector<uint64_t> part(nth, 0);
			std::vector<std::thread> pool;
			for(unsigned w = 0; w < nth; ++w) {
				pool.emplace_back([&, w]() {
					uint64_t b = 0;
					for(uint32_t k = w; k < n; k += nth) {
						volatile float g = expf(libm::u2f(uint32_t(first) + k));
						if(libm::f2u(g) != libm::f2u(h[k])) b++;
					}
					part[w] = b;
				});
			}
			for(auto& th : pool) th.join();
			for(uint64_t b : part) bad += b;
		}
	}
	cudaFree(slots);
	cudaFree(dout);
	return bad;
}

uint64_t
Simulation::libmCheck()
{
	stopResident();
	using namespace libm;
	const LibmTables& t = libmTables();
	cudaStream_t stream = STREAM(m_stream);
	float *dsin, *dlog;
	uint32_t *ds, *dl;
	NEMO_CUDA(cudaMalloc(&dsin, size_t(TABLE_ENTRIES) * 4));
	NEMO_CUDA(cudaMalloc(&dlog, size_t(TABLE_ENTRIES) * 4));
	NEMO_CUDA(cudaMalloc(&ds, t.sinCodes.size() * 4));
	NEMO_CUDA(cudaMalloc(&dl, t.logCodes.size() * 4));
	NEMO_CUDA(cudaMemcpyAsync(ds, t.sinCodes.data(), t.sinCodes.size() * 4, cudaMemcpyHostToDevice, stream));
	NEMO_CUDA(cudaMemcpyAsync(dl, t.logCodes.data(), t.logCodes.size() * 4, cudaMemcpyHostToDevice, stream));
	launchLibmEval(dsin, dlog, ds, dl, m_stream);
	std::vector<float> hs(TABLE_ENTRIES), hl(TABLE_ENTRIES);
	NEMO_CUDA(cudaMemcpyAsync(hs.data(), dsin, size_t(TABLE_ENTRIES) * 4, cudaMemcpyDeviceToHost, stream));
	NEMO_CUDA(cudaMemcpyAsync(hl.data(), dlog, size_t(TABLE_ENTRIES) * 4, cudaMemcpyDeviceToHost, stream));
	NEMO_CUDA(cudaStreamSynchronize(stream));
	cudaFree(dsin);
	cudaFree(dlog);
	cudaFree(ds);
	cudaFree(dl);
	unsigned nth = std::max(1u, std::thread::hardware_concurrency());
	std::vector<uint64_t> bad(nth, 0);
	std::vector<std::thread> pool;
	for(unsigned k = 0; k < nth; ++k) {
		pool.emplace_back([&, k]() {
			for(uint32_t idx = k; idx < TABLE_ENTRIES; idx += nth) {
				float fu = libm_value(idx);
				volatile float gs = sinf(sin_argument(fu));
				volatile float gl = logf(log_argument(fu));
				if(f2u(gs) != f2u(hs[idx]) || f2u(gl) != f2u(hl[idx])) bad[k]++;
			}
		});
	}
	for(auto& th : pool) th.join();
	uint64_t total = 0;
	for(uint64_t b : bad) total += b;
	return total;
}

void
hhDivisionCheck(uint64_t mismatches[3])
{
	unsigned long long* bad = nullptr;
	NEMO_CUDA(cudaMalloc(&bad, 3 * sizeof(unsigned long long)));
	NEMO_CUDA(cudaMemset(bad, 0, 3 * sizeof(unsigned long long)));
	launchHhDivCheck(bad, nullptr);
	unsigned long long h[3] = {0, 0, 0};
	const cudaError_t err = cudaMemcpy(h, bad, sizeof(h), cudaMemcpyDeviceToHost);
	cudaFree(bad);
	NEMO_CUDA(err);
	for(int q = 0; q < 3; ++q) mismatches[q] = h[q];
}

void
shardWarps(uint32_t totalWarps, unsigned rank, unsigned world, uint32_t* lo, uint32_t* hi)
{
	if(world == 0 || rank >= world) {
		fail(NEMO_INVALID_INPUT, "Shard: rank " + std::to_string(rank) + " of " + std::to_string(world));
	}
	const uint32_t q = totalWarps / world, r = totalWarps % world;
	*lo = rank * q + std::min<uint32_t>(rank, r);
	*hi = *lo + q + (rank < r ? 1u : 0u);
}

Network
shardNetwork(const Network& net, unsigned rank, unsigned world, ShardSpec* spec)
{
	/* the device layout of Simulation's constructor */
	std::unordered_map<uint32_t, uint32_t> g2d;
	uint64_t devPos = 0;
	for(const NeuronGroup& ng : net.groups) {
		const uint32_t n = uint32_t(ng.gidx.size());
		if(n == 0) continue;
		const uint32_t shift = ng.type.kind == MODEL_HH ? 3u : 0u;
		for(uint32_t i = 0; i < n; ++i) g2d.emplace(ng.gidx[i], uint32_t(devPos + (uint64_t(i) << shift)));
		devPos = roundUp(devPos + (uint64_t(n) << shift), 32);
	}
	const uint32_t total = uint32_t(std::max<uint64_t>(devPos, 32) / 32);
	ShardSpec sp;
	sp.rank = rank;
	sp.world = world;
	sp.totalWarps = total;
	sp.maxDelay = net.maxDelay();
	shardWarps(total, rank, world, &sp.warpLo, &sp.warpHi);
	*spec = sp;
	return net.subsetByTarget([&](uint32_t tgt) {
		auto it = g2d.find(tgt);
		return it != g2d.end() && it->second / 32 >= sp.warpLo && it->second / 32 < sp.warpHi;
	});
}

} // namespace nemo_b200
