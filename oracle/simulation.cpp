/* ORACLE — TEST INFRASTRUCTURE ONLY (see oracle.hpp).
 *
 * The CPU step loop and connectivity, restating src/nemo/cpu/Simulation.cpp,
 * src/nemo/cpu/Neurons.cpp, src/nemo/ConnectivityMatrix.cpp,
 * src/nemo/construction/RCM.cpp, src/nemo/runtime/RCM.cpp,
 * src/nemo/OutgoingDelays.cpp and src/nemo/nemo.cpp:110-134.
 *
 * Containers differ from the reference (flat CSR arrays instead of std::map
 * and boost::unordered_map) but every observable ordering is kept: synapses
 * are visited source-major in ascending user index and per-source insertion
 * order (NetworkImpl.cpp:225-247), rows keep that order, fired neurons are
 * reported in ascending simulation index. Neuron getters and setters use the
 * type-local index; the reference passes the simulation index there
 * (cpu/Simulation.cpp:221-247), which only coincides for the first type. */

#include "oracle.hpp"

#include <algorithm>
#include <chrono>
#include <sstream>

namespace oracle {

static double
nowMs()
{
	using namespace std::chrono;
	return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

static inline uint64_t shl64(uint64_t x, unsigned n) { return x << (n & 63); }
static inline uint64_t shr64(uint64_t x, unsigned n) { return x >> (n & 63); }

/* src/nemo/nemo.cpp:110-134 (checks) and src/nemo/cpu/Simulation.cpp:36-82 */
Simulation::Simulation(const Network& net, const Configuration& conf) :
	m_neuronCount(net.neuronCount()),
	m_fbits(conf.fractionalBits),
	m_maxDelay(0),
	m_stdpOn(conf.hasStdp),
	m_writeOnly(conf.writeOnlySynapses),
	m_cycles(0)
{
	if(m_neuronCount == 0) {
		throw Error(NEMO_INVALID_INPUT, "Cannot create simulation from empty network");
	}
	if(conf.hasStdp) {
		conf.stdp[0].verifyDynamicWindowLength(net.maxDelay());
	}
	if(net.maxDelay() > 64) {
		std::ostringstream msg;
		msg << "The network has synapses with delay " << net.maxDelay()
			<< "ms. The CPU backend supports a maximum of 64 ms";
		throw Error(NEMO_INVALID_INPUT, msg.str());
	}

	const unsigned N = m_neuronCount;
	m_fired.assign(N, 0);
	m_recentFiring.assign(N, 0);
	m_delays.assign(N, 0);
	mfx_currentE.assign(N, 0);
	mfx_currentI.assign(N, 0);
	m_currentE.assign(N, 0.0f);
	m_currentI.assign(N, 0.0f);
	m_currentExt.assign(N, 0.0f);
	m_fstim.assign(N, 0);

	/* contiguous simulation indices, types in registration order
	 * (cpu/Simulation.cpp:58-73, cpu/Neurons.cpp:7-48) */
	unsigned l_idx = 0;
	for(unsigned t = 0; t < net.groups.size(); ++t) {
		m_typeBase.push_back(l_idx);
		const NeuronGroup& ng = net.groups[t];
		unsigned n = unsigned(ng.gidx.size());
		if(n == 0) {
			continue;
		}
		Group g;
		g.type = ng.type;
		g.base = l_idx;
		g.size = n;
		g.param.resize(size_t(ng.type.nParam) * n);
		g.state.resize(size_t(ng.type.nState) * n);
		for(unsigned p = 0; p < ng.type.nParam; ++p)
			std::copy(ng.param[p].begin(), ng.param[p].end(), g.param.begin() + size_t(p) * n);
		for(unsigned s = 0; s < ng.type.nState; ++s)
			std::copy(ng.state[s].begin(), ng.state[s].end(), g.state.begin() + size_t(s) * n);
		for(unsigned i = 0; i < n; ++i) {
			unsigned sim = l_idx + i;
			if(!m_g2l.emplace(ng.gidx[i], sim).second) {
				std::ostringstream msg;
				msg << "Duplicate neuron index " << ng.gidx[i];
				throw Error(NEMO_INVALID_INPUT, msg.str());
			}
			m_l2g.push_back(ng.gidx[i]);
			m_typeOfLocal.push_back(unsigned(m_groups.size()));
		}
		g.rng.resize(n);
		initialiseRng(l_idx, l_idx + n - 1, g.rng);
		m_groups.push_back(std::move(g));
		l_idx += n;
	}

	/* ---- connectivity (ConnectivityMatrix.cpp:65-193) ---- */
	if(m_stdpOn) {
		m_stdp.emplace_back(conf.stdp[0], m_fbits);
	}

	/* pass 1: validate in iteration order, find max delay, count rows */
	size_t nsyn = 0;
	for(const auto& kv : net.fcm) {
		const Axon& ax = kv.second;
		for(size_t i = 0; i < ax.targets.size(); ++i) {
			localIdx(kv.first);
			localIdx(ax.targets[i]);
			fx_toFix(ax.weights[i], m_fbits);
			m_maxDelay = std::max(m_maxDelay, ax.delays[i]);
			nsyn++;
		}
	}

	size_t nrows = size_t(N) * m_maxDelay;
	std::vector<size_t> rowCount(nrows + 1, 0);
	std::vector<size_t> rcmCount(size_t(N) + 1, 0);
	for(const auto& kv : net.fcm) {
		unsigned src = localIdx(kv.first);
		const Axon& ax = kv.second;
		for(size_t i = 0; i < ax.targets.size(); ++i) {
			rowCount[addressOf(src, ax.delays[i])]++;
			if(m_stdpOn && ax.plastic[i]) {
				rcmCount[localIdx(ax.targets[i])]++;
			}
		}
	}
	m_rowStart.assign(nrows + 1, 0);
	for(size_t r = 0; r < nrows; ++r) m_rowStart[r + 1] = m_rowStart[r] + rowCount[r];
	m_terminals.resize(nsyn);
	m_rcmStart.assign(size_t(N) + 1, 0);
	for(size_t t = 0; t < N; ++t) m_rcmStart[t + 1] = m_rcmStart[t] + rcmCount[t];
	size_t nrcm = m_rcmStart[N];
	m_rcmSource.resize(nrcm);
	m_rcmDelay.resize(nrcm);
	m_rcmForward.resize(nrcm);
	m_rcmAcc.assign(nrcm, 0);
	if(!m_writeOnly) {
		m_aux.resize(nsyn);
	}

	/* pass 2: fill rows (insertion order), RCM and query data */
	std::vector<size_t> rowFill(m_rowStart.begin(), m_rowStart.end() - 1);
	std::vector<size_t> rcmFill(m_rcmStart.begin(), m_rcmStart.end() - 1);
	size_t auxPos = 0;
	for(const auto& kv : net.fcm) {
		unsigned src = localIdx(kv.first);
		const Axon& ax = kv.second;
		if(!m_writeOnly) {
			m_auxRange[kv.first] = std::make_pair(auxPos, ax.targets.size());
		}
		for(size_t i = 0; i < ax.targets.size(); ++i) {
			unsigned delay = ax.delays[i];
			unsigned tgt = localIdx(ax.targets[i]);
			size_t r = addressOf(src, delay);
			size_t pos = rowFill[r]++;
			unsigned sidx = unsigned(pos - m_rowStart[r]);
			m_terminals[pos].target = tgt;
			m_terminals[pos].weight = fx_toFix(ax.weights[i], m_fbits);
			m_delays[src] |= uint64_t(1) << (delay - 1); /* OutgoingDelays.cpp:74-85 */
			if(!m_writeOnly) {
				m_aux[auxPos + i] = Aux{sidx, delay, ax.plastic[i] != 0};
			}
			if(m_stdpOn && ax.plastic[i]) {
				size_t j = rcmFill[tgt]++;
				m_rcmSource[j] = src;
				m_rcmDelay[j] = delay;
				m_rcmForward[j] = sidx;
			}
		}
		auxPos += ax.targets.size();
	}

	resetTimer();
}

unsigned
Simulation::localIdx(unsigned gidx) const
{
	auto it = m_g2l.find(gidx);
	if(it == m_g2l.end()) {
		std::ostringstream msg;
		msg << "Non-existing neuron index " << gidx;
		throw Error(NEMO_INVALID_INPUT, msg.str());
	}
	return it->second;
}

unsigned
Simulation::globalIdx(unsigned lidx) const
{
	return m_l2g.at(lidx);
}

const Simulation::Group&
Simulation::groupOf(unsigned lidx, unsigned* nl) const
{
	const Group& g = m_groups.at(m_typeOfLocal.at(lidx));
	*nl = lidx - g.base;
	return g;
}

Simulation::Group&
Simulation::groupOf(unsigned lidx, unsigned* nl)
{
	Group& g = m_groups.at(m_typeOfLocal.at(lidx));
	*nl = lidx - g.base;
	return g;
}

/* cpu/Simulation.cpp:140-147 */
void
Simulation::setFiringStimulus(const std::vector<unsigned>& fstim)
{
	for(unsigned n : fstim) {
		m_fstim.at(localIdx(n)) = 1;
	}
}

/* cpu/Simulation.cpp:159-163 */
void
Simulation::addCurrentStimulus(unsigned gidx, float current)
{
	m_currentExt[localIdx(gidx)] = current;
}

/* cpu/Simulation.cpp:259-308 */
void
Simulation::deliverSpikes()
{
	uint64_t validSpikes = ~shl64(~uint64_t(0), m_maxDelay);
	for(size_t source = 0; source < m_neuronCount; ++source) {
		uint64_t f = m_recentFiring[source] & validSpikes & m_delays[source];
		unsigned delay = 0;
		while(f) {
			unsigned shift = 1 + unsigned(__builtin_ctzll(f));
			delay += shift;
			f = shr64(f, shift);
			size_t r = addressOf(unsigned(source), delay);
			for(size_t s = m_rowStart[r]; s < m_rowStart[r + 1]; ++s) {
				const FAxonTerminal& term = m_terminals[s];
				std::vector<wfix_t>& current = term.weight >= 0 ? mfx_currentE : mfx_currentI;
				current.at(term.target) += term.weight;
			}
		}
	}
	int ncount = int(m_neuronCount);
#pragma omp parallel for default(shared)
	for(int n = 0; n < ncount; n++) {
		m_currentE[n] = wfx_toFloat(mfx_currentE[n], m_fbits);
		mfx_currentE[n] = 0;
		m_currentI[n] = wfx_toFloat(mfx_currentI[n], m_fbits);
		mfx_currentI[n] = 0;
	}
}

/* ConnectivityMatrix.cpp:224-258 */
void
Simulation::accumulateStdp()
{
	if(!m_stdpOn) {
		return;
	}
	const StdpProcess& stdp = m_stdp[0];
	for(size_t target = 0; target < m_neuronCount; ++target) {
		if(m_rcmStart[target] == m_rcmStart[target + 1]) continue;
		if(m_recentFiring[target] & stdp.postFireMask()) {
			for(size_t j = m_rcmStart[target]; j < m_rcmStart[target + 1]; ++j) {
				uint64_t preFiring = shr64(m_recentFiring[m_rcmSource[j]], m_rcmDelay[j]);
				fix_t w_diff = stdp.weightChange(preFiring);
				if(w_diff != 0) {
					m_rcmAcc[j] = fix_t(uint32_t(m_rcmAcc[j]) + uint32_t(w_diff));
				}
			}
		}
	}
}

/* cpu/Simulation.cpp:199-209 */
void
Simulation::setFiring()
{
	m_firedList.clear();
	for(unsigned n = 0; n < m_neuronCount; ++n) {
		if(m_fired[n]) {
			m_firedList.push_back(globalIdx(n));
		}
	}
}

/* cpu/Simulation.cpp:94-111, cpu/Neurons.cpp:111-137 */
void
Simulation::fire()
{
	deliverSpikes();
	for(Group& g : m_groups) {
		unsigned nP = g.type.nParam, nS = g.type.nState;
		g.type.update(g.base, g.base + g.size, unsigned(m_cycles),
				g.param.data(), g.size,
				g.state.data(), size_t(nS) * g.size, g.size,
				m_fbits, m_fstim.data(), g.rng.data(),
				m_currentE.data(), m_currentI.data(), m_currentExt.data(),
				m_recentFiring.data(), m_fired.data(), nullptr);
		(void) nP;
	}
	accumulateStdp();
	setFiring();
	m_cycles++;
}

const std::vector<unsigned>&
Simulation::readFiring()
{
	return m_firedList;
}

/* ConnectivityMatrix.cpp:272-325 */
void
Simulation::applyStdp(float reward)
{
	if(!m_stdpOn) {
		throw Error(NEMO_LOGIC_ERROR, "applyStdp called, but no STDP model specified");
	}
	fix_t fx_reward = fx_toFix(reward, m_fbits);
	if(fx_reward == 0 && reward != 0) {
		std::ostringstream msg;
		msg << "STDP reward rounded down to zero. The smallest valid reward is "
			<< fx_toFloat(1, m_fbits);
		throw Error(NEMO_INVALID_INPUT, msg.str());
	}
	if(fx_reward == 0) {
		std::fill(m_rcmAcc.begin(), m_rcmAcc.end(), 0);
	}
	const StdpProcess& stdp = m_stdp[0];
	for(size_t j = 0; j < m_rcmAcc.size(); ++j) {
		size_t r = addressOf(m_rcmSource[j], m_rcmDelay[j]);
		fix_t& w_old = m_terminals[m_rowStart[r] + m_rcmForward[j]].weight;
		fix_t w_new = stdp.updatedWeight(w_old, fx_mul(fx_reward, m_rcmAcc[j], m_fbits));
		if(w_old != w_new) {
			w_old = w_new;
		}
		m_rcmAcc[j] = 0;
	}
}

static void
checkVar(unsigned i, unsigned n, const char* what)
{
	if(i >= n) {
		std::ostringstream msg;
		msg << "Invalid " << what << " index " << i;
		throw Error(NEMO_INVALID_INPUT, msg.str());
	}
}

float
Simulation::getNeuronState(unsigned gidx, unsigned var) const
{
	unsigned nl;
	const Group& g = groupOf(localIdx(gidx), &nl);
	checkVar(var, g.type.nState, "state variable");
	return g.state[size_t(var) * g.size + nl];
}

float
Simulation::getNeuronParameter(unsigned gidx, unsigned param) const
{
	unsigned nl;
	const Group& g = groupOf(localIdx(gidx), &nl);
	checkVar(param, g.type.nParam, "parameter");
	return g.param[size_t(param) * g.size + nl];
}

float
Simulation::getMembranePotential(unsigned gidx) const
{
	unsigned nl;
	const Group& g = groupOf(localIdx(gidx), &nl);
	return getNeuronState(gidx, g.type.membranePotential);
}

void
Simulation::setNeuron(unsigned gidx, unsigned nargs, const float args[])
{
	unsigned nl;
	Group& g = groupOf(localIdx(gidx), &nl);
	if(nargs != g.type.nParam + g.type.nState) {
		std::ostringstream msg;
		msg << "Unexpected number of parameters/state variables when modifying neuron. Expected "
			<< g.type.nParam + g.type.nState << ", found " << nargs;
		throw Error(NEMO_INVALID_INPUT, msg.str());
	}
	for(unsigned p = 0; p < g.type.nParam; ++p) g.param[size_t(p) * g.size + nl] = args[p];
	for(unsigned s = 0; s < g.type.nState; ++s) g.state[size_t(s) * g.size + nl] = args[g.type.nParam + s];
}

void
Simulation::setNeuronState(unsigned gidx, unsigned var, float val)
{
	unsigned nl;
	Group& g = groupOf(localIdx(gidx), &nl);
	checkVar(var, g.type.nState, "state variable");
	g.state[size_t(var) * g.size + nl] = val;
}

void
Simulation::setNeuronParameter(unsigned gidx, unsigned param, float val)
{
	unsigned nl;
	Group& g = groupOf(localIdx(gidx), &nl);
	checkVar(param, g.type.nParam, "parameter");
	g.param[size_t(param) * g.size + nl] = val;
}

/* ConnectivityMatrix.cpp:329-362 */
const std::vector<synapse_id>&
Simulation::getSynapsesFrom(unsigned source)
{
	if(m_writeOnly) {
		throw Error(NEMO_INVALID_INPUT, "Cannot read synapse state if simulation configured with write-only synapses");
	}
	size_t n = 0;
	auto it = m_auxRange.find(source);
	if(it == m_auxRange.end()) {
		if(m_g2l.find(source) == m_g2l.end()) {
			std::ostringstream msg;
			msg << "Non-existing source neuron id (" << source << ") in synapse id query";
			throw Error(NEMO_INVALID_INPUT, msg.str());
		}
	} else {
		n = it->second.second;
	}
	m_queried.resize(n);
	for(size_t i = 0; i < n; ++i) {
		m_queried[i] = (uint64_t(source) << 32) | uint64_t(i);
	}
	return m_queried;
}

/* ConnectivityMatrix.cpp:374-391 */
const Simulation::Aux&
Simulation::aux(synapse_id id) const
{
	if(m_writeOnly) {
		throw Error(NEMO_INVALID_INPUT, "Cannot read synapse state if simulation configured with write-only synapses");
	}
	unsigned neuron = unsigned(id >> 32);
	auto it = m_auxRange.find(neuron);
	if(it == m_auxRange.end()) {
		std::ostringstream msg;
		msg << "Non-existing neuron id (" << neuron << ") in synapse query";
		throw Error(NEMO_INVALID_INPUT, msg.str());
	}
	size_t idx = size_t(id & 0xffffffff);
	if(idx >= it->second.second) {
		throw std::out_of_range("synapse index out of range"); /* vector::at in the reference */
	}
	return m_aux[it->second.first + idx];
}

unsigned
Simulation::getSynapseTarget(synapse_id id) const
{
	const Aux& s = aux(id);
	unsigned src = localIdx(unsigned(id >> 32));
	return globalIdx(m_terminals[m_rowStart[addressOf(src, s.delay)] + s.idx].target);
}

unsigned
Simulation::getSynapseDelay(synapse_id id) const
{
	return aux(id).delay;
}

float
Simulation::getSynapseWeight(synapse_id id) const
{
	const Aux& s = aux(id);
	unsigned src = localIdx(unsigned(id >> 32));
	return fx_toFloat(m_terminals[m_rowStart[addressOf(src, s.delay)] + s.idx].weight, m_fbits);
}

/* getSynapseWeight over many ids, with the per-source lookups made once per
 * run of ids from the same source (the tests read every weight of large
 * networks) */
void
Simulation::getWeights(const synapse_id* ids, size_t n, float* out) const
{
	bool have = false;
	unsigned last = 0, src = 0;
	size_t first = 0, count = 0;
	for(size_t k = 0; k < n; ++k) {
		const unsigned neuron = unsigned(ids[k] >> 32);
		if(!have || neuron != last) {
			(void) aux(ids[k] & ~uint64_t(0xffffffffu));   /* errors of the single query */
			auto it = m_auxRange.find(neuron);
			first = it->second.first;
			count = it->second.second;
			src = localIdx(neuron);
			last = neuron;
			have = true;
		}
		const size_t idx = size_t(ids[k] & 0xffffffffu);
		if(idx >= count) {
			throw std::out_of_range("synapse index out of range");
		}
		const Aux& a = m_aux[first + idx];
		out[k] = fx_toFloat(m_terminals[m_rowStart[addressOf(src, a.delay)] + a.idx].weight, m_fbits);
	}
}

unsigned char
Simulation::getSynapsePlastic(synapse_id id) const
{
	return aux(id).plastic;
}

unsigned long
Simulation::elapsedWallclock() const
{
	return (unsigned long) (nowMs() - m_wallStart);
}

void
Simulation::resetTimer()
{
	m_wallStart = nowMs();
	m_cycles = 0;
}

} // namespace oracle
