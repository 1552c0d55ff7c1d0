/* ORACLE — TEST INFRASTRUCTURE ONLY (see oracle.hpp).
 *
 * Network construction, restating src/nemo/NetworkImpl.cpp, Neurons.cpp,
 * Axon.cpp and Network.cpp. */

#include "oracle.hpp"

#include <algorithm>
#include <limits>
#include <sstream>

namespace oracle {

Network::Network() :
	minIdx(std::numeric_limits<int>::max()),
	maxIdx(std::numeric_limits<int>::min()),
	m_maxDelay(0), minWeight(0), maxWeight(0), izType(~0U)
{
}

/* NetworkImpl.cpp:428-438: registering an existing name returns its id */
unsigned
Network::addNeuronType(const std::string& name)
{
	auto it = typeIds.find(name);
	if(it != typeIds.end()) {
		return it->second;
	}
	NeuronGroup g;
	g.type = neuronType(name);
	g.param.resize(g.type.nParam);
	g.state.resize(g.type.nState);
	unsigned id = unsigned(groups.size());
	groups.push_back(g);
	typeIds[name] = id;
	return id;
}

/* NetworkImpl.cpp:471-476 and Neurons.cpp:29-48. The neuron is appended to
 * its type before the duplicate-index check, as in the reference. */
void
Network::addNeuron(unsigned type, unsigned gidx, unsigned nargs, const float args[])
{
	maxIdx = std::max(maxIdx, int(gidx));
	minIdx = std::min(minIdx, int(gidx));
	if(type >= groups.size()) {
		std::ostringstream msg;
		msg << "Invalid neuron type id " << type;
		throw Error(NEMO_INVALID_INPUT, msg.str());
	}
	NeuronGroup& g = groups[type];
	if(nargs != g.type.nParam + g.type.nState) {
		std::ostringstream msg;
		msg << "Unexpected number of parameters/state variables when adding neuron. Expected "
			<< g.type.nParam + g.type.nState << ", found " << nargs;
		throw Error(NEMO_INVALID_INPUT, msg.str());
	}
	for(unsigned i = 0; i < g.type.nParam; ++i) g.param[i].push_back(*args++);
	for(unsigned i = 0; i < g.type.nState; ++i) g.state[i].push_back(*args++);
	g.gidx.push_back(gidx);
	unsigned index = unsigned(g.gidx.size() - 1);
	if(!mapper.emplace(gidx, std::make_pair(type, index)).second) {
		std::ostringstream msg;
		msg << "Duplicate neuron index " << gidx;
		throw Error(NEMO_INVALID_INPUT, msg.str());
	}
}

std::pair<unsigned, unsigned>
Network::address(unsigned gidx) const
{
	auto it = mapper.find(gidx);
	if(it == mapper.end()) {
		std::ostringstream msg;
		msg << "Non-existing neuron index " << gidx;
		throw Error(NEMO_INVALID_INPUT, msg.str());
	}
	return it->second;
}

/* Neurons.cpp:78-95 */
void
Network::setNeuron(unsigned gidx, unsigned nargs, const float args[])
{
	auto a = address(gidx);
	NeuronGroup& g = groups[a.first];
	if(nargs != g.type.nParam + g.type.nState) {
		std::ostringstream msg;
		msg << "Unexpected number of parameters/state variables when modifying neuron. Expected "
			<< g.type.nParam + g.type.nState << ", found " << nargs;
		throw Error(NEMO_INVALID_INPUT, msg.str());
	}
	for(unsigned i = 0; i < g.type.nParam; ++i) g.param[i][a.second] = *args++;
	for(unsigned i = 0; i < g.type.nState; ++i) g.state[i][a.second] = *args++;
}

static void
checkIndex(unsigned i, unsigned n, const char* what)
{
	if(i >= n) {
		std::ostringstream msg;
		msg << "Invalid " << what << " index " << i;
		throw Error(NEMO_INVALID_INPUT, msg.str());
	}
}

float
Network::getNeuronState(unsigned gidx, unsigned var) const
{
	auto a = address(gidx);
	const NeuronGroup& g = groups[a.first];
	checkIndex(var, g.type.nState, "state variable");
	return g.state[var][a.second];
}

float
Network::getNeuronParameter(unsigned gidx, unsigned param) const
{
	auto a = address(gidx);
	const NeuronGroup& g = groups[a.first];
	checkIndex(param, g.type.nParam, "parameter");
	return g.param[param][a.second];
}

void
Network::setNeuronState(unsigned gidx, unsigned var, float val)
{
	auto a = address(gidx);
	NeuronGroup& g = groups[a.first];
	checkIndex(var, g.type.nState, "state variable");
	g.state[var][a.second] = val;
}

void
Network::setNeuronParameter(unsigned gidx, unsigned param, float val)
{
	auto a = address(gidx);
	NeuronGroup& g = groups[a.first];
	checkIndex(param, g.type.nParam, "parameter");
	g.param[param][a.second] = val;
}

/* NetworkImpl.cpp:492-511 and Axon.cpp:9-19 */
synapse_id
Network::addSynapse(unsigned source, unsigned target, unsigned delay, float weight, unsigned char plastic)
{
	if(delay < 1) {
		std::ostringstream msg;
		msg << "Invalid delay (" << delay << ") for synapse between " << source << " and " << target;
		throw Error(NEMO_INVALID_INPUT, msg.str());
	}
	Axon& ax = fcm[source];
	uint32_t id = uint32_t(ax.targets.size());
	ax.targets.push_back(target);
	ax.delays.push_back(delay);
	ax.weights.push_back(weight);
	ax.plastic.push_back(plastic != 0);
	maxIdx = std::max(maxIdx, int(std::max(source, target)));
	minIdx = std::min(minIdx, int(std::min(source, target)));
	m_maxDelay = std::max(m_maxDelay, delay);
	maxWeight = std::max(maxWeight, weight);
	minWeight = std::min(minWeight, weight);
	return (uint64_t(source) << 32) | uint64_t(id);
}

/* NetworkImpl.cpp:533-541 */
const Axon&
Network::axon(unsigned source) const
{
	auto it = fcm.find(source);
	if(it == fcm.end()) {
		std::ostringstream msg;
		msg << "synapses of non-existing neuron (" << source << ") requested";
		throw Error(NEMO_INVALID_INPUT, msg.str());
	}
	return it->second;
}

/* NetworkImpl.cpp:559-569: unknown sources give an empty list */
const std::vector<synapse_id>&
Network::getSynapsesFrom(unsigned source)
{
	m_queried.clear();
	auto it = fcm.find(source);
	if(it != fcm.end()) {
		size_t n = it->second.targets.size();
		m_queried.resize(n);
		for(size_t i = 0; i < n; ++i) {
			m_queried[i] = (uint64_t(source) << 32) | uint64_t(i);
		}
	}
	return m_queried;
}

unsigned
Network::neuronCount() const
{
	unsigned total = 0;
	for(const NeuronGroup& g : groups) total += unsigned(g.gidx.size());
	return total;
}

} // namespace oracle
