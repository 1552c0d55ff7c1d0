#ifndef NEMO_B200_NETWORK_HPP
#define NEMO_B200_NETWORK_HPP

/* Host-side network description and configuration: the data behind the
 * nemo::Network and nemo::Configuration classes of the reference
 * (src/nemo/NetworkImpl.cpp, Neurons.cpp, Axon.cpp, ConfigurationImpl.cpp,
 * StdpFunction.cpp, NeuronType.cpp).
 *
 * Synapses are kept in flat insertion-order arrays (13 bytes each) rather than
 * per-source containers, so that networks of 1e8+ synapses build in seconds;
 * the per-source synapse ids of the reference ((source << 32) | index) are
 * preserved. */

#include <cstdint>
#include <functional>
#include <string>
#include <unordered_map>
#include <vector>

#include "common.hpp"

namespace nemo_b200 {

/* Built-in neuron models with B200 kernels. */
enum ModelKind {
	MODEL_IZHIKEVICH,
	MODEL_IF_CURR_EXP,
	MODEL_QIF,
	MODEL_HH,
	MODEL_POISSON_SOURCE,
	MODEL_INPUT,
	MODEL_EXTERNAL,   /* a plugin's kernels (nemo_b200_plugin.h) */
	MODEL_COUNT
};

/* Descriptor parsed from <name>.ini (the keys of src/nemo/NeuronType.cpp:94-158) */
struct NeuronType {
	std::string name;
	unsigned nParam = 0;
	unsigned nState = 0;
	unsigned membranePotential = 0;
	unsigned history = 1;
	bool nrand = false;
	bool rcmSources = false, rcmDelays = false, rcmForward = false, rcmWeights = false;
	bool backendCpu = false, backendCuda = false;
	std::string pluginDir;
	ModelKind kind = MODEL_COUNT;
	std::string b200Plugin;   /* MODEL_EXTERNAL: <pluginDir>/b200/lib<name>.so */
};

void addPluginPath(const std::string& dir);
NeuronType loadNeuronType(const std::string& name);

struct StdpFunction {
	StdpFunction() {}
	StdpFunction(const std::vector<float>& pre, const std::vector<float>& post,
			float minE, float maxE, float minI, float maxI);
	void verifyDynamicWindowLength(unsigned dmax) const;
	uint64_t potentiationBits() const;
	uint64_t depressionBits() const;
	std::vector<float> prefire, postfire;
	float minE = 0, maxE = 0, minI = 0, maxI = 0;
};

struct Configuration {
	bool logging = false;
	bool writeOnlySynapses = false;
	unsigned fractionalBits = 20;
	int cudaDevice = -1;
	bool hasStdp = false;
	StdpFunction stdp;
	std::string description = "B200 backend (sm_100a)";
};

struct NeuronGroup {
	NeuronType type;
	std::vector<std::vector<float>> param;  /* [nParam][n] */
	std::vector<std::vector<float>> state;  /* [nState][n] */
	std::vector<uint32_t> gidx;
};

class Network {
public:
	unsigned addNeuronType(const std::string& name);
	void addNeuron(unsigned type, unsigned gidx, unsigned nargs, const float* args);
	void setNeuron(unsigned gidx, unsigned nargs, const float* args);
	synapse_id addSynapse(unsigned source, unsigned target, unsigned delay, float weight, unsigned char plastic);

	float getNeuronState(unsigned gidx, unsigned var) const;
	float getNeuronParameter(unsigned gidx, unsigned param) const;
	void setNeuronState(unsigned gidx, unsigned var, float val);
	void setNeuronParameter(unsigned gidx, unsigned param, float val);

	/* synapse queries by id (src/nemo/NetworkImpl.cpp:533-569) */
	size_t synapsePosition(synapse_id id) const;
	const std::vector<synapse_id>& getSynapsesFrom(unsigned source);

	unsigned neuronCount() const;
	unsigned maxDelay() const { return m_maxDelay; }
	size_t synapseCount() const { return src.size(); }

	/* A batch: independent networks as one, instance j's user indices
	 * shifted by base[j] (base has one entry per instance and a final end);
	 * synapses never cross instances. seedKey[g][i] is (instance << 32) |
	 * simulation index within the instance for neuron i of group g, so that
	 * each instance's neurons get the random seeds they would get alone. */
	static Network merge(const std::vector<const Network*>& nets, std::vector<uint32_t>* base);

	/* Every neuron and the synapses whose target `keepTarget` accepts, in
	 * their order, with their ids; the maximum delay stays this network's
	 * (it decides delivery for every synapse). The network one shard of a
	 * sharded simulation builds. */
	Network subsetByTarget(const std::function<bool(uint32_t)>& keepTarget) const;
	std::vector<std::vector<uint64_t>> seedKey;

	std::vector<NeuronGroup> groups;
	std::unordered_map<std::string, unsigned> typeIds;
	std::unordered_map<uint32_t, std::pair<uint32_t, uint32_t>> mapper; /* gidx -> (type, index) */
	unsigned izType = ~0u;

	/* synapses in insertion order */
	std::vector<uint32_t> src, tgt, dly;
	std::vector<float> wgt;
	std::vector<uint8_t> plastic;
	std::vector<uint32_t> sid;   /* per-source index, i.e. the low word of the synapse id */

	/* per-source insertion-order positions (built on demand) */
	void indexBySource() const;
	mutable bool m_indexed = false;
	mutable std::unordered_map<uint32_t, std::pair<size_t, uint32_t>> m_srcRange; /* gidx -> (offset, count) */
	mutable std::vector<size_t> m_bySource;

private:
	std::pair<uint32_t, uint32_t> address(unsigned gidx) const;
	std::unordered_map<uint32_t, uint32_t> m_srcCount;
	uint32_t m_lastSrc = ~0u;
	uint32_t* m_lastCount = nullptr;
	unsigned m_maxDelay = 0;
	std::vector<synapse_id> m_queried;
};

} // namespace nemo_b200

#endif
