#ifndef NEMO_ORACLE_HPP
#define NEMO_ORACLE_HPP

/* ORACLE — TEST INFRASTRUCTURE ONLY.
 *
 * A Boost-free CPU restatement of the reference NeMo 0.7.2 CPU backend
 * (src/nemo/cpu/, src/nemo/ConnectivityMatrix.cpp, StdpProcess.cpp,
 * fixedpoint.cpp, RNG.cpp, the CPU neuron plugins). It exports the same C ABI
 * as the product (include/nemo.h) so that the same test code drives both.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * it, always as the checker or the timed CPU baseline, never as part of the
 * product path.
 *
 * Parity pins: the reference's known-answer tests (ring networks, firing and
 * current stimulus, fixed-point saturation, the analytic STDP test,
 * src/test/test.cpp, src/test/stdp.cpp) run against this restatement, and its
 * neuron updates are compared bit for bit with the reference's own CPU
 * plugin sources compiled into oracle/_ref/ (see oracle/Makefile). The
 * reference library as a whole cannot be built here (Boost and libltdl are
 * missing), so whole-simulation outputs of the reference are not available. */

#include <cstdint>
#include <cstddef>
#include <map>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include <nemo/types.h>

namespace oracle {

/* nemo::exception (src/nemo/exception.hpp:10-30) */
struct Error : public std::runtime_error {
	Error(int code, const std::string& msg) : std::runtime_error(msg), code(code) {}
	int code;
};

typedef int32_t fix_t;
typedef int64_t wfix_t;

/* src/nemo/fixedpoint.cpp:17-49, fixedpoint.hpp:86-99 */
fix_t fx_toFix(float f, unsigned fbits);
float fx_toFloat(fix_t v, unsigned fbits);
float wfx_toFloat(wfix_t v, unsigned fbits);
inline fix_t fx_mul(fix_t a, fix_t b, unsigned fbits) {
	int64_t r = int64_t(a) * int64_t(b);
	return fix_t(r >> fbits);
}
const fix_t fx_min = fix_t(uint32_t(1) << 31);
const fix_t fx_max = ~fix_t(uint32_t(1) << 31);

/* src/nemo/RNG.hpp:9-11 */
struct RNG { unsigned state[4]; };

/* src/nemo/RNG.cpp:39-62: per-neuron seeds for local indices [minIdx, maxIdx] */
void initialiseRng(unsigned minIdx, unsigned maxIdx, std::vector<RNG>& rngs);

} // namespace oracle

extern "C" {
/* src/nemo/RNG.cpp:10-34 (extern "C" in the reference as well) */
unsigned urand(oracle::RNG* rng);
float nrand(oracle::RNG* rng);
}

namespace oracle {

/* The CPU neuron-model plugin signature (src/nemo/cpu/plugins/neuron_model.h:25-38) */
typedef void cpu_update_neurons_t(
		unsigned start, unsigned end,
		unsigned cycle,
		float* paramBase, size_t paramStride,
		float* stateBase, size_t stateHistoryStride, size_t stateVarStride,
		unsigned fbits,
		unsigned fstim[],
		RNG rng[],
		float currentEPSP[],
		float currentIPSP[],
		float currentExternal[],
		uint64_t recentFiring[],
		unsigned fired[],
		void* rcm);

/* Neuron-type descriptor: the fields of the plugin .ini files
 * (src/nemo/NeuronType.cpp:94-158, src/nemo/plugins/<name>.ini). */
struct NeuronType {
	std::string name;
	unsigned nParam;
	unsigned nState;
	unsigned membranePotential;
	unsigned history;
	bool nrand;
	cpu_update_neurons_t* update;
};

NeuronType neuronType(const std::string& name);

/* Restated model updates (exported so tests can compare them with the
 * reference plugin sources compiled in oracle/_ref). */
cpu_update_neurons_t update_Izhikevich;
cpu_update_neurons_t update_IF_curr_exp;
cpu_update_neurons_t update_QIF;
cpu_update_neurons_t update_HH;
cpu_update_neurons_t update_PoissonSource;
cpu_update_neurons_t update_Input;

/* ---- StdpFunction (src/nemo/StdpFunction.cpp:9-107) ---- */
struct StdpFunction {
	StdpFunction(const std::vector<float>& pre, const std::vector<float>& post,
			float minE, float maxE, float minI, float maxI);
	void verifyDynamicWindowLength(unsigned d_max) const;
	uint64_t potentiationBits() const;
	uint64_t depressionBits() const;
	std::vector<float> prefire, postfire;
	float minE, maxE, minI, maxI;
private:
	uint64_t getBits(bool (*pred)(float)) const;
};

/* ---- StdpProcess (src/nemo/StdpProcess.cpp:20-137) ---- */
class StdpProcess {
public:
	StdpProcess(const StdpFunction& fn, unsigned fbits);
	fix_t weightChange(uint64_t preFiring) const;
	fix_t updatedWeight(fix_t w_old, fix_t w_diff) const;
	uint64_t postFireMask() const { return m_postFireMask; }
private:
	fix_t updateRegion(uint64_t arrivals) const;
	unsigned closestPreFire(uint64_t arrivals) const;
	unsigned closestPostFire(uint64_t arrivals) const;
	static const unsigned NONE = ~0U;
	std::vector<fix_t> m_fnPre, m_fnPost;
	int m_postPreWindow;
	uint64_t m_potentiationBits, m_depressionBits, m_prePostBits, m_postPreBits, m_postFireMask;
	fix_t m_minE, m_maxE, m_minI, m_maxI;
};

/* ---- Configuration (src/nemo/ConfigurationImpl.cpp:19-117) ---- */
struct Configuration {
	Configuration();
	bool logging;
	bool writeOnlySynapses;
	unsigned fractionalBits;
	backend_t backend;
	int cudaDevice;
	std::string description;
	bool hasStdp;
	std::vector<StdpFunction> stdp; /* 0 or 1 element */
};

/* ---- Network (src/nemo/NetworkImpl.cpp, Neurons.cpp, Axon.cpp) ---- */
struct NeuronGroup {
	NeuronType type;
	std::vector<std::vector<float>> param; /* [nParam][n] */
	std::vector<std::vector<float>> state; /* [nState][n] */
	std::vector<unsigned> gidx;
};

struct Axon {
	std::vector<unsigned> targets;
	std::vector<unsigned> delays;
	std::vector<float> weights;
	std::vector<unsigned char> plastic;
};

class Network {
public:
	Network();
	unsigned addNeuronType(const std::string& name);
	void addNeuron(unsigned type, unsigned gidx, unsigned nargs, const float args[]);
	void setNeuron(unsigned gidx, unsigned nargs, const float args[]);
	synapse_id addSynapse(unsigned source, unsigned target, unsigned delay, float weight, unsigned char plastic);
	float getNeuronState(unsigned gidx, unsigned var) const;
	float getNeuronParameter(unsigned gidx, unsigned param) const;
	void setNeuronState(unsigned gidx, unsigned var, float val);
	void setNeuronParameter(unsigned gidx, unsigned param, float val);
	const Axon& axon(unsigned source) const;
	const std::vector<synapse_id>& getSynapsesFrom(unsigned source);
	unsigned neuronCount() const;
	unsigned maxDelay() const { return m_maxDelay; }

	std::vector<NeuronGroup> groups;
	std::map<std::string, unsigned> typeIds;
	std::unordered_map<unsigned, std::pair<unsigned, unsigned>> mapper; /* gidx -> (type, index) */
	std::map<unsigned, Axon> fcm; /* ordered by source, like NetworkImpl::m_fcm */
	int minIdx, maxIdx;
	unsigned m_maxDelay;
	float minWeight, maxWeight;
	unsigned izType;
private:
	std::vector<synapse_id> m_queried;
	std::pair<unsigned, unsigned> address(unsigned gidx) const;
};

/* ---- CPU simulation (src/nemo/cpu/Simulation.cpp, Neurons.cpp,
 *      src/nemo/ConnectivityMatrix.cpp, runtime/RCM.cpp) ---- */
struct FAxonTerminal { unsigned target; fix_t weight; };

class Simulation {
public:
	Simulation(const Network& net, const Configuration& conf);

	void setFiringStimulus(const std::vector<unsigned>& fstim);
	void addCurrentStimulus(unsigned gidx, float current);
	void fire();
	const std::vector<unsigned>& readFiring();
	void applyStdp(float reward);

	float getNeuronState(unsigned gidx, unsigned var) const;
	float getNeuronParameter(unsigned gidx, unsigned param) const;
	float getMembranePotential(unsigned gidx) const;
	void setNeuron(unsigned gidx, unsigned nargs, const float args[]);
	void setNeuronState(unsigned gidx, unsigned var, float val);
	void setNeuronParameter(unsigned gidx, unsigned param, float val);

	const std::vector<synapse_id>& getSynapsesFrom(unsigned source);
	unsigned getSynapseTarget(synapse_id id) const;
	unsigned getSynapseDelay(synapse_id id) const;
	float getSynapseWeight(synapse_id id) const;
	void getWeights(const synapse_id* ids, size_t n, float* out) const;
	unsigned char getSynapsePlastic(synapse_id id) const;

	unsigned long elapsedWallclock() const;
	unsigned long elapsedSimulation() const { return m_cycles; }
	void resetTimer();

private:
	struct Group {
		NeuronType type;
		unsigned base;
		unsigned size;
		std::vector<float> param; /* nParam * size */
		std::vector<float> state; /* nState * size (history 1) */
		std::vector<RNG> rng;
	};

	unsigned localIdx(unsigned gidx) const;
	unsigned globalIdx(unsigned lidx) const;
	const Group& groupOf(unsigned lidx, unsigned* nl) const;
	Group& groupOf(unsigned lidx, unsigned* nl);
	void deliverSpikes();
	void accumulateStdp();
	void setFiring();
	struct Aux { unsigned idx; unsigned delay; bool plastic; };
	const Aux& aux(synapse_id id) const;
	size_t addressOf(unsigned source, unsigned delay) const { return size_t(source) * m_maxDelay + delay - 1; }

	unsigned m_neuronCount;
	std::vector<Group> m_groups;
	std::vector<unsigned> m_typeBase;
	std::unordered_map<unsigned, unsigned> m_g2l;
	std::vector<unsigned> m_l2g;
	std::vector<unsigned> m_typeOfLocal;

	std::vector<unsigned> m_fired;
	std::vector<uint64_t> m_recentFiring;
	std::vector<uint64_t> m_delays;
	std::vector<wfix_t> mfx_currentE, mfx_currentI;
	std::vector<float> m_currentE, m_currentI, m_currentExt;
	std::vector<unsigned> m_fstim;

	/* forward matrix: rows (source, delay) in CSR form */
	unsigned m_fbits;
	unsigned m_maxDelay;
	std::vector<size_t> m_rowStart; /* size nrows+1 */
	std::vector<FAxonTerminal> m_terminals;

	/* reverse matrix: per target, its (plastic) incoming synapses */
	std::vector<size_t> m_rcmStart; /* size N+1 */
	std::vector<unsigned> m_rcmSource, m_rcmDelay, m_rcmForward;
	std::vector<fix_t> m_rcmAcc;
	bool m_stdpOn;
	std::vector<StdpProcess> m_stdp;

	/* synapse queries keyed by global source (ConnectivityMatrix m_cmAux) */
	bool m_writeOnly;
	std::unordered_map<unsigned, std::pair<size_t, size_t>> m_auxRange;
	std::vector<Aux> m_aux;
	std::vector<synapse_id> m_queried;

	std::vector<unsigned> m_firedList;
	unsigned long m_cycles;
	double m_wallStart;
};

} // namespace oracle

#endif
