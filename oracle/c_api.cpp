/* ORACLE — TEST INFRASTRUCTURE ONLY (see oracle.hpp).
 *
 * The include/nemo.h C ABI over the oracle classes, restating
 * src/nemo/nemo_c.cpp (error capture in process-global state, CALL/CATCH
 * semantics, step() helper order). */

#include <nemo.h>
/* the bulk construction calls (nemo_add_neurons / nemo_add_synapses) and the
 * bulk weight read are declared with the B200 library's extensions; the
 * oracle defines them too, so that a network file builds through the same
 * calls on both libraries and the tests read weights the same way */
#include <nemo_b200.h>

#include <cstring>
#include <string>
#include <vector>

#include "oracle.hpp"

using namespace oracle;

struct nemo_network_class { Network net; };
struct nemo_configuration_class { Configuration conf; };
struct nemo_simulation_class {
	explicit nemo_simulation_class(const Network& n, const Configuration& c) : sim(n, c) {}
	Simulation sim;
	std::vector<unsigned> fired;
};

static std::string g_lastError;
static nemo_status_t g_lastCallStatus = NEMO_OK;

static void
setResult(const char* msg, nemo_status_t status)
{
	g_lastError = msg;
	g_lastCallStatus = status;
}

/* nemo_c.cpp:42-53 */
#define CALL(...) {                                                          \
        g_lastCallStatus = NEMO_OK;                                           \
        try {                                                                 \
            __VA_ARGS__;                                                      \
        } catch (oracle::Error& e) {                                          \
            setResult(e.what(), e.code);                                      \
        } catch (std::exception& e) {                                         \
            setResult(e.what(), NEMO_UNKNOWN_ERROR);                          \
        } catch (...) {                                                       \
            setResult("unknown exception", NEMO_UNKNOWN_ERROR);               \
        }                                                                     \
    }

#define RETURN_CALL(...) { CALL(__VA_ARGS__); return g_lastCallStatus; }

/* nemo_c.cpp:328-343 */
template<class T>
static void
synapsesFrom(T& obj, unsigned source, synapse_id* synapses[], size_t* len)
{
	const std::vector<synapse_id>& ids = obj.getSynapsesFrom(source);
	if(!ids.empty()) {
		*synapses = const_cast<synapse_id*>(ids.data());
		*len = ids.size();
	} else {
		*synapses = NULL;
		*len = 0;
	}
}

extern "C" {

const char* nemo_version(void) { return "0.7.2-oracle"; }

nemo_status_t nemo_add_plugin_path(const char*) { RETURN_CALL((void) 0); }

nemo_status_t
nemo_cuda_device_count(unsigned* count)
{
	*count = 0;
	RETURN_CALL((void) 0);
}

nemo_status_t
nemo_cuda_device_description(unsigned, const char**)
{
	RETURN_CALL(throw Error(NEMO_API_UNSUPPORTED, "the oracle has no CUDA backend"));
}

nemo_configuration_t nemo_new_configuration(void) { return new nemo_configuration_class(); }
void nemo_delete_configuration(nemo_configuration_t c) { delete c; }
nemo_status_t nemo_log_stdout(nemo_configuration_t c) { RETURN_CALL(c->conf.logging = true); }

nemo_status_t
nemo_set_stdp_function(nemo_configuration_t c,
		float* pre, size_t pre_len, float* post, size_t post_len,
		float we_min, float we_max, float wi_min, float wi_max)
{
	RETURN_CALL({
		StdpFunction fn(std::vector<float>(pre, pre + pre_len),
				std::vector<float>(post, post + post_len), we_min, we_max, wi_min, wi_max);
		c->conf.stdp.clear();
		c->conf.stdp.push_back(fn);
		c->conf.hasStdp = true;
	});
}

nemo_status_t nemo_set_cpu_backend(nemo_configuration_t c) { RETURN_CALL(c->conf.backend = NEMO_BACKEND_CPU); }

nemo_status_t
nemo_set_cuda_backend(nemo_configuration_t, int)
{
	RETURN_CALL(throw Error(NEMO_API_UNSUPPORTED, "the oracle has no CUDA backend"));
}

nemo_status_t nemo_cuda_device(nemo_configuration_t c, int* dev) { RETURN_CALL(*dev = c->conf.cudaDevice); }
nemo_status_t nemo_backend(nemo_configuration_t c, backend_t* b) { RETURN_CALL(*b = c->conf.backend); }
nemo_status_t nemo_backend_description(nemo_configuration_t c, const char** d) { RETURN_CALL(*d = c->conf.description.c_str()); }
nemo_status_t nemo_set_write_only_synapses(nemo_configuration_t c) { RETURN_CALL(c->conf.writeOnlySynapses = true); }

nemo_network_t nemo_new_network(void) { return new nemo_network_class(); }
void nemo_delete_network(nemo_network_t n) { delete n; }

nemo_status_t
nemo_add_neuron_type(nemo_network_t n, const char* name, unsigned* type)
{
	RETURN_CALL(*type = n->net.addNeuronType(name));
}

/* Network.cpp:46-56: parameters {a,b,c,d,sigma} then state {u,v} */
nemo_status_t
nemo_add_neuron_iz(nemo_network_t n, unsigned idx, float a, float b, float c, float d, float u, float v, float sigma)
{
	RETURN_CALL({
		if(n->net.izType == ~0U) n->net.izType = n->net.addNeuronType("Izhikevich");
		float args[7] = {a, b, c, d, sigma, u, v};
		n->net.addNeuron(n->net.izType, idx, 7, args);
	});
}

nemo_status_t
nemo_add_neuron(nemo_network_t n, unsigned type, unsigned idx, unsigned nargs, float args[])
{
	RETURN_CALL(n->net.addNeuron(type, idx, nargs, args));
}

nemo_status_t
nemo_add_neurons(nemo_network_t n, unsigned type, size_t count, const unsigned idx[], unsigned nargs, const float args[])
{
	RETURN_CALL({
		for(size_t i = 0; i < count; ++i) n->net.addNeuron(type, idx[i], nargs, args + i * nargs);
	});
}

nemo_status_t
nemo_add_synapse(nemo_network_t n, unsigned source, unsigned target, unsigned delay, float weight,
		unsigned char plastic, synapse_id* id)
{
	synapse_id sid = 0;
	CALL(sid = n->net.addSynapse(source, target, delay, weight, plastic));
	if(id != NULL) *id = sid;
	return g_lastCallStatus;
}

nemo_status_t
nemo_add_synapses(nemo_network_t n, size_t count, const unsigned source[], const unsigned target[],
		const unsigned delay[], const float weight[], const unsigned char plastic[], synapse_id ids[])
{
	RETURN_CALL({
		for(size_t i = 0; i < count; ++i) {
			synapse_id sid = n->net.addSynapse(source[i], target[i], delay[i], weight[i], plastic ? plastic[i] : 0);
			if(ids) ids[i] = sid;
		}
	});
}

nemo_status_t nemo_neuron_count(nemo_network_t n, unsigned* c) { RETURN_CALL(*c = n->net.neuronCount()); }

nemo_simulation_t
nemo_new_simulation(nemo_network_t n, nemo_configuration_t c)
{
	try {
		return new nemo_simulation_class(n->net, c->conf);
	} catch(oracle::Error& e) {
		setResult(e.what(), e.code);
	} catch(std::exception& e) {
		setResult(e.what(), NEMO_UNKNOWN_ERROR);
	} catch(...) {
		setResult("Unknown error", NEMO_UNKNOWN_ERROR);
	}
	return NULL;
}

void nemo_delete_simulation(nemo_simulation_t s) { delete s; }

/* nemo_c.cpp:439-476: firing stimulus, then current stimulus, then the cycle */
nemo_status_t
nemo_step(nemo_simulation_t s, unsigned fstim_nidx[], size_t fstim_count,
		unsigned istim_nidx[], float istim_current[], size_t istim_count,
		unsigned* fired[], size_t* fired_count)
{
	RETURN_CALL({
		s->sim.setFiringStimulus(std::vector<unsigned>(fstim_nidx, fstim_nidx + fstim_count));
		for(size_t i = 0; i < istim_count; ++i) {
			s->sim.addCurrentStimulus(istim_nidx[i], istim_current[i]);
		}
		s->sim.fire();
		s->fired = s->sim.readFiring();
		if(fired != NULL) *fired = s->fired.empty() ? NULL : s->fired.data();
		if(fired_count != NULL) *fired_count = s->fired.size();
	});
}

nemo_status_t nemo_apply_stdp(nemo_simulation_t s, float reward) { RETURN_CALL(s->sim.applyStdp(reward)); }

nemo_status_t nemo_get_membrane_potential(nemo_simulation_t s, unsigned n, float* v) { RETURN_CALL(*v = s->sim.getMembranePotential(n)); }
nemo_status_t nemo_get_neuron_state_n(nemo_network_t n, unsigned i, unsigned var, float* v) { RETURN_CALL(*v = n->net.getNeuronState(i, var)); }
nemo_status_t nemo_get_neuron_parameter_n(nemo_network_t n, unsigned i, unsigned p, float* v) { RETURN_CALL(*v = n->net.getNeuronParameter(i, p)); }
nemo_status_t nemo_get_neuron_state_s(nemo_simulation_t s, unsigned i, unsigned var, float* v) { RETURN_CALL(*v = s->sim.getNeuronState(i, var)); }
nemo_status_t nemo_get_neuron_parameter_s(nemo_simulation_t s, unsigned i, unsigned p, float* v) { RETURN_CALL(*v = s->sim.getNeuronParameter(i, p)); }

nemo_status_t nemo_get_synapse_source_n(nemo_network_t, synapse_id id, unsigned* src) { RETURN_CALL(*src = unsigned(id >> 32)); }
nemo_status_t nemo_get_synapse_source_s(nemo_simulation_t, synapse_id id, unsigned* src) { RETURN_CALL(*src = unsigned(id >> 32)); }
nemo_status_t nemo_get_synapse_target_n(nemo_network_t n, synapse_id id, unsigned* t) { RETURN_CALL(*t = n->net.axon(unsigned(id >> 32)).targets.at(id & 0xffffffff)); }
nemo_status_t nemo_get_synapse_target_s(nemo_simulation_t s, synapse_id id, unsigned* t) { RETURN_CALL(*t = s->sim.getSynapseTarget(id)); }
nemo_status_t nemo_get_synapse_delay_n(nemo_network_t n, synapse_id id, unsigned* d) { RETURN_CALL(*d = n->net.axon(unsigned(id >> 32)).delays.at(id & 0xffffffff)); }
nemo_status_t nemo_get_synapse_delay_s(nemo_simulation_t s, synapse_id id, unsigned* d) { RETURN_CALL(*d = s->sim.getSynapseDelay(id)); }
nemo_status_t nemo_get_synapse_weight_n(nemo_network_t n, synapse_id id, float* w) { RETURN_CALL(*w = n->net.axon(unsigned(id >> 32)).weights.at(id & 0xffffffff)); }
nemo_status_t nemo_get_synapse_weight_s(nemo_simulation_t s, synapse_id id, float* w) { RETURN_CALL(*w = s->sim.getSynapseWeight(id)); }
nemo_status_t
nemo_b200_get_weights(nemo_simulation_t s, const synapse_id ids[], size_t count, float weights[])
{
	RETURN_CALL(s->sim.getWeights(ids, count, weights));
}
nemo_status_t nemo_get_synapse_plastic_n(nemo_network_t n, synapse_id id, unsigned char* p) { RETURN_CALL(*p = n->net.axon(unsigned(id >> 32)).plastic.at(id & 0xffffffff)); }
nemo_status_t nemo_get_synapse_plastic_s(nemo_simulation_t s, synapse_id id, unsigned char* p) { RETURN_CALL(*p = s->sim.getSynapsePlastic(id)); }

nemo_status_t nemo_get_synapses_from_n(nemo_network_t n, unsigned src, synapse_id* ids[], size_t* len) { RETURN_CALL(synapsesFrom(n->net, src, ids, len)); }
nemo_status_t nemo_get_synapses_from_s(nemo_simulation_t s, unsigned src, synapse_id* ids[], size_t* len) { RETURN_CALL(synapsesFrom(s->sim, src, ids, len)); }

nemo_status_t nemo_set_neuron_n(nemo_network_t n, unsigned idx, unsigned nargs, float args[]) { RETURN_CALL(n->net.setNeuron(idx, nargs, args)); }
nemo_status_t nemo_set_neuron_s(nemo_simulation_t s, unsigned idx, unsigned nargs, float args[]) { RETURN_CALL(s->sim.setNeuron(idx, nargs, args)); }

nemo_status_t
nemo_set_neuron_iz_n(nemo_network_t n, unsigned idx, float a, float b, float c, float d, float u, float v, float sigma)
{
	float args[7] = {a, b, c, d, sigma, u, v};
	RETURN_CALL(n->net.setNeuron(idx, 7, args));
}

nemo_status_t
nemo_set_neuron_iz_s(nemo_simulation_t s, unsigned idx, float a, float b, float c, float d, float u, float v, float sigma)
{
	float args[7] = {a, b, c, d, sigma, u, v};
	RETURN_CALL(s->sim.setNeuron(idx, 7, args));
}

nemo_status_t nemo_set_neuron_state_n(nemo_network_t n, unsigned i, unsigned var, float v) { RETURN_CALL(n->net.setNeuronState(i, var, v)); }
nemo_status_t nemo_set_neuron_parameter_n(nemo_network_t n, unsigned i, unsigned p, float v) { RETURN_CALL(n->net.setNeuronParameter(i, p, v)); }
nemo_status_t nemo_set_neuron_state_s(nemo_simulation_t s, unsigned i, unsigned var, float v) { RETURN_CALL(s->sim.setNeuronState(i, var, v)); }
nemo_status_t nemo_set_neuron_parameter_s(nemo_simulation_t s, unsigned i, unsigned p, float v) { RETURN_CALL(s->sim.setNeuronParameter(i, p, v)); }

nemo_status_t nemo_elapsed_wallclock(nemo_simulation_t s, unsigned long* e) { RETURN_CALL(*e = s->sim.elapsedWallclock()); }
nemo_status_t nemo_elapsed_simulation(nemo_simulation_t s, unsigned long* e) { RETURN_CALL(*e = s->sim.elapsedSimulation()); }
nemo_status_t nemo_reset_timer(nemo_simulation_t s) { RETURN_CALL(s->sim.resetTimer()); }

const char* nemo_strerror(void) { return g_lastError.c_str(); }

/* Test hook: the restated model update for a named type, with the reference
 * plugin signature, so tests can run it beside the reference plugin code. */
void*
oracle_model_update(const char* name)
{
	try {
		return (void*) neuronType(name).update;
	} catch(...) {
		return NULL;
	}
}

} // extern "C"
