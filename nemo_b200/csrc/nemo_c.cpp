/* The NeMo C ABI (include/nemo.h, include/nemo_b200.h) over the B200 backend.
 *
 * Error handling follows src/nemo/nemo_c.cpp:24-65: every call clears the
 * process-global status, catches exceptions and records message and code;
 * constructors return NULL on failure. */

#include <nemo.h>
#include <nemo_b200.h>

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "libm_tables.hpp"
#include "network.hpp"
#include "simulation.hpp"

using namespace nemo_b200;

struct nemo_network_class { Network net; };
struct nemo_configuration_class { Configuration conf; };
struct nemo_simulation_class {
	nemo_simulation_class(const Network& n, const Configuration& c, const ShardSpec* shard = nullptr) :
		sim(n, c, shard) {}
	Simulation sim;
	std::vector<unsigned> fired;
};

static std::string g_lastError;
static nemo_status_t g_lastCallStatus = NEMO_OK;
static std::string g_deviceDescription;
static std::string g_cachePath;

static void
setResult(const char* msg, nemo_status_t status)
{
	g_lastError = msg;
	g_lastCallStatus = status;
}

#define CALL(...) {                                                           \
        g_lastCallStatus = NEMO_OK;                                           \
        try {                                                                 \
            __VA_ARGS__;                                                      \
        } catch(Exception& e) {                                               \
            setResult(e.what(), e.code());                                    \
        } catch(std::exception& e) {                                          \
            setResult(e.what(), NEMO_UNKNOWN_ERROR);                          \
        } catch(...) {                                                        \
            setResult("unknown exception", NEMO_UNKNOWN_ERROR);               \
        }                                                                     \
    }

#define RETURN_CALL(...) { CALL(__VA_ARGS__); return g_lastCallStatus; }

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

const char* nemo_version(void) { return "0.7.2-b200"; }

nemo_status_t nemo_add_plugin_path(const char* dir) { RETURN_CALL(addPluginPath(dir)); }

nemo_status_t
nemo_cuda_device_count(unsigned* count)
{
	*count = 0;
	RETURN_CALL({
		int n = 0;
		NEMO_CUDA(cudaGetDeviceCount(&n));
		*count = unsigned(n);
	});
}

nemo_status_t
nemo_cuda_device_description(unsigned device, const char** descr)
{
	RETURN_CALL({
		cudaDeviceProp p;
		NEMO_CUDA(cudaGetDeviceProperties(&p, int(device)));
		g_deviceDescription = std::string(p.name) + " (sm_" + std::to_string(p.major) + std::to_string(p.minor) + ")";
		*descr = g_deviceDescription.c_str();
	});
}

nemo_configuration_t
nemo_new_configuration(void)
{
	try {
		return new nemo_configuration_class();
	} catch(std::exception& e) {
		setResult(e.what(), NEMO_UNKNOWN_ERROR);
		return NULL;
	}
}

void nemo_delete_configuration(nemo_configuration_t c) { delete c; }
nemo_status_t nemo_log_stdout(nemo_configuration_t c) { RETURN_CALL(c->conf.logging = true); }

nemo_status_t
nemo_set_stdp_function(nemo_configuration_t c, float* pre, size_t pre_len, float* post, size_t post_len,
		float we_min, float we_max, float wi_min, float wi_max)
{
	RETURN_CALL({
		c->conf.stdp = StdpFunction(std::vector<float>(pre, pre + pre_len),
				std::vector<float>(post, post + post_len), we_min, we_max, wi_min, wi_max);
		c->conf.hasStdp = true;
	});
}

nemo_status_t
nemo_set_cpu_backend(nemo_configuration_t)
{
	RETURN_CALL(fail(NEMO_API_UNSUPPORTED, "libnemo_b200 provides the B200 (CUDA) backend only"));
}

nemo_status_t
nemo_set_cuda_backend(nemo_configuration_t c, int dev)
{
	RETURN_CALL({
		if(dev >= 0) {
			int n = 0;
			NEMO_CUDA(cudaGetDeviceCount(&n));
			if(dev >= n) {
				fail(NEMO_INVALID_INPUT, "Invalid CUDA device " + std::to_string(dev));
			}
		}
		c->conf.cudaDevice = dev;
	});
}

nemo_status_t nemo_cuda_device(nemo_configuration_t c, int* dev) { RETURN_CALL(*dev = c->conf.cudaDevice); }
nemo_status_t nemo_backend(nemo_configuration_t, backend_t* b) { RETURN_CALL(*b = NEMO_BACKEND_CUDA); }
nemo_status_t nemo_backend_description(nemo_configuration_t c, const char** d) { RETURN_CALL(*d = c->conf.description.c_str()); }
nemo_status_t nemo_set_write_only_synapses(nemo_configuration_t c) { RETURN_CALL(c->conf.writeOnlySynapses = true); }

nemo_network_t nemo_new_network(void) { return new nemo_network_class(); }
void nemo_delete_network(nemo_network_t n) { delete n; }

nemo_status_t
nemo_add_neuron_type(nemo_network_t n, const char* name, unsigned* type)
{
	RETURN_CALL(*type = n->net.addNeuronType(name));
}

/* src/nemo/Network.cpp:46-56: parameters {a,b,c,d,sigma}, state {u,v} */
nemo_status_t
nemo_add_neuron_iz(nemo_network_t n, unsigned idx, float a, float b, float c, float d, float u, float v, float sigma)
{
	RETURN_CALL({
		if(n->net.izType == ~0u) n->net.izType = n->net.addNeuronType("Izhikevich");
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
		Network& net = n->net;
		size_t want = net.src.size() + count;
		net.src.reserve(want); net.tgt.reserve(want); net.dly.reserve(want);
		net.wgt.reserve(want); net.plastic.reserve(want); net.sid.reserve(want);
		for(size_t i = 0; i < count; ++i) {
			synapse_id sid = net.addSynapse(source[i], target[i], delay[i], weight[i], plastic ? plastic[i] : 0);
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
	} catch(Exception& e) {
		setResult(e.what(), e.code());
	} catch(std::exception& e) {
		setResult(e.what(), NEMO_UNKNOWN_ERROR);
	} catch(...) {
		setResult("Unknown error", NEMO_UNKNOWN_ERROR);
	}
	return NULL;
}

void nemo_delete_simulation(nemo_simulation_t s) { delete s; }

nemo_simulation_t
nemo_b200_new_batch(nemo_network_t nets[], size_t count, nemo_configuration_t c)
{
	try {
		if(count == 0) {
			fail(NEMO_INVALID_INPUT, "Batch: no networks");
		}
		std::vector<const Network*> list(count);
		for(size_t j = 0; j < count; ++j) list[j] = &nets[j]->net;
		std::vector<uint32_t> base;
		Network merged = Network::merge(list, &base);
		nemo_simulation_class* s = new nemo_simulation_class(merged, c->conf);
		s->sim.setBatch(std::move(base));
		return s;
	} catch(Exception& e) {
		setResult(e.what(), e.code());
	} catch(std::exception& e) {
		setResult(e.what(), NEMO_UNKNOWN_ERROR);
	} catch(...) {
		setResult("Unknown error", NEMO_UNKNOWN_ERROR);
	}
	return NULL;
}

nemo_status_t nemo_b200_last_status(void) { return g_lastCallStatus; }

nemo_status_t
nemo_b200_network_stats(nemo_network_t n, unsigned* max_delay, float* min_weight, float* max_weight)
{
	RETURN_CALL({
		float lo = 0.0f, hi = 0.0f;
		for(float w : n->net.wgt) {
			lo = std::min(lo, w);
			hi = std::max(hi, w);
		}
		if(max_delay) *max_delay = n->net.maxDelay();
		if(min_weight) *min_weight = lo;
		if(max_weight) *max_weight = hi;
	});
}

nemo_simulation_t
nemo_b200_new_shard(nemo_network_t n, nemo_configuration_t c, unsigned rank, unsigned world)
{
	try {
		ShardSpec spec;
		Network local = shardNetwork(n->net, rank, world, &spec);
		return new nemo_simulation_class(local, c->conf, &spec);
	} catch(Exception& e) {
		setResult(e.what(), e.code());
	} catch(std::exception& e) {
		setResult(e.what(), NEMO_UNKNOWN_ERROR);
	} catch(...) {
		setResult("Unknown error", NEMO_UNKNOWN_ERROR);
	}
	return NULL;
}

nemo_status_t
nemo_b200_shard_warps(unsigned total_words, unsigned rank, unsigned world, unsigned* first_word, unsigned* words)
{
	RETURN_CALL({
		uint32_t lo = 0, hi = 0;
		shardWarps(total_words, rank, world, &lo, &hi);
		*first_word = lo;
		*words = hi - lo;
	});
}

nemo_status_t
nemo_b200_shard_range(nemo_simulation_t s, unsigned* first_word, unsigned* words, unsigned* total_words)
{
	RETURN_CALL({
		const ShardSpec& sp = s->sim.shard();
		*first_word = sp.warpLo;
		*words = sp.warpHi - sp.warpLo;
		*total_words = sp.totalWarps;
	});
}

nemo_status_t
nemo_b200_shard_step(nemo_simulation_t s, unsigned fstim_nidx[], size_t fstim_count,
		unsigned istim_nidx[], float istim_current[], size_t istim_count, uint32_t local_words[])
{
	RETURN_CALL(s->sim.shardStep(fstim_nidx, fstim_count, istim_nidx, istim_current, istim_count, local_words));
}

nemo_status_t
nemo_b200_shard_deliver(nemo_simulation_t s, const uint32_t all_words[], unsigned* fired[], size_t* fired_count)
{
	RETURN_CALL({
		const std::vector<unsigned>& f = s->sim.shardDeliver(all_words);
		s->fired = f;
		*fired = s->fired.empty() ? NULL : s->fired.data();
		*fired_count = s->fired.size();
	});
}

nemo_status_t
nemo_b200_shard_step_async(nemo_simulation_t s, const unsigned fstim_nidx[], size_t fstim_count,
		const unsigned istim_nidx[], const float istim_current[], size_t istim_count, uint32_t* local_words_dev,
		void* stream)
{
	RETURN_CALL(s->sim.shardStepAsync(fstim_nidx, fstim_count, istim_nidx, istim_current, istim_count,
				local_words_dev, stream));
}

nemo_status_t
nemo_b200_shard_deliver_async(nemo_simulation_t s, const uint32_t* all_words_dev, void* stream)
{
	RETURN_CALL(s->sim.shardDeliverAsync(all_words_dev, stream));
}

nemo_status_t
nemo_b200_stream_wait(nemo_simulation_t s, void* stream)
{
	RETURN_CALL(s->sim.streamWait(stream));
}

nemo_status_t
nemo_step(nemo_simulation_t s, unsigned fstim_nidx[], size_t fstim_count,
		unsigned istim_nidx[], float istim_current[], size_t istim_count,
		unsigned* fired[], size_t* fired_count)
{
	RETURN_CALL({
		const std::vector<unsigned>& f = s->sim.step(fstim_nidx, fstim_count, istim_nidx, istim_current, istim_count);
		if(fired != NULL) *fired = f.empty() ? NULL : const_cast<unsigned*>(f.data());
		if(fired_count != NULL) *fired_count = f.size();
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
nemo_status_t nemo_get_synapse_target_n(nemo_network_t n, synapse_id id, unsigned* t) { RETURN_CALL(*t = n->net.tgt[n->net.synapsePosition(id)]); }
nemo_status_t nemo_get_synapse_target_s(nemo_simulation_t s, synapse_id id, unsigned* t) { RETURN_CALL(*t = s->sim.getSynapseTarget(id)); }
nemo_status_t nemo_get_synapse_delay_n(nemo_network_t n, synapse_id id, unsigned* d) { RETURN_CALL(*d = n->net.dly[n->net.synapsePosition(id)]); }
nemo_status_t nemo_get_synapse_delay_s(nemo_simulation_t s, synapse_id id, unsigned* d) { RETURN_CALL(*d = s->sim.getSynapseDelay(id)); }
nemo_status_t nemo_get_synapse_weight_n(nemo_network_t n, synapse_id id, float* w) { RETURN_CALL(*w = n->net.wgt[n->net.synapsePosition(id)]); }
nemo_status_t nemo_get_synapse_weight_s(nemo_simulation_t s, synapse_id id, float* w) { RETURN_CALL(*w = s->sim.getSynapseWeight(id)); }
nemo_status_t
nemo_b200_get_weights(nemo_simulation_t s, const synapse_id ids[], size_t count, float weights[])
{
	RETURN_CALL(s->sim.getWeights(ids, count, weights));
}
nemo_status_t nemo_get_synapse_plastic_n(nemo_network_t n, synapse_id id, unsigned char* p) { RETURN_CALL(*p = n->net.plastic[n->net.synapsePosition(id)]); }
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

/* ---- include/nemo_b200.h ---- */

nemo_status_t
nemo_b200_run(nemo_simulation_t s, unsigned cycles, uint32_t fired_counts[], uint64_t events[])
{
	RETURN_CALL(s->sim.run(cycles, fired_counts, events));
}

nemo_status_t
nemo_b200_fired_at(nemo_simulation_t s, uint64_t cycle, unsigned* fired[], size_t* fired_count)
{
	RETURN_CALL({
		const std::vector<unsigned>& f = s->sim.firedAt(cycle);
		if(fired != NULL) *fired = f.empty() ? NULL : const_cast<unsigned*>(f.data());
		if(fired_count != NULL) *fired_count = f.size();
	});
}

nemo_status_t nemo_b200_cycle(nemo_simulation_t s, uint64_t* cycle) { RETURN_CALL(*cycle = s->sim.cycle()); }
nemo_status_t nemo_b200_synchronize(nemo_simulation_t s) { RETURN_CALL(s->sim.synchronize()); }

nemo_status_t
nemo_b200_step_noalloc(nemo_simulation_t s, const unsigned fstim_nidx[], size_t fstim_count,
		const unsigned istim_nidx[], const float istim_current[], size_t istim_count,
		unsigned fired[], size_t fired_capacity, size_t* fired_count)
{
	RETURN_CALL({
		size_t n = s->sim.stepNoAlloc(fstim_nidx, fstim_count, istim_nidx, istim_current, istim_count,
				fired, fired_capacity);
		if(fired_count != NULL) *fired_count = n;
	});
}

nemo_status_t
nemo_b200_nrand_probe(nemo_simulation_t s, const uint32_t u1[], const uint32_t u2[], float out[], size_t n)
{
	RETURN_CALL(s->sim.nrandProbe(u1, u2, out, n));
}

nemo_status_t
nemo_b200_timed_steps(nemo_simulation_t s, unsigned steps, unsigned cycles_per_step, int apply_stdp,
		float reward, double out[4])
{
	RETURN_CALL(s->sim.timedSteps(steps, cycles_per_step, apply_stdp != 0, reward, out));
}

nemo_status_t
nemo_b200_profile(nemo_simulation_t s, unsigned cycles, float reward, double out[10])
{
	RETURN_CALL(s->sim.profile(cycles, reward, out));
}

nemo_status_t
nemo_b200_trace(nemo_simulation_t s, unsigned cycles, double out[24])
{
	RETURN_CALL(s->sim.trace(cycles, out));
}

nemo_status_t
nemo_b200_apply_launches(nemo_simulation_t s, unsigned* launches)
{
	RETURN_CALL(*launches = s->sim.applyLaunches());
}

nemo_status_t
nemo_b200_counters(nemo_simulation_t s, uint64_t out[4])
{
	RETURN_CALL(s->sim.readStats(out));
}

nemo_status_t
nemo_b200_batch_instances(nemo_simulation_t s, size_t* count)
{
	RETURN_CALL(*count = s->sim.instances());
}

nemo_status_t
nemo_b200_batch_fired_at(nemo_simulation_t s, uint64_t cycle, const unsigned* fired[], const size_t* offsets[])
{
	RETURN_CALL({
		const std::vector<unsigned>* f;
		const std::vector<size_t>* o;
		s->sim.batchFiredAt(cycle, &f, &o);
		*fired = f->empty() ? NULL : f->data();
		*offsets = o->data();
	});
}

nemo_status_t
nemo_b200_run_graph(nemo_simulation_t s, unsigned cycles, unsigned cycles_per_launch, int* used_graph)
{
	RETURN_CALL(s->sim.runGraph(cycles, cycles_per_launch, used_graph));
}

nemo_status_t
nemo_b200_autotune(nemo_simulation_t s, unsigned trial_cycles, unsigned* threads, double ms[3])
{
	RETURN_CALL({
		double t[3];
		unsigned best = s->sim.autotune(trial_cycles, t);
		if(threads) *threads = best;
		if(ms) for(int k = 0; k < 3; ++k) ms[k] = t[k];
	});
}

nemo_status_t
nemo_b200_host_bytes(nemo_simulation_t s, unsigned long long out[2])
{
	RETURN_CALL(s->sim.hostBytes(out));
}

nemo_status_t
nemo_b200_autotune_shape(nemo_simulation_t s, unsigned trial_cycles, unsigned* threads, unsigned* stdp_run,
		double ms[6])
{
	RETURN_CALL({
		double t[6];
		const nemo_b200::AutotuneShape best = s->sim.autotuneShape(trial_cycles, t);
		if(threads) *threads = best.threads;
		if(stdp_run) *stdp_run = best.stdpRun;
		if(ms) for(int k = 0; k < 6; ++k) ms[k] = t[k];
	});
}

nemo_status_t
nemo_b200_expf_check(nemo_simulation_t s, uint64_t* mismatches)
{
	RETURN_CALL(*mismatches = s->sim.expfCheck());
}

nemo_status_t
nemo_b200_hh_division_check(uint64_t mismatches[3])
{
	RETURN_CALL(nemo_b200::hhDivisionCheck(mismatches));
}

nemo_status_t
nemo_b200_expf_exceptions(size_t* count, double* tau)
{
	RETURN_CALL({
		const nemo_b200::ExpExceptions& e = nemo_b200::expExceptions();
		if(count) *count = e.keys.size();
		if(tau) *tau = e.tau;
	});
}

nemo_status_t
nemo_b200_libm_check(nemo_simulation_t s, uint64_t* mismatches)
{
	RETURN_CALL(*mismatches = s->sim.libmCheck());
}

const char*
nemo_b200_libm_cache_path(void)
{
	g_cachePath = libmCachePath();
	return g_cachePath.c_str();
}

nemo_status_t nemo_b200_prepare_libm_tables(void) { RETURN_CALL((void) libmTables()); }

} // extern "C"
