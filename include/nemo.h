#ifndef NEMO_H
#define NEMO_H

/* NeMo C ABI, implemented by libnemo_b200.so (B200 backend).
 *
 * Every entry point keeps the signature, argument meaning, ownership rules
 * and error behaviour of the reference C ABI in src/nemo.h, so that a program
 * (or a ctypes/FFI binding) written against the reference links against this
 * library unchanged. Each declaration cites the reference declaration it
 * replaces and the wrapper that implements it in src/nemo/nemo_c.cpp.
 *
 * Error model (src/nemo/nemo_c.cpp:24-65): functions returning nemo_status_t
 * return NEMO_OK or an error code; the message of the last failing call is
 * kept in process-global state and read with nemo_strerror(). Constructors
 * return NULL on failure. The library is not thread-safe, like the reference.
 *
 * Ownership (src/nemo.h:337-343, nemo_c.cpp:454-460): arrays returned through
 * output pointers (fired lists, synapse id lists, descriptions) point into
 * library-owned memory that stays valid until the next call on the same
 * object. */

#include <stddef.h>
#include <nemo/types.h>

#ifdef __cplusplus
extern "C" {
#endif

struct nemo_network_class;
struct nemo_simulation_class;
struct nemo_configuration_class;

/* src/nemo.h:43-53 */
typedef struct nemo_network_class* nemo_network_t;
typedef struct nemo_simulation_class* nemo_simulation_t;
typedef struct nemo_configuration_class* nemo_configuration_t;
typedef int nemo_status_t;

/* src/nemo.h:56-57, nemo_c.cpp:68-72 */
const char* nemo_version(void);

/* src/nemo.h:72-74, nemo_c.cpp:76-81. Adds a directory searched (first) for
 * neuron-model descriptors (<name>.ini) and external model plugins. */
nemo_status_t nemo_add_plugin_path(const char* dir);

/* src/nemo.h:88-95, nemo_c.cpp:84-98 */
nemo_status_t nemo_cuda_device_count(unsigned* count);
nemo_status_t nemo_cuda_device_description(unsigned device, const char** descr);

/* ---- Configuration: src/nemo.h:105-191, nemo_c.cpp:116-136,493-587 ---- */

nemo_configuration_t nemo_new_configuration(void);
void nemo_delete_configuration(nemo_configuration_t);
nemo_status_t nemo_log_stdout(nemo_configuration_t);

/* src/nemo.h:148-156. Window lengths: prefire_len + postfire_len <= 64;
 * excitatory limits >= 0, inhibitory limits <= 0 (src/nemo/StdpFunction.cpp:20-55). */
nemo_status_t nemo_set_stdp_function(nemo_configuration_t,
		float prefire_fn[], size_t prefire_len,
		float postfire_fn[], size_t postfire_len,
		float min_excitatory_weight,
		float max_excitatory_weight,
		float min_inhibitory_weight,
		float max_inhibitory_weight);

/* src/nemo.h:159-168. This library provides only the B200 backend;
 * nemo_set_cpu_backend returns NEMO_API_UNSUPPORTED. */
nemo_status_t nemo_set_cpu_backend(nemo_configuration_t);
nemo_status_t nemo_set_cuda_backend(nemo_configuration_t conf, int dev);
nemo_status_t nemo_cuda_device(nemo_configuration_t conf, int* dev);
nemo_status_t nemo_backend(nemo_configuration_t conf, backend_t* backend);
nemo_status_t nemo_backend_description(nemo_configuration_t conf, const char** descr);
nemo_status_t nemo_set_write_only_synapses(nemo_configuration_t conf);

/* ---- Network construction: src/nemo.h:214-292, nemo_c.cpp:101-224 ---- */

nemo_network_t nemo_new_network(void);
void nemo_delete_network(nemo_network_t);
nemo_status_t nemo_add_neuron_type(nemo_network_t, const char* name, unsigned* neuron_type);
nemo_status_t nemo_add_neuron_iz(nemo_network_t, unsigned idx,
		float a, float b, float c, float d, float u, float v, float sigma);
nemo_status_t nemo_add_neuron(nemo_network_t, unsigned type, unsigned idx,
		unsigned nargs, float args[]);
nemo_status_t nemo_add_synapse(nemo_network_t, unsigned source, unsigned target,
		unsigned delay, float weight, unsigned char is_plastic, synapse_id* id);
nemo_status_t nemo_neuron_count(nemo_network_t net, unsigned* ncount);

/* ---- Simulation: src/nemo.h:311-358, nemo_c.cpp:140-166,439-484 ---- */

nemo_simulation_t nemo_new_simulation(nemo_network_t, nemo_configuration_t);
void nemo_delete_simulation(nemo_simulation_t);

/* One 1 ms cycle: gather -> neuron update -> scatter -> STDP accumulation.
 * *fired receives the fired neurons of this cycle in ascending simulation
 * order, valid until the next call (src/nemo.h:348-352, nemo_c.cpp:439-476). */
nemo_status_t nemo_step(nemo_simulation_t,
		unsigned fstim_nidx[], size_t fstim_count,
		unsigned istim_nidx[], float istim_current[], size_t istim_count,
		unsigned* fired[], size_t* fired_count);

/* src/nemo.h:356-358, nemo_c.cpp:480-484 */
nemo_status_t nemo_apply_stdp(nemo_simulation_t, float reward);

/* ---- Queries: src/nemo.h:380-581, nemo_c.cpp:228-436 ---- */

nemo_status_t nemo_get_membrane_potential(nemo_simulation_t sim, unsigned neuron, float* v);
nemo_status_t nemo_get_neuron_state_n(nemo_network_t net, unsigned neuron, unsigned var, float* val);
nemo_status_t nemo_get_neuron_parameter_n(nemo_network_t net, unsigned neuron, unsigned param, float* val);
nemo_status_t nemo_get_neuron_state_s(nemo_simulation_t sim, unsigned neuron, unsigned var, float* val);
nemo_status_t nemo_get_neuron_parameter_s(nemo_simulation_t sim, unsigned neuron, unsigned param, float* val);
nemo_status_t nemo_get_synapse_source_n(nemo_network_t, synapse_id synapse, unsigned* source);
nemo_status_t nemo_get_synapse_source_s(nemo_simulation_t, synapse_id synapse, unsigned* source);
nemo_status_t nemo_get_synapse_target_n(nemo_network_t, synapse_id synapse, unsigned* target);
nemo_status_t nemo_get_synapse_target_s(nemo_simulation_t, synapse_id synapse, unsigned* target);
nemo_status_t nemo_get_synapse_delay_n(nemo_network_t, synapse_id synapse, unsigned* delay);
nemo_status_t nemo_get_synapse_delay_s(nemo_simulation_t, synapse_id synapse, unsigned* delay);
nemo_status_t nemo_get_synapse_weight_n(nemo_network_t, synapse_id synapse, float* weight);
nemo_status_t nemo_get_synapse_weight_s(nemo_simulation_t, synapse_id synapse, float* weight);
nemo_status_t nemo_get_synapse_plastic_n(nemo_network_t, synapse_id synapse, unsigned char* plastic);
nemo_status_t nemo_get_synapse_plastic_s(nemo_simulation_t, synapse_id synapse, unsigned char* plastic);
nemo_status_t nemo_get_synapses_from_n(nemo_network_t, unsigned source, synapse_id* synapses[], size_t* len);
nemo_status_t nemo_get_synapses_from_s(nemo_simulation_t, unsigned source, synapse_id* synapses[], size_t* len);

/* ---- Modifying neurons: src/nemo.h:613-731, nemo_c.cpp:264-325 ---- */

nemo_status_t nemo_set_neuron_n(nemo_network_t, unsigned idx, unsigned nargs, float args[]);
nemo_status_t nemo_set_neuron_s(nemo_simulation_t, unsigned idx, unsigned nargs, float args[]);
nemo_status_t nemo_set_neuron_iz_n(nemo_network_t net, unsigned idx,
		float a, float b, float c, float d, float u, float v, float sigma);
nemo_status_t nemo_set_neuron_iz_s(nemo_simulation_t sim, unsigned idx,
		float a, float b, float c, float d, float u, float v, float sigma);
nemo_status_t nemo_set_neuron_state_n(nemo_network_t net, unsigned neuron, unsigned var, float val);
nemo_status_t nemo_set_neuron_parameter_n(nemo_network_t net, unsigned neuron, unsigned param, float val);
nemo_status_t nemo_set_neuron_state_s(nemo_simulation_t sim, unsigned neuron, unsigned var, float val);
nemo_status_t nemo_set_neuron_parameter_s(nemo_simulation_t sim, unsigned neuron, unsigned param, float val);

/* ---- Timers: src/nemo.h:753-762, nemo_c.cpp:501-521 ---- */

nemo_status_t nemo_elapsed_wallclock(nemo_simulation_t, unsigned long*);
nemo_status_t nemo_elapsed_simulation(nemo_simulation_t, unsigned long*);
nemo_status_t nemo_reset_timer(nemo_simulation_t);

/* ---- Errors: src/nemo.h:786-787, nemo_c.cpp:590-594 ---- */

const char* nemo_strerror(void);

#ifdef __cplusplus
}
#endif

#endif
