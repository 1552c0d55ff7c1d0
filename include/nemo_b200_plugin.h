#ifndef NEMO_B200_PLUGIN_H
#define NEMO_B200_PLUGIN_H

/* GPU neuron-model plugins for the B200 backend.
 *
 * The reference loads a neuron model as lib<Name>.so from
 * <plugindir>/{cpu,cuda}/ beside <Name>.ini (src/nemo/NeuronType.cpp:48-73)
 * and calls its cpu_update_neurons / cuda_update_neurons
 * (src/nemo/cpu/plugins/neuron_model.h:25-51,
 * src/nemo/cuda/plugins/neuron_model.h:26-62). The CUDA signature is tied to
 * the reference's partition layout; this is the B200 backend's own: a model
 * whose name is not one of the built-in models (Izhikevich, IF_curr_exp, QIF,
 * HH, PoissonSource, Input) is loaded from <plugindir>/b200/lib<Name>.so,
 * where <plugindir> is the directory of <Name>.ini. The .ini keeps the
 * reference's schema (parameters, state-variables, membrane-potential,
 * history, rng.normal, rcm.*, backends.*).
 *
 * Each cycle, for each population of the plugin's type, the simulation
 * calls b200_update_neurons on its own CUDA stream after the population's
 * synaptic currents of the cycle are complete and before the cycle's spikes
 * are delivered. The call launches the model's kernels on that stream and
 * returns without synchronising; it must write the population's firing bits
 * for the cycle. Everything else (the firing history, the fired list,
 * spike delivery, STDP) is the simulation's.
 *
 * All pointers in the batch are device pointers, valid for the duration of
 * the call's work on the stream. Neuron i of the population (0 <= i < count)
 * is the i-th neuron of its type in the simulation's order (ascending user
 * index within the type for networks built neuron by neuron).
 */

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct b200_neuron_batch {
	/* neurons of this type in the simulation */
	unsigned count;
	/* cycles since the last timer reset, the cycle being computed
	 * (the reference's `cycle` argument) */
	unsigned long long cycle;
	/* param[p * param_stride + i], p < the .ini's `parameters` */
	const float* param;
	size_t param_stride;
	/* state[s * state_stride + i], s < the .ini's `state-variables`; read
	 * and written by the model */
	float* state;
	size_t state_stride;
	/* this cycle's input currents from excitatory (w >= 0) and inhibitory
	 * synapses, after the fixed-point sums are saturated and converted
	 * (src/nemo/fixedpoint.cpp:40-49); read only */
	const float* current_epsp;
	const float* current_ipsp;
	/* user-provided current of this cycle: read, then cleared to 0 by the
	 * model (the reference's post-condition on currentExternal) */
	float* current_external;
	/* firing stimulus of this cycle: bit (i % 32) of word i / 32; a
	 * stimulated neuron fires (the model applies its reset) */
	const uint32_t* fstim;
	/* firing history before this cycle: bit k set if neuron i fired k + 1
	 * cycles ago */
	const uint64_t* recent_firing;
	/* output: bit (i % 32) of word i / 32 set if neuron i fires this cycle;
	 * every one of the (count + 31) / 32 words is written, bits at or above
	 * count are ignored */
	uint32_t* fired;
	/* per-neuron xorshift128 state, four words per neuron (rng[4 i .. 4 i + 3]),
	 * seeded as the reference seeds it (src/nemo/RNG.cpp:39-62) */
	uint32_t* rng;
} b200_neuron_batch;

/* The binary layout of b200_neuron_batch and of the calls below. Every
 * source that includes this header defines `b200_plugin_abi_version` (a weak,
 * exported constant; define NEMO_B200_PLUGIN_HOST before the include to leave
 * it out), so a plugin carries the layout it was compiled against, and the
 * simulation refuses a plugin whose version is missing or differs from its
 * own with NEMO_DL_ERROR instead of running it with wrong field offsets. */
#define NEMO_B200_PLUGIN_ABI_VERSION 1u

#if !defined(NEMO_B200_PLUGIN_HOST)
#ifdef __cplusplus
extern   /* a const at namespace scope has internal linkage in C++ otherwise */
#endif
__attribute__((weak, visibility("default"))) const unsigned b200_plugin_abi_version = NEMO_B200_PLUGIN_ABI_VERSION;
#endif

/* Update one population for one cycle. `stream` is the simulation's
 * cudaStream_t. Returns 0 (cudaSuccess) or a CUDA error code, which the
 * simulation reports as NEMO_CUDA_INVOCATION_ERROR. Exported by the plugin
 * as `b200_update_neurons`. */
typedef int b200_update_neurons_t(const b200_neuron_batch* batch, void* stream);

/* Optional: called once per population when the simulation is created,
 * after the parameters, state and RNG are on the device (`cycle` 0, the
 * currents, fstim and fired null), for models that derive state from
 * parameters. Exported as `b200_init_neurons`. */
typedef int b200_init_neurons_t(const b200_neuron_batch* batch, void* stream);

#ifdef __cplusplus
}
#endif

#endif
