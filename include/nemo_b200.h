#ifndef NEMO_B200_H
#define NEMO_B200_H

/* Extensions of the NeMo C ABI provided by libnemo_b200.so. None of these
 * has a counterpart in the reference C ABI (src/nemo.h); they expose the
 * device-resident forms of the step path. Errors follow the include/nemo.h
 * model (status code + nemo_strerror). */

#include <stddef.h>
#include <stdint.h>
#include <nemo.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Bulk construction: the C form of the vector overloads of the
 * reference Python binding (src/api/python/nemo_py.cpp:733-806); no
 * counterpart in the reference C ABI. Semantics are exactly those of calling
 * nemo_add_neuron / nemo_add_synapse once per element, in array order; on an
 * error the elements before the failing one stay added. ---- */

/* args is row-major: count rows of nargs floats (parameters, then state). */
nemo_status_t nemo_add_neurons(nemo_network_t, unsigned type, size_t count,
		const unsigned idx[], unsigned nargs, const float args[]);

/* plastic may be NULL (all static); ids may be NULL. */
nemo_status_t nemo_add_synapses(nemo_network_t, size_t count,
		const unsigned source[], const unsigned target[], const unsigned delay[],
		const float weight[], const unsigned char plastic[], synapse_id ids[]);

/* The vector form of nemo_get_synapse_weight_s (src/nemo.h:478-486; no
 * counterpart in the reference C ABI): weights[k] = the current weight of
 * synapse ids[k], for k < count. Errors as the single query: the first
 * invalid id fails the call (the weights before it are written). */
nemo_status_t nemo_b200_get_weights(nemo_simulation_t sim, const synapse_id ids[], size_t count, float weights[]);

/* Run `cycles` cycles (<= 1024 per call) without stimulus, entirely on the
 * device in one persistent launch of the step kernel (spike gather, neuron
 * update and STDP accumulation per cycle, one grid barrier per cycle); a
 * network with plugin neuron models (nemo_b200_plugin.h) instead queues
 * each cycle's plugin updates and step launch without host synchronisation.
 * Equivalent to `cycles` calls of nemo_step with empty stimulus. fired_counts[k] / events[k] (each may be NULL) receive the
 * number of neurons fired in cycle k and the synaptic events those firings
 * generate (fired neurons x out-degree, the throughput unit of the
 * reference benchmark, src/examples/common.cpp:93-98). */
nemo_status_t nemo_b200_run(nemo_simulation_t sim, unsigned cycles,
		uint32_t fired_counts[], uint64_t events[]);

/* Fired neurons of an earlier cycle (one of the last 1024 simulated), in the
 * same order and ownership as nemo_step's output. `cycle` counts from the
 * creation of the simulation. */
nemo_status_t nemo_b200_fired_at(nemo_simulation_t sim, uint64_t cycle,
		unsigned* fired[], size_t* fired_count);

/* Number of cycles simulated since the simulation was created. */
nemo_status_t nemo_b200_cycle(nemo_simulation_t sim, uint64_t* cycle);

/* Wait for all device work of the simulation. */
nemo_status_t nemo_b200_synchronize(nemo_simulation_t sim);

/* One simulation cycle like nemo_step, for callers that must not allocate
 * memory while the simulation runs. No counterpart in the reference C ABI.
 *
 * nemo_step grows a device and a pinned host staging buffer with cudaMalloc /
 * cudaMallocHost whenever a call brings more stimulus than any call before,
 * and returns the fired list in memory the simulation owns and resizes. A
 * device allocation synchronises the whole device and fails once the device
 * memory is fully committed; a closed-loop controller with a hard per-cycle
 * budget, or a host program whose device memory is owned by another
 * allocator, cannot accept either. This call allocates nothing, on the host or
 * the device, when it succeeds:
 *   - the stimulus is staged through one module-static device array per
 *     device (192 KB), so at most 16384 firing-stimulus entries and 16384
 *     current-stimulus entries are accepted per call; more is rejected with
 *     NEMO_INVALID_INPUT before anything runs;
 *   - the fired neurons (user indices, ascending simulation order, as
 *     nemo_step) are written to the caller's `fired` array, which must hold
 *     at least the network's neuron count (`fired_capacity`), else
 *     NEMO_INVALID_INPUT before anything runs; their number goes to
 *     *fired_count.
 * The simulation's device must be the calling thread's current device. The
 * first call on a device looks up the scratch address (cudaGetSymbolAddress)
 * and keeps it, so make one call before any latency-critical loop. Nothing in
 * the scratch has to start at zero: each call writes the entries it reads.
 * The scratch is shared by every simulation on the device, so calls for
 * simulations on the same device must not overlap in time (from several host
 * threads); calls that overlap race on the scratch. Stimulus and results are
 * otherwise identical to nemo_step's, including repeated current-stimulus
 * indices (the last entry wins) and invalid indices (the entries before the
 * invalid one are applied, then NEMO_INVALID_INPUT). */
nemo_status_t nemo_b200_step_noalloc(nemo_simulation_t sim,
		const unsigned fstim_nidx[], size_t fstim_count,
		const unsigned istim_nidx[], const float istim_current[], size_t istim_count,
		unsigned fired[], size_t fired_capacity, size_t* fired_count);

/* The status of the last call (NEMO_OK after a success): the code behind a
 * NULL returned by a constructor, whose message nemo_strerror gives. */
nemo_status_t nemo_b200_last_status(void);

/* The largest synapse delay and the weight range of a network, as the
 * reference's Network::maxDelay / minWeight / maxWeight give them (both
 * weight bounds start at 0; src/nemo/NetworkImpl.cpp:25,108-110). */
nemo_status_t nemo_b200_network_stats(nemo_network_t net, unsigned* max_delay, float* min_weight,
		float* max_weight);

/* Kernel launches one applyStdp makes (0 without plastic synapses). */
nemo_status_t nemo_b200_apply_launches(nemo_simulation_t sim, unsigned* launches);

/* Cumulative device counters since the simulation was created: out[0]
 * synapses delivered, out[1] STDP synapse visits, out[2] neurons fired,
 * out[3] synaptic events (fired neurons x out-degree). */
nemo_status_t nemo_b200_counters(nemo_simulation_t sim, uint64_t out[4]);

/* ---- batches: many independent networks in one simulation ----
 *
 * nemo_b200_new_batch builds one simulation from `count` networks that stay
 * independent (trials, parameter sweeps): they advance together in the same
 * persistent step kernel, and each gives exactly the firing it gives when
 * simulated alone (its own random seeds, its own neuron indices).
 * nemo_step / nemo_b200_run / nemo_b200_run_graph advance all instances; a
 * fired list of nemo_step holds the instances' neurons shifted by the
 * instance's base index (instances in order), so use
 * nemo_b200_batch_fired_at to read them per instance. Returns NULL on error
 * (nemo_strerror). */
nemo_simulation_t nemo_b200_new_batch(nemo_network_t nets[], size_t count, nemo_configuration_t conf);

/* ---- sharded simulation: one network over several GPUs ----
 *
 * A network too large for one GPU runs as `world` shards, one per process
 * and GPU (the reference's MPI workers, src/mpi/Worker.cpp:265-292, over
 * NVLink). Shard `rank` owns a contiguous range of the simulation's device
 * warps (32 neuron slots each, types in registration order; equal warp
 * counts) and holds only the synapses to its own neurons. Every cycle:
 *
 *   nemo_b200_shard_step     stimulus for this shard's neurons (entries for
 *                            other shards' neurons are skipped), the update
 *                            of its neurons; writes the fired words of its
 *                            own warps (shard_range: `words` uint32 from
 *                            `first_word`) to local_words (host memory);
 *   (the caller all-gathers the words of all shards, e.g. with
 *    torch.distributed, into the total_words words of the cycle)
 *   nemo_b200_shard_deliver  brings the other shards' firing of the cycle
 *                            in; returns every neuron fired in the cycle
 *                            (user indices), valid until the next call.
 *
 * Firing, currents and STDP equal those of the unsharded simulation bit for
 * bit. nemo_apply_stdp applies to the shard's synapses. A neuron's state is
 * read on the shard that owns it; synapse queries answer for the synapses
 * whose target the shard owns. nemo_step and the device-resident runs are
 * not available on a shard. Returns NULL on error (nemo_strerror). */
nemo_simulation_t nemo_b200_new_shard(nemo_network_t net, nemo_configuration_t conf, unsigned rank, unsigned world);

/* The warps shard `rank` of `world` owns out of total_words: [first_word,
 * first_word + words). Host arithmetic, no device needed. */
nemo_status_t nemo_b200_shard_warps(unsigned total_words, unsigned rank, unsigned world, unsigned* first_word,
		unsigned* words);

/* The shard's own warps and the simulation's total warps (the length of the
 * fired-word vector of a cycle). */
nemo_status_t nemo_b200_shard_range(nemo_simulation_t sim, unsigned* first_word, unsigned* words,
		unsigned* total_words);

nemo_status_t nemo_b200_shard_step(nemo_simulation_t sim, unsigned fstim_nidx[], size_t fstim_count,
		unsigned istim_nidx[], float istim_current[], size_t istim_count, uint32_t local_words[]);

nemo_status_t nemo_b200_shard_deliver(nemo_simulation_t sim, const uint32_t all_words[], unsigned* fired[],
		size_t* fired_count);

/* The same cycle with the fired words kept in device memory, for an exchange
 * by a collective on the GPUs (NCCL over NVLink) instead of through host
 * memory. Nothing waits on the host:
 *
 *   nemo_b200_shard_step_async     queues the stimulus, the update and a
 *                                  copy of the shard's own words (`words`
 *                                  of shard_range) into local_words_dev
 *                                  (device memory), and makes `stream` (a
 *                                  cudaStream_t; NULL: the legacy default
 *                                  stream) wait for that copy;
 *   (the caller all-gathers the words into all_words_dev on `stream`)
 *   nemo_b200_shard_deliver_async  makes the simulation wait for the work
 *                                  queued on `stream` so far, then brings
 *                                  the other shards' firing in from
 *                                  all_words_dev (device, total_words).
 *
 * Both buffers must stay allocated until the simulation's work that reads
 * them has run (nemo_b200_stream_wait orders a stream after it). The cycle's
 * fired neurons are read with nemo_b200_fired_at. No counterpart in the
 * reference (the MPI worker exchanges through host messages,
 * src/mpi/Worker.cpp:265-292). */
nemo_status_t nemo_b200_shard_step_async(nemo_simulation_t sim, const unsigned fstim_nidx[], size_t fstim_count,
		const unsigned istim_nidx[], const float istim_current[], size_t istim_count, uint32_t* local_words_dev,
		void* stream);
nemo_status_t nemo_b200_shard_deliver_async(nemo_simulation_t sim, const uint32_t* all_words_dev, void* stream);

/* Make `stream` (a cudaStream_t; NULL: the legacy default stream) wait for
 * every piece of work queued on the simulation so far, without waiting on the
 * host. */
nemo_status_t nemo_b200_stream_wait(nemo_simulation_t sim, void* stream);

/* Number of networks of a batch (1 for an ordinary simulation). */
nemo_status_t nemo_b200_batch_instances(nemo_simulation_t sim, size_t* count);

/* Fired neurons of every instance in `cycle` (one of the last 1024): each
 * instance's own neuron indices in its simulation order, instance after
 * instance; instance j's are fired[offsets[j] .. offsets[j+1]). Both arrays
 * belong to the simulation and stay valid until the next call. */
nemo_status_t nemo_b200_batch_fired_at(nemo_simulation_t sim, uint64_t cycle,
		const unsigned* fired[], const size_t* offsets[]);

/* Run `cycles` cycles (<= 1024) as a CUDA graph of persistent launches of at
 * most `cycles_per_launch` cycles each (0: one launch); the graph is captured
 * on the first call with given sizes and replayed afterwards. *used_graph
 * (may be NULL) is 0 when the device refused the capture and the launches
 * ran directly. Same results as nemo_b200_run. */
nemo_status_t nemo_b200_run_graph(nemo_simulation_t sim, unsigned cycles, unsigned cycles_per_launch,
		int* used_graph);

/* Choose the step kernel's work shape by timing `trial_cycles` cycles with
 * each candidate, twice, interleaved, keeping the fastest: threads per
 * partition (1024, 512 or 256; the partitions stay) and, for a network with
 * STDP, the synapses of a full STDP work entry (128 or 64: a post-spiking
 * target's plastic synapses are dealt to the warps in runs of that length).
 * The results do not depend on the shape; the trial cycles are simulated
 * like any others (2 x candidates x trial_cycles). nemo_b200_autotune:
 * ms[k] (may be NULL) the best device ms per cycle with thread size k.
 * nemo_b200_autotune_shape: ms[3 r + k] (may be NULL) with thread size k
 * and run length r (0 for r = 1 without STDP). */
nemo_status_t nemo_b200_autotune(nemo_simulation_t sim, unsigned trial_cycles, unsigned* threads, double ms[3]);
nemo_status_t nemo_b200_autotune_shape(nemo_simulation_t sim, unsigned trial_cycles, unsigned* threads,
		unsigned* stdp_run, double ms[6]);

/* Bytes that crossed the bus for nemo_step calls since the simulation was
 * made: out[0] host to device (stimulus: a resident step's command chunks,
 * else the staged stimulus), out[1] device to host (each step's fired
 * list: its count and error words, its {fired word, warp} pairs, and a
 * resident step's done word). */
nemo_status_t nemo_b200_host_bytes(nemo_simulation_t sim, unsigned long long out[2]);

/* ---- the differentiable form: discrete LIF network and its BPTT adjoint ----
 *
 * A recurrent network of leaky integrate-and-fire neurons (1 ms Euler step,
 * reset by subtraction) for up to 32 trials at once, and the exact adjoint of
 * its backpropagation through time with a fast-sigmoid surrogate
 * 1 / (1 + kappa |u - theta|)^2 standing in for the derivative of the
 * threshold (the model and the adjoint are written out in
 * nemo_b200/csrc/lif_bptt.cu). All pointers are device memory; `stream` is a
 * cudaStream_t (NULL: the default stream). Synapses are listed by target
 * (rowptr/pre: pre < N a recurrent neuron, whose spike arrives one step
 * later; pre >= N input channel pre - N, same step), and the recurrent ones
 * also by source (colptr/post/wpos, wpos the index in pre/w). Return a status;
 * nemo_b200_lif_error describes a failure. No counterpart in the reference. */
typedef struct nemo_b200_lif_net {
	int N;          /* neurons */
	int C;          /* input channels */
	int B;          /* trials, 1..32 */
	int T;          /* steps */
	int K;          /* steps between checkpoints */
	int bin_steps;  /* steps per counting bin (T a multiple of it) */
	float beta;     /* 1 - dt / tau_m */
	float theta;    /* threshold */
	float kappa;    /* surrogate slope */
	const int* rowptr;
	const int* pre;
	const int* colptr;
	const int* post;
	const int* wpos;
	int nnz_rec;    /* recurrent synapses (colptr[N]) */
} nemo_b200_lif_net;

/* Bytes of the work buffer both calls need. */
size_t nemo_b200_lif_work_bytes(const nemo_b200_lif_net* net);

/* Forward: in_bits [T][C] input spikes (bit b = trial b); outputs s_bits
 * [T][N] spikes (bit b = trial b), v_ckpt [ceil(T/K)][N][32] checkpoints and
 * counts [B][T/bin_steps] spikes per trial and bin. relaxed != 0 runs the
 * relaxed model (spike r(u - theta) = (u - theta) / (1 + kappa |u - theta|),
 * stored in s_float [T][N][32] instead of s_bits). */
int nemo_b200_lif_forward(const nemo_b200_lif_net* net, const float* w, const uint32_t* in_bits, int relaxed,
		uint32_t* s_bits, float* s_float, float* v_ckpt, float* counts, float* work, void* stream);

/* Backward: adds dL/dw into dw (pass zeros) for dL/dcounts dcounts
 * [B][T/bin_steps], from the forward's s_bits / s_float and v_ckpt, recomputing
 * each segment of K steps from its checkpoint. */
int nemo_b200_lif_backward(const nemo_b200_lif_net* net, const float* w, const uint32_t* in_bits, int relaxed,
		const uint32_t* s_bits, const float* s_float, const float* v_ckpt, const float* dcounts, float* dw,
		float* work, void* stream);

const char* nemo_b200_lif_error(void);

/* Device-timed throughput loop: `steps` repetitions of (`cycles_per_step`
 * cycles in one persistent launch, then applyStdp(reward) when apply_stdp != 0),
 * bracketed by CUDA events on the simulation's stream. out[0] = device ms,
 * out[1] = neurons fired, out[2] = synaptic events generated (fired x
 * out-degree), out[3] = synapses delivered. */
nemo_status_t nemo_b200_timed_steps(nemo_simulation_t sim, unsigned steps, unsigned cycles_per_step,
		int apply_stdp, float reward, double out[4]);

/* Device times of one persistent launch of `cycles` cycles and of one
 * applyStdp(reward) (when STDP is on), with the work they did (the cycles are
 * simulated). out[0] = step-kernel ms, out[1] = its grid blocks, out[2] = 0,
 * out[3] = synapses pushed, out[4] = neurons fired, out[5] = STDP synapse
 * visits, out[6] = neuron updates, out[7] = applyStdp ms, out[8] = plastic
 * synapses, out[9] = synaptic events generated. */
nemo_status_t nemo_b200_profile(nemo_simulation_t sim, unsigned cycles, float reward, double out[10]);

/* Phase timing of the step kernel over `cycles` cycles (one traced launch;
 * the cycles are simulated). Means over cycles, in ns: out[0] whole phase,
 * out[1] / out[2] slowest / mean block neuron update (with the delay-1
 * push), out[3] / out[4] slowest / mean block work of the phase, out[5]
 * phase start to the last block's arrival at the grid barrier, out[6] last
 * arrival to barrier exit, out[7] spread of the blocks' arrivals, out[8] /
 * out[9] slowest / mean block work left after its update, out[10] /
 * out[11] mean duration of one gather / STDP work unit of a warp, out[12] /
 * out[13] such units per block and cycle, out[14] / out[15] mean time of an
 * update warp to its model's result / to the end of its update, out[16]
 * mean time of a warp with fired neurons after its lists (delay-1 push,
 * prefetches), out[17] such warps per block and cycle, out[18] / out[19]
 * mean duration / count per block and cycle of a next-cycle noise unit,
 * out[20] mean time from a block's phase start to its last work unit taken,
 * out[21] mean time to a warp's leaving the work units, out[22] mean time
 * from a block's last unit taken to its work done, out[23] mean time from a
 * block's phase start to the end of its last unit. */
nemo_status_t nemo_b200_trace(nemo_simulation_t sim, unsigned cycles, double out[24]);

/* Diagnostics: the device noise transform of two RNG words per sample,
 * sin(2*pi*u1/2^32) * sqrt(-2 log(1 - u2/2^32)) as computed by the
 * Izhikevich kernel (glibc-matching), for n samples. */
nemo_status_t nemo_b200_nrand_probe(nemo_simulation_t sim, const uint32_t u1[], const uint32_t u2[],
		float out[], size_t n);

/* Diagnostics: evaluate the device sinf/logf of the noise generator on all
 * 83886081 inputs the RNG can produce and count results that differ from the
 * host glibc (0 when the device reproduces the reference bit for bit). */
nemo_status_t nemo_b200_libm_check(nemo_simulation_t sim, uint64_t* mismatches);

/* Diagnostics: evaluate the device expf of the Hodgkin-Huxley model on every
 * float in [-104, 89] (the range where expf is neither 0 nor infinity) and
 * count the results that differ from the host glibc (0 when the device
 * reproduces it bit for bit). */
nemo_status_t nemo_b200_expf_check(nemo_simulation_t sim, uint64_t* mismatches);

/* Diagnostics: the Hodgkin-Huxley model's divisions of -(v + 65) by 20, 80
 * and 18 (an FMA-corrected product with the rounded reciprocal) against the
 * device's correctly rounded division, on every float of magnitude at least
 * 2^-100 and on the zeros; mismatches[q] per divisor (0 when they agree). */
nemo_status_t nemo_b200_hh_division_check(uint64_t mismatches[3]);

/* The host-built table of inputs on which glibc expf rounds differently from
 * the device candidate: its size and its boundary distance (built or loaded
 * from the cache on first use; no device needed). */
nemo_status_t nemo_b200_expf_exceptions(size_t* count, double* tau);

/* Path of the glibc correction-table cache file used by this process. */
const char* nemo_b200_libm_cache_path(void);

/* Build the glibc correction tables now (and write the cache file). */
nemo_status_t nemo_b200_prepare_libm_tables(void);

#ifdef __cplusplus
}
#endif

#endif
