/* A second user's neuron model as a B200 plugin (include/nemo_b200_plugin.h),
 * for the tests: the leaky integrate-and-fire update with exponential
 * synaptic currents of the reference's IF_curr_exp plugin
 * (src/nemo/cpu/plugins/IF_curr_exp.cpp:27-122), with the reference's float
 * operation order. Nine parameters and four state variables, addressed
 * through the batch's strides. Built by nemo_b200.build.build_plugin into
 * b200/libLIFPlugin.so. */

#include <cuda_runtime.h>

#include <nemo_b200_plugin.h>

__global__ void
k_lif_plugin(b200_neuron_batch b)
{
	const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
	const unsigned lane = threadIdx.x & 31u;
	bool fired = false;
	if(i < b.count) {
		const float* P = b.param;
		float* S = b.state;
		const size_t ps = b.param_stride, ss = b.state_stride;
		const float v_rest = P[0 * ps + i], v_reset = P[1 * ps + i], c_m = P[2 * ps + i];
		const float tau_m = P[3 * ps + i], tau_refrac = P[4 * ps + i];
		const float tau_e = P[5 * ps + i], tau_i = P[6 * ps + i];
		const float v_thresh = P[7 * ps + i], i_offset = P[8 * ps + i];
		float v = S[0 * ss + i];
		const float ie0 = S[1 * ss + i], ii0 = S[2 * ss + i], lastfire = S[3 * ss + i];
		const float X = b.current_external[i];
		if(X != 0.0f) {
			b.current_external[i] = 0.0f;
		}
		const float ie = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, __fdiv_rn(1.0f, tau_e)), ie0), b.current_epsp[i]);
		const float ii = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, __fdiv_rn(1.0f, tau_i)), ii0), b.current_ipsp[i]);
		const float In = __fadd_rn(__fadd_rn(__fadd_rn(ie, ii), X), i_offset);
		S[1 * ss + i] = ie;
		S[2 * ss + i] = ii;
		const bool refractory = lastfire <= tau_refrac;
		if(!refractory) {
			v = __fadd_rn(v, __fadd_rn(__fdiv_rn(In, c_m), __fdiv_rn(__fsub_rn(v_rest, v), tau_m)));
		}
		const bool stim = (b.fstim[i >> 5] >> (i & 31u)) & 1u;
		fired = (!refractory && v > v_thresh) || stim;
		S[3 * ss + i] = fired ? 1.0f : __fadd_rn(lastfire, 1.0f);
		S[0 * ss + i] = fired ? v_reset : v;
	}
	/* blocks are whole warps: every lane reaches the ballot */
	const unsigned word = __ballot_sync(0xffffffffu, fired);
	if(lane == 0 && i < ((b.count + 31u) & ~31u)) {
		b.fired[i >> 5] = word;
	}
}

extern "C" int
b200_update_neurons(const b200_neuron_batch* batch, void* stream)
{
	if(batch->count == 0) {
		return 0;
	}
	k_lif_plugin<<<(batch->count + 255u) / 256u, 256, 0, (cudaStream_t) stream>>>(*batch);
	return (int) cudaGetLastError();
}
