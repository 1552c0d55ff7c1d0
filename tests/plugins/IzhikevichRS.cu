/* The reference's IzhikevichRS model, which it ships only as a CUDA kernel
 * (src/nemo/cuda/plugins/IzhikevichRS.cu:65-140), as a B200 plugin
 * (include/nemo_b200_plugin.h): a regular-spiking Izhikevich neuron with
 * fixed a = 0.02, b = 0.2 and reset v = -65, u += 8, no parameters, state u
 * and v, four float Euler substeps of 0.25 ms with u updated in each, firing
 * at v >= 30. Used by the tests to run the reference's no-parameter model
 * test (src/test/test.cpp:988-1006). Built by nemo_b200.build.build_plugin
 * into b200/libIzhikevichRS.so. */

#include <cuda_runtime.h>

#include <nemo_b200_plugin.h>

__global__ void
k_izhikevich_rs(b200_neuron_batch b)
{
	const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
	const unsigned lane = threadIdx.x & 31u;
	bool fired = false;
	if(i < b.count) {
		float* U = b.state;
		float* V = b.state + b.state_stride;
		float u = U[i];
		float v = V[i];
		const float a = 0.02f, bb = 0.2f;
		const float X = b.current_external[i];
		if(X != 0.0f) {
			b.current_external[i] = 0.0f;
		}
		const float I = __fadd_rn(__fadd_rn(b.current_epsp[i], b.current_ipsp[i]), X);
		for(int j = 0; j < 4; ++j) {
			if(!fired) {
				const float dv = __fadd_rn(__fsub_rn(__fadd_rn(__fmul_rn(__fadd_rn(__fmul_rn(0.04f, v), 5.0f), v),
								140.0f), u), I);
				v = __fadd_rn(v, __fmul_rn(0.25f, dv));
				u = __fadd_rn(u, __fmul_rn(0.25f, __fmul_rn(a, __fsub_rn(__fmul_rn(bb, v), u))));
				fired = v >= 30.0f;
			}
		}
		fired = fired || ((b.fstim[i >> 5] >> (i & 31u)) & 1u);
		if(fired) {
			v = -65.0f;
			u = __fadd_rn(u, 8.0f);
		}
		U[i] = u;
		V[i] = v;
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
	k_izhikevich_rs<<<(batch->count + 255u) / 256u, 256, 0, (cudaStream_t) stream>>>(*batch);
	return (int) cudaGetLastError();
}
