/* A user's neuron model as a B200 plugin (include/nemo_b200_plugin.h), for
 * the tests: the quadratic integrate-and-fire update of the reference's QIF
 * plugin (src/nemo/cpu/plugins/QIF.cpp:16-107: ten RK4 substeps of 0.1 ms
 * on dv/dt = a v (v - 1) + 0.015 I, firing at v >= 1, reset to 0), written
 * as a plain CUDA kernel with the reference's float operation order. A
 * network using it must behave exactly like one using the built-in QIF.
 *
 * Built by nemo_b200.build.build_plugin into b200/libQIFPlugin.so, and with
 * QIF_PLUGIN_INIT defined into b200/libQIFPluginInit.so, which also exports
 * b200_init_neurons (initial v = 5 a, replacing the state given). */

#include <cuda_runtime.h>

#include <nemo_b200_plugin.h>

__global__ void
k_qif_plugin(b200_neuron_batch b)
{
	const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
	const unsigned lane = threadIdx.x & 31u;
	bool fired = false;
	if(i < b.count) {
		const float dt = 0.1f;
		const float a1 = __fmul_rn(0.5f, dt);
		const float a2 = dt;
		const float bb1 = __fdiv_rn(dt, 6.0f);
		const float E = b.current_epsp[i];
		const float I = b.current_ipsp[i];
		const float X = b.current_external[i];
		if(X != 0.0f) {
			b.current_external[i] = 0.0f;
		}
		const float a = b.param[i];
		float v = b.state[i];
		for(int k = 0; k < 10; ++k) {
			if(!fired) {
				const float In = __fmul_rn(__fadd_rn(__fadd_rn(E, I), X), 0.015f);
				const float k1 = __fadd_rn(__fmul_rn(__fmul_rn(a, v), __fsub_rn(v, 1.0f)), In);
				const float x2 = __fadd_rn(v, __fmul_rn(a1, k1));
				const float k2 = __fadd_rn(__fmul_rn(__fmul_rn(a, x2), __fsub_rn(x2, 1.0f)), In);
				const float x3 = __fadd_rn(v, __fmul_rn(a1, k2));
				const float k3 = __fadd_rn(__fmul_rn(__fmul_rn(a, x3), __fsub_rn(x3, 1.0f)), In);
				const float x4 = __fadd_rn(v, __fmul_rn(a2, k3));
				const float k4 = __fadd_rn(__fmul_rn(__fmul_rn(a, x4), __fsub_rn(x4, 1.0f)), In);
				const float sum = __fadd_rn(__fadd_rn(__fadd_rn(k1, __fmul_rn(2.0f, k2)), __fmul_rn(2.0f, k3)), k4);
				v = __fadd_rn(v, __fmul_rn(bb1, sum));
				fired = v >= 1.0f;
			}
		}
		fired = fired || ((b.fstim[i >> 5] >> (i & 31u)) & 1u);
		if(fired) {
			v = 0.0f;
		}
		b.state[i] = v;
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
	k_qif_plugin<<<(batch->count + 255u) / 256u, 256, 0, (cudaStream_t) stream>>>(*batch);
	return (int) cudaGetLastError();
}

#ifdef QIF_PLUGIN_INIT
__global__ void
k_qif_plugin_init(b200_neuron_batch b)
{
	const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i < b.count) {
		b.state[i] = __fmul_rn(b.param[i], 5.0f);
	}
}

extern "C" int
b200_init_neurons(const b200_neuron_batch* batch, void* stream)
{
	if(batch->count == 0) {
		return 0;
	}
	k_qif_plugin_init<<<(batch->count + 255u) / 256u, 256, 0, (cudaStream_t) stream>>>(*batch);
	return (int) cudaGetLastError();
}
#endif
