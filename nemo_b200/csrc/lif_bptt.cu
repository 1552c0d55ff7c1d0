/* The differentiable form: a recurrent network of discrete leaky
 * integrate-and-fire neurons (1 ms Euler step, reset by subtraction) run
 * forward with exact spikes for up to 32 trials at once (one lane per trial),
 * and its backpropagation-through-time adjoint, with a fast-sigmoid surrogate
 * for the derivative of the threshold only. C ABI in include/nemo_b200.h
 * (nemo_b200_lif_*).
 *
 * Model, for neuron i, trial b, step t (v[-1] = 0):
 *   I[t] = sum over in-synapses k of i: w[k] * x_k[t]
 *          x_k[t] = s_j[t-1] for a recurrent synapse from neuron j (0 at t = 0),
 *                   the input channel's spike at t for an input synapse;
 *   u[t] = beta * v[t-1] + I[t];   s[t] = H(u[t] - theta);   v[t] = u[t] - theta * s[t].
 * The output is counts[b][bin] = sum over neurons and the bin's steps of s.
 *
 * Adjoint (backward through time), with s'(u) = 1 / (1 + kappa |u - theta|)^2
 * standing in for the derivative of H:
 *   gs[t]_j = dL/dcounts[b][bin(t)] + sum over recurrent out-synapses (j -> i, w):
 *             w * gu[t+1]_i
 *   gv[t]   = beta * gu[t+1]
 *   gu[t]   = s'(u[t]) * (gs[t] - theta * gv[t]) + gv[t]
 *   dL/dw[k] = sum over t, b of gu[t]_i * x_k[t]
 * The relaxed variant replaces the spike by s = r(u - theta) with
 * r(x) = x / (1 + kappa |x|), whose derivative is the surrogate exactly, so
 * that the adjoint is the true gradient of the relaxed forward (checked
 * against finite differences).
 *
 * Memory: the forward stores every step's spikes (a 32-bit word per neuron:
 * bit b = trial b) and v at every checkpoint (every K steps); the backward
 * recomputes u inside each K-step segment from its checkpoint (the same
 * operations in the same order, so u is bit-identical), then walks the
 * segment backwards. Sums run in a fixed order, so results are reproducible;
 * the weight gradient sums steps segment by segment, so its rounding (not u's)
 * depends on the checkpoint interval. */

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>

#include <nemo_b200.h>

#include "common.hpp"

namespace nemo_b200 {
namespace lif {
namespace {

const unsigned FULL = 0xffffffffu;
const unsigned THREADS = 256;

struct Net {
	int N, C, B, T, K, binSteps;
	float beta, theta, kappa;
	const int* rowptr;   /* [N + 1] in-synapses of each neuron */
	const int* pre;      /* [nnz] < N: recurrent source; >= N: input channel pre - N */
	const int* colptr;   /* [N + 1] recurrent out-synapses of each neuron */
	const int* post;     /* [nnzRec] target */
	const int* wpos;     /* [nnzRec] index of the synapse in w / pre */
	int nnzRec;          /* colptr[N] */
};

/* spike of presynaptic unit p for the lane's trial at step t */
template<bool RELAXED>
__device__ __forceinline__ float presyn(const Net& n, int p, int t, uint32_t lane, const uint32_t* sBits,
		const float* sF, const uint32_t* inBits)
{
	if(p >= n.N) {
		return float((inBits[size_t(t) * n.C + (p - n.N)] >> lane) & 1u);
	}
	if(t == 0) return 0.0f;
	if(RELAXED) {
		return sF[(size_t(t - 1) * n.N + p) * 32 + lane];
	}
	return float((sBits[size_t(t - 1) * n.N + p] >> lane) & 1u);
}

/* the spike word (bit b = trial b) of presynaptic unit p at step t */
__device__ __forceinline__ uint32_t presynWord(const Net& n, int p, int t, const uint32_t* sBits,
		const uint32_t* inBits)
{
	if(p >= n.N) return inBits[size_t(t) * n.C + (p - n.N)];
	return t == 0 ? 0u : sBits[size_t(t - 1) * n.N + p];
}

/* One forward step for every neuron (warp per neuron, lane per trial).
 * v: [N][32] state, read and written. RECOMPUTE: store u into uOut (a
 * segment buffer [K][N][32]) instead of the spikes and counts. */
template<bool RELAXED, bool RECOMPUTE>
__global__ void __launch_bounds__(THREADS)
k_step(Net n, int t, const float* w, const uint32_t* inBits, uint32_t* sBits, float* sF, float* v,
		float* vCkpt, float* counts, float* uOut, int segStart)
{
	__shared__ float sCount[32];
	const uint32_t lane = threadIdx.x & 31u;
	const bool active = lane < uint32_t(n.B);
	if(!RECOMPUTE) {
		if(threadIdx.x < 32) sCount[threadIdx.x] = 0.0f;
		__syncthreads();
	}
	const int warps = int((gridDim.x * blockDim.x) >> 5);
	for(int i = int((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < n.N; i += warps) {
		const size_t cell = size_t(i) * 32 + lane;
		const float vPrev = v[cell];
		if(!RECOMPUTE && t % n.K == 0) {
			vCkpt[size_t(t / n.K) * n.N * 32 + cell] = vPrev;
		}
		/* in-synapses in order, 32 at a time: lane L loads synapse base + L
		 * (and, for spikes as bits, the presynaptic word of all trials), then
		 * every lane takes them in turn; a word without spikes adds nothing */
		float I = 0.0f;
		const int k0 = n.rowptr[i], k1 = n.rowptr[i + 1];
		for(int base = k0; base < k1; base += 32) {
			const int k = base + int(lane);
			const int p = k < k1 ? n.pre[k] : 0;
			const float wk = k < k1 ? w[k] : 0.0f;
			const int cnt = min(32, k1 - base);
			if(RELAXED) {
				for(int q = 0; q < cnt; ++q) {
					const int pq = __shfl_sync(FULL, p, q);
					const float wq = __shfl_sync(FULL, wk, q);
					I = __fadd_rn(I, __fmul_rn(wq, presyn<RELAXED>(n, pq, t, lane, sBits, sF, inBits)));
				}
			} else {
				const uint32_t word = k < k1 ? presynWord(n, p, t, sBits, inBits) : 0u;
				uint32_t nz = __ballot_sync(FULL, word != 0u);
				while(nz) {
					const int q = __ffs(int(nz)) - 1;
					nz &= nz - 1u;
					const uint32_t wd = __shfl_sync(FULL, word, q);
					const float wq = __shfl_sync(FULL, wk, q);
					if((wd >> lane) & 1u) I = __fadd_rn(I, wq);
				}
			}
		}
		const float u = __fadd_rn(__fmul_rn(n.beta, vPrev), I);
		const float x = __fsub_rn(u, n.theta);
		float s;
		if(RELAXED) {
			s = __fdiv_rn(x, __fadd_rn(1.0f, __fmul_rn(n.kappa, fabsf(x))));
		} else {
			s = (active && u >= n.theta) ? 1.0f : 0.0f;
		}
		v[cell] = __fsub_rn(u, __fmul_rn(n.theta, s));
		if(RECOMPUTE) {
			uOut[(size_t(t - segStart) * n.N) * 32 + cell] = u;
		} else {
			if(RELAXED) {
				sF[(size_t(t) * n.N + i) * 32 + lane] = active ? s : 0.0f;
			} else {
				const uint32_t word = __ballot_sync(FULL, s != 0.0f);
				if(lane == 0) sBits[size_t(t) * n.N + i] = word;
			}
			if(active && s != 0.0f) atomicAdd(&sCount[lane], s);
		}
	}
	if(!RECOMPUTE) {
		__syncthreads();
		if(threadIdx.x < uint32_t(n.B)) {
			const float c = sCount[threadIdx.x];
			if(c != 0.0f) atomicAdd(&counts[size_t(threadIdx.x) * (n.T / n.binSteps) + t / n.binSteps], c);
		}
	}
}

/* wOut[e] = w[n.wpos[e]]: the recurrent weights in out-synapse order */
__global__ void
k_gather_out(Net n, int nnzRec, const float* w, float* wOut)
{
	for(int e = int(blockIdx.x * blockDim.x + threadIdx.x); e < nnzRec; e += int(gridDim.x * blockDim.x)) {
		wOut[e] = w[n.wpos[e]];
	}
}

/* One backward step: gu[t] of every neuron j from gu[t+1] (guNext, [N][32])
 * and u[t] (uSeg). Warp per neuron (source view), lane per trial; wOut: the
 * recurrent weights in out-synapse order. A chunk's 32 rows of guNext are
 * all loaded before they are summed (in synapse order), so that a warp keeps
 * 32 loads in flight. */
__global__ void __launch_bounds__(THREADS)
k_back(Net n, int t, const float* wOut, const float* uSeg, int segStart, const float* guNext, float* guOut,
		const float* dcounts, bool last)
{
	const uint32_t lane = threadIdx.x & 31u;
	const bool active = lane < uint32_t(n.B);
	const int warps = int((gridDim.x * blockDim.x) >> 5);
	const int bins = n.T / n.binSteps;
	for(int j = int((blockIdx.x * blockDim.x + threadIdx.x) >> 5); j < n.N; j += warps) {
		const size_t cell = size_t(j) * 32 + lane;
		float gs = active ? dcounts[size_t(lane) * bins + t / n.binSteps] : 0.0f;
		float gv = 0.0f;
		if(!last) {
			const int e0 = n.colptr[j], e1 = n.colptr[j + 1];
			for(int base = e0; base < e1; base += 32) {
				const int e = base + int(lane);
				const int i = e < e1 ? n.post[e] : 0;
				const float we = e < e1 ? wOut[e] : 0.0f;
				const int cnt = min(32, e1 - base);
				float g[32];
#pragma unroll
				for(int q = 0; q < 32; ++q) {
					const int iq = __shfl_sync(FULL, i, q);
					g[q] = q < cnt ? guNext[size_t(iq) * 32 + lane] : 0.0f;
				}
#pragma unroll
				for(int q = 0; q < 32; ++q) {
					const float wq = __shfl_sync(FULL, we, q);
					if(q < cnt) gs = __fadd_rn(gs, __fmul_rn(wq, g[q]));
				}
			}
			gv = __fmul_rn(n.beta, guNext[cell]);
		}
		const float u = uSeg[(size_t(t - segStart) * n.N) * 32 + cell];
		const float a = __fadd_rn(1.0f, __fmul_rn(n.kappa, fabsf(__fsub_rn(u, n.theta))));
		const float sp = __fdiv_rn(1.0f, __fmul_rn(a, a));
		const float gu = __fadd_rn(__fmul_rn(sp, __fsub_rn(gs, __fmul_rn(n.theta, gv))), gv);
		guOut[(size_t(t - segStart) * n.N) * 32 + cell] = active ? gu : 0.0f;
	}
}

/* dL/dw over one segment: for every in-synapse k of neuron i, the sum over
 * the segment's steps and the trials of gu[t]_i * x_k[t]; warp per neuron,
 * lanes summing their trial over the steps, one reduction per synapse. */
template<bool RELAXED>
__global__ void __launch_bounds__(THREADS)
k_dw(Net n, int segStart, int segEnd, const float* guSeg, const uint32_t* sBits, const float* sF,
		const uint32_t* inBits, float* dw)
{
	const uint32_t lane = threadIdx.x & 31u;
	const int warps = int((gridDim.x * blockDim.x) >> 5);
	for(int i = int((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < n.N; i += warps) {
		const int k0 = n.rowptr[i], k1 = n.rowptr[i + 1];
		for(int k = k0; k < k1; ++k) {
			const int p = n.pre[k];
			float acc = 0.0f;
			for(int t = segStart; t < segEnd; ++t) {
				if(RELAXED) {
					const float g = guSeg[(size_t(t - segStart) * n.N + i) * 32 + lane];
					acc = __fadd_rn(acc, __fmul_rn(g, presyn<RELAXED>(n, p, t, lane, sBits, sF, inBits)));
				} else {
					/* spikes are 0 or 1: add gu where the trial's bit is set */
					const uint32_t word = presynWord(n, p, t, sBits, inBits);
					if(word && ((word >> lane) & 1u)) {
						acc = __fadd_rn(acc, guSeg[(size_t(t - segStart) * n.N + i) * 32 + lane]);
					}
				}
			}
#pragma unroll
			for(int d = 16; d; d >>= 1) acc = __fadd_rn(acc, __shfl_xor_sync(FULL, acc, d));
			if(lane == 0) dw[k] = __fadd_rn(dw[k], acc);
		}
	}
}

/* dL/dw over one segment for spikes as bits: lanes over the neuron's
 * in-synapses, each lane walking its synapse's presynaptic words along the
 * segment (words stored source-major, [unit][T], so consecutive steps are
 * consecutive words) and adding gu[t]_i of every trial whose bit is set. */
__global__ void __launch_bounds__(THREADS)
k_dw_bits(Net n, int segStart, int segEnd, const float* guSeg, const uint32_t* sT, const uint32_t* inT, float* dw)
{
	const uint32_t lane = threadIdx.x & 31u;
	const int warps = int((gridDim.x * blockDim.x) >> 5);
	for(int i = int((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < n.N; i += warps) {
		const int k0 = n.rowptr[i], k1 = n.rowptr[i + 1];
		for(int base = k0; base < k1; base += 32) {
			const int k = base + int(lane);
			if(k >= k1) continue;
			const int p = n.pre[k];
			const bool input = p >= n.N;
			const uint32_t* words = input ? inT + size_t(p - n.N) * n.T : sT + size_t(p) * n.T;
			float acc = 0.0f;
			for(int t = segStart; t < segEnd; ++t) {
				uint32_t word = input ? words[t] : (t == 0 ? 0u : words[t - 1]);
				while(word) {
					const int b = __ffs(int(word)) - 1;
					word &= word - 1u;
					acc = __fadd_rn(acc, __ldg(&guSeg[(size_t(t - segStart) * n.N + i) * 32 + b]));
				}
			}
			dw[k] = __fadd_rn(dw[k], acc);
		}
	}
}

/* dst[c][r] = src[r][c] for a rows x cols array of words */
__global__ void
k_transpose(const uint32_t* src, uint32_t* dst, int rows, int cols)
{
	__shared__ uint32_t tile[32][33];
	const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
	for(int y = threadIdx.y; y < 32; y += blockDim.y) {
		const int r = r0 + y, c = c0 + int(threadIdx.x);
		if(r < rows && c < cols) tile[y][threadIdx.x] = src[size_t(r) * cols + c];
	}
	__syncthreads();
	for(int y = threadIdx.y; y < 32; y += blockDim.y) {
		const int c = c0 + y, r = r0 + int(threadIdx.x);
		if(r < rows && c < cols) dst[size_t(c) * rows + r] = tile[threadIdx.x][y];
	}
}

static void
transpose(const uint32_t* src, uint32_t* dst, int rows, int cols, cudaStream_t st)
{
	if(rows == 0 || cols == 0) return;
	dim3 g((cols + 31) / 32, (rows + 31) / 32), b(32, 8);
	k_transpose<<<g, b, 0, st>>>(src, dst, rows, cols);
}

static int
grid(int N)
{
	int dev = 0, sms = 148;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	const long warps = long(N);
	long blocks = (warps * 32 + THREADS - 1) / THREADS;
	const long cap = long(sms) * 8;
	return int(blocks < cap ? blocks : cap);
}

static void
validate(const Net& n)
{
	if(n.N <= 0 || n.T <= 0 || n.K <= 0 || n.binSteps <= 0 || n.C < 0) {
		fail(NEMO_INVALID_INPUT, "lif: sizes must be positive");
	}
	if(n.B < 1 || n.B > 32) {
		fail(NEMO_INVALID_INPUT, "lif: 1 to 32 trials per call (one lane each)");
	}
	if(n.T % n.binSteps != 0) {
		fail(NEMO_INVALID_INPUT, "lif: the steps must be a whole number of bins");
	}
	if(n.nnzRec < 0) {
		fail(NEMO_INVALID_INPUT, "lif: negative recurrent synapse count");
	}
}

} // namespace
} // namespace lif
} // namespace nemo_b200

using namespace nemo_b200;

/* work buffer: v state [N][32], gu of the step after the segment [N][32],
 * the segment's u and gu [K][N][32], the spike and input words transposed to
 * [unit][T], then the recurrent weights in out-synapse order [nnzRec] */
static size_t
workFloats(const lif::Net& n)
{
	return size_t(n.N) * 32 * (2 + 2 * size_t(n.K)) + (size_t(n.N) + size_t(n.C)) * size_t(n.T)
		+ size_t(n.nnzRec);
}

static std::string g_lifError;

#define LIF_CALL(...) \
	try { __VA_ARGS__; return NEMO_OK; } \
	catch(Exception& e) { g_lifError = e.what(); return e.code(); } \
	catch(std::exception& e) { g_lifError = e.what(); return NEMO_UNKNOWN_ERROR; }

extern "C" {

const char* nemo_b200_lif_error(void) { return g_lifError.c_str(); }

size_t
nemo_b200_lif_work_bytes(const nemo_b200_lif_net* net)
{
	lif::Net n;
	static_assert(sizeof(nemo_b200_lif_net) == sizeof(lif::Net), "layout");
	memcpy(&n, net, sizeof(n));
	return workFloats(n) * sizeof(float);
}

int
nemo_b200_lif_forward(const nemo_b200_lif_net* net, const float* w, const uint32_t* in_bits, int relaxed,
		uint32_t* s_bits, float* s_float, float* v_ckpt, float* counts, float* work, void* stream)
{
	LIF_CALL({
		lif::Net n;
		memcpy(&n, net, sizeof(n));
		lif::validate(n);
		cudaStream_t st = static_cast<cudaStream_t>(stream);
		float* v = work;
		NEMO_CUDA(cudaMemsetAsync(v, 0, size_t(n.N) * 32 * 4, st));
		NEMO_CUDA(cudaMemsetAsync(counts, 0, size_t(n.B) * (n.T / n.binSteps) * 4, st));
		const int g = lif::grid(n.N);
		for(int t = 0; t < n.T; ++t) {
			if(relaxed) {
				lif::k_step<true, false><<<g, lif::THREADS, 0, st>>>(n, t, w, in_bits, s_bits, s_float, v, v_ckpt,
						counts, nullptr, 0);
			} else {
				lif::k_step<false, false><<<g, lif::THREADS, 0, st>>>(n, t, w, in_bits, s_bits, s_float, v, v_ckpt,
						counts, nullptr, 0);
			}
		}
		NEMO_CUDA(cudaGetLastError());
	})
}

int
nemo_b200_lif_backward(const nemo_b200_lif_net* net, const float* w, const uint32_t* in_bits, int relaxed,
		const uint32_t* s_bits, const float* s_float, const float* v_ckpt, const float* dcounts, float* dw,
		float* work, void* stream)
{
	LIF_CALL({
		lif::Net n;
		memcpy(&n, net, sizeof(n));
		lif::validate(n);
		cudaStream_t st = static_cast<cudaStream_t>(stream);
		const size_t NS = size_t(n.N) * 32;
		float* v = work;
		float* guNextSeg = work + NS;          /* gu of the first step after the segment */
		float* uSeg = work + 2 * NS;
		float* guSeg = uSeg + size_t(n.K) * NS;
		uint32_t* sT = reinterpret_cast<uint32_t*>(guSeg + size_t(n.K) * NS);
		uint32_t* inT = sT + size_t(n.N) * n.T;
		if(!relaxed) {
			lif::transpose(s_bits, sT, n.T, n.N, st);
			lif::transpose(in_bits, inT, n.T, n.C, st);
		}
		const int g = lif::grid(n.N);
		/* the recurrent weights in out-synapse order, for k_back */
		float* wOut = reinterpret_cast<float*>(inT + size_t(n.C) * n.T);
		if(n.nnzRec) lif::k_gather_out<<<g, lif::THREADS, 0, st>>>(n, n.nnzRec, w, wOut);
		const int segments = (n.T + n.K - 1) / n.K;
		for(int sgi = segments - 1; sgi >= 0; --sgi) {
			const int c0 = sgi * n.K, c1 = std::min(n.T, c0 + n.K);
			/* recompute u over the segment from its checkpoint */
			NEMO_CUDA(cudaMemcpyAsync(v, v_ckpt + size_t(sgi) * NS, NS * 4, cudaMemcpyDeviceToDevice, st));
			for(int t = c0; t < c1; ++t) {
				if(relaxed) {
					lif::k_step<true, true><<<g, lif::THREADS, 0, st>>>(n, t, w, in_bits, nullptr,
							const_cast<float*>(s_float), v, nullptr, nullptr, uSeg, c0);
				} else {
					lif::k_step<false, true><<<g, lif::THREADS, 0, st>>>(n, t, w, in_bits,
							const_cast<uint32_t*>(s_bits), nullptr, v, nullptr, nullptr, uSeg, c0);
				}
			}
			/* backwards through the segment */
			for(int t = c1 - 1; t >= c0; --t) {
				const bool last = t == n.T - 1;
				const float* next = t == c1 - 1 ? guNextSeg : guSeg + size_t(t + 1 - c0) * NS;
				lif::k_back<<<g, lif::THREADS, 0, st>>>(n, t, wOut, uSeg, c0, next, guSeg, dcounts, last);
			}
			if(relaxed) {
				lif::k_dw<true><<<g, lif::THREADS, 0, st>>>(n, c0, c1, guSeg, s_bits, s_float, in_bits, dw);
			} else {
				lif::k_dw_bits<<<g, lif::THREADS, 0, st>>>(n, c0, c1, guSeg, sT, inT, dw);
			}
			NEMO_CUDA(cudaMemcpyAsync(guNextSeg, guSeg, NS * 4, cudaMemcpyDeviceToDevice, st));
		}
		NEMO_CUDA(cudaGetLastError());
	})
}

} // extern "C"
