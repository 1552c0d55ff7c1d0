/* The network compiler on the device (compile.hpp): stable radix sorts
 * (CUB) reproduce the constructor's host counting sorts exactly.
 *
 * Forward matrix. Each synapse gets the key of its bucket: a delay >= 2
 * synapse whose target block b belongs to block group g goes to
 * groupFirst[g] x nDev + source x blocks(g) + (b - groupFirst[g]), a delay-1
 * synapse to blocks x nDev + source, after every group. A stable sort of
 * (key, insertion index) puts the synapses in forward order: by group, in a
 * group by source, for a source by block, in a bucket by insertion order, as
 * the host fills them. The exclusive sum of the bucket counts gives the
 * bucket starts and the delay-1 starts.
 *
 * Reverse matrix. Walking the forward order, a plastic synapse gets the key
 * of its target and any other the key nDev (after all targets); a stable sort
 * of (key, forward position) groups the plastic synapses by target in
 * forward order, the order the host fills them in. */

#include "compile.hpp"

#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>

#include "common.hpp"

namespace nemo_b200 {

namespace {

/* a device temporary, freed on scope exit once the work queued on its
 * stream (which may still read it) has finished, on error paths too */
struct Temp {
	void* p = nullptr;
	cudaStream_t st;
	Temp(size_t bytes, cudaStream_t s) : st(s) { NEMO_CUDA(cudaMalloc(&p, bytes ? bytes : 16)); }
	~Temp()
	{
		if(p) {
			cudaStreamSynchronize(st);
			cudaFree(p);
		}
	}
	Temp(const Temp&) = delete;
	Temp& operator=(const Temp&) = delete;
	template<class T> T* as() const { return static_cast<T*>(p); }
};

unsigned
gridFor(size_t n)
{
	return unsigned(std::min<size_t>((n + 255) / 256, size_t(148) * 32));
}

/* bits needed for the values 0 .. x */
int
bitsFor(uint64_t x)
{
	int b = 1;
	while(b < 64 && (x >> b) != 0) ++b;
	return b;
}

__global__ void
k_forward_keys(size_t S, uint32_t nDev, uint32_t B, uint32_t warpLo, uint32_t ownedWarps, uint32_t G,
		const uint32_t* src, const uint32_t* tgt, const uint32_t* dly, const uint32_t* ownerOfWarp,
		const uint32_t* groupFirst, const uint32_t* groupOf,
		unsigned long long* key, uint32_t* val, uint32_t* cnt, uint32_t* bad)
{
	for(size_t s = blockIdx.x * size_t(blockDim.x) + threadIdx.x; s < S; s += size_t(gridDim.x) * blockDim.x) {
		const uint32_t a = src[s], t = tgt[s], d = dly[s];
		unsigned long long k = 0ull;
		bool ok = a < nDev && t < nDev && d >= 1u && d <= 64u;
		if(ok && d == 1u) {
			k = (unsigned long long) B * nDev + a;
		} else if(ok) {
			const uint32_t tw = t / 32u;
			ok = tw >= warpLo && tw - warpLo < ownedWarps;
			const uint32_t b = ok ? ownerOfWarp[tw - warpLo] : 0u;
			ok = ok && b < B;
			const uint32_t g = ok ? groupOf[b] : 0u;
			ok = ok && g < G;
			const uint32_t g0 = ok ? groupFirst[g] : 0u, g1 = ok ? groupFirst[g + 1] : 1u;
			ok = ok && g0 <= b && b < g1 && g1 <= B;
			k = ok ? (unsigned long long) g0 * nDev + (unsigned long long) a * (g1 - g0) + (b - g0) : 0ull;
		}
		if(ok) {
			atomicAdd(&cnt[k], 1u);
		} else {
			atomicOr(bad, 1u);
			k = 0ull;
		}
		key[s] = k;
		val[s] = uint32_t(s);
	}
}

__global__ void
k_forward_fill(size_t S, const uint32_t* synAt, const uint32_t* tgt, const uint32_t* dly, const int32_t* wfx,
		uint2* fcm, uint32_t* fcmPos, uint32_t* bad)
{
	for(size_t p = blockIdx.x * size_t(blockDim.x) + threadIdx.x; p < S; p += size_t(gridDim.x) * blockDim.x) {
		const uint32_t s = synAt[p];
		if(s >= S) {
			atomicOr(bad, 2u);
			continue;
		}
		fcm[p] = make_uint2((tgt[s] << 6) | (dly[s] - 1u), uint32_t(wfx[s]));
		if(fcmPos) fcmPos[s] = uint32_t(p);
	}
}

/* start: exclusive sum of the bucket counts, B x nDev + nDev + 1 entries:
 * the first B x nDev + 1 are the bucket starts, the rest (less the first
 * delay-1 position) the delay-1 starts */
__global__ void
k_forward_offsets(const uint32_t* start, uint32_t nDev, uint32_t B, uint32_t* d1Start)
{
	const size_t base = size_t(B) * nDev;
	for(size_t a = blockIdx.x * size_t(blockDim.x) + threadIdx.x; a <= nDev; a += size_t(gridDim.x) * blockDim.x) {
		d1Start[a] = start[base + a] - start[base];
	}
}

__global__ void
k_reverse_keys(size_t S, uint32_t nDev, const uint32_t* synAt, const uint32_t* tgt, const uint8_t* plastic,
		uint32_t* key, uint32_t* val, uint32_t* cntT)
{
	for(size_t p = blockIdx.x * size_t(blockDim.x) + threadIdx.x; p < S; p += size_t(gridDim.x) * blockDim.x) {
		const uint32_t s = synAt[p];
		const uint32_t t = tgt[s];
		const bool pl = plastic[s] != 0;
		key[p] = pl ? t : nDev;
		val[p] = uint32_t(p);
		if(pl) atomicAdd(&cntT[t], 1u);
	}
}

__global__ void
k_reverse_fill(size_t nrcm, const uint32_t* rpos, const uint32_t* synAt, const uint32_t* src, const uint32_t* dly,
		const int32_t* wfx, uint32_t* rcmSrcDelay, uint32_t* rcmForward, int32_t* rcmWeight)
{
	for(size_t j = blockIdx.x * size_t(blockDim.x) + threadIdx.x; j < nrcm; j += size_t(gridDim.x) * blockDim.x) {
		const uint32_t p = rpos[j];
		const uint32_t s = synAt[p];
		rcmSrcDelay[j] = (src[s] << 6) | (dly[s] - 1u);
		rcmForward[j] = p;
		rcmWeight[j] = wfx[s];
	}
}

} // namespace

bool
layoutOnDevice(size_t S, uint32_t nDev, uint32_t blocks)
{
	const uint64_t buckets = uint64_t(blocks) * nDev + nDev + 1;
	return S > 0 && S < (uint64_t(1) << 32) && buckets < (uint64_t(1) << 31);
}

void
buildLayoutOnDevice(const LayoutIn& in, const std::function<void*(size_t)>& keep, LayoutOut* out, void* streamPtr)
{
	cudaStream_t st = static_cast<cudaStream_t>(streamPtr);
	const size_t S = in.S;
	const uint32_t nDev = in.nDev, B = in.blocks;
	if(!layoutOnDevice(S, nDev, B)) {
		fail(NEMO_LOGIC_ERROR, "device layout build: sizes out of range");
	}
	const size_t buckets = size_t(B) * nDev + nDev + 1;

	/* inputs */
	Temp src(S * 4, st), tgt(S * 4, st), wfx(S * 4, st), dly(S * 4, st), plastic(S, st),
		owner(size_t(in.ownedWarps) * 4, st), bad(4, st), gFirst((size_t(in.groups) + 1) * 4, st),
		gOf(size_t(B) * 4, st);
	NEMO_CUDA(cudaMemcpyAsync(src.p, in.src, S * 4, cudaMemcpyHostToDevice, st));
	NEMO_CUDA(cudaMemcpyAsync(tgt.p, in.tgt, S * 4, cudaMemcpyHostToDevice, st));
	NEMO_CUDA(cudaMemcpyAsync(wfx.p, in.wfx, S * 4, cudaMemcpyHostToDevice, st));
	NEMO_CUDA(cudaMemcpyAsync(dly.p, in.dly, S * 4, cudaMemcpyHostToDevice, st));
	NEMO_CUDA(cudaMemcpyAsync(plastic.p, in.plastic, S, cudaMemcpyHostToDevice, st));
	if(in.ownedWarps) {
		NEMO_CUDA(cudaMemcpyAsync(owner.p, in.ownerOfWarp, size_t(in.ownedWarps) * 4, cudaMemcpyHostToDevice, st));
	}
	NEMO_CUDA(cudaMemcpyAsync(gFirst.p, in.groupFirst, (size_t(in.groups) + 1) * 4, cudaMemcpyHostToDevice, st));
	NEMO_CUDA(cudaMemcpyAsync(gOf.p, in.groupOf, size_t(B) * 4, cudaMemcpyHostToDevice, st));
	NEMO_CUDA(cudaMemsetAsync(bad.p, 0, 4, st));

	/* ---- forward matrix ---- */
	Temp cnt(buckets * 4, st), start(buckets * 4, st);
	NEMO_CUDA(cudaMemsetAsync(cnt.p, 0, buckets * 4, st));
	Temp keyIn(S * 8, st), keyOut(S * 8, st), valIn(S * 4, st), synAt(S * 4, st);
	k_forward_keys<<<gridFor(S), 256, 0, st>>>(S, nDev, B, in.warpLo, in.ownedWarps, in.groups, src.as<uint32_t>(),
			tgt.as<uint32_t>(), dly.as<uint32_t>(), owner.as<uint32_t>(), gFirst.as<uint32_t>(), gOf.as<uint32_t>(),
			keyIn.as<unsigned long long>(), valIn.as<uint32_t>(), cnt.as<uint32_t>(), bad.as<uint32_t>());
	NEMO_CUDA(cudaGetLastError());
	{
		size_t bytes = 0;
		const int bits = bitsFor(uint64_t(buckets) - 1);
		NEMO_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, keyIn.as<unsigned long long>(),
				keyOut.as<unsigned long long>(), valIn.as<uint32_t>(), synAt.as<uint32_t>(), uint32_t(S), 0, bits, st));
		Temp tmp(bytes, st);
		NEMO_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, bytes, keyIn.as<unsigned long long>(),
				keyOut.as<unsigned long long>(), valIn.as<uint32_t>(), synAt.as<uint32_t>(), uint32_t(S), 0, bits, st));
	}
	{
		size_t bytes = 0;
		NEMO_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, cnt.as<uint32_t>(), start.as<uint32_t>(), buckets, st));
		Temp tmp(bytes, st);
		NEMO_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, bytes, cnt.as<uint32_t>(), start.as<uint32_t>(), buckets, st));
	}
	out->fcm = static_cast<uint2*>(keep(S * 8));
	const size_t segEntries = size_t(B) * nDev + 1;
	out->segOff = static_cast<uint32_t*>(keep(segEntries * 4));
	out->d1Start = static_cast<uint32_t*>(keep((size_t(nDev) + 1) * 4));
	Temp fcmPos(in.wantFcmPos ? S * 4 : 16, st);
	k_forward_fill<<<gridFor(S), 256, 0, st>>>(S, synAt.as<uint32_t>(), tgt.as<uint32_t>(), dly.as<uint32_t>(),
			wfx.as<int32_t>(), out->fcm, in.wantFcmPos ? fcmPos.as<uint32_t>() : nullptr, bad.as<uint32_t>());
	NEMO_CUDA(cudaGetLastError());
	NEMO_CUDA(cudaMemcpyAsync(out->segOff, start.p, segEntries * 4, cudaMemcpyDeviceToDevice, st));
	k_forward_offsets<<<gridFor(size_t(nDev) + 1), 256, 0, st>>>(start.as<uint32_t>(), nDev, B, out->d1Start);
	NEMO_CUDA(cudaGetLastError());
	uint32_t hBad = 0, hD1 = 0;
	NEMO_CUDA(cudaMemcpyAsync(&hBad, bad.p, 4, cudaMemcpyDeviceToHost, st));
	NEMO_CUDA(cudaMemcpyAsync(&hD1, start.as<uint32_t>() + size_t(B) * nDev, 4, cudaMemcpyDeviceToHost, st));
	NEMO_CUDA(cudaStreamSynchronize(st));
	out->d1Base = hD1;
	if(hBad) {
		fail(NEMO_LOGIC_ERROR, "device layout build: a synapse's neuron, delay or owner is out of range");
	}
	if(in.wantFcmPos) {
		out->fcmPos.resize(S);
		NEMO_CUDA(cudaMemcpyAsync(out->fcmPos.data(), fcmPos.p, S * 4, cudaMemcpyDeviceToHost, st));
	}

	/* ---- reverse matrix of the plastic synapses ---- */
	if(in.stdp) {
		Temp cntT((size_t(nDev) + 1) * 4, st), rKeyIn(S * 4, st), rKeyOut(S * 4, st), rValIn(S * 4, st),
			rPos(S * 4, st);
		NEMO_CUDA(cudaMemsetAsync(cntT.p, 0, (size_t(nDev) + 1) * 4, st));
		k_reverse_keys<<<gridFor(S), 256, 0, st>>>(S, nDev, synAt.as<uint32_t>(), tgt.as<uint32_t>(),
				plastic.as<uint8_t>(), rKeyIn.as<uint32_t>(), rValIn.as<uint32_t>(), cntT.as<uint32_t>());
		NEMO_CUDA(cudaGetLastError());
		{
			size_t bytes = 0;
			const int bits = bitsFor(nDev);
			NEMO_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, rKeyIn.as<uint32_t>(), rKeyOut.as<uint32_t>(),
					rValIn.as<uint32_t>(), rPos.as<uint32_t>(), uint32_t(S), 0, bits, st));
			Temp tmp(bytes, st);
			NEMO_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, bytes, rKeyIn.as<uint32_t>(), rKeyOut.as<uint32_t>(),
					rValIn.as<uint32_t>(), rPos.as<uint32_t>(), uint32_t(S), 0, bits, st));
		}
		out->rcmStart = static_cast<uint32_t*>(keep((size_t(nDev) + 1) * 4));
		{
			size_t bytes = 0;
			NEMO_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, cntT.as<uint32_t>(), out->rcmStart,
					size_t(nDev) + 1, st));
			Temp tmp(bytes, st);
			NEMO_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, bytes, cntT.as<uint32_t>(), out->rcmStart,
					size_t(nDev) + 1, st));
		}
		std::vector<uint32_t> hStart(size_t(nDev) + 1);
		NEMO_CUDA(cudaMemcpyAsync(hStart.data(), out->rcmStart, hStart.size() * 4, cudaMemcpyDeviceToHost, st));
		NEMO_CUDA(cudaStreamSynchronize(st));
		out->nrcm = hStart[nDev];
		out->maxIn = 0;
		for(uint32_t n = 0; n < nDev; ++n) out->maxIn = std::max<uint64_t>(out->maxIn, hStart[n + 1] - hStart[n]);
		out->rcmSrcDelay = static_cast<uint32_t*>(keep(out->nrcm * 4));
		out->rcmForward = static_cast<uint32_t*>(keep(out->nrcm * 4));
		out->rcmWeight = static_cast<int32_t*>(keep(out->nrcm * 4));
		if(out->nrcm) {
			k_reverse_fill<<<gridFor(out->nrcm), 256, 0, st>>>(out->nrcm, rPos.as<uint32_t>(), synAt.as<uint32_t>(),
					src.as<uint32_t>(), dly.as<uint32_t>(), wfx.as<int32_t>(), out->rcmSrcDelay, out->rcmForward,
					out->rcmWeight);
			NEMO_CUDA(cudaGetLastError());
		}
	}
	NEMO_CUDA(cudaStreamSynchronize(st));
}

} // namespace nemo_b200
