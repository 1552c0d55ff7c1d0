#ifndef NEMO_B200_COMPILE_HPP
#define NEMO_B200_COMPILE_HPP

/* The network compiler on the device: the forward matrix (delay >= 2
 * synapses in buckets of block group, source and owner block, then the
 * delay-1 synapses by source; kernels.hpp NetDev::segOff) and the reverse
 * matrix of plastic synapses, built with stable radix sorts on the GPU
 * instead of the constructor's host counting sorts (the reference builds
 * them with maps on the host: src/nemo/ConnectivityMatrix.cpp:128-193,
 * src/nemo/cuda/ConnectivityMatrix.cpp:39-101). Element for element equal
 * to the host build. */

#include <cstddef>
#include <cstdint>
#include <functional>
#include <vector>

#include <vector_types.h>

namespace nemo_b200 {

struct LayoutIn {
	size_t S;                    /* synapses */
	uint32_t nDev;               /* device neurons */
	uint32_t blocks;             /* owner blocks (regions) */
	uint32_t warpLo;             /* first owned warp */
	uint32_t ownedWarps;         /* entries of ownerOfWarp */
	bool stdp;                   /* build the reverse matrix */
	bool wantFcmPos;             /* return each synapse's forward position */
	/* host arrays of S entries, in the network's insertion order */
	const uint32_t* src;         /* device index */
	const uint32_t* tgt;         /* device index */
	const int32_t* wfx;          /* Q11.20 weight */
	const uint32_t* dly;         /* 1 .. 64 */
	const uint8_t* plastic;
	const uint32_t* ownerOfWarp; /* owner block of each owned warp (host) */
	uint32_t groups;             /* block groups */
	const uint32_t* groupFirst;  /* [groups + 1] first block of each group (host) */
	const uint32_t* groupOf;     /* [blocks] group of each block (host) */
};

struct LayoutOut {
	/* device arrays, allocated through the caller's allocator */
	uint2* fcm = nullptr;            /* [S] */
	uint32_t* segOff = nullptr;      /* [blocks * nDev + 1] bucket starts */
	uint32_t* d1Start = nullptr;     /* [nDev + 1] */
	uint32_t* rcmStart = nullptr;    /* [nDev + 1] */
	uint32_t* rcmSrcDelay = nullptr; /* [nrcm] */
	uint32_t* rcmForward = nullptr;  /* [nrcm] */
	int32_t* rcmWeight = nullptr;    /* [nrcm] */
	/* host results */
	uint64_t d1Base = 0;              /* first delay-1 record */
	std::vector<uint32_t> fcmPos;     /* [S] when wantFcmPos */
	uint64_t nrcm = 0;
	uint64_t maxIn = 0;               /* most plastic in-synapses of a target */
};

/* Whether the device build handles these sizes (its bucket table of
 * blocks x nDev + nDev + 1 counters fits a 31-bit index). */
bool layoutOnDevice(size_t S, uint32_t nDev, uint32_t blocks);

/* Build the layout on the device on `stream` (a cudaStream_t). `keep`
 * allocates the device arrays that outlive the call; temporaries are freed
 * before it returns. Raises NEMO_LOGIC_ERROR if an input is out of range
 * (the host validates them first). */
void buildLayoutOnDevice(const LayoutIn& in, const std::function<void*(size_t)>& keep, LayoutOut* out,
		void* stream);

} // namespace nemo_b200

#endif
