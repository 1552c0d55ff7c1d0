#ifndef NEMO_B200_TYPES_H
#define NEMO_B200_TYPES_H

/* Status codes, backend identifiers and scalar types of the NeMo C ABI.
 *
 * The numeric values are part of the binary interface and therefore match
 * the reference exactly (src/nemo/types.h:31-71): a caller compiled against
 * the reference headers sees the same codes from this library. */

#include <stdint.h>

#define NEMO_OK 0
#define NEMO_CUDA_INVOCATION_ERROR 1
#define NEMO_CUDA_ASSERTION_FAILURE 2
#define NEMO_CUDA_MEMORY_ERROR 3
#define NEMO_CUDA_ERROR 4
#define NEMO_API_UNSUPPORTED 5
#define NEMO_INVALID_INPUT 6
#define NEMO_BUFFER_OVERFLOW 7
#define NEMO_BUFFER_UNDERFLOW 8
#define NEMO_LOGIC_ERROR 9
#define NEMO_ALLOCATION_ERROR 10
#define NEMO_MPI_ERROR 11
#define NEMO_DL_ERROR 12
#define NEMO_IO_ERROR 13
#define NEMO_UNKNOWN_ERROR 14

/* src/nemo/types.h:63-66. NEMO_BACKEND_CUDA selects the B200 backend here. */
enum {
	NEMO_BACKEND_CUDA,
	NEMO_BACKEND_CPU
};

typedef unsigned backend_t;
typedef unsigned long long cycle_t;

/* (source << 32) | per-source synapse index (src/nemo/synapse_indices.hpp:28-52) */
typedef uint64_t synapse_id;

#endif
