/* Stand-in for src/nemo/types.h: status codes, backend ids and basic
 * types, with the reference's include guard and values. */
#ifndef NEMO_TYPES_H
#define NEMO_TYPES_H
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
enum { NEMO_BACKEND_CUDA, NEMO_BACKEND_CPU };
typedef unsigned backend_t;
typedef unsigned long long cycle_t;
typedef uint64_t synapse_id;
#endif
