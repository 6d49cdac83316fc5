/* Stand-in for src/nemo/internal_types.h */
#ifndef NEMO_INTERNAL_TYPES_H
#define NEMO_INTERNAL_TYPES_H
#include <nemo/types.h>
typedef int32_t fix_t;
typedef int64_t wfix_t;
typedef unsigned nidx_t;
typedef unsigned sidx_t;
typedef unsigned delay_t;
typedef uint32_t id32_t;
typedef uint64_t id64_t;
#endif
