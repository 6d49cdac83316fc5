/* Stand-in for the reference's generated nemo/config.h (test
 * infrastructure: it lets the backend adapter compile without the
 * reference's build system).  No export attributes are needed. */
#ifndef NEMO_CONFIG_H
#define NEMO_CONFIG_H
#define NEMO_BASE_DLL_PUBLIC
#define NEMO_CUDA_DLL_PUBLIC
#endif
