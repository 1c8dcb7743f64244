/* Minimal stand-in for the CUDA-samples header the reference includes
 * (include/FAME_CUDA.h:7).  Only checkCudaErrors is used by the reference. */
#ifndef FAME_REF_SHIM_HELPER_CUDA_H
#define FAME_REF_SHIM_HELPER_CUDA_H
#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>
#define checkCudaErrors(call)                                                    \
  do {                                                                           \
    cudaError_t e_ = (call);                                                     \
    if (e_ != cudaSuccess) {                                                     \
      std::fprintf(stderr, "CUDA error %s at %s:%d\n", cudaGetErrorString(e_),   \
                   __FILE__, __LINE__);                                          \
      std::exit(3);                                                              \
    }                                                                            \
  } while (0)
#endif
