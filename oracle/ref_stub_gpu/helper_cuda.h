/* Stand-in for the CUDA-samples helper header the reference includes, for the
   reference's own GPU build (oracle/build_ref_gpu.sh): checkCudaErrors reports
   a failed CUDA call and ends the process, as the samples' macro does. */
#pragma once
#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>
#define checkCudaErrors(val)                                                                            \
    do {                                                                                                \
        cudaError_t e_ = (cudaError_t)(val);                                                            \
        if (e_ != cudaSuccess) {                                                                        \
            std::fprintf(stderr, "CUDA error %d (%s) at %s:%d\n", (int)e_, cudaGetErrorString(e_), __FILE__, \
                         __LINE__);                                                                     \
            std::exit(1);                                                                               \
        }                                                                                               \
    } while (0)
