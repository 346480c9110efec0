/* ref_shim.h — TEST INFRASTRUCTURE.  Force-included when the reference's own
 * CUDA sources (src/kernels.cu, src/device_math.cu, src/disparitymeasurementmodel.cu)
 * are compiled as plain host C++ by oracle/Makefile, so that their per-thread
 * kernels and __host__ __device__ math can be called on the CPU to pin the oracle.
 * CUDA qualifiers become no-ops and the thread/block indices become thread-local
 * variables that ref_glue.cpp sets before calling a kernel body.  Kernels that use
 * __syncthreads-based block reductions are compiled but never called. */
#ifndef SCPHD_REF_SHIM_H
#define SCPHD_REF_SHIM_H
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#undef __global__
#define __global__
#undef __device__
#define __device__
#undef __host__
#define __host__
#undef __shared__
#define __shared__ static
#undef __forceinline__
#define __forceinline__ inline
struct ShimDim3 { unsigned x, y, z; };
extern thread_local ShimDim3 threadIdx, blockIdx, blockDim, gridDim;
inline void __syncthreads() {}
using std::isnan;
#endif
