/* Host-side stand-in for the CUDA headers the reference includes, so that the
   reference's own kernel sources (LBFS.cu, immersed_boundary_method.cu,
   spring_network.cu, common_kernels.cu) compile with g++ as plain C++ and run
   serially on the CPU.  Test infrastructure only: it lets the oracle be pinned
   against the reference's unmodified kernel bodies.

   Execution model: every __global__ function becomes an ordinary function; a
   "launch" is a direct call with gridDim = blockDim = 1 and
   blockIdx = threadIdx = 0, so each grid-stride loop visits every element in
   index order on one host thread.  __shared__ variables become ordinary
   function locals (each kernel writes them before use; the shared-memory
   reduction templates are never called).  The CAS-based atomic add of
   the reference becomes a plain read-modify-write, which is exact on one
   thread. */
#pragma once
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>

struct uint3 { unsigned int x, y, z; };
struct dim3 { unsigned int x, y, z; };
struct int3 { int x, y, z; };
struct float3 { float x, y, z; };
struct double2 { double x, y; };
struct double3 { double x, y, z; };
struct double4 { double x, y, z, w; };
inline double3 make_double3(double x, double y, double z) { double3 r; r.x = x; r.y = y; r.z = z; return r; }
inline double4 make_double4(double x, double y, double z, double w) { double4 r; r.x = x; r.y = y; r.z = z; r.w = w; return r; }

#define __device__
#define __global__
#define __host__
#define __forceinline__ inline
#define __constant__
#define __shared__

extern uint3 threadIdx, blockIdx;
extern dim3 blockDim, gridDim;

inline void __syncthreads() {}
inline long long __double_as_longlong(double d) { long long r; std::memcpy(&r, &d, 8); return r; }
inline double __longlong_as_double(long long l) { double r; std::memcpy(&r, &l, 8); return r; }
inline unsigned long long atomicCAS(unsigned long long *addr, unsigned long long cmp, unsigned long long val) {
    unsigned long long old = *addr;
    if (old == cmp) *addr = val;
    return old;
}
/* CUDA device code resolves abs/min/max on doubles to the floating-point
   overloads; make the host build do the same. */
using std::abs;
using std::isnan;
using std::isinf;
inline double min(double a, double b) { return std::fmin(a, b); }
inline double max(double a, double b) { return std::fmax(a, b); }

typedef int cudaError_t;
/* The reference's unused NaN checker issues a GPU trap instruction; on the host it is a no-op. */
#define asm(...) ((void)0)
