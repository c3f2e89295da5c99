// Residual RMS norms without any device allocation.
//
// Some callers cannot call cudaMalloc: a host code that drives the step from
// inside a CUDA-graph capture or a stream callback (cudaMalloc is not a
// stream-ordered operation: it is illegal during capture and synchronises the
// device), and integrations whose device memory is entirely reserved by their
// own pool allocator, with nothing left for a library to allocate.  For them
// this file provides lbfs_residual_rms_noalloc, a variant of the residual
// reduction of the cell-update kernel (k_cell_update) whose block partial sums
// and completion ticket live in a file-scope __device__ array instead of
// memory the solver handle allocates.  The caller passes the residual field
// and the output in device memory.
//
// The array is LBFS_NOALLOC_MAX_BLOCKS * 4 doubles (2 MiB) plus one slot for
// the ticket;
// every GPU that loads this library holds it until the process exits.  All
// calls on a device share it and it keeps the last call's contents: the ticket
// is cleared (cudaMemsetAsync, no allocation) before every launch, the partial
// slots are written before they are read.  Calls that overlap on the GPU (two
// streams, or two threads) race on the array: serialise them.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "lbfs_b200.h"
#include "lbfs_internal.h"

namespace lbfs {
namespace {

constexpr int kNoallocThreads = 256;

// Scratch layout: 4 partial sums per block, then one 8-byte slot holding the
// completion ticket.
constexpr size_t kScratchDoubles = 4 * (size_t)LBFS_NOALLOC_MAX_BLOCKS + 1;
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

struct NoallocScratch {
    double *partials;
    unsigned int *ticket;
};

// Address of g_noalloc_scratch on each device, resolved once per device with
// that device current (the host-side symbol is only a stand-in, not a device
// address).  The table lives as long as the process: cudaDeviceReset (or any
// other reset of a device's primary context) unloads the module, and the next
// load may place the array elsewhere, so a caller that resets a device must
// not call lbfs_residual_rms_noalloc on it afterwards in the same process.
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
double *g_noalloc_ptr[kMaxDevices] = {};

int scratch_for_current_device(NoallocScratch *out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(LBFS_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return set_error(LBFS_ERR_LIMIT, "device index beyond the no-allocation table");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return set_error(LBFS_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_noalloc_ptr[dev] = (double *)p;
    }
    out->partials = g_noalloc_ptr[dev];
    out->ticket = (unsigned int *)(g_noalloc_ptr[dev] + 4 * (size_t)LBFS_NOALLOC_MAX_BLOCKS);
    return LBFS_OK;
}

// One cell per thread; block partials of the four squared residuals with the
// warp tree of k_cell_update, then the last block to finish sums the partials
// in a fixed assignment and writes the RMS norms.
__global__ void __launch_bounds__(kNoallocThreads)
    k_residual_rms_noalloc(const double *__restrict__ res, int n_cells, double ref_rho, double ref_mom,
                           NoallocScratch scratch, double *__restrict__ rms) {
    __shared__ double sh[4][kNoallocThreads / 32];
    __shared__ bool last_block;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double sq[4] = {0, 0, 0, 0};
    if (i < n_cells) {
#pragma unroll
        for (int m = 0; m < 4; m++) {
            const double r = res[4 * (size_t)i + m];
            sq[m] = r * r;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int m = 0; m < 4; m++) {
        double v = sq[m];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[m][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int m = 0; m < 4; m++) {
            double v = 0;
            for (int w = 0; w < kNoallocThreads / 32; w++) v += sh[m][w];
            scratch.partials[4 * blockIdx.x + m] = v;
        }
        __threadfence();
        last_block = atomicAdd(scratch.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last_block) return;
    __threadfence();
    double acc[4] = {0, 0, 0, 0};
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
#pragma unroll
        for (int m = 0; m < 4; m++) acc[m] += __ldcg(scratch.partials + 4 * b + m);
#pragma unroll
    for (int m = 0; m < 4; m++) {
        double v = acc[m];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[m][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double v = 0;
        for (int w = 0; w < kNoallocThreads / 32; w++) v += sh[threadIdx.x][w];
        rms[threadIdx.x] = sqrt(v / n_cells) / (threadIdx.x == 0 ? ref_rho : ref_mom);
    }
}

}  // namespace
}  // namespace lbfs

using namespace lbfs;

extern "C" int lbfs_residual_rms_noalloc(const double *d_res, int32_t n_cells, double ref_rho, double max_velocity,
                                         double *d_rms, void *stream) {
    if (!d_res || !d_rms || n_cells <= 0) return set_error(LBFS_ERR_ARG, "null pointer or no cells");
    const long long blocks = ((long long)n_cells + kNoallocThreads - 1) / kNoallocThreads;
    if (blocks > LBFS_NOALLOC_MAX_BLOCKS)
        return set_error(LBFS_ERR_LIMIT, "lbfs_residual_rms_noalloc: n_cells exceeds LBFS_NOALLOC_MAX_CELLS (" +
                                             std::to_string((long long)LBFS_NOALLOC_MAX_CELLS) + ")");
    cudaStream_t s = (cudaStream_t)stream;
    if (s) {
        // the scratch address is the current device's: the stream must belong to it
        int cur = 0, sdev = 0;
        cudaError_t e = cudaGetDevice(&cur);
        if (e == cudaSuccess) e = cudaStreamGetDevice(s, &sdev);
        if (e != cudaSuccess) return set_error(LBFS_ERR_CUDA, std::string("stream device: ") + cudaGetErrorString(e));
        if (sdev != cur)
            return set_error(LBFS_ERR_ARG, "lbfs_residual_rms_noalloc: the stream belongs to device " +
                                               std::to_string(sdev) + ", the current device is " + std::to_string(cur));
    }
    NoallocScratch scratch;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    cudaError_t e = cudaMemsetAsync(scratch.ticket, 0, sizeof(unsigned int), s);
    if (e != cudaSuccess) return set_error(LBFS_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    k_residual_rms_noalloc<<<(unsigned int)blocks, kNoallocThreads, 0, s>>>(d_res, n_cells, ref_rho,
                                                                          ref_rho * max_velocity, scratch, d_rms);
    e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(LBFS_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return LBFS_OK;
}
