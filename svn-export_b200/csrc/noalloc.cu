// Residual check of an edge system that allocates nothing.
//
// Same computation as the FP64 true-residual kernel the solver uses to judge convergence
// (solver.cu, k_residual64): r = b - S x, then the Jacobi-scaled and the unscaled relative
// residual norms.  That kernel keeps its per-block partial sums and its arrival ticket in
// memory owned by an mh_handle.  Here they live in a fixed file-scope device array, so a caller
// that cannot allocate device memory can still verify a solution: the caller passes the CSR
// matrix, b, x and the outputs, all already on the device.
//
// The scratch array is part of the library image: every GPU that loads the library holds it
// (about 512 KiB) until the process exits.  All calls share it and it keeps the last call's
// contents, so the arrival ticket is cleared at the start of every call; calls that overlap on
// the GPU (different streams, or different host threads) race on it.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "mh_darcy.h"

namespace {

constexpr int kRowsPerBlock = 256;
constexpr int kMaxBlocks = MH_NOALLOC_MAX_ROWS / kRowsPerBlock;
constexpr int kMaxDevices = 64;

struct NoAllocScratch {
    double partial[kMaxBlocks][4];  // per-block sums: r'D^-1 r, b'D^-1 b, r'r, b'b
    unsigned int ticket;            // blocks that have stored their partial sums
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// Device address of g_noalloc_scratch on each device, looked up once per device.
std::mutex g_setup_mutex;
NoAllocScratch *g_scratch_addr[kMaxDevices] = {};

__global__ void __launch_bounds__(kRowsPerBlock)
    k_csr_residual_noalloc(int64_t n, const int32_t *__restrict__ row_ptr, const int32_t *__restrict__ col,
                           const double *__restrict__ val, const double *__restrict__ b,
                           const double *__restrict__ x, double *__restrict__ r, NoAllocScratch *scratch,
                           double *__restrict__ out) {
    const int64_t row = (int64_t)blockIdx.x * kRowsPerBlock + threadIdx.x;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    if (row < n) {
        double y = 0.0, d = 0.0;
        for (int32_t k = row_ptr[row]; k < row_ptr[row + 1]; ++k) {
            const int32_t c = col[k];
            const double v = val[k];
            y += v * x[c];
            if (c == row) d += v;
        }
        const double bi = b[row];
        const double ri = bi - y;
        if (r) r[row] = ri;
        const double w = d > 0.0 ? 1.0 / d : 1.0;
        s[0] = ri * ri * w;
        s[1] = bi * bi * w;
        s[2] = ri * ri;
        s[3] = bi * bi;
    }
    __shared__ double sh[kRowsPerBlock / 32][4];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        double v = s[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) sh[warp][k] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < 4; ++k) {
            double v = 0.0;
            for (int w = 0; w < kRowsPerBlock / 32; ++w) v += sh[w][k];
            scratch->partial[blockIdx.x][k] = v;
        }
        __threadfence();
        last = (atomicAdd(&scratch->ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    // the last block to arrive sums every block's partials (fixed order: thread-strided, then
    // warp shuffles, then the warps in order)
    __threadfence();
    double t[4] = {0.0, 0.0, 0.0, 0.0};
    for (unsigned int blk = threadIdx.x; blk < gridDim.x; blk += kRowsPerBlock)
#pragma unroll
        for (int k = 0; k < 4; ++k) t[k] += __ldcg(&scratch->partial[blk][k]);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        double v = t[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) sh[warp][k] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < 4; ++k) {
            t[k] = 0.0;
            for (int w = 0; w < kRowsPerBlock / 32; ++w) t[k] += sh[w][k];
        }
        out[0] = t[1] > 0.0 ? sqrt(t[0] / t[1]) : 0.0;
        out[1] = t[3] > 0.0 ? sqrt(t[2] / t[3]) : 0.0;
        out[2] = sqrt(t[2]);
        out[3] = sqrt(t[3]);
        scratch->ticket = 0u;
    }
}

}  // namespace

extern "C" int mh_csr_residual_noalloc(int64_t n, const int32_t *row_ptr, const int32_t *col, const double *val,
                                       const double *b, const double *x, double *r, double *out,
                                       void *cuda_stream) {
    if (n <= 0 || !row_ptr || !col || !val || !b || !x || !out) return MH_ERR_INVALID;
    if (n > (int64_t)MH_NOALLOC_MAX_ROWS) return MH_ERR_INVALID;  // larger than the fixed scratch
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return MH_ERR_CUDA;
    }
    NoAllocScratch *scratch = nullptr;
    {
        // set-up on the first call per device: in host code g_noalloc_scratch names a host-side
        // stand-in, so the kernel gets the device address from cudaGetSymbolAddress
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_addr[dev]) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
                cudaGetLastError();
                return MH_ERR_CUDA;
            }
            g_scratch_addr[dev] = (NoAllocScratch *)p;
        }
        scratch = g_scratch_addr[dev];
    }
    cudaStream_t s = (cudaStream_t)cuda_stream;
    if (cudaMemsetAsync(&scratch->ticket, 0, sizeof(unsigned int), s) != cudaSuccess) {
        cudaGetLastError();
        return MH_ERR_CUDA;
    }
    const unsigned blocks = (unsigned)((n + kRowsPerBlock - 1) / kRowsPerBlock);
    k_csr_residual_noalloc<<<blocks, kRowsPerBlock, 0, s>>>(n, row_ptr, col, val, b, x, r, scratch, out);
    if (cudaGetLastError() != cudaSuccess) return MH_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) {
        cudaGetLastError();
        return MH_ERR_CUDA;
    }
    return MH_OK;
}
