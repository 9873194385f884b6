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
//
// In host code g_noalloc_scratch names a host-side stand-in, so the kernel is given the array's
// device address, looked up with cudaGetSymbolAddress.  That address belongs to a CUDA context
// (the module holding the array is loaded into each context separately), so it is cached per
// context id: a context created after cudaDeviceReset, or a driver-API context the caller made
// current, gets its own lookup.  CUDA loads modules lazily, and the first lookup in a context
// loads this file's module, which allocates device memory for its code and the array; a call
// with n == 0 does only that set-up, so callers can run it while allocation still succeeds.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "mh_darcy.h"

namespace {

constexpr int kRowsPerBlock = 256;
constexpr int kMaxBlocks = MH_NOALLOC_MAX_ROWS / kRowsPerBlock;
constexpr int kMaxContexts = 64;

struct NoAllocScratch {
    double partial[kMaxBlocks][4];  // per-block sums: r'D^-1 r, b'D^-1 b, r'r, b'b
    unsigned int ticket;            // blocks that have stored their partial sums
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

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

// ---- per-context cache of the scratch array's device address -----------------------------
typedef CUresult(CUDAAPI *PFN_ctx_current)(CUcontext *);
typedef CUresult(CUDAAPI *PFN_ctx_id)(CUcontext, unsigned long long *);

struct ContextEntry {
    unsigned long long ctx_id;
    NoAllocScratch *addr;
};

std::mutex g_setup_mutex;
std::once_flag g_driver_once;
PFN_ctx_current g_ctx_current = nullptr;
PFN_ctx_id g_ctx_id = nullptr;
ContextEntry g_contexts[kMaxContexts];
int g_n_contexts = 0;

void load_driver_entry_points() {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_ctx_current = (PFN_ctx_current)f;
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_ctx_id = (PFN_ctx_id)f;
    cudaGetLastError();  // a failed lookup only disables the cache; it is not this call's error
}

// Device address of g_noalloc_scratch in the context current on this thread.  Looked up once per
// context; when no context is current yet (the lookup then initialises the device's primary
// context) or the driver lacks cuCtxGetId (before CUDA 12.0), it is looked up without caching.
cudaError_t scratch_address(NoAllocScratch **out) {
    std::call_once(g_driver_once, load_driver_entry_points);
    unsigned long long id = 0;
    bool have_id = false;
    if (g_ctx_current && g_ctx_id) {
        CUcontext ctx = nullptr;
        have_id = g_ctx_current(&ctx) == CUDA_SUCCESS && ctx && g_ctx_id(ctx, &id) == CUDA_SUCCESS;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (have_id)
        for (int i = 0; i < g_n_contexts; ++i)
            if (g_contexts[i].ctx_id == id) {
                *out = g_contexts[i].addr;
                return cudaSuccess;
            }
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    if (!p) return cudaErrorInvalidSymbol;
    // load the kernel too, so that a set-up call leaves nothing for a later call to load
    cudaFuncAttributes attr;
    e = cudaFuncGetAttributes(&attr, k_csr_residual_noalloc);
    if (e != cudaSuccess) return e;
    if (have_id && g_n_contexts < kMaxContexts) g_contexts[g_n_contexts++] = {id, (NoAllocScratch *)p};
    *out = (NoAllocScratch *)p;
    return cudaSuccess;
}

bool overlaps(const void *a, const void *b, int64_t n) {
    const uintptr_t pa = (uintptr_t)a, pb = (uintptr_t)b, bytes = (uintptr_t)n * sizeof(double);
    return pa < pb + bytes && pb < pa + bytes;
}

}  // namespace

extern "C" int mh_csr_residual_noalloc(int64_t n, const int32_t *row_ptr, const int32_t *col, const double *val,
                                       const double *b, const double *x, double *r, double *out,
                                       void *cuda_stream) {
    if (n < 0 || n > (int64_t)MH_NOALLOC_MAX_ROWS) return MH_ERR_INVALID;  // beyond the fixed scratch
    if (n > 0) {
        if (!row_ptr || !col || !val || !b || !x || !out) return MH_ERR_INVALID;
        // the kernel reads x and b while other threads write r
        if (r && (overlaps(r, x, n) || overlaps(r, b, n))) return MH_ERR_INVALID;
    }
    // an error left by the caller's earlier work is not this call's: report it, leave it pending
    if (cudaPeekAtLastError() != cudaSuccess) return MH_ERR_CUDA;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
        cudaGetLastError();
        return MH_ERR_CUDA;
    }
    NoAllocScratch *scratch = nullptr;
    if (scratch_address(&scratch) != cudaSuccess) {
        cudaGetLastError();
        return MH_ERR_CUDA;
    }
    if (n == 0) return MH_OK;  // set-up only
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
