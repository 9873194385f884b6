// Aggregation multigrid preconditioner: GPU setup (pairwise aggregation, Galerkin products,
// dense coarsest inverse) and the V-cycle.  See amg.hpp for the method.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>

#include <cooperative_groups.h>
#include <cuda_fp16.h>

#include "amg.hpp"

namespace cg = cooperative_groups;

namespace mh {

template <class T> cudaError_t DBuf<T>::ensure(size_t n) {
    if (p && n <= cap) return cudaSuccess;
    release();
    const size_t m = n ? n : 1;
    cudaError_t e = cudaMalloc(&p, m * sizeof(T));
    if (e != cudaSuccess) {
        p = nullptr;
        return e;
    }
    cap = m;
    return cudaSuccess;
}
template <class T> void DBuf<T>::release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
}
template struct DBuf<int32_t>;
template struct DBuf<int64_t>;
template struct DBuf<float>;
template struct DBuf<double>;
template struct DBuf<unsigned int>;
template struct DBuf<uint16_t>;
template struct DBuf<unsigned char>;

namespace {

constexpr int kS = kSliceRows;  // SELL slice height
constexpr int32_t kUnmatched = -2, kSingle = -1, kExcluded = -3;
// Galerkin row kernel tiers: candidate entries per coarse row and warps per block (the shared
// gather buffer is warps x entries x 8 bytes; the large tier's 128 KB is dynamic)
constexpr int kGalCap0 = 256, kGalWarps0 = 4, kGalCapBig = 16384, kGalWarpsBig = 1;
constexpr unsigned kFull = 0xffffffffu;

inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }
inline int64_t round_up(int64_t n, int64_t m) { return (n + m - 1) / m * m; }

struct MatView {
    int64_t n;
    const int64_t *off;
    const int32_t *col;
    const float *val;
    const int32_t *rlen;  // entries of each row (coarse matrices), null: the slice width
    const __half *hval;   // FP16 copy of val read by the cycle's fine-level kernels, or null
};
MatView view(const AmgMatrix &A) { return {A.n, A.slice_off, A.col, A.val, A.rlen, nullptr}; }

// Rows longer than this (hub aggregates: a fracture intersection or a channel that couples to
// every aggregate along it) are skipped by the thread-per-row kernels and handled by a block
// each (k_long_rows), so that one row does not serialise its warp.
constexpr int kLongRow = 96;
__device__ __forceinline__ bool is_long(const MatView &A, int64_t i) { return A.rlen && A.rlen[i] > kLongRow; }

// Cycle kernels return at once when every instance of the Krylov run has finished: the
// captured iteration graph then costs only launches.
struct Gate {
    const int32_t *n_done;
    int32_t n_inst;
};
__device__ __forceinline__ bool closed(const Gate &g) { return g.n_done && *g.n_done >= g.n_inst; }

__device__ __forceinline__ void row_of(const MatView &A, int64_t i, int64_t &base, int &w, int &ln) {
    const int64_t sl = i / kS;
    ln = (int)(i - sl * kS);
    base = A.off[sl];
    w = (int)((A.off[sl + 1] - base) / kS);
    if (A.rlen && A.rlen[i] < w) w = A.rlen[i];  // a row stops at its own last entry
}

// ---- scans (exclusive, out[n] = total) ----------------------------------------------------
template <typename T> __device__ __forceinline__ T block_incl_scan(T v, T *ws, T &block_total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[warp] = x;
    __syncthreads();
    if (warp == 0) {
        T w = lane < (int)(blockDim.x >> 5) ? ws[lane] : T(0);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const T y = __shfl_up_sync(kFull, w, o);
            if (lane >= o) w += y;
        }
        ws[lane] = w;
    }
    __syncthreads();
    const T res = (warp ? ws[warp - 1] : T(0)) + x;
    block_total = ws[(blockDim.x >> 5) - 1];
    __syncthreads();
    return res;
}

template <typename T> __global__ void __launch_bounds__(1024) k_scan_block(const T *in, T *out, T *bsum, int64_t n) {
    __shared__ T ws[32];
    const int64_t i = (int64_t)blockIdx.x * 1024 + threadIdx.x;
    const T v = i < n ? in[i] : T(0);
    T tot;
    const T incl = block_incl_scan<T>(v, ws, tot);
    if (i < n) out[i] = incl - v;
    if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

template <typename T> __global__ void __launch_bounds__(1024) k_scan_sums(T *bsum, int64_t nb) {
    __shared__ T ws[32];
    T carry = 0;
    for (int64_t base = 0; base < nb; base += 1024) {
        const int64_t i = base + threadIdx.x;
        const T v = i < nb ? bsum[i] : T(0);
        T tot;
        const T incl = block_incl_scan<T>(v, ws, tot);
        if (i < nb) bsum[i] = carry + incl - v;
        carry += tot;
    }
    if (threadIdx.x == 0) bsum[nb] = carry;
}

template <typename T> __global__ void k_scan_add(T *out, const T *bsum, int64_t n, int64_t nb) {
    const int64_t i = (int64_t)blockIdx.x * 1024 + threadIdx.x;
    if (i < n) out[i] += bsum[blockIdx.x];
    if (i == 0) out[n] = bsum[nb];
}

// the whole scan in one block (small n: one launch instead of three)
constexpr int64_t kScanOneMax = 8192;
template <typename T> __global__ void __launch_bounds__(1024) k_scan_one(const T *in, T *out, int64_t n) {
    __shared__ T ws[32];
    T carry = 0;
    for (int64_t base = 0; base < n; base += 1024) {
        const int64_t i = base + threadIdx.x;
        const T v = i < n ? in[i] : T(0);
        T tot;
        const T incl = block_incl_scan<T>(v, ws, tot);
        if (i < n) out[i] = carry + incl - v;
        carry += tot;
    }
    if (threadIdx.x == 0) out[n] = carry;
}

// exclusive scan of in[0, n) into out[0, n], out[n] = total, stream-ordered
template <typename T> cudaError_t launch_scan(const T *in, T *out, int64_t n, DBuf<T> &blk, cudaStream_t s) {
    if (n <= 0) return cudaMemsetAsync(out, 0, sizeof(T), s);
    if (n <= kScanOneMax) {
        k_scan_one<T><<<1, 1024, 0, s>>>(in, out, n);
        return cudaGetLastError();
    }
    const int64_t nb = (n + 1023) / 1024;
    cudaError_t e = blk.ensure(nb + 1);
    if (e != cudaSuccess) return e;
    k_scan_block<T><<<(unsigned)nb, 1024, 0, s>>>(in, out, blk.p, n);
    k_scan_sums<T><<<1, 1024, 0, s>>>(blk.p, nb);
    k_scan_add<T><<<(unsigned)nb, 1024, 0, s>>>(out, blk.p, n, nb);
    return cudaGetLastError();
}

// Row kernels with G warps per 32-row slice (blocks of 8 warps): row i of warp g of its slice's
// group; the warp takes the slots g, g + G, g + 2G, ... of the row.
template <int G> __device__ __forceinline__ void split_row(int64_t &i, int &g) {
    const int64_t gw = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    i = (gw / G) * kS + (threadIdx.x & 31);
    g = (int)(gw % G);
}

// ---- level statistics ----------------------------------------------------------------------
// inv_diag = 1/a_ii, isd = 1/sqrt(a_ii) (0 where there is no positive diagonal) and the
// Gershgorin bound max_i sum_j |a_ij| / a_ii of D^-1 A.
template <int G>
__global__ void __launch_bounds__(256) k_level_diag(MatView A, float *inv_diag, float *isd, unsigned int *bound) {
    int64_t i;
    int g;
    split_row<G>(i, g);
    const bool live = i < A.n && !is_long(A, i);  // long rows: k_level_diag_long
    float dg = 0.f, sum = 0.f;
    if (live) {
        int64_t base;
        int w, ln;
        row_of(A, i, base, w, ln);
        constexpr int kB = 8;
        for (int j0 = g; j0 < w; j0 += kB * G) {
            int32_t c[kB];
            float v[kB];
#pragma unroll
            for (int k = 0; k < kB; ++k) {
                const int j = j0 + k * G;
                const int64_t slot = base + (int64_t)j * kS + ln;
                c[k] = j < w ? __ldg(A.col + slot) : -1;
                v[k] = j < w ? __ldg(A.val + slot) : 0.f;
            }
#pragma unroll
            for (int k = 0; k < kB; ++k) {
                if (c[k] == (int32_t)i) dg += v[k];
                sum += fabsf(v[k]);
            }
        }
    }
    if constexpr (G > 1) {
        __shared__ float part[2][8][32];
        const int wb = threadIdx.x >> 5, lane = threadIdx.x & 31;
        part[0][wb][lane] = dg;
        part[1][wb][lane] = sum;
        __syncthreads();
        if (wb % G == 0) {
            dg = sum = 0.f;
#pragma unroll
            for (int k = 0; k < G; ++k) {
                dg += part[0][wb + k][lane];
                sum += part[1][wb + k][lane];
            }
        }
    }
    float s = 0.f;
    if (live && g == 0) {
        const bool ok = dg > 0.f;
        inv_diag[i] = ok ? 1.f / dg : 0.f;
        isd[i] = ok ? rsqrtf(dg) : 0.f;
        s = ok ? sum / dg : 0.f;
    }
    // one atomic per block (one per warp on a single word serialises at the L2)
    __shared__ float wmax[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s = fmaxf(s, __shfl_xor_sync(kFull, s, o));
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float m = 0.f;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) m = fmaxf(m, wmax[k]);
        if (m > 0.f) atomicMax(bound, __float_as_uint(m));
    }
}

// the same for the long rows, one block each
__device__ void k_level_diag_long_row(MatView A, int64_t i, float *inv_diag, float *isd, unsigned int *bound) {
    int64_t base;
    int w, ln;
    row_of(A, i, base, w, ln);
    float dg = 0.f, sum = 0.f;
    for (int j = threadIdx.x; j < w; j += blockDim.x) {
        const int64_t slot = base + (int64_t)j * kS + ln;
        const float v = A.val[slot];
        if (A.col[slot] == (int32_t)i) dg += v;
        sum += fabsf(v);
    }
    __shared__ float red[2][8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        dg += __shfl_xor_sync(kFull, dg, o);
        sum += __shfl_xor_sync(kFull, sum, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = dg;
        red[1][threadIdx.x >> 5] = sum;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        dg = 0.f;
        sum = 0.f;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            dg += red[0][k];
            sum += red[1][k];
        }
        const bool ok = dg > 0.f;
        inv_diag[i] = ok ? 1.f / dg : 0.f;
        isd[i] = ok ? rsqrtf(dg) : 0.f;
        if (ok) atomicMax(bound, __float_as_uint(sum / dg));
    }
}

__global__ void __launch_bounds__(256) k_level_diag_long(MatView A, const int32_t *__restrict__ list, float *inv_diag,
                                                         float *isd, unsigned int *bound) {
    // list = [count, rows...]; the blocks stride over the rows
    for (int32_t k = blockIdx.x; k < list[0]; k += gridDim.x) {
        k_level_diag_long_row(A, list[1 + k], inv_diag, isd, bound);
        __syncthreads();
    }
}

// ---- pairwise aggregation ------------------------------------------------------------------
// A row takes part if it is a real row (row_edge >= 0 on the fine level) with at least one
// non-zero off-diagonal entry.  The rest (padding, decoupled Dirichlet edges, and coarse rows
// left without coupling, e.g. a whole batch instance reduced to one row) get agg = -1: they
// leave the hierarchy and the smoother solves them exactly (x = b / a_ii).
__global__ void k_pair_init(MatView A, const int32_t *row_edge, const float *isd, int32_t *mate) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    bool coupled = false;
    if ((!row_edge || row_edge[i] >= 0) && isd[i] > 0.f) {
        int64_t base;
        int w, ln;
        row_of(A, i, base, w, ln);
        for (int j = 0; j < w && !coupled; ++j) {
            const int64_t slot = base + (int64_t)j * kS + ln;
            coupled = A.col[slot] != (int32_t)i && A.val[slot] != 0.f;
        }
    }
    mate[i] = coupled ? kUnmatched : kExcluded;
}

// agg = -1 for rows without a non-zero off-diagonal (solved exactly by the smoother), else 0
__global__ void k_mark_isolated(MatView A, int32_t *agg) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    int64_t base;
    int w, ln;
    row_of(A, i, base, w, ln);
    bool coupled = false;
    for (int j = 0; j < w && !coupled; ++j) {
        const int64_t slot = base + (int64_t)j * kS + ln;
        coupled = A.col[slot] != (int32_t)i && A.val[slot] != 0.f;
    }
    agg[i] = coupled ? 0 : -1;
}

// Strongest negative coupling -a_ij / sqrt(a_ii a_jj) to a still unmatched row (ties: lower j).
// With mix, a row may also pair along a positive coupling, weighted 1e-3 so that any negative
// coupling is preferred (coarse Galerkin matrices, and unsteady systems, carry many positive
// off-diagonals; pairing only along negative ones stalls the coarsening there).
// The choice is the largest weight, and among equal weights the lowest column: it does not
// depend on the order the slots are visited in, so the G warps of a slice (split_row) combine
// their partial choices to the same row.
__device__ __forceinline__ bool better(float s, int32_t c, float bw, int32_t best) {
    return c >= 0 && (s > bw || (s == bw && best >= 0 && c < best));
}

template <int G>
__global__ void __launch_bounds__(256) k_pair_want(MatView A, const float *isd, const int32_t *mate, int32_t *want,
                                                   int mix) {
    int64_t i;
    int g;
    split_row<G>(i, g);
    int32_t best = -1;
    float bw = 0.f;
    if (i < A.n && mate[i] == kUnmatched && !is_long(A, i)) {  // a hub row stays an aggregate of its own
        int64_t base;
        int w, ln;
        row_of(A, i, base, w, ln);
        const float si = isd[i];
        constexpr int kB = 8;
        for (int j0 = g; j0 < w; j0 += kB * G) {
            int32_t c[kB];
            float v[kB];
#pragma unroll
            for (int k = 0; k < kB; ++k) {
                const int j = j0 + k * G;
                const int64_t slot = base + (int64_t)j * kS + ln;
                c[k] = j < w ? __ldg(A.col + slot) : (int32_t)i;
                v[k] = j < w ? __ldg(A.val + slot) : 0.f;
            }
            int32_t mt[kB];
            float sc[kB];
#pragma unroll
            for (int k = 0; k < kB; ++k) {
                const bool cand = c[k] != (int32_t)i && v[k] != 0.f && (mix || v[k] < 0.f);
                mt[k] = cand ? mate[c[k]] : kExcluded;
                sc[k] = cand ? isd[c[k]] : 0.f;
            }
#pragma unroll
            for (int k = 0; k < kB; ++k) {
                if (mt[k] != kUnmatched) continue;
                const float s = (v[k] < 0.f ? -v[k] : 1e-3f * v[k]) * si * sc[k];
                if (better(s, c[k], bw, best)) {
                    bw = s;
                    best = c[k];
                }
            }
        }
    }
    if constexpr (G > 1) {
        __shared__ float pw[8][32];
        __shared__ int32_t pc[8][32];
        const int wb = threadIdx.x >> 5, lane = threadIdx.x & 31;
        pw[wb][lane] = bw;
        pc[wb][lane] = best;
        __syncthreads();
        if (wb % G != 0) return;
#pragma unroll
        for (int k = 1; k < G; ++k)
            if (better(pw[wb + k][lane], pc[wb + k][lane], bw, best)) {
                bw = pw[wb + k][lane];
                best = pc[wb + k][lane];
            }
    }
    if (i < A.n) want[i] = best;
}

// Handshake: i and j pair when each is the other's choice; a row with no candidate is final.
__global__ void k_pair_match(int64_t n, const int32_t *want, int32_t *mate) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || mate[i] != kUnmatched) return;
    const int32_t j = want[i];
    if (j < 0) mate[i] = kSingle;
    else if (want[j] == (int32_t)i) mate[i] = j;
}

// Leader of each aggregate (a single row, or the lower row of a pair), packed for one scan:
// low 32 bits 1 for a leader, high 32 bits the aggregate's member count.  The exclusive scan
// then gives every leader its aggregate id (low) and member offset (high).
__global__ void k_pair_pack(int64_t n, const int32_t *mate, int64_t *packed) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t m = mate[i];
    const bool lead = m == kSingle || m == kUnmatched || (m >= 0 && (int32_t)i < m);
    packed[i] = lead ? (int64_t)1 | ((int64_t)(m >= 0 ? 2 : 1) << 32) : 0;
}

// agg of every row, and the member lists (leader first, then its pair)
__global__ void k_pair_finish(int64_t n, int64_t nc, int64_t members, const int32_t *mate, const int64_t *packed,
                              const int64_t *pscan, int32_t *agg, int32_t *mstart, int32_t *mrows) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) mstart[nc] = (int32_t)members;
    if (i >= n) return;
    const int32_t m = mate[i];
    if (packed[i] & 1) {
        const int64_t pre = pscan[i];
        const int32_t cid = (int32_t)(pre & 0xffffffff), off = (int32_t)(pre >> 32);
        agg[i] = cid;
        mstart[cid] = off;
        mrows[off] = (int32_t)i;
        if (m >= 0) mrows[off + 1] = m;
    } else {
        agg[i] = m >= 0 ? (int32_t)(pscan[m] & 0xffffffff) : -1;
    }
}

// Two pairing passes composed: agg = agg2[agg1[i]], members of each final row in order.
__global__ void k_compose_agg(int64_t n, const int32_t *agg1, const int32_t *agg2, int32_t *agg) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t a = agg1[i];
    agg[i] = a >= 0 ? agg2[a] : -1;
}

__global__ void k_compose_count(int64_t nc, const int32_t *ms2, const int32_t *mr2, const int32_t *ms1, int32_t *cnt) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    int32_t k = 0;
    for (int32_t q = ms2[c]; q < ms2[c + 1]; ++q) k += ms1[mr2[q] + 1] - ms1[mr2[q]];
    cnt[c] = k;
}

__global__ void k_compose_fill(int64_t nc, const int32_t *ms2, const int32_t *mr2, const int32_t *ms1,
                               const int32_t *mr1, const int32_t *ms, int32_t *mr) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    int32_t p = ms[c];
    for (int32_t q = ms2[c]; q < ms2[c + 1]; ++q)
        for (int32_t t = ms1[mr2[q]]; t < ms1[mr2[q] + 1]; ++t) mr[p++] = mr1[t];
}

// ---- Galerkin product A_c = P^T A P, one warp per coarse row -------------------------------
// Gathers (agg[col], val) of the coarse row's rows, sorts by coarse column (bitonic, in
// shared memory), and sums equal columns in sorted order (FP64 sums: deterministic).
// Pass 1 (WRITE = false) stores the row lengths; pass 2 writes the SELL slots, padding with
// (own row, 0).
// Each coarse row is gathered, sorted and reduced once; its entries go to a compact buffer at
// t_off[I] (sized by the candidate bound) and its length to rowlen[I]; k_sell_fill then lays
// the rows out as SELL.  Rows run in two tiers: every row first with the small static buffer
// (LIST = false); a row whose candidates do not fit is appended to a list, and the list then
// runs with a large dynamic buffer (LIST = true, one warp per block).  A row too wide even for
// that sets *overflow.
// Rows of at most S candidates (S = 16 or 32), one row per S-lane segment of the warp and one
// candidate per lane (key INT_MAX: none; cnt real ones in the segment; I < 0: no row).
// seg_gather loads lane t's candidate (the rows of the coarse row in member order, then their
// slots) with all the row's loads in flight at once; seg_reduce sorts the segment by coarse
// column (bitonic network in registers), sums equal columns in sorted order in FP64, and writes
// the row at t_off = ob and its length to rowlen[I].
template <int S>
__device__ __forceinline__ void seg_gather(const MatView &A, const int32_t *__restrict__ agg,
                                           const int32_t *__restrict__ mrows, const float *__restrict__ wt,
                                           int32_t m0, int32_t nm, int32_t &key, float &v) {
    const int sl = threadIdx.x & (S - 1);
    int64_t mb = 0;
    int mw = 0, mln = 0;
    float mwt = 1.f;
    if (sl < nm) {
        const int32_t mi = mrows[m0 + sl];
        row_of(A, mi, mb, mw, mln);
        if (wt) mwt = wt[mi];
    }
    int incl = mw;
#pragma unroll
    for (int o = 1; o < S; o <<= 1) {
        const int y = __shfl_up_sync(kFull, incl, o, S);
        if (sl >= o) incl += y;
    }
    const int excl = incl - mw, total = __shfl_sync(kFull, incl, S - 1, S);
    const int nmax = __reduce_max_sync(kFull, (unsigned)nm);
    int mem = 0;  // the last member starting at or before this lane
    for (int k = 1; k < nmax; ++k) {
        const int e = __shfl_sync(kFull, excl, k, S);
        if (k < nm && e <= sl) mem = k;
    }
    const int64_t b = __shfl_sync(kFull, mb, mem, S);
    const int lnm = __shfl_sync(kFull, mln, mem, S), e0 = __shfl_sync(kFull, excl, mem, S);
    const float wi = __shfl_sync(kFull, mwt, mem, S);
    key = INT_MAX;
    v = 0.f;
    if (sl < total) {
        const int64_t slot = b + (int64_t)(sl - e0) * kS + lnm;
        const float a = A.val[slot];
        if (a != 0.f) {
            const int32_t c = A.col[slot];
            const int32_t ac = agg[c];
            if (ac >= 0) {
                key = ac;
                v = wt ? a * wi * wt[c] : a;
            }
        }
    }
}

template <int S>
__device__ __forceinline__ void seg_reduce(int32_t key, float val, int cnt, int64_t ob, int64_t I,
                                           int32_t *__restrict__ t_col, float *__restrict__ t_val,
                                           int32_t *__restrict__ rowlen) {
    const int lane = threadIdx.x & 31, sl = lane & (S - 1);
#pragma unroll
    for (int k = 2; k <= S; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const int32_t pk = __shfl_xor_sync(kFull, key, j);
            const float pv = __shfl_xor_sync(kFull, val, j);
            const bool up = (sl & k) == 0, lower = (sl & j) == 0;
            // the pair (lower, upper) swaps when its keys are out of order (strictly)
            const bool swap = lower ? (up ? key > pk : key < pk) : (up ? pk > key : pk < key);
            if (swap) {
                key = pk;
                val = pv;
            }
        }
    const int32_t prev = __shfl_up_sync(kFull, key, 1);
    const bool head = sl < cnt && (sl == 0 || key != prev);
    const unsigned hall = __ballot_sync(kFull, head);
    const unsigned hm = S == 32 ? hall : (hall >> (lane & ~(S - 1))) & ((1u << (S & 31)) - 1u);
    double sum = (double)val;
    bool open = head;
    for (int dlt = 1; dlt < S; ++dlt) {
        const int32_t kd = __shfl_down_sync(kFull, key, dlt);
        const float vd = __shfl_down_sync(kFull, val, dlt);
        if (open) {
            if (sl + dlt < cnt && kd == key) sum += (double)vd;
            else open = false;
        }
        if (!__any_sync(kFull, open)) break;
    }
    if (head) {
        const int outk = __popc(hm & ((1u << sl) - 1u));
        t_col[ob + outk] = key;
        t_val[ob + outk] = (float)sum;
    }
    if (sl == 0 && I >= 0) rowlen[I] = __popc(hm);
}

template <int kGalCap, int kGalWarps, bool LIST>
__global__ void __launch_bounds__(kGalWarps * 32)
    k_galerkin(MatView A, const int32_t *__restrict__ agg, const int32_t *__restrict__ mstart,
               const int32_t *__restrict__ mrows, int64_t nc, int32_t *__restrict__ rowlen,
               const int64_t *__restrict__ t_off, int32_t *__restrict__ t_col, float *__restrict__ t_val,
               int32_t *overflow, const float *__restrict__ wt, int32_t *__restrict__ big_list,
               int32_t *big_count) {
    __shared__ int32_t s_k[LIST ? 1 : kGalWarps][LIST ? 1 : kGalCap];
    __shared__ float s_v[LIST ? 1 : kGalWarps][LIST ? 1 : kGalCap];
    extern __shared__ unsigned char dyn_sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int32_t *K = LIST ? reinterpret_cast<int32_t *>(dyn_sm) + (size_t)warp * kGalCap : s_k[warp];
    float *V = LIST ? reinterpret_cast<float *>(dyn_sm) + (size_t)(kGalWarps + warp) * kGalCap : s_v[warp];
    const unsigned lt = (1u << lane) - 1u;
    const int64_t n_iter = LIST ? *big_count : nc;
    constexpr int R = LIST ? 1 : 2;  // rows per warp and iteration
    for (int64_t it = ((int64_t)blockIdx.x * kGalWarps + warp) * R; it < n_iter;
         it += (int64_t)gridDim.x * kGalWarps * R) {
        if (!LIST) {
            // two rows of at most 16 candidates (the summed widths of their rows): one per
            // half-warp, lane t of a half taking candidate t of its row
            const int half = lane >> 4;
            const int64_t Ih = it + half < n_iter ? it + half : -1;
            int64_t obh = 0;
            int32_t m0h = 0, nmh = 0;
            bool fit = true;
            if (Ih >= 0) {
                obh = t_off[Ih];
                m0h = mstart[Ih];
                nmh = mstart[Ih + 1] - m0h;
                fit = t_off[Ih + 1] - obh <= 16 && nmh <= 16;
            }
            if (__all_sync(kFull, fit)) {
                int32_t key;
                float v;
                seg_gather<16>(A, agg, mrows, wt, m0h, nmh, key, v);
                const unsigned bal = __ballot_sync(kFull, key != INT_MAX);
                seg_reduce<16>(key, v, __popc(half ? bal >> 16 : bal & 0xffffu), obh, Ih, t_col, t_val, rowlen);
                __syncwarp();
                continue;
            }
        }
        for (int q = 0; q < R; ++q) {
            const int64_t I = LIST ? big_list[it] : it + q;
            if (I >= (LIST ? INT64_MAX : nc)) break;
            const int64_t ob = t_off[I];
            if (!LIST) {
                // at most 32 candidates: one row per warp, lane t taking candidate t
                const int32_t m0 = mstart[I], nm = mstart[I + 1] - m0;
                if (t_off[I + 1] - ob <= 32 && nm <= 32) {
                    int32_t key;
                    float v;
                    seg_gather<32>(A, agg, mrows, wt, m0, nm, key, v);
                    seg_reduce<32>(key, v, __popc(__ballot_sync(kFull, key != INT_MAX)), ob, I, t_col, t_val, rowlen);
                    __syncwarp();
                    continue;
                }
            }
            int cnt = 0;
            for (int32_t m = mstart[I]; m < mstart[I + 1]; ++m) {
                int64_t base;
                int w, ln;
                const int32_t mi = mrows[m];
                row_of(A, mi, base, w, ln);
                const float wi = wt ? wt[mi] : 1.f;
                for (int j0 = 0; j0 < w; j0 += 32) {
                    const int j = j0 + lane;
                    int32_t key = -1;
                    float v = 0.f;
                    if (j < w) {
                        const int64_t slot = base + (int64_t)j * kS + ln;
                        v = A.val[slot];
                        if (v != 0.f) {
                            const int32_t c = A.col[slot];
                            key = agg[c];
                            if (wt) v = v * wi * wt[c];
                        }
                    }
                    const unsigned mask = __ballot_sync(kFull, key >= 0);
                    const int pos = cnt + __popc(mask & lt);
                    if (key >= 0 && pos < kGalCap) {
                        K[pos] = key;
                        V[pos] = v;
                    }
                    cnt += __popc(mask);
                }
            }
            if (cnt > kGalCap) {
                if (lane == 0) {
                    if (LIST) atomicExch(overflow, 1);
                    else big_list[atomicAdd(big_count, 1)] = (int32_t)I;
                    rowlen[I] = 0;
                }
                __syncwarp();
                continue;
            }
            if (cnt <= 32) {  // one candidate per lane: the register network
                __syncwarp();
                const int32_t key = lane < cnt ? K[lane] : INT_MAX;
                const float val = lane < cnt ? V[lane] : 0.f;
                __syncwarp();
                seg_reduce<32>(key, val, cnt, ob, I, t_col, t_val, rowlen);
                __syncwarp();
                continue;
            }
            int cp = 32;
            while (cp < cnt) cp <<= 1;
            for (int k = cnt + lane; k < cp; k += 32) {
                K[k] = INT_MAX;
                V[k] = 0.f;
            }
            __syncwarp();
            for (int k = 2; k <= cp; k <<= 1)
                for (int j = k >> 1; j > 0; j >>= 1) {
                    for (int t = lane; t < cp; t += 32) {
                        const int u = t ^ j;
                        if (u > t) {
                            const int32_t a = K[t], b = K[u];
                            const bool up = (t & k) == 0;
                            if (up ? (a > b) : (a < b)) {
                                K[t] = b;
                                K[u] = a;
                                const float x = V[t];
                                V[t] = V[u];
                                V[u] = x;
                            }
                        }
                    }
                    __syncwarp();
                }
            int uniq = 0;
            for (int t0 = 0; t0 < cnt; t0 += 32) {
                const int t = t0 + lane;
                const bool head = t < cnt && (t == 0 || K[t] != K[t - 1]);
                const unsigned hm = __ballot_sync(kFull, head);
                if (head) {
                    const int outk = uniq + __popc(hm & lt);
                    const int32_t key = K[t];
                    double s = 0.0;
                    for (int q = t; q < cnt && K[q] == key; ++q) s += (double)V[q];
                    t_col[ob + outk] = key;
                    t_val[ob + outk] = (float)s;
                }
                uniq += __popc(hm);
            }
            if (lane == 0) rowlen[I] = uniq;
            __syncwarp();
        }
    }
}

// Candidate bound of each coarse row: the summed lengths of its rows
__global__ void k_cand_bound(MatView A, const int32_t *__restrict__ mstart, const int32_t *__restrict__ mrows,
                             int64_t nc, int64_t *__restrict__ bound) {
    const int64_t I = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= nc) return;
    int64_t b = 0;
    for (int32_t m = mstart[I]; m < mstart[I + 1]; ++m) {
        int64_t base;
        int w, ln;
        row_of(A, mrows[m], base, w, ln);
        b += w;
    }
    bound[I] = b;
}

// SELL layout of the compact rows: entries, then padding slots (own column, value 0)
__global__ void k_sell_fill(int64_t n_pad, int64_t nc, const int64_t *__restrict__ c_off,
                            const int32_t *__restrict__ rowlen, const int64_t *__restrict__ t_off,
                            const int32_t *__restrict__ t_col, const float *__restrict__ t_val,
                            int32_t *__restrict__ c_col, float *__restrict__ c_val) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pad) return;
    const int64_t sl = i / kS;
    const int ln = (int)(i - sl * kS);
    const int w = (int)((c_off[sl + 1] - c_off[sl]) / kS);
    const int len = i < nc ? rowlen[i] : 0;
    const int64_t src = i < nc ? t_off[i] : 0;
    for (int k = 0; k < w; ++k) {
        const int64_t slot = c_off[sl] + (int64_t)k * kS + ln;
        if (k < len) {
            c_col[slot] = t_col[src + k];
            c_val[slot] = t_val[src + k];
        } else {
            c_col[slot] = (int32_t)i;
            c_val[slot] = 0.f;
        }
    }
}

// slots of each slice: 32 x the longest row among its real rows
__global__ void k_slice_width(int64_t n_slices, int64_t nc, const int32_t *rowlen, int64_t *width) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_slices) return;
    int32_t m = 0;
    for (int k = 0; k < kS; ++k) {
        const int64_t i = s * kS + k;
        if (i < nc) m = max(m, rowlen[i]);
    }
    width[s] = (int64_t)m * kS;
}


// ---- dense coarsest level ----------------------------------------------------------------
// In-place Gauss-Jordan inversion in shared memory (FP64, no pivoting: the matrix is SPD), one
// block of 1024 threads, n <= kDenseMax.  The first n rows of the SELL matrix are gathered
// into shared memory, inverted, and written out as FP32.  flag = 1 on a non-positive or
// non-finite pivot.
constexpr int kDenseMax = 160;  // n^2 doubles + n factors fit in 227 KB of shared memory

__global__ void __launch_bounds__(1024) k_dense_inverse(MatView A, int n, float *inv, int32_t *flag) {
    extern __shared__ double sm[];
    double *M = sm, *fac = sm + n * n;
    __shared__ double pinv;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // launched with 1024 threads
    for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) M[idx] = 0.0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        int64_t base;
        int w, ln;
        row_of(A, i, base, w, ln);
        for (int j = 0; j < w; ++j) {
            const int64_t slot = base + (int64_t)j * kS + ln;
            const int32_t c = A.col[slot];
            if (c < n) M[i * n + c] += (double)A.val[slot];
        }
    }
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        if (threadIdx.x == 0) {
            const double p = M[k * n + k];
            const bool ok = p > 0.0 && isfinite(p);
            if (!ok) *flag = 1;
            pinv = ok ? 1.0 / p : 0.0;
        }
        for (int i = threadIdx.x; i < n; i += blockDim.x) fac[i] = M[i * n + k];
        __syncthreads();
        // row k: a_kj / p, with a_kk := 1 / p
        for (int j = threadIdx.x; j < n; j += blockDim.x) M[k * n + j] = (j == k ? 1.0 : M[k * n + j]) * pinv;
        __syncthreads();
        // rows i != k: a_ij -= f_i a_kj, with a_ik := -f_i / p (32 x 32 threads: lanes take
        // consecutive columns, warps rows; a_kj is loaded once per column, f_i is a broadcast)
        for (int j = tx; j < n; j += 32) {
            const double akj = M[k * n + j];
            const bool jk = j == k;
            for (int i = ty; i < n; i += 32) {
                if (i == k) continue;
                const double base = jk ? 0.0 : M[i * n + j];
                M[i * n + j] = base - fac[i] * akj;
            }
        }
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) inv[idx] = (float)M[idx];
}

// x[i] = sum_j inv[i][j] b[j] for i < n (one warp per row); rows n..n_pad-1 get 0
__global__ void k_dense_gemv(Gate gate, const float *__restrict__ inv, int64_t n, int64_t n_pad, const float *__restrict__ b,
                             float *__restrict__ x) {
    if (closed(gate)) return;
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= n_pad) return;
    float s = 0.f;
    if (i < n)
        for (int64_t j = lane; j < n; j += 32) s += inv[i * n + j] * b[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
    if (lane == 0) x[i] = s;
}

// ---- V-cycle kernels ------------------------------------------------------------------------
// (A x)_i.  On the fine level (no row lengths: 7-8 entries per row) the first 8 slots are
// loaded together, then gathered together, so each thread keeps 8 independent loads in flight
// instead of one dependent load chain per slot; coarse rows (longer, irregular) loop.
// the fine level's row: slots loaded 8 at a time, values from FP32 or their FP16 copy
template <bool HALF>
// The slots are a stream read once per pass: loaded evict-first (ld.global.cs) so that they
// do not push the gathered vector out of L2.
__device__ __forceinline__ float fine_dot(const MatView &A, int64_t base, int w, int ln, const float *__restrict__ x) {
    auto value = [&](int64_t slot) { return HALF ? __half2float(__ldcs(A.hval + slot)) : __ldcs(A.val + slot); };
    constexpr int kB = 8;
    int32_t c[kB];
    float v[kB];
#pragma unroll
    for (int k = 0; k < kB; ++k) {
        const int64_t slot = base + (int64_t)k * kS + ln;
        c[k] = k < w ? __ldcs(A.col + slot) : 0;
        v[k] = k < w ? value(slot) : 0.f;
    }
    float g[kB];
#pragma unroll
    for (int k = 0; k < kB; ++k) g[k] = k < w ? x[c[k]] : 0.f;
    float y = 0.f;
#pragma unroll
    for (int k = 0; k < kB; ++k) y += v[k] * g[k];
    for (int j = kB; j < w; ++j) {
        const int64_t slot = base + (int64_t)j * kS + ln;
        y += value(slot) * x[__ldcs(A.col + slot)];
    }
    return y;
}

__device__ __forceinline__ float row_dot(const MatView &A, int64_t i, const float *__restrict__ x) {
    int64_t base;
    int w, ln;
    row_of(A, i, base, w, ln);
    if (A.rlen) {
        float y = 0.f;
        for (int j = 0; j < w; ++j) {
            const int64_t slot = base + (int64_t)j * kS + ln;
            y += __ldg(A.val + slot) * x[__ldg(A.col + slot)];
        }
        return y;
    }
    return A.hval ? fine_dot<true>(A, base, w, ln, x) : fine_dot<false>(A, base, w, ln, x);
}

// Coarse rows are long (tens of entries), so one thread walking a row issues a long chain of
// dependent loads and the small coarse levels run at load latency.  The row kernels therefore
// take G warps per 32-row slice (G = AmgLevel::g, chosen from the level's mean slice width):
// warp g of a slice's group takes the slots g, g + G, g + 2G, ... of its 32 rows, eight loaded
// together, and the G partial sums meet in shared memory in warp order (deterministic).  Blocks
// hold 8 warps, i.e. 8 / G slices.  G = 1 is one thread per row (row_dot).
template <int G>
__device__ __forceinline__ float split_part(const MatView &A, int64_t i, int g, const float *__restrict__ x) {
    if (G == 1) return row_dot(A, i, x);
    int64_t base;
    int w, ln;
    row_of(A, i, base, w, ln);
    constexpr int kB = 8;
    float y = 0.f;
    for (int j0 = g; j0 < w; j0 += kB * G) {
        int32_t c[kB];
        float v[kB];
#pragma unroll
        for (int k = 0; k < kB; ++k) {
            const int j = j0 + k * G;
            const int64_t slot = base + (int64_t)j * kS + ln;
            c[k] = j < w ? __ldg(A.col + slot) : 0;
            v[k] = j < w ? __ldg(A.val + slot) : 0.f;
        }
        float gx[kB];
#pragma unroll
        for (int k = 0; k < kB; ++k) gx[k] = j0 + k * G < w ? x[c[k]] : 0.f;
#pragma unroll
        for (int k = 0; k < kB; ++k) y += v[k] * gx[k];
    }
    return y;
}

// the row's sum of the G partials (valid in the group's warp g = 0); every thread of the block
// calls it
template <int G> __device__ __forceinline__ float split_sum(float y) {
    if constexpr (G == 1) {
        return y;
    } else {
        __shared__ float part[8][32];
        const int wb = threadIdx.x >> 5, lane = threadIdx.x & 31;
        part[wb][lane] = y;
        __syncthreads();
        float t = 0.f;
        if (wb % G == 0)
#pragma unroll
            for (int k = 0; k < G; ++k) t += part[wb + k][lane];
        return t;
    }
}

// first Chebyshev step from x = 0: d = c2 D^-1 b, x = d
// (invd null: unit diagonal, the Jacobi-scaled fine level)
__global__ void k_sm_first(Gate gate, int64_t n, const float *__restrict__ b, const float *__restrict__ invd, float c2,
                           float *__restrict__ x, float *__restrict__ d, const int32_t *__restrict__ agg) {
    if (closed(gate)) return;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float di = invd ? invd[i] : 1.f;
    if (agg && agg[i] < 0) {  // a row outside the hierarchy: exact
        d[i] = 0.f;
        x[i] = di * b[i];
        return;
    }
    const float v = c2 * di * b[i];
    d[i] = v;
    x[i] = v;
}

// restriction fused with the first smoothing step of the coarse level:
// b_c[I] = sum over the rows of I of w r, then x = d = c2 D_c^-1 b_c
__global__ void k_restrict_first(Gate gate, int64_t nc, int64_t nc_pad, const int32_t *__restrict__ ms,
                                 const int32_t *__restrict__ mr, const float *__restrict__ r,
                                 const float *__restrict__ wt, const float *__restrict__ invd_c, float c2,
                                 float *__restrict__ bc, float *__restrict__ x, float *__restrict__ d,
                                 const int32_t *__restrict__ agg_c) {
    if (closed(gate)) return;
    const int64_t I = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= nc_pad) return;
    float s = 0.f;
    if (I < nc)
        for (int32_t k = ms[I]; k < ms[I + 1]; ++k) s += (wt ? wt[mr[k]] : 1.f) * r[mr[k]];
    bc[I] = s;
    const bool exact = agg_c[I] < 0;
    const float v = (exact ? 1.f : c2) * invd_c[I] * s;
    d[I] = exact ? 0.f : v;
    x[I] = v;
}

// Chebyshev step: d = c1 d + c2 D^-1 (b - A x_in), x_out = x_in + d (c1 = 0: d is not read)
template <int G>
__global__ void __launch_bounds__(256) k_sm_step(Gate gate, MatView A, const float *__restrict__ b,
                                                 const float *__restrict__ invd, const float *__restrict__ x_in,
                                                 float *__restrict__ x_out, float *__restrict__ d, float c1, float c2,
                                                 const int32_t *__restrict__ agg) {
    if (closed(gate)) return;
    int64_t i;
    int g;
    split_row<G>(i, g);
    const bool outside = i < A.n && agg && agg[i] < 0;
    const bool live = i < A.n && !outside && !is_long(A, i);  // long rows: k_long_rows
    const float y = split_sum<G>(live ? split_part<G>(A, i, g, x_in) : 0.f);
    if (g != 0 || i >= A.n) return;
    const float di = invd ? invd[i] : 1.f;
    if (outside) {  // a row outside the hierarchy: exact
        d[i] = 0.f;
        x_out[i] = di * b[i];
        return;
    }
    if (!live) return;
    const float r = b[i] - y;
    const float dn = (c1 != 0.f ? c1 * d[i] : 0.f) + c2 * di * r;
    d[i] = dn;
    x_out[i] = x_in[i] + dn;
}

// The fine level's first two Chebyshev steps from x = 0 in one pass (unit diagonal):
// x1 = c0 b (so A x1 = c0 A b), d = c1 c0 b + c2 (b - c0 A b), x_out = x1 + d
__global__ void k_sm_first_step(Gate gate, MatView A, const float *__restrict__ b, float *__restrict__ x_out,
                                float *__restrict__ d, float c0, float c1, float c2, const int32_t *__restrict__ agg) {
    if (closed(gate)) return;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    const float bi = b[i];
    if (agg && agg[i] < 0) {  // a row outside the hierarchy: exact
        d[i] = 0.f;
        x_out[i] = bi;
        return;
    }
    const float x1 = c0 * bi;
    const float r = bi - c0 * row_dot(A, i, b);
    const float dn = c1 * x1 + c2 * r;
    d[i] = dn;
    x_out[i] = x1 + dn;
}

// The same with smoother weights w (Omega S^): x1 = c0 w b, d = c1 x1 + c2 w (b - S^ x1); the
// product S^ (w b) gathers w and b together
__global__ void k_sm_first_step_w(Gate gate, MatView A, const float *__restrict__ b, const float *__restrict__ w,
                                  float *__restrict__ x_out, float *__restrict__ d, float c0, float c1, float c2,
                                  const int32_t *__restrict__ agg) {
    if (closed(gate)) return;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    const float bi = b[i];
    if (agg && agg[i] < 0) {  // a row outside the hierarchy: exact
        d[i] = 0.f;
        x_out[i] = bi;
        return;
    }
    int64_t base;
    int wd, ln;
    row_of(A, i, base, wd, ln);
    float y = 0.f;
    for (int j = 0; j < wd; ++j) {
        const int64_t slot = base + (int64_t)j * kS + ln;
        const int32_t c = __ldg(A.col + slot);
        const float v = A.hval ? __half2float(A.hval[slot]) : __ldg(A.val + slot);
        y += v * (w[c] * b[c]);
    }
    const float wi = w[i];
    const float x1 = c0 * wi * bi;
    const float dn = c1 * x1 + c2 * wi * (bi - c0 * y);
    d[i] = dn;
    x_out[i] = x1 + dn;
}

template <int G>
__global__ void __launch_bounds__(256) k_residual(Gate gate, MatView A, const float *__restrict__ b,
                                                  const float *__restrict__ x, float *__restrict__ r) {
    if (closed(gate)) return;
    int64_t i;
    int g;
    split_row<G>(i, g);
    const bool live = i < A.n && !is_long(A, i);  // long rows: k_long_rows
    const float y = split_sum<G>(live ? split_part<G>(A, i, g, x) : 0.f);
    if (g == 0 && live) r[i] = b[i] - y;
}

// b_c[I] = sum of r over the rows of coarse row I (in member order); padding rows get 0
__global__ void k_restrict(Gate gate, int64_t nc, int64_t nc_pad, const int32_t *__restrict__ ms, const int32_t *__restrict__ mr,
                           const float *__restrict__ r, float *__restrict__ bc, const float *__restrict__ wt) {
    if (closed(gate)) return;
    const int64_t I = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= nc_pad) return;
    float s = 0.f;
    if (I < nc)
        for (int32_t k = ms[I]; k < ms[I + 1]; ++k) s += (wt ? wt[mr[k]] : 1.f) * r[mr[k]];
    bc[I] = s;
}

__global__ void k_to_half(int64_t n, const float *__restrict__ a, uint16_t *__restrict__ h) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) h[i] = __half_as_ushort(__float2half_rn(a[i]));
}

__global__ void k_to_float(int64_t n, const double *__restrict__ a, float *__restrict__ b) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}

// x += alpha P x_c (alpha from the device scalar when given, else the constant)
__global__ void k_prolong(Gate gate, int64_t n, const int32_t *__restrict__ agg, const float *__restrict__ xc,
                          float *__restrict__ x, const double *__restrict__ alpha_dev, float alpha,
                          const float *__restrict__ wt) {
    if (closed(gate)) return;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t a = agg[i];
    const float al = alpha_dev ? (float)*alpha_dev : alpha;
    if (a >= 0) x[i] += al * (wt ? wt[i] : 1.f) * xc[a];
}

// One block per long row (kLongRow): y = (A x)_i by a block reduction, then the epilogue of
// the thread-per-row kernel it stands in for.  MODE 0: Chebyshev step (k_sm_step), 1: residual
// (k_residual), 2: the row's terms x_i b_i and x_i (A x)_i of the coarse-correction scaling
// (k_coarse_dots), written to long_part[2k], [2k+1], 3: power step D^-1 A x (k_power_step).
template <int MODE>
__global__ void __launch_bounds__(256) k_long_rows(Gate gate, MatView A, const int32_t *__restrict__ rows,
                                                   const float *__restrict__ b, const float *__restrict__ invd,
                                                   const float *__restrict__ x_in, float *__restrict__ out,
                                                   float *__restrict__ d, float c1, float c2,
                                                   double *__restrict__ long_part) {
    if (closed(gate)) return;
    const int64_t i = rows[blockIdx.x];
    int64_t base;
    int w, ln;
    row_of(A, i, base, w, ln);
    float y = 0.f;
    for (int j = threadIdx.x; j < w; j += blockDim.x) {
        const int64_t slot = base + (int64_t)j * kS + ln;
        y += __ldg(A.val + slot) * x_in[__ldg(A.col + slot)];
    }
    __shared__ float red[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) y += __shfl_xor_sync(kFull, y, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = y;
    __syncthreads();
    if (threadIdx.x != 0) return;
    y = 0.f;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) y += red[k];
    if (MODE == 0) {
        const float di = invd ? invd[i] : 1.f;
        const float dn = (c1 != 0.f ? c1 * d[i] : 0.f) + c2 * di * (b[i] - y);
        d[i] = dn;
        out[i] = x_in[i] + dn;
    } else if (MODE == 1) {
        out[i] = b[i] - y;
    } else if (MODE == 3) {
        out[i] = invd ? invd[i] * y : y;
    } else {
        long_part[2 * blockIdx.x] = (double)x_in[i] * (double)b[i];
        long_part[2 * blockIdx.x + 1] = (double)x_in[i] * (double)y;
    }
}

// long-row list: flags (1 where rlen > kLongRow) for a scan, then the compacted row indices
__global__ void k_flag_long(int64_t n, const int32_t *rlen, int32_t *flag) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flag[i] = rlen[i] > kLongRow ? 1 : 0;
}
__global__ void k_compact_long(int64_t n, const int32_t *flag, const int32_t *pos, int32_t *list) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) list[0] = pos[n];
    if (i < n && flag[i]) list[1 + pos[i]] = (int32_t)i;
}

// Energy-optimal scaling of a coarse correction: per block partials of x_c.b_c and
// x_c.(A_c x_c) (the fine-level quantities e.r and e.Ae for e = P x_c).
template <int G>
__global__ void __launch_bounds__(256) k_coarse_dots(Gate gate, MatView A, const float *__restrict__ x,
                                                     const float *__restrict__ b, double *__restrict__ part,
                                                     unsigned int *ticket, double *alpha,
                                                     const double *__restrict__ long_part, int32_t n_long) {
    if (closed(gate)) return;
    int64_t i;
    int g;
    split_row<G>(i, g);
    const bool live = i < A.n && !is_long(A, i);  // long rows' terms come from k_long_rows in long_part
    const float y = split_sum<G>(live ? split_part<G>(A, i, g, x) : 0.f);
    double xb = 0.0, xax = 0.0;
    if (g == 0 && live) {
        const double xi = (double)x[i];
        xb = xi * (double)b[i];
        xax = xi * (double)y;
    }
    __shared__ double sh[2][8];
    __shared__ bool am_last;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        xb += __shfl_xor_sync(kFull, xb, o);
        xax += __shfl_xor_sync(kFull, xax, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][warp] = xb;
        sh[1][warp] = xax;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, c = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            a += sh[0][w];
            c += sh[1][w];
        }
        part[2 * blockIdx.x] = a;
        part[2 * blockIdx.x + 1] = c;
        __threadfence();
        am_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!am_last) return;
    // the last block: alpha from the partials in block order (deterministic)
    __threadfence();
    __shared__ double red[2][256];
    double a = 0.0, c = 0.0;
    for (int64_t k = threadIdx.x; k < gridDim.x; k += blockDim.x) {
        a += __ldcg(part + 2 * k);
        c += __ldcg(part + 2 * k + 1);
    }
    for (int k = threadIdx.x; k < n_long; k += blockDim.x) {
        a += __ldcg(long_part + 2 * k);
        c += __ldcg(long_part + 2 * k + 1);
    }
    red[0][threadIdx.x] = a;
    red[1][threadIdx.x] = c;
    __syncthreads();
    for (int st = 128; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) {
            red[0][threadIdx.x] += red[0][threadIdx.x + st];
            red[1][threadIdx.x] += red[1][threadIdx.x + st];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double num = red[0][0], den = red[1][0];
        *alpha = (den > 0.0 && num > 0.0 && isfinite(num / den)) ? num / den : 1.0;
        *ticket = 0u;
    }
}

// ---- fine-level smoothing with the matrix streamed by TMA bulk copies ----------------------
// The fine level's row kernels are one long stream of SELL slots (column index and FP16 value,
// 6 bytes a slot) plus gathers of x[col] that mostly hit L2.  In the thread-per-row kernels each
// warp waits for its slots from DRAM before it can issue its gathers, and the kernel runs at
// load latency (about 0.6 of the copy bandwidth).  Here a CTA streams tiles of 8 slices
// (256 rows) through a ring of NST shared-memory stages with 1D bulk copies (cp.async.bulk,
// completion counted on an mbarrier), so the DRAM stream runs NST - 1 tiles ahead of the warps,
// which read their slots from shared memory and only wait on the gathers.  The row arithmetic
// and its summation order are those of k_sm_first_step, k_sm_step<1> and k_residual<1>
// (bit-identical results).  Measured, it is no faster: the gathers, not the slots, set the
// latency, and the stages halve the threads per SM (fine_tma, off by default).  Every wait is
// bounded: a stage that does not complete in kFineSpin polls sets *err, and the CTA waits
// (bounded again) for its copies in flight before it returns.
constexpr int kFineTileSlices = 8;
constexpr int kFineSpin = 1 << 22;

enum FineMode : int { kFineFirst = 0, kFineStep = 1, kFineResid = 2 };

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait on a phase of an mbarrier: false when it did not complete
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    for (int k = 0; k < kFineSpin; ++k)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// global -> shared bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned)
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

struct FineTma {
    const int64_t *off;  // slice offsets (slots)
    const int32_t *col;
    const __half *hval;
    int64_t n, n_slices, n_tiles;
    int32_t stage_slots;  // slots one stage holds (the widest tile, rounded up to 64)
};

template <int MODE, int NST>
__global__ void __launch_bounds__(256) k_fine_tma(Gate gate, FineTma F, const float *__restrict__ b,
                                                  const float *__restrict__ invd, const float *__restrict__ x_in,
                                                  float *__restrict__ x_out, float *__restrict__ d, float c0, float c1,
                                                  float c2, const int32_t *__restrict__ agg, int32_t *err) {
    if (closed(gate)) return;
    extern __shared__ __align__(128) unsigned char fsm[];
    __shared__ __align__(8) uint64_t bar[NST];
    int s_bad = 0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const size_t col_bytes = (size_t)F.stage_slots * 4, stage_bytes = (size_t)F.stage_slots * 6;
    auto stage_col = [&](int k) { return reinterpret_cast<int32_t *>(fsm + k * stage_bytes); };
    auto stage_val = [&](int k) { return reinterpret_cast<__half *>(fsm + k * stage_bytes + col_bytes); };
    // tiles of this CTA: blockIdx.x, blockIdx.x + gridDim.x, ...
    const int64_t my_tiles = F.n_tiles > blockIdx.x ? (F.n_tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    auto issue = [&](int64_t k) {  // copy this CTA's tile k into stage k % NST
        const int64_t t = blockIdx.x + k * gridDim.x;
        const int64_t s0 = t * kFineTileSlices, s1 = min(s0 + kFineTileSlices, F.n_slices);
        const int64_t a = F.off[s0], z = F.off[s1];
        const uint32_t slots = (uint32_t)(z - a);
        const int st = (int)(k % NST);
        mbar_expect_tx(&bar[st], slots * 6u);
        bulk_g2s(stage_col(st), F.col + a, slots * 4u, &bar[st]);
        bulk_g2s(stage_val(st), F.hval + a, slots * 2u, &bar[st]);
    };
    if (threadIdx.x == 0) {
        for (int k = 0; k < NST; ++k) mbar_init(&bar[k], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int64_t k = 0; k < (my_tiles < NST ? my_tiles : (int64_t)NST); ++k) issue(k);
    int64_t done = 0;  // tiles whose stage completed (for the drain on an error)
    for (int64_t k = 0; k < my_tiles; ++k) {
        const int st = (int)(k % NST);
        const uint32_t parity = (uint32_t)((k / NST) & 1);
        // every thread observes the stage's completed phase itself (bounded)
        if (!__syncthreads_and(mbar_wait(&bar[st], parity))) {
            s_bad = 1;
            break;
        }
        done = k + 1;
        const int64_t t = blockIdx.x + k * gridDim.x;
        const int64_t s = t * kFineTileSlices + warp;
        if (s < F.n_slices) {
            const int64_t a0 = F.off[t * kFineTileSlices];
            const int64_t base = F.off[s];
            const int w = (int)((F.off[s + 1] - base) / kS);
            const int32_t *cs = stage_col(st) + (base - a0) + lane;
            const __half *vs = stage_val(st) + (base - a0) + lane;
            const int64_t i = s * kS + lane;
            const float *xg = MODE == kFineFirst ? b : x_in;
            constexpr int kB = 8;
            int32_t c[kB];
            float v[kB];
#pragma unroll
            for (int q = 0; q < kB; ++q) {
                c[q] = q < w ? cs[q * kS] : 0;
                v[q] = q < w ? __half2float(vs[q * kS]) : 0.f;
            }
            float g[kB];
#pragma unroll
            for (int q = 0; q < kB; ++q) g[q] = q < w ? xg[c[q]] : 0.f;
            float y = 0.f;
#pragma unroll
            for (int q = 0; q < kB; ++q) y += v[q] * g[q];
            for (int j = kB; j < w; ++j) y += __half2float(vs[j * kS]) * xg[cs[j * kS]];
            if (i < F.n) {
                if (MODE == kFineResid) {
                    x_out[i] = b[i] - y;
                } else if (MODE == kFineFirst) {
                    const float bi = b[i];
                    if (agg && agg[i] < 0) {
                        d[i] = 0.f;
                        x_out[i] = bi;
                    } else {
                        const float x1 = c0 * bi;
                        const float r = bi - c0 * y;
                        const float dn = c1 * x1 + c2 * r;
                        d[i] = dn;
                        x_out[i] = x1 + dn;
                    }
                } else {
                    const float di = invd ? invd[i] : 1.f;
                    if (agg && agg[i] < 0) {
                        d[i] = 0.f;
                        x_out[i] = di * b[i];
                    } else {
                        const float r = b[i] - y;
                        const float dn = (c1 != 0.f ? c1 * d[i] : 0.f) + c2 * di * r;
                        d[i] = dn;
                        x_out[i] = x_in[i] + dn;
                    }
                }
            }
        }
        __syncthreads();  // the stage is free again
        if (threadIdx.x == 0 && k + NST < my_tiles) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue(k + NST);
        }
    }
    if (s_bad && threadIdx.x == 0) {
        atomicExch(err, 1);
        // let the copies this CTA still has in flight land before the CTA leaves
        for (int64_t k = done; k < (my_tiles < done + NST ? my_tiles : done + NST); ++k)
            mbar_wait(&bar[k % NST], (uint32_t)((k / NST) & 1));
    }
}

// widest tile of the fine level (slots), for the stage size
__global__ void k_fine_tile_max(const int64_t *__restrict__ off, int64_t n_slices, int64_t n_tiles,
                                unsigned int *mx) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tiles) return;
    const int64_t s0 = t * kFineTileSlices, s1 = min(s0 + kFineTileSlices, n_slices);
    atomicMax(mx, (unsigned int)(off[s1] - off[s0]));
}

// ---- the coarse tail of the V-cycle in one cluster launch -----------------------------------
// The levels below a few thousand rows are latency-bound: each of their kernels does a
// microsecond of work and costs a launch.  One thread-block cluster runs all of them: the host
// compiles the tail's part of the cycle into a list of phases (the operations, pointers and
// coefficients the per-level kernels would get), and the cluster executes the list with a
// cluster barrier after each phase.  Every phase keeps the per-level kernels' work split and
// summation order (rows in 32-row slices with G warps each, the 256-thread groups of the long
// rows and of the scaling's partial sums), so the tail gives the same bits as the separate
// launches.  Vectors written by one phase are read by later ones through L2 (ld.global.cg);
// the matrices through the read-only path.  Measured, a phase costs more than the launch it
// saves (the chain of dependent L2 loads stays), so the tail is off by default (tail_rows).
constexpr int kTailThreads = 1024, kTailWarps = kTailThreads / 32;
constexpr int kTailGroups = kTailThreads / 256;  // 256-thread groups per CTA

enum TailOp : int32_t {
    kTailStep = 0,           // Chebyshev step (k_sm_step + k_long_rows<0>)
    kTailResid = 1,          // residual (k_residual + k_long_rows<1>)
    kTailRestrict = 2,       // restriction (k_restrict)
    kTailRestrictFirst = 3,  // restriction and the coarse level's first step (k_restrict_first)
    kTailFirst = 4,          // first step from zero (k_sm_first)
    kTailDense = 5,          // dense coarsest solve (k_dense_gemv)
    kTailDots = 6,           // coarse-correction scaling (k_long_rows<2> + k_coarse_dots)
    kTailProlong = 7         // prolongation (k_prolong)
};

struct TailLevel {
    MatView A;
    const float *invd;
    const int32_t *agg;       // coarse row of each row of this level, -1: none
    const int32_t *ms, *mr;   // rows of each coarse row (restriction from this level)
    const int32_t *longrows;  // rows longer than kLongRow
    int64_t nc;               // coarse rows (restriction from this level)
    int32_t n_long, g;
};

struct TailPhase {
    int32_t op, level;   // level: index into the level table (Restrict*: the fine side)
    int32_t next;        // Restrict*: the coarse side's index
    int32_t use_alpha;   // Prolong: scale by *alpha (the last Dots), else by alpha_fixed
    const float *b;      // Step, Resid, First, Dense, Dots: the level's rhs
    const float *x_in;   // Step, Resid, Dots: x; Prolong: the coarse level's x; Restrict*: r
    float *x_out;        // Step: new x; Resid: r; First, Dense: x; Prolong: x (+=); Restrict*: b_c
    float *d;            // Step, First: d; RestrictFirst: the coarse level's d
    float *x2;           // RestrictFirst: the coarse level's x
    const float *dense;  // Dense: the inverse (n x n)
    double *alpha;       // Dots: written; Prolong: read
    float c1, c2, alpha_fixed;
    int32_t dense_n;
};

__device__ __forceinline__ float tail_part(const MatView &A, int64_t i, int g, int G, const float *__restrict__ x) {
    int64_t base;
    int w, ln;
    row_of(A, i, base, w, ln);
    constexpr int kB = 8;
    float y = 0.f;
    for (int j0 = g; j0 < w; j0 += kB * G) {
        int32_t c[kB];
        float v[kB];
#pragma unroll
        for (int k = 0; k < kB; ++k) {
            const int j = j0 + k * G;
            const int64_t slot = base + (int64_t)j * kS + ln;
            c[k] = j < w ? __ldg(A.col + slot) : 0;
            v[k] = j < w ? __ldg(A.val + slot) : 0.f;
        }
        float gx[kB];
#pragma unroll
        for (int k = 0; k < kB; ++k) gx[k] = j0 + k * G < w ? __ldcg(x + c[k]) : 0.f;
#pragma unroll
        for (int k = 0; k < kB; ++k) y += v[k] * gx[k];
    }
    return y;
}

// Step, Resid or Dots over the regular rows of a level: rounds of 32 warps per CTA, warp gw of
// the cluster-wide virtual grid taking slice gw / G, part g = gw % G (split_row's mapping);
// Dots leaves its per-256-thread-group partials (k_coarse_dots' blocks) in part.
__device__ void tail_rows(const TailPhase &p, const TailLevel &L, int cta, int n_cta, double *__restrict__ part,
                          float (*sh)[32], double (*shd)[kTailWarps]) {
    const MatView &A = L.A;
    const int G = L.g, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t warps_all = (int64_t)n_cta * kTailWarps;
    const int64_t tasks = A.n / kS * G;  // warps of the per-level launch (split_blocks * 8, rounded up)
    const int64_t n_vb = (tasks + 7) / 8;
    for (int64_t r0 = 0; r0 < n_vb * 8; r0 += warps_all) {
        const int64_t gw = r0 + (int64_t)cta * kTailWarps + warp;
        const int64_t i = (gw / G) * kS + lane;
        const int g = (int)(gw % G);
        const bool outside = p.op == kTailStep && i < A.n && L.agg && L.agg[i] < 0;
        const bool live = i < A.n && !outside && !is_long(A, i);
        float y = live ? tail_part(A, i, g, G, p.x_in) : 0.f;
        if (G > 1) {
            sh[warp][lane] = y;
            __syncthreads();
            float t = 0.f;
            if (warp % G == 0)
                for (int k = 0; k < G; ++k) t += sh[warp + k][lane];
            y = t;
            __syncthreads();
        }
        if (p.op == kTailDots) {
            double xb = 0.0, xax = 0.0;
            if (g == 0 && live) {
                const double xi = (double)__ldcg(p.x_in + i);
                xb = xi * (double)__ldcg(p.b + i);
                xax = xi * (double)y;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                xb += __shfl_xor_sync(kFull, xb, o);
                xax += __shfl_xor_sync(kFull, xax, o);
            }
            if (lane == 0) {
                shd[0][warp] = xb;
                shd[1][warp] = xax;
            }
            __syncthreads();
            if (threadIdx.x < kTailWarps / 8) {  // one thread per group of 8 warps
                const int64_t vb = (r0 + (int64_t)cta * kTailWarps) / 8 + threadIdx.x;
                double a = 0.0, c = 0.0;
                for (int w = 0; w < 8; ++w) {
                    a += shd[0][threadIdx.x * 8 + w];
                    c += shd[1][threadIdx.x * 8 + w];
                }
                if (vb < n_vb) {
                    __stcg(part + 2 * vb, a);
                    __stcg(part + 2 * vb + 1, c);
                }
            }
            __syncthreads();
            continue;
        }
        if (g != 0 || i >= A.n) continue;
        if (p.op == kTailResid) {
            if (live) p.x_out[i] = __ldcg(p.b + i) - y;
            continue;
        }
        const float di = L.invd ? __ldg(L.invd + i) : 1.f;
        if (outside) {
            p.d[i] = 0.f;
            p.x_out[i] = di * __ldcg(p.b + i);
            continue;
        }
        if (!live) continue;
        const float rr = __ldcg(p.b + i) - y;
        const float dn = (p.c1 != 0.f ? p.c1 * __ldcg(p.d + i) : 0.f) + p.c2 * di * rr;
        p.d[i] = dn;
        p.x_out[i] = __ldcg(p.x_in + i) + dn;
    }
}

// the long rows of a level: 256-thread groups, one row each (k_long_rows' block); Dots leaves
// the rows' terms in long_part
__device__ void tail_long(const TailPhase &p, const TailLevel &L, int cta, int n_cta, double *__restrict__ long_part,
                          float (*red)[8]) {
    if (L.n_long <= 0) return;
    const MatView &A = L.A;
    const int grp = threadIdx.x >> 8, t = threadIdx.x & 255;
    const int n_grp = n_cta * kTailGroups;
    for (int k0 = 0; k0 < L.n_long; k0 += n_grp) {
        const int k = k0 + cta * kTailGroups + grp;
        float y = 0.f;
        int64_t i = 0;
        if (k < L.n_long) {
            i = __ldg(L.longrows + k);
            int64_t base;
            int w, ln;
            row_of(A, i, base, w, ln);
            for (int j = t; j < w; j += 256) {
                const int64_t slot = base + (int64_t)j * kS + ln;
                y += __ldg(A.val + slot) * __ldcg(p.x_in + __ldg(A.col + slot));
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) y += __shfl_xor_sync(kFull, y, o);
        if ((t & 31) == 0) red[grp][t >> 5] = y;
        __syncthreads();
        if (t == 0 && k < L.n_long) {
            y = 0.f;
            for (int q = 0; q < 8; ++q) y += red[grp][q];
            if (p.op == kTailStep) {
                const float di = L.invd ? __ldg(L.invd + i) : 1.f;
                const float dn = (p.c1 != 0.f ? p.c1 * __ldcg(p.d + i) : 0.f) + p.c2 * di * (__ldcg(p.b + i) - y);
                p.d[i] = dn;
                p.x_out[i] = __ldcg(p.x_in + i) + dn;
            } else if (p.op == kTailResid) {
                p.x_out[i] = __ldcg(p.b + i) - y;
            } else {
                const double xi = (double)__ldcg(p.x_in + i);
                __stcg(long_part + 2 * k, xi * (double)__ldcg(p.b + i));
                __stcg(long_part + 2 * k + 1, xi * (double)y);
            }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kTailThreads, 1)
    k_tail(Gate gate, const TailPhase *__restrict__ prog, int n_phases, const TailLevel *__restrict__ levels,
           double *__restrict__ scratch, int64_t long_off) {
    if (closed(gate)) return;  // the same for every CTA: nothing else writes n_done meanwhile
    cg::cluster_group cluster = cg::this_cluster();
    const int cta = (int)cluster.block_rank(), n_cta = (int)cluster.num_blocks();
    __shared__ float sh[kTailWarps][32];
    __shared__ double shd[2][kTailWarps];
    __shared__ float red[kTailGroups][8];
    __shared__ double tree[2][256];
    const int64_t tid = (int64_t)cta * kTailThreads + threadIdx.x, n_thr = (int64_t)n_cta * kTailThreads;
    for (int ph = 0; ph < n_phases; ++ph) {
        const TailPhase &p = prog[ph];
        const TailLevel &L = levels[p.level];
        switch (p.op) {
            case kTailStep:
            case kTailResid:
                tail_rows(p, L, cta, n_cta, scratch, sh, shd);
                tail_long(p, L, cta, n_cta, scratch + long_off, red);
                break;
            case kTailDots: {
                tail_rows(p, L, cta, n_cta, scratch, sh, shd);
                tail_long(p, L, cta, n_cta, scratch + long_off, red);
                cluster.sync();
                // the factor from the partials in k_coarse_dots' order, by the first CTA
                if (cta == 0) {
                    const int64_t n_vb = (L.A.n / kS * L.g + 7) / 8;
                    double a = 0.0, c = 0.0;
                    if (threadIdx.x < 256) {
                        for (int64_t k = threadIdx.x; k < n_vb; k += 256) {
                            a += __ldcg(scratch + 2 * k);
                            c += __ldcg(scratch + 2 * k + 1);
                        }
                        for (int k = threadIdx.x; k < L.n_long; k += 256) {
                            a += __ldcg(scratch + long_off + 2 * k);
                            c += __ldcg(scratch + long_off + 2 * k + 1);
                        }
                        tree[0][threadIdx.x] = a;
                        tree[1][threadIdx.x] = c;
                    }
                    __syncthreads();
                    for (int st = 128; st > 0; st >>= 1) {
                        if ((int)threadIdx.x < st) {
                            tree[0][threadIdx.x] += tree[0][threadIdx.x + st];
                            tree[1][threadIdx.x] += tree[1][threadIdx.x + st];
                        }
                        __syncthreads();
                    }
                    if (threadIdx.x == 0) {
                        const double num = tree[0][0], den = tree[1][0];
                        __stcg(p.alpha, (den > 0.0 && num > 0.0 && isfinite(num / den)) ? num / den : 1.0);
                    }
                }
                break;
            }
            case kTailRestrict:
            case kTailRestrictFirst: {
                const TailLevel &C = levels[p.next];
                const int64_t nc_pad = C.A.n;
                for (int64_t I = tid; I < nc_pad; I += n_thr) {
                    float s = 0.f;
                    if (I < L.nc)
                        for (int32_t k = __ldg(L.ms + I); k < __ldg(L.ms + I + 1); ++k)
                            s += 1.f * __ldcg(p.x_in + __ldg(L.mr + k));
                    p.x_out[I] = s;
                    if (p.op == kTailRestrictFirst) {
                        const bool exact = __ldg(C.agg + I) < 0;
                        const float v = (exact ? 1.f : p.c2) * __ldg(C.invd + I) * s;
                        p.d[I] = exact ? 0.f : v;
                        p.x2[I] = v;
                    }
                }
                break;
            }
            case kTailFirst:
                for (int64_t i = tid; i < L.A.n; i += n_thr) {
                    const float di = L.invd ? __ldg(L.invd + i) : 1.f;
                    if (L.agg && __ldg(L.agg + i) < 0) {
                        p.d[i] = 0.f;
                        p.x_out[i] = di * __ldcg(p.b + i);
                        continue;
                    }
                    const float v = p.c2 * di * __ldcg(p.b + i);
                    p.d[i] = v;
                    p.x_out[i] = v;
                }
                break;
            case kTailDense: {
                const int64_t n = p.dense_n, n_pad = L.A.n;
                const int lane = threadIdx.x & 31;
                for (int64_t i = tid >> 5; i < n_pad; i += n_thr >> 5) {
                    float s = 0.f;
                    if (i < n)
                        for (int64_t j = lane; j < n; j += 32) s += __ldg(p.dense + i * n + j) * __ldcg(p.b + j);
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
                    if (lane == 0) p.x_out[i] = s;
                }
                break;
            }
            case kTailProlong: {
                const float al = p.use_alpha ? (float)__ldcg(p.alpha) : p.alpha_fixed;
                for (int64_t i = tid; i < L.A.n; i += n_thr) {
                    const int32_t a = __ldg(L.agg + i);
                    if (a >= 0) p.x_out[i] = __ldcg(p.x_out + i) + al * 1.f * __ldcg(p.x_in + a);
                }
                break;
            }
            default:
                break;
        }
        cluster.sync();
    }
}

// the row kernels of a level with G warps per slice (G = 1, 2, 4 or 8)
decltype(&k_sm_step<1>) sm_step_kernel(int g) {
    return g >= 8 ? k_sm_step<8> : g >= 4 ? k_sm_step<4> : g >= 2 ? k_sm_step<2> : k_sm_step<1>;
}
decltype(&k_residual<1>) residual_kernel(int g) {
    return g >= 8 ? k_residual<8> : g >= 4 ? k_residual<4> : g >= 2 ? k_residual<2> : k_residual<1>;
}
decltype(&k_coarse_dots<1>) coarse_dots_kernel(int g) {
    return g >= 8 ? k_coarse_dots<8> : g >= 4 ? k_coarse_dots<4> : g >= 2 ? k_coarse_dots<2> : k_coarse_dots<1>;
}
decltype(&k_level_diag<1>) level_diag_kernel(int g) {
    return g >= 8 ? k_level_diag<8> : g >= 4 ? k_level_diag<4> : g >= 2 ? k_level_diag<2> : k_level_diag<1>;
}
decltype(&k_pair_want<1>) pair_want_kernel(int g) {
    return g >= 8 ? k_pair_want<8> : g >= 4 ? k_pair_want<4> : g >= 2 ? k_pair_want<2> : k_pair_want<1>;
}
// blocks of 8 warps covering n rows (a multiple of 32) with G warps per slice
unsigned split_blocks(int64_t n, int g) { return nblk(n / kS * g, 8); }
unsigned row_blocks(const AmgLevel &L) { return split_blocks(L.A.n, L.g); }
// warps per slice for a matrix: the fewest with at most `width` slots per warp and row (one on
// the fine level, whose 7-8 entries per row are loaded together by each thread)
int split_of(const AmgMatrix &A, int forced, int width) {
    if (!A.rlen) return 1;
    int g = 1;
    if (forced > 0) g = forced;
    else {
        const double w = A.n > 0 ? (double)A.slots / (double)A.n : 0.0;
        while (g < 8 && w > (double)width * g) g *= 2;
    }
    return g >= 8 ? 8 : g >= 4 ? 4 : g >= 2 ? 2 : 1;
}

}  // namespace

// ---- host side -------------------------------------------------------------------------------
#define AMG_CK(call)                                          \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) {                              \
            err = std::string(#call) + ": " + cudaGetErrorString(e_); \
            return e_;                                        \
        }                                                     \
    } while (0)

void Amg::release() {
    for (auto &L : lv_) {
        L.slice_off.release();
        L.col.release();
        L.val.release();
        L.inv_diag.release();
        L.agg.release();
        L.rlen.release();
        L.longrows.release();
        L.mem_start.release();
        L.mem_rows.release();
        L.b.release();
        L.xa.release();
        L.xb.release();
        L.d.release();
        L.r.release();
    }
    lv_.clear();
    n_levels_ = 0;
    for (auto *b : {&mate_, &want_, &cid_, &tmp_agg_, &tmp_ms_, &tmp_mr_, &cnt_, &rowlen_, &scan32_blk_, &flag_})
        b->release();
    for (auto *b : {&width_, &scan64_, &scan64_blk_, &mid_off_[0], &mid_off_[1]}) b->release();
    mid_col_[0].release();
    mid_col_[1].release();
    mid_val_[0].release();
    mid_val_[1].release();
    mid_invd_.release();
    dots_.release();
    dots_long_.release();
    big_list_.release();
    big_count_.release();
    tbound_.release();
    packed_.release();
    pscan_.release();
    bounds_.release();
    toff_.release();
    tcol_.release();
    tval_.release();
    lflag_.release();
    lpos_.release();
    for (auto &b : mid_rlen_) b.release();
    for (auto &b : mid_long_) b.release();
    alpha_.release();
    tickets_.release();
    w0_.release();
    fine_half_.release();
    w0_used_ = nullptr;
    isd_.release();
    dense_inv_.release();
    bound_.release();
    tail_prog_.release();
    tail_levels_.release();
    tile_max_.release();
    tma_err_.release();
    fine_tma_ = false;
    tail_scratch_.release();
    tail_level_ = tail_phases_ = tail_regular_ = 0;
    tail_out_ = nullptr;
    if (h_flag_) cudaFreeHost(h_flag_);
    h_flag_ = nullptr;
}

cudaError_t Amg::scan_i32_dev(const int32_t *in, int32_t *out, int64_t n, cudaStream_t s) {
    AMG_CK(launch_scan<int32_t>(in, out, n, scan32_blk_, s));
    return cudaSuccess;
}

cudaError_t Amg::scan_i64_dev(const int64_t *in, int64_t *out, int64_t n, cudaStream_t s) {
    AMG_CK(launch_scan<int64_t>(in, out, n, scan64_blk_, s));
    return cudaSuccess;
}

cudaError_t Amg::scan_i32(const int32_t *in, int32_t *out, int64_t n, int64_t &total, cudaStream_t s) {
    AMG_CK(launch_scan<int32_t>(in, out, n, scan32_blk_, s));
    int32_t t = 0;
    AMG_CK(cudaMemcpyAsync(&t, out + n, sizeof(t), cudaMemcpyDeviceToHost, s));
    AMG_CK(cudaStreamSynchronize(s));
    total = t;
    return cudaSuccess;
}

cudaError_t Amg::scan_i64(const int64_t *in, int64_t *out, int64_t n, int64_t &total, cudaStream_t s) {
    AMG_CK(launch_scan<int64_t>(in, out, n, scan64_blk_, s));
    AMG_CK(cudaMemcpyAsync(&total, out + n, sizeof(total), cudaMemcpyDeviceToHost, s));
    AMG_CK(cudaStreamSynchronize(s));
    return cudaSuccess;
}

cudaError_t Amg::level_stats(AmgLevel &L, unsigned int *bound, cudaStream_t s) {
    const int64_t n = L.A.n;
    AMG_CK(L.inv_diag.ensure(n));
    AMG_CK(isd_.ensure(n));
    const int g = split_of(L.A, opt_.split, opt_.split_width);
    level_diag_kernel(g)<<<split_blocks(n, g), 256, 0, s>>>(view(L.A), L.inv_diag.p, isd_.p, bound);
    if (L.A.long_count)
        k_level_diag_long<<<148, 256, 0, s>>>(view(L.A), L.A.long_count, L.inv_diag.p, isd_.p, bound);
    AMG_CK(cudaGetLastError());
    return cudaSuccess;
}

// ---- spectral estimates ---------------------------------------------------------------------
// One power-iteration step y = D^-1 A x (thread per row over the whole row, long rows included:
// setup only).  The start vector is a fixed pseudo-random sign pattern of amplitude in [0.5, 1)
// (no scaling between steps: |D^-1 A| <= a few, so 12 steps stay far from FP32 overflow).
__global__ void k_power_start(int64_t n, float *x) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t h = (uint32_t)i * 2654435761u;
    h ^= h >> 15;
    h *= 2246822519u;
    h ^= h >> 13;
    x[i] = ((h & 1u) ? 1.f : -1.f) * (0.5f + (float)((h >> 8) & 0xffffu) * (0.5f / 65536.f));
}

// y = D^-1 A x with the cycle's row kernels' split (G warps per slice, eight loads in flight);
// the long rows are left to k_long_rows<3>
template <int G>
__global__ void __launch_bounds__(256) k_power_step(MatView A, const float *__restrict__ invd,
                                                    const float *__restrict__ x, float *__restrict__ y) {
    int64_t i;
    int g;
    split_row<G>(i, g);
    const bool live = i < A.n && !is_long(A, i);
    const float acc = split_sum<G>(live ? split_part<G>(A, i, g, x) : 0.f);
    if (g != 0 || !live) return;
    y[i] = invd ? invd[i] * acc : acc;
}

// per-block partial sums of x.x and y.y (fixed grid, fixed tree: deterministic)
constexpr int kPowerBlocks = 296;
__global__ void __launch_bounds__(256) k_power_norms(int64_t n, const float *__restrict__ x, const float *__restrict__ y,
                                                     double *__restrict__ part) {
    double sx = 0.0, sy = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        sx += (double)x[i] * x[i];
        sy += (double)y[i] * y[i];
    }
    __shared__ double sh[2][256];
    sh[0][threadIdx.x] = sx;
    sh[1][threadIdx.x] = sy;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + w];
            sh[1][threadIdx.x] += sh[1][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = sh[0][0];
        part[2 * blockIdx.x + 1] = sh[1][0];
    }
}

// fine smoother weights in effect: 1 on the rows outside the hierarchy (solved exactly, x = b)
__global__ void k_fine_weights_eff(int64_t n, const int32_t *__restrict__ agg, const float *__restrict__ w,
                                   float *__restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (agg && agg[i] < 0) ? 1.f : w[i];
}

// Gershgorin bound of Omega S^ on the fine level (unit diagonal): max_i w_i sum_j |a_ij|
__global__ void __launch_bounds__(256) k_fine_bound(MatView A, const float *__restrict__ w, unsigned int *bound) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    float m = 0.f;
    if (i < A.n) {
        int64_t base;
        int wd, ln;
        row_of(A, i, base, wd, ln);
        float sum = 0.f;
        for (int j = 0; j < wd; ++j) sum += fabsf(__ldg(A.val + base + (int64_t)j * kS + ln));
        m = w[i] * sum;
    }
    __shared__ float wm[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(kFull, m, o));
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t = fmaxf(t, wm[k]);
        if (t > 0.f) atomicMax(bound, __float_as_uint(t));
    }
}

__global__ void k_power_total(const double *__restrict__ part, int nb, double *__restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double a = 0.0, b = 0.0;
    for (int k = 0; k < nb; ++k) {
        a += part[2 * k];
        b += part[2 * k + 1];
    }
    out[0] = a;
    out[1] = b;
}

// One pairing pass on A (rows excluded by row_edge < 0 or without coupling get agg = -1):
// agg [A.n], nc aggregates, member lists mstart [nc+1], mrows.
cudaError_t Amg::pair_pass(const AmgMatrix &A, const float *isd, const int32_t *row_edge, DBuf<int32_t> &agg,
                           int64_t &nc, DBuf<int32_t> &mstart, DBuf<int32_t> &mrows, cudaStream_t s) {
    const int64_t n = A.n;
    const MatView V = view(A);
    AMG_CK(mate_.ensure(n));
    AMG_CK(want_.ensure(n));
    AMG_CK(packed_.ensure(n + 1));
    AMG_CK(pscan_.ensure(n + 1));
    AMG_CK(agg.ensure(n));
    const unsigned g = nblk(n, 256);
    const int gw = split_of(A, opt_.split, opt_.split_width);
    k_pair_init<<<g, 256, 0, s>>>(V, row_edge, isd, mate_.p);
    for (int r = 0; r < opt_.pair_rounds; ++r) {
        pair_want_kernel(gw)<<<split_blocks(n, gw), 256, 0, s>>>(V, isd, mate_.p, want_.p,
                                                                  row_edge ? 0 : opt_.mix_coarse);
        k_pair_match<<<g, 256, 0, s>>>(n, want_.p, mate_.p);
    }
    k_pair_pack<<<g, 256, 0, s>>>(n, mate_.p, packed_.p);
    AMG_CK(cudaGetLastError());
    int64_t tot = 0;
    cudaError_t e = scan_i64(packed_.p, pscan_.p, n, tot, s);  // the one host read of the pass
    if (e != cudaSuccess) return e;
    nc = tot & 0xffffffff;
    const int64_t members = tot >> 32;
    AMG_CK(mstart.ensure(nc + 1));
    AMG_CK(mrows.ensure(std::max<int64_t>(members, 1)));
    k_pair_finish<<<std::max(g, 1u), 256, 0, s>>>(n, nc, members, mate_.p, packed_.p, pscan_.p, agg.p, mstart.p,
                                                  mrows.p);
    AMG_CK(cudaGetLastError());
    return cudaSuccess;
}

cudaError_t Amg::galerkin(const AmgMatrix &A, const int32_t *agg, int64_t nc, const int32_t *mstart,
                          const int32_t *mrows, DBuf<int64_t> &c_off, DBuf<int32_t> &c_col, DBuf<float> &c_val,
                          DBuf<int32_t> &c_rlen, DBuf<int32_t> &c_long, AmgMatrix &C, cudaStream_t s,
                          const float *wt) {
    const int64_t n_pad = round_up(nc, kS), n_sl = n_pad / kS;
    AMG_CK(rowlen_.ensure(n_pad));
    AMG_CK(cudaMemsetAsync(rowlen_.p, 0, n_pad * sizeof(int32_t), s));  // padding rows: no entries
    AMG_CK(width_.ensure(n_sl));
    AMG_CK(c_off.ensure(n_sl + 1));
    // compact row buffer sized by the candidate bound of every coarse row
    const MatView V = view(A);
    AMG_CK(tbound_.ensure(nc + 1));
    AMG_CK(toff_.ensure(nc + 1));
    if (nc > 0) k_cand_bound<<<nblk(nc, 256), 256, 0, s>>>(V, mstart, mrows, nc, tbound_.p);
    AMG_CK(cudaGetLastError());
    cudaError_t e = scan_i64_dev(tbound_.p, toff_.p, nc, s);
    if (e != cudaSuccess) return e;
    // every row of A belongs to at most one coarse row and contributes at most its slice
    // width: the candidates fit in A's slot count
    AMG_CK(tcol_.ensure(std::max<int64_t>(A.slots, 1)));
    AMG_CK(tval_.ensure(std::max<int64_t>(A.slots, 1)));
    // every row first with the small buffer; rows that overflow it run again as a list with
    // the large one (wide rows appear only on coarse levels, next to hub rows)
    AMG_CK(big_list_.ensure(std::max<int64_t>(nc, 1)));
    AMG_CK(big_count_.ensure(1));
    AMG_CK(cudaMemsetAsync(big_count_.p, 0, sizeof(int32_t), s));
    const unsigned g0 =
        (unsigned)std::max<int64_t>(1, std::min<int64_t>((nc + kGalWarps0 - 1) / kGalWarps0, 148 * 32));
    const size_t big_smem = (size_t)kGalWarpsBig * kGalCapBig * 8;
    AMG_CK(cudaFuncSetAttribute(k_galerkin<kGalCapBig, kGalWarpsBig, true>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)big_smem));
    k_galerkin<kGalCap0, kGalWarps0, false><<<g0, kGalWarps0 * 32, 0, s>>>(
        V, agg, mstart, mrows, nc, rowlen_.p, toff_.p, tcol_.p, tval_.p, flag_.p, wt, big_list_.p, big_count_.p);
    // the list pass reads its row count on the device (usually none: the blocks return at once);
    // an overflow there is reported at the end of the setup
    k_galerkin<kGalCapBig, kGalWarpsBig, true><<<148 * 2, kGalWarpsBig * 32, big_smem, s>>>(
        V, agg, mstart, mrows, nc, rowlen_.p, toff_.p, tcol_.p, tval_.p, flag_.p, wt, big_list_.p, big_count_.p);
    AMG_CK(cudaGetLastError());
    k_slice_width<<<nblk(n_sl, 256), 256, 0, s>>>(n_sl, nc, rowlen_.p, width_.p);
    AMG_CK(cudaGetLastError());
    int64_t slots = 0;
    if ((e = scan_i64(width_.p, c_off.p, n_sl, slots, s)) != cudaSuccess) return e;
    AMG_CK(c_col.ensure(std::max<int64_t>(slots, 1)));
    AMG_CK(c_val.ensure(std::max<int64_t>(slots, 1)));
    k_sell_fill<<<nblk(n_pad, 256), 256, 0, s>>>(n_pad, nc, c_off.p, rowlen_.p, toff_.p, tcol_.p, tval_.p, c_col.p,
                                                  c_val.p);
    AMG_CK(cudaGetLastError());
    C.n = n_pad;
    C.n_slices = n_sl;
    C.slots = slots;
    C.slice_off = c_off.p;
    C.col = c_col.p;
    C.val = c_val.p;
    // row lengths, and the rows too long for the thread-per-row kernels
    AMG_CK(c_rlen.ensure(n_pad));
    AMG_CK(cudaMemcpyAsync(c_rlen.p, rowlen_.p, n_pad * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
    C.rlen = c_rlen.p;
    AMG_CK(lflag_.ensure(n_pad));
    AMG_CK(lpos_.ensure(n_pad + 1));
    k_flag_long<<<nblk(n_pad, 256), 256, 0, s>>>(n_pad, c_rlen.p, lflag_.p);
    AMG_CK(cudaGetLastError());
    cudaError_t e2 = scan_i32_dev(lflag_.p, lpos_.p, n_pad, s);
    if (e2 != cudaSuccess) return e2;
    // the list holds its count in front: [count, rows...]; the host reads the counts of all
    // levels at the end of the setup
    AMG_CK(c_long.ensure(n_pad + 1));
    k_compact_long<<<nblk(n_pad, 256), 256, 0, s>>>(n_pad, lflag_.p, lpos_.p, c_long.p);
    AMG_CK(cudaGetLastError());
    C.longrows = c_long.p + 1;
    C.long_count = c_long.p;
    C.n_long = -1;  // not known on the host yet
    return cudaSuccess;
}

cudaError_t Amg::dense_coarse(const AmgMatrix &A, cudaStream_t s) {
    const int64_t n = dense_n_;
    AMG_CK(dense_inv_.ensure((size_t)n * n));
    AMG_CK(flag_.ensure(1));
    AMG_CK(cudaMemsetAsync(flag_.p, 0, sizeof(int32_t), s));
    const size_t smem = (size_t)(n * n + n) * sizeof(double);
    AMG_CK(cudaFuncSetAttribute(k_dense_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_dense_inverse<<<1, 1024, smem, s>>>(view(A), (int)n, dense_inv_.p, flag_.p);
    AMG_CK(cudaGetLastError());
    AMG_CK(cudaMemcpyAsync(h_flag_, flag_.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    AMG_CK(cudaStreamSynchronize(s));
    if (*h_flag_) {
        err = "coarsest matrix is not positive definite";
        return cudaErrorInvalidValue;
    }
    return cudaSuccess;
}

cudaError_t Amg::setup(const DevSystem &sys, const AmgOptions &o, cudaStream_t s) {
    opt_ = o;
    if (!h_flag_) AMG_CK(cudaHostAlloc((void **)&h_flag_, sizeof(int32_t), cudaHostAllocDefault));
    // device words the setup fills and the host reads once at its end: the Gershgorin bound of
    // each level, and the Galerkin overflow flag
    AMG_CK(bounds_.ensure(o.max_levels + 1));
    AMG_CK(cudaMemsetAsync(bounds_.p, 0, (o.max_levels + 1) * sizeof(unsigned int), s));
    AMG_CK(flag_.ensure(1));
    AMG_CK(cudaMemsetAsync(flag_.p, 0, sizeof(int32_t), s));
    if ((int)lv_.size() < o.max_levels) lv_.resize(o.max_levels);
    n_levels_ = 0;
    // level 0: the solver's FP32 scaled matrix
    AmgLevel &L0 = lv_[0];
    L0.A.n = sys.n_rows;
    L0.A.n_slices = sys.n_slices;
    L0.A.slots = sys.n_slots;
    L0.A.slice_off = sys.slice_off;
    L0.A.col = sys.col;
    L0.A.val = sys.val32;
    L0.A.rlen = nullptr;  // fine rows are short: the slice width bounds them
    L0.A.longrows = nullptr;
    L0.A.n_long = 0;
    L0.A.long_count = nullptr;
    // the cycle's fine-level kernels read the values in FP16 (unit diagonal, off-diagonals of
    // magnitude <= 1: relative rounding 5e-4, the same for a_ij and a_ji, so the cycle stays
    // symmetric); the setup and the Krylov products use the FP32 values
    if (opt_.half_fine) {
        AMG_CK(fine_half_.ensure(std::max<int64_t>(sys.n_slots, 1)));
        k_to_half<<<nblk(sys.n_slots, 256), 256, 0, s>>>(sys.n_slots, sys.val32, fine_half_.p);
        AMG_CK(cudaGetLastError());
    }
    fine_tma_ = false;
    const int64_t fine_tiles = (sys.n_slices + kFineTileSlices - 1) / kFineTileSlices;
    if (opt_.fine_tma && opt_.half_fine && fine_tiles > 0) {  // the widest tile, read with the bounds
        AMG_CK(tile_max_.ensure(1));
        AMG_CK(cudaMemsetAsync(tile_max_.p, 0, sizeof(unsigned int), s));
        k_fine_tile_max<<<nblk(fine_tiles, 256), 256, 0, s>>>(sys.slice_off, sys.n_slices, fine_tiles, tile_max_.p);
        AMG_CK(cudaGetLastError());
    }
    // level-0 weights: the near-null vector of the scaled system S^ = D^-1/2 S D^-1/2 is
    // D^1/2 1 (constants are near-null for S), so the level-0 transfers carry sqrt(diag S)
    AMG_CK(w0_.ensure(sys.n_rows));
    k_to_float<<<nblk(sys.n_rows, 256), 256, 0, s>>>(sys.n_rows, sys.dsq, w0_.p);
    AMG_CK(cudaGetLastError());
    const float *w0 = opt_.weighted ? w0_.p : nullptr;
    cudaError_t e;
    int poor_run = 0;  // consecutive coarsenings that kept more than half of the rows
    for (int l = 0;; ++l) {
        AmgLevel &L = lv_[l];
        AmgLevel &C = lv_[l + 1 < (int)lv_.size() ? l + 1 : l];
        if ((e = level_stats(L, bounds_.p + l, s)) != cudaSuccess) return e;
        AMG_CK(L.b.ensure(L.A.n));
        AMG_CK(L.xa.ensure(L.A.n));
        AMG_CK(L.xb.ensure(L.A.n));
        AMG_CK(L.d.ensure(L.A.n));
        AMG_CK(L.r.ensure(L.A.n));
        L.nc = 0;
        n_levels_ = l + 1;
        const int64_t n_real = l == 0 ? sys.n_rows : (l > 0 ? lv_[l - 1].nc : 0);
        if (n_real <= opt_.coarse_max || l + 1 >= opt_.max_levels) break;
        // pairing passes: pass 1 on A_l, pass p on the Galerkin matrix of pass p-1's pairs;
        // the aggregation of the level is their composition
        const int passes = l == 0 ? opt_.pair_passes : opt_.pair_passes_coarse;
        AmgMatrix cur = L.A;
        const float *curw = l == 0 ? w0 : nullptr;
        int64_t nc = 0;
        if ((e = pair_pass(cur, isd_.p, l == 0 ? sys.row_edge : nullptr, L.agg, nc, L.mem_start, L.mem_rows, s)) !=
            cudaSuccess)
            return e;
        const int32_t *cagg = L.agg.p, *cms = L.mem_start.p, *cmr = L.mem_rows.p;
        for (int p = 1; p < passes && nc > opt_.coarse_max; ++p) {
            AmgMatrix M;
            const int slot = p & 1;
            if ((e = galerkin(cur, cagg, nc, cms, cmr, mid_off_[slot], mid_col_[slot], mid_val_[slot], mid_rlen_[slot],
                              mid_long_[slot], M, s, curw)) != cudaSuccess)
                return e;
            AMG_CK(isd_.ensure(M.n));
            AMG_CK(mid_invd_.ensure(M.n));
            // (the intermediate matrix's bound is not needed: its own slot past the levels')
            unsigned int *mb = bounds_.p + o.max_levels;
            const int gm = split_of(M, opt_.split, opt_.split_width);
            level_diag_kernel(gm)<<<split_blocks(M.n, gm), 256, 0, s>>>(view(M), mid_invd_.p, isd_.p, mb);
            if (M.long_count)
                k_level_diag_long<<<148, 256, 0, s>>>(view(M), M.long_count, mid_invd_.p, isd_.p, mb);
            AMG_CK(cudaGetLastError());
            int64_t np = 0;
            if ((e = pair_pass(M, isd_.p, nullptr, tmp_agg_, np, tmp_ms_, tmp_mr_, s)) != cudaSuccess) return e;
            // compose: agg = agg_p[agg], members of each new aggregate in order
            AMG_CK(cnt_.ensure(np + 1));
            AMG_CK(cid_.ensure(np + 1));
            k_compose_agg<<<nblk(L.A.n, 256), 256, 0, s>>>(L.A.n, L.agg.p, tmp_agg_.p, L.agg.p);
            k_compose_count<<<nblk(np, 256), 256, 0, s>>>(np, tmp_ms_.p, tmp_mr_.p, L.mem_start.p, cnt_.p);
            AMG_CK(cudaGetLastError());
            // member offsets by a device-side scan; the member lists hold at most A_l's rows
            if ((e = scan_i32_dev(cnt_.p, cid_.p, np, s)) != cudaSuccess) return e;
            AMG_CK(want_.ensure(std::max<int64_t>(L.A.n, 1)));
            k_compose_fill<<<nblk(np, 256), 256, 0, s>>>(np, tmp_ms_.p, tmp_mr_.p, L.mem_start.p, L.mem_rows.p, cid_.p,
                                                         want_.p);
            AMG_CK(cudaGetLastError());
            std::swap(L.mem_start, cid_);  // the composed lists become the level's
            std::swap(L.mem_rows, want_);
            cur = M;
            curw = nullptr;
            cagg = tmp_agg_.p;
            cms = tmp_ms_.p;
            cmr = tmp_mr_.p;
            nc = np;
        }
        // the coarse matrix from the last pass's pairs
        if ((e = galerkin(cur, cagg, nc, cms, cmr, C.slice_off, C.col, C.val, C.rlen, C.longrows, C.A, s, curw)) !=
            cudaSuccess)
            return e;
        L.nc = nc;
        if (L.nc == 0) {  // nothing couples: this level is the last
            break;
        }
        if ((double)L.nc > 0.85 * (double)n_real) {  // coarsening stalls: stop one level later
            opt_.max_levels = std::min(opt_.max_levels, l + 2);
        }
        // slow coarsening (hub-dominated levels keep more than half their rows, level after
        // level): once the next level is small, it becomes the coarsest, smoothed by the
        // coarse polynomial, instead of many more levels of a few kernels each
        poor_run = 2 * L.nc > n_real ? poor_run + 1 : 0;
        if (opt_.stall_rows > 0 && poor_run >= 2 && L.nc <= opt_.stall_rows)
            opt_.max_levels = std::min(opt_.max_levels, l + 2);
    }
    {
        cudaError_t e2 = fine_weights_eff(s);
        if (e2 != cudaSuccess || (e2 = fine_interval(s)) != cudaSuccess) return e2;
        // the bounds, the long-row counts and the overflow flag first: the power iteration's
        // row kernels need each level's split and long rows
        std::vector<unsigned int> bits(n_levels_);
        std::vector<int32_t> nlong(n_levels_, 0);
        std::vector<double> pw(2 * n_levels_, 0.0);
        AMG_CK(cudaMemcpyAsync(bits.data(), bounds_.p, n_levels_ * sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
        if (fine_w_)  // the fine level is smoothed on Omega S^: its own bound
            AMG_CK(cudaMemcpyAsync(bits.data(), bounds_.p + opt_.max_levels, sizeof(unsigned int),
                                   cudaMemcpyDeviceToHost, s));
        for (int l = 1; l < n_levels_; ++l)
            if (lv_[l].A.long_count)
                AMG_CK(cudaMemcpyAsync(&nlong[l], lv_[l].A.long_count, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        AMG_CK(cudaMemcpyAsync(h_flag_, flag_.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        unsigned int widest = 0;
        if (opt_.fine_tma && opt_.half_fine && fine_tiles > 0)
            AMG_CK(cudaMemcpyAsync(&widest, tile_max_.p, sizeof(widest), cudaMemcpyDeviceToHost, s));
        AMG_CK(cudaStreamSynchronize(s));
        if (*h_flag_) {
            err = "Galerkin row wider than the gather buffer";
            return cudaErrorInvalidValue;
        }
        if (widest > 0) AMG_CK(prepare_fine_tma(widest, s));
        for (int l = 0; l < n_levels_; ++l) {
            lv_[l].A.n_long = nlong[l];
            // warps per slice in the row kernels: at most split_width slots per warp and row
            // (the fine level, 7-8 entries per row, keeps one thread per row)
            lv_[l].g = split_of(lv_[l].A, opt_.split, opt_.split_width);
        }
        if ((e2 = power_estimates(s)) != cudaSuccess) return e2;
        if (opt_.power_steps > 0) {
            AMG_CK(cudaMemcpyAsync(pw.data(), pw_sums_.p, 2 * n_levels_ * sizeof(double), cudaMemcpyDeviceToHost, s));
            AMG_CK(cudaStreamSynchronize(s));
        }
        for (int l = 0; l < n_levels_; ++l) {
            float hi;
            std::memcpy(&hi, &bits[l], sizeof(hi));
            lv_[l].gershgorin = hi > 0.f ? hi : 2.f;
            lv_[l].hi = lv_[l].gershgorin;
            // |v_k| / |v_{k-1}| of the power iteration (a lower estimate of lambda_max)
            if (opt_.power_steps > 0 && pw[2 * l] > 0.0 && pw[2 * l + 1] > 0.0 && std::isfinite(pw[2 * l + 1])) {
                const double est = std::sqrt(pw[2 * l + 1] / pw[2 * l]);
                lv_[l].hi = (float)std::min((double)lv_[l].gershgorin, opt_.power_safety * est);
            }
        }
    }
    const AmgLevel &Lc = lv_[n_levels_ - 1];
    dense_n_ = n_levels_ == 1 ? Lc.A.n : lv_[n_levels_ - 2].nc;
    if (dense_n_ > kDenseMax) {  // too large for the shared-memory inverse: smooth it instead
        dense_n_ = 0;
        AmgLevel &Lm = lv_[n_levels_ - 1];
        AMG_CK(Lm.agg.ensure(Lm.A.n));
        k_mark_isolated<<<nblk(Lm.A.n, 256), 256, 0, s>>>(view(Lm.A), Lm.agg.p);
        AMG_CK(cudaGetLastError());
    }
    w0_used_ = w0;
    // partial sums of the coarse-correction scaling, one slice per level
    dots_off_.assign(n_levels_, 0);
    int64_t tot = 0;
    for (int l = 0; l + 1 < n_levels_; ++l) {
        dots_off_[l] = tot;
        tot += 2 * (int64_t)row_blocks(lv_[l + 1]);
    }
    AMG_CK(dots_.ensure(tot + 2));
    dots_long_off_.assign(n_levels_, 0);
    int64_t tl = 0;
    for (int l = 0; l + 1 < n_levels_; ++l) {
        dots_long_off_[l] = tl;
        tl += 2 * std::max<int64_t>(0, lv_[l + 1].A.n_long);
    }
    AMG_CK(dots_long_.ensure(tl + 2));
    AMG_CK(alpha_.ensure(n_levels_ + 1));
    AMG_CK(tickets_.ensure(n_levels_ + 1));
    AMG_CK(cudaMemsetAsync(tickets_.p, 0, (n_levels_ + 1) * sizeof(unsigned int), s));
    if (dense_n_ > 0) AMG_CK(dense_coarse(Lc.A, s));
    return build_tail(s);
}

cudaError_t Amg::power_estimates(cudaStream_t s, int only_level) {
    if (opt_.power_steps <= 0) return cudaSuccess;
    int64_t nmax = 0;
    for (int l = 0; l < n_levels_; ++l) nmax = std::max(nmax, lv_[l].A.n);
    AMG_CK(pw_a_.ensure(std::max<int64_t>(nmax, 1)));
    AMG_CK(pw_b_.ensure(std::max<int64_t>(nmax, 1)));
    AMG_CK(pw_part_.ensure(2 * kPowerBlocks));
    AMG_CK(pw_sums_.ensure(2 * (size_t)std::max(n_levels_, 1)));
    if (only_level < 0)
        AMG_CK(cudaMemsetAsync(pw_sums_.p, 0, 2 * (size_t)std::max(n_levels_, 1) * sizeof(double), s));
    // the coarsest level is solved, not smoothed (unless coarsening stalled: it then gets a
    // Chebyshev polynomial of its own and an estimate too)
    for (int l = 0; l < n_levels_; ++l) {
        if (only_level >= 0 && l != only_level) continue;
        AmgLevel &L = lv_[l];
        const int64_t n = L.A.n;
        if (n <= 0) continue;
        // the fine level is the Jacobi-scaled system (unit diagonal): no D^-1, or the
        // smoother's row weights
        const float *invd = l == 0 ? fw() : L.inv_diag.p;
        const MatView V = view(L.A);
        float *x = pw_a_.p, *y = pw_b_.p;
        k_power_start<<<nblk(n, 256), 256, 0, s>>>(n, x);
        for (int k = 0; k < opt_.power_steps; ++k) {
            const unsigned gs = row_blocks(L);
            switch (L.g >= 8 ? 8 : L.g >= 4 ? 4 : L.g >= 2 ? 2 : 1) {
                case 8: k_power_step<8><<<gs, 256, 0, s>>>(V, invd, x, y); break;
                case 4: k_power_step<4><<<gs, 256, 0, s>>>(V, invd, x, y); break;
                case 2: k_power_step<2><<<gs, 256, 0, s>>>(V, invd, x, y); break;
                default: k_power_step<1><<<gs, 256, 0, s>>>(V, invd, x, y); break;
            }
            if (L.A.n_long > 0)
                k_long_rows<3><<<(unsigned)L.A.n_long, 256, 0, s>>>(Gate{nullptr, 0}, V, L.A.longrows, nullptr, invd,
                                                                    x, y, nullptr, 0.f, 0.f, nullptr);
            if (k + 1 < opt_.power_steps) std::swap(x, y);
        }
        k_power_norms<<<kPowerBlocks, 256, 0, s>>>(n, x, y, pw_part_.p);
        k_power_total<<<1, 32, 0, s>>>(pw_part_.p, kPowerBlocks, pw_sums_.p + 2 * l);
        AMG_CK(cudaGetLastError());
    }
    return cudaSuccess;
}

cudaError_t Amg::fine_weights_eff(cudaStream_t s) {
    if (!fine_w_) return cudaSuccess;
    const int64_t n = lv_[0].A.n;
    AMG_CK(fine_w_eff_.ensure(std::max<int64_t>(n, 1)));
    k_fine_weights_eff<<<nblk(n, 256), 256, 0, s>>>(n, n_levels_ > 1 ? lv_[0].agg.p : nullptr, fine_w_,
                                                    fine_w_eff_.p);
    AMG_CK(cudaGetLastError());
    return cudaSuccess;
}

// Level 0's Gershgorin bound of Omega S^ (into the spare bound word) for fine weights
cudaError_t Amg::fine_interval(cudaStream_t s) {
    if (!fine_w_) return cudaSuccess;
    unsigned int *b = bounds_.p + opt_.max_levels;
    AMG_CK(cudaMemsetAsync(b, 0, sizeof(unsigned int), s));
    k_fine_bound<<<nblk(lv_[0].A.n, 256), 256, 0, s>>>(view(lv_[0].A), fw(), b);
    AMG_CK(cudaGetLastError());
    return cudaSuccess;
}

cudaError_t Amg::refresh_fine(cudaStream_t s) {
    if (n_levels_ < 1) return cudaSuccess;
    cudaError_t e;
    if ((e = fine_weights_eff(s)) != cudaSuccess || (e = fine_interval(s)) != cudaSuccess ||
        (e = power_estimates(s, 0)) != cudaSuccess)
        return e;
    unsigned int bits = 0;
    double pw[2] = {0.0, 0.0};
    AMG_CK(cudaMemcpyAsync(&bits, bounds_.p + (fine_w_ ? opt_.max_levels : 0), sizeof(bits), cudaMemcpyDeviceToHost, s));
    if (opt_.power_steps > 0) AMG_CK(cudaMemcpyAsync(pw, pw_sums_.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    AMG_CK(cudaStreamSynchronize(s));
    float hi;
    std::memcpy(&hi, &bits, sizeof(hi));
    AmgLevel &L = lv_[0];
    L.gershgorin = hi > 0.f ? hi : 2.f;
    L.hi = L.gershgorin;
    if (opt_.power_steps > 0 && pw[0] > 0.0 && pw[1] > 0.0 && std::isfinite(pw[1]))
        L.hi = (float)std::min((double)L.gershgorin, opt_.power_safety * std::sqrt(pw[1] / pw[0]));
    return cudaSuccess;
}

void Amg::cheb_coeffs(const AmgLevel &L, std::vector<double> &c1, std::vector<double> &c2, int degree,
                      float ratio) const {
    const int deg = std::max(1, degree > 0 ? degree : opt_.cheb_degree);
    const double hi = L.hi, lo = hi / std::max(1.5f, ratio > 0.f ? ratio : opt_.cheb_ratio);
    const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
    double rho = 1.0 / sigma;
    c1.assign(deg, 0.0);
    c2.assign(deg, 1.0 / theta);
    for (int k = 1; k < deg; ++k) {
        const double rn = 1.0 / (2.0 * sigma - rho);
        c1[k] = rn * rho;
        c2[k] = 2.0 * rn / delta;
        rho = rn;
    }
}

int Amg::kernels_per_apply() const {
    const int deg = std::max(1, opt_.cheb_degree), pre = pre_degree();
    const int coarse = dense_n_ > 0 ? 1 : std::max(1, opt_.coarse_degree);
    return last_long_launches_ + (n_levels_ - 1) * (pre + deg + 3) + coarse - std::max(0, n_levels_ - 2) -
           (n_levels_ > 1 && pre >= 2 ? 1 : 0) +
           (opt_.kcycle ? std::min(opt_.kcycle_levels, std::max(0, n_levels_ - (dense_n_ > 0 ? 2 : 1))) : 0) -
           (tail_phases_ > 0 ? tail_regular_ - 1 : 0);
}

// Compiles the cycle's part on levels tail_level_ .. coarsest (for the cycle from level 0) into
// the phase list k_tail runs: the same operations, buffers and coefficients, in the order
// cycle() launches them, with level tail_level_'s first step left to the restriction above it
// and the scaling of level tail_level_ - 1's coarse correction as the last phase.
cudaError_t Amg::build_tail(cudaStream_t s) {
    tail_level_ = tail_phases_ = tail_regular_ = 0;
    tail_out_ = nullptr;
    const int nl = n_levels_;
    if (opt_.tail_rows <= 0 || nl < 3) return cudaSuccess;
    int t = nl - 1;
    while (t - 1 >= 1 && lv_[t - 1].A.n <= opt_.tail_rows) --t;
    if (t > nl - 2) return cudaSuccess;  // only the coarsest solve would move: nothing to gain
    // the cluster: 16 CTAs where the device schedules them, else 8
    if (tail_cluster_ == 0) {
        cudaFuncSetAttribute(k_tail, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        cudaGetLastError();
        for (int cl : {16, 8}) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(cl);
            cfg.blockDim = dim3(kTailThreads);
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = cl;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            int n = 0;
            if (cudaOccupancyMaxActiveClusters(&n, k_tail, &cfg) == cudaSuccess && n > 0) {
                tail_cluster_ = cl;
                break;
            }
            cudaGetLastError();
        }
        if (tail_cluster_ == 0) tail_cluster_ = -1;  // clusters unavailable: no tail
    }
    if (tail_cluster_ < 0) return cudaSuccess;
    std::vector<TailLevel> tl(nl);
    for (int l = t; l < nl; ++l) {
        const AmgLevel &L = lv_[l];
        TailLevel &q = tl[l];
        q.A = view(L.A);
        q.invd = L.inv_diag.p;
        q.agg = L.agg.p;
        q.ms = l + 1 < nl ? L.mem_start.p : nullptr;
        q.mr = l + 1 < nl ? L.mem_rows.p : nullptr;
        q.longrows = L.A.longrows;
        q.nc = l + 1 < nl ? L.nc : 0;
        q.n_long = (int32_t)L.A.n_long;
        q.g = L.g;
    }
    std::vector<TailPhase> ph;
    int64_t max_vb = 1, max_long = 1;
    auto phase = [&](int32_t op, int level) {
        TailPhase p = {};
        p.op = op;
        p.level = level;
        p.alpha_fixed = opt_.alpha;
        tail_regular_ += 1;
        return p;
    };
    auto dots = [&](int lc, const float *x, double *alpha) {
        TailPhase p = phase(kTailDots, lc);
        p.x_in = x;
        p.b = lv_[lc].b.p;
        p.alpha = alpha;
        ph.push_back(p);
        max_vb = std::max<int64_t>(max_vb, (lv_[lc].A.n / kS * lv_[lc].g + 7) / 8);
        max_long = std::max<int64_t>(max_long, lv_[lc].A.n_long);
    };
    std::vector<double> c1, c2;
    std::vector<float *> xout(nl, nullptr);
    const int pre = pre_degree(), deg = std::max(1, opt_.cheb_degree);
    // descend (level t's first step: the restriction from level t - 1)
    for (int l = t; l < nl - 1; ++l) {
        AmgLevel &L = lv_[l];
        cheb_coeffs(L, c1, c2);
        float *xi = L.xa.p, *xo = L.xb.p;
        for (int k = 1; k < pre; ++k) {
            TailPhase p = phase(kTailStep, l);
            p.b = L.b.p;
            p.x_in = xi;
            p.x_out = xo;
            p.d = L.d.p;
            p.c1 = (float)c1[k];
            p.c2 = (float)c2[k];
            ph.push_back(p);
            std::swap(xi, xo);
        }
        xout[l] = xi;
        TailPhase r = phase(kTailResid, l);
        r.b = L.b.p;
        r.x_in = xi;
        r.x_out = L.r.p;
        ph.push_back(r);
        AmgLevel &C = lv_[l + 1];
        TailPhase q = phase(l + 2 < nl ? kTailRestrictFirst : kTailRestrict, l);
        q.next = l + 1;
        q.x_in = L.r.p;
        q.x_out = C.b.p;
        if (l + 2 < nl) {
            std::vector<double> cc1, cc2;
            cheb_coeffs(C, cc1, cc2);
            q.c2 = (float)cc2[0];
            q.d = C.d.p;
            q.x2 = C.xa.p;
        }
        ph.push_back(q);
    }
    // coarsest
    {
        AmgLevel &Lc = lv_[nl - 1];
        if (dense_n_ > 0) {
            TailPhase p = phase(kTailDense, nl - 1);
            p.b = Lc.b.p;
            p.x_out = Lc.xa.p;
            p.dense = dense_inv_.p;
            p.dense_n = (int32_t)dense_n_;
            ph.push_back(p);
            xout[nl - 1] = Lc.xa.p;
        } else {
            cheb_coeffs(Lc, c1, c2, std::max(1, opt_.coarse_degree), opt_.coarse_ratio);
            float *xi = Lc.xa.p, *xo = Lc.xb.p;
            TailPhase f = phase(kTailFirst, nl - 1);
            f.b = Lc.b.p;
            f.x_out = xi;
            f.d = Lc.d.p;
            f.c2 = (float)c2[0];
            ph.push_back(f);
            for (int k = 1; k < std::max(1, opt_.coarse_degree); ++k) {
                TailPhase p = phase(kTailStep, nl - 1);
                p.b = Lc.b.p;
                p.x_in = xi;
                p.x_out = xo;
                p.d = Lc.d.p;
                p.c1 = (float)c1[k];
                p.c2 = (float)c2[k];
                ph.push_back(p);
                float *xk = xo;
                xo = xi;
                xi = xk;
            }
            xout[nl - 1] = xi;
        }
    }
    // ascend
    auto kcycle_at = [&](int l) { return opt_.kcycle && l < opt_.kcycle_levels && (l + 2 < nl || dense_n_ == 0); };
    for (int l = nl - 2; l >= t; --l) {
        AmgLevel &L = lv_[l];
        cheb_coeffs(L, c1, c2);
        float *xi = xout[l];
        TailPhase pr = phase(kTailProlong, l);
        if (kcycle_at(l)) {
            dots(l + 1, xout[l + 1], alpha_.p + l);
            pr.use_alpha = 1;
            pr.alpha = alpha_.p + l;
        }
        pr.x_in = xout[l + 1];
        pr.x_out = xi;
        ph.push_back(pr);
        float *other = xi == L.xa.p ? L.xb.p : L.xa.p;
        for (int k = 0; k < deg; ++k) {
            TailPhase p = phase(kTailStep, l);
            p.b = L.b.p;
            p.x_in = xi;
            p.x_out = other;
            p.d = L.d.p;
            p.c1 = k == 0 ? 0.f : (float)c1[k];
            p.c2 = (float)c2[k];
            ph.push_back(p);
            float *xo = other;
            other = xi;
            xi = xo;
        }
        xout[l] = xi;
    }
    if (kcycle_at(t - 1)) dots(t, xout[t], alpha_.p + (t - 1));
    AMG_CK(tail_prog_.ensure(ph.size() * sizeof(TailPhase)));
    AMG_CK(tail_levels_.ensure(tl.size() * sizeof(TailLevel)));
    AMG_CK(tail_scratch_.ensure(2 * (size_t)(max_vb + max_long)));
    AMG_CK(cudaMemcpyAsync(tail_prog_.p, ph.data(), ph.size() * sizeof(TailPhase), cudaMemcpyHostToDevice, s));
    AMG_CK(cudaMemcpyAsync(tail_levels_.p, tl.data(), tl.size() * sizeof(TailLevel), cudaMemcpyHostToDevice, s));
    AMG_CK(cudaStreamSynchronize(s));  // the host vectors go out of scope
    tail_long_off_ = 2 * max_vb;
    tail_level_ = t;
    tail_phases_ = (int)ph.size();
    tail_out_ = xout[t];
    return cudaSuccess;
}

cudaError_t Amg::launch_tail(const int32_t *n_done, int32_t n_inst, cudaStream_t s) const {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(tail_cluster_);
    cfg.blockDim = dim3(kTailThreads);
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = tail_cluster_;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    const Gate gate{n_done, n_inst};
    return cudaLaunchKernelEx(&cfg, k_tail, gate, reinterpret_cast<const TailPhase *>(tail_prog_.p), tail_phases_,
                              reinterpret_cast<const TailLevel *>(tail_levels_.p), tail_scratch_.p, tail_long_off_);
}

// Stage size and grid of the fine level's TMA-staged kernels for the widest tile: the ring of
// fine_stages_ stages must fit 100 KB of shared memory, else the per-thread kernels stay in use.
cudaError_t Amg::prepare_fine_tma(unsigned int widest, cudaStream_t s) {
    fine_tma_ = false;
    const AmgMatrix &A = lv_[0].A;
    const int64_t stage_slots = ((int64_t)widest + 63) / 64 * 64;
    fine_stages_ = opt_.fine_tma_stages >= 3 ? 4 : 2;
    const size_t smem = (size_t)fine_stages_ * (size_t)stage_slots * 6;
    if (stage_slots <= 0 || smem > 100 * 1024 || A.n_slices <= 0) return cudaSuccess;
    for (auto f : {k_fine_tma<kFineFirst, 2>, k_fine_tma<kFineStep, 2>, k_fine_tma<kFineResid, 2>,
                   k_fine_tma<kFineFirst, 4>, k_fine_tma<kFineStep, 4>, k_fine_tma<kFineResid, 4>})
        AMG_CK(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0, dev = 0, sms = 0;
    AMG_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, fine_stages_ == 4 ? k_fine_tma<kFineStep, 4> : k_fine_tma<kFineStep, 2>, 256, smem));
    AMG_CK(cudaGetDevice(&dev));
    AMG_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (per_sm < 1) return cudaSuccess;
    const int64_t tiles = (A.n_slices + kFineTileSlices - 1) / kFineTileSlices;
    fine_stage_slots_ = (int32_t)stage_slots;
    fine_tma_grid_ = (int)std::min<int64_t>(tiles, (int64_t)per_sm * sms);
    AMG_CK(tma_err_.ensure(1));
    AMG_CK(cudaMemsetAsync(tma_err_.p, 0, sizeof(int32_t), s));
    fine_tma_ = true;
    return cudaSuccess;
}

template <int MODE>
void Amg::launch_fine(const int32_t *n_done, int32_t n_inst, const float *b, const float *invd, const float *x_in,
                      float *x_out, float *d, float c0, float c1, float c2, cudaStream_t s) const {
    const AmgMatrix &A = lv_[0].A;
    FineTma F;
    F.off = A.slice_off;
    F.col = A.col;
    F.hval = reinterpret_cast<const __half *>(fine_half_.p);
    F.n = A.n;
    F.n_slices = A.n_slices;
    F.n_tiles = (A.n_slices + kFineTileSlices - 1) / kFineTileSlices;
    F.stage_slots = fine_stage_slots_;
    const size_t smem = (size_t)fine_stages_ * (size_t)fine_stage_slots_ * 6;
    const int32_t *agg = n_levels_ > 1 ? lv_[0].agg.p : nullptr;
    if (fine_stages_ == 4)
        k_fine_tma<MODE, 4><<<fine_tma_grid_, 256, smem, s>>>(Gate{n_done, n_inst}, F, b, invd, x_in, x_out, d, c0, c1,
                                                              c2, agg, tma_err_.p);
    else
        k_fine_tma<MODE, 2><<<fine_tma_grid_, 256, smem, s>>>(Gate{n_done, n_inst}, F, b, invd, x_in, x_out, d, c0, c1,
                                                              c2, agg, tma_err_.p);
}

bool Amg::fine_tma_failed(cudaStream_t s) {
    if (!fine_tma_) return false;
    int32_t e = 0;
    if (cudaMemcpyAsync(&e, tma_err_.p, sizeof(e), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return true;
    if (e) cudaMemsetAsync(tma_err_.p, 0, sizeof(int32_t), s);
    return e != 0;
}

cudaError_t Amg::apply(const float *r, float *z, const int32_t *n_done, int32_t n_inst, cudaStream_t s,
                       AmgProf *prof) {
    return cycle(0, r, z, n_done, n_inst, s, prof, nullptr);
}

// The V-cycle from level l0: l0 = 0 is the preconditioner (rhs r, result z); l0 > 0 runs the
// cycle of the coarser levels on the rhs already in lv_[l0].b and leaves its result in
// *x_l0 (a level buffer), with no fine-level work.
cudaError_t Amg::cycle(int l0, const float *r, float *z, const int32_t *n_done, int32_t n_inst, cudaStream_t s,
                       AmgProf *prof, float **x_l0) {
    const Gate gate_{n_done, n_inst};
    const int pre = pre_degree();
    int launches = 0;  // kernels of one cycle, for the launch count
    auto long_rows = [&](const AmgMatrix &M, int mode, const float *b, const float *invd, const float *x_in,
                         float *out, float *d, float c1, float c2, double *part) {
        if (M.n_long <= 0) return;
        const unsigned gl = (unsigned)M.n_long;
        const MatView V = view(M);
        if (mode == 0)
            k_long_rows<0><<<gl, 256, 0, s>>>(gate_, V, M.longrows, b, invd, x_in, out, d, c1, c2, part);
        else if (mode == 1)
            k_long_rows<1><<<gl, 256, 0, s>>>(gate_, V, M.longrows, b, invd, x_in, out, d, c1, c2, part);
        else
            k_long_rows<2><<<gl, 256, 0, s>>>(gate_, V, M.longrows, b, invd, x_in, out, d, c1, c2, part);
        ++launches;
    };
    // inside a capture only cudaEventRecordExternal turns a record into a graph node
    auto rec = [&](cudaEvent_t ev) {
        if (prof && ev) cudaEventRecordWithFlags(ev, s, cudaEventRecordExternal);
    };
    int step0 = 0;  // fine-level smoothing steps recorded so far
    auto rec_step = [&](bool start) {
        if (prof && step0 < (int)prof->smooth.size() / 2) rec(prof->smooth[2 * step0 + (start ? 0 : 1)]);
        if (!start) ++step0;
    };
    if (prof) rec(prof->cycle[0]);
    // descend: smooth from zero, residual, restrict
    std::vector<double> c1, c2;
    const int deg = std::max(1, opt_.cheb_degree);
    const int nl = n_levels_;
    std::vector<float *> xout(nl);
    // the levels from tail_level_ down run as one cluster launch (the cycle from level 0 only)
    const bool use_tail = tail_phases_ > 0 && tail_level_ > l0;
    // the fine level's kernels stream its FP16 matrix through shared memory (k_fine_tma)
    const bool tma0 = fine_tma_ && opt_.half_fine && l0 == 0;
    for (int l = l0; l < (use_tail ? tail_level_ : nl - 1); ++l) {
        AmgLevel &L = lv_[l];
        const float *b = l == 0 ? r : L.b.p;
        // the scaled fine level has unit diagonal; with smoother weights Omega, D^-1 -> Omega
        const float *invd = l == 0 ? fw() : L.inv_diag.p;
        MatView A = view(L.A);
        if (l == 0 && opt_.half_fine) A.hval = reinterpret_cast<const __half *>(fine_half_.p);
        const unsigned g = nblk(L.A.n, 256), gs = row_blocks(L);
        const auto sm_step = sm_step_kernel(L.g);
        cheb_coeffs(L, c1, c2);
        float *xi = L.xa.p, *xo = L.xb.p;
        int k0 = 1;
        if (l == 0 && pre >= 2) {  // first two steps in one pass
            rec_step(true);
            if (fine_w_)
                k_sm_first_step_w<<<g, 256, 0, s>>>(gate_, A, b, fw(), xo, L.d.p, (float)c2[0], (float)c1[1],
                                                    (float)c2[1], L.agg.p);
            else if (tma0)
                launch_fine<kFineFirst>(n_done, n_inst, b, nullptr, nullptr, xo, L.d.p, (float)c2[0], (float)c1[1],
                                        (float)c2[1], s);
            else
                k_sm_first_step<<<g, 256, 0, s>>>(gate_, A, b, xo, L.d.p, (float)c2[0], (float)c1[1], (float)c2[1],
                                                  L.agg.p);
            rec_step(false);
            std::swap(xi, xo);
            k0 = 2;
        } else if (l == 0 || l == l0) {  // (a cycle started below the fine level: its first step)
            k_sm_first<<<g, 256, 0, s>>>(gate_, L.A.n, b, invd, (float)c2[0], xi, L.d.p, L.agg.p);
        }
        // (coarser levels: the first step was fused into the restriction from the level above)
        for (int k = k0; k < pre; ++k) {
            if (l == 0) rec_step(true);
            if (l == 0 && tma0)
                launch_fine<kFineStep>(n_done, n_inst, b, invd, xi, xo, L.d.p, 0.f, (float)c1[k], (float)c2[k], s);
            else
                sm_step<<<gs, 256, 0, s>>>(gate_, A, b, invd, xi, xo, L.d.p, (float)c1[k], (float)c2[k], L.agg.p);
            long_rows(L.A, 0, b, invd, xi, xo, L.d.p, (float)c1[k], (float)c2[k], nullptr);
            if (l == 0) rec_step(false);
            std::swap(xi, xo);
        }
        xout[l] = xi;
        if (l == 0 && tma0)
            launch_fine<kFineResid>(n_done, n_inst, b, nullptr, xi, L.r.p, nullptr, 0.f, 0.f, 0.f, s);
        else
            residual_kernel(L.g)<<<gs, 256, 0, s>>>(gate_, A, b, xi, L.r.p);
        long_rows(L.A, 1, b, nullptr, xi, L.r.p, nullptr, 0.f, 0.f, nullptr);
        AmgLevel &C = lv_[l + 1];
        const float *wt = l == 0 ? w0_used_ : nullptr;
        if (l + 2 < nl) {
            std::vector<double> cc1, cc2;
            cheb_coeffs(C, cc1, cc2);
            k_restrict_first<<<nblk(C.A.n, 256), 256, 0, s>>>(gate_, L.nc, C.A.n, L.mem_start.p, L.mem_rows.p, L.r.p, wt,
                                                              C.inv_diag.p, (float)cc2[0], C.b.p, C.xa.p, C.d.p,
                                                              C.agg.p);
        } else {
            k_restrict<<<nblk(C.A.n, 256), 256, 0, s>>>(gate_, L.nc, C.A.n, L.mem_start.p, L.mem_rows.p, L.r.p, C.b.p, wt);
        }
    }
    // coarsest: dense inverse, or (when coarsening stalled above the dense limit) a Chebyshev
    // polynomial of degree coarse_degree on a wide interval
    if (use_tail) {
        AMG_CK(launch_tail(n_done, n_inst, s));
        xout[tail_level_] = tail_out_;
    } else {
        AmgLevel &Lc = lv_[nl - 1];
        const float *b = nl == 1 ? r : Lc.b.p;
        if (dense_n_ > 0) {
            float *x = nl == 1 ? z : Lc.xa.p;
            k_dense_gemv<<<nblk(Lc.A.n * 32, 256), 256, 0, s>>>(gate_, dense_inv_.p, dense_n_, Lc.A.n, b, x);
            xout[nl - 1] = x;
        } else {
            const unsigned g = nblk(Lc.A.n, 256), gs = row_blocks(Lc);
            const auto sm_step = sm_step_kernel(Lc.g);
            cheb_coeffs(Lc, c1, c2, std::max(1, opt_.coarse_degree), opt_.coarse_ratio);
            float *xi = Lc.xa.p, *xo = Lc.xb.p;
            k_sm_first<<<g, 256, 0, s>>>(gate_, Lc.A.n, b, Lc.inv_diag.p, (float)c2[0], xi, Lc.d.p, Lc.agg.p);
            const int cdeg = std::max(1, opt_.coarse_degree);
            for (int k = 1; k < cdeg; ++k) {
                float *xk = (nl == 1 && k == cdeg - 1) ? z : xo;
                sm_step<<<gs, 256, 0, s>>>(gate_, view(Lc.A), b, Lc.inv_diag.p, xi, xk, Lc.d.p, (float)c1[k],
                                           (float)c2[k], Lc.agg.p);
                long_rows(Lc.A, 0, b, Lc.inv_diag.p, xi, xk, Lc.d.p, (float)c1[k], (float)c2[k], nullptr);
                xo = xi;
                xi = xk;
            }
            xout[nl - 1] = xi;
        }
    }
    // ascend: prolong, smooth
    for (int l = use_tail ? tail_level_ - 1 : nl - 2; l >= l0; --l) {
        AmgLevel &L = lv_[l];
        const float *b = l == 0 ? r : L.b.p;
        const float *invd = l == 0 ? fw() : L.inv_diag.p;
        MatView A = view(L.A);
        if (l == 0 && opt_.half_fine) A.hval = reinterpret_cast<const __half *>(fine_half_.p);
        const unsigned g = nblk(L.A.n, 256), gs = row_blocks(L);
        const auto sm_step = sm_step_kernel(L.g);
        cheb_coeffs(L, c1, c2);
        float *xi = xout[l];
        const double *al = nullptr;
        // (a dense coarsest correction is exact: its optimal scaling is 1)
        if (opt_.kcycle && l < opt_.kcycle_levels && (l + 2 < nl || dense_n_ == 0) && use_tail &&
            l == tail_level_ - 1) {
            al = alpha_.p + l;  // the tail's last phase
        } else if (opt_.kcycle && l < opt_.kcycle_levels && (l + 2 < nl || dense_n_ == 0)) {
            AmgLevel &C = lv_[l + 1];
            double *lp = dots_long_.p + dots_long_off_[l];
            long_rows(C.A, 2, C.b.p, nullptr, xout[l + 1], nullptr, nullptr, 0.f, 0.f, lp);
            coarse_dots_kernel(C.g)<<<row_blocks(C), 256, 0, s>>>(gate_, view(C.A), xout[l + 1], C.b.p,
                                                                  dots_.p + dots_off_[l], tickets_.p + l,
                                                                  alpha_.p + l, lp, (int32_t)C.A.n_long);
            al = alpha_.p + l;
        }
        k_prolong<<<g, 256, 0, s>>>(gate_, L.A.n, L.agg.p, xout[l + 1], xi, al, opt_.alpha, l == 0 ? w0_used_ : nullptr);
        float *other = xi == L.xa.p ? L.xb.p : L.xa.p;
        for (int k = 0; k < deg; ++k) {
            float *xo = (l == 0 && k == deg - 1) ? z : other;
            if (l == 0) rec_step(true);
            if (l == 0 && tma0)
                launch_fine<kFineStep>(n_done, n_inst, b, invd, xi, xo, L.d.p, 0.f, k == 0 ? 0.f : (float)c1[k],
                                       (float)c2[k], s);
            else
                sm_step<<<gs, 256, 0, s>>>(gate_, A, b, invd, xi, xo, L.d.p, k == 0 ? 0.f : (float)c1[k],
                                           (float)c2[k], L.agg.p);
            long_rows(L.A, 0, b, invd, xi, xo, L.d.p, k == 0 ? 0.f : (float)c1[k], (float)c2[k], nullptr);
            if (l == 0) rec_step(false);
            other = xi;
            xi = xo;
        }
        xout[l] = xi;
    }
    if (prof) rec(prof->cycle[1]);
    if (l0 == 0) last_long_launches_ = launches;
    if (x_l0) *x_l0 = xout[l0];
    return cudaGetLastError();
}

cudaError_t Amg::coarse_correct(const float *v, float *out, cudaStream_t s) {
    const int64_t n = lv_[0].A.n;
    AMG_CK(cudaMemsetAsync(out, 0, n * sizeof(float), s));
    if (n_levels_ < 2) return cudaSuccess;
    AmgLevel &L0 = lv_[0], &C = lv_[1];
    const Gate g{nullptr, 0};
    k_restrict<<<nblk(C.A.n, 256), 256, 0, s>>>(g, L0.nc, C.A.n, L0.mem_start.p, L0.mem_rows.p, v, C.b.p, w0_used_);
    AMG_CK(cudaGetLastError());
    float *xc = nullptr;
    cudaError_t e = cycle(1, nullptr, nullptr, nullptr, 0, s, nullptr, &xc);
    if (e != cudaSuccess) return e;
    k_prolong<<<nblk(n, 256), 256, 0, s>>>(g, n, L0.agg.p, xc, out, nullptr, 1.f, w0_used_);
    return cudaGetLastError();
}

cudaError_t Amg::smooth_fine(const float *b, float *x, cudaStream_t s) {
    AmgLevel &L = lv_[0];
    std::vector<double> c1, c2;
    cheb_coeffs(L, c1, c2);
    const int pre = pre_degree();
    const float *invd = fw();
    MatView A = view(L.A);
    if (opt_.half_fine) A.hval = reinterpret_cast<const __half *>(fine_half_.p);
    const int32_t *agg = n_levels_ > 1 ? L.agg.p : nullptr;
    const Gate g{nullptr, 0};
    float *xi = L.xa.p, *xo = L.xb.p;
    k_sm_first<<<nblk(L.A.n, 256), 256, 0, s>>>(g, L.A.n, b, invd, (float)c2[0], xi, L.d.p, agg);
    const auto sm_step = sm_step_kernel(L.g);
    for (int k = 1; k < pre; ++k) {
        sm_step<<<row_blocks(L), 256, 0, s>>>(g, A, b, invd, xi, xo, L.d.p, (float)c1[k], (float)c2[k], agg);
        std::swap(xi, xo);
    }
    AMG_CK(cudaGetLastError());
    AMG_CK(cudaMemcpyAsync(x, xi, L.A.n * sizeof(float), cudaMemcpyDeviceToDevice, s));
    return cudaSuccess;
}

bool Amg::fine_poly(double &a0, double &a1) const {
    if (n_levels_ < 1 || pre_degree() != 2) return false;
    std::vector<double> c1, c2;
    cheb_coeffs(lv_[0], c1, c2);
    a0 = c2[0] * (1.0 + c1[1]) + c2[1];
    a1 = -c2[1] * c2[0];
    return true;
}

}  // namespace mh
