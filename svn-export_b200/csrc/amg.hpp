// Aggregation multigrid preconditioner for the Jacobi-scaled edge system (FP32), built and
// applied on the GPU.  No counterpart in the reference, which preconditions the Schur system
// with PETSc ILU (src/la/solve.cc:370); it is the preconditioner of the MH_SOLVER_AMG solve.
//
// Setup (every solve, from the current matrix values):
//   level l -> l+1 by repeated pairwise aggregation: passes of handshake matching on the
//   strongest negative coupling -a_ij / sqrt(a_ii a_jj), each followed by the Galerkin product
//   A_c = P^T A P with the piecewise-constant P of the pairs; rows without off-diagonal
//   coupling (Dirichlet edges, padding) stay on the fine level only.  The fine level is the
//   Jacobi-scaled S^ = D^-1/2 S D^-1/2, whose near-null vector is D^1/2 1, so its transfers
//   carry the weights sqrt(diag S): P_0 = W P, and A_1 = P^T S P in the unscaled space.
//   Coarse matrices are stored as SELL-32 like the fine one; their rows are built by one warp each (gather,
//   bitonic sort by column, deterministic segmented sum).  The coarsest level (<= coarse_max
//   rows) is inverted densely in FP64 (in-place Gauss-Jordan in shared memory, one block); if
//   coarsening stalls above that size, the coarsest level gets a degree-12 Chebyshev polynomial.
// Apply (one V-cycle, FP32): Chebyshev smoothing of degree d on [hi/ratio, hi] of D^-1 A
// before and after the coarse correction (symmetric, so the cycle is an SPD operator).
#pragma once
#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "device_system.hpp"

namespace mh {

struct AmgOptions {
    int max_levels = 20;
    int coarse_max = 160;   // dense coarsest solve at or below this many rows (<= 160)
    int pair_rounds = 4;    // handshake rounds per pairing pass
    int pair_passes = 2;    // pairing passes from the fine level (2: aggregates of up to 4 rows)
    int pair_passes_coarse = 3;  // ... from the coarser levels (aggregates of up to 8)
    int cheb_degree = 2;    // smoothing steps after the coarse correction (and before, unless
    int pre_degree = 0;     // pre_degree > 0 sets a different number of steps before it)
    float cheb_ratio = 4.f; // smoothing interval [hi / ratio, hi]
    int kcycle = 1;         // 1: scale each coarse correction by its energy-optimal factor
    int kcycle_levels = 6;  // ... on the corrections of the first kcycle_levels levels
    float alpha = 1.f;      // fixed scaling of the coarse corrections when kcycle = 0
    int weighted = 1;       // level-0 transfers weighted by sqrt(diag S) (near-null vector)
    int mix_coarse = 1;     // coarse levels may pair along positive couplings (weakly preferred)
    int split = 0;          // warps per slice in the coarse row kernels (1, 2, 4, 8; 0: by row width)
    int split_width = 12;   // ... by row width: the fewest warps with at most this many slots each
    int half_fine = 1;      // 1: the cycle reads the fine matrix's values in FP16 (a copy made at setup)
    int power_steps = 12;   // power-iteration steps estimating lambda_max(D^-1 A) per level (0: the
                            // Gershgorin bound alone)
    float power_safety = 1.1f;  // smoothing interval top = min(Gershgorin, safety * estimate)
    int coarse_degree = 12;     // Chebyshev degree of a smoothed (not inverted) coarsest level
    float coarse_ratio = 50.f;  // ... on [hi / coarse_ratio, hi]
    int stall_rows = 32768; // after two coarsenings in a row that kept more than half of the rows, a
                            // next level of at most this many rows is the coarsest (0: off)
    int fine_tma = 0;       // 1: the fine level's cycle kernels stream the matrix through shared
                            // memory with TMA bulk copies (with half_fine; amg.cu k_fine_tma)
    int fine_tma_stages = 4;  // ... in a ring of 2 or 4 stages
    int tail_rows = 0;      // levels (below the fine one) from which every level has at most this
                            // many rows run in one cluster launch (0: every level on its own)
};

template <class T> struct DBuf {
    T *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n);  // grows (contents lost), never shrinks
    void release();
};

struct AmgMatrix {
    int64_t n = 0, n_slices = 0, slots = 0;
    const int64_t *slice_off = nullptr;
    const int32_t *col = nullptr;
    const float *val = nullptr;
    const int32_t *rlen = nullptr;      // entries per row (coarse matrices; null on the fine level)
    const int32_t *longrows = nullptr;  // rows with more than kLongRow entries (amg.cu)
    const int32_t *long_count = nullptr;  // their count, on the device (longrows[-1])
    int64_t n_long = 0;                 // ... on the host, once the setup has read it
};

struct AmgLevel {
    AmgMatrix A;                               // level 0 borrows the solver's SELL matrix
    DBuf<int64_t> slice_off;                   // owned storage of coarse levels
    DBuf<int32_t> col;
    DBuf<float> val;
    DBuf<float> inv_diag;
    DBuf<int32_t> rlen, longrows;              // row lengths and long rows of coarse levels
    DBuf<int32_t> agg;                         // [n] coarse row of each row, -1: none
    DBuf<int32_t> mem_start, mem_rows;         // rows of each coarse row: [nc+1], [n]
    DBuf<float> b, xa, xb, d, r;               // cycle vectors
    int64_t nc = 0;                            // coarse rows (0 on the coarsest level)
    float hi = 2.f;                            // top of the smoothing interval: the power-iteration
                                               // estimate of lambda_max(D^-1 A) times a safety
                                               // factor, at most the Gershgorin bound
    float gershgorin = 2.f;                    // Gershgorin bound of D^-1 A
    int g = 1;                                 // warps per slice in the row kernels (amg.cu)
};

// Events recorded inside a captured V-cycle (as external event nodes) to time it: the whole
// cycle, and each Chebyshev smoothing step of the fine level (start/end pairs).
struct AmgProf {
    cudaEvent_t cycle[2] = {nullptr, nullptr};
    std::vector<cudaEvent_t> smooth;
};

class Amg {
public:
    ~Amg() { release(); }
    // Builds the hierarchy from the FP32 scaled matrix (sys.val32) and sys.row_edge.
    cudaError_t setup(const DevSystem &sys, const AmgOptions &o, cudaStream_t s);
    // z = M r over all rows of the solver space (one V-cycle); stream-ordered, capturable.
    // The kernels do nothing once *n_done >= n_inst (n_done may be null).
    // With prof, events are recorded around the cycle and its fine-level smoothing steps.
    cudaError_t apply(const float *r, float *z, const int32_t *n_done, int32_t n_inst, cudaStream_t s,
                      AmgProf *prof = nullptr);
    // smoothing steps on the fine level per cycle (none when the fine level is the coarsest)
    int fine_steps() const { return n_levels_ > 1 ? pre_degree() - 1 + std::max(1, opt_.cheb_degree) : 0; }
    int pre_degree() const { return opt_.pre_degree > 0 ? opt_.pre_degree : std::max(1, opt_.cheb_degree); }
    int cheb_degree() const { return std::max(1, opt_.cheb_degree); }
    void release();
    int levels() const { return n_levels_; }
    const AmgLevel &level(int l) const { return lv_[l]; }
    int64_t coarse_rows() const { return n_levels_ ? lv_[n_levels_ - 1].A.n : 0; }
    // the first level of the coarse tail run as one cluster launch (0: none) and its CTAs
    int tail_level() const { return tail_phases_ > 0 ? tail_level_ : 0; }
    // the fine level's kernels stream the matrix with TMA; a stage wait that timed out (read
    // back and cleared: the cycle's results are then not usable)
    bool fine_tma() const { return fine_tma_; }
    bool fine_tma_failed(cudaStream_t s);
    int tail_cluster() const { return tail_cluster_; }
    int kernels_per_apply() const;
    const float *fine_weights() const { return w0_used_; }  // null when the transfers are unweighted
    // Per-row weights of the fine level's smoother (device array over the solver rows, owned by
    // the caller; null: none): the fine level is then smoothed with Chebyshev on Omega S^
    // instead of S^.  Takes effect at the next setup, or at refresh_fine for the current
    // hierarchy (the fine level's interval is re-estimated for the new weights).
    void set_fine_weights(const float *w) { fine_w_ = w; }
    const float *fine_smoother_weights() const { return fine_w_; }
    // the weights the cycle uses (1 on the rows outside the hierarchy), null when none are set
    const float *fine_smoother_weights_in_effect() const { return fw(); }
    cudaError_t refresh_fine(cudaStream_t s);
    // new values in the weights array, the smoothing interval kept as it is
    cudaError_t update_fine_weights(cudaStream_t s) { return fine_weights_eff(s); }
    // Parts of the cycle for training the fine smoother (the cycle is linear when kcycle = 0):
    //   coarse_correct: out = P B P^T v (restriction with the level-0 weights, the cycle of the
    //                   coarser levels B, prolongation), out over the fine rows;
    //   smooth_fine:    x = Q b, the fine level's smoothing from zero (Q = q(Omega S^) Omega);
    //   fine_poly:      Q = a0 Omega + a1 Omega S^ Omega for the degree-2 smoother (false for
    //                   other degrees).
    cudaError_t coarse_correct(const float *v, float *out, cudaStream_t s);
    cudaError_t smooth_fine(const float *b, float *x, cudaStream_t s);
    bool fine_poly(double &a0, double &a1) const;
    const AmgOptions &options() const { return opt_; }
    float level_hi(int l) const { return lv_[l].hi; }
    bool half_fine() const { return opt_.half_fine != 0; }
    std::string err;

private:
    cudaError_t pair_pass(const AmgMatrix &A, const float *inv_diag, const int32_t *exclude_row_edge,
                          DBuf<int32_t> &agg, int64_t &nc, DBuf<int32_t> &mstart, DBuf<int32_t> &mrows, cudaStream_t s);
    cudaError_t galerkin(const AmgMatrix &A, const int32_t *agg, int64_t nc, const int32_t *mstart,
                         const int32_t *mrows, DBuf<int64_t> &c_off, DBuf<int32_t> &c_col, DBuf<float> &c_val,
                         DBuf<int32_t> &c_rlen, DBuf<int32_t> &c_long, AmgMatrix &C, cudaStream_t s,
                         const float *wt);
    cudaError_t level_stats(AmgLevel &L, unsigned int *bound, cudaStream_t s);
    cudaError_t dense_coarse(const AmgMatrix &A, cudaStream_t s);
    // lambda_max estimates of D^-1 A on every level but the coarsest (power iteration from a
    // fixed pseudo-random start; deterministic sums), as |v_k|^2 and |v_{k-1}|^2 per level
    cudaError_t power_estimates(cudaStream_t s, int only_level = -1);
    cudaError_t cycle(int l0, const float *r, float *z, const int32_t *n_done, int32_t n_inst, cudaStream_t s,
                      AmgProf *prof, float **x_l0);
    cudaError_t scan_i32(const int32_t *in, int32_t *out, int64_t n, int64_t &total, cudaStream_t s);
    cudaError_t scan_i64(const int64_t *in, int64_t *out, int64_t n, int64_t &total, cudaStream_t s);
    // the same without reading the total back (out[n] holds it on the device)
    cudaError_t scan_i32_dev(const int32_t *in, int32_t *out, int64_t n, cudaStream_t s);
    cudaError_t scan_i64_dev(const int64_t *in, int64_t *out, int64_t n, cudaStream_t s);
    void cheb_coeffs(const AmgLevel &L, std::vector<double> &c1, std::vector<double> &c2, int degree = 0,
                     float ratio = 0.f) const;

    AmgOptions opt_;
    std::vector<AmgLevel> lv_;
    int n_levels_ = 0;
    // pairing and Galerkin scratch
    DBuf<int32_t> mate_, want_, cid_, tmp_agg_, tmp_ms_, tmp_mr_, cnt_;
    DBuf<int64_t> packed_, pscan_;  // pairing: packed (leader, member count) and its scan
    DBuf<unsigned int> bounds_;     // Gershgorin bound of each level (float bits)
    DBuf<int64_t> width_, scan64_;
    DBuf<int32_t> rowlen_, scan32_blk_;
    DBuf<int64_t> scan64_blk_;
    DBuf<int64_t> mid_off_[2];      // intermediate matrices of the pairing passes
    DBuf<int32_t> mid_col_[2];
    DBuf<float> mid_val_[2];
    DBuf<float> mid_invd_;
    DBuf<int32_t> mid_rlen_[2], mid_long_[2];
    DBuf<int32_t> lflag_, lpos_;    // long-row list construction
    DBuf<int32_t> big_list_, big_count_;  // Galerkin rows that need the large gather buffer
    DBuf<int64_t> tbound_, toff_;         // compact Galerkin rows: candidate bounds, offsets
    DBuf<int32_t> tcol_;
    DBuf<float> tval_;
    DBuf<double> dots_long_;        // long rows' terms of the coarse-correction scaling
    std::vector<int64_t> dots_long_off_;
    int last_long_launches_ = 0;
    DBuf<float> isd_;
    DBuf<float> dense_inv_;
    DBuf<int32_t> flag_;
    DBuf<unsigned int> bound_;
    DBuf<double> dots_, alpha_;     // coarse-correction scaling: partials, factor per level
    DBuf<unsigned int> tickets_;    // last-block tickets of the scaling reductions, per level
    std::vector<int64_t> dots_off_;
    const float *fine_w_ = nullptr;  // fine-level smoother weights (set_fine_weights)
    DBuf<float> fine_w_eff_;         // ... with 1 on the rows outside the hierarchy (solved exactly)
    const float *fw() const { return fine_w_ ? fine_w_eff_.p : nullptr; }
    cudaError_t fine_weights_eff(cudaStream_t s);
    cudaError_t fine_interval(cudaStream_t s);  // level 0's bound for the weights
    DBuf<float> pw_a_, pw_b_;       // power-iteration vectors
    DBuf<double> pw_part_, pw_sums_;  // its per-block partial norms and the two norms per level
    DBuf<float> w0_;                // sqrt(diag S) per fine row
    DBuf<uint16_t> fine_half_;      // FP16 bits of the fine matrix's values (half_fine)
    // the fine level's TMA-staged cycle kernels (k_fine_tma): ready, stage size, grid, the
    // widest tile read at setup and the stage-wait error flag
    bool fine_tma_ = false;
    int fine_stages_ = 4;
    int32_t fine_stage_slots_ = 0;
    int fine_tma_grid_ = 0;
    DBuf<unsigned int> tile_max_;
    DBuf<int32_t> tma_err_;
    cudaError_t prepare_fine_tma(unsigned int widest, cudaStream_t s);
    template <int MODE>
    void launch_fine(const int32_t *n_done, int32_t n_inst, const float *b, const float *invd, const float *x_in,
                     float *x_out, float *d, float c0, float c1, float c2, cudaStream_t s) const;
    // the coarse tail: levels tail_level_ .. coarsest of the cycle from level 0 as one cluster
    // launch running a list of phases (amg.cu, k_tail)
    cudaError_t build_tail(cudaStream_t s);
    cudaError_t launch_tail(const int32_t *n_done, int32_t n_inst, cudaStream_t s) const;
    int tail_level_ = 0;            // 0: no tail
    int tail_cluster_ = 0;          // CTAs of the cluster
    int tail_phases_ = 0;
    int tail_regular_ = 0;          // row kernels (not long-row ones) the tail stands in for
    float *tail_out_ = nullptr;     // the tail's result: x of level tail_level_
    int64_t tail_long_off_ = 0;     // long-row terms' offset in the scratch
    DBuf<unsigned char> tail_prog_, tail_levels_;
    DBuf<double> tail_scratch_;
    const float *w0_used_ = nullptr;
    int64_t dense_n_ = 0;
    int32_t *h_flag_ = nullptr;
};

}  // namespace mh
