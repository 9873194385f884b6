/*
 * linsys_cuda.hh -- C++ drop-ins for Flow123d's LinSys and DarcyFlowMH_Steady over the C ABI
 * of mh_darcy.h (header-only; link libmhdarcy.so).  No PETSc, no MPI: one process, one GPU.
 *
 * LinSys_CUDA mirrors the assembly interface of the abstract LinSys (src/la/linsys.hh:63-222):
 * the same method names, int / double* arguments and the ALLOCATE -> ADD|INSERT -> DONE
 * protocol of SetValuesMode (:66-72, :129-139):
 *   - start_allocation(): mat_set_values only records the pattern (preallocate_values);
 *     rhs_set_values does nothing (:147-156);
 *   - start_add_assembly() / start_insert_assembly(): the recorded pattern becomes the matrix
 *     (preallocate_matrix), its values start at zero, and mat_set_values / rhs_set_values add
 *     or insert (MatSetValues / VecSetValues with ADD_VALUES / INSERT_VALUES);
 *   - finalize(): the values go to the device (MatAssemblyBegin/End);
 *   - solve(): the solve that src/la/solve.cc:175-209 does with PETSc KSP (the proposed
 *     interface's `virtual int solve()`, src/la/linsys_proposed.hh:260), here any MH_SOLVER_*
 *     method of mh_solve on the GPU; the solution lands in the solution array (the one given
 *     to the constructor, as LinSys(lsize, sol_array), or an owned one).
 * set_symmetric / set_positive_definite keep the reference's coupling (:169-186); solve()
 * requires a symmetric positive definite system.  An entry outside the allocated pattern, a row
 * or column out of range, or a call in a state the reference disallows is recorded as an error
 * (error(), error_message()) and makes finalize() and solve() return MH_ERR_STATE or
 * MH_ERR_INVALID instead of aborting as the reference's ASSERT / xprintf(Err) would.
 *
 * DarcyFlowMH_Steady_CUDA is the seam of the steady MH flow: its constructor builds the mesh
 * topology as DarcyFlowMH_Steady's does (mh_create: Mesh::make_neighbours_and_edges,
 * src/mesh/mesh.cc:343-500), update_solution() replaces the n_schurs == 2 branch of
 * DarcyFlowMH_Steady::update_solution (src/flow/darcy_flow_mh.cc:407-416: make_schur1,
 * make_schur2, solve_system, resolve x2) with mh_assemble + mh_solve, and
 * get_solution_vector() / the MH_DofHandler accessors (src/flow/mh_dofhandler.cc:37-50) read
 * the solution in the reference's [side fluxes | element pressures | edge pressures] layout.
 */
#ifndef LINSYS_CUDA_HH
#define LINSYS_CUDA_HH

#include <algorithm>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "mh_darcy.h"

class LinSys_CUDA {
public:
    typedef enum { INSERT, ADD, ALLOCATE, DONE, NONE } SetValuesMode;

    /// A system of `lsize` unknowns; the solution is written to sol_array when given (not
    /// owned), else to an owned array (LinSys::LinSys, src/la/linsys.cc:55-61).
    explicit LinSys_CUDA(unsigned int lsize, double *sol_array = NULL)
        : n_(lsize), status_(NONE), symmetric_(false), positive_definite_(false), rows_(lsize), rhs_(lsize, 0.0),
          own_solution_(sol_array ? 0 : lsize, 0.0), solution_(sol_array ? sol_array : own_solution_.data()) {}
    ~LinSys_CUDA() {
        if (h_) mh_destroy(h_);
    }
    LinSys_CUDA(const LinSys_CUDA &) = delete;
    LinSys_CUDA &operator=(const LinSys_CUDA &) = delete;

    unsigned int size() const { return n_; }
    unsigned int vec_lsize() const { return n_; }

    void start_allocation() {
        if (status_ != NONE) fail(MH_ERR_STATE, "start_allocation after the matrix was allocated");
        status_ = ALLOCATE;
    }
    /// Records the pattern of a dense nrow x ncol block (LinSys_MPIAIJ::preallocate_values).
    void preallocate_values(int nrow, int *rows, int ncol, int *cols) {
        for (int i = 0; i < nrow; ++i) {
            if (!row_ok(rows[i])) continue;
            for (int j = 0; j < ncol; ++j)
                if (col_ok(cols[j])) rows_[rows[i]].push_back(cols[j]);
        }
    }
    /// Turns the recorded pattern into the matrix (every row also holds its diagonal).
    void preallocate_matrix() {
        row_ptr_.assign(n_ + 1, 0);
        col_.clear();
        for (unsigned int r = 0; r < n_; ++r) {
            std::vector<int32_t> &c = rows_[r];
            c.push_back((int32_t)r);
            std::sort(c.begin(), c.end());
            c.erase(std::unique(c.begin(), c.end()), c.end());
            col_.insert(col_.end(), c.begin(), c.end());
            row_ptr_[r + 1] = (int32_t)col_.size();
            std::vector<int32_t>().swap(c);
        }
        val_.assign(col_.size(), 0.0);
        if (h_) {
            mh_destroy(h_);
            h_ = NULL;
        }
        const int rc = mh_csr_create((int64_t)n_, row_ptr_.data(), col_.data(), &h_);
        if (rc < 0) fail(rc, "mh_csr_create failed");
    }
    void start_add_assembly() { start_assembly(ADD); }
    void start_insert_assembly() { start_assembly(INSERT); }
    /// End of an assembly pass: the values go to the device.  Returns a status code.
    int finalize() {
        if (status_ != ADD && status_ != INSERT) return fail(MH_ERR_STATE, "finalize outside an assembly pass");
        if (error_) return error_;
        status_ = DONE;
        if (!h_) return fail(MH_ERR_STATE, "no matrix");
        const int rc = mh_csr_set_values(h_, val_.data(), rhs_.data());
        if (rc < 0) return fail(rc, mh_last_error(h_));
        return MH_OK;
    }

    /// Sets (or adds, by the assembly mode) a dense nrow x ncol block, row-major
    /// (LinSys::mat_set_values, linsys.hh:129-139).
    void mat_set_values(int nrow, int *rows, int ncol, int *cols, double *vals) {
        switch (status_) {
            case ALLOCATE: preallocate_values(nrow, rows, ncol, cols); break;
            case INSERT:
            case ADD:
                for (int i = 0; i < nrow; ++i) {
                    if (!row_ok(rows[i])) continue;
                    for (int j = 0; j < ncol; ++j) {
                        const int64_t k = slot(rows[i], cols[j]);
                        if (k < 0) {
                            fail(MH_ERR_INVALID, "entry outside the allocated pattern");
                            continue;
                        }
                        if (status_ == ADD) val_[k] += vals[(int64_t)i * ncol + j];
                        else val_[k] = vals[(int64_t)i * ncol + j];
                    }
                }
                break;
            default: fail(MH_ERR_STATE, "mat_set_values outside allocation or assembly");
        }
    }
    void mat_set_value(int row, int col, double val) { mat_set_values(1, &row, 1, &col, &val); }
    /// Right-hand side values (LinSys::rhs_set_values, linsys.hh:147-156).
    void rhs_set_values(int nrow, int *rows, double *vals) {
        switch (status_) {
            case ALLOCATE: break;
            case INSERT:
            case ADD:
                for (int i = 0; i < nrow; ++i) {
                    if (!row_ok(rows[i])) continue;
                    if (status_ == ADD) rhs_[rows[i]] += vals[i];
                    else rhs_[rows[i]] = vals[i];
                }
                break;
            default: fail(MH_ERR_STATE, "rhs_set_values outside allocation or assembly");
        }
    }
    void rhs_set_value(int row, double val) { rhs_set_values(1, &row, &val); }
    void set_values(int nrow, int *rows, int ncol, int *cols, double *mat_vals, double *rhs_vals) {
        mat_set_values(nrow, rows, ncol, cols, mat_vals);
        rhs_set_values(nrow, rows, rhs_vals);
    }

    void set_symmetric(bool flag = true) {
        symmetric_ = flag;
        if (!flag) set_positive_definite(false);
    }
    bool is_symmetric() const { return symmetric_; }
    void set_positive_definite(bool flag = true) {
        positive_definite_ = flag;
        if (flag) set_symmetric();
    }
    bool is_positive_definite() const { return positive_definite_; }
    bool is_new() const { return status_ == NONE; }
    bool is_preallocated() const { return status_ == INSERT || status_ == ADD; }

    /// Solves the finalized system on the GPU (opts: NULL for mh_solve_opts_default with the
    /// reference's r_tol 1e-10 semantics of mh_solve).  Returns mh_solve's status; the stats of
    /// the last solve are in last_stats().
    int solve(const mh_solve_opts *opts = NULL) {
        if (error_) return error_;
        if (status_ != DONE || !h_) return fail(MH_ERR_STATE, "solve before finalize");
        if (!positive_definite_) return fail(MH_ERR_STATE, "solve needs set_positive_definite()");
        mh_solve_opts o;
        mh_solve_opts_default(&o);
        if (opts) o = *opts;
        int rc = mh_solve(h_, &o, &stats_);
        if (rc < 0) return fail(rc, mh_last_error(h_));
        const int rg = mh_csr_get_solution(h_, solution_, n_);
        if (rg < 0) return fail(rg, mh_last_error(h_));
        return stats_.status;
    }

    double *get_solution_array() { return solution_; }
    const std::vector<double> &get_rhs_array() const { return rhs_; }
    const mh_solve_stats &last_stats() const { return stats_; }
    /// The assembled matrix in CSR form (after start_add_assembly / start_insert_assembly).
    const std::vector<int32_t> &csr_row_ptr() const { return row_ptr_; }
    const std::vector<int32_t> &csr_col() const { return col_; }
    const std::vector<double> &csr_val() const { return val_; }
    SetValuesMode status() const { return status_; }
    int error() const { return error_; }
    const std::string &error_message() const { return msg_; }

private:
    bool row_ok(int r) {
        if (r >= 0 && (unsigned)r < n_) return true;
        fail(MH_ERR_INVALID, "row index out of range");
        return false;
    }
    bool col_ok(int c) {
        if (c >= 0 && (unsigned)c < n_) return true;
        fail(MH_ERR_INVALID, "column index out of range");
        return false;
    }
    int64_t slot(int r, int c) const {
        const int32_t *b = col_.data() + row_ptr_[r], *e = col_.data() + row_ptr_[r + 1];
        const int32_t *p = std::lower_bound(b, e, (int32_t)c);
        return (p != e && *p == c) ? (int64_t)(p - col_.data()) : -1;
    }
    void start_assembly(SetValuesMode mode) {
        if (status_ == ALLOCATE) preallocate_matrix();
        else if (status_ == NONE) fail(MH_ERR_STATE, "assembly before start_allocation");
        else if (status_ == DONE) {  // a new pass on the same pattern starts from zero (MatZeroEntries)
            std::fill(val_.begin(), val_.end(), 0.0);
            std::fill(rhs_.begin(), rhs_.end(), 0.0);
        }
        status_ = mode;
    }
    int fail(int code, const char *what) {
        if (!error_) {
            error_ = code;
            msg_ = what ? what : "";
        }
        return code;
    }

    unsigned int n_;
    SetValuesMode status_;
    bool symmetric_, positive_definite_;
    std::vector<std::vector<int32_t>> rows_;  // pattern recorded during allocation
    std::vector<int32_t> row_ptr_, col_;
    std::vector<double> val_, rhs_;
    std::vector<double> own_solution_;
    double *solution_;
    mh_handle *h_ = NULL;
    mh_solve_stats stats_ = {};
    int error_ = 0;
    std::string msg_;
};

/// The steady mixed-hybrid Darcy flow on the GPU behind the reference's class seam.
class DarcyFlowMH_Steady_CUDA {
public:
    /// Builds the topology of the mesh (edges, boundary objects, VB neighbours) and the edge
    /// system's layout; status() is MH_OK or the mh_create error.
    explicit DarcyFlowMH_Steady_CUDA(const mh_mesh_desc &mesh) { status_ = mh_create(&mesh, &h_); }
    ~DarcyFlowMH_Steady_CUDA() {
        if (h_) mh_destroy(h_);
    }
    DarcyFlowMH_Steady_CUDA(const DarcyFlowMH_Steady_CUDA &) = delete;
    DarcyFlowMH_Steady_CUDA &operator=(const DarcyFlowMH_Steady_CUDA &) = delete;

    int status() const { return status_; }
    mh_handle *handle() { return h_; }
    mh_sizes sizes() const {
        mh_sizes z = {};
        if (h_) mh_get_sizes(h_, &z);
        return z;
    }
    /// Element fields and boundary data (EqData, darcy_flow_mh.cc:154-183; one entry per
    /// boundary object in the topology's order).
    int set_data(const mh_coeffs &c, const mh_bc &bc) {
        int rc = mh_set_coeffs(h_, &c);
        if (rc >= 0) rc = mh_set_bc(h_, &bc);
        return rc;
    }
    /// Assembly, both Schur eliminations, the solve of the edge system and the
    /// back-substitution (darcy_flow_mh.cc:407-416).  Returns mh_solve's status.
    int update_solution(const mh_solve_opts *opts = NULL) {
        if (!h_) return status_;
        int rc = mh_assemble(h_);
        if (rc < 0) return rc;
        mh_solve_opts o;
        mh_solve_opts_default(&o);
        if (opts) o = *opts;
        rc = mh_solve(h_, &o, &stats_);
        if (rc < 0) return rc;
        solution_.resize(sizes().mh_size);
        const int rg = mh_get_solution(h_, solution_.data(), (int64_t)solution_.size());
        return rg < 0 ? rg : stats_.status;
    }
    /// The MH solution [side fluxes | element pressures | edge pressures]
    /// (DarcyFlowMH_Steady::get_solution_vector, darcy_flow_mh.cc:485-500).
    void get_solution_vector(double *&vec, unsigned int &vec_size) {
        vec = solution_.data();
        vec_size = (unsigned int)solution_.size();
    }
    const mh_solve_stats &last_stats() const { return stats_; }

    /// MH_DofHandler accessors (mh_dofhandler.cc:37-50): element e's local side i.
    double side_flux(int64_t e, int i) { return solution_[side_start(e) + i]; }
    double side_scalar(int64_t e, int i) {
        load_topology();
        const mh_sizes z = sizes();
        return solution_[z.n_sides + z.n_elements + side_edge_[el_side_start_[e] + i]];
    }
    double element_scalar(int64_t e) { return solution_[sizes().n_sides + e]; }

private:
    int64_t side_start(int64_t e) {
        load_topology();
        return el_side_start_[e];
    }
    void load_topology() {
        if (!el_side_start_.empty() || !h_) return;
        const mh_sizes z = sizes();
        el_side_start_.resize(z.n_elements + 1);
        side_edge_.resize(z.n_sides);
        mh_get_topology(h_, el_side_start_.data(), side_edge_.data(), NULL, NULL, NULL, NULL, NULL, NULL);
    }

    mh_handle *h_ = NULL;
    int status_ = 0;
    mh_solve_stats stats_ = {};
    std::vector<double> solution_;
    std::vector<int32_t> el_side_start_, side_edge_;
};

#endif /* LINSYS_CUDA_HH */
