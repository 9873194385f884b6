// Compiled C++ caller of include/linsys_cuda.hh, driven by tests/test_linsys_cpp.py.
//
//   linsys_driver linsys <dir> <solve>   LinSys_CUDA: ALLOCATE pass, ADD pass and (solve = 1)
//                                        finalize + GPU solve of the element blocks in
//                                        <dir>/blocks.bin and the right-hand side rhs_in.bin;
//                                        writes the assembled CSR (csr_*.bin, rhs.bin) and the
//                                        solution (x.bin)
//   linsys_driver darcy <dir> <solve>    DarcyFlowMH_Steady_CUDA on the mesh, coefficients and
//                                        boundary data in <dir>; writes sizes.bin and the
//                                        topology, and (solve = 1) the MH solution and the
//                                        MH_DofHandler accessors of every element
//
// Arrays are raw little-endian files, one per array (int32 / int64 / float64).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "linsys_cuda.hh"

template <class T> static std::vector<T> load(const std::string &path) {
    std::vector<T> v;
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return v;
    std::fseek(f, 0, SEEK_END);
    const long bytes = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    v.resize(bytes / sizeof(T));
    if (!v.empty() && std::fread(v.data(), sizeof(T), v.size(), f) != v.size()) v.clear();
    std::fclose(f);
    return v;
}

template <class T> static bool save(const std::string &path, const T *p, size_t n) {
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const bool ok = n == 0 || std::fwrite(p, sizeof(T), n, f) == n;
    std::fclose(f);
    return ok;
}

static int run_linsys(const std::string &dir, bool solve) {
    const std::vector<int64_t> nv = load<int64_t>(dir + "/n.bin");
    const std::vector<char> raw = load<char>(dir + "/blocks.bin");
    if (nv.size() != 1 || raw.empty()) return 2;
    std::vector<double> rhs_in = load<double>(dir + "/rhs_in.bin");
    if ((int64_t)rhs_in.size() != nv[0]) return 2;
    // blocks.bin: per element block int32 m, int32 rows[m], float64 vals[m*m] (row-major)
    struct Block {
        std::vector<int> rows;
        std::vector<double> vals;
    };
    std::vector<Block> blocks;
    size_t pos = 0;
    while (pos < raw.size()) {
        int32_t m;
        std::memcpy(&m, raw.data() + pos, 4);
        pos += 4;
        Block b;
        b.rows.resize(m);
        b.vals.resize((size_t)m * m);
        std::memcpy(b.rows.data(), raw.data() + pos, 4 * (size_t)m);
        pos += 4 * (size_t)m;
        std::memcpy(b.vals.data(), raw.data() + pos, 8 * (size_t)m * m);
        pos += 8 * (size_t)m * m;
        blocks.push_back(std::move(b));
    }
    std::vector<double> x(nv[0], 0.0);
    LinSys_CUDA ls((unsigned)nv[0], x.data());
    ls.set_positive_definite();
    ls.start_allocation();
    for (Block &b : blocks) ls.mat_set_values((int)b.rows.size(), b.rows.data(), (int)b.rows.size(), b.rows.data(),
                                              b.vals.data());
    ls.start_add_assembly();
    for (Block &b : blocks)
        ls.mat_set_values((int)b.rows.size(), b.rows.data(), (int)b.rows.size(), b.rows.data(), b.vals.data());
    // extra_add.bin (optional): int32 row, int32 col, float64 value entries set only in the ADD
    // pass, i.e. outside the allocated pattern unless an element block covered them
    const std::vector<char> extra = load<char>(dir + "/extra_add.bin");
    for (size_t p = 0; p + 16 <= extra.size(); p += 16) {
        int32_t rc[2];
        double v;
        std::memcpy(rc, extra.data() + p, 8);
        std::memcpy(&v, extra.data() + p + 8, 8);
        ls.mat_set_value(rc[0], rc[1], v);
    }
    std::vector<int> all(nv[0]);
    for (int64_t i = 0; i < nv[0]; ++i) all[i] = (int)i;
    ls.rhs_set_values((int)nv[0], all.data(), rhs_in.data());
    save(dir + "/csr_row_ptr.bin", ls.csr_row_ptr().data(), ls.csr_row_ptr().size());
    save(dir + "/csr_col.bin", ls.csr_col().data(), ls.csr_col().size());
    save(dir + "/csr_val.bin", ls.csr_val().data(), ls.csr_val().size());
    save(dir + "/rhs.bin", ls.get_rhs_array().data(), ls.get_rhs_array().size());
    if (ls.error()) {
        std::fprintf(stderr, "LinSys_CUDA: %s\n", ls.error_message().c_str());
        return 3;
    }
    if (!solve) return 0;
    int rc = ls.finalize();
    if (rc < 0) {
        std::fprintf(stderr, "finalize: %d %s\n", rc, ls.error_message().c_str());
        return 4;
    }
    mh_solve_opts o;
    mh_solve_opts_default(&o);
    o.method = MH_SOLVER_PCG64;
    o.r_tol = 1e-12;
    rc = ls.solve(&o);
    const mh_solve_stats &st = ls.last_stats();
    const double info[3] = {(double)rc, (double)st.iterations, st.rel_residual};
    save(dir + "/solve_info.bin", info, 3);
    save(dir + "/x.bin", ls.get_solution_array(), x.size());
    return rc < 0 ? 5 : 0;
}

static int run_darcy(const std::string &dir, bool solve) {
    const std::vector<double> xyz = load<double>(dir + "/nodes.bin");
    const std::vector<int32_t> el_dim = load<int32_t>(dir + "/el_dim.bin"), el_nodes = load<int32_t>(dir + "/el_nodes.bin");
    const std::vector<int32_t> bc_dim = load<int32_t>(dir + "/bc_dim.bin"), bc_nodes = load<int32_t>(dir + "/bc_nodes.bin");
    mh_mesh_desc d = {(int64_t)(xyz.size() / 3), xyz.data(), (int64_t)el_dim.size(), el_dim.data(), el_nodes.data(),
                      (int64_t)bc_dim.size(), bc_dim.empty() ? NULL : bc_dim.data(),
                      bc_dim.empty() ? NULL : bc_nodes.data()};
    DarcyFlowMH_Steady_CUDA flow(d);
    if (flow.status() < 0) {
        std::fprintf(stderr, "mh_create: %d\n", flow.status());
        return 2;
    }
    const mh_sizes z = flow.sizes();
    const int64_t sz[6] = {z.n_elements, z.n_sides, z.n_edges, z.n_boundaries, z.n_neighbours, z.schur_nnz};
    save(dir + "/sizes.bin", sz, 6);
    std::vector<int32_t> ess(z.n_elements + 1), se(z.n_sides), bbc(z.n_boundaries);
    mh_get_topology(flow.handle(), ess.data(), se.data(), NULL, bbc.data(), NULL, NULL, NULL, NULL);
    save(dir + "/el_side_start.bin", ess.data(), ess.size());
    save(dir + "/side_edge.bin", se.data(), se.size());
    save(dir + "/bdr_bc_element.bin", bbc.data(), bbc.size());
    if (!solve) return 0;
    const std::vector<double> K = load<double>(dir + "/conductivity.bin"), A = load<double>(dir + "/anisotropy.bin");
    const std::vector<double> cs = load<double>(dir + "/cross_section.bin"), sg = load<double>(dir + "/sigma.bin");
    const std::vector<double> f = load<double>(dir + "/water_source_density.bin");
    const std::vector<int32_t> bt = load<int32_t>(dir + "/bc_type.bin");
    const std::vector<double> bp = load<double>(dir + "/bc_pressure.bin"), bf = load<double>(dir + "/bc_flux.bin");
    const std::vector<double> br = load<double>(dir + "/bc_robin_sigma.bin");
    mh_coeffs c = {K.data(), A.empty() ? NULL : A.data(), cs.data(), sg.data(), f.data(), NULL};
    mh_bc bc = {bt.data(), bp.data(), bf.data(), br.data()};
    int rc = flow.set_data(c, bc);
    if (rc < 0) {
        std::fprintf(stderr, "set_data: %d\n", rc);
        return 3;
    }
    mh_solve_opts o;
    mh_solve_opts_default(&o);
    o.r_tol = 1e-12;
    rc = flow.update_solution(&o);
    if (rc < 0) {
        std::fprintf(stderr, "update_solution: %d %s\n", rc, mh_last_error(flow.handle()));
        return 4;
    }
    double *vec;
    unsigned int n;
    flow.get_solution_vector(vec, n);
    save(dir + "/solution.bin", vec, n);
    // the MH_DofHandler accessors, element by element: pressure, then (flux, side pressure) per side
    std::vector<double> acc;
    for (int64_t e = 0; e < z.n_elements; ++e) {
        acc.push_back(flow.element_scalar(e));
        for (int i = 0; i <= el_dim[e]; ++i) {
            acc.push_back(flow.side_flux(e, i));
            acc.push_back(flow.side_scalar(e, i));
        }
    }
    save(dir + "/accessors.bin", acc.data(), acc.size());
    return 0;
}

int main(int argc, char **argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: %s linsys|darcy <dir> <solve 0|1>\n", argv[0]);
        return 1;
    }
    const std::string mode = argv[1], dir = argv[2];
    const bool solve = std::atoi(argv[3]) != 0;
    if (mode == "linsys") return run_linsys(dir, solve);
    if (mode == "darcy") return run_darcy(dir, solve);
    return 1;
}
