// Mortar coupling of non-matching lower-dimensional elements: the constant blocks that
// DarcyFlowMH_Steady adds to the edge rows of the MH system when mortar_method is P0 or P1
// (coupling_P0_mortar_assembly, src/flow/darcy_flow_mh.cc:698-799, and
// mh_abstract_assembly_intersection, :815-937), from the intersections of 1D (master) and 2D
// (slave) elements that the reference reads from its neighbouring file
// (Mesh::read_intersections, src/mesh/mesh.cc:703-755; Intersection, src/mesh/intersection.cc).
// The blocks enter the edge system with the sign of the final scale(-1) (darcy_flow_mh.cc:1128):
// the reference adds -sigma (...) to the MH matrix, the edge system receives +sigma (...).
// Host work, once per handle; the device adds the summed values after every assembly.
#include <cmath>
#include <string>
#include <vector>

#include "mh_darcy.h"
#include "system_build.hpp"
#include "topology.hpp"

namespace mh {

namespace {

double line_length(const MeshData &m, int64_t e) {
    const int32_t a = m.nodes[4 * e], b = m.nodes[4 * e + 1];
    double s = 0.0;
    for (int k = 0; k < 3; ++k) {
        const double d = m.xyz[3 * b + k] - m.xyz[3 * a + k];
        s += d * d;
    }
    return std::sqrt(s);
}

int32_t side_edge_of(const Topology &t, int64_t e, int s) { return t.side_edge[t.el_side_start[e] + s]; }

}  // namespace

// Intersection k: master (1D) element, slave (2D) element, and its two points X, Y given by
// their local coordinates on the master (master_t[2k], [2k+1]) and on the slave
// (slave_xy[4k..4k+1] for X, [4k+2..4k+3] for Y), as in the reference's file.  Its size is
// |master| (t_Y - t_X) (Intersection::intersection_true_size: the master's measure times the
// determinant of the 1 x 1 map).
int mortar_blocks(const MeshData &m, const Topology &t, const mh_mortar_desc &d, ExtraBlocks &out, std::string *err) {
    out = ExtraBlocks();
    if (d.method == MH_MORTAR_NONE || d.n == 0) return MH_OK;
    if ((d.method != MH_MORTAR_P0 && d.method != MH_MORTAR_P1) || d.n < 0 || !d.master || !d.slave || !d.master_t ||
        !d.slave_xy || !std::isfinite(d.sigma)) {
        if (err) *err = "mortar: invalid description";
        return MH_ERR_INVALID;
    }
    for (int64_t k = 0; k < d.n; ++k) {
        const int64_t ma = d.master[k], sl = d.slave[k];
        if (ma < 0 || ma >= m.n_el || sl < 0 || sl >= m.n_el || m.dim[ma] != 1 || m.dim[sl] != 2) {
            if (err) *err = "mortar: intersection " + std::to_string(k) + " is not a (1D master, 2D slave) pair";
            return MH_ERR_INVALID;
        }
        for (int q = 0; q < 2; ++q)
            if (!std::isfinite(d.master_t[2 * k + q])) {
                if (err) *err = "mortar: non-finite local coordinate";
                return MH_ERR_NONFINITE;
            }
        for (int q = 0; q < 4; ++q)
            if (!std::isfinite(d.slave_xy[4 * k + q])) {
                if (err) *err = "mortar: non-finite local coordinate";
                return MH_ERR_NONFINITE;
            }
    }
    auto true_size = [&](int64_t k) { return line_length(m, d.master[k]) * (d.master_t[2 * k + 1] - d.master_t[2 * k]); };
    if (d.method == MH_MORTAR_P0) {
        // the intersections of every master, in element order and, per master, in input order
        // (Mesh::make_intersec_elements, mesh.cc:758-775); one rank-one block per master:
        // v = (delta_0 / 2, delta_0 / 2 | -delta_i / 3 x 3 per slave i), block = sigma v v' / delta_0
        std::vector<std::vector<int64_t>> lists(m.n_el);
        for (int64_t k = 0; k < d.n; ++k) lists[d.master[k]].push_back(k);
        for (int64_t ma = 0; ma < m.n_el; ++ma) {
            const auto &L = lists[ma];
            if (L.empty()) continue;
            const double d0 = line_length(m, ma);
            std::vector<int32_t> edges;
            std::vector<double> v;
            for (int64_t k : L) {
                const double di = true_size(k);
                for (int s = 0; s < 3; ++s) {
                    edges.push_back(side_edge_of(t, d.slave[k], s));
                    v.push_back(-di / 3.0);
                }
            }
            for (int s = 0; s < 2; ++s) {
                edges.push_back(side_edge_of(t, ma, s));
                v.push_back(d0 / 2.0);
            }
            const size_t q = edges.size();
            std::vector<double> blk(q * q);
            for (size_t a = 0; a < q; ++a)
                for (size_t b = 0; b < q; ++b) blk[a * q + b] = d.sigma * v[a] * v[b] / d0;
            out.edges.push_back(std::move(edges));
            out.vals.push_back(std::move(blk));
        }
        return MH_OK;
    }
    // P1: per intersection the integral over it of the squared jump between the slave's and
    // the master's nonconforming P1 traces, with the point values of the reference's basis:
    // triangle sides (mid-points) 1 - 2 t1, -1 + 2 t0 + 2 t1, 1 - 2 t0; line sides 1 - t, t.
    for (int64_t k = 0; k < d.n; ++k) {
        double dX[5], dY[5];
        const double *sx = d.slave_xy + 4 * k, *mt = d.master_t + 2 * k;
        auto slave_basis = [](double t0, double t1, double *out3) {
            out3[0] = 1.0 - 2.0 * t1;
            out3[1] = -1.0 + 2.0 * t0 + 2.0 * t1;
            out3[2] = 1.0 - 2.0 * t0;
        };
        double bX[3], bY[3];
        slave_basis(sx[0], sx[1], bX);
        slave_basis(sx[2], sx[3], bY);
        for (int i = 0; i < 3; ++i) {
            dX[i] = -bX[i];
            dY[i] = -bY[i];
        }
        dX[3] = 1.0 - mt[0];
        dX[4] = mt[0];
        dY[3] = 1.0 - mt[1];
        dY[4] = mt[1];
        const double sz = true_size(k);
        std::vector<int32_t> edges(5);
        for (int s = 0; s < 3; ++s) edges[s] = side_edge_of(t, d.slave[k], s);
        for (int s = 0; s < 2; ++s) edges[3 + s] = side_edge_of(t, d.master[k], s);
        std::vector<double> blk(25);
        for (int i = 0; i < 5; ++i)
            for (int j = 0; j < 5; ++j)
                blk[i * 5 + j] = d.sigma * sz *
                                 (dY[i] * dY[j] + dY[i] * dX[j] / 2.0 + dX[i] * dY[j] / 2.0 + dX[i] * dX[j]) * (1.0 / 3.0);
        out.edges.push_back(std::move(edges));
        out.vals.push_back(std::move(blk));
    }
    return MH_OK;
}

}  // namespace mh
