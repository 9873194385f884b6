// Element-local mixed-hybrid computation on the device, FP64 throughout.
//
// For one element E of dimension DIM (n = DIM+1 sides) this computes, in registers:
//   A_E      -- the RT0 resistance matrix of MHFEValues::update (src/flow/mh_fe_values.cc:34-60,
//               local_matrix_line :129-153, local_matrix_triangle :159-211,
//               local_matrix_tetrahedron :339-375 with polynom_integral_tetrahedron :452-514);
//   A_E^-1   -- adjugate inverse with the reference's singularity test (MatrixInverse,
//               src/system/math_fce.cc:124-229, NUM_ZERO = DBL_MIN/DBL_EPSILON, math_fce.h:51);
//   the element's rows of the saddle-point system (assembly_steady_mh_matrix,
//               src/flow/darcy_flow_mh.cc:551-671: C = c_val, B = -1, gravity and BC rhs,
//               sources, VB coupling [-v v; v -v] with v = sigma_lower*|side|*delta_higher);
//   the first elimination (sides)  S1 = Bt*IA*B - C, r1 = Bt*IA*RHS1 - RHS2   (schur.cc:583-602, 692)
//   the second elimination (element pressure, S1_ee is a scalar per element)
//       S2 = S1_ff - S1_fe S1_ee^-1 S1_ef,  r2 = r1_f - S1_fe S1_ee^-1 r1_e
//   i.e. the reference's schur2 after scale(-1) (darcy_flow_mh.cc:1123-1130).
// The local edge list is [own side edges (n) | VB-neighbour edges (k)].
#pragma once
#include <cstdint>

#include "mh_types.hpp"

namespace mh {

constexpr double kNumZero = 2.2250738585072014e-308 / 2.220446049250313e-16;

template <int DIM> struct MaxNgh { static constexpr int value = 0; };
template <> struct MaxNgh<1> { static constexpr int value = kMaxNgh1; };
template <> struct MaxNgh<2> { static constexpr int value = kMaxNgh2; };

struct V3 { double x, y, z; };
__device__ __forceinline__ V3 v3sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 v3cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double v3dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double v3norm(V3 a) { return sqrt(v3dot(a, a)); }
__device__ __forceinline__ V3 v3scale(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 v3div(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }

// Small-matrix inverses by the adjugate (cofactor matrix transposed over the determinant),
// MatrixInverse of src/system/math_fce.cc:124-229; the caller applies the NUM_ZERO test.
// The operation order is fixed (cofactors from cyclic 2x2 minors for n = 3, from 3x3 minor
// determinants for n = 4) and the file is compiled without FMA contraction, so the element
// arithmetic is reproducible bit for bit on any IEEE-754 FP64 unit.
__device__ __forceinline__ double det3(double a00, double a01, double a02, double a10, double a11, double a12,
                                       double a20, double a21, double a22) {
    return a00 * (a11 * a22 - a12 * a21) - a01 * (a10 * a22 - a12 * a20) + a02 * (a10 * a21 - a11 * a20);
}

template <int N> __device__ __forceinline__ double inv_small(const double (&a)[N][N], double (&b)[N][N]);

template <> __device__ __forceinline__ double inv_small<2>(const double (&a)[2][2], double (&b)[2][2]) {
    double det = a[0][0] * a[1][1] - a[0][1] * a[1][0];
    b[0][0] = a[1][1] / det;
    b[0][1] = -a[0][1] / det;
    b[1][0] = -a[1][0] / det;
    b[1][1] = a[0][0] / det;
    return det;
}

template <> __device__ __forceinline__ double inv_small<3>(const double (&a)[3][3], double (&b)[3][3]) {
    double cof[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int r0 = (i + 1) % 3, r1 = (i + 2) % 3, c0 = (j + 1) % 3, c1 = (j + 2) % 3;
            cof[i][j] = a[r0][c0] * a[r1][c1] - a[r0][c1] * a[r1][c0];
        }
    double det = a[0][0] * cof[0][0] + a[0][1] * cof[0][1] + a[0][2] * cof[0][2];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) b[i][j] = cof[j][i] / det;
    return det;
}

template <> __device__ __forceinline__ double inv_small<4>(const double (&a)[4][4], double (&b)[4][4]) {
    double cof[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            double m[9];
            int k = 0;
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                if (r == i) continue;
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    if (c == j) continue;
                    m[k++] = a[r][c];
                }
            }
            const double d = det3(m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], m[8]);
            cof[i][j] = ((i + j) % 2) ? -d : d;
        }
    double det = a[0][0] * cof[0][0] + a[0][1] * cof[0][1] + a[0][2] * cof[0][2] + a[0][3] * cof[0][3];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) b[i][j] = cof[j][i] / det;
    return det;
}

// Inverse of the anisotropy tensor; a diagonal tensor is inverted entry-wise.
__device__ __forceinline__ void inv3(const double *a, double *r) {
    if (a[1] == 0.0 && a[2] == 0.0 && a[3] == 0.0 && a[5] == 0.0 && a[6] == 0.0 && a[7] == 0.0) {
#pragma unroll
        for (int i = 0; i < 9; ++i) r[i] = 0.0;
        r[0] = 1.0 / a[0];
        r[4] = 1.0 / a[4];
        r[8] = 1.0 / a[8];
        return;
    }
    const double m[3][3] = {{a[0], a[1], a[2]}, {a[3], a[4], a[5]}, {a[6], a[7], a[8]}};
    double inv[3][3];
    inv_small<3>(m, inv);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r[3 * i + j] = inv[i][j];
}

// Side node tables (src/mesh/ref_element.cc:51-76).
__device__ __forceinline__ int dev_side_node(int dim, int side, int k) {
    if (dim == 3) return (k < side) ? k : k + 1;   // face opposite node `side`
    if (dim == 2) return (side == 2) ? (k == 0 ? 0 : 2) : side + k;
    return side;
}

// Local RT0 resistance matrix; returns the element measure.  X: node coordinates, R: the
// inverse anisotropy tensor (row-major), scale = 1/K/delta.
template <int DIM> __device__ __forceinline__ double local_matrix(const V3 (&X)[DIM + 1], const double *R,
                                                                  double scale,
                                                                  double (&A)[DIM + 1][DIM + 1]);

template <> __device__ __forceinline__ double local_matrix<1>(const V3 (&X)[2], const double *R, double scale,
                                                              double (&A)[2][2]) {
    V3 t = v3sub(X[1], X[0]);
    double len = v3norm(t);
    t = v3div(t, len);
    V3 Rt = {R[0] * t.x + R[1] * t.y + R[2] * t.z, R[3] * t.x + R[4] * t.y + R[5] * t.z,
             R[6] * t.x + R[7] * t.y + R[8] * t.z};
    double val = scale * v3dot(t, Rt) * len / 3.0;
    A[0][0] = val;
    A[1][1] = val;
    A[0][1] = -val / 2.0;
    A[1][0] = -val / 2.0;
    return len;
}

template <> __device__ __forceinline__ double local_matrix<2>(const V3 (&X)[3], const double *R, double scale,
                                                              double (&A)[3][3]) {
    // in-plane frame: ex along X1-X0, ez normal, ey = ez x ex
    V3 ex = v3sub(X[1], X[0]);
    ex = v3div(ex, v3norm(ex));
    V3 ac = v3sub(X[2], X[0]);
    V3 ez = v3cross(ex, ac);
    ez = v3div(ez, v3norm(ez));
    V3 ey = v3cross(ez, ex);
    ey = v3div(ey, v3norm(ey));
    // 2x2 resistance tensor r^T R r with r = [ex ey]
    V3 Rex = {R[0] * ex.x + R[1] * ex.y + R[2] * ex.z, R[3] * ex.x + R[4] * ex.y + R[5] * ex.z,
              R[6] * ex.x + R[7] * ex.y + R[8] * ex.z};
    V3 Rey = {R[0] * ey.x + R[1] * ey.y + R[2] * ey.z, R[3] * ey.x + R[4] * ey.y + R[5] * ey.z,
              R[6] * ey.x + R[7] * ey.y + R[8] * ey.z};
    double a00 = v3dot(ex, Rex), a01 = v3dot(ex, Rey), a10 = v3dot(ey, Rex), a11 = v3dot(ey, Rey);
    // planar node coordinates (node_coordinates_triangle, mh_fe_values.cc:218-245)
    V3 u = v3sub(X[1], X[0]), v = v3sub(X[2], X[0]);
    V3 nrm = v3cross(u, v);
    V3 tt = v3div(u, v3norm(u));
    nrm = v3div(nrm, v3norm(nrm));
    V3 bb = v3cross(nrm, u);
    bb = v3div(bb, v3norm(bb));
    double px[3] = {0.0, v3dot(tt, u), v3dot(tt, v)};
    double py[3] = {0.0, v3dot(bb, u), v3dot(bb, v)};
    // side midpoints: side0 = (0,1), side1 = (1,2), side2 = (2,0)
    double mx[3] = {(px[0] + px[1]) / 2.0, (px[1] + px[2]) / 2.0, (px[2] + px[0]) / 2.0};
    double my[3] = {(py[0] + py[1]) / 2.0, (py[1] + py[2]) / 2.0, (py[2] + py[0]) / 2.0};
    // basis phi_i = gamma_i (x - P_i), P_i the node opposite side i
    double al[3], be[3], ga[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        int i0 = i, i1 = (i + 1) % 3, i2 = (i + 2) % 3;
        al[i] = px[i2];
        be[i] = py[i2];
        ga[i] = 1.0 / fabs((px[i0] - px[i2]) * (py[i1] - py[i0]) + (py[i0] - py[i2]) * (px[i0] - px[i1]));
    }
    double area = v3norm(v3cross(v3sub(X[1], X[0]), v3sub(X[2], X[0]))) / 2.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j) {
            double p0 = a00 * al[i] * al[j] + a01 * be[i] * al[j] + a10 * al[i] * be[j] + a11 * be[i] * be[j];
            double p1 = (a00 * al[i] + a00 * al[j] + a01 * be[i] + a10 * be[j]) * -1.0;
            double p2 = (a11 * be[i] + a11 * be[j] + a10 * al[i] + a01 * al[j]) * -1.0;
            double p3 = a00, p4 = a01 + a10, p5 = a11;
            double s = 0.0;
#pragma unroll
            for (int q = 0; q < 3; ++q)
                s += p0 + p1 * mx[q] + p2 * my[q] + p3 * mx[q] * mx[q] + p4 * mx[q] * my[q] + p5 * my[q] * my[q];
            A[i][j] = scale * ga[i] * ga[j] * area * s / 3.0;
            A[j][i] = A[i][j];
        }
    return area;
}

template <> __device__ __forceinline__ double local_matrix<3>(const V3 (&X)[4], const double *R, double scale,
                                                              double (&A)[4][4]) {
    V3 e1 = v3sub(X[1], X[0]), e2 = v3sub(X[2], X[0]), e3 = v3sub(X[3], X[0]);
    double vol = fabs(v3dot(v3cross(e1, e2), e3)) / 6.0;
    V3 c = {(X[0].x + X[1].x + X[2].x + X[3].x) / 4.0, (X[0].y + X[1].y + X[2].y + X[3].y) / 4.0,
            (X[0].z + X[1].z + X[2].z + X[3].z) / 4.0};
    // delta_i = 1 / (|S_i| * n_i . (c_i - X_i)), n_i the outward unit normal of side i
    double delta[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        V3 a = X[dev_side_node(3, i, 0)], b = X[dev_side_node(3, i, 1)], d = X[dev_side_node(3, i, 2)];
        V3 cr = v3cross(v3sub(b, a), v3sub(d, a));
        double nr = v3norm(cr);
        double meas = 0.5 * nr;
        V3 n = v3div(cr, nr);
        if (v3dot(n, v3sub(c, a)) > 0.0) n = v3scale(n, -1.0);
        V3 sc = {(a.x + b.x + d.x) / 3.0, (a.y + b.y + d.y) / 3.0, (a.z + b.z + d.z) / 3.0};
        delta[i] = 1.0 / (meas * (n.x * sc.x + n.y * sc.y + n.z * sc.z - n.x * X[i].x - n.y * X[i].y - n.z * X[i].z));
    }
    // second moments about the centroid: the quadratic monomials integrate exactly to
    // |E| (t_r t_c + M_rc / 20) (polynom_integral_tetrahedron)
    double M[3][3];
    const double t[3] = {c.x, c.y, c.z};
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q) M[r][q] = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double d[3] = {X[k].x - t[0], X[k].y - t[1], X[k].z - t[2]};
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int q = 0; q < 3; ++q) M[r][q] += d[r] * d[q];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = i; j < 4; ++j) {
            // coefficients of (x - X_j)^T R (x - X_i) in the monomial basis
            // {1, x, y, z, xy, xz, yz, x^2, y^2, z^2} (calc_polynom_tetrahedron)
            const double Xi[3] = {X[i].x, X[i].y, X[i].z}, Xj[3] = {X[j].x, X[j].y, X[j].z};
            double poly[10];
            poly[0] = 0.0;
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int q = 0; q < 3; ++q) poly[0] += R[3 * r + q] * Xi[q] * Xj[r];
#pragma unroll
            for (int q = 0; q < 3; ++q)
                poly[1 + q] = -(R[3 * q] * Xi[0] + R[3 * q + 1] * Xi[1] + R[3 * q + 2] * Xi[2] + R[q] * Xj[0] +
                                R[3 + q] * Xj[1] + R[6 + q] * Xj[2]);
            poly[4] = R[1] + R[3];
            poly[5] = R[2] + R[6];
            poly[6] = R[5] + R[7];
            poly[7] = R[0];
            poly[8] = R[4];
            poly[9] = R[8];
            double rc = 0.0;
            rc += poly[0] * vol;
            rc += poly[1] * vol * t[0];
            rc += poly[2] * vol * t[1];
            rc += poly[3] * vol * t[2];
            rc += poly[4] * vol * (t[0] * t[1] + 1.0 / 20.0 * M[0][1]);
            rc += poly[5] * vol * (t[0] * t[2] + 1.0 / 20.0 * M[0][2]);
            rc += poly[6] * vol * (t[1] * t[2] + 1.0 / 20.0 * M[1][2]);
            rc += poly[7] * vol * (t[0] * t[0] + 1.0 / 20.0 * M[0][0]);
            rc += poly[8] * vol * (t[1] * t[1] + 1.0 / 20.0 * M[1][1]);
            rc += poly[9] * vol * (t[2] * t[2] + 1.0 / 20.0 * M[2][2]);
            A[i][j] = scale * delta[i] * delta[j] * rc;
            A[j][i] = A[i][j];
        }
    return vol;
}

// Everything K1 (assembly), K6 (time-term rhs) and K4 (back-substitution) need from one element.
template <int DIM> struct LocalMH {
    static constexpr int N = DIM + 1;
    static constexpr int K = MaxNgh<DIM>::value;
    static constexpr int M = N + K;
    int k;              // VB neighbours of this element
    int side0;          // first global side
    int32_t edge[M];    // local edge list [own | neighbours]
    double Ainv[N][N];
    double g[N];        // side rhs (gravity, Dirichlet)
    double c[N];        // c_val of each side
    double u[M];        // S1[E, edge_l]
    double s1ee;        // S1[E, E]
    double r1e;         // r1[E]
    double f_own[N];    // -F diagonal on own edges (BC and LMH time terms)
    double b_own[N];    // r1 edge rhs on own edges minus c*(A^-1 g)
    double v[K > 0 ? K : 1];
    double lmh_coef;    // LMH: |E| S delta / dt / n   (0 otherwise)
    double src_side;    // -|E| delta f / n (LMH flux postprocess)
    int singular;
};

// Build the local MH data of element e.
template <int DIM> __device__ __forceinline__ void build_local(const ElemData &d, int e, LocalMH<DIM> &L) {
    constexpr int N = DIM + 1;
    V3 X[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
        int nd = d.el_nodes[4 * e + i];
        X[i] = {d.xyz[3 * nd], d.xyz[3 * nd + 1], d.xyz[3 * nd + 2]};
    }
    double R[9];
    if (d.anisotropy) {
        double a[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) a[i] = d.anisotropy[9 * (size_t)e + i];
        inv3(a, R);
    } else {
#pragma unroll
        for (int i = 0; i < 9; ++i) R[i] = (i % 4 == 0) ? 1.0 : 0.0;
    }
    const double delta = d.cross_section[e];
    const double scale = 1.0 / d.conductivity[e] / delta;
    double A[N][N];
    const double meas = local_matrix<DIM>(X, R, scale, A);
    const double det = inv_small<N>(A, L.Ainv);
    L.singular = !(fabs(det) >= kNumZero);

    double cz = 0.0;
#pragma unroll
    for (int i = 0; i < N; ++i) cz += X[i].z;
    cz /= (double)N;

    L.side0 = d.el_side_start[e];
    double bE = -1.0 * meas * delta * d.source[e];
    double dEE = 0.0;
    L.lmh_coef = 0.0;
    if (d.time_mode == 1) {
        double tt = -d.storativity[e] * meas / d.dt;
        dEE += tt;
        bE += tt * d.prev_pressure[e];
    } else if (d.time_mode == 2) {
        L.lmh_coef = meas * d.storativity[e] * delta / d.dt / (double)N;
    }
    L.src_side = -1.0 * meas * delta * d.source[e] / (double)N;

#pragma unroll
    for (int i = 0; i < N; ++i) {
        const int s = L.side0 + i;
        L.edge[i] = d.side_edge[s];
        // side centre z and measure
        double sz = 0.0, smeas = 1.0;
        if (DIM == 1) {
            sz = X[i].z;
        } else if (DIM == 2) {
            V3 a = X[dev_side_node(2, i, 0)], b = X[dev_side_node(2, i, 1)];
            sz = (a.z + b.z) / 2.0;
            smeas = v3norm(v3sub(b, a));
        } else {
            V3 a = X[dev_side_node(3, i, 0)], b = X[dev_side_node(3, i, 1)], q = X[dev_side_node(3, i, 2)];
            sz = (a.z + b.z + q.z) / 3.0;
            smeas = 0.5 * v3norm(v3cross(v3sub(b, a), v3sub(q, a)));
        }
        double gi = cz - sz;
        double ci = 1.0, fdiag = 0.0, bedge = 0.0;
        const int bdr = d.side_bdr[s];
        if (bdr >= 0) {
            const int type = d.bc_type[bdr];
            if (type == 1) {          // Dirichlet
                ci = 0.0;
                double p = d.bc_pressure[bdr];
                gi -= p;
                bedge += -p;
                fdiag += -1.0;
            } else if (type == 2) {   // Neumann
                bedge += d.bc_flux[bdr] * smeas * delta;
            } else if (type == 3) {   // Robin
                double p = d.bc_pressure[bdr], sg = d.bc_sigma[bdr];
                bedge += -smeas * sg * p * delta;
                fdiag += -smeas * sg * delta;
            }
        }
        if (d.time_mode == 2) {
            fdiag += -L.lmh_coef;
            bedge += -L.lmh_coef * d.prev_edge[L.edge[i]];
        }
        L.g[i] = gi;
        L.c[i] = ci;
        L.f_own[i] = -fdiag;
        L.b_own[i] = -bedge;
    }

    // VB neighbours: this element is the lower-dimensional one
    L.k = 0;
    if (DIM < 3) {
        const int n0 = d.el_ngh_start[e], n1 = d.el_ngh_start[e + 1];
        const double sg = d.sigma[e];
#pragma unroll
        for (int m = 0; m < LocalMH<DIM>::K; ++m) {
            if (n0 + m < n1) {
                const int ng = d.el_ngh[n0 + m];
                const double vv = sg * d.ngh_side_measure[ng] * d.cross_section[d.ngh_hi_el[ng]];
                L.v[m] = vv;
                L.edge[N + m] = d.ngh_edge[ng];
                dEE += -vv;
                L.k = m + 1;
            } else {
                L.v[m] = 0.0;
                L.edge[N + m] = -1;
            }
        }
    }

    // first elimination
    double Ag[N], A1[N], s1 = 0.0, sg_ = 0.0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        double t1 = 0.0, t2 = 0.0;
#pragma unroll
        for (int j = 0; j < N; ++j) {
            t1 += L.Ainv[i][j];
            t2 += L.Ainv[i][j] * L.g[j];
        }
        A1[i] = t1;
        Ag[i] = t2;
        s1 += t1;
        sg_ += t2;
    }
    L.s1ee = s1 - dEE;
    L.r1e = -sg_ - bE;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        L.u[i] = -L.c[i] * A1[i];
        L.b_own[i] += L.c[i] * Ag[i];
    }
#pragma unroll
    for (int m = 0; m < LocalMH<DIM>::K; ++m) L.u[N + m] = -L.v[m];
}

// Local second-Schur block entry (l, m) of the (n+k) x (n+k) edge block.
template <int DIM> __device__ __forceinline__ double local_s2(const LocalMH<DIM> &L, int l, int m) {
    constexpr int N = DIM + 1;
    double s1ff = 0.0;
    if (l < N && m < N) {
        s1ff = L.c[l] * L.Ainv[l][m] * L.c[m];
        if (l == m) s1ff += L.f_own[l];
    } else if (l == m) {
        s1ff = L.v[l - N];
    }
    return s1ff - L.u[l] * L.u[m] / L.s1ee;
}

template <int DIM> __device__ __forceinline__ double local_r2(const LocalMH<DIM> &L, int l) {
    constexpr int N = DIM + 1;
    double r1f = (l < N) ? L.b_own[l] : 0.0;
    return r1f - L.u[l] * L.r1e / L.s1ee;
}

}  // namespace mh
