/*
 * mh_oracle.c -- TEST INFRASTRUCTURE ONLY.  A plain-C FP64 restatement of Flow123d's mixed-
 * hybrid Darcy path, used as the checker of the GPU library (tests/, __graft_entry__.smoke()
 * and bench.py's CPU baseline).  It is never linked into or called by the product.
 *
 * Restated from the reference (paths relative to the Flow123d source tree):
 *   geometry        src/mesh/elements.cc:108-150 (measure, centre),
 *                   src/mesh/sides.cc:42-148 (side measure, outward normal, centre)
 *   local matrices  src/flow/mh_fe_values.cc:34-60 (update), :129-153 (line),
 *                   :159-334 (triangle), :339-514 (tetrahedron)
 *   inverses        src/system/math_fce.cc:124-229 (adjugate / determinant,
 *                   singular when |det| < NUM_ZERO = DBL_MIN/DBL_EPSILON, math_fce.h:51)
 *   MH assembly     src/flow/darcy_flow_mh.cc:525-694 (assembly_steady_mh_matrix)
 *   time terms      darcy_flow_mh.cc:1614-1675 (MH), :1695-1766 (LMH)
 *   Schur algebra   src/la/schur.cc:566-611, 690-694, 714-773; darcy_flow_mh.cc:1009-1131
 *   LMH postprocess darcy_flow_mh.cc:1772-1827
 *   element vectors src/flow/darcy_flow_mh_output.cc:301-323 (make_element_vector) with
 *                   mh_fe_values.cc:76-118 (RT0_value)
 *   node pressures  darcy_flow_mh_output.cc:424-546 (make_node_scalar_param)
 *   water balance   darcy_flow_mh_output.cc:671-790 (water_balance)
 *
 * Parity is pinned against the reference's own golden outputs: the per-element pressures,
 * fluxes and edge pressures of tests/01_steady_flow_123d/ref_output/flow_gmsh.con/raw_output.txt,
 * the node pressures and the water balance of the same run,
 * the element pressures of the VTK outputs of tests 05, 06 and 10, and the analytic answers of
 * tests 06 (p2 = -3, p1 = -2.5).  The FP64 direct solve of the full saddle-point system is
 * done with scipy in oracle.py.
 *
 * Build: make -C oracle   (gcc -O3 -fopenmp, output oracle/libmhoracle.so)
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>

#define ORC_NUM_ZERO (DBL_MIN / DBL_EPSILON)

/* ------------------------------------------------------------------ geometry ---------- */
static const int SIDE_NODES_1[2][1] = {{0}, {1}};
static const int SIDE_NODES_2[3][2] = {{0, 1}, {1, 2}, {0, 2}};
static const int SIDE_NODES_3[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};

static int side_node(int dim, int s, int k) {
    if (dim == 1) return SIDE_NODES_1[s][k];
    if (dim == 2) return SIDE_NODES_2[s][k];
    return SIDE_NODES_3[s][k];
}

static void sub3(const double *a, const double *b, double *r) { r[0] = a[0] - b[0]; r[1] = a[1] - b[1]; r[2] = a[2] - b[2]; }
static void cross3(const double *a, const double *b, double *r) {
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}
static double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static double norm3(const double *a) { return sqrt(dot3(a, a)); }

typedef struct {
    int dim, n;
    double X[4][3];
} Elem;

static void load_elem(const double *xyz, const int32_t *el_nodes, const int32_t *el_dim, int64_t e, Elem *E) {
    E->dim = el_dim[e];
    E->n = E->dim + 1;
    for (int i = 0; i < E->n; ++i)
        for (int c = 0; c < 3; ++c) E->X[i][c] = xyz[3 * (int64_t)el_nodes[4 * e + i] + c];
}

static double elem_measure(const Elem *E) {
    double u[3], v[3], w[3], c[3];
    if (E->dim == 1) { sub3(E->X[1], E->X[0], u); return norm3(u); }
    if (E->dim == 2) { sub3(E->X[1], E->X[0], u); sub3(E->X[2], E->X[0], v); cross3(u, v, c); return norm3(c) / 2.0; }
    sub3(E->X[1], E->X[0], u); sub3(E->X[2], E->X[0], v); sub3(E->X[3], E->X[0], w);
    cross3(u, v, c);
    return fabs(dot3(c, w)) / 6.0;
}

static void elem_centre(const Elem *E, double *c) {
    c[0] = c[1] = c[2] = 0.0;
    for (int i = 0; i < E->n; ++i) { c[0] += E->X[i][0]; c[1] += E->X[i][1]; c[2] += E->X[i][2]; }
    c[0] /= E->n; c[1] /= E->n; c[2] /= E->n;
}

static double side_measure(const Elem *E, int s) {
    double u[3], v[3], c[3];
    if (E->dim == 1) return 1.0;
    const double *a = E->X[side_node(E->dim, s, 0)], *b = E->X[side_node(E->dim, s, 1)];
    if (E->dim == 2) { sub3(b, a, u); return norm3(u); }
    const double *d = E->X[side_node(E->dim, s, 2)];
    sub3(b, a, u); sub3(d, a, v); cross3(u, v, c);
    return 0.5 * norm3(c);
}

static void side_centre(const Elem *E, int s, double *c) {
    int m = E->dim;  /* nodes of a side */
    c[0] = c[1] = c[2] = 0.0;
    for (int k = 0; k < m; ++k) {
        const double *p = E->X[side_node(E->dim, s, k)];
        c[0] += p[0]; c[1] += p[1]; c[2] += p[2];
    }
    c[0] /= m; c[1] /= m; c[2] /= m;
}

/* outward unit normal of a triangular side of a tetrahedron (Side::normal_triangle) */
static void side_normal_tet(const Elem *E, int s, double *n) {
    double u[3], v[3], ce[3], w[3];
    const double *a = E->X[side_node(3, s, 0)], *b = E->X[side_node(3, s, 1)], *d = E->X[side_node(3, s, 2)];
    sub3(b, a, u); sub3(d, a, v); cross3(u, v, n);
    double l = norm3(n);
    n[0] /= l; n[1] /= l; n[2] /= l;
    elem_centre(E, ce);
    sub3(ce, a, w);
    if (dot3(n, w) > 0.0) { n[0] = -n[0]; n[1] = -n[1]; n[2] = -n[2]; }
}

/* ------------------------------------------------------------------ inverses ---------- */
static double det3(double a00, double a01, double a02, double a10, double a11, double a12, double a20, double a21,
                   double a22) {
    return a00 * (a11 * a22 - a12 * a21) - a01 * (a10 * a22 - a12 * a20) + a02 * (a10 * a21 - a11 * a20);
}

/* adjugate inverse of an n x n row-major matrix (n <= 4); returns the determinant and leaves
 * b untouched when |det| < NUM_ZERO, as MatrixInverse does */
double orc_matrix_inverse(const double *a, double *b, int n) {
    if (n == 1) { b[0] = 1.0 / a[0]; return a[0]; }
    if (n == 2) {
        double det = a[0] * a[3] - a[1] * a[2];
        if (fabs(det) < ORC_NUM_ZERO) return det;
        b[0] = a[3] / det; b[1] = -a[1] / det; b[2] = -a[2] / det; b[3] = a[0] / det;
        return det;
    }
    if (n == 3) {
        double cof[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                int r0 = (i + 1) % 3, r1 = (i + 2) % 3, c0 = (j + 1) % 3, c1 = (j + 2) % 3;
                cof[3 * i + j] = a[3 * r0 + c0] * a[3 * r1 + c1] - a[3 * r0 + c1] * a[3 * r1 + c0];
            }
        double det = a[0] * cof[0] + a[1] * cof[1] + a[2] * cof[2];
        if (fabs(det) < ORC_NUM_ZERO) return det;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) b[3 * i + j] = cof[3 * j + i] / det;
        return det;
    }
    /* n == 4: cofactor C_ij = (-1)^(i+j) * det(minor_ij) */
    double cof[16];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double m[9];
            int k = 0;
            for (int r = 0; r < 4; ++r) {
                if (r == i) continue;
                for (int c = 0; c < 4; ++c) {
                    if (c == j) continue;
                    m[k++] = a[4 * r + c];
                }
            }
            double d = det3(m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], m[8]);
            cof[4 * i + j] = ((i + j) % 2 ? -d : d);
        }
    double det = a[0] * cof[0] + a[1] * cof[1] + a[2] * cof[2] + a[3] * cof[3];
    if (fabs(det) < ORC_NUM_ZERO) return det;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) b[4 * i + j] = cof[4 * j + i] / det;
    return det;
}

static void inverse_tensor(const double *aniso, double *R) {
    if (!aniso) {
        memset(R, 0, 9 * sizeof(double));
        R[0] = R[4] = R[8] = 1.0;
        return;
    }
    if (aniso[1] == 0.0 && aniso[2] == 0.0 && aniso[3] == 0.0 && aniso[5] == 0.0 && aniso[6] == 0.0 &&
        aniso[7] == 0.0) {
        memset(R, 0, 9 * sizeof(double));
        R[0] = 1.0 / aniso[0]; R[4] = 1.0 / aniso[4]; R[8] = 1.0 / aniso[8];
        return;
    }
    orc_matrix_inverse(aniso, R, 3);
}

/* ------------------------------------------------------------ local matrices ---------- */
static void local_matrix_line(const Elem *E, const double *R, double scale, double *A) {
    double t[3], Rt[3];
    sub3(E->X[1], E->X[0], t);
    double l = norm3(t);
    t[0] /= l; t[1] /= l; t[2] /= l;
    for (int r = 0; r < 3; ++r) Rt[r] = R[3 * r] * t[0] + R[3 * r + 1] * t[1] + R[3 * r + 2] * t[2];
    double val = scale * dot3(t, Rt) * elem_measure(E) / 3.0;
    A[0] = val; A[3] = val; A[1] = -val / 2.0; A[2] = -val / 2.0;
}

static double tri_poly_value(const double *p, double x, double y) {
    return p[0] + p[1] * x + p[2] * y + p[3] * x * x + p[4] * x * y + p[5] * y * y;
}

static void local_matrix_triangle(const Elem *E, const double *R, double scale, double *A) {
    double ex[3], ac[3], ez[3], ey[3], l;
    sub3(E->X[1], E->X[0], ex); l = norm3(ex); ex[0] /= l; ex[1] /= l; ex[2] /= l;
    sub3(E->X[2], E->X[0], ac);
    cross3(ex, ac, ez); l = norm3(ez); ez[0] /= l; ez[1] /= l; ez[2] /= l;
    cross3(ez, ex, ey); l = norm3(ey); ey[0] /= l; ey[1] /= l; ey[2] /= l;
    /* 2x2 resistance r^T R r, r = [ex ey] */
    double Rex[3], Rey[3];
    for (int r = 0; r < 3; ++r) {
        Rex[r] = R[3 * r] * ex[0] + R[3 * r + 1] * ex[1] + R[3 * r + 2] * ex[2];
        Rey[r] = R[3 * r] * ey[0] + R[3 * r + 1] * ey[1] + R[3 * r + 2] * ey[2];
    }
    double a00 = dot3(ex, Rex), a01 = dot3(ex, Rey), a10 = dot3(ey, Rex), a11 = dot3(ey, Rey);
    /* node coordinates in the plane (node_coordinates_triangle) */
    double u[3], v[3], nn[3], t[3], b[3];
    sub3(E->X[1], E->X[0], u);
    sub3(E->X[2], E->X[0], v);
    cross3(u, v, nn);
    t[0] = u[0]; t[1] = u[1]; t[2] = u[2];
    l = norm3(t); t[0] /= l; t[1] /= l; t[2] /= l;
    l = norm3(nn); nn[0] /= l; nn[1] /= l; nn[2] /= l;
    cross3(nn, u, b); l = norm3(b); b[0] /= l; b[1] /= l; b[2] /= l;
    double nod[3][2] = {{0.0, 0.0}, {dot3(t, u), dot3(b, u)}, {dot3(t, v), dot3(b, v)}};
    double mid[3][2];
    for (int i = 0; i < 3; ++i) {
        int j = (i + 1) % 3;
        mid[i][0] = (nod[i][0] + nod[j][0]) / 2.0;
        mid[i][1] = (nod[i][1] + nod[j][1]) / 2.0;
    }
    /* RT0 basis parameters (bas_func_0_triangle with cyclic node order) */
    double al[3], be[3], ga[3];
    for (int i = 0; i < 3; ++i) {
        const double *p0 = nod[i], *p1 = nod[(i + 1) % 3], *p2 = nod[(i + 2) % 3];
        al[i] = p2[0];
        be[i] = p2[1];
        ga[i] = 1.0 / fabs((p0[0] - p2[0]) * (p1[1] - p0[1]) + (p0[1] - p2[1]) * (p0[0] - p1[0]));
    }
    double meas = elem_measure(E);
    for (int i = 0; i < 3; ++i)
        for (int j = i; j < 3; ++j) {
            double poly[6];
            poly[0] = a00 * al[i] * al[j] + a01 * be[i] * al[j] + a10 * al[i] * be[j] + a11 * be[i] * be[j];
            poly[1] = (a00 * al[i] + a00 * al[j] + a01 * be[i] + a10 * be[j]) * -1.0;
            poly[2] = (a11 * be[i] + a11 * be[j] + a10 * al[i] + a01 * al[j]) * -1.0;
            poly[3] = a00;
            poly[4] = a01 + a10;
            poly[5] = a11;
            double s = tri_poly_value(poly, mid[0][0], mid[0][1]) + tri_poly_value(poly, mid[1][0], mid[1][1]) +
                       tri_poly_value(poly, mid[2][0], mid[2][1]);
            A[3 * i + j] = scale * ga[i] * ga[j] * meas * s / 3.0;
            A[3 * j + i] = A[3 * i + j];
        }
}

/* exact integral of a quadratic over a tetrahedron (polynom_integral_tetrahedron) */
static double tet_poly_integral(const Elem *E, const double *poly) {
    double v = elem_measure(E), t[3];
    elem_centre(E, t);
    double m[3][3] = {{0}};
    for (int k = 0; k < 4; ++k)
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) m[r][c] += (E->X[k][r] - t[r]) * (E->X[k][c] - t[c]);
    double rc = 0.0;
    rc += poly[0] * v;
    rc += poly[1] * v * t[0];
    rc += poly[2] * v * t[1];
    rc += poly[3] * v * t[2];
    rc += poly[4] * v * (t[0] * t[1] + 1.0 / 20.0 * m[0][1]);
    rc += poly[5] * v * (t[0] * t[2] + 1.0 / 20.0 * m[0][2]);
    rc += poly[6] * v * (t[1] * t[2] + 1.0 / 20.0 * m[1][2]);
    rc += poly[7] * v * (t[0] * t[0] + 1.0 / 20.0 * m[0][0]);
    rc += poly[8] * v * (t[1] * t[1] + 1.0 / 20.0 * m[1][1]);
    rc += poly[9] * v * (t[2] * t[2] + 1.0 / 20.0 * m[2][2]);
    return rc;
}

static void local_matrix_tetrahedron(const Elem *E, const double *a, double scale, double *A) {
    double delta[4];
    for (int i = 0; i < 4; ++i) {
        double n[3], c[3];
        side_normal_tet(E, i, n);
        side_centre(E, i, c);
        delta[i] = 1.0 / (side_measure(E, i) * (n[0] * c[0] + n[1] * c[1] + n[2] * c[2] - n[0] * E->X[i][0] -
                                               n[1] * E->X[i][1] - n[2] * E->X[i][2]));
    }
#define AA(r, c) a[3 * (r) + (c)]
    for (int i = 0; i < 4; ++i)
        for (int j = i; j < 4; ++j) {
            const double *Xi = E->X[i], *Xj = E->X[j];
            double poly[10];
            /* (x - X_j)^T a (x - X_i) expanded in monomials (calc_polynom_tetrahedron) */
            poly[0] = 0.0;
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) poly[0] += AA(r, c) * Xi[c] * Xj[r];
            for (int q = 0; q < 3; ++q)
                poly[1 + q] = -(AA(q, 0) * Xi[0] + AA(q, 1) * Xi[1] + AA(q, 2) * Xi[2] + AA(0, q) * Xj[0] +
                                AA(1, q) * Xj[1] + AA(2, q) * Xj[2]);
            poly[4] = AA(0, 1) + AA(1, 0);
            poly[5] = AA(0, 2) + AA(2, 0);
            poly[6] = AA(1, 2) + AA(2, 1);
            poly[7] = AA(0, 0);
            poly[8] = AA(1, 1);
            poly[9] = AA(2, 2);
            A[4 * i + j] = scale * delta[i] * delta[j] * tet_poly_integral(E, poly);
            A[4 * j + i] = A[4 * i + j];
        }
#undef AA
}

/* MHFEValues::update: A and A^-1 of element e.  Returns 0, or -2 if singular. */
int orc_local_matrix(const double *xyz, const int32_t *el_nodes, const int32_t *el_dim, int64_t e,
                     const double *aniso9, double conductivity, double cross_section, double *A, double *Ainv,
                     double *det_out) {
    Elem E;
    load_elem(xyz, el_nodes, el_dim, e, &E);
    double R[9];
    inverse_tensor(aniso9, R);
    double scale = 1 / conductivity / cross_section;
    if (E.dim == 1) local_matrix_line(&E, R, scale, A);
    else if (E.dim == 2) local_matrix_triangle(&E, R, scale, A);
    else local_matrix_tetrahedron(&E, R, scale, A);
    double det = orc_matrix_inverse(A, Ainv, E.n);
    if (det_out) *det_out = det;
    return (fabs(det) < ORC_NUM_ZERO) ? -2 : 0;
}

/* ------------------------------------------------------------------ inputs ------------ */
typedef struct {
    int64_t n_nodes;
    const double *xyz;
    int64_t n_el;
    const int32_t *el_dim, *el_nodes;
    const int32_t *el_side_start, *side_edge, *side_bdr;
    int64_t n_edges, n_ngh;
    const int32_t *ngh_element, *ngh_edge, *ngh_side;
    const double *K, *aniso, *delta, *sigma, *source, *storativity;
    const int32_t *bc_type;
    const double *bc_p, *bc_flux, *bc_sigma;
    int32_t time_mode;       /* 0 steady, 1 MH, 2 LMH */
    double dt;
    const double *prev;      /* previous MH solution (time_mode != 0) */
} orc_problem;

static int64_t n_sides_of(const orc_problem *P) { return P->el_side_start[P->n_el]; }

static int64_t ngh_higher_element(const orc_problem *P, int32_t side) {
    int64_t lo = 0, hi = P->n_el;
    while (hi - lo > 1) {
        int64_t mid = (lo + hi) / 2;
        if (P->el_side_start[mid] <= side) lo = mid; else hi = mid;
    }
    return lo;
}

static double ngh_value(const orc_problem *P, int64_t ng, int64_t lower) {
    int32_t side = P->ngh_side[ng];
    int64_t hi = ngh_higher_element(P, side);
    Elem H;
    load_elem(P->xyz, P->el_nodes, P->el_dim, hi, &H);
    return P->sigma[lower] * side_measure(&H, side - P->el_side_start[hi]) * P->delta[hi];
}

/* --------------------------------------------------- full saddle-point assembly ------- */
/* COO triplets of the MH matrix in rows [sides | elements | edges] (duplicates are meant to be
 * summed) and the rhs, exactly as assembly_steady_mh_matrix adds them, plus the time terms of
 * setup_time_term/modify_system.  Returns the number of triplets, or -1 if cap is too small,
 * -2 on a singular local matrix. */
static void neighbour_lists(const orc_problem *P, int32_t *start, int32_t *list);

int64_t orc_assemble_mh(const orc_problem *P, int32_t *I, int32_t *J, double *V, int64_t cap, double *rhs) {
    const int64_t ns = n_sides_of(P), ne = P->n_el;
    const int64_t mh_size = ns + ne + P->n_edges;
    memset(rhs, 0, mh_size * sizeof(double));
    int32_t *nstart = (int32_t *)malloc((P->n_el + 1) * sizeof(int32_t));
    int32_t *nlist = (int32_t *)malloc((P->n_ngh + 1) * sizeof(int32_t));
    neighbour_lists(P, nstart, nlist);
    int64_t k = 0;
#define ADD(r, c, v)                                     \
    do {                                                 \
        if (k >= cap) { k = -1; goto done; }             \
        I[k] = (int32_t)(r);                             \
        J[k] = (int32_t)(c);                             \
        V[k] = (v);                                      \
        ++k;                                             \
    } while (0)
    for (int64_t e = 0; e < ne; ++e) {
        Elem E;
        load_elem(P->xyz, P->el_nodes, P->el_dim, e, &E);
        double A[16], Ai[16], det;
        if (orc_local_matrix(P->xyz, P->el_nodes, P->el_dim, e, P->aniso ? P->aniso + 9 * e : NULL, P->K[e],
                             P->delta[e], A, Ai, &det)) {
            k = -2;
            goto done;
        }
        const double cs = P->delta[e];
        const int64_t el_row = ns + e;
        double ce[3];
        elem_centre(&E, ce);
        int64_t side_rows[4];
        for (int i = 0; i < E.n; ++i) {
            const int64_t side = P->el_side_start[e] + i;
            const int64_t edge_row = ns + ne + P->side_edge[side];
            side_rows[i] = side;
            double sc[3];
            side_centre(&E, i, sc);
            double loc_rhs = ce[2] - sc[2];
            double c_val = 1.0;
            const int32_t b = P->side_bdr[side];
            if (b >= 0) {
                const double bmeas = side_measure(&E, i);
                switch (P->bc_type[b]) {
                    case 1: {
                        c_val = 0.0;
                        loc_rhs -= P->bc_p[b];
                        rhs[edge_row] += -P->bc_p[b];
                        ADD(edge_row, edge_row, -1.0);
                        break;
                    }
                    case 2: rhs[edge_row] += P->bc_flux[b] * bmeas * cs; break;
                    case 3:
                        rhs[edge_row] += -bmeas * P->bc_sigma[b] * P->bc_p[b] * cs;
                        ADD(edge_row, edge_row, -bmeas * P->bc_sigma[b] * cs);
                        break;
                    default: break;
                }
            }
            ADD(side, edge_row, c_val);
            ADD(edge_row, side, c_val);
            rhs[side] += loc_rhs;
        }
        for (int i = 0; i < E.n; ++i)
            for (int j = 0; j < E.n; ++j) ADD(side_rows[i], side_rows[j], A[E.n * i + j]);
        for (int i = 0; i < E.n; ++i) {
            ADD(el_row, side_rows[i], -1.0);
            ADD(side_rows[i], el_row, -1.0);
        }
        const double meas = elem_measure(&E);
        rhs[el_row] += -1.0 * meas * P->delta[e] * P->source[e];
        ADD(el_row, el_row, 0.0);
        for (int32_t j = nstart[e]; j < nstart[e + 1]; ++j) {
            const int64_t ng = nlist[j];
            const double v = ngh_value(P, ng, e);
            const int64_t er = ns + ne + P->ngh_edge[ng];
            ADD(el_row, el_row, -v);
            ADD(el_row, er, v);
            ADD(er, el_row, v);
            ADD(er, er, -v);
        }
        /* time terms */
        if (P->time_mode == 1) {
            const double d = -P->storativity[e] * meas / P->dt;
            ADD(el_row, el_row, d);
            rhs[el_row] += d * P->prev[el_row];
        } else if (P->time_mode == 2) {
            for (int i = 0; i < E.n; ++i) {
                const int64_t er = ns + ne + P->side_edge[P->el_side_start[e] + i];
                const double d = -meas * P->storativity[e] * P->delta[e] / P->dt / E.n;
                ADD(er, er, d);
                rhs[er] += d * P->prev[er];
            }
        }
    }
#undef ADD
done:
    free(nstart);
    free(nlist);
    return k;
}

/* ------------------------------------------- element-local double Schur --------------- */
/* Per element: the (n+k)x(n+k) block of the second Schur complement (reference schur2 after
 * scale(-1)) and its rhs, by the algebra of SchurComplement::form_schur/form_rhs applied to
 * one element (B couples an element only to its own sides, S1_EE is a scalar).  Local edges
 * are [own side edges | VB-neighbour edges]; edges_out gets them.  Returns m = n + k or -2. */
typedef struct {
    int n, k, m;
    int32_t edges[12];
    double Ainv[16], g[4], c[4], u[12], s1ee, r1e, f_own[4], b_own[4], v[8];
    double lmh_coef, src_side;
} orc_local;

static int build_local(const orc_problem *P, int64_t e, const int32_t *ngh_list, int n_ngh_e, orc_local *L) {
    Elem E;
    load_elem(P->xyz, P->el_nodes, P->el_dim, e, &E);
    double A[16], det;
    if (orc_local_matrix(P->xyz, P->el_nodes, P->el_dim, e, P->aniso ? P->aniso + 9 * e : NULL, P->K[e],
                         P->delta[e], A, L->Ainv, &det))
        return -2;
    const int n = E.n;
    L->n = n;
    L->k = n_ngh_e;
    L->m = n + n_ngh_e;
    const double cs = P->delta[e];
    const double meas = elem_measure(&E);
    const int64_t ns = n_sides_of(P), ne = P->n_el;
    double ce[3];
    elem_centre(&E, ce);
    double bE = -1.0 * meas * cs * P->source[e];
    double dEE = 0.0;
    L->lmh_coef = 0.0;
    if (P->time_mode == 1) {
        const double d = -P->storativity[e] * meas / P->dt;
        dEE += d;
        bE += d * P->prev[ns + e];
    } else if (P->time_mode == 2) {
        L->lmh_coef = meas * P->storativity[e] * cs / P->dt / n;
    }
    L->src_side = -1.0 * meas * cs * P->source[e] / n;
    for (int i = 0; i < n; ++i) {
        const int64_t side = P->el_side_start[e] + i;
        L->edges[i] = P->side_edge[side];
        double sc[3];
        side_centre(&E, i, sc);
        double g = ce[2] - sc[2], c = 1.0, F = 0.0, bed = 0.0;
        const int32_t b = P->side_bdr[side];
        if (b >= 0) {
            const double bm = side_measure(&E, i);
            if (P->bc_type[b] == 1) { c = 0.0; g -= P->bc_p[b]; bed += -P->bc_p[b]; F += -1.0; }
            else if (P->bc_type[b] == 2) { bed += P->bc_flux[b] * bm * cs; }
            else if (P->bc_type[b] == 3) { bed += -bm * P->bc_sigma[b] * P->bc_p[b] * cs; F += -bm * P->bc_sigma[b] * cs; }
        }
        if (P->time_mode == 2) {
            F += -L->lmh_coef;
            bed += -L->lmh_coef * P->prev[ns + ne + L->edges[i]];
        }
        L->g[i] = g;
        L->c[i] = c;
        L->f_own[i] = -F;
        L->b_own[i] = -bed;
    }
    for (int j = 0; j < n_ngh_e; ++j) {
        const int64_t ng = ngh_list[j];
        const double v = ngh_value(P, ng, e);
        L->v[j] = v;
        L->edges[n + j] = P->ngh_edge[ng];
        dEE += -v;
    }
    /* S1 = Bt IA B - C ; r1 = Bt IA RHS1 - RHS2 restricted to the element */
    double A1[4], Ag[4], s1 = 0.0, sg = 0.0;
    for (int i = 0; i < n; ++i) {
        A1[i] = 0.0; Ag[i] = 0.0;
        for (int j = 0; j < n; ++j) { A1[i] += L->Ainv[n * i + j]; Ag[i] += L->Ainv[n * i + j] * L->g[j]; }
        s1 += A1[i];
        sg += Ag[i];
    }
    L->s1ee = s1 - dEE;
    L->r1e = -sg - bE;
    for (int i = 0; i < n; ++i) {
        L->u[i] = -L->c[i] * A1[i];
        L->b_own[i] += L->c[i] * Ag[i];
    }
    for (int j = 0; j < n_ngh_e; ++j) L->u[n + j] = -L->v[j];
    return L->m;
}

static double local_s2(const orc_local *L, int a, int b) {
    double s1ff = 0.0;
    if (a < L->n && b < L->n) {
        s1ff = L->c[a] * L->Ainv[L->n * a + b] * L->c[b];
        if (a == b) s1ff += L->f_own[a];
    } else if (a == b) {
        s1ff = L->v[a - L->n];
    }
    return s1ff - L->u[a] * L->u[b] / L->s1ee;
}

static double local_r2(const orc_local *L, int a) {
    double r1f = (a < L->n) ? L->b_own[a] : 0.0;
    return r1f - L->u[a] * L->r1e / L->s1ee;
}

/* element -> its VB neighbours (element_to_neigh_vb order) */
static void neighbour_lists(const orc_problem *P, int32_t *start, int32_t *list) {
    memset(start, 0, (P->n_el + 1) * sizeof(int32_t));
    for (int64_t g = 0; g < P->n_ngh; ++g) start[P->ngh_element[g] + 1]++;
    for (int64_t e = 0; e < P->n_el; ++e) start[e + 1] += start[e];
    int32_t *fill = (int32_t *)malloc((P->n_el + 1) * sizeof(int32_t));
    memcpy(fill, start, (P->n_el + 1) * sizeof(int32_t));
    for (int64_t g = 0; g < P->n_ngh; ++g) list[fill[P->ngh_element[g]]++] = (int32_t)g;
    free(fill);
}

/* Local Schur blocks as COO triplets (row edge, col edge, value) plus rhs triplets.
 * Returns the number of matrix triplets or -1 (cap) / -2 (singular). */
int64_t orc_schur2_coo(const orc_problem *P, int32_t *I, int32_t *J, double *V, int64_t cap, double *rhs) {
    int32_t *start = (int32_t *)malloc((P->n_el + 1) * sizeof(int32_t));
    int32_t *list = (int32_t *)malloc((P->n_ngh + 1) * sizeof(int32_t));
    neighbour_lists(P, start, list);
    memset(rhs, 0, P->n_edges * sizeof(double));
    int64_t k = 0;
    for (int64_t e = 0; e < P->n_el; ++e) {
        orc_local L;
        if (build_local(P, e, list + start[e], start[e + 1] - start[e], &L) < 0) { k = -2; break; }
        for (int a = 0; a < L.m; ++a) {
            rhs[L.edges[a]] += local_r2(&L, a);
            for (int b = 0; b < L.m; ++b) {
                if (k >= cap) { free(start); free(list); return -1; }
                I[k] = L.edges[a];
                J[k] = L.edges[b];
                V[k] = local_s2(&L, a, b);
                ++k;
            }
        }
    }
    free(start);
    free(list);
    return k;
}

/* Values of the second Schur complement on a given CSR pattern (sorted columns per row),
 * threaded over elements with atomic adds: the CPU baseline's assembly.  Returns 0 or -2. */
int orc_schur2_csr(const orc_problem *P, const int32_t *row_ptr, const int32_t *col, double *val, double *rhs) {
    int32_t *start = (int32_t *)malloc((P->n_el + 1) * sizeof(int32_t));
    int32_t *list = (int32_t *)malloc((P->n_ngh + 1) * sizeof(int32_t));
    neighbour_lists(P, start, list);
    memset(val, 0, (size_t)row_ptr[P->n_edges] * sizeof(double));
    memset(rhs, 0, P->n_edges * sizeof(double));
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int64_t e = 0; e < P->n_el; ++e) {
        orc_local L;
        if (build_local(P, e, list + start[e], start[e + 1] - start[e], &L) < 0) { bad = 1; continue; }
        for (int a = 0; a < L.m; ++a) {
            const int32_t r = L.edges[a];
            const double rv = local_r2(&L, a);
#pragma omp atomic
            rhs[r] += rv;
            for (int b = 0; b < L.m; ++b) {
                int32_t lo = row_ptr[r], hi = row_ptr[r + 1] - 1, c = L.edges[b];
                while (lo < hi) {
                    int32_t mid = (lo + hi) / 2;
                    if (col[mid] < c) lo = mid + 1; else hi = mid;
                }
                const double sv = local_s2(&L, a, b);
#pragma omp atomic
                val[lo] += sv;
            }
        }
    }
    free(start);
    free(list);
    return bad ? -2 : 0;
}

/* Back-substitution (SchurComplement::resolve for schur2 then schur1, plus the LMH flux
 * postprocess) into the MH solution vector; sol's edge part must already hold lambda. */
int orc_resolve(const orc_problem *P, double *sol) {
    int32_t *start = (int32_t *)malloc((P->n_el + 1) * sizeof(int32_t));
    int32_t *list = (int32_t *)malloc((P->n_ngh + 1) * sizeof(int32_t));
    neighbour_lists(P, start, list);
    const int64_t ns = n_sides_of(P), ne = P->n_el;
    const double *lam = sol + ns + ne;
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int64_t e = 0; e < P->n_el; ++e) {
        orc_local L;
        if (build_local(P, e, list + start[e], start[e + 1] - start[e], &L) < 0) { bad = 1; continue; }
        double acc = L.r1e;
        for (int a = 0; a < L.m; ++a) acc -= L.u[a] * lam[L.edges[a]];
        const double p = acc / L.s1ee;
        double rhs[4];
        for (int i = 0; i < L.n; ++i) rhs[i] = L.g[i] + p - L.c[i] * lam[L.edges[i]];
        for (int i = 0; i < L.n; ++i) {
            double q = 0.0;
            for (int j = 0; j < L.n; ++j) q += L.Ainv[L.n * i + j] * rhs[j];
            if (P->time_mode == 2)
                q += -L.lmh_coef * (lam[L.edges[i]] - P->prev[ns + ne + L.edges[i]]) + L.src_side;
            sol[P->el_side_start[e] + i] = q;
        }
        sol[ns + e] = p;
    }
    free(start);
    free(list);
    return bad ? -2 : 0;
}

/* ------------------------------------------------------- element flux vectors --------- */
/* Darcy flux vector at each element centre from its side fluxes (DarcyFlowMHOutput::
 * make_element_vector, darcy_flow_mh_output.cc:301-323): u = sum_i q_i RT0_i(c) / delta_e,
 * with the RT0 basis of MHFEValues::RT0_value (mh_fe_values.cc:76-118) and its parameters
 * from the local-matrix routines: line :150-152, triangle :193-211 (bas_func_0_triangle
 * :293-301), tetrahedron :379-396.  out holds 3 values per element. */
static void rt0_at(const Elem *E, const double *x, int s, double *v) {
    double d[3];
    if (E->dim == 1) {
        double lv[3], w[3];
        sub3(E->X[1], E->X[0], lv);
        const double ll = dot3(lv, lv);
        sub3(x, E->X[s == 0 ? 1 : 0], w);
        const double f = (s == 0 ? -norm3(w) : norm3(w)) / ll;
        v[0] = f * lv[0]; v[1] = f * lv[1]; v[2] = f * lv[2];
        return;
    }
    if (E->dim == 2) {
        /* the plane frame of the local matrix: ex along AB, ey in the plane */
        double ex[3], ac[3], ez[3], ey[3], l;
        sub3(E->X[1], E->X[0], ex); l = norm3(ex); ex[0] /= l; ex[1] /= l; ex[2] /= l;
        sub3(E->X[2], E->X[0], ac);
        cross3(ex, ac, ez); l = norm3(ez); ez[0] /= l; ez[1] /= l; ez[2] /= l;
        cross3(ez, ex, ey); l = norm3(ey); ey[0] /= l; ey[1] /= l; ey[2] /= l;
        /* node coordinates in that frame; side s is centred on the node opposite it */
        double nod[3][2];
        for (int k = 0; k < 3; ++k) {
            sub3(E->X[k], E->X[0], d);
            nod[k][0] = k ? dot3(d, ex) : 0.0;
            nod[k][1] = k ? dot3(d, ey) : 0.0;
        }
        const double *p0 = nod[s], *p1 = nod[(s + 1) % 3], *p2 = nod[(s + 2) % 3];
        const double ga = 1.0 / fabs((p0[0] - p2[0]) * (p1[1] - p0[1]) + (p0[1] - p2[1]) * (p0[0] - p1[0]));
        sub3(x, E->X[0], d);
        const double a = dot3(d, ex) - p2[0], b = dot3(d, ey) - p2[1];
        for (int c = 0; c < 3; ++c) v[c] = ga * (a * ex[c] + b * ey[c]);
        return;
    }
    /* tetrahedron: delta_s (x - X_s), X_s the node opposite side s */
    double n[3], c[3];
    side_normal_tet(E, s, n);
    side_centre(E, s, c);
    const double dl = 1.0 / (side_measure(E, s) * (dot3(n, c) - dot3(n, E->X[s])));
    sub3(x, E->X[s], d);
    v[0] = dl * d[0]; v[1] = dl * d[1]; v[2] = dl * d[2];
}

int orc_element_flux(const orc_problem *P, const double *sol, double *out) {
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < P->n_el; ++e) {
        Elem E;
        load_elem(P->xyz, P->el_nodes, P->el_dim, e, &E);
        double c[3], u[3] = {0.0, 0.0, 0.0}, v[3];
        elem_centre(&E, c);
        const double cs = P->delta ? P->delta[e] : 1.0;
        for (int s = 0; s < E.n; ++s) {
            rt0_at(&E, c, s, v);
            const double q = sol[P->el_side_start[e] + s];
            for (int k = 0; k < 3; ++k) u[k] += q * v[k] / cs;
        }
        for (int k = 0; k < 3; ++k) out[3 * e + k] = u[k];
    }
    return 0;
}

/* ------------------------------------------------------------ node pressures ---------- */
/* Pressure at every node (DarcyFlowMHOutput::make_node_scalar_param, darcy_flow_mh_output.cc:
 * 424-546): a distance-weighted mean of the pressures of the elements containing the node and
 * of the sides (of every element) containing it, with weights (1 - d / D) / (n - 1), d the
 * distance from the node to the element or side centre, D the sum of those distances over
 * the node's elements and sides, n their number.  Two passes in element order, as there. */
static double dist3(const double *a, const double *b) {
    double d[3];
    sub3(a, b, d);
    return sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
}

int orc_node_pressure(const orc_problem *P, const double *sol, double *out) {
    const int64_t nn = P->n_nodes, ns = n_sides_of(P);
    int32_t *cnt = (int32_t *)calloc(nn, sizeof(int32_t));
    double *sd = (double *)calloc(nn, sizeof(double));
    for (int64_t i = 0; i < nn; ++i) out[i] = 0.0;
    for (int pass = 0; pass < 2; ++pass) {
        /* elements */
        for (int64_t e = 0; e < P->n_el; ++e) {
            Elem E;
            load_elem(P->xyz, P->el_nodes, P->el_dim, e, &E);
            double c[3];
            elem_centre(&E, c);
            for (int k = 0; k < E.n; ++k) {
                const int32_t nd = P->el_nodes[4 * e + k];
                const double d = dist3(E.X[k], c);
                if (pass == 0) { sd[nd] += d; cnt[nd]++; }
                else out[nd] += sol[ns + e] * (1.0 - d / sd[nd]) / (cnt[nd] - 1);
            }
        }
        /* sides of every element (a line's sides are its nodes: distance 0) */
        for (int64_t e = 0; e < P->n_el; ++e) {
            Elem E;
            load_elem(P->xyz, P->el_nodes, P->el_dim, e, &E);
            for (int s = 0; s < E.n; ++s) {
                double c[3];
                side_centre(&E, s, c);
                const int64_t side = P->el_side_start[e] + s;
                const double p = sol[ns + P->n_el + P->side_edge[side]];
                for (int k = 0; k < E.dim; ++k) {
                    const int ln = side_node(E.dim, s, k);
                    const int32_t nd = P->el_nodes[4 * e + ln];
                    const double d = dist3(E.X[ln], c);
                    if (pass == 0) { sd[nd] += d; cnt[nd]++; }
                    else out[nd] += p * (1.0 - d / sd[nd]) / (cnt[nd] - 1);
                }
            }
        }
    }
    free(cnt);
    free(sd);
    return 0;
}

/* ------------------------------------------------------------ water balance ----------- */
/* DarcyFlowMHOutput::water_balance (darcy_flow_mh_output.cc:671-790): for each boundary region
 * the sum of the side fluxes of its boundary objects (outward positive), of the positive ones
 * and of the negative ones; for each bulk region the sum of |E| delta_E f_E.  bdr_region[b]
 * (for each boundary object b, in topology order) and el_region[e] are region indices;
 * out_bdr[3 r + {0,1,2}] = total, outflow, inflow; out_src[r]. */
int orc_water_balance(const orc_problem *P, const double *sol, const int32_t *bdr_region, int32_t n_bdr_regions,
                      const int32_t *el_region, int32_t n_el_regions, double *out_bdr, double *out_src) {
    const int64_t ns = n_sides_of(P);
    for (int32_t r = 0; r < 3 * n_bdr_regions; ++r) out_bdr[r] = 0.0;
    for (int32_t r = 0; r < n_el_regions; ++r) out_src[r] = 0.0;
    for (int64_t s = 0; s < ns; ++s) {
        const int32_t b = P->side_bdr[s];
        if (b < 0) continue;
        const int32_t r = bdr_region[b];
        const double q = sol[s];
        out_bdr[3 * r] += q;
        if (q > 0) out_bdr[3 * r + 1] += q;
        else out_bdr[3 * r + 2] += q;
    }
    for (int64_t e = 0; e < P->n_el; ++e) {
        Elem E;
        load_elem(P->xyz, P->el_nodes, P->el_dim, e, &E);
        const double delta = P->delta ? P->delta[e] : 1.0, f = P->source ? P->source[e] : 0.0;
        out_src[el_region[e]] += elem_measure(&E) * delta * f;
    }
    return 0;
}

/* ------------------------------------------------------------ Jacobi PCG -------------- */
/* CG with diagonal preconditioning on a CSR SPD matrix, FP64, threaded with OpenMP.  Stops
 * when the recursively updated residual satisfies both |D^-1/2 r| <= rtol |D^-1/2 b| (for
 * Jacobi, r.z is that squared norm) and |r| <= rtol |b|; returns iterations, or -1 if max_it
 * was reached.  res_out gets the true Jacobi-scaled relative residual. */
static void csr_mv(int64_t n, const int32_t *rp, const int32_t *col, const double *val, const double *x, double *y) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double s = 0.0;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) s += val[k] * x[col[k]];
        y[i] = s;
    }
}

int orc_pcg_jacobi(int64_t n, const int32_t *rp, const int32_t *col, const double *val, const double *b, double *x,
                   double rtol, int max_it, double *res_out) {
    double *r = (double *)malloc(n * sizeof(double)), *z = (double *)malloc(n * sizeof(double));
    double *p = (double *)malloc(n * sizeof(double)), *q = (double *)malloc(n * sizeof(double));
    double *dinv = (double *)malloc(n * sizeof(double));
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double d = 1.0;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k)
            if (col[k] == i) d = val[k];
        dinv[i] = 1.0 / d;
    }
    csr_mv(n, rp, col, val, x, q);
    double bb = 0.0, bdb = 0.0, rz = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : bb, bdb, rz)
    for (int64_t i = 0; i < n; ++i) {
        r[i] = b[i] - q[i];
        z[i] = dinv[i] * r[i];
        p[i] = z[i];
        bb += b[i] * b[i];
        bdb += b[i] * dinv[i] * b[i];
        rz += r[i] * z[i];
    }
    const double tol2 = rtol * rtol * bb, tol2s = rtol * rtol * bdb;
    int it = 0;
    double rr = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : rr)
    for (int64_t i = 0; i < n; ++i) rr += r[i] * r[i];
    while ((rr > tol2 || rz > tol2s) && it < max_it) {
        csr_mv(n, rp, col, val, p, q);
        double pq = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : pq)
        for (int64_t i = 0; i < n; ++i) pq += p[i] * q[i];
        const double alpha = rz / pq;
        double rz_new = 0.0;
        rr = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : rz_new, rr)
        for (int64_t i = 0; i < n; ++i) {
            x[i] += alpha * p[i];
            r[i] -= alpha * q[i];
            z[i] = dinv[i] * r[i];
            rz_new += r[i] * z[i];
            rr += r[i] * r[i];
        }
        const double beta = rz_new / rz;
        rz = rz_new;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        ++it;
    }
    csr_mv(n, rp, col, val, x, q);
    double res = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : res)
    for (int64_t i = 0; i < n; ++i) res += (b[i] - q[i]) * dinv[i] * (b[i] - q[i]);
    if (res_out) *res_out = bdb > 0.0 ? sqrt(res / bdb) : 0.0;
    free(r); free(z); free(p); free(q); free(dinv);
    return (rr > tol2 || rz > tol2s) ? -1 : it;
}

/* Incomplete LU factorisation with zero fill, ILU(0), of a CSR matrix whose rows have sorted
 * column indices and a diagonal entry (IKJ form: row i is eliminated with the finished rows
 * k < i inside its own pattern).  For the SPD edge system this is IC(0) in LU form, the
 * zero-fill member of the incomplete factorisations the reference's PETSc solver uses
 * (PCILU with 3 levels of fill, solve.cc:355-374).  lu[nnz] receives L (unit lower, strictly
 * below the diagonal) and U; dpos[n] the diagonal positions.  Returns 0, or -1 for a missing
 * diagonal or a zero pivot. */
int orc_ilu0(int64_t n, const int32_t *rp, const int32_t *col, const double *val, double *lu, int32_t *dpos) {
    int32_t *mark = (int32_t *)malloc(n * sizeof(int32_t));
    int rc = 0;
    for (int64_t i = 0; i < n; ++i) mark[i] = -1;
    memcpy(lu, val, (size_t)rp[n] * sizeof(double));
    for (int64_t i = 0; i < n && !rc; ++i) {
        dpos[i] = -1;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
            mark[col[k]] = k;
            if (col[k] == i) dpos[i] = k;
        }
        if (dpos[i] < 0) {
            rc = -1;
            break;
        }
        for (int32_t k = rp[i]; k < dpos[i]; ++k) {
            const int32_t c = col[k];
            const double f = (lu[k] /= lu[dpos[c]]);
            for (int32_t j = dpos[c] + 1; j < rp[c + 1]; ++j) {
                const int32_t m = mark[col[j]];
                if (m >= 0) lu[m] -= f * lu[j];
            }
        }
        if (lu[dpos[i]] == 0.0) rc = -1;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) mark[col[k]] = -1;
    }
    free(mark);
    return rc;
}

/* z = (LU)^-1 r: forward substitution with the unit lower factor, then backward with U. */
static void ilu0_apply(int64_t n, const int32_t *rp, const int32_t *col, const double *lu, const int32_t *dpos,
                       const double *r, double *z) {
    for (int64_t i = 0; i < n; ++i) {
        double s = r[i];
        for (int32_t k = rp[i]; k < dpos[i]; ++k) s -= lu[k] * z[col[k]];
        z[i] = s;
    }
    for (int64_t i = n - 1; i >= 0; --i) {
        double s = z[i];
        for (int32_t k = dpos[i] + 1; k < rp[i + 1]; ++k) s -= lu[k] * z[col[k]];
        z[i] = s / lu[dpos[i]];
    }
}

/* CG preconditioned by ILU(0) on a CSR SPD matrix, FP64: the SpMV and the vector updates are
 * threaded, the two triangular solves sequential.  The same stopping rule as orc_pcg_jacobi:
 * the recursively updated residual satisfies |D^-1/2 r| <= rtol |D^-1/2 b| and
 * |r| <= rtol |b|.  Returns iterations, -1 if max_it was reached, -2 if the factorisation
 * failed; res_out gets the true Jacobi-scaled relative residual and t_factor_out the
 * factorisation's seconds. */
int orc_pcg_ilu0(int64_t n, const int32_t *rp, const int32_t *col, const double *val, const double *b, double *x,
                 double rtol, int max_it, double *res_out, double *t_factor_out) {
    extern double omp_get_wtime(void);
    double *lu = (double *)malloc((size_t)rp[n] * sizeof(double));
    int32_t *dpos = (int32_t *)malloc(n * sizeof(int32_t));
    const double t0 = omp_get_wtime();
    if (orc_ilu0(n, rp, col, val, lu, dpos)) {
        free(lu); free(dpos);
        return -2;
    }
    if (t_factor_out) *t_factor_out = omp_get_wtime() - t0;
    double *r = (double *)malloc(n * sizeof(double)), *z = (double *)malloc(n * sizeof(double));
    double *p = (double *)malloc(n * sizeof(double)), *q = (double *)malloc(n * sizeof(double));
    double *dinv = (double *)malloc(n * sizeof(double));
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) dinv[i] = 1.0 / val[dpos[i]];
    csr_mv(n, rp, col, val, x, q);
    double bb = 0.0, bdb = 0.0, rr = 0.0, rdr = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : bb, bdb, rr, rdr)
    for (int64_t i = 0; i < n; ++i) {
        r[i] = b[i] - q[i];
        bb += b[i] * b[i];
        bdb += b[i] * dinv[i] * b[i];
        rr += r[i] * r[i];
        rdr += r[i] * dinv[i] * r[i];
    }
    ilu0_apply(n, rp, col, lu, dpos, r, z);
    double rz = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : rz)
    for (int64_t i = 0; i < n; ++i) {
        p[i] = z[i];
        rz += r[i] * z[i];
    }
    const double tol2 = rtol * rtol * bb, tol2s = rtol * rtol * bdb;
    int it = 0;
    while ((rr > tol2 || rdr > tol2s) && it < max_it) {
        csr_mv(n, rp, col, val, p, q);
        double pq = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : pq)
        for (int64_t i = 0; i < n; ++i) pq += p[i] * q[i];
        const double alpha = rz / pq;
        rr = 0.0;
        rdr = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : rr, rdr)
        for (int64_t i = 0; i < n; ++i) {
            x[i] += alpha * p[i];
            r[i] -= alpha * q[i];
            rr += r[i] * r[i];
            rdr += r[i] * dinv[i] * r[i];
        }
        ilu0_apply(n, rp, col, lu, dpos, r, z);
        double rz_new = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : rz_new)
        for (int64_t i = 0; i < n; ++i) rz_new += r[i] * z[i];
        const double beta = rz_new / rz;
        rz = rz_new;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        ++it;
    }
    csr_mv(n, rp, col, val, x, q);
    double res = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : res)
    for (int64_t i = 0; i < n; ++i) res += (b[i] - q[i]) * dinv[i] * (b[i] - q[i]);
    if (res_out) *res_out = bdb > 0.0 ? sqrt(res / bdb) : 0.0;
    free(r); free(z); free(p); free(q); free(dinv); free(lu); free(dpos);
    return (rr > tol2 || rdr > tol2s) ? -1 : it;
}

/* OpenMP threads of the following oracle calls (the CPU baseline's 1-core figure). */
void orc_set_threads(int n) {
#ifdef _OPENMP
    extern void omp_set_num_threads(int);
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int orc_num_threads(void) {
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    return omp_get_max_threads();
#else
    return 1;
#endif
}
