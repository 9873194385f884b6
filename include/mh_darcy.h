/*
 * mh_darcy.h -- C ABI of the B200 mixed-hybrid (MH) Darcy flow library.
 *
 * The library replaces the MH Darcy hot path of Flow123d 1.7:
 *   assembly of the saddle-point system  (src/flow/darcy_flow_mh.cc:525-694,
 *                                          src/flow/mh_fe_values.cc:34-514)
 *   first Schur complement (face fluxes)  (darcy_flow_mh.cc:1009-1090, src/la/schur.cc:566-611)
 *   second Schur complement (pressures)   (darcy_flow_mh.cc:1095-1131)
 *   iterative solve of the edge system    (src/la/solve.cc:316-466)
 *   back-substitution                     (src/la/schur.cc:714-773, darcy_flow_mh.cc:414-415)
 *   unsteady time term                    (darcy_flow_mh.cc:1614-1827)
 * on one GPU.  All entry points are plain C: pointers, sizes and int status codes.
 * Caller-owned host arrays are copied in and never retained; device memory is owned
 * by the opaque handle.  Every function returns MH_OK (0), a positive "solved with a
 * caveat" code, or a negative error code; nothing aborts.
 *
 * Numbering conventions follow the reference exactly:
 *   - elements in input order; element sides numbered element-major
 *     (MH_DofHandler::reinit, src/flow/mh_dofhandler.cc:12-24);
 *   - side i of a simplex is the face opposite node i for tetrahedra and
 *     {0,1},{1,2},{0,2} for triangles (src/mesh/ref_element.cc:51-76);
 *   - edges (groups of coincident sides) and boundary objects in the creation order of
 *     Mesh::make_neighbours_and_edges (src/mesh/mesh.cc:343-500);
 *   - the solution vector is [side fluxes | element pressures | edge pressures]
 *     (darcy_flow_mh.cc:337-355, mh_dofhandler.cc:37-50).
 */
#ifndef MH_DARCY_H
#define MH_DARCY_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------ */
#define MH_OK               0
#define MH_NOT_CONVERGED    1   /* max_it reached; the result is the last iterate        */
#define MH_FELL_BACK        2   /* converged, but only after a fallback (see fell_back)   */
#define MH_ERR_INVALID     -1   /* bad argument, inconsistent mesh                        */
#define MH_ERR_SINGULAR    -2   /* singular local MH block (|det| < DBL_MIN/DBL_EPSILON)  */
#define MH_ERR_CUDA        -3   /* CUDA runtime error or no device                        */
#define MH_ERR_STATE       -4   /* call out of order (e.g. solve before set_coeffs)       */
#define MH_ERR_NOMEM       -5
#define MH_ERR_NONFINITE   -6   /* NaN/Inf in coefficients or in the iteration            */
#define MH_ERR_TOPOLOGY    -7   /* the mesh violates a rule of the reference topology     */
#define MH_ERR_BREAKDOWN   -8   /* CG breakdown (p'Sp <= 0): system not SPD               */
#define MH_ERR_IO          -9   /* a file cannot be opened or read                        */

/* ---- boundary condition types (DarcyFlowMH::EqData::BC_Type, darcy_flow_mh.cc:81-87) --- */
#define MH_BC_NONE       0
#define MH_BC_DIRICHLET  1
#define MH_BC_NEUMANN    2
#define MH_BC_ROBIN      3

/* ---- solver methods ------------------------------------------------------------------ */
#define MH_SOLVER_PCG64     0   /* Jacobi-preconditioned CG, all FP64                     */
#define MH_SOLVER_IR32      1   /* FP32 inner CG inside FP64 iterative refinement         */
#define MH_SOLVER_CHEB      2   /* Chebyshev-Jacobi polynomial preconditioner in flexible CG:
                                   FP32 inner iteration, FP64 residual replacements       */
#define MH_SOLVER_FCG_LEARNED 3 /* learned (message-passing) preconditioner in flexible CG,
                                   FP32 inner, FP64 replacements; falls back to Chebyshev-
                                   Jacobi when the learned iteration stalls              */
#define MH_SOLVER_AMG       4   /* aggregation multigrid V-cycle in flexible CG: FP32 inner,
                                   FP64 residual replacements; hierarchy built on the GPU
                                   from the current matrix at every solve                */

typedef struct mh_handle mh_handle;
typedef struct mh_mesh mh_mesh;

/* Flat description of a mixed 1D/2D/3D simplicial mesh.  Element and boundary-element
 * node lists have 4 slots per element; unused slots are -1.  Boundary elements are the
 * explicit ones of a gmsh file (regions whose name starts with '.'); implicit boundary
 * objects are created for every outer side without one, as in mesh.cc:445-472. */
typedef struct mh_mesh_desc {
    int64_t        n_nodes;
    const double  *node_xyz;     /* [n_nodes*3]                                   */
    int64_t        n_elements;
    const int32_t *el_dim;       /* [n_elements], 1..3                            */
    const int32_t *el_nodes;     /* [n_elements*4]                                */
    int64_t        n_bc_elements;
    const int32_t *bc_dim;       /* [n_bc_elements], 0..2 (may be NULL if 0)      */
    const int32_t *bc_nodes;     /* [n_bc_elements*4]                             */
} mh_mesh_desc;

typedef struct mh_sizes {
    int64_t n_nodes, n_elements, n_sides, n_edges, n_boundaries, n_neighbours;
    int64_t n_el_dim[4];         /* elements per dimension                       */
    int64_t mh_size;             /* n_sides + n_elements + n_edges               */
    int64_t schur_nnz;           /* nonzeros of the edge (second Schur) system   */
    int64_t sell_slots;          /* stored SELL-C-sigma slots incl. padding       */
    int64_t n_rows_padded;       /* solver rows incl. per-instance padding        */
    int64_t n_instances;
} mh_sizes;

/* Element-wise coefficient fields (EqData, darcy_flow_mh.cc:154-183).  NULL selects the
 * reference default: anisotropy = I, cross_section = 1, conductivity = 1, sigma = 1,
 * water_source_density = 0, storativity = 1. */
typedef struct mh_coeffs {
    const double *conductivity;          /* [n_elements]                          */
    const double *anisotropy;            /* [n_elements*9] row-major 3x3 tensor   */
    const double *cross_section;         /* [n_elements]                          */
    const double *sigma;                 /* [n_elements] (used on lower-dim elem) */
    const double *water_source_density;  /* [n_elements]                          */
    const double *storativity;           /* [n_elements] (unsteady only)          */
} mh_coeffs;

/* Boundary data per boundary object (assembly_steady_mh_matrix, darcy_flow_mh.cc:570-596).
 * Arrays may be NULL when no boundary uses them. */
typedef struct mh_bc {
    const int32_t *type;          /* [n_boundaries] MH_BC_*                        */
    const double  *pressure;      /* Dirichlet / Robin pressure                    */
    const double  *flux;          /* Neumann flux                                  */
    const double  *robin_sigma;   /* Robin transfer coefficient                    */
} mh_bc;

/* Convergence is judged on the FP64 true residual r = b - S x of the edge system S x = b:
 * both the Jacobi-scaled relative residual |D^-1/2 r|/|D^-1/2 b| (D = diag S; the norm
 * PETSc's preconditioned CG monitors) and the unscaled |r|/|b| must be <= r_tol, or
 * |r| <= a_tol. */
typedef struct mh_solve_opts {
    int32_t method;         /* MH_SOLVER_*                                          */
    int32_t max_it;         /* cap on (inner) iterations, default 20000              */
    double  r_tol;          /* relative tolerance (default 1e-10)                    */
    double  a_tol;          /* absolute tolerance on |b - S x| (default 0)           */
    int32_t use_initial_guess;  /* start from the current edge pressures             */
    int32_t cheb_degree;    /* MH_SOLVER_CHEB: polynomial degree (default 4)         */
    double  inner_rtol;     /* FP32 residual reduction between two FP64 residual
                               replacements; 0: 1e-3 for MH_SOLVER_AMG and
                               MH_SOLVER_FCG_LEARNED, else 0.1                       */
    int32_t inner_max_it;   /* FP32 iterations between two replacements at most (2000;
                               after the learned method fell back, at least 200)     */
    int32_t iters_per_graph;/* Krylov iterations per captured CUDA graph launch; 0:
                               16, or 4 for the multigrid methods (long iterations)  */
    int32_t profile_kernels;/* 1: time every Krylov kernel with CUDA events in-graph */
    int32_t host_loop;      /* 0: each Krylov run is one graph launch whose iterations
                               repeat on the device (a conditional loop that ends when
                               every instance is done); 1: graphs of iters_per_graph
                               iterations launched while the host sees one running   */
    int32_t reserved[5];
} mh_solve_opts;

/* kernel classes of mh_solve_stats.kernel_ms / kernel_count */
#define MH_KERNEL_SPMV64   0
#define MH_KERNEL_UPDATE64 1
#define MH_KERNEL_SPMV32   2
#define MH_KERNEL_UPDATE32 3
#define MH_KERNEL_SMOOTH0  4   /* MH_SOLVER_AMG: a Chebyshev smoothing step on the fine level */
#define MH_KERNEL_VCYCLE   5   /* MH_SOLVER_AMG: one whole V-cycle (all its kernels)          */
#define MH_KERNEL_CLASSES  6

typedef struct mh_solve_stats {
    int32_t status;
    int32_t iterations;         /* total Krylov iterations (inner ones for IR)       */
    int32_t outer_iterations;   /* refinement steps (IR/FCG), restarts (PCG)          */
    int32_t fell_back;          /* 1: IR32 stalled and finished in FP64 PCG, or the
                                   learned preconditioner stalled -> Chebyshev-Jacobi */
    double  rel_residual;       /* final Jacobi-scaled relative FP64 true residual    */
    double  ms_assembly;        /* device time of the last assembly                   */
    double  ms_solve;           /* device time of the Krylov solve                    */
    double  ms_backsub;         /* device time of back-substitution                   */
    double  rel_residual_unscaled; /* final |b - S x| / |b|                           */
    int64_t kernel_launches;    /* kernels launched by this call (graph nodes too)    */
    double  kernel_ms[MH_KERNEL_CLASSES];    /* with profile_kernels: summed device time */
    int32_t kernel_count[MH_KERNEL_CLASSES]; /* of the launches that did work, per class */
    double  ms_setup;           /* device time of the preconditioner setup (AMG), part
                                   of ms_solve                                         */
    double  reserved[3];
} mh_solve_stats;

/* ---- library ---------------------------------------------------------------------- */
const char *mh_version(void);
const char *mh_status_string(int status);
/* 1 if a CUDA device usable by the library is present, else 0. */
int mh_device_available(void);
/* Message of the last error recorded on a handle (empty if none). */
const char *mh_last_error(const mh_handle *h);

/* ---- synthetic meshes: unit cube of n^3 cubes, 6 Kuhn tetrahedra each -------------- */
/* Fracture planes: axis (0=x,1=y,2=z) at grid index; each adds the 2n^2 coincident face
 * triangles.  Channels: 1D segments along axis `line_axis` through grid indices
 * (line_a, line_b) of the two other axes in increasing axis order.  Element order:
 * tetrahedra (cube-major, x fastest), then triangles plane by plane, then segments. */
int mh_cube_mesh_create(int32_t n, int32_t n_planes, const int32_t *plane_axis,
                        const int32_t *plane_index, int32_t n_lines, const int32_t *line_axis,
                        const int32_t *line_a, const int32_t *line_b, mh_mesh **out);
int mh_mesh_describe(const mh_mesh *m, mh_mesh_desc *desc);
void mh_mesh_destroy(mh_mesh *m);

/* ---- gmsh 2.2 ASCII input (GmshMeshReader, src/mesh/msh_gmshreader.cc) -------------- */
/* Reads $PhysicalNames, $Nodes and $Elements (read_mesh, msh_gmshreader.cc:75-244) into a
 * mesh for mh_create.  Elements of types 1, 2, 4 and 15 (line, triangle, tetrahedron,
 * point) with at least two tags; the first tag is the physical region, the third (if any)
 * the partition.  Regions follow RegionDB::add_region (src/mesh/region.cc:107-175): a named
 * region is a boundary region when its name starts with '.', an id met only in $Elements
 * becomes the bulk region "region_<id>", and an element whose dimension differs from its
 * region's is an error.  Elements of boundary regions become boundary elements, the others
 * bulk elements (points in bulk regions are skipped), both in file order.  Empty lines and
 * lines starting with '#' are skipped and tokens may be quoted (Tokenizer,
 * src/system/tokenizer.cc).  Node ids may be sparse; a repeated node or element id is an
 * error.  Returns MH_ERR_IO when the file cannot be read and MH_ERR_INVALID for a format
 * error; the message (file line included) goes to err[err_len] when err is not NULL. */
int mh_gmsh_read(const char *path, mh_mesh **out, char *err, size_t err_len);

typedef struct mh_gmsh_info {
    const int64_t *node_id;            /* [n_nodes] ids of the file                       */
    const int64_t *el_id;              /* [n_elements]                                   */
    const int32_t *el_region;          /* [n_elements] physical id                       */
    const int32_t *el_partition;       /* [n_elements] third tag, 0 if absent            */
    const int64_t *bc_id;              /* [n_bc_elements]                                */
    const int32_t *bc_region;          /* [n_bc_elements]                                */
    int32_t        n_regions;          /* $PhysicalNames in file order, then the regions
                                          met only in $Elements, in order of appearance  */
    const int32_t *region_id;
    const int32_t *region_dim;
    const int32_t *region_boundary;    /* 1 for a boundary region                        */
    const char *const *region_name;
} mh_gmsh_info;
/* Ids and regions of a mesh read by mh_gmsh_read (MH_ERR_INVALID for other meshes).  The
 * arrays live as long as the mesh. */
int mh_gmsh_info_get(const mh_mesh *m, mh_gmsh_info *info);

/* Values of the element field `field` at `time` for the elements with ids el_ids[n_ids]
 * (strictly ascending), n_components per element, into out[n_ids*n_components]
 * (GmshMeshReader::read_element_data, msh_gmshreader.cc:251-396): the $ElementData
 * sections of the field are taken in file order while their time is <= time*(1 + 2 eps),
 * each overwriting the elements it lists; a row "id v_1 .. v_n" is matched against el_ids
 * with a pointer that only moves forward, rows of other ids are skipped, and a row past the
 * last id ends its section.  Elements no section lists stay NaN.  A section's own component
 * and entity counts are only used to find its rows.  MH_ERR_INVALID when the file has no
 * section of the field, none at or before `time`, or a row that is read has fewer than
 * n_components values or a malformed number. */
int mh_gmsh_element_data(const char *path, const char *field, double time, int64_t n_ids,
                         const int64_t *el_ids, int32_t n_components, double *out, char *err,
                         size_t err_len);

/* ---- the MH system (DarcyFlowMH_Steady, darcy_flow_mh.cc:249-433) ------------------- */
/* Builds edges, boundaries and VB neighbours on the host (Mesh::setup_topology,
 * mesh.cc:227-245, 343-500, 660-685) and uploads mesh, connectivity and the Schur
 * pattern to the current CUDA device.  With no device the handle still builds the
 * topology (mh_get_sizes/mh_get_topology work) and compute calls return MH_ERR_CUDA. */
int mh_create(const mh_mesh_desc *mesh, mh_handle **out);
void mh_destroy(mh_handle *h);
/* Runs all further work of the handle on the caller's cudaStream_t (NULL: the handle's own
 * stream).  Every call still returns only after its work on that stream is complete. */
int mh_set_stream(mh_handle *h, void *cuda_stream);
/* Kernels launched by the handle so far (the graph nodes of captured iterations included). */
int64_t mh_kernel_launches(const mh_handle *h);
int mh_get_sizes(const mh_handle *h, mh_sizes *out);
/* Topology export (any pointer may be NULL):
 *   el_side_start [n_elements+1]  first global side of each element
 *   side_edge     [n_sides]       edge of each side
 *   side_bdr      [n_sides]       boundary object of each side or -1
 *   bdr_bc_element[n_boundaries]  explicit boundary element or -1 (implicit)
 *   bdr_edge      [n_boundaries]
 *   ngh_element   [n_neighbours]  lower-dimensional element of a VB neighbour
 *   ngh_edge      [n_neighbours]  edge holding the single higher-dimensional side
 *   ngh_side      [n_neighbours]  that side                                         */
int mh_get_topology(const mh_handle *h, int32_t *el_side_start, int32_t *side_edge,
                    int32_t *side_bdr, int32_t *bdr_bc_element, int32_t *bdr_edge,
                    int32_t *ngh_element, int32_t *ngh_edge, int32_t *ngh_side);

int mh_set_coeffs(mh_handle *h, const mh_coeffs *c);
int mh_set_bc(mh_handle *h, const mh_bc *bc);

/* K1: local RT0 matrices, FP64 inversion, both Schur eliminations and the SELL scatter
 * (assembly_steady_mh_matrix + make_schur1 + make_schur2). */
int mh_assemble(mh_handle *h);
/* Krylov solve of the edge system followed by back-substitution (K2-K5 + K4). */
int mh_solve(mh_handle *h, const mh_solve_opts *opts, mh_solve_stats *stats);
/* Copies the MH solution [sides | elements | edges] (length mh_size) to the host. */
int mh_get_solution(const mh_handle *h, double *out, int64_t len);
/* Same, into a device buffer (a plain device pointer). */
int mh_get_solution_device(const mh_handle *h, double *dev_out, int64_t len);
/* Darcy flux vector at every element centre from the side fluxes of the last solution,
 * out[3 e + k] for k = x, y, z (length 3 n_elements): DarcyFlowMHOutput::make_element_vector
 * (src/flow/darcy_flow_mh_output.cc:301-323), the three flux columns of the raw output.
 * Computed on the device; MH_ERR_STATE until a solve follows the last mh_set_coeffs. */
int mh_get_element_flux(const mh_handle *h, double *out, int64_t len);
/* Same, written directly into a device buffer (a plain device pointer); nothing allocated. */
int mh_get_element_flux_device(const mh_handle *h, double *dev_out, int64_t len);
/* Pressure at every node (length n_nodes) from the last solution: the distance-weighted mean
 * of the pressures of the elements and element sides containing the node,
 * DarcyFlowMHOutput::make_node_scalar_param (src/flow/darcy_flow_mh_output.cc:424-546).
 * Computed on the device; MH_ERR_STATE until a solve follows the last mh_set_coeffs. */
int mh_get_node_pressure(const mh_handle *h, double *out, int64_t len);
/* Water balance of the last solution, DarcyFlowMHOutput::water_balance
 * (src/flow/darcy_flow_mh_output.cc:671-790).  bdr_region [n_boundaries] (the boundary objects
 * in mh_get_topology's order) and el_region [n_elements] are region indices in
 * [0, n_bdr_regions) and [0, n_el_regions).  bdr_out [3 n_bdr_regions]: per boundary region
 * the sum of the outward side fluxes, of the positive ones (outflow) and of the negative ones
 * (inflow); src_out [n_el_regions]: per bulk region the sum of |E| cross_section f.  Computed
 * on the device; MH_ERR_INVALID for an index out of range, MH_ERR_STATE until a solve
 * follows the last mh_set_coeffs. */
int mh_water_balance(const mh_handle *h, const int32_t *bdr_region, int32_t n_bdr_regions,
                     const int32_t *el_region, int32_t n_el_regions, double *bdr_out, double *src_out);
/* Convection matrix of the explicit finite-volume transport from the side fluxes of the last
 * solution, ConvectionTransport::create_transport_matrix_mpi (src/transport/transport.cc:
 * 788-923): a CSR matrix [n_elements x n_elements] with the reference's entries (a zero
 * entry wherever the reference inserts one), columns ascending in each row, and
 * cfl_max_step = 1 / max |a_ii|.  porosity [n_elements] (the transport's por_m) may be NULL
 * (1).  Call with row_ptr, col, val and cfl_max_step all NULL to get *nnz; then row_ptr
 * [n_elements+1], col [nnz], val [nnz] (any may be NULL).  The pattern is built on the first
 * call; the values are computed on the device.  MH_ERR_STATE until a solve follows the last
 * mh_set_coeffs. */
int mh_transport_matrix(const mh_handle *h, const double *porosity, int64_t *nnz, int32_t *row_ptr,
                        int32_t *col, double *val, double *cfl_max_step);
/* Same values into a device buffer (len >= nnz, in the CSR order of mh_transport_matrix);
 * dev_porosity is a device pointer or NULL.  Nothing is copied to the host but the CFL step. */
int mh_transport_matrix_device(const mh_handle *h, const double *dev_porosity, double *dev_val,
                               int64_t len, double *cfl_max_step);
/* Writes (append = 0) or appends one "$FlowField" block of the flow field text output,
 * DarcyFlowMHOutput::output_internal_flow_data (src/flow/darcy_flow_mh_output.cc:793-829):
 * per element its id (el_id, or the element index when null), pressure, centre flux vector,
 * number of sides, side pressures and side fluxes, printed "%.8g " as the reference does.
 * Host arrays only (no device, no handle): solution as from mh_get_solution, el_flux as from
 * mh_get_element_flux, el_side_start [n_el+1] and side_edge as from mh_get_topology. */
int mh_raw_output_write(const char *path, int append, double time, int64_t n_el, const int32_t *el_id,
                        const int32_t *el_side_start, const int32_t *side_edge, const double *solution,
                        const double *el_flux);

/* Export of the assembled edge system in CSR form (rows = edges), for checking.  The
 * values are the reference's schur2 matrix after scale(-1) (darcy_flow_mh.cc:1128-1130),
 * rhs likewise.  row_ptr [n_edges+1], col/val [schur_nnz], rhs [n_edges]. */
int mh_get_schur_system(const mh_handle *h, int32_t *row_ptr, int32_t *col, double *val,
                        double *rhs);

/* Fills opts with defaults. */
void mh_solve_opts_default(mh_solve_opts *opts);

/* ---- batches of independent systems ---------------------------------------------------- */
/* n_inst independent meshes (for example conductivity realisations on meshes of uneven
 * size) in one handle.  Every Krylov launch covers all instances; each instance keeps its own
 * CG coefficients and stops on its own residual (per-instance masks); mh_solve returns when
 * all have finished.  Element-wise arrays (mh_set_coeffs), boundary arrays (mh_set_bc) and the
 * MH solution cover the union: each part is the concatenation over instances in order, i.e.
 * the solution is [sides of inst 0, 1, ... | elements of 0, 1, ... | edges of 0, 1, ...]. */
int mh_create_batch(const mh_mesh_desc *meshes, int32_t n_inst, mh_handle **out);
/* Offsets [n_inst+1] of each instance's elements, sides, edges and boundary objects in the
 * union numbering (any pointer may be NULL). */
int mh_get_instance_offsets(const mh_handle *h, int64_t *el_off, int64_t *side_off, int64_t *edge_off,
                            int64_t *bdr_off);
/* Per-instance results of the last solve: Krylov iterations, final Jacobi-scaled relative
 * residual, status (0 converged, 1 not converged, < 0 breakdown).  Arrays of n_inst. */
int mh_get_instance_stats(const mh_handle *h, int32_t *iterations, double *rel_residual, int32_t *status);

/* ---- mortar coupling of non-matching 1D and 2D elements ---------------------------------- */
/* The reference couples a 1D element to 2D elements that do not share its nodes through the
 * intersections read from its neighbouring file (Mesh::read_intersections, src/mesh/mesh.cc:
 * 703-755) with mortar_method P0 (coupling_P0_mortar_assembly, src/flow/darcy_flow_mh.cc:
 * 698-799) or P1 (mh_abstract_assembly_intersection, :815-937), with the coefficient
 * mortar_sigma.  Intersection k: the 1D master element master[k], the 2D slave element
 * slave[k] (element indices), and its two points X, Y given by their local coordinates on the
 * master, master_t[2k] and [2k+1] (0 and 1 at the line's nodes 0 and 1), and on the slave,
 * slave_xy[4k], [4k+1] for X and [4k+2], [4k+3] for Y (t0, t1 with nodes 0, 1, 2 at (0,0),
 * (1,0), (0,1)), as in the file's intersection points. */
#define MH_MORTAR_NONE 0
#define MH_MORTAR_P0   1
#define MH_MORTAR_P1   2
typedef struct mh_mortar_desc {
    int32_t        method;    /* MH_MORTAR_*                                               */
    double         sigma;     /* mortar_sigma                                              */
    int64_t        n;         /* intersections                                             */
    const int32_t *master;    /* [n]                                                       */
    const int32_t *slave;     /* [n]                                                       */
    const double  *master_t;  /* [2n]                                                      */
    const double  *slave_xy;  /* [4n]                                                      */
} mh_mortar_desc;
/* mh_create with the mortar blocks of the intersections added to the edge system at every
 * assembly (their pattern is part of the layout).  MH_ERR_INVALID for a pair that is not
 * (1D master, 2D slave) or an index out of range. */
int mh_create_mortar(const mh_mesh_desc *mesh, const mh_mortar_desc *mortar, mh_handle **out);

/* Autotuner: times `iterations` FP64 and FP32 CG iterations on the assembled system for
 * every launch shape (rows per thread R in {1, 2, 4}, blocks per SM from the occupancy of
 * that R's SpMV kernels) and keeps the fastest.  Writes the chosen R and the FP32 and FP64
 * microseconds per iteration (either pointer may be NULL). */
int mh_autotune(mh_handle *h, int32_t iterations, int32_t *rows_per_thread, double *us_per_iter);

/* The launch shapes mh_autotune_ex chose. */
typedef struct mh_tune_result {
    int32_t rows_per_thread;    /* R of the Krylov kernels (mh_autotune)                  */
    int32_t sell_rows_per_warp; /* rows one warp's SELL-32 tile covers: 32 R              */
    int32_t k1_group;           /* elements per K1 block (one per thread): 64, 128 or 256;
                                   0 for a general system (mh_csr_create: no assembly)      */
    int32_t amg_fine_passes;    /* multigrid pairing passes from the fine level: 2 or 3
                                   (0: not tuned, MH_AMG_PASSES set)                       */
    double  us_per_iter_fp32;   /* FP32 CG iteration at R                                  */
    double  us_per_iter_fp64;   /* FP64 CG iteration at R                                  */
    double  us_assembly;        /* K1 + gather at k1_group (median of three)               */
    double  ms_amg_solve;       /* complete MH_SOLVER_AMG solve (setup included), host clock,
                                   at amg_fine_passes                                       */
    double  reserved[2];
} mh_tune_result;

/* mh_autotune, then the element group of the assembly's K1 kernel (the matrix and rhs are
 * assembled again, same values, three times per group size; the fastest median is kept for
 * every later assembly), then the multigrid's pairing passes from the fine level (2 or 3: two
 * complete MH_SOLVER_AMG solves of the assembled system each, hierarchy rebuilt; the faster is
 * kept for the handle's later multigrid solves).  The solves overwrite the solution. */
int mh_autotune_ex(mh_handle *h, int32_t iterations, mh_tune_result *out);

/* ---- unsteady MH (DarcyFlowMH_Unsteady, darcy_flow_mh.cc:1601-1675) ----------------- */
/* lumped = 0: MH time term on element rows (setup_time_term :1614-1658);
 * lumped = 1: LMH time term on edge rows (DarcyFlowLMH_Unsteady :1695-1827).
 * init_pressure [n_elements] may be NULL (zero). */
int mh_unsteady_init(mh_handle *h, int32_t lumped, double dt, const double *init_pressure);
/* One implicit-Euler step of length dt with the boundary data currently set. */
int mh_unsteady_step(mh_handle *h, double dt, const mh_solve_opts *opts,
                     mh_solve_stats *stats);

/* ---- learned preconditioner (MH_SOLVER_FCG_LEARNED) ---------------------------------- */
/* No counterpart in the reference, which preconditions the Schur system with PETSc ILU
 * (src/la/solve.cc).  The learned method is the aggregation multigrid of MH_SOLVER_AMG whose
 * fine-level smoother is Chebyshev on diag(w) S^, with the weights w given by a message-
 * passing network over the Jacobi-scaled edge system S^ (off-diagonal o_ij):
 *   x_i = (1, sum|o_ij|, max|o_ij|, sum o_ij, sum max(o_ij,0), nnz_i/8, sum o_ij^2, [nnz_i = 0])
 *   h0 = relu(W0 x + b0)                                  8 -> 32
 *   3 layers: h = h + relu(W_l [h ; A h] + b_l),  A_ij = |o_ij|       64 -> 32 (bf16 tensor
 *                                                                     cores, fp32 sums)
 *   w_i = exp(ln2 tanh(w_out . h_i + b_out))              w in [1/2, 2]
 * The network reads the matrix, not the residual: during a solve the preconditioner is a
 * fixed symmetric positive definite operator (the V-cycle), so flexible CG keeps its
 * guarantees.  A new handle starts from random hidden layers and a zero output layer: w = 1,
 * the plain multigrid.  MH_NN_PARAMS floats: W0 [32][8], b0 [32], per layer W_l [32][64],
 * b_l [32], then w_out [32], b_out [1] (row-major). */
#define MH_NN_PARAMS 6561
int mh_learned_set_weights(mh_handle *h, const float *w, int64_t n);
int mh_learned_get_weights(const mh_handle *h, float *w, int64_t n);
/* Back to the parameters a new handle starts from (w = 1) and a fresh Adam state. */
int mh_learned_reset(mh_handle *h);

/* Loss and parameter gradient of one training pair (r, e) on the assembled system, for
 * checking the training kernels: r, e [n_edges] in edge order, in the Jacobi-scaled space
 * (S^ e = r for an exact pair).  loss = (M r - e)' S^ (M r - e) / (e' S^ e) with M the
 * training V-cycle (no energy-optimal coarse scaling, FP32 fine values) and the network's
 * smoother weights; grad [MH_NN_PARAMS] = d loss / d parameters, with the smoothing interval
 * held at its estimate for the current weights. */
int mh_learned_grad(mh_handle *h, const double *r, const double *e, float *grad, double *loss);
/* The same evaluation, returning dw [n_edges] = d loss / d w (the cycle's adjoint) and the
 * weights w [n_edges] (either may be NULL).  refresh = 0 keeps the smoothing interval of the
 * previous evaluation (so that finite differences see the same function the gradient is of);
 * refresh = 1 re-estimates it for the current weights. */
int mh_learned_grad_weights(mh_handle *h, const double *r, const double *e, int32_t refresh, float *dw, float *w,
                            double *loss);
/* The network's smoother weights for the assembled system: w [n_edges] in edge order. */
int mh_learned_smoother(mh_handle *h, float *w, int64_t n);
/* z = M r: one application of the learned preconditioner (the solver's V-cycle with the
 * network's smoother weights); r, z [n_edges] in edge order, Jacobi-scaled space. */
int mh_learned_apply(mh_handle *h, const double *r, double *z);

typedef struct mh_learn_opts {
    int32_t n_pairs;        /* training pairs: snapshots of the plain solver (default 12) */
    int32_t epochs;         /* passes over the pairs, one Adam step per pair (default 40) */
    float   lr;             /* Adam step size (default 2e-3)                          */
    int32_t train_bias;     /* unused (every parameter is trained)                    */
    double  solve_rtol;     /* accuracy of the reference solution x* (default 1e-9)   */
    uint64_t seed;          /* order of the pairs within an epoch                     */
    int32_t reserved[6];
} mh_learn_opts;

typedef struct mh_learn_stats {
    double  loss_initial;   /* mean pair loss of the first epoch                      */
    double  loss_final;     /* mean pair loss of the last epoch                       */
    int32_t n_pairs, epochs;
    double  ms_pairs;       /* device time: reference solve and snapshots             */
    double  ms_train;       /* device time: forward, backward and Adam steps          */
    double  reserved[4];
} mh_learn_stats;

void mh_learn_opts_default(mh_learn_opts *o);
/* Trains the network on the assembled system (the current coefficients and boundary data):
 * solves it with FP64 PCG to solve_rtol for x*, reruns FP64 PCG from zero and takes
 * n_pairs snapshots x_s at geometrically spaced iterations, giving pairs
 * (r_s = b^ - S^ x_s, e_s = x* - x_s) scaled by 1/|r_s|, and runs epochs x n_pairs Adam
 * steps on the loss of mh_learned_grad (the energy-norm error of the V-cycle's answer), the
 * smoothing interval re-estimated at every step.  The solution left in the handle is x*. */
int mh_learned_train(mh_handle *h, const mh_learn_opts *opts, mh_learn_stats *stats);

/* ---- aggregation multigrid (MH_SOLVER_AMG) ------------------------------------------- */
/* No counterpart in the reference (PETSc ILU there).  The hierarchy of the last AMG solve:
 * number of levels, real rows and SELL slots per level (arrays of cap entries). */
int mh_amg_info(const mh_handle *h, int32_t *n_levels, int64_t *rows, int64_t *slots, int32_t cap);
/* The coarse tail of that hierarchy's V-cycle: the first level of the levels (below the fine
 * one, each of at most MH_AMG_TAIL rows; the environment variable, default 0: off) that run
 * as one thread-block cluster launch, and the cluster's CTAs; 0 and 0 when every level runs
 * its own kernels. */
int mh_amg_tail(const mh_handle *h, int32_t *level, int32_t *cluster_ctas);
/* One level of that hierarchy in CSR without zero entries (level 0 = the FP32 Jacobi-scaled
 * edge system in padded solver-row order), its aggregation agg [n] (coarse row of each row,
 * -1: none; not on the last level) and transfer weights [n]: level l+1 is P^T W A_l W P with
 * P_{i,agg[i]} = 1 and W = diag(weight).  Call with NULL arrays to get n and nnz first. */
int mh_amg_level(const mh_handle *h, int32_t level, int64_t *n, int64_t *nnz, int32_t *agg, float *weight,
                 int32_t *row_ptr, int32_t *col, float *val);

/* Per-edge weights w of the multigrid's fine-level smoother for MH_SOLVER_AMG: Chebyshev
 * smoothing on diag(w) S^ instead of the Jacobi-scaled S^ (MH_SOLVER_FCG_LEARNED sets them
 * from its network instead).  w [n_edges] in edge order, every weight > 0 and finite; NULL
 * restores plain smoothing.  Rows outside the hierarchy (no coupling) keep weight 1 (they are
 * solved exactly).  Takes effect at the next solve (the fine level's smoothing interval is
 * re-estimated for the weights). */
int mh_smoother_weights_set(mh_handle *h, const float *w, int64_t n);
/* The weights of the last multigrid solve (1 where it used none); w [n_edges]. */
int mh_smoother_weights_get(const mh_handle *h, float *w, int64_t n);

/* ---- a general symmetric positive definite system (the LinSys seam) ------------------- */
/* The solvers of mh_solve on a sparse SPD system the caller assembles itself, as Flow123d's
 * LinSys hands a system to PETSc's KSP (src/la/linsys.hh:63-222, solve_system in
 * src/la/solve.cc:175-209): for example the schur2 complement that SchurComplement::form_schur
 * builds (src/la/schur.cc:566-611), or any other SPD system of the reference.  C++ callers use
 * it through LinSys_CUDA (include/linsys_cuda.hh).
 * mh_csr_create: n rows, CSR pattern row_ptr [n+1], col [row_ptr[n]] with the columns of every
 * row sorted and unique and the diagonal present (MH_ERR_INVALID otherwise).  Without a device
 * the handle is created (the layout is host work) and compute calls return MH_ERR_CUDA.
 * mh_csr_set_values: val [row_ptr[n]] in CSR order and rhs [n]; every diagonal value must be
 * > 0.  Then mh_solve (any MH_SOLVER_* method, the same convergence test on the FP64 true
 * residual) and mh_csr_get_solution (x [n]).  The mesh-based calls (mh_set_coeffs, mh_set_bc,
 * mh_assemble, mh_unsteady_*) return MH_ERR_STATE on such a handle; mh_get_sizes reports n as
 * n_edges and the pattern's nonzeros as schur_nnz. */
int mh_csr_create(int64_t n, const int32_t *row_ptr, const int32_t *col, mh_handle **out);
int mh_csr_set_values(mh_handle *h, const double *val, const double *rhs);
int mh_csr_get_solution(const mh_handle *h, double *x, int64_t n);

/* ---- residual check without device allocation --------------------------------------- */
/* No counterpart in the reference: Flow123d leaves this check to PETSc's KSP monitor.
 * For callers that cannot call cudaMalloc at the point where they need to check a solution:
 * code that runs after a device allocation has already failed and must decide whether the
 * last iterate is usable, or a host framework that reserves the whole device for its own
 * memory pool (PyTorch's caching allocator, a PETSc/MPI pool) and forbids raw allocations.
 *
 * Computes r = b - S x for an n x n CSR matrix (row_ptr [n+1], col/val [nnz]) and writes
 *   out[0] = |D^-1/2 r| / |D^-1/2 b|   (D = diag S; the norm mh_solve judges convergence by)
 *   out[1] = |r| / |b|,  out[2] = |r|,  out[3] = |b|
 * and, if r is not NULL, the residual vector.  r must not overlap x or b (MH_ERR_INVALID).
 * Every pointer is a device pointer owned by the caller; work runs on cuda_stream (NULL: the
 * legacy default stream) and is complete when the call returns.  The scratch is a fixed
 * array inside the library (about 512 KiB, held on every GPU that loads the library until
 * the process exits), so n is limited to MH_NOALLOC_MAX_ROWS and larger n is rejected with
 * MH_ERR_INVALID.
 *
 * Set-up: CUDA loads a library's device code lazily, per context.  The first call in a
 * context loads this entry point's code and array (which allocates device memory) and looks
 * up the array's device address (cudaGetSymbolAddress).  Call it once with n == 0 (all other
 * pointers may be NULL) in each context you will use, at start-up while allocation still
 * succeeds and before any stream capture: that call does only the set-up.  After it, calls in
 * that context allocate nothing and call no allocating routine.  A new context (one created
 * after cudaDeviceReset, or a driver-API context made current) needs its own set-up call.
 *
 * Errors: an error already pending from the caller's earlier CUDA work makes the call return
 * MH_ERR_CUDA and is left pending; errors of this call's own work are cleared and returned as
 * MH_ERR_CUDA.  All calls share the array: calls that overlap on the GPU race and must be
 * serialised by the caller. */
#define MH_NOALLOC_MAX_ROWS (16384 * 256)
int mh_csr_residual_noalloc(int64_t n, const int32_t *row_ptr, const int32_t *col, const double *val,
                            const double *b, const double *x, double *r, double *out, void *cuda_stream);

#ifdef __cplusplus
}
#endif
#endif /* MH_DARCY_H */
