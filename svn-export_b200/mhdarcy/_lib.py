"""ctypes binding of libmhdarcy.so (the C ABI declared in include/mh_darcy.h).

The shared library is built in-tree by ``make -C svn-export_b200/csrc`` and loaded from this
directory.  There is no Python or CPU fallback for any compute entry point: if the library
is missing the import fails, and compute calls on a machine without a CUDA device return
MH_ERR_CUDA, which is raised as :class:`MHError`.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmhdarcy.so")

MH_OK = 0
MH_NOT_CONVERGED = 1
MH_FELL_BACK = 2
MH_ERR_INVALID = -1
MH_ERR_SINGULAR = -2
MH_ERR_CUDA = -3
MH_ERR_STATE = -4
MH_ERR_NOMEM = -5
MH_ERR_NONFINITE = -6
MH_ERR_TOPOLOGY = -7
MH_ERR_BREAKDOWN = -8
MH_ERR_IO = -9

MH_BC_NONE, MH_BC_DIRICHLET, MH_BC_NEUMANN, MH_BC_ROBIN = 0, 1, 2, 3

MH_SOLVER_PCG64 = 0
MH_SOLVER_IR32 = 1
MH_SOLVER_CHEB = 2
MH_SOLVER_FCG_LEARNED = 3
MH_SOLVER_AMG = 4

_i32p = C.POINTER(C.c_int32)
_f64p = C.POINTER(C.c_double)
_f32p = C.POINTER(C.c_float)
_i64p = C.POINTER(C.c_int64)


class MeshDesc(C.Structure):
    _fields_ = [("n_nodes", C.c_int64), ("node_xyz", _f64p), ("n_elements", C.c_int64),
                ("el_dim", _i32p), ("el_nodes", _i32p), ("n_bc_elements", C.c_int64),
                ("bc_dim", _i32p), ("bc_nodes", _i32p)]


class MortarDesc(C.Structure):
    _fields_ = [("method", C.c_int32), ("sigma", C.c_double), ("n", C.c_int64), ("master", _i32p), ("slave", _i32p),
                ("master_t", _f64p), ("slave_xy", _f64p)]


class GmshInfo(C.Structure):
    _fields_ = [("node_id", _i64p), ("el_id", _i64p), ("el_region", _i32p), ("el_partition", _i32p),
                ("bc_id", _i64p), ("bc_region", _i32p), ("n_regions", C.c_int32), ("region_id", _i32p),
                ("region_dim", _i32p), ("region_boundary", _i32p), ("region_name", C.POINTER(C.c_char_p))]


class Sizes(C.Structure):
    _fields_ = [("n_nodes", C.c_int64), ("n_elements", C.c_int64), ("n_sides", C.c_int64),
                ("n_edges", C.c_int64), ("n_boundaries", C.c_int64), ("n_neighbours", C.c_int64),
                ("n_el_dim", C.c_int64 * 4), ("mh_size", C.c_int64), ("schur_nnz", C.c_int64),
                ("sell_slots", C.c_int64), ("n_rows_padded", C.c_int64), ("n_instances", C.c_int64)]


class Coeffs(C.Structure):
    _fields_ = [("conductivity", _f64p), ("anisotropy", _f64p), ("cross_section", _f64p),
                ("sigma", _f64p), ("water_source_density", _f64p), ("storativity", _f64p)]


class BC(C.Structure):
    _fields_ = [("type", _i32p), ("pressure", _f64p), ("flux", _f64p), ("robin_sigma", _f64p)]


class SolveOpts(C.Structure):
    _fields_ = [("method", C.c_int32), ("max_it", C.c_int32), ("r_tol", C.c_double),
                ("a_tol", C.c_double), ("use_initial_guess", C.c_int32), ("cheb_degree", C.c_int32),
                ("inner_rtol", C.c_double), ("inner_max_it", C.c_int32),
                ("iters_per_graph", C.c_int32), ("profile_kernels", C.c_int32), ("host_loop", C.c_int32),
                ("reserved", C.c_int32 * 5)]


class SolveStats(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32), ("outer_iterations", C.c_int32),
                ("fell_back", C.c_int32), ("rel_residual", C.c_double), ("ms_assembly", C.c_double),
                ("ms_solve", C.c_double), ("ms_backsub", C.c_double),
                ("rel_residual_unscaled", C.c_double), ("kernel_launches", C.c_int64),
                ("kernel_ms", C.c_double * 6), ("kernel_count", C.c_int32 * 6), ("ms_setup", C.c_double),
                ("reserved", C.c_double * 3)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}
        d["kernel_ms"] = list(self.kernel_ms)
        d["kernel_count"] = list(self.kernel_count)
        return d


class TuneResult(C.Structure):
    _fields_ = [("rows_per_thread", C.c_int32), ("sell_rows_per_warp", C.c_int32), ("k1_group", C.c_int32),
                ("amg_fine_passes", C.c_int32), ("us_per_iter_fp32", C.c_double), ("us_per_iter_fp64", C.c_double),
                ("us_assembly", C.c_double), ("ms_amg_solve", C.c_double), ("reserved", C.c_double * 2)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("reserved")}


class LearnOpts(C.Structure):
    _fields_ = [("n_pairs", C.c_int32), ("epochs", C.c_int32), ("lr", C.c_float), ("train_bias", C.c_int32),
                ("solve_rtol", C.c_double), ("seed", C.c_uint64), ("reserved", C.c_int32 * 6)]


class LearnStats(C.Structure):
    _fields_ = [("loss_initial", C.c_double), ("loss_final", C.c_double), ("n_pairs", C.c_int32),
                ("epochs", C.c_int32), ("ms_pairs", C.c_double), ("ms_train", C.c_double),
                ("reserved", C.c_double * 4)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class MHError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        super().__init__(f"{lib.mh_status_string(status).decode()} ({status}): {msg}")


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C svn-export_b200/csrc` "
                          "(there is no fallback implementation)")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    sig = {
        "mh_version": (C.c_char_p, []),
        "mh_status_string": (C.c_char_p, [C.c_int]),
        "mh_device_available": (C.c_int, []),
        "mh_last_error": (C.c_char_p, [vp]),
        "mh_cube_mesh_create": (C.c_int, [C.c_int32, C.c_int32, _i32p, _i32p, C.c_int32, _i32p, _i32p,
                                          _i32p, C.POINTER(vp)]),
        "mh_mesh_describe": (C.c_int, [vp, C.POINTER(MeshDesc)]),
        "mh_mesh_destroy": (None, [vp]),
        "mh_gmsh_read": (C.c_int, [C.c_char_p, C.POINTER(vp), C.c_char_p, C.c_size_t]),
        "mh_gmsh_info_get": (C.c_int, [vp, C.POINTER(GmshInfo)]),
        "mh_gmsh_element_data": (C.c_int, [C.c_char_p, C.c_char_p, C.c_double, C.c_int64, vp, C.c_int32, vp,
                                           C.c_char_p, C.c_size_t]),
        "mh_create": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(vp)]),
        "mh_destroy": (None, [vp]),
        "mh_set_stream": (C.c_int, [vp, vp]),
        "mh_kernel_launches": (C.c_int64, [vp]),
        "mh_get_sizes": (C.c_int, [vp, C.POINTER(Sizes)]),
        "mh_get_topology": (C.c_int, [vp] + [_i32p] * 8),
        "mh_set_coeffs": (C.c_int, [vp, C.POINTER(Coeffs)]),
        "mh_set_bc": (C.c_int, [vp, C.POINTER(BC)]),
        "mh_assemble": (C.c_int, [vp]),
        "mh_solve": (C.c_int, [vp, C.POINTER(SolveOpts), C.POINTER(SolveStats)]),
        "mh_get_solution": (C.c_int, [vp, _f64p, C.c_int64]),
        "mh_get_solution_device": (C.c_int, [vp, vp, C.c_int64]),
        "mh_get_element_flux": (C.c_int, [vp, vp, C.c_int64]),
        "mh_get_element_flux_device": (C.c_int, [vp, vp, C.c_int64]),
        "mh_raw_output_write": (C.c_int, [C.c_char_p, C.c_int, C.c_double, C.c_int64, vp, vp, vp, vp, vp]),
        "mh_get_node_pressure": (C.c_int, [vp, vp, C.c_int64]),
        "mh_water_balance": (C.c_int, [vp, vp, C.c_int32, vp, C.c_int32, vp, vp]),
        "mh_transport_matrix": (C.c_int, [vp, vp, vp, vp, vp, vp, vp]),
        "mh_transport_matrix_device": (C.c_int, [vp, vp, vp, C.c_int64, vp]),
        "mh_get_schur_system": (C.c_int, [vp, _i32p, _i32p, _f64p, _f64p]),
        "mh_solve_opts_default": (None, [C.POINTER(SolveOpts)]),
        "mh_unsteady_init": (C.c_int, [vp, C.c_int32, C.c_double, _f64p]),
        "mh_unsteady_step": (C.c_int, [vp, C.c_double, C.POINTER(SolveOpts), C.POINTER(SolveStats)]),
        "mh_csr_residual_noalloc": (C.c_int, [C.c_int64, vp, vp, vp, vp, vp, vp, vp, vp]),
        "mh_create_batch": (C.c_int, [C.POINTER(MeshDesc), C.c_int32, C.POINTER(vp)]),
        "mh_get_instance_offsets": (C.c_int, [vp] + [C.POINTER(C.c_int64)] * 4),
        "mh_get_instance_stats": (C.c_int, [vp, _i32p, _f64p, _i32p]),
        "mh_autotune": (C.c_int, [vp, C.c_int32, _i32p, _f64p]),
        "mh_autotune_ex": (C.c_int, [vp, C.c_int32, C.POINTER(TuneResult)]),
        "mh_learned_set_weights": (C.c_int, [vp, _f32p, C.c_int64]),
        "mh_learned_get_weights": (C.c_int, [vp, _f32p, C.c_int64]),
        "mh_learned_grad": (C.c_int, [vp, _f64p, _f64p, _f32p, _f64p]),
        "mh_learned_apply": (C.c_int, [vp, _f64p, _f64p]),
        "mh_amg_info": (C.c_int, [vp, _i32p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.c_int32]),
        "mh_amg_tail": (C.c_int, [vp, _i32p, _i32p]),
        "mh_amg_level": (C.c_int, [vp, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64), _i32p, _f32p, _i32p,
                                   _i32p, _f32p]),
        "mh_learn_opts_default": (None, [C.POINTER(LearnOpts)]),
        "mh_learned_train": (C.c_int, [vp, C.POINTER(LearnOpts), C.POINTER(LearnStats)]),
        "mh_smoother_weights_set": (C.c_int, [vp, _f32p, C.c_int64]),
        "mh_learned_grad_weights": (C.c_int, [vp, _f64p, _f64p, C.c_int32, _f32p, _f32p, _f64p]),
        "mh_learned_smoother": (C.c_int, [vp, _f32p, C.c_int64]),
        "mh_learned_reset": (C.c_int, [vp]),
        "mh_smoother_weights_get": (C.c_int, [vp, _f32p, C.c_int64]),
        "mh_csr_create": (C.c_int, [C.c_int64, _i32p, _i32p, C.POINTER(vp)]),
        "mh_create_mortar": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(MortarDesc), C.POINTER(vp)]),
        "mh_csr_set_values": (C.c_int, [vp, _f64p, _f64p]),
        "mh_csr_get_solution": (C.c_int, [vp, _f64p, C.c_int64]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    return L


lib = _load()

# every symbol the header declares, for the load/export check
EXPORTED = ("mh_version", "mh_status_string", "mh_device_available", "mh_last_error",
            "mh_cube_mesh_create", "mh_mesh_describe", "mh_mesh_destroy", "mh_create", "mh_destroy",
            "mh_gmsh_read", "mh_gmsh_info_get", "mh_gmsh_element_data", "mh_set_stream", "mh_kernel_launches",
            "mh_get_sizes", "mh_get_topology", "mh_set_coeffs", "mh_set_bc", "mh_assemble",
            "mh_solve", "mh_get_solution", "mh_get_solution_device",
            "mh_get_element_flux", "mh_get_element_flux_device", "mh_raw_output_write",
            "mh_get_node_pressure", "mh_water_balance", "mh_transport_matrix", "mh_transport_matrix_device", "mh_get_schur_system",
            "mh_solve_opts_default", "mh_unsteady_init", "mh_unsteady_step", "mh_csr_residual_noalloc",
            "mh_create_batch", "mh_get_instance_offsets", "mh_get_instance_stats", "mh_autotune", "mh_autotune_ex",
            "mh_learned_set_weights", "mh_learned_get_weights", "mh_learned_grad", "mh_learned_apply", "mh_learn_opts_default",
            "mh_amg_info", "mh_amg_tail", "mh_amg_level",
            "mh_learned_train", "mh_smoother_weights_set", "mh_smoother_weights_get",
            "mh_learned_grad_weights", "mh_learned_smoother", "mh_learned_reset",
            "mh_csr_create", "mh_csr_set_values", "mh_csr_get_solution", "mh_create_mortar")

MH_NN_PARAMS = 6561

MH_NOALLOC_MAX_ROWS = 16384 * 256
MH_MORTAR_NONE, MH_MORTAR_P0, MH_MORTAR_P1 = 0, 1, 2


def ptr(a, ctype):
    """Pointer to a C-contiguous numpy array (None -> NULL)."""
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


def f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def i32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32)


def check(status, handle=None):
    if status < 0:
        msg = lib.mh_last_error(handle).decode() if handle else ""
        raise MHError(status, msg)
    return status


def device_available():
    return bool(lib.mh_device_available())
