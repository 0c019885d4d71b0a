"""ctypes binding of libubolt_b200.so - the C ABI declared in include/ubolt_b200.h.

The library is built in-tree (python -m ubolt_b200.build). There is no
fallback: if the shared object is missing or does not load, importing this
module raises.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libubolt_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is missing - build it with `python -m ubolt_b200.build`")
lib = C.CDLL(LIB_PATH)

OK = 0
ERRORS = {1: "ARG", 2: "CUDA", 3: "SINGULAR", 4: "STATE", 5: "NOT_CONVERGED", 6: "TIMEOUT", 7: "NOMEM",
          8: "BREAKDOWN", 9: "NONFINITE"}
TRI, QUAD, TET, HEX = 3, 4, 10, 12
BC_VACUUM, BC_REFLECT = 0, 1

vp = C.c_void_p
i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
dp = C.POINTER(C.c_double)


class UboltError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"UBOLT_ERR_{ERRORS.get(status, status)}: {message}")
        self.status = status


def check(status):
    if status != OK:
        raise UboltError(status, lib.ubolt_last_error().decode())
    return status


class DGGeometry(C.Structure):
    _fields_ = [("dim", C.c_int32), ("n_basis", C.c_int32), ("faces_per_cell", C.c_int32), ("pad_", C.c_int32),
                ("n_cells", C.c_int64),
                ("volume", dp), ("centroid", dp), ("face_nA", dp), ("face_neighbour", i64p),
                ("face_bc", i32p), ("face_side", i32p), ("face_axis", i32p), ("face_centroid", dp),
                ("face_distance", dp), ("face_own", dp), ("face_up", dp), ("basis_grad", dp),
                ("face_neighbour_grad", dp), ("face_basis_value", dp)]


class CGGeometry(C.Structure):
    _fields_ = [("dim", C.c_int32), ("n_element_vertices", C.c_int32), ("faces_per_element", C.c_int32),
                ("pad_", C.c_int32), ("n_vertices", C.c_int64), ("n_elements", C.c_int64), ("n_star", C.c_int64),
                ("n_bfaces", C.c_int64),
                ("elem_vertex", i64p), ("mass", dp), ("grad", dp), ("stiff", dp), ("centre_grad", dp),
                ("volume", dp), ("centroid", dp), ("lumped_mass", dp), ("vertex_coord", dp),
                ("star_offset", i64p), ("star_elem", i64p), ("star_li", i32p),
                ("bface_offset", i64p), ("bface_nA", dp), ("bface_mass", dp), ("bface_side", i32p),
                ("bface_bc", i32p), ("elem_face_neighbour", i64p), ("elem_face_area", dp), ("elem_face_bc", i32p)]


class Quadrature(C.Structure):
    _fields_ = [("dim", C.c_int32), ("n_angles", C.c_int32), ("sum_weights", C.c_double),
                ("omega", dp), ("w", dp), ("reflect", i32p)]


def _sig(name, restype, *argtypes):
    f = getattr(lib, name)
    f.restype = restype
    f.argtypes = list(argtypes)
    return f


_sig("ubolt_last_error", C.c_char_p)
_sig("ubolt_version", C.c_char_p)
_sig("ubolt_lqn_octant", C.c_int, C.c_int, dp, i32p, dp, i32p, i32p)
_sig("ubolt_quadrature_lqn", C.c_int, C.c_int, C.c_int, dp, dp, i32p, i32p, dp)
_sig("ubolt_geometry_build", C.c_int, C.c_int, C.c_int, C.c_int64, dp, C.c_int64, i64p, C.c_int, i32p,
     C.POINTER(vp))
_sig("ubolt_geometry_view", C.c_int, vp, C.POINTER(DGGeometry))
_sig("ubolt_geometry_free", None, vp)
_sig("ubolt_ctx_create", C.c_int, C.POINTER(DGGeometry), C.POINTER(Quadrature), C.POINTER(vp))
_sig("ubolt_cg_geometry_build", C.c_int, C.c_int, C.c_int, C.c_int64, dp, C.c_int64, i64p, i32p, C.POINTER(vp))
_sig("ubolt_cg_geometry_view", C.c_int, vp, C.POINTER(CGGeometry))
_sig("ubolt_cg_geometry_free", None, vp)
_sig("ubolt_ctx_create_cg", C.c_int, C.POINTER(CGGeometry), C.POINTER(Quadrature), C.c_double, C.POINTER(vp))
_sig("ubolt_ctx_is_cg", C.c_int, vp)
_sig("ubolt_ctx_destroy", C.c_int, vp)
_sig("ubolt_ctx_sizes", C.c_int, vp, i64p, i64p, i64p, i32p, i32p)
_sig("ubolt_set_group", C.c_int, vp, vp, vp, vp)
for _n in ("ubolt_apply", "ubolt_apply_f32", "ubolt_apply_unscattered", "ubolt_apply_unscattered_f32",
           "ubolt_apply_adjoint", "ubolt_apply_adjoint_f32", "ubolt_block_apply", "ubolt_block_apply_f32",
           "ubolt_block_apply_transpose", "ubolt_scalar_flux", "ubolt_scalar_flux_f32", "ubolt_add_source"):
    _sig(_n, C.c_int, vp, vp, vp, vp)
_sig("ubolt_diagonal", C.c_int, vp, vp, vp)
_sig("ubolt_block_setup", C.c_int, vp, i64p, vp)
_sig("ubolt_block_inverse", C.c_int, vp, vp, vp)
_sig("ubolt_current", C.c_int, vp, vp, vp, vp)
_sig("ubolt_expand_p1", C.c_int, vp, vp, vp, vp, vp)
_sig("ubolt_add_transfer", C.c_int, vp, vp, vp, vp, vp)
_sig("ubolt_add_ghost_inflow", C.c_int, vp, dp, vp, vp)


def declared_symbols(header=None):
    """Every function name include/ubolt_b200.h declares."""
    import re
    header = header or os.path.join(os.path.dirname(_HERE), "include", "ubolt_b200.h")
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ubolt_[a-z0-9_]+)\s*\(", text)))


class SweepInfo(C.Structure):
    _fields_ = [("patch_size", C.c_int32), ("n_patches", C.c_int32), ("n_tasks", C.c_int64),
                ("n_lagged", C.c_int64), ("n_split", C.c_int64), ("max_levels", C.c_int32), ("grid", C.c_int32),
                ("total_levels", C.c_int64), ("timeouts", C.c_uint32), ("kernel", C.c_int32),
                ("factor_bytes", C.c_int64), ("factor_bytes_fp64", C.c_int64)]


class SolveOptions(C.Structure):
    _fields_ = [("rtol", C.c_double), ("inner_rtol", C.c_double), ("max_it", C.c_int32), ("restart", C.c_int32),
                ("precision", C.c_int32), ("pc", C.c_int32), ("max_outer", C.c_int32), ("x_zero", C.c_int32),
                ("krylov", C.c_int32), ("pad_", C.c_int32)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("outer", C.c_int32), ("converged", C.c_int32), ("krylov", C.c_int32),
                ("residual", C.c_double), ("rnorm0", C.c_double), ("seconds", C.c_double)]


PC_NONE, PC_BLOCK, PC_SWEEP, PC_SWEEP_DSA, PC_BLOCK_DSA = 0, 1, 2, 3, 4
PRECISION_FP64, PRECISION_MIXED = 0, 1

_sig("ubolt_sweep_setup", C.c_int, vp, C.c_int)
_sig("ubolt_sweep", C.c_int, vp, vp, vp, vp)
_sig("ubolt_sweep_f32", C.c_int, vp, vp, vp, vp)
_sig("ubolt_sweep_iso", C.c_int, vp, vp, vp, vp, C.c_int, vp)
_sig("ubolt_sweep_iso_f32", C.c_int, vp, vp, vp, vp, C.c_int, vp)
_sig("ubolt_sweep_status", C.c_int, vp, C.POINTER(SweepInfo), vp)
_sig("ubolt_sweep_test_wait", C.c_int, vp, C.c_uint32, C.c_int)
_sig("ubolt_sweep_set_factor_limit", C.c_int, vp, C.c_int64)
_sig("ubolt_solve_defaults", None, C.POINTER(SolveOptions))
_sig("ubolt_solver_setup", C.c_int, vp, C.POINTER(SolveOptions))
_sig("ubolt_solve", C.c_int, vp, vp, vp, C.POINTER(SolveOptions), C.POINTER(SolveStats), vp)
_sig("ubolt_solve_host_batch", C.c_int, vp, C.c_int, C.POINTER(vp), C.POINTER(vp), C.POINTER(SolveOptions),
     C.POINTER(SolveStats), vp)


class SweepPlanView(C.Structure):
    _fields_ = [("patch_size", C.c_int32), ("n_patches", C.c_int32), ("n_tasks", C.c_int64),
                ("n_lagged", C.c_int64), ("n_split", C.c_int64), ("task_pa", i32p), ("dep_ptr", i32p),
                ("deps", i32p), ("cell_ptr", i64p), ("tcell", C.POINTER(C.c_uint8)),
                ("tmask", C.POINTER(C.c_uint16)), ("lvl_ptr", i32p), ("lvl", C.POINTER(C.c_uint16))]


_sig("ubolt_sweep_plan_build", C.c_int, C.POINTER(DGGeometry), C.POINTER(Quadrature), C.c_int, C.POINTER(vp),
     C.POINTER(SweepPlanView))
_sig("ubolt_sweep_plan_free", None, vp)


def sweep_plan(geometry, quad, patch_size=0):
    """The sweep plan built on the host, as NumPy arrays (for inspection and tests)."""
    import numpy as np
    h = vp()
    view = SweepPlanView()
    gs, qs = geometry.struct(), quad.struct()
    check(lib.ubolt_sweep_plan_build(C.byref(gs), C.byref(qs), patch_size, C.byref(h), C.byref(view)))
    try:
        nt = view.n_tasks
        arr = lambda p, n: np.ctypeslib.as_array(p, shape=(n,)).copy() if n > 0 else np.zeros(0)
        out = {"patch_size": view.patch_size, "n_patches": view.n_patches, "n_tasks": nt, "n_lagged": view.n_lagged,
               "n_split": view.n_split, "task_pa": arr(view.task_pa, nt), "dep_ptr": arr(view.dep_ptr, nt + 1),
               "cell_ptr": arr(view.cell_ptr, nt + 1), "lvl_ptr": arr(view.lvl_ptr, nt + 1)}
        out["deps"] = arr(view.deps, int(out["dep_ptr"][-1]))
        out["tcell"] = arr(view.tcell, int(out["cell_ptr"][-1]))
        out["tmask"] = arr(view.tmask, int(out["cell_ptr"][-1]))
        out["lvl"] = arr(view.lvl, int(out["lvl_ptr"][-1]))
        return out
    finally:
        lib.ubolt_sweep_plan_free(h)

SWEEP_AUTO, SWEEP_TASKS, SWEEP_WAVE = 0, 1, 2
_sig("ubolt_sweep_set_kernel", C.c_int, vp, C.c_int)


class WavePlanView(C.Structure):
    _fields_ = [("acyclic", C.c_int32), ("slots", C.c_int32), ("n_front", C.c_int32), ("max_width", C.c_int32),
                ("max_levels", C.c_int32), ("pad_", C.c_int32), ("total_levels", C.c_int64), ("lvl_base", i32p),
                ("lvl_pos", i32p), ("meta", i32p)]


_sig("ubolt_wave_plan_build", C.c_int, C.POINTER(DGGeometry), C.POINTER(Quadrature), C.POINTER(vp),
     C.POINTER(WavePlanView))
_sig("ubolt_wave_plan_free", None, vp)


class WaveLayoutView(C.Structure):
    _fields_ = [("front_off", C.c_int32), ("ring_base", C.c_int32), ("cap", C.c_int32), ("smem", C.c_int32),
                ("store_bytes", C.c_int64), ("region", i64p), ("chunk_rel", i32p), ("ring_off", i32p)]


_sig("ubolt_wave_plan_layout", C.c_int, vp, C.c_int, C.c_int, C.c_int, C.POINTER(WaveLayoutView))

B200_MAX_SHARED_PER_BLOCK = 232448  # cudaDevAttrMaxSharedMemoryPerBlockOptin on sm_100


def wave_plan(geometry, quad, layouts=()):
    """The wave plan built on the host, as NumPy arrays (for inspection and
    tests); layouts: (n_basis, elem_bytes, max_shared_bytes) triples whose
    store and shared-memory layouts to add under "layout"."""
    import numpy as np
    h = vp()
    view = WavePlanView()
    gs, qs = geometry.struct(), quad.struct()
    check(lib.ubolt_wave_plan_build(C.byref(gs), C.byref(qs), C.byref(h), C.byref(view)))
    try:
        A = quad.n_angles
        out = {"acyclic": bool(view.acyclic), "slots": view.slots, "n_front": view.n_front,
               "max_width": view.max_width, "max_levels": view.max_levels, "total_levels": view.total_levels,
               "lvl_base": np.ctypeslib.as_array(view.lvl_base, shape=(A + 1,)).copy()}
        if view.acyclic:
            out["lvl_pos"] = np.ctypeslib.as_array(view.lvl_pos, shape=(view.total_levels + A,)).copy()
            out["meta"] = np.ctypeslib.as_array(view.meta, shape=(A * geometry.n_cells * 4,)).copy().reshape(
                A, geometry.n_cells, 4)
        out["layout"] = {}
        for key in layouts:
            lv = WaveLayoutView()
            check(lib.ubolt_wave_plan_layout(h, *key, C.byref(lv)))
            n = view.total_levels + A
            out["layout"][tuple(key)] = {
                "front_off": lv.front_off, "ring_base": lv.ring_base, "cap": lv.cap, "smem": lv.smem,
                "store_bytes": lv.store_bytes, "region": np.ctypeslib.as_array(lv.region, shape=(A,)).copy(),
                "chunk_rel": np.ctypeslib.as_array(lv.chunk_rel, shape=(n,)).copy(),
                "ring_off": np.ctypeslib.as_array(lv.ring_off, shape=(n,)).copy()}
        return out
    finally:
        lib.ubolt_wave_plan_free(h)


_sig("ubolt_launch_count", C.c_uint64)
_sig("ubolt_solve_adjoint", C.c_int, vp, vp, vp, C.POINTER(SolveOptions), C.POINTER(SolveStats), vp)
_sig("ubolt_add_response_source", C.c_int, vp, vp, vp, vp)
_sig("ubolt_gradient", C.c_int, vp, vp, vp, vp, vp, vp)


class DsaOptions(C.Structure):
    _fields_ = [("penalty", C.c_double), ("consistent_power", C.c_double), ("consistent_d", C.c_int32),
                ("inner_iterations", C.c_int32), ("void_sigma_t", C.c_double), ("void_d", C.c_double),
                ("void_bridge", C.c_int32), ("pad_", C.c_int32)]


_sig("ubolt_dsa_defaults", None, C.POINTER(DsaOptions))
_sig("ubolt_dsa_setup", C.c_int, vp, C.c_void_p, C.POINTER(DsaOptions))
_sig("ubolt_dsa_set_group", C.c_int, vp, vp)
_sig("ubolt_dsa_void_info", C.c_int, vp, i64p, C.POINTER(C.c_int32), dp)
_sig("ubolt_dsa_apply", C.c_int, vp, vp, vp, vp)
_sig("ubolt_dsa_apply_static", C.c_int, vp, vp, vp, vp)
_sig("ubolt_dsa_spmv", C.c_int, vp, vp, vp, vp)
_sig("ubolt_dsa_restrict", C.c_int, vp, vp, vp, vp)
_sig("ubolt_dsa_prolong", C.c_int, vp, vp, vp, vp)
_sig("ubolt_dsa_matrix", C.c_int, vp, dp)
