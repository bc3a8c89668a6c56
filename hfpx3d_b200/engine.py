"""ctypes bindings of libhfpx_engine.so (include/hfpx_engine.h) and a Python
mirror of the reference's call surface for the assembly -> solve -> stress path.

The functions below keep the reference's names and argument meaning
(namespace hfp3d in src/Solvers/system_assembly.h:35-71,
src/Core/surface_mesh_utilities.h, and il::LU in
il/linear_algebra/dense/factorization/LU.h:46-61).  Every call goes through
the C-ABI; there is no CPU fallback: if the CUDA library is missing or no GPU
is present the calls raise EngineError.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, 'libhfpx_engine.so')

HFPX_OK, HFPX_ERR_ARG, HFPX_ERR_CUDA, HFPX_ERR_SINGULAR, HFPX_ERR_NOMEM, HFPX_ERR_STATE, \
    HFPX_ERR_NOT_CONVERGED = range(7)
HFPX_LU_FP64, HFPX_LU_MIXED = 0, 1
_STATUS_NAMES = {0: 'HFPX_OK', 1: 'HFPX_ERR_ARG', 2: 'HFPX_ERR_CUDA', 3: 'HFPX_ERR_SINGULAR',
                 4: 'HFPX_ERR_NOMEM', 5: 'HFPX_ERR_STATE', 6: 'HFPX_ERR_NOT_CONVERGED'}


class EngineError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f'{_STATUS_NAMES.get(code, code)}: {msg}')
        self.code = code


class SolveInfo(ctypes.Structure):
    _fields_ = [('iterations', ctypes.c_int), ('residual', ctypes.c_double), ('converged', ctypes.c_int)]


class CfMaterial(ctypes.Structure):
    """F_C_Param_T (src/Core/model_parameters.h:22-31) with the contact model
    ids of Properties_T::c_model_id (cohesion: 0 box, 1 linear weakening;
    friction: 0 constant, 1 linear slip weakening)."""
    _fields_ = [('cr_open', ctypes.c_double), ('peak_ts', ctypes.c_double), ('cr_slip', ctypes.c_double),
                ('peak_sc', ctypes.c_double), ('peak_sf', ctypes.c_double), ('res_sf', ctypes.c_double),
                ('cohesion_model', ctypes.c_int), ('friction_model', ctypes.c_int)]


class _CfStateC(ctypes.Structure):
    _fields_ = [('dd', ctypes.POINTER(ctypes.c_double)), ('pp', ctypes.POINTER(ctypes.c_double)),
                ('mr_open', ctypes.POINTER(ctypes.c_double)), ('mr_slip', ctypes.POINTER(ctypes.c_double)),
                ('friction_coef', ctypes.POINTER(ctypes.c_double)),
                ('slip_cohesion', ctypes.POINTER(ctypes.c_double)),
                ('open_cohesion', ctypes.POINTER(ctypes.c_double)),
                ('mat_id', ctypes.POINTER(ctypes.c_int32)), ('dof_h', ctypes.POINTER(ctypes.c_int64))]


class CfInfo(ctypes.Structure):
    _fields_ = [('residual', ctypes.c_double), ('volume', ctypes.c_double), ('pressure', ctypes.c_double),
                ('delta_p', ctypes.c_double), ('n_dof', ctypes.c_int64), ('n_fixed', ctypes.c_int64),
                ('solver', ctypes.c_int), ('refinement', ctypes.c_int)]


_D = ctypes.POINTER(ctypes.c_double)
_L = ctypes.POINTER(ctypes.c_int64)
_V = ctypes.c_void_p
_i64 = ctypes.c_int64
_f64 = ctypes.c_double
_int = ctypes.c_int

# name -> (restype, argtypes): the whole exported surface of include/hfpx_engine.h
SIGNATURES = {
    'hfpx_ctx_create': (_int, [_int, ctypes.POINTER(_V)]),
    'hfpx_ctx_destroy': (_int, [_V]),
    'hfpx_ctx_last_error': (ctypes.c_char_p, [_V]),
    'hfpx_ctx_stream': (_int, [_V, ctypes.POINTER(_V)]),
    'hfpx_ctx_synchronize': (_int, [_V]),
    'hfpx_dof_handle': (_i64, [_D, _i64, _i64, _L, _i64, _i64, _int, _L]),
    'hfpx_mesh_create': (_int, [_V, _D, _i64, _i64, _L, _i64, _i64, _f64, ctypes.POINTER(_V)]),
    'hfpx_mesh_destroy': (_int, [_V]),
    'hfpx_assemble': (_int, [_V, _V, _L, _i64, _f64, _f64, _int, _int, ctypes.POINTER(_V)]),
    'hfpx_assemble_into': (_int, [_V, _V, _L, _i64, _f64, _f64, _int, _int, _V]),
    'hfpx_assemble_mixed': (_int, [_V, _V, _L, _i64, _f64, _f64, _int, ctypes.POINTER(_V)]),
    'hfpx_matrix_is_mixed': (_int, [_V]),
    'hfpx_assemble_grow': (_int, [_V, _V, _i64, _L, _i64, _f64, _f64, _int, _V, ctypes.POINTER(_V)]),
    'hfpx_batch_create': (_int, [_V, _i64, ctypes.POINTER(_V), _f64, _f64, _int, _int, ctypes.POINTER(_V)]),
    'hfpx_batch_set_loads': (_int, [_V, _V, _D, _i64]),
    'hfpx_batch_run': (_int, [_V, _V, _f64, _int, _V]),
    'hfpx_batch_solution': (_int, [_V, _V, _i64, _D]),
    'hfpx_batch_residuals': (_int, [_V, _V, _D]),
    'hfpx_batch_launches': (_i64, [_V]),
    'hfpx_batch_phases': (_int, [_V, _V, _D]),
    'hfpx_batch_destroy': (_int, [_V]),
    'hfpx_cf_match': (_int, [_V, _i64, ctypes.POINTER(CfMaterial), _int, ctypes.POINTER(_CfStateC)]),
    'hfpx_cf_update_mrd': (_int, [_V, _i64, ctypes.POINTER(CfMaterial), _int, ctypes.POINTER(_CfStateC)]),
    'hfpx_vc_cf_iteration': (_int, [_V, _V, _V, _L, _i64, ctypes.POINTER(CfMaterial), _int, _D, _i64, _f64, _int,
                                    _int, _f64, ctypes.POINTER(_CfStateC), ctypes.POINTER(CfInfo)]),
    'hfpx_matrix_upload': (_int, [_V, _D, _i64, _i64, ctypes.POINTER(_V)]),
    'hfpx_matrix_dims': (_int, [_V, _L, _L]),
    'hfpx_matrix_download': (_int, [_V, _V, _D, _i64]),
    'hfpx_matrix_download_block': (_int, [_V, _V, _i64, _i64, _i64, _i64, _D, _i64]),
    'hfpx_matrix_destroy': (_int, [_V]),
    'hfpx_rhs_sinf': (_int, [_V, _V, _L, _i64, _D, _i64, _D, _i64]),
    'hfpx_lu_factor': (_int, [_V, _V, _int, _L]),
    'hfpx_lu_solve': (_int, [_V, _V, _D, _i64, _i64, _f64, _int, ctypes.POINTER(SolveInfo)]),
    'hfpx_lu_solve_device': (_int, [_V, _V, _V, _i64, _i64, _f64, _int, ctypes.POINTER(SolveInfo)]),
    'hfpx_matrix_truncate': (_int, [_V, _V, _L, _i64, _int, ctypes.POINTER(_V)]),
    'hfpx_lu_solve_fixed': (_int, [_V, _V, _L, _i64, _D, _f64, ctypes.POINTER(SolveInfo)]),
    'hfpx_gmres': (_int, [_V, _V, _D, _f64, _int, _int, ctypes.POINTER(SolveInfo)]),
    'hfpx_gmres_device': (_int, [_V, _V, _V, _f64, _int, _int, ctypes.POINTER(SolveInfo)]),
    'hfpx_ctx_launch_count': (_i64, [_V]),
    'hfpx_residual_device': (_int, [_V, _V, _V, _V, _V]),
    'hfpx_gemm_f16_update': (_int, [_V, _i64, _i64, _i64, _V, _i64, _V, _i64, _V, _i64, _V]),
    'hfpx_precond_create': (_int, [_V, _V, _V, _int, _V, _f64, ctypes.POINTER(_V)]),
    'hfpx_precond_destroy': (_int, [_V]),
    'hfpx_precond_update': (_int, [_V, _V, _V, _V, _f64]),
    'hfpx_precond_coarse': (_int, [_V, _V, _L, ctypes.POINTER(ctypes.c_int32), _D, _D, _D]),
    'hfpx_precond_blocks': (_int, [_V, _V, _L, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32), _D]),
    'hfpx_gmres_precond': (_int, [_V, _V, _V, _D, _f64, _int, _int, ctypes.POINTER(SolveInfo)]),
    'hfpx_gmres_precond_device': (_int, [_V, _V, _V, _V, _f64, _int, _int, ctypes.POINTER(SolveInfo)]),
    'hfpx_gnn_create': (_int, [_V, ctypes.c_uint64, ctypes.POINTER(_V)]),
    'hfpx_gnn_destroy': (_int, [_V]),
    'hfpx_gnn_param_count': (_i64, [_V]),
    'hfpx_gnn_get_params': (_int, [_V, _V, ctypes.POINTER(ctypes.c_float)]),
    'hfpx_gnn_set_params': (_int, [_V, _V, ctypes.POINTER(ctypes.c_float)]),
    'hfpx_gnn_save': (_int, [_V, _V, ctypes.c_char_p]),
    'hfpx_gnn_load': (_int, [_V, ctypes.c_char_p, ctypes.POINTER(_V)]),
    'hfpx_gnn_graph_create': (_int, [_V, _V, _V, _f64, _int, ctypes.POINTER(_V)]),
    'hfpx_gnn_graph_destroy': (_int, [_V]),
    'hfpx_gnn_graph_dims': (_int, [_V, _L, _L]),
    'hfpx_gnn_graph_data': (_int, [_V, _V, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                                   ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                                   ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]),
    'hfpx_gnn_forward': (_int, [_V, _V, _V, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]),
    'hfpx_gnn_gradients': (_int, [_V, _V, _V, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_float)]),
    'hfpx_gnn_train': (_int, [_V, _V, _V, _int, _f64, ctypes.POINTER(ctypes.c_double)]),
    'hfpx_lu_panel_factor_noalloc': (_int, [_V, _V, _i64, _i64, _int, _V, _L]),
    'hfpx_stress': (_int, [_V, _V, _f64, _f64, _int, _D, _D, _i64, _D, _D]),
    'hfpx_stress_batch': (_int, [_V, _V, _f64, _f64, _int, _D, _i64, _D, _i64, _D, _D]),
    'hfpx_matrix_pivots': (_int, [_V, _V, ctypes.POINTER(ctypes.c_int32)]),
    'hfpx_matrix_upload_lu': (_int, [_V, _D, _i64, _i64, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(_V)]),
    'hfpx_local_submatrix': (_int, [_V, _f64, _f64, _f64, _f64, _f64, _D, _D, _D]),
    'hfpx_element_frame': (_int, [_D, _D, _D, _D]),
}

_lib = None


def lib():
    """Load the engine library (fails loudly when it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise EngineError(HFPX_ERR_STATE, f'{LIB_PATH} not built (python -m hfpx3d_b200.build)')
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(_D)


def _lp(a):
    return a.ctypes.data_as(_L)


def _f(a, dtype=np.float64):
    return np.asfortranarray(a, dtype=dtype)


class Context:
    """One GPU, one CUDA stream (hfpx_ctx)."""

    def __init__(self, device=0):
        self.h = _V()
        rc = lib().hfpx_ctx_create(device, ctypes.byref(self.h))
        if rc != HFPX_OK:
            raise EngineError(rc, f'cannot create a context on device {device}')
        self.device = device

    def check(self, rc):
        if rc != HFPX_OK:
            raise EngineError(rc, lib().hfpx_ctx_last_error(self.h).decode())

    @property
    def stream(self):
        s = _V()
        self.check(lib().hfpx_ctx_stream(self.h, ctypes.byref(s)))
        return s.value

    def synchronize(self):
        self.check(lib().hfpx_ctx_synchronize(self.h))

    def close(self):
        if self.h:
            lib().hfpx_ctx_destroy(self.h)
            self.h = _V()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class MeshGeom:
    """Mesh_Geom_T (src/Core/surface_mesh_utilities.h:25-31): nods >=3 x Nn,
    conn >=3 x Ne (0-based), both column-major; rows 3,4 carry tip flags."""
    nods: np.ndarray
    conn: np.ndarray

    def __post_init__(self):
        self.nods = _f(self.nods)
        self.conn = _f(self.conn, np.int64)

    @property
    def n_el(self):
        return self.conn.shape[1]


@dataclass
class NumParam:
    """Num_Param_T (src/Core/model_parameters.h:75-95)."""
    beta: float = 0.125
    tip_type: int = 1
    is_dd_local: bool = False


def make_dof_h_crack(mesh: MeshGeom, tip_type: int):
    """surface_mesh_utilities.cpp:28-112 -> (dof_h n_el x 18 int64 F-order, n_dof)."""
    ne = mesh.n_el
    dof = np.zeros((ne, 18), dtype=np.int64, order='F')
    n = lib().hfpx_dof_handle(_dp(mesh.nods), mesh.nods.shape[0], mesh.nods.shape[1], _lp(mesh.conn),
                              mesh.conn.shape[0], ne, tip_type, _lp(dof))
    if n < 0:
        raise EngineError(-n, 'bad mesh for the DoF handle')
    return dof, int(n)


class DeviceMesh:
    """Mesh uploaded with its per-element precompute (hfpx_mesh)."""

    def __init__(self, ctx: Context, mesh: MeshGeom, beta=0.125):
        self.ctx, self.h = ctx, _V()
        ctx.check(lib().hfpx_mesh_create(ctx.h, _dp(mesh.nods), mesh.nods.shape[0], mesh.nods.shape[1],
                                         _lp(mesh.conn), mesh.conn.shape[0], mesh.n_el, beta,
                                         ctypes.byref(self.h)))
        self.n_el = mesh.n_el

    def close(self):
        if self.h:
            lib().hfpx_mesh_destroy(self.h)
            self.h = _V()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceMatrix:
    """Dense column-major matrix resident in HBM (hfpx_matrix)."""

    def __init__(self, ctx, handle):
        self.ctx, self.h = ctx, handle
        n, ld = _i64(), _i64()
        lib().hfpx_matrix_dims(self.h, ctypes.byref(n), ctypes.byref(ld))
        self.n, self.ld = n.value, ld.value
        self.mixed = bool(lib().hfpx_matrix_is_mixed(self.h))

    @classmethod
    def upload(cls, ctx, a):
        a = _f(a)
        h = _V()
        ctx.check(lib().hfpx_matrix_upload(ctx.h, _dp(a), a.shape[0], a.shape[0], ctypes.byref(h)))
        return cls(ctx, h)

    def download(self):
        out = np.empty((self.n, self.n), order='F')
        self.ctx.check(lib().hfpx_matrix_download(self.ctx.h, self.h, _dp(out), self.n))
        return out

    def block(self, i0, j0, rows, cols):
        """Rows [i0, i0 + rows) x columns [j0, j0 + cols) (column-major numpy)."""
        out = np.empty((rows, cols), order='F')
        self.ctx.check(lib().hfpx_matrix_download_block(self.ctx.h, self.h, i0, j0, rows, cols, _dp(out),
                                                        max(rows, 1)))
        return out

    def close(self):
        if self.h:
            lib().hfpx_matrix_destroy(self.h)
            self.h = _V()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def assemble(ctx, dmesh: DeviceMesh, dof_h, n_dof, G, nu, is_dd_local=False, vc=False) -> DeviceMatrix:
    h = _V()
    dof_h = _f(dof_h, np.int64)
    ctx.check(lib().hfpx_assemble(ctx.h, dmesh.h, _lp(dof_h), n_dof, G, nu, int(is_dd_local), int(vc),
                                  ctypes.byref(h)))
    return DeviceMatrix(ctx, h)


def assemble_mixed(ctx, dmesh: DeviceMesh, dof_h, n_dof, G, nu, is_dd_local=False) -> DeviceMatrix:
    """The operator of assemble() in mixed precision: FP32 entries, near-field
    blocks (self and vertex neighbours) kept to ~2^-48 by FP32 low parts."""
    h = _V()
    dof_h = _f(dof_h, np.int64)
    ctx.check(lib().hfpx_assemble_mixed(ctx.h, dmesh.h, _lp(dof_h), n_dof, G, nu, int(is_dd_local), ctypes.byref(h)))
    return DeviceMatrix(ctx, h)


def assemble_grow(ctx, dmesh: DeviceMesh, n_el_old, dof_h, n_dof, G, nu, old: DeviceMatrix,
                  is_dd_local=False) -> DeviceMatrix:
    """The operator of a mesh grown by appending elements to the one `old`
    was assembled for: the old block copied, only new rows and columns
    assembled (hfpx_assemble_grow)."""
    h = _V()
    dof_h = _f(dof_h, np.int64)
    ctx.check(lib().hfpx_assemble_grow(ctx.h, dmesh.h, n_el_old, _lp(dof_h), n_dof, G, nu, int(is_dd_local), old.h,
                                       ctypes.byref(h)))
    return DeviceMatrix(ctx, h)


def assemble_into(ctx, dmesh: DeviceMesh, dof_h, n_dof, G, nu, matrix: DeviceMatrix, is_dd_local=False, vc=False):
    """Re-assemble into an existing device matrix (storage reused)."""
    dof_h = _f(dof_h, np.int64)
    ctx.check(lib().hfpx_assemble_into(ctx.h, dmesh.h, _lp(dof_h), n_dof, G, nu, int(is_dd_local), int(vc),
                                       matrix.h))
    return matrix


def make_3dbem_matrix_s(ctx, shear_m, poiss_r, mesh: MeshGeom, n_par: NumParam, dof_h=None):
    """system_assembly.cpp:30-219 -> (host matrix, dof_h, n_dof)."""
    if dof_h is None:
        dof_h, n_dof = make_dof_h_crack(mesh, n_par.tip_type)
    else:
        n_dof = int(dof_h.max()) + 1
    dm = DeviceMesh(ctx, mesh, n_par.beta)
    m = assemble(ctx, dm, dof_h, n_dof, shear_m, poiss_r, n_par.is_dd_local, vc=False)
    return m.download(), dof_h, n_dof


def make_3dbem_matrix_vc(ctx, shear_m, poiss_r, mesh: MeshGeom, n_par: NumParam, dof_h=None):
    """system_assembly.cpp:458-557 (corner defined as 0) -> (host matrix, dof_h, n_dof)."""
    if dof_h is None:
        dof_h, n_dof = make_dof_h_crack(mesh, n_par.tip_type)
    else:
        n_dof = int(dof_h.max()) + 1
    dm = DeviceMesh(ctx, mesh, n_par.beta)
    m = assemble(ctx, dm, dof_h, n_dof, shear_m, poiss_r, n_par.is_dd_local, vc=True)
    return m.download(), dof_h, n_dof


def add_s_inf_to_3dbem_rhs(ctx, dmesh: DeviceMesh, dof_h, n_dof, s_inf, rhs=None):
    """system_assembly.cpp:222-274; s_inf is (6,) or 6 x n_rhs."""
    s = _f(np.asarray(s_inf, dtype=np.float64).reshape(6, -1))
    nr = s.shape[1]
    if rhs is None:
        rhs = np.zeros((n_dof, nr), order='F')
    rhs = _f(rhs.reshape(n_dof, nr) if rhs.ndim == 1 else rhs)
    dof_h = _f(dof_h, np.int64)
    ctx.check(lib().hfpx_rhs_sinf(ctx.h, dmesh.h, _lp(dof_h), n_dof, _dp(s), nr, _dp(rhs), rhs.shape[0]))
    return rhs[:, 0].copy() if nr == 1 else rhs


def truncate(ctx, matrix: DeviceMatrix, keep, keep_border=True) -> DeviceMatrix:
    """Device gather of the kept DD unknowns (and the VC border) of a
    matrix (hfpx_matrix_truncate)."""
    k = np.ascontiguousarray(keep, dtype=np.int64).reshape(-1)
    h = _V()
    ctx.check(lib().hfpx_matrix_truncate(ctx.h, matrix.h, _lp(k), k.size, int(keep_border), ctypes.byref(h)))
    return DeviceMatrix(ctx, h)


def vc_truncation_map(orig_dof_h, dof_h):
    """keep[t] = the original DoF of truncated DoF t, from the two DoF
    handles as mod_3dbem_system_vc reads them (system_assembly.cpp:596-606):
    entry (e, j) maps dof_h(e, j) >= 0 to orig_dof_h(e, j)."""
    o = np.asarray(orig_dof_h, dtype=np.int64).reshape(-1)
    t = np.asarray(dof_h, dtype=np.int64).reshape(-1)
    used = int(t.max()) + 1 if t.size and t.max() >= 0 else 0
    keep = np.full(used, -1, dtype=np.int64)
    sel = t >= 0
    if np.any(o[sel] < 0):
        raise ValueError('a truncated DoF without an original DoF')
    if np.unique(t[sel]).size != int(sel.sum()):
        raise ValueError('a truncated DoF at two element nodes')
    keep[t[sel]] = o[sel]
    if np.any(keep < 0):
        raise ValueError('the truncated numbering has gaps')
    return keep


def vc_rhs(orig_dof_h, dof_h, delta_t, delta_v, orig_ndof):
    """The right-hand side of mod_3dbem_system_vc (system_assembly.cpp:580-590,
    612-621): delta_t by the truncated numbering, delta_v last.  delta_t is
    indexed by the full element-node numbering (n_el * 18), the original DoF
    numbering or the truncated one, told apart by its length as there."""
    t = np.asarray(dof_h, dtype=np.int64).reshape(-1)
    o = np.asarray(orig_dof_h, dtype=np.int64).reshape(-1)
    used = vc_truncation_map(orig_dof_h, dof_h).size
    dt = np.asarray(delta_t, dtype=np.float64).reshape(-1)
    rhs = np.zeros(used + 1)
    rhs[used] = delta_v
    sel = t >= 0
    if dt.size == t.size:
        rhs[t[sel]] = dt[sel]
    elif dt.size == orig_ndof:
        rhs[t[sel]] = dt[o[sel]]
    elif dt.size == used:
        rhs[:used] = dt
    else:
        raise ValueError('delta_t must have the full, original or truncated DoF count')
    return rhs


def mod_3dbem_system_vc(ctx, matrix: DeviceMatrix, orig_dof_h, dof_h, delta_t, delta_v):
    """system_assembly.cpp:560-629: the truncated bordered system of the DoF
    dof_h keeps, gathered on the device from the bordered VC matrix ->
    (DeviceMatrix of used + 1 unknowns, host rhs)."""
    keep = vc_truncation_map(orig_dof_h, dof_h)
    rhs = vc_rhs(orig_dof_h, dof_h, delta_t, delta_v, matrix.n - 1)
    return truncate(ctx, matrix, keep, True), rhs


class LU:
    """il::LU<il::Array2D<double>> (LU.h:46-120) on the device: factor on
    construction (dgetrf), solve(y) (dgetrs).  mode HFPX_LU_MIXED factors an
    FP32 copy (FP16 tensor-core trailing updates with FP32 accumulation) and
    refines in FP64."""

    def __init__(self, ctx, matrix: DeviceMatrix, mode=HFPX_LU_FP64):
        self.ctx, self.matrix, self.mode = ctx, matrix, mode
        info = _i64()
        rc = lib().hfpx_lu_factor(ctx.h, matrix.h, mode, ctypes.byref(info))
        self.info = info.value
        ctx.check(rc)

    def solve(self, y, tol=0.0, max_iter=0):
        b = _f(np.array(y, dtype=np.float64, copy=True))
        one = b.ndim == 1
        if one:
            b = b.reshape(-1, 1, order='F')
        info = SolveInfo()
        rc = lib().hfpx_lu_solve(self.ctx.h, self.matrix.h, _dp(b), b.shape[1], b.shape[0], tol, max_iter,
                                 ctypes.byref(info))
        self.last_info = info
        self.ctx.check(rc)
        return b[:, 0].copy() if one else b

    def solve_fixed(self, y, fixed, tol=0.0):
        """x with x[fixed] = 0 solving the rows of A x = y outside `fixed`,
        from this factorisation (hfpx_lu_solve_fixed): the system that
        truncating `fixed` away makes, without a new factorisation."""
        b = np.array(y, dtype=np.float64, copy=True).reshape(-1)
        fx = np.ascontiguousarray(fixed, dtype=np.int64).reshape(-1)
        info = SolveInfo()
        rc = lib().hfpx_lu_solve_fixed(self.ctx.h, self.matrix.h, _lp(fx), fx.size, _dp(b), tol, ctypes.byref(info))
        self.last_info = info
        self.ctx.check(rc)
        return b

    def gmres(self, y, tol=0.0, restart=0, max_iter=0):
        """One right-hand side by flexible GMRES on the FP64 matrix,
        preconditioned by this (mixed) factorisation (hfpx_gmres)."""
        b = np.array(y, dtype=np.float64, copy=True).reshape(-1)
        info = SolveInfo()
        rc = lib().hfpx_gmres(self.ctx.h, self.matrix.h, _dp(b), tol, restart, max_iter, ctypes.byref(info))
        self.last_info = info
        self.ctx.check(rc)
        return b


def make_3dbem_stress_f_s(ctx, dmesh: DeviceMesh, shear_m, poiss_r, dd, pts, s_inf, is_dd_local=False):
    """system_assembly.cpp:279-455: dd (6 Ne) x 3, pts 3 x P -> P x 6."""
    dd = _f(dd)
    pts = _f(pts)
    s = np.ascontiguousarray(np.asarray(s_inf, dtype=np.float64).reshape(6))
    P = pts.shape[1]
    out = np.empty((P, 6), order='F')
    ctx.check(lib().hfpx_stress(ctx.h, dmesh.h, shear_m, poiss_r, int(is_dd_local), _dp(dd), _dp(pts), P,
                                _dp(s), _dp(out)))
    return out


def make_3dbem_stress_f_s_batch(ctx, dmesh: DeviceMesh, shear_m, poiss_r, dd_cases, pts, s_inf_cases,
                                is_dd_local=False):
    """make_3dbem_stress_f_s for many load cases: dd_cases (n_cases, 6 Ne, 3),
    s_inf_cases 6 x n_cases -> (n_cases, P, 6); one influence matrix and one
    FP64 GEMM on the device (hfpx_stress_batch)."""
    dd = np.asarray(dd_cases, dtype=np.float64)
    nc = dd.shape[0]
    # each case's (6 Ne) x 3 block column-major, blocks one after another
    flat = np.ascontiguousarray(np.stack([np.asfortranarray(dd[k]).reshape(-1, order='F') for k in range(nc)]))
    pts = _f(pts)
    s = _f(np.asarray(s_inf_cases, dtype=np.float64).reshape(6, nc))
    P = pts.shape[1]
    out = np.empty(nc * P * 6)
    ctx.check(lib().hfpx_stress_batch(ctx.h, dmesh.h, shear_m, poiss_r, int(is_dd_local), _dp(flat), nc, _dp(pts), P,
                                      _dp(s), _dp(out)))
    return np.stack([out[k * 6 * P:(k + 1) * 6 * P].reshape(P, 6, order='F') for k in range(nc)])


def make_local_3dbem_submatrix(ctx, shear_m, poiss_r, h, z, tau, sfm):
    """elasticity_kernel_integration.cpp:34-205 (kernel 1) -> 6 x 18."""
    tau = np.ascontiguousarray(np.column_stack([np.real(tau), np.imag(tau)]).reshape(-1))
    sfm = np.asarray(sfm)
    sfm = np.ascontiguousarray(np.stack([sfm.real, sfm.imag], axis=-1).reshape(-1))
    out = np.empty(108)
    ctx.check(lib().hfpx_local_submatrix(ctx.h, shear_m, poiss_r, h, complex(z).real, complex(z).imag,
                                         _dp(tau), _dp(sfm), _dp(out)))
    return out.reshape(6, 18)


def element_frame(vert):
    """make_el_sfm_uniform + make_el_tau_crd (element_utilities.cpp:89-238) on
    the host: vert is 3 x 3 (column j = vertex j) -> (r 3x3, tau (3,), sfm 6x6)."""
    v = np.ascontiguousarray(np.asarray(vert, dtype=np.float64).T)
    r, tau, sfm = np.empty(9), np.empty(6), np.empty(72)
    rc = lib().hfpx_element_frame(_dp(v), _dp(r), _dp(tau), _dp(sfm))
    if rc != HFPX_OK:
        raise EngineError(rc, 'element_frame')
    return r.reshape(3, 3), tau[0::2] + 1j * tau[1::2], (sfm[0::2] + 1j * sfm[1::2]).reshape(6, 6)


def write_dd_vector_to_md(sol, dof_h, n_el):
    """surface_mesh_utilities.cpp:256-328 -> nodal DD (6 n_el) x 3."""
    dd = np.zeros((6 * n_el, 3), order='F')
    d = np.asarray(dof_h)
    for j in range(18):
        rows = 6 * np.arange(n_el) + j // 3
        g = d[:, j]
        ok = g >= 0
        dd[rows[ok], j % 3] = sol[g[ok]]
    return dd


# ------------------------------------------------- near-field preconditioners
HFPX_PC_BLOCK_JACOBI, HFPX_PC_NEUMANN, HFPX_PC_LOCAL_INVERSE, HFPX_PC_LEARNED = 0, 1, 2, 3
HFPX_PC_COARSE = 16  # or'ed with a kind: the two-level form
# the trained network shipped with the engine (HFPX_PC_WEIGHTS overrides the path)
WEIGHTS_PATH = os.environ.get('HFPX_PC_WEIGHTS') or os.path.join(_HERE, 'data', 'pc_gnn.bin')


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


class Precond:
    """A near-field right preconditioner of the FP64 matrix (hfpx_precond)."""

    def __init__(self, ctx, dmesh: DeviceMesh, matrix: DeviceMatrix, kind, net=None, shear_m=1.0):
        self.ctx = ctx
        self.dmesh = dmesh  # updates read the mesh
        self.h = _V()
        ctx.check(lib().hfpx_precond_create(ctx.h, dmesh.h, matrix.h, kind, net.h if net is not None else None,
                                            shear_m, ctypes.byref(self.h)))

    def coarse(self, with_ap=False):
        """The coarse level (two-level kinds): (agg_of_el, weights[n_el, 6, 3],
        A P or None, inverse of P^T A P or None)."""
        na = _i64()
        self.ctx.check(lib().hfpx_precond_coarse(self.ctx.h, self.h, ctypes.byref(na), None, None, None, None))
        ne = self.dmesh.n_el
        n = 18 * ne
        nc = 9 * na.value
        agg = np.empty(ne, dtype=np.int32)
        w = np.empty(ne * 18)
        ap = np.empty((n, nc), order='F') if with_ap else None
        inv = np.empty((nc, nc), order='F') if with_ap else None
        self.ctx.check(lib().hfpx_precond_coarse(self.ctx.h, self.h, ctypes.byref(na), _ip(agg), _dp(w),
                                                 _dp(ap) if with_ap else None, _dp(inv) if with_ap else None))
        return agg, w.reshape(ne, 6, 3), ap, inv

    def update(self, matrix: DeviceMatrix, net=None, shear_m=1.0):
        """The blocks made again from a re-assembled matrix of the same mesh,
        in place (hfpx_precond_update)."""
        self.ctx.check(lib().hfpx_precond_update(self.ctx.h, self.h, matrix.h, net.h if net is not None else None,
                                                 shear_m))
        return self

    def blocks(self):
        """(block_row, block_col, blocks[nb, 18, 18]) with blocks[k][r, c] = M[18 row + r, 18 col + c]."""
        nb = _i64()
        self.ctx.check(lib().hfpx_precond_blocks(self.ctx.h, self.h, ctypes.byref(nb), None, None, None))
        r = np.empty(nb.value, dtype=np.int32)
        c = np.empty(nb.value, dtype=np.int32)
        b = np.empty(nb.value * 324)
        self.ctx.check(lib().hfpx_precond_blocks(self.ctx.h, self.h, ctypes.byref(nb), _ip(r), _ip(c), _dp(b)))
        return r, c, b.reshape(nb.value, 18, 18).transpose(0, 2, 1)

    def close(self):
        if self.h:
            lib().hfpx_precond_destroy(self.h)
            self.h = _V()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gmres(ctx, matrix: DeviceMatrix, b, precond: Precond = None, tol=1e-10, restart=50, max_iter=1000):
    """Flexible GMRES on the FP64 matrix with a near-field preconditioner
    (hfpx_gmres_precond); returns (x, SolveInfo)."""
    x = np.array(b, dtype=np.float64, copy=True).reshape(-1)
    info = SolveInfo()
    rc = lib().hfpx_gmres_precond(ctx.h, matrix.h, precond.h if precond is not None else None, _dp(x), tol, restart,
                                  max_iter, ctypes.byref(info))
    if rc not in (HFPX_OK, HFPX_ERR_NOT_CONVERGED):
        ctx.check(rc)
    return x, info


class Gnn:
    """The learned preconditioner's graph network (hfpx_gnn)."""

    def __init__(self, ctx, seed=0, path=None):
        self.ctx = ctx
        self.h = _V()
        if path is not None:
            ctx.check(lib().hfpx_gnn_load(ctx.h, os.fsencode(path), ctypes.byref(self.h)))
        else:
            ctx.check(lib().hfpx_gnn_create(ctx.h, seed, ctypes.byref(self.h)))

    @property
    def n_params(self):
        return int(lib().hfpx_gnn_param_count(self.h))

    def params(self):
        p = np.empty(self.n_params, dtype=np.float32)
        self.ctx.check(lib().hfpx_gnn_get_params(self.ctx.h, self.h, _fp(p)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        self.ctx.check(lib().hfpx_gnn_set_params(self.ctx.h, self.h, _fp(p)))

    def save(self, path):
        self.ctx.check(lib().hfpx_gnn_save(self.ctx.h, self.h, os.fsencode(path)))

    def gradients(self, graph):
        loss = ctypes.c_double()
        g = np.empty(self.n_params, dtype=np.float32)
        self.ctx.check(lib().hfpx_gnn_gradients(self.ctx.h, self.h, graph.h, ctypes.byref(loss), _fp(g)))
        return loss.value, g

    def forward(self, graph):
        on = np.empty((graph.n_nodes, 324), dtype=np.float32)
        oe = np.empty((graph.n_edges, 324), dtype=np.float32)
        self.ctx.check(lib().hfpx_gnn_forward(self.ctx.h, self.h, graph.h, _fp(on), _fp(oe)))
        return on, oe

    def train(self, graph, steps, lr):
        losses = np.empty(steps)
        self.ctx.check(lib().hfpx_gnn_train(self.ctx.h, self.h, graph.h, steps, lr,
                                            losses.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return losses

    def close(self):
        if self.h:
            lib().hfpx_gnn_destroy(self.h)
            self.h = _V()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GnnGraph:
    """The network's graph of a mesh and its assembled matrix (hfpx_gnn_graph)."""

    def __init__(self, ctx, dmesh: DeviceMesh, matrix: DeviceMatrix, shear_m=1.0, targets=True):
        self.ctx = ctx
        self.h = _V()
        ctx.check(lib().hfpx_gnn_graph_create(ctx.h, dmesh.h, matrix.h, shear_m, int(targets), ctypes.byref(self.h)))
        n, e = _i64(), _i64()
        lib().hfpx_gnn_graph_dims(self.h, ctypes.byref(n), ctypes.byref(e))
        self.n_nodes, self.n_edges = n.value, e.value
        self.targets = targets

    def data(self):
        """dict of xn, xe (inputs as the network reads them), src, dst and, with targets, tn, te."""
        n, E = self.n_nodes, self.n_edges
        d = dict(xn=np.empty((n, 336), dtype=np.float32), xe=np.empty((E, 336), dtype=np.float32),
                 src=np.empty(E, dtype=np.int32), dst=np.empty(E, dtype=np.int32))
        tn = np.empty((n, 324), dtype=np.float32) if self.targets else None
        te = np.empty((E, 324), dtype=np.float32) if self.targets else None
        self.ctx.check(lib().hfpx_gnn_graph_data(self.ctx.h, self.h, _fp(d['xn']), _fp(d['xe']), _ip(d['src']),
                                                 _ip(d['dst']), _fp(tn) if tn is not None else None,
                                                 _fp(te) if te is not None else None))
        if tn is not None:
            d.update(tn=tn, te=te)
        return d

    def close(self):
        if self.h:
            lib().hfpx_gnn_graph_destroy(self.h)
            self.h = _V()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchInfo(ctypes.Structure):
    _fields_ = [('n_mesh', ctypes.c_int64), ('residual', ctypes.c_double), ('converged', ctypes.c_int),
                ('singular_mesh', ctypes.c_int64), ('off_plane_pairs', ctypes.c_int), ('iterations', ctypes.c_int)]


BATCH_TILES_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'data', 'batch_tiles.json')


def batch_tiles():
    """The autotuner's choice of (block size, leaf rows) for the batched
    factorisation (hfpx3d_b200/data/batch_tiles.json), or the defaults."""
    import json
    try:
        with open(BATCH_TILES_PATH) as f:
            best = json.load(f)['best']
        return int(best['nb']), int(best['leaf_rows'])
    except (OSError, KeyError, ValueError):
        return 128, 512


class Batch:
    """Many meshes (DeviceMesh, no fixed DoF) assembled, factored and solved
    in one CUDA-graph launch (hfpx_batch_*); load cases are in-situ stress
    tensors (6 x n_cases per mesh)."""

    def __init__(self, ctx, dmeshes, G, nu, nb=None, leaf_rows=None):
        self.ctx = ctx
        self.dmeshes = list(dmeshes)  # the batch reads them: keep them alive
        if nb is None or leaf_rows is None:
            t_nb, t_leaf = batch_tiles()
            nb = t_nb if nb is None else nb
            leaf_rows = t_leaf if leaf_rows is None else leaf_rows
        self.nb, self.leaf_rows = nb, leaf_rows
        arr = (_V * len(self.dmeshes))(*[d.h for d in self.dmeshes])
        self.h = _V()
        ctx.check(lib().hfpx_batch_create(ctx.h, len(self.dmeshes), arr, G, nu, nb, leaf_rows, ctypes.byref(self.h)))
        self.n = [18 * d.n_el for d in self.dmeshes]
        self.n_cases = 0

    def set_loads(self, s_inf):
        """s_inf: (n_mesh, 6, n_cases) in-situ stress tensors (Voigt)."""
        s = np.ascontiguousarray(np.asarray(s_inf, dtype=np.float64).transpose(0, 2, 1))  # mesh, case, component
        self.n_cases = s.shape[1]
        self.ctx.check(lib().hfpx_batch_set_loads(self.ctx.h, self.h, _dp(s), self.n_cases))

    def run(self, tol=1e-10, max_iter=10):
        info = BatchInfo()
        rc = lib().hfpx_batch_run(self.ctx.h, self.h, tol, max_iter, ctypes.byref(info))
        if rc not in (HFPX_OK, HFPX_ERR_NOT_CONVERGED):
            self.ctx.check(rc)
        return info

    def solution(self, m):
        cols = self.n_cases if self.n_cases else 6
        x = np.empty((self.n[m], cols), order='F')
        self.ctx.check(lib().hfpx_batch_solution(self.ctx.h, self.h, m, _dp(x)))
        return x

    def residuals(self):
        r = np.empty(len(self.n))
        self.ctx.check(lib().hfpx_batch_residuals(self.ctx.h, self.h, _dp(r)))
        return r

    @property
    def launches(self):
        return int(lib().hfpx_batch_launches(self.h))

    def phases(self):
        """Device ms of the last run: assembly (+ right-hand sides), factorisation, solves."""
        ms = np.empty(3)
        self.ctx.check(lib().hfpx_batch_phases(self.ctx.h, self.h, _dp(ms)))
        return {'assembly': ms[0], 'factor': ms[1], 'solve': ms[2]}

    def close(self):
        if self.h:
            lib().hfpx_batch_destroy(self.h)
            self.h = _V()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- the volume-control iteration with cohesion and friction
# (vc_cf_iteration, src/Development/c_f_iteration.cpp:27-436; match_f_c and
# update_mrd, src/Development/cohesion_friction.cpp:22-194)

class CfState:
    """The solution part of the reference's Mesh_Data_T
    (src/Core/surface_mesh_utilities.h:51-101) per collocation point
    (n_cp = 6 n_el, point 6 el + local node): dd (n_cp x 3), pp, the
    Frac_State_T arrays, the material ids, and the step's truncated DoF
    handle dof_h (dof_h_dd) with its DoF count n_dof."""

    def __init__(self, n_el, dd=None, pp=None, mr_open=None, mr_slip=None, mat_id=None):
        n_cp = 6 * int(n_el)
        self.n_el = int(n_el)
        self.dd = np.asfortranarray(np.zeros((n_cp, 3)) if dd is None else dd, dtype=np.float64).copy(order='F')
        self.pp = np.ascontiguousarray(np.zeros(n_cp) if pp is None else pp, dtype=np.float64).copy()
        self.mr_open = np.ascontiguousarray(np.zeros(n_cp) if mr_open is None else mr_open, dtype=np.float64).copy()
        self.mr_slip = np.ascontiguousarray(np.zeros(n_cp) if mr_slip is None else mr_slip, dtype=np.float64).copy()
        self.mat_id = np.ascontiguousarray(np.zeros(n_cp) if mat_id is None else mat_id, dtype=np.int32).copy()
        self.friction_coef = np.zeros(n_cp)
        self.slip_cohesion = np.zeros(n_cp)
        self.open_cohesion = np.zeros(n_cp)
        self.dof_h = np.full((self.n_el, 18), -1, dtype=np.int64, order='F')
        self.n_dof = 0
        for a in (self.pp, self.mr_open, self.mr_slip, self.mat_id):
            if a.shape != (n_cp,):
                raise ValueError('per-point arrays must hold 6 n_el entries')
        if self.dd.shape != (n_cp, 3):
            raise ValueError('dd must be (6 n_el) x 3')

    def _c(self):
        d = lambda a: a.ctypes.data_as(_D)
        return _CfStateC(d(self.dd), d(self.pp), d(self.mr_open), d(self.mr_slip), d(self.friction_coef),
                         d(self.slip_cohesion), d(self.open_cohesion),
                         self.mat_id.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), _lp(self.dof_h))

    def copy(self):
        s = CfState(self.n_el, self.dd, self.pp, self.mr_open, self.mr_slip, self.mat_id)
        for k in ('friction_coef', 'slip_cohesion', 'open_cohesion', 'dof_h'):
            setattr(s, k, getattr(self, k).copy(order='K'))
        s.n_dof = self.n_dof
        return s


def _materials(materials):
    mats = (CfMaterial * len(materials))()
    for i, m in enumerate(materials):
        if isinstance(m, CfMaterial):
            mats[i] = m
        else:
            mats[i] = CfMaterial(**m)
    return mats


def match_f_c(ctx, materials, state: CfState):
    """cohesion_friction.cpp:22-130: cohesion and friction of every point."""
    mats = _materials(materials)
    st = state._c()
    ctx.check(lib().hfpx_cf_match(ctx.h, 6 * state.n_el, mats, len(mats), ctypes.byref(st)))


def update_mrd(ctx, materials, state: CfState):
    """cohesion_friction.cpp:134-194: the maximum relative opening and slip."""
    mats = _materials(materials)
    st = state._c()
    ctx.check(lib().hfpx_cf_update_mrd(ctx.h, 6 * state.n_el, mats, len(mats), ctypes.byref(st)))


def vc_cf_iteration(ctx, dmesh: DeviceMesh, matrix: DeviceMatrix, orig_dof_h, n_dof, materials, state: CfState,
                    s_inf, inj_cp, new_vol, is_dd_local=False, all_components=False, release_sign=False,
                    reuse_factors=False, tol=1e-12) -> CfInfo:
    """One volume-control iteration with cohesion and friction
    (c_f_iteration.cpp:27-436) on the bordered matrix of orig_dof_h
    (unfactored, or factored with HFPX_LU_MIXED); updates `state` in place
    and returns the step's CfInfo (residual as the reference's return value).
    all_components adds the normal traction adjustment to the right-hand side
    too (the reference adds the first two components); release_sign adds the
    adjustments with the sign that removes the excess traction (the
    reference's sign doubles it).  The truncated system is solved with the
    full system's mixed factors (capacitance correction) when that is the
    cheaper way, or always when reuse_factors is set and there are factors;
    otherwise the truncated system is factored."""
    mats = _materials(materials)
    dof = _f(orig_dof_h, np.int64)
    si = np.ascontiguousarray(s_inf, dtype=np.float64)
    if si.shape != (6,):
        raise ValueError('s_inf must hold 6 Voigt components')
    st = state._c()
    info = CfInfo()
    ctx.check(lib().hfpx_vc_cf_iteration(ctx.h, dmesh.h, matrix.h, _lp(dof), int(n_dof), mats, len(mats), _dp(si),
                                         int(inj_cp), float(new_vol), int(is_dd_local),
                                         (1 if all_components else 0) | (2 if release_sign else 0)
                                         | (4 if reuse_factors else 0),
                                         float(tol), ctypes.byref(st), ctypes.byref(info)))
    state.n_dof = int(info.n_dof)
    return info
