"""cfd_b200: B200-native pressure-correction solver (host-side mirror of ``cfd::gpu``).

Python front end (ctypes) of ``libcfdb.so``, the C ABI declared in ``include/cfdb.h``. The
names, argument meaning and error behaviour mirror the reference's accelerator interface
(Yipexnn/CFD ``src/gpu/include/cfd/gpu/krylov.hpp``):

* :func:`solve` / :func:`solve_amg_cg` / :func:`assemble_convection_diffusion`
* :class:`DeviceSolver` (``DeviceSolver(const LduPattern&)``, ``set_amg``, ``solve``)
* :func:`backend_name` / :func:`device_available` / :func:`device_description`

Errors: invalid arguments raise :class:`InvalidArgument` (a ``ValueError``, the reference's
``std::invalid_argument``); device failures raise :class:`CudaError` (a ``RuntimeError``, the
reference's ``std::runtime_error("CUDA ...")``). Non-convergence is reported in
:class:`SolveStats`, never raised. There is no CPU fallback: without the built library the import
fails, and without a GPU every compute call raises :class:`NoDevice`.
"""
from __future__ import annotations

import ctypes as C
import enum
import functools
import os
import sys
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcfdb.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"cfd_b200: {LIB_PATH} is missing; build it with `python -m cfd_b200.build`")
_lib = C.CDLL(LIB_PATH)

_i, _d, _sz = C.c_int, C.c_double, C.c_size_t
_pi, _pd = C.POINTER(C.c_int), C.POINTER(C.c_double)
_vp = C.c_void_p


class CsrStruct(C.Structure):
    _fields_ = [("n", _i), ("nnz", _i), ("row_ptr", _pi), ("col", _pi), ("val", _pd)]


class AmgLevelStruct(C.Structure):
    _fields_ = [("a", CsrStruct), ("p", CsrStruct), ("r", CsrStruct)]


class AmgViewStruct(C.Structure):
    _fields_ = [("n_levels", _i), ("levels", C.POINTER(AmgLevelStruct)), ("coarse_inverse", _pd),
                ("smooth_sweeps", _i), ("jacobi_weight", _d)]


class ControlStruct(C.Structure):
    _fields_ = [("abs_tolerance", _d), ("max_iterations", _i)]


class StatsStruct(C.Structure):
    _fields_ = [("iterations", _i), ("residual", _d), ("converged", _i), ("on_device", _i),
                ("true_residual", _d)]


class PatternStruct(C.Structure):
    _fields_ = [("n", _i), ("n_faces", _i), ("nnz", _i), ("row_ptr", _pi), ("col", _pi),
                ("diag_pos", _pi), ("upper_pos", _pi), ("lower_pos", _pi)]


class KernelRecordStruct(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("level", _i), ("ms", _d), ("bytes", _d)]


class LduSettingsStruct(C.Structure):
    _fields_ = [("method", _i), ("tolerance", _d), ("rel_tolerance", _d), ("max_iterations", _i),
                ("max_age", _i)]


class LduResultStruct(C.Structure):
    _fields_ = [("initial_residual", _d), ("final_residual", _d), ("iterations", _i),
                ("amg_rebuilt", _i)]


class AmgSettingsStruct(C.Structure):
    _fields_ = [("strength_threshold", _d), ("max_levels", _i), ("coarse_size", _i),
                ("smooth_sweeps", _i), ("jacobi_weight", _d), ("device_table_limit", _i)]


def _proto(name, args, res=_i):
    f = getattr(_lib, name)
    f.argtypes = args
    f.restype = res
    return f


_P = C.POINTER
_proto("cfdb_backend_name", [C.c_char_p, _sz])
_proto("cfdb_device_available", [])
_proto("cfdb_device_description", [C.c_char_p, _sz])
_proto("cfdb_last_error", [C.c_char_p, _sz])
_proto("cfdb_default_amg_settings", [_P(AmgSettingsStruct)], None)
_proto("cfdb_assemble", [_i, _i, _pi, _pi, _pd, _pd, _pd, _d, _pd, _pd, _pd, _pd])
_proto("cfdb_assemble_device", [_i, _i, _vp, _vp, _vp, _vp, _vp, _d, _vp, _vp, _vp, _vp])
_proto("cfdb_solve", [_P(CsrStruct), _pd, _pd, _i, _P(ControlStruct), _P(StatsStruct)])
_proto("cfdb_solve_amg_cg", [_P(AmgViewStruct), _pd, _pd, _P(ControlStruct), _P(StatsStruct)])
_proto("cfdb_build_pattern", [_i, _i, _pi, _pi, _pi, _pi, _pi, _pi, _pi, _pi])
_proto("cfdb_solve_device_noalloc", [_P(CsrStruct), _vp, _vp, _i, _P(ControlStruct),
                                     _P(StatsStruct)])
_proto("cfdb_amg_setup", [_P(CsrStruct), _P(AmgSettingsStruct), _P(_vp)])
_proto("cfdb_amg_setup_device", [_P(CsrStruct), _P(AmgSettingsStruct), _P(_vp)])
_proto("cfdb_hierarchy_destroy", [_vp])
_proto("cfdb_hierarchy_levels", [_vp, _pi])
_proto("cfdb_hierarchy_level", [_vp, _i, _i, _pi, _pi, _P(CsrStruct)])
_proto("cfdb_hierarchy_aggregates", [_vp, _i, _P(_pi), _pi])
_proto("cfdb_hierarchy_coarse_inverse", [_vp, _P(_pd), _pi])
_proto("cfdb_hierarchy_view", [_vp, _i, _d, _P(AmgViewStruct)])
_proto("cfdb_hierarchy_operator_complexity", [_vp, _pd])
_proto("cfdb_system_create", [_P(PatternStruct), _P(_vp)])
_proto("cfdb_system_create_mesh", [_i, _i, _pi, _pi, _P(_vp)])
_proto("cfdb_system_destroy", [_vp])
_proto("cfdb_system_on_device", [_vp])
_proto("cfdb_system_set_amg", [_vp, _P(AmgViewStruct)])
_proto("cfdb_system_setup_amg", [_vp, _pd, _pd, _pd, _P(AmgSettingsStruct)])
_proto("cfdb_system_setup_amg_device", [_vp, _vp, _vp, _vp, _P(AmgSettingsStruct), _i])
_proto("cfdb_system_setup_profile", [_vp, C.c_char_p, C.c_size_t])
_proto("cfdb_system_set_keep_levels", [_vp, _i])
_proto("cfdb_release_cached_memory", [])
_proto("cfdb_system_time_sweep", [_vp, _i, _i, _pd, _pd])
_proto("cfdb_system_solve_ldu", [_vp, _vp, _vp, _vp, _vp, _vp, _P(LduSettingsStruct),
                                 _P(AmgSettingsStruct), _i, _P(LduResultStruct)])
_proto("cfdb_system_set_precision", [_vp, _i])
_proto("cfdb_system_solve", [_vp, _pd, _pd, _pd, _pd, _pd, _i, _i, _P(ControlStruct),
                             _P(StatsStruct)])
_proto("cfdb_system_solve_device", [_vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _P(ControlStruct),
                                    _P(StatsStruct)])
_proto("cfdb_system_assemble_device", [_vp, _vp, _vp, _vp, _d, _vp, _vp, _vp, _vp])
_proto("cfdb_system_apply_amg", [_vp, _pd, _pd])
_proto("cfdb_system_set_ordered", [_vp, _i])
_proto("cfdb_system_assemble", [_vp, _pd, _pd, _pd, _d, _pd, _pd, _pd, _pd])
_proto("cfdb_system_assemble_pressure_device", [_vp, _vp, _vp, _vp, _vp, _vp, _i, _d, _vp, _vp,
                                                _vp, _vp])
_proto("cfdb_system_kernel_launches", [_vp, _P(C.c_ulonglong)])
_proto("cfdb_system_correct_pressure_device", [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _d, _vp, _vp])
_proto("cfdb_fv_create", [_i, _i, _i, _pi, _pi, _pd, _pd, _pd, _pd, _pd, _pi, _pd, _P(_vp)])
_proto("cfdb_fv_destroy", [_vp])
_proto("cfdb_fv_pressure_gradient_device", [_vp, _vp, _vp])
_proto("cfdb_fv_correct_velocity_device", [_vp, _vp, _vp, _vp, _vp])
_proto("cfdb_fv_delta_device", [_vp, _P(_vp)])
_proto("cfdb_fv_hbya_rau_device", [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp])
_proto("cfdb_fv_face_flux_device", [_vp, _vp, _vp, _vp, _vp, _vp, _d, _vp, _vp])
_proto("cfdb_fv_pressure_boundary_device", [_vp, _vp, _vp, _i, _d, _vp, _vp])
_proto("cfdb_fv_non_orth_device", [_vp, _vp, _vp, _vp, _vp, _vp])
_proto("cfdb_fv_correct_flux_device", [_vp, _vp, _vp, _vp, _vp, _vp])
_proto("cfdb_fv_relax_device", [_vp, _vp, _vp, _d, _vp])


class TuningStruct(C.Structure):
    _fields_ = [("target_tiles", _i), ("wide_row", _i), ("lanes_div", _i), ("fuse_first", _i),
                ("sell_rows", _i), ("krylov_pair", _i), ("tail_rows", _i),
                ("col16", _i), ("pdl", _i), ("wait_polls", _i), ("mixed_sweeps", _i),
                ("mixed_weight", _d), ("tail_cluster", _i), ("vcycle_pair", _i),
                ("krylov_stage", _i)]


_proto("cfdb_default_tuning", [_P(TuningStruct)], None)
_proto("cfdb_system_set_tuning", [_vp, _P(TuningStruct)])
_proto("cfdb_batch_create", [_i, _pi, _pi, _pi, _pi, _P(_vp)])
_proto("cfdb_batch_destroy", [_vp])
_proto("cfdb_batch_sizes", [_vp, _P(C.c_longlong), _P(C.c_longlong)])
_proto("cfdb_batch_setup_amg", [_vp, _pd, _pd, _pd, _P(AmgSettingsStruct)])
_proto("cfdb_batch_setup_amg_device", [_vp, _vp, _vp, _vp, _P(AmgSettingsStruct), _i])
_proto("cfdb_batch_set_precision", [_vp, _i])
_proto("cfdb_batch_set_tuning", [_vp, _P(TuningStruct)])
_proto("cfdb_batch_assemble_pressure_device", [_vp, _vp, _vp, _vp, _vp, _pi, _d, _vp, _vp, _vp,
                                               _vp])
_proto("cfdb_batch_solve_device", [_vp, _vp, _vp, _vp, _vp, _vp, _i, _P(ControlStruct),
                                   _P(StatsStruct)])
_proto("cfdb_batch_profile", [_vp, _i, _P(KernelRecordStruct), _i, _pi])
_proto("cfdb_batch_stream", [_vp, _P(_vp)])
_proto("cfdb_batch_device_bytes", [_vp, _P(_sz)])
_proto("cfdb_batch_setup_times", [_vp, _pd, _pd])
_proto("cfdb_batch_setup_profile", [_vp, C.c_char_p, C.c_size_t])
_proto("cfdb_batch_kernel_launches", [_vp, _P(C.c_ulonglong)])



_proto("cfdb_system_profile", [_vp, _i, _i, _P(KernelRecordStruct), _i, _pi])
_proto("cfdb_system_stream", [_vp, _P(_vp)])
_proto("cfdb_system_device_bytes", [_vp, _P(_sz)])
# synthetic workloads (include/cfdb_synth.h)
_proto("cfdb_mesh_box", [_i, _i, _i, _pd, _pd, _pd, _P(_vp)])
_proto("cfdb_mesh_tet", [_i, _i, _i, _pd, _pd, _pd, _d, C.c_uint64, _P(_vp)])
_proto("cfdb_mesh_destroy", [_vp])
_proto("cfdb_mesh_sizes", [_vp, _pi, _pi, _pi, _pi])
_proto("cfdb_mesh_addressing", [_vp, _P(_pi), _P(_pi)])
_proto("cfdb_mesh_geometry", [_vp, _P(_pd), _P(_pd), _P(_pd), _P(_pd), _P(_pd)])
_proto("cfdb_mesh_faces", [_vp, _P(_pi), _P(_pi)])
_proto("cfdb_mesh_fv", [_vp, _P(_pd), _P(_pd)])
_proto("cfdb_synth_pressure_inputs", [_vp, _d, _i, _i, _i, C.c_uint64, _pd, _pd, _pd])
_proto("cfdb_positions_graded", [_i, _d, _pd])
_proto("cfdb_positions_two_sided", [_i, _d, _pd])


# -------------------------------------------------------------------------------------------
# errors
# -------------------------------------------------------------------------------------------

class CfdbError(Exception):
    code = 0


class InvalidArgument(CfdbError, ValueError):
    code = 1


class CudaError(CfdbError, RuntimeError):
    code = 2


class OutOfMemory(CfdbError, MemoryError):
    code = 3


class NoDevice(CfdbError, RuntimeError):
    code = 4


class NotReady(CfdbError, RuntimeError):
    code = 5


class Timeout(CfdbError, RuntimeError):
    code = 6


_ERRORS = {1: InvalidArgument, 2: CudaError, 3: OutOfMemory, 4: NoDevice, 5: NotReady, 6: Timeout}


def last_error() -> str:
    buf = C.create_string_buffer(4096)
    _lib.cfdb_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def _check(rc: int) -> None:
    if rc != 0:
        raise _ERRORS.get(rc, CfdbError)(last_error())


# -------------------------------------------------------------------------------------------
# array helpers
# -------------------------------------------------------------------------------------------

def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _ip(a):
    return a.ctypes.data_as(_pi)


def _dp(a):
    return a.ctypes.data_as(_pd)


def _out_f64(a, name):
    if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous):
        raise InvalidArgument(f"{name} must be a C-contiguous float64 numpy array (updated in place)")
    return a


def _torch_ready() -> None:
    """The library's kernels run on its own CUDA streams. Before a call that reads or writes
    CUDA tensors, the work already queued on torch's current stream (tensor creation, zero
    fills, copies) must be finished, or the two could overlap on the same buffers."""
    torch = sys.modules.get("torch")
    if torch is not None and torch.cuda.is_initialized():
        torch.cuda.current_stream().synchronize()


def _stream_ordered(fn):
    """Decorator for the device-array entry points: torch's queued work first (_torch_ready);
    the library call itself returns when its own kernels are done."""
    @functools.wraps(fn)
    def call(*args, **kwargs):
        _torch_ready()
        return fn(*args, **kwargs)
    return call


def _devptr(t):
    """Device pointer of a torch CUDA tensor / object with data_ptr(), or a raw int."""
    if isinstance(t, int):
        return t
    if hasattr(t, "data_ptr"):
        return int(t.data_ptr())
    raise InvalidArgument("expected a device tensor or a raw device pointer")


# -------------------------------------------------------------------------------------------
# reference-mirroring types (krylov.hpp)
# -------------------------------------------------------------------------------------------

class Method(enum.IntEnum):
    Cg = 0
    BiCgStab = 1


class Precision(enum.IntEnum):
    FP64 = 0
    MIXED = 1


@dataclass
class SolveControl:
    abs_tolerance: float = 1e-10
    max_iterations: int = 1000

    def _c(self):
        return ControlStruct(float(self.abs_tolerance), int(self.max_iterations))


@dataclass
class SolveStats:
    iterations: int = 0
    residual: float = 0.0
    converged: bool = False
    on_device: bool = False
    true_residual: float = 0.0

    @staticmethod
    def _from(s: StatsStruct) -> "SolveStats":
        return SolveStats(s.iterations, s.residual, bool(s.converged), bool(s.on_device),
                          s.true_residual)


@dataclass
class CsrView:
    """krylov.hpp:10-16: square (or rectangular: n rows) CSR matrix."""
    n: int
    row_ptr: np.ndarray
    col: np.ndarray
    val: np.ndarray

    def __post_init__(self):
        self.row_ptr = _i32(self.row_ptr)
        self.col = _i32(self.col)
        self.val = _f64(self.val)

    @property
    def nnz(self):
        return int(self.row_ptr[-1]) if len(self.row_ptr) else 0

    def _c(self):
        return CsrStruct(int(self.n), self.nnz, _ip(self.row_ptr), _ip(self.col), _dp(self.val))


def _empty_csr():
    return CsrStruct(0, 0, None, None, None)


@dataclass
class AmgLevelView:
    a: CsrView | None = None
    p: CsrView | None = None
    r: CsrView | None = None


@dataclass
class AmgView:
    """krylov.hpp:48-58."""
    levels: list = field(default_factory=list)
    coarse_inverse: np.ndarray | None = None
    smooth_sweeps: int = 2
    jacobi_weight: float = 0.7

    def _c(self):
        L = len(self.levels)
        arr = (AmgLevelStruct * max(L, 1))()
        for l, lv in enumerate(self.levels):
            arr[l].a = lv.a._c() if lv.a is not None else _empty_csr()
            arr[l].p = lv.p._c() if lv.p is not None else _empty_csr()
            arr[l].r = lv.r._c() if lv.r is not None else _empty_csr()
        ci = _f64(self.coarse_inverse) if self.coarse_inverse is not None else None
        v = AmgViewStruct(L, arr, _dp(ci) if ci is not None else None, int(self.smooth_sweeps),
                          float(self.jacobi_weight))
        v._keep = (arr, ci)
        return v


@dataclass
class LduPattern:
    """krylov.hpp:68-77."""
    n: int
    n_faces: int
    row_ptr: np.ndarray
    col: np.ndarray
    diag_pos: np.ndarray
    upper_pos: np.ndarray
    lower_pos: np.ndarray

    def __post_init__(self):
        for k in ("row_ptr", "col", "diag_pos", "upper_pos", "lower_pos"):
            setattr(self, k, _i32(getattr(self, k)))

    @property
    def nnz(self):
        return int(self.row_ptr[-1])

    def _c(self):
        return PatternStruct(int(self.n), int(self.n_faces), self.nnz, _ip(self.row_ptr),
                             _ip(self.col), _ip(self.diag_pos), _ip(self.upper_pos),
                             _ip(self.lower_pos))


# -------------------------------------------------------------------------------------------
# backend queries (krylov.hpp:118-123)
# -------------------------------------------------------------------------------------------

def backend_name() -> str:
    buf = C.create_string_buffer(64)
    _check(_lib.cfdb_backend_name(buf, len(buf)))
    return buf.value.decode()


def device_available() -> bool:
    return bool(_lib.cfdb_device_available())


def release_cached_memory() -> None:
    """Return device memory cached in the library's pools to the driver (current device)."""
    _check(_lib.cfdb_release_cached_memory())


def device_description() -> str:
    buf = C.create_string_buffer(512)
    _check(_lib.cfdb_device_description(buf, len(buf)))
    return buf.value.decode()


# -------------------------------------------------------------------------------------------
# one-shot calls
# -------------------------------------------------------------------------------------------

def assemble_convection_diffusion(n_cells, n_faces, owner, neighbour, flux, gamma, delta_coeff,
                                  convection, upper, lower, diag, divergence) -> None:
    """krylov.hpp:105-116; upper/lower/diag/divergence are numpy float64 arrays updated in
    place (diag and divergence accumulated)."""
    own, nei = _i32(owner[:n_faces]), _i32(neighbour[:n_faces])
    flux, gamma, delta = _f64(flux), _f64(gamma), _f64(delta_coeff)
    for a, nm in ((upper, "upper"), (lower, "lower"), (diag, "diag"), (divergence, "divergence")):
        _out_f64(a, nm)
    if min(len(own), len(nei), len(flux), len(gamma), len(delta), len(upper), len(lower)) < n_faces \
            or min(len(diag), len(divergence)) < n_cells:
        raise InvalidArgument("array shorter than n_faces / n_cells")
    _check(_lib.cfdb_assemble(int(n_cells), int(n_faces), _ip(own), _ip(nei), _dp(flux),
                              _dp(gamma), _dp(delta), float(convection), _dp(upper), _dp(lower),
                              _dp(diag), _dp(divergence)))


@_stream_ordered
def assemble_convection_diffusion_device(n_cells, n_faces, owner, neighbour, flux, gamma,
                                         delta_coeff, convection, upper, lower, diag,
                                         divergence) -> None:
    """Same on device arrays (torch CUDA tensors or raw device pointers)."""
    _check(_lib.cfdb_assemble_device(int(n_cells), int(n_faces), _devptr(owner),
                                     _devptr(neighbour), _devptr(flux), _devptr(gamma),
                                     _devptr(delta_coeff), float(convection), _devptr(upper),
                                     _devptr(lower), _devptr(diag), _devptr(divergence)))


def solve(a: CsrView, b, x, method: Method, control: SolveControl) -> SolveStats:
    """krylov.hpp:37-38 (Jacobi-preconditioned CG); x: float64 array, initial guess in and
    solution out."""
    b = _f64(b)
    _out_f64(x, "x")
    st = StatsStruct()
    cs, ctl = a._c(), control._c()
    _check(_lib.cfdb_solve(C.byref(cs), _dp(b), _dp(x), int(method), C.byref(ctl), C.byref(st)))
    return SolveStats._from(st)


def solve_amg_cg(amg: AmgView, b, x, control: SolveControl) -> SolveStats:
    """krylov.hpp:61-62: AMG-preconditioned CG, A = amg.levels[0].a."""
    b = _f64(b)
    _out_f64(x, "x")
    st = StatsStruct()
    v, ctl = amg._c(), control._c()
    _check(_lib.cfdb_solve_amg_cg(C.byref(v), _dp(b), _dp(x), C.byref(ctl), C.byref(st)))
    return SolveStats._from(st)


def _noalloc_args(args):
    """The torch tensor arguments of solve_device_noalloc, (tensor, name, dtype, length), checked
    for the element type the kernels read, then layout, then device, then length. Raw integer
    pointers are the caller's responsibility (the library still checks where they point and the
    CSR structure)."""
    import torch
    ts = [a for a in args if not isinstance(a[0], int)]
    for t, name, _, _ in ts:
        if not isinstance(t, torch.Tensor):
            raise InvalidArgument(f"{name}: a torch CUDA tensor or a raw device pointer is required")
    for t, name, dt, _ in ts:
        if t.dtype != getattr(torch, dt):
            raise InvalidArgument(f"{name} must be torch.{dt}, got {t.dtype}")
    for t, name, _, _ in ts:
        if not t.is_contiguous():
            raise InvalidArgument(f"{name} must be contiguous")
    for t, name, _, _ in ts:
        if not t.is_cuda or t.device.index != torch.cuda.current_device():
            raise InvalidArgument(f"{name} must be on the current CUDA device")
    for t, name, _, ln in ts:
        if t.numel() < ln:
            raise InvalidArgument(f"{name} holds {t.numel()} elements, {ln} needed")


@_stream_ordered
def solve_device_noalloc(n, nnz, row_ptr, col, val, b, x, method: Method,
                         control: SolveControl) -> SolveStats:
    """Jacobi-preconditioned CG that allocates no device memory: every array is the caller's
    device memory (torch CUDA tensors or raw pointers), work vectors live in the library's
    static device array (at most 65,536 rows). For callers that cannot call cudaMalloc.
    Tensors must be row_ptr / col int32, val / b / x float64, contiguous, on the current
    device; the call runs on the legacy default stream after torch's current stream is done."""
    n, nnz = int(n), int(nnz)
    _noalloc_args(((row_ptr, "row_ptr", "int32", n + 1), (col, "col", "int32", nnz),
                   (val, "val", "float64", nnz), (b, "b", "float64", n), (x, "x", "float64", n)))
    cs = CsrStruct(int(n), int(nnz), C.cast(_devptr(row_ptr), _pi), C.cast(_devptr(col), _pi),
                   C.cast(_devptr(val), _pd))
    st = StatsStruct()
    ctl = control._c()
    _check(_lib.cfdb_solve_device_noalloc(C.byref(cs), _devptr(b), _devptr(x), int(method),
                                          C.byref(ctl), C.byref(st)))
    return SolveStats._from(st)


@dataclass
class LduSettings:
    """LinearSolverSettings (ldu_matrix.hpp:23-28) of the GPU path, with AmgCache::max_age."""
    method: int = 0  # Method.Cg (GpuCg) or Method.BiCgStab (GpuBiCgStab)
    tolerance: float = 1e-10
    rel_tolerance: float = 0.01
    max_iterations: int = 1000
    max_age: int = 20

    def _c(self):
        return LduSettingsStruct(int(self.method), float(self.tolerance), float(self.rel_tolerance),
                                 int(self.max_iterations), int(self.max_age))


@dataclass
class LduResult:
    """LinearSolveResult (ldu_matrix.hpp:30-34) plus whether the call rebuilt the hierarchy."""
    initial_residual: float
    final_residual: float
    iterations: int
    amg_rebuilt: bool


def build_csr_pattern(n, owner, neighbour) -> LduPattern:
    """fv::build_csr_pattern (ldu_matrix.cpp:572-612) from internal-face addressing."""
    nei = _i32(neighbour)
    nf = len(nei)
    own = _i32(owner[:nf])
    rp = np.zeros(n + 1, np.int32)
    col = np.zeros(n + 2 * nf, np.int32)
    dp, up, lp = np.zeros(n, np.int32), np.zeros(nf, np.int32), np.zeros(nf, np.int32)
    nnz = C.c_int()
    _check(_lib.cfdb_build_pattern(int(n), nf, _ip(own), _ip(nei), _ip(rp), _ip(col), _ip(dp),
                                   _ip(up), _ip(lp), C.byref(nnz)))
    return LduPattern(n, nf, rp, col[:nnz.value].copy(), dp, up, lp)


# -------------------------------------------------------------------------------------------
# AMG hierarchy (fv::AmgPreconditioner::setup, host)
# -------------------------------------------------------------------------------------------

@dataclass
class AmgSettings:
    strength_threshold: float = 0.08
    max_levels: int = 25
    coarse_size: int = 400
    smooth_sweeps: int = 2
    jacobi_weight: float = 0.7
    # device setup only: rows longer than this use device-memory tables (0: the default 6144)
    device_table_limit: int = 0

    def _c(self):
        return AmgSettingsStruct(float(self.strength_threshold), int(self.max_levels),
                                 int(self.coarse_size), int(self.smooth_sweeps),
                                 float(self.jacobi_weight), int(self.device_table_limit))


class AmgHierarchy:
    """Smoothed-aggregation hierarchy (amg.cpp:122-190) built by the library, on the host or
    (device=True) with the sparse algebra on the GPU; both builds are bit-identical."""

    def __init__(self, a: CsrView, settings: AmgSettings | None = None, device: bool = False):
        self.settings = settings or AmgSettings()
        h = _vp()
        cs, ss = a._c(), self.settings._c()
        fn = _lib.cfdb_amg_setup_device if device else _lib.cfdb_amg_setup
        _check(fn(C.byref(cs), C.byref(ss), C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:  # the library may be gone at interpreter exit
            _lib.cfdb_hierarchy_destroy(h)
            self._h = None

    def levels(self) -> int:
        n = C.c_int()
        _check(_lib.cfdb_hierarchy_levels(self._h, C.byref(n)))
        return n.value

    def _csr(self, level, which):
        nr, nc, m = C.c_int(), C.c_int(), CsrStruct()
        _check(_lib.cfdb_hierarchy_level(self._h, level, which, C.byref(nr), C.byref(nc), C.byref(m)))
        nnz = m.nnz
        rp = np.ctypeslib.as_array(m.row_ptr, (nr.value + 1,)).copy()
        ci = np.ctypeslib.as_array(m.col, (max(nnz, 1),))[:nnz].copy() if nnz else np.zeros(0, np.int32)
        va = np.ctypeslib.as_array(m.val, (max(nnz, 1),))[:nnz].copy() if nnz else np.zeros(0)
        return CsrView(nr.value, rp, ci, va), nc.value

    def level_matrix(self, level) -> CsrView:
        return self._csr(level, 0)[0]

    def level_prolongation(self, level) -> CsrView:
        return self._csr(level, 1)[0]

    def level_restriction(self, level) -> CsrView:
        return self._csr(level, 2)[0]

    def level_size(self, level) -> int:
        return self.level_matrix(level).n

    def aggregates(self, level):
        p, n = _pi(), C.c_int()
        _check(_lib.cfdb_hierarchy_aggregates(self._h, level, C.byref(p), C.byref(n)))
        return np.ctypeslib.as_array(p, (self.level_size(level),)).copy(), n.value

    def coarse_inverse(self) -> np.ndarray:
        p, n = _pd(), C.c_int()
        _check(_lib.cfdb_hierarchy_coarse_inverse(self._h, C.byref(p), C.byref(n)))
        return np.ctypeslib.as_array(p, (n.value * n.value,)).copy()

    def operator_complexity(self) -> float:
        v = C.c_double()
        _check(_lib.cfdb_hierarchy_operator_complexity(self._h, C.byref(v)))
        return v.value

    def view(self) -> AmgView:
        L = self.levels()
        lv = []
        for l in range(L):
            a = self.level_matrix(l)
            p = self.level_prolongation(l) if l + 1 < L else None
            r = self.level_restriction(l) if l + 1 < L else None
            lv.append(AmgLevelView(a, p, r))
        return AmgView(lv, self.coarse_inverse(), self.settings.smooth_sweeps,
                       self.settings.jacobi_weight)


# -------------------------------------------------------------------------------------------
# persistent system (DeviceSolver)
# -------------------------------------------------------------------------------------------

class DeviceSolver:
    """krylov.hpp:83-103: persistent solver for repeated solves on one LDU pattern."""

    def __init__(self, pattern: LduPattern | None = None, *, mesh=None):
        h = _vp()
        if pattern is not None:
            self.pattern = pattern
            ps = pattern._c()
            _check(_lib.cfdb_system_create(C.byref(ps), C.byref(h)))
            self.n, self.n_faces = pattern.n, pattern.n_faces
        elif mesh is not None:
            n, own, nei = mesh
            nei = _i32(nei)
            own = _i32(own[:len(nei)])
            _check(_lib.cfdb_system_create_mesh(int(n), len(nei), _ip(own), _ip(nei), C.byref(h)))
            self.n, self.n_faces = int(n), len(nei)
            self.pattern = None
        else:
            raise InvalidArgument("DeviceSolver needs a pattern or mesh addressing")
        self._h = h

    def close(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:  # the library may be gone at interpreter exit
            _lib.cfdb_system_destroy(h)
            self._h = None

    __del__ = close

    def on_device(self) -> bool:
        return bool(_lib.cfdb_system_on_device(self._h))

    def set_amg(self, amg: AmgView) -> None:
        v = amg._c()
        _check(_lib.cfdb_system_set_amg(self._h, C.byref(v)))

    def setup_amg(self, diag, upper, lower, settings: AmgSettings | None = None,
                  device: bool = True) -> None:
        """AmgPreconditioner::setup from LDU coefficients and installation of the hierarchy:
        built on the GPU (device=True, the default; the coefficients may also be CUDA tensors
        ready on the current stream) or on the host (device=False); both are bit-identical."""
        s = (settings or AmgSettings())._c()
        if not device:
            _check(_lib.cfdb_system_setup_amg(self._h, _dp(_f64(diag)), _dp(_f64(upper)),
                                              _dp(_f64(lower)), C.byref(s)))
            return
        if hasattr(diag, "is_cuda") and diag.is_cuda:
            import torch
            torch.cuda.current_stream().synchronize()
            _check(_lib.cfdb_system_setup_amg_device(self._h, _devptr(diag), _devptr(upper),
                                                     _devptr(lower), C.byref(s), 1))
            return
        d, u, lo = _f64(diag), _f64(upper), _f64(lower)
        _check(_lib.cfdb_system_setup_amg_device(self._h, d.ctypes.data, u.ctypes.data,
                                                 lo.ctypes.data, C.byref(s), 0))

    def time_sweep(self, level: int, reps: int = 20):
        """(ms, algorithmic bytes) of one Jacobi sweep of `level`, timed over `reps`
        back-to-back launches with CUDA events."""
        ms, by = C.c_double(), C.c_double()
        _check(_lib.cfdb_system_time_sweep(self._h, int(level), int(reps), C.byref(ms), C.byref(by)))
        return ms.value, by.value

    def set_keep_levels(self, keep: bool) -> None:
        """Keep a device setup's levels on the device so that later precision or tuning changes
        can rebuild the plan (default True)."""
        _check(_lib.cfdb_system_set_keep_levels(self._h, 1 if keep else 0))

    def setup_profile(self) -> dict:
        """Seconds per phase of the last hierarchy setup."""
        buf = C.create_string_buffer(1024)
        _check(_lib.cfdb_system_setup_profile(self._h, buf, len(buf)))
        out = {}
        for item in buf.value.decode().split(";"):
            if item:
                k, v = item.split("=")
                out[k] = float(v)
        return out

    def set_precision(self, precision: Precision) -> None:
        _check(_lib.cfdb_system_set_precision(self._h, int(precision)))

    def solve(self, diag, upper, lower, b, x, method: Method = Method.Cg, use_amg: bool = True,
              control: SolveControl | None = None) -> SolveStats:
        diag, upper, lower, b = _f64(diag), _f64(upper), _f64(lower), _f64(b)
        _out_f64(x, "x")
        if len(diag) != self.n or len(b) != self.n or len(x) != self.n or \
                len(upper) != self.n_faces or len(lower) != self.n_faces:
            raise InvalidArgument("array sizes do not match the pattern")
        st = StatsStruct()
        ctl = (control or SolveControl())._c()
        _check(_lib.cfdb_system_solve(self._h, _dp(diag), _dp(upper), _dp(lower), _dp(b), _dp(x),
                                      int(method), 1 if use_amg else 0, C.byref(ctl),
                                      C.byref(st)))
        return SolveStats._from(st)

    @_stream_ordered
    def solve_device(self, diag, upper, lower, b, x, method: Method = Method.Cg,
                     use_amg: bool = True, control: SolveControl | None = None) -> SolveStats:
        """All arrays device-resident (torch CUDA float64 tensors or raw pointers)."""
        st = StatsStruct()
        ctl = (control or SolveControl())._c()
        _check(_lib.cfdb_system_solve_device(self._h, _devptr(diag), _devptr(upper),
                                             _devptr(lower), _devptr(b), _devptr(x), int(method),
                                             1 if use_amg else 0, C.byref(ctl), C.byref(st)))
        return SolveStats._from(st)

    def solve_ldu(self, diag, upper, lower, source, x, settings: LduSettings | None = None,
                  amg: AmgSettings | None = None) -> LduResult:
        """LduMatrix::solve on the GPU path with the AmgCache rule (ldu_matrix.cpp:111-131,
        287-366): normalised residuals before and after, hierarchy (re)built on the device at
        the first CG call and every max_age calls. Host numpy arrays (x updated in place) or
        CUDA tensors (ready on the current stream)."""
        s = (settings or LduSettings())._c()
        a = (amg or AmgSettings())._c()
        r = LduResultStruct()
        if hasattr(diag, "is_cuda") and diag.is_cuda:
            import torch
            torch.cuda.current_stream().synchronize()
            _check(_lib.cfdb_system_solve_ldu(self._h, _devptr(diag), _devptr(upper), _devptr(lower),
                                              _devptr(source), _devptr(x), C.byref(s), C.byref(a), 1,
                                              C.byref(r)))
        else:
            d, u, lo, b = _f64(diag), _f64(upper), _f64(lower), _f64(source)
            _out_f64(x, "x")
            if len(d) != self.n or len(b) != self.n or len(x) != self.n or \
                    len(u) != self.n_faces or len(lo) != self.n_faces:
                raise InvalidArgument("array sizes do not match the pattern")
            _check(_lib.cfdb_system_solve_ldu(self._h, d.ctypes.data, u.ctypes.data, lo.ctypes.data,
                                              b.ctypes.data, x.ctypes.data, C.byref(s), C.byref(a), 0,
                                              C.byref(r)))
        return LduResult(r.initial_residual, r.final_residual, r.iterations, bool(r.amg_rebuilt))

    @_stream_ordered
    def assemble_device(self, flux, gamma, delta, convection, upper, lower, diag, div) -> None:
        _check(_lib.cfdb_system_assemble_device(self._h, _devptr(flux), _devptr(gamma),
                                                _devptr(delta), float(convection),
                                                _devptr(upper), _devptr(lower), _devptr(diag),
                                                _devptr(div)))

    def apply_amg(self, r) -> np.ndarray:
        """One V-cycle z = M^-1 r on the installed hierarchy (AmgPreconditioner::apply)."""
        r = _f64(r)
        z = np.zeros(self.n)
        _check(_lib.cfdb_system_apply_amg(self._h, _dp(r), _dp(z)))
        return z

    def assemble(self, flux, gamma, delta, convection, upper, lower, diag, div) -> None:
        """assemble_convection_diffusion on the system's mesh with host arrays (in place)."""
        for a, nm in ((upper, "upper"), (lower, "lower"), (diag, "diag"), (div, "div")):
            _out_f64(a, nm)
        flux, gamma, delta = _f64(flux), _f64(gamma), _f64(delta)
        _check(_lib.cfdb_system_assemble(self._h, _dp(flux), _dp(gamma), _dp(delta),
                                         float(convection), _dp(upper), _dp(lower), _dp(diag),
                                         _dp(div)))

    @_stream_ordered
    def assemble_pressure_device(self, flux, gamma, delta, source0, upper, lower, diag, source,
                                 diag0=None, ref_cell=0, ref_value=0.0) -> None:
        """Pressure-equation assembly on device arrays (flow_solver.cpp:757-796)."""
        _check(_lib.cfdb_system_assemble_pressure_device(
            self._h, _devptr(flux), _devptr(gamma), _devptr(delta),
            _devptr(diag0) if diag0 is not None else None, _devptr(source0), int(ref_cell),
            float(ref_value), _devptr(upper), _devptr(lower), _devptr(diag), _devptr(source)))

    @_stream_ordered
    def correct_pressure_device(self, flux, gamma, delta, p_new, phi, p, p_prev=None, alpha=1.0,
                                non_orth=None) -> None:
        """Conservative face flux phi and under-relaxed pressure p after the pressure solve
        (flow_solver.cpp:821-840), on device arrays; enqueued on the solver's stream."""
        _check(_lib.cfdb_system_correct_pressure_device(
            self._h, _devptr(flux), _devptr(gamma), _devptr(delta),
            _devptr(non_orth) if non_orth is not None else None, _devptr(p_new),
            _devptr(p_prev) if p_prev is not None else None, float(alpha), _devptr(phi), _devptr(p)))

    def kernel_launches(self) -> int:
        c = C.c_ulonglong()
        _check(_lib.cfdb_system_kernel_launches(self._h, C.byref(c)))
        return c.value

    def set_ordered(self, ordered: bool) -> None:
        """Bit-reproducible FP64 V-cycles (thread-per-row sums in CSR order on every level)."""
        _check(_lib.cfdb_system_set_ordered(self._h, 1 if ordered else 0))

    def profile(self, use_amg: bool = True, reps: int = 5) -> list:
        """Per-kernel device time (ms) and algorithmic bytes of the initial preconditioning and
        one iteration, in launch order: [(name, level, ms, bytes), ...]."""
        recs = (KernelRecordStruct * 512)()
        n = C.c_int()
        _check(_lib.cfdb_system_profile(self._h, 1 if use_amg else 0, int(reps), recs, 512,
                                        C.byref(n)))
        return [(recs[i].name.decode(), recs[i].level, recs[i].ms, recs[i].bytes)
                for i in range(n.value)]

    def stream(self) -> int:
        s = _vp()
        _check(_lib.cfdb_system_stream(self._h, C.byref(s)))
        return s.value or 0

    def device_bytes(self) -> int:
        b = C.c_size_t()
        _check(_lib.cfdb_system_device_bytes(self._h, C.byref(b)))
        return b.value


@dataclass
class Tuning:
    """Launch-shape / schedule knobs of the device plan (cfdb_tuning)."""
    target_tiles: int = 148 * 8
    wide_row: int = 48
    lanes_div: int = 16
    fuse_first: int = 0
    sell_rows: int = 256
    krylov_pair: int = 1
    tail_rows: int = 0
    col16: int = 0
    pdl: int = 1
    wait_polls: int = 1 << 22  # bounded device waits; < 0 makes them give up at once (tests)
    mixed_sweeps: int = 0  # mixed precision: Jacobi sweeps per level (0: the hierarchy's)
    mixed_weight: float = 0.0  # mixed precision: Jacobi weight (0: the hierarchy's)
    tail_cluster: int = 0  # tail as one cluster of this many CTAs (2..16); 0: cooperative grid
    vcycle_pair: int = 0  # V-cycle SELL kernels: two rows per thread per pass (1) or one (0)
    krylov_stage: int = 0  # level-0 Krylov SpMV staged through shared memory in 2..4 buffers; 0: off

    def _c(self):
        return TuningStruct(int(self.target_tiles), int(self.wide_row), int(self.lanes_div),
                            int(self.fuse_first), int(self.sell_rows), int(self.krylov_pair),
                            int(self.tail_rows), int(self.col16), int(self.pdl), int(self.wait_polls),
                            int(self.mixed_sweeps), float(self.mixed_weight), int(self.tail_cluster),
                            int(self.vcycle_pair), int(self.krylov_stage))


def _set_system_tuning(self, t: Tuning) -> None:
    ts = t._c()
    _check(_lib.cfdb_system_set_tuning(self._h, C.byref(ts)))


DeviceSolver.set_tuning = _set_system_tuning


def _profile_records(fn, handle, *args):
    recs = (KernelRecordStruct * 1024)()
    n = C.c_int()
    _check(fn(handle, *args, recs, 1024, C.byref(n)))
    return [(recs[i].name.decode(), recs[i].level, recs[i].ms, recs[i].bytes) for i in range(n.value)]


class Batch:
    """Many independent pressure systems of uneven size solved in one device plan: every
    kernel launch covers all systems, with per-system convergence and dot products. Arrays
    are concatenated in system order (cells of system 0, then 1, ...; faces likewise);
    owner / neighbour hold local cell indices."""

    def __init__(self, n_cells, n_faces, owner, neighbour):
        nc, nf = _i32(n_cells), _i32(n_faces)
        own, nei = _i32(owner), _i32(neighbour)
        if len(nc) != len(nf) or len(own) != int(nf.sum()) or len(nei) != int(nf.sum()):
            raise InvalidArgument("batch: inconsistent sizes")
        h = _vp()
        _check(_lib.cfdb_batch_create(len(nc), _ip(nc), _ip(nf), _ip(own), _ip(nei), C.byref(h)))
        self._h = h
        self.n_systems = len(nc)
        self.n_cells, self.n_faces = nc, nf
        self.total_cells, self.total_faces = int(nc.sum()), int(nf.sum())

    def close(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:  # the library may be gone at interpreter exit
            _lib.cfdb_batch_destroy(h)
            self._h = None

    __del__ = close

    def setup_amg(self, diag, upper, lower, settings: AmgSettings | None = None, device: bool = False,
                  concurrency: int = 0) -> None:
        """AmgPreconditioner::setup of every system: on the host (OpenMP over systems; host
        arrays) or on the device (device setup per system, `concurrency` systems at a time; CUDA
        tensors), bit-identical either way."""
        s = (settings or AmgSettings())._c()
        if device:
            _torch_ready()
            _check(_lib.cfdb_batch_setup_amg_device(self._h, _devptr(diag), _devptr(upper), _devptr(lower),
                                                    C.byref(s), int(concurrency)))
            return
        _check(_lib.cfdb_batch_setup_amg(self._h, _dp(_f64(diag)), _dp(_f64(upper)),
                                         _dp(_f64(lower)), C.byref(s)))

    def setup_times(self) -> dict:
        """Wall seconds of the last setup: per-system hierarchies and the batch plan."""
        h, p = C.c_double(), C.c_double()
        _check(_lib.cfdb_batch_setup_times(self._h, C.byref(h), C.byref(p)))
        out = {"hierarchies_s": h.value, "plan_s": p.value}
        buf = C.create_string_buffer(4096)
        _check(_lib.cfdb_batch_setup_profile(self._h, buf, len(buf)))
        for item in buf.value.decode().split(";"):
            name, _, v = item.partition("=")
            if v:
                out[name if name.startswith("plan") else "plan_" + name] = float(v)
        return out

    def set_precision(self, precision: Precision) -> None:
        _check(_lib.cfdb_batch_set_precision(self._h, int(precision)))

    def set_tuning(self, t: Tuning) -> None:
        ts = t._c()
        _check(_lib.cfdb_batch_set_tuning(self._h, C.byref(ts)))

    @_stream_ordered
    def assemble_pressure_device(self, flux, gamma, delta, source0, upper, lower, diag, source,
                                 ref_cells=None, ref_value=0.0) -> None:
        refs = _i32(ref_cells if ref_cells is not None else np.zeros(self.n_systems))
        _check(_lib.cfdb_batch_assemble_pressure_device(
            self._h, _devptr(flux), _devptr(gamma), _devptr(delta), _devptr(source0), _ip(refs),
            float(ref_value), _devptr(upper), _devptr(lower), _devptr(diag), _devptr(source)))

    @_stream_ordered
    def solve_device(self, diag, upper, lower, rhs, x, controls, use_amg=True):
        ctl = (ControlStruct * self.n_systems)(*[c._c() for c in controls])
        st = (StatsStruct * self.n_systems)()
        _check(_lib.cfdb_batch_solve_device(self._h, _devptr(diag), _devptr(upper), _devptr(lower),
                                            _devptr(rhs), _devptr(x), 1 if use_amg else 0, ctl, st))
        return [SolveStats._from(st[i]) for i in range(self.n_systems)]

    def profile(self, reps: int = 3) -> list:
        return _profile_records(_lib.cfdb_batch_profile, self._h, int(reps))

    def stream(self) -> int:
        s = _vp()
        _check(_lib.cfdb_batch_stream(self._h, C.byref(s)))
        return s.value or 0

    def device_bytes(self) -> int:
        b = C.c_size_t()
        _check(_lib.cfdb_batch_device_bytes(self._h, C.byref(b)))
        return b.value

    def kernel_launches(self) -> int:
        c = C.c_ulonglong()
        _check(_lib.cfdb_batch_kernel_launches(self._h, C.byref(c)))
        return c.value


# -------------------------------------------------------------------------------------------
# synthetic workloads (include/cfdb_synth.h)
# -------------------------------------------------------------------------------------------

def positions_graded(n: int, grading: float) -> np.ndarray:
    out = np.zeros(n + 1)
    _check(_lib.cfdb_positions_graded(n, float(grading), _dp(out)))
    return out


def positions_two_sided(n: int, ratio: float) -> np.ndarray:
    out = np.zeros(n + 1)
    _check(_lib.cfdb_positions_two_sided(n, float(ratio), _dp(out)))
    return out


def _view_copy(ptr, shape, dtype):
    """Copy of a library-owned array; an empty array may come back as a null pointer."""
    if int(np.prod(shape)) == 0:
        return np.zeros(shape, dtype)
    return np.ctypeslib.as_array(ptr, shape).copy()


class Mesh:
    """Box (hex) or jittered 6-tet mesh in the reference's face ordering, with geometry."""

    def __init__(self, h, nx, ny, nz):
        self._h = h
        self.shape = (nx, ny, nz)
        nc, nf, ni, npn = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _check(_lib.cfdb_mesh_sizes(h, C.byref(nc), C.byref(nf), C.byref(ni), C.byref(npn)))
        self.n_cells, self.n_faces, self.n_internal_faces, self.n_points = (
            nc.value, nf.value, ni.value, npn.value)
        o, n = _pi(), _pi()
        _check(_lib.cfdb_mesh_addressing(h, C.byref(o), C.byref(n)))
        self.owner = _view_copy(o, (self.n_faces,), np.int32)
        self.neighbour = _view_copy(n, (self.n_internal_faces,), np.int32)
        pts, fc, sf, cc, vol = _pd(), _pd(), _pd(), _pd(), _pd()
        _check(_lib.cfdb_mesh_geometry(h, C.byref(pts), C.byref(fc), C.byref(sf), C.byref(cc),
                                       C.byref(vol)))
        self.points = _view_copy(pts, (self.n_points, 3), np.float64)
        self.face_centres = _view_copy(fc, (self.n_faces, 3), np.float64)
        self.face_areas = _view_copy(sf, (self.n_faces, 3), np.float64)
        self.cell_centres = _view_copy(cc, (self.n_cells, 3), np.float64)
        self.cell_volumes = _view_copy(vol, (self.n_cells,), np.float64)
        dl, w = _pd(), _pd()
        _check(_lib.cfdb_mesh_fv(h, C.byref(dl), C.byref(w)))
        self.delta = _view_copy(dl, (self.n_internal_faces,), np.float64)
        self.weights = _view_copy(w, (self.n_internal_faces,), np.float64)
        fo, fn = _pi(), _pi()
        _check(_lib.cfdb_mesh_faces(h, C.byref(fo), C.byref(fn)))
        self.face_offsets = _view_copy(fo, (self.n_faces + 1,), np.int32)
        self.face_nodes = np.ctypeslib.as_array(fn, (int(self.face_offsets[-1]),)).copy()

    @staticmethod
    def box(nx, ny, nz, xs=None, ys=None, zs=None) -> "Mesh":
        xs = _f64(xs if xs is not None else np.linspace(0, 1, nx + 1))
        ys = _f64(ys if ys is not None else np.linspace(0, 1, ny + 1))
        zs = _f64(zs if zs is not None else np.linspace(0, 1, nz + 1))
        h = _vp()
        _check(_lib.cfdb_mesh_box(nx, ny, nz, _dp(xs), _dp(ys), _dp(zs), C.byref(h)))
        return Mesh(h, nx, ny, nz)

    @staticmethod
    def tet(nx, ny, nz, jitter=0.2, seed=0, xs=None, ys=None, zs=None) -> "Mesh":
        xs = _f64(xs if xs is not None else np.linspace(0, 1, nx + 1))
        ys = _f64(ys if ys is not None else np.linspace(0, 1, ny + 1))
        zs = _f64(zs if zs is not None else np.linspace(0, 1, nz + 1))
        h = _vp()
        _check(_lib.cfdb_mesh_tet(nx, ny, nz, _dp(xs), _dp(ys), _dp(zs), float(jitter),
                                  int(seed), C.byref(h)))
        return Mesh(h, nx, ny, nz)

    def pressure_inputs(self, sigma=0.0, unit_rau=False, flux_kind=0, rhs_kind=1, seed=0):
        """(gamma, flux, source) of a pressure system on this mesh."""
        g = np.zeros(self.n_internal_faces)
        f = np.zeros(self.n_internal_faces)
        s = np.zeros(self.n_cells)
        _check(_lib.cfdb_synth_pressure_inputs(self._h, float(sigma), 1 if unit_rau else 0,
                                               int(flux_kind), int(rhs_kind), int(seed), _dp(g),
                                               _dp(f), _dp(s)))
        return g, f, s

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:  # the library may be gone at interpreter exit
            _lib.cfdb_mesh_destroy(h)
            self._h = None


class BoundaryKind(enum.IntEnum):
    """flow_solver.hpp:16 FlowBoundary."""
    VelocityInlet = 0
    Wall = 1
    PressureOutlet = 2
    Symmetry = 3
    Empty = 4


class FvGeometry:
    """Device copy of a mesh's geometry for the pressure gradient and velocity correction of
    FlowSolver::pressure_correction (flow_solver.cpp:339-372, 843-846)."""

    def __init__(self, mesh: "Mesh", boundary_kind, boundary_pressure=None):
        nb = mesh.n_faces - mesh.n_internal_faces
        kinds = _i32(boundary_kind)
        pout = _f64(boundary_pressure if boundary_pressure is not None else np.zeros(nb))
        if len(kinds) != nb or len(pout) != nb:
            raise InvalidArgument("one boundary kind and pressure per boundary face")
        self.n_cells, self.n_faces, self.n_internal_faces = mesh.n_cells, mesh.n_faces, mesh.n_internal_faces
        own, nei = _i32(mesh.owner), _i32(mesh.neighbour)
        sf, cf = _f64(mesh.face_areas).ravel(), _f64(mesh.face_centres).ravel()
        cc, vol, w = _f64(mesh.cell_centres).ravel(), _f64(mesh.cell_volumes), _f64(mesh.weights)
        h = _vp()
        _check(_lib.cfdb_fv_create(mesh.n_cells, mesh.n_faces, mesh.n_internal_faces, _ip(own), _ip(nei),
                                   _dp(sf), _dp(cf), _dp(cc), _dp(vol), _dp(w), _ip(kinds), _dp(pout),
                                   C.byref(h)))
        self._h = h

    @_stream_ordered
    def pressure_gradient_device(self, p, grad) -> None:
        """grad (n_cells x 3, CUDA float64) of the cell pressure p (CUDA float64)."""
        _check(_lib.cfdb_fv_pressure_gradient_device(self._h, _devptr(p), _devptr(grad)))

    @_stream_ordered
    def correct_velocity_device(self, hbya, rau, grad, u) -> None:
        _check(_lib.cfdb_fv_correct_velocity_device(self._h, _devptr(hbya), _devptr(rau),
                                                    _devptr(grad), _devptr(u)))

    def delta_device(self) -> int:
        """Device pointer of the delta coefficients of all faces (owned by this object)."""
        d = _vp()
        _check(_lib.cfdb_fv_delta_device(self._h, C.byref(d)))
        return int(d.value)

    @_stream_ordered
    def hbya_rau_device(self, mom_diag, mom_upper, mom_lower, mom_source, u, hbya, rau) -> None:
        _check(_lib.cfdb_fv_hbya_rau_device(self._h, _devptr(mom_diag), _devptr(mom_upper),
                                            _devptr(mom_lower), _devptr(mom_source), _devptr(u),
                                            _devptr(hbya), _devptr(rau)))

    @_stream_ordered
    def face_flux_device(self, hbya, rau, fixed_velocity, phi_hbya, rau_f, u_prev=None,
                         phi_prev=None, beta=0.0) -> None:
        _check(_lib.cfdb_fv_face_flux_device(
            self._h, _devptr(hbya), _devptr(rau), _devptr(fixed_velocity),
            _devptr(u_prev) if u_prev is not None else None,
            _devptr(phi_prev) if phi_prev is not None else None, float(beta), _devptr(phi_hbya),
            _devptr(rau_f)))

    @_stream_ordered
    def pressure_boundary_device(self, phi_hbya, rau_f, diag, source, ref_cell=-1, ref_value=0.0):
        _check(_lib.cfdb_fv_pressure_boundary_device(self._h, _devptr(phi_hbya), _devptr(rau_f),
                                                     int(ref_cell), float(ref_value), _devptr(diag),
                                                     _devptr(source)))

    @_stream_ordered
    def non_orth_device(self, grad, rau_f, base_source, non_orth, source) -> None:
        _check(_lib.cfdb_fv_non_orth_device(self._h, _devptr(grad), _devptr(rau_f),
                                            _devptr(base_source), _devptr(non_orth), _devptr(source)))

    @_stream_ordered
    def correct_flux_device(self, phi_hbya, rau_f, p_new, phi, non_orth=None) -> None:
        _check(_lib.cfdb_fv_correct_flux_device(
            self._h, _devptr(phi_hbya), _devptr(rau_f),
            _devptr(non_orth) if non_orth is not None else None, _devptr(p_new), _devptr(phi)))

    @_stream_ordered
    def relax_device(self, p_prev, p_new, alpha, p) -> None:
        _check(_lib.cfdb_fv_relax_device(self._h, _devptr(p_prev), _devptr(p_new), float(alpha),
                                         _devptr(p)))

    def close(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:  # the library may be gone at interpreter exit
            _lib.cfdb_fv_destroy(h)
            self._h = None

    __del__ = close


from . import workloads  # noqa: E402,F401  (configs of the pressure systems)
