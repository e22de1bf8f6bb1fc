"""ctypes binding of ``include/meanas_fdfd.h`` (``libmeanas_fdfd.so``).

The structures below mirror the C declarations field for field.  Loading fails
loudly when the library is missing: there is no CPU fallback on the product path.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / 'libmeanas_fdfd.so'

ABI_VERSION = 1

STATUS_CONVERGED = 1
STATUS_MAXITER = 2
STATUS_BREAKDOWN = 3
STATUS_NONFINITE = 4
STATUS_NAMES = {0: 'running', 1: 'converged', 2: 'maxiter', 3: 'breakdown', 4: 'nonfinite'}

GRID_FP32 = 1
OP_A0, OP_SYM, OP_SYM_H = 0, 1, 2
C128, C64 = 0, 1
METHOD_COCG, METHOD_MIXED, METHOD_BICGSTAB = 0, 1, 2
CRIT_TRUE, CRIT_PRECOND = 0, 1


class GridDesc(C.Structure):
    _fields_ = [
        ('shape', C.c_int32 * 3),
        ('flags', C.c_int32),
        ('omega', C.c_double * 2),
        ('dxe', C.c_void_p * 3),
        ('dxh', C.c_void_p * 3),
        ('inv_dxe', C.c_void_p * 3),
        ('inv_dxh', C.c_void_p * 3),
        ('epsilon', C.c_void_p),
        ('mu', C.c_void_p),
        ('pec', C.c_void_p),
        ('pmc', C.c_void_p),
    ]


class SolveOpts(C.Structure):
    _fields_ = [
        ('method', C.c_int32),
        ('criterion', C.c_int32),
        ('adjoint', C.c_int32),
        ('maxiter', C.c_int32),
        ('rtol', C.c_double),
        ('atol', C.c_double),
        ('has_guess', C.c_int32),
        ('chunk', C.c_int32),
        ('use_graph', C.c_int32),
        ('max_outer', C.c_int32),
        ('inner_rtol', C.c_double),
        ('history', C.c_void_p),
        ('profile', C.c_int32),
        ('pad_', C.c_int32),
    ]


class SolveInfo(C.Structure):
    _fields_ = [
        ('status', C.c_int32),
        ('iterations', C.c_int32),
        ('outer_iterations', C.c_int32),
        ('kernel_launches', C.c_int32),
        ('residual', C.c_double),
        ('residual_pc', C.c_double),
        ('kernel_ms', C.c_double * 4),
        ('kernel_count', C.c_int32 * 4),
    ]


class CsrDesc(C.Structure):  # fdfd_csr_desc
    _fields_ = [('n', C.c_int64), ('nnz', C.c_int64), ('indptr', C.c_void_p), ('indices', C.c_void_p),
                ('data', C.c_void_p)]


class FdtdFace(C.Structure):  # fdfd_fdtd_face
    _fields_ = [('thickness', C.c_int32), ('pad_', C.c_int32), ('param_e', C.c_void_p), ('param_h', C.c_void_p),
                ('psi_e', C.c_void_p * 2), ('psi_h', C.c_void_p * 2)]


class FdtdDesc(C.Structure):  # fdfd_fdtd_desc
    _fields_ = [('shape', C.c_int32 * 3), ('field_type', C.c_int32), ('psi_type', C.c_int32), ('form', C.c_int32),
                ('dt', C.c_double), ('dxe', C.c_void_p * 3), ('dxh', C.c_void_p * 3), ('epsilon', C.c_void_p),
                ('mu', C.c_void_p), ('face', (FdtdFace * 2) * 3)]


class ModeSlice(C.Structure):  # fdfd_mode_slice
    _fields_ = [('axis', C.c_int32), ('polarity', C.c_int32), ('lo', C.c_int32 * 3), ('hi', C.c_int32 * 3),
                ('mask_lo', C.c_int32), ('mask_hi', C.c_int32)]


REAL64, REAL32 = 0, 1
FDTD_PLAIN, FDTD_CPML = 0, 1


EXPORTS = {
    'fdfd_abi_version': (C.c_int, []),
    'fdfd_last_error': (C.c_char_p, []),
    'fdfd_plan_workspace_bytes': (C.c_int, [C.POINTER(GridDesc), C.POINTER(C.c_size_t)]),
    'fdfd_plan_create': (C.c_int, [C.POINTER(GridDesc), C.c_void_p, C.c_size_t, C.c_void_p, C.POINTER(C.c_void_p)]),
    'fdfd_plan_update': (C.c_int, [C.c_void_p, C.POINTER(GridDesc), C.c_void_p]),
    'fdfd_plan_destroy': (C.c_int, [C.c_void_p]),
    'fdfd_plan_set_xchunk': (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    'fdfd_apply': (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    'fdfd_solve_workspace_bytes': (C.c_int, [C.c_void_p, C.POINTER(SolveOpts), C.POINTER(C.c_size_t)]),
    'fdfd_solve': (C.c_int, [C.c_void_p, C.POINTER(SolveOpts), C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                             C.POINTER(SolveInfo), C.c_void_p]),
    'fdfd_residual_workspace_bytes': (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    'fdfd_residual': (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.c_void_p,
                                C.c_size_t, C.c_void_p]),
    'fdfd_eps_gradient': (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    'fdfd_residual_static': (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.c_void_p]),
    'fdfd_e2h': (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    'fdfd_tfsf_source': (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    'fdfd_mode_expand': (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(ModeSlice), C.c_void_p,
                                   C.c_void_p, C.c_void_p]),
    'fdfd_mode_source': (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(ModeSlice), C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p]),
    'fdfd_csr_spmv': (C.c_int, [C.POINTER(CsrDesc), C.c_void_p, C.c_void_p, C.c_void_p]),
    'fdfd_csr_solve_workspace_bytes': (C.c_int, [C.POINTER(CsrDesc), C.POINTER(C.c_size_t)]),
    'fdfd_csr_solve': (C.c_int, [C.POINTER(CsrDesc), C.POINTER(SolveOpts), C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_size_t, C.POINTER(SolveInfo), C.c_void_p]),
    'fdfd_fdtd_update_h': (C.c_int, [C.POINTER(FdtdDesc), C.c_void_p, C.c_void_p, C.c_void_p]),
    'fdfd_fdtd_update_e': (C.c_int, [C.POINTER(FdtdDesc), C.c_void_p, C.c_void_p, C.c_void_p]),
}

# fdfd_tfsf_source flags
SRC_EDGES = 1
SRC_PERIODIC = 2

# fdfd_e2h flags (include/meanas_fdfd.h)
E2H_CONJ = 1
E2H_H_IN = 2

_lib: C.CDLL | None = None


class FDFDError(RuntimeError):
    """An argument or CUDA error reported by libmeanas_fdfd (negative return code)."""


def load() -> C.CDLL:
    """Load ``libmeanas_fdfd.so`` (building it first if the sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    from . import build as _build
    if _build.needs_build():
        _build.build()
    if not LIB_PATH.exists():
        raise FDFDError(f'{LIB_PATH} is missing and could not be built')
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.fdfd_abi_version() != ABI_VERSION:
        raise FDFDError(f'libmeanas_fdfd ABI {lib.fdfd_abi_version()} != {ABI_VERSION}')
    _lib = lib
    return lib


def check(rc: int) -> int:
    """Raise on negative return codes; pass solver statuses (>= 0) through."""
    if rc < 0:
        msg = load().fdfd_last_error().decode(errors='replace')
        raise FDFDError(f'libmeanas_fdfd error {rc}: {msg}')
    return rc
