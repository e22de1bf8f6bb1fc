"""GPU solver for the reference's second plugin point: ``matrix_solver(A, b, **opts) -> x``.

``meanas.fdfd.solvers.generic`` assembles the symmetrised CSR operator and hands it to
``matrix_solver`` (``meanas/fdfd/solvers.py:97-103,134``; the default is ``_scipy_qmr``,
``:21-63``).  ``matrix_solver`` below takes the same arguments and returns the same thing
(the last iterate, converged or not), solving on the GPU with complex128 BiCGSTAB over
the CSR matrix (``fdfd_csr_solve`` in ``libmeanas_fdfd.so``)::

    from meanas.fdfd import solvers
    from meanas_b200.csr import matrix_solver
    E = solvers.generic(omega, dxes, J, epsilon, matrix_solver=matrix_solver,
                        matrix_solver_opts=dict(rtol=1e-8))

It works for any square complex CSR matrix (for example operators built from ``eh_full``
or ``h_full``), where the matrix-free ``meanas_b200.generic`` covers only ``e_full``.
Stopping follows scipy: ``||r|| <= max(rtol ||b||, atol)`` on the recurrence residual,
``maxiter`` (default ``10 n``) iterations at most; ``x0`` is the initial guess.
"""
from __future__ import annotations

import ctypes as C
import logging
from typing import Any

import numpy
import torch
from scipy import sparse

from . import _lib
from .operators import _device, _stream_handle, as_device

logger = logging.getLogger(__name__)

_STATUS = {1: 'converged', 2: 'maxiter', 3: 'breakdown', 4: 'nonfinite'}


class CsrMatrix:
    """A square complex128 CSR matrix resident on the device."""

    def __init__(self, A, device: Any | None = None):
        A = sparse.csr_array(A)
        if A.shape[0] != A.shape[1]:
            raise ValueError(f'matrix must be square, got {A.shape}')
        if A.shape[0] >= 2 ** 31:
            raise ValueError('matrix too large for 32-bit column indices')
        A.sum_duplicates()
        self.device = _device(device)
        self.n = int(A.shape[0])
        self.indptr = torch.from_numpy(A.indptr.astype(numpy.int64)).to(self.device)
        self.indices = torch.from_numpy(A.indices.astype(numpy.int32)).to(self.device)
        self.data = torch.from_numpy(A.data.astype(numpy.complex128)).to(self.device)
        self.desc = _lib.CsrDesc(self.n, int(A.nnz), self.indptr.data_ptr(), self.indices.data_ptr(),
                                 self.data.data_ptr())
        self.lib = _lib.load()

    def __matmul__(self, x) -> torch.Tensor:
        xt = as_device(x, torch.complex128, self.device, self.n, 'x')
        y = torch.empty_like(xt)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.fdfd_csr_spmv(C.byref(self.desc), xt.data_ptr(), y.data_ptr(), _stream_handle()))
        return y

    def solve(self, b, x0=None, *, rtol: float = 1e-5, atol: float = 0.0, maxiter: int | None = None,
              chunk: int = 0) -> tuple[torch.Tensor, dict]:
        """BiCGSTAB for ``A x = b``; returns the last iterate and ``{status, iterations, residual}``."""
        bt = as_device(b, torch.complex128, self.device, self.n, 'b')
        x = (as_device(x0, torch.complex128, self.device, self.n, 'x0').clone() if x0 is not None
             else torch.zeros_like(bt))
        nbytes = C.c_size_t()
        _lib.check(self.lib.fdfd_csr_solve_workspace_bytes(C.byref(self.desc), C.byref(nbytes)))
        ws = torch.empty(int(nbytes.value) + 256, dtype=torch.uint8, device=self.device)
        off = (-ws.data_ptr()) % 256
        o = _lib.SolveOpts()
        o.method = 2
        o.rtol = float(rtol)
        o.atol = float(atol)
        o.maxiter = int(maxiter) if maxiter is not None else 10 * self.n
        o.has_guess = int(x0 is not None)
        o.chunk = int(chunk)
        info = _lib.SolveInfo()
        with torch.cuda.device(self.device):
            _lib.check(self.lib.fdfd_csr_solve(C.byref(self.desc), C.byref(o), bt.data_ptr(), x.data_ptr(),
                                               ws.data_ptr() + off, nbytes.value, C.byref(info),
                                               _stream_handle()))
        return x, dict(status=_STATUS.get(info.status, str(info.status)), iterations=int(info.iterations),
                       residual=float(info.residual))


def matrix_solver(A, b, **kwargs) -> numpy.ndarray:
    """Drop-in for ``meanas.fdfd.solvers._scipy_qmr(A, b, **kwargs)``: solve on the GPU and
    return x as a numpy array (the last iterate, converged or not).  Accepts scipy's
    ``rtol`` (default 1e-5), ``atol``, ``maxiter``, ``x0`` and ``callback`` (called once,
    with the result); ``device`` picks the GPU."""
    device = kwargs.pop('device', None)
    callback = kwargs.pop('callback', None)
    x0 = kwargs.pop('x0', None)
    opts = {k: kwargs.pop(k) for k in ('rtol', 'atol', 'maxiter') if k in kwargs}
    if kwargs:
        raise TypeError(f'unsupported matrix_solver options: {sorted(kwargs)}')
    M = CsrMatrix(A, device)
    x, info = M.solve(b, x0, **opts)
    if info['status'] != 'converged':
        logger.warning('GPU CSR solve stopped: %s after %d iterations, residual %.3g', info['status'],
                       info['iterations'], info['residual'])
    out = x.cpu().numpy()
    if callback is not None:
        callback(out)
    return out
