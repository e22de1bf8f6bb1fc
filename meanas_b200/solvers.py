"""Drop-in replacement for ``meanas.fdfd.solvers.generic`` running on a B200.

``generic(omega, dxes, J, epsilon, mu=None, *, pec=None, pmc=None, adjoint=False,
matrix_solver=None, matrix_solver_opts=None, E_guess=None)`` has the reference's
signature and meaning (``meanas/fdfd/solvers.py:66-141``): it solves
``A0 E = -i omega J`` with the wave operator of ``meanas/fdfd/operators.py:40-96``
(or ``A0^H E = -i omega J`` with ``adjoint=True``) and returns ``E`` as a 1D
complex128 array.

Differences from the reference, all deliberate:

* The solve runs matrix-free on the GPU (libmeanas_fdfd).  The default method is
  complex128 COCG on the same symmetrised system the reference hands to
  ``scipy.sparse.linalg.qmr``; ``precision='mixed'`` uses complex64 BiCGSTAB
  inner solves refined in complex128.
* ``matrix_solver_opts`` accepts scipy's ``rtol`` (default 1e-5), ``atol``
  (default 0), ``maxiter`` (default 10 * len(J)) and ``x0``, with scipy's
  meaning: by default the stopping test is scipy's, on the symmetrised system.
  ``criterion='true'`` stops on ``||b0 - A0 E|| <= rtol ||b0||`` instead.
  A ``callback`` cannot run per iteration on the device; it is called once with
  the final iterate of the symmetrised system.
* A custom ``matrix_solver`` (which expects an assembled CSR matrix) is not
  supported here and raises ``NotImplementedError``; to keep the reference's CSR flow
  and still solve on the GPU, pass ``meanas_b200.csr.matrix_solver`` to the reference's
  own ``generic()``.
* Non-convergence is not silent: it logs a WARNING, and the outcome of the last
  call is available from :func:`last_solve_info` (or ``return_info=True``).
* Progress is logged as the reference logs it: ``Solver residual at iteration i : r``
  every 100 iterations at INFO on the ``meanas.fdfd.solvers`` logger, after the solve
  (the iterations run on the device; their residuals are recorded only while that
  logger is enabled for INFO).
* The adjoint path works on current SciPy (the reference's ``.H`` on
  ``csr_array`` fails on SciPy >= 1.14).
"""
from __future__ import annotations

import logging
from collections.abc import Callable
from typing import Any

import numpy
import torch

from .operators import GridOperator, SolveInfo, as_device

logger = logging.getLogger(__name__)
# Progress lines go to the reference's own logger name, at its cadence (every 100
# iterations, ``meanas/fdfd/solvers.py:43-48``), so existing logging set-ups keep working.
progress_logger = logging.getLogger('meanas.fdfd.solvers')

_LAST_INFO: SolveInfo | None = None


def last_solve_info() -> SolveInfo | None:
    """Status, iterations and FP64 residual of the most recent :func:`generic` call."""
    return _LAST_INFO


def _pl_host(dxes) -> numpy.ndarray:
    """``Pl`` diagonal (principal sqrt of p^2), as ``e_full_preconditioners`` builds it."""
    (ex, ey, ez), (hx, hy, hz) = [[numpy.asarray(d, dtype=complex) for d in g] for g in dxes]
    p2 = numpy.stack([ex[:, None, None] * hy[None, :, None] * hz[None, None, :],
                      hx[:, None, None] * ey[None, :, None] * hz[None, None, :],
                      hx[:, None, None] * hy[None, :, None] * ez[None, None, :]])
    return numpy.sqrt(p2.ravel())


def generic(
        omega: complex,
        dxes,
        J,
        epsilon,
        mu=None,
        *,
        pec=None,
        pmc=None,
        adjoint: bool = False,
        matrix_solver: Callable[..., Any] | None = None,
        matrix_solver_opts: dict[str, Any] | None = None,
        E_guess=None,
        precision: str = 'fp64',
        criterion: str = 'precond',
        return_info: bool = False,
        device: Any | None = None,
        operator: GridOperator | None = None,
        ):
    """Solve the FDFD wave equation for E (see the module docstring).

    ``J``, ``epsilon``, ``mu``, ``pec``, ``pmc`` and ``E_guess`` are 1D arrays of
    length ``3*X*Y*Z`` (``meanas.fdmath.vec`` layout), numpy or torch.  The result
    is a numpy complex128 array, or a CUDA tensor when ``J`` is a CUDA tensor.
    ``operator`` reuses an existing :class:`GridOperator` for the same problem.
    """
    global _LAST_INFO
    if matrix_solver is not None:
        raise NotImplementedError('meanas_b200.generic runs its own matrix-free GPU solver; a CSR '
                                  'matrix_solver cannot be plugged in (for the CSR flow, pass '
                                  'meanas_b200.csr.matrix_solver to meanas.fdfd.solvers.generic)')
    opts = dict(matrix_solver_opts or {})
    rtol = float(opts.pop('rtol', 1e-5))
    atol = float(opts.pop('atol', 0.0))
    maxiter = opts.pop('maxiter', None)
    x0 = opts.pop('x0', None)
    callback = opts.pop('callback', None)
    if opts:
        raise TypeError(f'unsupported matrix_solver_opts: {sorted(opts)}')
    if precision not in ('fp64', 'mixed', 'bicgstab'):
        raise ValueError(f"precision must be 'fp64', 'mixed' or 'bicgstab', not {precision!r}")

    shape = tuple(int(numpy.size(d)) for d in dxes[0])
    n = 3 * int(numpy.prod(shape))
    for name, arr in (('J', J), ('epsilon', epsilon), ('mu', mu), ('pec', pec), ('pmc', pmc),
                      ('E_guess', E_guess)):
        if arr is not None and int(numpy.prod(tuple(arr.shape))) != n:
            raise ValueError(f'{name} has {int(numpy.prod(tuple(arr.shape)))} elements; the grid needs {n}')

    want_torch = isinstance(J, torch.Tensor) and J.is_cuda
    if E_guess is None and x0 is not None:
        # scipy's x0 lives in the symmetrised space: x0 = Pl E (forward) or Pr^H E (adjoint)
        pl = _pl_host(dxes)
        x0 = numpy.asarray(x0.cpu() if isinstance(x0, torch.Tensor) else x0)
        E_guess = (pl.conj() * x0) if adjoint else (x0 / pl)

    op = operator
    if op is None:
        op = GridOperator(omega, dxes, epsilon, mu, pec, pmc, device=device,
                          fp32=(precision == 'mixed'))
    method = {'fp64': 'cocg', 'mixed': 'mixed', 'bicgstab': 'bicgstab'}[precision]
    # the per-iteration residuals are kept on the device only when someone will read them
    log_progress = progress_logger.isEnabledFor(logging.INFO)
    E, info = op.solve(J, E_guess=E_guess, method=method, rtol=rtol, atol=atol,
                       maxiter=None if maxiter is None else int(maxiter), criterion=criterion,
                       adjoint=adjoint, record_history=log_progress)
    _LAST_INFO = info
    if log_progress and info.history is not None:
        # history[i] is the monitored relative residual after iteration i (the symmetrised
        # system's, as the reference logs, under the default criterion)
        for i in range(100, len(info.history), 100):
            progress_logger.info(f'Solver residual at iteration {i} : {info.history[i]}')
    if info.converged:
        logger.info(f'Solver converged: {info.iterations} iterations, residual {info.residual:.3e}')
    else:
        logger.warning(f'Solver stopped ({info.status}) after {info.iterations} iterations, '
                       f'residual {info.residual:.3e}')
    if callback is not None:
        pl = as_device(_pl_host(dxes), torch.complex128, E.device)
        callback((pl.conj() ** -1 * E if adjoint else pl * E).cpu().numpy())
    out = E if want_torch else E.cpu().numpy()
    if return_info:
        return out, info
    return out
