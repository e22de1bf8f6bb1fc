"""Differentiable FDFD solve: ``E = fdfd_solve(epsilon, ...)`` with ``dL/d(epsilon)``.

``FDFDSolve`` is a ``torch.autograd.Function``: the forward pass solves
``A0(eps) E = -i omega J`` (the system of ``meanas/fdfd/solvers.py:66-141``) on
the GPU; the backward pass runs one adjoint solve with the same kernels and plan.

Derivation.  ``A0 = pe (ch pm mu^-1 ce - omega^2 diag(eps)) pe``
(``meanas/fdfd/operators.py:95``), so ``dA0/deps_i = -omega^2 pe_i e_i e_i^T``
and ``dE/deps_i = A0^-1 omega^2 pe_i E_i e_i``.  With torch's complex gradient
``G = dL/dE`` (``G = 2 dL/dE*`` for real ``L``), ``dL = Re(sum conj(G) dE)``, so
``dL/deps_i = Re(omega^2 lambda_i E_i) pe_i`` with ``A0^T lambda = conj(G)``.
``A0^T lambda = conj(G)`` is ``A0^H conj(lambda) = G``: the reference's adjoint
solve ``generic(adjoint=True)`` with ``-i omega J_adj = G``.  The library solves it
with the forward kernels (``W A0`` is complex symmetric) and
``fdfd_eps_gradient`` forms ``Re(omega^2 conj(E_adj) E)``.
"""
from __future__ import annotations

from typing import Any

import torch

from .operators import GridOperator


class FDFDSolve(torch.autograd.Function):
    """``E = A0(epsilon)^-1 (-i omega J)``; differentiable with respect to ``epsilon``."""

    @staticmethod
    def forward(ctx, epsilon: torch.Tensor, J: torch.Tensor, omega: complex, dxes, mu, pec, pmc,
                solve_kw: dict[str, Any]):
        op = GridOperator(omega, dxes, epsilon.detach(), mu, pec, pmc, device=epsilon.device,
                          fp32=(solve_kw.get('method') == 'mixed'))
        E, info = op.solve(J, **solve_kw)
        if not info.converged:
            raise RuntimeError(f'forward FDFD solve did not converge: {info}')
        ctx.op = op
        ctx.omega = complex(omega)
        ctx.solve_kw = solve_kw
        ctx.save_for_backward(E)
        ctx.info = info
        return E

    @staticmethod
    def backward(ctx, grad_E: torch.Tensor):
        (E,) = ctx.saved_tensors
        op: GridOperator = ctx.op
        omega = ctx.omega
        kw = dict(ctx.solve_kw)
        kw['adjoint'] = True
        # -i omega J_adj = grad_E
        J_adj = grad_E.to(torch.complex128) * (1j / omega)
        E_adj, info = op.solve(J_adj, **kw)
        if not info.converged:
            raise RuntimeError(f'adjoint FDFD solve did not converge: {info}')
        g_eps = op.eps_gradient(E, E_adj)
        return g_eps, None, None, None, None, None, None, None


def fdfd_solve(epsilon: torch.Tensor, J, omega: complex, dxes, mu=None, pec=None, pmc=None, *,
               method: str = 'cocg', rtol: float = 1e-10, criterion: str = 'true',
               maxiter: int | None = None) -> torch.Tensor:
    """Differentiable solve.  ``epsilon``: real float64 CUDA tensor (3N, requires_grad for
    gradients); ``J``: complex (3N).  Returns ``E`` (complex128 CUDA tensor)."""
    if not isinstance(J, torch.Tensor):
        J = torch.as_tensor(J)
    J = J.to(device=epsilon.device, dtype=torch.complex128)
    kw = dict(method=method, rtol=rtol, criterion=criterion, maxiter=maxiter)
    return FDFDSolve.apply(epsilon, J, omega, dxes, mu, pec, pmc, kw)
