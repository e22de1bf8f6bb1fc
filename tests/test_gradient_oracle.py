"""The adjoint-gradient algebra on the CPU with exact (direct) sparse solves:
dL/deps from one adjoint solve equals central finite differences, and the adjoint
solve through the W-symmetry equals the reference's conjugate-transpose solve."""
from __future__ import annotations

import numpy
import scipy.sparse.linalg as sla

from meanas_b200 import workloads
from oracle import fdfd_oracle as O


def _problem():
    return workloads.adjoint_design(shape=(10, 9, 8), pml=3, wavelength=7.0, design=(4, 4, 2),
                                    source_x=3, monitor_x=6)


def _factor(p, eps):
    A = O.e_full_csr(p.omega, p.dxes, eps).tocsc()
    return A, sla.splu(A, permc_spec='MMD_AT_PLUS_A')


def _loss(p, eps):
    _, lu = _factor(p, eps)
    E = lu.solve(-1j * p.omega * p.J)
    return float(numpy.sum(numpy.abs(E[p.extra['monitor']]) ** 2))


def test_adjoint_gradient_matches_finite_differences():
    p = _problem()
    A, lu = _factor(p, p.epsilon)
    E = lu.solve(-1j * p.omega * p.J)
    mon = p.extra['monitor']
    L0 = float(numpy.sum(numpy.abs(E[mon]) ** 2))
    G = 2 * E * mon                            # torch's dL/dE for L = sum |E|^2
    # A0^T lambda = conj(G)  <=>  A0^H conj(lambda) = G (the reference's adjoint solve)
    lam = lu.solve(numpy.conj(G), trans='T')
    grad = numpy.real(p.omega ** 2 * lam * E)
    # the same lambda through the symmetriser: A0 y = W^-1 conj(G), lambda = W y
    W = O.precond_p2(p.dxes).ravel()
    y = lu.solve(numpy.conj(G) / W)
    assert numpy.allclose(W * y, lam, rtol=1e-9, atol=1e-12 * numpy.abs(lam).max())
    rng = numpy.random.default_rng(0)
    design = numpy.flatnonzero(numpy.tile(p.extra['design_mask'].ravel(), 3))
    h = 1e-4
    for idx in rng.choice(design, 5, replace=False):
        ep = p.epsilon.copy()
        em = p.epsilon.copy()
        ep[idx] += h
        em[idx] -= h
        fd = (_loss(p, ep) - _loss(p, em)) / (2 * h)
        assert abs(fd - grad[idx]) <= 1e-5 * abs(fd) + 1e-12 * L0, (idx, fd, grad[idx])
