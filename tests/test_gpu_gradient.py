"""GPU adjoint gradient (torch.autograd) against central finite differences of GPU
solves and against the oracle's direct-solve adjoint gradient."""
from __future__ import annotations

import numpy
import pytest

pytestmark = pytest.mark.gpu


def _problem():
    from meanas_b200 import workloads
    return workloads.adjoint_design(shape=(24, 20, 16), pml=4, wavelength=9.0, design=(8, 8, 4),
                                    source_x=6, monitor_x=18)


def test_autograd_gradient_matches_fd_and_oracle(cuda):
    import torch
    from meanas_b200.autograd import fdfd_solve
    from oracle import fdfd_oracle as O
    p = _problem()
    mon = torch.as_tensor(p.extra['monitor'], device=cuda)
    eps = torch.as_tensor(p.epsilon, device=cuda).requires_grad_(True)

    def loss(e):
        E = fdfd_solve(e, p.J, p.omega, p.dxes, rtol=1e-12)
        return (E.abs() ** 2)[mon].sum()
    L = loss(eps)
    L.backward()
    g = eps.grad.cpu().numpy()
    # oracle: CPU COCG solves (rtol 1e-12), adjoint through the W-symmetry
    W = O.precond_p2(p.dxes).ravel()
    E, _, st = O.cocg(p.omega, p.dxes, p.epsilon, -1j * p.omega * p.J, rtol=1e-12)
    assert st == 0
    y, _, st = O.cocg(p.omega, p.dxes, p.epsilon, numpy.conj(2 * E * p.extra['monitor']) / W, rtol=1e-12)
    assert st == 0
    g_ref = numpy.real(p.omega ** 2 * (W * y) * E)
    design = numpy.flatnonzero(numpy.tile(p.extra['design_mask'].ravel(), 3))
    err = numpy.linalg.norm(g[design] - g_ref[design]) / numpy.linalg.norm(g_ref[design])
    assert err < 1e-6, err
    # central finite differences with GPU FP64 solves (per cell: all three components move)
    rng = numpy.random.default_rng(1)
    cells = numpy.flatnonzero(p.extra['design_mask'].ravel())
    n = p.n_cells
    h = 1e-4
    with torch.no_grad():
        for cell in rng.choice(cells, 6, replace=False):
            idx = [cell, n + cell, 2 * n + cell]
            ep = eps.detach().clone()
            em = eps.detach().clone()
            ep[idx] += h
            em[idx] -= h
            fd = (loss(ep) - loss(em)).item() / (2 * h)
            ad = float(g[idx].sum())
            assert abs(fd - ad) <= 1e-5 * abs(fd) + 1e-9 * L.item(), (cell, fd, ad)


GRAD48 = __import__('conftest').GOLDEN / 'grad48.npz'


@pytest.mark.skipif(not GRAD48.exists(), reason='tests/golden/grad48.npz not generated')
def test_autograd_gradient_matches_reference_adjoint_at_48(cuda):
    """The design problem scaled to 48x48x40 (tests/golden/make_golden.py GRAD48): dL/deps
    from torch.autograd (GPU forward + adjoint solves) against the reference's own gradient,
    formed from its generic() and generic(adjoint=True) QMR solves, over the whole design
    region."""
    import torch
    from meanas_b200 import workloads
    from meanas_b200.autograd import fdfd_solve
    z = numpy.load(GRAD48)
    p = workloads.adjoint_design(shape=(48, 48, 40), pml=8, wavelength=26.0, design=(16, 16, 6),
                                 source_x=12, monitor_x=36)
    dsl = p.extra['design_slices']
    assert numpy.array_equal(z['eps_design'], p.epsilon.reshape(3, *p.shape)[(slice(None), *dsl)])
    mon = torch.as_tensor(p.extra['monitor'], device=cuda)
    eps = torch.as_tensor(p.epsilon, device=cuda).requires_grad_(True)
    E = fdfd_solve(eps, p.J, p.omega, p.dxes, rtol=1e-12)
    L = (E.abs() ** 2)[mon].sum()
    L.backward()
    g = eps.grad.cpu().numpy().reshape(3, *p.shape)[(slice(None), *dsl)]
    ref = z['grad_design']
    tol = max(1e-6, 100 * float(z['rtol']))   # the reference's QMR tolerance bounds its accuracy
    assert abs(L.item() - float(z['loss'])) <= tol * float(z['loss'])
    assert numpy.linalg.norm(g - ref) <= tol * numpy.linalg.norm(ref)
