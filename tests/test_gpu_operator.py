"""GPU operator parity: libmeanas_fdfd's matrix-free products against the reference's
sparse operators (golden vectors) and size-independent identities at full size."""
from __future__ import annotations

import numpy
import pytest

from conftest import golden_cases

pytestmark = pytest.mark.gpu

OPS = golden_cases('operator')


def _op(c, cuda, fp32=True):
    from meanas_b200.operators import GridOperator
    return GridOperator(complex(c['omega']), c['dxes'], c['eps'], c.get('mu'), c.get('pec'), c.get('pmc'),
                        device=cuda, fp32=fp32)


@pytest.mark.parametrize('c', OPS, ids=lambda c: f"op{c['index']}-{tuple(int(s) for s in c['shape'])}")
@pytest.mark.parametrize('which', ['A0', 'sym', 'sym_h'])
def test_apply_c128_matches_reference(cuda, c, which):
    op = _op(c, cuda)
    ref = {'A0': c['A0x'], 'sym': c['Sx'], 'sym_h': c['SHx']}[which]
    y = op.apply(c['x'], op=which, precision='c128').cpu().numpy()
    # complex128: within 1e-13 of the norm (summation order differs from the CSR product)
    assert numpy.linalg.norm(y - ref) <= 1e-13 * numpy.linalg.norm(ref)


@pytest.mark.parametrize('c', OPS, ids=lambda c: f"op{c['index']}")
def test_apply_c64_matches_reference(cuda, c):
    op = _op(c, cuda)
    y = op.apply(c['x'], op='A0', precision='c64').cpu().numpy()
    ref = c['A0x']
    # complex64: within 2e-6 of the norm
    assert numpy.linalg.norm(y - ref) <= 2e-6 * numpy.linalg.norm(ref)


def test_masks_are_exact(cuda):
    """E components on PEC cells come out exactly zero (pe applied on both sides)."""
    c = [c for c in OPS if 'pec' in c][0]
    op = _op(c, cuda)
    y = op.apply(c['x'], op='A0').cpu().numpy()
    assert numpy.all(y[c['pec'] != 0] == 0)


@pytest.mark.parametrize('shape', [(160, 160, 128), (96, 96, 64), (130, 70, 45), (512, 512, 1)])
def test_full_size_identities(cuda, shape):
    """Linearity and W-symmetry (x^T W A0 y = y^T W A0 x) at benchmark sizes."""
    import torch
    from meanas_b200 import workloads
    from meanas_b200.operators import GridOperator
    p = workloads.aniso_blocks(shape=shape, pml=10) if shape[2] > 1 else workloads.serving_request(
        numpy.random.default_rng(0), shape=shape)
    op = GridOperator(p.omega, p.dxes, p.epsilon, device=cuda)
    g = torch.Generator(device=cuda).manual_seed(0)
    n = p.n_unknowns
    x = torch.randn(n, dtype=torch.complex128, device=cuda, generator=g)
    y = torch.randn(n, dtype=torch.complex128, device=cuda, generator=g)
    a, b = 0.3 - 1.1j, -2.0 + 0.5j
    lhs = op.apply(a * x + b * y)
    rhs = a * op.apply(x) + b * op.apply(y)
    assert (torch.linalg.vector_norm(lhs - rhs) / torch.linalg.vector_norm(rhs)).item() < 1e-14
    (ex, ey, ez), (hx, hy, hz) = [[torch.as_tensor(numpy.asarray(d, dtype=complex), device=cuda) for d in gg]
                                  for gg in p.dxes]
    W = torch.stack([ex[:, None, None] * hy[None, :, None] * hz[None, None, :],
                     hx[:, None, None] * ey[None, :, None] * hz[None, None, :],
                     hx[:, None, None] * hy[None, :, None] * ez[None, None, :]]).reshape(-1)
    s1 = torch.sum(x * W * op.apply(y))
    s2 = torch.sum(y * W * op.apply(x))
    scale = torch.sum(torch.abs(x * W * op.apply(y)))
    assert (torch.abs(s1 - s2) / scale).item() < 1e-13
    # sym form is complex symmetric: x^T S y = y^T S x
    t1 = torch.sum(x * op.apply(y, op='sym'))
    t2 = torch.sum(y * op.apply(x, op='sym'))
    assert (torch.abs(t1 - t2) / torch.sum(torch.abs(x * op.apply(y, op='sym')))).item() < 1e-13


def test_full_size_matches_oracle_stencil(cuda):
    """The 160x160x128 anisotropic problem: GPU A0 x against the oracle's numpy stencil."""
    import torch
    from meanas_b200 import workloads
    from meanas_b200.operators import GridOperator
    from oracle import fdfd_oracle as O
    p = workloads.aniso_blocks()
    rng = numpy.random.default_rng(3)
    x = rng.standard_normal(p.n_unknowns) + 1j * rng.standard_normal(p.n_unknowns)
    op = GridOperator(p.omega, p.dxes, p.epsilon, device=cuda)
    y = op.apply(x).cpu().numpy()
    ref = O.e_full_apply(p.omega, p.dxes, p.epsilon, x)
    assert numpy.linalg.norm(y - ref) <= 1e-13 * numpy.linalg.norm(ref)
    y32 = op.apply(x, precision='c64').cpu().numpy()
    assert numpy.linalg.norm(y32 - ref) <= 2e-6 * numpy.linalg.norm(ref)
    del torch
