"""GPU E -> H and Poynting products (``fdfd_e2h``) against the reference's own outputs,
and the reference's energy-balance test (``meanas/test/test_fdfd.py:21-55``) on fields
solved, converted and multiplied on the GPU."""
from __future__ import annotations

import numpy
import pytest

from conftest import golden_cases

pytestmark = pytest.mark.gpu

E2H = golden_cases('e2h')
SOLVES = golden_cases('solve')


def _rel(a, b) -> float:
    return float(numpy.linalg.norm(a - b) / numpy.linalg.norm(b))


@pytest.mark.parametrize('c', E2H, ids=lambda c: f"e2h{c['index']}-{tuple(int(s) for s in c['shape'])}")
def test_e2h_and_poynting_match_reference(cuda, c):
    from meanas_b200 import fields
    from meanas_b200.operators import GridOperator
    om, mu, pmc = complex(c['omega']), c.get('mu'), c.get('pmc')
    shape = tuple(int(s) for s in c['shape'])
    # operators.e2h(omega, dxes, mu, pmc) @ x
    H = fields.e2h(om, c['dxes'], mu, pmc, device=cuda) @ c['x']
    assert isinstance(H, numpy.ndarray)
    assert _rel(H, c['H']) <= 1e-13
    # one pass over E: H and E x conj(H)
    grid = GridOperator(om, c['dxes'], numpy.ones(c['x'].size), mu, None, pmc, device=cuda, fp32=False)
    S, H2 = grid.poynting(c['x'])
    assert _rel(H2.cpu().numpy(), c['H']) <= 1e-13
    assert _rel(S.cpu().numpy(), c['S_op']) <= 1e-13
    # the reference's two forms with a given H: operators.poynting_e_cross(x) @ conj(H) and
    # functional.poynting_e_cross_h(dxes)(x, conj(H)) on (3, X, Y, Z) fields
    S_op = fields.poynting_e_cross(c['x'], c['dxes'], device=cuda) @ c['H'].conj()
    assert _rel(S_op, c['S_op']) <= 1e-13
    exh = fields.poynting_e_cross_h(c['dxes'], device=cuda)
    S_fn = exh(c['x'].reshape(3, *shape), c['H'].conj().reshape(3, *shape))
    assert S_fn.shape == (3, *shape)
    assert _rel(S_fn.ravel(), c['S_fn']) <= 1e-13


def test_pmc_cells_have_zero_h_and_device_tensors_stay_on_device(cuda):
    import torch
    from meanas_b200 import fields
    c = next(c for c in E2H if 'pmc' in c)
    x = torch.as_tensor(c['x'], device=cuda)
    H = fields.e2h(complex(c['omega']), c['dxes'], c.get('mu'), c['pmc'], device=cuda) @ x
    assert isinstance(H, torch.Tensor) and H.is_cuda
    assert torch.count_nonzero(H[torch.as_tensor(c['pmc'] != 0, device=cuda)]) == 0


@pytest.mark.parametrize('c', [c for c in SOLVES if c['tag'] == 'test_fdfd'],
                         ids=lambda c: f"s{c['index']}-{tuple(int(s) for s in c['shape'])}")
def test_poynting_planes_like_reference_test(cuda, c):
    """meanas/test/test_fdfd.py:21-55: the Poynting flux through the six faces around the
    second source point equals the power that point delivers (rtol 1e-6), here with E from
    the GPU solve and H, E x conj(H) from the GPU kernel."""
    from meanas_b200 import generic
    from meanas_b200.operators import GridOperator
    shape = tuple(int(s) for s in c['shape'])
    om = complex(c['omega'])
    E = generic(omega=om, dxes=c['dxes'], J=c['J'], epsilon=c['eps'],
                matrix_solver_opts=dict(atol=1e-15, rtol=1e-11), device=cuda)
    J = c['J'].reshape(3, *shape)
    mask = (J != 0).any(axis=0)
    assert mask.sum() == 2
    points = numpy.where(mask)
    mask[points[0][0], points[1][0], points[2][0]] = 0
    mx, my, mz = (numpy.roll(mask, -1, axis=a) for a in range(3))
    grid = GridOperator(om, c['dxes'], c['eps'], device=cuda, fp32=False)
    S, _ = grid.poynting(E)
    s = (S.real / 2).cpu().numpy().reshape(3, *shape)
    planes = [s[0, mask].sum(), -s[0, mx].sum(), s[1, mask].sum(), -s[1, my].sum(),
              s[2, mask].sum(), -s[2, mz].sum()]
    e = E.reshape(3, *shape)
    dv = (c['dxes'][0][0][:, None, None] * c['dxes'][0][1][None, :, None] * c['dxes'][0][2][None, None, :])
    src_energy = -((e * J.conj()).real * dv)[:, mask] / 2
    numpy.testing.assert_allclose(sum(planes), src_energy.sum(), rtol=1e-6)


SOURCES = golden_cases('sources')


@pytest.mark.parametrize('c', SOURCES, ids=lambda c: f"src{c['index']}-{tuple(int(s) for s in c['shape'])}")
def test_tfsf_and_boundary_sources_match_reference(cuda, c):
    from meanas_b200 import fields
    om, mu = complex(c['omega']), c.get('mu')
    args = (c['q'], om, c['dxes'], c['eps'], mu)
    J = fields.e_tfsf_source(*args, device=cuda) @ c['x']
    assert _rel(J, c['tfsf']) <= 1e-13
    for periodic, key in ((False, 'edge_mirror'), (True, 'edge_periodic')):
        Jb = fields.e_boundary_source(*args, periodic_mask_edges=periodic, device=cuda) @ c['x']
        assert _rel(Jb, c[key]) <= 1e-13
        # the edge mask is exact: the same cells are zero
        assert numpy.array_equal(Jb == 0, c[key] == 0)


def test_source_operator_refuses_masked_plans(cuda):
    from meanas_b200 import _lib
    from meanas_b200.operators import GridOperator
    c = SOURCES[0]
    grid = GridOperator(complex(c['omega']), c['dxes'], c['eps'], pec=numpy.zeros_like(c['eps']), device=cuda)
    with pytest.raises(_lib.FDFDError, match='no PEC/PMC'):
        grid.tfsf_source(c['x'], c['q'])
