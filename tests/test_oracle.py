"""The CPU oracle and the host-side SC-PML builder against the reference's own outputs."""
from __future__ import annotations

import numpy
import pytest

from conftest import golden_cases
from oracle import fdfd_oracle as O
from meanas_b200 import scpml

OPS = golden_cases('operator')
SOLVES = golden_cases('solve')
E2H = golden_cases('e2h')
SOURCES = golden_cases('sources')


def _opt(c, k):
    return c.get(k)


@pytest.mark.parametrize('c', OPS, ids=lambda c: f"op{c['index']}-{tuple(c['shape'])}")
def test_oracle_apply_matches_reference(c):
    om = complex(c['omega'])
    y = O.e_full_apply(om, c['dxes'], c['eps'], c['x'], _opt(c, 'mu'), _opt(c, 'pec'), _opt(c, 'pmc'))
    ref = c['A0x']
    assert numpy.linalg.norm(y - ref) <= 1e-14 * numpy.linalg.norm(ref)


@pytest.mark.parametrize('c', E2H, ids=lambda c: f"e2h{c['index']}-{tuple(c['shape'])}")
def test_oracle_e2h_and_poynting_match_reference(c):
    H = O.e2h(complex(c['omega']), c['dxes'], c['x'], _opt(c, 'mu'), _opt(c, 'pmc'))
    assert numpy.linalg.norm(H - c['H']) <= 1e-14 * numpy.linalg.norm(c['H'])
    S = O.poynting_e_cross_h(c['dxes'], c['x'], c['H'].conj())
    # the operator and the functional forms of the reference agree with each other
    for ref in (c['S_op'], c['S_fn']):
        assert numpy.linalg.norm(S - ref) <= 1e-14 * numpy.linalg.norm(ref)


@pytest.mark.parametrize('c', SOURCES, ids=lambda c: f"src{c['index']}-{tuple(c['shape'])}")
def test_oracle_sources_match_reference(c):
    args = (complex(c['omega']), c['dxes'], c['eps'], c['x'], c['q'], _opt(c, 'mu'))
    for kw, key in ((dict(), 'tfsf'), (dict(edges=True), 'edge_mirror'),
                    (dict(edges=True, periodic=True), 'edge_periodic')):
        j = O.tfsf_source(*args, **kw)
        assert numpy.linalg.norm(j - c[key]) <= 1e-14 * numpy.linalg.norm(c[key])
        assert numpy.array_equal(j == 0, c[key] == 0)


@pytest.mark.parametrize('c', OPS, ids=lambda c: f"op{c['index']}")
def test_oracle_csr_and_preconditioners_match_reference(c):
    om = complex(c['omega'])
    A = O.e_full_csr(om, c['dxes'], c['eps'], _opt(c, 'mu'), _opt(c, 'pec'), _opt(c, 'pmc'))
    assert numpy.linalg.norm(A @ c['x'] - c['A0x']) <= 1e-14 * numpy.linalg.norm(c['A0x'])
    pl = O.precond_pl(c['dxes'])
    assert numpy.array_equal(pl, c['pl'])
    S = (pl[:, None] * A.toarray()) / pl[None, :]
    assert numpy.linalg.norm(S @ c['x'] - c['Sx']) <= 1e-13 * numpy.linalg.norm(c['Sx'])
    assert numpy.linalg.norm(S.conj().T @ c['x'] - c['SHx']) <= 1e-13 * numpy.linalg.norm(c['SHx'])
    # the symmetrised operator is complex symmetric
    assert numpy.linalg.norm(S - S.T) <= 1e-13 * numpy.linalg.norm(S)


@pytest.mark.parametrize('c', [c for c in SOLVES if c['shape'].prod() <= 1000],
                         ids=lambda c: f"s{c['index']}-{c['tag']}")
def test_reference_solutions_pin_the_oracle_residual(c):
    """The oracle's residual of the reference's own solutions is tiny (pins operator + b0)."""
    om = complex(c['omega'])
    E, J = c['E'], c['J']
    if bool(c['adjoint']):
        A = O.e_full_csr(om, c['dxes'], c['eps'], _opt(c, 'mu'), _opt(c, 'pec'), _opt(c, 'pmc'))
        r = A.conj().T @ E + 1j * om * J
        rel = numpy.linalg.norm(r) / numpy.linalg.norm(om * J)
    else:
        rel = O.true_residual(om, c['dxes'], c['eps'], E, J, _opt(c, 'mu'), _opt(c, 'pec'), _opt(c, 'pmc'))
    assert rel < 1e-6


@pytest.mark.parametrize('c', [c for c in SOLVES if c['tag'] == 'test_fdfd'][:12],
                         ids=lambda c: f"s{c['index']}")
def test_oracle_cocg_detects_breakdown_of_paired_source(c):
    """The reference fixture's source (1+1j, 1-1j) gives r^T W r = 0 at the start:
    COCG must report breakdown there instead of dividing by rounding noise."""
    om = complex(c['omega'])
    b0 = -1j * om * c['J']
    E, it, st = O.cocg(om, c['dxes'], c['eps'], b0, rtol=1e-12)
    assert (st, it) == (2, 0)


@pytest.mark.parametrize('c', [c for c in SOLVES if c['tag'] in ('pml3d', 'test_pml') and not c['adjoint']],
                         ids=lambda c: f"s{c['index']}")
def test_oracle_cocg_matches_reference_solution(c):
    om = complex(c['omega'])
    b0 = -1j * om * c['J']
    E, it, st = O.cocg(om, c['dxes'], c['eps'], b0, _opt(c, 'mu'), _opt(c, 'pec'), _opt(c, 'pmc'), rtol=1e-12)
    assert st == 0
    ref = c['E']
    # the reference fields are themselves solved to scipy rtol 1e-11/1e-12; the 1D PML
    # cases are ill-conditioned enough that this bounds the agreement to ~1e-7
    tol = 1e-6 if c['tag'] == 'test_pml' else 1e-8
    assert numpy.linalg.norm(E - ref) <= tol * numpy.linalg.norm(ref)


@pytest.mark.parametrize('c', [c for c in SOLVES if c['tag'] == 'pml3d' and not c['adjoint']],
                         ids=lambda c: f"s{c['index']}")
def test_oracle_qmr_port_matches_reference_generic(c):
    om = complex(c['omega'])
    E, info = O.generic_qmr(om, c['dxes'], c['J'], c['eps'], _opt(c, 'mu'), pec=_opt(c, 'pec'),
                            pmc=_opt(c, 'pmc'), rtol=1e-12)
    ref = c['E']
    assert numpy.linalg.norm(E - ref) <= 1e-8 * numpy.linalg.norm(ref)


@pytest.mark.parametrize('c', [c for c in SOLVES if c['tag'] == 'pml3d' and c['adjoint']],
                         ids=lambda c: f"s{c['index']}")
def test_oracle_qmr_port_adjoint_matches_reference_generic(c):
    om = complex(c['omega'])
    E, info = O.generic_qmr(om, c['dxes'], c['J'], c['eps'], _opt(c, 'mu'), pec=_opt(c, 'pec'),
                            pmc=_opt(c, 'pmc'), rtol=1e-12, adjoint=True)
    ref = c['E']
    assert numpy.linalg.norm(E - ref) <= 1e-8 * numpy.linalg.norm(ref)


def test_scpml_matches_reference():
    z = numpy.load('tests/golden/scpml.npz') if False else None
    from conftest import GOLDEN, unpack_dxes
    z = numpy.load(GOLDEN / 'scpml.npz')
    for n in range(int(z['n'])):
        om, th, eff, lnr, m = z[f'c{n}_params']
        shape = tuple(int(s) for s in z[f'c{n}_shape'])
        th = int(th)
        dxes = [[numpy.ones(s) for s in shape] for _ in range(2)]
        sf = scpml.prepare_s_function(ln_R=lnr, m=m)
        for ax in range(3):
            if shape[ax] <= 2 * th:
                continue
            for pol in (-1, 1):
                dxes = scpml.stretch_with_scpml(dxes, axis=ax, polarity=pol, omega=om,
                                                epsilon_effective=eff, thickness=th, s_function=sf)
        ref = unpack_dxes(z, f'c{n}_')
        for g in range(2):
            for a in range(3):
                assert numpy.array_equal(numpy.asarray(dxes[g][a], dtype=complex), ref[g][a])
        u = scpml.uniform_grid_scpml(shape, list(z[f'c{n}_uth']), om, eff)
        refu = unpack_dxes(z, f'c{n}_u')
        for g in range(2):
            for a in range(3):
                assert numpy.array_equal(numpy.asarray(u[g][a], dtype=complex), refu[g][a])


def test_pml_fixture_assertions_hold_for_reference_solutions():
    """meanas/test/test_fdfd_pml.py:14-28 on the stored reference fields."""
    for c in [c for c in SOLVES if c['tag'] == 'test_pml']:
        e = c['E'].reshape(3, *c['shape'])
        e_sqr = numpy.squeeze((e.conj() * e).sum(axis=0))
        tgt, rev = e_sqr[16:19], e_sqr[10:13]
        if int(c['src_polarity']) < 0:
            tgt, rev = rev, tgt
        numpy.testing.assert_allclose(rev, 0, atol=1e-12)
        numpy.testing.assert_allclose(tgt, 1, rtol=3e-6)


MODESRC = golden_cases('modesrc')


def _slices(c):
    big = 10 ** 9
    return [slice(None if lo == -big else int(lo), None if hi == big else int(hi)) for lo, hi in c['slices']]


@pytest.mark.parametrize('c', MODESRC, ids=lambda c: f"mode{c['index']}-{tuple(int(s) for s in c['shape'])}")
def test_oracle_mode_source_matches_reference(c):
    args = (c['E'], complex(c['k']))
    axis, pol = int(c['axis']), int(c['polarity'])
    Ee = O.expand_e(*args, c['dxes'], axis, pol, _slices(c))
    assert numpy.linalg.norm(Ee - c['E_expanded']) <= 1e-14 * numpy.linalg.norm(c['E_expanded'])
    J = O.mode_source(*args, complex(c['omega']), c['dxes'], axis, pol, _slices(c), c['eps'], c.get('mu'))
    assert numpy.linalg.norm(J - c['J']) <= 1e-13 * numpy.linalg.norm(c['J'])
    assert numpy.array_equal(J == 0, c['J'] == 0)
