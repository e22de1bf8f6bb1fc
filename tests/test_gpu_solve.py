"""GPU solver parity: meanas_b200.generic against the reference generic() outputs
(golden vectors), the reference tests' own assertions, and failure statuses."""
from __future__ import annotations

import numpy
import pytest

from conftest import golden_cases

pytestmark = pytest.mark.gpu

SOLVES = golden_cases('solve')


def _args(c):
    return dict(omega=complex(c['omega']), dxes=c['dxes'], J=c['J'], epsilon=c['eps'], mu=c.get('mu'),
                pec=c.get('pec'), pmc=c.get('pmc'))


@pytest.mark.parametrize('c', [c for c in SOLVES if c['tag'] == 'test_fdfd'],
                         ids=lambda c: f"s{c['index']}-{tuple(int(s) for s in c['shape'])}")
def test_residual_like_reference_test(cuda, c):
    """meanas/test/test_fdfd.py:14-18 with the same solver options (rtol 1e-11, atol 1e-15)."""
    from meanas_b200 import generic
    from oracle import fdfd_oracle as O
    E, info = generic(**_args(c), matrix_solver_opts=dict(atol=1e-15, rtol=1e-11), return_info=True, device=cuda)
    om = complex(c['omega'])
    r = O.e_full_apply(om, c['dxes'], c['eps'], E) - (-1j * om * c['J'])
    assert numpy.linalg.norm(r) < 1e-10
    ref = c['E']
    assert numpy.linalg.norm(E - ref) <= 1e-6 * numpy.linalg.norm(ref)


@pytest.mark.parametrize('c', [c for c in SOLVES if c['tag'] == 'test_pml'], ids=lambda c: f"s{c['index']}")
def test_pml_like_reference_test(cuda, c):
    """meanas/test/test_fdfd_pml.py:14-28 on our solution."""
    from meanas_b200 import generic
    E = generic(**_args(c), matrix_solver_opts={'atol': 1e-15, 'rtol': 1e-11}, device=cuda)
    e = E.reshape(3, *c['shape'])
    e_sqr = numpy.squeeze((e.conj() * e).sum(axis=0))
    tgt, rev = e_sqr[16:19], e_sqr[10:13]
    if int(c['src_polarity']) < 0:
        tgt, rev = rev, tgt
    numpy.testing.assert_allclose(rev, 0, atol=1e-12)
    numpy.testing.assert_allclose(tgt, 1, rtol=3e-6)
    assert numpy.linalg.norm(E - c['E']) <= 1e-6 * numpy.linalg.norm(c['E'])


@pytest.mark.parametrize('precision', ['fp64', 'mixed', 'bicgstab'])
@pytest.mark.parametrize('c', [c for c in SOLVES if c['tag'] == 'pml3d'],
                         ids=lambda c: f"s{c['index']}-{'adj' if c['adjoint'] else 'fwd'}")
def test_pml3d_matches_reference(cuda, c, precision):
    """3D PML problems with mu/PEC/PMC, forward and adjoint (reference generic, rtol 1e-12)."""
    from meanas_b200 import generic
    if precision == 'bicgstab' and bool(c['adjoint']):
        pytest.skip('complex128 BiCGSTAB method supports the forward true-residual criterion')
    E, info = generic(**_args(c), adjoint=bool(c['adjoint']), precision=precision, criterion='true',
                      matrix_solver_opts=dict(rtol=1e-11), return_info=True, device=cuda)
    assert info.converged, info
    assert info.residual <= 1e-11 * 1.01
    ref = c['E']
    assert numpy.linalg.norm(E - ref) <= 1e-7 * numpy.linalg.norm(ref)


def test_dipole48_matches_reference_field(cuda):
    """The 48^3 dipole-in-core problem against the stored reference scipy-QMR field."""
    from meanas_b200 import workloads
    from meanas_b200.operators import GridOperator
    from conftest import GOLDEN
    z = numpy.load(GOLDEN / 'dipole48.npz')
    p = workloads.dipole_core(48)
    op = GridOperator(p.omega, p.dxes, p.epsilon, device=cuda)
    for method in ('cocg', 'mixed'):
        E, info = op.solve(p.J, method=method, rtol=1e-8, criterion='true')
        assert info.converged and info.residual <= 1e-8
        E = E.cpu().numpy()
        ref = z['E'].astype(complex)
        # both fields are solved to 1e-8 residual: they agree to ~cond x 1e-8
        assert numpy.linalg.norm(E - ref) <= 1e-5 * numpy.linalg.norm(ref), method


@pytest.mark.parametrize('method', ['cocg', 'mixed'])
def test_reported_residual_agrees_with_host_oracle_at_96(cuda, method):
    """The solver's FP64 true residual, on the 96x96x64 design problem (1.77M unknowns),
    equals ||b0 - A0 E|| / ||b0|| formed on the host with the reference's CSR operator
    (oracle port of meanas/fdfd/operators.py:40-96), and both meet rtol."""
    from meanas_b200 import workloads
    from meanas_b200.operators import GridOperator
    from oracle import fdfd_oracle as O
    p = workloads.adjoint_design()
    op = GridOperator(p.omega, p.dxes, p.epsilon, device=cuda)
    E, info = op.solve(p.J, method=method, rtol=1e-8, criterion='true')
    assert info.converged, info
    A0 = O.e_full_csr(p.omega, p.dxes, p.epsilon)
    b0 = -1j * p.omega * p.J
    host = numpy.linalg.norm(A0 @ E.cpu().numpy() - b0) / numpy.linalg.norm(b0)
    assert abs(host - info.residual) <= 1e-3 * host, (host, info.residual)
    assert host <= 1e-8 and info.residual <= 1e-8


def test_warm_start_and_history(cuda):
    from meanas_b200 import workloads
    from meanas_b200.operators import GridOperator
    p = workloads.dipole_core(32, pml=8)
    op = GridOperator(p.omega, p.dxes, p.epsilon, device=cuda)
    E1, i1 = op.solve(p.J, rtol=1e-6, criterion='true', record_history=True)
    assert i1.converged and i1.history is not None and len(i1.history) == i1.iterations + 1
    assert i1.history[-1] <= 1e-6
    E2, i2 = op.solve(p.J, rtol=1e-9, criterion='true', E_guess=E1)
    assert i2.converged and i2.residual <= 1e-9
    E3, i3 = op.solve(p.J, rtol=1e-9, criterion='true')
    assert i2.iterations < i3.iterations


def test_maxiter_status_is_reported(cuda):
    from meanas_b200 import workloads, generic, last_solve_info
    p = workloads.dipole_core(24, pml=6)
    E = generic(p.omega, p.dxes, p.J, p.epsilon, matrix_solver_opts=dict(rtol=1e-12, maxiter=5),
                criterion='true', device=cuda)
    info = last_solve_info()
    assert info.status == 'maxiter' and info.iterations == 5
    assert numpy.all(numpy.isfinite(E))


def test_nonfinite_input_is_reported(cuda):
    from meanas_b200 import workloads, generic, last_solve_info
    p = workloads.dipole_core(16, pml=4)
    eps = p.epsilon.copy()
    eps[100] = numpy.nan
    generic(p.omega, p.dxes, p.J, eps, matrix_solver_opts=dict(rtol=1e-8, maxiter=50), device=cuda)
    assert last_solve_info().status == 'nonfinite'


def test_zero_source_gives_zero_field(cuda):
    from meanas_b200 import workloads, generic, last_solve_info
    p = workloads.dipole_core(16, pml=4)
    E = generic(p.omega, p.dxes, numpy.zeros_like(p.J), p.epsilon, device=cuda)
    assert numpy.all(E == 0) and last_solve_info().converged


def test_sizes_mismatch_raise(cuda):
    from meanas_b200 import workloads, generic
    p = workloads.dipole_core(16, pml=4)
    with pytest.raises(ValueError):
        generic(p.omega, p.dxes, p.J[:-3], p.epsilon, device=cuda)
    with pytest.raises(NotImplementedError):
        generic(p.omega, p.dxes, p.J, p.epsilon, matrix_solver=lambda A, b: b, device=cuda)


def test_progress_logged_every_100_iterations_like_the_reference(cuda, caplog):
    """meanas/fdfd/solvers.py:43-48 logs ||A x - b|| / ||b|| every 100 iterations at INFO on
    the 'meanas.fdfd.solvers' logger; the drop-in logs the same lines after its solve."""
    import logging
    from meanas_b200 import generic, workloads
    p = workloads.dipole_core(24, pml=6)
    with caplog.at_level(logging.INFO, logger='meanas.fdfd.solvers'):
        E, info = generic(p.omega, p.dxes, p.J, p.epsilon, matrix_solver_opts=dict(rtol=1e-8),
                          return_info=True, device=cuda)
    lines = [r.getMessage() for r in caplog.records if r.name == 'meanas.fdfd.solvers']
    assert info.converged and info.iterations >= 200
    assert len(lines) == info.iterations // 100
    assert lines[0].startswith('Solver residual at iteration 100 : ')
    assert float(lines[0].split(':')[-1]) == pytest.approx(info.history[100], rel=1e-12)
