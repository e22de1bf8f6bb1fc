"""The GPU CSR solver behind ``meanas_b200.csr.matrix_solver``, the drop-in for the
reference's ``matrix_solver`` hook (``meanas/fdfd/solvers.py:97-103,134``): products
against scipy, solves against direct solutions, and the reference ``generic()`` flow
(the oracle's port of it) run with this hook against the reference's own fields."""
from __future__ import annotations

import numpy
import pytest
from scipy import sparse
import scipy.sparse.linalg

from conftest import golden_cases

pytestmark = pytest.mark.gpu

SOLVES = golden_cases('solve')
OPS = golden_cases('operator')


def _random_csr(n: int, seed: int, dominant: bool) -> sparse.csr_array:
    rng = numpy.random.default_rng(seed)
    nnz_row = rng.integers(0, 17, n)
    nnz_row[rng.random(n) < 0.02] = 0        # some empty rows
    rows = numpy.repeat(numpy.arange(n), nnz_row)
    cols = rng.integers(0, n, rows.size)
    vals = rng.standard_normal(rows.size) + 1j * rng.standard_normal(rows.size)
    A = sparse.csr_array((vals, (rows, cols)), shape=(n, n))
    if dominant:
        A = A + sparse.diags_array(4.0 + numpy.abs(A).sum(axis=1) + 1j * rng.standard_normal(n))
    return sparse.csr_array(A)


@pytest.mark.parametrize('n', [1, 37, 5000, 70001])
def test_spmv_matches_scipy(cuda, n):
    from meanas_b200.csr import CsrMatrix
    A = _random_csr(n, n, dominant=False)
    x = numpy.random.default_rng(1).standard_normal(n) + 1j * numpy.random.default_rng(2).standard_normal(n)
    y = (CsrMatrix(A, cuda) @ x).cpu().numpy()
    ref = A @ x
    assert numpy.linalg.norm(y - ref) <= 1e-14 * max(numpy.linalg.norm(ref), 1e-300)


@pytest.mark.parametrize('c', OPS, ids=lambda c: f"op{c['index']}")
def test_spmv_of_assembled_wave_operator(cuda, c):
    from oracle import fdfd_oracle as O
    from meanas_b200.csr import CsrMatrix
    A = O.e_full_csr(complex(c['omega']), c['dxes'], c['eps'], c.get('mu'), c.get('pec'), c.get('pmc'))
    y = (CsrMatrix(A, cuda) @ c['x']).cpu().numpy()
    assert numpy.linalg.norm(y - c['A0x']) <= 1e-13 * numpy.linalg.norm(c['A0x'])


@pytest.mark.parametrize('n', [50, 20000])
def test_solve_matches_direct_solution(cuda, n):
    from meanas_b200.csr import CsrMatrix
    A = _random_csr(n, 7 + n, dominant=True)
    b = numpy.random.default_rng(3).standard_normal(n) + 1j
    M = CsrMatrix(A, cuda)
    x, info = M.solve(b, rtol=1e-12)
    assert info['status'] == 'converged', info
    xh = x.cpu().numpy()
    if n <= 1000:  # a direct solve of a random sparsity pattern fills in: small n only
        ref = scipy.sparse.linalg.spsolve(A.tocsc(), b)
        assert numpy.linalg.norm(xh - ref) <= 1e-10 * numpy.linalg.norm(ref)
    # the true residual, recomputed on the host
    assert numpy.linalg.norm(A @ xh - b) <= 1.01e-12 * numpy.linalg.norm(b)
    assert info['residual'] <= 1e-12 * 1.01
    # warm start from the answer: converged before the first iteration
    x2, info2 = M.solve(b, x.cpu().numpy(), rtol=1e-10)
    assert info2['status'] == 'converged' and info2['iterations'] == 0


def test_maxiter_returns_the_last_iterate(cuda):
    from meanas_b200.csr import matrix_solver
    A = _random_csr(3000, 11, dominant=True)
    b = numpy.ones(3000, dtype=complex)
    x = matrix_solver(A, b, rtol=1e-14, maxiter=2)
    assert x.shape == (3000,) and numpy.isfinite(x).all()
    assert numpy.linalg.norm(A @ x - b) < numpy.linalg.norm(b)


@pytest.mark.parametrize('c', [c for c in SOLVES if c['tag'] == 'pml3d'],
                         ids=lambda c: f"s{c['index']}-{'adj' if c['adjoint'] else 'fwd'}")
def test_reference_generic_with_gpu_matrix_solver(cuda, c):
    """generic()'s own flow (assemble, symmetrise, matrix_solver, unscale) with the GPU hook,
    forward and adjoint, against the reference's generic() fields."""
    from oracle import fdfd_oracle as O
    from meanas_b200.csr import matrix_solver
    om = complex(c['omega'])
    E, _ = O.generic_qmr(om, c['dxes'], c['J'], c['eps'], c.get('mu'), pec=c.get('pec'), pmc=c.get('pmc'),
                         adjoint=bool(c['adjoint']), rtol=1e-12, matrix_solver=matrix_solver)
    ref = c['E']
    assert numpy.linalg.norm(E - ref) <= 1e-7 * numpy.linalg.norm(ref)


def test_unsupported_options_raise():
    from meanas_b200.csr import matrix_solver
    with pytest.raises(TypeError, match='M1'):
        matrix_solver(sparse.eye_array(3, format='csr', dtype=complex), numpy.ones(3), M1=None)
