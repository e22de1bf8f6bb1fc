"""GPU waveguide-mode source (row f3) against the reference's compute_source / expand_e
(tests/golden/modesrc.npz) and the reference's own unidirectional-source test
(meanas/test/test_fdfd_pml.py:14-28) run on GPU-built sources and GPU solves."""
from __future__ import annotations

import numpy
import pytest

from conftest import golden_cases

pytestmark = pytest.mark.gpu

MODESRC = golden_cases('modesrc')


def _slices(c):
    big = 10 ** 9
    return [slice(None if lo == -big else int(lo), None if hi == big else int(hi)) for lo, hi in c['slices']]


def _rel(a, b):
    return numpy.linalg.norm(numpy.asarray(a) - b) / numpy.linalg.norm(b)


@pytest.mark.parametrize('c', MODESRC, ids=lambda c: f"mode{c['index']}-{tuple(int(s) for s in c['shape'])}")
def test_mode_source_matches_reference(cuda, c):
    from meanas_b200 import waveguide
    axis, pol, k, om = int(c['axis']), int(c['polarity']), complex(c['k']), complex(c['omega'])
    Ee = waveguide.expand_e(c['E'], k, c['dxes'], axis, pol, _slices(c), device=cuda)
    assert Ee.shape == c['E'].shape
    assert _rel(Ee, c['E_expanded']) <= 1e-13
    assert numpy.array_equal(Ee == 0, c['E_expanded'] == 0)
    J = waveguide.compute_source(c['E'], k, om, c['dxes'], axis, pol, _slices(c), c['eps'], c.get('mu'),
                                 device=cuda)
    assert J.shape == c['E'].shape
    assert _rel(J, c['J']) <= 1e-13
    # the source sits on exactly the reference's two planes
    assert numpy.array_equal(J == 0, c['J'] == 0)


def test_mode_source_keeps_cuda_tensors_on_the_device(cuda):
    import torch
    from meanas_b200 import waveguide
    c = MODESRC[-1]
    E = torch.as_tensor(c['E'], device=cuda)
    J = waveguide.compute_source(E, complex(c['k']), complex(c['omega']), c['dxes'], int(c['axis']),
                                 int(c['polarity']), _slices(c), c['eps'], c.get('mu'))
    assert isinstance(J, torch.Tensor) and J.is_cuda
    assert _rel(J.cpu().numpy(), c['J']) <= 1e-13


@pytest.mark.parametrize('c', [c for c in MODESRC if 1 in tuple(int(s) for s in c['shape'][:3])
                               and int(numpy.prod(c['shape'])) == 30],
                         ids=lambda c: f"pml{c['index']}")
def test_reference_pml_test_passes_with_gpu_source_and_solve(cuda, c):
    """meanas/test/test_fdfd_pml.py:14-28: the GPU-built unidirectional source, solved on the
    GPU, leaves |E|^2 = 1 ahead of the source and 0 behind it."""
    from meanas_b200 import waveguide
    from meanas_b200.solvers import generic
    axis, pol = int(c['axis']), int(c['polarity'])
    om = complex(c['omega'])
    J = waveguide.compute_source(c['E'], complex(c['k']), om, c['dxes'], axis, pol, _slices(c), c['eps'],
                                 device=cuda)
    E = generic(om, c['dxes'], J.ravel(), c['eps'].ravel(), matrix_solver_opts={'atol': 1e-15, 'rtol': 1e-11},
                device=cuda)
    e = E.reshape(3, *[int(s) for s in c['shape']])
    e_sqr = numpy.squeeze((e.conj() * e).sum(axis=0))
    tgt, rev = e_sqr[16:19], e_sqr[10:13]
    if pol < 0:
        tgt, rev = rev, tgt
    numpy.testing.assert_allclose(rev, 0, atol=1e-12)
    numpy.testing.assert_allclose(tgt, 1, rtol=3e-6)
