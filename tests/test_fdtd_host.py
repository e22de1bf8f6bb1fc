"""FDTD host side without a GPU: the CPML coefficients against the reference's tables, and
the oracle's FDTD restatement against the reference's trajectories."""
from __future__ import annotations

import numpy
import pytest

from conftest import GOLDEN
from oracle import fdfd_oracle as O

Z = numpy.load(GOLDEN / 'fdtd.npz')
CASES = list(range(int(Z['n'])))


def _case(n):
    p = f'c{n}_'
    shape = tuple(int(v) for v in Z[p + 'shape'])
    dxes = [[Z[f'{p}dx{g}{a}'] for a in range(3)] for g in range(2)]
    return p, str(Z[p + 'kind']), shape, float(Z[p + 'dt']), dxes


@pytest.mark.parametrize('n', CASES)
def test_cpml_params_match_reference_tables(n):
    from meanas_b200 import fdtd
    p, kind, shape, dt, _ = _case(n)
    if kind != 'cpml':
        pytest.skip('no PML in this case')
    th = int(Z[p + 'th'])
    for a in range(3):
        for pp, pol in enumerate((-1, 1)):
            key = f'{p}pml{a}{pp}e'
            if key not in Z:
                continue
            prm = fdtd.cpml_params(axis=a, polarity=pol, dt=dt, thickness=th, epsilon_eff=1.5, cfs_alpha=0.05)
            for side in ('e', 'h'):
                got = numpy.stack([numpy.ravel(v) for v in prm['param_' + side]])
                assert numpy.array_equal(got, Z[f'{p}pml{a}{pp}{side}'])


@pytest.mark.parametrize('n', CASES)
def test_oracle_fdtd_reproduces_reference_trajectories(n):
    p, kind, shape, dt, dxes = _case(n)
    eps = Z[p + 'eps']
    if kind == 'plain':
        e = numpy.zeros((3, *shape))
        h = numpy.zeros((3, *shape))
        for tt in range(10):
            O.fdtd_plain_step(e, h, eps, dt, dxes)
            if tt in (0, 4, 8):
                e += Z[p + 'j'] / eps
            assert numpy.array_equal(e, Z[p + 'es'][tt]) and numpy.array_equal(h, Z[p + 'hs'][tt])
    else:
        ft = numpy.dtype(str(Z[p + 'ftype']))
        params = [[None, None] for _ in range(3)]
        for a in range(3):
            for pp in range(2):
                if f'{p}pml{a}{pp}e' in Z:
                    params[a][pp] = (Z[f'{p}pml{a}{pp}e'], Z[f'{p}pml{a}{pp}h'])
        U = O.CpmlUpdates(params, dt, dxes, shape, numpy.float32)
        e = numpy.zeros((3, *shape), ft)
        h = numpy.zeros((3, *shape), ft)
        src = tuple(s // 2 for s in shape)
        k = 0
        for tt in range(40):
            U.update_H(e, h)
            U.update_E(e, h, eps)
            e[(2, *src)] += numpy.sin(0.35 * tt) * numpy.exp(-((tt - 12) / 6) ** 2)
            if tt % 8 == 7:
                assert numpy.array_equal(e, Z[p + 'es'][k]) and numpy.array_equal(h, Z[p + 'hs'][k])
                k += 1
