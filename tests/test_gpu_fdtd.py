"""GPU FDTD updates (``fdfd_fdtd_update_e`` / ``_h``) replaying the reference's own
trajectories: ``maxwell_h`` / ``maxwell_e`` with currents injected as in
``meanas/test/test_fdtd.py:203-235`` and ``updates_with_cpml`` with CPML on every face,
float32 and float64 fields.  The kernels follow the reference's arithmetic step by step,
so the fields must be the same bits."""
from __future__ import annotations

import numpy
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

Z = numpy.load(GOLDEN / 'fdtd.npz')
CASES = list(range(int(Z['n'])))


def _case(n):
    p = f'c{n}_'
    shape = tuple(int(v) for v in Z[p + 'shape'])
    dxes = [[Z[f'{p}dx{g}{a}'] for a in range(3)] for g in range(2)]
    return p, str(Z[p + 'kind']), shape, float(Z[p + 'dt']), dxes


@pytest.mark.parametrize('n', CASES)
def test_fdtd_matches_reference_bit_for_bit(cuda, n):
    import torch
    from meanas_b200 import fdtd
    p, kind, shape, dt, dxes = _case(n)
    eps = Z[p + 'eps']
    if kind == 'plain':
        eh2h = fdtd.maxwell_h(dt, dxes, device=cuda)
        eh2e = fdtd.maxwell_e(dt, dxes, device=cuda)
        e = torch.zeros((3, *shape), dtype=torch.float64, device=cuda)
        h = torch.zeros_like(e)
        j = torch.as_tensor(Z[p + 'j'], device=cuda)
        epst = torch.as_tensor(eps, device=cuda)
        for tt in range(10):
            eh2h(e, h)
            eh2e(e, h, eps)
            if tt in (0, 4, 8):
                e += j / epst
            assert numpy.array_equal(e.cpu().numpy(), Z[p + 'es'][tt]), tt
            assert numpy.array_equal(h.cpu().numpy(), Z[p + 'hs'][tt]), tt
    else:
        th = int(Z[p + 'th'])
        ft = torch.float32 if str(Z[p + 'ftype']) == 'float32' else torch.float64
        params = [[None, None] for _ in range(3)]
        for a in range(3):
            for pp, pol in enumerate((-1, 1)):
                if f'{p}pml{a}{pp}e' in Z:
                    params[a][pp] = fdtd.cpml_params(axis=a, polarity=pol, dt=dt, thickness=th,
                                                     epsilon_eff=1.5, cfs_alpha=0.05)
        upd_e, upd_h = fdtd.updates_with_cpml(params, dt, dxes, eps, dtype=numpy.float32, device=cuda)
        e = torch.zeros((3, *shape), dtype=ft, device=cuda)
        h = torch.zeros_like(e)
        src = tuple(s // 2 for s in shape)
        k = 0
        for tt in range(40):
            upd_h(e, h)
            upd_e(e, h, eps)
            # the reference adds a Python float to one element of e (float64 sum, cast to e's type)
            val = float(numpy.sin(0.35 * tt) * numpy.exp(-((tt - 12) / 6) ** 2))
            e[(2, *src)] = torch.tensor(float(e[(2, *src)].item()) + val, dtype=ft)
            if tt % 8 == 7:
                assert numpy.array_equal(e.cpu().numpy(), Z[p + 'es'][k]), tt
                assert numpy.array_equal(h.cpu().numpy(), Z[p + 'hs'][k]), tt
                k += 1


def test_numpy_fields_are_updated_in_place(cuda):
    from meanas_b200 import fdtd
    p, kind, shape, dt, dxes = _case(0)
    e = numpy.zeros((3, *shape))
    e[2, shape[0] // 2, shape[1] // 2, 0] = 1.0
    h = numpy.zeros_like(e)
    out = fdtd.maxwell_h(dt, dxes, device=cuda)(e, h)
    assert out is h and numpy.abs(h).sum() > 0
