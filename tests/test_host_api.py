"""Host-side checks of the drop-ins that need no GPU: argument errors raise before any
device work, and the CPML coefficients keep the reference's layout."""
from __future__ import annotations

import numpy
import pytest
from scipy import sparse


@pytest.mark.parametrize('kw, msg', [(dict(axis=3), 'axis'), (dict(polarity=0), 'polarity'),
                                     (dict(thickness=2), 'thickness'), (dict(epsilon_eff=0), 'epsilon_eff')])
def test_cpml_params_rejects_what_the_reference_rejects(kw, msg):
    from meanas_b200 import fdtd
    args = dict(axis=0, polarity=1, dt=0.3, thickness=8)
    args.update(kw)
    with pytest.raises(ValueError):
        fdtd.cpml_params(**args)


@pytest.mark.parametrize('axis', [0, 1, 2])
@pytest.mark.parametrize('polarity', [-1, 1])
def test_cpml_params_layout(axis, polarity):
    from meanas_b200 import fdtd
    prm = fdtd.cpml_params(axis=axis, polarity=polarity, dt=0.3, thickness=6)
    for side in ('param_e', 'param_h'):
        p0, p1, p2 = prm[side]
        want = [1, 1, 1]
        want[axis] = 6
        assert p0.shape == p1.shape == p2.shape == tuple(want)
        assert numpy.all((0 < p0) & (p0 <= 1)) and numpy.all(p1 <= 0) and numpy.all((0 < p2) & (p2 <= 1))
    # the region is the face's slab: the low face for polarity -1, the high one for +1
    sl = prm['region'][axis]
    assert (sl.start, sl.stop) == ((None, 6) if polarity < 0 else (-6, None))


def test_matrix_solver_rejects_unknown_options_before_device_work():
    from meanas_b200.csr import matrix_solver
    with pytest.raises(TypeError, match='M1'):
        matrix_solver(sparse.eye_array(3, format='csr', dtype=complex), numpy.ones(3), M1=None)
