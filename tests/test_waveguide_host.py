"""Host-side argument handling of the GPU mode source (no device work)."""
from __future__ import annotations

import numpy
import pytest

from meanas_b200 import waveguide as W


def test_window_and_mask_planes():
    lo, hi = W._window([slice(None), slice(3, 4), slice(2, -2)], (5, 8, 10), 1)
    assert (lo, hi) == ([0, 3, 2], [5, 4, 8])
    assert W._mask_planes([slice(None), slice(3, 4), slice(None)], 8, 1, +1) == (3, 8)
    assert W._mask_planes([slice(None), slice(3, 4), slice(None)], 8, 1, -1) == (0, 4)
    # negative indices follow Python slicing, as numpy indexing does in the reference
    assert W._mask_planes([slice(-3, -2), slice(None), slice(None)], 8, 0, +1) == (5, 8)


@pytest.mark.parametrize('slices, axis, msg', [
    ([slice(None), slice(3, 5), slice(None)], 1, 'exactly one index'),
    ([slice(None), slice(3, 4), slice(None, None, 2)], 1, 'unit-step'),
    ([slice(4, 2), slice(3, 4), slice(None)], 1, 'non-empty'),
    ([slice(None), slice(3, 4)], 1, 'one slice per axis'),
])
def test_bad_slices_are_refused(slices, axis, msg):
    with pytest.raises(ValueError, match=msg):
        W._slice_desc((5, 8, 10), axis, 1, slices)


def test_bad_axis_and_polarity_are_refused():
    with pytest.raises(ValueError, match='axis'):
        W._slice_desc((5, 8, 10), 3, 1, [slice(None)] * 3)
    with pytest.raises(ValueError, match='polarity'):
        W._slice_desc((5, 8, 10), 0, 0, [slice(1, 2), slice(None), slice(None)])


def test_phase_table_follows_the_reference_arithmetic():
    dxes = [[numpy.array([1.0, 2.0, 0.5 + 0.3j, 1.0]), numpy.ones(1), numpy.ones(1)],
            [numpy.ones(4), numpy.ones(1), numpy.ones(1)]]
    ph = W._phase(0.7 - 0.01j, dxes, 0, -1, [slice(1, 2), slice(None), slice(None)])
    r = numpy.array([1.0, 3.0, 3.5, 4.5]) - 3.0
    assert numpy.allclose(ph, numpy.exp(-1 * -1j * (0.7 - 0.01j) * r), rtol=1e-15)
