"""The step after the solve on the GPU: E -> H and the Poynting cross product.

Drop-ins for the reference's post-processing of a ``generic()`` result:

* ``e2h(omega, dxes, mu=None, pmc=None)``        ``meanas/fdfd/operators.py:253-282``
  (a sparse matrix there; here a matrix-free operator used the same way, ``op @ E``).
* ``poynting_e_cross(e, dxes)``                  ``meanas/fdfd/operators.py:310-336``
  (``P @ h`` is the Yee-grid ``E x h``).
* ``poynting_e_cross_h(dxes)``                   ``meanas/fdfd/functional.py:187-221``
  (``f(e, h)`` on ``(3, X, Y, Z)`` fields).

One kernel (``fdfd_e2h`` in ``libmeanas_fdfd.so``) forms H from E and the cross product
from the same loads; ``GridOperator.poynting(E)`` returns both in one pass.  Host (numpy)
inputs give numpy outputs; CUDA tensors stay on the device.
"""
from __future__ import annotations

from typing import Any, Callable

import numpy
import torch

from .operators import GridOperator, as_device


def _out(like: Any, t: torch.Tensor):
    return t if isinstance(like, torch.Tensor) and like.is_cuda else t.cpu().numpy()


def _grid(omega: complex, dxes, mu=None, pmc=None, device=None) -> GridOperator:
    shape = tuple(int(numpy.size(d)) for d in dxes[0])
    ones = numpy.ones(3 * int(numpy.prod(shape)))
    return GridOperator(omega, dxes, ones, mu, None, pmc, device=device, fp32=False)


class FieldOperator:
    """A matrix-free linear operator on 1D ``vec()`` fields: ``op @ v``."""

    def __init__(self, fn: Callable[[Any], Any], n: int):
        self._fn = fn
        self.shape = (n, n)

    def __matmul__(self, v):
        return self._fn(v)


def e2h(omega: complex, dxes, mu=None, pmc=None, *, device: Any | None = None,
        operator: GridOperator | None = None) -> FieldOperator:
    """``H = pm diag(1/mu) ce(E) / (-i omega)`` as ``e2h(...) @ E``
    (``meanas/fdfd/operators.py:253-282``).  ``operator`` reuses the plan of a solve
    (its omega, mu and PMC mask)."""
    grid = operator if operator is not None else _grid(omega, dxes, mu, pmc, device)
    return FieldOperator(lambda e: _out(e, grid.e2h(e)), grid.n)


def poynting_e_cross(e, dxes, *, device: Any | None = None,
                     operator: GridOperator | None = None) -> FieldOperator:
    """The ``(E x)`` operator of ``meanas/fdfd/operators.py:310-336``: ``P @ h`` is the
    Yee-grid cross product of ``e`` with ``h`` (pass ``h.conj()`` for the Poynting vector,
    as ``meanas/test/test_fdfd.py:38-40`` does)."""
    grid = operator if operator is not None else _grid(1.0, dxes, device=device)
    et = as_device(e, torch.complex128, grid.device, grid.n, 'e')
    return FieldOperator(lambda h: _out(h, grid.poynting(et, h, conj=False)[0]), grid.n)


def poynting_e_cross_h(dxes, *, device: Any | None = None) -> Callable[[Any, Any], Any]:
    """``f(e, h) = e x h`` on ``(3, X, Y, Z)`` fields (``meanas/fdfd/functional.py:187-221``)."""
    grid = _grid(1.0, dxes, device=device)
    shape = (3, *grid.shape)

    def exh(e, h):
        S, _ = grid.poynting(as_device(e, torch.complex128, grid.device, grid.n, 'e'), h, conj=False)
        return _out(e, S.reshape(shape))
    return exh
