"""The steps either side of the solve on the GPU: sources, E -> H, Poynting products.

Drop-ins for the reference's source construction (before ``generic()``):

* ``e_tfsf_source(TF_region, omega, dxes, epsilon, mu=None)``
  ``meanas/fdfd/operators.py:366-393``: ``op @ E`` is the current that injects E inside
  the total-field region.
* ``e_boundary_source(mask, omega, dxes, epsilon, mu=None, periodic_mask_edges=False)``
  ``meanas/fdfd/operators.py:396-450``: the same, kept on the edges of the mask.

and for the post-processing of a ``generic()`` result:

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


def e_tfsf_source(TF_region, omega: complex, dxes, epsilon, mu=None, *,
                  device: Any | None = None) -> FieldOperator:
    """``(A0 Q - Q A0) / (-i omega)`` with ``Q = diag(TF_region)`` as ``op @ E``
    (``meanas/fdfd/operators.py:366-393``; ``A0`` without PEC/PMC, as there)."""
    grid = GridOperator(omega, dxes, epsilon, mu, device=device, fp32=False)
    q = as_device(TF_region, torch.float64, grid.device, grid.n, 'TF_region')
    return FieldOperator(lambda e: _out(e, grid.tfsf_source(e, q)), grid.n)


def e_boundary_source(mask, omega: complex, dxes, epsilon, mu=None, periodic_mask_edges: bool = False, *,
                      device: Any | None = None) -> FieldOperator:
    """``e_tfsf_source`` kept only where shifting ``mask`` by one cell along a non-singleton
    axis changes it (``meanas/fdfd/operators.py:396-450``; past the grid edge the shift
    mirrors, or wraps with ``periodic_mask_edges``)."""
    grid = GridOperator(omega, dxes, epsilon, mu, device=device, fp32=False)
    q = as_device(mask, torch.float64, grid.device, grid.n, 'mask')
    return FieldOperator(lambda e: _out(e, grid.tfsf_source(e, q, edges=True, periodic=periodic_mask_edges)),
                         grid.n)
