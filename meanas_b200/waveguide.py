"""Unidirectional waveguide-mode sources on the GPU: drop-ins for ``meanas.fdfd.waveguide_3d``.

* ``expand_e(E, wavenumber, dxes, axis, polarity, slices)``
  ``meanas/fdfd/waveguide_3d.py:206-257``: the mode's cross-section at the source plane,
  repeated along the propagation axis with the phase ``exp(-i polarity wavenumber r)``
  (``r`` measured along the real parts of ``dx_e`` from the source plane), inside the
  transverse window of ``slices`` and zero outside it.
* ``compute_source(E, wavenumber, omega, dxes, axis, polarity, slices, epsilon, mu=None)``
  ``meanas/fdfd/waveguide_3d.py:113-156``: the current ``J`` that launches that mode in
  one direction only, ``e_boundary_source(mask, omega, dxes, epsilon, mu) @ expand_e(...)``
  with ``mask`` the half-space from the source plane onward (``polarity > 0``) or up to it.

Both run in the library (``fdfd_mode_expand`` / ``fdfd_mode_source``): one elementwise pass
builds the expanded field and the mask, then the two passes of the boundary-source
stencil form ``J``.  Only the 1D phase table (one entry per plane of the axis) is computed
on the host, with the reference's arithmetic.  ``E`` and the result are ``(3, X, Y, Z)``
fields; numpy inputs give numpy outputs, CUDA tensors stay on the device.
"""
from __future__ import annotations

import ctypes as C
from collections.abc import Sequence
from typing import Any

import numpy
import torch

from . import _lib
from .operators import GridOperator, _stream_handle, as_device


def _window(slices: Sequence[slice], shape: tuple[int, int, int], axis: int) -> tuple[list[int], list[int]]:
    """``[lo, hi)`` per axis of unit-step ``slices``; one index along ``axis``."""
    if len(slices) != 3:
        raise ValueError('slices needs one slice per axis')
    lo, hi = [], []
    for a, (sl, n) in enumerate(zip(slices, shape)):
        idx = numpy.arange(n)[sl]
        if idx.size == 0 or numpy.any(numpy.diff(idx) != 1):
            raise ValueError(f'slices[{a}] must select a non-empty unit-step range')
        lo.append(int(idx[0]))
        hi.append(int(idx[-1]) + 1)
    if hi[axis] - lo[axis] != 1:
        raise ValueError('slices[axis] must select exactly one index')
    return lo, hi


def _phase(wavenumber: complex, dxes, axis: int, polarity: int, slices: Sequence[slice]) -> numpy.ndarray:
    """Per-plane phase of ``expand_e``: ``r_E`` from the cumulative real ``dx_e`` along the
    axis, relative to the source plane (the order of operations of
    ``meanas/fdfd/waveguide_3d.py:238-242``)."""
    a_E = numpy.real(dxes[0][axis]).cumsum()
    r_E = a_E - a_E[slices[axis]]
    iphi = polarity * -1j * wavenumber
    return numpy.exp(iphi * r_E).astype(numpy.complex128)


def _mask_planes(slices: Sequence[slice], n_axis: int, axis: int, polarity: int) -> tuple[int, int]:
    """Planes ``[lo, hi)`` of compute_source's half-space mask (``slices[axis].start``
    onward for ``polarity > 0``, else up to ``slices[axis].stop``)."""
    sl = slices[axis]
    planes = numpy.arange(n_axis)[slice(sl.start, None) if polarity > 0 else slice(None, sl.stop)]
    if planes.size == 0:
        return 0, 0
    return int(planes[0]), int(planes[-1]) + 1


def _slice_desc(shape, axis: int, polarity: int, slices: Sequence[slice]) -> _lib.ModeSlice:
    if axis not in (0, 1, 2):
        raise ValueError(f'axis must be 0, 1 or 2, not {axis}')
    if polarity not in (1, -1):
        raise ValueError(f'polarity must be +1 or -1, not {polarity}')
    lo, hi = _window(slices, shape, axis)
    m = _lib.ModeSlice()
    m.axis = axis
    m.polarity = polarity
    m.lo[:] = lo
    m.hi[:] = hi
    m.mask_lo, m.mask_hi = _mask_planes(slices, shape[axis], axis, polarity)
    return m


def _field_shape(E) -> tuple[int, int, int]:
    shape = tuple(int(s) for s in E.shape)
    if len(shape) != 4 or shape[0] != 3:
        raise ValueError(f'E must be a (3, X, Y, Z) field, not {shape}')
    return shape[1:]


def _out(like: Any, t: torch.Tensor, shape) -> Any:
    t = t.reshape(3, *shape)
    return t if isinstance(like, torch.Tensor) and like.is_cuda else t.cpu().numpy()


def _grid(omega: complex, dxes, epsilon, mu, shape, device) -> GridOperator:
    n = 3 * int(numpy.prod(shape))
    eps = epsilon.reshape(-1) if isinstance(epsilon, torch.Tensor) else numpy.asarray(epsilon).reshape(-1)
    if mu is not None:
        mu = mu.reshape(-1) if isinstance(mu, torch.Tensor) else numpy.asarray(mu).reshape(-1)
    if eps.shape[0] != n:
        raise ValueError(f'epsilon has {eps.shape[0]} elements; the grid needs {n}')
    return GridOperator(omega, dxes, eps, mu, device=device, fp32=False)


def expand_e(E, wavenumber: complex, dxes, axis: int, polarity: int, slices: Sequence[slice], *,
             device: Any | None = None):
    """``meanas.fdfd.waveguide_3d.expand_e`` on the GPU (see the module docstring)."""
    shape = _field_shape(E)
    if tuple(int(numpy.size(d)) for d in dxes[0]) != shape:
        raise ValueError('dxes and E disagree on the grid shape')
    slices = tuple(slices)
    desc = _slice_desc(shape, axis, polarity, slices)
    dev = E.device if isinstance(E, torch.Tensor) and E.is_cuda else device
    grid = _grid(1.0, dxes, numpy.ones(3 * int(numpy.prod(shape))), None, shape, dev)
    Et = as_device(E, torch.complex128, grid.device, grid.n, 'E')
    ph = as_device(_phase(wavenumber, dxes, axis, polarity, slices), torch.complex128, grid.device)
    out = torch.empty_like(Et)
    with torch.cuda.device(grid.device):
        _lib.check(grid.lib.fdfd_mode_expand(grid.plan, Et.data_ptr(), ph.data_ptr(), C.byref(desc),
                                             out.data_ptr(), None, _stream_handle()))
    return _out(E, out, shape)


def compute_source(E, wavenumber: complex, omega: complex, dxes, axis: int, polarity: int,
                   slices: Sequence[slice], epsilon, mu=None, *, device: Any | None = None):
    """``meanas.fdfd.waveguide_3d.compute_source`` on the GPU: ``J`` (``(3, X, Y, Z)``) of
    the unidirectional source of mode ``E`` (see the module docstring)."""
    shape = _field_shape(E)
    if tuple(int(numpy.size(d)) for d in dxes[0]) != shape:
        raise ValueError('dxes and E disagree on the grid shape')
    slices = tuple(slices)
    desc = _slice_desc(shape, axis, polarity, slices)
    dev = E.device if isinstance(E, torch.Tensor) and E.is_cuda else device
    grid = _grid(omega, dxes, epsilon, mu, shape, dev)
    Et = as_device(E, torch.complex128, grid.device, grid.n, 'E')
    ph = as_device(_phase(wavenumber, dxes, axis, polarity, slices), torch.complex128, grid.device)
    e_work = torch.empty_like(Et)
    mask = torch.empty(grid.n, dtype=torch.float64, device=grid.device)
    J = torch.empty_like(Et)
    with torch.cuda.device(grid.device):
        _lib.check(grid.lib.fdfd_mode_source(grid.plan, Et.data_ptr(), ph.data_ptr(), C.byref(desc),
                                             e_work.data_ptr(), mask.data_ptr(), J.data_ptr(), _stream_handle()))
    return _out(E, J, shape)
