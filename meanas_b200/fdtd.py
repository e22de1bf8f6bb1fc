"""FDTD Yee updates with CPML on the GPU: drop-ins for ``meanas.fdtd``'s update builders.

* ``maxwell_h(dt, dxes)`` / ``maxwell_e(dt, dxes)``     ``meanas/fdtd/base.py:13-125``
* ``cpml_params(axis, polarity, dt, ...)``              ``meanas/fdtd/pml.py:20-91``
* ``updates_with_cpml(cpml_params, dt, dxes, epsilon, dtype=float32)``
                                                        ``meanas/fdtd/pml.py:94-230``

The returned update functions change their field arguments in place, like the
reference's.  Fields may be CUDA tensors (they stay on the device; the fast path) or
numpy arrays (copied to the device and back on every call).  Each half step is one
kernel (``fdfd_fdtd_update_e`` / ``fdfd_fdtd_update_h``) that follows the reference's
arithmetic step by step, so the fields equal the reference's bit for bit.
"""
from __future__ import annotations

import ctypes as C
from typing import Any, Callable, Sequence

import numpy
import torch

from . import _lib
from .operators import _device, _stream_handle


def cpml_params(axis: int, polarity: int, dt: float, thickness: int = 8, ln_R_per_layer: float = -1.6,
                epsilon_eff: float = 1, mu_eff: float = 1, m: float = 3.5, ma: float = 1,
                cfs_alpha: float = 0) -> dict[str, Any]:
    """CPML coefficients of one face (``meanas/fdtd/pml.py:20-91``): graded conductivity
    ``sigma_max (x/th)^m``, ``kappa = 1 + (kappa_max - 1)(x/th)^m``, CFS ``alpha``, and the
    recurrence factors ``p0 = exp(-(sigma/kappa + alpha) dt)``,
    ``p1 = sigma / (sigma + kappa alpha) (p0 - 1)``, ``p2 = 1/kappa`` at the E and H
    positions of the ``thickness`` layers."""
    if axis not in range(3):
        raise ValueError(f'Invalid axis: {axis}')
    if polarity not in (-1, 1):
        raise ValueError(f'Invalid polarity: {polarity}')
    if thickness <= 2:
        raise ValueError('It would be wise to have a pml with 4+ cells of thickness')
    if epsilon_eff <= 0:
        raise ValueError('epsilon_eff must be positive')
    sigma_max = -ln_R_per_layer / 2 * (m + 1)
    kappa_max = numpy.sqrt(epsilon_eff * mu_eff)
    xe = numpy.arange(1, thickness + 1, dtype=float)
    xh = numpy.arange(1, thickness + 1, dtype=float)
    if polarity > 0:
        xe -= 0.5
    else:
        xh -= 0.5
        xe = xe[::-1]
        xh = xh[::-1]
    shape = [1, 1, 1]
    shape[axis] = thickness

    def par(x):
        scaling = (x / thickness) ** m
        sigma = scaling * sigma_max
        kappa = 1 + scaling * (kappa_max - 1)
        alpha = ((1 - x / thickness) ** ma) * cfs_alpha
        p0 = numpy.exp(-(sigma / kappa + alpha) * dt)
        p1 = sigma / (sigma + kappa * alpha) * (p0 - 1)
        p2 = 1 / kappa
        return p0.reshape(shape), p1.reshape(shape), p2.reshape(shape)

    region = [slice(None)] * 3
    region[axis] = slice(None, thickness) if polarity < 0 else slice(-thickness, None)
    return {'param_e': par(xe), 'param_h': par(xh), 'region': tuple(region)}


def _real_type(t: torch.Tensor) -> int:
    if t.dtype == torch.float32:
        return _lib.REAL32
    if t.dtype == torch.float64:
        return _lib.REAL64
    raise TypeError(f'FDTD fields must be float32 or float64, got {t.dtype}')


class _Fields:
    """Device views of the caller's fields; numpy arrays are copied back on exit."""

    def __init__(self, device, *arrays):
        self.src = arrays
        self.dev = []
        for a in arrays:
            if isinstance(a, torch.Tensor):
                if not a.is_cuda or not a.is_contiguous():
                    raise ValueError('FDTD field tensors must be contiguous CUDA tensors')
                self.dev.append(a)
            else:
                if a.dtype not in (numpy.float32, numpy.float64):
                    raise TypeError(f'FDTD fields must be float32 or float64, got {a.dtype}')
                self.dev.append(torch.from_numpy(numpy.ascontiguousarray(a)).to(device))

    def copy_back(self, *which: int) -> None:
        for w in which:
            a = self.src[w]
            if not isinstance(a, torch.Tensor):
                a[...] = self.dev[w].cpu().numpy()


class _Grid:
    def __init__(self, dxes, device):
        self.device = _device(device)
        self.shape = tuple(int(numpy.size(d)) for d in dxes[0])
        self.n = 3 * int(numpy.prod(self.shape))
        self.dx = [[torch.as_tensor(numpy.asarray(d, dtype=numpy.float64).ravel(), device=self.device)
                    for d in g] for g in dxes]
        self.lib = _lib.load()
        self._mats: dict[int, torch.Tensor] = {}

    def desc(self, form: int, dt: float, field_type: int, psi_type: int = _lib.REAL32) -> _lib.FdtdDesc:
        d = _lib.FdtdDesc()
        d.shape[:] = self.shape
        d.field_type = field_type
        d.psi_type = psi_type
        d.form = form
        d.dt = float(dt)
        for a in range(3):
            d.dxe[a] = self.dx[0][a].data_ptr()
            d.dxh[a] = self.dx[1][a].data_ptr()
        return d

    def material(self, m, name: str) -> torch.Tensor | None:
        """A float64 [3N] device copy of epsilon / mu (scalars broadcast), cached per object."""
        if m is None:
            return None
        key = id(m)
        cached = self._mats.get(key)
        if cached is not None and cached[0] is m:
            return cached[1]
        if isinstance(m, torch.Tensor):
            t = m.to(device=self.device, dtype=torch.float64).reshape(-1).contiguous()
        else:
            arr = numpy.asarray(m, dtype=numpy.float64)
            if arr.size in (1, 3) and arr.size != self.n:
                arr = numpy.broadcast_to(arr.reshape(-1, 1), (3, self.n // 3)) if arr.size == 3 else \
                    numpy.full(self.n, float(arr.ravel()[0]))
            t = torch.from_numpy(numpy.ascontiguousarray(arr).ravel()).to(self.device)
        if t.numel() != self.n:
            raise ValueError(f'{name} has {t.numel()} elements, expected {self.n}')
        self._mats[key] = (m, t)
        return t


def maxwell_h(dt: float, dxes, *, device: Any | None = None) -> Callable:
    """``f(e, h, mu=None)``: ``h -= dt * curl_forward(dxes[0])(e) [/ mu]`` in place; returns h
    (``meanas/fdtd/base.py:70-125``)."""
    grid = _Grid(dxes, device)

    def mh_fun(e, h, mu=None):
        f = _Fields(grid.device, e, h)
        d = grid.desc(_lib.FDTD_PLAIN, dt, _real_type(f.dev[0]))
        m = grid.material(mu, 'mu')
        d.mu = m.data_ptr() if m is not None else None
        with torch.cuda.device(grid.device):
            _lib.check(grid.lib.fdfd_fdtd_update_h(C.byref(d), f.dev[0].data_ptr(), f.dev[1].data_ptr(),
                                                   _stream_handle()))
        f.copy_back(1)
        return h
    return mh_fun


def maxwell_e(dt: float, dxes, *, device: Any | None = None) -> Callable:
    """``f(e, h, epsilon)``: ``e += dt * curl_back(dxes[1])(h) / epsilon`` in place; returns e
    (``meanas/fdtd/base.py:13-67``)."""
    grid = _Grid(dxes, device)

    def me_fun(e, h, epsilon):
        f = _Fields(grid.device, e, h)
        d = grid.desc(_lib.FDTD_PLAIN, dt, _real_type(f.dev[0]))
        d.epsilon = grid.material(epsilon, 'epsilon').data_ptr()
        with torch.cuda.device(grid.device):
            _lib.check(grid.lib.fdfd_fdtd_update_e(C.byref(d), f.dev[0].data_ptr(), f.dev[1].data_ptr(),
                                                   _stream_handle()))
        f.copy_back(0)
        return e
    return me_fun


def updates_with_cpml(cpml_params: Sequence[Sequence[dict[str, Any] | None]], dt: float, dxes, epsilon, *,
                      dtype=numpy.float32, device: Any | None = None) -> tuple[Callable, Callable]:
    """``(update_E, update_H)`` with CPML on the faces whose ``cpml_params[axis][0 | 1]`` is
    set (``meanas/fdtd/pml.py:94-230``): ``update_E(e, h, epsilon)``,
    ``update_H(e, h, mu=(1, 1, 1))``, in place.  The psi arrays (``dtype``) live on the device."""
    grid = _Grid(dxes, device)
    psi_type = _lib.REAL32 if numpy.dtype(dtype) == numpy.float32 else _lib.REAL64
    tdt = torch.float32 if psi_type == _lib.REAL32 else torch.float64
    keep = []  # device arrays the descriptors point to
    faces = []
    for a in range(3):
        for pp in range(2):
            prm = cpml_params[a][pp]
            if prm is None:
                continue
            th = int(numpy.size(prm['param_e'][0]))
            rshape = list(grid.shape)
            rshape[a] = th
            pe = torch.as_tensor(numpy.stack([numpy.ravel(v) for v in prm['param_e']]), dtype=torch.float64,
                                 device=grid.device).contiguous()
            ph = torch.as_tensor(numpy.stack([numpy.ravel(v) for v in prm['param_h']]), dtype=torch.float64,
                                 device=grid.device).contiguous()
            psi = [torch.zeros(rshape, dtype=tdt, device=grid.device) for _ in range(4)]
            keep += [pe, ph, *psi]
            faces.append((a, pp, th, pe, ph, psi))

    def desc(field_type: int) -> _lib.FdtdDesc:
        d = grid.desc(_lib.FDTD_CPML, dt, field_type, psi_type)
        for a, pp, th, pe, ph, psi in faces:
            f = d.face[a][pp]
            f.thickness = th
            f.param_e = pe.data_ptr()
            f.param_h = ph.data_ptr()
            f.psi_e[0], f.psi_e[1] = psi[0].data_ptr(), psi[1].data_ptr()
            f.psi_h[0], f.psi_h[1] = psi[2].data_ptr(), psi[3].data_ptr()
        return d

    eps0 = grid.material(epsilon, 'epsilon')

    def update_E(e, h, epsilon=None) -> None:
        f = _Fields(grid.device, e, h)
        d = desc(_real_type(f.dev[0]))
        d.epsilon = (grid.material(epsilon, 'epsilon') if epsilon is not None else eps0).data_ptr()
        with torch.cuda.device(grid.device):
            _lib.check(grid.lib.fdfd_fdtd_update_e(C.byref(d), f.dev[0].data_ptr(), f.dev[1].data_ptr(),
                                                   _stream_handle()))
        f.copy_back(0)

    def update_H(e, h, mu=None) -> None:
        f = _Fields(grid.device, e, h)
        d = desc(_real_type(f.dev[0]))
        m = None if mu is None or (not isinstance(mu, torch.Tensor) and numpy.all(numpy.asarray(mu) == 1)
                                   and numpy.size(mu) <= 3) else grid.material(mu, 'mu')
        d.mu = m.data_ptr() if m is not None else None
        with torch.cuda.device(grid.device):
            _lib.check(grid.lib.fdfd_fdtd_update_h(C.byref(d), f.dev[0].data_ptr(), f.dev[1].data_ptr(),
                                                   _stream_handle()))
        f.copy_back(1)

    update_E.psi = update_H.psi = keep  # keeps the device arrays alive with the closures
    return update_E, update_H
