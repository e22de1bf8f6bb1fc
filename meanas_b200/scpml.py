"""Stretched-coordinate PML cell widths (host side, O(X+Y+Z) work).

Same API and arithmetic as the reference's ``meanas/fdfd/scpml.py``:

* ``prepare_s_function`` follows ``meanas/fdfd/scpml.py:18-38``:
  ``s(l) = (m + 1) * ln_R / 2 * l**m``.
* ``uniform_grid_scpml`` follows ``meanas/fdfd/scpml.py:41-95`` (including its
  lack of a ``/thickness`` normalisation).
* ``stretch_with_scpml`` follows ``meanas/fdfd/scpml.py:98-166``: the widths of
  the ``thickness`` outermost cells on one face are multiplied by
  ``1 + i * s(l) / d / (sqrt(eps_eff) * Re(omega))``, with ``l`` the normalised
  depth of the E-grid cell centre (``dx_e``) or H-grid edge (``dx_h``) inside
  the layer and ``d`` the layer's physical depth.  Like the reference it writes
  the stretched arrays back into ``dxes`` and returns it.

These are tiny 1D computations; they stay in numpy on the host and only their
results (1D complex tables) are uploaded to the device.
"""
from __future__ import annotations

from collections.abc import Callable, Sequence

import numpy
from numpy.typing import NDArray

s_function_t = Callable[[NDArray[numpy.float64]], NDArray[numpy.float64]]


def prepare_s_function(ln_R: float = -16, m: float = 4) -> s_function_t:
    """Polynomial PML conductivity profile ``s_max * l**m``, ``s_max = (m+1) ln_R / 2``."""
    s_max = (m + 1) * ln_R / 2

    def s_of_depth(depth: NDArray[numpy.float64]) -> NDArray[numpy.float64]:
        return s_max * depth ** m

    return s_of_depth


def uniform_grid_scpml(
        shape: Sequence[int],
        thicknesses: Sequence[int],
        omega: float,
        epsilon_effective: float = 1.0,
        s_function: s_function_t | None = None,
        ) -> list[list[NDArray]]:
    """Unit-width grid with a PML of ``thicknesses[a]`` cells on both faces of axis ``a``."""
    if s_function is None:
        s_function = prepare_s_function()
    scale = numpy.sqrt(epsilon_effective) * numpy.real(omega)
    widths_e: list[NDArray] = []
    widths_h: list[NDArray] = []
    for n, th in zip(tuple(shape), tuple(thicknesses)):
        if th <= 0:
            widths_e.append(numpy.ones((n,)))
            widths_h.append(numpy.ones((n,)))
            continue
        u = numpy.arange(n, dtype=numpy.float64)

        def depth(v: NDArray[numpy.float64]) -> NDArray[numpy.float64]:
            return ((th - v).clip(0) + (v - (n - th)).clip(0)) / th

        widths_e.append(1 + 1j * s_function(depth(u)) / scale)
        widths_h.append(1 + 1j * s_function(depth(u + 0.5)) / scale)
    return [widths_e, widths_h]


def stretch_with_scpml(
        dxes: list[list[NDArray]],
        axis: int,
        polarity: int,
        omega: float,
        epsilon_effective: float = 1.0,
        thickness: int = 10,
        s_function: s_function_t | None = None,
        ) -> list[list[NDArray]]:
    """Add a PML of ``thickness`` cells to the low (``polarity>0``) or high face of ``axis``.

    Mutates ``dxes[0][axis]`` and ``dxes[1][axis]`` (replacing them with complex
    copies) and returns ``dxes``, as the reference does.
    """
    if s_function is None:
        s_function = prepare_s_function()
    w_e = numpy.asarray(dxes[0][axis]).astype(complex)
    w_h = numpy.asarray(dxes[1][axis]).astype(complex)

    edges = numpy.concatenate(([0], numpy.cumsum(w_e)))
    centres = (edges[:-1] + edges[1:]) / 2
    starts = edges[:-1]
    scale = numpy.sqrt(epsilon_effective) * numpy.real(omega)

    if polarity > 0:
        inner = edges[thickness]
        depth = inner - edges[0]
        sel = slice(thickness)

        def norm_depth(p: NDArray) -> NDArray:
            return (inner - p) / (inner - edges[0])
    else:
        inner = edges[-thickness - 1]
        depth = edges[-1] - inner
        sel = slice(None) if thickness == 0 else slice(-thickness, None)

        def norm_depth(p: NDArray) -> NDArray:
            return (p - inner) / (edges[-1] - inner)

    w_e[sel] *= 1 + 1j * s_function(norm_depth(centres[sel])) / depth / scale
    w_h[sel] *= 1 + 1j * s_function(norm_depth(starts[sel])) / depth / scale
    dxes[0][axis] = w_e
    dxes[1][axis] = w_h
    return dxes


def stretch_all_faces(
        shape: Sequence[int],
        omega: float,
        thickness: int,
        *,
        ln_R: float = -16,
        m: float = 3.5,
        epsilon_effective: float = 1.0,
        dx: float = 1.0,
        ) -> list[list[NDArray]]:
    """Uniform grid of width ``dx`` with a ``stretch_with_scpml`` PML on every non-singleton face.

    This is the construction used by the reference's PML test and examples
    (``meanas/test/test_fdfd_pml.py:134-143``, ``examples/fdfd0.py:71-74``):
    one ``stretch_with_scpml`` call per face, +1 polarity then -1.
    """
    sf = prepare_s_function(ln_R=ln_R, m=m)
    dxes = [[numpy.full(n, float(dx)) for n in shape] for _ in range(2)]
    for a, n in enumerate(shape):
        if n <= 1 or thickness <= 0:
            continue
        for pol in (-1, 1):
            dxes = stretch_with_scpml(dxes, axis=a, polarity=pol, omega=omega,
                                      epsilon_effective=epsilon_effective,
                                      thickness=thickness, s_function=sf)
    return dxes
