"""Seeded synthetic FDFD problems with the shapes and value ranges of the benchmark cases.

Every generator returns a :class:`Problem` whose arrays are in the layout the
reference's ``generic()`` takes (``meanas/fdfd/solvers.py:66-79``): 1D C-order
vectors of length ``3*X*Y*Z`` (``meanas/fdmath/vectorization.py:51-68``) and
``dxes = [[dx_e, dy_e, dz_e], [dx_h, dy_h, dz_h]]``.  PMLs are built with one
``stretch_with_scpml`` call per face, ``s_function = prepare_s_function(ln_R=-16,
m=3.5)``.

Problems:

* ``dipole_core``      48^3 point dipole in a slab-waveguide core (reference CPU case).
* ``aniso_blocks``     160x160x128 diagonal-anisotropic random blocks + Gaussian Jy plane.
* ``serving_request``  one request of the mixed-size serving stream.
* ``adjoint_design``   96x96x64 waveguide with a 40x40x8 random design region.
* ``masked_large``     320x320x200 with eps, mu, PEC and PMC (61.4M unknowns).
"""
from __future__ import annotations

import dataclasses
from typing import Any

import numpy
from numpy.typing import NDArray

from .scpml import stretch_all_faces


@dataclasses.dataclass
class Problem:
    name: str
    shape: tuple[int, int, int]
    omega: complex
    dxes: list[list[NDArray]]
    J: NDArray            # (3N,) complex128
    epsilon: NDArray      # (3N,) float64
    mu: NDArray | None = None
    pec: NDArray | None = None
    pmc: NDArray | None = None
    pml: int = 0
    extra: dict[str, Any] = dataclasses.field(default_factory=dict)

    @property
    def n_cells(self) -> int:
        return int(numpy.prod(self.shape))

    @property
    def n_unknowns(self) -> int:
        return 3 * self.n_cells


def _fill_blocks(rng: numpy.random.Generator, field: NDArray, lo: tuple[int, int, int],
                 hi: tuple[int, int, int], side: tuple[int, int], fill: float,
                 draw) -> NDArray:
    """Paint random axis-aligned boxes (per-axis side in ``side``) inside ``[lo, hi)``
    until ``fill`` of that region is covered; ``draw()`` gives each box's per-component values."""
    covered = numpy.zeros(field.shape[1:], dtype=bool)
    region = tuple(slice(a, b) for a, b in zip(lo, hi))
    target = fill * covered[region].size
    n_covered = 0
    while n_covered < target:
        size = rng.integers(side[0], side[1] + 1, size=3)
        size = numpy.minimum(size, numpy.array(hi) - numpy.array(lo))
        start = [int(rng.integers(l, h - s + 1)) for l, h, s in zip(lo, hi, size)]
        sl = tuple(slice(s, s + n) for s, n in zip(start, size))
        vals = draw()
        for c in range(field.shape[0]):
            field[(c, *sl)] = vals[c]
        n_covered += int((~covered[sl]).sum())
        covered[sl] = True
    return field


def dipole_core(n: int = 48, pml: int = 10, wavelength: float = 30.0) -> Problem:
    """Unit Jz dipole at the centre of an ``n^3`` grid; core eps=12.1 spanning x, 10 cells in y, 4 in z."""
    shape = (n, n, n)
    omega = 2 * numpy.pi / wavelength
    dxes = stretch_all_faces(shape, omega, pml)
    eps = numpy.ones((3, *shape))
    c = n // 2
    eps[:, :, c - 5:c + 5, c - 2:c + 2] = 12.1
    J = numpy.zeros((3, *shape), dtype=complex)
    J[2, c, c, c] = 1
    return Problem('dipole_core', shape, omega, dxes, J.ravel(), eps.ravel(), pml=pml)


def aniso_blocks(shape: tuple[int, int, int] = (160, 160, 128), pml: int = 12,
                 wavelength: float = 24.0, seed: int = 0, fill: float = 0.30) -> Problem:
    """Diagonal anisotropic eps in {1, 2.1, 12.1} on random 8-20 cell blocks (30% of the
    non-PML interior) and a Gaussian (sigma=6 cells) Jy plane source at z=20."""
    rng = numpy.random.default_rng(seed)
    omega = 2 * numpy.pi / wavelength
    dxes = stretch_all_faces(shape, omega, pml)
    eps = numpy.ones((3, *shape))
    levels = numpy.array([1.0, 2.1, 12.1])
    lo = (pml, pml, pml)
    hi = tuple(s - pml for s in shape)
    _fill_blocks(rng, eps, lo, hi, (8, 20), fill, lambda: rng.choice(levels, size=3))
    X, Y, Z = shape
    x = numpy.arange(X)[:, None]
    y = numpy.arange(Y)[None, :]
    sigma = 6.0
    g = numpy.exp(-((x - X // 2) ** 2 + (y - Y // 2) ** 2) / (2 * sigma ** 2))
    J = numpy.zeros((3, *shape), dtype=complex)
    J[1, :, :, 20] = g
    return Problem('aniso_blocks', shape, omega, dxes, J.ravel(), eps.ravel(), pml=pml,
                   extra=dict(seed=seed, fill=fill))


SERVING_SHAPES = [(128, 128, 1), (256, 256, 1), (512, 512, 1), (1024, 1024, 1),
                  (32, 32, 32), (64, 64, 64), (96, 96, 96), (128, 128, 128)]


def serving_request(rng: numpy.random.Generator, shape: tuple[int, int, int] | None = None,
                    pml: int = 10) -> Problem:
    """One serving request: a random grid size, lambda ~ U[16, 40] cells, random eps blocks in
    [1, 12.1] (constant per block) and a random-component dipole outside the PML."""
    if shape is None:
        shape = SERVING_SHAPES[int(rng.integers(len(SERVING_SHAPES)))]
    shape = tuple(int(s) for s in shape)
    wavelength = float(rng.uniform(16, 40))
    omega = 2 * numpy.pi / wavelength
    dxes = stretch_all_faces(shape, omega, pml)
    eps = numpy.ones((3, *shape))
    lo = tuple(pml if s > 1 else 0 for s in shape)
    hi = tuple(s - pml if s > 1 else 1 for s in shape)
    lo_side = max(2, min(s for s in numpy.array(hi) - numpy.array(lo) if s > 1) // 12)
    side = (lo_side, 3 * lo_side)

    def draw():
        v = rng.uniform(1.0, 12.1)
        return (v, v, v)
    _fill_blocks(rng, eps, lo, hi, side, 0.25, draw)
    J = numpy.zeros((3, *shape), dtype=complex)
    pos = tuple(int(rng.integers(l, h)) for l, h in zip(lo, hi))
    comp = int(rng.integers(3)) if shape[2] > 1 else 2
    J[(comp, *pos)] = 1.0
    return Problem('serving_request', shape, omega, dxes, J.ravel(), eps.ravel(), pml=pml,
                   extra=dict(wavelength=wavelength))


def adjoint_design(shape: tuple[int, int, int] = (96, 96, 64), pml: int = 10,
                   wavelength: float = 26.0, seed: int = 0,
                   design: tuple[int, int, int] = (40, 40, 8), source_x: int = 20,
                   monitor_x: int = 76) -> Problem:
    """Waveguide core (12.1, full x, 10 cells in y, 4 in z) with a centred random design region
    (eps ~ U[1, 12.1], same value on the three components of a cell); Jz dipole at x=20;
    the loss is sum |E|^2 over the plane x=76."""
    rng = numpy.random.default_rng(seed)
    omega = 2 * numpy.pi / wavelength
    dxes = stretch_all_faces(shape, omega, pml)
    X, Y, Z = shape
    eps = numpy.ones((3, *shape))
    cy, cz = Y // 2, Z // 2
    eps[:, :, cy - 5:cy + 5, cz - 2:cz + 2] = 12.1
    d0 = tuple((s - d) // 2 for s, d in zip(shape, design))
    dsl = tuple(slice(a, a + d) for a, d in zip(d0, design))
    vals = rng.uniform(1.0, 12.1, size=design)
    for c in range(3):
        eps[(c, *dsl)] = vals
    J = numpy.zeros((3, *shape), dtype=complex)
    J[2, source_x, cy, cz] = 1.0
    design_mask = numpy.zeros(shape, dtype=bool)
    design_mask[dsl] = True
    monitor = numpy.zeros((3, *shape), dtype=bool)
    monitor[:, monitor_x, :, :] = True
    return Problem('adjoint_design', shape, omega, dxes, J.ravel(), eps.ravel(), pml=pml,
                   extra=dict(design_mask=design_mask, design_slices=dsl,
                              monitor=monitor.ravel(), seed=seed))


def masked_large(shape: tuple[int, int, int] = (320, 320, 200), pml: int = 16,
                 wavelength: float = 20.0, seed: int = 0) -> Problem:
    """Diagonal eps in [1, 12.1] and mu in [1, 1.5] on random blocks; PEC 2-cell slabs on ~5%
    of cells and PMC on ~2% (both per component, outside the PML); 3 random dipoles that
    avoid PEC/PMC cells and the PML."""
    rng = numpy.random.default_rng(seed)
    omega = 2 * numpy.pi / wavelength
    dxes = stretch_all_faces(shape, omega, pml)
    lo = (pml, pml, pml)
    hi = tuple(s - pml for s in shape)
    eps = numpy.ones((3, *shape))
    _fill_blocks(rng, eps, lo, hi, (8, 24), 0.30, lambda: rng.uniform(1.0, 12.1, size=3))
    mu = numpy.ones((3, *shape))
    _fill_blocks(rng, mu, lo, hi, (8, 24), 0.15, lambda: rng.uniform(1.0, 1.5, size=3))

    def slabs(frac: float) -> NDArray:
        m = numpy.zeros((3, *shape))
        n_target = frac * numpy.prod(shape)
        cov = numpy.zeros(shape, dtype=bool)
        n_cov = 0
        while n_cov < n_target:
            ax = int(rng.integers(3))
            size = [int(rng.integers(8, 33)) for _ in range(3)]
            size[ax] = 2
            start = [int(rng.integers(l, h - s + 1)) for l, h, s in zip(lo, hi, size)]
            sl = tuple(slice(s, s + n) for s, n in zip(start, size))
            m[(slice(None), *sl)] = 1.0
            n_cov += int((~cov[sl]).sum())
            cov[sl] = True
        return m
    pec = slabs(0.05)
    pmc = slabs(0.02)
    J = numpy.zeros((3, *shape), dtype=complex)
    placed = 0
    while placed < 3:
        c = int(rng.integers(3))
        pos = tuple(int(rng.integers(l, h)) for l, h in zip(lo, hi))
        if pec[(c, *pos)] or pmc[:, pos[0], pos[1], pos[2]].any():
            continue
        J[(c, *pos)] = 1.0
        placed += 1
    return Problem('masked_large', shape, omega, dxes, J.ravel(), eps.ravel(), mu=mu.ravel(),
                   pec=pec.ravel(), pmc=pmc.ravel(), pml=pml, extra=dict(seed=seed))


BY_NAME = {
    'dipole_core': dipole_core,
    'aniso_blocks': aniso_blocks,
    'adjoint_design': adjoint_design,
    'masked_large': masked_large,
}
