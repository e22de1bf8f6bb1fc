"""Seeded problem generators: deterministic, right sizes and value ranges."""
from __future__ import annotations

import numpy

from meanas_b200 import workloads


def test_generators_are_deterministic_and_sized():
    a = workloads.aniso_blocks(shape=(48, 40, 36), pml=6)
    b = workloads.aniso_blocks(shape=(48, 40, 36), pml=6)
    assert numpy.array_equal(a.epsilon, b.epsilon)
    assert a.epsilon.size == 3 * 48 * 40 * 36
    assert set(numpy.unique(a.epsilon)) <= {1.0, 2.1, 12.1}
    assert numpy.count_nonzero(a.J) == 48 * 40
    p = workloads.dipole_core(24, pml=6)
    assert p.J.size == 3 * 24 ** 3 and numpy.count_nonzero(p.J) == 1


def test_masked_problem_avoids_conductors_at_sources():
    p = workloads.masked_large(shape=(64, 60, 48), pml=8)
    sh = (3, *p.shape)
    pec = p.pec.reshape(sh)
    pmc = p.pmc.reshape(sh)
    J = p.J.reshape(sh)
    for c, i, j, k in zip(*numpy.nonzero(J)):
        assert pec[c, i, j, k] == 0 and not pmc[:, i, j, k].any()
    assert 0.04 < (pec[0] != 0).mean() < 0.07
    assert p.mu.min() >= 1.0 and p.mu.max() <= 1.5


def test_serving_requests_cover_all_sizes():
    rng = numpy.random.default_rng(0)
    shapes = set()
    for _ in range(60):
        s = workloads.SERVING_SHAPES[int(rng.integers(len(workloads.SERVING_SHAPES)))]
        shapes.add(s)
    assert shapes == set(workloads.SERVING_SHAPES)
    r = workloads.serving_request(numpy.random.default_rng(1), shape=(32, 32, 32))
    assert numpy.count_nonzero(r.J) == 1
