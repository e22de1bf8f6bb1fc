"""Serving on the GPU: every result is the same alone and in the mix (deterministic
kernels, fixed tiling per slot), meets the FP64 residual, and slots are reused."""
from __future__ import annotations

import numpy
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(64, 64, 1), (128, 128, 1), (32, 32, 32), (40, 40, 40)]


def test_results_alone_equal_results_in_the_mix(cuda):
    from meanas_b200 import serving
    from oracle import fdfd_oracle as O
    probs = [p for _, p in serving.poisson_stream(8, rate=1e6, seed=3, shapes=SHAPES)]
    alone = []
    with serving.FDFDServer(cuda, max_active=1, precision='mixed', rtol=1e-8) as srv:
        for p in probs:
            alone.append(srv.submit(serving.Request(p.omega, p.dxes, p.J, p.epsilon)).result())
        assert srv.stats['slot_reuse'] >= 1
    with serving.FDFDServer(cuda, max_active=6, precision='mixed', rtol=1e-8) as srv:
        futs = [srv.submit(serving.Request(p.omega, p.dxes, p.J, p.epsilon)) for p in probs]
        mixed = [f.result() for f in futs]
    for p, a, m in zip(probs, alone, mixed):
        assert a.info.converged and m.info.converged
        # identical arithmetic in the same order: the same field alone and in the mix
        assert numpy.array_equal(a.E, m.E)
        res = O.true_residual(p.omega, p.dxes, p.epsilon, m.E, p.J)
        assert res <= 1.01e-8, res
    # overlap: some request started before an earlier one finished
    assert any(b.start < a.finish for a, b in zip(mixed, mixed[1:]))


def test_fp64_server_and_slot_refill(cuda):
    """A slot refilled with new problems of its size (new omega and eps) solves each
    correctly (the captured graphs are reused across them)."""
    from meanas_b200 import serving, workloads
    from oracle import fdfd_oracle as O
    rng = numpy.random.default_rng(5)
    probs = [workloads.serving_request(rng, shape=(48, 48, 1)) for _ in range(4)]
    with serving.FDFDServer(cuda, max_active=1, precision='fp64', rtol=1e-9) as srv:
        res = [srv.submit(serving.Request(p.omega, p.dxes, p.J, p.epsilon)).result() for p in probs]
        assert srv.stats['slot_new'] == 1 and srv.stats['slot_reuse'] == 3
    for p, r in zip(probs, res):
        assert r.info.converged
        assert O.true_residual(p.omega, p.dxes, p.epsilon, r.E, p.J) <= 1.01e-9
