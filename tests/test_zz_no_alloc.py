"""fdfd_residual_static: the FP64 residual check for callers that cannot allocate
device memory (their allocator is exhausted or frozen, or the host program owns
every device buffer and passes only inputs and outputs).  It keeps its reduction
scratch in a fixed array inside the library instead of a caller workspace; its
results must equal those of fdfd_residual, call after call."""
from __future__ import annotations

import ctypes as C

import numpy
import pytest

pytestmark = pytest.mark.gpu


def _with_workspace(lib, op, E, J):
    import torch
    nbytes = C.c_size_t()
    assert lib.fdfd_residual_workspace_bytes(op.plan, C.byref(nbytes)) == 0
    ws = torch.empty(int(nbytes.value), dtype=torch.uint8, device=op.device)
    out = (C.c_double * 4)()
    rc = lib.fdfd_residual(op.plan, E.data_ptr(), J.data_ptr(), out, ws.data_ptr(), nbytes.value,
                           torch.cuda.current_stream().cuda_stream)
    assert rc == 0, lib.fdfd_last_error()
    return numpy.array(list(out))


def _static(lib, op, E, J):
    import torch
    out = (C.c_double * 4)()
    rc = lib.fdfd_residual_static(op.plan, E.data_ptr(), J.data_ptr(), out,
                                  torch.cuda.current_stream().cuda_stream)
    assert rc == 0, lib.fdfd_last_error()
    return numpy.array(list(out))


def test_static_residual_matches_workspace_residual(cuda):
    import torch
    from meanas_b200 import _lib, workloads
    from meanas_b200.operators import GridOperator
    lib = _lib.load()
    p = workloads.aniso_blocks(shape=(48, 40, 36), pml=6)
    op = GridOperator(p.omega, p.dxes, p.epsilon, device=cuda)
    J = torch.as_tensor(p.J, device=cuda)
    E, info = op.solve(J, rtol=1e-6, criterion='true')
    g = torch.Generator(device=cuda).manual_seed(0)
    E_noisy = E + 1e-3 * torch.randn(p.n_unknowns, dtype=torch.complex128, device=cuda, generator=g)
    results = {}
    for name, field in (('solved', E), ('noisy', E_noisy)):
        ref = _with_workspace(lib, op, field, J)
        first = _static(lib, op, field, J)
        second = _static(lib, op, field, J)
        for got in (first, second):
            # the same kernel and reduction order: equal to 1e-12 of each norm
            assert numpy.allclose(got, ref, rtol=1e-12, atol=0), (got, ref)
        results[name] = first
    solved = results['solved']
    assert solved[2] > 0 and solved[0] / solved[2] <= 1e-6 * 1.01  # ||b0 - A0 E|| / ||b0||
    assert info.converged


def test_static_residual_rejects_grids_beyond_its_scratch(cuda):
    import torch
    from meanas_b200 import _lib
    from meanas_b200.operators import GridOperator
    from meanas_b200.scpml import stretch_all_faces
    lib = _lib.load()
    # one partial sum per (8-plane block, 32 x 8 y/z tile): a single x plane of
    # 1024 x 8192 cells has 128 x 256 = 32768 of them, past the 32752 the scratch holds
    shape = (1, 1024, 8192)
    n = 3 * int(numpy.prod(shape))
    op = GridOperator(2 * numpy.pi / 20, stretch_all_faces(shape, 2 * numpy.pi / 20, 0),
                      torch.ones(n, dtype=torch.float64, device=cuda), device=cuda, fp32=False)
    E = torch.zeros(n, dtype=torch.complex128, device=cuda)
    out = (C.c_double * 4)()
    rc = lib.fdfd_residual_static(op.plan, E.data_ptr(), E.data_ptr(), out,
                                  torch.cuda.current_stream().cuda_stream)
    assert rc == -1
    assert b'32768 partial sums' in lib.fdfd_last_error()
