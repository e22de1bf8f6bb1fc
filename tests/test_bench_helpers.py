"""bench.py's host-side helpers on CPU tensors (the same torch calls run on the GPU)."""
from __future__ import annotations

import sys

import numpy
import torch

from conftest import GOLDEN, ROOT

sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def test_field_errors_against_each_other_and_the_reference_field():
    ref = numpy.load(GOLDEN / 'dipole48.npz')['E'].astype(numpy.complex128)
    e64 = torch.as_tensor(ref)
    emix = e64 * (1 + 1e-6)
    out = bench.field_errors({'cocg': e64, 'mixed': emix}, 'dipole_core')
    assert abs(out['mixed_vs_fp64'] - 1e-6) < 1e-9
    assert out['fp64_vs_reference_qmr'] == 0.0
    assert abs(out['mixed_vs_reference_qmr'] - 1e-6) < 1e-9
    # other workloads have no stored reference field
    assert set(bench.field_errors({'cocg': e64, 'mixed': emix}, 'aniso_blocks')) == {'mixed_vs_fp64'}
    # a failure is reported, not raised
    assert 'error' in bench.field_errors({'cocg': e64, 'mixed': torch.zeros(3)}, 'aniso_blocks')


def test_workload_config_and_peaks():
    from meanas_b200 import workloads
    p = workloads.dipole_core()
    cfg = bench.workload_config('dipole_core', p)
    assert cfg['shape'] == [48, 48, 48] and cfg['unknowns'] == 3 * 48 ** 3
    peak, kind = bench.peaks()
    assert peak > 1000 and kind in ('measured', 'fallback')
    traffic, source = bench.profile_traffic('cocg_stencil_c128', 'aniso_blocks')
    assert traffic > 1e9 and source.startswith('profiles/cocg_stencil_c128_aniso160.md')
    assert bench.profile_traffic('cocg_stencil_c128', 'dipole_core') == (None, None)


def test_reference_extrapolation_and_host_description():
    assert bench.extrapolated(10.0, 0.5, 100) == 60.0
    cpu = bench.host_cpu()
    assert cpu['nproc'] >= 1
