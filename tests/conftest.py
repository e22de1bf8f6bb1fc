"""Shared fixtures: the golden vectors made by tests/golden/make_golden.py."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / 'tests' / 'golden'
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200)')


def unpack_dxes(z, prefix: str):
    return [[z[f'{prefix}dx{g}{a}'] for a in range(3)] for g in range(2)]


def golden_cases(name: str) -> list[dict]:
    """All cases of a golden file as dicts with 'dxes' unpacked."""
    z = numpy.load(GOLDEN / f'{name}.npz')
    n = int(z['n'])
    cases = []
    for i in range(n):
        p = f'c{i}_'
        d = {k[len(p):]: z[k] for k in z.files if k.startswith(p)}
        d['dxes'] = unpack_dxes(z, p)
        d['index'] = i
        cases.append(d)
    return cases


@pytest.fixture(scope='session')
def cuda():
    torch = pytest.importorskip('torch')
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return torch.device('cuda', 0)
