"""The C-ABI library: it loads without a GPU, exports every declared entry point,
and its ctypes mirror matches the C structures byte for byte."""
from __future__ import annotations

import re
import shutil
import subprocess
from pathlib import Path

import ctypes as C
import pytest

from conftest import ROOT

HEADER = ROOT / 'include' / 'meanas_fdfd.h'


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(fdfd_[a-z0-9_]+)\s*\(', text)))


def test_library_loads_and_exports_every_declared_symbol():
    from meanas_b200 import _lib
    lib = _lib.load()
    names = declared_functions()
    assert names, 'no declarations found'
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(_lib.EXPORTS), set(names) ^ set(_lib.EXPORTS)
    assert lib.fdfd_abi_version() == _lib.ABI_VERSION


def test_struct_layouts_match_header(tmp_path: Path):
    from meanas_b200 import _lib
    cc = shutil.which('gcc') or shutil.which('cc')
    if cc is None:
        pytest.skip('no C compiler')
    src = tmp_path / 'sz.c'
    src.write_text(f'''#include <stdio.h>
#include <stddef.h>
#include "{HEADER}"
int main(void) {{
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(fdfd_grid_desc), sizeof(fdfd_solve_opts),
         sizeof(fdfd_solve_info), offsetof(fdfd_grid_desc, epsilon), offsetof(fdfd_solve_opts, history),
         offsetof(fdfd_solve_info, residual), sizeof(fdfd_csr_desc), offsetof(fdfd_csr_desc, data),
         sizeof(fdfd_fdtd_face), sizeof(fdfd_fdtd_desc), offsetof(fdfd_fdtd_desc, face),
         sizeof(fdfd_mode_slice), offsetof(fdfd_mode_slice, mask_lo));
  return 0;
}}
''')
    exe = tmp_path / 'sz'
    subprocess.run([cc, str(src), '-o', str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [C.sizeof(_lib.GridDesc), C.sizeof(_lib.SolveOpts), C.sizeof(_lib.SolveInfo),
            _lib.GridDesc.epsilon.offset, _lib.SolveOpts.history.offset, _lib.SolveInfo.residual.offset,
            C.sizeof(_lib.CsrDesc), _lib.CsrDesc.data.offset,
            C.sizeof(_lib.FdtdFace), C.sizeof(_lib.FdtdDesc), _lib.FdtdDesc.face.offset,
            C.sizeof(_lib.ModeSlice), _lib.ModeSlice.mask_lo.offset]
    assert got == want


def test_argument_errors_need_no_gpu():
    """Calls that fail argument checks return negative codes and a message."""
    from meanas_b200 import _lib
    lib = _lib.load()
    d = _lib.GridDesc()
    d.shape[:] = (0, 4, 4)
    nbytes = C.c_size_t()
    rc = lib.fdfd_plan_workspace_bytes(C.byref(d), C.byref(nbytes))
    assert rc == -1
    assert b'shape' in lib.fdfd_last_error()
    d.shape[:] = (4, 5, 6)
    d.mu = 1  # any non-NULL pointer: only the layout is computed
    assert lib.fdfd_plan_workspace_bytes(C.byref(d), C.byref(nbytes)) == 0
    assert nbytes.value > 3 * 120 * 8
    assert lib.fdfd_plan_destroy(None) == 0


def test_csr_argument_checks_and_workspace_need_no_gpu():
    from meanas_b200 import _lib
    lib = _lib.load()
    d = _lib.CsrDesc(0, 0, None, None, None)
    nbytes = C.c_size_t()
    assert lib.fdfd_csr_solve_workspace_bytes(C.byref(d), C.byref(nbytes)) == -1
    assert b'n = 0' in lib.fdfd_last_error()
    d = _lib.CsrDesc(1000, 13000, 1, 1, 1)  # any non-NULL pointers: only the layout is computed
    assert lib.fdfd_csr_solve_workspace_bytes(C.byref(d), C.byref(nbytes)) == 0
    assert nbytes.value >= 7 * 16 * 1000


def test_no_cpu_fallback_in_product_package():
    """The product package never imports the oracle."""
    for p in (ROOT / 'meanas_b200').rglob('*.py'):
        text = p.read_text()
        assert 'from oracle' not in text and 'import oracle' not in text, p


def test_fdtd_argument_checks_need_no_gpu():
    from meanas_b200 import _lib
    lib = _lib.load()
    d = _lib.FdtdDesc()
    d.shape[:] = (4, 4, 4)
    assert lib.fdfd_fdtd_update_h(C.byref(d), 1, 1, None) == -1
    assert b'cell widths' in lib.fdfd_last_error()
    for a in range(3):
        d.dxe[a] = d.dxh[a] = 1  # any non-NULL pointer: only the checks run
    d.shape[:] = (4, 0, 4)
    assert lib.fdfd_fdtd_update_h(C.byref(d), 1, 1, None) == -1
    assert b'shape[1]' in lib.fdfd_last_error()
    d.shape[:] = (4, 4, 4)
    d.field_type = 7
    assert lib.fdfd_fdtd_update_h(C.byref(d), 1, 1, None) == -1
    assert b'type' in lib.fdfd_last_error()
    d.field_type = _lib.REAL32
    assert lib.fdfd_fdtd_update_e(C.byref(d), 1, 1, None) == -1   # E step needs epsilon
    assert b'epsilon' in lib.fdfd_last_error()
    d.form = _lib.FDTD_CPML
    d.epsilon = 1
    d.face[0][0].thickness = 9                                      # thicker than the axis
    d.face[0][0].param_e = d.face[0][0].param_h = 1
    assert lib.fdfd_fdtd_update_e(C.byref(d), 1, 1, None) == -1
    assert b'thickness' in lib.fdfd_last_error()
