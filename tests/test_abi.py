"""The C-ABI library: it loads without a GPU, exports every entry point that
include/bclx.h declares, its struct layouts agree with the header, and it
fails with a status (not a crash or a CPU fallback) when no device is there."""
import ctypes
import os
import re
import subprocess

import pytest

from bcl_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "bclx.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^BCLX_API\s+[\w\s\*]+?\b(bclx_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared()
    assert len(names) >= 14
    for name in names:
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (bclx_\w+)", out))
    assert set(names) <= exported
    assert set(_lib.SIGNATURES) == set(names)


def test_struct_layouts_match_header(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include "bclx.h"\n#include <stdio.h>\n#include <stddef.h>\n'
                   'int main(void){printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(bclx_csr_t), sizeof(bclx_spgrid_t),'
                   ' sizeof(bclx_spgrid_out_t), sizeof(bclx_dgrid_t), offsetof(bclx_csr_t, dtype),'
                   ' offsetof(bclx_spgrid_out_t, vals)); return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    want = [ctypes.sizeof(_lib.CSRDesc), ctypes.sizeof(_lib.SpGrid), ctypes.sizeof(_lib.SpGridOut),
            ctypes.sizeof(_lib.DGrid), _lib.CSRDesc.dtype.offset, _lib.SpGridOut.vals.offset]
    assert got == want


def test_version_and_invalid_arguments():
    lib = _lib.load()
    assert lib.bclx_version() >= 100
    # null handles are rejected with a status, before any device work
    assert lib.bclx_context_create(0, None) == _lib.ERR_INVALID
    assert lib.bclx_spgemm_symbolic(None, None, None, None, None, None) == _lib.ERR_INVALID
    assert lib.bclx_spmm_grid(None, None, None, None) == _lib.ERR_INVALID
    assert lib.bclx_spgemm_plan_destroy(None) == _lib.OK


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    rc = _lib.load().bclx_context_create(0, ctypes.byref(h))
    assert rc == _lib.ERR_NO_DEVICE
    with pytest.raises(RuntimeError):
        from bcl_b200.containers import Context
        Context(0)
