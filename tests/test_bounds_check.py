"""The bounds-check build (-DJC_BOUNDS_CHECK, libjc_layout_bc.so): every
indirect index a kernel follows (neighbour ids, body indices, tree node
indices, sort destinations) is checked before the access; a failed check
records JC_ERR_BOUNDS in the device error word and skips the access (no
trap). CPU: the build compiles and exports the same C ABI. GPU: on valid
inputs no check fires and the results are bit-exact against the oracle."""
import ctypes
import os
import re
import subprocess
import sys
from pathlib import Path

import pytest

from conftest import ROOT, _load_build_module


@pytest.fixture(scope="module")
def bc_lib():
    return _load_build_module().build(bounds_check=True)


def test_bounds_check_build_exports_the_abi(bc_lib):
    decl = re.findall(r"^\s*(?:jc_status|void|uint32_t|int32_t|uint64_t|const char\*|const uint32_t\*|jc_engine\*)"
                      r"\s+\**(jc_\w+)\(", (ROOT / "include" / "jc_layout.h").read_text(), re.M)
    assert len(decl) > 40
    L = ctypes.CDLL(str(bc_lib))
    for name in decl:
        assert hasattr(L, name), name
    L.jc_build_info.restype = ctypes.c_char_p
    assert b"bounds-check" in L.jc_build_info()


@pytest.mark.gpu
def test_bounds_check_build_is_bit_exact_and_silent(bc_lib):
    env = dict(os.environ, JC_LAYOUT_LIB=str(bc_lib))
    r = subprocess.run([sys.executable, str(Path(__file__).parent / "bounds_check_parity.py")], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "no check fired" in r.stdout
