"""The C ABI library loads on a machine without a GPU and exports every
entry point include/tc_j2k.h declares; calls that need a device fail with a
status code rather than crashing."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from thousandthchicken_b200 import _lib as L

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    hdr = (ROOT / "include" / "tc_j2k.h").read_text()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(tc_[a-z0-9_]+)\s*\(", hdr)))


def test_header_declares_the_bound_symbols():
    assert set(declared_symbols()) == set(L.exported_symbols())


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", str(L.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (tc_[a-z0-9_]+)$", out, flags=re.M))
    missing = set(declared_symbols()) - exported
    assert not missing, missing
    lib = L.lib()
    for s in declared_symbols():
        assert getattr(lib, s) is not None


def test_status_strings_and_version():
    lib = L.lib()
    assert lib.tc_version() >= 10000
    assert lib.tc_status_string(L.TC_E_CODESTREAM) == b"malformed codestream"


def test_null_arguments_are_rejected():
    lib = L.lib()
    assert lib.tc_ctx_create(0, None, None) == L.TC_E_ARG
    assert lib.tc_j2k_read_header(None, 0, None) == L.TC_E_ARG
    assert lib.tc_t1_sort_order(None, 3, None) == L.TC_E_ARG


def test_ctx_create_without_device_fails_cleanly():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    assert L.lib().tc_ctx_create(0, None, C.byref(h)) == L.TC_E_DEVICE
    assert not h.value
