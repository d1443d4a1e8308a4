"""CPU tests of the C ABI: the native library builds for sm_100a, loads, and
exports every entry point that include/*.h declares.  No compute call is made
without a GPU; context creation must fail cleanly with SBG_ENODEV."""
import ctypes as C
import re
from pathlib import Path

import pytest

import simd_bigint_b200 as sbg

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    syms = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b(sbg_[a-z0-9_]+)\s*\(", text):
            syms.add(m.group(1))
    return sorted(syms)


def test_library_builds_and_loads():
    L = sbg.lib(build_if_missing=True)
    assert L is not None


def test_exports_every_declared_symbol():
    syms = declared_symbols()
    assert len(syms) >= 10
    L = C.CDLL(str(sbg.lib_path()))
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_host_only_entries():
    L = sbg.lib(build_if_missing=True)
    assert L.sbg_strerror(0) == b"ok"
    assert L.sbg_strerror(2).startswith(b"operands beyond")
    assert L.sbg_max_total_limbs() == (1 << 25) + 1


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(sbg.SbgError):
        sbg.Context(0)
