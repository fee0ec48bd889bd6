"""The C-ABI library loads and exports every symbol ``include/tenet_b200.h`` declares (CPU)."""

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "tenet_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tnt_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from tenet_b200 import _lib

    lib = _lib.lib()
    names = declared_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    from tenet_b200 import _lib

    assert set(declared_symbols()) == set(_lib._SIGS)


def test_errors_are_reported_not_raised_across_the_abi():
    from tenet_b200 import _lib

    lib = _lib.lib()
    out = ctypes.c_void_p()
    kinds = (ctypes.c_int32 * 1)(7)
    st = lib.tnt_rule_create(1, kinds, 0, ctypes.byref(out))
    assert st == 1  # TNT_INVALID_ARGUMENT
    assert "factor kind" in _lib.last_error()


def test_version_string():
    from tenet_b200 import _lib

    assert _lib.lib().tnt_version().decode().count(".") == 2


def test_ctx_create_without_gpu_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from tenet_b200 import _lib

    out = ctypes.c_void_p()
    st = _lib.lib().tnt_ctx_create(0, ctypes.byref(out))
    assert st != 0
    assert _lib.last_error()
