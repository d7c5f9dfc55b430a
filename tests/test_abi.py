"""The C-ABI library loads and exports every symbol include/brook_b200.h declares (CPU only)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    text = open(os.path.join(ROOT, "include", "brook_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(brook_\w+)\s*\(", text)))


def test_exports_every_declared_symbol():
    from brook_b200 import _native

    lib = ctypes.CDLL(_native.LIB_PATH)
    names = declared()
    assert names, "no declarations found"
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing
    assert sorted(_native.EXPORTS) == names


def test_version_and_abi():
    from brook_b200 import _native

    assert _native.lib.brook_abi_version() == 1
    assert _native.lib.brook_version().decode() == "0.1.0"


def test_errors_without_a_gpu():
    """Null arguments are refused with BROOK_INVALID_ARGUMENT and a message; no device is touched."""
    from brook_b200 import _native

    assert _native.lib.brook_context_create(0, None) == _native.INVALID_ARGUMENT
    assert "null" in _native.lib.brook_last_error().decode()
    opts = _native.Options()
    _native.lib.brook_skeletonize_options_init(ctypes.byref(opts))
    assert opts.teasar.scale == 1.5 and opts.teasar.constant == 300 and opts.dust_threshold == 1000
    assert opts.flags == _native.FIX_BRANCHING | _native.FIX_BORDERS
    assert _native.lib.brook_skeletonize(None, None, ctypes.byref(opts), None) == _native.INVALID_ARGUMENT
