"""The C-ABI library (CPU only: no compute calls).

* the in-tree shared library loads and exports every function ``include/*.h`` declares,
* the ctypes table of ``fastctqw_b200._native`` binds exactly those functions,
* without an sm_100 device every handle-creating call fails loudly with FX_ERR_NODEV
  (no CPU fallback exists).
"""
import ctypes
import glob
import os
import re

import pytest

from fastctqw_b200 import _native

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DECL = re.compile(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(fx_\w+)\s*\(", re.M)


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(REPO, "include", "*.h")):
        with open(h) as f:
            text = f.read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(DECL.findall(text))
    return names


def test_header_declares_the_drop_in_entry_points():
    names = declared_functions()
    for n in ("fx_create", "fx_run_host", "fx_run_device", "fx_walk_device", "fx_free",
              "fx_destroy", "fx_last_error", "fx_get_n"):
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = _native.lib()
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_table_matches_header():
    assert set(_native.SIGNATURES) == declared_functions()


def test_library_is_built_for_sm100a_only():
    assert b"sm_100a" in _native.lib().fx_version()


@pytest.mark.skipif(_native.device_ok(), reason="a B200 is present")
def test_no_device_fails_loudly():
    h = ctypes.c_void_p()
    rc = _native.lib().fx_create(16, _native.C64, ctypes.byref(h))
    assert rc == _native.ERR_NODEV and not h.value
    with pytest.raises(RuntimeError):
        _native.Engine(16, "complex64")
    from fastctqw_b200 import fastexpm
    with pytest.raises(RuntimeError):
        fastexpm.ExpMatComplex64(8)


def test_status_codes_map_to_python_exceptions():
    for rc, exc in ((_native.ERR_TYPE, TypeError), (_native.ERR_VALUE, ValueError),
                    (_native.ERR_NONFINITE, ValueError), (_native.ERR_NOMEM, MemoryError),
                    (_native.ERR_CUDA, RuntimeError), (_native.ERR_TIMEOUT, RuntimeError),
                    (_native.ERR_SINGULAR, RuntimeError), (_native.ERR_NODEV, RuntimeError)):
        with pytest.raises(exc):
            _native.check(rc)
