"""The C ABI library loads, exports every function include/cee.h declares, and its host-only
parts behave without a GPU."""
import ctypes
import pathlib
import re

import numpy as np
import pytest

from cudaedgeelimination_b200 import _native, device_count

HEADER = pathlib.Path(__file__).resolve().parents[1] / "include" / "cee.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(cee_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    lib = _native.lib()
    names = declared_functions()
    assert len(names) >= 20
    missing = [name for name in names if not hasattr(lib, name)]
    assert not missing, missing


def test_abi_version():
    assert _native.lib().cee_abi_version() == 1


@pytest.mark.parametrize("k,count,expected", [(3, 4, 0xE58AF5E08D290D04), (4, 25, 0x03179E3CA191CE82),
                                              (5, 208, 0x6696DDE548591BCE)])
def test_library_templates_match_pinned_hashes(port, k, count, expected):
    mates = np.full((208, 14), 0xFF, np.uint8)
    h = ctypes.c_uint64(0)
    assert _native.lib().cee_kopt_templates(k, mates.ctypes.data_as(_native.c_u8p), ctypes.byref(h)) == count
    assert h.value == expected
    np.testing.assert_array_equal(mates[:count], port.kopt_templates(k)[0])


def test_bad_k_rejected():
    assert _native.lib().cee_kopt_templates(6, None, None) == _native.CEE_ERR_INVALID


@pytest.mark.skipif(device_count() > 0, reason="checks the no-device path")
def test_no_device_fails_loudly():
    handle = ctypes.c_void_p()
    assert _native.lib().cee_create(-1, ctypes.byref(handle)) == _native.CEE_ERR_NODEVICE
    assert b"no visible CUDA device" in _native.lib().cee_last_error(None)
    from cudaedgeelimination_b200 import Context
    with pytest.raises(_native.NativeError):
        Context(0)
