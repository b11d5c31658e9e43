"""The C-ABI library loads and exports every entry point include/warpmd_rmsd.h
declares; argument validation that happens before any device work."""
import ctypes
import os
import re

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(REPO, "include", "warpmd_rmsd.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(wmd_[a-z_0-9]+)\s*\(", src)))


def test_header_matches_binding_list():
    from warp_md import _native

    assert set(_declared()) == set(_native.EXPORTED)


def test_library_exports_every_declared_symbol():
    from warp_md import _native

    lib = _native.load()
    for name in _declared():
        assert hasattr(lib, name), name
    assert _native.version().startswith("0.4.30")


def test_create_without_device_fails_cleanly():
    import torch

    from warp_md import _native

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    lib = _native.load()
    h = ctypes.c_void_p()
    rc = lib.wmd_create(0, ctypes.byref(h))
    assert rc == _native.WMD_ERR_NO_DEVICE
    assert b"device" in lib.wmd_last_error(None)
    with pytest.raises(_native.WarpMdError):
        _native.Context(0)


def test_null_context_is_rejected():
    from warp_md import _native

    lib = _native.load()
    assert lib.wmd_rmsd_frames(None, None, 0, 0, 3, None, 0, None, 1, None, None) == _native.WMD_ERR_INVALID_ARG
    assert lib.wmd_pairwise_rmsd(None, None, 0, 0, 3, None, 0, 0, 0, None, None) == _native.WMD_ERR_INVALID_ARG
    assert lib.wmd_destroy(None) == 0
