"""The C-ABI library loads and exports every entry point include/mphy.h declares (no GPU needed)."""
import os
import re

import pytest

from mphyfem_b200 import _lib, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(mphy_[a-z0-9_]+)\s*\(", src))
    return names


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _lib.load()


def test_every_declared_symbol_is_exported_and_bound(lib):
    names = _declared()
    assert len(names) >= 30
    for n in sorted(names):
        assert hasattr(lib, n), n
    # the Python binding covers the same set
    assert names == set(_lib.SIGNATURES), names ^ set(_lib.SIGNATURES)


def test_api_version_and_status_strings(lib):
    assert lib.mphy_api_version() == 1
    assert lib.mphy_status_string(_lib.ERR_NEG_JACOBIAN).decode() == "negative Jacobian in an element"


def test_no_device_is_reported_not_faked(lib):
    """Without a visible GPU the context call fails loudly; nothing falls back to the CPU."""
    import ctypes as C
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    h = C.c_void_p()
    assert lib.mphy_ctx_create(0, C.byref(h)) == _lib.ERR_NO_DEVICE
