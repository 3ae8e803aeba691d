"""The C ABI library: it loads, exports every symbol the header declares, and
fails cleanly (no GPU needed)."""
import ctypes
import os
import re

import pytest

from fomo_julia_b200 import _lib, build

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(REPO, "include", "fomo_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(fomo_b200_\w+)\s*\(", src, re.M)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _lib.load()


def test_every_declared_symbol_is_exported(lib):
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(_lib.SIGNATURES), "ctypes signature table out of sync with the header"


def test_calls_before_init_fail_cleanly(lib):
    h = ctypes.c_uint64(0)
    rc = lib.fomo_b200_alloc(16, ctypes.byref(h))
    assert rc == -7  # FOMO_ENOINIT
    assert b"fomo_b200_init" in lib.fomo_b200_last_error()
    assert lib.fomo_b200_medium_destroy(1) == -7
    assert lib.fomo_b200_version() >= 100


def test_init_without_gpu_reports_error(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    rc = lib.fomo_b200_init(0)
    assert rc in (-1, -3)
    assert lib.fomo_b200_last_error()
