"""CPU tests of the C ABI library: it loads without a GPU, exports every symbol that
include/fast_mul.h declares, and its host-only helpers behave.  No compute call needs a GPU."""
import ctypes
import os
import re

import numpy as np

import fast_mul_ntt_b200 as fmn
from fast_mul_ntt_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:[\w\*]+\s+)+\**(\w+)\s*\(", text, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_reference_entry_points():
    names = declared_functions()
    assert "abs_mul64" in names and "abs_sqr64" in names
    assert set(names) == set(fmn.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(fmn.LIB_PATH)
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_ntt_len_matches_int_ceil2():
    for la, lb in [(1, 1), (1, 2), (2, 2), (3, 3), (10000, 10000), (1000000, 1000000), (10**7, 10**7),
                   (64 * 10**6, 250000), (5, 0)]:
        if la + lb - 1 >= 1:
            assert fmn.ntt_len(la, lb) == synth.ntt_len(la, lb)


def test_workspace_size():
    n = synth.ntt_len(10000, 10000)
    ws = fmn.workspace_size(10000, 10000)
    assert ws >= 2 * 3 * n * 8 and ws % 256 == 0
    assert fmn.workspace_size(10000, 10000, sqr=True) < ws


def test_zero_length_products_need_no_gpu():
    a = synth.limbs("uniform", 7, 0)
    assert np.array_equal(fmn.abs_mul64(a, np.zeros(0, np.uint64)), np.zeros(7, np.uint64))
    assert len(fmn.abs_mul64(np.zeros(0, np.uint64), np.zeros(0, np.uint64))) == 0


def test_too_large_is_rejected_before_any_device_call():
    lib = fmn.load_library()
    rc = lib.fmn_mul_device(ctypes.c_void_p(16), 1 << 30, ctypes.c_void_p(32), 1 << 30, ctypes.c_void_p(64), None)
    assert rc == 5       # FMN_ERR_TOO_LARGE
    assert b"2^30" in lib.fmn_last_error()
