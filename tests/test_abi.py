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


class _FakeDeviceLimbs:
    """Stands in for a CUDA tensor of int64 limbs (only what the wrapper's checks read)."""

    def __init__(self, n, cuda=True, contiguous=True, dtype=None):
        import torch
        self.n, self.is_cuda, self.contig = n, cuda, contiguous
        self.dtype = dtype or torch.int64

    def numel(self):
        return self.n

    def element_size(self):
        return self.dtype.itemsize

    def is_contiguous(self):
        return self.contig


def test_device_wrappers_check_buffers_before_any_launch():
    """The C ABI takes plain pointers and sizes, so the Python wrappers check every device
    tensor first: a short output (which the kernels would write past) and non-CUDA or
    strided tensors raise ValueError before the library is called."""
    import pytest
    import torch
    a, b = _FakeDeviceLimbs(600), _FakeDeviceLimbs(500)
    with pytest.raises(ValueError, match="needs 1100"):
        fmn.mul_device(a, b, _FakeDeviceLimbs(1099))
    with pytest.raises(ValueError, match="needs 1200"):
        fmn.sqr_device(a, _FakeDeviceLimbs(1100))
    with pytest.raises(ValueError, match="needs 1100"):
        fmn.mul_batch_device([(a, b, _FakeDeviceLimbs(1000))])
    with pytest.raises(ValueError, match="needs 1200"):
        fmn.mul_batch_device([(a, a, _FakeDeviceLimbs(1100))])
    with pytest.raises(ValueError, match="CUDA"):
        fmn.mul_device(torch.zeros(4, dtype=torch.int64), b, _FakeDeviceLimbs(504))
    with pytest.raises(ValueError, match="contiguous"):
        fmn.sqr_device(_FakeDeviceLimbs(4, contiguous=False), _FakeDeviceLimbs(8))
    with pytest.raises(ValueError, match="64-bit"):
        fmn.mul_device(_FakeDeviceLimbs(4, dtype=torch.int32), b, _FakeDeviceLimbs(504))
    with pytest.raises(ValueError, match="64-bit"):
        fmn.mul_device(_FakeDeviceLimbs(4, dtype=torch.float64), b, _FakeDeviceLimbs(504))
