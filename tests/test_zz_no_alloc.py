"""The entry point that allocates nothing (fmn_mul_device_noalloc), for callers that cannot
call cudaMalloc while they run.  Its output must equal the allocating entry point's
(fmn_mul_device) bit for bit, on two calls in a row that share its fixed scratch array.
This file is collected last so that a failure here stops a run only after every other test."""
import ctypes

import numpy as np
import pytest

from fast_mul_ntt_b200 import synth

pytestmark = pytest.mark.gpu


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x).view(np.int64)).cuda()


def test_no_alloc_matches_allocating_entry_point(fmn):
    import torch
    lib = fmn.load_library()
    stream = torch.cuda.current_stream().cuda_stream
    # two calls in a row on the shared array: a larger product, then a smaller one whose
    # scratch overlaps what the first left behind
    for kind, l1, l2, seed in [("uniform", 40000, 25537, 5), ("ones", 4097, 777, 6)]:
        a, b = synth.operands(kind, l1, l2, seed)
        da, db = _dev(a), _dev(b)
        want = torch.empty(l1 + l2, dtype=torch.int64, device="cuda")
        fmn.mul_device(da, db, want)
        fmn.sync()
        got = torch.full((l1 + l2,), -1, dtype=torch.int64, device="cuda")
        rc = lib.fmn_mul_device_noalloc(da.data_ptr(), l1, db.data_ptr(), l2, got.data_ptr(), stream)
        assert rc == 0, lib.fmn_last_error()
        assert torch.equal(got, want), (kind, l1, l2)


def test_no_alloc_rejects_products_beyond_its_array(fmn):
    import torch
    lib = fmn.load_library()
    a = _dev(synth.limbs("uniform", 8, 1))
    out = torch.empty(16, dtype=torch.int64, device="cuda")
    # 40000 + 30000 limbs need a 2^17-point transform: rejected before any launch
    rc = lib.fmn_mul_device_noalloc(a.data_ptr(), 40000, a.data_ptr() + 8, 30000, out.data_ptr(),
                                    ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 5
    assert b"65536" in lib.fmn_last_error()
