"""The entry point that allocates nothing (fmn_mul_device_noalloc), for callers that cannot
call cudaMalloc while they run (a plugin whose host application owns the device memory, a
latency-critical loop, a process with a fixed memory plan).  Its output must equal the
allocating entry point's (fmn_mul_device) bit for bit, the oracle's, and, where one exists,
the reference's own output digest, on calls in a row that share its fixed scratch array.
This file is collected last so that a failure here stops a run only after every other test."""
import ctypes

import numpy as np
import pytest

from fast_mul_ntt_b200 import synth
from tests.helpers import digest

pytestmark = pytest.mark.gpu


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x).view(np.int64)).cuda()


def _noalloc(lib, da, l1, db, l2, n_out):
    import torch
    got = torch.full((n_out,), -1, dtype=torch.int64, device="cuda")
    rc = lib.fmn_mul_device_noalloc(da.data_ptr(), l1, db.data_ptr(), l2, got.data_ptr(),
                                    ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, lib.fmn_last_error()
    return got


def test_no_alloc_matches_allocating_entry_point(fmn, oracle):
    import torch
    lib = fmn.load_library()
    # calls in a row on the shared array: the largest accepted product, then smaller ones whose
    # scratch overlaps what the earlier calls left behind, including a square (no second
    # operand's residues in the layout) right after the largest multiply
    for kind, l1, l2, seed in [("uniform", 40000, 25537, 5), ("sqr", 32768, 32768, 7), ("ones", 4097, 777, 6),
                               ("sqr", 3, 3, 8)]:
        if kind == "sqr":
            a = synth.limbs("uniform", l1, seed)
            da = db = _dev(a)
            b = a
        else:
            a, b = synth.operands(kind, l1, l2, seed)
            da, db = _dev(a), _dev(b)
        want = torch.empty(l1 + l2, dtype=torch.int64, device="cuda")
        fmn.mul_device(da, db, want)
        fmn.sync()
        got = _noalloc(lib, da, l1, db, l2, l1 + l2)
        assert torch.equal(got, want), (kind, l1, l2)
        host = got.cpu().numpy().view(np.uint64)
        ref = oracle.sqr(a) if kind == "sqr" else oracle.mul(a, b)
        assert np.array_equal(host, ref), (kind, l1, l2)


def test_no_alloc_matches_reference_digest(fmn, golden):
    """10,000 x 10,000 uniform limbs (seed 0) and its square: the reference's own output."""
    lib = fmn.load_library()
    for op in ("mul", "sqr"):
        c = next(c for c in golden if (c["op"], c["kind"], c["len1"], c["len2"]) == (op, "uniform", 10000, 10000))
        a, b = synth.operands(c["kind"], c["len1"], c["len2"], c["seed"])
        da = _dev(a)
        db = da if op == "sqr" else _dev(b)
        got = _noalloc(lib, da, c["len1"], db, c["len2"], c["len1"] + c["len2"])
        assert digest(got.cpu().numpy().view(np.uint64)) == c["sha256"], op


def test_no_alloc_zero_length_operand_gives_zero(fmn):
    import torch
    lib = fmn.load_library()
    a = _dev(synth.limbs("uniform", 1000, 3))
    got = _noalloc(lib, a, 1000, a, 0, 1000)
    assert torch.count_nonzero(got).item() == 0


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
