"""GPU parity: every product computed by the CUDA kernels through the C ABI must equal the
reference's own output bit for bit (golden vectors from the reference's src/ code), the
oracle restatement, and, at full size, the residue property mod independent primes."""
import ctypes

import numpy as np
import pytest

from fast_mul_ntt_b200 import synth
from tests.helpers import digest, operands_for, residue_check

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["e32", "e64"])
def engine(request, fmn):
    """Runs a test once per residue engine: the 32-bit-digit engine (what AUTO picks for
    these sizes) and the 64-bit engine with the reference's primes."""
    fmn.set_engine(fmn.ENGINE_32 if request.param == "e32" else fmn.ENGINE_64)
    yield request.param
    fmn.set_engine(fmn.ENGINE_AUTO)


def run(fmn, c, a, b):
    return fmn.abs_sqr64(a) if c["op"] == "sqr" else fmn.abs_mul64(a, b)


def test_golden_small_and_medium(fmn, golden, engine):
    """All golden cases up to 140k output limbs: sizes 1..2000 in every pairing pattern,
    uniform / all-ones / sparse operands, squares, 10k x 10k (transform length 2^15),
    unbalanced products and transform-length boundaries."""
    n = 0
    for c in golden:
        if c["len1"] + c["len2"] > 140000:
            continue
        a, b = operands_for(c)
        out = run(fmn, c, a, b)
        assert digest(out) == c["sha256"], (c["op"], c["kind"], c["len1"], c["len2"])
        n += 1
    assert n > 800


def test_random_shapes_vs_oracle(fmn, oracle, engine):
    """Seeded random (possibly very unbalanced) shapes against the oracle restatement."""
    rng = np.random.default_rng(2024)
    for i in range(60):
        la = int(np.exp(rng.uniform(0, np.log(300000))))
        lb = int(np.exp(rng.uniform(0, np.log(300000))))
        kind = ("uniform", "ones", "sparse")[i % 3]
        a, b = synth.operands(kind, la, lb, 100 + i)
        got = fmn.abs_mul64(a, b)
        assert np.array_equal(got, oracle.mul(a, b)), (kind, la, lb)
        if i % 4 == 0:
            assert np.array_equal(fmn.abs_sqr64(a), oracle.sqr(a)), (kind, la)


def test_transform_length_boundaries(fmn, oracle, engine):
    """conv_len = 2^k - 1, 2^k, 2^k + 1 for every k up to 2^20: each pass plan (1, 2 and 3
    passes) and its edges."""
    for k in range(0, 21):
        for conv in (2**k - 1, 2**k, 2**k + 1):
            if conv < 1:
                continue
            la = max(1, (conv + 1) // 2)
            lb = conv + 1 - la
            if lb < 1:
                continue
            a, b = synth.operands("uniform", la, lb, k)
            assert np.array_equal(fmn.abs_mul64(a, b), oracle.mul(a, b)), (k, la, lb)


def test_carry_chains(fmn, oracle, engine):
    """All-ones operands (longest carry chains) and products that are all-ones runs."""
    for n in (1, 2, 3, 1000, 4096, 65537, 300000):
        a = synth.limbs("ones", n)
        assert np.array_equal(fmn.abs_sqr64(a), oracle.sqr(a)), n
        b = np.zeros(n, np.uint64)
        b[0] = 1
        assert np.array_equal(fmn.abs_mul64(a, b), np.concatenate([a, np.zeros(n, np.uint64)]))
    # (2^(64n) - 1) * (2^(64m) + 1): long runs of propagating limbs
    a = synth.limbs("ones", 100000)
    b = np.zeros(70001, np.uint64)
    b[0] = 1
    b[-1] = 1
    assert np.array_equal(fmn.abs_mul64(a, b), oracle.mul(a, b))


def test_out_aliases_input(fmn, oracle, engine):
    """out may alias in1 (the reference copies inputs before writing out)."""
    lib = fmn.load_library()
    a, b = synth.operands("uniform", 5000, 3000, 11)
    want = oracle.mul(a, b)
    buf = np.zeros(8000, np.uint64)
    buf[:5000] = a
    p = buf.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
    lib.abs_mul64(p, 5000, b.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), 3000, p)
    assert np.array_equal(buf, want)


def test_same_block_is_square(fmn, oracle, engine):
    a = synth.limbs("uniform", 12345, 4)
    lib = fmn.load_library()
    out = np.zeros(2 * len(a), np.uint64)
    p = a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
    lib.abs_mul64(p, len(a), p, len(a), out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
    assert np.array_equal(out, oracle.sqr(a))


def test_pinned_host_buffers(fmn, oracle, engine):
    """abs_mul64 / abs_sqr64 on pinned host memory take the overlapped path (second operand
    copied while the first is transformed, output copied back in chunks)."""
    import torch
    lib = fmn.load_library()
    P = ctypes.POINTER(ctypes.c_uint64)
    for la, lb in [(600000, 700001), (5, 3), (1 << 19, 1 << 19)]:
        a, b = synth.operands("uniform", la, lb, 31)
        ha = torch.from_numpy(a.view(np.int64)).pin_memory().numpy().view(np.uint64)
        hb = torch.from_numpy(b.view(np.int64)).pin_memory().numpy().view(np.uint64)
        ho = torch.zeros(la + lb, dtype=torch.int64).pin_memory().numpy().view(np.uint64)
        lib.abs_mul64(ha.ctypes.data_as(P), la, hb.ctypes.data_as(P), lb, ho.ctypes.data_as(P))
        assert np.array_equal(ho, oracle.mul(a, b)), (la, lb)
        hs = torch.zeros(2 * la, dtype=torch.int64).pin_memory().numpy().view(np.uint64)
        lib.abs_sqr64(ha.ctypes.data_as(P), la, hs.ctypes.data_as(P))
        assert np.array_equal(hs, oracle.sqr(a)), la


def test_pageable_staging_many_chunks(fmn, oracle, engine):
    """Pageable buffers go through the lane's 4 x 8 MiB pinned slots: operands and product
    several times larger than all slots together (slot reuse in both directions), the output
    aliasing the first operand, and a square, equal to the device path's product."""
    import torch
    lib = fmn.load_library()
    P = ctypes.POINTER(ctypes.c_uint64)
    la, lb = 3_000_003, 2_500_001           # 24 + 20 MB in, 44 MB out: 3 + 3 and 6 chunks
    a, b = synth.operands("uniform", la, lb, 41)
    da = torch.from_numpy(a.view(np.int64)).cuda()
    db = torch.from_numpy(b.view(np.int64)).cuda()
    dout = torch.empty(la + lb, dtype=torch.int64, device="cuda")
    fmn.mul_device(da, db, dout)
    fmn.sync()
    want = dout.cpu().numpy().view(np.uint64)
    assert residue_check(oracle, a, b, want)
    got = fmn.abs_mul64(a, b)
    assert np.array_equal(got, want)
    buf = np.zeros(la + lb, np.uint64)
    buf[:la] = a
    p = buf.ctypes.data_as(P)
    lib.abs_mul64(p, la, b.ctypes.data_as(P), lb, p)     # void, aborts on failure
    assert np.array_equal(buf, want)
    dsq = torch.empty(2 * la, dtype=torch.int64, device="cuda")
    fmn.sqr_device(da, dsq)
    fmn.sync()
    assert np.array_equal(fmn.abs_sqr64(a), dsq.cpu().numpy().view(np.uint64))


def test_pageable_staging_threads(fmn, oracle):
    """Several host threads on pageable buffers at once: each takes its own lane and its
    own staging slots."""
    from concurrent.futures import ThreadPoolExecutor
    shapes = [(1_200_000 + 7 * i, 900_000 + 3 * i) for i in range(6)]
    ops = [synth.operands("uniform", la, lb, 50 + i) for i, (la, lb) in enumerate(shapes)]
    with ThreadPoolExecutor(4) as ex:
        outs = list(ex.map(lambda ab: fmn.abs_mul64(*ab), ops))
    for (a, b), out in zip(ops, outs):
        assert residue_check(oracle, a, b, out)
    assert np.array_equal(outs[0], fmn.abs_mul64(*ops[0]))


def test_device_api_and_caller_workspace(fmn, oracle, engine):
    import torch
    a, b = synth.operands("uniform", 70000, 50000, 21)
    want = oracle.mul(a, b)
    da = torch.from_numpy(a.view(np.int64)).cuda()
    db = torch.from_numpy(b.view(np.int64)).cuda()
    out = torch.empty(len(a) + len(b), dtype=torch.int64, device="cuda")
    fmn.mul_device(da, db, out)
    fmn.sync()
    assert np.array_equal(out.cpu().numpy().view(np.uint64), want)
    sq = torch.empty(2 * len(a), dtype=torch.int64, device="cuda")
    fmn.sqr_device(da, sq)
    fmn.sync()
    assert np.array_equal(sq.cpu().numpy().view(np.uint64), oracle.sqr(a))
    ws = torch.empty(fmn.workspace_size(len(a), len(b)), dtype=torch.uint8, device="cuda")
    out2 = torch.zeros_like(out)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        fmn.mul_device_ws(da, db, out2, ws, stream=s)
    fmn.ws_status(ws, stream=s)
    assert torch.equal(out, out2)


@pytest.mark.parametrize("op,kind,l1,l2", [
    ("mul", "uniform", 1000000, 1000000), ("mul", "ones", 1000000, 1000000), ("sqr", "uniform", 1000000, 1000000),
    ("mul", "uniform", 10000000, 10000000), ("mul", "ones", 10000000, 10000000),
    ("sqr", "uniform", 10000000, 10000000),
    ("mul", "uniform", 64000000, 250000), ("mul", "sparse", 64000000, 250000),
    ("mul", "uniform", 64000000, 64000000), ("mul", "sparse", 64000000, 64000000),
])
def test_full_size_golden(fmn, oracle, golden, op, kind, l1, l2):
    """The full-size configurations against the reference's own outputs (SHA-256 of all
    limbs) and the residue property mod three 61-bit primes, on the engine AUTO picks."""
    c = next(c for c in golden if (c["op"], c["kind"], c["len1"], c["len2"]) == (op, kind, l1, l2))
    a, b = operands_for(c)
    out = run(fmn, c, a, b)
    assert digest(out) == c["sha256"]
    assert [f"{int(v):016x}" for v in out[:4]] == c["head"]
    assert residue_check(oracle, a, b, out, sqr=(op == "sqr"))


@pytest.mark.parametrize("op,kind,l1,l2", [
    ("mul", "uniform", 1000000, 1000000), ("sqr", "uniform", 10000000, 10000000),
    ("mul", "ones", 10000000, 10000000),
])
def test_full_size_golden_64bit_engine(fmn, oracle, golden, op, kind, l1, l2):
    """Sizes that AUTO runs on the 32-bit engine, forced onto the 64-bit engine."""
    c = next(c for c in golden if (c["op"], c["kind"], c["len1"], c["len2"]) == (op, kind, l1, l2))
    a, b = operands_for(c)
    fmn.set_engine(fmn.ENGINE_64)
    try:
        out = run(fmn, c, a, b)
    finally:
        fmn.set_engine(fmn.ENGINE_AUTO)
    assert digest(out) == c["sha256"]


@pytest.mark.parametrize("kind", ["uniform", "ones"])
def test_engines_agree_at_the_32bit_limit(fmn, oracle, kind):
    """2^24 x 2^24 limbs: the largest product the 32-bit engine takes (a 2^26-digit transform
    whose coefficients come closest to the product of its primes).  Both engines must give
    the same limbs, which must pass the residue check."""
    import torch
    n = 1 << 24
    a, b = synth.operands(kind, n, n, 77)
    da = torch.from_numpy(a.view(np.int64)).cuda()
    db = torch.from_numpy(b.view(np.int64)).cuda()
    outs = []
    for eng in (fmn.ENGINE_32, fmn.ENGINE_64):
        fmn.set_engine(eng)
        try:
            assert fmn.engine_for(n, n) == eng
            o = torch.empty(2 * n, dtype=torch.int64, device="cuda")
            fmn.mul_device(da, db, o)
            fmn.sync()
            outs.append(o)
        finally:
            fmn.set_engine(fmn.ENGINE_AUTO)
    assert torch.equal(outs[0], outs[1])
    assert residue_check(oracle, a, b, outs[0].cpu().numpy().view(np.uint64))
