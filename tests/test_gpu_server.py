"""Resident operands and the product server on the GPU.

Every product must equal the oracle's bit for bit, and the same in the mix (continuous
batching, overlapping batches) as alone; the plain per-call server must give the same
numbers; admission must respect the HBM budget."""
import ctypes

import numpy as np
import pytest

from fast_mul_ntt_b200 import synth

pytestmark = pytest.mark.gpu


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x).view(np.int64)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint64)


@pytest.fixture(params=["e32", "e64"])
def engine(request, fmn):
    """Resident spectra on the 32-bit engine (AUTO) and on the 64-bit engine (ENGINE_64 set
    while the operands are created and used)."""
    fmn.set_engine(fmn.ENGINE_AUTO if request.param == "e32" else fmn.ENGINE_64)
    yield request.param
    fmn.set_engine(fmn.ENGINE_AUTO)


def test_resident_operand_products(fmn, oracle, engine):
    import torch
    a = synth.limbs("uniform", 30000, 41)
    da = _dev(a)
    op = fmn.Operand(da, max_partner_len=50000)
    try:
        for l2, kind in [(1, "uniform"), (777, "ones"), (30000, "sparse"), (50000, "uniform")]:
            b = synth.limbs(kind, l2, l2)
            out = torch.empty(len(a) + l2, dtype=torch.int64, device="cuda")
            op.mul(_dev(b), out)
            fmn.sync()
            assert np.array_equal(_host(out), oracle.mul(a, b)), (kind, l2)
            out2 = torch.zeros_like(out)                     # again: the spectrum stays intact
            op.mul(_dev(b), out2)
            fmn.sync()
            assert torch.equal(out, out2)
    finally:
        op.close()


def _requests(fmn, oracle, count, seed, with_operand=True):
    """Mixed requests with host-side expected products: (FmnRequest list, outputs, wants)."""
    import torch
    rng = np.random.default_rng(seed)
    keep, reqs, outs, wants = [], [], [], []
    operands = []
    if with_operand:
        for k in range(2):
            a = synth.limbs("uniform", int(rng.integers(500, 20000)), 77 + k)
            da = _dev(a)
            operands.append((a, fmn.Operand(da, max_partner_len=20000), da))
    for i in range(count):
        r = fmn.FmnRequest()
        kind = rng.uniform()
        l1, l2 = int(np.exp(rng.uniform(np.log(1), np.log(20000)))), int(np.exp(rng.uniform(np.log(1), np.log(20000))))
        a, b = synth.operands(("uniform", "ones", "sparse")[i % 3], l1, l2, seed * 1000 + i)
        if with_operand and kind < 0.25:
            oa, op, _ = operands[i % len(operands)]
            db = _dev(b)
            keep.append(db)
            r.op, r.operand, r.in2, r.len2 = fmn.FMN_OP_MUL_OPERAND, op.handle.value, db.data_ptr(), l2
            want = oracle.mul(oa, b)
        elif kind < 0.55:
            da = _dev(a)
            keep.append(da)
            r.op, r.in1, r.len1 = fmn.FMN_OP_SQR, da.data_ptr(), l1
            want = oracle.sqr(a)
        else:
            da, db = _dev(a), _dev(b)
            keep += [da, db]
            r.op, r.in1, r.len1, r.in2, r.len2 = fmn.FMN_OP_MUL, da.data_ptr(), l1, db.data_ptr(), l2
            want = oracle.mul(a, b)
        out = torch.full((len(want),), -1, dtype=torch.int64, device="cuda")
        r.out = out.data_ptr()
        r.tag = i
        reqs.append(r)
        outs.append(out)
        wants.append(want)
    return reqs, outs, wants, (keep, operands)


def test_server_mix_equals_alone_and_oracle(fmn, oracle, engine):
    reqs, outs, wants, hold = _requests(fmn, oracle, 120, 3)
    srv = fmn.Server(batching=True, max_batch=32)
    try:
        for r in reqs:                     # all at once: batched, overlapping on the device
            srv.submit(r)
        srv.wait()
        mixed = [_host(o).copy() for o in outs]
        for o in outs:
            o.fill_(-1)
        for r in reqs:                     # one at a time: each alone on the device
            srv.submit(r)
            srv.wait()
        st = srv.stats()
        assert st["completed"] == 2 * len(reqs) and st["rejected"] == 0 and st["device_errors"] == 0
        assert st["batches"] > len(reqs)   # the second round ran one request per batch
        for o, m, w in zip(outs, mixed, wants):
            assert np.array_equal(m, w)
            assert np.array_equal(_host(o), w)
        done = srv.take()
        assert len(done) == 2 * len(reqs) and all(lat >= 0 for _, lat in done)
    finally:
        srv.close()
        for _, op, _ in hold[1]:
            op.close()


def test_plain_server_matches(fmn, oracle):
    reqs, outs, wants, hold = _requests(fmn, oracle, 60, 4)
    srv = fmn.Server(batching=False)
    try:
        for r in reqs:
            srv.submit(r)
        srv.wait()
        for o, w in zip(outs, wants):
            assert np.array_equal(_host(o), w)
    finally:
        srv.close()
        for _, op, _ in hold[1]:
            op.close()


def test_budget_admission(fmn, oracle):
    import torch
    big_a, big_b = synth.operands("uniform", 200000, 200000, 9)
    small_a, small_b = synth.operands("uniform", 100, 300, 10)
    tensors = [_dev(x) for x in (big_a, big_b, small_a, small_b)]
    outs = [torch.empty(400000, dtype=torch.int64, device="cuda"), torch.empty(400, dtype=torch.int64, device="cuda")]
    reqs = []
    for (da, db, out, la, lb) in [(tensors[0], tensors[1], outs[0], 200000, 200000),
                                  (tensors[2], tensors[3], outs[1], 100, 300)]:
        r = fmn.FmnRequest()
        r.op, r.in1, r.len1, r.in2, r.len2, r.out = fmn.FMN_OP_MUL, da.data_ptr(), la, db.data_ptr(), lb, out.data_ptr()
        reqs.append(r)
    srv = fmn.Server(batching=True, hbm_budget=8 << 20)    # 8 MB: the big product can never fit
    try:
        for r in reqs:
            srv.submit(r)
        srv.wait()
        st = srv.stats()
        assert st["rejected"] == 1 and st["completed"] == 2
        assert st["peak_bytes"] <= 8 << 20
        assert np.array_equal(_host(outs[1]), oracle.mul(small_a, small_b))
    finally:
        srv.close()


def test_open_loop_replay_checks_every_output(fmn, oracle):
    """A Poisson stream replayed open-loop; outputs go to server scratch and each is compared
    on the device with its expected product."""
    import torch
    reqs, outs, wants, hold = _requests(fmn, oracle, 80, 6)
    checks = [_dev(w) for w in wants]
    for r, c in zip(reqs, checks):
        r.out = None
        r.check = c.data_ptr()
    rng = np.random.default_rng(1)
    arrivals = list(np.cumsum(rng.exponential(1 / 2000.0, size=len(reqs))))
    for batching in (True, False):
        srv = fmn.Server(batching=batching, max_batch=64)
        try:
            lat, wall = srv.replay(reqs, arrivals)
            st = srv.stats()
            assert st["completed"] == len(reqs) and st["mismatches"] == 0 and st["device_errors"] == 0
            assert all(x > 0 for x in lat) and wall > 0
        finally:
            srv.close()
    bad = fmn.FmnRequest()                   # a planted wrong expectation is caught
    bad.op, bad.in1, bad.len1 = reqs[0].op, reqs[0].in1, reqs[0].len1
    bad.in2, bad.len2, bad.operand = reqs[0].in2, reqs[0].len2, reqs[0].operand
    wrong = torch.zeros_like(checks[0])
    bad.check = wrong.data_ptr()
    srv = fmn.Server(batching=True)
    try:
        srv.replay([bad], [0.0])
        assert srv.stats()["mismatches"] == 1
    finally:
        srv.close()
        for _, op, _ in hold[1]:
            op.close()
