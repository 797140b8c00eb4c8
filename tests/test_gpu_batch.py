"""Batched products on the GPU: every output of a mixed batch (uneven sizes, transform
lengths 2^0 .. 2^18, squares, zero-length operands) must equal the oracle's product bit for
bit, and a CUDA-graph batch must recompute from updated inputs."""
import numpy as np
import pytest

from fast_mul_ntt_b200 import synth

pytestmark = pytest.mark.gpu


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x).view(np.int64)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint64)


def make_batch(count, lo, hi, seed, sqr_frac=0.2):
    rng = np.random.default_rng(seed)
    cases = []
    for i in range(count):
        l1 = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        l2 = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        kind = ("uniform", "ones", "sparse")[i % 3]
        a, b = synth.operands(kind, l1, l2, seed * 7919 + i)
        cases.append((a, a if rng.uniform() < sqr_frac else b))
    return cases


@pytest.fixture(params=["e32", "e64"])
def engine(request, fmn):
    """Batches on the 32-bit engine (what AUTO picks for whole products) and on the 64-bit one."""
    fmn.set_engine(fmn.ENGINE_AUTO if request.param == "e32" else fmn.ENGINE_64)
    yield request.param
    fmn.set_engine(fmn.ENGINE_AUTO)


def test_mixed_batch_matches_oracle(fmn, oracle, engine):
    import torch
    cases = make_batch(300, 1, 40000, 3)
    cases.append((synth.limbs("uniform", 5, 1), np.zeros(0, np.uint64)))   # zero product
    cases.append((synth.limbs("uniform", 1, 2), synth.limbs("uniform", 1, 3)))   # one-point transform
    jobs, outs = [], []
    for a, b in cases:
        da = _dev(a)
        db = da if b is a else _dev(b)
        out = torch.full((len(a) + len(b),), -1, dtype=torch.int64, device="cuda")
        jobs.append((da, db, out))
        outs.append(out)
    fmn.mul_batch_device(jobs)
    fmn.sync()
    for (a, b), out in zip(cases, outs):
        want = oracle.sqr(a) if b is a else oracle.mul(a, b)
        assert np.array_equal(_host(out), want), (len(a), len(b), b is a)


def test_batch_equals_per_call_on_the_mixed_size_stream(fmn, engine):
    """The configuration the batched form is measured on: each side log-uniform in
    [1000, 100000] limbs, 20% squares (a 512-product sample of it)."""
    import torch
    jobs, ref = [], []
    for op, l1, l2, seed in synth.batch_mix(512, seed=11):
        a, b = synth.operands("uniform", l1, l2, seed)
        da = _dev(a)
        db = da if op == "sqr" else _dev(b)
        out = torch.empty(l1 + l2, dtype=torch.int64, device="cuda")
        r = torch.empty_like(out)
        if op == "sqr":
            fmn.sqr_device(da, r)
        else:
            fmn.mul_device(da, db, r)
        jobs.append((da, db, out))
        ref.append(r)
    fmn.mul_batch_device(jobs)
    fmn.sync()
    for (_, _, out), r in zip(jobs, ref):
        assert torch.equal(out, r)
    # the same jobs checked and marshalled once, launched twice
    prepared = fmn.BatchJobs(jobs)
    for _ in range(2):
        for _, _, out in jobs:
            out.fill_(-1)
        fmn.mul_batch_device(prepared)
        fmn.sync()
        for (_, _, out), r in zip(jobs, ref):
            assert torch.equal(out, r)


def test_batch_graph_recomputes_updated_inputs(fmn, oracle):
    import torch
    cases = make_batch(40, 100, 30000, 5)
    jobs = []
    for a, b in cases:
        da = _dev(a)
        db = da if b is a else _dev(b)
        jobs.append((da, db, torch.empty(len(a) + len(b), dtype=torch.int64, device="cuda")))
    g = fmn.BatchGraph(jobs)
    try:
        for rnd in range(2):
            if rnd == 1:            # new operand values in the same buffers
                for (da, db, _), (a, b) in zip(jobs, cases):
                    na = synth.limbs("uniform", len(a), 10_000 + len(a))
                    da.copy_(_dev(na))
                    if db.data_ptr() != da.data_ptr():
                        db.copy_(_dev(synth.limbs("ones", len(b), 0)))
            g.launch()
            g.sync()
            for (da, db, out) in jobs:
                a = _host(da)
                want = oracle.sqr(a) if db.data_ptr() == da.data_ptr() else oracle.mul(a, _host(db))
                assert np.array_equal(_host(out), want)
    finally:
        g.close()


def test_twisted_batched_products(fmn, oracle):
    """Batched products whose coefficient count is just above a power of two run twisted (a
    cyclic transform of 2^n digits plus the product modulo X^M - c), grouped by (2^n, M),
    in the same batch as whole products and squares: by the cost model, and with every
    product that allows it forced twisted.  Every output equals the oracle."""
    import torch
    shapes = []
    for k in range(11, 17):
        shapes += [(2 ** (k - 1) + 1, 2 ** (k - 1), False), (2 ** (k - 1) + 2 ** (k - 3), 2 ** (k - 1) - 5, False),
                   (2 ** k - 3, 7 * 2 ** (k - 4), False), (2 ** (k - 1) + 3, 2 ** (k - 1) + 3, True)]
    shapes += [(1000, 1200, False), (3000, 50, False), (777, 777, True)]
    for mode in (0, 2):
        fmn.force_wrap(mode)
        try:
            twisted = sum(fmn.batch_twist_for(la, lb, sq) > 0 for la, lb, sq in shapes)
            assert twisted >= (12 if mode == 0 else 18), (mode, twisted)
            jobs, cases = [], []
            for i, (la, lb, sq) in enumerate(shapes):
                a, b = synth.operands(("uniform", "ones")[i % 2], la, lb, 900 + i)
                da = _dev(a)
                db = da if sq else _dev(b)
                out = torch.full((2 * la if sq else la + lb,), -1, dtype=torch.int64, device="cuda")
                jobs.append((da, db, out))
                cases.append((a, None if sq else b))
            fmn.mul_batch_device(jobs)
            fmn.sync()
            for (a, b), (_, _, out) in zip(cases, jobs):
                want = oracle.sqr(a) if b is None else oracle.mul(a, b)
                assert np.array_equal(_host(out), want), (mode, len(a), None if b is None else len(b))
        finally:
            fmn.force_wrap(0)
