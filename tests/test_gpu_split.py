"""Split products on the 32-bit engine: the shorter operand transformed once, the longer one
in pieces whose coefficients are summed before one CRT + carry pass.  Every result must equal
the oracle's bit for bit, whatever the number of pieces."""
import ctypes

import numpy as np
import pytest

from fast_mul_ntt_b200 import synth

pytestmark = pytest.mark.gpu

SHAPES = [(1000, 5000), (5000, 1000), (1, 20000), (20000, 1), (3, 100000), (50000, 50000), (12345, 67891),
          (4096, 12288), (2, 2), (999, 1001)]


@pytest.fixture
def forced(fmn):
    yield
    fmn.force_pieces(0)


@pytest.mark.parametrize("pieces", [2, 3, 7])
def test_forced_split_matches_oracle(fmn, oracle, forced, pieces):
    fmn.force_pieces(pieces)
    for i, (la, lb) in enumerate(SHAPES):
        for kind in ("uniform", "ones", "sparse"):
            a, b = synth.operands(kind, la, lb, 7 * i + pieces)
            want = oracle.mul(a, b)
            assert np.array_equal(fmn.abs_mul64(a, b), want), (pieces, kind, la, lb, fmn.pieces_for(la, lb))
    assert fmn.pieces_for(50000, 50000) == pieces


def test_split_device_api_and_workspace(fmn, oracle, forced):
    """Split products through the device API and a caller workspace of fmn_workspace_size."""
    import torch
    fmn.force_pieces(4)
    a, b = synth.operands("uniform", 30001, 200003, 5)
    want = oracle.mul(a, b)
    assert fmn.pieces_for(len(a), len(b)) == 4
    da = torch.from_numpy(a.view(np.int64)).cuda()
    db = torch.from_numpy(b.view(np.int64)).cuda()
    out = torch.empty(len(a) + len(b), dtype=torch.int64, device="cuda")
    fmn.mul_device(da, db, out)
    fmn.sync()
    assert np.array_equal(out.cpu().numpy().view(np.uint64), want)
    ws = torch.empty(fmn.workspace_size(len(a), len(b)), dtype=torch.uint8, device="cuda")
    out2 = torch.zeros_like(out)
    fmn.mul_device_ws(db, da, out2, ws)          # operands swapped: the short one is now second
    fmn.ws_status(ws)
    assert torch.equal(out, out2)


def test_split_pinned_host_buffers(fmn, oracle, forced):
    """The overlapped host path (second operand copied while the first is transformed)."""
    import torch
    fmn.force_pieces(3)
    lib = fmn.load_library()
    P = ctypes.POINTER(ctypes.c_uint64)
    for la, lb in [(700001, 60000), (60000, 700001)]:
        a, b = synth.operands("uniform", la, lb, 41)
        ha = torch.from_numpy(a.view(np.int64)).pin_memory().numpy().view(np.uint64)
        hb = torch.from_numpy(b.view(np.int64)).pin_memory().numpy().view(np.uint64)
        ho = torch.zeros(la + lb, dtype=torch.int64).pin_memory().numpy().view(np.uint64)
        lib.abs_mul64(ha.ctypes.data_as(P), la, hb.ctypes.data_as(P), lb, ho.ctypes.data_as(P))
        assert np.array_equal(ho, oracle.mul(a, b)), (la, lb)


@pytest.mark.parametrize("la,lb", [(5_000_000, 100_000), (200_000, 3_000_000)])
def test_model_split_vs_oracle(fmn, oracle, la, lb):
    """Products the cost model splits by itself."""
    assert fmn.pieces_for(la, lb) > 1
    a, b = synth.operands("uniform", la, lb, 3)
    assert np.array_equal(fmn.abs_mul64(a, b), oracle.mul(a, b))
