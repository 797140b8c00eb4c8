"""Failure detection without a GPU fault.

* A bounded wait that expires: the CRT + carry kernel runs with one look-back tile withheld
  (tile 0 never publishes its carry), its waits give up after a few milliseconds, and the
  status word the host reads is FMN_ERR_DEVICE; the device stays usable.
* Allocation failure: forced on the host (fmn_test_fail_allocs), fmn_mul returns
  FMN_ERR_NOMEM and abs_mul64 prints the error and aborts, as the reference does when its
  allocation fails (src/fast_mul.c:320-323).  The abort runs in a child process.
* Request cancellation: requests withdrawn before admission are never computed; the rest of
  the stream is unaffected."""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

from fast_mul_ntt_b200 import synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FMN_ERR_ARG, FMN_ERR_NOMEM, FMN_ERR_DEVICE = 1, 3, 4


def test_expired_lookback_wait_reports_device_error(fmn, oracle):
    lib = fmn.load_library()
    for tiles in (2, 5):
        rc = lib.fmn_test_carry_timeout(tiles * 2048)
        assert rc == FMN_ERR_DEVICE, lib.fmn_last_error()
        assert b"bounded wait" in lib.fmn_last_error()
    assert lib.fmn_test_carry_timeout(2048) == FMN_ERR_ARG          # one tile: nothing to withhold
    a, b = synth.operands("uniform", 3000, 5000, 9)                  # the context still works
    assert np.array_equal(fmn.abs_mul64(a, b), oracle.mul(a, b))


def test_forced_allocation_failure_returns_nomem(fmn, oracle):
    lib = fmn.load_library()
    P = ctypes.POINTER(ctypes.c_uint64)
    a, b = synth.operands("uniform", 1000, 700, 11)
    out = np.zeros(1700, np.uint64)
    lib.fmn_shutdown()                     # no cached buffers: the next product must allocate
    try:
        assert lib.fmn_test_fail_allocs(1) == 0
        rc = lib.fmn_mul(a.ctypes.data_as(P), 1000, b.ctypes.data_as(P), 700, out.ctypes.data_as(P))
        assert rc == FMN_ERR_NOMEM, lib.fmn_last_error()
        assert b"cudaMalloc" in lib.fmn_last_error()
        assert not out.any()                                          # nothing was written
    finally:
        lib.fmn_test_fail_allocs(0)
    assert np.array_equal(fmn.abs_mul64(a, b), oracle.mul(a, b))     # recovers on the next call


def test_abs_mul64_aborts_on_allocation_failure():
    """The drop-in keeps the reference's contract: no status code, abort() with a message."""
    code = (
        "import sys, ctypes, numpy as np\n"
        f"sys.path.insert(0, {ROOT!r})\n"
        "import fast_mul_ntt_b200 as f\n"
        "lib = f.load_library(); f.init(0)\n"
        "lib.fmn_test_fail_allocs(1)\n"
        "a = np.arange(1, 501, dtype=np.uint64); b = np.arange(1, 301, dtype=np.uint64)\n"
        "out = np.zeros(800, np.uint64)\n"
        "P = ctypes.POINTER(ctypes.c_uint64)\n"
        "lib.abs_mul64(a.ctypes.data_as(P), 500, b.ctypes.data_as(P), 300, out.ctypes.data_as(P))\n"
        "print('returned')\n")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode != 0 and "returned" not in r.stdout
    assert r.returncode in (-6, 134), (r.returncode, r.stderr[-2000:])   # SIGABRT
    assert "abs_mul64 failed" in r.stderr and "cudaMalloc" in r.stderr


def test_server_cancel_withdraws_waiting_requests(fmn, oracle):
    import torch
    srv = fmn.Server(device=0, hbm_budget=8 << 30, max_batch=64, batching=True)
    keep, reqs, wants = [], [], []
    try:
        srv.pause(True)                                  # nothing is admitted while we cancel
        for i in range(24):
            l1, l2 = 3000 + 97 * i, 2000 + 31 * i
            a, b = synth.operands("uniform", l1, l2, 300 + i)
            da = torch.from_numpy(a.view(np.int64)).cuda()
            db = torch.from_numpy(b.view(np.int64)).cuda()
            out = torch.full((l1 + l2,), -1, dtype=torch.int64, device="cuda")
            keep += [da, db, out]
            r = fmn.FmnRequest()
            r.op, r.in1, r.len1, r.in2, r.len2 = fmn.FMN_OP_MUL, da.data_ptr(), l1, db.data_ptr(), l2
            r.out, r.tag = out.data_ptr(), i
            srv.submit(r)
            reqs.append(out)
            wants.append(oracle.mul(a, b))
        with pytest.raises(fmn.FastMulError):            # paused with requests queued
            srv.wait()
        cancelled = [i for i in range(24) if i % 3 == 0]
        for i in cancelled:
            assert srv.cancel(i)
        assert not srv.cancel(0)                         # already withdrawn
        srv.pause(False)
        srv.wait()
        st = srv.stats()
        assert st["cancelled"] == len(cancelled)
        assert st["completed"] == 24 and st["failed"] == 0 and st["device_errors"] == 0
        assert not srv.cancel(1)                         # finished: nothing to withdraw
        for i, out in enumerate(reqs):
            host = out.cpu().numpy().view(np.uint64)
            if i in cancelled:
                assert (host == np.uint64(0xFFFFFFFFFFFFFFFF)).all(), i    # never written
            else:
                assert np.array_equal(host, wants[i]), i
    finally:
        srv.close()
