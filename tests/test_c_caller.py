"""The drop-in boundary from C: tests/c_caller.c includes include/fast_mul.h, uses malloc'd
limb buffers and calls abs_mul64 / abs_sqr64 exactly as the reference's callers call
src/fast_mul.h (bench/bench.c:32-43,86), and links against libfastmul_b200.so alone.
The link is checked on the CPU; the GPU test runs the binary and compares its output file
with the reference's own output digest."""
import os
import subprocess

import numpy as np
import pytest

from fast_mul_ntt_b200 import synth
from tests.helpers import digest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "fast_mul_ntt_b200", "lib")


def build_caller(dst):
    """gcc, the library's header and -lfastmul_b200: nothing from the package's Python side."""
    from fast_mul_ntt_b200 import build
    build.build()
    exe = os.path.join(dst, "c_caller")
    cmd = ["gcc", "-O2", "-std=c99", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "c_caller.c"), "-L" + LIBDIR, "-lfastmul_b200",
           "-Wl,-rpath," + LIBDIR, "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


def test_c_caller_compiles_and_links(tmp_path):
    exe = build_caller(str(tmp_path))
    syms = subprocess.run(["nm", "-D", "--undefined-only", exe], check=True, capture_output=True,
                          text=True).stdout
    assert "abs_mul64" in syms and "abs_sqr64" in syms


@pytest.mark.gpu
def test_c_caller_output_equals_reference(tmp_path, golden):
    exe = build_caller(str(tmp_path))
    for op, kind, l1, l2 in [("mul", "uniform", 10000, 10000), ("sqr", "uniform", 10000, 10000),
                             ("mul", "sparse", 10000, 10000), ("mul", "uniform", 100000, 1000)]:
        c = next(c for c in golden if (c["op"], c["kind"], c["len1"], c["len2"]) == (op, kind, l1, l2))
        a, b = synth.operands(kind, l1, l2, c["seed"])
        fa, fb, fo = (str(tmp_path / n) for n in ("a.bin", "b.bin", "out.bin"))
        a.astype("<u8").tofile(fa)
        b.astype("<u8").tofile(fb)
        modes = ["sqr"] if op == "sqr" else ["mul", "alias"]
        for mode in modes:
            args = [exe, mode, fa, fo] if mode == "sqr" else [exe, mode, fa, fb, fo]
            r = subprocess.run(args, capture_output=True, text=True, timeout=300)
            assert r.returncode == 0, r.stderr
            out = np.fromfile(fo, dtype="<u8")
            assert len(out) == l1 + l2
            assert digest(out) == c["sha256"], (mode, kind, l1, l2)
