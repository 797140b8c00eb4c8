"""Generate the golden vectors in tests/golden/golden_vectors.json.

Run in a container that has the reference mounted, after ``make -C oracle ref``:

    python tests/golden/gen_golden.py [--big]

Every output comes from the reference's own src/ abs_mul64 / abs_sqr64 compiled unmodified
(oracle/_ref/libref_fastmul.so), on operands from fast_mul_ntt_b200.synth (splitmix64).  The
file stores, per case, the SHA-256 of the little-endian output limbs, the first and last
limbs, and for small outputs the full limb list, so tests can pin any implementation
without the reference present.  ``--big`` adds the full-size configurations (minutes of CPU).
"""
import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from fast_mul_ntt_b200 import synth  # noqa: E402
from oracle.oracle import RefFastMul, RefFftSmall, Oracle  # noqa: E402

SMALL = [1, 2, 3, 4, 5, 7, 8, 9, 15, 16, 17, 31, 33, 64, 100, 255, 256, 257, 1000, 1999, 2000]
FULL_LIMIT = 64          # store every limb for outputs up to this many limbs


def digest(out):
    return hashlib.sha256(np.ascontiguousarray(out, dtype="<u8").tobytes()).hexdigest()


def record(op, kind, l1, l2, seed, out, secs):
    rec = {"op": op, "kind": kind, "len1": l1, "len2": l2, "seed": seed,
           "sha256": digest(out), "head": [f"{int(v):016x}" for v in out[:4]],
           "tail": [f"{int(v):016x}" for v in out[-4:]], "ref_seconds": round(secs, 4)}
    if len(out) <= FULL_LIMIT:
        rec["limbs"] = [f"{int(v):016x}" for v in out]
    return rec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--big", action="store_true")
    args = ap.parse_args()
    ref, fs, orc = RefFastMul(), RefFftSmall(), Oracle()
    cases = []
    for kind in ("uniform", "ones", "sparse"):
        for i, a in enumerate(SMALL):
            for j, b in enumerate(SMALL):
                if kind != "uniform" and (i + j) % 3:
                    continue
                cases.append(("mul", kind, a, b, 0))
            cases.append(("sqr", kind, a, a, 0))
    cases += [("mul", "uniform", 10000, 10000, 0), ("sqr", "uniform", 10000, 10000, 0),
              ("mul", "ones", 10000, 10000, 0), ("mul", "sparse", 10000, 10000, 0),
              ("mul", "uniform", 10000, 3, 0), ("mul", "uniform", 3, 10000, 0),
              ("mul", "uniform", 65536, 65537, 0), ("mul", "uniform", 100000, 1000, 0)]
    if args.big:
        cases += [("mul", "uniform", 1000000, 1000000, 0), ("mul", "ones", 1000000, 1000000, 0),
                  ("sqr", "uniform", 1000000, 1000000, 0),
                  ("mul", "uniform", 10000000, 10000000, 0), ("mul", "ones", 10000000, 10000000, 0),
                  ("sqr", "uniform", 10000000, 10000000, 0),
                  ("mul", "uniform", 64000000, 250000, 0), ("mul", "sparse", 64000000, 250000, 0),
                  ("mul", "uniform", 64000000, 64000000, 0), ("mul", "sparse", 64000000, 64000000, 0)]
    recs = []
    for op, kind, l1, l2, seed in cases:
        a, b = synth.operands(kind, l1, l2, seed)
        t0 = time.perf_counter()
        out = ref.sqr(a) if op == "sqr" else ref.mul(a, b)
        secs = time.perf_counter() - t0
        if l1 + l2 <= 40000:                      # cross-check the reference itself
            chk = orc.sqr(a) if op == "sqr" else orc.mul(a, b)
            alt = fs.sqr(a) if op == "sqr" else fs.mul(a, b)
            assert np.array_equal(out, chk) and np.array_equal(out, alt), (op, kind, l1, l2)
            if l1 <= 2000 and l2 <= 2000:
                sb = orc.schoolbook(a, a if op == "sqr" else b)
                assert np.array_equal(out, sb), (op, kind, l1, l2)
        recs.append(record(op, kind, l1, l2, seed, out, secs))
        if l1 + l2 > 100000:
            print(f"{op} {kind} {l1}x{l2}: {secs:.2f} s", flush=True)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_vectors.json")
    with open(path, "w") as f:
        json.dump({"generator": "reference src/ abs_mul64/abs_sqr64 compiled by oracle/Makefile",
                   "operands": "fast_mul_ntt_b200.synth.operands(kind, len1, len2, seed)",
                   "cases": recs}, f, indent=0)
    print(f"wrote {len(recs)} cases to {path}")


if __name__ == "__main__":
    main()
