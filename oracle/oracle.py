"""ctypes front end of the CPU oracle (test infrastructure only).

Three checkers, all CPU:
  * ``Oracle``     -- our C restatement of the reference algorithm (oracle/fmn_oracle.c),
                      built by oracle/Makefile into oracle/_build/liboracle.so;
  * ``RefFastMul`` -- the reference's own src/fast_mul.c compiled unmodified into
                      oracle/_ref/libref_fastmul.so (present only where /root/reference was
                      available at build time; it travels as a built file);
  * ``RefFftSmall``-- the reference's fft_small/ library, the cross-check it ships.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref_fastmul.so")
FFTSMALL_SO = os.path.join(HERE, "_ref", "libref_fftsmall.so")

_u64p = ctypes.POINTER(ctypes.c_uint64)
_u64 = ctypes.c_uint64


def _ptr(a):
    return a.ctypes.data_as(_u64p)


def build(ref=False):
    """Compile the oracle (and, with ref=True, the reference) with make."""
    targets = ["all"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


def _as_limbs(x):
    x = np.ascontiguousarray(x, dtype=np.uint64)
    return x


class Oracle:
    """Our C restatement: abs_mul64 / abs_sqr64 semantics, plus schoolbook and mod checks."""

    def __init__(self):
        if not os.path.exists(ORACLE_SO):
            build(ref=False)
        lib = ctypes.CDLL(ORACLE_SO)
        lib.oracle_abs_mul64.argtypes = [_u64p, _u64, _u64p, _u64, _u64p]
        lib.oracle_abs_mul64.restype = ctypes.c_int
        lib.oracle_abs_sqr64.argtypes = [_u64p, _u64, _u64p]
        lib.oracle_abs_sqr64.restype = ctypes.c_int
        lib.oracle_schoolbook.argtypes = [_u64p, _u64, _u64p, _u64, _u64p]
        lib.oracle_schoolbook.restype = None
        lib.oracle_mod.argtypes = [_u64p, _u64, _u64]
        lib.oracle_mod.restype = _u64
        lib.oracle_constants.argtypes = [ctypes.c_int, _u64p]
        lib.oracle_crt_constants.argtypes = [_u64p]
        lib.oracle_conv_residues.argtypes = [ctypes.c_int, _u64p, _u64, _u64p, _u64, _u64, _u64p]
        lib.oracle_conv_residues.restype = ctypes.c_int
        self.lib = lib

    def mul(self, a, b):
        a, b = _as_limbs(a), _as_limbs(b)
        out = np.zeros(len(a) + len(b), dtype=np.uint64)
        if self.lib.oracle_abs_mul64(_ptr(a), len(a), _ptr(b), len(b), _ptr(out)):
            raise MemoryError("oracle allocation failed")
        return out

    def sqr(self, a):
        a = _as_limbs(a)
        out = np.zeros(2 * len(a), dtype=np.uint64)
        if self.lib.oracle_abs_sqr64(_ptr(a), len(a), _ptr(out)):
            raise MemoryError("oracle allocation failed")
        return out

    def schoolbook(self, a, b):
        a, b = _as_limbs(a), _as_limbs(b)
        out = np.zeros(len(a) + len(b), dtype=np.uint64)
        self.lib.oracle_schoolbook(_ptr(a), len(a), _ptr(b), len(b), _ptr(out))
        return out

    def mod(self, x, m):
        x = _as_limbs(x)
        return int(self.lib.oracle_mod(_ptr(x), len(x), m))

    def constants(self, i):
        out = np.zeros(5, dtype=np.uint64)
        self.lib.oracle_constants(i, _ptr(out))
        return [int(v) for v in out]

    def crt_constants(self):
        out = np.zeros(12, dtype=np.uint64)
        self.lib.oracle_crt_constants(_ptr(out))
        return [int(v) for v in out]

    def conv_residues(self, i, a, b, n):
        a, b = _as_limbs(a), _as_limbs(b)
        out = np.zeros(n, dtype=np.uint64)
        if self.lib.oracle_conv_residues(i, _ptr(a), len(a), _ptr(b), len(b), n, _ptr(out)):
            raise MemoryError("oracle allocation failed")
        return out


class _RefLib:
    SO = None
    PREFIX = None

    @classmethod
    def available(cls):
        return os.path.exists(cls.SO)

    def __init__(self):
        if not self.available():
            raise FileNotFoundError(self.SO)
        lib = ctypes.CDLL(self.SO)
        self._mul = getattr(lib, self.PREFIX + "abs_mul64")
        self._mul.argtypes = [_u64p, _u64, _u64p, _u64, _u64p]
        self._mul.restype = None
        self._sqr = getattr(lib, self.PREFIX + "abs_sqr64")
        self._sqr.argtypes = [_u64p, _u64, _u64p]
        self._sqr.restype = None
        self.lib = lib

    def mul(self, a, b, out=None):
        a, b = _as_limbs(a), _as_limbs(b)
        if a.ctypes.data == b.ctypes.data:      # in1 != in2 is a precondition (src/fast_mul.h:37)
            b = b.copy()
        if out is None:
            out = np.zeros(len(a) + len(b), dtype=np.uint64)
        self._mul(_ptr(a), len(a), _ptr(b), len(b), _ptr(out))
        return out

    def sqr(self, a, out=None):
        a = _as_limbs(a)
        if out is None:
            out = np.zeros(2 * len(a), dtype=np.uint64)
        self._sqr(_ptr(a), len(a), _ptr(out))
        return out


class RefFastMul(_RefLib):
    """The reference's src/ abs_mul64 / abs_sqr64, compiled unmodified (single-threaded)."""
    SO = REF_SO
    PREFIX = "ref_"


class RefFftSmall(_RefLib):
    """The reference's fft_small/ abs_mul64 / abs_sqr64 (the cross-check library it ships)."""
    SO = FFTSMALL_SO
    PREFIX = "fs_"
