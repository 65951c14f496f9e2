"""The oracle's NTT against the reference's own CPU transform, run here.

oracle/_ref/libfidesref.so is the reference's test/cpuNTT_nega.cpp (nega_fft,
nega_fft2) and test/cpuNTT.cpp (the cyclic fft nega_fft2 calls) with
src/Math.cu, compiled unmodified from the reference tree by `make -C oracle
ref`.  FIDESlib's own check of its GPU transform (test/NTTtests.cu:933-1040,
TestLimbNTT) is:  bitrev(NTT(v)) == nega_fft2(v)  and  nega_fft2 inverts.
The same identities pin oracle.ntt here, on the reference's primes (p64 of
test/ParametrizedTest.cuh) at logN 13..16, for the forward and the inverse
transform.  The tables passed are the oracle's bit-reversed psi powers; the
reference code reads the root and its inverse from them.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from gpu_helpers import GOLD

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libfidesref.so")


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(LIB):
        r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], capture_output=True, text=True)
        if r.returncode != 0 or not os.path.exists(LIB):
            pytest.skip("reference tree not available to build oracle/_ref: " + r.stderr[-300:])
    lib = C.CDLL(LIB)
    u64p = C.POINTER(C.c_uint64)
    for fn in (lib.ref_nega_fft2, lib.ref_nega_fft):
        fn.argtypes = [u64p, C.c_int, u64p, u64p, C.c_uint64, C.c_int]
        fn.restype = None
    return lib


def _call(fn, a, psi, ipsi, p, invert):
    a = np.ascontiguousarray(a, dtype=np.uint64).copy()
    u64p = C.POINTER(C.c_uint64)
    fn(a.ctypes.data_as(u64p), len(a), psi.ctypes.data_as(u64p), ipsi.ctypes.data_as(u64p), int(p), int(invert))
    return a


def _bitrev(a):
    n = len(a)
    bits = n.bit_length() - 1
    idx = np.array([int(format(i, "0%db" % bits)[::-1], 2) for i in range(n)])
    return a[idx]


@pytest.mark.parametrize("logN", [13, 14, 15, 16])
def test_oracle_ntt_equals_reference_nega_fft2(ref, logN):
    from oracle import oracle as O

    primes = [p for p in GOLD["p64"] if (p - 1) % (2 << logN) == 0][:2]
    assert primes
    oc = O.Ctx(logN, primes, [], 1)
    rng = np.random.default_rng(logN)
    for i, p in enumerate(primes):
        psi, ipsi = oc.psi_tables(i)
        v = (rng.integers(0, 2 ** 63, size=oc.N, dtype=np.uint64) % np.uint64(p)).astype(np.uint64)
        r2 = _call(ref.ref_nega_fft2, v, psi, ipsi, p, False)
        # the reference's own round trip
        assert np.array_equal(_call(ref.ref_nega_fft2, r2, psi, ipsi, p, True), v)
        # its two CPU forms agree
        assert np.array_equal(_call(ref.ref_nega_fft, v, psi, ipsi, p, False), r2)
        # forward: evaluation order is the bit reversal of nega_fft2's output
        got = oc.ntt(v[None, :], [i])[0]
        assert np.array_equal(_bitrev(got), r2), (logN, p)
        # inverse: the oracle's INTT of an evaluation vector y equals the
        # reference's inverse of bitrev(y)
        y = (rng.integers(0, 2 ** 63, size=oc.N, dtype=np.uint64) % np.uint64(p)).astype(np.uint64)
        assert np.array_equal(oc.ntt(y[None, :], [i], inverse=True)[0],
                              _call(ref.ref_nega_fft2, _bitrev(y), psi, ipsi, p, True)), (logN, p)
