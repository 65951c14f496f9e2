"""CPU checks of the exactness arguments behind the FP64 and tensor-core paths.

The CUDA kernels compute the same residues as the integer arithmetic only
because of value bounds (fp64.cuh, ntt.cu, conv_tc.cu).  These tests restate
the device arithmetic on the host and run it against exact integer
arithmetic on the cases the bounds are tight for:

* the double-precision NTT with the kernels' stage schedule (column pass
  centring on odd stages, row pass on even ones, doubles passed between the
  passes, one floor reduction at the end; inverse with centred sums) on primes
  just below 2^50, random residues, p-1 everywhere and alternating 0/p-1
  (tests/exact_arith_emu.c, C99 fma);
* the FP64 key-switch sums of up to 8 digit products, including maximal
  operands, and the tensor product's single products and sums of two
  (floor-reduced without centring);
* the int8-split conversion: byte layout of A and B in the canonical K-major
  shared-memory form, the matrix product of the tensor-core MMAs, the
  reassembly of V' and its one-correction Barrett step (numpy / Python ints).
The GPU parity tests then check the kernels themselves against the oracle.
"""
import ctypes
import os
import random
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _is_prime(n):
    if n < 2:
        return False
    for a in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        if n % a == 0:
            return n == a
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def _ntt_primes(top, count, two_n=1 << 17):
    out, p = [], (top - 1) // two_n * two_n + 1
    while len(out) < count:
        if p < top and _is_prime(p):
            out.append(p)
        p -= two_n
    return out


def _psi(p, two_n=1 << 17):
    rng = random.Random(p)
    while True:
        w = pow(rng.randrange(2, p - 1), (p - 1) // two_n, p)
        if pow(w, two_n // 2, p) == p - 1:
            return w


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("emu") / "libemu.so")
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-frounding-math", "-shared", "-fPIC",
                    os.path.join(HERE, "exact_arith_emu.c"), "-o", out, "-lm"], check=True)
    lib = ctypes.CDLL(out)
    lib.emu_ntt_check.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int]
    lib.emu_ntt_gen_check.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int]
    lib.emu_ntt_sg_check.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int]
    lib.emu_ks_check.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_uint64, ctypes.c_int, ctypes.c_int]
    lib.emu_tensor_check.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, ctypes.c_int]
    return lib


PRIMES_50 = _ntt_primes(1 << 50, 3) + _ntt_primes((1 << 49) + (1 << 47), 1)


@pytest.mark.parametrize("p", PRIMES_50)
def test_fp64_ntt_schedule_exact(emu, p):
    psi = _psi(p)
    for pattern in (0, 1, 2):
        assert emu.emu_ntt_check(p, psi, 1000 + pattern, pattern) == 0, pattern


@pytest.mark.parametrize("p", PRIMES_50)
def test_fp64_ntt_generated_row_twiddles_exact(emu, p):
    """Forward variant 9: the row pass forms its twiddles on the fly and
    takes their quotient companions as fl(w * pinv) (not correctly rounded),
    centring X at every row stage."""
    psi = _psi(p)
    for pattern in (0, 1, 2):
        assert emu.emu_ntt_gen_check(p, psi, 2000 + pattern, pattern) == 0, pattern


@pytest.mark.parametrize("p", PRIMES_50)
def test_fp64_ntt_staged_generated_row_twiddles_exact(emu, p):
    """Forward variant 9 and its inverse configuration: exact staged twiddles
    for the forward row pass's first four stages, products of a table entry
    and psi_br[g] (unreduced, sloppy quotient companion) for the last four,
    which centre X at every stage; the inverse row pass forms its per-thread
    twiddles the same way."""
    psi = _psi(p)
    for pattern in (0, 1, 2):
        assert emu.emu_ntt_sg_check(p, psi, 3000 + pattern, pattern) == 0, pattern


@pytest.mark.parametrize("p", PRIMES_50[:2])
def test_fp64_keyswitch_sums_exact(emu, p):
    for nd in range(1, 9):
        assert emu.emu_ks_check(p, nd, nd, 20000, 0) == 0, nd
        assert emu.emu_ks_check(p, nd, nd, 4, 1) == 0, nd


@pytest.mark.parametrize("p", PRIMES_50)
def test_fp64_tensor_products_exact(emu, p):
    """e0 = a0 b0 and e1 = a0 b1 + a1 b0 as k_tensor forms them on the FP64
    pipes: products reduced to |r| <= 0.875p, floor-reduced without centring."""
    assert emu.emu_tensor_check(p, 7, 100000, 0) == 0
    assert emu.emu_tensor_check(p, 7, 4, 1) == 0


def _conv_tc_emulate(ck, cnt, ntar, bits, seed):
    """Byte layouts, MMA and epilogue of the pre-shifted int8 conversion;
    returns the number of outputs that differ from sum_i x_i M_i mod p."""
    rnd = random.Random(seed)
    rows, lbo_a = 128, 2048
    ntar2 = (ntar + 1) & ~1
    lbo_b = ntar2 * 128
    A = np.zeros(2 * ck * lbo_a, np.uint8)
    B = np.zeros(2 * ck * lbo_b, np.uint8)
    ps = [rnd.randrange(2 ** (bits - 1), 2 ** bits) | 1 for _ in range(ntar)]
    x = [[(2 ** 62 - 1) if rnd.random() < 0.5 else rnd.randrange(2 ** 62) for _ in range(rows)] for _ in range(cnt)]
    M = [[ps[m] - 1 if rnd.random() < 0.5 else rnd.randrange(ps[m]) for m in range(ntar)] for _ in range(cnt)]
    for i in range(cnt):
        for r in range(rows):
            off = (i >> 1) * lbo_a + (r >> 3) * 128 + (r & 7) * 16 + (i & 1) * 8
            A[off:off + 8] = np.frombuffer(x[i][r].to_bytes(8, "little"), np.uint8)
    for u in range(2 * ck * ntar2):
        c, m = divmod(u, ntar2)
        mp = [0] * 16
        for h in range(2):
            i = 2 * c + h
            live = i < cnt and m < ntar
            v = M[i][m] if live else 0
            for a in range(8):
                mp[8 * h + a] = v
                if live and a < 7:
                    v = (v << 8) % ps[m]
        for sb in range(8):
            nn = m * 8 + sb
            off = c * lbo_b + (nn >> 3) * 128 + (nn & 7) * 16
            B[off:off + 16] = np.frombuffer(bytes((mp[pos] >> (8 * sb)) & 255 for pos in range(16)), np.uint8)

    def operand(buf, start, lbo, nrows):  # canonical K-major, no swizzle, K = 32 bytes
        idx = np.array([[start + (k // 16) * lbo + (r // 8) * 128 + (r % 8) * 16 + k % 16 for k in range(32)]
                        for r in range(nrows)])
        return buf[idx].astype(np.int64)

    bad, m64 = 0, (1 << 64) - 1
    for m0 in range(0, ntar2, 32):
        nt = min(32, ntar2 - m0)
        D = np.zeros((rows, nt * 8), np.int64)
        for k in range(ck):
            D += operand(A, 2 * k * lbo_a, lbo_a, rows) @ operand(B, 2 * k * lbo_b + m0 * 128, lbo_b, nt * 8).T
        assert D.max() < 2 ** 23
        for mm in range(nt):
            m = m0 + mm
            if m >= ntar:
                continue
            p = ps[m]
            mu = (1 << 80) // p
            for r in range(0, rows, 3):
                c = [int(v) for v in D[r, mm * 8:mm * 8 + 8]]
                w = [c[2 * k] + (c[2 * k + 1] << 8) for k in range(4)]
                e, o = (w[2] << 32) | w[0], (w[3] << 32) | w[1]
                q = (((e >> 16) + o) * mu) >> 64
                res = (e + ((o << 16) & m64) - q * p) & m64
                assert res < 2 * p
                res = res - p if res >= p else res
                bad += res != sum(x[i][r] * M[i][m] for i in range(cnt)) % p
    return bad


@pytest.mark.parametrize("ck,cnt,ntar,bits", [(3, 10, 30, 50), (3, 10, 39, 60), (4, 15, 25, 62), (1, 3, 9, 50)])
def test_tensor_conversion_layout_exact(ck, cnt, ntar, bits):
    assert _conv_tc_emulate(ck, cnt, ntar, bits, ck * 100 + ntar) == 0


def test_tensor_conversion_barrett_bound():
    """The reassembly and one-correction Barrett step on random and maximal
    column sums (16 limbs x 8 bytes of 255 x 255) for 18- to 62-bit primes."""
    rnd = random.Random(7)
    m64 = (1 << 64) - 1
    cmax = 16 * 8 * 255 * 255
    for trial in range(20000):
        c = [cmax if trial % 4 == 0 else rnd.randrange(cmax + 1) for _ in range(8)]
        p = rnd.randrange(2 ** (rnd.choice([18, 40, 50, 60, 62]) - 1), 2 ** 62) | 1
        p = min(p, 2 ** 62 - 1)
        v = sum(c[s] << (8 * s) for s in range(8))
        w = [c[2 * k] + (c[2 * k + 1] << 8) for k in range(4)]
        e, o = (w[2] << 32) | w[0], (w[3] << 32) | w[1]
        t = (e >> 16) + o
        assert t == v >> 16 and t < 2 ** 64
        q = (t * ((1 << 80) // p)) >> 64
        r = (e + ((o << 16) & m64) - q * p) & m64
        assert r < 2 * p
        assert (r - p if r >= p else r) == v % p
