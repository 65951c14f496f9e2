"""Bit-exact parity of the CUDA path with the CPU oracle, through the C ABI.

Shapes follow FIDESlib's own tests: per-limb NTT against the CPU transform at
logN 13..16 (test/NTTtests.cu), Mult/Square/MultRescale at every level
(test/OpenFheInterfaceTests.cu), rotations and hoisted rotations, on the
reference's own prime lists (test/ParametrizedTest.cuh p64/sp64) and on the
generated moduli of the HMult workload (N=2^16, L=30, K=10, dnum=3).
"""
import ctypes as C

import numpy as np
import pytest

from gpu_helpers import device_status, from_dev, make_pair, rand_ct, rand_key, to_dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("logN", [10, 12, 13, 14, 15, 16])
def test_ntt_roundtrip_and_parity(logN):
    cc, oc = make_pair(logN, 4, 2, 2, ref_primes=True)
    nl = 6
    x = oc.random(list(range(nl)), 100 + logN)
    d = to_dev(x)
    cc.ntt(d.data_ptr(), 0, nl)
    got = from_dev(d)
    want = oc.ntt(x, list(range(nl)))
    assert np.array_equal(got, want)
    cc.ntt(d.data_ptr(), 0, nl, inverse=True)
    assert np.array_equal(from_dev(d), x)


@pytest.mark.parametrize("logN", [10, 12, 13, 14, 15, 16])
def test_every_ntt_variant_bitexact(logN):
    """Every autotuner variant (occupancy, twiddle fetch, lazy or approximate
    quotient butterflies) gives the oracle's residues, forward and inverse,
    single and batched, on 50- and 60-bit primes."""
    from pyfideslib_b200._capi import lib

    cc, oc = make_pair(logN, 8, 3, 3)
    nl = 11  # 8 ciphertext moduli (60 + 7 x 50 bits) and 3 special 60-bit moduli
    pid = list(range(nl))
    x = oc.random(pid, 900 + logN)
    want = oc.ntt(x, pid)
    xs = np.stack([x, oc.random(pid, 901 + logN)])
    want_b = [want, oc.ntt(xs[1], pid)]
    pm1 = np.array([oc.primes[i] - 1 for i in pid], dtype=np.uint64)
    x_max = np.ascontiguousarray(np.broadcast_to(pm1[:, None], x.shape))
    x_alt = x_max.copy()
    x_alt[:, ::2] = 0
    extremes = [(x_max, oc.ntt(x_max, pid)), (x_alt, oc.ntt(x_alt, pid))]
    nv = C.c_int()
    lib.fides_autotune(cc._h, None, None, C.byref(nv))
    for v in range(nv.value):
        cc.set_ntt_variant(v)
        d = to_dev(x)
        cc.ntt(d.data_ptr(), 0, nl)
        assert np.array_equal(from_dev(d), want), v
        cc.ntt(d.data_ptr(), 0, nl, inverse=True)
        assert np.array_equal(from_dev(d), x), v
        db = to_dev(np.ascontiguousarray(xs))
        cc.ntt_batch(db.data_ptr(), nl * cc.N, 2, 0, nl)
        got = from_dev(db)
        assert np.array_equal(got[0], want_b[0]) and np.array_equal(got[1], want_b[1]), v
        # the largest residues everywhere and alternating 0 / p-1 drive the
        # lazy and double-precision bounds to their worst cases
        for xe, we in extremes:
            d = to_dev(xe)
            cc.ntt(d.data_ptr(), 0, nl)
            assert np.array_equal(from_dev(d), we), v
            cc.ntt(d.data_ptr(), 0, nl, inverse=True)
            assert np.array_equal(from_dev(d), xe), v
    cc.set_ntt_variant(-1)


def test_polymul_30_limbs_n16():
    """Plain RNS polynomial multiply: N=2^16, 30 limbs (fwd NTT x2, product, INTT)."""
    import torch

    cc, oc = make_pair(16, 30, 10, 3)
    pid = list(range(30))
    a, b = oc.random(pid, 1), oc.random(pid, 2)
    da, db = to_dev(a), to_dev(b)
    dc = torch.empty_like(da)
    sa, sb = torch.empty_like(da), torch.empty_like(da)
    cc.polymul(da.data_ptr(), db.data_ptr(), dc.data_ptr(), sa.data_ptr(), sb.data_ptr(), 0, 30)
    want = oc.ntt(oc.polymul(oc.ntt(a, pid), oc.ntt(b, pid), pid), pid, inverse=True)
    assert np.array_equal(from_dev(dc), want)


@pytest.mark.parametrize("ref", [True, False])
def test_hmult_all_levels_small(ref):
    cc, oc = make_pair(12, 8, 3, 3, ref_primes=ref)
    kb, ka = rand_key(oc, 50)
    cc.upload_relin_key(kb, ka)
    for level in range(0, 8):
        a0, a1 = rand_ct(oc, level, 10 * level + 1)
        b0, b1 = rand_ct(oc, level, 10 * level + 5)
        A, B = cc.upload(a0, a1), cc.upload(b0, b1)
        for rs in ([False, True] if level > 0 else [False]):
            got = cc.EvalMult(A, B, rescale=rs).download()
            want = oc.hmult(level, a0, a1, b0, b1, kb, ka, rescale=rs)
            assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), (level, rs)


def test_square_matches_mult_self():
    cc, oc = make_pair(12, 6, 2, 2)
    kb, ka = rand_key(oc, 7)
    cc.upload_relin_key(kb, ka)
    a0, a1 = rand_ct(oc, 5, 3)
    A = cc.upload(a0, a1)
    got = cc.EvalSquare(A, rescale=True).download()
    want = oc.hmult(5, a0, a1, a0, a1, kb, ka, rescale=True)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def test_rescale_parity():
    cc, oc = make_pair(13, 6, 2, 2, ref_primes=True)
    for level in (1, 3, 5):
        c0, c1 = rand_ct(oc, level, 77 + level)
        got = cc.Rescale(cc.upload(c0, c1)).download()
        assert np.array_equal(got[0], oc.rescale(level, c0))
        assert np.array_equal(got[1], oc.rescale(level, c1))


@pytest.mark.parametrize("ks_variant", [0, 1])
def test_rotate_and_hoisted_parity(ks_variant):
    """Rotations and hoisted rotations, with the inner product's integer and
    FP64 sums."""
    from pyfideslib_b200._capi import lib

    cc, oc = make_pair(12, 8, 3, 3)
    assert lib.fides_set_keyswitch_variant(cc._h, ks_variant) == 0
    idx = [1, -1, 5, 100]
    keys = {}
    for i, r in enumerate(idx):
        g = cc.rotation_galois(r)
        keys[g] = rand_key(oc, 300 + 2 * i)
        cc.upload_galois_key(g, *keys[g])
    for level in (7, 4, 0):
        c0, c1 = rand_ct(oc, level, 900 + level)
        A = cc.upload(c0, c1)
        for r in idx:
            g = cc.rotation_galois(r)
            got = cc.EvalRotate(A, r).download()
            want = oc.rotate(level, c0, c1, pow(g, -1, 2 * oc.N), *keys[g])
            assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), (level, r)
        outs = cc.EvalFastRotation(A, idx)
        gals = [cc.rotation_galois(r) for r in idx]
        w0, w1 = oc.rotate_hoisted(level, c0, c1, [pow(g, -1, 2 * oc.N) for g in gals],
                                   [keys[g][0] for g in gals], [keys[g][1] for g in gals])
        for o, x0, x1 in zip(outs, w0, w1):
            g0, g1 = o.download()
            assert np.array_equal(g0, x0) and np.array_equal(g1, x1)


def test_every_conversion_variant_bitexact():
    """Every base-conversion variant (two coefficients per thread with 128-bit
    or split 32-bit-product sums, one coefficient per thread, the int8-split
    tensor-core ModUp and ModDown with 32 or 16 targets per MMA) gives the
    oracle's residues (HMult with and without the fused rescale and a
    rotation at two levels, moduli below 2^60)."""
    from pyfideslib_b200._capi import lib

    cc, oc = make_pair(12, 9, 3, 3)
    kb, ka = rand_key(oc, 61)
    cc.upload_relin_key(kb, ka)
    g = cc.rotation_galois(3)
    rk = rand_key(oc, 63)
    cc.upload_galois_key(g, *rk)
    for acc in (0, 1, 2, 3, 4):
        assert lib.fides_set_conv_accumulator(cc._h, acc) == 0
        for level in (8, 4):
            a0, a1 = rand_ct(oc, level, 70 + level)
            b0, b1 = rand_ct(oc, level, 80 + level)
            A, B = cc.upload(a0, a1), cc.upload(b0, b1)
            for rs in (True, False):
                got = cc.EvalMult(A, B, rescale=rs).download()
                want = oc.hmult(level, a0, a1, b0, b1, kb, ka, rescale=rs)
                assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), (acc, level, rs)
            got = cc.EvalRotate(A, 3).download()
            want = oc.rotate(level, a0, a1, pow(g, -1, 2 * oc.N), *rk)
            assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), (acc, level)
    assert lib.fides_set_conv_accumulator(cc._h, -1) == 0
    assert device_status(cc) == 0


@pytest.mark.parametrize("variant", [3, 4])
def test_tensor_conversion_every_level(variant):
    """The tensor-core conversions at every level of a small context (digits
    of 1 to 3 moduli, ModDown with and without the fused rescale, level 0
    included)."""
    from pyfideslib_b200._capi import lib

    cc, oc = make_pair(12, 8, 3, 3)
    kb, ka = rand_key(oc, 70 + variant)
    cc.upload_relin_key(kb, ka)
    assert lib.fides_set_conv_accumulator(cc._h, variant) == 0
    for level in range(0, 8):
        a0, a1 = rand_ct(oc, level, 90 + level)
        b0, b1 = rand_ct(oc, level, 95 + level)
        A, B = cc.upload(a0, a1), cc.upload(b0, b1)
        for rs in ([False, True] if level > 0 else [False]):
            got = cc.EvalMult(A, B, rescale=rs).download()
            want = oc.hmult(level, a0, a1, b0, b1, kb, ka, rescale=rs)
            assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), (level, rs)
    assert lib.fides_set_conv_accumulator(cc._h, -1) == 0
    assert device_status(cc) == 0


@pytest.mark.parametrize("dnum,variant", [(3, 3), (3, 4), (2, 3)])
def test_tensor_conversion_c2_shape_bitexact(dnum, variant):
    """The tensor-core ModUp and ModDown conversions at N=2^16, L=30, K=10
    (digits of 10 and 15 moduli, 60-bit special primes, the largest residues)
    give the oracle's HMult residues at the top, a middle and a low level."""
    from pyfideslib_b200._capi import lib

    cc, oc = make_pair(16, 30, 10, dnum)
    kb, ka = rand_key(oc, 1300 + dnum)
    cc.upload_relin_key(kb, ka)
    assert lib.fides_set_conv_accumulator(cc._h, variant) == 0
    for level in (29, 17, 2):
        a0, a1 = rand_ct(oc, level, 11 + level)
        b0, b1 = rand_ct(oc, level, 13 + level)
        if level == 29:
            pm1 = np.array([q - 1 for q in oc.primes[:level + 1]], dtype=np.uint64)[:, None]
            a0 = np.ascontiguousarray(np.broadcast_to(pm1, a0.shape))
            b1 = a0.copy()
        got = cc.EvalMult(cc.upload(a0, a1), cc.upload(b0, b1), rescale=True).download()
        want = oc.hmult(level, a0, a1, b0, b1, kb, ka, rescale=True)
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), level
    assert lib.fides_set_conv_accumulator(cc._h, -1) == 0
    assert device_status(cc) == 0


@pytest.mark.parametrize("logN,L,K,dnum", [(12, 9, 3, 3), (16, 30, 10, 3)])
def test_keyswitch_variants_bitexact(logN, L, K, dnum):
    """The key-switch inner product with 128-bit integer sums and with exact
    FP64 sums (primes below 2^50) gives the oracle's HMult residues, on random
    ciphertexts and on the largest residues with the largest key values."""
    from pyfideslib_b200._capi import lib

    cc, oc = make_pair(logN, L, K, dnum)
    kb, ka = rand_key(oc, 1400 + logN)
    pm1_all = np.array([q - 1 for q in oc.primes], dtype=np.uint64)
    kbx = np.ascontiguousarray(np.broadcast_to(pm1_all[None, :, None], kb.shape))
    level = L - 1
    a0, a1 = rand_ct(oc, level, 21)
    b0, b1 = rand_ct(oc, level, 23)
    pm1 = np.array([q - 1 for q in oc.primes[:level + 1]], dtype=np.uint64)[:, None]
    e1 = np.ascontiguousarray(np.broadcast_to(pm1, a1.shape))
    for keys, (x0, x1, y0, y1) in (((kb, ka), (a0, a1, b0, b1)), ((kbx, kbx), (a0, e1, b0, e1))):
        cc.upload_relin_key(*keys)
        want = oc.hmult(level, x0, x1, y0, y1, keys[0], keys[1], rescale=True)
        for v in (0, 1, 2, 3):
            assert lib.fides_set_keyswitch_variant(cc._h, v) == 0
            got = cc.EvalMult(cc.upload(x0, x1), cc.upload(y0, y1), rescale=True).download()
            assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), v
    assert lib.fides_set_keyswitch_variant(cc._h, 13) == 0


def test_hmult_c2_shape_bitexact():
    """HMult+Relin+Rescale at N=2^16, L=30, K=10, dnum=3, top level, one pair."""
    cc, oc = make_pair(16, 30, 10, 3)
    kb, ka = rand_key(oc, 1234)
    cc.upload_relin_key(kb, ka)
    a0, a1 = rand_ct(oc, 29, 11)
    b0, b1 = rand_ct(oc, 29, 13)
    got = cc.EvalMult(cc.upload(a0, a1), cc.upload(b0, b1), rescale=True).download()
    want = oc.hmult(29, a0, a1, b0, b1, kb, ka, rescale=True)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


@pytest.mark.parametrize("logN,L,K", [(12, 9, 3), (16, 30, 10)])
def test_fused_keyswitch_every_ntt_variant(logN, L, K):
    """The inner product fused into the digits' NTT row pass (integer and FP64
    sums) with the row-pass arithmetic of every forward NTT variant gives the
    oracle's HMult residues, at every level of a small context and at the
    top, a middle and the lowest level of the workload's, batched too."""
    from pyfideslib_b200._capi import lib

    cc, oc = make_pair(logN, L, K, 3)
    kb, ka = rand_key(oc, 1500 + logN)
    cc.upload_relin_key(kb, ka)
    levels = list(range(L)) if logN < 16 else [L - 1, 12, 0]
    raw = {lv: (rand_ct(oc, lv, 1600 + lv), rand_ct(oc, lv, 1700 + lv)) for lv in levels}
    want = {lv: oc.hmult(lv, *raw[lv][0], *raw[lv][1], kb, ka, rescale=lv > 0) for lv in levels}
    A = {lv: cc.upload(*raw[lv][0]) for lv in levels}
    B = {lv: cc.upload(*raw[lv][1]) for lv in levels}
    nv = C.c_int()
    lib.fides_autotune(cc._h, None, None, C.byref(nv))
    for v in range(nv.value):
        cc.set_ntt_variant(v)
        # 2 / 3: fused (integer / FP64 sums); 10 / 11: the same in the split
        # launch (variant 9: ciphertext-prime outputs at 3 CTAs per SM)
        for ksv in (2, 3, 10, 11):
            assert lib.fides_set_keyswitch_variant(cc._h, ksv) == 0
            for lv in levels:
                got = cc.EvalMult(A[lv], B[lv], rescale=lv > 0).download()
                assert np.array_equal(got[0], want[lv][0]) and np.array_equal(got[1], want[lv][1]), (v, ksv, lv)
            outs = cc.EvalMultBatch([A[lv] for lv in levels] * 2, [B[lv] for lv in levels] * 2, rescale=True)
            for k, lv in enumerate(levels * 2):
                if lv == 0:
                    continue
                got = outs[k].download()
                assert np.array_equal(got[0], want[lv][0]) and np.array_equal(got[1], want[lv][1]), (v, ksv, lv)
    cc.set_ntt_variant(-1)
    assert lib.fides_set_keyswitch_variant(cc._h, 13) == 0
    assert device_status(cc) == 0
