"""Raw-residue interop through the C ABI: ciphertexts, plaintexts and switching
keys in the shapes FIDESlib exchanges with OpenFHE (RawCipherText,
RawPlainText, RawKeySwitchKey; src/CKKS/openfhe-interface/RawCiphertext.cuh:19-93).

A raw ciphertext pair and a raw relinearisation key (its limbs in a shuffled
modulus order, matched by modulus as loadDecompDigit does) go in, HMult +
relinearisation + rescale runs, the raw result comes out and equals the
oracle's residues bit for bit; COEFFICIENT-format limbs are transformed on the
way in and out; bad moduli and non-canonical residues are refused.
"""
import numpy as np
import pytest

from gpu_helpers import make_pair, rand_ct, rand_key

pytestmark = pytest.mark.gpu

BAD_ARG = 1


def _raw_key(oc, kb, ka, rng):
    """RawKeySwitchKey layout: r_key[h][d][i], h = 0 the a half, 1 the b half,
    limbs of each digit polynomial in a shuffled order with their moduli."""
    np_ = oc.L + oc.K
    r_key, r_mod = [], []
    for half in (ka, kb):
        hk, hm = [], []
        for d in range(oc.dnum):
            order = rng.permutation(np_)
            hk.append([half[d, i] for i in order])
            hm.append([oc.primes[i] for i in order])
        r_key.append(hk)
        r_mod.append(hm)
    return r_key, r_mod


@pytest.mark.parametrize("logN,L,K", [(12, 8, 3), (16, 30, 10)])
def test_raw_ciphertexts_and_key_hmult_bitexact(logN, L, K):
    from pyfideslib_b200._capi import FidesError

    cc, oc = make_pair(logN, L, K, 3)
    rng = np.random.default_rng(logN)
    kb, ka = rand_key(oc, 5100)
    r_key, r_mod = _raw_key(oc, kb, ka, rng)
    cc.import_raw_key(0, r_key, r_mod)
    back, back_mod = cc.export_raw_key(0)
    assert np.array_equal(back[0], ka) and np.array_equal(back[1], kb)
    assert [int(x) for x in back_mod[0, 0]] == oc.primes
    level = L - 2
    (a0, a1), (b0, b1) = rand_ct(oc, level, 5200), rand_ct(oc, level, 5210)
    mod = oc.primes[:level + 1]
    A = cc.import_raw_ct(list(a0), list(a1), mod, noise=2.0 ** 40, noise_level=1, slots=cc.N // 4)
    B = cc.import_raw_ct(list(b0), list(b1), mod, noise=2.0 ** 40, noise_level=1, slots=cc.N // 4)
    out = cc.EvalMult(A, B, rescale=True)
    s0, s1, m, noise, nl, slots = cc.export_raw_ct(out)
    w0, w1 = oc.hmult(level, a0, a1, b0, b1, kb, ka, rescale=True)
    assert np.array_equal(np.stack(s0), w0) and np.array_equal(np.stack(s1), w1)
    assert m == oc.primes[:level] and nl == 1 and slots == cc.N // 4
    assert noise == pytest.approx(2.0 ** 80 / oc.primes[level], rel=1e-12)
    # COEFFICIENT format: the limbs are transformed on the device, both ways
    c0, c1 = oc.ntt(a0, list(range(level + 1)), inverse=True), oc.ntt(a1, list(range(level + 1)), inverse=True)
    Ac = cc.import_raw_ct(list(c0), list(c1), mod, fmt=cc.FORMAT_COEFFICIENT)
    g0, g1 = Ac.download()
    assert np.array_equal(g0, a0) and np.array_equal(g1, a1)
    e0, e1, *_ = cc.export_raw_ct(A, fmt=cc.FORMAT_COEFFICIENT)
    assert np.array_equal(np.stack(e0), c0) and np.array_equal(np.stack(e1), c1)
    # refused: a limb whose modulus is not the context's, and a residue >= q
    bad_mod = list(mod)
    bad_mod[1], bad_mod[2] = bad_mod[2], bad_mod[1]
    with pytest.raises(FidesError) as e:
        cc.import_raw_ct(list(a0), list(a1), bad_mod)
    assert e.value.status == BAD_ARG
    big = a0.copy()
    big[3, 17] = oc.primes[3]
    with pytest.raises(FidesError) as e:
        cc.import_raw_ct(list(big), list(a1), mod)
    assert e.value.status == BAD_ARG
    bad_key = [[list(limbs) for limbs in h] for h in r_key]
    bad_key[1][0][5] = np.full(cc.N, r_mod[1][0][5], dtype=np.uint64)
    with pytest.raises(FidesError) as e:
        cc.import_raw_key(0, bad_key, r_mod)
    assert e.value.status == BAD_ARG


def test_raw_plaintext_mult():
    """A raw plaintext multiplies a ciphertext like the oracle's limb-wise product."""
    cc, oc = make_pair(12, 8, 3, 3)
    level = 5
    c0, c1 = rand_ct(oc, level, 5300)
    pid = list(range(level + 1))
    m = oc.random(pid, 5310)
    import pyfideslib_b200 as F
    from pyfideslib_b200._capi import check, lib

    pt = cc.import_raw_pt(list(m), oc.primes[:level + 1])

    ct = cc.upload(c0, c1)
    out = F.Ciphertext(cc)
    check(lib.fides_mult_pt(cc._h, ct._h, pt._h, out._h, 0), cc._h)
    got = out.download()
    assert np.array_equal(got[0], oc.polymul(c0, m, pid)) and np.array_equal(got[1], oc.polymul(c1, m, pid))
    # the same limbs in COEFFICIENT form
    ptc = cc.import_raw_pt(list(oc.ntt(m, pid, inverse=True)), oc.primes[:level + 1], fmt=cc.FORMAT_COEFFICIENT)
    out2 = F.Ciphertext(cc)
    check(lib.fides_mult_pt(cc._h, ct._h, ptc._h, out2._h, 0), cc._h)
    g2 = out2.download()
    assert np.array_equal(g2[0], got[0]) and np.array_equal(g2[1], got[1])


@pytest.mark.parametrize("logN,L,K", [(12, 8, 3), (16, 30, 10)])
def test_raw_rotation_key_roundtrip_and_rotate(logN, L, K):
    """A raw rotation key (plain layout, shuffled limbs) imported for a
    Galois element is held permuted to the rotation's output order; it
    exports unchanged, and the rotation with it equals the oracle's."""
    cc, oc = make_pair(logN, L, K, 3)
    rng = np.random.default_rng(logN + 1)
    kb, ka = rand_key(oc, 5300)
    r_key, r_mod = _raw_key(oc, kb, ka, rng)
    g = cc.rotation_galois(5)
    cc.import_raw_key(g, r_key, r_mod)
    back, _ = cc.export_raw_key(g)
    assert np.array_equal(back[0], ka) and np.array_equal(back[1], kb)
    level = L - 1
    c0, c1 = rand_ct(oc, level, 5400)
    got = cc.EvalRotate(cc.upload(c0, c1), 5).download()
    want = oc.rotate(level, c0, c1, pow(g, -1, 2 * oc.N), kb, ka)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
