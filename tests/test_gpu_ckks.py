"""Decrypted-error checks of the evaluation core against FP64 slot arithmetic.

FIDESlib checks rotations, conjugation and bootstrapping by decrypted error
(test/ParametrizedTest.cuh:517-530, max |delta| <= 2^-(logPrecision - 4));
here every operation is decrypted with the client-side half of the library
and compared with the same arithmetic on complex doubles.  Tolerances are
stated per test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import pyfideslib_b200 as F


def msgs(n, seed):
    r = np.random.default_rng(seed)
    rad = np.sqrt(r.uniform(0, 1, n))
    ang = r.uniform(0, 2 * np.pi, n)
    return rad * np.exp(1j * ang)  # uniform in the unit disk


@pytest.fixture(scope="module")
def small():
    cc = F.CryptoContext(log_n=13, num_q=8, dnum=3)
    sk = cc.KeyGen(seed=11, hamming_weight=64)
    cc.EvalMultKeyGen(sk)
    cc.EvalRotateKeyGen(sk, [1, 2, -1, 7, 100])
    cc.EvalConjugateKeyGen(sk)
    return cc, sk


def test_encrypt_decrypt(small):
    cc, sk = small
    z = msgs(cc.N // 2, 1)
    ct = cc.Encrypt(sk, z)
    assert np.max(np.abs(cc.Decrypt(sk, ct) - z)) < 1e-9


def test_sparse_slots(small):
    cc, sk = small
    z = msgs(64, 2)
    ct = cc.Encrypt(sk, z, slots=64)
    assert np.max(np.abs(cc.Decrypt(sk, ct) - z)) < 1e-9
    r = cc.EvalRotate(ct, 7)
    assert np.max(np.abs(cc.Decrypt(sk, r) - np.roll(z, -7))) < 1e-8


def test_hmult_rescale_error(small):
    cc, sk = small
    z1, z2 = msgs(cc.N // 2, 3), msgs(cc.N // 2, 4)
    a, b = cc.Encrypt(sk, z1, seed=1), cc.Encrypt(sk, z2, seed=2)
    c = cc.EvalMult(a, b, rescale=True)
    assert c.level == cc.L - 2
    assert np.max(np.abs(cc.Decrypt(sk, c) - z1 * z2)) < 1e-8
    # lazy path: mult, then explicit rescale gives identical residues
    d = cc.Rescale(cc.EvalMult(a, b))
    for x, y in zip(c.download(), d.download()):
        assert np.array_equal(x, y)


def test_depth_chain(small):
    cc, sk = small
    z = msgs(cc.N // 2, 5)
    ct = cc.Encrypt(sk, z)
    want = z.copy()
    for _ in range(cc.L - 2):
        ct = cc.EvalMult(ct, ct, rescale=True)
        want = want * want
    assert np.max(np.abs(cc.Decrypt(sk, ct) - want)) < 1e-6


def test_rotations(small):
    cc, sk = small
    z = msgs(cc.N // 2, 6)
    ct = cc.Encrypt(sk, z)
    for r in [1, 2, -1, 7, 100]:
        assert np.max(np.abs(cc.Decrypt(sk, cc.EvalRotate(ct, r)) - np.roll(z, -r))) < 1e-8, r
    outs = cc.EvalFastRotation(ct, [1, 2, 7])
    for o, r in zip(outs, [1, 2, 7]):
        assert np.max(np.abs(cc.Decrypt(sk, o) - np.roll(z, -r))) < 1e-8


def test_conjugate(small):
    cc, sk = small
    z = msgs(cc.N // 2, 7)
    ct = cc.Encrypt(sk, z)
    assert np.max(np.abs(cc.Decrypt(sk, cc.EvalConjugate(ct)) - np.conj(z))) < 1e-8


def test_add_sub_pt_scalar(small):
    cc, sk = small
    z1, z2 = msgs(cc.N // 2, 8), msgs(cc.N // 2, 9)
    a, b = cc.Encrypt(sk, z1), cc.Encrypt(sk, z2)
    assert np.max(np.abs(cc.Decrypt(sk, cc.EvalAdd(a, b)) - (z1 + z2))) < 1e-9
    assert np.max(np.abs(cc.Decrypt(sk, cc.EvalSub(a, b)) - (z1 - z2))) < 1e-9
    assert np.max(np.abs(cc.Decrypt(sk, cc.EvalNegate(a)) + z1)) < 1e-9
    pt = cc.MakeCKKSPackedPlaintext(z2)
    assert np.max(np.abs(cc.Decrypt(sk, cc.EvalMult(a, pt, rescale=True)) - z1 * z2)) < 1e-8
    assert np.max(np.abs(cc.Decrypt(sk, cc.EvalAdd(a, pt)) - (z1 + z2))) < 1e-9
    assert np.max(np.abs(cc.Decrypt(sk, cc.EvalMult(a, 0.75, rescale=True)) - 0.75 * z1)) < 1e-8
    assert np.max(np.abs(cc.Decrypt(sk, cc.EvalAdd(a, -0.5)) - (z1 - 0.5))) < 1e-9


def test_hmult_c2_decrypted_error():
    """N=2^16, L=30, K=10, dnum=3, scale 2^50, ternary h=192: HMult+Relin+Rescale.
    Stated bound: max slot error < 2^-30 against the FP64 product."""
    cc = F.CryptoContext(log_n=16, num_q=30, dnum=3, num_p=10)
    sk = cc.KeyGen(seed=21, hamming_weight=192)
    cc.EvalMultKeyGen(sk)
    z1, z2 = msgs(cc.N // 2, 31), msgs(cc.N // 2, 32)
    a, b = cc.Encrypt(sk, z1, seed=3), cc.Encrypt(sk, z2, seed=4)
    c = cc.EvalMult(a, b, rescale=True)
    err = np.max(np.abs(cc.Decrypt(sk, c) - z1 * z2))
    assert err < 2.0 ** -30, err


def test_rotation_keys_regenerated_for_new_secret():
    """EvalRotateKeyGen with a second secret key replaces the keys the first
    one left for the same indices (OpenFHE keeps keys per secret key)."""
    cc = F.CryptoContext(log_n=12, num_q=4, dnum=2)
    sk1 = cc.KeyGen(seed=1, hamming_weight=64)
    cc.EvalRotateKeyGen(sk1, [1, 5])
    sk2 = cc.KeyGen(seed=2, hamming_weight=64)
    cc.EvalRotateKeyGen(sk2, [5, 5, 7])
    rng = np.random.default_rng(0)
    z = rng.uniform(-1, 1, cc.N // 2)
    ct = cc.Encrypt(sk2, z)
    got = cc.Decrypt(sk2, cc.EvalRotate(ct, 5))
    assert np.max(np.abs(got - np.roll(z, -5))) < 1e-6
