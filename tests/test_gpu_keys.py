"""Compressed rotation keys: a Galois key generated with compression stores
its b half and the seed of its uniform a half, which the key-switch kernels
regenerate.  Rotations with such keys equal the oracle's with the exported
(materialised) key, and equal the same keys stored in full, bit for bit --
single, hoisted, batched and grouped-hoisted (batched linear transform)."""
import numpy as np
import pytest

from gpu_helpers import make_pair, rand_ct

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("logN,L,K", [(12, 8, 3), (16, 20, 6)])
def test_compressed_rotation_keys_bitexact(logN, L, K):
    import pyfideslib_b200 as F
    from pyfideslib_b200._capi import lib

    cc, oc = make_pair(logN, L, K, 3)
    sk = cc.KeyGen(seed=31, hamming_weight=64)
    idx = [1, -1, 5, 3]
    level = L - 1
    c0, c1 = rand_ct(oc, level, 3100)
    A = cc.upload(c0, c1)
    res = {}
    for comp in (1, 0):
        assert lib.fides_set_key_compression(cc._h, comp) == 0
        cc.EvalRotateKeyGen(sk, idx, seed=77)
        single = [cc.EvalRotate(A, r).download() for r in idx]
        hoisted = [o.download() for o in cc.EvalFastRotation(A, idx)]
        batch = [o.download() for o in cc.EvalRotateBatch([A] * len(idx), idx)]
        res[comp] = (single, hoisted, batch)
        if comp == 1:
            for r, got in zip(idx, single):
                g = cc.rotation_galois(r)
                kb, ka = cc.export_key(g)
                want = oc.rotate(level, c0, c1, pow(g, -1, 2 * oc.N), kb, ka)
                assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), r
    for a, b in zip(res[1], res[0]):
        for x, y in zip(a, b):
            assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1])
    for s, h in zip(res[1][0], res[1][1]):
        assert np.array_equal(s[0], h[0]) and np.array_equal(s[1], h[1])
    assert lib.fides_set_key_compression(cc._h, 1) == 0


def test_compressed_keys_in_batched_transform_and_bootstrap():
    """The grouped hoisted rotations of a batched linear transform and a
    bootstrap run on compressed keys as on full ones."""
    import pyfideslib_b200 as F
    from pyfideslib_b200._capi import lib

    cc = F.CryptoContext(log_n=12, num_q=20, dnum=4)
    sk = cc.KeyGen(seed=41, hamming_weight=32)
    cc.EvalMultKeyGen(sk)
    cc.EvalBootstrapSetup(level_budget=(3, 3), cheb_degree=63)
    slots = cc.N // 2
    rng = np.random.default_rng(41)
    ct = cc.Encrypt(sk, rng.uniform(-1, 1, slots), slots=slots, level=0, seed=3)
    outs = {}
    for comp in (1, 0):
        assert lib.fides_set_key_compression(cc._h, comp) == 0
        cc.EvalBootstrapKeyGen(sk, seed=11)
        outs[comp] = [o.download() for o in cc.EvalBootstrapBatch([ct, ct])]
    for x, y in zip(outs[1], outs[0]):
        assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1])


def test_compressed_relin_key_bitexact():
    """A compressed relinearisation key (mask bit 1): single and batched
    HMults (a batch of 8, which with a full key takes the key switch fused
    into the row pass) equal the same key stored in full and the oracle's
    HMult with the exported key."""
    from pyfideslib_b200._capi import lib

    cc, oc = make_pair(12, 8, 3, 3)
    sk = cc.KeyGen(seed=51, hamming_weight=64)
    level = 7
    raw = [(rand_ct(oc, level, 5100 + 4 * i), rand_ct(oc, level, 5102 + 4 * i)) for i in range(8)]
    A = [cc.upload(*a) for a, _ in raw]
    B = [cc.upload(*b) for _, b in raw]
    res = {}
    for mask in (3, 0):
        assert lib.fides_set_key_compression(cc._h, mask) == 0
        cc.EvalMultKeyGen(sk, seed=9)
        single = cc.EvalMult(A[0], B[0]).download()
        batch = [o.download() for o in cc.EvalMultBatch(A, B)]
        res[mask] = [single] + batch
        if mask == 3:
            kb, ka = cc.export_key(0)
            (a0, a1), (b0, b1) = raw[0]
            want = oc.hmult(level, a0, a1, b0, b1, kb, ka, rescale=False)
            assert np.array_equal(single[0], want[0]) and np.array_equal(single[1], want[1])
    for x, y in zip(res[3], res[0]):
        assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1])
    assert lib.fides_set_key_compression(cc._h, 1) == 0
