"""Bit-exact parity with the oracle at the full workload shapes, through the C ABI.

* C2 shape (N=2^16, L=30: 60 + 29 x 50-bit moduli, K=10, dnum=3): single and
  hoisted rotations at the top level (largest residues) and at level 2;
  FIDESlib's own rotation tests run the same operations against OpenFHE
  (test/OpenFheInterfaceTests.cu:1014,1084).
* C3 shape (N=2^16, L=20: 60 + 19 x 40-bit moduli, K=6, dnum=3): eight of the
  32 hoisted rotation indices, and a 64-diagonal baby-step giant-step
  transform against the oracle composition of the same steps
  (CKKS/LinearTransform.cu:67-258).
* C4 shape: pairs at uneven levels in 4..29 through the captured graph plan
  (HMult + relinearisation + rescale, then a rotation by a random index),
  against oracle.hmult followed by oracle.rotate.
* C5 shape: EvalBootstrap at N=2^16 with a sparse secret (h=32), level budget
  {3,3} and a degree-119 EvalMod, precision asserted against the FP64
  message (the reference bounds bootstrap error the same way,
  test/ParametrizedTest.cuh:517-530).
"""
import numpy as np
import pytest

from gpu_helpers import device_status, make_pair, rand_ct, rand_key

pytestmark = pytest.mark.gpu


def _same(got, want):
    return np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def _upload_keys(cc, oc, indices, seed):
    keys = {}
    for i, r in enumerate(indices):
        g = cc.rotation_galois(r)
        if g not in keys:
            keys[g] = rand_key(oc, seed + 2 * i)
            cc.upload_galois_key(g, *keys[g])
    return keys


@pytest.fixture(scope="module")
def c2():
    cc, oc = make_pair(16, 30, 10, 3)
    yield cc, oc
    cc.close()


def test_rotations_c2_shape(c2):
    cc, oc = c2
    idx = [1, -1, 1000, 2 ** 14]
    keys = _upload_keys(cc, oc, idx, 2100)
    for level in (29, 2):
        c0, c1 = rand_ct(oc, level, 2200 + level)
        if level == 29:
            # the largest residues in c1, the polynomial that is key-switched
            pm1 = np.array([q - 1 for q in oc.primes[:level + 1]], dtype=np.uint64)[:, None]
            c1 = np.ascontiguousarray(np.broadcast_to(pm1, c1.shape))
        A = cc.upload(c0, c1)
        for r in idx[:2]:
            g = cc.rotation_galois(r)
            got = cc.EvalRotate(A, r).download()
            want = oc.rotate(level, c0, c1, pow(g, -1, 2 * oc.N), *keys[g])
            assert _same(got, want), (level, r)
        gals = [cc.rotation_galois(r) for r in idx]
        outs = cc.EvalFastRotation(A, idx)
        w0, w1 = oc.rotate_hoisted(level, c0, c1, [pow(g, -1, 2 * oc.N) for g in gals],
                                   [keys[g][0] for g in gals], [keys[g][1] for g in gals])
        for k, o in enumerate(outs):
            assert _same(o.download(), (w0[k], w1[k])), (level, idx[k])
    assert device_status(cc) == 0


@pytest.fixture(scope="module")
def c3():
    import pyfideslib_b200 as F
    from oracle import oracle as O

    cc = F.CryptoContext(log_n=16, num_q=20, dnum=3, qi_bits=40)
    oc = O.Ctx(cc.logN, cc.q, cc.p, cc.dnum)
    yield cc, oc
    cc.close()


def test_hoisted_rotations_c3_shape(c3):
    cc, oc = c3
    assert cc.K == 6 and all(q < 2 ** 41 for q in cc.q[1:])
    # eight of the workload's 32 indices (+-2^k and 3, 5)
    idx = [1, -1, 2 ** 7, -(2 ** 7), 2 ** 14, -(2 ** 14), 3, 5]
    keys = _upload_keys(cc, oc, idx, 3100)
    level = 19
    c0, c1 = rand_ct(oc, level, 3200)
    A = cc.upload(c0, c1)
    gals = [cc.rotation_galois(r) for r in idx]
    outs = cc.EvalFastRotation(A, idx)
    w0, w1 = oc.rotate_hoisted(level, c0, c1, [pow(g, -1, 2 * oc.N) for g in gals],
                               [keys[g][0] for g in gals], [keys[g][1] for g in gals])
    for k, o in enumerate(outs):
        assert _same(o.download(), (w0[k], w1[k])), idx[k]


def test_bsgs_64_diagonals_c3_shape(c3):
    """out = sum_k pt_k (.) Rot(x, k) over 64 diagonals (offsets 0..63,
    8 baby steps), rescaled, equals the oracle composition bit for bit."""
    import pyfideslib_b200 as F
    from test_gpu_linear import _oracle_bsgs, _upload_pt

    cc, oc = c3
    offsets, bstep = list(range(64)), 8
    rots = F.CryptoContext.linear_transform_rotations(offsets, bstep)
    keys = {}
    for i, r in enumerate(rots):
        g = cc.rotation_galois(r)
        keys[r] = rand_key(oc, 3300 + 2 * i)
        cc.upload_galois_key(g, *keys[r])
    level = 19
    c0, c1 = rand_ct(oc, level, 3400)
    x = cc.upload(c0, c1)
    pts_r = [oc.random(list(range(level + 1)), 3500 + k) for k in range(len(offsets))]
    pts = [_upload_pt(cc, m, level) for m in pts_r]
    got = cc.EvalLinearTransform(x, offsets, pts, bstep, rescale=True).download()
    w0, w1 = _oracle_bsgs(oc, level, c0, c1, offsets, pts_r, bstep, keys, cc.rotation_galois)
    assert _same(got, (oc.rescale(level, w0), oc.rescale(level, w1)))


def test_graph_plan_c4_shape_vs_oracle(c2):
    """Pairs at uneven levels (4..29) through one captured graph: HMult +
    relinearisation + rescale, then a rotation by a random index in
    [1, 2^15); every result equals oracle.hmult then oracle.rotate."""
    cc, oc = c2
    rng = np.random.default_rng(44)
    levels = [4, 29, 17, 11, 29, 8]
    idx = [int(x) for x in rng.integers(1, 2 ** 15, size=len(levels))]
    kb, ka = rand_key(oc, 4000)
    cc.upload_relin_key(kb, ka)
    keys = _upload_keys(cc, oc, idx, 4100)
    raw = [(rand_ct(oc, lv, 4200 + 4 * i), rand_ct(oc, lv, 4202 + 4 * i)) for i, lv in enumerate(levels)]
    A = [cc.upload(*a) for a, _ in raw]
    B = [cc.upload(*b) for _, b in raw]
    plan, outs = cc.plan_hmult_rotate(A, B, idx, rescale=True)
    for rep in range(2):
        plan.launch()
        cc.Synchronize()
        for i, lv in enumerate(levels):
            (a0, a1), (b0, b1) = raw[i]
            h0, h1 = oc.hmult(lv, a0, a1, b0, b1, kb, ka, rescale=True)
            g = cc.rotation_galois(idx[i])
            want = oc.rotate(lv - 1, h0, h1, pow(g, -1, 2 * oc.N), *keys[g])
            assert _same(outs[i].download(), want), (rep, i, lv)
    del plan


def test_bootstrap_precision_c5_shape():
    """EvalBootstrap at N=2^16, L=30, 2^15 slots, h=32, budget {3,3}, degree
    119: the refreshed ciphertext decrypts to the message within the stated
    precision (12.5 bits by default; 17 bits with the correction factor 6,
    valid for these messages), at the advertised output level."""
    import pyfideslib_b200 as F

    cc = F.CryptoContext(log_n=16, num_q=30, dnum=3)
    try:
        sk = cc.KeyGen(seed=101, hamming_weight=32)
        cc.EvalMultKeyGen(sk)
        cc.EvalBootstrapSetup(level_budget=(3, 3), cheb_degree=119)
        cc.EvalBootstrapKeyGen(sk)
        out_level, _ = cc.bootstrap_info()
        slots = cc.N // 2
        rng = np.random.default_rng(101)
        m = rng.uniform(-1, 1, slots) + 1j * rng.uniform(-1, 1, slots)
        ct = cc.Encrypt(sk, m, slots=slots, level=0, seed=7)
        bt = cc.EvalBootstrap(ct)
        assert bt.level == out_level
        bits = -np.log2(np.max(np.abs(cc.Decrypt(sk, bt, slots=slots) - m)))
        assert bits > 12.5, bits
        cc.EvalBootstrapSetup(level_budget=(3, 3), cheb_degree=119, correction=6)
        bt6 = cc.EvalBootstrap(ct)
        bits6 = -np.log2(np.max(np.abs(cc.Decrypt(sk, bt6, slots=slots) - m)))
        assert bits6 > 17.0, bits6
        assert device_status(cc) == 0
    finally:
        cc.close()


def test_sparse_bootstrap_c5_shape():
    """EvalBootstrap with sparse packing at N=2^16, L=30: 2^12 slots, h=32,
    budget {2,2}, degree 119: the subring projection (3 rotate-and-add
    steps) and the 2^12-slot transforms; precision asserted against the
    FP64 message at the advertised output level."""
    import pyfideslib_b200 as F

    cc = F.CryptoContext(log_n=16, num_q=30, dnum=3)
    try:
        slots = 1 << 12
        sk = cc.KeyGen(seed=103, hamming_weight=32)
        cc.EvalMultKeyGen(sk)
        cc.EvalBootstrapSetup(level_budget=(2, 2), slots=slots, cheb_degree=119)
        cc.EvalBootstrapKeyGen(sk, slots=slots)
        out_level, _ = cc.bootstrap_info(slots)
        rng = np.random.default_rng(103)
        m = rng.uniform(-1, 1, slots) + 1j * rng.uniform(-1, 1, slots)
        ct = cc.Encrypt(sk, m, slots=slots, level=0, seed=9)
        bt = cc.EvalBootstrap(ct)
        assert bt.level == out_level and bt.slots == slots
        bits = -np.log2(np.max(np.abs(cc.Decrypt(sk, bt, slots=slots) - m)))
        assert bits > 13.0, bits
        assert device_status(cc) == 0
    finally:
        cc.close()
