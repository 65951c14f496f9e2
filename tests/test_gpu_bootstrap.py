"""Bootstrapping and the operations it is built from, through the C ABI.

Bit-exact against the oracle (random residues): integer scalar product,
monomial product X^k (the negacyclic shift restated with the oracle's NTT),
ModRaise (centred lift of limb 0 to every modulus, Bootstrap.cu:380).
Numerically against FP64: EvalChebyshevSeries (ApproxModEval.cu:370) and
EvalBootstrap (Bootstrap.cu:169-320) -- the reference's own bootstrap tests
state a precision bound the same way (test/ParametrizedTest.cuh:517-530).
"""
import numpy as np
import pytest

from gpu_helpers import device_status, make_pair, rand_ct

pytestmark = pytest.mark.gpu


def _negacyclic_shift(coef, k, p):
    """coef * X^k in Z_p[X]/(X^N + 1), coef of shape (limbs, N), p of shape (limbs,)."""
    N = coef.shape[-1]
    out = np.zeros_like(coef)
    for i in range(N):
        e = i + k
        v = coef[:, i] % p
        out[:, e % N] = (p - v) % p if (e // N) % 2 else v
    return out


def test_mult_int_monomial_modraise_bitexact():
    cc, oc = make_pair(10, 6, 2, 3)
    level = 4
    pid = list(range(level + 1))
    p = np.array(oc.primes[:level + 1], dtype=np.uint64)[:, None]
    c0, c1 = rand_ct(oc, level, 5)
    x = cc.upload(c0, c1)
    for z in (3, -7, 2 ** 40 + 11):
        g0, g1 = cc.EvalMultInt(x, z).download()
        zz = np.array([z % int(q) for q in oc.primes[:level + 1]], dtype=np.uint64)[:, None]
        w0 = oc.polymul(c0, np.ascontiguousarray(np.broadcast_to(zz, c0.shape)), pid)
        w1 = oc.polymul(c1, np.ascontiguousarray(np.broadcast_to(zz, c1.shape)), pid)
        assert np.array_equal(g0, w0) and np.array_equal(g1, w1), z
    for k in (1, 5, cc.N // 2, 3 * cc.N // 2, 2 * cc.N - 1):
        g0, g1 = cc.EvalMultMonomial(x, k).download()
        for got, src in ((g0, c0), (g1, c1)):
            coef = oc.ntt(src, pid, inverse=True)
            want = oc.ntt(np.ascontiguousarray(_negacyclic_shift(coef, k, p[:, 0])), pid)
            assert np.array_equal(got, want), k
    # ModRaise: limb 0 lifted to (-q0/2, q0/2] and reduced modulo every modulus
    r0, r1 = cc.ModRaise(x).download()
    q0 = int(oc.primes[0])
    allp = list(range(oc.L))
    for got, src in ((r0, c0), (r1, c1)):
        a = oc.ntt(np.ascontiguousarray(src[:1]), [0], inverse=True)[0].astype(object)
        a = np.where(a > q0 // 2, a - q0, a)
        lifted = np.array([[int(v) % int(q) for v in a] for q in oc.primes[:oc.L]], dtype=np.uint64)
        want = oc.ntt(lifted, allp)
        assert got.shape == want.shape and np.array_equal(got, want)


def test_chebyshev_series_matches_fp64():
    import pyfideslib_b200 as F

    cc = F.CryptoContext(log_n=12, num_q=12, dnum=3)
    sk = cc.KeyGen(seed=5, hamming_weight=64)
    cc.EvalMultKeyGen(sk)
    slots = cc.N // 2
    rng = np.random.default_rng(7)
    x = rng.uniform(-1, 1, slots)
    ct = cc.Encrypt(sk, x, slots=slots)
    from numpy.polynomial import chebyshev as Ch
    for deg, fn in ((7, lambda t: np.cos(3 * t)), (31, lambda t: np.exp(t) * np.sin(4 * t)),
                    (59, lambda t: 1.0 / (1.0 + 4 * t * t))):
        c = Ch.chebinterpolate(fn, deg)
        y = cc.EvalChebyshevSeries(ct, c)
        got = cc.Decrypt(sk, y, slots=slots).real
        err = np.max(np.abs(got - Ch.chebval(x, c)))
        assert err < 1e-9, (deg, err)
    # a general interval costs one more level
    c = Ch.chebinterpolate(lambda t: np.cos(t), 15)
    y = cc.EvalChebyshevSeries(ct, c, lo=-2.0, hi=2.0)
    err = np.max(np.abs(cc.Decrypt(sk, y, slots=slots).real - Ch.chebval(x / 2.0, c)))
    assert err < 1e-9, err


def test_bootstrap_precision():
    import pyfideslib_b200 as F

    cc = F.CryptoContext(log_n=12, num_q=20, dnum=4)
    sk = cc.KeyGen(seed=9, hamming_weight=32)
    cc.EvalMultKeyGen(sk)
    cc.EvalBootstrapSetup(level_budget=(3, 3), cheb_degree=63)
    cc.EvalBootstrapKeyGen(sk)
    out_level, _ = cc.bootstrap_info()
    slots = cc.N // 2
    rng = np.random.default_rng(3)
    for trial in range(2):
        m = rng.uniform(-1, 1, slots) + 1j * rng.uniform(-1, 1, slots)
        ct = cc.Encrypt(sk, m, slots=slots, level=0)
        bt = cc.EvalBootstrap(ct)
        assert bt.level == out_level
        got = cc.Decrypt(sk, bt, slots=slots)
        err = np.max(np.abs(got - m))
        bits = -np.log2(err)
        assert bits > 14, (trial, err)
        # the refreshed ciphertext still multiplies
        sq = cc.EvalMult(bt, bt, rescale=True)
        err2 = np.max(np.abs(cc.Decrypt(sk, sq, slots=slots) - m * m))
        assert err2 < 2 ** -10, err2
    # the correction factor lifts the message against EvalMod's noise (2^3:
    # beyond that, at N = 2^12, the sine's cubic term on the largest message
    # coefficients takes over)
    cc.EvalBootstrapSetup(level_budget=(3, 3), cheb_degree=63, correction=3)
    m = rng.uniform(-1, 1, slots) + 1j * rng.uniform(-1, 1, slots)
    ct = cc.Encrypt(sk, m, slots=slots, level=0)
    err5 = np.max(np.abs(cc.Decrypt(sk, cc.EvalBootstrap(ct), slots=slots) - m))
    assert -np.log2(err5) > bits + 1.5, (err5, err)


def test_bootstrap_requests_served_in_mix():
    """EvalBootstrap requests in the serving loop beside HMult / Rotate
    batches give the same residues as the call made alone."""
    import pyfideslib_b200 as F

    cc = F.CryptoContext(log_n=12, num_q=20, dnum=4)
    sk = cc.KeyGen(seed=4, hamming_weight=32)
    cc.EvalMultKeyGen(sk)
    cc.EvalBootstrapSetup(level_budget=(3, 3), cheb_degree=63)
    cc.EvalBootstrapKeyGen(sk)
    cc.EvalRotateKeyGen(sk, [1, 3])
    rng = np.random.default_rng(8)
    slots = cc.N // 2
    lo = [cc.Encrypt(sk, rng.uniform(-1, 1, slots), slots=slots, level=0, seed=20 + i) for i in range(2)]
    hi = [cc.Encrypt(sk, rng.uniform(-1, 1, slots), slots=slots, level=10, seed=30 + i) for i in range(3)]
    srv = F.Server(cc, hbm_budget=16 << 30, max_batch=4, num_streams=2)
    reqs = []
    for k in range(12):
        if k % 4 == 0:
            reqs.append((F.Server.BOOTSTRAP, lo[(k // 4) % 2], None, 0))
        elif k % 2:
            reqs.append((F.Server.HMULT, hi[k % 3], hi[(k + 1) % 3], 0))
        else:
            reqs.append((F.Server.ROTATE, hi[k % 3], None, 3))
    outs = [srv.submit(op, a, b, r) for op, a, b, r in reqs]
    for rid, _ in outs:
        srv.wait(rid, 120.0)
    assert srv.stats()["completed"] == len(reqs)
    srv.close()
    for (op, a, b, r), (_, out) in zip(reqs, outs):
        if op == F.Server.BOOTSTRAP:
            alone = cc.EvalBootstrap(a)
        elif op == F.Server.HMULT:
            alone = cc.EvalMult(a, b, rescale=True)
        else:
            alone = cc.EvalRotate(a, r)
        g, w = out.download(), alone.download()
        assert np.array_equal(g[0], w[0]) and np.array_equal(g[1], w[1]), op


def test_bootstrap_batch_equals_single():
    """fides_bootstrap_batch: the batched EvalMod lanes and giant-step
    rotations give every input the residues of its own EvalBootstrap."""
    import pyfideslib_b200 as F

    cc = F.CryptoContext(log_n=12, num_q=20, dnum=4)
    sk = cc.KeyGen(seed=12, hamming_weight=32)
    cc.EvalMultKeyGen(sk)
    cc.EvalBootstrapSetup(level_budget=(3, 3), cheb_degree=63)
    cc.EvalBootstrapKeyGen(sk)
    slots = cc.N // 2
    rng = np.random.default_rng(12)
    msgs = [rng.uniform(-1, 1, slots) + 1j * rng.uniform(-1, 1, slots) for _ in range(3)]
    cts = [cc.Encrypt(sk, m, slots=slots, level=i, seed=40 + i) for i, m in enumerate(msgs)]
    outs = cc.EvalBootstrapBatch(cts)
    for ct, o, m in zip(cts, outs, msgs):
        w = cc.EvalBootstrap(ct).download()
        g = o.download()
        assert np.array_equal(g[0], w[0]) and np.array_equal(g[1], w[1])
        assert np.max(np.abs(cc.Decrypt(sk, o, slots=slots) - m)) < 2 ** -14


def test_bootstrap_requests_queued_in_serving():
    """Several bootstraps submitted together are all served (one batched
    call per kBootBatch of them); each result equals the call made alone."""
    import pyfideslib_b200 as F

    cc = F.CryptoContext(log_n=12, num_q=20, dnum=4)
    sk = cc.KeyGen(seed=13, hamming_weight=32)
    cc.EvalMultKeyGen(sk)
    cc.EvalBootstrapSetup(level_budget=(3, 3), cheb_degree=63)
    cc.EvalBootstrapKeyGen(sk)
    slots = cc.N // 2
    rng = np.random.default_rng(13)
    cts = [cc.Encrypt(sk, rng.uniform(-1, 1, slots), slots=slots, level=0, seed=60 + i) for i in range(5)]
    srv = F.Server(cc, hbm_budget=16 << 30, max_batch=4, num_streams=1)
    outs = [srv.submit(F.Server.BOOTSTRAP, c) for c in cts]
    for rid, _ in outs:
        srv.wait(rid, 120.0)
    st = srv.stats()
    srv.close()
    assert st["completed"] == 5 and 1 <= st["batches"] <= 5
    for c, (_, o) in zip(cts, outs):
        g, w = o.download(), cc.EvalBootstrap(c).download()
        assert np.array_equal(g[0], w[0]) and np.array_equal(g[1], w[1])


@pytest.mark.parametrize("slots", [8, 512])
def test_sparse_bootstrap_precision(slots):
    """EvalBootstrap with sparse packing (slots < N/2; the reference's
    approxModReductionSparse path, src/CKKS/ApproxModEval.cu:94, and
    slot-count-dependent CoeffsToSlots, src/CKKS/CoeffsToSlots.cu:26,161):
    the raised polynomial is projected onto the n-slot subring by
    log2(N/2n) rotate-and-add steps, then the n-slot transforms run.  The
    refreshed ciphertext decrypts to the message, keeps its slot count, and
    still multiplies; a full-packing set-up in the same context is unaffected."""
    import pyfideslib_b200 as F

    cc = F.CryptoContext(log_n=12, num_q=20, dnum=4)
    sk = cc.KeyGen(seed=19, hamming_weight=32)
    cc.EvalMultKeyGen(sk)
    cc.EvalBootstrapSetup(level_budget=(2, 2), slots=slots, cheb_degree=63)
    cc.EvalBootstrapKeyGen(sk, slots=slots)
    out_level, rots = cc.bootstrap_info(slots)
    assert any(r >= slots for r in rots)  # the subring projection's rotations
    rng = np.random.default_rng(slots)
    m = rng.uniform(-1, 1, slots) + 1j * rng.uniform(-1, 1, slots)
    ct = cc.Encrypt(sk, m, slots=slots, level=0)
    bt = cc.EvalBootstrap(ct)
    assert bt.level == out_level and bt.slots == slots
    err = np.max(np.abs(cc.Decrypt(sk, bt, slots=slots) - m))
    assert -np.log2(err) > 14, err
    sq = cc.EvalMult(bt, bt, rescale=True)
    err2 = np.max(np.abs(cc.Decrypt(sk, sq, slots=slots) - m * m))
    assert err2 < 2 ** -10, err2
    # batched sparse bootstraps equal single ones
    b2 = cc.EvalBootstrapBatch([ct, ct])
    r0, r1 = bt.download()
    for o in b2:
        g0, g1 = o.download()
        assert np.array_equal(g0, r0) and np.array_equal(g1, r1)
    assert device_status(cc) == 0


def test_two_iteration_bootstrap_precision():
    """EvalBootstrap(ct, numIterations=2): the first result's error is
    bootstrapped again at 2^12 and subtracted; the result decrypts to the
    message with at least 8 more bits than one bootstrap, one level below a
    single bootstrap's output.  An input below the bootstrap's output level
    is refused for a second iteration."""
    import pyfideslib_b200 as F

    cc = F.CryptoContext(log_n=12, num_q=20, dnum=4)
    sk = cc.KeyGen(seed=29, hamming_weight=32)
    cc.EvalMultKeyGen(sk)
    cc.EvalBootstrapSetup(level_budget=(3, 3), cheb_degree=63)
    cc.EvalBootstrapKeyGen(sk)
    out_level, _ = cc.bootstrap_info()
    slots = cc.N // 2
    rng = np.random.default_rng(29)
    m = rng.uniform(-1, 1, slots) + 1j * rng.uniform(-1, 1, slots)
    ct = cc.Encrypt(sk, m, slots=slots, level=out_level + 2, seed=5)
    one = cc.EvalBootstrap(ct)
    two = cc.EvalBootstrap(ct, num_iterations=2, precision=12)
    assert two.level == out_level - 1
    b1 = -np.log2(np.max(np.abs(cc.Decrypt(sk, one, slots=slots) - m)))
    b2 = -np.log2(np.max(np.abs(cc.Decrypt(sk, two, slots=slots) - m)))
    assert b2 > b1 + 8, (b1, b2)
    low = cc.Encrypt(sk, m, slots=slots, level=0, seed=6)
    from pyfideslib_b200._capi import FidesError
    with pytest.raises(FidesError):
        cc.EvalBootstrap(low, num_iterations=2)
    assert device_status(cc) == 0


def test_bootstrap_giant_step_moddown_modes():
    """The bootstrap's transforms with one ModDown per giant-step rotation
    (scope 0) and with each input's giant steps brought down once (scope 1,
    the default): the same precision.  The two ModDowns differ by a few units
    per coefficient, which the rescale after each transform divides by a
    modulus of about 2^50, so the refreshed ciphertexts are usually
    identical; the bound allows for the rare rounding step."""
    import pyfideslib_b200 as F
    from pyfideslib_b200._capi import lib

    cc = F.CryptoContext(log_n=12, num_q=20, dnum=4)
    sk = cc.KeyGen(seed=19, hamming_weight=32)
    cc.EvalMultKeyGen(sk)
    cc.EvalBootstrapSetup(level_budget=(3, 3), cheb_degree=63)
    cc.EvalBootstrapKeyGen(sk)
    slots = cc.N // 2
    rng = np.random.default_rng(33)
    m = rng.uniform(-1, 1, slots) + 1j * rng.uniform(-1, 1, slots)
    ct = cc.Encrypt(sk, m, slots=slots, level=0)
    got = {}
    for scope in (0, 1):
        assert lib.fides_set_giant_step_moddown(cc._h, scope) == 0
        got[scope] = cc.Decrypt(sk, cc.EvalBootstrap(ct), slots=slots)
        assert -np.log2(np.max(np.abs(got[scope] - m))) > 14, scope
    d = np.max(np.abs(got[0] - got[1]))
    assert d < 2 ** -14, d
