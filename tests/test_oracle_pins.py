"""Pins of the CPU oracle against FIDESlib's own known answers and against
big-integer definitions of every formula it restates.

The oracle is the checker for the CUDA path, so before it is trusted:
  * scalar arithmetic matches test/MathTest.cu's known answers;
  * the N=8, p=17 negacyclic convolution of test/NegacyclicNTTtests.cu holds;
  * the evaluation order equals bitrev(nega_fft2(x)) at logN 13..16 on the
    reference's own test primes (test/NTTtests.cu:933-1040);
  * the CRT constants equal their big-integer definitions;
  * ModUp, ModDown and Rescale satisfy their exact integer semantics;
  * the automorphism scatter is the ring map a(X) -> a(X^(k^-1)).
"""
import json
import os
import random

import numpy as np
import pytest

from oracle import oracle as O

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.json")))


def bitrev(x, bits):
    return int(format(x, "0%db" % bits)[::-1], 2) if bits else 0


def test_math_known_answers():
    for a, e, p, r in GOLD["powmod"]:
        assert O.powmod(a, e, p) == r
    for a, p, r in GOLD["invmod"]:
        assert O.invmod(a, p) == r


def test_negacyclic_n8_p17():
    g = GOLD["negacyclic_n8"]
    p, logN = g["p"], g["logN"]
    ctx = O.Ctx(logN, [p], [], 1)
    a = np.array(g["v1"], dtype=np.uint64).reshape(1, -1)
    b = np.array(g["v2"], dtype=np.uint64).reshape(1, -1)
    fa, fb = ctx.ntt(a, [0]), ctx.ntt(b, [0])
    prod = ctx.ntt(ctx.polymul(fa, fb, [0]), [0], inverse=True)
    assert prod.ravel().tolist() == g["product"]
    # the same through the independent twist+cyclic formulation
    psi = O.unity_root(p, 2 << logN)
    na, nb = O.nega_fft2(a.ravel(), logN, p, psi), O.nega_fft2(b.ravel(), logN, p, psi)
    pr = O.nega_fft2(np.array([int(x) * int(y) % p for x, y in zip(na, nb)], dtype=np.uint64), logN, p, psi, True)
    assert pr.tolist() == g["product"]


@pytest.mark.parametrize("logN", [13, 14, 15, 16])
def test_eval_order_is_bitreversed_nega_fft2(logN):
    primes = [GOLD["p64"][0], GOLD["p64"][1], GOLD["sp64"][0]]
    ctx = O.Ctx(logN, primes[:2], primes[2:], 1)
    rng = np.random.default_rng(logN)
    for pid, p in enumerate(primes):
        x = (rng.integers(0, 2**63, size=1 << logN, dtype=np.uint64) % np.uint64(p)).astype(np.uint64)
        ev = ctx.ntt(x.reshape(1, -1), [pid]).ravel()
        psi = O.unity_root(p, 2 << logN)
        nat = O.nega_fft2(x, logN, p, psi)
        br = np.array([bitrev(i, logN) for i in range(1 << logN)])
        assert np.array_equal(ev, nat[br])
        back = ctx.ntt(ev.reshape(1, -1), [pid], inverse=True).ravel()
        assert np.array_equal(back, x)


def test_prime_search():
    ps = O.find_primes(16, 50, 8)
    assert len(ps) == 8 and ps == sorted(ps, reverse=True)
    for p in ps:
        assert O.is_prime(p) and (p - 1) % (1 << 17) == 0 and p < 2**50 and p.bit_length() == 50
    # the reference's own test primes are NTT-friendly for logN 16
    for p in GOLD["p64"] + GOLD["sp64"]:
        assert O.is_prime(p) and (p - 1) % (1 << 17) == 0


def _prod(xs):
    r = 1
    for x in xs:
        r *= x
    return r


def small_ctx(logN=10, L=7, K=3, dnum=3):
    q = GOLD["p64"][:L]
    p = GOLD["sp64"][:K]
    return O.Ctx(logN, q, p, dnum)


def test_crt_constants_bigint():
    ctx = small_ctx()
    L, K, alpha = ctx.L, ctx.K, ctx.alpha
    pr = ctx.primes
    for level in range(L):
        for d in range(ctx.num_digits(level)):
            lo, hi = d * alpha, min(d * alpha + alpha - 1, level)
            Qd = _prod(pr[lo:hi + 1])
            hi_inv, hm = ctx.modup_consts(level, d)
            for i in range(lo, hi + 1):
                qi = pr[i]
                assert int(hi_inv[i - lo]) == pow(Qd // qi % qi, -1, qi)
                for t in range(L + K):
                    assert int(hm[i - lo, t]) == (Qd // qi) % pr[t]
    phat_inv, phat_mod, p_inv = ctx.moddown_consts()
    P = _prod(pr[L:])
    for k in range(K):
        pk = pr[L + k]
        assert int(phat_inv[k]) == pow(P // pk % pk, -1, pk)
        for j in range(L):
            assert int(phat_mod[k, j]) == (P // pk) % pr[j]
    for j in range(L):
        assert int(p_inv[j]) == pow(P % pr[j], -1, pr[j])
    # Rescale constant: QlQlInvModqlDivqlModq (the name OpenFHE exports) is
    # floor(Q'*[Q'^-1]_{q_l} / q_l) mod q_j with Q' = q_0..q_{l-1}; it equals
    # -q_l^-1 mod q_j, which is what the oracle (and the kernels) use.
    for level in range(1, L):
        ql = pr[level]
        Qp = _prod(pr[:level])
        v = pow(Qp % ql, -1, ql)
        m = (Qp * v) // ql
        for j in range(level):
            assert m % pr[j] == (-pow(ql, -1, pr[j])) % pr[j]


def crt(res, mods):
    M = _prod(mods)
    x = 0
    for r, m in zip(res, mods):
        Mi = M // m
        x += int(r) * Mi * pow(Mi % m, -1, m)
    return x % M, M


def test_modup_exact_semantics():
    ctx = small_ctx()
    L, K, alpha, N = ctx.L, ctx.K, ctx.alpha, ctx.N
    pr = ctx.primes
    level = L - 1
    x = ctx.random(list(range(level + 1)), 11)
    dg = ctx.modup(level, x)
    coef_in = ctx.ntt(x, list(range(level + 1)), inverse=True)
    ext = ctx.ext_pidx(level)
    for d in range(ctx.num_digits(level)):
        lo, hi = d * alpha, min(d * alpha + alpha - 1, level)
        out_coef = ctx.ntt(dg[d], ext, inverse=True)
        mods = pr[lo:hi + 1]
        Qd = _prod(mods)
        for j in random.Random(d).sample(range(N), 12):
            X, _ = crt([coef_in[i, j] for i in range(lo, hi + 1)], mods)
            # fast base conversion: X + u*Q' for some 0 <= u < #digit primes
            cands = [(X + u * Qd) for u in range(len(mods))]
            got = [int(out_coef[m, j]) for m in range(len(ext))]
            ok = [all(got[m] == c % pr[ext[m]] for m in range(len(ext))) for c in cands]
            assert any(ok), (d, j)


def test_moddown_exact_semantics():
    ctx = small_ctx()
    L, K, N = ctx.L, ctx.K, ctx.N
    pr = ctx.primes
    level = 4
    ext = ctx.ext_pidx(level)
    x = ctx.random(ext, 5)
    out = ctx.moddown(level, x)
    xc = ctx.ntt(x, ext, inverse=True)
    oc = ctx.ntt(out, list(range(level + 1)), inverse=True)
    P = _prod(pr[L:])
    qmods = pr[:level + 1]
    for j in random.Random(3).sample(range(N), 16):
        Y, _ = crt([xc[L_, j] for L_ in range(level + 1, level + 1 + K)], pr[L:])
        # ModDown: (x - (y + v*P)) / P with the fast-converted y, 0 <= v < K
        got = [int(oc[i, j]) for i in range(level + 1)]
        ok = False
        for v in range(K):
            for i in range(level + 1):
                qi = qmods[i]
                want = (int(xc[i, j]) - (Y + v * P)) * pow(P % qi, -1, qi) % qi
                if got[i] != want:
                    break
            else:
                ok = True
        assert ok


def test_rescale_exact_division():
    ctx = small_ctx()
    N = ctx.N
    pr = ctx.primes
    level = 5
    pid = list(range(level + 1))
    x = ctx.random(pid, 9)
    out = ctx.rescale(level, x)
    xc = ctx.ntt(x, pid, inverse=True)
    oc = ctx.ntt(out, pid[:-1], inverse=True)
    ql = pr[level]
    Qm = _prod(pr[:level])
    for j in random.Random(4).sample(range(N), 20):
        X, Q = crt([xc[i, j] for i in pid], pr[:level + 1])
        t = X % ql
        if t > ql // 2:
            t -= ql
        Y = (X - t) // ql
        assert (X - t) % ql == 0
        for i in range(level):
            assert int(oc[i, j]) == Y % pr[i]


def test_automorph_is_ring_map():
    ctx = small_ctx(logN=8, L=2, K=1, dnum=1)
    N = ctx.N
    p = ctx.primes[0]
    rng = np.random.default_rng(1)
    a = (rng.integers(0, 2**62, size=N, dtype=np.uint64) % np.uint64(p)).reshape(1, -1)
    for idx in [1, 3, -1, 17]:
        k = ctx.rotation_galois(idx, N // 2)
        ev = ctx.ntt(a, [0])
        rot = ctx.ntt(ctx.automorph(ev, k), [0], inverse=True).ravel()
        g = pow(k, -1, 2 * N)
        want = [0] * N
        for i in range(N):
            e = (i * g) % (2 * N)
            v = int(a[0, i])
            if e >= N:
                want[e - N] = (want[e - N] - v) % p
            else:
                want[e] = (want[e] + v) % p
        assert rot.tolist() == want
        # rotation by idx uses X -> X^(5^idx)
        assert g == pow(5, idx % (N // 2), 2 * N)


def test_hoisted_equals_single_rotations():
    ctx = small_ctx()
    level = 5
    pid = list(range(level + 1))
    np_ = ctx.L + ctx.K
    c0, c1 = ctx.random(pid, 1), ctx.random(pid, 2)
    keys = [(ctx.random(list(range(np_)) * ctx.dnum, 10 + r).reshape(ctx.dnum, np_, ctx.N),
             ctx.random(list(range(np_)) * ctx.dnum, 20 + r).reshape(ctx.dnum, np_, ctx.N)) for r in range(2)]
    gal = [ctx.rotation_galois(i, ctx.N // 2) for i in (1, 5)]
    h0, h1 = ctx.rotate_hoisted(level, c0, c1, gal, [k[0] for k in keys], [k[1] for k in keys])
    for r in range(2):
        s0, s1 = ctx.rotate(level, c0, c1, gal[r], keys[r][0], keys[r][1])
        assert np.array_equal(s0, h0[r]) and np.array_equal(s1, h1[r])
