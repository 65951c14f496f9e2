"""Diagonal-form linear transform (baby-step giant-step) through the C ABI.

* Bit-exact: the CUDA path equals the oracle composition of the same steps
  (hoisted baby rotations, plaintext products summed per giant step, giant
  rotations, sum, rescale) on random residues and random switching keys; the
  reference's LinearTransform (CKKS/LinearTransform.cu:67-258) has this shape.
* Numerically: with real keys and encoded diagonals the decrypted result
  matches the FP64 matrix-vector product (the reference's tests bound the
  error of rotations the same way, test/ParametrizedTest.cuh:517-530).
"""
import ctypes as C

import numpy as np
import pytest

from gpu_helpers import make_pair, rand_ct, rand_key

pytestmark = pytest.mark.gpu


def _upload_pt(cc, m, level):
    import pyfideslib_b200 as F
    from pyfideslib_b200._capi import check, lib, u64p, vp

    h = vp()
    m = np.ascontiguousarray(m, dtype=np.uint64)
    check(lib.fides_pt_upload(cc._h, m.ctypes.data_as(u64p), level, 1.0, 1, cc.N // 2, C.byref(h)), cc._h)
    return F.Plaintext(cc, h.value)


def _oracle_bsgs(oc, level, c0, c1, offsets, pts, bstep, keys, gal_of):
    pid = list(range(level + 1))
    p = np.array(oc.primes[:level + 1], dtype=np.uint64)[:, None]
    babies = sorted({o - (o // bstep) * bstep for o in offsets} - {0})
    rot = {0: (c0, c1)}
    if babies:
        ks = [pow(gal_of(b), -1, 2 * oc.N) for b in babies]
        h0, h1 = oc.rotate_hoisted(level, c0, c1, ks, [keys[b][0] for b in babies], [keys[b][1] for b in babies])
        for i, b in enumerate(babies):
            rot[b] = (h0[i], h1[i])
    groups = {}
    for k, o in enumerate(offsets):
        groups.setdefault(o // bstep, []).append(k)
    acc = None
    for g in sorted(groups):
        s0 = np.zeros_like(c0)
        s1 = np.zeros_like(c1)
        for k in groups[g]:
            b = offsets[k] - g * bstep
            s0 = (s0 + oc.polymul(rot[b][0], pts[k], pid)) % p
            s1 = (s1 + oc.polymul(rot[b][1], pts[k], pid)) % p
        if g:
            G = g * bstep
            s0, s1 = oc.rotate(level, s0, s1, pow(gal_of(G), -1, 2 * oc.N), *keys[G])
        acc = (s0, s1) if acc is None else ((acc[0] + s0) % p, (acc[1] + s1) % p)
    return acc


@pytest.mark.parametrize("offsets,bstep", [(list(range(16)), 4), ([-7, -3, -1, 0, 2, 5, 9, 13], 4), ([0], 4)])
def test_linear_transform_bitexact_vs_oracle(offsets, bstep):
    import pyfideslib_b200 as F

    cc, oc = make_pair(12, 8, 3, 3)
    level = 6
    rots = F.CryptoContext.linear_transform_rotations(offsets, bstep)
    keys = {}
    for i, r in enumerate(rots):
        g = cc.rotation_galois(r)
        keys[r] = rand_key(oc, 500 + 2 * i)
        cc.upload_galois_key(g, *keys[r])
    c0, c1 = rand_ct(oc, level, 71)
    x = cc.upload(c0, c1)
    pts_r = [oc.random(list(range(level + 1)), 900 + k) for k in range(len(offsets))]
    pts = [_upload_pt(cc, m, level) for m in pts_r]
    for rescale in (False, True):
        got = cc.EvalLinearTransform(x, offsets, pts, bstep, rescale=rescale).download()
        w0, w1 = _oracle_bsgs(oc, level, c0, c1, offsets, pts_r, bstep, keys, cc.rotation_galois)
        if rescale:
            w0, w1 = oc.rescale(level, w0), oc.rescale(level, w1)
        assert np.array_equal(got[0], w0) and np.array_equal(got[1], w1), (offsets, rescale)


@pytest.mark.parametrize("offsets,bstep", [(list(range(16)), 4), ([-9, -4, -1, 0, 3, 6, 11], 4),
                                           (list(range(-20, 44)), 8)])
def test_linear_transform_matches_fp64(offsets, bstep):
    import pyfideslib_b200 as F

    cc = F.CryptoContext(log_n=12, num_q=6, dnum=2)
    slots = cc.N // 2
    sk = cc.KeyGen(seed=3, hamming_weight=64)
    cc.EvalRotateKeyGen(sk, F.CryptoContext.linear_transform_rotations(offsets, bstep))
    rng = np.random.default_rng(len(offsets))
    x = rng.uniform(-1, 1, slots) + 1j * rng.uniform(-1, 1, slots)
    diags = {o: rng.uniform(-1, 1, slots) for o in offsets}
    ct = cc.Encrypt(sk, x, slots=slots)
    offs, pts = cc.prepare_linear_transform(diags, bstep, level=ct.level, slots=slots)
    y = cc.EvalLinearTransform(ct, offs, pts, bstep, rescale=True)
    got = cc.Decrypt(sk, y, slots=slots)
    want = np.zeros(slots, dtype=np.complex128)
    for o, d in diags.items():
        want += d * np.roll(x, -o)
    err = np.max(np.abs(got - want))
    assert err < 1e-6, err
    assert y.level == ct.level - 1


def test_linear_transform_batch_equals_single():
    """One transform of several ciphertexts (giant rotations batched over
    the inputs) equals one call per ciphertext, bit for bit."""
    import pyfideslib_b200 as F

    cc, oc = make_pair(12, 8, 3, 3)
    level, offsets, bstep = 6, [-7, -3, -1, 0, 2, 5, 9, 13], 4
    for i, r in enumerate(F.CryptoContext.linear_transform_rotations(offsets, bstep)):
        cc.upload_galois_key(cc.rotation_galois(r), *rand_key(oc, 700 + 2 * i))
    xs = [cc.upload(*rand_ct(oc, level, 800 + 2 * u)) for u in range(3)]
    pts = [_upload_pt(cc, oc.random(list(range(level + 1)), 850 + k), level) for k in range(len(offsets))]
    outs = cc.EvalLinearTransformBatch(xs, offsets, pts, bstep, rescale=True)
    for x, o in zip(xs, outs):
        w = cc.EvalLinearTransform(x, offsets, pts, bstep, rescale=True).download()
        g = o.download()
        assert np.array_equal(g[0], w[0]) and np.array_equal(g[1], w[1])


def _oracle_bsgs_giant_sum(oc, level, c0, c1, offsets, pts, bstep, keys, gal_of):
    """The transform with its giant-step rotations added in the extended basis
    (Q and the special moduli) before one ModDown: per giant step the oracle's
    own steps of a rotation -- ModUp, inner product, P c0, automorphism --
    without the ModDown, then the sum brought down once."""
    n = level + 1
    pid = list(range(n))
    p = np.array(oc.primes[:n], dtype=np.uint64)[:, None]
    pe = np.array(oc.primes[:n] + oc.primes[oc.L:oc.L + oc.K], dtype=np.uint64)[:, None]
    P = 1
    for x in oc.primes[oc.L:oc.L + oc.K]:
        P *= x
    pmod = np.repeat(np.array([[P % q] for q in oc.primes[:n]], dtype=np.uint64), oc.N, axis=1)
    babies = sorted({o - (o // bstep) * bstep for o in offsets} - {0})
    rot = {0: (c0, c1)}
    if babies:
        ks = [pow(gal_of(b), -1, 2 * oc.N) for b in babies]
        h0, h1 = oc.rotate_hoisted(level, c0, c1, ks, [keys[b][0] for b in babies], [keys[b][1] for b in babies])
        for i, b in enumerate(babies):
            rot[b] = (h0[i], h1[i])
    groups = {}
    for k, o in enumerate(offsets):
        groups.setdefault(o // bstep, []).append(k)
    acc, ext = None, None
    for g in sorted(groups):
        s0 = np.zeros_like(c0)
        s1 = np.zeros_like(c1)
        for k in groups[g]:
            b = offsets[k] - g * bstep
            s0 = (s0 + oc.polymul(rot[b][0], pts[k], pid)) % p
            s1 = (s1 + oc.polymul(rot[b][1], pts[k], pid)) % p
        if g == 0:
            acc = (s0, s1)
            continue
        kb, ka = keys[g * bstep]
        xb, xa = oc.ks_inner(level, oc.modup(level, s1), kb, ka)
        xb[:n] = (xb[:n] + oc.polymul(s0, pmod, pid)) % p
        gal = pow(gal_of(g * bstep), -1, 2 * oc.N)
        e = (oc.automorph(xb, gal), oc.automorph(xa, gal))
        ext = e if ext is None else ((ext[0] + e[0]) % pe, (ext[1] + e[1]) % pe)
    if ext is not None:
        d = (oc.moddown(level, ext[0]), oc.moddown(level, ext[1]))
        acc = d if acc is None else ((acc[0] + d[0]) % p, (acc[1] + d[1]) % p)
    return acc


@pytest.mark.parametrize("offsets,bstep", [(list(range(16)), 4), ([-7, -3, -1, 0, 2, 5, 9, 13], 4),
                                           ([5, 6, 9, 14], 4)])
def test_linear_transform_giant_sum_bitexact_vs_oracle(offsets, bstep):
    """fides_set_giant_step_moddown(ctx, 2): each input's giant-step rotations
    are added before one ModDown.  Bit for bit the oracle composition of the
    same steps, single and batched over inputs, with and without rescale."""
    import pyfideslib_b200 as F
    from pyfideslib_b200._capi import lib

    cc, oc = make_pair(12, 8, 3, 3)
    assert lib.fides_set_giant_step_moddown(cc._h, 2) == 0
    level = 6
    keys = {}
    for i, r in enumerate(F.CryptoContext.linear_transform_rotations(offsets, bstep)):
        keys[r] = rand_key(oc, 600 + 2 * i)
        cc.upload_galois_key(cc.rotation_galois(r), *keys[r])
    cts = [rand_ct(oc, level, 1071 + 2 * u) for u in range(2)]
    xs = [cc.upload(*ct) for ct in cts]
    pts_r = [oc.random(list(range(level + 1)), 1900 + k) for k in range(len(offsets))]
    pts = [_upload_pt(cc, m, level) for m in pts_r]
    for rescale in (False, True):
        want = []
        for c0, c1 in cts:
            w0, w1 = _oracle_bsgs_giant_sum(oc, level, c0, c1, offsets, pts_r, bstep, keys, cc.rotation_galois)
            want.append((oc.rescale(level, w0), oc.rescale(level, w1)) if rescale else (w0, w1))
        got = cc.EvalLinearTransform(xs[0], offsets, pts, bstep, rescale=rescale).download()
        assert np.array_equal(got[0], want[0][0]) and np.array_equal(got[1], want[0][1]), (offsets, rescale)
        for o, w in zip(cc.EvalLinearTransformBatch(xs, offsets, pts, bstep, rescale=rescale), want):
            g = o.download()
            assert np.array_equal(g[0], w[0]) and np.array_equal(g[1], w[1]), (offsets, rescale, "batch")
    assert lib.fides_set_giant_step_moddown(cc._h, 3) == 1  # BAD_ARG


@pytest.mark.parametrize("offsets,bstep,nx", [(list(range(32)), 4, 5), (list(range(0, 40)), 32, 2)])
def test_linear_transform_giant_sum_chunks(offsets, bstep, nx):
    """More giant-step terms than one key-switch batch holds (5 inputs x 7
    giant steps = 35 > 32: the batches are formed of whole inputs, so each
    input still takes one ModDown), and 31 baby steps with one giant step:
    still bit for bit the oracle composition."""
    import pyfideslib_b200 as F
    from pyfideslib_b200._capi import lib

    cc, oc = make_pair(12, 8, 3, 3)
    assert lib.fides_set_giant_step_moddown(cc._h, 2) == 0
    level = 5
    keys = {}
    for i, r in enumerate(F.CryptoContext.linear_transform_rotations(offsets, bstep)):
        keys[r] = rand_key(oc, 3000 + 2 * i)
        cc.upload_galois_key(cc.rotation_galois(r), *keys[r])
    cts = [rand_ct(oc, level, 3500 + 2 * u) for u in range(nx)]
    xs = [cc.upload(*ct) for ct in cts]
    pts_r = [oc.random(list(range(level + 1)), 3900 + k) for k in range(len(offsets))]
    pts = [_upload_pt(cc, m, level) for m in pts_r]
    outs = cc.EvalLinearTransformBatch(xs, offsets, pts, bstep, rescale=False)
    for (c0, c1), o in zip(cts, outs):
        w0, w1 = _oracle_bsgs_giant_sum(oc, level, c0, c1, offsets, pts_r, bstep, keys, cc.rotation_galois)
        g = o.download()
        assert np.array_equal(g[0], w0) and np.array_equal(g[1], w1)
