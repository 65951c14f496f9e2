"""Batched evaluation (config 4 shape, scaled down): results of the batched
entry points are identical to the per-operation path and to the oracle."""
import numpy as np
import pytest

from gpu_helpers import make_pair, rand_ct, rand_key

pytestmark = pytest.mark.gpu


def test_hmult_batch_uneven_levels_equals_per_op():
    cc, oc = make_pair(12, 10, 4, 3)
    kb, ka = rand_key(oc, 77)
    cc.upload_relin_key(kb, ka)
    rng = np.random.default_rng(3)
    levels = [int(x) for x in rng.integers(0, 10, size=40)]  # > 32 per level group would chunk too
    A, B, raw = [], [], []
    for i, lv in enumerate(levels):
        a0, a1 = rand_ct(oc, lv, 1000 + 4 * i)
        b0, b1 = rand_ct(oc, lv, 1002 + 4 * i)
        A.append(cc.upload(a0, a1))
        B.append(cc.upload(b0, b1))
        raw.append((a0, a1, b0, b1))
    for rs in (True, False):
        outs = cc.EvalMultBatch(A, B, rescale=rs)
        for i, lv in enumerate(levels):
            got = outs[i].download()
            want = cc.EvalMult(A[i], B[i], rescale=rs).download()
            assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), (i, lv, rs)
        # spot-check against the oracle
        for i in (0, 7, 23):
            w = oc.hmult(levels[i], *raw[i], kb, ka, rescale=rs and levels[i] > 0)
            g = outs[i].download()
            assert np.array_equal(g[0], w[0]) and np.array_equal(g[1], w[1])


def test_hmult_batch_same_level_more_than_32():
    cc, oc = make_pair(11, 6, 2, 2)
    kb, ka = rand_key(oc, 5)
    cc.upload_relin_key(kb, ka)
    A, B = [], []
    for i in range(37):
        A.append(cc.upload(*rand_ct(oc, 5, 10 * i)))
        B.append(cc.upload(*rand_ct(oc, 5, 10 * i + 5)))
    outs = cc.EvalMultBatch(A, B, rescale=True)
    for i in (0, 31, 32, 36):
        want = cc.EvalMult(A[i], B[i], rescale=True).download()
        got = outs[i].download()
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def test_rotate_batch_equals_per_op_and_oracle():
    cc, oc = make_pair(12, 8, 3, 3)
    idx = [1, 3, -2, 17, 1, 100]
    keys = {}
    for i, r in enumerate(sorted(set(idx))):
        g = cc.rotation_galois(r)
        keys[g] = rand_key(oc, 400 + 2 * i)
        cc.upload_galois_key(g, *keys[g])
    levels = [7, 7, 4, 2, 4, 7]
    cts, raw = [], []
    for i, lv in enumerate(levels):
        c0, c1 = rand_ct(oc, lv, 50 + 3 * i)
        cts.append(cc.upload(c0, c1))
        raw.append((c0, c1))
    outs = cc.EvalRotateBatch(cts, idx)
    for i, r in enumerate(idx):
        g = cc.rotation_galois(r)
        want = oc.rotate(levels[i], *raw[i], pow(g, -1, 2 * oc.N), *keys[g])
        got = outs[i].download()
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), i


def test_hoisted_more_than_32_rotations():
    cc, oc = make_pair(11, 5, 2, 2)
    idx = list(range(1, 41))
    cc_keys = {}
    for i, r in enumerate(idx):
        g = cc.rotation_galois(r)
        cc_keys[g] = rand_key(oc, 900 + 2 * i)
        cc.upload_galois_key(g, *cc_keys[g])
    c0, c1 = rand_ct(oc, 4, 8)
    ct = cc.upload(c0, c1)
    outs = cc.EvalFastRotation(ct, idx)
    for i in (0, 31, 32, 39):
        want = cc.EvalRotate(ct, idx[i]).download()
        got = outs[i].download()
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def test_graph_plan_matches_eager_and_replays_new_inputs():
    """Config-4 shape, scaled down: uneven levels, HMult+Relin+Rescale then one
    rotation per pair, captured once and replayed."""
    cc, oc = make_pair(12, 8, 3, 3)
    kb, ka = rand_key(oc, 31)
    cc.upload_relin_key(kb, ka)
    rng = np.random.default_rng(9)
    n = 12
    levels = [int(x) for x in rng.integers(1, 8, size=n)]
    idx = [int(x) for x in rng.integers(1, cc.N // 2, size=n)]
    for i, r in enumerate(sorted(set(idx))):
        cc.upload_galois_key(cc.rotation_galois(r), *rand_key(oc, 600 + 2 * i))
    A = [cc.upload(*rand_ct(oc, lv, 7 * i)) for i, lv in enumerate(levels)]
    B = [cc.upload(*rand_ct(oc, lv, 7 * i + 3)) for i, lv in enumerate(levels)]
    plan, outs = cc.plan_hmult_rotate(A, B, idx, rescale=True)
    for rep in range(2):
        if rep == 1:  # new inputs through the same captured graph
            for i, lv in enumerate(levels):
                cc.write(A[i], *rand_ct(oc, lv, 999 + i))
        plan.launch()
        cc.Synchronize()
        prod = cc.EvalMultBatch(A, B, rescale=True)
        want = cc.EvalRotateBatch(prod, idx)
        for i in range(n):
            g0, g1 = outs[i].download()
            w0, w1 = want[i].download()
            assert np.array_equal(g0, w0) and np.array_equal(g1, w1), (rep, i)


def test_async_upload_download_pipeline_equals_sync():
    """Uploads on the copy stream, batched HMult, asynchronous downloads into
    pinned memory and frees, three rounds queued back to back (the pattern of
    the end-to-end benchmark): every result equals the synchronous path."""
    import ctypes as C

    import torch

    from pyfideslib_b200._capi import check, lib, u64p, vp

    cc, oc = make_pair(12, 6, 2, 3)
    kb, ka = rand_key(oc, 5)
    cc.upload_relin_key(kb, ka)
    lv, B, N = 5, 4, cc.N
    rounds = []
    for r in range(3):
        pins = []
        for i in range(B):
            pair = []
            for s in range(2):
                t = torch.empty((2, lv + 1, N), dtype=torch.int64, pin_memory=True)
                a = t.numpy().view(np.uint64)
                a[0], a[1] = rand_ct(oc, lv, 1000 * r + 10 * i + 2 * s)
                pair.append((t, a))
            pins.append(pair)
        rounds.append(pins)
    outs = [__import__("pyfideslib_b200").Ciphertext(cc) for _ in range(B)]
    O = (vp * B)(*[o._h for o in outs])
    host_out = [[torch.empty((2, lv, N), dtype=torch.int64, pin_memory=True) for _ in range(B)] for _ in range(3)]
    for r in range(3):
        ha = [vp() for _ in range(B)]
        hb = [vp() for _ in range(B)]
        for i in range(B):
            a, b = rounds[r][i][0][1], rounds[r][i][1][1]
            check(lib.fides_ct_upload(cc._h, a[0].ctypes.data_as(u64p), a[1].ctypes.data_as(u64p), lv, cc.scale, 1,
                                      N // 2, C.byref(ha[i])), cc._h)
            check(lib.fides_ct_upload(cc._h, b[0].ctypes.data_as(u64p), b[1].ctypes.data_as(u64p), lv, cc.scale, 1,
                                      N // 2, C.byref(hb[i])), cc._h)
        check(lib.fides_hmult_batch(cc._h, B, (vp * B)(*[h.value for h in ha]), (vp * B)(*[h.value for h in hb]),
                                    O, 1), cc._h)
        for i in range(B):
            ho = host_out[r][i].numpy().view(np.uint64)
            check(lib.fides_ct_download_async(cc._h, outs[i]._h, ho[0].ctypes.data_as(u64p),
                                              ho[1].ctypes.data_as(u64p)), cc._h)
            lib.fides_ct_free(cc._h, ha[i])
            lib.fides_ct_free(cc._h, hb[i])
    cc.Synchronize()
    for r in range(3):
        for i in range(B):
            a, b = rounds[r][i][0][1], rounds[r][i][1][1]
            want = oc.hmult(lv, a[0], a[1], b[0], b[1], kb, ka, rescale=True)
            got = host_out[r][i].numpy().view(np.uint64)
            assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), (r, i)
