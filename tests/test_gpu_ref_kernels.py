"""The reference's own GPU kernels beside the oracle and this library, on the same B200.

oracle/_ref/libfidesref_gpu.so is the reference's src/NTT.cu,
src/CKKS/Conv.cu and src/CKKS/ElemenwiseBatchKernels.cu compiled unmodified,
with oracle/ref_gpu.cu filling the constant and table blocks their kernels
read and launching them with the reference's geometry.  The library is built
where the reference tree is mounted (`make -C oracle ref-gpu`) and travels
prebuilt; without it these tests skip.

* Parity, bit for bit: the forward and inverse NTT pairs (NTT_ / INTT_)
  against the oracle's transforms and this library's; the ModUp conversion
  (DecompAndModUpConv) and the ModDown conversion (ModDown2) against the
  exact base-conversion sums over the oracle's CRT constants; the key-switch
  inner product (fusedDotKSK_2_) against the oracle's, at logN 12 and at the
  HMult shape (N = 2^16, L = 30, K = 10, dnum = 3); the tensor product
  (binomialMult_), the automorphism (automorph_multi_) and the hoisted
  rotations' inner product (hoistedRotateDotKSK_2_) against the oracle's, at
  logN 12 and at config 3's shape.
* Timing at the HMult shape and at config 3's, CUDA events, printed for the
  record: each reference kernel on the work one batched step gives it, and
  this library's batched NTT / INTT on the same residues.
"""
import ctypes as C
import os

import numpy as np
import pytest

from gpu_helpers import from_dev, make_pair, to_dev

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libfidesref_gpu.so")


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(LIB):
        pytest.skip("the reference's GPU kernels were not built (make -C oracle ref-gpu needs the reference tree)")
    lib = C.CDLL(LIB)
    u64p = C.POINTER(C.c_uint64)
    vp = C.c_void_p
    lib.refgpu_init.argtypes = [C.c_int, C.c_int, u64p, u64p]
    lib.refgpu_transform.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, vp]
    lib.refgpu_set_keyswitch.argtypes = [C.c_int, C.c_int, C.c_int, u64p, u64p, u64p, u64p]
    lib.refgpu_modup_conv.argtypes = [vp, vp, C.c_int, C.c_int, vp]
    lib.refgpu_moddown_conv.argtypes = [vp, vp, C.c_int, vp]
    lib.refgpu_dot.argtypes = [vp, vp, vp, vp, vp, vp, vp]
    lib.refgpu_binomial.argtypes = [vp, vp, vp, vp, vp, C.c_int, vp]
    lib.refgpu_automorph.argtypes = [vp, vp, C.c_int, C.c_int, vp]
    lib.refgpu_hoisted_dot.argtypes = [vp, vp, vp, C.c_int, vp, vp, vp, vp, vp, vp]
    for f in ("refgpu_init", "refgpu_transform", "refgpu_set_keyswitch", "refgpu_modup_conv",
              "refgpu_moddown_conv", "refgpu_dot", "refgpu_binomial", "refgpu_automorph", "refgpu_hoisted_dot"):
        getattr(lib, f).restype = C.c_int
    lib.refgpu_release.argtypes = []
    yield lib
    lib.refgpu_release()


def _u64p(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint64))


def _stream():
    import torch

    return torch.cuda.current_stream().cuda_stream


def _init(ref, oc, nprimes):
    psi = np.array([int(oc.psi_tables(i)[0][oc.N // 2]) for i in range(nprimes)], dtype=np.uint64)
    q = np.array(oc.primes[:nprimes], dtype=np.uint64)
    assert ref.refgpu_init(oc.logN, nprimes, _u64p(q), _u64p(psi)) == 0


def _set_keyswitch(ref, oc):
    """ModUp constants of every (digit, level) and the ModDown constants,
    from the oracle (or_modup_consts / or_moddown_consts)."""
    L, K, D, a = oc.L, oc.K, oc.dnum, oc.alpha
    hat_inv = np.zeros((D, L, a), dtype=np.uint64)
    hat_mod = np.zeros((D, L, a, L + K), dtype=np.uint64)
    for d in range(D):
        for lv in range(d * a, L):
            hat_inv[d, lv], hat_mod[d, lv] = oc.modup_consts(lv, d)
    phat_inv, phat_mod, _ = oc.moddown_consts()
    assert ref.refgpu_set_keyswitch(L, K, D, _u64p(hat_inv), _u64p(hat_mod), _u64p(phat_inv),
                                    _u64p(np.ascontiguousarray(phat_mod))) == 0


def _digit_targets(oc, level, d):
    """Prime ids of digit d's ModUp outputs in the reference's list order:
    the special primes, then the ciphertext primes <= level outside it."""
    lo, hi = d * oc.alpha, min((d + 1) * oc.alpha, oc.L) - 1
    return [oc.L + k for k in range(oc.K)] + [q for q in range(level + 1) if q < lo or q > hi]


def _conv_expected(x_limbs, hat_inv, in_primes, hat_mod_rows, out_primes):
    """Exact base conversion: out_t = sum_i [x_i hat_inv_i]_{q_i} * hat_mod[i][t] mod t."""
    s = [(x.astype(object) * int(h)) % int(q) for x, h, q in zip(x_limbs, hat_inv, in_primes)]
    out = []
    for t, pt in enumerate(out_primes):
        acc = sum(si * int(row[t]) for si, row in zip(s, hat_mod_rows))
        out.append(np.array(acc % int(pt), dtype=np.uint64))
    return np.stack(out)


@pytest.mark.parametrize("logN,L", [(12, 8), (16, 30)])
def test_reference_transforms_equal_oracle_and_ours(ref, logN, L):
    cc, oc = make_pair(logN, L, 3, 3)
    _init(ref, oc, L)
    pid = list(range(L))
    x = oc.random(pid, 700 + logN)
    pm1 = np.array([q - 1 for q in oc.primes[:L]], dtype=np.uint64)[:, None]
    import torch

    for inp in (x, np.ascontiguousarray(np.broadcast_to(pm1, x.shape))):
        for inverse in (0, 1):
            want = oc.ntt(inp, pid, inverse=bool(inverse))
            d = to_dev(inp)
            aux = torch.empty_like(d)
            assert ref.refgpu_transform(d.data_ptr(), aux.data_ptr(), 0, L, inverse, _stream()) == 0
            torch.cuda.synchronize()
            assert np.array_equal(from_dev(d), want), ("reference", inverse)
            ours = to_dev(inp)
            cc.ntt(ours.data_ptr(), 0, L, inverse=bool(inverse))
            cc.Synchronize()
            assert np.array_equal(from_dev(ours), want), ("ours", inverse)


def test_reference_conversions_equal_exact_sums(ref):
    """DecompAndModUpConv for every digit at the top level and at a level
    inside digit 1, and ModDown2, at logN 12 (L = 8, K = 3, dnum = 3)."""
    import torch

    cc, oc = make_pair(12, 8, 3, 3)
    _init(ref, oc, oc.L + oc.K)
    _set_keyswitch(ref, oc)
    for level in (oc.L - 1, 4):
        x = oc.random(list(range(level + 1)), 900 + level)
        xd = to_dev(x)
        for d in range(oc.num_digits(level)):
            lo, hi = d * oc.alpha, min((d + 1) * oc.alpha - 1, level)
            tg = _digit_targets(oc, level, d)
            out = torch.empty((len(tg), oc.N), dtype=torch.int64, device="cuda")
            assert ref.refgpu_modup_conv(xd.data_ptr(), out.data_ptr(), level, d, _stream()) == 0
            torch.cuda.synchronize()
            hi_inv, hm = oc.modup_consts(level, d)
            cnt = hi - lo + 1
            want = _conv_expected(x[lo:hi + 1], hi_inv[:cnt], oc.primes[lo:hi + 1],
                                  [hm[i][tg] for i in range(cnt)], [oc.primes[t] for t in tg])
            assert np.array_equal(from_dev(out), want), (level, d)
        y = oc.random([oc.L + k for k in range(oc.K)], 950 + level)
        out = torch.empty((level + 1, oc.N), dtype=torch.int64, device="cuda")
        assert ref.refgpu_moddown_conv(to_dev(y).data_ptr(), out.data_ptr(), level, _stream()) == 0
        torch.cuda.synchronize()
        phat_inv, phat_mod, _ = oc.moddown_consts()
        want = _conv_expected(y, phat_inv, oc.primes[oc.L:], [phat_mod[k][:level + 1] for k in range(oc.K)],
                              oc.primes[:level + 1])
        assert np.array_equal(from_dev(out), want), level


def _dot_inputs(oc, seed):
    """Digits in the oracle's layout ([dnum][L+K][N], own limbs = x) and the
    same values in the reference's per-digit list order."""
    L, K, D = oc.L, oc.K, oc.dnum
    level = L - 1
    ext = list(range(L)) + [L + k for k in range(K)]
    x = oc.random(list(range(L)), seed)
    dig_or = np.empty((D, L + K, oc.N), dtype=np.uint64)
    dig_ref = np.zeros((D, L + K, oc.N), dtype=np.uint64)
    for d in range(D):
        lo, hi = d * oc.alpha, min((d + 1) * oc.alpha, L) - 1
        vals = oc.random(ext, seed + 1 + d)
        vals[lo:hi + 1] = x[lo:hi + 1]
        dig_or[d] = vals
        for pos, t in enumerate(_digit_targets(oc, level, d)):
            dig_ref[d, pos] = vals[t]  # ext position of prime t is t at the top level
    kpid = list(range(L + K)) * D
    kb = oc.random(kpid, seed + 20).reshape(D, L + K, oc.N)
    ka = oc.random(kpid, seed + 21).reshape(D, L + K, oc.N)
    return x, dig_or, dig_ref, kb, ka


@pytest.mark.parametrize("logN,L,K", [(12, 8, 3), (16, 30, 10)])
def test_reference_dot_equals_oracle(ref, logN, L, K):
    import torch

    cc, oc = make_pair(logN, L, K, 3)
    _init(ref, oc, L + K)
    _set_keyswitch(ref, oc)
    x, dig_or, dig_ref, kb, ka = _dot_inputs(oc, 1300 + logN)
    want_b, want_a = oc.ks_inner(L - 1, dig_or, kb, ka)
    t = [to_dev(v) for v in (dig_ref, x, kb, ka)]
    ob = torch.empty((L + K, oc.N), dtype=torch.int64, device="cuda")
    oa = torch.empty_like(ob)
    assert ref.refgpu_dot(t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), t[3].data_ptr(), ob.data_ptr(),
                          oa.data_ptr(), _stream()) == 0
    torch.cuda.synchronize()
    assert np.array_equal(from_dev(ob), want_b)
    assert np.array_equal(from_dev(oa), want_a)


def _time(fn, reps=10, warm=3):
    import torch

    s = torch.cuda.current_stream()
    for _ in range(warm):
        fn()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for r in range(reps):
        fn()
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps * 1e3


def test_reference_kernel_timing_hmult_shape(ref):
    """Device time of each reference kernel at N = 2^16, L = 30, K = 10,
    dnum = 3, level 29, on the work of one batched HMult step of 32 pairs
    where that is one launch, else per launch; this library's batched
    forward / inverse NTT of the same 32 x 30 limbs beside it."""
    import torch

    cc, oc = make_pair(16, 30, 10, 3)
    L, K, N = oc.L, oc.K, oc.N
    _init(ref, oc, L)
    nl, nb = 30, 32
    bufs = [torch.randint(0, 2 ** 40, (nb * nl, N), dtype=torch.int64, device="cuda") for _ in range(2)]
    aux = torch.empty_like(bufs[0])
    a, b = bufs[0].clone(), bufs[0].clone()
    assert ref.refgpu_transform(a.data_ptr(), aux.data_ptr(), 0, nb * nl, 0, _stream()) == 0
    cc.ntt_batch(b.data_ptr(), nl * N, nb, 0, nl)
    cc.Synchronize()
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    del a, b
    res = {}
    st = torch.cuda.ExternalStream(cc.stream_ptr())
    for inv in (0, 1):
        k = [0]

        def ref_t():
            ref.refgpu_transform(bufs[k[0] % 2].data_ptr(), aux.data_ptr(), 0, nb * nl, inv, _stream())
            k[0] += 1

        res["ref_" + ("intt" if inv else "ntt")] = _time(ref_t)
        with torch.cuda.stream(st):
            def ours_t():
                cc.ntt_batch(bufs[k[0] % 2].data_ptr(), nl * N, nb, 0, nl, inverse=bool(inv))
                k[0] += 1

            res["ours_" + ("intt" if inv else "ntt")] = _time(ours_t)
    del bufs, aux
    torch.cuda.synchronize()
    _init(ref, oc, L + K)
    _set_keyswitch(ref, oc)
    level = L - 1
    x = to_dev(oc.random(list(range(L)), 1500))
    outs = [torch.empty((K + L - oc.alpha, N), dtype=torch.int64, device="cuda") for _ in range(oc.dnum)]
    res["ref_modup_conv_3_digits"] = _time(lambda: [ref.refgpu_modup_conv(x.data_ptr(), outs[d].data_ptr(), level,
                                                                           d, _stream()) for d in range(oc.dnum)])
    y = to_dev(oc.random([L + k for k in range(K)], 1501))
    md = torch.empty((L, N), dtype=torch.int64, device="cuda")
    res["ref_moddown_conv_1_poly"] = _time(lambda: ref.refgpu_moddown_conv(y.data_ptr(), md.data_ptr(), level,
                                                                           _stream()))
    xs, dig_or, dig_ref, kb, ka = _dot_inputs(oc, 1600)
    t = [to_dev(v) for v in (dig_ref, xs, kb, ka)]
    ob = torch.empty((L + K, N), dtype=torch.int64, device="cuda")
    oa = torch.empty_like(ob)
    res["ref_dot_1_element"] = _time(lambda: ref.refgpu_dot(t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(),
                                                            t[3].data_ptr(), ob.data_ptr(), oa.data_ptr(), _stream()))
    print("\nreference kernels at N=2^16 L=30 K=10 dnum=3 (us, CUDA events): " +
          ", ".join("%s %.1f" % kv for kv in res.items()))
    assert all(v > 0 for v in res.values())


def _slots(logN, g):
    """slot(g, j) for every j: the automorphism's image of evaluation slot j
    (bit-reversed order), as the reference's automorph_slot computes it."""
    N = 1 << logN
    j = np.arange(N, dtype=np.uint64)
    br = np.zeros_like(j)
    for b in range(logN):
        br |= ((j >> np.uint64(b)) & np.uint64(1)) << np.uint64(logN - 1 - b)
    r = (((2 * br + 1) * np.uint64(g)) & np.uint64(2 * N - 1)) >> np.uint64(1)
    out = np.zeros_like(r)
    for b in range(logN):
        out |= ((r >> np.uint64(b)) & np.uint64(1)) << np.uint64(logN - 1 - b)
    return out.astype(np.int64)


def _ref_ptrs(arrs):
    return (C.c_void_p * len(arrs))(*[a.data_ptr() for a in arrs])


def _hoisted_expected(oc, x, dig_or, c0, kbs, kas, gals):
    """oracle inner product + P c0 on the ciphertext primes, then scattered to
    the automorphism's slots: out[slot(g, j)] = value[j]."""
    L = oc.L
    _, _, p_inv = oc.moddown_consts()
    P = np.array([pow(int(v), -1, int(q)) for v, q in zip(p_inv, oc.primes[:L])], dtype=np.uint64)
    pc0 = oc.polymul(c0, np.ascontiguousarray(np.broadcast_to(P[:, None], c0.shape)), list(range(L)))
    q = np.array(oc.primes[:L], dtype=np.uint64)[:, None]
    want = []
    for kb, ka, g in zip(kbs, kas, gals):
        ob, oa = oc.ks_inner(L - 1, dig_or, kb, ka)
        ob[:L] = (ob[:L] + pc0) % q
        sl = _slots(oc.logN, g)
        wb, wa = np.empty_like(ob), np.empty_like(oa)
        wb[:, sl] = ob
        wa[:, sl] = oa
        want.append((wb, wa))
    return want


@pytest.mark.parametrize("logN,L,K,qi_bits", [(12, 8, 3, 50), (16, 20, 6, 40)])
def test_reference_tensor_automorph_hoisted_equal_oracle(ref, logN, L, K, qi_bits):
    """binomialMult_ against the oracle's tensor product, automorph_multi_
    against its automorphism, and hoistedRotateDotKSK_2_ (4 rotations of one
    ModUp, plain-layout keys) against the oracle's inner product permuted and
    with P c0 added: at logN 12 and at the hoisted-rotation shape of config 3
    (N = 2^16, L = 20 x 40-bit, K = 6)."""
    import torch

    import pyfideslib_b200 as F
    from oracle import oracle as O

    cc = F.CryptoContext(log_n=logN, num_q=L, dnum=3, num_p=K, qi_bits=qi_bits)
    oc = O.Ctx(cc.logN, cc.q, cc.p, cc.dnum)
    _init(ref, oc, L + K)
    lv = L - 1
    a0, a1, b0, b1 = (oc.random(list(range(L)), 2000 + s) for s in range(4))
    e0, e1, e2 = oc.tensor(lv, a0, a1, b0, b1)
    t = [to_dev(v) for v in (a0, a1, b0, b1)]
    c2 = torch.empty_like(t[0])
    assert ref.refgpu_binomial(t[0].data_ptr(), t[1].data_ptr(), c2.data_ptr(), t[2].data_ptr(), t[3].data_ptr(),
                               L, _stream()) == 0
    torch.cuda.synchronize()
    assert np.array_equal(from_dev(t[0]), e0) and np.array_equal(from_dev(t[1]), e1)
    assert np.array_equal(from_dev(c2), e2)
    gals = [cc.rotation_galois(r) for r in (1, -3, 2 ** (logN - 3))] + [2 * cc.N - 1]
    for g in gals:
        out = torch.empty_like(t[2])
        assert ref.refgpu_automorph(t[2].data_ptr(), out.data_ptr(), L, g, _stream()) == 0
        torch.cuda.synchronize()
        assert np.array_equal(from_dev(out), oc.automorph(b0, g)), g
    _set_keyswitch(ref, oc)
    x, dig_or, dig_ref, _, _ = _dot_inputs(oc, 2100)
    c0 = oc.random(list(range(L)), 2150)
    kpid = list(range(L + K)) * oc.dnum
    kbs = [oc.random(kpid, 2200 + 2 * r).reshape(oc.dnum, L + K, oc.N) for r in range(len(gals))]
    kas = [oc.random(kpid, 2201 + 2 * r).reshape(oc.dnum, L + K, oc.N) for r in range(len(gals))]
    want = _hoisted_expected(oc, x, dig_or, c0, kbs, kas, gals)
    dd, dx, dc0 = to_dev(dig_ref), to_dev(x), to_dev(c0)
    dkb, dka = [to_dev(k) for k in kbs], [to_dev(k) for k in kas]
    ob = [torch.empty((L + K, oc.N), dtype=torch.int64, device="cuda") for _ in gals]
    oa = [torch.empty_like(o) for o in ob]
    G = (C.c_int32 * len(gals))(*gals)
    assert ref.refgpu_hoisted_dot(dd.data_ptr(), dx.data_ptr(), dc0.data_ptr(), len(gals), _ref_ptrs(dkb),
                                  _ref_ptrs(dka), G, _ref_ptrs(ob), _ref_ptrs(oa), _stream()) == 0
    torch.cuda.synchronize()
    for r, (wb, wa) in enumerate(want):
        assert np.array_equal(from_dev(ob[r]), wb), r
        assert np.array_equal(from_dev(oa[r]), wa), r


def test_reference_hoisted_timing_c3_shape(ref):
    """hoistedRotateDotKSK_2_ over the 32 rotations of config 3 (N = 2^16,
    L = 20 x 40-bit, K = 6, dnum = 3, level 19), one launch with the
    reference's geometry; binomialMult_ and automorph_multi_ of one
    top-level HMult-shape element (N = 2^16, 30 limbs).  Device time, CUDA
    events, printed for the record."""
    import torch

    import pyfideslib_b200 as F
    from oracle import oracle as O

    cc = F.CryptoContext(log_n=16, num_q=20, dnum=3, qi_bits=40)
    oc = O.Ctx(cc.logN, cc.q, cc.p, cc.dnum)
    L, K, N = oc.L, oc.K, oc.N
    _init(ref, oc, L + K)
    _set_keyswitch(ref, oc)
    idx = sorted({s * (1 << k) for k in range(15) for s in (1, -1)} | {3, 5})
    gals = [cc.rotation_galois(r) for r in idx]
    x, dig_or, dig_ref, _, _ = _dot_inputs(oc, 2300)
    dd, dx, dc0 = to_dev(dig_ref), to_dev(x), to_dev(oc.random(list(range(L)), 2350))
    kpid = list(range(L + K)) * oc.dnum
    keys = [to_dev(oc.random(kpid, 2400 + r).reshape(oc.dnum, L + K, N)) for r in range(2 * len(gals))]
    kb, ka = keys[0::2], keys[1::2]
    ob = [torch.empty((L + K, N), dtype=torch.int64, device="cuda") for _ in gals]
    oa = [torch.empty_like(o) for o in ob]
    G = (C.c_int32 * len(gals))(*gals)
    P = [_ref_ptrs(kb), _ref_ptrs(ka), _ref_ptrs(ob), _ref_ptrs(oa)]
    res = {"ref_hoisted_dot_32_rotations": _time(lambda: ref.refgpu_hoisted_dot(
        dd.data_ptr(), dx.data_ptr(), dc0.data_ptr(), len(gals), P[0], P[1], G, P[2], P[3], _stream()), reps=5)}
    del keys, kb, ka, ob, oa
    cc2, oc2 = make_pair(16, 30, 10, 3)
    _init(ref, oc2, 30)
    t = [to_dev(oc2.random(list(range(30)), 2500 + s)) for s in range(4)]
    c2 = torch.empty_like(t[0])
    res["ref_binomial_1_element"] = _time(lambda: ref.refgpu_binomial(
        t[0].data_ptr(), t[1].data_ptr(), c2.data_ptr(), t[2].data_ptr(), t[3].data_ptr(), 30, _stream()))
    res["ref_automorph_2x30_limbs"] = _time(lambda: [ref.refgpu_automorph(
        t[2 + h].data_ptr(), t[h].data_ptr(), 30, gals[0], _stream()) for h in (0, 1)])
    print("\nreference kernels (us, CUDA events): " + ", ".join("%s %.1f" % kv for kv in res.items()))
    assert all(v > 0 for v in res.values())
