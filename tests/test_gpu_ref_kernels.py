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
  HMult shape (N = 2^16, L = 30, K = 10, dnum = 3).
* Timing at the HMult shape, CUDA events, printed for the record: each
  reference kernel on the work one batched step gives it, and this library's
  batched NTT / INTT on the same residues.
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
    for f in ("refgpu_init", "refgpu_transform", "refgpu_set_keyswitch", "refgpu_modup_conv",
              "refgpu_moddown_conv", "refgpu_dot"):
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
