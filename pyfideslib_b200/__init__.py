"""pyfideslib_b200 -- B200-native CKKS evaluation core with the FIDESlib
evaluation surface (api/fideslib.hpp: CryptoContext, Ciphertext, EvalAdd,
EvalMult, EvalRotate, EvalFastRotation, Rescale ...), driven through the C ABI
in include/fides_b200.h.

This Python layer is a thin host-side mirror used by tests and benchmarks; the
C++ mirror of the same surface is pyfideslib_b200/csrc/api/fideslib.hpp.
Residues cross the boundary as numpy uint64 arrays in evaluation
(bit-reversed NTT) order, limb-major.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._capi import BootParams, FidesError, FidesParams, RawCt, RawKey, RawPt, SrvStats, check, lib, u64p, vp

__all__ = ["CryptoContext", "Ciphertext", "Plaintext", "PrivateKey", "Server", "Plan", "FidesError", "lib"]


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(u64p)


class Ciphertext:
    """Device-resident ciphertext handle (FIDESlib CiphertextImpl)."""

    def __init__(self, ctx: "CryptoContext", handle=None):
        self.ctx = ctx
        if handle is None:
            h = vp()
            check(lib.fides_ct_create(ctx._h, C.byref(h)), ctx._h)
            handle = h.value
        self._h = handle

    def __del__(self):
        h, ctx = getattr(self, "_h", None), getattr(self, "ctx", None)
        if h and ctx is not None and ctx._h:
            lib.fides_ct_free(ctx._h, h)
        self._h = None

    def info(self):
        lv, sc, nd, sl = C.c_int(), C.c_double(), C.c_int(), C.c_int()
        check(lib.fides_ct_info(self._h, C.byref(lv), C.byref(sc), C.byref(nd), C.byref(sl)))
        return {"level": lv.value, "scale": sc.value, "noise_deg": nd.value, "slots": sl.value}

    @property
    def level(self):
        return self.info()["level"]

    @property
    def slots(self):
        return self.info()["slots"]

    def GetLevel(self):
        return self.level

    def download(self):
        lv = self.level
        c0 = np.empty((lv + 1, self.ctx.N), dtype=np.uint64)
        c1 = np.empty_like(c0)
        check(lib.fides_ct_download(self.ctx._h, self._h, _p(c0), _p(c1)), self.ctx._h)
        return c0, c1


class Plaintext:
    def __init__(self, ctx, handle, values=None, slots=0):
        self.ctx, self._h, self.values, self.slots = ctx, handle, values, slots

    def __del__(self):
        h, ctx = getattr(self, "_h", None), getattr(self, "ctx", None)
        if h and ctx is not None and ctx._h:
            lib.fides_pt_free(ctx._h, h)
        self._h = None


class Plan:
    """A captured CUDA graph of a batched evaluation (fides_plan)."""

    def __init__(self, ctx, handle, keep):
        self.ctx, self._h, self._keep = ctx, handle, keep

    def launch(self):
        check(lib.fides_plan_launch(self.ctx._h, self._h), self.ctx._h)

    def __del__(self):
        h, ctx = getattr(self, "_h", None), getattr(self, "ctx", None)
        if h and ctx is not None and ctx._h:
            lib.fides_plan_free(ctx._h, h)
        self._h = None


class Server:
    """Continuous-batching request loop (fides_srv_*): submit HMult / Rotate /
    Bootstrap requests from any thread, wait on request ids, read p50 / p99."""

    HMULT, ROTATE, BOOTSTRAP = 0, 1, 2

    def __init__(self, ctx, hbm_budget, max_batch=16, num_streams=2):
        self.ctx = ctx
        h = vp()
        check(lib.fides_srv_create(ctx._h, int(hbm_budget), max_batch, num_streams, C.byref(h)), ctx._h)
        self._h = h.value

    def submit(self, op, a, b=None, index=0, out=None):
        out = out if out is not None else Ciphertext(self.ctx)
        rid = C.c_uint64()
        check(lib.fides_srv_submit(self._h, op, a._h, b._h if b is not None else None, index, out._h,
                                   C.byref(rid)), self.ctx._h)
        return rid.value, out

    def wait(self, rid, timeout=60.0):
        check(lib.fides_srv_wait(self._h, rid, timeout), self.ctx._h)

    def stats(self):
        st = SrvStats()
        check(lib.fides_srv_stats(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in SrvStats._fields_}

    def reset_stats(self):
        check(lib.fides_srv_reset_stats(self._h))

    def close(self):
        if getattr(self, "_h", None):
            lib.fides_srv_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


class PrivateKey:
    def __init__(self, ctx, handle):
        self.ctx, self._h = ctx, handle

    def __del__(self):
        h, ctx = getattr(self, "_h", None), getattr(self, "ctx", None)
        if h and ctx is not None and ctx._h:
            lib.fides_sk_free(ctx._h, h)
        self._h = None


class CryptoContext:
    """Mirror of fideslib::CryptoContextImpl<DCRTPoly> (api/CryptoContext.hpp:24-245)."""

    def __init__(self, log_n=16, num_q=30, dnum=3, num_p=0, q=None, p=None, q0_bits=60, qi_bits=50, p_bits=60,
                 device=0, scale=None, q_root=None, p_root=None):
        """q_root / p_root: the primitive 2N-th roots of unity that fix the
        evaluation representation (OpenFHE's RawParams root_of_unity /
        SPECIALroot_of_unity); None for FIDESlib's smallest-generator rule."""
        prm = FidesParams()
        prm.log_n, prm.num_q, prm.num_p, prm.dnum = log_n, num_q, num_p, dnum
        self._qa = np.ascontiguousarray(q, dtype=np.uint64) if q is not None else None
        self._pa = np.ascontiguousarray(p, dtype=np.uint64) if p is not None else None
        self._qr = np.ascontiguousarray(q_root, dtype=np.uint64) if q_root is not None else None
        self._pr = np.ascontiguousarray(p_root, dtype=np.uint64) if p_root is not None else None
        prm.q = _p(self._qa)
        prm.p = _p(self._pa)
        prm.q_root = _p(self._qr)
        prm.p_root = _p(self._pr)
        if self._pa is not None:
            prm.num_p = len(self._pa)
        prm.q0_bits, prm.qi_bits, prm.p_bits = q0_bits, qi_bits, p_bits
        prm.device = device
        prm.default_scale = float(scale) if scale else 0.0
        h = vp()
        check(lib.fides_ctx_create(C.byref(prm), C.byref(h)))
        self._h = h.value
        ln, nq, npp, dn = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        lib.fides_ctx_info(self._h, C.byref(ln), C.byref(nq), C.byref(npp), C.byref(dn), None, None)
        self.logN, self.L, self.K, self.dnum = ln.value, nq.value, npp.value, dn.value
        self.N = 1 << self.logN
        qq = np.zeros(self.L, dtype=np.uint64)
        pp = np.zeros(max(self.K, 1), dtype=np.uint64)
        lib.fides_ctx_info(self._h, None, None, None, None, _p(qq), _p(pp))
        self.q = [int(x) for x in qq]
        self.p = [int(x) for x in pp[:self.K]]
        self.scale = float(scale) if scale else float(2 ** qi_bits)

    def close(self):
        if getattr(self, "_h", None):
            lib.fides_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    # ---- info ----
    def GetRingDimension(self):
        return self.N

    def GetCyclotomicOrder(self):
        return 2 * self.N

    def primes(self):
        return self.q + self.p

    def stream_ptr(self):
        """The context's CUDA stream (cudaStream_t as an int)."""
        h = vp()
        check(lib.fides_ctx_stream(self._h, C.byref(h)), self._h)
        return h.value

    def Synchronize(self):
        check(lib.fides_ctx_synchronize(self._h), self._h)

    # ---- raw residue interop (RawCipherText-shaped) ----
    def upload(self, c0, c1, level=None, scale=None, noise_deg=1, slots=None):
        c0 = np.ascontiguousarray(c0, dtype=np.uint64)
        c1 = np.ascontiguousarray(c1, dtype=np.uint64)
        lv = c0.shape[0] - 1 if level is None else level
        h = vp()
        check(lib.fides_ct_upload(self._h, _p(c0), _p(c1), lv, float(scale or self.scale), noise_deg,
                                  slots or self.N // 2, C.byref(h)), self._h)
        return Ciphertext(self, h.value)

    # ---- raw-residue interop (RawCipherText / RawPlainText / RawKeySwitchKey) ----
    FORMAT_EVALUATION, FORMAT_COEFFICIENT = 0, 1

    @staticmethod
    def _limb_ptrs(limbs):
        return (u64p * len(limbs))(*[_p(x) for x in limbs])

    def import_raw_ct(self, sub_0, sub_1, moduli, noise=None, noise_level=1, slots=None, fmt=0):
        """Device ciphertext from RawCipherText-shaped data: lists of per-limb
        uint64 arrays (N words each) and the limbs' moduli."""
        sub_0 = [np.ascontiguousarray(x, dtype=np.uint64) for x in sub_0]
        sub_1 = [np.ascontiguousarray(x, dtype=np.uint64) for x in sub_1]
        mod = np.ascontiguousarray(moduli, dtype=np.uint64)
        raw = RawCt(self._limb_ptrs(sub_0), self._limb_ptrs(sub_1), _p(mod), len(sub_0), self.N, fmt,
                    float(noise or self.scale), noise_level, slots or self.N // 2)
        h = vp()
        check(lib.fides_ct_import_raw(self._h, C.byref(raw), C.byref(h)), self._h)
        return Ciphertext(self, h.value)

    def export_raw_ct(self, ct, fmt=0):
        """RawCipherText-shaped copy of a device ciphertext:
        (sub_0, sub_1, moduli, noise, noise_level, slots)."""
        n = ct.level + 1
        s0 = [np.empty(self.N, dtype=np.uint64) for _ in range(n)]
        s1 = [np.empty(self.N, dtype=np.uint64) for _ in range(n)]
        mod = np.zeros(n, dtype=np.uint64)
        raw = RawCt(self._limb_ptrs(s0), self._limb_ptrs(s1), _p(mod), n, self.N, fmt, 0.0, 0, 0)
        check(lib.fides_ct_export_raw(self._h, ct._h, C.byref(raw)), self._h)
        return s0, s1, [int(x) for x in mod], raw.Noise, raw.NoiseLevel, raw.slots

    def import_raw_pt(self, sub_0, moduli, noise=None, noise_level=1, slots=None, fmt=0):
        sub_0 = [np.ascontiguousarray(x, dtype=np.uint64) for x in sub_0]
        mod = np.ascontiguousarray(moduli, dtype=np.uint64)
        raw = RawPt(self._limb_ptrs(sub_0), _p(mod), len(sub_0), self.N, fmt, float(noise or self.scale),
                    noise_level, slots or self.N // 2)
        h = vp()
        check(lib.fides_pt_import_raw(self._h, C.byref(raw), C.byref(h)), self._h)
        return Plaintext(self, h.value)

    def import_raw_key(self, galois, r_key, r_key_moduli):
        """Switching key from RawKeySwitchKey-shaped data: r_key[h][d][i] (h = 0
        for the a half, 1 for b) of N words, r_key_moduli[h][d][i] its modulus.
        galois 0 is the relinearisation key."""
        dnum, nl = len(r_key[0]), len(r_key[0][0])
        limbs = [np.ascontiguousarray(r_key[h][d][i], dtype=np.uint64)
                 for h in range(2) for d in range(dnum) for i in range(nl)]
        mod = np.ascontiguousarray([r_key_moduli[h][d][i] for h in range(2) for d in range(dnum) for i in range(nl)],
                                   dtype=np.uint64)
        raw = RawKey(self._limb_ptrs(limbs), _p(mod), dnum, nl, self.N)
        check(lib.fides_key_import_raw(self._h, galois, C.byref(raw)), self._h)

    def export_raw_key(self, galois=0):
        """(r_key [2][dnum][L+K][N], r_key_moduli [2][dnum][L+K]) of a resident key."""
        nl = self.L + self.K
        arr = np.empty((2, self.dnum, nl, self.N), dtype=np.uint64)
        limbs = [arr[h, d, i] for h in range(2) for d in range(self.dnum) for i in range(nl)]
        mod = np.zeros(2 * self.dnum * nl, dtype=np.uint64)
        raw = RawKey(self._limb_ptrs(limbs), _p(mod), self.dnum, nl, self.N)
        check(lib.fides_key_export_raw(self._h, galois, C.byref(raw)), self._h)
        return arr, mod.reshape(2, self.dnum, nl)

    def random_ct(self, level, seed):
        h = vp()
        check(lib.fides_ct_random(self._h, level, seed, C.byref(h)), self._h)
        return Ciphertext(self, h.value)

    def upload_relin_key(self, b, a):
        check(lib.fides_key_upload_relin(self._h, _p(np.ascontiguousarray(b, dtype=np.uint64)),
                                         _p(np.ascontiguousarray(a, dtype=np.uint64))), self._h)

    def upload_galois_key(self, galois, b, a):
        check(lib.fides_key_upload_galois(self._h, galois, _p(np.ascontiguousarray(b, dtype=np.uint64)),
                                          _p(np.ascontiguousarray(a, dtype=np.uint64))), self._h)

    def export_key(self, galois=0):
        shape = (self.dnum, self.L + self.K, self.N)
        b = np.empty(shape, dtype=np.uint64)
        a = np.empty(shape, dtype=np.uint64)
        check(lib.fides_key_export(self._h, galois, _p(b), _p(a)), self._h)
        return b, a

    def rotation_galois(self, index, slots=None):
        return lib.fides_rotation_galois(self._h, index, slots or self.N // 2)

    # ---- client side ----
    def KeyGen(self, seed=1, hamming_weight=0):
        h = vp()
        check(lib.fides_keygen(self._h, seed, hamming_weight, C.byref(h)), self._h)
        return PrivateKey(self, h.value)

    def EvalMultKeyGen(self, sk, seed=2):
        check(lib.fides_keygen_relin(self._h, sk._h, seed), self._h)

    def EvalRotateKeyGen(self, sk, indices, slots=None, seed=3):
        arr = (C.c_int32 * len(indices))(*indices)
        check(lib.fides_keygen_rotations(self._h, sk._h, len(indices), arr, slots or self.N // 2, seed), self._h)

    def EvalConjugateKeyGen(self, sk, seed=4):
        check(lib.fides_keygen_conjugate(self._h, sk._h, seed), self._h)

    @staticmethod
    def _vals(values, slots):
        v = np.zeros(2 * slots, dtype=np.float64)
        z = np.asarray(values, dtype=np.complex128)
        v[0:2 * len(z):2] = z.real
        v[1:2 * len(z):2] = z.imag
        return v

    def encode(self, values, slots=None, level=None, scale=None):
        slots = slots or self.N // 2
        lv = self.L - 1 if level is None else level
        v = self._vals(values, slots)
        m = np.empty((lv + 1, self.N), dtype=np.uint64)
        check(lib.fides_encode(self._h, v.ctypes.data_as(C.POINTER(C.c_double)), slots, lv,
                               float(scale or self.scale), _p(m)), self._h)
        return m

    def MakeCKKSPackedPlaintext(self, values, noise_deg=1, level=None, slots=None, scale=None):
        slots = slots or self.N // 2
        lv = self.L - 1 if level is None else level
        sc = float(scale or self.scale) if noise_deg == 1 else float(scale or self.scale) ** noise_deg
        m = self.encode(values, slots, lv, sc)
        h = vp()
        check(lib.fides_pt_upload(self._h, _p(m), lv, sc, noise_deg, slots, C.byref(h)), self._h)
        return Plaintext(self, h.value, values, slots)

    def Encrypt(self, sk, values, slots=None, level=None, scale=None, seed=5):
        slots = slots or self.N // 2
        lv = self.L - 1 if level is None else level
        v = self._vals(values, slots)
        h = vp()
        check(lib.fides_encrypt(self._h, sk._h, v.ctypes.data_as(C.POINTER(C.c_double)), slots, lv,
                                float(scale or self.scale), seed, C.byref(h)), self._h)
        return Ciphertext(self, h.value)

    def Decrypt(self, sk, ct, slots=None):
        slots = slots or ct.info()["slots"] or self.N // 2
        v = np.empty(2 * slots, dtype=np.float64)
        check(lib.fides_decrypt(self._h, sk._h, ct._h, v.ctypes.data_as(C.POINTER(C.c_double)), slots), self._h)
        return v[0::2] + 1j * v[1::2]

    # ---- evaluation ----
    def _out(self, out):
        return out if out is not None else Ciphertext(self)

    def EvalMult(self, a, b, rescale=False, out=None):
        out = self._out(out)
        if isinstance(b, Plaintext):
            check(lib.fides_mult_pt(self._h, a._h, b._h, out._h, int(rescale)), self._h)
        elif isinstance(b, (int, float)):
            check(lib.fides_mult_scalar(self._h, a._h, float(b), out._h, int(rescale)), self._h)
        else:
            check(lib.fides_hmult(self._h, a._h, b._h, out._h, int(rescale)), self._h)
        return out

    def EvalMultBatch(self, a_list, b_list, rescale=False, outs=None):
        """Batched HMult (+ rescale) of independent pairs; levels may differ."""
        n = len(a_list)
        outs = outs or [Ciphertext(self) for _ in range(n)]
        A = (vp * n)(*[x._h for x in a_list])
        B = (vp * n)(*[x._h for x in b_list])
        O = (vp * n)(*[o._h for o in outs])
        check(lib.fides_hmult_batch(self._h, n, A, B, O, int(rescale)), self._h)
        return outs

    def EvalRotateBatch(self, a_list, indices, outs=None):
        """Rotation of each ciphertext by its own index (own keys)."""
        n = len(a_list)
        outs = outs or [Ciphertext(self) for _ in range(n)]
        A = (vp * n)(*[x._h for x in a_list])
        I = (C.c_int32 * n)(*indices)
        O = (vp * n)(*[o._h for o in outs])
        check(lib.fides_rotate_batch(self._h, n, A, I, O), self._h)
        return outs

    def plan_hmult_rotate(self, a_list, b_list, indices=None, rescale=True, outs=None):
        """Capture batched HMult(+rescale)(+rotation) into one CUDA graph.
        Returns (plan, outs); plan.launch() replays it."""
        n = len(a_list)
        outs = outs or [Ciphertext(self) for _ in range(n)]
        A = (vp * n)(*[x._h for x in a_list])
        B = (vp * n)(*[x._h for x in b_list])
        O = (vp * n)(*[o._h for o in outs])
        I = (C.c_int32 * n)(*indices) if indices is not None else None
        h = vp()
        check(lib.fides_plan_hmult_rotate(self._h, n, A, B, I, int(rescale), O, C.byref(h)), self._h)
        return Plan(self, h.value, (a_list, b_list, outs)), outs

    def write(self, ct, c0, c1):
        check(lib.fides_ct_write(self._h, ct._h, _p(np.ascontiguousarray(c0, dtype=np.uint64)),
                                 _p(np.ascontiguousarray(c1, dtype=np.uint64))), self._h)
        self.Synchronize()

    def EvalSquare(self, a, rescale=False, out=None):
        out = self._out(out)
        check(lib.fides_square(self._h, a._h, out._h, int(rescale)), self._h)
        return out

    def Rescale(self, a, out=None):
        out = self._out(out)
        check(lib.fides_rescale(self._h, a._h, out._h), self._h)
        return out

    def EvalAdd(self, a, b, out=None):
        out = self._out(out)
        if isinstance(b, Plaintext):
            check(lib.fides_add_pt(self._h, a._h, b._h, out._h), self._h)
        elif isinstance(b, (int, float)):
            check(lib.fides_add_scalar(self._h, a._h, float(b), out._h), self._h)
        else:
            check(lib.fides_add(self._h, a._h, b._h, out._h), self._h)
        return out

    def EvalSub(self, a, b, out=None):
        out = self._out(out)
        check(lib.fides_sub(self._h, a._h, b._h, out._h), self._h)
        return out

    def EvalNegate(self, a, out=None):
        out = self._out(out)
        check(lib.fides_negate(self._h, a._h, out._h), self._h)
        return out

    def EvalRotate(self, a, index, out=None):
        out = self._out(out)
        check(lib.fides_rotate(self._h, a._h, index, out._h), self._h)
        return out

    def EvalFastRotation(self, a, indices):
        outs = [Ciphertext(self) for _ in indices]
        arr = (C.c_int32 * len(indices))(*indices)
        hs = (vp * len(outs))(*[o._h for o in outs])
        check(lib.fides_rotate_hoisted(self._h, a._h, len(indices), arr, hs), self._h)
        return outs

    # ---- scalar / monomial / polynomial evaluation ----
    def EvalMultInt(self, a, z, out=None):
        """a times the integer z (scale kept)."""
        out = self._out(out)
        check(lib.fides_mult_int(self._h, a._h, int(z), out._h), self._h)
        return out

    def EvalMultMonomial(self, a, power, out=None):
        out = self._out(out)
        check(lib.fides_mult_monomial(self._h, a._h, int(power) % (2 * self.N), out._h), self._h)
        return out

    def ModRaise(self, a, out=None):
        out = self._out(out)
        check(lib.fides_mod_raise(self._h, a._h, out._h), self._h)
        return out

    def EvalChebyshevSeries(self, a, coeffs, lo=-1.0, hi=1.0, out=None):
        out = self._out(out)
        cf = np.ascontiguousarray(coeffs, dtype=np.float64)
        check(lib.fides_chebyshev_series(self._h, a._h, cf.ctypes.data_as(C.POINTER(C.c_double)), len(cf) - 1,
                                         float(lo), float(hi), out._h), self._h)
        return out

    # ---- bootstrapping (EvalBootstrapSetup / EvalBootstrapKeyGen / EvalBootstrap) ----
    def EvalBootstrapSetup(self, level_budget=(3, 3), slots=None, cheb_degree=119, K=16.0, double_angle=3,
                           correction=0):
        prm = BootParams()
        prm.slots = slots or self.N // 2
        prm.level_budget[0], prm.level_budget[1] = level_budget
        prm.cheb_degree, prm.K, prm.double_angle, prm.correction = cheb_degree, K, double_angle, correction
        check(lib.fides_bootstrap_setup(self._h, C.byref(prm)), self._h)

    def bootstrap_info(self, slots=None):
        lv, n = C.c_int(), C.c_int()
        check(lib.fides_bootstrap_info(self._h, slots or self.N // 2, C.byref(lv), C.byref(n), None), self._h)
        rot = (C.c_int32 * max(1, n.value))()
        check(lib.fides_bootstrap_info(self._h, slots or self.N // 2, None, None, rot), self._h)
        return lv.value, [int(rot[i]) for i in range(n.value)]

    def EvalBootstrapKeyGen(self, sk, slots=None, seed=11):
        check(lib.fides_bootstrap_keygen(self._h, sk._h, slots or self.N // 2, seed), self._h)

    def EvalBootstrap(self, a, out=None, num_iterations=1, precision=0):
        """num_iterations 2: bootstraps the first result's error again (the
        input must still hold the bootstrap's output level)."""
        out = self._out(out)
        if num_iterations == 1:
            check(lib.fides_bootstrap(self._h, a._h, out._h), self._h)
        else:
            check(lib.fides_bootstrap_iter(self._h, a._h, num_iterations, precision, out._h), self._h)
        return out

    def EvalBootstrapBatch(self, a_list, outs=None):
        """EvalBootstrap of several ciphertexts together (batched EvalMod and
        giant-step rotations); results equal one EvalBootstrap each."""
        n = len(a_list)
        outs = outs or [Ciphertext(self) for _ in range(n)]
        A = (vp * n)(*[x._h for x in a_list])
        O = (vp * n)(*[o._h for o in outs])
        check(lib.fides_bootstrap_batch(self._h, n, A, O), self._h)
        return outs

    # ---- diagonal-form linear transforms (baby-step giant-step) ----
    @staticmethod
    def linear_transform_rotations(offsets, bstep):
        """Rotation indices a BSGS transform over `offsets` needs keys for."""
        need = set()
        for o in offsets:
            g = o // bstep
            b = o - g * bstep
            if b:
                need.add(b)
            if g:
                need.add(g * bstep)
        return sorted(need)

    def prepare_linear_transform(self, diags, bstep, level=None, slots=None, scale=None):
        """Encode the diagonals {offset: vector of `slots` values} of a slot
        matrix M (M[i, (i + offset) % slots] = diags[offset][i]) as the
        plaintexts EvalLinearTransform consumes: diagonal o = g*bstep + b is
        pre-rotated by g*bstep slots."""
        slots = slots or self.N // 2
        offs = sorted(diags)
        pts = []
        for o in offs:
            g = o // bstep
            v = np.roll(np.asarray(diags[o], dtype=np.complex128), g * bstep)
            pts.append(self.MakeCKKSPackedPlaintext(v, level=level, slots=slots, scale=scale))
        return offs, pts

    def EvalLinearTransformBatch(self, xs, offsets, pts, bstep, rescale=True, outs=None):
        """The same diagonal-form transform of several ciphertexts at one level."""
        n = len(xs)
        outs = outs or [Ciphertext(self) for _ in range(n)]
        X = (vp * n)(*[x._h for x in xs])
        O = (vp * n)(*[o._h for o in outs])
        off = (C.c_int32 * len(offsets))(*offsets)
        P = (vp * len(pts))(*[p._h for p in pts])
        check(lib.fides_linear_transform_batch(self._h, n, X, len(offsets), off, P, bstep, int(rescale), O), self._h)
        return outs

    def EvalLinearTransform(self, x, offsets, pts, bstep, rescale=True, out=None):
        out = self._out(out)
        n = len(offsets)
        check(lib.fides_linear_transform(self._h, x._h, n, (C.c_int32 * n)(*offsets),
                                         (vp * n)(*[p._h for p in pts]), bstep, int(rescale), out._h), self._h)
        return out

    def EvalConjugate(self, a, out=None):
        out = self._out(out)
        check(lib.fides_conjugate(self._h, a._h, out._h), self._h)
        return out

    def EvalAutomorphism(self, a, galois, out=None):
        out = self._out(out)
        check(lib.fides_automorphism(self._h, a._h, galois, out._h), self._h)
        return out

    def SetLevel(self, ct, level):
        check(lib.fides_ct_set_level(self._h, ct._h, level), self._h)

    # ---- raw device kernels (device pointers as ints, memory the caller owns
    #      and may touch from other streams: these return after completion) ----
    def ntt(self, dev_ptr, prime0, nlimbs, inverse=False):
        check(lib.fides_ntt(self._h, dev_ptr, prime0, nlimbs, int(inverse)), self._h)
        self.Synchronize()

    def ntt_batch(self, dev_ptr, poly_stride, npoly, prime0, nlimbs, inverse=False):
        check(lib.fides_ntt_batch(self._h, dev_ptr, poly_stride, npoly, prime0, nlimbs, int(inverse)), self._h)
        self.Synchronize()

    def set_ntt_variant(self, variant):
        """Force an NTT kernel variant (-1: back to the autotuned one)."""
        check(lib.fides_set_ntt_variant(self._h, variant), self._h)

    def set_giant_step_moddown(self, scope):
        """Giant-step rotations of linear transforms summed before one ModDown
        per input: 0 never, 1 in the bootstrap's transforms (default), 2 in
        every transform."""
        check(lib.fides_set_giant_step_moddown(self._h, scope), self._h)

    def polymul(self, a, b, c, a_ntt, b_ntt, prime0, nlimbs):
        check(lib.fides_polymul(self._h, a, b, c, a_ntt, b_ntt, prime0, nlimbs), self._h)
        self.Synchronize()
