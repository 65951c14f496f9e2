"""ctypes front end of the CPU oracle (oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline / reference legs, never by the product package.
Arrays are numpy uint64, limb-major ``[limbs, N]``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

u64p = C.POINTER(C.c_uint64)


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.or_mulmod.restype = C.c_uint64
        L.or_mulmod.argtypes = [C.c_uint64] * 3
        L.or_powmod.restype = C.c_uint64
        L.or_powmod.argtypes = [C.c_uint64] * 3
        L.or_invmod.restype = C.c_uint64
        L.or_invmod.argtypes = [C.c_uint64] * 2
        L.or_is_prime.restype = C.c_int
        L.or_is_prime.argtypes = [C.c_uint64]
        L.or_bitrev.restype = C.c_uint32
        L.or_bitrev.argtypes = [C.c_uint32, C.c_int]
        L.or_generator.restype = C.c_uint64
        L.or_generator.argtypes = [C.c_uint64]
        L.or_unity_root.restype = C.c_uint64
        L.or_unity_root.argtypes = [C.c_uint64, C.c_uint64]
        L.or_find_primes.restype = C.c_int
        L.or_find_primes.argtypes = [C.c_int, C.c_int, C.c_int, C.c_uint64, u64p]
        L.or_ctx_new.restype = C.c_void_p
        L.or_ctx_new.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, u64p]
        L.or_ctx_free.argtypes = [C.c_void_p]
        L.or_num_digits.restype = C.c_int
        L.or_num_digits.argtypes = [C.c_void_p, C.c_int]
        L.or_get_psi_tables.argtypes = [C.c_void_p, C.c_int, u64p, u64p]
        L.or_modup_consts.argtypes = [C.c_void_p, C.c_int, C.c_int, u64p, u64p]
        L.or_moddown_consts.argtypes = [C.c_void_p, u64p, u64p, u64p]
        L.or_ntt.argtypes = [C.c_void_p, u64p, C.c_int]
        L.or_intt.argtypes = [C.c_void_p, u64p, C.c_int]
        L.or_ntt_limbs.argtypes = [C.c_void_p, u64p, C.POINTER(C.c_int), C.c_int, C.c_int]
        L.or_nega_fft2.argtypes = [u64p, C.c_int, C.c_uint64, C.c_uint64, C.c_int]
        L.or_polymul.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), u64p, u64p, u64p]
        L.or_tensor.argtypes = [C.c_void_p, C.c_int] + [u64p] * 7
        L.or_automorph.argtypes = [C.c_void_p, C.c_int, u64p, u64p, C.c_uint32]
        L.or_rotation_galois.restype = C.c_uint32
        L.or_rotation_galois.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.or_modup.argtypes = [C.c_void_p, C.c_int, u64p, u64p]
        L.or_ks_inner.argtypes = [C.c_void_p, C.c_int, u64p, u64p, u64p, u64p, u64p]
        L.or_moddown.argtypes = [C.c_void_p, C.c_int, u64p, u64p]
        L.or_rescale.argtypes = [C.c_void_p, C.c_int, u64p, u64p]
        L.or_hmult.argtypes = [C.c_void_p, C.c_int] + [u64p] * 6 + [C.c_int, u64p, u64p]
        L.or_rotate_hoisted.argtypes = [C.c_void_p, C.c_int, u64p, u64p, C.c_int, C.POINTER(C.c_uint32),
                                        C.POINTER(u64p), C.POINTER(u64p), C.POINTER(u64p), C.POINTER(u64p)]
        L.or_rotate.argtypes = [C.c_void_p, C.c_int, u64p, u64p, C.c_uint32, u64p, u64p, u64p, u64p]
        L.or_set_threads.argtypes = [C.c_int]
        L.or_get_threads.restype = C.c_int
        L.or_random_residues.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_uint64, u64p]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"], "need C-contiguous uint64"
    return a.ctypes.data_as(u64p)


def _ip(lst):
    arr = (C.c_int * len(lst))(*lst)
    return arr


def mulmod(a, b, p):
    return lib().or_mulmod(a, b, p)


def powmod(a, e, p):
    return lib().or_powmod(a, e, p)


def invmod(a, p):
    return lib().or_invmod(a, p)


def is_prime(n):
    return bool(lib().or_is_prime(n))


def unity_root(p, order):
    return lib().or_unity_root(p, order)


def find_primes(logN, bits, count, upper=0):
    out = np.zeros(count, dtype=np.uint64)
    n = lib().or_find_primes(logN, bits, count, upper, _p(out))
    return [int(x) for x in out[:n]]


def moduli(logN, L, K=0, dnum=3, q0_bits=60, qi_bits=50, p_bits=60):
    """The (q, p) moduli of a context with these parameters, restated from the
    reference's parameter rules: one q0_bits prime and L-1 qi_bits primes by
    descending search for p = 1 mod 2N, then K special p_bits primes continuing
    the search and skipping the q's; K = 0 derives it from the widest digit
    (Parameters / computeK, src/CKKS/Context.cu:275-295)."""
    q = find_primes(logN, q0_bits, 1) + find_primes(logN, qi_bits, L - 1)
    if K <= 0:
        alpha = (L + dnum - 1) // dnum
        widest = max(sum(int(x).bit_length() for x in q[d * alpha:min(L, (d + 1) * alpha)]) for d in range(dnum))
        K = (widest + p_bits - 2) // (p_bits - 1)
    p = [x for x in find_primes(logN, p_bits, K + L + 2) if x not in q][:K]
    return q, p


def nega_fft2(a: np.ndarray, logN, p, psi, invert=False):
    a = np.ascontiguousarray(a, dtype=np.uint64).copy()
    lib().or_nega_fft2(_p(a), logN, p, psi, int(invert))
    return a


def set_threads(n):
    lib().or_set_threads(int(n))


def get_threads():
    return lib().or_get_threads()


class Ctx:
    """Oracle context: primes (Q then P), twiddle tables, digit layout."""

    def __init__(self, logN, q_primes, p_primes, dnum):
        self.logN = logN
        self.N = 1 << logN
        self.L = len(q_primes)
        self.K = len(p_primes)
        self.dnum = dnum
        self.alpha = -(-self.L // dnum)
        self.primes = [int(x) for x in list(q_primes) + list(p_primes)]
        arr = np.array(self.primes, dtype=np.uint64)
        h = lib().or_ctx_new(logN, self.L, self.K, dnum, _p(arr))
        if not h:
            raise ValueError("oracle: bad parameters (a prime is not 1 mod 2N?)")
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.or_ctx_free(h)
            self._h = None

    # ---- helpers ----
    def num_digits(self, level):
        return lib().or_num_digits(self._h, level)

    def ext_pidx(self, level):
        n = level + 1
        return list(range(n)) + [self.L + k for k in range(self.K)]

    def random(self, pidx, seed):
        out = np.empty((len(pidx), self.N), dtype=np.uint64)
        lib().or_random_residues(self._h, len(pidx), _ip(pidx), seed, _p(out))
        return out

    def psi_tables(self, pidx):
        a = np.empty(self.N, dtype=np.uint64)
        b = np.empty(self.N, dtype=np.uint64)
        lib().or_get_psi_tables(self._h, pidx, _p(a), _p(b))
        return a, b

    def modup_consts(self, level, d):
        np_ = self.L + self.K
        hi = np.zeros(self.alpha, dtype=np.uint64)
        hm = np.zeros((self.alpha, np_), dtype=np.uint64)
        lib().or_modup_consts(self._h, level, d, _p(hi), _p(hm))
        return hi, hm

    def moddown_consts(self):
        a = np.zeros(self.K, dtype=np.uint64)
        b = np.zeros((self.K, self.L), dtype=np.uint64)
        c = np.zeros(self.L, dtype=np.uint64)
        lib().or_moddown_consts(self._h, _p(a), _p(b), _p(c))
        return a, b, c

    # ---- transforms ----
    def ntt(self, a, pidx, inverse=False):
        a = np.ascontiguousarray(a, dtype=np.uint64).copy()
        a2 = a.reshape(-1, self.N)
        assert a2.shape[0] == len(pidx)
        lib().or_ntt_limbs(self._h, _p(a2), _ip(pidx), len(pidx), int(inverse))
        return a2.reshape(a.shape)

    def polymul(self, a, b, pidx):
        out = np.empty_like(a)
        lib().or_polymul(self._h, len(pidx), _ip(pidx), _p(a), _p(b), _p(out))
        return out

    def tensor(self, level, c0, c1, d0, d1):
        e0, e1, e2 = (np.empty_like(c0) for _ in range(3))
        lib().or_tensor(self._h, level, _p(c0), _p(c1), _p(d0), _p(d1), _p(e0), _p(e1), _p(e2))
        return e0, e1, e2

    def automorph(self, a, k):
        out = np.empty_like(a)
        lib().or_automorph(self._h, a.shape[0], _p(a), _p(out), k)
        return out

    def rotation_galois(self, index, slots):
        return lib().or_rotation_galois(self._h, index, slots)

    # ---- key switching ----
    def modup(self, level, x):
        n = level + 1
        out = np.empty((self.num_digits(level), n + self.K, self.N), dtype=np.uint64)
        lib().or_modup(self._h, level, _p(x), _p(out))
        return out

    def ks_inner(self, level, digits, ksk_b, ksk_a):
        n = level + 1
        ob = np.empty((n + self.K, self.N), dtype=np.uint64)
        oa = np.empty_like(ob)
        lib().or_ks_inner(self._h, level, _p(digits), _p(ksk_b), _p(ksk_a), _p(ob), _p(oa))
        return ob, oa

    def moddown(self, level, x):
        out = np.empty((level + 1, self.N), dtype=np.uint64)
        lib().or_moddown(self._h, level, _p(x), _p(out))
        return out

    def rescale(self, level, x):
        out = np.empty((level, self.N), dtype=np.uint64)
        lib().or_rescale(self._h, level, _p(x), _p(out))
        return out

    def hmult(self, level, a0, a1, b0, b1, ksk_b, ksk_a, rescale=True):
        rows = level if rescale else level + 1
        o0 = np.empty((rows, self.N), dtype=np.uint64)
        o1 = np.empty_like(o0)
        lib().or_hmult(self._h, level, _p(a0), _p(a1), _p(b0), _p(b1), _p(ksk_b), _p(ksk_a), int(rescale),
                       _p(o0), _p(o1))
        return o0, o1

    def rotate_hoisted(self, level, c0, c1, galois, kb_list, ka_list):
        n = len(galois)
        o0 = [np.empty((level + 1, self.N), dtype=np.uint64) for _ in range(n)]
        o1 = [np.empty((level + 1, self.N), dtype=np.uint64) for _ in range(n)]
        G = (C.c_uint32 * n)(*galois)
        KB = (u64p * n)(*[_p(k) for k in kb_list])
        KA = (u64p * n)(*[_p(k) for k in ka_list])
        O0 = (u64p * n)(*[_p(o) for o in o0])
        O1 = (u64p * n)(*[_p(o) for o in o1])
        lib().or_rotate_hoisted(self._h, level, _p(c0), _p(c1), n, G, KB, KA, O0, O1)
        return o0, o1

    def rotate(self, level, c0, c1, galois, kb, ka):
        o0, o1 = self.rotate_hoisted(level, c0, c1, [galois], [kb], [ka])
        return o0[0], o1[0]
