"""Shared helpers of the GPU parity tests: a context and an oracle context over
the same moduli, seeded residues, torch device buffers for raw-pointer calls."""
import json
import os

import numpy as np

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.json")))


def make_pair(logN, L, K, dnum, ref_primes=False):
    """(CryptoContext, oracle.Ctx) over identical moduli."""
    from oracle import oracle as O

    import pyfideslib_b200 as F

    if ref_primes:
        cc = F.CryptoContext(log_n=logN, num_q=L, dnum=dnum, q=GOLD["p64"][:L], p=GOLD["sp64"][:K])
    else:
        cc = F.CryptoContext(log_n=logN, num_q=L, dnum=dnum, num_p=K)
    oc = O.Ctx(logN, cc.q, cc.p, dnum)
    return cc, oc


def rand_ct(oc, level, seed):
    pid = list(range(level + 1))
    return oc.random(pid, seed), oc.random(pid, seed + 1)


def rand_key(oc, seed):
    np_ = oc.L + oc.K
    pid = list(range(np_)) * oc.dnum
    b = oc.random(pid, seed).reshape(oc.dnum, np_, oc.N)
    a = oc.random(pid, seed + 1).reshape(oc.dnum, np_, oc.N)
    return b, a


def to_dev(arr):
    import torch

    return torch.from_numpy(arr.view(np.int64)).cuda()


def from_dev(t):
    return t.cpu().numpy().view(np.uint64)


def device_status(cc):
    """The context's device error word (0 when no kernel gave up a wait)."""
    import ctypes as C

    from pyfideslib_b200._capi import lib

    w = C.c_uint32()
    assert lib.fides_ctx_device_status(cc._h, C.byref(w)) == 0
    return w.value
