"""Host-only helpers over the C ABI that need no GPU."""
from __future__ import annotations

import ctypes as C

from ._capi import FidesParams, check, lib, u64p


def generated_moduli(log_n, num_q, num_p=0, dnum=3, q0_bits=60, qi_bits=50, p_bits=60):
    """The (q, p) moduli fides_ctx_create generates for these parameters."""
    prm = FidesParams()
    prm.log_n, prm.num_q, prm.num_p, prm.dnum = log_n, num_q, num_p, dnum
    prm.q0_bits, prm.qi_bits, prm.p_bits = q0_bits, qi_bits, p_bits
    q = (C.c_uint64 * num_q)()
    p = (C.c_uint64 * 64)()
    k = C.c_int()
    check(lib.fides_generate_moduli(C.byref(prm), C.cast(q, u64p), C.cast(p, u64p), C.byref(k)))
    return [int(x) for x in q], [int(x) for x in p[:k.value]]
