"""ctypes bindings of include/fides_b200.h (libfidesb200.so, built in-tree).

There is no fallback: importing this module without the built library raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfidesb200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        "pyfideslib_b200: %s is missing; build it with `make -C pyfideslib_b200/csrc` "
        "(or __graft_entry__.build())" % LIB_PATH)

lib = C.CDLL(LIB_PATH)

u64 = C.c_uint64
u64p = C.POINTER(C.c_uint64)
i32p = C.POINTER(C.c_int32)
vp = C.c_void_p

STATUS = {0: "OK", 1: "BAD_ARG", 2: "OOM", 3: "LEVEL_MISMATCH", 4: "KEY_MISSING", 5: "TIMEOUT",
          6: "CUDA_ERR", 7: "UNSUPPORTED", 8: "BUSY"}


class SrvStats(C.Structure):
    _fields_ = [("completed", C.c_uint64), ("batches", C.c_uint64), ("p50_ms", C.c_double), ("p99_ms", C.c_double),
                ("mean_queue_ms", C.c_double), ("throughput", C.c_double), ("reserved_bytes", C.c_size_t)]


class FidesParams(C.Structure):
    _fields_ = [("log_n", C.c_int), ("num_q", C.c_int), ("num_p", C.c_int), ("dnum", C.c_int),
                ("q", u64p), ("p", u64p), ("q0_bits", C.c_int), ("qi_bits", C.c_int), ("p_bits", C.c_int),
                ("device", C.c_int), ("default_scale", C.c_double), ("q_root", u64p), ("p_root", u64p)]


class BootParams(C.Structure):
    _fields_ = [("slots", C.c_int), ("level_budget", C.c_int * 2), ("cheb_degree", C.c_int), ("K", C.c_double),
                ("double_angle", C.c_int), ("correction", C.c_int)]


class RawCt(C.Structure):
    """fides_raw_ct: RawCipherText's shape (limb arrays with their moduli)."""
    _fields_ = [("sub_0", C.POINTER(u64p)), ("sub_1", C.POINTER(u64p)), ("moduli", u64p), ("numRes", C.c_int),
                ("N", C.c_int), ("format", C.c_int), ("Noise", C.c_double), ("NoiseLevel", C.c_int),
                ("slots", C.c_int)]


class RawPt(C.Structure):
    _fields_ = [("sub_0", C.POINTER(u64p)), ("moduli", u64p), ("numRes", C.c_int), ("N", C.c_int),
                ("format", C.c_int), ("Noise", C.c_double), ("NoiseLevel", C.c_int), ("slots", C.c_int)]


class RawKey(C.Structure):
    _fields_ = [("r_key", C.POINTER(u64p)), ("r_key_moduli", u64p), ("dnum", C.c_int), ("nlimbs", C.c_int),
                ("N", C.c_int)]


def _sig(name, args, res=C.c_int):
    f = getattr(lib, name)
    f.argtypes = args
    f.restype = res
    return f


EXPORTS = {
    "fides_ctx_create": ([C.POINTER(FidesParams), C.POINTER(vp)], C.c_int),
    "fides_ctx_destroy": ([vp], C.c_int),
    "fides_generate_moduli": ([C.POINTER(FidesParams), u64p, u64p, C.POINTER(C.c_int)], C.c_int),
    "fides_ctx_info": ([vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), u64p,
                        u64p], C.c_int),
    "fides_ctx_synchronize": ([vp], C.c_int),
    "fides_ctx_last_error": ([vp], C.c_char_p),
    "fides_ctx_stream": ([vp, C.POINTER(vp)], C.c_int),
    "fides_kernel_launches": ([], C.c_uint64),
    "fides_autotune": ([vp, C.POINTER(C.c_int), C.POINTER(C.c_float), C.POINTER(C.c_int)], C.c_int),
    "fides_autotune_conv_info": ([vp, C.POINTER(C.c_int), C.POINTER(C.c_float)], C.c_int),
    "fides_set_conv_accumulator": ([vp, C.c_int], C.c_int),
    "fides_ctx_device_status": ([vp, C.POINTER(C.c_uint32)], C.c_int),
    "fides_ctx_inject_device_error": ([vp, C.c_uint32], C.c_int),
    "fides_set_keyswitch_variant": ([vp, C.c_int], C.c_int),
    "fides_set_giant_step_moddown": ([vp, C.c_int], C.c_int),
    "fides_set_ntt_variant": ([vp, C.c_int], C.c_int),
    "fides_key_upload_relin": ([vp, u64p, u64p], C.c_int),
    "fides_key_upload_galois": ([vp, C.c_uint32, u64p, u64p], C.c_int),
    "fides_rotation_galois": ([vp, C.c_int32, C.c_int], C.c_uint32),
    "fides_ct_upload": ([vp, u64p, u64p, C.c_int, C.c_double, C.c_int, C.c_int, C.POINTER(vp)], C.c_int),
    "fides_ct_download": ([vp, vp, u64p, u64p], C.c_int),
    "fides_ct_download_async": ([vp, vp, u64p, u64p], C.c_int),
    "fides_ct_info": ([vp, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_int)],
                      C.c_int),
    "fides_ct_create": ([vp, C.POINTER(vp)], C.c_int),
    "fides_ct_write": ([vp, vp, u64p, u64p], C.c_int),
    "fides_ct_copy": ([vp, vp, vp], C.c_int),
    "fides_ct_free": ([vp, vp], C.c_int),
    "fides_ct_device_ptrs": ([vp, C.POINTER(u64p), C.POINTER(u64p)], C.c_int),
    "fides_ct_set_level": ([vp, vp, C.c_int], C.c_int),
    "fides_pt_upload": ([vp, u64p, C.c_int, C.c_double, C.c_int, C.c_int, C.POINTER(vp)], C.c_int),
    "fides_pt_free": ([vp, vp], C.c_int),
    "fides_ct_import_raw": ([vp, C.POINTER(RawCt), C.POINTER(vp)], C.c_int),
    "fides_ct_export_raw": ([vp, vp, C.POINTER(RawCt)], C.c_int),
    "fides_pt_import_raw": ([vp, C.POINTER(RawPt), C.POINTER(vp)], C.c_int),
    "fides_key_import_raw": ([vp, C.c_uint32, C.POINTER(RawKey)], C.c_int),
    "fides_key_export_raw": ([vp, C.c_uint32, C.POINTER(RawKey)], C.c_int),
    "fides_hmult": ([vp, vp, vp, vp, C.c_int], C.c_int),
    "fides_square": ([vp, vp, vp, C.c_int], C.c_int),
    "fides_rescale": ([vp, vp, vp], C.c_int),
    "fides_rotate": ([vp, vp, C.c_int32, vp], C.c_int),
    "fides_rotate_hoisted": ([vp, vp, C.c_int, i32p, C.POINTER(vp)], C.c_int),
    "fides_conjugate": ([vp, vp, vp], C.c_int),
    "fides_hmult_batch": ([vp, C.c_int, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.c_int], C.c_int),
    "fides_rotate_batch": ([vp, C.c_int, C.POINTER(vp), i32p, C.POINTER(vp)], C.c_int),
    "fides_plan_hmult_rotate": ([vp, C.c_int, C.POINTER(vp), C.POINTER(vp), i32p, C.c_int, C.POINTER(vp),
                                 C.POINTER(vp)], C.c_int),
    "fides_plan_launch": ([vp, vp], C.c_int),
    "fides_plan_free": ([vp, vp], C.c_int),
    "fides_automorphism": ([vp, vp, C.c_uint32, vp], C.c_int),
    "fides_add": ([vp, vp, vp, vp], C.c_int),
    "fides_sub": ([vp, vp, vp, vp], C.c_int),
    "fides_negate": ([vp, vp, vp], C.c_int),
    "fides_add_pt": ([vp, vp, vp, vp], C.c_int),
    "fides_mult_pt": ([vp, vp, vp, vp, C.c_int], C.c_int),
    "fides_mult_int": ([vp, vp, C.c_int64, vp], C.c_int),
    "fides_mult_monomial": ([vp, vp, C.c_uint32, vp], C.c_int),
    "fides_mod_raise": ([vp, vp, vp], C.c_int),
    "fides_chebyshev_series": ([vp, vp, C.POINTER(C.c_double), C.c_int, C.c_double, C.c_double, vp], C.c_int),
    "fides_bootstrap_setup": ([vp, C.POINTER(BootParams)], C.c_int),
    "fides_bootstrap_info": ([vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), i32p], C.c_int),
    "fides_bootstrap_keygen": ([vp, vp, C.c_int, u64], C.c_int),
    "fides_bootstrap_iter": ([vp, vp, C.c_int, C.c_int, vp], C.c_int),
    "fides_bootstrap": ([vp, vp, vp], C.c_int),
    "fides_linear_transform": ([vp, vp, C.c_int, i32p, C.POINTER(vp), C.c_int, C.c_int, vp], C.c_int),
    "fides_linear_transform_batch": ([vp, C.c_int, C.POINTER(vp), C.c_int, i32p, C.POINTER(vp), C.c_int, C.c_int,
                                      C.POINTER(vp)], C.c_int),
    "fides_bootstrap_batch": ([vp, C.c_int, C.POINTER(vp), C.POINTER(vp)], C.c_int),
    "fides_add_scalar": ([vp, vp, C.c_double, vp], C.c_int),
    "fides_mult_scalar": ([vp, vp, C.c_double, vp, C.c_int], C.c_int),
    "fides_srv_create": ([vp, C.c_size_t, C.c_int, C.c_int, C.POINTER(vp)], C.c_int),
    "fides_srv_submit": ([vp, C.c_int, vp, vp, C.c_int32, vp, C.POINTER(C.c_uint64)], C.c_int),
    "fides_srv_wait": ([vp, C.c_uint64, C.c_double], C.c_int),
    "fides_srv_stats": ([vp, C.POINTER(SrvStats)], C.c_int),
    "fides_srv_reset_stats": ([vp], C.c_int),
    "fides_srv_destroy": ([vp], C.c_int),
    "fides_ntt": ([vp, vp, C.c_int, C.c_int, C.c_int], C.c_int),
    "fides_ntt_batch": ([vp, C.c_void_p, C.c_size_t, C.c_int, C.c_int, C.c_int, C.c_int], C.c_int),
    "fides_polymul": ([vp, vp, vp, vp, vp, vp, C.c_int, C.c_int], C.c_int),
    "fides_polymul_noalloc": ([vp, vp, vp, vp, C.c_int, C.c_int], C.c_int),
    "fides_keygen": ([vp, u64, C.c_int, C.POINTER(vp)], C.c_int),
    "fides_sk_free": ([vp, vp], C.c_int),
    "fides_keygen_public": ([vp, vp, u64, C.POINTER(vp)], C.c_int),
    "fides_pk_free": ([vp, vp], C.c_int),
    "fides_encrypt_pk": ([vp, vp, C.POINTER(C.c_double), C.c_int, C.c_int, C.c_double, u64, C.POINTER(vp)], C.c_int),
    "fides_keygen_relin": ([vp, vp, u64], C.c_int),
    "fides_keygen_rotations": ([vp, vp, C.c_int, i32p, C.c_int, u64], C.c_int),
    "fides_keygen_conjugate": ([vp, vp, u64], C.c_int),
    "fides_set_key_compression": ([vp, C.c_int], C.c_int),
    "fides_key_export": ([vp, C.c_uint32, u64p, u64p], C.c_int),
    "fides_encode": ([vp, C.POINTER(C.c_double), C.c_int, C.c_int, C.c_double, u64p], C.c_int),
    "fides_encrypt": ([vp, vp, C.POINTER(C.c_double), C.c_int, C.c_int, C.c_double, u64, C.POINTER(vp)], C.c_int),
    "fides_decrypt": ([vp, vp, vp, C.POINTER(C.c_double), C.c_int], C.c_int),
    "fides_ct_random": ([vp, C.c_int, u64, C.POINTER(vp)], C.c_int),
}

for _n, (_a, _r) in EXPORTS.items():
    _sig(_n, _a, _r)


class FidesError(RuntimeError):
    def __init__(self, status, msg=""):
        super().__init__("%s%s" % (STATUS.get(status, status), (": " + msg) if msg else ""))
        self.status = status


def check(status, ctx=None):
    if status != 0:
        msg = ""
        if ctx is not None:
            m = lib.fides_ctx_last_error(ctx)
            msg = m.decode() if m else ""
        raise FidesError(status, msg)
