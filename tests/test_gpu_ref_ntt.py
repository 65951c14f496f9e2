"""The reference's own GPU forward NTT beside this library's, on the same B200.

oracle/_ref/libfidesref_gpu.so is src/NTT.cu of the reference compiled
unmodified, with oracle/ref_gpu_ntt.cu filling the constant and table blocks
its kernels read and launching them with the geometry of the reference's
LimbPartition::ApplyNTT (src/CKKS/LimbPartition.cu:364-395, ALGO_SHOUP, the
multi-limb NTT_ kernel pair).  The library is built where the reference tree
is mounted (`make -C oracle ref-gpu`) and travels prebuilt; without it these
tests skip.

* Parity: the reference kernel's output equals the oracle's transform and
  this library's bit for bit (bit-reversed evaluation order, the same psi).
* Timing: one forward transform of 32 polynomials x 30 limbs at N = 2^16
  (the bench's roofline workload) by each, CUDA events, inputs larger than
  L2 alternating between two resident batches; printed for the record.
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
        pytest.skip("the reference's GPU NTT was not built (make -C oracle ref-gpu needs the reference tree)")
    lib = C.CDLL(LIB)
    u64p = C.POINTER(C.c_uint64)
    lib.refntt_init.argtypes = [C.c_int, C.c_int, u64p, u64p]
    lib.refntt_init.restype = C.c_int
    lib.refntt_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    lib.refntt_forward.restype = C.c_int
    lib.refntt_release.argtypes = []
    yield lib
    lib.refntt_release()


def _init(ref, cc, oc, nq):
    psi = np.array([int(oc.psi_tables(i)[0][cc.N // 2]) for i in range(nq)], dtype=np.uint64)
    q = np.array(oc.primes[:nq], dtype=np.uint64)
    u64p = C.POINTER(C.c_uint64)
    assert ref.refntt_init(cc.logN, nq, q.ctypes.data_as(u64p), psi.ctypes.data_as(u64p)) == 0


def _ref_forward(ref, data, aux, ptrs, nlimbs, stream):
    assert ref.refntt_forward(data.data_ptr(), aux.data_ptr(), ptrs.data_ptr(), 0, nlimbs, stream) == 0


@pytest.mark.parametrize("logN,L", [(12, 8), (16, 30)])
def test_reference_ntt_equals_oracle_and_ours(ref, logN, L):
    import torch

    cc, oc = make_pair(logN, L, 3, 3)
    _init(ref, cc, oc, L)
    pid = list(range(L))
    x = oc.random(pid, 700 + logN)
    pm1 = np.array([q - 1 for q in oc.primes[:L]], dtype=np.uint64)[:, None]
    for inp in (x, np.ascontiguousarray(np.broadcast_to(pm1, x.shape))):
        want = oc.ntt(inp, pid)
        d = to_dev(inp)
        aux = torch.empty_like(d)
        ptrs = torch.empty(2 * L, dtype=torch.int64, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        _ref_forward(ref, d, aux, ptrs, L, stream)
        torch.cuda.synchronize()
        assert np.array_equal(from_dev(d), want)
        ours = to_dev(inp)
        cc.ntt(ours.data_ptr(), 0, L)
        cc.Synchronize()
        assert np.array_equal(from_dev(ours), want)


def test_reference_ntt_timing_batch32x30(ref):
    """The forward NTT of 32 x 30 limbs at N = 2^16 by the reference kernel
    pair and by this library's (same residues), device time per transform."""
    import torch

    cc, oc = make_pair(16, 30, 10, 3)
    _init(ref, cc, oc, 30)
    nl, nb, N = 30, 32, cc.N
    bufs = [torch.randint(0, 2 ** 40, (nb * nl, N), dtype=torch.int64, device="cuda") for _ in range(2)]
    aux = torch.empty_like(bufs[0])
    ptrs = torch.empty(2 * nb * nl, dtype=torch.int64, device="cuda")
    # same input through both: identical residues
    a, b = bufs[0].clone(), bufs[0].clone()
    s = torch.cuda.current_stream()
    _ref_forward(ref, a, aux, ptrs, nb * nl, s.cuda_stream)
    cc.ntt_batch(b.data_ptr(), nl * N, nb, 0, nl)
    cc.Synchronize()
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    del a, b
    reps = 10
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for r in range(3):
        _ref_forward(ref, bufs[r % 2], aux, ptrs, nb * nl, s.cuda_stream)
    e0.record(s)
    for r in range(reps):
        _ref_forward(ref, bufs[r % 2], aux, ptrs, nb * nl, s.cuda_stream)
    e1.record(s)
    e1.synchronize()
    ref_us = e0.elapsed_time(e1) / reps * 1e3
    st = torch.cuda.ExternalStream(cc.stream_ptr())
    for r in range(3):
        cc.ntt_batch(bufs[r % 2].data_ptr(), nl * N, nb, 0, nl)
    cc.Synchronize()
    e0.record(st)
    for r in range(reps):
        cc.ntt_batch(bufs[r % 2].data_ptr(), nl * N, nb, 0, nl)
    e1.record(st)
    e1.synchronize()
    ours_us = e0.elapsed_time(e1) / reps * 1e3
    gb = 16.0 * N * nl * nb / 1e9
    print("\nforward NTT 32 x 30 limbs, N=2^16: reference NTT_ pair %.1f us (%.0f GB/s), this library %.1f us "
          "(%.0f GB/s), ratio %.2f" % (ref_us, gb / (ref_us * 1e-6), ours_us, gb / (ours_us * 1e-6), ref_us / ours_us))
    assert ref_us > 0 and ours_us > 0
