"""fides_polymul_noalloc: the polynomial multiply for callers that cannot
allocate device memory when they multiply (hosts whose own allocator owns the
whole device, loops that must not hit cudaMalloc/cudaFree, which synchronise
the device).  Its scratch is a fixed device array inside the
library, so its output must equal fides_polymul's, which takes caller
scratch — bit for bit, on two calls in a row, and sizes beyond the fixed
scratch must be refused.

This file is collected last so that a failure here comes after every other
test has run; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_polymul_matches_polymul_twice():
    import torch

    import pyfideslib_b200 as F
    from pyfideslib_b200._capi import lib

    cc = F.CryptoContext(log_n=16, num_q=12, dnum=3, num_p=4)
    nl = 8  # 8 limbs x 2^16 = 2^19 words: the largest call the fixed scratch holds
    g = torch.Generator().manual_seed(5)
    for call in range(2):
        q = torch.tensor([int(x) for x in cc.q[:nl]], dtype=torch.int64)[:, None]
        a = (torch.randint(0, 2 ** 62, (nl, cc.N), generator=g, dtype=torch.int64) % q).cuda()
        b = (torch.randint(0, 2 ** 62, (nl, cc.N), generator=g, dtype=torch.int64) % q).cuda()
        want = torch.empty_like(a)
        sa, sb = torch.empty_like(a), torch.empty_like(a)
        assert lib.fides_polymul(cc._h, a.data_ptr(), b.data_ptr(), want.data_ptr(), sa.data_ptr(), sb.data_ptr(),
                                 0, nl) == 0
        got = torch.full_like(a, -1)
        assert lib.fides_polymul_noalloc(cc._h, a.data_ptr(), b.data_ptr(), got.data_ptr(), 0, nl) == 0
        cc.Synchronize()
        torch.cuda.synchronize()
        assert torch.equal(got.cpu(), want.cpu()), "call %d differs" % call
    # refused beyond the fixed scratch, with a message
    big = torch.zeros((nl + 1, cc.N), dtype=torch.int64, device="cuda")
    assert lib.fides_polymul_noalloc(cc._h, big.data_ptr(), big.data_ptr(), big.data_ptr(), 0, nl + 1) == 1
    assert b"exceeds the fixed scratch" in lib.fides_ctx_last_error(cc._h)
