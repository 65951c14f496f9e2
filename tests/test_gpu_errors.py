"""Error behaviour of the C ABI on a live context: every refusal is a status
code with a message, never an exit or an exception across the boundary
(the reference throws OPENFHE_THROW for the same preconditions,
api/CryptoContext.cpp:150,168,235), and the context stays usable after it."""
import numpy as np
import pytest

import pyfideslib_b200 as F
from pyfideslib_b200._capi import FidesError

pytestmark = pytest.mark.gpu

BAD_ARG, KEY_MISSING, TIMEOUT, UNSUPPORTED = 1, 4, 5, 7


@pytest.fixture(scope="module")
def ctx():
    cc = F.CryptoContext(log_n=12, num_q=6, dnum=3)
    sk = cc.KeyGen(seed=1, hamming_weight=32)
    return cc, sk


def _status(fn):
    with pytest.raises(FidesError) as e:
        fn()
    return e.value.status


def test_missing_keys(ctx):
    cc, sk = ctx
    ct = cc.Encrypt(sk, np.ones(cc.N // 2))
    assert _status(lambda: cc.EvalMult(ct, ct)) == KEY_MISSING
    assert _status(lambda: cc.EvalRotate(ct, 3)) == KEY_MISSING
    offs, pts = cc.prepare_linear_transform({0: np.ones(cc.N // 2), 5: np.ones(cc.N // 2)}, 4, level=ct.level)
    assert _status(lambda: cc.EvalLinearTransform(ct, offs, pts, 4)) == KEY_MISSING
    # still usable: generate the keys and the same calls succeed
    cc.EvalMultKeyGen(sk)
    cc.EvalRotateKeyGen(sk, [3, 1, 4])
    out = cc.EvalMult(ct, ct, rescale=True)
    assert np.max(np.abs(cc.Decrypt(sk, out).real - 1.0)) < 1e-6
    cc.EvalLinearTransform(ct, offs, pts, 4)


def test_bootstrap_preconditions(ctx):
    cc, sk = ctx
    ct = cc.Encrypt(sk, np.ones(cc.N // 2), level=0)
    assert _status(lambda: cc.EvalBootstrap(ct)) == BAD_ARG  # not set up
    # six moduli are far too few levels for the default bootstrap
    assert _status(lambda: cc.EvalBootstrapSetup()) == BAD_ARG
    # sparse packing is set up the same way (and fails the same way here);
    # slot counts that are not powers of two up to N/2 are refused
    assert _status(lambda: cc.EvalBootstrapSetup(slots=cc.N // 4)) == BAD_ARG
    assert _status(lambda: cc.EvalBootstrapSetup(slots=3)) == BAD_ARG
    assert _status(lambda: cc.EvalBootstrapSetup(slots=cc.N)) == BAD_ARG
    # degree beyond the levels left for a Chebyshev series
    assert _status(lambda: cc.EvalChebyshevSeries(ct, np.ones(64))) == BAD_ARG


def test_bad_arguments(ctx):
    from pyfideslib_b200._capi import lib

    cc, sk = ctx
    ct = cc.Encrypt(sk, np.ones(cc.N // 2))
    assert lib.fides_mult_int(cc._h, None, 3, ct._h) == BAD_ARG
    assert lib.fides_mod_raise(cc._h, ct._h, None) == BAD_ARG
    assert lib.fides_mult_monomial(None, ct._h, 1, ct._h) == BAD_ARG
    assert lib.fides_ntt_batch(cc._h, None, 0, 1, 0, 1, 0) == BAD_ARG
    assert lib.fides_set_ntt_variant(cc._h, 99) == BAD_ARG
    assert lib.fides_set_conv_accumulator(cc._h, 9) == BAD_ARG
    cc.EvalMultKeyGen(sk)  # the serving loop needs the relinearisation key
    srv = F.Server(cc, hbm_budget=4 << 30, max_batch=2, num_streams=1)
    other = cc.Encrypt(sk, np.ones(cc.N // 2), level=ct.level - 1)
    assert _status(lambda: srv.submit(F.Server.HMULT, ct, other)) == BAD_ARG  # levels differ
    assert _status(lambda: srv.submit(F.Server.BOOTSTRAP, ct)) == BAD_ARG  # not set up
    srv.close()


def test_device_error_word_is_reported_once(ctx):
    """A kernel that gives up a bounded wait sets the context's device error
    word.  The word is set here from the host (no kernel fails): the next
    synchronising call returns FIDES_TIMEOUT with a message, clears the word,
    and the call after it is clean; downloads and serving completions report
    it the same way."""
    import ctypes as C

    from pyfideslib_b200._capi import lib

    cc, sk = ctx
    cc.EvalMultKeyGen(sk)
    w = C.c_uint32()
    assert lib.fides_ctx_device_status(cc._h, C.byref(w)) == 0 and w.value == 0
    assert lib.fides_ctx_inject_device_error(cc._h, 1) == 0
    assert lib.fides_ctx_device_status(cc._h, C.byref(w)) == 0 and w.value == 1  # reading does not clear
    assert lib.fides_ctx_synchronize(cc._h) == TIMEOUT
    assert b"tensor-core" in lib.fides_ctx_last_error(cc._h)
    assert lib.fides_ctx_synchronize(cc._h) == 0
    assert lib.fides_ctx_device_status(cc._h, C.byref(w)) == 0 and w.value == 0
    # a download reports it too, and the next download is clean
    ct = cc.Encrypt(sk, np.ones(cc.N // 2))
    assert lib.fides_ctx_inject_device_error(cc._h, 1) == 0
    assert _status(lambda: ct.download()) == TIMEOUT
    c0, c1 = ct.download()
    assert c0.shape == (ct.level + 1, cc.N)
    # a serving completion fails the batch that completes next, not later ones
    srv = F.Server(cc, hbm_budget=4 << 30, max_batch=2, num_streams=1)
    assert lib.fides_ctx_inject_device_error(cc._h, 1) == 0
    rid, _ = srv.submit(F.Server.HMULT, ct, ct)
    assert _status(lambda: srv.wait(rid, 60.0)) == TIMEOUT
    rid, _ = srv.submit(F.Server.HMULT, ct, ct)
    srv.wait(rid, 60.0)
    srv.close()
    assert lib.fides_ctx_synchronize(cc._h) == 0
