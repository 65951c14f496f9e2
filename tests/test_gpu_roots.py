"""Caller-supplied roots of unity (fides_params.q_root / p_root): the
evaluation representation OpenFHE's residues carry is fixed by OpenFHE's
choice of the 2N-th root psi per modulus, which RawParams hands over
(root_of_unity / SPECIALroot_of_unity, src/CKKS/openfhe-interface/
RawCiphertext.cu:235,306) and SetupConstants adopts (src/ConstantsGPU.cu:
195-199).  With another primitive root the forward NTT must equal the
oracle's negacyclic transform at that root in bit-reversed order (the
reference's own check, test/NTTtests.cu:933-1040), the inverse must undo it,
and the evaluation must still decrypt; a root that is not primitive is
refused."""
import numpy as np
import pytest

from gpu_helpers import from_dev, to_dev

pytestmark = pytest.mark.gpu

BAD_ARG = 1


def _bitrev(a):
    n = a.shape[-1]
    lg = n.bit_length() - 1
    idx = [int(format(i, "0%db" % lg)[::-1], 2) for i in range(n)]
    return a[..., idx]


def _other_roots(primes, logN, k):
    """psi^k for the smallest-generator root psi (k odd: still primitive)."""
    from oracle import oracle as O

    return [pow(int(O.unity_root(p, 2 << logN)), k, p) for p in primes]


@pytest.mark.parametrize("logN", [10, 13])
def test_ntt_with_given_roots_matches_oracle(logN):
    import pyfideslib_b200 as F
    from oracle import oracle as O

    q, p = O.moduli(logN, 4, 2)
    qr, pr = _other_roots(q, logN, 3), _other_roots(p, logN, 5)
    cc = F.CryptoContext(log_n=logN, num_q=4, dnum=2, q=q, p=p, q_root=qr, p_root=pr)
    N = 1 << logN
    primes, roots = q + p, qr + pr
    rng = np.random.default_rng(logN)
    v = np.stack([rng.integers(0, pp, N, dtype=np.uint64) for pp in primes])
    d = to_dev(v.copy())
    cc.ntt(d.data_ptr(), 0, len(primes))
    got = from_dev(d)
    for i, (pp, psi) in enumerate(zip(primes, roots)):
        want = O.nega_fft2(v[i], logN, pp, psi)
        assert np.array_equal(_bitrev(got[i]), want), i
    cc.ntt(d.data_ptr(), 0, len(primes), inverse=True)
    assert np.array_equal(from_dev(d), v)


def test_evaluation_with_given_roots_decrypts():
    import pyfideslib_b200 as F
    from oracle import oracle as O

    logN = 12
    q, p = O.moduli(logN, 6, 0, dnum=3)
    cc = F.CryptoContext(log_n=logN, num_q=6, dnum=3, q=q, p=p, q_root=_other_roots(q, logN, 7),
                         p_root=_other_roots(p, logN, 9))
    sk = cc.KeyGen(seed=5, hamming_weight=32)
    cc.EvalMultKeyGen(sk)
    cc.EvalRotateKeyGen(sk, [3])
    rng = np.random.default_rng(2)
    x = rng.uniform(-1, 1, cc.N // 2)
    y = rng.uniform(-1, 1, cc.N // 2)
    ct = cc.EvalMult(cc.Encrypt(sk, x), cc.Encrypt(sk, y), rescale=True)
    assert np.max(np.abs(cc.Decrypt(sk, ct).real - x * y)) < 1e-6
    r = cc.EvalRotate(cc.Encrypt(sk, x), 3)
    assert np.max(np.abs(cc.Decrypt(sk, r).real - np.roll(x, -3))) < 1e-6


def test_non_primitive_root_is_refused():
    import pyfideslib_b200 as F
    from oracle import oracle as O
    from pyfideslib_b200._capi import FidesError

    logN = 10
    q, p = O.moduli(logN, 3, 1)
    bad = _other_roots(q, logN, 1)
    bad[1] = pow(bad[1], 2, q[1])  # order N: psi^N = 1, not -1
    with pytest.raises(FidesError) as e:
        F.CryptoContext(log_n=logN, num_q=3, dnum=1, q=q, p=p, q_root=bad)
    assert e.value.status == BAD_ARG
