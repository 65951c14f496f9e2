"""Decryption's decoding on the device: the mixed-radix CRT of the first three
moduli and the forward embedding FFT (the client-side step FIDESlib leaves to
OpenFHE's Decrypt, api/CryptoContext.cpp:560-626).

A trivial ciphertext (c1 = 0) holds known signed integer coefficients, so
that decryption with any key returns their canonical embedding divided by the
scale; it is compared with numpy's FFT of the same integers.  Magnitudes reach
past q0 (two moduli in the CRT) and past q0 q1 (three), negative values
included.
"""
import random

import numpy as np
import pytest

from gpu_helpers import make_pair

pytestmark = pytest.mark.gpu


def _embed(x, N, scale, slots):
    """slot j = sum_t (x_t / scale) zeta^(5^j t), zeta = exp(i pi / N)."""
    a = np.array([float(v) for v in x]) / scale * np.exp(1j * np.pi * np.arange(N) / N)
    A = np.fft.ifft(a) * N  # sum_t a_t exp(+2 pi i t k / N)
    idx = [(pow(5, j, 2 * N) - 1) // 2 for j in range(slots)]
    return A[idx]


def _residues(x, primes):
    return np.array([[v % p for v in x] for p in primes], dtype=np.uint64)


@pytest.mark.parametrize("level,bits", [(0, 58), (1, 100), (5, 150)])
def test_decrypt_decodes_trivial_ciphertext(level, bits):
    logN = 12
    cc, oc = make_pair(logN, 8, 3, 3)
    N = cc.N
    sk = cc.KeyGen(seed=7, hamming_weight=32)
    r = random.Random(bits)
    x = [r.getrandbits(r.randrange(bits)) * r.choice((1, -1)) for _ in range(N)]
    x[0], x[1] = (1 << bits) - 1, -(1 << bits) + 1
    primes = oc.primes[:level + 1]
    bound = 1
    for p in primes[:3]:
        bound *= p
    assert max(abs(v) for v in x) < bound // 2
    c0 = oc.ntt(_residues(x, primes), list(range(level + 1)))
    c1 = np.zeros_like(c0)
    scale = 2.0 ** (bits - 20)
    ct = cc.upload(c0, c1, level=level, scale=scale)
    for slots in (N // 2, 8):
        got = cc.Decrypt(sk, ct, slots=slots)
        want = _embed(x, N, scale, slots)
        # FP64: the CRT's conversion and the FFT's stages, relative to the
        # largest possible slot value
        tol = 1e-12 * sum(abs(float(v)) for v in x) / scale
        assert np.max(np.abs(got - want)) < tol


def test_encryption_error_has_sigma_3_2():
    """Encryption's error is drawn on the device (rounded Gaussian, sigma 3.2).
    An encryption of zeros at scale 1 decrypts to the embedding of the error
    itself, whose mean squared slot is N (sigma^2 + 1/12) by Parseval."""
    import pyfideslib_b200 as F

    cc = F.CryptoContext(log_n=12, num_q=4, dnum=2)
    sk = cc.KeyGen(seed=3, hamming_weight=32)
    N = cc.N
    ests = []
    for seed in (11, 12, 13, 14):
        ct = cc.Encrypt(sk, np.zeros(N // 2), level=0, scale=1.0, seed=seed)
        z = cc.Decrypt(sk, ct)
        ests.append(np.sqrt(np.mean(np.abs(z) ** 2) / N))
    want = np.sqrt(3.2 ** 2 + 1.0 / 12)
    assert all(abs(e - want) < 0.12 * want for e in ests)
    assert len(set(float(e) for e in ests)) == 4  # seeds give different draws
    assert abs(np.mean(ests) - want) < 0.06 * want
