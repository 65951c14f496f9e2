"""Extract the known-answer data FIDESlib's own test suite holds for this path
into tests/golden/reference_vectors.json.

Usage: python make_golden.py <path of the reference source tree>.  Sources
read (as text, nothing is executed):
  test/ParametrizedTest.cuh:42-76   prime lists p64 / sp64 (NTT-friendly for logN <= 16)
  test/MathTest.cu:14-39            modpow / modinv known answers
  test/NegacyclicNTTtests.cu:25-125 N=8, p=17 negacyclic convolution vectors
The schoolbook negacyclic product of the N=8 vectors is recomputed here with
Python integers, exactly as the reference test computes its `res` vector.
"""
import json
import os
import re
import sys

if len(sys.argv) != 2:
    sys.exit("usage: python make_golden.py <path of the reference source tree>")
REF = sys.argv[1]
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_vectors.json")


def read(rel):
    with open(os.path.join(REF, rel)) as f:
        return f.read()


def prime_list(src, name):
    m = re.search(r"std::vector<FIDESlib::PrimeRecord>\s+%s\s*\{(.*?)\};" % name, src, re.S)
    return [int(x) for x in re.findall(r"\.p\s*=\s*(\d+)", m.group(1))]


def main():
    pt = read("test/ParametrizedTest.cuh")
    p64 = prime_list(pt, "p64")
    sp64 = prime_list(pt, "sp64")

    mt = read("test/MathTest.cu")
    powmod = []
    for a, e, p, r in re.findall(r"modpow\((\d+),\s*(\d+),\s*(\d+)\),\s*(\d+)\)", mt):
        powmod.append([int(a), int(e), int(p), int(r)])
    invmod = []
    for a, p, r in re.findall(r"modinv\((\d+)(?:ll)?,\s*(\d+)\),\s*(\d+)(?:ll)?\)", mt):
        invmod.append([int(a), int(p), int(r)])
    m = re.search(r"modinv\((\d+)ll,\s*\(\(1ll << (\d+)\) - 1\)\),\s*(\d+)ll\)", mt)
    if m:
        invmod.append([int(m.group(1)), (1 << int(m.group(2))) - 1, int(m.group(3))])

    nt = read("test/NegacyclicNTTtests.cu")
    body = nt[nt.index("TEST_P(NegacyclicNTTTest, TestCpuNTT)"):]
    v1 = [int(x) for x in re.search(r"v1\{([^}]*)\}", body).group(1).split(",")]
    v2 = [int(x) for x in re.search(r"v2\{([^}]*)\}", body).group(1).split(",")]
    p = int(re.search(r"primes\[0\]\.p\s*=\s*(\d+)", body).group(1))
    logN = int(re.search(r"custom\.logN\s*=\s*(\d+)", body).group(1))
    N = 1 << logN
    res = [0] * N
    for i in range(N):
        for j in range(N):
            if i + j >= N:
                res[i + j - N] = (res[i + j - N] - v1[i] * v2[j]) % p
            else:
                res[i + j] = (res[i + j] + v1[i] * v2[j]) % p

    data = {
        "source": "FIDESlib test suite (test/ParametrizedTest.cuh, test/MathTest.cu, test/NegacyclicNTTtests.cu)",
        "p64": p64,
        "sp64": sp64,
        "powmod": powmod,
        "invmod": invmod,
        "negacyclic_n8": {"logN": logN, "p": p, "v1": v1, "v2": v2, "product": res},
    }
    with open(OUT, "w") as f:
        json.dump(data, f, indent=1)
    print("wrote", OUT, "p64:", len(p64), "sp64:", len(sp64), "powmod:", len(powmod), "invmod:", len(invmod))


if __name__ == "__main__":
    main()
