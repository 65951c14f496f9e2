"""CPU-side checks of the boundary: the C-ABI library loads and exports every
symbol include/fides_b200.h declares (no compute call is made without a GPU),
and the host-side modular arithmetic used by the kernels agrees with 128-bit
integer arithmetic."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"^\s*(?:[\w\*]+\s+)+\**(fides_\w+)\s*\(", src, re.M))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    import ctypes

    path = os.path.join(ROOT, "pyfideslib_b200", "libfidesb200.so")
    assert os.path.exists(path), "build the library first (__graft_entry__.build())"
    lib = ctypes.CDLL(path)
    names = declared_symbols()
    assert len(names) > 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_bindings_cover_header():
    from pyfideslib_b200 import _capi

    assert set(declared_symbols()) <= set(_capi.EXPORTS)


def test_bad_arguments_rejected_without_gpu():
    import ctypes

    from pyfideslib_b200 import _capi

    lib = _capi.lib
    assert lib.fides_ctx_create(None, None) == 1
    prm = _capi.FidesParams()
    prm.log_n, prm.num_q, prm.dnum = 20, 4, 2  # unsupported ring dimension
    h = ctypes.c_void_p()
    assert lib.fides_ctx_create(ctypes.byref(prm), ctypes.byref(h)) == 1
    assert lib.fides_ctx_destroy(None) == 1


HOST_TEST = r"""
#include "modarith.cuh"
#include <cstdio>
#include <random>
using namespace fides;
int main(int argc, char** argv) {
    std::mt19937_64 r(1);
    const uint64_t primes[] = {17ull, 2305843009218281473ull, 2251799661248513ull, 2305843009247641601ull,
                               (1ull << 61) - 1, 4611686018427387847ull /* < 2^62 */,
                               1152921504606830593ull /* < 2^60 */};
    for (uint64_t p : primes) {
        PrimeConst c{};
        c.p = p; c.two_p = 2 * p;
        c.mu64 = (uint64_t)((((unsigned __int128)1) << 64) / p);
        c.r64 = (uint64_t)((((unsigned __int128)1) << 64) % p);
        c.r64_sh = shoup_precompute(c.r64, p);
        for (int t = 0; t < 200000; ++t) {
            uint64_t a = r() % p, b = r() % p, w = r() % p;
            if (mul_mod(a, b, c) != (uint64_t)((unsigned __int128)a * b % p)) { printf("mul_mod %llu\n", (unsigned long long)p); return 1; }
            uint64_t ws = shoup_precompute(w, p);
            uint64_t big = r();
            if (mul_shoup(big, w, ws, p) != (uint64_t)((unsigned __int128)big * w % p)) { printf("shoup\n"); return 1; }
            unsigned __int128 z = ((unsigned __int128)r() << 64) | r();
            if (reduce128((uint64_t)(z >> 64), (uint64_t)z, c) != (uint64_t)(z % p)) { printf("reduce128\n"); return 1; }
            Acc128 acc; unsigned __int128 ref = 0;
            for (int k = 0; k < 15; ++k) { uint64_t x = r() % p, y = r() % p; acc.mac(x, y); ref += (unsigned __int128)x * y; }
            if (acc.reduce(c) != (uint64_t)(ref % p)) { printf("acc\n"); return 1; }
            if (p < (1ull << 60)) {
                AccSplit sa; unsigned __int128 sref = 0;
                for (int k = 0; k < 16; ++k) {
                    uint64_t x = (t & 1) ? p - 1 - (r() & 7) : r() % p, y = (t & 2) ? p - 1 : r() % p;
                    sa.mac(x, y); sref += (unsigned __int128)x * y;
                }
                if (sa.reduce(c) != (uint64_t)(sref % p)) { printf("accsplit\n"); return 1; }
            }
        }
    }
    printf("ok\n");
    return 0;
}
"""


def test_host_modular_arithmetic(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text(HOST_TEST)
    exe = tmp_path / "t"
    inc = os.path.join(ROOT, "pyfideslib_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", inc, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and "ok" in out.stdout, out.stdout


def test_generated_moduli_match_oracle_search():
    """The product's prime search and the oracle's independent one agree."""
    from oracle import oracle as O
    from pyfideslib_b200.host_params import generated_moduli

    q, p = generated_moduli(16, 30, 10, 3)
    assert len(q) == 30 and len(p) == 10
    assert q[0] == O.find_primes(16, 60, 1)[0]
    assert q[1:] == O.find_primes(16, 50, 29)
    assert p == [x for x in O.find_primes(16, 60, 12) if x not in q][:10]
    for x in q + p:
        assert O.is_prime(x) and (x - 1) % (1 << 17) == 0
    q2, p2 = generated_moduli(16, 30, 0, 3)  # K derived from the widest digit
    assert len(p2) == 9


@pytest.mark.parametrize("args", [dict(logN=16, L=30, K=10), dict(logN=16, L=20, K=0, qi_bits=40),
                                  dict(logN=12, L=8, K=3), dict(logN=16, L=30, K=0)])
def test_oracle_moduli_match_library(args):
    """The oracle's restated parameter rule gives the library's moduli, so the
    CPU reference arm of bench.py needs no product code to build its context."""
    from oracle import oracle as O
    from pyfideslib_b200.host_params import generated_moduli

    q, p = O.moduli(args["logN"], args["L"], args["K"], 3, qi_bits=args.get("qi_bits", 50))
    gq, gp = generated_moduli(args["logN"], args["L"], args["K"], 3, qi_bits=args.get("qi_bits", 50))
    assert (q, p) == (gq, gp)


def test_reference_arm_loads_no_product_code():
    """bench.py --impl reference maps only oracle/ libraries (checked in a
    child process on a tiny run: the import graph, not the timing)."""
    code = ("import sys, runpy; sys.argv=['bench.py','--impl','reference','--steps','1','--warmup','0','--batch','1'];"
            "import bench; bench.LOGN=12; bench.L=6; bench.K=2;"
            "bench.run_reference(bench.argparse.Namespace(steps=1, warmup=0, batch=1, gpus=1));"
            "maps=open('/proc/self/maps').read(); print('LOADED' if 'libfidesb200' in maps else 'CLEAN');"
            "print('MOD' if any(m.startswith('pyfideslib_b200') for m in sys.modules) else 'NOMOD')")
    r = subprocess.run([os.environ.get("PYTHON", "python"), "-c", code], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "CLEAN" in r.stdout and "NOMOD" in r.stdout, r.stdout


def test_reference_gpu_harness_loads():
    """The reference-kernel harness (oracle/_ref/libfidesref_gpu.so, built
    where the reference tree is mounted) resolves every symbol it links and
    exports its entry points; loading needs no GPU."""
    import ctypes

    lib_path = os.path.join(ROOT, "oracle", "_ref", "libfidesref_gpu.so")
    if not os.path.exists(lib_path):
        pytest.skip("the reference's GPU kernels were not built here")
    lib = ctypes.CDLL(lib_path)
    for name in ("refgpu_init", "refgpu_transform", "refgpu_set_keyswitch", "refgpu_modup_conv",
                 "refgpu_moddown_conv", "refgpu_dot", "refgpu_binomial", "refgpu_automorph",
                 "refgpu_hoisted_dot", "refgpu_release"):
        assert hasattr(lib, name), name
