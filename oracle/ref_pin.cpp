// ref_pin.cpp -- C entry points over the reference's own CPU negacyclic NTT
// (test/cpuNTT_nega.cpp:24-264, nega_fft and nega_fft2, and the cyclic fft of
// test/cpuNTT.cpp:14-47 that nega_fft2 calls), compiled unmodified from the
// reference tree into oracle/_ref/libfidesref.so.  TEST INFRASTRUCTURE ONLY:
// tests/test_oracle_ref_pin.py checks the oracle's transform against it.
#include <cstdint>
#include <vector>

#include "cpuNTT_nega.hpp"

extern "C" {

// a[0..n) in place; psi / inv_psi are the bit-reversed power tables of the
// 2n-th root (only entries n/2 and n/4 are read by nega_fft2); natural-order output
void ref_nega_fft2(uint64_t* a, int n, const uint64_t* psi, const uint64_t* inv_psi, uint64_t mod, int invert) {
    std::vector<uint64_t> v(a, a + n);
    FIDESlib::Testing::nega_fft2(v, invert != 0, psi, inv_psi, mod);
    for (int i = 0; i < n; ++i) a[i] = v[i];
}

// the in-place Cooley-Tukey form over the same tables, bit-reversal swap included
void ref_nega_fft(uint64_t* a, int n, const uint64_t* psi, const uint64_t* inv_psi, uint64_t mod, int invert) {
    std::vector<uint64_t> v(a, a + n);
    FIDESlib::Testing::nega_fft(v, invert != 0, psi, inv_psi, mod);
    for (int i = 0; i < n; ++i) a[i] = v[i];
}

}  // extern "C"
