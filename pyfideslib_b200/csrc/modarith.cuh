// modarith.cuh -- 64-bit modular arithmetic for residues modulo NTT primes
// p < 2^62, shared by the CUDA kernels and the host code.
//
// All products here are on the integer pipes (IMAD); nothing is approximated.
// (The NTT also has exact double-precision butterflies for primes below
// 2^50, in ntt.cu.)
// Canonical residues live in [0, p); the transforms keep Harvey's lazy
// ranges [0, 2p) / [0, 4p) internally and reduce at the end.
//
// Role in the reference: src/ModMult.cuh:46-313 (Shoup_mult_64, Neal_mult_64,
// modreduce on 128-bit values) and src/AddSub.cuh:37-49.  The formulations
// below are independent: Shoup's precomputed-quotient product (V. Shoup,
// NTL; D. Harvey, "Faster arithmetic for number-theoretic transforms", 2014)
// for products by a constant, and a two-step reduction of 128-bit values
// (high word by Shoup with 2^64 mod p, low word by a one-word Barrett
// quotient) for products of two variables and for 128-bit accumulators.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define FHD __host__ __device__ __forceinline__
#else
#define FHD inline
#endif

namespace fides {

FHD uint64_t mulhi64(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

// Per-prime constants needed by the reductions.
struct PrimeConst {
    uint64_t p;
    uint64_t two_p;
    uint64_t mu64;    // floor(2^64 / p)
    uint64_t r64;     // 2^64 mod p
    uint64_t r64_sh;  // Shoup companion of r64
    uint64_t ninv;    // N^-1 mod p
    uint64_t ninv_sh;
    uint64_t pinv_f64;  // bit pattern of the double 1/p rounded up (p < 2^50; 0 otherwise)
};

// Forward transforms of primes below this bound run their butterflies on the
// FP64 pipes (residues held exactly as doubles, see ntt.cu).
constexpr uint64_t kFpPrimeBound = 1ull << 50;

// floor(w * 2^64 / p), host only (needs a 128-bit division).
inline uint64_t shoup_precompute(uint64_t w, uint64_t p) {
    return (uint64_t)(((unsigned __int128)w << 64) / p);
}

FHD uint64_t csub(uint64_t x, uint64_t m) { return x >= m ? x - m : x; }

FHD uint64_t add_mod(uint64_t a, uint64_t b, uint64_t p) { return csub(a + b, p); }
FHD uint64_t sub_mod(uint64_t a, uint64_t b, uint64_t p) { return a >= b ? a - b : a + p - b; }
FHD uint64_t neg_mod(uint64_t a, uint64_t p) { return a ? p - a : 0; }

// a * w mod p in [0, 2p) for any a < 2^64 (w < p, w_sh = floor(w 2^64 / p)).
FHD uint64_t mul_shoup_lazy(uint64_t a, uint64_t w, uint64_t w_sh, uint64_t p) {
    const uint64_t q = mulhi64(a, w_sh);
    return a * w - q * p;
}
FHD uint64_t mul_shoup(uint64_t a, uint64_t w, uint64_t w_sh, uint64_t p) {
    return csub(mul_shoup_lazy(a, w, w_sh, p), p);
}

// x mod p for x < 2^64 via q = floor(x * mu64 / 2^64) (q >= floor(x/p) - 1).
FHD uint64_t reduce64_lazy(uint64_t x, const PrimeConst& c) {  // result in [0, 2p)
    return x - mulhi64(x, c.mu64) * c.p;
}

// (hi*2^64 + lo) mod p, any 128-bit value, canonical result.
FHD uint64_t reduce128(uint64_t hi, uint64_t lo, const PrimeConst& c) {
    uint64_t a = mul_shoup_lazy(hi, c.r64, c.r64_sh, c.p);  // [0, 2p)
    uint64_t b = reduce64_lazy(lo, c);                       // [0, 2p)
    uint64_t s = a + b;                                      // [0, 4p) < 2^64 for p < 2^62
    s = csub(s, c.two_p);
    return csub(s, c.p);
}

// Centred lift of a residue a mod om into the modulus of nc
// (src/CKKS/Rescale.cuh:45-62): a > om/2 stands for a - om.
FHD uint64_t switch_modulus(uint64_t a, uint64_t om, const PrimeConst& nc) {
    const uint64_t nm = nc.p;
    if (nm > om) return a > (om >> 1) ? a + (nm - om) : a;
    const uint64_t om_mod = csub(reduce64_lazy(om, nc), nm);
    uint64_t v = a > (om >> 1) ? a + (nm - om_mod) : a;
    return csub(reduce64_lazy(v, nc), nm);
}

// 128-bit accumulator of 64x64 products.
struct Acc128 {
    uint64_t lo, hi;
    FHD Acc128() : lo(0), hi(0) {}
    FHD void mac(uint64_t a, uint64_t b) {
        const uint64_t l = a * b;
        const uint64_t h = mulhi64(a, b);
        lo += l;
        hi += h + (lo < l ? 1 : 0);
    }
    FHD uint64_t reduce(const PrimeConst& c) const { return reduce128(hi, lo, c); }
};

// Sum of up to 16 products of residues below 2^60 kept as 32-bit partial
// products (a = a1 2^32 + a0, b = b1 2^32 + b0, a1, b1 < 2^28):
//   s11 = sum a1 b1 < 2^60,  s10 = sum a1 b0 < 2^64,  s01 = sum a0 b1 < 2^64,
//   w = sum a0 b0 < 2^68 in three 32-bit words.
// Each product costs four multiply-adds and no carry handling between 64-bit
// halves; the 128-bit total is formed once, in reduce().  Same value as Acc128.
struct AccSplit {
    uint64_t s11, s10, s01;
    uint32_t w0, w1, w2;
    FHD AccSplit() : s11(0), s10(0), s01(0), w0(0), w1(0), w2(0) {}
    FHD void mac(uint64_t a, uint64_t b) {
        const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32), b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
        s11 += (uint64_t)a1 * b1;
        s10 += (uint64_t)a1 * b0;
        s01 += (uint64_t)a0 * b1;
#if defined(__CUDA_ARCH__)
        asm("mad.lo.cc.u32 %0, %3, %4, %0;\n\t"
            "madc.hi.cc.u32 %1, %3, %4, %1;\n\t"
            "addc.u32 %2, %2, 0;"
            : "+r"(w0), "+r"(w1), "+r"(w2)
            : "r"(a0), "r"(b0));
#else
        const unsigned __int128 w = (((unsigned __int128)w2 << 64) | ((uint64_t)w1 << 32) | w0) + (uint64_t)a0 * b0;
        w0 = (uint32_t)w;
        w1 = (uint32_t)(w >> 32);
        w2 = (uint32_t)(w >> 64);
#endif
    }
    // total = s11 2^64 + (s10 + s01) 2^32 + (w2 2^64 + w1 2^32 + w0)
    FHD uint64_t reduce(const PrimeConst& c) const {
        const uint64_t mid = s10 + s01;
        const uint64_t mid_carry = mid < s10 ? 1 : 0;  // bit 64 of s10 + s01
        const uint64_t lo0 = ((uint64_t)w1 << 32) | w0;
        const uint64_t lo = lo0 + (mid << 32);
        const uint64_t hi = s11 + (mid >> 32) + (mid_carry << 32) + w2 + (lo < lo0 ? 1 : 0);
        return reduce128(hi, lo, c);
    }
};

FHD uint64_t mul_mod(uint64_t a, uint64_t b, const PrimeConst& c) {
    return reduce128(mulhi64(a, b), a * b, c);
}

}  // namespace fides
