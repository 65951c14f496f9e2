// fp64.cuh -- exact modular arithmetic on the FP64 pipes for primes below 2^50.
//
// Residues are held exactly as integer-valued doubles (values below 2^53 in
// magnitude are exact).  A product y w = h + l is split exactly by an FMA
// (h = fl(y w), l = fma(y, w, -h)); a quotient estimate q, rounded to an
// integer through the 1.5 * 2^52 shift (valid while |q| < 2^51), gives the
// remainder fma(-q, p, h) + l exactly.  Used by the NTT butterflies (ntt.cu)
// and the key-switch inner product (ks.cu); the integer pipes that the 64-bit
// Shoup/Barrett forms keep busy are left free.
#pragma once
#include <stdint.h>

namespace fides {

constexpr double kRint = 6755399441055744.0;  // 1.5 * 2^52
constexpr double kTwo52 = 4503599627370496.0;
constexpr uint64_t kMant52 = (1ull << 52) - 1;

__device__ __forceinline__ double as_f64(uint64_t v) { return __longlong_as_double((long long)v); }
__device__ __forceinline__ uint64_t as_u64(double v) { return (uint64_t)__double_as_longlong(v); }

// residue below 2^52 -> the same integer as a double
__device__ __forceinline__ uint64_t fp_from_u(uint64_t v) {
    return as_u64(__dsub_rn(as_f64(v | 0x4330000000000000ull), kTwo52));
}

// y w - q p with q = rint(y w / p) to within 1/2 + |y| 2^-54 (|y| < 2^51)
__device__ __forceinline__ double fp_mulw(double y, double w, double wq, double p) {
    const double h = __dmul_rn(y, w);
    const double l = __fma_rn(y, w, -h);
    const double q = __dsub_rn(__fma_rn(y, wq, kRint), kRint);
    return __dadd_rn(__fma_rn(-q, p, h), l);
}

// x - rint(x / p) p, magnitude <= p/2 + |x| 2^-52 (|x| < 2^51)
__device__ __forceinline__ double fp_center(double x, double p, double pinv) {
    const double q = __dsub_rn(__fma_rn(x, pinv, kRint), kRint);
    return __fma_rn(-q, p, x);
}

// canonical residue of an integer-valued v in (-2p, 2p); pinv_up >= 1/p.
// a = v + 2p lies in (0, 4p); floor(a pinv_up) = floor(a / p) because a / p
// is at least 1/p > 2^-50 away from the next integer while the rounding of
// 1/p moves it by at most 4 * 2^-52.
__device__ __forceinline__ uint64_t fp_to_u(double v, double p, double pinv_up) {
    const double two_p = __dadd_rn(p, p);
    const double a = __dadd_rn(v, two_p);
    const double b = __dadd_rn(v, __dadd_rn(two_p, kTwo52));  // a + 2^52, exact
    const double q = __dsub_rn(__fma_rd(a, pinv_up, kRint), kRint);
    return as_u64(__fma_rn(-q, p, b)) & kMant52;  // (a - q p) + 2^52 -> low 52 bits
}

// x y mod p up to a multiple of p for residues x, y < p < 2^50 (pinv >= 1/p,
// within 2^-52 relative): q = rint(fl(x y) pinv) is within 1/2 + 3/8 of x y / p,
// so the result r = x y - q p is exact with |r| <= 0.875 p.
__device__ __forceinline__ double fp_mulmod(double x, double y, double p, double pinv) {
    const double h = __dmul_rn(x, y);
    const double l = __fma_rn(x, y, -h);
    const double q = __dsub_rn(__fma_rn(h, pinv, kRint), kRint);
    return __dadd_rn(__fma_rn(-q, p, h), l);
}

}  // namespace fides
