// common.cuh -- device-side context view and limb addressing shared by all
// kernels of the evaluation core.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "modarith.cuh"

namespace fides {

constexpr int kMaxPrimes = 128;
constexpr int kMaxSeg = 8;
constexpr int kMaxBatch = 32;  // ciphertexts per batched launch (blockIdx.z)

// Bits of a context's device error word (DevCtx::err).  A kernel whose
// bounded wait gives up sets its bit and leaves invalid outputs; the next
// synchronising call of the context reports FIDES_TIMEOUT and clears the word.
constexpr uint32_t kDevErrTensorWait = 1u;  // a tensor-core conversion stopped waiting for its MMAs

// Counter-based generator behind every seeded uniform draw (a halves of keys
// and public keys, synthetic ciphertexts).  hash64 is a 64-bit finaliser of
// MurmurHash3's form (a bijection with full avalanche).  A draw is keyed by a
// stream word, uniform_stream(seed, tag) = hash64(seed) ^ tag << 48, mixed
// once on the host; residue j of prime t is
//   uniform_mod(stream, t, j, p) = floor(hash64(stream ^ t << 32 ^ j) * p / 2^64),
// one finaliser per residue.  The counter stream ^ t << 32 ^ j is distinct for
// every (tag, t, j) of a seed (tag, t < 2^16, j < 2^32).  Not a cryptographic
// generator.
__host__ __device__ __forceinline__ uint64_t hash64(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}
__host__ __device__ __forceinline__ uint64_t uniform_stream(uint64_t seed, uint32_t tag) {
    return hash64(seed) ^ ((uint64_t)tag << 48);
}
__device__ __forceinline__ uint64_t uniform_mod(uint64_t stream, int prime, uint32_t j, uint64_t p) {
    return __umul64hi(hash64(stream ^ ((uint64_t)prime << 32) ^ j), p);
}

// Read-only view of the context tables in HBM, passed by value to kernels.
// Index conventions: prime ids 0..L-1 are the Q primes, L..L+K-1 the special
// primes.  Every table entry with a Shoup companion stores (value, companion)
// adjacently.
struct DevCtx {
    int logN, N, L, K, dnum, alpha;
    int ntt_variant;             // forward NTT kernel variant chosen by the autotuner
    int intt_variant;            // inverse NTT kernel configuration (0..2)
    int ks_variant;              // key-switch inner product: bit 0 set: FP64 sums on primes below 2^50
                                 // (else integer sums); bit 1 set: HMult's inner product runs in the
                                 // epilogue of the ModUp digits' NTT row pass (else its own kernel);
                                 // bit 2 set: the same for HMult batches of 8 or more elements;
                                 // bit 3 set: that fused row pass in two launches (ciphertext-
                                 // prime outputs at 3 CTAs per SM, special-prime outputs at 2)
    int conv_variant;            // base conversions: 0 2 coefficients/thread 128-bit sums, 1 the same with
                                 // split 32-bit products (moduli < 2^60), 2 one coefficient/thread,
                                 // 3 and 4 ModUp and ModDown on the tensor cores (int8 split, 32
                                 // or 16 targets per MMA)
    const PrimeConst* pc;        // [L+K]
    const uint64_t* fwd_tw;      // [L+K][N][2]  psi^{bitrev(i)}, companion
    const uint64_t* inv_tw;      // [L+K][N][2]  psi^{-bitrev(i)}, companion
    const uint64_t* fwd_twf;     // [L+K][N][2]  bit patterns of the doubles w = psi^{bitrev(i)} and w / p
                                 //              (primes below 2^50; zero rows otherwise)
    const uint64_t* inv_twf;     // [L+K][N][2]  the same for psi^{-bitrev(i)}
    const uint64_t* intt_scale;  // [L+K][4]     s=N^-1, s', s*w1, (s*w1)'  (w1 = inverse twiddle 1)
    const uint64_t* modup_scale; // [L][L][4]    same with s = N^-1 * (Q'/q_i)^-1 for level, prime
    const uint64_t* modup_mat;   // [L][L][L+K]  (Q'/q_i) mod t for level, input prime i, target prime t
    const uint64_t* md_scale;    // [K][4]       same with s = N^-1 * (P/p_k)^-1
    const uint64_t* md_mat;      // [K][L]       (P/p_k) mod q_j
    const uint64_t* md_pinv;     // [L][2]       P^-1 mod q_j
    const uint64_t* md_pmod;     // [L][2]       P mod q_j
    const uint64_t* rs_qinv;     // [L][L][2]    q_l^-1 mod q_j (row l, column j < l)
    const uint8_t* tc_btab;      // tensor-core conversions: byte matrices B per (level, digit) and
    const uint64_t* tc_boff;     //   per (level, fused) for ModDown, and their byte offsets (or null)
    uint32_t* err;               // the context's device error word (kDevErr* bits)
};

// A launch covers up to kMaxSeg segments of contiguous limbs.  Within a
// segment, limb i (0 <= i < count) sits at in/out + i*N and maps to prime
//   j = i < skip_lo ? i : i + skip_cnt;   prime = j < nq ? q0 + j : L + (j - nq).
struct LimbSeg {
    const uint64_t* in;
    const uint64_t* in2;
    const uint64_t* in3;
    uint64_t* out;
    int count;
    int skip_lo, skip_cnt;
    int nq, q0;
    int level;  // level used by level-dependent tables (-1 if unused)
    int in_stride_zero;  // 1: every limb reads the same input limb
    int8_t lmode;  // transform prologue mode (FL_* forward, IL_* inverse)
    int8_t smode;  // transform epilogue mode (FS_* forward, IS_* inverse)
    int8_t out_tab;  // t > 0: batch element b writes to LimbMap::bout[t - 1][b] (+ limb offset)
    int8_t pad;
    size_t bstride;  // batch element b adds b * bstride words to in/in2/in3/out
};

struct LimbMap {
    int nseg;
    int total;
    int nb;  // batch elements (gridDim.z); 0 means 1
    LimbSeg seg[kMaxSeg];
    uint64_t* bout[2][kMaxBatch];
};

struct LimbRef {
    const uint64_t* in;
    const uint64_t* in2;
    const uint64_t* in3;
    uint64_t* out;
    int prime;
    int level;
    int lmode, smode;
};

__device__ __forceinline__ LimbRef resolve_limb(const LimbMap& m, int f, int b, int N, int L) {
    int s = 0;
#pragma unroll 1
    while (s < m.nseg - 1 && f >= m.seg[s].count) {
        f -= m.seg[s].count;
        ++s;
    }
    const LimbSeg& g = m.seg[s];
    LimbRef r;
    const size_t off = (size_t)f * N;
    const size_t bo = (size_t)b * g.bstride;
    r.in = g.in ? g.in + bo + (g.in_stride_zero ? 0 : off) : nullptr;
    r.in2 = g.in2 ? g.in2 + bo + off : nullptr;
    r.in3 = g.in3 ? g.in3 + bo + off : nullptr;
    if (g.out_tab > 0)
        r.out = m.bout[g.out_tab - 1][b] + off;
    else
        r.out = g.out ? g.out + bo + off : nullptr;
    const int j = f < g.skip_lo ? f : f + g.skip_cnt;
    r.prime = j < g.nq ? g.q0 + j : L + (j - g.nq);
    r.level = g.level;
    r.lmode = g.lmode;
    r.smode = g.smode;
    return r;
}

}  // namespace fides
