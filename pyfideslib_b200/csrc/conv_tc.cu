// conv_tc.cu -- ModUp and ModDown base conversions on the 5th-generation
// tensor cores.
//
// Role in the reference: DecompAndModUpConv and ModDown2 (src/CKKS/Conv.cu),
// the same contractions as k_modup_conv / k_moddown_conv in ks.cu:
//   out[m][j] = sum_i x_i[j] * M[i][m]  (mod p_m),
// with M[i][m] = (Q'/q_i) mod p_m over the cnt limbs i of one digit (ModUp),
// or (P/p_k) mod q_m over the K special limbs (ModDown), for ntar targets m.
//
// Exact int8 split (this file's own design): with x_i = sum_a x_{i,a} 2^{8a}
// (bytes) and the pre-shifted constants M'_{i,m,a} = M[i][m] 2^{8a} mod p_m
// = sum_s M'_{i,m,a,s} 2^{8s} (bytes), the value
//   V'[j][m] = sum_i sum_a x_{i,a} M'_{i,m,a} = sum_{s<8} c_s 2^{8s},
//   c_s = sum_i sum_a x_{i,a} M'_{i,m,a,s},
// is congruent to V mod p_m, and every c_s is one entry of an unsigned 8-bit
// matrix product A[j][(i,a)] = x_{i,a}, B[(i,a)][(m,s)] = M'_{i,m,a,s},
// accumulated exactly in 32 bits (c_s < 16 * 8 * 255^2 < 2^23).  Folding the
// byte position of x into the constants keeps V' below 2^80 and needs 8
// columns per target, against 2^128 and 15 columns for the plain split.
// A tile of 128 coefficients is multiplied by B with tcgen05.mma kind::i8
// (M = 128, N = 8 columns per target, K = 32 bytes per instruction) into
// tensor memory; the epilogue reads each coefficient's column sums with
// tcgen05.ld, reassembles V' and reduces it with one Barrett step
// (q = floor(floor(V'/2^16) floor(2^80/p) / 2^64), remainder in [0, 2p)).
// The tensor cores take the 64x64-bit products off the integer pipes; what
// is left there is a few shifts and adds and one 64-bit quotient per output.
//
// Operands sit in shared memory in the canonical K-major layout without
// swizzle: core matrices of 8 rows x 16 bytes stored contiguously, 8-row
// groups 128 bytes apart (SBO) and 16-byte K chunks LBO bytes apart.  A is
// rebuilt per tile from coalesced limb loads; every B (per level and digit,
// per level for ModDown) is built once per context and copied in by each
// CTA.  Every wait on the MMA completion barrier is bounded; a timeout sets an
// error flag and the CTA releases its tensor memory and returns.
#include <algorithm>
#include <mutex>
#include <vector>

#include "kernels.hpp"

namespace fides {

namespace {

constexpr int kTcThreads = 256;     // 8 warps: two per tensor-memory lane quarter
constexpr int kTcRows = 128;        // coefficients per tile (MMA M)
constexpr int kTcCols = 8;          // accumulator columns per target (byte positions 0..7 of V')
constexpr uint32_t kTcLboA = (kTcRows / 8) * 128;  // A: K-chunk stride in bytes
constexpr uint32_t kSpinLimit = 1u << 20;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor (canonical K-major, no swizzle)
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100; base offset 0, no swizzle
    return d;
}

// instruction descriptor of kind::i8: unsigned A and B, s32 accumulator,
// both operands K-major, shape M x N
__host__ __device__ constexpr uint32_t idesc_u8(int M, int N) {
    return (2u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_u8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ bool wait_parity(uint32_t bar, uint32_t phase) {
    for (uint32_t it = 0; it < kSpinLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

// 16 consecutive accumulator columns of this thread's lane (no wait)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&c)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];\n"
        : "=r"(c[0]), "=r"(c[1]), "=r"(c[2]), "=r"(c[3]), "=r"(c[4]), "=r"(c[5]), "=r"(c[6]), "=r"(c[7]),
          "=r"(c[8]), "=r"(c[9]), "=r"(c[10]), "=r"(c[11]), "=r"(c[12]), "=r"(c[13]), "=r"(c[14]), "=r"(c[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

// V' mod p for V' = sum_{s<8} c_s 2^{8s}, c_s < 2^23, 2^17 <= p < 2^62.
// The pairs w_k = c_{2k} + c_{2k+1} 2^8 fit 32 bits, and with
// e = w_0 + w_2 2^32, o = w_1 + w_3 2^32:  V' = e + o 2^16,
// floor(V'/2^16) = floor(e/2^16) + o  and  V' mod 2^64 = e + (o << 16).
// V' < 2^79.01, so with mu = floor(2^80/p) the Barrett quotient
// q = floor(floor(V'/2^16) mu / 2^64) is floor(V'/p) or one less, and
// V' - q p (formed modulo 2^64) lies in [0, 2p).
__device__ __forceinline__ uint64_t reduce_cols(const uint32_t* c, uint64_t mu, uint64_t p) {
    const uint32_t w0 = c[0] + (c[1] << 8), w1 = c[2] + (c[3] << 8);
    const uint32_t w2 = c[4] + (c[5] << 8), w3 = c[6] + (c[7] << 8);
    const uint64_t e = ((uint64_t)w2 << 32) | w0;
    const uint64_t o = ((uint64_t)w3 << 32) | w1;
    const uint64_t q = __umul64hi((e >> 16) + o, mu);
    const uint64_t r = e + (o << 16) - q * p;
    return r >= p ? r - p : r;
}

// target index m of a digit -> prime id (the other Q primes, then the special ones)
__device__ __forceinline__ int target_prime(int m, int lo, int cnt, int n, int L) {
    const int jj = m < lo ? m : m + cnt;
    return jj < n ? jj : L + (jj - n);
}

// Geometry of one conversion: the digit's limbs (ModUp) or the K special
// limbs (ModDown) against the target primes of a level.
struct TcShape {
    int level, n, lo, cnt, ntar, ntar2;
    bool md, fused;
    __device__ TcShape(const DevCtx& ctx, int lev, bool is_md, bool is_fused, int d)
        : level(lev), n(lev + 1), lo(0), md(is_md), fused(is_md && is_fused) {
        if (md) {
            cnt = ctx.K;
            ntar = n;  // level targets (+ the top limb) or level + 1 targets
        } else {
            lo = d * ctx.alpha;
            cnt = min(lo + ctx.alpha - 1, level) - lo + 1;
            ntar = n - cnt + ctx.K;
        }
        ntar2 = (ntar + 1) & ~1;  // MMA widths are multiples of 16 columns
    }
    // prime of target m
    __device__ int tprime(const DevCtx& ctx, int m) const {
        if (md) return fused ? (m == 0 ? level : m - 1) : m;
        return target_prime(m, lo, cnt, n, ctx.L);
    }
    // conversion constant of input limb i for target m; ModDown with the fused
    // rescale converts P^-1 x directly, so its constants carry P^-1 mod q
    __device__ uint64_t matrix(const DevCtx& ctx, int i, int m) const {
        const int t = tprime(ctx, m);
        if (md) {
            const uint64_t M = ctx.md_mat[(size_t)i * ctx.L + t];
            if (!fused) return M;
            const ulonglong2 pinv = reinterpret_cast<const ulonglong2*>(ctx.md_pinv)[t];
            return mul_shoup(M, pinv.x, pinv.y, ctx.pc[t].p);
        }
        return ctx.modup_mat[((size_t)level * ctx.L + lo + i) * (ctx.L + ctx.K) + t];
    }
    __device__ uint32_t lbo_b() const { return (uint32_t)ntar2 * kTcCols / 8 * 128; }
};

// B of a conversion in its shared-memory layout: for K chunk c (limbs 2c,
// 2c+1) and target m, the 16 constants M'_{i,m,a} = M[i][m] 2^{8a} mod p_m;
// column 8m + s of the chunk holds their bytes s (16 bytes: a of limb 2c,
// then a of limb 2c+1), 2*CK chunks lbo_b bytes apart.
template <int CK>
__device__ void tc_build_b(const DevCtx& ctx, const TcShape& sh, uint8_t* dst) {
    const uint32_t lbo_b = sh.lbo_b();
    for (int u = threadIdx.x; u < 2 * CK * sh.ntar2; u += blockDim.x) {
        const int c = u / sh.ntar2, m = u % sh.ntar2;
        uint64_t mp[16];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int i = 2 * c + h;
            const bool live = i < sh.cnt && m < sh.ntar;
            const PrimeConst pc = ctx.pc[live ? sh.tprime(ctx, m) : 0];
            uint64_t v = live ? sh.matrix(ctx, i, m) : 0;
#pragma unroll
            for (int a = 0; a < 8; ++a) {
                mp[8 * h + a] = v;
                if (live && a < 7) v = reduce128(v >> 56, v << 8, pc);  // v 2^8 mod p
            }
        }
#pragma unroll
        for (int sb = 0; sb < kTcCols; ++sb) {
            uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
            for (int pos = 0; pos < 16; ++pos) w[pos >> 2] |= (uint32_t)((mp[pos] >> (8 * sb)) & 0xFF) << (8 * (pos & 3));
            const int nn = m * kTcCols + sb;
            *reinterpret_cast<uint4*>(dst + (size_t)c * lbo_b + (nn >> 3) * 128 + (nn & 7) * 16) =
                make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
}

// index of a conversion's B in the context table
__host__ __device__ inline int tc_table_index(int L, int dnum, bool md, int level, int d_or_fused) {
    return md ? L * dnum + 2 * level + d_or_fused : level * dnum + d_or_fused;
}

// One CTA per table entry of one kind (blockIdx.x = level, blockIdx.y =
// digit or fused flag); entries that do not exist at a level are skipped.
template <int CK, bool MD>
__global__ void __launch_bounds__(256) k_conv_tc_table(const __grid_constant__ DevCtx ctx, uint8_t* tab,
                                                      const uint64_t* __restrict__ offs) {
    const int level = blockIdx.x, y = blockIdx.y;
    if (!MD && y > level / ctx.alpha) return;
    const TcShape sh(ctx, level, MD, y != 0, y);
    tc_build_b<CK>(ctx, sh, tab + offs[tc_table_index(ctx.L, ctx.dnum, MD, level, y)]);
}

// One conversion launch: ModUp (blockIdx.y = element * digits + digit) or
// ModDown (blockIdx.y = 2 * element + half).
struct TcArgs {
    const uint64_t* xt;  // ModUp: scaled limbs of element 0
    uint64_t* dig;       // ModUp: digit outputs of element 0
    size_t dig_stride;   // ModUp: limbs per digit
    size_t bstride;      // ModUp: words between batch elements
    int nb;              // batch elements
    MdArgs md;           // ModDown
};

// CK: K = 32*CK bytes of A per row, up to 4*CK input limbs.  CHUNK: targets
// per MMA (N = 8*CHUNK), also the tensor-memory columns a CTA holds / 8 (32
// targets: 256 columns, two CTAs per SM; 16 targets: 128 columns, up to three).
// MD: the ModDown conversion, K special limbs -> the Q primes of the level,
// with the fused Rescale of the top limb when md.ttop is set:
//   tl = ttop - P^-1 conv_l (mod q_l),  w_q = P^-1 conv_q + SwitchModulus(tl).
template <int CK, int CHUNK, bool MD>
__global__ void __launch_bounds__(kTcThreads, CHUNK == 16 ? 3 : 2)
    k_conv_tc(const __grid_constant__ DevCtx ctx, int level, const __grid_constant__ TcArgs args) {
    extern __shared__ __align__(1024) uint8_t smem[];
    const int ntiles = ctx.N / kTcRows;
    // ModDown with the top limb (target 0 = prime `level`); both halves alike
    const bool fused = MD && args.md.ttop[0] != nullptr;
    const int d = MD ? 0 : blockIdx.y;
    const TcShape sh(ctx, level, MD, fused, d);
    const int lo = sh.lo, cnt = sh.cnt, ntar = sh.ntar, ntar2 = sh.ntar2;
    // work items: (element, tile) of digit d (ModUp) or (element, half, tile)
    // (ModDown), split evenly over the CTAs of the row
    const int nitems = (MD ? 2 : 1) * args.nb * ntiles;
    const int it_begin = (int)((long long)blockIdx.x * nitems / gridDim.x);
    const int it_end = (int)((long long)(blockIdx.x + 1) * nitems / gridDim.x);
    // element offset (words) and half of item `it`
    auto item_off = [&](int it, int& half) -> size_t {
        if (MD) {
            const int bh = it / ntiles;
            half = bh & 1;
            return (size_t)(bh >> 1) * args.md.bstride;
        }
        half = 0;
        return (size_t)(it / ntiles) * args.bstride;
    };
    auto item_in = [&](int it) -> const uint64_t* {
        int h;
        const size_t off = item_off(it, h) + (size_t)(it % ntiles) * kTcRows;
        return MD ? args.md.y[h] + off : args.xt + off + (size_t)lo * ctx.N;
    };
    const uint32_t lbo_b = sh.lbo_b();

    uint8_t* sA = smem;                                   // 2*CK chunks x kTcLboA
    uint8_t* sB = smem + 2 * CK * kTcLboA;                // 2*CK chunks x lbo_b
    PrimeConst* sP = reinterpret_cast<PrimeConst*>(sB + 2 * CK * lbo_b);
    uint64_t* sMu = reinterpret_cast<uint64_t*>(sP + ntar2);       // floor(2^80 / p) per target
    uint64_t* sOm = sMu + ntar2;                         // ModDown: q_level mod target
    uint64_t* sTL = sOm + (MD ? ntar2 : 0);               // ModDown: tl per row
    uint64_t* bar = sTL + (MD ? kTcRows : 0);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);

    for (int m = threadIdx.x; m < ntar; m += kTcThreads) {
        const PrimeConst pc = ctx.pc[sh.tprime(ctx, m)];
        sP[m] = pc;
        sMu[m] = (uint64_t)(((unsigned __int128)1 << 80) / pc.p);
        if (MD) sOm[m] = csub(reduce64_lazy(ctx.pc[level].p, pc), pc.p);
    }
    // A: zero once (limbs cnt..4*CK-1 stay zero)
    for (int i = threadIdx.x; i < 2 * CK * (int)kTcLboA / 16; i += kTcThreads)
        reinterpret_cast<uint4*>(sA)[i] = make_uint4(0, 0, 0, 0);
    // B from the context's table (built once per level and digit)
    {
        const uint4* src = reinterpret_cast<const uint4*>(
            ctx.tc_btab + ctx.tc_boff[tc_table_index(ctx.L, ctx.dnum, MD, level, MD ? (fused ? 1 : 0) : d)]);
        for (int i = threadIdx.x; i < 2 * CK * (int)lbo_b / 16; i += kTcThreads)
            reinterpret_cast<uint4*>(sB)[i] = __ldg(src + i);
    }

    const uint32_t bar_a = smem_u32(bar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar_a), "r"(1u));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    constexpr uint32_t kTcTmemCols = CHUNK * kTcCols;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tslot)),
                     "r"(kTcTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tslot;

    const int quarter = warp & 3, wh = warp >> 2;
    const int row = quarter * 32 + lane;
    const uint32_t t_lane = tmem + ((uint32_t)(quarter * 32) << 16);
    const uint32_t a_base = smem_u32(sA), b_base = smem_u32(sB);
    uint32_t phase = 0;
    bool ok = true;
    // this thread's share of an A tile: element e = threadIdx.x + q * kTcThreads
    // is limb e / kTcRows, row e % kTcRows (at most 2*CK elements)
    constexpr int kPer = 2 * CK;
    uint64_t pre[kPer];
    auto fetch = [&](int it) {
        const uint64_t* src = item_in(it);
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            const int e = threadIdx.x + q * kTcThreads;
            if (e < cnt * kTcRows) pre[q] = src[(size_t)(e / kTcRows) * ctx.N + e % kTcRows];
        }
    };
    auto value = [&](const uint32_t* c, int m) { return reduce_cols(c, sMu[m], sP[m].p); };
    if (it_begin < it_end) fetch(it_begin);
    for (int it = it_begin; it < it_end && ok; ++it) {
        int half;
        const size_t boff = item_off(it, half);
        const size_t j = (size_t)(it % ntiles) * kTcRows + row;  // this thread's coefficient
        // output of target m for this thread's row (v = conversion value mod p_m)
        auto finish = [&](int m, uint64_t v) {
            if (MD) {
                if (fused) {
                    // v = P^-1 conv_q (folded into the constants)
                    // SwitchModulus(tl, q_l -> q) with q_l mod q precomputed
                    const PrimeConst pc = sP[m];
                    const uint64_t tl = sTL[row], ql = sP[0].p;
                    uint64_t sw = tl > (ql >> 1) ? tl + (pc.p - sOm[m]) : tl;
                    if (pc.p < ql) sw = csub(reduce64_lazy(sw, pc), pc.p);
                    args.md.w[half][boff + (size_t)(m - 1) * ctx.N + j] = add_mod(v, sw, pc.p);
                } else {
                    args.md.w[half][boff + (size_t)m * ctx.N + j] = v;
                }
            } else {
                args.dig[boff + ((size_t)d * args.dig_stride + m) * ctx.N + j] = v;
            }
        };
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            const int e = threadIdx.x + q * kTcThreads;
            if (e < cnt * kTcRows) {
                const int i = e / kTcRows, r = e % kTcRows;
                *reinterpret_cast<uint64_t*>(sA + (i >> 1) * kTcLboA + (r >> 3) * 128 + (r & 7) * 16 + (i & 1) * 8) =
                    pre[q];
            }
        }
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        for (int m0 = 0; m0 < ntar2 && ok; m0 += CHUNK) {
            const int nt = min(CHUNK, ntar2 - m0);  // even
            // the A tile is written and the previous chunk's accumulators are read
            asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
            __syncthreads();
            if (threadIdx.x == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint32_t idesc = idesc_u8(kTcRows, nt * kTcCols);
#pragma unroll
                for (int k = 0; k < CK; ++k) {
                    const uint64_t ad = smem_desc(a_base + 2 * k * kTcLboA, kTcLboA, 128);
                    const uint64_t bd = smem_desc(b_base + 2 * k * lbo_b + m0 * (kTcCols / 8) * 128, lbo_b, 128);
                    mma_u8(tmem, ad, bd, idesc, k > 0 ? 1u : 0u);
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                                 bar_a)
                             : "memory");
            }
            const bool got = wait_parity(bar_a, phase);
            phase ^= 1;
            ok = __syncthreads_and(got) != 0;
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            // the next item's limbs load while this chunk's outputs are formed
            if (m0 + CHUNK >= ntar2 && it + 1 < it_end) fetch(it + 1);
            // target pairs (2p, 2p+1) share one 16-column load; warps of half
            // wh take pairs wh, wh+2, ... two at a time
            int first = wh;
            if (MD && fused && m0 == 0) {
                // pair 0 holds the top limb: every row's tl first, shared through smem
                uint32_t c[16];
                uint64_t v1 = 0;
                if (wh == 0) {
                    tmem_ld16(t_lane, c);
                    tmem_wait_ld();
                    const uint64_t ql = sP[0].p;
                    sTL[row] = sub_mod(args.md.ttop[half][boff + j], value(c, 0), ql);  // ttop - P^-1 conv_l
                    if (ntar > 1) v1 = value(c + 8, 1);
                }
                __syncthreads();
                if (wh == 0) {
                    if (ntar > 1) finish(1, v1);
                    first = 2;
                }
            }
            for (int pp = first; 2 * pp < nt; pp += 4) {
                const bool two = 2 * (pp + 2) < nt;
                uint32_t c0[16], c1[16];
                tmem_ld16(t_lane + (uint32_t)(2 * pp * kTcCols), c0);
                if (two) tmem_ld16(t_lane + (uint32_t)(2 * (pp + 2) * kTcCols), c1);
                tmem_wait_ld();
                const int m = m0 + 2 * pp;
                finish(m, value(c0, m));
                if (m + 1 < ntar) finish(m + 1, value(c0 + 8, m + 1));
                if (two) {
                    const int m2 = m + 4;
                    finish(m2, value(c1, m2));
                    if (m2 + 1 < ntar) finish(m2 + 1, value(c1 + 8, m2 + 1));
                }
            }
        }
    }
    // a gave-up wait invalidates this launch's outputs: flagged in the
    // context's error word, which the next synchronising call reports
    if (!ok && threadIdx.x == 0 && ctx.err) atomicOr(ctx.err, kDevErrTensorWait);
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTcTmemCols));
    }
}

// dynamic shared memory of one CTA for ntar targets
size_t tc_smem_bytes(int ck, int ntar, bool md) {
    const size_t t2 = (size_t)((ntar + 1) & ~1);
    return (size_t)2 * ck * kTcLboA + (size_t)2 * ck * t2 * kTcCols / 8 * 128 + t2 * (sizeof(PrimeConst) + 8) +
           (md ? t2 * 8 + (size_t)kTcRows * 8 : 0) + 16;
}

constexpr int kTcMaxTargets = 48;
constexpr size_t kTcSmemCap = 160 * 1024;

template <int CK, int CHUNK, bool MD>
void set_smem_attr() {
    static std::once_flag once;
    std::call_once(once, [] {
        cudaFuncSetAttribute(k_conv_tc<CK, CHUNK, MD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmemCap);
    });
}

template <int CHUNK, bool MD>
void launch_ck(int ck, dim3 g, size_t smem, const DevCtx& ctx, int level, const TcArgs& a, cudaStream_t st) {
    switch (ck) {
        case 1:
            set_smem_attr<1, CHUNK, MD>();
            k_conv_tc<1, CHUNK, MD><<<g, kTcThreads, smem, st>>>(ctx, level, a);
            break;
        case 2:
            set_smem_attr<2, CHUNK, MD>();
            k_conv_tc<2, CHUNK, MD><<<g, kTcThreads, smem, st>>>(ctx, level, a);
            break;
        case 3:
            set_smem_attr<3, CHUNK, MD>();
            k_conv_tc<3, CHUNK, MD><<<g, kTcThreads, smem, st>>>(ctx, level, a);
            break;
        default:
            set_smem_attr<4, CHUNK, MD>();
            k_conv_tc<4, CHUNK, MD><<<g, kTcThreads, smem, st>>>(ctx, level, a);
            break;
    }
}

// grid, shared memory and launch; a floor on the shared memory keeps the
// CTAs of an SM within its 512 tensor-memory columns (80 KB: at most two
// CTAs of 256 columns; 58 KB: at most three of 128)
template <bool MD>
void launch_tc(const DevCtx& ctx, int level, int groups, int items, int ck, int ntar, const TcArgs& a,
               cudaStream_t st, int chunk) {
    const size_t floor_bytes = chunk == 32 ? (size_t)80 * 1024 : (size_t)58 * 1024;
    const size_t smem = std::max(tc_smem_bytes(ck, ntar, MD), floor_bytes);
    // one wave: the CTAs of all rows fill the SMs at the occupancy above
    const int ctas = chunk == 32 ? 2 * 148 : 3 * 148;
    const dim3 g(std::max(1, std::min(items, ctas / groups)), groups);
    count_launches(1);
    if (chunk == 32)
        launch_ck<32, MD>(ck, g, smem, ctx, level, a, st);
    else
        launch_ck<16, MD>(ck, g, smem, ctx, level, a, st);
}

}  // namespace

bool conv_tc_eligible(const DevCtx& ctx) {
    if (ctx.alpha > 16 || ctx.K > 16) return false;
    const int up = ctx.L - 1 + ctx.K;  // ModUp: at most L-1 other Q primes plus K
    return up <= kTcMaxTargets && ctx.L <= kTcMaxTargets &&
           tc_smem_bytes((ctx.alpha + 3) / 4, up, false) <= kTcSmemCap &&
           tc_smem_bytes((ctx.K + 3) / 4, ctx.L, true) <= kTcSmemCap;
}

bool conv_tc_supported(const DevCtx& ctx) { return ctx.tc_btab != nullptr && conv_tc_eligible(ctx); }

size_t conv_tc_table_layout(const DevCtx& ctx, std::vector<uint64_t>& offs) {
    const int L = ctx.L, K = ctx.K, dn = ctx.dnum;
    offs.assign((size_t)L * dn + 2 * L, 0);
    size_t off = 0;
    auto add = [&](int idx, int ck, int ntar) {
        offs[idx] = off;
        off += (size_t)2 * ck * (size_t)((ntar + 1) & ~1) * kTcCols / 8 * 128;
    };
    for (int level = 0; level < L; ++level) {
        const int n = level + 1;
        for (int d = 0; d <= level / ctx.alpha && d < dn; ++d) {
            const int lo = d * ctx.alpha, cnt = std::min(lo + ctx.alpha - 1, level) - lo + 1;
            add(tc_table_index(L, dn, false, level, d), (ctx.alpha + 3) / 4, n - cnt + K);
        }
        for (int f = 0; f < 2; ++f) add(tc_table_index(L, dn, true, level, f), (K + 3) / 4, n);
    }
    return off;
}

void conv_tc_build_tables(const DevCtx& ctx, cudaStream_t st) {
    const dim3 gu(ctx.L, ctx.dnum), gd(ctx.L, 2);
    uint8_t* tab = const_cast<uint8_t*>(ctx.tc_btab);
    switch ((ctx.alpha + 3) / 4) {
        case 1: k_conv_tc_table<1, false><<<gu, 256, 0, st>>>(ctx, tab, ctx.tc_boff); break;
        case 2: k_conv_tc_table<2, false><<<gu, 256, 0, st>>>(ctx, tab, ctx.tc_boff); break;
        case 3: k_conv_tc_table<3, false><<<gu, 256, 0, st>>>(ctx, tab, ctx.tc_boff); break;
        default: k_conv_tc_table<4, false><<<gu, 256, 0, st>>>(ctx, tab, ctx.tc_boff); break;
    }
    switch ((ctx.K + 3) / 4) {
        case 1: k_conv_tc_table<1, true><<<gd, 256, 0, st>>>(ctx, tab, ctx.tc_boff); break;
        case 2: k_conv_tc_table<2, true><<<gd, 256, 0, st>>>(ctx, tab, ctx.tc_boff); break;
        case 3: k_conv_tc_table<3, true><<<gd, 256, 0, st>>>(ctx, tab, ctx.tc_boff); break;
        default: k_conv_tc_table<4, true><<<gd, 256, 0, st>>>(ctx, tab, ctx.tc_boff); break;
    }
    count_launches(2);
}

void launch_modup_conv_tc(const DevCtx& ctx, int level, int nb, const uint64_t* xt, uint64_t* dig, size_t dig_stride,
                          size_t bstride, cudaStream_t st, int chunk) {
    const int nd = level / ctx.alpha + 1;
    const int n = level + 1, last = n - (nd - 1) * ctx.alpha;
    const int ntar = n - std::min(last, ctx.alpha) + ctx.K;  // largest over the digits
    TcArgs a{};
    a.xt = xt;
    a.dig = dig;
    a.dig_stride = dig_stride;
    a.bstride = bstride;
    a.nb = nb;
    launch_tc<false>(ctx, level, nd, nb * (ctx.N / kTcRows), (ctx.alpha + 3) / 4, ntar, a, st, chunk);
}

void launch_moddown_conv_tc(const DevCtx& ctx, int level, int nb, const MdArgs& md, cudaStream_t st, int chunk) {
    TcArgs a{};
    a.md = md;
    a.nb = nb;
    launch_tc<true>(ctx, level, 1, 2 * nb * (ctx.N / kTcRows), (ctx.K + 3) / 4, level + 1, a, st, chunk);
}

}  // namespace fides
