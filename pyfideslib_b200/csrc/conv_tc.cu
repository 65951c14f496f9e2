// conv_tc.cu -- ModUp base conversion on the 5th-generation tensor cores.
//
// Role in the reference: DecompAndModUpConv (src/CKKS/Conv.cu), the same
// contraction as k_modup_conv in ks.cu:
//   out[m][j] = sum_i x_i[j] * M[i][m]  (mod p_m),  M[i][m] = (Q'/q_i) mod p_m,
// over the cnt limbs i of one digit and the ntar target primes m.
//
// Exact int8 split (this file's own design): with x_i = sum_a x_{i,a} 2^{8a}
// and M[i][m] = sum_b M_{i,m,b} 2^{8b} (bytes), the value before reduction is
//   V[j][m] = sum_s c_s 2^{8s},  c_s = sum_i sum_{a+b=s} x_{i,a} M_{i,m,b},
// and every c_s (s = 0..14) is one entry of an unsigned 8-bit matrix product
//   A[j][(i,a)] = x_{i,a},   B[(i,a)][(m,s)] = M_{i,m,s-a} (0 outside 0..7),
// accumulated exactly in 32 bits (at most 8 products per limb, each below
// 2^16, for at most 16 limbs).
// A tile of 128 coefficients is multiplied by B with tcgen05.mma kind::i8
// (M = 128, N = 16 columns per target, K = 32 bytes per instruction) into
// tensor memory; the epilogue reads each coefficient's 16 column sums with
// tcgen05.ld, recombines them into the 128-bit V and reduces it mod p_m.  The
// tensor cores take the 64x64-bit products off the integer pipes; what is
// left there is one recombination and one 128-bit reduction per output.
//
// Operands sit in shared memory in the canonical K-major layout without
// swizzle: core matrices of 8 rows x 16 bytes stored contiguously, 8-row
// groups 128 bytes apart (SBO) and 16-byte K chunks LBO bytes apart.  A is
// rebuilt per tile from coalesced limb loads; B is built once per CTA.  Every
// wait on the MMA completion barrier is bounded; a timeout sets an error flag
// and the CTA releases its tensor memory and returns.
#include <algorithm>
#include <mutex>

#include "kernels.hpp"

namespace fides {

namespace {

constexpr int kTcThreads = 256;     // 8 warps: two per tensor-memory lane quarter
constexpr int kTcRows = 128;        // coefficients per tile (MMA M)
constexpr int kTcCols = 16;         // accumulator columns per target (15 byte shifts, 1 zero)
constexpr uint32_t kTcLboA = (kTcRows / 8) * 128;  // A: K-chunk stride in bytes
constexpr uint32_t kSpinLimit = 1u << 20;

__device__ int g_tc_error;

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

__device__ __forceinline__ uint64_t mad_wide(uint32_t a, uint32_t b, uint64_t c) {
    uint64_t d;
    asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(d) : "r"(a), "r"(b), "l"(c));
    return d;
}

// V = sum_s c_s 2^{8s} as (hi, lo).  Every c_s < 2^23, so the four groups
// g_k = c_{4k} + c_{4k+1} 2^8 + c_{4k+2} 2^16 + c_{4k+3} 2^24 are below 2^48
// and V = g_0 + g_1 2^32 + g_2 2^64 + g_3 2^96 is assembled word by word.
// V < 2^128 (at most 16 products of values below 2^62), so the high word of
// g_3 and the last carry are zero.
__device__ __forceinline__ void recombine(const uint32_t (&c)[16], uint64_t& hi, uint64_t& lo) {
    uint64_t g[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t t = c[4 * k] + (c[4 * k + 1] << 8);  // < 2^32
        g[k] = mad_wide(c[4 * k + 3], 1u << 24, mad_wide(c[4 * k + 2], 1u << 16, (uint64_t)t));
    }
    uint32_t w1, w2, w3;
    asm("add.cc.u32 %0, %3, %4;\n\t"
        "addc.cc.u32 %1, %5, %6;\n\t"
        "addc.u32 %2, %7, %8;"
        : "=r"(w1), "=r"(w2), "=r"(w3)
        : "r"((uint32_t)(g[0] >> 32)), "r"((uint32_t)g[1]), "r"((uint32_t)(g[1] >> 32)), "r"((uint32_t)g[2]),
          "r"((uint32_t)(g[2] >> 32)), "r"((uint32_t)g[3]));
    lo = ((uint64_t)w1 << 32) | (uint32_t)g[0];
    hi = ((uint64_t)w3 << 32) | w2;
}

// target index m of a digit -> prime id (the other Q primes, then the special ones)
__device__ __forceinline__ int target_prime(int m, int lo, int cnt, int n, int L) {
    const int jj = m < lo ? m : m + cnt;
    return jj < n ? jj : L + (jj - n);
}

// One conversion launch: ModUp (blockIdx.y = element * digits + digit) or
// ModDown (blockIdx.y = 2 * element + half).
struct TcArgs {
    const uint64_t* xt;  // ModUp: scaled limbs of element 0
    uint64_t* dig;       // ModUp: digit outputs of element 0
    size_t dig_stride;   // ModUp: limbs per digit
    size_t bstride;      // words between batch elements
    MdArgs md;           // ModDown
};

// CK: K = 32*CK bytes of A per row, up to 4*CK input limbs.  CHUNK: targets
// per MMA (N = 16*CHUNK), also the tensor-memory columns a CTA holds / 16
// (16 targets: two CTAs per SM, 8 targets: up to three; registers bounded to match).  MD: the ModDown
// conversion, K special limbs -> the Q primes of the level, with the fused
// Rescale of the top limb when md.ttop is set:
//   tl = ttop - P^-1 conv_l (mod q_l),  w_q = P^-1 conv_q + SwitchModulus(tl).
template <int CK, int CHUNK, bool MD>
__global__ void __launch_bounds__(kTcThreads, CHUNK == 8 ? 3 : 2)
    k_conv_tc(const __grid_constant__ DevCtx ctx, int level, const __grid_constant__ TcArgs args) {
    extern __shared__ __align__(1024) uint8_t smem[];
    const int n = level + 1;
    const uint64_t* in;   // input limb i at in + i * N
    int lo = 0, cnt, ntar, d = 0, half = 0;
    size_t boff;
    bool fused = false;   // ModDown with the top limb (target 0 = prime `level`)
    if (MD) {
        half = blockIdx.y & 1;
        boff = (size_t)(blockIdx.y >> 1) * args.md.bstride;
        in = args.md.y[half] + boff;
        cnt = ctx.K;
        fused = args.md.ttop[half] != nullptr;
        ntar = n;  // level targets (+ the top limb) or level + 1 targets
    } else {
        const int ndig = level / ctx.alpha + 1;
        d = blockIdx.y % ndig;
        boff = (size_t)(blockIdx.y / ndig) * args.bstride;
        lo = d * ctx.alpha;
        cnt = min(lo + ctx.alpha - 1, level) - lo + 1;
        ntar = n - cnt + ctx.K;
        in = args.xt + boff + (size_t)lo * ctx.N;
    }
    // prime and matrix column of target m
    auto tprime = [&](int m) {
        if (MD) return fused ? (m == 0 ? level : m - 1) : m;
        return target_prime(m, lo, cnt, n, ctx.L);
    };
    const int NP = ctx.L + ctx.K;
    auto matrix = [&](int i, int m) -> uint64_t {
        if (MD) return ctx.md_mat[(size_t)i * ctx.L + tprime(m)];
        return ctx.modup_mat[((size_t)level * ctx.L + lo + i) * NP + tprime(m)];
    };
    const uint32_t lbo_b = (uint32_t)ntar * kTcCols / 8 * 128;

    uint8_t* sA = smem;                                   // 2*CK chunks x kTcLboA
    uint8_t* sB = smem + 2 * CK * kTcLboA;                // 2*CK chunks x lbo_b
    PrimeConst* sP = reinterpret_cast<PrimeConst*>(sB + 2 * CK * lbo_b);
    ulonglong2* sPinv = reinterpret_cast<ulonglong2*>(sP + ntar);  // ModDown: P^-1 mod target
    uint64_t* sTL = reinterpret_cast<uint64_t*>(sPinv + (MD ? ntar : 0));  // ModDown: tl per row
    uint64_t* bar = sTL + (MD ? kTcRows : 0);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);

    // A: zero once (limbs cnt..4*CK-1 stay zero)
    for (int i = threadIdx.x; i < 2 * CK * (int)kTcLboA / 16; i += kTcThreads)
        reinterpret_cast<uint4*>(sA)[i] = make_uint4(0, 0, 0, 0);
    // B: 16-byte unit (chunk c, column nn = 16 m + s) holds K bytes 16c..16c+15,
    // i.e. bytes a of limbs 2c and 2c+1 against byte s-a of M[i][m]
    const int ncol = ntar * kTcCols;
    for (int u = threadIdx.x; u < 2 * CK * ncol; u += kTcThreads) {
        const int c = u / ncol, nn = u % ncol;
        const int m = nn / kTcCols, s = nn % kTcCols;
        uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int i = 2 * c + h;
            if (i >= cnt || s > 14) continue;
            const uint64_t M = matrix(i, m);
#pragma unroll
            for (int a = 0; a < 8; ++a) {
                const int b = s - a;
                if (b < 0 || b > 7) continue;
                const int pos = 8 * h + a;
                w[pos >> 2] |= (uint32_t)((M >> (8 * b)) & 0xFF) << (8 * (pos & 3));
            }
        }
        *reinterpret_cast<uint4*>(sB + (size_t)c * lbo_b + (nn >> 3) * 128 + (nn & 7) * 16) =
            make_uint4(w[0], w[1], w[2], w[3]);
    }
    for (int m = threadIdx.x; m < ntar; m += kTcThreads) {
        sP[m] = ctx.pc[tprime(m)];
        if (MD) sPinv[m] = reinterpret_cast<const ulonglong2*>(ctx.md_pinv)[tprime(m)];
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
    const int ntiles = ctx.N / kTcRows;
    // this thread's share of an A tile: element e = threadIdx.x + q * kTcThreads
    // is limb e / kTcRows, row e % kTcRows (at most 2*CK elements)
    constexpr int kPer = 2 * CK;
    uint64_t pre[kPer];
    auto fetch = [&](int tile) {
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            const int e = threadIdx.x + q * kTcThreads;
            if (e < cnt * kTcRows) pre[q] = in[(size_t)(e / kTcRows) * ctx.N + (size_t)tile * kTcRows + e % kTcRows];
        }
    };
    // output of target m for this thread's row (v = conversion value mod p_m)
    auto finish = [&](int m, uint64_t v, size_t j) {
        if (MD) {
            if (fused) {
                const PrimeConst pc = sP[m];
                const ulonglong2 pinv = sPinv[m];
                v = add_mod(mul_shoup(v, pinv.x, pinv.y, pc.p), switch_modulus(sTL[row], sP[0].p, pc), pc.p);
                args.md.w[half][boff + (size_t)(m - 1) * ctx.N + j] = v;
            } else {
                args.md.w[half][boff + (size_t)m * ctx.N + j] = v;
            }
        } else {
            args.dig[boff + ((size_t)d * args.dig_stride + m) * ctx.N + j] = v;
        }
    };
    if (blockIdx.x < ntiles) fetch(blockIdx.x);
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const size_t j0 = (size_t)tile * kTcRows;
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
        for (int m0 = 0; m0 < ntar && ok; m0 += CHUNK) {
            const int nt = min(CHUNK, ntar - m0);
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
            // the next tile's limbs load while this chunk's outputs are formed
            if (m0 + CHUNK >= ntar && tile + (int)gridDim.x < ntiles) fetch(tile + gridDim.x);
            int first = wh;
            if (MD && fused && m0 == 0) {
                // the top limb's value first: every row's tl, shared through smem
                if (wh == 0) {
                    uint32_t c[16];
                    tmem_ld16(t_lane, c);
                    tmem_wait_ld();
                    uint64_t vh, vl;
                    recombine(c, vh, vl);
                    const PrimeConst pl = sP[0];
                    const ulonglong2 pinv = sPinv[0];
                    const uint64_t conv = reduce128(vh, vl, pl);
                    sTL[row] = sub_mod(args.md.ttop[half][boff + j0 + row], mul_shoup(conv, pinv.x, pinv.y, pl.p), pl.p);
                }
                __syncthreads();
                if (wh == 0) first = 2;
            }
            // two targets per step (warp-uniform), one wait for both loads
            for (int mm = first; mm < nt; mm += 4) {
                const bool two = mm + 2 < nt;
                uint32_t c0[16], c1[16];
                tmem_ld16(t_lane + (uint32_t)(mm * kTcCols), c0);
                if (two) tmem_ld16(t_lane + (uint32_t)((mm + 2) * kTcCols), c1);
                tmem_wait_ld();
                uint64_t vh, vl;
                recombine(c0, vh, vl);
                finish(m0 + mm, reduce128(vh, vl, sP[m0 + mm]), j0 + row);
                if (two) {
                    recombine(c1, vh, vl);
                    finish(m0 + mm + 2, reduce128(vh, vl, sP[m0 + mm + 2]), j0 + row);
                }
            }
        }
    }
    if (!ok && threadIdx.x == 0) atomicExch(&g_tc_error, 1);
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTcTmemCols));
    }
}

// dynamic shared memory of one CTA for ntar targets
size_t tc_smem_bytes(int ck, int ntar, bool md) {
    return (size_t)2 * ck * kTcLboA + (size_t)2 * ck * ntar * kTcCols / 8 * 128 + (size_t)ntar * sizeof(PrimeConst) +
           (md ? (size_t)ntar * 16 + (size_t)kTcRows * 8 : 0) + 16;
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
void launch_tc(const DevCtx& ctx, int level, int groups, int ck, int ntar, const TcArgs& a, cudaStream_t st,
               int chunk) {
    const size_t floor_bytes = chunk == 16 ? (size_t)80 * 1024 : (size_t)58 * 1024;
    const size_t smem = std::max(tc_smem_bytes(ck, ntar, MD), floor_bytes);
    const int ctas = chunk == 16 ? 2 * 148 : 3 * 148;
    const int per = std::max(1, std::min(ctx.N / kTcRows, ctas / std::max(1, groups)));
    const dim3 g(per, groups);
    count_launches(1);
    if (chunk == 16)
        launch_ck<16, MD>(ck, g, smem, ctx, level, a, st);
    else
        launch_ck<8, MD>(ck, g, smem, ctx, level, a, st);
}

}  // namespace

bool conv_tc_supported(const DevCtx& ctx) {
    if (ctx.alpha > 16 || ctx.K > 16) return false;
    const int up = ctx.L - 1 + ctx.K;  // ModUp: at most L-1 other Q primes plus K
    return up <= kTcMaxTargets && ctx.L <= kTcMaxTargets &&
           tc_smem_bytes((ctx.alpha + 3) / 4, up, false) <= kTcSmemCap &&
           tc_smem_bytes((ctx.K + 3) / 4, ctx.L, true) <= kTcSmemCap;
}

int conv_tc_error() {
    int e = 0;
    cudaMemcpyFromSymbol(&e, g_tc_error, sizeof(int));
    return e;
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
    launch_tc<false>(ctx, level, nd * nb, (ctx.alpha + 3) / 4, ntar, a, st, chunk);
}

void launch_moddown_conv_tc(const DevCtx& ctx, int level, int nb, const MdArgs& md, cudaStream_t st, int chunk) {
    TcArgs a{};
    a.md = md;
    launch_tc<true>(ctx, level, 2 * nb, (ctx.K + 3) / 4, level + 1, a, st, chunk);
}

}  // namespace fides
