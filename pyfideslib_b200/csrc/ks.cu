// ks.cu -- tensor product, ModUp / ModDown base conversions, the hybrid
// key-switch inner product and the element-wise kernels, for sm_100a.
//
// Role in the reference: src/CKKS/Conv.cu (DecompAndModUpConv, ModDown2),
// src/CKKS/ElemenwiseBatchKernels.cu (binomialMult_, fusedDotKSK_2_,
// hoistedRotateDotKSK_2_, element-wise ops) and src/Rotation.cu
// (automorph_multi_).  Same arithmetic (exact 128-bit accumulation of the
// base-conversion sums with one reduction per output), own kernels:
//   * one thread per coefficient; the inputs of a conversion are staged once
//     in shared memory and every output limb of the digit is produced from
//     them, so each input limb is read from HBM once per digit;
//   * the inner product reads each key limb once and accumulates both key
//     halves in 128-bit registers, reducing once per output;
//   * rotations fold the automorphism into the inner product as a gather of
//     the digit values; Galois keys are held permuted to the output order, so
//     key loads and stores stay coalesced and vectorised.
#include "fp64.cuh"
#include "kernels.hpp"

namespace fides {

__device__ __forceinline__ uint32_t brev_bits(uint32_t x, int bits) { return __brev(x) >> (32 - bits); }

// src/Rotation.cuh:14-26 automorph_slot: slot of the image of slot j.
__device__ __forceinline__ uint32_t automorph_slot(int logN, uint32_t k, uint32_t j) {
    const uint32_t e = (brev_bits(j, logN) << 1) + 1;
    const uint32_t r = ((e * k) & ((2u << logN) - 1)) >> 1;
    return brev_bits(r, logN);
}

// ---------------------------------------------------------------------------
// tensor product (binomialMult_): e0 = a0 b0, e1 = a0 b1 + a1 b0, e2 = a1 b1,
// for every batch element (blockIdx.z)
// ---------------------------------------------------------------------------
__global__ void k_tensor(const __grid_constant__ DevCtx ctx, const __grid_constant__ TensorArgs args) {
    const int limb = blockIdx.y, bi = blockIdx.z;
    const PrimeConst pc = ctx.pc[limb];
    const size_t i = ((size_t)limb * ctx.N + (size_t)(blockIdx.x * blockDim.x + threadIdx.x) * 2);
    const size_t o = i + (size_t)bi * args.bstride;
    const ulonglong2 x0 = *reinterpret_cast<const ulonglong2*>(args.a0[bi] + i);
    const ulonglong2 x1 = *reinterpret_cast<const ulonglong2*>(args.a1[bi] + i);
    const ulonglong2 y0 = *reinterpret_cast<const ulonglong2*>(args.b0[bi] + i);
    const ulonglong2 y1 = *reinterpret_cast<const ulonglong2*>(args.b1[bi] + i);
    ulonglong2 r0, r1, r2;
    if (pc.p < kFpPrimeBound) {
        // all three on the FP64 pipes (fp64.cuh: each product reduced to
        // |r| <= 0.875p, e1's sum of two below 1.75p, then the floor
        // reduction, exact for (-2p, 2p)): with 128-bit integer products the
        // IMAD pipe, not HBM, bounds this kernel
        const double p = __ull2double_rn(pc.p), pinv = as_f64(pc.pinv_f64);
        auto fmul = [&](uint64_t a, uint64_t b) {
            return fp_to_u(fp_mulmod(as_f64(fp_from_u(a)), as_f64(fp_from_u(b)), p, pinv), p, pinv);
        };
        r0.x = fmul(x0.x, y0.x);
        r0.y = fmul(x0.y, y0.y);
        r2.x = fmul(x1.x, y1.x);
        r2.y = fmul(x1.y, y1.y);
        auto fsum = [&](uint64_t a, uint64_t b, uint64_t c, uint64_t d) {
            const double s = __dadd_rn(fp_mulmod(as_f64(fp_from_u(a)), as_f64(fp_from_u(b)), p, pinv),
                                       fp_mulmod(as_f64(fp_from_u(c)), as_f64(fp_from_u(d)), p, pinv));
            return fp_to_u(s, p, pinv);
        };
        r1.x = fsum(x0.x, y1.x, x1.x, y0.x);
        r1.y = fsum(x0.y, y1.y, x1.y, y0.y);
    } else {
        r0.x = mul_mod(x0.x, y0.x, pc);
        r0.y = mul_mod(x0.y, y0.y, pc);
        r2.x = mul_mod(x1.x, y1.x, pc);
        r2.y = mul_mod(x1.y, y1.y, pc);
        Acc128 s;
        s.mac(x0.x, y1.x);
        s.mac(x1.x, y0.x);
        r1.x = s.reduce(pc);
        Acc128 t;
        t.mac(x0.y, y1.y);
        t.mac(x1.y, y0.y);
        r1.y = t.reduce(pc);
    }
    *reinterpret_cast<ulonglong2*>(args.e0 + o) = r0;
    *reinterpret_cast<ulonglong2*>(args.e1 + o) = r1;
    *reinterpret_cast<ulonglong2*>(args.e2 + o) = r2;
}

void launch_tensor(const DevCtx& ctx, int n, int nb, const TensorArgs& args, cudaStream_t st) {
    dim3 g(ctx.N / 256, n, nb);
    count_launches(1);
    k_tensor<<<g, 128, 0, st>>>(ctx, args);
}

// ---------------------------------------------------------------------------
// ModUp base conversion (DecompAndModUpConv): for digit d at `level`, with
// inputs xt_i = [x_i * (Q'/q_i)^-1]_{q_i} (produced by the scaled INTT), every
// target prime t outside the digit gets  sum_i xt_i * [Q'/q_i]_t  mod t.
// Digit d's targets are stored at dig + (d*dig_stride + m)*N, m = target index
// (Q primes below the digit, Q primes above it up to `level`, then P).
//
// Each thread owns two adjacent coefficients and keeps the digit's inputs in
// registers; the block stages its slice of the conversion matrix and the
// target constants in shared memory.  Sums of up to 16 products of residues
// below 2^62 stay below 2^128, so one reduction per output suffices.
// ---------------------------------------------------------------------------
constexpr int kConvThreads = 128;
constexpr int kConvTargets = 32;  // targets per block
constexpr int kMaxConvIn = 16;    // digit size / special count handled in registers

template <class ACC>
__device__ __forceinline__ void conv_store(uint64_t* out, const ACC& a, const ACC& b, const PrimeConst& pc) {
    ulonglong2 o;
    o.x = a.reduce(pc);
    o.y = b.reduce(pc);
    *reinterpret_cast<ulonglong2*>(out) = o;
}

// MAXIN: the register arrays and unrolled loops cover MAXIN inputs (the digit
// size rounded up to a multiple of 4), so no issue slot goes to inputs that
// do not exist.  ACC: Acc128, or AccSplit when every modulus is below 2^60;
// the autotuner picks per context (identical sums).
template <int MAXIN, class ACC>
__global__ void __launch_bounds__(kConvThreads) k_modup_conv(const __grid_constant__ DevCtx ctx, int level,
                                                             const uint64_t* __restrict__ xt,
                                                             uint64_t* __restrict__ dig, size_t dig_stride,
                                                             size_t bstride) {
    __shared__ uint64_t sM[MAXIN][kConvTargets];
    __shared__ PrimeConst sP[kConvTargets];
    const int ndig = level / ctx.alpha + 1;
    const int d = blockIdx.y % ndig;
    const size_t boff = (size_t)(blockIdx.y / ndig) * bstride;
    xt += boff;
    dig += boff;
    const int n = level + 1;
    const int lo = d * ctx.alpha;
    const int hi = min(lo + ctx.alpha - 1, level);
    const int cnt = hi - lo + 1;
    const int ntar = n - cnt + ctx.K;
    const int m0 = blockIdx.z * kConvTargets;
    if (m0 >= ntar) return;
    const int nt = min(kConvTargets, ntar - m0);
    const int NP = ctx.L + ctx.K;
    const uint64_t* mat = ctx.modup_mat + (size_t)level * ctx.L * NP;
    for (int e = threadIdx.x; e < cnt * nt; e += kConvThreads) {
        const int i = e / nt, mm = e % nt, m = m0 + mm;
        const int jj = m < lo ? m : m + cnt;
        const int t = jj < n ? jj : ctx.L + (jj - n);
        sM[i][mm] = mat[(size_t)(lo + i) * NP + t];
        if (i == 0) sP[mm] = ctx.pc[t];
    }
    const size_t j = ((size_t)blockIdx.x * kConvThreads + threadIdx.x) * 2;
    uint64_t x0[MAXIN], x1[MAXIN];
#pragma unroll
    for (int i = 0; i < MAXIN; ++i) {
        if (i < cnt) {
            const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(xt + (size_t)(lo + i) * ctx.N + j);
            x0[i] = v.x;
            x1[i] = v.y;
        }
    }
    __syncthreads();
    uint64_t* out = dig + ((size_t)d * dig_stride + m0) * ctx.N + j;
    // two targets per iteration: four independent 128-bit accumulators
#pragma unroll 1
    for (int mm = 0; mm < nt; mm += 2) {
        const int m2 = mm + 1 < nt ? mm + 1 : mm;
        ACC a, b, c2, d2;
#pragma unroll
        for (int i = 0; i < MAXIN; ++i) {
            if (i < cnt) {
                const uint64_t M = sM[i][mm], M2 = sM[i][m2];
                a.mac(x0[i], M);
                b.mac(x1[i], M);
                c2.mac(x0[i], M2);
                d2.mac(x1[i], M2);
            }
        }
        conv_store(out + (size_t)mm * ctx.N, a, b, sP[mm]);
        if (m2 != mm) conv_store(out + (size_t)m2 * ctx.N, c2, d2, sP[m2]);
    }
}

// One coefficient per thread, four targets per iteration: half the input
// registers of k_modup_conv (twice the resident warps), the same products.
template <int MAXIN>
__global__ void __launch_bounds__(kConvThreads) k_modup_conv_c1(const __grid_constant__ DevCtx ctx, int level,
                                                                const uint64_t* __restrict__ xt,
                                                                uint64_t* __restrict__ dig, size_t dig_stride,
                                                                size_t bstride) {
    __shared__ uint64_t sM[MAXIN][kConvTargets];
    __shared__ PrimeConst sP[kConvTargets];
    const int ndig = level / ctx.alpha + 1;
    const int d = blockIdx.y % ndig;
    const size_t boff = (size_t)(blockIdx.y / ndig) * bstride;
    xt += boff;
    dig += boff;
    const int n = level + 1;
    const int lo = d * ctx.alpha;
    const int hi = min(lo + ctx.alpha - 1, level);
    const int cnt = hi - lo + 1;
    const int ntar = n - cnt + ctx.K;
    const int m0 = blockIdx.z * kConvTargets;
    if (m0 >= ntar) return;
    const int nt = min(kConvTargets, ntar - m0);
    const int NP = ctx.L + ctx.K;
    const uint64_t* mat = ctx.modup_mat + (size_t)level * ctx.L * NP;
    for (int e = threadIdx.x; e < cnt * nt; e += kConvThreads) {
        const int i = e / nt, mm = e % nt, m = m0 + mm;
        const int jj = m < lo ? m : m + cnt;
        const int t = jj < n ? jj : ctx.L + (jj - n);
        sM[i][mm] = mat[(size_t)(lo + i) * NP + t];
        if (i == 0) sP[mm] = ctx.pc[t];
    }
    const size_t j = (size_t)blockIdx.x * kConvThreads + threadIdx.x;
    uint64_t x[MAXIN];
#pragma unroll
    for (int i = 0; i < MAXIN; ++i)
        if (i < cnt) x[i] = xt[(size_t)(lo + i) * ctx.N + j];
    __syncthreads();
    uint64_t* out = dig + ((size_t)d * dig_stride + m0) * ctx.N + j;
#pragma unroll 1
    for (int mm = 0; mm < nt; mm += 4) {
        int m[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) m[u] = min(mm + u, nt - 1);
        Acc128 acc[4];
#pragma unroll
        for (int i = 0; i < MAXIN; ++i) {
            if (i < cnt) {
#pragma unroll
                for (int u = 0; u < 4; ++u) acc[u].mac(x[i], sM[i][m[u]]);
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (mm + u < nt) out[(size_t)(mm + u) * ctx.N] = acc[u].reduce(sP[mm + u]);
    }
}

bool conv_supported(const DevCtx& ctx) { return ctx.alpha <= kMaxConvIn && ctx.K <= kMaxConvIn; }

void launch_modup_conv(const DevCtx& ctx, int level, int nb, const uint64_t* xt, uint64_t* dig, size_t dig_stride,
                       size_t bstride, cudaStream_t st) {
    if ((ctx.conv_variant == 3 || ctx.conv_variant == 4) && conv_tc_supported(ctx)) {
        launch_modup_conv_tc(ctx, level, nb, xt, dig, dig_stride, bstride, st, ctx.conv_variant == 3 ? 32 : 16);
        return;
    }
    const int nd = level / ctx.alpha + 1;
    const int maxtar = level + 1 + ctx.K;
    dim3 g(ctx.N / (2 * kConvThreads), nd * nb, (maxtar + kConvTargets - 1) / kConvTargets);
    count_launches(1);
    const dim3 g1(ctx.N / kConvThreads, g.y, g.z);
#define FIDES_MODUP(M)                                                                                       \
    if (ctx.conv_variant == 2)                                                                              \
        k_modup_conv_c1<M><<<g1, kConvThreads, 0, st>>>(ctx, level, xt, dig, dig_stride, bstride);          \
    else if (ctx.conv_variant == 1)                                                                         \
        k_modup_conv<M, AccSplit><<<g, kConvThreads, 0, st>>>(ctx, level, xt, dig, dig_stride, bstride);    \
    else                                                                                                    \
        k_modup_conv<M, Acc128><<<g, kConvThreads, 0, st>>>(ctx, level, xt, dig, dig_stride, bstride);
    if (ctx.alpha <= 4) {
        FIDES_MODUP(4)
    } else if (ctx.alpha <= 8) {
        FIDES_MODUP(8)
    } else if (ctx.alpha <= 12) {
        FIDES_MODUP(12)
    } else {
        FIDES_MODUP(16)
    }
#undef FIDES_MODUP
}

// ---------------------------------------------------------------------------
// key-switch inner product (fusedDotKSK_2_ / hoistedRotateDotKSK_2_)
//   xb[m] = sum_d D_d[t] * kb[d][t] (+ P * c0[t] for Q primes when c0 given)
//   xa[m] = sum_d D_d[t] * ka[d][t]
// over the extended basis m in [0, n+K) (prime t = m or L + m - n).  D_d[t] is
// the original evaluation value e2[t] when t lies in digit d, otherwise the
// ModUp output.  Rotations (galois g != 0): out[j] = sum_d D_d[slot(g, j)] *
// k'_d[j] (+ P * c0[slot(g, j)]), where a Galois key is held permuted,
// k'_d[j] = k_d[slot(g, j)] (the key that switches sigma_g(s) back to s):
// only the digit values and c0 are gathered, the key streams in order.
// ---------------------------------------------------------------------------
// Batch element b = blockIdx.x % nb varies fastest, so the blocks that read
// one key tile for the different elements run back to back and the key is
// fetched from HBM once and served from L2 to the rest of the batch.
// FPK: limbs of primes below 2^50 accumulate on the FP64 pipes (fp64.cuh):
// each product x k is reduced to |r| <= 0.875p, the sum of up to 8 digits
// stays below 7p < 2^53, and one centring plus a floor reduction give the
// canonical residue -- the same values as the 128-bit integer sums.
// SEED: some element's key is seeded (ka null), its a half regenerated per
// coefficient; the instantiation without it carries no generator code and
// keeps the register count of the plain streaming loop (32-40).  Left free,
// the unrolled digit loop with the generator takes 56-72 registers; the
// bound holds it at 48 (FP64 sums) or 40 so that 5-6 blocks stay resident
// (not the split-product accumulator, which would spill).
template <class ACC>
constexpr bool kIsSplitAcc = false;
template <>
constexpr bool kIsSplitAcc<AccSplit> = true;

template <int VEC, class ACC, bool FPK, bool GRP = false, bool SEED = false>
__global__ void __launch_bounds__(256, SEED ? (FPK ? 5 : (kIsSplitAcc<ACC> ? 0 : 6)) : 0)
    k_ks_inner(const __grid_constant__ DevCtx ctx, int level, int nb, const __grid_constant__ KsArgs args) {
    const int n = level + 1;
    const int m = blockIdx.y;
    const int bi = blockIdx.x % nb;
    const int bx = blockIdx.x / nb;
    const int t = m < n ? m : ctx.L + (m - n);
    const PrimeConst pc = ctx.pc[t];
    const int nd = level / ctx.alpha + 1;
    const size_t kstride = (size_t)(ctx.L + ctx.K) * ctx.N;
    const size_t boff = (size_t)bi * args.bstride;
    const uint64_t* kb = args.kb[bi];
    const uint64_t* ka = args.ka[bi];  // null: seeded, digit d's a half is uniform_mod(astream ^ (d+1) << 48, t, j)
    const uint64_t astream = args.a_seed[bi];
    // source limb of each digit for this prime (GRP, grouped hoisting: the
    // element's ModUp is that of its group, a table entry)
    const int gi = GRP ? (int)args.dig_elem[bi] : bi;
    const uint64_t* srcs[8];
#pragma unroll
    for (int d = 0; d < 8; ++d) {
        if (d < nd) {
            const int lo = d * ctx.alpha;
            const int hi = min(lo + ctx.alpha - 1, level);
            const int cnt = hi - lo + 1;
            if (m < n && t >= lo && t <= hi) {
                srcs[d] = args.own[bi] + (size_t)t * ctx.N;
            } else {
                const int md = m < n ? (t < lo ? t : t - cnt) : (n - cnt) + (m - n);
                srcs[d] = args.dig + (size_t)gi * args.dig_bstride + ((size_t)d * args.dig_stride + md) * ctx.N;
            }
        }
    }
    uint64_t* xb = args.xb + boff + (size_t)m * ctx.N;
    uint64_t* xa = args.xa + boff + (size_t)m * ctx.N;
    if constexpr (VEC && FPK) {
        if (pc.p < kFpPrimeBound) {
            const size_t j = ((size_t)bx * blockDim.x + threadIdx.x) * 2;
            const double p = __ull2double_rn(pc.p), pinv = as_f64(pc.pinv_f64);
            double sb0 = 0, sb1 = 0, sa0 = 0, sa1 = 0;
#pragma unroll
            for (int d = 0; d < 8; ++d) {
                if (d < nd) {
                    const ulonglong2 x = *reinterpret_cast<const ulonglong2*>(srcs[d] + j);
                    const ulonglong2 b = *reinterpret_cast<const ulonglong2*>(kb + d * kstride + (size_t)t * ctx.N + j);
                    ulonglong2 a;
                    if (!SEED || ka) {
                        a = *reinterpret_cast<const ulonglong2*>(ka + d * kstride + (size_t)t * ctx.N + j);
                    } else {
                        a.x = uniform_mod(astream ^ ((uint64_t)(d + 1) << 48), t, (uint32_t)j, pc.p);
                        a.y = uniform_mod(astream ^ ((uint64_t)(d + 1) << 48), t, (uint32_t)j + 1, pc.p);
                    }
                    const double x0 = as_f64(fp_from_u(x.x)), x1 = as_f64(fp_from_u(x.y));
                    sb0 = __dadd_rn(sb0, fp_mulmod(x0, as_f64(fp_from_u(b.x)), p, pinv));
                    sb1 = __dadd_rn(sb1, fp_mulmod(x1, as_f64(fp_from_u(b.y)), p, pinv));
                    sa0 = __dadd_rn(sa0, fp_mulmod(x0, as_f64(fp_from_u(a.x)), p, pinv));
                    sa1 = __dadd_rn(sa1, fp_mulmod(x1, as_f64(fp_from_u(a.y)), p, pinv));
                }
            }
            ulonglong2 ob, oa;
            ob.x = fp_to_u(fp_center(sb0, p, pinv), p, pinv);
            ob.y = fp_to_u(fp_center(sb1, p, pinv), p, pinv);
            oa.x = fp_to_u(fp_center(sa0, p, pinv), p, pinv);
            oa.y = fp_to_u(fp_center(sa1, p, pinv), p, pinv);
            *reinterpret_cast<ulonglong2*>(xb + j) = ob;
            *reinterpret_cast<ulonglong2*>(xa + j) = oa;
            return;
        }
    }
    if constexpr (VEC) {
        const size_t j = ((size_t)bx * blockDim.x + threadIdx.x) * 2;
        ACC sb0, sb1, sa0, sa1;
#pragma unroll
        for (int d = 0; d < 8; ++d) {
            if (d < nd) {
                const ulonglong2 x = *reinterpret_cast<const ulonglong2*>(srcs[d] + j);
                const ulonglong2 b = *reinterpret_cast<const ulonglong2*>(kb + d * kstride + (size_t)t * ctx.N + j);
                ulonglong2 a;
                if (!SEED || ka) {
                    a = *reinterpret_cast<const ulonglong2*>(ka + d * kstride + (size_t)t * ctx.N + j);
                } else {
                    a.x = uniform_mod(astream ^ ((uint64_t)(d + 1) << 48), t, (uint32_t)j, pc.p);
                    a.y = uniform_mod(astream ^ ((uint64_t)(d + 1) << 48), t, (uint32_t)j + 1, pc.p);
                }
                sb0.mac(x.x, b.x);
                sb1.mac(x.y, b.y);
                sa0.mac(x.x, a.x);
                sa1.mac(x.y, a.y);
            }
        }
        ulonglong2 ob, oa;
        ob.x = sb0.reduce(pc);
        ob.y = sb1.reduce(pc);
        oa.x = sa0.reduce(pc);
        oa.y = sa1.reduce(pc);
        *reinterpret_cast<ulonglong2*>(xb + j) = ob;
        *reinterpret_cast<ulonglong2*>(xa + j) = oa;
    } else {
        // rotation: outputs j, j+1 gather the digit values (and c0) at the
        // automorphism's source slots; the key is stored permuted (entry j is
        // the one that pairs with output j), so its loads stay vectorised
        const size_t j = ((size_t)bx * blockDim.x + threadIdx.x) * 2;
        const uint32_t g = args.galois[bi];
        const uint32_t s0 = g ? automorph_slot(ctx.logN, g, (uint32_t)j) : (uint32_t)j;
        const uint32_t s1 = g ? automorph_slot(ctx.logN, g, (uint32_t)j + 1) : (uint32_t)j + 1;
        const size_t koff = (size_t)t * ctx.N + j;
        const uint64_t* c0 = args.c0[bi];
        if constexpr (FPK) {
            // up to 6 digits: |sum| <= 6 * 0.875p + p (the P c0 term) < 2^53
            if (pc.p < kFpPrimeBound && nd <= 6) {
                const double p = __ull2double_rn(pc.p), pinv = as_f64(pc.pinv_f64);
                double sb0 = 0, sb1 = 0, sa0 = 0, sa1 = 0;
#pragma unroll
                for (int d = 0; d < 6; ++d) {
                    if (d < nd) {
                        const double x0 = as_f64(fp_from_u(srcs[d][s0])), x1 = as_f64(fp_from_u(srcs[d][s1]));
                        const ulonglong2 b = *reinterpret_cast<const ulonglong2*>(kb + d * kstride + koff);
                        ulonglong2 a;
                        if (!SEED || ka) {
                            a = *reinterpret_cast<const ulonglong2*>(ka + d * kstride + koff);
                        } else {
                            a.x = uniform_mod(astream ^ ((uint64_t)(d + 1) << 48), t, (uint32_t)j, pc.p);
                            a.y = uniform_mod(astream ^ ((uint64_t)(d + 1) << 48), t, (uint32_t)j + 1, pc.p);
                        }
                        sb0 = __dadd_rn(sb0, fp_mulmod(x0, as_f64(fp_from_u(b.x)), p, pinv));
                        sb1 = __dadd_rn(sb1, fp_mulmod(x1, as_f64(fp_from_u(b.y)), p, pinv));
                        sa0 = __dadd_rn(sa0, fp_mulmod(x0, as_f64(fp_from_u(a.x)), p, pinv));
                        sa1 = __dadd_rn(sa1, fp_mulmod(x1, as_f64(fp_from_u(a.y)), p, pinv));
                    }
                }
                if (c0 && m < n) {
                    const ulonglong2 pm = __ldg(reinterpret_cast<const ulonglong2*>(ctx.md_pmod) + t);
                    const uint64_t* cm = c0 + (size_t)m * ctx.N;
                    sb0 = __dadd_rn(sb0, as_f64(fp_from_u(mul_shoup(cm[s0], pm.x, pm.y, pc.p))));
                    sb1 = __dadd_rn(sb1, as_f64(fp_from_u(mul_shoup(cm[s1], pm.x, pm.y, pc.p))));
                }
                ulonglong2 ob, oa;
                ob.x = fp_to_u(fp_center(sb0, p, pinv), p, pinv);
                ob.y = fp_to_u(fp_center(sb1, p, pinv), p, pinv);
                oa.x = fp_to_u(fp_center(sa0, p, pinv), p, pinv);
                oa.y = fp_to_u(fp_center(sa1, p, pinv), p, pinv);
                *reinterpret_cast<ulonglong2*>(xb + j) = ob;
                *reinterpret_cast<ulonglong2*>(xa + j) = oa;
                return;
            }
        }
        ACC sb0, sb1, sa0, sa1;
#pragma unroll
        for (int d = 0; d < 8; ++d) {
            if (d < nd) {
                const uint64_t x0 = srcs[d][s0], x1 = srcs[d][s1];
                const ulonglong2 b = *reinterpret_cast<const ulonglong2*>(kb + d * kstride + koff);
                ulonglong2 a;
                if (!SEED || ka) {
                    a = *reinterpret_cast<const ulonglong2*>(ka + d * kstride + koff);
                } else {
                    a.x = uniform_mod(astream ^ ((uint64_t)(d + 1) << 48), t, (uint32_t)j, pc.p);
                    a.y = uniform_mod(astream ^ ((uint64_t)(d + 1) << 48), t, (uint32_t)j + 1, pc.p);
                }
                sb0.mac(x0, b.x);
                sb1.mac(x1, b.y);
                sa0.mac(x0, a.x);
                sa1.mac(x1, a.y);
            }
        }
        if (c0 && m < n) {
            const ulonglong2 pm = __ldg(reinterpret_cast<const ulonglong2*>(ctx.md_pmod) + t);
            const uint64_t* cm = c0 + (size_t)m * ctx.N;
            sb0.mac(mul_shoup(cm[s0], pm.x, pm.y, pc.p), 1);
            sb1.mac(mul_shoup(cm[s1], pm.x, pm.y, pc.p), 1);
        }
        ulonglong2 ob, oa;
        ob.x = sb0.reduce(pc);
        ob.y = sb1.reduce(pc);
        oa.x = sa0.reduce(pc);
        oa.y = sa1.reduce(pc);
        *reinterpret_cast<ulonglong2*>(xb + j) = ob;
        *reinterpret_cast<ulonglong2*>(xa + j) = oa;
    }
}

template <int VEC, class ACC, bool FPK, bool GRP>
static void ks_inner_go(const DevCtx& ctx, int level, int nb, const KsArgs& args, bool seeded, dim3 g,
                        cudaStream_t st) {
    if (seeded)
        k_ks_inner<VEC, ACC, FPK, GRP, true><<<g, 256, 0, st>>>(ctx, level, nb, args);
    else
        k_ks_inner<VEC, ACC, FPK, GRP, false><<<g, 256, 0, st>>>(ctx, level, nb, args);
}

void launch_ks_inner(const DevCtx& ctx, int level, int nb, const KsArgs& args, bool plain, cudaStream_t st) {
    count_launches(1);
    bool seeded = false;
    for (int b = 0; b < nb; ++b) seeded = seeded || args.ka[b] == nullptr;
    if (plain) {
        dim3 g(ctx.N / 512 * nb, level + 1 + ctx.K);
        if (ctx.ks_variant & 1)
            ks_inner_go<1, Acc128, true, false>(ctx, level, nb, args, seeded, g, st);
        else if (ctx.conv_variant == 1)
            ks_inner_go<1, AccSplit, false, false>(ctx, level, nb, args, seeded, g, st);
        else
            ks_inner_go<1, Acc128, false, false>(ctx, level, nb, args, seeded, g, st);
    } else if (args.dig_group > 0) {
        dim3 g(ctx.N / 512 * nb, level + 1 + ctx.K);
        if (ctx.ks_variant & 1)
            ks_inner_go<0, Acc128, true, true>(ctx, level, nb, args, seeded, g, st);
        else
            ks_inner_go<0, Acc128, false, true>(ctx, level, nb, args, seeded, g, st);
    } else {
        dim3 g(ctx.N / 512 * nb, level + 1 + ctx.K);
        if (ctx.ks_variant & 1)
            ks_inner_go<0, Acc128, true, false>(ctx, level, nb, args, seeded, g, st);
        else if (ctx.conv_variant == 1)
            ks_inner_go<0, AccSplit, false, false>(ctx, level, nb, args, seeded, g, st);
        else
            ks_inner_go<0, Acc128, false, false>(ctx, level, nb, args, seeded, g, st);
    }
}

// ---------------------------------------------------------------------------
// ModDown base conversion (ModDown2), both halves of a key-switch result in
// one launch (blockIdx.z = half).  y = special limbs already scaled by
// (P/p_k)^-1 (scaled INTT).  Without ttop: w_j = sum_k y_k [P/p_k]_{q_j} for
// j = 0..level.  With ttop (fused rescale; ttop = INTT(e_l + P^-1 x_l)):
//   conv_l = sum_k y_k [P/p_k]_{q_l};  tl = ttop - P^-1 conv_l  (mod q_l)
//   w_j = P^-1 conv_j + SwitchModulus(tl, q_l -> q_j)  for j < level.
// ---------------------------------------------------------------------------


template <int MAXIN, class ACC>
__global__ void __launch_bounds__(kConvThreads) k_moddown_conv(const __grid_constant__ DevCtx ctx, int level,
                                                               const __grid_constant__ MdArgs args) {
    __shared__ uint64_t sM[MAXIN][kConvTargets];
    __shared__ PrimeConst sP[kConvTargets];
    __shared__ ulonglong2 sPinv[kConvTargets];
    const int half = blockIdx.z & 1;
    const size_t boff = (size_t)(blockIdx.z >> 1) * args.bstride;
    const uint64_t* __restrict__ y = args.y[half] + boff;
    uint64_t* __restrict__ w = args.w[half] + boff;
    const uint64_t* __restrict__ ttop = args.ttop[half] ? args.ttop[half] + boff : nullptr;
    const int K = ctx.K, L = ctx.L;
    const int nout = ttop ? level : level + 1;
    const int q0 = blockIdx.y * kConvTargets;
    const int nt = min(kConvTargets, nout - q0);
    if (nt <= 0) return;
    for (int e = threadIdx.x; e < K * nt; e += kConvThreads) {
        const int k = e / nt, qq = e % nt;
        sM[k][qq] = ctx.md_mat[(size_t)k * L + q0 + qq];
        if (k == 0) {
            sP[qq] = ctx.pc[q0 + qq];
            sPinv[qq] = reinterpret_cast<const ulonglong2*>(ctx.md_pinv)[q0 + qq];
        }
    }
    const size_t j = ((size_t)blockIdx.x * kConvThreads + threadIdx.x) * 2;
    uint64_t y0[MAXIN], y1[MAXIN];
#pragma unroll
    for (int k = 0; k < MAXIN; ++k) {
        if (k < K) {
            const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(y + (size_t)k * ctx.N + j);
            y0[k] = v.x;
            y1[k] = v.y;
        }
    }
    uint64_t tl0 = 0, tl1 = 0;
    uint64_t ql = 0;
    if (ttop) {
        const PrimeConst pl = ctx.pc[level];
        const ulonglong2 pinv_l = reinterpret_cast<const ulonglong2*>(ctx.md_pinv)[level];
        ACC a, b;
#pragma unroll
        for (int k = 0; k < MAXIN; ++k) {
            if (k < K) {
                const uint64_t M = ctx.md_mat[(size_t)k * L + level];
                a.mac(y0[k], M);
                b.mac(y1[k], M);
            }
        }
        const ulonglong2 tv = *reinterpret_cast<const ulonglong2*>(ttop + j);
        tl0 = sub_mod(tv.x, mul_shoup(a.reduce(pl), pinv_l.x, pinv_l.y, pl.p), pl.p);
        tl1 = sub_mod(tv.y, mul_shoup(b.reduce(pl), pinv_l.x, pinv_l.y, pl.p), pl.p);
        ql = pl.p;
    }
    __syncthreads();
    auto finish = [&](int qq, const ACC& a, const ACC& b) {
        const PrimeConst pc = sP[qq];
        ulonglong2 o;
        o.x = a.reduce(pc);
        o.y = b.reduce(pc);
        if (ttop) {
            const ulonglong2 pinv = sPinv[qq];
            o.x = add_mod(mul_shoup(o.x, pinv.x, pinv.y, pc.p), switch_modulus(tl0, ql, pc), pc.p);
            o.y = add_mod(mul_shoup(o.y, pinv.x, pinv.y, pc.p), switch_modulus(tl1, ql, pc), pc.p);
        }
        *reinterpret_cast<ulonglong2*>(w + (size_t)(q0 + qq) * ctx.N + j) = o;
    };
#pragma unroll 1
    for (int qq = 0; qq < nt; qq += 2) {
        const int q2 = qq + 1 < nt ? qq + 1 : qq;
        ACC a, b, c2, d2;
#pragma unroll
        for (int k = 0; k < MAXIN; ++k) {
            if (k < K) {
                const uint64_t M = sM[k][qq], M2 = sM[k][q2];
                a.mac(y0[k], M);
                b.mac(y1[k], M);
                c2.mac(y0[k], M2);
                d2.mac(y1[k], M2);
            }
        }
        finish(qq, a, b);
        if (q2 != qq) finish(q2, c2, d2);
    }
}

void launch_moddown_conv(const DevCtx& ctx, int level, int nb, const MdArgs& a, cudaStream_t st) {
    const int nout = a.ttop[0] ? level : level + 1;
    if (nout <= 0) return;
    if ((ctx.conv_variant == 3 || ctx.conv_variant == 4) && conv_tc_supported(ctx)) {
        launch_moddown_conv_tc(ctx, level, nb, a, st, ctx.conv_variant == 3 ? 32 : 16);
        return;
    }
    dim3 g(ctx.N / (2 * kConvThreads), (nout + kConvTargets - 1) / kConvTargets, 2 * nb);
    count_launches(1);
#define FIDES_MODDOWN(M)                                                      \
    if (ctx.conv_variant == 1)                                                \
        k_moddown_conv<M, AccSplit><<<g, kConvThreads, 0, st>>>(ctx, level, a); \
    else                                                                      \
        k_moddown_conv<M, Acc128><<<g, kConvThreads, 0, st>>>(ctx, level, a);
    if (ctx.K <= 4) {
        FIDES_MODDOWN(4)
    } else if (ctx.K <= 8) {
        FIDES_MODDOWN(8)
    } else if (ctx.K <= 12) {
        FIDES_MODDOWN(12)
    } else {
        FIDES_MODDOWN(16)
    }
#undef FIDES_MODDOWN
}

// ---------------------------------------------------------------------------
// element-wise
// ---------------------------------------------------------------------------
template <int OP>
__global__ void k_elementwise(const __grid_constant__ DevCtx ctx, int q0, const uint64_t* __restrict__ a,
                              const uint64_t* __restrict__ b, uint64_t* __restrict__ out) {
    const int limb = blockIdx.y;
    const PrimeConst pc = ctx.pc[q0 + limb];
    const size_t i = (size_t)limb * ctx.N + (size_t)(blockIdx.x * blockDim.x + threadIdx.x) * 2;
    const ulonglong2 x = *reinterpret_cast<const ulonglong2*>(a + i);
    ulonglong2 r;
    if constexpr (OP == EW_COPY) {
        r = x;
    } else if constexpr (OP == EW_NEG) {
        r.x = neg_mod(x.x, pc.p);
        r.y = neg_mod(x.y, pc.p);
    } else {
        const ulonglong2 y = *reinterpret_cast<const ulonglong2*>(b + i);
        if constexpr (OP == EW_ADD) {
            r.x = add_mod(x.x, y.x, pc.p);
            r.y = add_mod(x.y, y.y, pc.p);
        } else if constexpr (OP == EW_SUB) {
            r.x = sub_mod(x.x, y.x, pc.p);
            r.y = sub_mod(x.y, y.y, pc.p);
        } else {
            r.x = mul_mod(x.x, y.x, pc);
            r.y = mul_mod(x.y, y.y, pc);
        }
    }
    *reinterpret_cast<ulonglong2*>(out + i) = r;
}

void launch_elementwise(const DevCtx& ctx, int op, int n, int q0, const uint64_t* a, const uint64_t* b,
                        uint64_t* out, cudaStream_t st) {
    if (n <= 0) return;
    dim3 g(ctx.N / 256, n);
    switch (op) {
        case EW_ADD: count_launches(1); k_elementwise<EW_ADD><<<g, 128, 0, st>>>(ctx, q0, a, b, out); break;
        case EW_SUB: count_launches(1); k_elementwise<EW_SUB><<<g, 128, 0, st>>>(ctx, q0, a, b, out); break;
        case EW_NEG: count_launches(1); k_elementwise<EW_NEG><<<g, 128, 0, st>>>(ctx, q0, a, b, out); break;
        case EW_MUL: count_launches(1); k_elementwise<EW_MUL><<<g, 128, 0, st>>>(ctx, q0, a, b, out); break;
        default: count_launches(1); k_elementwise<EW_COPY><<<g, 128, 0, st>>>(ctx, q0, a, b, out); break;
    }
}

// Extended-basis sums of key-switch results: for output u, the elements
// start[u] .. start[u+1]-1 of XB and XA (n ciphertext limbs, then K special
// limbs, at bstride) are added into element start[u].  Two coefficients per
// thread.
__global__ void k_ext_sum(const __grid_constant__ DevCtx ctx, const __grid_constant__ ExtSumArgs a) {
    const int limb = blockIdx.y, u = blockIdx.z;
    const int j = (blockIdx.x * blockDim.x + threadIdx.x) * 2;
    if (j >= ctx.N) return;
    const uint64_t p = ctx.pc[limb < a.n ? limb : ctx.L + (limb - a.n)].p;
    const size_t i = (size_t)limb * ctx.N + j;
    const int b0 = a.start[u], b1 = a.start[u + 1];
    for (int h = 0; h < 2; ++h) {
        ulonglong2* dst = reinterpret_cast<ulonglong2*>(a.x[h] + (size_t)b0 * a.bstride + i);
        ulonglong2 s = *dst;
        for (int b = b0 + 1; b < b1; ++b) {
            const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(a.x[h] + (size_t)b * a.bstride + i);
            s.x = add_mod(s.x, v.x, p);
            s.y = add_mod(s.y, v.y, p);
        }
        *dst = s;
    }
}

void launch_ext_sum(const DevCtx& ctx, const ExtSumArgs& a, cudaStream_t st) {
    if (a.nout <= 0) return;
    count_launches(1);
    k_ext_sum<<<dim3((ctx.N + 511) / 512, a.n + ctx.K, a.nout), 256, 0, st>>>(ctx, a);
}

__global__ void k_scalar_mac(const __grid_constant__ DevCtx ctx, const uint64_t* __restrict__ a,
                             const uint64_t* __restrict__ cj, const uint64_t* __restrict__ b,
                             uint64_t* __restrict__ out) {
    const int limb = blockIdx.y;
    const PrimeConst pc = ctx.pc[limb];
    const ulonglong2 c = __ldg(reinterpret_cast<const ulonglong2*>(cj) + limb);
    const size_t i = (size_t)limb * ctx.N + (size_t)(blockIdx.x * blockDim.x + threadIdx.x) * 2;
    const ulonglong2 x = *reinterpret_cast<const ulonglong2*>(a + i);
    ulonglong2 r;
    r.x = mul_shoup(x.x, c.x, c.y, pc.p);
    r.y = mul_shoup(x.y, c.x, c.y, pc.p);
    if (b) {
        const ulonglong2 y = *reinterpret_cast<const ulonglong2*>(b + i);
        r.x = add_mod(r.x, y.x, pc.p);
        r.y = add_mod(r.y, y.y, pc.p);
    }
    *reinterpret_cast<ulonglong2*>(out + i) = r;
}

void launch_scalar_mac(const DevCtx& ctx, int n, const uint64_t* a, const uint64_t* cj, const uint64_t* b,
                       uint64_t* out, cudaStream_t st) {
    if (n <= 0) return;
    dim3 g(ctx.N / 256, n);
    count_launches(1);
    k_scalar_mac<<<g, 128, 0, st>>>(ctx, a, cj, b, out);
}

__global__ void k_scalar_add(const __grid_constant__ DevCtx ctx, const uint64_t* __restrict__ a,
                             const uint64_t* __restrict__ cj, uint64_t* __restrict__ out) {
    const int limb = blockIdx.y;
    const PrimeConst pc = ctx.pc[limb];
    const uint64_t c = __ldg(cj + limb);
    const size_t i = (size_t)limb * ctx.N + (size_t)(blockIdx.x * blockDim.x + threadIdx.x) * 2;
    const ulonglong2 x = *reinterpret_cast<const ulonglong2*>(a + i);
    ulonglong2 r;
    r.x = add_mod(x.x, c, pc.p);
    r.y = add_mod(x.y, c, pc.p);
    *reinterpret_cast<ulonglong2*>(out + i) = r;
}

void launch_scalar_add(const DevCtx& ctx, int n, const uint64_t* a, const uint64_t* cj, uint64_t* out,
                       cudaStream_t st) {
    if (n <= 0) return;
    dim3 g(ctx.N / 256, n);
    count_launches(1);
    k_scalar_add<<<g, 128, 0, st>>>(ctx, a, cj, out);
}

// Plaintext dot product: each thread owns two coefficients of both halves,
// reads each plaintext term once for c0 and c1.  Products of residues below
// 2^62 are below 2^124, so 15 of them plus a folded residue fit in 128 bits;
// the accumulators are folded back to one residue every 15 terms.
// Role in the reference: dotProductPt_ (CKKS/ElemenwiseBatchKernels.cu:651).
__global__ void k_dot_pt(const __grid_constant__ DevCtx ctx, const __grid_constant__ DotArgs args) {
    const int limb = blockIdx.y;
    const PrimeConst pc = ctx.pc[limb];
    const size_t i = (size_t)limb * ctx.N + (size_t)(blockIdx.x * blockDim.x + threadIdx.x) * 2;
    Acc128 a0, a1, b0, b1;
    if (args.accumulate) {
        const ulonglong2 x = *reinterpret_cast<const ulonglong2*>(args.o0 + i);
        const ulonglong2 y = *reinterpret_cast<const ulonglong2*>(args.o1 + i);
        a0.lo = x.x;
        a1.lo = x.y;
        b0.lo = y.x;
        b1.lo = y.y;
    }
    int since = 0;
#pragma unroll 1
    for (int k = 0; k < args.n; ++k) {
        const ulonglong2 w = __ldg(reinterpret_cast<const ulonglong2*>(args.p[k] + i));
        const ulonglong2 x = *reinterpret_cast<const ulonglong2*>(args.c0[k] + i);
        const ulonglong2 y = *reinterpret_cast<const ulonglong2*>(args.c1[k] + i);
        a0.mac(x.x, w.x);
        a1.mac(x.y, w.y);
        b0.mac(y.x, w.x);
        b1.mac(y.y, w.y);
        if (++since == 15) {
            a0.lo = a0.reduce(pc), a0.hi = 0;
            a1.lo = a1.reduce(pc), a1.hi = 0;
            b0.lo = b0.reduce(pc), b0.hi = 0;
            b1.lo = b1.reduce(pc), b1.hi = 0;
            since = 0;
        }
    }
    ulonglong2 r;
    r.x = a0.reduce(pc);
    r.y = a1.reduce(pc);
    *reinterpret_cast<ulonglong2*>(args.o0 + i) = r;
    r.x = b0.reduce(pc);
    r.y = b1.reduce(pc);
    *reinterpret_cast<ulonglong2*>(args.o1 + i) = r;
}

void launch_dot_pt(const DevCtx& ctx, int nlimbs, const DotArgs& args, cudaStream_t st) {
    if (nlimbs <= 0 || args.n <= 0 || args.n > kMaxBatch) return;
    dim3 g(ctx.N / 256, nlimbs);
    count_launches(1);
    k_dot_pt<<<g, 128, 0, st>>>(ctx, args);
}

// Integer linear combination (leaf sums of polynomial evaluation, integer
// scalar products): each thread owns two coefficients of both components.
__global__ void k_lincomb(const __grid_constant__ DevCtx ctx, const __grid_constant__ LinArgs args) {
    const int limb = blockIdx.y;
    const PrimeConst pc = ctx.pc[args.q0 + limb];
    const size_t i = (size_t)limb * ctx.N + (size_t)(blockIdx.x * blockDim.x + threadIdx.x) * 2;
    ulonglong2 r0 = make_ulonglong2(0, 0), r1 = make_ulonglong2(0, 0);
#pragma unroll 1
    for (int k = 0; k < args.n; ++k) {
        const uint64_t z = args.z[k][limb][0], zs = args.z[k][limb][1];
        const ulonglong2 x = *reinterpret_cast<const ulonglong2*>(args.in0[k] + i);
        const ulonglong2 y = *reinterpret_cast<const ulonglong2*>(args.in1[k] + i);
        r0.x = add_mod(r0.x, mul_shoup(x.x, z, zs, pc.p), pc.p);
        r0.y = add_mod(r0.y, mul_shoup(x.y, z, zs, pc.p), pc.p);
        r1.x = add_mod(r1.x, mul_shoup(y.x, z, zs, pc.p), pc.p);
        r1.y = add_mod(r1.y, mul_shoup(y.y, z, zs, pc.p), pc.p);
    }
    if (args.has_add) {
        r0.x = add_mod(r0.x, args.add0[limb], pc.p);
        r0.y = add_mod(r0.y, args.add0[limb], pc.p);
    }
    *reinterpret_cast<ulonglong2*>(args.out0 + i) = r0;
    *reinterpret_cast<ulonglong2*>(args.out1 + i) = r1;
}

void launch_lincomb(const DevCtx& ctx, int nlimbs, const LinArgs& args, cudaStream_t st) {
    if (nlimbs <= 0 || nlimbs > kMaxLinLimbs || args.n < 0 || args.n > kMaxLin) return;
    dim3 g(ctx.N / 256, nlimbs);
    count_launches(1);
    k_lincomb<<<g, 128, 0, st>>>(ctx, args);
}

// X^k in evaluation form: slot i of prime j holds psi_j^e, e = (2 brev(i) + 1) k
// mod 2N; psi^m = fwd_tw[j][brev(m)] for m < N and psi^N = -1.
// Role in the reference: Ciphertext::multMonomial (used by Bootstrap.cu:268).
__global__ void k_mult_monomial(const __grid_constant__ DevCtx ctx, const uint64_t* __restrict__ in0,
                                const uint64_t* __restrict__ in1, uint64_t* __restrict__ out0,
                                uint64_t* __restrict__ out1, uint32_t k) {
    const int limb = blockIdx.y;
    const uint64_t* in = blockIdx.z ? in1 : in0;
    uint64_t* out = blockIdx.z ? out1 : out0;
    const uint64_t p = ctx.pc[limb].p;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t mask2n = (2u << ctx.logN) - 1;
    const uint32_t e = (((brev_bits(i, ctx.logN) << 1) + 1) * k) & mask2n;
    const uint32_t m = e & ((uint32_t)ctx.N - 1);
    const ulonglong2 w = __ldg(reinterpret_cast<const ulonglong2*>(ctx.fwd_tw) + (size_t)limb * ctx.N +
                               brev_bits(m, ctx.logN));
    const size_t o = (size_t)limb * ctx.N + i;
    const uint64_t v = mul_shoup(in[o], w.x, w.y, p);
    out[o] = (e >= (uint32_t)ctx.N) ? neg_mod(v, p) : v;
}

void launch_mult_monomial(const DevCtx& ctx, int nlimbs, const uint64_t* in0, const uint64_t* in1, uint64_t* out0,
                          uint64_t* out1, uint32_t k, cudaStream_t st) {
    if (nlimbs <= 0) return;
    dim3 g(ctx.N / 256, nlimbs, 2);
    count_launches(1);
    k_mult_monomial<<<g, 256, 0, st>>>(ctx, in0, in1, out0, out1, k);
}

__global__ void k_automorph(const __grid_constant__ DevCtx ctx, const uint64_t* __restrict__ in,
                            uint64_t* __restrict__ out, uint32_t galois_inv) {
    const size_t base = (size_t)blockIdx.y * ctx.N;
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    out[base + j] = in[base + automorph_slot(ctx.logN, galois_inv, j)];
}

void launch_automorph(const DevCtx& ctx, int nlimbs, const uint64_t* in, uint64_t* out, uint32_t galois_inv,
                      cudaStream_t st) {
    if (nlimbs <= 0) return;
    dim3 g(ctx.N / 256, nlimbs);
    count_launches(1);
    k_automorph<<<g, 256, 0, st>>>(ctx, in, out, galois_inv);
}

}  // namespace fides
