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
//   * rotations fold the automorphism into the inner product as a gather, so
//     stores stay coalesced.
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
// tensor product (binomialMult_): e0 = a0 b0, e1 = a0 b1 + a1 b0, e2 = a1 b1
// ---------------------------------------------------------------------------
__global__ void k_tensor(const __grid_constant__ DevCtx ctx, const uint64_t* __restrict__ a0,
                         const uint64_t* __restrict__ a1, const uint64_t* __restrict__ b0,
                         const uint64_t* __restrict__ b1, uint64_t* __restrict__ e0, uint64_t* __restrict__ e1,
                         uint64_t* __restrict__ e2) {
    const int limb = blockIdx.y;
    const PrimeConst pc = ctx.pc[limb];
    const size_t i = ((size_t)limb * ctx.N + (size_t)(blockIdx.x * blockDim.x + threadIdx.x) * 2);
    const ulonglong2 x0 = *reinterpret_cast<const ulonglong2*>(a0 + i);
    const ulonglong2 x1 = *reinterpret_cast<const ulonglong2*>(a1 + i);
    const ulonglong2 y0 = *reinterpret_cast<const ulonglong2*>(b0 + i);
    const ulonglong2 y1 = *reinterpret_cast<const ulonglong2*>(b1 + i);
    ulonglong2 r0, r1, r2;
    r0.x = mul_mod(x0.x, y0.x, pc);
    r0.y = mul_mod(x0.y, y0.y, pc);
    {
        Acc128 s;
        s.mac(x0.x, y1.x);
        s.mac(x1.x, y0.x);
        r1.x = s.reduce(pc);
        Acc128 t;
        t.mac(x0.y, y1.y);
        t.mac(x1.y, y0.y);
        r1.y = t.reduce(pc);
    }
    r2.x = mul_mod(x1.x, y1.x, pc);
    r2.y = mul_mod(x1.y, y1.y, pc);
    *reinterpret_cast<ulonglong2*>(e0 + i) = r0;
    *reinterpret_cast<ulonglong2*>(e1 + i) = r1;
    *reinterpret_cast<ulonglong2*>(e2 + i) = r2;
}

void launch_tensor(const DevCtx& ctx, int n, const uint64_t* a0, const uint64_t* a1, const uint64_t* b0,
                   const uint64_t* b1, uint64_t* e0, uint64_t* e1, uint64_t* e2, cudaStream_t st) {
    dim3 g(ctx.N / 256, n);
    count_launches(1);
    k_tensor<<<g, 128, 0, st>>>(ctx, a0, a1, b0, b1, e0, e1, e2);
}

// ---------------------------------------------------------------------------
// ModUp base conversion (DecompAndModUpConv): for digit d at `level`, with
// inputs xt_i = [x_i * (Q'/q_i)^-1]_{q_i} (produced by the scaled INTT), every
// target prime t outside the digit gets  sum_i xt_i * [Q'/q_i]_t  mod t.
// Digit d's targets are stored at dig + (d*dig_stride + m)*N, m = target index
// (Q primes below the digit, Q primes above it up to `level`, then P).
// ---------------------------------------------------------------------------
constexpr int kConvThreads = 128;
constexpr int kTargetsPerBlock = 8;

__global__ void __launch_bounds__(kConvThreads) k_modup_conv(const __grid_constant__ DevCtx ctx, int level,
                                                             const uint64_t* __restrict__ xt,
                                                             uint64_t* __restrict__ dig, size_t dig_stride) {
    extern __shared__ uint64_t xs[];  // [cnt][kConvThreads]
    const int d = blockIdx.y;
    const int n = level + 1;
    const int lo = d * ctx.alpha;
    int hi = lo + ctx.alpha - 1;
    if (hi > level) hi = level;
    const int cnt = hi - lo + 1;
    const int ntar = n - cnt + ctx.K;
    const int m0 = blockIdx.z * kTargetsPerBlock;
    if (m0 >= ntar) return;
    const int m1 = min(m0 + kTargetsPerBlock, ntar);
    const int j = blockIdx.x * kConvThreads + threadIdx.x;
    for (int i = 0; i < cnt; ++i) xs[i * kConvThreads + threadIdx.x] = xt[(size_t)(lo + i) * ctx.N + j];
    const uint64_t* mat = ctx.modup_mat + (size_t)level * ctx.L * (ctx.L + ctx.K);
    const int NP = ctx.L + ctx.K;
    for (int m = m0; m < m1; ++m) {
        const int jj = m < lo ? m : m + cnt;
        const int t = jj < n ? jj : ctx.L + (jj - n);
        const PrimeConst pc = ctx.pc[t];
        Acc128 acc;
        int run = 0;
        for (int i = 0; i < cnt; ++i) {
            acc.mac(xs[i * kConvThreads + threadIdx.x], __ldg(mat + (size_t)(lo + i) * NP + t));
            if (++run == 15 && i + 1 < cnt) {  // keep the 128-bit sum from overflowing
                const uint64_t v = acc.reduce(pc);
                acc = Acc128();
                acc.lo = v;
                run = 1;
            }
        }
        dig[((size_t)d * dig_stride + m) * ctx.N + j] = acc.reduce(pc);
    }
}

void launch_modup_conv(const DevCtx& ctx, int level, const uint64_t* xt, uint64_t* dig, size_t dig_stride,
                       cudaStream_t st) {
    const int nd = level / ctx.alpha + 1;
    const int maxtar = level + 1 + ctx.K;
    dim3 g(ctx.N / kConvThreads, nd, (maxtar + kTargetsPerBlock - 1) / kTargetsPerBlock);
    const size_t smem = sizeof(uint64_t) * kConvThreads * ctx.alpha;
    count_launches(1);
    k_modup_conv<<<g, kConvThreads, smem, st>>>(ctx, level, xt, dig, dig_stride);
}

// ---------------------------------------------------------------------------
// key-switch inner product (fusedDotKSK_2_ / hoistedRotateDotKSK_2_)
//   xb[m] = sum_d D_d[t] * kb[d][t] (+ P * c0[t] for Q primes when c0 given)
//   xa[m] = sum_d D_d[t] * ka[d][t]
// over the extended basis m in [0, n+K) (prime t = m or L + m - n).  D_d[t] is
// the original evaluation value e2[t] when t lies in digit d, otherwise the
// ModUp output.  With galois_inv != 0 the result is written permuted:
// out[j] = value at slot(galois_inv, j).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_ks_inner(const __grid_constant__ DevCtx ctx, int level,
                                                  const uint64_t* __restrict__ e2, const uint64_t* __restrict__ dig,
                                                  size_t dig_stride, const uint64_t* __restrict__ kb,
                                                  const uint64_t* __restrict__ ka, uint64_t* __restrict__ xb,
                                                  uint64_t* __restrict__ xa, const uint64_t* __restrict__ c0,
                                                  uint32_t galois_inv) {
    const int n = level + 1;
    const int m = blockIdx.y;
    const int t = m < n ? m : ctx.L + (m - n);
    const PrimeConst pc = ctx.pc[t];
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t src = galois_inv ? automorph_slot(ctx.logN, galois_inv, j) : (uint32_t)j;
    const int nd = level / ctx.alpha + 1;
    const size_t kstride = (size_t)(ctx.L + ctx.K) * ctx.N;
    Acc128 sb, sa;
    for (int d = 0; d < nd; ++d) {
        const int lo = d * ctx.alpha;
        const int hi = min(lo + ctx.alpha - 1, level);
        const int cnt = hi - lo + 1;
        uint64_t x;
        if (m < n && t >= lo && t <= hi) {
            x = e2[(size_t)t * ctx.N + src];
        } else {
            const int md = m < n ? (t < lo ? t : t - cnt) : (n - cnt) + (m - n);
            x = dig[((size_t)d * dig_stride + md) * ctx.N + src];
        }
        sb.mac(x, kb[d * kstride + (size_t)t * ctx.N + src]);
        sa.mac(x, ka[d * kstride + (size_t)t * ctx.N + src]);
    }
    if (c0 && m < n) {
        const ulonglong2 pm = __ldg(reinterpret_cast<const ulonglong2*>(ctx.md_pmod) + t);
        sb.mac(mul_shoup(c0[(size_t)m * ctx.N + src], pm.x, pm.y, pc.p), 1);
    }
    xb[(size_t)m * ctx.N + j] = sb.reduce(pc);
    xa[(size_t)m * ctx.N + j] = sa.reduce(pc);
}

void launch_ks_inner(const DevCtx& ctx, int level, const uint64_t* e2, const uint64_t* dig, size_t dig_stride,
                     const uint64_t* kb, const uint64_t* ka, uint64_t* xb, uint64_t* xa, const uint64_t* c0,
                     uint32_t galois_inv, cudaStream_t st) {
    dim3 g(ctx.N / 256, level + 1 + ctx.K);
    count_launches(1);
    k_ks_inner<<<g, 256, 0, st>>>(ctx, level, e2, dig, dig_stride, kb, ka, xb, xa, c0, galois_inv);
}

// ---------------------------------------------------------------------------
// ModDown base conversion (ModDown2).  y = special limbs already scaled by
// (P/p_k)^-1 (scaled INTT).  Without ttop: w_j = sum_k y_k [P/p_k]_{q_j} for
// j = 0..level.  With ttop (fused rescale; ttop = INTT(e_l + P^-1 x_l)):
//   conv_l = sum_k y_k [P/p_k]_{q_l};  tl = ttop - P^-1 conv_l  (mod q_l)
//   w_j = P^-1 conv_j + SwitchModulus(tl, q_l -> q_j)  for j < level.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t switch_modulus_d(uint64_t a, uint64_t om, const PrimeConst& nc) {
    const uint64_t nm = nc.p;
    if (nm > om) return a > (om >> 1) ? a + (nm - om) : a;
    const uint64_t om_mod = csub(reduce64_lazy(om, nc), nm);
    uint64_t v = a > (om >> 1) ? a + (nm - om_mod) : a;
    return csub(reduce64_lazy(v, nc), nm);
}

__global__ void __launch_bounds__(kConvThreads) k_moddown_conv(const __grid_constant__ DevCtx ctx, int level,
                                                               const uint64_t* __restrict__ y,
                                                               uint64_t* __restrict__ w,
                                                               const uint64_t* __restrict__ ttop) {
    extern __shared__ uint64_t ys[];  // [K][kConvThreads]
    const int j = blockIdx.x * kConvThreads + threadIdx.x;
    const int K = ctx.K, L = ctx.L;
    for (int k = 0; k < K; ++k) ys[k * kConvThreads + threadIdx.x] = y[(size_t)k * ctx.N + j];
    auto conv = [&](int q) -> uint64_t {
        const PrimeConst pc = ctx.pc[q];
        Acc128 acc;
        int run = 0;
        for (int k = 0; k < K; ++k) {
            acc.mac(ys[k * kConvThreads + threadIdx.x], __ldg(ctx.md_mat + (size_t)k * L + q));
            if (++run == 15 && k + 1 < K) {
                const uint64_t v = acc.reduce(pc);
                acc = Acc128();
                acc.lo = v;
                run = 1;
            }
        }
        return acc.reduce(pc);
    };
    if (!ttop) {
        for (int q = blockIdx.y * kTargetsPerBlock; q < min((int)(blockIdx.y + 1) * kTargetsPerBlock, level + 1); ++q)
            w[(size_t)q * ctx.N + j] = conv(q);
        return;
    }
    const PrimeConst pl = ctx.pc[level];
    const ulonglong2 pinv_l = __ldg(reinterpret_cast<const ulonglong2*>(ctx.md_pinv) + level);
    const uint64_t tl = sub_mod(ttop[j], mul_shoup(conv(level), pinv_l.x, pinv_l.y, pl.p), pl.p);
    for (int q = blockIdx.y * kTargetsPerBlock; q < min((int)(blockIdx.y + 1) * kTargetsPerBlock, level); ++q) {
        const PrimeConst pc = ctx.pc[q];
        const ulonglong2 pinv = __ldg(reinterpret_cast<const ulonglong2*>(ctx.md_pinv) + q);
        const uint64_t a = mul_shoup(conv(q), pinv.x, pinv.y, pc.p);
        w[(size_t)q * ctx.N + j] = add_mod(a, switch_modulus_d(tl, pl.p, pc), pc.p);
    }
}

void launch_moddown_conv(const DevCtx& ctx, int level, const uint64_t* y, uint64_t* w, const uint64_t* ttop,
                         cudaStream_t st) {
    const int nout = ttop ? level : level + 1;
    if (nout <= 0) return;
    dim3 g(ctx.N / kConvThreads, (nout + kTargetsPerBlock - 1) / kTargetsPerBlock);
    const size_t smem = sizeof(uint64_t) * kConvThreads * ctx.K;
    count_launches(1);
    k_moddown_conv<<<g, kConvThreads, smem, st>>>(ctx, level, y, w, ttop);
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
