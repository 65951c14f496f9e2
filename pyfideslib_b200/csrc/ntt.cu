// ntt.cu -- negacyclic NTT / INTT over RNS limbs for sm_100a.
//
// Role in the reference: src/NTT.cu NTT_/INTT_ (two-pass 2-D decomposition with
// fused prologues/epilogues, NTTfusions.cuh).  The transform computed is the
// same one: natural-order coefficients -> evaluations in bit-reversed order,
//   out[i] = sum_j a_j psi^{(2 bitrev(i) + 1) j}  (mod p),
// i.e. the in-place Cooley-Tukey loop over the bit-reversed psi table, and its
// Gentleman-Sande inverse with N^-1 folded into the last stage.
//
// Layout and schedule (this file's own design):
//   * N = R x C with R = 2^LR rows of C = 2^LC contiguous coefficients.  The
//     first LR stages only pair elements of one column, the last LC stages
//     only elements of one row.  Pass 1 runs the column stages, pass 2 the
//     row stages; the intermediate limb (512 KiB at N=2^16) stays in L2.
//   * Each thread owns 16 elements of one column/row in registers and runs 4
//     butterfly stages on them (radix-16 register blocking); the next group
//     of stages follows one shared-memory exchange.  Column passes move 16
//     consecutive columns per CTA (128-byte coalesced rows); row passes stage
//     through shared memory so that global stores are coalesced.
//   * Harvey lazy butterflies: values stay in [0,4p) (forward) or [0,2p)
//     (inverse) and are reduced once at the end; twiddles are read as
//     16-byte (w, Shoup companion) pairs.
//   * Prologues/epilogues fuse the surrounding element-wise work (products of
//     two inputs, ModDown/Rescale combinations, per-limb CRT scalings).
#include <atomic>

#include "kernels.hpp"

namespace fides {

__device__ __forceinline__ void ct_bfly(uint64_t& X, uint64_t& Y, const ulonglong2 w, const uint64_t p,
                                        const uint64_t two_p) {
    const uint64_t x = csub(X, two_p);
    const uint64_t t = mul_shoup_lazy(Y, w.x, w.y, p);
    X = x + t;
    Y = x - t + two_p;
}

__device__ __forceinline__ void gs_bfly(uint64_t& X, uint64_t& Y, const ulonglong2 w, const uint64_t p,
                                        const uint64_t two_p) {
    const uint64_t s = csub(X + Y, two_p);
    const uint64_t d = X - Y + two_p;
    X = s;
    Y = mul_shoup_lazy(d, w.x, w.y, p);
}

__device__ __forceinline__ uint64_t reduce4p(uint64_t v, const PrimeConst& c) { return csub(csub(v, c.two_p), c.p); }

// Centred lift of a residue mod om into nm (src/CKKS/Rescale.cuh:45-62).
__device__ __forceinline__ uint64_t switch_modulus(uint64_t a, uint64_t om, const PrimeConst& nc) {
    const uint64_t nm = nc.p;
    if (nm > om) return a > (om >> 1) ? a + (nm - om) : a;
    const uint64_t om_mod = csub(reduce64_lazy(om, nc), nm);
    uint64_t v = a > (om >> 1) ? a + (nm - om_mod) : a;
    return csub(reduce64_lazy(v, nc), nm);
}

__device__ __forceinline__ ulonglong2 ldg2(const uint64_t* base, size_t idx) {
    return __ldg(reinterpret_cast<const ulonglong2*>(base) + idx);
}

// ---------------------------------------------------------------------------
// forward, pass 1: column stages 0..LR-1
// ---------------------------------------------------------------------------
template <int LR, int LC, int LOAD>
__global__ void __launch_bounds__(256, 2) k_ntt_fwd_cols(const __grid_constant__ DevCtx ctx,
                                                         const __grid_constant__ LimbMap map) {
    constexpr int R = 1 << LR, C = 1 << LC;
    constexpr int TPL = 1 << (LR - 4);
    constexpr int TC = (256 / TPL) < C ? (256 / TPL) : C;
    constexpr int NT = TPL * TC;
    __shared__ __align__(16) uint64_t sm[R * TC];
    __shared__ ulonglong2 tw[R];

    const LimbRef lr = resolve_limb(map, blockIdx.y, ctx.N, ctx.L);
    const PrimeConst pc = ctx.pc[lr.prime];
    const ulonglong2* twg = reinterpret_cast<const ulonglong2*>(ctx.fwd_tw) + (size_t)lr.prime * ctx.N;
    for (int i = threadIdx.x; i < R; i += NT) tw[i] = twg[i];

    const int c = threadIdx.x % TC, th = threadIdx.x / TC;
    const int col = blockIdx.x * TC + c;
    uint64_t x[16];
    if constexpr (LOAD == FL_SWITCHMOD) {
        const uint64_t om = ctx.pc[lr.level].p;
#pragma unroll
        for (int k = 0; k < 16; ++k) x[k] = switch_modulus(lr.in[(size_t)(th + (k << (LR - 4))) * C + col], om, pc);
    } else {
#pragma unroll
        for (int k = 0; k < 16; ++k) x[k] = lr.in[(size_t)(th + (k << (LR - 4))) * C + col];
    }
    __syncthreads();

#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const int kb = 3 - t;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            if (k & (1 << kb)) continue;
            const int r = th + (k << (LR - 4));
            ct_bfly(x[k], x[k | (1 << kb)], tw[(1 << t) + (r >> (LR - t))], pc.p, pc.two_p);
        }
    }
    if constexpr (LR > 4) {
#pragma unroll
        for (int k = 0; k < 16; ++k) sm[(th + (k << (LR - 4))) * TC + c] = x[k];
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 16; ++k) x[k] = sm[((th << 4) + k) * TC + c];
#pragma unroll
        for (int t = 4; t < LR; ++t) {
            const int kb = LR - 1 - t;
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                if (k & (1 << kb)) continue;
                const int r = (th << 4) + k;
                ct_bfly(x[k], x[k | (1 << kb)], tw[(1 << t) + (r >> (LR - t))], pc.p, pc.two_p);
            }
        }
#pragma unroll
        for (int k = 0; k < 16; ++k) lr.out[(size_t)((th << 4) + k) * C + col] = x[k];
    } else {
#pragma unroll
        for (int k = 0; k < 16; ++k) lr.out[(size_t)(th + k) * C + col] = x[k];
    }
}

// ---------------------------------------------------------------------------
// forward, pass 2: row stages LR..logN-1, with fused epilogue
// ---------------------------------------------------------------------------
template <int STORE>
__device__ __forceinline__ uint64_t fwd_epilogue(const DevCtx& ctx, const LimbRef& lr, const PrimeConst& pc,
                                                 size_t g, uint64_t v) {
    v = reduce4p(v, pc);
    if constexpr (STORE == FS_PLAIN) {
        return v;
    } else if constexpr (STORE == FS_MODDOWN) {
        const ulonglong2 pinv = ldg2(ctx.md_pinv, lr.prime);
        uint64_t r = mul_shoup(sub_mod(lr.in2[g], v, pc.p), pinv.x, pinv.y, pc.p);
        if (lr.in3) r = add_mod(r, lr.in3[g], pc.p);
        return r;
    } else if constexpr (STORE == FS_RESCALE) {
        const ulonglong2 qi = ldg2(ctx.rs_qinv, (size_t)lr.level * ctx.L + lr.prime);
        return mul_shoup(sub_mod(lr.in2[g], v, pc.p), qi.x, qi.y, pc.p);
    } else {  // FS_MDRS
        const ulonglong2 pinv = ldg2(ctx.md_pinv, lr.prime);
        const ulonglong2 qi = ldg2(ctx.rs_qinv, (size_t)lr.level * ctx.L + lr.prime);
        const uint64_t u = add_mod(lr.in3[g], mul_shoup(lr.in2[g], pinv.x, pinv.y, pc.p), pc.p);
        return mul_shoup(sub_mod(u, v, pc.p), qi.x, qi.y, pc.p);
    }
}

// Row passes keep each row in shared memory padded by one word per 16, so
// that both the strided (k*16 + th) and the contiguous (16*th + k) register
// mappings hit 16 distinct bank pairs.
__device__ __forceinline__ int padi(int r) { return r + (r >> 4); }

template <int LR, int LC, int STORE>
__global__ void __launch_bounds__(256, 2) k_ntt_fwd_rows(const __grid_constant__ DevCtx ctx,
                                                         const __grid_constant__ LimbMap map) {
    constexpr int R = 1 << LR, C = 1 << LC;
    constexpr int CP = C + C / 16;  // padded row stride
    constexpr int TPL = 1 << (LC - 4);
    constexpr int TR = (256 / TPL) < R ? (256 / TPL) : R;
    constexpr int NT = TPL * TR;
    __shared__ __align__(16) uint64_t sm[TR * CP];

    const LimbRef lr = resolve_limb(map, blockIdx.y, ctx.N, ctx.L);
    const PrimeConst pc = ctx.pc[lr.prime];
    const uint64_t* twg = ctx.fwd_tw + (size_t)lr.prime * 2 * ctx.N;

    const int th = threadIdx.x % TPL, rl = threadIdx.x / TPL;
    const int row = blockIdx.x * TR + rl;
    const uint64_t* src = lr.out + (size_t)row * C;
    uint64_t x[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) x[k] = src[th + (k << (LC - 4))];

#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const int kb = 3 - t;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            if (k & (1 << kb)) continue;
            const int r = th + (k << (LC - 4));
            ct_bfly(x[k], x[k | (1 << kb)], ldg2(twg, ((size_t)(R + row) << t) + (r >> (LC - t))), pc.p, pc.two_p);
        }
    }
    uint64_t* srow = sm + rl * CP;
    if constexpr (LC > 4) {
#pragma unroll
        for (int k = 0; k < 16; ++k) srow[padi(th + (k << (LC - 4)))] = x[k];
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 16; ++k) x[k] = srow[padi((th << 4) + k)];
#pragma unroll
        for (int t = 4; t < LC; ++t) {
            const int kb = LC - 1 - t;
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                if (k & (1 << kb)) continue;
                const int r = (th << 4) + k;
                ct_bfly(x[k], x[k | (1 << kb)], ldg2(twg, ((size_t)(R + row) << t) + (r >> (LC - t))), pc.p,
                        pc.two_p);
            }
        }
        // each thread rewrites exactly the slots it read
#pragma unroll
        for (int k = 0; k < 16; ++k) srow[padi((th << 4) + k)] = x[k];
    } else {
#pragma unroll
        for (int k = 0; k < 16; ++k) srow[padi(th + k)] = x[k];
    }
    __syncthreads();
    const size_t base = (size_t)blockIdx.x * TR * C;
#pragma unroll 4
    for (int i = threadIdx.x * 2; i < TR * C; i += NT * 2) {
        const int w = (i / C) * CP + padi(i % C);
        ulonglong2 o;
        o.x = fwd_epilogue<STORE>(ctx, lr, pc, base + i, sm[w]);
        o.y = fwd_epilogue<STORE>(ctx, lr, pc, base + i + 1, sm[w + 1]);
        *reinterpret_cast<ulonglong2*>(lr.out + base + i) = o;
    }
}

// ---------------------------------------------------------------------------
// inverse, pass A: row stages logN-1..LR (GS), with fused prologue
// ---------------------------------------------------------------------------
template <int LOAD>
__device__ __forceinline__ uint64_t inv_prologue(const DevCtx& ctx, const LimbRef& lr, const PrimeConst& pc,
                                                 size_t g) {
    if constexpr (LOAD == IL_PLAIN) {
        return lr.in[g];
    } else if constexpr (LOAD == IL_MUL) {
        return mul_mod(lr.in[g], lr.in2[g], pc);
    } else {  // IL_AXPY_PINV: in + in2 * P^-1
        const ulonglong2 pinv = ldg2(ctx.md_pinv, lr.prime);
        return add_mod(lr.in[g], mul_shoup(lr.in2[g], pinv.x, pinv.y, pc.p), pc.p);
    }
}

template <int LR, int LC, int LOAD>
__global__ void __launch_bounds__(256, 2) k_ntt_inv_rows(const __grid_constant__ DevCtx ctx,
                                                         const __grid_constant__ LimbMap map) {
    constexpr int R = 1 << LR, C = 1 << LC;
    constexpr int CP = C + C / 16;
    constexpr int TPL = 1 << (LC - 4);
    constexpr int TR = (256 / TPL) < R ? (256 / TPL) : R;
    constexpr int NT = TPL * TR;
    __shared__ __align__(16) uint64_t sm[TR * CP];

    const LimbRef lr = resolve_limb(map, blockIdx.y, ctx.N, ctx.L);
    const PrimeConst pc = ctx.pc[lr.prime];
    const uint64_t* twg = ctx.inv_tw + (size_t)lr.prime * 2 * ctx.N;

    const size_t base = (size_t)blockIdx.x * TR * C;
#pragma unroll 4
    for (int i = threadIdx.x * 2; i < TR * C; i += NT * 2) {
        const int w = (i / C) * CP + padi(i % C);
        sm[w] = inv_prologue<LOAD>(ctx, lr, pc, base + i);
        sm[w + 1] = inv_prologue<LOAD>(ctx, lr, pc, base + i + 1);
    }
    __syncthreads();

    const int th = threadIdx.x % TPL, rl = threadIdx.x / TPL;
    const int row = blockIdx.x * TR + rl;
    uint64_t* srow = sm + rl * CP;
    uint64_t x[16];
    if constexpr (LC > 4) {
#pragma unroll
        for (int k = 0; k < 16; ++k) x[k] = srow[padi((th << 4) + k)];
#pragma unroll
        for (int t = LC - 1; t >= 4; --t) {
            const int kb = LC - 1 - t;
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                if (k & (1 << kb)) continue;
                const int r = (th << 4) + k;
                gs_bfly(x[k], x[k | (1 << kb)], ldg2(twg, ((size_t)(R + row) << t) + (r >> (LC - t))), pc.p,
                        pc.two_p);
            }
        }
#pragma unroll
        for (int k = 0; k < 16; ++k) srow[padi((th << 4) + k)] = x[k];
        __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) x[k] = srow[padi(th + (k << (LC - 4)))];
#pragma unroll
    for (int t = 3; t >= 0; --t) {
        const int kb = 3 - t;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            if (k & (1 << kb)) continue;
            const int r = th + (k << (LC - 4));
            gs_bfly(x[k], x[k | (1 << kb)], ldg2(twg, ((size_t)(R + row) << t) + (r >> (LC - t))), pc.p, pc.two_p);
        }
    }
    uint64_t* dst = lr.out + (size_t)row * C;
#pragma unroll
    for (int k = 0; k < 16; ++k) dst[th + (k << (LC - 4))] = x[k];
}

// ---------------------------------------------------------------------------
// inverse, pass B: column stages LR-1..0 (GS), N^-1 and CRT scale folded in
// ---------------------------------------------------------------------------
template <int STORE>
__device__ __forceinline__ const uint64_t* inv_scale_entry(const DevCtx& ctx, const LimbRef& lr) {
    if constexpr (STORE == IS_PLAIN) {
        return ctx.intt_scale + (size_t)lr.prime * 4;
    } else if constexpr (STORE == IS_MODUP) {
        return ctx.modup_scale + ((size_t)lr.level * ctx.L + lr.prime) * 4;
    } else {  // IS_MODDOWN
        return ctx.md_scale + (size_t)(lr.prime - ctx.L) * 4;
    }
}

template <int LR, int LC, int STORE>
__global__ void __launch_bounds__(256, 2) k_ntt_inv_cols(const __grid_constant__ DevCtx ctx,
                                                         const __grid_constant__ LimbMap map) {
    constexpr int R = 1 << LR, C = 1 << LC;
    constexpr int TPL = 1 << (LR - 4);
    constexpr int TC = (256 / TPL) < C ? (256 / TPL) : C;
    constexpr int NT = TPL * TC;
    __shared__ __align__(16) uint64_t sm[R * TC];
    __shared__ ulonglong2 tw[R];

    const LimbRef lr = resolve_limb(map, blockIdx.y, ctx.N, ctx.L);
    const PrimeConst pc = ctx.pc[lr.prime];
    const ulonglong2* twg = reinterpret_cast<const ulonglong2*>(ctx.inv_tw) + (size_t)lr.prime * ctx.N;
    for (int i = threadIdx.x; i < R; i += NT) tw[i] = twg[i];
    const uint64_t* se = inv_scale_entry<STORE>(ctx, lr);
    const ulonglong2 s0 = ldg2(se, 0), s1 = ldg2(se, 1);

    const int c = threadIdx.x % TC, th = threadIdx.x / TC;
    const int col = blockIdx.x * TC + c;
    uint64_t x[16];
    if constexpr (LR > 4) {
#pragma unroll
        for (int k = 0; k < 16; ++k) x[k] = lr.out[(size_t)((th << 4) + k) * C + col];
        __syncthreads();
#pragma unroll
        for (int t = LR - 1; t >= 4; --t) {
            const int kb = LR - 1 - t;
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                if (k & (1 << kb)) continue;
                const int r = (th << 4) + k;
                gs_bfly(x[k], x[k | (1 << kb)], tw[(1 << t) + (r >> (LR - t))], pc.p, pc.two_p);
            }
        }
#pragma unroll
        for (int k = 0; k < 16; ++k) sm[((th << 4) + k) * TC + c] = x[k];
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 16; ++k) x[k] = sm[(th + (k << (LR - 4))) * TC + c];
    } else {
#pragma unroll
        for (int k = 0; k < 16; ++k) x[k] = lr.out[(size_t)(th + k) * C + col];
        __syncthreads();
    }
#pragma unroll
    for (int t = 3; t >= 1; --t) {
        const int kb = 3 - t;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            if (k & (1 << kb)) continue;
            const int r = th + (k << (LR - 4));
            gs_bfly(x[k], x[k | (1 << kb)], tw[(1 << t) + (r >> (LR - t))], pc.p, pc.two_p);
        }
    }
    // last stage (twiddle index 1) with the N^-1 * scale fold
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const uint64_t X = x[k], Y = x[k + 8];
        x[k] = mul_shoup(X + Y, s0.x, s0.y, pc.p);
        x[k + 8] = mul_shoup(X - Y + pc.two_p, s1.x, s1.y, pc.p);
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) lr.out[(size_t)(th + (k << (LR - 4))) * C + col] = x[k];
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
template <int LR, int LC>
static void launch_fwd(const DevCtx& ctx, const LimbMap& map, int load, int store, cudaStream_t st) {
    constexpr int R = 1 << LR, C = 1 << LC;
    constexpr int TC = (256 >> (LR - 4)) < C ? (256 >> (LR - 4)) : C;
    constexpr int TR = (256 >> (LC - 4)) < R ? (256 >> (LC - 4)) : R;
    dim3 g1(C / TC, map.total), g2(R / TR, map.total);
    const int nt1 = (1 << (LR - 4)) * TC, nt2 = (1 << (LC - 4)) * TR;
    if (load == FL_SWITCHMOD)
        k_ntt_fwd_cols<LR, LC, FL_SWITCHMOD><<<g1, nt1, 0, st>>>(ctx, map);
    else
        k_ntt_fwd_cols<LR, LC, FL_PLAIN><<<g1, nt1, 0, st>>>(ctx, map);
    switch (store) {
        case FS_MODDOWN: k_ntt_fwd_rows<LR, LC, FS_MODDOWN><<<g2, nt2, 0, st>>>(ctx, map); break;
        case FS_RESCALE: k_ntt_fwd_rows<LR, LC, FS_RESCALE><<<g2, nt2, 0, st>>>(ctx, map); break;
        case FS_MDRS: k_ntt_fwd_rows<LR, LC, FS_MDRS><<<g2, nt2, 0, st>>>(ctx, map); break;
        default: k_ntt_fwd_rows<LR, LC, FS_PLAIN><<<g2, nt2, 0, st>>>(ctx, map); break;
    }
}

template <int LR, int LC>
static void launch_inv(const DevCtx& ctx, const LimbMap& map, int load, int store, cudaStream_t st) {
    constexpr int R = 1 << LR, C = 1 << LC;
    constexpr int TC = (256 >> (LR - 4)) < C ? (256 >> (LR - 4)) : C;
    constexpr int TR = (256 >> (LC - 4)) < R ? (256 >> (LC - 4)) : R;
    dim3 g1(C / TC, map.total), g2(R / TR, map.total);
    const int nt1 = (1 << (LR - 4)) * TC, nt2 = (1 << (LC - 4)) * TR;
    switch (load) {
        case IL_MUL: k_ntt_inv_rows<LR, LC, IL_MUL><<<g2, nt2, 0, st>>>(ctx, map); break;
        case IL_AXPY_PINV: k_ntt_inv_rows<LR, LC, IL_AXPY_PINV><<<g2, nt2, 0, st>>>(ctx, map); break;
        default: k_ntt_inv_rows<LR, LC, IL_PLAIN><<<g2, nt2, 0, st>>>(ctx, map); break;
    }
    switch (store) {
        case IS_MODUP: k_ntt_inv_cols<LR, LC, IS_MODUP><<<g1, nt1, 0, st>>>(ctx, map); break;
        case IS_MODDOWN: k_ntt_inv_cols<LR, LC, IS_MODDOWN><<<g1, nt1, 0, st>>>(ctx, map); break;
        default: k_ntt_inv_cols<LR, LC, IS_PLAIN><<<g1, nt1, 0, st>>>(ctx, map); break;
    }
}

static std::atomic<uint64_t> g_launches{0};
uint64_t launch_count() { return g_launches.load(); }
void count_launches(int n) { g_launches.fetch_add((uint64_t)n); }

bool ntt_supported(int logN) { return logN >= 8 && logN <= 16; }

void ntt_forward(const DevCtx& ctx, const LimbMap& map, int load, int store, cudaStream_t st) {
    if (map.total <= 0) return;
    count_launches(2);
    switch (ctx.logN) {
        case 8: launch_fwd<4, 4>(ctx, map, load, store, st); break;
        case 9: launch_fwd<4, 5>(ctx, map, load, store, st); break;
        case 10: launch_fwd<5, 5>(ctx, map, load, store, st); break;
        case 11: launch_fwd<5, 6>(ctx, map, load, store, st); break;
        case 12: launch_fwd<6, 6>(ctx, map, load, store, st); break;
        case 13: launch_fwd<6, 7>(ctx, map, load, store, st); break;
        case 14: launch_fwd<7, 7>(ctx, map, load, store, st); break;
        case 15: launch_fwd<7, 8>(ctx, map, load, store, st); break;
        case 16: launch_fwd<8, 8>(ctx, map, load, store, st); break;
        default: break;
    }
}

void ntt_inverse(const DevCtx& ctx, const LimbMap& map, int load, int store, cudaStream_t st) {
    if (map.total <= 0) return;
    count_launches(2);
    switch (ctx.logN) {
        case 8: launch_inv<4, 4>(ctx, map, load, store, st); break;
        case 9: launch_inv<4, 5>(ctx, map, load, store, st); break;
        case 10: launch_inv<5, 5>(ctx, map, load, store, st); break;
        case 11: launch_inv<5, 6>(ctx, map, load, store, st); break;
        case 12: launch_inv<6, 6>(ctx, map, load, store, st); break;
        case 13: launch_inv<6, 7>(ctx, map, load, store, st); break;
        case 14: launch_inv<7, 7>(ctx, map, load, store, st); break;
        case 15: launch_inv<7, 8>(ctx, map, load, store, st); break;
        case 16: launch_inv<8, 8>(ctx, map, load, store, st); break;
        default: break;
    }
}

}  // namespace fides
