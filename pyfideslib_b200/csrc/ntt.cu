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
//   * Each thread owns 16 elements of one column/row in registers and runs up
//     to 4 butterfly stages on them (radix-16 register blocking); the next
//     group of stages follows one shared-memory exchange.  Column passes move
//     16 consecutive columns per CTA (128-byte coalesced rows); row passes
//     stage through padded shared memory so that global stores are coalesced.
//   * In a group of stages the twiddle of a butterfly only depends on the
//     high bits of its register index, so every group needs 1+2+4+8 = 15
//     twiddles per thread; they are fetched together (16-byte (w, Shoup)
//     pairs) before the butterflies, keeping 15 loads in flight instead of
//     one dependent load per butterfly.
//   * Harvey lazy butterflies: values stay in [0,4p) (forward) or [0,2p)
//     (inverse) and are reduced once at the end.
//   * For primes below 2^50 the butterflies can instead run on the FP64
//     pipes with residues held exactly as integer-valued doubles (products
//     split into h + l by an FMA, quotients from a precomputed w / p); the
//     integer pipes are the bottleneck of the 64-bit Shoup butterflies and
//     the FP64 pipes would otherwise stay idle.  Results are the same
//     canonical residues; the autotuner picks the arithmetic per context.
//   * Prologues/epilogues fuse the surrounding element-wise work (products of
//     two inputs, ModDown/Rescale combinations, per-limb CRT scalings).  The
//     mode is a per-segment field, so one launch can mix limbs with different
//     fusions.
#include <atomic>

#include "fp64.cuh"
#include "kernels.hpp"

namespace fides {

// Forward butterfly.  MODE 0 is Harvey's form: X kept in [0, 4p) with one
// conditional subtraction per butterfly.  For primes below 2^57, MODE 1 drops
// the subtraction: each stage adds at most 2p to the bound, so after the 16
// stages of a 2^16 transform values stay below 33p < 2^63 (the Shoup product
// accepts any 64-bit input) and one reduction in the epilogue suffices.
// MODE 3 (primes below 2^56) also forms the Shoup quotient from three of the
// four 32x32 partial products: it is low by at most 2, the product lands in
// [0, 4p), and the bound after 16 stages is 65p < 2^63.
constexpr uint64_t kLazyPrimeBound = 1ull << 57;
constexpr uint64_t kApproxPrimeBound = 1ull << 56;

// floor(a * b / 2^64) - d with d in {0, 1, 2}
__device__ __forceinline__ uint64_t mulhi64_approx(uint64_t a, uint64_t b) {
    const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32), b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
    uint64_t h = (uint64_t)a1 * b1;
    h += __umulhi(a1, b0);
    h += __umulhi(a0, b1);
    return h;
}

// ---- double-precision butterflies (MODE 4, primes below 2^50) ----
// Residues are held exactly as signed integer-valued doubles (bit patterns in
// the uint64_t registers) and every product runs on the FP64 pipes, which the
// integer butterflies leave idle.  With w < p and wq = fl(w / p):
//   h = fl(y w), l = fma(y, w, -h)          y w = h + l exactly
//   q = rint(y wq)                          |q - y w / p| <= 1/2 + |y| 2^-54
//   t = fma(-q, p, h) + l = y w - q p       exact, |t| <= p (1/2 + |y| 2^-54)
// (rint through the 1.5 * 2^52 shift, valid for |y wq| < 2^51; the fma of
// the shift rounds the exact product).  Starting from residues below p,
// alternating plain stages with stages that first centre X (x - rint(x/p) p,
// |.| <= p/2 + 1) keeps every value below 1.7p < 2^51, so the bounds above
// hold at every stage and all sums are exact.  The column pass hands these
// doubles to the row pass as they are; the row pass centres on the other
// stage parity (MODE 6) and ends with a floor reduction against 1/p rounded
// up, which is exact for values in (-2p, 2p).
// forward butterfly on doubles; RED centres X first
template <bool RED>
__device__ __forceinline__ void ct_bfly_fp(uint64_t& X, uint64_t& Y, const ulonglong2 w, const double p,
                                           const double pinv) {
    double x = as_f64(X);
    if constexpr (RED) x = fp_center(x, p, pinv);
    const double t = fp_mulw(as_f64(Y), as_f64(w.x), as_f64(w.y), p);
    X = as_u64(__dadd_rn(x, t));
    Y = as_u64(__dsub_rn(x, t));
}

// inverse (Gentleman-Sande) butterfly on doubles: the sum is centred every
// stage, the difference goes through the product, so every value stays
// below 0.58p and |x - y| < 1.2p keeps the product's quotient within range
__device__ __forceinline__ void gs_bfly_fp(uint64_t& X, uint64_t& Y, const ulonglong2 w, const double p,
                                           const double pinv) {
    const double x = as_f64(X), y = as_f64(Y);
    X = as_u64(fp_center(__dadd_rn(x, y), p, pinv));
    Y = as_u64(fp_mulw(__dsub_rn(x, y), as_f64(w.x), as_f64(w.y), p));
}

template <int MODE>
__device__ __forceinline__ void ct_bfly(uint64_t& X, uint64_t& Y, const ulonglong2 w, const uint64_t p,
                                        const uint64_t two_p) {
    if constexpr (MODE == 3) {
        const uint64_t t = Y * w.x - mulhi64_approx(Y, w.y) * p;  // [0, 4p)
        const uint64_t x = X;
        X = x + t;
        Y = x - t + 2 * two_p;
    } else {
        const uint64_t x = MODE == 1 ? X : csub(X, two_p);
        const uint64_t t = mul_shoup_lazy(Y, w.x, w.y, p);
        X = x + t;
        Y = x - t + two_p;
    }
}

__device__ __forceinline__ void gs_bfly(uint64_t& X, uint64_t& Y, const ulonglong2 w, const uint64_t p,
                                        const uint64_t two_p) {
    const uint64_t s = csub(X + Y, two_p);
    const uint64_t d = X - Y + two_p;
    X = s;
    Y = mul_shoup_lazy(d, w.x, w.y, p);
}

__device__ __forceinline__ uint64_t reduce4p(uint64_t v, const PrimeConst& c) { return csub(csub(v, c.two_p), c.p); }
// canonical residue of any forward-NTT output (below 33p, see ct_bfly)
__device__ __forceinline__ uint64_t reduce_fwd(uint64_t v, const PrimeConst& c) {
    return csub(reduce64_lazy(v, c), c.p);
}

__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

__device__ __forceinline__ ulonglong2 ldg2(const uint64_t* base, size_t idx) {
    return __ldg(reinterpret_cast<const ulonglong2*>(base) + idx);
}

// A stage whose register partner bit is kb pairs k and k | (1 << kb) and uses
// twiddle  (B << t) + (th_hi << (3 - kb)) + (k >> (kb + 1)),  t = t_of_kb0 - kb;
// its 8 >> kb twiddles sit at offset (8 >> kb) - 1 of the group's block.
__device__ __forceinline__ constexpr int tw_off(int kb) { return (8 >> kb) - 1; }

template <int KB, class Tab>
__device__ __forceinline__ void load_stage_tw(ulonglong2 (&w)[15], Tab tab, int t_of_kb0, size_t B, int th_hi) {
    const int t = t_of_kb0 - KB;
    const size_t base = (B << t) + ((size_t)th_hi << (3 - KB));
#pragma unroll
    for (int g = 0; g < (8 >> KB); ++g) w[tw_off(KB) + g] = tab(base + g);
}

// Twiddle-fetch policy of a group: PF = true fetches the 15 twiddles of the
// whole group up front (more loads in flight, +30 registers); PF = false
// fetches each stage's twiddles right before the stage (fewer registers,
// higher occupancy).  The autotuner picks per context.
// p and two_p carry the prime's constants for the butterfly mode: (p, 2p) for
// the integer modes, the bit patterns of the doubles (p, 1/p rounded up) for
// MODEs 4 to 6.  POS counts the stages of the group: MODE 4 (column pass, fed
// residues below p) centres X on odd ones and leaves values below 1.7p;
// MODE 6 (row pass, fed those doubles unconverted) centres X on even ones,
// so that its first stage already brings X down to p/2 and every value stays
// below 1.7p < 2^51.
template <int MODE, int POS>
__device__ __forceinline__ void bfly(uint64_t& X, uint64_t& Y, const ulonglong2 w, uint64_t p, uint64_t two_p) {
    if constexpr (MODE == 7)
        ct_bfly_fp<true>(X, Y, w, as_f64(p), as_f64(two_p));
    else if constexpr (MODE == 4)
        ct_bfly_fp<(POS & 1) != 0>(X, Y, w, as_f64(p), as_f64(two_p));
    else if constexpr (MODE == 6)
        ct_bfly_fp<(POS & 1) == 0>(X, Y, w, as_f64(p), as_f64(two_p));
    else if constexpr (MODE == 5)
        gs_bfly_fp(X, Y, w, as_f64(p), as_f64(two_p));
    else if constexpr (MODE != 2)
        ct_bfly<MODE>(X, Y, w, p, two_p);
    else
        gs_bfly(X, Y, w, p, two_p);
}

template <int KB, int KB_END, int STEP, bool PF, int MODE, int POS, class Tab>
__device__ __forceinline__ void run_stages(uint64_t (&x)[16], ulonglong2 (&w)[15], Tab tab, int t_of_kb0, size_t B,
                                           int th_hi, uint64_t p, uint64_t two_p) {
    if constexpr (!PF) load_stage_tw<KB>(w, tab, t_of_kb0, B, th_hi);
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        if (k & (1 << KB)) continue;
        bfly<MODE, POS>(x[k], x[k | (1 << KB)], w[tw_off(KB) + (k >> (KB + 1))], p, two_p);
    }
    if constexpr (KB != KB_END)
        run_stages<KB + STEP, KB_END, STEP, PF, MODE, POS + 1>(x, w, tab, t_of_kb0, B, th_hi, p, two_p);
}

// All twiddles of a group (stages with partner bits KB_FIRST..KB_LAST) into
// registers.
template <int KB_FIRST, int KB_LAST, class Tab>
__device__ __forceinline__ void load_group_tw(ulonglong2 (&w)[15], Tab tab, int t_of_kb0, size_t B, int th_hi) {
#pragma unroll
    for (int kb = 0; kb < 4; ++kb) {
        if ((kb < KB_FIRST && kb < KB_LAST) || (kb > KB_FIRST && kb > KB_LAST)) continue;
        const int t = t_of_kb0 - kb;
        const size_t base = (B << t) + ((size_t)th_hi << (3 - kb));
#pragma unroll
        for (int g = 0; g < (8 >> kb); ++g) w[tw_off(kb) + g] = tab(base + g);
    }
}

// MODE: 0 forward, 1 forward without the per-butterfly reduction, 2 inverse,
// 3 forward lazy with the approximate Shoup quotient, 4 forward on doubles
// (column pass), 5 inverse on doubles, 6 forward on doubles (row pass)
template <int KB_FIRST, int KB_LAST, bool PF, int MODE, class Tab>
__device__ __forceinline__ void run_group(uint64_t (&x)[16], Tab tab, int t_of_kb0, size_t B, int th_hi, uint64_t p,
                                          uint64_t two_p) {
    ulonglong2 w[15];
    constexpr int STEP = KB_FIRST > KB_LAST ? -1 : 1;
    if constexpr (PF) load_group_tw<KB_FIRST, KB_LAST>(w, tab, t_of_kb0, B, th_hi);
    run_stages<KB_FIRST, KB_LAST, STEP, PF, MODE, 0>(x, w, tab, t_of_kb0, B, th_hi, p, two_p);
}

// Forward group in the mode of this limb's prime (uniform per CTA); ROWS
// selects the row pass's centring schedule for the double-precision mode.
template <int KF, int KL, bool PF, bool AQ, bool FP, bool ROWS, class Tab>
__device__ __forceinline__ void fwd_group(int fmode, uint64_t (&x)[16], Tab tab, int t_of_kb0, size_t B, int th_hi,
                                          uint64_t p, uint64_t two_p) {
    if constexpr (FP) {
        if (fmode == 4) {
            run_group<KF, KL, PF, ROWS ? 6 : 4>(x, tab, t_of_kb0, B, th_hi, p, two_p);
            return;
        }
    }
    if constexpr (AQ) {
        if (fmode == 3) {
            run_group<KF, KL, PF, 3>(x, tab, t_of_kb0, B, th_hi, p, two_p);
            return;
        }
    } else {
        if (fmode == 1) {
            run_group<KF, KL, PF, 1>(x, tab, t_of_kb0, B, th_hi, p, two_p);
            return;
        }
    }
    run_group<KF, KL, PF, 0>(x, tab, t_of_kb0, B, th_hi, p, two_p);
}

template <bool AQ, bool FP>
__device__ __forceinline__ int fwd_mode(uint64_t p) {
    if constexpr (FP)
        if (p < kFpPrimeBound) return 4;
    if constexpr (AQ) return p < kApproxPrimeBound ? 3 : 0;
    return p < kLazyPrimeBound ? 1 : 0;
}

// Per-prime butterfly constants of a mode (see run_stages).
struct FwdK {
    uint64_t k0, k1;
};
__device__ __forceinline__ FwdK fwd_consts(int mode, const PrimeConst& pc) {
    if (mode == 4 || mode == 5) return {as_u64(__ull2double_rn(pc.p)), pc.pinv_f64};
    return {pc.p, pc.two_p};
}

template <bool FP>
__device__ __forceinline__ int inv_mode(uint64_t p) {
    if constexpr (FP)
        if (p < kFpPrimeBound) return 5;
    return 2;
}

// Inverse group in the mode of this limb's prime (uniform per CTA).
template <int KF, int KL, bool PF, bool FP, class Tab>
__device__ __forceinline__ void inv_group(int imode, uint64_t (&x)[16], Tab tab, int t_of_kb0, size_t B, int th_hi,
                                          uint64_t k0, uint64_t k1) {
    if (FP && imode == 5)
        run_group<KF, KL, PF, 5>(x, tab, t_of_kb0, B, th_hi, k0, k1);
    else
        run_group<KF, KL, PF, 2>(x, tab, t_of_kb0, B, th_hi, k0, k1);
}

// Row-pass twiddles of forward variant 10 (double-precision limbs, C = 256).
// Row r's stage s' (0 <= s' < 8) uses psi_br[((R + r) << s') + h], h < 2^s'.
// The first four stages' 15 twiddles per row are the same for the 16 threads
// of the row: they are staged in shared memory once per CTA, loaded at
// kernel start beside the data.  In the last four, thread th needs
// h = th 2^(s'-4) + g (g < 2^(s'-4)), and since the bit reversals of disjoint
// bit groups add,
//   psi_br[((R + r) << s') + (th << (s'-4)) + g] = D_s' * psi_br[g]  (mod p),
// D_s' = psi_br[((R + r) << s') + (th << (s'-4))]: four table loads per
// thread, issued before the row exchange, and 11 products on the
// FP64 pipes (fp_mulmod, |w| <= 0.875p, quotient companion fl(w * pinv))
// instead of 15 dependent L2 loads per group.  The looser companion widens
// the butterfly's quotient error, so these stages centre X at every stage
// (MODE 7); every value stays below 1.7p.
template <int KB>
__device__ __forceinline__ void sg_stage1(uint64_t (&x)[16], const ulonglong2* g1, uint64_t p, uint64_t pinv) {
    constexpr int t = 3 - KB;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        if (k & (1 << KB)) continue;
        bfly<6, t>(x[k], x[k | (1 << KB)], g1[(1 << t) - 1 + (k >> (KB + 1))], p, pinv);
    }
    if constexpr (KB > 0) sg_stage1<KB - 1>(x, g1, p, pinv);
}

template <int KB>
__device__ __forceinline__ void sg_stage2(uint64_t (&x)[16], const ulonglong2 (&d)[4], const double* gw, uint64_t p,
                                          uint64_t pinv) {
    constexpr int t = 7 - KB, NG = 8 >> KB;
    const ulonglong2 D = d[t - 4];
    ulonglong2 w[NG];
    w[0] = D;
#pragma unroll
    for (int g = 1; g < NG; ++g) {
        const double wd = fp_mulmod(as_f64(D.x), gw[g], as_f64(p), as_f64(pinv));
        w[g].x = as_u64(wd);
        w[g].y = as_u64(__dmul_rn(wd, as_f64(pinv)));
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        if (k & (1 << KB)) continue;
        bfly<7, 0>(x[k], x[k | (1 << KB)], w[k >> (KB + 1)], p, pinv);
    }
    if constexpr (KB > 0) sg_stage2<KB - 1>(x, d, gw, p, pinv);
}

// The inverse row pass of configuration 5 takes its twiddles the same way
// from the inverse table: its first four stages (s' = 7..4) form the
// per-thread ones from D_s' and psi^-1_br[g], its last four (s' = 3..0)
// read the row's 15 from shared memory.  The GS sums are centred at every
// stage already; the differences stay below 1.6p.
template <int KB>
__device__ __forceinline__ void sg_inv_stageA(uint64_t (&x)[16], const ulonglong2 (&d)[4], const double* gw,
                                              uint64_t p, uint64_t pinv) {
    constexpr int t = 7 - KB, NG = 8 >> KB;
    const ulonglong2 D = d[t - 4];
    ulonglong2 w[NG];
    w[0] = D;
#pragma unroll
    for (int g = 1; g < NG; ++g) {
        const double wd = fp_mulmod(as_f64(D.x), gw[g], as_f64(p), as_f64(pinv));
        w[g].x = as_u64(wd);
        w[g].y = as_u64(__dmul_rn(wd, as_f64(pinv)));
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        if (k & (1 << KB)) continue;
        bfly<5, 0>(x[k], x[k | (1 << KB)], w[k >> (KB + 1)], p, pinv);
    }
    if constexpr (KB < 3) sg_inv_stageA<KB + 1>(x, d, gw, p, pinv);
}

template <int KB>
__device__ __forceinline__ void sg_inv_stageB(uint64_t (&x)[16], const ulonglong2* g1, uint64_t p, uint64_t pinv) {
    constexpr int t = 3 - KB;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        if (k & (1 << KB)) continue;
        bfly<5, 0>(x[k], x[k | (1 << KB)], g1[(1 << t) - 1 + (k >> (KB + 1))], p, pinv);
    }
    if constexpr (KB < 3) sg_inv_stageB<KB + 1>(x, g1, p, pinv);
}

// Tile geometry shared by kernels and launchers.
template <int LR, int LC>
struct Geo {
    static constexpr int R = 1 << LR, C = 1 << LC;
    static constexpr int TPC = 1 << (LR - 4);                       // threads per column
    static constexpr int TC = (256 / TPC) < C ? (256 / TPC) : C;    // columns per CTA
    static constexpr int NTC = TPC * TC;
    static constexpr int TPR = 1 << (LC - 4);                       // threads per row
    static constexpr int TR = (256 / TPR) < R ? (256 / TPR) : R;    // rows per CTA
    static constexpr int NTR = TPR * TR;
    static constexpr int CP = C + C / 16;                           // padded row stride
};

// ---------------------------------------------------------------------------
// forward, pass 1: column stages 0..LR-1
// ---------------------------------------------------------------------------
template <int LR, int LC, int MINB, bool PF, bool AQ, bool FP>
__global__ void __launch_bounds__(256, MINB) k_ntt_fwd_cols(const __grid_constant__ DevCtx ctx,
                                                            const __grid_constant__ LimbMap map) {
    using G = Geo<LR, LC>;
    constexpr int C = G::C, TC = G::TC;
    __shared__ __align__(16) uint64_t sm[G::R * TC];
    __shared__ ulonglong2 tws[G::R];

    const LimbRef lr = resolve_limb(map, blockIdx.z, blockIdx.y, ctx.N, ctx.L);
    const PrimeConst pc = ctx.pc[lr.prime];
    const int fmode = fwd_mode<AQ, FP>(pc.p);
    const FwdK kk = fwd_consts(fmode, pc);
    const ulonglong2* twg =
        reinterpret_cast<const ulonglong2*>(fmode == 4 ? ctx.fwd_twf : ctx.fwd_tw) + (size_t)lr.prime * ctx.N;
    for (int i = threadIdx.x; i < G::R; i += G::NTC) tws[i] = twg[i];

    const int c = threadIdx.x % TC, th = threadIdx.x / TC;
    const int col = blockIdx.x * TC + c;
    uint64_t x[16];
    if (lr.lmode == FL_SWITCHMOD) {
        const uint64_t om = ctx.pc[lr.level].p;
#pragma unroll
        for (int k = 0; k < 16; ++k) x[k] = switch_modulus(lr.in[(size_t)(th + (k << (LR - 4))) * C + col], om, pc);
    } else {
#pragma unroll
        for (int k = 0; k < 16; ++k) x[k] = lr.in[(size_t)(th + (k << (LR - 4))) * C + col];
    }
    __syncthreads();
    auto tab = [&](size_t i) { return tws[i]; };
    if (FP && fmode == 4) {
#pragma unroll
        for (int k = 0; k < 16; ++k) x[k] = fp_from_u(x[k]);
    }
    // stages 0..3: r = th + (k << (LR - 4)), twiddle (1 << t) + (k >> (4 - t))
    fwd_group<3, 0, PF, AQ, FP, false>(fmode, x, tab, 3, 1, 0, kk.k0, kk.k1);
    if constexpr (LR > 4) {
#pragma unroll
        for (int k = 0; k < 16; ++k) sm[(th + (k << (LR - 4))) * TC + c] = x[k];
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 16; ++k) x[k] = sm[((th << 4) + k) * TC + c];
        // stages 4..LR-1: r = 16 th + k
        fwd_group<LR - 5, 0, PF, AQ, FP, false>(fmode, x, tab, LR - 1, 1, th, kk.k0, kk.k1);
    }
    // double-precision limbs leave as doubles below 1.7p; the row pass
    // continues on them without converting
    if constexpr (LR > 4) {
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
// v is the lazy butterfly output (canonical already when CANON, the
// double-precision path)
template <bool CANON>
__device__ __forceinline__ uint64_t fwd_epilogue(const DevCtx& ctx, const LimbRef& lr, const PrimeConst& pc, size_t g,
                                                 uint64_t v) {
    if constexpr (!CANON) v = reduce_fwd(v, pc);
    switch (lr.smode) {
        case FS_MODDOWN: {
            const ulonglong2 pinv = ldg2(ctx.md_pinv, lr.prime);
            uint64_t r = mul_shoup(sub_mod(lr.in2[g], v, pc.p), pinv.x, pinv.y, pc.p);
            if (lr.in3) r = add_mod(r, lr.in3[g], pc.p);
            return r;
        }
        case FS_RESCALE: {
            const ulonglong2 qi = ldg2(ctx.rs_qinv, (size_t)lr.level * ctx.L + lr.prime);
            return mul_shoup(sub_mod(lr.in2[g], v, pc.p), qi.x, qi.y, pc.p);
        }
        case FS_MDRS: {
            const ulonglong2 pinv = ldg2(ctx.md_pinv, lr.prime);
            const ulonglong2 qi = ldg2(ctx.rs_qinv, (size_t)lr.level * ctx.L + lr.prime);
            const uint64_t u = add_mod(lr.in3[g], mul_shoup(lr.in2[g], pinv.x, pinv.y, pc.p), pc.p);
            return mul_shoup(sub_mod(u, v, pc.p), qi.x, qi.y, pc.p);
        }
        default:
            return v;
    }
}

// Row passes keep each row in shared memory padded by one word per 16, so
// that both the strided (k*16 + th) and the contiguous (16*th + k) register
// mappings hit 16 distinct bank pairs.
__device__ __forceinline__ int padi(int r) { return r + (r >> 4); }

template <int LR, int LC, int MINB, bool PF, bool AQ, bool FP, bool SG = false>
__global__ void __launch_bounds__(256, MINB) k_ntt_fwd_rows(const __grid_constant__ DevCtx ctx,
                                                            const __grid_constant__ LimbMap map) {
    using G = Geo<LR, LC>;
    constexpr int R = G::R, C = G::C, CP = G::CP, TPR = G::TPR, TR = G::TR, NT = G::NTR;
    constexpr bool kSG = SG && FP && LC == 8;
    __shared__ __align__(16) uint64_t sm[TR * CP];
    __shared__ ulonglong2 s_g1[kSG ? TR * 16 : 1];  // first four stages' twiddles per row, entry 2^t - 1 + g
    __shared__ double s_gw[kSG ? 8 : 1];            // psi_br[g], g < 8

    const LimbRef lr = resolve_limb(map, blockIdx.z, blockIdx.y, ctx.N, ctx.L);
    const PrimeConst pc = ctx.pc[lr.prime];
    const int fmode = fwd_mode<AQ, FP>(pc.p);
    const FwdK kk = fwd_consts(fmode, pc);
    const uint64_t* twg = (fmode == 4 ? ctx.fwd_twf : ctx.fwd_tw) + (size_t)lr.prime * 2 * ctx.N;
    auto tab = [&](size_t i) { return ldg2(twg, i); };

    const int th = threadIdx.x % TPR, rl = threadIdx.x / TPR;
    const int row = blockIdx.x * TR + rl;
    const uint64_t* src = lr.out + (size_t)row * C;
    uint64_t x[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) x[k] = src[th + (k << (LC - 4))];
    if constexpr (kSG) {
        if (fmode == 4) {
            // the twiddle loads go out right behind the data loads
            const ulonglong2* tw2 = reinterpret_cast<const ulonglong2*>(twg);
            for (int e = threadIdx.x; e < TR * 15; e += NT) {
                const int r = e / 15, j = e % 15, t = 31 - __clz(j + 1);
                s_g1[r * 16 + j] = tw2[((size_t)(R + blockIdx.x * TR + r) << t) + (j + 1 - (1 << t))];
            }
            if (threadIdx.x < 8) s_gw[threadIdx.x] = as_f64(tw2[threadIdx.x].x);
            __syncthreads();
        }
    }
    if (lr.smode != FS_PLAIN && lr.in2 && gridDim.y > 1) {
        // the epilogue's operands for this tile (one 128-byte line per thread
        // and operand): start their HBM reads now, under the butterflies.
        // Batched launches only: a single element's grid is about two waves,
        // where the early reads only compete with the row loads (measured
        // 1.5% slower per operation, 0.5% faster batched)
        const size_t tile = (size_t)blockIdx.x * TR * C;
        for (int i = threadIdx.x * 16; i < TR * C; i += NT * 16) {
            prefetch_l2(lr.in2 + tile + i);
            if (lr.in3) prefetch_l2(lr.in3 + tile + i);
        }
    }
    if (kSG && fmode == 4) {
        if constexpr (kSG) sg_stage1<3>(x, s_g1 + rl * 16, kk.k0, kk.k1);
    } else {
        fwd_group<3, 0, PF, AQ, FP, true>(fmode, x, tab, 3, (size_t)(R + row), 0, kk.k0, kk.k1);
    }
    uint64_t* srow = sm + rl * CP;
    if constexpr (LC > 4) {
        // the last four stages' D_s' go out before the row exchange
        ulonglong2 dtw[kSG ? 4 : 1];
        if constexpr (kSG) {
            if (fmode == 4) {
#pragma unroll
                for (int t = 4; t < 8; ++t)
                    dtw[t - 4] = ldg2(twg, ((size_t)(R + row) << t) + ((size_t)th << (t - 4)));
            }
        }
#pragma unroll
        for (int k = 0; k < 16; ++k) srow[padi(th + (k << (LC - 4)))] = x[k];
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 16; ++k) x[k] = srow[padi((th << 4) + k)];
        if (kSG && fmode == 4) {
            if constexpr (kSG) sg_stage2<3>(x, dtw, s_gw, kk.k0, kk.k1);
        } else {
            fwd_group<LC - 5, 0, PF, AQ, FP, true>(fmode, x, tab, LC - 1, (size_t)(R + row), th, kk.k0, kk.k1);
        }
        if (FP && fmode == 4) {
#pragma unroll
            for (int k = 0; k < 16; ++k) x[k] = fp_to_u(as_f64(x[k]), as_f64(kk.k0), as_f64(kk.k1));
        }
        // each thread rewrites exactly the slots it read
#pragma unroll
        for (int k = 0; k < 16; ++k) srow[padi((th << 4) + k)] = x[k];
    } else {
        if (FP && fmode == 4) {
#pragma unroll
            for (int k = 0; k < 16; ++k) x[k] = fp_to_u(as_f64(x[k]), as_f64(kk.k0), as_f64(kk.k1));
        }
#pragma unroll
        for (int k = 0; k < 16; ++k) srow[padi(th + k)] = x[k];
    }
    __syncthreads();
    const size_t base = (size_t)blockIdx.x * TR * C;
    if (FP && fmode == 4) {
#pragma unroll 4
        for (int i = threadIdx.x * 2; i < TR * C; i += NT * 2) {
            const int wi = (i / C) * CP + padi(i % C);
            ulonglong2 o;
            o.x = fwd_epilogue<true>(ctx, lr, pc, base + i, sm[wi]);
            o.y = fwd_epilogue<true>(ctx, lr, pc, base + i + 1, sm[wi + 1]);
            *reinterpret_cast<ulonglong2*>(lr.out + base + i) = o;
        }
    } else {
#pragma unroll 4
        for (int i = threadIdx.x * 2; i < TR * C; i += NT * 2) {
            const int wi = (i / C) * CP + padi(i % C);
            ulonglong2 o;
            o.x = fwd_epilogue<false>(ctx, lr, pc, base + i, sm[wi]);
            o.y = fwd_epilogue<false>(ctx, lr, pc, base + i + 1, sm[wi + 1]);
            *reinterpret_cast<ulonglong2*>(lr.out + base + i) = o;
        }
    }
}

// ---------------------------------------------------------------------------
// forward, pass 2 of the ModUp digits fused with the key-switch inner product
// ---------------------------------------------------------------------------
// One CTA owns a tile of TR rows of output limb m (prime t) of batch element
// b.  First it runs the row stages of every digit limb of prime t that needs
// them (the column pass has already run in place), each into its own
// shared-memory tile; when t lies inside digit d, that digit's value is the
// original evaluation limb instead and is read in the epilogue.  Then one
// epilogue forms  XB[m] = sum_d D_d kb[d][t],  XA[m] = sum_d D_d ka[d][t]
// with the key and own-limb loads of all digits in flight together.  The
// digit limbs never return to HBM in evaluation form and are not read back
// by a separate inner-product kernel.  The prime, and so the twiddles, are
// the same for every digit of the CTA.  Reference: the key-switch dot
// products fused into the NTT epilogue, ksk_dot_fusion / ksk_dot_acc_fusion
// (src/NTTfusions.cuh:295-345) in the KSK_DOT modes of NTT_ (src/NTT.cu:680-700).
//
// Sums: for primes below 2^50 with fp_sums, each product is an exact FP64
// fp_mulmod of operands of magnitude <= p/2 (transformed values centred
// first) or < p (own limb, key): |r| <= 0.69p, and up to 8 digits sum below
// 5.6p < 2^53; otherwise products are reduced on the integer pipes (mul_mod)
// and added mod p.  Results are canonical residues, identical to k_ks_inner's.
template <int LR, int LC>
constexpr size_t ks_tile_words() {
    using G = Geo<LR, LC>;
    return (size_t)G::TR * G::CP;
}

// MB: CTAs per SM the register budget is cut for (2, or 3 for the launch of
// the ciphertext-prime outputs, which hold one digit tile less)
template <int LR, int LC, bool PF, bool AQ, bool FP, bool SG = false, int MB = 2>
__global__ void __launch_bounds__(256, MB) k_ntt_fwd_rows_ks(const __grid_constant__ DevCtx ctx,
                                                             const __grid_constant__ KsFuseArgs a) {
    using G = Geo<LR, LC>;
    constexpr int R = G::R, C = G::C, CP = G::CP, TPR = G::TPR, TR = G::TR, NT = G::NTR;
    constexpr int TILE = TR * C;
    constexpr int TW = TR * CP;
    constexpr bool kSG = SG && FP && LC == 8;
    extern __shared__ __align__(16) uint64_t ks_sm[];  // [digits needing rows][TR][CP]
    __shared__ ulonglong2 s_g1[kSG ? TR * 16 : 1];    // staged row twiddles (variant 9), shared by the digits
    __shared__ double s_gw[kSG ? 8 : 1];

    const int level = a.level, n = level + 1;
    const int m = a.m0 + (int)blockIdx.z;
    const size_t boff = (size_t)blockIdx.y * a.bstride;
    const int t = m < n ? m : ctx.L + (m - n);
    const PrimeConst pc = ctx.pc[t];
    const int fmode = fwd_mode<AQ, FP>(pc.p);
    const FwdK kk = fwd_consts(fmode, pc);
    const uint64_t* twg = (fmode == 4 ? ctx.fwd_twf : ctx.fwd_tw) + (size_t)t * 2 * ctx.N;
    auto tab = [&](size_t i) { return ldg2(twg, i); };

    const int th = threadIdx.x % TPR, rl = threadIdx.x / TPR;
    const int row = blockIdx.x * TR + rl;
    const size_t base = (size_t)blockIdx.x * TILE;
    const size_t kstride = (size_t)(ctx.L + ctx.K) * ctx.N;
    const size_t limb_off = (size_t)t * ctx.N + base;
    const int nd = level / ctx.alpha + 1;
    const int d_own = m < n ? t / ctx.alpha : -1;  // digit holding t (its value is the own limb)
    // variant 9: the row twiddles of this prime and these rows, for every digit
    ulonglong2 dtw[kSG ? 4 : 1];
    if constexpr (kSG) {
        if (fmode == 4) {
#pragma unroll
            for (int tt = 4; tt < 8; ++tt)
                dtw[tt - 4] = ldg2(twg, ((size_t)(R + row) << tt) + ((size_t)th << (tt - 4)));
            const ulonglong2* tw2 = reinterpret_cast<const ulonglong2*>(twg);
            for (int e = threadIdx.x; e < TR * 15; e += NT) {
                const int r = e / 15, j = e % 15, tt = 31 - __clz(j + 1);
                s_g1[r * 16 + j] = tw2[((size_t)(R + blockIdx.x * TR + r) << tt) + (j + 1 - (1 << tt))];
            }
            if (threadIdx.x < 8) s_gw[threadIdx.x] = as_f64(tw2[threadIdx.x].x);
            __syncthreads();
        }
    }

    // the epilogue's key tiles (and own tile) are read once per batch from
    // HBM; start those reads now, under the transforms
    for (int i = threadIdx.x * 16; i < TILE; i += NT * 16) {
        for (int d = 0; d < nd; ++d) {
            prefetch_l2(a.kb + d * kstride + limb_off + i);
            prefetch_l2(a.ka + d * kstride + limb_off + i);
        }
        if (d_own >= 0) prefetch_l2(a.own + boff + limb_off + i);
    }

#pragma unroll 1
    for (int d = 0, slot = 0; d < nd; ++d) {
        if (d == d_own) continue;
        const int lo = d * ctx.alpha, hi = min(lo + ctx.alpha - 1, level), cnt = hi - lo + 1;
        const int md = m < n ? (t < lo ? t : t - cnt) : (n - cnt) + (m - n);
        const uint64_t* src = a.dig + boff + ((size_t)d * a.dig_stride + md) * ctx.N + (size_t)row * C;
        uint64_t* srow = ks_sm + (size_t)slot * TW + rl * CP;
        ++slot;
        uint64_t x[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) x[k] = src[th + (k << (LC - 4))];
        if (kSG && fmode == 4) {
            if constexpr (kSG) sg_stage1<3>(x, s_g1 + rl * 16, kk.k0, kk.k1);
        } else {
            fwd_group<3, 0, PF, AQ, FP, true>(fmode, x, tab, 3, (size_t)(R + row), 0, kk.k0, kk.k1);
        }
        if constexpr (LC > 4) {
#pragma unroll
            for (int k = 0; k < 16; ++k) srow[padi(th + (k << (LC - 4)))] = x[k];
            __syncthreads();
#pragma unroll
            for (int k = 0; k < 16; ++k) x[k] = srow[padi((th << 4) + k)];
            if (kSG && fmode == 4) {
                if constexpr (kSG) sg_stage2<3>(x, dtw, s_gw, kk.k0, kk.k1);
            } else {
                fwd_group<LC - 5, 0, PF, AQ, FP, true>(fmode, x, tab, LC - 1, (size_t)(R + row), th, kk.k0, kk.k1);
            }
            // each thread rewrites exactly the slots it read
#pragma unroll
            for (int k = 0; k < 16; ++k) srow[padi((th << 4) + k)] = x[k];
        } else {
#pragma unroll
            for (int k = 0; k < 16; ++k) srow[padi(th + k)] = x[k];
        }
    }
    __syncthreads();

    const bool fpk = a.fp_sums && pc.p < kFpPrimeBound;
    const double pf = __ull2double_rn(pc.p), pinv = as_f64(pc.pinv_f64);
    uint64_t* xb = a.xb + boff + (size_t)m * ctx.N + base;
    uint64_t* xa = a.xa + boff + (size_t)m * ctx.N + base;
    for (int i = threadIdx.x * 2; i < TILE; i += NT * 2) {
        const int wi = (i / C) * CP + padi(i % C);
        ulonglong2 ob, oa;
        if (fpk) {
            double sb0 = 0, sb1 = 0, sa0 = 0, sa1 = 0;
#pragma unroll
            for (int d = 0; d < 8; ++d) {
                if (d < nd) {
                    const ulonglong2 kb2 = *reinterpret_cast<const ulonglong2*>(a.kb + d * kstride + limb_off + i);
                    const ulonglong2 ka2 = *reinterpret_cast<const ulonglong2*>(a.ka + d * kstride + limb_off + i);
                    double x0, x1;
                    if (d == d_own) {
                        const ulonglong2 o = *reinterpret_cast<const ulonglong2*>(a.own + boff + limb_off + i);
                        x0 = as_f64(fp_from_u(o.x));
                        x1 = as_f64(fp_from_u(o.y));
                    } else {
                        const uint64_t* tile = ks_sm + (size_t)(d_own >= 0 && d > d_own ? d - 1 : d) * TW;
                        if (fmode == 4) {
                            x0 = fp_center(as_f64(tile[wi]), pf, pinv);
                            x1 = fp_center(as_f64(tile[wi + 1]), pf, pinv);
                        } else {
                            x0 = as_f64(fp_from_u(reduce_fwd(tile[wi], pc)));
                            x1 = as_f64(fp_from_u(reduce_fwd(tile[wi + 1], pc)));
                        }
                    }
                    sb0 = __dadd_rn(sb0, fp_mulmod(x0, as_f64(fp_from_u(kb2.x)), pf, pinv));
                    sb1 = __dadd_rn(sb1, fp_mulmod(x1, as_f64(fp_from_u(kb2.y)), pf, pinv));
                    sa0 = __dadd_rn(sa0, fp_mulmod(x0, as_f64(fp_from_u(ka2.x)), pf, pinv));
                    sa1 = __dadd_rn(sa1, fp_mulmod(x1, as_f64(fp_from_u(ka2.y)), pf, pinv));
                }
            }
            ob.x = fp_to_u(fp_center(sb0, pf, pinv), pf, pinv);
            ob.y = fp_to_u(fp_center(sb1, pf, pinv), pf, pinv);
            oa.x = fp_to_u(fp_center(sa0, pf, pinv), pf, pinv);
            oa.y = fp_to_u(fp_center(sa1, pf, pinv), pf, pinv);
        } else {
            Acc128 sb0, sb1, sa0, sa1;
#pragma unroll
            for (int d = 0; d < 8; ++d) {
                if (d < nd) {
                    const ulonglong2 kb2 = *reinterpret_cast<const ulonglong2*>(a.kb + d * kstride + limb_off + i);
                    const ulonglong2 ka2 = *reinterpret_cast<const ulonglong2*>(a.ka + d * kstride + limb_off + i);
                    uint64_t x0, x1;
                    if (d == d_own) {
                        const ulonglong2 o = *reinterpret_cast<const ulonglong2*>(a.own + boff + limb_off + i);
                        x0 = o.x;
                        x1 = o.y;
                    } else {
                        const uint64_t* tile = ks_sm + (size_t)(d_own >= 0 && d > d_own ? d - 1 : d) * TW;
                        if (FP && fmode == 4) {
                            x0 = fp_to_u(as_f64(tile[wi]), as_f64(kk.k0), as_f64(kk.k1));
                            x1 = fp_to_u(as_f64(tile[wi + 1]), as_f64(kk.k0), as_f64(kk.k1));
                        } else {
                            x0 = reduce_fwd(tile[wi], pc);
                            x1 = reduce_fwd(tile[wi + 1], pc);
                        }
                    }
                    sb0.mac(x0, kb2.x);
                    sb1.mac(x1, kb2.y);
                    sa0.mac(x0, ka2.x);
                    sa1.mac(x1, ka2.y);
                }
            }
            ob.x = sb0.reduce(pc);
            ob.y = sb1.reduce(pc);
            oa.x = sa0.reduce(pc);
            oa.y = sa1.reduce(pc);
        }
        *reinterpret_cast<ulonglong2*>(xb + i) = ob;
        *reinterpret_cast<ulonglong2*>(xa + i) = oa;
    }
}

// ---------------------------------------------------------------------------
// inverse, pass A: row stages logN-1..LR (GS), with fused prologue
// ---------------------------------------------------------------------------
// Prologue modes of the inverse row pass (per segment): IL_PLAIN reads `in`,
// IL_MUL the product in*in2, IL_AXPY_PINV in + in2*P^-1.
template <int LR, int LC, int MINB, bool PF, bool FP, bool SG = false>
__global__ void __launch_bounds__(256, MINB) k_ntt_inv_rows(const __grid_constant__ DevCtx ctx,
                                                            const __grid_constant__ LimbMap map) {
    using G = Geo<LR, LC>;
    constexpr int R = G::R, C = G::C, CP = G::CP, TPR = G::TPR, TR = G::TR, NT = G::NTR;
    constexpr bool kSG = SG && FP && LC == 8;
    __shared__ __align__(16) uint64_t sm[TR * CP];
    __shared__ ulonglong2 s_g1[kSG ? TR * 16 : 1];  // last four stages' twiddles per row, entry 2^t - 1 + g
    __shared__ double s_gw[kSG ? 8 : 1];            // psi^-1_br[g], g < 8

    const LimbRef lr = resolve_limb(map, blockIdx.z, blockIdx.y, ctx.N, ctx.L);
    const PrimeConst pc = ctx.pc[lr.prime];
    const int imode = inv_mode<FP>(pc.p);
    const FwdK kk = fwd_consts(imode, pc);
    const uint64_t* twg = (imode == 5 ? ctx.inv_twf : ctx.inv_tw) + (size_t)lr.prime * 2 * ctx.N;
    auto tab = [&](size_t i) { return ldg2(twg, i); };

    const int th = threadIdx.x % TPR, rl = threadIdx.x / TPR;
    const int row = blockIdx.x * TR + rl;
    // all 16 elements of the thread are loaded before any is used, so the
    // 16 global loads (32 with a second operand) are in flight together
    const size_t base = (size_t)blockIdx.x * TR * C;
    constexpr int PER = TR * C / NT;  // elements per thread (16)
    static_assert(PER == 16, "row tile holds 16 elements per thread");
    uint64_t x[16];
    {
        uint64_t v[16];
#pragma unroll
        for (int q = 0; q < PER; ++q) v[q] = lr.in[base + threadIdx.x + q * NT];
        if (lr.lmode == IL_MUL) {
#pragma unroll
            for (int q = 0; q < PER; ++q) v[q] = mul_mod(v[q], lr.in2[base + threadIdx.x + q * NT], pc);
        } else if (lr.lmode == IL_AXPY_PINV) {
            const ulonglong2 pinv = ldg2(ctx.md_pinv, lr.prime);
#pragma unroll
            for (int q = 0; q < PER; ++q)
                v[q] = add_mod(v[q], mul_shoup(lr.in2[base + threadIdx.x + q * NT], pinv.x, pinv.y, pc.p), pc.p);
        }
        if (FP && imode == 5) {
#pragma unroll
            for (int q = 0; q < PER; ++q) v[q] = fp_from_u(v[q]);
        }
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            const int i = threadIdx.x + q * NT;
            sm[(i / C) * CP + padi(i % C)] = v[q];
        }
    }
    // configuration 5: this thread's D_s' and the rows' staged twiddles
    ulonglong2 dtw[kSG ? 4 : 1];
    if constexpr (kSG) {
        if (imode == 5) {
#pragma unroll
            for (int t = 4; t < 8; ++t) dtw[t - 4] = ldg2(twg, ((size_t)(R + row) << t) + ((size_t)th << (t - 4)));
            const ulonglong2* tw2 = reinterpret_cast<const ulonglong2*>(twg);
            for (int e = threadIdx.x; e < TR * 15; e += NT) {
                const int r = e / 15, j = e % 15, t = 31 - __clz(j + 1);
                s_g1[r * 16 + j] = tw2[((size_t)(R + blockIdx.x * TR + r) << t) + (j + 1 - (1 << t))];
            }
            if (threadIdx.x < 8) s_gw[threadIdx.x] = as_f64(tw2[threadIdx.x].x);
        }
    }
    __syncthreads();

    uint64_t* srow = sm + rl * CP;
    if constexpr (LC > 4) {
#pragma unroll
        for (int k = 0; k < 16; ++k) x[k] = srow[padi((th << 4) + k)];
        if (kSG && imode == 5) {
            if constexpr (kSG) sg_inv_stageA<0>(x, dtw, s_gw, kk.k0, kk.k1);
        } else {
            inv_group<0, LC - 5, PF, FP>(imode, x, tab, LC - 1, (size_t)(R + row), th, kk.k0, kk.k1);
        }
#pragma unroll
        for (int k = 0; k < 16; ++k) srow[padi((th << 4) + k)] = x[k];
        __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) x[k] = srow[padi(th + (k << (LC - 4)))];
    if (kSG && imode == 5) {
        if constexpr (kSG) sg_inv_stageB<0>(x, s_g1 + rl * 16, kk.k0, kk.k1);
    } else {
        inv_group<0, 3, PF, FP>(imode, x, tab, 3, (size_t)(R + row), 0, kk.k0, kk.k1);
    }
    // double-precision limbs leave as doubles below 0.6p in magnitude; the
    // column pass continues on them without converting
    uint64_t* dst = lr.out + (size_t)row * C;
#pragma unroll
    for (int k = 0; k < 16; ++k) dst[th + (k << (LC - 4))] = x[k];
}

// ---------------------------------------------------------------------------
// inverse, pass B: column stages LR-1..0 (GS), N^-1 and CRT scale folded in
// ---------------------------------------------------------------------------
__device__ __forceinline__ const uint64_t* inv_scale_entry(const DevCtx& ctx, const LimbRef& lr) {
    switch (lr.smode) {
        case IS_MODUP: return ctx.modup_scale + ((size_t)lr.level * ctx.L + lr.prime) * 4;
        case IS_MODDOWN: return ctx.md_scale + (size_t)(lr.prime - ctx.L) * 4;
        default: return ctx.intt_scale + (size_t)lr.prime * 4;
    }
}

template <int LR, int LC, int MINB, bool PF, bool FP>
__global__ void __launch_bounds__(256, MINB) k_ntt_inv_cols(const __grid_constant__ DevCtx ctx,
                                                            const __grid_constant__ LimbMap map) {
    using G = Geo<LR, LC>;
    constexpr int C = G::C, TC = G::TC;
    __shared__ __align__(16) uint64_t sm[G::R * TC];
    __shared__ ulonglong2 tws[G::R];

    const LimbRef lr = resolve_limb(map, blockIdx.z, blockIdx.y, ctx.N, ctx.L);
    const PrimeConst pc = ctx.pc[lr.prime];
    const int imode = inv_mode<FP>(pc.p);
    const FwdK kk = fwd_consts(imode, pc);
    const ulonglong2* twg =
        reinterpret_cast<const ulonglong2*>(imode == 5 ? ctx.inv_twf : ctx.inv_tw) + (size_t)lr.prime * ctx.N;
    for (int i = threadIdx.x; i < G::R; i += G::NTC) tws[i] = twg[i];
    const uint64_t* se = inv_scale_entry(ctx, lr);
    const ulonglong2 s0 = ldg2(se, 0), s1 = ldg2(se, 1);
    auto tab = [&](size_t i) { return tws[i]; };

    const int c = threadIdx.x % TC, th = threadIdx.x / TC;
    const int col = blockIdx.x * TC + c;
    uint64_t x[16];
    if constexpr (LR > 4) {
#pragma unroll
        for (int k = 0; k < 16; ++k) x[k] = lr.out[(size_t)((th << 4) + k) * C + col];
        __syncthreads();
        inv_group<0, LR - 5, PF, FP>(imode, x, tab, LR - 1, 1, th, kk.k0, kk.k1);
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
    inv_group<0, 2, PF, FP>(imode, x, tab, 3, 1, 0, kk.k0, kk.k1);
    // last stage (twiddle index 1) with the N^-1 * scale fold
    if (FP && imode == 5) {
        const double p = as_f64(kk.k0), a0 = (double)s0.x, a1 = (double)s1.x;
        const double a0q = __ddiv_rn(a0, p), a1q = __ddiv_rn(a1, p);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const double X = as_f64(x[k]), Y = as_f64(x[k + 8]);
            x[k] = fp_to_u(fp_mulw(__dadd_rn(X, Y), a0, a0q, p), p, as_f64(kk.k1));
            x[k + 8] = fp_to_u(fp_mulw(__dsub_rn(X, Y), a1, a1q, p), p, as_f64(kk.k1));
        }
    } else {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint64_t X = x[k], Y = x[k + 8];
            x[k] = mul_shoup(X + Y, s0.x, s0.y, pc.p);
            x[k + 8] = mul_shoup(X - Y + pc.two_p, s1.x, s1.y, pc.p);
        }
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) lr.out[(size_t)(th + (k << (LR - 4))) * C + col] = x[k];
}

// ---------------------------------------------------------------------------
// host launchers and variant dispatch
// ---------------------------------------------------------------------------
static std::atomic<uint64_t> g_launches{0};
uint64_t launch_count() { return g_launches.load(); }
void count_launches(int n) { g_launches.fetch_add((uint64_t)n); }

bool ntt_supported(int logN) { return logN >= 8 && logN <= 16; }

// Forward variants: (min CTAs per SM, twiddle policy, butterflies).
// 0: (2, group prefetch, Harvey / lazy), 1: (3, per-stage, lazy),
// 2: (4, per-stage, lazy), 3: (3, per-stage, approximate quotient),
// 4: (2, group prefetch, approximate quotient), 5 and 6: as 3 and 4 with the
// double-precision butterflies for primes below 2^50, 7: column pass of 5
// with the row pass of 6, 8: column pass of 5 with a row pass at 4 CTAs per
// SM, 9: column pass of 5 with a row pass whose twiddles are staged in
// shared memory or formed from a staged factor (sg_stage1 / sg_stage2, C =
// 256 only; other sizes run variant 5's row pass).  Inverse configurations:
// 5: configuration 3 with the row pass's twiddles staged or formed the
// same way (sg_inv_stageA / sg_inv_stageB); 0 (2, group prefetch),
// 1 (3, per-stage), 2 (4, per-stage), 3 and 4: as 1 and 0 with
// double-precision butterflies for primes below 2^50; ntt_inverse_of(v)
// pairs each forward variant with an inverse configuration of the same
// arithmetic.
int ntt_num_variants() { return 10; }
int ntt_num_inverse_variants() { return 6; }
int ntt_inverse_of(int v) {
    static const int inv[10] = {0, 1, 2, 1, 0, 3, 4, 3, 3, 5};
    return v >= 0 && v < 10 ? inv[v] : 0;
}

template <int LR, int LC, int MINB, bool PF, bool AQ, bool FP>
static void launch_fwd_v(const DevCtx& ctx, const LimbMap& map, cudaStream_t st) {
    using G = Geo<LR, LC>;
    // grid (tiles, batch element, limb): CTAs run x fastest, then y, so the
    // elements of a batch that share a prime run together and its twiddle
    // table is fetched from HBM once per launch rather than once per element
    dim3 g1(G::C / G::TC, map.nb > 0 ? map.nb : 1, map.total), g2(G::R / G::TR, map.nb > 0 ? map.nb : 1, map.total);
    k_ntt_fwd_cols<LR, LC, MINB, PF, AQ, FP><<<g1, G::NTC, 0, st>>>(ctx, map);
    k_ntt_fwd_rows<LR, LC, MINB, PF, AQ, FP><<<g2, G::NTR, 0, st>>>(ctx, map);
}

template <int LR, int LC, int MINB, bool PF, bool FP, bool SG = false>
static void launch_inv_v(const DevCtx& ctx, const LimbMap& map, cudaStream_t st) {
    using G = Geo<LR, LC>;
    // grid (tiles, batch element, limb): CTAs run x fastest, then y, so the
    // elements of a batch that share a prime run together and its twiddle
    // table is fetched from HBM once per launch rather than once per element
    dim3 g1(G::C / G::TC, map.nb > 0 ? map.nb : 1, map.total), g2(G::R / G::TR, map.nb > 0 ? map.nb : 1, map.total);
    k_ntt_inv_rows<LR, LC, MINB, PF, FP, SG><<<g2, G::NTR, 0, st>>>(ctx, map);
    k_ntt_inv_cols<LR, LC, MINB, PF, FP><<<g1, G::NTC, 0, st>>>(ctx, map);
}

// column pass with one configuration, row pass with another (SG2: the row
// pass's staged and formed twiddles, see sg_stage1 / sg_stage2)
template <int LR, int LC, int MB1, bool PF1, int MB2, bool PF2, bool AQ, bool FP, bool SG2 = false>
static void launch_fwd_mix(const DevCtx& ctx, const LimbMap& map, cudaStream_t st) {
    using G = Geo<LR, LC>;
    dim3 g1(G::C / G::TC, map.nb > 0 ? map.nb : 1, map.total), g2(G::R / G::TR, map.nb > 0 ? map.nb : 1, map.total);
    k_ntt_fwd_cols<LR, LC, MB1, PF1, AQ, FP><<<g1, G::NTC, 0, st>>>(ctx, map);
    k_ntt_fwd_rows<LR, LC, MB2, PF2, AQ, FP, SG2><<<g2, G::NTR, 0, st>>>(ctx, map);
}

template <int LR, int LC>
static void launch_fwd(const DevCtx& ctx, const LimbMap& map, cudaStream_t st) {
    switch (ctx.ntt_variant) {
        case 1: launch_fwd_v<LR, LC, 3, false, false, false>(ctx, map, st); break;
        case 2: launch_fwd_v<LR, LC, 4, false, false, false>(ctx, map, st); break;
        case 3: launch_fwd_v<LR, LC, 3, false, true, false>(ctx, map, st); break;
        case 4: launch_fwd_v<LR, LC, 2, true, true, false>(ctx, map, st); break;
        case 5: launch_fwd_v<LR, LC, 3, false, true, true>(ctx, map, st); break;
        case 6: launch_fwd_v<LR, LC, 2, true, true, true>(ctx, map, st); break;
        case 7: launch_fwd_mix<LR, LC, 3, false, 2, true, true, true>(ctx, map, st); break;
        case 8: launch_fwd_mix<LR, LC, 3, false, 4, false, true, true>(ctx, map, st); break;
        case 9: launch_fwd_mix<LR, LC, 3, false, 3, false, true, true, true>(ctx, map, st); break;
        default: launch_fwd_v<LR, LC, 2, true, false, false>(ctx, map, st); break;
    }
}

template <int LR, int LC>
static void launch_inv(const DevCtx& ctx, const LimbMap& map, cudaStream_t st) {
    switch (ctx.intt_variant) {
        case 1: launch_inv_v<LR, LC, 3, false, false>(ctx, map, st); break;
        case 2: launch_inv_v<LR, LC, 4, false, false>(ctx, map, st); break;
        case 3: launch_inv_v<LR, LC, 3, false, true>(ctx, map, st); break;
        case 4: launch_inv_v<LR, LC, 2, true, true>(ctx, map, st); break;
        case 5: launch_inv_v<LR, LC, 3, false, true, true>(ctx, map, st); break;
        default: launch_inv_v<LR, LC, 2, true, false>(ctx, map, st); break;
    }
}

// forward column pass alone (the row pass of the ModUp digits is fused with
// the key-switch inner product)
template <int LR, int LC, int MINB, bool PF, bool AQ, bool FP>
static void launch_fwd_cols_v(const DevCtx& ctx, const LimbMap& map, cudaStream_t st) {
    using G = Geo<LR, LC>;
    dim3 g1(G::C / G::TC, map.nb > 0 ? map.nb : 1, map.total);
    k_ntt_fwd_cols<LR, LC, MINB, PF, AQ, FP><<<g1, G::NTC, 0, st>>>(ctx, map);
}

template <int LR, int LC>
static void launch_fwd_cols(const DevCtx& ctx, const LimbMap& map, cudaStream_t st) {
    switch (ctx.ntt_variant) {
        case 1: launch_fwd_cols_v<LR, LC, 3, false, false, false>(ctx, map, st); break;
        case 2: launch_fwd_cols_v<LR, LC, 4, false, false, false>(ctx, map, st); break;
        case 3: launch_fwd_cols_v<LR, LC, 3, false, true, false>(ctx, map, st); break;
        case 4: launch_fwd_cols_v<LR, LC, 2, true, true, false>(ctx, map, st); break;
        case 5: case 7: case 8: case 9: launch_fwd_cols_v<LR, LC, 3, false, true, true>(ctx, map, st); break;
        case 6: launch_fwd_cols_v<LR, LC, 2, true, true, true>(ctx, map, st); break;
        default: launch_fwd_cols_v<LR, LC, 2, true, false, false>(ctx, map, st); break;
    }
}

template <int LR, int LC, bool PF, bool AQ, bool FP, bool SG = false>
static void launch_rows_ks_v(const DevCtx& ctx, const KsFuseArgs& a, int nb, cudaStream_t st) {
    using G = Geo<LR, LC>;
    const size_t tile = ks_tile_words<LR, LC>() * 8;
    const int n = a.level + 1;
    if constexpr (SG) {
      if (ctx.ks_variant & 8) {
        // split launch: the ciphertext-prime outputs need one tile less (their
        // own digit's value is the input limb) and run at 3 CTAs per SM; the
        // special-prime outputs keep every digit's tile at 2 per SM
        const int nd = a.level / ctx.alpha + 1;
        KsFuseArgs q = a, sp = a;
        q.m0 = 0;
        sp.m0 = n;
        count_launches(1);
        k_ntt_fwd_rows_ks<LR, LC, PF, AQ, FP, SG, 3>
            <<<dim3(G::R / G::TR, nb, n), G::NTR, tile * (size_t)(nd - 1), st>>>(ctx, q);
        k_ntt_fwd_rows_ks<LR, LC, PF, AQ, FP, SG, 2>
            <<<dim3(G::R / G::TR, nb, ctx.K), G::NTR, tile * (size_t)nd, st>>>(ctx, sp);
        return;
      }
    }
    KsFuseArgs all = a;
    all.m0 = 0;
    const size_t smem = tile * (size_t)ctx.dnum;  // opted in by ntt_prepare
    dim3 g(G::R / G::TR, nb, n + ctx.K);
    k_ntt_fwd_rows_ks<LR, LC, PF, AQ, FP, SG><<<g, G::NTR, smem, st>>>(ctx, all);
}

template <int LR, int LC, bool PF, bool AQ, bool FP, bool SG = false>
static void prepare_rows_ks_v(int dnum) {
    const int bytes = (int)(ks_tile_words<LR, LC>() * 8 * (size_t)dnum);
    cudaFuncSetAttribute(k_ntt_fwd_rows_ks<LR, LC, PF, AQ, FP, SG>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if constexpr (SG)
        cudaFuncSetAttribute(k_ntt_fwd_rows_ks<LR, LC, PF, AQ, FP, SG, 3>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

template <int LR, int LC>
static void prepare_rows_ks(const DevCtx& ctx, const LimbMap&, cudaStream_t) {
    prepare_rows_ks_v<LR, LC, true, false, false>(ctx.dnum);
    prepare_rows_ks_v<LR, LC, false, false, false>(ctx.dnum);
    prepare_rows_ks_v<LR, LC, false, true, false>(ctx.dnum);
    prepare_rows_ks_v<LR, LC, true, true, true>(ctx.dnum);
    prepare_rows_ks_v<LR, LC, false, true, true>(ctx.dnum);
    prepare_rows_ks_v<LR, LC, false, true, true, true>(ctx.dnum);
}

bool ntt_rows_keyswitch_supported(const DevCtx& ctx) {
    // one transformed tile per digit in shared memory (at most 227 KB)
    return ctx.dnum <= 6;
}

// the row-pass arithmetic of the context's forward variant (butterfly form,
// twiddle fetch); occupancy is set by the fused kernel's shared memory
template <int LR, int LC>
static void launch_rows_ks(const DevCtx& ctx, const KsFuseArgs& a, int nb, cudaStream_t st) {
    switch (ctx.ntt_variant) {
        case 0: launch_rows_ks_v<LR, LC, true, false, false>(ctx, a, nb, st); break;
        case 1: case 2: launch_rows_ks_v<LR, LC, false, false, false>(ctx, a, nb, st); break;
        case 3: case 4: launch_rows_ks_v<LR, LC, false, true, false>(ctx, a, nb, st); break;
        case 6: case 7: launch_rows_ks_v<LR, LC, true, true, true>(ctx, a, nb, st); break;
        case 9: launch_rows_ks_v<LR, LC, false, true, true, true>(ctx, a, nb, st); break;
        default: launch_rows_ks_v<LR, LC, false, true, true>(ctx, a, nb, st); break;
    }
}

#define FIDES_NTT_DISPATCH(FN)                        \
    switch (ctx.logN) {                               \
        case 8: FN<4, 4>(ctx, map, st); break;        \
        case 9: FN<4, 5>(ctx, map, st); break;        \
        case 10: FN<5, 5>(ctx, map, st); break;       \
        case 11: FN<5, 6>(ctx, map, st); break;       \
        case 12: FN<6, 6>(ctx, map, st); break;       \
        case 13: FN<6, 7>(ctx, map, st); break;       \
        case 14: FN<7, 7>(ctx, map, st); break;       \
        case 15: FN<7, 8>(ctx, map, st); break;       \
        case 16: FN<8, 8>(ctx, map, st); break;       \
        default: return;                              \
    }

void set_modes(LimbMap& map, int lmode, int smode) {
    for (int s = 0; s < map.nseg; ++s) {
        if (lmode >= 0) map.seg[s].lmode = (int8_t)lmode;
        if (smode >= 0) map.seg[s].smode = (int8_t)smode;
    }
}

void ntt_forward(const DevCtx& ctx, const LimbMap& m, int load, int store, cudaStream_t st) {
    if (m.total <= 0) return;
    LimbMap map = m;
    set_modes(map, load, store);
    count_launches(2);
    FIDES_NTT_DISPATCH(launch_fwd)
}

void ntt_prepare(const DevCtx& ctx) {
    const LimbMap map{};
    cudaStream_t st = nullptr;
    FIDES_NTT_DISPATCH(prepare_rows_ks)
}

void ntt_forward_cols(const DevCtx& ctx, const LimbMap& m, int load, cudaStream_t st) {
    if (m.total <= 0) return;
    LimbMap map = m;
    set_modes(map, load, -1);
    count_launches(1);
    FIDES_NTT_DISPATCH(launch_fwd_cols)
}

void ntt_rows_keyswitch(const DevCtx& ctx, const KsFuseArgs& a, int nb, cudaStream_t st) {
    count_launches(1);
    switch (ctx.logN) {
        case 8: launch_rows_ks<4, 4>(ctx, a, nb, st); break;
        case 9: launch_rows_ks<4, 5>(ctx, a, nb, st); break;
        case 10: launch_rows_ks<5, 5>(ctx, a, nb, st); break;
        case 11: launch_rows_ks<5, 6>(ctx, a, nb, st); break;
        case 12: launch_rows_ks<6, 6>(ctx, a, nb, st); break;
        case 13: launch_rows_ks<6, 7>(ctx, a, nb, st); break;
        case 14: launch_rows_ks<7, 7>(ctx, a, nb, st); break;
        case 15: launch_rows_ks<7, 8>(ctx, a, nb, st); break;
        case 16: launch_rows_ks<8, 8>(ctx, a, nb, st); break;
        default: return;
    }
}

void ntt_inverse(const DevCtx& ctx, const LimbMap& m, int load, int store, cudaStream_t st) {
    if (m.total <= 0) return;
    LimbMap map = m;
    set_modes(map, load, store);
    count_launches(2);
    FIDES_NTT_DISPATCH(launch_inv)
}

}  // namespace fides
