// engine.cpp -- the key-switching pipeline over a batch of nb <= kMaxBatch
// elements at one level, queued on the workspace's stream.  A single operation is a batch of one; batches
// share every launch (blockIdx.z or an interleaved grid dimension), so wave
// tails, launch overheads and, for HMult, switching-key reads are amortised.
//
// Reference flow (src/CKKS/LimbPartitionMGPU.cu:573-1748 modup_ksk_moddown_mgpu,
// :458-571 fusedHoistRotate; Ciphertext.cpp:409-622, :756-926, :1053-1226):
//   tensor -> INTT -> ModUp conversion -> NTT -> inner product with the key
//   -> INTT of the special limbs -> ModDown conversion -> NTT -> combine
//   (-> rescale).  Here ModDown and Rescale share their NTT (see
//   moddown_finish) and every step runs once for the whole batch.
#include "context.hpp"

namespace fides {

namespace {

// batch size from which the key switch fused into the digits' row pass wins
// (B200, N=2^16, L=30, dnum=3, ms per batched step unfused / fused: 4 pairs
// 0.986 / 0.997, 8 pairs 1.854 / 1.844, 16 pairs 3.578 / 3.529, 32 pairs
// 7.008 / 6.886)
constexpr int kFuseMinBatch = 8;

LimbSeg seg_ws(const uint64_t* in, uint64_t* out, int count, int nq, int q0, int level, size_t bstride) {
    LimbSeg g{};
    g.in = in;
    g.out = out;
    g.count = count;
    g.skip_lo = count;
    g.nq = nq;
    g.q0 = q0;
    g.level = level;
    g.bstride = bstride;
    return g;
}

// Special limbs of XB / XA -> INTT scaled by (P/p_k)^-1 (in place), and, for
// the fused rescale, INTT(e_l + P^-1 x_l) of both halves into T.
void special_intt(fides_ctx* c, Workspace& w, int level, int nb, bool with_top) {
    const int n = level + 1, N = c->N;
    LimbMap m{};
    m.nb = nb;
    uint64_t* xs[2] = {w.XB, w.XA};
    for (int s = 0; s < 2; ++s) {
        LimbSeg g = seg_ws(xs[s] + (size_t)n * N, xs[s] + (size_t)n * N, c->K, 0, 0, level, w.stride);
        g.lmode = IL_PLAIN;
        g.smode = IS_MODDOWN;
        m.seg[m.nseg++] = g;
        m.total += c->K;
    }
    if (with_top) {
        const uint64_t* es[2] = {w.E0, w.E1};
        for (int s = 0; s < 2; ++s) {
            LimbSeg g = seg_ws(es[s] + (size_t)level * N, w.T + (size_t)s * N, 1, 1, level, level, w.stride);
            g.in2 = xs[s] + (size_t)level * N;
            g.lmode = IL_AXPY_PINV;
            g.smode = IS_PLAIN;
            m.seg[m.nseg++] = g;
            m.total += 1;
        }
    }
    ntt_inverse(c->dev, m, -1, -1, w.st);
}

// ModDown of XB -> out0, XA -> out1 for every element, adding e0/e1 (E0/E1 of
// the workspace) when `add_e`; with `rescale` the result is also rescaled:
//   out = Rescale(e + ModDown(x)), computed as one NTT per output limb.
void moddown_finish(fides_ctx* c, Workspace& w, int level, int nb, uint64_t* const* out0, uint64_t* const* out1,
                    bool add_e, bool rescale) {
    const int n = level + 1, N = c->N, L = c->L;
    special_intt(c, w, level, nb, rescale);
    MdArgs md{};
    md.y[0] = w.XB + (size_t)n * N;
    md.y[1] = w.XA + (size_t)n * N;
    md.w[0] = w.W;
    md.w[1] = w.W + (size_t)L * N;
    md.ttop[0] = rescale ? w.T : nullptr;
    md.ttop[1] = rescale ? w.T + N : nullptr;
    md.bstride = w.stride;
    launch_moddown_conv(c->dev, level, nb, md, w.st);
    LimbMap m{};
    m.nb = nb;
    m.nseg = 2;
    const uint64_t* xs[2] = {w.XB, w.XA};
    const uint64_t* es[2] = {w.E0, w.E1};
    const int nout = rescale ? level : n;
    for (int s = 0; s < 2; ++s) {
        LimbSeg g = seg_ws(w.W + (size_t)s * L * N, nullptr, nout, nout, 0, level, w.stride);
        g.in2 = xs[s];
        g.in3 = add_e ? es[s] : nullptr;
        g.out_tab = (int8_t)(s + 1);
        m.seg[s] = g;
        m.total += nout;
    }
    for (int b = 0; b < nb; ++b) {
        m.bout[0][b] = out0[b];
        m.bout[1][b] = out1[b];
    }
    ntt_forward(c->dev, m, FL_PLAIN, rescale ? FS_MDRS : FS_MODDOWN, w.st);
}

}  // namespace

// Limbs of the ModUp digits in DIG (transformed in place): digit d holds the
// Q primes outside it up to `level`, then the K special primes.
static LimbMap digit_map(fides_ctx* c, Workspace& w, int level, int nb) {
    const int n = level + 1, N = c->N;
    LimbMap dm{};
    dm.nb = nb;
    const int nd = level / c->alpha + 1;
    for (int d = 0; d < nd; ++d) {
        const int lo = d * c->alpha, hi = std::min(lo + c->alpha - 1, level), cnt = hi - lo + 1;
        uint64_t* p = w.DIG + (size_t)d * w.dig_stride * N;
        LimbSeg g = seg_ws(p, p, n - cnt + c->K, n, 0, level, w.stride);
        g.skip_lo = lo;
        g.skip_cnt = cnt;
        dm.seg[dm.nseg++] = g;
        dm.total += g.count;
    }
    return dm;
}

// ModUp conversion + NTT of the digits, from the scaled coefficients in XT.
static void modup_from_xt(fides_ctx* c, Workspace& w, int level, int nb) {
    launch_modup_conv(c->dev, level, nb, w.XT, w.DIG, w.dig_stride, w.stride, w.st);
    ntt_forward(c->dev, digit_map(c, w, level, nb), FL_PLAIN, FS_PLAIN, w.st);
}

void eng_modup(fides_ctx* c, Workspace& w, int level, int nb, const uint64_t* const* x) {
    const int n = level + 1;
    // scaled INTT of each element's input (separate buffers: one segment per
    // element) into its XT
    int done = 0;
    while (done < nb) {
        LimbMap im{};
        im.nb = 1;
        for (; done < nb && im.nseg < kMaxSeg; ++done) {
            im.seg[im.nseg++] = seg_ws(x[done], w.XT + (size_t)done * w.stride, n, n, 0, level, 0);
            im.total += n;
        }
        ntt_inverse(c->dev, im, IL_PLAIN, IS_MODUP, w.st);
    }
    modup_from_xt(c, w, level, nb);
}

void eng_hmult(fides_ctx* c, Workspace& w, int level, int nb, const uint64_t* const* a0, const uint64_t* const* a1,
               const uint64_t* const* b0, const uint64_t* const* b1, uint64_t* const* out0, uint64_t* const* out1,
               bool rescale, const SwitchKey& key) {
    const int n = level + 1;
    TensorArgs ta{};
    for (int b = 0; b < nb; ++b) {
        ta.a0[b] = a0[b];
        ta.a1[b] = a1[b];
        ta.b0[b] = b0[b];
        ta.b1[b] = b1[b];
    }
    ta.e0 = w.E0;
    ta.e1 = w.E1;
    ta.e2 = w.E2;
    ta.bstride = w.stride;
    launch_tensor(c->dev, n, nb, ta, w.st);
    // scaled INTT of E2 (workspace: batch dimension with the element stride)
    LimbMap im{};
    im.nb = nb;
    im.seg[im.nseg++] = seg_ws(w.E2, w.XT, n, n, 0, level, w.stride);
    im.total = n;
    ntt_inverse(c->dev, im, IL_PLAIN, IS_MODUP, w.st);
    // fused inner product: forced (bit 1), or for batches of at least
    // kFuseMinBatch elements (bit 2; a small batch's fused launch is a few
    // waves of long CTAs at 2 per SM and measured slower than the two kernels)
    const bool fuse = ((c->dev.ks_variant & 2) || ((c->dev.ks_variant & 4) && nb >= kFuseMinBatch)) &&
                      ntt_rows_keyswitch_supported(c->dev) && key.a != nullptr;
    if (fuse) {
        // ModUp conversion and the digits' column pass; the row pass runs
        // fused with the inner product, so the digits' evaluation limbs never
        // reach HBM
        launch_modup_conv(c->dev, level, nb, w.XT, w.DIG, w.dig_stride, w.stride, w.st);
        ntt_forward_cols(c->dev, digit_map(c, w, level, nb), FL_PLAIN, w.st);
        KsFuseArgs fa{};
        fa.dig = w.DIG;
        fa.own = w.E2;
        fa.kb = key.b;
        fa.ka = key.a;
        fa.xb = w.XB;
        fa.xa = w.XA;
        fa.dig_stride = w.dig_stride;
        fa.bstride = w.stride;
        fa.level = level;
        fa.fp_sums = c->dev.ks_variant & 1;
        ntt_rows_keyswitch(c->dev, fa, nb, w.st);
        moddown_finish(c, w, level, nb, out0, out1, true, rescale && level > 0);
        return;
    }
    modup_from_xt(c, w, level, nb);
    KsArgs ka{};
    for (int b = 0; b < nb; ++b) {
        ka.own[b] = w.E2 + (size_t)b * w.stride;
        ka.kb[b] = key.b;
        ka.ka[b] = key.a;
        ka.a_seed[b] = key.a ? 0 : uniform_stream(key.a_seed, 0);
    }
    ka.dig = w.DIG;
    ka.xb = w.XB;
    ka.xa = w.XA;
    ka.dig_stride = w.dig_stride;
    ka.bstride = w.stride;
    ka.dig_bstride = w.stride;
    launch_ks_inner(c->dev, level, nb, ka, true, w.st);
    moddown_finish(c, w, level, nb, out0, out1, true, rescale && level > 0);
}

void eng_rotate(fides_ctx* c, Workspace& w, int level, int nb, const uint64_t* const* c0, const uint64_t* const* c1,
                const SwitchKey* const* keys, const uint32_t* galois, uint64_t* const* out0, uint64_t* const* out1,
                bool hoisted) {
    if (hoisted) {
        eng_modup(c, w, level, 1, c1);
    } else {
        eng_modup(c, w, level, nb, c1);
    }
    KsArgs ka{};
    for (int b = 0; b < nb; ++b) {
        ka.own[b] = hoisted ? c1[0] : c1[b];
        ka.c0[b] = hoisted ? c0[0] : c0[b];
        ka.kb[b] = keys[b]->b;
        ka.ka[b] = keys[b]->a;
        ka.a_seed[b] = keys[b]->a ? 0 : uniform_stream(keys[b]->a_seed, 0);
        ka.galois[b] = galois[b];
    }
    ka.dig = w.DIG;
    ka.xb = w.XB;
    ka.xa = w.XA;
    ka.dig_stride = w.dig_stride;
    ka.bstride = w.stride;
    ka.dig_bstride = hoisted ? 0 : w.stride;
    launch_ks_inner(c->dev, level, nb, ka, false, w.st);
    moddown_finish(c, w, level, nb, out0, out1, false, false);
}

void eng_rotate_sum(fides_ctx* c, Workspace& w, int level, int nb, const uint64_t* const* c0,
                    const uint64_t* const* c1, const SwitchKey* const* keys, const uint32_t* galois, int nout,
                    const int* start, uint64_t* const* out0, uint64_t* const* out1) {
    eng_modup(c, w, level, nb, c1);
    KsArgs ka{};
    for (int b = 0; b < nb; ++b) {
        ka.own[b] = c1[b];
        ka.c0[b] = c0[b];
        ka.kb[b] = keys[b]->b;
        ka.ka[b] = keys[b]->a;
        ka.a_seed[b] = keys[b]->a ? 0 : uniform_stream(keys[b]->a_seed, 0);
        ka.galois[b] = galois[b];
    }
    ka.dig = w.DIG;
    ka.xb = w.XB;
    ka.xa = w.XA;
    ka.dig_stride = w.dig_stride;
    ka.bstride = w.stride;
    ka.dig_bstride = w.stride;
    launch_ks_inner(c->dev, level, nb, ka, false, w.st);
    ExtSumArgs sa{};
    sa.nout = nout;
    sa.n = level + 1;
    for (int u = 0; u <= nout; ++u) sa.start[u] = start[u];
    sa.x[0] = w.XB;
    sa.x[1] = w.XA;
    sa.bstride = w.stride;
    launch_ext_sum(c->dev, sa, w.st);
    // one ModDown per output, on a view of the workspace whose element 0 is
    // the output's first element (every per-element buffer moves together)
    for (int u = 0; u < nout; ++u) {
        Workspace v = w;
        const size_t off = (size_t)start[u] * w.stride;
        for (uint64_t** p : {&v.E0, &v.E1, &v.E2, &v.XT, &v.DIG, &v.XB, &v.XA, &v.W, &v.T}) *p += off;
        moddown_finish(c, v, level, 1, out0 + u, out1 + u, false, false);
    }
}

void eng_rotate_groups(fides_ctx* c, Workspace& w, int level, int ngroups, int nper, const uint64_t* const* c0,
                       const uint64_t* const* c1, const SwitchKey* const* keys, const uint32_t* galois,
                       uint64_t* const* out0, uint64_t* const* out1) {
    eng_modup(c, w, level, ngroups, c1);
    const int nb = ngroups * nper;
    KsArgs ka{};
    for (int b = 0; b < nb; ++b) {
        ka.own[b] = c1[b / nper];
        ka.c0[b] = c0[b / nper];
        ka.kb[b] = keys[b]->b;
        ka.ka[b] = keys[b]->a;
        ka.a_seed[b] = keys[b]->a ? 0 : uniform_stream(keys[b]->a_seed, 0);
        ka.galois[b] = galois[b];
        ka.dig_elem[b] = (uint8_t)(b / nper);
    }
    ka.dig = w.DIG;
    ka.xb = w.XB;
    ka.xa = w.XA;
    ka.dig_stride = w.dig_stride;
    ka.bstride = w.stride;
    ka.dig_bstride = w.stride;
    ka.dig_group = nper;
    launch_ks_inner(c->dev, level, nb, ka, false, w.st);
    moddown_finish(c, w, level, nb, out0, out1, false, false);
}

}  // namespace fides
