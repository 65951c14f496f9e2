// api.cpp -- the C ABI of the evaluation core (include/fides_b200.h).
//
// Operations are queued on the context's stream and return immediately;
// downloads synchronise.  Every result is computed into a fresh buffer from
// the stream-ordered pool and then swapped into the output object, so an
// output may alias an input.
#include <algorithm>
#include <cmath>
#include <map>
#include <cstring>
#include <new>

#include "context.hpp"

using namespace fides;

namespace {

struct Guard {
    std::lock_guard<std::recursive_mutex> lk;
    explicit Guard(fides_ctx* c) : lk(c->mu) { cudaSetDevice(c->device); }
};

// Swap a freshly computed buffer into `out` and release the old one.
void commit(fides_ctx* c, fides_ct* out, fides_ct& tmp) {
    ct_quiesce(c, out);
    std::swap(out->buf, tmp.buf);
    std::swap(out->cap, tmp.cap);
    std::swap(out->ring, tmp.ring);
    if (tmp.buf) cudaFreeAsync(tmp.buf, c->st);
    tmp.buf = nullptr;
    tmp.cap = 0;
}

bool valid_ct(const fides_ctx* c, const fides_ct* a) { return a && a->buf && a->level >= 0 && a->level < c->L; }

uint64_t round_to_mod(long double v, uint64_t p) {
    // v rounded to the nearest integer, reduced mod p (|v| < 2^126)
    const bool neg = v < 0;
    long double a = neg ? -v : v;
    a = floorl(a + 0.5L);
    const unsigned __int128 big = (unsigned __int128)a;
    uint64_t r = (uint64_t)(big % p);
    return neg ? (r ? p - r : 0) : r;
}

}  // namespace

extern "C" {

fides_status fides_ctx_create(const fides_params* params, fides_ctx** out) {
    if (!params || !out) return FIDES_BAD_ARG;
    *out = nullptr;
    if (!ntt_supported(params->log_n) || params->num_q < 1 || params->dnum < 1 || params->dnum > params->num_q ||
        (params->p && params->num_p < 1))
        return FIDES_BAD_ARG;
    fides_ctx* c = new (std::nothrow) fides_ctx();
    if (!c) return FIDES_OOM;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || params->device < 0 || params->device >= ndev) {
        cudaGetLastError();
        delete c;
        return FIDES_CUDA_ERR;
    }
    cudaSetDevice(params->device);
    {
        cudaMemPool_t mp;
        if (cudaDeviceGetDefaultMemPool(&mp, params->device) == cudaSuccess) {
            uint64_t thr = UINT64_MAX;
            cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &thr);
        }
    }
    fides_status s = build_context(c, params);
    if (s == FIDES_OK) s = fides_autotune(c, nullptr, nullptr, nullptr);
    if (s != FIDES_OK) {
        free_context(c);
        delete c;
        return s;
    }
    *out = c;
    return FIDES_OK;
}

fides_status fides_generate_moduli(const fides_params* params, uint64_t* q, uint64_t* p, int* num_p_out) {
    if (!params || !q || !p || !num_p_out || !ntt_supported(params->log_n) || params->num_q < 1 || params->dnum < 1 ||
        params->dnum > params->num_q)
        return FIDES_BAD_ARG;
    std::vector<uint64_t> qq, pp;
    if (!select_moduli(params, qq, pp)) return FIDES_BAD_ARG;
    std::copy(qq.begin(), qq.end(), q);
    std::copy(pp.begin(), pp.end(), p);
    *num_p_out = (int)pp.size();
    return FIDES_OK;
}

fides_status fides_ctx_destroy(fides_ctx* ctx) {
    if (!ctx) return FIDES_BAD_ARG;
    free_context(ctx);
    delete ctx;
    return FIDES_OK;
}

fides_status fides_ctx_info(const fides_ctx* ctx, int* log_n, int* num_q, int* num_p, int* dnum, uint64_t* q,
                            uint64_t* p) {
    if (!ctx) return FIDES_BAD_ARG;
    if (log_n) *log_n = ctx->logN;
    if (num_q) *num_q = ctx->L;
    if (num_p) *num_p = ctx->K;
    if (dnum) *dnum = ctx->dnum;
    if (q) memcpy(q, ctx->host.prime.data(), sizeof(uint64_t) * ctx->L);
    if (p) memcpy(p, ctx->host.prime.data() + ctx->L, sizeof(uint64_t) * ctx->K);
    return FIDES_OK;
}

fides_status fides_ctx_synchronize(fides_ctx* ctx) {
    if (!ctx) return FIDES_BAD_ARG;
    Guard g(ctx);
    if (cudaStreamSynchronize(ctx->st) != cudaSuccess || cudaStreamSynchronize(ctx->h2d) != cudaSuccess ||
        cudaStreamSynchronize(ctx->d2h) != cudaSuccess)
        return check_cuda(ctx, "synchronize");
    const fides_status s = check_cuda(ctx, "synchronize");
    return s != FIDES_OK ? s : consume_device_error(ctx);
}

const char* fides_ctx_last_error(const fides_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

fides_status fides_ctx_stream(const fides_ctx* ctx, void** stream) {
    if (!ctx || !stream) return FIDES_BAD_ARG;
    *stream = (void*)ctx->st;
    return FIDES_OK;
}

uint64_t fides_kernel_launches(void) { return fides::launch_count(); }

fides_status fides_autotune(fides_ctx* c, int* variant, float* times_ms, int* num_variants) {
    if (!c) return FIDES_BAD_ARG;
    Guard g(c);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto elapsed = [&]() {
        cudaEventRecord(e1, c->st);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        return ms;
    };
    // Every candidate is timed in three interleaved rounds and keeps its best
    // round, so that clock or cache drift during tuning does not decide.
    constexpr int kRounds = 3, kReps = 3;
    // NTT variants: forward + inverse over the limbs of one element's ModUp
    // digits (up to 3 x (L+K) limbs in the workspace), the shape of the
    // key-switch pipeline's largest transforms; any residues work for timing
    const int nv = ntt_num_variants();
    const int np = std::min(c->L + c->K, kMaxPrimes);
    const int nseg = std::max(1, std::min(c->dnum, 3));
    cudaMemsetAsync(c->ws1.DIG, 0, (size_t)nseg * np * c->limb_bytes(), c->st);
    LimbMap m{};
    for (int sgi = 0; sgi < nseg; ++sgi) {
        LimbMap one = map_single(c->ws1.DIG + (size_t)sgi * np * c->N, c->ws1.DIG + (size_t)sgi * np * c->N, np, np, 0);
        m.seg[m.nseg++] = one.seg[0];
        m.total += np;
    }
    // forward variants and inverse configurations are timed (and chosen)
    // separately, each on one element's digits and on the same shape batched
    // over four elements (the batched key switch's launches), the score being
    // the sum; tune_ms[v] reports forward v plus its paired inverse
    constexpr int kTuneElems = 4;
    const size_t elem = (size_t)(c->L + c->dnum * (c->L + c->K)) * c->N;  // XT then the digits
    uint64_t* tbuf = nullptr;
    if (cudaMallocAsync((void**)&tbuf, kTuneElems * elem * sizeof(uint64_t), c->st) == cudaSuccess) {
        cudaMemsetAsync(tbuf, 0, kTuneElems * elem * sizeof(uint64_t), c->st);
    } else {
        cudaGetLastError();
        tbuf = nullptr;
    }
    LimbMap mb{};
    if (tbuf) {
        mb.nb = kTuneElems;
        for (int sgi = 0; sgi < nseg; ++sgi) {
            uint64_t* d0 = tbuf + (size_t)c->L * c->N + (size_t)sgi * np * c->N;
            LimbMap one = map_single(d0, d0, np, np, 0);
            one.seg[0].bstride = elem;
            mb.seg[mb.nseg++] = one.seg[0];
            mb.total += np;
        }
    }
    const int niv = ntt_num_inverse_variants();
    std::vector<float> fwd_ms(nv, 1e30f), inv_ms(niv, 1e30f), fwd_bms(nv, 1e30f), inv_bms(niv, 1e30f);
    for (int r = 0; r < kRounds; ++r) {
        for (int v = 0; v < nv; ++v) {
            c->dev.ntt_variant = v;
            ntt_forward(c->dev, m, FL_PLAIN, FS_PLAIN, c->st);
            cudaEventRecord(e0, c->st);
            for (int k = 0; k < kReps; ++k) ntt_forward(c->dev, m, FL_PLAIN, FS_PLAIN, c->st);
            fwd_ms[v] = std::min(fwd_ms[v], elapsed() / kReps);
            if (!tbuf) continue;
            cudaEventRecord(e0, c->st);
            for (int k = 0; k < kReps; ++k) ntt_forward(c->dev, mb, FL_PLAIN, FS_PLAIN, c->st);
            fwd_bms[v] = std::min(fwd_bms[v], elapsed() / kReps);
        }
        for (int v = 0; v < niv; ++v) {
            c->dev.intt_variant = v;
            ntt_inverse(c->dev, m, IL_PLAIN, IS_PLAIN, c->st);
            cudaEventRecord(e0, c->st);
            for (int k = 0; k < kReps; ++k) ntt_inverse(c->dev, m, IL_PLAIN, IS_PLAIN, c->st);
            inv_ms[v] = std::min(inv_ms[v], elapsed() / kReps);
            if (!tbuf) continue;
            cudaEventRecord(e0, c->st);
            for (int k = 0; k < kReps; ++k) ntt_inverse(c->dev, mb, IL_PLAIN, IS_PLAIN, c->st);
            inv_bms[v] = std::min(inv_bms[v], elapsed() / kReps);
        }
    }
    if (tbuf) {
        // the zero residues the batched timings transformed are reused below
        for (int v = 0; v < nv; ++v) fwd_ms[v] += fwd_bms[v];
        for (int v = 0; v < niv; ++v) inv_ms[v] += inv_bms[v];
    }
    c->tune_ms.assign(nv, 0.f);
    for (int v = 0; v < nv; ++v) c->tune_ms[v] = fwd_ms[v] + inv_ms[ntt_inverse_of(v)];
    int best = 0, best_inv = 0;
    for (int v = 1; v < nv; ++v)
        if (fwd_ms[v] < fwd_ms[best]) best = v;
    for (int v = 1; v < niv; ++v)
        if (inv_ms[v] < inv_ms[best_inv]) best_inv = v;
    // base-conversion variants (split products need every modulus below
    // 2^60): the ModUp conversion of four top-level elements in one launch,
    // as the batched key switch runs it, in a scratch buffer freed after
    bool split_ok = true;
    for (uint64_t q : c->host.prime) split_ok = split_ok && q < (1ull << 60);
    const bool tc_tune = conv_tc_supported(c->dev);  // tensor-core ModUp (int8 split)
    c->conv_ms.assign(kConvVariants, 0.f);
    int conv_best = 0;
    const int top = c->L - 1;
    if (conv_supported(c->dev) && tbuf) {
        cudaMemsetAsync(tbuf, 0, kTuneElems * elem * sizeof(uint64_t), c->st);
        uint64_t* xt = tbuf;
        uint64_t* dig = tbuf + (size_t)c->L * c->N;
        const size_t dstride = (size_t)(c->L + c->K);
        std::vector<float> best_ms(kConvVariants, 1e30f);
        for (int r = 0; r < kRounds; ++r)
            for (int v = 0; v < kConvVariants; ++v) {
                if (v == 1 && !split_ok) continue;
                if (v >= 3 && !tc_tune) continue;
                c->dev.conv_variant = v;
                launch_modup_conv(c->dev, top, kTuneElems, xt, dig, dstride, elem, c->st);
                cudaEventRecord(e0, c->st);
                for (int k = 0; k < kReps; ++k) launch_modup_conv(c->dev, top, kTuneElems, xt, dig, dstride, elem, c->st);
                best_ms[v] = std::min(best_ms[v], elapsed() / kReps);
            }
        for (int v = 0; v < kConvVariants; ++v) {
            c->conv_ms[v] = best_ms[v] < 1e29f ? best_ms[v] : 0.f;
            if (c->conv_ms[v] > 0.f && c->conv_ms[v] < c->conv_ms[conv_best]) conv_best = v;
        }
    }
    if (tbuf) cudaFreeAsync(tbuf, c->st);
    c->dev.conv_variant = conv_best;
    c->tuned_conv = conv_best;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->tuned_variant = best;
    c->tuned_inverse = best_inv;
    c->dev.ntt_variant = best;
    c->dev.intt_variant = best_inv;
    if (variant) *variant = best;
    if (num_variants) *num_variants = nv;
    if (times_ms)
        for (int v = 0; v < nv; ++v) times_ms[v] = c->tune_ms[v];
    return check_cuda(c, "autotune");
}

fides_status fides_autotune_conv_info(const fides_ctx* c, int* accumulator, float* times_ms) {
    if (!c) return FIDES_BAD_ARG;
    if (accumulator) *accumulator = c->tuned_conv;
    if (times_ms)
        for (size_t v = 0; v < (size_t)kConvVariants; ++v) times_ms[v] = v < c->conv_ms.size() ? c->conv_ms[v] : 0.f;
    return FIDES_OK;
}

fides_status fides_set_conv_accumulator(fides_ctx* c, int accumulator) {
    if (!c || accumulator < -1 || accumulator >= kConvVariants) return FIDES_BAD_ARG;
    Guard g(c);
    if (accumulator == 1)
        for (uint64_t q : c->host.prime)
            if (q >= (1ull << 60)) return set_err(c, FIDES_UNSUPPORTED, "split products need moduli below 2^60");
    if (accumulator >= 3 && !conv_tc_supported(c->dev))
        return set_err(c, FIDES_UNSUPPORTED, "tensor-core conversion needs digits of at most 16 moduli and at most 48 targets");
    c->dev.conv_variant = accumulator < 0 ? c->tuned_conv : accumulator;
    return FIDES_OK;
}

fides_status fides_ctx_device_status(fides_ctx* ctx, uint32_t* flags) {
    if (!ctx || !flags) return FIDES_BAD_ARG;
    Guard g(ctx);
    *flags = read_device_error(ctx, nullptr, false);
    return check_cuda(ctx, "device status");
}

fides_status fides_ctx_inject_device_error(fides_ctx* ctx, uint32_t flags) {
    if (!ctx || !ctx->dev.err) return FIDES_BAD_ARG;
    Guard g(ctx);
    // a host-side write into the word, ordered after the work already queued:
    // exercises the reporting path without any kernel failing
    const uint32_t w = flags;
    cudaMemcpyAsync(ctx->dev.err, &w, sizeof(w), cudaMemcpyHostToDevice, ctx->st);
    cudaStreamSynchronize(ctx->st);
    return check_cuda(ctx, "inject device error");
}

fides_status fides_set_giant_step_moddown(fides_ctx* c, int scope) {
    if (!c || scope < 0 || scope > 2) return FIDES_BAD_ARG;
    Guard g(c);
    c->giant_moddown = scope;
    return FIDES_OK;
}

fides_status fides_set_keyswitch_variant(fides_ctx* c, int variant) {
    if (!c || variant < 0 || variant > 15) return FIDES_BAD_ARG;
    Guard g(c);
    c->dev.ks_variant = variant;
    return FIDES_OK;
}

fides_status fides_set_ntt_variant(fides_ctx* c, int variant) {
    if (!c || variant >= ntt_num_variants() || variant < -1) return FIDES_BAD_ARG;
    Guard g(c);
    c->dev.ntt_variant = variant < 0 ? c->tuned_variant : variant;
    c->dev.intt_variant = variant < 0 ? c->tuned_inverse : ntt_inverse_of(variant);
    return FIDES_OK;
}

// galois != 0: the key is stored permuted to the rotation's output order,
// entry j = uploaded entry slot(galois, j) (the key-switch kernel's layout)
static fides_status upload_key(fides_ctx* c, SwitchKey& k, const uint64_t* b, const uint64_t* a,
                               uint32_t galois = 0) {
    const int nlimbs = c->dnum * (c->L + c->K);
    const size_t words = (size_t)nlimbs * c->N;
    fides_status s = key_alloc(c, k, false);
    if (s != FIDES_OK) return s;
    if (!galois) {
        cudaMemcpyAsync(k.b, b, words * 8, cudaMemcpyHostToDevice, c->st);
        cudaMemcpyAsync(k.a, a, words * 8, cudaMemcpyHostToDevice, c->st);
    } else {
        uint64_t* tmp = nullptr;
        if (cudaMallocAsync((void**)&tmp, words * 8, c->st) != cudaSuccess) {
            cudaGetLastError();
            return set_err(c, FIDES_OOM, "key upload scratch");
        }
        cudaMemcpyAsync(tmp, b, words * 8, cudaMemcpyHostToDevice, c->st);
        launch_automorph(c->dev, nlimbs, tmp, k.b, galois, c->st);
        cudaMemcpyAsync(tmp, a, words * 8, cudaMemcpyHostToDevice, c->st);
        launch_automorph(c->dev, nlimbs, tmp, k.a, galois, c->st);
        cudaFreeAsync(tmp, c->st);
    }
    cudaStreamSynchronize(c->st);
    return check_cuda(c, "key upload");
}

fides_status fides_key_upload_relin(fides_ctx* ctx, const uint64_t* b, const uint64_t* a) {
    if (!ctx || !b || !a) return FIDES_BAD_ARG;
    Guard g(ctx);
    fides_status s = upload_key(ctx, ctx->relin, b, a);
    if (s == FIDES_OK) ctx->has_relin = true;
    return s;
}

fides_status fides_key_upload_galois(fides_ctx* ctx, uint32_t galois, const uint64_t* b, const uint64_t* a) {
    if (!ctx || !b || !a || !(galois & 1) || galois >= 2u * (uint32_t)ctx->N) return FIDES_BAD_ARG;
    Guard g(ctx);
    SwitchKey& k = ctx->galois_keys[galois];
    return upload_key(ctx, k, b, a, galois);
}

uint32_t fides_rotation_galois(const fides_ctx* ctx, int32_t index, int slots) {
    if (!ctx || slots <= 0) return 0;
    const int N = ctx->N;
    int idx = index % slots;
    if (idx < 0) idx += slots;
    if (idx > slots / 2) idx += N / 2 - slots;
    return (uint32_t)powmod(5, (uint64_t)idx, 2ull * N);
}

fides_status fides_ct_create(fides_ctx* ctx, fides_ct** out) {
    if (!ctx || !out) return FIDES_BAD_ARG;
    *out = new (std::nothrow) fides_ct();
    return *out ? FIDES_OK : FIDES_OOM;
}

fides_status fides_ct_upload(fides_ctx* ctx, const uint64_t* c0, const uint64_t* c1, int level, double scale,
                             int noise_deg, int slots, fides_ct** out) {
    if (!ctx || !c0 || !c1 || !out || level < 0 || level >= ctx->L) return FIDES_BAD_ARG;
    Guard g(ctx);
    fides_ct* ct = new (std::nothrow) fides_ct();
    if (!ct) return FIDES_OOM;
    // allocated and filled on the upload stream, so that the copy runs beside
    // kernels already queued on the context stream, which then waits for it
    fides_status s = ct_reserve(ctx, ct, level, ctx->h2d);
    if (s != FIDES_OK) {
        delete ct;
        return s;
    }
    const size_t bytes = (size_t)(level + 1) * ctx->limb_bytes();
    cudaMemcpyAsync(ct->c0(), c0, bytes, cudaMemcpyHostToDevice, ctx->h2d);
    cudaMemcpyAsync(ct->c1(ctx->N), c1, bytes, cudaMemcpyHostToDevice, ctx->h2d);
    cudaEvent_t ev;
    cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    cudaEventRecord(ev, ctx->h2d);
    cudaStreamWaitEvent(ctx->st, ev, 0);
    cudaEventDestroy(ev);
    ct->level = level;
    ct->scale = scale;
    ct->noise_deg = noise_deg;
    ct->slots = slots;
    *out = ct;
    return check_cuda(ctx, "ct upload");
}

fides_status fides_ct_download(fides_ctx* ctx, const fides_ct* ct, uint64_t* c0, uint64_t* c1) {
    if (!ctx || !valid_ct(ctx, ct)) return FIDES_BAD_ARG;
    Guard g(ctx);
    const size_t bytes = (size_t)(ct->level + 1) * ctx->limb_bytes();
    if (c0) cudaMemcpyAsync(c0, ct->c0(), bytes, cudaMemcpyDeviceToHost, ctx->st);
    if (c1) cudaMemcpyAsync(c1, ct->c1(ctx->N), bytes, cudaMemcpyDeviceToHost, ctx->st);
    cudaStreamSynchronize(ctx->st);
    const fides_status s = check_cuda(ctx, "ct download");
    return s != FIDES_OK ? s : consume_device_error(ctx);
}

fides_status fides_ct_download_async(fides_ctx* ctx, const fides_ct* ct, uint64_t* c0, uint64_t* c1) {
    if (!ctx || !valid_ct(ctx, ct)) return FIDES_BAD_ARG;
    Guard g(ctx);
    // on the download stream after the kernels queued so far; later work that
    // releases or overwrites the buffer waits for the copy (ct_quiesce)
    cudaEvent_t ready;
    cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
    cudaEventRecord(ready, ctx->st);
    cudaStreamWaitEvent(ctx->d2h, ready, 0);
    cudaEventDestroy(ready);
    const size_t bytes = (size_t)(ct->level + 1) * ctx->limb_bytes();
    if (c0) cudaMemcpyAsync(c0, ct->c0(), bytes, cudaMemcpyDeviceToHost, ctx->d2h);
    if (c1) cudaMemcpyAsync(c1, ct->c1(ctx->N), bytes, cudaMemcpyDeviceToHost, ctx->d2h);
    if (ct->d2h_ev) cudaEventDestroy(ct->d2h_ev);  // superseded: same stream, later copy
    cudaEventCreateWithFlags(&ct->d2h_ev, cudaEventDisableTiming);
    cudaEventRecord(ct->d2h_ev, ctx->d2h);
    return check_cuda(ctx, "ct download");
}

fides_status fides_ct_info(const fides_ct* ct, int* level, double* scale, int* noise_deg, int* slots) {
    if (!ct) return FIDES_BAD_ARG;
    if (level) *level = ct->level;
    if (scale) *scale = ct->scale;
    if (noise_deg) *noise_deg = ct->noise_deg;
    if (slots) *slots = ct->slots;
    return FIDES_OK;
}

fides_status fides_ct_device_ptrs(const fides_ct* ct, uint64_t** c0, uint64_t** c1) {
    if (!ct || !ct->buf) return FIDES_BAD_ARG;
    if (c0) *c0 = ct->c0();
    if (c1) *c1 = ct->c1(ct->ring);
    return FIDES_OK;
}

fides_status fides_ct_write(fides_ctx* ctx, fides_ct* ct, const uint64_t* c0, const uint64_t* c1) {
    if (!ctx || !valid_ct(ctx, ct) || !c0 || !c1) return FIDES_BAD_ARG;
    Guard g(ctx);
    ct_quiesce(ctx, ct);
    const size_t bytes = (size_t)(ct->level + 1) * ctx->limb_bytes();
    cudaMemcpyAsync(ct->c0(), c0, bytes, cudaMemcpyHostToDevice, ctx->st);
    cudaMemcpyAsync(ct->c1(ctx->N), c1, bytes, cudaMemcpyHostToDevice, ctx->st);
    return check_cuda(ctx, "ct write");
}

fides_status fides_ct_copy(fides_ctx* ctx, const fides_ct* src, fides_ct* dst) {
    if (!ctx || !valid_ct(ctx, src) || !dst) return FIDES_BAD_ARG;
    if (src == dst) return FIDES_OK;
    Guard g(ctx);
    fides_status s = ct_reserve(ctx, dst, src->level);
    if (s != FIDES_OK) return s;
    const size_t bytes = (size_t)(src->level + 1) * ctx->limb_bytes();
    cudaMemcpyAsync(dst->c0(), src->c0(), bytes, cudaMemcpyDeviceToDevice, ctx->st);
    cudaMemcpyAsync(dst->c1(ctx->N), src->c1(ctx->N), bytes, cudaMemcpyDeviceToDevice, ctx->st);
    dst->level = src->level;
    dst->scale = src->scale;
    dst->noise_deg = src->noise_deg;
    dst->slots = src->slots;
    return check_cuda(ctx, "ct copy");
}

fides_status fides_ct_free(fides_ctx* ctx, fides_ct* ct) {
    if (!ctx || !ct) return FIDES_BAD_ARG;
    Guard g(ctx);
    ct_quiesce(ctx, ct);
    if (ct->buf) cudaFreeAsync(ct->buf, ctx->st);
    delete ct;
    return FIDES_OK;
}

fides_status fides_ct_set_level(fides_ctx* ctx, fides_ct* ct, int level) {
    if (!ctx || !valid_ct(ctx, ct) || level < 0 || level > ct->level) return FIDES_BAD_ARG;
    Guard g(ctx);
    if (level == ct->level) return FIDES_OK;
    fides_ct tmp;
    fides_status s = ct_reserve(ctx, &tmp, level);
    if (s != FIDES_OK) return s;
    const size_t bytes = (size_t)(level + 1) * ctx->limb_bytes();
    cudaMemcpyAsync(tmp.c0(), ct->c0(), bytes, cudaMemcpyDeviceToDevice, ctx->st);
    cudaMemcpyAsync(tmp.c1(ctx->N), ct->c1(ctx->N), bytes, cudaMemcpyDeviceToDevice, ctx->st);
    commit(ctx, ct, tmp);
    ct->level = level;
    return check_cuda(ctx, "set level");
}

fides_status fides_pt_upload(fides_ctx* ctx, const uint64_t* m, int level, double scale, int noise_deg, int slots,
                             fides_pt** out) {
    if (!ctx || !m || !out || level < 0 || level >= ctx->L) return FIDES_BAD_ARG;
    Guard g(ctx);
    fides_pt* pt = new (std::nothrow) fides_pt();
    if (!pt) return FIDES_OOM;
    pt->cap = level + 1;
    if (cudaMallocAsync((void**)&pt->m, (size_t)pt->cap * ctx->limb_bytes(), ctx->st) != cudaSuccess) {
        cudaGetLastError();
        delete pt;
        return set_err(ctx, FIDES_OOM, "plaintext allocation failed");
    }
    cudaMemcpyAsync(pt->m, m, (size_t)pt->cap * ctx->limb_bytes(), cudaMemcpyHostToDevice, ctx->st);
    pt->level = level;
    pt->scale = scale;
    pt->noise_deg = noise_deg;
    pt->slots = slots;
    *out = pt;
    return check_cuda(ctx, "pt upload");
}

fides_status fides_pt_free(fides_ctx* ctx, fides_pt* pt) {
    if (!ctx || !pt) return FIDES_BAD_ARG;
    Guard g(ctx);
    if (pt->m) cudaFreeAsync(pt->m, ctx->st);
    delete pt;
    return FIDES_OK;
}

// ---------------------------------------------------------------------------

static fides_status hmult_impl(fides_ctx* c, const fides_ct* a, const fides_ct* b, fides_ct* out, int rescale) {
    if (!valid_ct(c, a) || !valid_ct(c, b) || !out) return FIDES_BAD_ARG;
    if (!c->has_relin) return set_err(c, FIDES_KEY_MISSING, "no relinearisation key");
    const int level = std::min(a->level, b->level);
    const bool rs = rescale && level > 0;
    const int N = c->N;
    fides_ct tmp;
    fides_status s = ct_reserve(c, &tmp, rs ? level - 1 : level);
    if (s != FIDES_OK) return s;
    const uint64_t *a0 = a->c0(), *a1 = a->c1(N), *b0 = b->c0(), *b1 = b->c1(N);
    uint64_t *o0 = tmp.c0(), *o1 = tmp.c1(N);
    eng_hmult(c, c->ws1, level, 1, &a0, &a1, &b0, &b1, &o0, &o1, rs, c->relin);
    const double sc = a->scale * b->scale;
    const int nd = a->noise_deg + b->noise_deg;
    const int sl = std::max(a->slots, b->slots);
    commit(c, out, tmp);
    out->level = rs ? level - 1 : level;
    out->scale = rs ? sc / (double)c->host.prime[level] : sc;
    out->noise_deg = rs ? nd - 1 : nd;
    out->slots = sl;
    return check_cuda(c, "hmult");
}

fides_status fides_hmult(fides_ctx* ctx, const fides_ct* a, const fides_ct* b, fides_ct* out, int rescale) {
    if (!ctx) return FIDES_BAD_ARG;
    Guard g(ctx);
    return hmult_impl(ctx, a, b, out, rescale);
}

fides_status fides_square(fides_ctx* ctx, const fides_ct* a, fides_ct* out, int rescale) {
    if (!ctx) return FIDES_BAD_ARG;
    Guard g(ctx);
    return hmult_impl(ctx, a, a, out, rescale);
}

}  // extern "C"

// In-place rescale of n ciphertexts at one level, the same per-ciphertext
// steps as fides_rescale (INTT of the top limb, then one NTT per remaining
// limb with the switch-modulus prologue and the rescale epilogue), up to four
// ciphertexts per launch pair: small single-ciphertext launches leave most
// SMs idle, a batch fills them.  Results equal one fides_rescale each.
fides_status fides::rescale_batch(fides_ctx* c, int n, fides_ct* const* cts) {
    if (!c || n < 0) return FIDES_BAD_ARG;
    for (int i = 0; i < n; ++i)
        if (!valid_ct(c, cts[i]) || cts[i]->level < 1 || cts[i]->level != cts[0]->level) return FIDES_BAD_ARG;
    if (n == 0) return FIDES_OK;
    Guard g(c);
    const int l = cts[0]->level, N = c->N;
    constexpr int kPer = kMaxSeg / 2;
    uint64_t* top = nullptr;  // INTT of the top limbs, two per ciphertext
    if (cudaMallocAsync((void**)&top, (size_t)2 * kPer * N * 8, c->st) != cudaSuccess) {
        cudaGetLastError();
        return set_err(c, FIDES_OOM, "rescale scratch");
    }
    fides_status s = FIDES_OK;
    for (int i0 = 0; i0 < n && s == FIDES_OK; i0 += kPer) {
        const int k = std::min(kPer, n - i0);
        std::vector<fides_ct> tmp(k);
        LimbMap t{}, m{};
        for (int j = 0; j < k && s == FIDES_OK; ++j) {
            s = ct_reserve(c, &tmp[j], l - 1);
            const uint64_t* ins[2] = {cts[i0 + j]->c0(), cts[i0 + j]->c1(N)};
            uint64_t* os[2] = {tmp[j].c0(), tmp[j].c1(N)};
            for (int h = 0; h < 2; ++h) {
                uint64_t* tl = top + (size_t)(2 * j + h) * N;
                LimbSeg& a = t.seg[t.nseg++];
                a.in = ins[h] + (size_t)l * N;
                a.out = tl;
                a.count = 1;
                a.skip_lo = 1;
                a.nq = 1;
                a.q0 = l;
                a.level = l;
                t.total += 1;
                LimbSeg& b = m.seg[m.nseg++];
                b.in = tl;
                b.in_stride_zero = 1;
                b.in2 = ins[h];
                b.out = os[h];
                b.count = l;
                b.skip_lo = l;
                b.nq = l;
                b.level = l;
                m.total += l;
            }
        }
        if (s != FIDES_OK) break;
        ntt_inverse(c->dev, t, IL_PLAIN, IS_PLAIN, c->st);
        ntt_forward(c->dev, m, FL_SWITCHMOD, FS_RESCALE, c->st);
        for (int j = 0; j < k; ++j) {
            fides_ct* o = cts[i0 + j];
            const double sc = o->scale / (double)c->host.prime[l];
            const int nd = o->noise_deg - 1, sl = o->slots;
            commit(c, o, tmp[j]);
            o->level = l - 1;
            o->scale = sc;
            o->noise_deg = nd;
            o->slots = sl;
        }
    }
    cudaFreeAsync(top, c->st);
    return s != FIDES_OK ? s : check_cuda(c, "rescale");
}

extern "C" {

fides_status fides_rescale(fides_ctx* c, const fides_ct* a, fides_ct* out) {
    if (!c || !valid_ct(c, a) || !out || a->level < 1) return FIDES_BAD_ARG;
    Guard g(c);
    const int l = a->level, N = c->N;
    fides_ct tmp;
    fides_status s = ct_reserve(c, &tmp, l - 1);
    if (s != FIDES_OK) return s;
    LimbMap t{};
    t.nseg = 2;
    const uint64_t* ins[2] = {a->c0(), a->c1(N)};
    for (int i = 0; i < 2; ++i) {
        LimbSeg& g2 = t.seg[i];
        g2.in = ins[i] + (size_t)l * N;
        g2.out = c->ws1.T + (size_t)i * N;
        g2.count = 1;
        g2.skip_lo = 1;
        g2.nq = 1;
        g2.q0 = l;
        g2.level = l;
        t.total += 1;
    }
    ntt_inverse(c->dev, t, IL_PLAIN, IS_PLAIN, c->st);
    LimbMap m{};
    m.nseg = 2;
    uint64_t* os[2] = {tmp.c0(), tmp.c1(N)};
    for (int i = 0; i < 2; ++i) {
        LimbSeg& g2 = m.seg[i];
        g2.in = c->ws1.T + (size_t)i * N;
        g2.in_stride_zero = 1;
        g2.in2 = ins[i];
        g2.out = os[i];
        g2.count = l;
        g2.skip_lo = l;
        g2.nq = l;
        g2.level = l;
        m.total += l;
    }
    ntt_forward(c->dev, m, FL_SWITCHMOD, FS_RESCALE, c->st);
    const double sc = a->scale / (double)c->host.prime[l];
    const int nd = a->noise_deg - 1, sl = a->slots;
    commit(c, out, tmp);
    out->level = l - 1;
    out->scale = sc;
    out->noise_deg = nd;
    out->slots = sl;
    return check_cuda(c, "rescale");
}

// n rotations of one ciphertext sharing one ModUp (hoisted); n = 1 is a plain
// rotation.  Rotations are processed in batches of up to kMaxBatch.
static fides_status rotate_many(fides_ctx* c, const fides_ct* a, int n, const uint32_t* galois, fides_ct** outs) {
    if (!valid_ct(c, a) || n < 1) return FIDES_BAD_ARG;
    std::vector<const SwitchKey*> keys(n);
    for (int r = 0; r < n; ++r) {
        if (!outs[r]) return FIDES_BAD_ARG;
        auto it = c->galois_keys.find(galois[r]);
        if (it == c->galois_keys.end())
            return set_err(c, FIDES_KEY_MISSING, "no key for galois element " + std::to_string(galois[r]));
        keys[r] = &it->second;
    }
    const int level = a->level, N = c->N;
    std::vector<fides_ct> tmp(n);
    for (int r = 0; r < n; ++r) {
        fides_status s = ct_reserve(c, &tmp[r], level);
        if (s != FIDES_OK) return s;
    }
    Workspace* w = &c->ws1;
    if (n > 1) {
        fides_status s = ws_reserve(c, c->wsb, std::min(n, kMaxBatch));
        if (s != FIDES_OK) return s;
        w = &c->wsb;
    }
    const uint64_t *c0 = a->c0(), *c1 = a->c1(N);
    for (int r0 = 0; r0 < n; r0 += w->cap) {
        const int nb = std::min(w->cap, n - r0);
        std::vector<uint64_t*> o0(nb), o1(nb);
        for (int b = 0; b < nb; ++b) {
            o0[b] = tmp[r0 + b].c0();
            o1[b] = tmp[r0 + b].c1(N);
        }
        eng_rotate(c, *w, level, nb, &c0, &c1, keys.data() + r0, galois + r0, o0.data(), o1.data(), true);
    }
    const double sc = a->scale;
    const int nd = a->noise_deg, sl = a->slots;
    for (int r = 0; r < n; ++r) {
        commit(c, outs[r], tmp[r]);
        outs[r]->level = level;
        outs[r]->scale = sc;
        outs[r]->noise_deg = nd;
        outs[r]->slots = sl;
    }
    return check_cuda(c, "rotate");
}

// Hoisted rotations of nx ciphertexts at one level by the same n indices:
// groups of inputs share one batched ModUp and one inner-product / ModDown
// launch sequence (outs[u * n + r] = rotation of xs[u] by galois[r]).
static fides_status rotate_many_groups(fides_ctx* c, int nx, const fides_ct* const* xs, int n, const uint32_t* galois,
                                       fides_ct* const* outs) {
    if (n < 1 || nx < 1) return FIDES_BAD_ARG;
    if (nx == 1 || n > kMaxBatch / 2) {
        for (int u = 0; u < nx; ++u) {
            std::vector<fides_ct*> o(outs + (size_t)u * n, outs + (size_t)(u + 1) * n);
            fides_status s = rotate_many(c, xs[u], n, galois, o.data());
            if (s != FIDES_OK) return s;
        }
        return FIDES_OK;
    }
    std::vector<const SwitchKey*> keys(n);
    for (int r = 0; r < n; ++r) {
        auto it = c->galois_keys.find(galois[r]);
        if (it == c->galois_keys.end())
            return set_err(c, FIDES_KEY_MISSING, "no key for galois element " + std::to_string(galois[r]));
        keys[r] = &it->second;
    }
    const int level = xs[0]->level, N = c->N;
    fides_status s = ws_reserve(c, c->wsb, std::min(nx * n, kMaxBatch));
    if (s != FIDES_OK) return s;
    const int gmax = std::max(1, c->wsb.cap / n);
    std::vector<fides_ct> tmp((size_t)nx * n);
    for (auto& t : tmp)
        if ((s = ct_reserve(c, &t, level)) != FIDES_OK) return s;
    for (int u0 = 0; u0 < nx; u0 += gmax) {
        const int ng = std::min(gmax, nx - u0), nb = ng * n;
        std::vector<const uint64_t*> c0(ng), c1(ng);
        for (int g = 0; g < ng; ++g) {
            c0[g] = xs[u0 + g]->c0();
            c1[g] = xs[u0 + g]->c1(N);
        }
        std::vector<const SwitchKey*> kk(nb);
        std::vector<uint32_t> gg(nb);
        std::vector<uint64_t*> o0(nb), o1(nb);
        for (int b = 0; b < nb; ++b) {
            kk[b] = keys[b % n];
            gg[b] = galois[b % n];
            o0[b] = tmp[(size_t)u0 * n + b].c0();
            o1[b] = tmp[(size_t)u0 * n + b].c1(N);
        }
        eng_rotate_groups(c, c->wsb, level, ng, n, c0.data(), c1.data(), kk.data(), gg.data(), o0.data(), o1.data());
    }
    for (int u = 0; u < nx; ++u)
        for (int r = 0; r < n; ++r) {
            const fides_ct meta = *xs[u];
            fides_ct* o = outs[(size_t)u * n + r];
            commit(c, o, tmp[(size_t)u * n + r]);
            o->level = level;
            o->scale = meta.scale;
            o->noise_deg = meta.noise_deg;
            o->slots = meta.slots;
        }
    return check_cuda(c, "rotate groups");
}

fides_status fides_rotate(fides_ctx* ctx, const fides_ct* a, int32_t index, fides_ct* out) {
    if (!ctx || !valid_ct(ctx, a) || !out) return FIDES_BAD_ARG;
    Guard g(ctx);
    const int slots = a->slots > 0 ? a->slots : ctx->N / 2;
    const uint32_t gal = fides_rotation_galois(ctx, index, slots);
    if (gal == 1) return fides_ct_copy(ctx, a, out);
    return rotate_many(ctx, a, 1, &gal, &out);
}

fides_status fides_rotate_hoisted(fides_ctx* ctx, const fides_ct* a, int n, const int32_t* indices, fides_ct** outs) {
    if (!ctx || !valid_ct(ctx, a) || n < 1 || !indices || !outs) return FIDES_BAD_ARG;
    Guard g(ctx);
    const int slots = a->slots > 0 ? a->slots : ctx->N / 2;
    std::vector<uint32_t> gal;
    std::vector<fides_ct*> o;
    for (int r = 0; r < n; ++r) {
        const uint32_t ge = fides_rotation_galois(ctx, indices[r], slots);
        if (ge == 1) {
            fides_status s = fides_ct_copy(ctx, a, outs[r]);
            if (s != FIDES_OK) return s;
            continue;
        }
        gal.push_back(ge);
        o.push_back(outs[r]);
    }
    if (gal.empty()) return FIDES_OK;
    return rotate_many(ctx, a, (int)gal.size(), gal.data(), o.data());
}

fides_status fides_conjugate(fides_ctx* ctx, const fides_ct* a, fides_ct* out) {
    if (!ctx || !valid_ct(ctx, a) || !out) return FIDES_BAD_ARG;
    Guard g(ctx);
    const uint32_t gal = 2u * (uint32_t)ctx->N - 1;
    return rotate_many(ctx, a, 1, &gal, &out);
}

fides_status fides_automorphism(fides_ctx* ctx, const fides_ct* a, uint32_t galois, fides_ct* out) {
    if (!ctx || !valid_ct(ctx, a) || !out) return FIDES_BAD_ARG;
    Guard g(ctx);
    return rotate_many(ctx, a, 1, &galois, &out);
}

static fides_status binary_op(fides_ctx* c, int op, const fides_ct* a, const fides_ct* b, fides_ct* out) {
    if (!valid_ct(c, a) || (op != EW_NEG && !valid_ct(c, b)) || !out) return FIDES_BAD_ARG;
    const int level = op == EW_NEG ? a->level : std::min(a->level, b->level);
    const int n = level + 1, N = c->N;
    fides_ct tmp;
    fides_status s = ct_reserve(c, &tmp, level);
    if (s != FIDES_OK) return s;
    launch_elementwise(c->dev, op, n, 0, a->c0(), b ? b->c0() : nullptr, tmp.c0(), c->st);
    launch_elementwise(c->dev, op, n, 0, a->c1(N), b ? b->c1(N) : nullptr, tmp.c1(N), c->st);
    const double sc = a->scale;
    const int nd = a->noise_deg, sl = std::max(a->slots, b ? b->slots : 0);
    commit(c, out, tmp);
    out->level = level;
    out->scale = sc;
    out->noise_deg = nd;
    out->slots = sl;
    return check_cuda(c, "elementwise");
}

fides_status fides_add(fides_ctx* ctx, const fides_ct* a, const fides_ct* b, fides_ct* out) {
    if (!ctx) return FIDES_BAD_ARG;
    Guard g(ctx);
    return binary_op(ctx, EW_ADD, a, b, out);
}
fides_status fides_sub(fides_ctx* ctx, const fides_ct* a, const fides_ct* b, fides_ct* out) {
    if (!ctx) return FIDES_BAD_ARG;
    Guard g(ctx);
    return binary_op(ctx, EW_SUB, a, b, out);
}
fides_status fides_negate(fides_ctx* ctx, const fides_ct* a, fides_ct* out) {
    if (!ctx) return FIDES_BAD_ARG;
    Guard g(ctx);
    return binary_op(ctx, EW_NEG, a, nullptr, out);
}

fides_status fides_add_pt(fides_ctx* c, const fides_ct* a, const fides_pt* p, fides_ct* out) {
    if (!c || !valid_ct(c, a) || !p || !p->m || !out) return FIDES_BAD_ARG;
    Guard g(c);
    const int level = std::min(a->level, p->level), n = level + 1, N = c->N;
    fides_ct tmp;
    fides_status s = ct_reserve(c, &tmp, level);
    if (s != FIDES_OK) return s;
    launch_elementwise(c->dev, EW_ADD, n, 0, a->c0(), p->m, tmp.c0(), c->st);
    launch_elementwise(c->dev, EW_COPY, n, 0, a->c1(N), nullptr, tmp.c1(N), c->st);
    const double sc = a->scale;
    const int nd = a->noise_deg, sl = std::max(a->slots, p->slots);
    commit(c, out, tmp);
    out->level = level;
    out->scale = sc;
    out->noise_deg = nd;
    out->slots = sl;
    return check_cuda(c, "add_pt");
}

fides_status fides_mult_pt(fides_ctx* c, const fides_ct* a, const fides_pt* p, fides_ct* out, int rescale) {
    if (!c || !valid_ct(c, a) || !p || !p->m || !out) return FIDES_BAD_ARG;
    Guard g(c);
    const int level = std::min(a->level, p->level), n = level + 1, N = c->N;
    fides_ct tmp;
    fides_status s = ct_reserve(c, &tmp, level);
    if (s != FIDES_OK) return s;
    launch_elementwise(c->dev, EW_MUL, n, 0, a->c0(), p->m, tmp.c0(), c->st);
    launch_elementwise(c->dev, EW_MUL, n, 0, a->c1(N), p->m, tmp.c1(N), c->st);
    const double sc = a->scale * p->scale;
    const int nd = a->noise_deg + p->noise_deg, sl = std::max(a->slots, p->slots);
    commit(c, out, tmp);
    out->level = level;
    out->scale = sc;
    out->noise_deg = nd;
    out->slots = sl;
    fides_status st = check_cuda(c, "mult_pt");
    if (st == FIDES_OK && rescale && level > 0) st = fides_rescale(c, out, out);
    return st;
}

fides_status fides_add_scalar(fides_ctx* c, const fides_ct* a, double v, fides_ct* out) {
    if (!c || !valid_ct(c, a) || !out) return FIDES_BAD_ARG;
    Guard g(c);
    const int n = a->level + 1, N = c->N;
    std::vector<uint64_t> k(n);
    for (int j = 0; j < n; ++j) k[j] = round_to_mod((long double)v * a->scale, c->host.prime[j]);
    fides_ct tmp;
    fides_status s = ct_reserve(c, &tmp, a->level);
    if (s != FIDES_OK) return s;
    uint64_t* dk = nullptr;
    if (cudaMallocAsync((void**)&dk, n * 8, c->st) != cudaSuccess) return set_err(c, FIDES_OOM, "scalar table");
    cudaMemcpyAsync(dk, k.data(), n * 8, cudaMemcpyHostToDevice, c->st);
    launch_scalar_add(c->dev, n, a->c0(), dk, tmp.c0(), c->st);
    launch_elementwise(c->dev, EW_COPY, n, 0, a->c1(N), nullptr, tmp.c1(N), c->st);
    cudaStreamSynchronize(c->st);
    cudaFreeAsync(dk, c->st);
    const fides_ct meta = *a;
    commit(c, out, tmp);
    out->level = meta.level;
    out->scale = meta.scale;
    out->noise_deg = meta.noise_deg;
    out->slots = meta.slots;
    return check_cuda(c, "add_scalar");
}

fides_status fides_mult_scalar(fides_ctx* c, const fides_ct* a, double v, fides_ct* out, int rescale) {
    if (!c || !valid_ct(c, a) || !out) return FIDES_BAD_ARG;
    Guard g(c);
    const int n = a->level + 1, N = c->N;
    const double delta = c->default_scale;
    std::vector<uint64_t> k(2 * n);
    for (int j = 0; j < n; ++j) {
        const uint64_t p = c->host.prime[j];
        k[2 * j] = round_to_mod((long double)v * delta, p);
        k[2 * j + 1] = shoup_precompute(k[2 * j], p);
    }
    fides_ct tmp;
    fides_status s = ct_reserve(c, &tmp, a->level);
    if (s != FIDES_OK) return s;
    uint64_t* dk = nullptr;
    if (cudaMallocAsync((void**)&dk, 2 * n * 8, c->st) != cudaSuccess) return set_err(c, FIDES_OOM, "scalar table");
    cudaMemcpyAsync(dk, k.data(), 2 * n * 8, cudaMemcpyHostToDevice, c->st);
    launch_scalar_mac(c->dev, n, a->c0(), dk, nullptr, tmp.c0(), c->st);
    launch_scalar_mac(c->dev, n, a->c1(N), dk, nullptr, tmp.c1(N), c->st);
    cudaStreamSynchronize(c->st);
    cudaFreeAsync(dk, c->st);
    const fides_ct meta = *a;
    commit(c, out, tmp);
    out->level = meta.level;
    out->scale = meta.scale * delta;
    out->noise_deg = meta.noise_deg + 1;
    out->slots = meta.slots;
    fides_status st = check_cuda(c, "mult_scalar");
    if (st == FIDES_OK && rescale && out->level > 0) st = fides_rescale(c, out, out);
    return st;
}

// Elements grouped by level (stable), each group processed in chunks of the
// batch workspace's capacity.
static std::vector<std::vector<int>> level_groups(const fides_ctx* c, int n, const int* levels) {
    std::vector<std::vector<int>> g(c->L);
    for (int i = 0; i < n; ++i) g[levels[i]].push_back(i);
    std::vector<std::vector<int>> out;
    for (int l = c->L - 1; l >= 0; --l)
        if (!g[l].empty()) out.push_back(std::move(g[l]));
    return out;
}

fides_status fides_hmult_batch(fides_ctx* c, int n, const fides_ct* const* a, const fides_ct* const* b,
                               fides_ct* const* out, int rescale) {
    if (!c || n < 0 || (n && (!a || !b || !out))) return FIDES_BAD_ARG;
    Guard g(c);
    if (!c->has_relin) return set_err(c, FIDES_KEY_MISSING, "no relinearisation key");
    for (int i = 0; i < n; ++i)
        if (!valid_ct(c, a[i]) || !valid_ct(c, b[i]) || !out[i]) return FIDES_BAD_ARG;
    if (n == 0) return FIDES_OK;
    fides_status s = ws_reserve(c, c->wsb, std::min(n, kMaxBatch));
    if (s != FIDES_OK) return s;
    const int N = c->N;
    std::vector<int> lv(n);
    for (int i = 0; i < n; ++i) lv[i] = std::min(a[i]->level, b[i]->level);
    std::vector<fides_ct> tmp(n);
    for (auto& grp : level_groups(c, n, lv.data())) {
        const int level = lv[grp[0]];
        const bool rs = rescale && level > 0;
        for (int i : grp) {
            s = ct_reserve(c, &tmp[i], rs ? level - 1 : level);
            if (s != FIDES_OK) return s;
        }
        for (size_t k0 = 0; k0 < grp.size(); k0 += c->wsb.cap) {
            const int nb = (int)std::min(grp.size() - k0, (size_t)c->wsb.cap);
            std::vector<const uint64_t*> a0(nb), a1(nb), b0(nb), b1(nb);
            std::vector<uint64_t*> o0(nb), o1(nb);
            for (int j = 0; j < nb; ++j) {
                const int i = grp[k0 + j];
                a0[j] = a[i]->c0();
                a1[j] = a[i]->c1(N);
                b0[j] = b[i]->c0();
                b1[j] = b[i]->c1(N);
                o0[j] = tmp[i].c0();
                o1[j] = tmp[i].c1(N);
            }
            eng_hmult(c, c->wsb, level, nb, a0.data(), a1.data(), b0.data(), b1.data(), o0.data(), o1.data(), rs,
                      c->relin);
        }
    }
    for (int i = 0; i < n; ++i) {
        const int level = lv[i];
        const bool rs = rescale && level > 0;
        const double sc = a[i]->scale * b[i]->scale;
        const int nd = a[i]->noise_deg + b[i]->noise_deg;
        const int sl = std::max(a[i]->slots, b[i]->slots);
        commit(c, out[i], tmp[i]);
        out[i]->level = rs ? level - 1 : level;
        out[i]->scale = rs ? sc / (double)c->host.prime[level] : sc;
        out[i]->noise_deg = rs ? nd - 1 : nd;
        out[i]->slots = sl;
    }
    return check_cuda(c, "hmult_batch");
}

fides_status fides_rotate_batch(fides_ctx* c, int n, const fides_ct* const* a, const int32_t* indices,
                                fides_ct* const* out) {
    if (!c || n < 0 || (n && (!a || !indices || !out))) return FIDES_BAD_ARG;
    Guard g(c);
    for (int i = 0; i < n; ++i)
        if (!valid_ct(c, a[i]) || !out[i]) return FIDES_BAD_ARG;
    if (n == 0) return FIDES_OK;
    const int N = c->N;
    std::vector<uint32_t> gal(n);
    std::vector<const SwitchKey*> keys(n, nullptr);
    std::vector<int> lv(n);
    for (int i = 0; i < n; ++i) {
        gal[i] = fides_rotation_galois(c, indices[i], a[i]->slots > 0 ? a[i]->slots : N / 2);
        lv[i] = a[i]->level;
        if (gal[i] == 1) continue;
        auto it = c->galois_keys.find(gal[i]);
        if (it == c->galois_keys.end())
            return set_err(c, FIDES_KEY_MISSING, "no key for galois element " + std::to_string(gal[i]));
        keys[i] = &it->second;
    }
    fides_status s = ws_reserve(c, c->wsb, std::min(n, kMaxBatch));
    if (s != FIDES_OK) return s;
    std::vector<fides_ct> tmp(n);
    for (auto& grp0 : level_groups(c, n, lv.data())) {
        std::vector<int> grp;
        for (int i : grp0) {
            if (gal[i] == 1) {
                s = ct_reserve(c, &tmp[i], lv[i]);
                if (s != FIDES_OK) return s;
                const size_t bytes = (size_t)(lv[i] + 1) * c->limb_bytes();
                cudaMemcpyAsync(tmp[i].c0(), a[i]->c0(), bytes, cudaMemcpyDeviceToDevice, c->st);
                cudaMemcpyAsync(tmp[i].c1(N), a[i]->c1(N), bytes, cudaMemcpyDeviceToDevice, c->st);
            } else {
                grp.push_back(i);
            }
        }
        if (grp.empty()) continue;
        const int level = lv[grp[0]];
        for (int i : grp) {
            s = ct_reserve(c, &tmp[i], level);
            if (s != FIDES_OK) return s;
        }
        for (size_t k0 = 0; k0 < grp.size(); k0 += c->wsb.cap) {
            const int nb = (int)std::min(grp.size() - k0, (size_t)c->wsb.cap);
            std::vector<const uint64_t*> c0(nb), c1(nb);
            std::vector<uint64_t*> o0(nb), o1(nb);
            std::vector<const SwitchKey*> kk(nb);
            std::vector<uint32_t> gg(nb);
            for (int j = 0; j < nb; ++j) {
                const int i = grp[k0 + j];
                c0[j] = a[i]->c0();
                c1[j] = a[i]->c1(N);
                o0[j] = tmp[i].c0();
                o1[j] = tmp[i].c1(N);
                kk[j] = keys[i];
                gg[j] = gal[i];
            }
            eng_rotate(c, c->wsb, level, nb, c0.data(), c1.data(), kk.data(), gg.data(), o0.data(), o1.data(), false);
        }
    }
    for (int i = 0; i < n; ++i) {
        const fides_ct meta = *a[i];
        commit(c, out[i], tmp[i]);
        out[i]->level = meta.level;
        out[i]->scale = meta.scale;
        out[i]->noise_deg = meta.noise_deg;
        out[i]->slots = meta.slots;
    }
    return check_cuda(c, "rotate_batch");
}

// out = z * a (integer z), both components, level and scale of a.
fides_status fides_mult_int(fides_ctx* c, const fides_ct* a, int64_t z, fides_ct* out) {
    if (!c || !valid_ct(c, a) || !out) return FIDES_BAD_ARG;
    Guard g(c);
    const int n = a->level + 1, N = c->N;
    fides_ct tmp;
    fides_status s = ct_reserve(c, &tmp, a->level);
    if (s != FIDES_OK) return s;
    for (int j0 = 0; j0 < n; j0 += kMaxLinLimbs) {
        const int nl = std::min(kMaxLinLimbs, n - j0);
        LinArgs la{};
        la.n = 1;
        la.q0 = j0;
        la.in0[0] = a->c0() + (size_t)j0 * N;
        la.in1[0] = a->c1(N) + (size_t)j0 * N;
        la.out0 = tmp.c0() + (size_t)j0 * N;
        la.out1 = tmp.c1(N) + (size_t)j0 * N;
        uint64_t zz[kMaxPrimes][2];
        int_const_limbs(c, z, n, zz);
        for (int j = 0; j < nl; ++j) {
            la.z[0][j][0] = zz[j0 + j][0];
            la.z[0][j][1] = zz[j0 + j][1];
        }
        launch_lincomb(c->dev, nl, la, c->st);
    }
    const fides_ct meta = *a;
    commit(c, out, tmp);
    out->level = meta.level;
    out->scale = meta.scale;
    out->noise_deg = meta.noise_deg;
    out->slots = meta.slots;
    return check_cuda(c, "mult_int");
}

fides_status fides_mult_monomial(fides_ctx* c, const fides_ct* a, uint32_t power, fides_ct* out) {
    if (!c || !valid_ct(c, a) || !out) return FIDES_BAD_ARG;
    Guard g(c);
    const int N = c->N;
    fides_ct tmp;
    fides_status s = ct_reserve(c, &tmp, a->level);
    if (s != FIDES_OK) return s;
    launch_mult_monomial(c->dev, a->level + 1, a->c0(), a->c1(N), tmp.c0(), tmp.c1(N), power % (2u * (uint32_t)N),
                         c->st);
    const fides_ct meta = *a;
    commit(c, out, tmp);
    out->level = meta.level;
    out->scale = meta.scale;
    out->noise_deg = meta.noise_deg;
    out->slots = meta.slots;
    return check_cuda(c, "mult_monomial");
}

// ModRaise: the residues of limb 0 (mod q_0), lifted to (-q_0/2, q_0/2] in
// coefficient form, reduced modulo every ciphertext modulus and transformed
// back: one INTT of 2 limbs, one forward NTT of 2L limbs whose prologue does
// the centred lift (the SwitchModulus of the rescale with source prime q_0).
fides_status fides_mod_raise(fides_ctx* c, const fides_ct* a, fides_ct* out) {
    if (!c || !valid_ct(c, a) || !out) return FIDES_BAD_ARG;
    Guard g(c);
    const int N = c->N, top = c->L - 1;
    fides_ct tmp;
    fides_status s = ct_reserve(c, &tmp, top);
    if (s != FIDES_OK) return s;
    LimbMap t{};
    t.nseg = 2;
    const uint64_t* ins[2] = {a->c0(), a->c1(N)};
    for (int i = 0; i < 2; ++i) {
        LimbSeg& g2 = t.seg[i];
        g2.in = ins[i];
        g2.out = c->ws1.T + (size_t)i * N;
        g2.count = 1;
        g2.skip_lo = 1;
        g2.nq = 1;
        g2.q0 = 0;
        g2.level = 0;
        t.total += 1;
    }
    ntt_inverse(c->dev, t, IL_PLAIN, IS_PLAIN, c->st);
    LimbMap m{};
    m.nseg = 2;
    uint64_t* os[2] = {tmp.c0(), tmp.c1(N)};
    for (int i = 0; i < 2; ++i) {
        LimbSeg& g2 = m.seg[i];
        g2.in = c->ws1.T + (size_t)i * N;
        g2.in_stride_zero = 1;
        g2.out = os[i];
        g2.count = top + 1;
        g2.skip_lo = top + 1;
        g2.nq = top + 1;
        g2.q0 = 0;
        g2.level = 0;  // source prime of the centred lift
        m.total += top + 1;
    }
    ntt_forward(c->dev, m, FL_SWITCHMOD, FS_PLAIN, c->st);
    const fides_ct meta = *a;
    commit(c, out, tmp);
    out->level = top;
    out->scale = meta.scale;
    out->noise_deg = meta.noise_deg;
    out->slots = meta.slots;
    return check_cuda(c, "mod_raise");
}

// Offsets split as o = g*bstep + b with g = floor(o / bstep), 0 <= b < bstep.
static int floor_div(int a, int b) {
    int q = a / b;
    if ((a % b) != 0 && ((a < 0) != (b < 0))) --q;
    return q;
}

namespace {
// Temporary ciphertexts released on the context stream when the call ends.
struct CtTemps {
    fides_ctx* c;
    std::vector<fides_ct*> v;
    fides_ct* make() {
        v.push_back(new fides_ct());
        return v.back();
    }
    ~CtTemps() {
        for (fides_ct* t : v) {
            if (t->buf) cudaFreeAsync(t->buf, c->st);
            delete t;
        }
    }
};
}  // namespace

fides_status fides_linear_transform(fides_ctx* c, const fides_ct* x, int n, const int32_t* offsets,
                                    const fides_pt* const* pts, int bstep, int rescale, fides_ct* out) {
    return fides_linear_transform_batch(c, 1, &x, n, offsets, pts, bstep, rescale, &out);
}

fides_status fides_linear_transform_batch(fides_ctx* c, int nx, const fides_ct* const* xs, int n,
                                          const int32_t* offsets, const fides_pt* const* pts, int bstep, int rescale,
                                          fides_ct* const* outs) {
    return linear_transform_batch(c, nx, xs, n, offsets, pts, bstep, rescale, outs, false);
}

}  // extern "C"

namespace {
// The giant-step rotations of the transform's inputs with one ModDown per
// input (eng_rotate_sum): inner[i] belongs to input owner[i] (runs of equal
// owners) and rotates by gidx[i]; each input's rotated sum is added to
// acc[owner] (copied when have_acc is 0).
fides_status giant_rotate_sum(fides_ctx* c, int level, const std::vector<const fides_ct*>& inner,
                              const std::vector<int32_t>& gidx, const std::vector<int>& owner,
                              std::vector<fides_ct*>& acc, std::vector<char>& have_acc, CtTemps& tmp) {
    const int N = c->N, nl = level + 1;
    const size_t bytes = (size_t)nl * c->limb_bytes();
    auto add_into = [&](int u, const fides_ct* r) -> fides_status {
        fides_ct* a = acc[u];
        if (!have_acc[u]) {
            fides_status s = ct_reserve(c, a, level);
            if (s != FIDES_OK) return s;
            cudaMemcpyAsync(a->c0(), r->c0(), bytes, cudaMemcpyDeviceToDevice, c->st);
            cudaMemcpyAsync(a->c1(N), r->c1(N), bytes, cudaMemcpyDeviceToDevice, c->st);
            have_acc[u] = 1;
            return FIDES_OK;
        }
        launch_elementwise(c->dev, EW_ADD, nl, 0, a->c0(), r->c0(), a->c0(), c->st);
        launch_elementwise(c->dev, EW_ADD, nl, 0, a->c1(N), r->c1(N), a->c1(N), c->st);
        return FIDES_OK;
    };
    std::vector<int> terms;  // rotations that need a key switch, in owner order
    std::vector<uint32_t> gal(inner.size());
    std::vector<const SwitchKey*> keys(inner.size(), nullptr);
    for (size_t i = 0; i < inner.size(); ++i) {
        gal[i] = fides_rotation_galois(c, gidx[i], inner[i]->slots > 0 ? inner[i]->slots : N / 2);
        if (gal[i] == 1) {  // a rotation by a multiple of the slot count
            fides_status s = add_into(owner[i], inner[i]);
            if (s != FIDES_OK) return s;
            continue;
        }
        auto it = c->galois_keys.find(gal[i]);
        if (it == c->galois_keys.end())
            return set_err(c, FIDES_KEY_MISSING, "no key for galois element " + std::to_string(gal[i]));
        keys[i] = &it->second;
        terms.push_back((int)i);
    }
    if (terms.empty()) return FIDES_OK;
    fides_status s = ws_reserve(c, c->wsb, std::min((int)terms.size(), kMaxBatch));
    if (s != FIDES_OK) return s;
    // batches of whole inputs, so that every input's rotations share one
    // ModDown; only an input with more rotations than a batch holds is split
    // (one ModDown per part)
    const int cap = c->wsb.cap;
    std::vector<std::pair<size_t, size_t>> pieces;  // [begin, end) in terms
    for (size_t t0 = 0; t0 < terms.size();) {
        size_t t1 = t0;
        while (t1 < terms.size() && owner[terms[t1]] == owner[terms[t0]] && t1 - t0 < (size_t)cap) ++t1;
        pieces.push_back({t0, t1});
        t0 = t1;
    }
    for (size_t p0 = 0; p0 < pieces.size();) {
        size_t p1 = p0, nbz = 0;
        while (p1 < pieces.size() && nbz + (pieces[p1].second - pieces[p1].first) <= (size_t)cap)
            nbz += pieces[p1].second - pieces[p1].first, ++p1;
        const int nb = (int)nbz;
        std::vector<const uint64_t*> c0(nb), c1(nb);
        std::vector<const SwitchKey*> kk(nb);
        std::vector<uint32_t> gg(nb);
        std::vector<int> start, runs;  // run r: elements start[r] .. start[r+1]-1 of input runs[r]
        int j = 0;
        for (size_t q = p0; q < p1; ++q) {
            start.push_back(j);
            runs.push_back(owner[terms[pieces[q].first]]);
            for (size_t t = pieces[q].first; t < pieces[q].second; ++t, ++j) {
                const int i = terms[t];
                c0[j] = inner[i]->c0();
                c1[j] = inner[i]->c1(N);
                kk[j] = keys[i];
                gg[j] = gal[i];
            }
        }
        start.push_back(nb);
        p0 = p1;
        const int nout = (int)runs.size();
        std::vector<fides_ct*> r(nout);
        std::vector<uint64_t*> o0(nout), o1(nout);
        for (int u = 0; u < nout; ++u) {
            r[u] = tmp.make();
            s = ct_reserve(c, r[u], level);
            if (s != FIDES_OK) return s;
            o0[u] = r[u]->c0();
            o1[u] = r[u]->c1(N);
        }
        eng_rotate_sum(c, c->wsb, level, nb, c0.data(), c1.data(), kk.data(), gg.data(), nout, start.data(),
                       o0.data(), o1.data());
        for (int u = 0; u < nout; ++u) {
            s = add_into(runs[u], r[u]);
            if (s != FIDES_OK) return s;
        }
    }
    return FIDES_OK;
}
}  // namespace

// The same transform of nx ciphertexts at one level: the baby steps are one
// hoisted rotation group per input, the giant rotations of every input form
// one batched key switch (nx times the elements per launch), with one
// ModDown per rotation or, when `boot` and the context's giant_moddown
// select it, one per input.
fides_status fides::linear_transform_batch(fides_ctx* c, int nx, const fides_ct* const* xs, int n,
                                           const int32_t* offsets, const fides_pt* const* pts, int bstep,
                                           int rescale, fides_ct* const* outs, bool boot) {
    if (!c || nx < 1 || !xs || !outs || n < 1 || !offsets || !pts || bstep < 1) return FIDES_BAD_ARG;
    for (int u = 0; u < nx; ++u)
        if (!valid_ct(c, xs[u]) || !outs[u] || xs[u]->level != xs[0]->level) return FIDES_BAD_ARG;
    Guard g(c);
    const int level = xs[0]->level, nl = level + 1, N = c->N;
    for (int k = 0; k < n; ++k)
        if (!pts[k] || !pts[k]->m || pts[k]->level < level) return FIDES_BAD_ARG;
    std::vector<int> baby(n);
    std::vector<int32_t> babies;
    std::map<int, std::vector<int>> groups;  // giant step -> terms
    for (int k = 0; k < n; ++k) {
        const int gs = floor_div(offsets[k], bstep);
        baby[k] = offsets[k] - gs * bstep;
        if (baby[k] && std::find(babies.begin(), babies.end(), baby[k]) == babies.end()) babies.push_back(baby[k]);
        groups[gs].push_back(k);
    }
    CtTemps tmp{c, {}};
    fides_status s = FIDES_OK;
    std::vector<fides_ct*> acc(nx);
    std::vector<char> have_acc(nx, 0);
    std::vector<const fides_ct*> inner;
    std::vector<int32_t> gidx;
    std::vector<int> owner;  // input of each giant-step term
    // baby steps of every input: hoisted rotations, grouped over the inputs
    std::vector<fides_ct*> bo((size_t)nx * babies.size());
    if (!babies.empty()) {
        for (auto& p : bo) p = tmp.make();
        std::vector<uint32_t> bgal(babies.size());
        for (size_t i = 0; i < babies.size(); ++i)
            bgal[i] = fides_rotation_galois(c, babies[i], xs[0]->slots > 0 ? xs[0]->slots : N / 2);
        bool grouped = std::find(bgal.begin(), bgal.end(), 1u) == bgal.end();
        for (int u = 1; u < nx; ++u) grouped = grouped && xs[u]->slots == xs[0]->slots;
        if (grouped) {
            s = rotate_many_groups(c, nx, xs, (int)babies.size(), bgal.data(), bo.data());
        } else {
            for (int u = 0; u < nx && s == FIDES_OK; ++u)
                s = fides_rotate_hoisted(c, xs[u], (int)babies.size(), babies.data(), bo.data() + (size_t)u * babies.size());
        }
        if (s != FIDES_OK) return s;
    }
    for (int u = 0; u < nx; ++u) {
        const fides_ct* x = xs[u];
        std::map<int, const fides_ct*> bct;
        bct[0] = x;
        for (size_t i = 0; i < babies.size(); ++i) bct[babies[i]] = bo[(size_t)u * babies.size() + i];
        const double sc = x->scale * pts[0]->scale;
        const int nd = x->noise_deg + pts[0]->noise_deg, sl = x->slots;
        acc[u] = tmp.make();
        for (auto& kv : groups) {
            const int gs = kv.first;
            const std::vector<int>& ks = kv.second;
            fides_ct* dst = gs == 0 ? acc[u] : tmp.make();
            s = ct_reserve(c, dst, level);
            if (s != FIDES_OK) return s;
            for (size_t k0 = 0; k0 < ks.size(); k0 += kMaxBatch) {
                DotArgs d{};
                d.n = (int)std::min(ks.size() - k0, (size_t)kMaxBatch);
                d.accumulate = k0 > 0;
                for (int j = 0; j < d.n; ++j) {
                    const fides_ct* b = bct[baby[ks[k0 + j]]];
                    d.c0[j] = b->c0();
                    d.c1[j] = b->c1(N);
                    d.p[j] = pts[ks[k0 + j]]->m;
                }
                d.o0 = dst->c0();
                d.o1 = dst->c1(N);
                launch_dot_pt(c->dev, nl, d, c->st);
            }
            dst->level = level;
            dst->scale = sc;
            dst->noise_deg = nd;
            dst->slots = sl;
            if (gs == 0) {
                have_acc[u] = 1;
            } else {
                inner.push_back(dst);
                gidx.push_back(gs * bstep);
                owner.push_back(u);
            }
        }
    }
    if (!inner.empty() && (c->giant_moddown == 2 || (c->giant_moddown == 1 && boot))) {
        s = giant_rotate_sum(c, level, inner, gidx, owner, acc, have_acc, tmp);
        if (s != FIDES_OK) return s;
    } else if (!inner.empty()) {
        std::vector<fides_ct*> rot;
        for (size_t i = 0; i < inner.size(); ++i) rot.push_back(tmp.make());
        s = fides_rotate_batch(c, (int)inner.size(), inner.data(), gidx.data(), rot.data());
        if (s != FIDES_OK) return s;
        const size_t bytes = (size_t)nl * c->limb_bytes();
        for (size_t i = 0; i < rot.size(); ++i) {
            fides_ct* a = acc[owner[i]];
            if (!have_acc[owner[i]]) {
                s = ct_reserve(c, a, level);
                if (s != FIDES_OK) return s;
                cudaMemcpyAsync(a->c0(), rot[i]->c0(), bytes, cudaMemcpyDeviceToDevice, c->st);
                cudaMemcpyAsync(a->c1(N), rot[i]->c1(N), bytes, cudaMemcpyDeviceToDevice, c->st);
                have_acc[owner[i]] = 1;
                continue;
            }
            launch_elementwise(c->dev, EW_ADD, nl, 0, a->c0(), rot[i]->c0(), a->c0(), c->st);
            launch_elementwise(c->dev, EW_ADD, nl, 0, a->c1(N), rot[i]->c1(N), a->c1(N), c->st);
        }
    }
    for (int u = 0; u < nx; ++u) {
        const double sc = xs[u]->scale * pts[0]->scale;
        const int nd = xs[u]->noise_deg + pts[0]->noise_deg, sl = xs[u]->slots;
        commit(c, outs[u], *acc[u]);
        outs[u]->level = level;
        outs[u]->scale = sc;
        outs[u]->noise_deg = nd;
        outs[u]->slots = sl;
    }
    if (rescale && level > 0) {
        s = rescale_batch(c, nx, outs);
        if (s != FIDES_OK) return s;
    }
    return check_cuda(c, "linear_transform");
}

extern "C" {

}  // extern "C"

struct fides_plan {
    uint64_t nkernels = 0;  // kernels per replay
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<fides_ct> inter;  // products feeding the rotations
    std::vector<fides_ct*> outs;  // written by every replay
};

extern "C" {

fides_status fides_plan_hmult_rotate(fides_ctx* c, int n, const fides_ct* const* a, const fides_ct* const* b,
                                     const int32_t* indices, int rescale, fides_ct* const* out, fides_plan** plan) {
    if (!c || n < 1 || !a || !b || !out || !plan) return FIDES_BAD_ARG;
    Guard g(c);
    *plan = nullptr;
    if (!c->has_relin) return set_err(c, FIDES_KEY_MISSING, "no relinearisation key");
    const int N = c->N;
    std::vector<int> lv(n), lv2(n);
    std::vector<uint32_t> gal(n, 1);
    std::vector<const SwitchKey*> keys(n, nullptr);
    for (int i = 0; i < n; ++i) {
        if (!valid_ct(c, a[i]) || !valid_ct(c, b[i]) || !out[i]) return FIDES_BAD_ARG;
        lv[i] = std::min(a[i]->level, b[i]->level);
        lv2[i] = (rescale && lv[i] > 0) ? lv[i] - 1 : lv[i];
        if (indices) {
            gal[i] = fides_rotation_galois(c, indices[i], std::max(a[i]->slots, b[i]->slots));
            if (gal[i] != 1) {
                auto it = c->galois_keys.find(gal[i]);
                if (it == c->galois_keys.end())
                    return set_err(c, FIDES_KEY_MISSING, "no key for galois element " + std::to_string(gal[i]));
                keys[i] = &it->second;
            }
        }
    }
    fides_status s = ws_reserve(c, c->wsb, std::min(n, kMaxBatch));
    if (s != FIDES_OK) return s;
    auto* p = new (std::nothrow) fides_plan();
    if (!p) return FIDES_OOM;
    const bool rot = indices != nullptr;
    if (rot) p->inter.resize(n);
    p->outs.assign(out, out + n);
    for (int i = 0; i < n; ++i) {
        if (rot) s = ct_reserve(c, &p->inter[i], lv2[i]);
        if (s == FIDES_OK) s = ct_reserve(c, out[i], lv2[i]);
        if (s != FIDES_OK) {
            fides_plan_free(c, p);
            return s;
        }
    }
    cudaStreamSynchronize(c->st);
    // capture: kernels and device-to-device copies only, no allocation
    const uint64_t k0count = launch_count();
    if (cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        fides_plan_free(c, p);
        return check_cuda(c, "begin capture");
    }
    auto stage_out = [&](int i) -> fides_ct* { return rot ? &p->inter[i] : out[i]; };
    for (auto& grp : level_groups(c, n, lv.data())) {
        const int level = lv[grp[0]];
        for (size_t k0 = 0; k0 < grp.size(); k0 += c->wsb.cap) {
            const int nb = (int)std::min(grp.size() - k0, (size_t)c->wsb.cap);
            std::vector<const uint64_t*> a0(nb), a1(nb), b0(nb), b1(nb);
            std::vector<uint64_t*> o0(nb), o1(nb);
            for (int j = 0; j < nb; ++j) {
                const int i = grp[k0 + j];
                a0[j] = a[i]->c0();
                a1[j] = a[i]->c1(N);
                b0[j] = b[i]->c0();
                b1[j] = b[i]->c1(N);
                o0[j] = stage_out(i)->c0();
                o1[j] = stage_out(i)->c1(N);
            }
            eng_hmult(c, c->wsb, level, nb, a0.data(), a1.data(), b0.data(), b1.data(), o0.data(), o1.data(),
                      rescale && level > 0, c->relin);
        }
    }
    if (rot) {
        for (auto& grp0 : level_groups(c, n, lv2.data())) {
            std::vector<int> grp;
            for (int i : grp0) {
                if (gal[i] == 1) {
                    const size_t bytes = (size_t)(lv2[i] + 1) * c->limb_bytes();
                    cudaMemcpyAsync(out[i]->c0(), p->inter[i].c0(), bytes, cudaMemcpyDeviceToDevice, c->st);
                    cudaMemcpyAsync(out[i]->c1(N), p->inter[i].c1(N), bytes, cudaMemcpyDeviceToDevice, c->st);
                } else {
                    grp.push_back(i);
                }
            }
            if (grp.empty()) continue;
            const int level = lv2[grp[0]];
            for (size_t k0 = 0; k0 < grp.size(); k0 += c->wsb.cap) {
                const int nb = (int)std::min(grp.size() - k0, (size_t)c->wsb.cap);
                std::vector<const uint64_t*> c0(nb), c1(nb);
                std::vector<uint64_t*> o0(nb), o1(nb);
                std::vector<const SwitchKey*> kk(nb);
                std::vector<uint32_t> gg(nb);
                for (int j = 0; j < nb; ++j) {
                    const int i = grp[k0 + j];
                    c0[j] = p->inter[i].c0();
                    c1[j] = p->inter[i].c1(N);
                    o0[j] = out[i]->c0();
                    o1[j] = out[i]->c1(N);
                    kk[j] = keys[i];
                    gg[j] = gal[i];
                }
                eng_rotate(c, c->wsb, level, nb, c0.data(), c1.data(), kk.data(), gg.data(), o0.data(), o1.data(),
                           false);
            }
        }
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t e1 = cudaStreamEndCapture(c->st, &graph);
    if (e1 != cudaSuccess || !graph) {
        fides_plan_free(c, p);
        return set_err(c, FIDES_CUDA_ERR, std::string("end capture: ") + cudaGetErrorString(e1));
    }
    p->graph = graph;
    p->nkernels = launch_count() - k0count;
    const cudaError_t e2 = cudaGraphInstantiate(&p->exec, graph, 0);
    if (e2 != cudaSuccess) {
        fides_plan_free(c, p);
        return set_err(c, FIDES_CUDA_ERR, std::string("graph instantiate: ") + cudaGetErrorString(e2));
    }
    for (int i = 0; i < n; ++i) {
        const double sc = a[i]->scale * b[i]->scale;
        const bool rs = rescale && lv[i] > 0;
        out[i]->level = lv2[i];
        out[i]->scale = rs ? sc / (double)c->host.prime[lv[i]] : sc;
        out[i]->noise_deg = a[i]->noise_deg + b[i]->noise_deg - (rs ? 1 : 0);
        out[i]->slots = std::max(a[i]->slots, b[i]->slots);
    }
    *plan = p;
    return check_cuda(c, "plan");
}

fides_status fides_plan_launch(fides_ctx* c, fides_plan* plan) {
    if (!c || !plan || !plan->exec) return FIDES_BAD_ARG;
    Guard g(c);
    for (fides_ct* o : plan->outs) ct_quiesce(c, o);  // pending downloads of the last replay's results
    count_launches((int)plan->nkernels);
    if (cudaGraphLaunch(plan->exec, c->st) != cudaSuccess) return check_cuda(c, "graph launch");
    return FIDES_OK;
}

fides_status fides_plan_free(fides_ctx* c, fides_plan* plan) {
    if (!c || !plan) return FIDES_BAD_ARG;
    Guard g(c);
    cudaStreamSynchronize(c->st);
    if (plan->exec) cudaGraphExecDestroy(plan->exec);
    if (plan->graph) cudaGraphDestroy(plan->graph);
    for (auto& t : plan->inter)
        if (t.buf) cudaFreeAsync(t.buf, c->st);
    delete plan;
    return FIDES_OK;
}

fides_status fides_ntt(fides_ctx* ctx, uint64_t* data, int prime0, int nlimbs, int inverse) {
    if (!ctx || !data || prime0 < 0 || nlimbs < 1 || prime0 + nlimbs > ctx->L + ctx->K || nlimbs > 65535)
        return FIDES_BAD_ARG;
    Guard g(ctx);
    LimbMap m = map_single(data, data, nlimbs, nlimbs, prime0);
    if (inverse)
        ntt_inverse(ctx->dev, m, IL_PLAIN, IS_PLAIN, ctx->st);
    else
        ntt_forward(ctx->dev, m, FL_PLAIN, FS_PLAIN, ctx->st);
    return check_cuda(ctx, "ntt");
}

fides_status fides_ntt_batch(fides_ctx* ctx, uint64_t* data, size_t poly_stride, int npoly, int prime0, int nlimbs,
                             int inverse) {
    if (!ctx || !data || npoly < 1 || npoly > 65535 || prime0 < 0 || nlimbs < 1 ||
        prime0 + nlimbs > ctx->L + ctx->K || poly_stride < (size_t)nlimbs * ctx->N)
        return FIDES_BAD_ARG;
    Guard g(ctx);
    LimbMap m = map_single(data, data, nlimbs, nlimbs, prime0);
    m.nb = npoly;
    m.seg[0].bstride = poly_stride;
    if (inverse)
        ntt_inverse(ctx->dev, m, IL_PLAIN, IS_PLAIN, ctx->st);
    else
        ntt_forward(ctx->dev, m, FL_PLAIN, FS_PLAIN, ctx->st);
    return check_cuda(ctx, "ntt batch");
}

fides_status fides_polymul(fides_ctx* ctx, const uint64_t* a, const uint64_t* b, uint64_t* c, uint64_t* a_ntt,
                           uint64_t* b_ntt, int prime0, int nlimbs) {
    if (!ctx || !a || !b || !c || !a_ntt || !b_ntt || prime0 < 0 || nlimbs < 1 ||
        prime0 + nlimbs > ctx->L + ctx->K || nlimbs > 32767)
        return FIDES_BAD_ARG;
    Guard g(ctx);
    LimbMap m{};
    m.nseg = 2;
    const uint64_t* ins[2] = {a, b};
    uint64_t* outs[2] = {a_ntt, b_ntt};
    for (int s = 0; s < 2; ++s) {
        LimbSeg& g2 = m.seg[s];
        g2.in = ins[s];
        g2.out = outs[s];
        g2.count = nlimbs;
        g2.skip_lo = nlimbs;
        g2.nq = nlimbs;
        g2.q0 = prime0;
        m.total += nlimbs;
    }
    ntt_forward(ctx->dev, m, FL_PLAIN, FS_PLAIN, ctx->st);
    ntt_inverse(ctx->dev, map_single(a_ntt, c, nlimbs, nlimbs, prime0, -1, b_ntt), IL_MUL, IS_PLAIN, ctx->st);
    return check_cuda(ctx, "polymul");
}

}  // extern "C"
