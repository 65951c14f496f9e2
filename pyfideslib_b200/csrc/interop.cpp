// interop.cpp -- raw-residue import and export in the shapes FIDESlib exchanges
// with OpenFHE: RawCipherText, RawPlainText and RawKeySwitchKey
// (src/CKKS/openfhe-interface/RawCiphertext.cuh:19-93), i.e. one vector of N
// words per limb with the limb's modulus beside it, in OpenFHE's EVALUATION
// (bit-reversed NTT) or COEFFICIENT format.
//
// Limbs are matched to the context's primes by their moduli (the reference
// loads key limbs the same way, through the moduli lists that
// loadDecompDigit receives, src/CKKS/LimbPartition.cu:1076).  Residues coming
// from outside are checked to be canonical on the host before they reach the
// exact kernels, which rely on it.
#include <cstring>
#include <new>

#include "context.hpp"

using namespace fides;

namespace {

struct Guard {
    std::lock_guard<std::recursive_mutex> lk;
    explicit Guard(fides_ctx* c) : lk(c->mu) { cudaSetDevice(c->device); }
};

// prime index of modulus q in the context (Q primes first), or -1
int prime_index(const fides_ctx* c, uint64_t q) {
    for (size_t i = 0; i < c->host.prime.size(); ++i)
        if (c->host.prime[i] == q) return (int)i;
    return -1;
}

bool canonical(const uint64_t* v, size_t n, uint64_t p) {
    uint64_t bad = 0;
    for (size_t j = 0; j < n; ++j) bad |= (uint64_t)(v[j] >= p);
    return bad == 0;
}

// In-place forward or inverse NTT of `nlimbs` limbs (primes 0..nlimbs-1).
fides_status transform(fides_ctx* c, uint64_t* d, int nlimbs, bool inverse) {
    LimbMap m = map_single(d, d, nlimbs, nlimbs, 0);
    if (inverse)
        ntt_inverse(c->dev, m, IL_PLAIN, IS_PLAIN, c->st);
    else
        ntt_forward(c->dev, m, FL_PLAIN, FS_PLAIN, c->st);
    return check_cuda(c, "raw format transform");
}

// Check a raw polynomial (numRes limbs over q_0..q_{numRes-1}) and gather it
// into one limb-major host buffer.
fides_status gather_q(fides_ctx* c, const uint64_t* const* sub, const uint64_t* moduli, int numRes,
                      std::vector<uint64_t>& out) {
    const size_t N = (size_t)c->N;
    out.resize((size_t)numRes * N);
    for (int i = 0; i < numRes; ++i) {
        if (!sub[i]) return set_err(c, FIDES_BAD_ARG, "raw import: null limb");
        if (moduli[i] != c->host.prime[i])
            return set_err(c, FIDES_BAD_ARG, "raw import: limb " + std::to_string(i) + " has modulus " +
                                                 std::to_string(moduli[i]) + ", the context's q_" +
                                                 std::to_string(i) + " is " + std::to_string(c->host.prime[i]));
        if (!canonical(sub[i], N, moduli[i]))
            return set_err(c, FIDES_BAD_ARG, "raw import: limb " + std::to_string(i) + " holds non-canonical residues");
        memcpy(out.data() + (size_t)i * N, sub[i], N * sizeof(uint64_t));
    }
    return FIDES_OK;
}

}  // namespace

extern "C" {

fides_status fides_ct_import_raw(fides_ctx* c, const fides_raw_ct* raw, fides_ct** out) {
    if (!c || !raw || !out || !raw->sub_0 || !raw->sub_1 || !raw->moduli) return FIDES_BAD_ARG;
    *out = nullptr;
    if (raw->N != c->N || raw->numRes < 1 || raw->numRes > c->L ||
        (raw->format != FIDES_FORMAT_EVALUATION && raw->format != FIDES_FORMAT_COEFFICIENT))
        return set_err(c, FIDES_BAD_ARG, "raw import: ring dimension, limb count or format does not fit the context");
    Guard g(c);
    std::vector<uint64_t> h0, h1;
    fides_status s = gather_q(c, raw->sub_0, raw->moduli, raw->numRes, h0);
    if (s == FIDES_OK) s = gather_q(c, raw->sub_1, raw->moduli, raw->numRes, h1);
    if (s != FIDES_OK) return s;
    fides_ct* ct = nullptr;
    s = fides_ct_upload(c, h0.data(), h1.data(), raw->numRes - 1, raw->Noise, raw->NoiseLevel, raw->slots, &ct);
    if (s != FIDES_OK) return s;
    if (raw->format == FIDES_FORMAT_COEFFICIENT) {
        s = transform(c, ct->c0(), raw->numRes, false);
        if (s == FIDES_OK) s = transform(c, ct->c1(c->N), raw->numRes, false);
    }
    // the host staging buffers are released on return: wait for the copies
    cudaStreamSynchronize(c->h2d);
    if (s != FIDES_OK) {
        fides_ct_free(c, ct);
        return s;
    }
    *out = ct;
    return check_cuda(c, "raw ciphertext import");
}

fides_status fides_ct_export_raw(fides_ctx* c, const fides_ct* ct, fides_raw_ct* raw) {
    if (!c || !ct || !raw || !raw->sub_0 || !raw->sub_1 || !raw->moduli || !ct->buf) return FIDES_BAD_ARG;
    const int n = ct->level + 1;
    if (raw->numRes < n || (raw->format != FIDES_FORMAT_EVALUATION && raw->format != FIDES_FORMAT_COEFFICIENT))
        return set_err(c, FIDES_BAD_ARG, "raw export: fewer limb buffers than the ciphertext has limbs, or bad format");
    for (int i = 0; i < n; ++i)
        if (!raw->sub_0[i] || !raw->sub_1[i]) return set_err(c, FIDES_BAD_ARG, "raw export: null limb buffer");
    Guard g(c);
    ct_quiesce(c, ct);
    const size_t N = (size_t)c->N, bytes = N * sizeof(uint64_t);
    const uint64_t* src0 = ct->c0();
    const uint64_t* src1 = ct->c1(c->N);
    uint64_t* tmp = nullptr;
    if (raw->format == FIDES_FORMAT_COEFFICIENT) {
        if (cudaMallocAsync((void**)&tmp, 2 * (size_t)n * bytes, c->st) != cudaSuccess) {
            cudaGetLastError();
            return set_err(c, FIDES_OOM, "raw export: scratch allocation failed");
        }
        cudaMemcpyAsync(tmp, src0, (size_t)n * bytes, cudaMemcpyDeviceToDevice, c->st);
        cudaMemcpyAsync(tmp + (size_t)n * N, src1, (size_t)n * bytes, cudaMemcpyDeviceToDevice, c->st);
        fides_status s = transform(c, tmp, n, true);
        if (s == FIDES_OK) s = transform(c, tmp + (size_t)n * N, n, true);
        if (s != FIDES_OK) {
            cudaFreeAsync(tmp, c->st);
            return s;
        }
        src0 = tmp;
        src1 = tmp + (size_t)n * N;
    }
    for (int i = 0; i < n; ++i) {
        cudaMemcpyAsync(raw->sub_0[i], src0 + (size_t)i * N, bytes, cudaMemcpyDeviceToHost, c->st);
        cudaMemcpyAsync(raw->sub_1[i], src1 + (size_t)i * N, bytes, cudaMemcpyDeviceToHost, c->st);
        raw->moduli[i] = c->host.prime[i];
    }
    if (tmp) cudaFreeAsync(tmp, c->st);
    cudaStreamSynchronize(c->st);
    raw->numRes = n;
    raw->N = c->N;
    raw->Noise = ct->scale;
    raw->NoiseLevel = ct->noise_deg;
    raw->slots = ct->slots;
    const fides_status s = check_cuda(c, "raw ciphertext export");
    return s != FIDES_OK ? s : consume_device_error(c);
}

fides_status fides_pt_import_raw(fides_ctx* c, const fides_raw_pt* raw, fides_pt** out) {
    if (!c || !raw || !out || !raw->sub_0 || !raw->moduli) return FIDES_BAD_ARG;
    *out = nullptr;
    if (raw->N != c->N || raw->numRes < 1 || raw->numRes > c->L ||
        (raw->format != FIDES_FORMAT_EVALUATION && raw->format != FIDES_FORMAT_COEFFICIENT))
        return set_err(c, FIDES_BAD_ARG, "raw import: ring dimension, limb count or format does not fit the context");
    Guard g(c);
    std::vector<uint64_t> h;
    fides_status s = gather_q(c, raw->sub_0, raw->moduli, raw->numRes, h);
    if (s != FIDES_OK) return s;
    fides_pt* pt = nullptr;
    s = fides_pt_upload(c, h.data(), raw->numRes - 1, raw->Noise, raw->NoiseLevel, raw->slots, &pt);
    if (s != FIDES_OK) return s;
    if (raw->format == FIDES_FORMAT_COEFFICIENT) s = transform(c, pt->m, raw->numRes, false);
    cudaStreamSynchronize(c->st);  // the upload reads the host staging buffer
    if (s != FIDES_OK) {
        fides_pt_free(c, pt);
        return s;
    }
    *out = pt;
    return check_cuda(c, "raw plaintext import");
}

fides_status fides_key_import_raw(fides_ctx* c, uint32_t galois, const fides_raw_key* raw) {
    if (!c || !raw || !raw->r_key || !raw->r_key_moduli) return FIDES_BAD_ARG;
    const int np = c->L + c->K;
    if (raw->N != c->N || raw->dnum != c->dnum || raw->nlimbs != np)
        return set_err(c, FIDES_BAD_ARG, "raw key: ring dimension, digit count or limb count does not fit the context");
    Guard g(c);
    const size_t N = (size_t)c->N, words = (size_t)c->dnum * np * N;
    std::vector<uint64_t> half[2] = {std::vector<uint64_t>(words), std::vector<uint64_t>(words)};  // a, b
    for (int h = 0; h < 2; ++h)
        for (int d = 0; d < c->dnum; ++d) {
            std::vector<char> seen(np, 0);
            for (int i = 0; i < np; ++i) {
                const size_t k = ((size_t)h * c->dnum + d) * np + i;
                const uint64_t q = raw->r_key_moduli[k];
                const int pi = prime_index(c, q);
                if (pi < 0 || seen[pi])
                    return set_err(c, FIDES_BAD_ARG, "raw key: modulus " + std::to_string(q) +
                                                         " is not one of the context's primes, or repeats");
                seen[pi] = 1;
                if (!raw->r_key[k] || !canonical(raw->r_key[k], N, q))
                    return set_err(c, FIDES_BAD_ARG, "raw key: null limb or non-canonical residues");
                memcpy(half[h].data() + ((size_t)d * np + pi) * N, raw->r_key[k], N * sizeof(uint64_t));
            }
        }
    // RawKeySwitchKey holds the a half first, then b
    return galois == 0 ? fides_key_upload_relin(c, half[1].data(), half[0].data())
                       : fides_key_upload_galois(c, galois, half[1].data(), half[0].data());
}

fides_status fides_key_export_raw(fides_ctx* c, uint32_t galois, fides_raw_key* raw) {
    if (!c || !raw || !raw->r_key || !raw->r_key_moduli) return FIDES_BAD_ARG;
    const int np = c->L + c->K;
    if (raw->dnum != c->dnum || raw->nlimbs != np)
        return set_err(c, FIDES_BAD_ARG, "raw key export: digit or limb count does not fit the context");
    const size_t N = (size_t)c->N, words = (size_t)c->dnum * np * N;
    std::vector<uint64_t> b(words), a(words);
    fides_status s = fides_key_export(c, galois, b.data(), a.data());
    if (s != FIDES_OK) return s;
    for (int h = 0; h < 2; ++h)
        for (int d = 0; d < c->dnum; ++d)
            for (int i = 0; i < np; ++i) {
                const size_t k = ((size_t)h * c->dnum + d) * np + i;
                if (!raw->r_key[k]) return set_err(c, FIDES_BAD_ARG, "raw key export: null limb buffer");
                memcpy(raw->r_key[k], (h == 0 ? a : b).data() + ((size_t)d * np + i) * N, N * sizeof(uint64_t));
                raw->r_key_moduli[k] = c->host.prime[i];
            }
    raw->N = c->N;
    return FIDES_OK;
}

}  // extern "C"
