// fideslib.hpp -- C++ mirror of FIDESlib's public API (api/fideslib.hpp) over
// the C ABI in include/fides_b200.h.  Header-only; link libfidesb200.so.
//
// The names, argument meanings and ownership follow the reference surface
// (api/CryptoContext.hpp:24-245, api/Ciphertext.hpp:13-56,
// api/Plaintext.hpp:15-58, api/CCParams.hpp, api/Definitions.hpp):
//   * CryptoContext / Ciphertext / Plaintext are shared_ptr handles; the
//     device objects live behind C-ABI handles owned by the context.
//   * Operations return new ciphertexts; the *InPlace variants overwrite.
//   * Errors throw fideslib::Exception (the reference throws OPENFHE_THROW at
//     the API; its CUDA errors exit, ours come back as a status).
// The client-side operations (KeyGen, Encrypt, Decrypt, encoding) that the
// reference delegates to OpenFHE are served by the library's own client half.
// Scaling: FIXEDMANUAL (explicit Rescale) and FLEXIBLEAUTO / FIXEDAUTO (inputs
// of degree 2 are rescaled before the next multiplication; levels aligned
// before additions), as Ciphertext.cpp:409-423 / adjustForMult does.
#pragma once
#include <complex>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../../include/fides_b200.h"

namespace fideslib {

class Exception : public std::runtime_error {
  public:
    Exception(fides_status s, const std::string& what) : std::runtime_error(what), status(s) {}
    fides_status status;
};

enum ScalingTechnique { FIXEDMANUAL = 0, FIXEDAUTO, FLEXIBLEAUTO, FLEXIBLEAUTOEXT, NORESCALE };
enum KeySwitchTechnique { INVALID_KS_TECH = 0, BV, HYBRID };
enum SecretKeyDist { GAUSSIAN = 0, UNIFORM_TERNARY = 1, SPARSE_TERNARY = 2 };
enum PKESchemeFeature { PKE = 0x01, KEYSWITCH = 0x02, LEVELEDSHE = 0x08, ADVANCEDSHE = 0x10, FHE = 0x40 };
struct DCRTPoly {};
struct CryptoContextCKKSRNS {};
enum Format { EVALUATION = 0, COEFFICIENT = 1 };

// The raw-residue shapes FIDESlib exchanges with OpenFHE
// (src/CKKS/openfhe-interface/RawCiphertext.cuh:19-93), without the OpenFHE
// objects they were read from: one vector of N words per limb, limb i mod
// moduli[i], EVALUATION meaning OpenFHE's bit-reversed NTT order.
struct RawCipherText {
    std::vector<std::vector<uint64_t>> sub_0, sub_1;
    std::vector<uint64_t> moduli;
    int numRes = 0;
    int N = 0;
    Format format = EVALUATION;
    double Noise = 0;
    int NoiseLevel = 1;
    int slots = 0;
};
struct RawPlainText {
    std::vector<std::vector<uint64_t>> sub_0;
    std::vector<uint64_t> moduli;
    int numRes = 0;
    int N = 0;
    Format format = EVALUATION;
    double Noise = 0;
    int slots = 0;
    int NoiseLevel = 1;
};
// The part of the reference's RawParams (src/CKKS/openfhe-interface/
// RawCiphertext.cuh:50-88) a context is built from when OpenFHE supplies it:
// the moduli and the 2N-th roots of unity that fix OpenFHE's evaluation
// representation (SetupConstants takes them, src/ConstantsGPU.cu:195-199).
// L counts the levels: moduli holds L + 1 entries.
struct RawParams {
    int N = 0, L = 0, K = 0, logN = 0, dnum = 0;
    std::vector<uint64_t> moduli, root_of_unity, SPECIALmoduli, SPECIALroot_of_unity;
};

// r_key[h][d][i]: half h (0 = a, 1 = b), digit d, limb i; r_key_moduli alike
struct RawKeySwitchKey {
    std::vector<std::vector<std::vector<uint64_t>>> r_key_moduli;
    std::vector<std::vector<std::vector<std::vector<uint64_t>>>> r_key;
    std::string keyid;
};

template <typename T>
class CCParams;

template <>
class CCParams<CryptoContextCKKSRNS> {
  public:
    void SetMultiplicativeDepth(uint32_t d) { depth = d; }
    void SetScalingModSize(uint32_t s) { scaleBits = s; }
    void SetFirstModSize(uint32_t s) { firstBits = s; }
    void SetBatchSize(uint32_t b) { batch = b; }
    void SetRingDim(uint32_t n) { ringDim = n; }
    void SetScalingTechnique(ScalingTechnique t) { tech = t; }
    void SetNumLargeDigits(uint32_t d) { dnum = d; }
    void SetKeySwitchTechnique(KeySwitchTechnique) {}
    void SetSecretKeyDist(SecretKeyDist d) { keyDist = d; }
    void SetSecretKeyHammingWeight(uint32_t h) { hamming = h; }
    void SetDevices(std::vector<int>&& d) { devices = std::move(d); }
    uint32_t GetMultiplicativeDepth() const { return depth; }
    uint32_t GetBatchSize() const { return batch; }
    SecretKeyDist GetSecretKeyDist() const { return keyDist; }

    uint32_t depth = 1, scaleBits = 50, firstBits = 60, batch = 0, ringDim = 1 << 16, dnum = 3, hamming = 192;
    ScalingTechnique tech = FLEXIBLEAUTO;
    SecretKeyDist keyDist = UNIFORM_TERNARY;
    std::vector<int> devices = {0};
};

inline void check(fides_status s, const fides_ctx* c = nullptr) {
    if (s != FIDES_OK) throw Exception(s, std::string("fides status ") + std::to_string((int)s) + ": " +
                                              (c ? fides_ctx_last_error(c) : ""));
}

template <typename T>
class CryptoContextImpl;

class CiphertextImpl {
  public:
    CiphertextImpl(fides_ctx* c, fides_ct* h) : ctx(c), handle(h), loaded(h != nullptr) {}
    // host-side (raw) ciphertext, moved to the device by LoadCiphertext
    CiphertextImpl(fides_ctx* c, RawCipherText r)
        : ctx(c), handle(nullptr), raw(std::make_shared<RawCipherText>(std::move(r))), loaded(false) {}
    ~CiphertextImpl() {
        if (handle) fides_ct_free(ctx, handle);
    }
    CiphertextImpl(const CiphertextImpl&) = delete;
    CiphertextImpl& operator=(const CiphertextImpl&) = delete;
    uint32_t GetLevel() const {
        int l = 0;
        fides_ct_info(handle, &l, nullptr, nullptr, nullptr);
        return (uint32_t)l;
    }
    size_t GetNoiseScaleDeg() const {
        int d = 0;
        fides_ct_info(handle, nullptr, nullptr, &d, nullptr);
        return (size_t)d;
    }
    double GetScalingFactor() const {
        double s = 0;
        fides_ct_info(handle, nullptr, &s, nullptr, nullptr);
        return s;
    }
    uint32_t GetSlots() const {
        int s = 0;
        fides_ct_info(handle, nullptr, nullptr, nullptr, &s);
        return (uint32_t)s;
    }
    fides_ctx* ctx;
    fides_ct* handle;
    std::shared_ptr<RawCipherText> raw;
    bool loaded;
};
template <typename T = DCRTPoly>
using Ciphertext = std::shared_ptr<CiphertextImpl>;

class PlaintextImpl {
  public:
    PlaintextImpl(fides_ctx* c, fides_pt* h, uint32_t s) : ctx(c), handle(h), slots(s), loaded(h != nullptr) {}
    PlaintextImpl(fides_ctx* c, RawPlainText r)
        : ctx(c), handle(nullptr), slots((uint32_t)r.slots), raw(std::make_shared<RawPlainText>(std::move(r))),
          loaded(false) {}
    ~PlaintextImpl() {
        if (handle) fides_pt_free(ctx, handle);
    }
    void SetLength(size_t n) { length = n; }
    void SetSlots(uint32_t s) { slots = s; }
    std::vector<std::complex<double>> GetCKKSPackedValue() const {
        return std::vector<std::complex<double>>(values.begin(), values.begin() + std::min(length, values.size()));
    }
    std::vector<double> GetRealPackedValue() const {
        std::vector<double> r;
        for (size_t i = 0; i < std::min(length, values.size()); ++i) r.push_back(values[i].real());
        return r;
    }
    fides_ctx* ctx;
    fides_pt* handle;
    uint32_t slots;
    std::shared_ptr<RawPlainText> raw;
    bool loaded;
    size_t length = 0;
    std::vector<std::complex<double>> values;
};
using Plaintext = std::shared_ptr<PlaintextImpl>;

template <typename T>
struct PrivateKeyImpl {
    fides_ctx* ctx = nullptr;
    fides_sk* handle = nullptr;
    ~PrivateKeyImpl() {
        if (handle) fides_sk_free(ctx, handle);
    }
};
template <typename T>
using PrivateKey = std::shared_ptr<PrivateKeyImpl<T>>;
template <typename T>
struct PublicKeyImpl {
    fides_ctx* ctx = nullptr;
    fides_pk* handle = nullptr;
    ~PublicKeyImpl() {
        if (handle) fides_pk_free(ctx, handle);
    }
};
template <typename T>
using PublicKey = std::shared_ptr<PublicKeyImpl<T>>;
template <typename T>
struct KeyPair {
    PublicKey<T> publicKey;
    PrivateKey<T> secretKey;
};
using DecryptResult = bool;

template <>
class CryptoContextImpl<DCRTPoly> {
  public:
    explicit CryptoContextImpl(const CCParams<CryptoContextCKKSRNS>& p) : tech(p.tech), hamming(p.hamming) {
        fides_params prm{};
        prm.log_n = 0;
        for (uint32_t n = p.ringDim; n > 1; n >>= 1) ++prm.log_n;
        prm.num_q = (int)p.depth + 1;
        prm.dnum = (int)p.dnum;
        prm.q0_bits = (int)p.firstBits;
        prm.qi_bits = (int)p.scaleBits;
        prm.p_bits = 60;
        prm.device = p.devices.empty() ? 0 : p.devices[0];
        check(fides_ctx_create(&prm, &ctx));
        slots = p.batch ? p.batch : (1u << prm.log_n) / 2;
        sparse = p.keyDist == SPARSE_TERNARY;
    }
    // A context over OpenFHE's moduli and roots (the reference builds its
    // CKKS::Context from RawParams the same way, src/CKKS/Context.cu:37-98),
    // so that raw ciphertexts and keys in EVALUATION format load unchanged.
    CryptoContextImpl(const CCParams<CryptoContextCKKSRNS>& p, const RawParams& raw)
        : tech(p.tech), hamming(p.hamming) {
        if (raw.moduli.empty() || raw.root_of_unity.size() != raw.moduli.size() ||
            raw.SPECIALroot_of_unity.size() != raw.SPECIALmoduli.size())
            throw Exception(FIDES_BAD_ARG, "RawParams: moduli and roots of unity differ in count");
        fides_params prm{};
        prm.log_n = raw.logN;
        prm.num_q = (int)raw.moduli.size();
        prm.num_p = (int)raw.SPECIALmoduli.size();
        prm.dnum = raw.dnum > 0 ? raw.dnum : (int)p.dnum;
        prm.q = raw.moduli.data();
        prm.p = raw.SPECIALmoduli.empty() ? nullptr : raw.SPECIALmoduli.data();
        prm.q_root = raw.root_of_unity.data();
        prm.p_root = raw.SPECIALroot_of_unity.empty() ? nullptr : raw.SPECIALroot_of_unity.data();
        prm.qi_bits = (int)p.scaleBits;
        prm.device = p.devices.empty() ? 0 : p.devices[0];
        check(fides_ctx_create(&prm, &ctx));
        slots = p.batch ? p.batch : (1u << prm.log_n) / 2;
        sparse = p.keyDist == SPARSE_TERNARY;
    }
    ~CryptoContextImpl() {
        if (ctx) fides_ctx_destroy(ctx);
    }
    CryptoContextImpl(const CryptoContextImpl&) = delete;

    void Enable(PKESchemeFeature) {}
    uint32_t GetRingDimension() const {
        int l = 0;
        fides_ctx_info(ctx, &l, nullptr, nullptr, nullptr, nullptr, nullptr);
        return 1u << l;
    }
    uint32_t GetCyclotomicOrder() const { return 2 * GetRingDimension(); }
    void Enable(uint32_t) {}
    // The bootstrap here takes its input at any scale and level (it reads the
    // first limb and tracks the scale exactly), so no pre-scaling is needed:
    // the factor a caller multiplies by before a `prescaled` EvalBootstrap
    // (api/CryptoContext.cpp:148-153) is 1.
    double GetPreScaleFactor(uint32_t) const { return 1.0; }
    // Ciphertexts and plaintexts of this API live on the device from the
    // start; there is nothing to load lazily (api/CryptoContext.cpp:158-165).
    void SetAutoLoadPlaintexts(bool) {}
    void SetAutoLoadCiphertexts(bool) {}

    KeyPair<DCRTPoly> KeyGen() {
        KeyPair<DCRTPoly> kp;
        kp.secretKey = std::make_shared<PrivateKeyImpl<DCRTPoly>>();
        kp.secretKey->ctx = ctx;
        check(fides_keygen(ctx, seed++, sparse ? (int)hamming : 0, &kp.secretKey->handle), ctx);
        kp.publicKey = std::make_shared<PublicKeyImpl<DCRTPoly>>();
        kp.publicKey->ctx = ctx;
        check(fides_keygen_public(ctx, kp.secretKey->handle, seed++, &kp.publicKey->handle), ctx);
        return kp;
    }
    void EvalMultKeyGen(const PrivateKey<DCRTPoly>& sk) { check(fides_keygen_relin(ctx, sk->handle, seed++), ctx); }
    void EvalRotateKeyGen(const PrivateKey<DCRTPoly>& sk, const std::vector<int32_t>& steps) {
        check(fides_keygen_rotations(ctx, sk->handle, (int)steps.size(), steps.data(), (int)slots, seed++), ctx);
    }
    void EvalConjugateKeyGen(const PrivateKey<DCRTPoly>& sk) { check(fides_keygen_conjugate(ctx, sk->handle, seed++), ctx); }
    // ---- loading (api/CryptoContext.hpp:60-66) ----
    // Raw switching keys (RawKeySwitchKey, e.g. read from OpenFHE) queued here
    // are uploaded by LoadContext, as the reference loads the OpenFHE
    // context's evaluation keys there (api/CryptoContext.cpp:176-228).  Keys
    // made by EvalMultKeyGen / EvalRotateKeyGen are device-resident already.
    void AddEvalMultKey(RawKeySwitchKey k) { pending.emplace_back(0u, std::move(k)); }
    void AddRotationKey(int32_t index, RawKeySwitchKey k) {
        pending.emplace_back(fides_rotation_galois(ctx, index, (int)slots), std::move(k));
    }
    void LoadContext(const PublicKey<DCRTPoly>&) {
        for (auto& pk : pending) load_key(pk.first, pk.second);
        pending.clear();
        loadedCtx = true;
    }
    void LoadCiphertext(Ciphertext<DCRTPoly>& ct) {
        if (ct->loaded) return;
        auto& r = *ct->raw;
        std::vector<uint64_t*> p0, p1;
        for (auto& v : r.sub_0) p0.push_back(v.data());
        for (auto& v : r.sub_1) p1.push_back(v.data());
        fides_raw_ct rc{p0.data(), p1.data(), r.moduli.data(), r.numRes, r.N, (int)r.format,
                        r.Noise, r.NoiseLevel, r.slots};
        check(fides_ct_import_raw(ctx, &rc, &ct->handle), ctx);
        ct->loaded = true;
    }
    void LoadPlaintext(Plaintext& pt) {
        if (pt->loaded) return;
        auto& r = *pt->raw;
        std::vector<uint64_t*> p0;
        for (auto& v : r.sub_0) p0.push_back(v.data());
        fides_raw_pt rp{p0.data(), r.moduli.data(), r.numRes, r.N, (int)r.format, r.Noise, r.NoiseLevel, r.slots};
        check(fides_pt_import_raw(ctx, &rp, &pt->handle), ctx);
        pt->loaded = true;
    }
    // A host-side ciphertext / plaintext from raw residues (what
    // GetRawCipherText / GetRawPlainText return for an OpenFHE object); it
    // is moved to the device by LoadCiphertext / LoadPlaintext.
    Ciphertext<DCRTPoly> CiphertextFromRaw(RawCipherText r) { return std::make_shared<CiphertextImpl>(ctx, std::move(r)); }
    Plaintext PlaintextFromRaw(RawPlainText r) { return std::make_shared<PlaintextImpl>(ctx, std::move(r)); }
    // The raw residues of a device ciphertext (GetRawCipherText,
    // src/CKKS/openfhe-interface/RawCiphertext.cu:48-75), in either format.
    RawCipherText GetRawCipherText(const Ciphertext<DCRTPoly>& ct, Format f = EVALUATION) {
        RawCipherText r;
        const int n = (int)ct->GetLevel() + 1;
        const size_t N = GetRingDimension();
        r.sub_0.assign(n, std::vector<uint64_t>(N));
        r.sub_1.assign(n, std::vector<uint64_t>(N));
        r.moduli.assign(n, 0);
        std::vector<uint64_t*> p0, p1;
        for (auto& v : r.sub_0) p0.push_back(v.data());
        for (auto& v : r.sub_1) p1.push_back(v.data());
        fides_raw_ct rc{p0.data(), p1.data(), r.moduli.data(), n, (int)N, (int)f, 0.0, 0, 0};
        check(fides_ct_export_raw(ctx, ct->handle, &rc), ctx);
        r.numRes = rc.numRes;
        r.N = rc.N;
        r.format = f;
        r.Noise = rc.Noise;
        r.NoiseLevel = rc.NoiseLevel;
        r.slots = rc.slots;
        return r;
    }

    Plaintext MakeCKKSPackedPlaintext(const std::vector<std::complex<double>>& v, size_t noiseScaleDeg = 1,
                                      uint32_t level = 0, std::shared_ptr<void> = nullptr, uint32_t nslots = 0) {
        const uint32_t s = nslots ? nslots : slots;
        int L = 0;
        fides_ctx_info(ctx, nullptr, &L, nullptr, nullptr, nullptr, nullptr);
        const int lv = L - 1 - (int)level;  // OpenFHE's level counts consumed levels
        std::vector<double> iv(2 * s, 0.0);
        for (size_t i = 0; i < v.size() && i < s; ++i) {
            iv[2 * i] = v[i].real();
            iv[2 * i + 1] = v[i].imag();
        }
        const double sc = scale_for(noiseScaleDeg);
        std::vector<uint64_t> m((size_t)(lv + 1) * GetRingDimension());
        check(fides_encode(ctx, iv.data(), (int)s, lv, sc, m.data()), ctx);
        fides_pt* h = nullptr;
        check(fides_pt_upload(ctx, m.data(), lv, sc, (int)noiseScaleDeg, (int)s, &h), ctx);
        auto pt = std::make_shared<PlaintextImpl>(ctx, h, s);
        pt->values = v;
        pt->length = v.size();
        return pt;
    }
    Plaintext MakeCKKSPackedPlaintext(const std::vector<double>& v, size_t noiseScaleDeg = 1, uint32_t level = 0,
                                      std::shared_ptr<void> params = nullptr, uint32_t nslots = 0) {
        std::vector<std::complex<double>> c(v.begin(), v.end());
        return MakeCKKSPackedPlaintext(c, noiseScaleDeg, level, params, nslots);
    }

    Ciphertext<DCRTPoly> Encrypt(const PublicKey<DCRTPoly>& pk, Plaintext& pt) {
        fides_ct* h = nullptr;
        auto iv = interleave(pt);
        check(fides_encrypt_pk(ctx, pk->handle, iv.data(), (int)pt->slots, top_level(), scale_for(1), seed++, &h), ctx);
        return wrap(h);
    }
    Ciphertext<DCRTPoly> Encrypt(Plaintext& pt, const PublicKey<DCRTPoly>& pk) { return Encrypt(pk, pt); }
    Ciphertext<DCRTPoly> Encrypt(const PrivateKey<DCRTPoly>& sk, Plaintext& pt) {
        fides_ct* h = nullptr;
        auto iv = interleave(pt);
        check(fides_encrypt(ctx, sk->handle, iv.data(), (int)pt->slots, top_level(), scale_for(1), seed++, &h), ctx);
        return wrap(h);
    }
    DecryptResult Decrypt(const PrivateKey<DCRTPoly>& sk, Ciphertext<DCRTPoly>& ct, Plaintext* out) {
        const uint32_t s = ct->GetSlots() ? ct->GetSlots() : slots;
        std::vector<double> v(2 * s);
        check(fides_decrypt(ctx, sk->handle, ct->handle, v.data(), (int)s), ctx);
        auto pt = std::make_shared<PlaintextImpl>(ctx, nullptr, s);
        for (uint32_t i = 0; i < s; ++i) pt->values.emplace_back(v[2 * i], v[2 * i + 1]);
        pt->length = s;
        *out = pt;
        return true;
    }
    DecryptResult Decrypt(Ciphertext<DCRTPoly>& ct, const PrivateKey<DCRTPoly>& sk, Plaintext* out) {
        return Decrypt(sk, ct, out);
    }

    // ---- evaluation ----
    Ciphertext<DCRTPoly> EvalAdd(const Ciphertext<DCRTPoly>& a, const Ciphertext<DCRTPoly>& b) {
        auto x = match(a, b);
        return op2(fides_add, x.first, x.second);
    }
    Ciphertext<DCRTPoly> EvalSub(const Ciphertext<DCRTPoly>& a, const Ciphertext<DCRTPoly>& b) {
        auto x = match(a, b);
        return op2(fides_sub, x.first, x.second);
    }
    Ciphertext<DCRTPoly> EvalAdd(const Ciphertext<DCRTPoly>& a, Plaintext& p) {
        auto o = empty();
        check(fides_add_pt(ctx, a->handle, p->handle, o->handle), ctx);
        return o;
    }
    Ciphertext<DCRTPoly> EvalAdd(const Ciphertext<DCRTPoly>& a, double v) {
        auto o = empty();
        check(fides_add_scalar(ctx, a->handle, v, o->handle), ctx);
        return o;
    }
    Ciphertext<DCRTPoly> EvalNegate(const Ciphertext<DCRTPoly>& a) {
        auto o = empty();
        check(fides_negate(ctx, a->handle, o->handle), ctx);
        return o;
    }
    Ciphertext<DCRTPoly> EvalMult(const Ciphertext<DCRTPoly>& a, const Ciphertext<DCRTPoly>& b) {
        auto x = align(prepare(a), prepare(b));
        auto o = empty();
        check(fides_hmult(ctx, x.first->handle, x.second->handle, o->handle, 0), ctx);
        return o;
    }
    Ciphertext<DCRTPoly> EvalMult(const Ciphertext<DCRTPoly>& a, Plaintext& p) {
        auto o = empty();
        check(fides_mult_pt(ctx, prepare(a)->handle, p->handle, o->handle, 0), ctx);
        return o;
    }
    Ciphertext<DCRTPoly> EvalMult(const Ciphertext<DCRTPoly>& a, double v) {
        auto o = empty();
        check(fides_mult_scalar(ctx, prepare(a)->handle, v, o->handle, 0), ctx);
        return o;
    }
    Ciphertext<DCRTPoly> EvalSquare(const Ciphertext<DCRTPoly>& a) {
        auto o = empty();
        check(fides_square(ctx, prepare(a)->handle, o->handle, 0), ctx);
        return o;
    }
    // ---- the commuted, in-place, mutable and many-operand forms
    //      (api/CryptoContext.hpp:110-159); Mutable forms may rescale or
    //      level-align their operands in place, as OpenFHE's do ----
    void EvalNegateInPlace(Ciphertext<DCRTPoly>& a) { a = EvalNegate(a); }
    Ciphertext<DCRTPoly> EvalAdd(Plaintext& p, const Ciphertext<DCRTPoly>& a) { return EvalAdd(a, p); }
    Ciphertext<DCRTPoly> EvalAdd(double v, const Ciphertext<DCRTPoly>& a) { return EvalAdd(a, v); }
    void EvalAddInPlace(Ciphertext<DCRTPoly>& a, const Ciphertext<DCRTPoly>& b) { a = EvalAdd(a, b); }
    void EvalAddInPlace(Ciphertext<DCRTPoly>& a, Plaintext& p) { a = EvalAdd(a, p); }
    void EvalAddInPlace(Plaintext& p, Ciphertext<DCRTPoly>& a) { a = EvalAdd(a, p); }
    void EvalAddInPlace(Ciphertext<DCRTPoly>& a, double v) { a = EvalAdd(a, v); }
    void EvalAddInPlace(double v, Ciphertext<DCRTPoly>& a) { a = EvalAdd(a, v); }
    Ciphertext<DCRTPoly> EvalAddMutable(Ciphertext<DCRTPoly>& a, Ciphertext<DCRTPoly>& b) {
        auto x = match(a, b);
        a = x.first;
        b = x.second;
        return op2(fides_add, a, b);
    }
    Ciphertext<DCRTPoly> EvalAddMutable(Ciphertext<DCRTPoly>& a, Plaintext& p) { return EvalAdd(a, p); }
    Ciphertext<DCRTPoly> EvalAddMutable(Plaintext& p, Ciphertext<DCRTPoly>& a) { return EvalAdd(a, p); }
    void EvalAddMutableInPlace(Ciphertext<DCRTPoly>& a, Ciphertext<DCRTPoly>& b) { a = EvalAddMutable(a, b); }
    // Sum of many ciphertexts as a balanced tree of additions.
    Ciphertext<DCRTPoly> EvalAddMany(const std::vector<Ciphertext<DCRTPoly>>& cts) {
        if (cts.empty()) throw Exception(FIDES_BAD_ARG, "EvalAddMany: no ciphertexts");
        std::vector<Ciphertext<DCRTPoly>> v(cts);
        while (v.size() > 1) {
            std::vector<Ciphertext<DCRTPoly>> next;
            for (size_t i = 0; i + 1 < v.size(); i += 2) next.push_back(EvalAdd(v[i], v[i + 1]));
            if (v.size() & 1) next.push_back(v.back());
            v.swap(next);
        }
        return v[0];
    }
    void EvalAddManyInPlace(std::vector<Ciphertext<DCRTPoly>>& cts) {
        auto s = EvalAddMany(cts);
        cts[0] = s;
    }
    // ct - pt = -(-ct + pt)
    Ciphertext<DCRTPoly> EvalSub(const Ciphertext<DCRTPoly>& a, Plaintext& p) { return EvalNegate(EvalAdd(EvalNegate(a), p)); }
    Ciphertext<DCRTPoly> EvalSub(Plaintext& p, const Ciphertext<DCRTPoly>& a) { return EvalAdd(EvalNegate(a), p); }
    Ciphertext<DCRTPoly> EvalSub(const Ciphertext<DCRTPoly>& a, double v) { return EvalAdd(a, -v); }
    Ciphertext<DCRTPoly> EvalSub(double v, const Ciphertext<DCRTPoly>& a) { return EvalAdd(EvalNegate(a), v); }
    void EvalSubInPlace(Ciphertext<DCRTPoly>& a, const Ciphertext<DCRTPoly>& b) { a = EvalSub(a, b); }
    void EvalSubInPlace(Ciphertext<DCRTPoly>& a, double v) { a = EvalSub(a, v); }
    void EvalSubInPlace(double v, Ciphertext<DCRTPoly>& a) { a = EvalSub(v, a); }
    Ciphertext<DCRTPoly> EvalSubMutable(Ciphertext<DCRTPoly>& a, Ciphertext<DCRTPoly>& b) {
        auto x = match(a, b);
        a = x.first;
        b = x.second;
        return op2(fides_sub, a, b);
    }
    Ciphertext<DCRTPoly> EvalSubMutable(Ciphertext<DCRTPoly>& a, Plaintext& p) { return EvalSub(a, p); }
    Ciphertext<DCRTPoly> EvalSubMutable(Plaintext& p, Ciphertext<DCRTPoly>& a) { return EvalSub(p, a); }
    void EvalSubMutableInPlace(Ciphertext<DCRTPoly>& a, Ciphertext<DCRTPoly>& b) { a = EvalSubMutable(a, b); }
    Ciphertext<DCRTPoly> EvalMult(Plaintext& p, const Ciphertext<DCRTPoly>& a) { return EvalMult(a, p); }
    Ciphertext<DCRTPoly> EvalMult(double v, const Ciphertext<DCRTPoly>& a) { return EvalMult(a, v); }
    void EvalMultInPlace(Ciphertext<DCRTPoly>& a, const Ciphertext<DCRTPoly>& b) { a = EvalMult(a, b); }
    void EvalMultInPlace(Ciphertext<DCRTPoly>& a, Plaintext& p) { a = EvalMult(a, p); }
    void EvalMultInPlace(Ciphertext<DCRTPoly>& a, double v) { a = EvalMult(a, v); }
    void EvalMultInPlace(double v, Ciphertext<DCRTPoly>& a) { a = EvalMult(a, v); }
    Ciphertext<DCRTPoly> EvalMultMutable(Ciphertext<DCRTPoly>& a, Ciphertext<DCRTPoly>& b) {
        a = prepare(a);
        b = prepare(b);
        auto x = align(a, b);
        a = x.first;
        b = x.second;
        auto o = empty();
        check(fides_hmult(ctx, a->handle, b->handle, o->handle, 0), ctx);
        return o;
    }
    Ciphertext<DCRTPoly> EvalMultMutable(Ciphertext<DCRTPoly>& a, Plaintext& p) {
        a = prepare(a);
        return EvalMult(a, p);
    }
    Ciphertext<DCRTPoly> EvalMultMutable(Plaintext& p, Ciphertext<DCRTPoly>& a) { return EvalMultMutable(a, p); }
    void EvalMultMutableInPlace(Ciphertext<DCRTPoly>& a, Ciphertext<DCRTPoly>& b) { a = EvalMultMutable(a, b); }
    void EvalSquareInPlace(Ciphertext<DCRTPoly>& a) { a = EvalSquare(a); }
    Ciphertext<DCRTPoly> EvalSquareMutable(Ciphertext<DCRTPoly>& a) {
        a = prepare(a);
        return EvalSquare(a);
    }
    Ciphertext<DCRTPoly> Rescale(const Ciphertext<DCRTPoly>& a) {
        auto o = empty();
        check(fides_rescale(ctx, a->handle, o->handle), ctx);
        return o;
    }
    void RescaleInPlace(Ciphertext<DCRTPoly>& a) { a = Rescale(a); }
    Ciphertext<DCRTPoly> EvalRotate(const Ciphertext<DCRTPoly>& a, int32_t index) {
        auto o = empty();
        check(fides_rotate(ctx, a->handle, index, o->handle), ctx);
        return o;
    }
    void EvalRotateInPlace(Ciphertext<DCRTPoly>& a, int32_t index) { a = EvalRotate(a, index); }
    // The hoisted ModUp happens inside EvalFastRotation; the precomputation
    // handle is kept for signature compatibility (the reference returns
    // nullptr on GPU too, api/CryptoContext.cpp:1360-1373).
    // m is the cyclotomic order 2N (OpenFHE's argument); 0 is accepted too.
    std::shared_ptr<void> EvalFastRotationPrecompute(const Ciphertext<DCRTPoly>&) { return nullptr; }
    Ciphertext<DCRTPoly> EvalFastRotation(const Ciphertext<DCRTPoly>& a, int32_t index, uint32_t m,
                                          const std::shared_ptr<void>&) {
        check_order(m);
        return EvalRotate(a, index);
    }
    std::vector<Ciphertext<DCRTPoly>> EvalFastRotation(const Ciphertext<DCRTPoly>& a, const std::vector<int32_t>& idx,
                                                       uint32_t m, const std::shared_ptr<void>&) {
        check_order(m);
        std::vector<Ciphertext<DCRTPoly>> outs;
        std::vector<fides_ct*> hs;
        for (size_t i = 0; i < idx.size(); ++i) {
            outs.push_back(empty());
            hs.push_back(outs.back()->handle);
        }
        check(fides_rotate_hoisted(ctx, a->handle, (int)idx.size(), idx.data(), hs.data()), ctx);
        return outs;
    }
    // The precomputed-digit forms: the hoisted ModUp is shared inside one
    // EvalFastRotation call; addFirst (the P c0 term) is always part of it.
    Ciphertext<DCRTPoly> EvalFastRotationExt(const Ciphertext<DCRTPoly>& a, int32_t index, const std::shared_ptr<void>&,
                                             bool) {
        return EvalRotate(a, index);
    }
    std::vector<Ciphertext<DCRTPoly>> EvalFastRotationExt(const Ciphertext<DCRTPoly>& a,
                                                          const std::vector<int32_t>& idx,
                                                          const std::shared_ptr<void>& pre, bool) {
        return EvalFastRotation(a, idx, 0, pre);
    }
    // Sum of `n` slots spaced `stride` apart into every slot: log2(n)
    // rotate-and-add steps (AccumulateSum, api/CryptoContext.hpp:183-184);
    // needs rotation keys for stride * 2^k, k < log2(n).
    Ciphertext<DCRTPoly> AccumulateSum(const Ciphertext<DCRTPoly>& a, int n, int stride = 1) {
        Ciphertext<DCRTPoly> acc = a;
        for (int k = 1; k < n; k <<= 1) acc = EvalAdd(acc, EvalRotate(acc, k * stride));
        return acc;
    }
    void AccumulateSumInPlace(Ciphertext<DCRTPoly>& a, int n, int stride = 1) { a = AccumulateSum(a, n, stride); }
    Ciphertext<DCRTPoly> EvalConjugate(const Ciphertext<DCRTPoly>& a) {
        auto o = empty();
        check(fides_conjugate(ctx, a->handle, o->handle), ctx);
        return o;
    }
    // EvalChebyshevSeries (api/CryptoContext.hpp:171-173).  The coefficients
    // follow OpenFHE's convention, which the reference keeps: the series is
    // c_0 / 2 + sum_{k >= 1} c_k T_k(y) (the reference adds q.front() / 2,
    // src/CKKS/ApproxModEval.cu:216); the C ABI takes the plain sum.
    Ciphertext<DCRTPoly> EvalChebyshevSeries(const Ciphertext<DCRTPoly>& a, const std::vector<double>& coeffs,
                                             double lo, double hi) {
        if (coeffs.empty()) throw Exception(FIDES_BAD_ARG, "EvalChebyshevSeries: no coefficients");
        std::vector<double> c(coeffs);
        c[0] *= 0.5;
        auto o = empty();
        check(fides_chebyshev_series(ctx, prepare(a)->handle, c.data(), (int)c.size() - 1, lo, hi, o->handle), ctx);
        return o;
    }
    void EvalChebyshevSeriesInPlace(Ciphertext<DCRTPoly>& a, const std::vector<double>& coeffs, double lo, double hi) {
        a = EvalChebyshevSeries(a, coeffs, lo, hi);
    }
    // Coefficients c_0..c_degree of the Chebyshev interpolant of func on
    // [a, b] at the degree + 1 Chebyshev nodes (GetChebyshevCoefficients,
    // api/CryptoContext.hpp:173, src/PolyApprox.cu:11), in OpenFHE's
    // convention c_0 / 2 + sum_{k >= 1} c_k T_k(y), y = (2x - (a + b)) / (b - a),
    // which EvalChebyshevSeries takes.
    template <class F>
    static std::vector<double> GetChebyshevCoefficients(F&& func, double a, double b, size_t degree) {
        const size_t n = degree + 1;
        const double pi = 3.14159265358979323846;
        std::vector<double> f(n), c(n, 0.0);
        for (size_t j = 0; j < n; ++j) {
            const double y = std::cos(pi * (j + 0.5) / n);
            f[j] = func(0.5 * (b - a) * y + 0.5 * (a + b));
        }
        for (size_t k = 0; k < n; ++k) {
            double s = 0;
            for (size_t j = 0; j < n; ++j) s += f[j] * std::cos(pi * k * (j + 0.5) / n);
            c[k] = 2.0 * s / n;
        }
        return c;
    }
    // EvalBootstrapSetup / EvalBootstrapKeyGen / EvalBootstrap (api/CryptoContext.hpp:80-82,180-181).
    // dim1 (the baby-step sizes of OpenFHE's linear transforms) is accepted
    // and not needed: each CoeffsToSlots / SlotsToCoeffs group here picks its
    // baby step from its own diagonals.  correctionFactor scales the message
    // by 2^correctionFactor through EvalMod (fides_boot_params.correction).
    void EvalBootstrapSetup(const std::vector<uint32_t>& levelBudget = {3, 3}, std::vector<uint32_t> dim1 = {0, 0},
                            uint32_t numSlots = 0, uint32_t correctionFactor = 0) {
        (void)dim1;
        fides_boot_params bp{};
        bp.slots = (int)(numSlots ? numSlots : slots);
        bp.level_budget[0] = levelBudget.size() > 0 ? (int)levelBudget[0] : 3;
        bp.level_budget[1] = levelBudget.size() > 1 ? (int)levelBudget[1] : 3;
        bp.correction = (int)correctionFactor;
        check(fides_bootstrap_setup(ctx, &bp), ctx);
    }
    void EvalBootstrapKeyGen(const PrivateKey<DCRTPoly>& sk, uint32_t numSlots = 0) {
        const int s = (int)(numSlots ? numSlots : slots);
        check(fides_bootstrap_keygen(ctx, sk->handle, s, seed), ctx);
        seed += 2;
    }
    // numIterations 2: the first result's error is bootstrapped again, scaled
    // by 2^precision (0: 12), and subtracted; the input must still hold the
    // bootstrap's output level (fides_bootstrap_iter).
    Ciphertext<DCRTPoly> EvalBootstrap(const Ciphertext<DCRTPoly>& a, uint32_t numIterations = 1,
                                       uint32_t precision = 0, bool prescaled = false) {
        (void)prescaled;
        auto o = empty();
        check(fides_bootstrap_iter(ctx, prepare(a)->handle, (int)numIterations, (int)precision, o->handle), ctx);
        return o;
    }
    void EvalBootstrapInPlace(Ciphertext<DCRTPoly>& a, uint32_t numIterations = 1, uint32_t precision = 0,
                              bool prescaled = false) {
        a = EvalBootstrap(a, numIterations, precision, prescaled);
    }
    static void SetLevel(Ciphertext<DCRTPoly>& ct, size_t level) {
        int L = 0;
        fides_ctx_info(ct->ctx, nullptr, &L, nullptr, nullptr, nullptr, nullptr);
        check(fides_ct_set_level(ct->ctx, ct->handle, L - 1 - (int)level), ct->ctx);
    }
    void Synchronize() const { check(fides_ctx_synchronize(ctx), ctx); }

    fides_ctx* ctx = nullptr;

  private:
    void check_order(uint32_t m) const {
        int logN = 0;
        fides_ctx_info(ctx, &logN, nullptr, nullptr, nullptr, nullptr, nullptr);
        if (m != 0 && m != (2u << logN)) throw Exception(FIDES_BAD_ARG, "EvalFastRotation: m is not the cyclotomic order 2N");
    }
    ScalingTechnique tech;
    uint32_t hamming;
    uint32_t slots = 0;
    bool sparse = false;
    bool loadedCtx = false;
    uint64_t seed = 0x5EEDull;
    std::vector<std::pair<uint32_t, RawKeySwitchKey>> pending;

    void load_key(uint32_t galois, RawKeySwitchKey& k) {
        if (k.r_key.size() != 2 || k.r_key_moduli.size() != 2) throw Exception(FIDES_BAD_ARG, "raw key: two halves");
        const int dn = (int)k.r_key[0].size();
        const int nl = dn ? (int)k.r_key[0][0].size() : 0;
        std::vector<uint64_t*> limbs;
        std::vector<uint64_t> mods;
        for (int h = 0; h < 2; ++h)
            for (int d = 0; d < dn; ++d)
                for (int i = 0; i < nl; ++i) {
                    limbs.push_back(k.r_key[h][d][i].data());
                    mods.push_back(k.r_key_moduli[h][d][i]);
                }
        fides_raw_key rk{limbs.data(), mods.data(), dn, nl, (int)GetRingDimension()};
        check(fides_key_import_raw(ctx, galois, &rk), ctx);
    }

    int top_level() const {
        int L = 0;
        fides_ctx_info(ctx, nullptr, &L, nullptr, nullptr, nullptr, nullptr);
        return L - 1;
    }
    double scale_for(size_t deg) const {
        const double base = 1125899906842624.0;  // 2^50, the context's default scale
        double s = 1;
        for (size_t i = 0; i < deg; ++i) s *= base;
        return s;
    }
    std::vector<double> interleave(const Plaintext& pt) const {
        std::vector<double> iv(2 * pt->slots, 0.0);
        for (size_t i = 0; i < pt->values.size() && i < pt->slots; ++i) {
            iv[2 * i] = pt->values[i].real();
            iv[2 * i + 1] = pt->values[i].imag();
        }
        return iv;
    }
    Ciphertext<DCRTPoly> wrap(fides_ct* h) { return std::make_shared<CiphertextImpl>(ctx, h); }
    Ciphertext<DCRTPoly> empty() {
        fides_ct* h = nullptr;
        check(fides_ct_create(ctx, &h), ctx);
        return wrap(h);
    }
    Ciphertext<DCRTPoly> op2(fides_status (*f)(fides_ctx*, const fides_ct*, const fides_ct*, fides_ct*),
                             const Ciphertext<DCRTPoly>& a, const Ciphertext<DCRTPoly>& b) {
        auto o = empty();
        check(f(ctx, a->handle, b->handle, o->handle), ctx);
        return o;
    }
    // FLEXIBLEAUTO / FIXEDAUTO: rescale a degree-2 input before multiplying.
    Ciphertext<DCRTPoly> prepare(const Ciphertext<DCRTPoly>& a) {
        if (tech != FIXEDMANUAL && a->GetNoiseScaleDeg() >= 2) return Rescale(a);
        return a;
    }
    // Automatic modes before an addition: bring both operands to the same
    // noise degree (rescaling the degree-2 one) and the same level
    // (adjustForAddOrSub, Ciphertext.cpp:177-230).
    std::pair<Ciphertext<DCRTPoly>, Ciphertext<DCRTPoly>> match(Ciphertext<DCRTPoly> a, Ciphertext<DCRTPoly> b) {
        if (tech != FIXEDMANUAL) {
            if (a->GetNoiseScaleDeg() > b->GetNoiseScaleDeg()) a = Rescale(a);
            if (b->GetNoiseScaleDeg() > a->GetNoiseScaleDeg()) b = Rescale(b);
        }
        return align(a, b);
    }
    // Drop the higher-level operand to the lower level (automatic modes).
    std::pair<Ciphertext<DCRTPoly>, Ciphertext<DCRTPoly>> align(Ciphertext<DCRTPoly> a, Ciphertext<DCRTPoly> b) {
        if (a->GetLevel() == b->GetLevel()) return {a, b};
        auto& hi = a->GetLevel() > b->GetLevel() ? a : b;
        const int target = (int)std::min(a->GetLevel(), b->GetLevel());
        auto c = empty();
        check(fides_ct_copy(ctx, hi->handle, c->handle), ctx);
        check(fides_ct_set_level(ctx, c->handle, target), ctx);
        hi = c;
        return {a, b};
    }
};

template <typename T = DCRTPoly>
using CryptoContext = std::shared_ptr<CryptoContextImpl<DCRTPoly>>;

inline CryptoContext<DCRTPoly> GenCryptoContext(const CCParams<CryptoContextCKKSRNS>& p) {
    return std::make_shared<CryptoContextImpl<DCRTPoly>>(p);
}
// over the moduli and roots of an OpenFHE context (RawParams from GetRawParams)
inline CryptoContext<DCRTPoly> GenCryptoContext(const CCParams<CryptoContextCKKSRNS>& p, const RawParams& raw) {
    return std::make_shared<CryptoContextImpl<DCRTPoly>>(p, raw);
}

}  // namespace fideslib
