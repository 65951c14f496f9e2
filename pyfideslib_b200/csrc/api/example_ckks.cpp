// example_ckks.cpp -- the FIDESlib-style C++ surface end to end: context,
// keys, encrypt, EvalMult + Rescale, EvalRotate, EvalFastRotation, raw
// (RawCipherText) export and LoadCiphertext in both formats, EvalAddMany,
// the in-place forms, AccumulateSum, a Chebyshev series from
// GetChebyshevCoefficients, decrypt.  Prints the maximum slot error of each
// step and "OK" when all are small.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>

#include "fideslib.hpp"

using namespace fideslib;

int main(int argc, char** argv) {
    const uint32_t logn = argc > 1 ? (uint32_t)atoi(argv[1]) : 13;
    CCParams<CryptoContextCKKSRNS> p;
    p.SetMultiplicativeDepth(6);
    p.SetScalingModSize(50);
    p.SetFirstModSize(60);
    p.SetRingDim(1u << logn);
    p.SetNumLargeDigits(3);
    p.SetScalingTechnique(FLEXIBLEAUTO);
    auto cc = GenCryptoContext(p);
    auto keys = cc->KeyGen();
    cc->EvalMultKeyGen(keys.secretKey);
    cc->EvalRotateKeyGen(keys.secretKey, {1, -3, 2});
    const size_t n = cc->GetRingDimension() / 2;
    std::mt19937 rng(7);
    std::uniform_real_distribution<double> u(-1, 1);
    std::vector<std::complex<double>> x(n), y(n);
    for (size_t i = 0; i < n; ++i) {
        x[i] = {u(rng), u(rng)};
        y[i] = {u(rng), u(rng)};
    }
    Plaintext px = cc->MakeCKKSPackedPlaintext(x), py = cc->MakeCKKSPackedPlaintext(y);
    auto cx = cc->Encrypt(keys.publicKey, px);
    auto cy = cc->Encrypt(keys.publicKey, py);
    auto cm = cc->EvalMult(cx, cy);   // degree 2
    auto cs = cc->EvalAdd(cc->EvalMult(cm, cx), cy);  // auto-rescale of cm, level alignment of cy
    auto cr = cc->EvalRotate(cx, 1);
    auto fr = cc->EvalFastRotation(cx, std::vector<int32_t>{1, -3}, 0, nullptr);
    auto err = [&](Ciphertext<DCRTPoly>& c, auto f) {
        Plaintext out;
        cc->Decrypt(keys.secretKey, c, &out);
        auto v = out->GetCKKSPackedValue();
        double e = 0;
        for (size_t i = 0; i < n; ++i) e = std::max(e, std::abs(v[i] - f(i)));
        return e;
    };
    const double e1 = err(cm, [&](size_t i) { return x[i] * y[i]; });
    const double e2 = err(cs, [&](size_t i) { return x[i] * y[i] * x[i] + y[i]; });
    const double e3 = err(cr, [&](size_t i) { return x[(i + 1) % n]; });
    const double e4 = err(fr[1], [&](size_t i) { return x[(i + n - 3) % n]; });
    // raw residues out and back in (LoadCiphertext), in both formats
    RawCipherText raw = cc->GetRawCipherText(cx);
    auto cx2 = cc->CiphertextFromRaw(raw);
    cc->LoadCiphertext(cx2);
    auto cx3 = cc->CiphertextFromRaw(cc->GetRawCipherText(cx, COEFFICIENT));
    cc->LoadCiphertext(cx3);
    const double e5 = std::max(err(cx2, [&](size_t i) { return x[i]; }), err(cx3, [&](size_t i) { return x[i]; }));
    // many-operand and in-place forms, slot accumulation
    auto many = cc->EvalAddMany({cx, cy, cx2});
    auto acc = cc->AccumulateSum(cx, 4, 1);
    auto ip = cx;
    cc->EvalMultInPlace(ip, 2.0);
    cc->EvalAddInPlace(ip, cy);
    cc->EvalSubInPlace(ip, 0.25);
    const double e6 = std::max({err(many, [&](size_t i) { return 2.0 * x[i] + y[i]; }),
                                err(acc, [&](size_t i) { return x[i] + x[(i + 1) % n] + x[(i + 2) % n] + x[(i + 3) % n]; }),
                                err(ip, [&](size_t i) { return 2.0 * x[i] + y[i] - 0.25; })});
    // cos on [-1, 1] by its degree-15 Chebyshev interpolant (OpenFHE's convention)
    std::vector<double> r(n);
    for (size_t i = 0; i < n; ++i) r[i] = u(rng);
    Plaintext pr = cc->MakeCKKSPackedPlaintext(r);
    auto crr = cc->Encrypt(keys.publicKey, pr);
    auto coeffs = CryptoContextImpl<DCRTPoly>::GetChebyshevCoefficients([](double t) { return std::cos(t); }, -1.0,
                                                                         1.0, 15);
    auto ccos = cc->EvalChebyshevSeries(crr, coeffs, -1.0, 1.0);
    const double e7 = err(ccos, [&](size_t i) { return std::complex<double>(std::cos(r[i]), 0.0); });
    printf("mult %.2e  mult-add %.2e  rotate %.2e  fast-rotate %.2e  raw %.2e  many/acc/in-place %.2e  cheb %.2e\n",
           e1, e2, e3, e4, e5, e6, e7);
    const bool ok = e1 < 1e-6 && e2 < 1e-6 && e3 < 1e-6 && e4 < 1e-6 && e5 < 1e-6 && e6 < 1e-6 && e7 < 1e-6;
    printf("%s\n", ok ? "OK" : "FAIL");
    return ok ? 0 : 1;
}
