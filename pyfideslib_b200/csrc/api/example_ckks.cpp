// example_ckks.cpp -- the FIDESlib-style C++ surface end to end: context,
// keys, encrypt, EvalMult + Rescale, EvalRotate, EvalFastRotation, decrypt.
// Prints the maximum slot error of each step and "OK" when all are small.
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
    cc->EvalRotateKeyGen(keys.secretKey, {1, -3});
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
    printf("mult %.2e  mult-add %.2e  rotate %.2e  fast-rotate %.2e\n", e1, e2, e3, e4);
    const bool ok = e1 < 1e-6 && e2 < 1e-6 && e3 < 1e-6 && e4 < 1e-6;
    printf("%s\n", ok ? "OK" : "FAIL");
    return ok ? 0 : 1;
}
