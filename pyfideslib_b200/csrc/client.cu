// client.cu -- the client-side half of CKKS that FIDESlib delegates to OpenFHE
// (api/CryptoContext.cpp:475-626: KeyGen, EvalMultKeyGen, EvalRotateKeyGen,
// MakeCKKSPackedPlaintext, Encrypt, Decrypt).  It is provided so that the
// evaluation core can be exercised end to end without OpenFHE; the
// evaluation path does not depend on it.
//
//   * encoding: canonical embedding with slot j at the root zeta^(5^j)
//     (zeta = e^{i pi / N}); sparse packings repeat the slots with period n.
//     Evaluated with one complex FFT of size N over the odd powers of zeta.
//   * secrets: ternary, uniform or with a fixed Hamming weight (host, then
//     uploaded); errors (rounded Gaussian, sigma 3.2, Box-Muller), ephemeral
//     ternary polynomials and uniform polynomials drawn on the device from a
//     counter-based hash.
//   * switching keys (hybrid, digits of alpha moduli):
//       b_d = -a_d * s_b + e_d + [P]_{q_i} * s_g   on the moduli of digit d,
//       b_d = -a_d * s_b + e_d                    elsewhere,
//     with (s_b, s_g) = (s, s^2) for relinearisation and
//     (sigma_g^-1(s), s) for the automorphism sigma_g: X -> X^g, matching the
//     order in which the evaluation applies the permutation (after the inner
//     product, before ModDown).
//   * decryption: c0 + c1 s, INTT, a mixed-radix CRT of the first three
//     moduli (values of decryptable ciphertexts are far below q0 q1 q2 / 2)
//     and the forward embedding FFT, all on the device; only the slots come
//     back to the host.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <random>
#include <vector>

#include "context.hpp"

using namespace fides;

namespace {

struct Xoshiro {
    uint64_t s[4];
    explicit Xoshiro(uint64_t seed) {
        for (int i = 0; i < 4; ++i) {
            uint64_t z = (seed += 0x9E3779B97F4A7C15ull);
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            s[i] = z ^ (z >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
};

__global__ void k_small_to_rns(const int64_t* __restrict__ v, uint64_t* __restrict__ out, int N, int q0,
                               const PrimeConst* __restrict__ pcs) {
    const int limb = blockIdx.y;
    const PrimeConst pc = pcs[q0 + limb];
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t x = v[j];
    uint64_t a = x < 0 ? (uint64_t)(-x) : (uint64_t)x;
    a = csub(reduce64_lazy(a, pc), pc.p);
    out[(size_t)limb * N + j] = x < 0 ? neg_mod(a, pc.p) : a;
}

__global__ void k_fill_uniform(uint64_t* __restrict__ out, int N, int q0, const PrimeConst* __restrict__ pcs,
                               uint64_t stream) {
    const int limb = blockIdx.y;
    const uint64_t p = pcs[q0 + limb].p;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    out[(size_t)limb * N + j] = uniform_mod(stream, q0 + limb, (uint32_t)j, p);
}

// Small polynomials drawn on the device, coefficient form, on limbs
// 0..nlimbs-1: KIND 0 a rounded Gaussian (Box-Muller, one pair of
// coefficients per thread, standard deviation sigma), KIND 1 uniform ternary.
// Pair i draws the counters stream ^ 2i and stream ^ (2i + 1).
constexpr double kErrorSigma = 3.2;
template <int KIND>
__global__ void k_sample_small(uint64_t* __restrict__ out, int N, int nlimbs, const PrimeConst* __restrict__ pcs,
                               uint64_t stream) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (2 * i >= N) return;
    const uint64_t h0 = hash64(stream ^ (uint64_t)(2 * i)), h1 = hash64(stream ^ (uint64_t)(2 * i + 1));
    int64_t x0, x1;
    if (KIND == 0) {
        const double u1 = (double)((h0 >> 11) + 1) * 0x1p-53;  // (0, 1]
        const double u2 = (double)(h1 >> 11) * 0x1p-53;        // [0, 1)
        const double r = sqrt(-2.0 * log(u1)) * kErrorSigma;
        double sn, cs;
        sincospi(2.0 * u2, &sn, &cs);
        x0 = llrint(r * cs);
        x1 = llrint(r * sn);
    } else {
        x0 = (int64_t)__umul64hi(h0, 3) - 1;
        x1 = (int64_t)__umul64hi(h1, 3) - 1;
    }
    for (int limb = 0; limb < nlimbs; ++limb) {
        const uint64_t p = pcs[limb].p;
        ulonglong2 v;
        v.x = x0 < 0 ? p - (uint64_t)(-x0) : (uint64_t)x0;
        v.y = x1 < 0 ? p - (uint64_t)(-x1) : (uint64_t)x1;
        *(ulonglong2*)(out + (size_t)limb * N + 2 * i) = v;
    }
}

// b = -a * sb + e (+ pmod_i * sg on limbs with lo <= prime < hi)
__global__ void k_key_combine(uint64_t* __restrict__ b, const uint64_t* __restrict__ a,
                              const uint64_t* __restrict__ sb, const uint64_t* __restrict__ e,
                              const uint64_t* __restrict__ sg, const PrimeConst* __restrict__ pcs,
                              const uint64_t* __restrict__ pmod, int N, int lo, int hi) {
    const int limb = blockIdx.y;
    const PrimeConst pc = pcs[limb];
    const size_t i = (size_t)limb * N + blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t v = sub_mod(e[i], mul_mod(a[i], sb[i], pc), pc.p);
    if (limb >= lo && limb < hi) v = add_mod(v, mul_shoup(sg[i], pmod[2 * limb], pmod[2 * limb + 1], pc.p), pc.p);
    b[i] = v;
}

fides_status upload_small(fides_ctx* c, const std::vector<int64_t>& v, uint64_t* out, int q0, int nlimbs) {
    int64_t* dv = nullptr;
    if (cudaMallocAsync((void**)&dv, sizeof(int64_t) * c->N, c->st) != cudaSuccess) return set_err(c, FIDES_OOM, "small");
    cudaMemcpyAsync(dv, v.data(), sizeof(int64_t) * c->N, cudaMemcpyHostToDevice, c->st);
    count_launches(1);
    k_small_to_rns<<<dim3(c->N / 256, nlimbs), 256, 0, c->st>>>(dv, out, c->N, q0, c->dev.pc);
    cudaStreamSynchronize(c->st);
    cudaFreeAsync(dv, c->st);
    return check_cuda(c, "small_to_rns");
}

// A small polynomial on limbs 0..nlimbs-1 (coefficient form), drawn on the
// device from the stream word: kind 0 error (Gaussian), 1 ternary.
void sample_small(fides_ctx* c, int kind, uint64_t stream, uint64_t* out, int nlimbs) {
    count_launches(1);
    const int grid = (c->N / 2 + 255) / 256;
    if (kind == 0)
        k_sample_small<0><<<grid, 256, 0, c->st>>>(out, c->N, nlimbs, c->dev.pc, stream);
    else
        k_sample_small<1><<<grid, 256, 0, c->st>>>(out, c->N, nlimbs, c->dev.pc, stream);
}

// stream words of the error and ternary draws (tags above any key digit's)
constexpr uint32_t kTagError = 0xE0, kTagTernary = 0xE1;

// A switching key b = -a sb + e + P sg (per digit), a uniform from the seed.
// compress: only b is stored; the a half is regenerated from the seed by the
// key-switch kernels (key.a null, key.a_seed set).
fides_status gen_switch_key(fides_ctx* c, const uint64_t* sb, const uint64_t* sg, uint64_t seed, SwitchKey& key,
                            bool compress) {
    const int N = c->N, NP = c->L + c->K;
    fides_status st = key_alloc(c, key, compress);
    if (st != FIDES_OK) return st;
    key.a_seed = seed * 1315423911ull;
    uint64_t* e = nullptr;
    uint64_t* atmp = nullptr;
    if (cudaMallocAsync((void**)&e, (size_t)NP * N * 8, c->st) != cudaSuccess) return set_err(c, FIDES_OOM, "key tmp");
    if (compress && cudaMallocAsync((void**)&atmp, (size_t)NP * N * 8, c->st) != cudaSuccess) {
        cudaFreeAsync(e, c->st);
        return set_err(c, FIDES_OOM, "key tmp");
    }
    for (int d = 0; d < c->dnum; ++d) {
        uint64_t* kb = key.b + (size_t)d * NP * N;
        uint64_t* ka = compress ? atmp : key.a + (size_t)d * NP * N;
        count_launches(1);
        k_fill_uniform<<<dim3(N / 256, NP), 256, 0, c->st>>>(ka, N, 0, c->dev.pc, uniform_stream(key.a_seed, d + 1));
        sample_small(c, 0, uniform_stream(seed ^ (0xABCDull + d), kTagError), e, NP);
        ntt_forward(c->dev, map_single(e, e, NP, NP, 0), FL_PLAIN, FS_PLAIN, c->st);
        const int lo = d * c->alpha, hi = std::min(c->L, lo + c->alpha);
        count_launches(1);
        k_key_combine<<<dim3(N / 256, NP), 256, 0, c->st>>>(kb, ka, sb, e, sg, c->dev.pc, c->dev.md_pmod, N, lo, hi);
    }
    cudaStreamSynchronize(c->st);
    cudaFreeAsync(e, c->st);
    if (atmp) cudaFreeAsync(atmp, c->st);
    return check_cuda(c, "switch key");
}

}  // namespace

// ---- encoding on the device ----
// The canonical embedding's inverse: slot j of the N/2 (slot k = j mod slots repeated) goes to the root
// zeta^(5^j) and its conjugate to zeta^(-5^j); an inverse complex FFT of
// length N, the twist by exp(-i pi t / N) / N and the real part give the
// coefficients, scaled and rounded to integers.  FP64 throughout.

// M[bitrev(pos_j)] = z_(j mod slots), M[bitrev(neg_j)] = conj(z): the FFT's
// input permutation folded into the scatter
// 5^j mod 2N by squaring (products in 64 bits: 2N - 1 can exceed 2^16)
__device__ __forceinline__ uint32_t pow5_mod_2n(uint32_t j, int logN) {
    const uint32_t mask = (2u << logN) - 1;
    uint32_t g = 1, b = 5;
    for (uint32_t e = j; e; e >>= 1) {
        if (e & 1) g = (uint32_t)(((uint64_t)g * b) & mask);
        b = (uint32_t)(((uint64_t)b * b) & mask);
    }
    return g;
}

// (slot j of the N/2 takes factor * z[(j - shift) mod slots])
__global__ void k_embed_scatter(const double2* __restrict__ z, int slots, int shift, double factor, int logN,
                                double2* __restrict__ M) {
    const int N = 1 << logN;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= N / 2) return;
    const uint32_t g = pow5_mod_2n((uint32_t)j, logN);
    double2 v = z[(j - shift) & (slots - 1)];
    v.x *= factor;
    v.y *= factor;
    const uint32_t pos = (g - 1) / 2, neg = (2u * (uint32_t)N - g - 1) / 2;
    M[__brev(pos) >> (32 - logN)] = v;
    M[__brev(neg) >> (32 - logN)] = make_double2(v.x, -v.y);
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(__fma_rn(a.x, b.x, -a.y * b.y), __fma_rn(a.x, b.y, a.y * b.x));
}

// radix-2 FFT butterflies on bit-reversed input, blocks of length 2^s
// (a[i] +- w a[i + h], w = exp(dir 2 pi i k / 2^s); dir = -1 for encoding,
// +1 for decoding): stages 1..log2(tile) in shared memory, one CTA per tile
// of 2 blockDim.x <= 2048 elements, then one launch per further stage
constexpr int kFftTile = 2048;
__global__ void __launch_bounds__(1024) k_fft_tile(double2* __restrict__ M, int s_hi, double dir) {
    __shared__ double2 t[kFftTile];
    const int T = 2 * blockDim.x;
    double2* base = M + (size_t)blockIdx.x * T;
    for (int i = threadIdx.x; i < T; i += blockDim.x) t[i] = base[i];
    __syncthreads();
    for (int s = 1; s <= s_hi; ++s) {
        const int h = 1 << (s - 1);
        const int i = threadIdx.x;  // one butterfly per thread and stage
        const int k = i & (h - 1), a = ((i >> (s - 1)) << s) + k;
        double sn, cs;
        sincospi(dir * (double)k / (double)h, &sn, &cs);
        const double2 u = t[a], v = cmul(t[a + h], make_double2(cs, sn));
        t[a] = make_double2(u.x + v.x, u.y + v.y);
        t[a + h] = make_double2(u.x - v.x, u.y - v.y);
        __syncthreads();
    }
    for (int i = threadIdx.x; i < T; i += blockDim.x) base[i] = t[i];
}

__global__ void k_fft_stage(double2* __restrict__ M, int s, int N, double dir) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N / 2) return;
    const int h = 1 << (s - 1);
    const int k = i & (h - 1), a = ((i >> (s - 1)) << s) + k;
    double sn, cs;
    sincospi(dir * (double)k / (double)h, &sn, &cs);
    const double2 u = M[a], v = cmul(M[a + h], make_double2(cs, sn));
    M[a] = make_double2(u.x + v.x, u.y + v.y);
    M[a + h] = make_double2(u.x - v.x, u.y - v.y);
}

// v_t = round(Re(M_t exp(-i pi t / N)) / N * scale); a magnitude at or above
// 9e18 sets *bad and writes 0
__global__ void k_embed_round(const double2* __restrict__ M, int N, double scale, int64_t* __restrict__ v,
                              int* __restrict__ bad) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N) return;
    double sn, cs;
    sincospi(-(double)t / (double)N, &sn, &cs);
    const double2 m = M[t];
    const double x = (m.x * cs - m.y * sn) / (double)N * scale;
    if (!(fabs(x) < 9.0e18)) {
        *bad = 1;
        v[t] = 0;
        return;
    }
    v[t] = llround(x);
}

// the FFT of length N on M (bit-reversed input, natural-order output)
static void fft_dev(fides_ctx* c, double2* M, double dir) {
    const int N = c->N, logN = c->logN;
    const int s_tile = std::min(logN, 11);  // tiles of 2^s_tile <= kFftTile elements
    count_launches(1 + logN - s_tile);
    k_fft_tile<<<N >> s_tile, (1 << s_tile) / 2, 0, c->st>>>(M, s_tile, dir);
    for (int s = s_tile + 1; s <= logN; ++s) k_fft_stage<<<(N / 2 + 255) / 256, 256, 0, c->st>>>(M, s, N, dir);
}

fides_status fides::encode_dev_z(fides_ctx* c, const double2* z, int slots, int shift, double factor, int level,
                                 double scale, uint64_t* dm, int* bad) {
    const int N = c->N, logN = c->logN;
    if (slots < 1 || slots > N / 2 || (slots & (slots - 1))) return set_err(c, FIDES_BAD_ARG, "encode: slots");
    // scratch: N complex (FFT), N int64
    char* buf = nullptr;
    const size_t b_m = (size_t)N * 16, b_v = (size_t)N * 8;
    if (cudaMallocAsync((void**)&buf, b_m + b_v, c->st) != cudaSuccess) {
        cudaGetLastError();
        return set_err(c, FIDES_OOM, "encode scratch");
    }
    double2* M = (double2*)buf;
    int64_t* v = (int64_t*)(buf + b_m);
    count_launches(3);
    k_embed_scatter<<<(N / 2 + 255) / 256, 256, 0, c->st>>>(z, slots, shift & (slots - 1), factor, logN, M);
    fft_dev(c, M, -1.0);
    k_embed_round<<<(N + 255) / 256, 256, 0, c->st>>>(M, N, scale, v, bad);
    k_small_to_rns<<<dim3(N / 256, level + 1), 256, 0, c->st>>>(v, dm, N, 0, c->dev.pc);
    cudaFreeAsync(buf, c->st);
    ntt_forward(c->dev, map_single(dm, dm, level + 1, level + 1, 0), FL_PLAIN, FS_PLAIN, c->st);
    return FIDES_OK;
}

fides_status fides::encode_dev(fides_ctx* c, const double* values, int slots, int level, double scale, uint64_t* dm) {
    if (slots < 1 || slots > c->N / 2 || (slots & (slots - 1))) return set_err(c, FIDES_BAD_ARG, "encode: slots");
    // slots complex (input) and one flag
    char* buf = nullptr;
    const size_t b_z = (size_t)slots * 16;
    if (cudaMallocAsync((void**)&buf, b_z + 16, c->st) != cudaSuccess) {
        cudaGetLastError();
        return set_err(c, FIDES_OOM, "encode scratch");
    }
    double2* z = (double2*)buf;
    int* bad = (int*)(buf + b_z);
    cudaMemcpyAsync(z, values, b_z, cudaMemcpyHostToDevice, c->st);
    cudaMemsetAsync(bad, 0, sizeof(int), c->st);
    fides_status s = encode_dev_z(c, z, slots, 0, 1.0, level, scale, dm, bad);
    int hbad = 0;
    if (s == FIDES_OK) cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, c->st);
    cudaFreeAsync(buf, c->st);
    cudaStreamSynchronize(c->st);
    if (s != FIDES_OK) return s;
    if (hbad) return set_err(c, FIDES_BAD_ARG, "encoded coefficient exceeds 2^63");
    return check_cuda(c, "encode");
}

// ---- decoding on the device ----
// The canonical embedding itself: the centred integer coefficients (a
// mixed-radix CRT of the first `use` <= 3 moduli, converted to FP64 and
// divided by the scale), twisted by exp(i pi t / N), then a forward complex
// FFT of length N; slot j reads the transform at the index t of the root
// zeta^(5^j), t = (5^j - 1) / 2.
struct CrtConst {
    uint64_t q[3];
    uint64_t inv01, inv02, inv12;  // q0^-1 mod q1, q0^-1 mod q2, q1^-1 mod q2
    int use;
};

// M[bitrev(t)] = x_t exp(i pi t / N), x_t the centred value of coefficient t
// over q0..q_{use-1} divided by scale; the FFT's input permutation folded in
__global__ void k_decode_crt(const uint64_t* __restrict__ m, int logN, CrtConst k, const PrimeConst* __restrict__ pcs,
                             double scale, double2* __restrict__ M) {
    const int N = 1 << logN;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N) return;
    uint64_t v[3] = {m[t], 0, 0};
    if (k.use > 1) v[1] = mul_mod(sub_mod(m[N + t], v[0] % k.q[1], k.q[1]), k.inv01, pcs[1]);
    if (k.use > 2) {
        const uint64_t u = mul_mod(sub_mod(m[2 * N + t], v[0] % k.q[2], k.q[2]), k.inv02, pcs[2]);
        v[2] = mul_mod(sub_mod(u, v[1] % k.q[2], k.q[2]), k.inv12, pcs[2]);
    }
    // the value is v0 + q0 (v1 + q1 v2); above half the product it stands
    // for a negative one, -(1 + sum (q_i - 1 - v_i) prod_{j<i} q_j)
    const bool neg = v[k.use - 1] > k.q[k.use - 1] / 2;
    double x = 0;
    for (int i = k.use - 1; i >= 0; --i) {
        const uint64_t d = neg ? k.q[i] - 1 - v[i] : v[i];
        x = i == k.use - 1 ? (double)d : __fma_rn(x, (double)k.q[i], (double)d);
    }
    x = (neg ? -(x + 1.0) : x) / scale;
    double sn, cs;
    sincospi((double)t / (double)N, &sn, &cs);
    M[__brev((uint32_t)t) >> (32 - logN)] = make_double2(x * cs, x * sn);
}

__global__ void k_decode_gather(const double2* __restrict__ M, int slots, int logN, double2* __restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= slots) return;
    out[j] = M[(pow5_mod_2n((uint32_t)j, logN) - 1) / 2];
}

extern "C" {

fides_status fides_keygen(fides_ctx* c, uint64_t seed, int hamming_weight, fides_sk** out) {
    if (!c || !out || hamming_weight < 0 || hamming_weight > c->N) return FIDES_BAD_ARG;
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    cudaSetDevice(c->device);
    fides_sk* sk = new (std::nothrow) fides_sk();
    if (!sk) return FIDES_OOM;
    const int N = c->N, NP = c->L + c->K;
    sk->coeff.assign(N, 0);
    Xoshiro r(seed);
    if (hamming_weight == 0) {
        for (int i = 0; i < N; ++i) sk->coeff[i] = (int8_t)((int)(r.next() % 3) - 1);
    } else {
        int placed = 0;
        while (placed < hamming_weight) {
            const int i = (int)(r.next() % N);
            if (sk->coeff[i]) continue;
            sk->coeff[i] = (r.next() & 1) ? 1 : -1;
            ++placed;
        }
    }
    if (cudaMalloc((void**)&sk->s, (size_t)NP * N * 8) != cudaSuccess) {
        cudaGetLastError();
        delete sk;
        return set_err(c, FIDES_OOM, "secret key");
    }
    std::vector<int64_t> v(sk->coeff.begin(), sk->coeff.end());
    fides_status s = upload_small(c, v, sk->s, 0, NP);
    if (s != FIDES_OK) return s;
    ntt_forward(c->dev, map_single(sk->s, sk->s, NP, NP, 0), FL_PLAIN, FS_PLAIN, c->st);
    cudaStreamSynchronize(c->st);
    *out = sk;
    return check_cuda(c, "keygen");
}

fides_status fides_sk_free(fides_ctx* c, fides_sk* sk) {
    if (!c || !sk) return FIDES_BAD_ARG;
    cudaSetDevice(c->device);
    if (sk->s) cudaFree(sk->s);
    delete sk;
    return FIDES_OK;
}

fides_status fides_keygen_relin(fides_ctx* c, const fides_sk* sk, uint64_t seed) {
    if (!c || !sk || !sk->s) return FIDES_BAD_ARG;
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    cudaSetDevice(c->device);
    const int NP = c->L + c->K;
    uint64_t* s2 = nullptr;
    if (cudaMallocAsync((void**)&s2, (size_t)NP * c->N * 8, c->st) != cudaSuccess) return set_err(c, FIDES_OOM, "s^2");
    launch_elementwise(c->dev, EW_MUL, NP, 0, sk->s, sk->s, s2, c->st);
    // bit 1 of the compression mask: batched HMults read an explicit a half
    // once per batch and serve it from L2, where a seeded one is regenerated
    // for every element (and the fused row-pass key switch needs it stored)
    fides_status s = gen_switch_key(c, sk->s, s2, seed, c->relin, (c->compress_keys & 2) != 0);
    cudaFreeAsync(s2, c->st);
    if (s == FIDES_OK) c->has_relin = true;
    return s;
}

// inverse of an odd g modulo 2N (extended Euclid; 2N is not prime)
static uint32_t inv_mod_2n(uint32_t g, uint32_t m) {
    int64_t t = 0, nt = 1, r = m, nr = g % m;
    while (nr) {
        const int64_t q = r / nr;
        const int64_t t2 = t - q * nt, r2 = r - q * nr;
        t = nt;
        nt = t2;
        r = nr;
        nr = r2;
    }
    return (uint32_t)(t < 0 ? t + m : t);
}

// The Galois key of g in the permuted layout of the key-switch kernel: entry j
// pairs with rotation output j, k'[j] = k[slot(g, j)] for the key k that
// switches sigma_g^-1(s) to s.  Written out, k' = (-a' s + e' + P sigma_g(s), a')
// with sigma_g(s)[j] = s[slot(g, j)]: a switching key from sigma_g(s) to s in
// the plain layout, a' uniform and e' fresh noise (both distributions are
// invariant under the permutation).
static fides_status keygen_galois(fides_ctx* c, const fides_sk* sk, uint32_t g, uint64_t seed) {
    const int NP = c->L + c->K, N = c->N;
    uint64_t* sr = nullptr;
    if (cudaMallocAsync((void**)&sr, (size_t)NP * N * 8, c->st) != cudaSuccess) return set_err(c, FIDES_OOM, "s rot");
    launch_automorph(c->dev, NP, sk->s, sr, g, c->st);
    fides_status s = gen_switch_key(c, sk->s, sr, seed ^ ((uint64_t)g << 20), c->galois_keys[g],
                                    (c->compress_keys & 1) != 0);
    cudaFreeAsync(sr, c->st);
    return s;
}

fides_status fides_keygen_rotations(fides_ctx* c, const fides_sk* sk, int n, const int32_t* indices, int slots,
                                    uint64_t seed) {
    if (!c || !sk || !sk->s || n < 0 || (n && !indices)) return FIDES_BAD_ARG;
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    cudaSetDevice(c->device);
    if (slots <= 0) slots = c->N / 2;
    // a key already held for an element is regenerated: it may belong to
    // another secret key; repeats within this call are generated once
    std::vector<uint32_t> done;
    for (int i = 0; i < n; ++i) {
        const uint32_t g = fides_rotation_galois(c, indices[i], slots);
        if (g == 1 || std::find(done.begin(), done.end(), g) != done.end()) continue;
        done.push_back(g);
        fides_status s = keygen_galois(c, sk, g, seed + 7919ull * (uint64_t)i);
        if (s != FIDES_OK) return s;
    }
    return FIDES_OK;
}

fides_status fides_set_key_compression(fides_ctx* c, int mask) {
    if (!c || mask < 0 || mask > 3) return FIDES_BAD_ARG;
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    c->compress_keys = mask;
    return FIDES_OK;
}

fides_status fides_keygen_conjugate(fides_ctx* c, const fides_sk* sk, uint64_t seed) {
    if (!c || !sk || !sk->s) return FIDES_BAD_ARG;
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    cudaSetDevice(c->device);
    return keygen_galois(c, sk, 2u * (uint32_t)c->N - 1, seed);
}

fides_status fides_key_export(fides_ctx* c, uint32_t galois, uint64_t* b, uint64_t* a) {
    if (!c || !b || !a) return FIDES_BAD_ARG;
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    cudaSetDevice(c->device);
    const SwitchKey* k = nullptr;
    if (galois == 0) {
        if (!c->has_relin) return FIDES_KEY_MISSING;
        k = &c->relin;
    } else {
        auto it = c->galois_keys.find(galois);
        if (it == c->galois_keys.end()) return FIDES_KEY_MISSING;
        k = &it->second;
    }
    const int NP = c->L + c->K, N = c->N;
    const int nlimbs = c->dnum * NP;
    const size_t words = (size_t)nlimbs * N;
    // a Galois key leaves in the plain layout: entry slot(g, j) = held entry j,
    // i.e. plain[i] = held[slot(g^-1, i)]
    const uint32_t ginv = galois ? inv_mod_2n(galois, 2u * (uint32_t)N) : 0;
    uint64_t* t = nullptr;
    if ((galois || !k->a) && cudaMallocAsync((void**)&t, 2 * words * 8, c->st) != cudaSuccess) {
        cudaGetLastError();
        return set_err(c, FIDES_OOM, "key export");
    }
    const uint64_t* ka = k->a;
    if (!ka) {
        // a seeded key: its a half regenerated digit by digit
        uint64_t* ta = t + words;
        for (int d = 0; d < c->dnum; ++d) {
            count_launches(1);
            k_fill_uniform<<<dim3(N / 256, NP), 256, 0, c->st>>>(ta + (size_t)d * NP * N, N, 0, c->dev.pc,
                                                                 uniform_stream(k->a_seed, d + 1));
        }
        ka = ta;
    }
    if (galois) {
        launch_automorph(c->dev, nlimbs, k->b, t, ginv, c->st);
        cudaMemcpyAsync(b, t, words * 8, cudaMemcpyDeviceToHost, c->st);
        // stream order: the gather below overwrites t's first half only after
        // the copy of b has read it (a regenerated a sits in the second half)
        launch_automorph(c->dev, nlimbs, ka, t, ginv, c->st);
        cudaMemcpyAsync(a, t, words * 8, cudaMemcpyDeviceToHost, c->st);
    } else {
        cudaMemcpyAsync(b, k->b, words * 8, cudaMemcpyDeviceToHost, c->st);
        cudaMemcpyAsync(a, ka, words * 8, cudaMemcpyDeviceToHost, c->st);
    }
    if (t) cudaFreeAsync(t, c->st);
    cudaStreamSynchronize(c->st);
    return check_cuda(c, "key export");
}


fides_status fides_encode(fides_ctx* c, const double* values, int slots, int level, double scale, uint64_t* m) {
    if (!c || !values || !m || slots < 1 || slots > c->N / 2 || (slots & (slots - 1)) || level < 0 || level >= c->L)
        return FIDES_BAD_ARG;
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    cudaSetDevice(c->device);
    uint64_t* dm = nullptr;
    if (cudaMallocAsync((void**)&dm, (size_t)(level + 1) * c->N * 8, c->st) != cudaSuccess)
        return set_err(c, FIDES_OOM, "encode");
    fides_status s = encode_dev(c, values, slots, level, scale > 0 ? scale : c->default_scale, dm);
    if (s == FIDES_OK) {
        cudaMemcpyAsync(m, dm, (size_t)(level + 1) * c->N * 8, cudaMemcpyDeviceToHost, c->st);
        cudaStreamSynchronize(c->st);
    }
    cudaFreeAsync(dm, c->st);
    return s == FIDES_OK ? check_cuda(c, "encode") : s;
}

fides_status fides_encrypt(fides_ctx* c, const fides_sk* sk, const double* values, int slots, int level,
                           double scale, uint64_t seed, fides_ct** out) {
    if (!c || !sk || !sk->s || !values || !out || slots < 1 || slots > c->N / 2 || (slots & (slots - 1)) ||
        level < 0 || level >= c->L)
        return FIDES_BAD_ARG;
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    cudaSetDevice(c->device);
    if (scale <= 0) scale = c->default_scale;
    const int n = level + 1, N = c->N;
    fides_ct* ct = new (std::nothrow) fides_ct();
    if (!ct) return FIDES_OOM;
    fides_status s = ct_reserve(c, ct, level);
    if (s != FIDES_OK) {
        delete ct;
        return s;
    }
    uint64_t *m = nullptr, *e = nullptr;
    cudaMallocAsync((void**)&m, (size_t)n * N * 8, c->st);
    cudaMallocAsync((void**)&e, (size_t)n * N * 8, c->st);
    s = encode_dev(c, values, slots, level, scale, m);
    if (s == FIDES_OK) {
        sample_small(c, 0, uniform_stream(seed ^ 0x5EED, kTagError), e, n);
        ntt_forward(c->dev, map_single(e, e, n, n, 0), FL_PLAIN, FS_PLAIN, c->st);
        count_launches(1);
        k_fill_uniform<<<dim3(N / 256, n), 256, 0, c->st>>>(ct->c1(N), N, 0, c->dev.pc, uniform_stream(seed * 2654435761ull + 17, 0));
        launch_elementwise(c->dev, EW_ADD, n, 0, e, m, e, c->st);  // e + m
        // c0 = -a s + (e + m): key_combine with no gadget term
        count_launches(1);
        k_key_combine<<<dim3(N / 256, n), 256, 0, c->st>>>(ct->c0(), ct->c1(N), sk->s, e, sk->s, c->dev.pc,
                                                           c->dev.md_pmod, N, 0, 0);
        cudaStreamSynchronize(c->st);
    }
    cudaFreeAsync(m, c->st);
    cudaFreeAsync(e, c->st);
    if (s != FIDES_OK) {
        fides_ct_free(c, ct);
        return s;
    }
    ct->level = level;
    ct->scale = scale;
    ct->noise_deg = 1;
    ct->slots = slots;
    *out = ct;
    return check_cuda(c, "encrypt");
}

fides_status fides_keygen_public(fides_ctx* c, const fides_sk* sk, uint64_t seed, fides_pk** out) {
    if (!c || !sk || !sk->s || !out) return FIDES_BAD_ARG;
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    cudaSetDevice(c->device);
    const int N = c->N, L = c->L;
    fides_pk* pk = new (std::nothrow) fides_pk();
    if (!pk) return FIDES_OOM;
    if (cudaMalloc((void**)&pk->b, 2 * (size_t)L * N * 8) != cudaSuccess) {
        cudaGetLastError();
        delete pk;
        return set_err(c, FIDES_OOM, "public key");
    }
    pk->a = pk->b + (size_t)L * N;
    uint64_t* e = nullptr;
    if (cudaMallocAsync((void**)&e, (size_t)L * N * 8, c->st) != cudaSuccess) return set_err(c, FIDES_OOM, "pk tmp");
    count_launches(1);
    k_fill_uniform<<<dim3(N / 256, L), 256, 0, c->st>>>(pk->a, N, 0, c->dev.pc, uniform_stream(seed * 0x9E3779B97F4A7C15ull + 99, 0));
    sample_small(c, 0, uniform_stream(seed ^ 0x7EA5, kTagError), e, L);
    ntt_forward(c->dev, map_single(e, e, L, L, 0), FL_PLAIN, FS_PLAIN, c->st);
    count_launches(1);
    k_key_combine<<<dim3(N / 256, L), 256, 0, c->st>>>(pk->b, pk->a, sk->s, e, sk->s, c->dev.pc, c->dev.md_pmod, N, 0,
                                                       0);
    cudaFreeAsync(e, c->st);
    cudaStreamSynchronize(c->st);
    fides_status s = check_cuda(c, "public key");
    if (s != FIDES_OK) {
        cudaFree(pk->b);
        delete pk;
        return s;
    }
    *out = pk;
    return FIDES_OK;
}

fides_status fides_pk_free(fides_ctx* c, fides_pk* pk) {
    if (!c || !pk) return FIDES_BAD_ARG;
    cudaSetDevice(c->device);
    if (pk->b) cudaFree(pk->b);
    delete pk;
    return FIDES_OK;
}

fides_status fides_encrypt_pk(fides_ctx* c, const fides_pk* pk, const double* values, int slots, int level,
                              double scale, uint64_t seed, fides_ct** out) {
    if (!c || !pk || !pk->b || !values || !out || slots < 1 || slots > c->N / 2 || (slots & (slots - 1)) ||
        level < 0 || level >= c->L)
        return FIDES_BAD_ARG;
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    cudaSetDevice(c->device);
    if (scale <= 0) scale = c->default_scale;
    const int n = level + 1, N = c->N, L = c->L;
    fides_ct* ct = new (std::nothrow) fides_ct();
    if (!ct) return FIDES_OOM;
    fides_status s = ct_reserve(c, ct, level);
    if (s != FIDES_OK) {
        delete ct;
        return s;
    }
    uint64_t* tmp = nullptr;  // m, v, e0, e1
    if (cudaMallocAsync((void**)&tmp, 4 * (size_t)n * N * 8, c->st) != cudaSuccess) {
        fides_ct_free(c, ct);
        return set_err(c, FIDES_OOM, "encrypt tmp");
    }
    uint64_t *m = tmp, *v = tmp + (size_t)n * N, *e0 = tmp + 2 * (size_t)n * N, *e1 = tmp + 3 * (size_t)n * N;
    s = encode_dev(c, values, slots, level, scale, m);
    if (s == FIDES_OK) {
        sample_small(c, 1, uniform_stream(seed ^ 0xC0FFEE, kTagTernary), v, n);
        sample_small(c, 0, uniform_stream(seed ^ 0xE0, kTagError), e0, n);
        sample_small(c, 0, uniform_stream(seed ^ 0xE1, kTagError), e1, n);
        LimbMap mm{};
        mm.nseg = 3;
        uint64_t* bufs[3] = {v, e0, e1};
        for (int i = 0; i < 3; ++i) {
            LimbSeg& g = mm.seg[i];
            g.in = g.out = bufs[i];
            g.count = n;
            g.skip_lo = n;
            g.nq = n;
            mm.total += n;
        }
        ntt_forward(c->dev, mm, FL_PLAIN, FS_PLAIN, c->st);
        launch_elementwise(c->dev, EW_ADD, n, 0, e0, m, e0, c->st);
        // c0 = v b + (e0 + m), c1 = v a + e1  (pk limbs 0..level)
        launch_elementwise(c->dev, EW_MUL, n, 0, pk->b, v, ct->c0(), c->st);
        launch_elementwise(c->dev, EW_ADD, n, 0, ct->c0(), e0, ct->c0(), c->st);
        launch_elementwise(c->dev, EW_MUL, n, 0, pk->a, v, ct->c1(N), c->st);
        launch_elementwise(c->dev, EW_ADD, n, 0, ct->c1(N), e1, ct->c1(N), c->st);
        cudaStreamSynchronize(c->st);
    }
    (void)L;
    cudaFreeAsync(tmp, c->st);
    if (s != FIDES_OK) {
        fides_ct_free(c, ct);
        return s;
    }
    ct->level = level;
    ct->scale = scale;
    ct->noise_deg = 1;
    ct->slots = slots;
    *out = ct;
    return check_cuda(c, "encrypt_pk");
}

fides_status fides_ct_random(fides_ctx* c, int level, uint64_t seed, fides_ct** out) {
    if (!c || !out || level < 0 || level >= c->L) return FIDES_BAD_ARG;
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    cudaSetDevice(c->device);
    fides_ct* ct = new (std::nothrow) fides_ct();
    if (!ct) return FIDES_OOM;
    fides_status s = ct_reserve(c, ct, level);
    if (s != FIDES_OK) {
        delete ct;
        return s;
    }
    const int N = c->N, n = level + 1;
    count_launches(2);
    k_fill_uniform<<<dim3(N / 256, n), 256, 0, c->st>>>(ct->c0(), N, 0, c->dev.pc, uniform_stream(seed * 0x9E3779B97F4A7C15ull + 1, 0));
    k_fill_uniform<<<dim3(N / 256, n), 256, 0, c->st>>>(ct->c1(N), N, 0, c->dev.pc, uniform_stream(seed * 0x9E3779B97F4A7C15ull + 2, 0));
    ct->level = level;
    ct->scale = c->default_scale;
    ct->noise_deg = 1;
    ct->slots = N / 2;
    *out = ct;
    return check_cuda(c, "ct random");
}

fides_status fides_decrypt(fides_ctx* c, const fides_sk* sk, const fides_ct* ct, double* values, int slots) {
    if (!c || !sk || !sk->s || !ct || !ct->buf || !values || slots < 1 || slots > c->N / 2) return FIDES_BAD_ARG;
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    cudaSetDevice(c->device);
    const int n = ct->level + 1, N = c->N;
    // scratch: the n limbs of c0 + c1 s, N complex (FFT), slots complex (output)
    char* buf = nullptr;
    const size_t b_m = (size_t)n * N * 8, b_f = (size_t)N * 16, b_o = (size_t)slots * 16;
    if (cudaMallocAsync((void**)&buf, b_m + b_f + b_o, c->st) != cudaSuccess) {
        cudaGetLastError();
        return set_err(c, FIDES_OOM, "decrypt");
    }
    uint64_t* m = (uint64_t*)buf;
    double2* M = (double2*)(buf + b_m);
    double2* o = (double2*)(buf + b_m + b_f);
    launch_elementwise(c->dev, EW_MUL, n, 0, ct->c1(N), sk->s, m, c->st);
    launch_elementwise(c->dev, EW_ADD, n, 0, m, ct->c0(), m, c->st);
    ntt_inverse(c->dev, map_single(m, m, n, n, 0), IL_PLAIN, IS_PLAIN, c->st);
    CrtConst k{};
    k.use = std::min(n, 3);
    const uint64_t* q = c->host.prime.data();
    for (int i = 0; i < k.use; ++i) k.q[i] = q[i];
    if (k.use > 1) k.inv01 = invmod(q[0] % q[1], q[1]);
    if (k.use > 2) {
        k.inv02 = invmod(q[0] % q[2], q[2]);
        k.inv12 = invmod(q[1] % q[2], q[2]);
    }
    count_launches(2);
    k_decode_crt<<<(N + 255) / 256, 256, 0, c->st>>>(m, c->logN, k, c->dev.pc, ct->scale, M);
    fft_dev(c, M, 1.0);
    k_decode_gather<<<(slots + 255) / 256, 256, 0, c->st>>>(M, slots, c->logN, o);
    cudaMemcpyAsync(values, o, b_o, cudaMemcpyDeviceToHost, c->st);
    cudaFreeAsync(buf, c->st);
    cudaStreamSynchronize(c->st);
    return check_cuda(c, "decrypt");
}

}  // extern "C"
