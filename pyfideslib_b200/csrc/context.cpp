// context.cpp -- context construction: moduli, per-prime constants, twiddle
// and CRT tables in HBM, key-switch workspace.
//
// Role in the reference: CKKS::ContextData (src/CKKS/Context.cu:37-98) and
// SetupConstants (src/ConstantsGPU.cu:127-708), which upload per-prime
// scalars to __constant__ memory and 16+16 MiB of dense [MAXP][MAXD][MAXP][MAXP]
// conversion matrices.  Here every table is compact and level-indexed
// (~0.3 MiB of CRT data at L=30, K=10) and the twiddles are stored as
// (value, Shoup companion) pairs so that a butterfly reads one 16-byte word.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <thread>

#include "context.hpp"

namespace fides {

using u128 = unsigned __int128;

uint64_t mulmod(uint64_t a, uint64_t b, uint64_t p) { return (uint64_t)((u128)a * b % p); }

static uint64_t f64_bits(double x) {
    uint64_t u;
    std::memcpy(&u, &x, 8);
    return u;
}

// The double nearest above 1/p (p < 2^50): x = m 2^e with a 53-bit m, and
// x >= 1/p  <=>  m p >= 2^-e, checked in exact integer arithmetic.
static double recip_up(uint64_t p) {
    double x = 1.0 / (double)p;
    int e = 0;
    const double f = std::frexp(x, &e);                  // x = f 2^e, f in [0.5, 1)
    const uint64_t m = (uint64_t)std::ldexp(f, 53);      // x = m 2^(e - 53)
    const int sh = 53 - e;                               // 2^-(e-53) = 2^sh, sh <= 104 for p < 2^50
    if (sh < 128 && (u128)m * p < ((u128)1 << sh)) x = std::nextafter(x, 1.0);
    return x;
}

uint64_t powmod(uint64_t a, uint64_t e, uint64_t p) {
    uint64_t r = 1 % p;
    a %= p;
    while (e) {
        if (e & 1) r = mulmod(r, a, p);
        a = mulmod(a, a, p);
        e >>= 1;
    }
    return r;
}

uint64_t invmod(uint64_t a, uint64_t p) { return powmod(a % p, p - 2, p); }

bool is_prime(uint64_t n) {
    if (n < 2) return false;
    static const uint64_t small[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    for (uint64_t b : small) {
        if (n == b) return true;
        if (n % b == 0) return false;
    }
    uint64_t d = n - 1;
    int s = 0;
    while (!(d & 1)) {
        d >>= 1;
        ++s;
    }
    for (uint64_t b : small) {
        uint64_t x = powmod(b, d, n);
        if (x == 1 || x == n - 1) continue;
        bool comp = true;
        for (int r = 1; r < s && comp; ++r) {
            x = mulmod(x, x, n);
            if (x == n - 1) comp = false;
        }
        if (comp) return false;
    }
    return true;
}

// Pollard's rho (Brent variant) for the factorisation of p-1.
static uint64_t rho(uint64_t n, uint64_t c) {
    if (n % 2 == 0) return 2;
    uint64_t y = 2, x = 2, g = 1, q = 1, ys = 2;
    const uint64_t m = 128;
    uint64_t r = 1;
    auto f = [&](uint64_t v) { return (mulmod(v, v, n) + c) % n; };
    while (g == 1) {
        x = y;
        for (uint64_t i = 0; i < r; ++i) y = f(y);
        uint64_t k = 0;
        while (k < r && g == 1) {
            ys = y;
            for (uint64_t i = 0; i < std::min(m, r - k); ++i) {
                y = f(y);
                q = mulmod(q, x > y ? x - y : y - x, n);
            }
            g = std::gcd(q, n);
            k += m;
        }
        r <<= 1;
    }
    if (g == n) {
        do {
            ys = f(ys);
            g = std::gcd(x > ys ? x - ys : ys - x, n);
        } while (g == 1);
    }
    return g;
}

static void factor(uint64_t n, std::vector<uint64_t>& out) {
    if (n == 1) return;
    for (uint64_t p : {2ull, 3ull, 5ull, 7ull, 11ull, 13ull}) {
        if (n % p == 0) {
            out.push_back(p);
            while (n % p == 0) n /= p;
        }
    }
    if (n == 1) return;
    if (is_prime(n)) {
        out.push_back(n);
        return;
    }
    uint64_t d = n;
    for (uint64_t c = 1; d == n; ++c) d = rho(n, c);
    factor(d, out);
    factor(n / d, out);
}

// The smallest generator of (Z/p)^*: the rule FIDESlib applies when it builds
// its own roots (src/ConstantsGPU.cu:40-72 generator / unity_root).
uint64_t smallest_generator(uint64_t p) {
    std::vector<uint64_t> f;
    factor(p - 1, f);
    std::sort(f.begin(), f.end());
    f.erase(std::unique(f.begin(), f.end()), f.end());
    for (uint64_t g = 2; g < p; ++g) {
        bool ok = true;
        for (uint64_t q : f)
            if (powmod(g, (p - 1) / q, p) == 1) {
                ok = false;
                break;
            }
        if (ok) return g;
    }
    return 0;
}

std::vector<uint64_t> find_ntt_primes(int logN, int bits, int count, uint64_t upper_exclusive) {
    std::vector<uint64_t> out;
    const uint64_t step = 2ull << logN;
    uint64_t lim = (bits < 64) ? (1ull << bits) : ~0ull;
    if (upper_exclusive && upper_exclusive < lim) lim = upper_exclusive;
    const uint64_t lo = 1ull << (bits - 1);
    uint64_t cand = ((lim - 2) / step) * step + 1;
    while ((int)out.size() < count && cand > lo) {
        if (is_prime(cand)) out.push_back(cand);
        cand -= step;
    }
    return out;
}

static uint32_t bitrev(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int i = 0; i < bits; ++i) {
        r = (r << 1) | (x & 1);
        x >>= 1;
    }
    return r;
}

fides_status set_err(fides_ctx* c, fides_status s, const std::string& msg) {
    if (c) c->last_error = msg;
    return s;
}

fides_status check_cuda(fides_ctx* c, const char* where) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_err(c, FIDES_CUDA_ERR, std::string(where) + ": " + cudaGetErrorString(e));
    return FIDES_OK;
}

uint32_t read_device_error(fides_ctx* c, cudaStream_t st, bool clear) {
    if (!c->dev.err) return 0;
    if (!st) st = c->st;
    uint32_t w = 0;
    if (cudaMemcpyAsync(&w, c->dev.err, sizeof(w), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return 0;  // the CUDA error itself is reported by check_cuda
    if (w && clear) {
        cudaMemsetAsync(c->dev.err, 0, sizeof(uint32_t), st);
        cudaStreamSynchronize(st);
    }
    return w;
}

fides_status consume_device_error(fides_ctx* c, cudaStream_t st) {
    const uint32_t w = read_device_error(c, st, true);
    if (w & kDevErrTensorWait)
        return set_err(c, FIDES_TIMEOUT,
                       "a tensor-core base conversion stopped waiting for its matrix products: results computed "
                       "since the previous synchronising call are invalid");
    if (w) return set_err(c, FIDES_TIMEOUT, "device error word " + std::to_string(w));
    return FIDES_OK;
}

LimbMap map_single(const uint64_t* in, uint64_t* out, int count, int nq, int q0, int level, const uint64_t* in2,
                   const uint64_t* in3) {
    LimbMap m{};
    m.nseg = 1;
    m.total = count;
    LimbSeg& s = m.seg[0];
    s.in = in;
    s.in2 = in2;
    s.in3 = in3;
    s.out = out;
    s.count = count;
    s.skip_lo = count;
    s.skip_cnt = 0;
    s.nq = nq;
    s.q0 = q0;
    s.level = level;
    s.in_stride_zero = 0;
    return m;
}

// ---------------------------------------------------------------------------

static void put4(uint64_t* dst, uint64_t s, uint64_t w1, uint64_t p) {
    const uint64_t sw = mulmod(s, w1, p);
    dst[0] = s;
    dst[1] = shoup_precompute(s, p);
    dst[2] = sw;
    dst[3] = shoup_precompute(sw, p);
}

bool select_moduli(const fides_params* prm, std::vector<uint64_t>& q, std::vector<uint64_t>& p) {
    const int logN = prm->log_n, L = prm->num_q, dnum = prm->dnum;
    const int alpha = (L + dnum - 1) / dnum;
    const int q0b = prm->q0_bits ? prm->q0_bits : 60;
    const int qib = prm->qi_bits ? prm->qi_bits : 50;
    const int pb = prm->p_bits ? prm->p_bits : 60;
    q.clear();
    p.clear();
    if (prm->q) {
        q.assign(prm->q, prm->q + L);
    } else {
        auto a = find_ntt_primes(logN, q0b, 1, 0);
        auto b = find_ntt_primes(logN, qib, L - 1, 0);
        if ((int)a.size() < 1 || (int)b.size() < L - 1) return false;
        q.push_back(a[0]);
        for (uint64_t x : b) {
            if (x == a[0]) return false;
            q.push_back(x);
        }
    }
    int K = prm->num_p;
    if (prm->p) {
        if (K < 1) return false;
        p.assign(prm->p, prm->p + K);
        return true;
    }
    if (K <= 0) {
        // enough special bits to cover the widest digit (Context.cu:283 computeK)
        int maxbits = 0;
        for (int d = 0; d < dnum; ++d) {
            int bits = 0;
            for (int i = d * alpha; i < std::min(L, (d + 1) * alpha); ++i) bits += 64 - __builtin_clzll(q[i]);
            maxbits = std::max(maxbits, bits);
        }
        K = (maxbits + pb - 2) / (pb - 1);
    }
    // special moduli continue the same descending search, skipping the q's
    std::vector<uint64_t> cand = find_ntt_primes(logN, pb, K + L + 2, 0);
    for (uint64_t x : cand) {
        if ((int)p.size() == K) break;
        if (std::find(q.begin(), q.end(), x) == q.end()) p.push_back(x);
    }
    return (int)p.size() == K;
}

fides_status build_context(fides_ctx* c, const fides_params* prm) {
    c->logN = prm->log_n;
    c->N = 1 << c->logN;
    c->L = prm->num_q;
    c->dnum = prm->dnum;
    c->alpha = (c->L + c->dnum - 1) / c->dnum;
    const int logN = c->logN, N = c->N, L = c->L;
    const int qib = prm->qi_bits ? prm->qi_bits : 50;

    std::vector<uint64_t> q, p;
    if (!select_moduli(prm, q, p)) return set_err(c, FIDES_BAD_ARG, "cannot select moduli for these parameters");
    const int K = (int)p.size();
    c->K = K;
    const int NP = L + K;
    if (c->alpha > 16 || K > 16 || c->dnum > 8)
        return set_err(c, FIDES_UNSUPPORTED, "need digit size <= 16, special moduli <= 16, dnum <= 8");
    if (NP > kMaxPrimes) return set_err(c, FIDES_BAD_ARG, "too many primes");
    for (int i = 0; i < NP; ++i) {
        uint64_t x = i < L ? q[i] : p[i - L];
        if (x >= (1ull << 62) || (x - 1) % (2ull * N) != 0 || !is_prime(x))
            return set_err(c, FIDES_BAD_ARG, "modulus " + std::to_string(x) + " is not an NTT prime < 2^62");
        for (int j = 0; j < i; ++j)
            if (c->host.prime.size() > (size_t)j && c->host.prime[j] == x) return set_err(c, FIDES_BAD_ARG, "duplicate modulus");
        c->host.prime.push_back(x);
    }
    c->default_scale = prm->default_scale > 0 ? prm->default_scale : (double)(1ull << qib);

    // ---- per-prime constants and twiddles (host) ----
    c->host.pc.resize(NP);
    c->host.root.resize(NP);
    std::vector<uint64_t> fwd((size_t)NP * N * 2), inv((size_t)NP * N * 2), fwdf((size_t)NP * N * 2, 0),
        invf((size_t)NP * N * 2, 0);
    auto work = [&](int i) {
        const uint64_t pr = c->host.prime[i];
        PrimeConst& k = c->host.pc[i];
        k.p = pr;
        k.two_p = 2 * pr;
        k.mu64 = (uint64_t)((((u128)1) << 64) / pr);
        k.r64 = (uint64_t)((((u128)1) << 64) % pr);
        k.r64_sh = shoup_precompute(k.r64, pr);
        k.ninv = invmod((uint64_t)N % pr, pr);
        k.ninv_sh = shoup_precompute(k.ninv, pr);
        const uint64_t* given = i < L ? prm->q_root : prm->p_root;
        uint64_t psi = 0;
        if (given) {
            psi = given[i < L ? i : i - L];
            // a primitive 2N-th root: psi^N = -1 (its order divides 2N, not N)
            if (psi == 0 || psi >= pr || powmod(psi, (uint64_t)N, pr) != pr - 1) {
                c->host.root[i] = 0;
                return;
            }
        } else {
            psi = powmod(smallest_generator(pr), (pr - 1) / (2ull * N), pr);
        }
        const uint64_t ipsi = invmod(psi, pr);
        c->host.root[i] = psi;
        std::vector<uint64_t> a(N), b(N);
        a[0] = b[0] = 1;
        for (int j = 1; j < N; ++j) {
            a[j] = mulmod(a[j - 1], psi, pr);
            b[j] = mulmod(b[j - 1], ipsi, pr);
        }
        uint64_t* F = fwd.data() + (size_t)i * N * 2;
        uint64_t* I = inv.data() + (size_t)i * N * 2;
        for (int j = 0; j < N; ++j) {
            const uint32_t r = bitrev((uint32_t)j, logN);
            F[2 * j] = a[r];
            F[2 * j + 1] = shoup_precompute(a[r], pr);
            I[2 * j] = b[r];
            I[2 * j + 1] = shoup_precompute(b[r], pr);
        }
        // double-precision butterflies (primes below 2^50): w and the
        // correctly rounded quotient w / p
        if (pr < kFpPrimeBound) {
            k.pinv_f64 = f64_bits(recip_up(pr));
            uint64_t* D = fwdf.data() + (size_t)i * N * 2;
            uint64_t* E = invf.data() + (size_t)i * N * 2;
            for (int j = 0; j < N; ++j) {
                const double w = (double)F[2 * j], v = (double)I[2 * j];
                D[2 * j] = f64_bits(w);
                D[2 * j + 1] = f64_bits(w / (double)pr);
                E[2 * j] = f64_bits(v);
                E[2 * j + 1] = f64_bits(v / (double)pr);
            }
        }
    };
    {
        unsigned nth = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        std::vector<std::thread> th;
        for (unsigned t = 0; t < nth; ++t)
            th.emplace_back([&, t] {
                for (int i = (int)t; i < NP; i += (int)nth) work(i);
            });
        for (auto& x : th) x.join();
    }
    for (int i = 0; i < NP; ++i)
        if (c->host.root[i] == 0)
            return set_err(c, FIDES_BAD_ARG, "modulus " + std::to_string(c->host.prime[i]) +
                                                 ": no primitive 2N-th root (or the given one is not)");

    // ---- CRT tables ----
    auto P = [&](int i) { return c->host.prime[i]; };
    std::vector<uint64_t> intt_scale((size_t)NP * 4);
    for (int i = 0; i < NP; ++i) put4(&intt_scale[(size_t)i * 4], c->host.pc[i].ninv, inv[(size_t)i * N * 2 + 2], P(i));

    std::vector<uint64_t> modup_scale((size_t)L * L * 4, 0), modup_mat((size_t)L * L * NP, 0);
    for (int lev = 0; lev < L; ++lev) {
        for (int d = 0; d * c->alpha <= lev; ++d) {
            const int lo = d * c->alpha, hi = std::min(lo + c->alpha - 1, lev);
            for (int i = lo; i <= hi; ++i) {
                uint64_t acc = 1;
                for (int k = lo; k <= hi; ++k)
                    if (k != i) acc = mulmod(acc, P(k) % P(i), P(i));
                const uint64_t hinv = invmod(acc, P(i));
                put4(&modup_scale[((size_t)lev * L + i) * 4], mulmod(hinv, c->host.pc[i].ninv, P(i)),
                     inv[(size_t)i * N * 2 + 2], P(i));
                for (int t = 0; t < NP; ++t) {
                    uint64_t a2 = 1;
                    for (int k = lo; k <= hi; ++k)
                        if (k != i) a2 = mulmod(a2, P(k) % P(t), P(t));
                    modup_mat[((size_t)lev * L + i) * NP + t] = a2;
                }
            }
        }
    }
    std::vector<uint64_t> md_scale((size_t)std::max(K, 1) * 4), md_mat((size_t)std::max(K, 1) * L),
        md_pinv((size_t)L * 2), md_pmod((size_t)L * 2);
    for (int k = 0; k < K; ++k) {
        const uint64_t pk = P(L + k);
        uint64_t acc = 1;
        for (int m = 0; m < K; ++m)
            if (m != k) acc = mulmod(acc, P(L + m) % pk, pk);
        put4(&md_scale[(size_t)k * 4], mulmod(invmod(acc, pk), c->host.pc[L + k].ninv, pk),
             inv[(size_t)(L + k) * N * 2 + 2], pk);
        for (int j = 0; j < L; ++j) {
            uint64_t a2 = 1;
            for (int m = 0; m < K; ++m)
                if (m != k) a2 = mulmod(a2, P(L + m) % P(j), P(j));
            md_mat[(size_t)k * L + j] = a2;
        }
    }
    for (int j = 0; j < L; ++j) {
        uint64_t acc = 1;
        for (int m = 0; m < K; ++m) acc = mulmod(acc, P(L + m) % P(j), P(j));
        const uint64_t pinv = invmod(acc, P(j));
        md_pinv[2 * j] = pinv;
        md_pinv[2 * j + 1] = shoup_precompute(pinv, P(j));
        md_pmod[2 * j] = acc;
        md_pmod[2 * j + 1] = shoup_precompute(acc, P(j));
    }
    std::vector<uint64_t> rs_qinv((size_t)L * L * 2, 0);
    for (int l = 1; l < L; ++l)
        for (int j = 0; j < l; ++j) {
            const uint64_t v = invmod(P(l) % P(j), P(j));
            rs_qinv[((size_t)l * L + j) * 2] = v;
            rs_qinv[((size_t)l * L + j) * 2 + 1] = shoup_precompute(v, P(j));
        }

    // ---- upload ----
    if (cudaSetDevice(prm->device) != cudaSuccess) return set_err(c, FIDES_CUDA_ERR, "cudaSetDevice failed");
    c->device = prm->device;
    if (cudaStreamCreateWithFlags(&c->h2d, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->d2h, cudaStreamNonBlocking) != cudaSuccess)
        return set_err(c, FIDES_CUDA_ERR, "copy stream creation failed");
    if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess)
        return set_err(c, FIDES_CUDA_ERR, "stream create failed");
    struct Part {
        const void* src;
        size_t bytes;
        size_t off;
    };
    std::vector<Part> parts;
    size_t off = 0;
    auto add = [&](const void* src, size_t bytes) {
        off = (off + 255) & ~(size_t)255;
        parts.push_back({src, bytes, off});
        off += bytes;
        return parts.size() - 1;
    };
    size_t i_pc = add(c->host.pc.data(), sizeof(PrimeConst) * NP);
    size_t i_fwd = add(fwd.data(), fwd.size() * 8);
    size_t i_inv = add(inv.data(), inv.size() * 8);
    size_t i_fwdf = add(fwdf.data(), fwdf.size() * 8);
    size_t i_invf = add(invf.data(), invf.size() * 8);
    size_t i_is = add(intt_scale.data(), intt_scale.size() * 8);
    size_t i_ms = add(modup_scale.data(), modup_scale.size() * 8);
    size_t i_mm = add(modup_mat.data(), modup_mat.size() * 8);
    size_t i_ds = add(md_scale.data(), md_scale.size() * 8);
    size_t i_dm = add(md_mat.data(), md_mat.size() * 8);
    size_t i_dp = add(md_pinv.data(), md_pinv.size() * 8);
    size_t i_dq = add(md_pmod.data(), md_pmod.size() * 8);
    size_t i_rq = add(rs_qinv.data(), rs_qinv.size() * 8);
    const uint64_t zero_word = 0;
    size_t i_err = add(&zero_word, sizeof(zero_word));
    c->table_bytes = off;
    if (cudaMalloc(&c->table_mem, off) != cudaSuccess) return set_err(c, FIDES_OOM, "table allocation failed");
    char* base = (char*)c->table_mem;
    for (auto& pt : parts)
        if (cudaMemcpy(base + pt.off, pt.src, pt.bytes, cudaMemcpyHostToDevice) != cudaSuccess)
            return set_err(c, FIDES_CUDA_ERR, "table upload failed");
    DevCtx& d = c->dev;
    d.logN = logN;
    d.N = N;
    d.L = L;
    d.K = K;
    d.dnum = c->dnum;
    d.alpha = c->alpha;
    d.ntt_variant = d.intt_variant = d.conv_variant = 0;  // chosen by the autotuner
    d.ks_variant = 1 | 4 | 8;  // FP64 sums; fused into the row pass (split launch) for batches of 8 or more
    d.pc = (const PrimeConst*)(base + parts[i_pc].off);
    d.fwd_tw = (const uint64_t*)(base + parts[i_fwd].off);
    d.inv_tw = (const uint64_t*)(base + parts[i_inv].off);
    d.fwd_twf = (const uint64_t*)(base + parts[i_fwdf].off);
    d.inv_twf = (const uint64_t*)(base + parts[i_invf].off);
    d.intt_scale = (const uint64_t*)(base + parts[i_is].off);
    d.modup_scale = (const uint64_t*)(base + parts[i_ms].off);
    d.modup_mat = (const uint64_t*)(base + parts[i_mm].off);
    d.md_scale = (const uint64_t*)(base + parts[i_ds].off);
    d.md_mat = (const uint64_t*)(base + parts[i_dm].off);
    d.md_pinv = (const uint64_t*)(base + parts[i_dp].off);
    d.md_pmod = (const uint64_t*)(base + parts[i_dq].off);
    d.rs_qinv = (const uint64_t*)(base + parts[i_rq].off);
    d.err = (uint32_t*)(base + parts[i_err].off);
    ntt_prepare(d);
    d.tc_btab = nullptr;
    d.tc_boff = nullptr;
    if (conv_tc_eligible(d)) {
        // byte matrices of the tensor-core conversions, one per (level, digit)
        // and per (level, fused) ModDown (a few MB); without them the
        // conversions run on the integer pipes
        std::vector<uint64_t> offs;
        const size_t bytes = conv_tc_table_layout(d, offs);
        const size_t obytes = offs.size() * sizeof(uint64_t);
        if (cudaMalloc(&c->tc_mem, bytes + obytes) == cudaSuccess) {
            uint8_t* tb = (uint8_t*)c->tc_mem;
            if (cudaMemcpy(tb + bytes, offs.data(), obytes, cudaMemcpyHostToDevice) == cudaSuccess) {
                d.tc_btab = tb;
                d.tc_boff = (const uint64_t*)(tb + bytes);
                conv_tc_build_tables(d, c->st);
                if (cudaStreamSynchronize(c->st) != cudaSuccess) return set_err(c, FIDES_CUDA_ERR, "table build failed");
            }
        } else {
            cudaGetLastError();
        }
    }

    // ---- key-switch workspace for single operations ----
    return ws_reserve(c, c->ws1, 1);
}

fides_status key_alloc(fides_ctx* c, SwitchKey& k, bool seeded) {
    const size_t words = (size_t)c->dnum * (c->L + c->K) * c->N;
    if (k.b && k.seeded != seeded) {
        cudaStreamSynchronize(c->st);  // kernels queued with the old key
        cudaFree(k.b);
        k.b = k.a = nullptr;
    }
    if (!k.b) {
        if (cudaMalloc((void**)&k.b, (seeded ? 1 : 2) * words * sizeof(uint64_t)) != cudaSuccess) {
            cudaGetLastError();
            k.b = nullptr;
            return set_err(c, FIDES_OOM, "key allocation failed");
        }
    }
    k.seeded = seeded;
    k.a = seeded ? nullptr : k.b + words;
    if (!seeded) k.a_seed = 0;
    return FIDES_OK;
}

fides_status ws_reserve(fides_ctx* c, Workspace& w, int cap) {
    if (!w.st) w.st = c->st;
    if (w.base && w.cap >= cap) return FIDES_OK;
    cudaStream_t keep = w.st;
    ws_free(w);
    w.st = keep;
    const size_t L = c->L, K = c->K, N = c->N;
    w.dig_stride = L + K;
    const size_t limbs = 4 * L /*E0,E1,E2,XT*/ + c->dnum * w.dig_stride /*DIG*/ + 2 * (L + K) /*XB,XA*/ +
                         2 * L /*W*/ + 2 /*T*/;
    w.stride = limbs * N;
    if (cudaMalloc((void**)&w.base, w.stride * 8 * (size_t)cap) != cudaSuccess) {
        cudaGetLastError();
        w.base = nullptr;
        return set_err(c, FIDES_OOM, "workspace allocation failed");
    }
    w.cap = cap;
    uint64_t* p = w.base;
    auto take = [&](size_t n) {
        uint64_t* r = p;
        p += n * N;
        return r;
    };
    w.E0 = take(L);
    w.E1 = take(L);
    w.E2 = take(L);
    w.XT = take(L);
    w.DIG = take(c->dnum * w.dig_stride);
    w.XB = take(L + K);
    w.XA = take(L + K);
    w.W = take(2 * L);
    w.T = take(2);
    return FIDES_OK;
}

void ws_free(Workspace& w) {
    if (w.base) cudaFree(w.base);
    w = Workspace{};
}

void free_context(fides_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->st) cudaStreamSynchronize(c->st);
    c->boot.clear();
    auto freek = [](SwitchKey& k) {
        if (k.b) cudaFree(k.b);
        k.b = k.a = nullptr;
        k.seeded = false;
    };
    if (c->has_relin) freek(c->relin);
    for (auto& kv : c->galois_keys) freek(kv.second);
    c->galois_keys.clear();
    ws_free(c->ws1);
    ws_free(c->wsb);
    if (c->table_mem) cudaFree(c->table_mem);
    if (c->tc_mem) cudaFree(c->tc_mem);
    c->tc_mem = nullptr;
    if (c->st) cudaStreamDestroy(c->st);
    if (c->h2d) cudaStreamSynchronize(c->h2d), cudaStreamDestroy(c->h2d);
    if (c->d2h) cudaStreamSynchronize(c->d2h), cudaStreamDestroy(c->d2h);
    c->table_mem = nullptr;
    c->st = nullptr;
    c->h2d = c->d2h = nullptr;
}

void int_const_limbs(const fides_ctx* c, int64_t z, int nlimbs, uint64_t (*out)[2]) {
    const uint64_t mag = z < 0 ? (uint64_t)(-(z + 1)) + 1 : (uint64_t)z;
    for (int j = 0; j < nlimbs; ++j) {
        const uint64_t p = c->host.prime[j];
        uint64_t r = mag % p;
        if (z < 0 && r) r = p - r;
        out[j][0] = r;
        out[j][1] = shoup_precompute(r, p);
    }
}

void ct_quiesce(fides_ctx* c, const fides_ct* ct, cudaStream_t st) {
    if (!ct->d2h_ev) return;
    cudaStreamWaitEvent(st ? st : c->st, ct->d2h_ev, 0);
    cudaEventDestroy(ct->d2h_ev);
    ct->d2h_ev = nullptr;
}

fides_status ct_reserve(fides_ctx* c, fides_ct* ct, int level, cudaStream_t st) {
    if (!st) st = c->st;
    ct_quiesce(c, ct, st);
    if (ct->buf && ct->cap >= level + 1) return FIDES_OK;
    if (ct->buf) cudaFreeAsync(ct->buf, st);
    ct->buf = nullptr;
    ct->cap = level + 1;
    ct->ring = c->N;
    const size_t bytes = 2 * (size_t)ct->cap * c->limb_bytes();
    const cudaError_t e = cudaMallocAsync((void**)&ct->buf, bytes, st);
    if (e != cudaSuccess) {
        ct->cap = 0;
        cudaGetLastError();
        return set_err(c, FIDES_OOM, "ciphertext allocation failed");
    }
    return FIDES_OK;
}

}  // namespace fides
