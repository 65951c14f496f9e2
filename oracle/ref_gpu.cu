// ref_gpu.cu -- a harness that runs the reference's own GPU kernels of the
// evaluation path on this machine's GPU, for the per-kernel comparison with
// this library.  TEST INFRASTRUCTURE ONLY: built by `make -C oracle ref-gpu`
// from the reference tree (src/NTT.cu, src/CKKS/Conv.cu,
// src/CKKS/ElemenwiseBatchKernels.cu and src/Rotation.cu compiled unmodified)
// into oracle/_ref/,
// loaded only by tests/test_gpu_ref_kernels.py.
//
// Kernels and the launch geometry each entry point repeats:
//   * forward NTT_<second, ALGO_SHOUP, NTT_NONE> pair and inverse INTT_ pair,
//     LimbPartition::ApplyNTT / ApplyINTT (src/CKKS/LimbPartition.cu:364-395,
//     :425-446);
//   * DecompAndModUpConv<ALGO_SHOUP>, grid N/64 x (64, 2), one digit per
//     launch (src/CKKS/LimbPartitionMGPU.cu:823-832);
//   * ModDown2<ALGO_SHOUP>, grid N/64 x (64, 2), one polynomial per launch
//     (src/CKKS/LimbPartitionMGPU.cu:1121-1129);
//   * fusedDotKSK_2_, grid (N/128, K + n) x 128 (src/CKKS/LimbPartitionMGPU.cu:444);
//   * hoistedRotateDotKSK_2_, grid (N/128, K + n) x 128, 128 num_d words of
//     shared memory (src/CKKS/LimbPartitionMGPU.cu:553);
//   * binomialMult_ and automorph_multi_, grid (N/128, limbs) x 128
//     (src/CKKS/LimbPartition.cu:2592, :2004).
//
// The reference reads its tables from a __constant__ Constants block and a
// device Global::Globals block that SetupConstants fills from OpenFHE
// (src/ConstantsGPU.cu:127-708).  Here both are allocated at their full
// declared sizes (src/ConstantsGPU.cuh:30-71,136-160), so every table index the
// kernels form from values below MAXP / MAXD is inside them; every field the
// kernels read is filled with the definition SetupConstants uses: primes,
// Barrett mu and bit widths (:32-35 mu_new), Shoup companions (:71-74), the psi
// tables (:188-320), the digit lists and counts (:660-690), PartQlHatInvModq /
// PartQlHatModp (:545-620), PHatInvModp / PHatModq (:493-541).  The host checks
// every count and id against MAXP / MAXD before a table is uploaded.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <map>
#include <vector>

#include "CKKS/Conv.cuh"
#include "CKKS/ElemenwiseBatchKernels.cuh"
#include "ConstantsGPU.cuh"
#include "NTT.cuh"
#include "Rotation.cuh"

namespace FIDESlib {
__constant__ Constants constants;
}

using namespace FIDESlib;

namespace {

typedef unsigned __int128 u128;

uint64_t mulmod(uint64_t a, uint64_t b, uint64_t p) { return (uint64_t)((u128)a * b % p); }
uint64_t powmod(uint64_t a, uint64_t e, uint64_t p) {
    uint64_t r = 1;
    while (e) {
        if (e & 1) r = mulmod(r, a, p);
        a = mulmod(a, a, p);
        e >>= 1;
    }
    return r;
}
uint32_t bitrev(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int b = 0; b < bits; ++b)
        if (x >> b & 1) r |= 1u << (bits - 1 - b);
    return r;
}
int bit_width(uint64_t x) {
    int b = 0;
    while (x) {
        ++b;
        x >>= 1;
    }
    return b;
}
uint64_t shoup(uint64_t v, uint64_t p) { return (uint64_t)(((u128)(v << 1) << 63) / p); }

struct State {
    int logN = 0, N = 0, np = 0;
    int L = 0, K = 0, dnum = 0, alpha = 0;  // key-switch shape (set_keyswitch)
    Global::Globals* dglob = nullptr;        // device copy of the table block
    std::vector<void*> tables;               // device tables owned here
    // device pointer arrays of the launches, by their arguments: a repeated
    // call launches without uploading anything
    std::map<std::vector<const void*>, void**> ptr_tables;
} g;
Constants hc;           // host image of the constant block
Global::Globals hg;     // host image of the table block

void release() {
    for (void* t : g.tables) cudaFree(t);
    g.tables.clear();
    if (g.dglob) cudaFree(g.dglob);
    g.dglob = nullptr;
    for (auto& kv : g.ptr_tables) cudaFree(kv.second);
    g.ptr_tables.clear();
}

// the limb-to-prime map the multi-limb NTT kernels read: entry k is prime
// k mod np over the whole flattened index table
void flat_identity() {
    for (int k = 0; k < (MAXD * 3 + 1) * MAXP; ++k) hc.primeid_flattened[k] = k % g.np;
}

int upload_constants() {
    if (cudaMemcpyToSymbol(constants, &hc, sizeof(hc)) != cudaSuccess) return 5;
    if (cudaMemcpy(g.dglob, &hg, sizeof(hg), cudaMemcpyHostToDevice) != cudaSuccess) return 5;
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 5;
}

// The device array of n pointers for a launch with arguments `key`: built by
// fill(host, device_base) on first use (the device base lets a table point
// into itself), then reused.  Null on allocation failure.
template <class F>
void** ptr_table(const std::vector<const void*>& key, size_t n, cudaStream_t st, F fill) {
    auto it = g.ptr_tables.find(key);
    if (it != g.ptr_tables.end()) return it->second;
    if (g.ptr_tables.size() >= 64) {
        cudaStreamSynchronize(st);
        for (auto& kv : g.ptr_tables) cudaFree(kv.second);
        g.ptr_tables.clear();
    }
    void** d = nullptr;
    if (cudaMalloc((void**)&d, n * sizeof(void*)) != cudaSuccess) return nullptr;
    std::vector<void*> h(n, nullptr);
    fill(h, d);
    if (cudaMemcpy(d, h.data(), n * sizeof(void*), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(d);
        return nullptr;
    }
    g.ptr_tables[key] = d;
    return d;
}

}  // namespace

extern "C" {

// Tables for nprimes primes (p_i = 1 mod 2N, below 2^62) with the primitive
// 2N-th roots psi[i], ring dimension 2^logN, 12 <= logN <= 16.  The prime ids
// of the other entry points are indices into this list.  0 on success.
int refgpu_init(int logN, int nprimes, const uint64_t* primes, const uint64_t* psi) {
    if (logN < 12 || logN > 16 || nprimes < 1 || nprimes > MAXP || !primes || !psi) return 1;
    release();
    const int N = 1 << logN;
    for (int i = 0; i < nprimes; ++i) {
        const uint64_t p = primes[i];
        if (p >= (1ull << 62) || (p - 1) % (2ull * N) != 0) return 2;
        if (powmod(psi[i], N, p) != p - 1) return 3;  // not a primitive 2N-th root
    }
    memset(&hc, 0, sizeof(hc));
    hc.N = N;
    hc.L = nprimes;
    hc.K = 0;
    hc.logN = logN;
    hc.dnum = 1;
    hc.type = 0;
    memset(&hg, 0, sizeof(hg));
    for (int i = 0; i < nprimes; ++i) {
        const uint64_t p = primes[i];
        const int bits = bit_width(p);
        hc.type |= (uint64_t)1 << i;  // 64-bit limbs
        hc.primes[i] = p;
        hc.prime_bits[i] = (uint32_t)bits;
        hc.prime_better_barret_mu[i] = (uint64_t)(((u128)1 << (2 * bits + 1)) / p);  // mu_new, NEIL
        const uint64_t ninv = powmod(N, p - 2, p), iroot = powmod(psi[i], p - 2, p);
        hc.N_shoup[i] = shoup(N % p, p);
        hc.N_inv[i] = ninv;
        hc.N_inv_shoup[i] = shoup(ninv, p);
        hc.root[i] = psi[i];
        hc.root_shoup[i] = shoup(psi[i], p);
        hc.inv_root[i] = iroot;
        hc.inv_root_shoup[i] = shoup(iroot, p);
        std::vector<uint64_t> no(2 * (size_t)N), ino(2 * (size_t)N), br(N), ibr(N), sh(N), ish(N), ms(N), ims(N);
        no[0] = ino[0] = 1;
        for (int j = 1; j < 2 * N; ++j) {
            no[j] = mulmod(no[j - 1], psi[i], p);
            ino[j] = mulmod(ino[j - 1], iroot, p);
        }
        for (int j = 0; j < N; ++j) {
            br[j] = no[bitrev(j, logN)];
            ibr[j] = ino[bitrev(j, logN)];
        }
        const int aw = (logN + 1) / 2;
        for (int j = 0; j < N / (1 << aw); ++j)
            for (int k = 0; k < (1 << aw); ++k) {
                ms[(size_t)j * (1 << aw) + k] = no[(size_t)j * bitrev(k, aw)];
                ims[(size_t)j * (1 << aw) + k] = mulmod(ino[(size_t)j * bitrev(k, aw)], ninv, p);
            }
        for (int j = 0; j < 2 * N; ++j) ino[j] = mulmod(ino[j], ninv, p);
        for (int j = 0; j < N; ++j) {
            sh[j] = shoup(br[j], p);
            ish[j] = shoup(ibr[j], p);
        }
        auto up = [&](const std::vector<uint64_t>& v) -> void* {
            void* d = nullptr;
            if (cudaMalloc(&d, v.size() * 8) != cudaSuccess) return nullptr;
            g.tables.push_back(d);
            cudaMemcpy(d, v.data(), v.size() * 8, cudaMemcpyHostToDevice);
            return d;
        };
        hg.psi[i] = up(br);
        hg.inv_psi[i] = up(ibr);
        hg.psi_no[i] = up(no);
        hg.inv_psi_no[i] = up(ino);
        hg.psi_middle_scale[i] = up(ms);
        hg.inv_psi_middle_scale[i] = up(ims);
        hg.psi_shoup[i] = up(sh);
        hg.inv_psi_shoup[i] = up(ish);
        if (!hg.psi[i] || !hg.inv_psi[i] || !hg.psi_no[i] || !hg.inv_psi_no[i] || !hg.psi_middle_scale[i] ||
            !hg.inv_psi_middle_scale[i] || !hg.psi_shoup[i] || !hg.inv_psi_shoup[i]) {
            release();
            return 4;
        }
    }
    g.logN = logN;
    g.N = N;
    g.np = nprimes;
    g.L = g.K = g.dnum = g.alpha = 0;
    flat_identity();
    if (cudaMalloc((void**)&g.dglob, sizeof(Global::Globals)) != cudaSuccess) {
        release();
        return 4;
    }
    const int rc = upload_constants();
    if (rc) release();
    return rc;
}

// Forward (inverse = 0) or inverse (1) NTT of nlimbs limbs in place: limb k
// at data + k*N uses prime (prime0 + k) mod nprimes; aux (nlimbs*N words)
// holds the first pass's output.  The two launches of ApplyNTT / ApplyINTT
// with their geometry.  Needs the identity limb map: call before
// refgpu_set_keyswitch, or after refgpu_init again.  0 on success.
int refgpu_transform(uint64_t* data, uint64_t* aux, int prime0, int nlimbs, int inverse, void* stream) {
    if (!g.dglob || !data || !aux || nlimbs < 1 || prime0 < 0 || g.L ||
        prime0 + nlimbs > (MAXD * 3 + 1) * MAXP || nlimbs > 65535)
        return 1;
    const int N = g.N, logN = g.logN;
    cudaStream_t st = (cudaStream_t)stream;
    void** ptrs = ptr_table({"transform", data, aux, (const void*)(size_t)nlimbs}, 2 * (size_t)nlimbs, st,
                            [&](std::vector<void*>& h, void**) {
                                for (int k = 0; k < nlimbs; ++k) {
                                    h[k] = data + (size_t)k * N;
                                    h[nlimbs + k] = aux + (size_t)k * N;
                                }
                            });
    if (!ptrs) return 2;
    constexpr int M = 4;
    constexpr ALGO algo = ALGO_SHOUP;
    void** dptr = ptrs;
    void** aptr = ptrs + nlimbs;
    if (!inverse) {
        const dim3 b1{(uint32_t)(1 << ((logN + 1) / 2 - 1))};
        const dim3 b2{(uint32_t)(1 << (logN / 2 - 1))};
        const int bytes1 = 8 * b1.x * (2 * M + 1 + 1);
        const int bytes2 = 8 * b2.x * (2 * M + 1 + 1);
        NTT_<false, algo, NTT_NONE><<<dim3{(uint32_t)N / (b1.x * M * 2), (uint32_t)nlimbs}, b1, bytes1, st>>>(
            g.dglob, dptr, prime0, aptr, nullptr, 0, nullptr, nullptr);
        NTT_<true, algo, NTT_NONE><<<dim3{(uint32_t)N / (b2.x * M * 2), (uint32_t)nlimbs}, b2, bytes2, st>>>(
            g.dglob, aptr, prime0, dptr, nullptr, 0, nullptr, nullptr);
    } else {
        const dim3 b1{(uint32_t)(1 << (logN / 2 - 1))};
        const dim3 b2{(uint32_t)(1 << ((logN + 1) / 2 - 1))};
        const int bytes1 = 8 * b1.x * (2 * M + 1 + 1);
        const int bytes2 = 8 * b2.x * (2 * M + 1 + 1);
        INTT_<false, algo, INTT_NONE><<<dim3{(uint32_t)N / (b1.x * M * 2), (uint32_t)nlimbs}, b1, bytes1, st>>>(
            g.dglob, dptr, prime0, aptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
        INTT_<true, algo, INTT_NONE><<<dim3{(uint32_t)N / (b2.x * M * 2), (uint32_t)nlimbs}, b2, bytes2, st>>>(
            g.dglob, aptr, prime0, dptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

// Key-switch shape: the init's primes are L ciphertext primes then K special
// primes (L + K == nprimes), digits of alpha = ceil(L / dnum) primes.
// hat_inv[d][l][i] / hat_mod[d][l][i][t] (d < dnum, l < L, i < alpha,
// t < L + K): ModUp's (Q_hat_i)^-1 mod q_i and Q_hat_i mod prime t of digit d
// at level l (PartQlHatInvModq / PartQlHatModp, zero where unused);
// phat_inv[k], phat_mod[k][j] (k < K, j < L): ModDown's (P_hat_k)^-1 mod p_k
// and P_hat_k mod q_j (PHatInvModp / PHatModq).  Replaces the identity limb
// map with the digit and partition lists.  0 on success.
int refgpu_set_keyswitch(int L, int K, int dnum, const uint64_t* hat_inv, const uint64_t* hat_mod,
                         const uint64_t* phat_inv, const uint64_t* phat_mod) {
    if (!g.dglob || L < 1 || K < 1 || L + K != g.np || dnum < 1 || dnum > MAXD || !hat_inv || !hat_mod ||
        !phat_inv || !phat_mod)
        return 1;
    const int alpha = (L + dnum - 1) / dnum;
    if ((L + alpha - 1) / alpha != dnum) return 1;  // every digit non-empty
    const int NP = L + K;
    cudaDeviceSynchronize();
    for (auto& kv : g.ptr_tables) cudaFree(kv.second);  // tables built from the previous lists
    g.ptr_tables.clear();
    hc.L = L;
    hc.K = K;
    hc.dnum = dnum;
    memset(hc.primeid_flattened, 0, sizeof(hc.primeid_flattened));
    memset(hc.num_primeid_digit_from, 0, sizeof(hc.num_primeid_digit_from));
    memset(hc.num_primeid_digit_to, 0, sizeof(hc.num_primeid_digit_to));
    memset(hc.pos_in_digit, 0, sizeof(hc.pos_in_digit));
    for (int t = 0; t < MAXP; ++t) hc.primeid_digit[t] = -1;  // special primes belong to no digit
    for (int q = 0; q < L; ++q) {
        hc.primeid_partition[0][q] = q;
        hc.primeid_digit[q] = q / alpha;
        uint64_t P = 1;  // the special primes' product mod q
        for (int k = 0; k < K; ++k) P = mulmod(P, hc.primes[L + k] % hc.primes[q], hc.primes[q]);
        hc.P[q] = P;
        hc.P_shoup[q] = shoup(P, hc.primes[q]);
    }
    for (int k = 0; k < K; ++k) hc.primeid_special_partition[k] = L + k;
    for (int d = 0; d < dnum; ++d) {
        const int lo = d * alpha, hi = (lo + alpha < L ? lo + alpha : L) - 1;
        for (int i = lo; i <= hi; ++i) {
            hc.primeid_digit_from[d][i - lo] = i;
            hc.pos_in_digit[d][i] = i - lo;
        }
        // the digit's targets: the special primes, then the ciphertext
        // primes outside the digit (src/CKKS/Context.cu generateDigitMeta)
        int num = 0;
        for (int k = 0; k < K; ++k) {
            hc.primeid_digit_to[d][num] = L + k;
            hc.pos_in_digit[d][L + k] = num++;
        }
        for (int q = 0; q < L; ++q)
            if (q < lo || q > hi) {
                hc.primeid_digit_to[d][num] = q;
                hc.pos_in_digit[d][q] = num++;
            }
        for (int l = 0; l < L; ++l) {
            int nf = 0, nt = K;
            for (int i = lo; i <= hi; ++i) nf += i <= l;
            for (int q = 0; q < L; ++q) nt += (q < lo || q > hi) && q <= l;
            hc.num_primeid_digit_from[d][l] = nf;
            hc.num_primeid_digit_to[d][l] = nt;
        }
    }
    memset(hg.DecompAndModUp_pre_scale, 0, sizeof(hg.DecompAndModUp_pre_scale));
    memset(hg.DecompAndModUp_pre_scale_shoup, 0, sizeof(hg.DecompAndModUp_pre_scale_shoup));
    memset(hg.DecompAndModUp_matrix, 0, sizeof(hg.DecompAndModUp_matrix));
    memset(hg.DecompAndModUp_matrix_shoup, 0, sizeof(hg.DecompAndModUp_matrix_shoup));
    for (int d = 0; d < dnum; ++d) {
        const int lo = d * alpha, hi = (lo + alpha < L ? lo + alpha : L) - 1;
        for (int l = lo; l < L; ++l) {
            const int cnt = (l < hi ? l : hi) - lo + 1;  // digit primes at level l
            for (int i = 0; i < cnt; ++i) {
                const int pid = lo + i;
                const size_t src = ((size_t)d * L + l) * alpha + i;
                // PartQlHatInvModq[d][cnt - 1][i] at [d][cnt - 1][pid]
                const uint64_t v = hat_inv[src];
                hg.DecompAndModUp_pre_scale[MODUPIDX_SCALE(d, cnt - 1, pid)] = v;
                hg.DecompAndModUp_pre_scale_shoup[MODUPIDX_SCALE(d, cnt - 1, pid)] = shoup(v, hc.primes[pid]);
                for (int t = 0; t < NP; ++t) {
                    const uint64_t m = hat_mod[src * NP + t];
                    hg.DecompAndModUp_matrix[MODUPIDX_MATRIX(l, d, pid, t)] = m;
                    hg.DecompAndModUp_matrix_shoup[MODUPIDX_MATRIX(l, d, pid, t)] = shoup(m, hc.primes[t]);
                }
            }
        }
    }
    memset(hg.ModDown_pre_scale, 0, sizeof(hg.ModDown_pre_scale));
    memset(hg.ModDown_pre_scale_shoup, 0, sizeof(hg.ModDown_pre_scale_shoup));
    memset(hg.ModDown_matrix, 0, sizeof(hg.ModDown_matrix));
    memset(hg.ModDown_matrix_shoup, 0, sizeof(hg.ModDown_matrix_shoup));
    for (int k = 0; k < K; ++k) {
        hg.ModDown_pre_scale[L + k] = phat_inv[k];
        hg.ModDown_pre_scale_shoup[L + k] = shoup(phat_inv[k], hc.primes[L + k]);
        for (int j = 0; j < L; ++j) {
            hg.ModDown_matrix[MODDOWN_MATRIX(k, j)] = phat_mod[(size_t)k * L + j];
            hg.ModDown_matrix_shoup[MODDOWN_MATRIX(k, j)] = shoup(phat_mod[(size_t)k * L + j], hc.primes[j]);
        }
    }
    g.L = L;
    g.K = K;
    g.dnum = dnum;
    g.alpha = alpha;
    return upload_constants();
}

// ModUp base conversion of digit d at `level` (coefficient domain):
// x = the level + 1 limbs of the polynomial ([level + 1][N]); out receives
// the digit's targets in its list order, the K special primes then the
// ciphertext primes <= level outside the digit ([K + level + 1 - cnt][N]).
int refgpu_modup_conv(const uint64_t* x, uint64_t* out, int level, int d, void* stream) {
    if (!g.L || !x || !out || level < 0 || level >= g.L || d < 0 || d >= g.dnum) return 1;
    const int lo = d * g.alpha;
    if (lo > level) return 1;  // the digit has no prime at this level
    const int nf = hc.num_primeid_digit_from[d][level], nt = hc.num_primeid_digit_to[d][level];
    cudaStream_t st = (cudaStream_t)stream;
    void** ptrs = ptr_table({"modup", x, out, (const void*)(size_t)level, (const void*)(size_t)d}, (size_t)nf + nt,
                            st, [&](std::vector<void*>& h, void**) {
                                for (int i = 0; i < nf; ++i) h[i] = (void*)(x + (size_t)(lo + i) * g.N);
                                for (int j = 0; j < nt; ++j) h[nf + j] = out + (size_t)j * g.N;
                            });
    if (!ptrs) return 2;
    const dim3 block{64, 2};
    const dim3 grid{(uint32_t)g.N / block.x};
    const int shared = (int)sizeof(uint64_t) * nf * (int)block.x;
    CKKS::DecompAndModUpConv<ALGO_SHOUP><<<grid, block, shared, st>>>(ptrs, level + 1, ptrs + nf, d, g.dglob);
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

// ModDown base conversion (coefficient domain): y = the K special limbs
// ([K][N]); out receives the level + 1 ciphertext limbs ([level + 1][N]).
int refgpu_moddown_conv(const uint64_t* y, uint64_t* out, int level, void* stream) {
    if (!g.L || !y || !out || level < 0 || level >= g.L) return 1;
    const int n = level + 1, K = g.K;
    cudaStream_t st = (cudaStream_t)stream;
    void** ptrs = ptr_table({"moddown", y, out, (const void*)(size_t)level}, (size_t)n + K, st,
                            [&](std::vector<void*>& h, void**) {
                                for (int j = 0; j < n; ++j) h[j] = out + (size_t)j * g.N;
                                for (int k = 0; k < K; ++k) h[n + k] = (void*)(y + (size_t)k * g.N);
                            });
    if (!ptrs) return 2;
    const dim3 block{64, 2};
    const dim3 grid{(uint32_t)g.N / block.x};
    const int shared = (int)sizeof(uint64_t) * K * (int)block.x;
    CKKS::ModDown2<ALGO_SHOUP><<<grid, block, shared, st>>>(ptrs, n, ptrs + n, PARTITION(0, 0), g.dglob);
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

// Key-switch inner product at the top level (level L - 1), fusedDotKSK_2_:
// dig = ModUp outputs [dnum][K + L - cnt_d][N] per digit in its list order
// (digit d's block starts at dig + d * (K + L) * N), x = the key-switched
// polynomial's own limbs [L][N] (evaluation form), ksk_b / ksk_a = the key
// halves [dnum][L + K][N]; out_b / out_a ([L + K][N], ciphertext primes then
// special primes) receive sum_d D_d * ksk_b[d] and sum_d D_d * ksk_a[d].
int refgpu_dot(const uint64_t* dig, const uint64_t* x, const uint64_t* ksk_b, const uint64_t* ksk_a,
               uint64_t* out_b, uint64_t* out_a, void* stream) {
    if (!g.L || !dig || !x || !ksk_b || !ksk_a || !out_b || !out_a) return 1;
    const int L = g.L, K = g.K, D = g.dnum, NP = L + K;
    const size_t N = g.N;
    cudaStream_t st = (cudaStream_t)stream;
    // 6 dnum pointer tables of NP entries each, then out1, sout1, out2, sout2
    // and the table of the 6 dnum table pointers
    const size_t ntab = 6 * (size_t)D;
    const size_t o = ntab * NP;
    void** ptrs = ptr_table({"dot", dig, x, ksk_b, ksk_a, out_b, out_a}, o + 2 * (size_t)NP + ntab, st,
                            [&](std::vector<void*>& h, void** base) {
        for (int i = 0; i < D; ++i) {
            const int lo = i * g.alpha, hi = (lo + g.alpha < L ? lo + g.alpha : L) - 1;
            const int nt = K + L - (hi - lo + 1);
            for (int pos = 0; pos < nt; ++pos) {
                const int t = hc.primeid_digit_to[i][pos];
                h[(size_t)i * NP + pos] = (void*)(dig + ((size_t)i * NP + pos) * N);            // digit values
                h[(size_t)(D + i) * NP + pos] = (void*)(ksk_a + ((size_t)i * NP + t) * N);      // kska
                h[(size_t)(2 * D + i) * NP + pos] = (void*)(ksk_b + ((size_t)i * NP + t) * N);  // kskb
            }
            for (int q = 0; q < L; ++q) {
                h[(size_t)(3 * D + i) * NP + q] = (void*)(x + (size_t)q * N);  // own limbs
                h[(size_t)(4 * D + i) * NP + q] = (void*)(ksk_a + ((size_t)i * NP + q) * N);
                h[(size_t)(5 * D + i) * NP + q] = (void*)(ksk_b + ((size_t)i * NP + q) * N);
            }
        }
        for (int q = 0; q < L; ++q) {
            h[o + q] = out_a + (size_t)q * N;       // out1
            h[o + NP + q] = out_b + (size_t)q * N;  // out2
        }
        for (int k = 0; k < K; ++k) {
            h[o + L + k] = out_a + (size_t)(L + k) * N;       // sout1
            h[o + NP + L + k] = out_b + (size_t)(L + k) * N;  // sout2
        }
        for (size_t k = 0; k < ntab; ++k) h[o + 2 * NP + k] = (void*)(base + k * NP);
    });
    if (!ptrs) return 2;
    void** out1 = ptrs + o;
    void** sout1 = ptrs + o + L;
    void** out2 = ptrs + o + NP;
    void** sout2 = ptrs + o + NP + L;
    void*** tabs = (void***)(ptrs + o + 2 * NP);
    CKKS::fusedDotKSK_2_<<<dim3{(uint32_t)N / 128, (uint32_t)(K + L)}, 128, 0, st>>>(out1, sout1, out2, sout2, tabs,
                                                                                   D, 0, K, 0);
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

// Tensor product over nlimbs limbs (limb k: prime k; at most L once the
// key-switch lists are set), binomialMult_ in place: c0 <- c0 d0,
// c1 <- c0 d1 + c1 d0, c2 <- c1 d1.
int refgpu_binomial(uint64_t* c0, uint64_t* c1, uint64_t* c2, const uint64_t* d0, const uint64_t* d1, int nlimbs,
                    void* stream) {
    if (!g.dglob || !c0 || !c1 || !c2 || !d0 || !d1 || nlimbs < 1 || nlimbs > (g.L ? g.L : g.np)) return 1;
    const size_t N = g.N;
    cudaStream_t st = (cudaStream_t)stream;
    void** ptrs = ptr_table({"binomial", c0, c1, c2, d0, d1, (const void*)(size_t)nlimbs}, 5 * (size_t)nlimbs, st,
                            [&](std::vector<void*>& h, void**) {
                                for (int k = 0; k < nlimbs; ++k) {
                                    h[k] = c0 + k * N;
                                    h[nlimbs + k] = c1 + k * N;
                                    h[2 * nlimbs + k] = c2 + k * N;
                                    h[3 * nlimbs + k] = (void*)(d0 + k * N);
                                    h[4 * nlimbs + k] = (void*)(d1 + k * N);
                                }
                            });
    if (!ptrs) return 2;
    CKKS::binomialMult_<<<dim3{(uint32_t)N / 128, (uint32_t)nlimbs}, 128, 0, st>>>(
        0, ptrs, ptrs + nlimbs, ptrs + 2 * nlimbs, ptrs + 3 * nlimbs, ptrs + 4 * nlimbs);
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

// Automorphism X -> X^k of nlimbs limbs (evaluation form), automorph_multi_:
// out[slot(k, j)] = a[j] per limb.
int refgpu_automorph(const uint64_t* a, uint64_t* out, int nlimbs, int k, void* stream) {
    if (!g.dglob || !a || !out || nlimbs < 1 || nlimbs > (g.L ? g.L : g.np) || !(k & 1) || k >= 2 * g.N) return 1;
    const size_t N = g.N;
    cudaStream_t st = (cudaStream_t)stream;
    void** ptrs = ptr_table({"automorph", a, out, (const void*)(size_t)nlimbs}, 2 * (size_t)nlimbs, st,
                            [&](std::vector<void*>& h, void**) {
                                for (int l = 0; l < nlimbs; ++l) {
                                    h[l] = (void*)(a + l * N);
                                    h[nlimbs + l] = out + l * N;
                                }
                            });
    if (!ptrs) return 2;
    CKKS::automorph_multi_<<<dim3{(uint32_t)N / 128, (uint32_t)nlimbs}, 128, 0, st>>>(ptrs, ptrs + nlimbs, k, 1, 0);
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

// Hoisted rotations' inner product at the top level, hoistedRotateDotKSK_2_:
// for rotation r (Galois element galois[r]) and output slot j,
//   out_b[r][slot(g, j)] = sum_d D_d[j] kb[r][d][j] (+ P c0[j] on the
//   ciphertext primes),  out_a[r][slot(g, j)] = sum_d D_d[j] ka[r][d][j];
// dig and x as for refgpu_dot, c0 = [L][N]; kb[r], ka[r] point to keys
// [dnum][L + K][N] in the plain layout; out_b[r], out_a[r] to [L + K][N]
// (ciphertext primes then special primes).  1 <= n <= 64.
int refgpu_hoisted_dot(const uint64_t* dig, const uint64_t* x, const uint64_t* c0, int n,
                       const uint64_t* const* kb, const uint64_t* const* ka, const int32_t* galois,
                       uint64_t* const* out_b, uint64_t* const* out_a, void* stream) {
    if (!g.L || !dig || !x || !c0 || n < 1 || n > 64 || !kb || !ka || !galois || !out_b || !out_a) return 1;
    for (int r = 0; r < n; ++r)
        if (!kb[r] || !ka[r] || !out_b[r] || !out_a[r] || !(galois[r] & 1) || galois[r] >= 2 * g.N) return 1;
    const int L = g.L, K = g.K, D = g.dnum, NP = L + K;
    const size_t N = g.N;
    cudaStream_t st = (cudaStream_t)stream;
    // layout (pointer slots): din1 tables [4 D][NP] | c0 [L] | out1, sout1,
    // out2, sout2 tables [n][L] / [n][K] | key tables [n][6 D][NP] |
    // table-of-tables: din1 [4 D], out1 [n], sout1 [n], out2 [n], sout2 [n],
    // keys [n 6 D] | galois as ints [n]
    const size_t o_din = 0, o_c0 = o_din + 4 * (size_t)D * NP, o_out = o_c0 + L;
    const size_t o_key = o_out + (size_t)n * (2 * L + 2 * K);
    const size_t o_tt = o_key + (size_t)n * 6 * D * NP;
    const size_t o_tt_din = o_tt, o_tt_o1 = o_tt_din + 4 * D, o_tt_s1 = o_tt_o1 + n, o_tt_o2 = o_tt_s1 + n,
                 o_tt_s2 = o_tt_o2 + n, o_tt_key = o_tt_s2 + n, o_idx = o_tt_key + (size_t)n * 6 * D;
    const size_t total = o_idx + ((size_t)n + 1) / 2;
    std::vector<const void*> key{"hoisted", dig, x, c0, (const void*)(size_t)n};
    for (int r = 0; r < n; ++r) {
        key.push_back(kb[r]);
        key.push_back(ka[r]);
        key.push_back(out_b[r]);
        key.push_back(out_a[r]);
        key.push_back((const void*)(size_t)galois[r]);
    }
    void** ptrs = ptr_table(key, total, st, [&](std::vector<void*>& h, void** base) {
        for (int i = 0; i < D; ++i) {
            const int lo = i * g.alpha, hi = (lo + g.alpha < L ? lo + g.alpha : L) - 1;
            const int nt = K + L - (hi - lo + 1);
            for (int pos = 0; pos < nt; ++pos) h[o_din + (size_t)i * NP + pos] = (void*)(dig + ((size_t)i * NP + pos) * N);
            for (int q = 0; q < L; ++q) h[o_din + (size_t)(3 * D + i) * NP + q] = (void*)(x + (size_t)q * N);
        }
        for (int q = 0; q < L; ++q) h[o_c0 + q] = (void*)(c0 + (size_t)q * N);
        for (int r = 0; r < n; ++r) {
            const size_t b1 = o_out + (size_t)r * (2 * L + 2 * K);  // out1 [L], sout1 [K], out2 [L], sout2 [K]
            for (int q = 0; q < L; ++q) {
                h[b1 + q] = out_a[r] + (size_t)q * N;
                h[b1 + L + K + q] = out_b[r] + (size_t)q * N;
            }
            for (int k = 0; k < K; ++k) {
                h[b1 + L + k] = out_a[r] + (size_t)(L + k) * N;
                h[b1 + 2 * L + K + k] = out_b[r] + (size_t)(L + k) * N;
            }
            h[o_tt_o1 + r] = (void*)(base + b1);
            h[o_tt_s1 + r] = (void*)(base + b1 + L);
            h[o_tt_o2 + r] = (void*)(base + b1 + L + K);
            h[o_tt_s2 + r] = (void*)(base + b1 + 2 * L + K);
            for (int i = 0; i < D; ++i) {
                const int lo = i * g.alpha, hi = (lo + g.alpha < L ? lo + g.alpha : L) - 1;
                const int nt = K + L - (hi - lo + 1);
                const size_t kt = o_key + ((size_t)r * 6 * D) * NP;
                for (int pos = 0; pos < nt; ++pos) {
                    const int t = hc.primeid_digit_to[i][pos];
                    h[kt + (size_t)(D + i) * NP + pos] = (void*)(ka[r] + ((size_t)i * NP + t) * N);
                    h[kt + (size_t)(2 * D + i) * NP + pos] = (void*)(kb[r] + ((size_t)i * NP + t) * N);
                }
                for (int q = 0; q < L; ++q) {
                    h[kt + (size_t)(4 * D + i) * NP + q] = (void*)(ka[r] + ((size_t)i * NP + q) * N);
                    h[kt + (size_t)(5 * D + i) * NP + q] = (void*)(kb[r] + ((size_t)i * NP + q) * N);
                }
            }
            for (int t6 = 0; t6 < 6 * D; ++t6)
                h[o_tt_key + (size_t)r * 6 * D + t6] = (void*)(base + o_key + ((size_t)r * 6 * D + t6) * NP);
        }
        for (int t4 = 0; t4 < 4 * D; ++t4) h[o_tt_din + t4] = (void*)(base + o_din + (size_t)t4 * NP);
        int32_t* idx = reinterpret_cast<int32_t*>(h.data() + o_idx);
        for (int r = 0; r < n; ++r) idx[r] = galois[r];
    });
    if (!ptrs) return 2;
    CKKS::hoistedRotateDotKSK_2_<<<dim3{(uint32_t)N / 128, (uint32_t)(K + L)}, 128, sizeof(uint64_t) * 128 * D, st>>>(
        (void***)(ptrs + o_tt_din), ptrs + o_c0, (void***)(ptrs + o_tt_o1), (void***)(ptrs + o_tt_s1),
        (void***)(ptrs + o_tt_o2), (void***)(ptrs + o_tt_s2), n, (const int*)(ptrs + o_idx),
        (void***)(ptrs + o_tt_key), D, 0, K, 0, nullptr, false);
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

void refgpu_release(void) { release(); }

}  // extern "C"
