// serve.cpp -- continuous-batching request loop over one context.
//
// Requests (HMult+Relin+Rescale, Rotate, Bootstrap) are queued by any
// thread.  A scheduler thread keeps forming batches from whatever is pending
// -- HMult / Rotate grouped by operation and level, up to max_batch per
// batch -- and launches each batch on the next free stream; every stream owns
// a key-switch workspace, so a batch admitted while others are still running
// overlaps them on the device.  Bootstraps run on their own lane (the
// context stream and workspaces), beside the batches, up to
// min(max_batch, kBootBatch) per batched EvalBootstrap call.  Admission is
// against a fixed HBM budget: the workspaces are
// charged once at start-up, and every admitted request reserves its output
// buffer until the request completes.  Completion is detected with one CUDA
// event per batch; the caller waits on a request id.  Ciphertexts and keys
// stay device-resident; the per-request latency (submit -> completion seen
// by the scheduler) feeds the p50 / p99 statistics.
//
// No counterpart in the reference (FIDESlib has no serving layer); each
// batch is the same engine call as fides_hmult_batch / fides_rotate_batch,
// so a result is bit-identical whether the request ran alone or in a mix.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

#include "context.hpp"

using namespace fides;
using clk = std::chrono::steady_clock;

// bootstraps batched together at most.  One: a batched EvalBootstrap of 2
// (4) ciphertexts at N = 2^16 runs 59.6 (115.3) ms against 31.4 ms for one,
// so batching gains 5-8% throughput while every member waits for the whole
// batch; with up to 4 per batch the p99 of the mix with 10% bootstraps at
// 70% of the lane's capacity measured 735 ms against 126 ms one at a time.
constexpr int kBootBatch = 1;

namespace {

struct Request {
    uint64_t id = 0;
    int op = 0;
    const fides_ct* a = nullptr;
    const fides_ct* b = nullptr;
    int32_t index = 0;
    fides_ct* out = nullptr;
    int level = 0;
    size_t bytes = 0;  // reserved output bytes
    clk::time_point t_submit, t_start, t_done;
    fides_status status = FIDES_OK;
    bool done = false;
};

struct Lane {
    cudaStream_t st = nullptr;
    Workspace ws;
    cudaEvent_t ev = nullptr;
    std::vector<Request*> batch;
    bool busy = false;
};

bool is_boot(const Request* r) { return r->op == FIDES_OP_BOOTSTRAP; }

}  // namespace

struct fides_server {
    fides_ctx* c = nullptr;
    size_t budget = 0, reserved = 0, ws_bytes = 0;
    int max_batch = 16;
    std::vector<Lane> lanes;
    Lane boot;                // bootstrap lane: context stream, one request at a time
    size_t boot_scratch = 0;  // HBM charged per bootstrap besides its output
    std::mutex mu;
    std::condition_variable cv_sched, cv_done;
    std::deque<Request*> pending;
    std::unordered_map<uint64_t, Request*> all;
    uint64_t next_id = 1;
    bool stop = false;
    std::thread th;
    std::vector<double> lat_ms, queue_ms;
    uint64_t completed = 0, batches = 0;
    clk::time_point t_first, t_last;
};

namespace {

size_t out_bytes(const fides_ctx* c, int level) { return 2 * (size_t)(level + 1) * c->limb_bytes(); }

// Launch one batch of same-op, same-level requests on a lane.  A request
// whose output cannot be allocated fails alone; the rest of the batch runs.
void launch_batch(fides_server* s, Lane& ln) {
    fides_ctx* c = s->c;
    const int N = c->N;
    const int op = ln.batch[0]->op;
    const int level = ln.batch[0]->level;
    if (op == FIDES_OP_BOOTSTRAP) {
        // the batch's bootstraps together (one batched EvalMod, batched
        // giant-step rotations), queued on the context stream by the
        // host-side orchestration
        std::vector<const fides_ct*> in;
        std::vector<fides_ct*> outs;
        for (Request* r : ln.batch) {
            r->t_start = clk::now();
            in.push_back(r->a);
            outs.push_back(r->out);
        }
        const fides_status st = fides_bootstrap_batch(c, (int)in.size(), in.data(), outs.data());
        for (Request* r : ln.batch) r->status = st;
        cudaEventRecord(ln.ev, ln.st);
        ln.busy = true;
        return;
    }
    std::vector<Request*> b;
    for (Request* r : ln.batch) {
        r->t_start = clk::now();
        const int out_level = (op == FIDES_OP_HMULT && level > 0) ? level - 1 : level;
        if (ct_reserve(c, r->out, out_level, ln.st) != FIDES_OK) {
            r->status = FIDES_OOM;
            continue;
        }
        b.push_back(r);
    }
    const int nb = (int)b.size();
    std::vector<uint64_t*> o0(nb), o1(nb);
    for (int j = 0; j < nb; ++j) {
        o0[j] = b[j]->out->c0();
        o1[j] = b[j]->out->c1(N);
    }
    if (nb > 0 && op == FIDES_OP_HMULT) {
        std::vector<const uint64_t*> a0(nb), a1(nb), b0(nb), b1(nb);
        for (int j = 0; j < nb; ++j) {
            a0[j] = b[j]->a->c0();
            a1[j] = b[j]->a->c1(N);
            b0[j] = b[j]->b->c0();
            b1[j] = b[j]->b->c1(N);
        }
        eng_hmult(c, ln.ws, level, nb, a0.data(), a1.data(), b0.data(), b1.data(), o0.data(), o1.data(), level > 0,
                  c->relin);
    } else if (nb > 0) {
        std::vector<const uint64_t*> c0(nb), c1(nb);
        std::vector<const SwitchKey*> keys(nb);
        std::vector<uint32_t> gal(nb);
        for (int j = 0; j < nb; ++j) {
            c0[j] = b[j]->a->c0();
            c1[j] = b[j]->a->c1(N);
            gal[j] = fides_rotation_galois(c, b[j]->index, b[j]->a->slots > 0 ? b[j]->a->slots : N / 2);
            keys[j] = &c->galois_keys.at(gal[j]);
        }
        eng_rotate(c, ln.ws, level, nb, c0.data(), c1.data(), keys.data(), gal.data(), o0.data(), o1.data(), false);
    }
    cudaEventRecord(ln.ev, ln.st);
    ln.busy = true;
}

void finish_lane(fides_server* s, Lane& ln, clk::time_point now, cudaError_t q) {
    const cudaError_t e = cudaGetLastError();
    // a kernel that gave up a bounded wait flags the context's error word:
    // the batch that completes next fails with FIDES_TIMEOUT
    const uint32_t dev_err = (e == cudaSuccess && q == cudaSuccess) ? read_device_error(s->c, ln.st, true) : 0;
    for (Request* r : ln.batch) {
        if (e != cudaSuccess || q != cudaSuccess) r->status = FIDES_CUDA_ERR;
        else if (dev_err && r->status == FIDES_OK) r->status = FIDES_TIMEOUT;
        const fides_ct* a = r->a;
        if (r->status != FIDES_OK || r->op == FIDES_OP_BOOTSTRAP) {
            // failed, or metadata set by fides_bootstrap
        } else if (r->op == FIDES_OP_HMULT) {
            const bool rs = r->level > 0;
            const double sc = a->scale * r->b->scale;
            r->out->level = rs ? r->level - 1 : r->level;
            r->out->scale = rs ? sc / (double)s->c->host.prime[r->level] : sc;
            r->out->noise_deg = a->noise_deg + r->b->noise_deg - (rs ? 1 : 0);
            r->out->slots = std::max(a->slots, r->b->slots);
        } else {
            r->out->level = a->level;
            r->out->scale = a->scale;
            r->out->noise_deg = a->noise_deg;
            r->out->slots = a->slots;
        }
        r->t_done = now;
        r->done = true;
        s->reserved -= r->bytes;
        s->lat_ms.push_back(std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count());
        s->queue_ms.push_back(std::chrono::duration<double, std::milli>(r->t_start - r->t_submit).count());
        s->completed++;
        s->t_last = now;
    }
    ln.batch.clear();
    ln.busy = false;
}

void scheduler(fides_server* s) {
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        // retire finished batches
        bool any_busy = false;
        auto retire = [&](Lane& ln) {
            if (!ln.busy) return;
            const cudaError_t q = cudaEventQuery(ln.ev);
            if (q != cudaErrorNotReady) {  // done, or failed: either way the batch ends here
                finish_lane(s, ln, clk::now(), q);
                s->cv_done.notify_all();
            } else {
                any_busy = true;
            }
        };
        for (auto& ln : s->lanes) retire(ln);
        retire(s->boot);
        if (s->stop && s->pending.empty() && !any_busy) break;
        // admit: form one batch per free lane from the head of the queue
        for (auto& ln : s->lanes) {
            if (ln.busy || s->pending.empty()) continue;
            auto hit = std::find_if(s->pending.begin(), s->pending.end(), [](Request* r) { return !is_boot(r); });
            if (hit == s->pending.end()) break;
            Request* head = *hit;
            std::vector<Request*> pick;
            size_t need = 0;
            for (auto it = hit; it != s->pending.end() && (int)pick.size() < s->max_batch;) {
                Request* r = *it;
                if (r->op == head->op && r->level == head->level && s->reserved + need + r->bytes <= s->budget) {
                    need += r->bytes;
                    pick.push_back(r);
                    it = s->pending.erase(it);
                } else {
                    ++it;
                }
            }
            if (pick.empty()) break;  // budget exhausted: wait for completions
            s->reserved += need;
            ln.batch = std::move(pick);
            s->batches++;
            // submitters are not held up while the batch is queued
            lk.unlock();
            {
                std::lock_guard<std::recursive_mutex> g(s->c->mu);
                cudaSetDevice(s->c->device);
                launch_batch(s, ln);
            }
            lk.lock();
            any_busy = true;
        }
        // the oldest bootstraps, up to max_batch with the same slot count,
        // when their lane is free and the budget allows
        if (!s->boot.busy) {
            auto hit = std::find_if(s->pending.begin(), s->pending.end(), [](Request* r) { return is_boot(r); });
            if (hit != s->pending.end() && s->reserved + (*hit)->bytes <= s->budget) {
                const int slots = (*hit)->a->slots;
                std::vector<Request*> pick;
                size_t need = 0;
                const int cap = std::min(s->max_batch, kBootBatch);
                for (auto it = hit; it != s->pending.end() && (int)pick.size() < cap;) {
                    Request* r = *it;
                    if (is_boot(r) && r->a->slots == slots && s->reserved + need + r->bytes <= s->budget) {
                        need += r->bytes;
                        pick.push_back(r);
                        it = s->pending.erase(it);
                    } else {
                        ++it;
                    }
                }
                s->reserved += need;
                s->boot.batch = std::move(pick);
                s->batches++;
                lk.unlock();
                {
                    std::lock_guard<std::recursive_mutex> g(s->c->mu);
                    cudaSetDevice(s->c->device);
                    launch_batch(s, s->boot);
                }
                lk.lock();
                any_busy = true;
            }
        }
        if (any_busy) {
            s->cv_sched.wait_for(lk, std::chrono::microseconds(50));
        } else {
            s->cv_sched.wait_for(lk, std::chrono::milliseconds(5));
        }
    }
}

}  // namespace

extern "C" {

fides_status fides_srv_create(fides_ctx* c, size_t hbm_budget, int max_batch, int num_streams, fides_server** out) {
    if (!c || !out || max_batch < 1 || max_batch > kMaxBatch || num_streams < 1 || num_streams > 8)
        return FIDES_BAD_ARG;
    *out = nullptr;
    std::lock_guard<std::recursive_mutex> g(c->mu);
    cudaSetDevice(c->device);
    if (!c->has_relin) return set_err(c, FIDES_KEY_MISSING, "serving needs the relinearisation key");
    auto* s = new (std::nothrow) fides_server();
    if (!s) return FIDES_OOM;
    s->c = c;
    s->budget = hbm_budget;
    s->max_batch = max_batch;
    s->lanes.resize(num_streams);
    for (auto& ln : s->lanes) {
        cudaStreamCreateWithFlags(&ln.st, cudaStreamNonBlocking);
        cudaEventCreateWithFlags(&ln.ev, cudaEventDisableTiming);
        ln.ws.st = ln.st;
        fides_status st = ws_reserve(c, ln.ws, max_batch);
        if (st != FIDES_OK) {
            fides_srv_destroy(s);
            return st;
        }
        s->ws_bytes += ln.ws.stride * 8 * (size_t)ln.ws.cap;
    }
    if (s->ws_bytes >= s->budget) {
        fides_srv_destroy(s);
        return set_err(c, FIDES_OOM, "HBM budget smaller than the serving workspaces");
    }
    s->reserved = s->ws_bytes;
    s->boot.st = c->st;
    cudaEventCreateWithFlags(&s->boot.ev, cudaEventDisableTiming);
    // a bootstrap holds about 64 top-level ciphertexts of intermediates
    s->boot_scratch = 64 * out_bytes(c, c->L - 1);
    s->th = std::thread(scheduler, s);
    *out = s;
    return FIDES_OK;
}

fides_status fides_srv_submit(fides_server* s, int op, const fides_ct* a, const fides_ct* b, int32_t index,
                              fides_ct* out, uint64_t* request_id) {
    if (!s || !a || !out || !request_id || !a->buf) return FIDES_BAD_ARG;
    fides_ctx* c = s->c;
    if (op == FIDES_OP_HMULT) {
        if (!b || !b->buf || b->level != a->level) return FIDES_BAD_ARG;
    } else if (op == FIDES_OP_ROTATE) {
        std::lock_guard<std::recursive_mutex> g(c->mu);
        const uint32_t gal = fides_rotation_galois(c, index, a->slots > 0 ? a->slots : c->N / 2);
        if (gal == 1 || !c->galois_keys.count(gal)) return set_err(c, FIDES_KEY_MISSING, "no rotation key");
    } else if (op == FIDES_OP_BOOTSTRAP) {
        std::lock_guard<std::recursive_mutex> g(c->mu);
        if (!c->boot.count(a->slots > 0 ? a->slots : c->N / 2))
            return set_err(c, FIDES_BAD_ARG, "bootstrapping not set up for these slots");
    } else {
        return FIDES_UNSUPPORTED;
    }
    auto* r = new (std::nothrow) Request();
    if (!r) return FIDES_OOM;
    r->op = op;
    r->a = a;
    r->b = b;
    r->index = index;
    r->out = out;
    r->level = a->level;
    r->bytes = op == FIDES_OP_BOOTSTRAP ? out_bytes(c, c->L - 1) + s->boot_scratch : out_bytes(c, a->level);
    std::lock_guard<std::mutex> lk(s->mu);
    if (r->bytes + s->ws_bytes > s->budget) {
        delete r;
        return set_err(c, FIDES_OOM, "request larger than the serving HBM budget");
    }
    r->id = s->next_id++;
    r->t_submit = clk::now();
    if (s->completed == 0 && s->all.empty()) s->t_first = r->t_submit;
    s->all[r->id] = r;
    s->pending.push_back(r);
    *request_id = r->id;
    s->cv_sched.notify_one();
    return FIDES_OK;
}

fides_status fides_srv_wait(fides_server* s, uint64_t request_id, double timeout_s) {
    if (!s) return FIDES_BAD_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(request_id);
    if (it == s->all.end()) return FIDES_BAD_ARG;
    Request* r = it->second;
    const auto deadline = clk::now() + std::chrono::duration<double>(timeout_s);
    while (!r->done) {
        if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && !r->done) return FIDES_TIMEOUT;
    }
    const fides_status st = r->status;
    s->all.erase(it);
    delete r;
    return st;
}

fides_status fides_srv_stats(fides_server* s, fides_srv_stats_t* out) {
    if (!s || !out) return FIDES_BAD_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto pct = [](std::vector<double> v, double q) {
        if (v.empty()) return 0.0;
        std::sort(v.begin(), v.end());
        return v[std::min(v.size() - 1, (size_t)(q * (v.size() - 1) + 0.5))];
    };
    out->completed = s->completed;
    out->batches = s->batches;
    out->p50_ms = pct(s->lat_ms, 0.50);
    out->p99_ms = pct(s->lat_ms, 0.99);
    out->mean_queue_ms = 0;
    for (double q : s->queue_ms) out->mean_queue_ms += q;
    if (!s->queue_ms.empty()) out->mean_queue_ms /= (double)s->queue_ms.size();
    const double span = std::chrono::duration<double>(s->t_last - s->t_first).count();
    out->throughput = span > 0 ? (double)s->completed / span : 0.0;
    out->reserved_bytes = s->reserved;
    return FIDES_OK;
}

fides_status fides_srv_reset_stats(fides_server* s) {
    if (!s) return FIDES_BAD_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    s->lat_ms.clear();
    s->queue_ms.clear();
    s->completed = 0;
    s->batches = 0;
    s->t_first = s->t_last = clk::now();
    return FIDES_OK;
}

fides_status fides_srv_destroy(fides_server* s) {
    if (!s) return FIDES_BAD_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_sched.notify_all();
    if (s->th.joinable()) s->th.join();
    cudaSetDevice(s->c->device);
    for (auto& ln : s->lanes) {
        if (ln.st) cudaStreamSynchronize(ln.st);
        ws_free(ln.ws);
        if (ln.ev) cudaEventDestroy(ln.ev);
        if (ln.st) cudaStreamDestroy(ln.st);
    }
    if (s->boot.st) cudaStreamSynchronize(s->boot.st);  // the context's stream: not destroyed here
    if (s->boot.ev) cudaEventDestroy(s->boot.ev);
    for (auto& kv : s->all) delete kv.second;
    delete s;
    return FIDES_OK;
}

}  // extern "C"
