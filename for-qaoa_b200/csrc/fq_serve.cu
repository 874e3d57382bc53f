// fq_serve.cu -- continuous batching of QAOA energy+gradient requests.
//
// Requests are admitted as resources free up and their work overlaps on the
// GPU; a scheduler thread runs the small-instance batches and every lane has
// a thread of its own, so the ~30 kernel launches of a larger request are
// issued by its lane's thread, in parallel with the other lanes':
//   - small instances (N <= 15) are packed into launches of k_small_jobs,
//     the whole instance in shared memory: one CTA each up to 12 qubits, a
//     cluster of 2^(N-12) CTAs above (distributed shared memory), one launch
//     per size class; two batches can be in flight on their own streams,
//     and a batch takes every small request queued when it launches (up to
//     its capacity);
//   - larger instances run on lanes (an fq_ctx each: its own stream and
//     scratch), so independent requests overlap; a free lane takes the
//     oldest queued request whose session is idle and whose buffers are
//     resident or fit the HBM budget.
// A session is a sequence of steps on one graph (an optimiser loop).  For
// N >= 16 its state and costate buffers (2 x 16 x 2^N bytes) stay resident
// across steps in a pool owned by the server and are released when the
// session is closed or, least recently used first, when another session
// needs the room.  Cut values are recomputed on the fly from the weights, so
// no 2^N diagonal is stored.  Steps of one session run in submission order.
// Results carry the submit, start and completion times (steady clock, s).
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <set>
#include <thread>
#include <vector>

#include "fq_ctx.h"
#include "fq_engine.h"
#include "fq_small.h"

namespace fq {
namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

size_t session_bytes(int N) { return 2 * (sizeof(double2) << N); }

struct Req {
    uint64_t ticket = 0, session = 0;
    int N = 0, P = 0;
    std::vector<double> w;      // N*N symmetric (small instances)
    std::vector<double> graph;  // N*N upper triangle (large instances)
    std::vector<double> gammas, betas;
    double t_submit = 0, t_start = 0;
};

struct Session {
    int N = 0;
    void* sv = nullptr;
    void* cs = nullptr;
    bool busy = false;
    bool heavy = false;   // its running step counts against the heavy cap
    bool closed = false;  // release once the running step completes
    int queued = 0;       // its requests waiting for a lane
    double last_used = 0;
};

struct Lane {
    fq_ctx* ctx = nullptr;
    cudaStream_t st = nullptr;  // low priority: one-CTA batches go first
    cudaEvent_t done = nullptr;
    bool busy = false;
    Req cur;
    std::thread th;  // the lane's own thread: takes requests, launches, completes them
};

constexpr int kBatchCap = 4096;           // small instances per launch
constexpr int kExpressN = 20;             // lane requests up to this size go first
constexpr double kEvictIdleS = 0.05;      // a session idle this long may lose its buffers
constexpr int kHeavyN = 24;               // requests this large fill the GPU on their own

// Requests with N >= kHeavyN in flight at once (FQ_SERVE_HEAVY, 0 = no
// cap; default 1).  Each one alone keeps HBM busy, so running two together
// gains no throughput (10,000-request stream on B200: 167 evals/s with the
// cap, 166 without) and holds the other lanes' short requests back: p50
// latency 3.5 ms with the cap, 12.9 ms without.
static int heavy_cap() {
    static int c = -1;
    if (c < 0) {
        const char* e = getenv("FQ_SERVE_HEAVY");
        c = e ? std::max(0, atoi(e)) : 1;
    }
    return c;
}
constexpr size_t kBatchBytes = 8u << 20;  // descriptors + data per launch
constexpr int kBatchOut = kBatchCap * (1 + 2 * FQ_SERVE_MAX_LAYERS);

struct Batch {
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    unsigned char* h_in = nullptr;  // pinned
    unsigned char* d_in = nullptr;
    double* h_out = nullptr;  // pinned
    double* d_out = nullptr;
    std::vector<Req> reqs;
    std::vector<int> out_off;
    bool busy = false;
    double t_start = 0;
};

}  // namespace
}  // namespace fq

using namespace fq;

struct fq_server {
    int device = 0;
    double budget = 0;
    size_t used = 0;  // bytes of resident session buffers
    int heavy_running = 0;  // steps with N >= kHeavyN on lanes (guarded by mu)
    cudaMemPool_t pool = nullptr;
    cudaStream_t free_stream = nullptr;
    std::vector<Lane> lanes;
    Batch batches[2];
    std::map<uint64_t, Session> sessions;  // guarded by mu
    std::deque<Req> small_q, large_q;      // guarded by mu
    std::vector<fq_result> done;           // guarded by mu
    std::mutex mu;
    std::condition_variable cv_done, cv_work, cv_lane;
    std::thread worker;
    bool stop = false;
    uint64_t next_ticket = 1;
    long long in_flight = 0;
    // Written by the worker, read by fq_server_stats.
    std::atomic<long long> launches{0}, batched{0}, laned{0};
    int error = FQ_OK;
    char errmsg[256] = "";

    // Records the first failure for fq_server_poll (worker thread).
    void fail(int st) {
        std::lock_guard<std::mutex> lk(mu);
        if (error == FQ_OK) {
            error = st;
            snprintf(errmsg, sizeof(errmsg), "%s", fq_last_error());
        }
    }

    void finish(const Req& r, int status, const double* e, const double* gg, const double* gb,
                double t_start) {
        fq_result o;
        memset(&o, 0, sizeof(o));
        o.ticket = r.ticket;
        o.session = r.session;
        o.N = r.N;
        o.P = r.P;
        o.status = status;
        if (status == FQ_OK) {
            o.energy = *e;
            for (int k = 0; k < r.P; k++) {
                o.grad_gamma[k] = gg[k];
                o.grad_beta[k] = gb[k];
            }
        }
        o.t_submit = r.t_submit;
        o.t_start = t_start;
        o.t_done = now_s();
        std::lock_guard<std::mutex> lk(mu);
        done.push_back(o);
        in_flight--;
        cv_done.notify_all();
    }

    // ---- small instances (one CTA each, or one cluster of CTAs) --------------
    static size_t job_bytes(const Req& r) {
        return sizeof(SmallJob) + sizeof(double) * (r.N * r.N + 2 * r.P);
    }

    int launch_batch(Batch& B) {
        const int nj = (int)B.reqs.size();
        // One launch per size class (one CTA, clusters of 2, 4, 8 CTAs):
        // the batch in class order.
        std::stable_sort(B.reqs.begin(), B.reqs.end(), [](const Req& a, const Req& b) {
            return small_class(a.N) < small_class(b.N);
        });
        int nmax = 1, counts[kSmallClasses] = {};
        for (auto& r : B.reqs) {
            counts[small_class(r.N)]++;
            if (small_class(r.N) == 0) nmax = std::max(nmax, r.N);
        }
        SmallJob* hj = reinterpret_cast<SmallJob*>(B.h_in);
        double* hd = reinterpret_cast<double*>(B.h_in + sizeof(SmallJob) * nj);
        const double* dd = reinterpret_cast<const double*>(B.d_in + sizeof(SmallJob) * nj);
        size_t off = 0;
        int o = 0;
        B.out_off.assign(nj, 0);
        for (int i = 0; i < nj; i++) {
            const Req& r = B.reqs[i];
            SmallJob d;
            d.N = r.N;
            d.P = r.P;
            d.flags = SJ_ENERGY | SJ_GRAD;
            d.pad = 0;
            memcpy(hd + off, r.w.data(), sizeof(double) * r.N * r.N);
            d.w = dd + off;
            off += r.N * r.N;
            memcpy(hd + off, r.gammas.data(), sizeof(double) * r.P);
            d.gammas = dd + off;
            off += r.P;
            memcpy(hd + off, r.betas.data(), sizeof(double) * r.P);
            d.betas = dd + off;
            off += r.P;
            d.out = B.d_out + o;
            B.out_off[i] = o;
            o += 1 + 2 * r.P;
            d.state = nullptr;
            hj[i] = d;
        }
        const size_t need = sizeof(SmallJob) * nj + sizeof(double) * off;
        FQ_CUDA(cudaMemcpyAsync(B.d_in, B.h_in, need, cudaMemcpyHostToDevice, B.st));
        FQ_TRY(launch_small_jobs(reinterpret_cast<const SmallJob*>(B.d_in), counts, nmax, B.st));
        FQ_CUDA(cudaMemcpyAsync(B.h_out, B.d_out, sizeof(double) * o, cudaMemcpyDeviceToHost,
                                B.st));
        FQ_CUDA(cudaEventRecord(B.done, B.st));
        B.busy = true;
        B.t_start = now_s();
        launches++;
        batched += nj;
        return FQ_OK;
    }

    void complete_batch(Batch& B) {
        for (size_t i = 0; i < B.reqs.size(); i++) {
            const Req& r = B.reqs[i];
            const double* out = B.h_out + B.out_off[i];
            finish(r, FQ_OK, out, out + 1, out + 1 + r.P, B.t_start);
        }
        B.reqs.clear();
        B.busy = false;
    }

    // Takes queued small requests that fit one launch (in order).
    void take_small(Batch& B) {
        size_t bytes = 0;
        int outw = 0;
        std::lock_guard<std::mutex> lk(mu);
        while (!small_q.empty() && (int)B.reqs.size() < kBatchCap) {
            const Req& r = small_q.front();
            if (bytes + job_bytes(r) > kBatchBytes || outw + 1 + 2 * r.P > kBatchOut) break;
            bytes += job_bytes(r);
            outw += 1 + 2 * r.P;
            B.reqs.push_back(std::move(small_q.front()));
            small_q.pop_front();
        }
    }

    // ---- large instances (lanes) --------------------------------------------
    // Frees a session's buffers (mu held; the session must be idle).
    void drop_buffers(Session& s) {
        if (!s.sv) return;
        cudaFreeAsync(s.sv, free_stream);
        cudaFreeAsync(s.cs, free_stream);
        used -= session_bytes(s.N);
        s.sv = s.cs = nullptr;
    }

    // Room for `bytes` more resident bytes: evict idle sessions, least
    // recently used first (mu held).
    // Only sessions with no step running or queued and idle for kEvictIdleS
    // are evicted, so a session between two steps of its optimiser loop
    // keeps its buffers and new sessions wait for room instead of evicting
    // busy ones (admission by budget, not thrashing).
    bool make_room(size_t bytes) {
        const double now = now_s();
        while ((double)(used + bytes) > budget) {
            Session* victim = nullptr;
            for (auto& kv : sessions)
                if (!kv.second.busy && kv.second.sv && kv.second.queued == 0 &&
                    now - kv.second.last_used >= kEvictIdleS &&
                    (!victim || kv.second.last_used < victim->last_used))
                    victim = &kv.second;
            if (!victim) return false;
            drop_buffers(*victim);
        }
        return true;
    }

    // Picks a runnable large request and reserves its session's buffers (mu
    // held): the oldest with N <= kExpressN if any (short requests are not
    // queued behind long ones), else the oldest.  Steps of a session keep
    // their order: a request is skipped if its session is running or an
    // earlier request of the same session is still queued.
    bool pick_large(Req& out, Session*& sess) {
        return pick_large_if(out, sess, kExpressN, false) ||
               pick_large_if(out, sess, kMaxQubits, true) ||
               pick_large_if(out, sess, kMaxQubits, false);
    }

    // resident_only: only sessions whose buffers are already allocated.
    bool pick_large_if(Req& out, Session*& sess, int nmax, bool resident_only) {
        std::set<uint64_t> blocked;
        for (auto it = large_q.begin(); it != large_q.end(); ++it) {
            if (blocked.count(it->session)) continue;
            blocked.insert(it->session);
            if (it->N > nmax) continue;
            Session& s = sessions[it->session];
            if (s.busy) continue;
            const bool heavy = it->N >= kHeavyN;
            if (heavy && heavy_cap() > 0 && heavy_running >= heavy_cap()) continue;
            if (resident_only && !(s.sv && s.N == it->N)) continue;
            if (s.sv && s.N != it->N) drop_buffers(s);  // the session changed size
            if (!s.sv) {
                const size_t bytes = session_bytes(it->N);
                if (!make_room(bytes)) continue;
                used += bytes;  // allocated by the lane on its stream
            }
            s.N = it->N;
            s.busy = true;
            s.heavy = heavy;
            heavy_running += heavy ? 1 : 0;
            s.queued--;
            s.last_used = now_s();
            out = std::move(*it);
            large_q.erase(it);
            sess = &s;
            return true;
        }
        return false;
    }

    int start_large(Lane& L, Req& r, Session& s) {
        cudaStream_t st = (cudaStream_t)fq_ctx_stream(L.ctx);
        if (!s.sv) {
            const size_t half = session_bytes(r.N) / 2;
            void *sv = nullptr, *cs = nullptr;
            if (cudaMallocFromPoolAsync(&sv, half, pool, st) != cudaSuccess ||
                cudaMallocFromPoolAsync(&cs, half, pool, st) != cudaSuccess) {
                cudaGetLastError();
                if (sv) cudaFreeAsync(sv, st);
                std::lock_guard<std::mutex> lk(mu);
                used -= session_bytes(r.N);
                set_error("session buffers of %zu bytes could not be allocated", 2 * half);
                return FQ_ERR_OOM;
            }
            std::lock_guard<std::mutex> lk(mu);
            s.sv = sv;
            s.cs = cs;
        }
        r.t_start = now_s();
        long long k0 = 0, k1 = 0;
        fq_ctx_kernel_launches(L.ctx, &k0);
        FQ_TRY(grad_enqueue(L.ctx, s.sv, s.cs, r.N, r.P, r.graph.data(), r.gammas.data(),
                            r.betas.data()));
        FQ_CUDA(cudaEventRecord(L.done, st));
        fq_ctx_kernel_launches(L.ctx, &k1);
        L.cur = std::move(r);
        L.busy = true;
        launches += k1 - k0;
        laned++;
        return FQ_OK;
    }

    void end_step(uint64_t id) {
        std::lock_guard<std::mutex> lk(mu);
        auto it = sessions.find(id);
        if (it == sessions.end()) return;
        if (it->second.heavy) heavy_running--;
        it->second.heavy = false;
        it->second.busy = false;
        it->second.last_used = now_s();
        if (it->second.closed && it->second.queued == 0) {
            drop_buffers(it->second);
            sessions.erase(it);
        }
    }

    void complete_large(Lane& L) {
        double e = 0, gg[FQ_SERVE_MAX_LAYERS], gb[FQ_SERVE_MAX_LAYERS];
        const int st = grad_collect(L.ctx, L.cur.N, L.cur.P, &e, gg, gb);
        if (st != FQ_OK) fail(st);
        end_step(L.cur.session);
        finish(L.cur, st, &e, gg, gb, L.cur.t_start);
        L.busy = false;
    }

    // ---- lane threads ----------------------------------------------------------
    // A lane takes the next runnable large request (pick_large), enqueues its
    // kernels on the lane's stream, waits for its event (polling, so that
    // sixteen lanes do not hold sixteen cores in a blocking wait) and
    // completes it.  It leaves once the server stops and no large request is
    // queued.
    void lane_loop(Lane& L) {
        cudaSetDevice(device);
        while (true) {
            Req r;
            Session* s = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                while (!pick_large(r, s)) {
                    if (stop && large_q.empty()) return;
                    cv_lane.wait_for(lk, std::chrono::milliseconds(2));
                }
            }
            const int st = start_large(L, r, *s);
            if (st != FQ_OK) {
                fail(st);
                end_step(r.session);
                finish(r, st, nullptr, nullptr, nullptr, now_s());
                cv_lane.notify_all();
                continue;
            }
            while (true) {
                const cudaError_t q = cudaEventQuery(L.done);
                if (q == cudaSuccess) break;
                if (q != cudaErrorNotReady) {
                    cudaGetLastError();
                    break;  // grad_collect reports the failure
                }
                std::this_thread::sleep_for(std::chrono::microseconds(20));
            }
            complete_large(L);
            cv_lane.notify_all();  // the session may have a next step queued
        }
    }

    // ---- scheduler loop -----------------------------------------------------
    void loop() {
        cudaSetDevice(device);
        while (true) {
            bool worked = false, pending = false;
            for (auto& B : batches) {
                if (B.busy && cudaEventQuery(B.done) == cudaSuccess) {
                    complete_batch(B);
                    worked = true;
                }
                if (!B.busy) {
                    take_small(B);
                    if (!B.reqs.empty()) {
                        const int st = launch_batch(B);
                        if (st != FQ_OK) {
                            fail(st);
                            for (auto& r : B.reqs) finish(r, st, nullptr, nullptr, nullptr, now_s());
                            B.reqs.clear();
                        }
                        worked = true;
                    }
                }
                pending |= B.busy;
            }
            if (worked) continue;
            std::unique_lock<std::mutex> lk(mu);
            if (stop && small_q.empty() && !pending) break;
            if (pending) {
                lk.unlock();
                std::this_thread::sleep_for(std::chrono::microseconds(10));
            } else {
                cv_work.wait_for(lk, std::chrono::milliseconds(5));
            }
        }
    }
};

extern "C" {

int fq_server_create(int device, double hbm_budget_bytes, int lanes, fq_server** out) {
    FQ_CHECK(out != nullptr, FQ_ERR_INVALID, "null output pointer");
    FQ_CHECK(lanes >= 1 && lanes <= 16, FQ_ERR_INVALID, "lanes=%d outside [1,16]", lanes);
    FQ_CHECK(hbm_budget_bytes > 0, FQ_ERR_INVALID, "the HBM budget must be positive");
    *out = nullptr;
    int ndev = 0;
    FQ_CUDA(cudaGetDeviceCount(&ndev));
    FQ_CHECK(device >= 0 && device < ndev, FQ_ERR_INVALID, "device %d not present (%d)", device,
             ndev);
    FQ_CUDA(cudaSetDevice(device));
    // Batches of one-CTA instances run at the highest stream priority, so
    // their CTAs are scheduled ahead of the lanes' pass kernels.
    int prio_low = 0, prio_high = 0;
    FQ_CUDA(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
    fq_server* S = new fq_server();
    S->device = device;
    S->budget = hbm_budget_bytes;
    int st = FQ_OK;
    for (int i = 0; i < lanes && st == FQ_OK; i++) {
        Lane L;
        if (cudaStreamCreateWithPriority(&L.st, cudaStreamNonBlocking, prio_low) != cudaSuccess)
            st = FQ_ERR_CUDA;
        if (st == FQ_OK) st = fq_ctx_create(device, L.st, &L.ctx);
        if (st == FQ_OK &&
            cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming) != cudaSuccess)
            st = FQ_ERR_CUDA;
        S->lanes.push_back(std::move(L));
    }
    for (auto& B : S->batches) {
        if (st != FQ_OK) break;
        if (cudaStreamCreateWithPriority(&B.st, cudaStreamNonBlocking, prio_high) != cudaSuccess ||
            cudaEventCreateWithFlags(&B.done, cudaEventDisableTiming) != cudaSuccess ||
            cudaMallocHost(&B.h_in, kBatchBytes) != cudaSuccess ||
            cudaMalloc(&B.d_in, kBatchBytes) != cudaSuccess ||
            cudaMallocHost(&B.h_out, sizeof(double) * kBatchOut) != cudaSuccess ||
            cudaMalloc(&B.d_out, sizeof(double) * kBatchOut) != cudaSuccess)
            st = FQ_ERR_OOM;
    }
    if (st == FQ_OK) {
        // A pool of its own that keeps freed session buffers for reuse.
        cudaMemPoolProps props;
        memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        uint64_t keep = (uint64_t)hbm_budget_bytes;
        if (cudaMemPoolCreate(&S->pool, &props) != cudaSuccess ||
            cudaMemPoolSetAttribute(S->pool, cudaMemPoolAttrReleaseThreshold, &keep) !=
                cudaSuccess ||
            cudaStreamCreateWithFlags(&S->free_stream, cudaStreamNonBlocking) != cudaSuccess)
            st = FQ_ERR_CUDA;
    }
    if (st != FQ_OK) {
        set_error("server creation failed: %s", cudaGetErrorString(cudaGetLastError()));
        fq_server_destroy(S);
        return st;
    }
    S->worker = std::thread([S] { S->loop(); });
    for (auto& L : S->lanes) {
        Lane* lp = &L;
        L.th = std::thread([S, lp] { S->lane_loop(*lp); });
    }
    *out = S;
    return FQ_OK;
}

int fq_server_destroy(fq_server* S) {
    if (!S) return FQ_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        S->cv_work.notify_all();
        S->cv_lane.notify_all();
    }
    if (S->worker.joinable()) S->worker.join();
    for (auto& L : S->lanes)
        if (L.th.joinable()) L.th.join();
    cudaSetDevice(S->device);
    for (auto& L : S->lanes)
        if (L.st) cudaStreamSynchronize(L.st);
    for (auto& kv : S->sessions) {
        if (kv.second.sv) cudaFreeAsync(kv.second.sv, S->free_stream);
        if (kv.second.cs) cudaFreeAsync(kv.second.cs, S->free_stream);
    }
    if (S->free_stream) {
        cudaStreamSynchronize(S->free_stream);
        cudaStreamDestroy(S->free_stream);
    }
    if (S->pool) cudaMemPoolDestroy(S->pool);
    for (auto& L : S->lanes) {
        if (L.done) cudaEventDestroy(L.done);
        fq_ctx_destroy(L.ctx);
        if (L.st) cudaStreamDestroy(L.st);
    }
    for (auto& B : S->batches) {
        if (B.st) cudaStreamSynchronize(B.st);
        if (B.done) cudaEventDestroy(B.done);
        if (B.st) cudaStreamDestroy(B.st);
        if (B.h_in) cudaFreeHost(B.h_in);
        cudaFree(B.d_in);
        if (B.h_out) cudaFreeHost(B.h_out);
        cudaFree(B.d_out);
    }
    delete S;
    return FQ_OK;
}

int fq_server_submit(fq_server* S, const fq_request* q, uint64_t* ticket) {
    FQ_CHECK(S && q && ticket, FQ_ERR_INVALID, "null argument");
    FQ_CHECK(q->N >= 2 && q->N <= kMaxQubits, FQ_ERR_INVALID, "N=%d out of range [2,%d]", q->N,
             kMaxQubits);
    FQ_CHECK(q->P >= 1 && q->P <= FQ_SERVE_MAX_LAYERS, FQ_ERR_INVALID, "P=%d outside [1,%d]",
             q->P, FQ_SERVE_MAX_LAYERS);
    FQ_CHECK(q->graph_upper && q->gammas && q->betas, FQ_ERR_INVALID, "null request arrays");
    for (int p = 0; p < q->P; p++)
        FQ_CHECK(isfinite(q->gammas[p]) && isfinite(q->betas[p]), FQ_ERR_INVALID,
                 "non-finite angle at layer %d", p);
    GraphPrep g;
    FQ_TRY(prep_graph(q->graph_upper, q->N, g));
    Req r;
    r.session = q->session;
    r.N = q->N;
    r.P = q->P;
    r.gammas.assign(q->gammas, q->gammas + q->P);
    r.betas.assign(q->betas, q->betas + q->P);
    const bool small = q->N <= kSmallJobMaxQubits;
    if (small)
        r.w = g.wd;
    else
        r.graph.assign(q->graph_upper, q->graph_upper + (size_t)q->N * q->N);
    r.t_submit = now_s();
    std::lock_guard<std::mutex> lk(S->mu);
    FQ_CHECK(!S->stop, FQ_ERR_INVALID, "the server is stopping");
    FQ_CHECK(small || (double)session_bytes(q->N) <= S->budget, FQ_ERR_OOM,
             "a %d-qubit session needs %zu bytes, over the %.0f-byte budget", q->N,
             session_bytes(q->N), S->budget);
    r.ticket = S->next_ticket++;
    *ticket = r.ticket;
    S->in_flight++;
    if (small)
        S->small_q.push_back(std::move(r));
    else {
        Session& ss = S->sessions[r.session];
        ss.queued++;
        ss.closed = false;  // new work reopens a closed session
        S->large_q.push_back(std::move(r));
    }
    S->cv_work.notify_one();
    S->cv_lane.notify_one();
    return FQ_OK;
}

int fq_server_poll(fq_server* S, fq_result* out, int max_results, int* n_out, int wait_ms) {
    FQ_CHECK(S && n_out && max_results >= 0 && (max_results == 0 || out), FQ_ERR_INVALID,
             "bad argument");
    std::unique_lock<std::mutex> lk(S->mu);
    if (S->done.empty() && wait_ms > 0)
        S->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms),
                            [S] { return !S->done.empty(); });
    const int n = std::min<int>(max_results, (int)S->done.size());
    for (int i = 0; i < n; i++) out[i] = S->done[i];
    S->done.erase(S->done.begin(), S->done.begin() + n);
    *n_out = n;
    if (S->error != FQ_OK) {
        set_error("%s", S->errmsg);
        return S->error;
    }
    return FQ_OK;
}

int fq_server_close_session(fq_server* S, uint64_t session) {
    FQ_CHECK(S, FQ_ERR_INVALID, "null server");
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->sessions.find(session);
    if (it == S->sessions.end()) return FQ_OK;
    if (it->second.busy || it->second.queued > 0) {
        it->second.closed = true;  // released once its queued steps have run
    } else {
        S->drop_buffers(it->second);
        S->sessions.erase(it);
    }
    return FQ_OK;
}

int fq_server_stats(fq_server* S, fq_server_counters* c) {
    FQ_CHECK(S && c, FQ_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    c->pending = S->in_flight;
    c->kernel_launches = S->launches;
    c->batched_requests = S->batched;
    c->lane_requests = S->laned;
    c->resident_bytes = (double)S->used;
    long long n = 0;
    for (auto& kv : S->sessions) n += kv.second.sv ? 1 : 0;
    c->resident_sessions = n;
    return FQ_OK;
}

}  // extern "C"
