// serve_replay.cpp -- replays a served request stream through the C ABI
// natively, so that neither the served run nor the one-at-a-time runs it is
// compared with carry the per-request cost of a Python client loop.
//
// A stream is a set of sessions (optimiser loops): each has a graph, a depth
// P, starting angles and an arrival time, and takes `steps` energy+gradient
// evaluations, every step moving the angles against the previous step's
// gradient (the same deterministic rule as serve_stream.next_angles).
//
//   serve_replay STREAM MODE OUT [lanes] [budget_gb]
//     MODE served      sessions arrive at their arrival times and run through
//                      the server (fq_server_*: continuous batching);
//          sequential  the same evaluations one at a time through
//                      fq_qaoa_energy_grad on one context, state and costate
//                      allocated once per session;
//          plain       the same, every call allocating its own buffers (a
//                      plain call of the public API).
//
// STREAM (little endian): int32 n_sessions, int32 steps; per session int32
// id, N, P, then float64 arrival_s, graph[N*N] (upper triangle read),
// gammas[P], betas[P].
// OUT: per evaluation int32 session, step, N, P; float64 energy, latency_s,
// queue_s; float64 grad_gamma[P], grad_beta[P].  Prints one JSON line with
// the wall time (and the server's counters in served mode).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <string>
#include <vector>

#include "forqaoa.h"

namespace {

struct Sess {
    int id = 0, N = 0, P = 0;
    double arrival = 0;
    std::vector<double> graph, g, b;
    int left = 0;
};

struct Rec {
    int session, step, N, P;
    double energy, latency, queue;
    std::vector<double> gg, gb;
};

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

[[noreturn]] void die(const char* what, int st = 0) {
    fprintf(stderr, "serve_replay: %s (status %d: %s)\n", what, st, st ? fq_last_error() : "");
    exit(2);
}

bool rd(FILE* f, void* p, size_t n) { return fread(p, 1, n, f) == n; }

// One optimiser step (serve_stream.next_angles).
void next_angles(std::vector<double>& g, std::vector<double>& b, const double* gg,
                 const double* gb, int P) {
    double m = 1.0;
    for (int k = 0; k < P; k++) m = std::max(m, std::max(std::fabs(gg[k]), std::fabs(gb[k])));
    const double s = 0.05 / m;
    for (int k = 0; k < P; k++) {
        g[k] = g[k] - s * gg[k];
        b[k] = b[k] - s * gb[k];
    }
}

void run_served(std::vector<Sess>& ss, int steps, int lanes, double budget, std::vector<Rec>& out,
                double& wall, fq_server_counters& cnt) {
    fq_server* srv = nullptr;
    int st = fq_server_create(0, budget, lanes, &srv);
    if (st) die("fq_server_create", st);
    std::vector<int> order(ss.size());
    for (size_t i = 0; i < ss.size(); i++) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return ss[a].arrival < ss[b].arrival; });
    std::vector<int> by_id;
    for (size_t i = 0; i < ss.size(); i++) {
        if (ss[i].id >= (int)by_id.size()) by_id.resize(ss[i].id + 1, -1);
        by_id[ss[i].id] = (int)i;
    }
    auto submit = [&](Sess& s) {
        fq_request r;
        r.session = (uint64_t)s.id;
        r.N = s.N;
        r.P = s.P;
        r.graph_upper = s.graph.data();
        r.gammas = s.g.data();
        r.betas = s.b.data();
        uint64_t t;
        const int e = fq_server_submit(srv, &r, &t);
        if (e) die("fq_server_submit", e);
    };
    std::vector<fq_result> res(4096);
    size_t nxt = 0;
    long long outstanding = 0;
    const double t0 = now_s();
    while (nxt < order.size() || outstanding) {
        const double now = now_s() - t0;
        while (nxt < order.size() && ss[order[nxt]].arrival <= now) {
            submit(ss[order[nxt]]);
            outstanding++;
            nxt++;
        }
        int wait = 20;
        if (nxt < order.size())
            wait = std::max(0, std::min(20, (int)((ss[order[nxt]].arrival - now) * 1000.0)));
        int n = 0;
        const int e = fq_server_poll(srv, res.data(), (int)res.size(), &n, wait);
        if (e) die("fq_server_poll", e);
        for (int i = 0; i < n; i++) {
            const fq_result& r = res[i];
            if (r.status) die("a request failed", r.status);
            outstanding--;
            Sess& s = ss[by_id[(int)r.session]];
            Rec rec{(int)r.session, steps - s.left, r.N, r.P, r.energy, r.t_done - r.t_submit,
                    r.t_start - r.t_submit,
                    std::vector<double>(r.grad_gamma, r.grad_gamma + r.P),
                    std::vector<double>(r.grad_beta, r.grad_beta + r.P)};
            out.push_back(std::move(rec));
            s.left--;
            next_angles(s.g, s.b, r.grad_gamma, r.grad_beta, s.P);
            if (s.left)
                submit(s), outstanding++;
            else if ((st = fq_server_close_session(srv, (uint64_t)s.id)))
                die("fq_server_close_session", st);
        }
    }
    wall = now_s() - t0;
    fq_server_stats(srv, &cnt);
    if ((st = fq_server_destroy(srv))) die("fq_server_destroy", st);
}

void run_sequential(std::vector<Sess>& ss, int steps, bool reuse, std::vector<Rec>& out,
                    double& wall) {
    fq_ctx* ctx = nullptr;
    int st = fq_ctx_create(0, nullptr, &ctx);
    if (st) die("fq_ctx_create", st);
    std::vector<int> order(ss.size());
    for (size_t i = 0; i < ss.size(); i++) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return ss[a].arrival < ss[b].arrival; });
    const double t0 = now_s();
    for (int i : order) {
        Sess& s = ss[i];
        void *sv = nullptr, *cs = nullptr;
        if (reuse && s.N > FQ_SMALL_MAX_QUBITS) {
            if ((st = fq_state_alloc(ctx, s.N, &sv)) || (st = fq_state_alloc(ctx, s.N, &cs)))
                die("fq_state_alloc", st);
        }
        std::vector<double> gg(s.P), gb(s.P);
        for (int k = 0; k < steps; k++) {
            double e;
            const double t1 = now_s();
            // A plain call allocates its state and costate (above
            // FQ_SMALL_MAX_QUBITS) and frees them afterwards, inside the
            // timed call.
            const bool own = !reuse && s.N > FQ_SMALL_MAX_QUBITS;
            if (own && ((st = fq_state_alloc(ctx, s.N, &sv)) || (st = fq_state_alloc(ctx, s.N, &cs))))
                die("fq_state_alloc", st);
            st = fq_qaoa_energy_grad(ctx, sv, cs, s.N, s.P, s.graph.data(), s.g.data(),
                                     s.b.data(), &e, gg.data(), gb.data());
            if (st) die("fq_qaoa_energy_grad", st);
            if (own) {
                if ((st = fq_state_free(ctx, sv)) || (st = fq_state_free(ctx, cs)))
                    die("fq_state_free", st);
                sv = cs = nullptr;
            }
            out.push_back(Rec{s.id, k, s.N, s.P, e, now_s() - t1, 0.0, gg, gb});
            next_angles(s.g, s.b, gg.data(), gb.data(), s.P);
        }
        if (sv) fq_state_free(ctx, sv);
        if (cs) fq_state_free(ctx, cs);
    }
    wall = now_s() - t0;
    fq_ctx_destroy(ctx);
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 4) {
        fprintf(stderr, "usage: serve_replay STREAM served|sequential|plain OUT [lanes] [budget_gb]\n");
        return 2;
    }
    const std::string mode = argv[2];
    const int lanes = argc > 4 ? atoi(argv[4]) : 4;
    const double budget = (argc > 5 ? atof(argv[5]) : 150.0) * 1e9;
    FILE* f = fopen(argv[1], "rb");
    if (!f) die("cannot open the stream file");
    int hdr[2];
    if (!rd(f, hdr, sizeof(hdr)) || hdr[0] < 0 || hdr[1] < 1) die("bad stream header");
    const int steps = hdr[1];
    std::vector<Sess> ss(hdr[0]);
    for (Sess& s : ss) {
        int h[3];
        if (!rd(f, h, sizeof(h)) || !rd(f, &s.arrival, sizeof(double))) die("short stream");
        s.id = h[0];
        s.N = h[1];
        s.P = h[2];
        if (s.id < 0 || s.N < 2 || s.N > 33 || s.P < 1 || s.P > FQ_SERVE_MAX_LAYERS)
            die("bad session record");
        s.graph.resize((size_t)s.N * s.N);
        s.g.resize(s.P);
        s.b.resize(s.P);
        if (!rd(f, s.graph.data(), s.graph.size() * sizeof(double)) ||
            !rd(f, s.g.data(), s.P * sizeof(double)) || !rd(f, s.b.data(), s.P * sizeof(double)))
            die("short stream");
        s.left = steps;
    }
    fclose(f);

    std::vector<Rec> recs;
    recs.reserve(ss.size() * steps);
    double wall = 0;
    fq_server_counters cnt;
    memset(&cnt, 0, sizeof(cnt));
    if (mode == "served")
        run_served(ss, steps, lanes, budget, recs, wall, cnt);
    else if (mode == "sequential" || mode == "plain")
        run_sequential(ss, steps, mode == "sequential", recs, wall);
    else
        die("mode must be served, sequential or plain");

    FILE* o = fopen(argv[3], "wb");
    if (!o) die("cannot open the output file");
    for (const Rec& r : recs) {
        const int h[4] = {r.session, r.step, r.N, r.P};
        const double d[3] = {r.energy, r.latency, r.queue};
        fwrite(h, sizeof(int), 4, o);
        fwrite(d, sizeof(double), 3, o);
        fwrite(r.gg.data(), sizeof(double), r.P, o);
        fwrite(r.gb.data(), sizeof(double), r.P, o);
    }
    fclose(o);
    printf("{\"mode\": \"%s\", \"evals\": %zu, \"wall_s\": %.6f, \"kernel_launches\": %lld, "
           "\"batched_requests\": %lld, \"lane_requests\": %lld}\n",
           mode.c_str(), recs.size(), wall, cnt.kernel_launches, cnt.batched_requests,
           cnt.lane_requests);
    return 0;
}
