// fq_ctx.cu -- context, status reporting, state memory and host-side graph
// handling of the FOR-QAOA B200 library.
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>

#include "fq_ctx.h"
#include "fq_pass.cuh"

namespace fq {

static thread_local char g_err[512] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int validate_ctx(fq_ctx* ctx) {
    FQ_CHECK(ctx != nullptr, FQ_ERR_INVALID, "null context");
    FQ_CUDA(cudaSetDevice(ctx->device));
    return FQ_OK;
}

int check_device_error(fq_ctx* ctx) {
    int flag = 0;
    FQ_CUDA(cudaMemcpy(&flag, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
        FQ_CUDA(cudaMemset(ctx->d_err, 0, sizeof(int)));
        set_error("a device-side bounded wait gave up (flag %d); results are incomplete", flag);
        return FQ_ERR_TIMEOUT;
    }
    return FQ_OK;
}

int stage_acquire(fq_ctx* ctx) {
    FQ_CUDA(cudaEventSynchronize(ctx->stage_evt));
    return FQ_OK;
}

// Weights must be finite; the integer path needs every weight integral and
// the cut range small enough for a phase table (src/rzz.cu:131-146 sums
// +-w in FP64, which is exact for such weights).
int prep_graph(const double* upper, int N, GraphPrep& g) {
    FQ_CHECK(upper != nullptr, FQ_ERR_INVALID, "null graph");
    FQ_CHECK(N >= 1 && N <= kMaxQubits, FQ_ERR_INVALID, "N=%d out of range [1,%d]", N,
             kMaxQubits);
    g.N = N;
    g.wabs = 0;
    g.wd.assign((size_t)N * N, 0.0);
    g.wi.assign((size_t)N * N, 0);
    bool integral = true;
    long long pos = 0, neg = 0, absum = 0;
    double W = 0;
    for (int i = 0; i < N; i++)
        for (int j = i + 1; j < N; j++) {
            const double w = upper[i * N + j];
            FQ_CHECK(isfinite(w), FQ_ERR_INVALID, "non-finite weight at (%d,%d)", i, j);
            g.wd[i * N + j] = g.wd[j * N + i] = w;
            W += w;
            g.wabs += fabs(w);
            if (w != rint(w) || fabs(w) > (double)(1 << 20)) {
                integral = false;
            } else {
                const long long wl = (long long)w;
                if (wl > 0) pos += wl; else neg += wl;
                absum += wl > 0 ? wl : -wl;
                g.wi[i * N + j] = g.wi[j * N + i] = (int)wl;
            }
        }
    g.W = W;
    g.gmax = 0;
    if (integral)
        for (int u = 0; u < N; u++) {
            long long d = 0;
            for (int v = 0; v < N; v++) d += g.wi[u * N + v] > 0 ? g.wi[u * N + v] : -g.wi[u * N + v];
            g.gmax = std::max(g.gmax, d);
        }
    g.integer = integral && absum < (1ll << 30) && (pos - neg + 1) <= kMaxPhaseTable;
    g.W_int = pos + neg;
    g.cmin = neg;
    g.cmax = pos;
    return FQ_OK;
}

int upload_graph(fq_ctx* ctx, const GraphPrep& g, const double* upper) {
    const size_t nn = (size_t)g.N * g.N;
    // Key: the upper triangle plus the path taken.
    if (ctx->g_n == g.N && ctx->g_key.size() == nn + 1 &&
        memcmp(ctx->g_key.data(), upper, nn * sizeof(double)) == 0 &&
        ctx->g_key[nn] == (g.integer ? 1.0 : 0.0))
        return FQ_OK;
    FQ_TRY(stage_acquire(ctx));
    const size_t bytes = g.integer ? nn * sizeof(int) : nn * sizeof(double);
    memcpy(ctx->h_stage, g.integer ? (const void*)g.wi.data() : (const void*)g.wd.data(), bytes);
    FQ_CUDA(cudaMemcpyAsync(ctx->d_w, ctx->h_stage, bytes, cudaMemcpyHostToDevice, ctx->stream));
    FQ_CUDA(cudaEventRecord(ctx->stage_evt, ctx->stream));
    ctx->g_key.assign(upper, upper + nn);
    ctx->g_key.push_back(g.integer ? 1.0 : 0.0);
    ctx->g_n = g.N;
    ctx->g_version++;
    return FQ_OK;
}

static cudaEvent_t pool_get(fq_ctx* ctx) {
    cudaEvent_t e = nullptr;
    if (!ctx->prof_pool.empty()) {
        e = ctx->prof_pool.back();
        ctx->prof_pool.pop_back();
    } else if (cudaEventCreate(&e) != cudaSuccess) {
        e = nullptr;
    }
    return e;
}

int prof_begin(fq_ctx* ctx) {
    if (!ctx->profiling) return -1;
    cudaEvent_t a = pool_get(ctx), b = pool_get(ctx);
    if (!a || !b) return -1;
    cudaEventRecord(a, ctx->stream);
    ctx->prof_pending.push_back({a, b, FQ_KIND_OTHER, 0.0});
    return (int)ctx->prof_pending.size() - 1;
}

void prof_end(fq_ctx* ctx, int token, int kind, double bytes) {
    if (token < 0 || token >= (int)ctx->prof_pending.size()) return;
    fq_ctx::ProfRec& r = ctx->prof_pending[token];
    cudaEventRecord(r.b, ctx->stream);
    r.kind = kind;
    r.bytes = bytes;
}

static int prof_resolve(fq_ctx* ctx) {
    if (ctx->prof_pending.empty()) return FQ_OK;
    FQ_CUDA(cudaStreamSynchronize(ctx->stream));
    for (auto& r : ctx->prof_pending) {
        float ms = 0;
        FQ_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
        if (r.kind >= 0 && r.kind < FQ_KIND_COUNT) {
            ctx->prof_ms[r.kind] += ms;
            ctx->prof_bytes[r.kind] += r.bytes;
            ctx->prof_count[r.kind]++;
        }
        ctx->prof_pool.push_back(r.a);
        ctx->prof_pool.push_back(r.b);
    }
    ctx->prof_pending.clear();
    return FQ_OK;
}

}  // namespace fq

using namespace fq;

extern "C" {

const char* fq_status_string(int status) {
    switch (status) {
        case FQ_OK: return "ok";
        case FQ_ERR_INVALID: return "invalid argument";
        case FQ_ERR_UNSUPPORTED: return "unsupported";
        case FQ_ERR_CUDA: return "CUDA error";
        case FQ_ERR_OOM: return "out of memory";
        case FQ_ERR_TIMEOUT: return "timeout";
        case FQ_ERR_BUSY: return "busy";
        default: return "unknown status";
    }
}

const char* fq_last_error(void) { return g_err; }

int fq_version(void) { return 100; }

int fq_ctx_create(int device, void* stream, fq_ctx** out) {
    FQ_CHECK(out != nullptr, FQ_ERR_INVALID, "null output pointer");
    *out = nullptr;
    int ndev = 0;
    FQ_CUDA(cudaGetDeviceCount(&ndev));
    FQ_CHECK(device >= 0 && device < ndev, FQ_ERR_INVALID, "device %d not present (%d)", device,
             ndev);
    FQ_CUDA(cudaSetDevice(device));
    fq_ctx* c = new fq_ctx();
    c->device = device;
    int st = FQ_OK;
    do {
        if (stream) {
            c->stream = (cudaStream_t)stream;
        } else {
            if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
                st = FQ_ERR_CUDA;
                break;
            }
            c->own_stream = true;
        }
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) { st = FQ_ERR_CUDA; break; }
        c->num_sms = prop.multiProcessorCount;
        c->partial_cap = 256 * c->num_sms;  // room for every pass of a gradient's reverse sweep
        const size_t wbytes = sizeof(double) * kMaxQubits * kMaxQubits;
        if (cudaMalloc(&c->d_w, wbytes) != cudaSuccess ||
            cudaMalloc(&c->d_ptab, sizeof(double2) * kMaxPhaseTable) != cudaSuccess ||
            cudaMalloc(&c->d_partial, sizeof(double) * c->partial_cap) != cudaSuccess ||
            cudaMalloc(&c->d_result, sizeof(double) * kResultWords) != cudaSuccess ||
            cudaMalloc(&c->d_scratch, kScratchBytes) != cudaSuccess ||
            cudaMalloc(&c->d_err, sizeof(int)) != cudaSuccess ||
            cudaMemset(c->d_err, 0, sizeof(int)) != cudaSuccess) {
            st = FQ_ERR_OOM;
            break;
        }
        c->h_stage_bytes = std::max(wbytes, (size_t)256 * 1024);
        if (cudaMallocHost(&c->h_stage, c->h_stage_bytes) != cudaSuccess ||
            cudaMallocHost(&c->h_result, sizeof(double) * kResultWords) != cudaSuccess) {
            st = FQ_ERR_OOM;
            break;
        }
        if (cudaEventCreateWithFlags(&c->stage_evt, cudaEventDisableTiming) != cudaSuccess) {
            st = FQ_ERR_CUDA;
            break;
        }
        if (cudaEventRecord(c->stage_evt, c->stream) != cudaSuccess) { st = FQ_ERR_CUDA; break; }
    } while (0);
    if (st != FQ_OK) {
        set_error("context creation failed: %s", cudaGetErrorString(cudaGetLastError()));
        fq_ctx_destroy(c);
        return st;
    }
    *out = c;
    return FQ_OK;
}

int fq_ctx_destroy(fq_ctx* c) {
    if (!c) return FQ_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    cudaFree(c->d_w);
    cudaFree(c->d_ptab);
    cudaFree(c->d_partial);
    cudaFree(c->d_result);
    cudaFree(c->d_err);
    cudaFree(c->d_scratch);
    cudaFree(c->d_tcut);
    if (c->h_stage) cudaFreeHost(c->h_stage);
    if (c->h_result) cudaFreeHost(c->h_result);
    if (c->stage_evt) cudaEventDestroy(c->stage_evt);
    for (auto& r : c->prof_pending) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (cudaEvent_t e : c->prof_pool) cudaEventDestroy(e);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return FQ_OK;
}

int fq_ctx_synchronize(fq_ctx* ctx) {
    FQ_TRY(validate_ctx(ctx));
    FQ_CUDA(cudaStreamSynchronize(ctx->stream));
    return check_device_error(ctx);
}

void* fq_ctx_stream(fq_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int fq_ctx_kernel_launches(fq_ctx* ctx, long long* count) {
    FQ_CHECK(ctx && count, FQ_ERR_INVALID, "null argument");
    *count = ctx->launches;
    return FQ_OK;
}

int fq_ctx_set_profiling(fq_ctx* ctx, int enable) {
    FQ_TRY(validate_ctx(ctx));
    ctx->profiling = enable != 0;
    return FQ_OK;
}

int fq_ctx_profile(fq_ctx* ctx, int kind, double* total_ms, long long* launches, double* bytes) {
    FQ_TRY(validate_ctx(ctx));
    FQ_CHECK(kind >= 0 && kind < FQ_KIND_COUNT, FQ_ERR_INVALID, "kind %d out of range", kind);
    FQ_TRY(prof_resolve(ctx));
    if (total_ms) *total_ms = ctx->prof_ms[kind];
    if (launches) *launches = ctx->prof_count[kind];
    if (bytes) *bytes = ctx->prof_bytes[kind];
    return FQ_OK;
}

int fq_ctx_profile_reset(fq_ctx* ctx) {
    FQ_TRY(validate_ctx(ctx));
    FQ_TRY(prof_resolve(ctx));
    for (int k = 0; k < FQ_KIND_COUNT; k++) {
        ctx->prof_ms[k] = 0;
        ctx->prof_bytes[k] = 0;
        ctx->prof_count[k] = 0;
    }
    return FQ_OK;
}

int fq_ctx_device_info(fq_ctx* ctx, int* num_sms, int* ctas_per_sm) {
    FQ_CHECK(ctx, FQ_ERR_INVALID, "null context");
    if (num_sms) *num_sms = ctx->num_sms;
    if (ctas_per_sm) *ctas_per_sm = ctx->ctas_per_sm;
    return FQ_OK;
}

int fq_state_alloc(fq_ctx* ctx, int N, void** sv) {
    FQ_TRY(validate_ctx(ctx));
    FQ_CHECK(sv, FQ_ERR_INVALID, "null output pointer");
    FQ_CHECK(N >= 1 && N <= kMaxQubits, FQ_ERR_INVALID, "N=%d out of range", N);
    *sv = nullptr;
    cudaError_t e = cudaMalloc(sv, sizeof(double2) << N);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("cudaMalloc of %llu bytes: %s", (unsigned long long)(sizeof(double2) << N),
                  cudaGetErrorString(e));
        return FQ_ERR_OOM;
    }
    return FQ_OK;
}

int fq_state_free(fq_ctx* ctx, void* sv) {
    FQ_TRY(validate_ctx(ctx));
    FQ_CUDA(cudaStreamSynchronize(ctx->stream));
    FQ_CUDA(cudaFree(sv));
    return FQ_OK;
}

int fq_state_init_basis0(fq_ctx* ctx, void* sv, int N) {
    FQ_TRY(validate_ctx(ctx));
    FQ_CHECK(sv && N >= 1 && N <= kMaxQubits, FQ_ERR_INVALID, "bad state");
    FQ_CUDA(cudaMemsetAsync(sv, 0, sizeof(double2) << N, ctx->stream));
    FQ_TRY(stage_acquire(ctx));
    double one[2] = {1.0, 0.0};
    memcpy(ctx->h_stage, one, sizeof(one));
    FQ_CUDA(cudaMemcpyAsync(sv, ctx->h_stage, sizeof(one), cudaMemcpyHostToDevice, ctx->stream));
    FQ_CUDA(cudaEventRecord(ctx->stage_evt, ctx->stream));
    return FQ_OK;
}

int fq_state_to_host(fq_ctx* ctx, const void* sv, int N, void* host) {
    FQ_TRY(validate_ctx(ctx));
    FQ_CHECK(sv && host && N >= 1 && N <= kMaxQubits, FQ_ERR_INVALID, "bad arguments");
    FQ_CUDA(cudaMemcpyAsync(host, sv, sizeof(double2) << N, cudaMemcpyDeviceToHost, ctx->stream));
    FQ_CUDA(cudaStreamSynchronize(ctx->stream));
    return check_device_error(ctx);
}

int fq_state_from_host(fq_ctx* ctx, void* sv, int N, const void* host) {
    FQ_TRY(validate_ctx(ctx));
    FQ_CHECK(sv && host && N >= 1 && N <= kMaxQubits, FQ_ERR_INVALID, "bad arguments");
    FQ_CUDA(cudaMemcpyAsync(sv, host, sizeof(double2) << N, cudaMemcpyHostToDevice, ctx->stream));
    FQ_CUDA(cudaStreamSynchronize(ctx->stream));
    return FQ_OK;
}

double fq_init_amp(int N) { return pow(1. / sqrt(2.), N); }

// src/swap.cu:27-50: relabel physical qubits swap_out+m <-> swap_in+m in the
// upper-triangular matrix, one pair at a time.
int fq_relabel_graph(double* g, int N, int swap_out, int swap_in, int num_swap) {
    FQ_CHECK(g != nullptr, FQ_ERR_INVALID, "null graph");
    FQ_CHECK(N >= 1 && N <= kMaxQubits && num_swap >= 0 && swap_out >= 0 &&
                 swap_out + num_swap <= swap_in && swap_in + num_swap <= N,
             FQ_ERR_INVALID, "bad block swap out=%d in=%d k=%d N=%d", swap_out, swap_in,
             num_swap, N);
    for (; num_swap > 0; num_swap--, swap_in++, swap_out++) {
        for (int i = 0; i < N; i++) {
            if (i == swap_in || i == swap_out) continue;
            if (i < swap_out)
                std::swap(g[N * i + swap_in], g[N * i + swap_out]);
            else if (i < swap_in)
                std::swap(g[N * swap_out + i], g[N * i + swap_in]);
            else
                std::swap(g[N * swap_out + i], g[N * swap_in + i]);
        }
    }
    return FQ_OK;
}

// src/Weighted.cpp:97-138: per layer the schedule swaps [0,k_{i+1}) with
// [sum_{<=i} k, +k_{i+1}) after RX chunk i; labels follow the swaps.
int fq_reference_label_map(int N, int C, int P, int* label_map) {
    FQ_CHECK(label_map && N >= 1 && N <= kMaxQubits && C >= 1 && P >= 0, FQ_ERR_INVALID,
             "bad arguments");
    std::vector<int> sizes;
    for (int i = 0; i < N; i += C) sizes.push_back(std::min(C, N - i));
    for (int b = 0; b < N; b++) label_map[b] = b;
    for (int p = 0; p < P; p++) {
        int swap_in = 0;
        for (size_t i = 0; i + 1 < sizes.size(); i++) {
            swap_in += sizes[i];
            for (int m = 0; m < sizes[i + 1]; m++) std::swap(label_map[m], label_map[swap_in + m]);
        }
    }
    return FQ_OK;
}

}  // extern "C"
