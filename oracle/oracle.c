/*
 * oracle.c -- CPU FP64 (OpenMP) restatement of FOR-QAOA's D=0 QAOA path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library, never part of
 * it.  Each function cites the reference file:line it restates.  Reference
 * paths are relative to the FOR-QAOA project root.
 */
#define _GNU_SOURCE
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef long long i64;
typedef unsigned long long u64;

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* rzz.cu:26-28: initialAmp = pow(1./sqrt(2.), numQubits) */
double orc_init_amp(int N) { return pow(1. / sqrt(2.), N); }

/* rzz.cu:158-171: (i,j) lexicographic packing of the strict upper triangle */
void orc_upper_tri_to_1d(int N, const double* upper, double* out) {
    int cnt = 0;
    for (int i = 0; i < N; i++)
        for (int j = i + 1; j < N; j++) out[cnt++] = upper[i * N + j];
}

/* rzz.cu:131-143: S(b) accumulated over pairs in packing order, zero skipped */
static double pair_sum(u64 b, int N, const double* g1d) {
    double sum = 0;
    int cnt = 0;
    for (int i = 0; i < N; i++) {
        for (int j = i + 1; j < N; j++) {
            if (g1d[cnt] != 0) {
                if (((b >> i) & 1ull) ^ ((b >> j) & 1ull))
                    sum += g1d[cnt];
                else
                    sum -= g1d[cnt];
            }
            cnt++;
        }
    }
    return sum;
}

/* rzz.cu:121-156 (kernel body) for every amplitude; rzz.cu:173-206 launches
 * it over all 2^N amplitudes with the packed graph. */
void orc_cost_phase(double* sv, int N, double angle, const double* graph1d,
                    int is_first_layer, double init_amp) {
    const i64 n = 1ll << N;
#pragma omp parallel for schedule(static)
    for (i64 b = 0; b < n; b++) {
        double sum = pair_sum((u64)b, N, graph1d);
        double s, c;
        sincos(sum * angle / 2, &s, &c); /* rzz.cu:146 */
        if (is_first_layer) {            /* rzz.cu:148-150: write-only */
            sv[2 * b] = c * init_amp;
            sv[2 * b + 1] = s * init_amp;
        } else { /* rzz.cu:152-154 */
            double re = sv[2 * b], im = sv[2 * b + 1];
            sv[2 * b] = re * c - im * s;
            sv[2 * b + 1] = re * s + im * c;
        }
    }
}

/* rx.cu:24-28 bit_string: insert a 0 bit at position `target` */
static inline u64 insert_zero(u64 task, int target) {
    u64 mask = (1ull << target) - 1;
    return ((task >> target) << (target + 1)) | (task & mask);
}

/* rx.cu:32-53 pair update, rx.cu:278-281 applied target by target, rx.cu:121
 * host sincos(angle/2). */
void orc_multi_rotate_x(double* sv, int N, const int* targets, int gate_size,
                        double angle) {
    double s, c;
    sincos(angle / 2, &s, &c);
    const i64 half = 1ll << (N - 1);
    for (int g = 0; g < gate_size; g++) {
        const int t = targets[g];
#pragma omp parallel for schedule(static)
        for (i64 k = 0; k < half; k++) {
            u64 up = insert_zero((u64)k, t);
            u64 lo = up + (1ull << t);
            double q0r = sv[2 * up], q0i = sv[2 * up + 1];
            double q1r = sv[2 * lo], q1i = sv[2 * lo + 1];
            sv[2 * up] = q0r * c + q1i * s;
            sv[2 * up + 1] = q0i * c - q1r * s;
            sv[2 * lo] = q0i * s + q1r * c;
            sv[2 * lo + 1] = -q0r * s + q1i * c;
        }
    }
}

/* swap.cu:76-102 + swap.cu:173-187: for every pair s1<s2 of k-bit block
 * values and every index g with both blocks zero, exchange
 *   (s1<<in) + (s2<<out) + g   <->   (s1<<out) + (s2<<in) + g.
 * That is the involution "exchange the two bit blocks" of the index. */
void orc_swap_gate_conti(double* sv, int N, int swap_out, int swap_in, int num_swap) {
    const i64 n = 1ll << N;
    const u64 kmask = (1ull << num_swap) - 1;
#pragma omp parallel for schedule(static)
    for (i64 x = 0; x < n; x++) {
        u64 a = ((u64)x >> swap_out) & kmask; /* block at out */
        u64 b = ((u64)x >> swap_in) & kmask;  /* block at in  */
        if (a >= b) continue;                  /* visit each pair once, s1<s2 */
        u64 y = ((u64)x & ~(kmask << swap_out) & ~(kmask << swap_in)) |
                (a << swap_in) | (b << swap_out);
        double r = sv[2 * x], i = sv[2 * x + 1];
        sv[2 * x] = sv[2 * y];
        sv[2 * x + 1] = sv[2 * y + 1];
        sv[2 * y] = r;
        sv[2 * y + 1] = i;
    }
}

static inline void dswap(double* a, double* b) {
    double t = *a;
    *a = *b;
    *b = t;
}

/* swap.cu:27-50, literal */
void orc_mapping_after_swap_conti(double* graph, int N, int swap_out, int swap_in,
                                  int num_swap) {
    const int num = N;
    while (num_swap > 0) {
        for (int i = 0; i < num; i++) {
            if (i == swap_in || i == swap_out) continue;
            else if (i < swap_out)
                dswap(&graph[num * i + swap_in], &graph[num * i + swap_out]);
            else if (i > swap_out && i < swap_in)
                dswap(&graph[num * swap_out + i], &graph[num * i + swap_in]);
            else
                dswap(&graph[num * swap_out + i], &graph[num * swap_in + i]);
        }
        num_swap--;
        swap_in++;
        swap_out++;
    }
}

/* Weighted.cpp:97-108 (subcircuits of C qubits) and Weighted.cpp:115-138
 * (layer loop), with per-layer angles instead of the fixed pi/4. */
void orc_weighted_run(int N, int C, int P, const double* graph_upper,
                      const double* gammas, const double* betas, double* sv,
                      double* graph_final, int* label_map) {
    double* g = (double*)malloc(sizeof(double) * N * N);
    double* g1d = (double*)malloc(sizeof(double) * (N * (N - 1) / 2 + 1));
    int* lab = (int*)malloc(sizeof(int) * N);
    int nsub = 0, sizes[64], targets[64];
    memcpy(g, graph_upper, sizeof(double) * N * N);
    for (int i = 0; i < N; i++) lab[i] = i;
    for (int i = 0; i < N; i += C) sizes[nsub++] = (i + C <= N) ? C : N - i;
    for (int j = 0; j < C && j < N; j++) targets[j] = j; /* subcirs[0] */
    const double init_amp = orc_init_amp(N);              /* Weighted.cpp:93 */
    for (int p = 0; p < P; p++) {
        orc_upper_tri_to_1d(N, g, g1d); /* rzz.cu:181 */
        orc_cost_phase(sv, N, gammas[p], g1d, p == 0, init_amp);
        int swap_in = 0;
        for (int i = 0; i < nsub; i++) {
            orc_multi_rotate_x(sv, N, targets, sizes[i], betas[p]);
            if (i < nsub - 1) {
                swap_in += sizes[i];
                orc_swap_gate_conti(sv, N, 0, swap_in, sizes[i + 1]);
                orc_mapping_after_swap_conti(g, N, 0, swap_in, sizes[i + 1]);
                for (int m = 0; m < sizes[i + 1]; m++) {
                    int t = lab[m];
                    lab[m] = lab[swap_in + m];
                    lab[swap_in + m] = t;
                }
            }
        }
    }
    if (graph_final) memcpy(graph_final, g, sizeof(double) * N * N);
    if (label_map) memcpy(label_map, lab, sizeof(int) * N);
    free(g);
    free(g1d);
    free(lab);
}

/* The circuit in logical order.  S(z) is the pair-order sum of
 * rzz.cu:131-143, computed once (it does not change between layers without
 * relabelling); each layer then applies rzz.cu:146-154 and the mixer. */
void orc_qaoa_logical(int N, int P, const double* graph_upper, const double* gammas,
                      const double* betas, double* sv) {
    const i64 n = 1ll << N;
    double* S = (double*)malloc(sizeof(double) * n);
    int targets[64];
    for (int q = 0; q < N; q++) targets[q] = q;
    orc_cost_diag_S(N, graph_upper, S);
    const double init_amp = orc_init_amp(N);
    for (int p = 0; p < P; p++) {
        const double angle = gammas[p];
#pragma omp parallel for schedule(static)
        for (i64 b = 0; b < n; b++) {
            double s, c;
            sincos(S[b] * angle / 2, &s, &c);
            if (p == 0) {
                sv[2 * b] = c * init_amp;
                sv[2 * b + 1] = s * init_amp;
            } else {
                double re = sv[2 * b], im = sv[2 * b + 1];
                sv[2 * b] = re * c - im * s;
                sv[2 * b + 1] = re * s + im * c;
            }
        }
        orc_multi_rotate_x(sv, N, targets, N, betas[p]);
    }
    free(S);
}

void orc_cost_diag_S(int N, const double* graph_upper, double* S) {
    double* g1d = (double*)malloc(sizeof(double) * (N * (N - 1) / 2 + 1));
    orc_upper_tri_to_1d(N, graph_upper, g1d);
    const i64 n = 1ll << N;
#pragma omp parallel for schedule(static)
    for (i64 b = 0; b < n; b++) S[b] = pair_sum((u64)b, N, g1d);
    free(g1d);
}

/* C(z) = sum over cut edges of w.  Computed by doubling:
 * C(z + 2^k) = C(z) + sum_{i<k} w_ik (1 - 2 z_i) + sum_{i>k} w_ik  for z<2^k
 * (bits >= k of z are zero).  Exact for integer weights. */
void orc_cut_values(int N, const double* graph_upper, double* Cz) {
    Cz[0] = 0;
    for (int k = 0; k < N; k++) {
        const i64 half = 1ll << k;
        double above = 0;
        for (int i = k + 1; i < N; i++) above += graph_upper[k * N + i];
#pragma omp parallel for schedule(static)
        for (i64 z = 0; z < half; z++) {
            double d = above;
            for (int i = 0; i < k; i++) {
                double w = graph_upper[i * N + k];
                if (w != 0) d += ((z >> i) & 1) ? -w : w;
            }
            Cz[z + half] = Cz[z] + d;
        }
    }
}

double orc_expectation(const double* sv, int N, const double* graph_upper) {
    const i64 n = 1ll << N;
    double* Cz = (double*)malloc(sizeof(double) * n);
    orc_cut_values(N, graph_upper, Cz);
    long double acc = 0;
#pragma omp parallel for schedule(static) reduction(+ : acc)
    for (i64 z = 0; z < n; z++) {
        long double p = (long double)sv[2 * z] * sv[2 * z] +
                        (long double)sv[2 * z + 1] * sv[2 * z + 1];
        acc += p * Cz[z];
    }
    free(Cz);
    return (double)acc;
}

/* Multiply psi by exp(+i*gamma*S/2) (sign=+1) or its inverse (sign=-1). */
static void phase_apply(double* v, i64 n, const double* S, double gamma, int sign) {
#pragma omp parallel for schedule(static)
    for (i64 z = 0; z < n; z++) {
        double s, c;
        sincos(S[z] * gamma / 2, &s, &c);
        s *= sign;
        double re = v[2 * z], im = v[2 * z + 1];
        v[2 * z] = re * c - im * s;
        v[2 * z + 1] = re * s + im * c;
    }
}

/* RX(angle) on every qubit. */
static void mixer_apply(double* v, int N, double angle) {
    int targets[64];
    for (int q = 0; q < N; q++) targets[q] = q;
    orc_multi_rotate_x(v, N, targets, N, angle);
}

/* Adjoint differentiation of E = <psi|C|psi>:
 *   lambda = C psi at the end; walking layers backwards,
 *   dE/dbeta_k  =  Im <lambda| sum_q X_q |psi>   (after mixer k)
 *   dE/dgamma_k = -Im <lambda| S |psi>           (after cost k)
 * with psi and lambda both moved back through the exact inverse of each
 * layer (recompute, no stored states). */
void orc_energy_grad(int N, int P, const double* graph_upper, const double* gammas,
                     const double* betas, double* energy, double* grad_gamma,
                     double* grad_beta) {
    const i64 n = 1ll << N;
    double* S = (double*)malloc(sizeof(double) * n);
    double* Cz = (double*)malloc(sizeof(double) * n);
    double* psi = (double*)malloc(sizeof(double) * 2 * n);
    double* lam = (double*)malloc(sizeof(double) * 2 * n);
    orc_cost_diag_S(N, graph_upper, S);
    orc_cut_values(N, graph_upper, Cz);
    orc_qaoa_logical(N, P, graph_upper, gammas, betas, psi);
    long double e = 0;
#pragma omp parallel for schedule(static) reduction(+ : e)
    for (i64 z = 0; z < n; z++) {
        lam[2 * z] = Cz[z] * psi[2 * z];
        lam[2 * z + 1] = Cz[z] * psi[2 * z + 1];
        e += ((long double)psi[2 * z] * psi[2 * z] +
              (long double)psi[2 * z + 1] * psi[2 * z + 1]) * Cz[z];
    }
    *energy = (double)e;
    for (int k = P - 1; k >= 0; k--) {
        /* Im <lam|B|psi> = sum_q sum_z Im(conj(lam_z) psi_{z^q}) */
        long double gb = 0;
        for (int q = 0; q < N; q++) {
            const u64 bit = 1ull << q;
#pragma omp parallel for schedule(static) reduction(+ : gb)
            for (i64 z = 0; z < n; z++) {
                u64 y = (u64)z ^ bit;
                double lr = lam[2 * z], li = lam[2 * z + 1];
                double pr = psi[2 * y], pi = psi[2 * y + 1];
                gb += (long double)lr * pi - (long double)li * pr;
            }
        }
        grad_beta[k] = (double)gb;
        mixer_apply(psi, N, -betas[k]);
        mixer_apply(lam, N, -betas[k]);
        long double gg = 0;
#pragma omp parallel for schedule(static) reduction(+ : gg)
        for (i64 z = 0; z < n; z++) {
            double lr = lam[2 * z], li = lam[2 * z + 1];
            double pr = psi[2 * z], pi = psi[2 * z + 1];
            gg += ((long double)lr * pi - (long double)li * pr) * S[z];
        }
        grad_gamma[k] = -(double)gg;
        if (k > 0) {
            phase_apply(psi, n, S, gammas[k], -1);
            phase_apply(lam, n, S, gammas[k], -1);
        }
    }
    free(S);
    free(Cz);
    free(psi);
    free(lam);
}

void orc_state_fill(double* sv, int N, double re, double im) {
    const i64 n = 1ll << N;
#pragma omp parallel for schedule(static)
    for (i64 z = 0; z < n; z++) {
        sv[2 * z] = re;
        sv[2 * z + 1] = im;
    }
}

void orc_layer_chunk(double* sv, int N, const double* graph1d, double gamma, double beta,
                     int first_layer, int chunk, int nchunks, double* t_cost, double* t_rx) {
    const i64 per = (1ll << N) / nchunks, pper = (1ll << (N - 1)) / nchunks;
    const double amp = orc_init_amp(N);
    const i64 a0 = (i64)chunk * per, p0 = (i64)chunk * pper;
    double t0 = omp_get_wtime();
    /* rzz.cu:121-156 on amplitudes [a0, a0 + per) */
#pragma omp parallel for schedule(static)
    for (i64 b = a0; b < a0 + per; b++) {
        double sum = pair_sum((u64)b, N, graph1d);
        double sn, cs;
        sincos(sum * gamma / 2, &sn, &cs);
        if (first_layer) {
            sv[2 * b] = cs * amp;
            sv[2 * b + 1] = sn * amp;
        } else {
            double re = sv[2 * b], im = sv[2 * b + 1];
            sv[2 * b] = re * cs - im * sn;
            sv[2 * b + 1] = re * sn + im * cs;
        }
    }
    double t1 = omp_get_wtime();
    /* rx.cu:32-53 for every qubit on pairs [p0, p0 + pper) */
    double s, c;
    sincos(beta / 2, &s, &c);
    for (int t = 0; t < N; t++) {
#pragma omp parallel for schedule(static)
        for (i64 k = p0; k < p0 + pper; k++) {
            u64 up = insert_zero((u64)k, t);
            u64 lo = up + (1ull << t);
            double q0r = sv[2 * up], q0i = sv[2 * up + 1];
            double q1r = sv[2 * lo], q1i = sv[2 * lo + 1];
            sv[2 * up] = q0r * c + q1i * s;
            sv[2 * up + 1] = q0i * c - q1r * s;
            sv[2 * lo] = q0i * s + q1r * c;
            sv[2 * lo + 1] = -q0r * s + q1i * c;
        }
    }
    double t2 = omp_get_wtime();
    *t_cost = t1 - t0;
    *t_rx = t2 - t1;
}

void orc_permute_qubits(const double* src, double* dst, int N, const int* perm) {
    const i64 n = 1ll << N;
#pragma omp parallel for schedule(static)
    for (i64 x = 0; x < n; x++) {
        u64 y = 0;
        for (int b = 0; b < N; b++) y |= (((u64)x >> b) & 1ull) << perm[b];
        dst[2 * y] = src[2 * x];
        dst[2 * y + 1] = src[2 * x + 1];
    }
}
