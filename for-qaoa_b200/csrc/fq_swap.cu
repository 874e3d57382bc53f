// fq_swap.cu -- qubit-block exchange in HBM (replaces swap_gate_conti's
// single-device path, src/swap.cu:104-202, kernel :76-102).
//
// Exchanging bit blocks [o, o+k) and [i, i+k) of every index is, for each
// value of the other bits, a transpose of a 2^k x 2^k matrix of "elements"
// (runs of 2^o contiguous amplitudes) whose rows are 2^i apart.  The
// reference walks a host-built table of all (s1, s2) block-value pairs and
// swaps one 16-byte amplitude per thread, so one side of every access is
// strided.  Here each CTA owns a PAIR of 2^a x 2^a sub-tiles, (I, J) and its
// mirror (J, I) (I, J = high k-a bits of each block), loads both with rows
// of >= 2^(a + eb) contiguous amplitudes, and writes each one transposed
// into the other's place through a padded shared tile, so reads and writes
// are both row-contiguous.  Diagonal sub-tiles (I == J) transpose in place.
#include <math.h>

#include <algorithm>

#include "fq_ctx.h"

namespace fq {

struct SwapArgs {
    double2* sv;
    int N, o, i, k;
    int eb;      // element bits kept inside a tile row (<= o)
    int a;       // sub-tile bits taken from each block
    int m;       // bits [o+k, o+k+m) also kept inside a row (only when a == k)
    int nob;     // "other" bits: [eb,o), [o+k+m,i), [i+k,N)
    i64 npairs;  // sub-tile pairs (I <= J)
    i64 nitems;
};

__global__ void __launch_bounds__(256) k_swap_blocks(const SwapArgs S) {
    extern __shared__ __align__(16) double2 sm[];
    // A row holds the element bits e (eb), the out-block low bits x (a) and
    // the free bits f above the out block (m): 2^(eb+a+m) amplitudes,
    // contiguous when o <= 6 and a == k.
    const int rowlen = 1 << (S.a + S.eb + S.m);
    const int rows = 1 << S.a;
    const int stride = rowlen + 1;  // padding keeps the transposed read conflict-free
    const int tsize = rows * rowlen;
    double2* t0 = sm;
    double2* t1 = sm + rows * stride;
    const int n1 = S.o - S.eb, n2 = S.i - S.o - S.k - S.m;
    const int xeb = S.a + S.eb;  // bits of (e, x) in a row index
    for (i64 item = blockIdx.x; item < S.nitems; item += gridDim.x) {
        const i64 oi = item & ((1ll << S.nob) - 1);
        const i64 p = item >> S.nob;
        i64 J = (i64)((sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
        while (J * (J + 1) / 2 > p) J--;
        while ((J + 1) * (J + 2) / 2 <= p) J++;
        const i64 I = p - J * (J + 1) / 2;
        const i64 base = ((oi & ((1ll << n1) - 1)) << S.eb) |
                         (((oi >> n1) & ((1ll << n2) - 1)) << (S.o + S.k + S.m)) |
                         ((oi >> (n1 + n2)) << (S.i + S.k));
        const i64 bIJ = base | (I << (S.o + S.a)) | (J << (S.i + S.a));
        const i64 bJI = base | (J << (S.o + S.a)) | (I << (S.i + S.a));
        const bool diag = (I == J);
        // Load: row y of a sub-tile = in-block low bits y; a row holds the
        // out-block low bits x and the element bits e (contiguous when o <= 6,
        // runs of 2^eb = 64 amplitudes otherwise).
        for (int idx = threadIdx.x; idx < tsize; idx += 256) {
            const int y = idx >> (xeb + S.m), xe = idx & (rowlen - 1);
            const int f = xe >> xeb, x = (xe >> S.eb) & ((1 << S.a) - 1);
            const i64 off = (xe & ((1 << S.eb) - 1)) + ((i64)x << S.o) +
                            ((i64)f << (S.o + S.k)) + ((i64)y << S.i);
            t0[y * stride + xe] = __ldcs(S.sv + bIJ + off);
            if (!diag) t1[y * stride + xe] = __ldcs(S.sv + bJI + off);
        }
        __syncthreads();
        // Element (x, y) of (I, J) lands at (y, x) of (J, I), and vice versa.
        for (int idx = threadIdx.x; idx < tsize; idx += 256) {
            const int yd = idx >> (xeb + S.m), xe = idx & (rowlen - 1);
            const int f = xe >> xeb, xd = (xe >> S.eb) & ((1 << S.a) - 1);
            const int e = xe & ((1 << S.eb) - 1);
            const int src = xd * stride + (f << xeb) + (yd << S.eb) + e;
            const i64 off = e + ((i64)xd << S.o) + ((i64)f << (S.o + S.k)) + ((i64)yd << S.i);
            __stcs(S.sv + bJI + off, t0[src]);
            if (!diag) __stcs(S.sv + bIJ + off, t1[src]);
        }
        __syncthreads();
    }
}

}  // namespace fq

using namespace fq;

extern "C" int fq_swap_blocks(fq_ctx* ctx, void* sv, int N, int swap_out, int swap_in,
                              int num_swap) {
    FQ_TRY(validate_ctx(ctx));
    FQ_CHECK(sv != nullptr && ((uintptr_t)sv & 15) == 0, FQ_ERR_INVALID, "bad state pointer");
    FQ_CHECK(N >= 1 && N <= kMaxQubits, FQ_ERR_INVALID, "N=%d out of range", N);
    FQ_CHECK(num_swap >= 0 && swap_out >= 0 && swap_out + num_swap <= swap_in &&
                 swap_in + num_swap <= N,
             FQ_ERR_INVALID,
             "block swap needs out + k <= in and in + k <= N (out=%d in=%d k=%d N=%d)", swap_out,
             swap_in, num_swap, N);
    if (num_swap == 0) return FQ_OK;
    SwapArgs S;
    S.sv = (double2*)sv;
    S.N = N;
    S.o = swap_out;
    S.i = swap_in;
    S.k = num_swap;
    S.eb = std::min(swap_out, 6);
    S.a = std::min(num_swap, std::max(0, (10 - S.eb) / 2));
    // A small block (the whole block in one sub-tile) leaves rows short;
    // the free bits right above the out block fill them up to 2^10
    // amplitudes per sub-tile (a swap of 2-qubit blocks at bit 0 took 7.9 ms
    // at N=26 with 4-amplitude rows).
    S.m = S.a == num_swap ? std::max(0, std::min(swap_in - swap_out - num_swap,
                                                  10 - 2 * S.a - S.eb))
                          : 0;
    S.nob = (swap_out - S.eb) + (swap_in - swap_out - num_swap - S.m) +
            (N - swap_in - num_swap);
    const i64 M = 1ll << (num_swap - S.a);
    S.npairs = M * (M + 1) / 2;
    S.nitems = S.npairs << S.nob;
    const size_t smem = sizeof(double2) * 2 * (1 << S.a) * ((1 << (S.a + S.eb + S.m)) + 1);
    const i64 grid = std::min<i64>(S.nitems, (i64)ctx->num_sms * 8);
    const int tok = prof_begin(ctx);
    k_swap_blocks<<<(unsigned)grid, 256, smem, ctx->stream>>>(S);
    FQ_CUDA(cudaGetLastError());
    // Amplitudes whose two blocks hold equal values stay put.
    prof_end(ctx, tok, FQ_KIND_SWAP, 32.0 * (double)(1ull << N) * (1.0 - 1.0 / (1ull << num_swap)));
    ctx->launches++;
    return FQ_OK;
}
