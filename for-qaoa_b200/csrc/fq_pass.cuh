// fq_pass.cuh -- the streaming tile pass every state sweep is built from.
//
// A pass walks the 2^N state in tiles of 2^12 amplitudes (64 KB).  A tile
// is every amplitude whose "tile bits" vary while all other ("fixed") index
// bits are held: tile bits 0..l-1 are physical bits 0..l-1 (contiguous rows
// of 2^l amplitudes, for coalescing) and tile bits l..11 are physical bits
// a..a+11-l.  With l = 12 the tile is 4096 contiguous amplitudes.  Within a
// tile a pass can
//   - multiply by (or, in layer 0, write) the QAOA cost phase,
//   - apply RX to any subset of the 12 tile qubits,
//   - accumulate <C> = sum |psi|^2 C(z),
// so one HBM read + write covers what the reference does in separate cost,
// RX-chunk and block-swap sweeps (src/rzz.cu:121-156, src/rx.cu:56-87,
// src/swap.cu:76-102): high qubits are brought on chip by the strided tile
// instead of being transposed in HBM.
//
// Thread layout: 256 threads x 16 amplitudes in registers.  The 16 register
// slots of a thread are 4 tile bits; RX on those 4 qubits is register-local.
// Three layouts rotate which 4 tile bits are register bits; moving between
// them goes through a shared buffer padded by one slot every 16 (pslot: 68
// KB per tile), which keeps every quarter-warp's 16-byte accesses in
// distinct banks in all three layouts:
//   L0 (load):       regs = tile bits 8..11, lanes = 0..4,  warps = 5..7
//   L1 (store):      regs = tile bits 4..7,  lanes = 0..3,8, warps = 9..11
//   L2:              regs = tile bits 0..3,  lanes = 4..8,  warps = 9..11
// L0 and L1 both keep the row bits on consecutive lanes, so a tile is loaded
// in L0 and stored from L1 without a layout change of its own: 12 qubits
// take two exchanges (L0 -> L2 -> L1), 8 take one (L0 -> L1).  Passes that
// alternate (ALT, ALTM) load their odd tiles in L1 and store them from L0.
// A single qubit among tile bits 0..3 is rotated with warp shuffles instead
// (those bits are lane bits in L0 and L1), so a strided pass with 128-byte
// rows (9 qubits, tile bits 3..11) also needs one exchange.
//
// Cut value of an amplitude (exact in integers for integer weights):
//   C(z) = K(fixed) + C_TT(tile bits) + sum_{u in tile} z_u e_u(fixed)
// with K = cut inside the fixed bits + sum_m z_m D_m, D_m = sum_{u in tile}
// w_um, and e_u = R_u - 2 sum_m w_um z_m, R_u = sum_{m fixed} w_um.  C_TT is
// split into the thread's 8 tile bits (constant per thread), the 4 register
// bits (16-entry table) and their cross term (4 per-thread coefficients), so
// each amplitude costs a few integer adds.
#pragma once

#include <type_traits>

#include "fq_common.cuh"

namespace fq {

constexpr int kTileBits = 12;
constexpr int kTile = 1 << kTileBits;
constexpr int kPassThreads = 256;
constexpr int kRegs = 16;
constexpr int kMaxFixed = kMaxQubits - kTileBits;  // 21

// Phase modes
enum { PH_NONE = 0, PH_MUL = 1, PH_INIT = 2 };
// Extra outputs: none, <C> partial sums, cut value of every amplitude
enum { EX_NONE = 0, EX_ENERGY = 1, EX_DIAG = 2, EX_COSTATE = 3 };
// EX_COSTATE: <C> partial sums and the costate lambda = C psi written to sv2.
// Round schedules: L0 only; L0 -> L1; L0 -> L2 -> L1 (see header comment).
enum { SC_L0 = 0, SC_L01 = 1, SC_L021 = 2 };

// Schedule a target mask needs.
__host__ __device__ inline int schedule_for(unsigned tmask) {
    const unsigned lo = tmask & 15u, mid = (tmask >> 4) & 15u;
    if (lo & (lo - 1)) return SC_L021;  // two or more of tile bits 0..3
    if (mid) return SC_L01;
    return SC_L0;
}
// Gate modes: reduced RX [[1,-it],[-it,1]] (t = tan(b/2)), reduced RX
// [[u,-i],[-i,u]] (u = cot(b/2)), the full RX of src/rx.cu:47-50.
enum { GM_NONE = 0, GM_TAN = 1, GM_COT = 2, GM_FULL = 3 };

struct PassArgs {
    double2* sv;
    double2* sv2;         // second vector: costate output (EX_COSTATE)
    const void* w;        // N*N symmetric weights (int32 or float64), device
    // Integer path: the phase of cut value c.  nhi == 0: one table in global
    // memory, ptab[c - cmin] = scale * exp(i*gamma*(2c - W)/2).  nhi > 0:
    // powers of z = exp(i*gamma) in two small tables copied to shared
    // memory, ptab[j] = z^j (j < 32) and ptab[32 + h] = z^(dlo + 32h), so
    // z^d = hi[(d - dlo) >> 5] * lo[(d - dlo) & 31] for d in [dlo, dlo + ntab)
    // and phase(c) = ph0 * z^c with ph0 = scale * exp(-i*gamma*W/2).
    const double2* ptab;
    double* partial;      // <C> partial sums, one per CTA
    double* diag;         // cut-value output (EX_DIAG)
    i64 ntiles;
    int N, l, a;
    unsigned tmask;  // RX targets among the 12 tile bits
    int cmin, ntab, nhi, dlo;
    double ph0x, ph0y;  // ph0 of the two-level table (see ptab)
    double gx;       // t or u of the reduced gate
    double gx2;      // fused passes (GM2 != GM_NONE): t or u of the next layer's gate
    double c, s;     // cos, sin of angle/2 for GM_FULL
    double gamma;    // FP64 phase path: exp(i*(2C-W)*gamma/2)
    double W;        // total weight
    double scale;    // multiplies the phase
    int tree;        // FP64 weights: phases by product tree (else one sincos per amplitude)
    double sc0, f2;  // adjoint passes: scale of the inner products at the pass's start, and
                     // the factor (f^2) it gains with every reduced rotation
    double f2b;      // fused adjoint passes: f^2 of the earlier layer's gate (A.gx2)
    int pf_dist;     // prefetch the tile pf_dist grid-strides ahead into L2 (0 = off)
    i64 goff;        // shard of a larger state: global index of sv[0] (enters cut values only)
    // Non-fused PH_MUL passes: RX (full form, pc = cos, ps = sin of angle/2)
    // on the layout-L0 register bits pre_mask (tile bits 8..11) of each
    // loaded tile before the phase; a shard's exchange brings the qubits it
    // swaps in to those bits of the next layer's first pass (0 = none).
    unsigned pre_mask;
    double pc, ps;
    // Cut constants of every tile of this pass's geometry, kTcutStride WT per
    // tile (K, then e_0..e_11; k_tile_cuts), or null: each tile computes its
    // own (CutTables::tile, warps 0 and 1, then a barrier).
    const void* tcut;
    int* err;        // device error flag (bounded waits that gave up)
};

__device__ __forceinline__ int tile_phys(int j, int l, int a) { return j < l ? j : a + j - l; }

constexpr int kPhaseLo = 32;     // low-part entries of the two-level phase table
constexpr int kPhaseHiMax = 512; // high-part entries kept in shared memory at most
// Layer tables of the two-level kind built in one launch, kTableStride
// entries apart in the context's table buffer (kMaxPhaseTable entries).
constexpr int kTableStride = kPhaseLo + kPhaseHiMax;
constexpr int kMaxTableLayers = 64;
static_assert(kTableStride * kMaxTableLayers <= kMaxPhaseTable, "layer tables fit the buffer");

// Shared-memory bytes reserved for the two-level phase table.
__host__ __device__ inline size_t phase_smem_bytes() {
    return sizeof(double2) * (kPhaseLo + kPhaseHiMax);
}

// Copy the two-level phase table into shared memory (all threads).
__device__ __forceinline__ void load_phase_tables(const PassArgs& A, double2* smtab, int tid,
                                                  int nthreads) {
    if (A.nhi > 0)
        for (int i = tid; i < kPhaseLo + A.nhi; i += nthreads) smtab[i] = A.ptab[i];
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// z^d from the two-level table in shared memory (nhi > 0).
__device__ __forceinline__ double2 tab_pow(const PassArgs& A, const double2* smtab, int d) {
    const int ti = min(max(d - A.dlo, 0), A.ntab - 1);  // guards the table read only
    return cmul(smtab[kPhaseLo + (ti >> 5)], smtab[ti & 31]);
}

// Phase (times the layer's scale) of a cut value on the integer path.
__device__ __forceinline__ double2 int_phase(const PassArgs& A, const double2* smtab, int cr) {
    if (A.nhi > 0) return cmul(make_double2(A.ph0x, A.ph0y), tab_pow(A, smtab, cr));
    const int ti = min(max(cr - A.cmin, 0), A.ntab - 1);  // guards the table read only
    return __ldg(A.ptab + ti);
}

// Swizzled slot of tile index t in a 64 KB exchange buffer (the TMA pass,
// whose landed stage is the buffer): bits 0..2 XORed with bits 4..6.
__device__ __forceinline__ int xslot(int t) { return t ^ ((t >> 4) & 7); }
// Padded slot of tile index t (k_pass, k_pass_dual): one empty 16-byte slot
// after every 16, so every quarter-warp's accesses fall in distinct banks in
// all three layouts, and -- unlike the XOR swizzle -- the slots of a
// thread's 16 registers are its first slot plus constants (the register
// bits have strides of 16 or more tile indices, or sit in bits 0..3 of a
// multiple of 16), which the compiler folds into the access instructions.
__device__ __forceinline__ int pslot(int t) { return t + (t >> 4); }
constexpr int kXTile = kTile + kTile / 16;  // slots of a padded buffer

template <int GM>
__device__ __forceinline__ void rx_pair(double2& p, double2& q, double g, double c, double s) {
    const double2 a = p, b = q;
    if (GM == GM_TAN) {
        p.x = fma(g, b.y, a.x);
        p.y = fma(-g, b.x, a.y);
        q.x = fma(g, a.y, b.x);
        q.y = fma(-g, a.x, b.y);
    } else if (GM == GM_COT) {
        p.x = fma(g, a.x, b.y);
        p.y = fma(g, a.y, -b.x);
        q.x = fma(g, b.x, a.y);
        q.y = fma(g, b.y, -a.x);
    } else {  // src/rx.cu:47-50
        p.x = a.x * c + b.y * s;
        p.y = a.y * c - b.x * s;
        q.x = a.y * s + b.x * c;
        q.y = -a.x * s + b.y * c;
    }
}

// RX on the register bits selected by m4 (uniform across the block).
template <int GM>
__device__ __forceinline__ void rx_regs(double2 (&v)[kRegs], unsigned m4, double g, double c,
                                        double s) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if ((m4 >> k) & 1u) {
#pragma unroll
            for (int r = 0; r < kRegs; r++)
                if (!((r >> k) & 1)) rx_pair<GM>(v[r], v[r | (1 << k)], g, c, s);
        }
    }
}

// One amplitude of an RX pair from its own value m and its partner's q (the
// gate is symmetric in the pair: self' = a*self - i*b*partner).
template <int GM>
__device__ __forceinline__ double2 rx_self(double2 m, double2 q, double g, double c, double s) {
    if (GM == GM_TAN) return make_double2(fma(g, q.y, m.x), fma(-g, q.x, m.y));
    if (GM == GM_COT) return make_double2(fma(g, m.x, q.y), fma(g, m.y, -q.x));
    return make_double2(m.x * c + q.y * s, m.y * c - q.x * s);
}

// RX on a qubit held in lane bit j: every lane updates its own amplitude
// from its partner's.
template <int GM>
__device__ __forceinline__ void rx_lane(double2 (&v)[kRegs], int j, double g, double c, double s) {
    const unsigned lm = 1u << j;
#pragma unroll
    for (int r = 0; r < kRegs; r++) {
        double2 q;
        q.x = __shfl_xor_sync(0xffffffffu, v[r].x, lm);
        q.y = __shfl_xor_sync(0xffffffffu, v[r].y, lm);
        v[r] = rx_self<GM>(v[r], q, g, c, s);
    }
}

// x through an empty volatile asm inside a tile loop: the compiler must take
// it as a new value there, so what is derived from it (addresses) is
// recomputed where it is used instead of being hoisted out of the loop and
// held in registers the amplitudes of a thread need (the adjoint pass).
__device__ __forceinline__ i64 opaque(i64 x) {
    asm volatile("" : "+l"(x));
    return x;
}

// Offset of register slot r from the strides b0..b3 of its 4 tile bits.
__device__ __forceinline__ i64 offr(int r, i64 b0, i64 b1, i64 b2, i64 b3) {
    return ((r & 1) ? b0 : 0) + ((r & 2) ? b1 : 0) + ((r & 4) ? b2 : 0) + ((r & 8) ? b3 : 0);
}

// Tile index held in register r under layout L (see header comment).
template <int L>
__device__ __forceinline__ int lay_index(int tid, int r) {
    const int lane = tid & 31, warp = tid >> 5;
    if (L == 0) return tid | (r << 8);
    if (L == 1) return (lane & 15) | ((lane >> 4) << 8) | (warp << 9) | (r << 4);
    return (lane << 4) | (warp << 9) | r;
}

// Barrier of one 256-thread group (named barrier 1 + g; 0 is __syncthreads).
__device__ __forceinline__ void group_sync(int g) {
    asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(kPassThreads) : "memory");
}

// Layouts L1 and L2 both put tile bits 9..11 on the warp index, so a change
// between them stays inside each warp's 512-amplitude region of buf
// (neither the padding nor the TMA pass's swizzle, which permutes bits 0..2,
// moves a slot out of it): a warp barrier is enough.  Such an
// exchange must follow reads of buf in L1 or L2 (the warp's own region), as
// every schedule here does; exchanges from or to L0 cross warps and use the
// block barrier.
// PAIR: the CTA holds two 256-thread groups, each on its own tile and
// buffer; the block barrier is then the group's named barrier.
template <bool PAIR>
__device__ __forceinline__ void tile_sync(int grp) {
    if (PAIR)
        group_sync(grp);
    else
        __syncthreads();
}

template <int LF, int LT, bool PAIR = false>
__device__ __forceinline__ void buf_sync(int grp = 0) {
    if (LF != 0 && LT != 0)
        __syncwarp();
    else
        tile_sync<PAIR>(grp);
}

// First padded slot of a thread's registers in layout L, taken through an
// empty volatile asm so that it is recomputed (two or three integer ops) at
// each exchange instead of being kept in a register across the tile loop.
// The slot of register r is this plus pslot(lay_index<L>(0, r)), a constant:
// pslot is additive over the thread part and the register part of a tile
// index in every layout.
template <int L>
__device__ __forceinline__ int pbase(int tid) {
    int b = pslot(lay_index<L>(tid, 0));
    asm volatile("" : "+r"(b));
    return b;
}

// Registers from layout LF to LT through buf.  Each thread writes its own
// LF slots and, after the barrier, reads its own LT slots.  wait_readers
// adds a barrier before the writes, which only a change of layout needs:
// an exchange that writes the layout the thread last read (the previous
// exchange's LT, with no partner reads since, or those behind
// exchange_lane's warp barrier) writes slots that no other thread reads
// until the next barrier, and skips it.
template <int LF, int LT, bool PAIR = false, bool PAD = true>
__device__ __forceinline__ void exchange(double2 (&v)[kRegs], double2* buf, int tid,
                                         bool wait_readers = true, int grp = 0) {
    if (wait_readers) buf_sync<LF, LT, PAIR>(grp);  // previous readers of buf are done
    if (PAD) {
        double2* const wb = buf + pbase<LF>(tid);
#pragma unroll
        for (int r = 0; r < kRegs; r++) wb[pslot(lay_index<LF>(0, r))] = v[r];
    } else {
#pragma unroll
        for (int r = 0; r < kRegs; r++) buf[xslot(lay_index<LF>(tid, r))] = v[r];
    }
    buf_sync<LF, LT, PAIR>(grp);
    if (PAD) {
        const double2* const rb = buf + pbase<LT>(tid);
#pragma unroll
        for (int r = 0; r < kRegs; r++) v[r] = rb[pslot(lay_index<LT>(0, r))];
    } else {
#pragma unroll
        for (int r = 0; r < kRegs; r++) v[r] = buf[xslot(lay_index<LT>(tid, r))];
    }
}

// exchange<LF, LT> that also applies RX on the qubit of lane bit j (a
// single target among tile bits 0..3, which is lane bit j in layouts L0 and
// L1 alike): each thread reads its own slots and its partner lane's
// (tid ^ 2^j) and combines them as rx_lane does, 16 more 16-byte shared
// loads in place of rx_lane's 64 shuffles.  The rotation then takes effect
// after the exchange instead of before it, which is the same state: it acts
// on another qubit than the register rounds around it.  The closing warp
// barrier keeps a partner's slots unwritten until both lanes have read them,
// whatever the caller writes next.  On B200 at N=30 the layer-0 pass takes
// 5.16-5.29 ms with it against 5.39-5.42 with rx_lane; the fused passes
// measured no faster with it (A/B in one call) and use exchange_lanet.
template <int LF, int LT, int GM, bool PAIR = false>
__device__ __forceinline__ void exchange_lane(double2 (&v)[kRegs], double2* buf, int tid,
                                              bool wait_readers, int grp, int j, double g,
                                              double c, double s) {
    if (wait_readers) buf_sync<LF, LT, PAIR>(grp);
    double2* const wb = buf + pbase<LF>(tid);
#pragma unroll
    for (int r = 0; r < kRegs; r++) wb[pslot(lay_index<LF>(0, r))] = v[r];
    buf_sync<LF, LT, PAIR>(grp);
    const double2* const rb = buf + pbase<LT>(tid);
    const double2* const qb = buf + pbase<LT>(tid ^ (1 << j));
#pragma unroll
    for (int r = 0; r < kRegs; r++) {
        const int o = pslot(lay_index<LT>(0, r));
        v[r] = rx_self<GM>(rb[o], qb[o], g, c, s);
    }
    __syncwarp();
}

// exchange<LF, LT> preceded by RX on the qubit of lane bit j, with half of
// rx_lane's shuffles: the two lanes of a pair (lane bit j = 0, 1) trade the
// registers whose bit 0 differs from their lane bit (8 values each way),
// after which each register pair (r, r|1) holds the lane qubit's two
// amplitudes of one register index and is rotated in place, by rx_lane's
// own arithmetic.  Every value then goes to the slot of the thread and
// register that held it before the trade.  A partner's slots written here
// are those whose values it has just sent, so its reads of them are done:
// the leading-barrier rule of exchange holds as before.  On B200 at N=30,
// p=5: fused passes 8.82-8.86 against 8.94-9.02 ms with rx_lane, 65.0-65.3
// against 64.4-64.6 layers/s (A/B in one call, bit-identical states).
template <int LF, int LT, int GM, bool PAIR = false>
__device__ __forceinline__ void exchange_lanet(double2 (&v)[kRegs], double2* buf, int tid,
                                               bool wait_readers, int grp, int j, double g,
                                               double c, double s) {
    const unsigned lm = 1u << j;
    const bool hi = (tid >> j) & 1;
#pragma unroll
    for (int r = 0; r < kRegs; r += 2) {
        const double2 keep = hi ? v[r | 1] : v[r], send = hi ? v[r] : v[r | 1];
        double2 q;
        q.x = __shfl_xor_sync(0xffffffffu, send.x, lm);
        q.y = __shfl_xor_sync(0xffffffffu, send.y, lm);
        v[r] = rx_self<GM>(keep, q, g, c, s);      // this lane's amplitude of register r|hi
        v[r | 1] = rx_self<GM>(q, keep, g, c, s);  // the partner's
    }
    if (wait_readers) buf_sync<LF, LT, PAIR>(grp);
    const int d = hi ? pslot(lay_index<LF>(0, 1)) : 0;
    double2* const wk = buf + pbase<LF>(tid) + d;
    double2* const wp = buf + pbase<LF>(tid ^ (int)lm) + d;
#pragma unroll
    for (int r = 0; r < kRegs; r += 2) {
        const int o = pslot(lay_index<LF>(0, r));
        wk[o] = v[r];
        wp[o] = v[r | 1];
    }
    buf_sync<LF, LT, PAIR>(grp);
    const double2* const rb = buf + pbase<LT>(tid);
#pragma unroll
    for (int r = 0; r < kRegs; r++) v[r] = rb[pslot(lay_index<LT>(0, r))];
}

constexpr int kWfStride = 21;  // row stride of the compact weight tables (odd: no bank conflicts)
static_assert(kWfStride >= kMaxFixed, "compact weight rows hold every fixed bit");

// Physical bit of fixed (non-tile) index i, ascending.
__device__ __forceinline__ int fixed_phys(int i, int l, int a) {
    const int nmid = a - l;
    return i < nmid ? l + i : a + (kTileBits - l) + (i - nmid);
}

// Offset of tile index t (12 bits) from the tile's base amplitude.
__device__ __forceinline__ i64 tile_off(int t, int l, int a) {
    return (i64)(t & ((1 << l) - 1)) | ((i64)(t >> l) << a);
}

// Shared-memory layout of k_pass after its padded exchange buffer (which
// also holds the N*N weights while the kernel sets up).
template <typename WT>
struct PassSmem {
    static constexpr size_t red = 0;                                // 16 double
    static constexpr size_t ke = red + 16 * sizeof(double);         // 2 groups x 2 x 32 WT
    static constexpr size_t creg = ke + 128 * sizeof(WT);           // 2 x 16 WT (L0, L1)
    static constexpr size_t Dm = creg + 32 * sizeof(WT);            // 24 WT
    static constexpr size_t Ru = Dm + 24 * sizeof(WT);              // 16 WT
    static constexpr size_t wf = Ru + 16 * sizeof(WT);              // kMaxFixed x kWfStride
    static constexpr size_t wu = wf + kMaxFixed * kWfStride * sizeof(WT);  // 12 x kWfStride
    static constexpr size_t thrc = wu + kTileBits * kWfStride * sizeof(WT);  // 2 x 5 x 256 WT
    static constexpr size_t qtab = (thrc + 10 * kPassThreads * sizeof(WT) + 15) & ~(size_t)15;
    static constexpr size_t smtab = qtab + 32 * sizeof(double2);    // after 2 x 16 qtab
    static constexpr size_t bytes = smtab + sizeof(double2) * (kPhaseLo + kPhaseHiMax);
};

// Shared-memory bytes k_pass needs (independent of N: the weights are
// staged in the exchange buffer); a paired CTA has two exchange buffers.
template <typename WT>
__host__ __device__ inline size_t pass_smem_bytes(int, bool pair = false) {
    return sizeof(double2) * kXTile * (pair ? 2 : 1) + PassSmem<WT>::bytes;
}

// Cut value of register slot r: c_r = cbase + creg[r] + sum_k r_k g_k, so
// its phase factors as phase(c_r) = P * Q_r * prod_k E_k^(r_k) with
// P = phase(cbase), Q_r = z^creg[r] (per pass, shared memory) and
// E_k = z^g_k, z = exp(i*gamma): 5 table lookups (or sincos) per thread and
// tile instead of 16.  The products run over four groups of four slots:
// B_q = P * E2^(q&1) * E3^(q>>1), then B_q {1, E0, E1, E0 E1} for the
// group's slots, each times Q_r: 48 complex products per thread where
// multiplying P * Q_r in and then E_k into the slots with bit k set takes
// 64 (on B200 at N=30, p=5, fused passes: 8.73-8.96 against 9.12-9.21 ms
// in one call, 9.46-9.49 against 9.63-9.68 in another, on a box with lower
// clocks).  PH_INIT writes the phase, PH_MUL multiplies it in
// (src/rzz.cu:153-154).
template <int PH>
__device__ __forceinline__ void phase_tree(double2 (&v)[kRegs], double2 P, const double2* qt,
                                           double2 E0, double2 E1, double2 E2, double2 E3) {
    const double2 E01 = cmul(E0, E1);
    const double2 B1 = cmul(P, E2);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const double2 B = q == 0 ? P : q == 1 ? B1 : q == 2 ? cmul(P, E3) : cmul(B1, E3);
        const double2 T[4] = {B, cmul(B, E0), cmul(B, E1), cmul(B, E01)};
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int r = 4 * q + i;
            const double2 ph = cmul(T[i], qt[r]);
            v[r] = (PH == PH_INIT) ? ph : cmul(v[r], ph);
        }
    }
}

// Shared-memory tables of the cut decomposition for one pass geometry.
template <typename WT>
struct CutTables {
    WT* ke;        // 2 x 32 per group, double-buffered per tile: [0] = K, [1+u] = e_u
    WT* creg;      // 16 per layout (L0, then L1): cut among the 4 register bits
    WT* Dm;        // nF: sum of weights between fixed bit m and the tile bits
    WT* Ru;        // 12: sum of weights between tile bit u and the fixed bits
    WT* wf;        // wf[i * kWfStride + j] = w(fixed i, fixed j)
    WT* wu;        // wu[u * kWfStride + j] = w(tile u, fixed j)
    WT* thrc;      // 5 x 256 per-thread constants per layout (L0, then L1):
                   // [0] cut among the thread's 8 tile bits (plus their
                   // edges to set register bits), [1+k] = f_k, the thread's
                   // part of g_k
    double2* qtab; // 16 per layout: z^creg[r], z = exp(i*gamma) (phase passes)

    __device__ CutTables(unsigned char* sm) {
        using SM = PassSmem<WT>;
        ke = reinterpret_cast<WT*>(sm + SM::ke);
        creg = reinterpret_cast<WT*>(sm + SM::creg);
        Dm = reinterpret_cast<WT*>(sm + SM::Dm);
        Ru = reinterpret_cast<WT*>(sm + SM::Ru);
        wf = reinterpret_cast<WT*>(sm + SM::wf);
        wu = reinterpret_cast<WT*>(sm + SM::wu);
        thrc = reinterpret_cast<WT*>(sm + SM::thrc);
        qtab = reinterpret_cast<double2*>(sm + SM::qtab);
    }

    // Fill the tables from the N*N weights sw (shared memory, all threads;
    // the caller synchronises before and after).  QT: also z^creg[r].
    // THR: also the per-thread constants (thrc), which the tile-cut table
    // kernel does not need.
    template <bool QT, bool THR = true>
    __device__ void setup(const WT* sw, int N, int l, int a, int tid, double gamma) const {
        const int nF = N - kTileBits;
        for (int idx = tid; idx < nF * nF; idx += kPassThreads) {
            const int i = idx / nF, j = idx - i * nF;
            wf[i * kWfStride + j] = sw[fixed_phys(i, l, a) * N + fixed_phys(j, l, a)];
        }
        for (int idx = tid; idx < kTileBits * nF; idx += kPassThreads) {
            const int u = idx / nF, j = idx - u * nF;
            wu[u * kWfStride + j] = sw[tile_phys(u, l, a) * N + fixed_phys(j, l, a)];
        }
        if (tid < nF) {
            const int m = fixed_phys(tid, l, a);
            WT d = 0;
            for (int u = 0; u < kTileBits; u++) d += sw[m * N + tile_phys(u, l, a)];
            Dm[tid] = d;
        } else if (tid >= 32 && tid < 32 + kTileBits) {
            const int u = tile_phys(tid - 32, l, a);
            WT r = 0;
            for (int i = 0; i < nF; i++) r += sw[u * N + fixed_phys(i, l, a)];
            Ru[tid - 32] = r;
        } else if (tid >= 64 && tid < 96) {
            const int L = (tid - 64) >> 4, r = tid & 15;
            WT c = 0;
            for (int k = 0; k < 4; k++)
                for (int k2 = k + 1; k2 < 4; k2++)
                    if (((r >> k) ^ (r >> k2)) & 1)
                        c += sw[tile_phys(rbit(L, k), l, a) * N + tile_phys(rbit(L, k2), l, a)];
            creg[16 * L + r] = c;
            if (QT) {
                double sn, cs;
                sincos(gamma * (double)c, &sn, &cs);
                qtab[16 * L + r] = make_double2(cs, sn);
            }
        }
        for (int L = 0; L < (THR ? 2 : 0); L++) {
            const int T = L == 0 ? tid : lay_index<1>(tid, 0);  // slot 0's tile index
            WT athr = 0, f[4] = {0, 0, 0, 0};
            for (int j = 0; j < 8; j++) {
                const int pj = tile_phys(tbit(L, j), l, a);
                const int tj = (T >> tbit(L, j)) & 1;
                for (int j2 = j + 1; j2 < 8; j2++)
                    if (tj ^ ((T >> tbit(L, j2)) & 1))
                        athr += sw[pj * N + tile_phys(tbit(L, j2), l, a)];
                // Edge (thread bit j, register bit k) is cut iff t_j != r_k:
                // t_j + r_k (1 - 2 t_j).
                for (int k = 0; k < 4; k++) {
                    const WT w = sw[pj * N + tile_phys(rbit(L, k), l, a)];
                    if (tj) {
                        athr += w;
                        f[k] -= w;
                    } else {
                        f[k] += w;
                    }
                }
            }
            WT* tc = thrc + 5 * kPassThreads * L;
            tc[tid] = athr;
            for (int k = 0; k < 4; k++) tc[(1 + k) * kPassThreads + tid] = f[k];
        }
    }

    // Tile bit of register bit k and of thread bit j in layout L (L0: the
    // thread's bits are tile bits 0..7, registers 8..11; L1: thread bits
    // 0..3 and 8..11, registers 4..7).
    __host__ __device__ static int rbit(int L, int k) { return L == 0 ? 8 + k : 4 + k; }
    __host__ __device__ static int tbit(int L, int j) { return L == 0 ? j : (j < 4 ? j : j + 4); }

    // K and e_u of the tile at `base` into kp (warps 0 and 1 of the block;
    // the caller synchronises before reading kp).
    __device__ void tile(WT* kp, i64 base, int nF, int l, int a, int warp, int lane) const {
        if (warp >= 2) return;
        const int zi = lane < nF ? (int)((base >> fixed_phys(lane, l, a)) & 1) : 0;
        const unsigned F = __ballot_sync(0xffffffffu, zi);
        if (warp == 0) {
            WT h = 0;
            if (lane < nF) {
                if (zi) h = Dm[lane];
                const WT* row = wf + lane * kWfStride;
#pragma unroll
                for (int j = 1; j < kMaxFixed; j++)
                    if (j > lane && j < nF && (((F >> j) & 1u) != (unsigned)zi)) h += row[j];
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
            if (lane == 0) kp[0] = h;
        } else if (lane < kTileBits) {
            WT e = Ru[lane];
            const WT* row = wu + lane * kWfStride;
#pragma unroll
            for (int j = 0; j < kMaxFixed; j++)
                if (j < nF && ((F >> j) & 1u)) e -= 2 * row[j];
            kp[1 + lane] = e;
        }
    }

    // K (role 0) or e_u (role 1) of the tile at `base` into out (one warp):
    // tile()'s warp 0 or warp 1 work in the same order, so the values are
    // the same.
    __device__ void tile_part(WT* out, i64 base, int nF, int l, int a, int lane,
                              int role) const {
        const int zi = lane < nF ? (int)((base >> fixed_phys(lane, l, a)) & 1) : 0;
        const unsigned F = __ballot_sync(0xffffffffu, zi);
        if (role == 0) {
            WT h = 0;
            if (lane < nF) {
                if (zi) h = Dm[lane];
                const WT* row = wf + lane * kWfStride;
#pragma unroll
                for (int j = 1; j < kMaxFixed; j++)
                    if (j > lane && j < nF && (((F >> j) & 1u) != (unsigned)zi)) h += row[j];
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
            if (lane == 0) out[0] = h;
        } else if (lane < kTileBits) {
            WT e = Ru[lane];
            const WT* row = wu + lane * kWfStride;
#pragma unroll
            for (int j = 0; j < kMaxFixed; j++)
                if (j < nF && ((F >> j) & 1u)) e -= 2 * row[j];
            out[1 + lane] = e;
        }
    }

    // cb = cut value of the thread's register slot 0, g_k = change of the
    // cut when register bit k is set; slot r has c_r = cb + creg[r] +
    // sum_k r_k g_k.
    template <int L = 0>
    __device__ void consts(const WT* kp, int tid, WT& cb, WT& g0, WT& g1, WT& g2, WT& g3) const {
        const WT* tc = thrc + 5 * kPassThreads * L;
        const int T = L == 0 ? tid : lay_index<1>(tid, 0);
        cb = kp[0] + tc[tid];
#pragma unroll
        for (int j = 0; j < 8; j++)
            if ((T >> tbit(L, j)) & 1) cb += kp[1 + tbit(L, j)];
        g0 = tc[kPassThreads + tid] + kp[1 + rbit(L, 0)];
        g1 = tc[2 * kPassThreads + tid] + kp[1 + rbit(L, 1)];
        g2 = tc[3 * kPassThreads + tid] + kp[1 + rbit(L, 2)];
        g3 = tc[4 * kPassThreads + tid] + kp[1 + rbit(L, 3)];
    }
};

// Cut constants of every tile of up to four pass geometries (blockIdx.y
// picks one) for the tile passes to read instead of computing them per
// tile: out[y * ntiles * kTcutStride + T * kTcutStride] = K, then
// e_0..e_11 (CutTables::tile).  256 threads set up the tables, then each
// pair of warps takes tiles, K on one, the e_u on the other.  Shared
// memory: the N*N weights, rounded up to 16 bytes, then PassSmem<WT>.
constexpr int kTcutStride = 16;
struct TcutGeoms {
    int l[4], a[4];
};
template <typename WT>
__host__ __device__ inline size_t tcut_smem_bytes(int N) {
    return ((N * N * sizeof(WT) + 15) & ~(size_t)15) + PassSmem<WT>::bytes;
}

template <typename WT>
__global__ void __launch_bounds__(kPassThreads) k_tile_cuts(const WT* w, int N, TcutGeoms G,
                                                            i64 ntiles, WT* out) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const int l = G.l[blockIdx.y], a = G.a[blockIdx.y];
    out += (i64)blockIdx.y * ntiles * kTcutStride;
    WT* sw = reinterpret_cast<WT*>(smraw);
    const CutTables<WT> ct(smraw + ((N * N * sizeof(WT) + 15) & ~(size_t)15));
    for (int i = threadIdx.x; i < N * N; i += kPassThreads) sw[i] = w[i];
    __syncthreads();
    ct.template setup<false, false>(sw, N, l, a, threadIdx.x, 0.0);
    __syncthreads();
    const int nF = N - kTileBits, nmid = a - l, lane = threadIdx.x & 31;
    const int role = (threadIdx.x >> 5) & 1, tpb = kPassThreads / 64;  // tiles per block and round
    for (i64 T = (i64)blockIdx.x * tpb + (threadIdx.x >> 6); T < ntiles; T += (i64)gridDim.x * tpb) {
        const i64 base = ((T & ((1ll << nmid) - 1)) << l) | ((T >> nmid) << (a + kTileBits - l));
        ct.tile_part(out + T * kTcutStride, base, nF, l, a, lane, role);
    }
}

// z^d with z = exp(i*gamma): the two-level table (integer weights) or sincos.
template <typename WT>
__device__ __forceinline__ double2 zpow(const PassArgs& A, const double2* smtab, WT d) {
    if (sizeof(WT) == sizeof(int)) return tab_pow(A, smtab, (int)d);
    double sn, cs;
    sincos(A.gamma * (double)d, &sn, &cs);
    return make_double2(cs, sn);
}

// P = phase(cbase) without the layer-0 scale: ph0 * z^cbase (integer
// weights) or scale * exp(i*gamma*(cbase - W/2)).
template <typename WT>
__device__ __forceinline__ double2 phase_of(const PassArgs& A, const double2* smtab, WT cbase) {
    if (sizeof(WT) == sizeof(int))
        return cmul(make_double2(A.ph0x, A.ph0y), tab_pow(A, smtab, (int)cbase));
    double sn, cs;
    sincos(A.gamma * ((double)cbase - 0.5 * A.W), &sn, &cs);
    return make_double2(cs * A.scale, sn * A.scale);
}

// GM2 != GM_NONE makes a fused pass: RX (GM, A.gx) on the tile's targets,
// then the phase of the next layer (PH_MUL, the tables and angle in A), then
// that layer's RX (GM2, A.gx2) on the same targets.  With the layer order
// reversed every other layer, the last pass of one layer and the first of
// the next share a tile geometry, so two sweeps become one.
//
// PAIR (strided tiles with rows of 2 to 8 amplitudes, l = 1..3): 512
// threads, one CTA per SM, as two 256-thread groups that take the two tiles
// differing only in physical bit l (tile numbers 2t and 2t+1) at the same
// time, each with its own exchange buffer, tile constants and named
// barrier.  Their loads and stores then meet DRAM as rows twice as long
// (256 bytes at l = 3): per-thread sweeps over 128-byte rows measured
// 4.1-4.9 TB/s on B200 at N=30, over 256-byte rows 5.6 TB/s.
template <typename WT, int PH, int GM, int EX, bool ST, int SC, int GM2 = GM_NONE,
          bool PAIR = false>
__global__ void __launch_bounds__(PAIR ? 2 * kPassThreads : kPassThreads, PAIR ? 1 : 2)
    k_pass(const PassArgs A) {
    extern __shared__ __align__(16) unsigned char smraw[];
    using SM = PassSmem<WT>;
    const int grp = PAIR ? (int)(threadIdx.x >> 8) : 0;  // the thread's group (tile of the pair)
    double2* buf = reinterpret_cast<double2*>(smraw) + (size_t)grp * kXTile;
    unsigned char* const sm = smraw + sizeof(double2) * kXTile * (PAIR ? 2 : 1);
    double* red = reinterpret_cast<double*>(sm + SM::red);
    const CutTables<WT> ct(sm);
    double2* smtab = reinterpret_cast<double2*>(sm + SM::smtab);
    const int N = A.N, l = A.l, a = A.a;
    const int nF = N - kTileBits;
    constexpr bool CUT = (PH != PH_NONE) || (EX != EX_NONE);
    // Passes with a phase or rotations may read their tiles' cut constants
    // from A.tcut (the read-only <C> pass always computes them per tile).
    constexpr bool TCUT = CUT && (PH != PH_NONE || GM != GM_NONE);
    constexpr bool LOAD = (PH != PH_INIT) && (ST || EX == EX_ENERGY || EX == EX_COSTATE);
    constexpr bool ACC = (EX == EX_ENERGY || EX == EX_COSTATE);
    constexpr bool INTW = sizeof(WT) == sizeof(int);
    // tid, lane and warp index the thread within its group of 256.
    const int tid = threadIdx.x & (kPassThreads - 1), lane = tid & 31, warp = tid >> 5;
    const int nmid = a - l;  // fixed bits between the row bits and the high tile bits
    // Product-tree phases: integer weights with the two-level table (nhi ==
    // 0 keeps one global-table lookup per amplitude), FP64 weights when the
    // host allows it (A.tree: small |gamma| * sum|w|, see phase_tree_ok).
    const bool tree = PH != PH_NONE && (INTW ? A.nhi > 0 : A.tree != 0);

    // ---- set-up: compact weight tables of this pass's tile geometry (the
    // tables depend on the geometry only: one copy serves both groups)
    WT* sw = reinterpret_cast<WT*>(smraw);  // N*N weights while setting up
    if (CUT) {
        const WT* gw = reinterpret_cast<const WT*>(A.w);
        for (int i = threadIdx.x; i < N * N; i += blockDim.x) sw[i] = gw[i];
    }
    if (PH != PH_NONE && INTW) load_phase_tables(A, smtab, threadIdx.x, blockDim.x);
    __syncthreads();
    if (CUT && threadIdx.x < kPassThreads)
        ct.template setup<PH != PH_NONE>(sw, N, l, a, tid, A.gamma);
    __syncthreads();  // the weights in the buffer are dead from here on

    // Address pieces: the thread's offsets in layouts L0 and L1 and the
    // strides of the 4 register bits of each (uniform across the grid).
    const i64 thr_off = tile_off(tid, l, a);
    const i64 thr_off1 = tile_off(lay_index<1>(tid, 0), l, a);
    const i64 s8 = 1ll << tile_phys(8, l, a), s9 = 1ll << tile_phys(9, l, a);
    const i64 s10 = 1ll << tile_phys(10, l, a), s11 = 1ll << tile_phys(11, l, a);
    const i64 s4 = 1ll << tile_phys(4, l, a), s5 = 1ll << tile_phys(5, l, a);
    const i64 s6 = 1ll << tile_phys(6, l, a), s7 = 1ll << tile_phys(7, l, a);
    auto off0 = [&](int r) -> i64 {
        return ((r & 1) ? s8 : 0) + ((r & 2) ? s9 : 0) + ((r & 4) ? s10 : 0) + ((r & 8) ? s11 : 0);
    };
    auto off1 = [&](int r) -> i64 {
        return ((r & 1) ? s4 : 0) + ((r & 2) ? s5 : 0) + ((r & 4) ? s6 : 0) + ((r & 8) ? s7 : 0);
    };
    const bool contiguous = (l == kTileBits);
    const unsigned m_hi = (A.tmask >> 8) & 15u, m_mid = (A.tmask >> 4) & 15u, m_lo = A.tmask & 15u;
    // Tile bits 0..3: two or more targets take a register round in L2
    // (SC_L021), a single one is rotated by shuffles in L0.
    const int lo_lane = (SC != SC_L021 && m_lo) ? __ffs(m_lo) - 1 : -1;
    double acc = 0, comp = 0;  // Kahan-compensated <C> accumulator

    int par = 0;
    const i64 nunits = PAIR ? A.ntiles / 2 : A.ntiles;
    // Fused passes end their rounds with an exchange into layout L0, after
    // which each thread's L0 slots of the buffer are its own until the next
    // tile's first exchange: the thread copies its part of the next tile
    // there (cp.async, 16 B each) before its last rotations and stores, and
    // reads it back at the next tile's start, so the next tile's loads are
    // in flight while this one finishes (on B200 at N=30, p=5: fused
    // passes 9.56-9.61 against 9.91-10.15 ms, A/B in one call).
    constexpr bool CPF = (GM2 != GM_NONE) && LOAD && ST && (SC != SC_L0);
    bool have_next = false;  // this thread's part of the tile is in buf
    // Write-only layer-0 passes reading table constants alternate the
    // direction of their exchange from tile to tile (L0 -> L1 on even
    // iterations, L1 -> L0 on odd ones, the phase and rounds in the matching
    // layouts): each thread then writes only slots that it, or its partner
    // lane behind exchange_lane's warp barrier, read last, so no exchange
    // needs a leading barrier and a tile takes one barrier.
    constexpr bool ALT = PH == PH_INIT && GM2 == GM_NONE && SC == SC_L01 && EX == EX_NONE &&
                         GM != GM_NONE && TCUT;
    const bool alt = ALT && A.tcut != nullptr;
    // Mixer passes with a round in L2 alternate the same way: odd tiles are
    // loaded in L1 and run L1 -> L2 -> L0 (the L1 <-> L2 exchange stays in
    // the warp), so the next tile's L0 -> L2 exchange writes only slots its
    // thread has just read, and a tile takes one block barrier, not two (on
    // B200 at N=30, p=5: mixer passes 5.89-5.97 against 6.00-6.08 ms, A/B in
    // one call).
    constexpr bool ALTM = PH == PH_NONE && GM != GM_NONE && GM2 == GM_NONE && SC == SC_L021 &&
                          EX == EX_NONE && ST && !PAIR;
    const bool skip_lead = (CUT && !(TCUT && A.tcut)) || CPF || alt || ALTM;
    for (i64 U = blockIdx.x; U < nunits; U += gridDim.x, par ^= 1) {
        const i64 T = PAIR ? 2 * U + grp : U;
        const i64 base = ((T & ((1ll << nmid) - 1)) << l) | ((T >> nmid) << (a + kTileBits - l));
        double2* const p = A.sv + base + thr_off;
        double2 v[kRegs];
        // The loads go out first; the tile's cut constants are computed
        // while they are in flight.
        if (CPF && have_next) {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
            const double2* const own = buf + pbase<0>(tid);
#pragma unroll
            for (int r = 0; r < kRegs; r++) v[r] = own[pslot(lay_index<0>(0, r))];
        } else {
#pragma unroll
            for (int r = 0; r < kRegs; r++) {
                if (ALTM && par) v[r] = __ldcs(A.sv + base + thr_off1 + off1(r));
                else if (LOAD) v[r] = __ldcs(p + off0(r));
                else v[r] = make_double2(0.0, 0.0);
            }
        }
        if (!PAIR && LOAD && A.pf_dist > 0 && contiguous) {
            // Stream this CTA's tile pf_dist strides ahead from HBM into L2
            // (one bulk prefetch).  Strided tiles are not prefetched: per-
            // thread row prefetches cost more than they saved (12.2 against
            // 11.2 ms on the fused strided pass at N=30), and so did a tensor
            // prefetch of the tile as a TMA box (61.5 against 58.1-61.0
            // layers/s at N=30, p=5; A/B in one call).
            const i64 T2 = T + (i64)A.pf_dist * gridDim.x;
            if (T2 < A.ntiles && tid == 0) {
                const i64 b2 = ((T2 & ((1ll << nmid) - 1)) << l) |
                               ((T2 >> nmid) << (a + kTileBits - l));
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(A.sv + b2),
                             "r"((unsigned)(kTile * sizeof(double2)))
                             : "memory");
            }
        }
        // The tile's cut constants: from the table (kp in global memory), or
        // computed by warps 0 and 1 into shared memory (double-buffered per
        // group: no barrier for the previous readers) and a barrier.
        const WT* kp = ct.ke + 64 * grp + 32 * par;
        WT cbase = 0, g0 = 0, g1 = 0, g2 = 0, g3 = 0;
        if (CUT) {
            if (TCUT && A.tcut) {
                kp = reinterpret_cast<const WT*>(A.tcut) + T * kTcutStride;
                // The next tile's constants into L1 now: the passes' sweeps
                // evict the table from L2, and a miss on it would stall the
                // next tile's phase.
                const i64 Tn = T + (PAIR ? 2 * (i64)gridDim.x : (i64)gridDim.x);
                if (tid == 0 && Tn < A.ntiles)
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(
                                     reinterpret_cast<const WT*>(A.tcut) + Tn * kTcutStride)
                                 : "memory");
            } else {
                ct.tile(ct.ke + 64 * grp + 32 * par, base | A.goff, nF, l, a, warp, lane);
                tile_sync<PAIR>(grp);
            }
            if (!(alt && par)) ct.consts(kp, tid, cbase, g0, g1, g2, g3);
        }
        // The cost phase (PH_INIT writes it, PH_MUL multiplies it in), with
        // the registers in layout LL (0 or 1) and that layout's constants.
        auto apply_phase = [&](auto lay_tag, WT cb, WT h0, WT h1, WT h2, WT h3) {
            constexpr int LL = decltype(lay_tag)::value;
            const double2* qt = ct.qtab + 16 * LL;
            const WT* crg = ct.creg + 16 * LL;
            if (tree) {
                double2 P = phase_of<WT>(A, smtab, cb);
                if (INTW && PH == PH_INIT) P = make_double2(P.x * A.scale, P.y * A.scale);
                phase_tree<PH>(v, P, qt, zpow<WT>(A, smtab, h0), zpow<WT>(A, smtab, h1),
                               zpow<WT>(A, smtab, h2), zpow<WT>(A, smtab, h3));
            } else {
#pragma unroll
                for (int r = 0; r < kRegs; r++) {
                    const WT cr = cb + crg[r] + ((r & 1) ? h0 : WT(0)) +
                                  ((r & 2) ? h1 : WT(0)) + ((r & 4) ? h2 : WT(0)) +
                                  ((r & 8) ? h3 : WT(0));
                    double2 ph;
                    if (INTW) {
                        ph = int_phase(A, smtab, (int)cr);
                        if (PH == PH_INIT) ph = make_double2(ph.x * A.scale, ph.y * A.scale);
                    } else {  // the reference's own argument (src/rzz.cu:146-150)
                        const double S = 2.0 * (double)cr - A.W;
                        double sn, cs;
                        sincos(S * A.gamma / 2, &sn, &cs);
                        ph = make_double2(cs * A.scale, sn * A.scale);
                    }
                    v[r] = (PH == PH_INIT) ? ph : cmul(v[r], ph);
                }
            }
        };
        // RX rounds on the tile's targets, from layout L0 to L1 (or L0 with
        // SC_L0).  first: the tile's first exchange skips its leading barrier
        // when the buffer's previous readers are already past one (the cut
        // barrier), or when the thread writes only slots that no other
        // thread reads after the previous tile's last barrier: its own L0
        // slots in a fused pass, whose previous tile ended by reading them.
        auto rx_rounds = [&](auto gm_tag, double gx, bool first) {
            constexpr int G = decltype(gm_tag)::value;
            rx_regs<G>(v, m_hi, gx, A.c, A.s);
            if (SC == SC_L0 && lo_lane >= 0) rx_lane<G>(v, lo_lane, gx, A.c, A.s);
            if (SC == SC_L021) {
                exchange<0, 2, PAIR>(v, buf, tid, !(first && skip_lead), grp);
                rx_regs<G>(v, m_lo, gx, A.c, A.s);
                exchange<2, 1, PAIR>(v, buf, tid, false, grp);
            } else if (SC == SC_L01) {
                if (GM2 == GM_NONE && lo_lane >= 0)
                    exchange_lane<0, 1, G, PAIR>(v, buf, tid, !(first && skip_lead), grp, lo_lane, gx,
                                                 A.c, A.s);
                else if (lo_lane >= 0)
                    exchange_lanet<0, 1, G, PAIR>(v, buf, tid, !(first && skip_lead), grp, lo_lane,
                                                  gx, A.c, A.s);
                else
                    exchange<0, 1, PAIR>(v, buf, tid, !(first && skip_lead), grp);
            }
            if (SC != SC_L0) rx_regs<G>(v, m_mid, gx, A.c, A.s);
        };
        constexpr bool FUSED = GM2 != GM_NONE;
        using L0t = std::integral_constant<int, 0>;
        using L1t = std::integral_constant<int, 1>;
        if (ALT && alt && par) {  // the odd iteration of an alternating pass (see ALT)
            WT cb, h0, h1, h2, h3;
            ct.template consts<1>(kp, tid, cb, h0, h1, h2, h3);
            apply_phase(L1t(), cb, h0, h1, h2, h3);
            rx_regs<GM>(v, m_mid, A.gx, A.c, A.s);
            if (lo_lane >= 0)
                exchange_lane<1, 0, GM, PAIR>(v, buf, tid, false, grp, lo_lane, A.gx, A.c, A.s);
            else
                exchange<1, 0, PAIR>(v, buf, tid, false, grp);
            rx_regs<GM>(v, m_hi, A.gx, A.c, A.s);
#pragma unroll
            for (int r = 0; r < kRegs; r++) __stcs(p + off0(r), v[r]);
            continue;
        }
        if (ALTM && par) {  // the odd iteration of an alternating mixer pass (see ALTM)
            rx_regs<GM>(v, m_mid, A.gx, A.c, A.s);
            exchange<1, 2, PAIR>(v, buf, tid, true, grp);
            rx_regs<GM>(v, m_lo, A.gx, A.c, A.s);
            exchange<2, 0, PAIR>(v, buf, tid, false, grp);
            rx_regs<GM>(v, m_hi, A.gx, A.c, A.s);
#pragma unroll
            for (int r = 0; r < kRegs; r++) __stcs(p + off0(r), v[r]);
            continue;
        }
        if constexpr (PH == PH_MUL && !FUSED) {
            if (A.pre_mask) rx_regs<GM_FULL>(v, A.pre_mask, 0.0, A.pc, A.ps);
        }
        if (PH != PH_NONE && !FUSED) apply_phase(L0t(), cbase, g0, g1, g2, g3);
        // Final layout: L1 after an exchange (<C> then takes the cut
        // constants of L1), L0 for the costate and the diagonal (written at
        // L0 addresses) and for fused passes (their second rounds run back
        // from L1 to L0).
        constexpr int LAY =
            (GM != GM_NONE && SC != SC_L0 && (EX == EX_NONE || EX == EX_ENERGY) && !FUSED) ? 1
                                                                                          : 0;
        if (GM != GM_NONE) {
            rx_rounds(std::integral_constant<int, GM>(), A.gx, true);
            if (FUSED) {
                constexpr int G2 = FUSED ? GM2 : GM;
                WT cb, h0, h1, h2, h3;
                if (SC == SC_L0) {
                    ct.consts(kp, tid, cb, h0, h1, h2, h3);
                    apply_phase(L0t(), cb, h0, h1, h2, h3);
                    rx_rounds(std::integral_constant<int, G2>(), A.gx2, false);
                } else {
                    // The next layer's phase in L1, then its rounds in the
                    // opposite order: L1 -> (L2 ->) L0.
                    ct.template consts<1>(kp, tid, cb, h0, h1, h2, h3);
                    apply_phase(L1t(), cb, h0, h1, h2, h3);
                    rx_regs<G2>(v, m_mid, A.gx2, A.c, A.s);
                    if (SC == SC_L021) {
                        exchange<1, 2, PAIR>(v, buf, tid, false, grp);
                        rx_regs<G2>(v, m_lo, A.gx2, A.c, A.s);
                        exchange<2, 0, PAIR>(v, buf, tid, false, grp);
                    } else if (lo_lane >= 0) {
                        // A single target among tile bits 0..3 is a lane bit
                        // in L1 as in L0.
                        exchange_lanet<1, 0, G2, PAIR>(v, buf, tid, false, grp, lo_lane, A.gx2,
                                                       A.c, A.s);
                    } else {
                        exchange<1, 0, PAIR>(v, buf, tid, false, grp);
                    }
                    if (CPF) {
                        const i64 U2 = U + gridDim.x;
                        have_next = U2 < nunits;
                        if (have_next) {
                            const i64 T2 = PAIR ? 2 * U2 + grp : U2;
                            const i64 b2 = ((T2 & ((1ll << nmid) - 1)) << l) |
                                           ((T2 >> nmid) << (a + kTileBits - l));
                            const double2* const src = A.sv + b2 + thr_off;
                            const unsigned dst = (unsigned)__cvta_generic_to_shared(
                                buf + pbase<0>(tid));
#pragma unroll
                            for (int r = 0; r < kRegs; r++)
                                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                                                 dst + (unsigned)(16 * pslot(lay_index<0>(0, r)))),
                                             "l"(src + off0(r))
                                             : "memory");
                            asm volatile("cp.async.commit_group;" ::: "memory");
                        }
                    }
                    rx_regs<G2>(v, m_hi, A.gx2, A.c, A.s);
                }
            } else if (SC != SC_L0 && LAY == 0) {
                exchange<1, 0, PAIR>(v, buf, tid, false, grp);
            }
        }
        // The cut constants again for the outputs that need them (read back
        // instead of held in registers through the rounds above).
        if (EX != EX_NONE) ct.template consts<LAY>(kp, tid, cbase, g0, g1, g2, g3);
        const WT* const crg = ct.creg + 16 * LAY;
        if (EX == EX_DIAG) {
#pragma unroll
            for (int r = 0; r < kRegs; r++) {
                const WT cr = cbase + crg[r] + ((r & 1) ? g0 : WT(0)) + ((r & 2) ? g1 : WT(0)) +
                              ((r & 4) ? g2 : WT(0)) + ((r & 8) ? g3 : WT(0));
                __stcs(A.diag + base + thr_off + off0(r), (double)cr);
            }
        }
        if (ACC) {
            double ts = 0;
#pragma unroll
            for (int r = 0; r < kRegs; r++) {
                const WT cr = cbase + crg[r] + ((r & 1) ? g0 : WT(0)) + ((r & 2) ? g1 : WT(0)) +
                              ((r & 4) ? g2 : WT(0)) + ((r & 8) ? g3 : WT(0));
                ts = fma(fma(v[r].x, v[r].x, v[r].y * v[r].y), (double)cr, ts);
                if (EX == EX_COSTATE) {
                    const double c = (double)cr;
                    __stcs(A.sv2 + base + thr_off + off0(r), make_double2(c * v[r].x, c * v[r].y));
                }
            }
            const double y = ts - comp;
            const double t2 = acc + y;
            comp = (t2 - acc) - y;
            acc = t2;
        }
        if (ST) {
            if (LAY == 0) {
#pragma unroll
                for (int r = 0; r < kRegs; r++) __stcs(p + off0(r), v[r]);
            } else {
                double2* const p1 = A.sv + base + thr_off1;
#pragma unroll
                for (int r = 0; r < kRegs; r++) __stcs(p1 + off1(r), v[r]);
            }
        }
    }
    if (ACC) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        __syncthreads();
        if (lane == 0) red[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
            A.partial[blockIdx.x] = s;
        }
    }
}

}  // namespace fq
