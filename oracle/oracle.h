/*
 * oracle.h -- CPU FP64 restatement of FOR-QAOA's single-device (D=0) QAOA
 * Max-Cut state-vector path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * only the test suite, the smoke check and the CPU-baseline leg of the bench
 * may load it.  The product library never links, loads or calls it.
 *
 * Parity pin: the restatement follows the reference's source line by line
 * (file:line cited at each function) and is checked against golden vectors
 * produced by the reference's own CUDA code (built from its unmodified
 * sources into oracle/_ref by oracle/Makefile.ref and run through
 * oracle/ref_harness.cpp); see tests/golden/.
 *
 * Conventions (all from the reference):
 *  - amplitudes are AoS complex128 {re, im}; bit q of the index is qubit q;
 *  - graphs are N x N row-major FP64 upper triangles, entry [i*N+j], i<j,
 *    zero meaning "no edge" (graph.cpp:54-64);
 *  - cost layer multiplies by exp(+i*gamma*S(z)/2) with
 *    S(z) = sum_{i<j, w!=0} (z_i xor z_j ? +w : -w)   (rzz.cu:121-156);
 *  - mixer is RX(beta) = exp(-i*beta*X/2) on each qubit (rx.cu:32-53,121).
 */
#ifndef FQ_ORACLE_H
#define FQ_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* rzz.cu:26-28 */
double orc_init_amp(int N);
/* rzz.cu:158-171 */
void orc_upper_tri_to_1d(int N, const double* upper, double* out);
/* rzz.cu:121-156 (kernel) + rzz.cu:173-206 (launcher), literal pair-order sum */
void orc_cost_phase(double* sv, int N, double angle, const double* graph1d,
                    int is_first_layer, double init_amp);
/* rx.cu:24-53, 56-87, 118-126: RX(angle) on targets[0..gate_size) in order */
void orc_multi_rotate_x(double* sv, int N, const int* targets, int gate_size,
                        double angle);
/* swap.cu:76-102, 166-187: exchange qubit blocks [out,out+k) <-> [in,in+k) */
void orc_swap_gate_conti(double* sv, int N, int swap_out, int swap_in, int num_swap);
/* swap.cu:27-50: relabel the upper-triangular graph the same way */
void orc_mapping_after_swap_conti(double* graph, int N, int swap_out, int swap_in,
                                  int num_swap);
/* Weighted.cpp:97-138 with per-layer angles: the reference's own schedule
 * (cost, then per chunk RX + block swap + relabel).  sv receives the final
 * state in the reference's PHYSICAL order; graph_final (may be NULL) the
 * relabelled graph; label_map (may be NULL) phys position -> logical qubit. */
void orc_weighted_run(int N, int C, int P, const double* graph_upper,
                      const double* gammas, const double* betas, double* sv,
                      double* graph_final, int* label_map);
/* The same circuit in logical qubit order (no swaps). */
void orc_qaoa_logical(int N, int P, const double* graph_upper,
                      const double* gammas, const double* betas, double* sv);
/* S(z) for every z, literal pair-order sum (rzz.cu:127-143). */
void orc_cost_diag_S(int N, const double* graph_upper, double* S);
/* C(z) = sum of cut edge weights for every z (integer weights: exact). */
void orc_cut_values(int N, const double* graph_upper, double* Cz);
/* <C> = sum_z |psi_z|^2 C(z), long-double accumulation. */
double orc_expectation(const double* sv, int N, const double* graph_upper);
/* Energy and adjoint gradient of <C> w.r.t. gammas[k], betas[k]. */
void orc_energy_grad(int N, int P, const double* graph_upper, const double* gammas,
                     const double* betas, double* energy, double* grad_gamma,
                     double* grad_beta);
/* dst[y] = src[x] where y has bit perm[b] equal to bit b of x. */
void orc_permute_qubits(const double* src, double* dst, int N, const int* perm);
/* Every amplitude set to re + i*im (OpenMP first touch). */
void orc_state_fill(double* sv, int N, double re, double im);
/* CPU-baseline unit of work: chunk `chunk` of `nchunks` equal parts of one
 * QAOA layer on a full 2^N state -- the cost phase of rzz.cu:121-156 (pair
 * loop over the whole graph) on amplitudes [chunk, chunk+1) * 2^N/nchunks,
 * then RX (rx.cu:32-53) for every qubit t on pairs [chunk, chunk+1) *
 * 2^(N-1)/nchunks of t's pair enumeration.  The nchunks parts together do
 * exactly one layer's amplitude and pair updates.  Returns each half's
 * seconds. */
void orc_layer_chunk(double* sv, int N, const double* graph1d, double gamma, double beta,
                     int first_layer, int chunk, int nchunks, double* t_cost, double* t_rx);
/* Threads OpenMP will use. */
int orc_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
