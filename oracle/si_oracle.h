/*
 * si_oracle.h — CPU oracle for the imputation hot path (TEST INFRASTRUCTURE).
 *
 * This is the checker, not the product. Only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline / reference arm may load it. The product path
 * (libswiftimpute_b200.so) never links, calls or falls back to it.
 *
 * Each function restates one step of the reference (tcBio/SwiftImpute) in
 * plain C, citing the reference file:line it follows. Pinning:
 *   - sio_pbwt_build is checked bit-for-bit against the reference's own
 *     PBWTBuilder::build compiled from its sources (oracle/_ref, see Makefile).
 *   - sio_select_row / sio_fb_sample are checked against the reference's own
 *     GPU kernels compiled from source and run on a B200 (tests/golden/).
 */
#ifndef SI_ORACLE_H
#define SI_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Selection patterns the reference kernels produce when every divergence at a
 * marker ties (pbwt_index.cpp:173-191 makes every divergence equal m). */
enum { SIO_SEL_AUTO = 0, SIO_SEL_WARP = 1, SIO_SEL_INSERTION = 2, SIO_SEL_FIRST_PAIRS = 3 };

/* Transition modes: the reference reads matrix 0 for every gap
 * (forward_backward.cu:108,201,234,269); PER_GAP uses each gap's own matrix. */
enum { SIO_TRANS_MATRIX0 = 0, SIO_TRANS_PER_GAP = 1 };

/* PBWT prefix sweep over a u8 panel [M][N] (reference layout). Writes the
 * prefix array [M][N]. Divergence is implicit: every entry of row m equals m. */
void sio_pbwt_build(const uint8_t* panel, uint32_t M, uint32_t N, uint32_t* prefix);

/* Same sweep over a bit-packed panel [M][W] u32 (bit i of word w = haplotype
 * 32w+i). Either output may be NULL. row_hash[m] = sio_row_hash(prefix row m). */
void sio_pbwt_build_packed(const uint32_t* words, uint32_t M, uint32_t N, uint32_t W,
                           uint32_t* prefix, uint64_t* row_hash);

/* Order-sensitive 64-bit hash of one prefix row (sum of mixed (value, position)). */
uint64_t sio_row_hash(const uint32_t* row, uint32_t N);

/* Slot haplotypes for one marker, given that marker's prefix row. */
int sio_select_kind(uint32_t N, uint32_t L);
void sio_select_row(const uint32_t* prefix_row, uint32_t N, uint32_t L, int kind, uint32_t* slots);
void sio_select_target(const uint32_t* prefix, const uint8_t* panel, const uint8_t* codes, uint32_t M, uint32_t N,
                       uint32_t L, uint32_t* pairs);

/* Li–Stephens log10 transition values (transition.cu:83-115), stored as float
 * like the reference. gd0/gd1 are genetic positions in Morgans. */
void sio_transition_log10(double gd0, double gd1, double ne, double rho_rate,
                          float* t_diag, float* t_off);

/* Philox4x32-10 (Salmon et al., SC'11): first output word for
 * counter (c0, c1, c2, c3) and key (k0, k1). */
uint32_t sio_philox_u32(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1);

/* Uniform in [0, 1) used for sampling cell (sample_id, marker). */
double sio_uniform(uint64_t seed, uint64_t sample_id, uint32_t marker);

/* One target sample through the FP64 log-space forward-backward.
 *   gl         [M][3] float log10 genotype likelihoods (reference TargetData)
 *   pairs      [M][L][2] haplotype ids per slot (reference selected_states)
 *   panel      [M][N] u8 alleles
 *   t_diag/t_off: one pair (MATRIX0) or M-1 pairs (PER_GAP), log10 floats
 * Outputs (any may be NULL):
 *   dosage [M], p0 [M], p1 [M]          posterior dosage and P(hap=1)
 *   hap_argmax [2][M]                    alleles of the argmax slot (tie_eps rule)
 *   hap_sampled [2][M]                   alleles of the Philox-sampled slot
 *   logpost [M][L]                       unnormalised alpha+beta (natural log)
 */
typedef struct {
    uint32_t M, N, L;
    int trans_mode;
    double tie_eps;
    uint64_t seed;
    uint64_t sample_id;
} sio_fb_args;

void sio_fb_sample(const sio_fb_args* a, const float* gl, const uint32_t* pairs,
                   const uint8_t* panel, const float* t_diag, const float* t_off,
                   float* dosage, float* p0, float* p1,
                   uint8_t* hap_argmax, uint8_t* hap_sampled, double* logpost);

/* Many samples over one shared slot table, threaded over samples.
 * gl [B][M][3]; outputs [B][M] (dosage/p0/p1) and [B][2][M] (haplotypes). */
void sio_fb_batch(const sio_fb_args* a, uint32_t B, const float* gl, const uint32_t* pairs,
                  const uint8_t* panel, const float* t_diag, const float* t_off,
                  float* dosage, float* p0, float* p1,
                  uint8_t* hap_argmax, uint8_t* hap_sampled, int n_threads);

/* Genotype code (0/1/2, 3 = missing) to the reference's hard-call GL triple
 * (imputer.cpp:244-295). */
void sio_codes_to_gl(const uint8_t* codes, uint64_t n, float* gl);

#ifdef __cplusplus
}
#endif
#endif
