/*
 * si_oracle.c — CPU oracle for the imputation hot path (TEST INFRASTRUCTURE).
 *
 * The checker, never the product: only tests/, __graft_entry__.smoke() and
 * bench.py (cpu_baseline leg, reference arm) load this library. Every function
 * restates one reference step in plain C; file:line citations are relative to
 * the tcBio/SwiftImpute source tree.
 *
 * Pinning: the PBWT sweep is compared bit-for-bit with the reference's own
 * PBWTBuilder compiled from source (oracle/_ref). Selection and the
 * forward-backward are compared with the reference's own CUDA kernels
 * compiled from source and run on a B200 (fixtures in tests/golden/).
 */
#include "si_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* PBWT prefix sweep                                                         */
/* ------------------------------------------------------------------------ */

/* One marker of the sweep: stable partition of the previous order by allele,
 * allele 0 first, any non-zero allele (incl. ALLELE_MISSING=255) second
 * (pbwt_index.cpp:176-207). The reference also pushes divergence values, but
 * it seeds p = q = m and resets them to m after every push
 * (pbwt_index.cpp:173-191), so each divergence entry of row m is m. */
static void sweep_step(const uint32_t* prev, uint32_t* cur, uint32_t N,
                       const uint8_t* row_u8, const uint32_t* row_bits) {
    uint32_t zeros = 0;
    for (uint32_t i = 0; i < N; ++i) {
        uint32_t h = prev[i];
        int one = row_u8 ? (row_u8[h] != 0) : (int)((row_bits[h >> 5] >> (h & 31)) & 1u);
        zeros += !one;
    }
    uint32_t z = 0, o = zeros;
    for (uint32_t i = 0; i < N; ++i) {
        uint32_t h = prev[i];
        int one = row_u8 ? (row_u8[h] != 0) : (int)((row_bits[h >> 5] >> (h & 31)) & 1u);
        if (one) cur[o++] = h; else cur[z++] = h;
    }
}

uint64_t sio_row_hash(const uint32_t* row, uint32_t N) {
    /* sum over positions of splitmix64(value + position * golden): addition
     * makes it order-independent to compute, the position makes it
     * order-sensitive as a function of the row. */
    uint64_t acc = 0;
    for (uint32_t i = 0; i < N; ++i) {
        uint64_t x = (uint64_t)row[i] + (uint64_t)i * 0x9E3779B97F4A7C15ull;
        x ^= x >> 30; x *= 0xBF58476D1CE4E5B9ull;
        x ^= x >> 27; x *= 0x94D049BB133111EBull;
        x ^= x >> 31;
        acc += x;
    }
    return acc;
}

/* Initial order is iota (pbwt_index.cpp:226); markers are swept in order
 * (pbwt_index.cpp:229-246). */
void sio_pbwt_build(const uint8_t* panel, uint32_t M, uint32_t N, uint32_t* prefix) {
    uint32_t* a = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)N);
    uint32_t* b = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)N);
    for (uint32_t i = 0; i < N; ++i) a[i] = i;
    for (uint32_t m = 0; m < M; ++m) {
        sweep_step(a, b, N, panel + (size_t)m * N, NULL);
        memcpy(prefix + (size_t)m * N, b, sizeof(uint32_t) * (size_t)N);
        uint32_t* t = a; a = b; b = t;
    }
    free(a); free(b);
}

void sio_pbwt_build_packed(const uint32_t* words, uint32_t M, uint32_t N, uint32_t W,
                           uint32_t* prefix, uint64_t* row_hash) {
    uint32_t* a = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)N);
    uint32_t* b = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)N);
    for (uint32_t i = 0; i < N; ++i) a[i] = i;
    for (uint32_t m = 0; m < M; ++m) {
        sweep_step(a, b, N, NULL, words + (size_t)m * W);
        if (prefix) memcpy(prefix + (size_t)m * N, b, sizeof(uint32_t) * (size_t)N);
        if (row_hash) row_hash[m] = sio_row_hash(b, N);
        uint32_t* t = a; a = b; b = t;
    }
    free(a); free(b);
}

/* ------------------------------------------------------------------------ */
/* L-state selection                                                         */
/* ------------------------------------------------------------------------ */

/* Kernel choice of launch_select_states (pbwt_selector.cu:413,428,441). */
int sio_select_kind(uint32_t N, uint32_t L) {
    return (L <= 32 && N <= 10000) ? SIO_SEL_WARP : SIO_SEL_INSERTION;
}

/* With every divergence of the row tied:
 *  - warp kernel (pbwt_selector.cu:212-312): each lane keeps its first four
 *    strided entries (:243-261); every round's max ties and __ffs picks
 *    lane 0 (:290-291), so round r emits row[32 r]; at most min(L, count of
 *    lane 0) rounds run (:276) and lane 0 fills the rest with i % N (:307-310).
 *    For N < 128 lanes hold different counts and the reference's full-mask
 *    shuffles run with lanes outside the loop; the value here is what the
 *    kernel computes when lane 0 wins, as it does whenever every lane joins.
 *  - insertion kernels (bitonic :320-394; block :47-204 in its defined case):
 *    strict '>' keeps the first L entries in scan order, rest i % N. */
void sio_select_row(const uint32_t* prefix_row, uint32_t N, uint32_t L, int kind, uint32_t* slots) {
    if (kind == SIO_SEL_AUTO) kind = sio_select_kind(N, L);
    if (kind == SIO_SEL_FIRST_PAIRS) {
        /* Imputer without an index: pairs (2k, 2k+1) (imputer.cpp:929-942) */
        for (uint32_t i = 0; i < L; ++i) slots[i] = 2 * i;
    } else if (kind == SIO_SEL_WARP) {
        uint32_t lane0 = (N + 31) / 32;
        if (lane0 > 4) lane0 = 4;
        for (uint32_t i = 0; i < L; ++i)
            slots[i] = (i < lane0) ? prefix_row[32 * i] : (i % N);
    } else {
        uint32_t top = N < L ? N : L;
        for (uint32_t i = 0; i < L; ++i)
            slots[i] = (i < top) ? prefix_row[i] : (i % N);
    }
}

/* Target-aware selection (the opt-in SI_SEL_TARGET; the reference has none:
 * its select_states, pbwt_index.cpp:20-79, sees only divergences equal to m).
 * One target, the Durbin (2014) PBWT extension of an inserted sequence: the
 * pseudo-haplotype carries 0 at code 0, 1 at code 2, else the allele of the
 * panel haplotype at its current position of the previous order (the last
 * entry when it sits past the end); its position p counts the haplotypes whose
 * reversed prefix sorts before it (it goes before equal keys):
 *   p' = zeros among prev[0, p)                   (allele 0)
 *   p' = Z + (p - zeros among prev[0, p))          (allele 1), Z = zeros at m.
 * Slots: positions clamp(p - L/2, 0, N - L) .. + L of the marker's order
 * (r % N when L > N), each as (h, (h + 1) % N). Non-zero alleles sort as 1,
 * as in the sweep. pairs: [M][L][2]. */
void sio_select_target(const uint32_t* prefix, const uint8_t* panel, const uint8_t* codes, uint32_t M, uint32_t N,
                       uint32_t L, uint32_t* pairs) {
    uint32_t p = 0;
    for (uint32_t m = 0; m < M; ++m) {
        const uint8_t* x = panel + (size_t)m * N;
        const uint32_t* prev = m ? prefix + (size_t)(m - 1) * N : NULL;
        uint32_t Z = 0, zb = 0;
        for (uint32_t i = 0; i < N; ++i) {
            const uint32_t h = prev ? prev[i] : i;
            const uint32_t z = x[h] == 0;
            Z += z;
            if (i < p) zb += z;
        }
        const uint32_t q = p < N ? p : N - 1;
        const uint32_t hq = prev ? prev[q] : q;
        const uint32_t xt = codes[m] == 0 ? 0u : codes[m] == 2 ? 1u : (x[hq] != 0);
        p = xt ? Z + (p - zb) : zb;
        const uint32_t* row = prefix + (size_t)m * N;
        uint32_t s0 = 0;
        if (L <= N) {
            s0 = p > L / 2 ? p - L / 2 : 0;
            if (s0 > N - L) s0 = N - L;
        }
        for (uint32_t r = 0; r < L; ++r) {
            const uint32_t h = L <= N ? row[s0 + r] : row[r % N];
            pairs[((size_t)m * L + r) * 2] = h;
            pairs[((size_t)m * L + r) * 2 + 1] = (h + 1) % N;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Transition (transition.cu:83-115)                                         */
/* ------------------------------------------------------------------------ */

void sio_transition_log10(double gd0, double gd1, double ne, double rho_rate,
                          float* t_diag, float* t_off) {
    double dist = gd1 - gd0;
    if (dist < 0.0) dist = 0.0;
    double exponent = -4.0 * ne * dist * rho_rate;
    double rho = 1.0 - exp(exponent);
    if (rho < 0.0) rho = 0.0;
    if (rho > 1.0) rho = 1.0;
    double stay = (1.0 - rho) + rho / (2.0 * ne);
    double sw = rho / (2.0 * ne);
    *t_diag = (float)log10(stay);
    *t_off = (sw < 1e-300) ? -999.0f : (float)log10(sw);
}

/* ------------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11)                          */
/* ------------------------------------------------------------------------ */

uint32_t sio_philox_u32(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    return c0;
}

double sio_uniform(uint64_t seed, uint64_t sample_id, uint32_t marker) {
    uint32_t x = sio_philox_u32(marker, (uint32_t)sample_id, (uint32_t)(sample_id >> 32), 0u,
                                (uint32_t)seed, (uint32_t)(seed >> 32));
    return (double)(x >> 8) * (1.0 / 16777216.0);
}

/* ------------------------------------------------------------------------ */
/* FP64 log-space forward-backward                                           */
/* ------------------------------------------------------------------------ */

#define SIO_LOG_ZERO (-999.0)

/* logsumexp2 (logsumexp.cuh:67-70), in double. */
static inline double lse2(double a, double b) {
    double m = a > b ? a : b;
    return log(exp(a - m) + exp(b - m)) + m;
}

/* Emission (emission.cu:35-54): the GL entry picked by the sum of the pair's
 * panel alleles; the log10 value is used unchanged in the natural-log
 * recursions, as the reference does. */
static inline double emission(const float* gl3, uint8_t a0, uint8_t a1) {
    int s = (int)a0 + (int)a1;
    return (double)(s == 0 ? gl3[0] : (s == 1 ? gl3[1] : gl3[2]));
}

void sio_codes_to_gl(const uint8_t* codes, uint64_t n, float* gl) {
    for (uint64_t i = 0; i < n; ++i) {
        float* g = gl + 3 * i;
        switch (codes[i]) {
            case 0: g[0] = 0.0f; g[1] = -999.0f; g[2] = -999.0f; break;
            case 1: g[0] = -999.0f; g[1] = 0.0f; g[2] = -999.0f; break;
            case 2: g[0] = -999.0f; g[1] = -999.0f; g[2] = 0.0f; break;
            default: g[0] = 0.0f; g[1] = 0.0f; g[2] = 0.0f; break;
        }
    }
}

/* Forward pass_kernel (forward_backward.cu:41-142): alpha_0 = E_0, then
 * alpha_m[j] = LSE(-999, alpha_{m-1}[i] + T[i][j] over i) + E_m[j], each row
 * shifted by its max. The sqrt(M) checkpoint/recompute schedule of
 * backward_pass_kernel (:186-280) reproduces these rows exactly, so every row
 * is simply kept. Backward (:181-242): beta_{M-1} = 0, beta_m[i] =
 * LSE(-999, T[i][j] + E_{m+1}[j] + beta_{m+1}[j] over j), never rescaled.
 * Posterior (:283-287): alpha + beta. The reference sampler (sampling.cu:80-100)
 * draws from softmax of that row; dosage and P(hap=1) are taken under the same
 * distribution. */
void sio_fb_sample(const sio_fb_args* a, const float* gl, const uint32_t* pairs,
                   const uint8_t* panel, const float* t_diag, const float* t_off,
                   float* dosage, float* p0, float* p1,
                   uint8_t* hap_argmax, uint8_t* hap_sampled, double* logpost) {
    const uint32_t M = a->M, N = a->N, L = a->L;
    double* alpha = (double*)malloc(sizeof(double) * (size_t)M * L);
    double* e_cur = (double*)malloc(sizeof(double) * L);
    double* beta = (double*)malloc(sizeof(double) * L);
    double* beta_next = (double*)malloc(sizeof(double) * L);
    double* e_next = (double*)malloc(sizeof(double) * L);
    double* w = (double*)malloc(sizeof(double) * L);

#define PAIR0(m, k) pairs[(((size_t)(m) * L + (k)) * 2) + 0]
#define PAIR1(m, k) pairs[(((size_t)(m) * L + (k)) * 2) + 1]
#define ALLELE(m, h) panel[(size_t)(m) * N + (h)]
#define EMIS(m, k) emission(gl + 3 * (size_t)(m), ALLELE(m, PAIR0(m, k)), ALLELE(m, PAIR1(m, k)))

    /* forward */
    for (uint32_t k = 0; k < L; ++k) alpha[k] = EMIS(0, k);
    {
        double mx = alpha[0];
        for (uint32_t k = 1; k < L; ++k) mx = alpha[k] > mx ? alpha[k] : mx;
        for (uint32_t k = 0; k < L; ++k) alpha[k] -= mx;
    }
    for (uint32_t m = 1; m < M; ++m) {
        double td = (double)(a->trans_mode == SIO_TRANS_PER_GAP ? t_diag[m - 1] : t_diag[0]);
        double to = (double)(a->trans_mode == SIO_TRANS_PER_GAP ? t_off[m - 1] : t_off[0]);
        const double* prev = alpha + (size_t)(m - 1) * L;
        double* cur = alpha + (size_t)m * L;
        for (uint32_t j = 0; j < L; ++j) {
            double s = SIO_LOG_ZERO;
            for (uint32_t i = 0; i < L; ++i) s = lse2(s, prev[i] + (i == j ? td : to));
            cur[j] = s + EMIS(m, j);
        }
        double mx = cur[0];
        for (uint32_t k = 1; k < L; ++k) mx = cur[k] > mx ? cur[k] : mx;
        for (uint32_t k = 0; k < L; ++k) cur[k] -= mx;
    }

    /* backward with posterior outputs */
    for (uint32_t k = 0; k < L; ++k) beta[k] = 0.0;
    for (int64_t mm = (int64_t)M - 1; mm >= 0; --mm) {
        uint32_t m = (uint32_t)mm;
        if (m < M - 1) {
            double td = (double)(a->trans_mode == SIO_TRANS_PER_GAP ? t_diag[m] : t_diag[0]);
            double to = (double)(a->trans_mode == SIO_TRANS_PER_GAP ? t_off[m] : t_off[0]);
            for (uint32_t j = 0; j < L; ++j) e_next[j] = EMIS(m + 1, j);
            for (uint32_t i = 0; i < L; ++i) {
                double s = SIO_LOG_ZERO;
                for (uint32_t j = 0; j < L; ++j) s = lse2(s, ((i == j ? td : to) + e_next[j]) + beta_next[j]);
                beta[i] = s;
            }
        }
        /* posterior row */
        const double* al = alpha + (size_t)m * L;
        double mx = -INFINITY;
        for (uint32_t k = 0; k < L; ++k) {
            w[k] = al[k] + beta[k];
            if (logpost) logpost[(size_t)m * L + k] = w[k];
            mx = w[k] > mx ? w[k] : mx;
        }
        double tot = 0.0;
        for (uint32_t k = 0; k < L; ++k) { w[k] = exp(w[k] - mx); tot += w[k]; }
        double ds = 0.0, q0 = 0.0, q1 = 0.0, pmax = 0.0;
        for (uint32_t k = 0; k < L; ++k) {
            double p = w[k] / tot;
            w[k] = p;
            uint8_t x0 = ALLELE(m, PAIR0(m, k)) ? 1 : 0, x1 = ALLELE(m, PAIR1(m, k)) ? 1 : 0;
            ds += p * (x0 + x1); q0 += p * x0; q1 += p * x1;
            pmax = p > pmax ? p : pmax;
        }
        if (dosage) dosage[m] = (float)ds;
        if (p0) p0[m] = (float)q0;
        if (p1) p1[m] = (float)q1;
        if (hap_argmax) {
            /* first slot within tie_eps of the max (sampling.cu:160-169 is the
             * tie_eps = 0 case: strict first max) */
            uint32_t best = 0;
            double thr = pmax * (1.0 - a->tie_eps);
            for (uint32_t k = 0; k < L; ++k) if (w[k] >= thr) { best = k; break; }
            hap_argmax[m] = ALLELE(m, PAIR0(m, best));
            hap_argmax[M + m] = ALLELE(m, PAIR1(m, best));
        }
        if (hap_sampled) {
            /* inverse CDF, first slot whose running sum exceeds u
             * (sampling.cu:103-113), u from Philox instead of XORWOW */
            double u = sio_uniform(a->seed, a->sample_id, m);
            double cum = 0.0;
            uint32_t pick = L;
            for (uint32_t k = 0; k < L; ++k) { cum += w[k]; if (u < cum) { pick = k; break; } }
            if (pick == L) { pick = 0; for (uint32_t k = 0; k < L; ++k) if (w[k] > 0.0) pick = k; }
            hap_sampled[m] = ALLELE(m, PAIR0(m, pick));
            hap_sampled[M + m] = ALLELE(m, PAIR1(m, pick));
        }
        memcpy(beta_next, beta, sizeof(double) * L);
    }
#undef PAIR0
#undef PAIR1
#undef ALLELE
#undef EMIS
    free(alpha); free(e_cur); free(beta); free(beta_next); free(e_next); free(w);
}

typedef struct {
    const sio_fb_args* a;
    uint32_t B;
    const float* gl;
    const uint32_t* pairs;
    const uint8_t* panel;
    const float* t_diag;
    const float* t_off;
    float *dosage, *p0, *p1;
    uint8_t *hap_argmax, *hap_sampled;
    atomic_uint next;
} batch_job;

static void* batch_worker(void* arg) {
    batch_job* j = (batch_job*)arg;
    const uint32_t M = j->a->M;
    for (;;) {
        uint32_t s = atomic_fetch_add(&j->next, 1u);
        if (s >= j->B) break;
        sio_fb_args a = *j->a;
        a.sample_id = j->a->sample_id + s;
        size_t o = (size_t)s * M;
        sio_fb_sample(&a, j->gl + 3 * o, j->pairs, j->panel, j->t_diag, j->t_off,
                      j->dosage ? j->dosage + o : NULL, j->p0 ? j->p0 + o : NULL,
                      j->p1 ? j->p1 + o : NULL,
                      j->hap_argmax ? j->hap_argmax + 2 * o : NULL,
                      j->hap_sampled ? j->hap_sampled + 2 * o : NULL, NULL);
    }
    return NULL;
}

void sio_fb_batch(const sio_fb_args* a, uint32_t B, const float* gl, const uint32_t* pairs,
                  const uint8_t* panel, const float* t_diag, const float* t_off,
                  float* dosage, float* p0, float* p1,
                  uint8_t* hap_argmax, uint8_t* hap_sampled, int n_threads) {
    batch_job j;
    j.a = a; j.B = B; j.gl = gl; j.pairs = pairs; j.panel = panel;
    j.t_diag = t_diag; j.t_off = t_off; j.dosage = dosage; j.p0 = p0; j.p1 = p1;
    j.hap_argmax = hap_argmax; j.hap_sampled = hap_sampled;
    atomic_init(&j.next, 0u);
    if (n_threads < 1) n_threads = 1;
    if (n_threads > 256) n_threads = 256;
    pthread_t th[256];
    for (int t = 0; t < n_threads; ++t) pthread_create(&th[t], NULL, batch_worker, &j);
    for (int t = 0; t < n_threads; ++t) pthread_join(th[t], NULL);
}
