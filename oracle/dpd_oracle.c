/*
 * dpd_oracle.c -- CPU restatement of the 2D DPD step of the reference engine.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker for the CUDA library.  Only
 * tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py load
 * it; the product path never does.
 *
 * Parity status:
 *   - Philox4x32-10 is pinned by the published known-answer vectors of its
 *     authors' Random123 distribution (tests/test_oracle.py);
 *   - mix13 noise, the cell key, the stable cell sort, pair and bond forces,
 *     the Groot-Warren integrator and the soup initialisation are pinned
 *     against the reference engine itself (oracle/_ref, built from
 *     cel/engine/oercel.c) through the fixtures in tests/golden/;
 *   - the three-rule chemistry (ora_chemistry) is PARITY UNPINNED: the
 *     reference has no such reactions.  It follows the reference's mechanism
 *     (keyed per-bead decisions, oercel.c:819-826; nearest partner with gid
 *     tie-break, oercel.c:1387-1396) and resolves conflicts by lowest gid.
 *
 * Built with -ffp-contract=off: every FP32 expression below that mirrors the
 * CUDA kernels spells out its fused multiply-adds with fmaf().
 */
#include "dpd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#define SQRT12 3.4641016151377545870548926830117

/* ------------------------------------------------------------------ counter-based RNGs */

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
 * as 1, 2, 3", SC'11): 10 rounds of two 32x32->64 multiplies with a Weyl key
 * schedule.  Constants are the paper's. */
void ora_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; r++) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* first output word of Philox4x32-10 at counter (a, b, step), key = seed */
uint32_t ora_philox_word(uint64_t seed, uint32_t a, uint32_t b, int64_t step) {
    const uint32_t ctr[4] = {a, b, (uint32_t)(uint64_t)step, (uint32_t)((uint64_t)step >> 32)};
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t o[4];
    ora_philox4x32_10(ctr, key, o);
    return o[0];
}

/* splitmix64 finaliser, oercel.c:124-128 */
uint64_t ora_mix13(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

/* per-step noise key, oercel.c:131-133 */
uint64_t ora_step_seed(uint64_t seed, int64_t step) {
    return ora_mix13(ora_mix13(seed ^ 0x5851f42d4c957f2dULL) ^ ora_mix13((uint64_t)step + 0x632be59bd9b4e019ULL));
}

/* raw 64-bit pair hash of the reference, oercel.c:137-141 (before the map to theta) */
uint64_t ora_mix13_pair(uint64_t sseed, uint32_t gi, uint32_t gj) {
    const uint64_t key = gi < gj ? (((uint64_t)gi << 32) | gj) : (((uint64_t)gj << 32) | gi);
    return ora_mix13((key * 0x9e3779b97f4a7c15ULL) ^ sseed);
}

/* symmetric pair noise theta in FP64, uniform on [-sqrt3, sqrt3).
 * noise 1: the reference's mapping of the full 64-bit hash (oercel.c:140);
 * noise 0: Philox word 0 at counter (min gid, max gid, step), key = seed,
 *          read as a signed 32-bit integer and scaled the same way. */
double ora_theta(const ora_params *P, int64_t step, uint32_t gi, uint32_t gj) {
    const uint32_t lo = gi < gj ? gi : gj, hi = gi < gj ? gj : gi;
    if (P->noise == 1) {
        const uint64_t h = ora_mix13_pair(ora_step_seed(P->seed, step), lo, hi);
        return (double)(int64_t)h * (SQRT12 / 18446744073709551616.0);
    }
    const uint32_t u = ora_philox_word(P->seed, lo, hi, step);
    return (double)(int32_t)u * (SQRT12 / 4294967296.0);
}

/* theta of every pair of n beads at one step (the test models' noise table):
 * out[i n + j] = theta(gid[i], gid[j]), 0 on the diagonal */
void ora_theta_matrix(const ora_params *P, int64_t step, int n, const uint32_t *gid, double *out) {
    for (int i = 0; i < n; i++) {
        out[(size_t)i * n + i] = 0.0;
        for (int j = i + 1; j < n; j++)
            out[(size_t)i * n + j] = out[(size_t)j * n + i] = ora_theta(P, step, gid[i], gid[j]);
    }
}

/* keyed uniform decision word for the chemistry: Philox word 0 at counter
 * (gid, salt, step), key = seed.  Mechanism of oercel.c:819-826 (hash_key /
 * hash_u01: a pure function of seed, step, salt and gid). */
uint32_t ora_decision_word(uint64_t seed, int64_t step, uint32_t salt, uint32_t gid) {
    return ora_philox_word(seed, gid, salt, step);
}

/* ------------------------------------------------------------------ cells and the sort */

/* cell of a position, oercel.c:779-786 with nsub = 1 (the product is taken in
 * FP64 exactly as the reference does; the input is an FP32 coordinate) */
int32_t ora_cell_of(const ora_params *P, float x, float y) {
    int cx = (int)((double)x * P->icsx), cy = (int)((double)y * P->icsy);
    if (cx >= P->ncx) cx = P->ncx - 1;
    if (cy >= P->ncy) cy = P->ncy - 1;
    if (cx < 0) cx = 0;
    if (cy < 0) cy = 0;
    return cx * P->ncy + cy;
}

/* Stable counting sort by cell, oercel.c:832-933: new slot d holds old bead
 * src[d]; beads of one cell keep their old relative order.  cstart has
 * ncell + 1 entries; key[i] is the cell of OLD bead i. */
void ora_sort(const ora_params *P, int32_t n, const float *x, const float *y, int32_t *key, int32_t *cstart,
              int32_t *src) {
    const int nc = P->ncx * P->ncy;
    memset(cstart, 0, (size_t)(nc + 1) * sizeof(int32_t));
    for (int i = 0; i < n; i++) {
        key[i] = ora_cell_of(P, x[i], y[i]);
        cstart[key[i] + 1]++;
    }
    for (int c = 0; c < nc; c++) cstart[c + 1] += cstart[c];
    int32_t *cur = malloc((size_t)(nc + 1) * sizeof(int32_t));
    memcpy(cur, cstart, (size_t)(nc + 1) * sizeof(int32_t));
    for (int i = 0; i < n; i++) src[cur[key[i]]++] = i;
    free(cur);
}

/* ------------------------------------------------------------------ forces (FP64) */

static inline double minimg(double d, double L) {
    const double h = 0.5 * L;
    if (d > h) d -= L;
    else if (d < -h) d += L;
    return d;
}

/* one pair term on bead i from bead j: F = w [a - gamma w (rhat . v_ij) + sigma theta / sqrt(dt)] rhat,
 * w = 1 - r, r < 1 (oercel.c:970-981; SPEC section 2).  dx = x_i - x_j. */
static inline void pair_term(const ora_params *P, double sdt, int64_t step, double dx, double dy, double dvx,
                             double dvy, int ti, int tj, uint32_t gi, uint32_t gj, double *fx, double *fy) {
    const double r2 = dx * dx + dy * dy;
    if (!(r2 < 1.0 && r2 > 1e-24)) return;
    const double r = sqrt(r2), ir = 1.0 / r, w = 1.0 - r;
    const double rv = (dx * dvx + dy * dvy) * ir;
    const double th = sdt != 0.0 ? ora_theta(P, step, gi, gj) : 0.0;
    const double fm = w * (P->a[ti * ORA_MAXT + tj] - P->gamma * w * rv + sdt * th) * ir;
    *fx += fm * dx;
    *fy += fm * dy;
}

/* sigma / sqrt(dt) with sigma = sqrt(2 gamma kT), oercel.c:579, 1204 */
double ora_sdt(const ora_params *P) { return sqrt(2.0 * P->gamma * P->kT) / sqrt(P->dt); }

/* sigma / sqrt(dt) of a step with the temperature cycle: kT_at (oercel.c:622-624)
 * at t = t_anchor + (step - step_anchor) dt (oercel.c:2353), then oercel.c:1204 */
double ora_sdt_at(const ora_params *P, int64_t step) {
    if (P->kT_amp == 0.0) return ora_sdt(P);
    const double t = P->t_anchor + (double)(step - P->step_anchor) * P->dt;
    const double kT = P->kT + P->kT_amp * sin(2.0 * M_PI * t / P->kT_period);
    return sqrt(2.0 * P->gamma * kT) / sqrt(P->dt);
}

/* Stirring body force (oercel.c:1166-1195): f_x = A sin(2 pi n y / L) on every
 * bead, minus the mean over the beads so that the net force is zero. Added to fx. */
void ora_stir_forces(const ora_params *P, int32_t n, const float *y, double *fx) {
    if (P->stir_A == 0.0 || n < 1) return;
    const double kn = (double)P->stir_n / P->L;
    double sum = 0.0;
    for (int i = 0; i < n; i++) sum += P->stir_A * sin(2.0 * M_PI * kn * (double)y[i]);
    const double mean = sum / n;
    for (int i = 0; i < n; i++) fx[i] += P->stir_A * sin(2.0 * M_PI * kn * (double)y[i]) - mean;
}

/* Pair forces through the cell list (input sorted by ora_sort): every bead
 * sums over the 3x3 neighbour cells (reference stencil oercel.c:1060-1120
 * visits the same pairs once each; here each pair is seen from both ends). */
void ora_pair_forces(const ora_params *P, int32_t n, const float *x, const float *y, const float *vtx,
                     const float *vty, const uint8_t *type, const uint32_t *gid, const int32_t *cstart, int64_t step,
                     int32_t with_noise, double *fx, double *fy) {
    const int ncx = P->ncx, ncy = P->ncy;
    const double L = P->L, sdt = with_noise ? ora_sdt_at(P, step) : 0.0;
    (void)n;
    for (int cx = 0; cx < ncx; cx++)
        for (int cy = 0; cy < ncy; cy++) {
            const int c = cx * ncy + cy;
            for (int i = cstart[c]; i < cstart[c + 1]; i++) {
                double ax = 0.0, ay = 0.0;
                for (int ox = -1; ox <= 1; ox++)
                    for (int oy = -1; oy <= 1; oy++) {
                        const int nx = (cx + ox + ncx) % ncx, ny = (cy + oy + ncy) % ncy;
                        const int cc = nx * ncy + ny;
                        for (int j = cstart[cc]; j < cstart[cc + 1]; j++) {
                            if (j == i) continue;
                            pair_term(P, sdt, step, minimg((double)x[i] - (double)x[j], L),
                                      minimg((double)y[i] - (double)y[j], L), (double)vtx[i] - (double)vtx[j],
                                      (double)vty[i] - (double)vty[j], type[i], type[j], gid[i], gid[j], &ax, &ay);
                        }
                    }
                fx[i] = ax;
                fy[i] = ay;
            }
        }
}

/* O(N^2) brute force over all pairs with the minimum image, the template of
 * cel/engine/tests/forcetest.c:91-101 */
void ora_pair_forces_brute(const ora_params *P, int32_t n, const float *x, const float *y, const float *vtx,
                           const float *vty, const uint8_t *type, const uint32_t *gid, int64_t step,
                           int32_t with_noise, double *fx, double *fy) {
    const double L = P->L, sdt = with_noise ? ora_sdt_at(P, step) : 0.0;
    for (int i = 0; i < n; i++) {
        double ax = 0.0, ay = 0.0;
        for (int j = 0; j < n; j++) {
            if (j == i) continue;
            pair_term(P, sdt, step, minimg((double)x[i] - (double)x[j], L), minimg((double)y[i] - (double)y[j], L),
                      (double)vtx[i] - (double)vtx[j], (double)vty[i] - (double)vty[j], type[i], type[j], gid[i],
                      gid[j], &ax, &ay);
        }
        fx[i] = ax;
        fy[i] = ay;
    }
}

/* Harmonic bonds U = k/2 (r - r0)^2 along the prev/next links, added to
 * fx/fy (oercel.c:1272-1308), and the angle terms when k_angle != 0.  Returns the largest bond
 * length in *maxbond (running max, oercel.c:1292). */
void ora_bond_forces(const ora_params *P, int32_t n, const float *x, const float *y, const int32_t *next,
                     double *fx, double *fy, double *maxbond) {
    const double L = P->L;
    double mb = *maxbond;
    for (int i = 0; i < n; i++) {
        const int j = next[i];
        if (j < 0) continue;
        const double dx = minimg((double)x[j] - (double)x[i], L), dy = minimg((double)y[j] - (double)y[i], L);
        const double r = sqrt(dx * dx + dy * dy);
        if (r > mb) mb = r;
        const double f = -P->k_bond * (r - P->r0) / r; /* force on j along (dx, dy) */
        fx[j] += f * dx;
        fy[j] += f * dy;
        fx[i] -= f * dx;
        fy[i] -= f * dy;
    }
    /* angle terms U = k (1 - cos theta) of every consecutive triplet (prev, j,
     * next) along the links (chain_forces_linear, oercel.c:1290-1307) */
    if (P->k_angle != 0.0) {
        int32_t *prev = (int32_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int32_t));
        for (int i = 0; i < n; i++) prev[i] = -1;
        for (int i = 0; i < n; i++)
            if (next[i] >= 0) prev[next[i]] = i;
        const double ka = P->k_angle;
        for (int j = 0; j < n; j++) {
            const int i = prev[j], k = next[j];
            if (i < 0 || k < 0) continue;
            const double ax = minimg((double)x[j] - (double)x[i], L), ay = minimg((double)y[j] - (double)y[i], L);
            const double cx = minimg((double)x[k] - (double)x[j], L), cy = minimg((double)y[k] - (double)y[j], L);
            const double la = sqrt(ax * ax + ay * ay), lc = sqrt(cx * cx + cy * cy);
            const double ilac = 1.0 / (la * lc);
            const double cs = (ax * cx + ay * cy) * ilac;
            const double dUax = -ka * (cx * ilac - cs * ax / (la * la));
            const double dUay = -ka * (cy * ilac - cs * ay / (la * la));
            const double dUcx = -ka * (ax * ilac - cs * cx / (lc * lc));
            const double dUcy = -ka * (ay * ilac - cs * cy / (lc * lc));
            fx[i] += dUax;
            fy[i] += dUay;
            fx[j] += -dUax + dUcx;
            fy[j] += -dUay + dUcy;
            fx[k] -= dUcx;
            fy[k] -= dUcy;
        }
        free(prev);
    }
    *maxbond = mb;
}

/* Bonded forces of branched lipids from a molecule template (mol_forces,
 * oercel.c:1221-1257): for every molecule (a bead with no prev and a next; its
 * beads follow next in template order) each template bond (position pair,
 * rest length, spring k_bond) and angle term (kind 0: U = K (1 - cos), kind 1:
 * U = K (cos - c0)^2) is added to the beads it joins. */
void ora_mol_forces(const ora_params *P, const ora_mol *M, int32_t n, const float *x, const float *y,
                    const int32_t *next, double *fx, double *fy, double *maxbond) {
    const double L = P->L;
    double mb = *maxbond;
    char *haspv = (char *)calloc((size_t)(n > 0 ? n : 1), 1);
    for (int i = 0; i < n; i++)
        if (next[i] >= 0) haspv[next[i]] = 1;
    for (int h = 0; h < n; h++) {
        if (haspv[h] || next[h] < 0) continue;
        int sl[ORA_MAXML], m = 0;
        for (int d = h; d >= 0 && m < M->mlen; d = next[d]) sl[m++] = d;
        if (m != M->mlen) continue;
        for (int q = 0; q < M->nb; q++) {
            const int i = sl[M->bi[q]], j = sl[M->bj[q]];
            const double dx = minimg((double)x[j] - (double)x[i], L), dy = minimg((double)y[j] - (double)y[i], L);
            const double r = sqrt(dx * dx + dy * dy);
            if (r > mb) mb = r;
            const double f = -P->k_bond * (r - M->br0[q]) / r; /* force on j along (dx, dy) */
            fx[j] += f * dx;
            fy[j] += f * dy;
            fx[i] -= f * dx;
            fy[i] -= f * dy;
        }
        for (int q = 0; q < M->na; q++) {
            const int i = sl[M->ai[q]], j = sl[M->aj[q]], k = sl[M->ak[q]];
            const double ax = minimg((double)x[j] - (double)x[i], L), ay = minimg((double)y[j] - (double)y[i], L);
            const double cx = minimg((double)x[k] - (double)x[j], L), cy = minimg((double)y[k] - (double)y[j], L);
            const double la = sqrt(ax * ax + ay * ay), lc = sqrt(cx * cx + cy * cy);
            const double ilac = 1.0 / (la * lc);
            const double cs = (ax * cx + ay * cy) * ilac;
            const double g = M->akind[q] == 0 ? -M->aK[q] : 2.0 * M->aK[q] * (cs - M->ac0[q]); /* dU/dcos */
            const double dUax = g * (cx * ilac - cs * ax / (la * la)), dUay = g * (cy * ilac - cs * ay / (la * la));
            const double dUcx = g * (ax * ilac - cs * cx / (lc * lc)), dUcy = g * (ay * ilac - cs * cy / (lc * lc));
            fx[i] += dUax;
            fy[i] += dUay;
            fx[j] += -dUax + dUcx;
            fy[j] += -dUay + dUcy;
            fx[k] -= dUcx;
            fy[k] -= dUcy;
        }
    }
    free(haspv);
    *maxbond = mb;
}

/* ------------------------------------------------------------------ integrator */

/* Groot-Warren step with stored half-step velocity (oercel.c:2303-2334):
 *   x += dt vh + dt^2 f ; vt = vh + (1/2 + lambda) dt f ; vh += dt f ; wrap.
 * FP32 mirror of the CUDA kernel: the same roundings in the same order.
 * Returns the number of beads whose wrapped coordinate left [0, L). */
int32_t ora_integrate_f32(const ora_f32c *C, int32_t n, float *x, float *y, float *vhx, float *vhy, float *vtx,
                          float *vty, const float *fx, const float *fy) {
    int32_t bad = 0;
    for (int i = 0; i < n; i++) {
        const float ddx = fmaf(C->dt2, fx[i], C->dt * vhx[i]);
        const float ddy = fmaf(C->dt2, fy[i], C->dt * vhy[i]);
        float xi = x[i] + ddx, yi = y[i] + ddy;
        xi = xi < 0.0f ? xi + C->L : xi;
        yi = yi < 0.0f ? yi + C->L : yi;
        xi = xi >= C->L ? xi - C->L : xi;
        yi = yi >= C->L ? yi - C->L : yi;
        bad += !(xi >= 0.0f && xi < C->L && yi >= 0.0f && yi < C->L);
        x[i] = xi;
        y[i] = yi;
        vtx[i] = fmaf(C->cvt, fx[i], vhx[i]);
        vty[i] = fmaf(C->cvt, fy[i], vhy[i]);
        vhx[i] = fmaf(C->dt, fx[i], vhx[i]);
        vhy[i] = fmaf(C->dt, fy[i], vhy[i]);
    }
    return bad;
}

/* the same step in FP64, as the reference computes it */
void ora_integrate_f64(const ora_params *P, int32_t n, double *x, double *y, double *vhx, double *vhy, double *vtx,
                       double *vty, const double *fx, const double *fy) {
    const double dt = P->dt, dt2 = dt * dt, cvt = (0.5 + P->lambda) * dt, L = P->L;
    for (int i = 0; i < n; i++) {
        const double ddx = dt * vhx[i] + dt2 * fx[i], ddy = dt * vhy[i] + dt2 * fy[i];
        double xi = x[i] + ddx, yi = y[i] + ddy;
        xi = xi < 0.0 ? xi + L : xi;
        yi = yi < 0.0 ? yi + L : yi;
        xi = xi >= L ? xi - L : xi;
        yi = yi >= L ? yi - L : yi;
        x[i] = xi;
        y[i] = yi;
        vtx[i] = vhx[i] + cvt * fx[i];
        vty[i] = vhy[i] + cvt * fy[i];
        vhx[i] += dt * fx[i];
        vhy[i] += dt * fy[i];
    }
}

/* ------------------------------------------------------------------ chemistry (parity unpinned) */

enum { T_W = 0, T_H = 1, T_T = 2, T_P = 3 };

/* squared minimum-image distance in FP32, mirroring the CUDA kernel */
static inline float dist2_f32(float xa, float ya, float xb, float yb, float L) {
    const float h = 0.5f * L;
    float dx = xb - xa, dy = yb - ya;
    dx = dx > h ? dx - L : (dx < -h ? dx + L : dx);
    dy = dy > h ? dy - L : (dy < -h ? dy + L : dy);
    return dx * dx + dy * dy;
}

/* chain length and head type of the chain that contains tail end e (walk prev) */
static int chain_from_tail(const int32_t *prev, const uint8_t *type, int e, int maxwalk, int *head_type) {
    int len = 1, c = e;
    while (prev[c] >= 0 && len <= maxwalk) {
        c = prev[c];
        len++;
    }
    *head_type = type[c];
    return len;
}

/* is bead e a growable H-terminated chain end: the tail of a chain whose head
 * is H and which is shorter than max_chain, or a lone (unbonded) H */
static int growable_end(const int32_t *prev, const int32_t *next, const uint8_t *type, int e, int max_chain) {
    if (next[e] >= 0) return 0;
    if (type[e] == T_H) return prev[e] < 0;
    if (type[e] != T_T || prev[e] < 0) return 0;
    int ht;
    const int len = chain_from_tail(prev, type, e, max_chain, &ht);
    return ht == T_H && len < max_chain;
}

typedef struct { int target; uint32_t d_gid; float d2; } req_t;

/* nearest bead satisfying `want` within r2 of bead p through the 3x3 cells
 * (ties: lowest gid, oercel.c:1387-1396); returns slot or -1 */
static int nearest(const ora_params *P, int32_t n, const float *x, const float *y, const uint32_t *gid,
                   const int32_t *cstart, int p, float r2, int (*want)(void *, int), void *ctx, float *d2out) {
    const int ncx = P->ncx, ncy = P->ncy;
    const float L = (float)P->L;
    const int c = ora_cell_of(P, x[p], y[p]);
    const int cx = c / ncy, cy = c % ncy;
    int best = -1;
    float bd = 0.0f;
    for (int ox = -1; ox <= 1; ox++)
        for (int oy = -1; oy <= 1; oy++) {
            const int cc = ((cx + ox + ncx) % ncx) * ncy + (cy + oy + ncy) % ncy;
            for (int j = cstart[cc]; j < cstart[cc + 1]; j++) {
                if (j == p || !want(ctx, j)) continue;
                const float d2 = dist2_f32(x[p], y[p], x[j], y[j], L);
                if (!(d2 < r2)) continue;
                if (best < 0 || d2 < bd || (d2 == bd && gid[j] < gid[best])) {
                    best = j;
                    bd = d2;
                }
            }
        }
    (void)n;
    if (d2out) *d2out = bd;
    return best;
}

typedef struct { const int32_t *prev, *next; const uint8_t *type; int max_chain; } wctx_t;
static int want_t(void *c, int j) { return ((wctx_t *)c)->type[j] == T_T; }
static int want_end(void *c, int j) {
    wctx_t *w = c;
    return growable_end(w->prev, w->next, w->type, j, w->max_chain);
}
static int want_free_h(void *c, int j) {
    wctx_t *w = c;
    return w->type[j] == T_H && w->prev[j] < 0 && w->next[j] < 0;
}

static int count_t_within(const ora_params *P, const float *x, const float *y, const uint8_t *type,
                          const int32_t *cstart, int p, float r2) {
    const int ncx = P->ncx, ncy = P->ncy;
    const float L = (float)P->L;
    const int c = ora_cell_of(P, x[p], y[p]);
    const int cx = c / ncy, cy = c % ncy;
    int k = 0;
    for (int ox = -1; ox <= 1; ox++)
        for (int oy = -1; oy <= 1; oy++) {
            const int cc = ((cx + ox + ncx) % ncx) * ncy + (cy + oy + ncy) % ncy;
            for (int j = cstart[cc]; j < cstart[cc + 1]; j++)
                if (j != p && type[j] == T_T && dist2_f32(x[p], y[p], x[j], y[j], L) < r2) k++;
        }
    return k;
}

static void push_event(ora_event *ev, int evcap, int *nev, int64_t step, int kind, uint32_t g, uint32_t pg, float x,
                       float y) {
    if (*nev < evcap) {
        ev[*nev].step = step;
        ev[*nev].kind = kind;
        ev[*nev].gid = g;
        ev[*nev].partner = pg;
        ev[*nev].x = x;
        ev[*nev].y = y;
        ev[*nev].pad = 0;
    }
    (*nev)++;
}

/* One chemistry pass on a cell-sorted state, three stages in this order, each
 * decided on the state left by the previous stage:
 *   1 brk : every H whose next bead is T breaks that bond if u(1, gid_H) < thr_break;
 *   2 grow: every P with >= n_t_min T beads within r_grow and u(2, gid_P) < thr_grow
 *           requests its nearest growable H-terminated chain end within r_grow;
 *           per end the lowest requesting gid wins; the winner becomes T and
 *           the end's new next bead;
 *   3 bond: every free T with u(3, gid_T) < thr_bond requests its nearest free
 *           H within r_bond; per H the lowest requesting gid wins; H.next = T.
 * Within a stage, requests see the stage's starting state only.  Events are
 * appended stage by stage in increasing gid order.  Returns the event count. */
int32_t ora_chemistry(const ora_params *P, const ora_chem *C, int32_t n, const float *x, const float *y, uint8_t *type,
                      const uint32_t *gid, int32_t *prev, int32_t *next, const int32_t *cstart, int64_t step,
                      ora_event *ev, int32_t evcap) {
    int nev = 0;
    /* order of beads by gid, for the serial lowest-gid-first application */
    int32_t *byg = malloc((size_t)n * sizeof(int32_t));
    for (int i = 0; i < n; i++) byg[gid[i]] = i;
    /* stage 1: breaks */
    for (int g = 0; g < n; g++) {
        const int h = byg[g];
        const int t = next[h];
        if (type[h] != T_H || t < 0 || type[t] != T_T) continue;
        if (ora_decision_word(P->seed, step, 1, gid[h]) < C->thr_break) {
            next[h] = -1;
            prev[t] = -1;
            push_event(ev, evcap, &nev, step, 1, gid[h], gid[t], x[h], y[h]);
        }
    }
    /* stage 2: growth, requests on the stage-2 snapshot */
    {
        wctx_t w = {prev, next, type, C->max_chain};
        int *tgt = malloc((size_t)n * sizeof(int));
        for (int g = 0; g < n; g++) {
            const int p = byg[g];
            tgt[g] = -1;
            if (type[p] != T_P) continue;
            if (!(ora_decision_word(P->seed, step, 2, gid[p]) < C->thr_grow)) continue;
            if (count_t_within(P, x, y, type, cstart, p, C->r2_grow) < C->n_t_min) continue;
            tgt[g] = nearest(P, n, x, y, gid, cstart, p, C->r2_grow, want_end, &w, NULL);
        }
        /* lowest gid wins: apply in gid order, a claimed end refuses later requests */
        uint8_t *taken = calloc((size_t)n, 1);
        for (int g = 0; g < n; g++) {
            const int e = tgt[g];
            if (e < 0 || taken[e]) continue;
            taken[e] = 1;
            const int p = byg[g];
            type[p] = T_T;
            next[e] = p;
            prev[p] = e;
            next[p] = -1;
            push_event(ev, evcap, &nev, step, 0, gid[p], gid[e], x[p], y[p]);
        }
        free(taken);
        free(tgt);
    }
    /* stage 3: free T + free H bonding, requests on the stage-3 snapshot */
    {
        wctx_t w = {prev, next, type, C->max_chain};
        int *tgt = malloc((size_t)n * sizeof(int));
        for (int g = 0; g < n; g++) {
            const int t = byg[g];
            tgt[g] = -1;
            if (type[t] != T_T || prev[t] >= 0 || next[t] >= 0) continue;
            if (!(ora_decision_word(P->seed, step, 3, gid[t]) < C->thr_bond)) continue;
            tgt[g] = nearest(P, n, x, y, gid, cstart, t, C->r2_bond, want_free_h, &w, NULL);
        }
        uint8_t *taken = calloc((size_t)n, 1);
        for (int g = 0; g < n; g++) {
            const int h = tgt[g];
            if (h < 0 || taken[h]) continue;
            taken[h] = 1;
            const int t = byg[g];
            next[h] = t;
            prev[t] = h;
            push_event(ev, evcap, &nev, step, 2, gid[t], gid[h], x[t], y[t]);
        }
        free(taken);
        free(tgt);
    }
    (void)want_t;
    free(byg);
    return nev;
}

/* ------------------------------------------------------------------ observables */

/* Kinetic temperature from the full velocity v = vh + dt/2 f over 2N - 2
 * degrees of freedom (oercel.c:2059-2071), total momentum, conservative
 * virial (1/V) sum_{i<j} a_ij (1 - r) r (cel/engine_gpu/tests/compare.py:96),
 * and the largest bond length.  out = {T, px, py, virial, maxbond}. */
void ora_observables(const ora_params *P, int32_t n, const float *x, const float *y, const float *vhx,
                     const float *vhy, const float *fx, const float *fy, const uint8_t *type, const int32_t *next,
                     const int32_t *cstart, double *out) {
    const double h = 0.5 * P->dt, L = P->L;
    double k2 = 0, sx = 0, sy = 0;
    for (int i = 0; i < n; i++) {
        const double vx = (double)vhx[i] + h * (double)fx[i], vy = (double)vhy[i] + h * (double)fy[i];
        k2 += vx * vx + vy * vy;
        sx += vx;
        sy += vy;
    }
    double vir = 0.0, mb = 0.0;
    const int ncx = P->ncx, ncy = P->ncy;
    for (int cx = 0; cx < ncx; cx++)
        for (int cy = 0; cy < ncy; cy++) {
            const int c = cx * ncy + cy;
            for (int i = cstart[c]; i < cstart[c + 1]; i++)
                for (int ox = -1; ox <= 1; ox++)
                    for (int oy = -1; oy <= 1; oy++) {
                        const int cc = ((cx + ox + ncx) % ncx) * ncy + (cy + oy + ncy) % ncy;
                        for (int j = cstart[cc]; j < cstart[cc + 1]; j++) {
                            if (j <= i) continue;
                            const double dx = minimg((double)x[i] - (double)x[j], L);
                            const double dy = minimg((double)y[i] - (double)y[j], L);
                            const double r2 = dx * dx + dy * dy;
                            if (!(r2 < 1.0 && r2 > 1e-24)) continue;
                            const double r = sqrt(r2);
                            vir += P->a[type[i] * ORA_MAXT + type[j]] * (1.0 - r) * r;
                        }
                    }
        }
    for (int i = 0; i < n; i++) {
        const int j = next[i];
        if (j < 0) continue;
        const double dx = minimg((double)x[j] - (double)x[i], L), dy = minimg((double)y[j] - (double)y[i], L);
        const double r = sqrt(dx * dx + dy * dy);
        if (r > mb) mb = r;
    }
    out[0] = k2 / (2.0 * n - 2.0);
    out[1] = sx;
    out[2] = sy;
    out[3] = vir / (L * L);
    out[4] = mb;
}

/* Histogram of minimum-image distances between beads of types ta and tb
 * (each unordered pair once; ta == tb allowed) in nbin bins on [0, rmax),
 * over the (2R+1)^2 cells with R = ceil(rmax * ncx / L).  Pattern of
 * cel/engine/tests/snapcheck.py:86-117. */
void ora_pair_hist(const ora_params *P, int32_t n, const float *x, const float *y, const uint8_t *type,
                   const int32_t *cstart, int32_t ta, int32_t tb, double rmax, int32_t nbin, double *hist) {
    const int ncx = P->ncx, ncy = P->ncy;
    const double L = P->L;
    int R = (int)ceil(rmax * P->icsx);
    if (2 * R + 1 > ncx) R = (ncx - 1) / 2;
    (void)n;
    for (int cx = 0; cx < ncx; cx++)
        for (int cy = 0; cy < ncy; cy++) {
            const int c = cx * ncy + cy;
            for (int i = cstart[c]; i < cstart[c + 1]; i++)
                for (int ox = -R; ox <= R; ox++)
                    for (int oy = -R; oy <= R; oy++) {
                        const int cc = ((cx + ox + ncx) % ncx) * ncy + (cy + oy + ncy) % ncy;
                        for (int j = cstart[cc]; j < cstart[cc + 1]; j++) {
                            if (j <= i) continue;
                            if (!((type[i] == ta && type[j] == tb) || (type[i] == tb && type[j] == ta))) continue;
                            const double dx = minimg((double)x[i] - (double)x[j], L);
                            const double dy = minimg((double)y[i] - (double)y[j], L);
                            const double r = sqrt(dx * dx + dy * dy);
                            if (r >= rmax) continue;
                            const int b = (int)(r / rmax * nbin);
                            if (b >= 0 && b < nbin) hist[b] += 1.0;
                        }
                    }
        }
}

/* ------------------------------------------------------------------ soup initialisation */

/* xoshiro256** and its seeding, oercel.c:143-174 */
typedef struct { uint64_t s[4]; } rng_t;
static inline uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static uint64_t rng_next(rng_t *r) {
    uint64_t *s = r->s;
    const uint64_t result = rotl64(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl64(s[3], 45);
    return result;
}
static void rng_seed(rng_t *r, uint64_t seed) {
    uint64_t z = seed;
    for (int k = 0; k < 4; k++) {
        z += 0x9e3779b97f4a7c15ULL;
        r->s[k] = ora_mix13(z);
    }
}
static double rng_unif(rng_t *r) { return (double)(rng_next(r) >> 11) * 0x1.0p-53; }
static double rng_normal(rng_t *r) {
    double u1 = rng_unif(r);
    const double u2 = rng_unif(r);
    if (u1 < 1e-300) u1 = 1e-300;
    return sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
}

static void wrap1(double *p, double L) {
    double v = *p;
    if (v < 0.0) {
        v += L;
        if (v >= L) v -= L;
    } else if (v >= L) {
        v -= L;
        if (v >= L || v < 0.0) v = fmod(v, L);
    }
    *p = v;
}

/* Random soup of the reference (init_soup oercel.c:1774-1814 for the linear
 * lipid, then set_velocities oercel.c:1757-1772) with the same draws in the
 * same order, so one seed gives the reference's state.  Lipids of nH heads +
 * nT tails are straight chains at spacing r0 from a uniform head position;
 * the remaining beads are uniform: first nKa beads type 4, nKb type 5, nN
 * type 3 (P here, N in the reference), the rest W.  next[] links each lipid
 * bead to the following one (the reference's nxt[]), prev[] the inverse.
 * Returns the number of beads placed in lipids. */
int32_t ora_init_soup(double L, int32_t N, uint64_t seed, double kT, double r0, int32_t nH, int32_t nT,
                      double f_lip, double f_Ka, double f_Kb, double c_N, double *x, double *y, double *vx, double *vy,
                      uint8_t *type, uint32_t *gid, int32_t *prev, int32_t *next) {
    rng_t rng;
    rng_seed(&rng, seed);
    const int ml = nH + nT;
    const long nlip = lround(f_lip * N / ml);
    const long nKa = lround(f_Ka * N), nKb = lround(f_Kb * N), nNn = lround(c_N * N);
    if (nlip * ml + nKa + nKb + nNn > N) return -1;
    for (int i = 0; i < N; i++) prev[i] = next[i] = -1;
    int gi = 0;
    for (long m = 0; m < nlip; m++) {
        const double hx = L * rng_unif(&rng), hy = L * rng_unif(&rng);
        const double phi = 2.0 * M_PI * rng_unif(&rng);
        for (int b = 0; b < ml; b++) {
            x[gi] = hx + b * r0 * cos(phi);
            y[gi] = hy + b * r0 * sin(phi);
            wrap1(&x[gi], L);
            wrap1(&y[gi], L);
            type[gi] = b < nH ? 1 : 2;
            gid[gi] = (uint32_t)gi;
            if (b + 1 < ml) next[gi] = gi + 1;
            if (b > 0) prev[gi] = gi - 1;
            gi++;
        }
    }
    const int nl = gi;
    long cnt = 0;
    for (; gi < N; gi++, cnt++) {
        x[gi] = L * rng_unif(&rng);
        y[gi] = L * rng_unif(&rng);
        gid[gi] = (uint32_t)gi;
        if (cnt < nKa) type[gi] = 4;
        else if (cnt < nKa + nKb) type[gi] = 5;
        else if (cnt < nKa + nKb + nNn) type[gi] = 3;
        else type[gi] = 0;
    }
    /* set_velocities */
    double px = 0, py = 0;
    for (int i = 0; i < N; i++) {
        vx[i] = rng_normal(&rng) * sqrt(kT);
        vy[i] = rng_normal(&rng) * sqrt(kT);
        px += vx[i];
        py += vy[i];
    }
    px /= N;
    py /= N;
    double k2 = 0;
    for (int i = 0; i < N; i++) {
        vx[i] -= px;
        vy[i] -= py;
        k2 += vx[i] * vx[i] + vy[i] * vy[i];
    }
    const double sc = sqrt(kT * (2.0 * N - 2.0) / k2);
    for (int i = 0; i < N; i++) {
        vx[i] *= sc;
        vy[i] *= sc;
    }
    return nl;
}

/* ------------------------------------------------------------------ the catalyst chemistry */

/* counter-based uniform deviate of the reference, oercel.c:819-826 */
static uint64_t cat_hash_key(uint64_t seed, int64_t step, uint64_t salt) {
    return ora_mix13(seed ^ ora_mix13((uint64_t)step * 0x9e3779b97f4a7c15ULL + salt));
}
static double cat_hash_u01(uint64_t key, uint32_t g) {
    return (double)(ora_mix13(key ^ ((uint64_t)g * 0xd1b54a32d192ed03ULL)) >> 11) * 0x1.0p-53;
}
/* oercel.c:164-167 */
static long cat_rng_below(rng_t *r, long n) {
    long k = (long)(rng_unif(r) * (double)n);
    return k >= n ? n - 1 : k;
}

/* cell of an FP64 position (cell_of_pos with nsub = 1, oercel.c:779-786) */
static int cat_cell(const ora_params *P, double x, double y) {
    int cx = (int)(x * P->icsx), cy = (int)(y * P->icsy);
    cx = cx >= P->ncx ? P->ncx - 1 : (cx < 0 ? 0 : cx);
    cy = cy >= P->ncy ? P->ncy - 1 : (cy < 0 ? 0 : cy);
    return cx * P->ncy + cy;
}

#define CAT_MARGIN 0.5 /* oercel.c:1348 */
typedef struct { int slot; double d2; } cat_nbr;

/* beads of one type within rcut of (xk, yk), nearest first, ties by lower gid
 * (find_type_near, oercel.c:1353-1398; at most maxout, counted in scan order) */
static int cat_find(const ora_params *P, const float *x, const float *y, const uint8_t *type, const uint32_t *gid,
                    const int32_t *cstart, int ks, double xk, double yk, double rcut, int want, cat_nbr *out,
                    int maxout) {
    const double L = P->L, r2c = rcut * rcut;
    const int ncx = P->ncx, ncy = P->ncy;
    const int c = cat_cell(P, xk, yk), cx = c / ncy, cy = c % ncy;
    const int rx = (int)ceil((rcut + CAT_MARGIN) * P->icsx), ry = (int)ceil((rcut + CAT_MARGIN) * P->icsy);
    int n = 0;
    for (int ox = -rx; ox <= rx; ox++) {
        int cxx = cx + ox;
        cxx += cxx < 0 ? ncx : 0;
        cxx -= cxx >= ncx ? ncx : 0;
        const int base = cxx * ncy, lo = cy - ry, hi = cy + ry;
        int r0[2], r1[2], nr = 0;
        if (lo >= 0 && hi < ncy) { r0[nr] = cstart[base + lo]; r1[nr] = cstart[base + hi + 1]; nr++; }
        else if (lo < 0) {
            r0[nr] = cstart[base + lo + ncy]; r1[nr] = cstart[base + ncy]; nr++;
            r0[nr] = cstart[base]; r1[nr] = cstart[base + hi + 1]; nr++;
        } else {
            r0[nr] = cstart[base + lo]; r1[nr] = cstart[base + ncy]; nr++;
            r0[nr] = cstart[base]; r1[nr] = cstart[base + hi - ncy + 1]; nr++;
        }
        for (int q = 0; q < nr; q++)
            for (int j = r0[q]; j < r1[q]; j++) {
                if (type[j] != want || j == ks) continue;
                const double dx = minimg((double)x[j] - xk, L), dy = minimg((double)y[j] - yk, L);
                const double d2 = dx * dx + dy * dy;
                if (d2 < r2c && n < maxout) { out[n].slot = j; out[n].d2 = d2; n++; }
            }
    }
    for (int a = 1; a < n; a++) {
        const cat_nbr t = out[a];
        int b = a - 1;
        while (b >= 0 && (out[b].d2 > t.d2 || (out[b].d2 == t.d2 && gid[out[b].slot] > gid[t.slot]))) {
            out[b + 1] = out[b];
            b--;
        }
        out[b + 1] = t;
    }
    return n;
}

/* overlap energy of a would-be straight chain (centre c0, direction u) with
 * every bead outside it (chain_overlap_energy, oercel.c:1425-1468) */
static double cat_chain_energy(const ora_params *P, const ora_cat *K, const float *x, const float *y,
                               const uint8_t *type, const int32_t *cstart, double cx0, double cy0, double ux, double uy,
                               const int *sl, int ml) {
    const int ncx = P->ncx, ncy = P->ncy;
    const double L = P->L;
    double U = 0.0;
    for (int b = 0; b < ml; b++) {
        const double off = (b - 0.5 * (ml - 1)) * P->r0;
        double px = cx0 + off * ux, py = cy0 + off * uy;
        wrap1(&px, L);
        wrap1(&py, L);
        const int tb = b < K->nH ? 1 : 2;
        const int c = cat_cell(P, px, py), cx = c / ncy, cy = c % ncy;
        const int rx = (int)ceil((1.0 + CAT_MARGIN) * P->icsx), ry = (int)ceil((1.0 + CAT_MARGIN) * P->icsy);
        for (int ox = -rx; ox <= rx; ox++) {
            int cxx = cx + ox;
            cxx += cxx < 0 ? ncx : 0;
            cxx -= cxx >= ncx ? ncx : 0;
            for (int oy = -ry; oy <= ry; oy++) {
                int cyy = cy + oy;
                cyy += cyy < 0 ? ncy : 0;
                cyy -= cyy >= ncy ? ncy : 0;
                const int cc = cxx * ncy + cyy;
                for (int j = cstart[cc]; j < cstart[cc + 1]; j++) {
                    int skip = 0;
                    for (int q = 0; q < ml; q++) skip |= j == sl[q];
                    if (skip) continue;
                    const double dx = minimg((double)x[j] - px, L), dy = minimg((double)y[j] - py, L);
                    const double r2 = dx * dx + dy * dy;
                    if (r2 >= 1.0) continue;
                    const double w = 1.0 - sqrt(r2);
                    U += 0.5 * P->a[tb * ORA_MAXT + type[j]] * w * w;
                }
            }
        }
    }
    return U;
}

/* steepest-descent relaxation of a new chain whose FP64 positions are
 * (px, py)[0..ml) against its frozen surroundings (relax_new_chain,
 * oercel.c:1473-1560, the linear-template branch) */
static void cat_relax(const ora_params *P, const ora_cat *K, const float *x, const float *y, const uint8_t *type,
                      const int32_t *cstart, const int *sl, int ml, double *px, double *py) {
    const int ncx = P->ncx, ncy = P->ncy;
    const double L = P->L, cap = 0.05, alpha = 0.002;
    enum { MAXNB = 512 };
    int nbj[MAXNB], nnb = 0;
    const double reach = 1.0 + cap * K->syn_relax, reach2 = reach * reach;
    for (int b = 0; b < ml && nnb < MAXNB; b++) {
        const int c = cat_cell(P, px[b], py[b]), cx = c / ncy, cy = c % ncy;
        const int rx = (int)ceil((reach + CAT_MARGIN) * P->icsx), ry = (int)ceil((reach + CAT_MARGIN) * P->icsy);
        for (int ox = -rx; ox <= rx; ox++) {
            int cxx = cx + ox;
            cxx += cxx < 0 ? ncx : 0;
            cxx -= cxx >= ncx ? ncx : 0;
            for (int oy = -ry; oy <= ry; oy++) {
                int cyy = cy + oy;
                cyy += cyy < 0 ? ncy : 0;
                cyy -= cyy >= ncy ? ncy : 0;
                const int cc = cxx * ncy + cyy;
                for (int j = cstart[cc]; j < cstart[cc + 1]; j++) {
                    int skip = 0;
                    for (int q = 0; q < ml; q++) skip |= j == sl[q];
                    for (int q = 0; q < nnb && !skip; q++) skip |= nbj[q] == j;
                    if (skip) continue;
                    const double dx = minimg((double)x[j] - px[b], L), dy = minimg((double)y[j] - py[b], L);
                    if (dx * dx + dy * dy < reach2 && nnb < MAXNB) nbj[nnb++] = j;
                }
            }
        }
    }
    for (int it = 0; it < K->syn_relax; it++) {
        double fx[64] = {0}, fy[64] = {0};
        for (int b = 0; b < ml; b++) {
            const int ti = b < K->nH ? 1 : 2;
            for (int q = 0; q < nnb; q++) {
                const int j = nbj[q];
                const double dx = minimg(px[b] - (double)x[j], L), dy = minimg(py[b] - (double)y[j], L);
                const double r2 = dx * dx + dy * dy;
                if (r2 >= 1.0 || r2 < 1e-24) continue;
                const double r = sqrt(r2);
                const double f = P->a[ti * ORA_MAXT + type[j]] * (1.0 - r) / r;
                fx[b] += f * dx;
                fy[b] += f * dy;
            }
        }
        double bx[64], by[64], bl[64];
        for (int b = 0; b < ml - 1; b++) {
            bx[b] = minimg(px[b + 1] - px[b], L);
            by[b] = minimg(py[b + 1] - py[b], L);
            bl[b] = sqrt(bx[b] * bx[b] + by[b] * by[b]);
            const double f = -P->k_bond * (bl[b] - P->r0) / bl[b];
            fx[b + 1] += f * bx[b]; fy[b + 1] += f * by[b];
            fx[b] -= f * bx[b]; fy[b] -= f * by[b];
        }
        for (int b = 0; b < ml - 2 && P->k_angle != 0.0; b++) {
            const double ax = bx[b], ay = by[b], cxv = bx[b + 1], cyv = by[b + 1], la = bl[b], lc = bl[b + 1];
            const double ilac = 1.0 / (la * lc), cs = (ax * cxv + ay * cyv) * ilac, ka = P->k_angle;
            const double dUax = -ka * (cxv * ilac - cs * ax / (la * la)), dUay = -ka * (cyv * ilac - cs * ay / (la * la));
            const double dUcx = -ka * (ax * ilac - cs * cxv / (lc * lc)), dUcy = -ka * (ay * ilac - cs * cyv / (lc * lc));
            fx[b] += dUax; fy[b] += dUay;
            fx[b + 1] += -dUax + dUcx; fy[b + 1] += -dUay + dUcy;
            fx[b + 2] -= dUcx; fy[b + 2] -= dUcy;
        }
        for (int b = 0; b < ml; b++) {
            double mx = alpha * fx[b], my = alpha * fy[b];
            const double m = sqrt(mx * mx + my * my);
            if (m > cap) { mx *= cap / m; my *= cap / m; }
            px[b] += mx;
            py[b] += my;
            wrap1(&px[b], L);
            wrap1(&py[b], L);
        }
    }
}

static int cat_in_vent(const ora_cat *K, double L, double x, double y) {
    if (K->vent_kind == 0) {
        const double dx = minimg(x - K->vent_x, L), dy = minimg(y - K->vent_y, L);
        return dx * dx + dy * dy < K->vent_r * K->vent_r;
    }
    if (K->vent_kind == 1) return fabs(minimg(x - K->vent_x, L)) < 0.5 * K->vent_w;
    return fabs(minimg(y - K->vent_y, L)) < 0.5 * K->vent_w;
}

static void cat_event(ora_event *ev, int32_t evcap, int32_t *nev, int64_t step, int kind, uint32_t i, double x,
                      double y, int variant) {
    if (*nev < evcap) {
        ora_event *e = &ev[*nev];
        e->step = step;
        e->kind = kind;
        e->gid = i;
        e->partner = (uint32_t)variant;
        e->x = (float)x;
        e->y = (float)y;
        e->pad = 0;
    }
    (*nev)++;
}

/* One chemistry check of the reference (chemistry, oercel.c:1565-1700, and
 * feed_supply, :1721-1753) on a state sorted into cells (cstart): catalysts
 * in slot order shuffled with the serial generator rng, each with lipid
 * synthesis (nearest N, best of syn_tries orientations, relaxation) and
 * replication / mutation; then decay by keyed deviates; then the food
 * supply.  Positions are FP32 in and out, computed in FP64.  Returns 1 if
 * beads moved; *nev = number of events (those beyond evcap are dropped). */
int32_t ora_catalyst_chemistry(const ora_params *P, const ora_cat *K, uint64_t *rng_state, int32_t n, float *x,
                               float *y, float *vhx, float *vhy, float *vtx, float *vty, uint8_t *type,
                               const uint32_t *gid, int32_t *prev, int32_t *next, const int32_t *cstart, int64_t step,
                               ora_event *ev, int32_t evcap, int32_t *nev) {
    rng_t rng;
    memcpy(rng.s, rng_state, sizeof rng.s);
    const int ml = K->nH + K->nT;
    const double L = P->L;
    int moved = 0;
    *nev = 0;
    int *ks = malloc((size_t)(n + 1) * sizeof(int));
    int nk = 0;
    for (int d = 0; d < n; d++)
        if (type[d] == 4 || type[d] == 5) ks[nk++] = d;
    for (int a = nk - 1; a > 0; a--) {
        const int b = (int)cat_rng_below(&rng, a + 1);
        const int t = ks[a]; ks[a] = ks[b]; ks[b] = t;
    }
    cat_nbr nb[256], nbw[256];
    for (int q = 0; q < nk; q++) {
        const int k = ks[q];
        if (type[k] != 4 && type[k] != 5) continue;
        const int var = type[k] == 5;
        const double psyn = var ? K->p_syn_b : K->p_syn_a, prep = var ? K->p_rep_b : K->p_rep_a;
        const double xk = x[k], yk = y[k];
        const int nn = cat_find(P, x, y, type, gid, cstart, k, xk, yk, K->r_cat, 3, nb, 256);
        if (nn < 2) continue;
        int used = 0;
        const int nsynN = K->syn_nN > 0 ? K->syn_nN : ml;
        int nw = 0;
        if (nn >= nsynN && nsynN < ml) nw = cat_find(P, x, y, type, gid, cstart, k, xk, yk, K->r_cat, 0, nbw, 256);
        if (nn >= nsynN && nsynN + nw >= ml && rng_unif(&rng) < psyn) {
            double cxm = 0, cym = 0, mvx = 0, mvy = 0, mtx = 0, mty = 0;
            int sl[64];
            for (int b = 0; b < ml; b++) {
                const int j = b < nsynN ? nb[b].slot : nbw[b - nsynN].slot;
                sl[b] = j;
                cxm += minimg((double)x[j] - xk, L);
                cym += minimg((double)y[j] - yk, L);
                mvx += vhx[j]; mvy += vhy[j];
                mtx += vtx[j]; mty += vty[j];
            }
            cxm = xk + cxm / ml; cym = yk + cym / ml;
            mvx /= ml; mvy /= ml; mtx /= ml; mty /= ml;
            double ux = 1.0, uy = 0.0, ubest = INFINITY;
            for (int tr = 0; tr < K->syn_tries; tr++) {
                const double phi = 2.0 * M_PI * rng_unif(&rng);
                const double cx_ = cos(phi), cy_ = sin(phi);
                const double U = K->syn_tries > 1 ? cat_chain_energy(P, K, x, y, type, cstart, cxm, cym, cx_, cy_, sl, ml)
                                                  : 0.0;
                if (U < ubest) { ubest = U; ux = cx_; uy = cy_; }
            }
            double px[64], py[64];
            for (int b = 0; b < ml; b++) {
                const int j = sl[b];
                const double off = (b - 0.5 * (ml - 1)) * P->r0;
                px[b] = cxm + off * ux;
                py[b] = cym + off * uy;
                wrap1(&px[b], L);
                wrap1(&py[b], L);
                vhx[j] = (float)mvx; vhy[j] = (float)mvy;
                vtx[j] = (float)mtx; vty[j] = (float)mty;
                type[j] = b < K->nH ? 1 : 2;
            }
            for (int b = 0; b < ml; b++) {
                prev[sl[b]] = b > 0 ? sl[b - 1] : -1;
                next[sl[b]] = b + 1 < ml ? sl[b + 1] : -1;
            }
            if (K->syn_relax > 0) cat_relax(P, K, x, y, type, cstart, sl, ml, px, py);
            for (int b = 0; b < ml; b++) {
                float fx_ = (float)px[b], fy_ = (float)py[b];
                if (fx_ >= (float)L) fx_ = 0.0f;
                if (fy_ >= (float)L) fy_ = 0.0f;
                x[sl[b]] = fx_;
                y[sl[b]] = fy_;
            }
            cat_event(ev, evcap, nev, step, ORA_EV_SYN, gid[k], xk, yk, var);
            used = nsynN;
            moved = 1;
        }
        if (nn - used >= 2 && rng_unif(&rng) < prep) {
            int nv = var, mut = 0;
            if (rng_unif(&rng) < K->mu) { nv = 1 - var; mut = 1; }
            const int j1 = nb[used].slot, j2 = nb[used + 1].slot;
            type[j1] = nv ? 5 : 4;
            type[j2] = 0;
            cat_event(ev, evcap, nev, step, mut ? ORA_EV_MUT : ORA_EV_REP, gid[j1], xk, yk, nv);
        }
    }
    /* decay: keyed per-bead decisions in slot order, applied after the scan */
    if (K->p_ld > 0 || K->p_kd > 0 || K->p_nd > 0) {
        const uint64_t kl = cat_hash_key(P->seed, step, 11), kk = cat_hash_key(P->seed, step, 12),
                       kn = cat_hash_key(P->seed, step, 13);
        int nd = 0;
        for (int d = 0; d < n; d++) {
            const int head = prev[d] < 0 && next[d] >= 0;
            if ((head && K->p_ld > 0 && cat_hash_u01(kl, gid[d]) < K->p_ld) ||
                ((type[d] == 4 || type[d] == 5) && K->p_kd > 0 && cat_hash_u01(kk, gid[d]) < K->p_kd) ||
                (type[d] == 3 && K->p_nd > 0 && cat_hash_u01(kn, gid[d]) < K->p_nd))
                ks[nd++] = d;
        }
        for (int q = 0; q < nd; q++) {
            const int d = ks[q], t = type[d];
            if (prev[d] < 0 && next[d] >= 0) {
                int c = d, m = 0;
                while (c >= 0 && m < ml) {
                    const int nx = next[c];
                    type[c] = 0;
                    prev[c] = -1;
                    next[c] = -1;
                    c = nx;
                    m++;
                }
                cat_event(ev, evcap, nev, step, ORA_EV_DLIP, gid[d], x[d], y[d], -1);
            } else if (t == 4 || t == 5) {
                type[d] = 0;
                cat_event(ev, evcap, nev, step, ORA_EV_DK, gid[d], x[d], y[d], t == 5);
            } else if (t == 3) {
                type[d] = 0;
                cat_event(ev, evcap, nev, step, ORA_EV_DN, gid[d], x[d], y[d], -1);
            }
        }
    }
    /* food supply (feed_supply, oercel.c:1721-1753) */
    if (K->feed_mode != 0 && K->p_feed > 0.0) {
        const uint64_t kf = cat_hash_key(P->seed, step, 14);
        int nc = 0;
        for (int d = 0; d < n; d++)
            if (type[d] == 0 && (K->feed_mode == 1 || cat_in_vent(K, L, x[d], y[d])) &&
                cat_hash_u01(kf, gid[d]) < K->p_feed)
                ks[nc++] = d;
        long add = nc;
        if (K->feed_cap > 0.0 && nc > 0) {
            long nN = 0;
            for (int i = 0; i < n; i++) nN += type[i] == 3;
            long room = (long)floor(K->feed_cap * (double)n + 1e-9) - nN;
            if (room < 0) room = 0;
            if (add > room) {
                for (long a = 0; a < room; a++) {
                    const long b = a + cat_rng_below(&rng, nc - a);
                    const int t = ks[a]; ks[a] = ks[b]; ks[b] = t;
                }
                add = room;
            }
        }
        for (long a = 0; a < add; a++) type[ks[a]] = 3;
        if (add > 0) cat_event(ev, evcap, nev, step, ORA_EV_FEED, (uint32_t)add, NAN, NAN, -1);
    }
    free(ks);
    memcpy(rng_state, rng.s, sizeof rng.s);
    return moved;
}
