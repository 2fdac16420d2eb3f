/*
 * dpd_oracle.h -- CPU restatement of the 2D DPD step (TEST INFRASTRUCTURE ONLY).
 *
 * This library is the checker for the CUDA path: only the tests, the smoke
 * check and the CPU-baseline leg of bench.py may load it.  The product
 * (libdpd.so) never links or calls it.
 *
 * Every function restates one piece of the reference engine
 * cel/engine/oercel.c (file:line cited at each definition in dpd_oracle.c),
 * with two deliberate extensions that the reference does not have:
 *   - Philox4x32-10 pair noise (Salmon et al., SC'11) next to the
 *     reference's mix13 hash noise (selected by ora_params.noise);
 *   - the three-rule lipid chemistry of the 1M-bead workload (chain growth
 *     from P, H-T bond breaking, free T + free H bonding), whose parity is
 *     UNPINNED by the reference (it has no such reactions).
 *
 * Conventions shared with the CUDA library:
 *   cells: ncx = ncy = floor(L), column-major c = cx * ncy + cy (the
 *          reference with nsub = 1, oercel.c:739-745, 779-786);
 *   links: prev/next slot of the bonded neighbour towards the chain head /
 *          tail, -1 if none (the reference's nxt[] is next[]).
 */
#ifndef DPD_ORACLE_H
#define DPD_ORACLE_H
#include <stdint.h>

#define ORA_MAXT 8

typedef struct {
    double L;
    int32_t ncx, ncy;
    double icsx, icsy;      /* ncx / L, ncy / L */
    double dt, lambda, gamma, kT;
    double a[ORA_MAXT * ORA_MAXT];
    double k_bond, r0;
    uint64_t seed;
    int32_t noise;          /* 0 = Philox4x32-10, 1 = reference mix13 hash */
    int32_t pad;
    double k_angle;         /* U = k_angle (1 - cos) on consecutive chain triplets */
    double stir_A;          /* stirring f_x = stir_A sin(2 pi stir_n y / L), mean removed */
    int32_t stir_n, pad2;
    double kT_amp, kT_period; /* kT(t) = kT + kT_amp sin(2 pi t / kT_period) */
    double t_anchor;        /* t(step) = t_anchor + (step - step_anchor) dt */
    int64_t step_anchor;
} ora_params;

typedef struct {
    float dt, dt2, cvt, L; /* FP32 integrator constants exactly as the kernel gets them */
} ora_f32c;

typedef struct {
    uint32_t thr_break, thr_grow, thr_bond; /* decision u32 < thr */
    float r2_grow, r2_bond;                  /* squared reaction radii (FP32) */
    int32_t n_t_min;                         /* T beads within r_grow needed by a P */
    int32_t max_chain;                       /* chains never grow beyond this many beads */
} ora_chem;

typedef struct {
    int64_t step;
    int32_t kind;      /* 0 = grow, 1 = brk, 2 = bond */
    uint32_t gid;      /* reacting bead */
    uint32_t partner;  /* gid of the bead it bonded to / unbonded from */
    float x, y;        /* position of the reacting bead */
    int32_t pad;
} ora_event;

/* A lipid molecule template (the reference's mol_t, oercel.c:451-462): bonds
 * as position pairs with rest lengths, angle terms as position triplets (j the
 * middle) with kind 0 U = K (1 - cos) or kind 1 U = K (cos - c0)^2. */
#define ORA_MAXML 16
#define ORA_MAXMB (2 * ORA_MAXML)
typedef struct {
    int32_t mlen, nb, na, pad;
    int32_t bi[ORA_MAXMB], bj[ORA_MAXMB];
    double br0[ORA_MAXMB];
    int32_t ai[ORA_MAXMB], aj[ORA_MAXMB], ak[ORA_MAXMB], akind[ORA_MAXMB];
    double aK[ORA_MAXMB], ac0[ORA_MAXMB];
} ora_mol;

/* the reference's catalyst chemistry (oercel.c:1345-1753): synthesis of
 * lipids from N beads around Ka/Kb catalysts, replication and mutation of
 * catalysts, decay, and the W -> N food supply */
typedef struct {
    double r_cat;                          /* catalyst reaction radius */
    int32_t syn_tries, syn_relax, syn_nN;  /* orientation trials, relaxation iterations, N per lipid (0 = mlen) */
    int32_t nH, nT;                        /* linear lipid template: nH heads then nT tails */
    int32_t feed_mode, vent_kind;          /* 0 none, 1 uniform, 2 vent; 0 disk, 1 vstrip, 2 hstrip */
    int32_t pad;
    double p_syn_a, p_syn_b, p_rep_a, p_rep_b, mu, p_ld, p_kd, p_nd;
    double p_feed, feed_cap, vent_x, vent_y, vent_r, vent_w;
} ora_cat;

/* event kinds of the catalyst chemistry (after the lipid chemistry's 0..2) */
#define ORA_EV_SYN 3
#define ORA_EV_REP 4
#define ORA_EV_MUT 5
#define ORA_EV_DLIP 6
#define ORA_EV_DK 7
#define ORA_EV_DN 8
#define ORA_EV_FEED 9

#endif
