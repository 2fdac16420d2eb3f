/*
 * dpd.h -- C ABI of libdpd.so, the B200 (sm_100a) implementation of the 2D
 * DPD step with lipid chemistry of the Oercel engine.
 *
 * The reference runs its step inside the engine process (cel/engine/oercel.c,
 * main loop :2300-2361) and is driven from Python only through a subprocess
 * CLI (cel/pc/pclib.py:973-986).  This ABI exposes the same step and its
 * phases in-process, for ctypes/cffi callers, with plain pointers and sizes:
 *
 *   reference phase (file:line)                       entry point here
 *   ------------------------------------------------  ---------------------------
 *   Params/PDEFS + finalize_params  oercel.c:178-299,578-619  dpd_params_default, dpd_create
 *   sys_alloc                       oercel.c:714-759   dpd_create
 *   init_soup + set_velocities      oercel.c:1757-1814 dpd_set_state (host-made soup)
 *   initial sort/forces/half kick   oercel.c:2203-2211 dpd_prime
 *   integrate block of main         oercel.c:2303-2334 dpd_integrate
 *   sort_cells                      oercel.c:832-933   dpd_build_cells
 *   pair_forces                     oercel.c:1198-1216 dpd_forces (pair part)
 *   bonded_forces                   oercel.c:1322-1343 dpd_forces (bond part)
 *   chemistry                       oercel.c:1565-1701 dpd_chemistry
 *   one loop iteration              oercel.c:2300-2361 dpd_step
 *   kinetic_T / count_types         oercel.c:2053-2071 dpd_observables
 *   write_snapshot/ckpt state read  oercel.c:1830-1936 dpd_get_state, dpd_get_cells
 *   add_event / flush_events        oercel.c:788-798,2036-2047 dpd_get_events
 *   die() error path                oercel.c:74-90     negative return + dpd_last_error
 *
 * Conventions
 *   - Every call returns DPD_OK (0) or a negative DPD_E_* code; the message of
 *     the last failure on the calling thread is dpd_last_error().  Nothing
 *     calls exit().
 *   - Array arguments may be host or device pointers (CUDA unified
 *     addressing decides); the caller owns them.  The library owns its device
 *     state and scratch.  Arrays are in "slot" order (cell-sorted order, as
 *     the reference's Sys arrays) unless a function says otherwise.
 *   - One handle = one CUDA stream; a handle is not thread safe.
 *   - Bead types: 0 W, 1 H, 2 T, 3 P (the reference's N), 4..7 free.  Lipid
 *     bonds are prev/next links (slot indices, -1 = none); the reference's
 *     nxt[] is next[] and mpos is implied by the chain.
 *   - Cells: ncx = ncy = floor(L), column-major c = cx * ncy + cy: the
 *     reference with nsub = 1 (oercel.c:739-745,779-786).
 */
#ifndef DPD_H
#define DPD_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define DPD_API __attribute__((visibility("default")))
#else
#define DPD_API
#endif

#define DPD_OK 0
#define DPD_E_ARG (-1)            /* bad argument or parameter (reference: die() on params) */
#define DPD_E_CUDA (-2)           /* CUDA runtime error */
#define DPD_E_SORT_OVERFLOW (-3)  /* cell sort could not place every bead (reference GPU: ERR_SORT) */
#define DPD_E_CHAIN (-4)          /* broken lipid chain (reference GPU: ERR_CHAIN) */
#define DPD_E_EVENT_OVERFLOW (-5) /* event buffer full (reference GPU: ERR_EVOVF) */
#define DPD_E_TIMEOUT (-6)        /* a bounded device wait gave up */
#define DPD_E_STATE (-7)          /* a bead left the box or a value is not finite */
#define DPD_E_NOMEM (-8)          /* device allocation failed */

#define DPD_MAXT 8

/* Physics and chemistry of one replica.  Defaults (dpd_params_default) are the
 * reference's PDEFS defaults where the reference has the key
 * (cel/engine/oercel.c:237-299) and the 1M-bead chemistry rules otherwise. */
typedef struct {
    double L;                  /* box side; ncx = ncy = floor(L) >= 3 */
    double dt;                 /* time step (reference key dt) */
    double lambda;             /* Groot-Warren lambda (lambda) */
    double gamma;              /* friction (gamma) */
    double kT;                 /* temperature; sigma = sqrt(2 gamma kT) (kT) */
    double a[DPD_MAXT * DPD_MAXT]; /* repulsion a_ij, symmetric (a_X_Y) */
    double k_bond;             /* harmonic bond constant (k_bond) */
    double r0;                 /* bond rest length (r0) */
    uint64_t seed;             /* noise and chemistry key (seed) */
    int32_t noise;             /* 0 = Philox4x32-10 (default), 1 = the reference's mix13 hash */
    int32_t chem;              /* 1 = run the chemistry pass */
    int32_t n_chem;            /* chemistry every n_chem steps (n_chem) */
    int32_t n_t_min;           /* T beads a P needs within r_grow */
    int32_t max_chain;         /* longest chain growth may produce */
    int32_t pad;
    double p_break;            /* H-T bond break probability per check */
    double p_grow;             /* P -> T chain growth probability per check */
    double p_bond;             /* free T + free H bonding probability per check */
    double r_grow;             /* growth reaction radius (r_c) */
    double r_bond;             /* free T - free H bonding radius */
    int64_t warmup;            /* repulsion ramp length (warmup; 0 = off) */
    int64_t warm_end;          /* step at which the ramp ends (a fresh soup: = warmup) */
    double k_angle;            /* U = k_angle (1 - cos theta) on consecutive chain triplets (k_angle) */
    double stir_A;             /* body force f_x = stir_A sin(2 pi stir_n y / L), net force removed (stir_A) */
    int32_t stir_n;            /* sine periods across the box (stir_n) */
    int32_t pad2;
    double kT_amp;             /* kT(t) = kT + kT_amp sin(2 pi t / kT_period) in the noise (kT_amp) */
    double kT_period;          /* (kT_period) */
    double t_anchor;           /* time of step step_anchor: t(step) = t_anchor + (step - step_anchor) dt */
    int64_t step_anchor;
    /* which chemistry chem = 1 runs: 0 = the lipid chemistry above (p_grow,
     * p_break, p_bond), 1 = the reference's catalyst chemistry (keys below,
     * oercel.c:1565-1753), which needs the serial generator state of
     * dpd_set_rng */
    int32_t chem_kind;
    int32_t syn_tries;         /* orientation trials of a new lipid (syn_tries) */
    int32_t syn_relax;         /* relaxation iterations of a new lipid (syn_relax) */
    int32_t syn_nN;            /* N beads consumed per lipid, 0 = all of it (syn_nN) */
    int32_t lip_nH, lip_nT;    /* linear lipid template: heads, tails (lip_nH, lip_nT) */
    int32_t feed_mode;         /* 0 none, 1 uniform, 2 vent (feed) */
    int32_t vent_kind;         /* 0 disk, 1 vstrip, 2 hstrip (vent_shape) */
    double r_cat;              /* catalyst reaction radius (r_cat) */
    double p_syn_a, p_syn_b;   /* synthesis probability per check, Ka / Kb */
    double p_rep_a, p_rep_b;   /* replication probability per check, Ka / Kb */
    double mu;                 /* mutation probability per replication */
    double p_ld, p_kd, p_nd;   /* decay probability per check: lipid, catalyst, N */
    double p_feed, feed_cap;   /* W -> N probability per check, cap on the N fraction (0 = none) */
    double vent_x, vent_y, vent_r, vent_w; /* vent region */
    /* lipid shape (lip_arch, oercel.c:436-576): 0 linear (lip_nH heads, lip_nT
     * tails), 1 pi (two bonded heads, a tail of lip_nT on each), 2 y (one head,
     * two tails of lip_nT), 3 bola (head pair, two tails of lip_nT, a third head
     * joining them); branched shapes take their bonds and angles from
     * dpd_lipid_template */
    int32_t lip_arch;
    int32_t lip_tie;           /* pi / y / bola: rungs between the two tails (lip_tie) */
    double r0_head;            /* pi / bola: head-head rest length (r0_head) */
    double k_head, cos_head;   /* junction angle term U = k_head (cos - cos_head)^2 (k_head, cos_head) */
} dpd_params;

/* The molecule template of a lipid shape: bead types by position (heads
 * first), bonds (position pairs with rest lengths, spring k_bond), angle terms
 * (position triplets, j the middle bead; kind 0: U = K (1 - cos), kind 1:
 * U = K (cos - c0)^2), the template coordinates (centroid at 0, long axis
 * along +x) used to place a newly synthesised lipid, and the offsets from
 * bead 0 used by the soup.  The beads of a molecule are linked prev/next in
 * position order.  Same numbers, same order as the reference's mol_build
 * (oercel.c:478-576). */
#define DPD_MAXML 16
#define DPD_MAXMB (2 * DPD_MAXML)
typedef struct {
    int32_t arch, mlen, nH, nb, na, pad;
    int32_t bi[DPD_MAXMB], bj[DPD_MAXMB];
    double br0[DPD_MAXMB];
    int32_t ai[DPD_MAXMB], aj[DPD_MAXMB], ak[DPD_MAXMB], akind[DPD_MAXMB];
    double aK[DPD_MAXMB], ac0[DPD_MAXMB];
    double px[DPD_MAXML], py[DPD_MAXML];
    double ix[DPD_MAXML], iy[DPD_MAXML];
} dpd_template;

/* The template of p's lipid shape (lip_arch, lip_nH, lip_nT, lip_tie, r0,
 * r0_head, k_angle, k_head, cos_head).  No counterpart call in the
 * reference, which builds it into a global (mol_build). */
DPD_API int dpd_lipid_template(const dpd_params *p, dpd_template *t);

/* One chemistry event, the reference's events.csv row (oercel.c:788-798)
 * with the partner bead added.  kind: 0 grow, 1 brk, 2 bond. */
typedef struct {
    int64_t step;
    int32_t kind;
    uint32_t gid;
    uint32_t partner;
    float x, y;
    int32_t replica;
} dpd_event;

typedef struct dpd_handle dpd_handle;

/* Launch choices of a handle (the autotuner's knobs).  force_kernel 0: cell
 * tiles of tile_w x tile_h cells staged in shared memory, each pair evaluated
 * once (default); 1: one thread per bead over its 3x3 cells, each pair
 * evaluated by both beads; 2: the cell tiles of 0 staged into shared memory
 * by bulk asynchronous copies, one per tile column (tile_w <= 30).  All give
 * bit-identical forces.
 * graph_steps: steps per captured CUDA graph.  sort_mode: the cell sort's
 * exclusive scan of the cell counts in two passes (0), in one pass with
 * decoupled look-back between blocks (1), or as a block-local pass whose
 * block prefixes the placement and fix-up kernels add themselves (2: one
 * kernel fewer; boxes of up to 4,194,304 cells, else as 0); the same cell
 * starts and order.  tile_threads: threads per CTA of force_kernel 0, 256
 * (four CTAs per SM) or 512 (two per SM, tiles of up to 512 cells with their
 * halo, so less halo per owned cell). */
typedef struct {
    int32_t force_kernel;
    int32_t tile_w, tile_h;   /* (tile_w + 2) * (tile_h + 2) <= 256, or <= tile_threads with force_kernel 0 */
    int32_t graph_steps;
    int32_t sort_mode;
    int32_t tile_threads;
} dpd_tuning;

/* message of the last failed call on this thread ("" if none) */
DPD_API const char *dpd_last_error(void);
/* library version string */
DPD_API const char *dpd_version(void);

/* Fill *p with the defaults. */
DPD_API int dpd_params_default(dpd_params *p);

/* Create a simulation of n_replicas independent boxes packed into one set of
 * device arrays.  params[r] and n_beads[r] describe replica r.  The step
 * counter starts at 0.  Replaces sys_alloc + finalize_params. */
DPD_API int dpd_create(const dpd_params *params, int32_t n_replicas, const int32_t *n_beads, dpd_handle **out);
DPD_API int dpd_destroy(dpd_handle *h);

/* sizes: total beads, beads of replica r, cells of replica r */
DPD_API int dpd_sizes(const dpd_handle *h, int32_t replica, int64_t *n_total, int32_t *n_beads, int32_t *n_cells);

/* Load replica r's state.  x, y in [0, L) (finite values outside are wrapped
 * in); vx, vy: velocity (see dpd_prime); type in 0..7; gid: permanent bead ids
 * 0..n-1 (NULL = 0..n-1); prev/next: link slot indices within the replica,
 * -1 = none (NULL = no links).  The slot order is the caller's; dpd_prime or
 * dpd_build_cells sorts it.  A non-finite position, a type above 7, a gid >= n
 * or a link out of range fails with DPD_E_ARG (checked on the device, so the
 * arrays may be host or device memory). */
DPD_API int dpd_set_state(dpd_handle *h, int32_t replica, const float *x, const float *y, const float *vx, const float *vy,
                  const uint8_t *type, const uint32_t *gid, const int32_t *prev, const int32_t *next);

/* Read replica r's state in slot order.  Any pointer may be NULL. vhx/vhy is
 * the stored half-step velocity, vtx/vty the predicted velocity, fx/fy the
 * force of the current configuration (the reference's vx/vy, vtx/vty, fx/fy). */
DPD_API int dpd_get_state(dpd_handle *h, int32_t replica, float *x, float *y, float *vhx, float *vhy, float *vtx, float *vty,
                  float *fx, float *fy, uint8_t *type, uint32_t *gid, int32_t *prev, int32_t *next);

/* Overwrite the stored half-step velocity, the force and the predicted
 * velocity of replica r (slot order), e.g. to continue from a checkpoint.
 * NULL leaves a field as is. */
DPD_API int dpd_set_dynamics(dpd_handle *h, int32_t replica, const float *vhx, const float *vhy, const float *fx,
                             const float *fy, const float *vtx, const float *vty);

/* Fresh start as the reference's main() (oercel.c:2203-2211): take the loaded
 * velocity as the full velocity v, sort by cell, compute the forces of the
 * current step, store vh = v - dt/2 f, and prepare the next sort. */
DPD_API int dpd_prime(dpd_handle *h);

/* Continue from a loaded (x, vh, f) state without recomputing forces: sort by
 * cell and prepare the next sort. */
DPD_API int dpd_resume(dpd_handle *h);

/* current step number (the step of the stored forces) */
DPD_API int dpd_get_step(const dpd_handle *h, int64_t *step);
DPD_API int dpd_set_step(dpd_handle *h, int64_t step);

/* Advance nsteps full steps: integrate, cell sort, chemistry (when due),
 * pair + bond forces (oercel.c:2300-2361), launched as CUDA graphs. */
DPD_API int dpd_step(dpd_handle *h, int64_t nsteps);

/* dpd_step without the final status check: enqueues the steps on the
 * handle's stream and returns; dpd_sync waits for them and reports any
 * device-side error flag (as dpd_step does). */
DPD_API int dpd_step_async(dpd_handle *h, int64_t nsteps);
DPD_API int dpd_sync(dpd_handle *h);
DPD_API int dpd_set_tuning(dpd_handle *h, const dpd_tuning *t);
DPD_API int dpd_get_tuning(const dpd_handle *h, dpd_tuning *t);
/* steps per captured CUDA graph (default: about 4M bead-steps per replay) */
DPD_API int dpd_set_graph_steps(dpd_handle *h, int32_t steps);
/* One real step launched kernel by kernel with CUDA events around each launch
 * on the handle's stream: ms[k] = device time of kernel k in launch order
 * (scan1, scan2, place, cellfix, permute, [2 chemistry kernels], [catalyst
 * check with its sort], forces); *n_out = number of kernels.  On a step with a
 * catalyst check the first entry is a one-thread step-counter kernel and the
 * next three are not launched (0 ms). */
DPD_API int dpd_profile_step(dpd_handle *h, float *ms, int32_t cap, int32_t *n_out);

/* The reference's random soup (init_soup + set_velocities,
 * cel/engine/oercel.c:1757-1814) with the same xoshiro256** draws, on the
 * host: linear lipids of nH heads + nT tails at spacing r0 from uniform head
 * positions (or, with a template of a branched shape, its soup offsets turned
 * by a random angle, its mlen beads and nH heads), then nKa = round(f_Ka N)
 * beads of type 4, nKb of type 5, round(c_N N) of type 3 (P), the rest W;
 * Gaussian velocities with the mean removed, rescaled to exactly kT.  HOST
 * arrays of N entries in gid order.  *n_lipid_beads receives the number of
 * beads placed in lipids; rng_out (4 words, may be NULL) the generator state
 * after the soup, from which the reference's serial chemistry continues.
 * mol may be NULL (linear lipids from nH, nT, r0). */
DPD_API int dpd_init_soup(double L, int32_t N, uint64_t seed, double kT, double r0, int32_t nH, int32_t nT,
                          double f_lip, double f_Ka, double f_Kb, double c_N, double *x, double *y, double *vx,
                          double *vy, uint8_t *type, int32_t *prev, int32_t *next, int32_t *n_lipid_beads,
                          uint64_t *rng_out, const dpd_template *mol);

/* The xoshiro256** state n draws after `state` (out may equal state), by a
 * jump through the generator's characteristic polynomial; the catalyst check
 * uses the same jumps to draw its stream in parallel.  No counterpart call in
 * the reference, which draws serially. */
DPD_API int dpd_xoshiro_jump(const uint64_t *state, uint64_t n, uint64_t *out);

/* The serial xoshiro256** state of the catalyst chemistry of replica r
 * (4 words; the reference's Sys.rng, checkpointed with the state). */
DPD_API int dpd_set_rng(dpd_handle *h, int32_t replica, const uint64_t *state);
DPD_API int dpd_get_rng(dpd_handle *h, int32_t replica, uint64_t *state);

/* ---- phases, for testing and custom loops ---- */

/* Stable counting sort of every replica by the cell of the CURRENT positions
 * (oercel.c:832-933); carries all per-bead arrays along, remaps links. */
DPD_API int dpd_build_cells(dpd_handle *h);
/* cell starts of replica r (n_cells + 1 entries, slot offsets within the replica) */
DPD_API int dpd_get_cells(dpd_handle *h, int32_t replica, int32_t *cstart);
/* pair + bond forces of the current configuration at the given step, stored
 * as the current forces (requires a sorted state) */
DPD_API int dpd_forces(dpd_handle *h, int64_t step);
/* pair part only / bond part only, written to fx, fy (slot order, replica r) */
DPD_API int dpd_pair_forces(dpd_handle *h, int32_t replica, int64_t step, float *fx, float *fy);
DPD_API int dpd_bond_forces(dpd_handle *h, int32_t replica, float *fx, float *fy, float *maxbond);
/* the Groot-Warren update in place, without sorting (oercel.c:2303-2334) */
DPD_API int dpd_integrate(dpd_handle *h);
/* one chemistry pass at the given step on the current sorted state */
DPD_API int dpd_chemistry(dpd_handle *h, int64_t step);

/* Events recorded since the last call, in device order; *n_out = count
 * returned (<= cap); the buffer is then cleared (events beyond cap are
 * dropped and reported as DPD_E_EVENT_OVERFLOW).  out == NULL only reports
 * the pending count in *n_out and clears nothing. */
DPD_API int dpd_get_events(dpd_handle *h, dpd_event *out, int32_t cap, int32_t *n_out);
/* dpd_get_events without waiting: enqueues on the handle's stream a copy of
 * the events recorded since the last read into out (at most cap) and of
 * their count into *n_out (all that were recorded: more than cap means the
 * rest were dropped), then clears the log.  out and n_out must be pinned host
 * memory the device can write (cudaHostAlloc, cudaHostRegister), else
 * DPD_E_ARG; they are valid once the stream has passed this point.  A driver
 * can read the events this way between steps without draining the stream.  No
 * counterpart call in the reference, which appends events.csv inside its step
 * loop (oercel.c:788-798). */
DPD_API int dpd_events_async(dpd_handle *h, dpd_event *out, int32_t cap, int32_t *n_out);

/* Observables of replica r (reference stats row, oercel.c:2364-2372):
 * out[0] T_kin = sum v^2 / (2N - 2) with v = vh + dt/2 f; out[1..2] total
 * momentum; out[3] conservative virial (1/L^2) sum_{i<j} a_ij (1-r) r;
 * out[4] largest bond length; out[5] number of chains (heads with a bond);
 * out[8 + t] number of beads of type t (t < 8).  out has 16 entries. */
DPD_API int dpd_observables(dpd_handle *h, int32_t replica, double *out);
/* the stats row only (out[3], the virial, is left 0): no pair loop */
DPD_API int dpd_stats(dpd_handle *h, int32_t replica, double *out);
/* dpd_stats without waiting: enqueues the row on the handle's stream and a
 * copy of its 16 raw sums into raw (host memory, pinned for a true async copy),
 * valid once the stream passes that point (dpd_sync); dpd_stats_decode turns
 * the raw sums into the 16 values of dpd_stats.  No counterpart call in the
 * reference, whose stats row is written by the step loop itself. */
DPD_API int dpd_stats_async(dpd_handle *h, int32_t replica, uint64_t *raw);
DPD_API int dpd_stats_decode(const dpd_handle *h, int32_t replica, const uint64_t *raw, double *out);
/* From now on every step (eager or inside a step graph) writes replica r's
 * stats row into ring[(step % nslots) * 16 ...] itself, as dpd_stats_async's
 * raw sums with word 6 set to the step number; ring: pinned host memory the
 * device can write (cudaHostAlloc, cudaHostRegister), else DPD_E_ARG.  A row
 * is complete once the stream has passed its step.  ring = NULL stops it.  A
 * driver can then run multi-step graphs and still read every step's row.  The
 * reference writes its stats row inside its own step loop (oercel.c:2262-2290). */
DPD_API int dpd_stats_ring(dpd_handle *h, int32_t replica, uint64_t *ring, int32_t nslots);

/* Clusters of the beads of one type of replica r (the reference's analysis
 * `snapcheck.py tclust`, cel/engine/tests/snapcheck.py:122-144): beads of the
 * type within rcut (0 < rcut <= 1) of each other are joined; out[0] beads of
 * the type, out[1] clusters, out[2] the largest, out[3] the sum of squared
 * sizes (bead-weighted mean size = out[3] / out[0]), out[4] neighbours within
 * 1.0 of the type's beads (any type, self excluded), out[5] those of the type
 * (neighbour fraction = out[5] / out[4]).  Distances in FP64 from the FP32
 * positions, <= as the reference's tree queries.  No counterpart call in the
 * reference engine, whose analysis reads snapshots on the CPU. */
DPD_API int dpd_type_clusters(dpd_handle *h, int32_t replica, int32_t type, double rcut, int64_t *out);

/* Membrane aggregates of replica r: the first stages of the reference's cell
 * detection (cel/tools/cells.py:64-86, 345-366, 605-608).  Molecules are the
 * bonded components of lipid beads (H, T); aggregates join molecules whose
 * tail beads lie within r_tail (0 < r_tail <= 1, distance <= r_tail).  out[0]
 * molecules, out[1] aggregates, out[2] membranes (aggregates of at least
 * min_lipids molecules), out[3] molecules in smaller aggregates, out[4] the
 * largest aggregate in molecules.  agg_of_gid (n entries, may be NULL): per
 * bead in gid order, the smallest gid of its aggregate, -1 for non-lipid
 * beads.  Uses the cell index of the last sort.  No counterpart call in the
 * reference engine, whose analysis reads snapshots on the CPU. */
DPD_API int dpd_aggregates(dpd_handle *h, int32_t replica, double r_tail, int32_t min_lipids, int64_t *out,
                           int32_t *agg_of_gid);

/* Histogram (nbin bins on [0, rmax], rmax <= 3) of distances between beads of
 * types ta and tb of replica r (ta < 0: all beads), each unordered pair once:
 * the pair counts of the reference's `snapcheck.py rdf`
 * (cel/engine/tests/snapcheck.py:86-107), distances in FP64 from the FP32
 * positions, binned as np.histogram bins them. */
DPD_API int dpd_pair_hist(dpd_handle *h, int32_t replica, int32_t ta, int32_t tb, double rmax, int32_t nbin, double *hist);

/* ---- cell detection in one snapshot (the reference's cel/tools/cells.py) ----
 * Stand-alone: no engine handle.  The thresholds of cells.py's DEFAULTS
 * (cells.py:37-56), with the same names and meaning. */
typedef struct {
    double r_tail, h, r_stamp;
    int32_t min_membrane_lipids, pad0;
    double min_lumen_area, min_aqueous_frac, rho, pad, leaflet_in, leaflet_max, min_exposure, wall_extra;
    double inner_frac_lo, inner_frac_hi;
} dpd_cells_cfg;

/* Columns of one detected cell, raw (unrounded) values:
 * x, y (lumen centroid, wrapped), area, n_lipids, n_Ka, n_Kb, n_N, n_W, n_Z,
 * agg, agg_lumens, agg_lipids, inner_heads, outer_heads, aspect, solidity
 * (not capped at 1), extent, wraps_membrane (0/1), exposure, wall (inf when
 * no distance to the bulk medium is finite).  Rounding as cells.py rounds its
 * dict (cells.py:582-601) is left to the caller. */
#define DPD_CELL_COLS 20
typedef struct dpd_cells dpd_cells;

DPD_API int dpd_cells_default(dpd_cells_cfg *cfg);
/* detect(snap, cfg) (cells.py:331-611) on the GPU: x, y (n host values,
 * already wrapped into [0, L), FP64 as the reference's snapshot reader gives
 * them), type (n), bonds (nbond x 2 bead indices).  *out receives the result;
 * free it with dpd_cells_free. */
DPD_API int dpd_cells_detect(const dpd_cells_cfg *cfg, double L, int64_t n, const double *x, const double *y,
                             const uint8_t *type, int64_t nbond, const int32_t *bonds, dpd_cells **out);
/* info[0..5]: n_molecules, n_aggregates, n_membranes, lipids_in_small_aggregates,
 * largest_aggregate, wrapping_membranes (the reference's summary); info[6] ng
 * (label grid side), info[7] cells, info[8] membranes listed by
 * dpd_cells_fetch's aggs; *h the pixel size. */
DPD_API int dpd_cells_info(const dpd_cells *c, int64_t *info, double *h);
/* Copies out (any pointer may be NULL): cells (cells x DPD_CELL_COLS), aggs
 * (membranes x 4: agg, n_lipids, wraps, n_holes), label (ng x ng, -1 = no
 * cell; label_bytes 2 gives int16 as cells.py does below 32767 cells, 4 gives
 * int32), bead_cell, mol and bead_agg (n each, as cells.py returns them).  The
 * grid and the per-bead arrays stay on the device until fetched. */
DPD_API int dpd_cells_fetch(const dpd_cells *c, double *cells, int64_t *aggs, void *label, int32_t label_bytes,
                            int32_t *bead_cell, int32_t *mol, int32_t *bead_agg);
DPD_API void dpd_cells_free(dpd_cells *c);

/* the CUDA stream (cudaStream_t) this handle enqueues its work on */
DPD_API int dpd_get_stream(const dpd_handle *h, void **stream);
/* kernels one step of dpd_step launches: *n_plain in total, of which *n_chem
 * belong to the chemistry pass (they return at once on non-chemistry steps) */
DPD_API int dpd_kernels_per_step(const dpd_handle *h, int32_t *n_plain, int32_t *n_chem);

/* ---- parameters in place, and reverse mode (no counterpart in the reference) ---- */

/* Replace replica r's physics and chemistry parameters (same box size); a fit
 * updates its repulsions this way between windows. */
DPD_API int dpd_set_params(dpd_handle *h, int32_t replica, const dpd_params *p);

/* Structural loss of a differentiated window: the pair distribution g(r) of
 * types ta and tb on nbin bins of [0, rmax), smoothed with a Gaussian of width
 * sigma, averaged over the last last_steps steps of the window;
 * loss = mean over bins of (g - target)^2, per replica.
 * horizon: the reverse pass runs back only `horizon` steps before the first
 * step that enters the loss (0 = through the whole window).  The exact
 * gradient through a long chaotic trajectory grows exponentially with the
 * window; a horizon of a few tens of steps keeps it bounded (truncated
 * backpropagation) and saves the recomputation of the earlier segments. */
typedef struct {
    int32_t ta, tb, nbin, last_steps;
    double rmax, sigma;
    int32_t horizon, pad;
} dpd_rdf_spec;

#define DPD_NGRAD 66 /* gradient layout per replica: d loss / d a_ij (64, entry [i*8+j] with i <= j holds the
                        symmetric pair's total), d loss / d gamma, d loss / d k_bond */

/* Advance every replica nsteps steps (chemistry must be off) and return the
 * loss (nrep values) and, if rdf_out, the averaged g(r) (nrep x nbin).  The
 * differentiated terms are those of the forces (dpd_force_vjp), the noise
 * amplitude following the temperature cycle. */
DPD_API int dpd_window_loss(dpd_handle *h, int64_t nsteps, const dpd_rdf_spec *spec, const double *target,
                            double *loss, double *rdf_out);
/* The same window, then its adjoint: the pair noise is replayed from its key,
 * the state is checkpointed every ckpt_every steps and each segment is
 * recomputed in reverse.  grad: nrep x DPD_NGRAD.  The handle ends at the end
 * of the window, as after dpd_window_loss. */
DPD_API int dpd_window_adjoint(dpd_handle *h, int64_t nsteps, int32_t ckpt_every, const dpd_rdf_spec *spec,
                               const double *target, double *loss, double *grad, double *rdf_out);
/* dpd_window_adjoint plus the cotangents of the window's start state: the
 * loss's gradient with respect to the positions (xbar), the stored half-step
 * velocities (vhbar) and the predicted velocities (vtbar) the window starts
 * from, the start forces being F(x, vt) of that state.  Each is 2 x N floats
 * (x, y interleaved) over all replicas packed, replica r's bead of gid g at
 * b0_r + g (b0_r = the bead counts of the replicas before r); any may be NULL.
 * Needs spec->horizon == 0 (the full reverse pass), else DPD_E_ARG.  No
 * counterpart in the reference (it has no reverse mode). */
DPD_API int dpd_window_adjoint_state(dpd_handle *h, int64_t nsteps, int32_t ckpt_every, const dpd_rdf_spec *spec,
                                     const double *target, double *loss, double *grad, double *rdf_out, float *xbar,
                                     float *vhbar, float *vtbar);
/* A fit of repulsions shared by every replica, run as one captured CUDA graph
 * replayed iters times: each iteration is the differentiated window of
 * dpd_window_adjoint (nsteps, ckpt_every, spec, target as there), its loss
 * and gradient computed on the device, the gradient of the fitted a_ij summed
 * over the replicas, and an Adam step (as torch.optim.Adam takes it, without
 * weight decay) that sets a_ij = a_ji in every replica.  The replicas continue
 * from the end of each window.  No host step comes between the iterations.
 * slot[k] = i * 8 + j (i <= j) names the fitted entries; they must start equal
 * in every replica.  Outputs (any may be NULL): loss (iters x nrep), grad
 * (iters x n, the summed gradient) and values ((iters + 1) x n: the values
 * each window ran with, then the last values).  Afterwards the handle holds
 * the last values, as if set by dpd_set_params.  No counterpart in the reference (it has no reverse mode). */
typedef struct {
    int32_t n, pad;
    int32_t slot[64];
    double lr, beta1, beta2, eps;
} dpd_fit_spec;
DPD_API int dpd_fit_graph(dpd_handle *h, int64_t nsteps, int32_t ckpt_every, const dpd_rdf_spec *spec,
                          const double *target, const dpd_fit_spec *fit, int32_t iters, double *loss, double *grad,
                          double *values);

/* Vector-Jacobian product of the forces of replica r's current configuration
 * at `step` (noise key and kT(t)): pair terms, bonds and angle terms (linear
 * chains and the templates of the branched shapes) and stirring.  Given the
 * force cotangent (gx, gy, slot order), the gradients with respect to
 * positions (xbar), predicted velocities (vbar) and parameters (grad,
 * DPD_NGRAD values). */
DPD_API int dpd_force_vjp(dpd_handle *h, int32_t replica, int64_t step, const float *gx, const float *gy,
                          float *xbar_x, float *xbar_y, float *vbar_x, float *vbar_y, double *grad);

/* ---- the cell sort without any allocation ----
 * No counterpart in the reference (its sort always runs inside the engine,
 * oercel.c:832-933, on buffers the engine allocated).  For callers that must
 * not allocate device memory, e.g. code inside another framework's operator
 * or plugin hook, where cudaMalloc's device-wide synchronisation is not
 * allowed: the stable cell sort of n positions (x, y: DEVICE arrays in [0, L))
 * with the cell grid of the handle API, writing cstart (floor(L)^2 + 1 DEVICE
 * entries) and order (n DEVICE entries: input index of each sorted slot).
 * The grid side is floor((float)L); an L whose rounding to float changes its
 * floor (31.9999999 -> 32.0f) is refused with DPD_E_ARG, so floor(L) is
 * always the side.  Positions outside [0, L) are clamped into the edge cells.
 * Any number of beads may share a cell (crowded cells are sorted by whole
 * CTAs; the work stays bounded even with every bead in one cell).
 * Scratch lives in one fixed device array of the library (8.0 MiB per GPU):
 * n <= DPD_NOALLOC_MAX_BEADS and floor(L)^2 <= DPD_NOALLOC_MAX_CELLS, else
 * DPD_E_ARG.  Calls whose work overlaps on the GPU race on that array.  The
 * first call on a device looks up the array's address and keeps it for the
 * life of the process: make it before any stream capture, and do not call
 * this on a device after a cudaDeviceReset of it.  stream: a cudaStream_t
 * (NULL = the default stream). */
#define DPD_NOALLOC_MAX_BEADS 1048576
#define DPD_NOALLOC_MAX_CELLS 524288
DPD_API int dpd_sort_cells_noalloc(const float *x, const float *y, int32_t n, double L, int32_t *cstart,
                                   int32_t *order, void *stream);

#ifdef __cplusplus
}
#endif
#endif
