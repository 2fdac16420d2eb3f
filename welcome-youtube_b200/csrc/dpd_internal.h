// dpd_internal.h -- device data layout shared by the kernels and the C ABI of libdpd.so.
//
// Layout in HBM (one set of arrays for all replicas, replica r owning the bead
// range [b0, b0 + n) and the cell range [c0, c0 + ncell)):
//   per bead, double-buffered (the cell sort permutes buffer cur -> 1 - cur):
//     pos  float2  x, y in [0, L)
//     vh   float2  stored half-step velocity (reference Sys.vx/vy)
//     vt   float2  Groot-Warren predicted velocity (reference Sys.vtx/vty)
//     f    float2  force of the current configuration
//     tg   u32     type << 29 | gid  (gid < 2^29)
//     link int2    prev, next slot of the bonded neighbours (-1 = none)
//   per bead, single: key (cell of the next position), src (old slot of each
//     new slot), dest (inverse), req/claim (chemistry requests)
//   per cell: count (beads whose next position falls in the cell), cstart
//     (exclusive scan of count; cstart of the packed cell C_total = N), fill
//     (placement cursor)
#pragma once
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "../../include/dpd.h"

#define DPD_MAXT 8
#define TYPE_SHIFT 29
#define GID_MASK 0x1FFFFFFFu

#define BEAD_TPB 256
#define CELL_TPB 256
#define SCAN_TPB 256
#define SCAN_PER_THREAD 4
#define SCAN_PER_BLOCK (SCAN_TPB * SCAN_PER_THREAD)

// status flags raised by kernels (read back once per API call)
#define DPD_F_OUTSIDE 0x1u      // a bead left [0, L) after integration
#define DPD_F_NONFINITE 0x2u    // non-finite force or position
#define DPD_F_EVENTS 0x4u       // event buffer overflow
#define DPD_F_CHAIN 0x8u        // broken chain link found
#define DPD_F_BIGCELL 0x10u     // a cell held more beads than the in-register sort handles (slow path used)
#define DPD_F_TILE 0x20u        // a cell tile held more beads than its shared-memory capacity
#define DPD_F_FORCE 0x40u       // a single pair or bond force term above the fixed-point range
#define DPD_F_CATALYST 0x80u    // a catalyst's neighbourhood exceeded the staging capacity
#define DPD_CAT_MAXTR 64        // orientation trials of one lipid synthesis (syn_tries)
#define DPD_F_ANALYSIS 0x200u   // a cluster union kept losing its compare-and-swap (analysis result invalid)
#define DPD_F_WAIT 0x800u       // a bounded device wait (an mbarrier, a look-back of the scan) gave up
#define DPD_F_INPUT 0x400u      // a state handed in had a non-finite position, a type >= DPD_MAXT, a gid >= n
                                // or a link outside [-1, n): stored sanitised, the call fails

struct RepDev {                 // constants of one replica, read by every kernel
    float L, halfL;
    int32_t ncx, ncy;
    double icsx, icsy;          // ncx / L, ncy / L (cell index product in FP64, as the reference)
    int32_t b0, n, c0, ncell;   // packed bead and cell offsets
    float dt, dt2, cvt, hdt;    // dt, dt^2, (1/2 + lambda) dt, dt / 2 (FP32)
    float gamma, sdt;           // gamma, sigma / sqrt(dt)
    float kb, r0;
    float a[DPD_MAXT * DPD_MAXT];
    uint64_t seed;
    int32_t noise;              // 0 Philox4x32-10, 1 reference mix13
    int32_t chem, n_chem;
    uint32_t thr_break, thr_grow, thr_bond;
    float r2_grow, r2_bond;
    int32_t n_t_min, max_chain;
    int32_t pad;
    long long warm_end;         // repulsions above 25 ramp in until this step (oercel.c:1124-1129)
    double warm_inv;            // 1 / warmup, 0 = no ramp
    float ka;                   // angle constant (0 = no angle terms)
    float stir_A;               // stirring amplitude (0 = off)
    double stir_k;              // stir_n / L (the argument of the sine is 2 pi stir_k y)
    double kT, kT_amp, kT_w;    // kT(t) = kT + kT_amp sin(kT_w t)
    double gamma_d, dt_d;       // gamma, dt in FP64 (sigma / sqrt(dt) of a step)
    double t_anchor;            // t(step) = t_anchor + (step - step_anchor) dt
    long long step_anchor;
    // the reference's catalyst chemistry (chem_kind 1, dpd_catalyst.cu)
    int32_t chem_kind, syn_tries, syn_relax, syn_nN, lip_nH, lip_nT, feed_mode, vent_kind;
    int32_t ch0, nch;           // this replica's chunks in the bead chunk table
    int32_t cat_E;              // half-width in cells of the window staged around a catalyst
    int32_t arch;               // lipid shape (0 linear: per-bead bond terms; else the template, k_mol_forces)
    long long so;               // first draw of this replica's catalyst stream (a multiple of 64)
    int32_t dcap, pad4;         // draws its stream holds (a multiple of 64)
    double r_cat, p_syn_a, p_syn_b, p_rep_a, p_rep_b, mu, p_ld, p_kd, p_nd, p_feed, feed_cap;
    double vent_x, vent_y, vent_r, vent_w;
    double kb_d, r0_d, ka_d;    // FP64 bond and angle constants for the relaxation of new chains
};

// sigma / sqrt(dt) at `step`: constant, or with the temperature cycle
// kT(t) = kT + kT_amp sin(2 pi t / kT_period) (oercel.c:622-624, 1204)
__device__ __forceinline__ float sdt_at(const RepDev &R, long long step) {
    if (R.kT_amp == 0.0) return R.sdt;
    const double t = R.t_anchor + (double)(step - R.step_anchor) * R.dt_d;
    const double kT = R.kT + R.kT_amp * sin(R.kT_w * t);
    return (float)(sqrt(2.0 * R.gamma_d * kT) / sqrt(R.dt_d));
}

// the repulsion in force at `step`: during the warm-up of a fresh soup the part
// of a_ij above the water value 25 is ramped in linearly (oercel.c:1124-1129)
__device__ __forceinline__ float a_at(const RepDev &R, int k, long long step) {
    const float a = R.a[k];
    if (R.warm_inv == 0.0 || step >= R.warm_end || a <= 25.0f) return a;
    double f = 1.0 - (double)(R.warm_end - step) * R.warm_inv;
    f = f < 0.0 ? 0.0 : f;
    return (float)(25.0 + ((double)a - 25.0) * f);
}

struct Chunk {                  // one CTA's work: packed indices [begin, end) of replica rep
    int32_t rep, begin, end, pad;
};

struct TileDesc {               // one CTA of the tiled force kernel: cells [cx0, cx0+w) x [cy0, cy0+h)
    int32_t rep, cx0, cy0, w, h;
    int32_t c0, ncx, ncy;       // the replica's first cell and grid (its RepDev's), read with the tile
};

struct DevStatus {
    unsigned int flags;
    unsigned int nevents;       // events appended (may exceed the capacity)
    unsigned int bigcell;       // largest cell population seen by the sort fix-up
    unsigned int n_grow;        // chemistry candidate lists of this step
    unsigned int n_bond;
    unsigned int done;          // CTAs finished in the current chemistry list kernel (the last one applies)
    unsigned int pad[2];
};

struct EventDev {
    long long step;
    int kind;
    unsigned int gid, partner;
    float x, y;
    int replica;
};

#define OBS_N 16
// per-replica observable accumulators (fixed point, integer atomics => deterministic)
//   0: sum vx * 2^24   1: sum vy * 2^24   2: sum v^2 * 2^24   3: virial sum a w r * 2^24
//   4: max bond length (float bits)   5: chain heads   8..15: type counts
#define OBS_FIX 16777216.0

struct Bufs {
    float2 *pos[2], *vh[2], *vt[2], *f[2];
    uint32_t *tg[2];
    int2 *link[2];
    uint32_t *key;
    uint32_t *fill;             // per cell: next free slot while beads are placed (cstart + count so far)
    int32_t *src, *dest;
    uint32_t *count;
    int32_t *cstart;            // C + 1
    int32_t *bsum;              // scan block totals
    unsigned long long *scan_state;   // single-pass scan: per block (epoch | flag | value), see k_scan_lb
    unsigned long long *scan_ticket;  // single-pass scan: block tickets taken so far (never reset)
    uint32_t *claim;            // per bead, 0xFFFFFFFF when unclaimed
    int32_t *req;               // per candidate chemistry request target (-1 none)
    int2 *grow_list;            // (slot, replica) of P beads whose growth draw succeeded
    int2 *bond_list;            // (slot, replica) of T beads whose bonding draw succeeded
    EventDev *events;
    int32_t evcap;
    DevStatus *status;
    long long *step;            // step number of the forces being computed
    unsigned long long *obs;    // OBS_N per replica: the running sums (zero between stats rows)
    unsigned long long *obs_out;  // OBS_N per replica: the last stats row, handed over by k_observables
    unsigned int *obs_done;     // per replica: blocks of k_observables finished
    unsigned long long *hist;   // pair histogram scratch
    long long *stir;            // per replica: sum of the stirring terms (fixed point) of the current positions
    uint64_t *rng;              // per replica: the serial xoshiro256** state of the catalyst chemistry (4 words)
    int32_t *cat_list;          // per bead slot: catalyst / feed candidates of a replica in slot order (at b0)
    int32_t *cat_cnt;           // per bead chunk: candidates in the chunk
    int32_t *cat_ncnt;          // per bead chunk: N beads in the chunk (the feed cap)
    int32_t *resort;            // [0]: some replica needs a sort before its catalyst check; [1 + r]: replica r
    int32_t *cat_nk;            // per replica: catalysts of the current check
    uint32_t *cat_near;         // per catalyst list entry: packed candidate counts (k_cat_near)
    int32_t *cat_cell;          // per catalyst list entry: its cell
    uint8_t *cat_mark;          // per cell: a bead near it changed type in the current check
    const dpd_template *mol;    // per replica: its lipid template
    const uint64_t *jump;       // x^(64 m) mod the xoshiro256** polynomial, 4 words per m (dpd_jump.cu)
    uint64_t *stream;           // the draws of a catalyst check, from RepDev::so per replica
    uint64_t *sblock;           // the generator state at every 64th draw of the stream
    long long *cat_dn;          // per replica: draws in the current check's stream
    int32_t *shuf;              // 8 x shuf_n scratch of the parallel shuffle (per replica at b0)
    long long shuf_n;
    int2 *fmol;                 // per bead: fixed-point bonded force of a branched lipid (k_mol_forces)
};

struct StateView {              // one stored configuration (slot order of its own step)
    const float2 *pos, *vt;
    const uint32_t *tg;
    const int2 *link;
    const int32_t *cstart;      // packed cells (C + 1)
};

#ifndef DPD_NGRAD
#define DPD_NGRAD (DPD_MAXT * DPD_MAXT + 2)
#endif

// launch a kernel of the step with programmatic dependent launch allowed (the
// kernel begins with pdl_begin(), which waits for its predecessor)
template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*k)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t s,
                       Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k, (KArgs)args...);
}

// the catalyst chemistry of one check (dpd_catalyst.cu): catalysts, decay, food supply
int catalyst_setup();
void launch_catalyst(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, int nrep, int64_t C,
                     int nmax, int stream_grid, cudaStream_t s);
int jump_table(int nblk, std::vector<uint64_t> &out);

// launchers (dpd_kernels.cu, dpd_chem.cu, dpd_adjoint.cu); every launcher enqueues on stream s
// PERM_KEEP: the step's update with the slot order kept (source = destination)
enum PermuteMode { PERM_STEP = 0, PERM_PRIME = 1, PERM_SORT = 2, PERM_KEEP = 3 };

void launch_keys(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, bool integrate,
                 cudaStream_t s);
void launch_scan(const Bufs &b, int64_t C, bool step_inc, cudaStream_t s);

void launch_scan_part(const Bufs &b, int64_t C, bool step_inc, int part, cudaStream_t s);
// the same exclusive scan in one pass (decoupled look-back between blocks)
void launch_scan_lb(const Bufs &b, int64_t C, bool step_inc, cudaStream_t s);
// the sort of a step in three kernels (block-local scan, placement and fix-up
// adding the block prefixes themselves); part 0..2 or all with part < 0
bool sort_pfx_fits(int64_t C);
void launch_sort_pfx(const Bufs &b, int64_t C, bool step_inc, const Chunk *bch, int nbch, const Chunk *cch, int ncch,
                     int part, cudaStream_t s);
void launch_place(const Bufs &b, const Chunk *bch, int nbch, cudaStream_t s);
void launch_cellfix(const Bufs &b, const Chunk *cch, int ncch, cudaStream_t s);
void launch_permute(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, PermuteMode mode,
                    cudaStream_t s);
void launch_forces(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, bool pair, bool bond,
                   bool next_keys, cudaStream_t s);
void launch_halfkick(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, cudaStream_t s);
void launch_integrate(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, cudaStream_t s);
void launch_step_begin(const Bufs &b, int nrep, cudaStream_t s);
void launch_events_out(const Bufs &b, EventDev *out, int cap, int *n_out, cudaStream_t s);
void launch_mol_forces(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, cudaStream_t s);
void launch_type_clusters(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, int rep_index, int t,
                          double rcut, int *parent, int *size, unsigned long long *acc, cudaStream_t s);
void launch_aggregates(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, int rep_index, int n,
                       double r_tail, int min_lipids, int *parent, int *size, int *minlab, unsigned long long *acc,
                       int32_t *out_label, cudaStream_t s);
void launch_resort(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, const Chunk *cch, int ncch,
                   int64_t C, cudaStream_t s);
void launch_observables(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, int rep_index,
                        bool virial, unsigned long long *host_out, int ring_slots, cudaStream_t s);
void launch_pair_hist(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, int rep_index, int ta,
                      int tb, double rmax, int nbin, cudaStream_t s);
void launch_pack(const Bufs &b, int cur, int b0, int n, float L, const float *x, const float *y, const float *vx,
                 const float *vy, const uint8_t *type, const uint32_t *gid, const int32_t *prev,
                 const int32_t *next, cudaStream_t s);
void launch_unpack(const Bufs &b, int cur, int b0, int n, float *x, float *y, float *vhx, float *vhy, float *vtx,
                   float *vty, float *fx, float *fy, uint8_t *type, uint32_t *gid, int32_t *prev, int32_t *next,
                   cudaStream_t s);
void launch_set_dynamics(const Bufs &b, int cur, int b0, int n, const float *vhx, const float *vhy,
                         const float *fx, const float *fy, const float *vtx, const float *vty, cudaStream_t s);
// A stats row that the tile force kernel assembles in its epilogue, in place
// of a separate pass over the beads: replica rep's row of this step (rep < 0:
// none), handed over to obs_out and, when host is set, into the ring
// host[step % slots] (the step in word 6), as k_observables does.
struct RowOut {
    int32_t rep, slots;
    unsigned long long *host;
};
void launch_forces_tile(const Bufs &b, int cur, const RepDev *rep, const TileDesc *tiles, int ntiles, int threads,
                        bool next_keys, cudaStream_t s, RowOut row = RowOut{-1, 0, nullptr});
int tile_setup();
size_t tile_smem_bytes();
size_t bulk_smem_bytes();
void launch_forces_bulk(const Bufs &b, int cur, const RepDev *rep, const TileDesc *tiles, int ntiles,
                        bool next_keys, cudaStream_t s);
// gsum: nrep doubles of scratch (the mean x cotangent of the stirring term), used when stir;
// mol: the replicas' lipid templates when some replica has branched lipids, else null
void launch_force_vjp(const StateView &sv, long long step, const RepDev *rep, const Chunk *bch, int nbch,
                      const float2 *g, float2 *xbar, float2 *vbar, double *grad, double *gsum, int nrep, bool stir,
                      const dpd_template *mol, cudaStream_t s, const long long *step_base = nullptr);
// the device side of a fit iteration that runs without the host (dpd_fit_graph); FitDev is in device memory
struct FitDev {
    long long base;             // the device step at the start of the iteration's window
    int iter;                   // iterations done
    int nfit;                   // fitted a_ij slots (i * DPD_MAXT + j, i <= j), shared by every replica
    int slot[DPD_MAXT * DPD_MAXT];
    double value[DPD_MAXT * DPD_MAXT], m[DPD_MAXT * DPD_MAXT], v[DPD_MAXT * DPD_MAXT];
    double lr, beta1, beta2, eps;
};
void launch_fit_begin(long long *step, FitDev *fd, cudaStream_t s);
void launch_set_step_rel(long long *step, const FitDev *fd, long long off, cudaStream_t s);
void launch_rdf_loss(const RepDev *rep, int nrep, const double *hist, const long long *npairs, const double *target,
                     int nbin, double rmax, int last_steps, double *loss_out, double *wgt, const FitDev *fd,
                     cudaStream_t s);
void launch_fit_update(RepDev *rep, int nrep, const double *grad, FitDev *fd, double *grad_out, double *value_out,
                       cudaStream_t s);
void launch_rdf(const StateView &sv, const RepDev *rep, const Chunk *bch, int nbch, int ta, int tb, int nbin,
                float rmax, float sigma, double *hist, cudaStream_t s);
void launch_rdf_vjp(const StateView &sv, const RepDev *rep, const Chunk *bch, int nbch, int ta, int tb, int nbin,
                    float rmax, float sigma, const double *wgt, float2 *xadd_gid, cudaStream_t s);
void launch_adj_update(const uint32_t *tg, const RepDev *rep, const Chunk *bch, int nbch, const float2 *xb,
                       const float2 *vb, float2 *X, float2 *V, float2 *F, cudaStream_t s);
void launch_adj_gather(const uint32_t *tg, const RepDev *rep, const Chunk *bch, int nbch, const float2 *F, float2 *g,
                       cudaStream_t s);
void launch_adj_state(const uint32_t *tg, const RepDev *rep, const Chunk *bch, int nbch, const float2 *xb,
                      const float2 *vb, float2 *X, float2 *VT, cudaStream_t s);
void launch_adj_save(int n, const float2 *pos, const float2 *vt, const uint32_t *tg, const int2 *link, float2 *opos,
                     float2 *ovt, uint32_t *otg, int2 *olink, cudaStream_t s);
int chem_kernel_count();
int lib_error(int code, const char *msg);  // sets dpd_last_error() and returns code
// the break stage and the candidate draws on the current sorted state (phase entry point)
void launch_chem_scan(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, cudaStream_t s);
// the growth and bonding stages over the candidate lists (part 0..3, or all with part < 0)
void launch_chem_lists(const Bufs &b, int cur, const RepDev *rep, int part, cudaStream_t s);
