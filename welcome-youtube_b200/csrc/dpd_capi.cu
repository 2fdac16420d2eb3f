// dpd_capi.cu -- the C ABI of libdpd.so (include/dpd.h): handles, device
// memory, CUDA graphs of the step, state in/out, error reporting.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <numeric>
#include <vector>

#include "../../include/dpd.h"
#include "dpd_internal.h"

static_assert(sizeof(dpd_event) == sizeof(EventDev), "event layout");

static thread_local std::string g_err;

static int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

// the error message of a call made outside this file (dpd_cells.cu)
int lib_error(int code, const char *msg) {
    g_err = msg;
    return code;
}

#define CK(call)                                                                                        \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) return fail(DPD_E_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                                           __FILE__, __LINE__);                                         \
    } while (0)

// reverse-mode storage (defined here: the handle keeps it between windows)
namespace {
struct FullCk {  // a full configuration of the engine's current buffer
    float2 *pos, *vh, *vt, *f;
    uint32_t *tg;
    int2 *link;
    int32_t *cstart;
};
struct SegState {  // what a force VJP needs of one configuration
    float2 *pos, *vt;
    uint32_t *tg;
    int2 *link;
    int32_t *cstart;
};
struct AdjBufs {
    std::vector<FullCk> ck;  // checkpoints + the end of the window (last)
    std::vector<SegState> seg;
    float2 *X, *V, *F, *g, *xb, *vb;
    double *hist, *wgt, *grad;
    double *gsum;            // per replica: the sum of the x cotangents (stirring)
};
}  // namespace

struct dpd_handle {
    int nrep = 0;
    std::vector<dpd_params> params;
    std::vector<RepDev> rh;
    int64_t N = 0, C = 0;
    int nmax = 0;
    cudaStream_t s = nullptr;
    RepDev *d_rep = nullptr;
    Chunk *d_bch = nullptr, *d_cch = nullptr;
    int nbch = 0, ncch = 0;
    Bufs b{};
    int cur = 0;
    // force kernel: 0 = cell tiles in shared memory (half shell), 1 = one thread per bead (full shell)
    int force_kernel = 0;      // 0 cell tiles, 1 thread per bead, 2 cell tiles staged by bulk copies
    int sort_mode = 2;
    int tile_threads = 256;    // threads per CTA of the tile kernel (256 or 512: tiles of up to that many local cells)         // 0 two scan passes, 1 one scan pass (k_scan_lb), 2 no second pass (block prefixes in place/cellfix)
    int tile_w = 8, tile_h = 16;
    TileDesc *d_tiles = nullptr;
    int ntiles = 0;
    bool any_chem = false;
    bool any_stir = false;      // some replica stirs: its term sums are cleared before each permute
    bool keys_valid = false;
    int64_t step = 0;
    // CUDA graphs of gsteps consecutive steps, one per starting buffer parity
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    // the stats ring: every step writes replica ring_rep's row into ring[step % ring_slots]
    unsigned long long *ring = nullptr;
    int32_t ring_rep = 0, ring_slots = 0;
    int gflip[2] = {0, 0};      // buffer parity change of one replay (steps + the extra sorts of catalyst checks)
    int gsteps = 0;
    // the reference's catalyst chemistry: replicas with chem_kind 1, the period of their checks
    bool any_cat = false, any_lipid = false;
    bool any_mol = false;       // some replica has branched lipids (k_mol_forces)
    int stream_grid = 1;        // blocks per replica of the catalyst stream kernel
    int64_t cat_period = 0;
    // reverse-mode storage, grown on demand (full checkpoints, the states of one
    // recomputed segment, adjoint arrays in gid order)
    std::vector<void *> adj_allocs;
    int adj_nck = 0, adj_nseg = 0, adj_nbin = 0;  // capacity of adj (0: none yet)
    AdjBufs adj;
    // staging for state in/out
    char *stage = nullptr;
    // cluster analysis scratch (allocated on first use): union-find parents, sizes, sums
    int *ana_parent = nullptr, *ana_size = nullptr, *ana_min = nullptr;
    int32_t *ana_label = nullptr;
    unsigned long long *ana_acc = nullptr;
    std::vector<void *> allocs;
};

extern "C" const char *dpd_last_error(void) { return g_err.c_str(); }
extern "C" const char *dpd_version(void) { return "libdpd 0.1 (sm_100a)"; }

extern "C" int dpd_params_default(dpd_params *p) {
    if (!p) return fail(DPD_E_ARG, "null params");
    memset(p, 0, sizeof *p);
    p->L = 64.0;   // reference defaults: cel/engine/oercel.c:237-299
    p->dt = 0.03;
    p->lambda = 0.65;
    p->gamma = 4.5;
    p->kT = 1.0;
    for (int i = 0; i < DPD_MAXT * DPD_MAXT; i++) p->a[i] = 25.0;
    p->k_bond = 100.0;
    p->r0 = 0.5;
    p->k_angle = 10.0;
    p->stir_n = 1;
    p->kT_period = 1000.0;
    p->chem_kind = 0;
    p->syn_tries = 8;   // catalyst chemistry: the reference's defaults, oercel.c:262-290
    p->syn_relax = 20;
    p->lip_nH = 1;
    p->lip_nT = 3;
    p->feed_mode = 1;
    p->r_cat = 1.2;
    p->p_syn_a = 0.02;
    p->p_syn_b = 0.06;
    p->p_rep_a = 0.001;
    p->p_rep_b = 0.001;
    p->mu = 0.02;
    p->p_ld = 2e-4;
    p->p_kd = 5e-4;
    p->p_nd = 1e-4;
    p->p_feed = 1e-3;
    p->feed_cap = 0.12;
    p->vent_x = -1.0;
    p->vent_y = -1.0;
    p->vent_r = 5.0;
    p->r0_head = 0.5;
    p->vent_w = 4.0;
    p->seed = 1;
    p->noise = 0;
    p->chem = 0;
    p->n_chem = 1;
    p->n_t_min = 2;
    p->max_chain = 12;  // reference MAXMLEN, oercel.c:50
    p->p_break = 1e-5;
    p->p_grow = 1e-3;
    p->p_bond = 1e-2;
    p->r_grow = 1.0;
    p->r_bond = 0.6;
    return DPD_OK;
}

static uint32_t threshold(double p) {
    const double t = std::floor(p * 4294967296.0);
    if (!(t > 0.0)) return 0u;
    if (t >= 4294967295.0) return 0xFFFFFFFFu;
    return (uint32_t)t;
}

static int make_rep(const dpd_params &p, int b0, int n, int c0, RepDev &R) {
    memset(&R, 0, sizeof R);
    if (!(p.L >= 3.0) || !std::isfinite(p.L)) return fail(DPD_E_ARG, "L must be >= 3 (got %g)", p.L);
    if (!(p.dt > 0.0)) return fail(DPD_E_ARG, "dt must be > 0");
    if (!(p.kT > 0.0)) return fail(DPD_E_ARG, "kT must be > 0");
    if (p.gamma < 0.0) return fail(DPD_E_ARG, "gamma must be >= 0");
    if (p.noise != 0 && p.noise != 1) return fail(DPD_E_ARG, "noise must be 0 (philox) or 1 (mix13)");
    if (p.chem && p.n_chem < 1) return fail(DPD_E_ARG, "n_chem must be >= 1");
    if (p.chem && (p.max_chain < 2 || p.max_chain > 1000)) return fail(DPD_E_ARG, "max_chain must be 2..1000");
    if (p.chem && !(p.r_grow > 0.0 && p.r_grow <= 1.0 && p.r_bond > 0.0 && p.r_bond <= 1.0))
        return fail(DPD_E_ARG, "reaction radii must lie in (0, 1]");
    for (int i = 0; i < DPD_MAXT; i++)
        for (int j = 0; j < DPD_MAXT; j++)
            if (p.a[i * DPD_MAXT + j] != p.a[j * DPD_MAXT + i]) return fail(DPD_E_ARG, "a_ij must be symmetric");
    R.L = (float)p.L;
    R.halfL = 0.5f * R.L;
    R.ncx = R.ncy = (int)std::floor((double)R.L);
    R.icsx = R.ncx / (double)R.L;
    R.icsy = R.ncy / (double)R.L;
    R.b0 = b0;
    R.n = n;
    R.c0 = c0;
    R.ncell = R.ncx * R.ncy;
    R.dt = (float)p.dt;
    R.dt2 = (float)(p.dt * p.dt);
    R.cvt = (float)((0.5 + p.lambda) * p.dt);
    R.hdt = (float)(0.5 * p.dt);
    R.gamma = (float)p.gamma;
    R.sdt = (float)(std::sqrt(2.0 * p.gamma * p.kT) / std::sqrt(p.dt));
    R.kb = (float)p.k_bond;
    R.r0 = (float)p.r0;
    for (int i = 0; i < DPD_MAXT * DPD_MAXT; i++) R.a[i] = (float)p.a[i];
    R.seed = p.seed;
    R.noise = p.noise;
    R.chem = p.chem;
    R.n_chem = p.n_chem;
    R.thr_break = threshold(p.p_break);
    R.thr_grow = threshold(p.p_grow);
    R.thr_bond = threshold(p.p_bond);
    R.r2_grow = (float)(p.r_grow * p.r_grow);
    R.r2_bond = (float)(p.r_bond * p.r_bond);
    R.n_t_min = p.n_t_min;
    R.max_chain = p.max_chain;
    if (p.warmup < 0) return fail(DPD_E_ARG, "warmup must be >= 0");
    R.warm_end = (long long)p.warm_end;
    R.warm_inv = p.warmup > 0 ? 1.0 / (double)p.warmup : 0.0;
    if (p.k_angle < 0.0 || !std::isfinite(p.k_angle)) return fail(DPD_E_ARG, "k_angle must be >= 0");
    R.ka = (float)p.k_angle;
    if (p.stir_A != 0.0 && p.stir_n < 1) return fail(DPD_E_ARG, "stir_n must be >= 1");
    if (!std::isfinite(p.stir_A)) return fail(DPD_E_ARG, "stir_A must be finite");
    R.stir_A = (float)p.stir_A;
    R.stir_k = p.stir_A != 0.0 ? (double)p.stir_n / p.L : 0.0;
    if (p.kT_amp != 0.0) {
        if (!(p.kT_period > 0.0)) return fail(DPD_E_ARG, "kT_period must be > 0");
        if (!(p.kT - std::fabs(p.kT_amp) > 0.0)) return fail(DPD_E_ARG, "kT - |kT_amp| must be > 0");
    }
    R.kT = p.kT;
    R.kT_amp = p.kT_amp;
    R.kT_w = p.kT_amp != 0.0 ? 2.0 * M_PI / p.kT_period : 0.0;
    R.gamma_d = p.gamma;
    R.dt_d = p.dt;
    R.t_anchor = p.t_anchor;
    R.step_anchor = (long long)p.step_anchor;
    R.kb_d = p.k_bond;
    R.r0_d = p.r0;
    R.ka_d = p.k_angle;
    R.chem_kind = p.chem_kind;
    if (p.chem_kind != 0 && p.chem_kind != 1) return fail(DPD_E_ARG, "chem_kind must be 0 (lipid) or 1 (catalyst)");
    // the lipid template: branched shapes need it for their bonds, the catalyst chemistry for new lipids
    dpd_template M;
    const bool need_mol = p.lip_arch != 0 || (p.chem && p.chem_kind == 1);
    if (dpd_lipid_template(&p, &M) != DPD_OK) {
        if (need_mol) return fail(DPD_E_ARG, "lipid shape: lip_arch 0..3 with 2..%d beads (lip_nH >= 1, lip_nT >= 1 "
                                             "for branched shapes)", DPD_MAXML);
        M.mlen = p.lip_nH + p.lip_nT;
        M.nH = p.lip_nH;
    }
    R.arch = p.lip_arch;
    if (p.chem && p.chem_kind == 1) {
        const int ml = M.mlen;
        double ext = 0.0;  // the template's reach from its centroid
        for (int b = 0; b < ml; b++) ext = std::max(ext, std::sqrt(M.px[b] * M.px[b] + M.py[b] * M.py[b]));
        if (!(p.r_cat > 0.0) || p.syn_tries < 1 || p.syn_tries > DPD_CAT_MAXTR || p.syn_relax < 0 || p.syn_nN < 0 ||
            p.syn_nN > ml)
            return fail(DPD_E_ARG, "need r_cat > 0, 1 <= syn_tries <= %d, syn_relax >= 0, 0 <= syn_nN <= mlen",
                        DPD_CAT_MAXTR);
        if (p.feed_mode < 0 || p.feed_mode > 2 || p.vent_kind < 0 || p.vent_kind > 2)
            return fail(DPD_E_ARG, "feed_mode 0..2, vent_kind 0..2");
        if (p.p_feed < 0.0 || p.p_feed > 1.0 || p.feed_cap < 0.0 || p.feed_cap >= 1.0)
            return fail(DPD_E_ARG, "p_feed in [0, 1], feed_cap in [0, 1)");
        // the cells a catalyst's visit can reach: the N window, the new chain's
        // extent around the centroid, and the energy and relaxation windows
        const double reach = 1.0 + 0.05 * p.syn_relax, ics = R.ncx / (double)R.L;
        const int wmax = std::max({(int)std::ceil((p.r_cat + 0.5) * ics), (int)std::ceil(1.5 * ics),
                                   (int)std::ceil((reach + 0.5) * ics)});
        R.cat_E = (int)std::ceil((p.r_cat + ext) * ics) + 2 + wmax;
        if (2 * (int)std::ceil((reach + 0.5) * ics) + 1 > R.ncx)
            return fail(DPD_E_ARG, "box too small for the catalyst windows (L must exceed 2 (r_cat, reach) + 1)");
    }
    R.syn_tries = p.syn_tries;
    R.syn_relax = p.syn_relax;
    R.syn_nN = p.syn_nN;
    R.lip_nH = M.nH;  // heads first, mlen beads (the template's, for every shape)
    R.lip_nT = M.mlen - M.nH;
    R.feed_mode = p.feed_mode;
    R.vent_kind = p.vent_kind;
    R.r_cat = p.r_cat;
    R.p_syn_a = p.p_syn_a;
    R.p_syn_b = p.p_syn_b;
    R.p_rep_a = p.p_rep_a;
    R.p_rep_b = p.p_rep_b;
    R.mu = p.mu;
    R.p_ld = p.p_ld;
    R.p_kd = p.p_kd;
    R.p_nd = p.p_nd;
    R.p_feed = p.p_feed;
    R.feed_cap = p.feed_cap;
    R.vent_x = p.vent_x < 0.0 ? 0.5 * p.L : p.vent_x;  // the reference centres an unset vent (oercel.c:607-608)
    R.vent_y = p.vent_y < 0.0 ? 0.5 * p.L : p.vent_y;
    R.vent_r = p.vent_r;
    R.vent_w = p.vent_w;
    return DPD_OK;
}

template <typename T>
static int dalloc(dpd_handle *h, T **p, size_t count) {
    void *q = nullptr;
    const size_t bytes = count * sizeof(T) + 64;
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) return fail(DPD_E_NOMEM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
    h->allocs.push_back(q);
    *p = (T *)q;
    return DPD_OK;
}

#define TRY(x)                       \
    do {                             \
        int r_ = (x);                \
        if (r_ != DPD_OK) return r_; \
    } while (0)

// graph length: with catalyst chemistry a multiple of its period (so that a
// replay starting on a multiple of the period holds the checks in place)
static int graph_len(const dpd_handle *h, int g) {
    g = std::max(1, g);
    const int64_t P = h->cat_period;
    if (P > 0 && P <= 1024) g = (int)(((g + P - 1) / P) * P);
    return g;
}

static void drop_graphs(dpd_handle *h) {
    for (int k = 0; k < 2; k++)
        if (h->gexec[k]) {
            cudaGraphExecDestroy(h->gexec[k]);
            h->gexec[k] = nullptr;
        }
}

static void free_adj(dpd_handle *h) {
    for (void *p : h->adj_allocs) cudaFree(p);
    h->adj_allocs.clear();
    h->adj_nck = h->adj_nseg = h->adj_nbin = 0;
    h->adj = AdjBufs();
}

static void free_all(dpd_handle *h) {
    drop_graphs(h);
    free_adj(h);
    for (void *p : h->allocs) cudaFree(p);
    h->allocs.clear();
    if (h->s) cudaStreamDestroy(h->s);
}

// cell tiles of every replica: w x h cells (narrower boxes get narrower tiles,
// so that a tile and its halo never hold the same column or row twice)
static int build_tiles(dpd_handle *h) {
    const int maxc = h->force_kernel == 0 ? h->tile_threads : 256;
    if (h->tile_w < 1 || h->tile_h < 1 || (h->tile_w + 2) * (h->tile_h + 2) > maxc)
        return fail(DPD_E_ARG, "tile shape %dx%d: need (w+2)(h+2) <= %d", h->tile_w, h->tile_h, maxc);
    std::vector<TileDesc> t;
    for (int r = 0; r < h->nrep; r++) {
        const RepDev &R = h->rh[r];
        const int w = std::min(h->tile_w, R.ncx - 2), hh = std::min(h->tile_h, R.ncy - 2);
        for (int cx = 0; cx < R.ncx; cx += w)
            for (int cy = 0; cy < R.ncy; cy += hh)
                t.push_back({r, cx, cy, std::min(w, R.ncx - cx), std::min(hh, R.ncy - cy), (int32_t)R.c0, R.ncx, R.ncy});
    }
    if (h->d_tiles) {
        cudaFree(h->d_tiles);
        for (auto &p : h->allocs)
            if (p == (void *)h->d_tiles) p = nullptr;
    }
    TRY(dalloc(h, &h->d_tiles, t.size()));
    CK(cudaMemcpy(h->d_tiles, t.data(), t.size() * sizeof(TileDesc), cudaMemcpyHostToDevice));
    h->ntiles = (int)t.size();
    return DPD_OK;
}

// the exclusive scan of the cell counts, in the form the handle's tuning picked
static void enqueue_scan(dpd_handle *h, bool step_inc) {
    if (h->sort_mode == 1) launch_scan_lb(h->b, h->C, step_inc, h->s);
    else launch_scan(h->b, h->C, step_inc, h->s);
}

// the sort of the counted keys into cell order (cell starts, src, dest)
static void enqueue_cell_sort(dpd_handle *h, bool step_inc) {
    if (h->sort_mode == 2 && sort_pfx_fits(h->C)) {
        launch_sort_pfx(h->b, h->C, step_inc, h->d_bch, h->nbch, h->d_cch, h->ncch, -1, h->s);
        return;
    }
    enqueue_scan(h, step_inc);
    launch_place(h->b, h->d_bch, h->nbch, h->s);
    launch_cellfix(h->b, h->d_cch, h->ncch, h->s);
}

// row: a stats row the tile kernel assembles on the way (the other kernels
// leave it to the caller)
static void enqueue_forces(dpd_handle *h, bool next_keys, RowOut row = RowOut{-1, 0, nullptr}) {
    if (h->any_mol) launch_mol_forces(h->b, h->cur, h->d_rep, h->d_bch, h->nbch, h->s);
    if (h->force_kernel == 0)
        launch_forces_tile(h->b, h->cur, h->d_rep, h->d_tiles, h->ntiles, h->tile_threads, next_keys, h->s, row);
    else if (h->force_kernel == 2) launch_forces_bulk(h->b, h->cur, h->d_rep, h->d_tiles, h->ntiles, next_keys, h->s);
    else launch_forces(h->b, h->cur, h->d_rep, h->d_bch, h->nbch, true, true, next_keys, h->s);
}

static int create_impl(dpd_handle *h, const dpd_params *params, int32_t nrep, const int32_t *n_beads) {
    h->nrep = nrep;
    h->params.assign(params, params + nrep);
    h->rh.resize(nrep);
    int64_t b0 = 0, c0 = 0;
    for (int r = 0; r < nrep; r++) {
        if (n_beads[r] < 2) return fail(DPD_E_ARG, "replica %d: need at least 2 beads", r);
        TRY(make_rep(params[r], (int)b0, n_beads[r], (int)c0, h->rh[r]));
        h->any_chem = h->any_chem || params[r].chem;
        h->any_lipid = h->any_lipid || (params[r].chem && params[r].chem_kind == 0);
        if (params[r].chem && params[r].chem_kind == 1) {
            h->any_cat = true;
            const int64_t a = h->cat_period ? h->cat_period : 1, c = params[r].n_chem;
            h->cat_period = a / std::gcd(a, c) * c;
        }
        h->any_stir = h->any_stir || params[r].stir_A != 0.0;
        h->any_mol = h->any_mol || params[r].lip_arch != 0;
        b0 += n_beads[r];
        c0 += h->rh[r].ncell;
        h->nmax = std::max(h->nmax, (int)n_beads[r]);
        if (b0 > (int64_t)GID_MASK || c0 > (int64_t)0x7fffffff - 8)
            return fail(DPD_E_ARG, "too many beads or cells (beads < 2^29 in total)");
    }
    h->N = b0;
    h->C = c0;
    // work chunks: CTAs never straddle replicas
    std::vector<Chunk> bch, cch;
    for (int r = 0; r < nrep; r++) {
        const RepDev &R = h->rh[r];
        h->rh[r].ch0 = (int32_t)bch.size();
        for (int k = 0; k < R.n; k += BEAD_TPB) bch.push_back({r, R.b0 + k, R.b0 + std::min(R.n, k + BEAD_TPB), 0});
        h->rh[r].nch = (int32_t)bch.size() - h->rh[r].ch0;
        for (int k = 0; k < R.ncell; k += CELL_TPB)
            cch.push_back({r, R.c0 + k, R.c0 + std::min(R.ncell, k + CELL_TPB), 0});
    }
    h->nbch = (int)bch.size();
    h->ncch = (int)cch.size();
    CK(cudaStreamCreateWithFlags(&h->s, cudaStreamNonBlocking));
    if (tile_setup() != 0) return fail(DPD_E_CUDA, "cannot reserve %zu bytes of shared memory per CTA", tile_smem_bytes());
    if (const char *e = getenv("DPD_FORCES"))
        h->force_kernel = strcmp(e, "bead") == 0 ? 1 : (strcmp(e, "bulk") == 0 ? 2 : 0);

    // default tile: 8 x 16 cells, smaller when that would leave SMs idle (at least ~4 tiles per SM)
    while (h->C / ((int64_t)h->tile_w * h->tile_h) < 4 * 148 && h->tile_w * h->tile_h > 4) {
        if (h->tile_h > h->tile_w) h->tile_h /= 2;
        else h->tile_w /= 2;
    }
    TRY(dalloc(h, &h->d_rep, nrep));
    TRY(dalloc(h, &h->d_bch, bch.size()));
    TRY(dalloc(h, &h->d_cch, cch.size()));
    CK(cudaMemcpy(h->d_rep, h->rh.data(), nrep * sizeof(RepDev), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->d_bch, bch.data(), bch.size() * sizeof(Chunk), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->d_cch, cch.data(), cch.size() * sizeof(Chunk), cudaMemcpyHostToDevice));
    Bufs &b = h->b;
    const size_t N = (size_t)h->N, C = (size_t)h->C;
    for (int k = 0; k < 2; k++) {
        TRY(dalloc(h, &b.pos[k], N));
        TRY(dalloc(h, &b.vh[k], N));
        TRY(dalloc(h, &b.vt[k], N));
        TRY(dalloc(h, &b.f[k], N));
        TRY(dalloc(h, &b.tg[k], N));
        TRY(dalloc(h, &b.link[k], N));
    }
    TRY(dalloc(h, &b.key, N));
    TRY(dalloc(h, &b.fill, C + 4));
    TRY(dalloc(h, &b.src, N));
    TRY(dalloc(h, &b.dest, N));
    TRY(dalloc(h, &b.count, C + 4));
    TRY(dalloc(h, &b.cstart, C + 4));
    TRY(dalloc(h, &b.bsum, C / SCAN_PER_BLOCK + 2));
    TRY(dalloc(h, &b.scan_state, C / SCAN_PER_BLOCK + 2));
    TRY(dalloc(h, &b.scan_ticket, 1));
    CK(cudaMemset(b.scan_state, 0, (C / SCAN_PER_BLOCK + 2) * sizeof(unsigned long long)));
    CK(cudaMemset(b.scan_ticket, 0, sizeof(unsigned long long)));
    TRY(dalloc(h, &b.claim, N));
    TRY(dalloc(h, &b.req, N));
    TRY(dalloc(h, &b.grow_list, N));
    TRY(dalloc(h, &b.bond_list, N));
    b.evcap = 1 << 20;
    TRY(dalloc(h, &b.events, (size_t)b.evcap));
    TRY(dalloc(h, &b.status, 1));
    TRY(dalloc(h, &b.step, 1));
    TRY(dalloc(h, &b.obs, (size_t)nrep * OBS_N));
    TRY(dalloc(h, &b.obs_out, (size_t)nrep * OBS_N));
    TRY(dalloc(h, &b.obs_done, (size_t)nrep));
    TRY(dalloc(h, &b.hist, 4096));
    TRY(dalloc(h, &b.stir, (size_t)nrep));
    TRY(dalloc(h, &b.rng, (size_t)4 * nrep));
    TRY(dalloc(h, &b.cat_list, N));
    TRY(dalloc(h, &b.cat_cnt, (size_t)h->nbch + 1));
    TRY(dalloc(h, &b.cat_ncnt, (size_t)h->nbch + 1));
    TRY(dalloc(h, &b.resort, (size_t)nrep + 1));
    TRY(dalloc(h, &b.cat_nk, (size_t)nrep));
    TRY(dalloc(h, &b.cat_near, N));
    TRY(dalloc(h, &b.cat_cell, N));
    TRY(dalloc(h, &b.cat_mark, C));
    TRY(dalloc(h, &b.fmol, N));
    if (h->any_cat) {
        // the catalyst checks' draw streams: 3 n + 4096 draws per replica, 64-draw blocks
        long long so = 0;
        int nblk = 1;
        for (int r = 0; r < nrep; r++) {
            const int dcap = (int)((3ll * h->rh[r].n + 4096 + 63) / 64 * 64);
            h->rh[r].so = so;
            h->rh[r].dcap = dcap;
            so += dcap;
            nblk = std::max(nblk, dcap / 64);
        }
        CK(cudaMemcpy(h->d_rep, h->rh.data(), (size_t)nrep * sizeof(RepDev), cudaMemcpyHostToDevice));
        std::vector<uint64_t> jt;
        if (jump_table(nblk, jt) != 0) return fail(DPD_E_STATE, "xoshiro256** polynomial not found");
        uint64_t *dj = nullptr;
        TRY(dalloc(h, &dj, jt.size()));
        CK(cudaMemcpy(dj, jt.data(), jt.size() * sizeof(uint64_t), cudaMemcpyHostToDevice));
        b.jump = dj;
        TRY(dalloc(h, &b.stream, (size_t)so));
        TRY(dalloc(h, &b.sblock, (size_t)so / 16));
        TRY(dalloc(h, &b.cat_dn, (size_t)nrep));
        TRY(dalloc(h, &b.shuf, 8 * N));
        b.shuf_n = (long long)N;
        h->stream_grid = (nblk + 255) / 256;
    }
    {
        std::vector<dpd_template> mols(nrep);
        for (int r = 0; r < nrep; r++)
            if (dpd_lipid_template(&h->params[r], &mols[r]) != DPD_OK) std::memset(&mols[r], 0, sizeof(dpd_template));
        dpd_template *dm = nullptr;
        TRY(dalloc(h, &dm, (size_t)nrep));
        CK(cudaMemcpy(dm, mols.data(), (size_t)nrep * sizeof(dpd_template), cudaMemcpyHostToDevice));
        b.mol = dm;
    }
    CK(cudaMemset(b.resort, 0, ((size_t)nrep + 1) * sizeof(int32_t)));
    CK(cudaMemset(b.rng, 0, (size_t)4 * nrep * sizeof(uint64_t)));
    if (h->any_cat && catalyst_setup() != 0)
        return fail(DPD_E_CUDA, "cannot reserve shared memory for the catalyst kernel");
    CK(cudaMemset(b.stir, 0, (size_t)nrep * sizeof(long long)));
    // staging for set/get state: 8 float + 3 int32 + 1 byte arrays of nmax
    TRY(dalloc(h, &h->stage, (size_t)h->nmax * (8 * 4 + 3 * 4 + 1) + 16 * 256));
    CK(cudaMemset(b.count, 0, (C + 4) * sizeof(uint32_t)));
    CK(cudaMemset(b.claim, 0xFF, N * sizeof(uint32_t)));
    CK(cudaMemset(b.req, 0xFF, N * sizeof(int32_t)));
    CK(cudaMemset(b.status, 0, sizeof(DevStatus)));
    CK(cudaMemset(b.step, 0, sizeof(long long)));
    CK(cudaMemset(b.obs, 0, (size_t)nrep * OBS_N * sizeof(unsigned long long)));
    CK(cudaMemset(b.obs_done, 0, (size_t)nrep * sizeof(unsigned int)));
    for (int k = 0; k < 2; k++) {
        CK(cudaMemset(b.pos[k], 0, N * sizeof(float2)));
        CK(cudaMemset(b.vh[k], 0, N * sizeof(float2)));
        CK(cudaMemset(b.vt[k], 0, N * sizeof(float2)));
        CK(cudaMemset(b.f[k], 0, N * sizeof(float2)));
        CK(cudaMemset(b.tg[k], 0, N * sizeof(uint32_t)));
        CK(cudaMemset(b.link[k], 0xFF, N * sizeof(int2)));
    }
    // graph length: even (the buffers alternate every step), ~4M bead-steps per replay
    int g = (int)std::max<int64_t>(1, std::min<int64_t>(64, (4 << 20) / std::max<int64_t>(1, h->N)));
    if (const char *e = getenv("DPD_GRAPH_STEPS")) g = atoi(e);
    h->gsteps = graph_len(h, g);
    TRY(build_tiles(h));
    return DPD_OK;
}

extern "C" int dpd_create(const dpd_params *params, int32_t n_replicas, const int32_t *n_beads, dpd_handle **out) {
    if (!params || !n_beads || !out || n_replicas < 1) return fail(DPD_E_ARG, "bad arguments to dpd_create");
    *out = nullptr;
    dpd_handle *h = new dpd_handle();
    const int r = create_impl(h, params, n_replicas, n_beads);
    if (r != DPD_OK) {
        free_all(h);
        delete h;
        return r;
    }
    *out = h;
    return DPD_OK;
}

extern "C" int dpd_destroy(dpd_handle *h) {
    if (!h) return DPD_OK;
    cudaStreamSynchronize(h->s);
    free_all(h);
    delete h;
    return DPD_OK;
}

extern "C" int dpd_sizes(const dpd_handle *h, int32_t r, int64_t *n_total, int32_t *n_beads, int32_t *n_cells) {
    if (!h) return fail(DPD_E_ARG, "null handle");
    if (n_total) *n_total = h->N;
    if (r >= 0 && r < h->nrep) {
        if (n_beads) *n_beads = h->rh[r].n;
        if (n_cells) *n_cells = h->rh[r].ncell;
    } else if (n_beads || n_cells) {
        return fail(DPD_E_ARG, "replica %d out of range", r);
    }
    return DPD_OK;
}

// ---------------------------------------------------------------- status

static int check_status(dpd_handle *h) {
    DevStatus st;
    CK(cudaMemcpyAsync(&st, h->b.status, sizeof st, cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    if (st.flags) {
        CK(cudaMemsetAsync(&h->b.status->flags, 0, sizeof(unsigned), h->s));
        CK(cudaStreamSynchronize(h->s));
        if (st.flags & DPD_F_WAIT)
            return fail(DPD_E_TIMEOUT, "a bounded device wait gave up (bulk copies of the force kernel, or the scan)");
        if (st.flags & DPD_F_ANALYSIS) return fail(DPD_E_STATE, "cluster analysis did not converge");
        if (st.flags & DPD_F_CATALYST)
            return fail(DPD_E_STATE, "a catalyst's neighbourhood did not fit the staging area, or a search found "
                                     "more than 256 candidates or 512 relaxation neighbours (too crowded)");
        if (st.flags & DPD_F_TILE)
            return fail(DPD_E_SORT_OVERFLOW, "a cell tile and its halo held more beads than fit in shared memory");
        if (st.flags & DPD_F_FORCE) return fail(DPD_E_STATE, "a pair or bond force above 2048 (fixed-point range)");
        if (st.flags & DPD_F_NONFINITE) return fail(DPD_E_STATE, "non-finite force (flags 0x%x)", st.flags);
        if (st.flags & DPD_F_OUTSIDE)
            return fail(DPD_E_STATE, "a bead moved more than one box length in one step (flags 0x%x)", st.flags);
        if (st.flags & DPD_F_EVENTS)
            return fail(DPD_E_EVENT_OVERFLOW, "event buffer full (%u events since the last read)", st.nevents);
        if (st.flags & DPD_F_CHAIN) return fail(DPD_E_CHAIN, "broken lipid chain");
    }
    return DPD_OK;
}

static int ensure_replica(const dpd_handle *h, int r) {
    if (!h) return fail(DPD_E_ARG, "null handle");
    if (r < 0 || r >= h->nrep) return fail(DPD_E_ARG, "replica %d out of range (0..%d)", r, h->nrep - 1);
    return DPD_OK;
}

// ---------------------------------------------------------------- state in/out

extern "C" int dpd_set_state(dpd_handle *h, int32_t r, const float *x, const float *y, const float *vx,
                             const float *vy, const uint8_t *type, const uint32_t *gid, const int32_t *prev,
                             const int32_t *next) {
    TRY(ensure_replica(h, r));
    if (!x || !y || !vx || !vy || !type) return fail(DPD_E_ARG, "x, y, vx, vy and type are required");
    const RepDev &R = h->rh[r];
    const size_t n = (size_t)R.n, a = ((n * 4 + 255) / 256) * 256;
    char *p = h->stage;
    float *sx = (float *)p, *sy = (float *)(p + a), *svx = (float *)(p + 2 * a), *svy = (float *)(p + 3 * a);
    uint32_t *sg = (uint32_t *)(p + 4 * a);
    int32_t *sp = (int32_t *)(p + 5 * a), *sn = (int32_t *)(p + 6 * a);
    uint8_t *st = (uint8_t *)(p + 7 * a);
    CK(cudaMemcpyAsync(sx, x, n * 4, cudaMemcpyDefault, h->s));
    CK(cudaMemcpyAsync(sy, y, n * 4, cudaMemcpyDefault, h->s));
    CK(cudaMemcpyAsync(svx, vx, n * 4, cudaMemcpyDefault, h->s));
    CK(cudaMemcpyAsync(svy, vy, n * 4, cudaMemcpyDefault, h->s));
    CK(cudaMemcpyAsync(st, type, n, cudaMemcpyDefault, h->s));
    if (gid) CK(cudaMemcpyAsync(sg, gid, n * 4, cudaMemcpyDefault, h->s));
    if (prev) CK(cudaMemcpyAsync(sp, prev, n * 4, cudaMemcpyDefault, h->s));
    if (next) CK(cudaMemcpyAsync(sn, next, n * 4, cudaMemcpyDefault, h->s));
    launch_pack(h->b, h->cur, R.b0, (int)n, R.L, sx, sy, svx, svy, st, gid ? sg : nullptr, prev ? sp : nullptr,
                next ? sn : nullptr, h->s);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->s));
    h->keys_valid = false;
    unsigned flags = 0;
    CK(cudaMemcpy(&flags, &h->b.status->flags, sizeof flags, cudaMemcpyDeviceToHost));
    if (flags & DPD_F_INPUT) {
        flags &= ~DPD_F_INPUT;
        CK(cudaMemcpy(&h->b.status->flags, &flags, sizeof flags, cudaMemcpyHostToDevice));
        return fail(DPD_E_ARG, "set_state: a non-finite position, a type >= %d, a gid >= n or a link outside "
                               "[-1, n) (replica %d)", DPD_MAXT, r);
    }
    return DPD_OK;
}

extern "C" int dpd_get_state(dpd_handle *h, int32_t r, float *x, float *y, float *vhx, float *vhy, float *vtx,
                             float *vty, float *fx, float *fy, uint8_t *type, uint32_t *gid, int32_t *prev,
                             int32_t *next) {
    TRY(ensure_replica(h, r));
    const RepDev &R = h->rh[r];
    const size_t n = (size_t)R.n, a = ((n * 4 + 255) / 256) * 256;
    char *p = h->stage;
    float *f8[8];
    for (int k = 0; k < 8; k++) f8[k] = (float *)(p + k * a);
    uint32_t *sg = (uint32_t *)(p + 8 * a);
    int32_t *sp = (int32_t *)(p + 9 * a), *sn = (int32_t *)(p + 10 * a);
    uint8_t *st = (uint8_t *)(p + 11 * a);
    launch_unpack(h->b, h->cur, R.b0, (int)n, f8[0], f8[1], f8[2], f8[3], f8[4], f8[5], f8[6], f8[7], st, sg, sp,
                  sn, h->s);
    CK(cudaGetLastError());
    float *outs[8] = {x, y, vhx, vhy, vtx, vty, fx, fy};
    for (int k = 0; k < 8; k++)
        if (outs[k]) CK(cudaMemcpyAsync(outs[k], f8[k], n * 4, cudaMemcpyDefault, h->s));
    if (type) CK(cudaMemcpyAsync(type, st, n, cudaMemcpyDefault, h->s));
    if (gid) CK(cudaMemcpyAsync(gid, sg, n * 4, cudaMemcpyDefault, h->s));
    if (prev) CK(cudaMemcpyAsync(prev, sp, n * 4, cudaMemcpyDefault, h->s));
    if (next) CK(cudaMemcpyAsync(next, sn, n * 4, cudaMemcpyDefault, h->s));
    CK(cudaStreamSynchronize(h->s));
    return DPD_OK;
}

extern "C" int dpd_set_dynamics(dpd_handle *h, int32_t r, const float *vhx, const float *vhy, const float *fx,
                                const float *fy, const float *vtx, const float *vty) {
    TRY(ensure_replica(h, r));
    const RepDev &R = h->rh[r];
    const size_t n = (size_t)R.n, a = ((n * 4 + 255) / 256) * 256;
    const float *in[6] = {vhx, vhy, fx, fy, vtx, vty};
    float *sg[6];
    for (int k = 0; k < 6; k++) {
        sg[k] = (float *)(h->stage + k * a);
        if (in[k]) CK(cudaMemcpyAsync(sg[k], in[k], n * 4, cudaMemcpyDefault, h->s));
    }
    launch_set_dynamics(h->b, h->cur, R.b0, (int)n, vhx ? sg[0] : nullptr, vhy ? sg[1] : nullptr,
                        fx ? sg[2] : nullptr, fy ? sg[3] : nullptr, vtx ? sg[4] : nullptr, vty ? sg[5] : nullptr,
                        h->s);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->s));
    h->keys_valid = false;
    return DPD_OK;
}

// ---------------------------------------------------------------- phases

// the stirring sums are accumulated by the permute kernel and read by the forces
static void clear_stir(dpd_handle *h) {
    if (h->any_stir) cudaMemsetAsync(h->b.stir, 0, (size_t)h->nrep * sizeof(long long), h->s);
}

static void enqueue_sort(dpd_handle *h, PermuteMode mode) {
    // counts of the CURRENT positions
    cudaMemsetAsync(h->b.count, 0, (size_t)(h->C + 4) * sizeof(uint32_t), h->s);
    launch_keys(h->b, h->cur, h->d_rep, h->d_bch, h->nbch, false, h->s);
    enqueue_cell_sort(h, false);
    clear_stir(h);
    launch_permute(h->b, h->cur, h->d_rep, h->d_bch, h->nbch, mode, h->s);
    h->cur ^= 1;
}

static int set_device_step(dpd_handle *h, int64_t step) {
    long long v = (long long)step;
    CK(cudaMemcpyAsync(h->b.step, &v, sizeof v, cudaMemcpyHostToDevice, h->s));
    CK(cudaStreamSynchronize(h->s));
    h->step = step;
    return DPD_OK;
}

static void enqueue_next_keys(dpd_handle *h) {
    cudaMemsetAsync(h->b.count, 0, (size_t)(h->C + 4) * sizeof(uint32_t), h->s);
    launch_keys(h->b, h->cur, h->d_rep, h->d_bch, h->nbch, true, h->s);
    h->keys_valid = true;
}

extern "C" int dpd_prime(dpd_handle *h) {
    if (!h) return fail(DPD_E_ARG, "null handle");
    enqueue_sort(h, PERM_PRIME);
    enqueue_forces(h, false);
    launch_halfkick(h->b, h->cur, h->d_rep, h->d_bch, h->nbch, h->s);
    enqueue_next_keys(h);
    CK(cudaGetLastError());
    return check_status(h);
}

extern "C" int dpd_resume(dpd_handle *h) {
    if (!h) return fail(DPD_E_ARG, "null handle");
    enqueue_sort(h, PERM_SORT);
    enqueue_next_keys(h);
    CK(cudaGetLastError());
    return check_status(h);
}

extern "C" int dpd_get_step(const dpd_handle *h, int64_t *step) {
    if (!h || !step) return fail(DPD_E_ARG, "null argument");
    *step = h->step;
    return DPD_OK;
}

extern "C" int dpd_set_step(dpd_handle *h, int64_t step) {
    if (!h) return fail(DPD_E_ARG, "null handle");
    return set_device_step(h, step);
}

extern "C" int dpd_build_cells(dpd_handle *h) {
    if (!h) return fail(DPD_E_ARG, "null handle");
    enqueue_sort(h, PERM_SORT);
    h->keys_valid = false;
    CK(cudaGetLastError());
    return check_status(h);
}

extern "C" int dpd_get_cells(dpd_handle *h, int32_t r, int32_t *cstart) {
    TRY(ensure_replica(h, r));
    if (!cstart) return fail(DPD_E_ARG, "null cstart");
    const RepDev &R = h->rh[r];
    std::vector<int32_t> tmp(R.ncell + 1);
    CK(cudaMemcpyAsync(tmp.data(), h->b.cstart + R.c0, (R.ncell + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost,
                       h->s));
    CK(cudaStreamSynchronize(h->s));
    for (auto &v : tmp) v -= R.b0;
    CK(cudaMemcpy(cstart, tmp.data(), tmp.size() * sizeof(int32_t), cudaMemcpyDefault));
    return DPD_OK;
}

extern "C" int dpd_forces(dpd_handle *h, int64_t step) {
    if (!h) return fail(DPD_E_ARG, "null handle");
    TRY(set_device_step(h, step));
    enqueue_forces(h, false);
    h->keys_valid = false;
    CK(cudaGetLastError());
    return check_status(h);
}

static int partial_forces(dpd_handle *h, int32_t r, bool pair, bool bond, float *fx, float *fy) {
    // computed into the spare force buffer so the stored forces stay untouched
    Bufs b = h->b;
    b.f[h->cur] = h->b.f[h->cur ^ 1];
    if (bond && h->any_mol) launch_mol_forces(b, h->cur, h->d_rep, h->d_bch, h->nbch, h->s);
    launch_forces(b, h->cur, h->d_rep, h->d_bch, h->nbch, pair, bond, false, h->s);
    CK(cudaGetLastError());
    const RepDev &R = h->rh[r];
    const size_t n = (size_t)R.n, a = ((n * 4 + 255) / 256) * 256;
    float *sx = (float *)h->stage, *sy = (float *)(h->stage + a);
    Bufs u = h->b;
    u.f[h->cur] = b.f[h->cur];
    launch_unpack(u, h->cur, R.b0, (int)n, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, sx, sy, nullptr,
                  nullptr, nullptr, nullptr, h->s);
    CK(cudaGetLastError());
    if (fx) CK(cudaMemcpyAsync(fx, sx, n * 4, cudaMemcpyDefault, h->s));
    if (fy) CK(cudaMemcpyAsync(fy, sy, n * 4, cudaMemcpyDefault, h->s));
    CK(cudaStreamSynchronize(h->s));
    return check_status(h);
}

extern "C" int dpd_pair_forces(dpd_handle *h, int32_t r, int64_t step, float *fx, float *fy) {
    TRY(ensure_replica(h, r));
    TRY(set_device_step(h, step));
    return partial_forces(h, r, true, false, fx, fy);
}

extern "C" int dpd_bond_forces(dpd_handle *h, int32_t r, float *fx, float *fy, float *maxbond) {
    TRY(ensure_replica(h, r));
    unsigned long long *slot = h->b.obs + (size_t)r * OBS_N + 4;
    CK(cudaMemsetAsync(slot, 0, sizeof(unsigned long long), h->s));
    TRY(partial_forces(h, r, false, true, fx, fy));
    if (maxbond) {
        unsigned long long v = 0;
        CK(cudaMemcpy(&v, slot, sizeof v, cudaMemcpyDeviceToHost));
        uint32_t bits = (uint32_t)v;
        memcpy(maxbond, &bits, 4);
    }
    return DPD_OK;
}

extern "C" int dpd_integrate(dpd_handle *h) {
    if (!h) return fail(DPD_E_ARG, "null handle");
    launch_integrate(h->b, h->cur, h->d_rep, h->d_bch, h->nbch, h->s);
    h->keys_valid = false;
    CK(cudaGetLastError());
    return check_status(h);
}

extern "C" int dpd_chemistry(dpd_handle *h, int64_t step) {
    if (!h) return fail(DPD_E_ARG, "null handle");
    TRY(set_device_step(h, step));
    CK(cudaMemsetAsync(&h->b.status->n_grow, 0, 2 * sizeof(unsigned), h->s));
    launch_chem_scan(h->b, h->cur, h->d_rep, h->d_bch, h->nbch, h->s);
    launch_chem_lists(h->b, h->cur, h->d_rep, -1, h->s);
    // the catalyst chemistry as the reference's chemistry(): no sort afterwards
    if (h->any_cat) launch_catalyst(h->b, h->cur, h->d_rep, h->d_bch, h->nbch, h->nrep, h->C, h->nmax, h->stream_grid, h->s);
    CK(cudaGetLastError());
    return check_status(h);
}

// ---------------------------------------------------------------- the step

// does a catalyst check of some replica fall on step s
static bool cat_at(const dpd_handle *h, int64_t s) {
    if (!h->any_cat) return false;
    for (const auto &p : h->params)
        if (p.chem && p.chem_kind == 1 && p.n_chem > 0 && s % p.n_chem == 0) return true;
    return false;
}

// one step producing step number s.  A step with a catalyst check follows the
// reference's order (oercel.c:2337-2349): the update with every bead kept in
// the slot of the last sort, the check on that order and cell index (the
// catalysts and the food candidates are taken in slot order), then the sort of
// the new configuration.  A replica in which a bead moved 0.5 or more is
// sorted before its check too (launch_resort, no-ops otherwise).  Other steps
// fuse the update into the sort whose counts the previous force kernel made.
static void enqueue_step(dpd_handle *h, int64_t s) {
    const bool cat = cat_at(h, s);
    if (!cat) {
        enqueue_cell_sort(h, true);
    } else {
        launch_step_begin(h->b, h->nrep, h->s);
    }
    clear_stir(h);
    launch_permute(h->b, h->cur, h->d_rep, h->d_bch, h->nbch, cat ? PERM_KEEP : PERM_STEP, h->s);
    h->cur ^= 1;
    if (h->any_lipid) launch_chem_lists(h->b, h->cur, h->d_rep, -1, h->s);
    if (cat) {
        launch_resort(h->b, h->cur, h->d_rep, h->d_bch, h->nbch, h->d_cch, h->ncch, h->C, h->s);
        launch_catalyst(h->b, h->cur, h->d_rep, h->d_bch, h->nbch, h->nrep, h->C, h->nmax, h->stream_grid, h->s);
        enqueue_sort(h, PERM_SORT);
    }
    // the step's stats row into the ring: assembled by the tile force kernel's
    // epilogue from the beads it holds anyway, else by a pass of its own
    if (h->ring && h->force_kernel == 0) {
        enqueue_forces(h, true, RowOut{h->ring_rep, h->ring_slots, h->ring});
    } else {
        enqueue_forces(h, true);
        if (h->ring)
            launch_observables(h->b, h->cur, h->d_rep, h->d_bch, h->nbch, h->ring_rep, false, h->ring, h->ring_slots,
                               h->s);
    }
}

// capture gsteps steps starting from the current buffer parity and step s0
// (with catalyst chemistry s0 is a multiple of its period: the graph then
// holds the checks at the same places on every replay)
static int build_graph(dpd_handle *h, int64_t s0) {
    const int cur0 = h->cur;
    if (h->gexec[cur0]) {
        CK(cudaGraphExecDestroy(h->gexec[cur0]));
        h->gexec[cur0] = nullptr;
    }
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(h->s, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < h->gsteps; k++) enqueue_step(h, s0 + 1 + k);
    const cudaError_t e = cudaStreamEndCapture(h->s, &g);
    h->gflip[cur0] = h->cur ^ cur0;
    h->cur = cur0;  // capture only recorded the launches
    if (e != cudaSuccess) return fail(DPD_E_CUDA, "graph capture: %s", cudaGetErrorString(e));
    const cudaError_t e2 = cudaGraphInstantiate(&h->gexec[cur0], g, 0);
    cudaGraphDestroy(g);
    if (e2 != cudaSuccess) return fail(DPD_E_CUDA, "graph instantiate: %s", cudaGetErrorString(e2));
    return DPD_OK;
}

// enqueue nsteps steps: whole graphs while they fit, eager launches for the rest
static int enqueue_steps(dpd_handle *h, int64_t nsteps) {
    if (nsteps < 0) return fail(DPD_E_ARG, "nsteps must be >= 0");
    if (nsteps == 0) return DPD_OK;
    if (!h->keys_valid) enqueue_next_keys(h);
    int64_t left = nsteps, s = h->step;
    const int64_t P = h->cat_period;
    const bool graphs = getenv("DPD_NO_GRAPH") == nullptr && (P == 0 || h->gsteps % P == 0);
    while (left > 0) {
        if (graphs && left >= h->gsteps && (P == 0 || s % P == 0)) {
            if (!h->gexec[h->cur]) TRY(build_graph(h, s));
            CK(cudaGraphLaunch(h->gexec[h->cur], h->s));
            h->cur ^= h->gflip[h->cur];
            left -= h->gsteps;
            s += h->gsteps;
        } else {
            enqueue_step(h, s + 1);
            left--;
            s++;
        }
    }
    CK(cudaGetLastError());
    h->step += nsteps;
    return DPD_OK;
}

extern "C" int dpd_step(dpd_handle *h, int64_t nsteps) {
    if (!h) return fail(DPD_E_ARG, "null handle");
    TRY(enqueue_steps(h, nsteps));
    return check_status(h);
}

extern "C" int dpd_step_async(dpd_handle *h, int64_t nsteps) {
    if (!h) return fail(DPD_E_ARG, "null handle");
    return enqueue_steps(h, nsteps);
}

extern "C" int dpd_sync(dpd_handle *h) {
    if (!h) return fail(DPD_E_ARG, "null handle");
    return check_status(h);
}

extern "C" int dpd_set_tuning(dpd_handle *h, const dpd_tuning *t) {
    if (!h || !t) return fail(DPD_E_ARG, "null argument");
    if (t->force_kernel < 0 || t->force_kernel > 2) return fail(DPD_E_ARG, "force_kernel must be 0, 1 or 2");
    if (t->force_kernel == 2 && t->tile_w + 2 > 32)
        return fail(DPD_E_ARG, "the bulk-staged force kernel takes tiles of at most 30 columns");
    if (t->graph_steps < 1) return fail(DPD_E_ARG, "graph_steps must be >= 1");
    if (t->sort_mode < 0 || t->sort_mode > 2) return fail(DPD_E_ARG, "sort_mode must be 0, 1 or 2");
    if (t->tile_threads != 256 && t->tile_threads != 512) return fail(DPD_E_ARG, "tile_threads must be 256 or 512");
    CK(cudaStreamSynchronize(h->s));
    const int ow = h->tile_w, oh = h->tile_h, ofk = h->force_kernel, ott = h->tile_threads;
    h->tile_w = t->tile_w;
    h->tile_h = t->tile_h;
    h->force_kernel = t->force_kernel;
    h->tile_threads = t->tile_threads;
    const int r = build_tiles(h);
    if (r != DPD_OK) {
        h->tile_w = ow;
        h->tile_h = oh;
        h->force_kernel = ofk;
        h->tile_threads = ott;
        build_tiles(h);
        return r;
    }
    h->sort_mode = t->sort_mode;
    h->gsteps = graph_len(h, t->graph_steps);
    drop_graphs(h);
    return DPD_OK;
}

extern "C" int dpd_get_tuning(const dpd_handle *h, dpd_tuning *t) {
    if (!h || !t) return fail(DPD_E_ARG, "null argument");
    t->force_kernel = h->force_kernel;
    t->tile_w = h->tile_w;
    t->tile_h = h->tile_h;
    t->graph_steps = h->gsteps;
    t->sort_mode = h->sort_mode;
    t->tile_threads = h->tile_threads;
    return DPD_OK;
}

extern "C" int dpd_set_graph_steps(dpd_handle *h, int32_t steps) {
    if (!h || steps < 1) return fail(DPD_E_ARG, "graph length must be >= 1");
    CK(cudaStreamSynchronize(h->s));
    drop_graphs(h);
    h->gsteps = graph_len(h, steps);
    return DPD_OK;
}

// One step launched kernel by kernel with CUDA events between the launches on
// the handle's stream; ms[k] = device time of kernel k (scan1 (the whole scan
// with sort_mode 1, the block-local scan with 2), scan2 (0 ms with sort_mode 1
// and 2), place, cellfix, permute, [2 chemistry], [catalyst check + its sort], forces).  The
// step is a real step; on a step with a catalyst check the first entry is the
// step counter's kernel, the next three are not launched (0 ms) and the
// permute keeps the slot order.
extern "C" int dpd_profile_step(dpd_handle *h, float *ms, int32_t cap, int32_t *n_out) {
    if (!h || !ms || !n_out) return fail(DPD_E_ARG, "null argument");
    if (!h->keys_valid) enqueue_next_keys(h);
    const bool cat = cat_at(h, h->step + 1);
    const int nk = 6 + (h->any_lipid ? chem_kernel_count() : 0) + (cat ? 1 : 0);
    if (cap < nk) return fail(DPD_E_ARG, "need room for %d kernel times", nk);
    std::vector<cudaEvent_t> ev(nk + 1);
    for (auto &e : ev) CK(cudaEventCreate(&e));
    int k = 0;
    CK(cudaEventRecord(ev[k++], h->s));
    const bool pfx = h->sort_mode == 2 && sort_pfx_fits(h->C);
    if (!cat) {
        if (pfx) launch_sort_pfx(h->b, h->C, true, h->d_bch, h->nbch, h->d_cch, h->ncch, 0, h->s);
        else if (h->sort_mode == 1) launch_scan_lb(h->b, h->C, true, h->s);
        else launch_scan_part(h->b, h->C, true, 1, h->s);
    } else {
        launch_step_begin(h->b, h->nrep, h->s);
    }
    CK(cudaEventRecord(ev[k++], h->s));
    if (!cat && h->sort_mode == 0) launch_scan_part(h->b, h->C, true, 2, h->s);
    CK(cudaEventRecord(ev[k++], h->s));
    if (!cat) {
        if (pfx) launch_sort_pfx(h->b, h->C, true, h->d_bch, h->nbch, h->d_cch, h->ncch, 1, h->s);
        else launch_place(h->b, h->d_bch, h->nbch, h->s);
    }
    CK(cudaEventRecord(ev[k++], h->s));
    if (!cat) {
        if (pfx) launch_sort_pfx(h->b, h->C, true, h->d_bch, h->nbch, h->d_cch, h->ncch, 2, h->s);
        else launch_cellfix(h->b, h->d_cch, h->ncch, h->s);
    }
    CK(cudaEventRecord(ev[k++], h->s));
    clear_stir(h);
    launch_permute(h->b, h->cur, h->d_rep, h->d_bch, h->nbch, cat ? PERM_KEEP : PERM_STEP, h->s);
    CK(cudaEventRecord(ev[k++], h->s));
    h->cur ^= 1;
    if (h->any_lipid)
        for (int c = 0; c < chem_kernel_count(); c++) {
            launch_chem_lists(h->b, h->cur, h->d_rep, c, h->s);
            CK(cudaEventRecord(ev[k++], h->s));
        }
    if (cat) {
        launch_resort(h->b, h->cur, h->d_rep, h->d_bch, h->nbch, h->d_cch, h->ncch, h->C, h->s);
        launch_catalyst(h->b, h->cur, h->d_rep, h->d_bch, h->nbch, h->nrep, h->C, h->nmax, h->stream_grid, h->s);
        enqueue_sort(h, PERM_SORT);
        CK(cudaEventRecord(ev[k++], h->s));
    }
    enqueue_forces(h, true);
    CK(cudaEventRecord(ev[k++], h->s));
    CK(cudaGetLastError());
    CK(cudaEventSynchronize(ev[nk]));
    for (int q = 0; q < nk; q++) CK(cudaEventElapsedTime(&ms[q], ev[q], ev[q + 1]));
    for (auto &e : ev) cudaEventDestroy(e);
    h->step += 1;
    *n_out = nk;
    return check_status(h);
}

extern "C" int dpd_type_clusters(dpd_handle *h, int32_t r, int32_t type, double rcut, int64_t *out) {
    TRY(ensure_replica(h, r));
    if (!out) return fail(DPD_E_ARG, "null output");
    if (type < 0 || type >= DPD_MAXT) return fail(DPD_E_ARG, "type must be 0..%d", DPD_MAXT - 1);
    if (!(rcut > 0.0 && rcut <= 1.0)) return fail(DPD_E_ARG, "rcut must be in (0, 1]");
    if (!h->ana_parent) {
        TRY(dalloc(h, &h->ana_parent, (size_t)h->N));
        TRY(dalloc(h, &h->ana_size, (size_t)h->N));
        TRY(dalloc(h, &h->ana_acc, 8));
    }
    launch_type_clusters(h->b, h->cur, h->d_rep, h->d_bch, h->nbch, r, type, rcut, h->ana_parent, h->ana_size,
                         h->ana_acc, h->s);
    CK(cudaGetLastError());
    unsigned long long acc[8];
    CK(cudaMemcpyAsync(acc, h->ana_acc, sizeof acc, cudaMemcpyDeviceToHost, h->s));
    TRY(check_status(h));
    out[0] = (int64_t)acc[4];  // beads of the type (the sum of the cluster sizes)
    out[1] = (int64_t)acc[2];  // clusters
    out[2] = (int64_t)acc[5];  // largest cluster
    out[3] = (int64_t)acc[3];  // sum of squared cluster sizes
    out[4] = (int64_t)acc[0];  // neighbours within 1 of the type's beads, all types
    out[5] = (int64_t)acc[1];  // the same, of the type
    return DPD_OK;
}

extern "C" int dpd_aggregates(dpd_handle *h, int32_t r, double r_tail, int32_t min_lipids, int64_t *out,
                              int32_t *agg_of_gid) {
    TRY(ensure_replica(h, r));
    if (!out) return fail(DPD_E_ARG, "null output");
    if (!(r_tail > 0.0 && r_tail <= 1.0)) return fail(DPD_E_ARG, "r_tail must be in (0, 1]");
    if (!h->ana_parent) {
        TRY(dalloc(h, &h->ana_parent, (size_t)h->N));
        TRY(dalloc(h, &h->ana_size, (size_t)h->N));
        TRY(dalloc(h, &h->ana_acc, 8));
    }
    if (!h->ana_min) {
        TRY(dalloc(h, &h->ana_min, (size_t)h->N));
        TRY(dalloc(h, &h->ana_label, (size_t)h->nmax));
    }
    const RepDev &R = h->rh[r];
    launch_aggregates(h->b, h->cur, h->d_rep, h->d_bch, h->nbch, r, R.n, r_tail, min_lipids, h->ana_parent,
                      h->ana_size, h->ana_min, h->ana_acc, agg_of_gid ? h->ana_label : nullptr, h->s);
    CK(cudaGetLastError());
    unsigned long long acc[8];
    CK(cudaMemcpyAsync(acc, h->ana_acc, sizeof acc, cudaMemcpyDeviceToHost, h->s));
    if (agg_of_gid) CK(cudaMemcpyAsync(agg_of_gid, h->ana_label, (size_t)R.n * sizeof(int32_t), cudaMemcpyDefault, h->s));
    TRY(check_status(h));
    out[0] = (int64_t)acc[4];  // molecules
    out[1] = (int64_t)acc[2];  // aggregates
    out[2] = (int64_t)acc[3];  // membranes (aggregates of >= min_lipids molecules)
    out[3] = (int64_t)acc[6];  // molecules in smaller aggregates
    out[4] = (int64_t)acc[5];  // the largest aggregate (molecules)
    return DPD_OK;
}

extern "C" int dpd_get_events(dpd_handle *h, dpd_event *out, int32_t cap, int32_t *n_out) {
    if (!h || !n_out) return fail(DPD_E_ARG, "null argument");
    DevStatus st;
    CK(cudaMemcpyAsync(&st, h->b.status, sizeof st, cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    const int have = (int)std::min<unsigned>(st.nevents, (unsigned)h->b.evcap);
    if (!out) {  // count only, nothing is cleared
        *n_out = have;
        return DPD_OK;
    }
    const int n = std::min(have, cap < 0 ? 0 : cap);
    if (n > 0) CK(cudaMemcpy(out, h->b.events, (size_t)n * sizeof(dpd_event), cudaMemcpyDefault));
    *n_out = n;
    CK(cudaMemset(&h->b.status->nevents, 0, sizeof(unsigned)));
    if (st.nevents > (unsigned)h->b.evcap)
        return fail(DPD_E_EVENT_OVERFLOW, "%u events were recorded, %d kept", st.nevents, h->b.evcap);
    if (have > n) return fail(DPD_E_EVENT_OVERFLOW, "%d events pending, %d copied: the rest were dropped", have, n);
    return DPD_OK;
}

// host memory the device can write through the same address (pinned, mapped)
static bool device_writable_host(const void *p) {
    cudaPointerAttributes pa;
    const bool ok = cudaPointerGetAttributes(&pa, p) == cudaSuccess && pa.type == cudaMemoryTypeHost &&
                    pa.devicePointer == p;
    cudaGetLastError();
    return ok;
}

extern "C" int dpd_events_async(dpd_handle *h, dpd_event *out, int32_t cap, int32_t *n_out) {
    if (!h || !out || !n_out) return fail(DPD_E_ARG, "null argument");
    if (cap < 1) return fail(DPD_E_ARG, "the event buffer needs room for at least one event");
    static_assert(sizeof(dpd_event) == sizeof(EventDev), "dpd_event and the device log agree");
    if (!device_writable_host(out) || !device_writable_host(n_out))
        return fail(DPD_E_ARG, "the event buffer and its count must be pinned host memory the device can write "
                               "(cudaHostAlloc, cudaHostRegister)");
    launch_events_out(h->b, (EventDev *)out, cap, (int *)n_out, h->s);
    CK(cudaGetLastError());
    return DPD_OK;
}

// the sums of a stats row on the stream, copied into v (OBS_N words) when the
// stream gets there: one kernel, whose last block hands the row over to obs_out
// and clears the running sums (the max bond restarts per stats row), and one copy
static int enqueue_observables(dpd_handle *h, int32_t r, bool virial, unsigned long long *v) {
    // pinned host memory the device can reach: the kernel writes the row there itself
    unsigned long long *direct = nullptr;
    cudaPointerAttributes pa;
    if (cudaPointerGetAttributes(&pa, v) == cudaSuccess && pa.type == cudaMemoryTypeHost &&
        pa.devicePointer == (void *)v)
        direct = v;
    cudaGetLastError();
    launch_observables(h->b, h->cur, h->d_rep, h->d_bch, h->nbch, r, virial, direct, 0, h->s);
    CK(cudaGetLastError());
    if (!direct)
        CK(cudaMemcpyAsync(v, h->b.obs_out + (size_t)r * OBS_N, OBS_N * sizeof(unsigned long long),
                           cudaMemcpyDeviceToHost, h->s));
    return DPD_OK;
}

static void decode_observables(const RepDev &R, const unsigned long long *v, double *out) {
    for (int k = 0; k < 16; k++) out[k] = 0.0;
    out[0] = (double)(long long)v[2] / OBS_FIX / (2.0 * R.n - 2.0);
    out[1] = (double)(long long)v[0] / OBS_FIX;
    out[2] = (double)(long long)v[1] / OBS_FIX;
    out[3] = (double)(long long)v[3] / OBS_FIX / ((double)R.L * (double)R.L);
    uint32_t bits = (uint32_t)v[4];
    float mb;
    memcpy(&mb, &bits, 4);
    out[4] = mb;
    out[5] = (double)v[5];
    for (int t = 0; t < 8; t++) out[8 + t] = (double)v[8 + t];
}

static int observables_impl(dpd_handle *h, int32_t r, bool virial, double *out) {
    TRY(ensure_replica(h, r));
    if (!out) return fail(DPD_E_ARG, "null out");
    unsigned long long v[OBS_N];
    TRY(enqueue_observables(h, r, virial, v));
    CK(cudaStreamSynchronize(h->s));
    decode_observables(h->rh[r], v, out);
    return DPD_OK;
}

extern "C" int dpd_stats_async(dpd_handle *h, int32_t r, uint64_t *raw) {
    TRY(ensure_replica(h, r));
    if (!raw) return fail(DPD_E_ARG, "null raw buffer");
    return enqueue_observables(h, r, false, (unsigned long long *)raw);
}

extern "C" int dpd_stats_ring(dpd_handle *h, int32_t r, uint64_t *ring, int32_t nslots) {
    TRY(ensure_replica(h, r));
    if (ring) {
        if (nslots < 1) return fail(DPD_E_ARG, "the ring needs at least one slot");
        cudaPointerAttributes pa;
        const bool ok = cudaPointerGetAttributes(&pa, ring) == cudaSuccess && pa.type == cudaMemoryTypeHost &&
                        pa.devicePointer == (void *)ring;
        cudaGetLastError();
        if (!ok) return fail(DPD_E_ARG, "the stats ring must be pinned host memory the device can write "
                                        "(cudaHostAlloc, cudaHostRegister)");
    }
    CK(cudaStreamSynchronize(h->s));
    h->ring = (unsigned long long *)ring;
    h->ring_rep = ring ? r : 0;
    h->ring_slots = ring ? nslots : 0;
    drop_graphs(h);  // the step graphs are captured again with (or without) the row
    return DPD_OK;
}

extern "C" int dpd_stats_decode(const dpd_handle *h, int32_t r, const uint64_t *raw, double *out) {
    if (!h || !raw || !out) return fail(DPD_E_ARG, "null argument");
    if (r < 0 || r >= h->nrep) return fail(DPD_E_ARG, "replica %d out of range", r);
    decode_observables(h->rh[r], (const unsigned long long *)raw, out);
    return DPD_OK;
}

extern "C" int dpd_observables(dpd_handle *h, int32_t r, double *out) { return observables_impl(h, r, true, out); }

extern "C" int dpd_stats(dpd_handle *h, int32_t r, double *out) { return observables_impl(h, r, false, out); }

extern "C" int dpd_pair_hist(dpd_handle *h, int32_t r, int32_t ta, int32_t tb, double rmax, int32_t nbin,
                             double *hist) {
    TRY(ensure_replica(h, r));
    if (!hist || nbin < 1 || nbin > 4096 || !(rmax > 0.0 && rmax <= 3.0))
        return fail(DPD_E_ARG, "need 1 <= nbin <= 4096 and 0 < rmax <= 3");
    CK(cudaMemsetAsync(h->b.hist, 0, nbin * sizeof(unsigned long long), h->s));
    launch_pair_hist(h->b, h->cur, h->d_rep, h->d_bch, h->nbch, r, ta, tb, rmax, nbin, h->s);
    CK(cudaGetLastError());
    std::vector<unsigned long long> v(nbin);
    CK(cudaMemcpyAsync(v.data(), h->b.hist, nbin * sizeof(unsigned long long), cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    for (int k = 0; k < nbin; k++) hist[k] = (double)v[k];
    return DPD_OK;
}

extern "C" int dpd_get_stream(const dpd_handle *h, void **stream) {
    if (!h || !stream) return fail(DPD_E_ARG, "null argument");
    *stream = (void *)h->s;
    return DPD_OK;
}

extern "C" int dpd_set_rng(dpd_handle *h, int32_t r, const uint64_t *state) {
    TRY(ensure_replica(h, r));
    if (!state) return fail(DPD_E_ARG, "null state");
    CK(cudaMemcpyAsync(h->b.rng + 4 * r, state, 4 * sizeof(uint64_t), cudaMemcpyDefault, h->s));
    CK(cudaStreamSynchronize(h->s));
    return DPD_OK;
}

extern "C" int dpd_get_rng(dpd_handle *h, int32_t r, uint64_t *state) {
    TRY(ensure_replica(h, r));
    if (!state) return fail(DPD_E_ARG, "null state");
    CK(cudaMemcpyAsync(state, h->b.rng + 4 * r, 4 * sizeof(uint64_t), cudaMemcpyDefault, h->s));
    CK(cudaStreamSynchronize(h->s));
    return DPD_OK;
}

extern "C" int dpd_kernels_per_step(const dpd_handle *h, int32_t *n_plain, int32_t *n_chem) {
    if (!h) return fail(DPD_E_ARG, "null handle");
    // scan1, scan2, place, cellfix, permute, forces (+ the chemistry kernels)
    if (n_plain) *n_plain = 6 + (h->any_lipid ? chem_kernel_count() : 0);
    if (n_chem) *n_chem = chem_kernel_count();
    return DPD_OK;
}

// ---------------------------------------------------------------- parameters in place

extern "C" int dpd_set_params(dpd_handle *h, int32_t r, const dpd_params *p) {
    TRY(ensure_replica(h, r));
    if (!p) return fail(DPD_E_ARG, "null params");
    RepDev R;
    const RepDev &old = h->rh[r];
    TRY(make_rep(*p, old.b0, old.n, old.c0, R));
    if (R.ncx != old.ncx || R.L != old.L) return fail(DPD_E_ARG, "dpd_set_params cannot change the box size");
    R.ch0 = old.ch0;
    R.nch = old.nch;
    R.so = old.so;
    R.dcap = old.dcap;
    if ((p->chem && p->chem_kind == 1) != (h->params[r].chem && h->params[r].chem_kind == 1) && !h->any_cat)
        return fail(DPD_E_ARG, "dpd_set_params cannot switch the catalyst chemistry on: create the handle with it");
    if (p->lip_arch != 0 && !h->any_mol)
        return fail(DPD_E_ARG, "dpd_set_params cannot switch to branched lipids: create the handle with them");
    CK(cudaStreamSynchronize(h->s));
    h->rh[r] = R;
    h->params[r] = *p;
    CK(cudaMemcpy(h->d_rep + r, &R, sizeof R, cudaMemcpyHostToDevice));
    {
        dpd_template M;
        if (dpd_lipid_template(p, &M) != DPD_OK) std::memset(&M, 0, sizeof M);
        CK(cudaMemcpy((dpd_template *)h->b.mol + r, &M, sizeof M, cudaMemcpyHostToDevice));
    }
    bool any = false;
    h->any_lipid = false;
    h->cat_period = 0;
    for (auto &q : h->params) {
        any = any || q.chem;
        h->any_lipid = h->any_lipid || (q.chem && q.chem_kind == 0);
        if (q.chem && q.chem_kind == 1) {
            const int64_t a = h->cat_period ? h->cat_period : 1, c = q.n_chem;
            h->cat_period = a / std::gcd(a, c) * c;
        }
    }
    h->gsteps = graph_len(h, h->gsteps);
    drop_graphs(h);
    bool stir = false;
    for (auto &q : h->params) stir = stir || q.stir_A != 0.0;
    if (stir && !h->any_stir) {
        // the current sums were not kept: rebuild them with a sort in place
        h->any_stir = true;
        drop_graphs(h);
        enqueue_sort(h, PERM_SORT);
        h->keys_valid = false;
    }
    h->any_stir = stir;
    if (any != h->any_chem) {
        h->any_chem = any;
        drop_graphs(h);
    }
    return DPD_OK;
}

// ---------------------------------------------------------------- reverse mode


template <typename T>
static int adj_alloc(dpd_handle *h, T **p, size_t count) {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, count * sizeof(T) + 64);
    if (e != cudaSuccess) return fail(DPD_E_NOMEM, "cudaMalloc for the adjoint: %s", cudaGetErrorString(e));
    h->adj_allocs.push_back(q);
    *p = (T *)q;
    return DPD_OK;
}

static int adj_setup(dpd_handle *h, int nck, int nseg, int nbin, AdjBufs &A) {
    // storage kept on the handle and grown on demand: a window that fits reuses
    // the buffers of the last one (freeing and allocating them every call costs a
    // device synchronisation per buffer)
    const int want_ck = nck, want_seg = nseg;
    if (h->adj_nbin > 0 && nck <= h->adj_nck && nseg <= h->adj_nseg && nbin <= h->adj_nbin) {
        A = h->adj;
        A.ck.resize(want_ck);
        A.seg.resize(want_seg);
        return DPD_OK;
    }
    nck = std::max(nck, h->adj_nck);
    nseg = std::max(nseg, h->adj_nseg);
    nbin = std::max(nbin, h->adj_nbin);
    free_adj(h);
    const size_t N = (size_t)h->N, C = (size_t)h->C;
    A = AdjBufs();
    // every buffer carved from one allocation (one cudaMalloc instead of a few hundred)
    std::vector<std::pair<void **, size_t>> plan;
    auto want = [&](auto **p, size_t count) { plan.push_back({(void **)p, count * sizeof(**p)}); };
    A.ck.resize(nck);
    for (auto &c : A.ck) {
        want(&c.pos, N);
        want(&c.vh, N);
        want(&c.vt, N);
        want(&c.f, N);
        want(&c.tg, N);
        want(&c.link, N);
        want(&c.cstart, C + 1);
    }
    A.seg.resize(nseg);
    for (auto &c : A.seg) {
        want(&c.pos, N);
        want(&c.vt, N);
        want(&c.tg, N);
        want(&c.link, N);
        want(&c.cstart, C + 1);
    }
    want(&A.X, N);
    want(&A.V, N);
    want(&A.F, N);
    want(&A.g, N);
    want(&A.xb, N);
    want(&A.vb, N);
    want(&A.hist, (size_t)h->nrep * nbin);
    want(&A.wgt, (size_t)h->nrep * nbin);
    want(&A.grad, (size_t)h->nrep * DPD_NGRAD);
    want(&A.gsum, (size_t)h->nrep);
    size_t total = 0;
    for (auto &q : plan) total += (q.second + 64 + 255) & ~(size_t)255;
    char *base = nullptr;
    TRY(adj_alloc(h, &base, total));
    for (auto &q : plan) {
        *q.first = base;
        base += (q.second + 64 + 255) & ~(size_t)255;
    }
    h->adj = A;
    h->adj_nck = nck;
    h->adj_nseg = nseg;
    h->adj_nbin = nbin;
    A.ck.resize(want_ck);
    A.seg.resize(want_seg);
    return DPD_OK;
}

static void ck_save(dpd_handle *h, const FullCk &c) {
    const size_t N = (size_t)h->N, C = (size_t)h->C;
    const int k = h->cur;
    cudaMemcpyAsync(c.pos, h->b.pos[k], N * sizeof(float2), cudaMemcpyDeviceToDevice, h->s);
    cudaMemcpyAsync(c.vh, h->b.vh[k], N * sizeof(float2), cudaMemcpyDeviceToDevice, h->s);
    cudaMemcpyAsync(c.vt, h->b.vt[k], N * sizeof(float2), cudaMemcpyDeviceToDevice, h->s);
    cudaMemcpyAsync(c.f, h->b.f[k], N * sizeof(float2), cudaMemcpyDeviceToDevice, h->s);
    cudaMemcpyAsync(c.tg, h->b.tg[k], N * sizeof(uint32_t), cudaMemcpyDeviceToDevice, h->s);
    cudaMemcpyAsync(c.link, h->b.link[k], N * sizeof(int2), cudaMemcpyDeviceToDevice, h->s);
    cudaMemcpyAsync(c.cstart, h->b.cstart, (C + 1) * sizeof(int32_t), cudaMemcpyDeviceToDevice, h->s);
}

static void ck_restore(dpd_handle *h, const FullCk &c) {
    const size_t N = (size_t)h->N, C = (size_t)h->C;
    const int k = h->cur;
    cudaMemcpyAsync(h->b.pos[k], c.pos, N * sizeof(float2), cudaMemcpyDeviceToDevice, h->s);
    cudaMemcpyAsync(h->b.vh[k], c.vh, N * sizeof(float2), cudaMemcpyDeviceToDevice, h->s);
    cudaMemcpyAsync(h->b.vt[k], c.vt, N * sizeof(float2), cudaMemcpyDeviceToDevice, h->s);
    cudaMemcpyAsync(h->b.f[k], c.f, N * sizeof(float2), cudaMemcpyDeviceToDevice, h->s);
    cudaMemcpyAsync(h->b.tg[k], c.tg, N * sizeof(uint32_t), cudaMemcpyDeviceToDevice, h->s);
    cudaMemcpyAsync(h->b.link[k], c.link, N * sizeof(int2), cudaMemcpyDeviceToDevice, h->s);
    cudaMemcpyAsync(h->b.cstart, c.cstart, (C + 1) * sizeof(int32_t), cudaMemcpyDeviceToDevice, h->s);
    h->keys_valid = false;
}

static void seg_save(dpd_handle *h, const SegState &c) {
    const int k = h->cur;
    launch_adj_save((int)h->N, h->b.pos[k], h->b.vt[k], h->b.tg[k], h->b.link[k], c.pos, c.vt, c.tg, c.link, h->s);
    cudaMemcpyAsync(c.cstart, h->b.cstart, (size_t)(h->C + 1) * sizeof(int32_t), cudaMemcpyDeviceToDevice, h->s);
}

static StateView view_of(const SegState &c) { return StateView{c.pos, c.vt, c.tg, c.link, c.cstart}; }

static StateView view_cur(dpd_handle *h) {
    const int k = h->cur;
    return StateView{h->b.pos[k], h->b.vt[k], h->b.tg[k], h->b.link[k], h->b.cstart};
}

static void enqueue_plain_step(dpd_handle *h) {  // one step without chemistry (windows require chem off)
    enqueue_cell_sort(h, true);
    clear_stir(h);
    launch_permute(h->b, h->cur, h->d_rep, h->d_bch, h->nbch, PERM_STEP, h->s);
    h->cur ^= 1;
    enqueue_forces(h, true);
}

static int check_window(dpd_handle *h, int64_t nsteps, const dpd_rdf_spec *spec, const double *target) {
    if (nsteps < 1) return fail(DPD_E_ARG, "window of at least one step");
    if (!spec || !target) return fail(DPD_E_ARG, "null loss specification");
    if (spec->nbin < 1 || spec->nbin > 4096 || !(spec->rmax > 0.0) || !(spec->sigma > 0.0) || spec->last_steps < 1 ||
        spec->last_steps > nsteps || spec->horizon < 0)
        return fail(DPD_E_ARG, "bad loss specification");
    for (auto &p : h->params) {
        if (p.chem) return fail(DPD_E_ARG, "chemistry must be off inside a differentiated window");
        if (p.warmup > 0 && h->step < p.warm_end)
            return fail(DPD_E_ARG, "the repulsion warm-up must be over before a differentiated window");
    }
    return DPD_OK;
}

// host side of the loss: mean histogram -> rdf, loss and the weights dL/dh of every bin
static void rdf_loss(dpd_handle *h, const dpd_rdf_spec *spec, const std::vector<double> &hist,
                     const std::vector<long long> &npairs, const double *target, double *loss, double *rdf_out,
                     std::vector<double> *wgt) {
    const int nb = spec->nbin;
    const double dr = spec->rmax / nb;
    for (int r = 0; r < h->nrep; r++) {
        const double L = (double)h->rh[r].L, area = L * L;
        double sum = 0.0;
        for (int b = 0; b < nb; b++) {
            const double rb = (b + 0.5) * dr;
            const double norm = (npairs[r] > 0) ? area / ((double)npairs[r] * 2.0 * M_PI * rb * dr) : 0.0;
            const double g = hist[(size_t)r * nb + b] / spec->last_steps * norm;
            if (rdf_out) rdf_out[(size_t)r * nb + b] = g;
            const double e = g - target[(size_t)r * nb + b];
            sum += e * e;
            if (wgt) (*wgt)[(size_t)r * nb + b] = 2.0 * e / nb * norm / spec->last_steps;
        }
        if (loss) loss[r] = sum / nb;
    }
}

// unordered pairs of the loss types per replica (the types do not change in a window)
static int count_pairs(dpd_handle *h, const dpd_rdf_spec *spec, std::vector<long long> &npairs) {
    npairs.assign(h->nrep, 0);
    for (int r = 0; r < h->nrep; r++) {
        double o[16];
        TRY(observables_impl(h, r, false, o));
        const long long na = (long long)o[8 + spec->ta], nb = (long long)o[8 + spec->tb];
        npairs[r] = spec->ta == spec->tb ? na * (na - 1) / 2 : na * nb;
    }
    return DPD_OK;
}

// state_out (optional): the cotangents of the start state, gid order packed by
// replica, x/y interleaved: [0] positions, [1] stored half-step velocities,
// [2] predicted velocities (2 N floats each; host or device memory)
static int window_impl(dpd_handle *h, int64_t nsteps, int32_t ckpt, const dpd_rdf_spec *spec, const double *target,
                       double *loss, double *grad, double *rdf_out, bool backward, float *const *state_out = nullptr) {
    TRY(check_window(h, nsteps, spec, target));
    if (state_out && spec->horizon > 0)
        return fail(DPD_E_ARG, "start-state cotangents need the full reverse pass (horizon 0)");
    if (ckpt < 1) ckpt = (int32_t)nsteps;
    const int nseg = (int)((nsteps + ckpt - 1) / ckpt);
    const int nb = spec->nbin;
    const float rmax = (float)spec->rmax, sig = (float)spec->sigma;
    std::vector<long long> npairs;
    TRY(count_pairs(h, spec, npairs));
    AdjBufs A;
    TRY(adj_setup(h, backward ? nseg + 1 : 0, backward ? ckpt + 1 : 0, nb, A));
    if (!h->keys_valid) enqueue_next_keys(h);
    const int64_t step0 = h->step;
    const int64_t first_loss = nsteps - spec->last_steps + 1;  // window steps whose state enters the loss
    CK(cudaMemsetAsync(A.hist, 0, (size_t)h->nrep * nb * sizeof(double), h->s));
    // ---- forward, with a full checkpoint at the start of every segment
    for (int64_t k = 1; k <= nsteps; k++) {
        if (backward && (k - 1) % ckpt == 0) ck_save(h, A.ck[(k - 1) / ckpt]);
        enqueue_plain_step(h);
        if (k >= first_loss) launch_rdf(view_cur(h), h->d_rep, h->d_bch, h->nbch, spec->ta, spec->tb, nb, rmax, sig, A.hist, h->s);
    }
    CK(cudaGetLastError());
    h->step = step0 + nsteps;
    std::vector<double> hist((size_t)h->nrep * nb), wgt((size_t)h->nrep * nb);
    CK(cudaMemcpyAsync(hist.data(), A.hist, hist.size() * sizeof(double), cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    TRY(check_status(h));
    rdf_loss(h, spec, hist, npairs, target, loss, rdf_out, &wgt);
    if (!backward) return DPD_OK;
    const FullCk &end = A.ck[nseg];
    ck_save(h, end);
    const int cur_end = h->cur;
    CK(cudaMemcpyAsync(A.wgt, wgt.data(), wgt.size() * sizeof(double), cudaMemcpyHostToDevice, h->s));
    const size_t N = (size_t)h->N;
    CK(cudaMemsetAsync(A.X, 0, N * sizeof(float2), h->s));
    CK(cudaMemsetAsync(A.V, 0, N * sizeof(float2), h->s));
    CK(cudaMemsetAsync(A.F, 0, N * sizeof(float2), h->s));
    CK(cudaMemsetAsync(A.grad, 0, (size_t)h->nrep * DPD_NGRAD * sizeof(double), h->s));
    // ---- reverse, segment by segment, recomputing each segment's states, down to k_stop
    const int64_t k_stop = spec->horizon > 0 ? std::max<int64_t>(0, first_loss - 1 - spec->horizon) : 0;
    const int sg_stop = (int)(k_stop / ckpt);
    int stop_slot = 0;  // slot of the configuration k_stop in the last recomputed segment
    for (int sg = nseg - 1; sg >= sg_stop; sg--) {
        const int64_t k0 = (int64_t)sg * ckpt;
        const int len = (int)std::min<int64_t>(ckpt, nsteps - k0);
        ck_restore(h, A.ck[sg]);
        TRY(set_device_step(h, step0 + k0));
        enqueue_next_keys(h);
        seg_save(h, A.seg[0]);
        for (int s = 1; s <= len; s++) {
            enqueue_plain_step(h);
            seg_save(h, A.seg[s]);
        }
        const int s_low = sg == sg_stop ? (int)(k_stop - k0) : 0;
        stop_slot = s_low;
        for (int s = len; s > s_low; s--) {
            const int64_t k = k0 + s;
            const StateView v = view_of(A.seg[s]);
            if (k >= first_loss)
                launch_rdf_vjp(v, h->d_rep, h->d_bch, h->nbch, spec->ta, spec->tb, nb, rmax, sig, A.wgt, A.X, h->s);
            launch_adj_gather(v.tg, h->d_rep, h->d_bch, h->nbch, A.F, A.g, h->s);
            launch_force_vjp(v, step0 + k, h->d_rep, h->d_bch, h->nbch, A.g, A.xb, A.vb, A.grad, A.gsum, h->nrep,
                     h->any_stir, h->any_mol ? h->b.mol : nullptr, h->s);
            launch_adj_update(v.tg, h->d_rep, h->d_bch, h->nbch, A.xb, A.vb, A.X, A.V, A.F, h->s);
        }
    }
    // the forces stored at step k_stop (the window start without a horizon) depend on the parameters too
    const StateView v0 = view_of(A.seg[stop_slot]);
    launch_adj_gather(v0.tg, h->d_rep, h->d_bch, h->nbch, A.F, A.g, h->s);
    launch_force_vjp(v0, step0 + k_stop, h->d_rep, h->d_bch, h->nbch, A.g, A.xb, A.vb, A.grad, A.gsum, h->nrep,
                     h->any_stir, h->any_mol ? h->b.mol : nullptr, h->s);
    CK(cudaGetLastError());
    if (state_out) {
        launch_adj_state(v0.tg, h->d_rep, h->d_bch, h->nbch, A.xb, A.vb, A.X, A.g, h->s);
        const float2 *src[3] = {A.X, A.V, A.g};
        for (int k = 0; k < 3; k++)
            if (state_out[k]) CK(cudaMemcpyAsync(state_out[k], src[k], N * sizeof(float2), cudaMemcpyDefault, h->s));
    }
    if (grad) {
        CK(cudaMemcpyAsync(grad, A.grad, (size_t)h->nrep * DPD_NGRAD * sizeof(double), cudaMemcpyDefault, h->s));
    }
    // back to the end of the window
    h->cur = cur_end;
    ck_restore(h, end);
    TRY(set_device_step(h, step0 + nsteps));
    CK(cudaStreamSynchronize(h->s));
    return check_status(h);
}

extern "C" int dpd_window_loss(dpd_handle *h, int64_t nsteps, const dpd_rdf_spec *spec, const double *target,
                               double *loss, double *rdf_out) {
    if (!h) return fail(DPD_E_ARG, "null handle");
    return window_impl(h, nsteps, (int32_t)nsteps, spec, target, loss, nullptr, rdf_out, false);
}

extern "C" int dpd_window_adjoint(dpd_handle *h, int64_t nsteps, int32_t ckpt_every, const dpd_rdf_spec *spec,
                                  const double *target, double *loss, double *grad, double *rdf_out) {
    if (!h) return fail(DPD_E_ARG, "null handle");
    return window_impl(h, nsteps, ckpt_every, spec, target, loss, grad, rdf_out, true);
}

extern "C" int dpd_window_adjoint_state(dpd_handle *h, int64_t nsteps, int32_t ckpt_every, const dpd_rdf_spec *spec,
                                        const double *target, double *loss, double *grad, double *rdf_out,
                                        float *xbar, float *vhbar, float *vtbar) {
    if (!h) return fail(DPD_E_ARG, "null handle");
    float *const out[3] = {xbar, vhbar, vtbar};
    return window_impl(h, nsteps, ckpt_every, spec, target, loss, grad, rdf_out, true, out);
}

// ---------------------------------------------------------------- a fit as one captured graph
//
// One optimizer iteration of a shared-a_ij fit, enqueued without any host
// step: the window (full checkpoints every ckpt steps), the loss and its bin
// weights (k_rdf_loss), the reverse pass (the steps relative to the window's
// first, kept on the device), and the update (k_fit_update).  The iteration
// ends with the window's last state in the buffers of the parity it started
// from, so the captured graph can be replayed for the next iteration.
struct FitArgs {
    int64_t nsteps;
    int ckpt, nseg, nb;
    const dpd_rdf_spec *spec;
    FitDev *fd;
    const long long *npairs;
    const double *target;
    double *loss, *grad, *value;  // iters x nrep, iters x nfit, iters x nfit
};

static void enqueue_fit_iteration(dpd_handle *h, AdjBufs &A, const FitArgs &a) {
    const dpd_rdf_spec *spec = a.spec;
    const int nb = a.nb, ckpt = a.ckpt, nseg = a.nseg;
    const int64_t nsteps = a.nsteps;
    const float rmax = (float)spec->rmax, sig = (float)spec->sigma;
    const int cur0 = h->cur;
    launch_fit_begin(h->b.step, a.fd, h->s);
    cudaMemsetAsync(A.hist, 0, (size_t)h->nrep * nb * sizeof(double), h->s);
    enqueue_next_keys(h);
    const int64_t first_loss = nsteps - spec->last_steps + 1;
    for (int64_t k = 1; k <= nsteps; k++) {
        if ((k - 1) % ckpt == 0) ck_save(h, A.ck[(k - 1) / ckpt]);
        enqueue_plain_step(h);
        if (k >= first_loss) launch_rdf(view_cur(h), h->d_rep, h->d_bch, h->nbch, spec->ta, spec->tb, nb, rmax, sig, A.hist, h->s);
    }
    const FullCk &end = A.ck[nseg];
    ck_save(h, end);
    launch_rdf_loss(h->d_rep, h->nrep, A.hist, a.npairs, a.target, nb, spec->rmax, spec->last_steps, a.loss, A.wgt,
                    a.fd, h->s);
    const size_t N = (size_t)h->N;
    cudaMemsetAsync(A.X, 0, N * sizeof(float2), h->s);
    cudaMemsetAsync(A.V, 0, N * sizeof(float2), h->s);
    cudaMemsetAsync(A.F, 0, N * sizeof(float2), h->s);
    cudaMemsetAsync(A.grad, 0, (size_t)h->nrep * DPD_NGRAD * sizeof(double), h->s);
    const long long *base = &a.fd->base;
    const int64_t k_stop = spec->horizon > 0 ? std::max<int64_t>(0, first_loss - 1 - spec->horizon) : 0;
    const int sg_stop = (int)(k_stop / ckpt);
    int stop_slot = 0;
    const dpd_template *mol = h->any_mol ? h->b.mol : nullptr;
    for (int sg = nseg - 1; sg >= sg_stop; sg--) {
        const int64_t k0 = (int64_t)sg * ckpt;
        const int len = (int)std::min<int64_t>(ckpt, nsteps - k0);
        ck_restore(h, A.ck[sg]);
        launch_set_step_rel(h->b.step, a.fd, k0, h->s);
        enqueue_next_keys(h);
        seg_save(h, A.seg[0]);
        for (int s = 1; s <= len; s++) {
            enqueue_plain_step(h);
            seg_save(h, A.seg[s]);
        }
        const int s_low = sg == sg_stop ? (int)(k_stop - k0) : 0;
        stop_slot = s_low;
        for (int s = len; s > s_low; s--) {
            const int64_t k = k0 + s;
            const StateView v = view_of(A.seg[s]);
            if (k >= first_loss)
                launch_rdf_vjp(v, h->d_rep, h->d_bch, h->nbch, spec->ta, spec->tb, nb, rmax, sig, A.wgt, A.X, h->s);
            launch_adj_gather(v.tg, h->d_rep, h->d_bch, h->nbch, A.F, A.g, h->s);
            launch_force_vjp(v, k, h->d_rep, h->d_bch, h->nbch, A.g, A.xb, A.vb, A.grad, A.gsum, h->nrep, h->any_stir,
                             mol, h->s, base);
            launch_adj_update(v.tg, h->d_rep, h->d_bch, h->nbch, A.xb, A.vb, A.X, A.V, A.F, h->s);
        }
    }
    const StateView v0 = view_of(A.seg[stop_slot]);
    launch_adj_gather(v0.tg, h->d_rep, h->d_bch, h->nbch, A.F, A.g, h->s);
    launch_force_vjp(v0, k_stop, h->d_rep, h->d_bch, h->nbch, A.g, A.xb, A.vb, A.grad, A.gsum, h->nrep, h->any_stir,
                     mol, h->s, base);
    // the window's end into the starting parity's buffers, the step after the window
    h->cur = cur0;
    ck_restore(h, end);
    launch_set_step_rel(h->b.step, a.fd, nsteps, h->s);
    launch_fit_update(h->d_rep, h->nrep, A.grad, a.fd, a.grad, a.value, h->s);
}

extern "C" int dpd_fit_graph(dpd_handle *h, int64_t nsteps, int32_t ckpt, const dpd_rdf_spec *spec,
                             const double *target, const dpd_fit_spec *fit, int32_t iters, double *loss, double *grad,
                             double *values) {
    TRY(check_window(h, nsteps, spec, target));
    if (!fit || fit->n < 1 || fit->n > DPD_MAXT * DPD_MAXT) return fail(DPD_E_ARG, "fit: 1 to 64 slots");
    if (iters < 1) return fail(DPD_E_ARG, "fit: at least one iteration");
    if (!(fit->lr > 0.0) || !(fit->beta1 >= 0.0 && fit->beta1 < 1.0) || !(fit->beta2 >= 0.0 && fit->beta2 < 1.0) ||
        !(fit->eps > 0.0))
        return fail(DPD_E_ARG, "fit: lr > 0, 0 <= beta < 1, eps > 0");
    FitDev F;
    std::memset(&F, 0, sizeof F);
    F.nfit = fit->n;
    F.lr = fit->lr;
    F.beta1 = fit->beta1;
    F.beta2 = fit->beta2;
    F.eps = fit->eps;
    for (int k = 0; k < fit->n; k++) {
        const int s = fit->slot[k], i = s / DPD_MAXT, j = s % DPD_MAXT;
        if (s < 0 || s >= DPD_MAXT * DPD_MAXT || i > j)
            return fail(DPD_E_ARG, "fit: slot %d is not i * 8 + j with i <= j", s);
        for (int q = 0; q < k; q++)
            if (fit->slot[q] == s) return fail(DPD_E_ARG, "fit: slot %d twice", s);
        F.slot[k] = s;
        F.value[k] = h->params[0].a[s];
        for (int r = 1; r < h->nrep; r++)
            if (h->params[r].a[s] != F.value[k])
                return fail(DPD_E_ARG, "fit: a shared slot (%d) must start equal in every replica", s);
    }
    if (ckpt < 1) ckpt = (int32_t)nsteps;
    const int nseg = (int)((nsteps + ckpt - 1) / ckpt), nb = spec->nbin, nrep = h->nrep;
    std::vector<long long> npairs;
    TRY(count_pairs(h, spec, npairs));
    AdjBufs A;
    TRY(adj_setup(h, nseg + 1, ckpt + 1, nb, A));
    // the fit's own device memory, freed before returning
    char *mem = nullptr;
    const size_t o_np = ((sizeof(FitDev) + 255) / 256) * 256, o_tg = o_np + (((size_t)nrep * 8 + 255) / 256) * 256;
    const size_t o_loss = o_tg + (((size_t)nrep * nb * 8 + 255) / 256) * 256;
    const size_t o_grad = o_loss + (((size_t)iters * nrep * 8 + 255) / 256) * 256;
    const size_t o_val = o_grad + (((size_t)iters * fit->n * 8 + 255) / 256) * 256;
    const size_t total = o_val + (((size_t)iters * fit->n * 8 + 255) / 256) * 256;
    if (cudaMalloc(&mem, total) != cudaSuccess) return fail(DPD_E_NOMEM, "cudaMalloc(%zu) for the fit", total);
    FitArgs a;
    a.nsteps = nsteps;
    a.ckpt = ckpt;
    a.nseg = nseg;
    a.nb = nb;
    a.spec = spec;
    a.fd = (FitDev *)mem;
    a.npairs = (const long long *)(mem + o_np);
    a.target = (const double *)(mem + o_tg);
    a.loss = (double *)(mem + o_loss);
    a.grad = (double *)(mem + o_grad);
    a.value = (double *)(mem + o_val);
    int rc = DPD_OK;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    const int cur0 = h->cur;
    do {
        if (cudaMemcpy(mem, &F, sizeof F, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(mem + o_np, npairs.data(), nrep * sizeof(long long), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(mem + o_tg, target, (size_t)nrep * nb * sizeof(double), cudaMemcpyDefault) != cudaSuccess) {
            rc = fail(DPD_E_CUDA, "fit: copies to the device: %s", cudaGetErrorString(cudaGetLastError()));
            break;
        }
        if (cudaStreamSynchronize(h->s) != cudaSuccess ||
            cudaStreamBeginCapture(h->s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            rc = fail(DPD_E_CUDA, "fit: capture: %s", cudaGetErrorString(cudaGetLastError()));
            break;
        }
        enqueue_fit_iteration(h, A, a);
        const cudaError_t e = cudaStreamEndCapture(h->s, &g);
        h->cur = cur0;
        if (e != cudaSuccess || cudaGraphInstantiate(&ge, g, 0) != cudaSuccess) {
            rc = fail(DPD_E_CUDA, "fit: graph: %s", cudaGetErrorString(e != cudaSuccess ? e : cudaGetLastError()));
            break;
        }
        for (int it = 0; it < iters && rc == DPD_OK; it++)
            if (cudaGraphLaunch(ge, h->s) != cudaSuccess) rc = fail(DPD_E_CUDA, "fit: launch");
        if (rc != DPD_OK) break;
        if (cudaStreamSynchronize(h->s) != cudaSuccess) {
            rc = fail(DPD_E_CUDA, "fit: %s", cudaGetErrorString(cudaGetLastError()));
            break;
        }
        if ((rc = check_status(h)) != DPD_OK) break;
        FitDev out;
        if (cudaMemcpy(&out, mem, sizeof out, cudaMemcpyDeviceToHost) != cudaSuccess ||
            (loss && cudaMemcpy(loss, a.loss, (size_t)iters * nrep * 8, cudaMemcpyDefault) != cudaSuccess) ||
            (grad && cudaMemcpy(grad, a.grad, (size_t)iters * fit->n * 8, cudaMemcpyDefault) != cudaSuccess) ||
            (values && cudaMemcpy(values, a.value, (size_t)iters * fit->n * 8, cudaMemcpyDefault) != cudaSuccess)) {
            rc = fail(DPD_E_CUDA, "fit: copies from the device");
            break;
        }
        if (values)
            for (int k = 0; k < fit->n; k++) values[(size_t)iters * fit->n + k] = out.value[k];
        // the host's view of the handle: the steps taken, the fitted values in every replica
        h->step += (int64_t)iters * nsteps;
        h->keys_valid = false;
        for (int r = 0; r < nrep && rc == DPD_OK; r++) {
            dpd_params p = h->params[r];
            for (int k = 0; k < fit->n; k++) {
                const int s = fit->slot[k], i = s / DPD_MAXT, j = s % DPD_MAXT;
                p.a[i * DPD_MAXT + j] = p.a[j * DPD_MAXT + i] = out.value[k];
            }
            rc = dpd_set_params(h, r, &p);
        }
    } while (false);
    if (ge) cudaGraphExecDestroy(ge);
    if (g) cudaGraphDestroy(g);
    cudaFree(mem);
    return rc;
}

extern "C" int dpd_force_vjp(dpd_handle *h, int32_t r, int64_t step, const float *gx, const float *gy, float *xbar_x,
                             float *xbar_y, float *vbar_x, float *vbar_y, double *grad) {
    TRY(ensure_replica(h, r));
    if (!gx || !gy) return fail(DPD_E_ARG, "null cotangent");
    const RepDev &R = h->rh[r];
    const size_t n = (size_t)R.n, N = (size_t)h->N, a = ((n * 4 + 255) / 256) * 256;
    AdjBufs A;
    TRY(adj_setup(h, 0, 0, 1, A));
    CK(cudaMemsetAsync(A.g, 0, N * sizeof(float2), h->s));
    CK(cudaMemsetAsync(A.grad, 0, (size_t)h->nrep * DPD_NGRAD * sizeof(double), h->s));
    float *sx = (float *)h->stage, *sy = (float *)(h->stage + a);
    CK(cudaMemcpyAsync(sx, gx, n * 4, cudaMemcpyDefault, h->s));
    CK(cudaMemcpyAsync(sy, gy, n * 4, cudaMemcpyDefault, h->s));
    // pack the cotangent into the replica's slots via the state packer's force field
    Bufs u = h->b;
    u.f[h->cur] = A.g;
    launch_set_dynamics(u, h->cur, R.b0, (int)n, nullptr, nullptr, sx, sy, nullptr, nullptr, h->s);
    launch_force_vjp(view_cur(h), step, h->d_rep, h->d_bch, h->nbch, A.g, A.xb, A.vb, A.grad, A.gsum, h->nrep,
                     h->any_stir, h->any_mol ? h->b.mol : nullptr, h->s);
    CK(cudaGetLastError());
    float *outs[4] = {xbar_x, xbar_y, vbar_x, vbar_y};
    float *st[4];
    for (int k = 0; k < 4; k++) st[k] = (float *)(h->stage + k * a);
    Bufs w = h->b;
    w.f[h->cur] = A.xb;
    w.vh[h->cur] = A.vb;
    launch_unpack(w, h->cur, R.b0, (int)n, nullptr, nullptr, st[2], st[3], nullptr, nullptr, st[0], st[1], nullptr,
                  nullptr, nullptr, nullptr, h->s);
    CK(cudaGetLastError());
    for (int k = 0; k < 4; k++)
        if (outs[k]) CK(cudaMemcpyAsync(outs[k], st[k], n * 4, cudaMemcpyDefault, h->s));
    if (grad) CK(cudaMemcpyAsync(grad, A.grad + (size_t)r * DPD_NGRAD, DPD_NGRAD * sizeof(double), cudaMemcpyDefault, h->s));
    CK(cudaStreamSynchronize(h->s));
    return DPD_OK;
}
