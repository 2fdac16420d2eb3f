// dpd_catalyst.cu -- the reference's catalyst chemistry (chem_kind 1) on the GPU.
//
// One chemistry check of cel/engine/oercel.c:1565-1753, with its semantics:
//   1. the catalysts (Ka, Kb) in slot order, shuffled with the serial
//      xoshiro256** generator, are visited one after the other: lipid
//      synthesis from the nearest N beads (centroid, best of syn_tries
//      random orientations by overlap energy, steepest-descent relaxation of
//      the new chain), then replication / mutation onto the next nearest N;
//   2. decay of lipids, catalysts and N by keyed deviates of (seed, step, gid);
//   3. the W -> N food supply, uniform or in a vent, with a cap on the N
//      fraction that keeps a random subset (serial generator) of the candidates.
// The catalysts of one replica form a chain of dependent decisions (each sees
// what the earlier ones did, and all draw from one serial stream), so one CTA
// per replica walks them in order.  Around each catalyst the CTA stages the
// cells within reach of everything the visit can touch into shared memory and
// does the neighbour searches, the overlap energies and the relaxation forces
// there in parallel; one thread makes the decisions.  All geometry is FP64 on
// the FP32 state, the reference's formulas in its order; sums over beads are
// block reductions in a fixed order, so a run is deterministic.
// Candidate sets are those of the reference: beads of the cells in the
// reference's windows around the cells the reference uses (the cell index of
// the last sort), then the distance tests.
#include <algorithm>

#include "dpd_chem.cuh"

#define CAT_TPB 256
#define CAT_WARPS (CAT_TPB / 32)
#define CAT_MAXS 2048    // staged beads around one catalyst
#define CAT_MAXC 1024    // staged cells
#define CAT_MAXML 16     // beads of a lipid
#define CAT_MAXNB 256    // N (or W) candidates of one catalyst (the reference keeps 256)
#define CAT_MAXRN 512    // relaxation neighbours of a new chain (the reference keeps 512)
#define CAT_MARGIN 0.5   // oercel.c:1348
#define CAT_WIN 1024     // catalysts per window of the walk
#define CAT_MAXTR DPD_CAT_MAXTR
// what the walk does with a catalyst: no draws (fewer than 2 N), the replication
// draw, the synthesis and replication draws, or a visit by the whole CTA
#define CAT_SHUF_SH 11264  // catalysts per replica whose shuffle scratch fits in shared memory (5 x 44 KB)
#define WALK_NONE 0
#define WALK_REP 1
#define WALK_SYN 2
#define WALK_VISIT 3

// event kinds after the lipid chemistry's 0..2
#define EV_SYN 3
#define EV_REP 4
#define EV_MUT 5
#define EV_DLIP 6
#define EV_DK 7
#define EV_DN 8
#define EV_FEED 9

struct CatSmem {
    float2 pos[CAT_MAXS];
    int32_t slot[CAT_MAXS];
    uint32_t gid[CAT_MAXS];
    int16_t cx[CAT_MAXS], cy[CAT_MAXS];  // cell of the bead's slot (the last sort)
    uint8_t type[CAT_MAXS];
    int32_t wstart[CAT_MAXC + 1];        // staged index of each window cell's first bead
    int32_t wg[CAT_MAXC];                // global slot of each window cell's first bead
    int16_t wcx[CAT_MAXC], wcy[CAT_MAXC];
    int32_t ns, ncw;
    int32_t nn, nw, nrn;
    int32_t nb[CAT_MAXNB], nbw[CAT_MAXNB];
    double nbd[CAT_MAXNB], nbwd[CAT_MAXNB];
    int32_t sl[CAT_MAXML];               // staged index of each bead of a new chain
    double px[CAT_MAXML], py[CAT_MAXML];
    double fx[CAT_MAXML], fy[CAT_MAXML];
    int32_t rn[CAT_MAXRN];
    double red[2][CAT_WARPS];
    int32_t scan[CAT_WARPS];
    uint64_t rng[4];
    int32_t go, k, var, ml;
    int32_t over;                        // a search found more than CAT_MAXNB candidates
    int32_t nd;                          // draws of the current visit
    int32_t serial, first, exhaust;      // walk state: serial mode, first stop of a segment, stop reason
    long long P, fpos;                   // stream position of the walk, of the first stop
    double tux[CAT_MAXTR], tuy[CAT_MAXTR], tU[CAT_MAXTR];  // trial directions of a synthesis, their energies
    int32_t nchg;                        // beads whose type the current visit changed
    float2 chg[CAT_MAXML + 2];           // and their positions before the change
    int32_t wk[CAT_WIN];                 // the window of the walk: catalyst slots and
    uint8_t wcode[CAT_WIN];              // their actions: WALK_* | Kb << 2
    double xk, yk, ux, uy, cxm, cym;
};

// ---------------------------------------------------------------- serial generator (oercel.c:143-174)

__device__ __forceinline__ uint64_t xo_rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
__device__ __forceinline__ uint64_t xo_next(uint64_t *s) {
    const uint64_t r = xo_rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = xo_rotl(s[3], 45);
    return r;
}
__device__ __forceinline__ double xo_unif(uint64_t *s) { return (double)(xo_next(s) >> 11) * 0x1.0p-53; }
// xo_unif(s) < p  <=>  (xo_next(s) >> 11) < u01_threshold(p): the draw is k 2^-53
// with an integer k < 2^53, and k < v <=> k < ceil(v) for real v = p 2^53
__host__ __device__ __forceinline__ uint64_t u01_threshold(double p) {
    if (!(p > 0.0)) return 0;
    if (p >= 1.0) return 1ull << 53;
    return (uint64_t)ceil(p * 0x1.0p53);
}
__device__ __forceinline__ long long xo_below(uint64_t *s, long long n) {
    const long long k = (long long)(xo_unif(s) * (double)n);
    return k >= n ? n - 1 : k;
}

// keyed uniform deviates of the parallel decisions (oercel.c:819-826)
__device__ __forceinline__ uint64_t cat_key(uint64_t seed, long long step, uint64_t salt) {
    return mix13(seed ^ mix13((uint64_t)step * 0x9e3779b97f4a7c15ULL + salt));
}
__device__ __forceinline__ double cat_u01(uint64_t key, uint32_t g) {
    return (double)(mix13(key ^ ((uint64_t)g * 0xd1b54a32d192ed03ULL)) >> 11) * 0x1.0p-53;
}

// ---------------------------------------------------------------- FP64 geometry of the reference

__device__ __forceinline__ double dmin(double d, double L) {
    const double h = 0.5 * L;
    return d > h ? d - L : (d < -h ? d + L : d);
}
__device__ __forceinline__ double dwrap(double v, double L) {
    if (v < 0.0) {
        v += L;
        if (v >= L) v -= L;
    } else if (v >= L) {
        v -= L;
        if (v >= L || v < 0.0) v = fmod(v, L);
    }
    return v;
}
__device__ __forceinline__ void dcell(const RepDev &R, double x, double y, int &cx, int &cy) {
    cx = (int)(x * R.icsx);
    cy = (int)(y * R.icsy);
    cx = cx >= R.ncx ? R.ncx - 1 : (cx < 0 ? 0 : cx);
    cy = cy >= R.ncy ? R.ncy - 1 : (cy < 0 ? 0 : cy);
}
// is cell column c within [c0 - r, c0 + r] (periodic, n columns, 2r + 1 <= n)
__device__ __forceinline__ bool in_band(int c, int c0, int r, int n) {
    int d = (c - c0 + r) % n;
    d += d < 0 ? n : 0;
    return d <= 2 * r;
}

// ---------------------------------------------------------------- block helpers

__device__ __forceinline__ int block_excl_scan(CatSmem &S, int v, int &total) {
    const int lane = (int)lane_id(), w = (int)threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    __syncthreads();
    if (lane == 31) S.scan[w] = x;
    __syncthreads();
    int before = 0;
    total = 0;
    for (int k = 0; k < CAT_WARPS; k++) {
        before += k < w ? S.scan[k] : 0;
        total += S.scan[k];
    }
    return before + x - v;
}

// ---------------------------------------------------------------- staging

// Stage the cells within R.cat_E of cell (cx0, cy0) (all columns / rows once
// if the window covers the box).  Returns false if they do not fit.
__device__ bool stage(CatSmem &S, const Bufs &b, int cur, const RepDev &R, int cx0, int cy0) {
    const int E = R.cat_E, ncx = R.ncx, ncy = R.ncy;
    const int ncol = 2 * E + 1 >= ncx ? ncx : 2 * E + 1, nrow = 2 * E + 1 >= ncy ? ncy : 2 * E + 1;
    const int c0 = 2 * E + 1 >= ncx ? 0 : cx0 - E, r0 = 2 * E + 1 >= ncy ? 0 : cy0 - E;
    const int ncw = ncol * nrow;
    if (ncw > CAT_MAXC) return false;
    const int32_t *cs = b.cstart + R.c0;
    int cnt[CAT_MAXC / CAT_TPB];
    int mine = 0;
    for (int q = 0; q < CAT_MAXC / CAT_TPB; q++) {
        const int w = q * CAT_TPB + (int)threadIdx.x;
        cnt[q] = 0;
        if (w < ncw) {
            int gx = c0 + w / nrow, gy = r0 + w % nrow;
            gx += gx < 0 ? ncx : (gx >= ncx ? -ncx : 0);
            gy += gy < 0 ? ncy : (gy >= ncy ? -ncy : 0);
            const int gc = gx * ncy + gy;
            const int g0 = __ldcg(cs + gc);
            cnt[q] = __ldcg(cs + gc + 1) - g0;
            S.wg[w] = g0;
            S.wcx[w] = (int16_t)gx;
            S.wcy[w] = (int16_t)gy;
        }
        mine += cnt[q];
    }
    // window cells of thread t are t, t + TPB, ...: scan them in window order
    int base = 0;
    for (int q = 0; q < CAT_MAXC / CAT_TPB; q++) {
        int tot;
        const int ex = block_excl_scan(S, cnt[q], tot);
        const int w = q * CAT_TPB + (int)threadIdx.x;
        if (w < ncw) S.wstart[w] = base + ex;
        base += tot;
    }
    (void)mine;
    if (threadIdx.x == 0) {
        S.wstart[ncw] = base;
        S.ns = base;
        S.ncw = ncw;
    }
    __syncthreads();
    const int ns = S.ns;
    if (ns > CAT_MAXS) return false;
    for (int i = (int)threadIdx.x; i < ns; i += CAT_TPB) {
        int lo = 0, hi = ncw;  // last window cell with wstart <= i
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (S.wstart[mid] <= i) lo = mid;
            else hi = mid;
        }
        const int g = S.wg[lo] + (i - S.wstart[lo]);
        S.slot[i] = g;
        S.pos[i] = __ldcg(b.pos[cur] + g);
        const uint32_t tg = __ldcg(b.tg[cur] + g);
        S.type[i] = (uint8_t)(tg >> TYPE_SHIFT);
        S.gid[i] = tg & GID_MASK;
        S.cx[i] = S.wcx[lo];
        S.cy[i] = S.wcy[lo];
    }
    __syncthreads();
    return true;
}

// beads of type `want` within rcut of (xk, yk) in the reference's cell window
// (find_type_near, oercel.c:1353-1398), nearest first, ties by lower gid
__device__ void find_near(CatSmem &S, const RepDev &R, int kslot, double xk, double yk, double rcut, int want,
                          int32_t *out, double *outd, int32_t *nout) {
    const double L = (double)R.L, r2c = rcut * rcut;
    int cx, cy;
    dcell(R, xk, yk, cx, cy);
    const int rx = (int)ceil((rcut + CAT_MARGIN) * R.icsx), ry = (int)ceil((rcut + CAT_MARGIN) * R.icsy);
    if (threadIdx.x == 0) *nout = 0;
    __syncthreads();
    for (int i = (int)threadIdx.x; i < S.ns; i += CAT_TPB) {
        if (S.type[i] != want || S.slot[i] == kslot) continue;
        if (!in_band(S.cx[i], cx, rx, R.ncx) || !in_band(S.cy[i], cy, ry, R.ncy)) continue;
        const double dx = dmin((double)S.pos[i].x - xk, L), dy = dmin((double)S.pos[i].y - yk, L);
        const double d2 = dx * dx + dy * dy;
        if (d2 < r2c) {
            const int q = atomicAdd(nout, 1);
            if (q < CAT_MAXNB) {
                out[q] = i;
                outd[q] = d2;
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        S.over |= *nout > CAT_MAXNB;  // which ones the atomics kept is arbitrary: reported, not used
        const int n = min(*nout, CAT_MAXNB);
        for (int a = 1; a < n; a++) {
            const int ti = out[a];
            const double td = outd[a];
            int c = a - 1;
            while (c >= 0 && (outd[c] > td || (outd[c] == td && S.gid[out[c]] > S.gid[ti]))) {
                out[c + 1] = out[c];
                outd[c + 1] = outd[c];
                c--;
            }
            out[c + 1] = ti;
            outd[c + 1] = td;
        }
        *nout = n;
    }
    __syncthreads();
}

// bead bb of a new lipid centred at (cx0, cy0) with long axis u: the linear
// chain along u (oercel.c:1433-1436), or the template turned onto u
// (oercel.c:1437-1440)
__device__ __forceinline__ void place(const RepDev &R, const dpd_template &M, int bb, int ml, double cx0, double cy0,
                                      double ux, double uy, double L, double &px, double &py) {
    if (R.arch == 0) {
        const double off = (bb - 0.5 * (ml - 1)) * R.r0_d;
        px = dwrap(cx0 + off * ux, L);
        py = dwrap(cy0 + off * uy, L);
    } else {
        px = dwrap(cx0 + (M.px[bb] * ux - M.py[bb] * uy), L);
        py = dwrap(cy0 + (M.px[bb] * uy + M.py[bb] * ux), L);
    }
}

// a draw of the visit from the generator state S.rng, counted (thread 0)
__device__ __forceinline__ double draw(CatSmem &S) {
    S.nd++;
    return xo_unif(S.rng);
}

__device__ __forceinline__ bool in_chain(const CatSmem &S, int i, int ml) {
    bool r = false;
    for (int q = 0; q < ml; q++) r |= S.sl[q] == i;
    return r;
}

// overlap energy of the would-be straight chain (centre, direction u) with the
// beads outside it (chain_overlap_energy, oercel.c:1425-1468), for each trial
// direction S.tu[tr] at once: trial tr on warp tr % CAT_WARPS, its lanes over
// the staged beads; S.tU[tr] receives the energy
__device__ void chain_energies(CatSmem &S, const RepDev &R, const dpd_template &M, double cx0, double cy0, int ntr,
                               int ml) {
    const double L = (double)R.L;
    const int rx = (int)ceil((1.0 + CAT_MARGIN) * R.icsx), ry = (int)ceil((1.0 + CAT_MARGIN) * R.icsy);
    const int lane = (int)lane_id(), warp = (int)threadIdx.x >> 5;
    for (int tr = warp; tr < ntr; tr += CAT_WARPS) {
        const double ux = S.tux[tr], uy = S.tuy[tr];
        double U = 0.0;
        for (int bb = 0; bb < ml; bb++) {
            double px, py;
            place(R, M, bb, ml, cx0, cy0, ux, uy, L, px, py);
            const int tb = bb < R.lip_nH ? 1 : 2;
            int cx, cy;
            dcell(R, px, py, cx, cy);
            for (int i = lane; i < S.ns; i += 32) {
                if (!in_band(S.cx[i], cx, rx, R.ncx) || !in_band(S.cy[i], cy, ry, R.ncy) || in_chain(S, i, ml))
                    continue;
                const double dx = dmin((double)S.pos[i].x - px, L), dy = dmin((double)S.pos[i].y - py, L);
                const double r2 = dx * dx + dy * dy;
                if (r2 >= 1.0) continue;
                const double w = 1.0 - sqrt(r2);
                U += 0.5 * (double)R.a[tb * DPD_MAXT + S.type[i]] * w * w;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) U += __shfl_down_sync(0xffffffffu, U, o);
        if (lane == 0) S.tU[tr] = U;
    }
    __syncthreads();
}

// steepest-descent relaxation of the new chain S.px/py against its frozen
// surroundings (relax_new_chain, oercel.c:1473-1560): pair repulsion, then the
// chain's bonds and angles (the linear terms, or the template's)
__device__ void relax_chain(CatSmem &S, const RepDev &R, const dpd_template &M, int ml, bool &overflow) {
    const double L = (double)R.L, cap = 0.05, alpha = 0.002;
    const double reach = 1.0 + cap * R.syn_relax, reach2 = reach * reach;
    const int rx = (int)ceil((reach + CAT_MARGIN) * R.icsx), ry = (int)ceil((reach + CAT_MARGIN) * R.icsy);
    int ccx[CAT_MAXML], ccy[CAT_MAXML];
    for (int bb = 0; bb < ml; bb++) dcell(R, S.px[bb], S.py[bb], ccx[bb], ccy[bb]);
    // neighbours within reach of any chain bead, in staged order
    int base = 0;
    for (int i0 = 0; i0 < S.ns; i0 += CAT_TPB) {
        const int i = i0 + (int)threadIdx.x;
        bool take = false;
        if (i < S.ns && !in_chain(S, i, ml))
            for (int bb = 0; bb < ml && !take; bb++) {
                if (!in_band(S.cx[i], ccx[bb], rx, R.ncx) || !in_band(S.cy[i], ccy[bb], ry, R.ncy)) continue;
                const double dx = dmin((double)S.pos[i].x - S.px[bb], L), dy = dmin((double)S.pos[i].y - S.py[bb], L);
                take = dx * dx + dy * dy < reach2;
            }
        int tot;
        const int ex = block_excl_scan(S, take ? 1 : 0, tot);
        if (take && base + ex < CAT_MAXRN) S.rn[base + ex] = i;
        base += tot;
    }
    if (base > CAT_MAXRN) overflow = true;
    const int nrn = min(base, CAT_MAXRN);
    const int lane = (int)lane_id(), warp = (int)threadIdx.x >> 5;
    for (int it = 0; it < R.syn_relax; it++) {
        // chain bead bb: warp bb % CAT_WARPS, its lanes over the neighbours
        for (int bb = warp; bb < ml; bb += CAT_WARPS) {
            const int ti = bb < R.lip_nH ? 1 : 2;
            double fx = 0.0, fy = 0.0;
            for (int q = lane; q < nrn; q += 32) {
                const int j = S.rn[q];
                const double dx = dmin(S.px[bb] - (double)S.pos[j].x, L), dy = dmin(S.py[bb] - (double)S.pos[j].y, L);
                const double r2 = dx * dx + dy * dy;
                if (r2 >= 1.0 || r2 < 1e-24) continue;
                const double r = sqrt(r2);
                const double f = (double)R.a[ti * DPD_MAXT + S.type[j]] * (1.0 - r) / r;
                fx += f * dx;
                fy += f * dy;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                fx += __shfl_down_sync(0xffffffffu, fx, o);
                fy += __shfl_down_sync(0xffffffffu, fy, o);
            }
            if (lane == 0) {
                S.fx[bb] = fx;
                S.fy[bb] = fy;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0 && R.arch != 0) {
            // the template's bonds and angles by position (mol_forces, oercel.c:1221-1257)
            for (int q = 0; q < M.nb; q++) {
                const int i = M.bi[q], j = M.bj[q];
                const double dx = dmin(S.px[j] - S.px[i], L), dy = dmin(S.py[j] - S.py[i], L);
                const double r = sqrt(dx * dx + dy * dy);
                const double f = -R.kb_d * (r - M.br0[q]) / r;
                S.fx[j] += f * dx;
                S.fy[j] += f * dy;
                S.fx[i] -= f * dx;
                S.fy[i] -= f * dy;
            }
            for (int q = 0; q < M.na; q++) {
                const int i = M.ai[q], j = M.aj[q], k = M.ak[q];
                const double ax = dmin(S.px[j] - S.px[i], L), ay = dmin(S.py[j] - S.py[i], L);
                const double cxv = dmin(S.px[k] - S.px[j], L), cyv = dmin(S.py[k] - S.py[j], L);
                const double la = sqrt(ax * ax + ay * ay), lc = sqrt(cxv * cxv + cyv * cyv);
                const double ilac = 1.0 / (la * lc), cs = (ax * cxv + ay * cyv) * ilac;
                const double g = M.akind[q] == 0 ? -M.aK[q] : 2.0 * M.aK[q] * (cs - M.ac0[q]);
                const double dUax = g * (cxv * ilac - cs * ax / (la * la)), dUay = g * (cyv * ilac - cs * ay / (la * la));
                const double dUcx = g * (ax * ilac - cs * cxv / (lc * lc)), dUcy = g * (ay * ilac - cs * cyv / (lc * lc));
                S.fx[i] += dUax;
                S.fy[i] += dUay;
                S.fx[j] += -dUax + dUcx;
                S.fy[j] += -dUay + dUcy;
                S.fx[k] -= dUcx;
                S.fy[k] -= dUcy;
            }
        }
        if (threadIdx.x == 0) {
            double bx[CAT_MAXML], by[CAT_MAXML], bl[CAT_MAXML];
            for (int bb = 0; bb < ml - 1 && R.arch == 0; bb++) {
                bx[bb] = dmin(S.px[bb + 1] - S.px[bb], L);
                by[bb] = dmin(S.py[bb + 1] - S.py[bb], L);
                bl[bb] = sqrt(bx[bb] * bx[bb] + by[bb] * by[bb]);
                const double f = -R.kb_d * (bl[bb] - R.r0_d) / bl[bb];
                S.fx[bb + 1] += f * bx[bb];
                S.fy[bb + 1] += f * by[bb];
                S.fx[bb] -= f * bx[bb];
                S.fy[bb] -= f * by[bb];
            }
            for (int bb = 0; bb < ml - 2 && R.ka_d != 0.0 && R.arch == 0; bb++) {
                const double ax = bx[bb], ay = by[bb], cxv = bx[bb + 1], cyv = by[bb + 1], la = bl[bb], lc = bl[bb + 1];
                const double ilac = 1.0 / (la * lc), cs = (ax * cxv + ay * cyv) * ilac, ka = R.ka_d;
                const double dUax = -ka * (cxv * ilac - cs * ax / (la * la)), dUay = -ka * (cyv * ilac - cs * ay / (la * la));
                const double dUcx = -ka * (ax * ilac - cs * cxv / (lc * lc)), dUcy = -ka * (ay * ilac - cs * cyv / (lc * lc));
                S.fx[bb] += dUax;
                S.fy[bb] += dUay;
                S.fx[bb + 1] += -dUax + dUcx;
                S.fy[bb + 1] += -dUay + dUcy;
                S.fx[bb + 2] -= dUcx;
                S.fy[bb + 2] -= dUcy;
            }
            for (int bb = 0; bb < ml; bb++) {
                double mx = alpha * S.fx[bb], my = alpha * S.fy[bb];
                const double m = sqrt(mx * mx + my * my);
                if (m > cap) {
                    mx *= cap / m;
                    my *= cap / m;
                }
                S.px[bb] = dwrap(S.px[bb] + mx, L);
                S.py[bb] = dwrap(S.py[bb] + my, L);
            }
        }
        __syncthreads();
    }
}

__device__ __forceinline__ void set_type(const Bufs &b, int cur, int g, int t) {
    uint32_t *tg = b.tg[cur];
    tg[g] = ((uint32_t)t << TYPE_SHIFT) | (__ldcg(tg + g) & GID_MASK);
}

// ---------------------------------------------------------------- 1. the catalysts

// per chunk: how many beads are catalysts (the list is built in slot order)
__global__ void __launch_bounds__(BEAD_TPB) k_cat_count(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                        const Chunk *__restrict__ ch, int mode) {
    __shared__ int red[BEAD_TPB / 32];
    const Chunk c = ch[blockIdx.x];
    const RepDev &R = reps[c.rep];
    const long long step = *b.step;
    const int d = c.begin + (int)threadIdx.x;
    int v = 0, vn = 0;
    if (cat_due(R, step) && d < c.end) {
        const uint32_t tg = b.tg[cur][d];
        const int t = (int)(tg >> TYPE_SHIFT);
        if (mode == 0) {
            v = t == 4 || t == 5;
        } else {
            const float2 p = b.pos[cur][d];
            const uint64_t kf = cat_key(R.seed, step, 14);
            bool in = true;
            if (R.feed_mode == 2) {
                const double L = (double)R.L;
                if (R.vent_kind == 0) {
                    const double dx = dmin((double)p.x - R.vent_x, L), dy = dmin((double)p.y - R.vent_y, L);
                    in = dx * dx + dy * dy < R.vent_r * R.vent_r;
                } else if (R.vent_kind == 1) {
                    in = fabs(dmin((double)p.x - R.vent_x, L)) < 0.5 * R.vent_w;
                } else {
                    in = fabs(dmin((double)p.y - R.vent_y, L)) < 0.5 * R.vent_w;
                }
            }
            v = R.feed_mode != 0 && R.p_feed > 0.0 && t == 0 && in && cat_u01(kf, tg & GID_MASK) < R.p_feed;
            vn = t == 3;
        }
    }
    v = __reduce_add_sync(0xffffffffu, v);
    vn = __reduce_add_sync(0xffffffffu, vn);
    if (lane_id() == 0) red[threadIdx.x >> 5] = v | (vn << 16);
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0, sn = 0;
        for (int w = 0; w < BEAD_TPB / 32; w++) {
            s += red[w] & 0xFFFF;
            sn += red[w] >> 16;
        }
        b.cat_cnt[blockIdx.x] = s;
        b.cat_ncnt[blockIdx.x] = sn;
    }
}

// per chunk: its candidates written to the replica's list in slot order
__global__ void __launch_bounds__(BEAD_TPB) k_cat_list(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                       const Chunk *__restrict__ ch, int mode) {
    __shared__ int ws[BEAD_TPB / 32];
    __shared__ int pre;
    const Chunk c = ch[blockIdx.x];
    const RepDev &R = reps[c.rep];
    const long long step = *b.step;
    if (!cat_due(R, step) || b.cat_cnt[blockIdx.x] == 0) return;
    {  // candidates of the replica's earlier chunks, summed by the whole block
        int part = 0;
        for (int k = R.ch0 + (int)threadIdx.x; k < (int)blockIdx.x; k += BEAD_TPB) part += b.cat_cnt[k];
        part = __reduce_add_sync(0xffffffffu, part);
        if (lane_id() == 0) ws[threadIdx.x >> 5] = part;
        __syncthreads();
        if (threadIdx.x == 0) {
            int s = 0;
            for (int w = 0; w < BEAD_TPB / 32; w++) s += ws[w];
            pre = s;
        }
        __syncthreads();
    }
    const int d = c.begin + (int)threadIdx.x;
    int v = 0;
    if (d < c.end) {
        const uint32_t tg = b.tg[cur][d];
        const int t = (int)(tg >> TYPE_SHIFT);
        if (mode == 0) {
            v = t == 4 || t == 5;
        } else {
            const float2 p = b.pos[cur][d];
            const uint64_t kf = cat_key(R.seed, step, 14);
            bool in = true;
            if (R.feed_mode == 2) {
                const double L = (double)R.L;
                if (R.vent_kind == 0) {
                    const double dx = dmin((double)p.x - R.vent_x, L), dy = dmin((double)p.y - R.vent_y, L);
                    in = dx * dx + dy * dy < R.vent_r * R.vent_r;
                } else if (R.vent_kind == 1) {
                    in = fabs(dmin((double)p.x - R.vent_x, L)) < 0.5 * R.vent_w;
                } else {
                    in = fabs(dmin((double)p.y - R.vent_y, L)) < 0.5 * R.vent_w;
                }
            }
            v = R.feed_mode != 0 && R.p_feed > 0.0 && t == 0 && in && cat_u01(kf, tg & GID_MASK) < R.p_feed;
        }
    }
    const unsigned m = __ballot_sync(0xffffffffu, v);
    if (lane_id() == 0) ws[threadIdx.x >> 5] = __popc(m);
    __syncthreads();
    int before = pre;
    for (int w = 0; w < (int)(threadIdx.x >> 5); w++) before += ws[w];
    if (v) b.cat_list[R.b0 + before + __popc(m & ((1u << lane_id()) - 1u))] = d;
}

// The draws of one check (per replica): draw p is the output of T^p s0, s0
// the generator state at the check's start, T one step.  One thread per block
// of 64 draws starts at T^(64 m) s0 by the jump table (x^(64 m) mod the
// generator's characteristic polynomial, dpd_jump.cu), then steps.  The
// shuffle takes nk - 1 draws and the walk at most two per catalyst plus those
// of its events; 3 nk + 4096 draws are made (the walk goes on serially past
// them).  Block start states are kept for the walk's visits.
__global__ void __launch_bounds__(256) k_cat_stream(Bufs b, const RepDev *__restrict__ reps) {
    __shared__ int red[8];
    const int rep = (int)blockIdx.y;
    const RepDev &R = reps[rep];
    if (!cat_due(R, *b.step)) return;
    const int tid = (int)threadIdx.x;
    int n = 0;
    for (int k = tid; k < R.nch; k += 256) n += b.cat_cnt[R.ch0 + k];
    n = __reduce_add_sync(0xffffffffu, n);
    if (lane_id() == 0) red[tid >> 5] = n;
    __syncthreads();
    int nk = 0;
    for (int w = 0; w < 8; w++) nk += red[w];
    const long long D = min((long long)R.dcap, (3ll * nk + 4096 + 63) / 64 * 64);
    if (blockIdx.x == 0 && tid == 0) {
        b.cat_nk[rep] = nk;
        b.cat_dn[rep] = D;
    }
    uint64_t s0[4];
    for (int q = 0; q < 4; q++) s0[q] = b.rng[4 * rep + q];
    for (long long m = (long long)blockIdx.x * 256 + tid; m < D / 64; m += (long long)gridDim.x * 256) {
        const uint64_t *J = b.jump + 4 * m;
        uint64_t t[4] = {s0[0], s0[1], s0[2], s0[3]}, acc[4] = {0, 0, 0, 0};
        for (int w = 0; w < 4; w++) {
            const uint64_t jw = J[w];
            for (int bit = 0; bit < 64; bit++) {
                if ((jw >> bit) & 1) {
                    acc[0] ^= t[0];
                    acc[1] ^= t[1];
                    acc[2] ^= t[2];
                    acc[3] ^= t[3];
                }
                xo_next(t);
            }
        }
        uint64_t *bs = b.sblock + 4 * (R.so / 64 + m);
        for (int q = 0; q < 4; q++) bs[q] = acc[q];
        uint64_t *out = b.stream + R.so + 64 * m;
        for (int j = 0; j < 64; j++) out[j] = xo_next(acc);
    }
}

// the generator state at draw p of the replica's stream (p < its length)
__device__ __forceinline__ void state_at(const Bufs &b, const RepDev &R, long long p, uint64_t *s) {
    const uint64_t *bs = b.sblock + 4 * (R.so / 64 + p / 64);
    for (int q = 0; q < 4; q++) s[q] = __ldcg(bs + q);
    for (int k = 0; k < (int)(p % 64); k++) xo_next(s);
}

// the catalyst list of one replica shuffled as the serial generator does it
// (oercel.c:1571-1580): step i = nk-1 .. 1 swaps entries i and c_i =
// xo_below(i + 1) of draw nk-1-i.  The swaps are resolved in parallel: the
// entry that ends at position i >= 1 is the one that sat at c_i just before
// step i, i.e. the one the latest earlier step (the smallest m > i with
// c_m = c_i) moved there, else the original a[c_i]; what step m moved is the
// entry that sat at m just before step m, i.e. the one moved there by the
// smallest m' > m with c_m' = m, else a[m].  These "moved by" links point to
// larger steps, so pointer jumping resolves them in O(log nk) rounds.  Position
// 0 ends with what the smallest step m with c_m = 0 moved, else a[0].  The
// steps are grouped by partner (a stable order within each group comes from
// sorting the group, at most a few steps).
__device__ __forceinline__ int swap_partner(const uint64_t *st, int nk, int i) {
    const double u = (double)(__ldcg(st + (nk - 1 - i)) >> 11) * 0x1.0p-53;
    const long long k = (long long)(u * (double)(i + 1));
    return (int)(k >= i + 1 ? i : k);
}

__device__ __forceinline__ int block_excl_scan_1k(int v, int &total, int *ws) {
    const int lane = (int)lane_id(), w = (int)threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    __syncthreads();
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
        int t = ws[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        ws[lane] = t;  // inclusive sums of the warps
    }
    __syncthreads();
    total = ws[31];
    return (w > 0 ? ws[w - 1] : 0) + x - v;
}

__global__ void __launch_bounds__(1024) k_cat_shuffle(Bufs b, const RepDev *__restrict__ reps, int sh) {
    extern __shared__ int32_t shs[];
    __shared__ int ws[32];
    const int rep = (int)blockIdx.x;
    const RepDev &R = reps[rep];
    if (!cat_due(R, *b.step)) return;
    const int tid = (int)threadIdx.x, nk = b.cat_nk[rep];
    if (nk < 2) return;
    const uint64_t *st = b.stream + R.so;
    int32_t *list = b.cat_list + R.b0;
    // scratch of nk entries each, in shared memory while it fits: bucket starts, fill (later the
    // result), the steps sorted by partner, the next step with the same partner, the "moved by" link
    int32_t *cnt, *fill, *occ, *nxt, *lnk;
    if (nk <= sh) {  // the launch gave 5 sh entries of shared memory
        cnt = shs;
        fill = shs + sh;
        occ = shs + 2 * sh;
        nxt = shs + 3 * sh;
        lnk = shs + 4 * sh;
    } else {
        cnt = b.shuf + 0 * b.shuf_n + R.b0;
        fill = b.shuf + 1 * b.shuf_n + R.b0;
        occ = b.shuf + 2 * b.shuf_n + R.b0;
        nxt = b.shuf + 3 * b.shuf_n + R.b0;
        lnk = b.shuf + 4 * b.shuf_n + R.b0;
    }
    for (int p = tid; p < nk; p += 1024) {
        cnt[p] = 0;
        fill[p] = 0;
    }
    __syncthreads();
    for (int k = 1 + tid; k < nk; k += 1024) atomicAdd(cnt + swap_partner(st, nk, k), 1);
    __syncthreads();
    int base = 0;  // bucket starts: exclusive scan of cnt, in place
    for (int p0 = 0; p0 < nk; p0 += 1024) {
        const int p = p0 + tid, v = p < nk ? cnt[p] : 0;
        int tot;
        const int ex = block_excl_scan_1k(v, tot, ws);
        if (p < nk) cnt[p] = base + ex;
        base += tot;
    }
    __syncthreads();
    for (int k = 1 + tid; k < nk; k += 1024) {
        const int c = swap_partner(st, nk, k);
        occ[cnt[c] + atomicAdd(fill + c, 1)] = k;
    }
    __syncthreads();
    // each bucket in ascending step order; the next step of the same partner
    for (int p = tid; p < nk; p += 1024) {
        const int s0 = cnt[p], n = fill[p];
        for (int a = 1; a < n; a++) {
            const int t = occ[s0 + a];
            int c = a - 1;
            while (c >= 0 && occ[s0 + c] > t) {
                occ[s0 + c + 1] = occ[s0 + c];
                c--;
            }
            occ[s0 + c + 1] = t;
        }
        for (int a = 0; a < n; a++) nxt[occ[s0 + a]] = a + 1 < n ? occ[s0 + a + 1] : -1;
    }
    __syncthreads();
    // step k moved what the first step m > k with c_m = k had moved there, else a[k]
    for (int k = 1 + tid; k < nk; k += 1024) {
        int m = fill[k] > 0 ? occ[cnt[k]] : -1;  // the smallest step with partner k (>= k)
        if (m == k) m = nxt[k];
        lnk[k] = m;
    }
    __syncthreads();
    // what ends at position i: what the smallest step m > i with c_m = c_i moved (following the
    // links, which only go to larger steps), else a[c_i]; position 0 likewise with partner 0.
    // Into fill: only position 0 reads fill (fill[0], by the thread that writes it).
    for (int i = tid; i < nk; i += 1024) {
        int m, src;
        if (i == 0) {
            m = fill[0] > 0 ? occ[cnt[0]] : -1;
            src = 0;
        } else {
            m = nxt[i];
            src = swap_partner(st, nk, i);
        }
        for (int hop = 0; m >= 0 && hop < nk; hop++) {
            src = m;
            m = lnk[m];
        }
        fill[i] = list[src];
    }
    __syncthreads();
    for (int i = tid; i < nk; i += 1024) list[i] = fill[i];
}

// per catalyst (a warp each, its lanes over the cells of the search window):
// the N and W counts its searches will find (the candidate rules of find_near
// on the cell index of the last sort), its type and its cell.  Packed:
// nn | nw << 16 | Kb << 31 (counts saturate).  Grid: blockIdx.y = replica,
// the replica's blocks stride over its catalysts.
__global__ void __launch_bounds__(BEAD_TPB) k_cat_near(Bufs b, int cur, const RepDev *__restrict__ reps) {
    const int rep = (int)blockIdx.y;
    const RepDev &R = reps[rep];
    if (!cat_due(R, *b.step)) return;
    const int nk = b.cat_nk[rep], lane = (int)lane_id();
    const int rx = (int)ceil((R.r_cat + CAT_MARGIN) * R.icsx), ry = (int)ceil((R.r_cat + CAT_MARGIN) * R.icsy);
    const int ncol = 2 * rx + 1 >= R.ncx ? R.ncx : 2 * rx + 1, nrow = 2 * ry + 1 >= R.ncy ? R.ncy : 2 * ry + 1;
    const double L = (double)R.L, r2c = R.r_cat * R.r_cat;
    const int32_t *cs = b.cstart + R.c0;
    const int warps = (int)gridDim.x * (BEAD_TPB / 32);
    for (int q = (int)blockIdx.x * (BEAD_TPB / 32) + (int)(threadIdx.x >> 5); q < nk; q += warps) {
        const int k = b.cat_list[R.b0 + q];
        const float2 pk = b.pos[cur][k];
        const double xk = pk.x, yk = pk.y;
        int cx, cy;
        dcell(R, xk, yk, cx, cy);
        const int x0 = 2 * rx + 1 >= R.ncx ? 0 : cx - rx, y0 = 2 * ry + 1 >= R.ncy ? 0 : cy - ry;
        int nn = 0, nw = 0;
        for (int e = lane; e < ncol * nrow; e += 32) {
            int gx = x0 + e / nrow, gy = y0 + e % nrow;
            gx += gx < 0 ? R.ncx : (gx >= R.ncx ? -R.ncx : 0);
            gy += gy < 0 ? R.ncy : (gy >= R.ncy ? -R.ncy : 0);
            const int gc = gx * R.ncy + gy, end = cs[gc + 1];
            for (int j = cs[gc]; j < end; j++) {
                const int tj = (int)(b.tg[cur][j] >> TYPE_SHIFT);
                if ((tj != 3 && tj != 0) || j == k) continue;
                const float2 pj = b.pos[cur][j];
                const double dx = dmin((double)pj.x - xk, L), dy = dmin((double)pj.y - yk, L);
                if (dx * dx + dy * dy < r2c) {
                    nn += tj == 3;
                    nw += tj == 0;
                }
            }
        }
        nn = __reduce_add_sync(0xffffffffu, nn);
        nw = __reduce_add_sync(0xffffffffu, nw);
        if (lane == 0) {
            const int t = (int)(b.tg[cur][k] >> TYPE_SHIFT);
            b.cat_near[R.b0 + q] =
                (uint32_t)min(nn, 0x7FFF) | ((uint32_t)min(nw, 0x7FFF) << 16) | (t == 5 ? 0x80000000u : 0u);
            b.cat_cell[R.b0 + q] = R.c0 + cx * R.ncy + cy;
        }
    }
}

// One catalyst visit with the whole CTA (oercel.c:1582-1653): staging, the
// searches, synthesis and replication.  Thread 0 records in S.chg the old
// positions of the beads whose type it changed.
__device__ void visit(CatSmem &S, const Bufs &b, int cur, const RepDev &R, int rep, long long step, int k,
                      bool &overflow) {
    const int tid = (int)threadIdx.x, ml = R.lip_nH + R.lip_nT;
    const double L = (double)R.L;
    const dpd_template &M = b.mol[rep];
    if (tid == 0) {
        const int t = (int)(__ldcg(b.tg[cur] + k) >> TYPE_SHIFT);
        const float2 pk = __ldcg(b.pos[cur] + k);
        S.go = t == 4 || t == 5;
        S.var = t == 5;
        S.xk = pk.x;
        S.yk = pk.y;
        S.nchg = 0;
    }
    __syncthreads();
    if (!S.go) return;
    const int var = S.var;
    const double xk = S.xk, yk = S.yk;
    int cxk, cyk;
    dcell(R, xk, yk, cxk, cyk);
    if (!stage(S, b, cur, R, cxk, cyk)) {
        overflow = true;
        return;
    }
    find_near(S, R, k, xk, yk, R.r_cat, 3, S.nb, S.nbd, &S.nn);
    const int nn = S.nn;
    if (nn < 2) return;
    const int nsynN = R.syn_nN > 0 ? R.syn_nN : ml;
    if (nn >= nsynN && nsynN < ml) find_near(S, R, k, xk, yk, R.r_cat, 0, S.nbw, S.nbwd, &S.nw);
    else if (tid == 0) S.nw = 0;
    __syncthreads();
    const int nw = S.nw;
    int used = 0;
    if (tid == 0) S.go = nn >= nsynN && nsynN + nw >= ml && draw(S) < (var ? R.p_syn_b : R.p_syn_a);
    __syncthreads();
    if (S.go) {
        // synthesis: the nsynN nearest N, then the nearest W
        if (tid == 0) {
            double cxm = 0, cym = 0;
            for (int bb = 0; bb < ml; bb++) {
                const int i = bb < nsynN ? S.nb[bb] : S.nbw[bb - nsynN];
                S.sl[bb] = i;
                S.chg[bb] = S.pos[i];
                cxm += dmin((double)S.pos[i].x - xk, L);
                cym += dmin((double)S.pos[i].y - yk, L);
            }
            S.nchg = ml;
            S.cxm = xk + cxm / ml;
            S.cym = yk + cym / ml;
            S.ux = 1.0;
            S.uy = 0.0;
        }
        // the trial directions: consecutive draws, as in the reference's loop
        const int ntr = R.syn_tries;
        if (tid == 0)
            for (int tr = 0; tr < ntr; tr++) {
                const double phi = 2.0 * M_PI * draw(S);
                S.tux[tr] = cos(phi);
                S.tuy[tr] = sin(phi);
            }
        __syncthreads();
        if (ntr > 1) chain_energies(S, R, M, S.cxm, S.cym, ntr, ml);
        if (tid == 0) {  // the first lowest energy wins
            double ubest = INFINITY;
            for (int tr = 0; tr < ntr; tr++) {
                const double U = ntr > 1 ? S.tU[tr] : 0.0;
                if (U < ubest) {
                    ubest = U;
                    S.ux = S.tux[tr];
                    S.uy = S.tuy[tr];
                }
            }
        }
        __syncthreads();
        if (tid == 0) {
            double mvx = 0, mvy = 0, mtx = 0, mty = 0;
            for (int bb = 0; bb < ml; bb++) {
                const int g = S.slot[S.sl[bb]];
                const float2 vh = __ldcg(b.vh[cur] + g), vt = __ldcg(b.vt[cur] + g);
                mvx += vh.x;
                mvy += vh.y;
                mtx += vt.x;
                mty += vt.y;
            }
            mvx /= ml;
            mvy /= ml;
            mtx /= ml;
            mty /= ml;
            for (int bb = 0; bb < ml; bb++) {
                const int i = S.sl[bb], g = S.slot[i];
                place(R, M, bb, ml, S.cxm, S.cym, S.ux, S.uy, L, S.px[bb], S.py[bb]);
                b.vh[cur][g] = make_float2((float)mvx, (float)mvy);
                b.vt[cur][g] = make_float2((float)mtx, (float)mty);
                const int t = bb < R.lip_nH ? 1 : 2;
                set_type(b, cur, g, t);
                S.type[i] = (uint8_t)t;
                b.link[cur][g] = make_int2(bb > 0 ? S.slot[S.sl[bb - 1]] : -1,
                                           bb + 1 < ml ? S.slot[S.sl[bb + 1]] : -1);
            }
        }
        __syncthreads();
        if (R.syn_relax > 0) relax_chain(S, R, M, ml, overflow);
        if (tid == 0) {
            const float Lf = R.L;
            for (int bb = 0; bb < ml; bb++) {
                float x = (float)S.px[bb], y = (float)S.py[bb];
                x = x >= Lf ? 0.0f : x;
                y = y >= Lf ? 0.0f : y;
                b.pos[cur][S.slot[S.sl[bb]]] = make_float2(x, y);
            }
            push_event(b, step, EV_SYN, __ldcg(b.tg[cur] + k) & GID_MASK, (uint32_t)var, (float)xk, (float)yk, rep);
        }
        used = nsynN;
    }
    // replication onto the next two nearest N, with mutation
    if (tid == 0 && nn - used >= 2 && draw(S) < (var ? R.p_rep_b : R.p_rep_a)) {
        int nv = var, mut = 0;
        if (draw(S) < R.mu) {
            nv = 1 - var;
            mut = 1;
        }
        const int i1 = S.nb[used], i2 = S.nb[used + 1], g1 = S.slot[i1], g2 = S.slot[i2];
        set_type(b, cur, g1, nv ? 5 : 4);
        set_type(b, cur, g2, 0);
        S.chg[S.nchg++] = S.pos[i1];
        S.chg[S.nchg++] = S.pos[i2];
        push_event(b, step, mut ? EV_MUT : EV_REP, __ldcg(b.tg[cur] + g1) & GID_MASK, (uint32_t)nv, (float)xk,
                   (float)yk, rep);
    }
    __syncthreads();
}

// the walk's action for a catalyst from its packed counts and its cell mark
__device__ __forceinline__ uint8_t walk_code(uint32_t v, uint8_t dirty, int nsynN, int ml) {
    const int nn = (int)(v & 0x7FFF), nw = (int)((v >> 16) & 0x7FFF), var = (int)(v >> 31);
    int code;
    if (dirty || nn > CAT_MAXNB || nw > CAT_MAXNB) code = WALK_VISIT;
    else if (nn < 2) code = WALK_NONE;
    else {
        const int nwe = nn >= nsynN && nsynN < ml ? nw : 0;
        code = nn >= nsynN && nsynN + nwe >= ml ? WALK_SYN : WALK_REP;
    }
    return (uint8_t)(code | var << 2);
}

// The catalysts of one replica, one after the other in the shuffled order
// (oercel.c:1582-1655).  Most visits end without an event: their decisions
// need only the draws and the two candidate counts, which k_cat_near found
// before the walk.  A catalyst's draws are the next 0 (fewer than 2 N), 1
// (replication) or 2 (synthesis, replication) of the check's stream, so a
// block-wide prefix sum over a window of the walk gives every catalyst its
// draw positions and the decisions are made in parallel; the first catalyst
// whose draws give an event, or near which an earlier event changed a bead
// (cell marks), is visited by the whole CTA (visit(), from the generator state
// at its position), which counts the draws it takes, and the walk goes on
// after it.  Past the end of the stream, thread 0 walks on serially.  The
// draws, their order and every decision are those of visiting each catalyst
// in full.
__global__ void __launch_bounds__(CAT_TPB) k_cat_serial(Bufs b, int cur, const RepDev *__restrict__ reps) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    CatSmem &S = *reinterpret_cast<CatSmem *>(smem_raw);
    const int rep = (int)blockIdx.x;
    const RepDev &R = reps[rep];
    const long long step = *b.step;
    if (!cat_due(R, step)) return;
    const int tid = (int)threadIdx.x;
    const int ml = R.lip_nH + R.lip_nT, nsynN = R.syn_nN > 0 ? R.syn_nN : ml;
    const int nk = b.cat_nk[rep];
    const long long D = b.cat_dn[rep];
    const int32_t *list = b.cat_list + R.b0;
    const uint32_t *near = b.cat_near + R.b0;
    const int32_t *cell = b.cat_cell + R.b0;
    const uint64_t *st = b.stream + R.so;
    uint8_t *mark = b.cat_mark;
    const uint64_t tsyn[2] = {u01_threshold(R.p_syn_a), u01_threshold(R.p_syn_b)};
    const uint64_t trep[2] = {u01_threshold(R.p_rep_a), u01_threshold(R.p_rep_b)};
    // marking reach: the search radius in cells (a changed bead within r_cat of a
    // catalyst lies within rx cells of it), plus one
    const int mx = (int)ceil((R.r_cat + CAT_MARGIN) * R.icsx) + 1, my = (int)ceil((R.r_cat + CAT_MARGIN) * R.icsy) + 1;
    const int mcol = 2 * mx + 1 >= R.ncx ? R.ncx : 2 * mx + 1, mrow = 2 * my + 1 >= R.ncy ? R.ncy : 2 * my + 1;
    if (tid == 0) {
        S.over = 0;
        S.serial = 0;
        S.P = nk > 0 ? nk - 1 : 0;  // after the shuffle's draws
    }
    bool overflow = false;
    for (int w0 = 0; w0 < nk; w0 += CAT_WIN) {
        const int wn = min(CAT_WIN, nk - w0);
        __syncthreads();
        for (int i = tid; i < wn; i += CAT_TPB) {
            S.wk[i] = list[w0 + i];
            S.wcode[i] = walk_code(near[w0 + i], __ldcg(mark + cell[w0 + i]), nsynN, ml);
        }
        __syncthreads();
        int i = 0;
        while (true) {
            if (!S.serial) {
                // entries i .. wn-1: CAT_WIN / CAT_TPB consecutive ones per thread
                constexpr int PER = CAT_WIN / CAT_TPB;
                const int q0 = i + tid * PER;
                int nd[PER], tot = 0;
#pragma unroll
                for (int e = 0; e < PER; e++) {
                    const int q = q0 + e, kind = q < wn ? S.wcode[q] & 3 : WALK_NONE;
                    nd[e] = kind == WALK_SYN ? 2 : kind == WALK_REP ? 1 : 0;
                    tot += nd[e];
                }
                int total;
                long long pos = S.P + block_excl_scan(S, tot, total);
                if (tid == 0) {
                    S.first = wn;
                    S.exhaust = 0;
                }
                __syncthreads();
                int mine = wn;
                long long mpos = 0;
                bool mex = false;
#pragma unroll
                for (int e = 0; e < PER; e++) {
                    const int q = q0 + e;
                    if (q >= wn || mine < wn) break;
                    const int code = S.wcode[q], kind = code & 3, var = code >> 2;
                    bool stop = kind == WALK_VISIT;
                    if (!stop && nd[e] > 0) {
                        if (pos + 2 > D - 128) {
                            stop = true;
                            mex = true;
                        } else {
                            stop = (kind == WALK_SYN && (__ldcg(st + pos) >> 11) < tsyn[var]) ||
                                   (__ldcg(st + pos + (kind == WALK_SYN)) >> 11) < trep[var];
                        }
                    }
                    if (stop) {
                        mine = q;
                        mpos = pos;
                    }
                    pos += nd[e];
                }
                if (mine < wn) atomicMin(&S.first, mine);
                __syncthreads();
                if (mine < wn && mine == S.first) {
                    S.fpos = mpos;
                    S.exhaust = mex;
                }
                __syncthreads();
                i = S.first;
                if (i >= wn) {
                    if (tid == 0) S.P += total;
                    break;
                }
                if (tid == 0) {
                    state_at(b, R, S.fpos, S.rng);
                    S.nd = 0;
                    if (S.exhaust) S.serial = 1;
                }
                __syncthreads();
                if (S.serial) continue;  // walk on serially from catalyst i
            } else {
                if (tid == 0) {
                    uint64_t r[4] = {S.rng[0], S.rng[1], S.rng[2], S.rng[3]};
                    for (; i < wn; i++) {
                        const int code = S.wcode[i], kind = code & 3, var = code >> 2;
                        if (kind == WALK_NONE) continue;
                        if (kind == WALK_VISIT) break;
                        uint64_t t[4] = {r[0], r[1], r[2], r[3]};
                        if (kind == WALK_SYN && (xo_next(t) >> 11) < tsyn[var]) break;
                        if ((xo_next(t) >> 11) < trep[var]) break;
                        r[0] = t[0];
                        r[1] = t[1];
                        r[2] = t[2];
                        r[3] = t[3];
                    }
                    for (int q = 0; q < 4; q++) S.rng[q] = r[q];
                    S.k = i;
                }
                __syncthreads();
                i = S.k;
                if (i >= wn) break;
            }
            visit(S, b, cur, R, rep, step, S.wk[i], overflow);
            if (tid == 0 && !S.serial) S.P = S.fpos + S.nd;
            // mark the cells around the beads it changed; re-test the rest of the window
            const int nchg = S.nchg;
            if (nchg > 0) {
                for (int e = tid; e < nchg * mcol * mrow; e += CAT_TPB) {
                    const int c = e / (mcol * mrow), u = (e / mrow) % mcol, w = e % mrow;
                    int cx, cy;
                    dcell(R, (double)S.chg[c].x, (double)S.chg[c].y, cx, cy);
                    int gx = (2 * mx + 1 >= R.ncx ? 0 : cx - mx) + u, gy = (2 * my + 1 >= R.ncy ? 0 : cy - my) + w;
                    gx += gx < 0 ? R.ncx : (gx >= R.ncx ? -R.ncx : 0);
                    gy += gy < 0 ? R.ncy : (gy >= R.ncy ? -R.ncy : 0);
                    mark[R.c0 + gx * R.ncy + gy] = 1;
                }
                __syncthreads();
                for (int j = i + 1 + tid; j < wn; j += CAT_TPB)
                    if (__ldcg(mark + cell[w0 + j])) S.wcode[j] = (uint8_t)(WALK_VISIT | (S.wcode[j] & 4));
            }
            __syncthreads();
            i++;
        }
    }
    __syncthreads();
    if (tid == 0) {
        if (!S.serial) state_at(b, R, S.P, S.rng);
        for (int q = 0; q < 4; q++) b.rng[4 * rep + q] = S.rng[q];
    }
    if ((overflow || S.over) && tid == 0) raise_flag(b.status, DPD_F_CATALYST);
}

// ---------------------------------------------------------------- 2. decay (oercel.c:1658-1694)

__global__ void __launch_bounds__(BEAD_TPB) k_cat_decay(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                        const Chunk *__restrict__ ch) {
    const Chunk c = ch[blockIdx.x];
    const RepDev &R = reps[c.rep];
    const long long step = *b.step;
    if (!cat_due(R, step) || !(R.p_ld > 0 || R.p_kd > 0 || R.p_nd > 0)) return;
    const int d = c.begin + (int)threadIdx.x;
    if (d >= c.end) return;
    const uint32_t tg = b.tg[cur][d];
    const int t = (int)(tg >> TYPE_SHIFT);
    const uint32_t g = tg & GID_MASK;
    const int2 lk = b.link[cur][d];
    const bool head = lk.x < 0 && lk.y >= 0;
    const bool lip = head && R.p_ld > 0 && cat_u01(cat_key(R.seed, step, 11), g) < R.p_ld;
    const bool kat = (t == 4 || t == 5) && R.p_kd > 0 && cat_u01(cat_key(R.seed, step, 12), g) < R.p_kd;
    const bool nut = t == 3 && R.p_nd > 0 && cat_u01(cat_key(R.seed, step, 13), g) < R.p_nd;
    const float2 p = b.pos[cur][d];
    if (lip) {
        // the whole chain becomes W (no other thread touches its beads)
        const int ml = R.lip_nH + R.lip_nT;
        int cc = d, m = 0;
        while (cc >= 0 && m < ml) {
            const int nx = b.link[cur][cc].y;
            set_type(b, cur, cc, 0);
            b.link[cur][cc] = make_int2(-1, -1);
            cc = nx;
            m++;
        }
        push_event(b, step, EV_DLIP, g, 0xFFFFFFFFu, p.x, p.y, c.rep);
    } else if (kat) {
        set_type(b, cur, d, 0);
        push_event(b, step, EV_DK, g, t == 5 ? 1u : 0u, p.x, p.y, c.rep);
    } else if (nut) {
        set_type(b, cur, d, 0);
        push_event(b, step, EV_DN, g, 0xFFFFFFFFu, p.x, p.y, c.rep);
    }
}

// ---------------------------------------------------------------- 3. food supply (oercel.c:1721-1753)

// candidates in slot order (k_cat_list, mode 1); the cap keeps a random subset
__global__ void __launch_bounds__(CAT_TPB) k_cat_feed(Bufs b, int cur, const RepDev *__restrict__ reps) {
    __shared__ double red[2][CAT_WARPS];
    __shared__ long long keep;
    const int rep = (int)blockIdx.x;
    const RepDev &R = reps[rep];
    const long long step = *b.step;
    if (!cat_due(R, step) || R.feed_mode == 0 || !(R.p_feed > 0.0)) return;
    const int tid = (int)threadIdx.x;
    long long nc = 0, nN = 0;
    for (int k = tid; k < R.nch; k += CAT_TPB) {
        nc += b.cat_cnt[R.ch0 + k];
        nN += b.cat_ncnt[R.ch0 + k];
    }
    double a = (double)nc, z = (double)nN;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        z += __shfl_down_sync(0xffffffffu, z, o);
    }
    if (lane_id() == 0) {
        red[0][tid >> 5] = a;
        red[1][tid >> 5] = z;
    }
    __syncthreads();
    int32_t *list = b.cat_list + R.b0;
    if (tid == 0) {
        double sa = 0, sz = 0;
        for (int w = 0; w < CAT_WARPS; w++) {
            sa += red[0][w];
            sz += red[1][w];
        }
        const long long ncand = (long long)sa, nNt = (long long)sz;
        long long add = ncand;
        if (R.feed_cap > 0.0 && ncand > 0) {
            long long room = (long long)floor(R.feed_cap * (double)R.n + 1e-9) - nNt;
            if (room < 0) room = 0;
            if (add > room) {
                uint64_t s[4];
                for (int q = 0; q < 4; q++) s[q] = b.rng[4 * rep + q];
                for (long long c = 0; c < room; c++) {  // partial Fisher-Yates: a random subset of size room
                    const long long d = c + xo_below(s, ncand - c);
                    const int t = list[c];
                    list[c] = list[d];
                    list[d] = t;
                }
                for (int q = 0; q < 4; q++) b.rng[4 * rep + q] = s[q];
                add = room;
            }
        }
        keep = add;
        if (add > 0) push_event(b, step, EV_FEED, (uint32_t)add, 0xFFFFFFFFu, __int_as_float(0x7fc00000),
                                __int_as_float(0x7fc00000), rep);
    }
    __syncthreads();
    for (long long c = tid; c < keep; c += CAT_TPB) set_type(b, cur, list[c], 3);
}

// ---------------------------------------------------------------- launch

int catalyst_setup() {
    cudaError_t e =
        cudaFuncSetAttribute(k_cat_serial, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(CatSmem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_cat_shuffle, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 CAT_SHUF_SH * 5 * (int)sizeof(int32_t));

    return e == cudaSuccess ? 0 : -1;
}

void launch_catalyst(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, int nrep, int64_t C,
                     int nmax, int stream_grid, cudaStream_t s) {
    k_cat_count<<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch, 0);
    k_cat_list<<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch, 0);
    k_cat_stream<<<dim3(stream_grid, nrep), 256, 0, s>>>(b, rep);
    const int sh = std::min(nmax, CAT_SHUF_SH);
    k_cat_shuffle<<<nrep, 1024, (size_t)sh * 5 * sizeof(int32_t), s>>>(b, rep, sh);
    k_cat_near<<<dim3(std::max(1, 148 * 8 / nrep), nrep), BEAD_TPB, 0, s>>>(b, cur, rep);
    cudaMemsetAsync(b.cat_mark, 0, (size_t)C, s);
    k_cat_serial<<<nrep, CAT_TPB, sizeof(CatSmem), s>>>(b, cur, rep);
    k_cat_decay<<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch);
    k_cat_count<<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch, 1);
    k_cat_list<<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch, 1);
    k_cat_feed<<<nrep, CAT_TPB, 0, s>>>(b, cur, rep);
}
