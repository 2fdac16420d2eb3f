// dpd_chem.cu -- the lipid chemistry pass (sm_100a).
//
// Three stages per chemistry step, each decided on the state the previous
// stage left (kernel boundaries), every decision a keyed Philox draw of
// (seed, step, salt, gid) -- the reference's counter-based mechanism
// (cel/engine/oercel.c:819-826) -- and every conflict resolved by the lowest
// requesting gid (atomicMin claim, then a check by each requester; the
// reference GPU port resolves its lock rounds the same way, lowest rank wins,
// cel/engine_gpu/oercel_gpu.cu:1746-1757):
//   1 brk : an H whose next bead is T breaks the bond with p_break;
//   2 grow: a P with >= n_t_min T beads within r_grow, with p_grow, becomes a
//           T bonded behind its nearest growable H-terminated chain end
//           (the tail of a chain headed by H and shorter than max_chain, or a
//           lone H) within r_grow;
//   3 bond: a free T, with p_bond, bonds to its nearest free H within r_bond.
// Nearest = smallest squared FP32 distance, ties to the lower gid
// (oercel.c:1387-1396).
#include "dpd_device.cuh"

#define T_W 0
#define T_H 1
#define T_T 2
#define T_P 3
#define SALT_BREAK 1u
#define SALT_GROW 2u
#define SALT_BOND 3u

__device__ __forceinline__ bool chem_due(const RepDev &R, long long step) {
    return R.chem && R.n_chem > 0 && (step % R.n_chem) == 0;
}

__device__ __forceinline__ int type_of(uint32_t tg) { return (int)(tg >> TYPE_SHIFT); }

__device__ __forceinline__ float dist2(float xa, float ya, float xb, float yb, float L, float h) {
    const float dx = minimg(__fsub_rn(xb, xa), L, h), dy = minimg(__fsub_rn(yb, ya), L, h);
    return __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
}

__device__ void push_event(const Bufs &b, long long step, int kind, uint32_t gid, uint32_t partner, float x, float y,
                           int rep) {
    const unsigned k = atomicAdd(&b.status->nevents, 1u);
    if ((int)k < b.evcap) {
        EventDev e;
        e.step = step;
        e.kind = kind;
        e.gid = gid;
        e.partner = partner;
        e.x = x;
        e.y = y;
        e.replica = rep;
        b.events[k] = e;
    } else {
        raise_flag(b.status, DPD_F_EVENTS);
    }
}

// tail end e of a chain headed by H that is shorter than max_chain, or a lone H
__device__ bool growable_end(const uint32_t *tg, const int2 *link, int e, int max_chain, DevStatus *st) {
    const int2 le = link[e];
    if (le.y >= 0) return false;
    const int te = type_of(tg[e]);
    if (te == T_H) return le.x < 0;
    if (te != T_T || le.x < 0) return false;
    int len = 1, c = e;
    while (true) {
        const int p = link[c].x;
        if (p < 0) break;
        c = p;
        len++;
        if (len > max_chain) return false;  // chain already full (or a loop): not growable
    }
    return type_of(tg[c]) == T_H && len < max_chain;
}

__global__ void __launch_bounds__(BEAD_TPB) k_chem_break(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                         const Chunk *__restrict__ ch) {
    const Chunk c = ch[blockIdx.x];
    const RepDev &R = reps[c.rep];
    const long long step = *b.step;
    if (!chem_due(R, step)) return;
    const int d = c.begin + (int)threadIdx.x;
    if (d >= c.end) return;
    const uint32_t *tg = b.tg[cur];
    int2 *link = b.link[cur];
    const uint32_t t0 = tg[d];
    if (type_of(t0) != T_H) return;
    const int t = link[d].y;
    if (t < 0 || type_of(tg[t]) != T_T) return;
    if (decision_word(R, step, SALT_BREAK, t0 & GID_MASK) >= R.thr_break) return;
    link[d].y = -1;
    link[t].x = -1;
    const float2 p = b.pos[cur][d];
    push_event(b, step, 1, t0 & GID_MASK, tg[t] & GID_MASK, p.x, p.y, c.rep);
}

// the 3x3 cells around bead d: calls body(j) for every other bead j
template <typename F>
__device__ __forceinline__ void for_neighbours(const Bufs &b, const RepDev &R, float2 pi, F body) {
    const int ncx = R.ncx, ncy = R.ncy;
    const int32_t *cs = b.cstart + R.c0;
    int cx, cy;
    cell_xy(R, pi.x, pi.y, cx, cy);
    for (int ox = -1; ox <= 1; ox++) {
        const int nx = (cx + ox + ncx) % ncx;
        for (int oy = -1; oy <= 1; oy++) {
            const int cc = nx * ncy + (cy + oy + ncy) % ncy;
            for (int j = cs[cc]; j < cs[cc + 1]; j++) body(j);
        }
    }
}

__global__ void __launch_bounds__(BEAD_TPB) k_chem_grow_req(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                            const Chunk *__restrict__ ch) {
    const Chunk c = ch[blockIdx.x];
    const RepDev &R = reps[c.rep];
    const long long step = *b.step;
    if (!chem_due(R, step)) return;
    const int d = c.begin + (int)threadIdx.x;
    if (d >= c.end) return;
    b.req[d] = -1;
    const uint32_t *tg = b.tg[cur];
    const uint32_t t0 = tg[d];
    if (type_of(t0) != T_P) return;
    const uint32_t g = t0 & GID_MASK;
    if (decision_word(R, step, SALT_GROW, g) >= R.thr_grow) return;
    const float2 *pos = b.pos[cur];
    const int2 *link = b.link[cur];
    const float2 pi = pos[d];
    const float L = R.L, h = R.halfL, r2 = R.r2_grow;
    int nt = 0;
    for_neighbours(b, R, pi, [&](int j) {
        if (j != d && type_of(tg[j]) == T_T) {
            const float2 pj = pos[j];
            if (dist2(pi.x, pi.y, pj.x, pj.y, L, h) < r2) nt++;
        }
    });
    if (nt < R.n_t_min) return;
    int best = -1;
    float bd = 0.0f;
    uint32_t bg = 0;
    for_neighbours(b, R, pi, [&](int j) {
        if (j == d) return;
        const float2 pj = pos[j];
        const float q = dist2(pi.x, pi.y, pj.x, pj.y, L, h);
        if (!(q < r2)) return;
        const uint32_t gj = tg[j] & GID_MASK;
        if (best >= 0 && !(q < bd || (q == bd && gj < bg))) return;
        if (!growable_end(tg, link, j, R.max_chain, b.status)) return;
        best = j;
        bd = q;
        bg = gj;
    });
    if (best < 0) return;
    b.req[d] = best;
    atomicMin(b.claim + best, g);
}

__global__ void __launch_bounds__(BEAD_TPB) k_chem_grow_apply(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                              const Chunk *__restrict__ ch) {
    const Chunk c = ch[blockIdx.x];
    const RepDev &R = reps[c.rep];
    const long long step = *b.step;
    if (!chem_due(R, step)) return;
    const int d = c.begin + (int)threadIdx.x;
    if (d >= c.end) return;
    const int e = b.req[d];
    if (e < 0) return;
    uint32_t *tg = b.tg[cur];
    const uint32_t g = tg[d] & GID_MASK;
    if (b.claim[e] != g) return;  // a lower gid claimed this end
    b.claim[e] = 0xFFFFFFFFu;
    int2 *link = b.link[cur];
    tg[d] = ((uint32_t)T_T << TYPE_SHIFT) | g;
    link[d] = make_int2(e, -1);
    link[e].y = d;
    const float2 p = b.pos[cur][d];
    push_event(b, step, 0, g, tg[e] & GID_MASK, p.x, p.y, c.rep);
}

__global__ void __launch_bounds__(BEAD_TPB) k_chem_bond_req(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                            const Chunk *__restrict__ ch) {
    const Chunk c = ch[blockIdx.x];
    const RepDev &R = reps[c.rep];
    const long long step = *b.step;
    if (!chem_due(R, step)) return;
    const int d = c.begin + (int)threadIdx.x;
    if (d >= c.end) return;
    b.req[d] = -1;
    const uint32_t *tg = b.tg[cur];
    const int2 *link = b.link[cur];
    const uint32_t t0 = tg[d];
    if (type_of(t0) != T_T) return;
    const int2 lk = link[d];
    if (lk.x >= 0 || lk.y >= 0) return;
    const uint32_t g = t0 & GID_MASK;
    if (decision_word(R, step, SALT_BOND, g) >= R.thr_bond) return;
    const float2 *pos = b.pos[cur];
    const float2 pi = pos[d];
    const float L = R.L, h = R.halfL, r2 = R.r2_bond;
    int best = -1;
    float bd = 0.0f;
    uint32_t bg = 0;
    for_neighbours(b, R, pi, [&](int j) {
        if (j == d) return;
        const uint32_t tj = tg[j];
        if (type_of(tj) != T_H) return;
        const int2 lj = link[j];
        if (lj.x >= 0 || lj.y >= 0) return;
        const float2 pj = pos[j];
        const float q = dist2(pi.x, pi.y, pj.x, pj.y, L, h);
        if (!(q < r2)) return;
        const uint32_t gj = tj & GID_MASK;
        if (best >= 0 && !(q < bd || (q == bd && gj < bg))) return;
        best = j;
        bd = q;
        bg = gj;
    });
    if (best < 0) return;
    b.req[d] = best;
    atomicMin(b.claim + best, g);
}

__global__ void __launch_bounds__(BEAD_TPB) k_chem_bond_apply(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                              const Chunk *__restrict__ ch) {
    const Chunk c = ch[blockIdx.x];
    const RepDev &R = reps[c.rep];
    const long long step = *b.step;
    if (!chem_due(R, step)) return;
    const int d = c.begin + (int)threadIdx.x;
    if (d >= c.end) return;
    const int h = b.req[d];
    if (h < 0) return;
    const uint32_t *tg = b.tg[cur];
    const uint32_t g = tg[d] & GID_MASK;
    if (b.claim[h] != g) return;
    b.claim[h] = 0xFFFFFFFFu;
    int2 *link = b.link[cur];
    link[h].y = d;
    link[d].x = h;
    const float2 p = b.pos[cur][d];
    push_event(b, step, 2, g, tg[h] & GID_MASK, p.x, p.y, c.rep);
}

int chem_kernel_count() { return 5; }

void launch_chemistry_part(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, int part,
                           cudaStream_t s) {
    switch (part) {
    case 0: k_chem_break<<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch); break;
    case 1: k_chem_grow_req<<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch); break;
    case 2: k_chem_grow_apply<<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch); break;
    case 3: k_chem_bond_req<<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch); break;
    default: k_chem_bond_apply<<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch); break;
    }
}

void launch_chemistry(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, cudaStream_t s) {
    for (int k = 0; k < chem_kernel_count(); k++) launch_chemistry_part(b, cur, rep, bch, nbch, k, s);
}
