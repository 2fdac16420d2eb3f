// dpd_chem.cu -- the lipid chemistry pass (sm_100a).
//
// Three stages per chemistry step, each decided on the state the previous
// stage left (kernel boundaries), every decision a keyed Philox draw of
// (seed, step, salt, gid) -- the reference's counter-based mechanism
// (cel/engine/oercel.c:819-826) -- and every conflict resolved by the lowest
// requesting gid (atomicMin claim, then a check by each requester; the
// reference GPU port resolves its lock rounds the same way, lowest rank wins,
// cel/engine_gpu/oercel_gpu.cu:1746-1757).  The draws do not depend on the
// state, so one pass over the beads (fused into the permute kernel of the step,
// or k_chem_scan for the phase entry point) applies the breaks and lists the
// few beads whose growth or bonding draw succeeded; the later stages run over
// those lists only.
//   1 brk : an H whose next bead is T breaks the bond with p_break;
//   2 grow: a P with >= n_t_min T beads within r_grow, with p_grow, becomes a
//           T bonded behind its nearest growable H-terminated chain end
//           (the tail of a chain headed by H and shorter than max_chain, or a
//           lone H) within r_grow;
//   3 bond: a free T, with p_bond, bonds to its nearest free H within r_bond.
// Nearest = smallest squared FP32 distance, ties to the lower gid
// (oercel.c:1387-1396).
#include "dpd_chem.cuh"

// stage 1 on a sorted state in place (the phase entry point dpd_chemistry)
__global__ void __launch_bounds__(BEAD_TPB) k_chem_scan(Bufs b, int cur, const RepDev *__restrict__ reps,
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
    const int t = link[d].y;
    if (type_of(t0) == T_H && t >= 0 && h_breaks(R, step, t0, tg[t])) {
        link[d].y = -1;
        link[t].x = -1;
        const float2 p = b.pos[cur][d];
        push_event(b, step, 1, t0 & GID_MASK, tg[t] & GID_MASK, p.x, p.y, c.rep);
    }
    chem_candidate(b, R, step, c.rep, d, t0);
}

// tail end e of a chain headed by H that is shorter than max_chain, or a lone H
__device__ bool growable_end(const uint32_t *tg, const int2 *link, int e, int max_chain) {
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

// the 3x3 cells around position pi as contiguous slot ranges: per column the
// rows cy-1..cy+1 are one range, or two where the rows wrap
struct NbrRanges {
    int s[6], e[6];
    int n, total;
};

__device__ __forceinline__ NbrRanges nbr_ranges(const Bufs &b, const RepDev &R, float2 pi) {
    NbrRanges q;
    const int ncx = R.ncx, ncy = R.ncy;
    const int32_t *cs = b.cstart + R.c0;
    int cx, cy;
    cell_xy(R, pi.x, pi.y, cx, cy);
    q.n = 0;
    q.total = 0;
#pragma unroll
    for (int ox = -1; ox <= 1; ox++) {
        const int col = ((cx + ox + ncx) % ncx) * ncy;
        if (cy >= 1 && cy + 1 < ncy) {
            q.s[q.n] = cs[col + cy - 1];
            q.e[q.n++] = cs[col + cy + 2];
        } else if (cy == 0) {
            q.s[q.n] = cs[col + ncy - 1];
            q.e[q.n++] = cs[col + ncy];
            q.s[q.n] = cs[col];
            q.e[q.n++] = cs[col + 2];
        } else {
            q.s[q.n] = cs[col + cy - 1];
            q.e[q.n++] = cs[col + ncy];
            q.s[q.n] = cs[col];
            q.e[q.n++] = cs[col + 1];
        }
    }
    for (int k = 0; k < q.n; k++) q.total += q.e[k] - q.s[k];
    return q;
}

// slot of the f-th bead of the ranges
__device__ __forceinline__ int nbr_slot(const NbrRanges &q, int f) {
    int k = 0;
    while (f >= q.e[k] - q.s[k]) {
        f -= q.e[k] - q.s[k];
        k++;
    }
    return q.s[k] + f;
}

// warp minimum of a 64-bit key (distance bits, gid): the lexicographic nearest
__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}

#define LIST_GRID 148
#define NONE_KEY 0xFFFFFFFFFFFFFFFFull

// stage 2 requests, one warp per listed P: it needs >= n_t_min T beads within
// r_grow and claims its nearest growable end within r_grow (req[k] = end or -1)
__global__ void __launch_bounds__(BEAD_TPB) k_chem_grow_req(Bufs b, int cur, const RepDev *__restrict__ reps) {
    const int n = (int)b.status->n_grow;
    const uint32_t *tg = b.tg[cur];
    const float2 *pos = b.pos[cur];
    const int2 *link = b.link[cur];
    const int lane = (int)lane_id();
    const int nw = (int)(gridDim.x * blockDim.x) >> 5;
    for (int k = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); k < n; k += nw) {
        const int2 it = b.grow_list[k];
        const int d = it.x;
        const RepDev &R = reps[it.y];
        const float2 pi = pos[d];
        const float L = R.L, h = R.halfL, r2 = R.r2_grow;
        const NbrRanges q = nbr_ranges(b, R, pi);
        int nt = 0;
        unsigned long long best = NONE_KEY;
        for (int f = lane; f < q.total; f += 32) {
            const int j = nbr_slot(q, f);
            if (j == d) continue;
            const float2 pj = pos[j];
            const float dd = dist2(pi.x, pi.y, pj.x, pj.y, L, h);
            if (!(dd < r2)) continue;
            const uint32_t tj = tg[j];
            nt += type_of(tj) == T_T;
            const unsigned long long key = ((unsigned long long)__float_as_uint(dd) << 32) | (tj & GID_MASK);
            if (key < best && growable_end(tg, link, j, R.max_chain)) best = key;
        }
        nt = (int)__reduce_add_sync(0xffffffffu, (unsigned)nt);
        best = warp_min_u64(best);
        int e = -1;
        if (nt >= R.n_t_min && best != NONE_KEY) {
            // the slot of the winning end: the lane that holds it reports it
            for (int f = lane; f < q.total; f += 32) {
                const int j = nbr_slot(q, f);
                if (j != d && (tg[j] & GID_MASK) == (uint32_t)(best & 0xFFFFFFFFu)) e = j;
            }
            e = (int)__reduce_max_sync(0xffffffffu, (unsigned)(e + 1)) - 1;
        }
        if (lane == 0) {
            b.req[k] = e;
            if (e >= 0) atomicMin(b.claim + e, tg[d] & GID_MASK);
        }
    }
}

// stage 2 application, one thread per listed P: the lowest claiming gid wins its end
__global__ void __launch_bounds__(BEAD_TPB) k_chem_grow_apply(Bufs b, int cur, const RepDev *__restrict__ reps) {
    const int n = (int)b.status->n_grow;
    const long long step = *b.step;
    uint32_t *tg = b.tg[cur];
    int2 *link = b.link[cur];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int e = b.req[k];
        if (e < 0) continue;
        const int2 it = b.grow_list[k];
        const int d = it.x;
        const uint32_t g = tg[d] & GID_MASK;
        if (b.claim[e] != g) continue;  // a lower gid claimed this end
        b.claim[e] = 0xFFFFFFFFu;
        tg[d] = ((uint32_t)T_T << TYPE_SHIFT) | g;
        link[d] = make_int2(e, -1);
        link[e].y = d;
        const float2 p = b.pos[cur][d];
        push_event(b, step, 0, g, tg[e] & GID_MASK, p.x, p.y, it.y);
    }
}

// stage 3 requests, one warp per listed T: if still free it claims its nearest
// free H within r_bond
__global__ void __launch_bounds__(BEAD_TPB) k_chem_bond_req(Bufs b, int cur, const RepDev *__restrict__ reps) {
    const int n = (int)b.status->n_bond;
    const uint32_t *tg = b.tg[cur];
    const float2 *pos = b.pos[cur];
    const int2 *link = b.link[cur];
    const int lane = (int)lane_id();
    const int nw = (int)(gridDim.x * blockDim.x) >> 5;
    for (int k = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); k < n; k += nw) {
        const int2 it = b.bond_list[k];
        const int d = it.x;
        const int2 lk = link[d];
        int e = -1;
        if (type_of(tg[d]) == T_T && lk.x < 0 && lk.y < 0) {
            const RepDev &R = reps[it.y];
            const float2 pi = pos[d];
            const float L = R.L, h = R.halfL, r2 = R.r2_bond;
            const NbrRanges q = nbr_ranges(b, R, pi);
            unsigned long long best = NONE_KEY;
            int bj = -1;
            for (int f = lane; f < q.total; f += 32) {
                const int j = nbr_slot(q, f);
                if (j == d) continue;
                const uint32_t tj = tg[j];
                if (type_of(tj) != T_H) continue;
                const int2 lj = link[j];
                if (lj.x >= 0 || lj.y >= 0) continue;
                const float2 pj = pos[j];
                const float dd = dist2(pi.x, pi.y, pj.x, pj.y, L, h);
                if (!(dd < r2)) continue;
                const unsigned long long key = ((unsigned long long)__float_as_uint(dd) << 32) | (tj & GID_MASK);
                if (key < best) {
                    best = key;
                    bj = j;
                }
            }
            const unsigned long long wbest = warp_min_u64(best);
            const int mine = (best == wbest && wbest != NONE_KEY) ? bj : -1;
            e = (int)__reduce_max_sync(0xffffffffu, (unsigned)(mine + 1)) - 1;
        }
        if (lane == 0) {
            b.req[k] = e;
            if (e >= 0) atomicMin(b.claim + e, tg[d] & GID_MASK);
        }
    }
}

__global__ void __launch_bounds__(BEAD_TPB) k_chem_bond_apply(Bufs b, int cur, const RepDev *__restrict__ reps) {
    const int n = (int)b.status->n_bond;
    const long long step = *b.step;
    const uint32_t *tg = b.tg[cur];
    int2 *link = b.link[cur];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int h = b.req[k];
        if (h < 0) continue;
        const int2 it = b.bond_list[k];
        const int d = it.x;
        const uint32_t g = tg[d] & GID_MASK;
        if (b.claim[h] != g) continue;
        b.claim[h] = 0xFFFFFFFFu;
        link[h].y = d;
        link[d].x = h;
        const float2 p = b.pos[cur][d];
        push_event(b, step, 2, g, tg[h] & GID_MASK, p.x, p.y, it.y);
    }
}

int chem_kernel_count() { return 4; }

void launch_chem_scan(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, cudaStream_t s) {
    k_chem_scan<<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch);
}

void launch_chem_lists(const Bufs &b, int cur, const RepDev *rep, int part, cudaStream_t s) {
    if (part < 0 || part == 0) k_chem_grow_req<<<LIST_GRID, BEAD_TPB, 0, s>>>(b, cur, rep);
    if (part < 0 || part == 1) k_chem_grow_apply<<<LIST_GRID, BEAD_TPB, 0, s>>>(b, cur, rep);
    if (part < 0 || part == 2) k_chem_bond_req<<<LIST_GRID, BEAD_TPB, 0, s>>>(b, cur, rep);
    if (part < 0 || part == 3) k_chem_bond_apply<<<LIST_GRID, BEAD_TPB, 0, s>>>(b, cur, rep);
}
