// dpd_chem.cuh -- device functions of the chemistry pass shared by the permute
// kernel (which runs stage 1 of every chemistry step) and dpd_chem.cu.
#pragma once
#include "dpd_device.cuh"

#define T_W 0
#define T_H 1
#define T_T 2
#define T_P 3
#define SALT_BREAK 1u
#define SALT_GROW 2u
#define SALT_BOND 3u

// the lipid chemistry (chem_kind 0) is due at this step
__device__ __forceinline__ bool chem_due(const RepDev &R, long long step) {
    return R.chem && R.chem_kind == 0 && R.n_chem > 0 && (step % R.n_chem) == 0;
}

// the reference's catalyst chemistry (chem_kind 1) is due at this step
__device__ __forceinline__ bool cat_due(const RepDev &R, long long step) {
    return R.chem && R.chem_kind == 1 && R.n_chem > 0 && (step % R.n_chem) == 0;
}

__device__ __forceinline__ int type_of(uint32_t tg) { return (int)(tg >> TYPE_SHIFT); }

__device__ __forceinline__ float dist2(float xa, float ya, float xb, float yb, float L, float h) {
    const float dx = minimg(__fsub_rn(xb, xa), L, h), dy = minimg(__fsub_rn(yb, ya), L, h);
    return __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
}

__device__ __forceinline__ void push_event(const Bufs &b, long long step, int kind, uint32_t gid, uint32_t partner, float x, float y,
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

// does the H bead (tg_h) break its bond to the T bead (tg_t) at this step
__device__ __forceinline__ bool h_breaks(const RepDev &R, long long step, uint32_t tg_h, uint32_t tg_t) {
    return type_of(tg_h) == T_H && type_of(tg_t) == T_T &&
           decision_word(R, step, SALT_BREAK, tg_h & GID_MASK) < R.thr_break;
}

// list the bead if its growth (P) or bonding (T) draw succeeds
__device__ __forceinline__ void chem_candidate(const Bufs &b, const RepDev &R, long long step, int rep, int d,
                                               uint32_t tg) {
    const int ty = type_of(tg);
    const uint32_t g = tg & GID_MASK;
    if (ty == T_P) {
        if (decision_word(R, step, SALT_GROW, g) < R.thr_grow) b.grow_list[atomicAdd(&b.status->n_grow, 1u)] = make_int2(d, rep);
    } else if (ty == T_T) {
        if (decision_word(R, step, SALT_BOND, g) < R.thr_bond) b.bond_list[atomicAdd(&b.status->n_bond, 1u)] = make_int2(d, rep);
    }
}

// stage 1 for new slot d inside the permute of a step (links already remapped
// to new slots in *nl): the H side drops its next and logs the event, the T
// side drops its prev; both evaluate the same draw (the H bead's).  Each lane
// makes at most two draws, each at one call site, so a warp runs the Philox
// rounds at most twice whatever its mix of bead types.
__device__ __forceinline__ void chem_in_permute(const Bufs &b, int cur, const RepDev &R, long long step, int rep, int d, float2 p,
                                uint32_t tg, int2 lk_old, int2 &nl) {
    const uint32_t *tg_old = b.tg[cur];
    const int ty = type_of(tg);
    const uint32_t g = tg & GID_MASK;
    // the H-T bond this bead is part of, if any: its H bead's gid decides
    uint32_t hgid = 0, partner = 0;
    int side = 0;  // 1: this bead is the H, 2: this bead is the T
    if (ty == T_H && lk_old.y >= 0) {
        partner = tg_old[lk_old.y];
        if (type_of(partner) == T_T) {
            side = 1;
            hgid = g;
        }
    } else if (ty == T_T && lk_old.x >= 0) {
        partner = tg_old[lk_old.x];
        if (type_of(partner) == T_H) {
            side = 2;
            hgid = partner & GID_MASK;
        }
    }
    if (side != 0 && decision_word(R, step, SALT_BREAK, hgid) < R.thr_break) {
        if (side == 1) {
            nl.y = -1;
            push_event(b, step, 1, g, partner & GID_MASK, p.x, p.y, rep);
        } else {
            nl.x = -1;
        }
    }
    // the growth (P) or bonding (T) draw; only a free T can bond (nothing in the
    // later stages of the step gives a free T a link before its bond request)
    if (ty == T_P || (ty == T_T && nl.x < 0 && nl.y < 0)) {
        const bool grow = ty == T_P;
        if (decision_word(R, step, grow ? SALT_GROW : SALT_BOND, g) < (grow ? R.thr_grow : R.thr_bond)) {
            if (grow) b.grow_list[atomicAdd(&b.status->n_grow, 1u)] = make_int2(d, rep);
            else b.bond_list[atomicAdd(&b.status->n_bond, 1u)] = make_int2(d, rep);
        }
    }
}

// tail end e of a chain headed by H that is shorter than max_chain, or a lone H
__device__ __forceinline__ bool growable_end(const uint32_t *tg, const int2 *link, int e, int max_chain) {
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


#define NONE_LIST_KEY 0xFFFFFFFFFFFFFFFFull

// a bead that could be a growable end, judged from itself alone: a lone H,
// or a T with a prev and no next (growable_end then walks its chain)
__device__ __forceinline__ bool maybe_end(uint32_t tj, int2 lj) {
    if (lj.y >= 0) return false;
    const int t = type_of(tj);
    return t == T_H ? lj.x < 0 : (t == T_T && lj.x >= 0);
}

#define GROW_KEEP 4  // candidate ends a lane keeps in registers (32 x 4 = 128 beads in the 3x3 cells)

// stage 2 request of list entry k, by one whole warp: the listed P needs
// >= n_t_min T beads within r_grow and claims its nearest growable end within
// r_grow (req[k] = end or -1).  Each lane keeps the possible ends among its
// candidates; the warp then takes them in increasing (distance, gid) order and
// walks the chain of one at a time, so that usually a single walk decides.
__device__ __forceinline__ void chem_grow_req_one(const Bufs &b, int cur, const RepDev *__restrict__ reps, int k,
                                                  int lane) {
    const uint32_t *tg = b.tg[cur];
    const float2 *pos = b.pos[cur];
    const int2 *link = b.link[cur];
    const int2 it = b.grow_list[k];
    const int d = it.x;
    const RepDev &R = reps[it.y];
    const float2 pi = pos[d];
    const float L = R.L, h = R.halfL, r2 = R.r2_grow;
    const NbrRanges q = nbr_ranges(b, R, pi);
    int nt = 0;
    unsigned long long key[GROW_KEEP];
    int slot[GROW_KEEP];
#pragma unroll
    for (int m = 0; m < GROW_KEEP; m++) {
        key[m] = NONE_LIST_KEY;
        slot[m] = -1;
    }
    const bool kept = q.total <= 32 * GROW_KEEP;
    unsigned long long best = NONE_LIST_KEY;  // the exhaustive path (a crowded neighbourhood)
    int bj = -1;
#pragma unroll
    for (int m = 0; m < GROW_KEEP; m++) {
        const int f = lane + 32 * m;
        if (f >= q.total) break;
        const int j = nbr_slot(q, f);
        if (j == d) continue;
        const float2 pj = pos[j];
        const float dd = dist2(pi.x, pi.y, pj.x, pj.y, L, h);
        if (!(dd < r2)) continue;
        const uint32_t tj = tg[j];
        nt += type_of(tj) == T_T;
        if (maybe_end(tj, link[j])) {
            key[m] = ((unsigned long long)__float_as_uint(dd) << 32) | (tj & GID_MASK);
            slot[m] = j;
        }
    }
    if (!kept)
        for (int f = lane + 32 * GROW_KEEP; f < q.total; f += 32) {
            const int j = nbr_slot(q, f);
            if (j == d) continue;
            const float2 pj = pos[j];
            const float dd = dist2(pi.x, pi.y, pj.x, pj.y, L, h);
            if (!(dd < r2)) continue;
            const uint32_t tj = tg[j];
            nt += type_of(tj) == T_T;
            const unsigned long long kk = ((unsigned long long)__float_as_uint(dd) << 32) | (tj & GID_MASK);
            if (kk < best && maybe_end(tj, link[j]) && growable_end(tg, link, j, R.max_chain)) {
                best = kk;
                bj = j;
            }
        }
    nt = (int)__reduce_add_sync(0xffffffffu, (unsigned)nt);
    const unsigned long long wb = warp_min_u64(best);  // the exhaustive path's nearest growable end
    int e = -1;
    if (nt >= R.n_t_min) {
        // the kept candidates in increasing key order, one chain walk each, until one is growable
        unsigned alive = 0;
#pragma unroll
        for (int m = 0; m < GROW_KEEP; m++) alive |= key[m] != NONE_LIST_KEY ? (1u << m) : 0u;
        unsigned long long found = NONE_LIST_KEY;
        int fslot = -1;
        while (true) {
            unsigned long long mine = NONE_LIST_KEY;
            int mm = -1;
#pragma unroll
            for (int m = 0; m < GROW_KEEP; m++)
                if ((alive >> m & 1u) && key[m] < mine) {
                    mine = key[m];
                    mm = m;
                }
            const unsigned long long w = warp_min_u64(mine);
            if (w == NONE_LIST_KEY || w > wb) break;  // (the exhaustive path's end is nearer)
            int ok = 0;
            int sj = -1;
            if (mine == w) {
#pragma unroll
                for (int m = 0; m < GROW_KEEP; m++)
                    if (m == mm) sj = slot[m];
                ok = growable_end(tg, link, sj, R.max_chain) ? 1 : 0;
                if (!ok) alive &= ~(1u << mm);
            }
            const unsigned okm = __ballot_sync(0xffffffffu, ok != 0);
            if (okm) {
                found = w;
                fslot = __shfl_sync(0xffffffffu, sj, __ffs(okm) - 1);
                break;
            }
        }
        // the exhaustive path's candidates compete too
        if (wb < found) {
            const unsigned hm = __ballot_sync(0xffffffffu, best == wb && wb != NONE_LIST_KEY);
            found = wb;
            fslot = __shfl_sync(0xffffffffu, bj, __ffs(hm) - 1);
        }
        e = found != NONE_LIST_KEY ? fslot : -1;
    }
    if (lane == 0) {
        b.req[k] = e;
        if (e >= 0) atomicMin(b.claim + e, tg[d] & GID_MASK);
    }
}

// stage 2 application of list entry k: the lowest claiming gid wins its end
__device__ __forceinline__ void chem_grow_apply_one(const Bufs &b, int cur, int k, long long step) {
    const int e = __ldcg(b.req + k);
    if (e < 0) return;
    uint32_t *tg = b.tg[cur];
    int2 *link = b.link[cur];
    const int2 it = b.grow_list[k];
    const int d = it.x;
    const uint32_t g = tg[d] & GID_MASK;
    if (__ldcg(b.claim + e) != g) return;  // a lower gid claimed this end
    b.claim[e] = 0xFFFFFFFFu;
    tg[d] = ((uint32_t)T_T << TYPE_SHIFT) | g;
    link[d] = make_int2(e, -1);
    link[e].y = d;
    const float2 p = b.pos[cur][d];
    push_event(b, step, 0, g, tg[e] & GID_MASK, p.x, p.y, it.y);
}

// stage 3 request of list entry k, by one whole warp: a T that is still free
// claims its nearest free H within r_bond
__device__ __forceinline__ void chem_bond_req_one(const Bufs &b, int cur, const RepDev *__restrict__ reps, int k,
                                                  int lane) {
    const uint32_t *tg = b.tg[cur];
    const float2 *pos = b.pos[cur];
    const int2 *link = b.link[cur];
    const int2 it = b.bond_list[k];
    const int d = it.x;
    const int2 lk = link[d];
    int e = -1;
    if (type_of(tg[d]) == T_T && lk.x < 0 && lk.y < 0) {
        const RepDev &R = reps[it.y];
        const float2 pi = pos[d];
        const float L = R.L, h = R.halfL, r2 = R.r2_bond;
        const NbrRanges q = nbr_ranges(b, R, pi);
        unsigned long long best = NONE_LIST_KEY;
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
        const int mine = (best == wbest && wbest != NONE_LIST_KEY) ? bj : -1;
        e = (int)__reduce_max_sync(0xffffffffu, (unsigned)(mine + 1)) - 1;
    }
    if (lane == 0) {
        b.req[k] = e;
        if (e >= 0) atomicMin(b.claim + e, tg[d] & GID_MASK);
    }
}

// stage 3 application of list entry k
__device__ __forceinline__ void chem_bond_apply_one(const Bufs &b, int cur, int k, long long step) {
    const int h = __ldcg(b.req + k);
    if (h < 0) return;
    const uint32_t *tg = b.tg[cur];
    int2 *link = b.link[cur];
    const int2 it = b.bond_list[k];
    const int d = it.x;
    const uint32_t g = tg[d] & GID_MASK;
    if (__ldcg(b.claim + h) != g) return;
    b.claim[h] = 0xFFFFFFFFu;
    link[h].y = d;
    link[d].x = h;
    const float2 p = b.pos[cur][d];
    push_event(b, step, 2, g, tg[h] & GID_MASK, p.x, p.y, it.y);
}
