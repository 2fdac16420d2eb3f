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

__device__ __forceinline__ bool chem_due(const RepDev &R, long long step) {
    return R.chem && R.n_chem > 0 && (step % R.n_chem) == 0;
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
// side drops its prev; both evaluate the same draw (the H bead's).
__device__ __forceinline__ void chem_in_permute(const Bufs &b, int cur, const RepDev &R, long long step, int rep, int d, float2 p,
                                uint32_t tg, int2 lk_old, int2 &nl) {
    const uint32_t *tg_old = b.tg[cur];
    if (type_of(tg) == T_H && lk_old.y >= 0) {
        const uint32_t tn = tg_old[lk_old.y];
        if (h_breaks(R, step, tg, tn)) {
            nl.y = -1;
            push_event(b, step, 1, tg & GID_MASK, tn & GID_MASK, p.x, p.y, rep);
        }
    } else if (type_of(tg) == T_T && lk_old.x >= 0) {
        if (h_breaks(R, step, tg_old[lk_old.x], tg)) nl.x = -1;
    }
    chem_candidate(b, R, step, rep, d, tg);
}

