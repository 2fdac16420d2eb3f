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

#define LIST_GRID 148

// stage 2: requests, one warp per listed P, then the claims applied by the last CTA
__global__ void __launch_bounds__(BEAD_TPB) k_chem_grow(Bufs b, int cur, const RepDev *__restrict__ reps) {
    pdl_begin();
    const int n = (int)b.status->n_grow;
    const int nw = (int)(gridDim.x * blockDim.x) >> 5;
    for (int k = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); k < n; k += nw)
        chem_grow_req_one(b, cur, reps, k, (int)lane_id());
    if (!last_cta(&b.status->done)) return;
    const long long step = *b.step;
    for (int k = (int)threadIdx.x; k < n; k += (int)blockDim.x) chem_grow_apply_one(b, cur, k, step);
}

// stage 3: requests, one warp per listed T, then the claims applied by the last CTA
__global__ void __launch_bounds__(BEAD_TPB) k_chem_bond(Bufs b, int cur, const RepDev *__restrict__ reps) {
    pdl_begin();
    const int n = (int)b.status->n_bond;
    const int nw = (int)(gridDim.x * blockDim.x) >> 5;
    for (int k = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); k < n; k += nw)
        chem_bond_req_one(b, cur, reps, k, (int)lane_id());
    if (!last_cta(&b.status->done)) return;
    const long long step = *b.step;
    for (int k = (int)threadIdx.x; k < n; k += (int)blockDim.x) chem_bond_apply_one(b, cur, k, step);
}

int chem_kernel_count() { return 2; }

void launch_chem_scan(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, cudaStream_t s) {
    k_chem_scan<<<nbch, BEAD_TPB, 0, s>>>(b, cur, rep, bch);
}

void launch_chem_lists(const Bufs &b, int cur, const RepDev *rep, int part, cudaStream_t s) {
    if (part < 0 || part == 0) launch_pdl(k_chem_grow, LIST_GRID, BEAD_TPB, 0, s, b, cur, rep);
    if (part < 0 || part == 1) launch_pdl(k_chem_bond, LIST_GRID, BEAD_TPB, 0, s, b, cur, rep);
}
