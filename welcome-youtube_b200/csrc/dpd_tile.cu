// dpd_tile.cu -- pair + bond forces over cell tiles staged in shared memory (sm_100a).
//
// One CTA owns a tile of w x h cells of one replica.  It copies the beads of
// the tile and of a one-cell halo around it into shared memory and enumerates
// every pair that touches an owned bead ONCE (half shell: a cell pairs with
// itself and with its 4 forward neighbours (x, y+1), (x+1, y-1..y+1)).  The
// pair force q, rounded to a multiple of 2^-16, goes +q to one bead and -q to
// the other (32-bit shared atomics).  A pair between an owned bead and a halo
// bead is computed by both CTAs, each keeping its own side; the operands are
// exactly negated, so both sides agree bit for bit and sum F = 0 holds exactly.
// The sums equal those of the per-bead kernel (k_forces) bit for bit: the same
// terms, rounded the same way, added in integers.
//
// Screening: cells are column-major, so for a source bead s in local cell
// (lx, ly) its half-shell partners are two contiguous index ranges of the
// local arrays: the rest of its own cell plus the cell above, and cells
// ly-1..ly+1 of the next column.  A lane owns one source and walks its two
// ranges, four candidates a round; hits (r < 1) go through a warp ballot into
// a per-warp queue, which is drained 64 pairs at a time (two per lane), so the
// noise and force arithmetic always runs on full warps.  Halo sources only
// pair with owned beads: their ranges are clipped to the owned rows of the
// column.
//
// Epilogue per owned bead: harmonic bonds to prev/next, the force written to
// HBM, and the cell of the next position with its count (the first half of
// the next step's sort).  When the step's stats row is wanted (the stats ring),
// the epilogue also sums the row's terms of the beads it holds, and the last
// CTA hands the row over (RowAcc, row_handover).  A tile whose beads do not
// fit in shared memory computes its owned beads straight from HBM instead
// (bead_pairs_direct).
#include <algorithm>

#include "dpd_device.cuh"

#define TILE_TPB 256
#define TILE_WARPS (TILE_TPB / 32)
#define TILE_MAXB 1408
#define TILE_MAXC 256
#define TILE_QCAP 192  // per-warp queue; < 64 entries wait between drains, at most 128 arrive per round

// one tile's staged beads and their local layout, for tiles of up to MAXC local
// cells (tile and halo) and MAXB beads
template <int MAXB, int MAXC>
struct __align__(16) TileBeadT {
    static constexpr int maxb = MAXB;
    float2 pos[MAXB];
    float2 vt[MAXB];
    uint32_t tg[MAXB];
    int32_t accx[MAXB];           // fixed-point force sums (separate arrays: 32 banks for the atomics)
    int32_t accy[MAXB];
    uint16_t lxy[MAXB];           // local cell of each bead: lx << 8 | ly (TILE_PAD: a padding slot)
    uint8_t img[MAXB];            // periodic image code: (ix + 1) | (iy + 1) << 2
    int32_t lcs[MAXC + 1];        // local cell starts (column-major over (w+2) x (h+2))
    int32_t gst[MAXC];            // global slot of each local cell's first bead
    float a[DPD_MAXT * DPD_MAXT];
    int32_t n;
    // The screen reads pos[t] and img[t] for t <= 2 MAXB + 2 (past a range's
    // end, masked out): pos is followed by vt and tg, and img by at least
    // MAXB + 8 bytes.
    static_assert((MAXC + 1) * 4 + MAXC * 4 >= MAXB + 8, "img must be followed by MAXB + 8 bytes of the tile");
};
using TileBead = TileBeadT<TILE_MAXB, TILE_MAXC>;

// the shared memory of k_forces_tile with TPB threads: tiles of up to TPB
// local cells, and beads in proportion
template <int TPB>
struct TileSmemT {
    TileBeadT<TILE_MAXB * (TPB / 256), TPB> t;
    uint32_t q[TPB / 32][TILE_QCAP];
    int32_t scan[TPB / 32];
    int32_t next_chunk;           // source chunks are handed to warps as they finish their last one
    long long rsum[TPB / 32][3];  // per warp, the stats-row sums of the tile's owned beads (RowAcc)
    uint32_t rcnt[TPB / 32][DPD_MAXT / 2 + 1];
    int32_t rlast;                // this CTA hands the row over
};

#define TILE_PAD 0xFFFFu          // lxy of a slot that holds no bead of the tile (bulk-copy padding)

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// asynchronous global -> shared copies of one 8- or 4-byte element
// (cp.async, completed by cp.async.wait_all): a thread keeps all of its
// elements in flight at once, with no registers held for them
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// periodic image shift of a pair along one axis: (code_s - code_t) L, exactly 0 or +-L
__device__ __forceinline__ float img_shift(int dc, float L) { return dc == 0 ? 0.0f : (dc > 0 ? L : -L); }

struct PairConst {
    NoiseKey nk;
    float L, gam, sdt;
};

// the pair force on s from t as fixed-point terms (a queued pair: inside the cutoff)
template <bool WRAP, int NOISE, class TB>
__device__ __forceinline__ void tile_pair(const TB &S, const PairConst &pc, int s, int t, int &qx, int &qy,
                                          float &fmax) {
    const float2 ps = S.pos[s], pt = S.pos[t];
    float dx = __fsub_rn(ps.x, pt.x), dy = __fsub_rn(ps.y, pt.y);
    if (WRAP) {
        const int is = S.img[s], it = S.img[t];
        dx = __fadd_rn(dx, img_shift((is & 3) - (it & 3), pc.L));
        dy = __fadd_rn(dy, img_shift((is >> 2) - (it >> 2), pc.L));
    }
    const float r2 = __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
    const float2 vs = S.vt[s], vtt = S.vt[t];
    const uint32_t tgs = S.tg[s], tgt = S.tg[t];
    float r, ir;
    r_and_ir(r2, r, ir);
    const float w = __fsub_rn(1.0f, r);
    const float dvx = __fsub_rn(vs.x, vtt.x), dvy = __fsub_rn(vs.y, vtt.y);
    const float rv = __fmul_rn(__fmaf_rn(dx, dvx, __fmul_rn(dy, dvy)), ir);
    const uint32_t gs = tgs & GID_MASK, gt = tgt & GID_MASK;
    int32_t u;
    if (NOISE == 1) {
        const uint64_t key = ((uint64_t)min(gs, gt) << 32) | max(gs, gt);
        u = (int32_t)(uint32_t)(mix13((key * 0x9e3779b97f4a7c15ULL) ^ pc.nk.sseed) >> 32);
    } else {
        u = (int32_t)philox_w0k(min(gs, gt), max(gs, gt), pc.nk.s0, pc.nk.s1, pc.nk.ks);
    }
    const float th = __fmul_rn(__int2float_rn(u), THETA_SCALE);
    const float a = S.a[(tgs >> TYPE_SHIFT) * DPD_MAXT + (tgt >> TYPE_SHIFT)];
    const float inner = __fmaf_rn(pc.sdt, th, __fmaf_rn(-__fmul_rn(pc.gam, w), rv, a));
    const float fm = __fmul_rn(__fmul_rn(w, inner), ir);
    const float tx = __fmul_rn(fm, dx), ty = __fmul_rn(fm, dy);
    fmax = fmaxf(fmax, fmaxf(fabsf(tx), fabsf(ty)));
    qx = f2fix16(tx);
    qy = f2fix16(ty);
}

// +q to s, -q to t; halo accumulators take their share too and are ignored
template <class TB>
__device__ __forceinline__ void tile_add(TB &S, uint32_t v, int qx, int qy) {
    const int s = (int)(v >> 16), t = (int)(v & 0xFFFFu);
    atomicAdd(&S.accx[s], qx);
    atomicAdd(&S.accy[s], qy);
    atomicAdd(&S.accx[t], -qx);
    atomicAdd(&S.accy[t], -qy);
}

// evaluate queue entries [0, cnt), cnt <= 64: two independent chains per lane
template <bool WRAP, int NOISE, class TB>
__device__ __forceinline__ void drain(TB &S, const PairConst &pc, const uint32_t *q, int cnt, int lane,
                                      float &fmax) {
    const int e1 = lane, e2 = lane + 32;
    const bool has1 = e1 < cnt, has2 = e2 < cnt;
    if (has1) {
        const uint32_t v1 = q[e1];
        const uint32_t v2 = q[has2 ? e2 : e1];
        int qx1, qy1, qx2, qy2;
        tile_pair<WRAP, NOISE>(S, pc, (int)(v1 >> 16), (int)(v1 & 0xFFFFu), qx1, qy1, fmax);
        tile_pair<WRAP, NOISE>(S, pc, (int)(v2 >> 16), (int)(v2 & 0xFFFFu), qx2, qy2, fmax);
        tile_add(S, v1, qx1, qy1);
        if (has2) tile_add(S, v2, qx2, qy2);
    }
    __syncwarp();
}

// rows [lo, hi] of local column c that hold owned cells, as a bead index range
template <class TB>
__device__ __forceinline__ void owned_rows(const TB &S, int c, int LH, int tw, int th, int &b0, int &b1) {
    if (c >= 1 && c <= tw) {
        b0 = S.lcs[c * LH + 1];
        b1 = S.lcs[c * LH + th + 1];
    } else {
        b0 = b1 = 0;
    }
}

// The half-shell partners of source s (local cell code v) as two local index
// ranges, [r1s, r1s + len1) and [s2m + len1, s2m + len): the rest of its own
// cell with the cell above, and rows ly-1..ly+1 of the next column.  A halo
// source keeps its owned partners only.  Returns len.
template <class TB>
__device__ __forceinline__ int src_ranges(const TB &S, int s, int v, int LH, int tw, int th, int &r1s, int &len1,
                                          int &s2m) {
    const int lx = v >> 8, ly = v & 255, l = lx * LH + ly;
    int r1e = S.lcs[l + (ly + 1 < LH ? 2 : 1)];
    r1s = s + 1;
    const int c2 = (lx + 1) * LH;
    int r2s = S.lcs[c2 + (ly > 0 ? ly - 1 : 0)];
    int r2e = S.lcs[c2 + (ly + 1 < LH ? ly + 1 : LH - 1) + 1];
    if (!(lx >= 1 && lx <= tw && ly >= 1 && ly <= th)) {  // halo source: owned partners only
        int o0, o1;
        owned_rows(S, lx, LH, tw, th, o0, o1);
        r1s = max(r1s, o0);
        r1e = min(r1e, o1);
        owned_rows(S, lx + 1, LH, tw, th, o0, o1);
        r2s = max(r2s, o0);
        r2e = min(r2e, o1);
    }
    len1 = max(r1e - r1s, 0);
    s2m = r2s - len1;
    return len1 + max(r2e - r2s, 0);
}

// The screened pairs of the staged tile S, evaluated on full warps.  q: this
// warp's queue; next_chunk: the CTA's chunk counter (starts at the warp count);
// first: this warp's first chunk of 32 sources.
template <bool WRAP, int NOISE, class TB>
__device__ void tile_pairs(TB &S, uint32_t *q, int *next_chunk, int first, const PairConst &pc, int LW, int LH,
                           int tw, int th, DevStatus *status) {
    const int lane = (int)lane_id();
    const uint32_t below = (1u << lane) - 1u;
    const int nsrc = S.lcs[(LW - 1) * LH];  // the last column (right halo) holds no sources
    int tail = 0;  // queued pairs: fewer than 64 between rounds
    float fmax = 0.0f;
    for (int base = first * 32; base < nsrc;) {
        const int s = base + lane;
        int r1s = 0, len1 = 0, s2m = 0, len = 0;
        float2 ps = make_float2(0.0f, 0.0f);
        int is = 0;
        const int v = s < nsrc ? S.lxy[s] : (int)TILE_PAD;
        if (v != (int)TILE_PAD) {
            ps = S.pos[s];
            if (WRAP) is = S.img[s];
            len = src_ranges(S, s, v, LH, tw, th, r1s, len1, s2m);
        }
        const int maxlen = __reduce_max_sync(0xffffffffu, len);
        for (int k = 0; k < maxlen; k += 4) {
            bool hit[4];
            int tt[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int kk = k + u;
                const int t = kk + (kk < len1 ? r1s : s2m);
                tt[u] = t;
                const int tc = t;  // past the end (t <= 2 MAXB + 2): an in-bounds read, masked out below
                const float2 pt = S.pos[tc];
                float dx = __fsub_rn(ps.x, pt.x), dy = __fsub_rn(ps.y, pt.y);
                if (WRAP) {
                    const int it = S.img[tc];
                    dx = __fadd_rn(dx, img_shift((is & 3) - (it & 3), pc.L));
                    dy = __fadd_rn(dy, img_shift((is >> 2) - (it >> 2), pc.L));
                }
                const float r2 = __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
                hit[u] = kk < len && r2 < 1.0f && r2 > 1e-24f;
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const uint32_t hm = __ballot_sync(0xffffffffu, hit[u]);
                if (hit[u]) q[tail + __popc(hm & below)] = ((uint32_t)s << 16) | (uint32_t)tt[u];
                tail += __popc(hm);
            }
            while (tail >= 64) {  // uniform over the warp
                __syncwarp();
                drain<WRAP, NOISE>(S, pc, q, 64, lane, fmax);
                // move the rest, fewer than 128, to the front (all read before any is written)
                const int rest = tail - 64;
                uint32_t m[4];
#pragma unroll
                for (int e = 0; e < 4; e++) m[e] = 64 + lane + 32 * e < 192 ? q[64 + lane + 32 * e] : 0u;
                __syncwarp();
#pragma unroll
                for (int e = 0; e < 4; e++)
                    if (lane + 32 * e < rest) q[lane + 32 * e] = m[e];
                tail = rest;
                __syncwarp();
            }
        }
        int nxt = 0;
        if (lane == 0) nxt = atomicAdd(next_chunk, 1);
        base = __shfl_sync(0xffffffffu, nxt, 0) * 32;
    }
    __syncwarp();
    if (tail > 0) drain<WRAP, NOISE>(S, pc, q, tail, lane, fmax);
    if (fmax > 2048.0f) raise_flag(status, DPD_F_FORCE);
}

// bonds, the force to HBM and the next cell key of one owned bead, from its
// links lk, its bond partners' positions pj[2] and its half-step velocity v
// (loaded by the caller)
template <bool NEXTKEY>
__device__ __forceinline__ float2 finish_loaded(const Bufs &b, int cur, const RepDev &R, int rep, int g, float2 pi,
                                                long long qx, long long qy, int2 lk, const float2 (&pj)[2], float2 v,
                                                float &mb, uint32_t &key) {
    const float L = R.L, h = R.halfL, kb = R.kb, r0 = R.r0;
    if (R.arch != 0) {  // branched lipids: the template terms of k_mol_forces
        if (lk.x >= 0 || lk.y >= 0) {
            const int2 q = b.fmol[g];
            qx += q.x;
            qy += q.y;
        }
    } else {
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const int j = e ? lk.y : lk.x;
            if (j < 0) continue;
            const float dx = minimg(__fsub_rn(pj[e].x, pi.x), L, h), dy = minimg(__fsub_rn(pj[e].y, pi.y), L, h);
            const float r = __fsqrt_rn(__fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
            mb = fmaxf(mb, r);
            const float fb = __fdiv_rn(__fmul_rn(kb, __fsub_rn(r, r0)), r);
            qx += f2fix16(__fmul_rn(fb, dx));
            qy += f2fix16(__fmul_rn(fb, dy));
        }
        angle_terms(b, cur, R, pi, lk, pj[0], pj[1], qx, qy);
    }
    if (R.stir_A != 0.0f) qx += stir_force(R, pi.y, b.tg[cur][g] & GID_MASK, b.stir[rep]);
    const float2 fs = make_float2(fix16_to_f(qx), fix16_to_f(qy));
    if (!(isfinite(fs.x) && isfinite(fs.y))) raise_flag(b.status, DPD_F_NONFINITE);
    b.f[cur][g] = fs;
    if (NEXTKEY) {
        int cx, cy;
        key = (uint32_t)(R.c0 + cell_xy(R, advance1(pi.x, v.x, fs.x, R.dt, R.dt2, L),
                                        advance1(pi.y, v.y, fs.y, R.dt, R.dt2, L), cx, cy));
    }
    return fs;
}

// The stats-row terms of a thread's owned beads, as k_observables sums them:
// momentum and kinetic energy of v = vh + dt/2 F in fixed point, the bead
// count of each type (16-bit fields, two types per word) and the molecule
// heads.  flush() adds the warp's sums into its slot of the CTA's sums in
// shared memory (all lanes of the warp call it; the slot starts at zero).
struct RowAcc {
    long long sx = 0, sy = 0, s2 = 0;
    uint32_t c[DPD_MAXT / 2] = {0, 0, 0, 0};
    uint32_t heads = 0;
    __device__ __forceinline__ void add(const RepDev &R, float2 v, float2 f, uint32_t tg, int2 lk) {
        const double vx = (double)v.x + (double)R.hdt * (double)f.x;
        const double vy = (double)v.y + (double)R.hdt * (double)f.y;
        sx += __double2ll_rn(vx * OBS_FIX);
        sy += __double2ll_rn(vy * OBS_FIX);
        s2 += __double2ll_rn((vx * vx + vy * vy) * OBS_FIX);
        const int ty = (int)(tg >> TYPE_SHIFT);
#pragma unroll
        for (int w = 0; w < DPD_MAXT / 2; w++)
            c[w] += ty == 2 * w ? 1u : (ty == 2 * w + 1 ? 0x10000u : 0u);
        heads += (lk.x < 0 && lk.y >= 0) ? 1u : 0u;
    }
    __device__ __forceinline__ void flush(long long (*rs)[3], uint32_t (*rc)[DPD_MAXT / 2 + 1]) {
        const long long a = warp_sum_ll(sx), bb = warp_sum_ll(sy), d = warp_sum_ll(s2);
        uint32_t cw[DPD_MAXT / 2 + 1];
#pragma unroll
        for (int w = 0; w < DPD_MAXT / 2; w++) cw[w] = __reduce_add_sync(0xffffffffu, c[w]);
        cw[DPD_MAXT / 2] = __reduce_add_sync(0xffffffffu, heads);
        if (lane_id() == 0) {  // the warp's own slot: no other thread writes it
            const int w = (int)threadIdx.x >> 5;
            rs[w][0] += a;
            rs[w][1] += bb;
            rs[w][2] += d;
#pragma unroll
            for (int k = 0; k < DPD_MAXT / 2 + 1; k++) rc[w][k] += cw[k];
        }
    }
};

// the same with its own loads (the crowded-tile path)
template <bool NEXTKEY>
__device__ __forceinline__ float2 finish_bead(const Bufs &b, int cur, const RepDev &R, int rep, int g, float2 pi,
                                              long long qx, long long qy, float &mb, uint32_t &key) {
    const int2 lk = b.link[cur][g];
    float2 pj[2];
    pj[0] = lk.x >= 0 ? b.pos[cur][lk.x] : pi;
    pj[1] = lk.y >= 0 ? b.pos[cur][lk.y] : pi;
    const float2 v = NEXTKEY ? b.vh[cur][g] : make_float2(0.0f, 0.0f);
    return finish_loaded<NEXTKEY>(b, cur, R, rep, g, pi, qx, qy, lk, pj, v, mb, key);
}

#define EPI_ITEMS 2   // owned beads per thread per round of the epilogue
// Four CTAs of k_forces_tile per SM (32 warps): the register budget is set for
// it (64 per thread).  Left to itself the compiler takes 104 registers, which
// leaves room for two CTAs; measured on the 1,048,576-bead box, four are 11 %
// faster.
#define TILE_MINB 4

// The owned beads of tile td straight from HBM (full-shell sums, bonds, force,
// next key): the path for a tile too crowded for shared memory (rare; the
// same bits).  arow: the tile's a_ij table in shared memory.
template <bool NEXTKEY>
__device__ void tile_direct(const Bufs &b, int cur, const RepDev &R, const TileDesc &td, const float *a, long long step,
                            float &mb, long long (*rs)[3], uint32_t (*rc)[DPD_MAXT / 2 + 1]) {
    const int ncy = R.ncy, tid = (int)threadIdx.x;
    const int32_t *__restrict__ cs = b.cstart + R.c0;
    PairConst pk;
    pk.nk = make_noise_key(R, step);
    for (int c = 1; c <= td.w; c++) {
        const int gx = td.cx0 + c - 1, g0 = cs[gx * ncy + td.cy0], g1 = cs[gx * ncy + td.cy0 + td.h];
        for (int base = g0; base < g1; base += blockDim.x) {
            RowAcc acc;  // this round's row terms
            const int g = base + tid;
            const bool act = g < g1;
            uint32_t key = 0;
            float2 fs = make_float2(0.0f, 0.0f);
            if (act) {
                PairCtx pc;
                pc.pos = b.pos[cur];
                pc.vt = b.vt[cur];
                pc.tg = b.tg[cur];
                pc.pi = pc.pos[g];
                pc.vi = pc.vt[g];
                const uint32_t tgi = pc.tg[g];
                pc.gi = tgi & GID_MASK;
                pc.arow = a + (tgi >> TYPE_SHIFT) * DPD_MAXT;
                pc.nk = pk.nk;
                pc.L = R.L;
                pc.h = R.halfL;
                pc.gam = R.gamma;
                pc.sdt = sdt_at(R, step);
                long long ax = 0, ay = 0;
                bead_pairs_direct(pc, R, cs, g, ax, ay);
                fs = finish_bead<NEXTKEY>(b, cur, R, td.rep, g, pc.pi, ax, ay, mb, key);
            }
            if (rs && act) acc.add(R, b.vh[cur][g], fs, b.tg[cur][g], b.link[cur][g]);
            if (rs) acc.flush(rs, rc);  // (uniform over the CTA)
            if (NEXTKEY) {
                count_key(b.count, key, act);
                if (act) b.key[g] = key;
            }
        }
    }
}

// The pairs of a staged tile: the screen and the queue, one instantiation per
// image mode and noise generator
template <class TB>
__device__ __forceinline__ void tile_pairs_any(TB &S, uint32_t *q, int *next_chunk, int first,
                                               const RepDev &R, const TileDesc &td, long long step,
                                               DevStatus *status) {
    PairConst pc;
    pc.nk = make_noise_key(R, step);
    pc.L = R.L;
    pc.gam = R.gamma;
    pc.sdt = sdt_at(R, step);
    const int LW = td.w + 2, LH = td.h + 2;
    const bool wrap = td.cx0 == 0 || td.cy0 == 0 || td.cx0 + td.w >= R.ncx || td.cy0 + td.h >= R.ncy;
    if (R.noise == 1) {
        if (wrap) tile_pairs<true, 1>(S, q, next_chunk, first, pc, LW, LH, td.w, td.h, status);
        else tile_pairs<false, 1>(S, q, next_chunk, first, pc, LW, LH, td.w, td.h, status);
    } else {
        if (wrap) tile_pairs<true, 0>(S, q, next_chunk, first, pc, LW, LH, td.w, td.h, status);
        else tile_pairs<false, 0>(S, q, next_chunk, first, pc, LW, LH, td.w, td.h, status);
    }
}

// The epilogue of a staged tile: over the local index range of the owned
// columns, every owned bead (halo rows and padding slots in that range are
// skipped) gets its bonds, its force written to HBM and its next cell key.
// The loads of a round are issued first.
template <bool NEXTKEY, class TB>
__device__ __forceinline__ void tile_epilogue(const Bufs &b, int cur, const RepDev &R, const TileDesc &td,
                                              const TB &S, float &mb, long long (*rs)[3],
                                              uint32_t (*rc)[DPD_MAXT / 2 + 1]) {
    const int LH = td.h + 2, tid = (int)threadIdx.x;
    const int e0 = S.lcs[LH + 1], e1 = S.lcs[td.w * LH + td.h + 1];
    const float2 *__restrict__ gpos = b.pos[cur];
    for (int base = e0; base < e1; base += EPI_ITEMS * blockDim.x) {
        RowAcc acc;  // this round's row terms
        int gg[EPI_ITEMS];
        bool own[EPI_ITEMS];
#pragma unroll
        for (int j = 0; j < EPI_ITEMS; j++) {
            const int k = base + j * (int)blockDim.x + tid;
            own[j] = false;
            gg[j] = 0;
            if (k < e1) {
                const int v = S.lxy[k], ly = v & 255, l = (v >> 8) * LH + ly;
                own[j] = v != (int)TILE_PAD && ly >= 1 && ly <= td.h;
                if (own[j]) gg[j] = S.gst[l] + (k - S.lcs[l]);
            }
        }
        int2 lk[EPI_ITEMS];
        float2 vv[EPI_ITEMS];
#pragma unroll
        for (int j = 0; j < EPI_ITEMS; j++) {
            lk[j] = own[j] ? b.link[cur][gg[j]] : make_int2(-1, -1);
            vv[j] = (NEXTKEY && own[j]) ? b.vh[cur][gg[j]] : make_float2(0.0f, 0.0f);
        }
        float2 pj[EPI_ITEMS][2];
#pragma unroll
        for (int j = 0; j < EPI_ITEMS; j++) {
            pj[j][0] = lk[j].x >= 0 ? gpos[lk[j].x] : make_float2(0.0f, 0.0f);
            pj[j][1] = lk[j].y >= 0 ? gpos[lk[j].y] : make_float2(0.0f, 0.0f);
        }
#pragma unroll
        for (int j = 0; j < EPI_ITEMS; j++) {
            const int k = base + j * (int)blockDim.x + tid;
            uint32_t key = 0;
            float2 fs = make_float2(0.0f, 0.0f);
            if (own[j])
                fs = finish_loaded<NEXTKEY>(b, cur, R, td.rep, gg[j], S.pos[k], S.accx[k], S.accy[k], lk[j], pj[j],
                                            vv[j], mb, key);
            if (NEXTKEY) {
                count_key(b.count, key, own[j]);
                if (own[j]) b.key[gg[j]] = key;
            }
            if (rs && own[j]) acc.add(R, vv[j], fs, S.tg[k], lk[j]);
        }
        if (rs) acc.flush(rs, rc);  // (uniform over the CTA)
    }
}

// The end of a launch that assembles a stats row: the CTA's row sums go to
// the replica's running sums (the slots of k_observables: 0, 1 momentum,
// 2 kinetic, 5 heads, 8 + t type counts; 4, the max bond, is max_bond_out's),
// and the last CTA of the grid hands the row over, to obs_out and into the
// host ring, and clears the sums for the next row, as k_observables does.
__device__ __forceinline__ void row_handover(const Bufs &b, const RowOut &row, const long long (*rs)[3],
                                             const uint32_t (*rc)[DPD_MAXT / 2 + 1], bool mine, int32_t *last) {
    __syncthreads();
    unsigned long long *obs = b.obs + (size_t)row.rep * OBS_N;
    const int tid = (int)threadIdx.x, nw = (int)blockDim.x >> 5;
    if (mine && tid < 3 + DPD_MAXT + 1) {  // the warps' sums: 3 fixed-point sums, the type counts, the heads
        unsigned long long v = 0;
        int slot;
        if (tid < 3) {
            for (int w = 0; w < nw; w++) v += (unsigned long long)rs[w][tid];
            slot = tid;
        } else if (tid < 3 + DPD_MAXT) {
            const int t = tid - 3;
            for (int w = 0; w < nw; w++) v += (rc[w][t >> 1] >> (16 * (t & 1))) & 0xFFFFu;
            slot = 8 + t;
        } else {
            for (int w = 0; w < nw; w++) v += rc[w][DPD_MAXT / 2];
            slot = 5;
        }
        if (v != 0) atomicAdd(obs + slot, v);
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) *last = atomicAdd(b.obs_done + row.rep, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!*last) return;
    __threadfence();
    unsigned long long *out = row.host;
    const long long step = *b.step;
    if (out && row.slots > 0) out += (size_t)(step % row.slots) * OBS_N;
    if (tid < OBS_N) {
        const unsigned long long v = atomicExch(obs + tid, 0ull);
        b.obs_out[(size_t)row.rep * OBS_N + tid] = v;
        if (out) out[tid] = (row.slots > 0 && tid == 6) ? (unsigned long long)step : v;
    }
    if (tid == 0) b.obs_done[row.rep] = 0u;
}

// the running max bond of a tile's replica (one atomic per warp)
__device__ __forceinline__ void max_bond_out(const Bufs &b, int rep, float mb) {
    const unsigned mbb = __reduce_max_sync(0xffffffffu, __float_as_uint(mb));
    if (lane_id() == 0 && mbb != 0u) atomicMax(b.obs + (size_t)rep * OBS_N + 4, (unsigned long long)mbb);
}

template <bool NEXTKEY, int TPB>
__global__ void __launch_bounds__(TPB, TILE_MINB * 256 / TPB) k_forces_tile(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                          const TileDesc *__restrict__ tiles, RowOut row) {
    // The successor may be scheduled only once this grid's CTAs reach their
    // epilogue: scheduled earlier, its waiting CTAs would hold SM slots that
    // later tiles need (1 % of the step at 1M beads).
    pdl_wait();
    extern __shared__ __align__(128) unsigned char smem_raw[];
    TileSmemT<TPB> &SS = *reinterpret_cast<TileSmemT<TPB> *>(smem_raw);
    auto &S = SS.t;
    constexpr int MAXB = TILE_MAXB * (TPB / 256);
    const TileDesc td = tiles[blockIdx.x];
    const RepDev &R = reps[td.rep];
    const int ncx = td.ncx, ncy = td.ncy;  // from the tile: the cell starts need no load of R first
    const int LH = td.h + 2, nl = (td.w + 2) * LH;
    const int32_t *__restrict__ cs = b.cstart + td.c0;
    const int tid = (int)threadIdx.x, lane = (int)lane_id(), wq = tid >> 5;
    const long long step = *b.step;
    if (tid < DPD_MAXT * DPD_MAXT) S.a[tid] = a_at(R, tid, step);
    const bool want_row = NEXTKEY && row.rep == td.rep;  // this tile's beads enter the step's stats row
    long long(*rs)[3] = want_row ? SS.rsum : nullptr;
    uint32_t(*rc)[DPD_MAXT / 2 + 1] = want_row ? SS.rcnt : nullptr;
    if (want_row && lane == 0) {  // each warp's slot of the row sums (only that warp's lane 0 writes it)
        SS.rsum[wq][0] = SS.rsum[wq][1] = SS.rsum[wq][2] = 0;
        for (int k = 0; k < DPD_MAXT / 2 + 1; k++) SS.rcnt[wq][k] = 0;
    }
    // ---- phase 0: local cells, their bead counts, exclusive scan
    int cnt = 0, lx = 0, ly = 0, code = 0;
    if (tid < nl) {
        lx = tid / LH;
        ly = tid - lx * LH;
        int gx = td.cx0 - 1 + lx, gy = td.cy0 - 1 + ly;
        const int ix = gx < 0 ? -1 : (gx >= ncx ? 1 : 0), iy = gy < 0 ? -1 : (gy >= ncy ? 1 : 0);
        gx -= ix * ncx;
        gy -= iy * ncy;
        code = (ix + 1) | ((iy + 1) << 2);
        const int gc = gx * ncy + gy;
        S.gst[tid] = cs[gc];
        cnt = cs[gc + 1] - cs[gc];
    }
    int before;
    {   // block exclusive scan of cnt (nl <= TPB)
        int x = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) SS.scan[wq] = x;
        __syncthreads();
        before = 0;
        for (int k = 0; k < wq; k++) before += SS.scan[k];
        before += x - cnt;
        if (tid < nl) S.lcs[tid] = before;
        if (tid == TPB - 1) {
            S.n = before + cnt;
            S.lcs[nl] = before + cnt;
        }
        __syncthreads();
    }
    const int n = S.n;
    float mb = 0.0f;
    if (n > MAXB) {
        tile_direct<NEXTKEY>(b, cur, R, td, S.a, step, mb, rs, rc);
    } else {
        // per local cell: its beads' cell and image code
        if (tid < nl)
            for (int k = before; k < before + cnt; k++) {
                S.lxy[k] = (uint16_t)((lx << 8) | ly);
                S.img[k] = (uint8_t)code;
            }
        __syncthreads();
        // copy in: consecutive beads of a column are consecutive in HBM
        // (coalesced); every copy of a thread is issued before it waits
        for (int k = tid; k < n; k += TPB) {
            const int v = S.lxy[k], l = (v >> 8) * LH + (v & 255);
            const int g = S.gst[l] + (k - S.lcs[l]);
            cp_async8(&S.pos[k], b.pos[cur] + g);
            cp_async8(&S.vt[k], b.vt[cur] + g);
            cp_async4(&S.tg[k], b.tg[cur] + g);
            S.accx[k] = 0;
            S.accy[k] = 0;
        }
        if (tid == 0) SS.next_chunk = TPB / 32;  // chunk w goes to warp w first
        cp_async_wait_all();
        __syncthreads();
        tile_pairs_any(S, SS.q[wq], &SS.next_chunk, wq, R, td, step, b.status);
        __syncthreads();
        pdl_trigger();
        tile_epilogue<NEXTKEY>(b, cur, R, td, S, mb, rs, rc);
    }
    max_bond_out(b, td.rep, mb);
    if (NEXTKEY && row.rep >= 0) row_handover(b, row, SS.rsum, SS.rcnt, want_row, &SS.rlast);
}

// ---------------------------------------------------------------- the bulk-staged kernel
//
// k_forces_bulk computes the same sums as k_forces_tile, one CTA per tile, but
// stages the tile's beads with bulk asynchronous copies (cp.async.bulk, global
// -> shared, completion counted on an mbarrier) instead of per-bead loads and
// stores.  Cells are column-major, so a local column of the tile and its halo
// is one contiguous slot range (two where the rows wrap around the box): warp
// 0 issues one bulk copy per array and range as soon as it has the ranges'
// ends, while the other threads load the per-cell starts.  A bulk copy moves
// 16-byte aligned blocks, so each range is widened to a multiple of 4 slots;
// the extra slots are padding, marked with TILE_PAD and placed far away, so
// that no screen ever hits them.  All copies read this GPU's own memory; no
// copy uses cluster multicast.  The epilogue takes a bond partner's position
// from shared memory when the partner is staged (almost always: bonds are
// shorter than a cell), else from HBM.
//
// The wait on the mbarrier is bounded (STAGE_WAIT_NS of global time); a CTA
// that gives up raises DPD_F_WAIT (the call returns DPD_E_TIMEOUT), waits once
// more, bounded, for its copies, and returns.

#define STAGE_MAXP 64                 // column ranges of one tile (w + 2 <= 32 columns, at most 2 ranges each)
#define STAGE_MAXLW 32
#define STAGE_WAIT_NS 200000000ull    // 0.2 s
#define STAGE_FAR 1.0e18f             // padding slots sit here: no distance to them is below the cutoff

struct StagePiece {                   // one contiguous slot range of a local column, staged by bulk copies
    int32_t a4, n4;                   // first global slot copied (a multiple of 4), slots copied (a multiple of 4)
    int32_t sm;                       // local slot of a4
    int32_t lo, hi;                   // the tile's beads in the range: global slots [lo, hi)
};

struct BulkSmem {
    TileBead t;
    StagePiece pc[STAGE_MAXP];
    int32_t np;                       // ranges of the tile
    int8_t colp[STAGE_MAXLW];         // first range of each local column
    int8_t split[STAGE_MAXLW];        // local rows in that first range (the rest are in the next)
    uint32_t q[TILE_WARPS][TILE_QCAP];
    int32_t next_chunk;
    int32_t fail;
    unsigned long long mbar;
};


__device__ __forceinline__ void mbar_init(unsigned long long *m, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(m)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(unsigned long long *m, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(m)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *m, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(m)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// wait for the phase of parity `parity` of m to complete, at most STAGE_WAIT_NS
__device__ __forceinline__ bool mbar_wait(unsigned long long *m, unsigned parity) {
    if (mbar_try_wait(m, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(m, parity))
        if (global_ns() - t0 > STAGE_WAIT_NS) return false;
    return true;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *m) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(m))
                 : "memory");
}

// Warp 0: the tile's column ranges, their local slots and the bulk copies of
// the bead data (none if the tile does not fit: T.n > TILE_MAXB)
__device__ void stage_ranges(BulkSmem &S, const TileDesc &td, const Bufs &b, int cur, const RepDev &R) {
    const int lane = (int)lane_id();
    TileBead &T = S.t;
    const int ncx = R.ncx, ncy = R.ncy, LW = td.w + 2, LH = td.h + 2;
    const int32_t *__restrict__ cs = b.cstart + R.c0;
    // lane = local column; its rows cy0 - 1 .. cy0 + h wrap at most once (h + 2 <= ncy)
    int nr = 0, sp = LH;
    StagePiece p0 = {0, 0, 0, 0, 0}, p1 = {0, 0, 0, 0, 0};
    if (lane < LW) {
        int gx = td.cx0 - 1 + lane;
        gx = gx < 0 ? gx + ncx : (gx >= ncx ? gx - ncx : gx);
        const int gy0 = td.cy0 - 1, col = gx * ncy;
        if (gy0 < 0) sp = 1;                       // row ncy - 1, then rows 0 .. h
        else if (gy0 + LH > ncy) sp = ncy - gy0;   // rows gy0 .. ncy - 1, then row 0 ..
        const int ya = gy0 < 0 ? ncy - 1 : gy0;
        p0.lo = cs[col + ya];
        p0.hi = cs[col + ya + sp];
        nr = 1;
        if (sp < LH) {
            p1.lo = cs[col];
            p1.hi = cs[col + LH - sp];
            nr = 2;
        }
    }
    int slots = 0;
    StagePiece *pp[2] = {&p0, &p1};
#pragma unroll
    for (int k = 0; k < 2; k++) {
        StagePiece &q = *pp[k];
        const bool any = k < nr && q.hi > q.lo;
        q.a4 = any ? q.lo & ~3 : q.lo;  // an empty range copies nothing; its cells start at its local slot
        q.n4 = any ? ((q.hi + 3) & ~3) - q.a4 : 0;
        slots += q.n4;
    }
    // local slot of each range and index of each column's first range: exclusive warp scans
    int x = slots, y = nr;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, x, o), v = __shfl_up_sync(0xffffffffu, y, o);
        if (lane >= o) {
            x += u;
            y += v;
        }
    }
    const int total = __shfl_sync(0xffffffffu, x, 31), np = __shfl_sync(0xffffffffu, y, 31);
    p0.sm = x - slots;
    p1.sm = p0.sm + p0.n4;
    const int pidx = y - nr;
    if (lane < LW) {
        S.pc[pidx] = p0;
        if (nr == 2) S.pc[pidx + 1] = p1;
        S.colp[lane] = (int8_t)pidx;
        S.split[lane] = (int8_t)sp;
    }
    if (lane == 0) {
        S.np = np;
        T.n = total;
    }
    const bool fits = total <= TILE_MAXB;
    __syncwarp();
    if (lane == 0) mbar_arrive_tx(&S.mbar, fits ? (unsigned)total * 20u : 0u);
    __syncwarp();
    if (fits && lane < LW) {
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const StagePiece &q = *pp[k];
            if (k >= nr || q.n4 == 0) continue;
            bulk_g2s(&T.pos[q.sm], b.pos[cur] + q.a4, (unsigned)q.n4 * 8u, &S.mbar);
            bulk_g2s(&T.vt[q.sm], b.vt[cur] + q.a4, (unsigned)q.n4 * 8u, &S.mbar);
            bulk_g2s(&T.tg[q.sm], b.tg[cur] + q.a4, (unsigned)q.n4 * 4u, &S.mbar);
        }
    }
}

// local slot of a staged bead of column lx - 1 .. lx + 1 from its global slot g (-1: not staged)
__device__ __forceinline__ int staged_slot(const BulkSmem &S, int lx, int LW, int LH, int g) {
    for (int c = max(lx - 1, 0); c <= min(lx + 1, LW - 1); c++) {
        const int k0 = S.colp[c], nk = S.split[c] < LH ? 2 : 1;
        for (int k = k0; k < k0 + nk; k++) {
            const StagePiece &q = S.pc[k];
            if (g >= q.lo && g < q.hi) return q.sm + (g - q.a4);
        }
    }
    return -1;
}

// the epilogue of a bulk-staged tile: tile_epilogue with the bond partners'
// positions taken from shared memory where staged
template <bool NEXTKEY>
__device__ __forceinline__ void bulk_epilogue(const Bufs &b, int cur, const RepDev &R, const TileDesc &td,
                                              const BulkSmem &S, float &mb) {
    const TileBead &T = S.t;
    const int LH = td.h + 2, LW = td.w + 2, tid = (int)threadIdx.x;
    const int e0 = T.lcs[LH + 1], e1 = T.lcs[td.w * LH + td.h + 1];
    const float2 *__restrict__ gpos = b.pos[cur];
    for (int base = e0; base < e1; base += EPI_ITEMS * blockDim.x) {
        int gg[EPI_ITEMS], lx[EPI_ITEMS];
        bool own[EPI_ITEMS];
#pragma unroll
        for (int j = 0; j < EPI_ITEMS; j++) {
            const int k = base + j * (int)blockDim.x + tid;
            own[j] = false;
            gg[j] = 0;
            lx[j] = 0;
            if (k < e1) {
                const int v = T.lxy[k], ly = v & 255, l = (v >> 8) * LH + ly;
                own[j] = v != (int)TILE_PAD && ly >= 1 && ly <= td.h;
                if (own[j]) {
                    gg[j] = T.gst[l] + (k - T.lcs[l]);
                    lx[j] = v >> 8;
                }
            }
        }
        int2 lk[EPI_ITEMS];
        float2 vv[EPI_ITEMS];
#pragma unroll
        for (int j = 0; j < EPI_ITEMS; j++) {
            lk[j] = own[j] ? b.link[cur][gg[j]] : make_int2(-1, -1);
            vv[j] = (NEXTKEY && own[j]) ? b.vh[cur][gg[j]] : make_float2(0.0f, 0.0f);
        }
        float2 pj[EPI_ITEMS][2];
#pragma unroll
        for (int j = 0; j < EPI_ITEMS; j++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int g = e ? lk[j].y : lk[j].x;
                pj[j][e] = make_float2(0.0f, 0.0f);
                if (g >= 0) {
                    const int ks = staged_slot(S, lx[j], LW, LH, g);
                    pj[j][e] = ks >= 0 ? T.pos[ks] : gpos[g];
                }
            }
#pragma unroll
        for (int j = 0; j < EPI_ITEMS; j++) {
            const int k = base + j * (int)blockDim.x + tid;
            uint32_t key = 0;
            if (own[j])
                finish_loaded<NEXTKEY>(b, cur, R, td.rep, gg[j], T.pos[k], T.accx[k], T.accy[k], lk[j], pj[j], vv[j],
                                       mb, key);
            if (NEXTKEY) {
                count_key(b.count, key, own[j]);
                if (own[j]) b.key[gg[j]] = key;
            }
        }
    }
}

template <bool NEXTKEY>
__global__ void __launch_bounds__(TILE_TPB, TILE_MINB) k_forces_bulk(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                          const TileDesc *__restrict__ tiles) {
    pdl_begin();
    extern __shared__ __align__(128) unsigned char smem_raw[];
    BulkSmem &S = *reinterpret_cast<BulkSmem *>(smem_raw);
    TileBead &T = S.t;
    const int tid = (int)threadIdx.x, wq = tid >> 5;
    const TileDesc td = tiles[blockIdx.x];
    const RepDev &R = reps[td.rep];
    const int ncx = R.ncx, ncy = R.ncy, LH = td.h + 2, nl = (td.w + 2) * LH;
    const int32_t *__restrict__ cs = b.cstart + R.c0;
    const long long step = *b.step;
    if (tid == 0) {
        mbar_init(&S.mbar, 1);
        S.fail = 0;
        S.next_chunk = TILE_WARPS;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (tid < DPD_MAXT * DPD_MAXT) T.a[tid] = a_at(R, tid, step);
    // every thread of a local cell loads its cell starts while warp 0 starts the copies
    int lx = 0, ly = 0, code = 0, s0 = 0, s1 = 0;
    if (tid < nl) {
        lx = tid / LH;
        ly = tid - lx * LH;
        int gx = td.cx0 - 1 + lx, gy = td.cy0 - 1 + ly;
        const int ix = gx < 0 ? -1 : (gx >= ncx ? 1 : 0), iy = gy < 0 ? -1 : (gy >= ncy ? 1 : 0);
        gx -= ix * ncx;
        gy -= iy * ncy;
        code = (ix + 1) | ((iy + 1) << 2);
        const int gc = gx * ncy + gy;
        s0 = cs[gc];
        s1 = cs[gc + 1];
    }
    __syncthreads();  // the mbarrier is initialised
    if (wq == 0) stage_ranges(S, td, b, cur, R);
    __syncthreads();  // ranges known
    const bool fits = T.n <= TILE_MAXB;
    if (tid < nl) {
        const StagePiece &q = S.pc[S.colp[lx] + (ly < S.split[lx] ? 0 : 1)];
        const int k0 = q.sm + (s0 - q.a4);
        T.lcs[tid] = k0;
        T.gst[tid] = s0;
        if (fits)
            for (int k = k0; k < k0 + (s1 - s0); k++) {
                T.lxy[k] = (uint16_t)((lx << 8) | ly);
                T.img[k] = (uint8_t)code;
            }
    }
    if (tid == 0) T.lcs[nl] = T.n;
    if (fits)
        for (int k = tid; k < S.np; k += blockDim.x) {  // padding slots: no bead
            const StagePiece q = S.pc[k];
            for (int j = q.sm; j < q.sm + (q.lo - q.a4); j++) T.lxy[j] = (uint16_t)TILE_PAD;
            for (int j = q.sm + (q.hi - q.a4); j < q.sm + q.n4; j++) T.lxy[j] = (uint16_t)TILE_PAD;
        }
    // the staged beads
    if (!mbar_wait(&S.mbar, 0u)) S.fail = 1;
    if (fits) {
        for (int k = tid; k < S.np; k += blockDim.x) {  // padding slots sit far away
            const StagePiece q = S.pc[k];
            for (int j = q.sm; j < q.sm + (q.lo - q.a4); j++) T.pos[j] = make_float2(STAGE_FAR, STAGE_FAR);
            for (int j = q.sm + (q.hi - q.a4); j < q.sm + q.n4; j++) T.pos[j] = make_float2(STAGE_FAR, STAGE_FAR);
        }
        for (int k = tid; k < T.n; k += blockDim.x) {
            T.accx[k] = 0;
            T.accy[k] = 0;
        }
    }
    __syncthreads();
    if (S.fail) {
        // a copy never completed: report it, wait once more (bounded) so that none is
        // still writing when the CTA ends, and return
        if (tid == 0) raise_flag(b.status, DPD_F_WAIT);
        mbar_wait(&S.mbar, 0u);
        return;
    }
    float mb = 0.0f;
    if (fits) {
        tile_pairs_any(T, S.q[wq], &S.next_chunk, wq, R, td, step, b.status);
        __syncthreads();
        bulk_epilogue<NEXTKEY>(b, cur, R, td, S, mb);
    } else {
        tile_direct<NEXTKEY>(b, cur, R, td, T.a, step, mb, nullptr, nullptr);
    }
    max_bond_out(b, td.rep, mb);
}

size_t tile_smem_bytes() { return sizeof(TileSmemT<512>); }
size_t bulk_smem_bytes() { return sizeof(BulkSmem); }

int tile_setup() {
    const size_t bytes = sizeof(TileSmemT<256>), bytes2 = sizeof(TileSmemT<512>), bbytes = sizeof(BulkSmem);
    cudaError_t e =
        cudaFuncSetAttribute(k_forces_tile<true, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_forces_tile<false, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_forces_tile<true, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes2);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_forces_tile<false, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes2);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_forces_bulk<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bbytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_forces_bulk<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bbytes);
    return e == cudaSuccess ? 0 : -1;
}

void launch_forces_tile(const Bufs &b, int cur, const RepDev *rep, const TileDesc *tiles, int ntiles, int threads,
                        bool next_keys, cudaStream_t s, RowOut row) {
    if (!next_keys) row.rep = -1;
    if (threads == 512) {
        const size_t bytes = sizeof(TileSmemT<512>);
        if (next_keys) launch_pdl(k_forces_tile<true, 512>, ntiles, 512, bytes, s, b, cur, rep, tiles, row);
        else k_forces_tile<false, 512><<<ntiles, 512, bytes, s>>>(b, cur, rep, tiles, row);
        return;
    }
    const size_t bytes = sizeof(TileSmemT<256>);
    if (next_keys) launch_pdl(k_forces_tile<true, 256>, ntiles, 256, bytes, s, b, cur, rep, tiles, row);
    else k_forces_tile<false, 256><<<ntiles, 256, bytes, s>>>(b, cur, rep, tiles, row);
}

void launch_forces_bulk(const Bufs &b, int cur, const RepDev *rep, const TileDesc *tiles, int ntiles,
                        bool next_keys, cudaStream_t s) {
    const size_t bytes = sizeof(BulkSmem);
    if (next_keys) launch_pdl(k_forces_bulk<true>, ntiles, TILE_TPB, bytes, s, b, cur, rep, tiles);
    else k_forces_bulk<false><<<ntiles, TILE_TPB, bytes, s>>>(b, cur, rep, tiles);
}
