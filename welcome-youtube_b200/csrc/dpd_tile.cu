// dpd_tile.cu -- pair + bond forces over cell tiles staged in shared memory (sm_100a).
//
// One CTA owns a tile of w x h cells of one replica.  It copies the beads of
// the tile and of a one-cell halo around it into shared memory, enumerates
// every pair that touches an owned bead ONCE (half shell: a cell pairs with
// itself and with its 4 forward neighbours (x, y+1), (x+1, y-1..y+1)), and adds
// +q to one bead and -q to the other (q = the pair force rounded to a multiple
// of 2^-16, 32-bit shared atomics).  A pair between an owned bead and a halo
// bead is computed by both CTAs, each keeping its own side; the operands are
// exactly negated, so both sides agree bit for bit and sum F = 0 holds exactly.
// The sums equal those of the per-bead kernel (k_forces) bit for bit: the same
// terms, rounded the same way, added in integers.
//
// Per warp the candidate pairs are screened (r < 1) into a queue in shared
// memory and the queue is evaluated 32 pairs at a time, so the noise and force
// arithmetic runs on full warps.  Epilogue per owned bead: harmonic bonds to
// prev/next, the force written to HBM, and the cell of the next position with
// its count (the first half of the next step's sort).
#include "dpd_device.cuh"

#define TILE_TPB 256
#define TILE_WARPS (TILE_TPB / 32)
#define TILE_MAXB 1536
#define TILE_MAXC 256
#define TILE_QCAP 512

struct TileSmem {
    float2 pos[TILE_MAXB];
    float2 vt[TILE_MAXB];
    uint32_t tg[TILE_MAXB];
    int32_t gslot[TILE_MAXB];
    int2 acc[TILE_MAXB];
    uint16_t lcell[TILE_MAXB];
    uint8_t flag[TILE_MAXB];      // bit 0 owned; bits 1-2 x image code + 1; bits 3-4 y image code + 1
    int32_t lcs[TILE_MAXC + 1];   // local cell starts (column-major over (w+2) x (h+2))
    int32_t gst[TILE_MAXC];       // global slot of each local cell's first bead
    uint32_t q[TILE_WARPS][TILE_QCAP];
    float a[DPD_MAXT * DPD_MAXT];
    int32_t scan[TILE_TPB / 32];
    int32_t n;
};

__device__ __forceinline__ int img_x(uint8_t f) { return (int)((f >> 1) & 3u) - 1; }
__device__ __forceinline__ int img_y(uint8_t f) { return (int)((f >> 3) & 3u) - 1; }

// periodic image shift of a pair: (code_s - code_t) L, exactly 0 or +-L
__device__ __forceinline__ float img_shift(int dc, float L) { return dc == 0 ? 0.0f : (dc > 0 ? L : -L); }

struct PairConst {
    NoiseKey nk;
    float L, gam, sdt;
    DevStatus *status;
};

// the pair force on s from t as fixed-point terms; only called for queued
// pairs, which the screen already found inside the cutoff with the same r^2
template <bool WRAP, int NOISE>
__device__ __forceinline__ void tile_pair(const TileSmem &S, const PairConst &pc, int s, int t, int &qx, int &qy) {
    const float2 ps = S.pos[s], pt = S.pos[t];
    float dx = __fsub_rn(ps.x, pt.x), dy = __fsub_rn(ps.y, pt.y);
    if (WRAP) {
        const uint8_t fs = S.flag[s], ft = S.flag[t];
        dx = __fadd_rn(dx, img_shift(img_x(fs) - img_x(ft), pc.L));
        dy = __fadd_rn(dy, img_shift(img_y(fs) - img_y(ft), pc.L));
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
    qx = f2fix16(__fmul_rn(fm, dx));
    qy = f2fix16(__fmul_rn(fm, dy));
}

// +q to s, -q to t; halo accumulators take their share too and are ignored
__device__ __forceinline__ void tile_add(TileSmem &S, int s, int t, int qx, int qy) {
    atomicAdd(&S.acc[s].x, qx);
    atomicAdd(&S.acc[s].y, qy);
    atomicAdd(&S.acc[t].x, -qx);
    atomicAdd(&S.acc[t].y, -qy);
}

template <bool WRAP, int NOISE>
__device__ __forceinline__ void flush_queue(TileSmem &S, const PairConst &pc, int wq, int qn, int lane,
                                            int &qmax) {
    // two queue entries per lane per round: two independent noise + force chains
    for (int e = lane; e < qn; e += 64) {
        const int e2 = e + 32;
        const uint32_t v = S.q[wq][e];
        const bool two = e2 < qn;
        const uint32_t v2 = two ? S.q[wq][e2] : v;
        int qx, qy, qx2, qy2;
        tile_pair<WRAP, NOISE>(S, pc, (int)(v >> 16), (int)(v & 0xFFFFu), qx, qy);
        tile_pair<WRAP, NOISE>(S, pc, (int)(v2 >> 16), (int)(v2 & 0xFFFFu), qx2, qy2);
        qx2 = two ? qx2 : 0;
        qy2 = two ? qy2 : 0;
        qmax = max(qmax, max(max(abs(qx), abs(qy)), max(abs(qx2), abs(qy2))));
        tile_add(S, (int)(v >> 16), (int)(v & 0xFFFFu), qx, qy);
        tile_add(S, (int)(v2 >> 16), (int)(v2 & 0xFFFFu), qx2, qy2);
    }
    __syncwarp();
}

// Screening by cell: a warp takes a source cell A; its lanes hold up to 32
// candidate beads t of the half-shell set of A (A itself, the cell above, and
// the three cells of the next column) in registers and the warp walks the
// beads s of A (a shared-memory broadcast), queueing every (s, t) inside the
// cutoff that touches an owned bead.
template <bool WRAP, int NOISE>
__device__ void tile_pairs(TileSmem &S, const PairConst &pc, int LW, int LH, int tw, int th) {
    const int lane = (int)lane_id(), wq = (int)threadIdx.x >> 5;
    const int nl = LW * LH;
    int qn = 0, qmax = 0;
    for (int l = wq; l < nl; l += TILE_WARPS) {
        const int A0 = S.lcs[l], A1 = S.lcs[l + 1];
        if (A0 == A1) continue;
        const int lx = l / LH, ly = l - lx * LH;
        const bool aown = lx >= 1 && lx <= tw && ly >= 1 && ly <= th;
        if (!aown) {  // a halo cell matters only if its half-shell set holds an owned cell
            const bool up = lx >= 1 && lx <= tw && ly + 1 >= 1 && ly + 1 <= th;
            const bool right = lx + 1 >= 1 && lx + 1 <= tw && ly + 1 >= 1 && ly - 1 <= th;
            if (!up && !right) continue;
        }
        const int b1s = A0, b1e = S.lcs[ly + 1 < LH ? l + 2 : l + 1];
        int b2s = 0, b2e = 0;
        if (lx + 1 < LW) {
            b2s = S.lcs[(lx + 1) * LH + (ly > 0 ? ly - 1 : 0)];
            b2e = S.lcs[(lx + 1) * LH + (ly + 1 < LH ? ly + 1 : LH - 1) + 1];
        }
        const int nb1 = b1e - b1s, nb = nb1 + (b2e - b2s), na = A1 - A0;
        for (int c0 = 0; c0 < nb; c0 += 32) {
            const int k = c0 + lane;
            const bool tv = k < nb;
            const int t = tv ? (k < nb1 ? b1s + k : b2s + (k - nb1)) : 0;
            const float2 pt = S.pos[t];
            const uint8_t ft = S.flag[t];
            const bool tok = tv && (aown || (ft & 1u));
            const int tin = k < na ? A0 + k : -1;  // t's slot when t lies in A (only s < t pairs there)
            if (qn + 32 * na > TILE_QCAP) {  // room for every pair of this source cell and chunk
                flush_queue<WRAP, NOISE>(S, pc, wq, qn, lane, qmax);
                qn = 0;
            }
            // four sources per round: independent screening chains for the scheduler
            for (int s0 = A0; s0 < A1; s0 += 4) {
                if (qn > TILE_QCAP - 128) {  // only for cells of more than QCAP / 32 beads
                    flush_queue<WRAP, NOISE>(S, pc, wq, qn, lane, qmax);
                    qn = 0;
                }
                bool hit[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int s = min(s0 + u, A1 - 1);  // past the cell end: repeat the last bead, masked below
                    const float2 ps = S.pos[s];
                    float dx = __fsub_rn(ps.x, pt.x), dy = __fsub_rn(ps.y, pt.y);
                    if (WRAP) {
                        const uint8_t fs = S.flag[s];
                        dx = __fadd_rn(dx, img_shift(img_x(fs) - img_x(ft), pc.L));
                        dy = __fadd_rn(dy, img_shift(img_y(fs) - img_y(ft), pc.L));
                    }
                    const float r2 = __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
                    hit[u] = (s0 + u < A1) && tok && (tin < 0 || tin > s) && r2 < 1.0f && r2 > 1e-24f;
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const unsigned hm = __ballot_sync(0xffffffffu, hit[u]);
                    if (hit[u]) S.q[wq][qn + __popc(hm & ((1u << lane) - 1u))] = ((uint32_t)(s0 + u) << 16) | (uint32_t)t;
                    qn += __popc(hm);
                }
            }
        }
    }
    flush_queue<WRAP, NOISE>(S, pc, wq, qn, lane, qmax);
    if (qmax > FIX_TERM_LIMIT) raise_flag(pc.status, DPD_F_FORCE);
}

template <bool NEXTKEY>
__global__ void __launch_bounds__(TILE_TPB) k_forces_tile(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                          const TileDesc *__restrict__ tiles) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TileSmem &S = *reinterpret_cast<TileSmem *>(smem_raw);
    const TileDesc td = tiles[blockIdx.x];
    const RepDev &R = reps[td.rep];
    const int ncx = R.ncx, ncy = R.ncy;
    const int LW = td.w + 2, LH = td.h + 2, nl = LW * LH;
    const int32_t *__restrict__ cs = b.cstart + R.c0;
    const int tid = (int)threadIdx.x;
    if (tid < DPD_MAXT * DPD_MAXT) S.a[tid] = a_at(R, tid, *b.step);
    // ---- phase 0: local cells, their bead counts, exclusive scan, copy in
    int cnt = 0;
    if (tid < nl) {
        const int lx = tid / LH, ly = tid - lx * LH;
        int gx = td.cx0 - 1 + lx, gy = td.cy0 - 1 + ly;
        gx += gx < 0 ? ncx : (gx >= ncx ? -ncx : 0);
        gy += gy < 0 ? ncy : (gy >= ncy ? -ncy : 0);
        const int gc = gx * ncy + gy;
        S.gst[tid] = cs[gc];
        cnt = cs[gc + 1] - cs[gc];
    }
    {   // block exclusive scan of cnt (nl <= TILE_TPB)
        const int lane = (int)lane_id(), w = tid >> 5;
        int x = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) S.scan[w] = x;
        __syncthreads();
        int before = 0;
        for (int k = 0; k < w; k++) before += S.scan[k];
        if (tid < nl) S.lcs[tid] = before + x - cnt;
        if (tid == TILE_TPB - 1) {
            S.n = before + x;
            S.lcs[nl] = before + x;
        }
        __syncthreads();
    }
    const int n = S.n;
    if (n > TILE_MAXB) {  // tile too crowded for shared memory: report, leave the forces to the host check
        if (tid == 0) raise_flag(b.status, DPD_F_TILE);
        return;
    }
    const bool wrap = td.cx0 == 0 || td.cy0 == 0 || td.cx0 + td.w >= ncx || td.cy0 + td.h >= ncy;
    for (int k = tid; k < n; k += TILE_TPB) {
        int lo = 0, hi = nl;  // last local cell with lcs <= k
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (S.lcs[mid] <= k) lo = mid;
            else hi = mid;
        }
        const int l = lo, lx = l / LH, ly = l - lx * LH;
        const int g = S.gst[l] + (k - S.lcs[l]);
        const int gx = td.cx0 - 1 + lx, gy = td.cy0 - 1 + ly;
        const int ix = gx < 0 ? -1 : (gx >= ncx ? 1 : 0), iy = gy < 0 ? -1 : (gy >= ncy ? 1 : 0);
        const bool own = lx >= 1 && lx <= td.w && ly >= 1 && ly <= td.h;
        S.pos[k] = b.pos[cur][g];
        S.vt[k] = b.vt[cur][g];
        S.tg[k] = b.tg[cur][g];
        S.gslot[k] = g;
        S.lcell[k] = (uint16_t)l;
        S.flag[k] = (uint8_t)((own ? 1u : 0u) | ((uint32_t)(ix + 1) << 1) | ((uint32_t)(iy + 1) << 3));
        S.acc[k] = make_int2(0, 0);
    }
    __syncthreads();
    // ---- phases 1 + 2: screened pair queue per warp, evaluated on full warps
    PairConst pc;
    pc.nk = make_noise_key(R, *b.step);
    pc.L = R.L;
    pc.gam = R.gamma;
    pc.sdt = R.sdt;
    pc.status = b.status;
    if (R.noise == 1) {
        if (wrap) tile_pairs<true, 1>(S, pc, LW, LH, td.w, td.h);
        else tile_pairs<false, 1>(S, pc, LW, LH, td.w, td.h);
    } else {
        if (wrap) tile_pairs<true, 0>(S, pc, LW, LH, td.w, td.h);
        else tile_pairs<false, 0>(S, pc, LW, LH, td.w, td.h);
    }
    __syncthreads();
    // ---- phase 3: bonds, the force to HBM, next cell key + count
    const float2 *__restrict__ pos = b.pos[cur];
    const float L = R.L, h = R.halfL, kb = R.kb, r0 = R.r0;
    float mb = 0.0f;
    for (int base = 0; base < n; base += TILE_TPB) {
        const int k = base + tid;
        const bool act = k < n && (S.flag[k] & 1u);
        uint32_t key = 0;
        int g = 0;
        if (act) {
            g = S.gslot[k];
            int2 q = S.acc[k];
            const float2 pi = S.pos[k];
            const int2 lk = b.link[cur][g];
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int j = e ? lk.y : lk.x;
                if (j < 0) continue;
                const float2 pj = pos[j];
                const float dx = minimg(__fsub_rn(pj.x, pi.x), L, h), dy = minimg(__fsub_rn(pj.y, pi.y), L, h);
                const float r = __fsqrt_rn(__fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
                mb = fmaxf(mb, r);
                const float fb = __fdiv_rn(__fmul_rn(kb, __fsub_rn(r, r0)), r);
                q.x += f2fix16(__fmul_rn(fb, dx));
                q.y += f2fix16(__fmul_rn(fb, dy));
            }
            const float2 fs = make_float2(fix16_to_f(q.x), fix16_to_f(q.y));
            b.f[cur][g] = fs;
            if (NEXTKEY) {
                const float2 v = b.vh[cur][g];
                int cx, cy;
                key = (uint32_t)(R.c0 + cell_xy(R, advance1(pi.x, v.x, fs.x, R.dt, R.dt2, L),
                                                advance1(pi.y, v.y, fs.y, R.dt, R.dt2, L), cx, cy));
            }
        }
        if (NEXTKEY) {
            count_key(b.count, key, act);
            if (act) b.key[g] = key;
        }
    }
    const unsigned mbb = __reduce_max_sync(0xffffffffu, __float_as_uint(mb));
    if (lane_id() == 0 && mbb != 0u) atomicMax(b.obs + (size_t)td.rep * OBS_N + 4, (unsigned long long)mbb);
}

size_t tile_smem_bytes() { return sizeof(TileSmem); }

int tile_setup() {
    const size_t bytes = sizeof(TileSmem);
    cudaError_t e = cudaFuncSetAttribute(k_forces_tile<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_forces_tile<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    return e == cudaSuccess ? 0 : -1;
}

void launch_forces_tile(const Bufs &b, int cur, const RepDev *rep, const TileDesc *tiles, int ntiles,
                        bool next_keys, cudaStream_t s) {
    const size_t bytes = sizeof(TileSmem);
    if (next_keys) k_forces_tile<true><<<ntiles, TILE_TPB, bytes, s>>>(b, cur, rep, tiles);
    else k_forces_tile<false><<<ntiles, TILE_TPB, bytes, s>>>(b, cur, rep, tiles);
}
