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
// ranges; hits (r < 1) go through a warp ballot into a per-warp ring buffer,
// which is drained 64 pairs at a time (two per lane), so the noise and force
// arithmetic always runs on full warps.  Halo sources only pair with owned
// beads: their ranges are clipped to the owned rows of the column.
//
// Epilogue per owned bead: harmonic bonds to prev/next, the force written to
// HBM, and the cell of the next position with its count (the first half of
// the next step's sort).  A tile whose beads do not fit in shared memory
// computes its owned beads straight from HBM instead (bead_pairs_direct).
#include "dpd_device.cuh"

#define TILE_TPB 256
#define TILE_WARPS (TILE_TPB / 32)
#define TILE_MAXB 1408
#define TILE_MAXC 256
#define TILE_QCAP 128  // per-warp ring; < 64 entries wait between drains, at most 64 arrive per round

struct TileSmem {
    float2 pos[TILE_MAXB];
    float2 vt[TILE_MAXB];
    uint32_t tg[TILE_MAXB];
    int32_t accx[TILE_MAXB];      // fixed-point force sums (separate arrays: 32 banks for the atomics)
    int32_t accy[TILE_MAXB];
    uint16_t lxy[TILE_MAXB];      // local cell of each bead: lx << 8 | ly
    uint8_t img[TILE_MAXB];       // periodic image code: (ix + 1) | (iy + 1) << 2
    int32_t lcs[TILE_MAXC + 1];   // local cell starts (column-major over (w+2) x (h+2))
    int32_t gst[TILE_MAXC];       // global slot of each local cell's first bead
    uint32_t q[TILE_WARPS][TILE_QCAP];
    float a[DPD_MAXT * DPD_MAXT];
    int32_t scan[TILE_WARPS];
    int32_t n;
    int32_t next_chunk;           // source chunks are handed to warps as they finish their last one
};

// periodic image shift of a pair along one axis: (code_s - code_t) L, exactly 0 or +-L
__device__ __forceinline__ float img_shift(int dc, float L) { return dc == 0 ? 0.0f : (dc > 0 ? L : -L); }

struct PairConst {
    NoiseKey nk;
    float L, gam, sdt;
};

// the pair force on s from t as fixed-point terms (a queued pair: inside the cutoff)
template <bool WRAP, int NOISE>
__device__ __forceinline__ void tile_pair(const TileSmem &S, const PairConst &pc, int s, int t, int &qx, int &qy,
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
__device__ __forceinline__ void tile_add(TileSmem &S, uint32_t v, int qx, int qy) {
    const int s = (int)(v >> 16), t = (int)(v & 0xFFFFu);
    atomicAdd(&S.accx[s], qx);
    atomicAdd(&S.accy[s], qy);
    atomicAdd(&S.accx[t], -qx);
    atomicAdd(&S.accy[t], -qy);
}

// evaluate ring entries [head, head + cnt), cnt <= 64: two independent chains per lane
template <bool WRAP, int NOISE>
__device__ __forceinline__ void drain(TileSmem &S, const PairConst &pc, const uint32_t *q, int head, int cnt,
                                      int lane, float &fmax) {
    const int e1 = lane, e2 = lane + 32;
    const bool has1 = e1 < cnt, has2 = e2 < cnt;
    if (has1) {
        const uint32_t v1 = q[(head + e1) & (TILE_QCAP - 1)];
        const uint32_t v2 = q[(head + (has2 ? e2 : e1)) & (TILE_QCAP - 1)];
        int qx1, qy1, qx2, qy2;
        tile_pair<WRAP, NOISE>(S, pc, (int)(v1 >> 16), (int)(v1 & 0xFFFFu), qx1, qy1, fmax);
        tile_pair<WRAP, NOISE>(S, pc, (int)(v2 >> 16), (int)(v2 & 0xFFFFu), qx2, qy2, fmax);
        tile_add(S, v1, qx1, qy1);
        if (has2) tile_add(S, v2, qx2, qy2);
    }
    __syncwarp();
}

// rows [lo, hi] of local column c that hold owned cells, as a bead index range
__device__ __forceinline__ void owned_rows(const TileSmem &S, int c, int LH, int tw, int th, int &b0, int &b1) {
    if (c >= 1 && c <= tw) {
        b0 = S.lcs[c * LH + 1];
        b1 = S.lcs[c * LH + th + 1];
    } else {
        b0 = b1 = 0;
    }
}

template <bool WRAP, int NOISE>
__device__ void tile_pairs(TileSmem &S, const PairConst &pc, int LW, int LH, int tw, int th, DevStatus *status) {
    const int lane = (int)lane_id(), wq = (int)threadIdx.x >> 5;
    const uint32_t below = (1u << lane) - 1u;
    uint32_t *q = S.q[wq];
    const int nsrc = S.lcs[(LW - 1) * LH];  // the last column (right halo) holds no sources
    int head = 0, tail = 0;
    float fmax = 0.0f;
    for (int base = wq * 32; base < nsrc;) {
        const int s = base + lane;
        int r1s = 0, len1 = 0, r2s = 0, len = 0;
        float2 ps = make_float2(0.0f, 0.0f);
        int is = 0;
        if (s < nsrc) {
            const int v = S.lxy[s], lx = v >> 8, ly = v & 255, l = lx * LH + ly;
            ps = S.pos[s];
            if (WRAP) is = S.img[s];
            int r1e = S.lcs[l + (ly + 1 < LH ? 2 : 1)];
            r1s = s + 1;
            const int c2 = (lx + 1) * LH;
            r2s = S.lcs[c2 + (ly > 0 ? ly - 1 : 0)];
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
            len = len1 + max(r2e - r2s, 0);
        }
        const int s2m = r2s - len1;
        const int maxlen = __reduce_max_sync(0xffffffffu, len);
        for (int k = 0; k < maxlen; k += 2) {
            bool hit[2];
            int tt[2];
#pragma unroll
            for (int u = 0; u < 2; u++) {
                const int kk = k + u;
                const int t = kk + (kk < len1 ? r1s : s2m);
                tt[u] = t;
                const int tc = kk < len ? t : 0;  // past the end: a harmless in-range read
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
            for (int u = 0; u < 2; u++) {
                const uint32_t hm = __ballot_sync(0xffffffffu, hit[u]);
                if (hit[u]) q[(tail + __popc(hm & below)) & (TILE_QCAP - 1)] = ((uint32_t)s << 16) | (uint32_t)tt[u];
                tail += __popc(hm);
            }
            __syncwarp();
            if (tail - head >= 64) {
                drain<WRAP, NOISE>(S, pc, q, head, 64, lane, fmax);
                head += 64;
            }
        }
        int nxt = 0;
        if (lane == 0) nxt = atomicAdd(&S.next_chunk, 1);
        base = __shfl_sync(0xffffffffu, nxt, 0) * 32;
    }
    while (tail > head) {
        const int cnt = min(tail - head, 64);
        drain<WRAP, NOISE>(S, pc, q, head, cnt, lane, fmax);
        head += cnt;
    }
    if (fmax > 2048.0f) raise_flag(status, DPD_F_FORCE);
}

// bonds, the force to HBM and the next cell key of one owned bead, from its
// links lk, its bond partners' positions pj[2] and its half-step velocity v
// (loaded by the caller)
template <bool NEXTKEY>
__device__ __forceinline__ void finish_loaded(const Bufs &b, int cur, const RepDev &R, int rep, int g, float2 pi,
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
}

// the same with its own loads (the crowded-tile path)
template <bool NEXTKEY>
__device__ __forceinline__ void finish_bead(const Bufs &b, int cur, const RepDev &R, int rep, int g, float2 pi,
                                            long long qx, long long qy, float &mb, uint32_t &key) {
    const int2 lk = b.link[cur][g];
    float2 pj[2];
    pj[0] = lk.x >= 0 ? b.pos[cur][lk.x] : pi;
    pj[1] = lk.y >= 0 ? b.pos[cur][lk.y] : pi;
    const float2 v = NEXTKEY ? b.vh[cur][g] : make_float2(0.0f, 0.0f);
    finish_loaded<NEXTKEY>(b, cur, R, rep, g, pi, qx, qy, lk, pj, v, mb, key);
}

#define EPI_ITEMS 2  // owned beads per thread per round of the epilogue

template <bool NEXTKEY>
__global__ void __launch_bounds__(TILE_TPB) k_forces_tile(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                          const TileDesc *__restrict__ tiles) {
    pdl_begin();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TileSmem &S = *reinterpret_cast<TileSmem *>(smem_raw);
    const TileDesc td = tiles[blockIdx.x];
    const RepDev &R = reps[td.rep];
    const int ncx = R.ncx, ncy = R.ncy;
    const int LW = td.w + 2, LH = td.h + 2, nl = LW * LH;
    const int32_t *__restrict__ cs = b.cstart + R.c0;
    const int tid = (int)threadIdx.x, lane = (int)lane_id(), wq = tid >> 5;
    const long long step = *b.step;
    if (tid < DPD_MAXT * DPD_MAXT) S.a[tid] = a_at(R, tid, step);
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
    {   // block exclusive scan of cnt (nl <= TILE_TPB)
        int x = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) S.scan[wq] = x;
        __syncthreads();
        before = 0;
        for (int k = 0; k < wq; k++) before += S.scan[k];
        before += x - cnt;
        if (tid < nl) S.lcs[tid] = before;
        if (tid == TILE_TPB - 1) {
            S.n = before + cnt;
            S.lcs[nl] = before + cnt;
        }
        __syncthreads();
    }
    const int n = S.n;
    float mb = 0.0f;
    if (n > TILE_MAXB) {
        // too crowded for shared memory: the owned beads straight from HBM (rare; same bits)
        PairConst pk;
        pk.nk = make_noise_key(R, step);
        for (int c = 1; c <= td.w; c++) {
            const int gx = td.cx0 + c - 1, g0 = cs[gx * ncy + td.cy0], g1 = cs[gx * ncy + td.cy0 + td.h];
            for (int base = g0; base < g1; base += TILE_TPB) {
                const int g = base + tid;
                const bool act = g < g1;
                uint32_t key = 0;
                if (act) {
                    PairCtx pc;
                    pc.pos = b.pos[cur];
                    pc.vt = b.vt[cur];
                    pc.tg = b.tg[cur];
                    pc.pi = pc.pos[g];
                    pc.vi = pc.vt[g];
                    const uint32_t tgi = pc.tg[g];
                    pc.gi = tgi & GID_MASK;
                    pc.arow = S.a + (tgi >> TYPE_SHIFT) * DPD_MAXT;
                    pc.nk = pk.nk;
                    pc.L = R.L;
                    pc.h = R.halfL;
                    pc.gam = R.gamma;
                    pc.sdt = sdt_at(R, step);
                    long long ax = 0, ay = 0;
                    bead_pairs_direct(pc, R, cs, g, ax, ay);
                    finish_bead<NEXTKEY>(b, cur, R, td.rep, g, pc.pi, ax, ay, mb, key);
                }
                if (NEXTKEY) {
                    count_key(b.count, key, act);
                    if (act) b.key[g] = key;
                }
            }
        }
    } else {
        // per local cell: its beads' cell and image code
        if (tid < nl)
            for (int k = before; k < before + cnt; k++) {
                S.lxy[k] = (uint16_t)((lx << 8) | ly);
                S.img[k] = (uint8_t)code;
            }
        __syncthreads();
        // copy in: consecutive beads of a column are consecutive in HBM (coalesced)
        for (int k = tid; k < n; k += TILE_TPB) {
            const int v = S.lxy[k], l = (v >> 8) * LH + (v & 255);
            const int g = S.gst[l] + (k - S.lcs[l]);
            S.pos[k] = b.pos[cur][g];
            S.vt[k] = b.vt[cur][g];
            S.tg[k] = b.tg[cur][g];
            S.accx[k] = 0;
            S.accy[k] = 0;
        }
        if (tid == 0) S.next_chunk = TILE_WARPS;  // chunks 0..7 go to warps 0..7 first
        __syncthreads();
        // ---- screened pairs, evaluated on full warps
        PairConst pc;
        pc.nk = make_noise_key(R, step);
        pc.L = R.L;
        pc.gam = R.gamma;
        pc.sdt = sdt_at(R, step);
        const bool wrap = td.cx0 == 0 || td.cy0 == 0 || td.cx0 + td.w >= ncx || td.cy0 + td.h >= ncy;
        if (R.noise == 1) {
            if (wrap) tile_pairs<true, 1>(S, pc, LW, LH, td.w, td.h, b.status);
            else tile_pairs<false, 1>(S, pc, LW, LH, td.w, td.h, b.status);
        } else {
            if (wrap) tile_pairs<true, 0>(S, pc, LW, LH, td.w, td.h, b.status);
            else tile_pairs<false, 0>(S, pc, LW, LH, td.w, td.h, b.status);
        }
        __syncthreads();
        // ---- epilogue over the local index range of the owned columns; halo beads
        // (rows 0 and h + 1) in that range are skipped.  Loads of a round first.
        const int e0 = S.lcs[LH + 1], e1 = S.lcs[td.w * LH + td.h + 1];
        const float2 *__restrict__ gpos = b.pos[cur];
        for (int base = e0; base < e1; base += EPI_ITEMS * TILE_TPB) {
            int gg[EPI_ITEMS];
            bool own[EPI_ITEMS];
#pragma unroll
            for (int j = 0; j < EPI_ITEMS; j++) {
                const int k = base + j * TILE_TPB + tid;
                own[j] = false;
                gg[j] = 0;
                if (k < e1) {
                    const int v = S.lxy[k], ly = v & 255, l = (v >> 8) * LH + ly;
                    own[j] = ly >= 1 && ly <= td.h;
                    gg[j] = S.gst[l] + (k - S.lcs[l]);
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
                const int k = base + j * TILE_TPB + tid;
                uint32_t key = 0;
                if (own[j])
                    finish_loaded<NEXTKEY>(b, cur, R, td.rep, gg[j], S.pos[k], S.accx[k], S.accy[k], lk[j], pj[j],
                                           vv[j], mb, key);
                if (NEXTKEY) {
                    count_key(b.count, key, own[j]);
                    if (own[j]) b.key[gg[j]] = key;
                }
            }
        }
    }
    const unsigned mbb = __reduce_max_sync(0xffffffffu, __float_as_uint(mb));
    if (lane == 0 && mbb != 0u) atomicMax(b.obs + (size_t)td.rep * OBS_N + 4, (unsigned long long)mbb);
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
    if (next_keys) launch_pdl(k_forces_tile<true>, ntiles, TILE_TPB, bytes, s, b, cur, rep, tiles);
    else k_forces_tile<false><<<ntiles, TILE_TPB, bytes, s>>>(b, cur, rep, tiles);
}
