// dpd_device.cuh -- device helpers shared by the kernels of libdpd.so.
#pragma once
#include "dpd_internal.h"

// ---------------------------------------------------------------- counter-based RNGs

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), first output word.
// Counter (c0, c1, c2, c3); the round keys (k0 + r W0, k1 + r W1) come
// precomputed in ks (see PhiloxKeys); constants from the paper.
struct PhiloxKeys {
    uint32_t k0[10], k1[10];
};

__device__ __forceinline__ PhiloxKeys philox_keys(uint32_t k0, uint32_t k1) {
    PhiloxKeys ks;
#pragma unroll
    for (int r = 0; r < 10; r++) {
        ks.k0[r] = k0 + (uint32_t)r * 0x9E3779B9u;
        ks.k1[r] = k1 + (uint32_t)r * 0xBB67AE85u;
    }
    return ks;
}

__device__ __forceinline__ uint32_t philox_w0k(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                               const PhiloxKeys &ks) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ ks.k0[r];
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ ks.k1[r];
        c1 = (uint32_t)p1;
        c3 = (uint32_t)p0;
        c0 = n0;
        c2 = n2;
    }
    return c0;
}

__device__ __forceinline__ uint32_t philox_w0(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                              uint32_t k1) {
    return philox_w0k(c0, c1, c2, c3, philox_keys(k0, k1));
}

// splitmix64 finaliser of the reference (cel/engine/oercel.c:124-128)
__device__ __forceinline__ uint64_t mix13(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// per-step noise key of the reference (oercel.c:131-133)
__device__ __forceinline__ uint64_t step_seed(uint64_t seed, long long step) {
    return mix13(mix13(seed ^ 0x5851f42d4c957f2dULL) ^ mix13((uint64_t)step + 0x632be59bd9b4e019ULL));
}

#define THETA_SCALE (3.4641016151377545870548926830117f / 4294967296.0f)  // sqrt(12) / 2^32

// symmetric pair noise theta, uniform on [-sqrt3, sqrt3).
// noise 0: Philox word 0 at counter (min gid, max gid, step), key = seed;
// noise 1: the reference's mix13 pair hash (oercel.c:137-141), top 32 bits.
struct NoiseKey {
    PhiloxKeys ks;             // Philox round keys of the seed
    uint32_t s0, s1;           // step words of the counter
    uint64_t sseed;            // mix13 per-step key
    int mode;
};

__device__ __forceinline__ NoiseKey make_noise_key(const RepDev &R, long long step) {
    NoiseKey k;
    k.ks = philox_keys((uint32_t)R.seed, (uint32_t)(R.seed >> 32));
    k.s0 = (uint32_t)(unsigned long long)step;
    k.s1 = (uint32_t)((unsigned long long)step >> 32);
    k.mode = R.noise;
    k.sseed = R.noise == 1 ? step_seed(R.seed, step) : 0ull;
    return k;
}

__device__ __forceinline__ float pair_theta(const NoiseKey &k, uint32_t gi, uint32_t gj) {
    const uint32_t lo = min(gi, gj), hi = max(gi, gj);
    int32_t u;
    if (k.mode == 1) {
        const uint64_t key = ((uint64_t)lo << 32) | hi;
        u = (int32_t)(uint32_t)(mix13((key * 0x9e3779b97f4a7c15ULL) ^ k.sseed) >> 32);
    } else {
        u = (int32_t)philox_w0k(lo, hi, k.s0, k.s1, k.ks);
    }
    return __fmul_rn(__int2float_rn(u), THETA_SCALE);
}

// keyed decision word for the chemistry: Philox word 0 at counter (gid, salt, step), key = seed
__device__ __forceinline__ uint32_t decision_word(const RepDev &R, long long step, uint32_t salt, uint32_t gid) {
    return philox_w0(gid, salt, (uint32_t)(unsigned long long)step, (uint32_t)((unsigned long long)step >> 32),
                     (uint32_t)R.seed, (uint32_t)(R.seed >> 32));
}

// ---------------------------------------------------------------- the pair force

// 1/r and r from r^2 with the hardware reciprocal square root: r^2 -> (r, 1/r)
__device__ __forceinline__ void r_and_ir(float r2, float &r, float &ir) {
    ir = rsqrtf(r2);
    r = __fmul_rn(r2, ir);
}

// ---------------------------------------------------------------- fixed-point force sums

// Each pair or bond term is rounded once to a multiple of 2^-16 (a 32-bit
// integer) and the terms are summed in integers: the sum does not depend on the
// order of the terms, and the two halves of a pair, computed with exactly
// negated operands, cancel exactly.  A bead's sum stays far below 2^31 (|F| <
// 32768) for any physical state; a single term above 2048 raises a flag.
#define FIX_TERM_LIMIT (1 << 27)
__device__ __forceinline__ int f2fix16(float v) { return __float2int_rn(__fmul_rn(v, 65536.0f)); }
__device__ __forceinline__ float fix16_to_f(int a) { return __fmul_rn(__int2float_rn(a), 1.52587890625e-05f); }
__device__ __forceinline__ float fix16_to_f(long long a) { return __fmul_rn(__ll2float_rn(a), 1.52587890625e-05f); }

// ---------------------------------------------------------------- cells and the integrator

// cell of a position: the reference's cell_of_pos (oercel.c:779-786) with nsub = 1
__device__ __forceinline__ int cell_xy(const RepDev &R, float x, float y, int &cx, int &cy) {
    cx = (int)((double)x * R.icsx);
    cy = (int)((double)y * R.icsy);
    cx = cx >= R.ncx ? R.ncx - 1 : cx;
    cy = cy >= R.ncy ? R.ncy - 1 : cy;
    cx = cx < 0 ? 0 : cx;
    cy = cy < 0 ? 0 : cy;
    return cx * R.ncy + cy;
}

// Groot-Warren position update x + dt vh + dt^2 f, wrapped into [0, L)
// (oercel.c:2314-2324); every rounding spelled out so that the copy in the
// force kernel's next-key epilogue and the one in the permute kernel agree.
__device__ __forceinline__ float advance1(float x, float vh, float f, float dt, float dt2, float L) {
    const float dd = __fmaf_rn(dt2, f, __fmul_rn(dt, vh));
    float xi = __fadd_rn(x, dd);
    xi = xi < 0.0f ? __fadd_rn(xi, L) : xi;
    xi = xi >= L ? __fsub_rn(xi, L) : xi;
    return xi;
}

__device__ __forceinline__ float minimg(float d, float L, float h) {
    return d > h ? __fsub_rn(d, L) : (d < -h ? __fadd_rn(d, L) : d);
}

// ---------------------------------------------------------------- the pair term

// one pair term on bead i from bead j in fixed point; dx = minimg(x_i - x_j),
// which equals (x_i - x_j) + shift of the cell stencil bit for bit
struct PairCtx {
    const float2 *__restrict__ pos;
    const float2 *__restrict__ vt;
    const uint32_t *__restrict__ tg;
    const float *arow;
    NoiseKey nk;
    float2 pi, vi;
    uint32_t gi;
    float L, h, gam, sdt;
};

__device__ __forceinline__ void pair_term(const PairCtx &c, int j, long long &ax, long long &ay) {
    const float2 pj = c.pos[j];
    const float dx = minimg(__fsub_rn(c.pi.x, pj.x), c.L, c.h);
    const float dy = minimg(__fsub_rn(c.pi.y, pj.y), c.L, c.h);
    const float r2 = __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
    const float2 vj = c.vt[j];
    const uint32_t tgj = c.tg[j];
    float r, ir;
    r_and_ir(r2, r, ir);
    const float w = __fsub_rn(1.0f, r);
    const float dvx = __fsub_rn(c.vi.x, vj.x), dvy = __fsub_rn(c.vi.y, vj.y);
    const float rv = __fmul_rn(__fmaf_rn(dx, dvx, __fmul_rn(dy, dvy)), ir);
    const float th = pair_theta(c.nk, c.gi, tgj & GID_MASK);
    const float inner = __fmaf_rn(c.sdt, th, __fmaf_rn(-__fmul_rn(c.gam, w), rv, c.arow[tgj >> TYPE_SHIFT]));
    const float fm = __fmul_rn(__fmul_rn(w, inner), ir);
    ax += f2fix16(__fmul_rn(fm, dx));
    ay += f2fix16(__fmul_rn(fm, dy));
}


// The full-shell pair sum of bead d straight from HBM (3 x 3 cells around its
// own, every term evaluated on the spot): the force kernels' slow path for
// tiles too crowded for shared memory.  Same terms and roundings as k_forces.
__device__ __forceinline__ void bead_pairs_direct(const PairCtx &pc, const RepDev &R, const int32_t *__restrict__ cs,
                                                  int d, long long &ax, long long &ay) {
    const int ncx = R.ncx, ncy = R.ncy;
    const float L = R.L;
    int cx, cy;
    cell_xy(R, pc.pi.x, pc.pi.y, cx, cy);
    for (int ox = -1; ox <= 1; ox++) {
        int nx = cx + ox;
        float sx = 0.0f;
        if (nx < 0) {
            nx += ncx;
            sx = L;
        } else if (nx >= ncx) {
            nx -= ncx;
            sx = -L;
        }
        for (int oy = -1; oy <= 1; oy++) {
            int ny = cy + oy;
            float sy = 0.0f;
            if (ny < 0) {
                ny += ncy;
                sy = L;
            } else if (ny >= ncy) {
                ny -= ncy;
                sy = -L;
            }
            const int cc = nx * ncy + ny;
            for (int j = cs[cc]; j < cs[cc + 1]; j++) {
                const float2 pj = pc.pos[j];
                const float dx = __fadd_rn(__fsub_rn(pc.pi.x, pj.x), sx);
                const float dy = __fadd_rn(__fsub_rn(pc.pi.y, pj.y), sy);
                const float r2 = __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
                if (r2 < 1.0f && r2 > 1e-24f && j != d) pair_term(pc, j, ax, ay);
            }
        }
    }
}

// ---------------------------------------------------------------- angle terms and stirring

// The outer shares of one angle term of the triplet (i, j, k), theta the angle
// between a = x_j - x_i and c = x_k - x_j: kind 0, U = K (1 - cos theta) (the
// chain terms, chain_forces_linear, oercel.c:1290-1307); kind 1,
// U = K (cos theta - c0)^2 (the junction terms of branched lipids,
// mol_forces, oercel.c:1237-1256).  In fixed point: (qix, qiy) on the end i,
// (qkx, qky) on the end k; the middle bead j takes -(qi + qk), so the three
// shares cancel exactly.  Every rounding is explicit: each of the three beads
// recomputes the term from the same positions and gets the same bits.
__device__ __forceinline__ void angle_shares_g(float2 xi, float2 xj, float2 xk, int kind, float K, float c0, float L,
                                               float h, int &qix, int &qiy, int &qkx, int &qky) {
    const float ax = minimg(__fsub_rn(xj.x, xi.x), L, h), ay = minimg(__fsub_rn(xj.y, xi.y), L, h);
    const float cx = minimg(__fsub_rn(xk.x, xj.x), L, h), cy = minimg(__fsub_rn(xk.y, xj.y), L, h);
    const float la2 = __fmaf_rn(ax, ax, __fmul_rn(ay, ay)), lc2 = __fmaf_rn(cx, cx, __fmul_rn(cy, cy));
    const float ilac = __fdiv_rn(1.0f, __fmul_rn(__fsqrt_rn(la2), __fsqrt_rn(lc2)));
    const float cs = __fmul_rn(__fmaf_rn(ax, cx, __fmul_rn(ay, cy)), ilac);
    const float csa = __fdiv_rn(cs, la2), csc = __fdiv_rn(cs, lc2);
    // g = dU/dcos: kind 0, U = K (1 - cos): -K; kind 1, U = K (cos - c0)^2: 2 K (cos - c0) (oercel.c:1243-1245)
    // on i: dU/da = g (c / (la lc) - cos a / la^2); on k: -dU/dc = -g (a / (la lc) - cos c / lc^2)
    const float g = kind == 0 ? -K : __fmul_rn(2.0f * K, __fsub_rn(cs, c0));
    qix = f2fix16(__fmul_rn(g, __fsub_rn(__fmul_rn(cx, ilac), __fmul_rn(csa, ax))));
    qiy = f2fix16(__fmul_rn(g, __fsub_rn(__fmul_rn(cy, ilac), __fmul_rn(csa, ay))));
    qkx = f2fix16(__fmul_rn(-g, __fsub_rn(__fmul_rn(ax, ilac), __fmul_rn(csc, cx))));
    qky = f2fix16(__fmul_rn(-g, __fsub_rn(__fmul_rn(ay, ilac), __fmul_rn(csc, cy))));
}

// the straight-chain term U = ka (1 - cos) of the linear lipids
__device__ __forceinline__ void angle_shares(float2 xi, float2 xj, float2 xk, float ka, float L, float h, int &qix,
                                             int &qiy, int &qkx, int &qky) {
    angle_shares_g(xi, xj, xk, 0, ka, 0.0f, L, h, qix, qiy, qkx, qky);
}

// The angle shares of bead g at position pg with chain neighbours p (prev),
// n (next), pp (prev of p) and nn (next of n); has* say which exist.  g is
// the middle of (p, g, n), the end k of (pp, p, g) and the end i of (g, n, nn).
__device__ __forceinline__ void angle_sum(float ka, float L, float h, float2 pg, bool hp, float2 pp_, bool hn,
                                          float2 pn, bool hpp, float2 ppp, bool hnn, float2 pnn, long long &qx,
                                          long long &qy) {
    int ix, iy, kx, ky;
    if (hp && hn) {
        angle_shares(pp_, pg, pn, ka, L, h, ix, iy, kx, ky);
        qx -= (long long)ix + kx;
        qy -= (long long)iy + ky;
    }
    if (hp && hpp) {
        angle_shares(ppp, pp_, pg, ka, L, h, ix, iy, kx, ky);
        qx += kx;
        qy += ky;
    }
    if (hn && hnn) {
        angle_shares(pg, pn, pnn, ka, L, h, ix, iy, kx, ky);
        qx += ix;
        qy += iy;
    }
}

// The stirring term A sin(2 pi n y / L) of a bead at height y (oercel.c:1183),
// in fixed point.
__device__ __forceinline__ long long stir_fix(const RepDev &R, float y) {
    return __double2ll_rn((double)R.stir_A * sinpi(2.0 * R.stir_k * (double)y) * 65536.0);
}

// The stirring force of bead gid (fixed point): its term minus its share of
// the replica's sum S of all terms, the share being floor(S / n) plus one
// for gids below the remainder, so the shares add up to S exactly and the net
// stirring force is exactly zero (the reference subtracts the mean,
// oercel.c:1191-1195).
__device__ __forceinline__ long long stir_force(const RepDev &R, float y, uint32_t gid, long long S) {
    long long base = S / R.n;
    if (S - base * R.n < 0) base -= 1;
    const long long rem = S - base * R.n;
    return stir_fix(R, y) - base - ((long long)gid < rem ? 1 : 0);
}

// The angle terms of bead g (slot), added to its fixed-point force: pg its
// position, lk its links, pp_/pn the positions of its prev/next (valid where
// the link is).  Loads the second neighbours itself; nothing when ka = 0.
__device__ __forceinline__ void angle_terms(const Bufs &b, int cur, const RepDev &R, float2 pg, int2 lk, float2 pp_,
                                            float2 pn, long long &qx, long long &qy) {
    if (R.ka == 0.0f || (lk.x < 0 && lk.y < 0)) return;
    const int2 *__restrict__ link = b.link[cur];
    const float2 *__restrict__ pos = b.pos[cur];
    const int pp = lk.x >= 0 ? link[lk.x].x : -1, nn = lk.y >= 0 ? link[lk.y].y : -1;
    const float2 ppp = pp >= 0 ? pos[pp] : pg, pnn = nn >= 0 ? pos[nn] : pg;
    angle_sum(R.ka, R.L, R.halfL, pg, lk.x >= 0, pp_, lk.y >= 0, pn, pp >= 0, ppp, nn >= 0, pnn, qx, qy);
}

// ---------------------------------------------------------------- programmatic dependent launch

// The kernels of a step are launched with programmatic stream serialization
// (launch_pdl): a kernel may be scheduled while its predecessor drains.  It
// waits for the predecessor's completion (and its memory) before touching
// anything, and lets its own successor be scheduled once all its CTAs run.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_begin() {
    pdl_wait();
    pdl_trigger();
}

// ---------------------------------------------------------------- grid helpers

// True in the last CTA of the grid to get here, after every CTA's writes are
// visible to it (fence, then a counter; nothing waits).  The last CTA resets
// the counter for the next launch.
__device__ __forceinline__ bool last_cta(unsigned int *done) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        last = atomicAdd(done, 1u) == gridDim.x - 1;
        if (last) *done = 0u;
    }
    __syncthreads();
    if (last) __threadfence();
    return last;
}

// ---------------------------------------------------------------- warp helpers

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

// count a bead into its next cell (no value returned: the add is fire-and-forget)
__device__ __forceinline__ void count_key(uint32_t *count, uint32_t key, bool active) {
    if (active) atomicAdd(count + key, 1u);
}

__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ void raise_flag(DevStatus *st, unsigned f) { atomicOr(&st->flags, f); }
