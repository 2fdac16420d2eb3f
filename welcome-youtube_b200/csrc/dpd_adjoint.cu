// dpd_adjoint.cu -- reverse mode through the DPD step (sm_100a).
//
// k_force_vjp    vector-Jacobian product of the pair + bond forces of one
//                configuration: given the cotangent g of the forces, the
//                gradients with respect to positions, predicted velocities,
//                the repulsions a_ij, gamma and the bond constant.  The pair
//                noise theta is replayed from its key (frozen noise).
// k_rdf_smooth   Gaussian-smoothed pair distribution of two bead types
//                (the structural target of a fit) and k_rdf_vjp its gradient.
// k_adj_update   the adjoint of the Groot-Warren update, with the adjoint
//                state kept in gid order so the sort of every step does not
//                matter.
//
// Pair term (w = 1 - r, A = a - gamma w rv + s theta, s = sigma / sqrt(dt)):
//   f = fm d,  fm = w A / r,  rv = d . dv / r
//   d(c.f)/dd  = (c.d) [dfm/dr dhat + dfm/drv (dv - rv dhat) / r] + fm c
//   d(c.f)/ddv = (c.d) dfm/drv dhat
//   dfm/dr  = (-A + w gamma rv) / r - w A / r^2,   dfm/drv = -gamma w^2 / r
//   d(c.f)/da_ij = (c.d) w / r,  d(c.f)/dgamma = (c.d) w (-w rv + s theta / (2 gamma)) / r
// with c = g_i - g_j for the pair (i, j).  Every bead sums over its 3x3 cells
// (each pair from both ends; the two halves are exact negatives), the
// parameter gradients count each pair once.
#include "dpd_device.cuh"

#define NGRAD DPD_NGRAD

__device__ __forceinline__ float theta_of(const NoiseKey &nk, uint32_t gi, uint32_t gj) { return pair_theta(nk, gi, gj); }

__global__ void __launch_bounds__(BEAD_TPB) k_force_vjp(StateView sv, long long step, const RepDev *__restrict__ reps,
                                                        const Chunk *__restrict__ ch, const float2 *__restrict__ g,
                                                        float2 *__restrict__ xbar, float2 *__restrict__ vbar,
                                                        double *__restrict__ grad) {
    __shared__ double sgrad[NGRAD];
    for (int k = threadIdx.x; k < NGRAD; k += blockDim.x) sgrad[k] = 0.0;
    __syncthreads();
    const Chunk c = ch[blockIdx.x];
    const RepDev &R = reps[c.rep];
    const int d = c.begin + (int)threadIdx.x;
    if (d < c.end) {
        const float2 pi = sv.pos[d], vi = sv.vt[d], gi2 = g[d];
        const uint32_t tgi = sv.tg[d], gi = tgi & GID_MASK;
        const int ti = (int)(tgi >> TYPE_SHIFT);
        const float L = R.L, h = R.halfL, gam = R.gamma, s = R.sdt;
        const NoiseKey nk = make_noise_key(R, step);
        const int ncx = R.ncx, ncy = R.ncy;
        const int32_t *cs = sv.cstart + R.c0;
        int cx, cy;
        cell_xy(R, pi.x, pi.y, cx, cy);
        float xbx = 0.f, xby = 0.f, vbx = 0.f, vby = 0.f;
        double ggam = 0.0;
        for (int ox = -1; ox <= 1; ox++)
            for (int oy = -1; oy <= 1; oy++) {
                const int cc = ((cx + ox + ncx) % ncx) * ncy + (cy + oy + ncy) % ncy;
                for (int j = cs[cc]; j < cs[cc + 1]; j++) {
                    if (j == d) continue;
                    const float2 pj = sv.pos[j];
                    const float dx = minimg(__fsub_rn(pi.x, pj.x), L, h), dy = minimg(__fsub_rn(pi.y, pj.y), L, h);
                    const float r2 = __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
                    if (!(r2 < 1.0f && r2 > 1e-24f)) continue;
                    const float2 vj = sv.vt[j], gj = g[j];
                    const uint32_t tgj = sv.tg[j];
                    const int tj = (int)(tgj >> TYPE_SHIFT);
                    float r, ir;
                    r_and_ir(r2, r, ir);
                    const float w = 1.0f - r;
                    const float dvx = vi.x - vj.x, dvy = vi.y - vj.y;
                    const float rv = (dx * dvx + dy * dvy) * ir;
                    const float th = theta_of(nk, gi, tgj & GID_MASK);
                    const float a = R.a[ti * DPD_MAXT + tj];
                    const float A = a - gam * w * rv + s * th;
                    const float fm = w * A * ir;
                    const float cxv = gi2.x - gj.x, cyv = gi2.y - gj.y;
                    const float cd = cxv * dx + cyv * dy;
                    const float dfr = (-A + w * gam * rv) * ir - w * A * ir * ir;
                    const float dfv = -gam * w * w * ir;
                    const float hx = dx * ir, hy = dy * ir;
                    xbx += cd * (dfr * hx + dfv * (dvx - rv * hx) * ir) + fm * cxv;
                    xby += cd * (dfr * hy + dfv * (dvy - rv * hy) * ir) + fm * cyv;
                    vbx += cd * dfv * hx;
                    vby += cd * dfv * hy;
                    if (gi < (tgj & GID_MASK)) {  // parameter gradients: each pair once
                        const int lo = min(ti, tj), hi = max(ti, tj);
                        atomicAdd(&sgrad[lo * DPD_MAXT + hi], (double)(cd * w * ir));
                        ggam += (double)(cd * w * (-w * rv + (gam > 0.0f ? s * th / (2.0f * gam) : 0.0f)) * ir);
                    }
                }
            }
        // bonds: f_i = kb (1 - r0/r) d with d = x_p - x_i
        const int2 lk = sv.link[d];
        double gkb = 0.0;
        for (int q = 0; q < 2; q++) {
            const int p = q ? lk.y : lk.x;
            if (p < 0) continue;
            const float2 pp = sv.pos[p], gp = g[p];
            const float dx = minimg(pp.x - pi.x, L, h), dy = minimg(pp.y - pi.y, L, h);
            const float r = sqrtf(dx * dx + dy * dy);
            const float cxv = gi2.x - gp.x, cyv = gi2.y - gp.y;
            const float cd = cxv * dx + cyv * dy;
            const float u = 1.0f - R.r0 / r;
            const float k0 = R.kb * R.r0 / (r * r) * cd / r;
            xbx -= k0 * dx + R.kb * u * cxv;
            xby -= k0 * dy + R.kb * u * cyv;
            if (q == 1) gkb += (double)(u * cd);  // each bond once, from its prev end
        }
        xbar[d] = make_float2(xbx, xby);
        vbar[d] = make_float2(vbx, vby);
        if (ggam != 0.0) atomicAdd(&sgrad[DPD_MAXT * DPD_MAXT], ggam);
        if (gkb != 0.0) atomicAdd(&sgrad[DPD_MAXT * DPD_MAXT + 1], gkb);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < NGRAD; k += blockDim.x)
        if (sgrad[k] != 0.0) atomicAdd(&grad[(size_t)c.rep * NGRAD + k], sgrad[k]);
}

// Gaussian-smoothed distribution of (ta, tb) pairs: h_b += K(r - r_b) dr for
// each unordered pair with r < rmax + 4 sigma, K the unit Gaussian of width sigma
struct RdfConst {
    int ta, tb, nbin;
    float rmax, sigma;
};

__device__ __forceinline__ bool rdf_types(const RdfConst &q, int ti, int tj) {
    return (ti == q.ta && tj == q.tb) || (ti == q.tb && tj == q.ta);
}

template <bool VJP>
__global__ void __launch_bounds__(BEAD_TPB) k_rdf(StateView sv, const RepDev *__restrict__ reps,
                                                  const Chunk *__restrict__ ch, RdfConst q, double *__restrict__ hist,
                                                  const double *__restrict__ wgt, float2 *__restrict__ xadd,
                                                  const uint32_t *__restrict__ gid_map) {
    extern __shared__ double sh[];
    const Chunk c = ch[blockIdx.x];
    if (!VJP) {
        for (int k = threadIdx.x; k < q.nbin; k += blockDim.x) sh[k] = 0.0;
        __syncthreads();
    }
    const RepDev &R = reps[c.rep];
    const int d = c.begin + (int)threadIdx.x;
    if (d < c.end) {
        const uint32_t tgi = sv.tg[d];
        const int ti = (int)(tgi >> TYPE_SHIFT);
        if (ti == q.ta || ti == q.tb) {
            const float2 pi = sv.pos[d];
            const float L = R.L, h = R.halfL;
            const float rc = q.rmax + 4.0f * q.sigma, dr = q.rmax / q.nbin;
            const float inv2s2 = 0.5f / (q.sigma * q.sigma), kn = dr * 0.3989422804f / q.sigma;
            const int ncx = R.ncx, ncy = R.ncy;
            const int rcell = min((int)ceilf(rc * (float)R.icsx), (min(ncx, ncy) - 1) / 2);
            const int32_t *cs = sv.cstart + R.c0;
            int cx, cy;
            cell_xy(R, pi.x, pi.y, cx, cy);
            const double *wr = VJP ? wgt + (size_t)c.rep * q.nbin : nullptr;
            float gx = 0.f, gy = 0.f;
            for (int ox = -rcell; ox <= rcell; ox++)
                for (int oy = -rcell; oy <= rcell; oy++) {
                    const int cc = ((cx + ox + ncx) % ncx) * ncy + (cy + oy + ncy) % ncy;
                    for (int j = cs[cc]; j < cs[cc + 1]; j++) {
                        if (j == d) continue;
                        if (!VJP && j < d) continue;  // the histogram counts each pair once
                        if (!rdf_types(q, ti, (int)(sv.tg[j] >> TYPE_SHIFT))) continue;
                        const float2 pj = sv.pos[j];
                        const float dx = minimg(pi.x - pj.x, L, h), dy = minimg(pi.y - pj.y, L, h);
                        const float r = sqrtf(dx * dx + dy * dy);
                        if (!(r < rc) || r == 0.0f) continue;
                        const int b0 = max(0, (int)floorf((r - 4.0f * q.sigma) / dr));
                        const int b1 = min(q.nbin - 1, (int)floorf((r + 4.0f * q.sigma) / dr));
                        float dldr = 0.f;
                        for (int b = b0; b <= b1; b++) {
                            const float rb = (b + 0.5f) * dr, e = r - rb;
                            const float k = kn * __expf(-e * e * inv2s2);
                            if (VJP) dldr += (float)wr[b] * k * (-e * 2.0f * inv2s2);
                            else atomicAdd(&sh[b], (double)k);
                        }
                        if (VJP) {
                            gx += dldr * dx / r;
                            gy += dldr * dy / r;
                        }
                    }
                }
            if (VJP) {
                const uint32_t gg = gid_map ? (tgi & GID_MASK) + (uint32_t)R.b0 : (uint32_t)d;
                float2 x = xadd[gg];
                xadd[gg] = make_float2(x.x + gx, x.y + gy);
            }
        }
    }
    if (!VJP) {
        __syncthreads();
        for (int k = threadIdx.x; k < q.nbin; k += blockDim.x)
            if (sh[k] != 0.0) atomicAdd(&hist[(size_t)c.rep * q.nbin + k], sh[k]);
    }
}

// Adjoint of one Groot-Warren step, slot order of the configuration n+1 mapped
// to gid order (packed: gid + b0 of the replica):
//   x_bar(n)  = x_bar(n+1) + J_x^T F_bar
//   vh_bar(n) = dt x_bar(n) + vh_bar(n+1) + J_v^T F_bar
//   F_bar(n)  = dt^2 x_bar(n) + dt vh_bar(n+1) + cvt J_v^T F_bar
// (X, V, F hold x_bar, vh_bar, F_bar in gid order; xb, vb are J_x^T F_bar, J_v^T F_bar in slot order)
__global__ void __launch_bounds__(BEAD_TPB) k_adj_update(const uint32_t *__restrict__ tg, const RepDev *__restrict__ reps,
                                                         const Chunk *__restrict__ ch, const float2 *__restrict__ xb,
                                                         const float2 *__restrict__ vb, float2 *__restrict__ X,
                                                         float2 *__restrict__ V, float2 *__restrict__ F) {
    const Chunk c = ch[blockIdx.x];
    const int d = c.begin + (int)threadIdx.x;
    if (d >= c.end) return;
    const RepDev &R = reps[c.rep];
    const uint32_t g = (tg[d] & GID_MASK) + (uint32_t)R.b0;
    const float2 x0 = X[g], v0 = V[g], xf = xb[d], vf = vb[d];
    const float2 x = make_float2(x0.x + xf.x, x0.y + xf.y);
    X[g] = x;
    V[g] = make_float2(R.dt * x.x + v0.x + vf.x, R.dt * x.y + v0.y + vf.y);
    F[g] = make_float2(R.dt2 * x.x + R.dt * v0.x + R.cvt * vf.x, R.dt2 * x.y + R.dt * v0.y + R.cvt * vf.y);
}

// gather F_bar (gid order) into slot order of one configuration
__global__ void __launch_bounds__(BEAD_TPB) k_adj_gather(const uint32_t *__restrict__ tg, const RepDev *__restrict__ reps,
                                                         const Chunk *__restrict__ ch, const float2 *__restrict__ F,
                                                         float2 *__restrict__ g) {
    const Chunk c = ch[blockIdx.x];
    const int d = c.begin + (int)threadIdx.x;
    if (d >= c.end) return;
    g[d] = F[(tg[d] & GID_MASK) + (uint32_t)reps[c.rep].b0];
}

// cotangents of the window's start state in gid order: x_bar(0) gains the part
// that flows through the start forces (xb = J_x^T F_bar(0)), and the predicted
// velocity's cotangent is that force VJP's vb; vh_bar(0) is V as it stands
__global__ void __launch_bounds__(BEAD_TPB) k_adj_state(const uint32_t *__restrict__ tg, const RepDev *__restrict__ reps,
                                                        const Chunk *__restrict__ ch, const float2 *__restrict__ xb,
                                                        const float2 *__restrict__ vb, float2 *__restrict__ X,
                                                        float2 *__restrict__ VT) {
    const Chunk c = ch[blockIdx.x];
    const int d = c.begin + (int)threadIdx.x;
    if (d >= c.end) return;
    const uint32_t g = (tg[d] & GID_MASK) + (uint32_t)reps[c.rep].b0;
    const float2 x = X[g], a = xb[d];
    X[g] = make_float2(x.x + a.x, x.y + a.y);
    VT[g] = vb[d];
}

// copy a configuration out of the engine's buffers (for recomputation)
__global__ void k_adj_save(int n, const float2 *pos, const float2 *vt, const uint32_t *tg, const int2 *link,
                           float2 *opos, float2 *ovt, uint32_t *otg, int2 *olink) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    opos[k] = pos[k];
    ovt[k] = vt[k];
    otg[k] = tg[k];
    olink[k] = link[k];
}

void launch_force_vjp(const StateView &sv, long long step, const RepDev *rep, const Chunk *bch, int nbch,
                      const float2 *g, float2 *xbar, float2 *vbar, double *grad, cudaStream_t s) {
    k_force_vjp<<<nbch, BEAD_TPB, 0, s>>>(sv, step, rep, bch, g, xbar, vbar, grad);
}

void launch_rdf(const StateView &sv, const RepDev *rep, const Chunk *bch, int nbch, int ta, int tb, int nbin,
                float rmax, float sigma, double *hist, cudaStream_t s) {
    RdfConst q{ta, tb, nbin, rmax, sigma};
    k_rdf<false><<<nbch, BEAD_TPB, nbin * sizeof(double), s>>>(sv, rep, bch, q, hist, nullptr, nullptr, nullptr);
}

void launch_rdf_vjp(const StateView &sv, const RepDev *rep, const Chunk *bch, int nbch, int ta, int tb, int nbin,
                    float rmax, float sigma, const double *wgt, float2 *xadd_gid, cudaStream_t s) {
    RdfConst q{ta, tb, nbin, rmax, sigma};
    k_rdf<true><<<nbch, BEAD_TPB, 0, s>>>(sv, rep, bch, q, nullptr, wgt, xadd_gid, sv.tg);
}

void launch_adj_update(const uint32_t *tg, const RepDev *rep, const Chunk *bch, int nbch, const float2 *xb,
                       const float2 *vb, float2 *X, float2 *V, float2 *F, cudaStream_t s) {
    k_adj_update<<<nbch, BEAD_TPB, 0, s>>>(tg, rep, bch, xb, vb, X, V, F);
}

void launch_adj_gather(const uint32_t *tg, const RepDev *rep, const Chunk *bch, int nbch, const float2 *F, float2 *g,
                       cudaStream_t s) {
    k_adj_gather<<<nbch, BEAD_TPB, 0, s>>>(tg, rep, bch, F, g);
}

void launch_adj_state(const uint32_t *tg, const RepDev *rep, const Chunk *bch, int nbch, const float2 *xb,
                      const float2 *vb, float2 *X, float2 *VT, cudaStream_t s) {
    k_adj_state<<<nbch, BEAD_TPB, 0, s>>>(tg, rep, bch, xb, vb, X, VT);
}

void launch_adj_save(int n, const float2 *pos, const float2 *vt, const uint32_t *tg, const int2 *link, float2 *opos,
                     float2 *ovt, uint32_t *otg, int2 *olink, cudaStream_t s) {
    k_adj_save<<<(n + 255) / 256, 256, 0, s>>>(n, pos, vt, tg, link, opos, ovt, otg, olink);
}
