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
// parameter gradients count each pair once.  s follows the temperature cycle
// (s(step) = sqrt(2 gamma kT(t) / dt)), as the forward forces do.
//
// Angle terms (U = K (1 - cos), or K (cos - c0)^2 at the junctions of the
// branched shapes, per triplet i-j-k, a = x_j - x_i, c = x_k - x_j): with
// F = -grad U the VJP on bead m is -d phi / d x_m, phi = sum over beads of
// g . dU/dx = D U(a, c)[da, dc], da = g_j - g_i, dc = g_k - g_j.  dphi/da and
// dphi/dc are Hessian-vector products of U, written out in angle_hvp; then
// d/dx_i = -d/da, d/dx_j = d/da - d/dc, d/dx_k = d/dc.  Linear chains: each
// bead gathers the triplets it is part of (as middle, as last of its prev's,
// as first of its next's), so no two threads write one bead.  Branched
// shapes: k_mol_vjp, one thread per molecule.
//
// Stirring (f_x,i = A sin(2 pi k y_i) minus its replica mean): the VJP on y_m
// is A 2 pi k cos(2 pi k y_m) (g_x,m - mean of g_x), the mean from k_gsum.
#include "dpd_device.cuh"

#define NGRAD DPD_NGRAD

__device__ __forceinline__ float theta_of(const NoiseKey &nk, uint32_t gi, uint32_t gj) { return pair_theta(nk, gi, gj); }

__device__ __forceinline__ float dot2(float2 u, float2 v) { return u.x * v.x + u.y * v.y; }

// dphi/da (pa) and dphi/dc (pc) of phi = D U(a, c)[da, dc] for an angle term
// U(cos) of kind 0, U = K (1 - cos) (U' = -K, U'' = 0), or kind 1,
// U = K (cos - c0)^2 (U' = 2 K (cos - c0), U'' = 2 K):
//   cos = (a.c) / (|a| |c|),  Dcos = q / AC - cos (a.da) / A2 - cos (c.dc) / C2,  q = da.c + a.dc
//   dDcos/da = dc / AC - q a / (AC A2) - gca ((a.da) / A2 + (c.dc) / C2) - cos (da / A2 - 2 (a.da) a / A2^2)
//   dDcos/dc = da / AC - q c / (AC C2) - gcc ((a.da) / A2 + (c.dc) / C2) - cos (dc / C2 - 2 (c.dc) c / C2^2)
// with gca = dcos/da = c / AC - cos a / A2, gcc = dcos/dc = a / AC - cos c / C2;
// phi = U' Dcos, so dphi/da = U'' Dcos gca + U' dDcos/da (and likewise for c)
__device__ __forceinline__ void angle_hvp(float2 a, float2 c, float2 da, float2 dc, int kind, float K, float c0,
                                          float2 &pa, float2 &pc) {
    const float A2 = dot2(a, a), C2 = dot2(c, c);
    const float iac = rsqrtf(A2 * C2), iA2 = 1.0f / A2, iC2 = 1.0f / C2;
    const float cs = dot2(a, c) * iac;
    const float q = dot2(da, c) + dot2(a, dc), ada = dot2(a, da), cdc = dot2(c, dc);
    const float m = ada * iA2 + cdc * iC2;
    const float2 gca = make_float2(c.x * iac - cs * a.x * iA2, c.y * iac - cs * a.y * iA2);
    const float2 gcc = make_float2(a.x * iac - cs * c.x * iC2, a.y * iac - cs * c.y * iC2);
    const float ta = q * iac * iA2, tc = q * iac * iC2;
    const float ka2 = 2.0f * ada * iA2 * iA2, kc2 = 2.0f * cdc * iC2 * iC2;
    const float u1 = kind == 0 ? -K : 2.0f * K * (cs - c0), u2 = kind == 0 ? 0.0f : 2.0f * K;
    const float dcos = q * iac - cs * m;
    pa = make_float2(u2 * dcos * gca.x + u1 * (dc.x * iac - ta * a.x - gca.x * m - cs * (da.x * iA2 - ka2 * a.x)),
                     u2 * dcos * gca.y + u1 * (dc.y * iac - ta * a.y - gca.y * m - cs * (da.y * iA2 - ka2 * a.y)));
    pc = make_float2(u2 * dcos * gcc.x + u1 * (da.x * iac - tc * c.x - gcc.x * m - cs * (dc.x * iC2 - kc2 * c.x)),
                     u2 * dcos * gcc.y + u1 * (da.y * iac - tc * c.y - gcc.y * m - cs * (dc.y * iC2 - kc2 * c.y)));
}

// the angle-term VJP of a bead of a linear chain at pi with cotangent gi and
// links lk (x_bar increment): the triplets (p, d, n), (pp, p, d) and
// (d, n, nn) of its chain, where they exist
__device__ __forceinline__ float2 angle_vjp(const StateView &sv, const float2 *__restrict__ g, const RepDev &R, float2 pi,
                                           float2 gi, int2 lk) {
    const float L = R.L, h = R.halfL, ka = R.ka;
    float2 out = make_float2(0.0f, 0.0f);
    auto vec = [&](float2 u, float2 v) {  // v - u, minimum image
        return make_float2(minimg(v.x - u.x, L, h), minimg(v.y - u.y, L, h));
    };
    auto dif = [](float2 u, float2 v) { return make_float2(v.x - u.x, v.y - u.y); };
    float2 pp_ = pi, pn = pi, gp = gi, gn = gi;
    if (lk.x >= 0) {
        pp_ = sv.pos[lk.x];
        gp = g[lk.x];
    }
    if (lk.y >= 0) {
        pn = sv.pos[lk.y];
        gn = g[lk.y];
    }
    float2 pa, pc;
    if (lk.x >= 0 && lk.y >= 0) {  // the bead in the middle: -(dphi/da - dphi/dc)
        angle_hvp(vec(pp_, pi), vec(pi, pn), dif(gp, gi), dif(gi, gn), 0, ka, 0.0f, pa, pc);
        out.x -= pa.x - pc.x;
        out.y -= pa.y - pc.y;
    }
    if (lk.x >= 0) {
        const int q = sv.link[lk.x].x;
        if (q >= 0) {  // (q, p, d): the bead last, -dphi/dc
            const float2 pq = sv.pos[q], gq = g[q];
            angle_hvp(vec(pq, pp_), vec(pp_, pi), dif(gq, gp), dif(gp, gi), 0, ka, 0.0f, pa, pc);
            out.x -= pc.x;
            out.y -= pc.y;
        }
    }
    if (lk.y >= 0) {
        const int q = sv.link[lk.y].y;
        if (q >= 0) {  // (d, n, q): the bead first, +dphi/da
            const float2 pq = sv.pos[q], gq = g[q];
            angle_hvp(vec(pi, pn), vec(pn, pq), dif(gi, gn), dif(gn, gq), 0, ka, 0.0f, pa, pc);
            out.x += pa.x;
            out.y += pa.y;
        }
    }
    return out;
}

// per replica, the sum of the x cotangents (the stirring term's mean)
__global__ void __launch_bounds__(BEAD_TPB) k_gsum(const RepDev *__restrict__ reps, const Chunk *__restrict__ ch,
                                                   const float2 *__restrict__ g, double *__restrict__ gsum) {
    const Chunk c = ch[blockIdx.x];
    if (reps[c.rep].stir_A == 0.0f) return;
    const int d = c.begin + (int)threadIdx.x;
    double v = d < c.end ? (double)g[d].x : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane_id() == 0 && v != 0.0) atomicAdd(gsum + c.rep, v);
}

__global__ void __launch_bounds__(BEAD_TPB) k_force_vjp(StateView sv, long long step, const RepDev *__restrict__ reps,
                                                        const Chunk *__restrict__ ch, const float2 *__restrict__ g,
                                                        float2 *__restrict__ xbar, float2 *__restrict__ vbar,
                                                        double *__restrict__ grad, const double *__restrict__ gsum,
                                                        const long long *__restrict__ step_base) {
    if (step_base) step += *step_base;  // the step relative to a step number kept on the device
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
        const float L = R.L, h = R.halfL, gam = R.gamma, s = sdt_at(R, step);
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
        // bonds: f_i = kb (1 - r0/r) d with d = x_p - x_i (linear chains; the
        // branched shapes' bonds and angles are k_mol_vjp's)
        const int2 lk = R.arch == 0 ? sv.link[d] : make_int2(-1, -1);
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
        if (R.ka != 0.0f && (lk.x >= 0 || lk.y >= 0)) {
            const float2 t = angle_vjp(sv, g, R, pi, gi2, lk);
            xbx += t.x;
            xby += t.y;
        }
        if (R.stir_A != 0.0f) {
            const double w2 = 2.0 * R.stir_k;
            const double dfy = (double)R.stir_A * M_PI * w2 * cospi(w2 * (double)pi.y);
            xby += (float)(dfy * ((double)gi2.x - gsum[c.rep] / (double)R.n));
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

// The bonded terms of the branched shapes (the template terms of
// k_mol_forces): one thread per molecule (its first bead) adds each of its
// beads' share to x_bar after k_force_vjp, so no two threads write one bead.
// Bond (i, j), d = x_j - x_i, F_i = kb (1 - r0/r) d = -F_j, c = g_i - g_j:
//   d(c.F_i)/dd = kb ((1 - r0/r) c + r0 (c.d) d / r^3),  d(c.F_i)/dkb = (1 - r0/r) (c.d)
// Angle (i, j, k): x_bar_i += dphi/da, x_bar_j -= dphi/da - dphi/dc, x_bar_k -= dphi/dc.
__global__ void __launch_bounds__(BEAD_TPB) k_mol_vjp(StateView sv, const RepDev *__restrict__ reps,
                                                      const Chunk *__restrict__ ch, const dpd_template *__restrict__ mol,
                                                      const float2 *__restrict__ g, float2 *__restrict__ xbar,
                                                      double *__restrict__ grad) {
    const Chunk c = ch[blockIdx.x];
    const RepDev &R = reps[c.rep];
    if (R.arch == 0) return;
    const int d = c.begin + (int)threadIdx.x;
    double gkb = 0.0;
    if (d < c.end) {
        const int2 lk0 = sv.link[d];
        if (lk0.x < 0 && lk0.y >= 0) {
            const dpd_template &M = mol[c.rep];
            const int ml = M.mlen;
            int sl[DPD_MAXML];
            float2 p[DPD_MAXML], gg[DPD_MAXML], xb[DPD_MAXML];
            int n = 0;
            for (int q = d; q >= 0 && n < ml; q = sv.link[q].y) {
                sl[n] = q;
                p[n] = sv.pos[q];
                gg[n] = g[q];
                xb[n] = make_float2(0.0f, 0.0f);
                n++;
            }
            if (n == ml) {  // (an incomplete molecule raised DPD_F_CHAIN in the forward pass)
                const float L = R.L, h = R.halfL, kb = R.kb;
                for (int q = 0; q < M.nb; q++) {
                    const int i = M.bi[q], j = M.bj[q];
                    const float dx = minimg(p[j].x - p[i].x, L, h), dy = minimg(p[j].y - p[i].y, L, h);
                    const float r = sqrtf(dx * dx + dy * dy), r0 = (float)M.br0[q];
                    const float cx = gg[i].x - gg[j].x, cy = gg[i].y - gg[j].y, cd = cx * dx + cy * dy;
                    const float u = 1.0f - r0 / r, k3 = kb * r0 * cd / (r * r * r);
                    const float tx = kb * u * cx + k3 * dx, ty = kb * u * cy + k3 * dy;  // d(c.F_i)/dd
                    xb[i].x -= tx;
                    xb[i].y -= ty;
                    xb[j].x += tx;
                    xb[j].y += ty;
                    gkb += (double)(u * cd);
                }
                for (int q = 0; q < M.na; q++) {
                    const int i = M.ai[q], j = M.aj[q], k = M.ak[q];
                    const float2 a = make_float2(minimg(p[j].x - p[i].x, L, h), minimg(p[j].y - p[i].y, L, h));
                    const float2 cc = make_float2(minimg(p[k].x - p[j].x, L, h), minimg(p[k].y - p[j].y, L, h));
                    const float2 da = make_float2(gg[j].x - gg[i].x, gg[j].y - gg[i].y);
                    const float2 dc = make_float2(gg[k].x - gg[j].x, gg[k].y - gg[j].y);
                    float2 pa, pc;
                    angle_hvp(a, cc, da, dc, M.akind[q], (float)M.aK[q], (float)M.ac0[q], pa, pc);
                    xb[i].x += pa.x;
                    xb[i].y += pa.y;
                    xb[j].x -= pa.x - pc.x;
                    xb[j].y -= pa.y - pc.y;
                    xb[k].x -= pc.x;
                    xb[k].y -= pc.y;
                }
                for (int e = 0; e < ml; e++) {
                    const float2 o = xbar[sl[e]];
                    xbar[sl[e]] = make_float2(o.x + xb[e].x, o.y + xb[e].y);
                }
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) gkb += __shfl_down_sync(0xffffffffu, gkb, o);
    if (lane_id() == 0 && gkb != 0.0) atomicAdd(&grad[(size_t)c.rep * NGRAD + DPD_MAXT * DPD_MAXT + 1], gkb);
}

void launch_force_vjp(const StateView &sv, long long step, const RepDev *rep, const Chunk *bch, int nbch,
                      const float2 *g, float2 *xbar, float2 *vbar, double *grad, double *gsum, int nrep, bool stir,
                      const dpd_template *mol, cudaStream_t s, const long long *step_base) {
    if (stir) {
        cudaMemsetAsync(gsum, 0, (size_t)nrep * sizeof(double), s);
        k_gsum<<<nbch, BEAD_TPB, 0, s>>>(rep, bch, g, gsum);
    }
    k_force_vjp<<<nbch, BEAD_TPB, 0, s>>>(sv, step, rep, bch, g, xbar, vbar, grad, gsum, step_base);
    if (mol) k_mol_vjp<<<nbch, BEAD_TPB, 0, s>>>(sv, rep, bch, mol, g, xbar, grad);
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

// ---------------------------------------------------------------- a fit iteration without the host
//
// dpd_fit_graph captures one optimizer iteration (the window, its adjoint, the
// loss and the parameter update) as a CUDA graph and replays it: every value
// that changes from one iteration to the next lives on the device (FitDev).

__global__ void k_fit_begin(const long long *__restrict__ step, FitDev *__restrict__ fd) { fd->base = *step; }

__global__ void k_set_step_rel(long long *__restrict__ step, const FitDev *__restrict__ fd, long long off) {
    *step = fd->base + off;
}

// The smoothed-RDF loss of each replica (one block each) and the weights dL/dh
// of its bins, as the host computes them for dpd_window_adjoint:
// g = h / last_steps * L^2 / (npairs 2 pi r_b dr), loss = mean over bins of
// (g - target)^2, w = 2 (g - target) / nbin * L^2 / (npairs 2 pi r_b dr) / last_steps.
// The loss goes to loss_out[iter * nrep + replica].
__global__ void k_rdf_loss(const RepDev *__restrict__ reps, const double *__restrict__ hist,
                           const long long *__restrict__ npairs, const double *__restrict__ target, int nbin,
                           double rmax, int last_steps, double *__restrict__ loss_out, double *__restrict__ wgt,
                           const FitDev *__restrict__ fd) {
    __shared__ double red[32];
    const int r = (int)blockIdx.x, nrep = (int)gridDim.x;
    const double L = (double)reps[r].L, area = L * L, dr = rmax / nbin;
    const long long np = npairs[r];
    double sum = 0.0;
    for (int b = (int)threadIdx.x; b < nbin; b += (int)blockDim.x) {
        const double rb = (b + 0.5) * dr;
        const double norm = np > 0 ? area / ((double)np * 2.0 * M_PI * rb * dr) : 0.0;
        const double g = hist[(size_t)r * nbin + b] / last_steps * norm;
        const double e = g - target[(size_t)r * nbin + b];
        sum += e * e;
        wgt[(size_t)r * nbin + b] = 2.0 * e / nbin * norm / last_steps;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
    if (lane_id() == 0) red[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
        loss_out[(size_t)fd->iter * nrep + r] = t / nbin;
    }
}

// The optimizer step of the shared a_ij (one thread per fitted slot): the
// gradient summed over the replicas in replica order, then Adam as
// torch.optim.Adam takes it (no weight decay): m += (1 - b1)(g - m),
// v = b2 v + (1 - b2) g^2, a -= lr / (1 - b1^t) m / (sqrt(v) / sqrt(1 - b2^t) + eps).
// The new value goes into a_ij and a_ji of every replica; the gradient and the
// value the window ran with go to grad_out / value_out[iter * nfit + k].
__global__ void k_fit_update(RepDev *__restrict__ reps, int nrep, const double *__restrict__ grad,
                             FitDev *__restrict__ fd, double *__restrict__ grad_out, double *__restrict__ value_out) {
    const int k = (int)threadIdx.x, it = fd->iter;
    if (k < fd->nfit) {
        const int slot = fd->slot[k];
        double g = 0.0;
        for (int r = 0; r < nrep; r++) g += grad[(size_t)r * NGRAD + slot];
        const double t = (double)(it + 1);
        const double m = fd->m[k] + (1.0 - fd->beta1) * (g - fd->m[k]);
        const double v = fd->beta2 * fd->v[k] + (1.0 - fd->beta2) * g * g;
        fd->m[k] = m;
        fd->v[k] = v;
        const double bc1 = 1.0 - pow(fd->beta1, t), bc2 = 1.0 - pow(fd->beta2, t);
        const double denom = sqrt(v) / sqrt(bc2) + fd->eps;
        const double val = fd->value[k] - fd->lr / bc1 * m / denom;
        grad_out[(size_t)it * fd->nfit + k] = g;
        value_out[(size_t)it * fd->nfit + k] = fd->value[k];
        fd->value[k] = val;
        const int i = slot / DPD_MAXT, j = slot % DPD_MAXT;
        for (int r = 0; r < nrep; r++) {
            reps[r].a[i * DPD_MAXT + j] = (float)val;
            reps[r].a[j * DPD_MAXT + i] = (float)val;
        }
    }
    __syncthreads();
    if (k == 0) fd->iter = it + 1;
}

void launch_fit_begin(long long *step, FitDev *fd, cudaStream_t s) { k_fit_begin<<<1, 1, 0, s>>>(step, fd); }

void launch_set_step_rel(long long *step, const FitDev *fd, long long off, cudaStream_t s) {
    k_set_step_rel<<<1, 1, 0, s>>>(step, fd, off);
}

void launch_rdf_loss(const RepDev *rep, int nrep, const double *hist, const long long *npairs, const double *target,
                     int nbin, double rmax, int last_steps, double *loss_out, double *wgt, const FitDev *fd,
                     cudaStream_t s) {
    k_rdf_loss<<<nrep, 256, 0, s>>>(rep, hist, npairs, target, nbin, rmax, last_steps, loss_out, wgt, fd);
}

void launch_fit_update(RepDev *rep, int nrep, const double *grad, FitDev *fd, double *grad_out, double *value_out,
                       cudaStream_t s) {
    k_fit_update<<<1, DPD_MAXT * DPD_MAXT, 0, s>>>(rep, nrep, grad, fd, grad_out, value_out);
}
