// dpd_mol.cu -- lipid molecule templates (linear, pi, y, bola) and the bonded
// forces of the branched shapes.
//
// A template lists a lipid's bonds (position pairs with rest lengths) and
// angle terms (position triplets) and its coordinates; the shapes and their
// numbers are those of the reference's mol_build (cel/engine/oercel.c:478-576),
// in the same order, because the order fixes the snapshot bond list and the
// summation order of the relaxation.  Linear lipids keep the per-bead bond and
// angle terms of the force kernels; k_mol_forces handles the branched shapes:
// one thread per molecule (its first bead) computes every bond and angle term
// of the template in fixed point and leaves each bead's sum in Bufs::fmol,
// which the force kernels' epilogue adds.  Every term is rounded once to
// fixed point and added with opposite signs (angles: three shares that
// cancel), so F_ij = -F_ji and the net bonded force are exactly zero.
#include <cmath>
#include <cstring>

#include "dpd_device.cuh"

namespace {

struct TemplateBuilder {
    dpd_template &M;
    void bond(int i, int j, double r0) {
        M.bi[M.nb] = i;
        M.bj[M.nb] = j;
        M.br0[M.nb] = r0;
        M.nb++;
    }
    // zero terms are left out, as the reference does (oercel.c:469)
    void angle(int i, int j, int k, int kind, double K, double c0) {
        if (K == 0.0) return;
        M.ai[M.na] = i;
        M.aj[M.na] = j;
        M.ak[M.na] = k;
        M.akind[M.na] = kind;
        M.aK[M.na] = K;
        M.ac0[M.na] = c0;
        M.na++;
    }
    // straight chain through positions c[0..n-1]: bonds at r0, then the angles
    void chain(const int *c, int n, double r0, double ka) {
        for (int b = 0; b + 1 < n; b++) bond(c[b], c[b + 1], r0);
        for (int b = 0; b + 2 < n; b++) angle(c[b], c[b + 1], c[b + 2], 0, ka, 0.0);
    }
};

}  // namespace

extern "C" int dpd_lipid_template(const dpd_params *p, dpd_template *t) {
    if (!p || !t) return DPD_E_ARG;
    dpd_template &M = *t;
    std::memset(&M, 0, sizeof M);
    TemplateBuilder B{M};
    const double r0 = p->r0, h = p->r0_head;
    const int nT = p->lip_nT;
    M.arch = p->lip_arch;
    if (p->lip_arch == 0) {
        M.nH = p->lip_nH;
        M.mlen = p->lip_nH + nT;
        if (p->lip_nH < 1 || nT < 0 || M.mlen < 2 || M.mlen > DPD_MAXML) return DPD_E_ARG;
        for (int b = 0; b + 1 < M.mlen; b++) B.bond(b, b + 1, r0);
        for (int b = 0; b + 2 < M.mlen; b++) B.angle(b, b + 1, b + 2, 0, p->k_angle, 0.0);
        for (int b = 0; b < M.mlen; b++) {
            M.px[b] = (b - 0.5 * (M.mlen - 1)) * r0;
            M.ix[b] = b * r0;
        }
        return DPD_OK;
    }
    if (nT < 1) return DPD_E_ARG;
    int ca[DPD_MAXML + 1], cb[DPD_MAXML + 1];
    if (p->lip_arch == 1) {  // pi: heads 0-1 bonded, tail A on 0 (2..nT+1), tail B on 1
        M.nH = 2;
        M.mlen = 2 + 2 * nT;
        if (M.mlen > DPD_MAXML) return DPD_E_ARG;
        B.bond(0, 1, h);
        ca[0] = 0;
        cb[0] = 1;
        for (int k = 1; k <= nT; k++) {
            ca[k] = 1 + k;
            cb[k] = 1 + nT + k;
        }
        B.chain(ca, nT + 1, r0, p->k_angle);
        B.chain(cb, nT + 1, r0, p->k_angle);
        for (int m = 1; m <= p->lip_tie && m <= nT; m++) B.bond(ca[m], cb[m], h);
        B.angle(1, 0, ca[1], 1, p->k_head, p->cos_head);
        B.angle(0, 1, cb[1], 1, p->k_head, p->cos_head);
        M.py[0] = -0.5 * h;
        M.py[1] = 0.5 * h;
        for (int k = 1; k <= nT; k++) {
            M.px[ca[k]] = k * r0;
            M.py[ca[k]] = -0.5 * h;
            M.px[cb[k]] = k * r0;
            M.py[cb[k]] = 0.5 * h;
        }
    } else if (p->lip_arch == 2) {  // y: one head carrying two tails
        M.nH = 1;
        M.mlen = 1 + 2 * nT;
        if (M.mlen > DPD_MAXML) return DPD_E_ARG;
        ca[0] = cb[0] = 0;
        for (int k = 1; k <= nT; k++) {
            ca[k] = k;
            cb[k] = nT + k;
        }
        B.chain(ca, nT + 1, r0, p->k_angle);
        B.chain(cb, nT + 1, r0, p->k_angle);
        for (int m = 1; m <= p->lip_tie && m <= nT; m++) B.bond(ca[m], cb[m], 1.2 * r0);
        B.angle(ca[1], 0, cb[1], 1, p->k_head, p->cos_head);
        for (int k = 1; k <= nT; k++) {
            M.px[ca[k]] = 0.8 * r0 + (k - 1) * r0;
            M.py[ca[k]] = -0.6 * r0;
            M.px[cb[k]] = 0.8 * r0 + (k - 1) * r0;
            M.py[cb[k]] = 0.6 * r0;
        }
    } else if (p->lip_arch == 3) {  // bola: head pair 0-1, tails to a third head 2
        M.nH = 3;
        M.mlen = 3 + 2 * nT;
        if (M.mlen > DPD_MAXML) return DPD_E_ARG;
        B.bond(0, 1, h);
        ca[0] = 0;
        cb[0] = 1;
        for (int k = 1; k <= nT; k++) {
            ca[k] = 2 + k;
            cb[k] = 2 + nT + k;
        }
        ca[nT + 1] = cb[nT + 1] = 2;
        B.chain(ca, nT + 2, r0, p->k_angle);
        B.chain(cb, nT + 2, r0, p->k_angle);
        for (int m = 1; m <= p->lip_tie && m <= nT; m++) B.bond(ca[m], cb[m], h * (1.0 - (double)m / (nT + 1)));
        B.angle(1, 0, ca[1], 1, p->k_head, p->cos_head);
        B.angle(0, 1, cb[1], 1, p->k_head, p->cos_head);
        const double X = std::sqrt((nT + 1) * r0 * (nT + 1) * r0 - 0.25 * h * h);
        M.py[0] = -0.5 * h;
        M.py[1] = 0.5 * h;
        M.px[2] = X;
        for (int k = 1; k <= nT; k++) {
            const double f = (double)k / (nT + 1);
            M.px[ca[k]] = f * X;
            M.py[ca[k]] = -0.5 * h * (1.0 - f);
            M.px[cb[k]] = f * X;
            M.py[cb[k]] = 0.5 * h * (1.0 - f);
        }
    } else {
        return DPD_E_ARG;
    }
    double mx = 0.0, my = 0.0;
    for (int b = 0; b < M.mlen; b++) {
        mx += M.px[b];
        my += M.py[b];
    }
    mx /= M.mlen;
    my /= M.mlen;
    for (int b = 0; b < M.mlen; b++) {
        M.px[b] -= mx;
        M.py[b] -= my;
    }
    for (int b = 0; b < M.mlen; b++) {
        M.ix[b] = M.px[b] - M.px[0];
        M.iy[b] = M.py[b] - M.py[0];
    }
    return DPD_OK;
}

// ---------------------------------------------------------------- bonded forces of branched lipids

// The template's bonds and angles of the molecule whose first bead is slot d
// (mol_forces, oercel.c:1221-1257, with the FP32 roundings of the linear
// terms): each bead's fixed-point sum goes to fmol.  Threads of replicas with
// linear lipids, and of beads that do not start a molecule, do nothing.
__global__ void __launch_bounds__(BEAD_TPB) k_mol_forces(Bufs b, int cur, const RepDev *__restrict__ reps,
                                                         const Chunk *__restrict__ ch) {
    pdl_begin();
    const Chunk c = ch[blockIdx.x];
    const RepDev &R = reps[c.rep];
    const int d = c.begin + (int)threadIdx.x;
    float mb = 0.0f;
    if (R.arch != 0 && d < c.end) {
        const int2 lk0 = b.link[cur][d];
        if (lk0.x < 0 && lk0.y >= 0) {
            const dpd_template &M = b.mol[c.rep];
            const int ml = M.mlen;
            int sl[DPD_MAXML];
            float2 p[DPD_MAXML];
            int qx[DPD_MAXML], qy[DPD_MAXML];
            int n = 0;
            for (int s = d; s >= 0 && n < ml; s = b.link[cur][s].y) {
                sl[n] = s;
                p[n] = b.pos[cur][s];
                qx[n] = qy[n] = 0;
                n++;
            }
            if (n != ml) {
                raise_flag(b.status, DPD_F_CHAIN);
            } else {
                const float L = R.L, h = R.halfL, kb = R.kb;
                for (int q = 0; q < M.nb; q++) {
                    const int i = M.bi[q], j = M.bj[q];
                    const float dx = minimg(__fsub_rn(p[j].x, p[i].x), L, h), dy = minimg(__fsub_rn(p[j].y, p[i].y), L, h);
                    const float r = __fsqrt_rn(__fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
                    mb = fmaxf(mb, r);
                    const float fb = __fdiv_rn(__fmul_rn(kb, __fsub_rn(r, (float)M.br0[q])), r);
                    const int tx = f2fix16(__fmul_rn(fb, dx)), ty = f2fix16(__fmul_rn(fb, dy));
                    qx[i] += tx;  // a stretched bond pulls i toward j
                    qy[i] += ty;
                    qx[j] -= tx;
                    qy[j] -= ty;
                }
                for (int q = 0; q < M.na; q++) {
                    const int i = M.ai[q], j = M.aj[q], k = M.ak[q];
                    int ix, iy, kx, ky;
                    angle_shares_g(p[i], p[j], p[k], M.akind[q], (float)M.aK[q], (float)M.ac0[q], L, h, ix, iy, kx,
                                   ky);
                    qx[i] += ix;
                    qy[i] += iy;
                    qx[k] += kx;
                    qy[k] += ky;
                    qx[j] -= ix + kx;
                    qy[j] -= iy + ky;
                }
                for (int e = 0; e < ml; e++) b.fmol[sl[e]] = make_int2(qx[e], qy[e]);
            }
        }
    }
    // running max bond length of the replica (obs slot 4, float bits; r >= 0)
    const unsigned mbb = __reduce_max_sync(0xffffffffu, __float_as_uint(mb));
    if (lane_id() == 0 && mbb != 0u) atomicMax(b.obs + (size_t)c.rep * OBS_N + 4, (unsigned long long)mbb);
}

void launch_mol_forces(const Bufs &b, int cur, const RepDev *rep, const Chunk *bch, int nbch, cudaStream_t s) {
    launch_pdl(k_mol_forces, nbch, BEAD_TPB, 0, s, b, cur, rep, bch);
}
