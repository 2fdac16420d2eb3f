// dpd_soup.cu -- host-side random soup of the reference (dpd_init_soup).
//
// init_soup + set_velocities of cel/engine/oercel.c:1757-1814, for linear
// lipids and for the branched templates (dpd_mol.cu): the same xoshiro256**
// stream seeded as rng_seed (oercel.c:143-174), drawn in the same order, so
// one seed gives the reference's initial state.
#include <cmath>
#include <cstdint>

#include "../../include/dpd.h"

namespace {

struct Xoshiro {
    uint64_t s[4];
    static uint64_t mix(uint64_t z) {
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        return z ^ (z >> 31);
    }
    explicit Xoshiro(uint64_t seed) {
        uint64_t z = seed;
        for (int k = 0; k < 4; k++) {
            z += 0x9e3779b97f4a7c15ULL;
            s[k] = mix(z);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double unif() { return (double)(next() >> 11) * 0x1.0p-53; }
    double normal() {  // Box-Muller, cosine branch
        double u1 = unif();
        const double u2 = unif();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
    }
};

double wrap(double v, double L) {
    if (v < 0.0) {
        v += L;
        if (v >= L) v -= L;
    } else if (v >= L) {
        v -= L;
        if (v >= L || v < 0.0) v = std::fmod(v, L);
    }
    return v;
}

}  // namespace

extern "C" int dpd_init_soup(double L, int32_t N, uint64_t seed, double kT, double r0, int32_t nH, int32_t nT,
                             double f_lip, double f_Ka, double f_Kb, double c_N, double *x, double *y, double *vx,
                             double *vy, uint8_t *type, int32_t *prev, int32_t *next, int32_t *n_lipid_beads,
                             uint64_t *rng_out, const dpd_template *mol) {
    const bool branched = mol && mol->arch != 0;
    if (branched) {
        nH = mol->nH;
        nT = mol->mlen - mol->nH;
    }
    if (!x || !y || !vx || !vy || !type || N < 2 || nH < 1 || nT < 0 || !(L > 0.0) || !(kT > 0.0) ||
        nH + nT > DPD_MAXML)
        return DPD_E_ARG;
    const int ml = nH + nT;
    const long nlip = std::lround(f_lip * N / ml);
    const long nKa = std::lround(f_Ka * N), nKb = std::lround(f_Kb * N), nP = std::lround(c_N * N);
    if (nlip * ml + nKa + nKb + nP > N) return DPD_E_ARG;
    Xoshiro rng(seed);
    for (int i = 0; i < N; i++) {
        if (prev) prev[i] = -1;
        if (next) next[i] = -1;
    }
    int gi = 0;
    for (long m = 0; m < nlip; m++) {
        const double hx = L * rng.unif(), hy = L * rng.unif();
        const double phi = 2.0 * M_PI * rng.unif();
        const double cph = std::cos(phi), sph = std::sin(phi);
        for (int b = 0; b < ml; b++) {
            if (branched) {  // the template's soup offsets, turned by phi
                x[gi] = wrap(hx + (mol->ix[b] * cph - mol->iy[b] * sph), L);
                y[gi] = wrap(hy + (mol->ix[b] * sph + mol->iy[b] * cph), L);
            } else {
                x[gi] = wrap(hx + b * r0 * cph, L);
                y[gi] = wrap(hy + b * r0 * sph, L);
            }
            type[gi] = b < nH ? 1 : 2;
            if (next && b + 1 < ml) next[gi] = gi + 1;
            if (prev && b > 0) prev[gi] = gi - 1;
            gi++;
        }
    }
    if (n_lipid_beads) *n_lipid_beads = gi;
    for (long cnt = 0; gi < N; gi++, cnt++) {
        x[gi] = L * rng.unif();
        y[gi] = L * rng.unif();
        type[gi] = cnt < nKa ? 4 : cnt < nKa + nKb ? 5 : cnt < nKa + nKb + nP ? 3 : 0;
    }
    double px = 0, py = 0;
    for (int i = 0; i < N; i++) {
        vx[i] = rng.normal() * std::sqrt(kT);
        vy[i] = rng.normal() * std::sqrt(kT);
        px += vx[i];
        py += vy[i];
    }
    px /= N;
    py /= N;
    double k2 = 0;
    for (int i = 0; i < N; i++) {
        vx[i] -= px;
        vy[i] -= py;
        k2 += vx[i] * vx[i] + vy[i] * vy[i];
    }
    const double sc = std::sqrt(kT * (2.0 * N - 2.0) / k2);
    for (int i = 0; i < N; i++) {
        vx[i] *= sc;
        vy[i] *= sc;
    }
    if (rng_out)
        for (int k = 0; k < 4; k++) rng_out[k] = rng.s[k];
    return DPD_OK;
}
