/*
 * ref_shim.c -- ctypes entry points into the reference engine itself
 * (TEST INFRASTRUCTURE ONLY: used to pin the oracle restatement and to
 * generate tests/golden/ fixtures; never part of the product).
 *
 * The reference source cel/engine/oercel.c is compiled unmodified from where
 * it lies, with the include trick of cel/engine/tests/forcetest.c:3-5.
 * oracle/Makefile passes its directory with -I.  Every function below only
 * calls the reference's own routines, except ref_integrate, which restates
 * the integrator block that the reference keeps inline in main()
 * (oercel.c:2303-2334).
 */
#define main oercel_main
#include "oercel.c"
#undef main

typedef struct {
    Params P;
    Sys S;
} ref_t;

/* Parameters: the reference defaults (oercel.c:2139-2140), then the
 * "key=value" lines of kv, generic a_K_X keys first (oercel.c:2155-2158),
 * then finalize_params. */
static void ref_params(Params *P, const char *kv) {
    memset(P, 0, sizeof *P);
    for (int k = 0; k < NPDEFS; k++) set_param(P, PDEFS[k].key, PDEFS[k].def);
    default_amatrix(P);
    char *buf = strdup(kv ? kv : "");
    kv_t items[256];
    int n = 0;
    for (char *line = strtok(buf, "\n"); line && n < 256; line = strtok(NULL, "\n")) {
        char *eq = strchr(line, '=');
        if (!eq) continue;
        *eq = 0;
        snprintf(items[n].key, sizeof items[n].key, "%s", trim(line));
        snprintf(items[n].val, sizeof items[n].val, "%s", trim(eq + 1));
        n++;
    }
    for (int pass = 0; pass < 2; pass++)
        for (int k = 0; k < n; k++)
            if (is_generic_akey(items[k].key) == (pass == 0)) set_param(P, items[k].key, items[k].val);
    free(buf);
    finalize_params(P);
}

/* A fresh soup exactly as main() builds it (oercel.c:2185-2202), without the
 * initial force evaluation (ref_prime does that). */
void *ref_create(const char *kv) {
    ref_t *r = calloc(1, sizeof *r);
    ref_params(&r->P, kv);
    Params *P = &r->P;
    Sys *s = &r->S;
    omp_set_num_threads(P->threads);
    omp_set_dynamic(0);
    const int N = (int)lround(P->rho * P->L * P->L);
    sys_alloc(s, N, P->L, g_mol.mlen, g_mol.nH, P->threads, P->nsub);
    s->seed = P->seed;
    s->soup_seed = P->seed;
    rng_seed(&s->rng, P->seed);
    init_soup(s, P);
    set_velocities(s, P);
    g_warm_end = P->warmup;
    for (int i = 0; i < N; i++) {
        s->vtx[i] = s->vx[i];
        s->vty[i] = s->vy[i];
    }
    s->step = 0;
    s->time = 0.0;
    s->t_anchor = 0.0;
    s->step_anchor = 0;
    s->dt_anchor = P->dt;
    return r;
}

/* initial sort, forces at step 0 and the half kick vh = v - dt/2 f (oercel.c:2203-2211) */
void ref_prime(void *h) {
    ref_t *r = h;
    Sys *s = &r->S;
    sort_cells(s);
    pair_forces(s, &r->P, 0, 0.0);
    bonded_forces(s, &r->P);
    for (int i = 0; i < s->N; i++) {
        s->vx[i] -= 0.5 * r->P.dt * s->fx[i];
        s->vy[i] -= 0.5 * r->P.dt * s->fy[i];
    }
}

int32_t ref_n(void *h) { return ((ref_t *)h)->S.N; }
int32_t ref_ncell(void *h) { return ((ref_t *)h)->S.ncell; }
int32_t ref_ncy(void *h) { return ((ref_t *)h)->S.ncy; }

void ref_get(void *h, double *x, double *y, double *vx, double *vy, double *vtx, double *vty, double *fx, double *fy,
             uint8_t *type, uint32_t *gid, int32_t *nxt, int8_t *mpos) {
    Sys *s = &((ref_t *)h)->S;
    const size_t N = (size_t)s->N;
    memcpy(x, s->x, N * 8); memcpy(y, s->y, N * 8);
    memcpy(vx, s->vx, N * 8); memcpy(vy, s->vy, N * 8);
    memcpy(vtx, s->vtx, N * 8); memcpy(vty, s->vty, N * 8);
    memcpy(fx, s->fx, N * 8); memcpy(fy, s->fy, N * 8);
    memcpy(type, s->type, N); memcpy(gid, s->gid, N * 4);
    memcpy(nxt, s->nxt, N * 4); memcpy(mpos, s->mpos, N);
}

void ref_set(void *h, const double *x, const double *y, const double *vx, const double *vy, const double *vtx,
             const double *vty, const double *fx, const double *fy, const uint8_t *type, const uint32_t *gid,
             const int32_t *nxt, const int8_t *mpos) {
    Sys *s = &((ref_t *)h)->S;
    const size_t N = (size_t)s->N;
    memcpy(s->x, x, N * 8); memcpy(s->y, y, N * 8);
    memcpy(s->vx, vx, N * 8); memcpy(s->vy, vy, N * 8);
    memcpy(s->vtx, vtx, N * 8); memcpy(s->vty, vty, N * 8);
    memcpy(s->fx, fx, N * 8); memcpy(s->fy, fy, N * 8);
    memcpy(s->type, type, N); memcpy(s->gid, gid, N * 4);
    memcpy(s->nxt, nxt, N * 4); memcpy(s->mpos, mpos, N);
}

void ref_sort(void *h) { sort_cells(&((ref_t *)h)->S); }

void ref_cells(void *h, int32_t *cstart) {
    Sys *s = &((ref_t *)h)->S;
    memcpy(cstart, s->cstart, (size_t)(s->ncell + 1) * sizeof(int32_t));
}

int32_t ref_cell_of(void *h, double x, double y) { return cell_of_pos(&((ref_t *)h)->S, x, y); }

void ref_pair(void *h, int64_t step) {
    ref_t *r = h;
    pair_forces(&r->S, &r->P, step, r->S.t_anchor + (double)(step - r->S.step_anchor) * r->P.dt);
}

double ref_bonded(void *h) {
    ref_t *r = h;
    r->S.maxbond = 0.0;
    bonded_forces(&r->S, &r->P);
    return r->S.maxbond;
}

/* the integrator block of main(), oercel.c:2303-2334 */
void ref_integrate(void *h) {
    ref_t *r = h;
    Sys *s = &r->S;
    const double dt = r->P.dt, dt2 = dt * dt, cvt = (0.5 + r->P.lambda) * dt, L = s->L;
    for (int i = 0; i < s->N; i++) {
        const double ddx = dt * s->vx[i] + dt2 * s->fx[i], ddy = dt * s->vy[i] + dt2 * s->fy[i];
        double xi = s->x[i] + ddx, yi = s->y[i] + ddy;
        xi = xi < 0.0 ? xi + L : xi;
        yi = yi < 0.0 ? yi + L : yi;
        xi = xi >= L ? xi - L : xi;
        yi = yi >= L ? yi - L : yi;
        s->x[i] = xi;
        s->y[i] = yi;
        s->vtx[i] = s->vx[i] + cvt * s->fx[i];
        s->vty[i] = s->vy[i] + cvt * s->fy[i];
        s->vx[i] += dt * s->fx[i];
        s->vy[i] += dt * s->fy[i];
    }
}

/* nsteps plain steps (no chemistry, no IO) in main()'s order: integrate,
 * sort, pair forces of the new step, bonded forces (oercel.c:2300-2361). */
void ref_run(void *h, int64_t nsteps) {
    ref_t *r = h;
    Sys *s = &r->S;
    for (int64_t k = 0; k < nsteps; k++) {
        const int64_t ns = s->step + 1;
        ref_integrate(h);
        sort_cells(s);
        const double tn = s->t_anchor + (double)(ns - s->step_anchor) * r->P.dt;
        pair_forces(s, &r->P, ns, tn);
        bonded_forces(s, &r->P);
        s->step = ns;
        s->time = tn;
    }
}

int64_t ref_step(void *h) { return ((ref_t *)h)->S.step; }

double ref_theta(uint64_t seed, int64_t step, uint32_t gi, uint32_t gj) {
    return pair_theta(step_seed(seed, step), gi, gj);
}

double ref_kinetic_T(void *h, double *px, double *py) {
    ref_t *r = h;
    return kinetic_T(&r->S, r->P.dt, px, py);
}

void ref_destroy(void *h) { free(h); /* per-bead arrays are never freed by the reference either */ }

/* the reference's chemistry check at `step` (oercel.c:1565-1700), its event
 * list and its serial generator state */
int32_t ref_chemistry(void *h, int64_t step) {
    ref_t *r = h;
    r->S.nev = 0;
    return chemistry(&r->S, &r->P, step);
}

int32_t ref_nev(void *h) { return ((ref_t *)h)->S.nev; }

void ref_events(void *h, int64_t *step, int32_t *kind, int64_t *i, double *x, double *y, int32_t *variant) {
    Sys *s = &((ref_t *)h)->S;
    for (int k = 0; k < s->nev; k++) {
        step[k] = s->ev[k].step;
        kind[k] = s->ev[k].kind;
        i[k] = s->ev[k].i;
        x[k] = s->ev[k].x;
        y[k] = s->ev[k].y;
        variant[k] = s->ev[k].variant;
    }
}

void ref_get_rng(void *h, uint64_t *s4) { memcpy(s4, ((ref_t *)h)->S.rng.s, 4 * sizeof(uint64_t)); }
void ref_set_rng(void *h, const uint64_t *s4) { memcpy(((ref_t *)h)->S.rng.s, s4, 4 * sizeof(uint64_t)); }

/* the reference's lipid template g_mol (built by finalize_params from the
 * parameters of ref_create): ints = arch, mlen, nH, nb, na, then bi, bj (nb
 * each), ai, aj, ak, akind (na each); dbls = br0 (nb), aK, ac0 (na each), then
 * px, py, ix, iy (mlen each) */
void ref_template(void *h, int32_t *ints, double *dbls) {
    (void)h;
    const mol_t *M = &g_mol;
    int k = 0, d = 0;
    ints[k++] = M->arch; ints[k++] = M->mlen; ints[k++] = M->nH; ints[k++] = M->nb; ints[k++] = M->na;
    for (int q = 0; q < M->nb; q++) ints[k++] = M->bi[q];
    for (int q = 0; q < M->nb; q++) ints[k++] = M->bj[q];
    for (int q = 0; q < M->na; q++) ints[k++] = M->ai[q];
    for (int q = 0; q < M->na; q++) ints[k++] = M->aj[q];
    for (int q = 0; q < M->na; q++) ints[k++] = M->ak[q];
    for (int q = 0; q < M->na; q++) ints[k++] = M->akind[q];
    for (int q = 0; q < M->nb; q++) dbls[d++] = M->br0[q];
    for (int q = 0; q < M->na; q++) dbls[d++] = M->aK[q];
    for (int q = 0; q < M->na; q++) dbls[d++] = M->ac0[q];
    for (int b = 0; b < M->mlen; b++) dbls[d++] = M->px[b];
    for (int b = 0; b < M->mlen; b++) dbls[d++] = M->py[b];
    for (int b = 0; b < M->mlen; b++) dbls[d++] = M->ix[b];
    for (int b = 0; b < M->mlen; b++) dbls[d++] = M->iy[b];
}
