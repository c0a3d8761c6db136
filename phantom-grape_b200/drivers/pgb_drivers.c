/*
 * pgb_drivers.c -- call-sequence drivers for the GRAPE-5 / GRAPE-6 C APIs.
 *
 * Each driver dlopen()s a library that exports the GRAPE API -- this project's lib/libpg*.so
 * or the reference's own build -- and replays the call sequence of the reference's sample
 * programs, timing it with CLOCK_MONOTONIC.  The benchmark uses the same driver for both
 * implementations, so the two arms make identical API calls:
 *
 *  g6drv_schedule  block time-step force calls as PG6/banana/hermite.c:214-275 makes them:
 *                  g6_set_ti, then per npipes-sized chunk g6calc_firsthalf + g6calc_lasthalf2p,
 *                  then g6_set_j_particle for the corrected active particles.
 *  g5drv_direct    PG5/newton/direct/direct.c:133-176: g5_set_xmj, g5_set_eps_to_all,
 *                  g5_set_n, g5_calculate_force_on_x.
 *  g5drv_groups    PG5/newton_quad/source.cpp:813-860 style: OpenMP over i-groups, each thread
 *                  with its own devid: g5_set_xmjMC, g5_set_nMC, g5_calculate_force_on_xMC.
 *  g5drv_bh        the same with the quadrupole-cell lists through g5c_* (source.cpp:813-866).
 *
 * Libraries are opened with RTLD_LOCAL so several GRAPE libraries can coexist in one process.
 */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static double now(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

#define LOAD(h, var, name)                                                       \
    do {                                                                         \
        *(void **)(&(var)) = dlsym((h), (name));                                 \
        if (!(var)) {                                                            \
            fprintf(stderr, "pgb_drivers: %s has no symbol %s\n", path, (name)); \
            return NULL;                                                         \
        }                                                                        \
    } while (0)

/* ---------------------------------------------------------------------------------------- */
/* GRAPE-6 (PG6/libpg6/gp6util.h) */

typedef struct {
    void *h;
    void (*open)(int);
    int (*npipes)(void);
    void (*set_j)(int, int, int, double, double, double, double *, double *, double *, double *, double *);
    void (*set_ti)(int, double);
    void (*firsthalf)(int, int, int, int *, double (*)[3], double (*)[3], double (*)[3], double (*)[3], double *,
                      double, double *);
    int (*lasthalf2p)(int, int, int, int *, double (*)[3], double (*)[3], double, double *, double (*)[3],
                      double (*)[3], double *, int *, float *);
    int (*lasthalf)(int, int, int, int *, double (*)[3], double (*)[3], double, double *, double (*)[3],
                    double (*)[3], double *);
} g6api;

void *g6drv_open(const char *path) {
    void *h = dlopen(path, RTLD_LOCAL | RTLD_NOW);
    if (!h) {
        fprintf(stderr, "pgb_drivers: dlopen(%s): %s\n", path, dlerror());
        return NULL;
    }
    g6api *a = (g6api *)calloc(1, sizeof(g6api));
    a->h = h;
    LOAD(h, a->open, "g6_open");
    LOAD(h, a->npipes, "g6_npipes");
    LOAD(h, a->set_j, "g6_set_j_particle");
    LOAD(h, a->set_ti, "g6_set_ti");
    LOAD(h, a->firsthalf, "g6calc_firsthalf");
    LOAD(h, a->lasthalf2p, "g6calc_lasthalf2p");
    LOAD(h, a->lasthalf, "g6calc_lasthalf");
    a->open(0);
    return a;
}

int g6drv_npipes(void *handle) { return ((g6api *)handle)->npipes(); }

/* g6_set_j_particle for n particles (addr NULL: address = index). */
double g6drv_set_j(void *handle, int n, const double *pos, const double *vel, const double *acc2, const double *jrk6,
                   const double *mass, const double *tj, const int *idx, const int *addr) {
    g6api *a = (g6api *)handle;
    double snp[3] = {0, 0, 0};
    double t0 = now();
    for (int k = 0; k < n; k++) {
        int j = addr ? addr[k] : k;
        a->set_j(0, j, idx[j], tj[j], 0.0, mass[j], snp, (double *)jrk6 + 3 * j, (double *)acc2 + 3 * j,
                 (double *)vel + 3 * j, (double *)pos + 3 * j);
    }
    return now() - t0;
}

/* Seconds per drop-in call of one shape: `calls` x (g6calc_firsthalf + g6calc_lasthalf2p) for the
 * first ni of the given i-particles against j-records [0, nj) of the j-memory (set before),
 * after 100 untimed calls; the best of three runs. */
double g6drv_call_time(void *handle, int ni, int nj, int calls, const double *xi, const double *vi, const int *idx,
                       double eps2) {
    g6api *a = (g6api *)handle;
    if (ni < 1 || ni > a->npipes() || calls < 1) return -1.0;
    int *pidx = (int *)malloc(sizeof(int) * ni);
    double(*pos)[3] = malloc(sizeof(double) * 3 * ni);
    double(*vel)[3] = malloc(sizeof(double) * 3 * ni);
    double(*acc)[3] = malloc(sizeof(double) * 3 * ni);
    double(*jrk)[3] = malloc(sizeof(double) * 3 * ni);
    double *pot = (double *)malloc(sizeof(double) * ni), *h2 = (double *)calloc(ni, sizeof(double));
    int *nnb = (int *)malloc(sizeof(int) * ni);
    float *rnnb = (float *)malloc(sizeof(float) * ni);
    for (int i = 0; i < ni; i++) {
        pidx[i] = idx[i];
        for (int c = 0; c < 3; c++) {
            pos[i][c] = xi[3 * i + c];
            vel[i][c] = vi[3 * i + c];
        }
    }
    double best = 1e30;
    for (int run = 0; run < 4; run++) {
        const int n = run == 0 ? 100 : calls;
        double t0 = now();
        for (int k = 0; k < n; k++) {
            a->firsthalf(0, nj, ni, pidx, pos, vel, acc, jrk, pot, eps2, h2);
            a->lasthalf2p(0, nj, ni, pidx, pos, vel, eps2, h2, acc, jrk, pot, nnb, rnnb);
        }
        double t = (now() - t0) / n;
        if (run > 0 && t < best) best = t;
    }
    free(pidx);
    free(pos);
    free(vel);
    free(acc);
    free(jrk);
    free(pot);
    free(h2);
    free(nnb);
    free(rnnb);
    return best;
}

/* One pass over `ncalls` block steps.  Call c uses time t_calls[c] and the active particles
 * set_idx[set_off[c] .. set_off[c+1]) whose predicted positions / velocities are
 * xi/vi[set_off[c] ..].  With `resend`, the active particles' j-records (from pos..tj) are
 * re-sent after each call, as the corrector does (hermite.c:255-275).  Outputs (optional) are
 * written per active particle in the same concatenated order.  Returns the elapsed seconds. */
double g6drv_schedule2(void *handle, int nj, int ncalls, const int *set_off, const int *set_idx,
                       const double *t_calls, const double *xi, const double *vi, double eps2, int with_nnb,
                       int resend, const int *rs_off, const int *rs_idx, const double *pos, const double *vel,
                       const double *acc2, const double *jrk6, const double *mass, const double *tj, const int *idx,
                       double *acc_out, double *jrk_out, double *pot_out, int *nnb_out, float *rnnb_out);

double g6drv_schedule(void *handle, int nj, int ncalls, const int *set_off, const int *set_idx,
                      const double *t_calls, const double *xi, const double *vi, double eps2, int with_nnb,
                      int resend, const double *pos, const double *vel, const double *acc2, const double *jrk6,
                      const double *mass, const double *tj, const int *idx, double *acc_out, double *jrk_out,
                      double *pot_out, int *nnb_out, float *rnnb_out) {
    return g6drv_schedule2(handle, nj, ncalls, set_off, set_idx, t_calls, xi, vi, eps2, with_nnb, resend, NULL, NULL,
                           pos, vel, acc2, jrk6, mass, tj, idx, acc_out, jrk_out, pot_out, nnb_out, rnnb_out);
}

/* As g6drv_schedule, with the particles re-sent after call c given separately (rs_off / rs_idx,
 * NULL: the call's own set): a rank of a sharded schedule computes the forces of a slice of each
 * active set but updates its j-memory with the whole set. */
double g6drv_schedule2(void *handle, int nj, int ncalls, const int *set_off, const int *set_idx,
                       const double *t_calls, const double *xi, const double *vi, double eps2, int with_nnb,
                       int resend, const int *rs_off, const int *rs_idx, const double *pos, const double *vel,
                       const double *acc2, const double *jrk6, const double *mass, const double *tj, const int *idx,
                       double *acc_out, double *jrk_out, double *pot_out, int *nnb_out, float *rnnb_out) {
    if (!rs_off || !rs_idx) {
        rs_off = set_off;
        rs_idx = set_idx;
    }
    g6api *a = (g6api *)handle;
    int npipe = a->npipes();
    int *pidx = (int *)malloc(sizeof(int) * npipe);
    double(*acc)[3] = malloc(sizeof(double) * 3 * npipe);
    double(*jrk)[3] = malloc(sizeof(double) * 3 * npipe);
    double *pot = (double *)malloc(sizeof(double) * npipe);
    double *h2 = (double *)calloc(npipe, sizeof(double));
    int *nnb = (int *)malloc(sizeof(int) * npipe);
    float *rnnb = (float *)malloc(sizeof(float) * npipe);
    double snp[3] = {0, 0, 0};
    double t0 = now();
    for (int c = 0; c < ncalls; c++) {
        int off = set_off[c], ni = set_off[c + 1] - set_off[c];
        a->set_ti(0, t_calls[c]);
        for (int i = 0; i < ni; i += npipe) {
            int nii = ni - i < npipe ? ni - i : npipe;
            for (int k = 0; k < nii; k++) pidx[k] = idx[set_idx[off + i + k]];
            double(*px)[3] = (double(*)[3])(xi + 3 * (size_t)(off + i));
            double(*pv)[3] = (double(*)[3])(vi + 3 * (size_t)(off + i));
            a->firsthalf(0, nj, nii, pidx, px, pv, acc, jrk, pot, eps2, h2);
            if (with_nnb)
                a->lasthalf2p(0, nj, nii, pidx, px, pv, eps2, h2, acc, jrk, pot, nnb, rnnb);
            else
                a->lasthalf(0, nj, nii, pidx, px, pv, eps2, h2, acc, jrk, pot);
            size_t o = (size_t)(off + i);
            if (acc_out) memcpy(acc_out + 3 * o, acc, sizeof(double) * 3 * nii);
            if (jrk_out) memcpy(jrk_out + 3 * o, jrk, sizeof(double) * 3 * nii);
            if (pot_out) memcpy(pot_out + o, pot, sizeof(double) * nii);
            if (nnb_out && with_nnb) memcpy(nnb_out + o, nnb, sizeof(int) * nii);
            if (rnnb_out && with_nnb) memcpy(rnnb_out + o, rnnb, sizeof(float) * nii);
        }
        if (resend) {
            for (int k = rs_off[c]; k < rs_off[c + 1]; k++) {
                int j = rs_idx[k];
                a->set_j(0, j, idx[j], tj[j], 0.0, mass[j], snp, (double *)jrk6 + 3 * j, (double *)acc2 + 3 * j,
                         (double *)vel + 3 * j, (double *)pos + 3 * j);
            }
        }
    }
    double el = now() - t0;
    free(pidx);
    free(acc);
    free(jrk);
    free(pot);
    free(h2);
    free(nnb);
    free(rnnb);
    return el;
}

/* ---------------------------------------------------------------------------------------- */
/* GRAPE-5 (PG5/newton/libpg5/gp5util.h, PG5/table/libpg5/gp5util.h) */

typedef struct {
    void *h;
    void (*open)(void);
    void (*set_eps_to_all)(double);
    void (*set_xmj)(int, int, double (*)[3], double *);
    void (*set_n)(int);
    void (*calc)(double (*)[3], double (*)[3], double *, int);
    void (*set_xmjMC)(int, int, int, double (*)[3], double *);
    void (*set_nMC)(int, int);
    void (*calcMC)(int, double (*)[3], double (*)[3], double *, int);
    /* quadrupole cells (PG5/newton_quad/quad/quad_util.h:8-15); NULL in libraries without them */
    void (*c_set_xmjMC)(int, int, int, double (*)[3], double *, double (*)[6]);
    void (*c_set_nMC)(int, int);
    void (*c_calcMC)(int, double (*)[3], double (*)[3], double *, int);
} g5api;

void *g5drv_open(const char *path) {
    void *h = dlopen(path, RTLD_LOCAL | RTLD_NOW);
    if (!h) {
        fprintf(stderr, "pgb_drivers: dlopen(%s): %s\n", path, dlerror());
        return NULL;
    }
    g5api *a = (g5api *)calloc(1, sizeof(g5api));
    a->h = h;
    LOAD(h, a->open, "g5_open");
    LOAD(h, a->set_eps_to_all, "g5_set_eps_to_all");
    LOAD(h, a->set_xmj, "g5_set_xmj");
    LOAD(h, a->set_n, "g5_set_n");
    LOAD(h, a->calc, "g5_calculate_force_on_x");
    LOAD(h, a->set_xmjMC, "g5_set_xmjMC");
    LOAD(h, a->set_nMC, "g5_set_nMC");
    LOAD(h, a->calcMC, "g5_calculate_force_on_xMC");
    *(void **)(&a->c_set_xmjMC) = dlsym(h, "g5c_set_xmjMC");
    *(void **)(&a->c_set_nMC) = dlsym(h, "g5c_set_nMC");
    *(void **)(&a->c_calcMC) = dlsym(h, "g5c_calculate_force_on_xMC");
    a->open();
    return a;
}

/* Direct summation, all i against all j (direct.c:133-176). */
double g5drv_direct(void *handle, int n, const double *x, const double *m, double eps, double *acc, double *pot) {
    g5api *a = (g5api *)handle;
    double t0 = now();
    a->set_xmj(0, n, (double(*)[3])x, (double *)m);
    a->set_eps_to_all(eps);
    a->set_n(n);
    a->calc((double(*)[3])x, (double(*)[3])acc, pot, n);
    return now() - t0;
}

/* Interaction-list groups: items[k] = {i_off, i_cnt, j_off, j_cnt}; OpenMP over groups with
 * devid = thread id (source.cpp:813-860).  nthreads <= 0: OpenMP default. */
double g5drv_groups(void *handle, int ngroups, const int *items, const double *xi, const double *xj,
                    const double *mj, double eps, double *acc, double *pot, int nthreads) {
    g5api *a = (g5api *)handle;
    a->set_eps_to_all(eps);
    if (nthreads > 0) omp_set_num_threads(nthreads);
    double t0 = now();
#pragma omp parallel for schedule(dynamic, 1)
    for (int g = 0; g < ngroups; g++) {
        int dev = omp_get_thread_num();
        const int *it = items + 4 * g;
        a->set_xmjMC(dev, 0, it[3], (double(*)[3])(xj + 3 * (size_t)it[2]), (double *)mj + it[2]);
        a->set_nMC(dev, it[3]);
        a->calcMC(dev, (double(*)[3])(xi + 3 * (size_t)it[0]), (double(*)[3])(acc + 3 * (size_t)it[0]),
                  pot + it[0], it[1]);
    }
    return now() - t0;
}

/* Barnes-Hut groups with point-mass and quadrupole-cell lists, the way
 * PG5/newton_quad/source.cpp:813-866 drives the libraries: OpenMP over groups, devid = thread
 * id; per group the point-mass list through g5_set_xmjMC + g5_set_nMC +
 * g5_calculate_force_on_xMC and the cell list through g5c_set_xmjMC + g5c_set_nMC +
 * g5c_calculate_force_on_xMC, then acc = a_mono + a_quad and phi = -p_mono + p_quad (the sign
 * reconciliation of source.cpp:854, 866; its self-term correction epsinv*m is left out).
 * Lists are index lists into tree-order particle (xp, mp) and cell (cpos, cmass, cquad) arrays,
 * gathered per group into thread-local buffers inside the timed loop (the reference writes
 * them in its tree walk just before the calls).  Groups [g0, g1); returns elapsed seconds,
 * or -1 when the library has no g5c_* entry points. */
double g5drv_bh(void *handle, int g0, int g1, const int *gfirst, const int *gcount, const double *xi,
                const double *xp, const double *mp, const long long *poff, const int *pidx, const double *cpos,
                const double *cmass, const double *cquad, const long long *coff, const int *cidx, double eps,
                double *acc, double *phi, int nthreads) {
    g5api *a = (g5api *)handle;
    if (!a->c_set_xmjMC || !a->c_set_nMC || !a->c_calcMC) return -1.0;
    long long maxp = 1, maxc = 1;
    int maxi = 1;
    for (int g = g0; g < g1; g++) {
        if (poff[g + 1] - poff[g] > maxp) maxp = poff[g + 1] - poff[g];
        if (coff[g + 1] - coff[g] > maxc) maxc = coff[g + 1] - coff[g];
        if (gcount[g] > maxi) maxi = gcount[g];
    }
    a->set_eps_to_all(eps);
    if (nthreads > 0) omp_set_num_threads(nthreads);
    double t0 = now();
#pragma omp parallel
    {
        double(*xj)[3] = malloc(sizeof(double) * 3 * maxp);
        double *mj = malloc(sizeof(double) * maxp);
        double(*xc)[3] = malloc(sizeof(double) * 3 * maxc);
        double *mc = malloc(sizeof(double) * maxc);
        double(*qc)[6] = malloc(sizeof(double) * 6 * maxc);
        double(*a2)[3] = malloc(sizeof(double) * 3 * maxi);
        double *p1 = malloc(sizeof(double) * maxi), *p2 = malloc(sizeof(double) * maxi);
        int dev = omp_get_thread_num();
#pragma omp for schedule(dynamic, 1)
        for (int g = g0; g < g1; g++) {
            const int f = gfirst[g], ni = gcount[g];
            const int np = (int)(poff[g + 1] - poff[g]), nc = (int)(coff[g + 1] - coff[g]);
            for (int k = 0; k < np; k++) {
                const int p = pidx[poff[g] + k];
                xj[k][0] = xp[3 * (size_t)p];
                xj[k][1] = xp[3 * (size_t)p + 1];
                xj[k][2] = xp[3 * (size_t)p + 2];
                mj[k] = mp[p];
            }
            for (int k = 0; k < nc; k++) {
                const int c = cidx[coff[g] + k];
                for (int d = 0; d < 3; d++) xc[k][d] = cpos[3 * (size_t)c + d];
                mc[k] = cmass[c];
                for (int d = 0; d < 6; d++) qc[k][d] = cquad[6 * (size_t)c + d];
            }
            double(*xg)[3] = (double(*)[3])(xi + 3 * (size_t)f);
            double(*ag)[3] = (double(*)[3])(acc + 3 * (size_t)f);
            a->set_xmjMC(dev, 0, np, xj, mj);
            a->set_nMC(dev, np);
            a->calcMC(dev, xg, ag, p1, ni);
            a->c_set_xmjMC(dev, 0, nc, xc, mc, qc);
            a->c_set_nMC(dev, nc);
            a->c_calcMC(dev, xg, a2, p2, ni);
            for (int i = 0; i < ni; i++) {
                ag[i][0] += a2[i][0];
                ag[i][1] += a2[i][1];
                ag[i][2] += a2[i][2];
                phi[f + i] = -p1[i] + p2[i];
            }
        }
        free(xj);
        free(mj);
        free(xc);
        free(mc);
        free(qc);
        free(a2);
        free(p1);
        free(p2);
    }
    return now() - t0;
}

/* Independent clusters through the plain GRAPE-6 calls: for cluster c (particles
 * [off[c], off[c+1]) of the arrays), its particles are written to j-addresses 0..n_c-1 with
 * g6_set_j_particle (zero acc/2, jerk/6, time 0), then g6_set_ti(0) and npipes-sized
 * g6calc_firsthalf / g6calc_lasthalf2p over all of them.  Outputs per particle (optional).
 * Clusters [c0, c1) only.  Returns the elapsed seconds. */
double g6drv_clusters(void *handle, int c0, int c1, const int *off, const double *pos, const double *vel,
                      const double *mass, double eps2, double *acc_out, double *jrk_out, double *pot_out,
                      int *nnb_out, float *rnnb_out) {
    g6api *a = (g6api *)handle;
    int npipe = a->npipes();
    int *pidx = (int *)malloc(sizeof(int) * npipe);
    double(*acc)[3] = malloc(sizeof(double) * 3 * npipe);
    double(*jrk)[3] = malloc(sizeof(double) * 3 * npipe);
    double *pot = (double *)malloc(sizeof(double) * npipe);
    double *h2 = (double *)calloc(npipe, sizeof(double));
    int *nnb = (int *)malloc(sizeof(int) * npipe);
    float *rnnb = (float *)malloc(sizeof(float) * npipe);
    double zero3[3] = {0, 0, 0};
    double t0 = now();
    for (int c = c0; c < c1; c++) {
        int o = off[c], n = off[c + 1] - off[c];
        for (int k = 0; k < n; k++)
            a->set_j(0, k, k, 0.0, 0.0, mass[o + k], zero3, zero3, zero3, (double *)vel + 3 * (size_t)(o + k),
                     (double *)pos + 3 * (size_t)(o + k));
        a->set_ti(0, 0.0);
        for (int i = 0; i < n; i += npipe) {
            int nii = n - i < npipe ? n - i : npipe;
            for (int k = 0; k < nii; k++) pidx[k] = i + k;
            double(*px)[3] = (double(*)[3])(pos + 3 * (size_t)(o + i));
            double(*pv)[3] = (double(*)[3])(vel + 3 * (size_t)(o + i));
            a->firsthalf(0, n, nii, pidx, px, pv, acc, jrk, pot, eps2, h2);
            a->lasthalf2p(0, n, nii, pidx, px, pv, eps2, h2, acc, jrk, pot, nnb, rnnb);
            size_t q = (size_t)(o + i);
            if (acc_out) memcpy(acc_out + 3 * q, acc, sizeof(double) * 3 * nii);
            if (jrk_out) memcpy(jrk_out + 3 * q, jrk, sizeof(double) * 3 * nii);
            if (pot_out) memcpy(pot_out + q, pot, sizeof(double) * nii);
            if (nnb_out) memcpy(nnb_out + q, nnb, sizeof(int) * nii);
            if (rnnb_out) memcpy(rnnb_out + q, rnnb, sizeof(float) * nii);
        }
    }
    double el = now() - t0;
    free(pidx);
    free(acc);
    free(jrk);
    free(pot);
    free(h2);
    free(nnb);
    free(rnnb);
    return el;
}
