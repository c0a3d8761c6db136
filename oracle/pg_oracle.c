/*
 * pg_oracle.c -- FP64 CPU restatement of Phantom-GRAPE's pairwise-force algorithms.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA force engine: only the
 * test suite, the smoke check and the benchmark's CPU-baseline leg load it.  Nothing in the
 * shipped libraries links or calls it.
 *
 * Every function evaluates the reference's formula in double precision, without the
 * reference's reduced-precision shortcuts (12-bit rsqrt, FP32 accumulation), so that the
 * GPU results and the reference's own AVX results can both be measured against it.  Each
 * function names the reference lines it follows (paths inside the Phantom-GRAPE tree).
 *
 * Pinning: the restatement is checked against the unmodified reference libraries compiled
 * from their own sources (oracle/Makefile `ref` target) and against golden vectors they
 * produced (tests/golden/), within the reference's own measured error.
 *
 * Array conventions: positions/velocities are [n][3] row-major doubles; all outputs are
 * overwritten (not accumulated).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

/* ------------------------------------------------------------------------------------ */
/* PG5 Newtonian direct sum.
 * PG5/newton/libpg5/gravity_avx2.c:95-153 (GravityKernel): r2 = eps2_i + |xj - xi|^2,
 * pot -= m/r, acc += m/r^3 (xj - xi), self pair included.
 * PG5/newton/libpg5/phantom_g5.c:244-269 (g5_get_forceMC): the returned pot has its sign
 * flipped (Pot_correct = -(1-bias)), i.e. g5_get_force returns +sum m/r.
 * Symmetric softening (GravityKernel0, gravity_avx2.c:178-250; -DSYMMETRIC):
 * r2 = eps2_i + eps2_j + |dx|^2 -- pass eps2j != NULL.
 * Output: acc[i] = sum_j m_j dx / r^3, pot[i] = +sum_j m_j / r  (GRAPE-5 return convention). */
void orc_g5_newton(int ni, const double *xi, const double *eps2i,
                   int nj, const double *xj, const double *mj, const double *eps2j,
                   double *acc, double *pot)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < ni; i++) {
        double ax = 0, ay = 0, az = 0, p = 0;
        const double x = xi[3*i], y = xi[3*i+1], z = xi[3*i+2];
        for (int j = 0; j < nj; j++) {
            double dx = xj[3*j] - x, dy = xj[3*j+1] - y, dz = xj[3*j+2] - z;
            double r2 = eps2i[i] + dx*dx + dy*dy + dz*dz;
            if (eps2j) r2 += eps2j[j];
            double ri = 1.0 / sqrt(r2);
            double mri = mj[j] * ri;
            double mri3 = mri * ri * ri;
            p += mri;
            ax += mri3 * dx; ay += mri3 * dy; az += mri3 * dz;
        }
        acc[3*i] = ax; acc[3*i+1] = ay; acc[3*i+2] = az;
        pot[i] = p;
    }
}

/* ------------------------------------------------------------------------------------ */
/* PG5 table: force-shape table generation, restated in the reference's own float
 * arithmetic so that the table is bit-identical to the reference's.
 * PG5/table/libpg5/pg5_table.c:43-113 (pg5_gen_force_table):
 *   fmax = 2^(2^EXP_BIT) * (2 - 2^-FRC_BIT)  (float), r2scale = (fmax - 2) / rcut^2 (float),
 *   entry i sits at s_i = float with bits 0x40000000 + i * 2^(23-FRC_BIT),
 *   r_i = sqrtf((s_i - 2) / r2scale), T[i][0] = f(r_i), T[i][1] = (T[i+1][0]-T[i][0])/(s_{i+1}-s_i),
 *   last slope 0; xscale = sqrtf(r2scale) (pg5_table.c:61).
 * Table size = 2^(EXP_BIT+FRC_BIT) (pg5_table.h:17-18). */
typedef double (*orc_force_fn)(double);

static float bits_to_float(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static uint32_t float_to_bits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

void orc_pg5_gen_force_table(int exp_bit, int frc_bit, orc_force_fn force_func, double rcut,
                             float *table /* [tbl][2] */, double *xscale_out)
{
    const int tbl = 1 << (exp_bit + frc_bit);
    const uint32_t tick = 1u << (23 - frc_bit);
    const float r2max = (float)(rcut * rcut);
    const float fmax = (float)(1 << (1 << exp_bit)) * (2.0f - 1.0f / (float)(1 << frc_bit));
    const float r2scale = (fmax - 2.0f) / r2max;
    uint32_t u = float_to_bits(2.0f);
    for (int i = 0; i < tbl; i++, u += tick) {
        float f = bits_to_float(u);
        float r2 = (float)((f - 2.0) / r2scale);
        float r = sqrtf(r2);
        table[2*i] = (float)force_func(r);
    }
    u = float_to_bits(2.0f);
    int i;
    for (i = 0; i < tbl - 1; i++) {
        float x0 = bits_to_float(u);
        u += tick;
        float x1 = bits_to_float(u);
        float y0 = table[2*i], y1 = table[2*(i+1)];
        table[2*i+1] = (y1 - y0) / (x1 - x0);
    }
    table[2*i+1] = 0.0f;
    if (xscale_out) *xscale_out = (double)sqrtf(r2scale);
}

/* S2 softening difference used by g5_open's default table.
 * PG5/table/libpg5/pg5_table.c:8-22 (reff) and :27-29 (s2_force = reff(PP) - reff(PM)). */
static double orc_reff(double sft, double r)
{
    double eta = 2.0 * r / sft;
    if (eta < 1.0)
        return (224. + eta*eta*(-224. + eta*(70. + eta*(48. - eta*21.)))) * 2.0 / (35.0 * pow(sft, 3));
    if (eta < 2.0)
        return (12./(eta*eta) - 224. + eta*(896. + eta*(-840. + eta*(224. + eta*(70. + eta*(-48. + eta*7.))))))
               * 2.0 / (35.0 * eta * pow(sft, 3));
    return 1.0 / pow(r, 3);
}

double orc_s2_force(double r, double sft_pp, double sft_pm)
{
    return orc_reff(sft_pp, r) - orc_reff(sft_pm, r);
}

/* FP64 evaluation of the table force with the same table and linear interpolation.
 * PG5/table/libpg5/gravity_kernel_avx2.c:70-124 (gravity_kernel loop):
 *   s = 2 + |(xj - xi) * xscale|^2, s = min(s, r2cut), r2cut = float bits
 *   (1<<30) | ((TBL-1) << (23-FRC_BIT)) (phantom_g5.c:37-42);
 *   idx = bin of s in the float-bit grid, f = T[idx][0] + (s - s_idx) T[idx][1];
 *   acc += m (xj - xi) xscale f;  acc *= 1/xscale  (gravity_kernel_avx2.c:127-129).
 * Here s, the bin and the lerp are evaluated in FP64 (the bin from frexp, not float bits). */
void orc_g5_table(int ni, const double *xi, int nj, const double *xj, const double *mj,
                  const float *table, int exp_bit, int frc_bit, double xscale, double *acc)
{
    const int tbl = 1 << (exp_bit + frc_bit);
    const double r2cut = (double)bits_to_float((1u << 30) | ((uint32_t)(tbl - 1) << (23 - frc_bit)));
    const double nfrac = (double)(1 << frc_bit);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < ni; i++) {
        double ax = 0, ay = 0, az = 0;
        const double x = xi[3*i] * xscale, y = xi[3*i+1] * xscale, z = xi[3*i+2] * xscale;
        for (int j = 0; j < nj; j++) {
            double dx = xj[3*j] * xscale - x, dy = xj[3*j+1] * xscale - y, dz = xj[3*j+2] * xscale - z;
            double s = 2.0 + dx*dx + dy*dy + dz*dz;
            if (s > r2cut) s = r2cut;
            int e;
            double m = frexp(s, &e);          /* s = m 2^e, m in [0.5, 1) */
            m *= 2.0; e -= 1;                 /* s = m 2^e, m in [1, 2), e >= 1 */
            int fbin = (int)floor((m - 1.0) * nfrac);
            if (fbin >= (1 << frc_bit)) fbin = (1 << frc_bit) - 1;
            int idx = (e - 1) * (1 << frc_bit) + fbin;
            if (idx > tbl - 1) idx = tbl - 1;
            double node = ldexp(1.0 + fbin / nfrac, e);
            double f = (double)table[2*idx] + (s - node) * (double)table[2*idx+1];
            double mf = mj[j] * f;
            ax += mf * dx; ay += mf * dy; az += mf * dz;
        }
        acc[3*i] = ax / xscale; acc[3*i+1] = ay / xscale; acc[3*i+2] = az / xscale;
    }
}

/* ------------------------------------------------------------------------------------ */
/* Quadrupole j-cells.  PG5/newton_quad/source.cpp:1160-1184 (calc_force_nopg, the
 * reference's own FP64 restatement of c_GravityKernel, quad/quad_avx2.c:35-149):
 *   qdr = Q dr, phi_p = m/r, phi_q = (1/2) dr.Q.dr / r^5,
 *   pot += phi_p + phi_q, acc += (phi_p + 5 phi_q) dr / r^2 - qdr / r^5,
 * with Q = (xx, xy, xz, yy, yz, zz) (quad_util.h:8-15, source.cpp:215-248).
 * Output pot is the kernel's accumulated +sum (phi_p + phi_q) before any API sign change. */
void orc_g5_quad(int ni, const double *xi, const double *eps2i,
                 int nc, const double *xc, const double *mc, const double *qc,
                 double *acc, double *pot)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < ni; i++) {
        double a[3] = {0, 0, 0}, p = 0;
        for (int k = 0; k < nc; k++) {
            double dx[3], qdr[3];
            for (int d = 0; d < 3; d++) dx[d] = xc[3*k+d] - xi[3*i+d];
            const double *q = qc + 6*k;
            double r2 = 1.0 / (dx[0]*dx[0] + dx[1]*dx[1] + dx[2]*dx[2] + eps2i[i]);
            double drab = sqrt(r2);
            double phi_p = mc[k] * drab;
            qdr[0] = q[0]*dx[0] + q[1]*dx[1] + q[2]*dx[2];
            qdr[1] = q[1]*dx[0] + q[3]*dx[1] + q[4]*dx[2];
            qdr[2] = q[2]*dx[0] + q[4]*dx[1] + q[5]*dx[2];
            double drqdr = dx[0]*qdr[0] + dx[1]*qdr[1] + dx[2]*qdr[2];
            double dr5i = r2 * r2 * drab;
            double phi_q = 0.5 * dr5i * drqdr;
            p += phi_p + phi_q;
            double mr3i = (phi_p + 5.0 * phi_q) * r2;
            for (int d = 0; d < 3; d++) a[d] += dx[d] * mr3i - qdr[d] * dr5i;
        }
        acc[3*i] = a[0]; acc[3*i+1] = a[1]; acc[3*i+2] = a[2];
        pot[i] = p;
    }
}

/* ------------------------------------------------------------------------------------ */
/* PG6 j-particle predictor.  PG6/libpg6/gravity.c:149-193 (avx_predict_j_particle) with
 * the macro predict() at gravity.c:17-18:
 *   dt = t_i - t_j, x_p = x + v dt + a2 dt^2 + j6 dt^3, v_p = v + 2 a2 dt + 3 j6 dt^2,
 * where a2 = acc/2 and j6 = jerk/6 as stored by g6_set_j_particle (banana01.c:206-212).
 * Kept in FP64 here (the reference stores v_p as float). */
void orc_g6_predict(int nj, double ti, const double *pos, const double *vel,
                    const double *acc2, const double *jrk6, const double *tj,
                    double *xp, double *vp)
{
#pragma omp parallel for schedule(static)
    for (int j = 0; j < nj; j++) {
        double dt = ti - tj[j];
        for (int d = 0; d < 3; d++) {
            int k = 3*j + d;
            xp[k] = pos[k] + vel[k]*dt + acc2[k]*dt*dt + jrk6[k]*dt*dt*dt;
            vp[k] = vel[k] + 2.0*acc2[k]*dt + 3.0*jrk6[k]*dt*dt;
        }
    }
}

/* PG6 Hermite force, jerk, potential, nearest neighbour and neighbour list in FP64.
 * Formulae: PG6/libpg6/gravity.c:195-258 (gravity_kernels, the scalar FP64 kernel) and the
 * output scaling of phantom_g6.c:200-208 (acc, jerk x -1/8 and pot x 1/2 of the -2/r sums),
 * which together give
 *   acc = sum m dx / r^3, jerk = sum m (dv / r^3 - 3 (dx.dv) dx / r^5), pot = -sum m / r,
 * with r^2 = |dx|^2 + eps2 and the self pair excluded by index (gravity.c:347-351).
 * Nearest neighbour (gravity_kernel2, gravity.c:554-564, 651-657): the j != i with the
 * smallest softened r^2; rnnb = softened r (-2 / key_min).  The FP64 oracle breaks exact ties
 * by the smaller j and also reports the second-smallest softened r^2, so tests can skip
 * near-ties where FP32 keys may legitimately order differently.
 * Neighbour list (gravity_kerneln, gravity.c:788-793, 895-906): j flagged when
 * -2/r <= -2/h_i, i.e. softened r <= h_i, none when h2_i == 0; lists in j order, at most
 * maxlen entries stored per i, counts always exact; returns 1 if any count > maxlen.
 * Any of nnb/rnnb/r2nn/r2nn2/h2/nbcount/nblist may be NULL to skip that output. */
int orc_g6_force(int ni, const double *xi, const double *vi, const int *idi, double eps2,
                 const double *h2,
                 int nj, const double *xj, const double *vj, const double *mj, const int *idj,
                 double *acc, double *jrk, double *pot,
                 int *nnb, double *rnnb, double *r2nn, double *r2nn2,
                 int *nbcount, int *nblist, int maxlen)
{
    int overflow = 0;
#pragma omp parallel for schedule(dynamic, 8) reduction(|:overflow)
    for (int i = 0; i < ni; i++) {
        double a[3] = {0, 0, 0}, jk[3] = {0, 0, 0}, p = 0;
        double best = INFINITY, second = INFINITY;
        int bestj = -1, cnt = 0;
        double hh = h2 ? h2[i] : 0.0;
        for (int j = 0; j < nj; j++) {
            if (idj[j] == idi[i]) continue;
            double dx[3], dv[3];
            for (int d = 0; d < 3; d++) {
                dx[d] = xj[3*j+d] - xi[3*i+d];
                dv[d] = vj[3*j+d] - vi[3*i+d];
            }
            double r2 = dx[0]*dx[0] + dx[1]*dx[1] + dx[2]*dx[2] + eps2;
            double rv = dx[0]*dv[0] + dx[1]*dv[1] + dx[2]*dv[2];
            double rinv2 = 1.0 / r2;
            double rinv = sqrt(rinv2);
            double mr = mj[j] * rinv;
            double mr3 = mr * rinv2;
            double rv3 = 3.0 * rv * rinv2;
            p -= mr;
            for (int d = 0; d < 3; d++) {
                a[d] += mr3 * dx[d];
                jk[d] += mr3 * (dv[d] - rv3 * dx[d]);
            }
            if (r2 < best) { second = best; best = r2; bestj = j; }
            else if (r2 < second) { second = r2; }
            if (hh > 0.0 && r2 <= hh) {
                if (nblist && cnt < maxlen) nblist[(long)i * maxlen + cnt] = idj[j];
                cnt++;
            }
        }
        for (int d = 0; d < 3; d++) { acc[3*i+d] = a[d]; jrk[3*i+d] = jk[d]; }
        pot[i] = p;
        if (nnb) nnb[i] = bestj >= 0 ? idj[bestj] : -1;
        if (rnnb) rnnb[i] = sqrt(best);
        if (r2nn) r2nn[i] = best;
        if (r2nn2) r2nn2[i] = second;
        if (nbcount) nbcount[i] = cnt;
        if (cnt > maxlen) overflow = 1;
    }
    return overflow;
}

/* Pairwise potential energy sum_{i<j} -m_i m_j / sqrt(r^2 + eps2), FP64.
 * PG6/banana/calc_energy.c:34-54 (the ACCURACYTEST exact potential). */
double orc_potential_energy(int n, const double *x, const double *m, double eps2)
{
    double w = 0.0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+:w)
    for (int i = 0; i < n; i++) {
        for (int j = i + 1; j < n; j++) {
            double dx = x[3*j] - x[3*i], dy = x[3*j+1] - x[3*i+1], dz = x[3*j+2] - x[3*i+2];
            w -= m[i] * m[j] / sqrt(dx*dx + dy*dy + dz*dz + eps2);
        }
    }
    return w;
}

/* ------------------------------------------------------------------------------------ */
/* PG6 4th-order Hermite block-time-step integrator (the reference's sample integrator,
 * PG6/banana, built with -DNORMAL as its setting.mk does).  State per particle i, as
 * struct Particle (PG6/banana/particle.h) stores it: t, dt, pos[3], vel[3], acc[3] (double),
 * jrk[3], mass, pot (float, held here as the double of a float).
 *
 * orc_hermite_select -- the block step: t_gl = min_i (t_i + dt_i) and the active set
 *   {i : t_i + dt_i == t_gl} in index order (timestep.c:87-98 global_time, whose sorted
 *   index list yields that set under the block-step invariant).  Returns ni.
 * orc_hermite_predict -- the i-particle predictor (hermite.c:39-63 predict_exmotion):
 *   x + v dt + a dt^2 (1/2) + j dt^3 (1/6), v + a dt + j dt^2 (1/2), with the reference's
 *   decimal constants 5e-1 and 1.666666666666667e-1.
 * orc_hermite_correct -- the corrector and the new step (hermite.c:67-108 correct,
 *   143-205 correct_sgmotion, timestep.c:53-85 dt_criterion) for the active set, given the
 *   new force (acc1 double; jrk1 and pot1 rounded to float as NewAccJerk stores them).
 * orc_hermite_startup -- the first step (hermite.c:110-141 startup_sgmotion,
 *   timestep.c:24-51 dt_startup).
 * calc_modulus (timestep.c:137-150) decides whether t is a multiple of a block step. */
static double orc_calc_modulus(double num, double mod, double modmax)
{
    double tmpmod = modmax;
    while (num > 0.0) {
        while (tmpmod > num) tmpmod *= 0.5;
        if (tmpmod < mod) break;
        num -= tmpmod;
    }
    return num;
}

int orc_hermite_select(int n, const double *t, const double *dt, double *t_gl, int *active)
{
    double tm = 1e300;
    for (int i = 0; i < n; i++)
        if (t[i] + dt[i] < tm) tm = t[i] + dt[i];
    int ni = 0;
    for (int i = 0; i < n; i++)
        if (t[i] + dt[i] == tm) active[ni++] = i;
    *t_gl = tm;
    return ni;
}

void orc_hermite_predict(int ni, const int *active, double t_gl, const double *t, const double *pos,
                         const double *vel, const double *acc, const double *jrk, double *xp, double *vp)
{
    const double second = 5e-1, third = 1.666666666666667e-1;
    for (int k = 0; k < ni; k++) {
        const int i = active[k];
        const double d = t_gl - t[i], d2 = d * d, d3 = d * d2;
        for (int c = 0; c < 3; c++) {
            xp[3*k+c] = pos[3*i+c] + vel[3*i+c] * d + acc[3*i+c] * d2 * second + jrk[3*i+c] * d3 * third;
            vp[3*k+c] = vel[3*i+c] + acc[3*i+c] * d + jrk[3*i+c] * d2 * second;
        }
    }
}

/* In place on the state arrays; t_gl is the step's time (= t_i + dt_i of every active i). */
void orc_hermite_correct(int ni, const int *active, double t_gl, const double *xp, const double *vp,
                         const double *acc1, const double *jrk1, const double *pot1, double eta,
                         double dtmax, double *t, double *dt, double *pos, double *vel, double *acc,
                         double *jrk, double *pot)
{
    const double third = 1.666666666666667e-1, fourth = 4.166666666666667e-2, fifth = 8.333333333333333e-3;
    const double dtmin = dtmax / pow(2.0, 51.0);
    for (int k = 0; k < ni; k++) {
        const int i = active[k];
        const double dts = dt[i], dtsinv = 1.0 / dts;
        double s0[3], c0[3], x1[3], v1[3], a1[3], j1[3];
        for (int c = 0; c < 3; c++) {
            a1[c] = acc1[3*k+c];
            j1[c] = (double)(float)jrk1[3*k+c];
            x1[c] = xp[3*k+c];
            v1[c] = vp[3*k+c];
            const double a0 = acc[3*i+c], j0 = jrk[3*i+c];
            s0[c] = 2.0 * (-3.0 * (a0 - a1[c]) - (2.0 * j0 + j1[c]) * dts) * dtsinv * dtsinv;
            c0[c] = 6.0 * (2.0 * (a0 - a1[c]) + (j0 + j1[c]) * dts) * dtsinv * dtsinv * dtsinv;
            x1[c] += s0[c] * dts * dts * dts * dts * fourth + c0[c] * dts * dts * dts * dts * dts * fifth;
            v1[c] += s0[c] * dts * dts * dts * third + c0[c] * dts * dts * dts * dts * fourth;
        }
        /* dt_criterion at the new time t_gl with the old step */
        double s1[3], a = 0, jj = 0, sn = 0, cr = 0, dnew = dts;
        for (int c = 0; c < 3; c++) {
            s1[c] = s0[c] + c0[c] * dts;
            a += a1[c] * a1[c];
            jj += j1[c] * j1[c];
            sn += s1[c] * s1[c];
            cr += c0[c] * c0[c];
        }
        a = sqrt(a); jj = sqrt(jj); sn = sqrt(sn); cr = sqrt(cr);
        const double dti = eta * sqrt((a * sn + jj * jj) / (jj * cr + sn * sn));
        if (dti < dnew) {
            while (dnew > dti && dnew > dtmin) dnew *= 0.5;
        } else if (dti > 2.0 * dnew) {
            if (orc_calc_modulus(t_gl, 2.0 * dnew, dtmax) == 0.0) dnew = 2.0 * dnew;
        }
        t[i] = t_gl;
        dt[i] = dnew;
        for (int c = 0; c < 3; c++) {
            pos[3*i+c] = x1[c];
            vel[3*i+c] = v1[c];
            acc[3*i+c] = a1[c];
            jrk[3*i+c] = j1[c];
        }
        pot[i] = (double)(float)pot1[k];
    }
}

/* Returns the number of particles whose step fell below dtmin (the reference exits there). */
int orc_hermite_startup(int ni, const int *active, const double *acc1, const double *jrk1, const double *pot1,
                        double eta_s, double dtmax, const double *t, double *dt, double *acc, double *jrk,
                        double *pot)
{
    const double dtmin = dtmax / pow(2.0, 51.0);
    int bad = 0;
    for (int k = 0; k < ni; k++) {
        const int i = active[k];
        double a = 0, jj = 0;
        for (int c = 0; c < 3; c++) {
            acc[3*i+c] = acc1[3*k+c];
            jrk[3*i+c] = (double)(float)jrk1[3*k+c];
            a += acc[3*i+c] * acc[3*i+c];
            jj += jrk[3*i+c] * jrk[3*i+c];
        }
        pot[i] = (double)(float)pot1[k];
        const double dtcrit = eta_s * sqrt(a / jj);
        double d = dtmax;
        while (d > dtcrit && d > dtmin) d *= 0.5;
        while (orc_calc_modulus(t[i], d, dtmax) != 0.0) {
            d *= 0.5;
            if (d < dtmin) { bad++; break; }
        }
        dt[i] = d;
    }
    return bad;
}
