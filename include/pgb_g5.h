/*
 * pgb_g5.h -- C ABI of lib/libpg5.so (and lib/libpg5sym.so with PGB_SYMMETRIC defined):
 * the GRAPE-5 direct-summation API and the newton_quad quadrupole-cell API on the B200 engine.
 *
 * Drop-in replacement for the reference libraries built from PG5/newton/libpg5 and
 * PG5/newton_quad/quad: same symbols, same argument meaning, same return conventions
 * (acc = sum m dx / r^3, pot = +sum m / r including the self pair; the quadrupole potential
 * comes back negated, as the reference returns it).  Differences are listed in the library
 * source (csrc/pgb_g5.cu header comment).
 *
 * Errors: the reference asserts; this library records the error (pgb5_last_error) and, unless
 * PGB_NOABORT=1 or pgb5_set_abort(0), prints it and aborts.
 */
#ifndef PGB_G5_H
#define PGB_G5_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- GRAPE-5 API: PG5/newton/libpg5/gp5util.h:10-39 ------------------------------------ */
void g5_open(void);                                   /* phantom_g5.c:45-60 (no rsqrt bias) */
void g5_close(void);                                  /* phantom_g5.c:62-65 (frees GPU memory) */
int  g5_get_number_of_pipelines(void);                /* phantom_g5.c:35-38 (4; PGB_G5_NPIPES) */
int  g5_get_jmemsize(void);                           /* phantom_g5.c:40-43 (1 Mi; PGB_G5_JMEMSIZE) */
void g5_set_eps_to_all(double eps);                   /* phantom_g5.c:67-70 */
void g5_set_eps(int ni, double *eps);                 /* phantom_g5.c:84-87 */
void g5_set_epsMC(int devid, int ni, double *eps);    /* phantom_g5.c:72-82 */
void g5_set_n(int n);                                 /* phantom_g5.c:95-98 */
void g5_set_nMC(int devid, int n);                    /* phantom_g5.c:89-93 */
void g5_set_xi(int ni, double (*xi)[3]);              /* phantom_g5.c:130-133 */
void g5_set_xiMC(int devid, int ni, double (*xi)[3]); /* phantom_g5.c:100-113 */
void g5_set_xei(int ni, double (*xi)[3], double *eps2);                 /* phantom_g5.c:135-138 */
void g5_set_xeiMC(int devid, int ni, double (*xi)[3], double *eps2);    /* phantom_g5.c:115-128 */
#ifdef PGB_SYMMETRIC
/* symmetric softening r^2 = |dx|^2 + eps2_i + epsj2[j] (phantom_g5.c:140-186, -DSYMMETRIC) */
void g5_set_xmj(int adr, int nj, double (*xj)[3], double *mj, double *epsj2);
void g5_set_xmjMC(int devid, int adr, int nj, double (*xj)[3], double *mj, double *epsj2);
#else
void g5_set_xmj(int adr, int nj, double (*xj)[3], double *mj);               /* phantom_g5.c:215-218 */
void g5_set_xmjMC(int devid, int adr, int nj, double (*xj)[3], double *mj);  /* phantom_g5.c:188-205 */
#endif
void g5_run(void);                                    /* phantom_g5.c:239-242 */
void g5_runMC(int devid);                             /* phantom_g5.c:222-237 */
void g5_get_force(int ni, double (*a)[3], double *p);               /* phantom_g5.c:271-274 */
void g5_get_forceMC(int devid, int ni, double (*a)[3], double *p);  /* phantom_g5.c:244-269 */
void g5_calculate_force_on_x(double (*x)[3], double (*a)[3], double *p, int ni);       /* :303-306 */
void g5_calculate_force_on_xMC(int devid, double (*x)[3], double (*a)[3], double *p, int ni); /* :276-287 */
void g5_calculate_force_on_xe(double (*x)[3], double *eps2, double (*a)[3], double *p, int ni); /* :308-312 */
void g5_calculate_force_on_xeMC(int devid, double (*x)[3], double *eps2, double (*a)[3], double *p,
                                int ni);                                                 /* :289-300 */

/* ---- quadrupole j-cells: PG5/newton_quad/quad/quad_util.h:8-15 -------------------------- */
/* qj = (xx, xy, xz, yy, yz, zz) of sum m (3 d d - |d|^2 I) (source.cpp:215-248)            */
void g5c_set_nMC(int devid, int n);                                                     /* quad_g5c.c:14-17 */
void g5c_set_xmjMC(int devid, int adr, int nj, double (*xj)[3], double *mj, double (*qj)[6]);  /* :198-283 */
void g5c_set_xmjMC0(int devid, int adr, int nj, double (*xj)[3], double *mj, double (*qj)[6]); /* :19-188 */
void g5c_runMC(int devid);                                                              /* :297-303 */
void g5c_runMC0(int devid);                                                             /* :190-196 */
void g5c_calculate_force_on_xMC(int devid, double (*x)[3], double (*a)[3], double *p, int ni);  /* :285-295 */
void g5c_calculate_force_on_xMC0(int devid, double (*x)[3], double (*a)[3], double *p, int ni); /* (SoA twin) */

/* ---- Fortran bindings: PG5/newton/libpg5/pg5_fortran.c:1-119 ---------------------------- */
int  g5_get_number_of_pipelines_(void);
int  g5_get_jmemsize_(void);
void g5_open_(void);
void g5_close_(void);
void g5_set_eps_to_all_(double *eps);
void g5_set_n_(int *n);
void g5_set_nMC_(int *devid, int *n);
void g5_set_xi_(int *ni, double (*xi)[3]);
void g5_set_xei_(int *ni, double (*xi)[3], double *eps2);
void g5_set_xiMC_(int *devid, int *ni, double (*xi)[3]);
void g5_set_xeiMC_(int *devid, int *ni, double (*xi)[3], double *eps2);
#ifdef PGB_SYMMETRIC
void g5_set_xmj_(int *adr, int *nj, double (*xj)[3], double *mj, double *eps2);
void g5_set_xmjMC_(int *devid, int *adr, int *nj, double (*xj)[3], double *mj, double *eps2);
#else
void g5_set_xmj_(int *adr, int *nj, double (*xj)[3], double *mj);
void g5_set_xmjMC_(int *devid, int *adr, int *nj, double (*xj)[3], double *mj);
#endif
void g5_run_(void);
void g5_runMC_(int *devid);
void g5_get_force_(int *ni, double (*a)[3], double *p);
void g5_get_forceMC_(int *devid, int *ni, double (*a)[3], double *p);
void g5_calculate_force_on_x_(double (*x)[3], double (*a)[3], double *p, int *ni);
void g5_calculate_force_on_xe_(double (*x)[3], double *eps2, double (*a)[3], double *p, int *ni);
void g5_calculate_force_on_xMC_(int *devid, double (*x)[3], double (*a)[3], double *p, int *ni);
void g5_calculate_force_on_xeMC_(int *devid, double (*x)[3], double *eps2, double (*a)[3], double *p, int *ni);

/* ---- library status (no reference counterpart: replaces assert()) ----------------------- */
int  pgb5_last_error(char *buf, int len);   /* returns the last error code, copies its message */
void pgb5_clear_error(void);
void pgb5_set_abort(int on);                /* 1 (default): abort on error, as assert() does */

/* ---- batched path (no reference counterpart) --------------------------------------------
 * Replaces a loop over i-groups of g5_set_xmjMC + g5_set_nMC + g5_calculate_force_on_xMC
 * (PG5/newton_quad/source.cpp:847-860) by one persistent launch over all groups.
 * items[k] = {i_offset, i_count, j_offset, j_count} into the device i- and j-arrays.
 * kind: PGB5_NEWTON, PGB5_SYMMETRIC, PGB5_QUAD (libpg5*.so) or PGB5_TABLE (libpg5table.so).
 * Device layouts: ipos float4 (x, y, z, eps2); jpos float4 (x, y, z, m); jaux: symmetric
 * float4 (eps2_j, 0, 0, 0) per j, quad two float4 (q0 q1 q2 q3)(q4 q5 0 0) per cell;
 * out double4 (ax, ay, az, pot_raw) with pot_raw = -sum m/r (newton) or +sum(phi_p + phi_q)
 * (quad), indexed by absolute i.  pgb5_plan_launch launches one kernel on `stream` (a
 * cudaStream_t) and uploads nothing, so it can be captured in a CUDA graph.
 * pgb5_plan_tune times the plan once per kernel configuration (threads x i per thread) on
 * the caller's data (out is overwritten), keeps the fastest for this plan and for later
 * plans of the same shape, and returns its index (-1 on error; *best_ms its launch time).
 * pgb5_plan_config returns the plan's configuration index; pgb5_plan_set_config pins one
 * (an error for a configuration the kind cannot use: the table kind takes CTAs of <= 256
 * threads, the quadrupole kind <= 512).                                                  */
enum { PGB5_NEWTON = 0, PGB5_SYMMETRIC = 1, PGB5_QUAD = 2, PGB5_TABLE = 3 };
typedef struct pgb5_plan pgb5_plan;
int  pgb5_plan_create(pgb5_plan **plan, int kind, int nitem, const int *items);
int  pgb5_plan_launch(pgb5_plan *plan, const void *ipos, const void *jpos, const void *jaux, void *out,
                      void *stream);
void pgb5_plan_destroy(pgb5_plan *plan);
long long pgb5_plan_interactions(const pgb5_plan *plan);
int  pgb5_plan_tasks(const pgb5_plan *plan);
int  pgb5_plan_tune(pgb5_plan *plan, const void *ipos, const void *jpos, const void *jaux, void *out,
                    void *stream, float *best_ms);
int  pgb5_plan_config(const pgb5_plan *plan);
int  pgb5_plan_set_config(pgb5_plan *plan, int cfg);   /* pin one (PGB5_NCFG configurations) */
/* New items for an existing plan of the same kind, its configuration kept: re-planned on the
 * host, staged into the plan's own buffers (grown only when needed, so no device allocation in
 * a step loop); waits until the plan's previous stream launches have finished with its task
 * list (replays of a CUDA graph that captured the plan must be finished by the caller).
 * For codes whose lists change every step (tree codes): one plan per kind for the whole run. */
int  pgb5_plan_update(pgb5_plan *plan, int nitem, const int *items);
/* Tree-code interaction lists without copies: the items' j-ranges address the device index
 * list jidx (int32), record k of an item being jpos[jidx[j_offset + k]] (and its jaux words):
 * one plan for the point-mass lists (PGB5_NEWTON over the particle array) and one for the
 * cell lists (PGB5_QUAD over the cell array) of every group.  Tune with the same list.       */
int  pgb5_plan_launch_indexed(pgb5_plan *plan, const void *ipos, const void *jpos, const void *jaux,
                              const int *jidx, void *out, void *stream);
int  pgb5_plan_tune_indexed(pgb5_plan *plan, const void *ipos, const void *jpos, const void *jaux,
                            const int *jidx, void *out, void *stream, float *best_ms);
enum { PGB5_NCFG = 8 };

#ifdef __cplusplus
}
#endif

#endif /* PGB_G5_H */
