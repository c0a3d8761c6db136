/*
 * pgb_g5table.h -- C ABI of lib/libpg5table.so: the GRAPE-5 API with a table-interpolated
 * cutoff force (the TreePM particle-particle part) on the B200 engine.
 *
 * Drop-in replacement for the reference library built from PG5/table/libpg5 (gp5util.h,
 * pg5_table.h): same symbols and conventions (positions scaled by xscale on set_*, forces
 * a = sum m dx f(s), no potential: g5_get_force returns pot = 0).  The table is generated in
 * the reference's float arithmetic, bit-identical to the reference's Force_table.
 */
#ifndef PGB_G5TABLE_H
#define PGB_G5TABLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- GRAPE-5 API of the table library: PG5/table/libpg5/gp5util.h:9-35 ------------------ */
void g5_open(void);                 /* phantom_g5.c:56-61: builds the default S2 table */
void g5_close(void);                /* phantom_g5.c:63-67 */
int  g5_get_number_of_pipelines(void);                                 /* phantom_g5.c:52-54 */
void g5_set_range(double xmin, double xmax, double mmin);             /* phantom_g5.c:77-78 (no-op) */
void g5_set_eta(double eta);                                           /* phantom_g5.c:69-71 */
void g5_set_eps_to_all(double eps);                                    /* phantom_g5.c:73-75 (unused) */
void g5_set_n(int n);                                                  /* phantom_g5.c:92-94 */
void g5_set_nMC(int devid, int n);                                     /* phantom_g5.c:86-90 */
void g5_set_xmj(int adr, int nj, double (*xj)[3], double *mj);         /* phantom_g5.c:130-132 */
void g5_set_xmjMC(int devid, int adr, int nj, double (*xj)[3], double *mj);  /* phantom_g5.c:112-128 */
void g5_set_xi(int ni, double (*xi)[3]);                               /* phantom_g5.c:108-110 */
void g5_set_xiMC(int devid, int ni, double (*xi)[3]);                  /* phantom_g5.c:96-106 */
void g5_run(void);                                                     /* phantom_g5.c:141-143 */
void g5_runMC(int devid);                                              /* phantom_g5.c:134-139 */
void g5_get_force(int ni, double (*a)[3], double *p);                  /* phantom_g5.c:156-158 */
void g5_get_forceMC(int devid, int ni, double (*a)[3], double *p);     /* phantom_g5.c:145-154 */
void g5_calculate_force_on_x(double (*x)[3], double (*a)[3], double *p, int ni);             /* :173-176 */
void g5_calculate_force_on_xMC(int devid, double (*x)[3], double (*a)[3], double *p, int ni);  /* :160-170 */
/* a stub in the reference (phantom_g5.c:80-84); here it installs ffunc with cutoff fcut */
void g5_set_cutoff_table(double (*ffunc)(double), double fcut, double fcor,
                         double (*pfunc)(double), double pcut, double pcor);

/* ---- table generation: PG5/table/libpg5/pg5_table.h:38-40 -------------------------------- */
void pg5_gen_force_table(double (*force_func)(double), double rcut);   /* pg5_table.c:43-113 */
void pg5_gen_s2_force_table(double sft_for_PP, double sft_for_PM);    /* pg5_table.c:31-35 */
void pg5_set_xscale(double xscale);                                    /* phantom_g5.c:43-50 */
/* the reference's table entries as a global (pg5_table.h:31); here [4096][2], first rows used */
extern float Force_table[4096][2];

/* ---- extensions (no reference counterpart) ----------------------------------------------- */
/* table resolution 2^(exp_bit+frc_bit); the reference fixes EXP_BIT 4, FRC_BIT 5 at compile
 * time (pg5_table.h:7-17); exp_bit must be 4, frc_bit 1..8; applies at the next generation */
int  pg5_set_table_bits(int exp_bit, int frc_bit);
/* copy of the current table (min(n, max_entries) rows of (f, df/ds)); returns n, sets xscale */
int  pg5_get_table(float *out, int max_entries, double *xscale);
int  pgb5_last_error(char *buf, int len);
void pgb5_clear_error(void);
void pgb5_set_abort(int on);

/* batched path (see pgb_g5.h): kind must be PGB5_TABLE (3); ipos/jpos are float4 records in
 * table units (coordinates multiplied by xscale, as g5_set_xi / g5_set_xmj do); jaux unused;
 * out double4 (ax, ay, az, 0) with acc already divided by xscale. */
typedef struct pgb5_plan pgb5_plan;
int  pgb5_plan_create(pgb5_plan **plan, int kind, int nitem, const int *items);
int  pgb5_plan_launch(pgb5_plan *plan, const void *ipos, const void *jpos, const void *jaux, void *out,
                      void *stream);
void pgb5_plan_destroy(pgb5_plan *plan);
long long pgb5_plan_interactions(const pgb5_plan *plan);
int  pgb5_plan_tasks(const pgb5_plan *plan);
/* autotuner and configuration pinning, as in pgb_g5.h (the table kind uses configurations
 * 0, 1, 5, 6 and 7: CTAs of at most 256 threads) */
int  pgb5_plan_tune(pgb5_plan *plan, const void *ipos, const void *jpos, const void *jaux, void *out,
                    void *stream, float *best_ms);
int  pgb5_plan_config(const pgb5_plan *plan);
int  pgb5_plan_set_config(pgb5_plan *plan, int cfg);   /* pin one (PGB5_NCFG configurations) */
int  pgb5_plan_update(pgb5_plan *plan, int nitem, const int *items);   /* as in pgb_g5.h */
/* index-list launch and tuning, as in pgb_g5.h */
int  pgb5_plan_launch_indexed(pgb5_plan *plan, const void *ipos, const void *jpos, const void *jaux,
                              const int *jidx, void *out, void *stream);
int  pgb5_plan_tune_indexed(pgb5_plan *plan, const void *ipos, const void *jpos, const void *jaux,
                            const int *jidx, void *out, void *stream, float *best_ms);
enum { PGB5_NCFG = 8 };

#ifdef __cplusplus
}
#endif

#endif /* PGB_G5TABLE_H */
