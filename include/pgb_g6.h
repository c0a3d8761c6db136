/*
 * pgb_g6.h -- C ABI of lib/libpg6.so: the GRAPE-6 4th-order Hermite API on the B200 engine.
 *
 * Drop-in replacement for the reference library built from PG6/libpg6 (gp6util.h:1-101):
 * same symbols (each with its Fortran `_` twin), same conventions: g6_set_j_particle takes
 * acc/2 and jerk/6, g6calc_lasthalf* return acc = sum m dx/r^3, jerk, pot = -sum m/r with the
 * self pair excluded by id, nnb = nearest-neighbour id, rnnb = its softened distance.
 * Differences are listed in the library source (csrc/pgb_g6.cu header comment).
 */
#ifndef PGB_G6_H
#define PGB_G6_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- GRAPE-6 API: PG6/libpg6/gp6util.h:1-101 (phantom_g6.c line numbers) ---------------- */
void g6_open(int gpid);                   /* :18-26 */
void g6_open_(int *gpid);
void g6_set_tunit(int tunit);             /* :36-40 (no-op) */
void g6_set_tunit_(int *tunit);
void g6_set_xunit(int xunit);             /* :50-54 (no-op) */
void g6_set_xunit_(int *xunit);
void g6_reset(int gpid);                  /* :64-68 (no-op) */
void g6_reset_(int *gpid);
void g6_reset_fofpga(int gpid);           /* :78-82 (no-op) */
void g6_reset_fofpga_(int *gpid);
void g6_close(int gpid);                  /* :92-96 */
void g6_close_(int *gpid);
int  g6_npipes(void);                     /* :106-109 (48; PGB_G6_NPIPES) */
int  g6_npipes_(void);
void g6_set_j_particle(int gpid, int padr, int pidx, double t, double dt, double mss,
                       double *snp, double *jrk, double *acc, double *vel, double *pos);   /* :118-125 */
void g6_set_j_particle_(int *gpid, int *padr, int *pidx, double *t, double *dt, double *mss,
                        double *snp, double *jrk, double *acc, double *vel, double *pos);
void g6_set_ti(int gpid, double time);    /* :138-143 */
void g6_set_ti_(int *gpid, double *time);
void g6calc_firsthalf(int gpid, int nj, int ni, int *pidx, double (*pos)[3], double (*vel)[3],
                      double (*acc)[3], double (*jrk)[3], double *pot, double eps2, double *h2);  /* :153-164 */
void g6calc_firsthalf_(int *gpid, int *nj, int *ni, int *pidx, double (*pos)[3], double (*vel)[3],
                       double (*acc)[3], double (*jrk)[3], double *pot, double *eps2, double *h2);
int  g6calc_lasthalf(int gpid, int nj, int ni, int *pidx, double (*pos)[3], double (*vel)[3], double eps2,
                     double *h2, double (*acc)[3], double (*jrk)[3], double *pot);                 /* :177-211 */
int  g6calc_lasthalf_(int *gpid, int *nj, int *ni, int *pidx, double (*pos)[3], double (*vel)[3], double *eps2,
                      double *h2, double (*acc)[3], double (*jrk)[3], double *pot);
int  g6calc_lasthalf2(int gpid, int nj, int ni, int *pidx, double (*pos)[3], double (*vel)[3], double eps2,
                      double *h2, double (*acc)[3], double (*jrk)[3], double *pot, int *nnb);      /* :223-258 */
int  g6calc_lasthalf2_(int *gpid, int *nj, int *ni, int *pidx, double (*pos)[3], double (*vel)[3],
                       double *eps2, double *h2, double (*acc)[3], double (*jrk)[3], double *pot, int *nnb);
int  g6calc_lasthalf2p(int gpid, int nj, int ni, int *pidx, double (*pos)[3], double (*vel)[3], double eps2,
                       double *h2, double (*acc)[3], double (*jrk)[3], double *pot, int *nnb,
                       float *rnnb);                                                            /* :270-306 */
int  g6calc_lasthalf2p_(int *gpid, int *nj, int *ni, int *pidx, double (*pos)[3], double (*vel)[3],
                        double *eps2, double *h2, double (*acc)[3], double (*jrk)[3], double *pot, int *nnb,
                        float *rnnb);
int  g6calc_lasthalfn(int gpid, int nj, int ni, int *pidx, double (*pos)[3], double (*vel)[3], double eps2,
                      double *h2, double (*acc)[3], double (*jrk)[3], double *pot);                /* :318-355 */
int  g6calc_lasthalfn_(int *gpid, int *nj, int *ni, int *pidx, double (*pos)[3], double (*vel)[3],
                       double *eps2, double *h2, double (*acc)[3], double (*jrk)[3], double *pot);
int  g6calc_lasthalf2n(int gpid, int nj, int ni, int *pidx, double (*pos)[3], double (*vel)[3], double eps2,
                       double *h2, double (*acc)[3], double (*jrk)[3], double *pot, int *nnb);     /* :367-405 */
int  g6calc_lasthalf2n_(int *gpid, int *nj, int *ni, int *pidx, double (*pos)[3], double (*vel)[3],
                        double *eps2, double *h2, double (*acc)[3], double (*jrk)[3], double *pot, int *nnb);
int  g6calc_lasthalf2np(int gpid, int nj, int ni, int *pidx, double (*pos)[3], double (*vel)[3], double eps2,
                        double *h2, double (*acc)[3], double (*jrk)[3], double *pot, int *nnb,
                        float *rnnb);                                                           /* :417-456 */
int  g6calc_lasthalf2np_(int *gpid, int *nj, int *ni, int *pidx, double (*pos)[3], double (*vel)[3],
                         double *eps2, double *h2, double (*acc)[3], double (*jrk)[3], double *pot, int *nnb,
                         float *rnnb);
void g6_setup_njdata(int gpid, int nj);   /* :468-472 (no-op) */
void g6_setup_njdata_(int *gpid, int *nj);
int  g6_read_neighbour_list(int gpid);    /* :482-486: 0 ok, 1 overflow */
int  g6_read_neighbour_list_(int *gpid);
int  g6_get_neighbour_list(int gpid, int ipipe, int maxlen, int *nblen, int *nbl);   /* :495-499 */
int  g6_get_neighbour_list_(int *gpid, int *ipipe, int *maxlen, int *nblen, int *nbl);
void g6_debugfunc(int tmp);               /* :508-517 */
void g6_debugfunc_(int *tmp);
void g6_debugfunc_double(double tmp);     /* :527-535 */
void g6_debugfunc_double_(double *tmp);
void g6_dump(double tim, int n, double *m, double (*x)[3], double (*v)[3]);   /* :545-561 */
void g6_dump_(double *tim, int *n, double *m, double (*x)[3], double (*v)[3]);

/* ---- library status (no reference counterpart: the reference has no error reporting) ---- */
int  pgb6_last_error(char *buf, int len);
void pgb6_clear_error(void);
void pgb6_set_abort(int on);
/* Device time of the drop-in calls (no reference counterpart): with timing on, every
 * g6calc_firsthalf (j update + prediction) and g6calc_lasthalf* (force) adds the device time
 * between CUDA events around its work to a total, read (and cleared with reset != 0) in ms. */
void   pgb6_set_call_timing(int on);
double pgb6_call_device_ms(int reset);

/* ---- batched path (no reference counterpart) ----------------------------------------------
 * Replaces loops of g6calc_firsthalf/lasthalf over npipes-sized i chunks (PG6/banana/
 * hermite.c:214-252), or over independent clusters, by one persistent launch.
 * items[k] = {i_offset, i_count, j_offset, j_count}.  Device records (sizes from
 * pgb6_record_sizes): j-memory G6Ptcl {double pos[3], vel[3], acc2[3], jrk6[3], mass, tim;
 * int idx, pad[3]} (128 B), predicted j G6PredJ {POS p; float m; int id; float vx, vy, vz,
 * pad} (48 B), i G6I {POS p; float vx, vy, vz; int id; float h2, pad} (48 B), where POS is
 * 24 bytes: by default the double-float layout {float xh, yh, zh, xl, yl, zl} (x = xh + xl,
 * xh = (float)x), with flag PGB6_POS_F64 {double x, y, z}; result G6Out {double ax, ay, az,
 * jx, jy, jz, pot; float key; int jadr} (64 B) with key = -2/r_soft of the nearest neighbour
 * and jadr its j address (flags & PGB6_NN).                                                 */
enum { PGB6_NN = 1, PGB6_POS_F64 = 2 };
typedef struct pgb6_plan pgb6_plan;
void pgb6_record_sizes(int *ptcl, int *predj, int *irec, int *out);
int  pgb6_plan_create(pgb6_plan **plan, int nitem, const int *items, int flags);
int  pgb6_plan_launch(pgb6_plan *plan, const void *ipart, const void *jpred, double eps2, void *out,
                      void *stream);
void pgb6_plan_destroy(pgb6_plan *plan);
long long pgb6_plan_interactions(const pgb6_plan *plan);
int  pgb6_plan_tasks(const pgb6_plan *plan);
int  pgb6_plan_config(const pgb6_plan *plan);
/* j-chunks per i-tile of a one-item plan (1: unsplit; 0: a plan of several items) */
int  pgb6_plan_chunks(const pgb6_plan *plan);
/* kernels one pgb6_plan_launch issues (the force kernel, plus the nearest-neighbour lookup kernel
 * of split i-tiles when the plan's configuration defers them) */
int  pgb6_plan_kernels(const pgb6_plan *plan);
/* new items for an existing plan (its flags and configuration kept), staged into its own buffers
 * (no device allocation in a step loop); waits for the plan's previous stream launches */
int  pgb6_plan_update(pgb6_plan *plan, int nitem, const int *items);
int  pgb6_plan_set_config(pgb6_plan *plan, int cfg);   /* pin one of PGB6_NCFG configurations */
enum { PGB6_NCFG = 10 };
/* autotuner: times every kernel configuration on the caller's data, keeps the fastest for this
 * plan and for later plans of the same shape; returns the configuration, *best_ms its time */
int  pgb6_plan_tune(pgb6_plan *plan, const void *ipart, const void *jpred, double eps2, void *out,
                    void *stream, float *best_ms);
/* FP64 j predictor on device records (gravity.c:149-193): pred[j] = predict(ptcl[j], ti);
 * flags & PGB6_POS_F64 writes FP64 positions, else the double-float layout */
int  pgb6_predict(const void *ptcl, int nj, double ti, void *pred, int flags, void *stream);
/* host-buffer batch: inputs and outputs in host memory, copies included; nnb/rnnb optional */
int  pgb6_batch_host(int nitem, const int *items, int ni, const double (*xi)[3], const double (*vi)[3],
                     const int *idi, int nj, const double (*xj)[3], const double (*vj)[3], const double *mj,
                     const int *idj, double eps2, double (*acc)[3], double (*jrk)[3], double *pot, int *nnb,
                     float *rnnb);

/* ---- allocation-free force call (no counterpart in the reference) ------------------------
 * For callers that cannot let a library allocate GPU memory: codes whose device memory is
 * owned by their own pool allocator, and step loops that cannot afford the device-wide
 * synchronisation of cudaMalloc / cudaFree.  Same kernel and results as a one-item plan
 * (ni G6I records against nj G6PredJ records, G6Out results, flags PGB6_NN / PGB6_POS_F64),
 * but its work list and partial sums live in a fixed 16 MiB array of the library's static
 * device memory (held on every GPU the library is loaded on until exit); it never calls
 * cudaMalloc or cudaFree.  Limit: at most 4096 i-tiles (ni <= 1,048,576 with the 256-particle
 * tile that large calls use); larger ni returns
 * PGB_ERR_CAPACITY.  The first call on a device looks up the array's address there and
 * should come before any stream capture.  All calls share the array: calls that overlap on
 * the GPU race and must be serialised by the caller. */
int  pgb6_force_noalloc(const void *ipart, int ni, const void *jpred, int nj, double eps2, void *out, int flags,
                        void *stream);

/* ---- Hermite block-time-step integrator on the device (no counterpart in the reference's
 * libraries).  Replaces the steps of the reference's sample integrator around the force call
 * (PG6/banana, -DNORMAL): global_time (timestep.c:87-98), predict_exmotion (hermite.c:39-63),
 * the g6_set_j_particle re-send of the active particles (hermite.c:240-265), correct /
 * correct_sgmotion (hermite.c:67-108, 143-205), dt_criterion (timestep.c:53-85), the start-up
 * step startup_sgmotion / dt_startup (hermite.c:110-141, timestep.c:24-51) and reset_time every
 * dtmax (timestep.c:127-135, banana01.c:161-179).  The state stays in device memory between
 * steps; given the same forces a step's new state equals the reference's formulas evaluated in
 * plain FP64 bit for bit.  The force is the GRAPE-6 kernel of this library (eps2, id-excluded
 * self pair).                                                                                  */
typedef struct pgb6_hermite pgb6_hermite;
/* 2 <= n <= 2^20 particles; takes the start-up step (forces at t = 0, first steps); PGB_ERR_ARG
 * when a start-up step falls below dtmax / 2^51 */
int  pgb6_hermite_create(pgb6_hermite **h, int n, const double *mass, const double (*pos)[3],
                         const double (*vel)[3], double eps2, double eta, double eta_s, double dtmax);
/* one block step; *time = global time after it, *ni = particles advanced (both optional) */
int  pgb6_hermite_step(pgb6_hermite *h, double *time, int *ni);
/* block steps while the global time is below tend; steps taken by this call (optional) */
int  pgb6_hermite_advance(pgb6_hermite *h, double tend, long long *psteps, long long *bsteps);
double pgb6_hermite_time(pgb6_hermite *h);
/* Fault handling of the step kernel: every wait (grid barrier, segment / task flag) gives up
 * after a limit of SM cycles (default about a second; cycles <= 0 restores it), after which
 * every CTA returns, the call reports PGB_ERR_DEVICE and the integrator is unusable.
 * wait_status reads whether a wait gave up, how many CTAs have returned from the kernel (over
 * all launches) and the CTAs per launch. */
int  pgb6_hermite_set_wait_limit(pgb6_hermite *h, long long cycles);
int  pgb6_hermite_wait_status(pgb6_hermite *h, int *gave_up, int *exits, int *grid);
/* state as struct Particle holds it (any pointer may be NULL; jrk, pot with float values) */
int  pgb6_hermite_get(pgb6_hermite *h, double *t, double *dt, double (*pos)[3], double (*vel)[3],
                      double (*acc)[3], double (*jrk)[3], double *pot);
/* the last step's active particles and their force-kernel results; returns their count */
int  pgb6_hermite_last_step(pgb6_hermite *h, int *active, double (*acc)[3], double (*jrk)[3], double *pot);
/* kinetic and potential energy, calc_energy.c:9-33 */
int  pgb6_hermite_energy(pgb6_hermite *h, double *ek, double *ew);
/* particle and block steps since creation (the start-up step counts n and 1) */
void pgb6_hermite_counts(pgb6_hermite *h, long long *psteps, long long *bsteps);
/* the integrator's CUDA stream (cudaStream_t) */
void *pgb6_hermite_stream(pgb6_hermite *h);
/* pair interactions so far (active x n) and steps by force decomposition (i-tile 16, 32, 64,
 * 128, 512); any pointer may be NULL */
void pgb6_hermite_stats(pgb6_hermite *h, long long *pairs, long long *steps_by_tile);
void pgb6_hermite_destroy(pgb6_hermite *h);

#ifdef __cplusplus
}
#endif

#endif /* PGB_G6_H */
