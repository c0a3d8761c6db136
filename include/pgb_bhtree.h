/*
 * pgb_bhtree.h -- C ABI of lib/libpgbtree.so: the Barnes-Hut octree, cell moments, i-groups and
 * interaction lists of the quadrupole tree code, built on the GPU.
 *
 * No counterpart among the reference's libraries: it replaces the tree construction and
 * make_interaction_list of the reference's tree code PG5/newton_quad/source.cpp (:418-514 tree,
 * :215-248 and :544-576 moments, :477-482 and :510-514 groups, :581-707 lists), whose lists feed
 * g5_* / g5c_* per group -- or, here, one batched pgb5_plan_launch_indexed per entry kind.  The
 * tree is the one the host builder (phantom-grape_b200/drivers/pgb_bhtree.c, bh_* accessors)
 * makes, bit for bit: same particle order, pre-order node numbering, FP64 moments, groups and
 * list entries.
 */
#ifndef PGB_BHTREE_H
#define PGB_BHTREE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pgbt_tree pgbt_tree;

/* n particles (x: n x 3, m: n, host arrays), opening angle theta, leaf size nleaf, group size
 * ncrit; NULL on bad arguments or failure (message in pgbt_last_error) */
pgbt_tree *pgbt_build(int n, const double *x, const double *m, double theta, int nleaf, int ncrit);
/* rebuild for n new particles with the same parameters, reusing the tree's device buffers (a
 * code that builds every step saves the allocations); PGB_OK or an error code */
int  pgbt_rebuild(pgbt_tree *tree, int n, const double *x, const double *m);
void pgbt_free(pgbt_tree *tree);
int  pgbt_n(const pgbt_tree *tree);
int  pgbt_ngroups(const pgbt_tree *tree);
int  pgbt_nnodes(const pgbt_tree *tree);
long long pgbt_np(const pgbt_tree *tree);   /* point-mass list entries of all groups */
long long pgbt_nc(const pgbt_tree *tree);   /* cell list entries of all groups */
float pgbt_build_ms(const pgbt_tree *tree); /* device time of the build (CUDA events) */

/* host copies, the layouts of the host builder's bh_* accessors */
int  pgbt_perm(pgbt_tree *tree, int *perm);                                   /* tree order -> input index */
int  pgbt_groups(pgbt_tree *tree, int *first, int *count, double *centre, double *half);
int  pgbt_cells(pgbt_tree *tree, double *com, double *mass, double *quad);    /* per node: com[3], mass, Q[6] */
int  pgbt_nodes(pgbt_tree *tree, int *first, int *count, double *half, double *centre, int *child);
int  pgbt_lists(pgbt_tree *tree, long long *poff, int *pidx, long long *coff, int *cidx);

/* device pointers for the batched force launch (valid until pgbt_free): particles float4
 * (x, y, z, m) in tree order; cells float4 (com, mass) and two float4 of quadrupole per cell
 * (xx, xy, xz, yy) (yz, zz, 0, 0); list offsets (int64) and entries (int32) */
int  pgbt_device(pgbt_tree *tree, void **part, void **cell, void **cquad, void **poff, void **pidx, void **coff,
                 void **cidx);
/* host copies of those records: part [n][4], cell [nnodes][4], cquad [nnodes][8] (any may be NULL) */
int  pgbt_records(pgbt_tree *tree, float *part, float *cell, float *cquad);
/* i-records float4 (x, y, z, eps2) in tree order into the caller's device buffer out[n] */
int  pgbt_irecords(pgbt_tree *tree, double eps2, void *out);
/* the groups' particle ranges (ngroup) and list offsets (ngroup + 1): the work items of the
 * batched launches (any pointer may be NULL) */
int  pgbt_group_table(pgbt_tree *tree, int *first, int *count, long long *poff, long long *coff);

int  pgbt_last_error(char *buf, int len);
void pgbt_clear_error(void);
void pgbt_set_abort(int on);

#ifdef __cplusplus
}
#endif

#endif /* PGB_BHTREE_H */
