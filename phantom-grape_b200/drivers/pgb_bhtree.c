/* pgb_bhtree.c -- host octree, multipole moments and interaction lists of the Barnes-Hut
 * quadrupole workload: the tree code that drives PG5/newton_quad's g5_* / g5c_* calls
 * (PG5/newton_quad/source.cpp), rebuilt as a flat C builder whose lists feed either the
 * per-group drop-in calls or one batched, index-list launch per entry kind.
 *
 * The tree follows the reference's rules:
 *  - an octree over a cube centred on the origin; a node is split while it holds more than
 *    `nleaf` particles (source.cpp:470-503); a particle goes to the child whose centre it
 *    exceeds on each axis, x the most significant octant bit (childindex, source.cpp:177-197);
 *  - a group (one set of i-particles) is the first node on each root-to-leaf path holding at
 *    most `ncrit` particles (source.cpp:477-482, 510-514);
 *  - node moments: mass, centre of mass and the traceless quadrupole
 *    Q = sum m (3 d d^T - |d|^2 I) about the centre of mass, leaves from their particles and
 *    internal nodes from their children by the parallel-axis shift (source.cpp:215-248,
 *    544-576), stored (xx, xy, xz, yy, yz, zz) with zz = -(xx + yy);
 *  - the interaction list of a group with cell centre g and half side h, from the root: a node
 *    with at most nleaf particles contributes its particles; otherwise each non-empty child
 *    contributes its particle if it holds one, itself as a quadrupole cell if
 *    theta^2 d^2 > (child side)^2 with d the distance from the child's centre of mass to the
 *    group's cube (per axis max(|x - g| - h, 0)), else its own list (make_interaction_list and
 *    calc_dist, source.cpp:581-707).
 * Differences: the root cube is the smallest power-of-two cube containing every particle
 * (the reference's calculate_size doubles at most once per coordinate); a group so far from
 * the whole tree that the root itself passes the opening test gets the root as one quadrupole
 * cell (the reference: one point mass) -- a case no group inside the root cube reaches.
 * Particles are kept in tree order (each node's particles are contiguous); perm maps tree
 * order to input order.  The builder is serial (O(N depth)); the lists are built by OpenMP
 * threads over groups (count pass, prefix sum, fill pass: deterministic). */
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    double c[3], half;  /* geometric centre and half side */
    int first, count;   /* particle range in tree order */
    int child[8];       /* node index, -1 for an empty octant; all -1 for a leaf */
    double com[3], mass, quad[6];
} bh_node;

typedef struct {
    int n;
    int *perm;          /* tree order -> input index */
    double *x, *m;      /* tree-order positions (3n) and masses */
    int nnode, capnode;
    bh_node *node;
    int nleaf;
    int ngroup;
    int *gnode;         /* node of each group, in tree order */
    long long *poff, *coff;  /* list offsets per group (ngroup + 1) */
    int *pidx, *cidx;   /* point-mass entries (tree-order particle indices), cells (node indices) */
} bh_tree;

#define BH_MAXDEPTH 40

static int new_node(bh_tree *T) {
    if (T->nnode == T->capnode) {
        int cap = T->capnode ? 2 * T->capnode : 1024;
        bh_node *p = (bh_node *)realloc(T->node, (size_t)cap * sizeof(bh_node));
        if (!p) return -1;
        T->node = p;
        T->capnode = cap;
    }
    return T->nnode++;
}

static int octant(const double *x, const double *c) {
    return ((x[0] > c[0]) << 2) | ((x[1] > c[1]) << 1) | (x[2] > c[2]);
}

/* Split node v (particles perm[first, first+count)) recursively; tmp is scratch of size n. */
static int build(bh_tree *T, const double *xin, int v, int depth, int *tmp) {
    bh_node *N = &T->node[v];
    for (int o = 0; o < 8; o++) N->child[o] = -1;
    if (N->count <= T->nleaf || depth >= BH_MAXDEPTH) return 0;
    int cnt[8] = {0}, start[8];
    const int first = N->first, count = N->count;
    const double c[3] = {N->c[0], N->c[1], N->c[2]}, half = N->half;
    for (int k = first; k < first + count; k++) cnt[octant(xin + 3 * (size_t)T->perm[k], c)]++;
    start[0] = first;
    for (int o = 1; o < 8; o++) start[o] = start[o - 1] + cnt[o - 1];
    int pos[8];
    memcpy(pos, start, sizeof pos);
    for (int k = first; k < first + count; k++) {
        const int p = T->perm[k];
        tmp[pos[octant(xin + 3 * (size_t)p, c)]++] = p;
    }
    memcpy(T->perm + first, tmp + first, (size_t)count * sizeof(int));
    for (int o = 0; o < 8; o++) {
        if (!cnt[o]) continue;
        const int w = new_node(T);
        if (w < 0) return -1;
        bh_node *C = &T->node[w];
        C->half = 0.5 * half;
        C->c[0] = c[0] + ((o & 4) ? C->half : -C->half);
        C->c[1] = c[1] + ((o & 2) ? C->half : -C->half);
        C->c[2] = c[2] + ((o & 1) ? C->half : -C->half);
        C->first = start[o];
        C->count = cnt[o];
        T->node[v].child[o] = w;  /* T->node may have moved: index again */
        if (build(T, xin, w, depth + 1, tmp)) return -1;
    }
    return 0;
}

static void quad_add(double q[6], double m, const double d[3]) {
    const double dd = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    q[0] += m * (3.0 * d[0] * d[0] - dd);
    q[1] += m * (3.0 * d[0] * d[1]);
    q[2] += m * (3.0 * d[0] * d[2]);
    q[3] += m * (3.0 * d[1] * d[1] - dd);
    q[4] += m * (3.0 * d[1] * d[2]);
}

/* Moments of node v and its subtree (children first). */
static void moments(bh_tree *T, int v) {
    bh_node *N = &T->node[v];
    int leaf = 1;
    for (int o = 0; o < 8; o++)
        if (N->child[o] >= 0) leaf = 0;
    double m = 0, s[3] = {0, 0, 0}, q[6] = {0, 0, 0, 0, 0, 0};
    if (leaf) {
        for (int k = N->first; k < N->first + N->count; k++) {
            m += T->m[k];
            for (int a = 0; a < 3; a++) s[a] += T->m[k] * T->x[3 * (size_t)k + a];
        }
        for (int a = 0; a < 3; a++) N->com[a] = s[a] / m;
        for (int k = N->first; k < N->first + N->count; k++) {
            const double d[3] = {T->x[3 * (size_t)k] - N->com[0], T->x[3 * (size_t)k + 1] - N->com[1],
                                 T->x[3 * (size_t)k + 2] - N->com[2]};
            if (N->count > 1) quad_add(q, T->m[k], d);
        }
    } else {
        for (int o = 0; o < 8; o++) {
            const int w = N->child[o];
            if (w < 0) continue;
            moments(T, w);
            N = &T->node[v];
            const bh_node *C = &T->node[w];
            m += C->mass;
            for (int a = 0; a < 3; a++) s[a] += C->mass * C->com[a];
        }
        for (int a = 0; a < 3; a++) N->com[a] = s[a] / m;
        for (int o = 0; o < 8; o++) {
            const int w = N->child[o];
            if (w < 0) continue;
            const bh_node *C = &T->node[w];
            const double d[3] = {C->com[0] - N->com[0], C->com[1] - N->com[1], C->com[2] - N->com[2]};
            quad_add(q, C->mass, d);
            if (C->count > 1)
                for (int k = 0; k < 5; k++) q[k] += C->quad[k];
        }
    }
    N->mass = m;
    q[5] = -(q[0] + q[3]);
    memcpy(N->quad, q, sizeof q);
}

static void find_groups(bh_tree *T, int v, int ncrit, int *out, int *ng) {
    const bh_node *N = &T->node[v];
    int leaf = 1;
    for (int o = 0; o < 8; o++)
        if (N->child[o] >= 0) leaf = 0;
    if (N->count <= ncrit || leaf) {
        if (out) out[*ng] = v;
        (*ng)++;
        return;
    }
    for (int o = 0; o < 8; o++)
        if (N->child[o] >= 0) find_groups(T, N->child[o], ncrit, out, ng);
}

/* distance^2 from point p to the cube (centre g, half side h) */
static double box_d2(const double p[3], const double g[3], double h) {
    double d2 = 0.0;
    for (int a = 0; a < 3; a++) {
        double d = fabs(p[a] - g[a]) - h;
        if (d > 0) d2 += d * d;
    }
    return d2;
}

/* Walk for one group; with pl/cl NULL only counts. */
static void walk(const bh_tree *T, int v, const double g[3], double h, double th2, int *pl, long long *np, int *cl,
                 long long *nc) {
    const bh_node *N = &T->node[v];
    if (N->count <= T->nleaf) {
        for (int k = N->first; k < N->first + N->count; k++) {
            if (pl) pl[*np] = k;
            (*np)++;
        }
        return;
    }
    int leaf = 1;
    for (int o = 0; o < 8; o++)
        if (N->child[o] >= 0) leaf = 0;
    if (leaf) {  /* depth-capped node of more than nleaf coincident particles */
        for (int k = N->first; k < N->first + N->count; k++) {
            if (pl) pl[*np] = k;
            (*np)++;
        }
        return;
    }
    for (int o = 0; o < 8; o++) {
        const int w = N->child[o];
        if (w < 0) continue;
        const bh_node *C = &T->node[w];
        if (C->count == 1) {
            if (pl) pl[*np] = C->first;
            (*np)++;
            continue;
        }
        const double side = 2.0 * C->half;
        if (box_d2(C->com, g, h) * th2 > side * side) {
            if (cl) cl[*nc] = w;
            (*nc)++;
        } else {
            walk(T, w, g, h, th2, pl, np, cl, nc);
        }
    }
}

static void group_list(const bh_tree *T, int gi, double th2, int *pl, long long *np, int *cl, long long *nc) {
    const bh_node *G = &T->node[T->gnode[gi]];
    const bh_node *R = &T->node[0];
    const double side = 2.0 * R->half;
    if (box_d2(R->com, G->c, G->half) * th2 < side * side) {
        walk(T, 0, G->c, G->half, th2, pl, np, cl, nc);
    } else {
        if (cl) cl[*nc] = 0;
        (*nc)++;
    }
}

void bh_free(bh_tree *T) {
    if (!T) return;
    free(T->perm);
    free(T->x);
    free(T->m);
    free(T->node);
    free(T->gnode);
    free(T->poff);
    free(T->coff);
    free(T->pidx);
    free(T->cidx);
    free(T);
}

/* Build the tree of n particles (x: n x 3, m: n) and every group's interaction list.
 * Returns NULL on allocation failure or bad arguments. */
bh_tree *bh_build(int n, const double *x, const double *m, double theta, int nleaf, int ncrit) {
    if (n <= 0 || !x || !m || nleaf < 1 || ncrit < 1 || theta <= 0) return NULL;
    bh_tree *T = (bh_tree *)calloc(1, sizeof(bh_tree));
    if (!T) return NULL;
    T->n = n;
    T->nleaf = nleaf;
    T->perm = (int *)malloc((size_t)n * sizeof(int));
    int *tmp = (int *)malloc((size_t)n * sizeof(int));
    if (!T->perm || !tmp) goto fail;
    double maxabs = 0.0;
    for (size_t k = 0; k < 3 * (size_t)n; k++) maxabs = fmax(maxabs, fabs(x[k]));
    double R = 1.0;  /* the smallest power of two above every |coordinate| */
    if (maxabs > 0) {
        while (R <= maxabs) R *= 2.0;
        while (R * 0.5 > maxabs) R *= 0.5;
    }
    for (int k = 0; k < n; k++) T->perm[k] = k;
    {
        const int r = new_node(T);
        if (r < 0) goto fail;
        bh_node *N = &T->node[r];
        N->c[0] = N->c[1] = N->c[2] = 0.0;
        N->half = R;
        N->first = 0;
        N->count = n;
    }
    if (build(T, x, 0, 0, tmp)) goto fail;
    free(tmp);
    tmp = NULL;
    T->x = (double *)malloc(3 * (size_t)n * sizeof(double));
    T->m = (double *)malloc((size_t)n * sizeof(double));
    if (!T->x || !T->m) goto fail;
    for (int k = 0; k < n; k++) {
        const int p = T->perm[k];
        T->x[3 * (size_t)k] = x[3 * (size_t)p];
        T->x[3 * (size_t)k + 1] = x[3 * (size_t)p + 1];
        T->x[3 * (size_t)k + 2] = x[3 * (size_t)p + 2];
        T->m[k] = m[p];
    }
    moments(T, 0);
    {
        int ng = 0;
        find_groups(T, 0, ncrit, NULL, &ng);
        T->gnode = (int *)malloc((size_t)ng * sizeof(int));
        if (!T->gnode) goto fail;
        T->ngroup = 0;
        find_groups(T, 0, ncrit, T->gnode, &T->ngroup);
    }
    {
        const int ng = T->ngroup;
        const double th2 = theta * theta;
        long long *np = (long long *)calloc((size_t)ng, sizeof(long long));
        long long *nc = (long long *)calloc((size_t)ng, sizeof(long long));
        T->poff = (long long *)malloc(((size_t)ng + 1) * sizeof(long long));
        T->coff = (long long *)malloc(((size_t)ng + 1) * sizeof(long long));
        if (!np || !nc || !T->poff || !T->coff) {
            free(np);
            free(nc);
            goto fail;
        }
#pragma omp parallel for schedule(dynamic, 16)
        for (int g = 0; g < ng; g++) group_list(T, g, th2, NULL, &np[g], NULL, &nc[g]);
        T->poff[0] = T->coff[0] = 0;
        for (int g = 0; g < ng; g++) {
            T->poff[g + 1] = T->poff[g] + np[g];
            T->coff[g + 1] = T->coff[g] + nc[g];
        }
        T->pidx = (int *)malloc((size_t)(T->poff[ng] > 0 ? T->poff[ng] : 1) * sizeof(int));
        T->cidx = (int *)malloc((size_t)(T->coff[ng] > 0 ? T->coff[ng] : 1) * sizeof(int));
        if (!T->pidx || !T->cidx) {
            free(np);
            free(nc);
            goto fail;
        }
#pragma omp parallel for schedule(dynamic, 16)
        for (int g = 0; g < ng; g++) {
            long long a = 0, b = 0;
            group_list(T, g, th2, T->pidx + T->poff[g], &a, T->cidx + T->coff[g], &b);
        }
        free(np);
        free(nc);
    }
    return T;
fail:
    free(tmp);
    bh_free(T);
    return NULL;
}

/* ---- accessors (plain arrays for ctypes callers) ---- */
int bh_n(const bh_tree *T) { return T->n; }
int bh_ngroups(const bh_tree *T) { return T->ngroup; }
int bh_nnodes(const bh_tree *T) { return T->nnode; }
long long bh_np(const bh_tree *T) { return T->poff[T->ngroup]; }
long long bh_nc(const bh_tree *T) { return T->coff[T->ngroup]; }

/* perm[n]: tree order -> input index */
void bh_perm(const bh_tree *T, int *perm) { memcpy(perm, T->perm, (size_t)T->n * sizeof(int)); }

/* per group: first particle (tree order), count, cell centre (3), half side */
void bh_groups(const bh_tree *T, int *first, int *count, double *centre, double *half) {
    for (int g = 0; g < T->ngroup; g++) {
        const bh_node *G = &T->node[T->gnode[g]];
        first[g] = G->first;
        count[g] = G->count;
        for (int a = 0; a < 3; a++) centre[3 * g + a] = G->c[a];
        half[g] = G->half;
    }
}

/* per node: centre of mass (3), mass, quadrupole (6) */
void bh_cells(const bh_tree *T, double *com, double *mass, double *quad) {
    for (int v = 0; v < T->nnode; v++) {
        const bh_node *N = &T->node[v];
        for (int a = 0; a < 3; a++) com[3 * (size_t)v + a] = N->com[a];
        mass[v] = N->mass;
        for (int k = 0; k < 6; k++) quad[6 * (size_t)v + k] = N->quad[k];
    }
}

/* per node: particle range (tree order), half side, centre (3), children (8, -1 = empty) */
void bh_nodes(const bh_tree *T, int *first, int *count, double *half, double *centre, int *child) {
    for (int v = 0; v < T->nnode; v++) {
        const bh_node *N = &T->node[v];
        first[v] = N->first;
        count[v] = N->count;
        half[v] = N->half;
        for (int a = 0; a < 3; a++) centre[3 * (size_t)v + a] = N->c[a];
        for (int o = 0; o < 8; o++) child[8 * (size_t)v + o] = N->child[o];
    }
}

/* list offsets (ngroup + 1 each) and entries */
void bh_lists(const bh_tree *T, long long *poff, int *pidx, long long *coff, int *cidx) {
    memcpy(poff, T->poff, ((size_t)T->ngroup + 1) * sizeof(long long));
    memcpy(coff, T->coff, ((size_t)T->ngroup + 1) * sizeof(long long));
    memcpy(pidx, T->pidx, (size_t)T->poff[T->ngroup] * sizeof(int));
    memcpy(cidx, T->cidx, (size_t)T->coff[T->ngroup] * sizeof(int));
}
