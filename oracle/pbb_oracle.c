/*
 * pbb_oracle.c -- CPU restatement of the PBBPerm flow-shop bounds and of its
 * sequential IVM branch-and-bound, used ONLY as a test oracle and as the
 * timed CPU port in bench.py.  Nothing in the product links this file.
 *
 * Parity is pinned by tests/ against (1) the reference's own bounds library
 * and multicore B&B built from source into oracle/_ref/ (oracle/build_ref.py)
 * and (2) golden fixtures those binaries produced (tests/golden/).
 *
 * Every function names the reference file:line whose behaviour it restates.
 * All arithmetic is int32, exactly as in the reference.
 */
#include <limits.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MAXN 128
#define ORC_MAXM 64

typedef struct {
    int n, m, P;
    int *p;         /* [m][n] processing times, row-major (machine-major)       */
    int *min_arr;   /* earliest start per machine  (bound_fsp_weak.cpp:249-286) */
    int *min_dep;   /* min run-out per machine                                 */
    int *mach0;     /* [P] first machine of pair  (bound_fsp_strong.cpp:283-297)*/
    int *mach1;     /* [P] second machine of pair                              */
    int *lag;       /* [P][n] sum of p over machines strictly between the pair  */
    int *johnson;   /* [P][n] Johnson order of jobs for the pair               */
    int pair_mode;  /* JohnsonMode 0 (all pairs) / 1 (k,m-1) / 2 (k,k+1)         */
} orc_inst;

static int imax(int a, int b) { return a > b ? a : b; }

/* ------------------------------------------------------------------------ */
/* instances                                                                */
/* ------------------------------------------------------------------------ */

static uint64_t splitmix64_next(uint64_t *s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

/* Project PRNG for synthetic instances: p = lo + (u mod span) with rejection
 * of the biased tail, row-major m x n.  Mirrored bit-for-bit by
 * pbbperm_b200/instances.py and the C++ host (csrc/pbb_host.cpp). */
uint64_t orc_uniform(uint64_t *state, uint32_t lo, uint32_t hi)
{
    uint64_t span = (uint64_t)(hi - lo + 1);
    uint64_t limit = UINT64_MAX - (UINT64_MAX % span);
    uint64_t u;
    do { u = splitmix64_next(state); } while (u >= limit);
    return lo + (u % span);
}

void orc_synthetic_instance(uint64_t seed, int n, int m, int lo, int hi, int *p)
{
    uint64_t s = seed;
    for (int k = 0; k < m; k++)
        for (int j = 0; j < n; j++)
            p[k * n + j] = (int)orc_uniform(&s, (uint32_t)lo, (uint32_t)hi);
}

/* Taillard's generator (bounds/src/instance_flowshop.cpp:78-101): the
 * Park-Miller minimal-standard LCG via Schrage's method, mapped to [lo,hi]
 * through a float division.  The caller supplies the time seed. */
void orc_taillard_instance(long seed, int n, int m, int *p)
{
    const long M = 2147483647, A = 16807, Q = 127773, R = 2836;
    for (int k = 0; k < m; k++)
        for (int j = 0; j < n; j++) {
            long hi = seed / Q;
            seed = A * (seed % Q) - hi * R;
            if (seed < 0) seed += M;
            double u01 = (float)seed / (float)M;
            p[k * n + j] = (int)(1 + (long)(u01 * 99));
        }
}

/* ------------------------------------------------------------------------ */
/* tables                                                                   */
/* ------------------------------------------------------------------------ */

/* bound_fsp_weak.cpp:249-286 (and its twin bound_fsp_strong.cpp:300-340). */
static void fill_min_times(orc_inst *I)
{
    int n = I->n, m = I->m;
    int acc[ORC_MAXM];
    for (int k = 0; k < m; k++) { I->min_dep[k] = INT_MAX; I->min_arr[k] = INT_MAX; }
    I->min_dep[m - 1] = 0;
    I->min_arr[0] = 0;
    for (int j = 0; j < n; j++) {
        /* suffix sums from the last machine */
        acc[m - 1] = I->p[(m - 1) * n + j];
        for (int k = m - 2; k >= 0; k--) acc[k] = acc[k + 1] + I->p[k * n + j];
        for (int k = m - 2; k >= 0; k--) if (acc[k + 1] < I->min_dep[k]) I->min_dep[k] = acc[k + 1];
        /* prefix sums from the first machine */
        acc[0] = I->p[j];
        for (int k = 1; k < m; k++) acc[k] = acc[k - 1] + I->p[k * n + j];
        for (int k = 1; k < m; k++) if (acc[k - 1] < I->min_arr[k]) I->min_arr[k] = acc[k - 1];
    }
}

/* Johnson ordering keys (bound_fsp_strong.cpp:417-436): group 1 = jobs whose
 * first-machine time is strictly smaller, sorted by increasing (p1+lag);
 * group 2 sorted by decreasing (p2+lag).  The order among equal keys is the
 * one produced by the reference's Hoare-partition quicksort with the first
 * element as pivot (:359-414); restated here because ties change the LB. */
typedef struct { const int *grp; const int *key; } jkeys;

static int j_less(const jkeys *K, int a, int b)
{
    if (K->grp[a] == K->grp[b])
        return K->grp[a] == 1 ? K->key[a] < K->key[b] : K->key[a] > K->key[b];
    return K->grp[a] < K->grp[b];
}

static int j_greater(const jkeys *K, int a, int b)
{
    if (K->grp[a] == K->grp[b])
        return K->grp[a] == 1 ? K->key[a] > K->key[b] : K->key[a] < K->key[b];
    return K->grp[a] > K->grp[b];
}

static void j_sort(const jkeys *K, int *v, int lo, int hi)
{
    while (hi - lo > 0) {
        int pivot = v[lo];
        int i = lo - 1, j = hi + 1;
        for (;;) {
            do j--; while (j_greater(K, v[j], pivot));
            do i++; while (j_less(K, v[i], pivot));
            if (i < j) { int t = v[i]; v[i] = v[j]; v[j] = t; } else break;
        }
        j_sort(K, v, lo, j);
        lo = j + 1;
    }
}

orc_inst *orc_create(int n, int m, const int *p, int pair_mode)
{
    if (n < 1 || n > ORC_MAXN || m < 2 || m > ORC_MAXM) return NULL;
    orc_inst *I = (orc_inst *)calloc(1, sizeof(orc_inst));
    I->n = n; I->m = m; I->P = m * (m - 1) / 2; I->pair_mode = pair_mode;
    I->p = (int *)malloc(sizeof(int) * n * m);
    memcpy(I->p, p, sizeof(int) * n * m);
    I->min_arr = (int *)malloc(sizeof(int) * m);
    I->min_dep = (int *)malloc(sizeof(int) * m);
    fill_min_times(I);
    I->mach0 = (int *)malloc(sizeof(int) * I->P);
    I->mach1 = (int *)malloc(sizeof(int) * I->P);
    I->lag = (int *)malloc(sizeof(int) * I->P * n);
    I->johnson = (int *)malloc(sizeof(int) * I->P * n);
    int s = 0;
    for (int a = 0; a < m - 1; a++)
        for (int b = a + 1; b < m; b++, s++) { I->mach0[s] = a; I->mach1[s] = b; }
    int grp[ORC_MAXN], key[ORC_MAXN];
    for (s = 0; s < I->P; s++) {
        int a = I->mach0[s], b = I->mach1[s];
        for (int j = 0; j < n; j++) {
            int l = 0;
            for (int k = a + 1; k < b; k++) l += p[k * n + j];
            I->lag[s * n + j] = l;
        }
        for (int j = 0; j < n; j++) {
            I->johnson[s * n + j] = j;
            if (p[a * n + j] < p[b * n + j]) { grp[j] = 1; key[j] = p[a * n + j] + I->lag[s * n + j]; }
            else                             { grp[j] = 2; key[j] = p[b * n + j] + I->lag[s * n + j]; }
        }
        jkeys K = { grp, key };
        j_sort(&K, I->johnson + s * n, 0, n - 1);
    }
    return I;
}

void orc_destroy(orc_inst *I)
{
    if (!I) return;
    free(I->p); free(I->min_arr); free(I->min_dep); free(I->mach0); free(I->mach1);
    free(I->lag); free(I->johnson); free(I);
}

void orc_johnson_row(const orc_inst *I, int s, int *out) { memcpy(out, I->johnson + s * I->n, sizeof(int) * I->n); }
void orc_lag_row(const orc_inst *I, int s, int *out) { memcpy(out, I->lag + s * I->n, sizeof(int) * I->n); }
void orc_min_times(const orc_inst *I, int *arr, int *dep)
{
    memcpy(arr, I->min_arr, sizeof(int) * I->m);
    memcpy(dep, I->min_dep, sizeof(int) * I->m);
}

/* ------------------------------------------------------------------------ */
/* weak (one-machine) bound                                                  */
/* ------------------------------------------------------------------------ */

/* makespan of a full permutation (bound_fsp_weak.cpp:224-244) */
int orc_eval(const orc_inst *I, const int *perm)
{
    int c[ORC_MAXM] = {0};
    int n = I->n, m = I->m;
    for (int i = 0; i < n; i++) {
        int j = perm[i];
        c[0] += I->p[j];
        for (int k = 1; k < m; k++) c[k] = imax(c[k - 1], c[k]) + I->p[k * n + j];
    }
    return c[m - 1];
}

/* heads of the jobs fixed in front, tails of the jobs fixed at the back and
 * machine loads of the free jobs (bound_fsp_weak.cpp:62-122) */
static void weak_partial(const orc_inst *I, const int *s, int l1, int l2, int *front, int *back, int *remain)
{
    int n = I->n, m = I->m;
    if (l1 == -1) {
        for (int k = 0; k < m; k++) front[k] = I->min_arr[k];
    } else {
        for (int k = 0; k < m; k++) front[k] = 0;
        for (int i = 0; i <= l1; i++) {
            int j = s[i];
            front[0] += I->p[j];
            for (int k = 1; k < m; k++) front[k] = imax(front[k - 1], front[k]) + I->p[k * n + j];
        }
    }
    if (l2 == n) {
        for (int k = 0; k < m; k++) back[k] = I->min_dep[k];
    } else {
        for (int k = 0; k < m; k++) back[k] = 0;
        for (int i = n - 1; i >= l2; i--) {
            int j = s[i];
            back[m - 1] += I->p[(m - 1) * n + j];
            for (int k = m - 2; k >= 0; k--) back[k] = imax(back[k], back[k + 1]) + I->p[k * n + j];
        }
    }
    for (int k = 0; k < m; k++) remain[k] = 0;
    for (int i = l1 + 1; i < l2; i++)
        for (int k = 0; k < m; k++) remain[k] += I->p[k * n + s[i]];
}

/* node LB (bound_fsp_weak.cpp:289-311, `bornes_calculer`) */
int orc_weak_node(const orc_inst *I, const int *s, int l1, int l2)
{
    int front[ORC_MAXM], back[ORC_MAXM], remain[ORC_MAXM];
    weak_partial(I, s, l1, l2, front, back, remain);
    int t0 = front[0] + remain[0];
    int lb = t0 + back[0];
    for (int k = 1; k < I->m; k++) {
        int t1 = imax(front[k] + remain[k], t0);
        lb = imax(lb, t1 + back[k]);
        t0 = t1;
    }
    return lb;
}

/* LB of child `j` appended at the front / prepended at the back, with the
 * idle-time priority (bound_fsp_weak.cpp:134-191) */
static int weak_add_front(const orc_inst *I, const int *front, const int *back, const int *remain, int j, int *prio)
{
    int n = I->n, m = I->m;
    int t0 = front[0] + I->p[j];
    int lb = front[0] + remain[0] + back[0];
    int pr = 0;
    for (int k = 1; k < m; k++) {
        int d = t0 - front[k];
        pr += d < 0 ? -d : d;
        int t1 = imax(front[k], t0);
        lb = imax(lb, t1 + remain[k] + back[k]);
        t0 = t1 + I->p[k * n + j];
    }
    *prio = pr;
    return lb;
}

static int weak_add_back(const orc_inst *I, const int *front, const int *back, const int *remain, int j, int *prio)
{
    int n = I->n, m = I->m;
    int t0 = back[m - 1] + I->p[(m - 1) * n + j];
    int lb = front[m - 1] + remain[m - 1] + back[m - 1];
    int pr = 0;
    for (int k = m - 2; k >= 0; k--) {
        int d = t0 - back[k];
        pr += d < 0 ? -d : d;
        int t1 = imax(t0, back[k]);
        lb = imax(lb, front[k] + remain[k] + t1);
        t0 = t1 + I->p[k * n + j];
    }
    *prio = pr;
    return lb;
}

/* children LBs indexed by job id, 0 for fixed jobs (bound_fsp_weak.cpp:194-221).
 * both_ends != 0 is branchingMode > 0; otherwise only cb is written. */
void orc_weak_children(const orc_inst *I, const int *s, int l1, int l2, int both_ends,
                       int *cb, int *ce, int *pb, int *pe)
{
    int front[ORC_MAXM], back[ORC_MAXM], remain[ORC_MAXM];
    memset(cb, 0, sizeof(int) * I->n);
    if (both_ends) memset(ce, 0, sizeof(int) * I->n);
    weak_partial(I, s, l1, l2, front, back, remain);
    for (int i = l1 + 1; i < l2; i++) {
        int j = s[i];
        cb[j] = weak_add_front(I, front, back, remain, j, &pb[j]);
        if (both_ends) ce[j] = weak_add_back(I, front, back, remain, j, &pe[j]);
    }
}

/* ------------------------------------------------------------------------ */
/* strong (Johnson two-machine) bound                                        */
/* ------------------------------------------------------------------------ */

/* bound_fsp_strong.cpp:541-560 with best = -1 (no early exit), which calls
 * setFlags :481-486, scheduleFront :457-478, scheduleBack :490-509 and
 * borneInfMakespan :103-162 -> initCmax :52-62, heuristiqueCmax :76-100,
 * cmaxFin :66-72.  For at most one free job the exact makespan is returned. */
int orc_strong_node(const orc_inst *I, const int *s, int l1, int l2)
{
    int n = I->n, m = I->m;
    if (l2 - l1 <= 2) return orc_eval(I, s);
    unsigned char fixed[ORC_MAXN];
    memset(fixed, 0, (size_t)n);
    for (int i = 0; i <= l1; i++) fixed[s[i]] = 1;
    for (int i = l2; i < n; i++) fixed[s[i]] = 1;
    int front[ORC_MAXM], back[ORC_MAXM];
    if (l1 == -1) {
        for (int k = 0; k < m; k++) front[k] = I->min_arr[k];
    } else {
        for (int k = 0; k < m; k++) front[k] = 0;
        for (int i = 0; i <= l1; i++) {
            int j = s[i];
            front[0] += I->p[j];
            for (int k = 1; k < m; k++) front[k] = imax(front[k], front[k - 1]) + I->p[k * n + j];
        }
    }
    if (l2 == n) {
        for (int k = 0; k < m; k++) back[k] = I->min_dep[k];
    } else {
        for (int k = 0; k < m; k++) back[k] = 0;
        for (int i = n - 1; i >= l2; i--) {
            int j = s[i];
            back[m - 1] += I->p[(m - 1) * n + j];
            for (int k = m - 2; k >= 0; k--) back[k] = imax(back[k], back[k + 1]) + I->p[k * n + j];
        }
    }
    int lb = 0;
    for (int q = 0; q < I->P; q++) {
        int a = I->mach0[q], b = I->mach1[q];
        if (I->pair_mode == 1 && b < m - 1) continue;
        if (I->pair_mode == 2 && b != a + 1) continue;
        int t0 = front[a], t1 = front[b];
        const int *ord = I->johnson + q * n;
        const int *lg = I->lag + q * n;
        for (int t = 0; t < n; t++) {
            int j = ord[t];
            if (fixed[j]) continue;
            t0 += I->p[a * n + j];
            t1 = imax(t1, t0 + lg[j]) + I->p[b * n + j];
        }
        int fin = imax(t1 + back[b], t0 + back[a]);
        if (fin > lb) lb = fin;
    }
    return lb;
}

/* ------------------------------------------------------------------------ */
/* sequential IVM branch-and-bound                                           */
/* ------------------------------------------------------------------------ */

typedef struct {
    int bound_mode;    /* [bb] boundingMode: 0 weak, 1 strong, 2 weak then strong */
    int branch_mode;   /* [bb] adaptiveBranchingMode: -3,-2,-1,1,2,3 (CPU numbering) */
    int find_all;      /* [bb] findAll */
    int sort_nodes;    /* [bb] sortedDFS: 0 row reversal; 1 sort by the first cost; 2, 4 by (first
                          cost, priority); 3 by priority (ivm_bound.cpp:338-370) */
    int64_t node_limit;/* stop after this many decomposed nodes (<=0: none) */
    int sort_crit;     /* [bb] sortingCriterion: priority of siblings, 1 chosen side's cost,
                          2 its difference with the other side's, 3 idle time (:506-544) */
} orc_cfg;

typedef struct {
    int64_t decomposed, johnson_bounds, simple_bounds, leaves;
    int best;          /* best cost known at the end (initial UB if not improved) */
    int found;         /* a leaf improved (or, with findAll, matched) the UB */
    int complete;      /* the whole interval was explored */
} orc_result;

typedef struct {
    const orc_inst *I;
    orc_cfg cfg;
    int n;
    int *mat;          /* [n][n] jobs; pruned/visited cells hold -j-1 (common/include/misc.h:20-29) */
    int pos[ORC_MAXN], end[ORC_MAXN], dir[ORC_MAXN];
    int line;
    int sched[ORC_MAXN];
    int l1, l2;
    int best;
    int *best_perm;
    /* per-node cost tables indexed by job (ivm_bound.cpp:27-31) */
    int cb_w[ORC_MAXN], ce_w[ORC_MAXN], cb_s[ORC_MAXN], ce_s[ORC_MAXN];
    int pb_w[ORC_MAXN], pe_w[ORC_MAXN];   /* weak idle-time priorities (priorityBegin/End) */
    int prio[ORC_MAXN];                   /* sibling priorities set by chooseChildrenSet */
    orc_result res;
} orc_bb;

static int flag_neg(int v) { return v < 0 ? v : -v - 1; }    /* misc.h negative() */
static int flag_abs(int v) { return v >= 0 ? v : -v - 1; }   /* misc.h absolute() */

static int gt_best(const orc_bb *B, int v)                    /* ivm_bound.cpp:678-682 */
{
    return B->cfg.find_all ? v > B->best : v >= B->best;
}

/* ivm.cpp:153-162 */
static int before_end(const orc_bb *B)
{
    for (int i = 0; i < B->n; i++) {
        if (B->pos[i] < B->end[i]) return 1;
        if (B->pos[i] > B->end[i]) return 0;
    }
    return 1;
}

/* ivm.cpp:116-133: row `l` is row l-1 without the cell at pos[l-1], flags removed */
static void generate_line(orc_bb *B, int l, int explore)
{
    int n = B->n, c = B->pos[l - 1];
    int *dst = B->mat + l * n, *src = B->mat + (l - 1) * n;
    for (int i = 0; i < c; i++) dst[i] = flag_abs(src[i]);
    for (int i = c; i < n - l; i++) dst[i] = flag_abs(src[i + 1]);
    if (explore) { B->pos[l] = 0; B->dir[l] = 0; }
}

/* ivm_bound.cpp:112-138 */
static void prepare_schedule(orc_bb *B)
{
    int n = B->n;
    B->l1 = -1; B->l2 = n;
    for (int l = 0; l < B->line; l++) {
        int j = flag_abs(B->mat[l * n + B->pos[l]]);
        if (B->dir[l] == 0) B->sched[++B->l1] = j; else B->sched[--B->l2] = j;
    }
    for (int l = 0; l < n - B->line; l++) B->sched[B->l1 + 1 + l] = flag_abs(B->mat[B->line * n + l]);
}

static void weak_bounds(orc_bb *B)                              /* ivm_bound.cpp:216-236 */
{
    memset(B->cb_s, 0, sizeof(int) * B->n);
    memset(B->ce_s, 0, sizeof(int) * B->n);
    int both = B->cfg.branch_mode > 0;
    orc_weak_children(B->I, B->sched, B->l1, B->l2, both, B->cb_w, B->ce_w, B->pb_w, B->pe_w);
    B->res.simple_bounds += both ? 2 * (B->l2 - B->l1 - 1) : (B->l2 - B->l1 - 1);
}

/* ivm_bound.cpp:141-195 with the Johnson call restored (P4) */
static void strong_bounds(orc_bb *B, int front_side)
{
    int n = B->n;
    int L1 = B->l1 + (front_side ? 1 : 0);
    int L2 = B->l2 - (front_side ? 0 : 1);
    int *first = front_side ? B->cb_s : B->ce_s;
    int *second = front_side ? B->cb_w : B->ce_w;
    int fill = front_side ? L1 : L2;
    memset(first, 0, sizeof(int) * n);
    for (int i = B->l1 + 1; i < B->l2; i++) {
        int j = B->sched[i];
        if (gt_best(B, second[j])) continue;
        int t = B->sched[fill]; B->sched[fill] = B->sched[i]; B->sched[i] = t;
        first[j] = orc_strong_node(B->I, B->sched, L1, L2);
        t = B->sched[fill]; B->sched[fill] = B->sched[i]; B->sched[i] = t;
        B->res.johnson_bounds++;
    }
}

/* ivm_bound.cpp:413-504 (CPU rule numbering); 0 = FRONT, 1 = BACK.  The
 * multicore B&B forces singleNode (multicore/src/main.cpp:21), so MinBranch
 * and MinMin count pruned children against the incumbent (:458-459). */
static int choose_side(const orc_bb *B, const int *cb, const int *ce)
{
    int n = B->n, ub = B->best;
    switch (B->cfg.branch_mode) {
    case -3: return (B->line % 2) ? 1 : 0;
    case -2: return 1;
    case -1: return 0;
    case 1: {
        int sum = 0;
        for (int i = 0; i < n; i++) sum += cb[i] - ce[i];
        return sum < 0 ? 1 : 0;
    }
    case 2: {
        int elim = 0, sum = 0;
        for (int i = 0; i < n; i++) {
            if (cb[i] >= ub) elim++; else sum += cb[i];
            if (ce[i] >= ub) elim--; else sum -= ce[i];
        }
        if (elim > 0) return 0;
        if (elim < 0) return 1;
        return sum < 0 ? 1 : 0;
    }
    case 3:
    default: {
        int mn = INT_MAX, cnt = 0, elim = 0;
        for (int i = 0; i < n; i++) {
            if (cb[i] < mn && cb[i] > 0) mn = cb[i];
            if (ce[i] < mn && ce[i] > 0) mn = ce[i];
        }
        for (int i = 0; i < n; i++) {
            if (cb[i] == mn) cnt++;
            if (ce[i] == mn) cnt--;
            if (cb[i] >= ub) elim++;
            if (ce[i] >= ub) elim--;
        }
        if (cnt > 0) return 1;
        if (cnt < 0) return 0;
        return elim > 0 ? 0 : 1;
    }
    }
}

/* chooseChildrenSet (ivm_bound.cpp:413-560): the side, then the siblings'
 * priorities for sortedDFS 2-4 (:506-544).  Priority 3 reads the weak
 * bound's idle times (priorityBegin/End); criteria 4 and the strong bound's
 * idle times are rejected by the engine and never reach here. */
static int choose_dir(orc_bb *B, const int *cb, const int *ce)
{
    int n = B->n;
    int side = choose_side(B, cb, ce);
    for (int i = 0; i < n; i++) {
        int mine = side ? ce[i] : cb[i], other = side ? cb[i] : ce[i];
        if (B->cfg.sort_crit == 1) B->prio[i] = mine;
        else if (B->cfg.sort_crit == 2) B->prio[i] = mine - other;
        else if (B->cfg.sort_crit == 3) B->prio[i] = mine > 0 ? (side ? B->pe_w[i] : B->pb_w[i]) : 99999;
    }
    return side;
}

/* misc.h:33-48 gnomeSortByKeyInc: stable, swaps neighbours while the left key
 * is strictly larger */
static void gnome_sort_by_key(int *arr, const int *key, int from, int to)
{
    int i = from + 1, j = i + 1;
    while (i <= to) {
        if (key[arr[i - 1]] > key[arr[i]]) {
            int t = arr[i - 1]; arr[i - 1] = arr[i]; arr[i] = t;
            if (--i) continue;
        }
        i = j++;
    }
}

/* misc.h:50-65 gnomeSortByKeysInc: the same, with key2 breaking ties of key1 */
static void gnome_sort_by_keys(int *arr, const int *key1, const int *key2, int from, int to)
{
    int i = from + 1, j = i + 1;
    while (i <= to) {
        if (key1[arr[i - 1]] > key1[arr[i]] ||
            (key1[arr[i - 1]] == key1[arr[i]] && key2[arr[i - 1]] > key2[arr[i]])) {
            int t = arr[i - 1]; arr[i - 1] = arr[i]; arr[i] = t;
            if (--i) continue;
        }
        i = j++;
    }
}

/* ivm_bound.cpp:611-646 -> eliminateJobs :338-410.  sortedDFS = 0 reverses the
 * row when the side changes; sortedDFS = 1 sorts it by the chosen side's first
 * cost instead (:344-349), 2 and 4 by that cost then the priority (:350-354,
 * :360-364), 3 by the priority (:355-359). */
static void prune(orc_bb *B, const int *c1b, const int *c1e, const int *c2b, const int *c2e)
{
    int n = B->n, l = B->line;
    int *row = B->mat + l * n;
    int prev = l > 0 ? B->dir[l - 1] : 0;
    if (B->cfg.sort_nodes == 0 && prev != B->dir[l]) {
        for (int a = 0, b = n - l - 1; a < b; a++, b--) { int t = row[a]; row[a] = row[b]; row[b] = t; }
    }
    const int *c1 = B->dir[l] == 1 ? c1e : c1b;
    const int *c2 = B->dir[l] == 1 ? c2e : c2b;
    if (B->cfg.sort_nodes == 1) gnome_sort_by_key(row, c1, 0, n - l - 1);
    else if (B->cfg.sort_nodes == 2 || B->cfg.sort_nodes == 4) gnome_sort_by_keys(row, c1, B->prio, 0, n - l - 1);
    else if (B->cfg.sort_nodes == 3) gnome_sort_by_key(row, B->prio, 0, n - l - 1);
    for (int i = 0; i < n - l; i++) {
        int j = row[i];
        if (gt_best(B, c1[j]) || gt_best(B, c2[j])) row[i] = flag_neg(j);
    }
}

static void bound_and_prune(orc_bb *B, int mode)
{
    switch (mode) {
    case 0:                                         /* weakBoundPrune :650-658 */
        weak_bounds(B);
        B->dir[B->line] = choose_dir(B, B->cb_w, B->ce_w);
        prune(B, B->cb_w, B->ce_w, B->cb_w, B->ce_w);
        break;
    case 1:                                         /* strongBoundPrune :669-676 */
        for (int i = 0; i < B->n; i++) { B->cb_w[i] = -1; B->ce_w[i] = -1; }
        strong_bounds(B, 1);
        strong_bounds(B, 0);
        B->dir[B->line] = choose_dir(B, B->cb_s, B->ce_s);
        prune(B, B->cb_s, B->ce_s, B->cb_s, B->ce_s);
        break;
    case 2:                                         /* mixedBoundPrune :661-666 */
    default:
        weak_bounds(B);
        B->dir[B->line] = choose_dir(B, B->cb_w, B->ce_w);
        strong_bounds(B, B->dir[B->line] == 0);
        prune(B, B->cb_w, B->ce_w, B->cb_s, B->ce_s);
        break;
    }
}

/* ivm_bound.cpp:239-271 */
static void bound_leaf(orc_bb *B)
{
    int n = B->n;
    B->res.leaves++;
    int c = orc_eval(B->I, B->sched);
    if (!gt_best(B, c)) {
        if (c < B->best || !B->res.found) memcpy(B->best_perm, B->sched, sizeof(int) * n);
        B->best = c;
        B->res.found = 1;
    }
    int *cell = B->mat + B->line * n + B->pos[B->line];
    *cell = flag_neg(*cell);
}

/* sequentialbb.cpp:207-264 (uncounted descent along the interval's start) */
static void unfold(orc_bb *B)
{
    int n = B->n;
    while (B->line < n - 2) {
        if (B->mat[B->line * n + B->pos[B->line]] < 0) {
            for (int i = B->line + 1; i < n; i++) B->pos[i] = 0;
            break;
        }
        B->line++;
        generate_line(B, B->line, 0);
        prepare_schedule(B);
        bound_and_prune(B, B->cfg.bound_mode);
    }
}

/* sequentialbb.cpp:110-190; returns 1 when a node was bounded */
static int bb_next(orc_bb *B)
{
    int n = B->n;
    while (before_end(B)) {
        int l = B->line;
        if (B->pos[l] >= n - l) {                             /* goUp ivm.cpp:56-72 */
            if (l > 0) {
                B->pos[l] = 0;
                B->line--;
                int *cell = B->mat + B->line * n + B->pos[B->line];
                *cell = flag_neg(*cell);
            } else {
                B->pos[0]++;
            }
            continue;
        }
        if (B->mat[l * n + B->pos[l]] < 0) { B->pos[l]++; continue; }   /* goRight */
        B->res.decomposed++;
        B->line++;                                          /* goDown ivm.cpp:73-104 */
        generate_line(B, B->line, 1);
        prepare_schedule(B);
        if (B->line == n - 1) { bound_leaf(B); continue; }
        bound_and_prune(B, B->cfg.bound_mode);
        return 1;
    }
    return 0;
}

/* Solve the interval [pos, end] (NULL = the whole space) from the root row
 * `root`: sequentialbb::setRoot :28-46 -> boundRoot (weak, uncounted), then
 * initAtInterval :84-106 (stats reset, unfold :207-264), then next() until
 * the interval is exhausted or node_limit. */
int orc_solve_interval(const orc_inst *I, const orc_cfg *cfg, int ub, const int *root, const int *pos,
                       const int *end, orc_result *out, int *best_perm)
{
    int n = I->n;
    orc_bb B;
    memset(&B, 0, sizeof(B));
    B.I = I; B.cfg = *cfg; B.n = n; B.best = ub; B.best_perm = best_perm;
    B.mat = (int *)calloc((size_t)n * n, sizeof(int));
    if (!B.mat) return -1;
    for (int i = 0; i < n; i++) B.mat[i] = root[i];
    B.line = 0;
    prepare_schedule(&B);
    /* boundRoot: always the weak bound (ivm_bound.cpp:274-336) */
    weak_bounds(&B);
    B.dir[0] = choose_dir(&B, B.cb_w, B.ce_w);
    prune(&B, B.cb_w, B.ce_w, B.cb_w, B.ce_w);
    memset(&B.res, 0, sizeof(B.res));                     /* initAtInterval resets the stats */
    for (int i = 0; i < n; i++) {
        B.pos[i] = pos ? pos[i] : 0;
        B.end[i] = end ? end[i] : n - i - 1;
        if (B.pos[i] < 0 || B.pos[i] >= n - i || B.end[i] < 0 || B.end[i] >= n - i) { free(B.mat); return -2; }
    }
    if (before_end(&B)) unfold(&B);
    int complete = 1;
    while (bb_next(&B)) {
        if (cfg->node_limit > 0 && B.res.decomposed >= cfg->node_limit) { complete = !before_end(&B); break; }
    }
    B.res.best = B.best;
    B.res.complete = complete;
    *out = B.res;
    free(B.mat);
    return 0;
}

int orc_solve(const orc_inst *I, const orc_cfg *cfg, int ub, const int *root, orc_result *out, int *best_perm)
{
    return orc_solve_interval(I, cfg, ub, root, NULL, NULL, out, best_perm);
}

/* ------------------------------------------------------------------------ */
/* NEH initial upper bound                                                   */
/* ------------------------------------------------------------------------ */

/* NEH: jobs by decreasing total processing time (ties: lower id first); the
 * first pair keeps the swapped order unless the original is strictly better
 * (heuristic/src/fastNEH.cpp:230-243); every further job goes to the first
 * position of minimum partial makespan (findBestPos :151-178).  Partial
 * makespans are evaluated directly, O(n^3 m). */
static int partial_makespan(const orc_inst *I, const int *seq, int len)
{
    int c[ORC_MAXM] = {0};
    int n = I->n, m = I->m;
    for (int i = 0; i < len; i++) {
        int j = seq[i];
        c[0] += I->p[j];
        for (int k = 1; k < m; k++) c[k] = imax(c[k - 1], c[k]) + I->p[k * n + j];
    }
    return c[m - 1];
}

int orc_neh(const orc_inst *I, int *perm)
{
    int n = I->n, m = I->m;
    int tot[ORC_MAXN], order[ORC_MAXN], seq[ORC_MAXN], trial[ORC_MAXN];
    for (int j = 0; j < n; j++) {
        tot[j] = 0;
        for (int k = 0; k < m; k++) tot[j] += I->p[k * n + j];
        order[j] = j;
    }
    for (int a = 1; a < n; a++) {             /* stable insertion sort, decreasing total */
        int v = order[a], b = a - 1;
        while (b >= 0 && tot[order[b]] < tot[v]) { order[b + 1] = order[b]; b--; }
        order[b + 1] = v;
    }
    if (n == 1) { perm[0] = order[0]; return partial_makespan(I, perm, 1); }
    seq[0] = order[0]; seq[1] = order[1];
    int c1 = partial_makespan(I, seq, 2);
    seq[0] = order[1]; seq[1] = order[0];
    int c2 = partial_makespan(I, seq, 2);
    if (c1 < c2) { seq[0] = order[0]; seq[1] = order[1]; }
    for (int k = 2; k < n; k++) {
        int job = order[k], best = INT_MAX, bpos = 0;
        for (int q = 0; q <= k; q++) {
            for (int i = 0, t = 0; i <= k; i++) trial[i] = (i == q) ? job : seq[t++];
            int c = partial_makespan(I, trial, k + 1);
            if (c < best) { best = c; bpos = q; }
        }
        for (int i = k; i > bpos; i--) seq[i] = seq[i - 1];
        seq[bpos] = job;
    }
    memcpy(perm, seq, sizeof(int) * n);
    return partial_makespan(I, perm, n);
}

/* ------------------------------------------------------------------------ */
/* Iterated greedy, the checker of the device IG                             */
/* ------------------------------------------------------------------------ */

/* The reference's IG (heuristic/src/IG.cpp:341-416) draws its decisions from
 * std::random_device, so no run of it can be reproduced.  The engine's IG
 * follows the same steps with a seeded splitmix64 stream; this is a plain
 * restatement of that definition, evaluating every candidate by a direct
 * makespan, used to check the device kernel draw for draw:
 *   start: NEH (orc_neh);
 *   round: d = perturbation (2, growing to 5 after rejections, :393-396)
 *     destruction (:120-160): r uniform in [d, n], the first r entries of the
 *       middle-out visit order (:33-45) shuffled (Fisher-Yates, j uniform in
 *       [i, r-1]), the jobs at the first d shuffled positions removed in draw
 *       order, the rest compacted;
 *     construction (:229-255): each removed job at the first position of least
 *       makespan;
 *     local search (localSearchKI :567-612): passes over the visit order; the
 *       job at position i goes to the first best place within isqrt(n) of i;
 *       a strict improvement is kept and starts a new pass; at most
 *       `ls_passes` passes;
 *     acceptance (:258-274): one draw u (the high 32 bits of the next value);
 *       kept when not worse, or when u < 2^32 T / (T + 1000 delta) with
 *       T = 20 x total time / (n m), i.e. 1000 x 0.2 x mean time / 10. */
static uint64_t ig_next(uint64_t *s)
{
    *s += 0x9E3779B97F4A7C15ull;
    uint64_t z = *s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static int ig_range(uint64_t *s, int a, int b)
{
    return a + (int)(((unsigned __int128)ig_next(s) * (uint64_t)(b - a + 1)) >> 64);
}

/* first position in [lo, hi] of least makespan for x inserted into seq[0..len) */
static int ig_best_pos(const orc_inst *I, const int *seq, int len, int x, int lo, int hi, int *cost)
{
    int trial[ORC_MAXN], best = INT_MAX, bpos = lo;
    for (int q = lo; q <= hi; q++) {
        for (int i = 0, t = 0; i <= len; i++) trial[i] = (i == q) ? x : seq[t++];
        int c = partial_makespan(I, trial, len + 1);
        if (c < best) { best = c; bpos = q; }
    }
    *cost = best;
    return bpos;
}

static void ig_insert(int *seq, int len, int pos, int x)
{
    for (int i = len; i > pos; i--) seq[i] = seq[i - 1];
    seq[pos] = x;
}

int orc_ig(const orc_inst *I, int iterations, int destruct, int destruct_max, int ls_passes, uint64_t seed,
           int *perm)
{
    int n = I->n, m = I->m;
    int cur[ORC_MAXN], best[ORC_MAXN], seq[ORC_MAXN], vo[ORC_MAXN], order[ORC_MAXN], removed[ORC_MAXN];
    int cur_cost = orc_neh(I, cur);
    int best_cost = cur_cost;
    memcpy(best, cur, sizeof(int) * n);
    long long sum = 0;
    for (int i = 0; i < n * m; i++) sum += I->p[i];
    long long temp1000 = 20 * sum / ((long long)n * m);
    int start = n / 2, ind = 0;
    for (int i = start; i < n; i++) { vo[ind] = i; ind += 2; }
    ind = 1;
    for (int i = start - 1; i >= 0; i--) { vo[ind] = i; ind += 2; }
    int kmax = 1;
    while ((kmax + 1) * (kmax + 1) <= n) kmax++;
    uint64_t rs = seed;
    int perturb = destruct;
    for (int it = 0; it < iterations && n >= 3; it++) {
        int d = perturb < n - 1 ? perturb : n - 1;
        memcpy(seq, cur, sizeof(int) * n);
        int r = ig_range(&rs, d, n);
        for (int i = 0; i < r; i++) order[i] = vo[i];
        for (int i = 0; i < r - 1; i++) {
            int j = ig_range(&rs, i, r - 1);
            int t = order[i]; order[i] = order[j]; order[j] = t;
        }
        unsigned char gone[ORC_MAXN];
        memset(gone, 0, sizeof(gone));
        for (int i = 0; i < d; i++) { removed[i] = seq[order[i]]; gone[order[i]] = 1; }
        int w = 0;
        for (int i = 0; i < n; i++) if (!gone[i]) seq[w++] = seq[i];
        int len = n - d, c;
        for (int i = 0; i < d; i++) {
            int pos = ig_best_pos(I, seq, len, removed[i], 0, len, &c);
            ig_insert(seq, len, pos, removed[i]);
            len++;
        }
        int cost = partial_makespan(I, seq, n);
        for (int pass = 0; pass < ls_passes; pass++) {
            int improved = 0;
            for (int j = 0; j < n && !improved; j++) {
                int i = vo[j], x = seq[i];
                for (int q = i; q < n - 1; q++) seq[q] = seq[q + 1];
                int lo = i - kmax > 0 ? i - kmax : 0, hi = i + kmax < n - 1 ? i + kmax : n - 1;
                int pos = ig_best_pos(I, seq, n - 1, x, lo, hi, &c);
                if (c < cost) { ig_insert(seq, n - 1, pos, x); cost = c; improved = 1; }
                else ig_insert(seq, n - 1, i, x);
            }
            if (!improved) break;
        }
        long long delta = (long long)cost - cur_cost;
        uint64_t u = ig_next(&rs) >> 32;
        int accept = delta <= 0 || u < ((uint64_t)temp1000 << 32) / (uint64_t)(temp1000 + 1000 * delta);
        if (accept) {
            memcpy(cur, seq, sizeof(int) * n);
            cur_cost = cost;
            perturb = destruct;
        } else {
            perturb = perturb + 1 > destruct_max ? destruct : perturb + 1;
        }
        if (cost < best_cost) { best_cost = cost; memcpy(best, seq, sizeof(int) * n); }
    }
    memcpy(perm, best, sizeof(int) * n);
    return best_cost;
}

/* couts[1] of bound_fsp_strong::bornes_calculer (bound_fsp_strong.cpp:541-560):
 * the idle time of the front jobs' schedule (scheduleFront :457-478; 0 when
 * nothing is fixed in front) plus that of the back jobs' (scheduleBack
 * :490-509), all reset to 0 when nothing is fixed at the back; 0 with at most
 * one free job, where the reference leaves the value as it was. */
int orc_strong_idle(const orc_inst *I, const int *s, int l1, int l2)
{
    int n = I->n, m = I->m;
    if (l2 - l1 <= 2 || l2 == n) return 0;
    int fr[ORC_MAXM], bk[ORC_MAXM], idle = 0;
    for (int k = 0; k < m; k++) { fr[k] = 0; bk[k] = 0; }
    for (int i = 0; i <= l1; i++) {
        int j = s[i];
        fr[0] += I->p[j];
        for (int k = 1; k < m; k++) {
            idle += imax(0, fr[k - 1] - fr[k]);
            fr[k] = imax(fr[k], fr[k - 1]) + I->p[k * n + j];
        }
    }
    for (int i = n - 1; i >= l2; i--) {
        int j = s[i];
        bk[m - 1] += I->p[(m - 1) * n + j];
        for (int k = m - 2; k >= 0; k--) {
            idle += imax(0, bk[k + 1] - bk[k]);
            bk[k] = imax(bk[k], bk[k + 1]) + I->p[k * n + j];
        }
    }
    return idle;
}
