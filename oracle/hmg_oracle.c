/*
 * hmg_oracle.c -- CPU restatement of the kadircs/hmglib H-matrix hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product; see hmg_oracle.h).
 * Built with -ffp-contract=off so that the only fused multiply-adds are the
 * explicit fma() calls, which mirror the contractions nvcc makes in the
 * reference's device code (nvcc's default is --fmad=true).
 */
#include "hmg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------- */
/* Morton codes                                                               */
/* ------------------------------------------------------------------------- */

/* helper.cu:108-138 -- thrust::minmax_element per dimension (exact). */
void orc_minmax(const double* coords, int n, int dim, double* mn, double* mx)
{
    for (int d = 0; d < dim; d++) {
        const double* c = coords + (size_t)d * n;
        double lo = c[0], hi = c[0];
        for (int i = 1; i < n; i++) {
            if (c[i] < lo) lo = c[i];
            if (c[i] > hi) hi = c[i];
        }
        mn[d] = lo;
        mx[d] = hi;
    }
}

/* morton.cu:71-75 (coord_to_fp).  A NaN quotient (a dimension with max == min)
 * converts to the largest fixed-point value, as the device conversion of the
 * reference's `(uint64_t)floor(NaN)` does on sm_100 (observed on a B200). */
static uint64_t coord_to_fixed(double c, double lo, double range, int bits)
{
    double t = (c - lo) / range;
    double f = floor(t * (double)(1ull << bits));
    uint64_t q;
    if (f != f)
        q = ~0ull;
    else if (f <= 0.0)
        q = 0;
    else if (f >= 18446744073709551616.0)
        q = ~0ull;
    else
        q = (uint64_t)f;
    uint64_t cap = (1ull << bits) - 1;
    return q < cap ? q : cap;
}

/* morton.cu:21-67 (stretch) restated as the plain definition of bit interleaving:
 * bit b of the fixed-point coordinate of dimension d lands on bit b*dim+d.  The
 * reference only supports (dim,bits) in {(2,32),(3,20),(10,4)} and yields 0
 * otherwise; the same restriction is applied here. */
static int morton_supported(int dim, int bits)
{
    return (dim == 2 && bits == 32) || (dim == 3 && bits == 20) || (dim == 10 && bits == 4);
}

void orc_morton(const double* coords, int n, int dim, int bits, const double* mn,
                const double* mx, uint64_t* codes)
{
    int ok = morton_supported(dim, bits);
    for (int i = 0; i < n; i++) {
        uint64_t code = 0;
        if (ok) {
            for (int d = 0; d < dim; d++) {
                uint64_t q = coord_to_fixed(coords[(size_t)d * n + i], mn[d], mx[d] - mn[d], bits);
                for (int b = 0; b < bits; b++)
                    code |= ((q >> b) & 1ull) << (b * dim + d);
            }
        }
        codes[i] = code;
    }
}

/* helper.cu:140-167 -- stable sort of (code, index): LSD radix sort, 8-bit digits. */
void orc_sort(const uint64_t* codes, int n, uint64_t* sorted, int64_t* order)
{
    uint64_t* k0 = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(n > 0 ? n : 1));
    uint64_t* k1 = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(n > 0 ? n : 1));
    int64_t* v0 = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    int64_t* v1 = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; i++) {
        k0[i] = codes[i];
        v0[i] = i;
    }
    for (int pass = 0; pass < 8; pass++) {
        int shift = pass * 8;
        size_t cnt[257];
        memset(cnt, 0, sizeof(cnt));
        for (int i = 0; i < n; i++) cnt[((k0[i] >> shift) & 255u) + 1]++;
        for (int b = 0; b < 256; b++) cnt[b + 1] += cnt[b];
        for (int i = 0; i < n; i++) {
            size_t p = cnt[(k0[i] >> shift) & 255u]++;
            k1[p] = k0[i];
            v1[p] = v0[i];
        }
        uint64_t* tk = k0; k0 = k1; k1 = tk;
        int64_t* tv = v0; v0 = v1; v1 = tv;
    }
    for (int i = 0; i < n; i++) {
        sorted[i] = k0[i];
        order[i] = v0[i];
    }
    free(k0); free(k1); free(v0); free(v1);
}

/* helper.cu:69-78,293-328 -- out[d][i] = coords[d][order[i]] */
void orc_reorder(const double* coords, int n, int dim, const int64_t* order, double* out)
{
    for (int d = 0; d < dim; d++)
        for (int i = 0; i < n; i++)
            out[(size_t)d * n + i] = coords[(size_t)d * n + order[i]];
}

/* ------------------------------------------------------------------------- */
/* Block-cluster tree                                                         */
/* ------------------------------------------------------------------------- */

static int clz64(uint64_t x) { return x ? __builtin_clzll(x) : 64; }

/* tree.cu:40-78 (findSplit): the last index s in [first,last) whose code shares more
 * than the common prefix of codes[first] and codes[last] with codes[first]; the
 * midpoint when the two end codes are equal.  Restated as a linear scan. */
static int split_index(const uint64_t* codes, int first, int last)
{
    uint64_t a = codes[first], b = codes[last];
    if (a == b) return (first + last) >> 1;
    int common = clz64(a ^ b);
    int s = first;
    for (int t = first + 1; t < last; t++) {
        if (clz64(a ^ codes[t]) > common)
            s = t;
        else
            break;
    }
    return s;
}

typedef struct {
    int l1, u1, l2, u2;
    int lev1, lev2;
} orc_node;

struct orc_blocks {
    int count, cap, levels;
    int *s1l, *s1u, *s2l, *s2u, *type, *lev1, *lev2;
};

static void blocks_push(orc_blocks* b, const orc_node* nd, int type)
{
    if (b->count == b->cap) {
        b->cap = b->cap ? 2 * b->cap : 1024;
        b->s1l = (int*)realloc(b->s1l, sizeof(int) * b->cap);
        b->s1u = (int*)realloc(b->s1u, sizeof(int) * b->cap);
        b->s2l = (int*)realloc(b->s2l, sizeof(int) * b->cap);
        b->s2u = (int*)realloc(b->s2u, sizeof(int) * b->cap);
        b->type = (int*)realloc(b->type, sizeof(int) * b->cap);
        b->lev1 = (int*)realloc(b->lev1, sizeof(int) * b->cap);
        b->lev2 = (int*)realloc(b->lev2, sizeof(int) * b->cap);
    }
    int k = b->count++;
    b->s1l[k] = nd->l1; b->s1u[k] = nd->u1;
    b->s2l[k] = nd->l2; b->s2u[k] = nd->u2;
    b->type[k] = type;
    b->lev1[k] = nd->lev1; b->lev2[k] = nd->lev2;
}

/* exact per-cluster bounding box, memoised per level by the lower bound (within one
 * level a lower bound identifies the cluster, tree.cu:909-918). */
typedef struct {
    int n, dim;
    const double* c;
    int* stamp;
    double* lo;
    double* hi;
} bbox_cache;

static void bbox_get(bbox_cache* bc, int level_stamp, int l, int u, const double** lo,
                     const double** hi)
{
    int dim = bc->dim;
    if (bc->stamp[l] != level_stamp) {
        for (int d = 0; d < dim; d++) {
            const double* c = bc->c + (size_t)d * bc->n;
            double a = c[l], b = c[l];
            for (int i = l + 1; i <= u; i++) {
                a = fmin(a, c[i]);
                b = fmax(b, c[i]);
            }
            bc->lo[(size_t)l * dim + d] = a;
            bc->hi[(size_t)l * dim + d] = b;
        }
        bc->stamp[l] = level_stamp;
    }
    *lo = bc->lo + (size_t)l * dim;
    *hi = bc->hi + (size_t)l * dim;
}

/* tree.cu:94-105: nvcc contracts diam += t*t into fma(t,t,diam). */
static double box_diameter(const double* lo, const double* hi, int dim)
{
    double s = 0.0;
    for (int d = 0; d < dim; d++) {
        double t = hi[d] - lo[d];
        s = fma(t, t, s);
    }
    return sqrt(s);
}

/* tree.cu:107-118: at most one of the two gaps per dimension is nonzero, so the
 * contracted and uncontracted forms give the same sum. */
static double box_distance(const double* lo1, const double* hi1, const double* lo2,
                           const double* hi2, int dim)
{
    double s = 0.0;
    for (int d = 0; d < dim; d++) {
        double a = fmax(0.0, lo1[d] - hi2[d]);
        double b = fmax(0.0, lo2[d] - hi1[d]);
        s = s + (a * a + b * b);
    }
    return sqrt(s);
}

/* tree.cu:121-160 (max rule, :159) or the min rule (:158, commented out there). */
static int admissible(const double* lo1, const double* hi1, const double* lo2,
                      const double* hi2, int dim, double eta, int rule)
{
    double d1 = box_diameter(lo1, hi1, dim);
    double d2 = box_diameter(lo2, hi2, dim);
    double dist = box_distance(lo1, hi1, lo2, hi2, dim);
    double lhs = rule == 0 ? fmax(d1, d2) : fmin(d1, d2);
    return lhs <= eta * dist;
}

orc_blocks* orc_tree(const double* coords1, const uint64_t* codes1, int n1,
                     const double* coords2, const uint64_t* codes2, int n2, int dim,
                     double eta, int c_leaf, int max_level, int root_level1,
                     int root_level2, int rule, int sort_dense_first)
{
    orc_blocks* out = (orc_blocks*)calloc(1, sizeof(orc_blocks));
    bbox_cache bc1 = {n1, dim, coords1, (int*)malloc(sizeof(int) * n1),
                      (double*)malloc(sizeof(double) * (size_t)n1 * dim),
                      (double*)malloc(sizeof(double) * (size_t)n1 * dim)};
    bbox_cache bc2 = {n2, dim, coords2, (int*)malloc(sizeof(int) * n2),
                      (double*)malloc(sizeof(double) * (size_t)n2 * dim),
                      (double*)malloc(sizeof(double) * (size_t)n2 * dim)};
    for (int i = 0; i < n1; i++) bc1.stamp[i] = -1;
    for (int i = 0; i < n2; i++) bc2.stamp[i] = -1;

    size_t cap = 1, cnt = 1;
    orc_node* cur = (orc_node*)malloc(sizeof(orc_node) * cap);
    cur[0].l1 = 0; cur[0].u1 = n1 - 1; cur[0].l2 = 0; cur[0].u2 = n2 - 1;
    cur[0].lev1 = root_level1; cur[0].lev2 = root_level2;

    /* tree.cu:1462-1556: one iteration per level */
    for (int it = 0; it < max_level && cnt > 0; it++) {
        out->levels = it + 1;
        size_t ncap = cnt * 4, ncnt = 0;
        orc_node* nxt = (orc_node*)malloc(sizeof(orc_node) * (ncap ? ncap : 1));
        for (size_t q = 0; q < cnt; q++) {
            orc_node nd = cur[q];
            const double *lo1, *hi1, *lo2, *hi2;
            bbox_get(&bc1, it, nd.l1, nd.u1, &lo1, &hi1);
            bbox_get(&bc2, it, nd.l2, nd.u2, &lo2, &hi2);
            if (nd.lev1 == nd.lev2) {
                /* tree.cu:230-257 (count_for_new_level) and :431-446 (leaf emission) */
                int adm = admissible(lo1, hi1, lo2, hi2, dim, eta, rule);
                int m1 = nd.u1 - nd.l1 + 1, m2 = nd.u2 - nd.l2 + 1;
                if (adm) {
                    blocks_push(out, &nd, ORC_WT_ACA);
                } else if (m1 <= c_leaf || m2 <= c_leaf || it + 1 >= max_level) {
                    blocks_push(out, &nd, ORC_WT_DENSE);
                } else {
                    /* tree.cu:336-374: children 11, 12, 21, 22 */
                    int s1 = split_index(codes1, nd.l1, nd.u1);
                    int s2 = split_index(codes2, nd.l2, nd.u2);
                    orc_node c;
                    c.lev1 = nd.lev1 + 1; c.lev2 = nd.lev2 + 1;
                    c.l1 = nd.l1; c.u1 = s1; c.l2 = nd.l2; c.u2 = s2; nxt[ncnt++] = c;
                    c.l1 = nd.l1; c.u1 = s1; c.l2 = s2 + 1; c.u2 = nd.u2; nxt[ncnt++] = c;
                    c.l1 = s1 + 1; c.u1 = nd.u1; c.l2 = nd.l2; c.u2 = s2; nxt[ncnt++] = c;
                    c.l1 = s1 + 1; c.u1 = nd.u1; c.l2 = s2 + 1; c.u2 = nd.u2; nxt[ncnt++] = c;
                }
            } else if (nd.lev1 < nd.lev2) {
                /* tree.cu:376-402: split set 1 only */
                int s1 = split_index(codes1, nd.l1, nd.u1);
                orc_node c = nd;
                c.lev1 = nd.lev1 + 1;
                c.u1 = s1; nxt[ncnt++] = c;
                c.l1 = s1 + 1; c.u1 = nd.u1; nxt[ncnt++] = c;
            } else {
                /* tree.cu:403-428: split set 2 only */
                int s2 = split_index(codes2, nd.l2, nd.u2);
                orc_node c = nd;
                c.lev2 = nd.lev2 + 1;
                c.u2 = s2; nxt[ncnt++] = c;
                c.l2 = s2 + 1; c.u2 = nd.u2; nxt[ncnt++] = c;
            }
        }
        free(cur);
        cur = nxt;
        cnt = ncnt;
        cap = ncap;
    }
    free(cur);
    free(bc1.stamp); free(bc1.lo); free(bc1.hi);
    free(bc2.stamp); free(bc2.lo); free(bc2.hi);
    (void)cap;

    if (sort_dense_first) {
        /* linear_algebra.cu:63-86: stable sort by work_type descending (DENSE=2 first) */
        orc_blocks* s = (orc_blocks*)calloc(1, sizeof(orc_blocks));
        s->levels = out->levels;
        for (int pass = 0; pass < 2; pass++) {
            int want = pass == 0 ? ORC_WT_DENSE : ORC_WT_ACA;
            for (int k = 0; k < out->count; k++) {
                if (out->type[k] != want) continue;
                orc_node nd = {out->s1l[k], out->s1u[k], out->s2l[k], out->s2u[k],
                               out->lev1[k], out->lev2[k]};
                blocks_push(s, &nd, want);
            }
        }
        orc_blocks_free(out);
        out = s;
    }
    return out;
}

int orc_blocks_count(const orc_blocks* b) { return b->count; }
int orc_blocks_levels(const orc_blocks* b) { return b->levels; }

void orc_blocks_get(const orc_blocks* b, int* s1l, int* s1u, int* s2l, int* s2u,
                    int* type, int* level1, int* level2)
{
    size_t sz = sizeof(int) * (size_t)b->count;
    if (!b->count) return;
    if (s1l) memcpy(s1l, b->s1l, sz);
    if (s1u) memcpy(s1u, b->s1u, sz);
    if (s2l) memcpy(s2l, b->s2l, sz);
    if (s2u) memcpy(s2u, b->s2u, sz);
    if (type) memcpy(type, b->type, sz);
    if (level1) memcpy(level1, b->lev1, sz);
    if (level2) memcpy(level2, b->lev2, sz);
}

void orc_blocks_free(orc_blocks* b)
{
    if (!b) return;
    free(b->s1l); free(b->s1u); free(b->s2l); free(b->s2u);
    free(b->type); free(b->lev1); free(b->lev2);
    free(b);
}

/* ------------------------------------------------------------------------- */
/* Kernel entries                                                             */
/* ------------------------------------------------------------------------- */

/* kernel_system_assembler.h:38-52 / 82-96: r^2 accumulated with fma (nvcc contracts
 * result += t*t), regularisation added when the Z-ordered indices coincide.
 * param: kind 3 -> 1/l^2, kind 4 -> sqrt(3)/rho; unused for the reference kinds. */
double orc_entry(int kind, double param, double reg, const double* c1, int n1,
                 const double* c2, int n2, int dim, int i, int j)
{
    double s = 0.0;
    for (int d = 0; d < dim; d++) {
        double t = c1[(size_t)d * n1 + i] - c2[(size_t)d * n2 + j];
        s = fma(t, t, s);
    }
    double k;
    switch (kind) {
    case ORC_KERNEL_GAUSSIAN_REF: {
        double r = sqrt(s);
        k = exp(-r * r);
        break;
    }
    case ORC_KERNEL_MATERN_REF: {
        double r = sqrt(s);
        k = (yn(1, r + 1.0e-15) * pow(r, 1.0)) /
            (pow(2.0, (double)dim / 2.0) * tgamma(1.0 + (double)dim / 2.0));
        break;
    }
    case ORC_KERNEL_GAUSSIAN:
        k = exp(-(s * param));
        break;
    case ORC_KERNEL_MATERN32: {
        double a = sqrt(s) * param;
        k = (1.0 + a) * exp(-a);
        break;
    }
    default:
        k = 0.0;
    }
    if (i == j) k += reg;
    return k;
}

/* ------------------------------------------------------------------------- */
/* ACA                                                                        */
/* ------------------------------------------------------------------------- */

/* One admissible block with the reference's batched-ACA semantics. */
static void aca_fixed_block(int kind, double param, double reg, const double* c1,
                            int n1, const double* c2, int n2, int dim, int r0, int m1,
                            int q0, int m2, int kb, double* U, double* V, int* rank_out,
                            double* v)
{
    memset(U, 0, sizeof(double) * (size_t)m1 * kb);
    memset(V, 0, sizeof(double) * (size_t)m2 * kb);
    int ir = -1, rank = 0;
    for (int r = 0; r < kb; r++) {
        /* linear_algebra.cu:2036-2146: find the next row with residual norm >= 1e-13 */
        int stop = 0;
        for (;;) {
            if (ir >= m1 - 1) { stop = 1; break; }                  /* :2009-2024 */
            ir += 1;                                                /* :2091 */
            for (int j = 0; j < m2; j++) {                          /* :918-959 */
                double val = orc_entry(kind, param, reg, c1, n1, c2, n2, dim, r0 + ir, q0 + j);
                for (int l = 0; l < r; l++)
                    val = fma(-U[(size_t)l * m1 + ir], V[(size_t)l * m2 + j], val);
                v[j] = val;
            }
            double ss = 0.0;
            for (int j = 0; j < m2; j++) ss += v[j] * v[j];
            if (fabs(sqrt(ss)) >= 1.0e-13) break;                  /* :1213-1230 */
        }
        if (stop) {
            /* the stale residual stays in V's column, U's column stays zero */
            memcpy(V + (size_t)r * m2, v, sizeof(double) * m2);
            break;
        }
        /* :2179 reduce_by_key with tuple_absolute_maximum (:991-1018): the right
         * operand wins ties, i.e. the last index of the largest |v| */
        int jr = 0;
        double best = fabs(v[0]);
        for (int j = 1; j < m2; j++) {
            if (!(best > fabs(v[j]))) { best = fabs(v[j]); jr = j; }
        }
        double piv = v[jr];
        for (int j = 0; j < m2; j++) V[(size_t)r * m2 + j] = v[j] / piv; /* :963-986 */
        for (int i = 0; i < m1; i++) {                                   /* :1091-1147 */
            double val = orc_entry(kind, param, reg, c1, n1, c2, n2, dim, r0 + i, q0 + jr);
            for (int l = 0; l < r; l++)
                val = fma(-V[(size_t)l * m2 + jr], U[(size_t)l * m1 + i], val);
            U[(size_t)r * m1 + i] = val;
        }
        rank = r + 1;
    }
    *rank_out = rank;
}

void orc_aca_fixed(int kind, double param, double reg, const double* c1, int n1,
                   const double* c2, int n2, int dim, int nb, const int* s1l,
                   const int* s1u, const int* s2l, const int* s2u, int k,
                   const int64_t* uoff, const int64_t* voff, double* U, double* V,
                   int* ranks)
{
#pragma omp parallel
    {
        double* v = NULL;
        int vcap = 0;
#pragma omp for schedule(dynamic, 4)
        for (int b = 0; b < nb; b++) {
            int m1 = s1u[b] - s1l[b] + 1, m2 = s2u[b] - s2l[b] + 1;
            int kb = k;                                      /* :769-787 */
            if (kb > m1) kb = m1;
            if (kb > m2) kb = m2;
            if (m2 > vcap) { vcap = m2; v = (double*)realloc(v, sizeof(double) * vcap); }
            aca_fixed_block(kind, param, reg, c1, n1, c2, n2, dim, s1l[b], m1, s2l[b], m2,
                            kb, U + uoff[b], V + voff[b], &ranks[b], v);
        }
        free(v);
    }
}

/* The engine's adaptive ACA on one block (standard partial pivoting with the
 * Frobenius stopping rule; the reference keeps such a rule dormant at
 * linear_algebra.cu:1595-1755). */
static void aca_adaptive_block(int kind, double param, double reg, const double* c1,
                               int n1, const double* c2, int n2, int dim, int r0, int m1,
                               int q0, int m2, int kb, double eps, double* U, double* V,
                               int* rank_out, double* v, unsigned char* used)
{
    memset(U, 0, sizeof(double) * (size_t)m1 * kb);
    memset(V, 0, sizeof(double) * (size_t)m2 * kb);
    memset(used, 0, (size_t)m1);
    double S2 = 0.0;
    int rank = 0, ir = 0, nused = 0;
    for (int r = 0; r < kb; r++) {
        int jr = -1;
        double piv = 0.0;
        for (;;) {
            used[ir] = 1;
            nused++;
            for (int j = 0; j < m2; j++) {
                double val = orc_entry(kind, param, reg, c1, n1, c2, n2, dim, r0 + ir, q0 + j);
                for (int l = 0; l < r; l++)
                    val = fma(-U[(size_t)l * m1 + ir], V[(size_t)l * m2 + j], val);
                v[j] = val;
            }
            double best = -1.0;
            for (int j = 0; j < m2; j++) {
                double a = fabs(v[j]);
                if (a > best) { best = a; jr = j; }
            }
            if (best > 0.0) { piv = v[jr]; break; }
            /* zero residual row: take the next unused row in index order */
            ir = -1;
            for (int i = 0; i < m1; i++) if (!used[i]) { ir = i; break; }
            if (ir < 0) break;
        }
        if (ir < 0 || piv == 0.0) break;
        double* Vr = V + (size_t)r * m2;
        double* Ur = U + (size_t)r * m1;
        for (int j = 0; j < m2; j++) Vr[j] = v[j] / piv;
        for (int i = 0; i < m1; i++) {
            double val = orc_entry(kind, param, reg, c1, n1, c2, n2, dim, r0 + i, q0 + jr);
            for (int l = 0; l < r; l++)
                val = fma(-V[(size_t)l * m2 + jr], U[(size_t)l * m1 + i], val);
            Ur[i] = val;
        }
        double nu2 = 0.0, nv2 = 0.0, cross = 0.0;
        for (int i = 0; i < m1; i++) nu2 += Ur[i] * Ur[i];
        for (int j = 0; j < m2; j++) nv2 += Vr[j] * Vr[j];
        for (int l = 0; l < r; l++) {
            double du = 0.0, dv = 0.0;
            for (int i = 0; i < m1; i++) du += Ur[i] * U[(size_t)l * m1 + i];
            for (int j = 0; j < m2; j++) dv += Vr[j] * V[(size_t)l * m2 + j];
            cross += du * dv;
        }
        S2 = S2 + 2.0 * cross + nu2 * nv2;
        rank = r + 1;
        if (sqrt(nu2 * nv2) <= eps * sqrt(fabs(S2))) break;
        if (nused >= m1) break;
        /* next row: largest |u_r| among unused rows (first index on ties) */
        double best = -1.0;
        ir = -1;
        for (int i = 0; i < m1; i++) {
            if (used[i]) continue;
            double a = fabs(Ur[i]);
            if (a > best) { best = a; ir = i; }
        }
        if (ir < 0) break;
    }
    *rank_out = rank;
}

void orc_aca_adaptive(int kind, double param, double reg, const double* c1, int n1,
                      const double* c2, int n2, int dim, int nb, const int* s1l,
                      const int* s1u, const int* s2l, const int* s2u, int kmax,
                      double eps, const int64_t* uoff, const int64_t* voff, double* U,
                      double* V, int* ranks)
{
#pragma omp parallel
    {
        double* v = NULL;
        unsigned char* used = NULL;
        int vcap = 0, ucap = 0;
#pragma omp for schedule(dynamic, 4)
        for (int b = 0; b < nb; b++) {
            int m1 = s1u[b] - s1l[b] + 1, m2 = s2u[b] - s2l[b] + 1;
            int kb = kmax;
            if (kb > m1) kb = m1;
            if (kb > m2) kb = m2;
            if (m2 > vcap) { vcap = m2; v = (double*)realloc(v, sizeof(double) * vcap); }
            if (m1 > ucap) { ucap = m1; used = (unsigned char*)realloc(used, (size_t)ucap); }
            aca_adaptive_block(kind, param, reg, c1, n1, c2, n2, dim, s1l[b], m1, s2l[b], m2,
                               kb, eps, U + uoff[b], V + voff[b], &ranks[b], v, used);
        }
        free(v);
        free(used);
    }
}

/* ------------------------------------------------------------------------- */
/* Products                                                                   */
/* ------------------------------------------------------------------------- */

void orc_hmatvec(int kind, double param, double reg, const double* c1, int n1,
                 const double* c2, int n2, int dim, int nb, const int* s1l,
                 const int* s1u, const int* s2l, const int* s2u, const int* type,
                 const int64_t* uoff, const int64_t* voff, const double* U,
                 const double* V, const int* ranks, const double* xs, double* ys)
{
    for (int i = 0; i < n1; i++) ys[i] = 0.0;
    int maxm = 1;
    for (int b = 0; b < nb; b++) {
        int m1 = s1u[b] - s1l[b] + 1;
        if (m1 > maxm) maxm = m1;
    }
    double* loc = (double*)malloc(sizeof(double) * maxm);
    double* t = NULL;
    int tcap = 0;
    for (int b = 0; b < nb; b++) {
        int r0 = s1l[b], m1 = s1u[b] - s1l[b] + 1;
        int q0 = s2l[b], m2 = s2u[b] - s2l[b] + 1;
        if (type[b] == ORC_WT_DENSE) {
            /* linear_algebra.cu:2817-3137: y_b = A_b x_b, then added into y */
            for (int i = 0; i < m1; i++) {
                double acc = 0.0;
                for (int j = 0; j < m2; j++)
                    acc += orc_entry(kind, param, reg, c1, n1, c2, n2, dim, r0 + i, q0 + j) *
                           xs[q0 + j];
                loc[i] = acc;
            }
        } else {
            /* linear_algebra.cu:1429-1591: t = V_b^T x_b, y_b = U_b t */
            int rk = ranks[b];
            if (rk > tcap) { tcap = rk; t = (double*)realloc(t, sizeof(double) * tcap); }
            const double* Ub = U + uoff[b];
            const double* Vb = V + voff[b];
            for (int l = 0; l < rk; l++) {
                double acc = 0.0;
                for (int j = 0; j < m2; j++) acc += Vb[(size_t)l * m2 + j] * xs[q0 + j];
                t[l] = acc;
            }
            for (int i = 0; i < m1; i++) {
                double acc = 0.0;
                for (int l = 0; l < rk; l++) acc += Ub[(size_t)l * m1 + i] * t[l];
                loc[i] = acc;
            }
        }
        for (int i = 0; i < m1; i++) ys[r0 + i] += loc[i];
    }
    free(loc);
    free(t);
}

void orc_direct(int kind, double param, double reg, const double* c1, int n1,
                const double* c2, int n2, int dim, const double* xs, const int* rows,
                int nrows, double* y, int nthreads)
{
    int cnt = rows ? nrows : n1;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 16)
    for (int t = 0; t < cnt; t++) {
        int i = rows ? rows[t] : t;
        double acc = 0.0;
        for (int j = 0; j < n2; j++)
            acc += orc_entry(kind, param, reg, c1, n1, c2, n2, dim, i, j) * xs[j];
        y[t] = acc;
    }
}

/* hmglib.cu:403-418: rhs_i = prod_d sqrt(pi) (erf(1-x_d) - erf(-x_d)) / 2 */
void orc_gaussian_rhs(const double* coords, int n, int dim, double* b)
{
    const double pi = 3.14159265358979323846;
    for (int i = 0; i < n; i++) {
        double r = 1.0;
        for (int d = 0; d < dim; d++) {
            double x = coords[(size_t)d * n + i];
            r = r * sqrt(pi) * (erf(1.0 - x) - erf(0.0 - x)) / 2.0;
        }
        b[i] = r;
    }
}
