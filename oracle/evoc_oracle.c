/*
 * ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the evoc-rs kNN-graph path, used as the checker
 * for the CUDA library.  Only tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py load it; the product library never links it and
 * never falls back to it.
 *
 * What is restated (paths relative to the evoc-rs source tree):
 *   NumPy RandomState MT19937 + randint ............ src/numpy_rng.rs:35-112,204-212
 *   tau RNG ........................................ src/rng.rs:5-35
 *   prepare_float / normalize_float_rows ........... src/knn.rs:78-113
 *   knn_graph_impl defaults + RNG draw order ....... src/knn.rs:377-454, 115-154
 *   random-projection splits / trees / forests ..... src/nndescent/float.rs:13-177,
 *                                                    int8.rs:24-204, uint8.rs:38-190
 *   heap push / sift / deheap_sort ................. src/heap.rs:29-200
 *   build_candidates ............................... src/heap.rs:203-343
 *   apply_sorted_graph_updates ..................... src/heap.rs:425-502
 *   leaf-pair init, random init .................... src/nndescent/float.rs:179-390
 *   sorted local join .............................. src/nndescent/float.rs:517-669
 *   nn_descent_*_sorted driver ..................... src/nndescent/float.rs:775-879
 *   distances ...................................... src/fast_cosine.rs:33-63,
 *                                                    src/nndescent/int8.rs:15-21,
 *                                                    src/nndescent/uint8.rs:21-35
 *   transforms ..................................... src/knn.rs:156-187
 *   brute_force_knn ................................ src/knn.rs:189-281
 *   smooth_knn_dist / membership / fuzzy union ..... src/graph_construction.rs:16-115,
 *                                                    191-248; src/csr_matmul.rs:62-150
 *
 * Logical threads: the reference partitions work by rayon thread count T and
 * its results depend on T (RNG offsets, vertex blocks).  Every function here
 * takes T as a parameter and runs the T logical partitions either serially or
 * under OpenMP; the partitions touch disjoint rows, so the result is the same
 * either way.  The one deliberate departure: when a source thread's region of
 * the sorted-update buffer overflows, the reference (T > 1) writes into the
 * next thread's region; here each logical thread keeps its own region with the
 * same capacity bound.  The reference's own buffer sizing makes that overflow
 * impossible while n <= 65536.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_F32 0
#define ORC_I8 1
#define ORC_U8 2

static const float ORC_EPS = 1e-8f;
static const float ORC_INF = 3.40282347e+38f; /* f32::MAX, heap.rs:8 */
static const float ORC_MIN_POSITIVE = 1.17549435e-38f;

/* ------------------------------------------------------------------ */
/* NumPy RandomState (MT19937), src/numpy_rng.rs                        */
/* ------------------------------------------------------------------ */
typedef struct {
    uint32_t key[624];
    int32_t pos;
    int32_t has_gauss;
    double gauss;
} orc_mt;

void orc_mt_seed(orc_mt *s, uint32_t seed) {
    s->key[0] = seed;
    for (uint32_t i = 1; i < 624; i++) {
        seed = 1812433253u * (seed ^ (seed >> 30)) + i;
        s->key[i] = seed;
    }
    s->pos = 624;
    s->has_gauss = 0;
    s->gauss = 0.0;
}

static void mt_regen(orc_mt *s) {
    const uint32_t UP = 0x80000000u, LO = 0x7fffffffu, A = 0x9908b0dfu;
    int i;
    for (i = 0; i < 624 - 397; i++) {
        uint32_t y = (s->key[i] & UP) | (s->key[i + 1] & LO);
        s->key[i] = s->key[i + 397] ^ (y >> 1) ^ ((0u - (y & 1u)) & A);
    }
    for (; i < 623; i++) {
        uint32_t y = (s->key[i] & UP) | (s->key[i + 1] & LO);
        s->key[i] = s->key[i + 397 - 624] ^ (y >> 1) ^ ((0u - (y & 1u)) & A);
    }
    uint32_t y = (s->key[623] & UP) | (s->key[0] & LO);
    s->key[623] = s->key[396] ^ (y >> 1) ^ ((0u - (y & 1u)) & A);
    s->pos = 0;
}

uint32_t orc_mt_next_u32(orc_mt *s) {
    if (s->pos >= 624) mt_regen(s);
    uint32_t y = s->key[s->pos++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

static uint64_t mt_interval(orc_mt *s, uint64_t max) {
    if (max == 0) return 0;
    uint64_t mask = max;
    mask |= mask >> 1; mask |= mask >> 2; mask |= mask >> 4;
    mask |= mask >> 8; mask |= mask >> 16; mask |= mask >> 32;
    for (;;) {
        uint64_t v = (uint64_t)orc_mt_next_u32(s) & mask;
        if (v <= max) return v;
    }
}

int64_t orc_mt_randint(orc_mt *s, int64_t low, int64_t high) {
    uint64_t range = (uint64_t)(high - low);
    if (range == 0) return low;
    return low + (int64_t)mt_interval(s, range - 1);
}

static double mt_double(orc_mt *s) {
    int32_t a = (int32_t)(orc_mt_next_u32(s) >> 5);
    int32_t b = (int32_t)(orc_mt_next_u32(s) >> 6);
    return ((double)a * 67108864.0 + (double)b) / 9007199254740992.0;
}

double orc_mt_normal(orc_mt *s) {
    if (s->has_gauss) {
        s->has_gauss = 0;
        double t = s->gauss;
        s->gauss = 0.0;
        return t;
    }
    for (;;) {
        double x1 = 2.0 * mt_double(s) - 1.0;
        double x2 = 2.0 * mt_double(s) - 1.0;
        double r2 = x1 * x1 + x2 * x2;
        if (r2 < 1.0 && r2 != 0.0) {
            double f = sqrt(-2.0 * log(r2) / r2);
            s->gauss = f * x1;
            s->has_gauss = 1;
            return f * x2;
        }
    }
}

#define TAU_LO (-(int64_t)2147483647)      /* i32::MIN + 1 */
#define TAU_HI ((int64_t)2147483646)       /* i32::MAX - 1 */

void orc_mt_randint3_for_tau(orc_mt *s, int64_t out[3]) {
    for (int j = 0; j < 3; j++) out[j] = orc_mt_randint(s, TAU_LO, TAU_HI);
}

/* ------------------------------------------------------------------ */
/* tau RNG, src/rng.rs                                                  */
/* ------------------------------------------------------------------ */
static inline int64_t shl64(int64_t v, int sh) { return (int64_t)((uint64_t)v << sh); }

int32_t orc_tau_rand_int(int64_t st[3]) {
    st[0] = ((shl64(st[0] & 4294967294LL, 12)) & 0xFFFFFFFFLL) ^
            ((((shl64(st[0], 13)) & 0xFFFFFFFFLL) ^ st[0]) >> 19);
    st[1] = ((shl64(st[1] & 4294967288LL, 4)) & 0xFFFFFFFFLL) ^
            ((((shl64(st[1], 2)) & 0xFFFFFFFFLL) ^ st[1]) >> 25);
    st[2] = ((shl64(st[2] & 4294967280LL, 17)) & 0xFFFFFFFFLL) ^
            ((((shl64(st[2], 3)) & 0xFFFFFFFFLL) ^ st[2]) >> 11);
    return (int32_t)(uint32_t)(uint64_t)(st[0] ^ st[1] ^ st[2]);
}

static inline int32_t wrap_abs32(int32_t v) {
    return v == INT32_MIN ? INT32_MIN : (v < 0 ? -v : v);
}

float orc_tau_rand(int64_t st[3]) {
    int32_t v = orc_tau_rand_int(st);
    return (float)wrap_abs32(v) / 2147483648.0f; /* 0x7FFF_FFFF as f32 */
}

static inline int32_t tau_rand_mod(int64_t st[3], int32_t m) {
    int32_t r = orc_tau_rand_int(st) % m;
    return r < 0 ? r + m : r;
}

static inline void offset_state(const int64_t base[3], int64_t off, int64_t out[3]) {
    for (int j = 0; j < 3; j++) out[j] = (int64_t)((uint64_t)base[j] + (uint64_t)off);
}

/* ------------------------------------------------------------------ */
/* Distances                                                            */
/* ------------------------------------------------------------------ */
float orc_fast_cosine_fastmath(const float *x, const float *y, int dim); /* oracle_cosine.c */
typedef float (*orc_cos_fn)(const float *, const float *, int);
static orc_cos_fn g_strict_cos = orc_fast_cosine_fastmath;

/* Swap in the reference's own compiled fast_cosine_numba (oracle/_ref). */
void orc_set_strict_cosine(orc_cos_fn fn) { g_strict_cos = fn ? fn : orc_fast_cosine_fastmath; }

/* Serial-order f32 dot: the x86 branch of src/fast_cosine.rs:55-62. */
static float cos_serial(const float *x, const float *y, int dim) {
    float acc = 0.0f;
    for (int t = 0; t < dim; t++) acc += x[t] * y[t];
    return acc > 0.0f ? -acc : ORC_MIN_POSITIVE;
}

typedef struct {
    int dtype;
    const void *data;
    int64_t n, dim;
    int strict;
} orc_data;

static inline float dist_i8(const int8_t *x, const int8_t *y, int64_t dim) {
    int32_t acc = 0;
    for (int64_t t = 0; t < dim; t++) acc += (int32_t)x[t] * (int32_t)y[t];
    return -(float)acc;
}

static inline float dist_u8(const uint8_t *x, const uint8_t *y, int64_t dim) {
    uint32_t inter = 0, uni = 0;
    for (int64_t t = 0; t < dim; t++) {
        inter += (uint32_t)__builtin_popcount((unsigned)(x[t] & y[t]));
        uni += (uint32_t)__builtin_popcount((unsigned)(x[t] | y[t]));
    }
    if (uni > 0) return -((float)inter / (float)uni);
    return 0.0f;
}

static inline float dist(const orc_data *D, int64_t a, int64_t b) {
    switch (D->dtype) {
    case ORC_F32: {
        const float *X = (const float *)D->data;
        if (D->strict) return g_strict_cos(X + a * D->dim, X + b * D->dim, (int)D->dim);
        return cos_serial(X + a * D->dim, X + b * D->dim, (int)D->dim);
    }
    case ORC_I8: {
        const int8_t *X = (const int8_t *)D->data;
        return dist_i8(X + a * D->dim, X + b * D->dim, D->dim);
    }
    default: {
        const uint8_t *X = (const uint8_t *)D->data;
        return dist_u8(X + a * D->dim, X + b * D->dim, D->dim);
    }
    }
}

/* Exported single-pair distance (for KAT tests). */
float orc_distance(int dtype, const void *data, int64_t n, int64_t dim, int strict, int64_t a, int64_t b) {
    orc_data D = {dtype, data, n, dim, strict};
    return dist(&D, a, b);
}

/* ------------------------------------------------------------------ */
/* prepare_float, src/knn.rs:78-113                                      */
/* ------------------------------------------------------------------ */
/* Returns 1 when rows were renormalised (data modified in place). */
int orc_prepare_float(float *X, int64_t n, int64_t dim) {
    int all_unit = 1;
    for (int64_t i = 0; i < n && all_unit; i++) {
        float s = 0.0f;
        for (int64_t t = 0; t < dim; t++) s += X[i * dim + t] * X[i * dim + t];
        s = sqrtf(s);
        if (fabsf(s - 1.0f) > 1e-5f) all_unit = 0;
    }
    if (all_unit) return 0;
    for (int64_t i = 0; i < n; i++) {
        float s = 0.0f;
        for (int64_t t = 0; t < dim; t++) s += X[i * dim + t] * X[i * dim + t];
        s = sqrtf(s);
        if (s == 0.0f) s = 1.0f;
        for (int64_t t = 0; t < dim; t++) X[i * dim + t] /= s;
    }
    return 1;
}

/* ------------------------------------------------------------------ */
/* Random projection trees                                              */
/* ------------------------------------------------------------------ */
typedef struct {
    int32_t *pts;
    int64_t npts, cap_pts;
    int64_t *off, *len;
    int64_t nleaves, cap_leaves;
} leafset;

static void leafset_push(leafset *L, const int32_t *idx, int64_t cnt) {
    if (L->npts + cnt > L->cap_pts) {
        while (L->npts + cnt > L->cap_pts) L->cap_pts = L->cap_pts ? 2 * L->cap_pts : 1024;
        L->pts = (int32_t *)realloc(L->pts, (size_t)L->cap_pts * sizeof(int32_t));
    }
    if (L->nleaves == L->cap_leaves) {
        L->cap_leaves = L->cap_leaves ? 2 * L->cap_leaves : 64;
        L->off = (int64_t *)realloc(L->off, (size_t)L->cap_leaves * sizeof(int64_t));
        L->len = (int64_t *)realloc(L->len, (size_t)L->cap_leaves * sizeof(int64_t));
    }
    memcpy(L->pts + L->npts, idx, (size_t)cnt * sizeof(int32_t));
    L->off[L->nleaves] = L->npts;
    L->len[L->nleaves] = cnt;
    L->nleaves++;
    L->npts += cnt;
}

/* Split `idx[0..cnt)` into left/right (caller-provided buffers of size cnt). */
static void rp_split(const orc_data *D, const int32_t *idx, int64_t cnt, int64_t st[3],
                     int32_t *lft, int64_t *nl, int32_t *rgt, int64_t *nr) {
    const int64_t dim = D->dim;
    int32_t isz = (int32_t)cnt;
    uint32_t li = (uint32_t)tau_rand_mod(st, isz);
    uint32_t ri = (uint32_t)tau_rand_mod(st, isz);
    ri += (li == ri);
    ri %= (uint32_t)cnt;
    int64_t left = idx[li], right = idx[ri];

    float *hv = NULL;
    uint8_t *pos = NULL, *neg = NULL;
    if (D->dtype == ORC_F32) {
        const float *X = (const float *)D->data;
        const float *l = X + left * dim, *r = X + right * dim;
        hv = (float *)malloc((size_t)dim * sizeof(float));
        float hn = 0.0f;
        for (int64_t t = 0; t < dim; t++) {
            hv[t] = l[t] - r[t];
            hn += hv[t] * hv[t];
        }
        hn = sqrtf(hn);
        if (fabsf(hn) < ORC_EPS) hn = 1.0f;
        for (int64_t t = 0; t < dim; t++) hv[t] /= hn;
    } else if (D->dtype == ORC_I8) {
        const int8_t *X = (const int8_t *)D->data;
        const int8_t *l = X + left * dim, *r = X + right * dim;
        float ln = 0.0f, rn = 0.0f;
        for (int64_t t = 0; t < dim; t++) {
            float lv = (float)l[t], rv = (float)r[t];
            ln += lv * lv;
            rn += rv * rv;
        }
        ln = sqrtf(ln);
        rn = sqrtf(rn);
        hv = (float *)malloc((size_t)dim * sizeof(float));
        float hn = 0.0f;
        for (int64_t t = 0; t < dim; t++) {
            float lv = ln > 0.0f ? (float)l[t] / ln : 0.0f;
            float rv = rn > 0.0f ? (float)r[t] / rn : 0.0f;
            hv[t] = lv - rv;
            hn += hv[t] * hv[t];
        }
        hn = sqrtf(hn);
        if (fabsf(hn) < ORC_EPS) hn = 1.0f;
        for (int64_t t = 0; t < dim; t++) hv[t] /= hn;
    } else {
        const uint8_t *X = (const uint8_t *)D->data;
        const uint8_t *l = X + left * dim, *r = X + right * dim;
        pos = (uint8_t *)malloc((size_t)dim);
        neg = (uint8_t *)malloc((size_t)dim);
        for (int64_t t = 0; t < dim; t++) {
            uint8_t xv = l[t] ^ r[t];
            pos[t] = xv & l[t];
            neg[t] = xv & r[t];
        }
    }

    int64_t a = 0, b = 0;
    for (int64_t p = 0; p < cnt; p++) {
        int64_t loc[3];
        offset_state(st, p, loc);
        int64_t pt = idx[p];
        float margin = 0.0f;
        if (D->dtype == ORC_F32) {
            const float *x = (const float *)D->data + pt * dim;
            for (int64_t t = 0; t < dim; t++) margin += hv[t] * x[t];
        } else if (D->dtype == ORC_I8) {
            const int8_t *x = (const int8_t *)D->data + pt * dim;
            for (int64_t t = 0; t < dim; t++) margin += hv[t] * (float)x[t];
        } else {
            const uint8_t *x = (const uint8_t *)D->data + pt * dim;
            for (int64_t t = 0; t < dim; t++) {
                margin += (float)__builtin_popcount((unsigned)(pos[t] & x[t]));
                margin -= (float)__builtin_popcount((unsigned)(neg[t] & x[t]));
            }
        }
        int side;
        if (fabsf(margin) < ORC_EPS) side = tau_rand_mod(loc, 2);
        else if (margin > 0.0f) side = 0;
        else side = 1;
        if (side == 0) lft[a++] = (int32_t)pt;
        else rgt[b++] = (int32_t)pt;
    }
    if (a == 0 || b == 0) {
        a = b = 0;
        for (int64_t p = 0; p < cnt; p++) {
            if (tau_rand_mod(st, 2) == 0) lft[a++] = idx[p];
            else rgt[b++] = idx[p];
        }
    }
    free(hv);
    free(pos);
    free(neg);
    *nl = a;
    *nr = b;
}

static void make_tree(const orc_data *D, const int32_t *idx, int64_t cnt, leafset *L, int64_t st[3],
                      int64_t leaf_size, int64_t max_depth) {
    if (cnt > leaf_size && max_depth > 0) {
        int32_t *lft = (int32_t *)malloc((size_t)cnt * sizeof(int32_t));
        int32_t *rgt = (int32_t *)malloc((size_t)cnt * sizeof(int32_t));
        int64_t nl, nr;
        rp_split(D, idx, cnt, st, lft, &nl, rgt, &nr);
        make_tree(D, lft, nl, L, st, leaf_size, max_depth - 1);
        make_tree(D, rgt, nr, L, st, leaf_size, max_depth - 1);
        free(lft);
        free(rgt);
    } else {
        leafset_push(L, idx, cnt);
    }
}

/*
 * make_forest (src/knn.rs:115-154): draws 3*n_trees randint values from the
 * caller's MT state, builds one tree per state, concatenates the leaf arrays.
 * Returns a malloc'd (n_leaves_total x width) int32 array padded with -1.
 */
int32_t *orc_make_forest(const orc_data *D, int64_t n_neighbors, int64_t n_trees, int64_t leaf_size,
                         orc_mt *rng, int64_t max_depth, int64_t *out_rows, int64_t *out_width) {
    leaf_size = leaf_size < 10 ? 10 : leaf_size;
    leaf_size = leaf_size < n_neighbors ? n_neighbors : leaf_size;
    int64_t *states = (int64_t *)malloc((size_t)n_trees * 3 * sizeof(int64_t));
    for (int64_t t = 0; t < n_trees; t++)
        for (int j = 0; j < 3; j++) states[t * 3 + j] = orc_mt_randint(rng, TAU_LO, TAU_HI);
    leafset *Ls = (leafset *)calloc((size_t)n_trees, sizeof(leafset));
    int32_t *all = (int32_t *)malloc((size_t)D->n * sizeof(int32_t));
    for (int64_t i = 0; i < D->n; i++) all[i] = (int32_t)i;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t t = 0; t < n_trees; t++) {
        int64_t st[3] = {states[t * 3], states[t * 3 + 1], states[t * 3 + 2]};
        make_tree(D, all, D->n, &Ls[t], st, leaf_size, max_depth);
    }
    int64_t rows = 0, width = 0;
    for (int64_t t = 0; t < n_trees; t++) {
        int64_t w = leaf_size;
        for (int64_t l = 0; l < Ls[t].nleaves; l++) w = Ls[t].len[l] > w ? Ls[t].len[l] : w;
        width = w > width ? w : width;
        rows += Ls[t].nleaves;
    }
    int32_t *arr = (int32_t *)malloc((size_t)(rows * width) * sizeof(int32_t));
    for (int64_t i = 0; i < rows * width; i++) arr[i] = -1;
    int64_t r = 0;
    for (int64_t t = 0; t < n_trees; t++) {
        for (int64_t l = 0; l < Ls[t].nleaves; l++, r++)
            memcpy(arr + r * width, Ls[t].pts + Ls[t].off[l], (size_t)Ls[t].len[l] * sizeof(int32_t));
        free(Ls[t].pts);
        free(Ls[t].off);
        free(Ls[t].len);
    }
    free(Ls);
    free(all);
    free(states);
    *out_rows = rows;
    *out_width = width;
    return arr;
}

/* Exported wrapper: forest only (for the leaf_array golden). */
int64_t orc_forest(int dtype, const void *data, int64_t n, int64_t dim, int64_t n_neighbors, int64_t n_trees,
                   int64_t leaf_size, orc_mt *rng, int64_t max_depth, int32_t *out, int64_t out_cap,
                   int64_t *out_width) {
    orc_data D = {dtype, data, n, dim, 1};
    int64_t rows, width;
    int32_t *arr = orc_make_forest(&D, n_neighbors, n_trees, leaf_size, rng, max_depth, &rows, &width);
    *out_width = width;
    if (rows * width <= out_cap) memcpy(out, arr, (size_t)(rows * width) * sizeof(int32_t));
    free(arr);
    return rows;
}

/* ------------------------------------------------------------------ */
/* Heaps, src/heap.rs                                                    */
/* ------------------------------------------------------------------ */
static int cand_heap_push(float *pri, int32_t *ind, int64_t size, float p, int32_t n) {
    if (p >= pri[0]) return 0;
    for (int64_t i = 0; i < size; i++)
        if (ind[i] == n) return 0;
    pri[0] = p;
    ind[0] = n;
    int64_t i = 0;
    for (;;) {
        int64_t c1 = 2 * i + 1, c2 = c1 + 1, sw;
        if (c1 >= size) break;
        else if (c2 >= size) {
            if (pri[c1] > p) sw = c1;
            else break;
        } else if (pri[c1] >= pri[c2]) {
            if (p < pri[c1]) sw = c1;
            else break;
        } else if (p < pri[c2]) sw = c2;
        else break;
        pri[i] = pri[sw];
        ind[i] = ind[sw];
        i = sw;
    }
    pri[i] = p;
    ind[i] = n;
    return 1;
}

static int flagged_push(float *pri, int32_t *ind, uint8_t *flg, int64_t size, float p, int32_t n) {
    if (p >= pri[0]) return 0;
    for (int64_t i = 0; i < size; i++)
        if (ind[i] == n) return 0;
    pri[0] = p;
    ind[0] = n;
    int64_t i = 0;
    for (;;) {
        int64_t c1 = 2 * i + 1, c2 = c1 + 1, sw;
        if (c1 >= size) break;
        else if (c2 >= size) {
            if (pri[c1] > p) sw = c1;
            else break;
        } else if (pri[c1] >= pri[c2]) {
            if (p < pri[c1]) sw = c1;
            else break;
        } else if (p < pri[c2]) sw = c2;
        else break;
        pri[i] = pri[sw];
        ind[i] = ind[sw];
        flg[i] = flg[sw];
        i = sw;
    }
    pri[i] = p;
    ind[i] = n;
    flg[i] = 1;
    return 1;
}

static void siftdown(float *h1, int32_t *h2, int64_t n, int64_t e) {
    while (e * 2 + 1 < n) {
        int64_t l = e * 2 + 1, r = l + 1, sw = e;
        if (h1[sw] < h1[l]) sw = l;
        if (r < n && h1[sw] < h1[r]) sw = r;
        if (sw == e) break;
        float tf = h1[e]; h1[e] = h1[sw]; h1[sw] = tf;
        int32_t ti = h2[e]; h2[e] = h2[sw]; h2[sw] = ti;
        e = sw;
    }
}

static void deheap_sort(int32_t *ind, float *dst, int64_t n, int64_t k) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
        int32_t *ir = ind + i * k;
        float *dr = dst + i * k;
        for (int64_t j = k - 1; j >= 1; j--) {
            int32_t ti = ir[0]; ir[0] = ir[j]; ir[j] = ti;
            float tf = dr[0]; dr[0] = dr[j]; dr[j] = tf;
            siftdown(dr, ir, j, 0);
        }
    }
}

typedef struct {
    int32_t *ind;
    float *dst;
    uint8_t *flg;
    int64_t n, k;
} graph_heap;

/* build_candidates, src/heap.rs:203-343 */
static void build_candidates(graph_heap *G, int64_t mc, const int64_t rng_state[3], int64_t T,
                             int32_t *new_ind, int32_t *old_ind, float *new_pri, float *old_pri) {
    const int64_t n = G->n, k = G->k;
    for (int64_t i = 0; i < n * mc; i++) {
        new_ind[i] = -1; old_ind[i] = -1;
        new_pri[i] = ORC_INF; old_pri[i] = ORC_INF;
    }
    const int64_t bs = n / T + 1;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t t = 0; t < T; t++) {
        int64_t loc[3];
        offset_state(rng_state, t, loc);
        const int64_t b0 = t * bs, b1 = (b0 + bs) < n ? (b0 + bs) : n;
        for (int64_t i = 0; i < n; i++) {
            for (int64_t j = 0; j < k; j++) {
                int32_t idx = G->ind[i * k + j];
                if (idx < 0) continue;
                int in_i = (i >= b0 && i < b1), in_x = ((int64_t)idx >= b0 && (int64_t)idx < b1);
                if (!(in_i || in_x)) continue;
                int isn = G->flg[i * k + j] != 0;
                float d = orc_tau_rand(loc);
                int32_t *ci = isn ? new_ind : old_ind;
                float *cp = isn ? new_pri : old_pri;
                if (in_i) cand_heap_push(cp + i * mc, ci + i * mc, mc, d, idx);
                if (in_x) cand_heap_push(cp + (int64_t)idx * mc, ci + (int64_t)idx * mc, mc, d, (int32_t)i);
            }
        }
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
        for (int64_t j = 0; j < k; j++) {
            int32_t idx = G->ind[i * k + j];
            if (idx < 0) continue;
            for (int64_t c = 0; c < mc; c++)
                if (new_ind[i * mc + c] == idx) {
                    G->flg[i * k + j] = 0;
                    break;
                }
        }
    }
}

typedef struct {
    int32_t p, q;
    float d;
} upd;

typedef struct {
    upd *e;
    int64_t cnt, cap, limit;
} updvec;

static inline void updvec_push(updvec *v, int32_t p, int32_t q, float d) {
    if (v->cnt >= v->limit) return; /* reference drops writes past its buffer */
    if (v->cnt == v->cap) {
        v->cap = v->cap ? 2 * v->cap : 256;
        if (v->cap > v->limit) v->cap = v->limit;
        v->e = (upd *)realloc(v->e, (size_t)v->cap * sizeof(upd));
    }
    v->e[v->cnt].p = p;
    v->e[v->cnt].q = q;
    v->e[v->cnt].d = d;
    v->cnt++;
}

/* init_rp_tree_*, src/nndescent/float.rs:179-348 */
static void init_rp_tree(const orc_data *D, graph_heap *G, const int32_t *leaf, int64_t n_leaves, int64_t width,
                         int64_t T) {
    const int64_t n = G->n, k = G->k;
    const int64_t block = T * 64;
    const int64_t n_blocks = n_leaves / block;
    const int64_t vbs = n / T + 1;
    updvec *U = (updvec *)calloc((size_t)T, sizeof(updvec));
    float *thr = (float *)malloc((size_t)n * sizeof(float));
    for (int64_t t = 0; t < T; t++) U[t].limit = INT64_MAX;
    for (int64_t bi = 0; bi <= n_blocks; bi++) {
        int64_t s = bi * block, e = (bi + 1) * block < n_leaves ? (bi + 1) * block : n_leaves;
        if (s >= e) continue;
        for (int64_t v = 0; v < n; v++) thr[v] = G->dst[v * k];
        const int64_t rows = e - s, rpt = rows / T + 1;
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t t = 0; t < T; t++) {
            U[t].cnt = 0;
            for (int64_t r = 0; r < rpt; r++) {
                int64_t li = t * rpt + r;
                if (li >= rows) break;
                const int32_t *lf = leaf + (s + li) * width;
                for (int64_t i = 0; i < width; i++) {
                    int32_t p = lf[i];
                    if (p < 0) break;
                    updvec_push(&U[t], p, p, -1.0f);
                    for (int64_t j = i + 1; j < width; j++) {
                        int32_t q = lf[j];
                        if (q < 0) break;
                        float d = dist(D, p, q);
                        float mt = thr[p] > thr[q] ? thr[p] : thr[q];
                        if (d < mt) updvec_push(&U[t], p, q, d);
                    }
                }
            }
        }
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t t = 0; t < T; t++) {
            const int64_t v0 = t * vbs, v1 = (v0 + vbs) < n ? (v0 + vbs) : n;
            for (int64_t j = 0; j < T; j++) {
                for (int64_t u = 0; u < U[j].cnt; u++) {
                    int32_t p = U[j].e[u].p, q = U[j].e[u].q;
                    float d = U[j].e[u].d;
                    if (p == -1) continue;
                    if (p >= v0 && p < v1) flagged_push(G->dst + p * k, G->ind + p * k, G->flg + p * k, k, d, q);
                    if (q >= v0 && q < v1) flagged_push(G->dst + q * k, G->ind + q * k, G->flg + q * k, k, d, p);
                }
            }
        }
    }
    for (int64_t t = 0; t < T; t++) free(U[t].e);
    free(U);
    free(thr);
}

/* init_random_*, src/nndescent/float.rs:350-390 */
static void init_random(const orc_data *D, graph_heap *G, int64_t n_neighbors, const int64_t rng_state[3]) {
    const int64_t n = G->n, k = G->k;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; i++) {
        int64_t loc[3];
        offset_state(rng_state, i, loc);
        int32_t *ir = G->ind + i * k;
        if (ir[0] >= 0) continue;
        int64_t filled = 0;
        for (int64_t j = 0; j < k; j++) filled += ir[j] >= 0;
        int64_t to_fill = n_neighbors > filled ? n_neighbors - filled : 0;
        for (int64_t f = 0; f < to_fill; f++) {
            int32_t r = wrap_abs32(orc_tau_rand_int(loc));
            int64_t idx = (int64_t)((uint64_t)(int64_t)r % (uint64_t)n);
            int seen = 0;
            for (int64_t j = 0; j < k; j++)
                if (ir[j] == (int32_t)idx) { seen = 1; break; }
            if (seen) continue;
            float d = dist(D, idx, i);
            flagged_push(G->dst + i * k, ir, G->flg + i * k, k, d, (int32_t)idx);
        }
    }
}

/* nn_descent_*_sorted, src/nndescent/float.rs:775-879 (with 517-669, heap.rs:425-502) */
static void nn_descent_sorted(const orc_data *D, int64_t k, int64_t rng_state[3], int64_t mc, int64_t n_iters,
                              float delta, float delta_improv, const int32_t *leaf, int64_t n_leaves,
                              int64_t width, int64_t T, int32_t *out_ind, float *out_dst, int64_t *iters_run) {
    const int64_t n = D->n;
    graph_heap G = {out_ind, out_dst, (uint8_t *)calloc((size_t)(n * k), 1), n, k};
    for (int64_t i = 0; i < n * k; i++) { G.ind[i] = -1; G.dst[i] = ORC_INF; }
    if (leaf) init_rp_tree(D, &G, leaf, n_leaves, width, T);
    init_random(D, &G, k, rng_state);

    int64_t block = 65536 / (T > 0 ? T : 1);
    int64_t n_blocks = n / block;
    const int64_t max_updates = (mc * mc + mc * (mc > 0 ? mc - 1 : 0) / 2) * block;
    const int64_t per_src = max_updates / T;
    updvec *U = (updvec *)calloc((size_t)(T * T), sizeof(updvec)); /* [bucket][src] */
    int32_t *new_ind = (int32_t *)malloc((size_t)(n * mc) * sizeof(int32_t));
    int32_t *old_ind = (int32_t *)malloc((size_t)(n * mc) * sizeof(int32_t));
    float *new_pri = (float *)malloc((size_t)(n * mc) * sizeof(float));
    float *old_pri = (float *)malloc((size_t)(n * mc) * sizeof(float));
    float *thr = (float *)malloc((size_t)n * sizeof(float));
    const int64_t vbs = n / T + 1;
    int have_prev = 0;
    double prev = 0.0;
    int64_t it;
    for (it = 0; it < n_iters; it++) {
        build_candidates(&G, mc, rng_state, T, new_ind, old_ind, new_pri, old_pri);
        uint32_t c = 0;
        for (int64_t bi = 0; bi <= n_blocks; bi++) {
            int64_t s = bi * block, e = (bi + 1) * block < n ? (bi + 1) * block : n;
            if (s >= e) continue;
            for (int64_t v = 0; v < n; v++) thr[v] = G.dst[v * k];
            const int64_t rows = e - s, rpt = rows / T + 1;
#pragma omp parallel for schedule(dynamic, 1)
            for (int64_t t = 0; t < T; t++) {
                for (int64_t b = 0; b < T; b++) {
                    U[b * T + t].cnt = 0;
                    U[b * T + t].limit = max_updates - t * per_src;
                }
                for (int64_t r = 0; r < rpt; r++) {
                    int64_t li = t * rpt + r;
                    if (li >= rows) break;
                    const int32_t *nr = new_ind + (s + li) * mc, *orr = old_ind + (s + li) * mc;
                    for (int64_t j = 0; j < mc; j++) {
                        int32_t p = nr[j];
                        if (p < 0) continue;
                        float tp = thr[p];
                        int64_t pb = p / vbs;
                        if (pb >= T) pb = T - 1;
                        for (int pass = 0; pass < 2; pass++) {
                            const int32_t *qs = pass == 0 ? nr : orr;
                            for (int64_t kk = pass == 0 ? j + 1 : 0; kk < mc; kk++) {
                                int32_t q = qs[kk];
                                if (q < 0) continue;
                                float d = dist(D, p, q);
                                float tq = thr[q];
                                float mt = tp > tq ? tp : tq;
                                if (d <= mt) {
                                    int64_t qb = q / vbs;
                                    if (qb >= T) qb = T - 1;
                                    updvec_push(&U[pb * T + t], p, q, d);
                                    if (qb != pb) updvec_push(&U[qb * T + t], p, q, d);
                                }
                            }
                        }
                    }
                }
            }
            uint32_t cs = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : cs)
            for (int64_t b = 0; b < T; b++) {
                const int64_t v0 = b * vbs, v1 = (v0 + vbs) < n ? (v0 + vbs) : n;
                uint32_t local = 0;
                for (int64_t t = 0; t < T; t++) {
                    const updvec *V = &U[b * T + t];
                    for (int64_t u = 0; u < V->cnt; u++) {
                        int32_t p = V->e[u].p, q = V->e[u].q;
                        float d = V->e[u].d;
                        if (p >= v0 && p < v1)
                            local += flagged_push(G.dst + p * k, G.ind + p * k, G.flg + p * k, k, d, q);
                        if (q >= v0 && q < v1)
                            local += flagged_push(G.dst + q * k, G.ind + q * k, G.flg + q * k, k, d, p);
                    }
                }
                cs += local;
            }
            c += cs;
        }
        float lim = delta * (float)k * (float)n;
        uint32_t ulim = lim <= 0.0f ? 0u : (lim >= 4294967295.0f ? 4294967295u : (uint32_t)lim);
        if (c <= ulim) { it++; break; }
        if (delta_improv >= 0.0f) {
            double sum = 0.0;
            for (int64_t i = 0; i < n * k; i++)
                if (G.dst[i] < ORC_INF) sum += (double)G.dst[i];
            if (have_prev) {
                double rel = fabs(sum - prev) / fabs(prev);
                if (rel < (double)delta_improv) { it++; break; }
            }
            prev = sum;
            have_prev = 1;
        }
        block = (block < n ? block : n) * 2;
        if (block < 1) block = 1;
        n_blocks = n / block;
    }
    if (iters_run) *iters_run = it;
    deheap_sort(G.ind, G.dst, n, k);
    for (int64_t i = 0; i < T * T; i++) free(U[i].e);
    free(U);
    free(new_ind); free(old_ind); free(new_pri); free(old_pri); free(thr);
    free(G.flg);
}

/* ------------------------------------------------------------------ */
/* Transforms, src/knn.rs:156-187                                       */
/* ------------------------------------------------------------------ */
void orc_transform(int dtype, const float *raw, int64_t count, float *out) {
    for (int64_t i = 0; i < count; i++) {
        float d = raw[i];
        float r;
        if (dtype == ORC_F32) {
            if (d >= 0.0f) r = 0.0f;
            else {
                double sim = (double)(-d);
                if (sim >= 1.0) r = 0.0f;
                else r = (float)fmax(-log2(sim), 0.0);
            }
        } else if (dtype == ORC_I8) {
            r = d >= 0.0f ? 0.0f : 1.0f / (-d);
        } else {
            r = d >= 0.0f ? 0.0f : (float)(-log2((double)(-d)));
        }
        out[i] = r;
    }
}

/* ------------------------------------------------------------------ */
/* knn_graph_impl, src/knn.rs:377-454                                    */
/* ------------------------------------------------------------------ */
typedef struct {
    int64_t n_neighbors;
    int64_t n_trees;         /* <= 0: clamp(T, 4, 8) */
    int64_t leaf_size;       /* <= 0: max(10, k) */
    int64_t max_candidates;  /* <= 0: min(60, floor(1.5 k)) */
    int64_t max_rptree_depth;
    int64_t n_iters;         /* <= 0: max(5, round(log2 n)) */
    float delta;
    float delta_improv;      /* < 0 disables the improvement test */
    int64_t brute_force_max_n;
    int32_t deterministic;   /* 1: one logical thread, fast-math cosine */
    int32_t n_threads;       /* logical thread count when not deterministic */
} orc_knn_opts;

/* Error codes mirror KnnError (src/knn.rs:32-41). */
#define ORC_OK 0
#define ORC_ERR_EMPTY 1
#define ORC_ERR_K 2

static void brute_force(const orc_data *D, int64_t k, int32_t *ind, float *dst) {
    const int64_t n = D->n;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < n; i++) {
        float *hd = dst + i * k;
        int32_t *hi = ind + i * k;
        for (int64_t t = 0; t < k; t++) { hd[t] = INFINITY; hi[t] = -1; }
        for (int64_t j = 0; j < n; j++) {
            if (i == j) continue;
            float d;
            if (D->dtype == ORC_F32) d = cos_serial((const float *)D->data + i * D->dim,
                                                     (const float *)D->data + j * D->dim, (int)D->dim);
            else d = dist(D, i, j);
            if (d < hd[0]) {
                hd[0] = d;
                hi[0] = (int32_t)j;
                int64_t pos = 0;
                for (;;) {
                    int64_t l = pos * 2 + 1;
                    if (l >= k) break;
                    int64_t r = l + 1, sw = pos;
                    if (hd[sw] < hd[l]) sw = l;
                    if (r < k && hd[sw] < hd[r]) sw = r;
                    if (sw == pos) break;
                    float tf = hd[pos]; hd[pos] = hd[sw]; hd[sw] = tf;
                    int32_t ti = hi[pos]; hi[pos] = hi[sw]; hi[sw] = ti;
                    pos = sw;
                }
            }
        }
    }
}

/* Exported brute_force_knn (src/knn.rs:189-281): raw distances, heap order. */
int orc_brute_force_knn(int dtype, const void *data, int64_t n, int64_t dim, int64_t k, int32_t *ind,
                        float *raw) {
    orc_data D = {dtype, data, n, dim, 0};
    int64_t kk = k < n - 1 ? k : n - 1;
    if (kk < 1) kk = 1;
    brute_force(&D, kk, ind, raw);
    return (int)kk;
}

int orc_knn_graph(int dtype, const void *data_in, int64_t n, int64_t dim, const orc_knn_opts *o, orc_mt *rng,
                  int32_t *out_ind, float *out_raw, float *out_dist, int64_t *out_k, int64_t *iters_run) {
    if (o->n_neighbors <= 0) return ORC_ERR_K;
    if (n <= 0) return ORC_ERR_EMPTY;
    void *data = (void *)data_in;
    float *owned = NULL;
    if (dtype == ORC_F32) {
        owned = (float *)malloc((size_t)(n * dim) * sizeof(float));
        memcpy(owned, data_in, (size_t)(n * dim) * sizeof(float));
        orc_prepare_float(owned, n, dim);
        data = owned;
    }
    const int64_t T = o->deterministic ? 1 : (o->n_threads > 0 ? o->n_threads : 1);
    orc_data D = {dtype, data, n, dim, o->deterministic ? 1 : 0};
    int64_t k = o->n_neighbors < n - 1 ? o->n_neighbors : n - 1;
    if (k < 1) k = 1;
    int64_t n_trees = o->n_trees > 0 ? o->n_trees : (T < 4 ? 4 : (T > 8 ? 8 : T));
    int64_t leaf_size = o->leaf_size > 0 ? o->leaf_size : (k > 10 ? k : 10);
    int64_t n_iters = o->n_iters > 0 ? o->n_iters : (int64_t)fmax(5.0, round(log2((double)n)));
    int64_t mc = o->max_candidates > 0 ? o->max_candidates : (int64_t)((float)k * 1.5f);
    if (o->max_candidates <= 0 && mc > 60) mc = 60;
    int64_t rs[3];
    orc_mt_randint3_for_tau(rng, rs);
    *out_k = k;
    if (n <= o->brute_force_max_n && dtype != ORC_F32) {
        brute_force(&D, k, out_ind, out_raw);
        if (iters_run) *iters_run = 0;
    } else {
        int64_t rows, width;
        int32_t *leaf = orc_make_forest(&D, k, n_trees, leaf_size, rng, o->max_rptree_depth, &rows, &width);
        nn_descent_sorted(&D, k, rs, mc, n_iters, o->delta, o->delta_improv, leaf, rows, width, T, out_ind,
                          out_raw, iters_run);
        free(leaf);
    }
    orc_transform(dtype, out_raw, n * k, out_dist);
    free(owned);
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* Exact selector: the contract the CUDA exact forms are held to.        */
/* Per row: self offered with raw -1.0 (the NN-descent leaf-init rule,   */
/* src/nndescent/float.rs:209-215), every other row with its raw         */
/* dissimilarity; keep the k smallest by (raw, index) with f32 equality  */
/* (so -0.0 == +0.0); rows come out sorted ascending.                     */
/* f32 dissimilarities use the reference's deterministic cosine           */
/* (native/fast_cosine.c, the path knn_graph takes with deterministic).   */
/* ------------------------------------------------------------------ */
static inline int worse(float da, int32_t ia, float db, int32_t ib) {
    /* (da, ia) > (db, ib) */
    return da > db || (da == db && ia > ib);
}

static void sift_max(float *d, int32_t *ix, int64_t k, int64_t e) {
    for (;;) {
        int64_t l = 2 * e + 1, r = l + 1, m = e;
        if (l < k && worse(d[l], ix[l], d[m], ix[m])) m = l;
        if (r < k && worse(d[r], ix[r], d[m], ix[m])) m = r;
        if (m == e) break;
        float tf = d[e]; d[e] = d[m]; d[m] = tf;
        int32_t ti = ix[e]; ix[e] = ix[m]; ix[m] = ti;
        e = m;
    }
}

static int cmp_pair(const void *a, const void *b) {
    const upd *x = (const upd *)a, *y = (const upd *)b;
    if (x->d < y->d) return -1;
    if (x->d > y->d) return 1;
    return (x->q > y->q) - (x->q < y->q);
}

void orc_exact_knn(int dtype, const void *data, int64_t n, int64_t dim, int64_t k, int64_t row0, int64_t row1,
                   int32_t *out_ind, float *out_raw) {
#pragma omp parallel for schedule(dynamic, 8)
    for (int64_t i = row0; i < row1; i++) {
        orc_data D = {dtype, data, n, dim, 1};
        float *hd = (float *)malloc((size_t)k * sizeof(float));
        int32_t *hi = (int32_t *)malloc((size_t)k * sizeof(int32_t));
        int64_t cnt = 0;
        for (int64_t j = 0; j < n; j++) {
            float d = (j == i) ? -1.0f : dist(&D, i, j);
            if (d != d) continue; /* NaN never enters */
            if (cnt < k) {
                hd[cnt] = d; hi[cnt] = (int32_t)j; cnt++;
                if (cnt == k)
                    for (int64_t e = k / 2 - 1; e >= 0; e--) sift_max(hd, hi, k, e);
            } else if (d < hd[0]) {
                hd[0] = d; hi[0] = (int32_t)j;
                sift_max(hd, hi, k, 0);
            }
        }
        upd *tmp = (upd *)malloc((size_t)k * sizeof(upd));
        for (int64_t t = 0; t < cnt; t++) { tmp[t].d = hd[t]; tmp[t].q = hi[t]; tmp[t].p = 0; }
        qsort(tmp, (size_t)cnt, sizeof(upd), cmp_pair);
        int64_t r = i - row0;
        for (int64_t t = 0; t < k; t++) {
            out_ind[r * k + t] = t < cnt ? tmp[t].q : -1;
            out_raw[r * k + t] = t < cnt ? tmp[t].d : ORC_INF;
        }
        free(tmp); free(hd); free(hi);
    }
}

/* ------------------------------------------------------------------ */
/* Fuzzy graph, src/graph_construction.rs:16-248, csr_matmul.rs:62-150   */
/* ------------------------------------------------------------------ */
/* ndarray's contiguous f32 sum: 8 partial accumulators, then a short tail. */
static float ndarray_sum_f32(const float *x, int64_t len) {
    float acc = 0.0f, p[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int64_t i = 0;
    for (; i + 8 <= len; i += 8)
        for (int j = 0; j < 8; j++) p[j] += x[i + j];
    acc = acc + (p[0] + p[4]);
    acc = acc + (p[1] + p[5]);
    acc = acc + (p[2] + p[6]);
    acc = acc + (p[3] + p[7]);
    for (int64_t j = 0; i < len && j < 7; i++, j++) acc = acc + x[i];
    return acc;
}

void orc_smooth_knn_dist(const float *dists, int64_t n, int64_t k, float kf, float *sigma, float *rho) {
    const double target = log2((double)kf);
    const double mean_all = n * k > 0 ? (double)(ndarray_sum_f32(dists, n * k) / (float)(n * k)) : 0.0;
    const double tol = (double)1e-5f;
    for (int64_t i = 0; i < n; i++) {
        const float *row = dists + i * k;
        double r = 0.0;
        for (int64_t j = 0; j < k; j++)
            if ((double)row[j] > 0.0) { r = (double)row[j]; break; }
        double lo = 0.0, hi = INFINITY, mid = 1.0;
        for (int it = 0; it < 64; it++) {
            double ps = 0.0;
            for (int64_t j = 1; j < k; j++) {
                double d = (double)row[j] - r;
                ps += d > 0.0 ? exp(-(d / mid)) : 1.0;
            }
            if (fabs(ps - target) < tol) break;
            if (ps > target) { hi = mid; mid = (lo + hi) / 2.0; }
            else { lo = mid; if (hi == INFINITY) mid *= 2.0; else mid = (lo + hi) / 2.0; }
        }
        double s = mid;
        if (r > 0.0) {
            double m = 0.0;
            for (int64_t j = 0; j < k; j++) m += (double)row[j];
            m /= (double)k;
            double fl = (double)1e-3f * m;
            if (s < fl) s = fl;
        } else {
            double fl = (double)1e-3f * mean_all;
            if (s < fl) s = fl;
        }
        sigma[i] = (float)s;
        rho[i] = (float)r;
    }
}

void orc_membership(const int32_t *ind, const float *dists, int64_t n, int64_t k, const float *sigma,
                    const float *rho, float *vals) {
    for (int64_t i = 0; i < n; i++)
        for (int64_t j = 0; j < k; j++) {
            int32_t idx = ind[i * k + j];
            float v;
            if (idx == -1) v = 0.0f;
            else if (idx == (int32_t)i) v = 0.0f;
            else if ((dists[i * k + j] - rho[i]) <= 0.0f || sigma[i] == 0.0f) v = 1.0f;
            else v = expf(-((dists[i * k + j] - rho[i]) / sigma[i]));
            vals[i * k + j] = v;
        }
}

typedef struct {
    int64_t *ptr;
    int32_t *col;
    float *val;
    int64_t n, nnz;
} csr;

static int cmp_cv(const void *a, const void *b) {
    const upd *x = (const upd *)a, *y = (const upd *)b;
    return (x->q > y->q) - (x->q < y->q);
}

/* TriMat -> CSR: rows grouped, columns sorted, duplicates summed. */
static csr coo_to_csr(int64_t n, const int32_t *r, const int32_t *c, const float *v, int64_t m) {
    csr A;
    A.n = n;
    A.ptr = (int64_t *)calloc((size_t)(n + 1), sizeof(int64_t));
    for (int64_t e = 0; e < m; e++) A.ptr[r[e] + 1]++;
    for (int64_t i = 0; i < n; i++) A.ptr[i + 1] += A.ptr[i];
    upd *tmp = (upd *)malloc((size_t)(m > 0 ? m : 1) * sizeof(upd));
    int64_t *fill = (int64_t *)calloc((size_t)n, sizeof(int64_t));
    for (int64_t e = 0; e < m; e++) {
        int64_t at = A.ptr[r[e]] + fill[r[e]]++;
        tmp[at].p = (int32_t)e; /* insertion order for stable duplicate sums */
        tmp[at].q = c[e];
        tmp[at].d = v[e];
    }
    A.col = (int32_t *)malloc((size_t)(m > 0 ? m : 1) * sizeof(int32_t));
    A.val = (float *)malloc((size_t)(m > 0 ? m : 1) * sizeof(float));
    int64_t out = 0;
    int64_t *np = (int64_t *)calloc((size_t)(n + 1), sizeof(int64_t));
    for (int64_t i = 0; i < n; i++) {
        int64_t s = A.ptr[i], e = A.ptr[i + 1];
        qsort(tmp + s, (size_t)(e - s), sizeof(upd), cmp_cv);
        for (int64_t t = s; t < e; t++) {
            if (out > np[i] && A.col[out - 1] == tmp[t].q) A.val[out - 1] += tmp[t].d;
            else { A.col[out] = tmp[t].q; A.val[out] = tmp[t].d; out++; }
        }
        np[i + 1] = out;
    }
    free(A.ptr);
    A.ptr = np;
    A.nnz = out;
    free(tmp);
    free(fill);
    return A;
}

static csr csr_transpose(const csr *A) {
    int64_t m = A->nnz;
    int32_t *r = (int32_t *)malloc((size_t)(m > 0 ? m : 1) * sizeof(int32_t));
    int32_t *c = (int32_t *)malloc((size_t)(m > 0 ? m : 1) * sizeof(int32_t));
    for (int64_t i = 0; i < A->n; i++)
        for (int64_t e = A->ptr[i]; e < A->ptr[i + 1]; e++) { r[e] = A->col[e]; c[e] = (int32_t)i; }
    csr T = coo_to_csr(A->n, r, c, A->val, m);
    free(r);
    free(c);
    return T;
}

/* scipy_csr_rowwise_binop; op 0 = mul (intersect), 1 = add, 2 = sub (union). */
static csr csr_binop(const csr *A, const csr *B, int op) {
    csr C;
    C.n = A->n;
    C.ptr = (int64_t *)calloc((size_t)(A->n + 1), sizeof(int64_t));
    int64_t cap = A->nnz + B->nnz + 1;
    C.col = (int32_t *)malloc((size_t)cap * sizeof(int32_t));
    C.val = (float *)malloc((size_t)cap * sizeof(float));
    int64_t out = 0;
    for (int64_t i = 0; i < A->n; i++) {
        int64_t ja = A->ptr[i], jb = B->ptr[i], ea = A->ptr[i + 1], eb = B->ptr[i + 1];
        while (ja < ea || jb < eb) {
            int64_t ca = ja < ea ? A->col[ja] : INT64_MAX, cb = jb < eb ? B->col[jb] : INT64_MAX;
            int64_t col = ca < cb ? ca : cb;
            int ha = ca == col, hb = cb == col;
            float va = ha ? A->val[ja] : 0.0f, vb = hb ? B->val[jb] : 0.0f;
            int emit;
            float v;
            if (op == 0) { emit = ha && hb; v = va * vb; }
            else if (op == 1) { emit = 1; v = va + vb; }
            else { emit = 1; v = va - vb; }
            if (emit && v != 0.0f) { C.col[out] = (int32_t)col; C.val[out] = v; out++; }
            if (ha) ja++;
            if (hb) jb++;
        }
        C.ptr[i + 1] = out;
    }
    C.nnz = out;
    return C;
}

static void csr_free(csr *A) { free(A->ptr); free(A->col); free(A->val); }

/*
 * neighbor_graph_matrix (src/graph_construction.rs:176-235).  Writes sigma,
 * rho and the CSR (indptr n+1, indices/data up to cap).  Returns nnz, or
 * -(nnz) when `cap` is too small.
 */
int64_t orc_fuzzy_graph(const int32_t *ind, const float *dists, int64_t n, int64_t k, float kf, int symmetrize,
                        float *sigma, float *rho, int64_t *indptr, int32_t *indices, float *data, int64_t cap) {
    orc_smooth_knn_dist(dists, n, k, kf, sigma, rho);
    float *vals = (float *)malloc((size_t)(n * k) * sizeof(float));
    orc_membership(ind, dists, n, k, sigma, rho, vals);
    int32_t *r = (int32_t *)malloc((size_t)(n * k) * sizeof(int32_t));
    int32_t *c = (int32_t *)malloc((size_t)(n * k) * sizeof(int32_t));
    float *v = (float *)malloc((size_t)(n * k) * sizeof(float));
    int64_t m = 0;
    for (int64_t i = 0; i < n; i++)
        for (int64_t j = 0; j < k; j++) {
            int32_t idx = ind[i * k + j];
            if (idx == -1) continue;
            float w = vals[i * k + j];
            if (w != 0.0f) { r[m] = (int32_t)i; c[m] = idx; v[m] = w; m++; }
        }
    csr A = coo_to_csr(n, r, c, v, m);
    csr R;
    if (symmetrize) {
        csr At = csr_transpose(&A);
        csr P = csr_binop(&A, &At, 0);
        csr S = csr_binop(&A, &At, 1);
        R = csr_binop(&S, &P, 2);
        csr_free(&At); csr_free(&P); csr_free(&S); csr_free(&A);
    } else {
        R = A;
    }
    /* canonicalize_csr_rows: rows and columns already sorted; drop zeros. */
    int64_t out = 0;
    indptr[0] = 0;
    for (int64_t i = 0; i < n; i++) {
        for (int64_t e = R.ptr[i]; e < R.ptr[i + 1]; e++) {
            if (R.val[e] == 0.0f) continue;
            if (out < cap) { indices[out] = R.col[e]; data[out] = R.val[e]; }
            out++;
        }
        indptr[i + 1] = out;
    }
    csr_free(&R);
    free(vals); free(r); free(c); free(v);
    return out <= cap ? out : -out;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
#else
    (void)t;
#endif
}
