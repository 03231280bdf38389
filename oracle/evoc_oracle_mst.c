/*
 * ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of evoc-rs's KD-tree and Borůvka minimum spanning tree
 * over the node embedding (the mutual-reachability MST that the cluster
 * layers are built from), used as the checker for a GPU version.  Only tests/
 * load it; the product library never links it.
 *
 * What is restated (paths relative to the evoc-rs source tree):
 *   introselect / heapsort / partition .. src/kdtree.rs:20-230
 *   build_kdtree ........................ src/kdtree.rs:232-413
 *   rdist, point-to-box bound ........... src/kdtree.rs:415-447
 *   simple_heap_push, deheap_sort ....... src/kdtree.rs:449-541
 *   tree_query_recursion / parallel_tree_query  src/kdtree.rs:543-629
 *   disjoint set (path halving, rank) ... src/disjoint_set.rs:1-45
 *   merge_components .................... src/boruvka.rs:36-85
 *   update_component_vectors ............ src/boruvka.rs:87-131
 *   component_aware_query_recursion ..... src/boruvka.rs:133-261
 *   calculate_block_size, reproducible query  src/boruvka.rs:321-435
 *   initialize_boruvka_from_knn ......... src/boruvka.rs:437-480
 *   parallel_boruvka .................... src/boruvka.rs:492-593
 *
 * The reproducible path (one logical thread, block-sequential component
 * bounds) is the one restated; compiled with -ffp-contract=off.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    const float *data; /* n x d */
    int64_t n, d;
    int64_t n_nodes;
    int64_t *idx_array; /* n */
    int64_t *idx_start, *idx_end; /* n_nodes */
    float *radius;
    uint8_t *is_leaf;
    float *lo, *hi; /* n_nodes x d: node_bounds[0] and node_bounds[1] */
} orc_kdtree;

static inline float X(const orc_kdtree *t, int64_t i, int64_t j) { return t->data[i * t->d + j]; }

static int cmp_idx(const orc_kdtree *t, int64_t axis, int64_t a, int64_t b) {
    float va = X(t, a, axis), vb = X(t, b, axis);
    if (va < vb) return -1;
    if (va > vb) return 1;
    if (a < b) return -1;
    if (a > b) return 1;
    return 0;
}

static void insertion_sort(const orc_kdtree *t, int64_t *ia, int64_t axis, int64_t left, int64_t right) {
    for (int64_t i = left + 1; i < right; i++) {
        int64_t key = ia[i], j = i;
        while (j > left && cmp_idx(t, axis, ia[j - 1], key) > 0) {
            ia[j] = ia[j - 1];
            j--;
        }
        ia[j] = key;
    }
}

static void swap64(int64_t *a, int64_t i, int64_t j) {
    int64_t v = a[i];
    a[i] = a[j];
    a[j] = v;
}

static void sift_down_idx(const orc_kdtree *t, int64_t *ia, int64_t axis, int64_t off, int64_t start, int64_t end) {
    int64_t root = start;
    while (root * 2 + 1 < end) {
        int64_t child = root * 2 + 1, sw = root;
        if (cmp_idx(t, axis, ia[off + sw], ia[off + child]) < 0) sw = child;
        if (child + 1 < end && cmp_idx(t, axis, ia[off + sw], ia[off + child + 1]) < 0) sw = child + 1;
        if (sw == root) return;
        swap64(ia, off + root, off + sw);
        root = sw;
    }
}

static void heapsort_idx(const orc_kdtree *t, int64_t *ia, int64_t axis, int64_t left, int64_t right) {
    int64_t size = right - left;
    if (size <= 1) return;
    for (int64_t i = (size / 2 > 0 ? size / 2 - 1 : 0); i >= 0; i--) sift_down_idx(t, ia, axis, left, i, size);
    for (int64_t i = size - 1; i >= 1; i--) {
        swap64(ia, left, left + i);
        sift_down_idx(t, ia, axis, left, 0, i);
    }
}

static int64_t median3(const orc_kdtree *t, int64_t *ia, int64_t axis, int64_t left, int64_t right) {
    int64_t mid = (left + right - 1) / 2;
    int64_t l = ia[left], m = ia[mid], r = ia[right - 1];
    if (cmp_idx(t, axis, l, m) > 0) {
        swap64(ia, left, mid);
        int64_t v = l;
        l = m;
        m = v;
    }
    if (cmp_idx(t, axis, m, r) > 0) {
        swap64(ia, mid, right - 1);
        int64_t v = m;
        m = r;
        r = v;
        if (cmp_idx(t, axis, l, m) > 0) swap64(ia, left, mid);
    }
    return mid;
}

static int64_t partition_idx(const orc_kdtree *t, int64_t *ia, int64_t axis, int64_t left, int64_t right,
                             int64_t pivot) {
    swap64(ia, pivot, right - 1);
    int64_t pv = ia[right - 1];
    int64_t i = left, j = right - 2;
    for (;;) {
        while (i <= j && cmp_idx(t, axis, ia[i], pv) < 0) i++;
        while (i <= j && cmp_idx(t, axis, ia[j], pv) >= 0) j--;
        if (i >= j) break;
        swap64(ia, i, j);
        i++;
        j--;
    }
    swap64(ia, i, right - 1);
    return i;
}

static void introselect(const orc_kdtree *t, int64_t *ia, int64_t axis, int64_t left, int64_t right, int64_t nth) {
    int64_t size = right - left;
    if (size <= 16) {
        insertion_sort(t, ia, axis, left, right);
        return;
    }
    int64_t depth = (int64_t)(2.0 * log2((double)size));
    while (right - left > 16) {
        if (depth == 0) {
            heapsort_idx(t, ia, axis, left, right);
            return;
        }
        depth--;
        int64_t p = median3(t, ia, axis, left, right);
        int64_t pos = partition_idx(t, ia, axis, left, right, p);
        if (nth < pos) right = pos;
        else if (nth > pos) left = pos + 1;
        else return;
    }
    insertion_sort(t, ia, axis, left, right);
}

static int64_t split_dim(const orc_kdtree *t, int64_t s, int64_t e) {
    int64_t res = 0;
    float best = 0.0f;
    for (int64_t j = 0; j < t->d; j++) {
        float mx = X(t, t->idx_array[s], j), mn = mx;
        for (int64_t i = s + 1; i < e; i++) {
            float v = X(t, t->idx_array[i], j);
            if (v > mx) mx = v;
            if (v < mn) mn = v;
        }
        float spread = mx - mn;
        if (spread > best) {
            best = spread;
            res = j;
        }
    }
    return res;
}

static void init_node(orc_kdtree *t, int64_t node, int64_t s, int64_t e) {
    float *lo = t->lo + node * t->d, *hi = t->hi + node * t->d;
    for (int64_t j = 0; j < t->d; j++) {
        lo[j] = INFINITY;
        hi[j] = -INFINITY;
    }
    for (int64_t i = s; i < e; i++)
        for (int64_t j = 0; j < t->d; j++) {
            float v = X(t, t->idx_array[i], j);
            if (v < lo[j]) lo[j] = v;
            if (v > hi[j]) hi[j] = v;
        }
    float r = 0.0f;
    for (int64_t j = 0; j < t->d; j++) {
        float df = fabsf(hi[j] - lo[j]) * 0.5f;
        r += df * df;
    }
    t->idx_start[node] = s;
    t->idx_end[node] = e;
    t->radius[node] = sqrtf(r);
}

static void build_rec(orc_kdtree *t, int64_t s, int64_t e, int64_t node) {
    int64_t mid = (e - s) / 2;
    init_node(t, node, s, e);
    if (2 * node + 1 >= t->n_nodes || e - s < 2) {
        t->is_leaf[node] = 1;
        return;
    }
    t->is_leaf[node] = 0;
    int64_t axis = split_dim(t, s, e);
    introselect(t, t->idx_array, axis, s, e, s + mid);
    build_rec(t, s, s + mid, 2 * node + 1);
    build_rec(t, s + mid, e, 2 * node + 2);
}

int64_t orc_kdtree_nodes(int64_t n, int64_t leaf_size) {
    double m = (double)(n > 1 ? n - 1 : 1);
    double l = floor(fmax(log2(m / (double)leaf_size), 0.0));
    int64_t levels = (int64_t)l + 1;
    return ((int64_t)1 << levels) - 1;
}

/* Arrays are caller-owned, n_nodes = orc_kdtree_nodes(n, leaf_size). */
void orc_kdtree_build(const float *data, int64_t n, int64_t d, int64_t leaf_size, int64_t *idx_array,
                      int64_t *idx_start, int64_t *idx_end, float *radius, uint8_t *is_leaf, float *lo, float *hi) {
    orc_kdtree t = {data, n, d, orc_kdtree_nodes(n, leaf_size), idx_array, idx_start, idx_end, radius, is_leaf,
                    lo, hi};
    for (int64_t i = 0; i < n; i++) idx_array[i] = i;
    build_rec(&t, 0, n, 0);
}

static inline float rdist(const float *x, const float *y, int64_t d) {
    float r = 0.0f;
    for (int64_t i = 0; i < d; i++) {
        float df = x[i] - y[i];
        r += df * df;
    }
    return r;
}

/* point_to_node_lower_bound_rdist(node_bounds[0], node_bounds[1], pt) */
static inline float box_rdist(const float *lo, const float *hi, const float *pt, int64_t d) {
    float r = 0.0f;
    for (int64_t i = 0; i < d; i++) {
        float a = lo[i] > pt[i] ? lo[i] - pt[i] : 0.0f;
        float b = pt[i] > hi[i] ? pt[i] - hi[i] : 0.0f;
        float s = a + b;
        r += s * s;
    }
    return r;
}

static void heap_push(float *pr, int32_t *ix, int64_t size, float p, int32_t n) {
    if (p >= pr[0]) return;
    int64_t i = 0;
    for (;;) {
        int64_t c1 = 2 * i + 1, c2 = c1 + 1, sw;
        if (c1 >= size) break;
        if (c2 >= size) {
            if (pr[c1] > p) sw = c1;
            else break;
        } else if (pr[c1] >= pr[c2]) {
            if (p < pr[c1]) sw = c1;
            else break;
        } else if (p < pr[c2]) {
            sw = c2;
        } else {
            break;
        }
        pr[i] = pr[sw];
        ix[i] = ix[sw];
        i = sw;
    }
    pr[i] = p;
    ix[i] = n;
}

static void query_rec(const orc_kdtree *t, int64_t node, const float *pt, float *hp, int32_t *hi, int64_t k,
                      float lb) {
    if (lb > hp[0]) return;
    if (t->is_leaf[node]) {
        for (int64_t i = t->idx_start[node]; i < t->idx_end[node]; i++) {
            int64_t idx = t->idx_array[i];
            float dd = rdist(pt, t->data + idx * t->d, t->d);
            if (dd < hp[0]) heap_push(hp, hi, k, dd, (int32_t)idx);
        }
        return;
    }
    int64_t l = 2 * node + 1, r = l + 1;
    float bl = box_rdist(t->lo + l * t->d, t->hi + l * t->d, pt, t->d);
    float br = box_rdist(t->lo + r * t->d, t->hi + r * t->d, pt, t->d);
    if (bl <= br) {
        query_rec(t, l, pt, hp, hi, k, bl);
        query_rec(t, r, pt, hp, hi, k, br);
    } else {
        query_rec(t, r, pt, hp, hi, k, br);
        query_rec(t, l, pt, hp, hi, k, bl);
    }
}

static void siftdown2(float *h1, int32_t *h2, int64_t len, int64_t elt) {
    while (elt * 2 + 1 < len) {
        int64_t l = elt * 2 + 1, r = l + 1, sw = elt;
        if (h1[sw] < h1[l]) sw = l;
        if (r < len && h1[sw] < h1[r]) sw = r;
        if (sw == elt) break;
        float a = h1[elt];
        h1[elt] = h1[sw];
        h1[sw] = a;
        int32_t b = h2[elt];
        h2[elt] = h2[sw];
        h2[sw] = b;
        elt = sw;
    }
}

/* parallel_tree_query(tree, tree.data, k, output_rdist) on every point of the tree. */
static void tree_query_all(const orc_kdtree *t, int64_t k, int output_rdist, float *dist, int32_t *ind) {
    for (int64_t q = 0; q < t->n; q++) {
        float *hp = dist + q * k;
        int32_t *hi = ind + q * k;
        for (int64_t j = 0; j < k; j++) {
            hp[j] = INFINITY;
            hi[j] = -1;
        }
        const float *pt = t->data + q * t->d;
        query_rec(t, 0, pt, hp, hi, k, box_rdist(t->lo, t->hi, pt, t->d));
        if (!output_rdist)
            for (int64_t j = 0; j < k; j++) hp[j] = sqrtf(hp[j]);
        for (int64_t j = k - 1; j >= 1; j--) {
            float a = hp[0];
            hp[0] = hp[j];
            hp[j] = a;
            int32_t b = hi[0];
            hi[0] = hi[j];
            hi[j] = b;
            siftdown2(hp, hi, j, 0);
        }
    }
}

/* ------------------------------------------------------------------ Borůvka */

typedef struct {
    int32_t *parent, *rank;
} dset;

static int32_t ds_find(dset *s, int32_t x) {
    while (s->parent[x] != x) {
        int32_t gp = s->parent[s->parent[x]];
        s->parent[x] = gp;
        x = gp;
    }
    return x;
}

static void ds_union(dset *s, int32_t x, int32_t y) {
    x = ds_find(s, x);
    y = ds_find(s, y);
    if (x == y) return;
    if (s->rank[x] < s->rank[y]) {
        int32_t v = x;
        x = y;
        y = v;
    }
    s->parent[y] = x;
    if (s->rank[x] == s->rank[y]) s->rank[x]++;
}

static void update_components(const orc_kdtree *t, dset *s, int64_t *node_comp, int64_t *point_comp) {
    for (int64_t i = 0; i < t->n; i++) point_comp[i] = ds_find(s, (int32_t)i);
    for (int64_t i = t->n_nodes - 1; i >= 0; i--) {
        if (t->is_leaf[i]) {
            int64_t st = t->idx_start[i], en = t->idx_end[i];
            int64_t c = point_comp[t->idx_array[st]];
            int uniform = 1;
            for (int64_t j = st + 1; j < en; j++)
                if (point_comp[t->idx_array[j]] != c) {
                    uniform = 0;
                    break;
                }
            if (uniform) node_comp[i] = c;
        } else {
            int64_t l = 2 * i + 1, r = l + 1;
            if (node_comp[l] == node_comp[r]) node_comp[i] = node_comp[l];
        }
    }
}

static void comp_query_rec(const orc_kdtree *t, int64_t node, const float *pt, float *hp, int32_t *hi, float core_i,
                           const float *core, int64_t comp, const int64_t *node_comp, const int64_t *point_comp,
                           float lb, float *bound) {
    if (lb > hp[0]) return;
    if (lb > bound[0] || core_i > bound[0]) return;
    if (node_comp[node] == comp) return;
    if (t->is_leaf[node]) {
        for (int64_t i = t->idx_start[node]; i < t->idx_end[node]; i++) {
            int64_t idx = t->idx_array[i];
            if (point_comp[idx] != comp && core[idx] < bound[0]) {
                float dd = rdist(pt, t->data + idx * t->d, t->d);
                dd = fmaxf(fmaxf(dd, core_i), core[idx]);
                if (dd < hp[0]) {
                    hp[0] = dd;
                    hi[0] = (int32_t)idx;
                    if (dd < bound[0]) bound[0] = dd;
                }
            }
        }
        return;
    }
    int64_t l = 2 * node + 1, r = l + 1;
    float bl = box_rdist(t->lo + l * t->d, t->hi + l * t->d, pt, t->d);
    float br = box_rdist(t->lo + r * t->d, t->hi + r * t->d, pt, t->d);
    if (bl <= br) {
        comp_query_rec(t, l, pt, hp, hi, core_i, core, comp, node_comp, point_comp, bl, bound);
        comp_query_rec(t, r, pt, hp, hi, core_i, core, comp, node_comp, point_comp, br, bound);
    } else {
        comp_query_rec(t, r, pt, hp, hi, core_i, core, comp, node_comp, point_comp, br, bound);
        comp_query_rec(t, l, pt, hp, hi, core_i, core, comp, node_comp, point_comp, bl, bound);
    }
}

static int64_t block_size_for(int64_t n_components, int64_t n) {
    double ppc = n_components == 0 ? (double)n : (double)n / (double)n_components;
    int64_t bs = ppc < 10.0 ? 512 : (ppc < 100.0 ? 128 : (ppc < 1000.0 ? 32 : 8)); /* one logical thread */
    if (bs < 1) bs = 1;
    if (bs > n / 4 + 1) bs = n / 4 + 1;
    return bs;
}

/* Returns the number of edges written to edges (n - 1 rows of (from, to, weight)). */
int64_t orc_boruvka_mst(const float *data, int64_t n, int64_t d, int64_t leaf_size, int64_t min_samples,
                        float *edges, float *core_out, int64_t *idx_array_out) {
    int64_t nn = orc_kdtree_nodes(n, leaf_size);
    orc_kdtree t = {data, n, d, nn, malloc(sizeof(int64_t) * n), malloc(sizeof(int64_t) * nn),
                    malloc(sizeof(int64_t) * nn), malloc(sizeof(float) * nn), malloc(nn),
                    malloc(sizeof(float) * nn * d), malloc(sizeof(float) * nn * d)};
    orc_kdtree_build(data, n, d, leaf_size, t.idx_array, t.idx_start, t.idx_end, t.radius, t.is_leaf, t.lo, t.hi);
    if (idx_array_out) memcpy(idx_array_out, t.idx_array, sizeof(int64_t) * n);
    dset s = {malloc(sizeof(int32_t) * n), calloc(n, sizeof(int32_t))};
    for (int64_t i = 0; i < n; i++) s.parent[i] = (int32_t)i;
    int64_t *point_comp = malloc(sizeof(int64_t) * n), *node_comp = malloc(sizeof(int64_t) * nn);
    for (int64_t i = 0; i < nn; i++) node_comp[i] = -1;
    int64_t k = min_samples > 1 ? min_samples + 1 : 2;
    float *kd = malloc(sizeof(float) * n * k);
    int32_t *ki = malloc(sizeof(int32_t) * n * k);
    float *core = malloc(sizeof(float) * n);
    tree_query_all(&t, k, 1, kd, ki);
    for (int64_t i = 0; i < n; i++) core[i] = min_samples > 1 ? kd[i * k + k - 1] : 0.0f;
    if (core_out) memcpy(core_out, core, sizeof(float) * n);
    int64_t ne = 0;
    /* initialize_boruvka_from_knn */
    for (int64_t i = 0; i < n; i++) {
        int64_t nb = -1;
        float w = 0.0f;
        for (int64_t j = 1; j < k; j++) {
            int32_t q = ki[i * k + j];
            if (core[i] >= core[q]) {
                nb = q;
                w = fmaxf(core[i], kd[i * k + j]);
                break;
            }
        }
        if (nb < 0) continue;
        int32_t a = ds_find(&s, (int32_t)i), b = ds_find(&s, (int32_t)nb);
        if (a != b) {
            edges[ne * 3] = (float)i;
            edges[ne * 3 + 1] = (float)nb;
            edges[ne * 3 + 2] = w;
            ne++;
            ds_union(&s, a, b);
        }
    }
    update_components(&t, &s, node_comp, point_comp);
    int64_t ncomp = 0;
    {
        uint8_t *seen = calloc(n, 1);
        for (int64_t i = 0; i < n; i++)
            if (!seen[point_comp[i]]) {
                seen[point_comp[i]] = 1;
                ncomp++;
            }
        free(seen);
    }
    float *cand_d = malloc(sizeof(float) * n), *cbound = malloc(sizeof(float) * n);
    int32_t *cand_i = malloc(sizeof(int32_t) * n);
    int64_t *best = malloc(sizeof(int64_t) * n), *order = malloc(sizeof(int64_t) * n);
    while (ncomp > 1) {
        int64_t bs = block_size_for(ncomp, n);
        float *blockb = malloc(sizeof(float) * bs);
        for (int64_t i = 0; i < n; i++) cbound[i] = INFINITY;
        for (int64_t b0 = 0; b0 < n; b0 += bs) {
            int64_t b1 = b0 + bs < n ? b0 + bs : n;
            for (int64_t i = b0; i < b1; i++) {
                const float *pt = data + i * d;
                float hp = INFINITY;
                int32_t hix = -1;
                float bound = cbound[point_comp[i]];
                comp_query_rec(&t, 0, pt, &hp, &hix, core[i], core, point_comp[i], node_comp, point_comp,
                               box_rdist(t.lo, t.hi, pt, d), &bound);
                cand_d[i] = hp;
                cand_i[i] = hix;
                blockb[i - b0] = bound;
            }
            for (int64_t i = b0; i < b1; i++)
                if (blockb[i - b0] < cbound[point_comp[i]]) cbound[point_comp[i]] = blockb[i - b0];
        }
        free(blockb);
        /* merge_components: first-seen component order, strict improvement */
        for (int64_t i = 0; i < n; i++) best[i] = -1;
        int64_t no = 0;
        for (int64_t i = 0; i < n; i++) {
            int64_t c = point_comp[i];
            if (best[c] < 0) {
                best[c] = i;
                order[no++] = c;
            } else if (cand_d[i] < cand_d[best[c]]) {
                best[c] = i;
            }
        }
        int64_t added = 0;
        for (int64_t o = 0; o < no; o++) {
            int64_t i = best[order[o]];
            if (cand_i[i] < 0) continue; /* nothing outside the component was reachable */
            int32_t a = ds_find(&s, (int32_t)i), b = ds_find(&s, cand_i[i]);
            if (a != b) {
                edges[ne * 3] = (float)i;
                edges[ne * 3 + 1] = (float)cand_i[i];
                edges[ne * 3 + 2] = cand_d[i];
                ne++;
                added++;
                ds_union(&s, a, b);
            }
        }
        ncomp = ncomp > added ? ncomp - added : 0;
        update_components(&t, &s, node_comp, point_comp);
        if (added == 0) break; /* no progress (cannot happen for finite data) */
    }
    for (int64_t e = 0; e < ne; e++) edges[e * 3 + 2] = sqrtf(edges[e * 3 + 2]);
    free(cand_d);
    free(cbound);
    free(cand_i);
    free(best);
    free(order);
    free(kd);
    free(ki);
    free(core);
    free(point_comp);
    free(node_comp);
    free(s.parent);
    free(s.rank);
    free(t.idx_array);
    free(t.idx_start);
    free(t.idx_end);
    free(t.radius);
    free(t.is_leaf);
    free(t.lo);
    free(t.hi);
    return ne;
}
