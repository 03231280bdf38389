/*
 * ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of evoc-rs's label-propagation initialisation and its
 * reproducible (block-synchronous) node embedding, used as the checker for the
 * CUDA library.  Only tests/, __graft_entry__.smoke() and the CPU-baseline leg
 * of bench.py load it; the product library never links it.
 *
 * What is restated (paths relative to the evoc-rs source tree):
 *   label_prop_iteration ............ src/label_prop.rs:39-91
 *   label_outliers .................. src/label_prop.rs:94-132
 *   remap_labels .................... src/label_prop.rs:135-157
 *   label_prop_loop ................. src/label_prop.rs:160-185
 *   scipy_csr_matmul (SciPy SMMP) ... src/csr_matmul.rs:6-59
 *   csr_matmul_dense ................ src/label_prop.rs:233-250
 *   make_epochs_per_sample .......... src/embed.rs:10-23
 *   node_embedding_epoch_repr ....... src/embed.rs:138-248
 *   node_embedding (reproducible) ... src/embed.rs:251-369
 *   node_embedding_epoch ............ src/embed.rs:57-135 (non-reproducible: serial, in place)
 *   NumPy shuffle ................... src/numpy_rng.rs:136-141
 *
 * Compiled with -ffp-contract=off so every f32 expression rounds the way the
 * reference's Rust code does (no fused multiply-add).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    uint32_t key[624];
    int32_t pos;
    int32_t has_gauss;
    double gauss;
} orc_mt;

int64_t orc_mt_randint(orc_mt *s, int64_t low, int64_t high);
double orc_mt_normal(orc_mt *s);
void orc_mt_randint3_for_tau(orc_mt *s, int64_t out[3]);
int32_t orc_tau_rand_int(int64_t st[3]);
float orc_tau_rand(int64_t st[3]);

static void offset3(const int64_t base[3], int64_t off, int64_t out[3]) {
    for (int j = 0; j < 3; j++) out[j] = (int64_t)((uint64_t)base[j] + (uint64_t)off);
}

/* ------------------------------------------------------------------ */
/* label propagation                                                    */
/* ------------------------------------------------------------------ */

/* One Jacobi sweep: rows with a label keep it; an unlabelled row takes the
 * label whose f64 vote (edge weights summed in CSR order, labels in order of
 * first appearance) is largest and at least 1.0, the last such on ties. */
void orc_lp_iteration(const int64_t *indptr, const int32_t *indices, const float *data, int64_t n,
                      const int64_t *labels, const int64_t rng_state[3], int64_t *out) {
    int64_t maxdeg = 0;
    for (int64_t i = 0; i < n; i++)
        if (indptr[i + 1] - indptr[i] > maxdeg) maxdeg = indptr[i + 1] - indptr[i];
    int64_t *vl = (int64_t *)malloc(sizeof(int64_t) * (size_t)(maxdeg + 1));
    double *vw = (double *)malloc(sizeof(double) * (size_t)(maxdeg + 1));
    for (int64_t i = 0; i < n; i++) {
        int64_t cur = labels[i];
        out[i] = cur;
        if (cur >= 0) continue;
        int64_t loc[3];
        offset3(rng_state, i, loc);
        int64_t nv = 0;
        for (int64_t k = indptr[i]; k < indptr[i + 1]; k++) {
            int64_t l = labels[indices[k]];
            double w = (double)data[k];
            int64_t t = 0;
            while (t < nv && vl[t] != l) t++;
            if (t < nv) {
                vw[t] += w;
            } else {
                vl[nv] = l;
                vw[nv] = w;
                nv++;
            }
        }
        double max_vote = 1.0;
        int64_t tie = 1, res = cur;
        for (int64_t t = 0; t < nv; t++) {
            if (vl[t] == -1) continue;
            if (vw[t] > max_vote) {
                max_vote = vw[t];
                res = vl[t];
                tie = 1;
            } else if (vw[t] == max_vote) {
                tie++;
                if (cur == -1) res = vl[t];
                else if ((double)orc_tau_rand(loc) < 1.0 / (double)tie) res = vl[t];
            }
        }
        out[i] = res;
    }
    free(vl);
    free(vw);
}

/* Rows still unlabelled take the first labelled neighbour met by a
 * depth-first walk of at most 64 pops (labels set earlier in this pass are
 * visible); a walk that runs 64 pops, or ends without one, draws a random
 * label from the row's tau stream. */
void orc_lp_outliers(const int64_t *indptr, const int32_t *indices, int64_t n, int64_t *labels,
                     const int64_t rng_state[3]) {
    int64_t max_label = 0;
    for (int64_t i = 0; i < n; i++)
        if (labels[i] > max_label) max_label = labels[i];
    int64_t maxdeg = 0;
    for (int64_t i = 0; i < n; i++)
        if (indptr[i + 1] - indptr[i] > maxdeg) maxdeg = indptr[i + 1] - indptr[i];
    size_t cap = (size_t)(64 * maxdeg + 2);
    int64_t *queue = (int64_t *)malloc(sizeof(int64_t) * cap);
    for (int64_t i = 0; i < n; i++) {
        if (labels[i] >= 0) continue;
        int64_t loc[3];
        offset3(rng_state, i, loc);
        size_t qn = 0;
        queue[qn++] = i;
        int unlabelled = 1;
        int n_iter = 0;
        while (unlabelled && n_iter < 64 && qn > 0) {
            n_iter++;
            int64_t node = queue[--qn];
            for (int64_t k = indptr[node]; k < indptr[node + 1]; k++) {
                int64_t j = indices[k];
                if (labels[j] >= 0) {
                    labels[i] = labels[j];
                    unlabelled = 0;
                    break;
                }
                queue[qn++] = j;
            }
        }
        if (n_iter >= 64 || unlabelled) {
            int64_t draw = (int64_t)orc_tau_rand_int(loc);
            int64_t m = max_label + 1;
            int64_t r = draw % m;
            labels[i] = r < 0 ? r + m : r;
        }
    }
    free(queue);
}

static int cmp_i64(const void *a, const void *b) {
    int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
    return (x > y) - (x < y);
}

/* Labels -> 0..u-1 by rank among the distinct non-negative labels; negative
 * labels get u, u+1, ... in row order. */
void orc_lp_remap(int64_t *labels, int64_t n) {
    int64_t *u = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n + 1));
    memcpy(u, labels, sizeof(int64_t) * (size_t)n);
    qsort(u, (size_t)n, sizeof(int64_t), cmp_i64);
    int64_t nu = 0;
    for (int64_t i = 0; i < n; i++)
        if (nu == 0 || u[nu - 1] != u[i]) u[nu++] = u[i];
    int64_t first = 0;
    if (nu > 0 && u[0] == -1) first = 1;
    int64_t next = nu - first;
    for (int64_t i = 0; i < n; i++) {
        if (labels[i] < 0) {
            labels[i] = next++;
        } else {
            int64_t lo = first, hi = nu;
            while (lo < hi) {
                int64_t mid = (lo + hi) / 2;
                if (u[mid] < labels[i]) lo = mid + 1;
                else hi = mid;
            }
            labels[i] = lo - first;
        }
    }
    free(u);
}

/* label_prop_loop: 3 tau-seed draws, approx_n_parts seeds labels[randint(0,n)]
 * = i, n_iter sweeps, outliers, remap.  labels[] holds the starting labels
 * (all -1 from label_propagation_init) and receives the partition. */
void orc_lp_loop(const int64_t *indptr, const int32_t *indices, const float *data, int64_t n, int64_t *labels,
                 orc_mt *rng, int32_t n_iter, int64_t approx_n_parts, int64_t *seeded_out) {
    int64_t rs[3];
    orc_mt_randint3_for_tau(rng, rs);
    for (int64_t i = 0; i < approx_n_parts; i++) {
        int64_t idx = orc_mt_randint(rng, 0, n);
        labels[idx] = i;
    }
    if (seeded_out) memcpy(seeded_out, labels, sizeof(int64_t) * (size_t)n);
    int64_t *tmp = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    for (int32_t it = 0; it < n_iter; it++) {
        orc_lp_iteration(indptr, indices, data, n, labels, rs, tmp);
        memcpy(labels, tmp, sizeof(int64_t) * (size_t)n);
    }
    free(tmp);
    orc_lp_outliers(indptr, indices, n, labels, rs);
    orc_lp_remap(labels, n);
}

/* ------------------------------------------------------------------ */
/* sparse products                                                      */
/* ------------------------------------------------------------------ */

/* C = A * B with SciPy's SMMP ordering: f32 sums accumulated in A-row /
 * B-row order, each output row listing its columns in reverse order of first
 * appearance, exact zeros dropped.  Returns nnz (or -1 if cap is too small). */
int64_t orc_smmp(int64_t n_row, int64_t n_col, const int64_t *ap, const int32_t *ai, const float *ad,
                 const int64_t *bp, const int32_t *bi, const float *bd, int64_t cap, int64_t *cp, int32_t *cj,
                 float *cd) {
    int32_t *next = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n_col + 1));
    float *sums = (float *)calloc((size_t)(n_col + 1), sizeof(float));
    for (int64_t k = 0; k < n_col; k++) next[k] = -1;
    int64_t nnz = 0;
    cp[0] = 0;
    for (int64_t i = 0; i < n_row; i++) {
        int32_t head = -2, length = 0;
        for (int64_t jj = ap[i]; jj < ap[i + 1]; jj++) {
            int64_t j = ai[jj];
            float v = ad[jj];
            for (int64_t kk = bp[j]; kk < bp[j + 1]; kk++) {
                int32_t k = bi[kk];
                sums[k] += v * bd[kk];
                if (next[k] == -1) {
                    next[k] = head;
                    head = k;
                    length++;
                }
            }
        }
        for (int32_t t = 0; t < length; t++) {
            int32_t k = head;
            if (sums[k] != 0.0f) {
                if (nnz >= cap) {
                    free(next);
                    free(sums);
                    return -1;
                }
                cj[nnz] = k;
                cd[nnz] = sums[k];
                nnz++;
            }
            head = next[k];
            next[k] = -1;
            sums[k] = 0.0f;
        }
        cp[i + 1] = nnz;
    }
    free(next);
    free(sums);
    return nnz;
}

/* Per-segment f32 sums, each segment's values added one at a time in order. */
void orc_seg_sum_f32(const float *v, const int64_t *seg, int64_t m, int64_t nseg, float *out) {
    memset(out, 0, sizeof(float) * (size_t)nseg);
    for (int64_t i = 0; i < m; i++) out[seg[i]] += v[i];
}

/* out[r, c] += (w as f64 * dense[col, c] as f64) as f32, entries in CSR order. */
void orc_csr_dense(int64_t n_row, const int64_t *ap, const int32_t *ai, const float *ad, const float *dense,
                   int64_t k, float *out) {
    memset(out, 0, sizeof(float) * (size_t)(n_row * k));
    for (int64_t r = 0; r < n_row; r++)
        for (int64_t e = ap[r]; e < ap[r + 1]; e++) {
            double w = (double)ad[e];
            const float *src = dense + (int64_t)ai[e] * k;
            float *dst = out + r * k;
            for (int64_t c = 0; c < k; c++) dst[c] += (float)(w * (double)src[c]);
        }
}

/* ------------------------------------------------------------------ */
/* reproducible node embedding                                          */
/* ------------------------------------------------------------------ */

void orc_make_epochs_per_sample(const float *w, int64_t m, int32_t n_epochs, float *out) {
    float nf = (float)n_epochs, mx = 0.0f;
    for (int64_t i = 0; i < m; i++)
        if (w[i] > mx) mx = w[i];
    for (int64_t i = 0; i < m; i++) {
        if (mx == 0.0f) {
            out[i] = nf;
            continue;
        }
        float ns = nf * (w[i] / mx);
        if (!(ns >= 1.0f)) ns = 1.0f; /* f32::max(ns, 1.0): NaN -> 1.0 */
        out[i] = nf / ns;
    }
}

static inline float rdist(const float *x, const float *y, int dim) {
    float r = 0.0f;
    for (int d = 0; d < dim; d++) {
        float df = x[d] - y[d];
        r += df * df;
    }
    return r;
}

static inline float clip4(float v) { return v > 4.0f ? 4.0f : (v < -4.0f ? -4.0f : v); }

static inline uint64_t neg_count(float nf, float eon, float rate) {
    float v = (nf - eon) / rate;
    if (v <= 0.0f) return 0;
    if (v != v) return 0;
    if (v >= 2147483647.0f) return 2147483647u;
    return (uint64_t)(int32_t)v;
}

void orc_node_embedding_epoch_repr(float *emb, int32_t ncomp, const uint32_t *indptr, const uint32_t *indices,
                                   uint32_t nv, const float *eps, uint32_t rng_state, int32_t dim, float alpha,
                                   const float *epns, float *eonn, float *eons, uint8_t n, float noise,
                                   float gamma, float *updates, const uint32_t *order, uint32_t block_size) {
    float nf = (float)n;
    float cur[256];
    for (uint64_t bs = 0; bs < nv; bs += block_size) {
        uint64_t be = bs + block_size < nv ? bs + block_size : nv;
        for (uint64_t ni = bs; ni < be; ni++) {
            uint64_t from = order[ni];
            if (from >= nv) continue;
            for (int d = 0; d < dim; d++) cur[d] = emb[from * ncomp + d];
            float *upd = updates + from * ncomp;
            for (uint64_t raw = indptr[from]; raw < indptr[from + 1]; raw++) {
                if (eons[raw] > nf) continue;
                uint64_t to = indices[raw];
                if (to >= nv) continue;
                const float *yt = emb + to * ncomp;
                float ds = rdist(cur, yt, dim);
                if (ds > 0.0f) {
                    float dist = sqrtf(ds);
                    float gc = (-2.0f * noise * dist - 2.0f) / (2.0f * ds - 0.5f * dist + 1.0f);
                    for (int d = 0; d < dim; d++) {
                        float g = gc * (cur[d] - yt[d]);
                        upd[d] += g * alpha;
                    }
                }
                eons[raw] += eps[raw];
                uint64_t nneg = neg_count(nf, eonn[raw], epns[raw]);
                for (uint64_t p = 0; p < nneg; p++) {
                    uint64_t idx = (raw * ((uint64_t)n + p + 1) * (uint64_t)rng_state) % (uint64_t)nv;
                    uint64_t tn = order[idx];
                    if (tn >= nv) continue;
                    const float *yn = emb + tn * ncomp;
                    float dn = rdist(cur, yn, dim);
                    if (dn > 1e-2f) {
                        float gc = gamma * 4.0f / ((1.0f + 0.25f * dn) * dn);
                        if (gc > 0.0f)
                            for (int d = 0; d < dim; d++) {
                                float g = clip4(gc * (cur[d] - yn[d]));
                                upd[d] += g * alpha;
                            }
                    }
                }
                eonn[raw] += (float)nneg * epns[raw];
            }
        }
        for (uint64_t ni = bs; ni < be; ni++) {
            uint64_t from = order[ni];
            if (from >= nv) continue;
            for (int d = 0; d < dim; d++) emb[from * ncomp + d] += updates[from * ncomp + d];
        }
    }
}

/* node_embedding(reproducible_flag = true).  emb (nv x ncomp) holds the
 * initial embedding when have_init, else it is drawn as normal(0.25) from rng
 * (row-major).  Draws n_epochs randint(0, i32::MAX - 1) epoch seeds, then one
 * shuffle of the node order per epoch.  n_run < n_epochs stops after that many
 * epochs (schedule unchanged); the optional *_out arrays receive the state
 * there (updates nv x ncomp, next-negative and next-sample epochs per edge). */
void orc_node_embedding_repr(int64_t nv, const int64_t *indptr64, const int32_t *indices, const float *w,
                             int32_t ncomp, int32_t n_epochs, float *emb, int32_t have_init, float initial_alpha,
                             float negative_sample_rate, float noise, orc_mt *rng, int32_t n_run,
                             float *updates_out, float *eonn_out, float *eons_out) {
    if (!have_init)
        for (int64_t i = 0; i < nv * ncomp; i++) emb[i] = (float)(0.25 * orc_mt_normal(rng));
    int64_t m = indptr64[nv];
    float *eps = (float *)malloc(sizeof(float) * (size_t)(m + 1));
    float *epns = (float *)malloc(sizeof(float) * (size_t)(m + 1));
    float *eonn = (float *)malloc(sizeof(float) * (size_t)(m + 1));
    float *eons = (float *)malloc(sizeof(float) * (size_t)(m + 1));
    uint32_t *ip = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(nv + 1));
    uint32_t *ix = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(m + 1));
    uint32_t *order = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(nv + 1));
    uint32_t *seeds = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n_epochs + 1));
    float *updates = (float *)calloc((size_t)(nv * ncomp + 1), sizeof(float));
    orc_make_epochs_per_sample(w, m, n_epochs, eps);
    for (int64_t e = 0; e < m; e++) {
        epns[e] = eps[e] / negative_sample_rate;
        epns[e] *= 1.5f;
        eonn[e] = epns[e];
        eons[e] = eps[e];
        ix[e] = (uint32_t)indices[e];
    }
    for (int64_t i = 0; i <= nv; i++) ip[i] = (uint32_t)indptr64[i];
    for (int64_t i = 0; i < nv; i++) order[i] = (uint32_t)i;
    uint32_t block = (uint32_t)(nv / 8 > 1024 ? nv / 8 : 1024);
    int32_t dim = ncomp < 255 ? ncomp : 255;
    float alpha = initial_alpha;
    for (int32_t e = 0; e < n_epochs; e++) seeds[e] = (uint32_t)orc_mt_randint(rng, 0, 2147483646);
    if (n_run < 0 || n_run > n_epochs) n_run = n_epochs;
    for (int32_t e = 0; e < n_run; e++) {
        float gamma = n_epochs <= 1 ? 1.0f : 0.5f + ((float)e / (float)(n_epochs - 1)) * 1.0f;
        orc_node_embedding_epoch_repr(emb, ncomp, ip, ix, (uint32_t)nv, eps, seeds[e], dim, alpha, epns, eonn, eons,
                                      (uint8_t)e, noise, gamma, updates, order, block);
        double om = 1.0 - (double)alpha;
        float decay = (float)(om * om * 0.5);
        for (int64_t i = 0; i < nv * ncomp; i++) updates[i] *= decay;
        for (int64_t i = nv - 1; i >= 1; i--) {
            int64_t j = orc_mt_randint(rng, 0, i + 1);
            uint32_t t = order[i];
            order[i] = order[j];
            order[j] = t;
        }
        alpha = initial_alpha * (1.0f - ((float)e / (float)n_epochs));
    }
    if (updates_out) memcpy(updates_out, updates, sizeof(float) * (size_t)(nv * ncomp));
    if (eonn_out) memcpy(eonn_out, eonn, sizeof(float) * (size_t)m);
    if (eons_out) memcpy(eons_out, eons, sizeof(float) * (size_t)m);
    free(eps);
    free(epns);
    free(eonn);
    free(eons);
    free(ip);
    free(ix);
    free(order);
    free(seeds);
    free(updates);
}

/* node_embedding(reproducible_flag = false): epochs of in-place SGD over the
 * edges in CSR order (src/embed.rs:57-135), no momentum, no shuffles.
 * Optional outputs: the per-edge next-negative / next-sample epochs. */
void orc_node_embedding_serial(int64_t nv, const int64_t *indptr64, const int32_t *indices, const float *w,
                               int32_t ncomp, int32_t n_epochs, float *emb, int32_t have_init, float initial_alpha,
                               float negative_sample_rate, float noise, orc_mt *rng, float *eonn_out,
                               float *eons_out) {
    if (!have_init)
        for (int64_t i = 0; i < nv * ncomp; i++) emb[i] = (float)(0.25 * orc_mt_normal(rng));
    int64_t m = indptr64[nv];
    float *eps = (float *)malloc(sizeof(float) * (size_t)(m + 1));
    float *epns = (float *)malloc(sizeof(float) * (size_t)(m + 1));
    float *eonn = (float *)malloc(sizeof(float) * (size_t)(m + 1));
    float *eons = (float *)malloc(sizeof(float) * (size_t)(m + 1));
    uint32_t *head = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(m + 1));
    uint32_t *seeds = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n_epochs + 1));
    orc_make_epochs_per_sample(w, m, n_epochs, eps);
    for (int64_t r = 0; r < nv; r++)
        for (int64_t e = indptr64[r]; e < indptr64[r + 1]; e++) head[e] = (uint32_t)r;
    for (int64_t e = 0; e < m; e++) {
        epns[e] = eps[e] / negative_sample_rate;
        eonn[e] = epns[e];
        eons[e] = eps[e];
    }
    int32_t dim = ncomp < 255 ? ncomp : 255;
    float alpha = initial_alpha;
    for (int32_t e = 0; e < n_epochs; e++) seeds[e] = (uint32_t)orc_mt_randint(rng, 0, 2147483646);
    for (int32_t ep = 0; ep < n_epochs; ep++) {
        float nf = (float)(uint8_t)ep;
        uint64_t n8 = (uint8_t)ep;
        for (int64_t i = 0; i < m; i++) {
            if (eons[i] > nf) continue;
            uint64_t j = head[i], k = (uint32_t)indices[i];
            if (j >= (uint64_t)nv || k >= (uint64_t)nv) continue;
            float *ej = emb + j * ncomp, *ek = emb + k * ncomp;
            float ds = 0.0f;
            for (int d = 0; d < dim; d++) {
                float df = ej[d] - ek[d];
                ds += df * df;
            }
            if (ds > 0.0f) {
                float dist = sqrtf(ds);
                float gc = (-2.0f * noise * dist - 2.0f) / (2.0f * ds - 0.5f * dist + 1.0f);
                for (int d = 0; d < dim; d++) {
                    float g = gc * (ej[d] - ek[d]);
                    ej[d] += g * alpha;
                    ek[d] -= g * alpha;
                }
            }
            eons[i] += eps[i];
            uint64_t nneg = neg_count(nf, eonn[i], epns[i]);
            for (uint64_t p = 0; p < nneg; p++) {
                uint64_t nk = ((n8 + p) * (uint64_t)i * (uint64_t)seeds[ep]) % (uint64_t)nv;
                float *en = emb + nk * ncomp;
                float dn = 0.0f;
                for (int d = 0; d < dim; d++) {
                    float df = ej[d] - en[d];
                    dn += df * df;
                }
                if (dn > 1e-2f) {
                    float gc = 4.0f / ((1.0f + 0.25f * dn) * dn);
                    for (int d = 0; d < dim; d++) {
                        float g = clip4(gc * (ej[d] - en[d]));
                        ej[d] += g * alpha;
                    }
                }
            }
            eonn[i] += (float)nneg * epns[i];
        }
        alpha = initial_alpha * (1.0f - ((float)ep / (float)n_epochs));
    }
    if (eonn_out) memcpy(eonn_out, eonn, sizeof(float) * (size_t)m);
    if (eons_out) memcpy(eons_out, eons, sizeof(float) * (size_t)m);
    free(eps);
    free(epns);
    free(eonn);
    free(eons);
    free(head);
    free(seeds);
}
