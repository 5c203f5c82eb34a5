/*
 * rover_oracle.c -- CPU restatement of Rover's quantized graph-search path.
 *
 * TEST INFRASTRUCTURE ONLY (see rover_oracle.h).  Compiled by
 * `make -C oracle port` with -O2 -ffp-contract=off: each FP32 expression is
 * written in the reference's operation order and the compiler must not fuse
 * multiply-adds, so results are bit-identical to the reference's host build.
 * Each function names the reference function (file:line, paths relative to
 * the reference checkout) it restates.
 */
#define _GNU_SOURCE
#include "rover_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* shared helpers                                                      */

typedef struct { int32_t id; float dist; } Cand;

static inline int code4(const uint8_t *p, int i) {
    return (i & 1) ? (p[i >> 1] >> 4) : (p[i >> 1] & 0x0f);
}

/* Strict total order on (distance, id): sqmd_pure_pq.c:97-112. */
static inline int pq_order(float ld, int li, float rd, int ri) {
    if (ld < rd) return -1;
    if (ld > rd) return 1;
    if (li < ri) return -1;
    if (li > ri) return 1;
    return 0;
}

static int pq_cand_cmp(const void *a, const void *b) {
    const Cand *x = (const Cand *)a, *y = (const Cand *)b;
    return pq_order(x->dist, x->id, y->dist, y->id);
}

/* ------------------------------------------------------------------ */
/* PQ: LUT, ADC, residual correction                                   */

/* retrieval_pq_build_lut + pq_sub_l2, retrieval_pq_core.c:362-390, :16-25 */
int oracle_pq_build_lut(const OraclePqIndex *ix, const float *query, float *lut) {
    for (int m = 0; m < ix->m; m++) {
        const float *q = query + (size_t)m * ix->subdim;
        for (int k = 0; k < ix->ks; k++) {
            const float *c = ix->codebook + ((size_t)m * ix->ks + k) * ix->subdim;
            float acc = 0.0f;
            for (int d = 0; d < ix->subdim; d++) {
                float diff = q[d] - c[d];
                acc += diff * diff;
            }
            if (!isfinite(acc)) return -1;
            lut[(size_t)m * ix->ks + k] = acc;
        }
    }
    return 0;
}

/* retrieval_pq_adc_scalar, retrieval_pq_core.c:392-416 (FLT_MAX = invalid) */
static float pq_adc_one(const OraclePqIndex *ix, const uint8_t *code, const float *lut) {
    float acc = 0.0f;
    for (int m = 0; m < ix->m; m++) {
        int c = ix->ks <= 16 ? code4(code, m) : code[m];
        float v;
        if (c >= ix->ks) return FLT_MAX;
        v = lut[(size_t)m * ix->ks + c];
        if (!isfinite(v)) return FLT_MAX;
        acc += v;
        if (!isfinite(acc)) return FLT_MAX;
    }
    return acc;
}

/* retrieval_pq_adc_ids_batch_scalar, retrieval_pq_core.c:280-360 */
int oracle_pq_adc(const OraclePqIndex *ix, const float *lut, const int32_t *ids, int count,
                  float *out) {
    for (int i = 0; i < count; i++) {
        float d;
        if (ids[i] < 0 || ids[i] >= ix->n) return -1;
        d = pq_adc_one(ix, ix->codes + (size_t)ids[i] * ix->code_bytes, lut);
        if (!isfinite(d) || d == FLT_MAX) return -1;
        out[i] = d;
    }
    return 0;
}

static inline const uint8_t *pq_residual_row(const OraclePqIndex *ix, int id) {
    /* pq_residual_query_block, retrieval_pq_residual.c:914-924 */
    size_t block = (size_t)id / (size_t)ix->vectors_per_block;
    size_t within = ((size_t)id % (size_t)ix->vectors_per_block) * (size_t)ix->residual_code_bytes;
    return ix->residual + block * 4096u + within;
}

/* pq_residual_decode_value, retrieval_pq_residual.c:946-952: ((c + q*s) + z),
 * each step rounded to float. */
static inline float pq_decode_value(float centroid, int code, float scale, float zero) {
    volatile float product = (float)code * scale;
    volatile float sum = centroid + product;
    volatile float value = sum + zero;
    return value;
}

/* retrieval_pq_residual_query_evaluate, retrieval_pq_residual.c:983-1042 */
static int pq_residual_eval_one(const OraclePqIndex *ix, const float *query, int id, float *out) {
    const uint8_t *codes, *res;
    float scale, zero, dist = 0.0f;
    int dim = 0;
    if (id < 0 || id >= ix->n) return -1;
    scale = ix->qparams[2 * (size_t)id];
    zero = ix->qparams[2 * (size_t)id + 1];
    if (!isfinite(scale) || !isfinite(zero) || scale <= 0.0f) return -1;
    codes = ix->codes + (size_t)id * ix->code_bytes;
    res = pq_residual_row(ix, id);
    for (int m = 0; m < ix->m; m++) {
        int c = ix->ks == 16 ? code4(codes, m) : codes[m];
        const float *cv = ix->codebook + ((size_t)m * ix->ks + c) * ix->subdim;
        for (int j = 0; j < ix->subdim; j++, dim++) {
            int q = ix->residual_bits == 4 ? code4(res, dim) : res[dim];
            float x = pq_decode_value(cv[j], q, scale, zero);
            float diff = query[dim] - x;
            dist += diff * diff;
        }
    }
    if (!isfinite(dist)) return -1;
    *out = dist;
    return 0;
}

int oracle_pq_residual_eval(const OraclePqIndex *ix, const float *query, const int32_t *ids,
                            int count, float *out) {
    for (int i = 0; i < count; i++)
        if (pq_residual_eval_one(ix, query, ids[i], &out[i]) != 0) return -1;
    return 0;
}

/* retrieval_pq_residual_query_decode, retrieval_pq_residual.c:954-981 */
int oracle_pq_decode(const OraclePqIndex *ix, int id, float *out) {
    const uint8_t *codes, *res;
    float scale, zero;
    int dim = 0;
    if (id < 0 || id >= ix->n) return -1;
    scale = ix->qparams[2 * (size_t)id];
    zero = ix->qparams[2 * (size_t)id + 1];
    if (!isfinite(scale) || scale <= 0 || !isfinite(zero)) return -1;
    codes = ix->codes + (size_t)id * ix->code_bytes;
    res = pq_residual_row(ix, id);
    for (int m = 0; m < ix->m; m++) {
        int c = ix->ks == 16 ? code4(codes, m) : codes[m];
        const float *cv = ix->codebook + ((size_t)m * ix->ks + c) * ix->subdim;
        for (int j = 0; j < ix->subdim; j++, dim++) {
            int q = ix->residual_bits == 4 ? code4(res, dim) : res[dim];
            out[dim] = pq_decode_value(cv[j], q, scale, zero);
            if (!isfinite(out[dim])) return -1;
        }
    }
    return 0;
}

/* pure_pq_make_seed_ids, retrieval_rpc_demo_pure_pq.c:192-208 */
int oracle_pq_seed_ids(int n, int entry_count, int graph_entry, uint32_t seed, int32_t *ids) {
    int count = entry_count < n ? entry_count : n;
    for (int i = 0; i < count; i++) {
        if (i == 0 && graph_entry >= 0 && graph_entry < n) {
            ids[i] = graph_entry;
        } else {
            seed = seed * 1103515245u + 12345u;
            ids[i] = (int32_t)(((uint64_t)seed * (uint64_t)n) >> 32);
        }
    }
    return count;
}

/* ------------------------------------------------------------------ */
/* PQ beam search, retrieval_pure_pq_search_scalar_with_policy,        */
/* retrieval_sqmd_pure_pq.c:793-969, with its heaps (:121-249).        */

static void pq_pool_up(Cand *h, int pos) {
    Cand c = h[pos];
    while (pos > 0) {
        int parent = (pos - 1) / 2;
        if (pq_order(c.dist, c.id, h[parent].dist, h[parent].id) <= 0) break;
        h[pos] = h[parent];
        pos = parent;
    }
    h[pos] = c;
}

static void pq_pool_down(Cand *h, int size, int pos) {
    Cand c = h[pos];
    for (;;) {
        int child = pos * 2 + 1;
        if (child >= size) break;
        if (child + 1 < size && pq_order(h[child + 1].dist, h[child + 1].id,
                                         h[child].dist, h[child].id) > 0)
            child++;
        if (pq_order(c.dist, c.id, h[child].dist, h[child].id) >= 0) break;
        h[pos] = h[child];
        pos = child;
    }
    h[pos] = c;
}

static int pq_pool_insert(Cand *h, int *size, int cap, int id, float dist) {
    if (*size < cap) {
        h[*size].id = id; h[*size].dist = dist;
        pq_pool_up(h, *size);
        (*size)++;
        return 1;
    }
    if (pq_order(dist, id, h[0].dist, h[0].id) < 0) {
        h[0].id = id; h[0].dist = dist;
        pq_pool_down(h, *size, 0);
        return 1;
    }
    return 0;
}

static void pq_front_up(Cand *f, int pos) {
    Cand c = f[pos];
    while (pos > 0) {
        int parent = (pos - 1) / 2;
        if (pq_order(c.dist, c.id, f[parent].dist, f[parent].id) >= 0) break;
        f[pos] = f[parent];
        pos = parent;
    }
    f[pos] = c;
}

static void pq_front_down(Cand *f, int size, int pos) {
    Cand c = f[pos];
    for (;;) {
        int child = pos * 2 + 1;
        if (child >= size) break;
        if (child + 1 < size && pq_order(f[child + 1].dist, f[child + 1].id,
                                         f[child].dist, f[child].id) < 0)
            child++;
        if (pq_order(c.dist, c.id, f[child].dist, f[child].id) <= 0) break;
        f[pos] = f[child];
        pos = child;
    }
    f[pos] = c;
}

/* pure_pq_graph_row_count, retrieval_sqmd_pure_pq.c:59-87: the row is a
 * valid prefix followed only by -1 padding; anything else is an error. */
static int pq_row_count(const int32_t *row, int slots, int n) {
    for (int i = 0; i < slots; i++) {
        int id = row[i];
        if (id == -1) {
            for (int s = i + 1; s < slots; s++)
                if (row[s] != -1) return -1;
            return i;
        }
        if (id < 0 || id >= n) return -1;
    }
    return slots;
}

static int pq_score(const OraclePqIndex *ix, const float *query, const float *lut, int id,
                    int correction, float *out) {
    float d = pq_adc_one(ix, ix->codes + (size_t)id * ix->code_bytes, lut);
    if (!isfinite(d) || d == FLT_MAX) return -1;
    /* pure_pq_evaluate_distance, retrieval_sqmd_pure_pq.c:40-57 */
    if (correction) {
        float c;
        if (pq_residual_eval_one(ix, query, id, &c) != 0 || !isfinite(c)) return -1;
        d = c;
    }
    *out = d;
    return 0;
}

int oracle_pq_search(const OraclePqIndex *ix, const float *query, const int32_t *entry_ids,
                     int entry_count, int expand_count, int pool_capacity, int num_out,
                     int correction, int32_t *out_ids, float *out_dists, uint64_t *stats) {
    int n = ix->n, pool_size = 0, front_size = 0, result = -1;
    int expand = expand_count < ix->degree ? expand_count : ix->degree;
    uint64_t scored = 0, corrected = 0, expanded = 0, dedup = 0;
    Cand *pool = malloc((size_t)pool_capacity * sizeof(Cand));
    Cand *front = malloc((size_t)n * sizeof(Cand));
    uint32_t *visited = calloc(((size_t)n + 31) / 32, sizeof(uint32_t));
    float *lut = malloc((size_t)ix->m * ix->ks * sizeof(float));
    int32_t *batch = malloc((size_t)(expand > 0 ? expand : 1) * sizeof(int32_t));
    if (!pool || !front || !visited || !lut || !batch || entry_count <= 0 || expand <= 0 ||
        pool_capacity <= 0 || num_out <= 0 || num_out > pool_capacity ||
        oracle_pq_build_lut(ix, query, lut) != 0)
        goto done;
    for (int e = 0; e < entry_count; e++) {
        int id = entry_ids[e];
        float d;
        if (id < 0 || id >= n) goto done;
        if (visited[id >> 5] & (1u << (id & 31))) { dedup++; continue; }
        visited[id >> 5] |= 1u << (id & 31);
        if (pq_score(ix, query, lut, id, correction, &d) != 0) goto done;
        scored++;
        if (correction) corrected++;
        if (pq_pool_insert(pool, &pool_size, pool_capacity, id, d)) {
            front[front_size].id = id; front[front_size].dist = d;
            pq_front_up(front, front_size++);
        }
    }
    while (front_size > 0) {
        Cand src;
        int count, nb = 0, found = 0;
        const int32_t *row;
        if (pool_size == pool_capacity &&
            pq_order(front[0].dist, front[0].id, pool[0].dist, pool[0].id) > 0)
            break;
        src = front[0];
        front_size--;
        if (front_size > 0) { front[0] = front[front_size]; pq_front_down(front, front_size, 0); }
        /* pure_pq_pool_contains, retrieval_sqmd_pure_pq.c:240-249 */
        for (int i = 0; i < pool_size; i++)
            if (pool[i].id == src.id && pool[i].dist == src.dist) { found = 1; break; }
        if (!found) continue;
        row = ix->graph + (size_t)src.id * ix->degree;
        count = pq_row_count(row, expand, n);
        if (count < 0) goto done;
        for (int j = 0; j < count; j++) {
            int id = row[j];
            if (visited[id >> 5] & (1u << (id & 31))) { dedup++; continue; }
            visited[id >> 5] |= 1u << (id & 31);
            batch[nb++] = id;
        }
        expanded++;
        for (int j = 0; j < nb; j++) {
            float d;
            if (pq_score(ix, query, lut, batch[j], correction, &d) != 0) goto done;
            scored++;
            if (correction) corrected++;
            if (pq_pool_insert(pool, &pool_size, pool_capacity, batch[j], d)) {
                front[front_size].id = batch[j]; front[front_size].dist = d;
                pq_front_up(front, front_size++);
            }
        }
    }
    qsort(pool, (size_t)pool_size, sizeof(Cand), pq_cand_cmp);
    result = num_out < pool_size ? num_out : pool_size;
    for (int i = 0; i < result; i++) { out_ids[i] = pool[i].id; out_dists[i] = pool[i].dist; }
    if (stats) { stats[0] = scored; stats[1] = corrected; stats[2] = expanded; stats[3] = dedup; }
done:
    free(pool); free(front); free(visited); free(lut); free(batch);
    return result;
}

/* ------------------------------------------------------------------ */
/* SQ codes                                                            */

/* retrieval_quantize_query_u8 / _u4, retrieval_l1_int8_core.c:13-63 */
int oracle_sq_quantize(const OracleSqIndex *ix, const float *query, uint8_t *out) {
    int levels = ix->l1_bits == 4 ? 15 : 255;
    float inv;
    if (ix->l1_scale == 0.0f) return -1;
    inv = 1.0f / ix->l1_scale;
    for (int i = 0; i < ix->dim; i++) {
        int v = (int)roundf((query[i] - ix->l1_zero) * inv);
        if (v < 0) v = 0;
        else if (v > levels) v = levels;
        out[i] = (uint8_t)v;
    }
    return 0;
}

/* retrieval_compute_int8_native_distance_u8_scalar (:119-148) and
 * retrieval_compute_int4_packed_distance_u8_scalar (:150-169):
 * exact integer sum, then (float)acc * (scale * scale). */
float oracle_sq_coarse(const OracleSqIndex *ix, const uint8_t *qc, int id) {
    const uint8_t *x = ix->l1 + (size_t)id * ix->l1_code_bytes;
    int64_t acc = 0;
    float scale_sq = ix->l1_scale * ix->l1_scale;
    for (int i = 0; i < ix->dim; i++) {
        int d = ix->l1_bits == 4 ? (int)(qc[i] & 0x0f) - code4(x, i) : (int)qc[i] - (int)x[i];
        acc += (int64_t)(d * d);
    }
    return (float)acc * scale_sq;
}

/* retrieval_demo_exact_distance_residual_scalar,
 * retrieval_rpc_demo_support.c:1397-1443 */
float oracle_sq_exact(const OracleSqIndex *ix, const float *query, int id) {
    const uint8_t *l1 = ix->l1 + (size_t)id * ix->l1_code_bytes;
    const uint8_t *res = ix->residual ? ix->residual + (size_t)id * ix->residual_code_bytes : NULL;
    float rs = 0.0f, rz = 0.0f, dist = 0.0f;
    if (res) { rs = ix->qparams[2 * (size_t)id]; rz = ix->qparams[2 * (size_t)id + 1]; }
    for (int i = 0; i < ix->dim; i++) {
        int c = ix->l1_bits == 4 ? code4(l1, i) : l1[i];
        float value = (float)c * ix->l1_scale + ix->l1_zero;
        float diff;
        if (res) {
            int r = ix->residual_bits == 4 ? code4(res, i) : res[i];
            value += (float)r * rs + rz;
        }
        diff = query[i] - value;
        dist += diff * diff;
    }
    return dist;
}

/* demo_rerank_candidates (retrieval_rpc_demo_support.c:1833-1862) without a
 * reorder map: stable insertion sort of the candidates by id
 * (demo_sort_candidates_by_id :1776-1798), the exact residual distance of
 * each (FLT_MAX for an id outside the index, :1565-1567), stable insertion
 * sort by distance (demo_sort_candidates_by_distance :1800-1818), first
 * min(top_k, count).  ids/dists are scratch of count entries. */
int oracle_sq_rerank(const OracleSqIndex *ix, const float *query, int32_t *ids, float *dists, int count,
                     int top_k, int32_t *out_ids, float *out_dists) {
    int j, rc;
    if (!ix || !query || !ids || !dists || count < 0) return -1;
    for (j = 1; j < count; j++) {
        int32_t tid = ids[j];
        float tdt = dists[j];
        int k = j - 1;
        while (k >= 0 && !(ids[k] <= tid)) {
            ids[k + 1] = ids[k];
            dists[k + 1] = dists[k];
            k--;
        }
        ids[k + 1] = tid;
        dists[k + 1] = tdt;
    }
    for (j = 0; j < count; j++)
        dists[j] = (ids[j] < 0 || ids[j] >= ix->n) ? FLT_MAX : oracle_sq_exact(ix, query, ids[j]);
    for (j = 1; j < count; j++) {
        int32_t tid = ids[j];
        float tdt = dists[j];
        int k = j - 1;
        while (k >= 0 && dists[k] > tdt) {
            ids[k + 1] = ids[k];
            dists[k + 1] = dists[k];
            k--;
        }
        ids[k + 1] = tid;
        dists[k + 1] = tdt;
    }
    rc = top_k < count ? top_k : count;
    for (j = 0; j < rc; j++) {
        out_ids[j] = ids[j];
        out_dists[j] = dists[j];
    }
    return rc;
}

/* retrieval_sqmd_make_seed_ids, retrieval_sqmd_seed.c:15-63 */
int oracle_sq_seed_ids(int n, int entry_points, int graph_entry, uint32_t seed, int32_t *ids,
                       int capacity) {
    uint64_t limit, attempts = 0;
    int target = entry_points, count = 0;
    if (n <= 0 || entry_points <= 0 || capacity <= 0) return -1;
    if (target > capacity) target = capacity;
    if (target > n) target = n;
    if (graph_entry >= 0 && graph_entry < n) ids[count++] = graph_entry;
    limit = (uint64_t)target * 64u + 1024u;
    while (count < target && attempts < limit) {
        int id, dup = 0;
        seed = seed * 1103515245u + 12345u;
        id = (int)((seed / 65536u) % (uint32_t)n);
        attempts++;
        for (int i = 0; i < count; i++) if (ids[i] == id) { dup = 1; break; }
        if (dup) continue;
        ids[count++] = id;
    }
    for (int id = 0; count < target && id < n; id++) {
        int dup = 0;
        for (int i = 0; i < count; i++) if (ids[i] == id) { dup = 1; break; }
        if (!dup) ids[count++] = id;
    }
    return count;
}

/* SQ4 split distance ------------------------------------------------ */

/* retrieval_quantize_query_l1_aligned_u8, retrieval_l1_int8_core.c:65-111:
 * codes on the 4-bit L1 grid refined 17-fold, in double, lround, clamped. */
int oracle_split_query(const OracleSqIndex *ix, const float *query, OracleSplitQuery *out) {
    const double qs = (double)ix->l1_scale / 17.0;
    if (!query || !out || ix->dim <= 0 || ix->dim > 1024 || !isfinite(ix->l1_scale) ||
        !isfinite(ix->l1_zero) || ix->l1_scale <= 0.0f || !isfinite(qs) || qs <= 0.0)
        return -1;
    out->sum_q = 0;
    for (int i = 0; i < ix->dim; i++) {
        double raw = ((double)query[i] - (double)ix->l1_zero) / qs;
        long code;
        if (!isfinite(query[i]) || !isfinite(raw)) return -1;
        code = lround(raw);
        if (code < 0) code = 0;
        else if (code > 255) code = 255;
        out->q[i] = (uint8_t)code;
        out->sum_q += (uint64_t)code;
    }
    return 0;
}

/* retrieval_compute_u8_u4_l1_distance_scalar (:171-191) */
float oracle_split_coarse(const OracleSqIndex *ix, const OracleSplitQuery *sq, int id) {
    const uint8_t *x = ix->l1 + (size_t)id * ix->l1_code_bytes;
    const double qs = (double)ix->l1_scale / 17.0;
    int64_t acc = 0;
    if (ix->dim <= 0 || ix->dim > 33025 || !isfinite(ix->l1_scale) || ix->l1_scale <= 0.0f) return FLT_MAX;
    for (int i = 0; i < ix->dim; i++) {
        int32_t diff = (int32_t)sq->q[i] - 17 * (int32_t)code4(x, i);
        acc += (int64_t)diff * (int64_t)diff;
    }
    return (float)((double)acc * qs * qs);
}

/* sqmd_split_residual_delta_fn (retrieval_rpc_demo_pipeline.c:935-976) over
 * retrieval_compute_u8_u4 / u8_u8_residual_dot_scalar (:193-263):
 * bias[id] - 2 <q, r> with the dot product expanded over the integer sums. */
float oracle_split_delta(const OracleSqIndex *ix, const float *bias, const OracleSplitQuery *sq, int id) {
    const uint8_t *r = ix->residual + (size_t)id * ix->residual_code_bytes;
    const float rs = ix->qparams[2 * (size_t)id], rz = ix->qparams[2 * (size_t)id + 1];
    const double qs = (double)ix->l1_scale / 17.0;
    uint64_t sum_qv = 0, sum_v = 0;
    double dot, delta;
    if (!isfinite(ix->l1_scale) || !isfinite(ix->l1_zero) || !isfinite(rs) || !isfinite(rz) ||
        ix->l1_scale <= 0.0f || rs < 0.0f)
        return NAN;
    for (int i = 0; i < ix->dim; i++) {
        uint8_t v = ix->residual_bits == 4 ? (uint8_t)code4(r, i) : r[i];
        sum_qv += (uint64_t)sq->q[i] * (uint64_t)v;
        sum_v += (uint64_t)v;
    }
    dot = qs * (double)rs * (double)sum_qv + qs * (double)rz * (double)sq->sum_q +
          (double)ix->l1_zero * (double)rs * (double)sum_v +
          (double)ix->dim * (double)ix->l1_zero * (double)rz;
    delta = (double)bias[id] - 2.0 * dot;
    return isfinite(delta) ? (float)delta : NAN;
}

/* sqmd_split_distance_for_id (retrieval_rpc_demo_pipeline.c:978-995): the
 * seeds' distance; FLT_MAX when either part is not finite. */
float oracle_split_distance(const OracleSqIndex *ix, const float *bias, const OracleSplitQuery *sq, int id) {
    float coarse = oracle_split_coarse(ix, sq, id);
    float delta = oracle_split_delta(ix, bias, sq, id);
    if (!isfinite(coarse) || !isfinite(delta)) return FLT_MAX;
    coarse += delta;
    if (coarse < 0.0f && coarse > -1.0e-4f) coarse = 0.0f;
    return coarse;
}

/* Distance-only heaps with the reference's tie behaviour:
 * sqmd_heap_sift_up/down, sqmd_frontier_*, sqmd_candidate_insert,
 * sqmd_heap_sort (retrieval_sqmd_common.c:9-144); the DSP copies
 * (retrieval_async_dsp_search.c:101-217) are identical. */
static void sq_pool_up(Cand *p, int i) {
    Cand t = p[i];
    while (i > 0) {
        int parent = (i - 1) / 2;
        if (t.dist <= p[parent].dist) break;
        p[i] = p[parent];
        i = parent;
    }
    p[i] = t;
}

static void sq_pool_down(Cand *p, int size, int i) {
    Cand t = p[i];
    for (;;) {
        int child = 2 * i + 1;
        if (child >= size) break;
        if (child + 1 < size && p[child + 1].dist > p[child].dist) child++;
        if (t.dist >= p[child].dist) break;
        p[i] = p[child];
        i = child;
    }
    p[i] = t;
}

static int sq_pool_insert(Cand *p, int *size, int cap, int id, float dist) {
    if (*size < cap) {
        p[*size].id = id; p[*size].dist = dist;
        sq_pool_up(p, *size);
        (*size)++;
        return 1;
    }
    if (dist < p[0].dist) {
        p[0].id = id; p[0].dist = dist;
        sq_pool_down(p, *size, 0);
        return 1;
    }
    return 0;
}

static void sq_heap_sort(Cand *p, int size) {
    for (int i = size - 1; i > 0; i--) {
        Cand t = p[0]; p[0] = p[i]; p[i] = t;
        sq_pool_down(p, i, 0);
    }
}

static void sq_front_up(Cand *f, int i) {
    Cand t = f[i];
    while (i > 0) {
        int parent = (i - 1) / 2;
        if (t.dist >= f[parent].dist) break;
        f[i] = f[parent];
        i = parent;
    }
    f[i] = t;
}

static void sq_front_down(Cand *f, int size, int i) {
    Cand t = f[i];
    for (;;) {
        int child = 2 * i + 1;
        if (child >= size) break;
        if (child + 1 < size && f[child + 1].dist < f[child].dist) child++;
        if (t.dist <= f[child].dist) break;
        f[i] = f[child];
        i = child;
    }
    f[i] = t;
}

static int sq_front_pop(Cand *f, int *size) {
    int top = f[0].id;
    (*size)--;
    if (*size > 0) { f[0] = f[*size]; sq_front_down(f, *size, 0); }
    return top;
}

/*
 * SQMD search as the CLI runs it with a window of one source per turn:
 * sqmd_cpu_state_seed (retrieval_sqmd_common.c:446), the turn loop of
 * sqmd_cpu_state_run_fake_dsp (:2052-2152) with
 * sqmd_cpu_state_try_peek_source (:478), sqmd_dispatch_neighbors_to_lanes
 * (:283-383) and sqmd_cpu_state_apply_results_with_correction (:638-708);
 * seeds and seed distances from sqmd_make_seed (pipeline.c:1013-1055).
 * stats: {work_items, exact_corrected, turns, dedup_skips}.
 */
static int sqmd_search_core(const OracleSqIndex *ix, const float *bias, const float *query,
                            int entry_points, int graph_entry, uint32_t seed, int expand_count,
                            int pool_capacity, int correction, int32_t *out_ids, float *out_dists,
                            int out_capacity, uint64_t *stats) {
    int n = ix->n, pool_size = 0, front_size = 0, result = -1, seed_count;
    size_t front_cap = (size_t)entry_points + (size_t)pool_capacity * (size_t)expand_count;
    int expand = expand_count < ix->degree ? expand_count : ix->degree;
    uint64_t work = 0, corrected = 0, turns = 0, dedup = 0;
    uint8_t qc[1024];
    OracleSplitQuery split;
    Cand *pool = calloc((size_t)pool_capacity, sizeof(Cand));
    Cand *front = calloc(front_cap ? front_cap : 1, sizeof(Cand));
    uint32_t *visited = calloc(((size_t)n + 31) / 32, sizeof(uint32_t));
    int32_t *seeds = malloc((size_t)entry_points * sizeof(int32_t));
    int32_t wl[32];
    if (!pool || !front || !visited || !seeds || ix->dim > 1024 || pool_capacity <= 0 ||
        entry_points <= 0 || expand_count <= 0 || oracle_sq_quantize(ix, query, qc) != 0)
        goto done;
    /* sqmd_split_query_init (pipeline.c:916-933): 4-bit codes, residuals */
    if (bias && (!correction || ix->l1_bits != 4 || !ix->residual || !ix->qparams ||
                 oracle_split_query(ix, query, &split) != 0))
        goto done;
    seed_count = oracle_sq_seed_ids(n, entry_points, graph_entry, seed, seeds, entry_points);
    if (seed_count <= 0) goto done;
    for (int i = 0; i < seed_count; i++) {
        int id = seeds[i];
        float d;
        if (correction) {
            d = bias ? oracle_split_distance(ix, bias, &split, id) : oracle_sq_exact(ix, query, id);
            if (!isfinite(d) || d < 0.0f) goto done;
        } else {
            d = oracle_sq_coarse(ix, qc, id);
        }
        if (visited[id >> 5] & (1u << (id & 31))) continue;
        visited[id >> 5] |= 1u << (id & 31);
        if (sq_pool_insert(pool, &pool_size, pool_capacity, id, d) && (size_t)front_size < front_cap) {
            front[front_size].id = id; front[front_size].dist = d;
            sq_front_up(front, front_size++);
        }
    }
    for (;;) {
        int src, nw = 0;
        const int32_t *row;
        while (front_size > 0 && pool_size >= pool_capacity && front[0].dist > pool[0].dist)
            sq_front_pop(front, &front_size);
        if (front_size <= 0) break;
        src = sq_front_pop(front, &front_size);
        if (expand > 32) goto done; /* SQMD_STATUS_TOO_MUCH_WORK */
        row = ix->graph + (size_t)src * ix->degree;
        for (int j = 0; j < expand; j++) {
            int id = row[j], dup = 0;
            if (id < 0 || id >= n || id == src) continue;
            for (int w = 0; w < nw; w++) if (wl[w] == id) { dup = 1; break; }
            if (dup || (visited[id >> 5] & (1u << (id & 31)))) { dedup++; continue; }
            wl[nw++] = id;
        }
        turns++;
        work += (uint64_t)nw;
        for (int w = 0; w < nw; w++) visited[wl[w] >> 5] |= 1u << (wl[w] & 31);
        for (int w = 0; w < nw; w++) {
            float d = oracle_sq_coarse(ix, qc, wl[w]);
            if (bias) {
                /* sqmd_source_job_commit (sqmd_common.c:1533-1556): the
                 * lane's split coarse distance plus the host's delta */
                float delta = oracle_split_delta(ix, bias, &split, wl[w]);
                if (!isfinite(delta)) goto done;
                d = oracle_split_coarse(ix, &split, wl[w]) + delta;
                if (d < 0.0f && d > -1.0e-4f) d = 0.0f;
                if (!isfinite(d) || d < 0.0f) goto done;
            } else if (correction) {
                d = oracle_sq_exact(ix, query, wl[w]);
            }
            if (sq_pool_insert(pool, &pool_size, pool_capacity, wl[w], d) &&
                (size_t)front_size < front_cap) {
                front[front_size].id = wl[w]; front[front_size].dist = d;
                sq_front_up(front, front_size++);
            }
            corrected++;
        }
    }
    sq_heap_sort(pool, pool_size);
    result = pool_size < out_capacity ? pool_size : out_capacity;
    for (int i = 0; i < result; i++) { out_ids[i] = pool[i].id; out_dists[i] = pool[i].dist; }
    if (stats) { stats[0] = work; stats[1] = corrected; stats[2] = turns; stats[3] = dedup; }
done:
    free(pool); free(front); free(visited); free(seeds);
    return result;
}

int oracle_sqmd_search(const OracleSqIndex *ix, const float *query, int entry_points,
                       int graph_entry, uint32_t seed, int expand_count, int pool_capacity,
                       int correction, int32_t *out_ids, float *out_dists, int out_capacity,
                       uint64_t *stats) {
    return sqmd_search_core(ix, NULL, query, entry_points, graph_entry, seed, expand_count, pool_capacity,
                            correction, out_ids, out_dists, out_capacity, stats);
}

/* The SQMD session path with SQMD_SPLIT_DISTANCE on
 * (sqmd_cpu_state_run_source_pipeline_split, sqmd_common.c:2028-2050). */
int oracle_sqmd_search_split(const OracleSqIndex *ix, const float *bias, const float *query,
                             int entry_points, int graph_entry, uint32_t seed, int expand_count,
                             int pool_capacity, int32_t *out_ids, float *out_dists, int out_capacity,
                             uint64_t *stats) {
    if (!bias) return -1;
    return sqmd_search_core(ix, bias, query, entry_points, graph_entry, seed, expand_count, pool_capacity,
                            1, out_ids, out_dists, out_capacity, stats);
}

/*
 * Legacy device search, calculator_retrieval_search
 * (retrieval_async_dsp_search.c:368-509): entries from
 * dsp_search_select_entry_id (:219-230, seed 42), SQ coarse distances, the
 * same distance-only heaps; neighbours outside [0, n) are skipped one by one.
 */
int oracle_dsp_search(const OracleSqIndex *ix, const float *query, int entry_points,
                      int graph_entry, int expand_count, int pool_size, int num_out,
                      int32_t *out_ids, float *out_dists) {
    int n = ix->n, ps = 0, fs = 0, result = -1;
    int expand = expand_count < ix->degree ? expand_count : ix->degree;
    uint32_t seed = 42u;
    size_t fcap;
    uint8_t qc[1024];
    Cand *pool, *front;
    uint32_t *visited;
    if (pool_size <= 0 || num_out <= 0 || expand <= 0 || ix->dim > 1024) return -1;
    if (pool_size > 2000) pool_size = 2000;
    fcap = (size_t)(entry_points > 0 ? entry_points : 0) + (size_t)n * (size_t)expand + 1;
    pool = malloc(2000 * sizeof(Cand));
    front = malloc(fcap * sizeof(Cand));
    visited = calloc(((size_t)n + 31) / 32, sizeof(uint32_t));
    if (!pool || !front || !visited || oracle_sq_quantize(ix, query, qc) != 0) goto done;
    for (int i = 0; i < entry_points && i < n; i++) {
        int id;
        float d;
        if (i == 0 && graph_entry >= 0 && graph_entry < n) {
            id = graph_entry;
        } else {
            seed = seed * 1103515245u + 12345u;
            id = (int)(((uint64_t)seed * (uint64_t)n) >> 32);
        }
        if (visited[id >> 5] & (1u << (id & 31))) continue;
        visited[id >> 5] |= 1u << (id & 31);
        d = oracle_sq_coarse(ix, qc, id);
        if (sq_pool_insert(pool, &ps, pool_size, id, d)) {
            front[fs].id = id; front[fs].dist = d; sq_front_up(front, fs++);
        }
    }
    while (fs > 0) {
        int cur;
        const int32_t *row;
        if (ps >= pool_size && front[0].dist > pool[0].dist) { sq_front_pop(front, &fs); continue; }
        cur = sq_front_pop(front, &fs);
        row = ix->graph + (size_t)cur * ix->degree;
        for (int j = 0; j < expand; j++) {
            int id = row[j];
            float d;
            if (id < 0 || id >= n) continue;
            if (visited[id >> 5] & (1u << (id & 31))) continue;
            visited[id >> 5] |= 1u << (id & 31);
            d = oracle_sq_coarse(ix, qc, id);
            if (sq_pool_insert(pool, &ps, pool_size, id, d)) {
                front[fs].id = id; front[fs].dist = d; sq_front_up(front, fs++);
            }
        }
    }
    sq_heap_sort(pool, ps);
    result = num_out < ps ? num_out : ps;
    for (int i = 0; i < result; i++) { out_ids[i] = pool[i].id; out_dists[i] = pool[i].dist; }
done:
    free(pool); free(front); free(visited);
    return result;
}

/* ------------------------------------------------------------------ */
/* final refine, refine_impl (retrieval_final_refine.c:256-292), mode  */
/* CURRENT, no order maps (graph id == original id == storage row).    */

typedef struct { int32_t id; double dist; } RefineItem;

static int refine_by_id(const void *a, const void *b) {
    const RefineItem *x = (const RefineItem *)a, *y = (const RefineItem *)b;
    return (x->id > y->id) - (x->id < y->id);
}

static int refine_by_dist(const void *a, const void *b) {
    const RefineItem *x = (const RefineItem *)a, *y = (const RefineItem *)b;
    if (x->dist != y->dist) return x->dist < y->dist ? -1 : 1;
    return (x->id > y->id) - (x->id < y->id);
}

/* decode_value / add_f32 / retrieval_final_refine_decode_sq,
 * retrieval_final_refine.c:46-67 */
static inline float refine_decode_value(unsigned code, float scale, float zero) {
    volatile float product = (float)code * scale;
    volatile float value = product + zero;
    return value;
}

static int refine_decode_sq(const OracleSqIndex *ix, int id, float *out) {
    const uint8_t *l1 = ix->l1 + (size_t)id * ix->l1_code_bytes;
    const uint8_t *r = ix->residual + (size_t)id * ix->residual_code_bytes;
    float rs = ix->qparams[2 * (size_t)id], rz = ix->qparams[2 * (size_t)id + 1];
    if (!isfinite(ix->l1_scale) || ix->l1_scale <= 0 || !isfinite(ix->l1_zero) ||
        !isfinite(rs) || rs < 0 || !isfinite(rz))
        return -1;
    for (int d = 0; d < ix->dim; d++) {
        unsigned a = ix->l1_bits == 4 ? (unsigned)code4(l1, d) : l1[d];
        unsigned b = ix->residual_bits == 4 ? (unsigned)code4(r, d) : r[d];
        volatile float v = refine_decode_value(a, ix->l1_scale, ix->l1_zero) +
                           refine_decode_value(b, rs, rz);
        out[d] = v;
        if (!isfinite(out[d])) return -1;
    }
    return 0;
}

/* decode_vector's ERROR4 term (retrieval_final_refine.c:221-246): the
 * storage row's int4 code, scale and zero added to the base decode, each
 * product and sum rounded to float; the row is the graph id here (no
 * storage map). */
static int refine_add_error4(const OracleError4 *e4, int row, int dim, float *v) {
    const uint8_t *codes = e4->blocks + (size_t)(row / e4->vectors_per_block) * 4096u +
                           (size_t)(row % e4->vectors_per_block) * (size_t)e4->code_bytes;
    float s = e4->qparams[2 * (size_t)row], z = e4->qparams[2 * (size_t)row + 1];
    for (int d = 0; d < dim; d++) {
        volatile float value = v[d] + refine_decode_value((unsigned)code4(codes, d), s, z);
        if (!isfinite(value)) return -1;
        v[d] = value;
    }
    return 0;
}

int oracle_refine(int kind, const void *index, const float *query, const int32_t *ids,
                  int count, int output_k, int32_t *out_ids, float *out_dists) {
    return oracle_refine_ex(kind, index, NULL, query, ids, count, output_k, out_ids, out_dists);
}

int oracle_refine_ex(int kind, const void *index, const OracleError4 *e4, const float *query,
                     const int32_t *ids, int count, int output_k, int32_t *out_ids, float *out_dists) {
    int dim = kind == 0 ? ((const OracleSqIndex *)index)->dim : ((const OraclePqIndex *)index)->dim;
    int n = kind == 0 ? ((const OracleSqIndex *)index)->n : ((const OraclePqIndex *)index)->n;
    RefineItem *items = malloc((size_t)(count > 0 ? count : 1) * sizeof(RefineItem));
    float *v = malloc((size_t)dim * sizeof(float));
    int rc = -1;
    if (!items || !v || count < 0 || output_k <= 0) goto done;
    for (int d = 0; d < dim; d++) if (!isfinite(query[d])) goto done;
    for (int i = 0; i < count; i++) {
        if (ids[i] < 0 || ids[i] >= n) goto done;
        items[i].id = ids[i];
    }
    qsort(items, (size_t)count, sizeof(RefineItem), refine_by_id);
    for (int i = 1; i < count; i++) if (items[i].id == items[i - 1].id) goto done;
    for (int i = 0; i < count; i++) {
        int drc = kind == 0 ? refine_decode_sq((const OracleSqIndex *)index, items[i].id, v)
                            : oracle_pq_decode((const OraclePqIndex *)index, items[i].id, v);
        if (drc != 0) goto done;
        if (e4 && refine_add_error4(e4, items[i].id, dim, v) != 0) goto done;
        items[i].dist = 0;
        for (int d = 0; d < dim; d++) {
            double delta = (double)query[d] - (double)v[d];
            items[i].dist += delta * delta;
        }
        if (!isfinite(items[i].dist) || items[i].dist >= FLT_MAX) goto done;
    }
    qsort(items, (size_t)count, sizeof(RefineItem), refine_by_dist);
    rc = count < output_k ? count : output_k;
    for (int i = 0; i < rc; i++) { out_ids[i] = items[i].id; out_dists[i] = (float)items[i].dist; }
done:
    free(items); free(v);
    return rc;
}

/* ------------------------------------------------------------------ */
/* batch helper                                                        */

typedef struct {
    const OraclePqIndex *ix;
    const float *queries;
    const int32_t *pool_sizes;
    int nq, entry_points, graph_entry, expand_count, correction, refine_budget, top_k;
    uint32_t seed;
    int32_t *pool_ids; float *pool_dists; int pool_stride; int32_t *pool_counts;
    int32_t *out_ids; float *out_dists; int out_stride; int32_t *out_counts;
    uint64_t *stats;
    int next, failed;
    pthread_mutex_t lock;
} PqJob;

static void *pq_job_main(void *p) {
    PqJob *j = (PqJob *)p;
    int32_t *seeds = malloc((size_t)(j->entry_points > 0 ? j->entry_points : 1) * sizeof(int32_t));
    int max_pool = 1;
    for (int i = 0; i < j->nq; i++) if (j->pool_sizes[i] > max_pool) max_pool = j->pool_sizes[i];
    int32_t *ids = malloc((size_t)max_pool * sizeof(int32_t));
    float *dists = malloc((size_t)max_pool * sizeof(float));
    for (;;) {
        int q, count, sc;
        pthread_mutex_lock(&j->lock);
        q = j->failed ? j->nq : j->next++;
        pthread_mutex_unlock(&j->lock);
        if (q >= j->nq) break;
        const float *query = j->queries + (size_t)q * j->ix->dim;
        int pool = j->pool_sizes[q];
        sc = oracle_pq_seed_ids(j->ix->n, j->entry_points, j->graph_entry, j->seed, seeds);
        count = oracle_pq_search(j->ix, query, seeds, sc, j->expand_count, pool, pool,
                                 j->correction, ids, dists, j->stats ? j->stats + (size_t)q * 4 : NULL);
        if (count >= 0 && j->pool_ids) {
            for (int i = 0; i < count && i < j->pool_stride; i++) {
                j->pool_ids[(size_t)q * j->pool_stride + i] = ids[i];
                j->pool_dists[(size_t)q * j->pool_stride + i] = dists[i];
            }
            if (j->pool_counts) j->pool_counts[q] = count;
        }
        if (count >= 0 && j->out_ids) {
            int fc;
            if (j->refine_budget > 0) {
                int sel = count < j->refine_budget ? count : j->refine_budget;
                fc = oracle_refine(1, j->ix, query, ids, sel, j->top_k,
                                   j->out_ids + (size_t)q * j->out_stride,
                                   j->out_dists + (size_t)q * j->out_stride);
            } else {
                fc = count < j->top_k ? count : j->top_k;
                for (int i = 0; i < fc; i++) {
                    j->out_ids[(size_t)q * j->out_stride + i] = ids[i];
                    j->out_dists[(size_t)q * j->out_stride + i] = dists[i];
                }
            }
            if (fc < 0) count = -1;
            else if (j->out_counts) j->out_counts[q] = fc;
        }
        if (count < 0) {
            pthread_mutex_lock(&j->lock);
            if (!j->failed) j->failed = q + 1;
            pthread_mutex_unlock(&j->lock);
        }
    }
    free(seeds); free(ids); free(dists);
    return NULL;
}

int oracle_pq_search_batch(const OraclePqIndex *ix, const float *queries, int nq,
                           const int32_t *pool_sizes, int entry_points, int graph_entry,
                           uint32_t seed, int expand_count, int correction, int refine_budget,
                           int top_k, int threads, int32_t *pool_ids, float *pool_dists,
                           int pool_stride, int32_t *pool_counts, int32_t *out_ids,
                           float *out_dists, int out_stride, int32_t *out_counts,
                           uint64_t *stats) {
    PqJob j;
    pthread_t tid[256];
    int t;
    memset(&j, 0, sizeof(j));
    j.ix = ix; j.queries = queries; j.pool_sizes = pool_sizes; j.nq = nq;
    j.entry_points = entry_points; j.graph_entry = graph_entry; j.expand_count = expand_count;
    j.correction = correction; j.refine_budget = refine_budget; j.top_k = top_k; j.seed = seed;
    j.pool_ids = pool_ids; j.pool_dists = pool_dists; j.pool_stride = pool_stride;
    j.pool_counts = pool_counts; j.out_ids = out_ids; j.out_dists = out_dists;
    j.out_stride = out_stride; j.out_counts = out_counts; j.stats = stats;
    pthread_mutex_init(&j.lock, NULL);
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    for (t = 0; t < threads; t++)
        if (pthread_create(&tid[t], NULL, pq_job_main, &j) != 0) break;
    for (int i = 0; i < t; i++) pthread_join(tid[i], NULL);
    pthread_mutex_destroy(&j.lock);
    return j.failed;
}
