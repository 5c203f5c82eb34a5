/*
 * ref_harness.c -- batch driver around the UNMODIFIED reference functions
 * (test infrastructure: the oracle and the timed CPU baseline).
 *
 * Every distance, search, correction and refine below is computed by the
 * reference's own code linked from oracle/_ref/libref_host.so and
 * libref_dsp.so.  This file only
 *   - opens the reference's artifacts with the reference loaders,
 *   - restates two tiny static helpers the reference keeps private
 *     (PQ seed ids, retrieval_rpc_demo_pure_pq.c:192-208; the fake-DSP
 *     distance/correction callbacks, retrieval_rpc_demo_pipeline.c:881-1011),
 *   - fans independent queries out over POSIX threads (the reference itself
 *     runs one query at a time; queries share no state).
 */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "rover_config.h"
#include "dsp_demo/retrieval_final_refine.h"
#include "dsp_demo/retrieval_l1_int8_core.h"
#include "dsp_demo/retrieval_pq_artifact.h"
#include "dsp_demo/retrieval_pq_core.h"
#include "dsp_demo/retrieval_pq_residual.h"
#include "dsp_demo/retrieval_rpc_demo.h"
#include "dsp_demo/retrieval_sqmd_common.h"
#include "dsp_demo/retrieval_sqmd_pure_pq.h"
#include "dsp_demo/retrieval_sqmd_seed.h"
#include "calculator.h"

#define HARNESS_MAX_CHUNKS 64

/* ------------------------------------------------------------------ */
/* thread fan-out                                                      */

typedef struct {
    int count;
    int next;
    int failed;
    pthread_mutex_t lock;
    int (*fn)(void *ctx, int worker, int item);
    void *ctx;
} Fanout;

typedef struct { Fanout *f; int worker; } FanoutArg;

static void *fanout_main(void *p) {
    FanoutArg *a = (FanoutArg *)p;
    Fanout *f = a->f;
    for (;;) {
        int item;
        pthread_mutex_lock(&f->lock);
        item = f->failed ? f->count : f->next++;
        pthread_mutex_unlock(&f->lock);
        if (item >= f->count) break;
        if (f->fn(f->ctx, a->worker, item) != 0) {
            pthread_mutex_lock(&f->lock);
            if (!f->failed) f->failed = item + 1;
            pthread_mutex_unlock(&f->lock);
        }
    }
    return NULL;
}

/* Returns 0, or (1 + index of the first failing item). */
static int fanout_run(int count, int threads, int (*fn)(void *, int, int), void *ctx) {
    Fanout f;
    pthread_t tid[256];
    FanoutArg args[256];
    int t;
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    if (threads > count) threads = count > 0 ? count : 1;
    memset(&f, 0, sizeof(f));
    f.count = count; f.fn = fn; f.ctx = ctx;
    pthread_mutex_init(&f.lock, NULL);
    for (t = 0; t < threads; t++) {
        args[t].f = &f; args[t].worker = t;
        if (pthread_create(&tid[t], NULL, fanout_main, &args[t]) != 0) { threads = t; break; }
    }
    for (t = 0; t < threads; t++) pthread_join(tid[t], NULL);
    pthread_mutex_destroy(&f.lock);
    return f.failed;
}

/* ------------------------------------------------------------------ */
/* pure PQ                                                             */

typedef struct {
    RetrievalPqArtifacts artifacts;
    RetrievalPqResidualIndex *residual;
    const uint8_t *chunks[HARNESS_MAX_CHUNKS];
    int chunk_counts[HARNESS_MAX_CHUNKS];
    int chunk_count;
    int chunk_vectors;
    int residual_bits;
} RefPq;

/* Load <prefix>.pqbook/.pqcodes with retrieval_pq_artifacts_load and, when
 * residual_bits > 0, <prefix>.pqresN(.qparams) with
 * retrieval_pq_residual_index_open in memory mode (rover_config.disk = 0,
 * retrieval_pq_residual.c:807-812).  Codes are split into chunk_vectors-sized
 * chunks the way retrieval_pure_pq_index.c does. */
int ref_pq_open(const char *prefix, int residual_bits, int chunk_vectors, void **out) {
    RefPq *h;
    uint64_t n, start;
    if (!prefix || !out || chunk_vectors <= 0) return -1;
    *out = NULL;
    h = (RefPq *)calloc(1, sizeof(*h));
    if (!h) return -1;
    if (retrieval_pq_artifacts_load(prefix, &h->artifacts) != 0) { free(h); return -2; }
    n = h->artifacts.metadata.num_vectors;
    h->chunk_vectors = chunk_vectors;
    for (start = 0; start < n; start += (uint64_t)chunk_vectors) {
        uint64_t count = n - start < (uint64_t)chunk_vectors ? n - start : (uint64_t)chunk_vectors;
        if (h->chunk_count >= HARNESS_MAX_CHUNKS) { retrieval_pq_artifacts_release(&h->artifacts); free(h); return -3; }
        h->chunks[h->chunk_count] = h->artifacts.codes + start * h->artifacts.metadata.code_bytes;
        h->chunk_counts[h->chunk_count] = (int)count;
        h->chunk_count++;
    }
    h->residual_bits = residual_bits;
    if (residual_bits > 0) {
        RetrievalPqResidualOpenRequest request;
        memset(&request, 0, sizeof(request));
        rover_config.disk = 0;
        request.artifact_prefix = prefix;
        request.residual_bits = residual_bits;
        request.cache_slots = 2048;
        request.pq_metadata = &h->artifacts.metadata;
        request.codebook = h->artifacts.codebook;
        request.code_chunks = h->chunks;
        request.chunk_vector_counts = h->chunk_counts;
        request.chunk_count = h->chunk_count;
        request.chunk_vectors = h->chunk_vectors;
        if (retrieval_pq_residual_index_open(&request, &h->residual) != 0) {
            retrieval_pq_artifacts_release(&h->artifacts); free(h); return -4;
        }
    }
    *out = h;
    return 0;
}

void ref_pq_close(void *p) {
    RefPq *h = (RefPq *)p;
    if (!h) return;
    retrieval_pq_residual_index_close(h->residual);
    retrieval_pq_artifacts_release(&h->artifacts);
    free(h);
}

/* info = {n, dim, m, ks, subdim, code_bytes} */
int ref_pq_info(void *p, int32_t *info) {
    RefPq *h = (RefPq *)p;
    if (!h || !info) return -1;
    info[0] = (int32_t)h->artifacts.metadata.num_vectors;
    info[1] = (int32_t)h->artifacts.metadata.dim;
    info[2] = (int32_t)h->artifacts.metadata.m;
    info[3] = (int32_t)h->artifacts.metadata.ks;
    info[4] = (int32_t)h->artifacts.metadata.subdim;
    info[5] = (int32_t)h->artifacts.metadata.code_bytes;
    return 0;
}

const float *ref_pq_codebook(void *p) { return p ? ((RefPq *)p)->artifacts.codebook : NULL; }
const uint8_t *ref_pq_codes(void *p) { return p ? ((RefPq *)p)->artifacts.codes : NULL; }

/* retrieval_pq_build_lut, pq_core.c:362 */
int ref_pq_lut(void *p, const float *query, float *lut) {
    RefPq *h = (RefPq *)p;
    if (!h) return -1;
    return retrieval_pq_build_lut(query, h->artifacts.codebook, (int)h->artifacts.metadata.m,
                                  (int)h->artifacts.metadata.ks, (int)h->artifacts.metadata.subdim, lut);
}

/* retrieval_pq_adc_ids_batch_scalar, pq_core.c:347 */
int ref_pq_adc(void *p, const float *lut, const int32_t *ids, int count, float *out) {
    RefPq *h = (RefPq *)p;
    if (!h) return -1;
    return retrieval_pq_adc_ids_batch_scalar(h->chunks, h->chunk_counts, h->chunk_count,
                                             h->chunk_vectors, ids, count, lut,
                                             (int)h->artifacts.metadata.m,
                                             (int)h->artifacts.metadata.ks, out);
}

/* retrieval_pq_residual_query_evaluate, pq_residual.c:983 */
int ref_pq_residual_eval(void *p, const float *query, const int32_t *ids, int count, float *out) {
    RefPq *h = (RefPq *)p;
    RetrievalPqResidualQuery *q = NULL;
    int i, rc = 0;
    if (!h || !h->residual || retrieval_pq_residual_query_create(h->residual, &q) != 0) return -1;
    retrieval_pq_residual_query_bind(q, query);
    for (i = 0; i < count && rc == 0; i++)
        rc = retrieval_pq_residual_query_evaluate(q, ids[i], 0.0f, &out[i]);
    retrieval_pq_residual_query_destroy(q);
    return rc;
}

/* retrieval_pq_residual_query_decode, pq_residual.c:954 */
int ref_pq_residual_decode(void *p, int id, float *out) {
    RefPq *h = (RefPq *)p;
    RetrievalPqResidualQuery *q = NULL;
    int rc;
    if (!h || !h->residual || retrieval_pq_residual_query_create(h->residual, &q) != 0) return -1;
    rc = retrieval_pq_residual_query_decode(q, id, out);
    retrieval_pq_residual_query_destroy(q);
    return rc;
}

/* Seed ids of the pure-PQ CLI driver: graph entry first, then the LCG
 * seed = seed*1103515245 + 12345, id = (seed * N) >> 32; restated from the
 * static pure_pq_make_seed_ids, retrieval_rpc_demo_pure_pq.c:192-208. */
static int harness_pq_seed_ids(int num_vectors, int entry_count, int graph_entry,
                               unsigned int seed, int *seed_ids) {
    int count = entry_count < num_vectors ? entry_count : num_vectors;
    int index;
    for (index = 0; index < count; index++) {
        if (index == 0 && graph_entry >= 0 && graph_entry < num_vectors) {
            seed_ids[index] = graph_entry;
        } else {
            seed = seed * 1103515245u + 12345u;
            seed_ids[index] = (int)(((uint64_t)seed * (uint64_t)num_vectors) >> 32);
        }
    }
    return count;
}

int ref_pq_seed_ids(int num_vectors, int entry_count, int graph_entry, unsigned int seed,
                    int *seed_ids) {
    return harness_pq_seed_ids(num_vectors, entry_count, graph_entry, seed, seed_ids);
}

typedef struct {
    RefPq *h;
    const int32_t *graph;
    int degree, graph_entry;
    const float *queries;
    const int32_t *pool_sizes;
    int entry_points, expand_count, correction, refine_budget, top_k;
    unsigned int seed;
    int32_t *pool_ids; float *pool_dists; int pool_stride; int32_t *pool_counts;
    int32_t *out_ids; float *out_dists; int out_stride; int32_t *out_counts;
    uint64_t *stats;
    RetrievalPqResidualQuery **queries_res;
    RetrievalFinalRefineContext **refine;
    int *scratch_ids; float *scratch_dists; int scratch_stride;
} PqBatch;

static int harness_pq_decode(void *provider, int id, float *out) {
    return retrieval_pq_residual_query_decode((RetrievalPqResidualQuery *)provider, id, out);
}

static int harness_pq_evaluator(void *context, int id, float coarse, float *out) {
    return retrieval_pq_residual_query_evaluate((RetrievalPqResidualQuery *)context, id, coarse, out);
}

static int pq_batch_item(void *ctx, int worker, int qi) {
    PqBatch *b = (PqBatch *)ctx;
    RefPq *h = b->h;
    const RetrievalPqArtifactMetadata *md = &h->artifacts.metadata;
    const float *query = b->queries + (size_t)qi * md->dim;
    int pool = b->pool_sizes[qi];
    int *ids = b->scratch_ids + (size_t)worker * b->scratch_stride;
    float *dists = b->scratch_dists + (size_t)worker * b->scratch_stride;
    int seeds[4096];
    PurePqSearchIndexView view;
    PurePqSearchRequest request;
    PurePqDistancePolicy policy;
    PurePqSearchStats stats;
    int seed_count, count, i;
    if (pool <= 0 || pool > b->scratch_stride || b->entry_points > 4096) return -1;
    seed_count = harness_pq_seed_ids((int)md->num_vectors, b->entry_points, b->graph_entry,
                                     b->seed, seeds);
    memset(&view, 0, sizeof(view));
    view.graph = b->graph; view.graph_degree = b->degree; view.num_vectors = (int)md->num_vectors;
    view.code_chunks = h->chunks; view.chunk_vector_counts = h->chunk_counts;
    view.chunk_count = h->chunk_count; view.chunk_vectors = h->chunk_vectors;
    view.codebook = h->artifacts.codebook; view.dim = (int)md->dim; view.m = (int)md->m;
    view.ks = (int)md->ks; view.subdim = (int)md->subdim;
    memset(&request, 0, sizeof(request));
    request.query = query; request.entry_ids = seeds; request.entry_count = seed_count;
    request.expand_count = b->expand_count; request.pool_capacity = pool; request.num_out = pool;
    memset(&policy, 0, sizeof(policy));
    if (b->correction) {
        RetrievalPqResidualQuery *rq = b->queries_res[worker];
        if (!rq || retrieval_pq_residual_query_bind(rq, query) != 0) return -1;
        policy.mode = PURE_PQ_CORRECTION_ONLINE;
        policy.evaluator = harness_pq_evaluator;
        policy.context = rq;
    }
    count = retrieval_pure_pq_search_scalar_with_policy(&view, &request, b->correction ? &policy : NULL,
                                                        ids, dists, pool, &stats);
    if (count < 0) return -1;
    if (b->stats) {
        uint64_t *s = b->stats + (size_t)qi * 4;
        s[0] = stats.pq_scored_candidates; s[1] = stats.corrected_candidates;
        s[2] = stats.expanded_nodes; s[3] = stats.visited_dedup_skips;
    }
    if (b->pool_ids) {
        for (i = 0; i < count && i < b->pool_stride; i++) {
            b->pool_ids[(size_t)qi * b->pool_stride + i] = ids[i];
            b->pool_dists[(size_t)qi * b->pool_stride + i] = dists[i];
        }
        if (b->pool_counts) b->pool_counts[qi] = count;
    }
    if (b->out_ids) {
        int final_count;
        if (b->refine_budget > 0) {
            int selected = count < b->refine_budget ? count : b->refine_budget;
            RetrievalFinalRefineContext *rc = b->refine[worker];
            if (!rc) return -1;
            final_count = retrieval_final_refine(rc, query, ids, dists, selected, b->top_k, NULL);
            if (final_count < 0) return -1;
        } else {
            final_count = count < b->top_k ? count : b->top_k;
        }
        for (i = 0; i < final_count && i < b->out_stride; i++) {
            b->out_ids[(size_t)qi * b->out_stride + i] = ids[i];
            b->out_dists[(size_t)qi * b->out_stride + i] = dists[i];
        }
        if (b->out_counts) b->out_counts[qi] = final_count;
    }
    return 0;
}

/*
 * Batched pure-PQ search through the reference's scalar search
 * (retrieval_pure_pq_search_scalar_with_policy, sqmd_pure_pq.c:793) with the
 * ONLINE residual policy (retrieval_pq_residual_query_evaluate) when
 * correction != 0, then the reference final refine (retrieval_final_refine,
 * final_refine.c:294, mode CURRENT with the residual decode provider) of the
 * first refine_budget pool entries when refine_budget > 0.
 * pool_ids/pool_dists receive the sorted pool (num_out = pool size);
 * out_ids/out_dists the final top_k.  stats: 4 x u64 per query
 * {pq_scored, corrected, expanded, visited_dedup_skips}.
 * Returns 0, or 1 + the index of the first failing query.
 */
int ref_pq_search_batch(void *p, const int32_t *graph, int degree, int graph_entry,
                        const float *queries, int nq, const int32_t *pool_sizes,
                        int entry_points, int expand_count, unsigned int seed,
                        int correction, int refine_budget, int top_k, int threads,
                        int32_t *pool_ids, float *pool_dists, int pool_stride, int32_t *pool_counts,
                        int32_t *out_ids, float *out_dists, int out_stride, int32_t *out_counts,
                        uint64_t *stats) {
    RefPq *h = (RefPq *)p;
    PqBatch b;
    int t, rc, max_pool = 0, i;
    if (!h || !graph || !queries || nq < 0 || !pool_sizes || threads < 1) return -1;
    if (correction && !h->residual) return -1;
    for (i = 0; i < nq; i++) if (pool_sizes[i] > max_pool) max_pool = pool_sizes[i];
    if (threads > 256) threads = 256;
    memset(&b, 0, sizeof(b));
    b.h = h; b.graph = graph; b.degree = degree; b.graph_entry = graph_entry;
    b.queries = queries; b.pool_sizes = pool_sizes; b.entry_points = entry_points;
    b.expand_count = expand_count; b.correction = correction; b.refine_budget = refine_budget;
    b.top_k = top_k; b.seed = seed;
    b.pool_ids = pool_ids; b.pool_dists = pool_dists; b.pool_stride = pool_stride; b.pool_counts = pool_counts;
    b.out_ids = out_ids; b.out_dists = out_dists; b.out_stride = out_stride; b.out_counts = out_counts;
    b.stats = stats;
    b.scratch_stride = max_pool > 0 ? max_pool : 1;
    b.scratch_ids = (int *)malloc((size_t)threads * b.scratch_stride * sizeof(int));
    b.scratch_dists = (float *)malloc((size_t)threads * b.scratch_stride * sizeof(float));
    b.queries_res = (RetrievalPqResidualQuery **)calloc((size_t)threads, sizeof(void *));
    b.refine = (RetrievalFinalRefineContext **)calloc((size_t)threads, sizeof(void *));
    rc = (!b.scratch_ids || !b.scratch_dists || !b.queries_res || !b.refine) ? -1 : 0;
    for (t = 0; t < threads && rc == 0; t++) {
        if (h->residual && retrieval_pq_residual_query_create(h->residual, &b.queries_res[t]) != 0) rc = -1;
        if (rc == 0 && refine_budget > 0) {
            RetrievalFinalRefineConfig config;
            memset(&config, 0, sizeof(config));
            config.mode = RETRIEVAL_REFINE_CURRENT;
            config.num_vectors = (int)h->artifacts.metadata.num_vectors;
            config.dim = (int)h->artifacts.metadata.dim;
            config.capacity = refine_budget;
            config.cache_slots = 1;
            config.decode = harness_pq_decode;
            config.provider = b.queries_res[t];
            if (!b.queries_res[t] || retrieval_final_refine_open(&config, &b.refine[t]) != 0) rc = -1;
        }
    }
    if (rc == 0) rc = fanout_run(nq, threads, pq_batch_item, &b);
    for (t = 0; t < threads; t++) {
        if (b.refine) retrieval_final_refine_close(b.refine[t]);
        if (b.queries_res) retrieval_pq_residual_query_destroy(b.queries_res[t]);
    }
    free(b.scratch_ids); free(b.scratch_dists); free(b.queries_res); free(b.refine);
    return rc;
}

/* ------------------------------------------------------------------ */
/* SQ                                                                  */

typedef struct {
    RetrievalDemoEncodedDataset ds;
} RefSq;

/* An in-memory SQ dataset laid out as the reference's host keeps it:
 * flat L1 codes (the L1MS payload), per-vector residual qparams, and flat
 * residual rows (RetrievalDemoEncodedDataset, retrieval_rpc_demo.h:24). */
int ref_sq_open(int num_vectors, int dim, int l1_bits, float l1_scale, float l1_zero,
                const uint8_t *l1_codes, int residual_bits, const uint8_t *residual_codes,
                const float *residual_qparams, void **out) {
    RefSq *h;
    if (!out || num_vectors <= 0 || dim <= 0 || (l1_bits != 4 && l1_bits != 8)) return -1;
    h = (RefSq *)calloc(1, sizeof(*h));
    if (!h) return -1;
    h->ds.num_vectors = num_vectors;
    h->ds.dim = dim;
    h->ds.l1_bits = l1_bits;
    h->ds.l1_code_bytes = l1_bits == 4 ? (dim + 1) / 2 : dim;
    h->ds.l1_qparams.scale = l1_scale;
    h->ds.l1_qparams.zero_point = l1_zero;
    h->ds.l1_codes = (uint8_t *)l1_codes;
    if (residual_codes && residual_qparams && (residual_bits == 4 || residual_bits == 8)) {
        h->ds.residual_bits = residual_bits;
        h->ds.residual_code_bytes = residual_bits == 4 ? (dim + 1) / 2 : dim;
        h->ds.residual_codes = (uint8_t *)residual_codes;
        h->ds.residual_qparams = (QCResidualQuantParams *)residual_qparams;
    }
    *out = h;
    return 0;
}

void ref_sq_close(void *p) { free(p); }

static int harness_sq_quantize(const RefSq *h, const float *query, uint8_t *query_l1) {
    if (h->ds.l1_bits == 4)
        return retrieval_quantize_query_u4(query, h->ds.dim, h->ds.l1_qparams.scale,
                                           h->ds.l1_qparams.zero_point, query_l1);
    return retrieval_quantize_query_u8(query, h->ds.dim, h->ds.l1_qparams.scale,
                                       h->ds.l1_qparams.zero_point, query_l1);
}

static float harness_sq_coarse(const RefSq *h, const uint8_t *query_l1, int id) {
    const uint8_t *code = h->ds.l1_codes + (size_t)id * h->ds.l1_code_bytes;
    if (h->ds.l1_bits == 4)
        return retrieval_compute_int4_packed_distance_u8(query_l1, code, h->ds.dim,
                                                         h->ds.l1_qparams.scale);
    return retrieval_compute_int8_native_distance_u8(query_l1, code, h->ds.dim,
                                                     h->ds.l1_qparams.scale);
}

/* retrieval_quantize_query_u8/_u4, l1_int8_core.c:13/:39 */
int ref_sq_quantize(void *p, const float *query, uint8_t *out) {
    return p ? harness_sq_quantize((RefSq *)p, query, out) : -1;
}

/* retrieval_compute_int8_native_distance_u8 / int4_packed, l1_int8_core.c:463/:477 */
int ref_sq_coarse(void *p, const float *query, const int32_t *ids, int count, float *out) {
    RefSq *h = (RefSq *)p;
    uint8_t q[RETRIEVAL_ASYNC_DEMO_MAX_DIM];
    int i;
    if (!h || h->ds.dim > RETRIEVAL_ASYNC_DEMO_MAX_DIM || harness_sq_quantize(h, query, q) != 0) return -1;
    for (i = 0; i < count; i++) out[i] = harness_sq_coarse(h, q, ids[i]);
    return 0;
}

/* retrieval_demo_exact_distance_residual, retrieval_rpc_demo_support.c:1577 */
int ref_sq_exact(void *p, const float *query, const int32_t *ids, int count, float *out) {
    RefSq *h = (RefSq *)p;
    int i;
    if (!h) return -1;
    for (i = 0; i < count; i++) out[i] = retrieval_demo_exact_distance_residual(query, &h->ds, ids[i]);
    return 0;
}

typedef struct { const RefSq *h; const uint8_t *query_l1; } SqDistCtx;
typedef struct { const RefSq *h; const float *query; int correction; } SqCorrCtx;

/* The fake-DSP callbacks of the reference host, retrieval_rpc_demo_pipeline.c:881-898
 * (coarse SQ distance) and :996-1011 (exact residual distance when
 * correction is on, else the coarse distance). */
static int harness_sqmd_distance(const SqmdWorkItem *work, float *coarse, void *ctx) {
    SqDistCtx *c = (SqDistCtx *)ctx;
    if (!work || !coarse || work->neighbor_id < 0 || work->neighbor_id >= c->h->ds.num_vectors) return -1;
    *coarse = harness_sq_coarse(c->h, c->query_l1, work->neighbor_id);
    return 0;
}

static float harness_sqmd_correction(int neighbor_id, int source_id, float coarse, void *ctx) {
    SqCorrCtx *c = (SqCorrCtx *)ctx;
    (void)source_id;
    if (!c->correction) return coarse;
    return retrieval_demo_exact_distance_residual(c->query, &c->h->ds, neighbor_id);
}

typedef struct {
    RefSq *h;
    const int32_t *graph;
    int degree, graph_entry;
    const float *queries;
    const int32_t *pool_sizes;
    int entry_points, expand_count, lanes, correction;
    unsigned int seed;
    int32_t *out_ids; float *out_dists; int out_stride; int32_t *out_counts;
} SqBatch;

static int sqmd_batch_item(void *ctx, int worker, int qi) {
    SqBatch *b = (SqBatch *)ctx;
    RefSq *h = b->h;
    const float *query = b->queries + (size_t)qi * h->ds.dim;
    int pool = b->pool_sizes[qi];
    uint8_t q[RETRIEVAL_ASYNC_DEMO_MAX_DIM];
    int seeds[4096];
    float seed_dists[4096];
    SqDistCtx dctx;
    SqCorrCtx cctx;
    int count, i, n;
    (void)worker;
    if (b->entry_points > 4096 || h->ds.dim > RETRIEVAL_ASYNC_DEMO_MAX_DIM ||
        harness_sq_quantize(h, query, q) != 0)
        return -1;
    /* seeds: retrieval_sqmd_make_seed_ids (sqmd_seed.c:15) with the distances
     * sqmd_make_seed (pipeline.c:1013) assigns */
    n = retrieval_sqmd_make_seed_ids(h->ds.num_vectors, b->entry_points, b->graph_entry, b->seed,
                                     seeds, b->entry_points);
    if (n <= 0) return -1;
    for (i = 0; i < n; i++) {
        if (b->correction) {
            seed_dists[i] = retrieval_demo_exact_distance_residual(query, &h->ds, seeds[i]);
            if (!isfinite(seed_dists[i]) || seed_dists[i] < 0.0f) return -1;
        } else {
            seed_dists[i] = harness_sq_coarse(h, q, seeds[i]);
        }
    }
    dctx.h = h; dctx.query_l1 = q;
    cctx.h = h; cctx.query = query; cctx.correction = b->correction;
    count = sqmd_cpu_state_run_fake_dsp(b->graph, b->degree, h->ds.num_vectors, pool,
                                        b->entry_points, b->expand_count, seeds, seed_dists, n,
                                        b->lanes, harness_sqmd_distance, &dctx,
                                        harness_sqmd_correction, &cctx,
                                        b->out_ids + (size_t)qi * b->out_stride,
                                        b->out_dists + (size_t)qi * b->out_stride,
                                        b->out_stride);
    if (count < 0) return -1;
    if (b->out_counts) b->out_counts[qi] = count;
    return 0;
}

/*
 * Batched SQMD search through the reference's in-process protocol driver
 * sqmd_cpu_state_run_fake_dsp (sqmd_common.c:2052): the CLI's SQ path with
 * the DSP lanes replaced by the reference's own fake-DSP loop.
 * Returns 0, or 1 + the index of the first failing query.
 */
int ref_sq_sqmd_batch(void *p, const int32_t *graph, int degree, int graph_entry,
                      const float *queries, int nq, const int32_t *pool_sizes,
                      int entry_points, int expand_count, unsigned int seed, int lanes,
                      int correction, int threads, int32_t *out_ids, float *out_dists,
                      int out_stride, int32_t *out_counts) {
    SqBatch b;
    if (!p || !graph || !queries || !pool_sizes || !out_ids || !out_dists) return -1;
    memset(&b, 0, sizeof(b));
    b.h = (RefSq *)p; b.graph = graph; b.degree = degree; b.graph_entry = graph_entry;
    b.queries = queries; b.pool_sizes = pool_sizes; b.entry_points = entry_points;
    b.expand_count = expand_count; b.lanes = lanes; b.correction = correction; b.seed = seed;
    b.out_ids = out_ids; b.out_dists = out_dists; b.out_stride = out_stride; b.out_counts = out_counts;
    return fanout_run(nq, threads, sqmd_batch_item, &b);
}

/* SQ final refine, mode CURRENT: decode = retrieval_final_refine_decode_sq
 * (final_refine.c:55) over the dataset's L1 + residual rows. */
typedef struct { const RefSq *h; } SqRefineProvider;

static int harness_sq_refine_decode(void *provider, int id, float *out) {
    const RefSq *h = ((SqRefineProvider *)provider)->h;
    if (id < 0 || id >= h->ds.num_vectors || !h->ds.residual_codes) return -1;
    return retrieval_final_refine_decode_sq(
        h->ds.l1_codes + (size_t)id * h->ds.l1_code_bytes, h->ds.l1_bits,
        h->ds.l1_qparams.scale, h->ds.l1_qparams.zero_point,
        h->ds.residual_codes + (size_t)id * h->ds.residual_code_bytes, h->ds.residual_bits,
        h->ds.residual_qparams[id].scale, h->ds.residual_qparams[id].zero_point,
        h->ds.dim, out);
}

/* retrieval_final_refine (final_refine.c:294) of cand_counts[q] candidates per
 * query, with either the SQ decode (kind 0, handle from ref_sq_open) or the
 * PQ residual decode (kind 1, handle from ref_pq_open). */
int ref_refine_batch(int kind, void *p, const float *queries, int dim, int nq,
                     int32_t *cand_ids, float *cand_dists, int cand_stride,
                     const int32_t *cand_counts, int top_k, int32_t *out_counts) {
    RetrievalFinalRefineConfig config;
    RetrievalFinalRefineContext *ctx = NULL;
    SqRefineProvider sqp;
    RetrievalPqResidualQuery *pq = NULL;
    int q, max_count = 1, rc = 0;
    for (q = 0; q < nq; q++) if (cand_counts[q] > max_count) max_count = cand_counts[q];
    memset(&config, 0, sizeof(config));
    config.mode = RETRIEVAL_REFINE_CURRENT;
    config.dim = dim;
    config.capacity = max_count;
    config.cache_slots = 1;
    if (kind == 0) {
        sqp.h = (const RefSq *)p;
        config.num_vectors = sqp.h->ds.num_vectors;
        config.decode = harness_sq_refine_decode;
        config.provider = &sqp;
    } else {
        RefPq *h = (RefPq *)p;
        if (!h->residual || retrieval_pq_residual_query_create(h->residual, &pq) != 0) return -1;
        config.num_vectors = (int)h->artifacts.metadata.num_vectors;
        config.decode = harness_pq_decode;
        config.provider = pq;
    }
    if (retrieval_final_refine_open(&config, &ctx) != 0) rc = -1;
    for (q = 0; q < nq && rc == 0; q++) {
        int n = retrieval_final_refine(ctx, queries + (size_t)q * dim,
                                       cand_ids + (size_t)q * cand_stride,
                                       cand_dists + (size_t)q * cand_stride,
                                       cand_counts[q], top_k, NULL);
        if (n < 0) rc = q + 1;
        else out_counts[q] = n;
    }
    retrieval_final_refine_close(ctx);
    retrieval_pq_residual_query_destroy(pq);
    return rc;
}

/* ------------------------------------------------------------------ */
/* legacy full device search (calculator_retrieval_search, the DSP TU)  */

typedef struct {
    const float *queries; int dim;
    const int32_t *pool_sizes;
    int entry_points, expand_count, num_out;
    int32_t *out_ids; float *out_dists; int out_stride; int32_t *out_counts;
} DspBatch;

static int dsp_batch_item(void *ctx, int worker, int qi) {
    DspBatch *b = (DspBatch *)ctx;
    int32 actual = 0;
    (void)worker;
    if (calculator_retrieval_search(0, b->queries + (size_t)qi * b->dim, b->dim, b->entry_points,
                                    b->expand_count, b->pool_sizes[qi], b->num_out,
                                    b->out_ids + (size_t)qi * b->out_stride, b->out_stride,
                                    b->out_dists + (size_t)qi * b->out_stride, b->out_stride,
                                    &actual) != AEE_SUCCESS)
        return -1;
    if (b->out_counts) b->out_counts[qi] = actual;
    return 0;
}

/* calculator_retrieval_load (async_dsp_search.c:293) then
 * calculator_retrieval_search (:368) per query, at most 8 concurrent
 * (DSP_SEARCH_MAX_CONCURRENT search contexts), then unload. */
int ref_dsp_search_batch(int l1_bits, const int32_t *graph, int n, int degree, int graph_entry,
                         const uint8_t *l1_codes, int l1_len, int dim, float scale, float zero,
                         const float *queries, int nq, const int32_t *pool_sizes,
                         int entry_points, int expand_count, int num_out, int threads,
                         int32_t *out_ids, float *out_dists, int out_stride, int32_t *out_counts) {
    DspBatch b;
    int rc;
    /* Built for the host, the DSP TU reads its code width through
     * RETRIEVAL_DEMO_L1_BITS == rover_config.sq_bits (retrieval_demo_params.h). */
    rover_config.sq_bits = l1_bits;
    if (calculator_rover_configure(0, 1, l1_bits) != AEE_SUCCESS) return -1;
    if (calculator_retrieval_load(0, graph, n * degree, l1_codes, l1_len, n, dim, degree,
                                  graph_entry, scale, zero) != AEE_SUCCESS)
        return -1;
    memset(&b, 0, sizeof(b));
    b.queries = queries; b.dim = dim; b.pool_sizes = pool_sizes; b.entry_points = entry_points;
    b.expand_count = expand_count; b.num_out = num_out; b.out_ids = out_ids;
    b.out_dists = out_dists; b.out_stride = out_stride; b.out_counts = out_counts;
    if (threads > 8) threads = 8;
    rc = fanout_run(nq, threads, dsp_batch_item, &b);
    calculator_retrieval_unload(0);
    return rc;
}
