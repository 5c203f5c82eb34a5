/* rover_cli.c -- `Rover search`, the reference's command line on the B200.
 *
 * Same options, defaults and checks as the reference's `Rover` executable
 * (src/app/main.c, src/app/config.c:6-118), same outputs: results.jsonl
 * lines `{"query":q,"ids":[...],"distances":[...]}` (config.c:145-156, ids
 * mapped back through --order-map), recall@1/10/100 against --gt
 * (demo_recall_hits_at_k, retrieval_rpc_demo_support.c:1709), the summary
 * lines and the metrics CSV row of the pure-PQ driver
 * (retrieval_rpc_demo_pure_pq.c:402-760, including its FNV-1a fingerprint of
 * every query's search pool before refinement) or the SQMD driver
 * (retrieval_rpc_demo_pipeline.c:2745-3340).
 *
 * The difference is where the search runs: the reference drives each query
 * through FastRPC lanes; this host loads the bundle with librover_host
 * (index.json, member SHA-256, header checks) and hands the whole query set
 * to libcalculator.so in one batched call (calculator_rover_pq_search /
 * calculator_rover_sq_search + calculator_rover_refine), whose kernels run
 * every query on the GPU.  Options that configure the phone's DSP sessions
 * (--lanes, --domain, --cache-pages, ...) are accepted and have no effect.
 * Index construction (build-index / insert / resume) is not part of this
 * search path. */
#define _GNU_SOURCE
#include <errno.h>
#include <limits.h>
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>

#include "calculator.h"
#include "rover_b200.h"
#include "rover_host.h"

typedef struct {
    const char* command;
    int parent_n, expand_count, rnn_s, rnn_t1, gt_k, n, dim, nq, degree, sq_bits, residual_bits, pq_bits, pq_m,
        pq_compression, top_k, pool, entry_points, lanes, source_window, first_factor, cache_pages,
        refine_cache_pages, refine_factor, train_samples, train_iters, seed, domain, unsigned_pd, build_pool,
        build_candidates, build_iterations, build_threads, build_refine_candidates, backlink_threads,
        checkpoint_every, reverse_candidates, cooldown_every, cooldown_ms;
    int graph_entry, third_residual, correction, disk, split_distance, refine_all, refine_mode;
    const char *parent_graph, *build_distance, *method, *search_mode, *build_method, *graph_format, *index_dir, *base,
        *query, *gt, *graph, *order_map, *output, *l1, *residual, *qparams, *residual_map, *error4, *bias, *pq_prefix,
        *pq_book, *pq_codes, *pq_residual, *pq_qparams, *result_dir, *metrics, *checkpoint, *identity, *layout,
        *layout_hash, *dataset;
} Config;

/* config.c:11-25 defaults */
static Config cfg = {
    .graph_entry = -1, .expand_count = 32, .rnn_s = 16, .rnn_t1 = 4, .build_distance = "cpu", .gt_k = 100,
    .sq_bits = 4, .residual_bits = 4, .pq_bits = 8, .disk = 1, .top_k = 10, .pool = 128, .entry_points = 32,
    .lanes = 4, .source_window = 1, .first_factor = 3, .cache_pages = 2048, .refine_cache_pages = 2048,
    .refine_factor = 2, .correction = 1, .train_samples = 100000, .train_iters = 20, .seed = 42, .domain = 3,
    .unsigned_pd = 1, .degree = 16, .build_pool = 128, .build_candidates = 16, .build_iterations = 1,
    .build_threads = 1, .backlink_threads = 1, .checkpoint_every = 1000000, .cooldown_ms = 10000,
    .parent_graph = "", .method = "sq", .search_mode = "sqmd", .build_method = "stream-insert",
    .graph_format = "nndescent", .base = "", .query = "", .gt = "", .graph = "", .order_map = "", .index_dir = "",
    .residual_map = "", .l1 = "", .residual = "", .qparams = "", .error4 = "", .bias = "", .output = "results.jsonl",
    .pq_prefix = "", .pq_book = "", .pq_codes = "", .pq_residual = "", .pq_qparams = "", .result_dir = ".",
    .metrics = "metrics.csv", .checkpoint = "", .identity = "", .layout = "original",
    .layout_hash = "0000000000000000000000000000000000000000000000000000000000000000", .dataset = "dataset",
};

typedef struct { const char* name; size_t offset; int integer; } Option;
#define INT(name, field) {name, offsetof(Config, field), 1}
#define STR(name, field) {name, offsetof(Config, field), 0}
static const Option options[] = {
    INT("parent-n", parent_n), STR("parent-graph", parent_graph), STR("build-distance", build_distance),
    INT("expand-count", expand_count), INT("rnn-s", rnn_s), INT("rnn-t1", rnn_t1), INT("gt-k", gt_k), INT("n", n),
    INT("dim", dim), INT("nq", nq), INT("graph-degree", degree), INT("sq-bits", sq_bits),
    INT("residual-bits", residual_bits), INT("pq-bits", pq_bits), INT("pq-m", pq_m),
    INT("pq-compression", pq_compression), INT("top-k", top_k), INT("pool", pool), INT("entry-points", entry_points),
    INT("lanes", lanes), INT("source-window", source_window), INT("first-stage-factor", first_factor),
    INT("cache-pages", cache_pages), INT("refine-cache-pages", refine_cache_pages), INT("refine-factor", refine_factor),
    INT("pq-train-samples", train_samples), INT("pq-train-iters", train_iters), INT("seed", seed),
    INT("domain", domain), INT("unsigned-pd", unsigned_pd), INT("build-pool", build_pool),
    INT("build-candidates", build_candidates), INT("build-iterations", build_iterations),
    INT("build-threads", build_threads), INT("build-refine-candidates", build_refine_candidates),
    INT("backlink-threads", backlink_threads), INT("checkpoint-every", checkpoint_every),
    INT("reverse-candidates", reverse_candidates), INT("cooldown-every", cooldown_every),
    INT("cooldown-ms", cooldown_ms), STR("method", method), STR("search-mode", search_mode),
    STR("build-method", build_method), STR("graph-format", graph_format), STR("index-dir", index_dir),
    STR("base", base), STR("query", query), STR("gt", gt), STR("graph", graph), STR("order-map", order_map),
    STR("output", output), STR("l1", l1), STR("residual", residual), STR("qparams", qparams),
    STR("residual-map", residual_map), STR("error4", error4), STR("bias", bias), STR("pq-prefix", pq_prefix),
    STR("pq-book", pq_book), STR("pq-codes", pq_codes), STR("pq-residual", pq_residual),
    STR("pq-qparams", pq_qparams), STR("result-dir", result_dir), STR("metrics", metrics),
    STR("checkpoint", checkpoint), STR("identity", identity), STR("layout", layout), STR("layout-hash", layout_hash),
    STR("dataset", dataset),
};

static int number(const char* s, int* out) {
    char* end;
    errno = 0;
    long n = strtol(s, &end, 10);
    if (errno || !*s || *end || n < 0 || n > INT_MAX) return -1;
    *out = (int)n;
    return 0;
}

static int choice(const char* s, const char* a, const char* b, int* v) {
    if (!strcmp(s, a)) { *v = 0; return 0; }
    if (!strcmp(s, b)) { *v = 1; return 0; }
    return -1;
}

/* config.c:61-118: 1 = help printed, -1 = invalid, 0 = run */
static int parse(int argc, char** argv) {
    Config* c = &cfg;
    int refine = 0, subdim = 0;
    if (argc < 2 || !strcmp(argv[1], "--help")) {
        puts("Rover search|build-index|insert|resume [options]\n"
             "B200 build: `search` runs every query on the GPU through libcalculator.so.");
        for (size_t i = 0; i < sizeof(options) / sizeof(*options); i++) printf("  --%s VALUE\n", options[i].name);
        puts("  --third-residual off|on  --refine off|on  --refine-all\n  --correction off|online  "
             "--storage memory|disk  --split-distance off|on  --pq-subdim N  --graph-entry ID|-1");
        return 1;
    }
    c->command = argv[1];
    if (strcmp(c->command, "search") && strcmp(c->command, "build-index") && strcmp(c->command, "insert") &&
        strcmp(c->command, "resume"))
        return -1;
    for (int i = 2; i < argc; i++) {
        const char* key = argv[i];
        int found = 0;
        if (!strcmp(key, "--refine-all")) { c->refine_all = 1; continue; }
        if (strncmp(key, "--", 2) || ++i >= argc) { fprintf(stderr, "Missing option value: %s\n", key); return -1; }
        key += 2;
        const char* v = argv[i];
        if (!strcmp(key, "graph-entry")) {
            if (!strcmp(v, "-1")) c->graph_entry = -1;
            else if (number(v, &c->graph_entry)) return -1;
            continue;
        }
        if (!strcmp(key, "third-residual")) { if (choice(v, "off", "on", &c->third_residual)) return -1; continue; }
        if (!strcmp(key, "refine")) { if (choice(v, "off", "on", &refine)) return -1; continue; }
        if (!strcmp(key, "correction")) { if (choice(v, "off", "online", &c->correction)) return -1; continue; }
        if (!strcmp(key, "storage")) { if (choice(v, "memory", "disk", &c->disk)) return -1; continue; }
        if (!strcmp(key, "split-distance")) { if (choice(v, "off", "on", &c->split_distance)) return -1; continue; }
        if (!strcmp(key, "pq-subdim")) { if (number(v, &subdim)) return -1; continue; }
        for (size_t j = 0; j < sizeof(options) / sizeof(*options); j++)
            if (!strcmp(key, options[j].name)) {
                char* field = (char*)c + options[j].offset;
                if (options[j].integer) { if (number(v, (int*)field)) return -1; }
                else *(const char**)field = v;
                found = 1;
                break;
            }
        if (!found) { fprintf(stderr, "Unknown option: --%s\n", key); return -1; }
    }
#define REQUIRE(test, message) do { if (!(test)) { fprintf(stderr, "Rover: %s\n", message); return -1; } } while (0)
    REQUIRE(c->n > 0 && c->dim > 0 && c->dim <= 1024, "n > 0 and dim in 1..1024 required");
    REQUIRE(c->domain <= 3 && c->unsigned_pd <= 1, "domain 0..3 and unsigned-pd 0/1 required");
    REQUIRE(c->degree > 0 && c->degree < c->n, "graph-degree must be in 1..n-1");
    REQUIRE((c->sq_bits == 4 || c->sq_bits == 8) && (c->pq_bits == 4 || c->pq_bits == 8) &&
                (c->residual_bits == 4 || c->residual_bits == 8),
            "code and residual bits must be 4 or 8");
    REQUIRE(!strcmp(c->method, "sq") || !strcmp(c->method, "pq"), "method must be sq or pq");
    REQUIRE(c->top_k > 0 && c->top_k <= 100 && c->pool >= c->top_k && c->pool <= 2000, "top-k 1..100; pool top-k..2000");
    REQUIRE(c->expand_count >= 1 && c->expand_count <= 32 && c->graph_entry < c->n && c->rnn_s > 0 && c->rnn_t1 > 0,
            "invalid expand-count/graph-entry/RNN parameters");
    REQUIRE(c->entry_points > 0 && c->entry_points <= c->n && c->lanes > 0 && c->lanes <= 8 && c->source_window >= 1 &&
                c->source_window <= 2,
            "invalid entry/lane/source-window capacity");
    REQUIRE(c->first_factor > 0 && c->first_factor <= 2000 / c->top_k && c->refine_factor > 0 &&
                c->refine_factor <= 2000 / c->top_k,
            "candidate factor exceeds capacity");
    REQUIRE(c->cache_pages <= 65536 && !(c->cache_pages & (c->cache_pages - 1)) && c->refine_cache_pages <= 65536 &&
                !(c->refine_cache_pages & (c->refine_cache_pages - 1)),
            "cache pages must be powers of two up to 65536");
    REQUIRE(c->gt_k > 0 && c->gt_k <= 1000000, "invalid GT width");
    REQUIRE(c->cache_pages > 0 && (!c->third_residual || c->refine_cache_pages > 0), "positive cache size required");
    REQUIRE(!refine || c->correction, "coarse-only search with final residual refinement is outside this release");
    REQUIRE(!c->split_distance || (!strcmp(c->method, "sq") && c->sq_bits == 4 && c->correction && *c->bias),
            "split distance requires SQ4 online correction and a verified bias file");
    REQUIRE(!strcmp(c->search_mode, "sqmd") || !strcmp(c->search_mode, "db-pair"), "search-mode must be sqmd or db-pair");
    if (!strcmp(c->method, "pq")) {
        REQUIRE(strcmp(c->search_mode, "db-pair"), "PQ supports SQMD; DB Pair is an SQ path");
        REQUIRE((!!subdim + !!c->pq_m + !!c->pq_compression) <= 1, "choose only one PQ grouping parameter");
        if (subdim) { REQUIRE(c->dim % subdim == 0, "PQ subdim must divide dim"); c->pq_m = c->dim / subdim; }
        if (c->pq_compression) {
            int64_t divisor = (int64_t)c->pq_compression * c->pq_bits;
            REQUIRE((c->dim * 32) % divisor == 0, "non-integral PQ M");
            c->pq_m = (int)((c->dim * 32) / divisor);
        }
        if (!c->pq_m) { REQUIRE(c->dim % 16 == 0, "set pq-m or pq-subdim explicitly for this dimension"); c->pq_m = c->dim / 16; }
        REQUIRE(c->pq_m > 0 && c->pq_m <= c->dim && c->dim % c->pq_m == 0, "PQ M must divide dim");
        c->pq_compression = c->dim * 4 / ((c->pq_m * c->pq_bits + 7) / 8);
        c->search_mode = "pure_pq";
    } else if (!strcmp(c->search_mode, "db-pair")) {
        c->search_mode = "db_pair";
    }
    c->refine_mode = refine ? (c->third_residual ? 2 : 1) : 0;
    REQUIRE(!c->third_residual, "the third-level (ERROR4) refine is not part of this build");
    REQUIRE(!c->split_distance, "the SQ4 split-distance correction is not part of this build");
    REQUIRE(strcmp(c->search_mode, "db_pair"), "the DB-pair search mode is not part of this build");
    if (!strcmp(c->command, "search"))
        REQUIRE(c->nq > 0 && c->top_k <= c->n && *c->query && (*c->graph || *c->index_dir),
                "search requires query, graph, nq and top-k <= n");
    REQUIRE(c->train_iters > 0 && c->train_samples > 0, "positive PQ training settings required");
    return 0;
}

static unsigned long long now_us(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (unsigned long long)ts.tv_sec * 1000000ull + (unsigned long long)ts.tv_nsec / 1000ull;
}

/* results.jsonl and the order map (config.c:121-156) */
static FILE* results;
static int *original_ids, *index_ids;

static int results_open(void) {
    if (*cfg.order_map) {
        FILE* map = fopen(cfg.order_map, "r");
        original_ids = (int*)malloc((size_t)cfg.n * sizeof(int));
        index_ids = (int*)malloc((size_t)cfg.n * sizeof(int));
        if (!map || !original_ids || !index_ids) { if (map) fclose(map); return -1; }
        for (int i = 0; i < cfg.n; i++) index_ids[i] = -1;
        for (int i = 0; i < cfg.n; i++) {
            int id;
            if (fscanf(map, "%d", &id) != 1 || id < 0 || id >= cfg.n || index_ids[id] != -1) { fclose(map); return -1; }
            original_ids[i] = id;
            index_ids[id] = i;
        }
        int extra;
        if (fscanf(map, "%d", &extra) != EOF) { fclose(map); return -1; }
        fclose(map);
    }
    results = fopen(cfg.output, "wx");
    return results ? 0 : -1;
}

static int write_result(int query, const int* ids, const float* distances, int count) {
    for (int i = 0; i < count; i++)
        if (ids[i] < 0 || ids[i] >= cfg.n || (distances && !isfinite(distances[i]))) return -1;
    if (!results) return -1;
    fprintf(results, "{\"query\":%d,\"ids\":[", query);
    for (int i = 0; i < count; i++) fprintf(results, "%s%d", i ? "," : "", original_ids ? original_ids[ids[i]] : ids[i]);
    fprintf(results, "],\"distances\":[");
    for (int i = 0; i < count; i++) fprintf(results, "%s%.9g", i ? "," : "", distances ? distances[i] : 0.0);
    fprintf(results, "]}\n");
    return ferror(results) ? -1 : 0;
}

static int results_close(void) {
    const int rc = results ? fclose(results) : 0;
    results = NULL;
    free(original_ids);
    free(index_ids);
    original_ids = index_ids = NULL;
    return rc;
}

static int recall_hits(const int* ids, int count, const int32_t* gt_row, int gt_k, int k) {
    int hits = 0;
    for (int i = 0; i < k && i < count; i++)
        for (int j = 0; j < gt_k && j < k; j++)
            if (ids[i] == (int)gt_row[j]) { hits++; break; }
    return hits;
}

/* retrieval_rpc_demo_pure_pq.c:387-399 */
static uint64_t fingerprint(uint64_t hash, const int* ids, const float* distances, int count) {
    for (int i = 0; i < count; ++i) {
        uint32_t values[2];
        values[0] = (uint32_t)ids[i];
        memcpy(&values[1], &distances[i], sizeof(float));
        for (int byte = 0; byte < 8; ++byte) {
            hash ^= (values[byte / 4] >> (8 * (byte % 4))) & 255u;
            hash *= UINT64_C(1099511628211);
        }
    }
    return hash;
}

static int path_join(char* out, size_t cap, const char* a, const char* b) {
    return (size_t)snprintf(out, cap, "%s%s", a, b) < cap ? 0 : -1;
}

typedef struct {
    int32_t *ids, *counts, *status;
    float* dists;
    int32_t *pool_ids, *pool_counts;
    float* pool_dists;
    uint64_t* stats;
} Outputs;

static void free_outputs(Outputs* o) {
    free(o->ids); free(o->counts); free(o->status); free(o->dists);
    free(o->pool_ids); free(o->pool_counts); free(o->pool_dists); free(o->stats);
}

static int run_search(remote_handle64 h, const RoverBundle* b, const float* queries, const int32_t* gt) {
    const int nq = cfg.nq, pq = b->method == 1;
    const int refine_budget = cfg.refine_mode ? (cfg.refine_all ? cfg.pool : cfg.refine_factor * cfg.top_k) : 0;
    RoverSearchParams p;
    memset(&p, 0, sizeof(p));
    p.size = (int32_t)sizeof(p);
    p.mode = ROVER_MODE_EXACT;
    p.entry_points = cfg.entry_points;
    p.seed = (uint32_t)cfg.seed;
    p.expand_count = cfg.expand_count;
    p.correction = cfg.correction;
    p.refine_budget = pq ? refine_budget : 0;
    /* the SQMD driver asks its search for rerank_count results
       (retrieval_rpc_demo_pipeline.c:2754): the refine budget, or top-k x
       the first-stage factor */
    p.top_k = pq ? cfg.top_k : (refine_budget ? refine_budget : cfg.top_k * cfg.first_factor);
    p.pool_stride = pq ? cfg.pool : 0;
    p.sq_mode = 1;
    const int stride = p.top_k;
    Outputs o;
    memset(&o, 0, sizeof(o));
    o.ids = (int32_t*)malloc((size_t)nq * stride * 4);
    o.dists = (float*)malloc((size_t)nq * stride * 4);
    o.counts = (int32_t*)malloc((size_t)nq * 4);
    o.status = (int32_t*)malloc((size_t)nq * 4);
    o.stats = (uint64_t*)calloc((size_t)nq * 4, 8);
    int32_t* pools = (int32_t*)malloc((size_t)nq * 4);
    if (pq) {
        o.pool_ids = (int32_t*)malloc((size_t)nq * cfg.pool * 4);
        o.pool_dists = (float*)malloc((size_t)nq * cfg.pool * 4);
        o.pool_counts = (int32_t*)malloc((size_t)nq * 4);
    }
    if (!o.ids || !o.dists || !o.counts || !o.status || !o.stats || !pools ||
        (pq && (!o.pool_ids || !o.pool_dists || !o.pool_counts))) {
        free(pools);
        free_outputs(&o);
        fprintf(stderr, "Rover: out of memory\n");
        return -1;
    }
    for (int i = 0; i < nq; ++i) pools[i] = cfg.pool;
    RoverSearchOutputs out = {o.ids, o.dists, o.counts, stride, o.pool_ids, o.pool_dists, o.pool_counts, o.stats,
                              o.status};
    int rc = 0;
    unsigned long long refine_us = 0, refine_candidates = 0;
    const unsigned long long start = now_us();
    if (pq) {
        rc = calculator_rover_pq_search(h, &p, queries, nq, pools, NULL, &out);
        for (int i = 0; i < nq; ++i) refine_candidates += (unsigned long long)(
            refine_budget ? (o.pool_counts[i] < refine_budget ? o.pool_counts[i] : refine_budget) : 0);
    } else {
        rc = calculator_rover_sq_search(h, &p, queries, nq, pools, &out);
        if (!rc && refine_budget) {
            /* retrieval_final_refine over the first refine_budget entries of the SQMD pool */
            int32_t* cand_counts = (int32_t*)malloc((size_t)nq * 4);
            int32_t* rid = (int32_t*)malloc((size_t)nq * cfg.top_k * 4);
            float* rd = (float*)malloc((size_t)nq * cfg.top_k * 4);
            int32_t* rc_counts = (int32_t*)malloc((size_t)nq * 4);
            if (!cand_counts || !rid || !rd || !rc_counts) rc = -1;
            for (int i = 0; !rc && i < nq; ++i) {
                cand_counts[i] = o.counts[i] < refine_budget ? o.counts[i] : refine_budget;
                refine_candidates += (unsigned long long)cand_counts[i];
            }
            const unsigned long long r0 = now_us();
            if (!rc)
                rc = calculator_rover_refine(h, 0, queries, nq, o.ids, stride, cand_counts, cfg.top_k, rid, rd,
                                             rc_counts, o.status);
            refine_us = now_us() - r0;
            for (int i = 0; !rc && i < nq; ++i) {
                memcpy(o.ids + (size_t)i * stride, rid + (size_t)i * cfg.top_k, (size_t)cfg.top_k * 4);
                memcpy(o.dists + (size_t)i * stride, rd + (size_t)i * cfg.top_k, (size_t)cfg.top_k * 4);
                o.counts[i] = rc_counts[i];
            }
            free(cand_counts); free(rid); free(rd); free(rc_counts);
        }
    }
    const unsigned long long total_wall_us = now_us() - start;
    if (rc) {
        fprintf(stderr, "Rover: search failed (%d): %s\n", rc, calculator_rover_last_error());
        free(pools);
        free_outputs(&o);
        return -1;
    }
    uint64_t fp = UINT64_C(14695981039346656037);
    unsigned long long r1 = 0, r10 = 0, r100 = 0, corrected = 0, scored = 0, expanded = 0;
    for (int q = 0; q < nq && !rc; ++q) {
        const int* ids = o.ids + (size_t)q * stride;
        const float* dists = o.dists + (size_t)q * stride;
        int count = o.counts[q];
        if (pq) fp = fingerprint(fp, o.pool_ids + (size_t)q * cfg.pool, o.pool_dists + (size_t)q * cfg.pool,
                                 o.pool_counts[q]);
        if (pq && count != cfg.top_k) { fprintf(stderr, "Rover: query %d returned %d results\n", q, count); rc = -1; break; }
        const int limit = count < cfg.top_k ? count : cfg.top_k;
        if (write_result(q, ids, dists, limit)) { rc = -1; break; }
        if (gt) {
            const int32_t* row = gt + (size_t)q * cfg.gt_k;
            r1 += (unsigned long long)recall_hits(ids, limit, row, cfg.gt_k, 1);
            r10 += (unsigned long long)recall_hits(ids, limit, row, cfg.gt_k, 10);
            r100 += (unsigned long long)recall_hits(ids, limit, row, cfg.gt_k, 100);
        }
        scored += o.stats[(size_t)q * 4];
        corrected += o.stats[(size_t)q * 4 + 1];
        expanded += o.stats[(size_t)q * 4 + 2];
    }
    free(pools);
    if (rc) { free_outputs(&o); return -1; }
    const double recall_at_1 = 100.0 * (double)r1 / nq, recall_at_10 = 100.0 * (double)r10 / (nq * 10.0),
                 recall_at_100 = 100.0 * (double)r100 / (nq * 100.0);
    const unsigned long long wall_us = total_wall_us / (unsigned long long)nq;
    if (!pq) {
        /* the SQMD driver prints its summary and writes no metrics file
           (retrieval_rpc_demo_pipeline.c:3360) */
        printf("  [ 1/1] e=%3d p=%4d  R@1=%5.2f R@10=%5.2f R@100=%5.2f  wall=%4llu us (work=%llu corr=%llu expanded=%llu)\n",
               cfg.entry_points, cfg.pool, recall_at_1, recall_at_10, recall_at_100, wall_us, scored / nq,
               corrected / nq, expanded / nq);
        if (refine_budget)
            printf("  [Phase15 stats] top_k=%d mode=%d factor=%d budget=%d queries=%d candidates=%llu refine_us=%llu\n",
                   cfg.top_k, cfg.refine_mode, cfg.refine_factor, refine_budget, nq, refine_candidates, refine_us);
        free_outputs(&o);
        return 0;
    }
    printf("  e=%3d p=%4d R@1=%5.2f R@10=%5.2f R@100=%5.2f wall=%llu us work=%llu corr=%llu expanded=%llu\n",
           cfg.entry_points, cfg.pool, recall_at_1, recall_at_10, recall_at_100, wall_us, scored / nq,
           corrected / nq, expanded / nq);
    FILE* m = fopen(cfg.metrics, "w");
    if (!m) { free_outputs(&o); fprintf(stderr, "Rover: cannot create %s\n", cfg.metrics); return -1; }
    {
        char prefix[PATH_MAX];
        snprintf(prefix, sizeof(prefix), "%s", *cfg.pq_prefix ? cfg.pq_prefix : cfg.index_dir);
        const int code_bytes = b->pq.code_bytes;
        printf("PQ_PIPELINE window=%d jobs=%llu retired=%llu high_water=%d\n", cfg.source_window, expanded, expanded, 1);
        printf("PQ_REFINE K=%d mode=%d factor=%d budget=%d candidates=%llu us=%llu search=%016llx\n", cfg.top_k,
               cfg.refine_mode, cfg.refine_factor, refine_budget, refine_candidates, refine_us, (unsigned long long)fp);
        fprintf(m, "dataset,layout,code_bits,ks,m,code_bytes,compression_x,entry_points,pool_size,queries,recall_at_1,"
                   "recall_at_10,recall_at_100,wall_us,work_items,dsp_adc_us,dsp_wait_polls,correction_mode,"
                   "residual_bits,corrected_candidates,residual_cache_hits,residual_cache_misses,"
                   "residual_cache_errors,artifact_prefix,window,source_jobs,source_retired,source_high_water,top_k,"
                   "refine_mode,refine_factor,refine_budget,refine_candidates,refine_us,refine_blocks,refine_bytes,"
                   "refine_hits,search_pool_fingerprint,total_wall_us\n");
        fprintf(m, "%s,%s,%d,%d,%d,%d,%d,%d,%d,%d,%.8f,%.8f,%.8f,%llu,%llu,%llu,%llu,%s,%d,%llu,%llu,%llu,%llu,%s,%d,"
                   "%llu,%llu,%d,%d,%d,%d,%d,%llu,%llu,%llu,%llu,%llu,%016llx,%llu\n",
                cfg.dataset, cfg.layout, b->pq.ks == 16 ? 4 : 8, b->pq.ks, b->pq.m, code_bytes,
                b->dim * 4 / code_bytes, cfg.entry_points, cfg.pool, nq, recall_at_1, recall_at_10, recall_at_100,
                wall_us, scored / nq, 0ull, 0ull, cfg.correction ? "online" : "off",
                cfg.correction ? b->residual_bits : 0, corrected, 0ull, 0ull, 0ull, prefix, cfg.source_window,
                expanded, expanded, 1, cfg.top_k, cfg.refine_mode, cfg.refine_factor, refine_budget, refine_candidates,
                refine_us, 0ull, 0ull, 0ull, (unsigned long long)fp, total_wall_us);
    }
    const int bad = fclose(m) != 0;
    free_outputs(&o);
    return bad ? -1 : 0;
}

static int search(remote_handle64 h) {
    RoverBundle* b = NULL;
    const int pq = !strcmp(cfg.method, "pq");
    int rc;
    if (*cfg.index_dir) {
        rc = rover_bundle_open_dir(cfg.index_dir, 1, &b);
        if (!rc && (b->method != pq || b->n != cfg.n || b->dim != cfg.dim || b->degree != cfg.degree)) {
            fprintf(stderr, "Rover: --index-dir disagrees with --method/--n/--dim/--graph-degree\n");
            rover_bundle_close(b);
            return -1;
        }
        if (!rc && cfg.graph_entry >= 0) b->graph_entry = b->pq.graph_entry = b->sq.graph_entry = cfg.graph_entry;
    } else if (pq) {
        char book[PATH_MAX], codes[PATH_MAX], res[PATH_MAX], qp[PATH_MAX];
        char suffix[32];
        snprintf(suffix, sizeof(suffix), ".pqres%d", cfg.residual_bits);
        if (path_join(book, sizeof(book), *cfg.pq_book ? cfg.pq_book : cfg.pq_prefix, *cfg.pq_book ? "" : ".pqbook") ||
            path_join(codes, sizeof(codes), *cfg.pq_codes ? cfg.pq_codes : cfg.pq_prefix, *cfg.pq_codes ? "" : ".pqcodes") ||
            path_join(res, sizeof(res), *cfg.pq_residual ? cfg.pq_residual : cfg.pq_prefix, *cfg.pq_residual ? "" : suffix) ||
            path_join(qp, sizeof(qp), *cfg.pq_qparams ? cfg.pq_qparams : res, *cfg.pq_qparams ? "" : ".qparams"))
            return -1;
        rc = rover_bundle_open_pq(cfg.graph, cfg.graph_format, cfg.n, cfg.dim, cfg.degree, cfg.graph_entry, book,
                                  codes, res, qp, cfg.correction ? cfg.residual_bits : 0, 1, &b);
    } else {
        rc = rover_bundle_open_sq(cfg.graph, cfg.graph_format, cfg.n, cfg.dim, cfg.degree, cfg.graph_entry, cfg.l1,
                                  cfg.residual, cfg.qparams, &b);
    }
    if (rc) { fprintf(stderr, "Rover: %s\n", rover_host_error()); return -1; }
    if (pq && (b->pq.m != cfg.pq_m || b->pq.ks != (cfg.pq_bits == 4 ? 16 : 256))) {
        fprintf(stderr, "Rover: the PQ bundle is M=%d x %d, the options M=%d x %d\n", b->pq.m, b->pq.ks, cfg.pq_m,
                cfg.pq_bits == 4 ? 16 : 256);
        rover_bundle_close(b);
        return -1;
    }
    float* queries = NULL;
    int32_t* gt = NULL;
    if (rover_read_fvecs(cfg.query, cfg.nq, cfg.dim, &queries) ||
        (*cfg.gt && rover_read_ivecs(cfg.gt, cfg.nq, cfg.gt_k, &gt))) {
        fprintf(stderr, "Rover: %s\n", rover_host_error());
        rover_bundle_close(b);
        free(queries);
        return -1;
    }
    if (gt && index_ids)   /* ground truth in original ids -> index ids (support.c:2273) */
        for (size_t j = 0; j < (size_t)cfg.nq * cfg.gt_k; j++)
            if (gt[j] >= 0 && gt[j] < cfg.n) gt[j] = index_ids[gt[j]];
    if (pq) {
        printf("RETRIEVAL_DB_MODE=pure_pq\n\n=== Pure-PQ SQMD Search (B200) ===\n");
        printf("dataset=%s N=%d dim=%d bits=%d M=%d Ks=%d compression=%dx correction=%s residual_bits=%d result=%s\n",
               cfg.dataset, cfg.n, cfg.dim, b->pq.ks == 16 ? 4 : 8, b->pq.m, b->pq.ks, cfg.pq_compression,
               cfg.correction ? "online" : "off", cfg.correction ? b->residual_bits : 0, cfg.metrics);
        rc = calculator_rover_pq_load(h, &b->pq);
    } else {
        printf("RETRIEVAL_DB_MODE=sqmd\n\n=== SQMD Search (B200) ===\n");
        printf("dataset=%s N=%d dim=%d sq_bits=%d residual_bits=%d correction=%s result=%s\n", cfg.dataset, cfg.n,
               cfg.dim, b->sq.l1_bits, b->residual_bits, cfg.correction ? "online" : "off", cfg.metrics);
        rc = calculator_rover_sq_load(h, &b->sq);
    }
    fflush(stdout);
    if (rc) fprintf(stderr, "Rover: index load failed (%d): %s\n", rc, calculator_rover_last_error());
    else rc = run_search(h, b, queries, gt);
    if (pq) calculator_rover_pq_unload(h);
    else calculator_rover_sq_unload(h);
    rover_bundle_close(b);
    free(queries);
    free(gt);
    return rc;
}

int main(int argc, char** argv) {
    int rc = parse(argc, argv);
    if (rc) return rc > 0 ? 0 : 2;
    if (strcmp(cfg.command, "search")) {
        fprintf(stderr, "Construction is available on graph-build-insert.\n");
        return 1;
    }
    remote_handle64 handle = 0;
    rc = calculator_open(calculator_URI "&_dom=cdsp", &handle);
    if (!rc) rc = calculator_rover_configure(handle, 1, cfg.sq_bits);
    if (!rc) {
        printf("ROVER_EVALUATION enabled=%d\n", *cfg.gt != 0);
        rc = results_open();
        if (rc) fprintf(stderr, "Rover: cannot create %s (it must not exist)\n", cfg.output);
        if (!rc) rc = search(handle);
        if (results_close()) rc = -1;
    }
    if (handle) {
        const int close_rc = calculator_close(handle);
        if (!rc) rc = close_rc;
    }
    if (rc) fprintf(stderr, "Rover failed: %d\n", rc);
    return rc ? 1 : 0;
}
