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
#include <ctype.h>
#include <errno.h>
#include <limits.h>
#include <math.h>
#include <stdarg.h>
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

/* ---- configuration ------------------------------------------------------
 *
 * The option names, their defaults and the wording of every refusal are the
 * reference CLI's interface (src/app/config.c:12-116) and stay identical, so
 * scripts written for `Rover search` drive this binary unchanged.  The
 * parser itself is a table of typed option specs bound to the fields they
 * set, and the checks are an ordered list of rules; the first failing rule's
 * message is printed, as the reference does. */
typedef struct {
    const char* command;
    /* integers */
    int parent_n, expand_count, rnn_s, rnn_t1, gt_k, n, dim, nq, degree, sq_bits, residual_bits, pq_bits, pq_m,
        pq_compression, pq_subdim, top_k, pool, entry_points, lanes, source_window, first_factor, cache_pages,
        refine_cache_pages, refine_factor, train_samples, train_iters, seed, domain, unsigned_pd, build_pool,
        build_candidates, build_iterations, build_threads, build_refine_candidates, backlink_threads,
        checkpoint_every, reverse_candidates, cooldown_every, cooldown_ms, graph_entry;
    /* two-way switches (0 = first spelling) */
    int third_residual, refine, correction, disk, split_distance, refine_all;
    int refine_mode;   /* derived: 0 none, 1 residual refine, 2 with the third residual */
    /* text */
    const char *parent_graph, *build_distance, *method, *search_mode, *build_method, *graph_format, *index_dir, *base,
        *query, *gt, *graph, *order_map, *output, *l1, *residual, *qparams, *residual_map, *error4, *bias, *pq_prefix,
        *pq_book, *pq_codes, *pq_residual, *pq_qparams, *result_dir, *metrics, *checkpoint, *identity, *layout,
        *layout_hash, *dataset;
} Config;

static Config cfg;

static void config_defaults(Config* c) {
    memset(c, 0, sizeof(*c));
    c->graph_entry = -1;
    c->expand_count = 32; c->rnn_s = 16; c->rnn_t1 = 4; c->gt_k = 100;
    c->sq_bits = 4; c->residual_bits = 4; c->pq_bits = 8; c->disk = 1;
    c->top_k = 10; c->pool = 128; c->entry_points = 32; c->lanes = 4; c->source_window = 1;
    c->first_factor = 3; c->refine_factor = 2; c->cache_pages = 2048; c->refine_cache_pages = 2048;
    c->correction = 1; c->train_samples = 100000; c->train_iters = 20; c->seed = 42;
    c->domain = 3; c->unsigned_pd = 1; c->degree = 16;
    c->build_pool = 128; c->build_candidates = 16; c->build_iterations = 1; c->build_threads = 1;
    c->backlink_threads = 1; c->checkpoint_every = 1000000; c->cooldown_ms = 10000;
    const char* empty = "";
    c->parent_graph = c->base = c->query = c->gt = c->graph = c->order_map = c->index_dir = empty;
    c->residual_map = c->l1 = c->residual = c->qparams = c->error4 = c->bias = empty;
    c->pq_prefix = c->pq_book = c->pq_codes = c->pq_residual = c->pq_qparams = empty;
    c->checkpoint = c->identity = empty;
    c->build_distance = "cpu"; c->method = "sq"; c->search_mode = "sqmd"; c->build_method = "stream-insert";
    c->graph_format = "nndescent"; c->output = "results.jsonl"; c->result_dir = "."; c->metrics = "metrics.csv";
    c->layout = "original"; c->dataset = "dataset";
    c->layout_hash = "0000000000000000000000000000000000000000000000000000000000000000";
}

enum OptKind { OPT_COUNT, OPT_ENTRY, OPT_TEXT, OPT_SWITCH };

typedef struct {
    const char* name;
    enum OptKind kind;
    void* field;
    const char* spellings;   /* OPT_SWITCH: "first|second" */
} OptSpec;

static const OptSpec kOptions[] = {
    {"parent-n", OPT_COUNT, &cfg.parent_n, 0},             {"parent-graph", OPT_TEXT, &cfg.parent_graph, 0},
    {"build-distance", OPT_TEXT, &cfg.build_distance, 0},  {"expand-count", OPT_COUNT, &cfg.expand_count, 0},
    {"rnn-s", OPT_COUNT, &cfg.rnn_s, 0},                   {"rnn-t1", OPT_COUNT, &cfg.rnn_t1, 0},
    {"gt-k", OPT_COUNT, &cfg.gt_k, 0},                     {"n", OPT_COUNT, &cfg.n, 0},
    {"dim", OPT_COUNT, &cfg.dim, 0},                       {"nq", OPT_COUNT, &cfg.nq, 0},
    {"graph-degree", OPT_COUNT, &cfg.degree, 0},           {"sq-bits", OPT_COUNT, &cfg.sq_bits, 0},
    {"residual-bits", OPT_COUNT, &cfg.residual_bits, 0},   {"pq-bits", OPT_COUNT, &cfg.pq_bits, 0},
    {"pq-m", OPT_COUNT, &cfg.pq_m, 0},                     {"pq-compression", OPT_COUNT, &cfg.pq_compression, 0},
    {"top-k", OPT_COUNT, &cfg.top_k, 0},                   {"pool", OPT_COUNT, &cfg.pool, 0},
    {"entry-points", OPT_COUNT, &cfg.entry_points, 0},     {"lanes", OPT_COUNT, &cfg.lanes, 0},
    {"source-window", OPT_COUNT, &cfg.source_window, 0},   {"first-stage-factor", OPT_COUNT, &cfg.first_factor, 0},
    {"cache-pages", OPT_COUNT, &cfg.cache_pages, 0},       {"refine-cache-pages", OPT_COUNT, &cfg.refine_cache_pages, 0},
    {"refine-factor", OPT_COUNT, &cfg.refine_factor, 0},   {"pq-train-samples", OPT_COUNT, &cfg.train_samples, 0},
    {"pq-train-iters", OPT_COUNT, &cfg.train_iters, 0},    {"seed", OPT_COUNT, &cfg.seed, 0},
    {"domain", OPT_COUNT, &cfg.domain, 0},                 {"unsigned-pd", OPT_COUNT, &cfg.unsigned_pd, 0},
    {"build-pool", OPT_COUNT, &cfg.build_pool, 0},         {"build-candidates", OPT_COUNT, &cfg.build_candidates, 0},
    {"build-iterations", OPT_COUNT, &cfg.build_iterations, 0},
    {"build-threads", OPT_COUNT, &cfg.build_threads, 0},
    {"build-refine-candidates", OPT_COUNT, &cfg.build_refine_candidates, 0},
    {"backlink-threads", OPT_COUNT, &cfg.backlink_threads, 0},
    {"checkpoint-every", OPT_COUNT, &cfg.checkpoint_every, 0},
    {"reverse-candidates", OPT_COUNT, &cfg.reverse_candidates, 0},
    {"cooldown-every", OPT_COUNT, &cfg.cooldown_every, 0}, {"cooldown-ms", OPT_COUNT, &cfg.cooldown_ms, 0},
    {"method", OPT_TEXT, &cfg.method, 0},                  {"search-mode", OPT_TEXT, &cfg.search_mode, 0},
    {"build-method", OPT_TEXT, &cfg.build_method, 0},      {"graph-format", OPT_TEXT, &cfg.graph_format, 0},
    {"index-dir", OPT_TEXT, &cfg.index_dir, 0},            {"base", OPT_TEXT, &cfg.base, 0},
    {"query", OPT_TEXT, &cfg.query, 0},                    {"gt", OPT_TEXT, &cfg.gt, 0},
    {"graph", OPT_TEXT, &cfg.graph, 0},                    {"order-map", OPT_TEXT, &cfg.order_map, 0},
    {"output", OPT_TEXT, &cfg.output, 0},                  {"l1", OPT_TEXT, &cfg.l1, 0},
    {"residual", OPT_TEXT, &cfg.residual, 0},              {"qparams", OPT_TEXT, &cfg.qparams, 0},
    {"residual-map", OPT_TEXT, &cfg.residual_map, 0},      {"error4", OPT_TEXT, &cfg.error4, 0},
    {"bias", OPT_TEXT, &cfg.bias, 0},                      {"pq-prefix", OPT_TEXT, &cfg.pq_prefix, 0},
    {"pq-book", OPT_TEXT, &cfg.pq_book, 0},                {"pq-codes", OPT_TEXT, &cfg.pq_codes, 0},
    {"pq-residual", OPT_TEXT, &cfg.pq_residual, 0},        {"pq-qparams", OPT_TEXT, &cfg.pq_qparams, 0},
    {"result-dir", OPT_TEXT, &cfg.result_dir, 0},          {"metrics", OPT_TEXT, &cfg.metrics, 0},
    {"checkpoint", OPT_TEXT, &cfg.checkpoint, 0},          {"identity", OPT_TEXT, &cfg.identity, 0},
    {"layout", OPT_TEXT, &cfg.layout, 0},                  {"layout-hash", OPT_TEXT, &cfg.layout_hash, 0},
    {"dataset", OPT_TEXT, &cfg.dataset, 0},
    /* options the reference lists on a separate help line */
    {"third-residual", OPT_SWITCH, &cfg.third_residual, "off|on"},
    {"refine", OPT_SWITCH, &cfg.refine, "off|on"},
    {"correction", OPT_SWITCH, &cfg.correction, "off|online"},
    {"storage", OPT_SWITCH, &cfg.disk, "memory|disk"},
    {"split-distance", OPT_SWITCH, &cfg.split_distance, "off|on"},
    {"pq-subdim", OPT_COUNT, &cfg.pq_subdim, 0},
    {"graph-entry", OPT_ENTRY, &cfg.graph_entry, 0},
};
#define OPTION_COUNT (sizeof(kOptions) / sizeof(kOptions[0]))

/* A decimal count in [0, INT_MAX]; nothing else may follow the digits. */
static int read_count(const char* text, int* out) {
    if (!*text) return -1;
    long long v = 0;
    for (const char* p = text; *p; ++p) {
        if (*p < '0' || *p > '9') return -1;
        v = v * 10 + (*p - '0');
        if (v > INT_MAX) return -1;
    }
    *out = (int)v;
    return 0;
}

/* Index of `word` among the '|'-separated spellings, or -1. */
static int spelling_index(const char* spellings, const char* word) {
    const size_t len = strlen(word);
    int index = 0;
    for (const char* s = spellings;; ++index) {
        const char* bar = strchr(s, '|');
        const size_t n = bar ? (size_t)(bar - s) : strlen(s);
        if (n == len && !strncmp(s, word, n)) return index;
        if (!bar) return -1;
        s = bar + 1;
    }
}

static const OptSpec* find_option(const char* name) {
    for (size_t i = 0; i < OPTION_COUNT; ++i)
        if (!strcmp(kOptions[i].name, name)) return &kOptions[i];
    return NULL;
}

/* 0 = stored, -1 = the value does not parse for this option. */
static int store_option(const OptSpec* o, const char* value) {
    switch (o->kind) {
    case OPT_TEXT: *(const char**)o->field = value; return 0;
    case OPT_COUNT: return read_count(value, (int*)o->field);
    case OPT_ENTRY:
        if (!strcmp(value, "-1")) { *(int*)o->field = -1; return 0; }
        return read_count(value, (int*)o->field);
    case OPT_SWITCH: {
        const int k = spelling_index(o->spellings, value);
        if (k < 0) return -1;
        *(int*)o->field = k;
        return 0;
    }
    }
    return -1;
}

static void print_help(void) {
    puts("Rover search|build-index|insert|resume [options]\n"
         "B200 build: `search` runs every query on the GPU through libcalculator.so.");
    for (size_t i = 0; i < OPTION_COUNT; ++i)
        if (kOptions[i].kind == OPT_COUNT || kOptions[i].kind == OPT_TEXT)
            if (strcmp(kOptions[i].name, "pq-subdim")) printf("  --%s VALUE\n", kOptions[i].name);
    fputs(" ", stdout);
    for (size_t i = 0; i < OPTION_COUNT; ++i)
        if (kOptions[i].kind == OPT_SWITCH) printf(" --%s %s", kOptions[i].name, kOptions[i].spellings);
    puts("  --refine-all  --pq-subdim N  --graph-entry ID|-1");
}

/* ---- checks, in the reference's order (config.c:82-116) ---------------- */
static int is(const char* a, const char* b) { return !strcmp(a, b); }
static int pow2_upto(int v, int cap) { return v <= cap && !(v & (v - 1)); }

static int rule_shape(const Config* c) { return c->n > 0 && c->dim > 0 && c->dim <= 1024; }
static int rule_domain(const Config* c) { return c->domain <= 3 && c->unsigned_pd <= 1; }
static int rule_degree(const Config* c) { return c->degree > 0 && c->degree < c->n; }
static int rule_bits(const Config* c) {
    return (c->sq_bits == 4 || c->sq_bits == 8) && (c->pq_bits == 4 || c->pq_bits == 8) &&
           (c->residual_bits == 4 || c->residual_bits == 8);
}
static int rule_method(const Config* c) { return is(c->method, "sq") || is(c->method, "pq"); }
static int rule_topk(const Config* c) {
    return c->top_k > 0 && c->top_k <= 100 && c->pool >= c->top_k && c->pool <= 2000;
}
static int rule_expand(const Config* c) {
    return c->expand_count >= 1 && c->expand_count <= 32 && c->graph_entry < c->n && c->rnn_s > 0 && c->rnn_t1 > 0;
}
static int rule_capacity(const Config* c) {
    return c->entry_points > 0 && c->entry_points <= c->n && c->lanes > 0 && c->lanes <= 8 &&
           c->source_window >= 1 && c->source_window <= 2;
}
static int rule_factors(const Config* c) {
    const int cap = 2000 / c->top_k;
    return c->first_factor > 0 && c->first_factor <= cap && c->refine_factor > 0 && c->refine_factor <= cap;
}
static int rule_cache_shape(const Config* c) {
    return pow2_upto(c->cache_pages, 65536) && pow2_upto(c->refine_cache_pages, 65536);
}
static int rule_gt(const Config* c) { return c->gt_k > 0 && c->gt_k <= 1000000; }
static int rule_cache_size(const Config* c) {
    return c->cache_pages > 0 && (!c->third_residual || c->refine_cache_pages > 0);
}
static int rule_refine(const Config* c) { return !c->refine || c->correction; }
static int rule_split(const Config* c) {
    return !c->split_distance || (is(c->method, "sq") && c->sq_bits == 4 && c->correction && *c->bias);
}
static int rule_mode(const Config* c) { return is(c->search_mode, "sqmd") || is(c->search_mode, "db-pair"); }

typedef struct { int (*holds)(const Config*); const char* message; } Rule;
static const Rule kRules[] = {
    {rule_shape, "n > 0 and dim in 1..1024 required"},
    {rule_domain, "domain 0..3 and unsigned-pd 0/1 required"},
    {rule_degree, "graph-degree must be in 1..n-1"},
    {rule_bits, "code and residual bits must be 4 or 8"},
    {rule_method, "method must be sq or pq"},
    {rule_topk, "top-k 1..100; pool top-k..2000"},
    {rule_expand, "invalid expand-count/graph-entry/RNN parameters"},
    {rule_capacity, "invalid entry/lane/source-window capacity"},
    {rule_factors, "candidate factor exceeds capacity"},
    {rule_cache_shape, "cache pages must be powers of two up to 65536"},
    {rule_gt, "invalid GT width"},
    {rule_cache_size, "positive cache size required"},
    {rule_refine, "coarse-only search with final residual refinement is outside this release"},
    {rule_split, "split distance requires SQ4 online correction and a verified bias file"},
    {rule_mode, "search-mode must be sqmd or db-pair"},
};

static int refuse(const char* message) {
    fprintf(stderr, "Rover: %s\n", message);
    return -1;
}

/* PQ grouping: at most one of --pq-subdim / --pq-m / --pq-compression picks
 * M; without one, M = dim / 16.  Then the compression figure follows from M
 * (config.c:99-105). */
static int settle_pq_grouping(Config* c) {
    const int chosen = (c->pq_subdim != 0) + (c->pq_m != 0) + (c->pq_compression != 0);
    if (chosen > 1) return refuse("choose only one PQ grouping parameter");
    if (c->pq_subdim) {
        if (c->dim % c->pq_subdim) return refuse("PQ subdim must divide dim");
        c->pq_m = c->dim / c->pq_subdim;
    } else if (c->pq_compression) {
        const int64_t bits_per_code = (int64_t)c->pq_compression * c->pq_bits;
        const int64_t total_bits = (int64_t)c->dim * 32;
        if (total_bits % bits_per_code) return refuse("non-integral PQ M");
        c->pq_m = (int)(total_bits / bits_per_code);
    } else if (!c->pq_m) {
        if (c->dim % 16) return refuse("set pq-m or pq-subdim explicitly for this dimension");
        c->pq_m = c->dim / 16;
    }
    if (!(c->pq_m > 0 && c->pq_m <= c->dim && c->dim % c->pq_m == 0)) return refuse("PQ M must divide dim");
    c->pq_compression = c->dim * 4 / ((c->pq_m * c->pq_bits + 7) / 8);
    return 0;
}

/* 1 = help printed, -1 = invalid, 0 = run */
static int parse(int argc, char** argv) {
    static const char* const commands[] = {"search", "build-index", "insert", "resume"};
    Config* c = &cfg;
    config_defaults(c);
    if (argc < 2 || is(argv[1], "--help")) { print_help(); return 1; }
    c->command = argv[1];
    int known = 0;
    for (size_t i = 0; i < sizeof(commands) / sizeof(commands[0]); ++i) known |= is(c->command, commands[i]);
    if (!known) return -1;
    for (int i = 2; i < argc; ++i) {
        const char* arg = argv[i];
        if (is(arg, "--refine-all")) { c->refine_all = 1; continue; }
        if (strncmp(arg, "--", 2) || i + 1 >= argc) { fprintf(stderr, "Missing option value: %s\n", arg); return -1; }
        const OptSpec* o = find_option(arg + 2);
        const char* value = argv[++i];
        if (!o) { fprintf(stderr, "Unknown option: %s\n", arg); return -1; }
        if (store_option(o, value)) return -1;
    }
    for (size_t r = 0; r < sizeof(kRules) / sizeof(kRules[0]); ++r)
        if (!kRules[r].holds(c)) return refuse(kRules[r].message);
    if (is(c->method, "pq")) {
        if (is(c->search_mode, "db-pair")) return refuse("PQ supports SQMD; DB Pair is an SQ path");
        if (settle_pq_grouping(c)) return -1;
        c->search_mode = "pure_pq";
    } else if (is(c->search_mode, "db-pair")) {
        c->search_mode = "db_pair";
    }
    c->refine_mode = c->refine ? 1 + (c->third_residual != 0) : 0;
    /* A residual file in a storage order of its own (retrieval_rpc_demo_
       reorder.c layouts B/C/D, read through --residual-map) is refused
       rather than read as if it were in graph order. */
    if (*c->residual_map)
        return refuse("reordered residual files (--residual-map) are not supported; use residual layout a");
    if (c->third_residual) {
        /* the artifact must exist and hash (config.c:118); it is checked
           against the index when the refine opens it */
        uint8_t digest[32];
        if (!*c->error4 || rover_sha256_file(c->error4, 0, digest) != 0)
            return refuse("missing or unreadable third residual artifact");
    }
    if (is(c->command, "search") &&
        !(c->nq > 0 && c->top_k <= c->n && *c->query && (*c->graph || *c->index_dir)))
        return refuse("search requires query, graph, nq and top-k <= n");
    if (!(c->train_iters > 0 && c->train_samples > 0)) return refuse("positive PQ training settings required");
    return 0;
}

static unsigned long long now_us(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (unsigned long long)ts.tv_sec * 1000000ull + (unsigned long long)ts.tv_nsec / 1000ull;
}

/* ---- results ------------------------------------------------------------
 *
 * --order-map lists, for each index row, the original id of the vector
 * stored there: a permutation of 0..n-1 as whitespace-separated decimals.
 * Results are written in original ids; ground truth (original ids) is
 * translated to index ids.  Each results.jsonl line is
 * {"query":Q,"ids":[...],"distances":[...]} with distances in %.9g, the
 * reference's format (config.c:145-156), built in memory and written once. */
typedef struct {
    FILE* out;
    int* to_original;   /* index row -> original id, NULL without a map */
    int* to_index;      /* original id -> index row */
    char* line;
    size_t cap;
} ResultSink;

static ResultSink sink;

static int load_order_map(const char* path, int n) {
    FILE* f = fopen(path, "rb");
    if (!f) return -1;
    fseek(f, 0, SEEK_END);
    const long size = ftell(f);
    fseek(f, 0, SEEK_SET);
    char* text = size >= 0 ? (char*)malloc((size_t)size + 1) : NULL;
    const int ok_read = text && fread(text, 1, (size_t)size, f) == (size_t)size;
    fclose(f);
    sink.to_original = (int*)malloc((size_t)n * sizeof(int));
    sink.to_index = (int*)malloc((size_t)n * sizeof(int));
    if (!ok_read || !sink.to_original || !sink.to_index) { free(text); return -1; }
    text[size] = 0;
    for (int i = 0; i < n; ++i) sink.to_index[i] = -1;
    const char* p = text;
    int rows = 0, bad = 0;
    for (;;) {
        while (*p && isspace((unsigned char)*p)) ++p;
        if (!*p) break;
        char* end;
        errno = 0;
        const long id = strtol(p, &end, 10);
        if (end == p || errno || rows >= n || id < 0 || id >= n || sink.to_index[id] != -1) { bad = 1; break; }
        sink.to_original[rows] = (int)id;
        sink.to_index[id] = rows++;
        p = end;
    }
    free(text);
    return bad || rows != n ? -1 : 0;
}

static int results_open(void) {
    if (*cfg.order_map && load_order_map(cfg.order_map, cfg.n)) return -1;
    sink.out = fopen(cfg.output, "wx");
    return sink.out ? 0 : -1;
}

static int append(size_t* len, const char* fmt, ...) {
    for (;;) {
        va_list ap;
        va_start(ap, fmt);
        const int n = vsnprintf(sink.line + *len, sink.cap - *len, fmt, ap);
        va_end(ap);
        if (n < 0) return -1;
        if (*len + (size_t)n < sink.cap) { *len += (size_t)n; return 0; }
        const size_t cap = sink.cap ? 2 * sink.cap + (size_t)n : 4096;
        char* grown = (char*)realloc(sink.line, cap);
        if (!grown) return -1;
        sink.line = grown;
        sink.cap = cap;
    }
}

static int write_result(int query, const int* ids, const float* distances, int count) {
    if (!sink.out) return -1;
    for (int i = 0; i < count; i++)
        if (ids[i] < 0 || ids[i] >= cfg.n || (distances && !isfinite(distances[i]))) return -1;
    size_t len = 0;
    int rc = append(&len, "{\"query\":%d,\"ids\":[", query);
    for (int i = 0; !rc && i < count; i++)
        rc = append(&len, i ? ",%d" : "%d", sink.to_original ? sink.to_original[ids[i]] : ids[i]);
    if (!rc) rc = append(&len, "],\"distances\":[");
    for (int i = 0; !rc && i < count; i++) rc = append(&len, i ? ",%.9g" : "%.9g", distances ? distances[i] : 0.0);
    if (!rc) rc = append(&len, "]}\n");
    if (rc || fwrite(sink.line, 1, len, sink.out) != len) return -1;
    return 0;
}

static int results_close(void) {
    const int rc = sink.out ? fclose(sink.out) : 0;
    free(sink.to_original);
    free(sink.to_index);
    free(sink.line);
    memset(&sink, 0, sizeof(sink));
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
    p.third_residual = pq && cfg.refine_mode == 2;
    /* SQMD_SPLIT_DISTANCE (retrieval_rpc_demo_pipeline.c:2776, set from
       --split-distance by config.c:122) */
    p.split_distance = !pq && cfg.split_distance;
    /* the SQMD driver asks its search for rerank_count results
       (retrieval_rpc_demo_pipeline.c:2754): the refine budget, or top-k x
       the first-stage factor */
    p.top_k = pq ? cfg.top_k : (refine_budget ? refine_budget : cfg.top_k * cfg.first_factor);
    p.pool_stride = pq ? cfg.pool : 0;
    /* SQ: the SQMD loop, or the DB-pair search (retrieval_rpc_demo_pipeline.c:2496-2700) */
    const int db_pair = !pq && is(cfg.search_mode, "db_pair");
    p.sq_mode = db_pair ? 2 : 1;
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
        /* without final refine, demo_rerank_candidates over every candidate:
           the DB-pair re-rank worker (retrieval_rpc_demo_pipeline.c:204-226)
           and the split-distance SQMD path (:3310-3320) */
        const int rerank = !refine_budget && ((db_pair && cfg.correction) || cfg.split_distance);
        if (!rc && (refine_budget || rerank)) {
            /* retrieval_final_refine over the first refine_budget entries of the SQMD pool */
            int32_t* cand_counts = (int32_t*)malloc((size_t)nq * 4);
            int32_t* rid = (int32_t*)malloc((size_t)nq * cfg.top_k * 4);
            float* rd = (float*)malloc((size_t)nq * cfg.top_k * 4);
            int32_t* rc_counts = (int32_t*)malloc((size_t)nq * 4);
            if (!cand_counts || !rid || !rd || !rc_counts) rc = -1;
            for (int i = 0; !rc && i < nq; ++i) {
                cand_counts[i] = rerank || o.counts[i] < refine_budget ? o.counts[i] : refine_budget;
                refine_candidates += (unsigned long long)cand_counts[i];
            }
            const unsigned long long r0 = now_us();
            if (!rc)
                rc = calculator_rover_refine(h, rerank ? 2 : cfg.refine_mode == 2 ? 3 : 0, queries, nq, o.ids,
                                             stride, cand_counts, cfg.top_k, rid, rd, rc_counts, o.status);
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

/* The split-distance bias, checked as sqmd_load_correction_bias does
   (retrieval_rpc_demo_pipeline.c:3000-3019 prints the same refusal). */
static int load_split_bias(remote_handle64 h, const RoverBundle* b) {
    float* bias = NULL;
    if (rover_split_bias_open(b, cfg.bias, &bias) != 0) {
        printf("  ERROR: split distance requires verified U4/U4 or U4/U8 bias artifact %s\n", cfg.bias);
        fprintf(stderr, "Rover: %s\n", rover_artifact_error());
        return -1;
    }
    printf("  SQMD split distance: ON bias=%s bytes=%llu\n", cfg.bias, (unsigned long long)b->n * 4ull);
    const int rc = calculator_rover_sq_split_load(h, bias, b->n);
    if (rc) fprintf(stderr, "Rover: split bias load failed (%d): %s\n", rc, calculator_rover_last_error());
    free(bias);
    return rc ? -1 : 0;
}

/* The ERROR4 artifact of the final refine's mode 2, checked as
   retrieval_final_refine.c:118-166 does (the reference's two open-failure
   messages, retrieval_rpc_demo_pure_pq.c:530-533 and
   retrieval_rpc_demo_pipeline.c:3040-3043). */
static int load_error4(remote_handle64 h, const RoverBundle* b) {
    RoverError4* e = NULL;
    const int pq = b->method == 1;
    if (rover_error4_open(b, cfg.error4, sink.to_original, &e) != 0) {
        printf(pq ? "ERROR: PQ final refinement identity/open failed\n"
                  : "  ERROR: Phase15 refinement artifact/provider validation failed\n");
        fprintf(stderr, "Rover: %s\n", rover_artifact_error());
        return -1;
    }
    const int rc = calculator_rover_error4_load(h, pq ? 1 : 0, e->qparams, e->blocks, e->blocks_bytes,
                                                e->num_vectors, e->dim);
    if (rc) fprintf(stderr, "Rover: ERROR4 load failed (%d): %s\n", rc, calculator_rover_last_error());
    rover_error4_close(e);
    return rc ? -1 : 0;
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
    if (gt && sink.to_index)   /* ground truth in original ids -> index ids (support.c:2273) */
        for (size_t j = 0; j < (size_t)cfg.nq * cfg.gt_k; j++)
            if (gt[j] >= 0 && gt[j] < cfg.n) gt[j] = sink.to_index[gt[j]];
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
    if (!rc && cfg.split_distance) rc = load_split_bias(h, b);
    if (!rc && cfg.refine_mode == 2) rc = load_error4(h, b);
    if (!rc) rc = run_search(h, b, queries, gt);
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
