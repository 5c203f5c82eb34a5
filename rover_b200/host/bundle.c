/* bundle.c -- Rover index bundles in C: index.json validation, member
 * checksums, graph / PQ / SQ member readers.
 *
 * The checks follow the reference's own: tools/index_bundle.py:187-226
 * (index.json: schema, sizes, required members, member paths, sizes and
 * SHA-256, PQ member names), :84-92 (graph ids, self and duplicate edges),
 * src/dsp_demo/retrieval_pq_artifact.c:886-958 and
 * tools/build_pure_pq_index.py:67-97 (PUREPQ01 headers),
 * retrieval_pq_residual.c:216-246 / :716-835 and
 * tools/build_pure_pq_residual.py:46-66 (PQRES01 headers),
 * tools/encode_l1_residual.py:10-27 and retrieval_rpc_demo_support.c:1968
 * (L1MS / QPMS files), retrieval_rpc_demo_graph_index.c:1296 and
 * support.c:1866 (graph formats). */
#define _GNU_SOURCE
#include <errno.h>
#include <limits.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include "json.h"
#include "rover_host.h"

static __thread char g_error[512];

const char* rover_host_error(void) { return g_error; }

static int fail(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_error, sizeof(g_error), fmt, ap);
    va_end(ap);
    return -1;
}

static long long file_size(const char* path) {
    struct stat st;
    if (stat(path, &st) != 0 || !S_ISREG(st.st_mode)) return -1;
    return (long long)st.st_size;
}

/* the whole file into a malloc'd buffer (+1 NUL byte) */
static int read_file(const char* path, uint8_t** out, size_t* len) {
    const long long sz = file_size(path);
    if (sz < 0) return fail("%s: not a readable file", path);
    FILE* f = fopen(path, "rb");
    if (!f) return fail("%s: %s", path, strerror(errno));
    uint8_t* buf = (uint8_t*)malloc((size_t)sz + 1);
    if (!buf) { fclose(f); return fail("%s: out of memory", path); }
    const size_t got = fread(buf, 1, (size_t)sz, f);
    const int extra = fgetc(f);
    fclose(f);
    if (got != (size_t)sz || extra != EOF) { free(buf); return fail("%s: short read", path); }
    buf[sz] = 0;
    *out = buf;
    *len = (size_t)sz;
    return 0;
}

static uint32_t rd32(const uint8_t* p) { return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24; }
static uint16_t rd16(const uint8_t* p) { return (uint16_t)(p[0] | p[1] << 8); }
static uint64_t rd64(const uint8_t* p) { return (uint64_t)rd32(p) | (uint64_t)rd32(p + 4) << 32; }
static float rdf(const uint8_t* p) { uint32_t u = rd32(p); float f; memcpy(&f, &u, 4); return f; }

/* ------------------------------------------------------------ vectors */

static int read_vecs(const char* path, int32_t count, int32_t dim, void** out) {
    if (count <= 0 || dim <= 0) return fail("%s: count and dim must be positive", path);
    FILE* f = fopen(path, "rb");
    if (!f) return fail("%s: %s", path, strerror(errno));
    uint8_t* buf = (uint8_t*)malloc((size_t)count * dim * 4);
    if (!buf) { fclose(f); return fail("%s: out of memory", path); }
    for (int32_t i = 0; i < count; ++i) {
        int32_t d = 0;
        if (fread(&d, 4, 1, f) != 1 || d != dim ||
            fread(buf + (size_t)i * dim * 4, 4, (size_t)dim, f) != (size_t)dim) {
            fclose(f);
            free(buf);
            return fail("%s: record %d missing or of dimension other than %d", path, i, dim);
        }
    }
    fclose(f);
    *out = buf;
    return 0;
}

int rover_read_fvecs(const char* path, int32_t count, int32_t dim, float** out) {
    return read_vecs(path, count, dim, (void**)out);
}

int rover_read_ivecs(const char* path, int32_t count, int32_t dim, int32_t** out) {
    return read_vecs(path, count, dim, (void**)out);
}

/* ------------------------------------------------------------ graphs */

static int cmp_i32(const void* a, const void* b) {
    const int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
    return (x > y) - (x < y);
}

int rover_check_graph(const int32_t* graph, int32_t n, int32_t degree) {
    int32_t* row = (int32_t*)malloc((size_t)degree * 4);
    if (!row) return fail("out of memory");
    for (int32_t i = 0; i < n; ++i) {
        const int32_t* g = graph + (size_t)i * degree;
        for (int32_t j = 0; j < degree; ++j) {
            if (g[j] < -1 || g[j] >= n) { free(row); return fail("Out-of-range graph neighbor (row %d)", i); }
            if (g[j] == i) { free(row); return fail("Graph contains a self edge (row %d)", i); }
        }
        memcpy(row, g, (size_t)degree * 4);
        qsort(row, (size_t)degree, 4, cmp_i32);
        for (int32_t j = 1; j < degree; ++j)
            if (row[j] >= 0 && row[j] == row[j - 1]) { free(row); return fail("Graph contains duplicate edges (row %d)", i); }
    }
    free(row);
    return 0;
}

int rover_read_graph(const char* path, const char* format, int32_t n, int32_t dim, int32_t degree,
                     int32_t** out) {
    if (n <= 0 || degree <= 0) return fail("graph: n and degree must be positive");
    const size_t count = (size_t)n * degree;
    int32_t* graph = (int32_t*)malloc(count * 4);
    if (!graph) return fail("graph: out of memory");
    FILE* f = fopen(path, "rb");
    if (!f) { free(graph); return fail("%s: %s", path, strerror(errno)); }
    int ok = 0;
    if (!strcmp(format, "rover") || !strcmp(format, "dense")) {
        int header_ok = 1;
        if (!strcmp(format, "rover")) {
            int32_t h[4];
            header_ok = fread(h, sizeof(h), 1, f) == 1 && (uint32_t)h[0] == 0x35314252u && h[1] == n && h[2] == dim &&
                        h[3] == degree;
        }
        ok = header_ok && fread(graph, 4, count, f) == count && fgetc(f) == EOF && !ferror(f);
    } else if (!strcmp(format, "nndescent")) {
        int32_t h[3];
        ok = fread(h, sizeof(h), 1, f) == 1 && h[0] == n && h[1] == degree;
        float* skip = (float*)malloc((size_t)degree * 4);
        for (int32_t i = 0; ok && i < n; ++i)
            ok = skip && fread(graph + (size_t)i * degree, 4, (size_t)degree, f) == (size_t)degree &&
                 fread(skip, 4, (size_t)degree, f) == (size_t)degree;
        free(skip);
    } else {
        fclose(f);
        free(graph);
        return fail("Unknown graph format: %s", format);
    }
    fclose(f);
    if (!ok) { free(graph); return fail("%s: %s graph size or header mismatch", path, format); }
    for (size_t i = 0; i < count; ++i)
        if (graph[i] < -1 || graph[i] >= n) { free(graph); return fail("%s: out-of-range neighbour", path); }
    *out = graph;
    return 0;
}

/* ------------------------------------------------------------ pure PQ */

enum { PQ_HEADER = 256, BLOCK = 4096, PQ_KIND_BOOK = 1, PQ_KIND_CODES = 2, RES_KIND_BLOCKS = 1, RES_KIND_QPARAMS = 2 };
static const uint32_t kEndian = 0x01020304u;

typedef struct {
    uint8_t uuid[16];
    uint64_t n;
    uint32_t dim, m, ks, subdim, code_bytes, trainer, sample, iters, seed;
    uint64_t train_count;
    uint8_t dataset_fp[32], layout_fp[32];
    uint64_t payload_bytes;
    uint8_t payload_hash[32];
} PqHeader;

static uint32_t pq_code_bytes(uint32_t m, uint32_t ks) { return ks == 16 ? (m + 1) / 2 : ks == 256 ? m : 0; }
static uint32_t res_code_bytes(uint32_t dim, uint32_t bits) { return bits == 4 ? (dim + 1) / 2 : dim; }

static int parse_pq_header(const char* path, const uint8_t* h, size_t len, uint32_t kind, PqHeader* md) {
    if (len < PQ_HEADER || memcmp(h, "PUREPQ01", 8)) return fail("%s: invalid Pure-PQ magic/header length", path);
    const uint16_t major = rd16(h + 8), minor = rd16(h + 10);
    if (major != 1 || minor > 1 || rd32(h + 12) != PQ_HEADER || rd32(h + 20) != kEndian)
        return fail("%s: unsupported Pure-PQ header", path);
    if (rd32(h + 16) != kind) return fail("%s: artifact kind %u, expected %u", path, rd32(h + 16), kind);
    memcpy(md->uuid, h + 32, 16);
    md->n = rd64(h + 48);
    md->dim = rd32(h + 56); md->m = rd32(h + 60); md->ks = rd32(h + 64); md->subdim = rd32(h + 68);
    md->code_bytes = rd32(h + 72);
    if (rd32(h + 76) != 1 || rd32(h + 80) != 1 || rd32(h + 84) != 1)
        return fail("%s: unsupported metric or payload dtype", path);
    md->trainer = rd32(h + 88); md->sample = rd32(h + 92);
    md->train_count = rd64(h + 96);
    md->iters = rd32(h + 104); md->seed = rd32(h + 108);
    md->payload_bytes = rd64(h + 112);
    memcpy(md->payload_hash, h + 120, 32);
    memcpy(md->dataset_fp, h + 152, 32);
    memcpy(md->layout_fp, h + 184, 32);
    static const uint8_t zero16[16] = {0};
    if (!memcmp(md->uuid, zero16, 16) || md->n == 0 || md->n > INT32_MAX || md->dim == 0 || md->m == 0 ||
        md->subdim == 0 || (uint64_t)md->m * md->subdim != md->dim || md->code_bytes != pq_code_bytes(md->m, md->ks) ||
        md->train_count == 0 || md->train_count > md->n || md->iters == 0)
        return fail("%s: inconsistent Pure-PQ metadata", path);
    return 0;
}

static int same_meta(const PqHeader* a, const PqHeader* b) {
    return !memcmp(a->uuid, b->uuid, 16) && a->n == b->n && a->dim == b->dim && a->m == b->m && a->ks == b->ks &&
           a->subdim == b->subdim && a->code_bytes == b->code_bytes && a->trainer == b->trainer &&
           a->sample == b->sample && a->train_count == b->train_count && a->iters == b->iters &&
           a->seed == b->seed && !memcmp(a->dataset_fp, b->dataset_fp, 32) && !memcmp(a->layout_fp, b->layout_fp, 32);
}

/* header + payload of one .pqbook / .pqcodes file */
static int load_pq_member(const char* path, uint32_t kind, int verify, PqHeader* md, uint8_t** payload) {
    uint8_t* raw = NULL;
    size_t len = 0;
    if (read_file(path, &raw, &len) != 0) return -1;
    if (parse_pq_header(path, raw, len, kind, md) != 0) { free(raw); return -1; }
    if (len - PQ_HEADER != md->payload_bytes) { free(raw); return fail("%s: payload size mismatch", path); }
    if (verify) {
        uint8_t d[32];
        rover_sha256(raw + PQ_HEADER, len - PQ_HEADER, d);
        if (memcmp(d, md->payload_hash, 32)) { free(raw); return fail("%s: payload checksum mismatch", path); }
    }
    uint8_t* p = (uint8_t*)malloc(len - PQ_HEADER + 1);
    if (!p) { free(raw); return fail("%s: out of memory", path); }
    memcpy(p, raw + PQ_HEADER, len - PQ_HEADER);
    free(raw);
    *payload = p;
    return 0;
}

/* one .pqresN / .pqresN.qparams file checked against the PQ metadata */
static int load_res_member(const char* path, uint32_t kind, uint32_t bits, const PqHeader* md, int verify,
                           uint8_t** payload, size_t* payload_len) {
    uint8_t* raw = NULL;
    size_t len = 0;
    if (read_file(path, &raw, &len) != 0) return -1;
    const uint32_t storage = kind == RES_KIND_BLOCKS ? BLOCK : PQ_HEADER;
    const uint8_t* h = raw;
    if (len < storage || memcmp(h, "PQRES01\0", 8)) { free(raw); return fail("%s: invalid PQ residual header", path); }
    const uint32_t rcb = rd32(h + 28);
    const uint64_t n = rd64(h + 48);
    const uint32_t dim = rd32(h + 56), bb = rd32(h + 60), vpb = rd32(h + 64), blocks = rd32(h + 68);
    const uint64_t pbytes = rd64(h + 72);
    if (rd16(h + 8) != 1 || rd16(h + 10) > 0 || rd32(h + 12) != storage || rd32(h + 16) != kind ||
        rd32(h + 20) != kEndian || rd32(h + 176) != 8 || rd32(h + 24) != bits || rcb != res_code_bytes(dim, bits) ||
        bb != BLOCK || vpb != BLOCK / rcb || blocks != (n + vpb - 1) / vpb || n != md->n || dim != md->dim ||
        memcmp(h + 32, md->uuid, 16) || memcmp(h + 112, md->dataset_fp, 32) || memcmp(h + 144, md->layout_fp, 32)) {
        free(raw);
        return fail("%s: PQ residual metadata mismatch", path);
    }
    const uint64_t expect = kind == RES_KIND_BLOCKS ? (uint64_t)blocks * BLOCK : n * 8;
    if (pbytes != expect || len - storage != expect) { free(raw); return fail("%s: PQ residual payload size mismatch", path); }
    if (verify || kind == RES_KIND_QPARAMS) {
        uint8_t d[32];
        rover_sha256(raw + storage, len - storage, d);
        if (memcmp(d, h + 80, 32)) { free(raw); return fail("%s: PQ residual checksum mismatch", path); }
    }
    uint8_t* p = (uint8_t*)malloc(len - storage + 1);
    if (!p) { free(raw); return fail("%s: out of memory", path); }
    memcpy(p, raw + storage, len - storage);
    free(raw);
    *payload = p;
    *payload_len = len - storage;
    return 0;
}

void rover_bundle_close(RoverBundle* b) {
    if (!b) return;
    free(b->graph);
    free(b->pq_codebook);
    free(b->pq_codes);
    free(b->pq_residual_blocks);
    free(b->pq_qparams);
    free(b->sq_l1);
    free(b->sq_residual_rows);
    free(b->sq_qparams);
    free(b);
}

static int open_pq_members(RoverBundle* b, const char* book, const char* codes, const char* residual,
                           const char* qparams, int32_t residual_bits, int verify) {
    PqHeader mb, mc;
    uint8_t* pb = NULL;
    uint8_t* pc = NULL;
    if (load_pq_member(book, PQ_KIND_BOOK, verify, &mb, &pb) != 0) return -1;
    if (load_pq_member(codes, PQ_KIND_CODES, verify, &mc, &pc) != 0) { free(pb); return -1; }
    b->pq_codebook = (float*)pb;
    b->pq_codes = pc;
    if (!same_meta(&mb, &mc)) return fail("pqbook and pqcodes metadata mismatch");
    if ((int64_t)mb.n != b->n || (int32_t)mb.dim != b->dim)
        return fail("PQ bundle is %llu x %u, the index %d x %d", (unsigned long long)mb.n, mb.dim, b->n, b->dim);
    const size_t book_count = (size_t)mb.m * mb.ks * mb.subdim;
    if (mb.payload_bytes != book_count * 4) return fail("invalid codebook payload");
    for (size_t i = 0; i < book_count; ++i)
        if (!isfinite(rdf(pb + 4 * i))) return fail("invalid codebook payload");
    if (mc.payload_bytes != mc.n * mc.code_bytes) return fail("pqcodes payload size mismatch");
    memcpy(b->index_uuid, mb.uuid, 16);
    RoverPqIndexDesc* d = &b->pq;
    d->graph = b->graph;
    d->num_vectors = b->n;
    d->graph_degree = b->degree;
    d->graph_entry = b->graph_entry;
    d->dim = b->dim;
    d->codes = b->pq_codes;
    d->codebook = b->pq_codebook;
    d->m = (int32_t)mb.m;
    d->ks = (int32_t)mb.ks;
    d->subdim = (int32_t)mb.subdim;
    d->code_bytes = (int32_t)mb.code_bytes;
    b->residual_bits = residual_bits;
    if (residual_bits) {
        if (residual_bits != 4 && residual_bits != 8) return fail("residual bits must be 4 or 8");
        uint8_t* blocks = NULL;
        uint8_t* qp = NULL;
        size_t blen = 0, qlen = 0;
        if (load_res_member(residual, RES_KIND_BLOCKS, (uint32_t)residual_bits, &mb, verify, &blocks, &blen) != 0)
            return -1;
        b->pq_residual_blocks = blocks;
        if (load_res_member(qparams, RES_KIND_QPARAMS, (uint32_t)residual_bits, &mb, verify, &qp, &qlen) != 0)
            return -1;
        b->pq_qparams = (float*)qp;
        d->residual_blocks = blocks;
        d->residual_blocks_bytes = (int64_t)blen;
        d->residual_bits = residual_bits;
        d->residual_qparams = b->pq_qparams;
    }
    return 0;
}

int rover_bundle_open_pq(const char* graph_path, const char* graph_format, int32_t n, int32_t dim, int32_t degree,
                         int32_t graph_entry, const char* pq_book, const char* pq_codes, const char* pq_residual,
                         const char* pq_qparams, int32_t residual_bits, int verify, RoverBundle** out) {
    *out = NULL;
    RoverBundle* b = (RoverBundle*)calloc(1, sizeof(RoverBundle));
    if (!b) return fail("out of memory");
    b->method = 1;
    b->n = n;
    b->dim = dim;
    b->degree = degree;
    b->graph_entry = graph_entry;
    snprintf(b->base_paths[0], sizeof(b->base_paths[0]), "%s", pq_codes ? pq_codes : "");
    snprintf(b->base_paths[1], sizeof(b->base_paths[1]), "%s", pq_residual ? pq_residual : "");
    snprintf(b->base_paths[2], sizeof(b->base_paths[2]), "%s", pq_qparams ? pq_qparams : "");
    snprintf(b->pq_book_path, sizeof(b->pq_book_path), "%s", pq_book ? pq_book : "");
    if (rover_read_graph(graph_path, graph_format, n, dim, degree, &b->graph) != 0 ||
        (verify && rover_check_graph(b->graph, n, degree) != 0) ||
        open_pq_members(b, pq_book, pq_codes, pq_residual, pq_qparams, residual_bits, verify) != 0) {
        rover_bundle_close(b);
        return -1;
    }
    *out = b;
    return 0;
}

/* ------------------------------------------------------------ SQ */

int rover_bundle_open_sq(const char* graph_path, const char* graph_format, int32_t n, int32_t dim, int32_t degree,
                         int32_t graph_entry, const char* l1, const char* residual, const char* qparams,
                         RoverBundle** out) {
    *out = NULL;
    RoverBundle* b = (RoverBundle*)calloc(1, sizeof(RoverBundle));
    if (!b) return fail("out of memory");
    b->method = 0;
    b->n = n;
    b->dim = dim;
    b->degree = degree;
    b->graph_entry = graph_entry;
    snprintf(b->base_paths[0], sizeof(b->base_paths[0]), "%s", l1 ? l1 : "");
    snprintf(b->base_paths[1], sizeof(b->base_paths[1]), "%s", residual ? residual : "");
    snprintf(b->base_paths[2], sizeof(b->base_paths[2]), "%s", qparams ? qparams : "");
    uint8_t* raw = NULL;
    size_t len = 0;
    int rc = -1;
    if (rover_read_graph(graph_path, graph_format, n, dim, degree, &b->graph) != 0) goto done;
    /* l1.bin: "<IIiiiff4s" header (magic L1MS, version 1, n, dim, bits, scale, zero) + codes */
    if (read_file(l1, &raw, &len) != 0) goto done;
    if (len < 32 || rd32(raw) != 0x314C4D53u || rd32(raw + 4) != 1 || (int32_t)rd32(raw + 8) != n ||
        (int32_t)rd32(raw + 12) != dim || (rd32(raw + 16) != 4 && rd32(raw + 16) != 8)) {
        fail("%s: invalid L1 code file header", l1);
        goto done;
    }
    const uint32_t l1_bits = rd32(raw + 16);
    const float scale = rdf(raw + 20), zero = rdf(raw + 24);
    const size_t cb = res_code_bytes((uint32_t)dim, l1_bits);
    if (len != 32 + (size_t)n * cb) { fail("%s: L1 code file size mismatch", l1); goto done; }
    b->sq_l1 = (uint8_t*)malloc((size_t)n * cb);
    if (!b->sq_l1) { fail("out of memory"); goto done; }
    memcpy(b->sq_l1, raw + 32, (size_t)n * cb);
    free(raw);
    raw = NULL;
    /* qparams.bin: "<IIiiff8s" header (magic QPMS, version 1, n, residual bits, scale, zero) + pairs */
    if (read_file(qparams, &raw, &len) != 0) goto done;
    if (len < 32 || rd32(raw) != 0x51504D53u || rd32(raw + 4) != 1 || (int32_t)rd32(raw + 8) != n ||
        (rd32(raw + 12) != 4 && rd32(raw + 12) != 8) || rdf(raw + 16) != scale || rdf(raw + 20) != zero) {
        fail("%s: invalid qparams file header", qparams);
        goto done;
    }
    const uint32_t rbits = rd32(raw + 12);
    if (len != 32 + (size_t)n * 8) { fail("%s: qparams file size mismatch", qparams); goto done; }
    b->sq_qparams = (float*)malloc((size_t)n * 8);
    if (!b->sq_qparams) { fail("out of memory"); goto done; }
    memcpy(b->sq_qparams, raw + 32, (size_t)n * 8);
    free(raw);
    raw = NULL;
    /* residual.bin: 4096-byte blocks of 4096 / rcb rows, no header */
    {
        const size_t rcb = res_code_bytes((uint32_t)dim, rbits);
        const size_t vpb = BLOCK / rcb;
        const size_t blocks = ((size_t)n + vpb - 1) / vpb;
        if (read_file(residual, &raw, &len) != 0) goto done;
        if (len != blocks * BLOCK) { fail("%s: residual block file size mismatch", residual); goto done; }
        b->sq_residual_rows = (uint8_t*)malloc((size_t)n * rcb);
        if (!b->sq_residual_rows) { fail("out of memory"); goto done; }
        for (size_t i = 0; i < (size_t)n; ++i)
            memcpy(b->sq_residual_rows + i * rcb, raw + (i / vpb) * BLOCK + (i % vpb) * rcb, rcb);
    }
    b->residual_bits = (int32_t)rbits;
    RoverSqIndexDesc* d = &b->sq;
    d->graph = b->graph;
    d->num_vectors = n;
    d->graph_degree = degree;
    d->graph_entry = graph_entry;
    d->dim = dim;
    d->l1_codes = b->sq_l1;
    d->l1_bits = (int32_t)l1_bits;
    d->l1_scale = scale;
    d->l1_zero = zero;
    d->residual_rows = b->sq_residual_rows;
    d->residual_bits = (int32_t)rbits;
    d->residual_qparams = b->sq_qparams;
    rc = 0;
done:
    free(raw);
    if (rc != 0) rover_bundle_close(b);
    else *out = b;
    return rc;
}

/* ------------------------------------------------------------ index.json */

static const RoverJson* member(const RoverJson* files, const char* key) {
    const RoverJson* m = rover_json_get(files, key);
    return m && m->kind == ROVER_JSON_OBJECT ? m : NULL;
}

static int number_of(const RoverJson* obj, const char* key, double* out) {
    const RoverJson* v = rover_json_get(obj, key);
    if (!v || v->kind != ROVER_JSON_NUMBER) return -1;
    *out = v->num;
    return 0;
}

static const char* string_of(const RoverJson* obj, const char* key) {
    const RoverJson* v = rover_json_get(obj, key);
    return v && v->kind == ROVER_JSON_STRING ? v->str : NULL;
}

static const char* base_name(const char* p) {
    const char* s = strrchr(p, '/');
    return s ? s + 1 : p;
}

/* dir/member path, checked to resolve inside dir */
static int member_path(const char* root, const RoverJson* item, const char* key, char* out, size_t cap) {
    const char* rel = string_of(item, "path");
    if (!rel || !*rel || rel[0] == '/') return fail("Invalid index member %s", key);
    char joined[PATH_MAX];
    if ((size_t)snprintf(joined, sizeof(joined), "%s/%s", root, rel) >= sizeof(joined))
        return fail("Invalid index member %s", key);
    char real[PATH_MAX];
    if (!realpath(joined, real)) return fail("Invalid index member %s", key);
    const size_t rl = strlen(root);
    if (strncmp(real, root, rl) || real[rl] != '/' || file_size(real) < 0) return fail("Invalid index member %s", key);
    if ((size_t)snprintf(out, cap, "%s", real) >= cap) return fail("Invalid index member %s", key);
    return 0;
}

int rover_bundle_open_dir(const char* dir, int verify, RoverBundle** out) {
    *out = NULL;
    char root[PATH_MAX];
    if (!realpath(dir, root)) return fail("%s: %s", dir, strerror(errno));
    char path[PATH_MAX + 16];
    snprintf(path, sizeof(path), "%s/index.json", root);
    uint8_t* text = NULL;
    size_t len = 0;
    if (read_file(path, &text, &len) != 0) return -1;
    RoverJson doc;
    char err[128];
    if (rover_json_parse((const char*)text, len, &doc, err, sizeof(err)) != 0) {
        free(text);
        return fail("%s: %s", path, err);
    }
    free(text);
    int rc = -1;
    RoverBundle* b = NULL;
    char p_graph[PATH_MAX], p_a[PATH_MAX], p_b[PATH_MAX], p_c[PATH_MAX], p_d[PATH_MAX];
    const char* schema = string_of(&doc, "schema");
    const char* method = string_of(&doc, "method");
    const RoverJson* files = rover_json_get(&doc, "files");
    double n = 0, dim = 0, degree = 0, rbits = 0, cbits = 0, entry = -1;
    if (!schema || strcmp(schema, "rover.index.v1")) { fail("Unsupported Rover index schema"); goto done; }
    if (!method || (strcmp(method, "sq") && strcmp(method, "pq")) || number_of(&doc, "n", &n) ||
        number_of(&doc, "dim", &dim) || number_of(&doc, "graph_degree", &degree) || !(dim > 0 && dim <= 1024) ||
        !(degree > 0 && degree < n && n <= 2147483647.0) || n != floor(n) || dim != floor(dim) ||
        degree != floor(degree)) {
        fail("Invalid index method or dimensions");
        goto done;
    }
    const int pq = !strcmp(method, "pq");
    if (number_of(&doc, "residual_bits", &rbits) || (rbits != 4 && rbits != 8) ||
        number_of(&doc, pq ? "pq_bits" : "sq_bits", &cbits) || (cbits != 4 && cbits != 8)) {
        fail("Index bits must be 4 or 8");
        goto done;
    }
    if (!files || files->kind != ROVER_JSON_OBJECT) { fail("Index missing files"); goto done; }
    {
        static const char* sq_req[] = {"l1", "residual", "qparams", "graph", NULL};
        static const char* pq_req[] = {"pq_book", "pq_codes", "pq_residual", "pq_qparams", "pq_manifest",
                                       "pq_residual_manifest", "graph", NULL};
        for (const char** k = pq ? pq_req : sq_req; *k; ++k)
            if (!member(files, *k)) { fail("Index missing %s", *k); goto done; }
        const RoverJson* reordered = rover_json_get(&doc, "reordered");
        if (reordered && reordered->kind == ROVER_JSON_BOOL && reordered->boolean && !member(files, "order_map")) {
            fail("Index missing order_map");
            goto done;
        }
        const char* layout = string_of(&doc, "residual_layout");
        if (layout && strcmp(layout, "a") && !member(files, "residual_map")) { fail("Index missing residual_map"); goto done; }
        if (layout && strcmp(layout, "a")) {
            fail("residual layout %s (a reordered residual file) is not supported; use residual layout a", layout);
            goto done;
        }
    }
    /* every member: inside the directory, a regular file, unique name, recorded size and digest */
    for (int i = 0; i < files->count; ++i) {
        const char* key = files->keys[i];
        const RoverJson* item = &files->items[i];
        if (!strcmp(key, "error4")) continue;   /* the third-level residual is not read by this loader */
        if (item->kind != ROVER_JSON_OBJECT) { fail("Invalid index member %s", key); goto done; }
        char real[PATH_MAX];
        if (member_path(root, item, key, real, sizeof(real)) != 0) goto done;
        for (int j = 0; j < i; ++j) {
            const char* other = string_of(&files->items[j], "path");
            if (strcmp(files->keys[j], "error4") && other && !strcmp(base_name(other), base_name(real))) {
                fail("Colliding index member names");
                goto done;
            }
        }
        double bytes = -1;
        const char* digest = string_of(item, "sha256");
        if (number_of(item, "bytes", &bytes) || file_size(real) != (long long)bytes) {
            fail("Index member changed: %s", key);
            goto done;
        }
        if (verify) {
            uint8_t d[32];
            char hex[65];
            if (!digest || rover_sha256_file(real, 0, d) != 0) { fail("Index member changed: %s", key); goto done; }
            rover_hex(d, 32, hex);
            if (strcmp(hex, digest)) { fail("Index member changed: %s", key); goto done; }
        }
    }
    if (pq) {
        char suffix[16];
        snprintf(suffix, sizeof(suffix), ".pqres%d", (int)rbits);
        const char* keys[6] = {"pq_book", "pq_codes", "pq_manifest", "pq_residual", "pq_qparams", "pq_residual_manifest"};
        char names[6][40];
        snprintf(names[0], 40, "index.pqbook");
        snprintf(names[1], 40, "index.pqcodes");
        snprintf(names[2], 40, "index.pq.json");
        snprintf(names[3], 40, "index%s", suffix);
        snprintf(names[4], 40, "index%s.qparams", suffix);
        snprintf(names[5], 40, "index%s.json", suffix);
        for (int k = 0; k < 6; ++k)
            if (strcmp(base_name(string_of(member(files, keys[k]), "path")), names[k])) {
                fail("PQ bundle filenames must use the index prefix");
                goto done;
            }
    }
    const char* gformat = string_of(&doc, "graph_format");
    if (number_of(&doc, "graph_entry", &entry) != 0) entry = -1;
    if (member_path(root, member(files, "graph"), "graph", p_graph, sizeof(p_graph)) != 0) goto done;
    if (pq) {
        if (member_path(root, member(files, "pq_book"), "pq_book", p_a, sizeof(p_a)) ||
            member_path(root, member(files, "pq_codes"), "pq_codes", p_b, sizeof(p_b)) ||
            member_path(root, member(files, "pq_residual"), "pq_residual", p_c, sizeof(p_c)) ||
            member_path(root, member(files, "pq_qparams"), "pq_qparams", p_d, sizeof(p_d)))
            goto done;
        if (rover_bundle_open_pq(p_graph, gformat ? gformat : "rover", (int32_t)n, (int32_t)dim, (int32_t)degree,
                                 (int32_t)entry, p_a, p_b, p_c, p_d, (int32_t)rbits, verify, &b) != 0)
            goto done;
        if (b->pq.ks != (cbits == 4 ? 16 : 256)) {
            fail("PQ members disagree with index.json pq_bits");
            goto done;
        }
    } else {
        if (member_path(root, member(files, "l1"), "l1", p_a, sizeof(p_a)) ||
            member_path(root, member(files, "residual"), "residual", p_b, sizeof(p_b)) ||
            member_path(root, member(files, "qparams"), "qparams", p_c, sizeof(p_c)))
            goto done;
        if (rover_bundle_open_sq(p_graph, gformat ? gformat : "rover", (int32_t)n, (int32_t)dim, (int32_t)degree,
                                 (int32_t)entry, p_a, p_b, p_c, &b) != 0)
            goto done;
        if (verify && rover_check_graph(b->graph, b->n, b->degree) != 0) goto done;
        if (b->sq.l1_bits != (int32_t)cbits || b->residual_bits != (int32_t)rbits) {
            fail("SQ members disagree with index.json bits");
            goto done;
        }
    }
    rc = 0;
done:
    rover_json_free(&doc);
    if (rc == 0) *out = b;
    else rover_bundle_close(b);
    return rc;
}
