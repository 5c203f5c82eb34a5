/*
 * artifacts.c -- the two optional correction artifacts of `Rover search`:
 * the final refine's third-level ERROR4 file (--third-residual on --error4)
 * and the SQMD split-distance bias (--split-distance on --bias).
 *
 * Both are checked the way the reference host checks them before it uses
 * them -- retrieval_final_refine.c:118-166 (header fields, sizes, the
 * payload's SHA-256, the SHA-256 of the three base members, of the PQ
 * codebook and of the id maps, finite non-negative scales) and
 * retrieval_rpc_demo_support.c:237-297 (header fields, the source
 * fingerprint over the base members' digests, the payload's FNV-1a 64, finite
 * values) -- and handed back as host buffers for calculator_rover_error4_load
 * and calculator_rover_sq_split_load.
 */
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/rover_host.h"

#define E4_HEADER 256
#define E4_BLOCK 4096u
#define BIAS_HEADER 64

static __thread char g_error[512];

static int fail(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_error, sizeof(g_error), fmt, ap);
    va_end(ap);
    return -1;
}

const char* rover_artifact_error(void) { return g_error; }

static uint32_t rd32(const uint8_t* p) {
    return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24;
}
static uint64_t rd64(const uint8_t* p) { return (uint64_t)rd32(p) | (uint64_t)rd32(p + 4) << 32; }

/* The whole file in memory. */
static int slurp(const char* path, uint8_t** out, size_t* len) {
    FILE* f = fopen(path, "rb");
    if (!f) return fail("%s: cannot open", path);
    if (fseek(f, 0, SEEK_END) != 0) { fclose(f); return fail("%s: cannot seek", path); }
    const long size = ftell(f);
    if (size < 0 || fseek(f, 0, SEEK_SET) != 0) { fclose(f); return fail("%s: cannot size", path); }
    uint8_t* buf = (uint8_t*)malloc(size ? (size_t)size : 1);
    if (!buf) { fclose(f); return fail("out of memory"); }
    const size_t got = fread(buf, 1, (size_t)size, f);
    fclose(f);
    if (got != (size_t)size) { free(buf); return fail("%s: short read", path); }
    *out = buf;
    *len = (size_t)size;
    return 0;
}

static int file_digest_is(const char* path, const uint8_t want[32]) {
    uint8_t d[32];
    return path && *path && rover_sha256_file(path, 0, d) == 0 && memcmp(d, want, 32) == 0;
}

void rover_error4_close(RoverError4* e) {
    if (!e) return;
    free(e->file);
    free(e->qparams);
    free(e);
}

int rover_error4_open(const RoverBundle* b, const char* path, const int32_t* graph_to_original, RoverError4** out) {
    *out = NULL;
    const int pq = b->method == 1;
    const uint32_t n = (uint32_t)b->n, dim = (uint32_t)b->dim;
    const uint32_t cb = (dim + 1) / 2, vpb = E4_BLOCK / cb;
    if (!vpb) return fail("ERROR4 rows do not fit a block");
    const uint64_t qb = (uint64_t)n * 8u, blocks = ((uint64_t)n + vpb - 1) / vpb * E4_BLOCK;
    uint8_t* f = NULL;
    size_t len = 0;
    if (slurp(path, &f, &len) != 0) return -1;
    const uint8_t* h = f;
    uint8_t d[32];
    int ok = len >= E4_HEADER && memcmp(h, pq ? "PQERR4V1" : "SQERR4V1", 8) == 0 && rd32(h + 8) == 1 &&
             rd32(h + 12) == n && rd32(h + 16) == dim && (rd32(h + 20) == 4 || rd32(h + 20) == 8) &&
             (rd32(h + 24) == 4 || rd32(h + 24) == 8) && rd32(h + 28) == E4_BLOCK && rd32(h + 32) == 1 &&
             rd32(h + 36) == 1 && rd64(h + 40) == qb && rd64(h + 48) == blocks &&
             (uint64_t)len == E4_HEADER + qb + blocks;
    if (!ok) { free(f); return fail("%s: ERROR4 header does not match the index", path); }
    rover_sha256(f + E4_HEADER, len - E4_HEADER, d);
    if (memcmp(d, h + 56, 32) != 0) { free(f); return fail("%s: ERROR4 payload digest mismatch", path); }
    for (int i = 0; i < 3; ++i)
        if (!file_digest_is(b->base_paths[i], h + 88 + 32 * i)) {
            free(f);
            return fail("%s: ERROR4 artifact was built from other base members", path);
        }
    if (pq && !file_digest_is(b->pq_book_path, h + 184)) {
        free(f);
        return fail("%s: ERROR4 artifact was built from another codebook", path);
    }
    /* the id maps: graph -> original (or identity), then graph -> storage
       (identity: no storage map), or no bytes at all without a map */
    if (graph_to_original) {
        int32_t* maps = (int32_t*)malloc((size_t)n * 8);
        if (!maps) { free(f); return fail("out of memory"); }
        for (uint32_t i = 0; i < n; ++i) {
            maps[i] = graph_to_original[i];
            maps[n + i] = (int32_t)i;
        }
        rover_sha256(maps, (size_t)n * 8, d);
        free(maps);
    } else {
        static const uint8_t none = 0;
        rover_sha256(&none, 0, d);
    }
    if (memcmp(d, h + 216, 32) != 0) { free(f); return fail("%s: ERROR4 id-map digest mismatch", path); }
    RoverError4* e = (RoverError4*)calloc(1, sizeof(RoverError4));
    float* qp = (float*)malloc((size_t)qb);
    if (!e || !qp) { free(e); free(qp); free(f); return fail("out of memory"); }
    memcpy(qp, f + E4_HEADER, (size_t)qb);
    for (uint32_t i = 0; i < n; ++i)
        if (!isfinite(qp[2 * i]) || qp[2 * i] < 0.0f || !isfinite(qp[2 * i + 1])) {
            free(e); free(qp); free(f);
            return fail("%s: ERROR4 qparams of row %u are invalid", path, i);
        }
    e->file = f;
    e->qparams = qp;
    e->blocks = f + E4_HEADER + qb;
    e->blocks_bytes = (int64_t)blocks;
    e->num_vectors = b->n;
    e->dim = b->dim;
    *out = e;
    return 0;
}

int rover_split_bias_open(const RoverBundle* b, const char* path, float** out) {
    *out = NULL;
    if (b->method != 0 || b->sq.l1_bits != 4 || (b->residual_bits != 4 && b->residual_bits != 8))
        return fail("split distance needs 4-bit L1 codes with 4- or 8-bit residuals");
    const uint64_t payload = (uint64_t)b->n * 4u;
    uint8_t* f = NULL;
    size_t len = 0;
    if (slurp(path, &f, &len) != 0) return -1;
    /* source fingerprint: the first 16 bytes of SHA-256 over the three base
       members' digests */
    uint8_t hashes[96], fp[32];
    for (int i = 0; i < 3; ++i)
        if (!b->base_paths[i][0] || rover_sha256_file(b->base_paths[i], 0, hashes + 32 * i) != 0) {
            free(f);
            return fail("%s: cannot hash the base members", path);
        }
    rover_sha256(hashes, sizeof(hashes), fp);
    const uint8_t* h = f;
    int ok = len == BIAS_HEADER + payload && memcmp(h, "SQMDBIAS", 8) == 0 && rd32(h + 8) == 1 &&
             rd32(h + 12) == BIAS_HEADER && rd32(h + 16) == (uint32_t)b->n && rd32(h + 20) == (uint32_t)b->dim &&
             rd32(h + 24) == (uint32_t)b->sq.l1_bits && rd32(h + 28) == (uint32_t)b->residual_bits &&
             rd64(h + 32) == payload && memcmp(h + 48, fp, 16) == 0;
    if (!ok) { free(f); return fail("%s: bias header does not match the index", path); }
    uint64_t hash = UINT64_C(14695981039346656037);
    for (uint64_t i = 0; i < payload; ++i) {
        hash ^= f[BIAS_HEADER + i];
        hash *= UINT64_C(1099511628211);
    }
    if (hash != rd64(h + 40)) { free(f); return fail("%s: bias payload hash mismatch", path); }
    float* bias = (float*)malloc((size_t)payload);
    if (!bias) { free(f); return fail("out of memory"); }
    memcpy(bias, f + BIAS_HEADER, (size_t)payload);
    free(f);
    for (int32_t i = 0; i < b->n; ++i)
        if (!isfinite(bias[i])) { free(bias); return fail("%s: bias of row %d is not finite", path, i); }
    *out = bias;
    return 0;
}
