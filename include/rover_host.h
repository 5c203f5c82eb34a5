/*
 * rover_host.h -- the C host side of the B200 search path: Rover's index
 * bundle loader and its checks, and the vector / graph file readers the
 * `Rover search` command uses (librover_host.so, built with the `Rover`
 * executable).
 *
 * The reference prepares and validates a bundle in Python
 * (tools/index_bundle.py:187-226 validate, :229-345 prepare) and loads its
 * members in C (src/dsp_demo/retrieval_pq_artifact.c:886-958 for .pqbook /
 * .pqcodes, retrieval_pq_residual.c:716-835 for .pqresN / .qparams,
 * retrieval_rpc_demo_support.c:1968 for l1.bin / qparams.bin / residual.bin,
 * retrieval_rpc_demo_graph_index.c:1296 for graphs, support.c:2201/2234 for
 * fvecs / ivecs).  This library does both in C: it reads index.json, checks
 * every member's size and SHA-256, parses and cross-checks the binary
 * headers, and hands back host buffers in the layout of RoverPqIndexDesc /
 * RoverSqIndexDesc (rover_b200.h), ready for calculator_rover_pq_load /
 * calculator_rover_sq_load.
 *
 * Every function returns 0 on success and -1 on failure with a message in
 * rover_host_error().
 */
#ifndef ROVER_HOST_H
#define ROVER_HOST_H

#include <stddef.h>
#include <stdint.h>

#include "rover_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- SHA-256 (FIPS 180-4) ---- */
typedef struct RoverSha256 {
    uint32_t h[8];
    uint64_t bytes;
    uint8_t buf[64];
    size_t fill;
} RoverSha256;

void rover_sha256_init(RoverSha256 *s);
void rover_sha256_update(RoverSha256 *s, const void *data, size_t len);
void rover_sha256_final(RoverSha256 *s, uint8_t out[32]);
void rover_sha256(const void *data, size_t len, uint8_t out[32]);
/* digest of the file's bytes from `offset` to the end */
int rover_sha256_file(const char *path, long long offset, uint8_t out[32]);
/* lower-case hex of `len` bytes into out[2 * len + 1] */
void rover_hex(const uint8_t *bytes, size_t len, char *out);

/* ---- vectors and graphs ---- */
/* The first `count` vectors of an fvecs / ivecs file (each record: int32
 * dimension, then `dim` values); every record must have dimension `dim`.
 * *out is malloc'd [count][dim]. */
int rover_read_fvecs(const char *path, int32_t count, int32_t dim, float **out);
int rover_read_ivecs(const char *path, int32_t count, int32_t dim, int32_t **out);
/* A dense INT32 adjacency [n][degree], -1 padded, in one of the reference's
 * graph formats: "rover" (16-byte header 0x35314252, n, dim, degree),
 * "dense" (raw rows), "nndescent" (int32 n, degree, pad; then per vector
 * `degree` ids and `degree` float distances).  Ids must lie in [-1, n). */
int rover_read_graph(const char *path, const char *format, int32_t n, int32_t dim, int32_t degree,
                     int32_t **out);
/* index_bundle.py's graph checks: no self edges, no duplicate edges. */
int rover_check_graph(const int32_t *graph, int32_t n, int32_t degree);

/* ---- index bundles ---- */
typedef struct RoverBundle {
    int32_t method;                 /* 0 = SQ, 1 = PQ */
    int32_t n, dim, degree, graph_entry, residual_bits;
    int32_t *graph;                 /* [n][degree] */
    /* PQ members (method 1) */
    RoverPqIndexDesc pq;            /* points into the buffers below */
    float *pq_codebook;
    uint8_t *pq_codes;
    uint8_t *pq_residual_blocks;
    float *pq_qparams;
    uint8_t index_uuid[16];
    /* SQ members (method 0) */
    RoverSqIndexDesc sq;
    uint8_t *sq_l1;
    uint8_t *sq_residual_rows;      /* unpacked [n][residual code bytes] */
    float *sq_qparams;
    /* the member files the index came from: PQ codes, residual, qparams (or
       SQ l1, residual, qparams), and the PQ codebook -- the digests the
       correction artifacts below are bound to */
    char base_paths[3][4096];
    char pq_book_path[4096];
} RoverBundle;

/* A rover.index.v1 directory: validate index.json (schema, method, sizes,
 * required members, paths inside the directory, sizes and -- with verify --
 * SHA-256 of every member, PQ member names), read the graph and the method's
 * members, check their headers against each other and the manifest. */
int rover_bundle_open_dir(const char *dir, int verify, RoverBundle **out);
/* The same members named one by one (the CLI's --graph / --pq-* options).
 * residual_bits 0 = no residuals. */
int rover_bundle_open_pq(const char *graph_path, const char *graph_format, int32_t n, int32_t dim,
                         int32_t degree, int32_t graph_entry, const char *pq_book, const char *pq_codes,
                         const char *pq_residual, const char *pq_qparams, int32_t residual_bits, int verify,
                         RoverBundle **out);
int rover_bundle_open_sq(const char *graph_path, const char *graph_format, int32_t n, int32_t dim,
                         int32_t degree, int32_t graph_entry, const char *l1, const char *residual,
                         const char *qparams, RoverBundle **out);
void rover_bundle_close(RoverBundle *b);

const char *rover_host_error(void);

/* ---- correction artifacts ---- */
/* The final refine's third-level ERROR4 file (PQERR4V1 / SQERR4V1), checked
 * as retrieval_final_refine.c:118-166 does against the bundle it refines
 * (the base members' and the PQ codebook's SHA-256, the id maps: the order
 * map graph -> original when one is used, else none) and loaded. */
typedef struct RoverError4 {
    int32_t num_vectors, dim;
    float *qparams;                 /* [n][2] {scale >= 0, zero}            */
    const uint8_t *blocks;          /* 4096-byte code blocks                */
    int64_t blocks_bytes;
    uint8_t *file;                  /* owns blocks                          */
} RoverError4;
int rover_error4_open(const RoverBundle *b, const char *path, const int32_t *graph_to_original, RoverError4 **out);
void rover_error4_close(RoverError4 *e);
/* The SQMD split-distance bias (SQMDBIAS, retrieval_rpc_demo_support.c:
 * 237-297): *out is malloc'd [n] floats. */
int rover_split_bias_open(const RoverBundle *b, const char *path, float **out);
/* message of the last failed artifact call on this thread */
const char *rover_artifact_error(void);

/* ---- neighbourhood-aware layout ---- */
/* The reference's clustered block ordering of a graph's ids (rover-layout,
 * src/graph/layout_opt_kmeans.cpp:55-712): graph [n][degree] (-1 padded
 * rows), one cluster label per node in [0, clusters); new_to_old[n]
 * receives, per new id, the old id.  rrf_c, max_reverse (0 = no limit),
 * use_cn / use_mnn as the tool's arguments; `threads` host threads.
 * 0 on success, -1 on invalid input. */
int rover_layout_order(const int32_t *graph, int32_t n, int32_t degree, const int32_t *labels, int32_t clusters,
                       int32_t vectors_per_block, double rrf_c, int32_t max_reverse, int32_t use_cn,
                       int32_t use_mnn, int32_t threads, int32_t *new_to_old);

#ifdef __cplusplus
}
#endif

#endif /* ROVER_HOST_H */
