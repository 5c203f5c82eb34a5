/*
 * rover_oracle.h -- CPU restatement of Rover's quantized graph-search path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load this library, and only as the checker.
 * The product path (rover_b200/libcalculator.so) never links or calls it.
 *
 * Every function restates the reference function cited beside it, with the
 * same operation order, so FP32 results are bit-identical when compiled with
 * -O2 -ffp-contract=off.  The restatement itself is pinned against the
 * compiled reference (oracle/_ref) and the golden fixtures in tests/golden/.
 */
#ifndef ROVER_ORACLE_H
#define ROVER_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Index views (flat device-style layouts, ids are graph ids). */
typedef struct {
    const int32_t *graph;       /* [n][degree], -1 padded rows            */
    int32_t n, degree, dim;
    const uint8_t *codes;       /* [n][code_bytes]                        */
    const float *codebook;      /* [m][ks][subdim]                        */
    int32_t m, ks, subdim, code_bytes;
    const uint8_t *residual;    /* .pqresN payload: 4096-B blocks         */
    int32_t residual_bits, residual_code_bytes, vectors_per_block;
    const float *qparams;       /* [n][2] = {scale, zero}                 */
} OraclePqIndex;

typedef struct {
    const int32_t *graph;
    int32_t n, degree, dim;
    const uint8_t *l1;          /* [n][l1_code_bytes]                     */
    int32_t l1_bits, l1_code_bytes;
    float l1_scale, l1_zero;
    const uint8_t *residual;    /* flat [n][residual_code_bytes] or NULL  */
    int32_t residual_bits, residual_code_bytes;
    const float *qparams;       /* [n][2]                                 */
} OracleSqIndex;

/* stats: {scored, corrected, expanded, dedup_skips} */
int oracle_pq_build_lut(const OraclePqIndex *ix, const float *query, float *lut);
int oracle_pq_adc(const OraclePqIndex *ix, const float *lut, const int32_t *ids, int count,
                  float *out);
int oracle_pq_residual_eval(const OraclePqIndex *ix, const float *query, const int32_t *ids,
                            int count, float *out);
int oracle_pq_decode(const OraclePqIndex *ix, int id, float *out);
int oracle_pq_seed_ids(int n, int entry_count, int graph_entry, uint32_t seed, int32_t *ids);
int oracle_pq_search(const OraclePqIndex *ix, const float *query, const int32_t *entry_ids,
                     int entry_count, int expand_count, int pool_capacity, int num_out,
                     int correction, int32_t *out_ids, float *out_dists, uint64_t *stats);

int oracle_sq_quantize(const OracleSqIndex *ix, const float *query, uint8_t *out);
float oracle_sq_coarse(const OracleSqIndex *ix, const uint8_t *query_code, int id);
float oracle_sq_exact(const OracleSqIndex *ix, const float *query, int id);
int oracle_sq_rerank(const OracleSqIndex *ix, const float *query, int32_t *ids, float *dists, int count,
                     int top_k, int32_t *out_ids, float *out_dists);
int oracle_sq_seed_ids(int n, int entry_points, int graph_entry, uint32_t seed, int32_t *ids,
                       int capacity);
int oracle_sqmd_search(const OracleSqIndex *ix, const float *query, int entry_points,
                       int graph_entry, uint32_t seed, int expand_count, int pool_capacity,
                       int correction, int32_t *out_ids, float *out_dists, int out_capacity,
                       uint64_t *stats);
int oracle_dsp_search(const OracleSqIndex *ix, const float *query, int entry_points,
                      int graph_entry, int expand_count, int pool_size, int num_out,
                      int32_t *out_ids, float *out_dists);

/* final refine, mode CURRENT: kind 0 = SQ decode, 1 = PQ residual decode */
int oracle_refine(int kind, const void *index, const float *query, const int32_t *ids,
                  int count, int output_k, int32_t *out_ids, float *out_dists);

/* Third-level ERROR4 artifact payload (PQERR4V1 / SQERR4V1 after the
 * 256-byte header): per storage row {scale, zero}, then 4096-byte blocks of
 * ceil(dim/2)-byte int4 codes, low nibble first. */
typedef struct {
    const float *qparams;        /* [n][2]                                 */
    const uint8_t *blocks;       /* vectors_per_block rows per 4096 bytes  */
    int32_t code_bytes, vectors_per_block;
} OracleError4;

/* final refine in mode ERROR4 when e4 != NULL (mode CURRENT otherwise) */
int oracle_refine_ex(int kind, const void *index, const OracleError4 *e4, const float *query,
                     const int32_t *ids, int count, int output_k, int32_t *out_ids, float *out_dists);

/* SQ4 split distance: the L1-aligned u8 query, the u8-vs-4-bit L1 code
 * distance, the residual delta bias[id] - 2 q.r and their sum. */
typedef struct {
    uint8_t q[1024];
    uint64_t sum_q;
} OracleSplitQuery;

int oracle_split_query(const OracleSqIndex *ix, const float *query, OracleSplitQuery *out);
float oracle_split_coarse(const OracleSqIndex *ix, const OracleSplitQuery *sq, int id);
float oracle_split_delta(const OracleSqIndex *ix, const float *bias, const OracleSplitQuery *sq, int id);
float oracle_split_distance(const OracleSqIndex *ix, const float *bias, const OracleSplitQuery *sq, int id);
/* oracle_sqmd_search with split distances (correction on, 4-bit L1 codes) */
int oracle_sqmd_search_split(const OracleSqIndex *ix, const float *bias, const float *query,
                             int entry_points, int graph_entry, uint32_t seed, int expand_count,
                             int pool_capacity, int32_t *out_ids, float *out_dists, int out_capacity,
                             uint64_t *stats);

/* batch helpers (threads over queries) */
int oracle_pq_search_batch(const OraclePqIndex *ix, const float *queries, int nq,
                           const int32_t *pool_sizes, int entry_points, int graph_entry,
                           uint32_t seed, int expand_count, int correction, int refine_budget,
                           int top_k, int threads, int32_t *pool_ids, float *pool_dists,
                           int pool_stride, int32_t *pool_counts, int32_t *out_ids,
                           float *out_dists, int out_stride, int32_t *out_counts,
                           uint64_t *stats);

#ifdef __cplusplus
}
#endif

#endif
