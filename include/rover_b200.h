/*
 * rover_b200.h -- batched extension entry points of libcalculator.so.
 *
 * The reference's accelerator interface (calculator.h) is per query: the
 * host drives every expansion of every query through FastRPC lane buffers.
 * On a GPU that protocol cannot fill 148 SMs, so the library adds batch
 * entry points that run thousands of complete searches in one launch.  They
 * follow the reference's conventions: plain C types, pointer + length
 * arguments, AEE result codes (calculator.h), and the reference's search
 * semantics, cited per entry.  No CUDA or torch types appear here; device
 * buffers and streams are passed as plain pointers.
 */
#ifndef ROVER_B200_H
#define ROVER_B200_H

#include <stdint.h>

#include "calculator.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Status values reported per query (out_status arrays). */
#define ROVER_QUERY_OK 0
#define ROVER_QUERY_BAD_ROW 1        /* graph row breaks the valid-prefix rule */
#define ROVER_QUERY_NUMERIC 2        /* non-finite distance or invalid qparams */
#define ROVER_QUERY_TABLE_FULL 3     /* internal: retried with a larger table  */
#define ROVER_QUERY_BAD_PARAM 4
#define ROVER_QUERY_FRONTIER_FULL 5

/* Search modes. */
#define ROVER_MODE_EXACT 0   /* reference expansion order, bit-exact results */

/* Residual layouts for PQ searches with correction (RoverSearchParams.layout).
 * Both give identical results; they trade device memory for arithmetic. */
#define ROVER_LAYOUT_AUTO 0     /* decoded when it fits, else packed */
#define ROVER_LAYOUT_PACKED 1   /* .pqresN rows decoded per candidate */
#define ROVER_LAYOUT_DECODED 2  /* FP32 rows ((c + code*s) + z) built once per index */

/* A pure-PQ index held in host memory (layouts of the reference bundle:
 * graph.rover rows, .pqcodes / .pqbook payloads, .pqresN block payload,
 * .pqresN.qparams payload).  Loaded once; the library keeps a device copy. */
typedef struct RoverPqIndexDesc {
    const int32_t *graph;            /* [num_vectors][graph_degree], -1 padded */
    int32_t num_vectors;
    int32_t graph_degree;
    int32_t graph_entry;             /* -1 = none */
    int32_t dim;
    const uint8_t *codes;            /* [num_vectors][code_bytes] */
    const float *codebook;           /* [m][ks][subdim] */
    int32_t m, ks, subdim, code_bytes;
    const uint8_t *residual_blocks;  /* 4096-byte blocks, 4096/rcb rows each */
    int64_t residual_blocks_bytes;
    int32_t residual_bits;           /* 0 = no residuals, else 4 or 8 */
    const float *residual_qparams;   /* [num_vectors][2] {scale, zero} */
} RoverPqIndexDesc;

/* An SQ index held in host memory (l1.bin payload, residual rows, qparams). */
typedef struct RoverSqIndexDesc {
    const int32_t *graph;
    int32_t num_vectors, graph_degree, graph_entry, dim;
    const uint8_t *l1_codes;         /* [num_vectors][l1_code_bytes] */
    int32_t l1_bits;                 /* 4 or 8 */
    float l1_scale, l1_zero;
    const uint8_t *residual_rows;    /* [num_vectors][rcb] or NULL */
    int32_t residual_bits;
    const float *residual_qparams;   /* [num_vectors][2] or NULL */
} RoverSqIndexDesc;

/* Per-call search options (all searches of one call share them). */
typedef struct RoverSearchParams {
    int32_t size;            /* sizeof(RoverSearchParams) */
    int32_t mode;            /* ROVER_MODE_* */
    int32_t entry_points;    /* seed count (graph entry first, then LCG) */
    uint32_t seed;           /* LCG seed, reference default 42 */
    int32_t expand_count;    /* neighbours read per expansion (<= degree) */
    int32_t correction;      /* 0 = coarse distances, 1 = online residual */
    int32_t refine_budget;   /* 0 = no final refine, else candidates re-ranked */
    int32_t top_k;           /* results per query when top_ks is NULL */
    int32_t pool_stride;     /* columns of the optional pool output */
    int32_t sq_mode;         /* SQ only: 0 = device search (calculator_retrieval_search),
                                1 = SQMD session semantics */
    int32_t layout;          /* PQ with correction: ROVER_LAYOUT_* */
    int32_t reserved[5];
} RoverSearchParams;

/* Per-call outputs.  Host pointers for calculator_rover_*_search, device
 * pointers for the *_device variants.  Any of pool_*, stats, status may be
 * NULL. */
typedef struct RoverSearchOutputs {
    int32_t *ids;            /* [nq][top_k stride] */
    float *dists;
    int32_t *counts;         /* [nq] */
    int32_t out_stride;
    int32_t *pool_ids;       /* [nq][pool_stride] sorted pool */
    float *pool_dists;
    int32_t *pool_counts;
    uint64_t *stats;         /* [nq][4] {scored, corrected, expanded, dedup} */
    int32_t *status;         /* [nq] ROVER_QUERY_* */
} RoverSearchOutputs;

/* Load / replace the handle's PQ index.  Reference counterpart:
 * calculator_retrieval_pure_pq_load_dma (retrieval_async_dsp_search.c:698)
 * plus the host's residual index open (retrieval_pq_residual.c:716). */
AEEResult calculator_rover_pq_load(remote_handle64 h, const RoverPqIndexDesc *desc);
AEEResult calculator_rover_pq_unload(remote_handle64 h);

/* Batched pure-PQ search (host buffers in and out).  Per query: the search
 * of retrieval_pure_pq_search_scalar_with_policy (retrieval_sqmd_pure_pq.c:793)
 * seeded as pure_pq_run_one_query_limited does (retrieval_rpc_demo_pure_pq.c:210),
 * then, with refine_budget > 0, retrieval_final_refine (retrieval_final_refine.c:294).
 * pool_sizes[nq] is the beam width L of each query (uneven widths allowed);
 * top_ks[nq] (or params->top_k when NULL) the result count.  Returns
 * AEE_SUCCESS when every query succeeded, else AEE_EFAILED with per-query
 * codes in out->status. */
AEEResult calculator_rover_pq_search(remote_handle64 h, const RoverSearchParams *params,
                                     const float *queries, int32_t num_queries,
                                     const int32_t *pool_sizes, const int32_t *top_ks,
                                     const RoverSearchOutputs *out);
/* Same with device-resident queries, sizes and outputs, enqueued on
 * `stream` (a cudaStream_t, NULL = the library's stream); returns after the
 * work completes. */
AEEResult calculator_rover_pq_search_device(remote_handle64 h, const RoverSearchParams *params,
                                            const float *queries, int32_t num_queries,
                                            const int32_t *pool_sizes, const int32_t *top_ks,
                                            const RoverSearchOutputs *out, void *stream);

/* Allocation-free variant of calculator_rover_pq_search_device.  It has no
 * counterpart in the reference: it exists for callers that cannot allocate
 * device memory while they search -- a server whose memory pool already owns
 * the GPU, or a latency-bound loop that must not take cudaMalloc/cudaFree's
 * implicit synchronization.  Nothing is allocated per call: the kernel's
 * visited tables, work counter and error flag live in a fixed 64 MiB device
 * array inside the library (held by every GPU that loads the library until
 * the process exits).  All pointers are device pointers; out->status is
 * required; max_pool must bound every pool_sizes[i] (the sizes are not read
 * back).  A request whose visited tables cannot fit the array is rejected
 * with AEE_EBADPARM, and a query that overflows its table fails the call
 * (AEE_EFAILED) instead of being retried.  The first call on each device
 * resolves the array's device address (cudaGetSymbolAddress) and clears it;
 * make that first call before any stream capture.  Calls share the array:
 * two calls whose kernels overlap on the GPU race, so issue them one after
 * another.  stream is a cudaStream_t (NULL = the legacy default stream). */
AEEResult calculator_rover_pq_search_noalloc(remote_handle64 h, const RoverSearchParams *params,
                                             const float *queries, int32_t num_queries,
                                             const int32_t *pool_sizes, int32_t max_pool,
                                             const int32_t *top_ks, const RoverSearchOutputs *out,
                                             void *stream);

/* Distances for explicit (query, id) lists: ids[offsets[q] .. offsets[q+1]).
 * kind 0 = PQ ADC (retrieval_pq_adc_ids_batch, retrieval_pq_core.c:332),
 * 1 = PQ residual-corrected (retrieval_pq_residual_query_evaluate,
 * retrieval_pq_residual.c:983), 2 = SQ coarse
 * (retrieval_compute_int8/int4 distance, retrieval_l1_int8_core.c:463-489),
 * 3 = SQ exact residual (retrieval_demo_exact_distance_residual,
 * retrieval_rpc_demo_support.c:1577). */
AEEResult calculator_rover_score(remote_handle64 h, int32_t kind, const float *queries,
                                 int32_t num_queries, const int32_t *ids, const int64_t *offsets,
                                 float *out_dists, int32_t *out_status);
/* Per-query PQ lookup tables [nq][m*ks] (retrieval_pq_build_lut, retrieval_pq_core.c:362). */
AEEResult calculator_rover_pq_lut(remote_handle64 h, const float *queries, int32_t num_queries,
                                  float *out_luts, int32_t *out_status);

/* Final refine of host-supplied candidate lists (refine_impl,
 * retrieval_final_refine.c:256): kind 0 = SQ decode, 1 = PQ residual decode. */
AEEResult calculator_rover_refine(remote_handle64 h, int32_t kind, const float *queries,
                                  int32_t num_queries, const int32_t *cand_ids, int32_t cand_stride,
                                  const int32_t *cand_counts, int32_t top_k, int32_t *out_ids,
                                  float *out_dists, int32_t *out_counts, int32_t *out_status);

/* SQ index and batched SQ search (sq_mode 0: calculator_retrieval_search,
 * retrieval_async_dsp_search.c:368; sq_mode 1: the SQMD loop,
 * retrieval_sqmd_common.c:2052 with the exact residual correction). */
AEEResult calculator_rover_sq_load(remote_handle64 h, const RoverSqIndexDesc *desc);
AEEResult calculator_rover_sq_unload(remote_handle64 h);
AEEResult calculator_rover_sq_search(remote_handle64 h, const RoverSearchParams *params,
                                     const float *queries, int32_t num_queries,
                                     const int32_t *pool_sizes, const RoverSearchOutputs *out);

/* Last CUDA / library error as text (thread-local). */
const char *calculator_rover_last_error(void);

/* Number of CUDA kernels this library has launched in this process. */
uint64_t calculator_rover_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* ROVER_B200_H */
