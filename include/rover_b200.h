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
#define ROVER_QUERY_SEED_RANK 6      /* a plan's tensor-core seed ranking gave up waiting */

/* Search modes. */
#define ROVER_MODE_EXACT 0    /* reference expansion order, bit-exact results */
#define ROVER_MODE_BATCHED 1  /* free-running: beam_width pool entries expanded per step,
                                 every candidate corrected (PQ with correction only;
                                 expand_count <= 64) */
#define ROVER_MODE_GATED 2    /* batched, with the learned gate choosing which candidates
                                 are corrected and when a query stops expanding;
                                 without a loaded gate it runs as ROVER_MODE_BATCHED */

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
                                1 = SQMD session semantics, 2 = DB-pair search
                                (calculator_retrieval_search_db: the device search with
                                each expansion candidate's exact residual distance when
                                correction is on) */
    int32_t layout;          /* PQ with correction: ROVER_LAYOUT_* */
    int32_t beam_width;      /* BATCHED / GATED: entries expanded per step, 1..4 (0 = the
                                largest with beam_width * expand_count <= 256) */
    int32_t third_residual;  /* PQ with refine_budget > 0: the final refine in mode ERROR4
                                (retrieval_final_refine.c:118-166, :221-246), adding the
                                artifact loaded by calculator_rover_error4_load to every
                                decoded candidate */
    int32_t split_distance;  /* SQ, sq_mode 1 with correction: the SQ4 split distance
                                (SQMD_SPLIT_DISTANCE on, retrieval_rpc_demo_pipeline.c:909-995)
                                with the bias loaded by calculator_rover_sq_split_load */
    int32_t reserved[2];
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
 * implicit synchronization.  It runs the exact search (params->mode
 * ROVER_MODE_EXACT) over the packed residual rows (params->layout AUTO or
 * PACKED) and refuses other modes and layouts with AEE_EBADPARM.  Nothing is
 * allocated per call: the kernel's
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

/* ---- search plans: one set of searches replayed on new queries ----------
 *
 * The reference serves queries one at a time; a plan serves thousands with
 * uneven beam widths and result counts (pool_sizes[i], top_ks[i], fixed when
 * the plan is made) as a fixed sequence of kernels: a bookkeeping kernel,
 * the all-queries entry-seed pass, one persistent search launch per
 * beam-width class (queries sorted by width, widest first, so each class's
 * shared-memory slices fit its widest query) and a second bookkeeping
 * kernel.  A launch allocates nothing, never waits on the host and reads its
 * per-launch state (visited-table generations, work counters) from device
 * memory, so a CUDA graph captured from one launch can be replayed on new
 * vectors written into the same query buffer.
 *
 * With tune_queries (device, [num_queries][dim]), creation times the
 * configurations that leave results unchanged -- warps per CTA (2, 4, 8),
 * shared-memory visited slots per warp (1024, 2048, 4096), beam-width
 * classes (one, two, one per power of two), and for ROVER_MODE_EXACT the
 * packed or decoded residual layout -- and keeps the fastest.  Every
 * configuration returns the same ids and distances as
 * calculator_rover_pq_search on the same inputs.
 *
 * A plan copies the entry seeds (and the loaded gate, for ROVER_MODE_GATED)
 * when it is made and refers to the loaded PQ index: destroy plans, and the
 * graphs captured from them, before unloading or replacing the index. */
#define ROVER_PLAN_MAX_CLASSES 8

typedef struct RoverPlanInfo {
    int32_t num_queries;
    int32_t mode;                    /* ROVER_MODE_* */
    int32_t layout;                  /* ROVER_LAYOUT_PACKED or ROVER_LAYOUT_DECODED */
    int32_t warps_per_cta;
    int32_t shared_visited_slots;    /* per warp; 0 for the packed layout */
    int32_t classes;                 /* beam-width classes = search launches */
    int32_t launches;                /* kernels one plan launch enqueues */
    int32_t candidates;              /* configurations timed at creation (0 = untuned) */
    int32_t max_pool;
    int32_t beam_width;              /* batched / gated modes */
    int32_t class_pool[ROVER_PLAN_MAX_CLASSES];     /* widest beam of each class */
    int32_t class_queries[ROVER_PLAN_MAX_CLASSES];
    int32_t class_blocks[ROVER_PLAN_MAX_CLASSES];   /* CTAs of each class launch */
    float tuned_ms;                  /* the kept configuration's launch time (0 = untuned) */
    float default_ms;                /* the untuned default's launch time (0 = untuned) */
    int64_t device_bytes;            /* device memory held by the plan */
    int32_t class_split;             /* RoverPlanConfig.class_split of the kept configuration */
    int32_t reserved[7];
} RoverPlanInfo;

/* One plan configuration (every one gives the same results). */
typedef struct RoverPlanConfig {
    int32_t layout;                  /* ROVER_LAYOUT_PACKED or ROVER_LAYOUT_DECODED */
    int32_t warps_per_cta;           /* 1..8 (the packed layout runs 4) */
    int32_t shared_visited_slots;    /* per warp, power of two 256..8192 (decoded layout) */
    int32_t class_split;             /* 0: one class, 1: two, 2: one per power of two of the beam width */
} RoverPlanConfig;

typedef struct RoverPqPlan RoverPqPlan;   /* opaque */

/* pool_sizes and top_ks (NULL = params->top_k) are host arrays of
 * num_queries entries.  tune_queries may be NULL (no tuning: decoded layout
 * when available, 4 warps, 2048 slots, one class). */
AEEResult calculator_rover_pq_plan_create(remote_handle64 h, const RoverSearchParams *params,
                                          int32_t num_queries, const int32_t *pool_sizes,
                                          const int32_t *top_ks, const float *tune_queries,
                                          RoverPqPlan **plan);
/* A plan with a given configuration, e.g. one that an earlier tuned plan
 * reported (calculator_rover_pq_plan_describe), without timing anything. */
AEEResult calculator_rover_pq_plan_create_fixed(remote_handle64 h, const RoverSearchParams *params,
                                                int32_t num_queries, const int32_t *pool_sizes,
                                                const int32_t *top_ks, const RoverPlanConfig *config,
                                                RoverPqPlan **plan);
/* Enqueues the plan's searches on stream (a cudaStream_t, NULL = the
 * library's stream) and returns without waiting.  queries and every output
 * pointer are device pointers; out->status is required and is rewritten by
 * every launch (ROVER_QUERY_TABLE_FULL marks a query whose visited table
 * overflowed: rerun it through calculator_rover_pq_search). */
AEEResult calculator_rover_pq_plan_launch(RoverPqPlan *plan, const float *queries,
                                          const RoverSearchOutputs *out, void *stream);
AEEResult calculator_rover_pq_plan_describe(const RoverPqPlan *plan, RoverPlanInfo *info);
AEEResult calculator_rover_pq_plan_destroy(RoverPqPlan *plan);

/* Distances for explicit (query, id) lists: ids[offsets[q] .. offsets[q+1]).
 * kind 0 = PQ ADC (retrieval_pq_adc_ids_batch, retrieval_pq_core.c:332),
 * 1 = PQ residual-corrected (retrieval_pq_residual_query_evaluate,
 * retrieval_pq_residual.c:983), 2 = SQ coarse
 * (retrieval_compute_int8/int4 distance, retrieval_l1_int8_core.c:463-489),
 * 3 = SQ exact residual (retrieval_demo_exact_distance_residual,
 * retrieval_rpc_demo_support.c:1577), 4 = kind 1 computed from the decoded
 * rows (same values bit for bit; builds them on first use; dim % 4 == 0,
 * dim <= 384). */
AEEResult calculator_rover_score(remote_handle64 h, int32_t kind, const float *queries,
                                 int32_t num_queries, const int32_t *ids, const int64_t *offsets,
                                 float *out_dists, int32_t *out_status);
/* Per-query PQ lookup tables [nq][m*ks] (retrieval_pq_build_lut, retrieval_pq_core.c:362). */
AEEResult calculator_rover_pq_lut(remote_handle64 h, const float *queries, int32_t num_queries,
                                  float *out_luts, int32_t *out_status);

/* PQ codebook training on the GPU: retrieval_pq_train
 * (retrieval_pq_core.c:202-224 over retrieval_pq_train_subspace :97-200),
 * bit for bit: per subspace, centroid k starts as training vector
 * k (count-1) / (ks-1) and kmeans_iters (at least 1) Lloyd iterations follow,
 * with the reference's FP32 distances, first-minimum ties and member sums in
 * vector order.  train_vectors [train_count][dim] (host, finite), codebook
 * out [m][ks][dim/m] (host).  ks in 1..256, dim % m == 0. */
AEEResult calculator_rover_pq_train(remote_handle64 h, const float *train_vectors, int32_t train_count,
                                    int32_t dim, int32_t m, int32_t ks, int32_t kmeans_iters,
                                    float *out_codebook);
/* PQ encoding on the GPU: retrieval_pq_encode_batch (retrieval_pq_core.c:
 * 226-268): the nearest centroid of every subspace (first minimum), codes
 * [count][code_bytes] with two 4-bit codes per byte (low nibble first) when
 * ks <= 16.  AEE_EBADPARM on a non-finite distance, as the reference fails. */
AEEResult calculator_rover_pq_encode(remote_handle64 h, const float *vectors, int64_t count, int32_t dim,
                                     const float *codebook, int32_t m, int32_t ks, uint8_t *out_codes);

/* The third-level ERROR4 artifact of the loaded index (kind 0 = the SQ index
 * of calculator_rover_sq_load, 1 = the PQ index): the payload of a
 * SQERR4V1 / PQERR4V1 file after its 256-byte header (retrieval_final_refine.c:
 * 118-166 validates the header; the host does that before calling), i.e.
 * qparams[num_vectors][2] {scale >= 0, zero}, then code_blocks: 4096-byte
 * blocks of 4096 / ceil(dim/2) rows of ceil(dim/2) int4 codes, low nibble
 * first.  Rows are graph ids (no storage map).  Unloading or replacing the
 * index drops it. */
AEEResult calculator_rover_error4_load(remote_handle64 h, int32_t kind, const float *qparams,
                                       const uint8_t *code_blocks, int64_t code_blocks_bytes,
                                       int32_t num_vectors, int32_t dim);
AEEResult calculator_rover_error4_unload(remote_handle64 h, int32_t kind);

/* The SQ4 split-distance bias of the loaded SQ index (the payload of a
 * SQMDBIAS file after its 64-byte header, one finite float per vector;
 * sqmd_load_correction_bias, retrieval_rpc_demo_support.c:237-297, holds the
 * header checks).  Needs 4-bit L1 codes and residuals. */
AEEResult calculator_rover_sq_split_load(remote_handle64 h, const float *bias, int32_t num_vectors);

/* Final refine of host-supplied candidate lists (refine_impl,
 * retrieval_final_refine.c:256): kind 0 = SQ decode, 1 = PQ residual decode.
 * kind 2 = the legacy SQ re-rank demo_rerank_candidates
 * (retrieval_rpc_demo_support.c:1833): stable sort by id, exact residual
 * distance (retrieval_demo_exact_distance_residual, :1397; FLT_MAX for an id
 * outside the index), stable sort by distance, first top_k; no reorder map.
 * kinds 3 / 4 = kinds 0 / 1 in mode ERROR4 (the index's loaded ERROR4
 * artifact added to each decode, decode_vector :221-246).
 * At most 2048 candidates per query. */
AEEResult calculator_rover_refine(remote_handle64 h, int32_t kind, const float *queries,
                                  int32_t num_queries, const int32_t *cand_ids, int32_t cand_stride,
                                  const int32_t *cand_counts, int32_t top_k, int32_t *out_ids,
                                  float *out_dists, int32_t *out_counts, int32_t *out_status);

/* SQ index and batched SQ search (sq_mode 0: calculator_retrieval_search,
 * retrieval_async_dsp_search.c:368; sq_mode 1: the SQMD loop,
 * retrieval_sqmd_common.c:2052 with the exact residual correction; sq_mode 2:
 * calculator_retrieval_search_db's per-query search,
 * retrieval_async_dsp_search.c:1205-1581, with the host correction of
 * retrieval_rpc_demo_pipeline.c:454-495 applied on the device). */
AEEResult calculator_rover_sq_load(remote_handle64 h, const RoverSqIndexDesc *desc);
AEEResult calculator_rover_sq_unload(remote_handle64 h);
AEEResult calculator_rover_sq_search(remote_handle64 h, const RoverSearchParams *params,
                                     const float *queries, int32_t num_queries,
                                     const int32_t *pool_sizes, const RoverSearchOutputs *out);

/* ---- learned gate (ROVER_MODE_GATED) ----------------------------------
 * A 5 -> 64 -> 64 -> 2 MLP with ReLU hidden layers.  Inputs per row: log
 * quantized (ADC) distance, pool rank / L, log worst-in-pool distance,
 * hop count / L, query norm; each standardised with mu / sigma.  Outputs:
 * refine-needed logit, stop-expanding logit.  Weights are FP32 row-major
 * [in][out] here and BF16 on the device; accumulation is FP32. */
#define ROVER_GATE_IN 5
#define ROVER_GATE_HIDDEN 64
#define ROVER_GATE_OUT 2
/* Packed parameter vector: w1[5][64] b1[64] w2[64][64] b2[64] w3[64][2] b3[2] */
#define ROVER_GATE_PARAMS (5 * 64 + 64 + 64 * 64 + 64 + 64 * 2 + 2)

typedef struct RoverGateThresholds {
    float band_lo;       /* quantized / worst ratio at or below which a candidate is corrected */
    float band_hi;       /* ratio at or above which it keeps its quantized distance */
    float refine_logit;  /* inside the band: corrected when the refine logit exceeds this */
    float stop_logit;    /* a query stops when its sources' mean stop logit exceeds this */
} RoverGateThresholds;

/* Loads a gate (params: ROVER_GATE_PARAMS floats; mu, sigma: 5 each). */
AEEResult calculator_rover_gate_load(remote_handle64 h, const float *params, const float *mu,
                                     const float *sigma, const RoverGateThresholds *thresholds);
AEEResult calculator_rover_gate_unload(remote_handle64 h);
/* MLP rows the loaded gate has evaluated inside searches (seed-shortlist
 * rows inside the refine band, plus one row per expansion source while the
 * stop head is on) since it was loaded: 0 means the thresholds kept the
 * network out of every search. */
AEEResult calculator_rover_gate_rows(remote_handle64 h, uint64_t *rows);
/* The loaded gate's logits [n][2] (refine-needed, stop-expanding) for raw
 * rows [n][5] = {quantized distance, pool rank / L, worst pool distance,
 * hop count / L, query norm} (host buffers), computed by the same device
 * code the gated search runs (log of the two distances, standardisation,
 * BF16 tensor-core tiles). */
AEEResult calculator_rover_gate_eval(remote_handle64 h, const float *rows, int64_t n, float *logits);

/* Seed selection of the verified exact seed pool, on host buffers: for each
 * row of rank[rows][n_seeds] (non-negative floats) the m smallest keys
 * (rank bits << 32 | seed index) ascending into keys[rows][m] (all ones past
 * the row's end) and the (m + 1)-th smallest rank into next[rows] (+inf when
 * n_seeds <= m; NaN, with every key all ones, when the row holds a rank of
 * 3e38 or more or more than 2,048 ranks tie with the (m + 1)-th, which the
 * search answers by scanning the row).  Runs the device code the searches
 * run. */
AEEResult calculator_rover_seed_topm(remote_handle64 h, const float *rank, int32_t rows, int32_t n_seeds, int32_t m,
                                     uint64_t *keys, float *next);

/* The seed ranking of the verified seed pool on host buffers:
 * out[nq][n_rows] = max(|q|^2 + |x|^2 - 2 q . x, 0) with the dot products on
 * the tensor cores from TF32-rounded operands -- tcgen05 (TMA-fed, TMEM
 * accumulators) for dim 32..128 in steps of 32, mma.sync otherwise or with
 * ROVER_SEED_RANK=mma in the environment.  Runs the device code the searches
 * run (pq_seed_rank, pq_seed_pool.cuh bounds its error). */
AEEResult calculator_rover_seed_rank(remote_handle64 h, const float *queries, int32_t num_queries,
                                     const float *rows, int32_t num_rows, int32_t dim, float *out);

/* One training row per scored candidate or expansion source. */
typedef struct RoverGateTraceRow {
    int32_t query, hop, id;
    int32_t flags;       /* bit0: entered the pool, bit1: expansion source, bit2: entry seed */
    float quantized;     /* ADC distance (sources: pool distance) */
    float rank;          /* pool rank / L */
    float worst;         /* worst pool distance */
    float qnorm;         /* query L2 norm */
    float dist;          /* corrected distance */
    float pad[3];
} RoverGateTraceRow;

/* Plain search with full correction in the reference's expansion order
 * (ROVER_MODE_BATCHED with beam width 1), recording trace rows.  Rows beyond
 * capacity are counted in *count but not written. */
AEEResult calculator_rover_pq_trace(remote_handle64 h, const RoverSearchParams *params, const float *queries,
                                    int32_t num_queries, const int32_t *pool_sizes,
                                    const RoverSearchOutputs *out, RoverGateTraceRow *rows,
                                    int64_t capacity, int64_t *count);

/* Training on the device (forward / backward / Adam kernels of this
 * library).  Inputs x[n][5] are the raw gate inputs (log quantized distance,
 * rank / L, log worst distance, hop / L, query norm); y[n][2] labels in
 * {0, 1} (refine-needed, stop-expanding); m[n][2] masks (0 = no label for that
 * head).  Standardisation statistics come from x.  Outputs: the FP32 master
 * parameters (ROVER_GATE_PARAMS floats), mu / sigma (5 each), and the mean
 * training loss of each epoch. */
typedef struct RoverGateTrainParams {
    int32_t size;            /* sizeof(RoverGateTrainParams) */
    int32_t epochs;
    int32_t batch;           /* rows per optimiser step */
    float lr;                /* Adam step size */
    float beta1, beta2, eps;
    float weight_decay;      /* decoupled */
    uint32_t seed;           /* initialisation and shuffling */
    float pos_weight[2];     /* positive-class weight per head */
    int32_t reserved[4];
} RoverGateTrainParams;

AEEResult calculator_rover_gate_train(remote_handle64 h, const float *x, const float *y, const float *m, int64_t n,
                                      const RoverGateTrainParams *tp, float *params_out, float *mu_out,
                                      float *sigma_out, float *epoch_loss);

/* One forward / backward pass over all n rows with the given parameters,
 * as one training step computes it: the mean loss and the gradient of every
 * parameter (ROVER_GATE_PARAMS floats), both divided by n. */
AEEResult calculator_rover_gate_grad(remote_handle64 h, const float *x, const float *y, const float *m, int64_t n,
                                     const float *params, const float *mu, const float *sigma,
                                     const float *pos_weight, float *grad_out, float *loss_out);

/* Last CUDA / library error as text (thread-local). */
const char *calculator_rover_last_error(void);

/* Number of CUDA kernels this library has launched in this process. */
uint64_t calculator_rover_launch_count(void);

/* Per-kernel device time.  While enabled, each search-path kernel launch is
 * bracketed by CUDA events on the stream it runs on; the events are read when
 * the call that launched it synchronizes.  calculator_rover_kernel_times
 * fills, per kind, the launches and summed milliseconds since the last
 * calculator_rover_kernel_timing call (which resets them) and returns the
 * number of kinds written. */
#define ROVER_KERNEL_PQ_PACKED 0    /* PQ search, packed residual rows */
#define ROVER_KERNEL_PQ_SEEDS 1     /* all-queries x entry-seeds distances */
#define ROVER_KERNEL_PQ_DECODED 2   /* PQ search, decoded rows */
#define ROVER_KERNEL_PQ_BATCHED 3   /* PQ search, batched / gated modes */
#define ROVER_KERNEL_SQ 4           /* SQ search */
#define ROVER_KERNEL_PQ_SEED_RANK 5 /* all-queries x entry-seeds quantized distances, tensor cores */
#define ROVER_KERNEL_PQ_LUT 6       /* calculator_rover_score kind 0: per-query LUTs */
#define ROVER_KERNEL_PQ_ADC 7       /* kind 0: ADC sums of the id lists */
#define ROVER_KERNEL_PQ_RESIDUAL 8  /* kind 1: corrected distances from packed residual rows */
#define ROVER_KERNEL_SQ_COARSE 9    /* kind 2: SQ code distances */
#define ROVER_KERNEL_SQ_EXACT 10    /* kind 3: SQ residual-corrected distances */
#define ROVER_KERNEL_REFINE 11      /* calculator_rover_refine */
#define ROVER_KERNEL_PQ_RESCORE 12  /* kind 4: corrected distances from decoded rows */
#define ROVER_KERNEL_PLAN 13        /* search plans: bookkeeping kernels */
#define ROVER_KERNEL_PQ_SEED_TOPM 14 /* per-query top-M of the seed ranks */
#define ROVER_KERNEL_PQ_TRAIN 15    /* calculator_rover_pq_train / _pq_encode */
#define ROVER_KERNEL_KINDS 16
void calculator_rover_kernel_timing(int32_t enable);
int32_t calculator_rover_kernel_times(int64_t *launches, double *ms, int32_t kinds);

#ifdef __cplusplus
}
#endif

#endif /* ROVER_B200_H */
