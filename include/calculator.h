/*
 * calculator.h -- the Rover accelerator C-ABI, served on NVIDIA B200 (sm_100a).
 *
 * These are the entry points the reference host binds through its FastRPC
 * stub.  The interface is declared in the reference's inc/calculator.idl and
 * qaic lowers it to C as follows: the first argument is the session handle;
 * every `in sequence<T>` becomes (const T *p, int pLen); every
 * `rout sequence<T>` becomes (T *p, int pLen); `rout int32` becomes int32 *;
 * `sequence<long>` is a sequence of 32-bit int.  The implementations in the
 * reference are the DSP skeleton functions cited per entry below
 * (src/app/dsp.c and src/dsp_demo/retrieval_async_dsp_*.c).
 *
 * In this library the "DSP" is a CUDA device: index buffers live in HBM and
 * every distance, beam search, correction and re-rank runs as a hand-written
 * sm_100a kernel.  The "fd" arguments of the *_dma entry points name buffers
 * registered with the rpcmem/fastrpc compatibility layer exported by the same
 * library (include/rpcmem.h, include/remote.h); the zero-copy contract is kept
 * by uploading a registered buffer once at load time.
 *
 * Return codes: AEE_SUCCESS (0) on success, otherwise one of the AEE_* values
 * below.  The reference pins only AEE_SUCCESS == 0 (its AEEStdErr.h comes from
 * the Hexagon SDK); the nonzero values are this library's own.
 */
#ifndef ROVER_CALCULATOR_H
#define ROVER_CALCULATOR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef ROVER_AEE_TYPES_DEFINED
#define ROVER_AEE_TYPES_DEFINED
typedef int32_t int32;
typedef uint8_t uint8;
typedef uint64_t uint64;
typedef uint64_t remote_handle64;
typedef int AEEResult;
#endif

#ifndef AEE_SUCCESS
#define AEE_SUCCESS 0
#define AEE_EFAILED 1
#define AEE_ENOMEMORY 2
#define AEE_EBADPARM 14
#define AEE_EUNSUPPORTED 20
#endif

/* URI prefix the reference main.c passes to calculator_open (main.c:20). */
#define calculator_URI "file:///libcalculator_skel.so?calculator_skel_handle_invoke&_modver=1.0"

/* src/app/dsp.c:18 -- open a session; the handle is opaque. */
int calculator_open(const char *uri, remote_handle64 *handle);
/* src/app/dsp.c:24 -- close; the last close resets the async service. */
int calculator_close(remote_handle64 handle);

/* calculator.idl:15, src/app/dsp.c:8 -- ABI handshake: abi_version must be 1
 * (search branch) and l1_bits 4 or 8, else AEE_EBADPARM. */
AEEResult calculator_rover_configure(remote_handle64 h, int32 abi_version,
                                     int32 l1_bits);

/* calculator.idl:16-25, retrieval_async_dsp_async_service.c:214 -- queue one
 * SQ8 batch distance task (<= 240 codes) and return its task id. */
AEEResult calculator_retrieval_async_submit(
    remote_handle64 h, const float *query, int queryLen,
    const int *candidate_ids, int candidate_idsLen,
    const uint8 *compressed_batch, int compressed_batchLen, int32 dim,
    int32 num_candidates, float scale, float zero_point, int32 *task_id);
/* calculator.idl:26-32, retrieval_async_dsp_async_service.c:300 */
AEEResult calculator_retrieval_async_poll(
    remote_handle64 h, int32 task_id, int32 *status, int *result_ids,
    int result_idsLen, float *distances, int distancesLen,
    int32 *num_results);
/* calculator.idl:33, retrieval_async_dsp_async_service.c:354 */
AEEResult calculator_retrieval_async_reset(remote_handle64 h);

/* calculator.idl:36-45, retrieval_async_dsp_search.c:293 -- copy a dense
 * INT32 graph (num_vectors x graph_k) and SQ codes (4 or 8 bit, as set by
 * calculator_rover_configure) to the device. */
AEEResult calculator_retrieval_load(
    remote_handle64 h, const int *graph, int graphLen, const uint8 *l1_codes,
    int l1_codesLen, int32 num_vectors, int32 dim, int32 graph_k,
    int32 graph_entry_point, float l1_scale, float l1_zero_point);
/* calculator.idl:46-55, retrieval_async_dsp_search.c:368 -- one complete SQ
 * beam search on the device; ids/dists ascending, *actual_count filled. */
AEEResult calculator_retrieval_search(
    remote_handle64 h, const float *query, int queryLen, int32 entry_points,
    int32 expand_count, int32 pool_size, int32 num_out, int *candidate_ids,
    int candidate_idsLen, float *candidate_dists, int candidate_distsLen,
    int32 *actual_count);
/* calculator.idl:56, retrieval_async_dsp_search.c:511 */
AEEResult calculator_retrieval_unload(remote_handle64 h);

/* calculator.idl:59-69, retrieval_async_dsp_search.c:558 -- zero-copy
 * variant: fd_graph == -1 means the host keeps the graph. */
AEEResult calculator_retrieval_load_dma(
    remote_handle64 h, int32 fd_graph, const int32 *fd_l1_codes,
    int fd_l1_codesLen, int32 l1_chunk_vectors, int32 num_vectors, int32 dim,
    int32 graph_k, int32 graph_entry_point, float l1_scale,
    float l1_zero_point);
/* calculator.idl:70, retrieval_async_dsp_search.c:526 */
AEEResult calculator_retrieval_unload_dma(remote_handle64 h);

/* calculator.idl:73-77, retrieval_rnn_l2_dsp.c:21 (graph construction) */
AEEResult calculator_retrieval_rnn_l2_load_dma(remote_handle64 h,
                                               int32 fd_base,
                                               int32 num_vectors, int32 dim);
/* calculator.idl:78-83, retrieval_rnn_l2_dsp.c:54 */
AEEResult calculator_retrieval_rnn_l2_batch(remote_handle64 h,
                                            const int *ids_a, int ids_aLen,
                                            const int *ids_b, int ids_bLen,
                                            int32 pair_count, float *distances,
                                            int distancesLen);
/* calculator.idl:84, retrieval_rnn_l2_dsp.c:6 */
AEEResult calculator_retrieval_rnn_l2_unload_dma(remote_handle64 h);

/* calculator.idl:87-101, retrieval_async_dsp_search.c:1399 -- two SQ
 * queries searched together; the host corrects coarse distances through the
 * ExpansionBuffer pair behind fd_expansion_buf. */
AEEResult calculator_retrieval_search_db(
    remote_handle64 h, const float *query_a, int query_aLen,
    const float *query_b, int query_bLen, int32 fd_expansion_buf,
    int32 entry_points, int32 expand_count, int32 pool_size, int32 num_out,
    int *candidate_ids_a, int candidate_ids_aLen, float *candidate_dists_a,
    int candidate_dists_aLen, int32 *actual_count_a, int *candidate_ids_b,
    int candidate_ids_bLen, float *candidate_dists_b,
    int candidate_dists_bLen, int32 *actual_count_b);

/* calculator.idl:104-110, retrieval_async_dsp_search.c:1584 -- serve one
 * query's SQMD lane buffers (blocking until the host finishes the query). */
AEEResult calculator_retrieval_expand_sqmd(remote_handle64 h,
                                           const float *query, int queryLen,
                                           int32 query_dim, int32 fd_sqmd_ctrl,
                                           int32 lane_count,
                                           int32 work_items_cap);
/* calculator.idl:113-117, retrieval_async_dsp_search.c:1791 -- blocking
 * SQMD session: serve lane buffers until SHUTDOWN/ABORT. */
AEEResult calculator_retrieval_expand_sqmd_run(remote_handle64 h,
                                               int32 fd_sqmd_ctrl,
                                               int32 lane_count,
                                               int32 work_items_cap);

/* calculator.idl:119-131, retrieval_async_dsp_search.c:698 -- register the
 * pure-PQ code chunks (all but the last full), codebook and index UUID. */
AEEResult calculator_retrieval_pure_pq_load_dma(
    remote_handle64 h, const int32 *fd_pq_codes, int fd_pq_codesLen,
    const int32 *pq_chunk_vector_counts, int pq_chunk_vector_countsLen,
    int32 pq_chunk_vectors, const float *pq_codebook, int pq_codebookLen,
    int32 num_vectors, int32 dim, int32 pq_m, int32 pq_ks, int32 pq_subdim,
    int32 pq_code_bytes, const uint8 *index_uuid, int index_uuidLen);
/* calculator.idl:132, retrieval_async_dsp_search.c:668 */
AEEResult calculator_retrieval_pure_pq_unload_dma(remote_handle64 h);
/* calculator.idl:133-138, retrieval_async_dsp_search.c:2269 -- blocking
 * pure-PQ session: ADC for every CPU_READY lane buffer. */
AEEResult calculator_retrieval_pure_pq_sqmd_run(remote_handle64 h,
                                                int32 fd_sqmd_ctrl,
                                                int32 fd_query_lut,
                                                int32 lane_count,
                                                int32 work_items_cap);

#ifdef __cplusplus
}
#endif

#endif /* ROVER_CALCULATOR_H */
