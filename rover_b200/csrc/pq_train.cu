// pq_train.cu -- PQ codebook training and encoding on the GPU, bit for bit
// the reference's C trainer (retrieval_pq_train / retrieval_pq_train_subspace,
// retrieval_pq_core.c:97-224) and encoder (retrieval_pq_encode_batch,
// :226-268).
//
// The trainer is Lloyd's k-means per subspace: centroid k starts as training
// vector k (count-1) / (ks-1); each iteration assigns every vector to its
// nearest centroid (sequential FP32 squared distance, strict < so the first
// minimum wins) and replaces every non-empty centroid by its members' FP32
// sum -- accumulated in vector order -- times 1 / count.  All subspaces run
// at once, one CUDA launch sequence per iteration:
//   pq_assign_kernel   each thread one (vector, subspace): the argmin, and a
//                      per-block histogram of the assignments;
//   pq_bucket_kernel   per subspace: each centroid's total and, per block of
//                      vectors, where its members of that block start in the
//                      centroid's member list (an exclusive scan over blocks);
//   pq_scatter_kernel  each vector's slot in its centroid's list: the block
//                      start plus its rank among the earlier vectors of its
//                      block with the same centroid, so every list is in
//                      vector order (a stable counting sort);
//   pq_update_kernel   each thread one (subspace, centroid, dimension): the
//                      sequential sum over the member list, then the mean.
// Summing a centroid's members in list order reproduces the reference's
// running sums exactly, since its per-centroid additions also happen in
// vector order.  Sums and means are separately rounded _rn operations.

#include <cfloat>
#include <vector>

#include "common.cuh"
#include "kernels.h"

namespace rover {
namespace {

constexpr int kTrainBlock = 256;   // vectors per assignment block

__device__ __forceinline__ float sub_l2(const float* a, const float* b, int subdim) {
  float acc = 0.0f;
  for (int d = 0; d < subdim; ++d) {
    const float diff = fsub(a[d], b[d]);
    acc = fadd(acc, fmul(diff, diff));
  }
  return acc;
}

__global__ void pq_train_init_kernel(const float* __restrict__ x, int n, int dim, int m, int ks, int subdim,
                                     float* __restrict__ book) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;   // (subspace, centroid, dimension)
  if (t >= m * ks * subdim) return;
  const int s = t / (ks * subdim), r = t - s * ks * subdim, k = r / subdim, d = r - k * subdim;
  const long long src = n == 1 ? 0 : (static_cast<long long>(k) * (n - 1)) / (ks > 1 ? ks - 1 : 1);
  book[t] = x[static_cast<size_t>(src) * dim + static_cast<size_t>(s) * subdim + d];
}

// grid (blocks of kTrainBlock vectors, m); the subspace's centroids are
// staged in shared memory when they fit.
__global__ void __launch_bounds__(kTrainBlock) pq_assign_kernel(const float* __restrict__ x, int n, int dim, int ks,
                                                                int subdim, const float* __restrict__ book,
                                                                int stage, uint8_t* __restrict__ assign,
                                                                int* __restrict__ block_hist) {
  extern __shared__ __align__(16) float cen[];
  __shared__ int hist[256];
  const int s = blockIdx.y, b = blockIdx.x;
  const float* c = book + static_cast<size_t>(s) * ks * subdim;
  for (int k = threadIdx.x; k < 256; k += blockDim.x) hist[k] = 0;
  if (stage)
    for (int i = threadIdx.x; i < ks * subdim; i += blockDim.x) cen[i] = c[i];
  __syncthreads();
  const float* cs = stage ? cen : c;
  const int i = b * kTrainBlock + threadIdx.x;
  if (i < n) {
    const float* xv = x + static_cast<size_t>(i) * dim + static_cast<size_t>(s) * subdim;
    float best = FLT_MAX;
    int best_k = 0;
    for (int k = 0; k < ks; ++k) {
      const float dist = sub_l2(xv, cs + static_cast<size_t>(k) * subdim, subdim);
      if (dist < best) { best = dist; best_k = k; }
    }
    assign[static_cast<size_t>(s) * n + i] = static_cast<uint8_t>(best_k);
    atomicAdd(&hist[best_k], 1);
  }
  __syncthreads();
  const int nb = gridDim.x;
  for (int k = threadIdx.x; k < ks; k += blockDim.x)
    block_hist[(static_cast<size_t>(s) * nb + b) * ks + k] = hist[k];
}

// one block per subspace, one thread per centroid: totals, member-list
// offsets, and each block's start inside the lists (block_hist is rewritten
// in place with the starts).
__global__ void pq_bucket_kernel(int ks, int nb, int* __restrict__ block_hist, int* __restrict__ counts) {
  __shared__ int total[256];
  const int s = blockIdx.x, k = threadIdx.x;
  int run = 0;
  if (k < ks) {
    for (int b = 0; b < nb; ++b) {
      int* h = block_hist + (static_cast<size_t>(s) * nb + b) * ks + k;
      const int c = *h;
      *h = run;
      run += c;
    }
    total[k] = run;
    counts[s * ks + k] = run;
  }
  __syncthreads();
  if (k < ks) {
    int off = 0;
    for (int j = 0; j < k; ++j) off += total[j];
    for (int b = 0; b < nb; ++b) block_hist[(static_cast<size_t>(s) * nb + b) * ks + k] += off;
  }
}

__global__ void __launch_bounds__(kTrainBlock) pq_scatter_kernel(int n, const uint8_t* __restrict__ assign, int ks,
                                                                 const int* __restrict__ block_start,
                                                                 int* __restrict__ members) {
  __shared__ uint8_t a[kTrainBlock];
  const int s = blockIdx.y, b = blockIdx.x, nb = gridDim.x;
  const int i = b * kTrainBlock + threadIdx.x;
  a[threadIdx.x] = i < n ? assign[static_cast<size_t>(s) * n + i] : 0;
  __syncthreads();
  if (i >= n) return;
  const uint8_t me = a[threadIdx.x];
  int rank = 0;
  for (int j = 0; j < static_cast<int>(threadIdx.x); ++j) rank += a[j] == me;
  members[static_cast<size_t>(s) * n + block_start[(static_cast<size_t>(s) * nb + b) * ks + me] + rank] = i;
}

__global__ void pq_update_kernel(const float* __restrict__ x, int n, int dim, int m, int ks, int subdim,
                                 const int* __restrict__ members, const int* __restrict__ counts,
                                 float* __restrict__ book) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;   // (subspace, centroid, dimension)
  if (t >= m * ks * subdim) return;
  const int s = t / (ks * subdim), r = t - s * ks * subdim, k = r / subdim, d = r - k * subdim;
  const int c = counts[s * ks + k];
  if (c <= 0) return;   // empty centroids keep their place
  int off = 0;
  for (int j = 0; j < k; ++j) off += counts[s * ks + j];
  const int* mem = members + static_cast<size_t>(s) * n + off;
  const float* col = x + static_cast<size_t>(s) * subdim + d;
  float sum = 0.0f;
  for (int j = 0; j < c; ++j) sum = fadd(sum, __ldg(col + static_cast<size_t>(__ldg(mem + j)) * dim));
  const float inv = __fdiv_rn(1.0f, __int2float_rn(c));
  book[t] = fmul(sum, inv);
}

// retrieval_pq_encode_batch: one thread per (vector, code byte); a
// non-finite distance marks *bad.
__global__ void pq_encode_kernel(const float* __restrict__ x, long long n, int dim, int m, int ks, int subdim,
                                 int code_bytes, const float* __restrict__ book, uint8_t* __restrict__ codes,
                                 int* bad) {
  const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= n * code_bytes) return;
  const long long i = t / code_bytes;
  const int byte = static_cast<int>(t - i * code_bytes);
  const int per = ks <= 16 ? 2 : 1;
  uint8_t out = 0;
  for (int h = 0; h < per; ++h) {
    const int s = byte * per + h;
    if (s >= m) break;
    const float* xv = x + static_cast<size_t>(i) * dim + static_cast<size_t>(s) * subdim;
    const float* c = book + static_cast<size_t>(s) * ks * subdim;
    float best = FLT_MAX;
    int best_k = 0;
    for (int k = 0; k < ks; ++k) {
      const float dist = sub_l2(xv, c + static_cast<size_t>(k) * subdim, subdim);
      if (!isfinite(dist)) { *bad = 1; return; }
      if (dist < best) { best = dist; best_k = k; }
    }
    out |= static_cast<uint8_t>(best_k << (4 * h));
  }
  codes[t] = out;
}

}  // namespace

PqTrainScratch::~PqTrainScratch() { release(); }

void PqTrainScratch::release() {
  for (void* p : {static_cast<void*>(assign), static_cast<void*>(block_hist), static_cast<void*>(counts),
                  static_cast<void*>(members)})
    if (p) cudaFree(p);
  assign = nullptr;
  block_hist = counts = members = nullptr;
}

cudaError_t pq_train_device(const float* x, int n, int dim, int m, int ks, int iters, float* book,
                            PqTrainScratch* sc, cudaStream_t s) {
  const int subdim = dim / m;
  const int nb = (n + kTrainBlock - 1) / kTrainBlock;
  sc->release();
  cudaError_t e;
  if ((e = cudaMalloc(&sc->assign, static_cast<size_t>(m) * n)) != cudaSuccess ||
      (e = cudaMalloc(&sc->block_hist, static_cast<size_t>(m) * nb * ks * sizeof(int))) != cudaSuccess ||
      (e = cudaMalloc(&sc->counts, static_cast<size_t>(m) * ks * sizeof(int))) != cudaSuccess ||
      (e = cudaMalloc(&sc->members, static_cast<size_t>(m) * n * sizeof(int))) != cudaSuccess)
    return e;
  const int cells = m * ks * subdim;
  pq_train_init_kernel<<<(cells + 255) / 256, 256, 0, s>>>(x, n, dim, m, ks, subdim, book);
  const size_t cen_bytes = static_cast<size_t>(ks) * subdim * sizeof(float);
  const int stage = cen_bytes <= 96 * 1024;
  if (stage && cen_bytes > 48 * 1024)
    cudaFuncSetAttribute(pq_assign_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(cen_bytes));
  for (int it = 0; it < (iters > 0 ? iters : 1); ++it) {
    pq_assign_kernel<<<dim3(nb, m), kTrainBlock, stage ? cen_bytes : 0, s>>>(x, n, dim, ks, subdim, book, stage,
                                                                            sc->assign, sc->block_hist);
    pq_bucket_kernel<<<m, 256, 0, s>>>(ks, nb, sc->block_hist, sc->counts);
    pq_scatter_kernel<<<dim3(nb, m), kTrainBlock, 0, s>>>(n, sc->assign, ks, sc->block_hist, sc->members);
    pq_update_kernel<<<(cells + 127) / 128, 128, 0, s>>>(x, n, dim, m, ks, subdim, sc->members, sc->counts, book);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

int pq_train_launches(int iters) { return 1 + 4 * (iters > 0 ? iters : 1); }

void launch_pq_encode(const float* x, long long n, int dim, int m, int ks, const float* book, uint8_t* codes,
                      int* bad, cudaStream_t s) {
  if (n <= 0) return;
  const int subdim = dim / m;
  const int code_bytes = ks <= 16 ? m / 2 + m % 2 : m;
  const long long cells = n * code_bytes;
  pq_encode_kernel<<<static_cast<unsigned>((cells + 255) / 256), 256, 0, s>>>(x, n, dim, m, ks, subdim, code_bytes,
                                                                               book, codes, bad);
}

}  // namespace rover
