// seed_rank_tc.cu -- the seed ranking on Blackwell's fifth-generation tensor
// cores: out[q][u] = max(|q|^2 + |x_u|^2 - 2 q . x_u, 0) for every query q of
// a chunk and every entry seed u, with the dot products as tcgen05.mma
// kind::tf32 (M = 128 queries x N = 128 seeds x K = 8 per instruction, FP32
// accumulators in tensor memory).
//
// One CTA owns 128 queries and a run of 128-seed tiles:
//   * warps 0-3 stage the 128 query rows, rounded to TF32, into shared
//     memory in the 128-byte-swizzled K-major layout the MMA descriptors
//     name, and sum |q|^2;
//   * warps 0-7 are the epilogue: warp w reads accumulator lanes
//     32 (w mod 4) .. +31 (its query rows) and columns 64 (w / 4) .. +63 of
//     each tile with tcgen05.ld, applies the rank formula (the tile's seed
//     norms read once per 32 columns and broadcast by shuffles) and stores
//     the row segments;
//   * warp 8 streams the seed tiles with TMA (cp.async.bulk.tensor, one
//     32-float x 128-row box per 128-byte swizzle column) into two stages;
//   * warp 9 allocates 256 tensor-memory columns (two accumulators) and one
//     of its threads issues the MMAs; tcgen05.commit hands each finished
//     accumulator to the epilogue and each consumed stage back to TMA.
// The seed rows come pre-rounded to TF32 (round to nearest, as cvt.rna),
// so the tensor cores see the operands the error bound of the verified seed
// pool assumes (pq_seed_pool.cuh: relative 2^-11 per operand).
//
// Every wait on an mbarrier is bounded; a wait that runs out sets *err,
// every role stops issuing work, the TMA thread waits (bounded) for the
// copies it started, and the CTA frees its tensor memory and returns.  The
// caller checks *err after the search and fails the call.

#include <algorithm>
#include <cstring>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "common.cuh"
#include "kernels.h"

namespace rover {
namespace {

constexpr int kTcM = 128;                 // queries per CTA (MMA M, TMEM lanes)
constexpr int kTcN = 128;                 // seeds per tile (MMA N)
constexpr int kTcEpiWarps = 8;            // two per accumulator lane quarter
constexpr int kTmaWarp = kTcEpiWarps, kMmaWarp = kTcEpiWarps + 1;
constexpr int kTcThreads = 32 * (kTcEpiWarps + 2);
constexpr int kAtomBytes = 128 * 128;     // one 32-float column block of 128 rows
constexpr uint32_t kWaitLimit = 1u << 22; // mbarrier polls before giving up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// True once the phase of the given parity has completed; false after
// kWaitLimit polls.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (uint32_t i = 0; i < kWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
      ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
      : "memory");
}

__device__ __forceinline__ uint32_t tf32_bits(float f) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(f));
  return r;
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1,024 bytes apart (start, leading and stride offsets in 16-byte units;
// version 1; layout type 2 = SWIZZLE_128B).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((addr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>(1u) << 16;            // leading byte offset: 16 B (unused for swizzled K-major)
  d |= static_cast<uint64_t>(1024u >> 4) << 32;    // stride byte offset: 1,024 B between 8-row groups
  d |= static_cast<uint64_t>(1u) << 46;            // descriptor version
  d |= static_cast<uint64_t>(2u) << 61;            // SWIZZLE_128B
  return d;
}

// Instruction descriptor of kind::tf32: FP32 accumulator, TF32 A and B,
// both K-major, N = 128, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((kTcN >> 3) << 17) | ((kTcM >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      ::"r"(tmem_d), "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive accumulator columns of this warp's 32 lanes.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}


__global__ void __launch_bounds__(kTcThreads, 1)
pq_seed_rank_tc_kernel(const __grid_constant__ CUtensorMap rows_map, const float* __restrict__ queries, int q_begin,
                       int q_end, int dim, const float* __restrict__ norms, int n_seeds, int tiles_per_cta,
                       float* __restrict__ out, int out_stride, int* err) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;        // swizzle atoms start on 1,024-byte boundaries
  uint8_t* gbase = smem_raw + (base - raw);
  const int dk = dim / 32;                              // 128-byte K columns per row
  const uint32_t a_s = base;                            // queries: dk columns of 128 rows
  const uint32_t b_s = a_s + dk * kAtomBytes;           // seeds: 2 stages x dk columns
  const uint32_t bars = b_s + 2 * dk * kAtomBytes;
  uint8_t* gbars = gbase + (bars - base);
  const uint32_t full0 = bars, empty0 = bars + 16, accf0 = bars + 32, acce0 = bars + 48;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(gbars + 64);
  volatile int* stop = reinterpret_cast<volatile int*>(gbars + 68);
  float* qn = reinterpret_cast<float*>(gbars + 128);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q0 = q_begin + static_cast<int>(blockIdx.y) * kTcM;
  const int nt = (n_seeds + kTcN - 1) / kTcN;
  const int t0 = static_cast<int>(blockIdx.x) * tiles_per_cta;
  const int ntiles = max(0, min(nt, t0 + tiles_per_cta) - t0);
  auto fail = [&]() {
    *stop = 1;
    atomicExch(err, 1);
  };

  if (threadIdx.x == 0) {
    for (int s = 0; s < 2; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
      mbar_init(accf0 + 8 * s, 1);
      mbar_init(acce0 + 8 * s, kTcEpiWarps);   // one arrival per epilogue warp
    }
    *stop = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(256u)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (warp < 4) {
    // one query row per thread: TF32-rounded into the swizzled layout
    // (16-byte chunk c of row r at chunk c ^ (r mod 8)), and |q|^2
    const int r = threadIdx.x;
    const int qq = q0 + r;
    const float4* src = reinterpret_cast<const float4*>(queries + static_cast<size_t>(qq) * dim);
    float sq = 0.0f;
    for (int c4 = 0; c4 < dim / 4; ++c4) {
      const float4 v = qq < q_end ? __ldg(src + c4) : make_float4(0.f, 0.f, 0.f, 0.f);
      sq += ((v.x * v.x + v.y * v.y) + v.z * v.z) + v.w * v.w;
      const int k = 4 * c4, col = k >> 5, chunk = (k & 31) >> 2;
      const uint32_t addr = a_s + col * kAtomBytes + r * 128 + ((chunk ^ (r & 7)) << 4);
      asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(tf32_bits(v.x)), "r"(tf32_bits(v.y)),
                   "r"(tf32_bits(v.z)), "r"(tf32_bits(v.w))
                   : "memory");
    }
    qn[r] = sq;
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // the MMAs read what the threads wrote
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == kTmaWarp) {
    if (lane == 0) {
      // TMA producer: seed tile t0 + i into stage i % 2
      int issued = 0;
      for (int i = 0; i < ntiles && !*stop; ++i) {
        const int s = i & 1;
        const uint32_t ph = (i >> 1) & 1;
        if (!mbar_wait(empty0 + 8 * s, ph ^ 1u)) { fail(); break; }
        mbar_expect_tx(full0 + 8 * s, static_cast<uint32_t>(dk * kAtomBytes));
        for (int col = 0; col < dk; ++col)
          tma_load_2d(b_s + (s * dk + col) * kAtomBytes, &rows_map, full0 + 8 * s, 32 * col, (t0 + i) * kTcN);
        ++issued;
      }
      // every copy this thread started lands before the CTA may leave
      for (int i = max(0, issued - 2); i < issued; ++i)
        if (!mbar_wait(full0 + 8 * (i & 1), (i >> 1) & 1)) atomicExch(err, 1);
    }
  } else if (warp == kMmaWarp) {
    if (lane == 0) {
      // MMA issuer: tile i into accumulator i % 2 (TMEM columns 128 (i % 2) ..)
      int committed = 0;
      for (int i = 0; i < ntiles && !*stop; ++i) {
        const int s = i & 1;
        const uint32_t ph = (i >> 1) & 1;
        if (!mbar_wait(acce0 + 8 * s, ph ^ 1u)) { fail(); break; }
        if (!mbar_wait(full0 + 8 * s, ph)) { fail(); break; }
        tc_fence_after();
        const uint32_t d = tmem + static_cast<uint32_t>(s * kTcN);
        for (int ks = 0; ks < dim / 8; ++ks) {
          const uint32_t off = static_cast<uint32_t>((ks >> 2) * kAtomBytes + (ks & 3) * 32);
          mma_tf32(d, sw128_desc(a_s + off), sw128_desc(b_s + s * dk * kAtomBytes + off), ks > 0 ? 1u : 0u);
        }
        mma_commit(empty0 + 8 * s);       // stage s may be refilled once these MMAs are done
        mma_commit(accf0 + 8 * s);        // accumulator s is ready for the epilogue
        ++committed;
      }
      // the last commit covers every MMA issued: none is in flight at exit
      if (committed > 0 && !mbar_wait(accf0 + 8 * ((committed - 1) & 1), ((committed - 1) >> 1) & 1))
        atomicExch(err, 1);
    }
  } else {
    // epilogue: accumulator lanes 32 (warp mod 4) .. +31 = this warp's query
    // rows; columns 64 (warp / 4) .. +63 of each tile
    const int quarter = warp & 3, half = warp >> 2;
    const int r = quarter * 32 + lane;
    const int qq = q0 + r;
    const float qv = qn[r];
    float* orow = out + static_cast<size_t>(qq - q_begin) * out_stride;
    const bool vec = (out_stride & 3) == 0;
    for (int i = 0; i < ntiles; ++i) {
      const int ab = i & 1;
      if (!mbar_wait(accf0 + 8 * ab, (i >> 1) & 1)) { fail(); break; }
      tc_fence_after();
      const int u0 = (t0 + i) * kTcN;
#pragma unroll 1
      for (int c = 2 * half; c < 2 * half + 2; ++c) {
        float v[32];
        tmem_ld32(tmem + (static_cast<uint32_t>(quarter * 32) << 16) + static_cast<uint32_t>(ab * kTcN + c * 32), v);
        const int ub = u0 + c * 32;
        const float nl = ub + lane < n_seeds ? __ldg(norms + ub + lane) : 0.0f;   // this chunk's 32 seed norms
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = fmaxf(qv + __shfl_sync(kFullMask, nl, j) - 2.0f * v[j], 0.0f);
        if (qq < q_end) {
          if (vec && ub + 32 <= n_seeds) {
#pragma unroll
            for (int j = 0; j < 32; j += 4)
              *reinterpret_cast<float4*>(orow + ub + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
          } else {
#pragma unroll
            for (int j = 0; j < 32; ++j)
              if (ub + j < n_seeds) orow[ub + j] = v[j];
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acce0 + 8 * ab);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256u) : "memory");
  }
}

__global__ void tf32_round_kernel(const float* __restrict__ in, float* __restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    out[i] = __uint_as_float(tf32_bits(in[i]));
}

// |x|^2 of each row (FP32, in dimension order).
__global__ void row_norms_kernel(const float* __restrict__ rows, int n, int dim, float* __restrict__ norms) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  float s = 0.0f;
  for (int d = 0; d < dim; ++d) {
    const float v = rows[static_cast<size_t>(r) * dim + d];
    s += v * v;
  }
  norms[r] = s;
}

size_t tc_smem_bytes(int dim) { return static_cast<size_t>(3 * (dim / 32)) * kAtomBytes + 1024 + 640; }

}  // namespace

bool seed_rank_tc_supported(int dim) { return dim >= 32 && dim <= 128 && dim % 32 == 0; }

void launch_tf32_round(const float* in, float* out, size_t n, cudaStream_t s) {
  if (n) tf32_round_kernel<<<static_cast<unsigned>(std::min<size_t>((n + 255) / 256, 4096)), 256, 0, s>>>(in, out, n);
}

void launch_row_norms(const float* rows, int n, int dim, float* norms, cudaStream_t s) {
  if (n > 0) row_norms_kernel<<<(n + 127) / 128, 128, 0, s>>>(rows, n, dim, norms);
}

// A TMA descriptor of [n_seeds][dim] FP32 rows (TF32-rounded), boxes of 32
// floats x 128 rows with the 128-byte swizzle; rows past n_seeds read as 0.
bool tc_seed_map_encode(TcSeedMap* m, const float* rows, int n_seeds, int dim) {
  m->valid = 0;
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
      cudaGetLastError();
      return false;
    }
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  if (!seed_rank_tc_supported(dim) || n_seeds <= 0 || (reinterpret_cast<uintptr_t>(rows) & 15u)) return false;
  const cuuint64_t gdim[2] = {static_cast<cuuint64_t>(dim), static_cast<cuuint64_t>(n_seeds)};
  const cuuint64_t gstride[1] = {static_cast<cuuint64_t>(dim) * sizeof(float)};
  const cuuint32_t box[2] = {32u, static_cast<cuuint32_t>(kTcN)};
  const cuuint32_t estride[2] = {1u, 1u};
  const CUresult r = encode(reinterpret_cast<CUtensorMap*>(m->bytes), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                            const_cast<float*>(rows), gdim, gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
                            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  m->valid = r == CUDA_SUCCESS ? 1 : 0;
  return m->valid != 0;
}

bool launch_pq_seed_rank_tc(const TcSeedMap& m, const float* queries, int q_begin, int q_end, int dim,
                            const float* norms, int n_seeds, float* out, int out_stride, int* err, int sms,
                            cudaStream_t s) {
  if (!m.valid || !seed_rank_tc_supported(dim) || q_end <= q_begin || n_seeds <= 0) return false;
  const size_t smem = tc_smem_bytes(dim);
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(pq_seed_rank_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem > 200000 ? smem : 200000)) != cudaSuccess)
      return false;
    attr = true;
  }
  const int qt = (q_end - q_begin + kTcM - 1) / kTcM;
  const int nt = (n_seeds + kTcN - 1) / kTcN;
  static int per_sm = 0;
  if (!per_sm && (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pq_seed_rank_tc_kernel, kTcThreads, smem) !=
                      cudaSuccess ||
                  per_sm < 1))
    per_sm = 1;
  // Split the seed tiles of each 128-query tile across CTAs.  The time is
  // about (waves of resident CTAs) x (tiles per CTA + the prologue, worth
  // about two tiles: query staging, tensor-memory allocation, pipeline
  // fill); take the split that minimises it.
  const int slots = std::max(1, sms) * per_sm;
  int per = nt;
  long long best = -1;
  for (int sp = 1; sp <= nt; ++sp) {
    const int p = (nt + sp - 1) / sp;
    const int used = (nt + p - 1) / p;
    const long long waves = (static_cast<long long>(qt) * used + slots - 1) / slots;
    const long long cost = waves * (p + 2);
    if (best < 0 || cost < best) { best = cost; per = p; }
  }
  const int splits = (nt + per - 1) / per;
  CUtensorMap map;
  std::memcpy(&map, m.bytes, sizeof(map));
  // a failure left behind by an earlier call that tolerated it (an occupancy
  // or attribute probe) must not read as this launch's: the caller would
  // then rank the seeds a second time on mma.sync
  cudaGetLastError();
  pq_seed_rank_tc_kernel<<<dim3(splits, qt), kTcThreads, smem, s>>>(map, queries, q_begin, q_end, dim, norms,
                                                                   n_seeds, per, out, out_stride ? out_stride : n_seeds,
                                                                   err);
  return cudaGetLastError() == cudaSuccess;
}

}  // namespace rover
