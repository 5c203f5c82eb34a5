// sq_search.cu -- SQ beam search with the reference's exact heap semantics.
//
// Two reference loops are served:
//  * kSqModeDsp: calculator_retrieval_search, the legacy full device search
//    (src/dsp_demo/retrieval_async_dsp_search.c:368-509): LCG entries
//    (dsp_search_select_entry_id :219), neighbours outside [0, n) skipped one
//    by one, coarse SQ distances only.
//  * kSqModeSqmd: the CLI's SQMD loop (retrieval_sqmd_common.c
//    sqmd_cpu_state_run_fake_dsp :2052 with dispatch :283 and apply :638),
//    seeds from retrieval_sqmd_make_seed_ids (retrieval_sqmd_seed.c:15), and
//    the exact residual distance (retrieval_rpc_demo_support.c:1397) replacing
//    the coarse one when correction is on.
//  * kSqModeDb: one query of calculator_retrieval_search_db, the DB-pair
//    search (retrieval_async_dsp_search.c:1205-1581): the device search of
//    kSqModeDsp (entries, pool clamp, neighbour filtering), except that every
//    expansion candidate enters the pool with the distance the host's
//    correction thread returns for it (retrieval_rpc_demo_pipeline.c:454-495:
//    the exact residual distance with correction on, the coarse one with it
//    off) and that the frontier grows as needed (db_search_reserve_frontier).
//
// SQ pool and frontier heaps order by distance only and break ties by heap
// position (strict '<' replacement, sqmd_common.c:51-80), so results depend
// on the insertion order.  The kernel therefore keeps the reference's heaps
// verbatim: one warp per query computes distances in parallel, lane 0 applies
// the heap operations in the reference's order.

#include "common.cuh"
#include "kernels.h"
#include "sq_split.cuh"

namespace rover {

struct HeapEntry { int32_t id; float dist; };

__device__ __forceinline__ void pool_sift_up(HeapEntry* p, int i) {
  HeapEntry t = p[i];
  while (i > 0) {
    const int parent = (i - 1) / 2;
    if (t.dist <= p[parent].dist) break;
    p[i] = p[parent];
    i = parent;
  }
  p[i] = t;
}

__device__ __forceinline__ void pool_sift_down(HeapEntry* p, int size, int i) {
  HeapEntry t = p[i];
  for (;;) {
    int child = 2 * i + 1;
    if (child >= size) break;
    if (child + 1 < size && p[child + 1].dist > p[child].dist) ++child;
    if (t.dist >= p[child].dist) break;
    p[i] = p[child];
    i = child;
  }
  p[i] = t;
}

__device__ __forceinline__ bool pool_insert(HeapEntry* p, int* size, int cap, int32_t id, float d) {
  if (*size < cap) {
    p[*size].id = id;
    p[*size].dist = d;
    pool_sift_up(p, *size);
    ++*size;
    return true;
  }
  if (d < p[0].dist) {
    p[0].id = id;
    p[0].dist = d;
    pool_sift_down(p, *size, 0);
    return true;
  }
  return false;
}

__device__ __forceinline__ void front_sift_up(HeapEntry* f, int i) {
  HeapEntry t = f[i];
  while (i > 0) {
    const int parent = (i - 1) / 2;
    if (t.dist >= f[parent].dist) break;
    f[i] = f[parent];
    i = parent;
  }
  f[i] = t;
}

__device__ __forceinline__ void front_sift_down(HeapEntry* f, int size, int i) {
  HeapEntry t = f[i];
  for (;;) {
    int child = 2 * i + 1;
    if (child >= size) break;
    if (child + 1 < size && f[child + 1].dist < f[child].dist) ++child;
    if (t.dist <= f[child].dist) break;
    f[i] = f[child];
    i = child;
  }
  f[i] = t;
}

__device__ __forceinline__ int32_t front_pop(HeapEntry* f, int* size) {
  const int32_t top = f[0].id;
  --*size;
  if (*size > 0) {
    f[0] = f[*size];
    front_sift_down(f, *size, 0);
  }
  return top;
}

// retrieval_compute_int8_native_distance_u8_scalar / int4_packed (l1_int8_core.c:119-169):
// exact integer sum of squared code differences, then (float)acc * scale^2.
__device__ __forceinline__ float sq_coarse(const SqIndexView& ix, const uint8_t* qc, int32_t id) {
  const uint8_t* x = ix.l1 + static_cast<size_t>(id) * ix.l1_code_bytes;
  long long acc = 0;
  if (ix.l1_bits == 8) {
    int d = 0;
    if ((ix.dim & 3) == 0) {
      const uint32_t* xw = reinterpret_cast<const uint32_t*>(x);
      const uint32_t* qw = reinterpret_cast<const uint32_t*>(qc);
      int iacc = 0;
      for (; d < ix.dim; d += 4) {
        const uint32_t a = qw[d >> 2];
        const uint32_t b = __ldg(xw + (d >> 2));
        // sum (a_i - b_i)^2 = sum a^2 - 2 sum ab + sum b^2, exact in int32 per word
        iacc += __dp4a(a, a, 0u) - 2 * static_cast<int>(__dp4a(a, b, 0u)) + __dp4a(b, b, 0u);
        if ((d & 1023) == 1020) { acc += iacc; iacc = 0; }
      }
      acc += iacc;
    } else {
      for (; d < ix.dim; ++d) {
        const int df = static_cast<int>(qc[d]) - static_cast<int>(__ldg(x + d));
        acc += df * df;
      }
    }
  } else {
    for (int d = 0; d < ix.dim; ++d) {
      const int df = static_cast<int>(qc[d] & 15) - nibble(x, d);
      acc += df * df;
    }
  }
  const float scale_sq = fmul(ix.l1_scale, ix.l1_scale);
  return fmul(__ll2float_rn(acc), scale_sq);
}

// retrieval_demo_exact_distance_residual_scalar (support.c:1397-1443)
__device__ __forceinline__ float sq_exact(const SqIndexView& ix, const float* q, int32_t id) {
  const uint8_t* l1 = ix.l1 + static_cast<size_t>(id) * ix.l1_code_bytes;
  const uint8_t* res = ix.residual ? ix.residual + static_cast<size_t>(id) * ix.rcb : nullptr;
  float rs = 0.0f, rz = 0.0f, dist = 0.0f;
  if (res) {
    const float2 qp = __ldg(reinterpret_cast<const float2*>(ix.qparams) + id);
    rs = qp.x;
    rz = qp.y;
  }
  for (int i = 0; i < ix.dim; ++i) {
    const uint32_t c = ix.l1_bits == 4 ? static_cast<uint32_t>(nibble(l1, i)) : __ldg(l1 + i);
    float value = fadd(fmul(u8f(c), ix.l1_scale), ix.l1_zero);
    if (res) {
      const uint32_t r = ix.residual_bits == 4 ? static_cast<uint32_t>(nibble(res, i)) : __ldg(res + i);
      value = fadd(value, fadd(fmul(u8f(r), rs), rz));
    }
    const float diff = fsub(q[i], value);
    dist = fadd(dist, fmul(diff, diff));
  }
  return dist;
}

// First occurrence in lane order among lanes that hold the same id.
__device__ __forceinline__ bool first_of_equal(bool active, int32_t id, int lane) {
  const unsigned act = __ballot_sync(kFullMask, active);
  const unsigned same = __match_any_sync(kFullMask, active ? id : -2 - lane) & act;
  return active && (__ffs(same) - 1) == lane;
}

template <bool kSplit>
__global__ void __launch_bounds__(kSearchWarps * 32)
sq_search_kernel_t(SqSearchArgs a) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const SqIndexView& ix = a.ix;
  const int qbytes = ((ix.dim * 4) + 15) & ~15;
  const int cbytes = ((ix.dim + 15) & ~15);
  uint8_t* base = smem + static_cast<size_t>(warp) * (qbytes + cbytes + 64 * 8);
  float* q = reinterpret_cast<float*>(base);
  uint8_t* qc = base + qbytes;
  HeapEntry* work = reinterpret_cast<HeapEntry*>(base + qbytes + cbytes);  // 32 results
  int32_t* seeds = reinterpret_cast<int32_t*>(work + 32);                   // 32 ids
  const int slot = blockIdx.x * kSearchWarps + warp;
  HeapEntry* pool = reinterpret_cast<HeapEntry*>(a.heaps) +
                    static_cast<size_t>(slot) * (a.max_pool + a.frontier_cap);
  HeapEntry* front = pool + a.max_pool;
  VisitedTable vt;
  vt.slots = a.visited + static_cast<size_t>(slot) * (a.visited_mask + 1ull);
  vt.mask = a.visited_mask;
  const bool sqmd = a.mode == kSqModeSqmd;
  const bool db = a.mode == kSqModeDb;
  const bool split = kSplit && sqmd && a.correction;   // the host checks the index supports it

  for (;;) {
    int qi = 0;
    if (lane == 0) qi = static_cast<int>(atomicAdd(a.next_query, 1u));
    qi = __shfl_sync(kFullMask, qi, 0);
    if (qi >= a.nq) break;
    int32_t* status = a.status + qi;
    int cap = a.pool_sizes[qi];
    if (!sqmd && cap > 2000) cap = 2000;  // DSP_SEARCH_MAX_POOL
    const int expand = min(a.expand_count, ix.degree);
    if (cap <= 0 || cap > a.max_pool || expand <= 0 || a.entry_points <= 0 ||
        (sqmd && expand > 32) || (!sqmd && a.num_out <= 0)) {
      if (lane == 0) *status = kStatusBadParam;
      continue;
    }
    // frontier capacity the reference allocates for this request
    // (the DB-pair search grows its frontier up to n entries)
    const long long fcap_ref = db ? static_cast<long long>(ix.n)
                               : sqmd ? static_cast<long long>(a.entry_points) + static_cast<long long>(cap) * a.expand_count
                                      : static_cast<long long>(a.entry_points) + static_cast<long long>(cap) * expand;
    const int fcap = static_cast<int>(min(fcap_ref, static_cast<long long>(a.frontier_cap)));
    // query and its quantized codes (retrieval_quantize_query_u8/_u4,
    // l1_int8_core.c:13-63); with the split distance the codes of the
    // 17-fold refined grid instead (sq_split.cuh) and their sum
    const float inv = __frcp_rn(ix.l1_scale);
    const int levels = ix.l1_bits == 4 ? 15 : 255;
    const double step = split ? split_step(ix.l1_scale) : 0.0;
    unsigned long long sum_q = 0;
    bool qbad = false;
    for (int d = lane; d < ix.dim; d += kWarp) {
      const float v = a.queries[static_cast<size_t>(qi) * ix.dim + d];
      q[d] = v;
      if (split) {
        uint8_t c = 0;
        qbad |= !split_code(v, ix.l1_zero, step, &c);
        qc[d] = c;
        sum_q += c;
      } else {
        int c = static_cast<int>(roundf(fmul(fsub(v, ix.l1_zero), inv)));
        c = c < 0 ? 0 : (c > levels ? levels : c);
        qc[d] = static_cast<uint8_t>(c);
      }
    }
    if (split) {
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) sum_q += __shfl_xor_sync(kFullMask, sum_q, off);
      if (__any_sync(kFullMask, qbad)) {
        if (lane == 0) *status = kStatusNumeric;
        continue;
      }
    }
    __syncwarp();
    vt.gen = a.gen_base + static_cast<uint32_t>(qi);
    int psize = 0, fsize = 0;
    int32_t st = kStatusOk;
    unsigned long long scored = 0, turns = 0, dedup = 0;

    // ---- entries
    const int entries = min(a.entry_points, ix.n);
    uint32_t lcg = sqmd ? a.seed : 42u;
    uint64_t attempts = 0;
    const uint64_t attempt_limit = static_cast<uint64_t>(entries) * 64u + 1024u;
    int sweep = 0;
    bool graph_entry_used = false;
    for (int base_e = 0; base_e < entries && st == kStatusOk; base_e += kWarp) {
      // lane 0 produces the next chunk of entry ids in reference order
      if (lane == 0) {
        for (int t = 0; t < kWarp && base_e + t < entries; ++t) {
          const int i = base_e + t;
          int32_t id = -1;
          if (!sqmd) {
            if (i == 0 && a.graph_entry >= 0 && a.graph_entry < ix.n) {
              id = a.graph_entry;
            } else {
              lcg = lcg * 1103515245u + 12345u;
              id = static_cast<int32_t>((static_cast<uint64_t>(lcg) * static_cast<uint64_t>(ix.n)) >> 32);
            }
          } else {
            // retrieval_sqmd_make_seed_ids: graph entry, LCG (seed/65536)%n
            // with de-duplication, then an increasing sweep.  Seeds are
            // claimed in the visited table as they are drawn, which is both
            // the reference's de-duplication and sqmd_cpu_state_seed's claim.
            if (!graph_entry_used && a.graph_entry >= 0 && a.graph_entry < ix.n) {
              graph_entry_used = true;
              const int r = visited_insert(vt, static_cast<uint32_t>(a.graph_entry));
              if (r == 1) id = a.graph_entry;
              else if (r < 0) st = kStatusTableFull;
            }
            while (id < 0 && st == kStatusOk && attempts < attempt_limit) {
              lcg = lcg * 1103515245u + 12345u;
              const int32_t cand = static_cast<int32_t>((lcg / 65536u) % static_cast<uint32_t>(ix.n));
              ++attempts;
              const int r = visited_insert(vt, static_cast<uint32_t>(cand));
              if (r == 1) id = cand;
              else if (r < 0) st = kStatusTableFull;
            }
            while (id < 0 && st == kStatusOk && sweep < ix.n) {
              const int r = visited_insert(vt, static_cast<uint32_t>(sweep));
              if (r == 1) id = sweep;
              else if (r < 0) st = kStatusTableFull;
              ++sweep;
            }
          }
          seeds[t] = id;
        }
      }
      st = __shfl_sync(kFullMask, st, 0);
      __syncwarp();
      const int e = base_e + lane;
      const bool active = e < entries && seeds[lane] >= 0;
      const int32_t id = active ? seeds[lane] : -1;
      bool fresh = false;
      if (!sqmd) {
        // DSP: claim in entry order; duplicates after the first are skipped
        const bool first = first_of_equal(active, id, lane);
        if (first) {
          const int r = visited_insert(vt, static_cast<uint32_t>(id));
          if (r < 0) st = kStatusTableFull;
          fresh = r == 1;
        }
      } else {
        // SQMD seeds were claimed while being drawn (unique by construction)
        fresh = active;
      }
      float d = 0.0f;
      if (fresh) {
        d = split ? split_seed_distance(ix, qc, sum_q, id, step)
                  : (sqmd && a.correction) ? sq_exact(ix, q, id) : sq_coarse(ix, qc, id);
        if (sqmd && a.correction && (!isfinite(d) || d < 0.0f)) st = kStatusNumeric;
      }
      if (__any_sync(kFullMask, st != kStatusOk)) { st = st != kStatusOk ? st : kStatusNumeric; break; }
      work[lane].id = fresh ? id : -1;
      work[lane].dist = d;
      __syncwarp();
      if (lane == 0) {
        for (int t = 0; t < kWarp; ++t) {
          if (work[t].id < 0) continue;
          if (pool_insert(pool, &psize, cap, work[t].id, work[t].dist)) {
            if (fsize < fcap) {
              front[fsize] = work[t];
              front_sift_up(front, fsize);
              ++fsize;
            } else if (!sqmd) {
              st = kStatusFrontierFull;
            }
          }
        }
      }
      st = __shfl_sync(kFullMask, st, 0);
      __syncwarp();
    }
    st = __shfl_sync(kFullMask, st, 0);

    // ---- expansion loop
    while (st == kStatusOk) {
      int32_t src = -1;
      if (lane == 0) {
        while (fsize > 0 && psize >= cap && front[0].dist > pool[0].dist) front_pop(front, &fsize);
        if (fsize > 0) src = front_pop(front, &fsize);
      }
      src = __shfl_sync(kFullMask, src, 0);
      if (src < 0) break;
      const int32_t* row = ix.graph + static_cast<size_t>(src) * ix.degree;
      int nw = 0;
      for (int b = 0; b < expand; b += kWarp) {
        const int j = b + lane;
        int32_t nid = j < expand ? __ldg(row + j) : -1;
        bool ok = j < expand && nid >= 0 && nid < ix.n && (!sqmd || nid != src);
        const bool first = first_of_equal(ok, nid, lane);
        if (ok && !first) ++dedup;        // duplicate earlier in this row
        bool fresh = false;
        if (first) {
          const int r = visited_insert(vt, static_cast<uint32_t>(nid));
          if (r < 0) st = kStatusTableFull;
          fresh = r == 1;
          if (r == 0) ++dedup;
        }
        const unsigned fm = __ballot_sync(kFullMask, fresh);
        float d = 0.0f;
        bool dbad = false;
        if (fresh && split) {
          // sqmd_source_job_commit (sqmd_common.c:1533-1556): the lane's
          // coarse distance plus the host's delta, tiny negatives clamped
          const float dl = split_delta(ix, qc, sum_q, nid, step);
          d = split_sum(split_coarse(ix, qc, nid, step), dl);
          dbad = !isfinite(dl) || !isfinite(d) || d < 0.0f;
        } else if (fresh) {
          d = sq_coarse(ix, qc, nid);
          if ((sqmd || db) && a.correction) d = sq_exact(ix, q, nid);
        }
        if (split && __any_sync(kFullMask, dbad)) { st = kStatusNumeric; break; }
        const int slot_i = __popc(fm & ((1u << lane) - 1u));
        if (fresh) {
          work[slot_i].id = nid;
          work[slot_i].dist = d;
        }
        __syncwarp();
        if (__any_sync(kFullMask, st != kStatusOk)) { st = kStatusTableFull; break; }
        const int cnt = __popc(fm);
        if (lane == 0) {
          for (int t = 0; t < cnt; ++t) {
            if (pool_insert(pool, &psize, cap, work[t].id, work[t].dist)) {
              if (fsize < fcap) {
                front[fsize] = work[t];
                front_sift_up(front, fsize);
                ++fsize;
              } else if (!sqmd) {
                st = kStatusFrontierFull;
              }
            }
          }
        }
        nw += cnt;
        st = __shfl_sync(kFullMask, st, 0);
        __syncwarp();
        if (st != kStatusOk) break;
      }
      ++turns;
      scored += nw;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) dedup += __shfl_xor_sync(kFullMask, dedup, off);
    if (st != kStatusOk) {
      if (lane == 0) *status = st;
      continue;
    }
    if (lane == 0) {
      // sqmd_heap_sort / dsp_heap_sort: in-place heap sort, ascending
      for (int i = psize - 1; i > 0; --i) {
        const HeapEntry t = pool[0];
        pool[0] = pool[i];
        pool[i] = t;
        pool_sift_down(pool, i, 0);
      }
    }
    // the heaps (and their sizes) are lane 0's: broadcast the pool size
    psize = __shfl_sync(kFullMask, psize, 0);
    __syncwarp();
    const int limit = sqmd ? a.out_stride : a.num_out;
    const int outn = min(psize, min(limit, a.out_stride));
    for (int i = lane; i < outn; i += kWarp) {
      a.out_ids[static_cast<size_t>(qi) * a.out_stride + i] = pool[i].id;
      a.out_dists[static_cast<size_t>(qi) * a.out_stride + i] = pool[i].dist;
    }
    if (lane == 0) {
      a.out_counts[qi] = outn;
      if (a.stats) {
        unsigned long long* s = a.stats + static_cast<size_t>(qi) * 4;
        s[0] = scored;
        s[1] = sqmd ? scored : 0ull;
        s[2] = turns;
        s[3] = dedup;
      }
    }
    __syncwarp();
  }
}


SqSearchFn sq_search_kernel_for(bool split) {
  return split ? sq_search_kernel_t<true> : sq_search_kernel_t<false>;
}

// ---------------------------------------------------------------------------
// DB-pair search, one step per launch (calculator_retrieval_search_db).  Warp
// w serves slot w when io.op[w] asks for it:
//   kDbInit   db_search_state_init (retrieval_async_dsp_search.c:1205-1301):
//             quantized query, cleared visited bitmap, entries (graph entry,
//             then the LCG of dsp_search_select_entry_id) with their coarse
//             distances inserted in draw order;
//   kDbStep   db_search_apply_corrections (:1371-1389) for the ids the last
//             step returned, with the corrected distances the caller wrote
//             into io.corr, then db_search_expand_one_step (:1303-1369): pop
//             (dropping entries worse than a full pool's worst), read up to
//             expand_limit neighbours, skip invalid and visited ids, and
//             return the rest with their coarse distances -- or finished;
//   kDbFinish dsp_heap_sort and the first num_out entries.
// Heap operations run on lane 0 in the reference's order; lanes compute the
// coarse distances.
__global__ void __launch_bounds__(kDbSlots * 32) db_step_kernel(DbArgs a) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  DbIo& io = *a.io;
  const int op = io.op[w];
  if (op == kDbNone) return;
  const SqIndexView& ix = a.ix;
  DbSlot& s = a.slots[w];
  HeapEntry* pool = reinterpret_cast<HeapEntry*>(a.pools) + static_cast<size_t>(w) * a.pool_cap;
  HeapEntry* front = reinterpret_cast<HeapEntry*>(a.fronts) + static_cast<size_t>(w) * a.frontier_cap;
  const size_t vwords = (static_cast<size_t>(ix.n) + 31) / 32;
  uint32_t* visited = a.visited + static_cast<size_t>(w) * vwords;
  __shared__ HeapEntry work[kDbSlots][32];
  __shared__ int32_t ids[kDbSlots][32];
  int st = kStatusOk;
  auto push = [&](int32_t id, float d) {   // lane 0: pool insert, then frontier push
    if (pool_insert(pool, &s.psize, a.pool_cap, id, d)) {
      if (s.fsize >= a.frontier_cap) { st = kStatusFrontierFull; return; }
      front[s.fsize] = HeapEntry{id, d};
      front_sift_up(front, s.fsize);
      ++s.fsize;
    }
  };
  auto test_and_set = [&](int32_t id) {     // lane 0 only
    uint32_t& word = visited[id >> 5];
    const uint32_t bit = 1u << (id & 31);
    const bool seen = (word & bit) != 0;
    word |= bit;
    return !seen;
  };
  if (op == kDbInit) {
    const float* q = a.queries + static_cast<size_t>(w) * ix.dim;
    const float inv = __frcp_rn(ix.l1_scale);
    const int levels = ix.l1_bits == 4 ? 15 : 255;
    for (int d = lane; d < ix.dim; d += kWarp) {
      int c = static_cast<int>(roundf(fmul(fsub(q[d], ix.l1_zero), inv)));
      s.qc[d] = static_cast<uint8_t>(c < 0 ? 0 : (c > levels ? levels : c));
    }
    for (size_t i = lane; i < vwords; i += kWarp) visited[i] = 0u;
    if (lane == 0) { s.psize = s.fsize = s.finished = s.last_count = 0; }
    __syncwarp();
    __threadfence_block();
    const int entries = min(a.entry_points, ix.n);
    uint32_t lcg = 42u;   // DSP_SEARCH_ENTRY_SEED
    for (int e0 = 0; e0 < entries && st == kStatusOk; e0 += kWarp) {
      if (lane == 0) {
        for (int t = 0; t < kWarp; ++t) {
          const int i = e0 + t;
          int32_t id = -1;
          if (i < entries) {
            if (i == 0 && a.graph_entry >= 0 && a.graph_entry < ix.n) {
              id = a.graph_entry;
            } else {
              lcg = lcg * 1103515245u + 12345u;
              id = static_cast<int32_t>((static_cast<uint64_t>(lcg) * static_cast<uint64_t>(ix.n)) >> 32);
            }
            if (!test_and_set(id)) id = -1;
          }
          ids[w][t] = id;
        }
      }
      __syncwarp();
      const int32_t id = ids[w][lane];
      work[w][lane] = HeapEntry{id, id >= 0 ? sq_coarse(ix, s.qc, id) : 0.0f};
      __syncwarp();
      if (lane == 0)
        for (int t = 0; t < kWarp && st == kStatusOk; ++t)
          if (work[w][t].id >= 0) push(work[w][t].id, work[w][t].dist);
      st = __shfl_sync(kFullMask, st, 0);
      __syncwarp();
    }
    if (lane == 0) io.status[w] = st;
    return;
  }
  if (op == kDbFinish) {
    if (lane == 0) {
      for (int i = s.psize - 1; i > 0; --i) {     // dsp_heap_sort
        const HeapEntry t = pool[0];
        pool[0] = pool[i];
        pool[i] = t;
        pool_sift_down(pool, i, 0);
      }
      const int outn = min(a.num_out, s.psize);
      for (int i = 0; i < outn; ++i) {
        a.out_ids[static_cast<size_t>(w) * a.num_out + i] = pool[i].id;
        a.out_dists[static_cast<size_t>(w) * a.num_out + i] = pool[i].dist;
      }
      io.out_count[w] = outn;
      io.status[w] = kStatusOk;
    }
    return;
  }
  // kDbStep: the caller's corrections of the last step, then the next step
  int32_t src = -1;
  if (lane == 0) {
    const int nc = s.last_count;
    for (int t = 0; t < nc && st == kStatusOk; ++t) push(s.last_ids[t], io.corr[w][t]);
    if (st == kStatusOk) {
      while (s.fsize > 0 && s.psize >= a.pool_cap && front[0].dist > pool[0].dist) front_pop(front, &s.fsize);
      if (s.fsize > 0) src = front_pop(front, &s.fsize);
    }
  }
  st = __shfl_sync(kFullMask, st, 0);
  src = __shfl_sync(kFullMask, src, 0);
  if (st != kStatusOk || src < 0) {
    if (lane == 0) {
      s.finished = src < 0 ? 1 : s.finished;
      s.last_count = 0;
      io.count[w] = 0;
      io.finished[w] = src < 0;
      io.status[w] = st;
    }
    return;
  }
  if (lane == 0) {
    const int32_t* row = ix.graph + static_cast<size_t>(src) * ix.degree;
    int cnt = 0;
    for (int j = 0; j < a.expand_limit && cnt < kDbItems; ++j) {
      const int32_t nid = row[j];
      if (nid < 0 || nid >= ix.n) continue;
      if (!test_and_set(nid)) continue;
      ids[w][cnt++] = nid;
    }
    s.last_count = cnt;
    io.count[w] = cnt;
    io.finished[w] = 0;
    io.status[w] = kStatusOk;
  }
  __syncwarp();
  const int cnt = __shfl_sync(kFullMask, lane == 0 ? s.last_count : 0, 0);
  if (lane < cnt) {
    const int32_t nid = ids[w][lane];
    s.last_ids[lane] = nid;
    io.ids[w][lane] = nid;
    io.coarse[w][lane] = sq_coarse(ix, s.qc, nid);
  }
}

void launch_db_step(const DbArgs& a, cudaStream_t s) { db_step_kernel<<<1, kDbSlots * 32, 0, s>>>(a); }

}  // namespace rover
