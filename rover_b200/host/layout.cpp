// layout.cpp -- neighbourhood-aware id layout of an index (the reference's
// rover-layout tool, src/graph/layout_opt_kmeans.cpp:55-712): nodes that a
// search expands together get neighbouring ids, so their codes, residual rows
// and decoded rows share blocks.
//
// Nodes come grouped by a clustering (one label per node).  Inside each
// cluster, ids are handed out block by block (vectors_per_block nodes per
// block): a block starts at the unplaced node of highest in-degree (ties: lower
// id) and grows greedily by the unplaced node of the cluster with the highest
// accumulated affinity to the nodes already in the block (ties: higher
// in-degree, then lower id).  The affinity a newly placed node u passes to a
// candidate v is a reciprocal-rank fusion, 1 / (c + rank), of two rankings
// of the cluster's unplaced nodes:
//   common neighbours  sum over u's out-neighbours z of
//                      degree(z) / sqrt(rank of z in u's row * rank of z in
//                      v's row), over z's reverse edges (v -> z);
//   mutual neighbours  1 / rank of v in u's row, plus 1 / rank of u in v's
//                      row;
// each ranking by score, descending, ties by lower id.  A node's reverse
// edges are the (rank, source) pairs of the rows that point at it, smallest
// first, at most max_reverse of them.  The final order lists every cluster's
// full blocks, cluster by cluster, then every cluster's last partial block.
//
// The reference keeps per-node hash maps; here each cluster works on dense
// arrays indexed by the node's position in its cluster, with lists of the
// positions touched, and clusters run on a pool of host threads.  Every sum
// is formed in the reference's order, so the layout is the reference's
// exactly (tests/test_layout.py runs both on the same graphs and labels).

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

namespace {

constexpr uint32_t kNone = 0xffffffffu;

struct Graph {
  const int32_t* rows;
  int32_t n, degree;
  std::vector<int32_t> len;                 // valid prefix of each row
  std::vector<uint32_t> in_degree, degree_sum;
  std::vector<size_t> rev_off;              // reverse edges of node v: rev[rev_off[v] .. rev_off[v + 1])
  std::vector<uint64_t> rev;                // (rank << 32) | source
  const int32_t* row(uint32_t u) const { return rows + static_cast<size_t>(u) * degree; }
};

// Row lengths, degrees and the reverse edges (preprocessGraphSparse,
// layout_opt_kmeans.cpp:55-156).  False on an id outside the graph.
bool prepare(Graph& g, uint32_t max_reverse) {
  const uint32_t n = static_cast<uint32_t>(g.n);
  g.len.assign(n, 0);
  g.in_degree.assign(n, 0);
  std::vector<uint32_t> out(n, 0);
  for (uint32_t u = 0; u < n; ++u) {
    const int32_t* r = g.row(u);
    int32_t k = 0;
    while (k < g.degree && r[k] >= 0) ++k;
    g.len[u] = k;
    for (int32_t j = 0; j < k; ++j) {
      if (r[j] >= g.n) return false;
      if (static_cast<uint32_t>(r[j]) == u) continue;
      ++g.in_degree[r[j]];
      ++out[u];
    }
  }
  std::vector<size_t> fill(n + 1, 0);
  for (uint32_t v = 0; v < n; ++v) fill[v + 1] = fill[v] + g.in_degree[v];
  std::vector<uint64_t> all(fill[n]);
  std::vector<size_t> pos(fill.begin(), fill.end() - 1);
  for (uint32_t u = 0; u < n; ++u) {
    const int32_t* r = g.row(u);
    uint64_t rank = 1;
    for (int32_t j = 0; j < g.len[u]; ++j) {
      const uint32_t v = static_cast<uint32_t>(r[j]);
      if (v == u) continue;
      all[pos[v]++] = (rank << 32) | u;
      ++rank;
    }
  }
  g.rev_off.assign(n + 1, 0);
  for (uint32_t v = 0; v < n; ++v) {
    const size_t cnt = fill[v + 1] - fill[v];
    const size_t keep = max_reverse > 0 ? std::min<size_t>(cnt, max_reverse) : cnt;
    g.rev_off[v + 1] = g.rev_off[v] + keep;
  }
  g.rev.resize(g.rev_off[n]);
  for (uint32_t v = 0; v < n; ++v) {
    // (rank, source) pairs are distinct, so the smallest `keep` of a full
    // sort are the ones the reference keeps
    std::sort(all.begin() + fill[v], all.begin() + fill[v + 1]);
    std::copy(all.begin() + fill[v], all.begin() + fill[v] + (g.rev_off[v + 1] - g.rev_off[v]),
              g.rev.begin() + g.rev_off[v]);
  }
  g.degree_sum.resize(n);
  for (uint32_t v = 0; v < n; ++v) g.degree_sum[v] = g.in_degree[v] + out[v];
  return true;
}

// One cluster's order (reorderOneCluster, :418-562).
class ClusterOrder {
 public:
  ClusterOrder(const Graph& g, const std::vector<uint32_t>& nodes, const std::vector<uint32_t>& local,
               const std::vector<int32_t>& label, int32_t cluster, uint32_t per_block, double rrf_c, bool use_cn,
               bool use_mnn)
      : g_(g), nodes_(nodes), local_(local), label_(label), cluster_(cluster), per_block_(per_block),
        rrf_c_(rrf_c), use_cn_(use_cn), use_mnn_(use_mnn), open_(nodes.size(), 1), cn_(nodes.size(), 0.0),
        mnn_(nodes.size(), 0.0), block_(nodes.size(), 0.0), seen_(nodes.size(), 0), in_block_list_(nodes.size(), 0) {}

  std::vector<uint32_t> run() {
    std::vector<uint32_t> order;
    order.reserve(nodes_.size());
    size_t remaining = nodes_.size(), seed = 0;
    while (remaining > 0) {
      const uint32_t first = next_seed(&seed);
      if (first == kNone) break;
      for (uint32_t p : block_list_) { block_[p] = 0.0; in_block_list_[p] = 0; }
      block_list_.clear();
      uint32_t in_block = 0;
      place(first, &order, &remaining);
      ++in_block;
      while (in_block < per_block_ && remaining > 0) {
        uint32_t best = kNone;
        double best_score = -1.0;
        for (uint32_t p : block_list_) {
          if (!open_[p]) continue;
          const uint32_t v = nodes_[p];
          const double s = block_[p];
          if (best == kNone || s > best_score ||
              (s == best_score && (g_.in_degree[v] > g_.in_degree[best] ||
                                   (g_.in_degree[v] == g_.in_degree[best] && v < best)))) {
            best = v;
            best_score = s;
          }
        }
        if (best == kNone) best = next_seed(&seed);
        if (best == kNone) break;
        place(best, &order, &remaining);
        ++in_block;
      }
    }
    return order;
  }

 private:
  bool candidate(uint32_t v) const {
    return label_[v] == cluster_ && open_[local_[v]];
  }

  uint32_t next_seed(size_t* seed) const {
    while (*seed < nodes_.size()) {
      const uint32_t v = nodes_[(*seed)++];
      if (open_[local_[v]]) return v;
    }
    return kNone;
  }

  void touch(uint32_t p) {
    if (!seen_[p]) { seen_[p] = 1; touched_.push_back(p); }
  }

  // Places u and passes its affinities to the block's candidates
  // (computeDirectedRRFForNodeInCluster, :180-395).
  void place(uint32_t u, std::vector<uint32_t>* order, size_t* remaining) {
    open_[local_[u]] = 0;
    --*remaining;
    order->push_back(u);
    const int32_t* r = g_.row(u);
    const int32_t len = g_.len[u];
    if (use_cn_) {
      double rank_uz = 1.0;
      for (int32_t j = 0; j < len; ++j, rank_uz += 1.0) {
        const uint32_t z = static_cast<uint32_t>(r[j]);
        if (z == u) continue;
        for (size_t e = g_.rev_off[z]; e < g_.rev_off[z + 1]; ++e) {
          const uint32_t v = static_cast<uint32_t>(g_.rev[e]);
          if (v == u || !candidate(v)) continue;
          const double rank_vz = static_cast<double>(g_.rev[e] >> 32);
          const uint32_t p = local_[v];
          touch(p);
          cn_[p] += static_cast<double>(g_.degree_sum[z]) / std::sqrt(rank_uz * rank_vz);
        }
      }
    }
    if (use_mnn_) {
      double rank_uv = 1.0;
      for (int32_t j = 0; j < len; ++j, rank_uv += 1.0) {
        const uint32_t v = static_cast<uint32_t>(r[j]);
        if (v == u || !candidate(v)) continue;
        touch(local_[v]);
        mnn_[local_[v]] += 1.0 / rank_uv;
      }
      for (size_t e = g_.rev_off[u]; e < g_.rev_off[u + 1]; ++e) {
        const uint32_t v = static_cast<uint32_t>(g_.rev[e]);
        if (v == u || !candidate(v)) continue;
        touch(local_[v]);
        mnn_[local_[v]] += 1.0 / static_cast<double>(g_.rev[e] >> 32);
      }
    }
    // the two rankings, fused
    rrf_.assign(touched_.size(), 0.0);
    for (int which = 0; which < 2; ++which) {
      if (which == 0 ? !use_cn_ : !use_mnn_) continue;
      const std::vector<double>& sc = which == 0 ? cn_ : mnn_;
      ranked_.clear();
      for (size_t t = 0; t < touched_.size(); ++t)
        if (sc[touched_[t]] > 0.0) ranked_.push_back(static_cast<uint32_t>(t));
      std::sort(ranked_.begin(), ranked_.end(), [&](uint32_t a, uint32_t b) {
        const double sa = sc[touched_[a]], sb = sc[touched_[b]];
        if (sa != sb) return sa > sb;
        return nodes_[touched_[a]] < nodes_[touched_[b]];
      });
      for (size_t k = 0; k < ranked_.size(); ++k) rrf_[ranked_[k]] += 1.0 / (rrf_c_ + static_cast<double>(k + 1));
    }
    for (size_t t = 0; t < touched_.size(); ++t) {
      const uint32_t p = touched_[t];
      if (rrf_[t] > 0.0 && open_[p]) {
        if (!in_block_list_[p]) { in_block_list_[p] = 1; block_list_.push_back(p); }
        block_[p] += rrf_[t];
      }
      cn_[p] = mnn_[p] = 0.0;
      seen_[p] = 0;
    }
    touched_.clear();
  }

  const Graph& g_;
  const std::vector<uint32_t>& nodes_;
  const std::vector<uint32_t>& local_;
  const std::vector<int32_t>& label_;
  const int32_t cluster_;
  const uint32_t per_block_;
  const double rrf_c_;
  const bool use_cn_, use_mnn_;
  std::vector<char> open_;
  std::vector<double> cn_, mnn_, block_, rrf_;
  std::vector<char> seen_, in_block_list_;
  std::vector<uint32_t> touched_, block_list_, ranked_;
};

}  // namespace

extern "C" int rover_layout_order(const int32_t* graph, int32_t n, int32_t degree, const int32_t* labels,
                                  int32_t clusters, int32_t vectors_per_block, double rrf_c, int32_t max_reverse,
                                  int32_t use_cn, int32_t use_mnn, int32_t threads, int32_t* new_to_old) {
  if (!graph || !labels || !new_to_old || n <= 0 || degree <= 0 || clusters <= 0 || vectors_per_block <= 0 ||
      (!use_cn && !use_mnn) || max_reverse < 0)
    return -1;
  Graph g{graph, n, degree, {}, {}, {}, {}, {}};
  if (!prepare(g, static_cast<uint32_t>(max_reverse))) return -1;
  std::vector<int32_t> label(labels, labels + n);
  std::vector<std::vector<uint32_t>> members(clusters);
  for (int32_t i = 0; i < n; ++i) {
    if (label[i] < 0 || label[i] >= clusters) return -1;
    members[label[i]].push_back(static_cast<uint32_t>(i));
  }
  std::vector<uint32_t> local(n, kNone);
  for (auto& m : members) {
    std::sort(m.begin(), m.end(), [&](uint32_t a, uint32_t b) {
      if (g.in_degree[a] != g.in_degree[b]) return g.in_degree[a] > g.in_degree[b];
      return a < b;
    });
    for (size_t p = 0; p < m.size(); ++p) local[m[p]] = static_cast<uint32_t>(p);
  }
  std::vector<std::vector<uint32_t>> orders(clusters);
  std::atomic<int32_t> next{0};
  auto worker = [&]() {
    for (int32_t c; (c = next.fetch_add(1)) < clusters;)
      orders[c] = ClusterOrder(g, members[c], local, label, c, static_cast<uint32_t>(vectors_per_block), rrf_c,
                               use_cn != 0, use_mnn != 0).run();
  };
  const int nt = std::max(1, std::min<int>(threads > 0 ? threads : 1, clusters));
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
  worker();
  for (auto& t : pool) t.join();
  size_t k = 0;
  for (int pass = 0; pass < 2; ++pass)
    for (int32_t c = 0; c < clusters; ++c) {
      const auto& o = orders[c];
      if (o.size() != members[c].size()) return -1;
      const size_t full = o.size() / vectors_per_block * vectors_per_block;
      const size_t b = pass == 0 ? 0 : full, e = pass == 0 ? full : o.size();
      for (size_t i = b; i < e; ++i) new_to_old[k++] = static_cast<int32_t>(o[i]);
    }
  return k == static_cast<size_t>(n) ? 0 : -1;
}
