// Multilevel recursive graph bisection: the partitioner for matrices without
// row coordinates, in the role METIS_PartGraphRecursive plays in the
// reference (CRSHostMatrix.cpp:139-271: vertex weight = off-diagonals of the
// row + 1, unit edge weights, minimum edge cut, C numbering).
//
// Each bisection follows the multilevel scheme of Karypis and Kumar ("A fast
// and high quality multilevel scheme for partitioning irregular graphs",
// SIAM J. Sci. Comput. 20(1), 1998):
//   1. coarsening by heavy-edge matching in a seeded random vertex order,
//      merging matched pairs (coarse vertex weight capped) until the graph
//      has at most kCoarsest vertices or stops shrinking;
//   2. an initial bisection of the coarsest graph by greedy graph growing
//      from several seeds, each refined, the smallest balanced cut kept;
//   3. uncoarsening: the sides projected level by level, each level refined
//      by Fiduccia-Mattheyses passes over the boundary vertices (gain
//      buckets as heaps, moves that break the balance skipped, a pass
//      rolled back to its best prefix, an overweight side emptied first).
// The graph is the symmetrised off-diagonal pattern. Parts are split as
// p1 = parts / 2 against parts - p1 with the weight target in proportion, and
// the two induced subgraphs are partitioned recursively (in parallel near the
// top). Everything is seeded, so the result is deterministic.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <numeric>
#include <queue>
#include <thread>
#include <utility>
#include <vector>

#include "host_matrix.hpp"

namespace gr {

namespace {

constexpr i64 kCoarsest = 160;       // stop coarsening at this many vertices
constexpr double kImbalance = 0.002;  // allowed excess over a side's target, per bisection
constexpr int kInitialTries = 8;
constexpr int kFmPasses = 8;
constexpr int kCycles = 4;  // independent multilevel bisections, the best kept

struct Graph {
  i64 n = 0;
  std::vector<i64> xadj;  // n + 1
  std::vector<i32> adj;
  std::vector<i32> ew;
  std::vector<i64> vw;
  i64 totalW = 0;
};

struct Rng {
  u64 s;
  explicit Rng(u64 seed) : s(seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull) {}
  u64 next() {
    u64 z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  i64 below(i64 k) { return static_cast<i64>(next() % static_cast<u64>(k)); }
};

std::vector<i32> randomOrder(i64 n, Rng& rng) {
  std::vector<i32> p(n);
  std::iota(p.begin(), p.end(), 0);
  for (i64 i = n - 1; i > 0; --i) std::swap(p[i], p[rng.below(i + 1)]);
  return p;
}

// One coarsening step: heavy-edge matching and the contracted graph.
// Returns false when the graph would shrink by less than 5 %.
bool coarsen(const Graph& G, Rng& rng, Graph& C, std::vector<i32>& cmap) {
  const i64 n = G.n;
  const i64 maxVw = std::max<i64>(1, (3 * G.totalW) / (2 * kCoarsest));
  std::vector<i32> match(n, -1);
  const u64 salt = rng.next();
  for (i32 v : randomOrder(n, rng)) {
    if (match[v] != -1) continue;
    // The heaviest edge; ties to the lighter vertex, then a seeded hash
    // (not the adjacency order, which would contract a grid along one axis).
    i32 best = -1, bw = -1;
    i64 bvw = 0;
    u64 bh = 0;
    for (i64 k = G.xadj[v]; k < G.xadj[v + 1]; ++k) {
      const i32 u = G.adj[k];
      if (match[u] != -1 || u == v || G.vw[v] + G.vw[u] > maxVw) continue;
      const u64 h = (static_cast<u64>(u) + salt) * 0x9E3779B97F4A7C15ull;
      if (G.ew[k] > bw || (G.ew[k] == bw && (G.vw[u] < bvw || (G.vw[u] == bvw && h > bh)))) {
        best = u;
        bw = G.ew[k];
        bvw = G.vw[u];
        bh = h;
      }
    }
    if (best < 0) {
      match[v] = v;
    } else {
      match[v] = best;
      match[best] = v;
    }
  }
  cmap.assign(n, -1);
  i64 cn = 0;
  for (i64 v = 0; v < n; ++v) {
    if (cmap[v] != -1) continue;
    cmap[v] = static_cast<i32>(cn);
    cmap[match[v]] = static_cast<i32>(cn);
    ++cn;
  }
  if (cn > n - n / 20) return false;
  C.n = cn;
  C.vw.assign(cn, 0);
  C.xadj.assign(cn + 1, 0);
  C.adj.clear();
  C.ew.clear();
  C.adj.reserve(G.adj.size());
  C.ew.reserve(G.adj.size());
  C.totalW = G.totalW;
  std::vector<i64> slot(cn, -1);
  std::vector<i32> first(cn, -1);
  for (i64 v = 0; v < n; ++v)
    if (first[cmap[v]] < 0) first[cmap[v]] = static_cast<i32>(v);
  for (i64 c = 0; c < cn; ++c) {
    const i64 start = static_cast<i64>(C.adj.size());
    const i32 v = first[c], u = match[v];
    for (i32 w : {v, u}) {
      C.vw[c] += G.vw[w];
      for (i64 k = G.xadj[w]; k < G.xadj[w + 1]; ++k) {
        const i32 cw = cmap[G.adj[k]];
        if (cw == c) continue;
        if (slot[cw] < start) {
          slot[cw] = static_cast<i64>(C.adj.size());
          C.adj.push_back(cw);
          C.ew.push_back(G.ew[k]);
        } else {
          C.ew[slot[cw]] += G.ew[k];
        }
      }
      if (u == v) break;
    }
    C.xadj[c + 1] = static_cast<i64>(C.adj.size());
  }
  return true;
}

struct Bisection {
  std::vector<uint8_t> side;
  i64 w[2] = {0, 0};
  i64 cut = 0;
};

i64 cutOf(const Graph& G, const std::vector<uint8_t>& side) {
  i64 cut = 0;
  for (i64 v = 0; v < G.n; ++v)
    for (i64 k = G.xadj[v]; k < G.xadj[v + 1]; ++k)
      if (side[G.adj[k]] != side[v]) cut += G.ew[k];
  return cut / 2;
}

// Balance test: side s may hold at most maxW[s].
struct Limits {
  i64 target[2];
  i64 maxW[2];
};

Limits limitsFor(const Graph& G, double frac0) {
  Limits L;
  L.target[0] = static_cast<i64>(static_cast<double>(G.totalW) * frac0 + 0.5);
  L.target[1] = G.totalW - L.target[0];
  i64 maxVw = 1;
  for (i64 v = 0; v < G.n; ++v) maxVw = std::max(maxVw, G.vw[v]);
  for (int s = 0; s < 2; ++s) {
    const i64 slack = std::max<i64>(static_cast<i64>(kImbalance * static_cast<double>(L.target[s])), maxVw);
    L.maxW[s] = L.target[s] + slack;
  }
  return L;
}

double overload(const Bisection& B, const Limits& L) {
  double o = 0;
  for (int s = 0; s < 2; ++s)
    if (B.w[s] > L.maxW[s]) o += static_cast<double>(B.w[s] - L.maxW[s]);
  return o;
}

// Fiduccia-Mattheyses refinement of B in place.
void refine(const Graph& G, const Limits& L, Bisection& B) {
  const i64 n = G.n;
  std::vector<i64> id(n, 0), ed(n, 0);  // edge weight to own side / to the other side
  auto degrees = [&]() {
    for (i64 v = 0; v < n; ++v) {
      id[v] = ed[v] = 0;
      for (i64 k = G.xadj[v]; k < G.xadj[v + 1]; ++k) (B.side[G.adj[k]] == B.side[v] ? id[v] : ed[v]) += G.ew[k];
    }
  };
  std::vector<uint8_t> locked(n, 0);
  std::vector<i32> moved;
  using Item = std::pair<i64, i32>;  // (gain, vertex)
  for (int pass = 0; pass < kFmPasses; ++pass) {
    degrees();
    std::priority_queue<Item> q[2];
    for (i64 v = 0; v < n; ++v)
      if (ed[v] > 0 || B.w[B.side[v]] > L.maxW[B.side[v]]) q[B.side[v]].push({ed[v] - id[v], static_cast<i32>(v)});
    std::fill(locked.begin(), locked.end(), 0);
    moved.clear();
    const i64 startCut = B.cut;
    const double startOver = overload(B, L);
    i64 bestCut = B.cut;
    double bestOver = startOver;
    size_t bestLen = 0;
    const size_t patience = static_cast<size_t>(std::max<i64>(50, std::min<i64>(1000, n / 20)));
    for (;;) {
      // Source side: an overweight side first, else the side with the
      // larger top gain among feasible moves.
      int from = -1;
      for (int s = 0; s < 2; ++s)
        if (B.w[s] > L.maxW[s]) from = s;
      auto top = [&](int s) -> i64 {
        while (!q[s].empty()) {
          const auto [g, v] = q[s].top();
          if (locked[v] || B.side[v] != s || g != ed[v] - id[v]) {
            q[s].pop();
            continue;
          }
          return g;
        }
        return INT64_MIN;
      };
      if (from < 0) {
        const i64 g0 = top(0), g1 = top(1);
        if (g0 == INT64_MIN && g1 == INT64_MIN) break;
        from = g0 >= g1 ? 0 : 1;
        if (top(from) == INT64_MIN) from ^= 1;
      }
      if (top(from) == INT64_MIN) break;
      const i32 v = q[from].top().second;
      q[from].pop();
      const int to = from ^ 1;
      const bool fixesLoad = B.w[from] > L.maxW[from];
      if (!fixesLoad && B.w[to] + G.vw[v] > L.maxW[to]) {
        locked[v] = 1;  // would break the balance: not this pass
        continue;
      }
      // Move v.
      B.cut -= ed[v] - id[v];
      B.side[v] = static_cast<uint8_t>(to);
      B.w[from] -= G.vw[v];
      B.w[to] += G.vw[v];
      std::swap(id[v], ed[v]);
      locked[v] = 2;
      moved.push_back(v);
      for (i64 k = G.xadj[v]; k < G.xadj[v + 1]; ++k) {
        const i32 u = G.adj[k];
        if (B.side[u] == to) {
          id[u] += G.ew[k];
          ed[u] -= G.ew[k];
        } else {
          id[u] -= G.ew[k];
          ed[u] += G.ew[k];
        }
        if (!locked[u]) q[B.side[u]].push({ed[u] - id[u], u});
      }
      const double over = overload(B, L);
      if (over < bestOver || (over == bestOver && B.cut < bestCut)) {
        bestOver = over;
        bestCut = B.cut;
        bestLen = moved.size();
      } else if (moved.size() - bestLen > patience) {
        break;
      }
    }
    // Roll back the moves after the best prefix.
    for (size_t i = moved.size(); i > bestLen; --i) {
      const i32 v = moved[i - 1];
      const int from = B.side[v], to = from ^ 1;
      B.side[v] = static_cast<uint8_t>(to);
      B.w[from] -= G.vw[v];
      B.w[to] += G.vw[v];
    }
    B.cut = bestCut;
    if (bestCut >= startCut && bestOver >= startOver) break;
  }
}

// Greedy graph growing from `seed`: side 0 takes the boundary vertex that
// adds the least cut until it reaches its target.
Bisection grow(const Graph& G, const Limits& L, i32 seed, Rng& rng) {
  Bisection B;
  B.side.assign(G.n, 1);
  B.w[1] = G.totalW;
  std::vector<i64> gain(G.n, 0);  // edge weight into side 0 minus into side 1
  for (i64 v = 0; v < G.n; ++v)
    for (i64 k = G.xadj[v]; k < G.xadj[v + 1]; ++k) gain[v] -= G.ew[k];
  std::priority_queue<std::pair<i64, i32>> q;
  const std::vector<i32> order = randomOrder(G.n, rng);  // seeds for exhausted components
  i64 pos = 0;
  auto take = [&](i32 v) {
    B.side[v] = 0;
    B.w[0] += G.vw[v];
    B.w[1] -= G.vw[v];
    for (i64 k = G.xadj[v]; k < G.xadj[v + 1]; ++k) {
      const i32 u = G.adj[k];
      gain[u] += 2 * G.ew[k];
      if (B.side[u] == 1) q.push({gain[u], u});
    }
  };
  take(seed);
  while (B.w[0] < L.target[0]) {
    i32 v = -1;
    while (!q.empty()) {
      const auto [g, u] = q.top();
      q.pop();
      if (B.side[u] == 1 && g == gain[u]) {
        v = u;
        break;
      }
    }
    if (v < 0) {  // the region's component is exhausted: a new seed
      while (pos < G.n && B.side[order[pos]] == 0) ++pos;
      if (pos == G.n) break;
      v = order[pos];
    }
    if (B.w[0] + G.vw[v] > L.maxW[0] && B.w[0] > 0) break;
    take(v);
  }
  B.cut = cutOf(G, B.side);
  return B;
}

Bisection initialBisection(const Graph& G, const Limits& L, Rng& rng) {
  Bisection best;
  bool have = false;
  for (int t = 0; t < kInitialTries; ++t) {
    const i32 seed = static_cast<i32>(rng.below(G.n));
    Bisection B = grow(G, L, seed, rng);
    refine(G, L, B);
    const double o = overload(B, L);
    if (!have || o < overload(best, L) || (o == overload(best, L) && B.cut < best.cut)) {
      best = std::move(B);
      have = true;
    }
  }
  return best;
}

// Multilevel bisection of G with side 0 targeting frac0 of the weight.
Bisection bisectOnce(const Graph& G, double frac0, u64 seed) {
  Rng rng(seed);
  std::vector<Graph> levels;
  std::vector<std::vector<i32>> maps;
  const Graph* cur = &G;
  while (cur->n > kCoarsest) {
    Graph C;
    std::vector<i32> cmap;
    if (!coarsen(*cur, rng, C, cmap)) break;
    levels.push_back(std::move(C));
    maps.push_back(std::move(cmap));
    cur = &levels.back();
  }
  Bisection B = initialBisection(*cur, limitsFor(*cur, frac0), rng);
  for (size_t l = levels.size(); l-- > 0;) {
    const Graph& fine = l == 0 ? G : levels[l - 1];
    Bisection F;
    F.side.resize(fine.n);
    for (i64 v = 0; v < fine.n; ++v) F.side[v] = B.side[maps[l][v]];
    F.w[0] = B.w[0];
    F.w[1] = B.w[1];
    F.cut = B.cut;
    refine(fine, limitsFor(fine, frac0), F);
    B = std::move(F);
  }
  return B;
}

// The best (balanced first, then smallest cut) of kCycles multilevel
// bisections from different seeds.
std::vector<uint8_t> bisect(const Graph& G, double frac0, u64 seed) {
  const Limits L = limitsFor(G, frac0);
  Bisection best;
  for (int t = 0; t < kCycles; ++t) {
    Bisection B = bisectOnce(G, frac0, seed * 7919 + static_cast<u64>(t));
    if (t == 0 || overload(B, L) < overload(best, L) ||
        (overload(B, L) == overload(best, L) && B.cut < best.cut))
      best = std::move(B);
  }
  return std::move(best.side);
}

// The subgraph induced by the vertices with side == s; ids[k] is the
// parent id of subgraph vertex k.
Graph induced(const Graph& G, const std::vector<uint8_t>& side, int s, std::vector<i32>& ids) {
  std::vector<i32> loc(G.n, -1);
  ids.clear();
  for (i64 v = 0; v < G.n; ++v)
    if (side[v] == s) {
      loc[v] = static_cast<i32>(ids.size());
      ids.push_back(static_cast<i32>(v));
    }
  Graph S;
  S.n = static_cast<i64>(ids.size());
  S.xadj.assign(S.n + 1, 0);
  S.vw.resize(S.n);
  for (i64 k = 0; k < S.n; ++k) {
    const i32 v = ids[k];
    S.vw[k] = G.vw[v];
    S.totalW += G.vw[v];
    for (i64 e = G.xadj[v]; e < G.xadj[v + 1]; ++e)
      if (loc[G.adj[e]] >= 0) {
        S.adj.push_back(loc[G.adj[e]]);
        S.ew.push_back(G.ew[e]);
      }
    S.xadj[k + 1] = static_cast<i64>(S.adj.size());
  }
  return S;
}

void recurse(const Graph& G, const std::vector<i32>& ids, i32 parts, i32 first, i32* out, u64 seed, int depth) {
  if (G.n == 0) return;
  if (parts == 1 || G.n == 1) {
    for (i64 k = 0; k < G.n; ++k) out[ids[k]] = first;
    return;
  }
  const i32 p1 = parts / 2;
  const std::vector<uint8_t> side = bisect(G, static_cast<double>(p1) / parts, seed);
  std::vector<i32> id0, id1;
  Graph G0 = induced(G, side, 0, id0);
  Graph G1 = induced(G, side, 1, id1);
  for (auto& v : id0) v = ids[v];
  for (auto& v : id1) v = ids[v];
  const u64 s0 = seed * 2 + 1, s1 = seed * 2 + 2;
  if (depth < 5 && G.n > 100000) {
    std::thread th([&]() { recurse(G0, id0, p1, first, out, s0, depth + 1); });
    recurse(G1, id1, parts - p1, first + p1, out, s1, depth + 1);
    th.join();
  } else {
    recurse(G0, id0, p1, first, out, s0, depth + 1);
    recurse(G1, id1, parts - p1, first + p1, out, s1, depth + 1);
  }
}

}  // namespace

std::vector<i32> partitionMultilevel(const HostMatrix& A, i32 numParts) {
  const i64 n = A.n;
  if (n >= (i64(1) << 31)) fail(GR_EUNSUPPORTED, "multilevel partitioning supports fewer than 2^31 rows");
  // Symmetrised off-diagonal pattern, unit edge weights; vertex weight =
  // off-diagonals of the row + 1.
  Graph G;
  G.n = n;
  std::vector<i64> deg(n + 1, 0);
  for (i64 r = 0; r < n; ++r)
    for (i64 k = A.gRowPtr[r]; k < A.gRowPtr[r + 1]; ++k) {
      const i64 c = A.gCol[k];
      if (c == r) continue;
      ++deg[r + 1];
      ++deg[c + 1];
    }
  for (i64 r = 0; r < n; ++r) deg[r + 1] += deg[r];
  std::vector<i32> adj(deg[n]);
  std::vector<i64> fill(deg.begin(), deg.end() - 1);
  for (i64 r = 0; r < n; ++r)
    for (i64 k = A.gRowPtr[r]; k < A.gRowPtr[r + 1]; ++k) {
      const i64 c = A.gCol[k];
      if (c == r) continue;
      adj[fill[r]++] = static_cast<i32>(c);
      adj[fill[c]++] = static_cast<i32>(r);
    }
  G.xadj.assign(n + 1, 0);
  G.adj.reserve(adj.size());
  for (i64 r = 0; r < n; ++r) {
    auto b = adj.begin() + deg[r], e = adj.begin() + deg[r + 1];
    std::sort(b, e);
    e = std::unique(b, e);
    G.adj.insert(G.adj.end(), b, e);
    G.xadj[r + 1] = static_cast<i64>(G.adj.size());
  }
  G.ew.assign(G.adj.size(), 1);
  G.vw.resize(n);
  for (i64 r = 0; r < n; ++r) {
    G.vw[r] = A.gRowPtr[r + 1] - A.gRowPtr[r] + 1;
    G.totalW += G.vw[r];
  }
  std::vector<i32> part(n, 0), ids(n);
  std::iota(ids.begin(), ids.end(), 0);
  recurse(G, ids, numParts, 0, part.data(), 1, 0);
  return part;
}

i64 edgeCut(const HostMatrix& A, const std::vector<i32>& rowToTile) {
  i64 cut = 0;
  for (i64 r = 0; r < A.n; ++r)
    for (i64 k = A.gRowPtr[r]; k < A.gRowPtr[r + 1]; ++k)
      if (rowToTile[A.gCol[k]] != rowToTile[r]) ++cut;
  return cut;
}

}  // namespace gr
