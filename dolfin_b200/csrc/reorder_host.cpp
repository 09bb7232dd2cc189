// reorder_host.cpp -- reordered dof numbering (reorder_dofs_serial = True) and the
// reordered CSR of a pattern (host only).
//
// DofMapBuilder::build with reordering on a single process
// (dolfin/fem/DofMapBuilder.cpp:168-252, compute_node_reordering :1473-1667,
// build_dofmap :1669-1693) with dof_ordering_library = "Boost":
//   1. the node graph: for each cell in order, for each pair of its nodes
//      (i, j), i != j, in local order, graph[i].insert(j) into a dolfin::Set
//      (insertion order kept, duplicates skipped) (:1527-1556);
//   2. node_remap = BoostGraphOrdering::compute_cuthill_mckee(graph, true)
//      (dolfin/graph/BoostGraphOrdering.cpp:34-75): Boost's
//      cuthill_mckee_ordering over a compressed-sparse-row copy of the graph
//      (out-edges in Set order), written through a reverse iterator, i.e.
//      reverse Cuthill-McKee; map[old] = new;
//   3. dofs: dof(c, node) = bs * node_remap[node] + c (node-major blocks).
// Boost is not part of the reference tree; its published algorithm
// (boost/graph/cuthill_mckee_ordering.hpp, sparse_ordering.hpp) is restated:
// one start per connected component (the first unvisited vertex in index
// order), moved to a pseudo-peripheral vertex by repeated BFS (the
// minimum-degree vertex of the last level, first such vertex on ties; repeat
// while the eccentricity grows); then BFS in which the children of each
// dequeued vertex are sorted by degree (std::sort, ascending) as a block.
#include <algorithm>
#include <deque>
#include <thread>
#include <vector>

#include "internal.h"

namespace db2 {
namespace {

// Neighbour lists of the node graph in dolfin::Set insertion order.  For a
// node i, pairs (i, j) are inserted cell by cell, in ascending cell order
// over the cells containing i, j in the cell's local order -- so the first
// occurrence order follows from i's incident cells alone.
void node_graph(const Space& V, std::vector<int64_t>& ptr, std::vector<int32_t>& adj) {
  const int64_t nn = V.nnodes, nc = V.mesh->nc;
  const int k = V.k;
  std::vector<int64_t> ip(nn + 1, 0);
  for (uint32_t n : V.cell_nodes) ip[n + 1]++;
  for (int64_t i = 0; i < nn; ++i) ip[i + 1] += ip[i];
  std::vector<int32_t> icell(ip[nn]);
  {
    std::vector<int64_t> fill(ip.begin(), ip.end() - 1);
    for (int64_t c = 0; c < nc; ++c)
      for (int a = 0; a < k; ++a) icell[fill[V.cell_nodes[c * k + a]]++] = int32_t(c);
  }
  std::vector<int32_t> deg(nn, 0);
  std::vector<std::vector<int32_t>> parts;
  const int nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  const int64_t chunk = (nn + nt - 1) / nt;
  std::vector<std::vector<int32_t>> lists(nt);
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t)
    th.emplace_back([&, t] {
      std::vector<uint8_t> mark(nn, 0);
      const int64_t b = t * chunk, e = std::min(nn, b + chunk);
      std::vector<int32_t>& out = lists[t];
      for (int64_t i = b; i < e; ++i) {
        const size_t start = out.size();
        for (int64_t s = ip[i]; s < ip[i + 1]; ++s) {
          const uint32_t* cn = &V.cell_nodes[int64_t(icell[s]) * k];
          for (int a = 0; a < k; ++a) {
            const uint32_t j = cn[a];
            if (j == uint32_t(i) || mark[j]) continue;
            mark[j] = 1;
            out.push_back(int32_t(j));
          }
        }
        for (size_t q = start; q < out.size(); ++q) mark[out[q]] = 0;
        deg[i] = int32_t(out.size() - start);
      }
    });
  for (auto& x : th) x.join();
  ptr.assign(nn + 1, 0);
  for (int64_t i = 0; i < nn; ++i) ptr[i + 1] = ptr[i] + deg[i];
  adj.resize(ptr[nn]);
  for (int t = 0; t < nt; ++t) {
    const int64_t b = t * chunk;
    if (b < nn) std::copy(lists[t].begin(), lists[t].end(), adj.begin() + ptr[b]);
  }
}

}  // namespace

std::vector<int32_t> rcm_node_order(const Space& V) {
  std::vector<int64_t> ptr;
  std::vector<int32_t> adj;
  node_graph(V, ptr, adj);
  const int64_t n = V.nnodes;
  auto degree = [&](int32_t v) { return ptr[v + 1] - ptr[v]; };
  std::vector<int32_t> remap(n);
  if (adj.empty()) {
    for (int64_t i = 0; i < n; ++i) remap[i] = int32_t(i);
    return remap;
  }
  enum : uint8_t { WHITE = 0, GRAY = 1, BLACK = 2 };
  std::vector<uint8_t> color(n, WHITE);
  // one vertex per connected component: first unvisited in index order
  std::vector<int32_t> starts;
  {
    std::vector<int32_t> stack;
    for (int64_t v = 0; v < n; ++v) {
      if (color[v] != WHITE) continue;
      starts.push_back(int32_t(v));
      stack.push_back(int32_t(v));
      color[v] = BLACK;
      while (!stack.empty()) {
        const int32_t u = stack.back();
        stack.pop_back();
        for (int64_t e = ptr[u]; e < ptr[u + 1]; ++e)
          if (color[adj[e]] == WHITE) {
            color[adj[e]] = BLACK;
            stack.push_back(adj[e]);
          }
      }
    }
  }
  // BFS from u over the component (colors reset to white first); returns the
  // eccentricity of u and the minimum-degree vertex of the last level
  // (first encountered on ties).
  std::vector<int32_t> queue(n);
  std::vector<uint8_t> seen(n, 0);
  std::vector<int32_t> touched;
  auto peripheral_pair = [&](int32_t u, int& ecc) {
    for (int32_t t : touched) seen[t] = 0;
    touched.clear();
    int64_t head = 0, tail = 0;
    queue[tail++] = u;
    seen[u] = 1;
    touched.push_back(u);
    ecc = -1;
    int32_t w = u;
    while (head < tail) {
      const int64_t level_end = tail;
      ++ecc;
      bool first = true;
      for (; head < level_end; ++head) {
        const int32_t x = queue[head];
        if (first || degree(x) < degree(w)) w = x;
        first = false;
        for (int64_t e = ptr[x]; e < ptr[x + 1]; ++e) {
          const int32_t y = adj[e];
          if (!seen[y]) {
            seen[y] = 1;
            touched.push_back(y);
            queue[tail++] = y;
          }
        }
      }
    }
    return w;
  };
  for (int32_t& r : starts) {
    int er = 0, ex = 0;
    int32_t x = peripheral_pair(r, er);
    int32_t y = peripheral_pair(x, ex);
    while (ex > er) {
      r = x;
      er = ex;
      x = y;
      y = peripheral_pair(x, ex);
    }
    r = x;
  }
  // Cuthill-McKee BFS; children of each vertex sorted by degree as a block
  std::fill(color.begin(), color.end(), WHITE);
  std::deque<int32_t> Q;
  std::vector<int32_t> order;
  order.reserve(n);
  auto less_degree = [&](int32_t a, int32_t b) { return degree(a) < degree(b); };
  for (int32_t s : starts) {
    if (color[s] != WHITE) continue;
    color[s] = GRAY;
    Q.push_back(s);
    while (!Q.empty()) {
      const int32_t u = Q.front();
      Q.pop_front();
      order.push_back(u);
      const size_t begin = Q.size();
      for (int64_t e = ptr[u]; e < ptr[u + 1]; ++e) {
        const int32_t v = adj[e];
        if (color[v] == WHITE) {
          color[v] = GRAY;
          Q.push_back(v);
        }
      }
      color[u] = BLACK;
      // Tie rule: the same call on the same sequence (a std::deque block in
      // Set insertion order) as Boost, so equal degrees end where libstdc++'s
      // std::sort leaves them.  For blocks of at most 16 nodes (every block
      // of the unit square and cube meshes, P1 and P2, started from a
      // pseudo-peripheral node) that sort is an insertion sort, which is
      // stable: ties stay in Set insertion order, whatever the library's
      // introsort would do with longer blocks.
      std::sort(Q.begin() + begin, Q.end(), less_degree);
    }
  }
  // reversed: the k-th visited vertex gets number n-1-k
  for (int64_t i = 0; i < n; ++i) remap[order[i]] = int32_t(n - 1 - i);
  return remap;
}

// The reordered CSR of a pattern on a reordered space: row i (new dof) is the
// natural row of the same dof with its columns renumbered and sorted;
// val_src / dof_src index the natural arrays.
void build_reordered_csr(Pattern& P) {
  const Space& V = *P.V;
  const int64_t N = V.dim();
  const int bs = V.vsize;
  std::vector<int32_t> nat_rowptr(N + 1), nat_cols(P.nnz);
  P.csr_host_natural(nat_rowptr.data(), nat_cols.data());
  auto new_of_nat = [&](int64_t d) {  // natural dof c*nn + node -> bs*remap[node] + c
    const int64_t c = d / V.nnodes, node = d - c * V.nnodes;
    return int64_t(bs) * V.node_new[node] + c;
  };
  ReorderedCSR& R = P.reordered;
  R.dof_src.assign(N, 0);
  for (int64_t d = 0; d < N; ++d) R.dof_src[new_of_nat(d)] = int32_t(d);
  R.rowptr.assign(N + 1, 0);
  for (int64_t i = 0; i < N; ++i) {
    const int64_t d = R.dof_src[i];
    R.rowptr[i + 1] = R.rowptr[i] + (nat_rowptr[d + 1] - nat_rowptr[d]);
  }
  R.cols.assign(P.nnz, 0);
  R.val_src.assign(P.nnz, 0);
  std::vector<std::pair<int32_t, int32_t>> tmp;
  for (int64_t i = 0; i < N; ++i) {
    const int64_t d = R.dof_src[i];
    tmp.clear();
    for (int32_t q = nat_rowptr[d]; q < nat_rowptr[d + 1]; ++q)
      tmp.emplace_back(int32_t(new_of_nat(nat_cols[q])), q);
    std::sort(tmp.begin(), tmp.end());
    for (size_t q = 0; q < tmp.size(); ++q) {
      R.cols[R.rowptr[i] + q] = tmp[q].first;
      R.val_src[R.rowptr[i] + q] = tmp[q].second;
    }
  }
  R.built = true;
}

}  // namespace db2
