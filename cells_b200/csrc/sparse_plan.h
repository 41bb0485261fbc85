// sparse_plan.h - the host plan of a sparse Cholesky factor, shared by the N2 operator
// (n2_step.cu) and the resolved field's node-space Laplacian (field_step.cu).
//
// Restates numerics/sparse_cholesky.py's bind (:137-215): an elimination order (minimum degree:
// least current degree, ties by the least original degree, then the smallest index; the
// eliminated node's neighbours form a clique; or an order the caller supplies), the filled
// pattern by the elimination tree's union rule, the tree's levels, each column's update list and
// the relative positions of its update terms (left-looking, so a column's updates need no
// atomics), and each edge's off-diagonal entry.
#pragma once

#include <algorithm>
#include <queue>
#include <set>
#include <tuple>
#include <vector>

#include "handle.h"

namespace cbk {

struct WorldPlan {
  std::vector<int> order, rank, colp, lrow, uk_ptr, uk_col, uk_pos, uk_rel, rel, level_cols,
      level_ptr, edge_pos;
};

// n nodes, ne edges (snd[e], rcv[e]); order (optional) a permutation giving the elimination
// order, else minimum degree. who names the caller in the refusal messages.
inline int plan_world(int n, const int *snd, const int *rcv, int ne, WorldPlan &p,
                      const int *order = nullptr, const char *who = "N2") {
  std::vector<std::set<int>> adj(n);
  for (int e = 0; e < ne; ++e) {
    const int a = snd[e], b = rcv[e];
    if (a == b) return fail(CB_ERR_LAYOUT, std::string(who) + ": an edge joins a node to itself");
    if (!adj[a].insert(b).second)
      return fail(CB_ERR_LAYOUT, std::string(who) + ": two edges join the same pair");
    adj[b].insert(a);
  }
  if (order) {
    p.order.assign(order, order + n);
  } else {
    // Minimum degree.
    std::vector<int> original(n);
    for (int i = 0; i < n; ++i) original[i] = (int)adj[i].size();
    std::vector<std::set<int>> g = adj;
    using Key = std::tuple<int, int, int>;
    std::priority_queue<Key, std::vector<Key>, std::greater<Key>> heap;
    for (int i = 0; i < n; ++i) heap.push(Key(original[i], original[i], i));
    std::vector<char> alive(n, 1);
    p.order.clear();
    while (!heap.empty()) {
      const auto [degree, orig, node] = heap.top();
      heap.pop();
      if (!alive[node] || degree != (int)g[node].size()) continue;
      alive[node] = 0;
      p.order.push_back(node);
      const std::set<int> nb = g[node];
      for (int a : nb) {
        g[a].erase(node);
        for (int b : nb)
          if (b != a) g[a].insert(b);
        heap.push(Key((int)g[a].size(), original[a], a));
      }
      g[node].clear();
    }
  }
  p.rank.assign(n, 0);
  for (int r = 0; r < n; ++r) p.rank[p.order[r]] = r;
  // Symbolic factorisation (union rule) and the elimination tree.
  std::vector<std::set<int>> below(n);
  for (int i = 0; i < n; ++i) {
    const int r = p.rank[i];
    for (int a : adj[i])
      if (p.rank[a] > r) below[r].insert(p.rank[a]);
  }
  std::vector<int> parent(n, -1), level(n, 0);
  for (int kk = 0; kk < n; ++kk) {
    if (!below[kk].empty()) {
      const int par = *below[kk].begin();
      parent[kk] = par;
      for (int r : below[kk])
        if (r != par) below[par].insert(r);
    }
  }
  for (int kk = 0; kk < n; ++kk)
    if (parent[kk] >= 0) level[parent[kk]] = std::max(level[parent[kk]], level[kk] + 1);
  p.colp.assign(n + 1, 0);
  for (int kk = 0; kk < n; ++kk) p.colp[kk + 1] = p.colp[kk] + 1 + (int)below[kk].size();
  p.lrow.assign(p.colp[n], 0);
  for (int kk = 0; kk < n; ++kk) {
    int f = p.colp[kk];
    p.lrow[f++] = kk;
    for (int r : below[kk]) p.lrow[f++] = r;
  }
  // Update lists: for column j, every k < j whose column holds row j, ascending k; the
  // relative positions in column j of column k's rows at or below j.
  std::vector<std::vector<std::pair<int, int>>> rowlist(n);  // j -> (k, entry of L_jk)
  for (int kk = 0; kk < n; ++kk)
    for (int f = p.colp[kk] + 1; f < p.colp[kk + 1]; ++f) rowlist[p.lrow[f]].push_back({kk, f});
  std::vector<int> where(n, -1);
  p.uk_ptr.assign(n + 1, 0);
  p.uk_col.clear();
  p.uk_pos.clear();
  p.uk_rel.clear();
  p.rel.clear();
  for (int j = 0; j < n; ++j) {
    for (int f = p.colp[j]; f < p.colp[j + 1]; ++f) where[p.lrow[f]] = f - p.colp[j];
    for (const auto &[kk, f] : rowlist[j]) {
      p.uk_col.push_back(kk);
      p.uk_pos.push_back(f);
      p.uk_rel.push_back((int)p.rel.size());
      for (int t = f; t < p.colp[kk + 1]; ++t) {
        const int off = where[p.lrow[t]];
        if (off < 0) return fail(CB_ERR_LAYOUT, std::string(who) + ": inconsistent factor pattern");
        p.rel.push_back(off);
      }
    }
    for (int f = p.colp[j]; f < p.colp[j + 1]; ++f) where[p.lrow[f]] = -1;
    p.uk_ptr[j + 1] = (int)p.uk_col.size();
  }
  // Levels.
  const int levels = n ? 1 + *std::max_element(level.begin(), level.end()) : 0;
  p.level_ptr.assign(levels + 1, 0);
  for (int kk = 0; kk < n; ++kk) p.level_ptr[level[kk] + 1]++;
  for (int l = 0; l < levels; ++l) p.level_ptr[l + 1] += p.level_ptr[l];
  p.level_cols.assign(n, 0);
  std::vector<int> fill(p.level_ptr.begin(), p.level_ptr.end() - 1);
  for (int kk = 0; kk < n; ++kk) p.level_cols[fill[level[kk]]++] = kk;
  // Junctions' off-diagonal entries (row = the later rank, column = the earlier).
  p.edge_pos.assign(ne, 0);
  for (int e = 0; e < ne; ++e) {
    const int ra = p.rank[snd[e]], rb = p.rank[rcv[e]];
    const int col = std::min(ra, rb), row = std::max(ra, rb);
    int found = -1;
    for (int f = p.colp[col]; f < p.colp[col + 1]; ++f)
      if (p.lrow[f] == row) found = f;
    if (found < 0) return fail(CB_ERR_LAYOUT, std::string(who) + ": edge outside the factor pattern");
    p.edge_pos[e] = found;
  }
  return CB_OK;
}

}  // namespace cbk
