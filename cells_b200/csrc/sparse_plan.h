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

// Supernodes of a plan's factor (the multifrontal form of its factorisation): column j joins the
// supernode of column j - 1 when j - 1 is j's only child and struct(j - 1) = {j - 1} + struct(j), so a
// supernode's columns share one dense front: rows c0 .. c1 - 1 (its columns) then its boundary B
// (rows of later supernodes). Each front is factored densely (its s x s diagonal block, the b x s
// block below), leaving the update matrix B x B for its parent; the parent adds its children's
// update matrices into its own front (extend-add) in ascending child order. Levels: a
// supernode's level is one above its highest child's.
struct SuperPlan {
  int count = 0, levels = 0;
  std::vector<int> c0, s, m;                // first column, columns, front rows
  std::vector<long long> loff, uoff, voff;  // factor block (m x s), update matrix (packed
                                            // lower b x b), vector
  std::vector<int> rows_ptr, rows;          // each front's rows (factor columns, ascending)
  std::vector<int> ch_ptr, ch;              // each supernode's children, ascending
  std::vector<int> map_ptr, map;            // a child's boundary rows' positions in its parent
  std::vector<int> split;                   // a child's boundary rows that fall in its parent's
                                            // columns (the first `split`, as its map ascends)
  std::vector<int> parent;                  // -1 at a root
  std::vector<int> lv_ptr, lv_sn;           // supernodes level by level
  std::vector<int> sn_of;                   // column -> supernode
  long long lsize = 0, usize = 0, vsize = 0;
  long long max_block = 0;                  // largest m x s
  int max_m = 0;
};

// group (optional, by column): consecutive columns with the same non-negative id form one
// supernode (a relaxed supernode: a connected subtree of the elimination tree, its front rows the
// union of its columns' structures, its diagonal block dense); columns with id -1 follow the
// fundamental rule.
inline int build_supernodes(const WorldPlan &p, SuperPlan &sp,
                            const std::vector<int> *group = nullptr) {
  const int n = (int)p.colp.size() - 1;
  auto len = [&](int j) { return p.colp[j + 1] - p.colp[j]; };
  auto par = [&](int j) { return len(j) > 1 ? p.lrow[p.colp[j] + 1] : -1; };
  sp = SuperPlan();
  sp.sn_of.assign(n, -1);
  std::vector<int> children(n, 0);
  for (int j = 0; j < n; ++j)
    if (par(j) >= 0) children[par(j)]++;
  for (int j = 0; j < n; ++j) {
    // fundamental supernodes: j - 1 is j's only child
    bool join = j > 0 && par(j - 1) == j && children[j] == 1 && len(j - 1) == len(j) + 1;
    if (group) {
      const int gj = (*group)[j], gp = j > 0 ? (*group)[j - 1] : -2;
      if (gj >= 0 || gp >= 0) join = j > 0 && gj >= 0 && gj == gp;
    }
    if (!join) {
      sp.c0.push_back(j);
      sp.s.push_back(0);
    }
    sp.s.back() += 1;
    sp.sn_of[j] = (int)sp.c0.size() - 1;
  }
  const int S = sp.count = (int)sp.c0.size();
  sp.m.resize(S);
  sp.parent.assign(S, -1);
  sp.rows_ptr.assign(S + 1, 0);
  for (int q = 0; q < S; ++q) {
    const int c = sp.c0[q], c1 = c + sp.s[q];
    // Rows: the supernode's columns, then the union of its columns' rows beyond it.
    std::set<int> beyond;
    for (int k = c; k < c1; ++k)
      for (int t = p.colp[k]; t < p.colp[k + 1]; ++t)
        if (p.lrow[t] >= c1) beyond.insert(p.lrow[t]);
    for (int k = c; k < c1; ++k) sp.rows.push_back(k);
    sp.rows.insert(sp.rows.end(), beyond.begin(), beyond.end());
    sp.rows_ptr[q + 1] = (int)sp.rows.size();
    sp.m[q] = sp.rows_ptr[q + 1] - sp.rows_ptr[q];
    if (!beyond.empty()) sp.parent[q] = sp.sn_of[*beyond.begin()];
    for (int k = c; k < c1; ++k)  // a relaxed supernode must be one subtree
      if (par(k) >= 0 && par(k) >= c1 && par(k) != *beyond.begin())
        return fail(CB_ERR_LAYOUT, "supernodes: a group is not one subtree");
    // the supernode's columns are its first rows
    for (int k = 0; k < sp.s[q]; ++k)
      if (sp.rows[sp.rows_ptr[q] + k] != c + k)
        return fail(CB_ERR_LAYOUT, "supernodes: inconsistent front rows");
  }
  std::vector<std::vector<int>> kids(S);
  for (int q = 0; q < S; ++q)
    if (sp.parent[q] >= 0) kids[sp.parent[q]].push_back(q);
  sp.ch_ptr.assign(S + 1, 0);
  for (int q = 0; q < S; ++q) {
    sp.ch.insert(sp.ch.end(), kids[q].begin(), kids[q].end());
    sp.ch_ptr[q + 1] = (int)sp.ch.size();
  }
  sp.map_ptr.assign(S + 1, 0);
  for (int q = 0; q < S; ++q) {
    const int b = sp.m[q] - sp.s[q];
    if (sp.parent[q] >= 0) {
      const int pq = sp.parent[q];
      const int *pr = sp.rows.data() + sp.rows_ptr[pq];
      const int pm = sp.m[pq];
      for (int i = 0; i < b; ++i) {
        const int r = sp.rows[sp.rows_ptr[q] + sp.s[q] + i];
        const int *at = std::lower_bound(pr, pr + pm, r);
        if (at == pr + pm || *at != r)
          return fail(CB_ERR_LAYOUT, "supernodes: a boundary row is not in the parent's front");
        sp.map.push_back((int)(at - pr));
      }
    } else if (b != 0) {
      return fail(CB_ERR_LAYOUT, "supernodes: a root front has boundary rows");
    }
    sp.map_ptr[q + 1] = (int)sp.map.size();
  }
  sp.split.assign(S, 0);
  for (int q = 0; q < S; ++q)
    if (sp.parent[q] >= 0)
      for (int t = sp.map_ptr[q]; t < sp.map_ptr[q + 1]; ++t)
        if (sp.map[t] < sp.s[sp.parent[q]]) sp.split[q]++;
  // Levels (children precede parents: supernodes are numbered in column order).
  std::vector<int> level(S, 0);
  for (int q = 0; q < S; ++q)
    if (sp.parent[q] >= 0) level[sp.parent[q]] = std::max(level[sp.parent[q]], level[q] + 1);
  sp.levels = S ? 1 + *std::max_element(level.begin(), level.end()) : 0;
  sp.lv_ptr.assign(sp.levels + 1, 0);
  for (int q = 0; q < S; ++q) sp.lv_ptr[level[q] + 1]++;
  for (int l = 0; l < sp.levels; ++l) sp.lv_ptr[l + 1] += sp.lv_ptr[l];
  sp.lv_sn.assign(S, 0);
  std::vector<int> fill(sp.lv_ptr.begin(), sp.lv_ptr.end() - 1);
  for (int q = 0; q < S; ++q) sp.lv_sn[fill[level[q]]++] = q;
  sp.loff.resize(S);
  sp.uoff.resize(S);
  sp.voff.resize(S);
  for (int q = 0; q < S; ++q) {
    const long long mm = sp.m[q], ss = sp.s[q], b = mm - ss;
    sp.loff[q] = sp.lsize;
    sp.lsize += (mm * ss + 1) & ~1LL;  // even: every block 16-byte aligned, its copy padded
    sp.uoff[q] = sp.usize;
    sp.usize += b * (b + 1) / 2;  // the update matrix's lower triangle, packed by columns
    sp.voff[q] = sp.vsize;
    sp.vsize += b;
    sp.max_block = std::max(sp.max_block, mm * ss);
    sp.max_m = std::max(sp.max_m, (int)mm);
  }
  return CB_OK;
}

// Relaxed amalgamation of a supernode plan: a supernode q whose columns end where its parent p's
// begin joins p when the zeros the merge adds to q's columns (s_q (s_q + m_p - m_q) entries: p's
// rows that q's own structure lacks) are at most `frac` of the merged front block and that block
// stays within `cap` entries; repeated until nothing merges. On a nested-dissection grid plan the
// single-column fronts where two separators cross each become a level of their own; merged into
// the separator above, they leave fewer, larger fronts: fewer levels (level-synchronous launches)
// and update matrices for a few percent more factor entries and flops.
inline int amalgamate(const WorldPlan &p, SuperPlan &sp, double frac, long long cap) {
  const int n = (int)p.colp.size() - 1;
  std::vector<int> group(n);
  for (int pass = 0; pass < 64; ++pass) {
    std::vector<int> target(sp.count);
    for (int q = 0; q < sp.count; ++q) target[q] = q;
    int merges = 0;
    for (int q = sp.count - 1; q >= 0; --q) {
      const int pq = sp.parent[q];
      if (pq < 0 || sp.c0[q] + sp.s[q] != sp.c0[pq] || target[pq] != pq) continue;
      const long long extra = (long long)sp.s[q] * (sp.s[q] + sp.m[pq] - sp.m[q]);
      const long long merged = (long long)(sp.s[q] + sp.m[pq]) * (sp.s[q] + sp.s[pq]);
      if (extra > frac * (double)merged || merged > cap) continue;
      target[q] = pq;
      ++merges;
    }
    if (!merges) return CB_OK;
    for (int q = 0; q < sp.count; ++q) {
      int t = q;
      while (target[t] != t) t = target[t];
      for (int k = 0; k < sp.s[q]; ++k) group[sp.c0[q] + k] = t;
    }
    SuperPlan merged;
    if (int rc = build_supernodes(p, merged, &group)) return rc;
    sp = std::move(merged);
  }
  return CB_OK;
}

}  // namespace cbk
