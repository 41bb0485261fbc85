// n2_common.cuh - the per-world sparse Cholesky shared by the N2 and ROS2 steps (n2_step.cu)
// and the ROS2 step's reverse (ros2_adjoint.cu): the device plan arrays, the route slope
// conductance, and the one-CTA-per-world left-looking factor and level-scheduled substitutions.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "handle.h"

namespace cbk {

struct N2Dev {
  // World-local plan arrays; world w's entries start at the bases below.
  int *rank;      // [C] each cell's position (its minimum-degree rank in its world)
  int *colp;      // [C+W] per world n+1 first factor entries of its columns (world w at c0 + w)
  int *lrow;      // [F] each factor entry's row
  int *uk_ptr;    // [C+W] per world n+1: column j's update list (the k < j with L_jk != 0)
  int *uk_col;    // [U] k
  int *uk_pos;    // [U] the factor entry of L_jk
  int *uk_rel;    // [U] offset into rel of the pair's relative positions
  int *rel;       // [R] each entry of column k at or below row j -> its offset in column j
  int *lv_ptr;    // [levels+W] per world L+1 first columns of its levels (world w at lb[w] + w)
  int *lv_cols;   // [C] columns level by level (world w at c0)
  int *edge_pos;  // [E] each junction's off-diagonal factor entry
  int *fb, *ub, *rb, *lb;  // [W+1] bases: factor entries, update terms, rel, levels
  double *lval;   // [F] factor values (global mode)
  double *cs;     // cell scratch [NC_FIELDS][C]
  double *es;     // junction scratch [NE_FIELDS][E]
};

struct N2Plan {
  N2Dev d{};
  std::vector<void *> owned;
  long long factor_entries = 0, update_terms = 0;
  int levels = 0, max_level = 0;
  size_t smem_bytes = 0;  // dynamic shared memory per CTA (worlds that fit stage into it)
  int block = 256;        // CTA threads (256, or 128 for small worlds)
  int ros2_block = 256;   // the ROS2/RK4 kernel's CTA threads: 128 (four CTAs per SM) when no
                          // world's plan is staged in shared memory, else 256 (two)
  size_t smem_f32 = 0;    // the same staging with FP32 factor values (CB_METHOD_ROS2_MIXED)
  int ros2_block_f32 = 256;
  int min_blocks = 2;     // the register budget's target CTAs per SM (2: capped at 128
                          // registers, measured fastest on 16x16 grids; 1: uncapped)
};

// The ROS2 forward's record of one step for the reverse (ros2_adjoint.cu), world-packed as the
// state: the factor of the step's voltage operator (world w's entries from fb[w]), its Jacobi
// scale, the two stage solves' voltage rates, k1's dynamic rows and k2's gate rows. A null factor
// pointer records nothing.
struct R2Tape {
  double *factor;  // [F]
  double *scale;   // [C]
  double *u;       // [2][C]
  double *k1n;     // [3][C]
  double *k1gc;    // [2 NCH][C], row r of slot q at (r NCH + q) C
  double *k1g;     // [E]
  double *k2gc;    // [2 NCH][C]
  double *k2g;     // [E]
};

}  // namespace cbk

namespace {

using namespace cbk;

// B'(x), the reference's form (patch_electrodiffusion.bernoulli_slope): the series
// -1/2 + x/6 - x^3/180 below |x| < 1e-3, otherwise with em = e^-|x|:
// x > 0: (em (1 - x) - em^2) / (1 - em)^2; x < 0: (em - 1 - x em) / (em - 1)^2.
__device__ __forceinline__ double ref_bernoulli_slope(double x) {
  if (fabs(x) < 1e-3) return (-0.5 + x / 6.0) - ((x * x) * x) / 180.0;
  const double em = exp(-fabs(x));
  if (x > 0.0) {
    const double d = 1.0 - em;
    return (em * (1.0 - x) - em * em) / (d * d);
  }
  const double d = em - 1.0;
  return ((em - 1.0) - x * em) / (d * d);
}

// dJ/d(dv) of a route with prefactor g (fmol/s per mM) between c_from and c_to, valence z.
__device__ __forceinline__ double route_slope(double g, double c_from, double c_to, double dv,
                                              double zfrt) {
  const double x = zfrt * dv;
  return g * zfrt * (-c_from * ref_bernoulli_slope(-x) - c_to * ref_bernoulli_slope(x));
}

// The dense tail of a world's plan: the longest end of its final run of one-column levels (the
// top separator's chain) whose columns are the plan's last t columns n - t .. n - 1 in order, each
// dense below its diagonal. Returns t (0 when shorter than 2).
__device__ inline int dense_tail(const int *colp, const int *lvp, const int *lvc, int lv0, int lv1,
                                 int n) {
  int t = 0;
  for (int l = lv1 - 1; l >= lv0 && lvp[l + 1] - lvp[l] == 1; --l) {
    const int j = lvc[lvp[l]];
    if (j != n - 1 - t || colp[j + 1] - colp[j] != n - j) break;
    ++t;
  }
  return t >= 2 ? t : 0;
}

// One world's sparse Cholesky on its plan (local indices; values and vectors by position), as one
// CTA of BLOCK threads runs it: left-looking factor by levels of the elimination tree, a warp per
// column (update terms in ascending k, each term's rows at precomputed offsets in the column,
// so no atomics); a run of one-column levels (the top separator's chain) by warp 0 alone with
// warp syncs only, except a dense tail (dense_tail), whose columns' updates from the columns
// before it go one column per warp and whose own block is factored right-looking by the CTA;
// forward and back substitution of L L^T x = b (b in Yv, x to Xv), a thread per column on wide
// levels, a warp per column with the dot products across its lanes (a fixed xor tree) on narrow
// levels and on the runs. Each factor entry sees the same operations in the same order in every
// form.
template <typename FT, int BLOCK>
struct WorldCholesky {
  const int *colp, *lrow, *ukp, *ukc, *ukpos, *ukrel, *rel, *lvp, *lvc;
  FT *lval, *Yv, *Xv;
  int lv0, lv1;
  int n, tail;  // the world's columns; its dense tail's length (0: none)

  // Update terms u0 .. u1 of the column at cj (ascending k), those with k below klim, in order:
  // lanes over a term's rows, a warp sync between terms. While a term's rows are written, the
  // next term's multiplier, length and first 32 rows (their offsets in column j and their values)
  // are read, and the indices of the term after it: all lie in finished columns, so each term
  // waits on one round of loads, not on the index loads and the loads they address in turn.
  __device__ void apply_updates(int cj, int u0, int u1, int klim, int lane) const {
    if (u0 >= u1 || ukc[u0] >= klim) return;
    int p = ukpos[u0], r0 = ukrel[u0];
    int cnt = colp[ukc[u0] + 1] - p;
    FT ljk = lval[p];
    int off = lane < cnt ? rel[r0 + lane] : 0;
    FT src = lane < cnt ? lval[p + lane] : FT(0);
    bool m1 = u0 + 1 < u1;
    int k1 = 0, p1 = 0, r1 = 0;
    if (m1) {
      k1 = ukc[u0 + 1];
      p1 = ukpos[u0 + 1];
      r1 = ukrel[u0 + 1];
      m1 = k1 < klim;
    }
    for (int u = u0;; ++u) {
      int ncnt = 0, noff = 0;
      FT nl = 0, nsrc = 0;
      if (m1) {
        ncnt = colp[k1 + 1] - p1;
        nl = lval[p1];
        if (lane < ncnt) {
          noff = rel[r1 + lane];
          nsrc = lval[p1 + lane];
        }
      }
      bool m2 = m1 && u + 2 < u1;
      int k2 = 0, p2 = 0, r2 = 0;
      if (m2) {
        k2 = ukc[u + 2];
        p2 = ukpos[u + 2];
        r2 = ukrel[u + 2];
        m2 = k2 < klim;
      }
      if (lane < cnt) lval[cj + off] -= src * ljk;
      for (int t = lane + 32; t < cnt; t += 32) lval[cj + rel[r0 + t]] -= lval[p + t] * ljk;
      __syncwarp();
      if (!m1) break;
      p = p1;
      r0 = r1;
      cnt = ncnt;
      ljk = nl;
      off = noff;
      src = nsrc;
      m1 = m2;
      k1 = k2;
      p1 = p2;
      r1 = r2;
    }
  }
  __device__ uint32_t factor_column(int j, int lane) const {
    uint32_t bad = 0;
    const int cj = colp[j];
    apply_updates(cj, ukp[j], ukp[j + 1], j, lane);
    FT piv = 0;
    if (lane == 0) {
      const FT d = lval[cj];
      if (!(d > 0.0) || !is_finite(d)) bad = 1u;
      piv = sqrt(d);
      lval[cj] = piv;
    }
    piv = __shfl_sync(0xffffffffu, piv, 0);
    const FT inv = FT(1) / piv;
    const int len = colp[j + 1] - cj;
    for (int t = 1 + lane; t < len; t += 32) lval[cj + t] *= inv;
    __syncwarp();
    return bad;
  }
  // The end of the run of one-column levels starting at lv (uniform across the CTA).
  __device__ int single_run_end(int lv) const {
    int end = lv;
    while (end < lv1 && lvp[end + 1] - lvp[end] == 1) ++end;
    return end;
  }
  // The dense tail j0 .. n - 1: first each tail column's updates from the columns before the
  // tail (ascending k, as factor_column takes them), warps over the tail's columns, which touch
  // only their own column; then the tail block right-looking, a column at a time: warp 0 takes
  // the pivot and scales the column, the warps take its products out of the later columns (each
  // entry's updates still in ascending k, the same products as factor_column's).
  __device__ uint32_t factor_tail(int j0) const {
    constexpr int WARPS = BLOCK / 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t bad = 0;
    for (int j = j0 + warp; j < n; j += WARPS) apply_updates(colp[j], ukp[j], ukp[j + 1], j0, lane);
    __syncthreads();
    for (int j = j0; j < n; ++j) {
      const int cj = colp[j], len = n - j;
      if (warp == 0) {
        FT piv = 0;
        if (lane == 0) {
          const FT d = lval[cj];
          if (!(d > 0.0) || !is_finite(d)) bad = 1u;
          piv = sqrt(d);
          lval[cj] = piv;
        }
        piv = __shfl_sync(0xffffffffu, piv, 0);
        const FT inv = FT(1) / piv;
        for (int t = 1 + lane; t < len; t += 32) lval[cj + t] *= inv;
      }
      __syncthreads();
      for (int jj = j + 1 + warp; jj < n; jj += WARPS) {
        const FT l = lval[cj + (jj - j)];
        const int cjj = colp[jj];
        for (int r = jj + lane; r < n; r += 32) lval[cjj + (r - jj)] -= lval[cj + (r - j)] * l;
      }
      __syncthreads();
    }
    return bad;
  }
  __device__ uint32_t factor() const {
    constexpr int WARPS = BLOCK / 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t bad = 0;
    for (int lv = lv0; lv < lv1;) {
      const int a0 = lvp[lv], a1 = lvp[lv + 1];
      if (a1 - a0 == 1) {
        const int end = single_run_end(lv);
        if (tail > 0 && end == lv1) {  // the final run: its head by warp 0, then the dense tail
          const int head = end - tail;
          if (warp == 0)
            for (int l = lv; l < head; ++l) bad |= factor_column(lvc[lvp[l]], lane);
          __syncthreads();
          bad |= factor_tail(lvc[lvp[head]]);
          lv = end;
          continue;
        }
        if (warp == 0)
          for (int l = lv; l < end; ++l) bad |= factor_column(lvc[lvp[l]], lane);
        lv = end;
      } else {
        for (int a = a0 + warp; a < a1; a += WARPS) bad |= factor_column(lvc[a], lane);
        ++lv;
      }
      __syncthreads();
    }
    return bad;
  }
  __device__ static FT warp_sum(FT v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
  }
  __device__ void solve() const {
    constexpr int WARPS = BLOCK / 32;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int lv = lv0; lv < lv1;) {
      const int a0 = lvp[lv], a1 = lvp[lv + 1];
      if (a1 - a0 == 1) {
        const int end = single_run_end(lv);
        if (warp == 0) {
          // A chain of columns, each after the last: the next column's term indices, factor
          // entries and pivot are read while this one's dot product completes.
          int j = lvc[lvp[lv]], ue = ukp[j + 1], u0 = ukp[j] + lane;
          int col = u0 < ue ? ukc[u0] : 0;
          FT val = u0 < ue ? lval[ukpos[u0]] : FT(0), piv = lval[colp[j]];
          for (int l = lv; l < end; ++l) {
            int jn = 0, uen = 0, u0n = 0, coln = 0;
            FT valn = 0, pivn = 0;
            if (l + 1 < end) {
              jn = lvc[lvp[l + 1]];
              uen = ukp[jn + 1];
              u0n = ukp[jn] + lane;
              if (u0n < uen) {
                coln = ukc[u0n];
                valn = lval[ukpos[u0n]];
              }
              pivn = lval[colp[jn]];
            }
            FT part = 0;
            if (u0 < ue) part += val * Yv[col];
            for (int u = u0 + 32; u < ue; u += 32) part += lval[ukpos[u]] * Yv[ukc[u]];
            part = warp_sum(part);
            if (lane == 0) Yv[j] = (Yv[j] - part) / piv;
            __syncwarp();
            j = jn;
            ue = uen;
            u0 = u0n;
            col = coln;
            val = valn;
            piv = pivn;
          }
        }
        lv = end;
      } else if (a1 - a0 <= 2 * WARPS) {  // a narrow level: a warp per column
        for (int a = a0 + warp; a < a1; a += WARPS) {
          const int j = lvc[a];
          FT part = 0;
          for (int u = ukp[j] + lane; u < ukp[j + 1]; u += 32)
            part += lval[ukpos[u]] * Yv[ukc[u]];
          part = warp_sum(part);
          if (lane == 0) Yv[j] = (Yv[j] - part) / lval[colp[j]];
        }
        ++lv;
      } else {
        for (int a = a0 + tid; a < a1; a += BLOCK) {
          const int j = lvc[a];
          FT b = Yv[j];
          for (int u = ukp[j]; u < ukp[j + 1]; ++u) b -= lval[ukpos[u]] * Yv[ukc[u]];
          Yv[j] = b / lval[colp[j]];
        }
        ++lv;
      }
      __syncthreads();
    }
    for (int lv = lv1 - 1; lv >= lv0;) {
      const int a0 = lvp[lv], a1 = lvp[lv + 1];
      if (a1 - a0 == 1) {
        int begin = lv;  // the run of one-column levels ending at lv
        while (begin > lv0 && lvp[begin] - lvp[begin - 1] == 1) --begin;
        if (warp == 0) {
          // The chain backwards, the next column's rows, entries and pivot read ahead.
          int j = lvc[lvp[lv]], cj = colp[j], len = colp[j + 1] - cj;
          int row = 1 + lane < len ? lrow[cj + 1 + lane] : 0;
          FT val = 1 + lane < len ? lval[cj + 1 + lane] : FT(0), piv = lval[cj];
          for (int l = lv; l >= begin; --l) {
            int jn = 0, cjn = 0, lenn = 0, rown = 0;
            FT valn = 0, pivn = 0;
            if (l - 1 >= begin) {
              jn = lvc[lvp[l - 1]];
              cjn = colp[jn];
              lenn = colp[jn + 1] - cjn;
              if (1 + lane < lenn) {
                rown = lrow[cjn + 1 + lane];
                valn = lval[cjn + 1 + lane];
              }
              pivn = lval[cjn];
            }
            FT part = 0;
            if (1 + lane < len) part += val * Xv[row];
            for (int t = 33 + lane; t < len; t += 32) part += lval[cj + t] * Xv[lrow[cj + t]];
            part = warp_sum(part);
            if (lane == 0) Xv[j] = (Yv[j] - part) / piv;
            __syncwarp();
            j = jn;
            cj = cjn;
            len = lenn;
            row = rown;
            val = valn;
            piv = pivn;
          }
        }
        lv = begin - 1;
      } else if (a1 - a0 <= 2 * WARPS) {  // a narrow level: a warp per column
        for (int a = a0 + warp; a < a1; a += WARPS) {
          const int j = lvc[a];
          const int cj = colp[j], len = colp[j + 1] - cj;
          FT part = 0;
          for (int t = 1 + lane; t < len; t += 32) part += lval[cj + t] * Xv[lrow[cj + t]];
          part = warp_sum(part);
          if (lane == 0) Xv[j] = (Yv[j] - part) / lval[cj];
        }
        --lv;
      } else {
        for (int a = a0 + tid; a < a1; a += BLOCK) {
          const int j = lvc[a];
          const int cj = colp[j], len = colp[j + 1] - cj;
          FT x = Yv[j];
          for (int t = 1; t < len; ++t) x -= lval[cj + t] * Xv[lrow[cj + t]];
          Xv[j] = x / lval[cj];
        }
        --lv;
      }
      __syncthreads();
    }
  }
};

}  // namespace
