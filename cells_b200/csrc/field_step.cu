// field_step.cu - the resolved-field step (cb_field_*): tissues whose cells face a resolved
// extracellular grid with held boundary nodes, ARS(2,2,2) with implicit face electromigration.
//
// Reference: models/surface_pump.py:158-369 (explicit_rates, implicit_rates, imex_step) with the
// field closure numerics/surface_field.py:253-855 (bind, _capacitor_solve, the damped Newton on
// the floating offsets) and the face operator numerics/surface_imex.py:123-278 (face_weights,
// drift_flux, face_laplacian, factor_operator, solve_operator); transport and logmean of
// numerics/surface_transport.py:298-386 and numerics/extracellular_field.py:48-62.
//
// Algebra. Each cell's one membrane faces a free outside node, so a cell and its node form one
// capacitor component and every other free node is a component of its own. Eliminating each cell
// into its node (C (phi_c - phi_m) = q_c) leaves, on the free nodes:
//   start field   currents balance: sum of face and junction currents out of each component = 0,
//                 with phi_c = phi_m + q_c / C_c. Face currents are affine in the potentials at
//                 the step start's concentrations; junction currents are the constant-field law.
//                 Solved as the reference's Newton (initial solve with the face conductances, then
//                 corrections with a backtracking line search and its acceptance: max residual
//                 down, or within NEWTON_TARGET of the current scale), with the face Laplacian as
//                 the Newton matrix throughout (a chord: the junction slopes, five orders below the
//                 face conductances, are left out of the matrix, not out of the residual).
//   stage solve   gamma dt L(W) phi = q_m + q_c on the free nodes, the held nodes' potentials on
//                 the right, W the face weights at the half-step prediction.
// Both matrices are the face conductance Laplacian of the free nodes: one sparse pattern for
// every world, ordered by nested dissection of the grid (or minimum degree for other graphs),
// factored left-looking by the elimination tree's levels (a warp per column).
//
// One CTA advances one world n_steps steps; its vectors, rates and factor live in a global scratch
// slice of its own.

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cells_b200.h"
#include "handle.h"
#include "sparse_plan.h"

namespace {

using namespace cbk;

constexpr double kNewtonTarget = 0.01;   // surface_field.NEWTON_TARGET
constexpr double kCurrentAtol = 1e-23;   // CURRENT_ATOL_A
constexpr double kCurrentRtol = 2e-12;   // CURRENT_RTOL
constexpr int kMaxIterations = 16;       // solve's max_iterations
constexpr int kMaxBacktracks = 12;       // max_backtracks
constexpr int kFieldBlock = 512;
constexpr int kPhaseMinBlocks = 2;  // phase CTAs per SM the register budget aims for
constexpr int kWarpBlock = 1280;  // a level's fronts go one per warp when their blocks fit this
constexpr int kWarpVector = 256;  // ... and their fronts' rows this
constexpr int kWideColumns = 48;  // a CTA level's fronts take the wide factor from this many columns
// Dynamic shared memory a level kernel may ask for: the 227 KB per CTA less room for its static
// shared memory.
constexpr long long kMaxSmemBytes = 227 * 1024 - 1024;
constexpr double kChargeAtol = 3e-25;    // surface_field.CHARGE_ATOL_C
constexpr double kChargeRtol = 2e-12;    // CHARGE_RTOL

enum FieldWorldConst {
  FW_T = 0, FW_RT, FW_FRT, FW_INVRT, FW_DRIVE, FW_LOGKMK, FW_LATP, FW_LOGKMNA, FW_AFF0,
  FW_PUMPOK, FW_INVRTD, FW_STRIDE
};

struct Topo {  // shared by every world
  int N, O, E, F, U, levels;
  const int *cell_node;  // [N]
  const int *ncell;      // [O] the cell facing the node, or -1
  const int *upos;       // [O] the node's unknown (factor column), or -1 when held
  const int *nf_ptr, *nf_idx;  // node -> faces, face order: f << 1 | (1 when the receiver)
  const int *cj_ptr, *cj_idx;  // cell -> junctions, edge order: e << 1 | (1 when the receiver)
  const int *fs, *fr;    // [F]
  const int *js, *jr;    // [E]
  const int *col_node;   // [U] each factor column's node
  // Supernodes (the multifrontal factor): first column, columns, front rows; offsets of each
  // front's factor block (m x s, column-major), update matrix (b x b) and update vector (b);
  // front rows; children; a child's boundary rows' positions in its parent's front; levels and
  // whether a level's fronts are small enough for one warp each; each front's face entries.
  const int *sn_c0, *sn_s, *sn_m;
  const long long *sn_loff, *sn_uoff, *sn_voff;
  const int *rows_ptr, *rows, *ch_ptr, *ch, *map_ptr, *map, *split, *lv_ptr, *lv_sn;
  const int *af_ptr, *af_face, *af_pos;
};
struct Params {  // per world, world-major
  const double *wc;      // [W][FW_STRIDE]
  const double *vol, *icap, *q0, *pcap, *logpcap;  // [W*N]
  const double *ref, *ap;                          // [3][W*N]
  const double *jap;                               // [3][W*E]
  const double *thr, *jmin;                        // [W*E]
  const double *ovol, *q0o, *vb;                   // [W*O]
  const double *oref;                              // [3][W*O]
  const double *ff;                                // [3][W*F] D A / L
  long long WN, WO, WE, WF;
};

struct FLayout {
  long long s[CB_FIELD_STATE_FIELDS];
};

// Scratch fields of one world, in doubles (offsets from the world's slice).
struct Scratch {
  long long lval, uf, wv, ctl, x, xt, dx, r, rt, y, phi, pc, co, lco, ci, lci, fm, ld, wp, ifc, ijc, k0, k1,
      d1, d2, n1, o1, g1, cp, stride;
  // a rate block: cell amount [3N], membrane transferred [3N], md, cycles, pd, mw [N each],
  // junction transferred [3E], jd, gate [E each], face diffusion [3F], node extracellular [3O],
  // node supply [3O], the outward pump transfer "extra" [3N]
  long long rk_n, rk_mt, rk_md, rk_cy, rk_pd, rk_mw, rk_jt, rk_jd, rk_g, rk_fd, rk_x, rk_s, rk_ex,
      rk_size;
};

__device__ __forceinline__ void logmean(double l, double r, double &mean, double &lg) {
  // extracellular_field.logmean (:48-62)
  const double middle = 0.5 * l + 0.5 * r;
  const double difference = l - r;
  const double ratio = (0.5 * difference) / middle;
  const bool near = fabs(ratio) < 0.5;
  lg = near ? 2.0 * atanh(ratio) : log(l) - log(r);
  if (fabs(ratio) < 1e-4) {
    const double sq = ratio * ratio;
    mean = middle * ((1.0 - sq / 3.0) - 4.0 * sq * sq / 45.0);
  } else {
    mean = difference / lg;
  }
}

template <int BLOCK>
__device__ __forceinline__ double block_max_abs(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double m = red[0];
  for (int q = 1; q < BLOCK / 32; ++q) m = fmax(m, red[q]);
  return m;
}

template <int BLOCK>
__device__ __forceinline__ unsigned block_or(unsigned v, unsigned *red) {
  for (int o = 16; o > 0; o >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  unsigned m = 0;
  for (int q = 0; q < BLOCK / 32; ++q) m |= red[q];
  return m;
}

// Constant-field route flux of species s (z = +1 for Na, K; -1 for Cl), selective_flux with
// residual 0 and gate 1: g (c_from B(-x) - c_to B(x)) for z = +1, the pair swapped for z = -1.
__device__ __forceinline__ double ghk(int s, double g, double cf, double ct, double bp,
                                      double bm) {
  return s < 2 ? g * (cf * bm - ct * bp) : g * (cf * bp - ct * bm);
}

// The step's phases, launched in order by cb_field_step around the factor and solve levels.
enum Phase { PH_START = 0, PH_NEWTON_INIT, PH_NEWTON_SEARCH, PH_AFTER_NEWTON, PH_STAGE1, PH_FINISH };

// A factorisation's face conductances: a (b sum_s W_s(f)) over the faces' weights W.
struct Conductance {
  const double *w;
  int F;
  double a, b;
  __device__ double operator()(int f) const {
    return a * (b * ((w[f] + w[F + f]) + w[2 * F + f]));
  }
};

// kind 0: the start field's Newton matrix (F^2/RT sum factor mean); kind 1: the stage operator
// (gamma dt K F/(R T) sum W at the prediction).
__device__ __forceinline__ Conductance conductance(const Params &P, const Scratch &S, double *base,
                                                   int w, int F, int kind, double gamma_dt) {
  const double *wc = P.wc + (size_t)w * FW_STRIDE;
  if (kind == 0) return Conductance{base + S.fm, F, 1.0, kF * kF / wc[FW_RT]};
  return Conductance{base + S.wp, F, gamma_dt, kChargePerFmol * kF / (kR * wc[FW_T])};
}

// Visit entries [a0, a1) of the lower triangle (i >= j) of an n x n matrix packed by columns
// (column j's entries at j n - j (j - 1) / 2 + (i - j)): fn(i, j, packed index), strided by group.
template <class Fn>
__device__ __forceinline__ void packed_lower(int n, long long a0, long long a1, int gid,
                                             int gsize, Fn fn) {
  int j = 0;
  long long start = 0;
  for (long long a = a0 + gid; a < a1; a += gsize) {
    while (a >= start + (n - j)) {
      start += n - j;
      ++j;
    }
    fn(j + (int)(a - start), j, a);
  }
}
__device__ __forceinline__ long long packed_start(int n, int j) {
  return (long long)j * n - (long long)j * (j - 1) / 2;
}

// Stage a front's factor block (count doubles, global, 16-byte aligned, padded by the plan to an
// even count) into shared memory with one TMA bulk copy (cp.async.bulk, completion on an
// mbarrier that thread gid 0 initialises and arms). The wait is bounded: false when the copy did
// not complete (the caller flags the world; the copy is waited for once more before the CTA
// leaves, see drain_block).
constexpr int kBulkWaitRounds = 1 << 22;
__device__ __forceinline__ unsigned smem_addr(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ bool bulk_done(uint64_t *mbar) {
  unsigned ok = 0;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(mbar))
      : "memory");
  return ok != 0;
}
template <class Sync>
__device__ bool stage_block(double *dst, const double *src, int count, uint64_t *mbar, int gid,
                            Sync sync) {
  const unsigned bytes = (unsigned)((count + 1) & ~1) * 8u;
  if (gid == 0) {
    const unsigned mb = smem_addr(mbar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(mb)
        : "memory");
  }
  sync();
  bool done = false;
  for (int round = 0; round < kBulkWaitRounds && !done; ++round) done = bulk_done(mbar);
  return done;
}
// A copy that stage_block gave up on, waited for once more (bounded) so that it does not land in
// shared memory the CTA no longer owns.
__device__ void drain_block(uint64_t *mbar) {
  for (int round = 0; round < kBulkWaitRounds && !bulk_done(mbar); ++round) {
  }
}

// The trailing update of a block of columns [kb, ke) of an m x sc front in shared memory (column
// major, leading dimension m): A[i][j] -= sum_k A[i][k] A[j][k] for ke <= j < sc, j <= i < m, k in
// [kb, ke), 8x8 tiles of the lower part on the FP64 tensor cores (mma.m8n8k4, k in steps of 4;
// entries past the front read 0), tiles over the group's nw warps (this one wid; lane row r,
// column c of the fragments).
__device__ __forceinline__ void trailing_update(double *A, int m, int sc, int kb, int ke, int wid,
                                                int nw, int r, int c) {
  const int ti = (m - ke + 7) >> 3, tj = (sc - ke + 7) >> 3;
  for (int tile = wid; tile < ti * tj; tile += nw) {
    const int it = tile / tj, jt = tile % tj;
    if (jt > it) continue;  // wholly above the diagonal
    const int ia = ke + it * 8 + r, jb = ke + jt * 8 + r;
    double acc0 = 0.0, acc1 = 0.0;
    for (int k0 = kb; k0 < ke; k0 += 4) {
      const int k = k0 + c;
      const double av = (ia < m && k < ke) ? A[ia + k * m] : 0.0;
      const double bv = (jb < sc && k < ke) ? A[jb + k * m] : 0.0;
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, "
                   "{%0, %1};"
                   : "+d"(acc0), "+d"(acc1)
                   : "d"(av), "d"(bv));
    }
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int j = ke + jt * 8 + 2 * c + e;
      if (ia < m && j < sc && j <= ia) A[ia + j * m] -= e ? acc1 : acc0;
    }
  }
}

// One front q of one world by a group of gsize threads (gid in [0, gsize)) with shared region A
// (its m x s block) and piv (s doubles): assemble the face Laplacian's entries of its columns and
// the entries of its children's update matrices that fall in its columns (children ascending);
// factor its m x s panel right-looking; write its update matrix as minus the panel's product,
// then add the children's entries that fall in it (children ascending); store the panel. Update
// matrices are packed lower triangles. The stored panel holds each column's inverse pivot
// 1/sqrt(d) on its diagonal (the solves multiply by it). Returns nonzero (at gid 0) on a pivot
// that is not positive.
//
// Two factor forms:
//  * !WIDE (a warp, or a CTA): column by column, warps over the later columns, lanes over rows,
//    one sync per column. Few registers, many CTAs per SM: the fronts below the top of the tree;
//  * WIDE (a CTA): blocks of 16 columns, three barriers per block (below); more registers, two
//    CTAs per SM: the wide separators at the top of the tree, whose columns are the critical path.
template <bool WIDE, class Sync>
__device__ unsigned front_factor(const Topo &T, double *LF, double *UF, int q,
                                 const Conductance &g, double *A, double *piv, int gid,
                                 int gsize, Sync sync) {
  const int c0 = T.sn_c0[q], sc = T.sn_s[q], m = T.sn_m[q], b = m - sc;
  double *Uq = UF + T.sn_uoff[q];
  unsigned bad = 0;
  for (int a = gid; a < m * sc; a += gsize) A[a] = 0.0;
  sync();
  for (int k = gid; k < sc; k += gsize) {
    const int node = T.col_node[c0 + k];
    double d = 0.0;
    for (int a = T.nf_ptr[node]; a < T.nf_ptr[node + 1]; ++a) d += g(T.nf_idx[a] >> 1);
    A[k + k * m] = d;
  }
  for (int a = T.af_ptr[q] + gid; a < T.af_ptr[q + 1]; a += gsize) A[T.af_pos[a]] = -g(T.af_face[a]);
  sync();
  for (int t = T.ch_ptr[q]; t < T.ch_ptr[q + 1]; ++t) {
    const int c = T.ch[t];
    const int bc = T.sn_m[c] - T.sn_s[c];
    const double *Uc = UF + T.sn_uoff[c];
    const int *mp = T.map + T.map_ptr[c];
    packed_lower(bc, 0, packed_start(bc, T.split[c]), gid, gsize, [&](int i, int j, long long a) {
      A[mp[i] + mp[j] * m] += Uc[a];
    });
    sync();
  }
  const int nw = gsize >> 5, wid = gid >> 5, ln = gid & 31;
  if constexpr (WIDE) {
    // WIDE: blocks of kPanel columns, three barriers per block:
    //  * the block's diagonal part by warp 0 in registers (a lane per row, right-looking: each
    //    column scaled by its inverse pivot, then its products taken out of the block's later
    //    columns, the other rows' values by shuffle), its inverse pivots left on its diagonal;
    //  * every row below the block by the group, a thread per row in registers (the same scalings
    //    and subtractions, in the same column order);
    //  * the block's contribution taken out of the later columns by the group, 8x8 tiles of their
    //    lower part on the FP64 tensor cores (mma.m8n8k4, k over the block's columns).
    // Each entry sees the same operations in the same order as a column-by-column factor.
    constexpr int kPanel = 16;
    const int r = ln >> 2, c = ln & 3;
    for (int kb = 0; kb < sc; kb += kPanel) {
      const int ke = min(kb + kPanel, sc), nb = ke - kb;
      if (wid == 0) {
        const bool mine = ln < nb;
        double a[kPanel];
#pragma unroll
        for (int j = 0; j < kPanel; ++j)
          a[j] = (mine && j <= ln) ? A[(kb + ln) + (kb + j) * m] : 0.0;
#pragma unroll
        for (int k = 0; k < kPanel; ++k) {
          if (k < nb) {
            const double d = __shfl_sync(0xffffffffu, a[k], k);
            if (ln == 0 && (!(d > 0.0) || !is_finite(d))) bad = 1u;
            const double inv_p = 1.0 / sqrt(d);
            if (ln == k) A[(kb + k) + (kb + k) * m] = inv_p;  // for the rows below
            if (ln > k) a[k] *= inv_p;
#pragma unroll
            for (int j = k + 1; j < kPanel; ++j) {
              if (j < nb) {
                const double ljk = __shfl_sync(0xffffffffu, a[k], j);
                if (ln >= j) a[j] -= a[k] * ljk;
              }
            }
          }
        }
        if (mine) {
#pragma unroll
          for (int j = 0; j < kPanel; ++j)
            if (j < ln) A[(kb + ln) + (kb + j) * m] = a[j];
        }
      }
      sync();
      for (int i = ke + gid; i < m; i += gsize) {
        double x[kPanel];
#pragma unroll
        for (int k = 0; k < kPanel; ++k) x[k] = k < nb ? A[i + (kb + k) * m] : 0.0;
#pragma unroll
        for (int k = 0; k < kPanel; ++k) {
          if (k < nb) {
            x[k] *= A[(kb + k) + (kb + k) * m];
#pragma unroll
            for (int j = k + 1; j < kPanel; ++j)
              if (j < nb) x[j] -= x[k] * A[(kb + j) + (kb + k) * m];
          }
        }
#pragma unroll
        for (int k = 0; k < kPanel; ++k)
          if (k < nb) A[i + (kb + k) * m] = x[k];
      }
      sync();
      if (ke < sc) {
        trailing_update(A, m, sc, kb, ke, wid, nw, r, c);
        sync();
      }
    }
    sync();
  } else {
    // Column by column: warps of the group over the later columns, lanes over rows, a sync per
    // column (the trailing update uses the unscaled pivot column over the pivot; the column is
    // scaled after the sync).
    for (int k = 0; k < sc; ++k) {
      const double d = A[k + k * m];
      if (gid == 0 && (!(d > 0.0) || !is_finite(d))) bad = 1u;
      const double inv_d = 1.0 / d, inv_p = 1.0 / sqrt(d);
      if (gid == 0) piv[k] = inv_p;
      for (int j = k + 1 + wid; j < sc; j += nw) {
        const double ljk = A[j + k * m] * inv_d;
        for (int i = j + ln; i < m; i += 32) A[i + j * m] -= A[i + k * m] * ljk;
      }
      sync();
      for (int i = k + 1 + gid; i < m; i += gsize) A[i + k * m] *= inv_p;
    }
    sync();
    for (int k = gid; k < sc; k += gsize) A[k + k * m] = piv[k];
    sync();
  }
  // The update matrix -L_B L_B^T on the FP64 tensor cores: 8x8 tiles of its lower triangle,
  // one warp per tile, k in steps of 4 (mma.m8n8k4.f64; rows past b and columns past sc read 0).
  {
    const int nt = (b + 7) >> 3;
    const int r = ln >> 2, c = ln & 3;
    for (int tile = wid; tile < nt * (nt + 1) / 2; tile += nw) {
      int it = 0;
      while ((it + 1) * (it + 2) / 2 <= tile) ++it;
      const int jt = tile - it * (it + 1) / 2;
      const int ia = it * 8 + r, jb = jt * 8 + r;
      double acc0 = 0.0, acc1 = 0.0;
      for (int k0 = 0; k0 < sc; k0 += 4) {
        const int k = k0 + c;
        const double av = (ia < b && k < sc) ? A[sc + ia + k * m] : 0.0;
        const double bv = (jb < b && k < sc) ? A[sc + jb + k * m] : 0.0;
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, "
                     "{%0, %1};"
                     : "+d"(acc0), "+d"(acc1)
                     : "d"(av), "d"(bv));
      }
      const int i = it * 8 + r;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int j = jt * 8 + 2 * c + e;
        if (i < b && j <= i) Uq[packed_start(b, j) + (i - j)] = -(e ? acc1 : acc0);
      }
    }
  }
  sync();
  for (int t = T.ch_ptr[q]; t < T.ch_ptr[q + 1]; ++t) {
    const int c = T.ch[t];
    const int bc = T.sn_m[c] - T.sn_s[c];
    const double *Uc = UF + T.sn_uoff[c];
    const int *mp = T.map + T.map_ptr[c];
    packed_lower(bc, packed_start(bc, T.split[c]), packed_start(bc, bc), gid, gsize,
                 [&](int i, int j, long long a) {
                   const int pr = mp[i] - sc, pc = mp[j] - sc;
                   Uq[packed_start(b, pc) + (pr - pc)] += Uc[a];
                 });
    sync();
  }
  double *Lq = LF + T.sn_loff[q];
  for (int a = gid; a < m * sc; a += gsize) Lq[a] = A[a];
  sync();
  return bad;
}

// Forward substitution of front q: its columns' right-hand side (Y) plus its children's update
// vectors, the dense triangular solve on the staged block, the update vector for its parent.
template <class Sync>
__device__ bool front_forward(const Topo &T, const double *LF, double *WV, double *Y, int q,
                              double *A, double *v, uint64_t *mbar, int gid, int gsize,
                              Sync sync) {
  const int c0 = T.sn_c0[q], sc = T.sn_s[q], m = T.sn_m[q];
  const double *Lq = LF + T.sn_loff[q];
  for (int i = gid; i < m; i += gsize) v[i] = i < sc ? Y[c0 + i] : 0.0;
  if (!stage_block(A, Lq, m * sc, mbar, gid, sync)) {
    drain_block(mbar);
    return false;
  }
  sync();
  for (int t = T.ch_ptr[q]; t < T.ch_ptr[q + 1]; ++t) {
    const int c = T.ch[t];
    const int bc = T.sn_m[c] - T.sn_s[c];
    const double *vc = WV + T.sn_voff[c];
    const int *mp = T.map + T.map_ptr[c];
    for (int i = gid; i < bc; i += gsize) v[mp[i]] += vc[i];
    sync();
  }
  // Blocks of 32 columns: the diagonal block by warp 0 (a lane per row, the column's value by
  // shuffle, times the column's inverse pivot), then every row below it by the group, each
  // row's subtractions in column order (the same arithmetic as column by column, two barriers
  // per block).
  for (int kb = 0; kb < sc; kb += 32) {
    const int kw = min(32, sc - kb);
    if (gid < 32) {
      double x = gid < kw ? v[kb + gid] : 0.0;
      for (int k = 0; k < kw; ++k) {
        const double xk = __shfl_sync(0xffffffffu, x, k) * A[(kb + k) + (kb + k) * m];
        if (gid == k) x = xk;
        if (gid > k && gid < kw) x -= A[(kb + gid) + (kb + k) * m] * xk;
      }
      if (gid < kw) v[kb + gid] = x;
    }
    sync();
    for (int i = kb + kw + gid; i < m; i += gsize) {
      double t = v[i];
      for (int k = 0; k < kw; ++k) t -= A[i + (kb + k) * m] * v[kb + k];
      v[i] = t;
    }
    sync();
  }
  sync();
  double *vq = WV + T.sn_voff[q];
  for (int i = gid; i < m; i += gsize) {
    if (i < sc) Y[c0 + i] = v[i];
    else vq[i - sc] = v[i];
  }
  return true;
}

// Back substitution of front q: t = y_S - L_BS^T x_B (x_B from its ancestors, in out), one
// column per thread; then L_SS^T x_S = t in blocks of 32 columns.
template <class Sync>
__device__ bool front_backward(const Topo &T, const double *LF, const double *Y, double *out,
                               int q, double *A, double *v, uint64_t *mbar, int gid, int gsize,
                               Sync sync) {
  const int c0 = T.sn_c0[q], sc = T.sn_s[q], m = T.sn_m[q];
  const double *Lq = LF + T.sn_loff[q];
  const int *rq = T.rows + T.rows_ptr[q];
  for (int i = sc + gid; i < m; i += gsize) v[i] = out[rq[i]];
  if (!stage_block(A, Lq, m * sc, mbar, gid, sync)) {
    drain_block(mbar);
    return false;
  }
  sync();
  for (int k = gid; k < sc; k += gsize) {
    double t = Y[c0 + k];
    for (int i = sc; i < m; ++i) t -= A[i + k * m] * v[i];
    v[k] = t;
  }
  sync();
  // Blocks of 32 columns from the last: the diagonal block by warp 0, then every column before
  // it by the group, each one's subtractions in descending column order (the same arithmetic as
  // the column sweep, two barriers per block; the inverse pivots on the diagonal).
  for (int ke = sc; ke > 0; ke -= 32) {
    const int kb = max(0, ke - 32), kw = ke - kb;
    if (gid < 32) {
      double x = gid < kw ? v[kb + gid] : 0.0;
      for (int k = kw - 1; k > 0; --k) {
        const double xk = __shfl_sync(0xffffffffu, x, k) * A[(kb + k) + (kb + k) * m];
        if (gid < k) x -= A[(kb + k) + (kb + gid) * m] * xk;
      }
      if (gid < kw) v[kb + gid] = x;
    }
    sync();
    for (int j = gid; j < kb; j += gsize) {
      double t = v[j];
      for (int k = kw - 1; k >= 0; --k)
        t -= A[(kb + k) + j * m] * (v[kb + k] * A[(kb + k) + (kb + k) * m]);
      v[j] = t;
    }
    sync();
  }
  for (int k = gid; k < sc; k += gsize) out[c0 + k] = v[k] * A[k + k * m];
  return true;
}

// Level kernels. Warp form: each warp one (front, world) task of the level, world-major, with a
// slice of shared memory (the level's largest block, then its largest front's vector). CTA form:
// one CTA of kGroupThreads per (front, world). Refused worlds are skipped.
constexpr int kWarpsPerCta = 8;
constexpr int kGroupThreads = 256;
// Shared memory of a level's task: the front block (its TMA copy rounded up to an even count of
// doubles, 16 bytes), then the front's vector; a warp task's slice kept even so every block
// starts on a 16-byte boundary.
__host__ __device__ constexpr long long level_vec(long long block) { return (block + 1) & ~1LL; }
__host__ __device__ constexpr long long level_slice(long long block, long long rows) {
  return (level_vec(block) + rows + 1) & ~1LL;
}

struct LevelTask {
  int q, w;
  bool ok;
};

__device__ __forceinline__ LevelTask warp_task(const Topo &T, const uint32_t *status, int a0,
                                               int fronts, int W) {
  const long long task = (long long)blockIdx.x * kWarpsPerCta + (threadIdx.x >> 5);
  if (task >= (long long)fronts * W) return {0, 0, false};
  const int w = (int)(task / fronts);
  return {T.lv_sn[a0 + (int)(task % fronts)], w, status[w] == 0u};
}


__global__ void __launch_bounds__(kWarpsPerCta * 32)
    factor_warps(const Topo T, const Params P, const Scratch S, double *scratch,
                 const uint32_t *status, int kind, double gamma_dt, int a0, int fronts, int W,
                 int slice, int vec) {
  extern __shared__ __align__(16) double sm[];
  const LevelTask t = warp_task(T, status, a0, fronts, W);
  if (!t.ok) return;
  double *base = scratch + (size_t)t.w * S.stride;
  double *A = sm + (size_t)(threadIdx.x >> 5) * slice;
  const unsigned bad = front_factor<false>(T, base + S.lval, base + S.uf, t.q,
                                           conductance(P, S, base, t.w, T.F, kind, gamma_dt), A,
                                           A + vec, threadIdx.x & 31, 32, [] { __syncwarp(); });
  if (bad) base[S.ctl + 7] = 1.0;
}

// The narrow form's registers held to six CTAs per SM, the wide form's to two.
template <bool WIDE>
__global__ void __launch_bounds__(kGroupThreads, WIDE ? 2 : 6)
    factor_group(const Topo T, const Params P, const Scratch S, double *scratch,
                 const uint32_t *status, int kind, double gamma_dt, int a0, int vec) {
  extern __shared__ __align__(16) double sm[];
  const int w = blockIdx.y;
  if (status[w] != 0u) return;
  double *base = scratch + (size_t)w * S.stride;
  const unsigned bad = front_factor<WIDE>(T, base + S.lval, base + S.uf,
                                          T.lv_sn[a0 + blockIdx.x],
                                          conductance(P, S, base, w, T.F, kind, gamma_dt), sm,
                                          sm + vec, threadIdx.x, kGroupThreads,
                                          [] { __syncthreads(); });
  if (bad) base[S.ctl + 7] = 1.0;
}

// The substitutions' warp kernels at eight CTAs per SM's registers (their small leaf slices fit).
__global__ void __launch_bounds__(kWarpsPerCta * 32, 8)
    forward_warps(const Topo T, const Scratch S, double *scratch, const uint32_t *status, int a0,
                  int fronts, int W, int slice, int vec) {
  extern __shared__ __align__(16) double sm[];
  __shared__ uint64_t mbar[kWarpsPerCta];
  const LevelTask t = warp_task(T, status, a0, fronts, W);
  if (!t.ok) return;
  double *base = scratch + (size_t)t.w * S.stride;
  double *A = sm + (size_t)(threadIdx.x >> 5) * slice;
  if (!front_forward(T, base + S.lval, base + S.wv, base + S.y, t.q, A, A + vec,
                     mbar + (threadIdx.x >> 5), threadIdx.x & 31, 32, [] { __syncwarp(); }))
    base[S.ctl + 7] = 1.0;
}

__global__ void __launch_bounds__(kGroupThreads)
    forward_group(const Topo T, const Scratch S, double *scratch, const uint32_t *status, int a0,
                  int vec) {
  extern __shared__ __align__(16) double sm[];
  __shared__ uint64_t mbar;
  const int w = blockIdx.y;
  if (status[w] != 0u) return;
  double *base = scratch + (size_t)w * S.stride;
  if (!front_forward(T, base + S.lval, base + S.wv, base + S.y, T.lv_sn[a0 + blockIdx.x], sm,
                     sm + vec, &mbar, threadIdx.x, kGroupThreads, [] { __syncthreads(); }) &&
      threadIdx.x == 0)
    base[S.ctl + 7] = 1.0;
}

__global__ void __launch_bounds__(kWarpsPerCta * 32, 8)
    backward_warps(const Topo T, const Scratch S, double *scratch, const uint32_t *status,
                   long long out_off, int a0, int fronts, int W, int slice, int vec) {
  extern __shared__ __align__(16) double sm[];
  __shared__ uint64_t mbar[kWarpsPerCta];
  const LevelTask t = warp_task(T, status, a0, fronts, W);
  if (!t.ok) return;
  double *base = scratch + (size_t)t.w * S.stride;
  double *A = sm + (size_t)(threadIdx.x >> 5) * slice;
  if (!front_backward(T, base + S.lval, base + S.y, base + out_off, t.q, A, A + vec,
                      mbar + (threadIdx.x >> 5), threadIdx.x & 31, 32, [] { __syncwarp(); }))
    base[S.ctl + 7] = 1.0;
}

__global__ void __launch_bounds__(kGroupThreads)
    backward_group(const Topo T, const Scratch S, double *scratch, const uint32_t *status,
                   long long out_off, int a0, int vec) {
  extern __shared__ __align__(16) double sm[];
  __shared__ uint64_t mbar;
  const int w = blockIdx.y;
  if (status[w] != 0u) return;
  double *base = scratch + (size_t)w * S.stride;
  if (!front_backward(T, base + S.lval, base + S.y, base + out_off, T.lv_sn[a0 + blockIdx.x], sm,
                      sm + vec, &mbar, threadIdx.x, kGroupThreads, [] { __syncthreads(); }) &&
      threadIdx.x == 0)
    base[S.ctl + 7] = 1.0;
}

// One instantiation per phase, so each gets its own register allocation (MINB: CTAs per SM).
template <int BLOCK, int phase, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB)
    field_phase(const Topo T, const Params P, const FLayout L, const Scratch S,
                double *__restrict__ state, const double *__restrict__ control, const StepCoef k,
                int first, uint32_t *__restrict__ status,
                int32_t *__restrict__ taken_out, double *__restrict__ scratch,
                int *__restrict__ any_active) {
  __shared__ double sRed[BLOCK / 32];
  __shared__ unsigned sBits[BLOCK / 32];
  [[maybe_unused]] constexpr int WARPS = BLOCK / 32;
  const int w = blockIdx.x, tid = threadIdx.x;
  [[maybe_unused]] const int lane = tid & 31, warp = tid >> 5;
  const int N = T.N, O = T.O, E = T.E, F = T.F, U = T.U;
  const long long WN = P.WN, WO = P.WO, WE = P.WE, WF = P.WF;
  const long long c0 = (long long)w * N, o0 = (long long)w * O, e0 = (long long)w * E,
                  f0 = (long long)w * F;
  const double *wc = P.wc + (size_t)w * FW_STRIDE;
  const double RT = wc[FW_RT], FRT = wc[FW_FRT], temp = wc[FW_T];
  double *base = scratch + (size_t)w * S.stride;
  double *ctl = base + S.ctl;  // per world: bits, count, accepted, active, norm, rmax, taken, bad
  if (status[w] != 0u) return;  // refused earlier in this call
  double *X = base + S.x, *XT = base + S.xt, *DX = base + S.dx, *Rv = base + S.r,
         *RTv = base + S.rt, *Y = base + S.y;
  double *PHI = base + S.phi, *PC = base + S.pc;
  double *CO = base + S.co, *LCO = base + S.lco, *CI = base + S.ci, *LCI = base + S.lci;
  double *FM = base + S.fm, *LD = base + S.ld, *WP = base + S.wp;
  double *IFC = base + S.ifc, *IJC = base + S.ijc;
  double *K0 = base + S.k0, *K1 = base + S.k1, *D1 = base + S.d1, *D2 = base + S.d2;
  double *N1 = base + S.n1, *O1 = base + S.o1, *G1 = base + S.g1, *CP = base + S.cp;
  const double *cm = control, *cj = control + WN, *cpmp = control + WN + WE;
  auto st = [&](int f) { return state + L.s[f]; };
  const double dt = k.dt;
  const double omgamma_dt = (1.0 - (1.0 - 1.0 / sqrt(2.0))) * dt;  // (1 - gamma) dt

  // ---- transport pieces --------------------------------------------------------------------
  // Concentrations and logs of a stage: cells from amounts n (functor (s, i)), nodes from o.
  auto set_conc = [&](auto n, auto o) -> unsigned {
    unsigned bits = 0;
    for (int i = tid; i < N; i += BLOCK) {
      const double v = P.vol[c0 + i];
      for (int s = 0; s < 3; ++s) {
        const double c = (P.ref[s * WN + c0 + i] + n(s, i)) / v;
        if (!(is_finite(c) && c > 0.0)) bits |= CB_WORLD_TRANSPORT;
        CI[s * N + i] = c;
        LCI[s * N + i] = log(c);
      }
    }
    for (int m = tid; m < O; m += BLOCK) {
      const double v = P.ovol[o0 + m];
      for (int s = 0; s < 3; ++s) {
        const double c = (P.oref[s * WO + o0 + m] + o(s, m)) / v;
        if (!(is_finite(c) && c > 0.0)) bits |= CB_WORLD_TRANSPORT;
        CO[s * O + m] = c;
        LCO[s * O + m] = log(c);
      }
    }
    return bits;
  };
  // A junction's constant-field fluxes at voltage dv (opening = availability x gate).
  auto junction_flux = [&](int e, double dv, double opening, double (&jj)[3], double (&mu)[3],
                           unsigned &bits) {
    const int a = T.js[e], b = T.jr[e];
    const double x = dv * FRT;
    if (!(fabs(x) <= kMaxAbsX)) bits |= CB_WORLD_TRANSPORT;
    double bp, bm;
    bernoulli_pair<double>(x, bp, bm);
    for (int s = 0; s < 3; ++s) {
      const double g = P.jap[s * WE + e0 + e] * opening;
      jj[s] = ghk(s, g, CI[s * N + a], CI[s * N + b], bp, bm);
      mu[s] = RT * (LCI[s * N + a] - LCI[s * N + b]) + ((s < 2) ? kF * dv : (-kF) * dv);
    }
  };
  // A face's current (A) at potentials PHI with the step start's weights (transport's face
  // expression: flux = factor mean mu / (RT 1e-15)).
  auto face_current = [&](int f) {
    const double dv = PHI[T.fs[f]] - PHI[T.fr[f]];
    double cur = 0.0;
    for (int s = 0; s < 3; ++s) {
      const double z = s < 2 ? 1.0 : -1.0;
      const double mu = RT * LD[s * F + f] + z * kF * dv;
      const double flux = FM[s * F + f] * mu / (RT * 1e-15);
      cur += z * flux;
    }
    return kChargePerFmol * cur;
  };
  // Explicit rates at a stage (surface_pump.explicit_rates): concentrations in CI/CO, cell
  // potentials PC, node potentials PHI, gates g(e), into rate block K. Face diffusion uses the
  // stage's own weights (W ln(a/b)); at the step start (start) those are the start field's
  // factor means FM and log differences LD, the same values the logmean gives.
  auto explicit_rates = [&](double *Kb, auto gate, bool start) -> unsigned {
    unsigned bits = 0;
    double *kn = Kb + S.rk_n, *kmt = Kb + S.rk_mt, *kmd = Kb + S.rk_md, *kcy = Kb + S.rk_cy,
           *kpd = Kb + S.rk_pd, *kmw = Kb + S.rk_mw, *kjt = Kb + S.rk_jt, *kjd = Kb + S.rk_jd,
           *kg = Kb + S.rk_g, *kfd = Kb + S.rk_fd, *kx = Kb + S.rk_x, *ks = Kb + S.rk_s,
           *kex = Kb + S.rk_ex;
    for (int i = tid; i < N; i += BLOCK) {
      const int m = T.cell_node[i];
      const double dv = PC[i] - PHI[m];
      const double x = dv * FRT;
      if (!(fabs(x) <= kMaxAbsX)) bits |= CB_WORLD_TRANSPORT;
      double bp, bm;
      bernoulli_pair<double>(x, bp, bm);
      const double mc = cm[c0 + i], pcc = cpmp[c0 + i];
      if (!(is_finite(mc) && mc >= 0.0 && mc <= 1.0 && is_finite(pcc) && pcc >= 0.0 &&
            pcc <= 1.0))
        bits |= CB_WORLD_CONTROL;
      double jm[3], mu[3];
      for (int s = 0; s < 3; ++s) {
        const double g = P.ap[s * WN + c0 + i] * mc;
        jm[s] = ghk(s, g, CI[s * N + i], CO[s * O + m], bp, bm);
        mu[s] = RT * (LCI[s * N + i] - LCO[s * O + m]) + ((s < 2) ? kF * dv : (-kF) * dv);
        kmt[s * N + i] = jm[s];
      }
      const double md = 1e-3 * ((jm[0] * mu[0] + jm[1] * mu[1]) + jm[2] * mu[2]);
      kmd[i] = md;
      if (!(is_finite(jm[0]) && is_finite(jm[1]) && is_finite(jm[2]) && is_finite(md)))
        bits |= CB_WORLD_TRANSPORT;
      // Na/K-ATPase: Na inside, K at the cell's node.
      const double drive = wc[FW_DRIVE];
      const double energy = (drive + (-3.0) * mu[0]) + 2.0 * mu[1];
      const double a = energy * wc[FW_INVRT];
      double cycles = 0.0;
      const double cap = P.pcap[c0 + i];
      if (cap > 0.0 && pcc > 0.0) {
        const double lk = logaddexp0(2.0 * (wc[FW_LOGKMK] - LCO[O + m]));
        const double ls = ((-logaddexp0(3.0 * (wc[FW_LOGKMNA] - LCI[i]))) - lk) - wc[FW_LATP];
        const double mag = exp(((P.logpcap[c0 + i] + log(pcc)) + ls) + fmax(a, 0.0));
        const double dep = a >= 0.0 ? expm1(-a) : -expm1(a);
        cycles = mag * dep;
      }
      const double pd = (-1e-3 * cycles) * energy, mw = (-1e-3 * cycles) * drive;
      kcy[i] = cycles;
      kpd[i] = pd;
      kmw[i] = mw;
      kex[i] = 3.0 * cycles;
      kex[N + i] = -2.0 * cycles;
      kex[2 * N + i] = -0.0 * cycles;
      const double sna = mu[0] * wc[FW_INVRTD], sk = mu[1] * wc[FW_INVRTD];
      const double aff = (wc[FW_AFF0] + (-3.0) * sna) + 2.0 * sk;
      if (!(wc[FW_PUMPOK] != 0.0 && is_finite(cap) && cap >= 0.0 && is_finite(sna) &&
            fabs(sna) <= kMaxAbsIonPotentialOverRT && is_finite(sk) &&
            fabs(sk) <= kMaxAbsIonPotentialOverRT && is_finite(aff) &&
            fabs(aff) <= kMaxAbsAffinityOverRT))
        bits |= CB_WORLD_PUMP_DOMAIN;
      if (!(is_finite(cycles) && is_finite(pd) && is_finite(mw))) bits |= CB_WORLD_TRANSPORT;
    }
    for (int e = tid; e < E; e += BLOCK) {
      const double g = gate(e);
      const double dv = PC[T.js[e]] - PC[T.jr[e]];
      const double jc = cj[e0 + e];
      double jj[3], mu[3];
      junction_flux(e, dv, jc * g, jj, mu, bits);
      for (int s = 0; s < 3; ++s) kjt[s * E + e] = jj[s];
      const double jd = 1e-3 * ((jj[0] * mu[0] + jj[1] * mu[1]) + jj[2] * mu[2]);
      kjd[e] = jd;
      const double thr = P.thr[e0 + e], mn = P.jmin[e0 + e];
      double gr = 0.0;
      if (mn < 1.0) {
        const double shift = fabs(dv) - thr;
        const double alpha = 1.3 * exp(-77.0 * shift);
        const double log_beta = kLog0065 + 140.0 * shift;
        const double beta = 20.0 * exp(-logaddexp0(-log_beta));
        gr = alpha * (1.0 - g) - beta * (g - mn);
      }
      kg[e] = gr;
      const bool gate_ok = is_finite(thr) && thr >= 0.0 && thr <= kMaxAbsJunctionV &&
                           is_finite(mn) && mn >= 0.0 && mn <= 1.0 && is_finite(dv) &&
                           fabs(dv) <= kMaxAbsJunctionV && is_finite(g) && g >= mn && g <= 1.0 &&
                           is_finite(jc) && jc >= 0.0 && jc <= 1.0;
      if (!gate_ok) bits |= CB_WORLD_GATE_DOMAIN;
      if (!(is_finite(jj[0]) && is_finite(jj[1]) && is_finite(jj[2]) && is_finite(jd) &&
            is_finite(gr)))
        bits |= CB_WORLD_TRANSPORT;
    }
    for (int f = tid; f < F; f += BLOCK) {
      const int a = T.fs[f], b = T.fr[f];
      const double dv = PHI[a] - PHI[b];
      if (!(fabs(dv * FRT) <= kMaxAbsX)) bits |= CB_WORLD_TRANSPORT;
      for (int s = 0; s < 3; ++s) {
        double d;
        if (start) {  // the step start's concentrations: their factor mean and log difference
          d = (FM[s * F + f] / 1e-15) * LD[s * F + f];
        } else {
          double mean, lg;
          logmean(CO[s * O + a], CO[s * O + b], mean, lg);
          const double wgt = P.ff[s * WF + f0 + f] * mean / 1e-15;
          d = wgt * (LCO[s * O + a] - LCO[s * O + b]);
        }
        kfd[s * F + f] = d;
        if (!is_finite(d)) bits |= CB_WORLD_TRANSPORT;
      }
    }
    __syncthreads();
    for (int i = tid; i < N; i += BLOCK) {
      double snd[3] = {0.0, 0.0, 0.0}, rcv[3] = {0.0, 0.0, 0.0};
      for (int a = T.cj_ptr[i]; a < T.cj_ptr[i + 1]; ++a) {
        const int code = T.cj_idx[a], e = code >> 1;
        for (int s = 0; s < 3; ++s) {
          if (code & 1) rcv[s] += kjt[s * E + e];
          else snd[s] += -kjt[s * E + e];
        }
      }
      for (int s = 0; s < 3; ++s) {
        const double cell = ((-kmt[s * N + i]) + snd[s]) + rcv[s];
        kn[s * N + i] = cell - kex[s * N + i];
        if (!is_finite(kn[s * N + i])) bits |= CB_WORLD_TRANSPORT;
      }
    }
    for (int m = tid; m < O; m += BLOCK) {
      const int i = T.ncell[m];
      const bool held = T.upos[m] < 0;
      for (int s = 0; s < 3; ++s) {
        double a = 0.0, out = 0.0, in = 0.0;
        if (i >= 0) a = 0.0 + (kmt[s * N + i] + kex[s * N + i]);
        for (int q = T.nf_ptr[m]; q < T.nf_ptr[m + 1]; ++q) {
          const int code = T.nf_idx[q];
          if (code & 1) in += kfd[s * F + (code >> 1)];
          else out += kfd[s * F + (code >> 1)];
        }
        const double inflow = (a - out) + in;
        kx[s * O + m] = held ? 0.0 : inflow;
        ks[s * O + m] = held ? -inflow : 0.0;
      }
    }
    __syncthreads();
    return bits;
  };

  // Per-world control words across the phases (doubles holding small integers and flags).
  auto bits_in = [&]() { return (unsigned)ctl[0]; };
  auto bits_out = [&](unsigned b) {
    b = block_or<BLOCK>(b, sBits);
    if (tid == 0) ctl[0] = (double)b;
    __syncthreads();
  };
  const double *n0 = st(CB_FIELD_AMOUNT_INCREMENT), *x0 = st(CB_FIELD_EXTRACELLULAR_INCREMENT);
  const double *g0 = st(CB_FIELD_JUNCTION_GATE) + e0;
  const double cond = kChargePerFmol * kF / (kR * temp);
  auto gface = [&](int f) {
    return k.gamma_dt * (cond * ((WP[f] + WP[F + f]) + WP[2 * F + f]));
  };
    // residual at potentials PHI (cells PC = node + relative): face currents, then junctions.
    auto cell_potentials = [&](double *dst) {
      for (int i = tid; i < N; i += BLOCK) {
        const double *n = st(CB_FIELD_AMOUNT_INCREMENT);
        const double q = P.q0[c0 + i] +
                         kChargePerFmol * ((n[c0 + i] + n[WN + c0 + i]) + (-n[2 * WN + c0 + i]));
        dst[i] = q * P.icap[c0 + i] + PHI[T.cell_node[i]];
      }
    };
    // evaluate: residual into res (by factor column), returns (max |residual|, norm, valid).
    auto evaluate = [&](double *res, bool junctions, double &rmax, double &norm) -> bool {
      unsigned b = 0;
      cell_potentials(PC);
      for (int f = tid; f < F; f += BLOCK) {
        IFC[f] = face_current(f);
        if (!(fabs((PHI[T.fs[f]] - PHI[T.fr[f]]) * FRT) <= kMaxAbsX) || !is_finite(IFC[f]))
          b |= 1u;
      }
      __syncthreads();
      for (int e = tid; e < E; e += BLOCK) {
        double jj[3], mu[3];
        unsigned jb = 0;
        const double opening = cj[e0 + e] * st(CB_FIELD_JUNCTION_GATE)[e0 + e];
        junction_flux(e, PC[T.js[e]] - PC[T.jr[e]], opening, jj, mu, jb);
        IJC[e] = junctions ? kChargePerFmol * ((jj[0] + jj[1]) + (-jj[2])) : 0.0;
        if (jb || !is_finite(IJC[e])) b |= 1u;
      }
      __syncthreads();
      double mr = 0.0, sc = 0.0;
      for (int f = tid; f < F; f += BLOCK) sc = fmax(sc, fabs(IFC[f]));
      for (int e = tid; e < E; e += BLOCK) sc = fmax(sc, fabs(IJC[e]));
      for (int m = tid; m < O; m += BLOCK) {
        const int u = T.upos[m];
        if (u < 0) continue;
        double r = 0.0;
        for (int q = T.nf_ptr[m]; q < T.nf_ptr[m + 1]; ++q) {
          const int code = T.nf_idx[q];
          r += (code & 1) ? -IFC[code >> 1] : IFC[code >> 1];
        }
        const int i = T.ncell[m];
        if (i >= 0)
          for (int q = T.cj_ptr[i]; q < T.cj_ptr[i + 1]; ++q) {
            const int code = T.cj_idx[q];
            r += (code & 1) ? -IJC[code >> 1] : IJC[code >> 1];
          }
        res[u] = r;
        mr = fmax(mr, fabs(r));
        if (!is_finite(r)) b |= 1u;
      }
      for (int i = tid; i < N; i += BLOCK)
        if (!(fabs((PC[i] - PHI[T.cell_node[i]]) * FRT) <= kMaxAbsX)) b |= 1u;
      rmax = block_max_abs<BLOCK>(mr, sRed);
      const double scale = block_max_abs<BLOCK>(sc, sRed);
      norm = rmax / (kCurrentAtol + kCurrentRtol * scale);
      return block_or<BLOCK>(b, sBits) == 0u && is_finite(norm);
    };
    auto set_phi = [&](const double *x) {
      for (int m = tid; m < O; m += BLOCK) {
        const int u = T.upos[m];
        PHI[m] = u < 0 ? P.vb[o0 + m] : x[u];
      }
      __syncthreads();
    };
  // The stage solve's right-hand side on known amounts (cells n(s,i), nodes o3(m, v[3])), into Y
  // (and RTv, kept for the residual check).
  auto stage_rhs = [&](auto n, auto o3) {
    for (int m = tid; m < O; m += BLOCK) {
      const int u = T.upos[m];
      if (u < 0) continue;
      double ov[3];
      o3(m, ov);
      double q = P.q0o[o0 + m] + kChargePerFmol * ((ov[0] + ov[1]) + (-ov[2]));
      const int i = T.ncell[m];
      if (i >= 0)
        q = q + (P.q0[c0 + i] + kChargePerFmol * ((n(0, i) + n(1, i)) + (-n(2, i))));
      for (int a = T.nf_ptr[m]; a < T.nf_ptr[m + 1]; ++a) {
        const int f = T.nf_idx[a] >> 1;
        const int other = T.fs[f] == m ? T.fr[f] : T.fs[f];
        if (T.upos[other] < 0) q += gface(f) * P.vb[o0 + other];
      }
      Y[u] = q;
      RTv[u] = q;
    }
    __syncthreads();
  };
  // The stage solution X: potentials into PHI, PC, and the stage solve's acceptance (the
  // residual r = b - L x on the free rows within CHARGE_ATOL + CHARGE_RTOL max(|b|, |L x|),
  // numerics/surface_imex.py).
  auto stage_post = [&](auto n) -> unsigned {
    unsigned b = 0;
    for (int m = tid; m < O; m += BLOCK) {
      const int u = T.upos[m];
      PHI[m] = u < 0 ? P.vb[o0 + m] : X[u];
      if (u < 0) continue;
      double diag = 0.0, off = 0.0;
      for (int a = T.nf_ptr[m]; a < T.nf_ptr[m + 1]; ++a) {
        const int f = T.nf_idx[a] >> 1;
        const double g = gface(f);
        diag += g;
        const int other = T.fs[f] == m ? T.fr[f] : T.fs[f];
        const int v = T.upos[other];
        if (v >= 0) off += g * X[v];
      }
      const double lx = diag * X[u] - off;
      const double r = RTv[u] - lx;
      if (!(fabs(r) <= kChargeAtol + kChargeRtol * fmax(fabs(RTv[u]), fabs(lx)))) b = 1u;
    }
    __syncthreads();
    for (int i = tid; i < N; i += BLOCK) {
      const double q = P.q0[c0 + i] + kChargePerFmol * ((n(0, i) + n(1, i)) + (-n(2, i)));
      PC[i] = PHI[T.cell_node[i]] + q * P.icap[c0 + i];
      if (!is_finite(PC[i])) b = 1u;
    }
    for (int m = tid; m < O; m += BLOCK)
      if (!is_finite(PHI[m])) b = 1u;
    __syncthreads();
    return b ? (unsigned)CB_WORLD_RESIDUAL : 0u;
  };
    // The implicit drift W z F/RT dv at the stage potentials into D.
    auto drift = [&](double *D) {
      for (int f = tid; f < F; f += BLOCK) {
        const double dv = PHI[T.fs[f]] - PHI[T.fr[f]];
        for (int s = 0; s < 3; ++s) {
          const double z = s < 2 ? 1.0 : -1.0;
          D[s * F + f] = WP[s * F + f] * (z * FRT) * dv;
        }
      }
      __syncthreads();
    };
    // A node's drift inflow of each species (scatter to receivers less scatter from senders), in
    // one pass over its faces.
    auto drift_inflow3 = [&](const double *D, int m, double (&r)[3]) {
      double in[3] = {0.0, 0.0, 0.0}, out[3] = {0.0, 0.0, 0.0};
      for (int q = T.nf_ptr[m]; q < T.nf_ptr[m + 1]; ++q) {
        const int code = T.nf_idx[q], f = code >> 1;
        for (int s = 0; s < 3; ++s) {
          if (code & 1) in[s] += D[s * F + f];
          else out[s] += D[s * F + f];
        }
      }
      for (int s = 0; s < 3; ++s) r[s] = in[s] - out[s];
    };
  auto known1_cell = [&](int s, int i) {
    return n0[s * WN + c0 + i] + k.gamma_dt * K0[S.rk_n + s * N + i];
  };
  auto known1_node = [&](int s, int m) {
    return x0[s * WO + o0 + m] + k.gamma_dt * K0[S.rk_x + s * O + m];
  };
  auto known2_cell = [&](int s, int i) {
    return (n0[s * WN + c0 + i] + k.delta_dt * K0[S.rk_n + s * N + i]) +
           k.omdelta_dt * K1[S.rk_n + s * N + i];
  };
  auto known1_node3 = [&](int m, double (&v)[3]) {
    for (int s = 0; s < 3; ++s) v[s] = known1_node(s, m);
  };
  auto known2_node3 = [&](int m, double (&v)[3]) {
    const bool held = T.upos[m] < 0;
    double d1[3] = {0.0, 0.0, 0.0};
    if (!held) drift_inflow3(D1, m, d1);
    for (int s = 0; s < 3; ++s)
      v[s] = ((x0[s * WO + o0 + m] + k.delta_dt * K0[S.rk_x + s * O + m]) +
              k.omdelta_dt * K1[S.rk_x + s * O + m]) +
             omgamma_dt * (held ? 0.0 : d1[s]);
  };
  // The Newton's next right-hand side: -R for an active world, 0 otherwise.
  auto newton_rhs = [&](bool active) {
    for (int u = tid; u < U; u += BLOCK) Y[u] = active ? -Rv[u] : 0.0;
    if (active && tid == 0) atomicOr(any_active, 1);
    __syncthreads();
  };

  if (phase == PH_START) {
    // ---- start concentrations, face weights, base potentials, the initial offsets' rhs --------
    if (tid == 0) {
      if (first) ctl[6] = 0.0;
      ctl[0] = 0.0;
      ctl[7] = 0.0;
    }
    unsigned bits = set_conc([&](int s, int i) { return n0[s * WN + c0 + i]; },
                             [&](int s, int m) { return x0[s * WO + o0 + m]; });
    __syncthreads();
    for (int f = tid; f < F; f += BLOCK) {
      const int a = T.fs[f], b = T.fr[f];
      for (int s = 0; s < 3; ++s) {
        double mean, lg;
        logmean(CO[s * O + a], CO[s * O + b], mean, lg);
        FM[s * F + f] = P.ff[s * WF + f0 + f] * mean;
        LD[s * F + f] = LCO[s * O + a] - LCO[s * O + b];
      }
    }
    // Base potentials: free nodes 0, held nodes their boundary; cells q_c / C_c above their node.
    for (int m = tid; m < O; m += BLOCK) PHI[m] = T.upos[m] < 0 ? P.vb[o0 + m] : 0.0;
    __syncthreads();
    double rmax, norm;
    evaluate(Rv, false, rmax, norm);
    for (int u = tid; u < U; u += BLOCK) Y[u] = -Rv[u];
    bits_out(bits);
    return;
  }
  if (phase == PH_NEWTON_INIT || phase == PH_NEWTON_SEARCH) {
    // ---- the start field: Newton on the free nodes' potentials (the floating offsets) -------
    if (phase == PH_NEWTON_INIT) {
      unsigned bits = bits_in() | (ctl[7] != 0.0 ? (unsigned)CB_WORLD_FIELD : 0u);
      set_phi(X);
      double rmax, norm;
      const bool accepted = evaluate(Rv, true, rmax, norm);
      const bool active = accepted && norm > kNewtonTarget;
      __syncthreads();
      if (tid == 0) {
        ctl[1] = 0.0;
        ctl[2] = accepted ? 1.0 : 0.0;
        ctl[3] = active ? 1.0 : 0.0;
        ctl[4] = norm;
        ctl[5] = rmax;
      }
      newton_rhs(active);
      bits_out(bits);
      return;
    }
    if (ctl[3] == 0.0) {  // converged or stopped: keep the next solve's rhs at zero
      newton_rhs(false);
      return;
    }
    // One correction (DX, solved by the host's level launches) with its backtracking line search.
    const double before = ctl[5];
    double norm = ctl[4], tmax = 0.0, tnorm = norm;
    bool ok = false;
    for (int bt = 0; bt < kMaxBacktracks && !ok; ++bt) {
      const double h = ldexp(1.0, -bt);
      for (int u = tid; u < U; u += BLOCK) XT[u] = X[u] + DX[u] * h;
      __syncthreads();
      set_phi(XT);
      const bool valid = evaluate(RTv, true, tmax, tnorm);
      ok = valid && (tmax < before || tnorm <= kNewtonTarget);
    }
    norm = tnorm;
    double rmax = before;
    if (ok) {
      for (int u = tid; u < U; u += BLOCK) {
        X[u] = XT[u];
        Rv[u] = RTv[u];
      }
      rmax = tmax;
    }
    __syncthreads();
    const int count = (int)ctl[1] + 1;
    const bool active = count < kMaxIterations && norm > kNewtonTarget && ok;
    __syncthreads();
    if (tid == 0) {
      ctl[1] = (double)count;
      ctl[2] = ok ? 1.0 : 0.0;
      ctl[3] = active ? 1.0 : 0.0;
      ctl[4] = norm;
      ctl[5] = rmax;
    }
    newton_rhs(active);
    return;
  }
  if (phase == PH_AFTER_NEWTON) {
    // ctl[7]: a pivot or a staged copy that failed in the start field's factor or solves.
    unsigned bits = bits_in() | (ctl[7] != 0.0 ? (unsigned)CB_WORLD_FIELD : 0u);
    set_phi(X);
    {
      double rm2, n2;
      const bool valid = evaluate(Rv, true, rm2, n2);
      if (!(valid && ctl[2] != 0.0 && n2 <= kNewtonTarget)) bits |= CB_WORLD_FIELD;
    }
    // ---- stage 0: explicit rates at the start potentials ---------------------------------
    bits |= explicit_rates(K0, [&](int e) { return g0[e]; }, true);
    // The readouts' extracellular rate (membrane flux, whole face flux at the start field, the
    // pump's transfer) and the half-step prediction of the node concentrations.
    for (int m = tid; m < O; m += BLOCK) {
      const int i = T.ncell[m];
      const bool held = T.upos[m] < 0;
      double outs[3] = {0.0, 0.0, 0.0}, ins[3] = {0.0, 0.0, 0.0};
      for (int q = T.nf_ptr[m]; q < T.nf_ptr[m + 1]; ++q) {
        const int code = T.nf_idx[q], f = code >> 1;
        const double dv = PHI[T.fs[f]] - PHI[T.fr[f]];
        for (int s = 0; s < 3; ++s) {
          const double z = s < 2 ? 1.0 : -1.0;
          const double mu = RT * LD[s * F + f] + z * kF * dv;
          const double flux = FM[s * F + f] * mu / (RT * 1e-15);
          if (code & 1) ins[s] += flux;
          else outs[s] += flux;
        }
      }
      for (int s = 0; s < 3; ++s) {
        double a = 0.0;
        if (i >= 0) a = 0.0 + K0[S.rk_mt + s * N + i];
        double rate = held ? 0.0 : (a - outs[s]) + ins[s];
        if (!held && i >= 0) rate = rate + K0[S.rk_ex + s * N + i];
        const double amount = P.oref[s * WO + o0 + m] +
                              st(CB_FIELD_EXTRACELLULAR_INCREMENT)[s * WO + o0 + m];
        const double pred = (amount + (0.5 * dt) * rate) / P.ovol[o0 + m];
        if (!(is_finite(pred) && pred > 0.0)) bits |= CB_WORLD_OPERATOR;
        CP[s * O + m] = pred > 0.0 ? pred : 1.0;
      }
    }
    __syncthreads();
    // Frozen face weights at the prediction, and the operator gamma dt L(W).
    for (int f = tid; f < F; f += BLOCK) {
      const int a = T.fs[f], b = T.fr[f];
      for (int s = 0; s < 3; ++s) {
        double mean, lg;
        logmean(CP[s * O + a], CP[s * O + b], mean, lg);
        WP[s * F + f] = P.ff[s * WF + f0 + f] * mean / 1e-15;
      }
    }
    __syncthreads();
    __syncthreads();
    if (tid == 0) ctl[7] = 0.0;  // the operator factor's pivot flag
    stage_rhs(known1_cell, known1_node3);
    bits_out(bits);
    return;
  }
  if (phase == PH_STAGE1) {
    unsigned bits = bits_in() | (ctl[7] != 0.0 ? (unsigned)CB_WORLD_OPERATOR : 0u);
    bits |= stage_post(known1_cell);
    drift(D1);
    for (int i = tid; i < N; i += BLOCK)
      for (int s = 0; s < 3; ++s) N1[s * N + i] = known1_cell(s, i);
    for (int m = tid; m < O; m += BLOCK) {
      const bool held = T.upos[m] < 0;
      double d1[3] = {0.0, 0.0, 0.0};
      if (!held) drift_inflow3(D1, m, d1);
      for (int s = 0; s < 3; ++s)
        O1[s * O + m] = known1_node(s, m) + k.gamma_dt * (held ? 0.0 : d1[s]);
    }
    for (int e = tid; e < E; e += BLOCK) G1[e] = g0[e] + k.gamma_dt * K0[S.rk_g + e];
    __syncthreads();
    bits |= set_conc([&](int s, int i) { return N1[s * N + i]; },
                     [&](int s, int m) { return O1[s * O + m]; });
    __syncthreads();
    bits |= explicit_rates(K1, [&](int e) { return G1[e]; }, false);
    stage_rhs(known2_cell, known2_node3);
    bits_out(bits);
    return;
  }
  // PH_FINISH: the stage-2 solution, its drift, the step's end.
  {
    unsigned bits = bits_in() | (ctl[7] != 0.0 ? (unsigned)CB_WORLD_OPERATOR : 0u);
    bits |= stage_post(known2_cell);
    drift(D2);
    // ---- the step's end: ledgers, heat, domain; write or refuse ---------------------------
    unsigned dom = 0;
    const double gdt = k.gamma_dt, ddt = k.delta_dt, odt = k.omdelta_dt;
    const double dl = k.delta, od = k.omdelta, gm = 1.0 - 1.0 / sqrt(2.0), og = 1.0 - gm;
    // Cells.
    // The final amounts go to N1 / O1 (no longer needed) for the write below.
    for (int i = tid; i < N; i += BLOCK) {
      for (int s = 0; s < 3; ++s) {
        const double v = known2_cell(s, i);
        N1[s * N + i] = v;
        if (!(is_finite(v) && P.ref[s * WN + c0 + i] + v > 0.0)) dom = 1u;
      }
      for (int s = 0; s < 3; ++s) {
        const double v = (st(CB_FIELD_MEMBRANE_TRANSFERRED)[s * WN + c0 + i] +
                          ddt * K0[S.rk_mt + s * N + i]) + odt * K1[S.rk_mt + s * N + i];
        if (!is_finite(v)) dom = 1u;
      }
      const int f4[4] = {CB_FIELD_MEMBRANE_DISSIPATED, CB_FIELD_PUMP_CYCLES,
                         CB_FIELD_PUMP_DISSIPATED, CB_FIELD_METABOLIC_WORK};
      const long long r4[4] = {S.rk_md, S.rk_cy, S.rk_pd, S.rk_mw};
      for (int q = 0; q < 4; ++q) {
        const double v = (st(f4[q])[c0 + i] + ddt * K0[r4[q] + i]) + odt * K1[r4[q] + i];
        if (!is_finite(v)) dom = 1u;
      }
    }
    for (int e = tid; e < E; e += BLOCK) {
      for (int s = 0; s < 3; ++s) {
        const double v = (st(CB_FIELD_JUNCTION_TRANSFERRED)[s * WE + e0 + e] +
                          ddt * K0[S.rk_jt + s * E + e]) + odt * K1[S.rk_jt + s * E + e];
        if (!is_finite(v)) dom = 1u;
      }
      const double jd = (st(CB_FIELD_JUNCTION_DISSIPATED)[e0 + e] + ddt * K0[S.rk_jd + e]) +
                        odt * K1[S.rk_jd + e];
      const double g = (g0[e] + ddt * K0[S.rk_g + e]) + odt * K1[S.rk_g + e];
      if (!(is_finite(jd) && is_finite(g))) dom = 1u;
    }
    for (int m = tid; m < O; m += BLOCK) {
      const bool held = T.upos[m] < 0;
      double k2[3], d2[3] = {0.0, 0.0, 0.0};
      known2_node3(m, k2);
      if (!held) drift_inflow3(D2, m, d2);
      for (int s = 0; s < 3; ++s) {
        const double v = k2[s] + gdt * (held ? 0.0 : d2[s]);
        O1[s * O + m] = v;
        if (!(is_finite(v) && P.oref[s * WO + o0 + m] + v > 0.0)) dom = 1u;
      }
    }
    if (block_or<BLOCK>(dom, sBits)) bits |= CB_WORLD_DOMAIN;
    bits = block_or<BLOCK>(bits, sBits);
    if (bits) {
      if (tid == 0) status[w] = bits;
      return;
    }
    // Accepted: write the step in place, field by field (each from its own start value).
    for (int i = tid; i < N; i += BLOCK) {
      double nv[3];
      for (int s = 0; s < 3; ++s) nv[s] = N1[s * N + i];
      for (int s = 0; s < 3; ++s) {
        st(CB_FIELD_AMOUNT_INCREMENT)[s * WN + c0 + i] = nv[s];
        double *mt = st(CB_FIELD_MEMBRANE_TRANSFERRED) + s * WN + c0 + i;
        *mt = (*mt + ddt * K0[S.rk_mt + s * N + i]) + odt * K1[S.rk_mt + s * N + i];
      }
      const int f4[4] = {CB_FIELD_MEMBRANE_DISSIPATED, CB_FIELD_PUMP_CYCLES,
                         CB_FIELD_PUMP_DISSIPATED, CB_FIELD_METABOLIC_WORK};
      const long long r4[4] = {S.rk_md, S.rk_cy, S.rk_pd, S.rk_mw};
      for (int q = 0; q < 4; ++q) {
        double *v = st(f4[q]) + c0 + i;
        *v = (*v + ddt * K0[r4[q] + i]) + odt * K1[r4[q] + i];
      }
    }
    for (int e = tid; e < E; e += BLOCK) {
      for (int s = 0; s < 3; ++s) {
        double *v = st(CB_FIELD_JUNCTION_TRANSFERRED) + s * WE + e0 + e;
        *v = (*v + ddt * K0[S.rk_jt + s * E + e]) + odt * K1[S.rk_jt + s * E + e];
      }
      double *jd = st(CB_FIELD_JUNCTION_DISSIPATED) + e0 + e;
      *jd = (*jd + ddt * K0[S.rk_jd + e]) + odt * K1[S.rk_jd + e];
      double *g = st(CB_FIELD_JUNCTION_GATE) + e0 + e;
      *g = (*g + ddt * K0[S.rk_g + e]) + odt * K1[S.rk_g + e];
    }
    // Faces: transferred (explicit diffusion, both drifts), heat of the applied flux.
    for (int f = tid; f < F; f += BLOCK) {
      double heat = 0.0;
      for (int s = 0; s < 3; ++s) {
        const double k0d = K0[S.rk_fd + s * F + f], k1d = K1[S.rk_fd + s * F + f];
        const double d1 = D1[s * F + f], d2 = D2[s * F + f];
        double *v = st(CB_FIELD_FACE_TRANSFERRED) + s * WF + f0 + f;
        *v = (((*v + ddt * k0d) + odt * k1d) + omgamma_dt * d1) + gdt * d2;
        const double applied = ((0.0 + dl * k0d) + od * k1d) + ((0.0 + og * d1) + gm * d2);
        const double wgt = WP[s * F + f];
        heat += wgt > 0.0 ? applied * applied / wgt : 0.0;
      }
      double *fd = st(CB_FIELD_FACE_DISSIPATED) + f0 + f;
      *fd = *fd + dt * (1e-3 * kR * temp * heat);
    }
    // Nodes: amounts (free), supply and reservoir work (held); the held nodes face no capacitor,
    // so their electrodes deliver nothing (electrode charge and work unchanged).
    for (int m = tid; m < O; m += BLOCK) {
      const bool held = T.upos[m] < 0;
      double nv[3], sup[3], h1[3] = {0.0, 0.0, 0.0}, h2[3] = {0.0, 0.0, 0.0};
      if (held) {
        drift_inflow3(D1, m, h1);
        drift_inflow3(D2, m, h2);
      }
      for (int s = 0; s < 3; ++s) {
        nv[s] = O1[s * O + m];
        const double i1 = held ? -h1[s] : 0.0;
        const double i2 = held ? -h2[s] : 0.0;
        const double k0s = K0[S.rk_s + s * O + m], k1s = K1[S.rk_s + s * O + m];
        double *v = st(CB_FIELD_RESERVOIR_SUPPLIED) + s * WO + o0 + m;
        *v = (((*v + ddt * k0s) + odt * k1s) + omgamma_dt * i1) + gdt * i2;
        sup[s] = ((0.0 + dl * k0s) + od * k1s) + ((0.0 + og * i1) + gm * i2);
      }
      for (int s = 0; s < 3; ++s) st(CB_FIELD_EXTRACELLULAR_INCREMENT)[s * WO + o0 + m] = nv[s];
      if (held) {
        const double vb = P.vb[o0 + m];
        double work = 0.0;
        for (int s = 0; s < 3; ++s) {
          const double z = s < 2 ? 1.0 : -1.0;
          const double co = P.oref[s * WO + o0 + m] / P.ovol[o0 + m];
          const double mu = kR * temp * log(co) + z * kF * vb;
          work += mu * (dt * sup[s]);
        }
        double *rw = st(CB_FIELD_RESERVOIR_WORK) + o0 + m;
        *rw = *rw + 1e-3 * work;
      }
    }
    __syncthreads();
    if (tid == 0) {
      ctl[6] = ctl[6] + 1.0;
      if (taken_out) taken_out[w] = (int32_t)ctl[6];
    }
  }
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// Host

struct cb_field {
  int device = 0;
  int W = 0, N = 0, O = 0, E = 0, F = 0, U = 0, levels = 0;
  long long lsize = 0, usize = 0, vsize = 0, smem_doubles = 0;
  int supernodes = 0;
  // Levels of the fronts (host copies): first entry in lv_sn, one warp per front, the largest
  // block (m x s) and front rows.
  std::vector<int> lv_ptr, lv_warp, lv_wide, lv_block, lv_m;
  double factor_flops = 0.0, solve_flops = 0.0;  // per world: one factorisation, one solve
  long long launches = 0;   // kernels launched by the last cb_field_step
  long long solves = 0, factorisations = 0;  // ... and the solves and factorisations it ran
  double *host_state = nullptr, *host_control = nullptr;  // cb_field_step_host's device copies
  uint32_t *host_status = nullptr;
  int32_t *host_taken = nullptr;
  int *any = nullptr;       // device: some world's Newton goes on
  int *any_host = nullptr;  // pinned copy
  Topo topo{};
  Params params{};
  FLayout layout{};
  Scratch scratch{};
  long long state_total = 0;
  double *scratch_buf = nullptr;
  std::vector<void *> owned;
};

namespace {

template <typename V>
int upload(cb_field *f, const V *host, size_t count, V **dst) {
  void *p = nullptr;
  const size_t bytes = std::max<size_t>(count, 1) * sizeof(V);
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
  f->owned.push_back(p);
  if (count) {
    e = cudaMemcpy(p, host, count * sizeof(V), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy");
  }
  *dst = static_cast<V *>(p);
  return CB_OK;
}

template <typename V>
int upload(cb_field *f, const std::vector<V> &host, const V **dst) {
  V *p = nullptr;
  const int rc = upload(f, host.data(), host.size(), &p);
  *dst = p;
  return rc;
}

double host_logaddexp0(double y) {
  if (y == 0.0) return 0.6931471805599453;
  if (-y > 0) return std::log1p(std::exp(y));
  return y + std::log1p(std::exp(-y));
}

// Nested dissection of the free nodes of a side x side grid whose held nodes are its ring: the
// free box (side - 2)^2, split across its longer side by a middle line, the line last.
// Each leaf block (at most kLeafNodes nodes) becomes one relaxed supernode: group gets its id for
// the block's columns, -1 for separator columns.
constexpr int kLeafNodes = 16;
void nested_dissection(int x0, int x1, int y0, int y1, int width, std::vector<int> &order,
                       std::vector<int> &group, int &groups) {
  const int w = x1 - x0, h = y1 - y0;
  if (w <= 0 || h <= 0) return;
  if (w * h <= kLeafNodes) {
    for (int y = y0; y < y1; ++y)
      for (int x = x0; x < x1; ++x) {
        order.push_back(y * width + x);
        group.push_back(groups);
      }
    ++groups;
    return;
  }
  if (w >= h) {
    const int mid = x0 + w / 2;
    nested_dissection(x0, mid, y0, y1, width, order, group, groups);
    nested_dissection(mid + 1, x1, y0, y1, width, order, group, groups);
    for (int y = y0; y < y1; ++y) {
      order.push_back(y * width + mid);
      group.push_back(-1);
    }
  } else {
    const int mid = y0 + h / 2;
    nested_dissection(x0, x1, y0, mid, width, order, group, groups);
    nested_dissection(x0, x1, mid + 1, y1, width, order, group, groups);
    for (int x = x0; x < x1; ++x) {
      order.push_back(mid * width + x);
      group.push_back(-1);
    }
  }
}

}  // namespace

extern "C" int cb_field_bind(const cb_field_desc *d, int device, cb_field **out) {
  if (!d || !out) return fail(CB_ERR_ARGUMENT, "null argument");
  *out = nullptr;
  const int W = d->worlds, N = d->cells, O = d->nodes, E = d->junctions, F = d->faces;
  if (W <= 0 || N < 0 || O <= 0 || E < 0 || F < 0)
    return fail(CB_ERR_ARGUMENT, "field: sizes must be positive");
  for (const void *p : {(const void *)d->cell_node, (const void *)d->face_sender,
                        (const void *)d->face_receiver, (const void *)d->reservoir,
                        (const void *)d->temperature, (const void *)d->pump,
                        (const void *)d->volume, (const void *)d->capacitance,
                        (const void *)d->permeability, (const void *)d->pump_capacity,
                        (const void *)d->amount, (const void *)d->initial_charge,
                        (const void *)d->outside_volume, (const void *)d->outside_amount,
                        (const void *)d->outside_charge, (const void *)d->boundary_V,
                        (const void *)d->face_factor, (const void *)d->area})
    if (!p) return fail(CB_ERR_ARGUMENT, "field: null array");
  if (E && (!d->junction_sender || !d->junction_receiver || !d->junction_area ||
            !d->junction_permeability || !d->gate_threshold || !d->gate_minimum))
    return fail(CB_ERR_ARGUMENT, "field: null junction array");
  // Topology checks: the contract the eliminated algebra rests on.
  std::vector<int> ncell(O, -1), cell_node(N);
  for (int i = 0; i < N; ++i) {
    const long long m = d->cell_node[i];
    if (m < 0 || m >= O) return fail(CB_ERR_LAYOUT, "field: cell_node out of range");
    if (d->reservoir[m]) return fail(CB_ERR_LAYOUT, "field: a cell faces a held node");
    if (ncell[m] >= 0) return fail(CB_ERR_LAYOUT, "field: two cells face one node");
    ncell[m] = i;
    cell_node[i] = (int)m;
  }
  std::vector<int> fs(F), fr(F), js(E), jr(E);
  for (int f = 0; f < F; ++f) {
    const long long a = d->face_sender[f], b = d->face_receiver[f];
    if (a < 0 || a >= O || b < 0 || b >= O || a == b)
      return fail(CB_ERR_LAYOUT, "field: a face's nodes are out of range or equal");
    fs[f] = (int)a;
    fr[f] = (int)b;
  }
  for (int e = 0; e < E; ++e) {
    const long long a = d->junction_sender[e], b = d->junction_receiver[e];
    if (a < 0 || a >= N || b < 0 || b >= N || a == b)
      return fail(CB_ERR_LAYOUT, "field: a junction's cells are out of range or equal");
    js[e] = (int)a;
    jr[e] = (int)b;
  }
  // Free nodes, the Laplacian's graph (faces between free nodes), its order.
  std::vector<int> free_index(O, -1), free_nodes;
  for (int m = 0; m < O; ++m)
    if (!d->reservoir[m]) {
      free_index[m] = (int)free_nodes.size();
      free_nodes.push_back(m);
    }
  const int U = (int)free_nodes.size();
  if (U == 0) return fail(CB_ERR_LAYOUT, "field: no free node");
  std::vector<int> ga, gb, gface;
  std::vector<char> touches_held(U, 0);
  for (int f = 0; f < F; ++f) {
    const int a = free_index[fs[f]], b = free_index[fr[f]];
    if (a >= 0 && b >= 0) {
      ga.push_back(a);
      gb.push_back(b);
      gface.push_back(f);
    } else if (a >= 0) {
      touches_held[a] = 1;
    } else if (b >= 0) {
      touches_held[b] = 1;
    }
  }
  // Every free node must reach a held node through faces (the reference's return-path rule),
  // or the Laplacian is singular.
  {
    std::vector<std::vector<int>> adj(U);
    for (size_t q = 0; q < ga.size(); ++q) {
      adj[ga[q]].push_back(gb[q]);
      adj[gb[q]].push_back(ga[q]);
    }
    std::vector<char> seen(U, 0);
    std::vector<int> stack;
    for (int u = 0; u < U; ++u)
      if (touches_held[u]) {
        seen[u] = 1;
        stack.push_back(u);
      }
    while (!stack.empty()) {
      const int u = stack.back();
      stack.pop_back();
      for (int v : adj[u])
        if (!seen[v]) {
          seen[v] = 1;
          stack.push_back(v);
        }
    }
    for (int u = 0; u < U; ++u)
      if (!seen[u])
        return fail(CB_ERR_LAYOUT,
                    "field: a floating component has no face path to a held node");
  }
  // Grid detection: O = side^2 with the ring held and 4-neighbour faces -> nested dissection.
  std::vector<int> order;
  const int side = (int)std::lround(std::sqrt((double)O));
  bool grid = side * side == O && side >= 3 && F == 2 * side * (side - 1);
  if (grid) {
    for (int m = 0; m < O && grid; ++m) {
      const int x = m % side, y = m / side;
      const bool ring = x == 0 || y == 0 || x == side - 1 || y == side - 1;
      grid = (d->reservoir[m] != 0) == ring;
    }
    for (int f = 0; f < F && grid; ++f) {
      const int a = fs[f], b = fr[f];
      const int dx = std::abs(a % side - b % side), dy = std::abs(a / side - b / side);
      grid = dx + dy == 1;
    }
  }
  std::vector<int> group;
  if (grid) {
    std::vector<int> cells;
    int groups = 0;
    nested_dissection(0, side - 2, 0, side - 2, side - 2, cells, group, groups);
    // cells index the free box row-major; map to free-node indices.
    for (int c : cells) {
      const int x = c % (side - 2) + 1, y = c / (side - 2) + 1;
      order.push_back(free_index[y * side + x]);
    }
  }
  WorldPlan plan;
  int rc = plan_world(U, ga.data(), gb.data(), (int)ga.size(), plan,
                      grid ? order.data() : nullptr, "field");
  if (rc) return rc;
  cudaError_t ce = cudaSetDevice(device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
  auto *f = new cb_field();
  f->device = device;
  f->W = W, f->N = N, f->O = O, f->E = E, f->F = F, f->U = U;
  auto bail = [&](int code) {
    cb_field_free(f);
    return code;
  };
  // Shared topology.
  std::vector<int> upos(O, -1);
  for (int u = 0; u < U; ++u) upos[free_nodes[u]] = plan.rank[u];
  std::vector<int> nf_ptr(O + 1, 0), nf_idx;
  {
    std::vector<std::vector<int>> lists(O);
    for (int q = 0; q < F; ++q) {
      lists[fs[q]].push_back(q << 1);
      lists[fr[q]].push_back((q << 1) | 1);
    }
    for (int m = 0; m < O; ++m) {
      nf_ptr[m + 1] = nf_ptr[m] + (int)lists[m].size();
      nf_idx.insert(nf_idx.end(), lists[m].begin(), lists[m].end());
    }
  }
  std::vector<int> cj_ptr(N + 1, 0), cj_idx;
  {
    std::vector<std::vector<int>> lists(N);
    for (int e = 0; e < E; ++e) {
      lists[js[e]].push_back(e << 1);
      lists[jr[e]].push_back((e << 1) | 1);
    }
    for (int i = 0; i < N; ++i) {
      cj_ptr[i + 1] = cj_ptr[i] + (int)lists[i].size();
      cj_idx.insert(cj_idx.end(), lists[i].begin(), lists[i].end());
    }
  }
  // Supernodes and each front's face entries (row = the later column, column = the earlier).
  SuperPlan sp;
  if ((rc = build_supernodes(plan, sp, grid ? &group : nullptr))) return bail(rc);
  // Fewer levels: fronts merged into their parents where that adds at most 5% zeros and keeps
  // the front within 16384 entries (the 126-column root of the 128x128 grid is 15876).
  if ((rc = amalgamate(plan, sp, 0.05, 16384))) return bail(rc);
  std::vector<int> col_node(U), af_ptr(sp.count + 1, 0), af_face, af_pos;
  for (int u = 0; u < U; ++u) col_node[plan.rank[u]] = free_nodes[u];
  {
    std::vector<std::vector<std::pair<int, int>>> lists(sp.count);
    for (size_t q = 0; q < gface.size(); ++q) {
      const int ra = plan.rank[ga[q]], rb = plan.rank[gb[q]];
      const int col = std::min(ra, rb), row = std::max(ra, rb);
      const int sn = sp.sn_of[col];
      const int *rq = sp.rows.data() + sp.rows_ptr[sn];
      const int *at = std::lower_bound(rq, rq + sp.m[sn], row);
      if (at == rq + sp.m[sn] || *at != row) return bail(fail(CB_ERR_LAYOUT, "field: face outside its front"));
      lists[sn].push_back({gface[q], (int)(at - rq) + (col - sp.c0[sn]) * sp.m[sn]});
    }
    for (int q = 0; q < sp.count; ++q) {
      for (auto &pr : lists[q]) {
        af_face.push_back(pr.first);
        af_pos.push_back(pr.second);
      }
      af_ptr[q + 1] = (int)af_face.size();
    }
  }
  // A level's fronts go one per warp (their blocks and rows small) or one per CTA. Override for
  // sweeps: CELLS_B200_FIELD_WARP_BLOCK (the largest block, in doubles, a warp takes).
  long long warp_block = kWarpBlock;
  if (const char *env = std::getenv("CELLS_B200_FIELD_WARP_BLOCK"))
    warp_block = std::max(1, std::min(std::atoi(env), kWarpBlock));
  f->lv_ptr = sp.lv_ptr;
  f->lv_warp.assign(sp.levels, 0);
  f->lv_wide.assign(sp.levels, 0);
  f->lv_block.assign(sp.levels, 0);
  f->lv_m.assign(sp.levels, 0);
  for (int l = 0; l < sp.levels; ++l) {
    long long mb = 0;
    int mm = 0, ms = 0;
    for (int a = sp.lv_ptr[l]; a < sp.lv_ptr[l + 1]; ++a) {
      const int q = sp.lv_sn[a];
      mb = std::max(mb, (long long)sp.m[q] * sp.s[q]);
      mm = std::max(mm, sp.m[q]);
      ms = std::max(ms, sp.s[q]);
    }
    f->lv_block[l] = (int)mb;
    f->lv_m[l] = mm;
    f->lv_warp[l] = (mb <= warp_block && mm <= kWarpVector) ? 1 : 0;
    f->lv_wide[l] = (!f->lv_warp[l] && ms >= kWideColumns) ? 1 : 0;
    const long long need =
        f->lv_warp[l] ? (long long)kWarpsPerCta * level_slice(mb, mm) : level_vec(mb) + mm;
    f->smem_doubles = std::max(f->smem_doubles, need);
  }
  if (f->smem_doubles * (long long)sizeof(double) > kMaxSmemBytes)
    return bail(fail(CB_ERR_UNSUPPORTED, "field: a front exceeds shared memory"));
  // Arithmetic of the plan per world (FMA = 2 flops): the panel's scaling and right-looking
  // update, the update matrix (packed lower triangle), and one FMA per factor entry each way of a
  // solve.
  for (int q = 0; q < sp.count; ++q) {
    const double sq = sp.s[q], mq = sp.m[q], bq = mq - sq;
    for (int k = 0; k < sp.s[q]; ++k) {
      f->factor_flops += mq - k - 1;
      for (int j = k + 1; j < sp.s[q]; ++j) f->factor_flops += 2.0 * (mq - j);
    }
    f->factor_flops += bq * (bq + 1.0) * sq;
    f->solve_flops += 4.0 * (mq * sq - sq * (sq - 1.0) / 2.0);
  }
  f->levels = sp.levels;
  f->supernodes = sp.count;
  f->lsize = sp.lsize, f->usize = sp.usize, f->vsize = sp.vsize;
  Topo &T = f->topo;
  T.N = N, T.O = O, T.E = E, T.F = F, T.U = U, T.levels = sp.levels;
  std::vector<int> sn_c0 = sp.c0, sn_s = sp.s, sn_m = sp.m;
  if ((rc = upload(f, cell_node, &T.cell_node)) || (rc = upload(f, ncell, &T.ncell)) ||
      (rc = upload(f, upos, &T.upos)) || (rc = upload(f, nf_ptr, &T.nf_ptr)) ||
      (rc = upload(f, nf_idx, &T.nf_idx)) || (rc = upload(f, cj_ptr, &T.cj_ptr)) ||
      (rc = upload(f, cj_idx, &T.cj_idx)) || (rc = upload(f, fs, &T.fs)) ||
      (rc = upload(f, fr, &T.fr)) || (rc = upload(f, js, &T.js)) ||
      (rc = upload(f, jr, &T.jr)) || (rc = upload(f, col_node, &T.col_node)) ||
      (rc = upload(f, sn_c0, &T.sn_c0)) || (rc = upload(f, sn_s, &T.sn_s)) ||
      (rc = upload(f, sn_m, &T.sn_m)) || (rc = upload(f, sp.loff, &T.sn_loff)) ||
      (rc = upload(f, sp.uoff, &T.sn_uoff)) || (rc = upload(f, sp.voff, &T.sn_voff)) ||
      (rc = upload(f, sp.rows_ptr, &T.rows_ptr)) || (rc = upload(f, sp.rows, &T.rows)) ||
      (rc = upload(f, sp.ch_ptr, &T.ch_ptr)) || (rc = upload(f, sp.ch, &T.ch)) ||
      (rc = upload(f, sp.map_ptr, &T.map_ptr)) || (rc = upload(f, sp.map, &T.map)) ||
      (rc = upload(f, sp.split, &T.split)) ||
      (rc = upload(f, sp.lv_ptr, &T.lv_ptr)) || (rc = upload(f, sp.lv_sn, &T.lv_sn)) ||
      (rc = upload(f, af_ptr, &T.af_ptr)) ||
      (rc = upload(f, af_face, &T.af_face)) || (rc = upload(f, af_pos, &T.af_pos)))
    return bail(rc);
  // Per-world parameters.
  const long long WN = (long long)W * N, WO = (long long)W * O, WE = (long long)W * E,
                  WF = (long long)W * F;
  Params &P = f->params;
  P.WN = WN, P.WO = WO, P.WE = WE, P.WF = WF;
  std::vector<double> wcv((size_t)W * FW_STRIDE);
  const double ln1000 = std::log(1000.0);
  for (int w = 0; w < W; ++w) {
    double *c = wcv.data() + (size_t)w * FW_STRIDE;
    const double Tk = d->temperature[w], RT = kR * Tk;
    c[FW_T] = Tk;
    c[FW_RT] = RT;
    c[FW_FRT] = kF / RT;
    c[FW_INVRT] = 1.0 / RT;
    const double atp = d->pump[0 * W + w], adp = d->pump[1 * W + w], pi = d->pump[2 * W + w];
    const double km_na = d->pump[3 * W + w], km_k = d->pump[4 * W + w];
    const double km_atp = d->pump[5 * W + w], dg0 = d->pump[6 * W + w];
    c[FW_DRIVE] = dg0 + RT * (((std::log(adp) + std::log(pi)) - std::log(atp)) - ln1000);
    c[FW_LOGKMK] = std::log(km_k);
    c[FW_LATP] = host_logaddexp0(std::log(km_atp) - std::log(atp));
    c[FW_LOGKMNA] = std::log(km_na);
    const bool t_ok = std::isfinite(Tk) && Tk >= 200.0 && Tk <= 400.0;
    const double rtd = kR * (t_ok ? Tk : 298.15);
    bool ok = t_ok;
    for (double v : {atp, adp, pi, km_na, km_k, km_atp}) ok = ok && std::isfinite(v) && v > 0;
    ok = ok && std::isfinite(dg0);
    const double s_atp = ok ? atp : 1.0, s_adp = ok ? adp : 1.0, s_pi = ok ? pi : 1.0;
    c[FW_AFF0] = (((dg0 / rtd + std::log(s_adp)) + std::log(s_pi)) - std::log(s_atp)) - ln1000;
    c[FW_PUMPOK] = ok ? 1.0 : 0.0;
    c[FW_INVRTD] = 1.0 / rtd;
  }
  std::vector<double> icap(WN), logpcap(WN), ap(3 * WN), jap(3 * WE);
  for (long long i = 0; i < WN; ++i) {
    icap[i] = 1.0 / d->capacitance[i];
    logpcap[i] = d->pump_capacity[i] > 0 ? std::log(d->pump_capacity[i]) : 0.0;
    for (int s = 0; s < 3; ++s)
      ap[s * WN + i] = d->area[i] * d->permeability[s * WN + i] / 1e-15;
  }
  for (long long e = 0; e < WE; ++e)
    for (int s = 0; s < 3; ++s)
      jap[s * WE + e] = d->junction_area[e] * d->junction_permeability[s * WE + e] / 1e-15;
  double *tmp = nullptr;
  auto put = [&](const double *src, size_t count, const double **dst) {
    int r = upload(f, src, count, &tmp);
    *dst = tmp;
    return r;
  };
  if ((rc = upload(f, wcv, &P.wc)) || (rc = put(d->volume, WN, &P.vol)) ||
      (rc = upload(f, icap, &P.icap)) || (rc = put(d->initial_charge, WN, &P.q0)) ||
      (rc = put(d->pump_capacity, WN, &P.pcap)) || (rc = upload(f, logpcap, &P.logpcap)) ||
      (rc = put(d->amount, 3 * WN, &P.ref)) || (rc = upload(f, ap, &P.ap)) ||
      (rc = upload(f, jap, &P.jap)) || (rc = put(E ? d->gate_threshold : nullptr, WE, &P.thr)) ||
      (rc = put(E ? d->gate_minimum : nullptr, WE, &P.jmin)) ||
      (rc = put(d->outside_volume, WO, &P.ovol)) || (rc = put(d->outside_charge, WO, &P.q0o)) ||
      (rc = put(d->boundary_V, WO, &P.vb)) || (rc = put(d->outside_amount, 3 * WO, &P.oref)) ||
      (rc = put(d->face_factor, 3 * WF, &P.ff)))
    return bail(rc);
  // State layout.
  const long long sizes[CB_FIELD_STATE_FIELDS] = {3 * WN, 3 * WO, 3 * WN, 3 * WE, 3 * WF, 3 * WO,
                                                  WN, WE, WF, WO, WO, WO, WE, WN, WN, WN};
  long long off = 0;
  for (int q = 0; q < CB_FIELD_STATE_FIELDS; ++q) {
    f->layout.s[q] = off;
    off += sizes[q];
  }
  f->state_total = off;
  // Scratch slices.
  Scratch &S = f->scratch;
  long long o = 0;
  auto take = [&](long long n) {
    const long long at = o;
    o += (n + 31) / 32 * 32;  // 256-byte aligned sub-arrays
    return at;
  };
  S.rk_n = 0;
  S.rk_mt = 3LL * N;
  S.rk_md = 6LL * N;
  S.rk_cy = 7LL * N;
  S.rk_pd = 8LL * N;
  S.rk_mw = 9LL * N;
  S.rk_jt = 10LL * N;
  S.rk_jd = S.rk_jt + 3LL * E;
  S.rk_g = S.rk_jd + E;
  S.rk_fd = S.rk_g + E;
  S.rk_x = S.rk_fd + 3LL * F;
  S.rk_s = S.rk_x + 3LL * O;
  S.rk_ex = S.rk_s + 3LL * O;
  S.rk_size = S.rk_ex + 3LL * N;
  S.lval = take(f->lsize), S.uf = take(f->usize), S.wv = take(std::max(f->vsize, 1LL));
  // The solves stage each front block with a TMA bulk copy: its global start must be 16-byte
  // aligned (world slices and sub-arrays are 256-byte aligned; blocks start at even offsets).
  for (int q = 0; q < sp.count; ++q)
    if (sp.loff[q] % 2 != 0) return bail(fail(CB_ERR_LAYOUT, "field: a factor block is not 16-byte aligned"));
  S.ctl = take(8);
  S.x = take(U), S.xt = take(U), S.dx = take(U), S.r = take(U), S.rt = take(U), S.y = take(U);
  S.phi = take(O), S.pc = take(N);
  S.co = take(3LL * O), S.lco = take(3LL * O), S.ci = take(3LL * N), S.lci = take(3LL * N);
  S.fm = take(3LL * F), S.ld = take(3LL * F), S.wp = take(3LL * F);
  S.ifc = take(F), S.ijc = take(std::max(E, 1));
  S.k0 = take(S.rk_size), S.k1 = take(S.rk_size);
  S.d1 = take(3LL * F), S.d2 = take(3LL * F);
  S.n1 = take(3LL * N), S.o1 = take(3LL * O), S.g1 = take(std::max(E, 1));
  S.cp = take(3LL * O);
  S.stride = o;
  {
    void *p = nullptr;
    ce = cudaMalloc(&p, (size_t)S.stride * W * sizeof(double));
    if (ce != cudaSuccess) {
      cuda_fail(ce, "cudaMalloc field scratch");
      return bail(CB_ERR_CUDA);
    }
    f->owned.push_back(p);
    f->scratch_buf = static_cast<double *>(p);
  }
  {
    void *p = nullptr;
    if ((ce = cudaMalloc(&p, sizeof(int))) != cudaSuccess) {
      cuda_fail(ce, "cudaMalloc");
      return bail(CB_ERR_CUDA);
    }
    f->owned.push_back(p);
    f->any = static_cast<int *>(p);
    if ((ce = cudaMallocHost(&p, sizeof(int))) != cudaSuccess) {
      cuda_fail(ce, "cudaMallocHost");
      return bail(CB_ERR_CUDA);
    }
    f->any_host = static_cast<int *>(p);
  }
  for (const void *fn : {(const void *)factor_warps, (const void *)factor_group<false>,
                         (const void *)factor_group<true>, (const void *)forward_warps, (const void *)forward_group,
                         (const void *)backward_warps, (const void *)backward_group})
    if ((ce = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)kMaxSmemBytes)) != cudaSuccess) {
      cuda_fail(ce, "cudaFuncSetAttribute");
      return bail(CB_ERR_CUDA);
    }
  *out = f;
  return CB_OK;
}

extern "C" void cb_field_free(cb_field *f) {
  if (!f) return;
  cudaSetDevice(f->device);
  for (void *p : f->owned) cudaFree(p);
  if (f->any_host) cudaFreeHost(f->any_host);
  delete f;
}

extern "C" int cb_field_state_layout(const cb_field *f, int64_t offsets[CB_FIELD_STATE_FIELDS],
                                     int64_t *total) {
  if (!f || !offsets || !total) return fail(CB_ERR_ARGUMENT, "null argument");
  for (int q = 0; q < CB_FIELD_STATE_FIELDS; ++q) offsets[q] = f->layout.s[q];
  *total = f->state_total;
  return CB_OK;
}

extern "C" int cb_field_info(const cb_field *f, int64_t info[8]) {
  if (!f || !info) return fail(CB_ERR_ARGUMENT, "null argument");
  info[0] = f->U;
  info[1] = f->supernodes;
  info[2] = f->levels;
  info[3] = f->lsize;
  info[4] = f->usize;
  info[5] = f->vsize;
  info[6] = f->smem_doubles * (int64_t)sizeof(double);
  info[7] = f->scratch.stride * (int64_t)f->W * (int64_t)sizeof(double);
  return CB_OK;
}

extern "C" int cb_field_flops(const cb_field *f, double out[2]) {
  if (!f || !out) return fail(CB_ERR_ARGUMENT, "null argument");
  out[0] = f->factor_flops;
  out[1] = f->solve_flops;
  return CB_OK;
}

extern "C" int32_t cb_field_levels(const cb_field *f, int32_t *kinds, int32_t capacity) {
  if (!f) return fail(CB_ERR_ARGUMENT, "null argument"), -1;
  for (int l = 0; l < f->levels && kinds && l < capacity; ++l)
    kinds[l] = f->lv_warp[l] ? 0 : f->lv_wide[l] ? 2 : 1;
  return f->levels;
}

extern "C" int64_t cb_field_launches(const cb_field *f) { return f ? f->launches : -1; }

extern "C" int cb_field_counts(const cb_field *f, int64_t out[3]) {
  if (!f || !out) return fail(CB_ERR_ARGUMENT, "null argument");
  out[0] = f->launches;
  out[1] = f->factorisations;
  out[2] = f->solves;
  return CB_OK;
}

extern "C" int64_t cb_field_control_length(const cb_field *f) {
  if (!f) return -1;
  return (long long)f->W * (2LL * f->N + f->E);
}

extern "C" int cb_field_step(cb_field *f, const double *state_in, double *state_out, double dt,
                             const double *control, int n_steps, uint32_t *world_status,
                             int32_t *accepted_steps, void *stream) {
  if (!f || !state_in || !state_out || !control || !world_status)
    return fail(CB_ERR_ARGUMENT, "null argument");
  if (n_steps < 0) return fail(CB_ERR_ARGUMENT, "n_steps must be non-negative");
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(CB_ERR_ARGUMENT, "dt must be positive");
  cudaError_t ce = cudaSetDevice(f->device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
  auto s = static_cast<cudaStream_t>(stream);
  if (state_out != state_in) {
    ce = cudaMemcpyAsync(state_out, state_in, (size_t)f->state_total * sizeof(double),
                         cudaMemcpyDeviceToDevice, s);
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaMemcpyAsync");
  }
  if ((ce = cudaMemsetAsync(world_status, 0, f->W * sizeof(uint32_t), s)) != cudaSuccess ||
      (accepted_steps &&
       (ce = cudaMemsetAsync(accepted_steps, 0, f->W * sizeof(int32_t), s)) != cudaSuccess))
    return cuda_fail(ce, "cudaMemsetAsync");
  const StepCoef k = step_coef(dt);
  const Topo &T = f->topo;
  const Scratch &S = f->scratch;
  double *sc = f->scratch_buf;
  f->launches = 0;
  f->solves = 0;
  f->factorisations = 0;
  auto phase = [&](int ph, int first) {
    ++f->launches;
    auto go = [&](auto kernel) {
      kernel<<<f->W, kFieldBlock, 0, s>>>(T, f->params, f->layout, S, state_out, control, k, first,
                                          world_status, accepted_steps, sc, f->any);
    };
    switch (ph) {
      case PH_START: go(field_phase<kFieldBlock, PH_START, kPhaseMinBlocks>); break;
      case PH_NEWTON_INIT: go(field_phase<kFieldBlock, PH_NEWTON_INIT, kPhaseMinBlocks>); break;
      case PH_NEWTON_SEARCH: go(field_phase<kFieldBlock, PH_NEWTON_SEARCH, kPhaseMinBlocks>); break;
      case PH_AFTER_NEWTON: go(field_phase<kFieldBlock, PH_AFTER_NEWTON, kPhaseMinBlocks>); break;
      case PH_STAGE1: go(field_phase<kFieldBlock, PH_STAGE1, kPhaseMinBlocks>); break;
      default: go(field_phase<kFieldBlock, PH_FINISH, kPhaseMinBlocks>); break;
    }
    return cudaGetLastError();
  };
  auto level_launch = [&](int l, auto warps, auto group) {
    const int a0 = f->lv_ptr[l], fronts = f->lv_ptr[l + 1] - a0;
    const int vec = (int)level_vec(f->lv_block[l]);
    ++f->launches;
    if (f->lv_warp[l]) {
      const int slice = (int)level_slice(f->lv_block[l], f->lv_m[l]);
      const long long tasks = (long long)fronts * f->W;
      const int ctas = (int)((tasks + kWarpsPerCta - 1) / kWarpsPerCta);
      warps(ctas, (size_t)kWarpsPerCta * slice * sizeof(double), a0, fronts, slice, vec);
    } else {
      group(dim3(fronts, f->W), (size_t)(vec + f->lv_m[l]) * sizeof(double), a0, vec);
    }
    return cudaGetLastError();
  };
  auto factor = [&](int kind) {
    ++f->factorisations;
    for (int l = 0; l < f->levels; ++l) {
      ce = level_launch(
          l,
          [&](int ctas, size_t smem, int a0, int fronts, int slice, int vec) {
            factor_warps<<<ctas, kWarpsPerCta * 32, smem, s>>>(T, f->params, S, sc, world_status,
                                                               kind, k.gamma_dt, a0, fronts, f->W,
                                                               slice, vec);
          },
          [&](dim3 grid, size_t smem, int a0, int vec) {
            auto kern = f->lv_wide[l] ? factor_group<true> : factor_group<false>;
            kern<<<grid, kGroupThreads, smem, s>>>(T, f->params, S, sc, world_status, kind,
                                                   k.gamma_dt, a0, vec);
          });
      if (ce != cudaSuccess) return ce;
    }
    return cudaSuccess;
  };
  auto solve = [&](long long out_off) {
    ++f->solves;
    for (int l = 0; l < f->levels; ++l) {
      ce = level_launch(
          l,
          [&](int ctas, size_t smem, int a0, int fronts, int slice, int vec) {
            forward_warps<<<ctas, kWarpsPerCta * 32, smem, s>>>(T, S, sc, world_status, a0,
                                                                fronts, f->W, slice, vec);
          },
          [&](dim3 grid, size_t smem, int a0, int vec) {
            forward_group<<<grid, kGroupThreads, smem, s>>>(T, S, sc, world_status, a0, vec);
          });
      if (ce != cudaSuccess) return ce;
    }
    for (int l = f->levels - 1; l >= 0; --l) {
      ce = level_launch(
          l,
          [&](int ctas, size_t smem, int a0, int fronts, int slice, int vec) {
            backward_warps<<<ctas, kWarpsPerCta * 32, smem, s>>>(T, S, sc, world_status, out_off,
                                                                 a0, fronts, f->W, slice, vec);
          },
          [&](dim3 grid, size_t smem, int a0, int vec) {
            backward_group<<<grid, kGroupThreads, smem, s>>>(T, S, sc, world_status, out_off, a0,
                                                             vec);
          });
      if (ce != cudaSuccess) return ce;
    }
    return cudaSuccess;
  };
  auto check = [&](cudaError_t e, const char *what) {
    return e == cudaSuccess ? CB_OK : cuda_fail(e, what);
  };
  int rc = CB_OK;
  for (int step = 0; step < n_steps && rc == CB_OK; ++step) {
    if ((rc = check(phase(PH_START, step == 0), "field start")) ||
        (rc = check(factor(0), "field factor")) || (rc = check(solve(S.x), "field solve")) ||
        (rc = check(cudaMemsetAsync(f->any, 0, sizeof(int), s), "cudaMemsetAsync")) ||
        (rc = check(phase(PH_NEWTON_INIT, 0), "field newton")))
      break;
    // The Newton's corrections while some world's goes on (one flag read back per correction).
    for (int it = 0; it < kMaxIterations && rc == CB_OK; ++it) {
      if ((rc = check(cudaMemcpyAsync(f->any_host, f->any, sizeof(int), cudaMemcpyDeviceToHost,
                                      s), "cudaMemcpyAsync")) ||
          (rc = check(cudaStreamSynchronize(s), "cudaStreamSynchronize")))
        break;
      if (*f->any_host == 0) break;
      if ((rc = check(solve(S.dx), "field solve")) ||
          (rc = check(cudaMemsetAsync(f->any, 0, sizeof(int), s), "cudaMemsetAsync")) ||
          (rc = check(phase(PH_NEWTON_SEARCH, 0), "field newton")))
        break;
    }
    if (rc) break;
    if ((rc = check(phase(PH_AFTER_NEWTON, 0), "field stage 0")) ||
        (rc = check(factor(1), "field factor")) || (rc = check(solve(S.x), "field solve")) ||
        (rc = check(phase(PH_STAGE1, 0), "field stage 1")) ||
        (rc = check(solve(S.x), "field solve")) ||
        (rc = check(phase(PH_FINISH, 0), "field finish")))
      break;
  }
  return rc;
}

extern "C" int cb_field_step_host(cb_field *f, const double *state_in, double *state_out,
                                  double dt, const double *control, int n_steps,
                                  uint32_t *world_status, int32_t *accepted_steps) {
  if (!f || !state_in || !state_out || !control || !world_status)
    return fail(CB_ERR_ARGUMENT, "null argument");
  cudaError_t ce = cudaSetDevice(f->device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
  const size_t sb = (size_t)f->state_total * sizeof(double);
  const size_t cb = (size_t)cb_field_control_length(f) * sizeof(double);
  // The device buffers of host calls: allocated by the handle's first host call, kept until
  // cb_field_free.
  if (!f->host_state) {
    void *p = nullptr;
    const size_t bytes = sb + cb + f->W * (sizeof(uint32_t) + sizeof(int32_t)) + 256;
    if ((ce = cudaMalloc(&p, bytes)) != cudaSuccess) return cuda_fail(ce, "cudaMalloc");
    f->owned.push_back(p);
    char *c = static_cast<char *>(p);
    f->host_state = reinterpret_cast<double *>(c);
    f->host_control = reinterpret_cast<double *>(c + sb);
    f->host_status = reinterpret_cast<uint32_t *>(c + sb + cb);
    f->host_taken = reinterpret_cast<int32_t *>(c + sb + cb + f->W * sizeof(uint32_t));
  }
  double *ds = f->host_state, *dc = f->host_control;
  uint32_t *dst = f->host_status;
  int32_t *dacc = f->host_taken;
  int rc = CB_OK;
  if ((ce = cudaMemcpy(ds, state_in, sb, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (ce = cudaMemcpy(dc, control, cb, cudaMemcpyHostToDevice)) != cudaSuccess) {
    rc = cuda_fail(ce, "cudaMemcpy");
  } else if ((rc = cb_field_step(f, ds, ds, dt, dc, n_steps, dst, dacc, nullptr)) == CB_OK) {
    if ((ce = cudaMemcpy(state_out, ds, sb, cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (ce = cudaMemcpy(world_status, dst, f->W * sizeof(uint32_t), cudaMemcpyDeviceToHost)) !=
            cudaSuccess ||
        (accepted_steps && (ce = cudaMemcpy(accepted_steps, dacc, f->W * sizeof(int32_t),
                                            cudaMemcpyDeviceToHost)) != cudaSuccess))
      rc = cuda_fail(ce, "cudaMemcpy");
  }
  return rc;
}
