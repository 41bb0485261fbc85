// n2_step.cu - the N2 step (CB_METHOD_N2): ARS(2,2,2) with the routes' slope conductances in the
// implicit operator, for held-bath worlds, and the batched sparse Cholesky it factors each step.
//
// Reference: models/surface_pump_v3.py:3547-3955 (imex_step under
// cells.solver.imex_ars222_implicit_conductances@1): operator_time_conductances :2961-3029,
// conductance_weights / route_slope :2741-2813 (bernoulli_slope of
// laws/routes/patch_electrodiffusion.py:43-54), conductance_laplacian :2816-2841,
// explicit_remainder :2925-2946, implicit_rates :2659-2700, implicit_route_heat :2949-2958,
// stage_junction_gates :3130-3156; the operator factor and solve of numerics/surface_imex.py
// :207-225, :269-278; the sparse factor's plan of numerics/sparse_cholesky.py:137-215 (a
// minimum-degree order, the elimination tree's union rule, levels).
//
// One CTA advances one world n_steps steps; threads loop over the world's cells and junctions.
// Per step, for each world:
//   stage 0   whole rates at the start potentials (cells, then junctions, then each cell's gather
//             of its junction fluxes in edge order);
//   predict   amounts, channel gates and junction gates half a step ahead, their potentials; the
//             slopes W = dJ/d(dv) of every patch, channel population and junction there; the
//             conductances G = F/1e15 sum_s z_s W_s;
//   operator  M = C + gamma dt L on the cells (the held bath clamped), Jacobi scaled, assembled
//             into the world's factor pattern and factored left-looking, level by level of the
//             elimination tree (a warp per column; each update term's destination precomputed on
//             the host, so no atomics);
//   stage i   the stage's charges, forward and back substitution by levels, the potentials; the
//             routes' linear fluxes W dv there (the implicit drift), their heat at the stage; the
//             remainders J - W dv of the explicit rates; channel and junction gates by their
//             exponential updates from the step start;
//   book      ledgers as the plain step; accept or refuse the world's step as a whole.
// Stage values live in a global scratch that stays in L2 while the world's CTA runs.

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <type_traits>
#include <queue>
#include <set>
#include <string>
#include <tuple>
#include <vector>

#include "handle.h"
#include "sparse_plan.h"

#include "n2_common.cuh"

namespace {

using namespace cbk;

// The stage solve's acceptance (surface_field.CHARGE_ATOL_C, CHARGE_RTOL).
constexpr double kChargeAtol = 3e-25;
constexpr double kChargeRtol = 2e-12;
// The mixed form's refinement bound (corrections per stage solve).
constexpr int kRefine = 6;

// Cell scratch fields ([field][C]).
enum N2Cell {
  NC_CX = 0,    // 3: the current stage's concentrations
  NC_LX = 3,    // 3: their logs
  NC_VX = 6,    // the current stage's potential
  NC_CP = 7,    // 3: predicted concentrations
  NC_VP = 10,   // predicted potential
  NC_WM = 11,   // 3: patch slopes W (fmol/s per V)
  NC_GP = 14,   // patch conductance (its channels' included)
  NC_S = 15,    // Jacobi scale 1/sqrt(M_ii)
  NC_MD = 16,   // M_ii
  NC_MB = 17,   // M_i,bath
  NC_A = 18,    // 10: accumulators n[3], mt[3], md, pc, pd, mw
  NC_K1 = 28,   // 3: stage-1 known amounts
  NC_KN = 31,   // 3: the stage-0 whole amount rate, then the stage-1 drift's amount rate
  NC_JM = 34,   // 3: the stage's patch flux J_m
  NC_EX = 37,   // 3: the stage's outward pump + channel transfer ("extra")
  NC_R = 40,    // 4: the stage's md, cycles, pd, mw
  NC_Y = 44,    // forward solve (position-indexed)
  NC_X = 45,    // back solve (position-indexed)
  NC_CH = 46    // per channel slot q: W, t0[2], tau0[2], gate[2], acc transferred, acc heat,
                //   J, J heat: 11 fields
};
constexpr int kN2ChFields = 11;
enum N2ChField {
  CH_W = 0, CH_T0 = 1, CH_TAU0 = 3, CH_G = 5, CH_AT = 7, CH_AD = 8, CH_J = 9, CH_JD = 10
};
__host__ __device__ constexpr int n2_cell_fields(int nch) { return NC_CH + kN2ChFields * nch; }
// Junction scratch fields ([field][E]).
enum N2Edge {
  NE_J = 0,     // 3: flux for the cells' gather
  NE_W = 3,     // 3: slopes W
  NE_G = 6,     // conductance
  NE_T0 = 7,    // start target of the gate law
  NE_R0 = 8,    // start relaxation rate
  NE_GX = 9,    // predicted gate, then the stage gate
  NE_A = 10,    // 4: accumulators jt[3], jd
  NE_JJ = 14,   // 3: the stage's whole flux
  NE_JD = 17,   // the stage's whole heat
  NE_FIELDS = 18
};


__device__ __forceinline__ void junction_law(double dv, double thr, double mn, double &target,
                                             double &relaxation) {
  const double shift = fabs(dv) - thr;
  const double alpha = 1.3 * exp(-77.0 * shift);
  const double log_beta = kLog0065 + 140.0 * shift;
  const double beta = 20.0 * exp(-logaddexp0(-log_beta));
  relaxation = alpha + beta;
  target = (alpha + beta * mn) / relaxation;
}

__device__ __forceinline__ bool gate_domain(double g, double dv, double thr, double mn,
                                            double jc) {
  return is_finite(thr) && thr >= 0.0 && thr <= kMaxAbsJunctionV && is_finite(mn) && mn >= 0.0 &&
         mn <= 1.0 && is_finite(dv) && fabs(dv) <= kMaxAbsJunctionV && is_finite(g) && g >= mn &&
         g <= 1.0 && is_finite(jc) && jc >= 0.0 && jc <= 1.0;
}

// A cell's own whole rates at a stage (patch flux, pump, channel populations), the plain step's
// arithmetic: J_m[3], extra[3] (outward pump + channel transfer), md, cycles, pd, mw, each
// population's J and heat; validity bits. Gate m of slot q at gate[q slot_stride], h at
// gate[q slot_stride + row_stride].
template <int NCH>
__device__ __forceinline__ uint32_t own_rates(const Tissue &T, const double *__restrict__ wc,
                                              long long gi, const double (&c)[3],
                                              const double (&lc)[3], double V, const double *gate,
                                              long long slot_stride, long long row_stride,
                                              double mc, double pctl,
                                              double ldc, const double *chctl, double (&jm)[3],
                                              double (&extra)[3], double (&r4)[4],
                                              double (&chj)[NCH > 0 ? NCH : 1],
                                              double (&chd)[NCH > 0 ? NCH : 1]) {
  const long long C = T.C;
  uint32_t bits = 0;
  const double RT = wc[WC_RT], dv = V - wc[WC_VB];
  const double x = dv * wc[WC_FRT];
  if (!(fabs(x) <= kMaxAbsX)) bits |= CB_WORLD_TRANSPORT;
  if (!is_finite(V)) bits |= CB_WORLD_TRANSPORT;
  double bp, bm;
  bernoulli_pair<double>(x, bp, bm);
  double mu[3];
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    if (!(is_finite(c[s]) && c[s] > 0.0)) bits |= CB_WORLD_TRANSPORT;
    const double gs = __ldg(T.ap + s * C + gi) * mc;
    const double co = wc[WC_CO + s];
    jm[s] = (s < 2) ? gs * (c[s] * bm - co * bp) : gs * (c[s] * bp - co * bm);
    mu[s] = RT * (lc[s] - wc[WC_LOGCO + s]) + ((s < 2) ? kF * dv : (-kF) * dv);
  }
  const double md = 1e-3 * ((jm[0] * mu[0] + jm[1] * mu[1]) + jm[2] * mu[2]);
  if (!(is_finite(jm[0]) && is_finite(jm[1]) && is_finite(jm[2]) && is_finite(md)))
    bits |= CB_WORLD_TRANSPORT;
  if (!(is_finite(mc) && mc >= 0.0 && mc <= 1.0 && is_finite(pctl) && pctl >= 0.0 && pctl <= 1.0))
    bits |= CB_WORLD_CONTROL;
  double chm[3] = {0.0, 0.0, 0.0};
  if constexpr (NCH > 0) {
#pragma unroll
    for (int q = 0; q < NCH; ++q) {
      const int code = __ldg(T.ch_code + q * C + gi);
      const int sp = __ldg(T.ch_species + q * C + gi);
      const double ctl = __ldg(chctl + q * C);
      if (!(is_finite(ctl) && ctl >= 0.0 && ctl <= 1.0)) bits |= CB_WORLD_CONTROL;
      const double open =
          channel_opening(code, gate[q * slot_stride], gate[q * slot_stride + row_stride]);
      const double gq = __ldg(T.ch_ap + q * C + gi) * ((open * ctl) * __ldg(T.ch_ab + q * C + gi));
      const double cs_ = sp == 0 ? c[0] : sp == 1 ? c[1] : c[2];
      const double co = wc[WC_CO + sp];
      const double J = sp < 2 ? gq * (cs_ * bm - co * bp) : gq * (cs_ * bp - co * bm);
      const double Jd = 1e-3 * J * (sp == 0 ? mu[0] : sp == 1 ? mu[1] : mu[2]);
      chj[q] = J;
      chd[q] = Jd;
      chm[sp] += J;
      if (!(is_finite(J) && is_finite(Jd))) bits |= CB_WORLD_TRANSPORT;
    }
  }
  const double energy = (wc[WC_DRIVE] + (-3.0) * mu[0]) + 2.0 * mu[1];
  const double a = energy * wc[WC_INVRT];
  double cycles = 0.0;
  if (__ldg(T.pcap + gi) > 0.0 && pctl > 0.0) {
    const double ls = ((-logaddexp0(3.0 * (wc[WC_LOGKMNA] - lc[0]))) - wc[WC_LK]) - wc[WC_LATP];
    const double mag = exp((ldc + ls) + fmax(a, 0.0));
    cycles = mag * (a >= 0.0 ? expm1(-a) : -expm1(a));
  }
  r4[0] = md;
  r4[1] = cycles;
  r4[2] = (-1e-3 * cycles) * energy;
  r4[3] = (-1e-3 * cycles) * wc[WC_DRIVE];
  extra[0] = (3.0 * cycles - 0.0) + chm[0];
  extra[1] = (-2.0 * cycles - 0.0) + chm[1];
  extra[2] = (-0.0 * cycles - 0.0) + chm[2];
  const double sna = mu[0] * wc[WC_INVRTD], sk = mu[1] * wc[WC_INVRTD];
  const double aff = (wc[WC_AFF0] + (-3.0) * sna) + 2.0 * sk;
  const double capacity = __ldg(T.pcap + gi);
  const bool pump_ok = wc[WC_PUMPOK] != 0.0 && is_finite(capacity) && capacity >= 0.0 &&
                       is_finite(sna) && fabs(sna) <= kMaxAbsIonPotentialOverRT && is_finite(sk) &&
                       fabs(sk) <= kMaxAbsIonPotentialOverRT && is_finite(aff) &&
                       fabs(aff) <= kMaxAbsAffinityOverRT;
  if (!pump_ok) bits |= CB_WORLD_PUMP_DOMAIN;
  if (!(is_finite(cycles) && is_finite(r4[2]) && is_finite(r4[3]))) bits |= CB_WORLD_TRANSPORT;
  return bits;
}

// A junction's whole flux at a stage: jj[3], its heat; validity bits.
__device__ __forceinline__ uint32_t junction_flux(const Tissue &T, const double *__restrict__ wc,
                                                  long long ge, const double (&ca)[3],
                                                  const double (&cb)[3], const double (&la)[3],
                                                  const double (&lb)[3], double dv,
                                                  double opening, double (&jj)[3], double &jd) {
  const long long E = T.E;
  uint32_t bits = 0;
  const double x = dv * wc[WC_FRT];
  if (!(fabs(x) <= kMaxAbsX)) bits |= CB_WORLD_TRANSPORT;
  double bp, bm, mu[3];
  bernoulli_pair<double>(x, bp, bm);
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    const double gs = __ldg(T.jap + s * E + ge) * opening;
    jj[s] = (s < 2) ? gs * (ca[s] * bm - cb[s] * bp) : gs * (ca[s] * bp - cb[s] * bm);
    mu[s] = wc[WC_RT] * (la[s] - lb[s]) + ((s < 2) ? kF * dv : (-kF) * dv);
  }
  jd = 1e-3 * ((jj[0] * mu[0] + jj[1] * mu[1]) + jj[2] * mu[2]);
  if (!(is_finite(jj[0]) && is_finite(jj[1]) && is_finite(jj[2]) && is_finite(jd)))
    bits |= CB_WORLD_TRANSPORT;
  return bits;
}

// The electrochemical differences of a junction (sender minus receiver) and of a patch.
__device__ __forceinline__ void junction_mu(const double *__restrict__ wc, const double (&la)[3],
                                            const double (&lb)[3], double dv, double (&mu)[3]) {
#pragma unroll
  for (int s = 0; s < 3; ++s)
    mu[s] = wc[WC_RT] * (la[s] - lb[s]) + ((s < 2) ? kF * dv : (-kF) * dv);
}
__device__ __forceinline__ void patch_mu(const double *__restrict__ wc, const double (&lc)[3],
                                         double dv, double (&mu)[3]) {
#pragma unroll
  for (int s = 0; s < 3; ++s)
    mu[s] = wc[WC_RT] * (lc[s] - wc[WC_LOGCO + s]) + ((s < 2) ? kF * dv : (-kF) * dv);
}


// Each world's factor values, solve vectors and plan are copied to dynamic shared memory once per
// launch when they fit (`smem_bytes`): all of it, or all but the relative positions; otherwise the
// world works from global memory. The choice is per world (uniform within its CTA).
// MIX: the factor and its substitutions in FP32, the stage potentials recovered by FP64
// iterative refinement of the charge residual against the FP64 operator.
template <int BLOCK, int NCH, int MINB, bool MIX>
__global__ void __launch_bounds__(BLOCK, MINB)
    n2_kernel(const Tissue T, const Layout L, const N2Dev D, const double *state_in,
              double *state_out, const double *__restrict__ control, const StepCoef k,
              int n_steps, uint32_t *__restrict__ world_status,
              int32_t *__restrict__ accepted_steps, size_t smem_bytes) {
  extern __shared__ double n2_smem[];
  constexpr int NQ = NCH > 0 ? NCH : 1;
  __shared__ double sW[WC_STRIDE];
  __shared__ double sRed[(BLOCK / 32) * 16];
  __shared__ unsigned int sBits;
  const int w = blockIdx.x, tid = threadIdx.x;
  const int c0 = T.cell_offset[w], nc = T.cell_offset[w + 1] - c0;
  const int e0 = T.edge_offset[w], ne = T.edge_offset[w + 1] - e0;
  const long long C = T.C, E = T.E, W = T.W;
  if (tid < WC_STRIDE) sW[tid] = T.world[(size_t)w * WC_STRIDE + tid];
  if (tid == 0) sBits = 0u;
  double *cs = D.cs;
  double *es = D.es;
  // The world's factor plan (local indices), factor values and solve vectors (by position).
  const int wF = D.fb[blockIdx.x + 1] - D.fb[blockIdx.x];
  const int wU = D.ub[blockIdx.x + 1] - D.ub[blockIdx.x];
  const int wR = D.rb[blockIdx.x + 1] - D.rb[blockIdx.x];
  const int wL = D.lb[blockIdx.x + 1] - D.lb[blockIdx.x];
  const int wc0 = T.cell_offset[blockIdx.x], wn = T.cell_offset[blockIdx.x + 1] - wc0;
  const int *colp = D.colp + wc0 + blockIdx.x, *lrow = D.lrow + D.fb[blockIdx.x];
  const int *ukp = D.uk_ptr + wc0 + blockIdx.x, *ukc = D.uk_col + D.ub[blockIdx.x];
  const int *ukpos = D.uk_pos + D.ub[blockIdx.x], *ukrel = D.uk_rel + D.ub[blockIdx.x];
  const int *rel = D.rel + D.rb[blockIdx.x];
  const int *lvp = D.lv_ptr + D.lb[blockIdx.x] + blockIdx.x, *lvc = D.lv_cols + wc0;
  using FT = typename std::conditional<MIX, float, double>::type;
  FT *lval = reinterpret_cast<FT *>(D.lval) + D.fb[blockIdx.x];
  FT *Yv = reinterpret_cast<FT *>(cs + (long long)NC_Y * T.C) + wc0;
  FT *Xv = reinterpret_cast<FT *>(cs + (long long)NC_X * T.C) + wc0;
  const size_t values = sizeof(FT) * (size_t)(wF + 2 * wn);
  const size_t plan_ints = sizeof(int) * (size_t)(2 * (wn + 1) + wF + 3 * wU + wL + 1 + wn);
  const size_t small_ints = sizeof(int) * (size_t)(2 * (wn + 1) + wL + 1 + wn);
  const int mode = values + plan_ints + sizeof(int) * (size_t)wR <= smem_bytes ? 2
                   : values + plan_ints <= smem_bytes                           ? 1
                   : values + small_ints <= smem_bytes                          ? 3
                                                                                : 0;
  if (mode > 0) {
    lval = reinterpret_cast<FT *>(n2_smem);
    Yv = lval + wF;
    Xv = Yv + wn;
    int *si = reinterpret_cast<int *>(Xv + wn);
    auto stage_ints = [&](const int *src, int count) {
      for (int i = threadIdx.x; i < count; i += BLOCK) si[i] = src[i];
      const int *out = si;
      si += count;
      return out;
    };
    colp = stage_ints(colp, wn + 1);
    if (mode != 3) lrow = stage_ints(lrow, wF);
    ukp = stage_ints(ukp, wn + 1);
    if (mode != 3) {
      ukc = stage_ints(ukc, wU);
      ukpos = stage_ints(ukpos, wU);
      ukrel = stage_ints(ukrel, wU);
    }
    lvp = stage_ints(lvp, wL + 1);
    lvc = stage_ints(lvc, wn);
    if (mode == 2) rel = stage_ints(rel, wR);
  }
  const long long oN = L.s[CB_AMOUNT_INCREMENT], oG = L.s[CB_JUNCTION_GATE];
  const long long oH = L.s[CB_CHANNEL_GATE];
  const double *mctl = control + L.c[CB_CONTROL_MEMBRANE];
  const double *pctlp = control + L.c[CB_CONTROL_PUMP];
  const double *jctl = control + L.c[CB_CONTROL_JUNCTION];
  const double *chctl0 = control + L.c[CB_CONTROL_CHANNEL];
  const double K = kChargePerFmol;
  const double gdt = k.gamma_dt;               // the implicit diagonal gamma dt (the operator's)
  const double theta = 0.5 * k.dt;             // the routes' operator time
  const double w1 = (1.0 - (1.0 - 1.0 / sqrt(2.0))) * k.dt;  // (1 - gamma) dt
  const int lv0 = 0, lv1 = wL;
  auto CF = [&](int f, long long gi) -> double & { return cs[(long long)f * C + gi]; };
  auto EF = [&](int f, long long ge) -> double & { return es[(long long)f * E + ge]; };
  auto CH = [&](int q, int f, long long gi) -> double & {
    return cs[(long long)(NC_CH + q * kN2ChFields + f) * C + gi];
  };
  __syncthreads();
  const double Vb = sW[WC_VB];
  double res[3], ec, rw, ew;
  for (int s = 0; s < 3; ++s) res[s] = state_in[L.s[CB_RESERVOIR_SUPPLIED] + s * W + w];
  ec = state_in[L.s[CB_ELECTRODE_CHARGE] + w];
  rw = state_in[L.s[CB_RESERVOIR_WORK] + w];
  ew = state_in[L.s[CB_ELECTRODE_WORK] + w];
  const double *cur = state_in;
  int taken = 0;
  uint32_t refused = 0u;

  const WorldCholesky<FT, BLOCK> chol{colp, lrow, ukp, ukc, ukpos, ukrel, rel, lvp, lvc,
                                       lval, Yv, Xv, lv0, lv1, wn,
                                       dense_tail(colp, lvp, lvc, lv0, lv1, wn)};
  auto factor = [&]() { return chol.factor(); };
  auto solve = [&]() { chol.solve(); };
  // A cell's gather over its junctions (senders first, then receivers, edge order) of field f.
  auto gather = [&](long long gi, int f, double (&send)[3], double (&recv)[3]) {
#pragma unroll
    for (int s = 0; s < 3; ++s) send[s] = recv[s] = 0.0;
    for (int a = __ldg(T.adj_ptr + gi); a < __ldg(T.adj_ptr + gi + 1); ++a) {
      const int code = __ldg(T.adj_idx + a);
      const long long ge = e0 + (code >> 1);
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        if (code & 1) recv[s] += EF(f + s, ge);
        else send[s] += EF(f + s, ge);
      }
    }
  };
  // Concentrations and logs of amounts n, into the current-stage fields.
  auto set_stage = [&](long long gi, const double (&n)[3], double V) {
    const double ivol = __ldg(T.ivol + gi);
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      const double c = (__ldg(T.ref + s * C + gi) + n[s]) * ivol;
      CF(NC_CX + s, gi) = c;
      CF(NC_LX + s, gi) = log(c);
    }
    CF(NC_VX, gi) = V;
  };
  auto potential_of = [&](long long gi, const double (&n)[3]) {
    return (__ldg(T.q0 + gi) + K * ((n[0] + n[1]) + (-n[2]))) * __ldg(T.icap + gi) + Vb;
  };
  // The operator's row product (M phi)_i (neighbours' potentials in NC_VX) less the charge q.
  auto row_residual = [&](long long gi, double q, double &product) {
    double sum = CF(NC_MD, gi) * CF(NC_VX, gi);
    for (int a = __ldg(T.adj_ptr + gi); a < __ldg(T.adj_ptr + gi + 1); ++a) {
      const int code = __ldg(T.adj_idx + a);
      const long long ge = e0 + (code >> 1);
      const long long nb = c0 + ((code & 1) ? __ldg(T.snd + ge) : __ldg(T.rcv + ge));
      sum += (gdt * (-EF(NE_G, ge))) * CF(NC_VX, nb);
    }
    product = sum + CF(NC_MB, gi) * Vb;
    return product - q;
  };

  for (int step = 0; step < n_steps; ++step) {
    uint32_t bits = 0;
    double inflow0[3] = {0, 0, 0}, outlin0[3] = {0, 0, 0}, plate0 = 0.0;
    // P1 (cells): the start: concentrations, potentials, own whole rates, start kinetics.
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      double n[3], c[3], lc[3];
      for (int s = 0; s < 3; ++s) n[s] = cur[oN + s * C + gi];
      const double V0 = potential_of(gi, n);
      set_stage(gi, n, V0);
      for (int s = 0; s < 3; ++s) {
        c[s] = CF(NC_CX + s, gi);
        lc[s] = CF(NC_LX + s, gi);
      }
      plate0 += -(K * ((n[0] + n[1]) + (-n[2])));
      const double pctl = pctlp[gi];
      const double ldc = pctl > 0.0 ? __ldg(T.logpcap + gi) + log(pctl) : 0.0;
      double jm[3], ex[3], r4[4], chj[NQ], chd[NQ];
      bits |= own_rates<NCH>(T, sW, gi, c, lc, V0, cur + oH + gi, C, NCH * C, mctl[gi], pctl,
                             ldc, chctl0 + gi, jm, ex, r4, chj, chd);
      for (int s = 0; s < 3; ++s) {
        CF(NC_JM + s, gi) = jm[s];
        CF(NC_EX + s, gi) = ex[s];
        inflow0[s] += jm[s] + ex[s];
      }
      for (int f = 0; f < 4; ++f) CF(NC_R + f, gi) = r4[f];
      if constexpr (NCH > 0) {
        for (int q = 0; q < NCH; ++q) {
          CH(q, CH_J, gi) = chj[q];
          CH(q, CH_JD, gi) = chd[q];
          double t[2], tau[2];
          channel_kinetics<false>(__ldg(T.ch_code + q * C + gi), V0 - Vb, t, tau);
          if (!channel_kinetics_ok(V0 - Vb, t, tau)) bits |= CB_WORLD_CHANNEL_DOMAIN;
          for (int r = 0; r < 2; ++r) {
            CH(q, CH_T0 + r, gi) = t[r];
            CH(q, CH_TAU0 + r, gi) = tau[r];
          }
        }
      }
      // Zero the world's factor columns held by this thread's cells.
      const int P = __ldg(D.rank + gi);
      for (int f = colp[P]; f < colp[P + 1]; ++f) lval[f] = 0.0;
    }
    __syncthreads();
    // E1 (junctions): stage-0 whole fluxes, the gate law at the start, the predicted gate.
    for (int e = tid; e < ne; e += BLOCK) {
      const long long ge = e0 + e;
      const long long ga = c0 + __ldg(T.snd + ge), gb = c0 + __ldg(T.rcv + ge);
      double ca[3], cb[3], la[3], lb[3], jj[3], jd;
      for (int s = 0; s < 3; ++s) {
        ca[s] = CF(NC_CX + s, ga);
        cb[s] = CF(NC_CX + s, gb);
        la[s] = CF(NC_LX + s, ga);
        lb[s] = CF(NC_LX + s, gb);
      }
      const double dv = CF(NC_VX, ga) - CF(NC_VX, gb);
      const double g = cur[oG + ge], jc = jctl[ge];
      bits |= junction_flux(T, sW, ge, ca, cb, la, lb, dv, jc * g, jj, jd);
      for (int s = 0; s < 3; ++s) {
        EF(NE_J + s, ge) = jj[s];
        EF(NE_JJ + s, ge) = jj[s];
      }
      EF(NE_JD, ge) = jd;
      const double thr = __ldg(T.thr + ge), mn = __ldg(T.jmin + ge);
      if (!gate_domain(g, dv, thr, mn, jc)) bits |= CB_WORLD_GATE_DOMAIN;
      double t0, r0;
      junction_law(dv, thr, mn, t0, r0);
      EF(NE_T0, ge) = t0;
      EF(NE_R0, ge) = r0;
      EF(NE_GX, ge) = g + (t0 - g) * -expm1(-r0 * theta);
    }
    __syncthreads();
    // P2 (cells): the whole stage-0 amount rate, the prediction, the patch slopes.
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      double send[3], recv[3], np_[3], cp[3];
      gather(gi, NE_J, send, recv);
      const double ivol = __ldg(T.ivol + gi);
      for (int s = 0; s < 3; ++s) {
        const double rate = ((-CF(NC_JM + s, gi) + (-send[s])) + recv[s]) - CF(NC_EX + s, gi);
        CF(NC_KN + s, gi) = rate;
        np_[s] = cur[oN + s * C + gi] + theta * rate;
        cp[s] = (__ldg(T.ref + s * C + gi) + np_[s]) * ivol;
        CF(NC_CP + s, gi) = cp[s];
        if (!(is_finite(cp[s]) && cp[s] > 0.0)) bits |= CB_WORLD_OPERATOR;
      }
      const double Vp = potential_of(gi, np_);
      CF(NC_VP, gi) = Vp;
      if (!is_finite(Vp)) bits |= CB_WORLD_OPERATOR;
      const double dv = Vp - Vb, mc = mctl[gi];
      double gp = 0.0;
      double zw[3];
      for (int s = 0; s < 3; ++s) {
        const double zfrt = (s < 2 ? 1.0 : -1.0) * sW[WC_FRT];
        const double W_ = route_slope(__ldg(T.ap + s * C + gi) * mc, cp[s], sW[WC_CO + s], dv,
                                      zfrt);
        CF(NC_WM + s, gi) = W_;
        zw[s] = (s < 2 ? 1.0 : -1.0) * W_;
        if (!is_finite(W_)) bits |= CB_WORLD_OPERATOR;
      }
      gp = K * ((zw[0] + zw[1]) + zw[2]);
      if constexpr (NCH > 0) {
        double extra = 0.0;
        for (int q = 0; q < NCH; ++q) {
          const int code = __ldg(T.ch_code + q * C + gi);
          const int sp = __ldg(T.ch_species + q * C + gi);
          double gq[2];
          for (int r = 0; r < 2; ++r) {
            const double g0 = cur[oH + (r * NCH + q) * C + gi];
            gq[r] = (r == 1 && code == kHhKn4)
                        ? g0
                        : advance_gate<false>(g0, CH(q, CH_T0 + r, gi), CH(q, CH_TAU0 + r, gi),
                                              CH(q, CH_T0 + r, gi), CH(q, CH_TAU0 + r, gi), theta);
          }
          const double available = (__ldg(T.ch_ab + q * C + gi) * channel_opening(code, gq[0], gq[1])) *
                                   __ldg(chctl0 + q * C + gi);
          const double zfrt = (sp < 2 ? 1.0 : -1.0) * sW[WC_FRT];
          const double W_ = route_slope(__ldg(T.ch_ap + q * C + gi) * available, cp[sp],
                                        sW[WC_CO + sp], dv, zfrt);
          CH(q, CH_W, gi) = W_;
          if (!is_finite(W_)) bits |= CB_WORLD_OPERATOR;
          extra = extra + K * ((sp < 2 ? 1.0 : -1.0) * W_);
        }
        gp = gp + extra;
      }
      CF(NC_GP, gi) = gp;
    }
    __syncthreads();
    // E2 (junctions): slopes and conductances at the prediction; the stage-0 linear part and its
    // heat; the junction accumulators y + delta dt (J - W dv).
    for (int e = tid; e < ne; e += BLOCK) {
      const long long ge = e0 + e;
      const long long ga = c0 + __ldg(T.snd + ge), gb = c0 + __ldg(T.rcv + ge);
      const double dvp = CF(NC_VP, ga) - CF(NC_VP, gb);
      const double opening = jctl[ge] * EF(NE_GX, ge);
      double zw[3], la[3], lb[3], mu[3];
      for (int s = 0; s < 3; ++s) {
        const double zfrt = (s < 2 ? 1.0 : -1.0) * sW[WC_FRT];
        const double W_ = route_slope(__ldg(T.jap + s * E + ge) * opening, CF(NC_CP + s, ga),
                                      CF(NC_CP + s, gb), dvp, zfrt);
        EF(NE_W + s, ge) = W_;
        zw[s] = (s < 2 ? 1.0 : -1.0) * W_;
        if (!is_finite(W_)) bits |= CB_WORLD_OPERATOR;
        la[s] = CF(NC_LX + s, ga);
        lb[s] = CF(NC_LX + s, gb);
      }
      EF(NE_G, ge) = K * ((zw[0] + zw[1]) + zw[2]);
      const double dv0 = CF(NC_VX, ga) - CF(NC_VX, gb);
      junction_mu(sW, la, lb, dv0, mu);
      double lin[3], hm[3];
      for (int s = 0; s < 3; ++s) {
        lin[s] = EF(NE_W + s, ge) * dv0;
        hm[s] = lin[s] * mu[s];
        EF(NE_J + s, ge) = lin[s];
        EF(NE_A + s, ge) =
            cur[L.s[CB_JUNCTION_TRANSFERRED] + s * E + ge] + k.delta_dt * (EF(NE_JJ + s, ge) - lin[s]);
      }
      const double heat = 1e-3 * ((hm[0] + hm[1]) + hm[2]);
      EF(NE_A + 3, ge) = cur[L.s[CB_JUNCTION_DISSIPATED] + ge] + k.delta_dt * (EF(NE_JD, ge) - heat);
    }
    __syncthreads();
    // P4 (cells): the stage-0 remainder, the accumulators, the operator's diagonal.
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      double send[3], recv[3], lc[3], mu[3];
      gather(gi, NE_J, send, recv);
      const double dv0 = CF(NC_VX, gi) - Vb;
      for (int s = 0; s < 3; ++s) lc[s] = CF(NC_LX + s, gi);
      patch_mu(sW, lc, dv0, mu);
      double lm[3], patches[3], hm[3];
      for (int s = 0; s < 3; ++s) {
        lm[s] = CF(NC_WM + s, gi) * dv0;
        patches[s] = lm[s];
        hm[s] = lm[s] * mu[s];
      }
      double lch[NQ], hch[NQ];
      if constexpr (NCH > 0) {
        for (int q = 0; q < NCH; ++q) {
          const int sp = __ldg(T.ch_species + q * C + gi);
          lch[q] = CH(q, CH_W, gi) * dv0;
          hch[q] = 1e-3 * lch[q] * mu[sp];
          patches[sp] = patches[sp] + lch[q];
        }
      }
      const double hmem = 1e-3 * ((hm[0] + hm[1]) + hm[2]);
      for (int s = 0; s < 3; ++s) {
        const double cells_lin = (recv[s] - send[s]) - patches[s];
        const double k0n = CF(NC_KN + s, gi) - cells_lin;
        const double n0 = cur[oN + s * C + gi];
        CF(NC_A + s, gi) = n0 + k.delta_dt * k0n;
        CF(NC_K1 + s, gi) = n0 + k.gamma_dt * k0n;
        CF(NC_A + 3 + s, gi) = cur[L.s[CB_MEMBRANE_TRANSFERRED] + s * C + gi] +
                               k.delta_dt * (CF(NC_JM + s, gi) - lm[s]);
        outlin0[s] += patches[s];
      }
      CF(NC_A + 6, gi) = cur[L.s[CB_MEMBRANE_DISSIPATED] + gi] + k.delta_dt * (CF(NC_R, gi) - hmem);
      CF(NC_A + 7, gi) = cur[L.s[CB_PUMP_CYCLES] + gi] + k.delta_dt * CF(NC_R + 1, gi);
      CF(NC_A + 8, gi) = cur[L.s[CB_PUMP_DISSIPATED] + gi] + k.delta_dt * CF(NC_R + 2, gi);
      CF(NC_A + 9, gi) = cur[L.s[CB_METABOLIC_WORK] + gi] + k.delta_dt * CF(NC_R + 3, gi);
      if constexpr (NCH > 0) {
        for (int q = 0; q < NCH; ++q) {
          CH(q, CH_AT, gi) = cur[L.s[CB_CHANNEL_TRANSFERRED] + q * C + gi] +
                             k.delta_dt * (CH(q, CH_J, gi) - lch[q]);
          CH(q, CH_AD, gi) = cur[L.s[CB_CHANNEL_DISSIPATED] + q * C + gi] +
                             k.delta_dt * (CH(q, CH_JD, gi) - hch[q]);
        }
      }
      // M_ii = C_i + gamma dt (G_patch + sum of its junctions' G), the junctions as the
      // Laplacian's scatter orders them (senders, then receivers).
      double gs = 0.0, gr = 0.0;
      for (int a = __ldg(T.adj_ptr + gi); a < __ldg(T.adj_ptr + gi + 1); ++a) {
        const int code = __ldg(T.adj_idx + a);
        const double g = EF(NE_G, e0 + (code >> 1));
        if (code & 1) gr += g;
        else gs += g;
      }
      const double cap = 1.0 / __ldg(T.icap + gi);
      const double gp = CF(NC_GP, gi);
      const double mii = cap + gdt * (gp + (gs + gr));
      CF(NC_MD, gi) = mii;
      CF(NC_MB, gi) = (-cap) + gdt * (-gp);
      if (!(mii > 0.0)) bits |= CB_WORLD_OPERATOR;
      const double sc = 1.0 / sqrt(mii > 0.0 ? mii : 1.0);
      CF(NC_S, gi) = sc;
      lval[colp[__ldg(D.rank + gi)]] = FT((mii * sc) * sc);
    }
    __syncthreads();
    // E3 (junctions): the operator's off-diagonal entries, scaled (row then column).
    for (int e = tid; e < ne; e += BLOCK) {
      const long long ge = e0 + e;
      const long long ga = c0 + __ldg(T.snd + ge), gb = c0 + __ldg(T.rcv + ge);
      const int ra = __ldg(D.rank + ga), rb = __ldg(D.rank + gb);
      const double m = 0.0 + gdt * (-EF(NE_G, ge));
      const double s_row = ra > rb ? CF(NC_S, ga) : CF(NC_S, gb);
      const double s_col = ra > rb ? CF(NC_S, gb) : CF(NC_S, ga);
      lval[__ldg(D.edge_pos + ge)] = FT((m * s_row) * s_col);
    }
    __syncthreads();
    if (factor()) bits |= CB_WORLD_OPERATOR;
    // Two stages: i = 1 (known K1) and i = 2 (known: the accumulators).
    double inflow1[3] = {0, 0, 0}, outlin1[3] = {0, 0, 0}, outlin2[3] = {0, 0, 0};
    double plate2 = 0.0;
    for (int st = 1; st <= 2; ++st) {
      const int kf = st == 1 ? NC_K1 : NC_A;
      if constexpr (!MIX) {
        // Charges and the scaled right-hand side (charge - M held) s; the FP64 solve.
        for (int i = tid; i < nc; i += BLOCK) {
          const long long gi = c0 + i;
          const double q = __ldg(T.q0 + gi) +
                           K * ((CF(kf, gi) + CF(kf + 1, gi)) + (-CF(kf + 2, gi)));
          Yv[__ldg(D.rank + gi)] = (q - CF(NC_MB, gi) * Vb) * CF(NC_S, gi);
        }
        __syncthreads();
        solve();
        for (int i = tid; i < nc; i += BLOCK) {
          const long long gi = c0 + i;
          CF(NC_VX, gi) = Xv[__ldg(D.rank + gi)] * CF(NC_S, gi);
        }
        __syncthreads();
      } else {
        // Iterative refinement from V = 0: the FP64 residual r = q - M V, its FP32 correction
        // (scaled), V += correction; until every row is within 1e-3 of the stage's acceptance
        // bound (3e-25 C + 2e-12 max(|q|, |M V|)), at most kRefine corrections.
        for (int i = tid; i < nc; i += BLOCK) CF(NC_VX, c0 + i) = 0.0;
        __syncthreads();
        for (int it = 0; it < kRefine; ++it) {
          int pending = 0;
          for (int i = tid; i < nc; i += BLOCK) {
            const long long gi = c0 + i;
            const double q = __ldg(T.q0 + gi) +
                             K * ((CF(kf, gi) + CF(kf + 1, gi)) + (-CF(kf + 2, gi)));
            double product;
            const double r = -row_residual(gi, q, product);
            const double bound = kChargeAtol + kChargeRtol * fmax(fabs(q), fabs(product));
            if (!(fabs(r) <= 1e-3 * bound)) pending = 1;
            Yv[__ldg(D.rank + gi)] = FT(r * CF(NC_S, gi));
          }
          if (!__syncthreads_or(pending)) break;
          solve();
          for (int i = tid; i < nc; i += BLOCK) {
            const long long gi = c0 + i;
            CF(NC_VX, gi) = CF(NC_VX, gi) + double(Xv[__ldg(D.rank + gi)]) * CF(NC_S, gi);
          }
          __syncthreads();
        }
      }
      // Junctions: the linear flux at the stage potentials, the stage gate.
      const double frac_dt = st == 1 ? k.frac1_dt : k.frac2_dt;
      for (int e = tid; e < ne; e += BLOCK) {
        const long long ge = e0 + e;
        const long long ga = c0 + __ldg(T.snd + ge), gb = c0 + __ldg(T.rcv + ge);
        const double dv = CF(NC_VX, ga) - CF(NC_VX, gb);
        for (int s = 0; s < 3; ++s) EF(NE_J + s, ge) = EF(NE_W + s, ge) * dv;
        const double thr = __ldg(T.thr + ge), mn = __ldg(T.jmin + ge);
        double t1, r1;
        junction_law(dv, thr, mn, t1, r1);
        const double g = advance_gate<false>(cur[oG + ge], EF(NE_T0, ge), 1.0 / EF(NE_R0, ge), t1,
                                             1.0 / r1, frac_dt);
        EF(NE_GX, ge) = g;
        if (!gate_domain(g, dv, thr, mn, jctl[ge])) bits |= CB_WORLD_GATE_DOMAIN;
      }
      __syncthreads();
      // Cells: the residual, the drift's amounts, the stage state, its gates, its own rates.
      for (int i = tid; i < nc; i += BLOCK) {
        const long long gi = c0 + i;
        const double q = __ldg(T.q0 + gi) +
                         K * ((CF(kf, gi) + CF(kf + 1, gi)) + (-CF(kf + 2, gi)));
        double product;
        const double r = row_residual(gi, q, product);
        const double V = CF(NC_VX, gi);
        if (!is_finite(V) || !(fabs(r) <= kChargeAtol + kChargeRtol * fmax(fabs(q), fabs(product))))
          bits |= CB_WORLD_RESIDUAL;
        double send[3], recv[3], patches[3], n[3];
        gather(gi, NE_J, send, recv);
        const double dv = V - Vb;
        for (int s = 0; s < 3; ++s) patches[s] = CF(NC_WM + s, gi) * dv;
        if constexpr (NCH > 0) {
          for (int q_ = 0; q_ < NCH; ++q_) {
            const int sp = __ldg(T.ch_species + q_ * C + gi);
            patches[sp] = patches[sp] + CH(q_, CH_W, gi) * dv;
          }
        }
        for (int s = 0; s < 3; ++s) {
          const double d = (recv[s] - send[s]) - patches[s];
          n[s] = CF(kf + s, gi) + k.gamma_dt * d;  // the stage state's amounts
          if (st == 1) {
            CF(NC_KN + s, gi) = d;
            outlin1[s] += patches[s];
          } else {
            CF(NC_A + s, gi) = n[s];  // the step's new amounts
            outlin2[s] += patches[s];
          }
        }
        if (st == 2) plate2 += -(K * ((n[0] + n[1]) + (-n[2])));
        const double ivol = __ldg(T.ivol + gi);
        double c[3], lc[3];
        for (int s = 0; s < 3; ++s) {
          c[s] = (__ldg(T.ref + s * C + gi) + n[s]) * ivol;
          lc[s] = log(c[s]);
          CF(NC_CX + s, gi) = c[s];
          CF(NC_LX + s, gi) = lc[s];
        }
        // Channel gates: the exponential update from the start to this stage's potential.
        if constexpr (NCH > 0) {
          for (int q_ = 0; q_ < NCH; ++q_) {
            const int code = __ldg(T.ch_code + q_ * C + gi);
            double t[2], tau[2];
            channel_kinetics<false>(code, dv, t, tau);
            if (!channel_kinetics_ok(dv, t, tau)) bits |= CB_WORLD_CHANNEL_DOMAIN;
            for (int r2 = 0; r2 < 2; ++r2) {
              const double g0 = cur[oH + (r2 * NCH + q_) * C + gi];
              CH(q_, CH_G + r2, gi) =
                  (r2 == 1 && code == kHhKn4)
                      ? g0
                      : advance_gate<false>(g0, CH(q_, CH_T0 + r2, gi), CH(q_, CH_TAU0 + r2, gi),
                                            t[r2], tau[r2], frac_dt);
            }
          }
        }
        // The linear parts' heat at the stage state and potential.
        double mu[3];
        patch_mu(sW, lc, dv, mu);
        double lm[3], hm[3];
        for (int s = 0; s < 3; ++s) {
          lm[s] = CF(NC_WM + s, gi) * dv;
          hm[s] = lm[s] * mu[s];
        }
        const double hmem = 1e-3 * ((hm[0] + hm[1]) + hm[2]);
        double lch[NQ], hch[NQ];
        if constexpr (NCH > 0) {
          for (int q_ = 0; q_ < NCH; ++q_) {
            const int sp = __ldg(T.ch_species + q_ * C + gi);
            lch[q_] = CH(q_, CH_W, gi) * dv;
            hch[q_] = 1e-3 * lch[q_] * mu[sp];
          }
        }
        if (st == 1) {
          // The stage-1 whole rates (own parts; the junctions' after their pass), the remainder
          // k1 = whole - linear and the drift d1 into the accumulators, as _combine orders them.
          const double pctl = pctlp[gi];
          const double ldc = pctl > 0.0 ? __ldg(T.logpcap + gi) + log(pctl) : 0.0;
          double jm[3], ex[3], r4[4], chj[NQ], chd[NQ];
          bits |= own_rates<NCH>(T, sW, gi, c, lc, V, cs + (long long)(NC_CH + CH_G) * C + gi,
                                 (long long)kN2ChFields * C, C, mctl[gi], pctl, ldc,
                                 chctl0 + gi, jm, ex, r4, chj, chd);
          for (int s = 0; s < 3; ++s) {
            CF(NC_JM + s, gi) = jm[s];
            CF(NC_EX + s, gi) = ex[s];
            inflow1[s] += jm[s] + ex[s];
            CF(NC_A + 3 + s, gi) = (CF(NC_A + 3 + s, gi) + k.omdelta_dt * (jm[s] - lm[s])) +
                                   w1 * lm[s];
          }
          CF(NC_A + 6, gi) = (CF(NC_A + 6, gi) + k.omdelta_dt * (r4[0] - hmem)) + w1 * hmem;
          CF(NC_A + 7, gi) = (CF(NC_A + 7, gi) + k.omdelta_dt * r4[1]) + w1 * 0.0;
          CF(NC_A + 8, gi) = (CF(NC_A + 8, gi) + k.omdelta_dt * r4[2]) + w1 * 0.0;
          CF(NC_A + 9, gi) = (CF(NC_A + 9, gi) + k.omdelta_dt * r4[3]) + w1 * 0.0;
          if constexpr (NCH > 0) {
            for (int q_ = 0; q_ < NCH; ++q_) {
              CH(q_, CH_AT, gi) = (CH(q_, CH_AT, gi) + k.omdelta_dt * (chj[q_] - lch[q_])) +
                                  w1 * lch[q_];
              CH(q_, CH_AD, gi) = (CH(q_, CH_AD, gi) + k.omdelta_dt * (chd[q_] - hch[q_])) +
                                  w1 * hch[q_];
            }
          }
        } else {
          // The new state's ledgers: the accumulators plus gamma dt of the stage-2 drift.
          for (int s = 0; s < 3; ++s)
            CF(NC_A + 3 + s, gi) = CF(NC_A + 3 + s, gi) + k.gamma_dt * lm[s];
          CF(NC_A + 6, gi) = CF(NC_A + 6, gi) + k.gamma_dt * hmem;
          CF(NC_A + 7, gi) = CF(NC_A + 7, gi) + k.gamma_dt * 0.0;
          CF(NC_A + 8, gi) = CF(NC_A + 8, gi) + k.gamma_dt * 0.0;
          CF(NC_A + 9, gi) = CF(NC_A + 9, gi) + k.gamma_dt * 0.0;
          bool ok = true;
          for (int f = 0; f < 10; ++f) ok = ok && is_finite(CF(NC_A + f, gi));
          for (int s = 0; s < 3; ++s) ok = ok && (__ldg(T.ref + s * C + gi) + n[s]) > 0.0;
          if constexpr (NCH > 0) {
            for (int q_ = 0; q_ < NCH; ++q_) {
              CH(q_, CH_AT, gi) = CH(q_, CH_AT, gi) + k.gamma_dt * lch[q_];
              CH(q_, CH_AD, gi) = CH(q_, CH_AD, gi) + k.gamma_dt * hch[q_];
              ok = ok && is_finite(CH(q_, CH_AT, gi)) && is_finite(CH(q_, CH_AD, gi));
              for (int r2 = 0; r2 < 2; ++r2) {
                const double g = CH(q_, CH_G + r2, gi);
                ok = ok && is_finite(g) && g >= 0.0 && g <= 1.0;
              }
            }
          }
          if (!ok) bits |= CB_WORLD_DOMAIN;
        }
      }
      __syncthreads();
      // Junctions: the linear part's heat at the stage; at stage 1 the whole flux too.
      for (int e = tid; e < ne; e += BLOCK) {
        const long long ge = e0 + e;
        const long long ga = c0 + __ldg(T.snd + ge), gb = c0 + __ldg(T.rcv + ge);
        double ca[3], cb[3], la[3], lb[3], mu[3], lin[3], hm[3];
        for (int s = 0; s < 3; ++s) {
          ca[s] = CF(NC_CX + s, ga);
          cb[s] = CF(NC_CX + s, gb);
          la[s] = CF(NC_LX + s, ga);
          lb[s] = CF(NC_LX + s, gb);
        }
        const double dv = CF(NC_VX, ga) - CF(NC_VX, gb);
        junction_mu(sW, la, lb, dv, mu);
        for (int s = 0; s < 3; ++s) {
          lin[s] = EF(NE_W + s, ge) * dv;
          hm[s] = lin[s] * mu[s];
        }
        const double heat = 1e-3 * ((hm[0] + hm[1]) + hm[2]);
        const double g = EF(NE_GX, ge), jc = jctl[ge];
        if (st == 1) {
          double jj[3], jd;
          bits |= junction_flux(T, sW, ge, ca, cb, la, lb, dv, jc * g, jj, jd);
          if (!gate_domain(g, dv, __ldg(T.thr + ge), __ldg(T.jmin + ge), jc))
            bits |= CB_WORLD_GATE_DOMAIN;
          for (int s = 0; s < 3; ++s) {
            EF(NE_J + s, ge) = jj[s];
            EF(NE_A + s, ge) = (EF(NE_A + s, ge) + k.omdelta_dt * (jj[s] - lin[s])) + w1 * lin[s];
          }
          EF(NE_A + 3, ge) = (EF(NE_A + 3, ge) + k.omdelta_dt * (jd - heat)) + w1 * heat;
        } else {
          bool ok = true;
          for (int s = 0; s < 3; ++s) {
            EF(NE_A + s, ge) = EF(NE_A + s, ge) + k.gamma_dt * lin[s];
            ok = ok && is_finite(EF(NE_A + s, ge));
          }
          EF(NE_A + 3, ge) = EF(NE_A + 3, ge) + k.gamma_dt * heat;
          ok = ok && is_finite(EF(NE_A + 3, ge)) && is_finite(g) && g >= __ldg(T.jmin + ge) &&
               g <= 1.0;
          if (!ok) bits |= CB_WORLD_DOMAIN;
        }
      }
      __syncthreads();
      if (st == 1) {
        // Cells: the stage-1 whole amount rate (own + junctions) less the drift, into the
        // accumulators: A += (1 - delta) dt k1 + (1 - gamma) dt d1.
        for (int i = tid; i < nc; i += BLOCK) {
          const long long gi = c0 + i;
          double send[3], recv[3];
          gather(gi, NE_J, send, recv);
          for (int s = 0; s < 3; ++s) {
            const double whole =
                ((-CF(NC_JM + s, gi) + (-send[s])) + recv[s]) - CF(NC_EX + s, gi);
            const double d1 = CF(NC_KN + s, gi);
            CF(NC_A + s, gi) = (CF(NC_A + s, gi) + k.omdelta_dt * (whole - d1)) + w1 * d1;
          }
        }
        __syncthreads();
      }
    }
    // World sums: the bath's inflow terms of both stages' rates and drifts, the end plate.
    double v[14] = {inflow0[0], inflow0[1], inflow0[2], outlin0[0], outlin0[1], outlin0[2],
                    inflow1[0], inflow1[1], inflow1[2], outlin1[0], outlin1[1], outlin1[2],
                    plate0, plate2};
    block_sum<BLOCK, 14>(v, sRed);
    double v2[3] = {outlin2[0], outlin2[1], outlin2[2]};
    block_sum<BLOCK, 3>(v2, sRed);
    double res2[3], applied[3];
    // The bath's supply rates: a whole stage rate supplies -inflow; the routes' linear parts
    // carry +outlin out through the patches, so a remainder supplies -inflow + outlin and a
    // drift -outlin.
    for (int s = 0; s < 3; ++s) {
      const double k0r = -v[s] + v[3 + s];
      const double k1r = -v[6 + s] + v[9 + s];
      const double d1r = -v[9 + s];
      const double d2r = -v2[s];
      res2[s] = (((res[s] + k.delta_dt * k0r) + k.omdelta_dt * k1r) + w1 * d1r) + k.gamma_dt * d2r;
      applied[s] = ((0.0 + k.delta * k0r) + k.omdelta * k1r) +
                   ((0.0 + (1.0 - (1.0 - 1.0 / sqrt(2.0))) * d1r) + (1.0 - 1.0 / sqrt(2.0)) * d2r);
    }
    const double electrode = v[13] - v[12];
    const double ec2 = ec + electrode;
    const double rw2 = rw + 1e-3 * ((sW[WC_MUB] * (k.dt * applied[0]) +
                                     sW[WC_MUB + 1] * (k.dt * applied[1])) +
                                    sW[WC_MUB + 2] * (k.dt * applied[2]));
    const double ew2 = ew + (1e12 * Vb) * electrode;
    if (!(is_finite(res2[0]) && is_finite(res2[1]) && is_finite(res2[2]) && is_finite(ec2) &&
          is_finite(rw2) && is_finite(ew2)))
      bits |= CB_WORLD_DOMAIN;
    if (bits) atomicOr(&sBits, bits);
    __syncthreads();
    const uint32_t world_bits = sBits;
    if (world_bits) {
      refused = world_bits;
      break;
    }
    // Commit the accepted state.
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      for (int s = 0; s < 3; ++s) {
        state_out[oN + s * C + gi] = CF(NC_A + s, gi);
        state_out[L.s[CB_MEMBRANE_TRANSFERRED] + s * C + gi] = CF(NC_A + 3 + s, gi);
      }
      state_out[L.s[CB_MEMBRANE_DISSIPATED] + gi] = CF(NC_A + 6, gi);
      state_out[L.s[CB_PUMP_CYCLES] + gi] = CF(NC_A + 7, gi);
      state_out[L.s[CB_PUMP_DISSIPATED] + gi] = CF(NC_A + 8, gi);
      state_out[L.s[CB_METABOLIC_WORK] + gi] = CF(NC_A + 9, gi);
      if constexpr (NCH > 0) {
        for (int q = 0; q < NCH; ++q) {
          state_out[L.s[CB_CHANNEL_TRANSFERRED] + q * C + gi] = CH(q, CH_AT, gi);
          state_out[L.s[CB_CHANNEL_DISSIPATED] + q * C + gi] = CH(q, CH_AD, gi);
          for (int r = 0; r < 2; ++r)
            state_out[oH + (r * NCH + q) * C + gi] = CH(q, CH_G + r, gi);
        }
      }
    }
    for (int e = tid; e < ne; e += BLOCK) {
      const long long ge = e0 + e;
      for (int s = 0; s < 3; ++s)
        state_out[L.s[CB_JUNCTION_TRANSFERRED] + s * E + ge] = EF(NE_A + s, ge);
      state_out[L.s[CB_JUNCTION_DISSIPATED] + ge] = EF(NE_A + 3, ge);
      state_out[oG + ge] = EF(NE_GX, ge);
    }
    for (int s = 0; s < 3; ++s) res[s] = res2[s];
    ec = ec2;
    rw = rw2;
    ew = ew2;
    ++taken;
    cur = state_out;
    __syncthreads();
  }
  // A world refused at its first step keeps its input state.
  if (taken == 0 && state_in != state_out) {
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      for (int f = CB_AMOUNT_INCREMENT; f <= CB_METABOLIC_WORK; ++f) {
        const int reps = (f <= CB_MEMBRANE_TRANSFERRED) ? 3 : 1;
        for (int s = 0; s < reps; ++s)
          state_out[L.s[f] + s * C + gi] = state_in[L.s[f] + s * C + gi];
      }
      for (int f = CB_CHANNEL_GATE; f <= CB_CHANNEL_DISSIPATED; ++f) {
        const int reps = (f == CB_CHANNEL_GATE) ? 2 * NCH : NCH;
        for (int s = 0; s < reps; ++s)
          state_out[L.s[f] + s * C + gi] = state_in[L.s[f] + s * C + gi];
      }
    }
    for (int e = tid; e < ne; e += BLOCK) {
      const long long ge = e0 + e;
      for (int f = CB_JUNCTION_TRANSFERRED; f <= CB_JUNCTION_GATE; ++f) {
        const int reps = (f == CB_JUNCTION_TRANSFERRED) ? 3 : 1;
        for (int s = 0; s < reps; ++s)
          state_out[L.s[f] + s * E + ge] = state_in[L.s[f] + s * E + ge];
      }
    }
  }
  if (tid == 0) {
    for (int s = 0; s < 3; ++s) state_out[L.s[CB_RESERVOIR_SUPPLIED] + s * W + w] = res[s];
    state_out[L.s[CB_ELECTRODE_CHARGE] + w] = ec;
    state_out[L.s[CB_RESERVOIR_WORK] + w] = rw;
    state_out[L.s[CB_ELECTRODE_WORK] + w] = ew;
    world_status[w] = refused;
    if (accepted_steps) accepted_steps[w] = taken;
  }
}

// ---------------------------------------------------------------------------------------------
// ROS2 (CB_METHOD_ROS2, this library's cells_b200.solver.ros2_verwer@1; the reference has no
// Rosenbrock method on its tissue path): Verwer, Spee, Blom and Hundsdorfer's two-stage,
// second-order, L-stable scheme, gamma = 1 + 1/sqrt(2),
//   W k1 = F(y),  W k2 = F(y + h k1) - 2 k1,  y' = y + (3/2) h k1 + (1/2) h k2,  W = I - gamma h J,
// the stage structure of the reference's only Rosenbrock integrator (numerics/
// rosenbrock_dense.py:123-141) on the held-bath step's whole right-hand side F (the readouts'
// derivative, models/surface_kinetic.py:221-410). J, fixed at y for the step: every route's slope
// conductance dJ/d(dv) (N2's route_slope) through each cell's dV/dn_s = z_s F/C, applied alike to
// the amounts and to every ledger whose rate is a route flux (so the ledgers balance to rounding);
// each gate's relaxation rate on the diagonal and, for channel gates, d/dV of (target - g)/tau;
// nothing for the pump. W k = r then reduces per world to (C + gamma h G) u = K sum_s z_s r_s in
// the cells' voltage rates u (G the conductance Laplacian of N2's operator, the bath held: the
// same sparse factor plan), after which a route's rate is r + gamma h W du and a gate's
// (r + gamma h dg'/dV u) / (1 + gamma h lambda). One factorisation and two solves per step.

// Cell scratch ([field][C]).
enum R2Cell {
  RC_CX = 0,    // 3: the evaluated state's concentrations
  RC_LX = 3,    // 3: their logs
  RC_VX = 6,    // its potential
  RC_WM = 7,    // 3: patch slopes W (fmol/s per V) at the step start
  RC_MD = 10,   // the operator's diagonal M_ii
  RC_S = 11,    // Jacobi scale 1/sqrt(M_ii)
  RC_JM0 = 12,  // 3: the start's patch fluxes
  RC_MU0 = 15,  // 3: the start's patch electrochemical differences
  RC_R = 18,    // 10: the evaluation's right-hand side: n[3], mt[3], md, cycles, pd, mw
  RC_K = 28,    // 10: k1 of those rows, then the step's new values
  RC_U = 38,    // the voltage rate u
  RC_YV = 39,   // forward solve (position-indexed)
  RC_XV = 40,   // back solve (position-indexed)
  RC_CH = 41    // per channel slot q: R2ChField
};
enum R2ChField {
  RH_W = 0,     // slope at the start
  RH_J0 = 1,    // flux at the start
  RH_DEC = 2,   // 2: each gate row's relaxation rate 1/tau at the start (0: no law)
  RH_CPL = 4,   // 2: d/dV of (target - g)/tau at the start
  RH_R = 6,     // 4: the evaluation's gate rates m, h, transferred, dissipated
  RH_K = 10,    // 4: k1 of those rows, then the new values
  RH_FIELDS = 14
};
__host__ __device__ constexpr int ros2_cell_fields(int nch) { return RC_CH + RH_FIELDS * nch; }
// Junction scratch ([field][E]).
enum R2Edge {
  RE_J = 0,     // 3: fluxes for the cells' gather (the evaluation's, then the corrections)
  RE_W = 3,     // 3: slopes at the start
  RE_G = 6,     // conductance
  RE_JJ0 = 7,   // 3: the start's fluxes
  RE_MU0 = 10,  // 3: the start's electrochemical differences
  RE_DEC = 13,  // the gate law's relaxation rate alpha + beta at the start
  RE_R = 14,    // 5: the evaluation's jt[3], jd, gate rate
  RE_K = 19,    // 5: k1 of those rows, then the new values
  RE_FIELDS = 24
};

// MIX (CB_METHOD_ROS2_MIXED): the voltage operator factored and both stage solves substituted in
// FP32, with no refinement. ROS2 is a W-method: its order and its ledger bookkeeping hold for any
// W, and an FP32 factor is the exact factor of a W within FP32 rounding of the FP64 one, so every
// rate, slope and accumulation stays FP64 and the step stays second order and conservative.
template <int BLOCK, int NCH, int MINB, bool RK4, bool MIX>
__global__ void __launch_bounds__(BLOCK, MINB)
    ros2_kernel(const Tissue T, const Layout L, const N2Dev D, const double *state_in,
                double *state_out, const double *__restrict__ control, const StepCoef k,
                int n_steps, uint32_t *__restrict__ world_status,
                int32_t *__restrict__ accepted_steps, size_t smem_bytes, const R2Tape tp) {
  extern __shared__ double n2_smem[];
  constexpr int NQ = NCH > 0 ? NCH : 1;
  __shared__ double sW[WC_STRIDE];
  __shared__ double sRed[(BLOCK / 32) * 16];
  __shared__ unsigned int sBits;
  const int w = blockIdx.x, tid = threadIdx.x;
  const int c0 = T.cell_offset[w], nc = T.cell_offset[w + 1] - c0;
  const int e0 = T.edge_offset[w], ne = T.edge_offset[w + 1] - e0;
  const long long C = T.C, E = T.E, W = T.W;
  if (tid < WC_STRIDE) sW[tid] = T.world[(size_t)w * WC_STRIDE + tid];
  if (tid == 0) sBits = 0u;
  double *cs = D.cs;
  double *es = D.es;
  // The world's factor plan (local indices), factor values and solve vectors (by position),
  // staged into shared memory as n2_kernel stages them.
  const int wF = D.fb[w + 1] - D.fb[w];
  const int wU = D.ub[w + 1] - D.ub[w];
  const int wR = D.rb[w + 1] - D.rb[w];
  const int wL = D.lb[w + 1] - D.lb[w];
  const int wn = nc;
  const int *colp = D.colp + c0 + w, *lrow = D.lrow + D.fb[w];
  const int *ukp = D.uk_ptr + c0 + w, *ukc = D.uk_col + D.ub[w];
  const int *ukpos = D.uk_pos + D.ub[w], *ukrel = D.uk_rel + D.ub[w];
  const int *rel = D.rel + D.rb[w];
  const int *lvp = D.lv_ptr + D.lb[w] + w, *lvc = D.lv_cols + c0;
  using FT = typename std::conditional<MIX, float, double>::type;
  FT *lval = reinterpret_cast<FT *>(D.lval) + D.fb[w];
  FT *Yv = reinterpret_cast<FT *>(cs + (long long)RC_YV * C) + c0;
  FT *Xv = reinterpret_cast<FT *>(cs + (long long)RC_XV * C) + c0;
  const size_t values = sizeof(FT) * (size_t)(wF + 2 * wn);
  const size_t plan_ints = sizeof(int) * (size_t)(2 * (wn + 1) + wF + 3 * wU + wL + 1 + wn);
  const size_t small_ints = sizeof(int) * (size_t)(2 * (wn + 1) + wL + 1 + wn);
  const int mode = values + plan_ints + sizeof(int) * (size_t)wR <= smem_bytes ? 2
                   : values + plan_ints <= smem_bytes                           ? 1
                   : values + small_ints <= smem_bytes                          ? 3
                                                                                : 0;
  if (mode > 0) {
    lval = reinterpret_cast<FT *>(n2_smem);
    Yv = lval + wF;
    Xv = Yv + wn;
    int *si = reinterpret_cast<int *>(Xv + wn);
    auto stage_ints = [&](const int *src, int count) {
      for (int i = threadIdx.x; i < count; i += BLOCK) si[i] = src[i];
      const int *out = si;
      si += count;
      return out;
    };
    colp = stage_ints(colp, wn + 1);
    if (mode != 3) lrow = stage_ints(lrow, wF);
    ukp = stage_ints(ukp, wn + 1);
    if (mode != 3) {
      ukc = stage_ints(ukc, wU);
      ukpos = stage_ints(ukpos, wU);
      ukrel = stage_ints(ukrel, wU);
    }
    lvp = stage_ints(lvp, wL + 1);
    lvc = stage_ints(lvc, wn);
    if (mode == 2) rel = stage_ints(rel, wR);
  }
  __syncthreads();  // the staged plan, read by dense_tail
  const WorldCholesky<FT, BLOCK> chol{colp, lrow, ukp, ukc, ukpos, ukrel, rel, lvp, lvc,
                                          lval, Yv, Xv, 0, wL, wn,
                                          dense_tail(colp, lvp, lvc, 0, wL, wn)};
  const long long oN = L.s[CB_AMOUNT_INCREMENT], oG = L.s[CB_JUNCTION_GATE];
  const long long oH = L.s[CB_CHANNEL_GATE];
  const double *mctl = control + L.c[CB_CONTROL_MEMBRANE];
  const double *pctlp = control + L.c[CB_CONTROL_PUMP];
  const double *jctl = control + L.c[CB_CONTROL_JUNCTION];
  const double *chctl0 = control + L.c[CB_CONTROL_CHANNEL];
  const double Kc = kChargePerFmol;
  const double h = k.dt;
  const double gh = (1.0 + 1.0 / sqrt(2.0)) * h;  // gamma h
  auto CF = [&](int f, long long gi) -> double & { return cs[(long long)f * C + gi]; };
  auto EF = [&](int f, long long ge) -> double & { return es[(long long)f * E + ge]; };
  auto CH = [&](int q, int f, long long gi) -> double & {
    return cs[(long long)(RC_CH + q * RH_FIELDS + f) * C + gi];
  };
  __syncthreads();
  const double Vb = sW[WC_VB];
  // The ledger fields of a cell's k / new-value rows (RC_K + f) in the state layout.
  const int kCellField[10] = {CB_AMOUNT_INCREMENT, CB_AMOUNT_INCREMENT, CB_AMOUNT_INCREMENT,
                              CB_MEMBRANE_TRANSFERRED, CB_MEMBRANE_TRANSFERRED,
                              CB_MEMBRANE_TRANSFERRED, CB_MEMBRANE_DISSIPATED, CB_PUMP_CYCLES,
                              CB_PUMP_DISSIPATED, CB_METABOLIC_WORK};
  auto cell_state = [&](const double *src, int f, long long gi) {
    return src[L.s[kCellField[f]] + (f < 6 ? (f % 3) * C : 0) + gi];
  };
  auto edge_state = [&](const double *src, int f, long long ge) {
    return f < 3 ? src[L.s[CB_JUNCTION_TRANSFERRED] + f * E + ge]
           : f == 3 ? src[L.s[CB_JUNCTION_DISSIPATED] + ge]
                    : src[oG + ge];
  };
  auto chan_state = [&](const double *src, int q, int f, long long gi) {
    return f < 2 ? src[oH + (f * NCH + q) * C + gi]
           : f == 2 ? src[L.s[CB_CHANNEL_TRANSFERRED] + q * C + gi]
                    : src[L.s[CB_CHANNEL_DISSIPATED] + q * C + gi];
  };
  auto gather = [&](long long gi, int f, double (&send)[3], double (&recv)[3]) {
#pragma unroll
    for (int s = 0; s < 3; ++s) send[s] = recv[s] = 0.0;
    for (int a = __ldg(T.adj_ptr + gi); a < __ldg(T.adj_ptr + gi + 1); ++a) {
      const int code = __ldg(T.adj_idx + a);
      const long long ge = e0 + (code >> 1);
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        if (code & 1) recv[s] += EF(f + s, ge);
        else send[s] += EF(f + s, ge);
      }
    }
  };
  auto potential_of = [&](long long gi, const double (&n)[3]) {
    return (__ldg(T.q0 + gi) + Kc * ((n[0] + n[1]) + (-n[2]))) * __ldg(T.icap + gi) + Vb;
  };
  double res[3], ec, rw, ew;
  for (int s = 0; s < 3; ++s) res[s] = state_in[L.s[CB_RESERVOIR_SUPPLIED] + s * W + w];
  ec = state_in[L.s[CB_ELECTRODE_CHARGE] + w];
  rw = state_in[L.s[CB_RESERVOIR_WORK] + w];
  ew = state_in[L.s[CB_ELECTRODE_WORK] + w];
  const double *cur = state_in;
  int taken = 0;
  uint32_t refused = 0u;

  // The rows that give a stage's state: ROS2's k1, or RK4's previous evaluation.
  constexpr int kCell = RK4 ? RC_R : RC_K, kChan = RK4 ? RH_R : RH_K, kEdge = RK4 ? RE_R : RE_K;
  // The evaluated state of a cell: y + (c h) k (c = 0 at the step's start).
  auto cell_amounts = [&](double c, long long gi, double (&n)[3]) {
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      n[s] = cur[oN + s * C + gi];
      if (c != 0.0) n[s] = n[s] + (c * h) * CF(kCell + s, gi);
    }
  };
  // Right-hand side r at stage st of the state y + (c h) k for every row (ROS2: r = F(y) at
  // st = 0, F(y + h k1) - 2 k1 at st = 1; RK4: r = F), its validity bits, and the world sums it
  // needs: v[0..2] the bath inflow, v[3] the cells' charge rate. At ROS2's st = 0 also the
  // start's slopes, kinetics and the operator's entries.
  auto evaluate = [&](int st, double c_stage, double (&v)[4]) -> uint32_t {
    uint32_t bits = 0;
    const bool sub = !RK4 && st;      // r = F - 2 k1
    const bool start = !RK4 && !st;   // the start's slopes and operator
    for (int q = 0; q < 4; ++q) v[q] = 0.0;
    // Cells: concentrations, potential, own rates (patch, pump, channels), gate rates.
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      double n[3], c[3], lc[3], gl[2 * NQ];
      cell_amounts(c_stage, gi, n);
      const double V = potential_of(gi, n);
      const double ivol = __ldg(T.ivol + gi);
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        c[s] = (__ldg(T.ref + s * C + gi) + n[s]) * ivol;
        lc[s] = log(c[s]);
        CF(RC_CX + s, gi) = c[s];
        CF(RC_LX + s, gi) = lc[s];
      }
      CF(RC_VX, gi) = V;
      for (int q = 0; q < NCH; ++q)
        for (int r = 0; r < 2; ++r) {
          double g = cur[oH + (r * NCH + q) * C + gi];
          if (c_stage != 0.0) g = g + (c_stage * h) * CH(q, kChan + r, gi);
          gl[r * NQ + q] = g;
          if (!(is_finite(g) && g >= 0.0 && g <= 1.0)) bits |= CB_WORLD_DOMAIN;
        }
      const double mc = mctl[gi], pctl = pctlp[gi];
      const double ldc = pctl > 0.0 ? __ldg(T.logpcap + gi) + log(pctl) : 0.0;
      double jm[3], ex[3], r4[4], chj[NQ], chd[NQ];
      bits |= own_rates<NCH>(T, sW, gi, c, lc, V, gl, 1, NQ, mc, pctl, ldc, chctl0 + gi, jm, ex,
                             r4, chj, chd);
      const double dv = V - Vb;
      for (int s = 0; s < 3; ++s) {
        v[s] += jm[s] + ex[s];
        CF(RC_R + s, gi) = ex[s];  // the amounts' rate follows in the gather pass
        CF(RC_R + 3 + s, gi) = sub ? jm[s] - 2.0 * CF(RC_K + 3 + s, gi) : jm[s];
      }
      for (int f = 0; f < 4; ++f)
        CF(RC_R + 6 + f, gi) = sub ? r4[f] - 2.0 * CF(RC_K + 6 + f, gi) : r4[f];
      for (int q = 0; q < NCH; ++q) {
        const int code = __ldg(T.ch_code + q * C + gi);
        double t[2], tau[2];
        channel_kinetics<false>(code, dv, t, tau);
        if (!channel_kinetics_ok(dv, t, tau)) bits |= CB_WORLD_CHANNEL_DOMAIN;
        // Gate rates (target - g)/tau of the rows with a law (HH K's h row has none).
        const double rr[4] = {(t[0] - gl[q]) / tau[0],
                              code == kHhKn4 ? 0.0 : (t[1] - gl[NQ + q]) / tau[1], chj[q],
                              chd[q]};
        for (int f = 0; f < 4; ++f)
          CH(q, RH_R + f, gi) = sub ? rr[f] - 2.0 * CH(q, RH_K + f, gi) : rr[f];
        if (start) {
          double dtg[2], dtau[2];
          channel_slope(code, dv, dtg, dtau);
          for (int r = 0; r < 2; ++r) {
            const bool live = !(r == 1 && code == kHhKn4);
            const double cpl = dtg[r] / tau[r] - (t[r] - gl[r * NQ + q]) * dtau[r] / (tau[r] * tau[r]);
            CH(q, RH_DEC + r, gi) = live ? 1.0 / tau[r] : 0.0;
            CH(q, RH_CPL + r, gi) = live && is_finite(cpl) ? cpl : 0.0;
          }
          CH(q, RH_J0, gi) = chj[q];
        }
      }
      if (start) {
        // The start's slopes (N2's route_slope at y), fluxes and differences for the heat rows;
        // the patch conductance into RC_MD until the operator pass.
        double mu[3], zw[3];
        patch_mu(sW, lc, dv, mu);
        for (int s = 0; s < 3; ++s) {
          const double zfrt = (s < 2 ? 1.0 : -1.0) * sW[WC_FRT];
          const double W_ = route_slope(__ldg(T.ap + s * C + gi) * mc, c[s], sW[WC_CO + s], dv,
                                        zfrt);
          CF(RC_WM + s, gi) = W_;
          CF(RC_JM0 + s, gi) = jm[s];
          CF(RC_MU0 + s, gi) = mu[s];
          zw[s] = (s < 2 ? 1.0 : -1.0) * W_;
          if (!is_finite(W_)) bits |= CB_WORLD_OPERATOR;
        }
        double gp = Kc * ((zw[0] + zw[1]) + zw[2]);
        if constexpr (NCH > 0) {
          double extra = 0.0;
          for (int q = 0; q < NCH; ++q) {
            const int code = __ldg(T.ch_code + q * C + gi);
            const int sp = __ldg(T.ch_species + q * C + gi);
            const double available =
                (__ldg(T.ch_ab + q * C + gi) * channel_opening(code, gl[q], gl[NQ + q])) *
                __ldg(chctl0 + q * C + gi);
            const double zfrt = (sp < 2 ? 1.0 : -1.0) * sW[WC_FRT];
            const double W_ = route_slope(__ldg(T.ch_ap + q * C + gi) * available, c[sp],
                                          sW[WC_CO + sp], dv, zfrt);
            CH(q, RH_W, gi) = W_;
            if (!is_finite(W_)) bits |= CB_WORLD_OPERATOR;
            extra = extra + Kc * ((sp < 2 ? 1.0 : -1.0) * W_);
          }
          gp = gp + extra;
        }
        CF(RC_MD, gi) = gp;
        const int P = __ldg(D.rank + gi);
        for (int f = colp[P]; f < colp[P + 1]; ++f) lval[f] = 0.0;
      }
    }
    __syncthreads();
    // Junctions: fluxes, heat, the gate law's rate; at st = 0 the start's slopes and kinetics.
    for (int e = tid; e < ne; e += BLOCK) {
      const long long ge = e0 + e;
      const long long ga = c0 + __ldg(T.snd + ge), gb = c0 + __ldg(T.rcv + ge);
      double ca[3], cb[3], la[3], lb[3], jj[3], jd;
      for (int s = 0; s < 3; ++s) {
        ca[s] = CF(RC_CX + s, ga);
        cb[s] = CF(RC_CX + s, gb);
        la[s] = CF(RC_LX + s, ga);
        lb[s] = CF(RC_LX + s, gb);
      }
      const double dv = CF(RC_VX, ga) - CF(RC_VX, gb);
      double g = cur[oG + ge];
      if (c_stage != 0.0) g = g + (c_stage * h) * EF(kEdge + 4, ge);
      const double jc = jctl[ge];
      bits |= junction_flux(T, sW, ge, ca, cb, la, lb, dv, jc * g, jj, jd);
      const double thr = __ldg(T.thr + ge), mn = __ldg(T.jmin + ge);
      if (!gate_domain(g, dv, thr, mn, jc)) bits |= CB_WORLD_GATE_DOMAIN;
      // junction_voltage_relaxation's rate; pinned gates (minimum 1) exactly 0.
      double gr = 0.0, relax = 0.0;
      if (mn < 1.0) {
        const double shift = fabs(dv) - thr;
        const double alpha = 1.3 * exp(-77.0 * shift);
        const double log_beta = kLog0065 + 140.0 * shift;
        const double beta = 20.0 * exp(-logaddexp0(-log_beta));
        gr = alpha * (1.0 - g) - beta * (g - mn);
        relax = alpha + beta;
      }
      if (!is_finite(gr)) bits |= CB_WORLD_TRANSPORT;
      const double rr[5] = {jj[0], jj[1], jj[2], jd, gr};
      for (int s = 0; s < 3; ++s) EF(RE_J + s, ge) = jj[s];
      for (int f = 0; f < 5; ++f) EF(RE_R + f, ge) = sub ? rr[f] - 2.0 * EF(RE_K + f, ge) : rr[f];
      if (start) {
        double mu[3], zw[3];
        junction_mu(sW, la, lb, dv, mu);
        for (int s = 0; s < 3; ++s) {
          const double zfrt = (s < 2 ? 1.0 : -1.0) * sW[WC_FRT];
          const double W_ = route_slope(__ldg(T.jap + s * E + ge) * (jc * g), ca[s], cb[s], dv,
                                        zfrt);
          EF(RE_W + s, ge) = W_;
          EF(RE_JJ0 + s, ge) = jj[s];
          EF(RE_MU0 + s, ge) = mu[s];
          zw[s] = (s < 2 ? 1.0 : -1.0) * W_;
          if (!is_finite(W_)) bits |= CB_WORLD_OPERATOR;
        }
        EF(RE_G, ge) = Kc * ((zw[0] + zw[1]) + zw[2]);
        EF(RE_DEC, ge) = is_finite(relax) ? relax : 0.0;
      }
    }
    __syncthreads();
    // Cells: the amounts' rate (own parts, then the junctions in edge order), the charge rate
    // and the scaled right-hand side of the voltage solve; at st = 0 the operator's diagonal.
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      double send[3], recv[3], r[3];
      gather(gi, RE_J, send, recv);
      for (int s = 0; s < 3; ++s) {
        // the patch flux J_m (RC_R + 3 holds J_m - 2 k1 at st = 1)
        const double jm = sub ? CF(RC_R + 3 + s, gi) + 2.0 * CF(RC_K + 3 + s, gi)
                              : CF(RC_R + 3 + s, gi);
        const double whole = ((-jm + (-send[s])) + recv[s]) - CF(RC_R + s, gi);
        r[s] = sub ? whole - 2.0 * CF(RC_K + s, gi) : whole;
        CF(RC_R + s, gi) = r[s];
        if (!is_finite(r[s])) bits |= CB_WORLD_TRANSPORT;
      }
      const double qdot = Kc * ((r[0] + r[1]) + (-r[2]));
      // F's charge rate for the electrode row (r = F - 2 k1 at st = 1)
      v[3] += sub ? Kc * (((r[0] + 2.0 * CF(RC_K, gi)) + (r[1] + 2.0 * CF(RC_K + 1, gi))) +
                         (-(r[2] + 2.0 * CF(RC_K + 2, gi))))
                 : qdot;
      if (start) {
        double gs = 0.0, gq = 0.0;
        for (int a = __ldg(T.adj_ptr + gi); a < __ldg(T.adj_ptr + gi + 1); ++a) {
          const int code = __ldg(T.adj_idx + a);
          const double g = EF(RE_G, e0 + (code >> 1));
          if (code & 1) gq += g;
          else gs += g;
        }
        const double cap = 1.0 / __ldg(T.icap + gi);
        const double mii = cap + gh * (CF(RC_MD, gi) + (gs + gq));
        CF(RC_MD, gi) = mii;
        if (!(mii > 0.0)) bits |= CB_WORLD_OPERATOR;
        const double sc = 1.0 / sqrt(mii > 0.0 ? mii : 1.0);
        CF(RC_S, gi) = sc;
        lval[colp[__ldg(D.rank + gi)]] = (FT)((mii * sc) * sc);
      }
      if (!RK4) Yv[__ldg(D.rank + gi)] = (FT)(qdot * CF(RC_S, gi));
    }
    __syncthreads();
    if (start) {
      // Junctions: the operator's off-diagonal entries, scaled (row then column).
      for (int e = tid; e < ne; e += BLOCK) {
        const long long ge = e0 + e;
        const long long ga = c0 + __ldg(T.snd + ge), gb = c0 + __ldg(T.rcv + ge);
        const int ra = __ldg(D.rank + ga), rb = __ldg(D.rank + gb);
        const double m = 0.0 + gh * (-EF(RE_G, ge));
        const double s_row = ra > rb ? CF(RC_S, ga) : CF(RC_S, gb);
        const double s_col = ra > rb ? CF(RC_S, gb) : CF(RC_S, ga);
        lval[__ldg(D.edge_pos + ge)] = (FT)((m * s_row) * s_col);
      }
      __syncthreads();
    }
    return bits;
  };
  // k = W^-1 r after the voltage solve: u, each route's rate r + gamma h W du, the heat rows
  // through W du mu + J z F du at the start, the gates' (r + gamma h dg'/dV u)/(1 + gamma h
  // lambda), the pump's k = r. st = 0 keeps k1; st = 1 writes the step's new values
  // y + 3/2 h k1 + 1/2 h k2 over it. v[0..2]: the bath's correction sum of the patches' route
  // corrections, v[3] the cells' charge correction.
  auto correct = [&](int st, double (&v)[4]) -> uint32_t {
    uint32_t bits = 0;
    for (int q = 0; q < 4; ++q) v[q] = 0.0;
    chol.solve();
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      const double u = (double)Xv[__ldg(D.rank + gi)] * CF(RC_S, gi);
      CF(RC_U, gi) = u;
      if (tp.factor) tp.u[st * C + gi] = u;
      if (!is_finite(u)) bits |= CB_WORLD_RESIDUAL;
    }
    __syncthreads();
    auto finish = [&](double r, double &kslot, double y) {
      const double kv = r;
      if (st == 0) {
        kslot = kv;
      } else {
        kslot = (y + (1.5 * h) * kslot) + (0.5 * h) * kv;
      }
    };
    // Junctions: route corrections W du (for the cells' gather), transfers, heat, gate.
    for (int e = tid; e < ne; e += BLOCK) {
      const long long ge = e0 + e;
      const long long ga = c0 + __ldg(T.snd + ge), gb = c0 + __ldg(T.rcv + ge);
      const double du = CF(RC_U, ga) - CF(RC_U, gb);
      double dj[3], hm[3];
      for (int s = 0; s < 3; ++s) {
        dj[s] = EF(RE_W + s, ge) * du;
        EF(RE_J + s, ge) = dj[s];
        hm[s] = dj[s] * EF(RE_MU0 + s, ge) + EF(RE_JJ0 + s, ge) * ((s < 2 ? kF : -kF) * du);
      }
      const double heat = 1e-3 * ((hm[0] + hm[1]) + hm[2]);
      double kv[5];
      for (int s = 0; s < 3; ++s) kv[s] = EF(RE_R + s, ge) + gh * dj[s];
      kv[3] = EF(RE_R + 3, ge) + gh * heat;
      kv[4] = EF(RE_R + 4, ge) / (1.0 + gh * EF(RE_DEC, ge));
      if (tp.factor) (st ? tp.k2g : tp.k1g)[ge] = kv[4];
      for (int f = 0; f < 5; ++f) {
        if (!is_finite(kv[f])) bits |= CB_WORLD_TRANSPORT;
        finish(kv[f], EF(RE_K + f, ge), st ? edge_state(cur, f, ge) : 0.0);
      }
    }
    __syncthreads();
    // Cells: the amounts through the patches' and junctions' corrections (route_rates' order:
    // receivers less senders less patches), the patch ledgers, the pump's rows, the channels.
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      const double u = CF(RC_U, gi);
      double send[3], recv[3], dm[3], pm[3], hm[3];
      gather(gi, RE_J, send, recv);
      for (int s = 0; s < 3; ++s) {
        dm[s] = CF(RC_WM + s, gi) * u;
        pm[s] = dm[s];
        hm[s] = dm[s] * CF(RC_MU0 + s, gi) + CF(RC_JM0 + s, gi) * ((s < 2 ? kF : -kF) * u);
      }
      double kch[NQ][4];
      for (int q = 0; q < NCH; ++q) {
        const int sp = __ldg(T.ch_species + q * C + gi);
        const double dc = CH(q, RH_W, gi) * u;
        pm[sp] = pm[sp] + dc;
        const double zf = sp < 2 ? kF : -kF;
        const double musp = CF(RC_MU0 + sp, gi);
        for (int r = 0; r < 2; ++r)
          kch[q][r] = (CH(q, RH_R + r, gi) + gh * (CH(q, RH_CPL + r, gi) * u)) /
                      (1.0 + gh * CH(q, RH_DEC + r, gi));
        kch[q][2] = CH(q, RH_R + 2, gi) + gh * dc;
        kch[q][3] = CH(q, RH_R + 3, gi) + gh * (1e-3 * (dc * musp + CH(q, RH_J0, gi) * (zf * u)));
      }
      double kv[10], corr[3];
      for (int s = 0; s < 3; ++s) {
        corr[s] = (recv[s] - send[s]) - pm[s];
        kv[s] = CF(RC_R + s, gi) + gh * corr[s];
        kv[3 + s] = CF(RC_R + 3 + s, gi) + gh * dm[s];
        v[s] += pm[s];
      }
      v[3] += Kc * ((corr[0] + corr[1]) + (-corr[2]));
      if (tp.factor) {
        if (st == 0)
          for (int s = 0; s < 3; ++s) tp.k1n[s * C + gi] = kv[s];
        for (int q = 0; q < NCH; ++q)
          for (int r = 0; r < 2; ++r) (st ? tp.k2gc : tp.k1gc)[(r * NCH + q) * C + gi] = kch[q][r];
      }
      kv[6] = CF(RC_R + 6, gi) + gh * (1e-3 * ((hm[0] + hm[1]) + hm[2]));
      for (int f = 7; f < 10; ++f) kv[f] = CF(RC_R + f, gi);
      for (int f = 0; f < 10; ++f) {
        if (!is_finite(kv[f])) bits |= CB_WORLD_TRANSPORT;
        finish(kv[f], CF(RC_K + f, gi), st ? cell_state(cur, f, gi) : 0.0);
      }
      for (int q = 0; q < NCH; ++q)
        for (int f = 0; f < 4; ++f) {
          if (!is_finite(kch[q][f])) bits |= CB_WORLD_TRANSPORT;
          finish(kch[q][f], CH(q, RH_K + f, gi), st ? chan_state(cur, q, f, gi) : 0.0);
        }
    }
    __syncthreads();
    return bits;
  };
  // The world rows (bath supply [3], electrode charge, reservoir work, electrode work): F's
  // from an evaluation's sums (the supply -inflow, the electrode -sum of the cells' charge
  // rates, the works 1e-3 mu_bath . supply and 1e12 V_bath electrode), and their correction
  // rows from the corrections' sums, the same linear maps.
  const double mub[3] = {sW[WC_MUB], sW[WC_MUB + 1], sW[WC_MUB + 2]};
  auto world_map = [&](const double (&v)[4], double (&out)[6]) {
    for (int s = 0; s < 3; ++s) out[s] = -v[s];
    out[3] = -v[3];
    out[4] = 1e-3 * ((mub[0] * out[0] + mub[1] * out[1]) + mub[2] * out[2]);
    out[5] = (1e12 * Vb) * out[3];
  };

  // RK4: the evaluation's rows into the running sum k1 + 2 k2 + 2 k3 + k4 (RC_K, RH_K, RE_K).
  auto accumulate = [&](int st, double wgt) {
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      for (int f = 0; f < 10; ++f)
        CF(RC_K + f, gi) = st ? CF(RC_K + f, gi) + wgt * CF(RC_R + f, gi) : CF(RC_R + f, gi);
      for (int q = 0; q < NCH; ++q)
        for (int f = 0; f < 4; ++f)
          CH(q, RH_K + f, gi) = st ? CH(q, RH_K + f, gi) + wgt * CH(q, RH_R + f, gi)
                                   : CH(q, RH_R + f, gi);
    }
    for (int e = tid; e < ne; e += BLOCK) {
      const long long ge = e0 + e;
      for (int f = 0; f < 5; ++f)
        EF(RE_K + f, ge) = st ? EF(RE_K + f, ge) + wgt * EF(RE_R + f, ge) : EF(RE_R + f, ge);
    }
  };
  // RK4: the new values y + (h / 6) (k1 + 2 k2 + 2 k3 + k4) over the sum.
  auto rk4_finish = [&]() {
    const double h6 = h / 6.0;
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      for (int f = 0; f < 10; ++f) CF(RC_K + f, gi) = cell_state(cur, f, gi) + h6 * CF(RC_K + f, gi);
      for (int q = 0; q < NCH; ++q)
        for (int f = 0; f < 4; ++f)
          CH(q, RH_K + f, gi) = chan_state(cur, q, f, gi) + h6 * CH(q, RH_K + f, gi);
    }
    for (int e = tid; e < ne; e += BLOCK) {
      const long long ge = e0 + e;
      for (int f = 0; f < 5; ++f) EF(RE_K + f, ge) = edge_state(cur, f, ge) + h6 * EF(RE_K + f, ge);
    }
  };

  for (int step = 0; step < n_steps; ++step) {
    uint32_t bits = 0;
    double ve[4], vc[4], fw[6], cw[6], k1w[6], k2w[6], neww[6];
    const double yw[6] = {res[0], res[1], res[2], ec, rw, ew};
    if constexpr (RK4) {
      // fixed_step.rk4_checked_step (:25-71): four evaluations at y, y + h/2 k1, y + h/2 k2,
      // y + h k3, each of a valid trial state.
      const double cst[4] = {0.0, 0.5, 0.5, 1.0}, wst[4] = {1.0, 2.0, 2.0, 1.0};
      for (int st = 0; st < 4; ++st) {
        bits |= evaluate(st, cst[st], ve);
        block_sum<BLOCK, 4>(ve, sRed);
        world_map(ve, fw);
        for (int f = 0; f < 6; ++f) k1w[f] = st ? k1w[f] + wst[st] * fw[f] : fw[f];
        accumulate(st, wst[st]);
        __syncthreads();
      }
      rk4_finish();
      __syncthreads();
      for (int f = 0; f < 6; ++f) {
        neww[f] = yw[f] + (h / 6.0) * k1w[f];
        if (!is_finite(neww[f])) bits |= CB_WORLD_DOMAIN;
      }
      (void)vc;
      (void)cw;
      (void)k2w;
    } else {
      // Stage 1: F(y), the operator at y, k1.
      bits |= evaluate(0, 0.0, ve);
      block_sum<BLOCK, 4>(ve, sRed);
      if (chol.factor()) bits |= CB_WORLD_OPERATOR;
      if (tp.factor) {  // the reverse's record: the factor and its scale
        for (int f = tid; f < wF; f += BLOCK) tp.factor[D.fb[w] + f] = (double)lval[f];
        for (int i = tid; i < nc; i += BLOCK) tp.scale[c0 + i] = CF(RC_S, c0 + i);
      }
      bits |= correct(0, vc);
      block_sum<BLOCK, 4>(vc, sRed);
      world_map(ve, fw);
      world_map(vc, cw);
      for (int f = 0; f < 6; ++f) k1w[f] = fw[f] + gh * cw[f];
      // Stage 2: F(y + h k1) - 2 k1 through the same factor; the new values.
      bits |= evaluate(1, 1.0, ve);
      block_sum<BLOCK, 4>(ve, sRed);
      bits |= correct(1, vc);
      block_sum<BLOCK, 4>(vc, sRed);
      world_map(ve, fw);
      world_map(vc, cw);
      for (int f = 0; f < 6; ++f) {
        k2w[f] = (fw[f] - 2.0 * k1w[f]) + gh * cw[f];
        neww[f] = (yw[f] + (1.5 * h) * k1w[f]) + (0.5 * h) * k2w[f];
        if (!is_finite(neww[f])) bits |= CB_WORLD_DOMAIN;
      }
    }
    // The new state's domain: positive amounts, gates in range, finite ledgers.
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      bool ok = true;
      for (int f = 0; f < 10; ++f) ok = ok && is_finite(CF(RC_K + f, gi));
      for (int s = 0; s < 3; ++s) ok = ok && (__ldg(T.ref + s * C + gi) + CF(RC_K + s, gi)) > 0.0;
      for (int q = 0; q < NCH; ++q) {
        for (int f = 0; f < 4; ++f) ok = ok && is_finite(CH(q, RH_K + f, gi));
        for (int r = 0; r < 2; ++r) {
          const double g = CH(q, RH_K + r, gi);
          ok = ok && g >= 0.0 && g <= 1.0;
        }
      }
      if (!ok) bits |= CB_WORLD_DOMAIN;
    }
    for (int e = tid; e < ne; e += BLOCK) {
      const long long ge = e0 + e;
      bool ok = true;
      for (int f = 0; f < 5; ++f) ok = ok && is_finite(EF(RE_K + f, ge));
      const double g = EF(RE_K + 4, ge);
      ok = ok && g >= __ldg(T.jmin + ge) && g <= 1.0;
      if (!ok) bits |= CB_WORLD_DOMAIN;
    }
    if (bits) atomicOr(&sBits, bits);
    __syncthreads();
    const uint32_t world_bits = sBits;
    if (world_bits) {
      refused = world_bits;
      break;
    }
    // Commit the accepted state.
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      for (int f = 0; f < 10; ++f)
        state_out[L.s[kCellField[f]] + (f < 6 ? (f % 3) * C : 0) + gi] = CF(RC_K + f, gi);
      for (int q = 0; q < NCH; ++q) {
        for (int r = 0; r < 2; ++r) state_out[oH + (r * NCH + q) * C + gi] = CH(q, RH_K + r, gi);
        state_out[L.s[CB_CHANNEL_TRANSFERRED] + q * C + gi] = CH(q, RH_K + 2, gi);
        state_out[L.s[CB_CHANNEL_DISSIPATED] + q * C + gi] = CH(q, RH_K + 3, gi);
      }
    }
    for (int e = tid; e < ne; e += BLOCK) {
      const long long ge = e0 + e;
      for (int s = 0; s < 3; ++s)
        state_out[L.s[CB_JUNCTION_TRANSFERRED] + s * E + ge] = EF(RE_K + s, ge);
      state_out[L.s[CB_JUNCTION_DISSIPATED] + ge] = EF(RE_K + 3, ge);
      state_out[oG + ge] = EF(RE_K + 4, ge);
    }
    for (int s = 0; s < 3; ++s) res[s] = neww[s];
    ec = neww[3];
    rw = neww[4];
    ew = neww[5];
    ++taken;
    cur = state_out;
    __syncthreads();
  }
  // A world refused at its first step keeps its input state.
  if (taken == 0 && state_in != state_out) {
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      for (int f = CB_AMOUNT_INCREMENT; f <= CB_METABOLIC_WORK; ++f) {
        const int reps = (f <= CB_MEMBRANE_TRANSFERRED) ? 3 : 1;
        for (int s = 0; s < reps; ++s)
          state_out[L.s[f] + s * C + gi] = state_in[L.s[f] + s * C + gi];
      }
      for (int f = CB_CHANNEL_GATE; f <= CB_CHANNEL_DISSIPATED; ++f) {
        const int reps = (f == CB_CHANNEL_GATE) ? 2 * NCH : NCH;
        for (int s = 0; s < reps; ++s)
          state_out[L.s[f] + s * C + gi] = state_in[L.s[f] + s * C + gi];
      }
    }
    for (int e = tid; e < ne; e += BLOCK) {
      const long long ge = e0 + e;
      for (int f = CB_JUNCTION_TRANSFERRED; f <= CB_JUNCTION_GATE; ++f) {
        const int reps = (f == CB_JUNCTION_TRANSFERRED) ? 3 : 1;
        for (int s = 0; s < reps; ++s)
          state_out[L.s[f] + s * E + ge] = state_in[L.s[f] + s * E + ge];
      }
    }
  }
  if (tid == 0) {
    for (int s = 0; s < 3; ++s) state_out[L.s[CB_RESERVOIR_SUPPLIED] + s * W + w] = res[s];
    state_out[L.s[CB_ELECTRODE_CHARGE] + w] = ec;
    state_out[L.s[CB_RESERVOIR_WORK] + w] = rw;
    state_out[L.s[CB_ELECTRODE_WORK] + w] = ew;
    world_status[w] = refused;
    if (accepted_steps) accepted_steps[w] = taken;
  }
}

template <typename V>
int upload_vec(N2Plan *plan, const std::vector<V> &host, V **dst) {
  void *ptr = nullptr;
  const size_t bytes = std::max<size_t>(host.size() * sizeof(V), 16);
  cudaError_t e = cudaMalloc(&ptr, bytes);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc (N2 plan)");
  plan->owned.push_back(ptr);
  if (!host.empty()) {
    e = cudaMemcpy(ptr, host.data(), host.size() * sizeof(V), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy (N2 plan)");
  }
  *dst = static_cast<V *>(ptr);
  return CB_OK;
}

int build_plan(cb_tissue *t) {
  if (t->n2) return CB_OK;
  auto *plan = new N2Plan();
  const int W = t->W;
  const long long C = t->C, E = t->E;
  std::vector<int> rank(C), colp, lrow, uk_ptr, uk_col, uk_pos, uk_rel, rel, lv_ptr, lv_cols(C),
      edge_pos(E), fb{0}, ub{0}, rb{0}, lb{0};
  // Shared memory per CTA: for each world the largest of its stagings that fits the cap (the
  // whole plan; all but the relative positions; the factor values, solve vectors and the
  // per-column index arrays), the batch's maximum of those. The cap keeps the register budget's
  // CTAs per SM resident (110 KB at two, 200 KB at one): measured on 512 1024-cell worlds, whose
  // factor values alone take 136 KB, the ROS2 step runs at 9.1 ms from global memory at two CTAs
  // per SM against 12.4 ms with the values staged at one. Overrides for sweeps:
  // CELLS_B200_N2_SMEM (KB), CELLS_B200_N2_BLOCK (128 or 256), CELLS_B200_N2_MINB (1, or 2:
  // registers capped for more resident CTAs).
  if (const char *env = std::getenv("CELLS_B200_N2_BLOCK"))
    plan->block = std::atoi(env) == 128 ? 128 : 256;
  if (const char *env = std::getenv("CELLS_B200_N2_MINB"))
    plan->min_blocks = std::atoi(env) >= 2 ? 2 : 1;
  size_t cap = plan->min_blocks >= 2 ? 110 * 1024 : 200 * 1024;
  if (const char *env = std::getenv("CELLS_B200_N2_SMEM")) cap = (size_t)std::atoi(env) * 1024;
  size_t shared = 0, shared_f32 = 0;  // FP64 values; FP32 values (CB_METHOD_ROS2_MIXED)
  int rc = CB_OK;
  for (int w = 0; w < W && !rc; ++w) {
    const long long c0 = t->h_cell_offset[w], n = t->h_cell_offset[w + 1] - c0;
    const long long e0 = t->h_edge_offset[w], ne = t->h_edge_offset[w + 1] - e0;
    WorldPlan p;
    rc = plan_world((int)n, t->h_snd.data() + e0, t->h_rcv.data() + e0, (int)ne, p);
    if (rc) break;
    const long long F = p.colp[n], U = (long long)p.uk_col.size(), R = (long long)p.rel.size();
    const long long L = (long long)p.level_ptr.size() - 1;
    if (fb.back() + F >= (1LL << 31) || ub.back() + U >= (1LL << 31) ||
        rb.back() + R >= (1LL << 31)) {
      rc = fail(CB_ERR_UNSUPPORTED, "N2: the batch's factor plan exceeds 2^31 entries");
      break;
    }
    for (long long i = 0; i < n; ++i) rank[c0 + i] = p.rank[i];
    colp.insert(colp.end(), p.colp.begin(), p.colp.end());
    lrow.insert(lrow.end(), p.lrow.begin(), p.lrow.end());
    uk_ptr.insert(uk_ptr.end(), p.uk_ptr.begin(), p.uk_ptr.end());
    uk_col.insert(uk_col.end(), p.uk_col.begin(), p.uk_col.end());
    uk_pos.insert(uk_pos.end(), p.uk_pos.begin(), p.uk_pos.end());
    uk_rel.insert(uk_rel.end(), p.uk_rel.begin(), p.uk_rel.end());
    rel.insert(rel.end(), p.rel.begin(), p.rel.end());
    lv_ptr.insert(lv_ptr.end(), p.level_ptr.begin(), p.level_ptr.end());
    for (long long r = 0; r < n; ++r) lv_cols[c0 + r] = p.level_cols[r];
    for (long long e = 0; e < ne; ++e) edge_pos[e0 + e] = p.edge_pos[e];
    fb.push_back((int)(fb.back() + F));
    ub.push_back((int)(ub.back() + U));
    rb.push_back((int)(rb.back() + R));
    lb.push_back((int)(lb.back() + L));
    plan->max_level = std::max(plan->max_level, (int)L);
    // Shared-memory footprint: values and vectors, then the plan's integers.
    const size_t values = sizeof(double) * (size_t)(F + 2 * n);
    const size_t ints = sizeof(int) * (size_t)(2 * (n + 1) + F + 3 * U + L + 1 + n);
    const size_t all = values + ints + sizeof(int) * (size_t)R;
    const size_t small = values + sizeof(int) * (size_t)(2 * (n + 1) + L + 1 + n);
    const size_t fits = all <= cap ? all : values + ints <= cap ? values + ints
                        : small <= cap ? small : 0;
    shared = std::max(shared, fits);
    const size_t v32 = values / 2, a32 = all - values / 2, s32 = small - values / 2;
    const size_t fits32 = a32 <= cap ? a32 : v32 + ints <= cap ? v32 + ints : s32 <= cap ? s32 : 0;
    shared_f32 = std::max(shared_f32, fits32);
  }
  if (rc) {
    delete plan;
    return rc;
  }
  plan->factor_entries = fb.back();
  plan->update_terms = rb.back();
  plan->levels = lb.back();
  // A world none of whose stagings fits works from global memory. With nothing staged the ROS2
  // kernel runs 128-thread CTAs, four per SM (512 1024-cell worlds: 7.2 ms per step against 8.97
  // at 256 threads, two per SM; the 16x16 grid, whose plans are staged: 5.3 against 4.4).
  plan->smem_bytes = shared;
  plan->smem_f32 = shared_f32;
  plan->ros2_block = shared == 0 ? 128 : 256;
  plan->ros2_block_f32 = shared_f32 == 0 ? 128 : 256;
  if (const char *env = std::getenv("CELLS_B200_N2_BLOCK"))
    plan->ros2_block = plan->ros2_block_f32 = std::atoi(env) == 128 ? 128 : 256;
  N2Dev &d = plan->d;
  if (!rc) rc = upload_vec(plan, rank, &d.rank);
  if (!rc) rc = upload_vec(plan, colp, &d.colp);
  if (!rc) rc = upload_vec(plan, lrow, &d.lrow);
  if (!rc) rc = upload_vec(plan, uk_ptr, &d.uk_ptr);
  if (!rc) rc = upload_vec(plan, uk_col, &d.uk_col);
  if (!rc) rc = upload_vec(plan, uk_pos, &d.uk_pos);
  if (!rc) rc = upload_vec(plan, uk_rel, &d.uk_rel);
  if (!rc) rc = upload_vec(plan, rel, &d.rel);
  if (!rc) rc = upload_vec(plan, lv_ptr, &d.lv_ptr);
  if (!rc) rc = upload_vec(plan, lv_cols, &d.lv_cols);
  if (!rc) rc = upload_vec(plan, edge_pos, &d.edge_pos);
  if (!rc) rc = upload_vec(plan, fb, &d.fb);
  if (!rc) rc = upload_vec(plan, ub, &d.ub);
  if (!rc) rc = upload_vec(plan, rb, &d.rb);
  if (!rc) rc = upload_vec(plan, lb, &d.lb);
  if (!rc) rc = upload_vec(plan, std::vector<double>((size_t)fb.back()), &d.lval);
  // Scratch for either kernel (N2's or ROS2's fields, whichever needs more).
  const size_t cell_fields = std::max(n2_cell_fields(t->t.nch), ros2_cell_fields(t->t.nch));
  const size_t edge_fields = std::max<size_t>(NE_FIELDS, RE_FIELDS);
  if (!rc) rc = upload_vec(plan, std::vector<double>(cell_fields * C), &d.cs);
  if (!rc) rc = upload_vec(plan, std::vector<double>(edge_fields * std::max(E, 1LL)), &d.es);
  if (rc) {
    for (void *ptr : plan->owned) cudaFree(ptr);
    delete plan;
    return rc;
  }
  t->n2 = plan;
  return CB_OK;
}

template <int NCH>
int launch_n2(cb_tissue *t, const double *in, double *out, const double *control,
              const StepCoef &k, int n_steps, uint32_t *status, int32_t *taken,
              cudaStream_t stream, bool mix) {
  const size_t smem = t->n2->smem_bytes;
  const int block = t->n2->block, minb = t->n2->min_blocks;
  auto kern = mix ? n2_kernel<256, NCH, 1, true> : n2_kernel<256, NCH, 1, false>;
  if (block == 128)
    kern = minb >= 2 ? (mix ? n2_kernel<128, NCH, 4, true> : n2_kernel<128, NCH, 4, false>)
                     : (mix ? n2_kernel<128, NCH, 1, true> : n2_kernel<128, NCH, 1, false>);
  else if (minb >= 2)
    kern = mix ? n2_kernel<256, NCH, 2, true> : n2_kernel<256, NCH, 2, false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute (n2)");
  kern<<<t->W, block, smem, stream>>>(t->t, t->layout, t->n2->d, in, out, control, k, n_steps,
                                      status, taken, smem);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "n2 launch");
  return CB_OK;
}

template <int NCH>
int launch_ros2(cb_tissue *t, const double *in, double *out, const double *control,
                const StepCoef &k, int n_steps, uint32_t *status, int32_t *taken,
                cudaStream_t stream, bool rk4, bool mix, const R2Tape &tape) {
  // Registers capped for two CTAs per SM (N2's measured choice), unless CELLS_B200_N2_MINB=1;
  // 128-thread CTAs at four per SM where the plan chose them (ros2_block).
  const int block = mix ? t->n2->ros2_block_f32 : t->n2->ros2_block;
  const size_t smem = mix ? t->n2->smem_f32 : t->n2->smem_bytes;
  auto kern = rk4   ? ros2_kernel<256, NCH, 2, true, false>
              : mix ? ros2_kernel<256, NCH, 2, false, true>
                    : ros2_kernel<256, NCH, 2, false, false>;
  if (block == 128)
    kern = rk4   ? ros2_kernel<128, NCH, 4, true, false>
           : mix ? ros2_kernel<128, NCH, 4, false, true>
                 : ros2_kernel<128, NCH, 4, false, false>;
  else if (t->n2->min_blocks < 2)
    kern = rk4   ? ros2_kernel<256, NCH, 1, true, false>
           : mix ? ros2_kernel<256, NCH, 1, false, true>
                 : ros2_kernel<256, NCH, 1, false, false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute (ros2)");
  kern<<<t->W, block, smem, stream>>>(t->t, t->layout, t->n2->d, in, out, control, k, n_steps,
                                      status, taken, smem, tape);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "ros2 launch");
  return CB_OK;
}

}  // namespace

namespace cbk {

int ros2_step(cb_tissue *t, const double *state_in, double *state_out, double dt,
              const double *control, int n_steps, uint32_t *world_status,
              int32_t *accepted_steps, cudaStream_t stream, bool rk4, bool mix) {
  return ros2_step_tape(t, state_in, state_out, dt, control, n_steps, world_status,
                        accepted_steps, stream, rk4, mix, R2Tape{});
}

int ros2_step_tape(cb_tissue *t, const double *state_in, double *state_out, double dt,
                   const double *control, int n_steps, uint32_t *world_status,
                   int32_t *accepted_steps, cudaStream_t stream, bool rk4, bool mix,
                   const R2Tape &tape) {
  if (tape.factor && (rk4 || mix || n_steps != 1))
    return fail(CB_ERR_ARGUMENT, "a ROS2 record covers one FP64 ROS2 step");
  int rc = build_plan(t);
  if (rc) return rc;
  const StepCoef k = step_coef(dt);
  if (t->t.nch == 2)
    return launch_ros2<2>(t, state_in, state_out, control, k, n_steps, world_status,
                          accepted_steps, stream, rk4, mix, tape);
  if (t->t.nch == 0)
    return launch_ros2<0>(t, state_in, state_out, control, k, n_steps, world_status,
                          accepted_steps, stream, rk4, mix, tape);
  return fail(CB_ERR_UNSUPPORTED, "channel slots must be 0 or 2");
}


int n2_step(cb_tissue *t, const double *state_in, double *state_out, double dt,
            const double *control, int n_steps, uint32_t *world_status, int32_t *accepted_steps,
            cudaStream_t stream, bool mix) {
  int rc = build_plan(t);
  if (rc) return rc;
  const StepCoef k = step_coef(dt);
  if (t->t.nch == 2)
    return launch_n2<2>(t, state_in, state_out, control, k, n_steps, world_status,
                        accepted_steps, stream, mix);
  if (t->t.nch == 0)
    return launch_n2<0>(t, state_in, state_out, control, k, n_steps, world_status,
                        accepted_steps, stream, mix);
  return fail(CB_ERR_UNSUPPORTED, "channel slots must be 0 or 2");
}

int n2_build_plan(cb_tissue *t) { return build_plan(t); }

}  // namespace cbk

extern "C" {

int cb_set_sparse_launch(cb_tissue *t, int block) {
  if (!t) return fail(CB_ERR_ARGUMENT, "null argument");
  if (block != 0 && block != 128 && block != 256)
    return fail(CB_ERR_ARGUMENT, "the sparse kernels' block is 128 or 256 (0: the plan's choice)");
  cudaError_t ce = cudaSetDevice(t->device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
  const int rc = build_plan(t);
  if (rc) return rc;
  N2Plan *p = t->n2;
  p->ros2_block = block ? block : (p->smem_bytes == 0 ? 128 : 256);
  p->ros2_block_f32 = block ? block : (p->smem_f32 == 0 ? 128 : 256);
  return CB_OK;
}

int cb_get_sparse_launch(cb_tissue *t, int *block) {
  if (!t || !block) return fail(CB_ERR_ARGUMENT, "null argument");
  cudaError_t ce = cudaSetDevice(t->device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
  const int rc = build_plan(t);
  if (rc) return rc;
  *block = t->n2->ros2_block;
  return CB_OK;
}

}  // extern "C"

namespace cbk {

void n2_release(cb_tissue *t) {
  if (!t->n2) return;
  for (void *ptr : t->n2->owned) cudaFree(ptr);
  delete t->n2;
  t->n2 = nullptr;
}

}  // namespace cbk
