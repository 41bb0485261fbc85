// ros2_adjoint.cu - the reverse-mode derivative of the ROS2 step (CB_METHOD_ROS2):
// cb_step_vjp_method(..., CB_METHOD_ROS2, ...).
//
// The step (n2_step.cu, ros2_kernel; Verwer, Spee, Blom and Hundsdorfer's ROS2, gamma = 1 +
// 1/sqrt(2)): W k1 = F(y), y1 = y + h k1, W k2 = F(y1) - 2 k1, y' = y + 3/2 h k1 + 1/2 h k2,
// W = I - gamma h J(y). On the dynamic rows (amounts n[3][C], junction gates g[E], channel gates
// gc[2][NCH][C]; the ledgers never feed back) W k = r is, per world,
//
//   M u = K sum_s z_s r_n,s,     M = C + gamma h (diag(G_patch) + L(G_junction)), bath held,
//   k_n = r_n + gamma h route_rates(W_m u, W_c u, W_j du),
//   k_g = r_g / (1 + gamma h lambda),  k_gc = (r_gc + gamma h cpl u) / (1 + gamma h dec),
//
// W_* the routes' slope conductances at y, G their charge sums, lambda the junction gate law's
// relaxation rate, dec = 1/tau and cpl = d/dV of (target - g)/tau of a channel gate row.
//
// cb_step_vjp_method first runs the n_steps steps forward, one step per launch, through the ROS2
// kernel with its record (R2Tape) on: every step-start state, the step's factor of M with its
// Jacobi scale, both stage solves' voltage rates u1, u2, k1's dynamic rows and k2's gate rows.
// Then one launch, one CTA per world, walks the steps backwards. Per step:
//
//   kbar1 = 3/2 h ybar', kbar2 = 1/2 h ybar'
//   solve^T(kbar2) -> rbar2      the transposed stage solve REUSES THE STEP'S FACTOR: M is
//                                symmetric, so rho_bar = M^-1 ubar is one forward and back
//                                substitution through the recorded factor; M's dependence on y
//                                gives G_patch_bar = -gamma h rho_bar u and G_junction_bar =
//                                -gamma h (rho_bar_a - rho_bar_b) du
//   kbar1 -= 2 rbar2; ybar1 = F^T(y1) rbar2; ybar += ybar1; kbar1 += h ybar1
//   solve^T(kbar1) -> rbar1; ybar += F^T(y) rbar1
//   ybar += J^T(y) Jbar          the slopes', relaxation rates', decays' and couplings'
//                                dependence on y and the permeabilities: B''(x), the channel
//                                laws' target'' and tau'', d lambda/dV
//
// F^T is the explicit rates' transposed linearisation shared with the ARS(2,2,2) reverse
// (adjoint_terms.cuh) plus the channel gate rows (target - g)/tau. Junction terms are formed
// once per edge, stored per edge and gathered by each cell over its CSR adjacency in edge order:
// no atomics, results bit-identical run to run. A step the forward refused is the identity for
// its world and adds nothing. The reference has no reverse-mode adjoint (it differentiates its
// step forward only, analysis/stationary.py:505-514) and no Rosenbrock method on its tissue path;
// this is the derivative jax.grad would take of the composed ROS2 step.

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <string>

#include "adjoint_terms.cuh"
#include "handle.h"
#include "n2_common.cuh"

namespace {

using namespace cbk;

// B''(x) for B(x) = x / expm1(x); even in x. With a = |x|, om = -expm1(-a):
// (1 - om)(a (2 - om) - 2 om) / om^3; below a < 0.1 the series 1/6 - x^2/60 + x^4/1008 -
// x^6/21600 + x^8/532224 (from the Bernoulli numbers B_2 .. B_10).
__device__ __forceinline__ double bernoulli_curvature(double x) {
  const double a = fabs(x);
  if (a < 0.1) {
    const double x2 = x * x;
    return 1.0 / 6.0 +
           x2 * (-1.0 / 60.0 + x2 * (1.0 / 1008.0 + x2 * (-1.0 / 21600.0 + x2 / 532224.0)));
  }
  const double om = -expm1(-a);
  return (1.0 - om) * (a * (2.0 - om) - 2.0 * om) / ((om * om) * om);
}

// A gate row's target t and rate kappa = 1/tau with their first and second voltage derivatives
// (the channel laws of laws.cuh: NaV1.2 m^3 h, Kv1.5 m h, Hodgkin-Huxley n).
struct GateCurve {
  double t[2], dt[2], d2t[2], k[2], dk[2], d2k[2];
};

__device__ inline GateCurve gate_curve(int code, double v) {
  GateCurve g;
  if (code == kNav1p2) {
    const double sh = (v + 0.025) / 0.009;
    double bp, bm, sp, sm;
    bernoulli_pair<double>(sh, bp, bm);
    bernoulli_slope_pair(sh, sp, sm);
    const double c2 = bernoulli_curvature(sh);
    const double a = (0.182 * 9) * bm, da = -(0.182 * 9) * sm / 0.009,
                 d2a = (0.182 * 9) * c2 / (0.009 * 0.009);
    const double d = (0.124 * 9) * bp, dd = (0.124 * 9) * sp / 0.009,
                 d2d = (0.124 * 9) * c2 / (0.009 * 0.009);
    const double s = a + d, ds = da + dd, d2s = d2a + d2d;
    const double t = a / s;
    const double dt = (da - t * ds) / s;
    g.t[0] = t;
    g.dt[0] = dt;
    g.d2t[0] = (d2a - 2.0 * dt * ds - t * d2s) / s;
    g.k[0] = 1000.0 * s;
    g.dk[0] = 1000.0 * ds;
    g.d2k[0] = 1000.0 * d2s;
    const double th = 1.0 / (1.0 + exp((v + 0.055) / 0.0062));
    const double dth = -th * (1.0 - th) / 0.0062;
    g.t[1] = th;
    g.dt[1] = dth;
    g.d2t[1] = -dth * (1.0 - 2.0 * th) / 0.0062;
    const double ur = -(v + 0.040) / 0.005, ui = (v + 0.065000123) / 0.005;
    const double q = (0.024 * 5) * bernoulli<double>(ur) + (0.0091 * 5) * bernoulli<double>(ui);
    const double dq = -(0.024 * 5) * bernoulli_slope(ur) / 0.005 +
                      (0.0091 * 5) * bernoulli_slope(ui) / 0.005;
    const double d2q = (0.024 * 5) * bernoulli_curvature(ur) / (0.005 * 0.005) +
                       (0.0091 * 5) * bernoulli_curvature(ui) / (0.005 * 0.005);
    g.k[1] = 1000.0 * q;
    g.dk[1] = 1000.0 * dq;
    g.d2k[1] = 1000.0 * d2q;
  } else if (code == kHhKn4) {
    const double ua = -(1000.0 * v + 55.0) / 10.0;
    const double al = 100.0 * bernoulli<double>(ua);
    const double dal = -100.0 * 100.0 * bernoulli_slope(ua);
    const double d2al = 100.0 * (100.0 * 100.0) * bernoulli_curvature(ua);
    const double be = 125.0 * exp(-(1000.0 * v + 65.0) / 80.0);
    const double dbe = -12.5 * be, d2be = 156.25 * be;
    const double s = al + be, ds = dal + dbe, d2s = d2al + d2be;
    const double t = al / s;
    const double dt = (dal - t * ds) / s;
    g.t[0] = t;
    g.dt[0] = dt;
    g.d2t[0] = (d2al - 2.0 * dt * ds - t * d2s) / s;
    g.k[0] = s;
    g.dk[0] = ds;
    g.d2k[0] = d2s;
    g.t[1] = g.dt[1] = g.d2t[1] = g.k[1] = g.dk[1] = g.d2k[1] = 0.0;
  } else {  // Kv1.5
    const double s0 = sigmoid((v + 0.0060) / 0.0064);
    const double ds0 = s0 * (1.0 - s0) / 0.0064;
    const double s1 = sigmoid(-(v + 0.0253) / 0.0035);
    const double ds1 = -s1 * (1.0 - s1) / 0.0035;
    g.t[0] = s0;
    g.dt[0] = ds0;
    g.d2t[0] = ds0 * (1.0 - 2.0 * s0) / 0.0064;
    g.t[1] = s1;
    g.dt[1] = ds1;
    g.d2t[1] = -ds1 * (1.0 - 2.0 * s1) / 0.0035;
    const double tau[2] = {0.008330 - 0.1163 * v, 1.620000 - 15.500 * v};
    const double dtau[2] = {-0.1163, -15.5};
    for (int r = 0; r < 2; ++r) {
      g.k[r] = 1.0 / tau[r];
      g.dk[r] = -dtau[r] / (tau[r] * tau[r]);
      g.d2k[r] = 2.0 * dtau[r] * dtau[r] / ((tau[r] * tau[r]) * tau[r]);
    }
  }
  return g;
}

// Partials of route_slope W = p z' (-c_from B'(-x) - c_to B'(x)), x = z' dv (z' = z F/RT, p the
// prefactor in fmol/s per mM): dW/dc_from, dW/dc_to, dW/d dv (B'' is even) and W / p.
struct SlopeParts {
  double d_from, d_to, d_dv, w1;
};
__device__ __forceinline__ SlopeParts slope_parts(double p, double c_from, double c_to, double dv,
                                                  double zfrt) {
  const double x = zfrt * dv;
  const double bm = ref_bernoulli_slope(-x), bp = ref_bernoulli_slope(x);
  SlopeParts r;
  r.d_from = p * zfrt * (-bm);
  r.d_to = p * zfrt * (-bp);
  r.d_dv = p * (zfrt * zfrt) * bernoulli_curvature(x) * (c_from - c_to);
  r.w1 = zfrt * (-c_from * bm - c_to * bp);
  return r;
}

// Cell scratch ([field][C]); the channel fields [field][NCH][C] from AR_CH.
enum R2RevCell {
  AR_C0 = 0,     // 3: concentrations at y
  AR_V0 = 3,     // potential at y
  AR_C1 = 4,     // 3: concentrations at y1 = y + h k1
  AR_V1 = 7,     // potential at y1
  AR_WM = 8,     // 3: patch slopes at y
  AR_KB1N = 11,  // 3: kbar1 of the amounts
  AR_RBN = 14,   // 3: rbar of the amounts (the current solve's)
  AR_JWM = 17,   // 3: the patch slopes' cotangent
  AR_UB = 20,    // ubar, then rho_bar
  AR_YV = 21,    // substitution vectors (position-indexed)
  AR_XV = 22,
  AR_CH = 23
};
enum R2RevChan {  // per channel slot, each field [NCH][C]
  AH_W = 0,       // slope at y
  AH_DEC = 1,     // 2: 1/tau per gate row at y (0: no law)
  AH_CPL = 3,     // 2: d/dV of (target - g)/tau at y
  AH_GC1 = 5,     // 2: gates at y1
  AH_KB1 = 7,     // 2: kbar1 of the gates
  AH_RB = 9,      // 2: rbar of the gates (the current solve's)
  AH_JW = 11,     // the slope's cotangent
  AH_JDEC = 12,   // 2: cotangents of dec and cpl
  AH_JCPL = 14,   // 2
  AH_FIELDS = 16
};
__host__ __device__ constexpr int r2rev_cell_fields(int nch) { return AR_CH + AH_FIELDS * nch; }
enum R2RevEdge {
  AJ_W = 0,      // 3: slopes at y
  AJ_LAM = 3,    // relaxation rate at y
  AJ_JW = 4,     // 3: the slopes' cotangent
  AJ_JLAM = 7,   // the relaxation rate's cotangent
  AJ_UJ = 8,     // the junction's ubar contribution (sender +, receiver -)
  AJ_KB1 = 9,    // kbar1 of the gate
  AJ_RB = 10,    // rbar of the gate (the current solve's)
  AJ_DA = 11,    // 3: cotangent contributions to the sender's concentrations
  AJ_DB = 14,    // 3: to the receiver's
  AJ_DV = 17,    // to the potential difference
  AJ_FIELDS = 18
};

struct R2Rev {
  const double *tape;        // step t's record at tape + t stride
  long long stride;          // doubles per step
  long long o_factor, o_scale, o_u, o_k1n, o_k1gc, o_k1g, o_k2gc, o_k2g;
};

template <int BLOCK, int NCH, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB)
    ros2_vjp_kernel(const Tissue T, const Layout L, const N2Dev D, const Adj A, const R2Rev R,
                    const double *__restrict__ control, double h, int n_steps) {
  constexpr int NQ = NCH > 0 ? NCH : 1;
  __shared__ double sW[WC_STRIDE];
  const int w = blockIdx.x, tid = threadIdx.x;
  const int c0 = T.cell_offset[w], nc = T.cell_offset[w + 1] - c0;
  const int e0 = T.edge_offset[w], ne = T.edge_offset[w + 1] - e0;
  const long long C = T.C, E = T.E, W = T.W;
  if (tid < WC_STRIDE) sW[tid] = T.world[(size_t)w * WC_STRIDE + tid];
  double *cs = A.cs, *es = A.es, *cot = A.cot;
  const long long oN = L.s[CB_AMOUNT_INCREMENT], oG = L.s[CB_JUNCTION_GATE];
  const long long oH = L.s[CB_CHANNEL_GATE];
  const double K = kChargePerFmol;
  const double gh = (1.0 + 1.0 / sqrt(2.0)) * h;
  const double z3[3] = {1.0, 1.0, -1.0};
  // A ledger cotangent that is not zero: its dependence on the parameters is not differentiated.
  int ledger = 0;
  for (int i = tid; i < nc; i += BLOCK) {
    const long long gi = c0 + i;
    for (int s = 0; s < 3; ++s) ledger |= cot[L.s[CB_MEMBRANE_TRANSFERRED] + s * C + gi] != 0.0;
    ledger |= cot[L.s[CB_MEMBRANE_DISSIPATED] + gi] != 0.0;
    ledger |= cot[L.s[CB_PUMP_CYCLES] + gi] != 0.0;
    ledger |= cot[L.s[CB_PUMP_DISSIPATED] + gi] != 0.0;
    ledger |= cot[L.s[CB_METABOLIC_WORK] + gi] != 0.0;
    for (int q = 0; q < NCH; ++q) {
      ledger |= cot[L.s[CB_CHANNEL_TRANSFERRED] + q * C + gi] != 0.0;
      ledger |= cot[L.s[CB_CHANNEL_DISSIPATED] + q * C + gi] != 0.0;
    }
  }
  for (int e = tid; e < ne; e += BLOCK) {
    const long long ge = e0 + e;
    for (int s = 0; s < 3; ++s) ledger |= cot[L.s[CB_JUNCTION_TRANSFERRED] + s * E + ge] != 0.0;
    ledger |= cot[L.s[CB_JUNCTION_DISSIPATED] + ge] != 0.0;
  }
  if (tid == 0) {
    for (int s = 0; s < 3; ++s) ledger |= cot[L.s[CB_RESERVOIR_SUPPLIED] + s * W + w] != 0.0;
    ledger |= cot[L.s[CB_ELECTRODE_CHARGE] + w] != 0.0;
    ledger |= cot[L.s[CB_RESERVOIR_WORK] + w] != 0.0;
    ledger |= cot[L.s[CB_ELECTRODE_WORK] + w] != 0.0;
  }
  ledger = __syncthreads_or(ledger);
  const double Vb = sW[WC_VB], FRT = sW[WC_FRT];
  const double *mctl = control + L.c[CB_CONTROL_MEMBRANE];
  const double *pctlp = control + L.c[CB_CONTROL_PUMP];
  const double *jctl = control + L.c[CB_CONTROL_JUNCTION];
  const double *chctl0 = control + L.c[CB_CONTROL_CHANNEL];
  auto CF = [&](int f, long long gi) -> double & { return cs[(long long)f * C + gi]; };
  auto EF = [&](int f, long long ge) -> double & { return es[(long long)f * E + ge]; };
  auto CH = [&](int q, int f, long long gi) -> double & {
    return cs[(long long)(AR_CH + f * NQ + q) * C + gi];
  };
  const int wL = D.lb[w + 1] - D.lb[w];
  const int *colp = D.colp + c0 + w, *lrow = D.lrow + D.fb[w];
  const int *ukp = D.uk_ptr + c0 + w, *ukc = D.uk_col + D.ub[w];
  const int *ukpos = D.uk_pos + D.ub[w], *ukrel = D.uk_rel + D.ub[w];
  const int *rel = D.rel + D.rb[w];
  const int *lvp = D.lv_ptr + D.lb[w] + w, *lvc = D.lv_cols + c0;
  double *Yv = cs + (long long)AR_YV * C + c0;
  double *Xv = cs + (long long)AR_XV * C + c0;
  // Each cell's gather of a junction field over its adjacency (senders +, receivers -).
  auto gather_signed = [&](long long gi, int f) {
    double v = 0.0;
    for (int a = __ldg(T.adj_ptr + gi); a < __ldg(T.adj_ptr + gi + 1); ++a) {
      const int code = __ldg(T.adj_idx + a);
      const long long ge = e0 + (code >> 1);
      if (code & 1) v -= EF(f, ge);
      else v += EF(f, ge);
    }
    return v;
  };
  // The junctions' F^T contributions to a cell: concentrations lc[3], potential lv.
  auto gather_terms = [&](long long gi, double (&lc)[3], double &lv) {
    for (int a = __ldg(T.adj_ptr + gi); a < __ldg(T.adj_ptr + gi + 1); ++a) {
      const int code = __ldg(T.adj_idx + a);
      const long long ge = e0 + (code >> 1);
      if (code & 1) {
        for (int s = 0; s < 3; ++s) lc[s] += EF(AJ_DB + s, ge);
        lv -= EF(AJ_DV, ge);
      } else {
        for (int s = 0; s < 3; ++s) lc[s] += EF(AJ_DA + s, ge);
        lv += EF(AJ_DV, ge);
      }
    }
  };

  for (int t = n_steps - 1; t >= 0; --t) {
    if (A.taken[(size_t)t * W + w] == 0) continue;  // refused: the identity, uniform per CTA
    const double *St = t == 0 ? A.state_in : A.states + (size_t)(t - 1) * A.state_total;
    const double *tp = R.tape + (size_t)t * R.stride;
    const double *tS = tp + R.o_scale, *tU1 = tp + R.o_u, *tU2 = tp + R.o_u + C;
    const double *tK1n = tp + R.o_k1n, *tK1gc = tp + R.o_k1gc, *tK1g = tp + R.o_k1g;
    const double *tK2gc = tp + R.o_k2gc, *tK2g = tp + R.o_k2g;
    const WorldCholesky<double, BLOCK> chol{colp, lrow, ukp, ukc, ukpos, ukrel, rel, lvp, lvc,
                                            const_cast<double *>(tp + R.o_factor + D.fb[w]),
                                            Yv, Xv, 0, wL, nc, 0};

    // A (cells): y and y1; the W-matrix's cell pieces at y; the cotangent accumulators zeroed.
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      const double ivol = __ldg(T.ivol + gi);
      double n[3], n1[3], c[3];
      for (int s = 0; s < 3; ++s) {
        n[s] = St[oN + s * C + gi];
        n1[s] = n[s] + h * tK1n[s * C + gi];
        c[s] = (__ldg(T.ref + s * C + gi) + n[s]) * ivol;
        CF(AR_C0 + s, gi) = c[s];
        CF(AR_C1 + s, gi) = (__ldg(T.ref + s * C + gi) + n1[s]) * ivol;
      }
      const double V0 = cell_potential(T, gi, Vb, n);
      CF(AR_V0, gi) = V0;
      CF(AR_V1, gi) = cell_potential(T, gi, Vb, n1);
      const double dv = V0 - Vb, mc = mctl[gi];
      for (int s = 0; s < 3; ++s) {
        CF(AR_WM + s, gi) = route_slope(__ldg(T.ap + s * C + gi) * mc, c[s], sW[WC_CO + s], dv,
                                        z3[s] * FRT);
        CF(AR_JWM + s, gi) = 0.0;
      }
      for (int q = 0; q < NCH; ++q) {
        const int code = __ldg(T.ch_code + q * C + gi);
        const int sp = __ldg(T.ch_species + q * C + gi);
        const double g0[2] = {St[oH + q * C + gi], St[oH + (NCH + q) * C + gi]};
        const double avail = (__ldg(T.ch_ab + q * C + gi) * channel_opening(code, g0[0], g0[1])) *
                             __ldg(chctl0 + q * C + gi);
        CH(q, AH_W, gi) = route_slope(__ldg(T.ch_ap + q * C + gi) * avail, c[sp], sW[WC_CO + sp],
                                      dv, z3[sp] * FRT);
        CH(q, AH_JW, gi) = 0.0;
        const GateCurve gk = gate_curve(code, dv);
        for (int r = 0; r < 2; ++r) {
          const bool live = !(r == 1 && code == kHhKn4);
          const double cpl = gk.dt[r] * gk.k[r] + (gk.t[r] - g0[r]) * gk.dk[r];
          CH(q, AH_DEC + r, gi) = live && is_finite(gk.k[r]) ? gk.k[r] : 0.0;
          CH(q, AH_CPL + r, gi) = live && is_finite(cpl) ? cpl : 0.0;
          CH(q, AH_GC1 + r, gi) = g0[r] + h * tK1gc[(r * NCH + q) * C + gi];
          CH(q, AH_JDEC + r, gi) = 0.0;
          CH(q, AH_JCPL + r, gi) = 0.0;
        }
      }
    }
    __syncthreads();
    // B (junctions): slopes and relaxation rate at y.
    for (int e = tid; e < ne; e += BLOCK) {
      const long long ge = e0 + e;
      const long long ga = c0 + __ldg(T.snd + ge), gb = c0 + __ldg(T.rcv + ge);
      const double dv = CF(AR_V0, ga) - CF(AR_V0, gb);
      const double p = jctl[ge] * St[oG + ge];
      for (int s = 0; s < 3; ++s) {
        EF(AJ_W + s, ge) = route_slope(__ldg(T.jap + s * E + ge) * p, CF(AR_C0 + s, ga),
                                       CF(AR_C0 + s, gb), dv, z3[s] * FRT);
        EF(AJ_JW + s, ge) = 0.0;
      }
      // The gate law's relaxation rate alpha + beta (its own form, pinned gates included).
      const double shift = fabs(dv) - __ldg(T.thr + ge);
      const double relax = 1.3 * exp(-77.0 * shift) + 20.0 * sigmoid(kLog0065 + 140.0 * shift);
      EF(AJ_LAM, ge) = is_finite(relax) ? relax : 0.0;
      EF(AJ_JLAM, ge) = 0.0;
    }
    __syncthreads();
    // C (cells): kbar2 = 1/2 h ybar', kbar1 = 3/2 h ybar'; solve^T(kbar2), the cells' part.
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      const double u2 = tU2[gi];
      double kb2[3], ub = 0.0;
      for (int s = 0; s < 3; ++s) {
        const double yb = cot[oN + s * C + gi];
        kb2[s] = (0.5 * h) * yb;
        CF(AR_KB1N + s, gi) = (1.5 * h) * yb;
        const double phi = -gh * kb2[s];
        CF(AR_JWM + s, gi) += phi * u2;
        ub += phi * CF(AR_WM + s, gi);
      }
      for (int q = 0; q < NCH; ++q) {
        const int sp = __ldg(T.ch_species + q * C + gi);
        const double phi = -gh * kb2[sp];
        CH(q, AH_JW, gi) += phi * u2;
        ub += phi * CH(q, AH_W, gi);
        for (int r = 0; r < 2; ++r) {
          const double yb = cot[oH + (r * NCH + q) * C + gi];
          const double k2 = (0.5 * h) * yb;
          const double den = 1.0 + gh * CH(q, AH_DEC + r, gi);
          const double rb = k2 / den;
          CH(q, AH_RB + r, gi) = rb;
          CH(q, AH_JCPL + r, gi) += gh * u2 * rb;
          CH(q, AH_JDEC + r, gi) += -gh * k2 * tK2gc[(r * NCH + q) * C + gi] / den;
          ub += gh * CH(q, AH_CPL + r, gi) * rb;
          CH(q, AH_KB1 + r, gi) = (1.5 * h) * yb;
        }
      }
      CF(AR_UB, gi) = ub;
    }
    // D (junctions): solve^T(kbar2), the junctions' part (reads ybar' of the end cells).
    for (int e = tid; e < ne; e += BLOCK) {
      const long long ge = e0 + e;
      const long long ga = c0 + __ldg(T.snd + ge), gb = c0 + __ldg(T.rcv + ge);
      const double du = tU2[ga] - tU2[gb];
      const double yb = cot[oG + ge];
      const double k2 = (0.5 * h) * yb;
      const double den = 1.0 + gh * EF(AJ_LAM, ge);
      const double rb = k2 / den;
      EF(AJ_RB, ge) = rb;
      EF(AJ_JLAM, ge) += -gh * k2 * tK2g[ge] / den;
      EF(AJ_KB1, ge) = (1.5 * h) * yb - 2.0 * rb;
      double uj = 0.0;
      for (int s = 0; s < 3; ++s) {
        const double phi =
            gh * ((0.5 * h) * cot[oN + s * C + gb] - (0.5 * h) * cot[oN + s * C + ga]);
        EF(AJ_JW + s, ge) += phi * du;
        uj += phi * EF(AJ_W + s, ge);
      }
      EF(AJ_UJ, ge) = uj;
    }
    __syncthreads();
    // E (cells): ubar complete; the right-hand side of rho_bar = M^-1 ubar.
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      Yv[__ldg(D.rank + gi)] = (CF(AR_UB, gi) + gather_signed(gi, AJ_UJ)) * tS[gi];
    }
    __syncthreads();
    chol.solve();
    // G (cells): rho_bar, rbar2 of the amounts, G_patch_bar; kbar1 -= 2 rbar2.
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      const double rho = Xv[__ldg(D.rank + gi)] * tS[gi];
      CF(AR_UB, gi) = rho;
      const double gp = -gh * rho * tU2[gi];
      for (int s = 0; s < 3; ++s) {
        const double rbn = (0.5 * h) * cot[oN + s * C + gi] + K * z3[s] * rho;
        CF(AR_RBN + s, gi) = rbn;
        CF(AR_KB1N + s, gi) -= 2.0 * rbn;
        CF(AR_JWM + s, gi) += K * z3[s] * gp;
      }
      for (int q = 0; q < NCH; ++q) {
        const int sp = __ldg(T.ch_species + q * C + gi);
        CH(q, AH_JW, gi) += K * z3[sp] * gp;
        for (int r = 0; r < 2; ++r) CH(q, AH_KB1 + r, gi) -= 2.0 * CH(q, AH_RB + r, gi);
      }
    }
    __syncthreads();
    // H (junctions): G_junction_bar of solve 2; F^T at y1, the junctions' part.
    for (int e = tid; e < ne; e += BLOCK) {
      const long long ge = e0 + e;
      const long long ga = c0 + __ldg(T.snd + ge), gb = c0 + __ldg(T.rcv + ge);
      const double gj = -gh * (CF(AR_UB, ga) - CF(AR_UB, gb)) * (tU2[ga] - tU2[gb]);
      double ca[3], cb[3], ma[3], mb[3], da[3], db[3], ddv;
      for (int s = 0; s < 3; ++s) {
        EF(AJ_JW + s, ge) += K * z3[s] * gj;
        ca[s] = CF(AR_C1 + s, ga);
        cb[s] = CF(AR_C1 + s, gb);
        ma[s] = CF(AR_RBN + s, ga);
        mb[s] = CF(AR_RBN + s, gb);
      }
      const double g1 = St[oG + ge] + h * tK1g[ge];
      const double lg = edge_vjp(T, A, sW, ge, ca, cb, CF(AR_V1, ga) - CF(AR_V1, gb), g1,
                                 jctl[ge], ma, mb, EF(AJ_RB, ge), da, db, ddv);
      for (int s = 0; s < 3; ++s) {
        EF(AJ_DA + s, ge) = da[s];
        EF(AJ_DB + s, ge) = db[s];
      }
      EF(AJ_DV, ge) = ddv;
      cot[oG + ge] += lg;
      EF(AJ_KB1, ge) += h * lg;
    }
    __syncthreads();
    // I (cells): F^T at y1, the cells' part (with the junctions' gathered), into ybar and kbar1;
    // then solve^T(kbar1), the cells' part.
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      const double mc = mctl[gi], pctl = pctlp[gi];
      const double ldc = pctl > 0.0 ? __ldg(T.logpcap + gi) + log(pctl) : 0.0;
      const double ivol = __ldg(T.ivol + gi), icap = __ldg(T.icap + gi);
      double c[3], mu[3], lc[3] = {0.0, 0.0, 0.0}, lv = 0.0, lgc[2][NQ] = {}, own[3];
      for (int s = 0; s < 3; ++s) {
        c[s] = CF(AR_C1 + s, gi);
        mu[s] = CF(AR_RBN + s, gi);
      }
      gather_terms(gi, lc, lv);
      const double V1 = CF(AR_V1, gi);
      const double *gc1 = cs + (long long)(AR_CH + AH_GC1 * NQ) * C + gi;
      cell_terms<NCH, false, true>(T, A, sW, gi, c, V1, gc1, NQ * C, mc, pctl, ldc, chctl0 + gi,
                                   mu, lc, lv, lgc, own);
      for (int q = 0; q < NCH; ++q) {
        const int code = __ldg(T.ch_code + q * C + gi);
        const GateCurve gk = gate_curve(code, V1 - Vb);
        for (int r = 0; r < 2; ++r) {
          if (r == 1 && code == kHhKn4) continue;
          const double rb = CH(q, AH_RB + r, gi);
          lgc[r][q] += -gk.k[r] * rb;
          lv += (gk.dt[r] * gk.k[r] + (gk.t[r] - CH(q, AH_GC1 + r, gi)) * gk.dk[r]) * rb;
        }
      }
      const double u1 = tU1[gi];
      double ub = 0.0;
      for (int s = 0; s < 3; ++s) {
        const double y1 = lc[s] * ivol + lv * (K * z3[s]) * icap;
        cot[oN + s * C + gi] += y1;
        const double kb = CF(AR_KB1N + s, gi) + h * y1;
        CF(AR_KB1N + s, gi) = kb;
        const double phi = -gh * kb;
        CF(AR_JWM + s, gi) += phi * u1;
        ub += phi * CF(AR_WM + s, gi);
      }
      for (int q = 0; q < NCH; ++q) {
        const int sp = __ldg(T.ch_species + q * C + gi);
        const double phi = -gh * CF(AR_KB1N + sp, gi);
        CH(q, AH_JW, gi) += phi * u1;
        ub += phi * CH(q, AH_W, gi);
        for (int r = 0; r < 2; ++r) {
          cot[oH + (r * NCH + q) * C + gi] += lgc[r][q];
          const double kb = CH(q, AH_KB1 + r, gi) + h * lgc[r][q];
          const double den = 1.0 + gh * CH(q, AH_DEC + r, gi);
          const double rb = kb / den;
          CH(q, AH_RB + r, gi) = rb;
          CH(q, AH_JCPL + r, gi) += gh * u1 * rb;
          CH(q, AH_JDEC + r, gi) += -gh * kb * tK1gc[(r * NCH + q) * C + gi] / den;
          ub += gh * CH(q, AH_CPL + r, gi) * rb;
        }
      }
      CF(AR_UB, gi) = ub;
    }
    __syncthreads();
    // J (junctions): solve^T(kbar1), the junctions' part.
    for (int e = tid; e < ne; e += BLOCK) {
      const long long ge = e0 + e;
      const long long ga = c0 + __ldg(T.snd + ge), gb = c0 + __ldg(T.rcv + ge);
      const double kb = EF(AJ_KB1, ge);
      const double den = 1.0 + gh * EF(AJ_LAM, ge);
      const double rb = kb / den;
      EF(AJ_RB, ge) = rb;
      EF(AJ_JLAM, ge) += -gh * kb * tK1g[ge] / den;
      const double du = tU1[ga] - tU1[gb];
      double uj = 0.0;
      for (int s = 0; s < 3; ++s) {
        const double phi = gh * (CF(AR_KB1N + s, gb) - CF(AR_KB1N + s, ga));
        EF(AJ_JW + s, ge) += phi * du;
        uj += phi * EF(AJ_W + s, ge);
      }
      EF(AJ_UJ, ge) = uj;
    }
    __syncthreads();
    // K (cells): the right-hand side of solve 1's rho_bar.
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      Yv[__ldg(D.rank + gi)] = (CF(AR_UB, gi) + gather_signed(gi, AJ_UJ)) * tS[gi];
    }
    __syncthreads();
    chol.solve();
    // L (cells): rho_bar, rbar1 of the amounts, G_patch_bar.
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      const double rho = Xv[__ldg(D.rank + gi)] * tS[gi];
      CF(AR_UB, gi) = rho;
      const double gp = -gh * rho * tU1[gi];
      for (int s = 0; s < 3; ++s) {
        CF(AR_RBN + s, gi) = CF(AR_KB1N + s, gi) + K * z3[s] * rho;
        CF(AR_JWM + s, gi) += K * z3[s] * gp;
      }
      for (int q = 0; q < NCH; ++q) {
        const int sp = __ldg(T.ch_species + q * C + gi);
        CH(q, AH_JW, gi) += K * z3[sp] * gp;
      }
    }
    __syncthreads();
    // M (junctions): G_junction_bar of solve 1; F^T at y and J^T(y), the junctions' parts.
    for (int e = tid; e < ne; e += BLOCK) {
      const long long ge = e0 + e;
      const long long ga = c0 + __ldg(T.snd + ge), gb = c0 + __ldg(T.rcv + ge);
      const double gj = -gh * (CF(AR_UB, ga) - CF(AR_UB, gb)) * (tU1[ga] - tU1[gb]);
      double ca[3], cb[3], ma[3], mb[3], da[3], db[3], ddv;
      for (int s = 0; s < 3; ++s) {
        EF(AJ_JW + s, ge) += K * z3[s] * gj;
        ca[s] = CF(AR_C0 + s, ga);
        cb[s] = CF(AR_C0 + s, gb);
        ma[s] = CF(AR_RBN + s, ga);
        mb[s] = CF(AR_RBN + s, gb);
      }
      const double dv = CF(AR_V0, ga) - CF(AR_V0, gb);
      const double g0 = St[oG + ge], jc = jctl[ge];
      double lg = edge_vjp(T, A, sW, ge, ca, cb, dv, g0, jc, ma, mb, EF(AJ_RB, ge), da, db, ddv);
      // J^T(y): the slopes (through both ends' concentrations, the potential difference, the
      // gate and the permeabilities) and the relaxation rate (through the potential difference).
      const double jarea_f = __ldg(A.jarea + ge) / 1e-15;
      for (int s = 0; s < 3; ++s) {
        const double jap = __ldg(T.jap + s * E + ge);
        const SlopeParts sp = slope_parts(jap * (jc * g0), ca[s], cb[s], dv, z3[s] * FRT);
        const double jb = EF(AJ_JW + s, ge);
        da[s] += jb * sp.d_from;
        db[s] += jb * sp.d_to;
        ddv += jb * sp.d_dv;
        A.gj[s * E + ge] += jb * sp.w1 * (jarea_f * (jc * g0));
        lg += jb * sp.w1 * (jap * jc);
      }
      const double shift = fabs(dv) - __ldg(T.thr + ge);
      const double alpha = 1.3 * exp(-77.0 * shift);
      const double sb = sigmoid(kLog0065 + 140.0 * shift);
      const double sgn = dv > 0.0 ? 1.0 : dv < 0.0 ? -1.0 : 0.0;
      if (EF(AJ_LAM, ge) != 0.0)
        ddv += EF(AJ_JLAM, ge) * sgn * (-77.0 * alpha + (20.0 * 140.0) * sb * (1.0 - sb));
      for (int s = 0; s < 3; ++s) {
        EF(AJ_DA + s, ge) = da[s];
        EF(AJ_DB + s, ge) = db[s];
      }
      EF(AJ_DV, ge) = ddv;
      cot[oG + ge] += lg;
    }
    __syncthreads();
    // N (cells): F^T at y and J^T(y), the cells' parts, into ybar.
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      const double mc = mctl[gi], pctl = pctlp[gi];
      const double ldc = pctl > 0.0 ? __ldg(T.logpcap + gi) + log(pctl) : 0.0;
      const double ivol = __ldg(T.ivol + gi), icap = __ldg(T.icap + gi);
      const double area_f = __ldg(A.area + gi) / 1e-15;
      double c[3], mu[3], lc[3] = {0.0, 0.0, 0.0}, lv = 0.0, lgc[2][NQ] = {}, own[3];
      for (int s = 0; s < 3; ++s) {
        c[s] = CF(AR_C0 + s, gi);
        mu[s] = CF(AR_RBN + s, gi);
      }
      gather_terms(gi, lc, lv);
      const double V0 = CF(AR_V0, gi), dv = V0 - Vb;
      cell_terms<NCH, false, true>(T, A, sW, gi, c, V0, St + oH + gi, NCH * C, mc, pctl, ldc,
                                   chctl0 + gi, mu, lc, lv, lgc, own);
      for (int s = 0; s < 3; ++s) {
        const double ap = __ldg(T.ap + s * C + gi);
        const SlopeParts sp = slope_parts(ap * mc, c[s], sW[WC_CO + s], dv, z3[s] * FRT);
        const double jb = CF(AR_JWM + s, gi);
        lc[s] += jb * sp.d_from;
        lv += jb * sp.d_dv;
        A.gm[s * C + gi] += jb * sp.w1 * (area_f * mc);
      }
      for (int q = 0; q < NCH; ++q) {
        const int code = __ldg(T.ch_code + q * C + gi);
        const int sp_ = __ldg(T.ch_species + q * C + gi);
        const double g0[2] = {St[oH + q * C + gi], St[oH + (NCH + q) * C + gi]};
        const double ab = __ldg(T.ch_ab + q * C + gi), ctl = __ldg(chctl0 + q * C + gi);
        const double chap = __ldg(T.ch_ap + q * C + gi);
        const double open = channel_opening(code, g0[0], g0[1]);
        const double avail = (ab * open) * ctl;
        const SlopeParts sp = slope_parts(chap * avail, c[sp_], sW[WC_CO + sp_], dv, z3[sp_] * FRT);
        const double jb = CH(q, AH_JW, gi);
        lc[sp_] += jb * sp.d_from;
        lv += jb * sp.d_dv;
        A.gch[q * C + gi] += jb * sp.w1 * (area_f * avail);
        double dm, dh;
        opening_partials(code, g0[0], g0[1], dm, dh);
        const double dopen = jb * sp.w1 * ((chap * ab) * ctl);
        lgc[0][q] += dopen * dm;
        lgc[1][q] += dopen * dh;
        const GateCurve gk = gate_curve(code, dv);
        for (int r = 0; r < 2; ++r) {
          if (r == 1 && code == kHhKn4) continue;
          // F's gate row (target - g) kappa, with the step's rbar1.
          const double rb = CH(q, AH_RB + r, gi);
          lgc[r][q] += -gk.k[r] * rb;
          lv += (gk.dt[r] * gk.k[r] + (gk.t[r] - g0[r]) * gk.dk[r]) * rb;
          // J^T(y): dec = kappa, cpl = t' kappa + (t - g) kappa'.
          if (CH(q, AH_DEC + r, gi) != 0.0) {
            const double jd = CH(q, AH_JDEC + r, gi), jc_ = CH(q, AH_JCPL + r, gi);
            lv += jd * gk.dk[r] + jc_ * ((gk.d2t[r] * gk.k[r] + 2.0 * gk.dt[r] * gk.dk[r]) +
                                         (gk.t[r] - g0[r]) * gk.d2k[r]);
            lgc[r][q] += -jc_ * gk.dk[r];
          }
        }
      }
      for (int s = 0; s < 3; ++s) cot[oN + s * C + gi] += lc[s] * ivol + lv * (K * z3[s]) * icap;
      for (int q = 0; q < NCH; ++q)
        for (int r = 0; r < 2; ++r) cot[oH + (r * NCH + q) * C + gi] += lgc[r][q];
    }
    __syncthreads();
  }
  if (tid == 0) {
    uint32_t bits = ledger ? CB_WORLD_LEDGER_COTANGENT : 0u;
    for (int t = 0; t < n_steps; ++t) bits |= A.fwd_status[(size_t)t * W + w];
    A.status[w] = bits;
  }
}

size_t align256(size_t n) { return (n + 255) / 256 * 256; }
long long pad32(long long n) { return (n + 31) / 32 * 32; }

// The workspace: every step's end state, accepted flags and status, every step's record, the
// reverse's scratch. Offsets in bytes; the record's parts in doubles within one step's record.
struct R2Workspace {
  size_t states, taken, status, tape, cells, edges, total;
  R2Rev rev;
};

R2Workspace plan_workspace(const cb_tissue *t, int n_steps) {
  R2Workspace p{};
  const long long C = t->C, E = std::max(t->E, 1), nch = t->t.nch;
  long long o = 0;
  p.rev.o_factor = o;
  o += pad32(t->n2->factor_entries);
  p.rev.o_scale = o;
  o += pad32(C);
  p.rev.o_u = o;
  o += pad32(2 * C);
  p.rev.o_k1n = o;
  o += pad32(3 * C);
  p.rev.o_k1gc = o;
  o += pad32(2 * nch * C);
  p.rev.o_k1g = o;
  o += pad32(E);
  p.rev.o_k2gc = o;
  o += pad32(2 * nch * C);
  p.rev.o_k2g = o;
  o += pad32(E);
  p.rev.stride = o;
  p.states = 0;
  p.taken = align256(sizeof(double) * (size_t)t->state_total * (size_t)n_steps);
  p.status = p.taken + align256(sizeof(int32_t) * (size_t)t->W * (size_t)n_steps);
  p.tape = p.status + align256(sizeof(uint32_t) * (size_t)t->W * (size_t)n_steps);
  p.cells = p.tape + align256(sizeof(double) * (size_t)o * (size_t)n_steps);
  p.edges = p.cells + align256(sizeof(double) * (size_t)r2rev_cell_fields((int)nch) * C);
  p.total = p.edges + align256(sizeof(double) * (size_t)AJ_FIELDS * E);
  return p;
}

template <int NCH>
int launch_ros2_vjp(cb_tissue *t, const Adj &A, const R2Rev &R, const double *control, double h,
                    int n_steps, cudaStream_t stream) {
  if (t->n2->block == 128)  // CELLS_B200_N2_BLOCK=128: four 128-thread CTAs per SM
    ros2_vjp_kernel<128, NCH, 4><<<t->W, 128, 0, stream>>>(t->t, t->layout, t->n2->d, A, R,
                                                           control, h, n_steps);
  else
    ros2_vjp_kernel<256, NCH, 2><<<t->W, 256, 0, stream>>>(t->t, t->layout, t->n2->d, A, R,
                                                           control, h, n_steps);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "ros2 vjp launch");
  return CB_OK;
}

int ros2_workspace(cb_tissue *t, int n_steps, size_t *bytes) {
  if (!t || !bytes) return fail(CB_ERR_ARGUMENT, "null argument");
  if (n_steps < 0) return fail(CB_ERR_ARGUMENT, "n_steps must be non-negative");
  cudaError_t ce = cudaSetDevice(t->device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
  const int rc = n2_build_plan(t);
  if (rc) return rc;
  *bytes = plan_workspace(t, n_steps).total;
  return CB_OK;
}

int ros2_vjp(cb_tissue *t, const double *state_in, double dt, const double *control, int n_steps,
             const double *cot_out, double *cot_in, double *grad_membrane, double *grad_junction,
             double *grad_channel, void *workspace, size_t workspace_bytes,
             uint32_t *world_status, void *stream) {
  if (!t || !state_in || !control || !cot_out || !cot_in || !grad_membrane || !world_status ||
      (t->E && !grad_junction) || (t->t.nch && !grad_channel) || !workspace)
    return fail(CB_ERR_ARGUMENT, "null argument");
  if (t->t.blk_modes > 0)
    return fail(CB_ERR_UNSUPPORTED, "the adjoint step has no open-channel block");
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(CB_ERR_ARGUMENT, "dt must be positive");
  if (n_steps < 0) return fail(CB_ERR_ARGUMENT, "n_steps must be non-negative");
  if (t->t.nch != 0 && t->t.nch != 2)
    return fail(CB_ERR_UNSUPPORTED, "channel slots must be 0 or 2");
  cudaError_t ce = cudaSetDevice(t->device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
  int rc = n2_build_plan(t);
  if (rc) return rc;
  const R2Workspace p = plan_workspace(t, n_steps);
  if (workspace_bytes < p.total) return fail(CB_ERR_ARGUMENT, "workspace too small");
  if (reinterpret_cast<uintptr_t>(workspace) % 256)
    return fail(CB_ERR_ARGUMENT, "workspace must be 256-byte aligned");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  char *ws = static_cast<char *>(workspace);
  double *states = reinterpret_cast<double *>(ws + p.states);
  int32_t *taken = reinterpret_cast<int32_t *>(ws + p.taken);
  uint32_t *status = reinterpret_cast<uint32_t *>(ws + p.status);
  double *tape = reinterpret_cast<double *>(ws + p.tape);
  // The forward, one recorded step per launch, every state kept.
  for (int step = 0; step < n_steps; ++step) {
    const double *in = step == 0 ? state_in : states + (size_t)(step - 1) * t->state_total;
    double *rec = tape + (size_t)step * p.rev.stride;
    const R2Tape tp{rec + p.rev.o_factor, rec + p.rev.o_scale, rec + p.rev.o_u,
                    rec + p.rev.o_k1n,    rec + p.rev.o_k1gc,  rec + p.rev.o_k1g,
                    rec + p.rev.o_k2gc,   rec + p.rev.o_k2g};
    rc = ros2_step_tape(t, in, states + (size_t)step * t->state_total, dt, control, 1,
                        status + (size_t)step * t->W, taken + (size_t)step * t->W, s, false,
                        false, tp);
    if (rc) return rc;
  }
  if (cot_in != cot_out) {
    ce = cudaMemcpyAsync(cot_in, cot_out, sizeof(double) * t->state_total,
                         cudaMemcpyDeviceToDevice, s);
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaMemcpyAsync");
  }
  Adj A{};
  A.state_in = state_in;
  A.states = states;
  A.state_total = t->state_total;
  A.taken = taken;
  A.fwd_status = status;
  A.cot = cot_in;
  A.gm = grad_membrane;
  A.gj = grad_junction;
  A.gch = grad_channel;
  A.cs = reinterpret_cast<double *>(ws + p.cells);
  A.es = reinterpret_cast<double *>(ws + p.edges);
  A.area = t->area;
  A.jarea = t->jarea;
  A.status = world_status;
  R2Rev R = p.rev;
  R.tape = tape;
  if (t->t.nch == 2) return launch_ros2_vjp<2>(t, A, R, control, dt, n_steps, s);
  return launch_ros2_vjp<0>(t, A, R, control, dt, n_steps, s);
}

}  // namespace

extern "C" {

int cb_vjp_workspace_method(cb_tissue *t, int method, int n_steps, size_t *bytes) {
  if (method == CB_METHOD_ARS222) return cb_vjp_workspace(t, n_steps, bytes);
  if (method == CB_METHOD_ROS2) return ros2_workspace(t, n_steps, bytes);
  return fail(CB_ERR_UNSUPPORTED, "the reverse covers CB_METHOD_ARS222 and CB_METHOD_ROS2");
}

int cb_step_vjp_method(cb_tissue *t, int method, const double *state_in, double dt,
                       const double *control, int n_steps, const double *cot_out,
                       double *cot_in, double *grad_membrane, double *grad_junction,
                       double *grad_channel, void *workspace, size_t workspace_bytes,
                       uint32_t *world_status, void *stream) {
  if (method == CB_METHOD_ARS222)
    return cb_step_vjp(t, state_in, dt, control, n_steps, cot_out, cot_in, grad_membrane,
                       grad_junction, grad_channel, workspace, workspace_bytes, world_status,
                       stream);
  if (method == CB_METHOD_ROS2)
    return ros2_vjp(t, state_in, dt, control, n_steps, cot_out, cot_in, grad_membrane,
                    grad_junction, grad_channel, workspace, workspace_bytes, world_status,
                    stream);
  return fail(CB_ERR_UNSUPPORTED, "the reverse covers CB_METHOD_ARS222 and CB_METHOD_ROS2");
}

}  // extern "C"
