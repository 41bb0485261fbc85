// adjoint_step.cu - the reverse-mode derivative of the FP64 ARS(2,2,2) tissue step
// (cb_step_vjp).
//
// The step's dynamic state is the amount increments n[3][C], the junction gates g[E] and the
// channel gates gc[2][NCH][C]; the ledgers never feed back into it. cb_step_vjp takes the
// cotangent of the state after n_steps steps and returns the cotangent of the state before them,
// adding each permeability's gradient. It first recomputes the n_steps steps through cb_step one
// step per launch, keeping every step-start state in the caller's workspace (so the forward it
// differentiates is the library's own step, refusals included), then runs one reverse launch:
// one CTA per world walks the steps backwards and, per step, rebuilds the stage values from the
// kept start state (stage-0 rates, the stage-1 amounts, gates and potentials) and applies the
// transposed linearisation of each stage in reverse order:
//
//   end gates  gc2 = adv(gc, kin(V0), kin(V2), dt)      -> cotangents of gc, V0, V2
//   end state  y2 = y + dt (delta k0 + (1 - delta) k1)   -> rate cotangents mu0, mu1
//   stage 1    k1 = f(n1, g1, gc1, V1)                   -> n1, g1, gc1, V1
//   stage-1 gates gc1 = adv(gc, kin(V0), kin(V1), gamma dt)
//   stage 1    y1 = y + gamma dt k0                      -> mu0 += gamma dt lambda1
//   stage 0    k0 = f(n, g, gc, V0)
//
// Each potential is the capacitor closure V = (Q0 + F sum z n) / C + V_bath: a diagonal map,
// its transposed solve the same diagonal. In f, each junction's terms are formed once per edge
// (its cotangent contributions to both end cells stored per edge) and each cell gathers them over
// its CSR adjacency in edge order: no atomics, results bit-identical run to run.
//
// Derivatives (restated from the laws' closed forms): B'(x) for B(x) = x / expm1(x) (the
// reference's bernoulli_slope, laws/routes/patch_electrodiffusion.py:43-54); the Na/K-ATPase
// cycles = -M expm1(a) on both branches of nak_atp_mass_action_positive.py:63-98; the junction
// gate law of junction_voltage_relaxation.py:43-67; the channel laws of kv1p5_mh.py:29-41 and
// nav1p2_m3h_regularized.py:22-44 and the Hodgkin-Huxley n law; the exponential gate update of
// numerics/exponential_gates.py:36-51.

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <string>

#include "adjoint_terms.cuh"
#include "handle.h"

namespace {

using namespace cbk;

// Scratch fields per cell ([field][C]): stage-0 and stage-1 concentrations and potentials, the
// amount-rate cotangents of both stages, the potential cotangent gathered for V0 from the gates,
// then the stage-1 channel gates [2][NCH].
enum AdjCell {
  AC_C0 = 0, AC_V0 = 3, AC_C1 = 4, AC_V1 = 7, AC_MU0 = 8, AC_MU1 = 11, AC_LV0 = 14, AC_GC1 = 15
};
__host__ __device__ constexpr int adj_cell_fields(int nch) { return AC_GC1 + 2 * nch; }
// Scratch fields per junction ([field][E]): stage-0 fluxes, the stage-1 gate, the cotangent
// contributions to the sender's and receiver's concentrations and to the potential difference,
// and the stage-0 gate-rate cotangent.
enum AdjEdge { AE_J = 0, AE_G1 = 3, AE_DA = 4, AE_DB = 7, AE_DV = 10, AE_MU0G = 11, AE_FIELDS = 12 };

// Partials of g + (ts - g)(1 - e^-z) + (te - ts) lag(z), z = h (1/taus + 1/taue) / 2,
// lag(z) = 1 - (1 - e^-z)/z: lag'(z) = -(em (1 + z) + z) / z^2 with em = expm1(-z), and its
// series 1/2 - z/3 + z^2/8 - z^3/30 below z < 1e-3 (where lag itself is a series).
struct GatePartials {
  double g, ts, taus, te, taue;
};
__device__ __forceinline__ GatePartials advance_partials(double g, double ts, double taus,
                                                         double te, double taue, double h) {
  const double z = 0.5 * h * (1.0 / taus + 1.0 / taue);
  const double em = expm1(-z);
  double lag, dlag;
  if (z < 1e-3) {
    lag = z * (0.5 - z * (1.0 / 6.0 - z * (1.0 / 24.0 - z / 120.0)));
    dlag = 0.5 - z * (1.0 / 3.0 - z * (1.0 / 8.0 - z / 30.0));
  } else {
    lag = (em + z) / z;
    dlag = -(em * (1.0 + z) + z) / (z * z);
  }
  const double dz = (ts - g) * (1.0 + em) + (te - ts) * dlag;
  GatePartials p;
  p.g = 1.0 + em;
  p.ts = -em - lag;
  p.taus = dz * (-0.5 * h / (taus * taus));
  p.te = lag;
  p.taue = dz * (-0.5 * h / (taue * taue));
  return p;
}

// A cell's gather of its junctions' contributions (senders first, then receivers, as the
// adjacency lists them): concentration cotangents and the potential cotangent.
__device__ __forceinline__ void gather_edges(const Tissue &T, const Adj &A, long long gi, int e0,
                                             double (&lc)[3], double &lv) {
  const long long E = T.E;
  const int a0 = __ldg(T.adj_ptr + gi), a1 = __ldg(T.adj_ptr + gi + 1);
  for (int a = a0; a < a1; ++a) {
    const int code = __ldg(T.adj_idx + a);
    const long long ge = e0 + (code >> 1);
    if (code & 1) {
#pragma unroll
      for (int s = 0; s < 3; ++s) lc[s] += A.es[(AE_DB + s) * E + ge];
      lv -= A.es[AE_DV * E + ge];
    } else {
#pragma unroll
      for (int s = 0; s < 3; ++s) lc[s] += A.es[(AE_DA + s) * E + ge];
      lv += A.es[AE_DV * E + ge];
    }
  }
}

template <int BLOCK, int NCH, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB)
    vjp_kernel(const Tissue T, const Layout L, const Adj A, const double *__restrict__ control,
               const StepCoef k, int n_steps) {
  constexpr int NQ = NCH > 0 ? NCH : 1;
  __shared__ double sW[WC_STRIDE];
  const int w = blockIdx.x, tid = threadIdx.x;
  const int c0 = T.cell_offset[w], nc = T.cell_offset[w + 1] - c0;
  const int e0 = T.edge_offset[w], ne = T.edge_offset[w + 1] - e0;
  const long long C = T.C, E = T.E, W = T.W;
  if (tid < WC_STRIDE) sW[tid] = T.world[(size_t)w * WC_STRIDE + tid];
  const double *cs = A.cs;
  double *cw = A.cs;
  double *es = A.es;
  double *cot = A.cot;
  const long long oN = L.s[CB_AMOUNT_INCREMENT], oG = L.s[CB_JUNCTION_GATE];
  const long long oH = L.s[CB_CHANNEL_GATE];
  const double K = kChargePerFmol;
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
  const double Vb = sW[WC_VB];
  const double *jctl = control + L.c[CB_CONTROL_JUNCTION];
  const double z3[3] = {1.0, 1.0, -1.0};

  for (int t = n_steps - 1; t >= 0; --t) {
    if (A.taken[(size_t)t * W + w] == 0) continue;  // refused: the identity, uniform per CTA
    const double *St = t == 0 ? A.state_in : A.states + (size_t)(t - 1) * A.state_total;
    const double *St1 = A.states + (size_t)t * A.state_total;

    // P1 (cells): stage-0 concentrations and potentials.
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      double n[3];
      const double ivol = __ldg(T.ivol + gi);
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        n[s] = St[oN + s * C + gi];
        cw[(AC_C0 + s) * C + gi] = (__ldg(T.ref + s * C + gi) + n[s]) * ivol;
      }
      cw[AC_V0 * C + gi] = cell_potential(T, gi, Vb, n);
    }
    __syncthreads();
    // P2 (junctions): stage-0 fluxes and the stage-1 gates.
    for (int e = tid; e < ne; e += BLOCK) {
      const long long ge = e0 + e;
      const long long ga = c0 + __ldg(T.snd + ge), gb = c0 + __ldg(T.rcv + ge);
      const double dv = cs[AC_V0 * C + ga] - cs[AC_V0 * C + gb];
      const double g = St[oG + ge];
      const double opening = __ldg(jctl + ge) * g;
      double bp, bm;
      bernoulli_pair<double>(dv * sW[WC_FRT], bp, bm);
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        const double ca = cs[(AC_C0 + s) * C + ga], cb = cs[(AC_C0 + s) * C + gb];
        const double gs = __ldg(T.jap + s * E + ge) * opening;
        es[(AE_J + s) * E + ge] = s < 2 ? gs * (ca * bm - cb * bp) : gs * (ca * bp - cb * bm);
      }
      const double thr = __ldg(T.thr + ge), mn = __ldg(T.jmin + ge);
      double gr = 0.0;
      if (mn < 1.0) {
        const double shift = fabs(dv) - thr;
        const double alpha = 1.3 * exp(-77.0 * shift);
        const double log_beta = kLog0065 + 140.0 * shift;
        const double beta = 20.0 * exp(-logaddexp0(-log_beta));
        gr = alpha * (1.0 - g) - beta * (g - mn);
      }
      es[AE_G1 * E + ge] = g + k.gamma_dt * gr;
    }
    __syncthreads();
    // P3 (cells): stage-0 amount rates, the stage-1 state; then the end state's cotangent
    // through the end gates and the end potential, split into the two stages' rate cotangents.
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      const double mc = control[L.c[CB_CONTROL_MEMBRANE] + gi];
      const double pctl = control[L.c[CB_CONTROL_PUMP] + gi];
      const double ldc = pctl > 0.0 ? __ldg(T.logpcap + gi) + log(pctl) : 0.0;
      const double *chctl = control + L.c[CB_CONTROL_CHANNEL] + gi;
      const double ivol = __ldg(T.ivol + gi), icap = __ldg(T.icap + gi);
      double c[3], n[3], n1[3], n2[3];
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        c[s] = cs[(AC_C0 + s) * C + gi];
        n[s] = St[oN + s * C + gi];
        n2[s] = St1[oN + s * C + gi];
      }
      const double V0 = cs[AC_V0 * C + gi];
      double own[3], lc_unused[3] = {0, 0, 0}, lv_unused = 0.0, lgc_unused[2][NQ] = {};
      const double mu0[3] = {0, 0, 0};
      cell_terms<NCH, true, false>(T, A, sW, gi, c, V0, St + oH + gi, NCH * C, mc, pctl, ldc,
                                   chctl, mu0, lc_unused, lv_unused, lgc_unused, own);
      double send[3] = {0, 0, 0}, recv[3] = {0, 0, 0};
      const int a0 = __ldg(T.adj_ptr + gi), a1 = __ldg(T.adj_ptr + gi + 1);
      for (int a = a0; a < a1; ++a) {
        const int code = __ldg(T.adj_idx + a);
        const long long ge = e0 + (code >> 1);
#pragma unroll
        for (int s = 0; s < 3; ++s) {
          if (code & 1) recv[s] += es[(AE_J + s) * E + ge];
          else send[s] += -es[(AE_J + s) * E + ge];
        }
      }
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        const double rate = (own[s] + send[s]) + recv[s];
        n1[s] = n[s] + k.gamma_dt * rate;
        cw[(AC_C1 + s) * C + gi] = (__ldg(T.ref + s * C + gi) + n1[s]) * ivol;
      }
      const double V1 = cell_potential(T, gi, Vb, n1);
      const double V2 = cell_potential(T, gi, Vb, n2);
      cw[AC_V1 * C + gi] = V1;
      double lv0 = 0.0, lv2 = 0.0;
      if constexpr (NCH > 0) {
#pragma unroll
        for (int q = 0; q < NCH; ++q) {
          const int code = __ldg(T.ch_code + q * C + gi);
          double t0[2], tau0[2], t1[2], tau1[2], t2[2], tau2[2], d0[2], dtau0[2], d2[2], dtau2[2];
          channel_kinetics<false>(code, V0 - Vb, t0, tau0);
          channel_kinetics<false>(code, V1 - Vb, t1, tau1);
          channel_kinetics<false>(code, V2 - Vb, t2, tau2);
          channel_slope(code, V0 - Vb, d0, dtau0);
          channel_slope(code, V2 - Vb, d2, dtau2);
#pragma unroll
          for (int r = 0; r < 2; ++r) {
            const long long slot = oH + (r * NCH + q) * C + gi;
            const double gc = St[slot];
            const bool active = !(r == 1 && code == kHhKn4);
            cw[(AC_GC1 + r * NCH + q) * C + gi] =
                active ? advance_gate<false>(gc, t0[r], tau0[r], t1[r], tau1[r], k.frac1_dt) : gc;
            const double lam = cot[slot];
            if (active) {
              const GatePartials p = advance_partials(gc, t0[r], tau0[r], t2[r], tau2[r],
                                                      k.frac2_dt);
              cot[slot] = lam * p.g;
              lv0 += lam * (p.ts * d0[r] + p.taus * dtau0[r]);
              lv2 += lam * (p.te * d2[r] + p.taue * dtau2[r]);
            }
          }
        }
      }
      cw[AC_LV0 * C + gi] = lv0;
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        const double lam = cot[oN + s * C + gi] + lv2 * (K * z3[s]) * icap;
        cot[oN + s * C + gi] = lam;
        cw[(AC_MU0 + s) * C + gi] = k.delta_dt * lam;
        cw[(AC_MU1 + s) * C + gi] = k.omdelta_dt * lam;
      }
    }
    __syncthreads();
    // P4 (junctions): stage 1, transposed.
    for (int e = tid; e < ne; e += BLOCK) {
      const long long ge = e0 + e;
      const long long ga = c0 + __ldg(T.snd + ge), gb = c0 + __ldg(T.rcv + ge);
      double ca[3], cb[3], ma[3], mb[3], da[3], db[3], ddv;
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        ca[s] = cs[(AC_C1 + s) * C + ga];
        cb[s] = cs[(AC_C1 + s) * C + gb];
        ma[s] = cs[(AC_MU1 + s) * C + ga];
        mb[s] = cs[(AC_MU1 + s) * C + gb];
      }
      const double lam_g = cot[oG + ge];
      const double lg1 = edge_vjp(T, A, sW, ge, ca, cb, cs[AC_V1 * C + ga] - cs[AC_V1 * C + gb],
                                  es[AE_G1 * E + ge], __ldg(jctl + ge), ma, mb,
                                  k.omdelta_dt * lam_g, da, db, ddv);
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        es[(AE_DA + s) * E + ge] = da[s];
        es[(AE_DB + s) * E + ge] = db[s];
      }
      es[AE_DV * E + ge] = ddv;
      cot[oG + ge] = lam_g + lg1;
      es[AE_MU0G * E + ge] = k.delta_dt * lam_g + k.gamma_dt * lg1;
    }
    __syncthreads();
    // P5 (cells): stage 1, transposed; the stage-1 gates' update, transposed.
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      const double mc = control[L.c[CB_CONTROL_MEMBRANE] + gi];
      const double pctl = control[L.c[CB_CONTROL_PUMP] + gi];
      const double ldc = pctl > 0.0 ? __ldg(T.logpcap + gi) + log(pctl) : 0.0;
      const double *chctl = control + L.c[CB_CONTROL_CHANNEL] + gi;
      double c[3], mu[3], lc[3] = {0, 0, 0}, lv = 0.0, lgc[2][NQ] = {}, own[3];
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        c[s] = cs[(AC_C1 + s) * C + gi];
        mu[s] = cs[(AC_MU1 + s) * C + gi];
      }
      gather_edges(T, A, gi, e0, lc, lv);
      const double V1 = cs[AC_V1 * C + gi];
      cell_terms<NCH, false, true>(T, A, sW, gi, c, V1, cs + AC_GC1 * C + gi, NCH * C, mc, pctl,
                                   ldc, chctl, mu, lc, lv, lgc, own);
      if constexpr (NCH > 0) {
        const double V0 = cs[AC_V0 * C + gi];
        double lv0 = cw[AC_LV0 * C + gi];
#pragma unroll
        for (int q = 0; q < NCH; ++q) {
          const int code = __ldg(T.ch_code + q * C + gi);
          double t0[2], tau0[2], t1[2], tau1[2], d0[2], dtau0[2], d1[2], dtau1[2];
          channel_kinetics<false>(code, V0 - Vb, t0, tau0);
          channel_kinetics<false>(code, V1 - Vb, t1, tau1);
          channel_slope(code, V0 - Vb, d0, dtau0);
          channel_slope(code, V1 - Vb, d1, dtau1);
#pragma unroll
          for (int r = 0; r < 2; ++r) {
            const long long slot = oH + (r * NCH + q) * C + gi;
            const bool active = !(r == 1 && code == kHhKn4);
            const double lam = lgc[r][q];
            if (active) {
              const GatePartials p =
                  advance_partials(St[slot], t0[r], tau0[r], t1[r], tau1[r], k.frac1_dt);
              cot[slot] += lam * p.g;
              lv0 += lam * (p.ts * d0[r] + p.taus * dtau0[r]);
              lv += lam * (p.te * d1[r] + p.taue * dtau1[r]);
            } else {
              cot[slot] += lam;
            }
          }
        }
        cw[AC_LV0 * C + gi] = lv0;
      }
      const double ivol = __ldg(T.ivol + gi), icap = __ldg(T.icap + gi);
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        const double lam1 = lc[s] * ivol + lv * (K * z3[s]) * icap;
        cot[oN + s * C + gi] += lam1;
        cw[(AC_MU0 + s) * C + gi] += k.gamma_dt * lam1;
      }
    }
    __syncthreads();
    // P6 (junctions): stage 0, transposed.
    for (int e = tid; e < ne; e += BLOCK) {
      const long long ge = e0 + e;
      const long long ga = c0 + __ldg(T.snd + ge), gb = c0 + __ldg(T.rcv + ge);
      double ca[3], cb[3], ma[3], mb[3], da[3], db[3], ddv;
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        ca[s] = cs[(AC_C0 + s) * C + ga];
        cb[s] = cs[(AC_C0 + s) * C + gb];
        ma[s] = cs[(AC_MU0 + s) * C + ga];
        mb[s] = cs[(AC_MU0 + s) * C + gb];
      }
      const double lg0 = edge_vjp(T, A, sW, ge, ca, cb, cs[AC_V0 * C + ga] - cs[AC_V0 * C + gb],
                                  St[oG + ge], __ldg(jctl + ge), ma, mb, es[AE_MU0G * E + ge],
                                  da, db, ddv);
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        es[(AE_DA + s) * E + ge] = da[s];
        es[(AE_DB + s) * E + ge] = db[s];
      }
      es[AE_DV * E + ge] = ddv;
      cot[oG + ge] += lg0;
    }
    __syncthreads();
    // P7 (cells): stage 0, transposed; the start potential's cotangent to the amounts.
    for (int i = tid; i < nc; i += BLOCK) {
      const long long gi = c0 + i;
      const double mc = control[L.c[CB_CONTROL_MEMBRANE] + gi];
      const double pctl = control[L.c[CB_CONTROL_PUMP] + gi];
      const double ldc = pctl > 0.0 ? __ldg(T.logpcap + gi) + log(pctl) : 0.0;
      const double *chctl = control + L.c[CB_CONTROL_CHANNEL] + gi;
      double c[3], mu[3], lc[3] = {0, 0, 0}, lv = 0.0, lgc[2][NQ] = {}, own[3];
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        c[s] = cs[(AC_C0 + s) * C + gi];
        mu[s] = cs[(AC_MU0 + s) * C + gi];
      }
      gather_edges(T, A, gi, e0, lc, lv);
      cell_terms<NCH, false, true>(T, A, sW, gi, c, cs[AC_V0 * C + gi], St + oH + gi, NCH * C,
                                   mc, pctl, ldc, chctl, mu, lc, lv, lgc, own);
      if constexpr (NCH > 0) {
#pragma unroll
        for (int q = 0; q < NCH; ++q)
#pragma unroll
          for (int r = 0; r < 2; ++r) cot[oH + (r * NCH + q) * C + gi] += lgc[r][q];
      }
      const double lv0 = cs[AC_LV0 * C + gi] + lv;
      const double ivol = __ldg(T.ivol + gi), icap = __ldg(T.icap + gi);
#pragma unroll
      for (int s = 0; s < 3; ++s)
        cot[oN + s * C + gi] += lc[s] * ivol + lv0 * (K * z3[s]) * icap;
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

struct WorkspacePlan {
  size_t states, taken, status, cells, edges, total;
};

WorkspacePlan plan(const cb_tissue *t, int n_steps) {
  WorkspacePlan p;
  p.states = 0;
  p.taken = align256(sizeof(double) * (size_t)t->state_total * (size_t)n_steps);
  p.status = p.taken + align256(sizeof(int32_t) * (size_t)t->W * (size_t)n_steps);
  p.cells = p.status + align256(sizeof(uint32_t) * (size_t)t->W * (size_t)n_steps);
  p.edges = p.cells + align256(sizeof(double) * (size_t)adj_cell_fields(t->t.nch) * t->C);
  p.total = p.edges + align256(sizeof(double) * (size_t)AE_FIELDS * std::max(t->E, 1));
  return p;
}

// CTA shape of the reverse kernel: 128 threads at 4 CTAs per SM (every world of a 512-world batch
// resident at once; measured 5% faster than 256 threads at 2 per SM, the same threads per SM), or
// 256. CELLS_B200_VJP_BLOCK overrides.
template <int NCH>
int launch_vjp(cb_tissue *t, const Adj &A, const double *control, const StepCoef &k,
               int n_steps, cudaStream_t stream) {
  int block = 128;
  if (const char *env = std::getenv("CELLS_B200_VJP_BLOCK")) block = std::atoi(env) == 128 ? 128 : 256;
  if (block == 128)
    vjp_kernel<128, NCH, 4><<<t->W, 128, 0, stream>>>(t->t, t->layout, A, control, k, n_steps);
  else
    vjp_kernel<256, NCH, 2><<<t->W, 256, 0, stream>>>(t->t, t->layout, A, control, k, n_steps);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "vjp launch");
  return CB_OK;
}

}  // namespace

extern "C" {

int cb_vjp_workspace(const cb_tissue *t, int n_steps, size_t *bytes) {
  if (!t || !bytes) return fail(CB_ERR_ARGUMENT, "null argument");
  if (n_steps < 0) return fail(CB_ERR_ARGUMENT, "n_steps must be non-negative");
  *bytes = plan(t, n_steps).total;
  return CB_OK;
}

int cb_step_vjp(cb_tissue *t, const double *state_in, double dt, const double *control,
                int n_steps, const double *cot_out, double *cot_in, double *grad_membrane,
                double *grad_junction, double *grad_channel, void *workspace,
                size_t workspace_bytes, uint32_t *world_status, void *stream) {
  if (!t || !state_in || !control || !cot_out || !cot_in || !grad_membrane || !world_status ||
      (t->E && !grad_junction) || (t->t.nch && !grad_channel) || !workspace)
    return fail(CB_ERR_ARGUMENT, "null argument");
  if (t->t.blk_modes > 0)
    return fail(CB_ERR_UNSUPPORTED, "the adjoint step has no open-channel block");
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(CB_ERR_ARGUMENT, "dt must be positive");
  if (n_steps < 0) return fail(CB_ERR_ARGUMENT, "n_steps must be non-negative");
  const WorkspacePlan p = plan(t, n_steps);
  if (workspace_bytes < p.total) return fail(CB_ERR_ARGUMENT, "workspace too small");
  if (reinterpret_cast<uintptr_t>(workspace) % 256)
    return fail(CB_ERR_ARGUMENT, "workspace must be 256-byte aligned");
  cudaError_t ce = cudaSetDevice(t->device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  char *ws = static_cast<char *>(workspace);
  double *states = reinterpret_cast<double *>(ws + p.states);
  int32_t *taken = reinterpret_cast<int32_t *>(ws + p.taken);
  uint32_t *status = reinterpret_cast<uint32_t *>(ws + p.status);
  // The forward, one step per launch, every state kept.
  for (int step = 0; step < n_steps; ++step) {
    const double *in = step == 0 ? state_in : states + (size_t)(step - 1) * t->state_total;
    const int rc = cb_step(t, CB_METHOD_ARS222, in, states + (size_t)step * t->state_total, dt,
                           control, 1, status + (size_t)step * t->W,
                           taken + (size_t)step * t->W, stream);
    if (rc) return rc;
  }
  if (cot_in != cot_out) {
    ce = cudaMemcpyAsync(cot_in, cot_out, sizeof(double) * t->state_total,
                         cudaMemcpyDeviceToDevice, s);
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaMemcpyAsync");
  }
  Adj A;
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
  const StepCoef k = step_coef(dt);
  if (t->t.nch == 2) return launch_vjp<2>(t, A, control, k, n_steps, s);
  if (t->t.nch == 0) return launch_vjp<0>(t, A, control, k, n_steps, s);
  return fail(CB_ERR_UNSUPPORTED, "channel slots must be 0 or 2");
}

}  // extern "C"
