// adjoint_terms.cuh - the transposed linearisation of the explicit rate terms, shared by the
// ARS(2,2,2) reverse (adjoint_step.cu) and the ROS2 reverse (ros2_adjoint.cu): a cell's own
// terms (patch flux, Na/K-ATPase, channel populations) and a junction's flux and gate rate, each
// with its permeability gradients.
#pragma once

#include <cuda_runtime.h>

#include "handle.h"

namespace {

using namespace cbk;

// The reverse pass's buffers: the segment's states, the running cotangent, the gradients and
// the scratch. The rate terms below use the gradients and the areas.
struct Adj {
  const double *state_in;  // the segment's first state
  const double *states;    // [n_steps][state_total]: the state after each step
  long long state_total;
  const int32_t *taken;    // [n_steps][W]: 1 when the world's step was accepted
  const uint32_t *fwd_status;  // [n_steps][W]
  double *cot;             // [state_total]: end cotangent in, start cotangent out
  double *gm;              // [3][C]  d/d membrane permeability (added)
  double *gj;              // [3][E]  d/d junction permeability (added)
  double *gch;             // [NCH][C] d/d channel permeability (added)
  double *cs;              // [adj_cell_fields][C]
  double *es;              // [AE_FIELDS][E]
  const double *area;      // [C]
  const double *jarea;     // [E]
  uint32_t *status;        // [W]
};

// B'(x), the channel laws' voltage slopes and sigmoid: laws.cuh.

__device__ __forceinline__ void opening_partials(int code, double m, double h, double &dm,
                                                 double &dh) {
  if (code == kNav1p2) {
    dm = 3.0 * m * m * h;
    dh = m * m * m;
  } else if (code == kHhKn4) {
    dm = 4.0 * m * m * m;
    dh = 0.0;
  } else {
    dm = h;
    dh = m;
  }
}

__device__ __forceinline__ double cell_potential(const Tissue &T, long long gi, double Vb,
                                                 const double (&n)[3]) {
  return (__ldg(T.q0 + gi) + kChargePerFmol * ((n[0] + n[1]) + (-n[2]))) * __ldg(T.icap + gi) +
         Vb;
}

// One cell's own rate terms at a stage (patch flux, pump, channel populations) and, given their
// amount-rate cotangents mu[3], their transposed linearisation: adds d/dc to lc[3], d/dV to lv,
// d/d gates to lgc, and the permeability gradients to A.gm / A.gch. With FWD, also returns the
// forward rate terms: rate_own[s] = -J_m,s + stoichiometry_s cycles - channel_s (the amount rate
// without the junctions).
template <int NCH, bool FWD, bool VJP>
__device__ __forceinline__ void cell_terms(const Tissue &T, const Adj &A,
                                           const double *__restrict__ wc, long long gi,
                                           const double (&c)[3], double V, const double *gcp,
                                           long long gstride, double mc, double pctl,
                                           double log_drive_cap, const double *chctl,
                                           const double (&mu)[3], double (&lc)[3], double &lv,
                                           double (&lgc)[2][NCH > 0 ? NCH : 1],
                                           double (&rate_own)[3]) {
  const long long C = T.C;
  const double Vb = wc[WC_VB], RT = wc[WC_RT], FRT = wc[WC_FRT];
  const double dv = V - Vb;
  const double x = dv * FRT;
  double bp, bm, sp = 0.0, sm = 0.0;
  bernoulli_pair<double>(x, bp, bm);
  if (VJP) bernoulli_slope_pair(x, sp, sm);
  const double area_f = VJP ? __ldg(A.area + gi) / 1e-15 : 0.0;
  double lcv[3];
#pragma unroll
  for (int s = 0; s < 3; ++s) lcv[s] = log(c[s]);
  // Patch: J_s = A P_s mc (c B(-x_s) - co B(x_s)) / 1e-15; the amount rate takes -J_s.
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    const double ap = __ldg(T.ap + s * C + gi);
    const double co = wc[WC_CO + s];
    const double diff = s < 2 ? c[s] * bm - co * bp : c[s] * bp - co * bm;
    if (FWD) rate_own[s] = -(ap * mc * diff);
    if (VJP) {
      const double g = ap * mc;
      const double m = -mu[s];
      lc[s] += m * g * (s < 2 ? bm : bp);
      lv += m * g * (s < 2 ? (-c[s] * sm - co * sp) : (c[s] * sp + co * sm)) * FRT;
      A.gm[s * C + gi] += m * (area_f * mc) * diff;
    }
  }
  // Na/K-ATPase: cycles = -M expm1(a), M = cap avail exp(log saturation); the amount rates take
  // -3 cycles (Na) and +2 cycles (K).
  if (__ldg(T.pcap + gi) > 0.0 && pctl > 0.0) {
    const double mu_na = RT * (lcv[0] - wc[WC_LOGCO]) + kF * dv;
    const double mu_k = RT * (lcv[1] - wc[WC_LOGCO + 1]) + kF * dv;
    const double energy = (wc[WC_DRIVE] + (-3.0) * mu_na) + 2.0 * mu_k;
    const double a = energy * wc[WC_INVRT];
    const double u = 3.0 * (wc[WC_LOGKMNA] - lcv[0]);
    const double ls = ((-logaddexp0(u)) - wc[WC_LK]) - wc[WC_LATP];
    const double mag = exp((log_drive_cap + ls) + fmax(a, 0.0));
    const double cycles = mag * (a >= 0.0 ? expm1(-a) : -expm1(a));
    if (FWD) {
      rate_own[0] += -3.0 * cycles;
      rate_own[1] += 2.0 * cycles;
    }
    if (VJP) {
      const double dcda = -(a >= 0.0 ? mag : mag * exp(a));  // -M e^a
      const double m = -3.0 * mu[0] + 2.0 * mu[1];
      lc[0] += m * (cycles * 3.0 * sigmoid(u) / c[0] - 3.0 * dcda / c[0]);
      lc[1] += m * (2.0 * dcda / c[1]);
      lv += m * dcda * (-FRT);
    }
  }
  // Channel populations: J = A P_ch open ctl ab (c B(-x) - co B(x)) / 1e-15 of the permeant
  // species; the amount rate takes -J.
  if constexpr (NCH > 0) {
#pragma unroll
    for (int q = 0; q < NCH; ++q) {
      const int code = __ldg(T.ch_code + q * C + gi);
      const int sp_ = __ldg(T.ch_species + q * C + gi);
      const double ctl = __ldg(chctl + q * C);
      const double ab = __ldg(T.ch_ab + q * C + gi);
      const double chap = __ldg(T.ch_ap + q * C + gi);
      const double m_ = gcp[q * C], h_ = gcp[gstride + q * C];
      const double open = channel_opening(code, m_, h_);
      const double cs = sp_ == 0 ? c[0] : sp_ == 1 ? c[1] : c[2];
      const double co = wc[WC_CO + sp_];
      const double diff = sp_ < 2 ? cs * bm - co * bp : cs * bp - co * bm;
      const double gq = chap * ((open * ctl) * ab);
      if (FWD) {
        const double J = gq * diff;
        if (sp_ == 0) rate_own[0] -= J;
        else if (sp_ == 1) rate_own[1] -= J;
        else rate_own[2] -= J;
      }
      if (VJP) {
        const double m = -(sp_ == 0 ? mu[0] : sp_ == 1 ? mu[1] : mu[2]);
        const double dcs = m * gq * (sp_ < 2 ? bm : bp);
        if (sp_ == 0) lc[0] += dcs;
        else if (sp_ == 1) lc[1] += dcs;
        else lc[2] += dcs;
        lv += m * gq * (sp_ < 2 ? (-cs * sm - co * sp) : (cs * sp + co * sm)) * FRT;
        A.gch[q * C + gi] += m * (area_f * ((open * ctl) * ab)) * diff;
        double dm, dh;
        opening_partials(code, m_, h_, dm, dh);
        const double dopen = m * (chap * ctl * ab) * diff;
        lgc[0][q] += dopen * dm;
        lgc[1][q] += dopen * dh;
      }
    }
  }
}

// One junction's transposed linearisation at a stage: amount-rate cotangents mu_a, mu_b of its
// sender and receiver and the gate-rate cotangent mu_g in; contributions to the end cells'
// concentrations (da, db) and to the potential difference (dv) out, the gate's cotangent
// returned, the junction permeability gradients added.
__device__ __forceinline__ double edge_vjp(const Tissue &T, const Adj &A,
                                           const double *__restrict__ wc, long long ge,
                                           const double (&ca)[3], const double (&cb)[3],
                                           double dve, double g, double jc,
                                           const double (&mu_a)[3], const double (&mu_b)[3],
                                           double mu_g, double (&da)[3], double (&db)[3],
                                           double &ddv) {
  const long long E = T.E;
  const double FRT = wc[WC_FRT];
  const double x = dve * FRT;
  double bp, bm, sp, sm;
  bernoulli_pair<double>(x, bp, bm);
  bernoulli_slope_pair(x, sp, sm);
  const double opening = jc * g;
  const double jarea_f = __ldg(A.jarea + ge) / 1e-15;
  double lg = 0.0;
  ddv = 0.0;
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    const double jap = __ldg(T.jap + s * E + ge);
    const double gs = jap * opening;
    const double xi = mu_b[s] - mu_a[s];  // sender takes -J, receiver +J
    const double diff = s < 2 ? ca[s] * bm - cb[s] * bp : ca[s] * bp - cb[s] * bm;
    da[s] = xi * gs * (s < 2 ? bm : bp);
    db[s] = -xi * gs * (s < 2 ? bp : bm);
    ddv += xi * gs * (s < 2 ? (-ca[s] * sm - cb[s] * sp) : (ca[s] * sp + cb[s] * sm)) * FRT;
    lg += xi * (jap * jc) * diff;
    A.gj[s * E + ge] += xi * (jarea_f * opening) * diff;
  }
  // Gate rate alpha (1 - g) - beta (g - min), shift = |dv| - threshold (the law's own form,
  // also for pinned gates, whose rate and voltage slope vanish at g = min = 1).
  const double thr = __ldg(T.thr + ge), mn = __ldg(T.jmin + ge);
  const double shift = fabs(dve) - thr;
  const double alpha = 1.3 * exp(-77.0 * shift);
  const double sb = sigmoid(kLog0065 + 140.0 * shift);
  const double beta = 20.0 * sb;
  lg += mu_g * (-alpha - beta);
  const double sgn = dve > 0.0 ? 1.0 : dve < 0.0 ? -1.0 : 0.0;
  ddv += mu_g * sgn * (-77.0 * alpha * (1.0 - g) - (20.0 * 140.0) * sb * (1.0 - sb) * (g - mn));
  return lg;
}

}  // namespace
