// tissue_step.cu - the B200 (sm_100a) pump-leak tissue step and its C ABI.
//
// One CTA advances one world. A thread owns one cell (its patch, its pump) and up to EPT
// junctions of that world (edge-parallel). Per right-hand-side evaluation:
//   1. cell phase: concentrations, their logs and the cell potential go to shared memory; the
//      patch's constant-field flux and the Na/K-ATPase are evaluated in registers;
//   2. edge phase: each junction's constant-field flux is evaluated once and stored in shared
//      memory (species-major), its dissipation and gate rate kept in registers;
//   3. gather phase: each cell sums its junction fluxes over its CSR adjacency in edge order
//      (senders first, then receivers, as the reference's scatter-adds order them), so results
//      are bit-identical run to run - no atomics anywhere.
// World sums (the held bath's inflow, the electrode plate charge) are fixed-order block
// reductions. State lives in registers across the n_steps of one launch; HBM sees it once in
// and once out per launch.
//
// Arithmetic follows the reference expressions (Cells src/cells):
//   laws/electrochemistry.py:25-48           bernoulli, ghk route flux
//   laws/junctions/selective.py:28-50         selective_flux (residual 0, gate 1)
//   laws/pumps/nak_atp_mass_action_positive.py:55-148  pump kinetics and domain
//   laws/junctions/junction_voltage_relaxation.py:43-97 gate rate and domain
//   numerics/surface_transport.py:298-386     route transport, scatters
//   models/surface_pump.py:158-362            explicit_rates, imex_step (ARS(2,2,2)), ledgers
//   numerics/surface_imex.py:47-69            the ARS(2,2,2) tableau
// Two deliberate differences, both at the last-ulp level: the cell potential is Q/C plus the
// bath potential (the reference reaches the same value through a diagonal Cholesky solve of the
// scaled capacitor matrix), and the pair B(x), B(-x) comes from one expm1 (B(-x) = x + B(x),
// taken on the side where it does not cancel).

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "handle.h"

namespace cbk {

thread_local std::string g_error;

int fail(int code, const std::string &msg) {
  g_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char *what) {
  g_error = std::string(what) + ": " + cudaGetErrorString(e);
  return CB_ERR_CUDA;
}

const char *last_error() { return g_error.c_str(); }

}  // namespace cbk

namespace {

using namespace cbk;

// One explicit stage (surface_pump.explicit_rates, surface_pump.py:158-240) for this thread's
// cell and junction slots, each rate folded into the step accumulator as soon as it is formed
// (surface_pump._combine's y + (w dt) k, one term at a time):
//   FIRST  (stage 0): acc = y + (delta dt) k, with y read from `cur`; and the stage-1 amounts
//                     and gates n1 = n + (gamma dt) k_n, g1 = g + (gamma dt) k_g;
//   !FIRST (stage 1): acc = acc + ((1 - delta) dt) k.
// n, g: the stage's amounts and gates; V: this thread's cell potential. sA/sE hold the cell and
// junction accumulators in slots private to each thread. inflow: this cell's patch flux plus pump
// transfer (the held bath's inflow terms).
template <int BLOCK, int EPT, int NCH, bool FIRST, bool MIX>
__device__ __forceinline__ void stage(
    const Tissue &T, const Layout &L, const double *__restrict__ wc, const StepCoef &k,
    const double *cur, int c0, int e0, int ne, int i, bool has_cell, const double (&n)[3],
    double V, const double (&g)[EPT], const double (&chg)[2][NCH > 0 ? NCH : 1], double mc,
    double pc_ctl, double log_drive_cap, const double *__restrict__ jctl,
    const double *__restrict__ chctl, double *sV, double *sC, double *sL, double *sJ, double *sA,
    double *sE, double *sH, double (&n1)[3], double (&g1)[EPT], double (&inflow)[3],
    uint32_t &bits) {
  constexpr int EB = EPT * BLOCK;
  const double w = FIRST ? k.delta_dt : k.omdelta_dt;
  const long long C = T.C, E = T.E;
  const double RT = wc[WC_RT];
  const double Vb = wc[WC_VB];
  const int gi = c0 + i;
  // Accumulate one cell ledger field f (slot f of sA) with rate r.
  auto cell_acc = [&](int f, long long off, double r) {
    double *slot = sA + f * BLOCK + i;
    if (FIRST)
      *slot = cur[off + gi] + w * r;
    else
      *slot = *slot + w * r;
  };
  double jm[3] = {0.0, 0.0, 0.0}, extra[3] = {0.0, 0.0, 0.0};
  if (has_cell) {
    double c[3], lc[3];
    const double ivol = __ldg(T.ivol + gi);
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      c[s] = (__ldg(T.ref + s * C + gi) + n[s]) * ivol;
      lc[s] = log(c[s]);
      sL[s * BLOCK + i] = lc[s];
      if (!(is_finite(c[s]) && c[s] > 0.0)) bits |= CB_WORLD_TRANSPORT;
      sC[s * BLOCK + i] = c[s];
    }
    sV[i] = V;
    if (!is_finite(V)) bits |= CB_WORLD_TRANSPORT;
    // Patch: constant-field flux per species (selective_flux with residual 0, gate 1).
    const double dv = V - Vb;
    const double x = dv * wc[WC_FRT];
    if (!(fabs(x) <= kMaxAbsX)) bits |= CB_WORLD_TRANSPORT;
    double bp, bm;
    bernoulli_pair_at<MIX>(x, bp, bm);
    double mu[3];
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      const double gs = __ldg(T.ap + s * C + gi) * mc;
      const double co = wc[WC_CO + s];
      const double zfdv = (s < 2) ? kF * dv : (-kF) * dv;
      if constexpr (MIX) {
        // FP32 with the concentration difference formed in FP64: c_in B(-x) - c_out B(x) =
        // (c_in - c_out) B(x) + c_in x for z = +1, (c_in - c_out) B(x) - c_out x for z = -1.
        const float d = (float)(c[s] - co);
        const float fb = (float)bp, fx = (float)x;
        const float J = (float)gs * ((s < 2) ? d * fb + (float)c[s] * fx
                                             : d * fb - (float)co * fx);
        jm[s] = J;
      } else {
        // Na, K: z = +1 -> (c_in B(-x) - c_out B(x)); Cl: z = -1 swaps the pair.
        jm[s] = (s < 2) ? gs * (c[s] * bm - co * bp) : gs * (c[s] * bp - co * bm);
      }
      mu[s] = RT * (lc[s] - wc[WC_LOGCO + s]) + zfdv;
      cell_acc(3 + s, L.s[CB_MEMBRANE_TRANSFERRED] + s * C, jm[s]);
    }
    const double md = 1e-3 * ((jm[0] * mu[0] + jm[1] * mu[1]) + jm[2] * mu[2]);
    cell_acc(6, L.s[CB_MEMBRANE_DISSIPATED], md);
    if (!(is_finite(jm[0]) && is_finite(jm[1]) && is_finite(jm[2]) && is_finite(md)))
      bits |= CB_WORLD_TRANSPORT;
    if (!(is_finite(mc) && mc >= 0.0 && mc <= 1.0 && is_finite(pc_ctl) && pc_ctl >= 0.0 &&
          pc_ctl <= 1.0))
      bits |= CB_WORLD_CONTROL;
    // Explicit-stability refusal (surface_pump_v3.membrane_rate, :4588-4660): dt times the
    // cell's constant-field slope conductance over its capacitance must stay <= 1.
    double largest[3];
#pragma unroll
    for (int s = 0; s < 3; ++s) largest[s] = fmax(c[s], wc[WC_CO + s]);
    double membrane =
        ((((__ldg(T.ap + gi) * largest[0]) + __ldg(T.ap + C + gi) * largest[1]) +
          __ldg(T.ap + 2 * C + gi) * largest[2]) * 1e-15) * mc;
    // Channel populations (surface_pump_v3.channel_rates, :937-963): the permeant species'
    // constant-field flux at the patch voltage (the patch's Bernoulli pair), opening times
    // availability times abundance.
    double chm[3] = {0.0, 0.0, 0.0};
    if constexpr (NCH > 0) {
#pragma unroll
      for (int q = 0; q < NCH; ++q) {
        const int code = __ldg(T.ch_code + q * C + gi);
        const int sp = __ldg(T.ch_species + q * C + gi);
        const double ctl = __ldg(chctl + q * C);
        if (!(is_finite(ctl) && ctl >= 0.0 && ctl <= 1.0)) bits |= CB_WORLD_CONTROL;
        const double open = channel_opening(code, chg[0][q], chg[1][q]);
        const double available = (open * ctl) * __ldg(T.ch_ab + q * C + gi);
        const double gq = __ldg(T.ch_ap + q * C + gi) * available;
        const double cs = sp == 0 ? c[0] : sp == 1 ? c[1] : c[2];
        const double cos_ = wc[WC_CO + sp];
        const double musp = sp == 0 ? mu[0] : sp == 1 ? mu[1] : mu[2];
        double J, Jd;
        if constexpr (MIX) {
          const float d = (float)(cs - cos_), fb = (float)bp, fx = (float)x;
          J = (float)gq * (sp < 2 ? d * fb + (float)cs * fx : d * fb - (float)cos_ * fx);
        } else {
          J = sp < 2 ? gq * (cs * bm - cos_ * bp) : gq * (cs * bp - cos_ * bm);
        }
        Jd = 1e-3 * J * musp;
        chm[sp] += J;
        membrane += ((__ldg(T.ch_ap + q * C + gi) * 1e-15) * (sp == 0 ? largest[0]
                     : sp == 1 ? largest[1] : largest[2])) * available;
        double *tr = sH + q * BLOCK + i, *dd = sH + (NCH + q) * BLOCK + i;
        if (FIRST) {
          *tr = cur[L.s[CB_CHANNEL_TRANSFERRED] + q * C + gi] + w * J;
          *dd = cur[L.s[CB_CHANNEL_DISSIPATED] + q * C + gi] + w * Jd;
        } else {
          *tr = *tr + w * J;
          *dd = *dd + w * Jd;
        }
        if (!(is_finite(J) && is_finite(Jd))) bits |= CB_WORLD_TRANSPORT;
      }
    }
    if (!(k.dt * (wc[WC_SLOPE] * membrane * __ldg(T.icap + gi)) <= 1.0)) bits |= CB_WORLD_STIFF;
    // Na/K-ATPase (nak_atp_mass_action_positive.kinetics), Na inside, K in the bath.
    const double drive = wc[WC_DRIVE];
    const double energy = (drive + (-3.0) * mu[0]) + 2.0 * mu[1];
    const double a = energy * wc[WC_INVRT];
    double cycles = 0.0;
    if (__ldg(T.pcap + gi) > 0.0 && pc_ctl > 0.0) {
      const double ls =
          ((-logaddexp0(3.0 * (wc[WC_LOGKMNA] - lc[0]))) - wc[WC_LK]) - wc[WC_LATP];
      const double mag = exp((log_drive_cap + ls) + fmax(a, 0.0));
      const double dep = a >= 0.0 ? expm1(-a) : -expm1(a);
      cycles = mag * dep;
    }
    const double pd = (-1e-3 * cycles) * energy;
    const double mw = (-1e-3 * cycles) * drive;
    cell_acc(7, L.s[CB_PUMP_CYCLES], cycles);
    cell_acc(8, L.s[CB_PUMP_DISSIPATED], pd);
    cell_acc(9, L.s[CB_METABOLIC_WORK], mw);
    // -stoichiometry * cycles (outward-positive) plus the channels' transfer.
    extra[0] = (3.0 * cycles - 0.0) + chm[0];
    extra[1] = (-2.0 * cycles - 0.0) + chm[1];
    extra[2] = (-0.0 * cycles - 0.0) + chm[2];
    // Pump domain (positive substrates, parameters, |mu/RT| <= 1600, |affinity| <= 80).
    const double sna = mu[0] * wc[WC_INVRTD], sk = mu[1] * wc[WC_INVRTD];
    const double aff = (wc[WC_AFF0] + (-3.0) * sna) + 2.0 * sk;
    const double capacity = __ldg(T.pcap + gi);
    const bool pump_ok = wc[WC_PUMPOK] != 0.0 && is_finite(capacity) && capacity >= 0.0 &&
                         is_finite(sna) && fabs(sna) <= kMaxAbsIonPotentialOverRT && is_finite(sk) &&
                         fabs(sk) <= kMaxAbsIonPotentialOverRT && is_finite(aff) &&
                         fabs(aff) <= kMaxAbsAffinityOverRT;
    if (!pump_ok) bits |= CB_WORLD_PUMP_DOMAIN;
    if (!(is_finite(cycles) && is_finite(pd) && is_finite(mw))) bits |= CB_WORLD_TRANSPORT;
  }
  __syncthreads();
  // Edge phase: each junction once, its fluxes to shared memory for the gather.
#pragma unroll
  for (int q = 0; q < EPT; ++q) {
    const int e = threadIdx.x + q * BLOCK;
    g1[q] = g[q];
    if (e < ne) {
      const int ge = e0 + e;
      const int s_ = __ldg(T.snd + ge), r_ = __ldg(T.rcv + ge);
      const double dv = sV[s_] - sV[r_];
      const double jc = __ldg(jctl + e);
      const double opening = jc * g[q];
      const double x = dv * wc[WC_FRT];
      if (!(fabs(x) <= kMaxAbsX)) bits |= CB_WORLD_TRANSPORT;
      double bp, bm;
      bernoulli_pair_at<MIX>(x, bp, bm);
      double jj[3], mu[3];
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        const double gs = __ldg(T.jap + s * E + ge) * opening;
        const double cs = sC[s * BLOCK + s_], cr = sC[s * BLOCK + r_];
        const double zfdv = (s < 2) ? kF * dv : (-kF) * dv;
        if constexpr (MIX) {
          // FP32 on the FP64 difference c_s - c_r (as the patch).
          const float d = (float)(cs - cr), fb = (float)bp, fx = (float)x;
          jj[s] = (float)gs * ((s < 2) ? d * fb + (float)cs * fx : d * fb - (float)cr * fx);
        } else {
          jj[s] = (s < 2) ? gs * (cs * bm - cr * bp) : gs * (cs * bp - cr * bm);
        }
        mu[s] = RT * (sL[s * BLOCK + s_] - sL[s * BLOCK + r_]) + zfdv;
        sJ[s * EB + e] = jj[s];
      }
      const double jd = 1e-3 * ((jj[0] * mu[0] + jj[1] * mu[1]) + jj[2] * mu[2]);
      // Junction gate (junction_voltage_relaxation.rhs); pinned gates (minimum 1) are exactly 0.
      const double thr = __ldg(T.thr + ge), mn = __ldg(T.jmin + ge);
      double gr = 0.0;
      if (mn < 1.0) {
        const double shift = fabs(dv) - thr;
        const double alpha = 1.3 * exp(-77.0 * shift);
        const double log_beta = kLog0065 + 140.0 * shift;
        const double beta = 20.0 * exp(-logaddexp0(-log_beta));
        gr = alpha * (1.0 - g[q]) - beta * (g[q] - mn);
      }
      if (FIRST) {
#pragma unroll
        for (int s = 0; s < 3; ++s)
          sE[s * EB + e] = cur[L.s[CB_JUNCTION_TRANSFERRED] + s * E + ge] + w * jj[s];
        sE[3 * EB + e] = cur[L.s[CB_JUNCTION_DISSIPATED] + ge] + w * jd;
        sE[4 * EB + e] = g[q] + w * gr;
        g1[q] = g[q] + k.gamma_dt * gr;
      } else {
#pragma unroll
        for (int s = 0; s < 3; ++s) sE[s * EB + e] = sE[s * EB + e] + w * jj[s];
        sE[3 * EB + e] = sE[3 * EB + e] + w * jd;
        sE[4 * EB + e] = sE[4 * EB + e] + w * gr;
      }
      if (!(is_finite(jj[0]) && is_finite(jj[1]) && is_finite(jj[2]) && is_finite(jd) && is_finite(gr)))
        bits |= CB_WORLD_TRANSPORT;
      const bool gate_ok = is_finite(thr) && thr >= 0.0 && thr <= kMaxAbsJunctionV && is_finite(mn) &&
                           mn >= 0.0 && mn <= 1.0 && is_finite(dv) && fabs(dv) <= kMaxAbsJunctionV &&
                           is_finite(g[q]) && g[q] >= mn && g[q] <= 1.0 && is_finite(jc) &&
                           jc >= 0.0 && jc <= 1.0;
      if (!gate_ok) bits |= CB_WORLD_GATE_DOMAIN;
    }
  }
  __syncthreads();
  // Gather phase: amount rate = ((-J_m + sum_send(-J)) + sum_recv(J)) - extra.
  if (has_cell) {
    double send[3] = {0.0, 0.0, 0.0}, recv[3] = {0.0, 0.0, 0.0};
    const int a0 = __ldg(T.adj_ptr + gi), a1 = __ldg(T.adj_ptr + gi + 1);
    for (int a = a0; a < a1; ++a) {
      const int code = __ldg(T.adj_idx + a);
      const int e = code >> 1;
      if (code & 1) {
#pragma unroll
        for (int s = 0; s < 3; ++s) recv[s] += sJ[s * EB + e];
      } else {
#pragma unroll
        for (int s = 0; s < 3; ++s) send[s] += -sJ[s * EB + e];
      }
    }
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      const double rate = ((-jm[s] + send[s]) + recv[s]) - extra[s];
      inflow[s] = jm[s] + extra[s];
      if (!is_finite(rate)) bits |= CB_WORLD_TRANSPORT;
      if (FIRST) {
        n1[s] = n[s] + k.gamma_dt * rate;
        sA[s * BLOCK + i] = n[s] + w * rate;
      } else {
        sA[s * BLOCK + i] = sA[s * BLOCK + i] + w * rate;
      }
    }
  } else {
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      inflow[s] = 0.0;
      if (FIRST) n1[s] = 0.0;
    }
  }
}

// Shared-memory words of one step CTA: stage potentials, concentrations and their logs, junction
// fluxes, the step accumulator (cells, junctions) and the reduction scratch.
__host__ __device__ constexpr size_t step_smem_words(int block, int ept, int nch) {
  return (size_t)(7 * block + 3 * ept * block + 10 * block + 5 * ept * block + 8 * nch * block +
                  (block / 32) * 8);
}

// The ARS(2,2,2) step of surface_pump.imex_step (surface_pump.py:259-362) for one world per CTA,
// n_steps times. Registers hold only one stage's transients: the step's start state is read from
// global memory (the launch's input, then this CTA's own last accepted state, which stays in L2
// across fused steps), and the accumulator y + delta dt k0 + (1 - delta) dt k1 lives in shared
// memory, in slots private to each thread.
template <int BLOCK, int EPT, int NCH, int MINB, bool MIX>
__global__ void __launch_bounds__(BLOCK, MINB)
    ars222_kernel(const Tissue T, const Layout L, const double *state_in, double *state_out,
                  const double *__restrict__ control, const StepCoef k, int n_steps,
                  uint32_t *__restrict__ world_status, int32_t *__restrict__ accepted_steps) {
  constexpr int EB = EPT * BLOCK;
  extern __shared__ double smem[];
  double *sV = smem;            // [BLOCK]
  double *sC = sV + BLOCK;      // [3][BLOCK]
  double *sL = sC + 3 * BLOCK;  // [3][BLOCK]
  double *sJ = sL + 3 * BLOCK;  // [3][EB]
  double *sA = sJ + 3 * EB;     // [10][BLOCK]: n[3], mt[3], md, pc, pd, mw
  double *sE = sA + 10 * BLOCK; // [5][EB]: jt[3], jd, g
  double *sH = sE + 5 * EB;     // [2*NCH][BLOCK]: channel transferred, dissipated accumulators
  double *sK = sH + 2 * NCH * BLOCK;  // [4*NCH][BLOCK]: start kinetics t[2][NCH], tau[2][NCH]
  double *sG = sK + 4 * NCH * BLOCK;  // [2*NCH][BLOCK]: the new state's gates
  double *sRed = sG + 2 * NCH * BLOCK;  // [BLOCK/32][8]
  __shared__ double sW[WC_STRIDE];
  __shared__ unsigned int sBits;

  const int w = k.world0 + blockIdx.x;
  const int tid = threadIdx.x;
  const int c0 = T.cell_offset[w], nc = T.cell_offset[w + 1] - c0;
  const int e0 = T.edge_offset[w], ne = T.edge_offset[w + 1] - e0;
  if (tid < WC_STRIDE) sW[tid] = T.world[(size_t)w * WC_STRIDE + tid];
  if (tid == 0) sBits = 0u;
  const bool has_cell = tid < nc;
  const int i = tid;
  const int gi = c0 + i;
  const long long C = T.C, E = T.E;

  double mc = 0.0, pctl = 0.0, log_drive_cap = 0.0;
  if (has_cell) {
    mc = control[L.c[CB_CONTROL_MEMBRANE] + gi];
    pctl = control[L.c[CB_CONTROL_PUMP] + gi];
    // log(capacity) + log(availability) of the pump's magnitude, constant over the launch.
    if (pctl > 0.0) log_drive_cap = __ldg(T.logpcap + gi) + log(pctl);
  }
  const double *jctl = control + L.c[CB_CONTROL_JUNCTION] + e0;
  const double *chctl = control + L.c[CB_CONTROL_CHANNEL] + gi;
  double res[3];
#pragma unroll
  for (int s = 0; s < 3; ++s) res[s] = state_in[L.s[CB_RESERVOIR_SUPPLIED] + s * (long long)T.W + w];
  double ec = state_in[L.s[CB_ELECTRODE_CHARGE] + w];
  double rw = state_in[L.s[CB_RESERVOIR_WORK] + w];
  double ew = state_in[L.s[CB_ELECTRODE_WORK] + w];
  __syncthreads();
  const double Vb = sW[WC_VB];

  // Bath plate charge of the charge-only increment (surface_tissue.capacitor_change): the sum
  // over the world's cells of -C_i dp_i with dp_i = q_i / C_i, i.e. -q_i.
  const double *cur = state_in;
  double plate0;
  {
    double v[1] = {0.0};
    if (has_cell) {
      const double *n = cur + L.s[CB_AMOUNT_INCREMENT] + gi;
      v[0] = -(kChargePerFmol * ((n[0] + n[C]) + (-n[2 * C])));
    }
    block_sum<BLOCK, 1>(v, sRed);
    plate0 = v[0];
  }

  // The start's channel kinetics (readouts at the start potentials), carried from step to step:
  // a step's final potential is the next step's start potential here (both Q/C + V_bath).
  bool k0_ok = true;
  if constexpr (NCH > 0) {
    if (has_cell) {
      const double *n = cur + L.s[CB_AMOUNT_INCREMENT] + gi;
      const double V = (__ldg(T.q0 + gi) + kChargePerFmol * ((n[0] + n[C]) + (-n[2 * C]))) *
                           __ldg(T.icap + gi) + Vb;
#pragma unroll
      for (int q = 0; q < NCH; ++q) {
        double t[2], tau[2];
        channel_kinetics<false>(__ldg(T.ch_code + q * C + gi), V - Vb, t, tau);
        k0_ok = k0_ok && channel_kinetics_ok(V - Vb, t, tau);
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          sK[(r * NCH + q) * BLOCK + i] = t[r];
          sK[((2 + r) * NCH + q) * BLOCK + i] = tau[r];
        }
      }
    }
  }

  int taken = 0;
  uint32_t refused = 0u;
  for (int step = 0; step < n_steps; ++step) {
    uint32_t bits = k0_ok ? 0u : CB_WORLD_CHANNEL_DOMAIN;
    // Stage 0 at the step's start: potential from the capacitor solve, Q / C plus the bath's.
    double n0[3] = {0.0, 0.0, 0.0}, g0[EPT];
    double icap = 1.0, q0 = 0.0;
    if (has_cell) {
#pragma unroll
      for (int s = 0; s < 3; ++s) n0[s] = cur[L.s[CB_AMOUNT_INCREMENT] + s * C + gi];
      icap = __ldg(T.icap + gi);
      q0 = __ldg(T.q0 + gi);
    }
#pragma unroll
    for (int q = 0; q < EPT; ++q) {
      const int e = tid + q * BLOCK;
      g0[q] = e < ne ? cur[L.s[CB_JUNCTION_GATE] + e0 + e] : 1.0;
    }
    const double V0 = (q0 + kChargePerFmol * ((n0[0] + n0[1]) + (-n0[2]))) * icap + Vb;
    constexpr int NQ = NCH > 0 ? NCH : 1;
    double chg0[2][NQ], chg1[2][NQ];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int q = 0; q < NQ; ++q)
        chg0[r][q] = (NCH > 0 && has_cell) ? cur[L.s[CB_CHANNEL_GATE] + (r * NCH + q) * C + gi]
                                           : 0.0;
    double n1[3], g1[EPT], in0[3], in1[3];
    stage<BLOCK, EPT, NCH, true, MIX>(T, L, sW, k, cur, c0, e0, ne, i, has_cell, n0, V0, g0, chg0, mc,
                                 pctl, log_drive_cap, jctl, chctl, sV, sC, sL, sJ, sA, sE, sH, n1,
                                 g1, in0, bits);
    // Stage 1 potential: the IMEX operator (capacitor only, no faces) solve. The operator is
    // diagonal on the cells, so Q/C leaves a charge residual within an ulp of Q and only a
    // non-finite potential exceeds 3e-25 C + 2e-12 |Q| (surface_imex.solve_operator).
    const double V1 = (q0 + kChargePerFmol * ((n1[0] + n1[1]) + (-n1[2]))) * icap + Vb;
    if (has_cell && !is_finite(V1)) bits |= CB_WORLD_RESIDUAL;
    // Stage-1 channel gates: the exponential update from the step start to the stage potential
    // (surface_pump_v3.stage_gates, :3061-3070; rows without a law keep their value).
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      chg1[0][q] = chg0[0][q];
      chg1[1][q] = chg0[1][q];
      if (NCH > 0 && has_cell) {
        const int code = __ldg(T.ch_code + q * C + gi);
        double t[2], tau[2];
        channel_kinetics<false>(code, V1 - Vb, t, tau);
        if (!channel_kinetics_ok(V1 - Vb, t, tau)) bits |= CB_WORLD_CHANNEL_DOMAIN;
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          if (r == 1 && code == kHhKn4) continue;
          chg1[r][q] = advance_gate<false>(chg0[r][q], sK[(r * NCH + q) * BLOCK + i],
                                    sK[((2 + r) * NCH + q) * BLOCK + i], t[r], tau[r], k.frac1_dt);
        }
      }
    }
    {
      double nd[3], gd[EPT];
      stage<BLOCK, EPT, NCH, false, MIX>(T, L, sW, k, cur, c0, e0, ne, i, has_cell, n1, V1, g1, chg1,
                                    mc, pctl, log_drive_cap, jctl, chctl, sV, sC, sL, sJ, sA, sE,
                                    sH, nd, gd, in1, bits);
    }
    // The new state's domain (surface_kinetic.domain_valid): positive amounts, finite ledgers,
    // gates in [minimum, 1].
    bool k2_ok = true;
    double k2t[2][NQ], k2tau[2][NQ];
    if (has_cell) {
      bool ok = true;
#pragma unroll
      for (int f = 0; f < 10; ++f) ok = ok && is_finite(sA[f * BLOCK + i]);
#pragma unroll
      for (int s = 0; s < 3; ++s) ok = ok && (__ldg(T.ref + s * C + gi) + sA[s * BLOCK + i]) > 0.0;
      const double q2 = q0 + kChargePerFmol * ((sA[i] + sA[BLOCK + i]) + (-sA[2 * BLOCK + i]));
      const double V2 = q2 * icap + Vb;
      if (!is_finite(V2)) bits |= CB_WORLD_RESIDUAL;
      // Final channel gates from the step start to the final potential; channel ledgers finite.
      if constexpr (NCH > 0) {
#pragma unroll
        for (int q = 0; q < NCH; ++q) {
          const int code = __ldg(T.ch_code + q * C + gi);
          double t[2], tau[2];
          channel_kinetics<false>(code, V2 - Vb, t, tau);
          k2_ok = k2_ok && channel_kinetics_ok(V2 - Vb, t, tau);
#pragma unroll
          for (int r = 0; r < 2; ++r) {
            k2t[r][q] = t[r];
            k2tau[r][q] = tau[r];
            double g = chg0[r][q];
            if (!(r == 1 && code == kHhKn4))
              g = advance_gate<false>(chg0[r][q], sK[(r * NCH + q) * BLOCK + i],
                               sK[((2 + r) * NCH + q) * BLOCK + i], t[r], tau[r], k.frac2_dt);
            sG[(r * NCH + q) * BLOCK + i] = g;
            ok = ok && is_finite(g) && g >= 0.0 && g <= 1.0;
          }
          ok = ok && is_finite(sH[q * BLOCK + i]) && is_finite(sH[(NCH + q) * BLOCK + i]);
        }
        if (!k2_ok) bits |= CB_WORLD_CHANNEL_DOMAIN;
      }
      if (!ok) bits |= CB_WORLD_DOMAIN;
    }
#pragma unroll
    for (int q = 0; q < EPT; ++q) {
      const int e = tid + q * BLOCK;
      if (e < ne) {
        bool ok = true;
#pragma unroll
        for (int f = 0; f < 5; ++f) ok = ok && is_finite(sE[f * EB + e]);
        const double g = sE[4 * EB + e];
        ok = ok && g >= __ldg(T.jmin + e0 + e) && g <= 1.0;
        if (!ok) bits |= CB_WORLD_DOMAIN;
      }
    }
    // World sums: the bath inflow of both stages and the end plate charge.
    double v[7] = {in0[0], in0[1], in0[2], in1[0], in1[1], in1[2], 0.0};
    if (has_cell)
      v[6] = -(kChargePerFmol * ((sA[i] + sA[BLOCK + i]) + (-sA[2 * BLOCK + i])));
    block_sum<BLOCK, 7>(v, sRed);
    double res2[3], applied[3];
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      const double k0r = -v[s], k1r = -v[3 + s];
      res2[s] = (res[s] + k.delta_dt * k0r) + k.omdelta_dt * k1r;
      applied[s] = k.delta * k0r + k.omdelta * k1r;
    }
    const double electrode = v[6] - plate0;
    const double ec2 = ec + electrode;
    const double rw2 =
        rw + 1e-3 * ((sW[WC_MUB] * (k.dt * applied[0]) + sW[WC_MUB + 1] * (k.dt * applied[1])) +
                     sW[WC_MUB + 2] * (k.dt * applied[2]));
    const double ew2 = ew + (1e12 * Vb) * electrode;
    if (!(is_finite(res2[0]) && is_finite(res2[1]) && is_finite(res2[2]) && is_finite(ec2) && is_finite(rw2) &&
          is_finite(ew2)))
      bits |= CB_WORLD_DOMAIN;
    // The step is accepted or refused for the whole world.
    if (bits) atomicOr(&sBits, bits);
    __syncthreads();
    const uint32_t world_bits = sBits;
    if (world_bits) {
      refused = world_bits;
      break;
    }
    // Commit the accepted state (each thread its own slots).
    if (has_cell) {
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        state_out[L.s[CB_AMOUNT_INCREMENT] + s * C + gi] = sA[s * BLOCK + i];
        state_out[L.s[CB_MEMBRANE_TRANSFERRED] + s * C + gi] = sA[(3 + s) * BLOCK + i];
      }
      state_out[L.s[CB_MEMBRANE_DISSIPATED] + gi] = sA[6 * BLOCK + i];
      state_out[L.s[CB_PUMP_CYCLES] + gi] = sA[7 * BLOCK + i];
      state_out[L.s[CB_PUMP_DISSIPATED] + gi] = sA[8 * BLOCK + i];
      state_out[L.s[CB_METABOLIC_WORK] + gi] = sA[9 * BLOCK + i];
      if constexpr (NCH > 0) {
#pragma unroll
        for (int q = 0; q < NCH; ++q) {
          state_out[L.s[CB_CHANNEL_TRANSFERRED] + q * C + gi] = sH[q * BLOCK + i];
          state_out[L.s[CB_CHANNEL_DISSIPATED] + q * C + gi] = sH[(NCH + q) * BLOCK + i];
#pragma unroll
          for (int r = 0; r < 2; ++r) {
            state_out[L.s[CB_CHANNEL_GATE] + (r * NCH + q) * C + gi] =
                sG[(r * NCH + q) * BLOCK + i];
            sK[(r * NCH + q) * BLOCK + i] = k2t[r][q];
            sK[((2 + r) * NCH + q) * BLOCK + i] = k2tau[r][q];
          }
        }
      }
    }
    k0_ok = k2_ok;
#pragma unroll
    for (int q = 0; q < EPT; ++q) {
      const int e = tid + q * BLOCK;
      if (e < ne) {
        const long long ge = e0 + e;
#pragma unroll
        for (int s = 0; s < 3; ++s)
          state_out[L.s[CB_JUNCTION_TRANSFERRED] + s * E + ge] = sE[s * EB + e];
        state_out[L.s[CB_JUNCTION_DISSIPATED] + ge] = sE[3 * EB + e];
        state_out[L.s[CB_JUNCTION_GATE] + ge] = sE[4 * EB + e];
      }
    }
#pragma unroll
    for (int s = 0; s < 3; ++s) res[s] = res2[s];
    ec = ec2;
    rw = rw2;
    ew = ew2;
    plate0 = v[6];
    ++taken;
    cur = state_out;
  }

  // A world refused at its first step keeps its input state.
  if (taken == 0 && state_in != state_out) {
    if (has_cell) {
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
    for (int q = 0; q < EPT; ++q) {
      const int e = tid + q * BLOCK;
      if (e < ne) {
        for (int f = CB_JUNCTION_TRANSFERRED; f <= CB_JUNCTION_GATE; ++f) {
          const int reps = (f == CB_JUNCTION_TRANSFERRED) ? 3 : 1;
          for (int s = 0; s < reps; ++s)
            state_out[L.s[f] + s * E + e0 + e] = state_in[L.s[f] + s * E + e0 + e];
        }
      }
    }
  }
  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < 3; ++s) state_out[L.s[CB_RESERVOIR_SUPPLIED] + s * (long long)T.W + w] = res[s];
    state_out[L.s[CB_ELECTRODE_CHARGE] + w] = ec;
    state_out[L.s[CB_RESERVOIR_WORK] + w] = rw;
    state_out[L.s[CB_ELECTRODE_WORK] + w] = ew;
    world_status[w] = refused;
    if (accepted_steps) accepted_steps[w] = taken;
  }
}

#include "packed_step.cuh"

// Ledger residuals per world (the reference's balances(), held-bath worlds): one 256-thread CTA
// per world, looping over its cells; junction transfers read through each cell's adjacency.
constexpr int kBalanceBlock = 256;

__global__ void __launch_bounds__(kBalanceBlock) balances_kernel(const Tissue T, const Layout L,
                                                                 const double *__restrict__ st,
                                                                 double *__restrict__ out) {
  __shared__ double sRed[(kBalanceBlock / 32) * 8];
  const int w = blockIdx.x, tid = threadIdx.x;
  const int c0 = T.cell_offset[w], nc = T.cell_offset[w + 1] - c0;
  const int e0 = T.edge_offset[w];
  const long long C = T.C, E = T.E;
  const int nch = T.nch;
  const double *wc = T.world + (size_t)w * WC_STRIDE;
  double local = 0.0, metabolic = 0.0;
  double v[7] = {0, 0, 0, 0, 0, 0, 0};  // moved[3], amounts[3], plate
  for (int cl = tid; cl < nc; cl += kBalanceBlock) {
    const long long gi = c0 + cl;
    const double stoich[3] = {-3.0, 2.0, 0.0};
    const double pc = st[L.s[CB_PUMP_CYCLES] + gi];
    double send[3] = {0, 0, 0}, recv[3] = {0, 0, 0};
    for (int a = T.adj_ptr[gi]; a < T.adj_ptr[gi + 1]; ++a) {
      const int code = T.adj_idx[a];
      const long long ge = e0 + (code >> 1);
      for (int s = 0; s < 3; ++s) {
        const double j = st[L.s[CB_JUNCTION_TRANSFERRED] + s * E + ge];
        if (code & 1) recv[s] += j;
        else send[s] += j;
      }
    }
    double n[3], moved[3];
    for (int s = 0; s < 3; ++s) {
      n[s] = st[L.s[CB_AMOUNT_INCREMENT] + s * C + gi];
      moved[s] = st[L.s[CB_MEMBRANE_TRANSFERRED] + s * C + gi];
    }
    for (int q = 0; q < nch; ++q) {  // channel_to_membrane
      const int sp = T.ch_species[q * C + gi];
      moved[sp] += st[L.s[CB_CHANNEL_TRANSFERRED] + q * C + gi];
    }
    for (int s = 0; s < 3; ++s) {
      const double total_m = moved[s] - stoich[s] * pc;
      local = fmax(local, fabs(((n[s] + total_m) + send[s]) - recv[s]));
      v[s] += total_m;
      v[3 + s] += n[s];
    }
    metabolic = fmax(metabolic, fabs(st[L.s[CB_METABOLIC_WORK] + gi] + 1e-3 * wc[WC_DRIVE] * pc));
    v[6] += -(kChargePerFmol * ((n[0] + n[1]) + (-n[2])));
  }
  block_sum<kBalanceBlock, 7>(v, sRed);
  double mx[2] = {local, metabolic};
  for (int q = 0; q < 2; ++q)
    for (int o = 16; o > 0; o >>= 1) mx[q] = fmax(mx[q], __shfl_xor_sync(0xffffffffu, mx[q], o));
  __syncthreads();
  if ((tid & 31) == 0) {
    sRed[(tid >> 5) * 8 + 0] = mx[0];
    sRed[(tid >> 5) * 8 + 1] = mx[1];
  }
  __syncthreads();
  if (tid == 0) {
    double ml = 0.0, mm = 0.0;
    for (int q = 0; q < kBalanceBlock / 32; ++q) {
      ml = fmax(ml, sRed[q * 8]);
      mm = fmax(mm, sRed[q * 8 + 1]);
    }
    double outside = 0.0, total = 0.0, sup[3];
    for (int s = 0; s < 3; ++s) {
      sup[s] = st[L.s[CB_RESERVOIR_SUPPLIED] + s * (long long)T.W + w];
      outside = fmax(outside, fabs(-v[s] - sup[s]));
      total = fmax(total, fabs(v[3 + s] - sup[s]));
    }
    const double ec = st[L.s[CB_ELECTRODE_CHARGE] + w];
    const double rw = st[L.s[CB_RESERVOIR_WORK] + w];
    const double ew = st[L.s[CB_ELECTRODE_WORK] + w];
    const double supply_charge = kChargePerFmol * ((sup[0] + sup[1]) - sup[2]);
    double *o = out + (size_t)w * 8;
    o[0] = ml;
    o[1] = outside;
    o[2] = total;
    o[3] = fabs(ec - v[6]);
    o[4] = fabs(ec + supply_charge);
    o[5] = fabs(rw - 1e-3 * ((wc[WC_MUB] * sup[0] + wc[WC_MUB + 1] * sup[1]) + wc[WC_MUB + 2] * sup[2]));
    o[6] = fabs(ew - 1e12 * wc[WC_VB] * ec);
    o[7] = mm;
  }
}

// numpy's logaddexp(0, y) on the host (libm), for the per-world pump constants.
double host_logaddexp0(double y) {
  if (y == 0.0) return 0.6931471805599453;
  const double tmp = -y;
  if (tmp > 0.0) return std::log1p(std::exp(-tmp));
  if (tmp <= 0.0) return y + std::log1p(std::exp(tmp));
  return tmp;
}

long long pad32(long long n) { return (n + 31) / 32 * 32; }

}  // namespace


namespace {

template <typename T>
int upload(cb_tissue *t, const std::vector<T> &host, const T **dst) {
  void *p = nullptr;
  size_t bytes = std::max<size_t>(host.size() * sizeof(T), 16);
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
  t->owned.push_back(p);
  if (!host.empty()) {
    e = cudaMemcpy(p, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy");
  }
  *dst = static_cast<const T *>(p);
  return CB_OK;
}

size_t step_smem(int block, int ept, int nch) {
  return sizeof(double) * step_smem_words(block, ept, nch);
}
constexpr size_t kMaxSmemPerBlock = 227 * 1024;
constexpr int kBlockMaxModes = 4;  // open_channel_block.MAX_MODES

template <int BLOCK, int EPT>
int launch_step(cb_tissue *t, const double *in, double *out, const double *control,
                const StepCoef &k, int n_steps, uint32_t *status, int32_t *taken,
                cudaStream_t stream, bool mix) {
  const int nch = t->t.nch;
  const size_t smem = step_smem(BLOCK, EPT, nch);
  // Resident CTAs per SM that the register budget targets: 128-thread CTAs at 2 (no spills),
  // 256-thread CTAs at 2 (no spills) or 3 (a few spilled words; worlds without channels), larger
  // CTAs at 1.
  constexpr int kMin = BLOCK <= 256 ? 2 : 1;
  auto kern = ars222_kernel<BLOCK, EPT, 0, kMin, false>;
  if (nch == 2) {
    kern = mix ? ars222_kernel<BLOCK, EPT, 2, kMin, true> : ars222_kernel<BLOCK, EPT, 2, kMin, false>;
  } else if (mix) {
    kern = ars222_kernel<BLOCK, EPT, 0, kMin, true>;
    if constexpr (BLOCK == 256) {
      if (t->occupancy == 3) kern = ars222_kernel<BLOCK, EPT, 0, 3, true>;
    }
  } else if constexpr (BLOCK == 256) {
    if (t->occupancy == 3) kern = ars222_kernel<BLOCK, EPT, 0, 3, false>;
  }
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
  const int grid = k.worlds > 0 ? k.worlds : t->W;
  kern<<<grid, BLOCK, smem, stream>>>(t->t, t->layout, in, out, control, k, n_steps, status,
                                      taken);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "ars222 launch");
  return CB_OK;
}

// The route prefactors A P / 1e-15 (selective_flux's conductance per mM, fmol/s) from
// permeabilities P on the device: cb_bind and cb_set_permeability both form them here, so a
// rebound handle steps bit for bit like a handle bound with the same permeabilities. In place
// (P read from the prefactor array itself) when pm/pj/pch alias T.ap/T.jap/T.ch_ap.
__global__ void set_permeability_kernel(const Tissue T, const double *__restrict__ area,
                                        const double *__restrict__ jarea, const double *pm,
                                        const double *pj, const double *pch) {
  const long long C = T.C, E = T.E, NQ = (long long)T.nch * C;
  const long long n = (pm ? 3 * C : 0) + (pj ? 3 * E : 0) + (pch ? NQ : 0);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    long long j = i;
    if (pm) {
      if (j < 3 * C) {
        const_cast<double *>(T.ap)[j] = area[j % C] * pm[j] / 1e-15;
        continue;
      }
      j -= 3 * C;
    }
    if (pj) {
      if (j < 3 * E) {
        const_cast<double *>(T.jap)[j] = jarea[j % E] * pj[j] / 1e-15;
        continue;
      }
      j -= 3 * E;
    }
    const_cast<double *>(T.ch_ap)[j] = area[j % C] * pch[j] / 1e-15;
  }
}

int launch_set_permeability(const cb_tissue *t, const double *pm, const double *pj,
                            const double *pch, cudaStream_t stream) {
  const long long n = 3LL * t->C + 3LL * t->E + (long long)t->t.nch * t->C;
  const int blocks = (int)std::min<long long>((n + 255) / 256, 148 * 8);
  set_permeability_kernel<<<blocks, 256, 0, stream>>>(t->t, t->area, t->jarea, pm,
                                                      t->E ? pj : nullptr, pch);
  cudaError_t ce = cudaGetLastError();
  if (ce != cudaSuccess) return cuda_fail(ce, "set_permeability launch");
  return CB_OK;
}

int launch_balances(cb_tissue *t, const double *st, double *out, cudaStream_t stream) {
  balances_kernel<<<t->W, kBalanceBlock, 0, stream>>>(t->t, t->layout, st, out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "balances launch");
  return CB_OK;
}

template <int BLOCK, int NCH, bool BLK = false, bool MIX = false>
int launch_packed_bn(cb_tissue *t, const double *in, double *out, const double *control,
                     const StepCoef &k, int n_steps, uint32_t *status, int32_t *taken,
                     cudaStream_t stream) {
  const size_t smem = packed_smem_bytes(t->pk.cap);
  auto kern = packed_kernel<BLOCK, NCH, BLK, MIX>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
  e = cudaMemsetAsync(t->pk.queue, 0, sizeof(unsigned int), stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
  kern<<<t->grid_ctas, BLOCK, smem, stream>>>(t->t, t->layout, t->pk, in, out, control, k,
                                              n_steps, status, taken);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "packed launch");
  return CB_OK;
}

int launch_packed(cb_tissue *t, const double *in, double *out, const double *control,
                  const StepCoef &k, int n_steps, uint32_t *status, int32_t *taken,
                  cudaStream_t stream, bool mix = false) {
  const int key = t->packed_block * 10 + t->t.nch + (t->t.blk_modes > 0 ? 100000 : 0) +
                  (mix ? 200000 : 0);
  switch (key) {
    case 202560: return launch_packed_bn<256, 0, false, true>(t, in, out, control, k, n_steps, status, taken, stream);
    case 202562: return launch_packed_bn<256, 2, false, true>(t, in, out, control, k, n_steps, status, taken, stream);
    case 205120: return launch_packed_bn<512, 0, false, true>(t, in, out, control, k, n_steps, status, taken, stream);
    case 205122: return launch_packed_bn<512, 2, false, true>(t, in, out, control, k, n_steps, status, taken, stream);
    case 210240: return launch_packed_bn<1024, 0, false, true>(t, in, out, control, k, n_steps, status, taken, stream);
    case 210242: return launch_packed_bn<1024, 2, false, true>(t, in, out, control, k, n_steps, status, taken, stream);
    case 102562: return launch_packed_bn<256, 2, true>(t, in, out, control, k, n_steps, status, taken, stream);
    case 105122: return launch_packed_bn<512, 2, true>(t, in, out, control, k, n_steps, status, taken, stream);
    case 110242: return launch_packed_bn<1024, 2, true>(t, in, out, control, k, n_steps, status, taken, stream);
    case 2560: return launch_packed_bn<256, 0>(t, in, out, control, k, n_steps, status, taken, stream);
    case 2562: return launch_packed_bn<256, 2>(t, in, out, control, k, n_steps, status, taken, stream);
    case 5120: return launch_packed_bn<512, 0>(t, in, out, control, k, n_steps, status, taken, stream);
    case 5122: return launch_packed_bn<512, 2>(t, in, out, control, k, n_steps, status, taken, stream);
    case 10240: return launch_packed_bn<1024, 0>(t, in, out, control, k, n_steps, status, taken, stream);
    case 10242: return launch_packed_bn<1024, 2>(t, in, out, control, k, n_steps, status, taken, stream);
    default: return fail(CB_ERR_UNSUPPORTED, "no packed kernel for this block size");
  }
}

#define CB_DISPATCH(FN, ...)                                                     \
  switch (t->block * 10 + t->ept) {                                              \
    case 1281: return FN<128, 1>(t, __VA_ARGS__);                                \
    case 1282: return FN<128, 2>(t, __VA_ARGS__);                                \
    case 1283: return FN<128, 3>(t, __VA_ARGS__);                                \
    case 1284: return FN<128, 4>(t, __VA_ARGS__);                                \
    case 2561: return FN<256, 1>(t, __VA_ARGS__);                                \
    case 2562: return FN<256, 2>(t, __VA_ARGS__);                                \
    case 2563: return FN<256, 3>(t, __VA_ARGS__);                                \
    case 2564: return FN<256, 4>(t, __VA_ARGS__);                                \
    case 5121: return FN<512, 1>(t, __VA_ARGS__);                                \
    case 5122: return FN<512, 2>(t, __VA_ARGS__);                                \
    case 5123: return FN<512, 3>(t, __VA_ARGS__);                                \
    case 5124: return FN<512, 4>(t, __VA_ARGS__);                                \
    case 10241: return FN<1024, 1>(t, __VA_ARGS__);                              \
    case 10242: return FN<1024, 2>(t, __VA_ARGS__);                              \
    case 10243: return FN<1024, 3>(t, __VA_ARGS__);                              \
    case 10244: return FN<1024, 4>(t, __VA_ARGS__);                              \
    default: return fail(CB_ERR_UNSUPPORTED, "no kernel for this block/edge shape"); \
  }

}  // namespace

namespace {

// The one-world-per-CTA step over the worlds k.world0 .. k.world0 + k.worlds - 1.
int launch_shared(cb_tissue *t, const double *in, double *out, const double *control,
                  const StepCoef &k, int n_steps, uint32_t *status, int32_t *taken,
                  cudaStream_t stream, bool mix) {
  CB_DISPATCH(launch_step, in, out, control, k, n_steps, status, taken, stream, mix);
}

// The host entry point's pipeline: the worlds in this many chunks, each on a stream of its own,
// so that one chunk's copies overlap another's steps.
constexpr int kHostChunks = 4;

// The state elements of worlds wa .. wb-1 between two packed states (one strided copy per
// field: a field's species or slot rows are C, E or W doubles apart).
int copy_world_range(const cb_tissue *t, const double *src, double *dst, int wa, int wb,
                     cudaMemcpyKind kind, cudaStream_t stream) {
  const long long C = t->C, E = t->E, W = t->W, nch = t->t.nch;
  const long long ca = t->h_cell_offset[wa], cb = t->h_cell_offset[wb];
  const long long ea = t->h_edge_offset[wa], eb = t->h_edge_offset[wb];
  struct Range {
    int field;
    long long reps, lo, n, pitch;
  };
  const Range ranges[CB_STATE_FIELDS] = {
      {CB_AMOUNT_INCREMENT, 3, ca, cb - ca, C},     {CB_MEMBRANE_TRANSFERRED, 3, ca, cb - ca, C},
      {CB_MEMBRANE_DISSIPATED, 1, ca, cb - ca, C},  {CB_PUMP_CYCLES, 1, ca, cb - ca, C},
      {CB_PUMP_DISSIPATED, 1, ca, cb - ca, C},      {CB_METABOLIC_WORK, 1, ca, cb - ca, C},
      {CB_JUNCTION_TRANSFERRED, 3, ea, eb - ea, E}, {CB_JUNCTION_DISSIPATED, 1, ea, eb - ea, E},
      {CB_JUNCTION_GATE, 1, ea, eb - ea, E},        {CB_RESERVOIR_SUPPLIED, 3, wa, wb - wa, W},
      {CB_ELECTRODE_CHARGE, 1, wa, wb - wa, W},     {CB_RESERVOIR_WORK, 1, wa, wb - wa, W},
      {CB_ELECTRODE_WORK, 1, wa, wb - wa, W},       {CB_CHANNEL_GATE, 2 * nch, ca, cb - ca, C},
      {CB_CHANNEL_TRANSFERRED, nch, ca, cb - ca, C}, {CB_CHANNEL_DISSIPATED, nch, ca, cb - ca, C}};
  for (const Range &r : ranges) {
    if (r.reps == 0 || r.n == 0) continue;
    const long long off = t->layout.s[r.field] + r.lo;
    const size_t pitch = sizeof(double) * (size_t)r.pitch;
    cudaError_t e = cudaMemcpy2DAsync(dst + off, pitch, src + off, pitch,
                                      sizeof(double) * (size_t)r.n, (size_t)r.reps, kind, stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy2DAsync (world range)");
  }
  return CB_OK;
}

// cb_step_host for the one-world-per-CTA kernel: chunk c's state goes to the device, takes its
// steps and comes back on stream c, so the copies of one chunk run beside the steps of the
// others. Every world's arithmetic is that of one launch over all worlds (one CTA per world).
int step_host_chunked(cb_tissue *t, int method, const double *state_in, double *state_out,
                      double dt, const double *control, int n_steps, uint32_t *world_status,
                      int32_t *accepted_steps) {
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(CB_ERR_ARGUMENT, "dt must be positive");
  if (n_steps < 0) return fail(CB_ERR_ARGUMENT, "n_steps must be non-negative");
  cudaError_t ce = cudaSuccess;
  if (!t->h_streams_ready) {
    int made = 0;
    for (; made < kHostChunks && ce == cudaSuccess; ++made)
      ce = cudaStreamCreateWithFlags(&t->h_streams[made], cudaStreamNonBlocking);
    if (ce != cudaSuccess) --made;  // the failed creation made nothing
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&t->h_event, cudaEventDisableTiming);
    if (ce != cudaSuccess) {  // release what was made, so a later call starts clean
      for (int c = 0; c < made; ++c) cudaStreamDestroy(t->h_streams[c]);
      return cuda_fail(ce, "stream creation");
    }
    t->h_streams_ready = true;
  }
  cudaStream_t *st = t->h_streams;
  int rc = CB_OK;
  ce = cudaMemcpyAsync(t->h_control, control, sizeof(double) * t->control_total,
                       cudaMemcpyHostToDevice, st[0]);
  if (ce == cudaSuccess) ce = cudaEventRecord(t->h_event, st[0]);
  for (int c = 1; c < kHostChunks && ce == cudaSuccess; ++c)
    ce = cudaStreamWaitEvent(st[c], t->h_event, 0);
  if (ce != cudaSuccess) rc = cuda_fail(ce, "control copy");
  StepCoef k = step_coef(dt);
  const bool mix = method == CB_METHOD_ARS222_MIXED;
  for (int c = 0; c < kHostChunks && rc == CB_OK; ++c) {
    const int wa = (int)((long long)t->W * c / kHostChunks);
    const int wb = (int)((long long)t->W * (c + 1) / kHostChunks);
    if (wb == wa) continue;
    rc = copy_world_range(t, state_in, t->h_state, wa, wb, cudaMemcpyHostToDevice, st[c]);
    k.world0 = wa;
    k.worlds = wb - wa;
    if (!rc)
      rc = launch_shared(t, t->h_state, t->h_state, t->h_control, k, n_steps, t->h_status,
                         t->h_taken, st[c], mix);
    if (!rc) rc = copy_world_range(t, t->h_state, state_out, wa, wb, cudaMemcpyDeviceToHost,
                                   st[c]);
    if (!rc) {
      ce = cudaMemcpyAsync(world_status + wa, t->h_status + wa, sizeof(uint32_t) * (wb - wa),
                           cudaMemcpyDeviceToHost, st[c]);
      if (ce == cudaSuccess && accepted_steps)
        ce = cudaMemcpyAsync(accepted_steps + wa, t->h_taken + wa, sizeof(int32_t) * (wb - wa),
                             cudaMemcpyDeviceToHost, st[c]);
      if (ce != cudaSuccess) rc = cuda_fail(ce, "status copy");
    }
  }
  // Every stream drains before the host buffers are handed back, also after an error.
  for (int c = 0; c < kHostChunks; ++c) {
    ce = cudaStreamSynchronize(st[c]);
    if (ce != cudaSuccess && rc == CB_OK) rc = cuda_fail(ce, "cudaStreamSynchronize");
  }
  return rc;
}

int alloc_packed_scratch(cb_tissue *t) {
  if (t->pk.sc) return CB_OK;
  void *sc = nullptr;
  cudaError_t e = cudaMalloc(&sc, t->scratch_bytes);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc scratch");
  t->owned.push_back(sc);
  t->pk.sc = static_cast<double *>(sc);
  return CB_OK;
}

}  // namespace

// cb_step_packed_static's array address on `device` (defined with the array below).
int static_scratch(int device, double **out, bool refresh);

extern "C" {

const char *cb_last_error(void) { return cbk::last_error(); }

int cb_set_launch(cb_tissue *t, int kernel, int block, int occupancy) {
  if (!t) return fail(CB_ERR_ARGUMENT, "null argument");
  if (kernel == CB_KERNEL_SHARED) {
    if (t->t.blk_modes > 0)
      return fail(CB_ERR_UNSUPPORTED, "a batch with an open-channel block runs on the packed "
                                      "kernel only");
    if (!t->shared_ok) return fail(CB_ERR_UNSUPPORTED, "the one-world-per-CTA kernel cannot hold "
                                                       "these worlds");
    if (occupancy != 2 && occupancy != 3) return fail(CB_ERR_ARGUMENT, "occupancy must be 2 or 3");
    t->packed = false;
    t->occupancy = occupancy;
    return CB_OK;
  }
  if (kernel == CB_KERNEL_PACKED) {
    if (!t->pk.order) return fail(CB_ERR_UNSUPPORTED, "worlds too large for the packed kernel");
    if (block != 256 && block != 512 && block != 1024)
      return fail(CB_ERR_ARGUMENT, "packed block must be 256, 512 or 1024");
    cudaError_t ce = cudaSetDevice(t->device);
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
    const int rc = alloc_packed_scratch(t);
    if (rc) return rc;
    t->packed = true;
    t->packed_block = block;
    return CB_OK;
  }
  return fail(CB_ERR_ARGUMENT, "kernel must be CB_KERNEL_SHARED or CB_KERNEL_PACKED");
}

int cb_get_launch(const cb_tissue *t, int *kernel, int *block, int *occupancy) {
  if (!t || !kernel || !block || !occupancy) return fail(CB_ERR_ARGUMENT, "null argument");
  *kernel = t->packed ? CB_KERNEL_PACKED : CB_KERNEL_SHARED;
  *block = t->packed ? t->packed_block : t->block;
  *occupancy = t->packed ? 1 : t->occupancy;
  return CB_OK;
}

const char *cb_version(void) { return "cells_b200 0.1 (sm_100a, fp64 ARS(2,2,2))"; }

int cb_bind(const cb_tissue_desc *d, int device, cb_tissue **out) {
  if (!d || !out) return fail(CB_ERR_ARGUMENT, "null argument");
  *out = nullptr;
  const int W = d->n_worlds;
  const long long C = d->n_cells, E = d->n_edges;
  if (W <= 0 || C <= 0 || E < 0 || C > (1LL << 30) || E > (1LL << 30))
    return fail(CB_ERR_LAYOUT, "world, cell or junction count out of range");
  if (!d->cell_offset || !d->edge_offset || !d->temperature || !d->bath_amount ||
      !d->bath_volume || !d->bath_potential || !d->pump || !d->volume || !d->area ||
      !d->capacitance || !d->permeability || !d->pump_capacity || !d->amount_reference ||
      !d->initial_charge || (E > 0 && (!d->sender || !d->receiver || !d->junction_area ||
                                       !d->junction_permeability || !d->gate_threshold ||
                                       !d->gate_minimum)))
    return fail(CB_ERR_ARGUMENT, "null array in the tissue description");
  if (d->cell_offset[0] != 0 || d->edge_offset[0] != 0 || d->cell_offset[W] != C ||
      d->edge_offset[W] != E)
    return fail(CB_ERR_LAYOUT, "offsets must run from 0 to the totals");
  int max_cells = 0;
  long long max_edges = 0;
  for (int w = 0; w < W; ++w) {
    const long long nc = d->cell_offset[w + 1] - d->cell_offset[w];
    const long long ne = d->edge_offset[w + 1] - d->edge_offset[w];
    if (nc < 1) return fail(CB_ERR_LAYOUT, "every world needs at least one cell");
    if (ne < 0) return fail(CB_ERR_LAYOUT, "junction offsets must not decrease");
    if (nc > 4096) return fail(CB_ERR_UNSUPPORTED, "worlds of more than 4096 cells");
    max_cells = std::max<int>(max_cells, (int)nc);
    max_edges = std::max(max_edges, ne);
  }
  int block = 128;
  while (block < max_cells) block *= 2;
  const int ept = (int)std::max<long long>(1, (max_edges + block - 1) / block);
  const int desc_nch = d->channel_slots;
  // Kernel path: one world per CTA in shared memory (uniform worlds of up to 1024 cells), or the
  // packed persistent kernel (uneven or large worlds, up to 4096 cells).
  bool min_eq_max = true;
  for (int w = 1; w < W; ++w)
    min_eq_max = min_eq_max && (d->cell_offset[w + 1] - d->cell_offset[w] ==
                                d->cell_offset[1] - d->cell_offset[0]);
  const bool shared_ok = block <= 1024 && ept <= 4 && desc_nch >= 0 && desc_nch <= 2 &&
                         step_smem(block, ept, desc_nch) <= kMaxSmemPerBlock;
  bool use_packed = !shared_ok || !(min_eq_max || max_cells <= 256);
  if (const char *env = std::getenv("CELLS_B200_KERNEL")) {
    if (!std::strcmp(env, "packed")) use_packed = true;
    if (!std::strcmp(env, "shared") && shared_ok) use_packed = false;
  }
  int cap = 1024;
  while (cap < max_cells) cap *= 2;
  if (use_packed && packed_smem_bytes(cap) > kMaxSmemPerBlock)
    return fail(CB_ERR_UNSUPPORTED, "world too large for the packed step");
  if (desc_nch != 0 && desc_nch != 2)
    return fail(CB_ERR_UNSUPPORTED, "channel slots per cell must be 0 or 2");
  if (desc_nch && (!d->channel_code || !d->channel_species || !d->channel_permeability ||
                   !d->channel_abundance))
    return fail(CB_ERR_ARGUMENT, "null channel array in the tissue description");

  for (long long q = 0; q < (long long)desc_nch * C; ++q) {
    const int code = d->channel_code[q], sp = d->channel_species[q];
    if (code != 0 && code != 2 && code != 100)
      return fail(CB_ERR_UNSUPPORTED, "channel law code must be 0, 2 or 100");
    if (sp < 0 || sp > 2) return fail(CB_ERR_LAYOUT, "channel species out of range");
    if (!(d->channel_permeability[q] >= 0) || !(d->channel_abundance[q] >= 0))
      return fail(CB_ERR_LAYOUT, "channel permeability and abundance must be non-negative");
  }
  // Adjacency (senders first, then receivers, each in edge order) and route checks.
  std::vector<int> adj_ptr(C + 1, 0), adj_idx;
  std::vector<std::vector<int>> out_e(C), in_e(C);
  for (int w = 0; w < W; ++w) {
    const long long c0 = d->cell_offset[w], nc = d->cell_offset[w + 1] - c0;
    for (long long e = d->edge_offset[w]; e < d->edge_offset[w + 1]; ++e) {
      const int s = d->sender[e], r = d->receiver[e];
      if (s < 0 || r < 0 || s >= nc || r >= nc || s == r)
        return fail(CB_ERR_LAYOUT, "junction endpoint out of its world or a self junction");
      const int local = (int)(e - d->edge_offset[w]);
      out_e[c0 + s].push_back(local << 1);
      in_e[c0 + r].push_back((local << 1) | 1);
    }
  }
  adj_idx.reserve(2 * E);
  for (long long c = 0; c < C; ++c) {
    for (int v : out_e[c]) adj_idx.push_back(v);
    for (int v : in_e[c]) adj_idx.push_back(v);
    adj_ptr[c + 1] = (int)adj_idx.size();
  }
  for (long long c = 0; c < C; ++c) {
    if (!(d->volume[c] > 0) || !(d->capacitance[c] > 0) || !(d->area[c] > 0) ||
        !std::isfinite(d->initial_charge[c]))
      return fail(CB_ERR_LAYOUT, "cell volume, area and capacitance must be positive");
  }
  // Per-world constants with the reference's expressions.
  const double ln1000 = std::log(1000.0);
  std::vector<double> world((size_t)W * WC_STRIDE, 0.0);
  for (int w = 0; w < W; ++w) {
    double *c = world.data() + (size_t)w * WC_STRIDE;
    const double T = d->temperature[w];
    const double RT = kR * T;
    const double vb = d->bath_potential[w], bv = d->bath_volume[w];
    if (!(bv > 0)) return fail(CB_ERR_LAYOUT, "bath volume must be positive");
    c[WC_T] = T;
    c[WC_RT] = RT;
    c[WC_VB] = vb;
    const double z[3] = {1.0, 1.0, -1.0};
    for (int s = 0; s < 3; ++s) {
      const double co = d->bath_amount[(size_t)s * W + w] / bv;
      if (!(co > 0) || !std::isfinite(co)) return fail(CB_ERR_LAYOUT, "bath must be positive");
      c[WC_CO + s] = co;
      c[WC_LOGCO + s] = std::log(co);
      c[WC_MUB + s] = RT * std::log(co) + z[s] * kF * vb;
    }
    const double atp = d->pump[0 * W + w], adp = d->pump[1 * W + w], pi = d->pump[2 * W + w];
    const double km_na = d->pump[3 * W + w], km_k = d->pump[4 * W + w];
    const double km_atp = d->pump[5 * W + w], dg0 = d->pump[6 * W + w];
    c[WC_DRIVE] = dg0 + RT * (((std::log(adp) + std::log(pi)) - std::log(atp)) - ln1000);
    c[WC_LK] = host_logaddexp0(2.0 * (std::log(km_k) - std::log(c[WC_CO + 1])));
    c[WC_LATP] = host_logaddexp0(std::log(km_atp) - std::log(atp));
    c[WC_LOGKMNA] = std::log(km_na);
    const bool t_ok = std::isfinite(T) && T >= 200.0 && T <= 400.0;
    const double rtd = kR * (t_ok ? T : 298.15);
    bool ok = t_ok;
    for (double v : {atp, adp, pi, km_na, km_k, km_atp}) ok = ok && std::isfinite(v) && v > 0;
    ok = ok && std::isfinite(dg0);
    const double s_atp = ok ? atp : 1.0, s_adp = ok ? adp : 1.0, s_pi = ok ? pi : 1.0;
    c[WC_AFF0] = (((dg0 / rtd + std::log(s_adp)) + std::log(s_pi)) - std::log(s_atp)) - ln1000;
    c[WC_RTDOM] = rtd;
    c[WC_PUMPOK] = ok ? 1.0 : 0.0;
    c[WC_FRT] = kF / RT;
    c[WC_INVRT] = 1.0 / RT;
    c[WC_INVRTD] = 1.0 / rtd;
    c[WC_SLOPE] = kF * kF / RT;
  }
  // Reciprocals. The route prefactors A P / 1e-15 are formed on the device once the
  // permeabilities are uploaded (set_permeability_kernel).
  std::vector<double> logpcap(C), ivol(C), icap(C);
  for (long long c = 0; c < C; ++c) {
    logpcap[c] = d->pump_capacity[c] > 0 ? std::log(d->pump_capacity[c]) : 0.0;
    ivol[c] = 1.0 / d->volume[c];
    icap[c] = 1.0 / d->capacitance[c];
  }

  cudaError_t ce = cudaSetDevice(device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
  if (int rc0 = static_scratch(device, nullptr, true)) return rc0;
  cb_tissue *t = new cb_tissue();
  t->device = device;
  t->W = W;
  t->C = (int)C;
  t->E = (int)E;
  t->block = block;
  t->ept = ept;
  t->packed = use_packed;
  if (const char *env = std::getenv("CELLS_B200_PACKED_BLOCK")) {
    const int b = std::atoi(env);
    if (b == 256 || b == 512 || b == 1024) t->packed_block = b;
  }
  if (const char *env = std::getenv("CELLS_B200_OCCUPANCY")) t->occupancy = std::atoi(env) == 2 ? 2 : 3;
  std::vector<int> co32(W + 1), eo32(W + 1), snd(E), rcv(E);
  for (int w = 0; w <= W; ++w) {
    co32[w] = (int)d->cell_offset[w];
    eo32[w] = (int)d->edge_offset[w];
  }
  for (long long e = 0; e < E; ++e) {
    snd[e] = d->sender[e];
    rcv[e] = d->receiver[e];
  }
  t->h_cell_offset.assign(d->cell_offset, d->cell_offset + W + 1);
  t->h_edge_offset.assign(d->edge_offset, d->edge_offset + W + 1);
  t->h_snd = snd;
  t->h_rcv = rcv;
  t->h_temperature.assign(d->temperature, d->temperature + W);
  auto vec = [](const double *p, long long n) { return std::vector<double>(p, p + n); };
  int rc = CB_OK;
  Tissue &T = t->t;
  T.W = W;
  T.C = (int)C;
  T.E = (int)E;
  if (!rc) rc = upload(t, co32, &T.cell_offset);
  if (!rc) rc = upload(t, eo32, &T.edge_offset);
  if (!rc) rc = upload(t, adj_ptr, &T.adj_ptr);
  if (!rc) rc = upload(t, adj_idx, &T.adj_idx);
  if (!rc) rc = upload(t, world, &T.world);
  if (!rc) rc = upload(t, ivol, &T.ivol);
  if (!rc) rc = upload(t, vec(d->amount_reference, 3 * C), &T.ref);
  if (!rc) rc = upload(t, vec(d->permeability, 3 * C), &T.ap);
  if (!rc) rc = upload(t, icap, &T.icap);
  if (!rc) rc = upload(t, vec(d->initial_charge, C), &T.q0);
  if (!rc) rc = upload(t, vec(d->pump_capacity, C), &T.pcap);
  if (!rc) rc = upload(t, logpcap, &T.logpcap);
  if (!rc) rc = upload(t, snd, &T.snd);
  if (!rc) rc = upload(t, rcv, &T.rcv);
  if (!rc) rc = upload(t, E ? vec(d->junction_permeability, 3 * E) : std::vector<double>(),
                       &T.jap);
  if (!rc) rc = upload(t, E ? vec(d->gate_threshold, E) : std::vector<double>(), &T.thr);
  if (!rc) rc = upload(t, E ? vec(d->gate_minimum, E) : std::vector<double>(), &T.jmin);
  if (!rc) rc = upload(t, vec(d->area, C), &t->area);
  if (!rc) rc = upload(t, E ? vec(d->junction_area, E) : std::vector<double>(), &t->jarea);
  T.nch = desc_nch;
  {
    const long long nq = (long long)desc_nch * C;
    std::vector<int> code(nq), species(nq);
    std::vector<double> chap(nq), chab(nq);
    for (long long q = 0; q < nq; ++q) {
      code[q] = d->channel_code[q];
      species[q] = d->channel_species[q];
      chap[q] = d->channel_permeability[q];
      chab[q] = d->channel_abundance[q];
    }
    if (!rc) rc = upload(t, code, &T.ch_code);
    if (!rc) rc = upload(t, species, &T.ch_species);
    if (!rc) rc = upload(t, chap, &T.ch_ap);
    if (!rc) rc = upload(t, chab, &T.ch_ab);
  }
  // A P / 1e-15 in place over the uploaded permeabilities.
  if (!rc) rc = launch_set_permeability(t, T.ap, T.jap, desc_nch ? T.ch_ap : nullptr, nullptr);
  if (!rc) {
    const cudaError_t se = cudaDeviceSynchronize();
    if (se != cudaSuccess) rc = cuda_fail(se, "permeability prefactors");
  }
  const bool packed_ok = packed_smem_bytes(cap) <= kMaxSmemPerBlock;
  t->shared_ok = shared_ok;
  if (!rc && packed_ok) {
    // Work items: runs of consecutive worlds of at most `target` cells (a larger world is an item
    // of its own, up to `cap`) and kPackedMaxWorlds worlds, queued largest first. The target sets
    // how many cells the running items hold at once, and so whether their scratch stays in L2.
    long long target = std::min<long long>(cap, 1024);  // measured best of 512..4096
    if (const char *env = std::getenv("CELLS_B200_ITEM_CELLS"))
      target = std::max(32LL, std::min<long long>(cap, std::atoll(env)));
    std::vector<int> item_world0{0}, cell_world(C), isnd(E), ircv(E), iadj(adj_idx.size());
    long long cells_in = 0;
    int worlds_in = 0;
    for (int w = 0; w < W; ++w) {
      const long long nc = d->cell_offset[w + 1] - d->cell_offset[w];
      if (worlds_in > 0 && (cells_in + nc > target || worlds_in == kPackedMaxWorlds)) {
        item_world0.push_back(w);
        cells_in = 0;
        worlds_in = 0;
      }
      cells_in += nc;
      ++worlds_in;
    }
    item_world0.push_back(W);
    const int n_items = (int)item_world0.size() - 1;
    std::vector<long long> item_cells(n_items);
    for (int it = 0; it < n_items; ++it) {
      const int a = item_world0[it], b = item_world0[it + 1];
      const long long ic0 = d->cell_offset[a], ie0 = d->edge_offset[a];
      item_cells[it] = d->cell_offset[b] - ic0;
      for (int w = a; w < b; ++w) {
        for (long long c = d->cell_offset[w]; c < d->cell_offset[w + 1]; ++c) {
          cell_world[c] = w - a;
          for (int q = adj_ptr[c]; q < adj_ptr[c + 1]; ++q) {
            const int code = adj_idx[q];
            const long long item_edge = d->edge_offset[w] + (code >> 1) - ie0;
            iadj[q] = (int)((item_edge << 1) | (code & 1));
          }
        }
        for (long long e = d->edge_offset[w]; e < d->edge_offset[w + 1]; ++e) {
          isnd[e] = (int)(d->cell_offset[w] - ic0 + d->sender[e]);
          ircv[e] = (int)(d->cell_offset[w] - ic0 + d->receiver[e]);
        }
      }
    }
    std::vector<int> order(n_items);
    for (int it = 0; it < n_items; ++it) order[it] = it;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return item_cells[a] > item_cells[b]; });
    Packed &P = t->pk;
    P.n_items = n_items;
    P.cap = cap;
    rc = upload(t, order, &P.order);
    if (!rc) rc = upload(t, item_world0, &P.item_world0);
    if (!rc) rc = upload(t, cell_world, &P.cell_world);
    if (!rc) rc = upload(t, isnd, &P.isnd);
    if (!rc) rc = upload(t, ircv, &P.ircv);
    if (!rc) rc = upload(t, iadj, &P.iadj);
    if (!rc) {
      void *q = nullptr;
      cudaError_t e = cudaMalloc(&q, sizeof(unsigned int));
      if (e != cudaSuccess) rc = cuda_fail(e, "cudaMalloc");
      else {
        t->owned.push_back(q);
        P.queue = static_cast<unsigned int *>(q);
      }
    }
    t->scratch_bytes = sizeof(double) * ((size_t)packed_cell_fields(desc_nch) * C +
                                         (size_t)SE_FIELDS * std::max<long long>(E, 1));
    if (!rc && use_packed) rc = alloc_packed_scratch(t);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    t->grid_ctas = std::max(1, std::min(sms, n_items));
  }
  if (rc) {
    cb_free(t);
    return rc;
  }
  // Packed state and control layouts: each field padded to 32 doubles (256-byte aligned).
  const long long nch = desc_nch;
  const long long sizes[CB_STATE_FIELDS] = {3 * C, 3 * C, C, C, C, C, 3 * E, E, E, 3 * (long long)W,
                                            W, W, W, 2 * nch * C, nch * C, nch * C};
  long long off = 0;
  for (int f = 0; f < CB_STATE_FIELDS; ++f) {
    t->layout.s[f] = off;
    off += pad32(sizes[f]);
  }
  t->state_total = off;
  const long long csz[CB_CONTROL_FIELDS] = {C, E, C, nch * C};
  off = 0;
  for (int f = 0; f < CB_CONTROL_FIELDS; ++f) {
    t->layout.c[f] = off;
    off += pad32(csz[f]);
  }
  t->control_total = off;
  *out = t;
  return CB_OK;
}

void cb_free(cb_tissue *t) {
  if (!t) return;
  cudaSetDevice(t->device);
  n2_release(t);
  for (void *p : t->owned) cudaFree(p);
  if (t->h_state) cudaFree(t->h_state);
  if (t->h_control) cudaFree(t->h_control);
  if (t->h_status) cudaFree(t->h_status);
  if (t->h_taken) cudaFree(t->h_taken);
  if (t->blk_buf) cudaFree(t->blk_buf);
  if (t->h_streams_ready) {
    for (cudaStream_t s : t->h_streams) cudaStreamDestroy(s);
    cudaEventDestroy(t->h_event);
  }
  delete t;
}

int cb_state_layout(const cb_tissue *t, int64_t offsets[CB_STATE_FIELDS], int64_t *total) {
  if (!t || !offsets || !total) return fail(CB_ERR_ARGUMENT, "null argument");
  for (int f = 0; f < CB_STATE_FIELDS; ++f) offsets[f] = t->layout.s[f];
  *total = t->state_total;
  return CB_OK;
}

int cb_control_layout(const cb_tissue *t, int64_t offsets[CB_CONTROL_FIELDS], int64_t *total) {
  if (!t || !offsets || !total) return fail(CB_ERR_ARGUMENT, "null argument");
  for (int f = 0; f < CB_CONTROL_FIELDS; ++f) offsets[f] = t->layout.c[f];
  *total = t->control_total;
  return CB_OK;
}

int cb_step(cb_tissue *t, int method, const double *state_in, double *state_out, double dt,
            const double *control, int n_steps, uint32_t *world_status, int32_t *accepted_steps,
            void *stream) {
  if (!t || !state_in || !state_out || !control || !world_status)
    return fail(CB_ERR_ARGUMENT, "null argument");
  if (t->t.blk_modes > 0 && method != CB_METHOD_ARS222)
    return fail(CB_ERR_UNSUPPORTED,
                method == CB_METHOD_N2 || method == CB_METHOD_N2_MIXED
                    ? "the implicit-conductance step (N2) refuses a blocked channel population: a "
                      "negative slope in its operator could make it indefinite"
                    : "a batch with an open-channel block takes the FP64 step (CB_METHOD_ARS222) "
                      "only");
  if (method == CB_METHOD_N2 || method == CB_METHOD_N2_MIXED) {
    if (!(dt > 0.0) || !std::isfinite(dt)) return fail(CB_ERR_ARGUMENT, "dt must be positive");
    if (n_steps < 0) return fail(CB_ERR_ARGUMENT, "n_steps must be non-negative");
    cudaError_t ce = cudaSetDevice(t->device);
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
    return n2_step(t, state_in, state_out, dt, control, n_steps, world_status, accepted_steps,
                   static_cast<cudaStream_t>(stream), method == CB_METHOD_N2_MIXED);
  }
  if (method == CB_METHOD_ROS2 || method == CB_METHOD_RK4 || method == CB_METHOD_ROS2_MIXED) {
    if (!(dt > 0.0) || !std::isfinite(dt)) return fail(CB_ERR_ARGUMENT, "dt must be positive");
    if (n_steps < 0) return fail(CB_ERR_ARGUMENT, "n_steps must be non-negative");
    cudaError_t ce = cudaSetDevice(t->device);
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
    return ros2_step(t, state_in, state_out, dt, control, n_steps, world_status, accepted_steps,
                     static_cast<cudaStream_t>(stream), method == CB_METHOD_RK4,
                     method == CB_METHOD_ROS2_MIXED);
  }
  if (method != CB_METHOD_ARS222 && method != CB_METHOD_ARS222_MIXED)
    return fail(CB_ERR_UNSUPPORTED, "unknown step method");
  const bool mix = method == CB_METHOD_ARS222_MIXED;
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(CB_ERR_ARGUMENT, "dt must be positive");
  if (n_steps < 0) return fail(CB_ERR_ARGUMENT, "n_steps must be non-negative");
  cudaError_t ce = cudaSetDevice(t->device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
  const StepCoef k = step_coef(dt);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (t->packed)
    return launch_packed(t, state_in, state_out, control, k, n_steps, world_status,
                         accepted_steps, s, mix);
  CB_DISPATCH(launch_step, state_in, state_out, control, k, n_steps, world_status,
              accepted_steps, s, mix);
}

int cb_step_host(cb_tissue *t, int method, const double *state_in, double *state_out, double dt,
                 const double *control, int n_steps, uint32_t *world_status,
                 int32_t *accepted_steps) {
  if (!t || !state_in || !state_out || !control || !world_status)
    return fail(CB_ERR_ARGUMENT, "null argument");
  cudaError_t ce = cudaSetDevice(t->device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
  if (!t->h_state) {
    ce = cudaMalloc(&t->h_state, sizeof(double) * t->state_total);
    if (ce == cudaSuccess) ce = cudaMalloc(&t->h_control, sizeof(double) * t->control_total);
    if (ce == cudaSuccess) ce = cudaMalloc(&t->h_status, sizeof(uint32_t) * t->W);
    if (ce == cudaSuccess) ce = cudaMalloc(&t->h_taken, sizeof(int32_t) * t->W);
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaMalloc");
  }
  if (!t->packed && (method == CB_METHOD_ARS222 || method == CB_METHOD_ARS222_MIXED) &&
      t->W >= 2 * kHostChunks)
    return step_host_chunked(t, method, state_in, state_out, dt, control, n_steps, world_status,
                             accepted_steps);
  ce = cudaMemcpy(t->h_state, state_in, sizeof(double) * t->state_total, cudaMemcpyHostToDevice);
  if (ce == cudaSuccess)
    ce = cudaMemcpy(t->h_control, control, sizeof(double) * t->control_total,
                    cudaMemcpyHostToDevice);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaMemcpy to device");
  int rc = cb_step(t, method, t->h_state, t->h_state, dt, t->h_control, n_steps, t->h_status,
                   t->h_taken, nullptr);
  if (rc) return rc;
  ce = cudaMemcpy(state_out, t->h_state, sizeof(double) * t->state_total, cudaMemcpyDeviceToHost);
  if (ce == cudaSuccess)
    ce = cudaMemcpy(world_status, t->h_status, sizeof(uint32_t) * t->W, cudaMemcpyDeviceToHost);
  if (ce == cudaSuccess && accepted_steps)
    ce = cudaMemcpy(accepted_steps, t->h_taken, sizeof(int32_t) * t->W, cudaMemcpyDeviceToHost);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaMemcpy to host");
  return CB_OK;
}

int cb_set_permeability(cb_tissue *t, const double *membrane, const double *junction,
                        const double *channel, void *stream) {
  if (!t) return fail(CB_ERR_ARGUMENT, "null argument");
  if (channel && t->t.nch == 0) return fail(CB_ERR_ARGUMENT, "the batch has no channel slots");
  if (!membrane && !(junction && t->E) && !channel) return CB_OK;
  cudaError_t ce = cudaSetDevice(t->device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
  return launch_set_permeability(t, membrane, junction, channel,
                                 static_cast<cudaStream_t>(stream));
}

int cb_set_channel_block(cb_tissue *t, int32_t modes, const double *weight,
                         const double *k0_mM, const double *steepness,
                         const double *concentration_mM) {
  if (!t) return fail(CB_ERR_ARGUMENT, "null argument");
  cudaError_t ce = cudaSetDevice(t->device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
  if (modes == 0) {
    t->t.blk_modes = 0;
    t->t.blk = nullptr;
    t->t.blk_conc = nullptr;
    return CB_OK;
  }
  if (modes < 0 || modes > kBlockMaxModes)
    return fail(CB_ERR_ARGUMENT, "block modes must be 0 (none) to 4");
  if (t->t.nch == 0) return fail(CB_ERR_ARGUMENT, "the batch has no channel slots");
  if (!weight || !k0_mM || !steepness || !concentration_mM)
    return fail(CB_ERR_ARGUMENT, "null block array");
  if (!t->pk.order)
    return fail(CB_ERR_UNSUPPORTED, "a blocked batch runs on the packed kernel, which cannot "
                                    "hold these worlds");
  const long long NC = (long long)t->t.nch * t->C;
  // The admitted domain (surface_pump_v3_spec.parse_block, _block_mode): weights in [0, 1]
  // summing to 1 within 8 ulps, K(0) in [1e-15, 1e15] mM, |steepness| <= 8, the blocker in
  // [0, 1e3] mM.
  for (long long q = 0; q < NC; ++q) {
    long double sum = 0.0L;
    for (int k = 0; k < modes; ++k) {
      const double w = weight[k * NC + q], k0 = k0_mM[k * NC + q], s = steepness[k * NC + q];
      if (!(w >= 0.0 && w <= 1.0))
        return fail(CB_ERR_LAYOUT, "block weights must lie in [0, 1]");
      if (!(k0 >= 1e-15 && k0 <= 1e15))
        return fail(CB_ERR_LAYOUT, "block K(0) must lie in [1e-15, 1e15] mM");
      if (!(std::fabs(s) <= 8.0)) return fail(CB_ERR_LAYOUT, "block steepness must be <= 8");
      sum += w;
    }
    if (!(std::fabs((double)(sum - 1.0L)) <= 8.0 * 2.220446049250313e-16))
      return fail(CB_ERR_LAYOUT, "each population's block weights must sum to 1");
    const double c = concentration_mM[q];
    if (!(c >= 0.0 && c <= 1e3))
      return fail(CB_ERR_LAYOUT, "blocker concentration must lie in [0, 1e3] mM");
  }
  // [3][M][NCH][C] (weight, K(0), a = steepness F/(R T) with the cell's world temperature),
  // then the concentrations [NCH][C].
  std::vector<double> host((size_t)(3 * modes + 1) * NC);
  for (int w = 0; w < t->W; ++w) {
    const double per_volt = kF / (kR * t->h_temperature[w]);
    for (long long c = t->h_cell_offset[w]; c < t->h_cell_offset[w + 1]; ++c)
      for (int q = 0; q < t->t.nch; ++q) {
        const long long at = (long long)q * t->C + c;
        for (int k = 0; k < modes; ++k) {
          host[(size_t)k * NC + at] = weight[k * NC + at];
          host[(size_t)(modes + k) * NC + at] = k0_mM[k * NC + at];
          host[(size_t)(2 * modes + k) * NC + at] = steepness[k * NC + at] * per_volt;
        }
        host[(size_t)3 * modes * NC + at] = concentration_mM[at];
      }
  }
  if (t->blk_doubles < host.size()) {
    if (t->blk_buf) cudaFree(t->blk_buf);
    t->blk_buf = nullptr;
    t->blk_doubles = 0;
    ce = cudaMalloc(&t->blk_buf, sizeof(double) * host.size());
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaMalloc block table");
    t->blk_doubles = host.size();
  }
  ce = cudaMemcpy(t->blk_buf, host.data(), sizeof(double) * host.size(), cudaMemcpyHostToDevice);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaMemcpy block table");
  if (!t->packed) {
    const int rc = alloc_packed_scratch(t);
    if (rc) return rc;
    t->packed = true;
  }
  t->t.blk_modes = modes;
  t->t.blk = t->blk_buf;
  t->t.blk_conc = t->blk_buf + (size_t)3 * modes * NC;
  return CB_OK;
}

int cb_balances(cb_tissue *t, const double *state, double *out, void *stream) {
  if (!t || !state || !out) return fail(CB_ERR_ARGUMENT, "null argument");
  cudaError_t ce = cudaSetDevice(t->device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  return launch_balances(t, state, out, s);
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// The packed step on library-held scratch (cb_step_packed_static).
//
// The packed kernel needs scratch beyond its inputs and outputs: stage accumulators, junction
// fluxes, world-sum terms and its work-queue ticket counter. cb_step takes that from memory the
// handle allocated at bind. This entry point takes it instead from one array that every process
// loading the library holds on each GPU it uses, so the call itself allocates nothing. The
// counter lives in the array's first 256 bytes and is cleared before every launch; the rest is
// written before it is read, so what a previous call left there does no harm. Two calls whose
// kernels overlap on a GPU (different streams, or different threads) share the array and race.

// 2^21 doubles = 16 MiB per GPU, held until the process exits.
constexpr size_t kStaticScratchDoubles = size_t(1) << 21;
constexpr size_t kStaticCounterDoubles = 32;  // 256 bytes: the ticket counter
static __device__ __align__(256) double g_static_scratch[kStaticScratchDoubles];

namespace {

constexpr int kStaticMaxDevices = 64;
double *g_static_ptr[kStaticMaxDevices] = {};
std::mutex g_static_mutex;

}  // namespace

// The device address of g_static_scratch on the current device (host code may not use the
// symbol itself: on the host it names a stand-in, not device memory). Looked up again at every
// bind on the device (refresh), so a context rebuilt after cudaDeviceReset, whose handles must
// be bound anew, never sees a stale address; otherwise once per device.
int static_scratch(int device, double **out, bool refresh) {
  if (device < 0 || device >= kStaticMaxDevices)
    return out ? fail(CB_ERR_UNSUPPORTED, "device ordinal beyond the static scratch table")
               : CB_OK;
  std::lock_guard<std::mutex> lock(g_static_mutex);
  if (refresh || !g_static_ptr[device]) {
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(static scratch)");
    g_static_ptr[device] = static_cast<double *>(ptr);
  }
  if (out) *out = g_static_ptr[device];
  return CB_OK;
}

namespace {

template <int BLOCK, int NCH, bool BLK = false>
int launch_packed_with(cb_tissue *t, const Packed &P, const double *in, double *out,
                       const double *control, const StepCoef &k, int n_steps, uint32_t *status,
                       int32_t *taken, cudaStream_t stream) {
  const size_t smem = packed_smem_bytes(P.cap);
  auto kern = packed_kernel<BLOCK, NCH, BLK>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
  e = cudaMemsetAsync(P.queue, 0, sizeof(unsigned int), stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
  kern<<<t->grid_ctas, BLOCK, smem, stream>>>(t->t, t->layout, P, in, out, control, k, n_steps,
                                              status, taken);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "packed launch (static scratch)");
  return CB_OK;
}

}  // namespace

extern "C" int cb_step_packed_static(cb_tissue *t, const double *state_in, double *state_out,
                                     double dt, const double *control, int n_steps,
                                     uint32_t *world_status, int32_t *accepted_steps,
                                     void *stream) {
  if (!t || !state_in || !state_out || !control || !world_status)
    return fail(CB_ERR_ARGUMENT, "null argument");
  if (!t->packed || !t->pk.order)
    return fail(CB_ERR_UNSUPPORTED,
                "the handle was not bound for the packed kernel (bind with CELLS_B200_KERNEL="
                "packed, or worlds that need it)");
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(CB_ERR_ARGUMENT, "dt must be positive");
  if (n_steps < 0) return fail(CB_ERR_ARGUMENT, "n_steps must be non-negative");
  const size_t need = (size_t)packed_cell_fields(t->t.nch) * (size_t)t->C +
                      (size_t)SE_FIELDS * (size_t)std::max(t->E, 1);
  if (need > kStaticScratchDoubles - kStaticCounterDoubles)
    return fail(CB_ERR_UNSUPPORTED,
                "batch needs " + std::to_string(need) + " scratch doubles; the static scratch "
                "holds " + std::to_string(kStaticScratchDoubles - kStaticCounterDoubles) +
                " (16 MiB): use cb_step");
  cudaError_t ce = cudaSetDevice(t->device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
  double *base = nullptr;
  int rc = static_scratch(t->device, &base, false);
  if (rc) return rc;
  Packed P = t->pk;
  P.queue = reinterpret_cast<unsigned int *>(base);
  P.sc = base + kStaticCounterDoubles;
  const StepCoef k = step_coef(dt);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  switch (t->packed_block * 10 + t->t.nch + (t->t.blk_modes > 0 ? 100000 : 0)) {
    case 102562: return launch_packed_with<256, 2, true>(t, P, state_in, state_out, control, k, n_steps, world_status, accepted_steps, s);
    case 105122: return launch_packed_with<512, 2, true>(t, P, state_in, state_out, control, k, n_steps, world_status, accepted_steps, s);
    case 110242: return launch_packed_with<1024, 2, true>(t, P, state_in, state_out, control, k, n_steps, world_status, accepted_steps, s);
    case 2560: return launch_packed_with<256, 0>(t, P, state_in, state_out, control, k, n_steps, world_status, accepted_steps, s);
    case 2562: return launch_packed_with<256, 2>(t, P, state_in, state_out, control, k, n_steps, world_status, accepted_steps, s);
    case 5120: return launch_packed_with<512, 0>(t, P, state_in, state_out, control, k, n_steps, world_status, accepted_steps, s);
    case 5122: return launch_packed_with<512, 2>(t, P, state_in, state_out, control, k, n_steps, world_status, accepted_steps, s);
    case 10240: return launch_packed_with<1024, 0>(t, P, state_in, state_out, control, k, n_steps, world_status, accepted_steps, s);
    case 10242: return launch_packed_with<1024, 2>(t, P, state_in, state_out, control, k, n_steps, world_status, accepted_steps, s);
    default: return fail(CB_ERR_UNSUPPORTED, "no packed kernel for this block size");
  }
}
