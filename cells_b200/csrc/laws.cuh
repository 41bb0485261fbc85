// laws.cuh - what the tissue step's kernels share: the reference's constants, the per-world
// constant table, the device views of a bound batch, the ARS(2,2,2) coefficients, and the point
// laws in device code (constant-field Bernoulli pair, logaddexp, channel kinetics, exponential
// gate update) with the fixed-order block sum.
//
// Arithmetic follows the reference expressions (Cells src/cells):
//   laws/electrochemistry.py:25-48           bernoulli, ghk route flux
//   laws/pumps/nak_atp_mass_action_positive.py:55-148  pump kinetics and domain
//   laws/junctions/junction_voltage_relaxation.py:43-97 gate rate and domain
//   laws/channels/kv1p5_mh.py:29-41, laws/channels/nav1p2_m3h_regularized.py:22-44
//   numerics/exponential_gates.py:36-51      exponential stage gates
//   numerics/surface_imex.py:47-69            the ARS(2,2,2) tableau
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <cmath>

#include "../../include/cells_b200.h"

namespace cbk {

// Constants of laws/electrochemistry.py:11-15, formed by the same products.
constexpr double kAvogadro = 6.02214076e23;
constexpr double kF = kAvogadro * 1.602176634e-19;
constexpr double kR = kAvogadro * 1.380649e-23;
constexpr double kChargePerFmol = kF * 1e-15;
constexpr double kNormalMin = 2.2250738585072014e-308;  // the smallest normal binary64
constexpr double kMaxAbsX = 50.0;
constexpr double kMaxAbsJunctionV = 0.120;
constexpr double kMaxAbsIonPotentialOverRT = 1600.0;
constexpr double kMaxAbsAffinityOverRT = 80.0;
constexpr double kLog0065 = -2.7333680090865;  // log(0.065), the gate law's closing constant

// Per-world constants (host-computed with the reference's expressions), stride in doubles.
enum WorldConst {
  WC_T = 0,
  WC_RT,
  WC_VB,
  WC_CO,      // 3: bath concentrations
  WC_LOGCO = WC_CO + 3,   // 3
  WC_DRIVE = WC_LOGCO + 3,
  WC_LK,      // logaddexp(0, 2 (log km_k - log k_o))
  WC_LATP,    // logaddexp(0, log km_atp - log atp)
  WC_LOGKMNA,
  WC_AFF0,    // dG0/rt + log adp + log pi - log atp - log 1000 (pump domain affinity)
  WC_RTDOM,   // rt of the pump domain predicate
  WC_PUMPOK,  // 1 when temperature and pump parameters lie in the law's domain
  WC_MUB,     // 3: bath mu (RT log co + z F Vb)
  WC_FRT = WC_MUB + 3,  // F / RT
  WC_INVRT,   // 1 / RT
  WC_INVRTD,  // 1 / rt of the pump domain predicate
  WC_SLOPE,   // F^2 / RT, the constant-field slope of the explicit-stability rate
  WC_STRIDE
};

struct Tissue {
  int W;
  int C;
  int E;
  const int *cell_offset;  // [W+1]
  const int *edge_offset;  // [W+1]
  const int *adj_ptr;      // [C+1], global cell -> adjacency entries
  const int *adj_idx;      // local edge index << 1 | (1 if the cell is the receiver)
  const double *world;     // [W * WC_STRIDE]
  const double *ivol;      // [C] 1 / volume
  const double *ref;       // [3][C]
  const double *ap;        // [3][C]  area * permeability / 1e-15 (fmol/s per mM)
  const double *icap;      // [C] 1 / capacitance
  const double *q0;        // [C]
  const double *pcap;      // [C]
  const double *logpcap;   // [C] log of the pump capacity where positive, else 0
  const int *snd;          // [E] local
  const int *rcv;          // [E] local
  const double *jap;       // [3][E]  junction area * permeability / 1e-15
  const double *thr;       // [E]
  const double *jmin;      // [E]
  int nch;                 // channel slots per cell (0 or 2)
  const int *ch_code;      // [NCH][C] law code
  const int *ch_species;   // [NCH][C] permeant species
  const double *ch_ap;     // [NCH][C] area * permeability / 1e-15
  const double *ch_ab;     // [NCH][C] abundance
  // Open-channel block of the populations (0 modes: none declared).
  int blk_modes;           // mode slots per population (1..4)
  const double *blk;       // [3][M][NCH][C]: weight, K(0) (mM), a = steepness F/(R T) (1/V)
  const double *blk_conc;  // [NCH][C] blocker concentration (mM)
};

struct Layout {  // offsets in doubles
  long long s[CB_STATE_FIELDS];
  long long c[CB_CONTROL_FIELDS];
};

struct StepCoef {
  double dt;
  double frac1_dt;      // the gates' stage-1 and final advance: sum of the tableau row times dt
  double frac2_dt;
  double gamma_dt;      // ARS(2,2,2) stage 1 weight times dt
  double delta_dt;      // final weights times dt
  double omdelta_dt;
  double delta;         // for the applied reservoir flux
  double omdelta;
  // The worlds of a launch of the one-world-per-CTA kernel: world0 .. world0 + worlds - 1
  // (worlds = 0: every world).
  int world0;
  int worlds;
};

template <typename R>
__device__ __forceinline__ void bernoulli_pair(R x, R &bp, R &bm) {
  // bp = B(x) = x/expm1(x), bm = B(-x), with the reference's series for |x| < 1e-4.
  const R ax = fabs(x);
  if (ax < R(1e-4)) {
    const R x2 = x * x;
    const R x4 = x2 * x2;
    bp = ((R(1) - x / R(2)) + x2 / R(12)) - x4 / R(720);
    bm = ((R(1) + x / R(2)) + x2 / R(12)) - x4 / R(720);
  } else {
    const R e = expm1(ax);
    const R small = ax / e;     // B(|x|), in (0, 1)
    const R large = ax + small; // B(-|x|) = |x| + B(|x|)
    bp = x >= R(0) ? small : large;
    bm = x >= R(0) ? large : small;
  }
}

// The mixed-precision pair: the series near x = 0 in FP64 (where the GHK term is a difference of
// nearly equal concentrations), the exponential form in FP32.
template <bool MIX>
__device__ __forceinline__ void bernoulli_pair_at(double x, double &bp, double &bm) {
  if (!MIX || fabs(x) < 1e-4) {
    bernoulli_pair<double>(x, bp, bm);
  } else {
    float fp, fm;
    bernoulli_pair<float>((float)x, fp, fm);
    bp = fp;
    bm = fm;
  }
}

// numpy's logaddexp(0, y).
template <typename R>
__device__ __forceinline__ R logaddexp0(R y) {
  if (y == R(0)) return R(0.6931471805599453);  // 0 + ln 2
  const R tmp = -y;
  if (tmp > R(0)) return log1p(exp(-tmp));
  if (tmp <= R(0)) return y + log1p(exp(tmp));
  return tmp;  // NaN
}

__device__ __forceinline__ bool is_finite(double v) { return isfinite(v); }

// B(x) alone (laws/electrochemistry.py:25-32).
template <typename R>
__device__ __forceinline__ R bernoulli(R x) {
  if (fabs(x) < R(1e-4)) {
    const R x2 = x * x;
    return ((R(1) - x / R(2)) + x2 / R(12)) - (x2 * x2) / R(720);
  }
  return x / expm1(x);
}

// Voltage-gated channel laws: gate targets t[2] and time constants tau[2] (s) at membrane
// voltage v (V). Codes: 0 Kv1.5 (laws/channels/kv1p5_mh.py:29-41), 2 NaV1.2
// (laws/channels/nav1p2_m3h_regularized.py:22-44), 100 Hodgkin-Huxley K n (Hodgkin and Huxley
// 1952: alpha_n = 0.01 (Vm+55)/(1 - exp(-(Vm+55)/10)), beta_n = 0.125 exp(-(Vm+65)/80) per ms,
// Vm in mV, alpha_n = 0.1 B(-(Vm+55)/10); one gate, row 1 unused).
constexpr int kKv1p5 = 0, kNav1p2 = 2, kHhKn4 = 100;

template <typename R>
__device__ __forceinline__ R kv_sigmoid(R value) {
  const R e = exp(-fabs(value));
  return value >= R(0) ? R(1) / (R(1) + e) : e / (R(1) + e);
}

template <typename R>
__device__ __forceinline__ void channel_kinetics_r(int code, R v, R (&t)[2], R (&tau)[2]) {
  if (code == kNav1p2) {
    const R shifted = (v + R(0.025)) / R(0.009);
    R bp, bm;
    bernoulli_pair<R>(shifted, bp, bm);
    const R activation = R(0.182 * 9) * bm;
    const R deactivation = R(0.124 * 9) * bp;
    const R recovery = R(0.024 * 5) * bernoulli<R>(-(v + R(0.040)) / R(0.005));
    const R inactivation = R(0.0091 * 5) * bernoulli<R>((v + R(0.065000123)) / R(0.005));
    t[0] = activation / (activation + deactivation);
    t[1] = R(1) / (R(1) + exp((v + R(0.055)) / R(0.0062)));
    tau[0] = R(0.001) / (activation + deactivation);
    tau[1] = R(0.001) / (recovery + inactivation);
  } else if (code == kHhKn4) {
    const R vm = R(1000) * v;
    const R alpha = R(100) * bernoulli<R>(-(vm + R(55)) / R(10));
    const R beta = R(125) * exp(-(vm + R(65)) / R(80));
    t[0] = alpha / (alpha + beta);
    t[1] = R(0);
    tau[0] = R(1) / (alpha + beta);
    tau[1] = R(1);
  } else {  // Kv1.5
    t[0] = kv_sigmoid<R>((v + R(0.0060)) / R(0.0064));
    t[1] = kv_sigmoid<R>(-(v + R(0.0253)) / R(0.0035));
    tau[0] = R(0.008330) - R(0.1163) * v;
    tau[1] = R(1.620000) - R(15.500) * v;
  }
}

// The kinetics in FP64, or in FP32 for the mixed-precision step, returned in FP64.
template <bool MIX = false>
__device__ __forceinline__ void channel_kinetics(int code, double v, double (&t)[2],
                                                 double (&tau)[2]) {
  if constexpr (MIX) {
    float tf[2], tauf[2];
    channel_kinetics_r<float>(code, (float)v, tf, tauf);
    t[0] = tf[0];
    t[1] = tf[1];
    tau[0] = tauf[0];
    tau[1] = tauf[1];
  } else {
    channel_kinetics_r<double>(code, v, t, tau);
  }
}

// channel_domain_valid (surface_pump_v3.py:848-858): the -120..60 mV domain, finite kinetics.
__device__ __forceinline__ bool channel_kinetics_ok(double v, const double (&t)[2],
                                                    const double (&tau)[2]) {
  bool ok = v >= -0.120 && v <= 0.060;
#pragma unroll
  for (int r = 0; r < 2; ++r)
    ok = ok && is_finite(t[r]) && t[r] >= 0.0 && t[r] <= 1.0 && is_finite(tau[r]) && tau[r] > 0.0;
  return ok;
}

__device__ __forceinline__ double channel_opening(int code, double m, double h) {
  if (code == kNav1p2) return ((m * m) * m) * h;
  if (code == kHhKn4) return (m * m) * (m * m);
  return m * h;
}

// The open-channel block of population q of cell gi at the patch voltage v
// (laws/channels/open_channel_block.py, the reference's kernels dissociation, fractions,
// unblocked_fraction, slope and domain_valid): K_k = K_k(0) exp(a_k v); both fractions formed
// directly, theta_k = c_B / (c_B + K_k), 1 - theta_k = K_k / (c_B + K_k); the unblocked fraction
// u = (sum_k w_k (1 - theta_k)) / sum_k w_k and u's slope bound
// (sum_k w_k |a_k| theta_k (1 - theta_k)) / sum_k w_k, each sum left to right over the modes.
// ok turns false where a K_k or c_B + K_k is not a finite normal number.
__device__ __forceinline__ void channel_block(const Tissue &T, int q, long long gi, double v,
                                              double &u, double &slope, bool &ok) {
  const int M = T.blk_modes;
  const long long NC = (long long)T.nch * T.C, at = (long long)q * T.C + gi;
  const double cb = __ldg(T.blk_conc + at);
  double num = 0.0, den = 0.0, snum = 0.0;
  for (int k = 0; k < M; ++k) {
    const double w = __ldg(T.blk + (long long)k * NC + at);
    const double k0 = __ldg(T.blk + (long long)(M + k) * NC + at);
    const double a = __ldg(T.blk + (long long)(2 * M + k) * NC + at);
    const double K = k0 * exp(a * v);
    const double total = cb + K;
    const double theta = cb / total, free = K / total;
    ok = ok && is_finite(K) && K >= kNormalMin && is_finite(total) && total >= kNormalMin;
    const double wf = w * free, ws = (w * fabs(a)) * (theta * free);
    num = k == 0 ? wf : num + wf;
    den = k == 0 ? w : den + w;
    snum = k == 0 ? ws : snum + ws;
  }
  u = num / den;
  slope = snum / den;
}

// Exponential gate update with a linearly varying target (numerics/exponential_gates.py:36-51).
template <typename R>
__device__ __forceinline__ R advance_gate_r(R g, R ts, R taus, R te, R taue, R h) {
  const R z = R(0.5) * h * (R(1) / taus + R(1) / taue);
  const R em = expm1(-z);
  const R lag = z < R(1e-3) ? z * (R(0.5) - z * (R(1.0 / 6.0) - z * (R(1.0 / 24.0) - z / R(120))))
                            : (em + z) / z;
  return g + (ts - g) * (-em) + (te - ts) * lag;
}

template <bool MIX = false>
__device__ __forceinline__ double advance_gate(double g, double ts, double taus, double te,
                                               double taue, double h) {
  if constexpr (MIX)
    return advance_gate_r<float>((float)g, (float)ts, (float)taus, (float)te, (float)taue,
                                 (float)h);
  else
    return advance_gate_r<double>(g, ts, taus, te, taue, h);
}

// Block-wide sum of NV values per thread, fixed tree order: xor-shuffle within warps, then the
// warp partials in warp order. Every thread receives the totals.
template <int BLOCK, int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *red) {
  constexpr int WARPS = BLOCK / 32;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();  // red may still be read from a previous reduction
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) red[warp * NV + k] = v[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double s = red[k];
    for (int q = 1; q < WARPS; ++q) s += red[q * NV + k];
    v[k] = s;
  }
}

// The ARS(2,2,2) coefficients of one step of size dt (numerics/surface_imex.py:47-48, :63-66).
inline StepCoef step_coef(double dt) {
  const double gamma = 1.0 - 1.0 / std::sqrt(2.0);
  const double delta = 1.0 - 1.0 / (2.0 * gamma);
  StepCoef k;
  k.dt = dt;
  k.gamma_dt = gamma * dt;
  k.delta_dt = delta * dt;
  k.omdelta_dt = (1.0 - delta) * dt;
  k.delta = delta;
  k.omdelta = 1.0 - delta;
  // The gates' advance fractions: each tableau row's sum, in numpy's order (gamma + 0 + 0 and
  // (delta + (1 - delta)) + 0), times dt (surface_pump_v3.py:3700, entity_sum).
  k.frac1_dt = ((gamma + 0.0) + 0.0) * dt;
  k.frac2_dt = ((delta + (1.0 - delta)) + 0.0) * dt;
  k.world0 = 0;
  k.worlds = 0;
  return k;
}

// B'(x) and B'(-x) from one expm1 of -|x|:
//   x > 0: B'(x) = -(1 + em)(x + em) / em^2,  x < 0: B'(x) = (em + |x| (1 + em)) / em^2,
// em = expm1(-|x|); below |x| < 1e-2 the series -1/2 + x/6 - x^3/180 + x^5/5040 - x^7/151200.
__device__ __forceinline__ void bernoulli_slope_pair(double x, double &sp, double &sm) {
  const double ax = fabs(x);
  if (ax < 1e-2) {
    const double x2 = x * x;
    const double even = -0.5;
    const double odd = x * (1.0 / 6.0 + x2 * (-1.0 / 180.0 + x2 * (1.0 / 5040.0 - x2 / 151200.0)));
    sp = even + odd;
    sm = even - odd;
    return;
  }
  const double em = expm1(-ax);
  const double d = em * em;
  const double at_pos = -(1.0 + em) * (ax + em) / d;  // B'(|x|)
  const double at_neg = (em + ax * (1.0 + em)) / d;   // B'(-|x|)
  sp = x > 0.0 ? at_pos : at_neg;
  sm = x > 0.0 ? at_neg : at_pos;
}

__device__ __forceinline__ double bernoulli_slope(double x) {
  double sp, sm;
  bernoulli_slope_pair(x, sp, sm);
  return sp;
}

__device__ __forceinline__ double sigmoid(double u) {
  const double e = exp(-fabs(u));
  return u >= 0.0 ? 1.0 / (1.0 + e) : e / (1.0 + e);
}

// Voltage derivatives of a channel law's targets dt[2] and time constants dtau[2] at v.
__device__ inline void channel_slope(int code, double v, double (&dt)[2], double (&dtau)[2]) {
  if (code == kNav1p2) {
    const double sh = (v + 0.025) / 0.009;
    double bp, bm;
    bernoulli_pair<double>(sh, bp, bm);
    double sp, sm;
    bernoulli_slope_pair(sh, sp, sm);
    const double act = (0.182 * 9) * bm, dact = -(0.182 * 9) * sm / 0.009;
    const double deact = (0.124 * 9) * bp, ddeact = (0.124 * 9) * sp / 0.009;
    const double ur = -(v + 0.040) / 0.005, ui = (v + 0.065000123) / 0.005;
    const double rec = (0.024 * 5) * bernoulli<double>(ur);
    const double drec = -(0.024 * 5) * bernoulli_slope(ur) / 0.005;
    const double ina = (0.0091 * 5) * bernoulli<double>(ui);
    const double dina = (0.0091 * 5) * bernoulli_slope(ui) / 0.005;
    const double s = act + deact, ds = dact + ddeact;
    const double t1 = 1.0 / (1.0 + exp((v + 0.055) / 0.0062));
    const double q = rec + ina, dq = drec + dina;
    dt[0] = (dact * s - act * ds) / (s * s);
    dt[1] = -t1 * (1.0 - t1) / 0.0062;
    dtau[0] = -0.001 * ds / (s * s);
    dtau[1] = -0.001 * dq / (q * q);
  } else if (code == kHhKn4) {
    const double ua = -(1000.0 * v + 55.0) / 10.0;
    const double alpha = 100.0 * bernoulli<double>(ua);
    const double dalpha = -100.0 * 100.0 * bernoulli_slope(ua);
    const double beta = 125.0 * exp(-(1000.0 * v + 65.0) / 80.0);
    const double dbeta = -12.5 * beta;
    const double s = alpha + beta, ds = dalpha + dbeta;
    dt[0] = (dalpha * beta - alpha * dbeta) / (s * s);
    dt[1] = 0.0;
    dtau[0] = -ds / (s * s);
    dtau[1] = 0.0;
  } else {  // Kv1.5
    const double s0 = sigmoid((v + 0.0060) / 0.0064), s1 = sigmoid(-(v + 0.0253) / 0.0035);
    dt[0] = s0 * (1.0 - s0) / 0.0064;
    dt[1] = -s1 * (1.0 - s1) / 0.0035;
    dtau[0] = -0.1163;
    dtau[1] = -15.5;
  }
}

}  // namespace cbk
