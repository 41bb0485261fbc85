// device_checks.cu - the accepted-row checks on the device (cb_device_checks).
//
// The reference decides a compiled window's refusals on the device: for each accepted row it
// evaluates models/surface_pump_checks.row_checks (:101-192), as @3's device_checks calls it
// (models/surface_pump_v3.py:5572-5597): the state's domain; ten ledgers (surface_pump.LEDGERS:
// local, outside and total material, capacitor, electrode and global charge, energy, reservoir,
// electrode and metabolic work), each against its bound plus a rounding allowance of
// 2.5 eps x accepted steps x the magnitudes rounded into it (ledger_limits :752-800,
// ledger_magnitudes :705-738, @3's channel_magnitudes :5243-5258); and dissipation that is
// negative or decreases since the previous row. This kernel evaluates them per world for
// held-bath worlds (each cell's capacitor component holds its world's bath: no representative
// rows, every cell grounded through the bath), one CTA per world, the world sums in fixed-order
// block reductions, and returns a bitmask (bit k: DEVICE_CHECKS[k] failed) and the twelve
// DEVICE_DIAGNOSTICS per world.

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <cfloat>
#include <string>

#include "handle.h"

namespace {

using namespace cbk;

constexpr int kChecksBlock = 256;
constexpr int kChecksMinBlocks = 4;  // resident CTAs per SM the registers target (64 each)
constexpr int kFailureShift = 1;  // vector_windows.FAILURE_SHIFT: bit 0 is the refused step
constexpr double kEps = DBL_EPSILON;
constexpr double kLedgerStepRounding = 2.5;     // surface_pump.LEDGER_STEP_ROUNDING
constexpr double kComponentStepRounding = 2.5;  // surface_field.COMPONENT_STEP_ROUNDING
constexpr double kGlobalChargeAtol = 3e-25;     // surface_pump.GLOBAL_CHARGE_ATOL_C
constexpr double kGlobalChargeRounding = 256 * kEps;
constexpr double kEnergyAtol = 2e-8;            // surface_tissue.ENERGY_ATOL_PJ
constexpr double kWorkBound = 3e-12;            // ledger_limits' fixed work bounds
constexpr double kDissipationAtol = 1e-12;      // surface_pump_checks.DISSIPATION_ATOL_PJ
constexpr double kChargeAtol = 3e-25;           // surface_field.CHARGE_ATOL_C
constexpr double kChargeRtol = 2e-12;           // surface_field.CHARGE_RTOL

enum Check {
  K_DOMAIN = 0, K_LOCAL, K_OUTSIDE, K_TOTAL, K_CHARGE, K_ELECTRODE, K_GLOBAL, K_ENERGY,
  K_RESERVOIR_WORK, K_ELECTRODE_WORK, K_METABOLIC, K_DISSIPATION
};

struct CheckArgs {
  double tol[3];   // material tolerance per species (fmol)
  double rtol;     // the solver's energy tolerance
  double rounding; // 2.5 eps x accepted steps
  double grounding;  // 2.5 eps x accepted steps (the grounded components' rule)
  const int64_t *steps;  // per-world accepted steps (device [W]), or null: rounding/grounding
  int64_t step_offset;   // added to steps[w]
};

// A vector window's per-world bookkeeping of one row (cb_window_row), or row < 0 for none.
struct WindowRow {
  int row;                        // 0: the start row; j > 0: the state after slot j
  const uint32_t *step_status;    // [W] the row's step status (row > 0)
  const int64_t *counts;          // [W] rows each world takes
  int32_t *ok;                    // [W] in/out: no failure so far
  int32_t *first;                 // [W] out: first failing row, -1 if none
  int64_t *bits;                  // [W] out: its failure bits
  double *maxima;                 // [W*12] out: diagnostic maxima over accepted rows
  int32_t *keep;                  // [W] out: 1 where the world stays at its current state
};

template <int BLOCK>
__device__ __forceinline__ double block_max(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double m = red[0];
  for (int q = 1; q < BLOCK / 32; ++q) m = fmax(m, red[q]);
  return m;
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, kChecksMinBlocks)
    checks_kernel(const Tissue T, const Layout L, const double *__restrict__ prev,
                  const double *__restrict__ row, const CheckArgs A, const WindowRow R,
                  uint32_t *__restrict__ failed_out, double *__restrict__ values_out) {
  __shared__ double sRed[(BLOCK / 32) * 16];
  __shared__ unsigned int sFail;
  const int w = blockIdx.x, tid = threadIdx.x;
  const int c0 = T.cell_offset[w], nc = T.cell_offset[w + 1] - c0;
  const int e0 = T.edge_offset[w], ne = T.edge_offset[w + 1] - e0;
  const long long C = T.C, E = T.E, W = T.W;
  const int nch = T.nch;
  const double *wc = T.world + (size_t)w * WC_STRIDE;
  // The step-scaled rounding allowances: the call's, or this world's own step count.
  const double rounding =
      A.steps ? kLedgerStepRounding * kEps * (double)(A.steps[w] + A.step_offset) : A.rounding;
  const double grounding =
      A.steps ? kComponentStepRounding * kEps * (double)(A.steps[w] + A.step_offset)
              : A.grounding;
  if (tid == 0) sFail = 0u;
  __syncthreads();
  uint32_t fail = 0;
  auto bad = [&](double value, double limit) { return !is_finite(value) || fabs(value) > limit; };
  const double stoich[3] = {-3.0, 2.0, 0.0};
  const double z[3] = {1.0, 1.0, -1.0};
  const double Vb = wc[WC_VB], temp = wc[WC_T];
  // Per-thread partials: maxima of |local|, |charge|, |metabolic|; world sums.
  double m_local = 0.0, m_charge = 0.0, m_metab = 0.0;
  double s[16];  // moved[3], amounts[3], |moved|[3], |amounts|[3], plate, increments, energy,
                 // flows
  for (int k = 0; k < 16; ++k) s[k] = 0.0;
  const long long oN = L.s[CB_AMOUNT_INCREMENT], oMT = L.s[CB_MEMBRANE_TRANSFERRED];
  for (int i = tid; i < nc; i += BLOCK) {
    const long long gi = c0 + i;
    double n[3], moved[3], absmoved[3];
    const double pc = row[L.s[CB_PUMP_CYCLES] + gi];
    for (int sp = 0; sp < 3; ++sp) {
      n[sp] = row[oN + sp * C + gi];
      moved[sp] = row[oMT + sp * C + gi];
      absmoved[sp] = fabs(moved[sp]) + fabs(stoich[sp] * pc);
    }
    // Domain: finite fields, positive amounts, zero transfer where nothing is permeable.
    bool ok = true;
    for (int sp = 0; sp < 3; ++sp) {
      ok = ok && is_finite(n[sp]) && is_finite(moved[sp]) &&
           (__ldg(T.ref + sp * C + gi) + n[sp]) > 0.0;
      if (__ldg(T.ap + sp * C + gi) == 0.0 && moved[sp] != 0.0) ok = false;
    }
    for (int f : {CB_MEMBRANE_DISSIPATED, CB_PUMP_CYCLES, CB_PUMP_DISSIPATED, CB_METABOLIC_WORK})
      ok = ok && is_finite(row[L.s[f] + gi]);
    if (!(__ldg(T.pcap + gi) > 0.0) && pc != 0.0) ok = false;
    double chd_sum = 0.0, chd_abs = 0.0;
    for (int q = 0; q < nch; ++q) {
      const int sp = __ldg(T.ch_species + q * C + gi);
      const double tr = row[L.s[CB_CHANNEL_TRANSFERRED] + q * C + gi];
      const double dd = row[L.s[CB_CHANNEL_DISSIPATED] + q * C + gi];
      moved[sp] += tr;
      absmoved[sp] += fabs(tr);
      chd_sum += dd;
      chd_abs += fabs(dd);
      ok = ok && is_finite(tr) && is_finite(dd);
      for (int r = 0; r < 2; ++r) {
        const double g = row[L.s[CB_CHANNEL_GATE] + (r * nch + q) * C + gi];
        ok = ok && is_finite(g) && g >= 0.0 && g <= 1.0;
      }
      const double dprev = prev[L.s[CB_CHANNEL_DISSIPATED] + q * C + gi];
      if (dd < -kDissipationAtol || dd - dprev < -kDissipationAtol) fail |= 1u << K_DISSIPATION;
    }
    if (!ok) fail |= 1u << K_DOMAIN;
    // Local material: n + total_m + sum over its junctions sent - received.
    double send[3] = {0, 0, 0}, recv[3] = {0, 0, 0}, abs_j[3] = {0, 0, 0};
    for (int a = __ldg(T.adj_ptr + gi); a < __ldg(T.adj_ptr + gi + 1); ++a) {
      const int code = __ldg(T.adj_idx + a);
      const long long ge = e0 + (code >> 1);
      for (int sp = 0; sp < 3; ++sp) {
        const double j = row[L.s[CB_JUNCTION_TRANSFERRED] + sp * E + ge];
        if (code & 1) recv[sp] += j;
        else send[sp] += j;
        abs_j[sp] += fabs(j);
      }
    }
    for (int sp = 0; sp < 3; ++sp) {
      const double total_m = moved[sp] - stoich[sp] * pc;
      const double local = ((n[sp] + total_m) + send[sp]) - recv[sp];
      const double mag = (fabs(n[sp]) + absmoved[sp]) + abs_j[sp];
      if (bad(local, A.tol[sp] + rounding * mag)) fail |= 1u << K_LOCAL;
      m_local = fmax(m_local, fabs(local));
      s[sp] += total_m;
      s[3 + sp] += n[sp];
      s[6 + sp] += absmoved[sp];
      s[9 + sp] += fabs(n[sp]);
    }
    // Capacitor: image - initial charge + plate change - charge increment (held bath).
    const double icap = __ldg(T.icap + gi), cap = 1.0 / icap, q0 = __ldg(T.q0 + gi);
    const double q = kChargePerFmol * ((n[0] + n[1]) + (-n[2]));
    const double base = q0 * icap + Vb;
    const double image = cap * base + (-cap) * Vb;
    const double dp = q * icap;
    const double charge = ((image - q0) + cap * dp) - q;
    if (bad(charge, kChargeAtol + kChargeRtol * fabs(q0 + q))) fail |= 1u << K_CHARGE;
    m_charge = fmax(m_charge, fabs(charge));
    s[12] += -(cap * dp);
    s[13] += kChargePerFmol * ((fabs(n[0]) + fabs(n[1])) + fabs(n[2]));
    // Metabolic work: mw + 1e-3 drive cycles.
    const double mw = row[L.s[CB_METABOLIC_WORK] + gi];
    const double met = mw + 1e-3 * wc[WC_DRIVE] * pc;
    if (bad(met, kWorkBound + rounding * (fabs(mw) + 1e-3 * fabs(wc[WC_DRIVE] * pc))))
      fail |= 1u << K_METABOLIC;
    m_metab = fmax(m_metab, fabs(met));
    // Energy: chemical free energy, capacitor energy, heat, less metabolic work.
    double chem = 0.0;
    for (int sp = 0; sp < 3; ++sp) {
      const double a = __ldg(T.ref + sp * C + gi);
      chem += n[sp] * (log(a * __ldg(T.ivol + gi)) - 1.0) + (a + n[sp]) * log1p(n[sp] / a);
    }
    chem *= 1e-3 * kR * temp;
    const double v0 = q0 * icap;
    const double electric = 0.5e12 * (cap * dp * (2.0 * v0 + dp));
    const double md = row[L.s[CB_MEMBRANE_DISSIPATED] + gi];
    const double pd = row[L.s[CB_PUMP_DISSIPATED] + gi];
    s[14] += (((chem + electric) + md + pd) - mw) + chd_sum;
    s[15] += ((fabs(md) + fabs(pd)) + fabs(mw)) + chd_abs;
    for (int f : {CB_MEMBRANE_DISSIPATED, CB_PUMP_DISSIPATED}) {
      const double v = row[L.s[f] + gi], p = prev[L.s[f] + gi];
      if (v < -kDissipationAtol || v - p < -kDissipationAtol) fail |= 1u << K_DISSIPATION;
    }
  }
  for (int e = tid; e < ne; e += BLOCK) {
    const long long ge = e0 + e;
    bool ok = true;
    for (int sp = 0; sp < 3; ++sp) {
      const double j = row[L.s[CB_JUNCTION_TRANSFERRED] + sp * E + ge];
      ok = ok && is_finite(j);
      if (__ldg(T.jap + sp * E + ge) == 0.0 && j != 0.0) ok = false;
    }
    const double jd = row[L.s[CB_JUNCTION_DISSIPATED] + ge];
    const double g = row[L.s[CB_JUNCTION_GATE] + ge];
    ok = ok && is_finite(jd) && is_finite(g) && g >= __ldg(T.jmin + ge) && g <= 1.0;
    if (!ok) fail |= 1u << K_DOMAIN;
    s[14] += jd;
    s[15] += fabs(jd);
    const double p = prev[L.s[CB_JUNCTION_DISSIPATED] + ge];
    if (jd < -kDissipationAtol || jd - p < -kDissipationAtol) fail |= 1u << K_DISSIPATION;
  }
  if (fail) atomicOr(&sFail, fail);
  block_sum<BLOCK, 16>(s, sRed);
  m_local = block_max<BLOCK>(m_local, sRed);
  m_charge = block_max<BLOCK>(m_charge, sRed);
  m_metab = block_max<BLOCK>(m_metab, sRed);
  __syncthreads();
  if (tid != 0) return;
  uint32_t bits = sFail;
  double sup[3], abs_sup[3];
  double m_out = 0.0, m_tot = 0.0;
  double moved_charge = 0.0;
  for (int sp = 0; sp < 3; ++sp) {
    sup[sp] = row[L.s[CB_RESERVOIR_SUPPLIED] + sp * W + w];
    abs_sup[sp] = fabs(sup[sp]);
    const double outside = -s[sp] - sup[sp];
    const double total = s[3 + sp] - sup[sp];
    if (bad(outside, A.tol[sp] + rounding * (s[6 + sp] + abs_sup[sp]))) bits |= 1u << K_OUTSIDE;
    if (bad(total, A.tol[sp] + rounding * (s[9 + sp] + abs_sup[sp]))) bits |= 1u << K_TOTAL;
    m_out = fmax(m_out, fabs(outside));
    m_tot = fmax(m_tot, fabs(total));
    moved_charge += fabs(z[sp] * sup[sp]);
  }
  const double ec = row[L.s[CB_ELECTRODE_CHARGE] + w];
  const double rw = row[L.s[CB_RESERVOIR_WORK] + w];
  const double ew = row[L.s[CB_ELECTRODE_WORK] + w];
  bool world_ok = is_finite(ec) && is_finite(rw) && is_finite(ew);
  for (int sp = 0; sp < 3; ++sp) world_ok = world_ok && is_finite(sup[sp]);
  if (!world_ok) bits |= 1u << K_DOMAIN;
  moved_charge = kChargePerFmol * moved_charge + fabs(ec);
  const double electrode = ec - s[12];
  if (bad(electrode, kChargeAtol + kChargeRtol * fabs(ec))) bits |= 1u << K_ELECTRODE;
  const double global = ec + kChargePerFmol * ((sup[0] + sup[1]) - sup[2]);
  const double gbound = kGlobalChargeAtol + kGlobalChargeRounding * moved_charge;
  const double glimit =
      fmax(gbound + rounding * moved_charge, gbound + grounding * s[13]);
  if (bad(global, glimit)) bits |= 1u << K_GLOBAL;
  const double energy = (s[14] - rw) - ew;
  const double flows = (s[15] + fabs(rw)) + fabs(ew);
  if (bad(energy, kEnergyAtol + A.rtol * flows)) bits |= 1u << K_ENERGY;
  const double res_w = rw - 1e-3 * ((wc[WC_MUB] * sup[0] + wc[WC_MUB + 1] * sup[1]) +
                                    wc[WC_MUB + 2] * sup[2]);
  const double mag_rw = fabs(rw) + 1e-3 * ((fabs(wc[WC_MUB]) * abs_sup[0] +
                                            fabs(wc[WC_MUB + 1]) * abs_sup[1]) +
                                           fabs(wc[WC_MUB + 2]) * abs_sup[2]);
  if (bad(res_w, kWorkBound + rounding * mag_rw)) bits |= 1u << K_RESERVOIR_WORK;
  const double res_e = ew - 1e12 * Vb * ec;
  if (bad(res_e, kWorkBound + rounding * (fabs(ew) + 1e12 * fabs(Vb * ec))))
    bits |= 1u << K_ELECTRODE_WORK;
  const double v[12] = {m_local,       m_out,          m_tot,         m_charge,
                        fabs(electrode), fabs(global),   fabs(energy),  fabs(res_w),
                        fabs(res_e),   m_metab,        fabs(energy) / fmax(flows, kEnergyAtol),
                        fabs(global) / glimit};
  if (failed_out) failed_out[w] = bits;
  if (values_out)
    for (int k = 0; k < 12; ++k) values_out[(size_t)w * 12 + k] = v[k];
  if (R.row < 0) return;
  // The window's row (execution/vector_windows.py:379-404): a refused step is bit 0, failed
  // checks bits 1 + k; the row counts for a world still live within its own row count.
  double *mx = R.maxima + (size_t)w * 12;
  const int64_t flags =
      (R.row > 0 && R.step_status[w] != 0u) ? 1 : (int64_t)bits << kFailureShift;
  if (R.row == 0) {
    const bool ok = flags == 0;
    R.ok[w] = ok;
    R.first[w] = ok ? -1 : 0;
    R.bits[w] = flags;
    for (int k = 0; k < 12; ++k) mx[k] = ok ? v[k] : 0.0;
    R.keep[w] = 1;
    return;
  }
  const bool live = R.row <= R.counts[w] && R.ok[w] != 0;
  const bool failing = live && flags != 0, accept = live && flags == 0;
  if (failing) {
    R.first[w] = R.row;
    R.bits[w] = flags;
    R.ok[w] = 0;
  }
  if (accept)
    for (int k = 0; k < 12; ++k) mx[k] = fmax(mx[k], v[k]);
  R.keep[w] = accept ? 0 : 1;
}

}  // namespace

extern "C" int cb_device_checks(cb_tissue *t, const double *previous, const double *row,
                                int64_t steps, const double *material_atol, double energy_rtol,
                                uint32_t *failed, double *values, void *stream) {
  if (!t || !previous || !row || !material_atol || !failed || !values)
    return fail(CB_ERR_ARGUMENT, "null argument");
  if (steps < 0) return fail(CB_ERR_ARGUMENT, "steps must be non-negative");
  cudaError_t ce = cudaSetDevice(t->device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
  CheckArgs A;
  for (int s = 0; s < 3; ++s) A.tol[s] = material_atol[s];
  A.rtol = energy_rtol;
  A.rounding = kLedgerStepRounding * kEps * (double)steps;
  A.grounding = kComponentStepRounding * kEps * (double)steps;
  A.steps = nullptr;
  A.step_offset = 0;
  WindowRow R{};
  R.row = -1;
  checks_kernel<kChecksBlock><<<t->W, kChecksBlock, 0, static_cast<cudaStream_t>(stream)>>>(
      t->t, t->layout, previous, row, A, R, failed, values);
  ce = cudaGetLastError();
  if (ce != cudaSuccess) return cuda_fail(ce, "device checks launch");
  return CB_OK;
}

extern "C" int cb_device_checks_each(cb_tissue *t, const double *previous, const double *row,
                                     const int64_t *steps, const double *material_atol,
                                     double energy_rtol, uint32_t *failed, double *values,
                                     void *stream) {
  if (!t || !previous || !row || !steps || !material_atol || !failed || !values)
    return fail(CB_ERR_ARGUMENT, "null argument");
  cudaError_t ce = cudaSetDevice(t->device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
  CheckArgs A;
  for (int s = 0; s < 3; ++s) A.tol[s] = material_atol[s];
  A.rtol = energy_rtol;
  A.rounding = 0.0;
  A.grounding = 0.0;
  A.steps = steps;
  A.step_offset = 0;
  WindowRow R{};
  R.row = -1;
  checks_kernel<kChecksBlock><<<t->W, kChecksBlock, 0, static_cast<cudaStream_t>(stream)>>>(
      t->t, t->layout, previous, row, A, R, failed, values);
  ce = cudaGetLastError();
  if (ce != cudaSuccess) return cuda_fail(ce, "device checks launch");
  return CB_OK;
}

// ---------------------------------------------------------------------------------------------
// Per-world state copies (cb_copy_worlds): the window's selects, done for the worlds that need
// them. One CTA per world; a world whose mask entry is zero returns at once.

namespace {

template <int BLOCK>
__device__ __forceinline__ void copy_world(const Tissue &T, const Layout &L, int w,
                                           const double *__restrict__ src,
                                           double *__restrict__ dst) {
  const int tid = threadIdx.x;
  const long long C = T.C, E = T.E, W = T.W;
  const int c0 = T.cell_offset[w], nc = T.cell_offset[w + 1] - c0;
  const int e0 = T.edge_offset[w], ne = T.edge_offset[w + 1] - e0;
  const int nch = T.nch;
  // Cell fields: [reps][C] each.
  const int cell_field[9] = {CB_AMOUNT_INCREMENT, CB_MEMBRANE_TRANSFERRED, CB_MEMBRANE_DISSIPATED,
                             CB_PUMP_CYCLES,      CB_PUMP_DISSIPATED,      CB_METABOLIC_WORK,
                             CB_CHANNEL_GATE,     CB_CHANNEL_TRANSFERRED,  CB_CHANNEL_DISSIPATED};
  const int cell_reps[9] = {3, 3, 1, 1, 1, 1, 2 * nch, nch, nch};
  for (int f = 0; f < 9; ++f)
    for (int r = 0; r < cell_reps[f]; ++r) {
      const long long base = L.s[cell_field[f]] + (long long)r * C + c0;
      for (int i = tid; i < nc; i += BLOCK) dst[base + i] = src[base + i];
    }
  // Junction fields: [reps][E] each.
  const int edge_field[3] = {CB_JUNCTION_TRANSFERRED, CB_JUNCTION_DISSIPATED, CB_JUNCTION_GATE};
  const int edge_reps[3] = {3, 1, 1};
  for (int f = 0; f < 3; ++f)
    for (int r = 0; r < edge_reps[f]; ++r) {
      const long long base = L.s[edge_field[f]] + (long long)r * E + e0;
      for (int i = tid; i < ne; i += BLOCK) dst[base + i] = src[base + i];
    }
  // World fields: [reps][W] each.
  if (tid < 6) {
    const int f = tid < 3 ? CB_RESERVOIR_SUPPLIED : CB_ELECTRODE_CHARGE + (tid - 3);
    const long long at = L.s[f] + (tid < 3 ? (long long)tid * W : 0) + w;
    dst[at] = src[at];
  }
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
    copy_worlds_kernel(const Tissue T, const Layout L, const int32_t *__restrict__ mask,
                       const double *__restrict__ src, double *__restrict__ dst) {
  if (mask[blockIdx.x] == 0) return;
  copy_world<BLOCK>(T, L, blockIdx.x, src, dst);
}

// World w's state into stored row slot[w] (rows of `stride` doubles) where keep[w] == 0 and
// 0 <= slot[w] < n_rows.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
    store_worlds_kernel(const Tissue T, const Layout L, const int32_t *__restrict__ keep,
                        const int64_t *__restrict__ slot, int n_rows, long long stride,
                        const double *__restrict__ src, double *__restrict__ rows) {
  const int w = blockIdx.x;
  const int64_t s = slot[w];
  if (keep[w] != 0 || s < 0 || s >= n_rows) return;
  copy_world<BLOCK>(T, L, w, src, rows + s * stride);
}

}  // namespace

extern "C" int cb_copy_worlds(cb_tissue *t, const int32_t *mask, const double *src, double *dst,
                              void *stream) {
  if (!t || !mask || !src || !dst) return fail(CB_ERR_ARGUMENT, "null argument");
  if (src == dst) return CB_OK;
  cudaError_t ce = cudaSetDevice(t->device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
  copy_worlds_kernel<256><<<t->W, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      t->t, t->layout, mask, src, dst);
  ce = cudaGetLastError();
  if (ce != cudaSuccess) return cuda_fail(ce, "copy worlds launch");
  return CB_OK;
}

extern "C" int cb_window_row(cb_tissue *t, const double *previous, const double *row,
                             int32_t row_index, const int64_t *first_step, int64_t first_all,
                             const double *material_atol, double energy_rtol,
                             const uint32_t *step_status, const int64_t *counts, int32_t *ok,
                             int32_t *first, int64_t *bits, double *maxima, int32_t *keep,
                             void *stream) {
  if (!t || !previous || !row || !material_atol || !counts || !ok || !first || !bits ||
      !maxima || !keep || (row_index > 0 && !step_status))
    return fail(CB_ERR_ARGUMENT, "null argument");
  if (row_index < 0) return fail(CB_ERR_ARGUMENT, "row_index must be non-negative");
  if (!first_step && first_all < 0) return fail(CB_ERR_ARGUMENT, "steps must be non-negative");
  cudaError_t ce = cudaSetDevice(t->device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
  CheckArgs A;
  for (int s = 0; s < 3; ++s) A.tol[s] = material_atol[s];
  A.rtol = energy_rtol;
  A.rounding = kLedgerStepRounding * kEps * (double)(first_all + row_index);
  A.grounding = kComponentStepRounding * kEps * (double)(first_all + row_index);
  A.steps = first_step;
  A.step_offset = row_index;
  WindowRow R{row_index, step_status, counts, ok, first, bits, maxima, keep};
  checks_kernel<kChecksBlock><<<t->W, kChecksBlock, 0, static_cast<cudaStream_t>(stream)>>>(
      t->t, t->layout, previous, row, A, R, nullptr, nullptr);
  ce = cudaGetLastError();
  if (ce != cudaSuccess) return cuda_fail(ce, "window row launch");
  return CB_OK;
}

extern "C" int cb_store_worlds(cb_tissue *t, const int32_t *keep, const int64_t *slot,
                               const double *src, double *rows, int32_t n_rows, void *stream) {
  if (!t || !keep || !slot || !src || !rows) return fail(CB_ERR_ARGUMENT, "null argument");
  if (n_rows <= 0) return CB_OK;
  cudaError_t ce = cudaSetDevice(t->device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
  store_worlds_kernel<256><<<t->W, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      t->t, t->layout, keep, slot, n_rows, t->state_total, src, rows);
  ce = cudaGetLastError();
  if (ce != cudaSuccess) return cuda_fail(ce, "store worlds launch");
  return CB_OK;
}
