// packed_step.cuh - the packed persistent form of the ARS(2,2,2) tissue step (included by
// tissue_step.cu inside its anonymous namespace).
//
// Worlds of uneven size (tens to thousands of cells) are grouped on the host into work items:
// runs of consecutive worlds whose cells fit one CTA's shared-memory exchange arrays (CAP cells,
// at most MAXW worlds). A persistent grid (one CTA per SM) takes items from a device ticket
// counter, largest item first, and advances every world of an item n_steps steps. Threads loop
// over the item's cells and junctions; the only shared-memory arrays are what neighbours read
// (potential, concentrations and their logs); the stage accumulators, junction fluxes and
// per-cell world-sum terms live in a scratch buffer that stays in L2 while its item runs.
// World sums (bath inflow, electrode plate charge) are warp-per-world reductions in a fixed
// order, so a world's bits do not depend on the item it was packed into. Each world is accepted
// or refused step by step on its own; a refused world freezes at its last accepted state while
// the rest of its item continues. Arithmetic per cell and junction is the shared-memory
// kernel's (tissue_step.cu), in the same order.


// Scratch fields (cells): the accumulator (n[3], mt[3], md, pc, pd, mw), the stage-1 amounts,
// the patch flux and outward extra transfer of the current stage, the world-sum terms (stage-0
// inflow[3], stage-1 inflow[3], end plate charge), then per channel slot: the transferred and
// dissipated accumulators, the new gates [2], the stage-1 gates [2] (then the end targets), the
// start targets [2] and time constants [2], and the end time constants [2].
enum ScratchCell { SC_ACC = 0, SC_N1 = 10, SC_JM = 13, SC_EX = 16, SC_RED = 19, SC_CH = 26 };
constexpr int kChFields = 12;
// Scratch fields (junctions): flux[3], accumulator (jt[3], jd, g), stage-1 gate.
enum ScratchEdge { SE_J = 0, SE_ACC = 3, SE_G1 = 8, SE_FIELDS = 9 };

__host__ __device__ constexpr int packed_cell_fields(int nch) { return SC_CH + kChFields * nch; }

__host__ __device__ constexpr size_t packed_smem_bytes(int cap) {
  return sizeof(double) * (size_t)(7 * cap + 8 * kPackedMaxWorlds) +
         sizeof(unsigned int) * 3 * kPackedMaxWorlds;
}

template <int BLOCK, int NCH, bool BLK = false, bool MIX = false>
__global__ void __launch_bounds__(BLOCK, 1)
    packed_kernel(const Tissue T, const Layout L, const Packed P, const double *state_in,
                  double *state_out, const double *__restrict__ control, const StepCoef k,
                  int n_steps, uint32_t *__restrict__ world_status,
                  int32_t *__restrict__ accepted_steps) {
  constexpr int WARPS = BLOCK / 32;
  constexpr int NQ = NCH > 0 ? NCH : 1;
  extern __shared__ double smem[];
  const int CAP = P.cap;
  double *sV = smem;                       // [CAP]
  double *sC = sV + CAP;                   // [3][CAP]
  double *sL = sC + 3 * CAP;               // [3][CAP]
  double *sWL = sL + 3 * CAP;              // [MAXW][8]: res[3], ec, rw, ew, plate0, -
  unsigned int *sBits = (unsigned int *)(sWL + 8 * kPackedMaxWorlds);  // [MAXW] this step
  unsigned int *sRef = sBits + kPackedMaxWorlds;                       // [MAXW] refused
  int *sTaken = (int *)(sRef + kPackedMaxWorlds);                      // [MAXW]
  __shared__ int sTicket;
  __shared__ int sLive;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long C = T.C, E = T.E;
  const int FC = packed_cell_fields(NCH);
  double *scC = P.sc;                      // [FC][C]
  double *scE = P.sc + (size_t)FC * C;     // [SE_FIELDS][E]
  auto SCc = [&](int f, long long gi) -> double & { return scC[f * C + gi]; };
  auto SCe = [&](int f, long long ge) -> double & { return scE[f * E + ge]; };
  auto CH = [&](int q, int f, long long gi) -> double & {  // channel slot q, field f
    return scC[(SC_CH + q * kChFields + f) * C + gi];
  };

  for (;;) {
    if (tid == 0) sTicket = (int)atomicAdd(P.queue, 1u);
    __syncthreads();
    const int ticket = sTicket;
    if (ticket >= P.n_items) break;
    const int item = P.order[ticket];
    const int w0 = P.item_world0[item], nw = P.item_world0[item + 1] - w0;
    const int c0 = T.cell_offset[w0], nc = T.cell_offset[w0 + nw] - c0;
    const int e0 = T.edge_offset[w0], ne = T.edge_offset[w0 + nw] - e0;

    // The item's state moves to state_out first; steps then update it in place.
    if (state_in != state_out) {
      for (int f = CB_AMOUNT_INCREMENT; f <= CB_METABOLIC_WORK; ++f) {
        const int reps = f <= CB_MEMBRANE_TRANSFERRED ? 3 : 1;
        for (int s = 0; s < reps; ++s)
          for (int cl = tid; cl < nc; cl += BLOCK)
            state_out[L.s[f] + s * C + c0 + cl] = state_in[L.s[f] + s * C + c0 + cl];
      }
      for (int f = CB_CHANNEL_GATE; f <= CB_CHANNEL_DISSIPATED; ++f) {
        const int reps = f == CB_CHANNEL_GATE ? 2 * NCH : NCH;
        for (int s = 0; s < reps; ++s)
          for (int cl = tid; cl < nc; cl += BLOCK)
            state_out[L.s[f] + s * C + c0 + cl] = state_in[L.s[f] + s * C + c0 + cl];
      }
      for (int f = CB_JUNCTION_TRANSFERRED; f <= CB_JUNCTION_GATE; ++f) {
        const int reps = f == CB_JUNCTION_TRANSFERRED ? 3 : 1;
        for (int s = 0; s < reps; ++s)
          for (int el = tid; el < ne; el += BLOCK)
            state_out[L.s[f] + s * E + e0 + el] = state_in[L.s[f] + s * E + e0 + el];
      }
    }
    const double *cur = state_out;
    for (int wl = tid; wl < nw; wl += BLOCK) {
      const int w = w0 + wl;
      double *r = sWL + 8 * wl;
      for (int s = 0; s < 3; ++s) r[s] = state_in[L.s[CB_RESERVOIR_SUPPLIED] + s * (long long)T.W + w];
      r[3] = state_in[L.s[CB_ELECTRODE_CHARGE] + w];
      r[4] = state_in[L.s[CB_RESERVOIR_WORK] + w];
      r[5] = state_in[L.s[CB_ELECTRODE_WORK] + w];
      sBits[wl] = 0u;
      sRef[wl] = 0u;
      sTaken[wl] = 0;
    }
    __syncthreads();
    // Start plate charge and, with channels, the start kinetics of every cell.
    for (int cl = tid; cl < nc; cl += BLOCK) {
      const long long gi = c0 + cl;
      const double n0 = cur[L.s[CB_AMOUNT_INCREMENT] + gi];
      const double n1 = cur[L.s[CB_AMOUNT_INCREMENT] + C + gi];
      const double n2 = cur[L.s[CB_AMOUNT_INCREMENT] + 2 * C + gi];
      SCc(SC_RED + 6, gi) = -(kChargePerFmol * ((n0 + n1) + (-n2)));
      if constexpr (NCH > 0) {
        const int wl = P.cell_world[gi];
        const double *wc = T.world + (size_t)(w0 + wl) * WC_STRIDE;
        const double Vb = __ldg(wc + WC_VB);
        const double V = (__ldg(T.q0 + gi) + kChargePerFmol * ((n0 + n1) + (-n2))) *
                             __ldg(T.icap + gi) + Vb;
        bool ok = true;
        for (int q = 0; q < NCH; ++q) {
          double t[2], tau[2];
          channel_kinetics<false>(__ldg(T.ch_code + q * C + gi), V - Vb, t, tau);
          ok = ok && channel_kinetics_ok(V - Vb, t, tau);
          for (int r = 0; r < 2; ++r) {
            CH(q, 6 + r, gi) = t[r];
            CH(q, 8 + r, gi) = tau[r];
          }
        }
        if (!ok) atomicOr(&sBits[wl], CB_WORLD_CHANNEL_DOMAIN);
      }
    }
    __syncthreads();
    // World sums, warp per world: the start plate charge.
    for (int wl = warp; wl < nw; wl += WARPS) {
      const int a = T.cell_offset[w0 + wl], b = T.cell_offset[w0 + wl + 1];
      double v = 0.0;
      for (long long gi = a + lane; gi < b; gi += 32) v += SCc(SC_RED + 6, gi);
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) sWL[8 * wl + 6] = v;
    }
    __syncthreads();

    for (int step = 0; step < n_steps; ++step) {
      // Two explicit stages; stage 1 reads the stage-1 amounts and gates from scratch.
      for (int st = 0; st < 2; ++st) {
        const bool first = st == 0;
        const double w_acc = first ? k.delta_dt : k.omdelta_dt;
        // Cell phase.
        for (int cl = tid; cl < nc; cl += BLOCK) {
          const long long gi = c0 + cl;
          const int wl = P.cell_world[gi];
          if (sRef[wl]) continue;
          const double *wc = T.world + (size_t)(w0 + wl) * WC_STRIDE;
          const double RT = __ldg(wc + WC_RT), Vb = __ldg(wc + WC_VB);
          uint32_t bits = 0u;
          double n[3];
          for (int s = 0; s < 3; ++s)
            n[s] = first ? cur[L.s[CB_AMOUNT_INCREMENT] + s * C + gi] : SCc(SC_N1 + s, gi);
          const double q0 = __ldg(T.q0 + gi), icap = __ldg(T.icap + gi);
          const double V = (q0 + kChargePerFmol * ((n[0] + n[1]) + (-n[2]))) * icap + Vb;
          if (!first && !is_finite(V)) bits |= CB_WORLD_RESIDUAL;
          // Stage gates: the start's (stage 0), or the exponential update to the stage-1
          // potential (surface_pump_v3.stage_gates).
          double chg[2][NQ];
          if constexpr (NCH > 0) {
            for (int q = 0; q < NCH; ++q) {
              const int code = __ldg(T.ch_code + q * C + gi);
              for (int r = 0; r < 2; ++r)
                chg[r][q] = cur[L.s[CB_CHANNEL_GATE] + (r * NCH + q) * C + gi];
              if (!first) {
                double t[2], tau[2];
                channel_kinetics<false>(code, V - Vb, t, tau);
                if (!channel_kinetics_ok(V - Vb, t, tau)) bits |= CB_WORLD_CHANNEL_DOMAIN;
                for (int r = 0; r < 2; ++r) {
                  if (!(r == 1 && code == kHhKn4))
                    chg[r][q] = advance_gate<false>(chg[r][q], CH(q, 6 + r, gi), CH(q, 8 + r, gi),
                                             t[r], tau[r], k.frac1_dt);
                  CH(q, 4 + r, gi) = chg[r][q];
                }
              }
            }
          }
          double c[3], lc[3];
          const double ivol = __ldg(T.ivol + gi);
          for (int s = 0; s < 3; ++s) {
            c[s] = (__ldg(T.ref + s * C + gi) + n[s]) * ivol;
            lc[s] = log(c[s]);
            sL[s * CAP + cl] = lc[s];
            if (!(is_finite(c[s]) && c[s] > 0.0)) bits |= CB_WORLD_TRANSPORT;
            sC[s * CAP + cl] = c[s];
          }
          sV[cl] = V;
          if (!is_finite(V)) bits |= CB_WORLD_TRANSPORT;
          const double mc = control[L.c[CB_CONTROL_MEMBRANE] + gi];
          const double pctl = control[L.c[CB_CONTROL_PUMP] + gi];
          const double dv = V - Vb;
          const double x = dv * __ldg(wc + WC_FRT);
          if (!(fabs(x) <= kMaxAbsX)) bits |= CB_WORLD_TRANSPORT;
          double bp, bm;
          bernoulli_pair_at<MIX>(x, bp, bm);
          double jm[3], mu[3];
          for (int s = 0; s < 3; ++s) {
            const double gs = __ldg(T.ap + s * C + gi) * mc;
            const double co = __ldg(wc + WC_CO + s);
            const double zfdv = (s < 2) ? kF * dv : (-kF) * dv;
            if constexpr (MIX) {
              // FP32 on the FP64 concentration difference (the shared kernel's mixed form).
              const float d = (float)(c[s] - co), fb = (float)bp, fx = (float)x;
              const float J = (float)gs * ((s < 2) ? d * fb + (float)c[s] * fx
                                                   : d * fb - (float)co * fx);
              jm[s] = J;
            } else {
              jm[s] = (s < 2) ? gs * (c[s] * bm - co * bp) : gs * (c[s] * bp - co * bm);
            }
            mu[s] = RT * (lc[s] - __ldg(wc + WC_LOGCO + s)) + zfdv;
          }
          const double md = 1e-3 * ((jm[0] * mu[0] + jm[1] * mu[1]) + jm[2] * mu[2]);
          if (!(is_finite(jm[0]) && is_finite(jm[1]) && is_finite(jm[2]) && is_finite(md)))
            bits |= CB_WORLD_TRANSPORT;
          if (!(is_finite(mc) && mc >= 0.0 && mc <= 1.0 && is_finite(pctl) && pctl >= 0.0 &&
                pctl <= 1.0))
            bits |= CB_WORLD_CONTROL;
          double largest[3];
          for (int s = 0; s < 3; ++s) largest[s] = fmax(c[s], __ldg(wc + WC_CO + s));
          double membrane =
              ((((__ldg(T.ap + gi) * largest[0]) + __ldg(T.ap + C + gi) * largest[1]) +
                __ldg(T.ap + 2 * C + gi) * largest[2]) * 1e-15) * mc;
          double chm[3] = {0.0, 0.0, 0.0};
          double blocked_tv = 0.0;  // the blocked populations' T_V (S)
          if constexpr (NCH > 0) {
            for (int q = 0; q < NCH; ++q) {
              const int code = __ldg(T.ch_code + q * C + gi);
              const int sp = __ldg(T.ch_species + q * C + gi);
              const double ctl = control[L.c[CB_CONTROL_CHANNEL] + q * C + gi];
              if (!(is_finite(ctl) && ctl >= 0.0 && ctl <= 1.0)) bits |= CB_WORLD_CONTROL;
              const double open = channel_opening(code, chg[0][q], chg[1][q]);
              const double available = (open * ctl) * __ldg(T.ch_ab + q * C + gi);
              const double gq = __ldg(T.ch_ap + q * C + gi) * available;
              const double cs = c[sp], cos_ = __ldg(wc + WC_CO + sp);
              double J;
              if constexpr (MIX) {
                const float d = (float)(cs - cos_), fb = (float)bp, fx = (float)x;
                J = (float)gq * (sp < 2 ? d * fb + (float)cs * fx : d * fb - (float)cos_ * fx);
              } else {
                J = sp < 2 ? gq * (cs * bm - cos_ * bp) : gq * (cs * bp - cos_ * bm);
              }
              const double gterm =
                  ((__ldg(T.ch_ap + q * C + gi) * 1e-15) * largest[sp]) * available;
              if constexpr (BLK) {
                // Open-channel block (surface_pump_v3.channel_rates :958-960, channel_block_terms
                // :1051-1090): u multiplies the flux; the stability rule takes the population's
                // T_V = u G_max + |I_free| slope in place of G_max.
                double u, su;
                bool bok = true;
                channel_block(T, q, gi, dv, u, su, bok);
                if (!bok) bits |= CB_WORLD_CHANNEL_DOMAIN;
                const double ifree = kChargePerFmol * ((sp < 2 ? 1.0 : -1.0) * J);
                blocked_tv += u * (__ldg(wc + WC_SLOPE) * gterm) + fabs(ifree) * su;
                J = J * u;
              } else {
                membrane += gterm;
              }
              const double Jd = 1e-3 * J * mu[sp];
              chm[sp] += J;
              if (first) {
                CH(q, 0, gi) = cur[L.s[CB_CHANNEL_TRANSFERRED] + q * C + gi] + w_acc * J;
                CH(q, 1, gi) = cur[L.s[CB_CHANNEL_DISSIPATED] + q * C + gi] + w_acc * Jd;
              } else {
                CH(q, 0, gi) = CH(q, 0, gi) + w_acc * J;
                CH(q, 1, gi) = CH(q, 1, gi) + w_acc * Jd;
              }
              if (!(is_finite(J) && is_finite(Jd))) bits |= CB_WORLD_TRANSPORT;
            }
          }
          if (!(k.dt * ((__ldg(wc + WC_SLOPE) * membrane + blocked_tv) * icap) <= 1.0))
            bits |= CB_WORLD_STIFF;
          // Pump.
          const double drive = __ldg(wc + WC_DRIVE);
          const double energy = (drive + (-3.0) * mu[0]) + 2.0 * mu[1];
          const double a = energy * __ldg(wc + WC_INVRT);
          double cycles = 0.0;
          const double capacity = __ldg(T.pcap + gi);
          if (capacity > 0.0 && pctl > 0.0) {
            const double ldc = __ldg(T.logpcap + gi) + log(pctl);
            const double ls = ((-logaddexp0(3.0 * (__ldg(wc + WC_LOGKMNA) - lc[0]))) -
                               __ldg(wc + WC_LK)) - __ldg(wc + WC_LATP);
            const double mag = exp((ldc + ls) + fmax(a, 0.0));
            const double dep = a >= 0.0 ? expm1(-a) : -expm1(a);
            cycles = mag * dep;
          }
          const double pd = (-1e-3 * cycles) * energy;
          const double mw = (-1e-3 * cycles) * drive;
          const double sna = mu[0] * __ldg(wc + WC_INVRTD), sk = mu[1] * __ldg(wc + WC_INVRTD);
          const double aff = (__ldg(wc + WC_AFF0) + (-3.0) * sna) + 2.0 * sk;
          if (!(__ldg(wc + WC_PUMPOK) != 0.0 && is_finite(capacity) && capacity >= 0.0 &&
                is_finite(sna) && fabs(sna) <= kMaxAbsIonPotentialOverRT && is_finite(sk) &&
                fabs(sk) <= kMaxAbsIonPotentialOverRT && is_finite(aff) &&
                fabs(aff) <= kMaxAbsAffinityOverRT))
            bits |= CB_WORLD_PUMP_DOMAIN;
          if (!(is_finite(cycles) && is_finite(pd) && is_finite(mw))) bits |= CB_WORLD_TRANSPORT;
          const double ex[3] = {(3.0 * cycles - 0.0) + chm[0], (-2.0 * cycles - 0.0) + chm[1],
                                (-0.0 * cycles - 0.0) + chm[2]};
          const double led[7] = {jm[0], jm[1], jm[2], md, cycles, pd, mw};
          const int offs[7] = {CB_MEMBRANE_TRANSFERRED, CB_MEMBRANE_TRANSFERRED,
                               CB_MEMBRANE_TRANSFERRED, CB_MEMBRANE_DISSIPATED, CB_PUMP_CYCLES,
                               CB_PUMP_DISSIPATED, CB_METABOLIC_WORK};
          for (int f = 0; f < 7; ++f) {
            const long long at = L.s[offs[f]] + (f < 3 ? f * C : 0) + gi;
            SCc(SC_ACC + 3 + f, gi) =
                first ? cur[at] + w_acc * led[f] : SCc(SC_ACC + 3 + f, gi) + w_acc * led[f];
          }
          for (int s = 0; s < 3; ++s) {
            SCc(SC_JM + s, gi) = jm[s];
            SCc(SC_EX + s, gi) = ex[s];
          }
          if (bits) atomicOr(&sBits[wl], bits);
        }
        __syncthreads();
        // Junction phase.
        for (int el = tid; el < ne; el += BLOCK) {
          const long long ge = e0 + el;
          const int s_ = P.isnd[ge], r_ = P.ircv[ge];
          const int wl = P.cell_world[c0 + s_];
          if (sRef[wl]) continue;
          const double *wc = T.world + (size_t)(w0 + wl) * WC_STRIDE;
          const double RT = __ldg(wc + WC_RT);
          uint32_t bits = 0u;
          const double g = first ? cur[L.s[CB_JUNCTION_GATE] + ge] : SCe(SE_G1, ge);
          const double dv = sV[s_] - sV[r_];
          const double jc = control[L.c[CB_CONTROL_JUNCTION] + ge];
          const double opening = jc * g;
          const double x = dv * __ldg(wc + WC_FRT);
          if (!(fabs(x) <= kMaxAbsX)) bits |= CB_WORLD_TRANSPORT;
          double bp, bm;
          bernoulli_pair_at<MIX>(x, bp, bm);
          double jj[3], mu[3];
          for (int s = 0; s < 3; ++s) {
            const double gs = __ldg(T.jap + s * E + ge) * opening;
            const double cs = sC[s * CAP + s_], cr = sC[s * CAP + r_];
            const double zfdv = (s < 2) ? kF * dv : (-kF) * dv;
            if constexpr (MIX) {
              // FP32 on the FP64 difference c_s - c_r.
              const float d = (float)(cs - cr), fb = (float)bp, fx = (float)x;
              jj[s] = (float)gs * ((s < 2) ? d * fb + (float)cs * fx : d * fb - (float)cr * fx);
            } else {
              jj[s] = (s < 2) ? gs * (cs * bm - cr * bp) : gs * (cs * bp - cr * bm);
            }
            mu[s] = RT * (sL[s * CAP + s_] - sL[s * CAP + r_]) + zfdv;
            SCe(SE_J + s, ge) = jj[s];
          }
          const double jd = 1e-3 * ((jj[0] * mu[0] + jj[1] * mu[1]) + jj[2] * mu[2]);
          const double thr = __ldg(T.thr + ge), mn = __ldg(T.jmin + ge);
          double gr = 0.0;
          if (mn < 1.0) {
            const double shift = fabs(dv) - thr;
            const double alpha = 1.3 * exp(-77.0 * shift);
            const double log_beta = kLog0065 + 140.0 * shift;
            const double beta = 20.0 * exp(-logaddexp0(-log_beta));
            gr = alpha * (1.0 - g) - beta * (g - mn);
          }
          const double led[5] = {jj[0], jj[1], jj[2], jd, gr};
          for (int f = 0; f < 5; ++f) {
            double y;
            if (first)
              y = f < 3   ? cur[L.s[CB_JUNCTION_TRANSFERRED] + f * E + ge]
                  : f == 3 ? cur[L.s[CB_JUNCTION_DISSIPATED] + ge]
                           : g;
            else
              y = SCe(SE_ACC + f, ge);
            SCe(SE_ACC + f, ge) = y + w_acc * led[f];
          }
          if (first) SCe(SE_G1, ge) = g + k.gamma_dt * gr;
          if (!(is_finite(jj[0]) && is_finite(jj[1]) && is_finite(jj[2]) && is_finite(jd) && is_finite(gr)))
            bits |= CB_WORLD_TRANSPORT;
          if (!(is_finite(thr) && thr >= 0.0 && thr <= kMaxAbsJunctionV && is_finite(mn) && mn >= 0.0 &&
                mn <= 1.0 && is_finite(dv) && fabs(dv) <= kMaxAbsJunctionV && is_finite(g) && g >= mn &&
                g <= 1.0 && is_finite(jc) && jc >= 0.0 && jc <= 1.0))
            bits |= CB_WORLD_GATE_DOMAIN;
          if (bits) atomicOr(&sBits[wl], bits);
        }
        __syncthreads();
        // Gather phase: the amount rates, in edge order (senders, then receivers).
        for (int cl = tid; cl < nc; cl += BLOCK) {
          const long long gi = c0 + cl;
          const int wl = P.cell_world[gi];
          if (sRef[wl]) continue;
          uint32_t bits = 0u;
          double send[3] = {0.0, 0.0, 0.0}, recv[3] = {0.0, 0.0, 0.0};
          const int a0 = __ldg(T.adj_ptr + gi), a1 = __ldg(T.adj_ptr + gi + 1);
          for (int a = a0; a < a1; ++a) {
            const int code = __ldg(P.iadj + a);
            const long long ge = e0 + (code >> 1);
            if (code & 1) {
              for (int s = 0; s < 3; ++s) recv[s] += SCe(SE_J + s, ge);
            } else {
              for (int s = 0; s < 3; ++s) send[s] += -SCe(SE_J + s, ge);
            }
          }
          for (int s = 0; s < 3; ++s) {
            const double jm = SCc(SC_JM + s, gi), ex = SCc(SC_EX + s, gi);
            const double rate = ((-jm + send[s]) + recv[s]) - ex;
            SCc(SC_RED + 3 * st + s, gi) = jm + ex;
            if (!is_finite(rate)) bits |= CB_WORLD_TRANSPORT;
            if (first) {
              const double n = cur[L.s[CB_AMOUNT_INCREMENT] + s * C + gi];
              SCc(SC_N1 + s, gi) = n + k.gamma_dt * rate;
              SCc(SC_ACC + s, gi) = n + w_acc * rate;
            } else {
              SCc(SC_ACC + s, gi) = SCc(SC_ACC + s, gi) + w_acc * rate;
            }
          }
          if (!first) {
            // The new state: its potential, final channel gates and domain; the end plate charge.
            bool ok = true;
            for (int f = 0; f < 10; ++f) ok = ok && is_finite(SCc(SC_ACC + f, gi));
            for (int s = 0; s < 3; ++s)
              ok = ok && (__ldg(T.ref + s * C + gi) + SCc(SC_ACC + s, gi)) > 0.0;
            const double *wc = T.world + (size_t)(w0 + wl) * WC_STRIDE;
            const double Vb = __ldg(wc + WC_VB);
            const double qn = kChargePerFmol *
                              ((SCc(SC_ACC, gi) + SCc(SC_ACC + 1, gi)) + (-SCc(SC_ACC + 2, gi)));
            const double V2 = (__ldg(T.q0 + gi) + qn) * __ldg(T.icap + gi) + Vb;
            if (!is_finite(V2)) bits |= CB_WORLD_RESIDUAL;
            SCc(SC_RED + 6, gi) = -qn;
            if constexpr (NCH > 0) {
              bool k2 = true;
              for (int q = 0; q < NCH; ++q) {
                const int code = __ldg(T.ch_code + q * C + gi);
                double t[2], tau[2];
                channel_kinetics<false>(code, V2 - Vb, t, tau);
                k2 = k2 && channel_kinetics_ok(V2 - Vb, t, tau);
                for (int r = 0; r < 2; ++r) {
                  const double g0 = cur[L.s[CB_CHANNEL_GATE] + (r * NCH + q) * C + gi];
                  double g = g0;
                  if (!(r == 1 && code == kHhKn4))
                    g = advance_gate<false>(g0, CH(q, 6 + r, gi), CH(q, 8 + r, gi), t[r], tau[r],
                                     k.frac2_dt);
                  CH(q, 2 + r, gi) = g;
                  // The end kinetics: the next step's start once this step is accepted.
                  CH(q, 4 + r, gi) = t[r];
                  CH(q, 10 + r, gi) = tau[r];
                  ok = ok && is_finite(g) && g >= 0.0 && g <= 1.0;
                }
                ok = ok && is_finite(CH(q, 0, gi)) && is_finite(CH(q, 1, gi));
              }
              if (!k2) bits |= CB_WORLD_CHANNEL_DOMAIN;
            }
            if (!ok) bits |= CB_WORLD_DOMAIN;
          }
          if (bits) atomicOr(&sBits[wl], bits);
        }
        __syncthreads();
      }
      // World sums, warp per world, and each world's decision.
      for (int wl = warp; wl < nw; wl += WARPS) {
        if (sRef[wl]) continue;
        const int a = T.cell_offset[w0 + wl], b = T.cell_offset[w0 + wl + 1];
        double v[7] = {0, 0, 0, 0, 0, 0, 0};
        for (long long gi = a + lane; gi < b; gi += 32)
          for (int f = 0; f < 7; ++f) v[f] += SCc(SC_RED + f, gi);
        for (int f = 0; f < 7; ++f)
          for (int o = 16; o > 0; o >>= 1) v[f] += __shfl_xor_sync(0xffffffffu, v[f], o);
        if (lane == 0) {
          const double *wc = T.world + (size_t)(w0 + wl) * WC_STRIDE;
          double *r = sWL + 8 * wl;
          double res2[3], applied[3];
          for (int s = 0; s < 3; ++s) {
            const double k0r = -v[s], k1r = -v[3 + s];
            res2[s] = (r[s] + k.delta_dt * k0r) + k.omdelta_dt * k1r;
            applied[s] = k.delta * k0r + k.omdelta * k1r;
          }
          const double electrode = v[6] - r[6];
          const double ec2 = r[3] + electrode;
          const double rw2 = r[4] + 1e-3 * ((__ldg(wc + WC_MUB) * (k.dt * applied[0]) +
                                             __ldg(wc + WC_MUB + 1) * (k.dt * applied[1])) +
                                            __ldg(wc + WC_MUB + 2) * (k.dt * applied[2]));
          const double ew2 = r[5] + (1e12 * __ldg(wc + WC_VB)) * electrode;
          unsigned int bits = sBits[wl];
          if (!(is_finite(res2[0]) && is_finite(res2[1]) && is_finite(res2[2]) && is_finite(ec2) &&
                is_finite(rw2) && is_finite(ew2)))
            bits |= CB_WORLD_DOMAIN;
          if (bits) {
            sRef[wl] = bits;
          } else {
            for (int s = 0; s < 3; ++s) r[s] = res2[s];
            r[3] = ec2;
            r[4] = rw2;
            r[5] = ew2;
            r[6] = v[6];
            sTaken[wl] += 1;
          }
        }
      }
      __syncthreads();
      // Commit each world accepted at this step (its slots only).
      for (int cl = tid; cl < nc; cl += BLOCK) {
        const long long gi = c0 + cl;
        if (sRef[P.cell_world[gi]]) continue;
        for (int s = 0; s < 3; ++s) {
          state_out[L.s[CB_AMOUNT_INCREMENT] + s * C + gi] = SCc(SC_ACC + s, gi);
          state_out[L.s[CB_MEMBRANE_TRANSFERRED] + s * C + gi] = SCc(SC_ACC + 3 + s, gi);
        }
        state_out[L.s[CB_MEMBRANE_DISSIPATED] + gi] = SCc(SC_ACC + 6, gi);
        state_out[L.s[CB_PUMP_CYCLES] + gi] = SCc(SC_ACC + 7, gi);
        state_out[L.s[CB_PUMP_DISSIPATED] + gi] = SCc(SC_ACC + 8, gi);
        state_out[L.s[CB_METABOLIC_WORK] + gi] = SCc(SC_ACC + 9, gi);
        if constexpr (NCH > 0) {
          for (int q = 0; q < NCH; ++q) {
            state_out[L.s[CB_CHANNEL_TRANSFERRED] + q * C + gi] = CH(q, 0, gi);
            state_out[L.s[CB_CHANNEL_DISSIPATED] + q * C + gi] = CH(q, 1, gi);
            for (int r = 0; r < 2; ++r) {
              state_out[L.s[CB_CHANNEL_GATE] + (r * NCH + q) * C + gi] = CH(q, 2 + r, gi);
              CH(q, 6 + r, gi) = CH(q, 4 + r, gi);   // end targets -> start
              CH(q, 8 + r, gi) = CH(q, 10 + r, gi);  // end time constants -> start
            }
          }
        }
      }
      for (int el = tid; el < ne; el += BLOCK) {
        const long long ge = e0 + el;
        if (sRef[P.cell_world[c0 + P.isnd[ge]]]) continue;
        for (int s = 0; s < 3; ++s)
          state_out[L.s[CB_JUNCTION_TRANSFERRED] + s * E + ge] = SCe(SE_ACC + s, ge);
        state_out[L.s[CB_JUNCTION_DISSIPATED] + ge] = SCe(SE_ACC + 3, ge);
        state_out[L.s[CB_JUNCTION_GATE] + ge] = SCe(SE_ACC + 4, ge);
      }
      if (tid == 0) {
        int live = 0;
        for (int wl = 0; wl < nw; ++wl) live += sRef[wl] == 0u;
        sLive = live;
      }
      __syncthreads();
      if (sLive == 0) break;
    }
    // World outputs.
    for (int wl = tid; wl < nw; wl += BLOCK) {
      const int w = w0 + wl;
      const double *r = sWL + 8 * wl;
      for (int s = 0; s < 3; ++s) state_out[L.s[CB_RESERVOIR_SUPPLIED] + s * (long long)T.W + w] = r[s];
      state_out[L.s[CB_ELECTRODE_CHARGE] + w] = r[3];
      state_out[L.s[CB_RESERVOIR_WORK] + w] = r[4];
      state_out[L.s[CB_ELECTRODE_WORK] + w] = r[5];
      world_status[w] = sRef[wl];
      if (accepted_steps) accepted_steps[w] = sTaken[wl];
    }
    __syncthreads();
  }
}
