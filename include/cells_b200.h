/*
 * cells_b200.h - C ABI of the B200 tissue electrodiffusion step.
 *
 * The library replaces the reference's model-module protocol for the resolved pump-leak tissue
 * (Cells, src/cells/models/surface_pump.py and src/cells/models/surface_pump_v3.py):
 *
 *   initial_values(spec) -> (state, layout)      ~ cb_bind            (surface_pump.py:124-138,
 *                                                                      surface_tissue.py:135-257)
 *   checked_step(state, dt, control, p, active)  ~ cb_step / cb_step_host
 *                                                  (surface_pump.py:365-369 -> imex_step :259-362;
 *                                                   surface_pump_v3.py:3989 -> imex_step :3547)
 *   balances(state, p)                            ~ cb_balances       (surface_tissue.py:536-611,
 *                                                                      surface_kinetic.py:470-482)
 *   device_checks(prev, row, p, constants, steps) ~ cb_device_checks (surface_pump_v3.py:5572,
 *                                                                      surface_pump_checks.py:101)
 *
 * Worlds are packed back to back (see cells_b200/worlds.py): world w owns cells
 * cell_offset[w] .. cell_offset[w+1]-1 and junctions edge_offset[w] .. edge_offset[w+1]-1.
 * Every cell has one membrane patch that faces its world's one held bath (a reservoir outside
 * node clamped at bath_potential). Species are Na, K, Cl with valences +1, +1, -1; the pump is
 * the Na/K-ATPase (3 Na out, 2 K in) of laws/pumps/nak_atp_mass_action_positive.py.
 *
 * Error convention (the reference's: a traced step never raises; it returns valid=False and the
 * unchanged state, surface_pump_v3.py:3934): cb_step returns 0 when the launch is well formed and
 * reports each world's refusal in world_status (bit mask below); a refused world keeps its last
 * accepted state and takes no further steps in that call. A nonzero return is a configuration
 * or CUDA error; cb_last_error() gives the message. Nothing falls back to the CPU.
 *
 * Threading: a handle is used by one host thread at a time. Every device pointer argument must
 * be device memory of the handle's device; stream may be NULL (the legacy default stream).
 */
#ifndef CELLS_B200_H
#define CELLS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cb_tissue cb_tissue;

/* Per-world refusal bits (world_status). */
#define CB_WORLD_OK 0u
#define CB_WORLD_TRANSPORT 1u      /* concentration <= 0 or non-finite, |zF dV/RT| > 50, flux */
#define CB_WORLD_PUMP_DOMAIN 2u    /* nak_atp_mass_action_positive.domain_valid */
#define CB_WORLD_GATE_DOMAIN 4u    /* junction_voltage_relaxation.domain_valid */
#define CB_WORLD_CONTROL 8u        /* an availability outside [0, 1] or non-finite */
#define CB_WORLD_RESIDUAL 16u      /* stage charge residual above 3e-25 C + 2e-12 |q| */
#define CB_WORLD_DOMAIN 32u        /* accepted-state domain: amounts, gates, finite ledgers */
#define CB_WORLD_STIFF 64u         /* dt x membrane charge-relaxation rate > 1 at a stage
                                      (surface_pump_v3.membrane_rate, :4588) */
#define CB_WORLD_CHANNEL_DOMAIN 128u /* a channel population off its law's -120..60 mV domain
                                        or with non-finite kinetics (:848-858) */
#define CB_WORLD_LEDGER_COTANGENT 256u /* cb_step_vjp: a ledger field's cotangent was not zero;
                                          the gradients leave out the ledgers' dependence */
#define CB_WORLD_OPERATOR 512u     /* N2: the half-step prediction (non-positive concentration,
                                      non-finite slopes) or the operator (a non-positive pivot);
                                      field worlds: the same for the face-drift operator */
#define CB_WORLD_FIELD 1024u       /* field worlds: the start field's Newton on the floating
                                      offsets found no root within its bounds */

/* Return codes. */
#define CB_OK 0
#define CB_ERR_ARGUMENT 1
#define CB_ERR_LAYOUT 2
#define CB_ERR_CUDA 3
#define CB_ERR_UNSUPPORTED 4

/*
 * Packed world description (HOST pointers; copied at bind). Units: pL, fmol, m^2, m/s, F, K, V,
 * mM, J/mol, as the reference's definition schema. Arrays marked [3*X] are species-major
 * (Na block, then K, then Cl).
 */
typedef struct cb_tissue_desc {
  int32_t n_worlds;
  int64_t n_cells;              /* total over worlds */
  int64_t n_edges;              /* total over worlds */
  const int64_t *cell_offset;   /* [n_worlds+1] */
  const int64_t *edge_offset;   /* [n_worlds+1] */
  const double *temperature;    /* [W] K */
  const double *bath_amount;    /* [3*W] fmol, the held bath's reference amounts */
  const double *bath_volume;    /* [W] pL */
  const double *bath_potential; /* [W] V */
  const double *pump;           /* [7*W]: atp, adp, pi, km_na, km_k, km_atp (mM), dG0 (J/mol) */
  const double *volume;         /* [C] pL */
  const double *area;           /* [C] m^2 */
  const double *capacitance;    /* [C] F */
  const double *permeability;   /* [3*C] m/s */
  const double *pump_capacity;  /* [C] fmol cycles/s */
  const double *amount_reference; /* [3*C] fmol (the state stores increments over these) */
  const double *initial_charge; /* [C] C, the charge anchor of each cell */
  const int32_t *sender;        /* [E] world-local cell index */
  const int32_t *receiver;      /* [E] world-local cell index */
  const double *junction_area;  /* [E] m^2 */
  const double *junction_permeability; /* [3*E] m/s */
  const double *gate_threshold; /* [E] V */
  const double *gate_minimum;   /* [E] minimum open fraction */
  /* Voltage-gated channel populations (surface_pump_v3.channel_rates, :909-970): NCH slots per
   * cell, NCH = 0 (none) or 2. Slot arrays are [NCH*C], slot-major. Law codes: 0 Kv1.5 (m h),
   * 2 NaV1.2 (m^3 h) - the reference's catalogue codes - and 100 the Hodgkin-Huxley K n^4 law
   * of this library (no counterpart in the reference). One permeant species per population. */
  int32_t channel_slots;
  const int32_t *channel_code;        /* [NCH*C] */
  const int32_t *channel_species;     /* [NCH*C] 0 Na, 1 K, 2 Cl */
  const double *channel_permeability; /* [NCH*C] m/s, maximum permeability x relative */
  const double *channel_abundance;    /* [NCH*C] */
} cb_tissue_desc;

/* State fields in a packed state buffer, in this order (cb_state_layout gives each offset). */
enum cb_state_field {
  CB_AMOUNT_INCREMENT = 0,      /* [3][C] fmol over amount_reference (STATE amount_increment) */
  CB_MEMBRANE_TRANSFERRED,      /* [3][C] fmol, passive, outward-positive */
  CB_MEMBRANE_DISSIPATED,       /* [C] pJ */
  CB_PUMP_CYCLES,               /* [C] fmol cycles */
  CB_PUMP_DISSIPATED,           /* [C] pJ */
  CB_METABOLIC_WORK,            /* [C] pJ */
  CB_JUNCTION_TRANSFERRED,      /* [3][E] fmol, sender -> receiver */
  CB_JUNCTION_DISSIPATED,       /* [E] pJ */
  CB_JUNCTION_GATE,             /* [E] relative conductance g */
  CB_RESERVOIR_SUPPLIED,        /* [3][W] fmol into the finite system */
  CB_ELECTRODE_CHARGE,          /* [W] C */
  CB_RESERVOIR_WORK,            /* [W] pJ */
  CB_ELECTRODE_WORK,            /* [W] pJ */
  CB_CHANNEL_GATE,              /* [2][NCH][C] gate rows (m, h) of each population */
  CB_CHANNEL_TRANSFERRED,       /* [NCH][C] fmol of each population's permeant species */
  CB_CHANNEL_DISSIPATED,        /* [NCH][C] pJ */
  CB_STATE_FIELDS
};

/* Control fields (availabilities in [0,1]; SurfaceKineticControl, execution/schedule.py:18-22). */
enum cb_control_field {
  CB_CONTROL_MEMBRANE = 0, /* [C] */
  CB_CONTROL_JUNCTION,     /* [E] */
  CB_CONTROL_PUMP,         /* [C] */
  CB_CONTROL_CHANNEL,      /* [NCH][C] */
  CB_CONTROL_FIELDS
};

/* Step methods. */
#define CB_METHOD_ARS222 0 /* cells.solver.imex_ars222_face_electromigration@1 */
/* The same ARS(2,2,2) step with its constant-field fluxes in FP32 (this library's
 * cells_b200.solver.imex_ars222_mixed_fp32@1; no reference method): the Bernoulli pair's
 * exponential form and the membrane, channel and junction flux products in FP32 on FP64
 * concentration differences; the near-zero Bernoulli series, concentrations, their logarithms
 * and potentials, the pump, the channel and junction gate laws and the gates' updates, world
 * sums and every state and ledger accumulation in FP64. The amounts stay within 1e-8 (about
 * 1e-11) of the FP64 step's and the ledgers balance to 1e-12; the gates, which follow the
 * membrane voltage, within about 5e-8 of their scale, and the ledgers that integrate a flux carry
 * its FP32 rounding (about 1e-7 of their scale). Both kernels (one world per CTA, and the packed
 * kernel for uneven batches); not with an open-channel block. */
#define CB_METHOD_ARS222_MIXED 1
/* N2 (cells.solver.imex_ars222_implicit_conductances@1, models/surface_pump_v3.py:3547-3955 under
 * an N2 ID): ARS(2,2,2) with every patch's, channel population's and junction's slope
 * conductance dJ/d(dv), frozen at the step's half-way prediction (operator_time_conductances,
 * :2961-3029), in the implicit operator C + gamma dt L beside the capacitors; the remainders
 * J - W dv explicit; junction gates by their exponential update at the stages. The operator of
 * each world is factored every step by a sparse Cholesky on its contact graph (a minimum-degree
 * order and elimination-tree levels bound on the host at the first N2 step; left-looking by
 * levels on the device, one CTA per world). FP64. */
#define CB_METHOD_N2 2
/* N2 with its operator factored and substituted in FP32, the stage potentials recovered by FP64
 * iterative refinement of the charge residual against the FP64 operator (corrections until every
 * row is within 1e-3 of the stage's acceptance bound, at most 6); rates, slopes and every
 * accumulation in FP64 (this library's cells_b200.solver.imex_ars222_implicit_conductances_
 * mixed@1; no reference method). */
#define CB_METHOD_N2_MIXED 3
/* ROS2 (this library's cells_b200.solver.ros2_verwer@1; the reference has no Rosenbrock method
 * on its tissue path): the two-stage, second-order, L-stable Rosenbrock method of Verwer, Spee,
 * Blom and Hundsdorfer (gamma = 1 + 1/sqrt(2); W k1 = F(y), W k2 = F(y + h k1) - 2 k1,
 * y' = y + 3/2 h k1 + 1/2 h k2, W = I - gamma h J), the stage structure of the reference's
 * dense Rodas (numerics/rosenbrock_dense.py:123-141) on the held-bath step's whole right-hand
 * side. J at y: every route's slope conductance through each cell's dV/dn = z F/C, applied alike
 * to the amounts and the route ledgers (so the ledgers balance to rounding); each gate's
 * relaxation rate and, for channel gates, their voltage slope; nothing for the pump. Each world's
 * W reduces to (C + gamma h G) u = K sum_s z_s r_s in the cells' voltage rates (N2's operator
 * pattern and sparse factor plan): one factorisation and two solves per step, one CTA per world.
 * A world is refused (state kept) when an evaluation is invalid, the operator is not positive
 * definite or the new state leaves the domain; no explicit-stability refusal applies. FP64. */
#define CB_METHOD_ROS2 4
/* The reference's reference-run method: classical RK4 over the same whole right-hand side
 * (numerics/fixed_step.py:25-71 rk4_checked_step, taken by checked_step for an empty tableau,
 * models/surface_pump_v3.py:3989-4001): four evaluations, each of a state that must be valid,
 * y' = y + h/6 (k1 + 2 k2 + 2 k3 + k4) for every state field, the new state's domain checked.
 * No explicit-stability refusal (the reference's RK4 has none). One CTA per world (ROS2's kernel
 * without its operator). FP64. */
#define CB_METHOD_RK4 5
/* This library's cells_b200.solver.ros2_verwer_fp32_factor@1: CB_METHOD_ROS2 with its voltage
 * operator factored and both stage solves substituted in FP32 and no refinement; every rate,
 * slope, potential and accumulation stays FP64. ROS2 is a W-method: its order and its ledgers'
 * balance hold for any W, and the FP32 factor is the exact factor of a W within FP32 rounding of
 * the FP64 one, so the step stays second order and conservative. Measured against the FP64 ROS2
 * (tests/test_ros2_gpu.py): within 1e-8 scaled difference on every state field over hundreds of
 * steps, ledgers balanced to 1e-12. Half the factor's bytes: 1024-cell worlds' factor values fit
 * shared memory beside a second CTA. */
#define CB_METHOD_ROS2_MIXED 6

/*
 * Host symbolic bind (replaces initial_values' layout binding, surface_tissue.py:135-257 and
 * surface_field.bind :253-361): validates the packed description, builds each cell's junction
 * adjacency (CSR, edge order), uploads parameters to `device`. Worlds of up to 1024 cells.
 */
int cb_bind(const cb_tissue_desc *desc, int device, cb_tissue **out);
void cb_free(cb_tissue *t);

/* Kernel paths of cb_step: one world per CTA in shared memory (uniform worlds of up to 1024
 * cells), or the packed persistent kernel (work items of several worlds, up to 4096 cells each,
 * taken from a device queue; scratch allocated on first selection). cb_bind picks one; an
 * autotuner may override it. Block: CTA threads of the packed kernel (256, 512, 1024);
 * occupancy: resident 256-thread CTAs per SM the shared kernel's registers target (2 or 3). */
#define CB_KERNEL_SHARED 0
#define CB_KERNEL_PACKED 1
int cb_set_launch(cb_tissue *t, int kernel, int block, int occupancy);
int cb_get_launch(const cb_tissue *t, int *kernel, int *block, int *occupancy);

/* CTA threads of the ROS2 and RK4 kernel (CB_METHOD_ROS2, CB_METHOD_ROS2_MIXED, CB_METHOD_RK4) on
 * the batch's sparse factor plan: 128 (four CTAs per SM) or 256 (two); 0 restores the plan's own
 * choice (128 when no world's plan is staged in shared memory). The first call builds the plan
 * (device memory the handle keeps, as the first step of these methods does): make it outside any
 * stream capture. cb_get_sparse_launch reports the block in use (building the plan if needed).
 * An autotuner's knob (cells_b200.autotune.tune_sparse); no counterpart in the reference. */
int cb_set_sparse_launch(cb_tissue *t, int block);
int cb_get_sparse_launch(cb_tissue *t, int *block);

/* Offsets (in doubles) of each state field in a packed state buffer, and its total length. */
int cb_state_layout(const cb_tissue *t, int64_t offsets[CB_STATE_FIELDS], int64_t *total);
/* Offsets (in doubles) of each control field in a packed control buffer, and its total length. */
int cb_control_layout(const cb_tissue *t, int64_t offsets[CB_CONTROL_FIELDS], int64_t *total);

/*
 * n_steps steps of length dt (s) for every world (checked_step, repeated). state_in and
 * state_out may alias. DEVICE pointers. world_status [W] receives the refusal bits of the first
 * refused step (0 if all accepted); accepted_steps [W] (may be NULL) the steps each world took.
 */
int cb_step(cb_tissue *t, int method, const double *state_in, double *state_out, double dt,
            const double *control, int n_steps, uint32_t *world_status, int32_t *accepted_steps,
            void *stream);

/*
 * cb_step with HOST buffers: copies in, steps, copies out, synchronizes (end-to-end call). On the
 * one-world-per-CTA kernel (ARS(2,2,2), FP64 or mixed, 8 worlds or more) the worlds go in four
 * chunks on four streams of the handle, so one chunk's copies run beside another's steps; from
 * pinned host memory the copies then overlap the steps. Results equal cb_step's bit for bit;
 * the layout's padding in state_out is not written.
 */
int cb_step_host(cb_tissue *t, int method, const double *state_in, double *state_out, double dt,
                 const double *control, int n_steps, uint32_t *world_status,
                 int32_t *accepted_steps);

/*
 * Conservation ledgers of one packed state (DEVICE pointers), per world:
 * out[w*8 + k] = max |residual| of ledger k: 0 local material (fmol), 1 bath material (fmol),
 * 2 world total material (fmol), 3 electrode charge (C), 4 global charge (C),
 * 5 reservoir work (pJ), 6 electrode work (pJ), 7 metabolic work (pJ).
 */
int cb_balances(cb_tissue *t, const double *state, double *out, void *stream);

/*
 * The accepted-row checks of one row against its predecessor (DEVICE pointers; replaces @3's
 * device_checks, models/surface_pump_v3.py:5572-5597, which evaluates
 * models/surface_pump_checks.row_checks :101-192 on the device). steps is the number of steps
 * accepted up to row (the rounding allowance of every ledger is 2.5 eps x steps x the magnitudes
 * rounded into it, surface_pump.ledger_limits :752-800); material_atol [3] (HOST, fmol per
 * species) and energy_rtol are the solver's tolerances (@3's device_check_constants).
 * failed [W]: bit k set when check k failed, in the order 0 domain, 1 local material,
 * 2 bath material, 3 world total material, 4 capacitor charge, 5 electrode charge,
 * 6 global charge, 7 energy, 8 reservoir work, 9 electrode work, 10 metabolic work,
 * 11 dissipation (negative, or decreasing since previous). values [W*12]: the max |residual| of
 * the ten ledgers in that order (fmol, C, pJ), then the energy residual over its flows and the
 * global-charge residual over its bound (DEVICE_DIAGNOSTICS).
 */
int cb_device_checks(cb_tissue *t, const double *previous, const double *row, int64_t steps,
                     const double *material_atol, double energy_rtol, uint32_t *failed,
                     double *values, void *stream);

/*
 * cb_device_checks with each world's own accepted-step count (steps: DEVICE int64 [W], each
 * non-negative), as the reference's vector windows give every world its own first_step
 * (execution/vector_windows.py:348-410, `checked(current, updated, params, constants,
 * first_step + row)`). A world's result equals cb_device_checks' at that world's count, bit for
 * bit.
 */
int cb_device_checks_each(cb_tissue *t, const double *previous, const double *row,
                          const int64_t *steps, const double *material_atol, double energy_rtol,
                          uint32_t *failed, double *values, void *stream);

/*
 * Copy every state element of each world w with mask[w] != 0 from src to dst (packed states,
 * DEVICE pointers; mask DEVICE int32 [W]); other worlds' elements and the layout's padding are
 * left as they are. One CTA per world, so a copy costs only the masked worlds' bytes. The
 * vector window's selects (`jnp.where(accept, updated, current)` and the stored rows,
 * execution/vector_windows.py:393-402) as copies of the worlds that need them.
 */
int cb_copy_worlds(cb_tissue *t, const int32_t *mask, const double *src, double *dst,
                   void *stream);

/*
 * One row of a vector window (execution/vector_windows.py:379-404) in one launch: the
 * accepted-row checks of `row` against `previous` (as cb_device_checks, each world at its own
 * count first_step[w] + row_index, or first_all + row_index where first_step is NULL) and each
 * world's bookkeeping. Row 0 is the window start (row == previous, step_status unused): ok[w] =
 * no failure, first[w] = -1 or 0, bits[w] = its failure bits, maxima = its diagnostics (0 where
 * failing). Row j > 0 (step_status: the row's cb_step status): a world still live (ok[w] and
 * j <= counts[w]) fails at j with bits = 1 (refused step) or failed << 1 (FAILURE_SHIFT), or is
 * accepted and raises its maxima; keep[w] = 0 for an accepted world, else 1 (its state stays:
 * cb_copy_worlds(keep, current, row) then makes `row` the window's next current state).
 * DEVICE arrays: counts int64 [W], ok int32 [W], first int32 [W], bits int64 [W], maxima
 * float64 [W*12], keep int32 [W], first_step int64 [W] or NULL.
 */
int cb_window_row(cb_tissue *t, const double *previous, const double *row, int32_t row_index,
                  const int64_t *first_step, int64_t first_all, const double *material_atol,
                  double energy_rtol, const uint32_t *step_status, const int64_t *counts,
                  int32_t *ok, int32_t *first, int64_t *bits, double *maxima, int32_t *keep,
                  void *stream);

/*
 * Store each world's state from src into observation row slot[w] of `rows` (n_rows rows of the
 * packed state's length) where keep[w] == 0 and 0 <= slot[w] < n_rows: the window's stored rows
 * (execution/vector_windows.py:400-402). DEVICE pointers; slot int64 [W].
 */
int cb_store_worlds(cb_tissue *t, const int32_t *keep, const int64_t *slot, const double *src,
                    double *rows, int32_t n_rows, void *stream);

/*
 * cb_step with method CB_METHOD_ARS222 (the FP64 ARS(2,2,2) step; there is no method argument)
 * for a handle bound for the packed kernel, with the kernel's per-call scratch (stage
 * accumulators, junction fluxes, world-sum terms, the work-queue counter) taken from a 16 MiB
 * array that the library holds on every GPU it is loaded on, so the call allocates nothing. No
 * counterpart in the reference: it exists for callers that may not allocate device memory
 * while a step runs, such as a plugin inside a host runtime (an XLA/JAX custom call) that hands
 * it only its input and output buffers, or a process whose device memory another allocator has
 * already reserved. It saves no memory: the handle still holds what cb_bind allocated. A batch
 * needs (26 + 12 NCH) C + 9 E doubles of scratch and must fit 2^21 - 32 doubles; a larger batch
 * is refused (CB_ERR_UNSUPPORTED) and should use cb_step. The array's device address is looked
 * up whenever a handle is bound on the device, and by the first call on a device if no bind
 * has; make that first call before any stream capture. Every call shares the array, which keeps
 * the last call's contents: calls whose kernels overlap on a GPU race and must be serialised by
 * the caller. DEVICE pointers, as cb_step.
 */
int cb_step_packed_static(cb_tissue *t, const double *state_in, double *state_out, double dt,
                          const double *control, int n_steps, uint32_t *world_status,
                          int32_t *accepted_steps, void *stream);

/*
 * Reverse-mode derivative of n_steps FP64 ARS(2,2,2) steps (CB_METHOD_ARS222) from state_in.
 * The reference has no reverse-mode adjoint of its time loop: its loss gradients would be
 * jax.grad of the composed checked_step (models/surface_pump.py:365, models/surface_pump_v3.py:
 * 3989), which this computes for the held-bath step by the transposed linearisation of each
 * stage in reverse order. cot_out is the cotangent of the state after the n_steps steps and
 * cot_in receives the cotangent of state_in (both in the state layout; they may alias). Only the
 * amount increments, junction gates and channel gates carry the dynamics: the ledgers never feed
 * back, so their cotangents pass through unchanged and must be zero for the gradients to be
 * complete (a world whose ledger cotangents are not zero gets CB_WORLD_LEDGER_COTANGENT). The
 * gradients of the loss with respect to the permeabilities (m/s) are ADDED to grad_membrane
 * [3*C], grad_junction [3*E] and grad_channel [NCH*C] (NULL when NCH = 0). A step the forward
 * refused for a world is the identity for it (the world's state did not move) and adds nothing.
 * The call recomputes the n_steps steps with cb_step, one step per launch, keeping every state in
 * `workspace` (cb_vjp_workspace bytes for n_steps, 256-byte aligned, device memory the caller
 * owns), then runs one reverse launch; callers checkpoint long trajectories by calling it once
 * per segment, last segment first. world_status[w]: the forward's refusal bits OR-ed over the
 * steps, plus CB_WORLD_LEDGER_COTANGENT. DEVICE pointers; stream-ordered, no host sync.
 */
int cb_step_vjp(cb_tissue *t, const double *state_in, double dt, const double *control,
                int n_steps, const double *cot_out, double *cot_in, double *grad_membrane,
                double *grad_junction, double *grad_channel, void *workspace,
                size_t workspace_bytes, uint32_t *world_status, void *stream);
/* Bytes of cb_step_vjp's workspace for n_steps steps. */
int cb_vjp_workspace(const cb_tissue *t, int n_steps, size_t *bytes);

/*
 * The reverse-mode derivative of n_steps steps of `method`: CB_METHOD_ARS222 (cb_step_vjp) or
 * CB_METHOD_ROS2, the same arguments and contract as cb_step_vjp. Replaces jax.vjp / jax.grad of
 * the composed checked_step (models/surface_pump_v3.py:3989) for this library's ROS2 method, which
 * has no counterpart in the reference (its only Rosenbrock integrator is the dense Rodas4 of
 * numerics/rosenbrock_dense.py:123-141). For ROS2 the call first runs the n_steps steps forward,
 * one step per launch, keeping in the workspace every state and each step's record: the factor of
 * its voltage operator M = C + gamma h (G_patch + L(G_junction)), both stage solves' voltage
 * rates, k1's dynamic rows and k2's gate rows. The reverse launch then transposes each step: its
 * two stage solves reuse the step's recorded factor (M is symmetric), and the W-matrix's own
 * dependence on the state and the permeabilities enters through the laws' second derivatives.
 * Only the amounts, junction gates and channel gates carry the dynamics (ledger cotangents must be
 * zero; CB_WORLD_LEDGER_COTANGENT otherwise). Gradients are ADDED to grad_membrane [3*C],
 * grad_junction [3*E], grad_channel [NCH*C]. DEVICE pointers; stream-ordered, no host sync.
 */
int cb_step_vjp_method(cb_tissue *t, int method, const double *state_in, double dt,
                       const double *control, int n_steps, const double *cot_out,
                       double *cot_in, double *grad_membrane, double *grad_junction,
                       double *grad_channel, void *workspace, size_t workspace_bytes,
                       uint32_t *world_status, void *stream);
/* Bytes of cb_step_vjp_method's workspace for n_steps steps of `method`. For CB_METHOD_ROS2 the
 * first call builds the batch's sparse factor plan (device memory the handle keeps, as the first
 * ROS2 step does): make it outside any stream capture. */
int cb_vjp_workspace_method(cb_tissue *t, int method, int n_steps, size_t *bytes);

/*
 * Replace the bound permeabilities (m/s) from DEVICE arrays: membrane [3*C], junction [3*E],
 * channel [NCH*C]; a NULL array keeps what is bound. The prefactors are formed by the same device
 * code as cb_bind's (area * P / 1e-15), so a step after this call is bit-identical to a step of a
 * handle bound with these permeabilities. The reference rebuilds its parameter pytree for new
 * permeabilities (models/surface_tissue.py:135-257 parses them); this is that rebuild for the
 * permeabilities alone, without a host round trip. Values must be finite and non-negative (the
 * bind's checks are not repeated on the device). Stream-ordered.
 */
int cb_set_permeability(cb_tissue *t, const double *membrane, const double *junction,
                        const double *channel, void *stream);

/*
 * Open-channel block of the channel populations (cells.channel_block.open_channel_block_weighted_modes@1,
 * laws/channels/open_channel_block.py; @3's channel_rates :958-960, channel_block :1003-1036,
 * channel_block_terms :1051-1126). Replaces the reference's block layout fields
 * (surface_pump_v3.block_initial_values :599-615): channel_block_weight, channel_block_k0_mM,
 * channel_block_steepness [modes][NCH*C] and channel_block_concentration_mM [NCH*C], host
 * arrays in the channel slots' order. An unblocked population in a blocked batch takes weights
 * (1, 0, ...), K(0) 1, steepness 0 and concentration 0 (u = 1 exactly), as the reference's layout
 * gives it. The block reads the patch voltage (no voltage shift). The step multiplies each
 * population's flux by its unblocked fraction u, takes T_V = u G_max + |I_free| du/dV in place of
 * G_max in the explicit-stability rule, and refuses a world where a K or c_B + K is not a finite
 * normal number (bit CB_WORLD_CHANNEL_DOMAIN). A blocked batch runs on the packed kernel (a
 * shared-kernel handle is switched to it), FP64 ARS(2,2,2) only: N2 (as the reference refuses
 * it), the mixed step and the adjoint return CB_ERR_UNSUPPORTED. modes = 0 removes the block.
 * Domain checks as the reference's parse: weights in [0, 1] summing to 1 within 8 ulps, K(0) in
 * [1e-15, 1e15] mM, |steepness| <= 8, the blocker in [0, 1e3] mM; modes at most 4. Host call
 * (it may allocate the device table and synchronizes): not inside a stream capture, and not while
 * a step of this handle runs.
 */
int cb_set_channel_block(cb_tissue *t, int32_t modes, const double *weight,
                         const double *k0_mM, const double *steepness,
                         const double *concentration_mM);

/* The device's FP64 fused multiply-add rate (FLOP/s), measured by one launch of independent FMA
 * chains over every SM (iterations rounds per thread, CUDA events around it; ms its duration):
 * the denominator of an FP64-pipe fraction. No counterpart in the reference. Allocates and
 * synchronizes: a measurement call, not for a step's path. */
int cb_probe_fp64(int device, int64_t iterations, double *flops_per_second, double *milliseconds);

/* Message of the last error on this thread. */
const char *cb_last_error(void);
/* Library version string. */
const char *cb_version(void);

/*
 * Field worlds: tissues whose cells face a resolved extracellular grid (cells_b200/field_worlds.py)
 * instead of one held bath. Replaces the reference's model-module protocol for
 * cells.model.resolved_pump_tissue@1 with outside nodes and faces under
 * cells.solver.imex_ars222_face_electromigration@1 (models/surface_pump.py:158-369, the field
 * closure of numerics/surface_field.py:253-855, the face operator of numerics/surface_imex.py).
 *
 * Every world of a batch shares one topology: N cells, O outside nodes, E junctions, F faces;
 * cell i's one membrane faces outside node cell_node[i]; at most one cell per node and none on a
 * held node; held (reservoir) nodes have no membrane. Per-world parameters are world-major
 * ([W*N] etc.; species arrays [3][W*X]). The start field is the reference's capacitor reduction
 * with a damped Newton on the floating offsets (one per capacitor component: a cell with its node,
 * or a lone node), here a chord Newton whose matrix is the face conductance Laplacian; the stage
 * potentials solve (C + gamma dt L) phi = q with each cell eliminated into its node. Both
 * matrices are the face Laplacian on the free nodes: one nested-dissection plan, one sparse
 * Cholesky per matrix per world per step.
 */
typedef struct cb_field cb_field;
typedef struct {
  int32_t worlds, cells, nodes, junctions, faces;
  const int64_t *cell_node;        /* [N] */
  const int64_t *junction_sender;  /* [E] cells */
  const int64_t *junction_receiver;
  const int64_t *face_sender;      /* [F] outside nodes */
  const int64_t *face_receiver;
  const uint8_t *reservoir;        /* [O] held nodes */
  const double *temperature;       /* [W] K */
  const double *pump;              /* [7][W] atp, adp, pi (mM), km_na, km_k, km_atp (mM), dG0 */
  const double *volume;            /* [W*N] pL */
  const double *area;              /* [W*N] m^2 */
  const double *capacitance;       /* [W*N] F */
  const double *permeability;      /* [3][W*N] m/s */
  const double *pump_capacity;     /* [W*N] fmol/s */
  const double *amount;            /* [3][W*N] reference amounts, fmol */
  const double *initial_charge;    /* [W*N] C */
  const double *junction_area;     /* [W*E] */
  const double *junction_permeability; /* [3][W*E] */
  const double *gate_threshold;    /* [W*E] V */
  const double *gate_minimum;      /* [W*E] */
  const double *outside_volume;    /* [W*O] pL */
  const double *outside_amount;    /* [3][W*O] fmol */
  const double *outside_charge;    /* [W*O] C */
  const double *boundary_V;        /* [W*O] held potentials (0 on free nodes) */
  const double *face_factor;       /* [3][W*F] D A / L, m^3/s */
} cb_field_desc;

/* State fields of a field batch (offsets from cb_field_state_layout), the reference's STATE_TYPE
 * without channels: cell fields [3][W*N] or [W*N], node fields [3][W*O] or [W*O], junction
 * fields [3][W*E] or [W*E], face fields [3][W*F] or [W*F]. */
enum {
  CB_FIELD_AMOUNT_INCREMENT = 0, CB_FIELD_EXTRACELLULAR_INCREMENT, CB_FIELD_MEMBRANE_TRANSFERRED,
  CB_FIELD_JUNCTION_TRANSFERRED, CB_FIELD_FACE_TRANSFERRED, CB_FIELD_RESERVOIR_SUPPLIED,
  CB_FIELD_MEMBRANE_DISSIPATED, CB_FIELD_JUNCTION_DISSIPATED, CB_FIELD_FACE_DISSIPATED,
  CB_FIELD_ELECTRODE_CHARGE, CB_FIELD_RESERVOIR_WORK, CB_FIELD_ELECTRODE_WORK,
  CB_FIELD_JUNCTION_GATE, CB_FIELD_PUMP_CYCLES, CB_FIELD_PUMP_DISSIPATED, CB_FIELD_METABOLIC_WORK,
  CB_FIELD_STATE_FIELDS
};

/* Bind (host analysis: components, the nested-dissection plan of the free nodes' Laplacian;
 * uploads) on `device`. Refuses (CB_ERR_LAYOUT) a topology outside the contract above. */
int cb_field_bind(const cb_field_desc *desc, int device, cb_field **out);
void cb_field_free(cb_field *f);
int cb_field_state_layout(const cb_field *f, int64_t offsets[CB_FIELD_STATE_FIELDS],
                          int64_t *total);
/* The bound solver's sizes: info[0] free nodes (unknowns), [1] supernodes (fronts), [2] their
 * levels, [3] factor doubles per world, [4] update-matrix doubles per world, [5] update-vector
 * doubles per world, [6] shared memory bytes per CTA, [7] scratch bytes (all worlds). */
int cb_field_info(const cb_field *f, int64_t info[8]);
/* Arithmetic of the bound plan per world (an FMA counts 2): out[0] flops of one factorisation
 * (panels and update matrices), out[1] of one solve (forward and back substitution). */
int cb_field_flops(const cb_field *f, double out[2]);
/* The factor plan's levels (leaves first): kinds[l] (l < capacity; kinds may be NULL) = 0 when
 * level l's fronts go one per warp (factor_warps, forward_warps, backward_warps), 1 when one per
 * CTA (factor_group, forward_group, backward_group: separators whose front block exceeds 1280
 * doubles or whose front has more than 256 rows), 2 when one per CTA with the wide factor (such
 * a level whose widest front has 48 columns or more). Returns the number of levels (-1: null
 * handle). */
int32_t cb_field_levels(const cb_field *f, int32_t *kinds, int32_t capacity);
/* Control: membrane [W*N], junction [W*E], pump [W*N] availabilities, back to back. */
int64_t cb_field_control_length(const cb_field *f);
/* n_steps ARS(2,2,2) steps of every world (checked_step repeated; a refused world keeps its
 * last accepted state and stops). DEVICE pointers; state_in and state_out may alias. Each step is
 * a sequence of launches on `stream` (per-world phases around the factor and substitution levels);
 * the Newton's corrections continue while some world's does, which the call reads back, so it
 * synchronizes `stream` once per correction. */
int cb_field_step(cb_field *f, const double *state_in, double *state_out, double dt,
                  const double *control, int n_steps, uint32_t *world_status,
                  int32_t *accepted_steps, void *stream);
/* Kernels launched by the handle's last cb_field_step call. */
int64_t cb_field_launches(const cb_field *f);
/* The handle's last cb_field_step call: out[0] kernels launched, out[1] factorisations (every
 * world's, counted once per level sweep), out[2] solves (forward and back sweeps). */
int cb_field_counts(const cb_field *f, int64_t out[3]);
/* cb_field_step with HOST buffers: copies in, steps, copies out, synchronizes. The device copies
 * are allocated by the handle's first host call and kept until cb_field_free. */
int cb_field_step_host(cb_field *f, const double *state_in, double *state_out, double dt,
                       const double *control, int n_steps, uint32_t *world_status,
                       int32_t *accepted_steps);

#ifdef __cplusplus
}
#endif

#endif /* CELLS_B200_H */
