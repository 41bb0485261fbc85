// handle.h - the bound batch (cb_tissue) as the library's translation units share it: its
// device views, launch choices, packed work items and owned allocations, and the error helpers
// behind cb_last_error.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "laws.cuh"

namespace cbk {

constexpr int kPackedMaxWorlds = 32;  // worlds per work item of the packed kernel

struct Packed {
  int n_items;
  int cap;                      // cells per item (shared exchange arrays)
  const int *order;             // [n_items] queue order, largest item first
  const int *item_world0;       // [n_items + 1] first world of each item
  const int *cell_world;        // [C] item-local world of each cell
  const int *isnd, *ircv;       // [E] item-local junction endpoints
  const int *iadj;              // [2E] item-local junction codes (edge << 1 | receiver)
  unsigned int *queue;          // ticket counter, zero at launch
  double *sc;                   // scratch: cell fields [SC_FIELDS][C], then edge fields [SE_][E]
};

// Set the calling thread's error text (cb_last_error) and return `code`.
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);
const char *last_error();

struct N2Plan;  // n2_step.cu

}  // namespace cbk

struct cb_tissue;

namespace cbk {
// The N2 method (n2_step.cu): n_steps steps of every world, device buffers (cb_step's contract).
int n2_step(cb_tissue *t, const double *state_in, double *state_out, double dt,
            const double *control, int n_steps, uint32_t *world_status, int32_t *accepted_steps,
            cudaStream_t stream, bool mix);
void n2_release(cb_tissue *t);
// The ROS2 method (n2_step.cu, on N2's factor plan; with mix its FP32-factor form), or with rk4
// the classical RK4 of the same right-hand side in the same kernel: n_steps steps of every world.
int ros2_step(cb_tissue *t, const double *state_in, double *state_out, double dt,
              const double *control, int n_steps, uint32_t *world_status,
              int32_t *accepted_steps, cudaStream_t stream, bool rk4, bool mix);
// One ROS2 step that also records what the reverse needs (R2Tape, n2_common.cuh).
struct R2Tape;
int ros2_step_tape(cb_tissue *t, const double *state_in, double *state_out, double dt,
                   const double *control, int n_steps, uint32_t *world_status,
                   int32_t *accepted_steps, cudaStream_t stream, bool rk4, bool mix,
                   const R2Tape &tape);
// The N2 plan's build (idempotent), for the ROS2 reverse.
int n2_build_plan(cb_tissue *t);
}  // namespace cbk

struct cb_tissue {
  int device = 0;
  int W = 0, C = 0, E = 0;
  int block = 0, ept = 0;
  int occupancy = 3;  // target resident 256-thread CTAs per SM (3, measured faster, or 2)
  cbk::Tissue t{};
  cbk::Layout layout{};
  long long state_total = 0, control_total = 0;
  std::vector<void *> owned;  // device allocations
  // The packed persistent kernel (uneven or large worlds): work items, scratch, ticket counter.
  bool packed = false;
  bool shared_ok = false;
  int packed_block = 1024;
  int grid_ctas = 0;
  cbk::Packed pk{};
  double *scratch = nullptr;
  size_t scratch_bytes = 0;
  // Buffers of the host-pointer entry point, allocated on first use.
  double *h_state = nullptr, *h_control = nullptr;
  uint32_t *h_status = nullptr;
  int32_t *h_taken = nullptr;
  // Streams of the host entry point's chunked pipeline (created on first use).
  cudaStream_t h_streams[4] = {};
  cudaEvent_t h_event = nullptr;
  bool h_streams_ready = false;
  // Patch and junction areas (m^2): the permeability prefactors and the adjoint's gradients.
  const double *area = nullptr;   // [C]
  const double *jarea = nullptr;  // [E]
  // Host copies of the contact graph for plans built after bind: world offsets and the
  // world-local junction endpoints.
  std::vector<long long> h_cell_offset, h_edge_offset;
  std::vector<int> h_snd, h_rcv;
  std::vector<double> h_temperature;  // [W] K
  // The open-channel block's device table (cb_set_channel_block), or null.
  double *blk_buf = nullptr;
  size_t blk_doubles = 0;
  // The N2 method's sparse-factor plan and workspace, built at its first step.
  cbk::N2Plan *n2 = nullptr;
};
