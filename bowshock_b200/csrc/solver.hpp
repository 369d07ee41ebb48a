// Host side of the GPU solve: a batch of cases (an engine is a batch of one)
// with its device arenas, its CUDA stream and the launches of the fused
// kernels, in the state type R (double: FP64 state and residual with the
// FP32 LU-SGS operator; float: the reference GPU engine's all-FP32 field).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "bowshock.h"
#include "host/metrics.hpp"

namespace bs {

struct HostCase {
  bs_config cfg{};
  std::vector<double> x, y;  // grid nodes
  Metrics64 m;
};

// Validates a configuration like validateGrid2DConfig (src/solver/config.ts:35-55)
// and the GPU engine's own checks (src/engine-gpu/euler2d-gpu.ts:217-239).
std::string validate_config(const bs_config& c);

// Per-case result of a batched steady solve.
struct CaseResult {
  int status = BS_OK;
  int64_t steps = 0;
  double residual = 0;
  double initial_residual = 0;
};

class SolverBase {
 public:
  virtual ~SolverBase() = default;
  virtual int n_cases() const = 0;
  virtual const HostCase& host_case(int c) const = 0;
  // All of these return a bs_status and set the error message on failure.
  virtual bs_status set_primitives(int c, const double* prim) = 0;
  virtual bs_status iterate(int steps) = 0;
  virtual bs_status iterate_implicit(int steps, double cfl_max, double omega, double growth) = 0;
  // As iterate_implicit with the Anderson settings applied and the
  // acceleration's history kept between calls (reset when the state or the
  // settings change).
  virtual bs_status iterate_accelerated(int steps, double cfl_max, double omega, double growth) = 0;
  // 64: two-float metrics in the residual (FP32 values and their FP32 low
  // parts); 32: FP32 metrics (the default).
  virtual bs_status set_metric_precision(int bits) = 0;
  virtual bs_status set_implicit_cfl(double cfl) = 0;
  virtual bs_status residual_norms(double* norms) = 0;
  virtual bs_status residual(int c, double* out) = 0;
  virtual bs_status time_steps(int c, double* out) = 0;
  virtual bs_status boundary_fluxes(int c, int side, bs_face_flux* out) = 0;
  virtual bs_status forebody_drag(int c, double p_inf, double q_inf, double base_radius,
                                  double* drag) = 0;
  virtual bs_status read_state(int c, float* out) = 0;
  virtual bs_status read_primitives(int c, double* out) = 0;
  virtual bs_status solve(int method, double cfl, double omega, double tolerance, int relative,
                          int max_steps, int check_every, std::vector<CaseResult>& results) = 0;
  virtual bs_status set_free_stream() = 0;
  virtual bs_status kernel_times(int method, double cfl, double omega, int iterations,
                                 double* ms) = 0;
  // Chooses how many lanes (concurrent groups of cases) the batch runs, by
  // timing `steps` steps with each candidate; the state is unchanged.
  virtual bs_status autotune(int method, int steps, double cfl, double omega, int* lanes,
                             double* ms_per_step) = 0;
  virtual int lanes() const = 0;
  // Sets the number of lanes (1 .. min(cases, 64)), as autotune would.
  virtual bs_status set_lanes(int lanes) = 0;
  // Which cases later iterate calls advance (1 active, 0 frozen); a solve
  // sets its own.
  virtual bs_status set_active(const int* flags) = 0;
  // Case c's display field (0 schlieren, 1 Mach, 2 Cp, 3 density ratio) per
  // cell, computed on the GPU (free: the free stream's primitives).
  virtual bs_status flow_field(int c, int field, const bs_primitive& free, double length, double* out) = 0;
  virtual int64_t steps(int c) const = 0;
  virtual cudaStream_t stream() const = 0;
  // Device time of the last solve, milliseconds (CUDA events on the stream).
  virtual double last_solve_ms() const = 0;
  // Kernel launches made by the last solve.
  virtual int64_t last_solve_launches() const = 0;
  // Anderson acceleration of the LU-SGS steps of later solves: `depth`
  // differences kept (0: plain steps), after `plain_steps` plain steps.
  virtual bs_status set_anderson(int depth, int plain_steps) = 0;
  // Per case, the times the last solve's acceleration forgot its history.
  virtual bs_status anderson_restarts(int* out) = 0;
  // Polls each bounded wait of later LU-SGS sweeps makes before it gives up
  // (-1: the default bound); the drain after a give-up keeps the default.
  virtual bs_status set_sweep_wait_limit(int polls) = 0;
  // The residual pass's tile shape (bsd::tile_shape index, -1 the default),
  // which autotune also chooses.
  virtual bs_status set_tile_shape(int shape) = 0;
  virtual int tile_shape() const = 0;
  // Whether an LU-SGS step's residual pass applies the previous step's
  // update as it reads (two launches a step) or a separate update kernel
  // follows each sweep (three), which autotune also chooses.
  virtual bs_status set_fused_update(bool fused) = 0;
  virtual bool fused_update() const = 0;
};

// Cells along i and j and threads of a residual-pass tile shape (-1: the
// default shape).
void tile_dims(int shape, int32_t* ti, int32_t* tj, int32_t* threads);

// precision: 64 (FP64 state and residual, FP32 LU-SGS operator) or 32 (all FP32).
bs_status make_solver(std::vector<HostCase>&& cases, int precision,
                      std::unique_ptr<SolverBase>& out);

}  // namespace bs
