// C ABI of the single-grid engine (include/bowshock.h): the GpuEuler2D
// surface (src/engine-gpu/euler2d-gpu.ts:183-723) over a solver batch of one
// case. Each engine owns its CUDA stream; overlapping calls on one engine
// return BS_BUSY instead of interleaving (ExclusiveRunner,
// src/engine-gpu/gpu-common.ts:122-140).
#include <cuda_runtime.h>

#include <atomic>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "bowshock.h"
#include "common.hpp"
#include "solver.hpp"

struct bs_engine {
  std::unique_ptr<bs::SolverBase> solver;
  std::atomic<bool> busy{false};
};

namespace {

// Holds the engine for the duration of one call.
class Exclusive {
 public:
  explicit Exclusive(bs_engine* e) : e_(e) {
    bool expected = false;
    owned_ = e != nullptr && e->busy.compare_exchange_strong(expected, true);
  }
  ~Exclusive() {
    if (owned_) e_->busy.store(false);
  }
  bs_status status() const {
    if (e_ == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null engine");
    if (!owned_) return bs::fail(BS_BUSY, "the engine is running another operation");
    return BS_OK;
  }

 private:
  bs_engine* e_;
  bool owned_ = false;
};

#define BS_ENGINE_CALL(engine, body)     \
  do {                                   \
    Exclusive guard_(engine);            \
    const bs_status s_ = guard_.status(); \
    if (s_ != BS_OK) return s_;          \
    body;                                \
  } while (0)

}  // namespace

namespace bs {
// Builds a HostCase from a configuration and its nodes: validation and FP64 metrics.
bs_status make_host_case(const bs_config* config, const double* x, const double* y, HostCase& h) {
  if (config == nullptr || x == nullptr || y == nullptr)
    return fail(BS_INVALID_ARGUMENT, "null argument");
  const std::string e = validate_config(*config);
  if (!e.empty()) return fail(BS_INVALID_ARGUMENT, e);
  h.cfg = *config;
  const size_t nn = size_t(config->ni + 1) * (config->nj + 1);
  h.x.assign(x, x + nn);
  h.y.assign(y, y + nn);
  const std::string m = compute_metrics64(config->ni, config->nj, x, y,
                                          config->geometry == BS_AXISYMMETRIC, h.m);
  if (!m.empty()) return fail(BS_INVALID_ARGUMENT, m);
  return BS_OK;
}
}  // namespace bs

extern "C" {

bs_status bs_device_count(int32_t* count) {
  if (count == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
  int n = 0;
  const cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *count = 0;
    return BS_OK;
  }
  *count = n;
  return BS_OK;
}

bs_status bs_set_device(int32_t device) {
  const cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return bs::fail(BS_INVALID_ARGUMENT, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  }
  return BS_OK;
}

bs_status bs_engine_create_ex(const bs_config* config, const double* x, const double* y,
                              int32_t precision, bs_engine** out) {
  if (out == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  std::vector<bs::HostCase> cases(1);
  const bs_status s = bs::make_host_case(config, x, y, cases[0]);
  if (s != BS_OK) return s;
  auto* e = new (std::nothrow) bs_engine;
  if (e == nullptr) return bs::fail(BS_MEMORY_LIMIT, "out of host memory");
  const bs_status st = bs::make_solver(std::move(cases), precision, e->solver);
  if (st != BS_OK) {
    delete e;
    return st;
  }
  *out = e;
  return BS_OK;
}

bs_status bs_engine_create(const bs_config* config, const double* x, const double* y,
                           bs_engine** out) {
  return bs_engine_create_ex(config, x, y, BS_PRECISION_FP64, out);
}

bs_status bs_engine_destroy(bs_engine* engine) {
  if (engine == nullptr) return BS_OK;
  bool expected = false;
  if (!engine->busy.compare_exchange_strong(expected, true))
    return bs::fail(BS_BUSY, "the engine is running another operation");
  delete engine;
  return BS_OK;
}

bs_status bs_engine_centroids(bs_engine* engine, double* cx, double* cy) {
  BS_ENGINE_CALL(engine, {
    if (cx == nullptr || cy == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    const bs::Metrics64& m = engine->solver->host_case(0).m;
    std::copy(m.cx.begin(), m.cx.end(), cx);
    std::copy(m.cy.begin(), m.cy.end(), cy);
    return BS_OK;
  });
}

bs_status bs_engine_set_primitives(bs_engine* engine, const double* primitives) {
  BS_ENGINE_CALL(engine, {
    if (primitives == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    return engine->solver->set_primitives(0, primitives);
  });
}

bs_status bs_engine_iterate(bs_engine* engine, int32_t steps) {
  BS_ENGINE_CALL(engine, { return engine->solver->iterate(steps); });
}

bs_status bs_engine_set_implicit_cfl(bs_engine* engine, double cfl) {
  BS_ENGINE_CALL(engine, { return engine->solver->set_implicit_cfl(cfl); });
}

bs_status bs_engine_iterate_implicit(bs_engine* engine, int32_t steps, double cfl_max,
                                     double omega, double growth) {
  BS_ENGINE_CALL(engine, { return engine->solver->iterate_implicit(steps, cfl_max, omega, growth); });
}

bs_status bs_engine_density_residual_norm(bs_engine* engine, double* norm) {
  BS_ENGINE_CALL(engine, {
    if (norm == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    return engine->solver->residual_norms(norm);
  });
}

bs_status bs_engine_residual(bs_engine* engine, double* residual) {
  BS_ENGINE_CALL(engine, {
    if (residual == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    return engine->solver->residual(0, residual);
  });
}

bs_status bs_engine_time_steps(bs_engine* engine, double* dt) {
  BS_ENGINE_CALL(engine, {
    if (dt == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    return engine->solver->time_steps(0, dt);
  });
}

bs_status bs_engine_boundary_fluxes(bs_engine* engine, int32_t side, bs_face_flux* out) {
  BS_ENGINE_CALL(engine, {
    if (out == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    return engine->solver->boundary_fluxes(0, side, out);
  });
}

bs_status bs_engine_forebody_drag(bs_engine* engine, double p_inf, double q_inf,
                                  double base_radius, double* drag) {
  BS_ENGINE_CALL(engine, {
    if (drag == nullptr || !(q_inf > 0) || !(base_radius > 0))
      return bs::fail(BS_INVALID_ARGUMENT, "the drag needs q_inf > 0 and base_radius > 0");
    return engine->solver->forebody_drag(0, p_inf, q_inf, base_radius, drag);
  });
}

bs_status bs_engine_read_state(bs_engine* engine, float* conserved) {
  BS_ENGINE_CALL(engine, {
    if (conserved == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    return engine->solver->read_state(0, conserved);
  });
}

bs_status bs_engine_read_primitives(bs_engine* engine, double* primitives) {
  BS_ENGINE_CALL(engine, {
    if (primitives == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    return engine->solver->read_primitives(0, primitives);
  });
}

bs_status bs_engine_steps(bs_engine* engine, int64_t* steps) {
  BS_ENGINE_CALL(engine, {
    if (steps == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    *steps = engine->solver->steps(0);
    return BS_OK;
  });
}

bs_status bs_engine_solve(bs_engine* engine, int32_t method, double cfl, double omega,
                          double tolerance, int32_t relative, int32_t max_steps,
                          int32_t check_every, bs_solve_result* result) {
  BS_ENGINE_CALL(engine, {
    if (result == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    if (method != 0 && method != 1) return bs::fail(BS_INVALID_ARGUMENT, "method must be 0 or 1");
    std::vector<bs::CaseResult> r;
    const bs_status s = engine->solver->solve(method, cfl, omega, tolerance, relative, max_steps,
                                              check_every, r);
    if (s != BS_OK) return s;
    result->status = r[0].status;
    result->steps = int32_t(r[0].steps);
    result->residual = r[0].residual;
    result->initial_residual = r[0].initial_residual;
    result->drag = 0;
    if (r[0].status == BS_NON_PHYSICAL)
      return bs::fail(BS_NON_PHYSICAL, "the GPU solution became non-physical");
    if (r[0].status != BS_OK)
      return bs::fail(BS_NOT_CONVERGED, "the residual did not reach the tolerance within the step budget");
    return BS_OK;
  });
}

bs_status bs_engine_iterate_accelerated(bs_engine* engine, int32_t steps, double cfl_max, double omega,
                                        double growth) {
  BS_ENGINE_CALL(engine, { return engine->solver->iterate_accelerated(steps, cfl_max, omega, growth); });
}

bs_status bs_engine_set_metric_precision(bs_engine* engine, int32_t bits) {
  BS_ENGINE_CALL(engine, { return engine->solver->set_metric_precision(bits); });
}

bs_status bs_engine_anderson_restarts(bs_engine* engine, int32_t* restarts) {
  BS_ENGINE_CALL(engine, {
    if (restarts == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    int r = 0;
    const bs_status s = engine->solver->anderson_restarts(&r);
    if (s != BS_OK) return s;
    *restarts = int32_t(r);
    return BS_OK;
  });
}

bs_status bs_engine_set_anderson(bs_engine* engine, int32_t depth, int32_t plain_steps) {
  BS_ENGINE_CALL(engine, { return engine->solver->set_anderson(depth, plain_steps); });
}

bs_status bs_engine_set_sweep_wait_limit(bs_engine* engine, int32_t polls) {
  BS_ENGINE_CALL(engine, { return engine->solver->set_sweep_wait_limit(polls); });
}

}  // extern "C"

// ---- batches ---------------------------------------------------------------

struct bs_batch {
  std::unique_ptr<bs::SolverBase> solver;
  std::atomic<bool> busy{false};
};

namespace {

class BatchExclusive {
 public:
  explicit BatchExclusive(bs_batch* b) : b_(b) {
    bool expected = false;
    owned_ = b != nullptr && b->busy.compare_exchange_strong(expected, true);
  }
  ~BatchExclusive() {
    if (owned_) b_->busy.store(false);
  }
  bs_status status() const {
    if (b_ == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null batch");
    if (!owned_) return bs::fail(BS_BUSY, "the batch is running another operation");
    return BS_OK;
  }

 private:
  bs_batch* b_;
  bool owned_ = false;
};

#define BS_BATCH_CALL(batch, body)            \
  do {                                        \
    BatchExclusive guard_(batch);             \
    const bs_status s_ = guard_.status();     \
    if (s_ != BS_OK) return s_;               \
    body;                                     \
  } while (0)

bs_status check_case(bs_batch* b, int32_t c) {
  if (c < 0 || c >= b->solver->n_cases())
    return bs::fail(BS_INVALID_ARGUMENT, "case index out of range");
  return BS_OK;
}

}  // namespace

extern "C" {

bs_status bs_batch_create(int32_t n, const bs_config* configs, const double* const* x,
                          const double* const* y, int32_t precision, bs_batch** out) {
  if (out == nullptr || configs == nullptr || x == nullptr || y == nullptr || n < 1)
    return bs::fail(BS_INVALID_ARGUMENT, "a batch needs n >= 1 configurations and grids");
  *out = nullptr;
  std::vector<bs::HostCase> cases(n);
  for (int k = 0; k < n; k++) {
    const bs_status s = bs::make_host_case(&configs[k], x[k], y[k], cases[k]);
    if (s != BS_OK) return bs::fail(s, "case " + std::to_string(k) + ": " + bs_last_error());
  }
  auto* b = new (std::nothrow) bs_batch;
  if (b == nullptr) return bs::fail(BS_MEMORY_LIMIT, "out of host memory");
  const bs_status st = bs::make_solver(std::move(cases), precision, b->solver);
  if (st != BS_OK) {
    delete b;
    return st;
  }
  *out = b;
  return BS_OK;
}

bs_status bs_batch_destroy(bs_batch* batch) {
  if (batch == nullptr) return BS_OK;
  bool expected = false;
  if (!batch->busy.compare_exchange_strong(expected, true))
    return bs::fail(BS_BUSY, "the batch is running another operation");
  delete batch;
  return BS_OK;
}

bs_status bs_batch_size(bs_batch* batch, int32_t* n) {
  BS_BATCH_CALL(batch, {
    if (n == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    *n = batch->solver->n_cases();
    return BS_OK;
  });
}

bs_status bs_batch_set_primitives(bs_batch* batch, int32_t c, const double* primitives) {
  BS_BATCH_CALL(batch, {
    if (primitives == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    const bs_status s = check_case(batch, c);
    if (s != BS_OK) return s;
    return batch->solver->set_primitives(c, primitives);
  });
}

bs_status bs_batch_set_free_stream(bs_batch* batch) {
  BS_BATCH_CALL(batch, { return batch->solver->set_free_stream(); });
}

bs_status bs_batch_solve(bs_batch* batch, int32_t method, double cfl, double omega,
                         double tolerance, int32_t relative, int32_t max_steps,
                         int32_t check_every, bs_solve_result* results) {
  BS_BATCH_CALL(batch, {
    if (results == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    if (method != 0 && method != 1) return bs::fail(BS_INVALID_ARGUMENT, "method must be 0 or 1");
    std::vector<bs::CaseResult> r;
    const bs_status s = batch->solver->solve(method, cfl, omega, tolerance, relative, max_steps,
                                             check_every, r);
    if (s != BS_OK) return s;
    for (size_t k = 0; k < r.size(); k++) {
      results[k].status = r[k].status;
      results[k].steps = int32_t(r[k].steps);
      results[k].residual = r[k].residual;
      results[k].initial_residual = r[k].initial_residual;
      results[k].drag = 0;
    }
    return BS_OK;
  });
}

bs_status bs_batch_set_anderson(bs_batch* batch, int32_t depth, int32_t plain_steps) {
  BS_BATCH_CALL(batch, { return batch->solver->set_anderson(depth, plain_steps); });
}

bs_status bs_batch_set_metric_precision(bs_batch* batch, int32_t bits) {
  BS_BATCH_CALL(batch, { return batch->solver->set_metric_precision(bits); });
}

bs_status bs_batch_set_tile_shape(bs_batch* batch, int32_t shape) {
  BS_BATCH_CALL(batch, { return batch->solver->set_tile_shape(shape); });
}

bs_status bs_batch_tuning(bs_batch* batch, int32_t* lanes, int32_t* shape, int32_t* tile_i, int32_t* tile_j,
                          int32_t* threads) {
  BS_BATCH_CALL(batch, {
    if (lanes == nullptr || shape == nullptr || tile_i == nullptr || tile_j == nullptr || threads == nullptr)
      return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    *lanes = batch->solver->lanes();
    *shape = batch->solver->tile_shape();
    bs::tile_dims(*shape, tile_i, tile_j, threads);
    return BS_OK;
  });
}

bs_status bs_batch_set_lanes(bs_batch* batch, int32_t lanes) {
  BS_BATCH_CALL(batch, { return batch->solver->set_lanes(lanes); });
}

bs_status bs_batch_set_update_mode(bs_batch* batch, int32_t fused) {
  BS_BATCH_CALL(batch, {
    if (fused != 0 && fused != 1) return bs::fail(BS_INVALID_ARGUMENT, "update mode: 1 fused, 0 separate");
    return batch->solver->set_fused_update(fused == 1);
  });
}

bs_status bs_batch_update_mode(bs_batch* batch, int32_t* fused) {
  BS_BATCH_CALL(batch, {
    if (fused == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    *fused = batch->solver->fused_update() ? 1 : 0;
    return BS_OK;
  });
}

bs_status bs_batch_set_sweep_wait_limit(bs_batch* batch, int32_t polls) {
  BS_BATCH_CALL(batch, { return batch->solver->set_sweep_wait_limit(polls); });
}

bs_status bs_batch_anderson_restarts(bs_batch* batch, int32_t* restarts) {
  BS_BATCH_CALL(batch, {
    if (restarts == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    std::vector<int> r(batch->solver->n_cases());
    const bs_status s = batch->solver->anderson_restarts(r.data());
    if (s != BS_OK) return s;
    for (size_t k = 0; k < r.size(); k++) restarts[k] = int32_t(r[k]);
    return BS_OK;
  });
}

bs_status bs_batch_forebody_drag(bs_batch* batch, int32_t c, double p_inf, double q_inf,
                                 double base_radius, double* drag) {
  BS_BATCH_CALL(batch, {
    if (drag == nullptr || !(q_inf > 0) || !(base_radius > 0))
      return bs::fail(BS_INVALID_ARGUMENT, "the drag needs q_inf > 0 and base_radius > 0");
    const bs_status s = check_case(batch, c);
    if (s != BS_OK) return s;
    return batch->solver->forebody_drag(c, p_inf, q_inf, base_radius, drag);
  });
}

bs_status bs_batch_read_primitives(bs_batch* batch, int32_t c, double* primitives) {
  BS_BATCH_CALL(batch, {
    if (primitives == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    const bs_status s = check_case(batch, c);
    if (s != BS_OK) return s;
    return batch->solver->read_primitives(c, primitives);
  });
}

bs_status bs_batch_density_residual_norms(bs_batch* batch, double* norms) {
  BS_BATCH_CALL(batch, {
    if (norms == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    return batch->solver->residual_norms(norms);
  });
}

bs_status bs_batch_last_solve_timing(bs_batch* batch, double* device_ms, int64_t* launches) {
  BS_BATCH_CALL(batch, {
    if (device_ms) *device_ms = batch->solver->last_solve_ms();
    if (launches) *launches = batch->solver->last_solve_launches();
    return BS_OK;
  });
}

bs_status bs_batch_kernel_times(bs_batch* batch, int32_t method, double cfl, double omega,
                                int32_t iterations, double* ms) {
  BS_BATCH_CALL(batch, {
    if (ms == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    return batch->solver->kernel_times(method, cfl, omega, iterations, ms);
  });
}

bs_status bs_batch_flow_field(bs_batch* batch, int32_t c, int32_t field, const bs_primitive* free, double length,
                              double* out) {
  BS_BATCH_CALL(batch, {
    if (free == nullptr || out == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    const bs_status s = check_case(batch, c);
    if (s != BS_OK) return s;
    return batch->solver->flow_field(c, field, *free, length, out);
  });
}

bs_status bs_batch_iterate(bs_batch* batch, int32_t steps) {
  BS_BATCH_CALL(batch, { return batch->solver->iterate(steps); });
}

bs_status bs_batch_set_active(bs_batch* batch, const int32_t* flags) {
  BS_BATCH_CALL(batch, {
    if (flags == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    return batch->solver->set_active(flags);
  });
}

bs_status bs_batch_autotune(bs_batch* batch, int32_t method, int32_t steps, double cfl, double omega,
                            int32_t* lanes, double* ms_per_step) {
  BS_BATCH_CALL(batch, {
    if (lanes == nullptr || ms_per_step == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
    int l = 0;
    double ms = 0;
    const bs_status st = batch->solver->autotune(method, steps, cfl, omega, &l, &ms);
    if (st == BS_OK) {
      *lanes = l;
      *ms_per_step = ms;
    }
    return st;
  });
}

}  // extern "C"
