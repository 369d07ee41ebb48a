// One case solved with its bow shock fitted as the outer boundary, all of it
// on the GPU: the fitted-shock iteration of src/solver/shock-fitting.ts:
// 170-314 (device/fitted.cuh) around the explicit steps of the cell kernel:
// a step is five launches (the shock boundary, two SSP-RK2 stages, the
// shock's move, the new grid with the remap), replayed from captured CUDA
// graphs of 16 steps, with the host reading the shock's speed and the
// residual at checks. C ABI: bs_fit_*.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <memory>
#include <vector>

#include "bowshock.h"
#include "common.hpp"
#include "device/fitted.cuh"
#include "device/tile.cuh"
#include "device/wall.cuh"

namespace {

using bs::fail;

bs_status cuda_fail(cudaError_t e, const char* what) {
  return fail(BS_EXECUTION, std::string(what) + ": " + cudaGetErrorString(e));
}

#define FIT_CUDA(expr)                                  \
  do {                                                  \
    const cudaError_t e_ = (expr);                      \
    if (e_ != cudaSuccess) return cuda_fail(e_, #expr); \
  } while (0)

#define FIT_TRY(expr)            \
  do {                           \
    const bs_status s_ = (expr); \
    if (s_ != BS_OK) return s_;  \
  } while (0)

template <class T>
struct Buf {
  T* p = nullptr;
  Buf() = default;
  Buf(const Buf&) = delete;
  Buf& operator=(const Buf&) = delete;
  ~Buf() {
    if (p != nullptr) cudaFree(p);
  }
  cudaError_t alloc(size_t n) { return cudaMalloc(reinterpret_cast<void**>(&p), std::max<size_t>(n, 1) * sizeof(T)); }
  cudaError_t upload(const T* h, size_t n, cudaStream_t s) {
    return cudaMemcpyAsync(p, h, n * sizeof(T), cudaMemcpyHostToDevice, s);
  }
};

constexpr int kChunk = 16;

class FittedSolver {
 public:
  ~FittedSolver() {
    if (graph_ != nullptr) cudaGraphExecDestroy(graph_);
    if (stream_ != nullptr) cudaStreamDestroy(stream_);
  }

  bs_status init(const bs_config& cfg, const double* line_x, const double* line_y, const double* line_dx,
                 const double* line_dy, const double* fractions, const double* heights, const bs_primitive& free,
                 const double* i_min_states, int first_node, const double* initial) {
    ni_ = cfg.ni;
    nj_ = cfg.nj;
    const int ni = ni_, nj = nj_;
    if (ni < 2 || nj < 3) return fail(BS_INVALID_ARGUMENT, "a fitted grid needs at least 2 x 3 cells");
    if (cfg.boundaries[BS_JMAX].kind != BS_BC_FACE_STATES)
      return fail(BS_INVALID_ARGUMENT, "the fitted shock is the jMax side: it must be a face-states side");
    if (cfg.boundaries[BS_JMIN].kind != BS_BC_WALL || cfg.boundaries[BS_IMAX].kind != BS_BC_OUTFLOW)
      return fail(BS_INVALID_ARGUMENT, "a fitted grid has the body (a wall) on jMin and the outflow on iMax");
    const int i_min = cfg.boundaries[BS_IMIN].kind;
    if (i_min != BS_BC_FACE_STATES && i_min != BS_BC_WALL)
      return fail(BS_INVALID_ARGUMENT, "iMin is the inflow plane's face states or the axis (a wall)");
    if (i_min == BS_BC_FACE_STATES && i_min_states == nullptr)
      return fail(BS_INVALID_ARGUMENT, "the inflow plane's face states are missing");
    if (cfg.integrator == BS_FORWARD_EULER || cfg.time_stepping != BS_TIME_LOCAL)
      return fail(BS_INVALID_ARGUMENT, "a fitted grid takes SSP-RK steps with local time steps");
    if (!(cfg.cfl > 0 && cfg.cfl <= 1)) return fail(BS_INVALID_ARGUMENT, "cfl must be in (0, 1]");
    if (first_node != 0 && first_node != 1) return fail(BS_INVALID_ARGUMENT, "first_node is 0 (fixed) or 1 (symmetry)");
    if (!(free.rho > 0 && free.p > 0)) return fail(BS_INVALID_ARGUMENT, "the free stream needs rho > 0 and p > 0");
    if (!(cfg.gamma > 1)) return fail(BS_INVALID_ARGUMENT, "gamma must exceed 1");
    const size_t nn = size_t(ni + 1) * (nj + 1), nc = size_t(ni) * nj;
    std::vector<double> line(4 * size_t(ni + 1));
    for (int k = 0; k <= ni; k++) {
      const double len = std::hypot(line_dx[k], line_dy[k]);
      if (!(std::fabs(len - 1) < 1e-12)) return fail(BS_INVALID_ARGUMENT, "the lines' directions must be unit vectors");
      if (!(heights[k] > 0)) return fail(BS_INVALID_ARGUMENT, "the shock heights must be positive");
      line[4 * k] = line_x[k];
      line[4 * k + 1] = line_y[k];
      line[4 * k + 2] = line_dx[k];
      line[4 * k + 3] = line_dy[k];
    }
    // The fractions of a stretched line end at expm1(b nj / nj) / expm1(b),
    // which rounds to 1 + 2^-52 for some b: a rounding above 1 is accepted.
    for (size_t k = 0; k < nn; k++)
      if (!(fractions[k] >= 0 && fractions[k] <= 1 + 1e-12))
        return fail(BS_INVALID_ARGUMENT, "the node fractions must lie in [0, 1]");
    gamma_ = cfg.gamma;
    integrator_ = cfg.integrator;
    FIT_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    FIT_CUDA(line_.alloc(line.size()));
    FIT_CUDA(line_.upload(line.data(), line.size(), stream_));
    FIT_CUDA(fraction_.alloc(nn));
    FIT_CUDA(fraction_.upload(fractions, nn, stream_));
    for (Buf<double>* b : {&heights_, &heights_old_, &heights_next_}) FIT_CUDA(b->alloc(ni + 1));
    FIT_CUDA(heights_.upload(heights, ni + 1, stream_));
    FIT_CUDA(heights_old_.upload(heights, ni + 1, stream_));
    FIT_CUDA(x_.alloc(nn));
    FIT_CUDA(y_.alloc(nn));
    for (int v = 0; v < 4; v++) {
      FIT_CUDA(q_[v].alloc(nc));
      FIT_CUDA(s1_[v].alloc(nc));
      FIT_CUDA(old_[v].alloc(nc));
      if (cfg.integrator != BS_SSPRK2) FIT_CUDA(s2_[v].alloc(nc));
    }
    FIT_CUDA(dt_.alloc(nc));
    FIT_CUDA(iface_.alloc(size_t(ni + 1) * nj));
    FIT_CUDA(jface_.alloc(size_t(ni) * (nj + 1)));
    FIT_CUDA(cellm_.alloc(nc));
    FIT_CUDA(iface_lo_.alloc(size_t(ni + 1) * nj));
    FIT_CUDA(jface_lo_.alloc(size_t(ni) * (nj + 1)));
    FIT_CUDA(cellm_lo_.alloc(nc));
    FIT_CUDA(bgeom_.alloc(3 * size_t(2 * (ni + nj))));
    FIT_CUDA(top_state_.alloc(4 * size_t(ni)));
    FIT_CUDA(top_flux_.alloc(4 * size_t(ni)));
    FIT_CUDA(speed_.alloc(ni));
    FIT_CUDA(words_.alloc(4));  // max speed, residual sum, force, spare
    FIT_CUDA(status_.alloc(1));
    FIT_CUDA(bflux_.alloc(4 * size_t(std::max(ni, nj))));
    FIT_CUDA(cudaMemsetAsync(status_.p, 0, sizeof(unsigned), stream_));
    FIT_CUDA(cudaMemsetAsync(words_.p, 0, 4 * sizeof(double), stream_));
    // The free stream's ghosts until the first boundary pass.
    {
      std::vector<double> top(4 * size_t(ni));
      const double e = free.p / (gamma_ - 1) + 0.5 * free.rho * (free.u * free.u + free.v * free.v);
      for (int i = 0; i < ni; i++) {
        top[4 * i] = free.rho;
        top[4 * i + 1] = free.rho * free.u;
        top[4 * i + 2] = free.rho * free.v;
        top[4 * i + 3] = e;
      }
      FIT_CUDA(top_state_.upload(top.data(), top.size(), stream_));
      FIT_CUDA(top_flux_.upload(top.data(), top.size(), stream_));
      FIT_CUDA(cudaStreamSynchronize(stream_));
    }
    bsd::CaseDev cd{};
    cd.ni = ni;
    cd.nj = nj;
    for (int s = 0; s < 4; s++) cd.bc[s] = cfg.boundaries[s].kind;
    cd.flux = cfg.flux;
    cd.limiter = cfg.limiter;
    cd.recon = cfg.reconstruction;
    cd.axisym = cfg.geometry == BS_AXISYMMETRIC ? 1 : 0;
    cd.integrator = cfg.integrator;
    cd.local_dt = 1;
    cd.gamma = gamma_;
    cd.cfl = cfg.cfl;
    cd.face_state[BS_JMAX] = top_state_.p;
    cd.face_flux[BS_JMAX] = top_flux_.p;
    if (i_min == BS_BC_FACE_STATES) {
      std::vector<double> st(4 * size_t(nj));
      for (int j = 0; j < nj; j++) {
        const double* w = i_min_states + 4 * j;
        st[4 * j] = w[0];
        st[4 * j + 1] = w[0] * w[1];
        st[4 * j + 2] = w[0] * w[2];
        st[4 * j + 3] = w[3] / (gamma_ - 1) + 0.5 * w[0] * (w[1] * w[1] + w[2] * w[2]);
      }
      FIT_CUDA(in_state_.alloc(st.size()));
      FIT_CUDA(in_state_.upload(st.data(), st.size(), stream_));
      FIT_CUDA(cudaStreamSynchronize(stream_));
      cd.face_state[BS_IMIN] = in_state_.p;
    }
    FIT_CUDA(case_.alloc(1));
    FIT_CUDA(case_.upload(&cd, 1, stream_));
    const int ti = (ni + bsd::TI - 1) / bsd::TI, tj = (nj + bsd::TJ - 1) / bsd::TJ;
    n_tiles_ = ti * tj;
    std::vector<int2> tiles(n_tiles_);
    for (int t = 0; t < n_tiles_; t++) tiles[t] = make_int2(0, t);
    FIT_CUDA(tiles_.alloc(n_tiles_));
    FIT_CUDA(tiles_.upload(tiles.data(), n_tiles_, stream_));
    FIT_CUDA(cudaStreamSynchronize(stream_));

    A_.cases = case_.p;
    A_.ni = ni;
    A_.nj = nj;
    A_.gamma = gamma_;
    A_.free[0] = free.rho;
    A_.free[1] = free.u;
    A_.free[2] = free.v;
    A_.free[3] = free.p;
    A_.a_free = std::sqrt(gamma_ * free.p / free.rho);
    A_.line = line_.p;
    A_.fraction = fraction_.p;
    A_.heights = heights_.p;
    A_.heights_old = heights_old_.p;
    A_.heights_next = heights_next_.p;
    A_.nx_ = x_.p;
    A_.ny_ = y_.p;
    A_.face_state = top_state_.p;
    A_.face_flux = top_flux_.p;
    A_.speed = speed_.p;
    A_.max_speed = words_.p;
    A_.first_node = first_node;
    A_.axisym = cd.axisym;
    A_.iface = iface_.p;
    A_.jface = jface_.p;
    A_.cellm = cellm_.p;
    A_.iface_lo = iface_lo_.p;
    A_.jface_lo = jface_lo_.p;
    A_.cellm_lo = cellm_lo_.p;
    A_.bgeom = bgeom_.p;
    A_.q = q_view();
    A_.q_old = {old_[0].p, old_[1].p, old_[2].p, old_[3].p};
    FIT_TRY(launch_grid());
    // The residual scale: the larger of the starting flow's and the free
    // stream's on the first grid, each with its shock boundary (fitShock, :232-245).
    std::vector<double> prim(4 * nc);
    for (size_t k = 0; k < nc; k++) {
      prim[4 * k] = free.rho;
      prim[4 * k + 1] = free.u;
      prim[4 * k + 2] = free.v;
      prim[4 * k + 3] = free.p;
    }
    FIT_TRY(set_primitives(prim.data()));
    double r_free = 0, r_start = 0;
    FIT_TRY(residual(&r_free));
    FIT_TRY(set_primitives(initial));
    FIT_TRY(residual(&r_start));
    initial_residual_ = std::max(r_free, r_start);
    return BS_OK;
  }

  bs_status set_primitives(const double* prim) {
    const size_t nc = size_t(ni_) * nj_;
    std::vector<double> c[4];
    for (int v = 0; v < 4; v++) c[v].resize(nc);
    for (size_t k = 0; k < nc; k++) {
      const double* w = prim + 4 * k;
      if (!(w[0] > 0 && w[3] > 0)) return fail(BS_NON_PHYSICAL, "a starting state has rho <= 0 or p <= 0");
      c[0][k] = w[0];
      c[1][k] = w[0] * w[1];
      c[2][k] = w[0] * w[2];
      c[3][k] = w[3] / (gamma_ - 1) + 0.5 * w[0] * (w[1] * w[1] + w[2] * w[2]);
    }
    for (int v = 0; v < 4; v++) FIT_CUDA(q_[v].upload(c[v].data(), nc, stream_));
    FIT_CUDA(cudaStreamSynchronize(stream_));
    return BS_OK;
  }

  // `steps` fitted steps (each: the shock boundary, an explicit step, the move,
  // the new grid, the remap), from graphs of up to kChunk steps.
  bs_status iterate(int steps) {
    if (steps < 0) return fail(BS_INVALID_ARGUMENT, "steps must be non-negative");
    int left = steps;
    while (left >= kChunk) {
      if (graph_ == nullptr) {
        cudaGraph_t g = nullptr;
        FIT_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        bs_status st = BS_OK;
        for (int s = 0; s < kChunk && st == BS_OK; s++) st = record_step();
        const cudaError_t end = cudaStreamEndCapture(stream_, &g);
        if (st != BS_OK) {
          if (g != nullptr) cudaGraphDestroy(g);
          return st;
        }
        FIT_CUDA(end);
        const cudaError_t inst = cudaGraphInstantiate(&graph_, g, 0);
        cudaGraphDestroy(g);
        FIT_CUDA(inst);
      }
      FIT_CUDA(cudaGraphLaunch(graph_, stream_));
      left -= kChunk;
    }
    for (int s = 0; s < left; s++) FIT_TRY(record_step());
    iterations_ += steps;
    FIT_CUDA(cudaStreamSynchronize(stream_));
    unsigned status = 0;
    FIT_CUDA(cudaMemcpy(&status, status_.p, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (status & bsd::STATUS_NON_PHYSICAL) return fail(BS_NON_PHYSICAL, "the fitted solution became non-physical");
    return BS_OK;
  }

  // The largest shock speed of the last move over a_inf, and the density
  // residual of the current flow with its shock boundary applied, relative to
  // the starting scale.
  bs_status check(double* max_speed, double* residual_rel) {
    double r = 0;
    FIT_TRY(residual(&r));
    FIT_CUDA(cudaMemcpy(max_speed, words_.p, sizeof(double), cudaMemcpyDeviceToHost));
    *residual_rel = r / initial_residual_;
    return BS_OK;
  }

  bs_status solve(double speed_tol, double residual_tol, int max_iterations, int check_every, int* iterations,
                  int* converged, double* max_speed, double* residual_rel) {
    if (!(speed_tol > 0 && residual_tol > 0) || max_iterations < 0 || check_every < 1)
      return fail(BS_INVALID_ARGUMENT, "a fit needs positive tolerances and check_every >= 1");
    *converged = 0;
    double speed = INFINITY, r = INFINITY;
    int done = 0;
    while (done < max_iterations) {
      const int n = std::min(check_every, max_iterations - done);
      FIT_TRY(iterate(n));
      done += n;
      FIT_TRY(check(&speed, &r));
      if (speed < speed_tol && r < residual_tol) {
        *converged = 1;
        break;
      }
    }
    *iterations = done;
    *max_speed = speed;
    *residual_rel = r;
    return BS_OK;
  }

  bs_status heights(double* out) {
    FIT_CUDA(cudaMemcpy(out, heights_.p, (ni_ + 1) * sizeof(double), cudaMemcpyDeviceToHost));
    return BS_OK;
  }

  bs_status nodes(double* x, double* y) {
    const size_t nn = size_t(ni_ + 1) * (nj_ + 1);
    FIT_CUDA(cudaMemcpy(x, x_.p, nn * sizeof(double), cudaMemcpyDeviceToHost));
    FIT_CUDA(cudaMemcpy(y, y_.p, nn * sizeof(double), cudaMemcpyDeviceToHost));
    return BS_OK;
  }

  bs_status primitives(double* out) {
    const size_t nc = size_t(ni_) * nj_;
    std::vector<double> c[4];
    for (int v = 0; v < 4; v++) {
      c[v].resize(nc);
      FIT_CUDA(cudaMemcpy(c[v].data(), q_[v].p, nc * sizeof(double), cudaMemcpyDeviceToHost));
    }
    for (size_t k = 0; k < nc; k++) {
      const double rho = c[0][k], u = c[1][k] / rho, v = c[2][k] / rho;
      out[4 * k] = rho;
      out[4 * k + 1] = u;
      out[4 * k + 2] = v;
      out[4 * k + 3] = (gamma_ - 1) * (c[3][k] - 0.5 * rho * (u * u + v * v));
    }
    return BS_OK;
  }

  // The metrics the residual and the wall fluxes read: two-float (FP32
  // values and low parts, both written by every regrid).
  bsd::MetricsView metrics() const {
    bsd::MetricsView m{iface_.p, jface_.p, cellm_.p};
    m.iface_lo = iface_lo_.p;
    m.jface_lo = jface_lo_.p;
    m.cell_lo = cellm_lo_.p;
    return m;
  }

  // Wall fluxes of jMin (FP64, as bs_engine_boundary_fluxes) and the drag.
  bs_status wall(double p_inf, double* flux_out, double* force) {
    bsd::BoundaryArgs<double> B{};
    B.cases = case_.p;
    B.case_index = 0;
    B.q = q_view();
    B.m = metrics();
    B.side = BS_JMIN;
    B.geom = bgeom_.p + 3 * size_t(2 * nj_);
    B.gamma_eval = gamma_;
    B.flux_out = bflux_.p;
    B.p_inf = p_inf;
    B.force_out = words_.p + 2;
    bsd::boundary_flux_kernel<double><<<1, 256, 0, stream_>>>(B);
    FIT_CUDA(cudaGetLastError());
    FIT_CUDA(cudaStreamSynchronize(stream_));
    if (flux_out != nullptr) FIT_CUDA(cudaMemcpy(flux_out, bflux_.p, 4 * size_t(ni_) * sizeof(double), cudaMemcpyDeviceToHost));
    FIT_CUDA(cudaMemcpy(force, words_.p + 2, sizeof(double), cudaMemcpyDeviceToHost));
    return BS_OK;
  }

  // The jMin wall's faces (boundaryFluxes('jMin'), src/engine-cpu/euler2d.ts:
  // 499-525): midpoint, outward normal, area and the FP64 flux.
  bs_status wall_fluxes(bs_face_flux* out) {
    double force = 0;
    std::vector<double> f(4 * size_t(ni_));
    FIT_TRY(wall(0.0, f.data(), &force));
    std::vector<double> g(3 * size_t(ni_)), x(ni_ + 1), y(ni_ + 1);
    FIT_CUDA(cudaMemcpy(g.data(), bgeom_.p + 3 * size_t(2 * nj_), g.size() * sizeof(double),
                        cudaMemcpyDeviceToHost));
    FIT_CUDA(cudaMemcpy(x.data(), x_.p, (ni_ + 1) * sizeof(double), cudaMemcpyDeviceToHost));
    FIT_CUDA(cudaMemcpy(y.data(), y_.p, (ni_ + 1) * sizeof(double), cudaMemcpyDeviceToHost));
    for (int t = 0; t < ni_; t++) {
      bs_face_flux& o = out[t];
      o.x = 0.5 * (x[t] + x[t + 1]);
      o.y = 0.5 * (y[t] + y[t + 1]);
      o.nx = -g[3 * t];
      o.ny = -g[3 * t + 1];
      o.area = g[3 * t + 2];
      for (int v = 0; v < 4; v++) o.flux[v] = f[4 * t + v];
    }
    return BS_OK;
  }

  int ni() const { return ni_; }
  int nj() const { return nj_; }
  int iterations() const { return iterations_; }

 private:
  bsd::StateView<double> q_view() const { return {q_[0].p, q_[1].p, q_[2].p, q_[3].p}; }
  bsd::StateView<double> s1_view() const { return {s1_[0].p, s1_[1].p, s1_[2].p, s1_[3].p}; }

  int blocks(int64_t n) const { return int(std::min<int64_t>((n + 255) / 256, 4096)); }

  // The grid on the current heights and its metrics; with `remap`, the flow
  // in q_old interpolated onto it into q.
  bs_status launch_grid(bool remap = false) {
    const int64_t nc = int64_t(ni_) * nj_;
    const int64_t all = int64_t(ni_ + 1) * (nj_ + 1) + int64_t(ni_ + 1) * nj_ + int64_t(ni_) * (nj_ + 1) + nc +
                        (remap ? nc : 0);
    bsd::fit_regrid_kernel<<<blocks(all), 256, 0, stream_>>>(A_, remap ? 1 : 0);
    FIT_CUDA(cudaGetLastError());
    return BS_OK;
  }

  bs_status launch_boundary() {
    bsd::fit_boundary_kernel<<<(ni_ + 127) / 128, 128, 0, stream_>>>(A_);
    FIT_CUDA(cudaGetLastError());
    return BS_OK;
  }

  template <int MODE>
  bs_status launch_tile(bsd::StateView<double> src, bsd::StateView<double> out, double a, double b, bool first,
                        double* norm) {
    bsd::TileArgs<double> T{};
    T.cases = case_.p;
    T.tiles = tiles_.p;
    T.active = nullptr;
    T.src = src;
    T.u0 = q_view();
    T.out = out;
    T.m = metrics();
    T.dt = dt_.p;
    T.dt_global = nullptr;
    T.norm = norm;
    T.status = status_.p;
    T.a = a;
    T.b = b;
    T.first_stage = first ? 1 : 0;
    bsd::tile_kernel<double, MODE><<<n_tiles_, bsd::TILE_THREADS, 0, stream_>>>(T);
    FIT_CUDA(cudaGetLastError());
    return BS_OK;
  }

  // The density residual RMS of the current flow with its shock boundary.
  bs_status residual(double* out) {
    FIT_TRY(launch_boundary());
    FIT_CUDA(cudaMemsetAsync(words_.p + 1, 0, sizeof(double), stream_));
    FIT_TRY(launch_tile<bsd::MODE_RESIDUAL>(q_view(), q_view(), 0, 1, false, words_.p + 1));
    FIT_CUDA(cudaStreamSynchronize(stream_));
    double s = 0;
    FIT_CUDA(cudaMemcpy(&s, words_.p + 1, sizeof(double), cudaMemcpyDeviceToHost));
    *out = std::sqrt(s / (double(ni_) * nj_));
    return BS_OK;
  }

  bs_status record_step() {
    FIT_TRY(launch_boundary());
    // The step's last stage writes the state on the grid before the move
    // (q_old), which the move reads and the remap carries into q.
    const bsd::StateView<double> q = q_view(), s1 = s1_view();
    const bsd::StateView<double> old = {old_[0].p, old_[1].p, old_[2].p, old_[3].p};
    if (integrator_ == BS_SSPRK2) {
      FIT_TRY(launch_tile<bsd::MODE_STAGE>(q, s1, 0, 1, true, nullptr));
      FIT_TRY(launch_tile<bsd::MODE_STAGE>(s1, old, 0.5, 0.5, false, nullptr));
    } else {
      const bsd::StateView<double> s2 = {s2_[0].p, s2_[1].p, s2_[2].p, s2_[3].p};
      FIT_TRY(launch_tile<bsd::MODE_STAGE>(q, s1, 0, 1, true, nullptr));
      FIT_TRY(launch_tile<bsd::MODE_STAGE>(s1, s2, 0.75, 0.25, false, nullptr));
      FIT_TRY(launch_tile<bsd::MODE_STAGE>(s2, old, 1.0 / 3.0, 2.0 / 3.0, false, nullptr));
    }
    bsd::fit_move_kernel<<<1, 256, 0, stream_>>>(A_);
    FIT_CUDA(cudaGetLastError());
    return launch_grid(true);
  }

  int ni_ = 0, nj_ = 0, n_tiles_ = 0, integrator_ = 0, iterations_ = 0;
  double gamma_ = 1.4, initial_residual_ = 1;
  cudaStream_t stream_ = nullptr;
  cudaGraphExec_t graph_ = nullptr;
  bsd::FitArgs A_{};
  Buf<bsd::CaseDev> case_;
  Buf<int2> tiles_;
  Buf<double> line_, fraction_, heights_, heights_old_, heights_next_, x_, y_;
  Buf<double> q_[4], s1_[4], s2_[4], old_[4];
  Buf<float> dt_;
  Buf<float4> iface_, jface_, iface_lo_, jface_lo_;
  Buf<float2> cellm_, cellm_lo_;
  Buf<double> bgeom_, top_state_, top_flux_, in_state_, speed_, words_, bflux_;
  Buf<unsigned> status_;
};

}  // namespace

struct bs_fit {
  FittedSolver solver;
  std::atomic<int> busy{0};
};

#define FIT_CALL(fit, ...)                                                                    \
  do {                                                                                        \
    if ((fit) == nullptr) return fail(BS_INVALID_ARGUMENT, "null fit");                       \
    if ((fit)->busy.exchange(1)) return fail(BS_BUSY, "another call is running on this fit"); \
    const bs_status r_ = [&]() -> bs_status __VA_ARGS__();                                    \
    (fit)->busy.store(0);                                                                     \
    return r_;                                                                                \
  } while (0)

extern "C" {

bs_status bs_fit_create(const bs_config* config, const double* line_x, const double* line_y, const double* line_dx,
                        const double* line_dy, const double* fractions, const double* heights,
                        const bs_primitive* free, const double* i_min_states, int32_t first_node,
                        const double* initial, bs_fit** out) {
  if (config == nullptr || line_x == nullptr || line_y == nullptr || line_dx == nullptr || line_dy == nullptr ||
      fractions == nullptr || heights == nullptr || free == nullptr || initial == nullptr || out == nullptr)
    return fail(BS_INVALID_ARGUMENT, "null argument");
  auto f = std::make_unique<bs_fit>();
  const bs_status s = f->solver.init(*config, line_x, line_y, line_dx, line_dy, fractions, heights, *free,
                                     i_min_states, first_node, initial);
  if (s != BS_OK) return s;
  *out = f.release();
  return BS_OK;
}

bs_status bs_fit_destroy(bs_fit* fit) {
  delete fit;
  return BS_OK;
}

bs_status bs_fit_iterate(bs_fit* fit, int32_t steps) {
  FIT_CALL(fit, { return fit->solver.iterate(steps); });
}

bs_status bs_fit_check(bs_fit* fit, double* max_speed, double* residual) {
  FIT_CALL(fit, {
    if (max_speed == nullptr || residual == nullptr) return fail(BS_INVALID_ARGUMENT, "null argument");
    return fit->solver.check(max_speed, residual);
  });
}

bs_status bs_fit_solve(bs_fit* fit, double speed_tolerance, double residual_tolerance, int32_t max_iterations,
                       int32_t check_every, int32_t* iterations, int32_t* converged, double* max_speed,
                       double* residual) {
  FIT_CALL(fit, {
    if (iterations == nullptr || converged == nullptr || max_speed == nullptr || residual == nullptr)
      return fail(BS_INVALID_ARGUMENT, "null argument");
    int it = 0, conv = 0;
    const bs_status s = fit->solver.solve(speed_tolerance, residual_tolerance, max_iterations, check_every, &it,
                                          &conv, max_speed, residual);
    *iterations = it;
    *converged = conv;
    return s;
  });
}

bs_status bs_fit_heights(bs_fit* fit, double* heights) {
  FIT_CALL(fit, {
    if (heights == nullptr) return fail(BS_INVALID_ARGUMENT, "null argument");
    return fit->solver.heights(heights);
  });
}

bs_status bs_fit_nodes(bs_fit* fit, double* x, double* y) {
  FIT_CALL(fit, {
    if (x == nullptr || y == nullptr) return fail(BS_INVALID_ARGUMENT, "null argument");
    return fit->solver.nodes(x, y);
  });
}

bs_status bs_fit_read_primitives(bs_fit* fit, double* primitives) {
  FIT_CALL(fit, {
    if (primitives == nullptr) return fail(BS_INVALID_ARGUMENT, "null argument");
    return fit->solver.primitives(primitives);
  });
}

bs_status bs_fit_wall_fluxes(bs_fit* fit, bs_face_flux* out) {
  FIT_CALL(fit, {
    if (out == nullptr) return fail(BS_INVALID_ARGUMENT, "null argument");
    return fit->solver.wall_fluxes(out);
  });
}

bs_status bs_fit_forebody_drag(bs_fit* fit, double p_inf, double q_inf, double base_radius, double* drag) {
  FIT_CALL(fit, {
    if (drag == nullptr || !(q_inf > 0) || !(base_radius > 0))
      return fail(BS_INVALID_ARGUMENT, "the drag needs q_inf > 0 and base_radius > 0");
    double force = 0;
    const bs_status s = fit->solver.wall(p_inf, nullptr, &force);
    if (s != BS_OK) return s;
    *drag = (2 * force) / (q_inf * base_radius * base_radius);
    return BS_OK;
  });
}

}  // extern "C"
