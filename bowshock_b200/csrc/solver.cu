// GPU solve of a batch of cases: device arenas, kernel launches, CUDA-graph
// replay of the step loop, convergence checks with one small device-to-host
// read per check, and the FP64 boundary evaluations.
#include "solver.hpp"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "common.hpp"
#include "device/anderson.cuh"
#include "device/fields.cuh"
#include "device/sweep.cuh"
#include "device/tile.cuh"
#include "device/wall.cuh"

namespace bs {

std::string validate_config(const bs_config& c) {
  if (!(c.cfl > 0 && c.cfl <= 1)) return "cfl must be in (0, 1]";
  if (c.ni < 2 || c.nj < 2) return "the grid needs at least 2 x 2 cells";
  if (c.nj > 512) return "the GPU engine takes at most 512 cells across (nj)";
  if (c.ni > (1 << 24)) return "too many cells along the grid (ni)";
  if (!(c.gamma > 1)) return "gamma must exceed 1";
  if (c.geometry != BS_PLANAR && c.geometry != BS_AXISYMMETRIC) return "unknown geometry";
  if (c.flux != BS_FLUX_HLLC && c.flux != BS_FLUX_RUSANOV)
    return "the GPU engine has only the hllc and rusanov fluxes";
  if (c.limiter < BS_LIMITER_FIRST_ORDER || c.limiter > BS_LIMITER_UNLIMITED_CENTRAL)
    return "unknown limiter";
  if (c.reconstruction < BS_RECON_PER_VARIABLE || c.reconstruction > BS_RECON_SHARED_SCALED)
    return "unknown reconstruction";
  if ((c.reconstruction == BS_RECON_SHARED || c.reconstruction == BS_RECON_SHARED_SCALED) &&
      c.limiter != BS_LIMITER_VAN_ALBADA)
    return "shared reconstruction requires the 'vanAlbada' limiter";
  if (c.integrator < BS_FORWARD_EULER || c.integrator > BS_SSPRK3) return "unknown time integrator";
  if (c.time_stepping != BS_TIME_LOCAL && c.time_stepping != BS_TIME_GLOBAL)
    return "unknown time stepping";
  for (int s = 0; s < 4; s++) {
    const bs_boundary& b = c.boundaries[s];
    if (b.kind < BS_BC_INFLOW || b.kind > BS_BC_PERIODIC) return "unknown boundary kind";
    if (b.kind == BS_BC_INFLOW || b.kind == BS_BC_FAR_FIELD) {
      const bs_primitive& w = b.state;
      if (!(w.rho > 0 && w.p > 0 && std::isfinite(w.u) && std::isfinite(w.v)))
        return "a boundary state must have positive density and pressure";
    }
  }
  if ((c.boundaries[0].kind == BS_BC_PERIODIC) != (c.boundaries[1].kind == BS_BC_PERIODIC))
    return "periodic boundaries must be used on both iMin and iMax";
  if ((c.boundaries[2].kind == BS_BC_PERIODIC) != (c.boundaries[3].kind == BS_BC_PERIODIC))
    return "periodic boundaries must be used on both jMin and jMax";
  return "";
}

namespace {

bs_status cuda_fail(cudaError_t e, const char* what) {
  cudaGetLastError();  // clear a non-sticky error
  if (e == cudaErrorMemoryAllocation)
    return fail(BS_MEMORY_LIMIT, std::string("device memory exhausted (") + what + ")");
  return fail(BS_EXECUTION, std::string(what) + ": " + cudaGetErrorString(e));
}

#define BS_CUDA(expr)                                   \
  do {                                                  \
    const cudaError_t e_ = (expr);                      \
    if (e_ != cudaSuccess) return cuda_fail(e_, #expr); \
  } while (0)

#define BS_TRY(expr)                       \
  do {                                     \
    const bs_status s_ = (expr);           \
    if (s_ != BS_OK) return s_;            \
  } while (0)

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() {
    if (p != nullptr) cudaFree(p);
  }
  cudaError_t alloc(size_t count) {
    if (p != nullptr) {
      cudaFree(p);
      p = nullptr;
    }
    n = count;
    return cudaMalloc(reinterpret_cast<void**>(&p), std::max<size_t>(count, 1) * sizeof(T));
  }
};

struct GraphKey {
  int method, count, norm_last;
  bool operator<(const GraphKey& o) const {
    if (method != o.method) return method < o.method;
    if (count != o.count) return count < o.count;
    return norm_last < o.norm_last;
  }
};

constexpr int kMethodExplicit = 0;
constexpr int kMethodImplicit = 1;
// LU-SGS steps with Anderson acceleration (graphs of their own; the C ABI's
// method stays LU-SGS, the acceleration is a setting of the batch).
constexpr int kMethodAnderson = 2;

// The launch geometry of a group of cases: its tile list, case list, widest
// case and stream. The whole batch is one lane; a batch of several cases is
// also split into lanes whose step chains run concurrently (a lane's residual
// pass fills the SMs that the other lanes' sweeps leave idle).
struct LaneView {
  const int2* tiles;
  int n_tiles;
  const int* case_list;
  int n_cases;
  int max_nj;
  int max_len;  // longest anti-diagonal, max min(ni, nj), of its cases
  cudaStream_t stream;
  // The residual pass's tiles when the batch runs a tuned tile shape (else
  // the default tiles above).
  const int2* rtiles = nullptr;
  int n_rtiles = 0;
};

// The tiles of `cases` for a tile shape of ti x tj cells, case by case.
std::vector<int2> tiles_for(const std::vector<bsd::CaseDev>& hc, const std::vector<int>& cases, int ti, int tj) {
  std::vector<int2> t;
  for (int c : cases) {
    const int n = ((hc[c].ni + ti - 1) / ti) * ((hc[c].nj + tj - 1) / tj);
    for (int k = 0; k < n; k++) t.push_back(make_int2(c, k));
  }
  return t;
}

constexpr int kMaxLanes = 64;
constexpr int kDefaultLanes = 16;

template <class R>
class Solver final : public SolverBase {
 public:
  explicit Solver(std::vector<HostCase>&& cases) : cases_(std::move(cases)) {}

  ~Solver() override {
    for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second);
    for (auto& l : lanes_)
      if (l->stream != nullptr) cudaStreamDestroy(l->stream);
    for (auto e : ev_join_) cudaEventDestroy(e);
    if (ev_fork_ != nullptr) cudaEventDestroy(ev_fork_);
    if (ev0_ != nullptr) cudaEventDestroy(ev0_);
    if (ev1_ != nullptr) cudaEventDestroy(ev1_);
    if (stream_ != nullptr) cudaStreamDestroy(stream_);
  }

  bs_status init() {
    n_ = int(cases_.size());
    BS_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    BS_CUDA(cudaEventCreate(&ev0_));
    BS_CUDA(cudaEventCreate(&ev1_));
    {
      int dev = 0;
      BS_CUDA(cudaGetDevice(&dev));
      BS_CUDA(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, dev));
    }
    std::vector<bsd::CaseDev> hc(n_);
    std::vector<int2> tiles;
    int64_t cell = 0, ifc = 0, jfc = 0, bfc = 0, slots = 0;
    boundary_off_.resize(n_);
    cell_off_.resize(n_);
    for (int c = 0; c < n_; c++) {
      cell_off_[c] = cell;
      const HostCase& h = cases_[c];
      const bs_config& cfg = h.cfg;
      bsd::CaseDev& d = hc[c];
      d.ni = cfg.ni;
      d.nj = cfg.nj;
      d.cell = cell;
      d.iface = ifc;
      d.jface = jfc;
      d.slot = slots;
      d.tile_base = int64_t(tiles.size());
      slots += bsd::sweep_slots(cfg.ni, cfg.nj);
      for (int s = 0; s < 4; s++) d.bc[s] = cfg.boundaries[s].kind;
      d.flux = cfg.flux;
      d.limiter = cfg.limiter;
      d.recon = cfg.reconstruction;
      d.axisym = cfg.geometry == BS_AXISYMMETRIC;
      d.integrator = cfg.integrator;
      d.local_dt = cfg.time_stepping == BS_TIME_LOCAL;
      any_global_dt_ = any_global_dt_ || !d.local_dt;
      d.gamma = solve_gamma(cfg.gamma);
      d.cfl = cfg.cfl;
      for (int s = 0; s < 4; s++) {
        const bs_primitive& w = cfg.boundaries[s].state;
        d.inflow_prim[s][0] = w.rho;
        d.inflow_prim[s][1] = w.u;
        d.inflow_prim[s][2] = w.v;
        d.inflow_prim[s][3] = w.p;
        const double g = d.gamma;
        d.inflow_cons[s][0] = w.rho;
        d.inflow_cons[s][1] = w.rho * w.u;
        d.inflow_cons[s][2] = w.rho * w.v;
        d.inflow_cons[s][3] = w.p / (g - 1) + 0.5 * w.rho * (w.u * w.u + w.v * w.v);
      }
      const int ti = (cfg.ni + bsd::TI - 1) / bsd::TI, tj = (cfg.nj + bsd::TJ - 1) / bsd::TJ;
      for (int t = 0; t < ti * tj; t++) tiles.push_back(make_int2(c, t));
      boundary_off_[c] = bfc;
      bfc += 2 * int64_t(cfg.ni + cfg.nj);
      cell += int64_t(cfg.ni) * cfg.nj;
      ifc += int64_t(cfg.ni + 1) * cfg.nj;
      jfc += int64_t(cfg.ni) * (cfg.nj + 1);
      max_nj_ = std::max(max_nj_, cfg.nj);
      max_len_ = std::max(max_len_, std::min(cfg.ni, cfg.nj));
      max_along_ = std::max(max_along_, std::max(cfg.ni, cfg.nj));
    }
    total_cells_ = cell;
    total_slots_ = slots;
    n_tiles_ = int(tiles.size());
    steps_.assign(n_, 0);
    active_h_.assign(n_, 1);

    BS_CUDA(d_cases_.alloc(n_));
    BS_CUDA(cudaMemcpy(d_cases_.p, hc.data(), n_ * sizeof(bsd::CaseDev), cudaMemcpyHostToDevice));
    BS_CUDA(d_tiles_.alloc(tiles.size()));
    BS_CUDA(cudaMemcpy(d_tiles_.p, tiles.data(), tiles.size() * sizeof(int2), cudaMemcpyHostToDevice));
    std::vector<int> list(n_);
    for (int c = 0; c < n_; c++) list[c] = c;
    BS_CUDA(d_case_list_.alloc(n_));
    BS_CUDA(cudaMemcpy(d_case_list_.p, list.data(), n_ * sizeof(int), cudaMemcpyHostToDevice));
    BS_CUDA(d_active_.alloc(n_));
    BS_CUDA(cudaMemcpy(d_active_.p, active_h_.data(), n_ * sizeof(int), cudaMemcpyHostToDevice));
    for (int v = 0; v < 4; v++) BS_CUDA(q_[v].alloc(total_cells_));
    BS_CUDA(dt_.alloc(total_cells_));
    BS_CUDA(iface_.alloc(ifc));
    BS_CUDA(jface_.alloc(jfc));
    BS_CUDA(cellm_.alloc(total_cells_));
    total_iface_ = ifc;
    total_jface_ = jfc;
    BS_CUDA(norm_.alloc(n_));
    BS_CUDA(status_.alloc(n_));
    BS_CUDA(dtmin_.alloc(n_));
    BS_CUDA(cfl_.alloc(n_));
    BS_CUDA(cflmax_.alloc(n_));
    BS_CUDA(growth_.alloc(n_));
    BS_CUDA(omega_.alloc(n_));
    BS_CUDA(bgeom_.alloc(3 * bfc));
    BS_CUDA(bflux_.alloc(4 * size_t(max_along_)));
    BS_CUDA(force_.alloc(1));
    BS_CUDA(cudaMemset(status_.p, 0, n_ * sizeof(unsigned)));
    std::vector<float> ones(n_, 1.f), fifteen(n_, 1.5f);
    BS_CUDA(cudaMemcpy(cfl_.p, ones.data(), n_ * sizeof(float), cudaMemcpyHostToDevice));
    BS_CUDA(cudaMemcpy(cflmax_.p, ones.data(), n_ * sizeof(float), cudaMemcpyHostToDevice));
    BS_CUDA(cudaMemcpy(growth_.p, ones.data(), n_ * sizeof(float), cudaMemcpyHostToDevice));
    BS_CUDA(cudaMemcpy(omega_.p, fifteen.data(), n_ * sizeof(float), cudaMemcpyHostToDevice));
    // Metrics, FP64 on the host, stored FP32 on the device.
    std::vector<float4> fi, fj;
    std::vector<float2> cm;
    std::vector<double> bg(3 * bfc);
    for (int c = 0; c < n_; c++) {
      const Metrics64& m = cases_[c].m;
      const int ni = m.ni, nj = m.nj;
      fi.resize(size_t(ni + 1) * nj);
      for (size_t k = 0; k < fi.size(); k++)
        fi[k] = make_float4(float(m.inx[k]), float(m.iny[k]), float(m.iarea[k]), 0.f);
      fj.resize(size_t(ni) * (nj + 1));
      for (size_t k = 0; k < fj.size(); k++)
        fj[k] = make_float4(float(m.jnx[k]), float(m.jny[k]), float(m.jarea[k]), 0.f);
      cm.resize(size_t(ni) * nj);
      for (size_t k = 0; k < cm.size(); k++)
        cm[k] = make_float2(float(m.volume[k]), float(m.planar[k]));
      BS_CUDA(cudaMemcpy(iface_.p + hc[c].iface, fi.data(), fi.size() * sizeof(float4),
                         cudaMemcpyHostToDevice));
      BS_CUDA(cudaMemcpy(jface_.p + hc[c].jface, fj.data(), fj.size() * sizeof(float4),
                         cudaMemcpyHostToDevice));
      BS_CUDA(cudaMemcpy(cellm_.p + hc[c].cell, cm.data(), cm.size() * sizeof(float2),
                         cudaMemcpyHostToDevice));
      // FP64 boundary geometry, sides in order iMin, iMax, jMin, jMax.
      double* g = bg.data() + 3 * boundary_off_[c];
      for (int s = 0; s < 4; s++) {
        const int along = s < 2 ? nj : ni;
        for (int t = 0; t < along; t++) {
          size_t f;
          if (s < 2) {
            f = (s == 0 ? 0 : ni) + size_t(t) * (ni + 1);
            g[0] = m.inx[f]; g[1] = m.iny[f]; g[2] = m.iarea[f];
          } else {
            f = t + size_t(s == 2 ? 0 : nj) * ni;
            g[0] = m.jnx[f]; g[1] = m.jny[f]; g[2] = m.jarea[f];
          }
          g += 3;
        }
      }
    }
    BS_CUDA(cudaMemcpy(bgeom_.p, bg.data(), bg.size() * sizeof(double), cudaMemcpyHostToDevice));
    hc_ = hc;
    return init_lanes(hc, std::min(n_, kDefaultLanes));
  }

  // Frees the lanes, their streams and events, and every captured graph
  // (whose launches reference the lanes).
  void release_lanes() {
    cudaStreamSynchronize(stream_);
    for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second);
    graphs_.clear();
    graph_launches_.clear();
    for (auto& l : lanes_)
      if (l->stream != nullptr) cudaStreamDestroy(l->stream);
    lanes_.clear();
    for (auto e : ev_join_) cudaEventDestroy(e);
    ev_join_.clear();
    if (ev_fork_ != nullptr) cudaEventDestroy(ev_fork_);
    ev_fork_ = nullptr;
  }

  // Splits the cases into lanes of about equal cell counts. A few cases per
  // lane: largest first, each to the lightest lane. Many: contiguous runs of
  // the cases sorted by width, so that a lane's sweep CTAs share one size
  // class (a sweep launch sizes its shared memory for its widest case).
  bs_status init_lanes(const std::vector<bsd::CaseDev>& hc, int lanes) {
    const int L = std::max(1, std::min({n_, kMaxLanes, lanes}));
    if (L < 2) return BS_OK;
    auto cells = [&](int c) { return int64_t(hc[c].ni) * hc[c].nj; };
    std::vector<int> order(n_);
    for (int c = 0; c < n_; c++) order[c] = c;
    std::vector<std::vector<int>> members(L);
    if (n_ < 4 * L) {
      std::sort(order.begin(), order.end(), [&](int a, int b) { return cells(a) > cells(b); });
      std::vector<int64_t> load(L, 0);
      for (int c : order) {
        const int l = int(std::min_element(load.begin(), load.end()) - load.begin());
        members[l].push_back(c);
        load[l] += cells(c);
      }
    } else {
      std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return hc[a].nj != hc[b].nj ? hc[a].nj > hc[b].nj : cells(a) > cells(b);
      });
      int64_t total = 0;
      for (int c = 0; c < n_; c++) total += cells(c);
      int64_t acc = 0;
      int l = 0;
      for (int k = 0; k < n_; k++) {
        // Move to the next lane once this one has its share, or when the
        // cases left are just enough to give every later lane one.
        const int after = L - 1 - l;
        const bool share = acc >= total * (l + 1) / L;
        if (after > 0 && !members[l].empty() && (share || n_ - k <= after)) l++;
        members[l].push_back(order[k]);
        acc += cells(order[k]);
      }
    }
    for (auto& m : members)
      if (m.empty()) return fail(BS_EXECUTION, "internal error: an empty lane");
    BS_CUDA(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming));
    for (int l = 0; l < L; l++) {
      auto lane = std::make_unique<Lane>();
      std::sort(members[l].begin(), members[l].end());
      std::vector<int2> tiles;
      for (int c : members[l]) {
        const int ti = (hc[c].ni + bsd::TI - 1) / bsd::TI, tj = (hc[c].nj + bsd::TJ - 1) / bsd::TJ;
        for (int t = 0; t < ti * tj; t++) tiles.push_back(make_int2(c, t));
        lane->max_nj = std::max(lane->max_nj, hc[c].nj);
        lane->max_len = std::max(lane->max_len, std::min(hc[c].ni, hc[c].nj));
      }
      lane->n_cases = int(members[l].size());
      lane->n_tiles = int(tiles.size());
      lane->members = members[l];
      BS_CUDA(lane->tiles.alloc(tiles.size()));
      BS_CUDA(cudaMemcpy(lane->tiles.p, tiles.data(), tiles.size() * sizeof(int2), cudaMemcpyHostToDevice));
      BS_CUDA(lane->case_list.alloc(members[l].size()));
      BS_CUDA(cudaMemcpy(lane->case_list.p, members[l].data(), members[l].size() * sizeof(int),
                         cudaMemcpyHostToDevice));
      BS_CUDA(cudaStreamCreateWithFlags(&lane->stream, cudaStreamNonBlocking));
      cudaEvent_t ev;
      BS_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      ev_join_.push_back(ev);
      lanes_.push_back(std::move(lane));
    }
    return build_rtiles();
  }

  int n_cases() const override { return n_; }
  const HostCase& host_case(int c) const override { return cases_[c]; }
  int64_t steps(int c) const override { return steps_[c]; }
  cudaStream_t stream() const override { return stream_; }
  double last_solve_ms() const override { return last_solve_ms_; }
  int64_t last_solve_launches() const override { return last_solve_launches_; }

  bs_status set_primitives(int c, const double* prim) override {
    const HostCase& h = cases_[c];
    const size_t n = size_t(h.cfg.ni) * h.cfg.nj;
    const double g = solve_gamma(h.cfg.gamma);
    std::vector<R> comp[4];
    for (int v = 0; v < 4; v++) comp[v].resize(n);
    for (size_t k = 0; k < n; k++) {
      const double rho = prim[4 * k], u = prim[4 * k + 1], v = prim[4 * k + 2], p = prim[4 * k + 3];
      if (!(rho > 0 && p > 0 && std::isfinite(u) && std::isfinite(v)))
        return fail(BS_NON_PHYSICAL, "non-physical state for cell " + std::to_string(k) +
                                         " (i " + std::to_string(k % h.cfg.ni) + ", j " +
                                         std::to_string(k / h.cfg.ni) + ")");
      comp[0][k] = R(rho);
      comp[1][k] = R(rho * u);
      comp[2][k] = R(rho * v);
      comp[3][k] = R(p / (g - 1) + 0.5 * rho * (u * u + v * v));
    }
    const int64_t off = cell_offset(c);
    for (int v = 0; v < 4; v++)
      BS_CUDA(cudaMemcpyAsync(q_[v].p + off, comp[v].data(), n * sizeof(R), cudaMemcpyHostToDevice,
                              stream_));
    unsigned zero = 0;
    BS_CUDA(cudaMemcpyAsync(status_.p + c, &zero, sizeof(unsigned), cudaMemcpyHostToDevice, stream_));
    BS_CUDA(cudaStreamSynchronize(stream_));
    steps_[c] = 0;
    anderson_stale_ = true;
    return BS_OK;
  }

  bs_status set_free_stream() override {
    for (int c = 0; c < n_; c++) {
      const bs_config& cfg = cases_[c].cfg;
      int side = -1;
      for (int s : {BS_JMAX, BS_IMIN, BS_IMAX, BS_JMIN})
        if (side < 0 && (cfg.boundaries[s].kind == BS_BC_INFLOW ||
                         cfg.boundaries[s].kind == BS_BC_FAR_FIELD))
          side = s;
      if (side < 0) return fail(BS_INVALID_ARGUMENT, "case " + std::to_string(c) + " has no free stream");
      const bs_primitive& w = cfg.boundaries[side].state;
      const size_t n = size_t(cfg.ni) * cfg.nj;
      std::vector<double> prim(4 * n);
      for (size_t k = 0; k < n; k++) {
        prim[4 * k] = w.rho;
        prim[4 * k + 1] = w.u;
        prim[4 * k + 2] = w.v;
        prim[4 * k + 3] = w.p;
      }
      BS_TRY(set_primitives(c, prim.data()));
    }
    return BS_OK;
  }

  // The residual-pass tile lists (whole batch and every lane) for rshape_.
  bs_status build_rtiles() {
    if (rshape_ < 0) return BS_OK;
    const bsd::TileShape sh = bsd::tile_shape(rshape_);
    std::vector<int> all(n_);
    for (int c = 0; c < n_; c++) all[c] = c;
    std::vector<int2> t = tiles_for(hc_, all, sh.ti, sh.tj);
    BS_CUDA(d_rtiles_.alloc(t.size()));
    BS_CUDA(cudaMemcpy(d_rtiles_.p, t.data(), t.size() * sizeof(int2), cudaMemcpyHostToDevice));
    n_rtiles_ = int(t.size());
    for (auto& l : lanes_) {
      t = tiles_for(hc_, l->members, sh.ti, sh.tj);
      BS_CUDA(l->rtiles.alloc(t.size()));
      BS_CUDA(cudaMemcpy(l->rtiles.p, t.data(), t.size() * sizeof(int2), cudaMemcpyHostToDevice));
      l->n_rtiles = int(t.size());
    }
    return BS_OK;
  }

  bs_status set_tile_shape(int shape) override {
    if (shape < -1 || shape >= bsd::kTileShapes)
      return fail(BS_INVALID_ARGUMENT, "tile shape: -1 (default) or 0 .. " + std::to_string(bsd::kTileShapes - 1));
    if (shape >= 0 && sizeof(R) != sizeof(double))
      return fail(BS_INVALID_ARGUMENT, "the all-FP32 engine keeps the default tile shape");
    BS_CUDA(cudaStreamSynchronize(stream_));
    rshape_ = shape;
    BS_TRY(build_rtiles());
    // Captured graphs hold the old launches.
    for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second);
    graphs_.clear();
    graph_launches_.clear();
    return BS_OK;
  }

  int tile_shape() const override { return rshape_; }

  bs_status set_fused_update(bool fused) override {
    BS_CUDA(cudaStreamSynchronize(stream_));
    fuse_update_ = fused;
    // Captured graphs hold the old launches.
    for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second);
    graphs_.clear();
    graph_launches_.clear();
    return BS_OK;
  }

  bool fused_update() const override { return fuse_update_; }

  // Times `steps` steps from the current state with 1, 2, 4, ... lanes (up to
  // 64 and the case count), then, with the fastest lane count, each tile shape
  // of the residual pass (FP64 batches), each run after one untimed run that
  // captures its graphs, restoring the state before every run; keeps the
  // fastest. The state, CFL numbers and status words are as before the call.
  bs_status autotune(int method, int steps, double cfl, double omega, int* lanes, double* ms_per_step) override {
    if (steps < 1) return fail(BS_INVALID_ARGUMENT, "autotune needs steps >= 1");
    if (method == kMethodImplicit) {
      if (!(cfl > 0 && omega >= 1)) return fail(BS_INVALID_ARGUMENT, "LU-SGS needs cfl > 0 and omega >= 1");
      BS_TRY(ensure_implicit());
      BS_TRY(set_implicit_params(cfl, omega, 1.0));
    } else {
      BS_TRY(ensure_explicit());
    }
    DevBuf<R> saved[4];
    for (int v = 0; v < 4; v++) {
      BS_CUDA(saved[v].alloc(total_cells_));
      BS_CUDA(cudaMemcpyAsync(saved[v].p, q_[v].p, total_cells_ * sizeof(R), cudaMemcpyDeviceToDevice, stream_));
    }
    auto restore = [&]() -> bs_status {
      for (int v = 0; v < 4; v++)
        BS_CUDA(cudaMemcpyAsync(q_[v].p, saved[v].p, total_cells_ * sizeof(R), cudaMemcpyDeviceToDevice, stream_));
      if (method == kMethodImplicit) BS_TRY(set_implicit_cfl(cfl));
      BS_CUDA(cudaMemsetAsync(status_.p, 0, n_ * sizeof(unsigned), stream_));
      return BS_OK;
    };
    std::fill(active_h_.begin(), active_h_.end(), 1);
    BS_TRY(upload_active());
    int best = 0;
    double best_ms = 0;
    for (int L = 1; L <= std::min(n_, kMaxLanes); L *= 2) {
      release_lanes();
      BS_TRY(init_lanes(hc_, L));
      BS_TRY(restore());
      BS_TRY(run_steps(method, steps, false));
      BS_TRY(restore());
      BS_CUDA(cudaEventRecord(ev0_, stream_));
      BS_TRY(run_steps(method, steps, false));
      BS_CUDA(cudaEventRecord(ev1_, stream_));
      BS_CUDA(cudaEventSynchronize(ev1_));
      float t = 0;
      BS_CUDA(cudaEventElapsedTime(&t, ev0_, ev1_));
      if (best == 0 || t < best_ms) {
        best = L;
        best_ms = t;
      }
    }
    release_lanes();
    BS_TRY(init_lanes(hc_, best));
    // Then the residual pass's tile shape, with those lanes (FP64 batches;
    // -1 is the untuned default).
    if (sizeof(R) == sizeof(double)) {
      const int before = rshape_;
      int best_shape = before;
      for (int k = -1; k < bsd::kTileShapes; k++) {
        BS_TRY(set_tile_shape(k));
        BS_TRY(restore());
        BS_TRY(run_steps(method, steps, false));
        BS_TRY(restore());
        BS_CUDA(cudaEventRecord(ev0_, stream_));
        BS_TRY(run_steps(method, steps, false));
        BS_CUDA(cudaEventRecord(ev1_, stream_));
        BS_CUDA(cudaEventSynchronize(ev1_));
        float t = 0;
        BS_CUDA(cudaEventElapsedTime(&t, ev0_, ev1_));
        if (t < best_ms) {
          best_ms = t;
          best_shape = k;
        }
      }
      BS_TRY(set_tile_shape(best_shape));
    }
    // Then, for LU-SGS, the update fused into the residual pass (fewer
    // launches, the latency-bound case) or a separate update kernel (less
    // work per step: the fused pass updates each halo cell again, which a
    // batch that fills the GPU pays for).
    if (method == kMethodImplicit) {
      float t_mode[2] = {0.f, 0.f};  // [0] separate update, [1] fused
      for (int fused = 1; fused >= 0; fused--) {
        BS_TRY(set_fused_update(fused == 1));
        BS_TRY(restore());
        BS_TRY(run_steps(method, steps, false));
        BS_TRY(restore());
        BS_CUDA(cudaEventRecord(ev0_, stream_));
        BS_TRY(run_steps(method, steps, false));
        BS_CUDA(cudaEventRecord(ev1_, stream_));
        BS_CUDA(cudaEventSynchronize(ev1_));
        BS_CUDA(cudaEventElapsedTime(&t_mode[fused], ev0_, ev1_));
      }
      BS_TRY(set_fused_update(t_mode[1] <= t_mode[0]));
      best_ms = std::min(t_mode[0], t_mode[1]);
    }
    BS_TRY(restore());
    BS_CUDA(cudaStreamSynchronize(stream_));
    *lanes = best;
    *ms_per_step = best_ms / steps;
    return BS_OK;
  }

  int lanes() const override { return std::max<int>(1, int(lanes_.size())); }

  bs_status set_lanes(int lanes) override {
    if (lanes < 1 || lanes > std::min(n_, kMaxLanes))
      return fail(BS_INVALID_ARGUMENT, "lanes: 1 .. " + std::to_string(std::min(n_, kMaxLanes)));
    release_lanes();
    return init_lanes(hc_, lanes);
  }

  bs_status flow_field(int c, int field, const bs_primitive& free, double length, double* out) override {
    if (field < bsd::FIELD_SCHLIEREN || field > bsd::FIELD_DENSITY)
      return fail(BS_INVALID_ARGUMENT, "field: 0 schlieren, 1 mach, 2 cp, 3 density");
    if (!(free.rho > 0 && free.p > 0)) return fail(BS_INVALID_ARGUMENT, "free stream density and pressure must be positive");
    if (nodes_x_.p == nullptr) {
      // The grids' nodes, uploaded on first use (the solve needs only metrics).
      node_off_.assign(n_, 0);
      int64_t total = 0;
      for (int k = 0; k < n_; k++) {
        node_off_[k] = total;
        total += int64_t(cases_[k].x.size());
      }
      BS_CUDA(nodes_x_.alloc(total));
      BS_CUDA(nodes_y_.alloc(total));
      for (int k = 0; k < n_; k++) {
        BS_CUDA(cudaMemcpy(nodes_x_.p + node_off_[k], cases_[k].x.data(), cases_[k].x.size() * sizeof(double),
                           cudaMemcpyHostToDevice));
        BS_CUDA(cudaMemcpy(nodes_y_.p + node_off_[k], cases_[k].y.data(), cases_[k].y.size() * sizeof(double),
                           cudaMemcpyHostToDevice));
      }
    }
    const int64_t cells = int64_t(cases_[c].cfg.ni) * cases_[c].cfg.nj;
    DevBuf<double> d_out;
    BS_CUDA(d_out.alloc(cells));
    bsd::flow_field_kernel<R><<<unsigned((cells + 255) / 256), 256, 0, stream_>>>(
        d_cases_.p, c, q_view(), nodes_x_.p + node_off_[c], nodes_y_.p + node_off_[c], field, length, free.rho,
        free.u, free.v, free.p, d_out.p);
    BS_CUDA(cudaGetLastError());
    BS_CUDA(cudaMemcpyAsync(out, d_out.p, cells * sizeof(double), cudaMemcpyDeviceToHost, stream_));
    BS_CUDA(cudaStreamSynchronize(stream_));
    return BS_OK;
  }

  bs_status set_active(const int* flags) override {
    for (int c = 0; c < n_; c++) active_h_[c] = flags[c] != 0 ? 1 : 0;
    return upload_active();
  }

  bs_status kernel_times(int method, double cfl, double omega, int iterations, double* ms) override {
    if (iterations < 1) return fail(BS_INVALID_ARGUMENT, "iterations must be positive");
    cudaEvent_t ev[6];
    for (auto& e : ev) BS_CUDA(cudaEventCreate(&e));
    double sum[3] = {0, 0, 0};
    bs_status st = BS_OK;
    if (method == kMethodImplicit) {
      st = ensure_implicit();
      if (st == BS_OK) st = set_implicit_params(cfl, omega, 1.0);
      if (st == BS_OK) st = set_implicit_cfl(cfl);
      // One untimed residual pass and sweep give the timed passes a correction to apply.
      const bsd::StateView<R> q = q_view();
      if (st == BS_OK) st = launch_tile<bsd::MODE_PREPARE>(q, q, q, 0, 1, false, nullptr, nullptr, false);
      if (st == BS_OK) st = launch_sweep();
    } else {
      st = ensure_explicit();
    }
    for (int it = 0; it < iterations && st == BS_OK; it++) {
      cudaEventRecord(ev[0], stream_);
      if (method == kMethodImplicit) {
        // A step's residual pass with the previous step's update fused in
        // (read from q, written to the other buffer, so q stays as it was),
        // the sweeps, and a run's closing update (out of place as well).
        const bsd::StateView<R> q = q_view(), qb = qb_view();
        st = launch_tile<bsd::MODE_PREPARE>(q, q, q, 0, 1, false, norm_.p, nullptr, false, dq_.p, qb);
        cudaEventRecord(ev[1], stream_);
        cudaEventRecord(ev[2], stream_);
        if (st == BS_OK) st = launch_sweep();
        cudaEventRecord(ev[3], stream_);
        cudaEventRecord(ev[4], stream_);
        if (st == BS_OK) st = launch_update_on(whole(), q, qb);
      } else {
        const bsd::StateView<R> q = q_view(), s1 = s1_view(), s2 = s2_view();
        st = launch_tile<bsd::MODE_STAGE>(q, q, s1, 0.0, 1.0, true, norm_.p, nullptr, false);
        cudaEventRecord(ev[1], stream_);
        cudaEventRecord(ev[2], stream_);
        if (st == BS_OK) st = launch_tile<bsd::MODE_STAGE>(s1, q, s2, 0.75, 0.25, false, nullptr, nullptr, false);
        cudaEventRecord(ev[3], stream_);
        cudaEventRecord(ev[4], stream_);
      }
      cudaEventRecord(ev[5], stream_);
      const cudaError_t e = cudaEventSynchronize(ev[5]);
      if (e != cudaSuccess) {
        st = cuda_fail(e, "kernel timing");
        break;
      }
      float a = 0, b = 0, u = 0;
      cudaEventElapsedTime(&a, ev[0], ev[1]);
      cudaEventElapsedTime(&b, ev[2], ev[3]);
      cudaEventElapsedTime(&u, ev[4], ev[5]);
      sum[0] += a;
      sum[1] += b;
      sum[2] += u;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (st != BS_OK) return st;
    for (int k = 0; k < 3; k++) ms[k] = sum[k] / iterations;
    return BS_OK;
  }

  bs_status iterate(int steps) override {
    if (steps < 0) return fail(BS_INVALID_ARGUMENT, "steps must be non-negative");
    BS_TRY(ensure_explicit());
    BS_TRY(run_steps(kMethodExplicit, steps, false));
    count_steps(steps);
    return check_status();
  }

  bs_status set_implicit_cfl(double cfl) override {
    if (!(cfl > 0)) return fail(BS_INVALID_ARGUMENT, "the CFL number must be positive");
    std::vector<float> v(n_, float(cfl));
    BS_CUDA(cudaMemcpyAsync(cfl_.p, v.data(), n_ * sizeof(float), cudaMemcpyHostToDevice, stream_));
    BS_CUDA(cudaStreamSynchronize(stream_));
    return BS_OK;
  }

  bs_status iterate_implicit(int steps, double cfl_max, double omega, double growth) override {
    if (steps < 0) return fail(BS_INVALID_ARGUMENT, "steps must be non-negative");
    if (!(cfl_max > 0 && omega >= 1 && growth >= 1))
      return fail(BS_INVALID_ARGUMENT, "implicit steps need cfl > 0, omega >= 1 and growth >= 1");
    BS_TRY(ensure_implicit());
    BS_TRY(set_implicit_params(cfl_max, omega, growth));
    BS_TRY(run_steps(kMethodImplicit, steps, false));
    count_steps(steps);
    return check_status();
  }

  // LU-SGS steps with the Anderson settings of set_anderson applied, the
  // acceleration's history kept from one call to the next: plain steps until
  // anderson_plain_ steps have been taken since the history was last reset
  // (by setting the state or the settings), accelerated ones after, as
  // solveTransonic steps (src/analysis/transonic-flow.ts:151-245).
  bs_status iterate_accelerated(int steps, double cfl_max, double omega, double growth) override {
    if (steps < 0) return fail(BS_INVALID_ARGUMENT, "steps must be non-negative");
    if (!(cfl_max > 0 && omega >= 1 && growth >= 1))
      return fail(BS_INVALID_ARGUMENT, "implicit steps need cfl > 0, omega >= 1 and growth >= 1");
    BS_TRY(ensure_implicit());
    BS_TRY(set_implicit_params(cfl_max, omega, growth));
    if (anderson_depth_ == 0) {
      BS_TRY(run_steps(kMethodImplicit, steps, false));
    } else {
      if (anderson_stale_) {
        BS_TRY(reset_anderson());
        anderson_stale_ = false;
        accelerated_steps_ = 0;
      }
      const int plain =
          int(std::max<int64_t>(0, std::min<int64_t>(steps, anderson_plain_ - accelerated_steps_)));
      if (plain > 0) BS_TRY(run_steps(kMethodImplicit, plain, false));
      if (steps > plain) BS_TRY(run_steps(kMethodAnderson, steps - plain, false));
      accelerated_steps_ += steps;
    }
    count_steps(steps);
    return check_status();
  }

  // Two-float metrics (bits 64): the FP32 low part of every face normal,
  // area, cell volume and planar area, which the residual and the ghost cells
  // add to the FP32 values, as the reference's two-float engine stores its
  // metrics (src/engine-gpu/euler2d-two-float.ts:584-605); the LU-SGS
  // operator and the time steps keep the FP32 values. Bits 32: FP32 metrics.
  bs_status set_metric_precision(int bits) override {
    if (bits != 32 && bits != 64) return fail(BS_INVALID_ARGUMENT, "metric precision is 32 or 64 bits");
    if (bits == 64 && sizeof(R) != sizeof(double))
      return fail(BS_INVALID_ARGUMENT, "the all-FP32 engine keeps FP32 metrics");
    const bool on = bits == 64;
    if (on == metrics_lo_) return BS_OK;
    BS_CUDA(cudaStreamSynchronize(stream_));
    if (on && iface_lo_.p == nullptr) {
      BS_CUDA(iface_lo_.alloc(total_iface_));
      BS_CUDA(jface_lo_.alloc(total_jface_));
      BS_CUDA(cellm_lo_.alloc(total_cells_));
      auto lo = [](double v) { return float(v - double(float(v))); };
      std::vector<float4> fi, fj;
      std::vector<float2> cm;
      for (int c = 0; c < n_; c++) {
        const Metrics64& m = cases_[c].m;
        fi.resize(m.inx.size());
        for (size_t k = 0; k < fi.size(); k++) fi[k] = make_float4(lo(m.inx[k]), lo(m.iny[k]), lo(m.iarea[k]), 0.f);
        fj.resize(m.jnx.size());
        for (size_t k = 0; k < fj.size(); k++) fj[k] = make_float4(lo(m.jnx[k]), lo(m.jny[k]), lo(m.jarea[k]), 0.f);
        cm.resize(m.volume.size());
        for (size_t k = 0; k < cm.size(); k++) cm[k] = make_float2(lo(m.volume[k]), lo(m.planar[k]));
        BS_CUDA(cudaMemcpy(iface_lo_.p + hc_[c].iface, fi.data(), fi.size() * sizeof(float4),
                           cudaMemcpyHostToDevice));
        BS_CUDA(cudaMemcpy(jface_lo_.p + hc_[c].jface, fj.data(), fj.size() * sizeof(float4),
                           cudaMemcpyHostToDevice));
        BS_CUDA(cudaMemcpy(cellm_lo_.p + hc_[c].cell, cm.data(), cm.size() * sizeof(float2),
                           cudaMemcpyHostToDevice));
      }
    }
    metrics_lo_ = on;
    // Captured graphs hold the old metric views.
    for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second);
    graphs_.clear();
    graph_launches_.clear();
    return BS_OK;
  }

  bs_status residual_norms(double* norms) override {
    BS_CUDA(cudaMemsetAsync(norm_.p, 0, n_ * sizeof(double), stream_));
    BS_TRY(launch_tile<bsd::MODE_RESIDUAL>(q_view(), q_view(), q_view(), 0, 1, false, norm_.p,
                                           nullptr, true));
    std::vector<double> s(n_);
    BS_CUDA(cudaMemcpyAsync(s.data(), norm_.p, n_ * sizeof(double), cudaMemcpyDeviceToHost, stream_));
    BS_CUDA(cudaStreamSynchronize(stream_));
    for (int c = 0; c < n_; c++)
      norms[c] = std::sqrt(s[c] / (double(cases_[c].cfg.ni) * cases_[c].cfg.nj));
    return BS_OK;
  }

  bs_status residual(int c, double* out) override {
    if (res_out_.p == nullptr) BS_CUDA(res_out_.alloc(4 * size_t(total_cells_)));
    BS_TRY(launch_tile<bsd::MODE_RESIDUAL>(q_view(), q_view(), q_view(), 0, 1, false, nullptr,
                                           res_out_.p, true));
    const size_t n = size_t(cases_[c].cfg.ni) * cases_[c].cfg.nj;
    BS_CUDA(cudaMemcpyAsync(out, res_out_.p + 4 * cell_offset(c), 4 * n * sizeof(double),
                            cudaMemcpyDeviceToHost, stream_));
    BS_CUDA(cudaStreamSynchronize(stream_));
    return BS_OK;
  }

  bs_status time_steps(int c, double* out) override {
    bsd::dt_kernel<R><<<n_tiles_, bsd::TILE_THREADS, 0, stream_>>>(
        d_cases_.p, d_tiles_.p, nullptr, q_view(), metrics(), dt_.p, nullptr);
    BS_CUDA(cudaGetLastError());
    const size_t n = size_t(cases_[c].cfg.ni) * cases_[c].cfg.nj;
    std::vector<float> d(n);
    BS_CUDA(cudaMemcpyAsync(d.data(), dt_.p + cell_offset(c), n * sizeof(float),
                            cudaMemcpyDeviceToHost, stream_));
    BS_CUDA(cudaStreamSynchronize(stream_));
    for (size_t k = 0; k < n; k++) out[k] = d[k];
    return BS_OK;
  }

  bs_status boundary_fluxes(int c, int side, bs_face_flux* out) override {
    if (side < 0 || side > 3) return fail(BS_INVALID_ARGUMENT, "unknown side");
    const HostCase& h = cases_[c];
    const int ni = h.cfg.ni, nj = h.cfg.nj;
    const int along = side < 2 ? nj : ni;
    BS_TRY(launch_boundary(c, side, 0.0, false));
    std::vector<double> f(4 * size_t(along));
    BS_CUDA(cudaMemcpyAsync(f.data(), bflux_.p, f.size() * sizeof(double), cudaMemcpyDeviceToHost,
                            stream_));
    BS_CUDA(cudaStreamSynchronize(stream_));
    const int outward = (side == BS_IMIN || side == BS_JMIN) ? -1 : 1;
    const Metrics64& m = h.m;
    for (int t = 0; t < along; t++) {
      size_t n0, n1;
      double nx, ny, area;
      if (side < 2) {
        const int i = side == BS_IMIN ? 0 : ni;
        const size_t fidx = i + size_t(t) * (ni + 1);
        n0 = fidx;
        n1 = fidx + ni + 1;
        nx = m.inx[fidx]; ny = m.iny[fidx]; area = m.iarea[fidx];
      } else {
        const int j = side == BS_JMIN ? 0 : nj;
        const size_t fidx = t + size_t(j) * ni;
        n0 = t + size_t(j) * (ni + 1);
        n1 = n0 + 1;
        nx = m.jnx[fidx]; ny = m.jny[fidx]; area = m.jarea[fidx];
      }
      bs_face_flux& o = out[t];
      o.x = 0.5 * (h.x[n0] + h.x[n1]);
      o.y = 0.5 * (h.y[n0] + h.y[n1]);
      o.nx = outward * nx;
      o.ny = outward * ny;
      o.area = area;
      for (int v = 0; v < 4; v++) o.flux[v] = f[4 * t + v];
    }
    return BS_OK;
  }

  bs_status forebody_drag(int c, double p_inf, double q_inf, double base_radius,
                          double* drag) override {
    BS_TRY(launch_boundary(c, BS_JMIN, p_inf, true));
    double force = 0;
    BS_CUDA(cudaMemcpyAsync(&force, force_.p, sizeof(double), cudaMemcpyDeviceToHost, stream_));
    BS_CUDA(cudaStreamSynchronize(stream_));
    *drag = (2 * force) / (q_inf * base_radius * base_radius);
    return BS_OK;
  }

  bs_status read_state(int c, float* out) override {
    const size_t n = size_t(cases_[c].cfg.ni) * cases_[c].cfg.nj;
    std::vector<R> comp[4];
    BS_TRY(copy_state(c, comp));
    for (size_t k = 0; k < n; k++)
      for (int v = 0; v < 4; v++) out[4 * k + v] = float(comp[v][k]);
    return BS_OK;
  }

  bs_status read_primitives(int c, double* out) override {
    const size_t n = size_t(cases_[c].cfg.ni) * cases_[c].cfg.nj;
    std::vector<R> comp[4];
    BS_TRY(copy_state(c, comp));
    const double g = solve_gamma(cases_[c].cfg.gamma);
    for (size_t k = 0; k < n; k++) {
      const double rho = comp[0][k], mu = comp[1][k], mv = comp[2][k], e = comp[3][k];
      out[4 * k] = rho;
      out[4 * k + 1] = mu / rho;
      out[4 * k + 2] = mv / rho;
      out[4 * k + 3] = (g - 1) * (e - (0.5 * (mu * mu + mv * mv)) / rho);
    }
    return BS_OK;
  }

  bs_status set_anderson(int depth, int plain_steps) override {
    if (depth < 0 || depth > bsd::kMaxAndersonDepth || plain_steps < 0)
      return fail(BS_INVALID_ARGUMENT, "Anderson acceleration keeps 0 to 16 differences after plain_steps >= 0");
    anderson_depth_ = depth;
    anderson_plain_ = plain_steps;
    anderson_stale_ = true;
    return BS_OK;
  }

  bs_status set_sweep_wait_limit(int polls) override {
    if (polls < -1) return fail(BS_INVALID_ARGUMENT, "the wait limit is -1 (default) or a number of polls");
    if (polls == sweep_wait_limit_) return BS_OK;
    BS_CUDA(cudaStreamSynchronize(stream_));
    sweep_wait_limit_ = polls;
    // Captured graphs hold the old limit.
    for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second);
    graphs_.clear();
    graph_launches_.clear();
    return BS_OK;
  }

  bs_status anderson_restarts(int* out) override {
    if (ac_.p == nullptr) {
      for (int c = 0; c < n_; c++) out[c] = 0;
      return BS_OK;
    }
    std::vector<bsd::AndersonCase> h(n_);
    BS_CUDA(cudaMemcpyAsync(h.data(), ac_.p, n_ * sizeof(bsd::AndersonCase), cudaMemcpyDeviceToHost, stream_));
    BS_CUDA(cudaStreamSynchronize(stream_));
    for (int c = 0; c < n_; c++) out[c] = h[c].restarts;
    return BS_OK;
  }

  bs_status solve(int method, double cfl, double omega, double tolerance, int relative,
                  int max_steps, int check_every, std::vector<CaseResult>& results) override {
    if (!(tolerance > 0) || max_steps < 0 || check_every < 1)
      return fail(BS_INVALID_ARGUMENT, "a solve needs tolerance > 0, max_steps >= 0, check_every >= 1");
    if (method == kMethodImplicit) {
      if (!(cfl > 0 && omega >= 1))
        return fail(BS_INVALID_ARGUMENT, "LU-SGS needs cfl > 0 and omega >= 1");
      BS_TRY(ensure_implicit());
      BS_TRY(set_implicit_params(cfl, omega, 1.0));
      BS_TRY(set_implicit_cfl(cfl));
      if (anderson_depth_ > 0) BS_TRY(reset_anderson());
      // A later iterate_accelerated starts its own history.
      anderson_stale_ = true;
    } else {
      BS_TRY(ensure_explicit());
    }
    const bool accelerate = method == kMethodImplicit && anderson_depth_ > 0;
    results.assign(n_, CaseResult{});
    launches_ = 0;
    BS_CUDA(cudaEventRecord(ev0_, stream_));
    std::vector<double> r0(n_);
    BS_TRY(residual_norms(r0.data()));
    std::vector<double> target(n_);
    for (int c = 0; c < n_; c++) {
      results[c].initial_residual = r0[c];
      results[c].residual = r0[c];
      target[c] = relative ? tolerance * r0[c] : tolerance;
      active_h_[c] = r0[c] <= target[c] ? 0 : 1;
      results[c].status = active_h_[c] ? BS_NOT_CONVERGED : BS_OK;
    }
    BS_TRY(upload_active());
    std::vector<int64_t> taken(n_, 0);
    std::vector<double> sums(n_);
    std::vector<unsigned> status(n_);
    int done = 0;
    for (int c = 0; c < n_; c++) done += active_h_[c] == 0;
    int64_t step = 0;
    std::vector<double> rf(n_);
    bool any_timeout = false;
    for (;;) {
    while (done < n_ && step < max_steps) {
      const int chunk = int(std::min<int64_t>(check_every, max_steps - step));
      BS_CUDA(cudaMemsetAsync(norm_.p, 0, n_ * sizeof(double), stream_));
      if (accelerate) {
        // Plain steps up to anderson_plain_, accelerated ones after.
        const int plain = int(std::max<int64_t>(0, std::min<int64_t>(chunk, anderson_plain_ - step)));
        if (plain > 0) BS_TRY(run_steps(kMethodImplicit, plain, plain == chunk));
        if (chunk > plain) BS_TRY(run_steps(kMethodAnderson, chunk - plain, true));
      } else {
        BS_TRY(run_steps(method, chunk, true));
      }
      step += chunk;
      BS_CUDA(cudaMemcpyAsync(sums.data(), norm_.p, n_ * sizeof(double), cudaMemcpyDeviceToHost, stream_));
      BS_CUDA(cudaMemcpyAsync(status.data(), status_.p, n_ * sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
      BS_CUDA(cudaStreamSynchronize(stream_));
      bool changed = false;
      for (int c = 0; c < n_; c++) {
        if (!active_h_[c]) continue;
        taken[c] += chunk;
        steps_[c] += chunk;
        // The residual of the state at the start of the chunk's last step.
        const double r = std::sqrt(sums[c] / (double(cases_[c].cfg.ni) * cases_[c].cfg.nj));
        results[c].residual = r;
        if (status[c] & bsd::STATUS_TIMEOUT) {
          // A sweep gave up waiting for its records: the case keeps the
          // state of its last complete step and stops.
          results[c].status = BS_EXECUTION;
          active_h_[c] = 0;
          any_timeout = true;
        } else if (status[c] & bsd::STATUS_NON_PHYSICAL) {
          results[c].status = BS_NON_PHYSICAL;
          active_h_[c] = 0;
        } else if (!(r == r)) {
          results[c].status = BS_NON_PHYSICAL;
          active_h_[c] = 0;
        } else if (r <= target[c]) {
          results[c].status = BS_OK;
          active_h_[c] = 0;
        }
        if (!active_h_[c]) {
          done++;
          changed = true;
        }
      }
      if (changed) BS_TRY(upload_active());
    }
    // The exact residual of each final state. The check above reads the
    // residual of the state at the start of a chunk's last step; a case it
    // passed whose returned state still misses the target marches on.
    BS_TRY(residual_norms(rf.data()));
    bool again = false;
    for (int c = 0; c < n_; c++)
      if (results[c].status == BS_OK && !(rf[c] <= target[c]) && step < max_steps) {
        results[c].status = BS_NOT_CONVERGED;
        active_h_[c] = 1;
        done--;
        again = true;
      }
    if (!again) break;
    BS_TRY(upload_active());
    }
    for (int c = 0; c < n_; c++) active_h_[c] = 1;
    BS_TRY(upload_active());
    if (any_timeout) {
      std::vector<unsigned> st(n_);
      BS_CUDA(cudaMemcpyAsync(st.data(), status_.p, n_ * sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
      BS_CUDA(cudaStreamSynchronize(stream_));
      BS_TRY(clear_timeouts(st));
    }
    BS_CUDA(cudaEventRecord(ev1_, stream_));
    BS_CUDA(cudaEventSynchronize(ev1_));
    float ms = 0;
    BS_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
    last_solve_ms_ = ms;
    last_solve_launches_ = launches_;
    for (int c = 0; c < n_; c++) {
      results[c].steps = taken[c];
      results[c].residual = rf[c];
      if (results[c].status == BS_OK && !(rf[c] <= target[c])) results[c].status = BS_NOT_CONVERGED;
    }
    return BS_OK;
  }

 private:
  static double solve_gamma(double gamma) {
    // An FP32 field is solved with gamma rounded to FP32, as the reference GPU does.
    return sizeof(R) == 4 ? double(float(gamma)) : gamma;
  }

  int64_t cell_offset(int c) const { return cell_off_[c]; }

  void count_steps(int steps) {
    for (int c = 0; c < n_; c++)
      if (active_h_[c]) steps_[c] += steps;
  }

  bsd::StateView<R> q_view() const { return {q_[0].p, q_[1].p, q_[2].p, q_[3].p}; }
  bsd::StateView<R> s1_view() const { return {s1_[0].p, s1_[1].p, s1_[2].p, s1_[3].p}; }
  // The other buffer of the state, which LU-SGS steps alternate with q.
  bsd::StateView<R> qb_view() const { return {qb_[0].p, qb_[1].p, qb_[2].p, qb_[3].p}; }
  bsd::StateView<R> s2_view() const { return {s2_[0].p, s2_[1].p, s2_[2].p, s2_[3].p}; }
  bsd::MetricsView metrics() const {
    bsd::MetricsView m{iface_.p, jface_.p, cellm_.p};
    if (metrics_lo_) {
      m.iface_lo = iface_lo_.p;
      m.jface_lo = jface_lo_.p;
      m.cell_lo = cellm_lo_.p;
    }
    return m;
  }

  bs_status ensure_explicit() {
    if (s1_[0].p != nullptr) return BS_OK;
    for (int v = 0; v < 4; v++) {
      BS_CUDA(s1_[v].alloc(total_cells_));
      BS_CUDA(s2_[v].alloc(total_cells_));
    }
    return BS_OK;
  }

  bs_status ensure_implicit() {
    if (rec_f_.p != nullptr) return BS_OK;
    // The sweep indexes a case's anti-diagonals in 32 bits.
    for (const auto& c : hc_)
      if (c.ni + c.nj > 65536)
        return fail(BS_INVALID_ARGUMENT, "the LU-SGS sweep takes grids of at most 65536 cells along plus across (ni + nj)");
    BS_CUDA(rec_f_.alloc(bsd::REC_SIZE * size_t(total_slots_)));
    BS_CUDA(rec_b_.alloc(bsd::REC_SIZE * size_t(total_slots_)));
    BS_CUDA(dq_.alloc(total_cells_));
    for (int v = 0; v < 4; v++) BS_CUDA(qb_[v].alloc(total_cells_));
    return BS_OK;
  }

  // The acceleration's arrays for the current depth, and a fresh history:
  // no columns, no previous iterate, |f|^2's smallest value +inf.
  bs_status reset_anderson() {
    const int m = anderson_depth_;
    if (anderson_alloc_depth_ != m) {
      BS_CUDA(adx_.alloc(size_t(m) * total_cells_));
      BS_CUDA(adf_.alloc(size_t(m) * total_cells_));
      BS_CUDA(alastf_.alloc(total_cells_));
      for (int v = 0; v < 4; v++) BS_CUDA(alastx_[v].alloc(total_cells_));
      BS_CUDA(ac_.alloc(n_));
      BS_CUDA(aacc_.alloc(size_t(n_tiles_) * (1 + 2 * m)));
      BS_CUDA(agram_.alloc(size_t(n_) * m * m));
      BS_CUDA(agamma_.alloc(size_t(n_) * m));
      anderson_alloc_depth_ = m;
      // Graphs of accelerated steps hold the old arrays.
      for (auto it = graphs_.begin(); it != graphs_.end();) {
        if (it->first.method == kMethodAnderson) {
          cudaGraphExecDestroy(it->second);
          graph_launches_.erase(it->first);
          it = graphs_.erase(it);
        } else {
          ++it;
        }
      }
    }
    bsd::AndersonCase fresh{};
    fresh.best = HUGE_VAL;
    std::vector<bsd::AndersonCase> h(n_, fresh);
    BS_CUDA(cudaMemcpyAsync(ac_.p, h.data(), n_ * sizeof(bsd::AndersonCase), cudaMemcpyHostToDevice, stream_));
    BS_CUDA(cudaMemsetAsync(agram_.p, 0, size_t(n_) * m * m * sizeof(double), stream_));
    BS_CUDA(cudaMemsetAsync(agamma_.p, 0, size_t(n_) * m * sizeof(double), stream_));
    BS_CUDA(cudaStreamSynchronize(stream_));
    return BS_OK;
  }

  bs_status set_implicit_params(double cfl_max, double omega, double growth) {
    std::vector<float> a(n_, float(cfl_max)), b(n_, float(omega)), g(n_, float(growth));
    BS_CUDA(cudaMemcpyAsync(cflmax_.p, a.data(), n_ * sizeof(float), cudaMemcpyHostToDevice, stream_));
    BS_CUDA(cudaMemcpyAsync(omega_.p, b.data(), n_ * sizeof(float), cudaMemcpyHostToDevice, stream_));
    BS_CUDA(cudaMemcpyAsync(growth_.p, g.data(), n_ * sizeof(float), cudaMemcpyHostToDevice, stream_));
    BS_CUDA(cudaStreamSynchronize(stream_));
    return BS_OK;
  }

  bs_status upload_active() {
    BS_CUDA(cudaMemcpyAsync(d_active_.p, active_h_.data(), n_ * sizeof(int), cudaMemcpyHostToDevice,
                            stream_));
    BS_CUDA(cudaStreamSynchronize(stream_));
    return BS_OK;
  }

  // Clears the timeout bits of the status words `st` read from the device.
  bs_status clear_timeouts(std::vector<unsigned>& st) {
    for (auto& v : st) v &= ~bsd::STATUS_TIMEOUT;
    BS_CUDA(cudaMemcpyAsync(status_.p, st.data(), n_ * sizeof(unsigned), cudaMemcpyHostToDevice, stream_));
    BS_CUDA(cudaStreamSynchronize(stream_));
    return BS_OK;
  }

  bs_status check_status() {
    std::vector<unsigned> st(n_);
    BS_CUDA(cudaMemcpyAsync(st.data(), status_.p, n_ * sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
    BS_CUDA(cudaStreamSynchronize(stream_));
    for (int c = 0; c < n_; c++)
      if (st[c] & bsd::STATUS_TIMEOUT) {
        BS_TRY(clear_timeouts(st));
        return fail(BS_EXECUTION, "the LU-SGS sweep of case " + std::to_string(c) +
                                      " gave up waiting for its records; the step was not applied in full");
      }
    for (int c = 0; c < n_; c++)
      if (st[c] & bsd::STATUS_NON_PHYSICAL)
        return fail(BS_NON_PHYSICAL, "the GPU solution of case " + std::to_string(c) +
                                         " became non-physical");
    return BS_OK;
  }

  LaneView whole() const {
    return {d_tiles_.p, n_tiles_, d_case_list_.p, n_, max_nj_, max_len_, stream_, d_rtiles_.p, n_rtiles_};
  }

  template <int MODE>
  bs_status launch_tile(bsd::StateView<R> src, bsd::StateView<R> u0, bsd::StateView<R> out,
                        double a, double b, bool first, double* norm, double* res_out,
                        bool all_cases, const float4* dq_in = nullptr, bsd::StateView<R> upd_out = {}) {
    return launch_tile_on<MODE>(whole(), src, u0, out, a, b, first, norm, res_out, all_cases, dq_in,
                                upd_out);
  }

  template <int MODE>
  bs_status launch_tile_on(const LaneView& lane, bsd::StateView<R> src, bsd::StateView<R> u0,
                           bsd::StateView<R> out, double a, double b, bool first, double* norm,
                           double* res_out, bool all_cases, const float4* dq_in = nullptr,
                           bsd::StateView<R> upd_out = {}) {
    bsd::TileArgs<R> A{};
    A.cases = d_cases_.p;
    A.tiles = lane.tiles;
    A.active = all_cases ? nullptr : d_active_.p;
    A.src = src;
    A.u0 = u0;
    A.out = out;
    A.m = metrics();
    A.dt = dt_.p;
    A.dt_global = dtmin_.p;
    A.norm = norm;
    A.status = status_.p;
    A.a = a;
    A.b = b;
    A.first_stage = first ? 1 : 0;
    A.rec_f = rec_f_.p;
    A.rec_b = rec_b_.p;
    A.cfl = cfl_.p;
    A.omega = omega_.p;
    A.res_out = res_out;
    A.dq_in = dq_in;
    A.upd_out = upd_out;
    // The residual pass of an LU-SGS step follows the previous step's sweep by
    // programmatic dependent launch (the kernel waits for it first thing).
    const bool pdl = MODE == bsd::MODE_PREPARE && pdl_;
    auto go = [&](auto kernel, int n, int threads) {
      return bsd::launch_maybe_pdl(kernel, dim3(n), dim3(threads), 0, lane.stream, pdl, A);
    };
    cudaError_t e = cudaSuccess;
    bool tuned = false;
    if constexpr (sizeof(R) == sizeof(double) && MODE != bsd::MODE_RESIDUAL) {
      if (rshape_ >= 0) {
        tuned = true;
        A.tiles = lane.rtiles;
        const int n = lane.n_rtiles;
        switch (rshape_) {
          case 0: e = go(bsd::tile_kernel<R, MODE, 1>, n, bsd::TILE_THREADS); break;
          case 1: e = go(bsd::tile_kernel<R, MODE, 4>, n, bsd::TILE_THREADS); break;
          case 2: e = go(bsd::tile_kernel<R, MODE, 1, 16, 15, 512>, n, 512); break;
          case 3: e = go(bsd::tile_kernel<R, MODE, 1, 8, 15, 256>, n, 256); break;
          case 4: e = go(bsd::tile_kernel<R, MODE, 1, 16, 7, 256>, n, 256); break;
          case 5: e = go(bsd::tile_kernel<R, MODE, 1, 24, 15, 384>, n, 384); break;
          case 6: e = go(bsd::tile_kernel<R, MODE, 1, 8, 15, 128>, n, 128); break;
          default: e = go(bsd::tile_kernel<R, MODE, 2>, n, bsd::TILE_THREADS); break;
        }
      }
    }
    if (!tuned) {
      // Untuned: the default tile, four resident CTAs asked for on launches
      // of at least four waves.
      if (lane.n_tiles >= 4 * sm_count_)
        e = go(bsd::tile_kernel<R, MODE, 4>, lane.n_tiles, bsd::TILE_THREADS);
      else
        e = go(bsd::tile_kernel<R, MODE>, lane.n_tiles, bsd::TILE_THREADS);
    }
    launches_++;
    BS_CUDA(e);
    BS_CUDA(cudaGetLastError());
    return BS_OK;
  }

  // One explicit step of every active case; `norm` adds the density
  // residual of the step's starting state to the per-case slots.
  bs_status record_explicit_step(bool norm) { return record_explicit_step_on(whole(), norm); }

  bs_status record_explicit_step_on(const LaneView& lane, bool norm) {
    double a[3], b[3];
    int n = 3;
    const int integrator = cases_[0].cfg.integrator;
    if (integrator == BS_FORWARD_EULER) {
      n = 1; a[0] = 0; b[0] = 1;
    } else if (integrator == BS_SSPRK2) {
      n = 2; a[0] = 0; b[0] = 1; a[1] = 0.5; b[1] = 0.5;
    } else {
      a[0] = 0; b[0] = 1; a[1] = 3.0 / 4.0; b[1] = 1.0 / 4.0; a[2] = 1.0 / 3.0; b[2] = 2.0 / 3.0;
    }
    if (any_global_dt_) {
      BS_CUDA(cudaMemsetAsync(dtmin_.p, 0x7f, n_ * sizeof(unsigned), lane.stream));
      bsd::dt_kernel<R><<<lane.n_tiles, bsd::TILE_THREADS, 0, lane.stream>>>(
          d_cases_.p, lane.tiles, d_active_.p, q_view(), metrics(), dt_.p, dtmin_.p);
      launches_++;
      BS_CUDA(cudaGetLastError());
    }
    const bsd::StateView<R> q = q_view(), s1 = s1_view(), s2 = s2_view();
    if (n == 1) {
      BS_TRY(launch_tile_on<bsd::MODE_STAGE>(lane, q, q, s1, a[0], b[0], true, norm ? norm_.p : nullptr,
                                             nullptr, false));
      for (int v = 0; v < 4; v++)
        BS_CUDA(cudaMemcpyAsync(q_[v].p, s1_[v].p, total_cells_ * sizeof(R), cudaMemcpyDeviceToDevice,
                                lane.stream));
      return BS_OK;
    }
    for (int s = 0; s < n; s++) {
      const bsd::StateView<R> src = s == 0 ? q : (s == 1 ? s1 : s2);
      const bsd::StateView<R> out = s == n - 1 ? q : (s == 0 ? s1 : s2);
      BS_TRY(launch_tile_on<bsd::MODE_STAGE>(lane, src, q, out, a[s], b[s], s == 0,
                                             (norm && s == 0) ? norm_.p : nullptr, nullptr, false));
    }
    return BS_OK;
  }

  // Step s (from 0) of a run of `count` LU-SGS steps on one lane. The update
  // of each step is applied by the next step's residual pass as it reads the
  // state (the first step has none to apply), which stores the updated state
  // in the other buffer: step s >= 1 reads q when s is odd and qb when even,
  // and writes the other. After the last step a closing update brings the
  // state back into q, so every run begins and ends with the state in q.
  bs_status record_implicit_step_on(const LaneView& lane, bool norm, int s, int count) {
    const bsd::StateView<R> q = q_view(), qb = qb_view();
    if (!fuse_update_) {
      // Residual pass, sweeps, then the update in place (three launches).
      BS_TRY(launch_tile_on<bsd::MODE_PREPARE>(lane, q, q, q, 0, 1, false, norm ? norm_.p : nullptr, nullptr,
                                               false));
      BS_TRY(launch_sweep_on(lane));
      return launch_update_on(lane, q, q);
    }
    const bsd::StateView<R> src = (s == 0 || s % 2 == 1) ? q : qb;
    const bsd::StateView<R> dst = s % 2 == 1 ? qb : q;
    BS_TRY(launch_tile_on<bsd::MODE_PREPARE>(lane, src, src, src, 0, 1, false, norm ? norm_.p : nullptr,
                                             nullptr, false, s == 0 ? nullptr : dq_.p, dst));
    BS_TRY(launch_sweep_on(lane));
    if (s == count - 1) {
      const bsd::StateView<R> last = (s == 0 || s % 2 == 0) ? q : qb;
      return launch_update_on(lane, last, q);
    }
    return BS_OK;
  }

  // One LU-SGS step with Anderson acceleration: the residual pass and the
  // sweeps as for a plain step, then the acceleration's kernels in place of
  // the update.
  bs_status record_anderson_step_on(const LaneView& lane, bool norm) {
    const bsd::StateView<R> q = q_view();
    BS_TRY(launch_tile_on<bsd::MODE_PREPARE>(lane, q, q, q, 0, 1, false, norm ? norm_.p : nullptr,
                                             nullptr, false));
    BS_TRY(launch_sweep_on(lane));
    bsd::AndersonArgs<R> A{};
    A.cases = d_cases_.p;
    A.tiles = lane.tiles;
    A.case_list = lane.case_list;
    A.n_cases = lane.n_cases;
    A.active = d_active_.p;
    A.q = q;
    A.last_x = {alastx_[0].p, alastx_[1].p, alastx_[2].p, alastx_[3].p};
    A.dq = dq_.p;
    A.last_f = alastf_.p;
    A.dx = adx_.p;
    A.df = adf_.p;
    A.total = total_cells_;
    A.depth = anderson_depth_;
    A.ac = ac_.p;
    A.part = aacc_.p;
    A.gram = agram_.p;
    A.gamma = agamma_.p;
    A.status = status_.p;
    bsd::anderson_push_kernel<R><<<lane.n_tiles, bsd::TILE_THREADS, 0, lane.stream>>>(A);
    bsd::anderson_solve_kernel<R><<<lane.n_cases, 32, 0, lane.stream>>>(A);
    bsd::anderson_apply_kernel<R><<<lane.n_tiles, bsd::TILE_THREADS, 0, lane.stream>>>(A);
    bsd::anderson_fallback_kernel<R><<<lane.n_tiles, bsd::TILE_THREADS, 0, lane.stream>>>(A);
    launches_ += 4;
    BS_CUDA(cudaGetLastError());
    return BS_OK;
  }

  bs_status launch_sweep() { return launch_sweep_on(whole()); }


  bs_status launch_sweep_on(const LaneView& lane) {
    bsd::SweepArgs S{};
    S.cases = d_cases_.p;
    S.case_list = lane.case_list;
    S.active = d_active_.p;
    S.rec_f = rec_f_.p;
    S.rec_b = rec_b_.p;
    S.dq = dq_.p;
    S.cfl = cfl_.p;
    S.cfl_max = cflmax_.p;
    S.growth = growth_.p;
    S.omega = omega_.p;
    S.status = status_.p;
    BS_CUDA(bsd::launch_sweep(S, lane.n_cases, lane.max_nj, lane.max_len, n_, lane.stream, sweep_wait_limit_,
                              sweep_max_chunk_, pdl_));
    launches_++;
    return BS_OK;
  }

  bs_status launch_update_on(const LaneView& lane, bsd::StateView<R> src, bsd::StateView<R> dst) {
    bsd::lusgs_update_kernel<R><<<lane.n_tiles, bsd::TILE_THREADS, 0, lane.stream>>>(
        d_cases_.p, lane.tiles, d_active_.p, src, dst, dq_.p, status_.p);
    launches_++;
    BS_CUDA(cudaGetLastError());
    return BS_OK;
  }

  bool lanes_apply(int method) const {
    if (lanes_.size() < 2) return false;
    // Forward Euler copies whole arenas and global stepping reduces over the
    // batch: those run as one lane.
    return method == kMethodImplicit || method == kMethodAnderson ||
           (!any_global_dt_ && cases_[0].cfg.integrator != BS_FORWARD_EULER);
  }

  bs_status record_steps(int method, int count, bool norm_last) {
    if (!lanes_apply(method)) {
      for (int s = 0; s < count; s++) {
        const bool norm = norm_last && s == count - 1;
        if (method == kMethodExplicit)
          BS_TRY(record_explicit_step(norm));
        else if (method == kMethodAnderson)
          BS_TRY(record_anderson_step_on(whole(), norm));
        else
          BS_TRY(record_implicit_step_on(whole(), norm, s, count));
      }
      return BS_OK;
    }
    // Fork one chain of `count` steps per lane off the batch stream, join them back.
    BS_CUDA(cudaEventRecord(ev_fork_, stream_));
    for (auto& l : lanes_) BS_CUDA(cudaStreamWaitEvent(l->stream, ev_fork_, 0));
    for (auto& l : lanes_) {
      const LaneView lane{l->tiles.p,  l->n_tiles, l->case_list.p, l->n_cases,
                          l->max_nj,   l->max_len, l->stream,      l->rtiles.p, l->n_rtiles};
      for (int s = 0; s < count; s++) {
        const bool norm = norm_last && s == count - 1;
        if (method == kMethodExplicit)
          BS_TRY(record_explicit_step_on(lane, norm));
        else if (method == kMethodAnderson)
          BS_TRY(record_anderson_step_on(lane, norm));
        else
          BS_TRY(record_implicit_step_on(lane, norm, s, count));
      }
    }
    for (size_t k = 0; k < lanes_.size(); k++) {
      BS_CUDA(cudaEventRecord(ev_join_[k], lanes_[k]->stream));
      BS_CUDA(cudaStreamWaitEvent(stream_, ev_join_[k], 0));
    }
    return BS_OK;
  }

  // Runs `count` steps by replaying captured graphs of up to kChunk steps.
  bs_status run_steps(int method, int count, bool norm_last) {
    constexpr int kChunk = 16;
    int left = count;
    while (left > 0) {
      const int n = std::min(left, kChunk);
      const bool norm = norm_last && n == left;
      cudaGraphExec_t exec = nullptr;
      BS_TRY(graph_for(method, n, norm, &exec));
      BS_CUDA(cudaGraphLaunch(exec, stream_));
      left -= n;
    }
    return BS_OK;
  }

  bs_status graph_for(int method, int count, bool norm_last, cudaGraphExec_t* out) {
    const GraphKey key{method, count, norm_last ? 1 : 0};
    auto it = graphs_.find(key);
    if (it != graphs_.end()) {
      *out = it->second;
      launches_ += graph_launches_[key];
      return BS_OK;
    }
    cudaGraph_t graph = nullptr;
    const int64_t before = launches_;
    BS_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    const bs_status st = record_steps(method, count, norm_last);
    const cudaError_t end = cudaStreamEndCapture(stream_, &graph);
    if (st != BS_OK) {
      if (graph != nullptr) cudaGraphDestroy(graph);
      return st;
    }
    BS_CUDA(end);
    cudaGraphExec_t exec = nullptr;
    const cudaError_t inst = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    BS_CUDA(inst);
    graphs_[key] = exec;
    graph_launches_[key] = launches_ - before;
    *out = exec;
    return BS_OK;
  }

  bs_status launch_boundary(int c, int side, double p_inf, bool drag) {
    bsd::BoundaryArgs<R> A{};
    A.cases = d_cases_.p;
    A.case_index = c;
    A.q = q_view();
    A.m = metrics();
    A.side = side;
    const HostCase& h = cases_[c];
    int64_t off = boundary_off_[c];
    for (int s = 0; s < side; s++) off += s < 2 ? h.cfg.nj : h.cfg.ni;
    A.geom = bgeom_.p + 3 * off;
    A.gamma_eval = h.cfg.gamma;
    A.flux_out = bflux_.p;
    A.p_inf = p_inf;
    A.force_out = drag ? force_.p : nullptr;
    bsd::boundary_flux_kernel<R><<<1, 256, 0, stream_>>>(A);
    launches_++;
    BS_CUDA(cudaGetLastError());
    return BS_OK;
  }

  bs_status copy_state(int c, std::vector<R> comp[4]) {
    const size_t n = size_t(cases_[c].cfg.ni) * cases_[c].cfg.nj;
    const int64_t off = cell_offset(c);
    for (int v = 0; v < 4; v++) {
      comp[v].resize(n);
      BS_CUDA(cudaMemcpyAsync(comp[v].data(), q_[v].p + off, n * sizeof(R), cudaMemcpyDeviceToHost,
                              stream_));
    }
    BS_CUDA(cudaStreamSynchronize(stream_));
    return BS_OK;
  }

  std::vector<HostCase> cases_;
  int n_ = 0;
  int64_t total_cells_ = 0;
  int64_t total_slots_ = 0;
  int n_tiles_ = 0;
  int max_nj_ = 0, max_len_ = 0, max_along_ = 0;
  // LU-SGS steps apply the update inside the next residual pass (true) or
  // by a separate kernel after each sweep; autotune chooses.
  bool fuse_update_ = true;
  // Programmatic dependent launch between the residual pass and the sweep
  // (off with BOWSHOCK_NO_PDL set, to compare).
  bool pdl_ = std::getenv("BOWSHOCK_NO_PDL") == nullptr;
  // Longest sweep chunk (diagonals per bulk copy; BOWSHOCK_SWEEP_CHUNK
  // overrides the default 8, to compare). With lanes overlapping, chunks of
  // 8 in four buffers (three chunks of copies ahead) beat chunks of 16 in two
  // (one ahead), although 16 is faster alone.
  int sweep_max_chunk_ = std::getenv("BOWSHOCK_SWEEP_CHUNK") ? std::atoi(std::getenv("BOWSHOCK_SWEEP_CHUNK")) : 8;
  bool any_global_dt_ = false;
  std::vector<int64_t> boundary_off_, cell_off_;
  std::vector<int64_t> steps_;
  std::vector<int> active_h_;
  DevBuf<bsd::CaseDev> d_cases_;
  DevBuf<int2> d_tiles_;
  DevBuf<int> d_case_list_, d_active_;
  DevBuf<R> q_[4], qb_[4], s1_[4], s2_[4];
  DevBuf<float> dt_, cfl_, cflmax_, growth_, omega_;
  DevBuf<float4> iface_, jface_, rec_f_, rec_b_, dq_;
  DevBuf<float2> cellm_;
  // The two-float metrics' low parts, allocated when first switched on.
  DevBuf<float4> iface_lo_, jface_lo_;
  DevBuf<float2> cellm_lo_;
  bool metrics_lo_ = false;
  int64_t total_iface_ = 0, total_jface_ = 0;
  DevBuf<double> norm_, bgeom_, bflux_, force_, res_out_;
  DevBuf<unsigned> status_, dtmin_;
  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  struct Lane {
    DevBuf<int2> tiles, rtiles;
    DevBuf<int> case_list;
    std::vector<int> members;
    int n_tiles = 0, n_rtiles = 0, n_cases = 0, max_nj = 0, max_len = 0;
    cudaStream_t stream = nullptr;
  };
  std::vector<std::unique_ptr<Lane>> lanes_;
  std::vector<bsd::CaseDev> hc_;  // the cases as uploaded (to rebuild lanes)
  int sm_count_ = 148;
  DevBuf<double> nodes_x_, nodes_y_;  // grid nodes (display fields only)
  std::vector<int64_t> node_off_;
  cudaEvent_t ev_fork_ = nullptr;
  std::vector<cudaEvent_t> ev_join_;
  std::map<GraphKey, cudaGraphExec_t> graphs_;
  std::map<GraphKey, int64_t> graph_launches_;
  int64_t launches_ = 0;
  int sweep_wait_limit_ = -1;
  // The residual pass's tile shape (bsd::tile_shape), or -1 for the default
  // choice; the whole batch's tiles of that shape.
  int rshape_ = -1;
  DevBuf<int2> d_rtiles_;
  int n_rtiles_ = 0;
  double last_solve_ms_ = 0;
  int64_t last_solve_launches_ = 0;
  // Anderson acceleration: settings and its per-case history.
  int anderson_depth_ = 0, anderson_plain_ = 30, anderson_alloc_depth_ = 0;
  // iterate_accelerated's history: reset before its next step when stale,
  // and the steps it has taken since.
  bool anderson_stale_ = true;
  int64_t accelerated_steps_ = 0;
  DevBuf<float4> adx_, adf_, alastf_;
  DevBuf<R> alastx_[4];
  DevBuf<bsd::AndersonCase> ac_;
  DevBuf<double> aacc_, agram_, agamma_;
};

}  // namespace

void tile_dims(int shape, int32_t* ti, int32_t* tj, int32_t* threads) {
  const bsd::TileShape sh = bsd::tile_shape(shape < 0 ? 0 : shape);
  *ti = sh.ti;
  *tj = sh.tj;
  *threads = sh.threads;
}

bs_status make_solver(std::vector<HostCase>&& cases, int precision,
                      std::unique_ptr<SolverBase>& out) {
  if (cases.empty()) return fail(BS_INVALID_ARGUMENT, "a batch needs at least one case");
  const int integrator = cases[0].cfg.integrator;
  for (const HostCase& h : cases)
    if (h.cfg.integrator != integrator)
      return fail(BS_INVALID_ARGUMENT, "the cases of a batch share one time integrator");
  if (precision == 64) {
    auto s = std::make_unique<Solver<double>>(std::move(cases));
    BS_TRY(s->init());
    out = std::move(s);
  } else if (precision == 32) {
    auto s = std::make_unique<Solver<float>>(std::move(cases));
    BS_TRY(s->init());
    out = std::move(s);
  } else {
    return fail(BS_INVALID_ARGUMENT, "precision must be 32 or 64");
  }
  return BS_OK;
}

}  // namespace bs
