// An LU-SGS step that allocates nothing.
//
// Some callers cannot let a library allocate device memory: applications that
// hand out every byte of the GPU from their own pool or arena (a library's
// cudaMalloc would bypass their budget, and cudaMalloc / cudaFree
// synchronise the device and stall the caller's other streams), and
// long-running solver loops that must not allocate once they have started.
// bs_lusgs_step_static serves them: the caller owns the state and the grid
// metrics on the device, and the step's scratch (residual, diagonal, state
// copy and correction of every cell, and the few per-case words of the
// kernels) lives in one file-scope static device array of fixed size that the
// library reserves on every GPU that loads it, for as long as the process runs.
//
// Limits and sharing: at most kStaticMaxCells cells (ni nj; the sweep records
// take one slot per cell) and 512 cells across (nj).
// Every call uses the same array, which keeps the last call's contents; the
// per-call words that must start at zero are cleared by each call. Calls
// whose work overlaps on the GPU (from several threads, or on several streams
// of one device) race on the array; the caller must order them.
//
// Each call waits for its stream (it reads back the residual and the status),
// so it must not be called while that stream is being captured into a graph.
// The device address of the array is looked up once per device, by the first
// call made on it with that device current; after cudaDeviceReset (or any
// teardown of the device's primary context) that address is stale and the
// entry point must not be used again in the process.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>

#include "bowshock.h"
#include "common.hpp"
#include "device/sweep.cuh"
#include "device/tile.cuh"
#include "solver.hpp"

namespace {

constexpr int64_t kStaticMaxCells = 65536;
// Slots of the LU-SGS sweep records (bsd::sweep_slots: one per cell).
constexpr int64_t kStaticMaxSlots = kStaticMaxCells;
constexpr int kStaticMaxTiles = 4096;
constexpr int kMaxDevices = 64;

// Byte layout of the static scratch array (each region 256-byte aligned).
constexpr size_t kAlign = 256;
constexpr size_t align_up(size_t n) { return (n + kAlign - 1) / kAlign * kAlign; }
constexpr size_t kOffCase = 0;
constexpr size_t kOffTiles = kOffCase + align_up(sizeof(bsd::CaseDev));
constexpr size_t kOffWords = kOffTiles + align_up(sizeof(int2) * kStaticMaxTiles);
constexpr size_t kOffRecF = kOffWords + kAlign;
constexpr size_t kOffRecB = kOffRecF + align_up(5 * sizeof(float4) * kStaticMaxSlots);
constexpr size_t kOffDq = kOffRecB + align_up(5 * sizeof(float4) * kStaticMaxSlots);
constexpr size_t kStaticBytes = kOffDq + align_up(sizeof(float4) * kStaticMaxCells);

// The scratch: about 11.6 MB on every device that loads the library.
static __device__ __align__(256) unsigned char g_step_scratch[kStaticBytes];

// The per-case words inside the kOffWords region.
struct Words {
  double norm;
  unsigned status;
  int case_list;
  float cfl, cfl_max, growth, omega;
};

// Device address of g_step_scratch per device, found once per device (with
// that device current) by the first call made on it.
void* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

bs_status scratch_address(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices)
    return bs::fail(BS_INVALID_ARGUMENT, "device index beyond the static scratch table");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (g_scratch_addr[device] == nullptr) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_step_scratch);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return bs::fail(BS_EXECUTION,
                      std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
    }
    g_scratch_addr[device] = p;
  }
  *out = static_cast<unsigned char*>(g_scratch_addr[device]);
  return BS_OK;
}

// Writes the tile list and the per-case words of one step into the scratch.
__global__ void init_static_step(int2* tiles, int n_tiles, Words* w, float cfl, float omega) {
  for (int t = threadIdx.x; t < n_tiles; t += blockDim.x) tiles[t] = make_int2(0, t);
  if (threadIdx.x == 0) {
    w->norm = 0.0;
    w->status = 0u;
    w->case_list = 0;
    w->cfl = cfl;
    w->cfl_max = cfl;
    w->growth = 1.f;
    w->omega = omega;
  }
}

}  // namespace

extern "C" {

bs_status bs_lusgs_step_static(const bs_config* config, const float* iface, const float* jface,
                               const float* cells, double* rho, double* mu, double* mv, double* e,
                               double cfl, double omega, void* stream, double* residual,
                               int32_t* non_physical) {
  if (config == nullptr || iface == nullptr || jface == nullptr || cells == nullptr ||
      rho == nullptr || mu == nullptr || mv == nullptr || e == nullptr || residual == nullptr ||
      non_physical == nullptr)
    return bs::fail(BS_INVALID_ARGUMENT, "null argument");
  const std::string v = bs::validate_config(*config);
  if (!v.empty()) return bs::fail(BS_INVALID_ARGUMENT, v);
  if (!(cfl > 0 && omega >= 1)) return bs::fail(BS_INVALID_ARGUMENT, "LU-SGS needs cfl > 0 and omega >= 1");
  const int ni = config->ni, nj = config->nj;
  const int64_t n_cells = int64_t(ni) * nj;
  if (n_cells > kStaticMaxCells)
    return bs::fail(BS_INVALID_ARGUMENT,
                    "the grid has " + std::to_string(n_cells) +
                        " cells; the allocation-free step takes at most " +
                        std::to_string(kStaticMaxCells));
  static_assert(kStaticMaxSlots >= kStaticMaxCells, "one sweep-record slot per cell");
  const int n_tiles = ((ni + bsd::TI - 1) / bsd::TI) * ((nj + bsd::TJ - 1) / bsd::TJ);
  if (n_tiles > kStaticMaxTiles)
    return bs::fail(BS_INVALID_ARGUMENT, "the grid needs more tiles than the static scratch holds");
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) {
    cudaGetLastError();
    return bs::fail(BS_EXECUTION, "no CUDA device");
  }
  unsigned char* base = nullptr;
  const bs_status s = scratch_address(device, &base);
  if (s != BS_OK) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  bsd::CaseDev cd{};
  cd.ni = ni;
  cd.nj = nj;
  cd.cell = 0;
  cd.iface = 0;
  cd.jface = 0;
  cd.slot = 0;
  for (int k = 0; k < 4; k++) cd.bc[k] = config->boundaries[k].kind;
  cd.flux = config->flux;
  cd.limiter = config->limiter;
  cd.recon = config->reconstruction;
  cd.axisym = config->geometry == BS_AXISYMMETRIC;
  cd.integrator = config->integrator;
  cd.local_dt = config->time_stepping == BS_TIME_LOCAL;
  cd.gamma = config->gamma;
  cd.cfl = config->cfl;
  for (int k = 0; k < 4; k++) {
    const bs_primitive& w = config->boundaries[k].state;
    cd.inflow_prim[k][0] = w.rho;
    cd.inflow_prim[k][1] = w.u;
    cd.inflow_prim[k][2] = w.v;
    cd.inflow_prim[k][3] = w.p;
    cd.inflow_cons[k][0] = w.rho;
    cd.inflow_cons[k][1] = w.rho * w.u;
    cd.inflow_cons[k][2] = w.rho * w.v;
    cd.inflow_cons[k][3] = w.p / (cd.gamma - 1) + 0.5 * w.rho * (w.u * w.u + w.v * w.v);
  }
  auto* d_case = reinterpret_cast<bsd::CaseDev*>(base + kOffCase);
  auto* d_tiles = reinterpret_cast<int2*>(base + kOffTiles);
  auto* d_words = reinterpret_cast<Words*>(base + kOffWords);
  auto* d_rec_f = reinterpret_cast<float4*>(base + kOffRecF);
  auto* d_rec_b = reinterpret_cast<float4*>(base + kOffRecB);
  auto* d_dq = reinterpret_cast<float4*>(base + kOffDq);

  cudaError_t err = cudaMemcpyAsync(d_case, &cd, sizeof(cd), cudaMemcpyHostToDevice, st);
  if (err == cudaSuccess) {
    init_static_step<<<1, 256, 0, st>>>(d_tiles, n_tiles, d_words, float(cfl), float(omega));
    err = cudaGetLastError();
  }
  const bsd::MetricsView m{reinterpret_cast<const float4*>(iface),
                           reinterpret_cast<const float4*>(jface),
                           reinterpret_cast<const float2*>(cells)};
  const bsd::StateView<double> q{rho, mu, mv, e};
  if (err == cudaSuccess) {
    bsd::TileArgs<double> A{};
    A.cases = d_case;
    A.tiles = d_tiles;
    A.src = q;
    A.u0 = q;
    A.out = q;
    A.m = m;
    A.norm = &d_words->norm;
    A.status = &d_words->status;
    A.a = 0;
    A.b = 1;
    A.rec_f = d_rec_f;
    A.rec_b = d_rec_b;
    A.cfl = &d_words->cfl;
    A.omega = &d_words->omega;
    bsd::tile_kernel<double, bsd::MODE_PREPARE><<<n_tiles, bsd::TILE_THREADS, 0, st>>>(A);
    err = cudaGetLastError();
  }
  if (err == cudaSuccess) {
    bsd::SweepArgs S{};
    S.cases = d_case;
    S.case_list = &d_words->case_list;
    S.rec_f = d_rec_f;
    S.rec_b = d_rec_b;
    S.dq = d_dq;
    S.cfl = &d_words->cfl;
    S.cfl_max = &d_words->cfl_max;
    S.growth = &d_words->growth;
    S.omega = &d_words->omega;
    S.status = &d_words->status;
    err = bsd::launch_sweep(S, 1, nj, std::min(ni, nj), 1, st);
  }
  if (err == cudaSuccess) {
    bsd::lusgs_update_kernel<double><<<n_tiles, bsd::TILE_THREADS, 0, st>>>(
        d_case, d_tiles, nullptr, q, q, d_dq, &d_words->status);
    err = cudaGetLastError();
  }
  double norm = 0;
  unsigned status = 0;
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(&norm, &d_words->norm, sizeof(norm), cudaMemcpyDeviceToHost, st);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(&status, &d_words->status, sizeof(status), cudaMemcpyDeviceToHost, st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(st);
  if (err != cudaSuccess) {
    cudaGetLastError();
    return bs::fail(BS_EXECUTION, std::string("allocation-free LU-SGS step: ") + cudaGetErrorString(err));
  }
  if (status & bsd::STATUS_TIMEOUT)
    return bs::fail(BS_EXECUTION,
                    "allocation-free LU-SGS step: the sweep gave up waiting for its records; "
                    "the state was left as it was before the step");
  *residual = std::sqrt(norm / double(n_cells));
  *non_physical = (status & bsd::STATUS_NON_PHYSICAL) ? 1 : 0;
  return BS_OK;
}

}  // extern "C"
