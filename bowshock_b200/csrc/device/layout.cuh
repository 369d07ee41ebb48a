// Device data layout of a batch of cases (one engine is a batch of one).
//
// Every case's arrays live in shared arenas at per-case offsets:
//   state      SoA, one array per conserved component (rho, rho u, rho v, E),
//              ni nj cells of the case at `cell`, cell (i, j) at i + j ni;
//   i-faces    float4 (nx, ny, area, 0), (ni + 1) nj at `iface`;
//   j-faces    float4 (nx, ny, area, 0), ni (nj + 1) at `jface`;
//   cells      float2 (volume, planar area) at `cell`;
//   LU-SGS     per-cell sweep records in anti-diagonal order (sweep_slot),
//              ni nj slots at `slot`; the final correction dQ is row-major
//              like the state.
// Metrics are computed in FP64 on the host and stored as FP32; with the
// two-float metrics on, also each value's FP32 low part (the FP64 value less
// the FP32 one), which the residual adds back (about 48 bits). The state is
// stored in the solve's arithmetic type R: double for the steady solves
// (the residual that decides convergence is evaluated in FP64), float for
// the reference GPU engine's all-FP32 arithmetic.
#pragma once

#include <cstdint>

#include "scheme.cuh"

namespace bsd {

// Tile of the fused cell kernels: TI cells along i by TJ along j, one
// thread per cell; a CTA has TILE_THREADS threads, thread t on cell
// (t % TI, t / TI), and threads past the tile's TJ rows only help with the
// halo and the faces. 16 x 15 has 511 faces, two per thread (32 x 8 has 552,
// which leaves a third round to 40 threads), and 124 halo cells for 240
// (32 x 8: 160 for 256): its residual pass is 7 % faster.
constexpr int TI = 16;
constexpr int TJ = 15;
constexpr int TILE_THREADS = 256;
static_assert(TI * TJ <= TILE_THREADS, "a tile has at most one cell per thread");

// Tile shapes the residual pass and the explicit stages can run with, the
// autotuner's choices: TI x TJ cells on `threads` threads, `min_blocks`
// resident CTAs asked of the compiler. Shape 0 is the default above (about
// two faces per thread) with one resident CTA asked for, shape 1 the same
// with four. Shapes 2 to 4 give each thread about one face, which halves the
// dependent FP64 work a thread does and so a CTA's latency (a case's pass on
// idle SMs is latency-bound); shape 5 reads the least halo (43 % of its
// cells against 52 %) and shape 6 puts twice as many CTAs on a case. Shape 7
// is the default tile with two resident CTAs asked for: at most 128 registers
// a thread, between shape 0's 140 (one CTA an SM) and shape 1's 64 (spilling).
struct TileShape {
  int ti, tj, threads, min_blocks;
};
constexpr int kTileShapes = 8;
__host__ __device__ constexpr TileShape tile_shape(int k) {
  return k == 0   ? TileShape{TI, TJ, TILE_THREADS, 1}
         : k == 1 ? TileShape{TI, TJ, TILE_THREADS, 4}
         : k == 2 ? TileShape{16, 15, 512, 1}
         : k == 3 ? TileShape{8, 15, 256, 1}
         : k == 4 ? TileShape{16, 7, 256, 1}
         : k == 5 ? TileShape{24, 15, 384, 1}
         : k == 6 ? TileShape{8, 15, 128, 1}
                  : TileShape{TI, TJ, TILE_THREADS, 2};
}

// Per-case status bits.
constexpr unsigned STATUS_NON_PHYSICAL = 1u;
// A kernel gave up waiting for an asynchronous copy (bounded wait).
constexpr unsigned STATUS_TIMEOUT = 2u;

// LU-SGS sweep records: one per cell and direction, stored by anti-diagonal
// d = i + j (the order the sweeps visit them) and along a diagonal by row j,
// with no slot for cells off the grid, so that any run of diagonals is one
// contiguous range that a single bulk copy brings into shared memory and a
// case has exactly ni nj slots. Diagonal d holds rows max(0, d - ni + 1) ..
// min(d, nj - 1) and starts after diag_cells(ni, nj, d) slots: the diagonals
// before it have min(k + 1, ni, nj, ni + nj - 1 - k) cells each, which sums
// to T(d) - T(d - min) - T(d - max) with T(x) = x (x + 1) / 2 for x > 0.
// 32-bit: the sweep launch requires ni + nj <= 65536 (so x (x + 1) < 2^32).
__host__ __device__ __forceinline__ unsigned diag_cells(int ni, int nj, int d) {
  const int a = ni < nj ? ni : nj, b = ni < nj ? nj : ni;
  const unsigned x = unsigned(d), xa = unsigned(d > a ? d - a : 0), xb = unsigned(d > b ? d - b : 0);
  return ((x * (x + 1)) >> 1) - ((xa * (xa + 1)) >> 1) - ((xb * (xb + 1)) >> 1);
}
// Slot of cell (i, j) within its case's records.
__host__ __device__ __forceinline__ int64_t sweep_slot(int ni, int nj, int i, int j) {
  const int d = i + j;
  return int64_t(diag_cells(ni, nj, d)) + (j - (d - ni + 1 > 0 ? d - ni + 1 : 0));
}
// Slots of a case's records.
__host__ __device__ __forceinline__ int64_t sweep_slots(int ni, int nj) { return int64_t(ni) * nj; }
// float4 fields of a record (listed with the sweep kernel).
constexpr int REC_SIZE = 5;

// Programmatic dependent launch: a kernel launched with the programmatic
// stream-serialization attribute may start before the kernel ahead of it in
// its stream has finished; it must wait (griddep_wait) before it reads what
// that kernel writes or writes what it reads. Without the attribute both
// instructions do nothing.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
// Lets the dependent kernel be launched once every CTA of this one has run it.
__device__ __forceinline__ void griddep_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

struct CaseDev {
  int32_t ni, nj;
  int64_t cell;   // offset of the case's cell arrays
  int64_t iface;  // offset of its i-face arrays
  int64_t jface;  // offset of its j-face arrays
  int64_t slot;   // offset of its LU-SGS sweep records, sweep_slots(ni, nj) = ni nj slots
  int32_t bc[4];  // bs_bc_kind per side
  int32_t flux, limiter, recon, axisym;
  int32_t integrator, local_dt;
  double gamma;   // rounded to FP32 for FP32 cases
  double cfl;     // explicit CFL number
  double inflow_prim[4][4];  // (rho, u, v, p) outside each inflow / far-field side
  double inflow_cons[4][4];  // the same as conserved variables
  // 'faceStates' sides: the conserved state outside each face (4 per face,
  // FP64), and the flux per unit area imposed on each face or null.
  const double* face_state[4] = {};
  const double* face_flux[4] = {};
  int64_t tile_base = 0;  // index of its first tile in the batch's tile order
};

template <class R>
struct StateView {
  R* rho;
  R* mu;
  R* mv;
  R* e;
  __device__ __forceinline__ Cons<R> load(int64_t k) const { return {rho[k], mu[k], mv[k], e[k]}; }
  __device__ __forceinline__ void store(int64_t k, const Cons<R>& q) const {
    rho[k] = q.rho;
    mu[k] = q.mu;
    mv[k] = q.mv;
    e[k] = q.e;
  }
};

struct MetricsView {
  const float4* iface;  // (nx, ny, area, 0)
  const float4* jface;
  const float2* cell;   // (volume, planar area)
  // Low parts of the same values, or null (FP32 metrics).
  const float4* iface_lo = nullptr;
  const float4* jface_lo = nullptr;
  const float2* cell_lo = nullptr;
};

// A face's unit normal and area in the arithmetic R: the FP32 values, plus
// their low parts where the two-float metrics are on.
template <class R>
struct FaceGeom {
  R nx, ny, area;
};

template <class R>
__device__ __forceinline__ FaceGeom<R> face_geom(const float4* hi, const float4* lo, int64_t idx) {
  const float4 h = hi[idx];
  if (lo == nullptr) return {R(h.x), R(h.y), R(h.z)};
  const float4 l = lo[idx];
  return {R(h.x) + R(l.x), R(h.y) + R(l.y), R(h.z) + R(l.z)};
}

// A cell's volume and planar area (the axisymmetric source's weight) in R.
template <class R>
__device__ __forceinline__ void cell_geom(const MetricsView& m, int64_t k, R* volume, R* planar) {
  const float2 h = m.cell[k];
  if (m.cell_lo == nullptr) {
    *volume = R(h.x);
    *planar = R(h.y);
    return;
  }
  const float2 l = m.cell_lo[k];
  *volume = R(h.x) + R(l.x);
  *planar = R(h.y) + R(l.y);
}

// The conserved state of cell (i, j) of a case, for i in [-2, ni + 1] with j in
// range or j in [-2, nj + 1] with i in range: interior cells from `at(k)`,
// ghost cells from the side's boundary condition as fillGhosts builds them
// (src/engine-cpu/euler2d.ts:1361-1423): ghost layer g mirrors interior
// layer g (outflow, wall with the momentum reflected about the boundary
// face), wraps (periodic), or holds the inflow / far-field state.
// `inflow_from_prim` rebuilds the inflow ghost from its primitives with this
// gamma instead of using the stored conserved copy.
template <class R, class At>
__device__ __forceinline__ Cons<R> cell_or_ghost(const CaseDev& cd, const MetricsView& m, int i,
                                                 int j, R gamma, bool inflow_from_prim, At&& at) {
  const int ni = cd.ni, nj = cd.nj;
  if (i >= 0 && i < ni && j >= 0 && j < nj) return at(cd.cell + i + int64_t(j) * ni);
  int side, mi, mj, wi, wj, ii, ij;
  // The boundary face's metrics: array, low parts and index.
  const float4* fa;
  const float4* fl;
  int64_t fk;
  if (i < 0) {
    side = BS_IMIN;
    mi = -1 - i; mj = j; wi = i + ni; wj = j; ii = 0; ij = j;
    fa = m.iface; fl = m.iface_lo; fk = cd.iface + int64_t(j) * (ni + 1);
  } else if (i >= ni) {
    side = BS_IMAX;
    mi = 2 * ni - 1 - i; mj = j; wi = i - ni; wj = j; ii = ni - 1; ij = j;
    fa = m.iface; fl = m.iface_lo; fk = cd.iface + ni + int64_t(j) * (ni + 1);
  } else if (j < 0) {
    side = BS_JMIN;
    mi = i; mj = -1 - j; wi = i; wj = j + nj; ii = i; ij = 0;
    fa = m.jface; fl = m.jface_lo; fk = cd.jface + i;
  } else {
    side = BS_JMAX;
    mi = i; mj = 2 * nj - 1 - j; wi = i; wj = j - nj; ii = i; ij = nj - 1;
    fa = m.jface; fl = m.jface_lo; fk = cd.jface + i + int64_t(nj) * ni;
  }
  const int kind = cd.bc[side];
  if (kind == BS_BC_FACE_STATES) {
    // Both ghost layers hold the state given outside the face.
    const double* s = cd.face_state[side] + 4 * (side < 2 ? ij : ii);
    return {R(s[0]), R(s[1]), R(s[2]), R(s[3])};
  }
  if (kind == BS_BC_INFLOW) {
    if (inflow_from_prim) {
      const double* s = cd.inflow_prim[side];
      return to_cons(Prim<R>{R(s[0]), R(s[1]), R(s[2]), R(s[3])}, gamma);
    }
    const double* s = cd.inflow_cons[side];
    return {R(s[0]), R(s[1]), R(s[2]), R(s[3])};
  }
  if (kind == BS_BC_FAR_FIELD) {
    // Both ghost layers take the face's state from the first interior cell.
    const Prim<R> inside = to_prim(at(cd.cell + ii + int64_t(ij) * ni), gamma);
    const double* s = cd.inflow_prim[side];
    const Prim<R> fr{R(s[0]), R(s[1]), R(s[2]), R(s[3])};
    const R sgn = (side == BS_IMIN || side == BS_JMIN) ? R(-1) : R(1);
    const FaceGeom<R> f = face_geom<R>(fa, fl, fk);
    return to_cons(far_field_state(inside, fr, sgn * f.nx, sgn * f.ny, gamma), gamma);
  }
  if (kind == BS_BC_PERIODIC) return at(cd.cell + wi + int64_t(wj) * ni);
  Cons<R> c = at(cd.cell + mi + int64_t(mj) * ni);
  if (kind == BS_BC_WALL) {
    const FaceGeom<R> f = face_geom<R>(fa, fl, fk);
    const R nx = f.nx, ny = f.ny;
    const R mn = c.mu * nx + c.mv * ny;
    c.mu = c.mu - R(2) * mn * nx;
    c.mv = c.mv - R(2) * mn * ny;
  }
  return c;
}

template <class R>
__device__ __forceinline__ Cons<R> load_cell(const CaseDev& cd, const StateView<R>& q,
                                             const MetricsView& m, int i, int j) {
  return cell_or_ghost<R>(cd, m, i, j, R(cd.gamma), false,
                          [&](int64_t k) { return q.load(k); });
}

// -1 / +1 when face index `at` on a line of `n` cells is a wall face on the
// minimum / maximum side, else 0.
__device__ __forceinline__ int wall_side(const CaseDev& cd, int at, int n, int min_side,
                                         int max_side) {
  if (at == 0 && cd.bc[min_side] == BS_BC_WALL) return -1;
  if (at == n && cd.bc[max_side] == BS_BC_WALL) return 1;
  return 0;
}

// Warp-level FP64 sum; lane 0 holds the result.
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace bsd
