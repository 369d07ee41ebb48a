// The fused cell kernel: one CTA per TI x TJ tile of a case. It stages the
// tile's primitives with a two-cell halo in shared memory (one conversion per
// cell, ghost cells built from the boundary conditions on the fly), evaluates
// every i- and j-face flux of the tile once (MUSCL reconstruction + HLLC in
// the face frame, src/engine-cpu/euler2d.ts:1237-1269), sums them into the
// residual with the axisymmetric source (:1287-1295), and then, by MODE:
//   STAGE    - one SSP-RK stage, out = a u0 + b (src + dt/V R) (:1160-1175),
//              with the local time step of the first stage fused (:1183-1205);
//   PREPARE  - LU-SGS pass A: each cell's two sweep records - the residual
//              (FP32 copy), the scalar diagonal (:926-971) and the
//              constants of the neighbour terms the sweeps will meet;
//   RESIDUAL - the residual itself, in FP64 (residualVector, :456-472).
// Every mode can add sum (R_rho / V)^2 of its cells to a per-case FP64 slot
// (densityResidualNorm, :480-491) with warp-shuffle reductions.
// No face-flux array goes through HBM.
#pragma once

#include "layout.cuh"

namespace bsd {

enum TileMode { MODE_STAGE = 0, MODE_PREPARE = 1, MODE_RESIDUAL = 2 };

template <class R>
struct TileArgs {
  const CaseDev* cases;
  const int2* tiles;      // (case, tile index within the case)
  const int* active;      // per case: 0 skips the case (may be null)
  StateView<R> src;       // the state the residual is evaluated on
  StateView<R> u0;        // STAGE: the state at the start of the step
  StateView<R> out;       // STAGE: the stage's output
  MetricsView m;
  float* dt;              // per cell local time step (arena like the state)
  const unsigned* dt_global; // per case FP32 bits of the global step (may be null)
  double* norm;           // per case sum of (R_rho / V)^2, or null
  unsigned* status;       // per case status bits
  double a, b;            // STAGE coefficients
  int first_stage;        // STAGE: compute the time step from src (== u0)
  float4* rec_f;          // PREPARE output: each cell's forward sweep record (5 float4)
  float4* rec_b;          // PREPARE output: its backward record, fields 1-4 (sweep_slot order)
  const float* cfl;       // PREPARE: per case current implicit CFL number
  const float* omega;     // PREPARE: per case omega
  double* res_out;        // RESIDUAL: 4 values per cell, arena like the state
  // PREPARE: the previous LU-SGS step's correction (row-major like the
  // state), or null. Each cell the tile reads (its own and its halo) is
  // src updated by it (applyImplicitUpdate), and the tile's own updated
  // cells are stored in upd_out - the other buffer of the state, since
  // neighbouring tiles still read src.
  const float4* dq_in;
  StateView<R> upd_out;
};

// Spectral radius |u . n| + a of a primitive state along (nx, ny), in FP32
// (the LU-SGS operator's face radii, src/engine-cpu/euler2d.ts:931-954).
template <class R>
__device__ __forceinline__ float radius32(R rho, R u, R v, R p, float gamma, float nx, float ny) {
  const float fr = float(rho), fu = float(u), fv = float(v), fp = float(p);
  return fabsf(fu * nx + fv * ny) + __fsqrt_rn((gamma * fp) / fr);
}

// The tile is TI x TJ cells on kThreads threads (the batch's default shape,
// or another the autotuner picked for the residual pass). kMinBlocks asks for
// that many resident CTAs per SM (at some spilling): on launches of several
// waves the extra CTA's warps fill the issue slots that the others leave
// while they wait at a barrier for their slowest face; on one wave fewer,
// larger register budgets are faster.
template <class R, int MODE, int kMinBlocks = 1, int TI = bsd::TI, int TJ = bsd::TJ, int kThreads = TILE_THREADS>
__global__ void __launch_bounds__(kThreads, kMinBlocks) tile_kernel(const TileArgs<R> A) {
  static_assert(TI * TJ <= kThreads, "a tile has at most one cell per thread");
  __shared__ R W[4][TJ + 4][TI + 4];
  __shared__ R Fi[4][TJ][TI + 1];
  __shared__ R Fj[4][TJ + 1][TI];

  // Launched behind the previous step's sweep (or a stage): everything below
  // reads its results. The residual pass then lets the sweep that follows it
  // be launched, so that kernel's launch and set-up overlap this one.
  griddep_wait();
  if (MODE == MODE_PREPARE) griddep_launch_dependents();
  const int2 tile = A.tiles[blockIdx.x];
  const int c = tile.x;
  if (A.active != nullptr && A.active[c] == 0) return;
  const CaseDev& cd = A.cases[c];
  const int ni = cd.ni, nj = cd.nj;
  const int tiles_i = (ni + TI - 1) / TI;
  const int i0 = (tile.y % tiles_i) * TI;
  const int j0 = (tile.y / tiles_i) * TJ;
  const int ti = min(TI, ni - i0), tj = min(TJ, nj - j0);
  const R gamma = R(cd.gamma);
  const int tid = threadIdx.x;
  const int li = tid % TI, lj = tid / TI;
  const bool mine = li < ti && lj < tj;
  const int i = i0 + li, j = j0 + lj;
  const int64_t k = cd.cell + i + int64_t(j) * ni;

  // Every cell is read through `at`: src, or src with the previous step's
  // correction applied (the same arithmetic in every tile that reads it, so
  // the halo of one tile is the interior of its neighbour exactly). A case
  // whose previous sweep gave up keeps its state.
  const bool apply = MODE == MODE_PREPARE && A.dq_in != nullptr && (A.status[c] & STATUS_TIMEOUT) == 0;
  auto at = [&](int64_t kk) -> Cons<R> {
    const Cons<R> q0 = A.src.load(kk);
    return apply ? implicit_update(q0, A.dq_in[kk], gamma) : q0;
  };

  // Own cell: conserved in registers, primitives in shared memory.
  Cons<R> qs{};
  if (mine) {
    qs = at(k);
    if (MODE == MODE_PREPARE && A.dq_in != nullptr) {
      A.upd_out.store(k, qs);
      if (!is_physical(qs, gamma)) atomicOr(&A.status[c], STATUS_NON_PHYSICAL);
    }
    const Prim<R> w = to_prim(qs, gamma);
    W[0][lj + 2][li + 2] = w.rho;
    W[1][lj + 2][li + 2] = w.u;
    W[2][lj + 2][li + 2] = w.v;
    W[3][lj + 2][li + 2] = w.p;
  }
  // Halo: two columns each side of the tile's rows, two rows each side of
  // its columns (the stencils are one-dimensional; corners are unused).
  for (int h = tid; h < 4 * TJ + 4 * TI; h += kThreads) {
    int hi, hj;
    bool valid;
    if (h < 4 * TJ) {
      const int col = h / TJ, row = h % TJ;
      valid = row < tj;
      hi = col < 2 ? i0 - 2 + col : i0 + ti + (col - 2);
      hj = j0 + row;
    } else {
      const int h2 = h - 4 * TJ;
      const int r = h2 / TI, col = h2 % TI;
      valid = col < ti;
      hj = r < 2 ? j0 - 2 + r : j0 + tj + (r - 2);
      hi = i0 + col;
    }
    if (valid) {
      const Prim<R> w = to_prim(cell_or_ghost<R>(cd, A.m, hi, hj, gamma, false, at), gamma);
      W[0][hj - j0 + 2][hi - i0 + 2] = w.rho;
      W[1][hj - j0 + 2][hi - i0 + 2] = w.u;
      W[2][hj - j0 + 2][hi - i0 + 2] = w.v;
      W[3][hj - j0 + 2][hi - i0 + 2] = w.p;
    }
  }
  __syncthreads();

  auto Wat = [&](int sj, int si) {
    return Prim<R>{W[0][sj][si], W[1][sj][si], W[2][sj][si], W[3][sj][si]};
  };

  // Every face of the tile once: its flux times its area.
  const int nfi = (ti + 1) * tj, nfj = ti * (tj + 1);
  for (int f = tid; f < nfi + nfj; f += kThreads) {
    R flux[4];
    Prim<R> left, right;
    if (f < nfi) {
      const int fl = f % (ti + 1), fr = f / (ti + 1);
      const int gi = i0 + fl, gj = j0 + fr;
      const FaceGeom<R> fm = face_geom<R>(A.m.iface, A.m.iface_lo, cd.iface + gi + int64_t(gj) * (ni + 1));
      const int sj = fr + 2, si = fl + 2;
      const double* imposed = (gi == 0 || gi == ni) ? cd.face_flux[gi == 0 ? BS_IMIN : BS_IMAX] : nullptr;
      if (imposed != nullptr) {
#pragma unroll
        for (int v = 0; v < 4; v++) flux[v] = R(imposed[4 * gj + v]);
      } else {
        face_states(cd.recon, cd.limiter, Wat(sj, si - 2), Wat(sj, si - 1), Wat(sj, si),
                    Wat(sj, si + 1), gamma, wall_side(cd, gi, ni, BS_IMIN, BS_IMAX), fm.nx, fm.ny,
                    left, right);
        face_flux(cd.flux, left, right, fm.nx, fm.ny, gamma, flux);
      }
      const R area = fm.area;
#pragma unroll
      for (int v = 0; v < 4; v++) Fi[v][fr][fl] = flux[v] * area;
    } else {
      const int f2 = f - nfi;
      const int fl = f2 % ti, fr = f2 / ti;
      const int gi = i0 + fl, gj = j0 + fr;
      const FaceGeom<R> fm = face_geom<R>(A.m.jface, A.m.jface_lo, cd.jface + gi + int64_t(gj) * ni);
      const int sj = fr + 2, si = fl + 2;
      const double* imposed = (gj == 0 || gj == nj) ? cd.face_flux[gj == 0 ? BS_JMIN : BS_JMAX] : nullptr;
      if (imposed != nullptr) {
#pragma unroll
        for (int v = 0; v < 4; v++) flux[v] = R(imposed[4 * gi + v]);
      } else {
        face_states(cd.recon, cd.limiter, Wat(sj - 2, si), Wat(sj - 1, si), Wat(sj, si),
                    Wat(sj + 1, si), gamma, wall_side(cd, gj, nj, BS_JMIN, BS_JMAX), fm.nx, fm.ny,
                    left, right);
        face_flux(cd.flux, left, right, fm.nx, fm.ny, gamma, flux);
      }
      const R area = fm.area;
#pragma unroll
      for (int v = 0; v < 4; v++) Fj[v][fr][fl] = flux[v] * area;
    }
  }
  __syncthreads();

  double nsq = 0;
  if (mine) {
    // Net inflow, in the order the reference accumulates it: west and east
    // i-faces, then south and north j-faces, then the source.
    R res[4];
#pragma unroll
    for (int v = 0; v < 4; v++)
      res[v] = ((Fi[v][lj][li] - Fi[v][lj][li + 1]) + Fj[v][lj][li]) - Fj[v][lj + 1][li];
    const float2 cm = A.m.cell[k];
    R V, planar;
    cell_geom<R>(A.m, k, &V, &planar);
    if (cd.axisym) res[2] = res[2] + pressure_of(qs.rho, qs.mu, qs.mv, qs.e, gamma) * planar;
    if (A.norm != nullptr) {
      const R r = res[0] / V;
      nsq = double(r) * double(r);
    }
    if (MODE == MODE_STAGE) {
      R dtc;
      if (!cd.local_dt) {
        dtc = R(__uint_as_float(A.dt_global[c]));
      } else if (A.first_stage) {
        const Prim<R> w = Wat(lj + 2, li + 2);
        const R a = dsqrt((gamma * w.p) / w.rho);
        const float4 fw = A.m.iface[cd.iface + i + int64_t(j) * (ni + 1)];
        const float4 fe = A.m.iface[cd.iface + i + 1 + int64_t(j) * (ni + 1)];
        const float4 fs = A.m.jface[cd.jface + i + int64_t(j) * ni];
        const float4 fn = A.m.jface[cd.jface + i + int64_t(j + 1) * ni];
        const R sxi = R(0.5) * (R(fw.x) * R(fw.z) + R(fe.x) * R(fe.z));
        const R syi = R(0.5) * (R(fw.y) * R(fw.z) + R(fe.y) * R(fe.z));
        const R sxj = R(0.5) * (R(fs.x) * R(fs.z) + R(fn.x) * R(fn.z));
        const R syj = R(0.5) * (R(fs.y) * R(fs.z) + R(fn.y) * R(fn.z));
        const R lambda = (fabs(w.u * sxi + w.v * syi) + a * hypot(sxi, syi)) +
                         (fabs(w.u * sxj + w.v * syj) + a * hypot(sxj, syj));
        const float d32 = float((R(cd.cfl) * V) / lambda);
        A.dt[k] = d32;
        dtc = R(d32);
      } else {
        dtc = R(A.dt[k]);
      }
      const R factor = dtc / V;
      const R a = R(A.a), b = R(A.b);
      Cons<R> o;
      if (A.a != 0.0) {
        const Cons<R> q0 = A.u0.load(k);
        o = {a * q0.rho + b * (qs.rho + factor * res[0]), a * q0.mu + b * (qs.mu + factor * res[1]),
             a * q0.mv + b * (qs.mv + factor * res[2]), a * q0.e + b * (qs.e + factor * res[3])};
      } else {
        o = {b * (qs.rho + factor * res[0]), b * (qs.mu + factor * res[1]),
             b * (qs.mv + factor * res[2]), b * (qs.e + factor * res[3])};
      }
      A.out.store(k, o);
      if (!is_physical(o, gamma)) atomicOr(&A.status[c], STATUS_NON_PHYSICAL);
    } else if (MODE == MODE_PREPARE) {
      // The sweep records (see lusgs_sweep_kernel): the residual, 1/D and,
      // for each neighbour the sweep meets, its density, velocity and
      // H = E + p with the face's signed normal times A/2 and hud =
      // (u, v) . (hnx, hny) - omega lambda A/2 - everything the sweeps need
      // that does not depend on dQ, computed here where every cell is
      // independent and the neighbours' states are in the tile.
      const float g = float(gamma);
      const float4 fw = A.m.iface[cd.iface + i + int64_t(j) * (ni + 1)];
      const float4 fe = A.m.iface[cd.iface + i + 1 + int64_t(j) * (ni + 1)];
      const float4 fs = A.m.jface[cd.jface + i + int64_t(j) * ni];
      const float4 fn = A.m.jface[cd.jface + i + int64_t(j + 1) * ni];
      const int sj = lj + 2, si = li + 2;
      auto rad = [&](int aj, int ai, float nx, float ny) {
        return radius32(W[0][aj][ai], W[1][aj][ai], W[2][aj][ai], W[3][aj][ai], g, nx, ny);
      };
      const float lw = fmaxf(i > 0 ? rad(sj, si - 1, fw.x, fw.y) : 0.f, rad(sj, si, fw.x, fw.y)) * fw.z;
      const float le = fmaxf(rad(sj, si, fe.x, fe.y), i + 1 < ni ? rad(sj, si + 1, fe.x, fe.y) : 0.f) * fe.z;
      const float ls = fmaxf(j > 0 ? rad(sj - 1, si, fs.x, fs.y) : 0.f, rad(sj, si, fs.x, fs.y)) * fs.z;
      const float ln = fmaxf(rad(sj, si, fn.x, fn.y), j + 1 < nj ? rad(sj + 1, si, fn.x, fn.y) : 0.f) * fn.z;
      const float omega = A.omega[c];
      const float scale = 0.5f * (omega + 1.f / A.cfl[c]);
      const float diag = scale * (lw + le + ls + ln) + (cd.axisym ? cm.y * rad(sj, si, 0.f, 1.f) : 0.f);
      const float hk = g / (g - 1.f);
      // (rho, u, v, H) and (hnx, hny, hud, 0) of the neighbour at (aj, ai)
      // across face f, the flux leaving through sgn n; an absent neighbour
      // gets the inert (1, 0, 0, 0), (0, 0, 0, 0).
      auto term = [&](bool present, int aj, int ai, float4 f, float sgn, float lam, float4& q4, float4& f4) {
        if (!present) {
          q4 = make_float4(1.f, 0.f, 0.f, 0.f);
          f4 = make_float4(0.f, 0.f, 0.f, 0.f);
          return;
        }
        const float rho = float(W[0][aj][ai]), u = float(W[1][aj][ai]), v = float(W[2][aj][ai]);
        const float p = float(W[3][aj][ai]);
        const float h = 0.5f * f.z * sgn;
        const float hnx = h * f.x, hny = h * f.y;
        q4 = make_float4(rho, u, v, fmaf(hk, p, 0.5f * rho * (u * u + v * v)));
        f4 = make_float4(hnx, hny, (hnx * u + hny * v) - 0.5f * omega * lam, 0.f);
      };
      float4 aq, af, bq, bf;
      const int64_t slot = REC_SIZE * (cd.slot + sweep_slot(ni, nj, i, j));
      float4* rf = A.rec_f + slot;
      term(i > 0, sj, si - 1, fw, -1.f, lw, aq, af);
      term(j > 0, sj - 1, si, fs, -1.f, ls, bq, bf);
      rf[0] = make_float4(float(res[0]), float(res[1]), float(res[2]), float(res[3]));
      rf[1] = make_float4(1.f / diag, aq.x, aq.y, aq.z);
      rf[2] = make_float4(aq.w, af.x, af.y, af.z);
      rf[3] = bq;
      rf[4] = make_float4(bf.x, bf.y, bf.z, 0.f);
      float4* rb = A.rec_b + slot;
      term(i + 1 < ni, sj, si + 1, fe, 1.f, le, aq, af);
      term(j + 1 < nj, sj + 1, si, fn, 1.f, ln, bq, bf);
      rb[1] = make_float4(1.f / diag, aq.x, aq.y, aq.z);
      rb[2] = make_float4(aq.w, af.x, af.y, af.z);
      rb[3] = bq;
      rb[4] = make_float4(bf.x, bf.y, bf.z, 0.f);
    } else if (A.res_out != nullptr) {
      double* o = A.res_out + 4 * k;
      o[0] = double(res[0]);
      o[1] = double(res[1]);
      o[2] = double(res[2]);
      o[3] = double(res[3]);
    }
  }
  if (A.norm != nullptr) {
    nsq = warp_sum(nsq);
    if ((tid & 31) == 0 && nsq != 0.0) atomicAdd(&A.norm[c], nsq);
  }
}

// Local time step of every cell of the tile (computeTimeSteps,
// src/engine-cpu/euler2d.ts:1183-1205), written as FP32; with `dt_min_bits`
// also each case's smallest step, as the bits of a positive float (ordered
// like its value) combined by atomicMin, for global time stepping.
template <class R>
__global__ void __launch_bounds__(TILE_THREADS) dt_kernel(const CaseDev* cases, const int2* tiles,
                                                          const int* active, StateView<R> q,
                                                          MetricsView m, float* dt,
                                                          unsigned* dt_min_bits) {
  const int2 tile = tiles[blockIdx.x];
  const int c = tile.x;
  if (active != nullptr && active[c] == 0) return;
  const CaseDev& cd = cases[c];
  const int ni = cd.ni, nj = cd.nj;
  const int tiles_i = (ni + TI - 1) / TI;
  const int i = (tile.y % tiles_i) * TI + threadIdx.x % TI;
  const int j = (tile.y / tiles_i) * TJ + threadIdx.x / TI;
  if (i >= ni || j >= nj || int(threadIdx.x) >= TI * TJ) return;
  const R gamma = R(cd.gamma);
  const int64_t k = cd.cell + i + int64_t(j) * ni;
  const Prim<R> w = to_prim(q.load(k), gamma);
  const R a = dsqrt((gamma * w.p) / w.rho);
  const float4 fw = m.iface[cd.iface + i + int64_t(j) * (ni + 1)];
  const float4 fe = m.iface[cd.iface + i + 1 + int64_t(j) * (ni + 1)];
  const float4 fs = m.jface[cd.jface + i + int64_t(j) * ni];
  const float4 fn = m.jface[cd.jface + i + int64_t(j + 1) * ni];
  const R sxi = R(0.5) * (R(fw.x) * R(fw.z) + R(fe.x) * R(fe.z));
  const R syi = R(0.5) * (R(fw.y) * R(fw.z) + R(fe.y) * R(fe.z));
  const R sxj = R(0.5) * (R(fs.x) * R(fs.z) + R(fn.x) * R(fn.z));
  const R syj = R(0.5) * (R(fs.y) * R(fs.z) + R(fn.y) * R(fn.z));
  const R lambda = (fabs(w.u * sxi + w.v * syi) + a * hypot(sxi, syi)) +
                   (fabs(w.u * sxj + w.v * syj) + a * hypot(sxj, syj));
  const float d32 = float((R(cd.cfl) * R(m.cell[k].x)) / lambda);
  dt[k] = d32;
  if (dt_min_bits != nullptr && d32 > 0.f) atomicMin(&dt_min_bits[c], __float_as_uint(d32));
}

}  // namespace bsd
