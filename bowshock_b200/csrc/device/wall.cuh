// Boundary-face fluxes and the forebody pressure drag, in FP64 on the GPU
// (boundaryFluxes, src/engine-cpu/euler2d.ts:499-525; forebodyPressureDrag,
// src/analysis/forces.ts:19-30). The state is read in its stored type; an
// FP32 state is taken to primitives with the FP32 gamma it was solved with and
// then evaluated in FP64 with the configured gamma, as the reference's GPU
// engine does on its host (gpuPrimitive2D, src/engine-gpu/euler2d-gpu.ts:136-146;
// src/analysis/gpu-engine.ts:27-31).
#pragma once

#include "layout.cuh"

namespace bsd {

template <class R>
struct BoundaryArgs {
  const CaseDev* cases;
  int case_index;
  StateView<R> q;
  MetricsView m;
  int side;
  const double* geom;   // per face of the side: stored unit normal (nx, ny) and area, FP64
  double gamma_eval;    // the configured gamma
  double* flux_out;     // per face: 4 values along the outward normal
  double p_inf;         // drag: free-stream pressure
  double* force_out;    // drag: sum (f_x - p_inf n_x) A, or null
};

template <class R>
__device__ __forceinline__ Cons<double> adapt_state(const Cons<R>& q, double gamma_state,
                                                    double gamma_eval) {
  const Cons<double> d{double(q.rho), double(q.mu), double(q.mv), double(q.e)};
  if (gamma_state == gamma_eval) return d;
  return to_cons(to_prim(d, gamma_state), gamma_eval);
}

template <class R>
__global__ void __launch_bounds__(256) boundary_flux_kernel(const BoundaryArgs<R> A) {
  __shared__ double partial[8];
  const CaseDev& cd = A.cases[A.case_index];
  const int ni = cd.ni, nj = cd.nj;
  const bool idir = A.side == BS_IMIN || A.side == BS_IMAX;
  const int along = idir ? nj : ni;
  const double ge = A.gamma_eval;
  const double gs = cd.gamma;
  const int outward = (A.side == BS_IMIN || A.side == BS_JMIN) ? -1 : 1;
  auto at = [&](int64_t k) { return adapt_state(A.q.load(k), gs, ge); };
  double force = 0;
  for (int t = threadIdx.x; t < along; t += blockDim.x) {
    const double nx = A.geom[3 * t], ny = A.geom[3 * t + 1], area = A.geom[3 * t + 2];
    Prim<double> w[4];
    if (idir) {
      const int i = A.side == BS_IMIN ? 0 : ni;
      for (int s = 0; s < 4; s++)
        w[s] = to_prim(cell_or_ghost<double>(cd, A.m, i - 2 + s, t, ge, true, at), ge);
    } else {
      const int j = A.side == BS_JMIN ? 0 : nj;
      for (int s = 0; s < 4; s++)
        w[s] = to_prim(cell_or_ghost<double>(cd, A.m, t, j - 2 + s, ge, true, at), ge);
    }
    const int wall = cd.bc[A.side] == BS_BC_WALL ? outward : 0;
    Prim<double> left, right;
    face_states(cd.recon, cd.limiter, w[0], w[1], w[2], w[3], ge, wall, nx, ny, left, right);
    double f[4];
    face_flux(cd.flux, left, right, nx, ny, ge, f);
    double* o = A.flux_out + 4 * t;
    for (int v = 0; v < 4; v++) o[v] = outward * f[v];
    force += (o[1] - A.p_inf * (outward * nx)) * area;
  }
  if (A.force_out == nullptr) return;
  force = warp_sum(force);
  if ((threadIdx.x & 31) == 0) partial[threadIdx.x >> 5] = force;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int w = 0; w < int(blockDim.x >> 5); w++) s += partial[w];
    *A.force_out = s;
  }
}

}  // namespace bsd
