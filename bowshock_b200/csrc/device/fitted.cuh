// The fitted bow shock on the GPU (fitShock, src/solver/shock-fitting.ts:
// 170-314): the shock is the jMax boundary, a curve of nodes on straight
// grid lines from the body; all of one step runs on the device:
//   fit_boundary_kernel  per jMax face, the shock compatible with the flow in
//                        the two cells below it (compatibleShock, :87-111):
//                        its post-shock state fills the ghosts, its physical
//                        flux is imposed on the face, its speed is kept;
//   (the explicit step, with those held; its last stage writes q_old)
//   fit_move_kernel      one block: each shock node moves along its line by
//                        W dt / (n . line), W from the face on its axis side,
//                        dt half the top cell's height over its fastest
//                        signal; the axis node keeps the shock normal to the
//                        axis ('symmetry') or stays ('fixed');
//   fit_regrid_kernel    the grid on the new heights (each node at its fixed
//                        fraction of its line's height) and its metrics,
//                        FP64 computed, stored as the solver stores them
//                        (src/grid/structured.ts:94-168), and the flow
//                        interpolated along the lines onto it
//                        (remapAlongLines, :324-358), in one launch.
// Everything is FP64 except the stored face and cell metrics (FP32, as for
// every grid here).
#pragma once

#include "layout.cuh"

namespace bsd {

struct FitArgs {
  const CaseDev* cases;      // the one case
  int ni, nj;
  double gamma;
  double free[4];            // free-stream primitives
  double a_free;
  const double* line;        // (ni + 1) x (x, y, dx, dy)
  const double* fraction;    // (ni + 1) x (nj + 1), line-major
  double* heights;           // (ni + 1) current
  double* heights_old;       // (ni + 1) before the last move
  double* heights_next;      // (ni + 1) scratch of the move
  double* nx_;               // node x, (ni + 1)(nj + 1), node (i, j) at i + j (ni + 1)
  double* ny_;               // node y
  double* face_state;        // jMax: 4 conserved per face
  double* face_flux;         // jMax: 4 per face, per unit area
  double* speed;             // jMax: shock speed per face
  double* max_speed;         // |W| / a_inf, largest over the faces of the last move
  int first_node;            // 0 fixed, 1 symmetry
  int axisym;
  float4* iface;
  float4* jface;
  float2* cellm;
  // The metrics' FP32 low parts (the FP64 value less the FP32 one): the
  // residual reads two-float metrics, its steady state that of FP64 metrics.
  float4* iface_lo;
  float4* jface_lo;
  float2* cellm_lo;
  double* bgeom;             // boundary faces iMin, iMax, jMin, jMax: (nx, ny, area)
  StateView<double> q;       // the state at the start of a step, and after the remap
  StateView<double> q_old;   // the state after the step's last stage, on the grid before the move
};

// The FP32 low part of an FP64 value: v less its FP32 rounding.
__device__ __forceinline__ float low_part(double v) { return float(v - double(float(v))); }

__device__ __forceinline__ void fit_shock_state(const FitArgs& A, double mach, double nx, double ny, double w[4],
                                                double* speed, double* un) {
  const double* f = A.free;
  const double g = A.gamma;
  const double vn = f[1] * nx + f[2] * ny;
  *speed = mach * A.a_free + vn;
  const double m2 = mach * mach;
  const double dr = ((g + 1) * m2) / ((g - 1) * m2 + 2);
  const double pr = 1 + ((2 * g) / (g + 1)) * (m2 - 1);
  *un = *speed - (mach * A.a_free) / dr;
  w[0] = f[0] * dr;
  w[1] = f[1] + (*un - vn) * nx;
  w[2] = f[2] + (*un - vn) * ny;
  w[3] = f[3] * pr;
}

// The jMax face i's unit normal, from the nodes (the face runs from node
// (i + 1, nj) to node (i, nj); its normal is on the right).
__device__ __forceinline__ void fit_top_normal(const FitArgs& A, int i, double* nx, double* ny) {
  const int64_t a = (i + 1) + int64_t(A.nj) * (A.ni + 1), b = i + int64_t(A.nj) * (A.ni + 1);
  const double dx = A.nx_[b] - A.nx_[a], dy = A.ny_[b] - A.ny_[a];
  const double len = hypot(dx, dy);
  *nx = len > 0 ? dy / len : 0;
  *ny = len > 0 ? -dx / len : 0;
}

__device__ __forceinline__ Prim<double> fit_prim(const FitArgs& A, const StateView<double>& q, int i, int j) {
  return to_prim(q.load(int64_t(i) + int64_t(j) * A.ni), A.gamma);
}

__global__ void fit_boundary_kernel(const FitArgs A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.ni) return;
  double nx, ny;
  fit_top_normal(A, i, &nx, &ny);
  const Prim<double> c1 = fit_prim(A, A.q, i, A.nj - 1), c2 = fit_prim(A, A.q, i, A.nj - 2);
  const double g = A.gamma;
  const double impedance = c1.rho * sqrt(g * c1.p / c1.rho);
  const double p_face = 1.5 * c1.p - 0.5 * c2.p;
  const double un_face = 1.5 * (c1.u * nx + c1.v * ny) - 0.5 * (c2.u * nx + c2.v * ny);
  const double target = p_face + impedance * un_face;
  double w[4], speed, un;
  auto mismatch = [&](double m) {
    fit_shock_state(A, m, nx, ny, w, &speed, &un);
    return w[3] + impedance * un - target;
  };
  double mach = 1;
  if (mismatch(1.0) < 0) {
    // The root of the increasing mismatch, where the reference bisects from
    // [1, 2] (doubling the top) to a bracket of 1e-15 of its top: Newton
    // steps kept inside the bracket that every evaluation narrows, halving
    // it instead where a step would leave it, to the same width. The
    // mismatch's derivative: dp_s/dM = p 4 gamma M / (gamma + 1) and
    // du_n,s/dM = 2 a (1 + 1 / M^2) / (gamma + 1).
    const double gp1 = g + 1;
    double low = 1, high = INFINITY, m = 1;
    for (int k = 0; k < 200; k++) {
      const double f = mismatch(m);
      if (f == 0) break;  // the root itself
      if (f < 0)
        low = m;
      else
        high = m;
      if (high < INFINITY && high - low <= 1e-15 * high) break;
      const double df = A.free[3] * 4 * g * m / gp1 + impedance * 2 * A.a_free * (1 + 1 / (m * m)) / gp1;
      double next = m - f / df;
      if (next == m) break;  // a step below the last bit
      if (!(next > low && next < high)) next = high < INFINITY ? 0.5 * (low + high) : 2 * low;
      m = next;
    }
    mach = m;
  }
  fit_shock_state(A, mach, nx, ny, w, &speed, &un);
  const double energy = w[3] / (g - 1) + 0.5 * w[0] * (w[1] * w[1] + w[2] * w[2]);
  const double wn = w[1] * nx + w[2] * ny;
  double* s = A.face_state + 4 * i;
  s[0] = w[0];
  s[1] = w[0] * w[1];
  s[2] = w[0] * w[2];
  s[3] = energy;
  double* f = A.face_flux + 4 * i;
  f[0] = w[0] * wn;
  f[1] = w[0] * w[1] * wn + w[3] * nx;
  f[2] = w[0] * w[2] * wn + w[3] * ny;
  f[3] = wn * (energy + w[3]);
  A.speed[i] = speed;
}

// One block: the new heights from the last boundary's speeds and the flow
// after the step (q_old), on the grid before the move.
__global__ void fit_move_kernel(const FitArgs A) {
  __shared__ double worst[32];
  const int ni = A.ni, nj = A.nj;
  const double g = A.gamma;
  double w_max = 0;
  for (int f = threadIdx.x; f < ni; f += blockDim.x) w_max = fmax(w_max, fabs(A.speed[f]) / A.a_free);
  for (int k = 1 + threadIdx.x; k <= ni; k += blockDim.x) {
    const int f = k - 1;
    double nx, ny;
    fit_top_normal(A, f, &nx, &ny);
    const Prim<double> cell = fit_prim(A, A.q_old, min(k, ni - 1), nj - 1);
    const int64_t top = k + int64_t(nj) * (ni + 1), below = k + int64_t(nj - 1) * (ni + 1);
    const double height = hypot(A.nx_[top] - A.nx_[below], A.ny_[top] - A.ny_[below]);
    const double dt = (0.5 * height) / (hypot(cell.u, cell.v) + sqrt(g * cell.p / cell.rho));
    const double* l = A.line + 4 * k;
    A.heights_next[k] = A.heights[k] + (A.speed[f] * dt) / (l[2] * nx + l[3] * ny);
  }
  // The largest speed over the block.
  for (int o = 16; o > 0; o >>= 1) w_max = fmax(w_max, __shfl_xor_sync(0xffffffffu, w_max, o));
  if ((threadIdx.x & 31) == 0) worst[threadIdx.x >> 5] = w_max;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0;
    for (int k = 0; k < int(blockDim.x + 31) / 32; k++) m = fmax(m, worst[k]);
    *A.max_speed = m;
    double h0 = A.heights[0];
    if (A.first_node == 1) {
      // Normal to the axis: on the parabola x = x0 + c y^2 through the next two nodes.
      const double* l0 = A.line;
      const double* l1 = A.line + 4;
      const double* l2 = A.line + 8;
      const double x1 = l1[0] + A.heights_next[1] * l1[2], y1 = l1[1] + A.heights_next[1] * l1[3];
      const double x2 = l2[0] + A.heights_next[2] * l2[2], y2 = l2[1] + A.heights_next[2] * l2[3];
      const double c = (x2 - x1) / (y2 * y2 - y1 * y1);
      h0 = (x1 - c * y1 * y1 - l0[0]) / l0[2];
    }
    A.heights_next[0] = h0;
  }
  __syncthreads();
  for (int k = threadIdx.x; k <= ni; k += blockDim.x) {
    A.heights_old[k] = A.heights[k];
    A.heights[k] = A.heights_next[k];
  }
}

// Node (i, j) on its line at the current heights (gridOnLines,
// src/grid/blunt-grid.ts:602-620).
__device__ __forceinline__ void fit_node(const FitArgs& A, int i, int j, double* x, double* y) {
  const double* l = A.line + 4 * i;
  const double d = A.heights[i] * A.fraction[int64_t(i) * (A.nj + 1) + j];
  *x = l[0] + d * l[2];
  *y = l[1] + d * l[3];
}

// The grid on the new heights and, with `remap`, the flow on it, in one
// pass over a flat index: the nodes; the metrics (computeMetrics,
// src/grid/structured.ts:94-168), i-faces, j-faces and cells, FP64 computed
// from the node positions evaluated here, stored FP32, with the boundary
// faces' FP64 geometry for the wall fluxes; and the remap along the lines
// (remapAlongLines, src/solver/shock-fitting.ts:324-358), linear in the
// primitives between the old cell centres of the column, held at the end
// cells beyond them, from q_old into q (a node's distance along its line is
// its height times its fraction: the lines' directions are unit vectors).
__global__ void fit_regrid_kernel(const FitArgs A, int remap) {
  const int ni = A.ni, nj = A.nj;
  const int64_t nn = int64_t(ni + 1) * (nj + 1), nif = int64_t(ni + 1) * nj, njf = int64_t(ni) * (nj + 1),
                nc = int64_t(ni) * nj;
  const int64_t total = nn + nif + njf + nc + (remap ? nc : 0);
  auto face = [&](int ia, int ja, int ib, int jb, double* fx, double* fy, double* fa) {
    double xa, ya, xb, yb;
    fit_node(A, ia, ja, &xa, &ya);
    fit_node(A, ib, jb, &xb, &yb);
    const double dx = xb - xa, dy = yb - ya;
    const double length = hypot(dx, dy);
    *fx = length > 0 ? dy / length : 0;
    *fy = length > 0 ? -dx / length : 0;
    *fa = A.axisym ? length * 0.5 * (ya + yb) : length;
  };
  for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x) {
    double fx, fy, fa;
    if (k < nn) {
      const int i = int(k % (ni + 1)), j = int(k / (ni + 1));
      fit_node(A, i, j, &A.nx_[k], &A.ny_[k]);
    } else if (k < nn + nif) {
      const int64_t m = k - nn;
      const int i = int(m % (ni + 1)), j = int(m / (ni + 1));
      face(i, j, i, j + 1, &fx, &fy, &fa);
      A.iface[m] = make_float4(float(fx), float(fy), float(fa), 0.f);
      A.iface_lo[m] = make_float4(low_part(fx), low_part(fy), low_part(fa), 0.f);
      if (i == 0 || i == ni) {
        double* g = A.bgeom + 3 * ((i == 0 ? 0 : nj) + j);
        g[0] = fx;
        g[1] = fy;
        g[2] = fa;
      }
    } else if (k < nn + nif + njf) {
      const int64_t m = k - nn - nif;
      const int i = int(m % ni), j = int(m / ni);
      face(i + 1, j, i, j, &fx, &fy, &fa);
      A.jface[m] = make_float4(float(fx), float(fy), float(fa), 0.f);
      A.jface_lo[m] = make_float4(low_part(fx), low_part(fy), low_part(fa), 0.f);
      if (j == 0 || j == nj) {
        double* g = A.bgeom + 3 * (2 * nj + (j == 0 ? 0 : ni) + i);
        g[0] = fx;
        g[1] = fy;
        g[2] = fa;
      }
    } else if (k < nn + nif + njf + nc) {
      const int64_t m = k - nn - nif - njf;
      const int i = int(m % ni), j = int(m / ni);
      double cx[4], cy[4];
      fit_node(A, i, j, &cx[0], &cy[0]);
      fit_node(A, i + 1, j, &cx[1], &cy[1]);
      fit_node(A, i + 1, j + 1, &cx[2], &cy[2]);
      fit_node(A, i, j + 1, &cx[3], &cy[3]);
      double area = 0, sy = 0;
      for (int e = 0; e < 4; e++) {
        const int r = (e + 1) % 4;
        const double cross = cx[e] * cy[r] - cx[r] * cy[e];
        area += cross;
        sy += (cy[e] + cy[r]) * cross;
      }
      area *= 0.5;
      const double ycen = sy / (6 * area);
      const double volume = A.axisym ? area * ycen : area;
      A.cellm[m] = make_float2(float(volume), float(area));
      A.cellm_lo[m] = make_float2(low_part(volume), low_part(area));
    } else {
      const int64_t m = k - nn - nif - njf - nc;
      const int i = int(m % ni), j = int(m / ni);
      const double* f0 = A.fraction + int64_t(i) * (nj + 1);
      const double* f1 = A.fraction + int64_t(i + 1) * (nj + 1);
      auto column = [&](const double* h, int jj) { return 0.5 * (h[i] * f0[jj] + h[i + 1] * f1[jj]); };
      const double d = 0.5 * (column(A.heights, j) + column(A.heights, j + 1));
      auto centre = [&](int jj) { return 0.5 * (column(A.heights_old, jj) + column(A.heights_old, jj + 1)); };
      int jj = 0;
      while (jj < nj - 2 && centre(jj + 1) < d) jj++;
      const double c0 = centre(jj), c1 = centre(jj + 1);
      const double t = fmin(fmax((d - c0) / (c1 - c0), 0.0), 1.0);
      const Prim<double> a = to_prim(A.q_old.load(int64_t(i) + int64_t(jj) * ni), A.gamma);
      const Prim<double> b = to_prim(A.q_old.load(int64_t(i) + int64_t(jj + 1) * ni), A.gamma);
      const Prim<double> w{a.rho + t * (b.rho - a.rho), a.u + t * (b.u - a.u), a.v + t * (b.v - a.v),
                           a.p + t * (b.p - a.p)};
      A.q.store(m, to_cons(w, A.gamma));
    }
  }
}

}  // namespace bsd
