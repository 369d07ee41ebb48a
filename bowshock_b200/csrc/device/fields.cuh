// Per-cell display fields of a case, computed on the GPU into a buffer (the
// compute half of the reference's flow view; drawing is graphics and is not
// done here): src/render/flow-fields.ts:36-117, the twin of
// src/render/shaders/flow-fields.wgsl.
//   0 schlieren: |grad rho| by Green-Gauss over the cell's four faces in the
//     plane of the grid, each face taking the mean density of the two cells
//     either side (the cell's own on the boundary), times `length` over the
//     free stream's density;
//   1 Mach number; 2 pressure coefficient (p - p_inf) / (rho_inf V_inf^2 / 2);
//   3 density over the free stream's.
#pragma once

#include "layout.cuh"

namespace bsd {

enum { FIELD_SCHLIEREN = 0, FIELD_MACH = 1, FIELD_CP = 2, FIELD_DENSITY = 3 };

template <class R>
__global__ void flow_field_kernel(const CaseDev* cases, int c, StateView<R> q, const double* x,
                                  const double* y, int field, double length, double rho_inf, double u_inf,
                                  double v_inf, double p_inf, double* out) {
  const CaseDev& cd = cases[c];
  const int ni = cd.ni, nj = cd.nj;
  const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= int64_t(ni) * nj) return;
  const int i = int(k % ni), j = int(k / ni);
  const double gamma = cd.gamma;
  auto rho_at = [&](int a, int b) { return double(q.rho[cd.cell + a + int64_t(b) * ni]); };
  if (field == FIELD_SCHLIEREN) {
    const int row = ni + 1;
    const int corner[4] = {i + j * row, i + 1 + j * row, i + 1 + (j + 1) * row, i + (j + 1) * row};
    const int across[4][2] = {{i, j - 1}, {i + 1, j}, {i, j + 1}, {i - 1, j}};
    const double own = rho_at(i, j);
    double gx = 0, gy = 0, area = 0;
    for (int e = 0; e < 4; e++) {
      const int a = corner[e], b = corner[(e + 1) & 3];
      const int ai = across[e][0], aj = across[e][1];
      const bool inside = ai >= 0 && ai < ni && aj >= 0 && aj < nj;
      const double qf = inside ? 0.5 * (own + rho_at(ai, aj)) : own;
      const double dx = x[b] - x[a], dy = y[b] - y[a];
      gx += qf * dy;
      gy -= qf * dx;
      area += 0.5 * (x[a] * y[b] - x[b] * y[a]);
    }
    out[k] = sqrt(gx * gx + gy * gy) / fabs(area) * length / rho_inf;
    return;
  }
  const int64_t kk = cd.cell + k;
  const double rho = double(q.rho[kk]), mu = double(q.mu[kk]), mv = double(q.mv[kk]), e = double(q.e[kk]);
  const double p = (gamma - 1) * (e - 0.5 * (mu * mu + mv * mv) / rho);
  if (field == FIELD_MACH) {
    out[k] = sqrt(mu * mu + mv * mv) / rho / sqrt(gamma * p / rho);
  } else if (field == FIELD_CP) {
    out[k] = (p - p_inf) / (0.5 * rho_inf * (u_inf * u_inf + v_inf * v_inf));
  } else {
    out[k] = rho / rho_inf;
  }
}

}  // namespace bsd
