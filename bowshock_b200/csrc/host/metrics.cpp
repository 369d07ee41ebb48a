// FP64 grid metrics on the host (src/grid/structured.ts:94-168).
#include "metrics.hpp"

#include <cmath>

namespace bs {

std::string compute_metrics64(int ni, int nj, const double* x, const double* y, bool axisym,
                              Metrics64& m) {
  m.ni = ni;
  m.nj = nj;
  m.axisymmetric = axisym;
  const size_t nn = size_t(ni + 1) * (nj + 1);
  if (axisym)
    for (size_t k = 0; k < nn; k++)
      if (y[k] < 0) return "axisymmetric grids must have y >= 0 (y is the radius)";
  auto node = [&](int i, int j) { return size_t(i) + size_t(j) * (ni + 1); };
  // A face from node a to node b has its normal on the right of a -> b.
  auto face = [&](std::vector<double>& fx, std::vector<double>& fy, std::vector<double>& fa,
                  size_t k, size_t a, size_t b) {
    const double dx = x[b] - x[a], dy = y[b] - y[a];
    const double length = std::hypot(dx, dy);
    fx[k] = length > 0 ? dy / length : 0;
    fy[k] = length > 0 ? -dx / length : 0;
    fa[k] = axisym ? length * 0.5 * (y[a] + y[b]) : length;
  };
  const size_t nif = size_t(ni + 1) * nj, njf = size_t(ni) * (nj + 1), nc = size_t(ni) * nj;
  m.inx.assign(nif, 0); m.iny.assign(nif, 0); m.iarea.assign(nif, 0);
  m.jnx.assign(njf, 0); m.jny.assign(njf, 0); m.jarea.assign(njf, 0);
  for (int j = 0; j < nj; j++)
    for (int i = 0; i <= ni; i++)
      face(m.inx, m.iny, m.iarea, i + size_t(j) * (ni + 1), node(i, j), node(i, j + 1));
  for (int j = 0; j <= nj; j++)
    for (int i = 0; i < ni; i++)
      face(m.jnx, m.jny, m.jarea, i + size_t(j) * ni, node(i + 1, j), node(i, j));
  m.volume.assign(nc, 0); m.planar.assign(nc, 0); m.cx.assign(nc, 0); m.cy.assign(nc, 0);
  for (int j = 0; j < nj; j++)
    for (int i = 0; i < ni; i++) {
      // Corners counter-clockwise for a right-handed grid.
      const size_t corner[4] = {node(i, j), node(i + 1, j), node(i + 1, j + 1), node(i, j + 1)};
      double area = 0, sx = 0, sy = 0;
      for (int c = 0; c < 4; c++) {
        const size_t p = corner[c], q = corner[(c + 1) % 4];
        const double cross = x[p] * y[q] - x[q] * y[p];
        area += cross;
        sx += (x[p] + x[q]) * cross;
        sy += (y[p] + y[q]) * cross;
      }
      area *= 0.5;
      if (!(area > 0))
        return "cell (" + std::to_string(i) + ", " + std::to_string(j) + ") has non-positive area";
      const size_t k = i + size_t(j) * ni;
      m.planar[k] = area;
      m.cx[k] = sx / (6 * area);
      m.cy[k] = sy / (6 * area);
      m.volume[k] = axisym ? area * m.cy[k] : area;
    }
  return "";
}

}  // namespace bs
