// Finite-volume metrics of a structured grid in FP64 on the host
// (computeMetrics, src/grid/structured.ts:94-168): face unit normals and
// areas (length times midpoint radius when axisymmetric), cell planar areas
// by the shoelace formula, centroids and volumes (planar area times centroid
// radius when axisymmetric).
#pragma once

#include <string>
#include <vector>

namespace bs {

struct Metrics64 {
  int ni = 0, nj = 0;
  bool axisymmetric = false;
  std::vector<double> inx, iny, iarea;  // (ni + 1) nj i-faces, normal towards +i
  std::vector<double> jnx, jny, jarea;  // ni (nj + 1) j-faces, normal towards +j
  std::vector<double> volume, planar, cx, cy;
};

// "" on success, else the reference's RangeError message.
std::string compute_metrics64(int ni, int nj, const double* x, const double* y, bool axisymmetric,
                              Metrics64& out);

}  // namespace bs
