// Structured grids around bodies of revolution and their quality measures:
// src/grid/body-grid.ts (H topology, sharp noses), src/grid/spacing.ts
// (column placement), src/grid/quality.ts (quality gates),
// src/grid/shapes.ts (ramp grids for validation).
#pragma once

#include <cmath>
#include <functional>
#include <string>
#include <vector>

#include "geometry.hpp"

namespace bs {

struct Grid {
  int ni = 0, nj = 0;
  std::vector<double> x, y;  // (ni + 1)(nj + 1) nodes, node (i, j) at i + j (ni + 1)
  int i_tip = 0;
  double outer_angle = 0;
  // A C grid whose boundary is placed at the tip's blunt part, narrower
  // than the body (BluntGrid.twoScale, src/grid/blunt-grid.ts:553).
  bool two_scale = false;
};

struct GridQuality {  // src/grid/quality.ts:6-21
  double min_angle, min_wall_angle, max_size_ratio, max_aspect_ratio, min_area;
};

struct QualityLimits {  // src/grid/quality.ts:24-38
  double min_angle = 12 * M_PI / 180;
  double min_wall_angle = 60 * M_PI / 180;
  double max_size_ratio = 1.3;
  double max_aspect_ratio = 10;
};

GridQuality grid_quality(int ni, int nj, const double* x, const double* y);
std::vector<std::string> quality_failures(const GridQuality& q, const QualityLimits& limits);

// columnPositions (src/grid/spacing.ts:31-71), without the slope limiter of
// the blunt grids. When `total` > 0 the whole line gets exactly `total`
// intervals, apportioned to the breakpoint intervals by their integrated
// density (largest remainders, at least one each) instead of rounding each
// interval's own count: the batched configurations name ni exactly.
std::vector<double> column_positions(const std::vector<double>& breakpoints,
                                     const std::function<double(double)>& density, int refinement,
                                     int total, double max_spacing_slope = 0);

struct BodyGridOptions {
  int nj = 20;          // least cells across on the base grid
  int refinement = 1;   // 1, 2, 4, ...
  int ni = 0;           // exact cells along the body when > 0 (refinement must be 1)
  double mach = 2;
  double gamma = 1.4;
};

// bodyGrid (src/grid/body-grid.ts:76-181). Returns "" or the error; a grid
// failing the quality gates sets *quality_error.
std::string body_grid(const Body& body, const BodyGridOptions& options, Grid* out,
                      bool* quality_error);

// bluntBodyGrid (src/grid/blunt-grid.ts:159-540): the C-topology grid of a
// blunt nose (or of a sharp one whose bow shock detaches): straight lines
// from the body, close to its smoothed normals, to an outer boundary made of
// an arc ahead of the tip and a straight line at the angle halfway between
// the normal shock and the Mach angle. iMin is the axis ahead of the tip,
// jMin the body, jMax the outer boundary, iMax the outflow plane. `ni` > 0
// asks for exactly that many columns (refinement 1). A given outer boundary
// (outer_x, outer_y: a polyline from a point on the axis outwards, y
// strictly increasing) replaces the arc and line (BluntGridOptions
// .outerBoundary, src/grid/blunt-grid.ts:42, 296-331).
struct BluntGridOptions {
  int nj = 20;
  int refinement = 1;
  int ni = 0;
  double mach = 2;
  bool gated = true;
  std::vector<double> outer_x, outer_y;
};
std::string blunt_body_grid(const Body& body, const BluntGridOptions& options, Grid* out,
                            bool* quality_error);

// The column positions of a sharp nose's fitted grid (sharpFitProblem,
// src/analysis/fitted-flow.ts:380-395): from `x0` to the end of the body,
// the breakpoints at the nose's end and the body's, spaced `aspect` times the
// geometric mean of the wall and outer cell heights of the first guess of
// the shock, the tip cone's shock line at angle `beta`; `nj` cells across
// (refined), `density` the columns' density factor.
std::vector<double> sharp_fit_columns(const Body& body, double beta, double x0, int nj, int refinement,
                                      double aspect, double density);

// The base grid's spacings of the transonic grids, in body radii
// (TRANSONIC_SPACING, src/grid/transonic-grid.ts:119-126).
struct TransonicSpacing {
  double wall = 0.05;         // cell height at the wall
  double growth = 0.2;        // e^growth: cell growth away from the body and along the axis
  double tip = 0.05;          // column spacing at the tip
  double shoulder = 0.02;     // column spacing at the shoulder (the end of the nose)
  double nose = 0.2;          // largest column spacing along the nose
  double nose_growth = 0.1;   // growth of the column spacing along the nose
};

struct TransonicGridOptions {
  int refinement = 1;
  double far_field = 100;   // far boundaries at least this many body radii out
  double cylinder = 10;     // calibers of cylinder solved behind the nose
  TransonicSpacing spacing;
  // The grid cut back or continued, node for node, to these far boundaries
  // and cylinder (0: the grid's own), for sharp noses (nestedGrid).
  bool nested = false;
  double nested_far_field = 0, nested_cylinder = 0;
};

struct TransonicGridInfo {
  int i_tip = 0, i_shoulder = 0, base_nj = 0;
  double far_radius = 0, x_upstream = 0, x_end = 0;
  bool c_topology = false;  // C grid of a blunt nose (else H)
};

// transonicGrid (src/grid/transonic-grid.ts:128-189): for sharp noses the H
// grid of a nose and a long cylinder in a domain reaching far upstream,
// sideways and downstream (jMin the axis ahead of the tip and the body,
// jMax the far radius, iMin the far boundary upstream, iMax the plane
// ending the cylinder), optionally cut back or continued to a nested domain
// (nestedGrid, :191-303); for blunt noses the C grid (bluntGrid, :319-460:
// jMin the body from the stagnation point, iMin the axis ahead of it, jMax a
// quarter circle about the stagnation point continued at the far radius).
// Cells grow geometrically away from the wall and from the tip and shoulder
// along the body; refined grids nest.
std::string transonic_grid(const Body& body, const TransonicGridOptions& options, Grid* out,
                           TransonicGridInfo* info);

// rampGrid (src/grid/shapes.ts:30-52).
std::string ramp_grid(int ni, int nj, double x_min, double x_corner, double x_max, double height,
                      double angle, Grid* out);

}  // namespace bs
