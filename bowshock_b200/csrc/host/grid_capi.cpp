// C ABI of the host-side grid generator and exact solutions.
#include <cmath>
#include <cstring>
#include <new>

#include "../common.hpp"
#include "bowshock.h"
#include "gasdyn.hpp"
#include "geometry.hpp"
#include "grids.hpp"

struct bs_grid {
  bs::Grid g;
  bool transonic = false;
  bs::TransonicGridInfo info;
};

namespace {

bs::Body to_body(const bs_body& b) {
  bs::Body body;
  body.nose.kind = b.nose_kind;
  body.nose.parameter = b.parameter;
  body.nose.length = b.nose_length;
  body.nose.base_radius = b.base_radius;
  body.cylinder_length = b.cylinder_length;
  return body;
}

}  // namespace

extern "C" {

bs_status bs_body_grid(const bs_body* body, const bs_body_grid_options* options, bs_grid** out) {
  if (body == nullptr || options == nullptr || out == nullptr)
    return bs::fail(BS_INVALID_ARGUMENT, "null argument");
  bs::BodyGridOptions o;
  o.nj = options->nj;
  o.refinement = options->refinement <= 0 ? 1 : options->refinement;
  o.ni = options->ni;
  o.mach = options->mach;
  o.gamma = options->gamma;
  auto* g = new (std::nothrow) bs_grid;
  if (g == nullptr) return bs::fail(BS_MEMORY_LIMIT, "out of host memory");
  bool quality = false;
  const std::string e = bs::body_grid(to_body(*body), o, &g->g, &quality);
  if (!e.empty()) {
    delete g;
    return bs::fail(quality ? BS_GRID_QUALITY : BS_INVALID_ARGUMENT, e);
  }
  *out = g;
  return bs::ok();
}

bs_status bs_blunt_body_grid(const bs_body* body, const bs_body_grid_options* options,
                             bs_grid** out) {
  return bs_blunt_body_grid_bounded(body, options, nullptr, nullptr, 0, out);
}

bs_status bs_blunt_body_grid_bounded(const bs_body* body, const bs_body_grid_options* options,
                                     const double* outer_x, const double* outer_y, int32_t n_outer,
                                     bs_grid** out) {
  if (body == nullptr || options == nullptr || out == nullptr)
    return bs::fail(BS_INVALID_ARGUMENT, "null argument");
  if (n_outer < 0 || (n_outer > 0 && (outer_x == nullptr || outer_y == nullptr)))
    return bs::fail(BS_INVALID_ARGUMENT, "the outer boundary's points are missing");
  if (n_outer == 1)
    return bs::fail(BS_INVALID_ARGUMENT, "the outer boundary needs at least two points, the first on the axis");
  bs::BluntGridOptions o;
  o.nj = options->nj;
  o.refinement = options->refinement <= 0 ? 1 : options->refinement;
  o.ni = options->ni;
  o.mach = options->mach;
  o.gated = (options->flags & BS_GRID_UNGATED) == 0;
  if (n_outer > 0) {
    o.outer_x.assign(outer_x, outer_x + n_outer);
    o.outer_y.assign(outer_y, outer_y + n_outer);
  }
  auto* g = new (std::nothrow) bs_grid;
  if (g == nullptr) return bs::fail(BS_MEMORY_LIMIT, "out of host memory");
  bool quality = false;
  const std::string e = bs::blunt_body_grid(to_body(*body), o, &g->g, &quality);
  if (!e.empty()) {
    delete g;
    return bs::fail(quality ? BS_GRID_QUALITY : BS_INVALID_ARGUMENT, e);
  }
  *out = g;
  return bs::ok();
}

bs_status bs_ramp_grid(int32_t ni, int32_t nj, double x_min, double x_corner, double x_max,
                       double height, double angle, bs_grid** out) {
  if (out == nullptr || ni < 1 || nj < 1) return bs::fail(BS_INVALID_ARGUMENT, "invalid argument");
  auto* g = new (std::nothrow) bs_grid;
  if (g == nullptr) return bs::fail(BS_MEMORY_LIMIT, "out of host memory");
  const std::string e = bs::ramp_grid(ni, nj, x_min, x_corner, x_max, height, angle, &g->g);
  if (!e.empty()) {
    delete g;
    return bs::fail(BS_INVALID_ARGUMENT, e);
  }
  *out = g;
  return bs::ok();
}

bs_status bs_grid_dims(const bs_grid* grid, int32_t* ni, int32_t* nj) {
  if (grid == nullptr || ni == nullptr || nj == nullptr)
    return bs::fail(BS_INVALID_ARGUMENT, "null argument");
  *ni = grid->g.ni;
  *nj = grid->g.nj;
  return bs::ok();
}

bs_status bs_grid_nodes(const bs_grid* grid, double* x, double* y) {
  if (grid == nullptr || x == nullptr || y == nullptr)
    return bs::fail(BS_INVALID_ARGUMENT, "null argument");
  std::memcpy(x, grid->g.x.data(), grid->g.x.size() * sizeof(double));
  std::memcpy(y, grid->g.y.data(), grid->g.y.size() * sizeof(double));
  return bs::ok();
}

bs_status bs_grid_info(const bs_grid* grid, int32_t* i_tip, double* outer_angle) {
  if (grid == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
  if (i_tip) *i_tip = grid->g.i_tip;
  if (outer_angle) *outer_angle = grid->g.outer_angle;
  return bs::ok();
}

bs_status bs_transonic_grid(const bs_body* body, const bs_transonic_grid_options* options, bs_grid** out) {
  if (body == nullptr || options == nullptr || out == nullptr)
    return bs::fail(BS_INVALID_ARGUMENT, "null argument");
  bs::TransonicGridOptions o;
  o.refinement = options->refinement;
  o.far_field = options->far_field;
  o.cylinder = options->cylinder;
  o.nested = options->nested != 0;
  o.nested_far_field = options->nested_far_field;
  o.nested_cylinder = options->nested_cylinder;
  if (!(std::isfinite(o.nested_far_field) && std::isfinite(o.nested_cylinder) && o.nested_far_field >= 0 &&
        o.nested_cylinder >= 0))
    return bs::fail(BS_INVALID_ARGUMENT, "the nested domain's far field and cylinder must be 0 or positive");
  // A spacing of 0 takes the default.
  const double given[6] = {options->wall, options->growth, options->tip, options->shoulder, options->nose,
                           options->nose_growth};
  double* fields[6] = {&o.spacing.wall, &o.spacing.growth, &o.spacing.tip, &o.spacing.shoulder,
                       &o.spacing.nose, &o.spacing.nose_growth};
  for (int k = 0; k < 6; k++)
    if (given[k] != 0) *fields[k] = given[k];
  auto* g = new (std::nothrow) bs_grid;
  if (g == nullptr) return bs::fail(BS_MEMORY_LIMIT, "out of host memory");
  const std::string e = bs::transonic_grid(to_body(*body), o, &g->g, &g->info);
  if (!e.empty()) {
    delete g;
    return bs::fail(BS_INVALID_ARGUMENT, e);
  }
  g->transonic = true;
  *out = g;
  return bs::ok();
}

bs_status bs_grid_transonic_info(const bs_grid* grid, int32_t* i_shoulder, int32_t* base_nj, double* far_radius,
                                 double* x_upstream, double* x_end, int32_t* c_topology) {
  if (grid == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
  if (!grid->transonic) return bs::fail(BS_INVALID_ARGUMENT, "not a transonic grid");
  if (i_shoulder) *i_shoulder = grid->info.i_shoulder;
  if (base_nj) *base_nj = grid->info.base_nj;
  if (far_radius) *far_radius = grid->info.far_radius;
  if (x_upstream) *x_upstream = grid->info.x_upstream;
  if (x_end) *x_end = grid->info.x_end;
  if (c_topology) *c_topology = grid->info.c_topology ? 1 : 0;
  return bs::ok();
}

bs_status bs_grid_two_scale(const bs_grid* grid, int32_t* two_scale) {
  if (grid == nullptr || two_scale == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
  *two_scale = grid->g.two_scale ? 1 : 0;
  return bs::ok();
}

bs_status bs_grid_destroy(bs_grid* grid) {
  delete grid;
  return bs::ok();
}

bs_status bs_grid_quality_of(int32_t ni, int32_t nj, const double* x, const double* y,
                             bs_grid_quality* out) {
  if (x == nullptr || y == nullptr || out == nullptr || ni < 1 || nj < 1)
    return bs::fail(BS_INVALID_ARGUMENT, "invalid argument");
  const bs::GridQuality q = bs::grid_quality(ni, nj, x, y);
  out->min_angle = q.min_angle;
  out->min_wall_angle = q.min_wall_angle;
  out->max_size_ratio = q.max_size_ratio;
  out->max_aspect_ratio = q.max_aspect_ratio;
  out->min_area = q.min_area;
  return bs::ok();
}

bs_status bs_taylor_maccoll(double mach, double cone_angle, double gamma, double tolerance,
                            bs_cone_flow* out) {
  if (out == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
  bs::ConeFlow f;
  const std::string e =
      bs::taylor_maccoll(mach, cone_angle, gamma, tolerance > 0 ? tolerance : 1e-13, &f);
  if (!e.empty()) return bs::fail(BS_INVALID_ARGUMENT, e);
  out->shock_angle = f.shock_angle;
  out->post_shock_mach = f.post_shock_mach;
  out->post_shock_pressure_ratio = f.post_shock_pressure_ratio;
  out->surface_mach = f.surface_mach;
  out->surface_pressure_ratio = f.surface_pressure_ratio;
  out->surface_pressure_coefficient = f.surface_pressure_coefficient;
  return bs::ok();
}

bs_status bs_oblique_shock(double mach, double theta, double gamma, bs_shock* out) {
  if (out == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
  bs::ObliqueShock s;
  const std::string e = bs::oblique_shock(mach, theta, gamma, &s);
  if (!e.empty()) return bs::fail(BS_INVALID_ARGUMENT, e);
  out->beta = s.beta;
  out->pressure_ratio = s.pressure_ratio;
  out->density_ratio = s.density_ratio;
  out->downstream_mach = s.downstream_mach;
  return bs::ok();
}

bs_status bs_normal_shock(double mach, double gamma, bs_shock* out) {
  if (out == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
  bs::NormalShock s;
  const std::string e = bs::normal_shock(mach, gamma, &s);
  if (!e.empty()) return bs::fail(BS_INVALID_ARGUMENT, e);
  out->beta = M_PI / 2;
  out->pressure_ratio = s.pressure_ratio;
  out->density_ratio = s.density_ratio;
  out->downstream_mach = s.downstream_mach;
  return bs::ok();
}

bs_status bs_cone_flow_field(double mach, double cone_angle, double gamma, double tolerance, int32_t n,
                             const double* polar, double* speed, double* flow_angle, bs_cone_flow* flow) {
  if (n < 0 || (n > 0 && (polar == nullptr || speed == nullptr || flow_angle == nullptr)))
    return bs::fail(BS_INVALID_ARGUMENT, "null argument");
  bs::ConeField f;
  std::string e = bs::cone_flow_field(mach, cone_angle, gamma, tolerance > 0 ? tolerance : 1e-13, &f);
  if (!e.empty()) return bs::fail(BS_INVALID_ARGUMENT, e);
  for (int32_t k = 0; k < n; k++) {
    e = f.at(polar[k], &speed[k], &flow_angle[k]);
    if (!e.empty()) return bs::fail(BS_INVALID_ARGUMENT, e);
  }
  if (flow != nullptr) {
    flow->shock_angle = f.flow.shock_angle;
    flow->post_shock_mach = f.flow.post_shock_mach;
    flow->post_shock_pressure_ratio = f.flow.post_shock_pressure_ratio;
    flow->surface_mach = f.flow.surface_mach;
    flow->surface_pressure_ratio = f.flow.surface_pressure_ratio;
    flow->surface_pressure_coefficient = f.flow.surface_pressure_coefficient;
  }
  return bs::ok();
}

static void to_fitted(const bs::ShockState& s, bs_fitted_shock* out) {
  out->state.rho = s.w[0];
  out->state.u = s.w[1];
  out->state.v = s.w[2];
  out->state.p = s.w[3];
  out->speed = s.speed;
  out->normal_velocity = s.normal_velocity;
  out->mach = s.mach;
}

bs_status bs_shock_state(const bs_primitive* free, double gamma, double mach, double nx, double ny,
                         bs_fitted_shock* out) {
  if (free == nullptr || out == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
  if (!(mach >= 1)) return bs::fail(BS_INVALID_ARGUMENT, "a shock needs a relative Mach number of at least 1");
  const double f[4] = {free->rho, free->u, free->v, free->p};
  to_fitted(bs::shock_state(f, gamma, mach, nx, ny), out);
  return bs::ok();
}

bs_status bs_compatible_shock(const bs_primitive* free, double gamma, double nx, double ny, double rho, double a,
                              double p, double un, bs_fitted_shock* out) {
  if (free == nullptr || out == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
  if (!(rho > 0 && a > 0)) return bs::fail(BS_INVALID_ARGUMENT, "the flow behind needs rho > 0 and a > 0");
  const double f[4] = {free->rho, free->u, free->v, free->p};
  to_fitted(bs::compatible_shock(f, gamma, nx, ny, rho, a, p, un), out);
  return bs::ok();
}

bs_status bs_column_positions(int32_t n_breakpoints, const double* breakpoints, bs_density_fn density, void* user,
                              int32_t refinement, int32_t total, int32_t capacity, double* out, int32_t* n_out) {
  if (n_breakpoints < 2 || breakpoints == nullptr || density == nullptr || out == nullptr || n_out == nullptr)
    return bs::fail(BS_INVALID_ARGUMENT, "column positions need two breakpoints, a density and an output");
  if (!(refinement >= 1)) return bs::fail(BS_INVALID_ARGUMENT, "the refinement must be at least 1");
  const std::vector<double> bp(breakpoints, breakpoints + n_breakpoints);
  const std::vector<double> xs =
      bs::column_positions(bp, [&](double x) { return density(x, user); }, refinement, total);
  if (int64_t(xs.size()) > capacity) return bs::fail(BS_INVALID_ARGUMENT, "more positions than the output holds");
  for (size_t k = 0; k < xs.size(); k++) out[k] = xs[k];
  *n_out = int32_t(xs.size());
  return bs::ok();
}

bs_status bs_body_radius(const bs_body* body, int32_t n, const double* x, double* r) {
  if (body == nullptr || n < 0 || (n > 0 && (x == nullptr || r == nullptr)))
    return bs::fail(BS_INVALID_ARGUMENT, "null argument");
  const bs::Body b = to_body(*body);
  const std::string e = bs::validate_body(b);
  if (!e.empty()) return bs::fail(BS_INVALID_ARGUMENT, e);
  for (int32_t k = 0; k < n; k++) r[k] = bs::body_radius(b, x[k]);
  return bs::ok();
}

bs_status bs_nose_slopes(const bs_body* body, double* tip, double* base) {
  if (body == nullptr || tip == nullptr || base == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
  const bs::Body b = to_body(*body);
  const std::string e = bs::validate_body(b);
  if (!e.empty()) return bs::fail(BS_INVALID_ARGUMENT, e);
  *tip = bs::nose_tip_slope(b.nose);
  *base = bs::nose_base_slope(b.nose);
  return bs::ok();
}

bs_status bs_sharp_fit_columns(const bs_body* body, double beta, double x0, int32_t nj, int32_t refinement,
                               double aspect, double density, int32_t capacity, double* out, int32_t* n_out) {
  if (body == nullptr || out == nullptr || n_out == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
  if (!(nj >= 2 && refinement >= 1 && beta > 0 && beta < M_PI / 2 && x0 > 0 && aspect > 0 && density > 0))
    return bs::fail(BS_INVALID_ARGUMENT, "sharp fitted columns need nj >= 2, refinement >= 1, 0 < beta < pi/2");
  const bs::Body b = to_body(*body);
  const std::string e = bs::validate_body(b);
  if (!e.empty()) return bs::fail(BS_INVALID_ARGUMENT, e);
  if (!(x0 < b.nose.length)) return bs::fail(BS_INVALID_ARGUMENT, "the domain must start on the nose");
  const std::vector<double> xs = bs::sharp_fit_columns(b, beta, x0, nj, refinement, aspect, density);
  if (int64_t(xs.size()) > capacity) return bs::fail(BS_INVALID_ARGUMENT, "more positions than the output holds");
  for (size_t k = 0; k < xs.size(); k++) out[k] = xs[k];
  *n_out = int32_t(xs.size());
  return bs::ok();
}

}  // extern "C"
