// TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.
//
// A CPU restatement of bowshock's FP64 engine, src/engine-cpu/euler2d.ts, and
// the scheme functions it calls (src/scheme/{gas,limiters,reconstruction,flux}.ts,
// src/solver/runge-kutta.ts, src/grid/structured.ts computeMetrics,
// src/analysis/forces.ts). Only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg load it, and only as the checker or the timed CPU baseline;
// the product library never links or calls it.
//
// The engine is templated on its scalar type: `double` is the oracle proper
// (the reference computes in IEEE FP64, as JavaScript numbers); `float`
// predicts the FP32 GPU field's rounding floor and is never used as a
// reference for parity.
//
// Loop orders, ghost-cell conventions and the order of floating-point
// operations follow the reference function by function; each function cites
// the lines it restates.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "bowshock.h"

namespace bso {

template <class T>
struct Prim {
  T rho, u, v, p;
};

template <class T>
struct FaceState {  // src/scheme/flux.ts:19-24
  T rho, un, ut, p;
};

// Math.min / Math.max of JavaScript: NaN if either argument is NaN.
template <class T>
inline T jmin(T a, T b) {
  if (a != a || b != b) return std::numeric_limits<T>::quiet_NaN();
  return a < b ? a : b;
}
template <class T>
inline T jmax(T a, T b) {
  if (a != a || b != b) return std::numeric_limits<T>::quiet_NaN();
  return a > b ? a : b;
}

// ---- gas law: src/scheme/gas.ts:51-66 ------------------------------------
template <class T>
inline T pressure2d(T rho, T mu, T mv, T e, T gamma) {
  return (gamma - T(1)) * (e - (T(0.5) * (mu * mu + mv * mv)) / rho);
}
template <class T>
inline T sound_speed(T rho, T p, T gamma) {
  return std::sqrt((gamma * p) / rho);
}

// ---- limiters: src/scheme/limiters.ts:24-94 --------------------------------
template <class T>
inline T limit(int limiter, T a, T b) {
  switch (limiter) {
    case BS_LIMITER_FIRST_ORDER:
      return T(0);
    case BS_LIMITER_MINMOD:  // :27-30
      if (a * b <= T(0)) return T(0);
      return std::fabs(a) < std::fabs(b) ? a : b;
    case BS_LIMITER_VAN_LEER:  // :37-40
      if (a * b <= T(0)) return T(0);
      return (T(2) * a * b) / (a + b);
    case BS_LIMITER_VAN_ALBADA: {  // :65-68, VAN_ALBADA_EPSILON :51
      const T eps = T(1e-6);
      return (a * (b * b + eps) + b * (a * a + eps)) / (a * a + b * b + T(2) * eps);
    }
    case BS_LIMITER_MONOTONIZED_CENTRAL: {  // :75-79
      if (a * b <= T(0)) return T(0);
      const T sign = a > T(0) ? T(1) : T(-1);
      return sign * jmin(jmin(T(2) * std::fabs(a), T(2) * std::fabs(b)),
                              T(0.5) * std::fabs(a + b));
    }
    default:  // BS_LIMITER_UNLIMITED_CENTRAL :85
      return T(0.5) * (a + b);
  }
}

// ---- reconstruction: src/scheme/reconstruction.ts:50-151 --------------------
template <class T>
inline Prim<T> reconstruct_per_variable(const Prim<T>& pv, const Prim<T>& c, const Prim<T>& nx,
                                        T side, int limiter) {  // :50-64
  auto value = [&](T p, T cc, T n) { return cc + T(0.5) * side * limit<T>(limiter, cc - p, n - cc); };
  return {value(pv.rho, c.rho, nx.rho), value(pv.u, c.u, nx.u), value(pv.v, c.v, nx.v),
          value(pv.p, c.p, nx.p)};
}

template <class T>
inline T van_albada_factor(T aR, T aU, T aV, T aP, T bR, T bU, T bV, T bP) {
  const T ab = aR * bR + aU * bU + aV * bV + aP * bP;
  const T aa = aR * aR + aU * aU + aV * aV + aP * aP;
  const T bb = bR * bR + bU * bU + bV * bV + bP * bP;
  const T eps = T(1e-6);
  return jmax(T(0), (T(2) * (ab + eps)) / (aa + bb + T(2) * eps));
}

template <class T>
inline T shared_factor(const Prim<T>& pv, const Prim<T>& c, const Prim<T>& n) {  // :70-84
  return van_albada_factor<T>(c.rho - pv.rho, c.u - pv.u, c.v - pv.v, c.p - pv.p, n.rho - c.rho,
                              n.u - c.u, n.v - c.v, n.p - c.p);
}

template <class T>
inline T shared_scaled_factor(const Prim<T>& pv, const Prim<T>& c, const Prim<T>& n,
                              T gamma) {  // :111-136
  const T rho = jmin(jmin(pv.rho, c.rho), n.rho);
  const T sRho = T(1) / rho;
  const T rhoA2 = gamma * jmin(jmin(pv.p, c.p), n.p);
  const T sU = std::sqrt(rho / rhoA2);
  const T sP = T(1) / rhoA2;
  return van_albada_factor<T>((c.rho - pv.rho) * sRho, (c.u - pv.u) * sU, (c.v - pv.v) * sU,
                              (c.p - pv.p) * sP, (n.rho - c.rho) * sRho, (n.u - c.u) * sU,
                              (n.v - c.v) * sU, (n.p - c.p) * sP);
}

template <class T>
inline Prim<T> reconstruct_with_factor(const Prim<T>& pv, const Prim<T>& c, const Prim<T>& n,
                                       T side, T factor) {  // :90-100, :139-151
  const T k = T(0.25) * side * factor;
  return {c.rho + k * (n.rho - pv.rho), c.u + k * (n.u - pv.u), c.v + k * (n.v - pv.v),
          c.p + k * (n.p - pv.p)};
}

template <class T>
inline Prim<T> reconstruct(int recon, int limiter, const Prim<T>& pv, const Prim<T>& c,
                           const Prim<T>& n, T side, T gamma) {
  if (recon == BS_RECON_SHARED) return reconstruct_with_factor(pv, c, n, side, shared_factor(pv, c, n));
  if (recon == BS_RECON_SHARED_SCALED)
    return reconstruct_with_factor(pv, c, n, side, shared_scaled_factor(pv, c, n, gamma));
  return reconstruct_per_variable(pv, c, n, side, limiter);
}

// ---- face fluxes: src/scheme/flux.ts ---------------------------------------
template <class T>
inline T energy_of(const FaceState<T>& w, T gamma) {  // :34-36
  return w.p / (gamma - T(1)) + T(0.5) * w.rho * (w.un * w.un + w.ut * w.ut);
}

template <class T>
inline void physical_face_flux(const FaceState<T>& w, T gamma, T* out) {  // :39-45
  const T mass = w.rho * w.un;
  out[0] = mass;
  out[1] = mass * w.un + w.p;
  out[2] = mass * w.ut;
  out[3] = w.un * (energy_of(w, gamma) + w.p);
}

template <class T>
inline void rusanov_face_flux(const FaceState<T>& l, const FaceState<T>& r, T gamma,
                              T* out) {  // :56-80
  const T sMax = jmax(std::fabs(l.un) + sound_speed(l.rho, l.p, gamma),
                           std::fabs(r.un) + sound_speed(r.rho, r.p, gamma));
  const T eL = energy_of(l, gamma), eR = energy_of(r, gamma);
  const T mL = l.rho * l.un, mR = r.rho * r.un;
  out[0] = T(0.5) * (mL + mR) - T(0.5) * sMax * (r.rho - l.rho);
  out[1] = T(0.5) * (mL * l.un + l.p + mR * r.un + r.p) - T(0.5) * sMax * (mR - mL);
  out[2] = T(0.5) * (mL * l.ut + mR * r.ut) - T(0.5) * sMax * (r.rho * r.ut - l.rho * l.ut);
  out[3] = T(0.5) * (l.un * (eL + l.p) + r.un * (eR + r.p)) - T(0.5) * sMax * (eR - eL);
}

template <class T>
inline void einfeldt_speeds(const FaceState<T>& l, const FaceState<T>& r, T gamma, T& sL,
                            T& sR) {  // :87-107
  const T aL = sound_speed(l.rho, l.p, gamma);
  const T aR = sound_speed(r.rho, r.p, gamma);
  const T wL = std::sqrt(l.rho);
  const T wR = std::sqrt(r.rho);
  const T unRoe = (wL * l.un + wR * r.un) / (wL + wR);
  const T utRoe = (wL * l.ut + wR * r.ut) / (wL + wR);
  const T hL = (energy_of(l, gamma) + l.p) / l.rho;
  const T hR = (energy_of(r, gamma) + r.p) / r.rho;
  const T hRoe = (wL * hL + wR * hR) / (wL + wR);
  const T aRoe =
      std::sqrt(jmax((gamma - T(1)) * (hRoe - T(0.5) * (unRoe * unRoe + utRoe * utRoe)), T(0)));
  sL = jmin(l.un - aL, unRoe - aRoe);
  sR = jmax(r.un + aR, unRoe + aRoe);
}

template <class T>
inline void hllc_face_flux(const FaceState<T>& l, const FaceState<T>& r, T gamma,
                           T* out) {  // :164-205
  const T energyL = energy_of(l, gamma);
  const T energyR = energy_of(r, gamma);
  T sL, sR;
  einfeldt_speeds(l, r, gamma, sL, sR);
  if (sL >= T(0)) {
    physical_face_flux(l, gamma, out);
    return;
  }
  if (sR <= T(0)) {
    physical_face_flux(r, gamma, out);
    return;
  }
  const T mL = l.rho * (sL - l.un);
  const T mR = r.rho * (sR - r.un);
  const T sStar = (r.p - l.p + l.un * mL - r.un * mR) / (mL - mR);
  const bool leftSide = sStar >= T(0);
  const FaceState<T>& s = leftSide ? l : r;
  const T sK = leftSide ? sL : sR;
  const T energyK = leftSide ? energyL : energyR;
  const T starRho = (s.rho * (sK - s.un)) / (sK - sStar);
  const T starEnergy =
      starRho * (energyK / s.rho + (sStar - s.un) * (sStar + s.p / (s.rho * (sK - s.un))));
  const T mass = s.rho * s.un;
  out[0] = mass + sK * (starRho - s.rho);
  out[1] = mass * s.un + s.p + sK * (starRho * sStar - mass);
  out[2] = mass * s.ut + sK * (starRho - s.rho) * s.ut;
  out[3] = s.un * (energyK + s.p) + sK * (starEnergy - energyK);
}

template <class T>
inline void face_flux_2d(int flux, const Prim<T>& left, const Prim<T>& right, T nx, T ny, T gamma,
                         T* out) {  // :342-366
  const FaceState<T> l{left.rho, left.u * nx + left.v * ny, -left.u * ny + left.v * nx, left.p};
  const FaceState<T> r{right.rho, right.u * nx + right.v * ny, -right.u * ny + right.v * nx,
                       right.p};
  if (flux == BS_FLUX_RUSANOV)
    rusanov_face_flux(l, r, gamma, out);
  else
    hllc_face_flux(l, r, gamma, out);
  const T normal = out[1];
  const T tangential = out[2];
  out[1] = normal * nx - tangential * ny;
  out[2] = normal * ny + tangential * nx;
}

// farFieldState: src/engine-cpu/euler2d.ts:139-165.
template <class T>
inline Prim<T> far_field_state(const Prim<T>& in, const Prim<T>& fr, T nx, T ny, T gamma) {
  const T g = T(2) / (gamma - T(1));
  const T aIn = std::sqrt((gamma * in.p) / in.rho);
  const T aFree = std::sqrt((gamma * fr.p) / fr.rho);
  const T unIn = in.u * nx + in.v * ny;
  const T unFree = fr.u * nx + fr.v * ny;
  const T plus = unIn + aIn > T(0) ? unIn + g * aIn : unFree + g * aFree;
  const T minus = unIn - aIn > T(0) ? unIn - g * aIn : unFree - g * aFree;
  const T un = T(0.5) * (plus + minus);
  const T a = (plus - minus) / (T(2) * g);
  const Prim<T>& up = unIn > T(0) ? in : fr;
  const T entropy = up.p / std::pow(up.rho, gamma);
  const T unUp = up.u * nx + up.v * ny;
  const T rho = std::pow((a * a) / (gamma * entropy), T(1) / (gamma - T(1)));
  return {rho, up.u + (un - unUp) * nx, up.v + (un - unUp) * ny, (rho * a * a) / gamma};
}

// ---- grid metrics: src/grid/structured.ts:94-168 (always in FP64) ----------
struct Metrics {
  int ni = 0, nj = 0;
  bool axisymmetric = false;
  std::vector<double> inx, iny, iarea;  // (ni + 1) nj i-faces
  std::vector<double> jnx, jny, jarea;  // ni (nj + 1) j-faces
  std::vector<double> volume, planar, cx, cy;
};

// Returns "" on success or the reference's RangeError message.
inline std::string compute_metrics(int ni, int nj, const double* x, const double* y, bool axisym,
                                   Metrics& m) {
  m.ni = ni;
  m.nj = nj;
  m.axisymmetric = axisym;
  const size_t nn = size_t(ni + 1) * size_t(nj + 1);
  if (axisym)
    for (size_t k = 0; k < nn; k++)
      if (y[k] < 0) return "axisymmetric grids must have y >= 0 (y is the radius)";
  auto node = [&](int i, int j) { return size_t(i) + size_t(j) * size_t(ni + 1); };
  auto face = [&](std::vector<double>& fx, std::vector<double>& fy, std::vector<double>& fa,
                  size_t k, size_t a, size_t b) {
    const double dx = x[b] - x[a];
    const double dy = y[b] - y[a];
    const double length = std::hypot(dx, dy);
    fx[k] = length > 0 ? dy / length : 0;
    fy[k] = length > 0 ? -dx / length : 0;
    fa[k] = axisym ? length * 0.5 * (y[a] + y[b]) : length;
  };
  const size_t nif = size_t(ni + 1) * nj, njf = size_t(ni) * (nj + 1), nc = size_t(ni) * nj;
  m.inx.assign(nif, 0);
  m.iny.assign(nif, 0);
  m.iarea.assign(nif, 0);
  m.jnx.assign(njf, 0);
  m.jny.assign(njf, 0);
  m.jarea.assign(njf, 0);
  for (int j = 0; j < nj; j++)
    for (int i = 0; i <= ni; i++)
      face(m.inx, m.iny, m.iarea, i + size_t(j) * (ni + 1), node(i, j), node(i, j + 1));
  for (int j = 0; j <= nj; j++)
    for (int i = 0; i < ni; i++)
      face(m.jnx, m.jny, m.jarea, i + size_t(j) * ni, node(i + 1, j), node(i, j));
  m.volume.assign(nc, 0);
  m.planar.assign(nc, 0);
  m.cx.assign(nc, 0);
  m.cy.assign(nc, 0);
  for (int j = 0; j < nj; j++) {
    for (int i = 0; i < ni; i++) {
      const size_t corners[4] = {node(i, j), node(i + 1, j), node(i + 1, j + 1), node(i, j + 1)};
      double area = 0, sx = 0, sy = 0;
      for (int c = 0; c < 4; c++) {
        const size_t p = corners[c], q = corners[(c + 1) % 4];
        const double cross = x[p] * y[q] - x[q] * y[p];
        area += cross;
        sx += (x[p] + x[q]) * cross;
        sy += (y[p] + y[q]) * cross;
      }
      area *= 0.5;
      if (!(area > 0))
        return "cell (" + std::to_string(i) + ", " + std::to_string(j) +
               ") has non-positive area";
      const size_t k = i + size_t(j) * ni;
      m.planar[k] = area;
      m.cx[k] = sx / (6 * area);
      m.cy[k] = sy / (6 * area);
      m.volume[k] = axisym ? area * m.cy[k] : area;
    }
  }
  return "";
}

// RUNGE_KUTTA_STAGES: src/solver/runge-kutta.ts:17-28.
inline int rk_stages(int integrator, double* a, double* b) {
  if (integrator == BS_FORWARD_EULER) {
    a[0] = 0; b[0] = 1;
    return 1;
  }
  if (integrator == BS_SSPRK2) {
    a[0] = 0; b[0] = 1;
    a[1] = 0.5; b[1] = 0.5;
    return 2;
  }
  a[0] = 0; b[0] = 1;
  a[1] = 3.0 / 4.0; b[1] = 1.0 / 4.0;
  a[2] = 1.0 / 3.0; b[2] = 2.0 / 3.0;
  return 3;
}

// validateGrid2DConfig: src/solver/config.ts:35-55.
inline std::string validate_config(const bs_config& c) {
  if (!(c.cfl > 0 && c.cfl <= 1)) return "cfl must be in (0, 1]";
  if (c.ni < 2 || c.nj < 2) return "the grid needs at least 2 x 2 cells";
  if ((c.reconstruction == BS_RECON_SHARED || c.reconstruction == BS_RECON_SHARED_SCALED) &&
      c.limiter != BS_LIMITER_VAN_ALBADA)
    return "shared reconstruction requires the 'vanAlbada' limiter";
  if ((c.boundaries[0].kind == BS_BC_PERIODIC) != (c.boundaries[1].kind == BS_BC_PERIODIC))
    return "periodic boundaries must be used on both iMin and iMax";
  if ((c.boundaries[2].kind == BS_BC_PERIODIC) != (c.boundaries[3].kind == BS_BC_PERIODIC))
    return "periodic boundaries must be used on both jMin and jMax";
  return "";
}

// ---- the engine: class Euler2D, src/engine-cpu/euler2d.ts:290-1484 ----------
template <class T>
class Engine {
 public:
  static constexpr int G = 2;  // GHOSTS, :127
  bs_config cfg{};
  Metrics m64;
  int ni = 0, nj = 0, stride = 0;
  T gamma;
  // Metrics in the engine's scalar type.
  std::vector<T> inx, iny, iarea, jnx, jny, jarea, volume, planar;
  // Padded SoA states: the solution, two stage buffers and the residual.
  struct State {
    std::vector<T> rho, mu, mv, en;
    void alloc(size_t n) {
      rho.assign(n, T(0));
      mu.assign(n, T(0));
      mv.assign(n, T(0));
      en.assign(n, T(0));
    }
  };
  State st, stage_buf[2], res;
  // 'faceStates' sides: the state outside each face, and the flux imposed
  // on each face if any (setFaceStates / setFaceFluxes, :356-398).
  std::vector<Prim<T>> face_states_[4];
  std::vector<T> face_fluxes_[4];
  std::vector<T> dt;
  int64_t steps = 0;
  double time = 0;
  // Experiment knob: round every stored state to FP32 after each update
  // (FP32 field, FP64 arithmetic). Off for the oracle proper.
  bool quantize_state = false;
  void quantize(State& u) {
    if (!quantize_state) return;
    for (size_t k = 0; k < u.rho.size(); k++) {
      u.rho[k] = T(float(u.rho[k]));
      u.mu[k] = T(float(u.mu[k]));
      u.mv[k] = T(float(u.mv[k]));
      u.en[k] = T(float(u.en[k]));
    }
  }
  std::string error;
  // LU-SGS work arrays (implicitWork, :849-861).
  std::vector<T> lamI, lamJ, diag, dq, q, pc, ac, resid;

  std::string init(const bs_config& c, const double* x, const double* y) {
    std::string e = validate_config(c);
    if (!e.empty()) return e;
    cfg = c;
    ni = c.ni;
    nj = c.nj;
    for (int side = 0; side < 4; side++) {
      face_fluxes_[side].clear();
      face_states_[side].clear();
      if (c.boundaries[side].kind == BS_BC_FACE_STATES)
        face_states_[side].assign(side < 2 ? nj : ni, Prim<T>{T(1), T(0), T(0), T(1)});
    }
    e = compute_metrics(ni, nj, x, y, c.geometry == BS_AXISYMMETRIC, m64);
    if (!e.empty()) return e;
    // The FP32 instantiation rounds gamma as the GPU engine does
    // (src/engine-gpu/euler2d-gpu.ts:129-146).
    gamma = T(c.gamma);
    auto cast = [](const std::vector<double>& v) { return std::vector<T>(v.begin(), v.end()); };
    inx = cast(m64.inx);
    iny = cast(m64.iny);
    iarea = cast(m64.iarea);
    jnx = cast(m64.jnx);
    jny = cast(m64.jny);
    jarea = cast(m64.jarea);
    volume = cast(m64.volume);
    planar = cast(m64.planar);
    stride = ni + 2 * G;
    const size_t size = size_t(stride) * (nj + 2 * G);
    st.alloc(size);
    stage_buf[0].alloc(size);
    stage_buf[1].alloc(size);
    res.alloc(size);
    dt.assign(size_t(ni) * nj, T(0));
    return "";
  }

  size_t index(int i, int j) const { return size_t(i + G) + size_t(j + G) * stride; }  // :401-403

  Prim<T> prim_at(const State& u, size_t k) const {  // :1348-1358
    const T rho = u.rho[k], mu = u.mu[k], mv = u.mv[k];
    return {rho, mu / rho, mv / rho, pressure2d(rho, mu, mv, u.en[k], gamma)};
  }

  void set_conserved_from(State& u, size_t k, const Prim<T>& w) const {
    u.rho[k] = w.rho;
    u.mu[k] = w.rho * w.u;
    u.mv[k] = w.rho * w.v;
    u.en[k] = w.p / (gamma - T(1)) + T(0.5) * w.rho * (w.u * w.u + w.v * w.v);
  }

  Prim<T> bc_state(int side) const {
    const bs_primitive& s = cfg.boundaries[side].state;
    return {T(s.rho), T(s.u), T(s.v), T(s.p)};
  }

  // setCellPrimitives (:428-445): returns false with `error` set if non-physical.
  bool set_primitives(const double* w) {
    for (int j = 0; j < nj; j++)
      for (int i = 0; i < ni; i++) {
        const double* c = w + 4 * (i + size_t(j) * ni);
        set_conserved_from(st, index(i, j), Prim<T>{T(c[0]), T(c[1]), T(c[2]), T(c[3])});
      }
    time = 0;
    steps = 0;
    return check_physical(st);
  }

  // Boundary face of a side at position t (:1430-1469).
  struct BFace {
    int i, j;
    T nx, ny, area;
    size_t n0, n1;
    int outward;
  };
  BFace boundary_face(int side, int t) const {
    if (side == BS_IMIN || side == BS_IMAX) {
      const int i = side == BS_IMIN ? 0 : ni;
      const size_t f = i + size_t(t) * (ni + 1);
      return {i, t, inx[f], iny[f], iarea[f], f, f + ni + 1, side == BS_IMIN ? -1 : 1};
    }
    const int j = side == BS_JMIN ? 0 : nj;
    const size_t f = t + size_t(j) * ni;
    const size_t node = t + size_t(j) * (ni + 1);
    return {t, j, jnx[f], jny[f], jarea[f], node, node + 1, side == BS_JMIN ? -1 : 1};
  }

  // ghostCells (:1406-1423): [ghost, mirror, periodic image].
  void ghost_cells(int side, int t, int g, size_t out[3]) const {
    switch (side) {
      case BS_IMIN:
        out[0] = index(-1 - g, t); out[1] = index(g, t); out[2] = index(ni - 1 - g, t);
        return;
      case BS_IMAX:
        out[0] = index(ni + g, t); out[1] = index(ni - 1 - g, t); out[2] = index(g, t);
        return;
      case BS_JMIN:
        out[0] = index(t, -1 - g); out[1] = index(t, g); out[2] = index(t, nj - 1 - g);
        return;
      default:
        out[0] = index(t, nj + g); out[1] = index(t, nj - 1 - g); out[2] = index(t, g);
        return;
    }
  }

  // fillGhosts (:1361-1403).
  void fill_ghosts(State& u) const {
    for (int side = 0; side < 4; side++) {
      const int kind = cfg.boundaries[side].kind;
      const int along = side < 2 ? nj : ni;
      for (int t = 0; t < along; t++) {
        const BFace bf = boundary_face(side, t);
        for (int g = 0; g < G; g++) {
          size_t gc[3];
          ghost_cells(side, t, g, gc);
          const size_t ghost = gc[0];
          const size_t source = kind == BS_BC_PERIODIC ? gc[2] : gc[1];
          if (kind == BS_BC_INFLOW || kind == BS_BC_FAR_FIELD || kind == BS_BC_FACE_STATES) {
            Prim<T> w;
            if (kind == BS_BC_INFLOW) {
              w = bc_state(side);
            } else if (kind == BS_BC_FACE_STATES) {
              w = face_states_[side][t];
            } else {
              size_t g0[3];
              ghost_cells(side, t, 0, g0);
              const Prim<T> inside = prim_at(u, g0[1]);
              w = far_field_state(inside, bc_state(side), T(bf.outward) * bf.nx,
                                  T(bf.outward) * bf.ny, gamma);
            }
            set_conserved_from(u, ghost, w);
            continue;
          }
          u.rho[ghost] = u.rho[source];
          u.en[ghost] = u.en[source];
          if (kind == BS_BC_WALL) {
            const T mn = u.mu[source] * bf.nx + u.mv[source] * bf.ny;
            u.mu[ghost] = u.mu[source] - T(2) * mn * bf.nx;
            u.mv[ghost] = u.mv[source] - T(2) * mn * bf.ny;
          } else {
            u.mu[ghost] = u.mu[source];
            u.mv[ghost] = u.mv[source];
          }
        }
      }
    }
  }

  // faceStates (:1303-1320): reconstructed states with first-order fallback.
  void face_states(const State& u, bool idir, int i, int j, Prim<T>& left, Prim<T>& right) const {
    const size_t step = idir ? 1 : size_t(stride);
    const size_t kR = index(i, j), kL = kR - step;
    const Prim<T> wLL = prim_at(u, kL - step), wL = prim_at(u, kL), wR = prim_at(u, kR),
                  wRR = prim_at(u, kR + step);
    left = reconstruct<T>(cfg.reconstruction, cfg.limiter, wLL, wL, wR, T(1), gamma);
    right = reconstruct<T>(cfg.reconstruction, cfg.limiter, wL, wR, wRR, T(-1), gamma);
    const bool ok = left.rho > 0 && left.p > 0 && right.rho > 0 && right.p > 0;
    if (!ok) {
      left = wL;
      right = wR;
    }
  }

  // wallMirrored (:1332-1346); side < 0 means an interior face.
  void wall_mirrored(int side, T nx, T ny, Prim<T>& left, Prim<T>& right) const {
    if (side < 0 || cfg.boundaries[side].kind != BS_BC_WALL) return;
    auto mirror = [&](const Prim<T>& w) {
      const T un = w.u * nx + w.v * ny;
      return Prim<T>{w.rho, w.u - T(2) * un * nx, w.v - T(2) * un * ny, w.p};
    };
    const bool minSide = side == BS_IMIN || side == BS_JMIN;
    const Prim<T> inside = minSide ? right : left;
    if (minSide) {
      left = mirror(inside);
      right = inside;
    } else {
      left = inside;
      right = mirror(inside);
    }
  }

  // computeResidual (:1208-1296).
  // The flux imposed on boundary face t of a side into f; false if none (:392-398).
  bool imposed_flux(int side, int t, T* f) const {
    if (side < 0 || face_fluxes_[side].empty()) return false;
    for (int k = 0; k < 4; k++) f[k] = face_fluxes_[side][4 * size_t(t) + k];
    return true;
  }

  void compute_residual(State& u) {
    fill_ghosts(u);
    std::fill(res.rho.begin(), res.rho.end(), T(0));
    std::fill(res.mu.begin(), res.mu.end(), T(0));
    std::fill(res.mv.begin(), res.mv.end(), T(0));
    std::fill(res.en.begin(), res.en.end(), T(0));
    T f[4];
    auto accumulate = [&](size_t kL, size_t kR, T area) {
      const T mass = f[0] * area, xm = f[1] * area, ym = f[2] * area, en = f[3] * area;
      res.rho[kL] = res.rho[kL] - mass;
      res.mu[kL] = res.mu[kL] - xm;
      res.mv[kL] = res.mv[kL] - ym;
      res.en[kL] = res.en[kL] - en;
      res.rho[kR] = res.rho[kR] + mass;
      res.mu[kR] = res.mu[kR] + xm;
      res.mv[kR] = res.mv[kR] + ym;
      res.en[kR] = res.en[kR] + en;
    };
    for (int j = 0; j < nj; j++) {
      for (int i = 0; i <= ni; i++) {
        const size_t fi = i + size_t(j) * (ni + 1);
        const int side = i == 0 ? BS_IMIN : i == ni ? BS_IMAX : -1;
        if (!imposed_flux(side, j, f)) {
          Prim<T> l, r;
          face_states(u, true, i, j, l, r);
          wall_mirrored(side, inx[fi], iny[fi], l, r);
          face_flux_2d(cfg.flux, l, r, inx[fi], iny[fi], gamma, f);
        }
        accumulate(index(i - 1, j), index(i, j), iarea[fi]);
      }
    }
    for (int j = 0; j <= nj; j++) {
      for (int i = 0; i < ni; i++) {
        const size_t fj = i + size_t(j) * ni;
        const int side = j == 0 ? BS_JMIN : j == nj ? BS_JMAX : -1;
        if (!imposed_flux(side, i, f)) {
          Prim<T> l, r;
          face_states(u, false, i, j, l, r);
          wall_mirrored(side, jnx[fj], jny[fj], l, r);
          face_flux_2d(cfg.flux, l, r, jnx[fj], jny[fj], gamma, f);
        }
        accumulate(index(i, j - 1), index(i, j), jarea[fj]);
      }
    }
    if (cfg.geometry == BS_AXISYMMETRIC) {
      for (int j = 0; j < nj; j++)
        for (int i = 0; i < ni; i++) {
          const size_t k = index(i, j);
          const T p = pressure2d(u.rho[k], u.mu[k], u.mv[k], u.en[k], gamma);
          res.mv[k] = res.mv[k] + p * planar[i + size_t(j) * ni];
        }
    }
  }

  // computeTimeSteps (:1183-1205).
  void compute_time_steps(double limitT) {
    T smallest = std::numeric_limits<T>::infinity();
    const T cfl = T(cfg.cfl);
    for (int j = 0; j < nj; j++) {
      for (int i = 0; i < ni; i++) {
        const Prim<T> w = prim_at(st, index(i, j));
        const T a = sound_speed(w.rho, w.p, gamma);
        auto sr = [&](const std::vector<T>& fx, const std::vector<T>& fy, const std::vector<T>& fa,
                      size_t f0, size_t f1) {
          const T sx = T(0.5) * (fx[f0] * fa[f0] + fx[f1] * fa[f1]);
          const T sy = T(0.5) * (fy[f0] * fa[f0] + fy[f1] * fa[f1]);
          return std::fabs(w.u * sx + w.v * sy) + a * std::hypot(sx, sy);
        };
        const size_t fi = i + size_t(j) * (ni + 1);
        const size_t fj = i + size_t(j) * ni;
        const T lambda = sr(inx, iny, iarea, fi, fi + 1) + sr(jnx, jny, jarea, fj, fj + ni);
        const T d = (cfl * volume[fj]) / lambda;
        dt[fj] = d;
        smallest = jmin(smallest, d);
      }
    }
    if (cfg.time_stepping == BS_TIME_GLOBAL) {
      const T v = jmin(smallest, T(limitT));
      std::fill(dt.begin(), dt.end(), v);
    }
  }

  // stage (:1160-1175): out = a u0 + b (src + dt/V R(src)).
  void stage(State& u0, State& src, T a, T b, State& out) {
    compute_residual(src);
    for (int j = 0; j < nj; j++)
      for (int i = 0; i < ni; i++) {
        const size_t k = index(i, j);
        const size_t c = i + size_t(j) * ni;
        const T factor = dt[c] / volume[c];
        out.rho[k] = a * u0.rho[k] + b * (src.rho[k] + factor * res.rho[k]);
        out.mu[k] = a * u0.mu[k] + b * (src.mu[k] + factor * res.mu[k]);
        out.mv[k] = a * u0.mv[k] + b * (src.mv[k] + factor * res.mv[k]);
        out.en[k] = a * u0.en[k] + b * (src.en[k] + factor * res.en[k]);
      }
  }

  // step (:1146-1157).
  bool step() {
    double a[3], b[3];
    const int n = rk_stages(cfg.integrator, a, b);
    State* previous = &st;
    for (int s = 0; s < n; s++) {
      State* out = s == n - 1 ? &st : &stage_buf[s % 2];
      stage(st, *previous, T(a[s]), T(b[s]), *out);
      quantize(*out);
      previous = out;
    }
    steps += 1;
    return check_physical(st);
  }

  // iterate (:554-560).
  bool iterate(int count) {
    for (int n = 0; n < count; n++) {
      compute_time_steps(std::numeric_limits<double>::infinity());
      if (cfg.time_stepping == BS_TIME_GLOBAL) time += double(dt[0]);
      if (!step()) return false;
    }
    return true;
  }

  // densityResidualNorm (:480-491).
  double density_residual_norm() {
    compute_residual(st);
    double sum = 0;
    for (int j = 0; j < nj; j++)
      for (int i = 0; i < ni; i++) {
        const T r = res.rho[index(i, j)] / volume[i + size_t(j) * ni];
        sum += double(r) * double(r);
      }
    return std::sqrt(sum / (double(ni) * nj));
  }

  void residual_vector(double* out) {  // residualVector (:456-472)
    compute_residual(st);
    for (int j = 0; j < nj; j++)
      for (int i = 0; i < ni; i++) {
        const size_t k = index(i, j), c = 4 * (i + size_t(j) * ni);
        out[c] = res.rho[k];
        out[c + 1] = res.mu[k];
        out[c + 2] = res.mv[k];
        out[c + 3] = res.en[k];
      }
  }

  // boundaryFluxes (:499-525).
  void boundary_fluxes(int side, const double* x, const double* y, bs_face_flux* out) {
    fill_ghosts(st);
    const bool idir = side < 2;
    const int along = idir ? nj : ni;
    T f[4];
    for (int t = 0; t < along; t++) {
      const BFace bf = boundary_face(side, t);
      Prim<T> l, r;
      face_states(st, idir, bf.i, bf.j, l, r);
      wall_mirrored(side, bf.nx, bf.ny, l, r);
      face_flux_2d(cfg.flux, l, r, bf.nx, bf.ny, gamma, f);
      bs_face_flux& o = out[t];
      o.x = 0.5 * (x[bf.n0] + x[bf.n1]);
      o.y = 0.5 * (y[bf.n0] + y[bf.n1]);
      o.nx = double(bf.outward * bf.nx);
      o.ny = double(bf.outward * bf.ny);
      o.area = double(bf.area);
      for (int k = 0; k < 4; k++) o.flux[k] = double(bf.outward * f[k]);
    }
  }

  // checkPhysical (:1471-1483).
  bool check_physical(const State& u) {
    for (int j = 0; j < nj; j++)
      for (int i = 0; i < ni; i++) {
        const Prim<T> w = prim_at(u, index(i, j));
        if (!(w.rho > 0 && w.p > 0 && std::isfinite(double(w.u)) && std::isfinite(double(w.v)))) {
          error = "non-physical state in cell (" + std::to_string(i) + ", " + std::to_string(j) +
                  ") after step " + std::to_string(steps);
          return false;
        }
      }
    return true;
  }

  // implicitCorrection with LU-SGS sweeps (:878-1105), leaving dQ in `dq`.
  void implicit_correction(T cfl, T omega) {
    compute_residual(st);
    const size_t n = size_t(ni) * nj;
    if (dq.size() != 4 * n) {
      lamI.assign(size_t(ni + 1) * nj, T(0));
      lamJ.assign(size_t(ni) * (nj + 1), T(0));
      diag.assign(n, T(0));
      dq.assign(4 * n, T(0));
      q.assign(4 * n, T(0));
      pc.assign(n, T(0));
      ac.assign(n, T(0));
      resid.assign(4 * n, T(0));
    }
    for (int j = 0; j < nj; j++)
      for (int i = 0; i < ni; i++) {
        const size_t k = index(i, j), c = i + size_t(j) * ni;
        const T rho = st.rho[k], mx = st.mu[k], my = st.mv[k], e = st.en[k];
        q[4 * c] = rho;
        q[4 * c + 1] = mx;
        q[4 * c + 2] = my;
        q[4 * c + 3] = e;
        const T p = (gamma - T(1)) * (e - (T(0.5) * (mx * mx + my * my)) / rho);
        pc[c] = p;
        ac[c] = std::sqrt((gamma * p) / rho);
        resid[4 * c] = res.rho[k];
        resid[4 * c + 1] = res.mu[k];
        resid[4 * c + 2] = res.mv[k];
        resid[4 * c + 3] = res.en[k];
      }
    auto radius = [&](size_t c, T nx, T ny) {
      return std::fabs((q[4 * c + 1] * nx + q[4 * c + 2] * ny) / q[4 * c]) + ac[c];
    };
    for (int j = 0; j < nj; j++)
      for (int i = 0; i <= ni; i++) {
        const size_t f = i + size_t(j) * (ni + 1);
        const size_t c = i + size_t(j) * ni;
        const T l = i > 0 ? radius(c - 1, inx[f], iny[f]) : T(0);
        const T r = i < ni ? radius(c, inx[f], iny[f]) : T(0);
        lamI[f] = jmax(l, r) * iarea[f];
      }
    for (int j = 0; j <= nj; j++)
      for (int i = 0; i < ni; i++) {
        const size_t f = i + size_t(j) * ni;
        const T below = j > 0 ? radius(f - ni, jnx[f], jny[f]) : T(0);
        const T above = j < nj ? radius(f, jnx[f], jny[f]) : T(0);
        lamJ[f] = jmax(below, above) * jarea[f];
      }
    const T scale = T(0.5) * (omega + T(1) / cfl);
    const bool axisym = cfg.geometry == BS_AXISYMMETRIC;
    for (int j = 0; j < nj; j++)
      for (int i = 0; i < ni; i++) {
        const size_t fi = i + size_t(j) * (ni + 1), fj = i + size_t(j) * ni;
        diag[fj] = scale * (lamI[fi] + lamI[fi + 1] + lamJ[fj] + lamJ[fj + ni]) +
                   (axisym ? planar[fj] * radius(fj, T(0), T(1)) : T(0));
      }
    T sum[4];
    auto neighbour = [&](size_t c, T nx, T ny, T area, T lambdaA) {  // :977-1005
      const size_t b = 4 * c;
      const T rho = q[b], mx = q[b + 1], my = q[b + 2], e = q[b + 3];
      const T d0 = dq[b], d1 = dq[b + 1], d2 = dq[b + 2], d3 = dq[b + 3];
      const T p0 = pc[c];
      const T un0 = (mx * nx + my * ny) / rho;
      const T rho1 = rho + d0, mx1 = mx + d1, my1 = my + d2, e1 = e + d3;
      const T p1 = (gamma - T(1)) * (e1 - (T(0.5) * (mx1 * mx1 + my1 * my1)) / rho1);
      const T un1 = (mx1 * nx + my1 * ny) / rho1;
      const T half = T(0.5) * area;
      const T damp = T(0.5) * omega * lambdaA;
      sum[0] = sum[0] + half * (rho1 * un1 - rho * un0) - damp * d0;
      sum[1] = sum[1] + half * (mx1 * un1 + p1 * nx - (mx * un0 + p0 * nx)) - damp * d1;
      sum[2] = sum[2] + half * (my1 * un1 + p1 * ny - (my * un0 + p0 * ny)) - damp * d2;
      sum[3] = sum[3] + half * ((e1 + p1) * un1 - (e + p0) * un0) - damp * d3;
    };
    for (int j = 0; j < nj; j++)  // forward sweep :1058-1079
      for (int i = 0; i < ni; i++) {
        const size_t c = i + size_t(j) * ni;
        sum[0] = sum[1] = sum[2] = sum[3] = T(0);
        if (i > 0) {
          const size_t f = i + size_t(j) * (ni + 1);
          neighbour(c - 1, -inx[f], -iny[f], iarea[f], lamI[f]);
        }
        if (j > 0) neighbour(c - ni, -jnx[c], -jny[c], jarea[c], lamJ[c]);
        const T d = diag[c];
        for (int v = 0; v < 4; v++) dq[4 * c + v] = (resid[4 * c + v] - sum[v]) / d;
      }
    for (int j = nj - 1; j >= 0; j--)  // backward sweep :1080-1102
      for (int i = ni - 1; i >= 0; i--) {
        const size_t c = i + size_t(j) * ni;
        sum[0] = sum[1] = sum[2] = sum[3] = T(0);
        if (i < ni - 1) {
          const size_t f = i + 1 + size_t(j) * (ni + 1);
          neighbour(c + 1, inx[f], iny[f], iarea[f], lamI[f]);
        }
        if (j < nj - 1) {
          const size_t f = c + ni;
          neighbour(c + ni, jnx[f], jny[f], jarea[f], lamJ[f]);
        }
        const T d = diag[c];
        for (int v = 0; v < 4; v++) dq[4 * c + v] = dq[4 * c + v] - sum[v] / d;
      }
  }

  // applyImplicitUpdate (:816-847).
  bool apply_implicit_update() {
    for (int j = 0; j < nj; j++)
      for (int i = 0; i < ni; i++) {
        const size_t c = i + size_t(j) * ni, k = index(i, j);
        const T rho = st.rho[k], mx = st.mu[k], my = st.mv[k], e = st.en[k];
        const T p = (gamma - T(1)) * (e - (T(0.5) * (mx * mx + my * my)) / rho);
        T alpha = T(1);
        for (int tries = 0; tries < 30; tries++) {
          const T rho1 = rho + alpha * dq[4 * c];
          const T mx1 = mx + alpha * dq[4 * c + 1];
          const T my1 = my + alpha * dq[4 * c + 2];
          const T e1 = e + alpha * dq[4 * c + 3];
          const T p1 = (gamma - T(1)) * (e1 - (T(0.5) * (mx1 * mx1 + my1 * my1)) / rho1);
          if (rho1 > T(0.5) * rho && rho1 < T(2) * rho && p1 > T(0.5) * p && p1 < T(2) * p) break;
          alpha *= T(0.5);
        }
        st.rho[k] = rho + alpha * dq[4 * c];
        st.mu[k] = mx + alpha * dq[4 * c + 1];
        st.mv[k] = my + alpha * dq[4 * c + 2];
        st.en[k] = e + alpha * dq[4 * c + 3];
      }
    quantize(st);
    steps += 1;
    return check_physical(st);
  }

  // iterateImplicit (:581-589) with LU-SGS sweeps.
  bool iterate_implicit(int count, double cfl, double omega) {
    for (int n = 0; n < count; n++) {
      implicit_correction(T(cfl), T(omega));
      if (!apply_implicit_update()) return false;
    }
    return true;
  }
};

// forebodyPressureDrag: src/analysis/forces.ts:19-30.
inline double forebody_pressure_drag(const bs_face_flux* wall, int n, double p_inf, double q_inf,
                                     double base_radius) {
  double force = 0;
  for (int t = 0; t < n; t++) force += (wall[t].flux[1] - p_inf * wall[t].nx) * wall[t].area;
  return (2 * force) / (q_inf * base_radius * base_radius);
}

}  // namespace bso
