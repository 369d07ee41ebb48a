// TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.
//
// C entry points of the FP64 CPU oracle (a restatement of
// src/engine-cpu/euler2d.ts, in euler2d_oracle.hpp), for the tests' ctypes
// harness and the CPU baseline. `precision` 64 is the oracle proper; 32 runs
// the same code in FP32 to predict the GPU field's rounding floor.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "euler2d_oracle.hpp"

namespace {
thread_local std::string g_error;

struct Handle {
  int precision = 64;
  std::unique_ptr<bso::Engine<double>> d;
  std::unique_ptr<bso::Engine<float>> f;
  std::vector<double> x, y;
};

template <class F>
int with_engine(void* h, F&& fn) {
  if (h == nullptr) {
    g_error = "null oracle handle";
    return BS_INVALID_ARGUMENT;
  }
  Handle* e = static_cast<Handle*>(h);
  if (e->precision == 64) return fn(*e->d);
  return fn(*e->f);
}
}  // namespace

extern "C" {

const char* bso_last_error(void) { return g_error.c_str(); }

int bso_create(const bs_config* config, const double* x, const double* y, int precision,
               void** out) {
  if (config == nullptr || x == nullptr || y == nullptr || out == nullptr ||
      (precision != 32 && precision != 64)) {
    g_error = "invalid argument";
    return BS_INVALID_ARGUMENT;
  }
  auto h = std::make_unique<Handle>();
  h->precision = precision;
  const size_t nn = size_t(config->ni + 1) * size_t(config->nj + 1);
  if (config->ni < 1 || config->nj < 1) {
    g_error = "the grid needs at least 2 x 2 cells";
    return BS_INVALID_ARGUMENT;
  }
  h->x.assign(x, x + nn);
  h->y.assign(y, y + nn);
  std::string e;
  if (precision == 64) {
    h->d = std::make_unique<bso::Engine<double>>();
    e = h->d->init(*config, x, y);
  } else {
    h->f = std::make_unique<bso::Engine<float>>();
    e = h->f->init(*config, x, y);
  }
  if (!e.empty()) {
    g_error = e;
    return BS_INVALID_ARGUMENT;
  }
  *out = h.release();
  return BS_OK;
}

void bso_destroy(void* h) { delete static_cast<Handle*>(h); }

// Experiment knob of the FP64 engine: round the stored state to FP32 after
// every update (FP32 storage with FP64 arithmetic).
int bso_set_quantize(void* h, int on) {
  Handle* e = static_cast<Handle*>(h);
  if (e == nullptr || e->precision != 64) return BS_INVALID_ARGUMENT;
  e->d->quantize_state = on != 0;
  return BS_OK;
}

int bso_centroids(void* h, double* cx, double* cy) {
  return with_engine(h, [&](auto& e) {
    std::copy(e.m64.cx.begin(), e.m64.cx.end(), cx);
    std::copy(e.m64.cy.begin(), e.m64.cy.end(), cy);
    return BS_OK;
  });
}

int bso_metrics(void* h, double* iface /*3 (ni+1) nj*/, double* jface /*3 ni (nj+1)*/,
                double* cells /*4 ni nj: volume, planar, cx, cy*/) {
  return with_engine(h, [&](auto& e) {
    const auto& m = e.m64;
    for (size_t k = 0; k < m.inx.size(); k++) {
      iface[3 * k] = m.inx[k];
      iface[3 * k + 1] = m.iny[k];
      iface[3 * k + 2] = m.iarea[k];
    }
    for (size_t k = 0; k < m.jnx.size(); k++) {
      jface[3 * k] = m.jnx[k];
      jface[3 * k + 1] = m.jny[k];
      jface[3 * k + 2] = m.jarea[k];
    }
    for (size_t k = 0; k < m.volume.size(); k++) {
      cells[4 * k] = m.volume[k];
      cells[4 * k + 1] = m.planar[k];
      cells[4 * k + 2] = m.cx[k];
      cells[4 * k + 3] = m.cy[k];
    }
    return BS_OK;
  });
}

int bso_set_primitives(void* h, const double* w) {
  return with_engine(h, [&](auto& e) {
    if (!e.set_primitives(w)) {
      g_error = e.error;
      return BS_NON_PHYSICAL;
    }
    return BS_OK;
  });
}

// Set the conserved state directly (four values per cell), e.g. the FP32
// state read back from the GPU, without counting a step.
int bso_set_conserved(void* h, const double* q) {
  return with_engine(h, [&](auto& e) {
    for (int j = 0; j < e.nj; j++)
      for (int i = 0; i < e.ni; i++) {
        const size_t k = e.index(i, j);
        const double* c = q + 4 * (i + size_t(j) * e.ni);
        e.st.rho[k] = c[0];
        e.st.mu[k] = c[1];
        e.st.mv[k] = c[2];
        e.st.en[k] = c[3];
      }
    return BS_OK;
  });
}

// setFaceStates / setFaceFluxes (src/engine-cpu/euler2d.ts:356-390) for a
// 'faceStates' side: primitives (4 per face), and fluxes per unit area (4
// per face) or null to go back to the Riemann flux.
int bso_set_face_states(void* h, int side, const double* prim) {
  return with_engine(h, [&](auto& e) {
    using T = decltype(e.gamma);
    if (side < 0 || side > 3 || e.cfg.boundaries[side].kind != BS_BC_FACE_STATES) {
      g_error = "the side does not take face states";
      return BS_INVALID_ARGUMENT;
    }
    const int along = side < 2 ? e.nj : e.ni;
    e.face_states_[side].resize(along);
    for (int t = 0; t < along; t++)
      e.face_states_[side][t] = {T(prim[4 * t]), T(prim[4 * t + 1]), T(prim[4 * t + 2]), T(prim[4 * t + 3])};
    return BS_OK;
  });
}

int bso_set_face_fluxes(void* h, int side, const double* flux) {
  return with_engine(h, [&](auto& e) {
    using T = decltype(e.gamma);
    if (side < 0 || side > 3 || e.cfg.boundaries[side].kind != BS_BC_FACE_STATES) {
      g_error = "the side does not take face fluxes";
      return BS_INVALID_ARGUMENT;
    }
    const int along = side < 2 ? e.nj : e.ni;
    if (flux == nullptr) {
      e.face_fluxes_[side].clear();
    } else {
      e.face_fluxes_[side].resize(4 * size_t(along));
      for (size_t k = 0; k < 4 * size_t(along); k++) e.face_fluxes_[side][k] = T(flux[k]);
    }
    return BS_OK;
  });
}

int bso_iterate(void* h, int steps) {
  return with_engine(h, [&](auto& e) {
    if (!e.iterate(steps)) {
      g_error = e.error;
      return BS_NON_PHYSICAL;
    }
    return BS_OK;
  });
}

int bso_iterate_implicit(void* h, int steps, double cfl, double omega) {
  if (!(cfl > 0 && omega >= 1)) {
    g_error = "LU-SGS needs cfl > 0 and omega >= 1";
    return BS_INVALID_ARGUMENT;
  }
  return with_engine(h, [&](auto& e) {
    if (!e.iterate_implicit(steps, cfl, omega)) {
      g_error = e.error;
      return BS_NON_PHYSICAL;
    }
    return BS_OK;
  });
}

// The LU-SGS correction dQ of the current state without applying it
// (implicitCorrection, src/engine-cpu/euler2d.ts:872-1105).
int bso_implicit_correction(void* h, double cfl, double omega, double* dq) {
  return with_engine(h, [&](auto& e) {
    e.implicit_correction(decltype(e.gamma)(cfl), decltype(e.gamma)(omega));
    for (size_t k = 0; k < e.dq.size(); k++) dq[k] = e.dq[k];
    return BS_OK;
  });
}

int bso_density_residual_norm(void* h, double* out) {
  return with_engine(h, [&](auto& e) {
    *out = e.density_residual_norm();
    return BS_OK;
  });
}

int bso_residual(void* h, double* out) {
  return with_engine(h, [&](auto& e) {
    e.residual_vector(out);
    return BS_OK;
  });
}

int bso_time_steps(void* h, double* out) {
  return with_engine(h, [&](auto& e) {
    e.compute_time_steps(std::numeric_limits<double>::infinity());
    for (size_t k = 0; k < e.dt.size(); k++) out[k] = e.dt[k];
    return BS_OK;
  });
}

int bso_boundary_fluxes(void* h, int side, bs_face_flux* out) {
  if (h == nullptr || side < 0 || side > 3) {
    g_error = "invalid side";
    return BS_INVALID_ARGUMENT;
  }
  Handle* hh = static_cast<Handle*>(h);
  return with_engine(h, [&](auto& e) {
    e.boundary_fluxes(side, hh->x.data(), hh->y.data(), out);
    return BS_OK;
  });
}

int bso_forebody_drag(void* h, double p_inf, double q_inf, double base_radius, double* cd) {
  return with_engine(h, [&](auto& e) {
    std::vector<bs_face_flux> wall(e.ni);
    Handle* hh = static_cast<Handle*>(h);
    e.boundary_fluxes(BS_JMIN, hh->x.data(), hh->y.data(), wall.data());
    *cd = bso::forebody_pressure_drag(wall.data(), e.ni, p_inf, q_inf, base_radius);
    return BS_OK;
  });
}

int bso_conserved(void* h, double* q) {
  return with_engine(h, [&](auto& e) {
    for (int j = 0; j < e.nj; j++)
      for (int i = 0; i < e.ni; i++) {
        const size_t k = e.index(i, j), c = 4 * (i + size_t(j) * e.ni);
        q[c] = e.st.rho[k];
        q[c + 1] = e.st.mu[k];
        q[c + 2] = e.st.mv[k];
        q[c + 3] = e.st.en[k];
      }
    return BS_OK;
  });
}

int bso_primitives(void* h, double* w) {
  return with_engine(h, [&](auto& e) {
    for (int j = 0; j < e.nj; j++)
      for (int i = 0; i < e.ni; i++) {
        const auto p = e.prim_at(e.st, e.index(i, j));
        double* c = w + 4 * (i + size_t(j) * e.ni);
        c[0] = p.rho;
        c[1] = p.u;
        c[2] = p.v;
        c[3] = p.p;
      }
    return BS_OK;
  });
}

int64_t bso_steps(void* h) {
  int64_t s = 0;
  with_engine(h, [&](auto& e) {
    s = e.steps;
    return BS_OK;
  });
  return s;
}

// Steady solve of one case in FP64: LU-SGS (method 1) at fixed CFL or explicit
// steps (method 0), checking the RMS density residual every `check_every`
// steps against `tol` (relative to the starting residual when `relative`).
// Writes steps taken, final and initial residual. Returns BS_NOT_CONVERGED
// when `max_steps` ran out.
int bso_solve(void* h, int method, double cfl, double omega, double tol, int relative,
              int max_steps, int check_every, int* steps_out, double* residual_out,
              double* initial_out) {
  return with_engine(h, [&](auto& e) {
    const double r0 = e.density_residual_norm();
    const double target = relative ? tol * r0 : tol;
    int taken = 0;
    double r = r0;
    int status = BS_NOT_CONVERGED;
    while (taken < max_steps) {
      const int n = std::min(check_every, max_steps - taken);
      const bool ok = method == 1 ? e.iterate_implicit(n, cfl, omega) : e.iterate(n);
      taken += n;
      if (!ok) {
        g_error = e.error;
        status = BS_NON_PHYSICAL;
        break;
      }
      r = e.density_residual_norm();
      if (r <= target) {
        status = BS_OK;
        break;
      }
    }
    if (steps_out) *steps_out = taken;
    if (residual_out) *residual_out = r;
    if (initial_out) *initial_out = r0;
    return status;
  });
}

// Run `fn(k)` for k in [0, n) over `threads` host threads (one case per
// thread at a time), for batched CPU baselines.
int bso_parallel_solve(int n, void** handles, int method, double cfl, double omega, double tol,
                       int relative, int max_steps, int check_every, int threads, int* steps,
                       double* residual, double* initial, int* status) {
  std::atomic<int> next{0};
  auto worker = [&]() {
    for (;;) {
      const int k = next.fetch_add(1);
      if (k >= n) return;
      status[k] = bso_solve(handles[k], method, cfl, omega, tol, relative, max_steps, check_every,
                            &steps[k], &residual[k], &initial[k]);
    }
  };
  threads = std::max(1, std::min(threads, n));
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; t++) pool.emplace_back(worker);
  for (auto& t : pool) t.join();
  return BS_OK;
}

}  // extern "C"
