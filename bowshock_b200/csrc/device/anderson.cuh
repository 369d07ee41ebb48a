// Anderson acceleration of the LU-SGS steps, every case of a batch at once
// (AndersonMixing, src/solver/anderson.ts:20-123, as the reference's
// transonic driver applies it, src/analysis/transonic-flow.ts:183-206).
// With x the state, f the LU-SGS correction dQ of x, and the last `depth`
// differences dX, dF of the iterates and corrections,
//
//   gamma = argmin |f - dF gamma|,   x <- x + f - (dX + dF) gamma
//
// (Walker and Ni's type II, undamped). A step on the GPU, after the residual
// pass and the sweeps have left f in the diagonal-major dQ array:
//   anderson_push_kernel   the new differences into the case's ring of
//                          columns, and in the same pass |f|^2 and their dot
//                          products with every stored column and with f,
//                          each tile's sums stored in a fixed order;
//   anderson_solve_kernel  one warp per case: the tiles' sums added in a
//                          fixed order, then in shared memory the Gram matrix
//                          of dF kept up to date, its Cholesky factor (the R
//                          of a Gram-Schmidt of dF) with the oldest columns
//                          dropped while a column keeps less than 1e-6 of its
//                          norm, and gamma (lane 0);
//   anderson_apply_kernel  x + f - (dX + dF) gamma, flagging a case whose new
//                          state is not physical;
//   anderson_fallback_kernel  for a flagged case, the plain LU-SGS update of
//                          the previous state instead, and the history is
//                          forgotten (as the reference does on a rejected
//                          step). So is it when |f|^2 exceeds 100 times its
//                          smallest value since the last restart.
// The differences are stored in FP32, the state, the dot products and the
// Gram matrix in FP64: the accelerated iterate only changes the path to the
// steady state, whose test is still the FP64 residual. The Gram form loses
// the square of the columns' condition number, hence the drop threshold of
// 1e-6 where the reference's modified Gram-Schmidt uses 1e-10.
#pragma once

#include "sweep.cuh"

namespace bsd {

constexpr int kMaxAndersonDepth = 16;

struct AndersonCase {
  int count;       // columns stored (at most depth)
  int head;        // oldest column's slot once the ring is full
  int have_last;   // last_x / last_f hold the previous iterate
  int bad;         // the accelerated state was not physical (set by apply)
  int restarts;    // times the history was forgotten
  int pad;
  double best;     // smallest |f|^2 since the last restart (+inf at first)
};

// Per tile, `part` holds 1 + 2 depth sums over the tile's cells for the
// current step (the tile's row at its case's tile_base plus its index):
// |f|^2, the new column's dot products with the columns by slot, and each
// column's dot product with f by slot. The solve kernel adds the rows of a
// case in a fixed order, so a step's result does not depend on the order in
// which the tiles ran.
template <class R>
struct AndersonArgs {
  const CaseDev* cases;
  const int2* tiles;
  const int* case_list;   // solve kernel: thread -> case
  int n_cases;            // solve kernel: cases in the list
  const int* active;
  StateView<R> q;
  StateView<R> last_x;
  const float4* dq;       // the sweeps' correction, row-major like the state
  float4* last_f;         // like the state
  float4* dx;             // depth columns: slot s of cell k at s * total + k
  float4* df;
  int64_t total;          // cells of the batch
  int depth;
  AndersonCase* ac;
  double* part;           // (1 + 2 depth) per tile
  double* gram;           // depth x depth per case, by slot
  double* gamma;          // depth per case, by slot (0 for a dropped column)
  unsigned* status;
};

// The cell of thread `tid` in tile `tile`, or false when the thread has none.
__device__ __forceinline__ bool anderson_cell(const CaseDev& cd, int2 tile, int tid, int* i, int* j) {
  const int tiles_i = (cd.ni + TI - 1) / TI;
  *i = (tile.y % tiles_i) * TI + tid % TI;
  *j = (tile.y / tiles_i) * TJ + tid / TI;
  return tid < TI * TJ && *i < cd.ni && *j < cd.nj;
}

// Adds per-thread values over the CTA in a fixed order and stores them to
// out[0 .. 1 + 2 n): the sum of vf, then those of va[p], then those of
// vb[p], p < n (n <= K, the same for every thread of the CTA).
template <int K>
__device__ __forceinline__ void cta_store(double vf, const double (&va)[K], const double (&vb)[K], int n,
                                          double* out) {
  __shared__ double part[TILE_THREADS / 32][1 + 2 * K];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double sf = warp_sum(vf);
  if (lane == 0) part[warp][0] = sf;
#pragma unroll
  for (int p = 0; p < K; p++) {
    if (p < n) {
      const double sa = warp_sum(va[p]);
      const double sb = warp_sum(vb[p]);
      if (lane == 0) {
        part[warp][1 + p] = sa;
        part[warp][1 + n + p] = sb;
      }
    }
  }
  __syncthreads();
  const int t = threadIdx.x;
  if (t < 1 + 2 * n) {
    double s = 0;
    for (int w = 0; w < TILE_THREADS / 32; w++) s += part[w][t];
    out[t] = s;
  }
}

__device__ __forceinline__ double dot4(float4 a, float4 b) {
  return double(a.x) * b.x + double(a.y) * b.y + double(a.z) * b.z + double(a.w) * b.w;
}

// Whether this step forgets the history: the previous accelerated state was
// rejected, or |f|^2 grew past 100 times its smallest value since the last
// restart (transonic-flow.ts:187-191). Every kernel of the step decides the
// same way from the same words.
__device__ __forceinline__ bool anderson_reset(const AndersonCase& a, double fnorm) {
  return a.bad != 0 || fnorm > 100.0 * a.best;
}

// |f|^2 and the push of the new difference columns. The column is pushed
// unless the previous accelerated state was rejected; if this step's |f|^2
// makes the solve kernel forget the history, the column goes with the rest.
template <class R>
__global__ void __launch_bounds__(TILE_THREADS) anderson_push_kernel(const AndersonArgs<R> A) {
  const int2 tile = A.tiles[blockIdx.x];
  const int c = tile.x;
  if (A.active != nullptr && A.active[c] == 0) return;
  const CaseDev& cd = A.cases[c];
  const AndersonCase a = A.ac[c];
  const bool push = a.have_last && a.bad == 0;
  const int slot = a.count < A.depth ? a.count : a.head;
  const int ncols = push ? min(a.count + 1, A.depth) : 0;
  int i, j;
  const bool mine = anderson_cell(cd, tile, threadIdx.x, &i, &j);
  const int64_t k = cd.cell + i + int64_t(j) * cd.ni;
  float4 f = make_float4(0.f, 0.f, 0.f, 0.f), dfn = f;
  if (mine) {
    f = A.dq[k];
    const Cons<R> x = A.q.load(k);
    if (push) {
      const Cons<R> lx = A.last_x.load(k);
      const float4 lf = A.last_f[k];
      dfn = make_float4(f.x - lf.x, f.y - lf.y, f.z - lf.z, f.w - lf.w);
      A.dx[slot * A.total + k] = make_float4(float(x.rho - lx.rho), float(x.mu - lx.mu),
                                             float(x.mv - lx.mv), float(x.e - lx.e));
      A.df[slot * A.total + k] = dfn;
    }
    A.last_x.store(k, x);
    A.last_f[k] = f;
  }
  // The tile's row: |f|^2, then new column . column p for p < ncols, then
  // column p . f (the solve kernel reads them with this packing).
  double vg[kMaxAndersonDepth], vb[kMaxAndersonDepth];
#pragma unroll
  for (int p = 0; p < kMaxAndersonDepth; p++) {
    vg[p] = 0.0;
    vb[p] = 0.0;
    if (mine && p < ncols) {
      const float4 col = p == slot ? dfn : A.df[p * A.total + k];
      vg[p] = dot4(dfn, col);
      vb[p] = dot4(col, f);
    }
  }
  cta_store<kMaxAndersonDepth>(mine ? dot4(f, f) : 0.0, vg, vb, ncols,
                               A.part + (cd.tile_base + tile.y) * (1 + 2 * A.depth));
}

// One warp per case of the lane: the case's tile rows added in a fixed order
// (lane v adds value v over the tiles in order, every value at once), then
// lane 0 updates the history and solves for the mixing coefficients.
template <class R>
__global__ void __launch_bounds__(32) anderson_solve_kernel(const AndersonArgs<R> A) {
  const int c = A.case_list[blockIdx.x];
  if (A.active != nullptr && A.active[c] == 0) return;
  const int m = A.depth;
  const CaseDev& cd = A.cases[c];
  AndersonCase a = A.ac[c];
  const int width = 1 + 2 * m;
  const int pushed = a.have_last && a.bad == 0 ? min(a.count + 1, m) : 0;
  const int nv = 1 + 2 * pushed;
  const int ntiles = ((cd.ni + TI - 1) / TI) * ((cd.nj + TJ - 1) / TJ);
  const double* rows = A.part + cd.tile_base * width;
  __shared__ double acc[1 + 2 * kMaxAndersonDepth];
  for (int v = int(threadIdx.x); v < nv; v += 32) {
    double s = 0;
    for (int t = 0; t < ntiles; t++) s += rows[int64_t(t) * width + v];
    acc[v] = s;
  }
  // The Gram matrix into shared memory (loaded by the warp), where lane 0
  // updates it and factors it; the factor and the vectors of the solve too.
  __shared__ double Gs[kMaxAndersonDepth * kMaxAndersonDepth];
  __shared__ double Rm[kMaxAndersonDepth][kMaxAndersonDepth];
  __shared__ double b[kMaxAndersonDepth], z[kMaxAndersonDepth], gs[kMaxAndersonDepth];
  __shared__ int ord[kMaxAndersonDepth];
  double* G = A.gram + int64_t(c) * m * m;
  for (int k = int(threadIdx.x); k < m * m; k += 32) Gs[k] = G[k];
  __syncwarp();
  if (threadIdx.x != 0) return;
  double* gam = A.gamma + int64_t(c) * m;
  const double fnorm = acc[0];
  const bool reset = anderson_reset(a, fnorm);
  const bool push = a.have_last && !reset;
  if (reset) {
    if (a.bad || fnorm > 100.0 * a.best) a.restarts++;
    if (fnorm > 100.0 * a.best) a.best = fnorm;
    a.count = 0;
    a.head = 0;
  } else if (push) {
    const int slot = a.count < m ? a.count : a.head;
    const int ncols = min(a.count + 1, m);
    for (int p = 0; p < ncols; p++) {
      Gs[slot * m + p] = acc[1 + p];
      Gs[p * m + slot] = acc[1 + p];
      G[slot * m + p] = acc[1 + p];
      G[p * m + slot] = acc[1 + p];
      b[p] = acc[1 + ncols + p];
    }
    if (a.count < m) {
      a.count++;
    } else {
      a.head = (a.head + 1) % m;
    }
  }
  a.best = fmin(a.best, fnorm);
  a.have_last = 1;
  a.bad = 0;
  for (int p = 0; p < m; p++) gs[p] = 0.0;
  const int n = push ? a.count : 0;
  // Columns oldest first; drop the oldest while the factor is not well
  // conditioned (anderson.ts:78-114 on the Gram matrix).
  for (int t = 0; t < n; t++) ord[t] = a.count < m ? t : (a.head + t) % m;
  for (int first = 0; first < n; first++) {
    const int cols = n - first;
    bool ok = true;
    for (int cc = 0; cc < cols && ok; cc++) {
      const int sc = ord[first + cc];
      for (int p = 0; p < cc; p++) {
        double s = Gs[ord[first + p] * m + sc];
        for (int r = 0; r < p; r++) s -= Rm[r][p] * Rm[r][cc];
        Rm[p][cc] = s / Rm[p][p];
      }
      double d = Gs[sc * m + sc];
      const double g0 = d;
      for (int p = 0; p < cc; p++) d -= Rm[p][cc] * Rm[p][cc];
      if (!(g0 > 0.0) || !(d > 1e-12 * g0)) {
        ok = false;
      } else {
        Rm[cc][cc] = sqrt(d);
      }
    }
    if (!ok) continue;
    for (int cc = 0; cc < cols; cc++) {
      double s = b[ord[first + cc]];
      for (int p = 0; p < cc; p++) s -= Rm[p][cc] * z[p];
      z[cc] = s / Rm[cc][cc];
    }
    for (int cc = cols - 1; cc >= 0; cc--) {
      double s = z[cc];
      for (int p = cc + 1; p < cols; p++) s -= Rm[cc][p] * gs[ord[first + p]];
      gs[ord[first + cc]] = s / Rm[cc][cc];
    }
    break;
  }
  for (int p = 0; p < m; p++) gam[p] = gs[p];
  A.ac[c] = a;
}

template <class R>
__global__ void __launch_bounds__(TILE_THREADS) anderson_apply_kernel(const AndersonArgs<R> A) {
  __shared__ double g[kMaxAndersonDepth];
  const int2 tile = A.tiles[blockIdx.x];
  const int c = tile.x;
  if (A.active != nullptr && A.active[c] == 0) return;
  const CaseDev& cd = A.cases[c];
  const int n = A.ac[c].count;
  if (int(threadIdx.x) < n) g[threadIdx.x] = A.gamma[int64_t(c) * A.depth + threadIdx.x];
  __syncthreads();
  int i, j;
  bool bad = false;
  if (anderson_cell(cd, tile, threadIdx.x, &i, &j)) {
    const int64_t k = cd.cell + i + int64_t(j) * cd.ni;
    const float4 f = A.dq[k];
    const Cons<R> x = A.q.load(k);
    R o0 = x.rho + R(f.x), o1 = x.mu + R(f.y), o2 = x.mv + R(f.z), o3 = x.e + R(f.w);
    for (int s = 0; s < n; s++) {
      const R gs = R(g[s]);
      if (gs == R(0)) continue;
      const float4 a = A.dx[s * A.total + k], b = A.df[s * A.total + k];
      o0 -= gs * (R(a.x) + R(b.x));
      o1 -= gs * (R(a.y) + R(b.y));
      o2 -= gs * (R(a.z) + R(b.z));
      o3 -= gs * (R(a.w) + R(b.w));
    }
    const Cons<R> o{o0, o1, o2, o3};
    A.q.store(k, o);
    bad = !is_physical(o, R(cd.gamma));
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicExch(&A.ac[c].bad, 1);
}

template <class R>
__global__ void __launch_bounds__(TILE_THREADS) anderson_fallback_kernel(const AndersonArgs<R> A) {
  const int2 tile = A.tiles[blockIdx.x];
  const int c = tile.x;
  if (A.active != nullptr && A.active[c] == 0) return;
  if (A.ac[c].bad == 0) return;
  const CaseDev& cd = A.cases[c];
  int i, j;
  bool bad = false;
  if (anderson_cell(cd, tile, threadIdx.x, &i, &j)) {
    const int64_t k = cd.cell + i + int64_t(j) * cd.ni;
    const Cons<R> q1 = implicit_update(A.last_x.load(k), A.dq[k], R(cd.gamma));
    A.q.store(k, q1);
    bad = !is_physical(q1, R(cd.gamma));
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&A.status[c], STATUS_NON_PHYSICAL);
}

}  // namespace bsd
