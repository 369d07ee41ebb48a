// LU-SGS forward and backward sweeps as anti-diagonal wavefronts
// (implicitCorrection's sweeps, src/engine-cpu/euler2d.ts:1058-1102), and
// the update that applies the correction (applyImplicitUpdate, :816-847).
//
// The forward sweep solves (D + L) dQ* = R cell by cell in the order j, then
// i; cell (i, j) needs only (i - 1, j) and (i, j - 1), both on the previous
// anti-diagonal i + j = d - 1, so every cell of a diagonal is independent and
// the sweep is ni + nj - 1 dependent steps. One CTA owns a case; thread j
// owns grid row j for the whole sweep and walks it along i as d advances:
//   - its west (forward) / east (backward) neighbour is the cell it finished
//     on the previous step, held in registers;
//   - its south / north neighbour is the cell thread j -+ 1 finished on the
//     previous step: its dQ by warp shuffle (shared memory across a warp
//     edge), its state and face through double-buffered shared memory;
//   - its own operands (residual or dQ*, state, (u, v, p, 1/D), faces) come
//     from the per-cell records that the residual pass wrote diagonal-major,
//     staged into shared memory by TMA bulk copies a chunk of diagonals at a
//     time, two chunks in flight.
// One barrier per diagonal orders the exchange. A step has no branch: every
// thread computes, and only cells on the grid store.
//
// The operator runs in FP32. The neighbour term is the change of the
// physical flux, F(Q + dQ) - F(Q), exactly as the reference forms it, but
// evaluated in a rearranged form whose every term is proportional to dQ
// (no difference of two O(|F|) numbers), so FP32 rounding is relative to the
// term itself and vanishes with dQ.
#pragma once

#include <algorithm>

#include "layout.cuh"

namespace bsd {

struct SweepArgs {
  const CaseDev* cases;
  const int* case_list;   // blockIdx.x -> case
  const int* active;      // per case (may be null)
  const float4* rec;      // sweep records, diagonal-major (5 float4 per slot, pass A)
  float4* dq;             // diagonal-major: forward result dQ*, then the final dQ
  float* cfl;             // per case current CFL number (ramped after the sweep)
  const float* cfl_max;   // per case
  const float* growth;    // per case
  const float* omega;     // per case
  unsigned* status;       // per case
  int chunk;              // diagonals per bulk copy
  int wait_limit;         // mbarrier polls before a wait gives up
};

// Fields of the sweep record (five float4 per cell, written by the residual
// pass): residual; state; (u, v, p, 1/D); west face and south face as
// (nx, ny, A/2, omega lambda A / 2).
enum { REC_R = 0, REC_Q = 1, REC_W = 2, REC_FW = 3, REC_FS = 4, REC_SIZE = 5 };

// ---- TMA bulk copies and mbarriers (sm_90 and later; no multicast) --------
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
               "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for phase `parity` of `bar`; false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int limit) {
  for (int k = 0; k < limit; k++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async;\n" ::: "memory");
}

// 1/x by the hardware approximation (rcp.approx.ftz.f32, within about one
// ulp): the LU-SGS operator runs in FP32 and only shapes the path to the
// steady state, whose residual is FP64.
__device__ __forceinline__ float approx_rcp(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Shared memory of the sweep for `nt` threads, `nj` rows and chunks of
// `chunk` diagonals: a 128-byte header (two mbarriers), the double-buffered
// exchange (state, (u, v, p, 1/D), dQ, south face) and two chunk buffers of
// records and of dQ*.
__host__ __device__ constexpr size_t sweep_smem_bytes(int nt, int nj, int chunk) {
  return 128 + size_t(nt) * 16 * 8 + 2 * size_t(chunk) * nj * 16 * (REC_SIZE + 1);
}

// The d-independent part of a neighbour's term: its state, the face normal
// (signed for the direction the flux leaves), A/2, omega lambda A/2, its
// normal velocity and the momentum and kinetic-energy weights of dK.
struct NeighbourTerm {
  float4 q;
  float nx, ny, half_area, damp, un, ku, kv, kk, p;
};

__device__ __forceinline__ NeighbourTerm neighbour_term(const float4 q, const float4 w, const float4 f,
                                                        float sgn) {
  NeighbourTerm t;
  t.q = q;
  t.nx = sgn * f.x;
  t.ny = sgn * f.y;
  t.half_area = f.z;
  t.damp = f.w;
  t.un = w.x * t.nx + w.y * t.ny;
  t.ku = q.x * w.x;
  t.kv = q.x * w.y;
  t.kk = q.x * (0.5f * (w.x * w.x + w.y * w.y));
  t.p = w.z;
  return t;
}

// The neighbour term of src/engine-cpu/euler2d.ts:977-1005 - the change of
// the physical flux across the face, F(Q + d) - F(Q), times A/2, less
// omega lambda A/2 d - added to `sum`. The exact difference is written so
// that every term is proportional to d (no difference of two O(|F|)
// numbers), so FP32 rounding is relative to the term and d = 0 adds exactly
// nothing, which stands for an absent neighbour.
__device__ __forceinline__ void add_neighbour(float4& sum, const NeighbourTerm& t, const float4 d,
                                              float gm1) {
  const float inv1 = approx_rcp(t.q.x + d.x);
  const float dmn = d.y * t.nx + d.z * t.ny;
  const float dun = (dmn - t.un * d.x) * inv1;
  const float dk = (t.ku * d.y + t.kv * d.z - t.kk * d.x + 0.5f * (d.y * d.y + d.z * d.z)) * inv1;
  const float dp = gm1 * (d.w - dk);
  sum.x += t.half_area * dmn - t.damp * d.x;
  sum.y += t.half_area * (d.y * t.un + (t.q.y + d.y) * dun + dp * t.nx) - t.damp * d.y;
  sum.z += t.half_area * (d.z * t.un + (t.q.z + d.z) * dun + dp * t.ny) - t.damp * d.z;
  sum.w += t.half_area * ((d.w + dp) * t.un + (t.q.w + d.w + t.p + dp) * dun) - t.damp * d.w;
}

// The forward and backward sweeps of every active case, one CTA per case,
// leaving the final correction dQ (diagonal-major) for lusgs_update_kernel.
static __global__ void __launch_bounds__(512) lusgs_sweep_kernel(const SweepArgs A) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int c = A.case_list[blockIdx.x];
  if (A.active != nullptr && A.active[c] == 0) return;
  const CaseDev& cd = A.cases[c];
  const int ni = cd.ni, nj = cd.nj;
  const int nt = blockDim.x;
  const int j = threadIdx.x;
  const bool row = j < nj;
  const float gm1 = float(cd.gamma) - 1.f;
  const int ndiag = ni + nj - 1;
  const int K = A.chunk;
  const int nchunks = (ndiag + K - 1) / K;

  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);
  float4* xq = reinterpret_cast<float4*>(smem_raw + 128);  // [2][nt] exchange: state
  float4* xw = xq + 2 * nt;                                 // (u, v, p, 1/D)
  float4* xd = xw + 2 * nt;                                 // dQ
  float4* xf = xd + 2 * nt;                                 // south face
  float4* ring_rec = xf + 2 * nt;                           // [2][K nj][5]
  float4* ring_dq = ring_rec + 2 * size_t(K) * nj * REC_SIZE;  // [2][K nj]
  const float4* rec_case = A.rec + REC_SIZE * cd.skew;
  float4* dq_case = A.dq + cd.skew;
  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);

  if (j == 0) {
    for (int b = 0; b < 2; b++) mbar_init(&bars[b], 1);
    mbar_fence_init();
  }
  // Benign exchange contents: a slot read for an absent neighbour is
  // multiplied by a zero dQ and must be finite.
  for (int k = j; k < 2 * nt; k += nt) {
    xq[k] = make_float4(1.f, 0.f, 0.f, 1.f);
    xw[k] = make_float4(0.f, 0.f, 1.f, 1.f);
    xd[k] = zero;
    xf[k] = zero;
  }
  __syncthreads();

  unsigned uses[2] = {};    // completed phases of each buffer's mbarrier
  unsigned issued[2] = {};  // copies issued into each buffer
  bool failed = false;
  for (int pass = 0; pass < 2 && !failed; pass++) {
    const bool fwd = pass == 0;
    // Chunk cc holds the diagonals [dlo, dlo + n) in memory order.
    auto chunk_range = [&](int cc, int& dlo, int& n) {
      n = min(K, ndiag - cc * K);
      dlo = fwd ? cc * K : ndiag - cc * K - n;
    };
    auto issue = [&](int cc) {  // one thread
      int dlo, n;
      chunk_range(cc, dlo, n);
      const int buf = cc % 2;
      const unsigned rec_bytes = unsigned(n) * nj * 16u * REC_SIZE;
      const unsigned dq_bytes = fwd ? 0u : unsigned(n) * nj * 16u;
      mbar_arrive_expect_tx(&bars[buf], rec_bytes + dq_bytes);
      bulk_load(ring_rec + size_t(buf) * K * nj * REC_SIZE, rec_case + size_t(REC_SIZE) * dlo * nj,
                rec_bytes, &bars[buf]);
      if (!fwd) bulk_load(ring_dq + size_t(buf) * K * nj, dq_case + size_t(dlo) * nj, dq_bytes, &bars[buf]);
    };
    if (j == 0) fence_proxy_async();
    for (int k = 0; k < 2 && k < nchunks; k++) {
      if (j == 0) issue(k);
      issued[k]++;
    }
    // The cell this thread finished last step (its neighbour along the row).
    float4 pq = make_float4(1.f, 0.f, 0.f, 1.f), pw = make_float4(0.f, 0.f, 1.f, 1.f);
    float4 pd = zero, pfw = zero;
    for (int cc = 0; cc < nchunks; cc++) {
      const int buf = cc % 2;
      const bool ok = mbar_wait(&bars[buf], uses[buf] & 1u, A.wait_limit);
      if (ok) uses[buf]++;
      if (__syncthreads_or(!ok)) {
        failed = true;
        break;
      }
      int dlo, n;
      chunk_range(cc, dlo, n);
      const float4* rb = ring_rec + size_t(buf) * K * nj * REC_SIZE;
      const float4* db = ring_dq + size_t(buf) * K * nj;
      for (int t = 0; t < n; t++) {
        const int step = cc * K + t;
        const int d = fwd ? step : ndiag - 1 - step;
        const int i = d - j;
        // The dQ row j -+ 1 finished on the previous step, inside the warp.
        float4 sh;
        sh.x = fwd ? __shfl_up_sync(0xffffffffu, pd.x, 1) : __shfl_down_sync(0xffffffffu, pd.x, 1);
        sh.y = fwd ? __shfl_up_sync(0xffffffffu, pd.y, 1) : __shfl_down_sync(0xffffffffu, pd.y, 1);
        sh.z = fwd ? __shfl_up_sync(0xffffffffu, pd.z, 1) : __shfl_down_sync(0xffffffffu, pd.z, 1);
        sh.w = fwd ? __shfl_up_sync(0xffffffffu, pd.w, 1) : __shfl_down_sync(0xffffffffu, pd.w, 1);
        const bool lane_edge = (j & 31) == (fwd ? 0 : 31);
        // Only cells on the grid store; the others compute on records of
        // their chunk (possibly padding) and discard the result.
        const bool active = row && i >= 0 && i < ni;
        {
          const int local = (d - dlo) * nj + min(j, nj - 1);
          const float4* r5 = rb + size_t(REC_SIZE) * local;
          const float4 q = r5[REC_Q], w = r5[REC_W], fw = r5[REC_FW], fs = r5[REC_FS];
          const float4 base = fwd ? r5[REC_R] : db[local];
          const bool has_i = fwd ? i > 0 : i < ni - 1;
          const bool has_j = fwd ? j > 0 : j < nj - 1;
          const int b = ((step - 1) & 1) * nt + (fwd ? j - 1 : j + 1);
          const int bb = has_j ? b : (step & 1) * nt + j;  // an in-range slot either way
          const float4 oq = xq[bb], ow = xw[bb], of = xf[bb];
          float4 od = zero;
          if (has_j) od = lane_edge ? xd[bb] : sh;
          // Forward: this cell's west and south faces, the flux leaving
          // through -n; backward: the east neighbour's west face and the
          // north neighbour's south face, through +n.
          const float sgn = fwd ? -1.f : 1.f;
          const float4 face_i = fwd ? fw : pfw;
          const float4 face_j = fwd ? fs : of;
          float4 sum = zero;
          const NeighbourTerm ti = neighbour_term(pq, pw, face_i, sgn);
          const NeighbourTerm tj = neighbour_term(oq, ow, face_j, sgn);
          add_neighbour(sum, ti, has_i ? pd : zero, gm1);
          add_neighbour(sum, tj, od, gm1);
          const float inv_d = w.w;
          float4 dq;
          if (fwd) {
            dq = make_float4((base.x - sum.x) * inv_d, (base.y - sum.y) * inv_d,
                             (base.z - sum.z) * inv_d, (base.w - sum.w) * inv_d);
          } else {
            dq = make_float4(base.x - sum.x * inv_d, base.y - sum.y * inv_d,
                             base.z - sum.z * inv_d, base.w - sum.w * inv_d);
          }
          const int o = (step & 1) * nt + j;
          if (active) {
            xq[o] = q;
            xw[o] = w;
            xd[o] = dq;
            xf[o] = fs;
            dq_case[size_t(d) * nj + j] = dq;
          }
          pq = active ? q : pq;
          pw = active ? w : pw;
          pd = active ? dq : pd;
          pfw = active ? fw : pfw;
        }
        __syncthreads();
      }
      if (cc + 2 < nchunks) {
        if (j == 0) issue(cc + 2);
        issued[buf]++;
      }
    }
    // dQ* written by this pass is read by the next pass's bulk copies.
    fence_proxy_async();
    __syncthreads();
  }
  if (failed) {
    // Let the copies still in flight land (bounded) before leaving.
    for (int b = 0; b < 2; b++)
      for (unsigned u = uses[b]; u < issued[b]; u++) mbar_wait(&bars[b], u & 1u, A.wait_limit);
    if (j == 0) atomicOr(&A.status[c], STATUS_TIMEOUT);
    return;
  }
  if (j == 0) A.cfl[c] = fminf(A.cfl_max[c], A.cfl[c] * A.growth[c]);
}

// applyImplicitUpdate (src/engine-cpu/euler2d.ts:816-847) for one cell:
// Q + alpha dQ with alpha halved until density and pressure stay within a
// factor of two of Q's.
template <class R>
__device__ __forceinline__ Cons<R> implicit_update(const Cons<R>& q0, float4 d4, R gamma) {
  const R p0 = pressure_of(q0.rho, q0.mu, q0.mv, q0.e, gamma);
  const R d0 = R(d4.x), d1 = R(d4.y), d2 = R(d4.z), d3 = R(d4.w);
  R alpha = R(1);
  for (int tries = 0; tries < 30; tries++) {
    const R rho1 = q0.rho + alpha * d0;
    const R p1 = pressure_of(rho1, q0.mu + alpha * d1, q0.mv + alpha * d2, q0.e + alpha * d3, gamma);
    if (rho1 > R(0.5) * q0.rho && rho1 < R(2) * q0.rho && p1 > R(0.5) * p0 && p1 < R(2) * p0) break;
    alpha *= R(0.5);
  }
  return {q0.rho + alpha * d0, q0.mu + alpha * d1, q0.mv + alpha * d2, q0.e + alpha * d3};
}

// The update for every cell of every active case; flags non-physical results.
template <class R>
__global__ void __launch_bounds__(TILE_THREADS) lusgs_update_kernel(const CaseDev* cases,
                                                                    const int2* tiles,
                                                                    const int* active,
                                                                    StateView<R> q,
                                                                    const float4* dq,
                                                                    unsigned* status) {
  const int2 tile = tiles[blockIdx.x];
  const int c = tile.x;
  if (active != nullptr && active[c] == 0) return;
  const CaseDev& cd = cases[c];
  const int ni = cd.ni, nj = cd.nj;
  const int tiles_i = (ni + TI - 1) / TI;
  const int i = (tile.y % tiles_i) * TI + threadIdx.x % TI;
  const int j = (tile.y / tiles_i) * TJ + threadIdx.x / TI;
  bool bad = false;
  if (i < ni && j < nj && int(threadIdx.x) < TI * TJ) {
    const R gamma = R(cd.gamma);
    const int64_t k = cd.cell + i + int64_t(j) * ni;
    const Cons<R> q1 = implicit_update(q.load(k), dq[cd.skew + skew_slot(i, j, nj)], gamma);
    q.store(k, q1);
    bad = !is_physical(q1, gamma);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&status[c], STATUS_NON_PHYSICAL);
}

// Diagonals per bulk copy for cases of up to `nj` rows (`nt` threads) when
// `cases_in_flight` cases sweep at once: the largest (up to 8) that lets
// the resident cases (up to 8 per SM) share an SM's shared memory, else the
// largest that fits one CTA; 0 if not even one diagonal does.
inline int sweep_chunk(int nt, int nj, int cases_in_flight) {
  const int per_sm = std::min(8, std::max(1, (cases_in_flight + 147) / 148));
  for (size_t budget : {size_t(200 * 1024) / per_sm, size_t(200 * 1024)})
    for (int k = 8; k >= 1; k--)
      if (sweep_smem_bytes(nt, nj, k) <= budget) return k;
  return 0;
}

// `cases_in_flight`: cases of the whole batch sweeping at the same time
// (other lanes included), which sets the shared memory each CTA may take.
inline cudaError_t launch_sweep(SweepArgs A, int n_cases, int max_nj, int cases_in_flight,
                                cudaStream_t stream) {
  const int nt = ((max_nj + 31) / 32) * 32;
  A.chunk = sweep_chunk(nt, max_nj, cases_in_flight);
  if (A.chunk == 0 || nt > 512) return cudaErrorInvalidConfiguration;
  A.wait_limit = 1 << 22;
  const size_t bytes = sweep_smem_bytes(nt, max_nj, A.chunk);
  const cudaError_t e = cudaFuncSetAttribute(lusgs_sweep_kernel,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
  if (e != cudaSuccess) return e;
  lusgs_sweep_kernel<<<n_cases, nt, bytes, stream>>>(A);
  return cudaGetLastError();
}

}  // namespace bsd
