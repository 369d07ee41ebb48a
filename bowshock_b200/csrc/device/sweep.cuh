// LU-SGS forward and backward sweeps as anti-diagonal wavefronts
// (implicitCorrection's sweeps, src/engine-cpu/euler2d.ts:1058-1102, and
// applyImplicitUpdate, :816-847, fused into the backward sweep).
//
// The forward sweep solves (D + L) dQ* = R cell by cell in the order j, then
// i; cell (i, j) needs only (i - 1, j) and (i, j - 1), both on the previous
// anti-diagonal i + j = d - 1, so every cell of a diagonal is independent and
// the sweep is ni + nj - 1 dependent steps. One CTA owns a case; thread j
// owns grid row j for the whole sweep and walks it along i as d advances:
//   - its west (forward) / east (backward) neighbour is the cell it finished
//     on the previous step, held in registers;
//   - its south / north neighbour is the cell thread j -+ 1 finished on the
//     previous step, exchanged through double-buffered shared memory;
//   - everything that does not depend on dQ (residual, diagonal, state, face
//     metrics) is prefetched one step ahead, so a step's critical path is the
//     exchange, the two neighbour terms and one division.
// One __syncthreads per diagonal orders the exchange.
//
// The operator runs in FP32. The neighbour term is the change of the
// physical flux, F(Q + dQ) - F(Q), exactly as the reference forms it, but
// evaluated in a rearranged form whose every term is proportional to dQ
// (no difference of two O(|F|) numbers), so FP32 rounding is relative to the
// term itself and vanishes with dQ.
#pragma once

#include "layout.cuh"

namespace bsd {

struct SweepArgs {
  const CaseDev* cases;
  const int* case_list;   // blockIdx.x -> case
  const int* active;      // per case (may be null)
  MetricsView m;
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

// Change of the physical flux along (nx, ny) of state q (with u, v, p in
// w) for the change d, times half_area, less damp d, added to `sum` (the
// neighbour term, src/engine-cpu/euler2d.ts:977-1005: half_area = A / 2,
// damp = omega lambda A / 2) - the exact difference F(Q + dQ) - F(Q) written
// so that every term is proportional to dQ. d = 0 contributes exactly
// nothing, which stands for an absent neighbour.
__device__ __forceinline__ void neighbour_change(float4& sum, const float4 q, const float4 w,
                                                 const float4 d, float nx, float ny,
                                                 float half_area, float damp, float gm1) {
  const float u = w.x, v = w.y, p = w.z;
  const float un = u * nx + v * ny;
  const float inv1 = __frcp_rn(q.x + d.x);
  const float dmn = d.y * nx + d.z * ny;
  const float dun = (dmn - un * d.x) * inv1;
  const float dk = (q.x * (u * d.y + v * d.z - 0.5f * (u * u + v * v) * d.x) +
                    0.5f * (d.y * d.y + d.z * d.z)) * inv1;
  const float dp = gm1 * (d.w - dk);
  sum.x += half_area * dmn - damp * d.x;
  sum.y += half_area * (d.y * un + (q.y + d.y) * dun + dp * nx) - damp * d.y;
  sum.z += half_area * (d.z * un + (q.z + d.z) * dun + dp * ny) - damp * d.z;
  sum.w += half_area * ((d.w + dp) * un + (q.w + d.w + p + dp) * dun) - damp * d.w;
}

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

// Shared memory of the sweep kernel for `nt` threads, `nj` rows and chunks
// of `chunk` diagonals: two mbarriers; the exchange (state, u/v/p/(1/D), dQ,
// south face; double-buffered); two chunk buffers of records and of dQ*.
__host__ __device__ constexpr size_t sweep_smem_bytes(int nt, int nj, int chunk) {
  return 128 + size_t(nt) * 16 * 8 + 2 * size_t(chunk) * nj * 16 * (REC_SIZE + 1);
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
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
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

  unsigned uses[2] = {0u, 0u};    // completed phases of each buffer's mbarrier
  unsigned issued[2] = {0u, 0u};  // copies issued into each buffer
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
      const int buf = cc & 1;
      const unsigned rec_bytes = unsigned(n) * nj * 16u * REC_SIZE;
      const unsigned dq_bytes = fwd ? 0u : unsigned(n) * nj * 16u;
      mbar_arrive_expect_tx(&bars[buf], rec_bytes + dq_bytes);
      bulk_load(ring_rec + size_t(buf) * K * nj * REC_SIZE, rec_case + size_t(REC_SIZE) * dlo * nj,
                rec_bytes, &bars[buf]);
      if (!fwd) bulk_load(ring_dq + size_t(buf) * K * nj, dq_case + size_t(dlo) * nj, dq_bytes, &bars[buf]);
    };
    if (j == 0) {
      fence_proxy_async();
      issue(0);
      issued[0]++;
      if (nchunks > 1) {
        issue(1);
        issued[1]++;
      }
    } else {
      issued[0]++;
      if (nchunks > 1) issued[1]++;
    }
    // The cell this thread finished last step (its neighbour along the row).
    float4 pq = make_float4(1.f, 0.f, 0.f, 1.f), pw = make_float4(0.f, 0.f, 1.f, 1.f);
    float4 pd = zero, pfw = zero;
    for (int cc = 0; cc < nchunks; cc++) {
      const int buf = cc & 1;
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
        if (row && i >= 0 && i < ni) {
          const int local = (d - dlo) * nj + j;
          const float4* r5 = rb + size_t(REC_SIZE) * local;
          const float4 q = r5[REC_Q], w = r5[REC_W], fw = r5[REC_FW], fs = r5[REC_FS];
          const float4 base = fwd ? r5[REC_R] : db[local];
          const bool has_i = fwd ? i > 0 : i < ni - 1;
          const bool has_j = fwd ? j > 0 : j < nj - 1;
          const int b = ((step - 1) & 1) * nt + (fwd ? j - 1 : j + 1);
          const int bb = has_j ? b : (step & 1) * nt + j;  // an in-range slot either way
          const float4 oq = xq[bb], ow = xw[bb], of = xf[bb];
          const float4 od = has_j ? xd[bb] : zero;
          // Forward: this cell's west and south faces, the flux leaving
          // through -n; backward: the east neighbour's west face and the
          // north neighbour's south face, through +n.
          const float sgn = fwd ? -1.f : 1.f;
          const float4 face_i = fwd ? fw : pfw;
          const float4 face_j = fwd ? fs : of;
          float4 sum = zero;
          neighbour_change(sum, pq, pw, has_i ? pd : zero, sgn * face_i.x, sgn * face_i.y, face_i.z,
                           face_i.w, gm1);
          neighbour_change(sum, oq, ow, od, sgn * face_j.x, sgn * face_j.y, face_j.z, face_j.w, gm1);
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
          xq[o] = q;
          xw[o] = w;
          xd[o] = dq;
          xf[o] = fs;
          dq_case[size_t(d) * nj + j] = dq;
          pq = q;
          pw = w;
          pd = dq;
          pfw = fw;
        }
        __syncthreads();
      }
      if (cc + 2 < nchunks) {
        // The buffer is free: order this CTA's reads of it before the next
        // asynchronous write into it.
        fence_proxy_async();
        __syncthreads();
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

// applyImplicitUpdate (src/engine-cpu/euler2d.ts:816-847) for every cell of
// every active case: Q += alpha dQ with alpha halved until density and
// pressure stay within a factor of two; flags non-physical results.
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
  if (i < ni && j < nj) {
    const R gamma = R(cd.gamma);
    const int64_t k = cd.cell + i + int64_t(j) * ni;
    const Cons<R> q0 = q.load(k);
    const float4 d4 = dq[cd.skew + skew_slot(i, j, nj)];
    const R p0 = pressure_of(q0.rho, q0.mu, q0.mv, q0.e, gamma);
    const R d0 = R(d4.x), d1 = R(d4.y), d2 = R(d4.z), d3 = R(d4.w);
    R alpha = R(1);
    for (int tries = 0; tries < 30; tries++) {
      const R rho1 = q0.rho + alpha * d0;
      const R p1 = pressure_of(rho1, q0.mu + alpha * d1, q0.mv + alpha * d2, q0.e + alpha * d3, gamma);
      if (rho1 > R(0.5) * q0.rho && rho1 < R(2) * q0.rho && p1 > R(0.5) * p0 && p1 < R(2) * p0) break;
      alpha *= R(0.5);
    }
    const Cons<R> q1{q0.rho + alpha * d0, q0.mu + alpha * d1, q0.mv + alpha * d2, q0.e + alpha * d3};
    q.store(k, q1);
    bad = !is_physical(q1, gamma);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&status[c], STATUS_NON_PHYSICAL);
}

// Diagonals per bulk copy for a case of `nj` rows: the largest of 8, 6, 4,
// 3, 2, 1 whose shared memory fits one CTA.
inline int sweep_chunk(int nt, int nj) {
  constexpr size_t kLimit = 200 * 1024;
  for (int k : {8, 6, 4, 3, 2, 1})
    if (sweep_smem_bytes(nt, nj, k) <= kLimit) return k;
  return 0;
}

inline cudaError_t launch_sweep(SweepArgs A, int n_cases, int max_nj, cudaStream_t stream) {
  const int nt = ((max_nj + 31) / 32) * 32;
  A.chunk = sweep_chunk(nt, max_nj);
  if (A.chunk == 0) return cudaErrorInvalidConfiguration;
  A.wait_limit = 1 << 22;
  const size_t bytes = sweep_smem_bytes(nt, max_nj, A.chunk);
  const cudaError_t e = cudaFuncSetAttribute(lusgs_sweep_kernel,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
  if (e != cudaSuccess) return e;
  lusgs_sweep_kernel<<<n_cases, nt, bytes, stream>>>(A);
  return cudaGetLastError();
}

}  // namespace bsd
