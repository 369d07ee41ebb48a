// BF16 GEMMs on the fifth-generation tensor cores (tcgen05, sm_100a) for the
// learned warm start's MLP.
//
// C (M x N) = A (M x K) . B (N x K)^T, both operands bf16 and K-major (each
// row's K elements contiguous), FP32 accumulation in tensor memory (TMEM).
// One CTA computes a 128 x BN tile of C (BN = 64, 128 or 256) over a range of
// K, in chunks of 64 (one 128-byte swizzle atom of bf16):
//   - warp 0, one lane: TMA tile loads (cp.async.bulk.tensor.2d, no
//     multicast) of A (128 x 64) and B (BN x 64) into a four-stage ring of
//     shared memory, 128-byte swizzled;
//   - warp 1, one lane: four tcgen05.mma (M 128, N BN, K 16) per chunk,
//     accumulating in TMEM; tcgen05.commit frees the ring stage, and after
//     the last chunk signals the epilogue;
//   - all four warps: the epilogue reads the accumulator (tcgen05.ld, warp w
//     owns TMEM lanes = tile rows 32w..32w+31) and applies `Epi`.
// Every mbarrier wait is bounded; a wait that gives up sets *error and the
// CTA still releases its TMEM and waits (bounded) for its own copies and
// MMAs before it returns.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace bsd {
namespace umma {

constexpr int kBM = 128;     // rows of C per CTA (the MMA's M)
constexpr int kBK = 64;      // K per ring stage: one 128-byte swizzle atom of bf16
constexpr int kStages = 4;
constexpr int kThreads = 128;
constexpr int kWaitLimit = 1 << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---- mbarriers -------------------------------------------------------------
__device__ __forceinline__ void bar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void bar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void bar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool bar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity) {
  for (int k = 0; k < kWaitLimit; k++)
    if (bar_try_wait(bar, parity)) return true;
  return false;
}

// ---- TMA --------------------------------------------------------------------
// A 2D tile of `map` at (c0 = inner coordinate, c1) into shared memory,
// completing `bar`'s transaction count. c0 is always a multiple of 64
// elements here (128 bytes), so the copy starts on a 16-byte boundary.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int c0, int c1, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
          smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_addr(bar))
      : "memory");
}

// ---- tcgen05 ----------------------------------------------------------------
// Shared-memory matrix descriptor of a K-major operand tile in the canonical
// 128-byte-swizzled layout: rows of 128 bytes, 8-row groups 1024 bytes apart
// (stride byte offset), descriptor version 1, layout type SWIZZLE_128B.
__device__ __forceinline__ uint64_t desc_k_sw128(uint32_t saddr) {
  return uint64_t((saddr >> 4) & 0x3FFFu) | (uint64_t(1) << 16) | (uint64_t(1024 >> 4) << 32) |
         (uint64_t(1) << 46) | (uint64_t(2) << 61);
}
// Instruction descriptor: FP32 accumulator, BF16 A and B, both K-major,
// M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(n >> 3) << 17) | (uint32_t(kBM >> 4) << 24);
}
__device__ __forceinline__ void mma_bf16(uint32_t tmem_c, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_c),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t cols) {  // one full warp
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_addr(dst)),
               "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t cols) {  // the allocating warp
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(cols) : "memory");
}
// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; k++) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ bool ld_error(const int* error) { return *reinterpret_cast<const volatile int*>(error) != 0; }

template <int BN>
__host__ __device__ constexpr size_t gemm_smem_bytes() {
  // 1024-byte alignment slack, the ring, then barriers and the TMEM address.
  return 1024 + size_t(kStages) * (kBM + BN) * kBK * 2 + 256;
}

// C tile rows [m0, m0 + 128) x columns [n0, n0 + BN), K chunks [kc0, kc1).
// `Epi::apply(row, col, v)` receives 16 consecutive columns of one row
// (rows at or beyond m are not passed).
template <int BN, class Epi>
__global__ void __launch_bounds__(kThreads, 1)
    gemm_bf16_tn(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b, int m,
                 int k_chunks_per_split, int k_chunks, Epi epi, int* error) {
  static_assert(BN == 64 || BN == 128 || BN == 256, "tile width");
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  constexpr uint32_t kABytes = kBM * kBK * 2, kBBytes = BN * kBK * 2;
  unsigned char* ring = base;  // stage s: A at s (A + B) bytes, B after it; 1024-byte aligned
  uint64_t* full = reinterpret_cast<uint64_t*>(base + kStages * (kABytes + kBBytes));
  uint64_t* empty = full + kStages;
  uint64_t* accum = empty + kStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accum + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;
  const int kc0 = blockIdx.z * k_chunks_per_split;
  const int nk = min(k_chunks, kc0 + k_chunks_per_split) - kc0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; s++) {
      bar_init(&full[s], 1);
      bar_init(&empty[s], 1);
    }
    bar_init(accum, 1);
    bar_fence_init();
  }
  if (warp == 0) tmem_alloc(tmem_slot, BN);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  bool bad = false;

  uint32_t* issued = tmem_slot + 1;  // [kStages] fills issued per stage (producer)
  if (threadIdx.x < kStages) issued[threadIdx.x] = 0;
  __syncthreads();
  if (nk > 0) {
    if (warp == 0 && lane == 0) {
      // Producer.
      for (int kc = 0; kc < nk && !bad; kc++) {
        const int s = kc % kStages;
        if (kc >= kStages && !bar_wait(&empty[s], uint32_t((kc / kStages - 1) & 1))) {
          bad = true;
          break;
        }
        unsigned char* a = ring + size_t(s) * (kABytes + kBBytes);
        bar_expect_tx(&full[s], kABytes + kBBytes);
        tma_load_2d(a, &map_a, (kc0 + kc) * kBK, m0, &full[s]);
        tma_load_2d(a + kABytes, &map_b, (kc0 + kc) * kBK, n0, &full[s]);
        issued[s]++;
      }
    } else if (warp == 1 && lane == 0) {
      // MMA issue.
      constexpr uint32_t idesc = idesc_bf16(BN);
      int kc = 0;
      for (; kc < nk; kc++) {
        const int s = kc % kStages;
        if (!bar_wait(&full[s], uint32_t((kc / kStages) & 1))) {
          bad = true;
          break;
        }
        fence_after_sync();
        const uint32_t a = smem_addr(ring + size_t(s) * (kABytes + kBBytes));
        const uint64_t da = desc_k_sw128(a), db = desc_k_sw128(a + kABytes);
#pragma unroll
        for (int kk = 0; kk < kBK / 16; kk++)  // 16 bf16 = 32 bytes = 2 descriptor units
          mma_bf16(tmem, da + 2 * kk, db + 2 * kk, idesc, (kc > 0 || kk > 0) ? 1u : 0u);
        mma_commit(&empty[s]);
      }
      // Signals the epilogue once every MMA issued has completed.
      mma_commit(accum);
    }
    __syncwarp();
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicExch(error, 1);

    // Epilogue (tcgen05.ld is warp-wide: the warp agrees on going ahead).
    const bool ready = __all_sync(0xffffffffu, bar_wait(accum, 0));
    if (!ready && lane == 0) atomicExch(error, 1);
    fence_after_sync();
    const int row = m0 + warp * 32 + lane;
    const uint32_t t_lane = tmem + (uint32_t(warp * 32) << 16);
    if (ready) {
#pragma unroll 1
      for (int c = 0; c < BN; c += 16) {
        float v[16];
        tmem_ld16(t_lane + uint32_t(c), v);
        if (row < m) epi.apply(row, n0 + c, v);
      }
    }
  }
  // After a failure, the last copy into each stage lands (bounded) before
  // the CTA leaves.
  fence_before_sync();
  __syncthreads();
  if (threadIdx.x == 0 && ld_error(error))
    for (int s = 0; s < kStages; s++)
      if (issued[s] > 0) bar_wait(&full[s], (issued[s] - 1) & 1u);
  if (warp == 0) {
    fence_after_sync();
    tmem_free(tmem, BN);
  }
}

// ---- epilogues ----------------------------------------------------------------
__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  const float cdf = 0.5f * (1.f + erff(z * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * __expf(-0.5f * z * z);
  return cdf + z * pdf;
}

// C = A B^T stored as FP32 (row stride ldc).
struct EpiStoreF32 {
  float* c;
  int ldc;
  __device__ void apply(int row, int col, const float* v) const {
    float4* p = reinterpret_cast<float4*>(c + size_t(row) * ldc + col);
#pragma unroll
    for (int k = 0; k < 4; k++) p[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
  }
};

// C += A B^T (FP32 atomics; the split-K weight gradients).
struct EpiAtomicF32 {
  float* c;
  int ldc;
  __device__ void apply(int row, int col, const float* v) const {
    float* p = c + size_t(row) * ldc + col;
#pragma unroll
    for (int k = 0; k < 16; k++) atomicAdd(p + k, v[k]);
  }
};

// Hidden layer forward: z = A B^T + bias; h = gelu(z). Stores z and h
// (bf16, row stride ld) and h transposed (bf16, column j at ht + j ldt).
struct EpiBiasGelu {
  const float* bias;
  __nv_bfloat16* z;
  __nv_bfloat16* h;
  __nv_bfloat16* ht;
  int ld, ldt;
  __device__ void apply(int row, int col, const float* v) const {
    __nv_bfloat16 zb[16], hb[16];
#pragma unroll
    for (int k = 0; k < 16; k++) {
      const float zz = v[k] + bias[col + k];
      zb[k] = __float2bfloat16_rn(zz);
      hb[k] = __float2bfloat16_rn(gelu(zz));
      ht[size_t(col + k) * ldt + row] = hb[k];
    }
    uint4* pz = reinterpret_cast<uint4*>(z + size_t(row) * ld + col);
    uint4* ph = reinterpret_cast<uint4*>(h + size_t(row) * ld + col);
    pz[0] = *reinterpret_cast<const uint4*>(zb);
    pz[1] = *reinterpret_cast<const uint4*>(zb + 8);
    ph[0] = *reinterpret_cast<const uint4*>(hb);
    ph[1] = *reinterpret_cast<const uint4*>(hb + 8);
  }
};

// Output layer forward: y = A B^T + bias, FP32.
struct EpiBiasF32 {
  const float* bias;
  float* y;
  int ld;
  __device__ void apply(int row, int col, const float* v) const {
    float4* p = reinterpret_cast<float4*>(y + size_t(row) * ld + col);
#pragma unroll
    for (int k = 0; k < 4; k++)
      p[k] = make_float4(v[4 * k] + bias[col + 4 * k], v[4 * k + 1] + bias[col + 4 * k + 1],
                         v[4 * k + 2] + bias[col + 4 * k + 2], v[4 * k + 3] + bias[col + 4 * k + 3]);
  }
};

// Hidden layer backward: dz = (dL/dh = A B^T) gelu'(z). Stores dz (bf16, row
// stride ld) and dz transposed (column j at dzt + j ldt).
struct EpiGeluGrad {
  const __nv_bfloat16* z;
  __nv_bfloat16* dz;
  __nv_bfloat16* dzt;
  int ld, ldt;
  __device__ void apply(int row, int col, const float* v) const {
    __nv_bfloat16 zb[16], db[16];
    const uint4* pz = reinterpret_cast<const uint4*>(z + size_t(row) * ld + col);
    *reinterpret_cast<uint4*>(zb) = pz[0];
    *reinterpret_cast<uint4*>(zb + 8) = pz[1];
#pragma unroll
    for (int k = 0; k < 16; k++) {
      db[k] = __float2bfloat16_rn(v[k] * gelu_grad(__bfloat162float(zb[k])));
      dzt[size_t(col + k) * ldt + row] = db[k];
    }
    uint4* pd = reinterpret_cast<uint4*>(dz + size_t(row) * ld + col);
    pd[0] = *reinterpret_cast<const uint4*>(db);
    pd[1] = *reinterpret_cast<const uint4*>(db + 8);
  }
};

}  // namespace umma
}  // namespace bsd
