// The learned warm start's network on the tensor cores: tensor maps and
// launches of the tcgen05 GEMMs (device/umma.cuh), and their C entry points.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "bowshock.h"
#include "common.hpp"
#include "device/umma.cuh"

#define BS_TRY_ST(expr)              \
  do {                               \
    const bs_status s_ = (expr);     \
    if (s_ != BS_OK) return s_;      \
  } while (0)

namespace bsm {

using bsd::umma::kBK;
using bsd::umma::kBM;

// cuTensorMapEncodeTiled from the driver, found through the runtime (the
// library does not link the driver library itself).
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// The tensor map of a row-major bf16 matrix (rows x cols, cols contiguous)
// read in tiles of box_rows x 64, 128-byte swizzled; rows past the end read
// as zero.
bs_status make_map(CUtensorMap* map, const void* ptr, int64_t rows, int64_t cols, int box_rows) {
  auto fn = encode_fn();
  if (fn == nullptr) return bs::fail(BS_EXECUTION, "cuTensorMapEncodeTiled is not available");
  if (cols % kBK != 0 || (reinterpret_cast<uintptr_t>(ptr) & 15) != 0)
    return bs::fail(BS_INVALID_ARGUMENT, "a GEMM operand needs 16-byte alignment and K a multiple of 64");
  const cuuint64_t dims[2] = {cuuint64_t(cols), cuuint64_t(rows)};
  const cuuint64_t strides[1] = {cuuint64_t(cols) * 2};
  const cuuint32_t box[2] = {cuuint32_t(kBK), cuuint32_t(box_rows)};
  const cuuint32_t elem[2] = {1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box,
                        elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return bs::fail(BS_EXECUTION, "cuTensorMapEncodeTiled failed: " + std::to_string(int(r)));
  return BS_OK;
}

// C (m x n) from A (m x k, map a) and B (n x k, map b) with epilogue `epi`,
// K split over `splits` CTAs per tile. n must be a multiple of BN and k of 64.
template <int BN, class Epi>
bs_status gemm(const CUtensorMap& a, const CUtensorMap& b, int m, int n, int k, int splits, const Epi& epi,
               int* error, cudaStream_t stream) {
  if (m <= 0 || n % BN != 0 || k % kBK != 0 || k <= 0 || splits < 1)
    return bs::fail(BS_INVALID_ARGUMENT, "GEMM shape: n a multiple of the tile, k of 64");
  constexpr size_t bytes = bsd::umma::gemm_smem_bytes<BN>();
  static_assert(bytes <= 227 * 1024, "GEMM shared memory");
  auto kernel = bsd::umma::gemm_bf16_tn<BN, Epi>;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
  if (e != cudaSuccess) return bs::fail(BS_EXECUTION, std::string("GEMM attribute: ") + cudaGetErrorString(e));
  const int k_chunks = k / kBK;
  const int per_split = (k_chunks + splits - 1) / splits;
  const dim3 grid((m + kBM - 1) / kBM, n / BN, (k_chunks + per_split - 1) / per_split);
  kernel<<<grid, bsd::umma::kThreads, bytes, stream>>>(a, b, m, per_split, k_chunks, epi, error);
  e = cudaGetLastError();
  if (e != cudaSuccess) return bs::fail(BS_EXECUTION, std::string("GEMM launch: ") + cudaGetErrorString(e));
  return BS_OK;
}

template <class Epi>
bs_status gemm_any(const void* a, const void* b, int m, int n, int k, int splits, const Epi& epi, int* error,
                   cudaStream_t stream) {
  const int bn = n % 256 == 0 ? 256 : n % 128 == 0 ? 128 : n % 64 == 0 ? 64 : 0;
  if (bn == 0) return bs::fail(BS_INVALID_ARGUMENT, "GEMM n must be a multiple of 64");
  CUtensorMap ma, mb;
  BS_TRY_ST(make_map(&ma, a, m, k, kBM));
  BS_TRY_ST(make_map(&mb, b, n, k, bn));
  if (bn == 256) return gemm<256>(ma, mb, m, n, k, splits, epi, error, stream);
  if (bn == 128) return gemm<128>(ma, mb, m, n, k, splits, epi, error, stream);
  return gemm<64>(ma, mb, m, n, k, splits, epi, error, stream);
}


// ---- the warm-start network ---------------------------------------------------
//
// Per sample (one grid cell of one case) the input is 10 floats: the cell
// centroid (x, r) in body diameters and 8 case values (nose family one-hot
// over 5 families, fineness / 5, body length / 8, Mach / 5). The features
// are (x / 8, r / 4), the 8 case values, and sin and cos of pi 2^(7k/15) x/8
// and of pi 2^(7k/15) r/4 for k = 0..15: 74 values, padded with zeros to
// kFeatures. The output is 4 values per sample, (log rho, u / u_inf,
// v / u_inf, log p) against the free stream; the last layer is padded to
// kOutPad outputs whose weights stay zero.
constexpr int kInputs = 10;
constexpr int kTargets = 4;
constexpr int kFeatures = 128;
constexpr int kOutPad = 128;
constexpr int kFreq = 16;

__device__ __forceinline__ void sample_features(const float* in, float* f) {
  const float x = in[0] * 0.125f, r = in[1] * 0.25f;
  f[0] = x;
  f[1] = r;
#pragma unroll
  for (int k = 0; k < 8; k++) f[2 + k] = in[2 + k];
#pragma unroll
  for (int k = 0; k < kFreq; k++) {
    const float w = 3.14159265358979f * exp2f(float(7 * k) / 15.f);
    float sx, cx, sr, cr;
    sincosf(w * x, &sx, &cx);
    sincosf(w * r, &sr, &cr);
    f[10 + 4 * k] = sx;
    f[11 + 4 * k] = cx;
    f[12 + 4 * k] = sr;
    f[13 + 4 * k] = cr;
  }
#pragma unroll
  for (int k = 10 + 4 * kFreq; k < kFeatures; k++) f[k] = 0.f;
}

// A stateless 64-bit mix (SplitMix64's finaliser) for sampling.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Row `row` of the batch: sample `idx` (random when `seed` != 0, else row
// `first + row`) of the data set; its features (row-major and transposed,
// bf16) and, when wanted, its targets. Rows at or past `m_valid` are zero.
__global__ void mlp_gather(const float* inputs, const float* targets, int64_t n, int64_t first, int M, int m_valid,
                           uint64_t seed, __nv_bfloat16* x0, __nv_bfloat16* x0t, float* tgt) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= M) return;
  float f[kFeatures];
  float t[kTargets] = {0.f, 0.f, 0.f, 0.f};
  if (row < m_valid) {
    const int64_t idx = seed != 0 ? int64_t(mix64(seed ^ (uint64_t(row) * 0xD1B54A32D192ED03ull)) % uint64_t(n))
                                  : first + row;
    sample_features(inputs + idx * kInputs, f);
    if (targets != nullptr)
      for (int c = 0; c < kTargets; c++) t[c] = targets[idx * kTargets + c];
  } else {
    for (int k = 0; k < kFeatures; k++) f[k] = 0.f;
  }
  __nv_bfloat16* xr = x0 + size_t(row) * kFeatures;
#pragma unroll
  for (int k = 0; k < kFeatures; k++) {
    const __nv_bfloat16 b = __float2bfloat16_rn(f[k]);
    xr[k] = b;
    x0t[size_t(k) * M + row] = b;
  }
  if (tgt != nullptr)
    for (int c = 0; c < kTargets; c++) tgt[size_t(row) * kTargets + c] = t[c];
}

// Mean squared error over the first 4 outputs of rows < m_valid, and its
// gradient with respect to the (padded) output, bf16, row-major and
// transposed. The loss is added to *loss.
__global__ void mlp_loss(const float* y, const float* tgt, int M, int m_valid, __nv_bfloat16* dy,
                         __nv_bfloat16* dyt, float* loss) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  float part = 0.f;
  if (row < M) {
    const float scale = 2.f / float(kTargets * m_valid);
    for (int c = 0; c < kOutPad; c++) {
      float g = 0.f;
      if (c < kTargets && row < m_valid) {
        const float d = y[size_t(row) * kOutPad + c] - tgt[size_t(row) * kTargets + c];
        part += d * d;
        g = scale * d;
      }
      const __nv_bfloat16 b = __float2bfloat16_rn(g);
      dy[size_t(row) * kOutPad + c] = b;
      dyt[size_t(c) * M + row] = b;
    }
  }
  for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
  if ((threadIdx.x & 31) == 0 && part != 0.f) atomicAdd(loss, part / float(kTargets * m_valid));
}

// gb[j] = sum over the batch of dz (given transposed: row j contiguous).
__global__ void mlp_bias_grad(const __nv_bfloat16* dzt, int M, float* gb) {
  const __nv_bfloat16* p = dzt + size_t(blockIdx.x) * M;
  float s = 0.f;
  for (int k = threadIdx.x; k < M; k += blockDim.x) s += __bfloat162float(p[k]);
  __shared__ float red[32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.f;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) gb[blockIdx.x] = s;
  }
}

// One Adam step (bias-corrected) of an out x in weight block (in = 1 for a
// bias); the bf16 copies are rewritten, row-major and transposed; rows at or
// past `out_valid` stay zero; the gradient is cleared.
__global__ void mlp_adam(float* w, float* g, float* m, float* v, int out, int in, int out_valid,
                         __nv_bfloat16* wb, __nv_bfloat16* wt, float lr, float c1, float c2) {
  const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= int64_t(out) * in) return;
  const int o = int(k / in), i = int(k % in);
  float wk = w[k];
  if (o < out_valid) {
    const float gk = g[k];
    const float mk = 0.9f * m[k] + 0.1f * gk;
    const float vk = 0.999f * v[k] + 0.001f * gk * gk;
    m[k] = mk;
    v[k] = vk;
    wk -= lr * (mk * c1) / (sqrtf(vk * c2) + 1e-8f);
    w[k] = wk;
  }
  g[k] = 0.f;
  if (wb != nullptr) {
    const __nv_bfloat16 b = __float2bfloat16_rn(wk);
    wb[k] = b;
    wt[size_t(i) * out + o] = b;
  }
}

// fp32 master weights to their bf16 copies (row-major and transposed).
__global__ void mlp_round_weights(const float* w, int out, int in, __nv_bfloat16* wb, __nv_bfloat16* wt) {
  const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= int64_t(out) * in) return;
  const int o = int(k / in), i = int(k % in);
  const __nv_bfloat16 b = __float2bfloat16_rn(w[k]);
  wb[k] = b;
  wt[size_t(i) * out + o] = b;
}

template <class T>
struct Buf {
  T* p = nullptr;
  size_t n = 0;
  Buf() = default;
  Buf(const Buf&) = delete;
  Buf& operator=(const Buf&) = delete;
  ~Buf() {
    if (p != nullptr) cudaFree(p);
  }
  cudaError_t alloc(size_t count) {
    n = count;
    const cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), std::max<size_t>(count, 1) * sizeof(T));
    if (e == cudaSuccess) cudaMemset(p, 0, std::max<size_t>(count, 1) * sizeof(T));
    return e;
  }
};

#define MLP_CUDA(expr)                                                                   \
  do {                                                                                   \
    const cudaError_t e_ = (expr);                                                       \
    if (e_ != cudaSuccess) return bs::fail(BS_EXECUTION, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

using bf16 = __nv_bfloat16;

struct Layer {
  int in = 0, out = 0, out_valid = 0;
  Buf<float> w, b, gw, gb, mw, vw, mb, vb;
  Buf<bf16> wb, wt;
  CUtensorMap map_w, map_wt;  // B operands: W (out x in) and W^T (in x out)
};

inline int tile_n(int n) { return n % 256 == 0 ? 256 : n % 128 == 0 ? 128 : 64; }

// The network, its Adam state, its batch buffers and its data set.
class Mlp {
 public:
  int hidden = 0, width = 0, M = 0;
  std::vector<std::unique_ptr<Layer>> layers;  // hidden + 1
  Buf<bf16> x0, x0t, dy, dyt;
  std::vector<std::unique_ptr<Buf<bf16>>> z, h, ht, dz, dzt;  // per hidden layer
  Buf<float> y, tgt, loss;
  Buf<int> err;
  Buf<float> data_in, data_tgt;
  int64_t n_data = 0;
  int steps_done = 0;
  CUtensorMap map_x0, map_x0t, map_dy, map_dyt;
  std::vector<CUtensorMap> map_h, map_ht, map_dz, map_dzt;
  cudaStream_t stream = nullptr;

  ~Mlp() {
    if (stream != nullptr) cudaStreamDestroy(stream);
  }

  bs_status init(int hidden_layers, int w, int batch, uint64_t seed) {
    hidden = hidden_layers;
    width = w;
    M = batch;
    MLP_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    for (int l = 0; l <= hidden; l++) {
      auto L = std::make_unique<Layer>();
      L->in = l == 0 ? kFeatures : width;
      L->out = l == hidden ? kOutPad : width;
      L->out_valid = l == hidden ? kTargets : width;
      const size_t nw = size_t(L->in) * L->out;
      MLP_CUDA(L->w.alloc(nw));
      MLP_CUDA(L->gw.alloc(nw));
      MLP_CUDA(L->mw.alloc(nw));
      MLP_CUDA(L->vw.alloc(nw));
      MLP_CUDA(L->b.alloc(L->out));
      MLP_CUDA(L->gb.alloc(L->out));
      MLP_CUDA(L->mb.alloc(L->out));
      MLP_CUDA(L->vb.alloc(L->out));
      MLP_CUDA(L->wb.alloc(nw));
      MLP_CUDA(L->wt.alloc(nw));
      // He initialisation (GELU layers), a tenth of it for the output layer;
      // zero biases and zero padded outputs.
      std::vector<float> hw(nw, 0.f);
      const float sd = std::sqrt(2.f / float(L->in)) * (l == hidden ? 0.1f : 1.f);
      uint64_t st = mix64(seed + 0x1000 * uint64_t(l + 1));
      for (int o = 0; o < L->out_valid; o++)
        for (int i = 0; i < L->in; i++) {
          st = mix64(st);
          const double u1 = (double(st >> 11) + 0.5) * (1.0 / 9007199254740992.0);
          st = mix64(st);
          const double u2 = double(st >> 11) * (1.0 / 9007199254740992.0);
          hw[size_t(o) * L->in + i] = float(sd * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2));
        }
      MLP_CUDA(cudaMemcpy(L->w.p, hw.data(), nw * sizeof(float), cudaMemcpyHostToDevice));
      BS_TRY_ST(make_map(&L->map_w, L->wb.p, L->out, L->in, tile_n(L->out)));
      BS_TRY_ST(make_map(&L->map_wt, L->wt.p, L->in, L->out, tile_n(L->in)));
      layers.push_back(std::move(L));
    }
    MLP_CUDA(x0.alloc(size_t(M) * kFeatures));
    MLP_CUDA(x0t.alloc(size_t(M) * kFeatures));
    MLP_CUDA(dy.alloc(size_t(M) * kOutPad));
    MLP_CUDA(dyt.alloc(size_t(M) * kOutPad));
    MLP_CUDA(y.alloc(size_t(M) * kOutPad));
    MLP_CUDA(tgt.alloc(size_t(M) * kTargets));
    MLP_CUDA(loss.alloc(1));
    MLP_CUDA(err.alloc(1));
    BS_TRY_ST(make_map(&map_x0, x0.p, M, kFeatures, kBM));
    BS_TRY_ST(make_map(&map_x0t, x0t.p, kFeatures, M, tile_n(kFeatures)));
    BS_TRY_ST(make_map(&map_dy, dy.p, M, kOutPad, kBM));
    BS_TRY_ST(make_map(&map_dyt, dyt.p, kOutPad, M, kBM));
    for (int l = 0; l < hidden; l++) {
      for (auto* v : {&z, &h, &ht, &dz, &dzt}) {
        v->push_back(std::make_unique<Buf<bf16>>());
        MLP_CUDA(v->back()->alloc(size_t(M) * width));
      }
      map_h.emplace_back();
      map_ht.emplace_back();
      map_dz.emplace_back();
      map_dzt.emplace_back();
      BS_TRY_ST(make_map(&map_h.back(), h[l]->p, M, width, kBM));
      BS_TRY_ST(make_map(&map_ht.back(), ht[l]->p, width, M, tile_n(width)));
      BS_TRY_ST(make_map(&map_dz.back(), dz[l]->p, M, width, kBM));
      BS_TRY_ST(make_map(&map_dzt.back(), dzt[l]->p, width, M, kBM));
    }
    return round_weights();
  }

  bs_status round_weights() {
    for (auto& L : layers) {
      const int64_t nw = int64_t(L->in) * L->out;
      mlp_round_weights<<<unsigned((nw + 255) / 256), 256, 0, stream>>>(L->w.p, L->out, L->in, L->wb.p, L->wt.p);
    }
    MLP_CUDA(cudaGetLastError());
    return BS_OK;
  }

  // Forward pass over the whole batch in x0 (rows past the samples are zero
  // features; every row is computed so that no stale row reaches a
  // gradient).
  bs_status forward() {
    using namespace bsd::umma;
    for (int l = 0; l <= hidden; l++) {
      Layer& L = *layers[l];
      const CUtensorMap& a = l == 0 ? map_x0 : map_h[l - 1];
      if (l < hidden) {
        const EpiBiasGelu epi{L.b.p, z[l]->p, h[l]->p, ht[l]->p, width, M};
        BS_TRY_ST(gemm<256>(a, L.map_w, M, L.out, L.in, 1, epi, err.p, stream));
      } else {
        const EpiBiasF32 epi{L.b.p, y.p, kOutPad};
        BS_TRY_ST(gemm<128>(a, L.map_w, M, L.out, L.in, 1, epi, err.p, stream));
      }
    }
    return BS_OK;
  }

  // Loss of the first m_valid rows of the batch (targets in tgt), added to
  // *loss_slot, and the gradients of every parameter (added to gw and gb,
  // which the caller has cleared). Rows past m_valid get a zero gradient.
  bs_status backward(int m_valid, float* loss_slot) {
    using namespace bsd::umma;
    mlp_loss<<<(M + 255) / 256, 256, 0, stream>>>(y.p, tgt.p, M, m_valid, dy.p, dyt.p, loss_slot);
    MLP_CUDA(cudaGetLastError());
    const int splits = std::max(1, M / (kBK * 4));  // four K chunks per CTA
    for (int l = hidden; l >= 0; l--) {
      Layer& L = *layers[l];
      // This layer's output gradient dz (M x out), transposed in gzt.
      const CUtensorMap& gzt = l == hidden ? map_dyt : map_dzt[l];
      const bf16* gzt_p = l == hidden ? dyt.p : dzt[l]->p;
      const CUtensorMap& xin_t = l == 0 ? map_x0t : map_ht[l - 1];
      // dW (out x in) += dz^T x, over the batch (split K).
      const EpiAtomicF32 gw{L.gw.p, L.in};
      if (L.in % 256 == 0)
        BS_TRY_ST(gemm<256>(gzt, xin_t, L.out, L.in, M, splits, gw, err.p, stream));
      else
        BS_TRY_ST(gemm<128>(gzt, xin_t, L.out, L.in, M, splits, gw, err.p, stream));
      mlp_bias_grad<<<L.out, 256, 0, stream>>>(gzt_p, M, L.gb.p);
      MLP_CUDA(cudaGetLastError());
      if (l > 0) {
        // dz of the layer below: (dz W) gelu'(z_below).
        const CUtensorMap& gz = l == hidden ? map_dy : map_dz[l];
        const EpiGeluGrad epi{z[l - 1]->p, dz[l - 1]->p, dzt[l - 1]->p, width, M};
        BS_TRY_ST(gemm<256>(gz, L.map_wt, M, L.in, L.out, 1, epi, err.p, stream));
      }
    }
    return BS_OK;
  }

  bs_status adam(float lr) {
    steps_done++;
    const float c1 = 1.f / (1.f - std::pow(0.9f, float(steps_done)));
    const float c2 = 1.f / (1.f - std::pow(0.999f, float(steps_done)));
    for (auto& Lp : layers) {
      Layer& L = *Lp;
      const int64_t nw = int64_t(L.in) * L.out;
      mlp_adam<<<unsigned((nw + 255) / 256), 256, 0, stream>>>(L.w.p, L.gw.p, L.mw.p, L.vw.p, L.out, L.in,
                                                               L.out_valid, L.wb.p, L.wt.p, lr, c1, c2);
      mlp_adam<<<unsigned((L.out + 255) / 256), 256, 0, stream>>>(L.b.p, L.gb.p, L.mb.p, L.vb.p, L.out, 1,
                                                                  L.out_valid, nullptr, nullptr, lr, c1, c2);
    }
    MLP_CUDA(cudaGetLastError());
    return BS_OK;
  }

  bs_status clear_grads() {
    for (auto& L : layers) {
      MLP_CUDA(cudaMemsetAsync(L->gw.p, 0, L->gw.n * sizeof(float), stream));
      MLP_CUDA(cudaMemsetAsync(L->gb.p, 0, L->gb.n * sizeof(float), stream));
    }
    return BS_OK;
  }

  bs_status check_error() {
    int h = 0;
    MLP_CUDA(cudaMemcpyAsync(&h, err.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
    MLP_CUDA(cudaStreamSynchronize(stream));
    if (h != 0) return bs::fail(BS_EXECUTION, "warm-start network: a GEMM pipeline wait timed out");
    return BS_OK;
  }

  int64_t param_count() const {
    int64_t n = 0;
    for (auto& L : layers) n += int64_t(L->in) * L->out + L->out;
    return n;
  }
};
}  // namespace bsm

struct bs_mlp {
  bsm::Mlp net;
  std::atomic<bool> busy{false};
};

namespace {

// One call at a time per network (BS_BUSY otherwise), as for engines.
class MlpGuard {
 public:
  explicit MlpGuard(bs_mlp* m) : m_(m) {
    bool expected = false;
    ok_ = m_ != nullptr && m_->busy.compare_exchange_strong(expected, true);
  }
  ~MlpGuard() {
    if (ok_) m_->busy.store(false);
  }
  bool ok() const { return ok_; }

 private:
  bs_mlp* m_;
  bool ok_ = false;
};

#define MLP_GUARD(m)                                                                  \
  if ((m) == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null network");           \
  MlpGuard guard_(m);                                                                 \
  if (!guard_.ok()) return bs::fail(BS_BUSY, "the network is running another call")

// Uploads n samples (and targets when given) into temporary device arrays.
bs_status upload(const float* in, const float* tgt, int64_t n, bsm::Buf<float>* din, bsm::Buf<float>* dtgt) {
  MLP_CUDA(din->alloc(size_t(n) * bsm::kInputs));
  MLP_CUDA(cudaMemcpy(din->p, in, size_t(n) * bsm::kInputs * sizeof(float), cudaMemcpyHostToDevice));
  if (tgt != nullptr) {
    MLP_CUDA(dtgt->alloc(size_t(n) * bsm::kTargets));
    MLP_CUDA(cudaMemcpy(dtgt->p, tgt, size_t(n) * bsm::kTargets * sizeof(float), cudaMemcpyHostToDevice));
  }
  return BS_OK;
}

}  // namespace

extern "C" {

bs_status bs_gemm_bf16(const void* a, const void* b, float* c, int32_t m, int32_t n, int32_t k, int32_t splits,
                       int32_t accumulate, void* stream) {
  if (a == nullptr || b == nullptr || c == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null pointer");
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  int* d_err = nullptr;
  // Test entry point: a small error word of its own.
  if (cudaMallocAsync(&d_err, sizeof(int), st) != cudaSuccess) return bs::fail(BS_MEMORY_LIMIT, "error word");
  cudaMemsetAsync(d_err, 0, sizeof(int), st);
  bs_status s;
  if (accumulate != 0)
    s = bsm::gemm_any(a, b, m, n, k, splits, bsd::umma::EpiAtomicF32{c, n}, d_err, st);
  else if (splits != 1)
    s = bs::fail(BS_INVALID_ARGUMENT, "split K needs accumulate");
  else
    s = bsm::gemm_any(a, b, m, n, k, 1, bsd::umma::EpiStoreF32{c, n}, d_err, st);
  int h_err = 0;
  cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(d_err, st);
  const cudaError_t e = cudaStreamSynchronize(st);
  if (s != BS_OK) return s;
  if (e != cudaSuccess) return bs::fail(BS_EXECUTION, std::string("GEMM: ") + cudaGetErrorString(e));
  if (h_err != 0) return bs::fail(BS_EXECUTION, "GEMM: a pipeline wait timed out");
  return BS_OK;
}

bs_status bs_gemm_bf16_time(const void* a, const void* b, float* c, int32_t m, int32_t n, int32_t k,
                            int32_t iterations, float* ms) {
  if (a == nullptr || b == nullptr || c == nullptr || ms == nullptr || iterations < 1)
    return bs::fail(BS_INVALID_ARGUMENT, "null pointer or no iterations");
  const int bn = n % 256 == 0 ? 256 : n % 128 == 0 ? 128 : n % 64 == 0 ? 64 : 0;
  if (bn == 0) return bs::fail(BS_INVALID_ARGUMENT, "GEMM n must be a multiple of 64");
  CUtensorMap ma, mb;
  BS_TRY_ST(bsm::make_map(&ma, a, m, k, bsm::kBM));
  BS_TRY_ST(bsm::make_map(&mb, b, n, k, bn));
  bsm::Buf<int> err;
  MLP_CUDA(err.alloc(1));
  const bsd::umma::EpiStoreF32 epi{c, n};
  auto run = [&]() -> bs_status {
    if (bn == 256) return bsm::gemm<256>(ma, mb, m, n, k, 1, epi, err.p, nullptr);
    if (bn == 128) return bsm::gemm<128>(ma, mb, m, n, k, 1, epi, err.p, nullptr);
    return bsm::gemm<64>(ma, mb, m, n, k, 1, epi, err.p, nullptr);
  };
  BS_TRY_ST(run());  // warm-up
  cudaEvent_t e0, e1;
  MLP_CUDA(cudaEventCreate(&e0));
  MLP_CUDA(cudaEventCreate(&e1));
  cudaEventRecord(e0, nullptr);
  bs_status st = BS_OK;
  for (int it = 0; it < iterations && st == BS_OK; it++) st = run();
  cudaEventRecord(e1, nullptr);
  const cudaError_t e = cudaEventSynchronize(e1);
  float total = 0.f;
  cudaEventElapsedTime(&total, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != BS_OK) return st;
  if (e != cudaSuccess) return bs::fail(BS_EXECUTION, std::string("GEMM timing: ") + cudaGetErrorString(e));
  int h = 0;
  MLP_CUDA(cudaMemcpy(&h, err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (h != 0) return bs::fail(BS_EXECUTION, "GEMM: a pipeline wait timed out");
  *ms = total / float(iterations);
  return BS_OK;
}

bs_status bs_mlp_create(int32_t hidden_layers, int32_t width, int32_t batch, uint64_t seed, bs_mlp** out) {
  if (out == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null output");
  *out = nullptr;
  if (hidden_layers < 1 || hidden_layers > 16 || width != 256 || batch < 128 || batch % 128 != 0)
    return bs::fail(BS_INVALID_ARGUMENT, "network: 1 to 16 hidden layers of width 256, batch a multiple of 128");
  auto* m = new (std::nothrow) bs_mlp;
  if (m == nullptr) return bs::fail(BS_MEMORY_LIMIT, "out of host memory");
  const bs_status st = m->net.init(hidden_layers, width, batch, seed);
  if (st != BS_OK) {
    delete m;
    return st;
  }
  *out = m;
  return BS_OK;
}

bs_status bs_mlp_destroy(bs_mlp* m) {
  if (m == nullptr) return BS_OK;
  bool expected = false;
  if (!m->busy.compare_exchange_strong(expected, true)) return bs::fail(BS_BUSY, "the network is running another call");
  cudaStreamSynchronize(m->net.stream);
  delete m;
  return BS_OK;
}

bs_status bs_mlp_param_count(const bs_mlp* m, int64_t* out) {
  if (m == nullptr || out == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null argument");
  *out = m->net.param_count();
  return BS_OK;
}

bs_status bs_mlp_get_params(bs_mlp* m, float* out) {
  MLP_GUARD(m);
  if (out == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null output");
  MLP_CUDA(cudaStreamSynchronize(m->net.stream));
  for (auto& L : m->net.layers) {
    MLP_CUDA(cudaMemcpy(out, L->w.p, L->w.n * sizeof(float), cudaMemcpyDeviceToHost));
    out += L->w.n;
    MLP_CUDA(cudaMemcpy(out, L->b.p, L->b.n * sizeof(float), cudaMemcpyDeviceToHost));
    out += L->b.n;
  }
  return BS_OK;
}

bs_status bs_mlp_set_params(bs_mlp* m, const float* in) {
  MLP_GUARD(m);
  if (in == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "null input");
  MLP_CUDA(cudaStreamSynchronize(m->net.stream));
  for (auto& L : m->net.layers) {
    MLP_CUDA(cudaMemcpy(L->w.p, in, L->w.n * sizeof(float), cudaMemcpyHostToDevice));
    in += L->w.n;
    MLP_CUDA(cudaMemcpy(L->b.p, in, L->b.n * sizeof(float), cudaMemcpyHostToDevice));
    in += L->b.n;
  }
  BS_TRY_ST(m->net.round_weights());
  MLP_CUDA(cudaStreamSynchronize(m->net.stream));
  return BS_OK;
}

bs_status bs_mlp_set_data(bs_mlp* m, int64_t n, const float* inputs, const float* targets) {
  MLP_GUARD(m);
  if (n < 1 || inputs == nullptr || targets == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "empty data set");
  MLP_CUDA(cudaStreamSynchronize(m->net.stream));
  BS_TRY_ST(upload(inputs, targets, n, &m->net.data_in, &m->net.data_tgt));
  m->net.n_data = n;
  return BS_OK;
}

bs_status bs_mlp_train(bs_mlp* m, int32_t steps, float lr, uint64_t seed, float* losses) {
  MLP_GUARD(m);
  bsm::Mlp& N = m->net;
  if (steps < 1 || !(lr > 0.f) || N.n_data < 1) return bs::fail(BS_INVALID_ARGUMENT, "no data or no steps");
  bsm::Buf<float> dloss;
  MLP_CUDA(dloss.alloc(size_t(steps)));
  BS_TRY_ST(N.clear_grads());
  for (int s = 0; s < steps; s++) {
    const uint64_t step_seed = bsm::mix64(seed ^ (uint64_t(N.steps_done + 1) << 20)) | 1u;
    bsm::mlp_gather<<<(N.M + 127) / 128, 128, 0, N.stream>>>(N.data_in.p, N.data_tgt.p, N.n_data, 0, N.M, N.M,
                                                           step_seed, N.x0.p, N.x0t.p, N.tgt.p);
    MLP_CUDA(cudaGetLastError());
    BS_TRY_ST(N.forward());
    BS_TRY_ST(N.backward(N.M, dloss.p + s));
    BS_TRY_ST(N.adam(lr));
  }
  BS_TRY_ST(N.check_error());
  if (losses != nullptr) MLP_CUDA(cudaMemcpy(losses, dloss.p, size_t(steps) * sizeof(float), cudaMemcpyDeviceToHost));
  return BS_OK;
}

bs_status bs_mlp_loss_grad(bs_mlp* m, int32_t n, const float* inputs, const float* targets, float* loss,
                           float* grads) {
  MLP_GUARD(m);
  bsm::Mlp& N = m->net;
  if (n < 1 || n > N.M || inputs == nullptr || targets == nullptr || loss == nullptr)
    return bs::fail(BS_INVALID_ARGUMENT, "loss_grad: 1 to batch samples");
  MLP_CUDA(cudaStreamSynchronize(N.stream));
  bsm::Buf<float> din, dtgt, dloss;
  BS_TRY_ST(upload(inputs, targets, n, &din, &dtgt));
  MLP_CUDA(dloss.alloc(1));
  BS_TRY_ST(N.clear_grads());
  bsm::mlp_gather<<<(N.M + 127) / 128, 128, 0, N.stream>>>(din.p, dtgt.p, n, 0, N.M, n, 0, N.x0.p, N.x0t.p,
                                                         N.tgt.p);
  MLP_CUDA(cudaGetLastError());
  BS_TRY_ST(N.forward());
  BS_TRY_ST(N.backward(n, dloss.p));
  BS_TRY_ST(N.check_error());
  MLP_CUDA(cudaMemcpy(loss, dloss.p, sizeof(float), cudaMemcpyDeviceToHost));
  if (grads != nullptr)
    for (auto& L : N.layers) {
      MLP_CUDA(cudaMemcpy(grads, L->gw.p, L->gw.n * sizeof(float), cudaMemcpyDeviceToHost));
      grads += L->gw.n;
      MLP_CUDA(cudaMemcpy(grads, L->gb.p, L->gb.n * sizeof(float), cudaMemcpyDeviceToHost));
      grads += L->gb.n;
    }
  return N.clear_grads();
}

bs_status bs_mlp_predict(bs_mlp* m, int64_t n, const float* inputs, float* outputs) {
  MLP_GUARD(m);
  bsm::Mlp& N = m->net;
  if (n < 1 || inputs == nullptr || outputs == nullptr) return bs::fail(BS_INVALID_ARGUMENT, "predict: no samples");
  MLP_CUDA(cudaStreamSynchronize(N.stream));
  bsm::Buf<float> din, none;
  BS_TRY_ST(upload(inputs, nullptr, n, &din, &none));
  for (int64_t first = 0; first < n; first += N.M) {
    const int rows = int(std::min<int64_t>(N.M, n - first));
    bsm::mlp_gather<<<(N.M + 127) / 128, 128, 0, N.stream>>>(din.p, nullptr, n, first, N.M, rows, 0, N.x0.p,
                                                           N.x0t.p, nullptr);
    MLP_CUDA(cudaGetLastError());
    BS_TRY_ST(N.forward());
    MLP_CUDA(cudaMemcpy2DAsync(outputs + first * bsm::kTargets, bsm::kTargets * sizeof(float), N.y.p,
                               bsm::kOutPad * sizeof(float), bsm::kTargets * sizeof(float), rows,
                               cudaMemcpyDeviceToHost, N.stream));
  }
  return N.check_error();
}

}  // extern "C"
