// pcg_mlp.cu — training and inference of the per-cell collision MLP on the
// tensor cores (BF16 operands, FP32 accumulate), behind the pcg_mlp_* C ABI.
//
// One 128-thread block takes 64 rows (a warp per 16).  The training kernel
// runs forward and backward for its rows with every operand in shared
// memory and adds its share of the weight gradients to the FP32 gradient
// with atomics; an Adam kernel then updates the FP32 master parameters.
// The loss is the mean squared error over rows and the 6 outputs.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pcg.h"
#include "pcg_device.h"
#include "pcg_mlp.cuh"
#include "pcg_mlp_tc.cuh"
#include "pcg_philox.cuh"

static_assert(pcg::mlp::kParams == PCG_MLP_PARAMS, "parameter count of the C ABI");

struct pcg_mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  float* params = nullptr;  // FP32 master
  float* grad = nullptr;
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  float* loss = nullptr;    // device accumulator
  float* x = nullptr;       // resident training data
  float* t = nullptr;
  size_t rows = 0;
  uint64_t seed = 0;
  long long step = 0;
};

namespace pcg {
namespace mlp {
namespace {

constexpr int kThreads = 128;

struct TrainSmem {
  __nv_bfloat16 W1t[kW1tElems], W2t[kW2tElems], W3t[kW3tElems];
  __nv_bfloat16 W2[kHid * kHid];       // [in][out] as stored: [n][k] for dH1 = dH2 W2^T
  __nv_bfloat16 W3p[kHid * kInPad];    // [in][out padded to 16]: [n][k] for dH2 = dY W3^T
  __nv_bfloat16 X[kRowsPerBlock * kInPad];
  __nv_bfloat16 H1[kRowsPerBlock * kHid], H2[kRowsPerBlock * kHid];
  __nv_bfloat16 dY[kRowsPerBlock * kInPad];
  __nv_bfloat16 dH2[kRowsPerBlock * kHid], dH1[kRowsPerBlock * kHid];
  float b1[kHid], b2[kHid], b3[kOutPad];
  float db[kHid + kHid + kOutPad];
};

// rows of this block: data index of block row r (a minibatch draw, or r itself)
__device__ __forceinline__ size_t data_row(size_t r, size_t rows, int sample, uint64_t seed, long long step) {
  if (!sample) return r;
  uint32_t o[4];
  philox4x32_10((uint32_t)r, (uint32_t)step, (uint32_t)(step >> 32), 0x6d6c7062u, (uint32_t)seed,
                (uint32_t)(seed >> 32), o);
  const double u = ((double)(o[0] >> 5) * 67108864.0 + (double)(o[1] >> 6)) * (1.0 / 9007199254740992.0);
  size_t q = (size_t)(u * (double)rows);
  return q < rows ? q : rows - 1;
}

template <class S>
__device__ __forceinline__ void load_rows(S& sm, const float* x, size_t r0, size_t nrows, size_t rows,
                                          int sample, uint64_t seed, long long step) {
  for (int q = threadIdx.x; q < kRowsPerBlock * kInPad; q += blockDim.x) {
    const int r = q / kInPad, k = q - r * kInPad;
    float v = 0.f;
    if (r0 + r < nrows && k < kIn) v = x[data_row(r0 + r, rows, sample, seed, step) * kIn + k];
    sm.X[q] = __float2bfloat16_rn(v);
  }
}

__global__ void __launch_bounds__(kThreads) forward_kernel(const float* P, const float* x, size_t rows, float* y) {
  extern __shared__ __align__(16) unsigned char raw[];
  FwdSmem& sm = *reinterpret_cast<FwdSmem*>(raw);
  const size_t r0 = (size_t)blockIdx.x * kRowsPerBlock;
  load_forward_weights(sm.W1t, sm.W2t, sm.W3t, P);
  load_biases(sm, P);
  load_rows(sm, x, r0, rows, rows, 0, 0, 0);
  __syncthreads();
  const int lane = threadIdx.x & 31, wr = (threadIdx.x >> 5) * 16;
  float out[1][4];
  forward_rows(sm, wr, lane, out);
  const int g = lane >> 2, t = lane & 3;
  for (int h = 0; h < 2; ++h) {
    const size_t r = r0 + wr + g + 8 * h;
    if (r >= rows) continue;
    for (int q = 0; q < 2; ++q) {
      const int n = 2 * t + q;
      if (n < kOut) y[r * kOut + n] = out[0][2 * h + q];
    }
  }
}

// Forward + backward of one block of rows; gradients of
// loss = sum((y - t)^2) / (batch * kOut) added to grad.
__global__ void __launch_bounds__(kThreads) train_kernel(const float* P, const float* x, const float* tgt,
                                                         size_t nrows, size_t rows, int sample, uint64_t seed,
                                                         long long step, float* grad, float* loss) {
  extern __shared__ __align__(16) unsigned char raw[];
  TrainSmem& sm = *reinterpret_cast<TrainSmem*>(raw);
  const size_t r0 = (size_t)blockIdx.x * kRowsPerBlock;
  load_forward_weights(sm.W1t, sm.W2t, sm.W3t, P);
  for (int q = threadIdx.x; q < kHid * kHid; q += blockDim.x) sm.W2[q] = __float2bfloat16_rn(P[kOffW2 + q]);
  for (int q = threadIdx.x; q < kHid * kInPad; q += blockDim.x) {
    const int n = q / kInPad, k = q - n * kInPad;
    sm.W3p[q] = __float2bfloat16_rn(k < kOut ? P[kOffW3 + n * kOut + k] : 0.f);
  }
  load_biases(sm, P);
  load_rows(sm, x, r0, nrows, rows, sample, seed, step);
  for (int q = threadIdx.x; q < kHid + kHid + kOutPad; q += blockDim.x) sm.db[q] = 0.f;
  __syncthreads();
  const int lane = threadIdx.x & 31, wr = (threadIdx.x >> 5) * 16, g = lane >> 2, t = lane & 3;
  float out[1][4];
  forward_rows(sm, wr, lane, out);
  // dY = 2 (y - t) / (nrows * kOut), zero for padding rows and columns
  const float scale = 2.f / (float)(nrows * kOut);
  float lsum = 0.f;
  for (int h = 0; h < 2; ++h) {
    const int rl = wr + g + 8 * h;
    const size_t r = r0 + rl;
    for (int q = 0; q < 2; ++q) {
      const int n = 2 * t + q;
      float d = 0.f;
      if (r < nrows && n < kOut) {
        const float e = out[0][2 * h + q] - tgt[data_row(r, rows, sample, seed, step) * kOut + n];
        lsum += e * e;
        d = scale * e;
      }
      sm.dY[rl * kInPad + n] = __float2bfloat16_rn(d);
      sm.dY[rl * kInPad + n + 8] = __float2bfloat16_rn(0.f);
    }
  }
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if (lane == 0) atomicAdd(loss, lsum / (float)(nrows * kOut));
  __syncwarp();
  // dH2 = (dY W3^T) * (H2 > 0)
  float acc[kHid / 8][4];
  for (int i = 0; i < kHid / 8; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.f;
  warp_gemm<kInPad, kHid>(acc, sm.dY, kInPad, wr, sm.W3p, kInPad, lane);
  for (int nt = 0; nt < kHid / 8; ++nt)
    for (int h = 0; h < 2; ++h)
      for (int q = 0; q < 2; ++q) {
        const int rl = wr + g + 8 * h, n = nt * 8 + 2 * t + q;
        const float m = __bfloat162float(sm.H2[rl * kHid + n]) > 0.f ? acc[nt][2 * h + q] : 0.f;
        sm.dH2[rl * kHid + n] = __float2bfloat16_rn(m);
      }
  __syncwarp();
  // dH1 = (dH2 W2^T) * (H1 > 0)
  for (int i = 0; i < kHid / 8; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.f;
  warp_gemm<kHid, kHid>(acc, sm.dH2, kHid, wr, sm.W2, kHid, lane);
  for (int nt = 0; nt < kHid / 8; ++nt)
    for (int h = 0; h < 2; ++h)
      for (int q = 0; q < 2; ++q) {
        const int rl = wr + g + 8 * h, n = nt * 8 + 2 * t + q;
        const float m = __bfloat162float(sm.H1[rl * kHid + n]) > 0.f ? acc[nt][2 * h + q] : 0.f;
        sm.dH1[rl * kHid + n] = __float2bfloat16_rn(m);
      }
  __syncthreads();
  const int warp = threadIdx.x >> 5;
  // dW3[k][n] = sum_r H2[r][k] dY[r][n]: M = 128 (k), N = 8, K = 64 rows; 2 m-tiles per warp
  for (int mt = warp * 2; mt < warp * 2 + 2; ++mt) {
    float c[4] = {0.f, 0.f, 0.f, 0.f};
    for (int k0 = 0; k0 < kRowsPerBlock; k0 += 16) {
      uint32_t a[4], b[2];
      load_a_transposed(a, sm.H2, kHid, mt * 16, k0, lane);
      load_b_kn(b, sm.dY, kInPad, 0, k0, lane);
      mma16816(c, a, b);
    }
    for (int h = 0; h < 2; ++h)
      for (int q = 0; q < 2; ++q) {
        const int kk = mt * 16 + g + 8 * h, n = 2 * t + q;
        if (n < kOut) atomicAdd(grad + kOffW3 + kk * kOut + n, c[2 * h + q]);
      }
  }
  // dW2[k][n] = sum_r H1[r][k] dH2[r][n]: M = 128, N = 128, K = 64; 2 m-tiles per warp
  for (int mt = warp * 2; mt < warp * 2 + 2; ++mt) {
    float c[kHid / 8][4];
    for (int i = 0; i < kHid / 8; ++i) c[i][0] = c[i][1] = c[i][2] = c[i][3] = 0.f;
    for (int k0 = 0; k0 < kRowsPerBlock; k0 += 16) {
      uint32_t a[4];
      load_a_transposed(a, sm.H1, kHid, mt * 16, k0, lane);
      for (int nt = 0; nt < kHid / 8; ++nt) {
        uint32_t b[2];
        load_b_kn(b, sm.dH2, kHid, nt * 8, k0, lane);
        mma16816(c[nt], a, b);
      }
    }
    for (int nt = 0; nt < kHid / 8; ++nt)
      for (int h = 0; h < 2; ++h)
        for (int q = 0; q < 2; ++q) {
          const int kk = mt * 16 + g + 8 * h, n = nt * 8 + 2 * t + q;
          atomicAdd(grad + kOffW2 + kk * kHid + n, c[nt][2 * h + q]);
        }
  }
  // dW1[k][n] = sum_r X[r][k] dH1[r][n]: M = 16, N = 128 (32 columns per warp), K = 64
  {
    float c[4][4];
    for (int i = 0; i < 4; ++i) c[i][0] = c[i][1] = c[i][2] = c[i][3] = 0.f;
    for (int k0 = 0; k0 < kRowsPerBlock; k0 += 16) {
      uint32_t a[4];
      load_a_transposed(a, sm.X, kInPad, 0, k0, lane);
      for (int nt = 0; nt < 4; ++nt) {
        uint32_t b[2];
        load_b_kn(b, sm.dH1, kHid, warp * 32 + nt * 8, k0, lane);
        mma16816(c[nt], a, b);
      }
    }
    for (int nt = 0; nt < 4; ++nt)
      for (int h = 0; h < 2; ++h)
        for (int q = 0; q < 2; ++q) {
          const int kk = g + 8 * h, n = warp * 32 + nt * 8 + 2 * t + q;
          if (kk < kIn) atomicAdd(grad + kOffW1 + kk * kHid + n, c[nt][2 * h + q]);
        }
  }
  // bias gradients: column sums of dH1, dH2, dY
  for (int col = threadIdx.x; col < kHid + kHid + kOut; col += blockDim.x) {
    float s = 0.f;
    for (int r = 0; r < kRowsPerBlock; ++r) {
      if (col < kHid) s += __bfloat162float(sm.dH1[r * kHid + col]);
      else if (col < 2 * kHid) s += __bfloat162float(sm.dH2[r * kHid + col - kHid]);
      else s += __bfloat162float(sm.dY[r * kInPad + col - 2 * kHid]);
    }
    const int off = col < kHid ? kOffB1 + col : (col < 2 * kHid ? kOffB2 + col - kHid : kOffB3 + col - 2 * kHid);
    atomicAdd(grad + off, s);
  }
}

__global__ void adam_kernel(float* P, float* G, float* M, float* V, float lr, float b1, float b2, float eps,
                            float c1, float c2) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= kParams) return;
  const float g = G[q];
  const float m = b1 * M[q] + (1.f - b1) * g;
  const float v = b2 * V[q] + (1.f - b2) * g * g;
  M[q] = m;
  V[q] = v;
  P[q] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
  G[q] = 0.f;
}

// The forward pass on tcgen05 (pcg_mlp_tc.cuh): persistent CTAs of 128
// threads, 128 rows per tile; *err is set when a wait timed out.
__global__ void __launch_bounds__(tc::kThreads, 1) forward_tc_kernel(const float* P, const float* x, size_t rows,
                                                                      float* y, int* err) {
  extern __shared__ __align__(16) unsigned char raw_tc[];
  tc::Smem& sm = *reinterpret_cast<tc::Smem*>((reinterpret_cast<uintptr_t>(raw_tc) + 1023) & ~uintptr_t(1023));
  tc::load_weights(sm, P);
  tc::begin(sm);
  uint32_t phase = 0;
  unsigned char* a1 = reinterpret_cast<unsigned char*>(sm.A1);
  const size_t tiles = (rows + tc::kRows - 1) / tc::kRows;
  for (size_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const size_t row = tile * tc::kRows + threadIdx.x;
    uint32_t pk[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int k = 2 * q;
      const float lo = row < rows && k < kIn ? x[row * kIn + k] : 0.f;
      const float hi = row < rows && k + 1 < kIn ? x[row * kIn + k + 1] : 0.f;
      pk[q] = pack2(__float2bfloat16_rn(lo), __float2bfloat16_rn(hi));
    }
    *reinterpret_cast<uint4*>(a1 + tc::canon(threadIdx.x, 0, kInPad)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    *reinterpret_cast<uint4*>(a1 + tc::canon(threadIdx.x, 8, kInPad)) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
    float out[kOut];
    if (!tc::forward_tile(sm, phase, out)) {
      if (threadIdx.x == 0) atomicExch(err, 1);
      break;
    }
    if (row < rows)
      for (int q = 0; q < kOut; ++q) y[row * kOut + q] = out[q];
  }
  tc::end(sm, phase);
}

}  // namespace
}  // namespace mlp
}  // namespace pcg

using namespace pcg::mlp;
using pcg::DeviceScope;

namespace {

int set_smem_limits() {
  static const bool ok = [] {
    return cudaFuncSetAttribute(train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TrainSmem)) ==
               cudaSuccess &&
           cudaFuncSetAttribute(forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(FwdSmem)) ==
               cudaSuccess;
  }();
  return ok ? 0 : -1;
}

int upload(float** d, const float* h, size_t n, cudaStream_t s) {
  cudaFree(*d);
  *d = nullptr;
  if (cudaMalloc((void**)d, std::max<size_t>(n, 1) * sizeof(float)) != cudaSuccess) return -1;
  return cudaMemcpyAsync(*d, h, n * sizeof(float), cudaMemcpyHostToDevice, s) == cudaSuccess ? 0 : -1;
}

}  // namespace

extern "C" {

int pcg_mlp_create(int device, uint64_t seed, pcg_mlp** out) {
  if (!out) return PCG_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return PCG_ERR_ARG;
  DeviceScope device_scope(device);
  pcg_mlp* m = new pcg_mlp();
  m->device = device;
  m->seed = seed;
  if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) { delete m; return PCG_ERR_CUDA; }
  float** bufs[] = {&m->params, &m->grad, &m->adam_m, &m->adam_v};
  for (float** b : bufs)
    if (cudaMalloc((void**)b, kParams * sizeof(float)) != cudaSuccess) { pcg_mlp_destroy(m); return PCG_ERR_NOMEM; }
  if (cudaMalloc((void**)&m->loss, sizeof(float)) != cudaSuccess) { pcg_mlp_destroy(m); return PCG_ERR_NOMEM; }
  // He-uniform initialisation from Philox, zero biases
  std::vector<float> p(kParams, 0.f);
  auto fill = [&](int off, int fan_in, int count) {
    const double a = std::sqrt(6.0 / fan_in);
    for (int q = 0; q < count; ++q) {
      uint32_t o[4];
      pcg::philox4x32_10((uint32_t)(off + q), 0u, 0u, 0x6d6c7069u, (uint32_t)seed, (uint32_t)(seed >> 32), o);
      const double u = ((double)(o[0] >> 5) * 67108864.0 + (double)(o[1] >> 6)) * (1.0 / 9007199254740992.0);
      p[off + q] = (float)((2.0 * u - 1.0) * a);
    }
  };
  fill(kOffW1, kIn, kIn * kHid);
  fill(kOffW2, kHid, kHid * kHid);
  fill(kOffW3, kHid, kHid * kOut);
  cudaMemcpyAsync(m->params, p.data(), kParams * sizeof(float), cudaMemcpyHostToDevice, m->stream);
  cudaMemsetAsync(m->grad, 0, kParams * sizeof(float), m->stream);
  cudaMemsetAsync(m->adam_m, 0, kParams * sizeof(float), m->stream);
  cudaMemsetAsync(m->adam_v, 0, kParams * sizeof(float), m->stream);
  if (cudaStreamSynchronize(m->stream) != cudaSuccess || set_smem_limits() != 0) { pcg_mlp_destroy(m); return PCG_ERR_CUDA; }
  *out = m;
  return PCG_OK;
}

int pcg_mlp_destroy(pcg_mlp* m) {
  DeviceScope device_scope(m ? m->device : -1);
  if (!m) return PCG_OK;
  if (m->stream) cudaStreamSynchronize(m->stream);
  cudaFree(m->params); cudaFree(m->grad); cudaFree(m->adam_m); cudaFree(m->adam_v); cudaFree(m->loss);
  cudaFree(m->x); cudaFree(m->t);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
  return PCG_OK;
}

int pcg_mlp_get_params(pcg_mlp* m, float* out) {
  DeviceScope device_scope(m ? m->device : -1);
  if (!m || !out) return PCG_ERR_ARG;
  if (cudaMemcpyAsync(out, m->params, kParams * sizeof(float), cudaMemcpyDeviceToHost, m->stream) != cudaSuccess ||
      cudaStreamSynchronize(m->stream) != cudaSuccess)
    return PCG_ERR_CUDA;
  return PCG_OK;
}

int pcg_mlp_set_params(pcg_mlp* m, const float* in) {
  DeviceScope device_scope(m ? m->device : -1);
  if (!m || !in) return PCG_ERR_ARG;
  if (cudaMemcpyAsync(m->params, in, kParams * sizeof(float), cudaMemcpyHostToDevice, m->stream) != cudaSuccess ||
      cudaMemsetAsync(m->adam_m, 0, kParams * sizeof(float), m->stream) != cudaSuccess ||
      cudaMemsetAsync(m->adam_v, 0, kParams * sizeof(float), m->stream) != cudaSuccess ||
      cudaStreamSynchronize(m->stream) != cudaSuccess)
    return PCG_ERR_CUDA;
  m->step = 0;
  return PCG_OK;
}

int pcg_mlp_forward(pcg_mlp* m, const float* x, size_t rows, float* y) {
  DeviceScope device_scope(m ? m->device : -1);
  if (!m || (!x && rows) || (!y && rows)) return PCG_ERR_ARG;
  if (rows == 0) return PCG_OK;
  float *dx = nullptr, *dy = nullptr;
  if (upload(&dx, x, rows * kIn, m->stream) != 0 || cudaMalloc((void**)&dy, rows * kOut * sizeof(float)) != cudaSuccess) {
    cudaFree(dx);
    return PCG_ERR_NOMEM;
  }
  forward_kernel<<<(unsigned)((rows + kRowsPerBlock - 1) / kRowsPerBlock), kThreads, sizeof(FwdSmem), m->stream>>>(
      m->params, dx, rows, dy);
  const bool ok = cudaMemcpyAsync(y, dy, rows * kOut * sizeof(float), cudaMemcpyDeviceToHost, m->stream) == cudaSuccess &&
                  cudaStreamSynchronize(m->stream) == cudaSuccess;
  cudaFree(dx);
  cudaFree(dy);
  return ok ? PCG_OK : PCG_ERR_CUDA;
}

int pcg_mlp_forward_tc(pcg_mlp* m, const float* x, size_t rows, float* y, float* device_ms) {
  DeviceScope device_scope(m ? m->device : -1);
  if (!m || (!x && rows) || (!y && rows)) return PCG_ERR_ARG;
  if (device_ms) *device_ms = 0.f;
  if (rows == 0) return PCG_OK;
  const size_t smem = sizeof(tc::Smem) + 1024;
  static const bool attr = cudaFuncSetAttribute(forward_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)smem) == cudaSuccess;
  if (!attr) return PCG_ERR_CUDA;
  float *dx = nullptr, *dy = nullptr;
  int* derr = nullptr;
  if (upload(&dx, x, rows * kIn, m->stream) != 0 || cudaMalloc((void**)&dy, rows * kOut * sizeof(float)) != cudaSuccess ||
      cudaMalloc((void**)&derr, sizeof(int)) != cudaSuccess) {
    cudaFree(dx);
    cudaFree(dy);
    return PCG_ERR_NOMEM;
  }
  cudaMemsetAsync(derr, 0, sizeof(int), m->stream);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m->device);
  const size_t tiles = (rows + tc::kRows - 1) / tc::kRows;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, m->stream);
  forward_tc_kernel<<<(unsigned)std::min<size_t>(tiles, (size_t)sms), tc::kThreads, smem, m->stream>>>(
      m->params, dx, rows, dy, derr);
  cudaEventRecord(e1, m->stream);
  int herr = 0;
  bool ok = cudaGetLastError() == cudaSuccess &&
            cudaMemcpyAsync(y, dy, rows * kOut * sizeof(float), cudaMemcpyDeviceToHost, m->stream) == cudaSuccess &&
            cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, m->stream) == cudaSuccess &&
            cudaStreamSynchronize(m->stream) == cudaSuccess;
  if (ok && device_ms) cudaEventElapsedTime(device_ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(dx);
  cudaFree(dy);
  cudaFree(derr);
  if (!ok) return PCG_ERR_CUDA;
  return herr ? PCG_ERR_TIMEOUT : PCG_OK;
}

int pcg_mlp_gradient(pcg_mlp* m, const float* x, const float* t, size_t rows, float* grad_out, float* loss_out) {
  DeviceScope device_scope(m ? m->device : -1);
  if (!m || !x || !t || !grad_out || rows == 0) return PCG_ERR_ARG;
  float *dx = nullptr, *dt = nullptr;
  if (upload(&dx, x, rows * kIn, m->stream) != 0 || upload(&dt, t, rows * kOut, m->stream) != 0) {
    cudaFree(dx); cudaFree(dt);
    return PCG_ERR_NOMEM;
  }
  cudaMemsetAsync(m->grad, 0, kParams * sizeof(float), m->stream);
  cudaMemsetAsync(m->loss, 0, sizeof(float), m->stream);
  train_kernel<<<(unsigned)((rows + kRowsPerBlock - 1) / kRowsPerBlock), kThreads, sizeof(TrainSmem), m->stream>>>(
      m->params, dx, dt, rows, rows, 0, 0, 0, m->grad, m->loss);
  bool ok = cudaMemcpyAsync(grad_out, m->grad, kParams * sizeof(float), cudaMemcpyDeviceToHost, m->stream) == cudaSuccess;
  float l = 0.f;
  ok = ok && cudaMemcpyAsync(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream) == cudaSuccess;
  ok = ok && cudaMemsetAsync(m->grad, 0, kParams * sizeof(float), m->stream) == cudaSuccess;
  ok = ok && cudaStreamSynchronize(m->stream) == cudaSuccess;
  cudaFree(dx);
  cudaFree(dt);
  if (loss_out) *loss_out = l;
  return ok ? PCG_OK : PCG_ERR_CUDA;
}

int pcg_mlp_set_data(pcg_mlp* m, const float* x, const float* t, size_t rows) {
  DeviceScope device_scope(m ? m->device : -1);
  if (!m || !x || !t || rows == 0) return PCG_ERR_ARG;
  if (upload(&m->x, x, rows * kIn, m->stream) != 0 || upload(&m->t, t, rows * kOut, m->stream) != 0)
    return PCG_ERR_NOMEM;
  m->rows = rows;
  return cudaStreamSynchronize(m->stream) == cudaSuccess ? PCG_OK : PCG_ERR_CUDA;
}

int pcg_mlp_train(pcg_mlp* m, int steps, int batch, float lr, float* last_loss) {
  DeviceScope device_scope(m ? m->device : -1);
  if (!m || steps < 0 || batch <= 0 || !m->rows) return PCG_ERR_ARG;
  const unsigned blocks = (unsigned)((batch + kRowsPerBlock - 1) / kRowsPerBlock);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int s = 0; s < steps; ++s) {
    ++m->step;
    cudaMemsetAsync(m->loss, 0, sizeof(float), m->stream);
    train_kernel<<<blocks, kThreads, sizeof(TrainSmem), m->stream>>>(m->params, m->x, m->t, (size_t)batch, m->rows,
                                                                     1, m->seed, m->step, m->grad, m->loss);
    const float c1 = 1.f - std::pow(b1, (float)m->step), c2 = 1.f - std::pow(b2, (float)m->step);
    adam_kernel<<<(kParams + 255) / 256, 256, 0, m->stream>>>(m->params, m->grad, m->adam_m, m->adam_v, lr, b1, b2,
                                                              eps, c1, c2);
  }
  float l = 0.f;
  if (cudaMemcpyAsync(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream) != cudaSuccess ||
      cudaStreamSynchronize(m->stream) != cudaSuccess)
    return PCG_ERR_CUDA;
  if (last_loss) *last_loss = l;
  return cudaGetLastError() == cudaSuccess ? PCG_OK : PCG_ERR_CUDA;
}

}  // extern "C"
