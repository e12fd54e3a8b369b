// pcg_mlp.cuh — the per-cell collision MLP (13 -> 128 -> 128 -> 6, ReLU):
// BF16 operands on the tensor cores (mma.sync m16n8k16, FP32 accumulate),
// one warp per 16 rows.  Shared by the training kernels (pcg_mlp.cu) and
// the learned collision step (pcg_learned.cu).
//
// Fragment layouts of mma.m16n8k16 with .bf16 operands (PTX ISA, "Matrix
// fragments for mma.m16n8k16"): g = lane / 4, t = lane % 4;
//   A (16x16, row): regs {a0a1, a2a3, a4a5, a6a7} hold (g, 2t..2t+1),
//     (g+8, 2t..), (g, 2t+8..), (g+8, 2t+8..);
//   B (16x8, col):  {b0b1, b2b3} hold (k = 2t..2t+1, n = g), (k = 2t+8.., n = g);
//   C (16x8, f32):  {c0, c1, c2, c3} = (g, 2t), (g, 2t+1), (g+8, 2t), (g+8, 2t+1).
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace pcg {
namespace mlp {

constexpr int kIn = 13, kInPad = 16, kHid = 128, kOut = 6, kOutPad = 8;
// FP32 parameters, row-major [in][out] per layer, in this order
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kIn * kHid, kOffW2 = kOffB1 + kHid,
              kOffB2 = kOffW2 + kHid * kHid, kOffW3 = kOffB2 + kHid, kOffB3 = kOffW3 + kHid * kOut,
              kParams = kOffB3 + kOut;
// BF16 operand blocks in shared memory, each [n][k] (k contiguous):
// W1t [128][16], W2t [128][128], W3t [8][128] for the forward pass;
// W2 [128][128] (as stored) and W3p [128][16] for the backward pass.
constexpr int kW1tElems = kHid * kInPad, kW2tElems = kHid * kHid, kW3tElems = kOutPad * kHid;
constexpr int kFwdWeightElems = kW1tElems + kW2tElems + kW3tElems;

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ void mma16816(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// A fragment of a row-major [rows][lda] BF16 block (k contiguous), rows r0..r0+15, cols k0..k0+15.
__device__ __forceinline__ void load_a_rowmajor(uint32_t a[4], const __nv_bfloat16* A, int lda, int r0,
                                                int k0, int lane) {
  const int g = lane >> 2, t = lane & 3;
  const __nv_bfloat16* p0 = A + (r0 + g) * lda + k0 + 2 * t;
  const __nv_bfloat16* p1 = p0 + 8 * lda;
  a[0] = *reinterpret_cast<const uint32_t*>(p0);
  a[1] = *reinterpret_cast<const uint32_t*>(p1);
  a[2] = *reinterpret_cast<const uint32_t*>(p0 + 8);
  a[3] = *reinterpret_cast<const uint32_t*>(p1 + 8);
}

// A fragment whose element (m, k) is X[k][m] of a row-major [k][ldx] block
// (the transpose of stored activations, for weight gradients).
__device__ __forceinline__ void load_a_transposed(uint32_t a[4], const __nv_bfloat16* X, int ldx, int m0,
                                                  int k0, int lane) {
  const int g = lane >> 2, t = lane & 3;
  auto e = [&](int m, int k) { return X[(k0 + k) * ldx + m0 + m]; };
  a[0] = pack2(e(g, 2 * t), e(g, 2 * t + 1));
  a[1] = pack2(e(g + 8, 2 * t), e(g + 8, 2 * t + 1));
  a[2] = pack2(e(g, 2 * t + 8), e(g, 2 * t + 9));
  a[3] = pack2(e(g + 8, 2 * t + 8), e(g + 8, 2 * t + 9));
}

// B fragment of an [n][ldb] block (k contiguous): cols n0..n0+7, k0..k0+15.
__device__ __forceinline__ void load_b_nk(uint32_t b[2], const __nv_bfloat16* B, int ldb, int n0, int k0,
                                          int lane) {
  const int g = lane >> 2, t = lane & 3;
  const __nv_bfloat16* p = B + (n0 + g) * ldb + k0 + 2 * t;
  b[0] = *reinterpret_cast<const uint32_t*>(p);
  b[1] = *reinterpret_cast<const uint32_t*>(p + 8);
}

// B fragment whose element (k, n) is Y[k][n] of a row-major [k][ldy] block.
__device__ __forceinline__ void load_b_kn(uint32_t b[2], const __nv_bfloat16* Y, int ldy, int n0, int k0,
                                          int lane) {
  const int g = lane >> 2, t = lane & 3;
  auto e = [&](int k, int n) { return Y[(k0 + k) * ldy + n0 + n]; };
  b[0] = pack2(e(2 * t, g), e(2 * t + 1, g));
  b[1] = pack2(e(2 * t + 8, g), e(2 * t + 9, g));
}

// One warp: out[16][N] (+)= A[16 rows from r0][K] . B, B given as [n][k]; the
// accumulators are acc[N/8][4] in the C layout.
template <int K, int N>
__device__ __forceinline__ void warp_gemm(float acc[N / 8][4], const __nv_bfloat16* A, int lda, int r0,
                                          const __nv_bfloat16* Bnk, int ldb, int lane) {
#pragma unroll
  for (int k0 = 0; k0 < K; k0 += 16) {
    uint32_t a[4];
    load_a_rowmajor(a, A, lda, r0, k0, lane);
#pragma unroll
    for (int nt = 0; nt < N / 8; ++nt) {
      uint32_t b[2];
      load_b_nk(b, Bnk, ldb, nt * 8, k0, lane);
      mma16816(acc[nt], a, b);
    }
  }
}

// Bias, optional ReLU, and BF16 store of a warp's 16 x N block to a
// row-major [rows][ldo] shared block; the FP32 values stay in acc.
template <int N>
__device__ __forceinline__ void bias_relu_store(float acc[N / 8][4], const float* bias, bool relu,
                                                __nv_bfloat16* out, int ldo, int r0, int lane) {
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int nt = 0; nt < N / 8; ++nt) {
    const int n = nt * 8 + 2 * t;
    float v[4] = {acc[nt][0] + bias[n], acc[nt][1] + bias[n + 1], acc[nt][2] + bias[n], acc[nt][3] + bias[n + 1]};
    if (relu)
      for (int q = 0; q < 4; ++q) v[q] = v[q] > 0.f ? v[q] : 0.f;
    for (int q = 0; q < 4; ++q) acc[nt][q] = v[q];
    *reinterpret_cast<uint32_t*>(out + (r0 + g) * ldo + n) =
        pack2(__float2bfloat16_rn(v[0]), __float2bfloat16_rn(v[1]));
    *reinterpret_cast<uint32_t*>(out + (r0 + g + 8) * ldo + n) =
        pack2(__float2bfloat16_rn(v[2]), __float2bfloat16_rn(v[3]));
  }
}

// Forward weights in shared memory ([n][k] BF16 blocks) from the FP32
// parameters; every thread of the block takes part.
__device__ __forceinline__ void load_forward_weights(__nv_bfloat16* W1t, __nv_bfloat16* W2t,
                                                     __nv_bfloat16* W3t, const float* P) {
  for (int q = threadIdx.x; q < kW1tElems; q += blockDim.x) {
    const int n = q / kInPad, k = q - n * kInPad;
    W1t[q] = __float2bfloat16_rn(k < kIn ? P[kOffW1 + k * kHid + n] : 0.f);
  }
  for (int q = threadIdx.x; q < kW2tElems; q += blockDim.x) {
    const int n = q / kHid, k = q - n * kHid;
    W2t[q] = __float2bfloat16_rn(P[kOffW2 + k * kHid + n]);
  }
  for (int q = threadIdx.x; q < kW3tElems; q += blockDim.x) {
    const int n = q / kHid, k = q - n * kHid;
    W3t[q] = __float2bfloat16_rn(n < kOut ? P[kOffW3 + k * kOut + n] : 0.f);
  }
}

// A block of kMlpThreads threads (4 warps) runs the forward pass of 64 rows.
constexpr int kRowsPerBlock = 64, kMlpThreads = 128;

struct FwdSmem {
  __nv_bfloat16 W1t[kW1tElems], W2t[kW2tElems], W3t[kW3tElems];
  __nv_bfloat16 X[kRowsPerBlock * kInPad];
  __nv_bfloat16 H1[kRowsPerBlock * kHid], H2[kRowsPerBlock * kHid];
  float b1[kHid], b2[kHid], b3[kOutPad];
};

template <class S>
__device__ __forceinline__ void load_biases(S& sm, const float* P) {
  for (int q = threadIdx.x; q < kHid; q += blockDim.x) {
    sm.b1[q] = P[kOffB1 + q];
    sm.b2[q] = P[kOffB2 + q];
  }
  if (threadIdx.x < kOutPad) sm.b3[threadIdx.x] = threadIdx.x < kOut ? P[kOffB3 + threadIdx.x] : 0.f;
}

// Forward pass of one warp's 16 rows of sm.X (BF16, [64][16]); the hidden
// activations go to sm.H1 / sm.H2 and the outputs stay in out (C layout:
// out[0][2h+q] is row g + 8h, column 2t + q).
template <class S>
__device__ __forceinline__ void forward_rows(S& sm, int r0, int lane, float out[1][4]) {
  float acc[kHid / 8][4];
  for (int i = 0; i < kHid / 8; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.f;
  warp_gemm<kInPad, kHid>(acc, sm.X, kInPad, r0, sm.W1t, kInPad, lane);
  bias_relu_store<kHid>(acc, sm.b1, true, sm.H1, kHid, r0, lane);
  __syncwarp();
  for (int i = 0; i < kHid / 8; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.f;
  warp_gemm<kHid, kHid>(acc, sm.H1, kHid, r0, sm.W2t, kHid, lane);
  bias_relu_store<kHid>(acc, sm.b2, true, sm.H2, kHid, r0, lane);
  __syncwarp();
  out[0][0] = out[0][1] = out[0][2] = out[0][3] = 0.f;
  warp_gemm<kHid, kOutPad>(out, sm.H2, kHid, r0, sm.W3t, kHid, lane);
  const int t = lane & 3;
  out[0][0] += sm.b3[2 * t];
  out[0][1] += sm.b3[2 * t + 1];
  out[0][2] += sm.b3[2 * t];
  out[0][3] += sm.b3[2 * t + 1];
}

}  // namespace mlp
}  // namespace pcg
