// pcg_mlp_tc.cuh — the collision MLP's forward pass (13 -> 128 -> 128 -> 6,
// ReLU, BF16 operands, FP32 accumulation) on the fifth-generation tensor
// cores: tcgen05.mma with the accumulators in tensor memory (TMEM), issued
// by one thread per CTA, completion signalled on an mbarrier, results read
// back with tcgen05.ld.
//
// A CTA of 128 threads takes 128 rows (cells) at a time; thread r owns row
// r (warp w reads TMEM lanes 32w..32w+31).  Operands sit in shared memory in
// the no-swizzle K-major layout of the UMMA shared-memory descriptor: 8 x 8
// "core matrices" of 8 rows x 16 bytes stored as 128 contiguous bytes, the
// core matrices along K 128 bytes apart (the descriptor's leading byte
// offset) and the 8-row groups K/8 x 128 bytes apart (its stride byte
// offset):
//   byte offset of (row r, column k) = (r/8)(K/8)128 + (k/8)128 + (r%8)16 + (k%8)2.
// Layer l computes D[128 x N] = A[128 x K] . B[N x K]^T with K = 16 per
// instruction: layer 1 (K 16, N 128) into TMEM columns 0..127, layer 2 (K
// 128, N 128) into columns 128..255, layer 3 (K 128, N 16; outputs 6..15
// zero) into columns 0..15 once layer 1's have been read.
//
// Every wait on the mbarrier is bounded; on a time-out the CTA sets *err,
// stops taking rows and frees its TMEM.
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

#include "pcg_mlp.cuh"

namespace pcg {
namespace mlp {
namespace tc {

constexpr int kRows = 128, kThreads = 128, kTmemCols = 256;
constexpr int kN3 = 16;  // layer 3 padded to the smallest N of an M = 128 instruction
constexpr uint32_t kWaitLimit = 1u << 22;

__host__ __device__ constexpr uint32_t canon(int r, int k, int K) {
  return (uint32_t)((r >> 3) * (K >> 3) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

struct Smem {
  alignas(1024) __nv_bfloat16 W1[kHid * kInPad];   // B of layer 1: [128 n][16 k]
  alignas(1024) __nv_bfloat16 W2[kHid * kHid];     // B of layer 2: [128][128]
  alignas(1024) __nv_bfloat16 W3[kN3 * kHid];      // B of layer 3: [16][128]
  alignas(1024) __nv_bfloat16 A1[kRows * kInPad];  // the tile's inputs: [128 rows][16]
  alignas(1024) __nv_bfloat16 A2[kRows * kHid];    // hidden activations: [128][128]
  float b1[kHid], b2[kHid], b3[kN3];
  alignas(8) unsigned long long mbar;
  uint32_t tmem;
  int stop;
};

// UMMA shared-memory descriptor: start address, leading (K) and stride (8-row
// group) byte offsets in 16-byte units, version 1, no swizzle.
__device__ __forceinline__ uint64_t desc(const void* p, uint32_t lbo, uint32_t sbo) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
  return (uint64_t)((a & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
         (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N x M.
__host__ __device__ constexpr uint32_t idesc(int n, int m) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t id, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(d_tmem), "l"(a), "l"(b), "r"(id), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
      : "memory");
}

__device__ __forceinline__ void commit(unsigned long long* bar) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(a)
               : "memory");
}

__device__ __forceinline__ bool wait(unsigned long long* bar, uint32_t phase) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
  for (uint32_t i = 0; i < kWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

// Weights (FP32 [in][out] parameters -> BF16 canonical B operands) and
// biases; every thread of the CTA takes part.
__device__ __forceinline__ void load_weights(Smem& sm, const float* P) {
  unsigned char* w1 = reinterpret_cast<unsigned char*>(sm.W1);
  unsigned char* w2 = reinterpret_cast<unsigned char*>(sm.W2);
  unsigned char* w3 = reinterpret_cast<unsigned char*>(sm.W3);
  for (int q = threadIdx.x; q < kHid * kInPad; q += blockDim.x) {
    const int n = q / kInPad, k = q - n * kInPad;
    *reinterpret_cast<__nv_bfloat16*>(w1 + canon(n, k, kInPad)) =
        __float2bfloat16_rn(k < kIn ? P[kOffW1 + k * kHid + n] : 0.f);
  }
  for (int q = threadIdx.x; q < kHid * kHid; q += blockDim.x) {
    const int n = q / kHid, k = q - n * kHid;
    *reinterpret_cast<__nv_bfloat16*>(w2 + canon(n, k, kHid)) = __float2bfloat16_rn(P[kOffW2 + k * kHid + n]);
  }
  for (int q = threadIdx.x; q < kN3 * kHid; q += blockDim.x) {
    const int n = q / kHid, k = q - n * kHid;
    *reinterpret_cast<__nv_bfloat16*>(w3 + canon(n, k, kHid)) =
        __float2bfloat16_rn(n < kOut ? P[kOffW3 + k * kOut + n] : 0.f);
  }
  for (int q = threadIdx.x; q < kHid; q += blockDim.x) {
    sm.b1[q] = P[kOffB1 + q];
    sm.b2[q] = P[kOffB2 + q];
  }
  if (threadIdx.x < kN3) sm.b3[threadIdx.x] = threadIdx.x < kOut ? P[kOffB3 + threadIdx.x] : 0.f;
}

// Set-up: mbarrier (one arrival per phase) and 256 TMEM columns (warp 0).
__device__ __forceinline__ void begin(Smem& sm) {
  if (threadIdx.x == 0) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(&sm.mbar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    sm.stop = 0;
  }
  if (threadIdx.x < 32) {
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&sm.tmem);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
}

// Release of the TMEM columns.  After a timed-out wait (sm.stop) the last
// committed MMA may still be writing them, so warp 0 first waits again,
// bounded, for that commit (phase counts the committed phases); if it has
// still not arrived the columns stay allocated rather than be handed to
// another CTA under a running MMA.  The caller has reported the time-out,
// and the host treats the kernel's results as invalid.
__device__ __forceinline__ void end(Smem& sm, uint32_t phase) {
  fence_before();
  __syncthreads();
  if (threadIdx.x < 32) {
    const bool drained = !sm.stop || phase == 0 || __all_sync(0xffffffffu, wait(&sm.mbar, (phase - 1) & 1));
    fence_after();
    if (drained)
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(sm.tmem), "r"(kTmemCols)
                   : "memory");
  }
}

// The forward pass of the tile whose inputs this thread wrote to sm.A1 (its
// row, canonical layout) before the call; y[0..5] receives its row's outputs.
// phase counts the mbarrier's completed phases across tiles.  Returns false
// (and sets sm.stop) when a wait timed out.
__device__ __forceinline__ bool forward_tile(Smem& sm, uint32_t& phase, float y[kOut]) {
  const int r = threadIdx.x, warp = r >> 5;
  const uint32_t t0 = sm.tmem, lane_off = (uint32_t)(warp * 32) << 16;
  const uint32_t sbo16 = (kInPad / 8) * 128, sbo128 = (kHid / 8) * 128;
  fence_async_smem();  // this thread's A1 row is visible to the tensor cores
  fence_before();
  __syncthreads();
  if (r == 0) {
    fence_after();
    mma(t0, desc(sm.A1, 128, sbo16), desc(sm.W1, 128, sbo16), idesc(kHid, kRows), 0);
    commit(&sm.mbar);
  }
  bool ok = __all_sync(0xffffffffu, wait(&sm.mbar, phase & 1));  // warp-uniform: tcgen05.ld is .aligned
  ++phase;
  fence_after();
  unsigned char* a2 = reinterpret_cast<unsigned char*>(sm.A2);
  // layer 1 epilogue: bias, ReLU, BF16 into A2 (this thread's row)
  for (int c0 = 0; ok && c0 < kHid; c0 += 16) {
    float v[16];
    ld16(t0 + lane_off + (uint32_t)c0, v);
    uint32_t pk[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float lo = fmaxf(v[2 * q] + sm.b1[c0 + 2 * q], 0.f), hi = fmaxf(v[2 * q + 1] + sm.b1[c0 + 2 * q + 1], 0.f);
      pk[q] = pack2(__float2bfloat16_rn(lo), __float2bfloat16_rn(hi));
    }
    *reinterpret_cast<uint4*>(a2 + canon(r, c0, kHid)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    *reinterpret_cast<uint4*>(a2 + canon(r, c0 + 8, kHid)) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
  }
  fence_async_smem();
  fence_before();
  if (!ok) sm.stop = 1;
  __syncthreads();
  if (sm.stop) return false;
  if (r == 0) {
    fence_after();
    for (int kk = 0; kk < kHid / 16; ++kk)
      mma(t0 + 128, desc(a2 + kk * 256, 128, sbo128), desc(reinterpret_cast<unsigned char*>(sm.W2) + kk * 256, 128, sbo128),
          idesc(kHid, kRows), kk > 0);
    commit(&sm.mbar);
  }
  ok = __all_sync(0xffffffffu, wait(&sm.mbar, phase & 1));
  ++phase;
  fence_after();
  // layer 2 epilogue: into A2 again (layer 2 has finished reading it)
  for (int c0 = 0; ok && c0 < kHid; c0 += 16) {
    float v[16];
    ld16(t0 + lane_off + 128u + (uint32_t)c0, v);
    uint32_t pk[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float lo = fmaxf(v[2 * q] + sm.b2[c0 + 2 * q], 0.f), hi = fmaxf(v[2 * q + 1] + sm.b2[c0 + 2 * q + 1], 0.f);
      pk[q] = pack2(__float2bfloat16_rn(lo), __float2bfloat16_rn(hi));
    }
    *reinterpret_cast<uint4*>(a2 + canon(r, c0, kHid)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    *reinterpret_cast<uint4*>(a2 + canon(r, c0 + 8, kHid)) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
  }
  fence_async_smem();
  fence_before();
  if (!ok) sm.stop = 1;
  __syncthreads();
  if (sm.stop) return false;
  if (r == 0) {
    fence_after();
    for (int kk = 0; kk < kHid / 16; ++kk)
      mma(t0, desc(a2 + kk * 256, 128, sbo128), desc(reinterpret_cast<unsigned char*>(sm.W3) + kk * 256, 128, sbo128),
          idesc(kN3, kRows), kk > 0);
    commit(&sm.mbar);
  }
  ok = __all_sync(0xffffffffu, wait(&sm.mbar, phase & 1));
  ++phase;
  fence_after();
  if (ok) {
    float v[16];
    ld16(t0 + lane_off, v);
#pragma unroll
    for (int q = 0; q < kOut; ++q) y[q] = v[q] + sm.b3[q];
  }
  fence_before();
  if (!ok) sm.stop = 1;
  __syncthreads();  // A1, A2 and the TMEM columns are free for the next tile
  return !sm.stop;
}

}  // namespace tc
}  // namespace mlp
}  // namespace pcg
