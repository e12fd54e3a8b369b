// pcg_util.cu — small device utilities: compaction flags, index ramps and
// the double-precision energy reductions reported by pcg_diag.
#include <cuda_runtime.h>

#include "pcg_kernels.h"

namespace pcg {

namespace {

constexpr int kThreads = 256;

__global__ void alive_kernel(const double* r, unsigned char* flags, size_t n) {
  size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j < n) flags[j] = r[j] >= 0 ? 1 : 0;
}

__global__ void iota_kernel(unsigned* a, size_t n) {
  size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j < n) a[j] = (unsigned)j;
}

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double part[kThreads / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) part[wid] = v;
  __syncthreads();
  v = threadIdx.x < kThreads / 32 ? part[threadIdx.x] : 0.0;
  if (wid == 0)
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__global__ void energy_kernel(GridGeom g, FieldsF64 f, double* out) {
  double ee = 0, eh = 0;
  const long long total = (long long)g.nr * g.nz;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q / g.nz), k = (int)(q % g.nz);
    const long long p = gidx(g, i, k);
    const double vol = kPi * g.dz * g.dr * g.dr * (2.0 * i + 1);
    double e2 = 0, h2 = 0;
    for (int c = 0; c < 3; ++c) {
      e2 += f.E[c][p] * f.E[c][p];
      h2 += f.H[c][p] * f.H[c][p];
    }
    ee += 0.5 * kEpsilon0 * e2 * vol;
    eh += 0.5 * kMagnConst * h2 * vol;
  }
  ee = block_sum(ee);
  __syncthreads();
  eh = block_sum(eh);
  if (threadIdx.x == 0) {
    atomicAdd(out, ee);
    atomicAdd(out + 1, eh);
  }
}

__global__ void kinetic_kernel(const double* vr, const double* vphi, const double* vz,
                               const double* w, const double* r, size_t n, double mass,
                               double* out) {
  double ek = 0;
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < n;
       j += (size_t)gridDim.x * blockDim.x) {
    if (r[j] < 0) continue;
    const double v2 = vr[j] * vr[j] + vphi[j] * vphi[j] + vz[j] * vz[j];
    const double gm = 1.0 / sqrt(1.0 - v2 / kLightVel2);
    ek += w[j] * mass * v2 * gm * gm / (gm + 1.0);
  }
  ek = block_sum(ek);
  if (threadIdx.x == 0) atomicAdd(out, ek);
}

}  // namespace

void f64_alive_flags(const double* r, unsigned char* flags, size_t n, cudaStream_t s) {
  if (n) alive_kernel<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, s>>>(r, flags, n);
}

void iota_u32(unsigned* a, size_t n, cudaStream_t s) {
  if (n) iota_kernel<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, s>>>(a, n);
}

int f64_energies(const GridGeom& g, const FieldsF64& f, double* ee, double* eh, cudaStream_t s) {
  double* d = nullptr;
  if (cudaMalloc((void**)&d, 2 * sizeof(double)) != cudaSuccess) return -1;
  cudaMemsetAsync(d, 0, 2 * sizeof(double), s);
  energy_kernel<<<296, kThreads, 0, s>>>(g, f, d);
  double hbuf[2];
  cudaMemcpyAsync(hbuf, d, sizeof(hbuf), cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaStreamSynchronize(s);
  cudaFree(d);
  *ee = hbuf[0];
  *eh = hbuf[1];
  return e == cudaSuccess ? 0 : -1;
}

int f64_kinetic(const double* vr, const double* vphi, const double* vz, const double* w,
                const double* r, size_t n, double mass, double* out, cudaStream_t s) {
  *out = 0;
  if (n == 0) return 0;
  double* d = nullptr;
  if (cudaMalloc((void**)&d, sizeof(double)) != cudaSuccess) return -1;
  cudaMemsetAsync(d, 0, sizeof(double), s);
  kinetic_kernel<<<296, kThreads, 0, s>>>(vr, vphi, vz, w, r, n, mass, d);
  cudaMemcpyAsync(out, d, sizeof(double), cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaStreamSynchronize(s);
  cudaFree(d);
  return e == cudaSuccess ? 0 : -1;
}

}  // namespace pcg
