// pcg_kernels_f32.cu — the single-precision production path: float Yee
// update, species buffers in (cell, offset) form, import/export, beam
// injection and the fused particle step.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "pcg_f32.h"
#include "pcg_f32_step.cuh"
#include "pcg_philox.cuh"
#include "pcg_yee.cuh"

namespace pcg {

namespace {

constexpr int kThreads = 256;

inline unsigned blocks_for(size_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

// Position in metres -> (cell, offset) with 0 <= offset < 1.
__device__ __forceinline__ void split_position(double x_m, double d, int* cell, float* off) {
  const double x = x_m / d;
  double c = floor(x);
  float f = (float)(x - c);
  if (f >= 1.0f) { f = 0.0f; c += 1.0; }
  *cell = (int)c;
  *off = f;
}

__global__ void import_kernel(GridGeom g, SpeciesF32Buffers b, size_t n0, size_t n,
                              const double* src) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  size_t j = n0 + i;
  int ci, ck;
  float fr, fz;
  split_position(src[i], g.dr, &ci, &fr);
  split_position(src[n + i], g.dz, &ck, &fz);
  b.cell[j] = pack_cell(ci, ck);
  b.off_r[j] = fr;
  b.off_z[j] = fz;
  b.vr[j] = (float)src[2 * n + i];
  b.vphi[j] = (float)src[3 * n + i];
  b.vz[j] = (float)src[4 * n + i];
  b.w[j] = (float)src[5 * n + i];
}

// BeamP::inject (beamP.cpp:100-145) with the same Philox stream as the
// double path; positions are computed in double and then split.
__global__ void inject_kernel(GridGeom g, SpeciesF32Buffers b, size_t n0, unsigned count,
                              BeamInject bi) {
  unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const double dr = g.dr, dz = g.dz;
  double u[2];
  philox_uniform2(bi.seed, bi.stream, bi.step, i, u);
  const double pos_r = bi.domain_radius * u[0] + dr / 2 + 0.0 * dr;
  const double pos_z = bi.dl * u[1] + bi.half_z;
  double norm;
  if (pos_r > dr / 2)
    norm = 2 * kPi * pos_r * dr * dz / bi.v_macro_avg;
  else
    norm = kPi * (pos_r * pos_r + pos_r * dr + dr * dr / 4.) * dz / bi.v_macro_avg;
  const size_t j = n0 + i;
  int ci, ck;
  float fr, fz;
  split_position(pos_r, dr, &ci, &fr);
  split_position(pos_z, dz, &ck, &fz);
  b.cell[j] = pack_cell(ci, ck);
  b.off_r[j] = fr;
  b.off_z[j] = fz;
  b.vr[j] = 0.f;
  b.vphi[j] = 0.f;
  b.vz[j] = (float)bi.velocity;
  b.w[j] = (float)(bi.n_per_macro_avg * norm);
}

__global__ void alive_kernel(const int* cell, unsigned char* flags, size_t n) {
  size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j < n) flags[j] = cell[j] >= 0 ? 1 : 0;
}

template <typename T>
__global__ void gather_kernel(const T* src, T* dst, const unsigned* idx, size_t n) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[idx[i]];
}

__global__ void export_kernel(GridGeom g, SpeciesF32Buffers b, size_t n, double* out,
                              int* cells) {
  size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int c = b.cell[j];
  const int ci = cell_r_of(c), ck = cell_z_of(c);
  out[j] = ((double)ci + (double)b.off_r[j]) * g.dr;
  out[n + j] = ((double)ck + (double)b.off_z[j]) * g.dz;
  out[2 * n + j] = b.vr[j];
  out[3 * n + j] = b.vphi[j];
  out[4 * n + j] = b.vz[j];
  out[5 * n + j] = b.w[j];
  cells[j] = ci;
  cells[n + j] = ck;
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

struct Fld12 {
  const float* f[12];
};

__global__ void energy_kernel(GridGeom g, Fld12 fl, double* out) {
  double ee = 0, eh = 0;
  const long long total = (long long)g.nr * g.nz;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q / g.nz), k = (int)(q % g.nz);
    const long long p = gidx(g, i, k);
    const double vol = kPi * g.dz * g.dr * g.dr * (2.0 * i + 1);
    double e2 = 0, h2 = 0;
    for (int c = 0; c < 3; ++c) {
      const double e = fl.f[c][p], hh = fl.f[3 + c][p];
      e2 += e * e;
      h2 += hh * hh;
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

__global__ void kinetic_kernel(SpeciesF32Buffers b, size_t n, double mass, double* out) {
  double ek = 0;
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < n;
       j += (size_t)gridDim.x * blockDim.x) {
    if (b.cell[j] < 0) continue;
    const double vr = b.vr[j], vp = b.vphi[j], vz = b.vz[j];
    const double v2 = vr * vr + vp * vp + vz * vz;
    const double gm = 1.0 / sqrt(1.0 - v2 / kLightVel2);
    ek += (double)b.w[j] * mass * v2 * gm * gm / (gm + 1.0);
  }
  ek = block_sum(ek);
  if (threadIdx.x == 0) atomicAdd(out, ek);
}

}  // namespace

int f32_alloc_species(SpeciesF32Buffers& b, size_t cap) {
  if (cap == 0) cap = 1;
  b.cap = cap;
  if (cudaMalloc((void**)&b.cell, cap * sizeof(int)) != cudaSuccess) return -1;
  float** arrs[] = {&b.off_r, &b.off_z, &b.vr, &b.vphi, &b.vz, &b.w};
  for (float** a : arrs)
    if (cudaMalloc((void**)a, cap * sizeof(float)) != cudaSuccess) return -1;
  return 0;
}

void f32_free_species(SpeciesF32Buffers& b) {
  void* arrs[] = {b.cell, b.off_r, b.off_z, b.vr, b.vphi, b.vz, b.w};
  for (void* a : arrs) cudaFree(a);
  b = SpeciesF32Buffers();
}

void f32_launch_yee_e(const YeeArgs<float>& a, cudaStream_t s) {
  dim3 grid((a.g.nz + 4 + kThreads - 1) / kThreads, a.g.nr + 4);
  yee_e_kernel<float><<<grid, kThreads, 0, s>>>(a);
}

void f32_launch_yee_h(const YeeArgs<float>& a, int fixed, cudaStream_t s) {
  dim3 grid((a.g.nz + 4 + kThreads - 1) / kThreads, a.g.nr + 4);
  yee_h_kernel<float><<<grid, kThreads, 0, s>>>(a, fixed);
}

void f32_launch_inject(const GridGeom& g, SpeciesF32Buffers& b, size_t n0, unsigned count,
                       const BeamInject& bi, cudaStream_t s) {
  if (count) inject_kernel<<<(count + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, b, n0, count, bi);
}

void f32_launch_import(const GridGeom& g, SpeciesF32Buffers& b, size_t n0, size_t n,
                       const double* src, cudaStream_t s) {
  if (n) import_kernel<<<blocks_for(n), kThreads, 0, s>>>(g, b, n0, n, src);
}

void f32_alive_flags(const SpeciesF32Buffers& b, unsigned char* flags, size_t n, cudaStream_t s) {
  if (n) alive_kernel<<<blocks_for(n), kThreads, 0, s>>>(b.cell, flags, n);
}

int f32_compact(SpeciesF32Buffers& b, const unsigned* idx, size_t kept, cudaStream_t s) {
  if (kept == 0) return 0;
  void* tmp = nullptr;
  if (cudaMalloc(&tmp, kept * sizeof(float)) != cudaSuccess) return -1;
  gather_kernel<int><<<blocks_for(kept), kThreads, 0, s>>>(b.cell, (int*)tmp, idx, kept);
  cudaMemcpyAsync(b.cell, tmp, kept * sizeof(int), cudaMemcpyDeviceToDevice, s);
  float* arrs[] = {b.off_r, b.off_z, b.vr, b.vphi, b.vz, b.w};
  for (float* a : arrs) {
    gather_kernel<float><<<blocks_for(kept), kThreads, 0, s>>>(a, (float*)tmp, idx, kept);
    cudaMemcpyAsync(a, tmp, kept * sizeof(float), cudaMemcpyDeviceToDevice, s);
  }
  cudaError_t e = cudaStreamSynchronize(s);
  cudaFree(tmp);
  return e == cudaSuccess ? 0 : -1;
}

int f32_export(const GridGeom& g, SpeciesF32Buffers& b, size_t n, double* r, double* z,
               double* vr, double* vphi, double* vz, double* w, int32_t* cell_r, int32_t* cell_z,
               cudaStream_t s) {
  double* d = nullptr;
  int* c = nullptr;
  if (cudaMalloc((void**)&d, 6 * n * sizeof(double)) != cudaSuccess) return -1;
  if (cudaMalloc((void**)&c, 2 * n * sizeof(int)) != cudaSuccess) { cudaFree(d); return -1; }
  export_kernel<<<blocks_for(n), kThreads, 0, s>>>(g, b, n, d, c);
  double* dst[6] = {r, z, vr, vphi, vz, w};
  for (int a = 0; a < 6; ++a)
    if (dst[a]) cudaMemcpyAsync(dst[a], d + a * n, n * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (cell_r) cudaMemcpyAsync(cell_r, c, n * sizeof(int), cudaMemcpyDeviceToHost, s);
  if (cell_z) cudaMemcpyAsync(cell_z, c + n, n * sizeof(int), cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaStreamSynchronize(s);
  cudaFree(d);
  cudaFree(c);
  return e == cudaSuccess ? 0 : -1;
}

int f32_energies(const GridGeom& g, float* const fld[12], double* ee, double* eh, cudaStream_t s) {
  double* d = nullptr;
  if (cudaMalloc((void**)&d, 2 * sizeof(double)) != cudaSuccess) return -1;
  cudaMemsetAsync(d, 0, 2 * sizeof(double), s);
  Fld12 fl;
  for (int c = 0; c < 12; ++c) fl.f[c] = fld[c];
  energy_kernel<<<296, kThreads, 0, s>>>(g, fl, d);
  double hbuf[2];
  cudaMemcpyAsync(hbuf, d, sizeof(hbuf), cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaStreamSynchronize(s);
  cudaFree(d);
  *ee = hbuf[0];
  *eh = hbuf[1];
  return e == cudaSuccess ? 0 : -1;
}

int f32_kinetic(const SpeciesF32Buffers& b, size_t n, double mass, double* out, cudaStream_t s) {
  *out = 0;
  if (n == 0) return 0;
  double* d = nullptr;
  if (cudaMalloc((void**)&d, sizeof(double)) != cudaSuccess) return -1;
  cudaMemsetAsync(d, 0, sizeof(double), s);
  kinetic_kernel<<<296, kThreads, 0, s>>>(b, n, mass, d);
  cudaMemcpyAsync(out, d, sizeof(double), cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaStreamSynchronize(s);
  cudaFree(d);
  return e == cudaSuccess ? 0 : -1;
}

void f32_launch_step(const F32Step& st, SpeciesF32Buffers& b, size_t n, double charge,
                     double mass, int is_beam, cudaStream_t s) {
  launch_f32_particle_step(st, b, n, charge, mass, is_beam, s);
}

}  // namespace pcg
