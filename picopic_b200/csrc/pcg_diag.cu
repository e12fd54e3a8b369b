// pcg_diag.cu — double-precision acceptance diagnostics of the deposit:
// node charges of the particles and the flux divergence of a staggered
// (r, z) vector field (J or E).  With them the host forms the charge
// continuity residual Q(n+1) - Q(n) + dt div J and the Gauss residual
// eps0 div E - Q.
//
// The node charge is the particle shape that the Villasenor-Buneman deposit
// (currentVB.cpp:22-173) conserves exactly: a particle at x = r/dr in cell
// i gives node i the radial share f_i(x) = 1/2 + i(i+1)/(2x) - x/2 and node
// i+1 the rest, times the linear axial shares 1-b, b.  The face areas of the
// divergence are those the reference's Yee update implies
// (maxwellSolverYee.cpp:161-257): J_r, E_r at (i+1/2, k) cross
// 2 pi (i+1/2) dr dz; J_z, E_z at (i, k+1/2) cross 2 pi i dr^2, or
// pi dr^2 / 4 on the axis (its 4/dr curl factor).
#include <cuda_runtime.h>

#include "pcg_diag.h"
#include "pcg_f32.h"

namespace pcg {

namespace {

constexpr int kThreads = 256;
constexpr double kPiD = 3.1415926535897932;

inline unsigned blocks_for(size_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

__device__ __forceinline__ void add_charge(const GridGeom& g, double* q, double x, double y,
                                           double qw) {
  const int i = (int)floor(x), k = (int)floor(y);
  if (i < 0 || k < 0 || i >= g.nr || k >= g.nz) return;
  const double fi = 0.5 + (double)i * (double)(i + 1) / (2.0 * x) - 0.5 * x;
  const double b = y - (double)k;
  const int ld = g.nz + 4;
  double* p = q + (size_t)(i + 2) * ld + (k + 2);
  atomicAdd(p, qw * fi * (1.0 - b));
  atomicAdd(p + 1, qw * fi * b);
  atomicAdd(p + ld, qw * (1.0 - fi) * (1.0 - b));
  atomicAdd(p + ld + 1, qw * (1.0 - fi) * b);
}

__global__ void charge_f64_kernel(GridGeom g, const double* r, const double* z, const double* w,
                                  size_t n, double charge, double* q) {
  const size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= n || !(r[j] >= 0.0)) return;  // dead slots have r < 0
  add_charge(g, q, r[j] / g.dr, z[j] / g.dz, charge * w[j]);
}

__global__ void charge_f32_kernel(GridGeom g, SpeciesF32Buffers b, size_t n, double charge,
                                  double* q) {
  const size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int c = b.cell[j];
  if (c < 0) return;
  add_charge(g, q, (double)cell_r_of(c) + (double)b.off_r[j], (double)cell_z_of(c) + (double)b.off_z[j],
             charge * (double)b.w[j]);
}

template <typename T>
__global__ void divergence_kernel(GridGeom g, const T* fr, const T* fz, double* out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x - 2;
  const int i = (int)blockIdx.y - 2;
  if (k > g.nz + 1) return;
  const int ld = g.nz + 4;
  const size_t p = (size_t)(i + 2) * ld + (k + 2);
  const double dr = g.dr, dz = g.dz;
  const double ar = 2.0 * kPiD * ((double)i + 0.5) * dr * dz;
  const double ar_in = 2.0 * kPiD * ((double)i - 0.5) * dr * dz;
  const double s = i > 0 ? 2.0 * kPiD * (double)i * dr * dr : (i == 0 ? 0.25 * kPiD * dr * dr : 0.0);
  double d = 0.0;
  if (i > -2) d += (double)fr[p] * ar - (double)fr[p - ld] * ar_in;
  if (k > -2) d += ((double)fz[p] - (double)fz[p - 1]) * s;
  out[p] = d;
}

}  // namespace

int diag_node_charge_f64(const GridGeom& g, const double* r, const double* z, const double* w,
                         size_t n, double charge, double* q, cudaStream_t s) {
  if (n) charge_f64_kernel<<<blocks_for(n), kThreads, 0, s>>>(g, r, z, w, n, charge, q);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int diag_node_charge_f32(const GridGeom& g, const SpeciesF32Buffers& b, size_t n, double charge,
                         double* q, cudaStream_t s) {
  if (n) charge_f32_kernel<<<blocks_for(n), kThreads, 0, s>>>(g, b, n, charge, q);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int diag_divergence(const GridGeom& g, const void* fr, const void* fz, int is_double, double* out,
                    cudaStream_t s) {
  const dim3 grid((g.nz + 4 + kThreads - 1) / kThreads, g.nr + 4);
  if (is_double)
    divergence_kernel<double><<<grid, kThreads, 0, s>>>(g, (const double*)fr, (const double*)fz, out);
  else
    divergence_kernel<float><<<grid, kThreads, 0, s>>>(g, (const float*)fr, (const float*)fz, out);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace pcg
