// pcg_init.cu — seeded synthetic initial conditions on the device: a
// uniform Maxwellian plasma (pcg_seed_plasma) for both particle layouts.
#include <cuda_runtime.h>

#include "pcg_f32.h"
#include "pcg_init.h"
#include "pcg_philox.cuh"

namespace pcg {

namespace {

constexpr int kThreads = 256;

struct Draw {
  double r, z, v[3], w;
};

// Particle j of a plasma: two Philox blocks give r, z and two normals, a
// third gives the last normal (Box-Muller).
__device__ __forceinline__ Draw draw(const GridGeom& g, const PlasmaSeed& p, size_t j) {
  double u[2], n1[2], n2[2];
  const uint32_t idx = (uint32_t)j, hi = (uint32_t)(j >> 32);
  philox_uniform2(p.seed, p.stream, ((uint64_t)hi << 32) | 0u, idx, u);
  philox_uniform2(p.seed, p.stream, ((uint64_t)hi << 32) | 1u, idx, n1);
  philox_uniform2(p.seed, p.stream, ((uint64_t)hi << 32) | 2u, idx, n2);
  Draw d;
  const double r0 = 0.5 * g.dr, r1 = g.R - 0.5 * g.dr;
  const double two_pi = 6.283185307179586;
  const double a1 = sqrt(-2.0 * log(1.0 - n1[0])), a2 = sqrt(-2.0 * log(1.0 - n2[0]));
  if (p.per_cell) {  // cell j / per_cell, uniform in its ring volume
    const size_t c = j / p.per_cell;
    const double ci = (double)(c / g.nz), ck = (double)(c % g.nz);
    d.r = g.dr * sqrt(ci * ci + u[0] * (2.0 * ci + 1.0));
    d.z = g.dz * (ck + u[1]);
    d.w = p.density * 3.1415926535897932 * g.dz * g.dr * g.dr * (2.0 * ci + 1.0) / p.per_cell;
    d.v[0] = p.sigma_v_perp * a1 * cos(two_pi * n1[1]);
    d.v[1] = p.sigma_v_perp * a1 * sin(two_pi * n1[1]);
    d.v[2] = p.sigma_v * a2 * cos(two_pi * n2[1]);
    return d;
  }
  d.r = sqrt(r0 * r0 + u[0] * (r1 * r1 - r0 * r0));
  d.z = 0.5 * g.dz + u[1] * (g.L - g.dz);
  d.w = p.weight;
  d.v[0] = p.sigma_v * a1 * cos(two_pi * n1[1]);
  d.v[1] = p.sigma_v * a1 * sin(two_pi * n1[1]);
  d.v[2] = p.sigma_v * a2 * cos(two_pi * n2[1]);
  // keep the sample inside the walls after rounding
  if (d.r < r0) d.r = r0;
  if (d.r > r1) d.r = r1;
  return d;
}

__global__ void seed_f64_kernel(GridGeom g, PlasmaSeed p, SpeciesF64 sp, size_t n0, size_t n) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Draw d = draw(g, p, i);
  const size_t j = n0 + i;
  sp.r[j] = d.r; sp.z[j] = d.z;
  sp.vr[j] = d.v[0]; sp.vphi[j] = d.v[1]; sp.vz[j] = d.v[2];
  sp.w[j] = d.w;
  sp.r_old[j] = 0; sp.z_old[j] = 0;
  if (sp.phi) { sp.phi[j] = 0; sp.phi_old[j] = 0; sp.sn[j] = 0; }
  if (sp.cell_r) { sp.cell_r[j] = (int)floor(d.r / g.dr); sp.cell_z[j] = (int)floor(d.z / g.dz); }
}

__global__ void seed_f32_kernel(GridGeom g, PlasmaSeed p, SpeciesF32Buffers b, size_t n0, size_t n) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Draw d = draw(g, p, i);
  const size_t j = n0 + i;
  const double x = d.r / g.dr, y = d.z / g.dz;
  double cx = floor(x), cy = floor(y);
  float fx = (float)(x - cx), fy = (float)(y - cy);
  if (fx >= 1.0f) { fx = 0.0f; cx += 1.0; }
  if (fy >= 1.0f) { fy = 0.0f; cy += 1.0; }
  b.cell[j] = pack_cell((int)cx, (int)cy);
  b.off_r[j] = fx;
  b.off_z[j] = fy;
  b.vr[j] = (float)d.v[0];
  b.vphi[j] = (float)d.v[1];
  b.vz[j] = (float)d.v[2];
  b.w[j] = (float)d.w;
  b.id[j] = b.next_id + (unsigned)i;
}

}  // namespace

void launch_seed_f64(const GridGeom& g, const PlasmaSeed& p, const SpeciesF64& sp, size_t n0,
                     size_t n, cudaStream_t s) {
  if (n) seed_f64_kernel<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, s>>>(g, p, sp, n0, n);
}

void launch_seed_f32(const GridGeom& g, const PlasmaSeed& p, const SpeciesF32Buffers& b,
                     size_t n0, size_t n, cudaStream_t s) {
  if (n) seed_f32_kernel<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, s>>>(g, p, b, n0, n);
}

}  // namespace pcg
