// pcg_maps.cu — SpecieP's diagnostic maps on the GPU.
//
// A particle's value v (its weight, a component of gamma m w v, or
// gamma m w |v|) spreads over the four nodes around it as
// weight_cylindrical does (weighter.hpp:27-130): a cloud of one cell
// centred on the particle, split at (i + 1/2) dr and (k + 1/2) dz, each
// part's ring volume over the node's CELL_VOLUME (the reference's macro
// expands CELL_VOLUME(i + 1) to 2i + 1 + 1), times v over the cloud's
// volume, with the reference's two axis branches (r <= dr/2: the cloud cut
// at r = 0; dr/2 < r <= dr: node 0's volume is CYL_VOL).  Per node the
// temperature and energy are energy_m(m, p^2 / n^2) in eV
// (specieP.cpp:679-710, 785-823), the momentum p / n (:825-839).  Sums are
// FP64 atomics, so they differ from the reference's particle-order sums in
// the last bits.
#include <cuda_runtime.h>

#include "pcg_f32.h"
#include "pcg_maps.h"

namespace pcg {

namespace {

constexpr int kThreads = 256;
constexpr double kPi = 3.1415926535897932;
constexpr double kRelLimit = 5e7, kRelLimit2 = kRelLimit * kRelLimit;
constexpr double kC2 = 3.0e8 * 3.0e8;
constexpr double kElCharge = 1.6e-19;

inline unsigned blocks_for(size_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

__device__ __forceinline__ void inc(const GridGeom& g, double* a, unsigned i, unsigned k, double v) {
  atomicAdd(a + (size_t)(i + 2) * g.ld + (k + 2), v);
}

__device__ void weight_cyl(const GridGeom& g, double* a, double pos_r, double pos_z, double value) {
  const double dr = g.dr, dz = g.dz;
  const unsigned ri = (unsigned)(int)floor(pos_r / dr), zk = (unsigned)(int)floor(pos_z / dz);
  double v1 = kPi * dz * dr * dr * (2.0 * ri + 1);
  const double v2 = kPi * dz * dr * dr * (2.0 * ri + 1 + 1);
  const double dz1 = (zk + 0.5) * dz - (pos_z - 0.5 * dz);
  const double dz2 = (pos_z + 0.5 * dz) - (zk + 0.5) * dz;
  const double r3 = pos_r + 0.5 * dr;
  double rho, w00, w01;  // node i's ring volumes of the two axial parts
  double r2;
  if (pos_r <= dr / 2.) {
    r2 = 0.5 * dr;
    rho = value / (kPi * dz * (2. * pos_r * pos_r + dr * dr / 2.));
    const double ring0 = dr * dr / 2. - pos_r * dr + pos_r * pos_r;
    w00 = kPi * dz1 * ring0;
    w01 = kPi * dz2 * ring0;
  } else {
    const double r1 = pos_r - 0.5 * dr;
    r2 = (ri + 0.5) * dr;
    rho = value / (2. * kPi * dz * dr * pos_r);
    if (pos_r <= dr) v1 = kPi * dz * dr * dr;  // CYL_VOL(dz, dr)
    w00 = kPi * dz1 * (r2 * r2 - r1 * r1);
    w01 = kPi * dz2 * (r2 * r2 - r1 * r1);
  }
  inc(g, a, ri, zk, rho * (w00 / v1));
  inc(g, a, ri + 1, zk, rho * (kPi * dz1 * (r3 * r3 - r2 * r2) / v2));
  inc(g, a, ri, zk + 1, rho * (w01 / v1));
  inc(g, a, ri + 1, zk + 1, rho * (kPi * dz2 * (r3 * r3 - r2 * r2) / v2));
}

// flags: 1 density, 2 momentum (3 grids), 4 absolute momentum
__global__ void weigh_kernel(GridGeom g, MapSpecies sp, int flags, int fixed, double* dens, double* m0,
                             double* m1, double* m2, double* abs_map) {
  const size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= sp.n) return;
  double pos_r, pos_z, v[3], w;
  if (sp.cell) {
    const int c = sp.cell[j];
    if (c < 0) return;
    pos_r = ((double)cell_r_of(c) + (double)sp.off_r[j]) * g.dr;
    pos_z = ((double)cell_z_of(c) + (double)sp.off_z[j]) * g.dz;
    v[0] = sp.vr32[j]; v[1] = sp.vphi32[j]; v[2] = sp.vz32[j];
    w = sp.w32[j];
  } else {
    pos_r = sp.r[j];
    if (!(pos_r >= 0.0)) return;
    pos_z = sp.z[j];
    v[0] = sp.vr[j]; v[1] = sp.vphi[j]; v[2] = sp.vz[j];
    w = sp.w[j];
  }
  if (flags & 1) weight_cyl(g, dens, pos_r, pos_z, w);
  if (flags & 2) {  // calc_momentum_w (specieP.cpp:740-782)
    const double mw = sp.mass * w;
    double p[3] = {mw * v[0], mw * v[1], mw * v[2]};
    const double v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    if (fixed || v2 < kRelLimit2) {
      const double gm = 1 / sqrt(1.0 - v2 / kC2);
      for (int c = 0; c < 3; ++c) p[c] *= gm;
    }
    weight_cyl(g, m0, pos_r, pos_z, p[0]);
    weight_cyl(g, m1, pos_r, pos_z, p[1]);
    weight_cyl(g, m2, pos_r, pos_z, p[2]);
  }
  if (flags & 4) {  // calc_momentum_abs_w (:714-738)
    const double va = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    double pa = sp.mass * w * va;
    if (fixed || va < kRelLimit) pa *= 1 / sqrt(1.0 - va * va / kC2);
    weight_cyl(g, abs_map, pos_r, pos_z, pa);
  }
}

// phys::rel::energy_m (rel.cpp:88-101)
__device__ __forceinline__ double energy_m(double mass, double p2) {
  if (p2 > kRelLimit2 * mass * mass) {
    const double e_rest = mass * kC2;
    return sqrt(p2 * kC2 + e_rest * e_rest) - e_rest;
  }
  return 0.5 * p2 / mass;
}

// per interior node (r < nr, z < nz); other nodes stay 0
__global__ void finish_kernel(GridGeom g, int which, double mass, const double* dens, const double* m0,
                              const double* m1, const double* m2, const double* abs_map, double* out,
                              size_t plane) {
  const size_t q0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (q0 >= (size_t)g.nr * g.nz) return;
  const int r = (int)(q0 / g.nz), z = (int)(q0 - (size_t)r * g.nz);
  const size_t q = (size_t)(r + 2) * g.ld + (z + 2);
  const double dl = dens[q];
  if (dl == 0) return;
  if (which == 3) {
    out[q] = m0[q] / dl;
    out[plane + q] = m1[q] / dl;
    out[2 * plane + q] = m2[q] / dl;
    return;
  }
  double p2 = abs_map[q] * abs_map[q];
  if (which == 1) p2 -= m0[q] * m0[q] + m1[q] * m1[q] + m2[q] * m2[q];
  p2 /= dl * dl;
  out[q] = energy_m(mass, p2) * (1. / kElCharge);
}

}  // namespace

int species_map(const GridGeom& g, const MapSpecies& sp, int which, int fixed, double* abs_map,
                double* scratch, double* out, cudaStream_t s) {
  if (which < 0 || which > 3) return -1;
  const size_t plane = (size_t)(g.nr + 4) * g.ld;
  double *dens = scratch, *m0 = scratch + plane, *m1 = scratch + 2 * plane, *m2 = scratch + 3 * plane;
  const bool need_abs = which == 2 || (which == 1 && fixed);
  int flags = 1 | ((which == 1 || which == 3) ? 2 : 0) | (need_abs ? 4 : 0);
  cudaMemsetAsync(scratch, 0, 4 * plane * sizeof(double), s);
  if (need_abs) cudaMemsetAsync(abs_map, 0, plane * sizeof(double), s);
  if (sp.n)
    weigh_kernel<<<blocks_for(sp.n), kThreads, 0, s>>>(g, sp, flags, fixed, dens, m0, m1, m2, abs_map);
  if (which == 0) {
    cudaMemcpyAsync(out, dens, plane * sizeof(double), cudaMemcpyDeviceToDevice, s);
  } else {
    cudaMemsetAsync(out, 0, (which == 3 ? 3 : 1) * plane * sizeof(double), s);
    const size_t cells = (size_t)g.nr * g.nz;
    finish_kernel<<<blocks_for(cells), kThreads, 0, s>>>(g, which, sp.mass, dens, m0, m1, m2, abs_map, out,
                                                         plane);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace pcg
