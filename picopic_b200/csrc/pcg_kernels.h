// pcg_kernels.h — device data views and kernel launchers shared by the host
// API (pcg_api.cu) and the kernel translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "pcg_common.cuh"

namespace pcg {

template <typename Real>
struct YeeArgs;

struct FieldsF64 {
  double* E[3];
  double* H[3];
  double* Hat[3];
  double* J[3];
  const double* sig_r;
  const double* sig_z0;
  const double* sig_zl;
  // external fields: E_r, E_phi, E_z, H_r, H_phi, H_z planes of (nr+4)(nz+4)
  // nodes, gathered and added to E and H by the push; null when none
  const double* ext = nullptr;
};

// One species in the double-precision layout (structure of arrays).
struct SpeciesF64 {
  size_t n;  // slots in use (dead slots have r < 0)
  double *r, *z, *vr, *vphi, *vz, *w, *r_old, *z_old;
  double *phi, *phi_old, *sn;  // stage-by-stage mode only, else null
  int *cell_r, *cell_z;        // stage-by-stage mode only, else null
  double charge, mass;         // SI
  double c2m;                  // charge * dt / (2 * mass), pusherBoris.cpp:67
  int is_beam;
};

// Per-step parameters of BeamP::inject (beamP.cpp:71-157).
struct BeamInject {
  uint64_t seed;
  uint32_t stream;
  uint64_t step;
  double domain_radius, dl, half_z, velocity, v_macro_avg, n_per_macro_avg;
  // Gaussian longitudinal profile (profile == 1): r^2 uniform in
  // [r_min^2, radius^2], weight w0 * exp(-(s - 3 sigma)^2 / (2 sigma^2)) with
  // s = head_dist - dl * u_z the particle's distance behind the bunch head.
  int profile;
  double r_min, radius, sigma, head_dist, w0;
};

// The shared particle placement of both layouts (beamP.cpp:100-145 for
// profile 0).  u[0], u[1] are the two Philox uniforms of the particle.
__host__ __device__ inline void beam_particle(const BeamInject& b, double dr, double dz,
                                              const double u[2], double* r, double* z,
                                              double* w) {
  if (b.profile == 1) {
    *r = sqrt(b.r_min * b.r_min + u[0] * (b.radius * b.radius - b.r_min * b.r_min));
    *z = b.dl * u[1] + b.half_z;
    const double s = b.head_dist - b.dl * u[1] - 3.0 * b.sigma;
    *w = b.w0 * exp(-s * s / (2.0 * b.sigma * b.sigma));
    return;
  }
  const double pos_r = b.domain_radius * u[0] + dr / 2 + 0.0 * dr;
  *r = pos_r;
  *z = b.dl * u[1] + b.half_z;
  double norm;
  if (pos_r > dr / 2)
    norm = 2 * 3.1415926535897932 * pos_r * dr * dz / b.v_macro_avg;
  else
    norm = 3.1415926535897932 * (pos_r * pos_r + pos_r * dr + dr * dr / 4.) * dz / b.v_macro_avg;
  *w = b.n_per_macro_avg * norm;
}

void launch_yee_e_f64(const YeeArgs<double>& a, cudaStream_t s);
void launch_yee_h_f64(const YeeArgs<double>& a, int fixed, cudaStream_t s);
void launch_stage_f64(int stage, const GridGeom& g, const FieldsF64& f, const SpeciesF64& sp,
                      int slot, int pusher, int fixed, DevStatus* st, cudaStream_t s);
void launch_current_stage_f64(const GridGeom& g, const FieldsF64& f, const SpeciesF64* sp,
                              int nsp, int fixed, int current, unsigned long long* reset,
                              DevStatus* st, cudaStream_t s);
void launch_advance_f64(const GridGeom& g, const FieldsF64& f, const SpeciesF64& sp, int slot,
                        int pusher, int fixed, int current, unsigned long long* reset,
                        DevStatus* st, cudaStream_t s, int do_push = 1);
void launch_deposit_f64(const GridGeom& g, const FieldsF64& f, const SpeciesF64& sp, int slot,
                        int fixed, int current, const unsigned long long* reset, DevStatus* st,
                        cudaStream_t s);
void launch_halo_zero_f64(const GridGeom& g, double* a0, double* a1, double* a2, cudaStream_t s);
void launch_inject_f64(const GridGeom& g, const SpeciesF64& sp, size_t n0, unsigned count,
                       const BeamInject& b, cudaStream_t s);
void launch_import_f64(const GridGeom& g, const SpeciesF64& sp, size_t n0, size_t n,
                       const double* src, cudaStream_t s);
void launch_gather_f64(const double* src, double* dst, const unsigned* idx, size_t n, cudaStream_t s);
void launch_gather_i32(const int* src, int* dst, const unsigned* idx, size_t n, cudaStream_t s);

}  // namespace pcg

namespace pcg {

// Utilities (pcg_util.cu)
void f64_alive_flags(const double* r, unsigned char* flags, size_t n, cudaStream_t s);
void iota_u32(unsigned* a, size_t n, cudaStream_t s);
// Field energies over interior nodes: sum of eps0/2 |E|^2 V_i and mu0/2 |H|^2 V_i
// with V_i = PI dz dr^2 (2i+1), H taken at the centred time (field_h).
int f64_energies(const GridGeom& g, const FieldsF64& f, double* ee, double* eh, cudaStream_t s);
// Kinetic energy sum w m v^2 gamma^2/(gamma+1) of live particles (r >= 0).
int f64_kinetic(const double* vr, const double* vphi, const double* vz, const double* w,
                const double* r, size_t n, double mass, double* out, cudaStream_t s);

}  // namespace pcg
