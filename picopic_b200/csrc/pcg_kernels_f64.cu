// pcg_kernels_f64.cu — the double-precision particle path: one kernel per
// reference stage (used by pcg_stage for stage-by-stage parity) and the
// fused two-kernel step used by pcg_step.  Built with --fmad=false so that
// the arithmetic follows the reference operation order.
#include <cuda_runtime.h>

#include "pcg_f64.cuh"
#include "pcg_kernels.h"
#include "pcg_philox.cuh"
#include "pcg_yee.cuh"

namespace pcg {

using namespace f64;

namespace {

constexpr int kThreads = 256;

__host__ __device__ inline Fields make_fields(const FieldsF64& d) {
  Fields f;
  for (int c = 0; c < 3; ++c) {
    f.E[c] = d.E[c]; f.H[c] = d.H[c]; f.Hat[c] = d.Hat[c]; f.J[c] = d.J[c];
  }
  f.sig_r = d.sig_r; f.sig_z0 = d.sig_z0; f.sig_zl = d.sig_zl;
  f.ext = d.ext;
  return f;
}

inline unsigned blocks_for(size_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

// ---------------------------------------------------------------------------
// Stage kernels (one per Domain method)

template <bool EXT>
__global__ void push_kernel(GridGeom g, FieldsF64 fd, SpeciesF64 sp, int pusher, int fixed,
                            DevStatus* st) {
  size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= sp.n) return;
  if (sp.r[j] < 0) return;  // dead slot
  Fields f = make_fields(fd);
  double v[3] = {sp.vr[j], sp.vphi[j], sp.vz[j]};
  if (!gather_push<EXT>(g, f, pusher, fixed, sp.c2m, sp.r[j], sp.z[j], v, st)) return;
  sp.vr[j] = v[0]; sp.vphi[j] = v[1]; sp.vz[j] = v[2];
}

__global__ void dump_old_kernel(SpeciesF64 sp) {
  size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= sp.n) return;
  sp.r_old[j] = sp.r[j]; sp.phi_old[j] = sp.phi[j]; sp.z_old[j] = sp.z[j];
}

__global__ void move_kernel(SpeciesF64 sp, double dt) {  // mover_cylindrical :482-491
  size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= sp.n || sp.r[j] < 0) return;
  sp.r[j] = sp.r[j] + sp.vr[j] * dt;
  sp.phi[j] = sp.phi[j] + sp.vphi[j] * dt;
  sp.z[j] = sp.z[j] + sp.vz[j] * dt;
}

__global__ void pos_rz_kernel(SpeciesF64 sp) {  // back_position_to_rz :609-622
  size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= sp.n || sp.r[j] < 0) return;
  double pr = sp.r[j], pp = sp.phi[j];
  double r = sqrt(pr * pr + pp * pp);
  sp.sn[j] = pp / r;
  sp.r[j] = r;
  sp.phi[j] = 0;
}

__global__ void reflect_kernel(GridGeom g, SpeciesF64 sp, int fixed, DevStatus* st) {
  size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= sp.n || sp.r[j] < 0) return;
  double r = sp.r[j], z = sp.z[j], vr = sp.vr[j], vz = sp.vz[j];
  if (sp.is_beam) {
    reflect_beam(g, &r, &vr);
  } else if (!reflect_one(g, fixed, &r, &z, sp.r_old[j], sp.z_old[j], &vr, &vz)) {
    raise_error(st, kErrReflectLoop);
  }
  sp.r[j] = r; sp.z[j] = z; sp.vr[j] = vr; sp.vz[j] = vz;
}

__global__ void vel_rz_kernel(SpeciesF64 sp) {  // back_velocity_to_rz :624-640
  size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= sp.n || sp.r[j] < 0) return;
  double sn = sp.sn[j];
  double cs = sqrt(1 - sn * sn);
  double vr = sp.vr[j], vp = sp.vphi[j];
  double u2 = cs * vr - sn * vp;
  double v2 = sn * vr + cs * vp;
  sp.vr[j] = u2;
  sp.vphi[j] = v2;
}

__global__ void bind_kernel(GridGeom g, SpeciesF64 sp) {  // bind_cell_numbers :652-663
  size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= sp.n || sp.r[j] < 0) return;
  sp.cell_r[j] = cell_number(sp.r[j], g.dr);
  sp.cell_z[j] = cell_number(sp.z[j], g.dz);
}

// Runaway test of SMB.cpp:252-337 for one domain: marks the slot dead.
__global__ void collect_mark_kernel(GridGeom g, SpeciesF64 sp, DevStatus* st) {
  size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= sp.n || sp.r[j] < 0) return;
  int cr = sp.cell_r[j], cz = sp.cell_z[j];
  if (cr < 0 || cz < 0 || cr >= g.nr || cz >= g.nz) {
    sp.r[j] = -1.0;
    atomicAdd(&st->removed, 1ull);
    atomicAdd(&st->dead_slots, 1ull);
  }
}

// The strict-axial J_r overwrite of currentVB.cpp:545-546: record, per J_r
// node, the last particle (in reference order) that overwrites it.
__global__ void vb_reset_kernel(GridGeom g, SpeciesF64 sp, int slot, int fixed,
                                unsigned long long* reset) {
  size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= sp.n || sp.r[j] < 0) return;
  int i_n, k_n;
  if (vb_strict_axial_nodes(g, fixed, sp.r[j], sp.z[j], sp.r_old[j], sp.z_old[j], sp.cell_r[j],
                            &i_n, &k_n)) {
    unsigned long long o1 = particle_order(slot, j) + 1;
    atomicMax(reset + gidx(g, i_n, k_n), o1);
    atomicMax(reset + gidx(g, i_n, k_n + 1), o1);
  }
}

__global__ void zero_reset_nodes_kernel(long long nodes, const unsigned long long* reset,
                                        double* jr) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p < nodes && reset[p] != 0) jr[p] = 0.0;
}

__global__ void halo_zero_kernel(GridGeom g, double* a0, double* a1, double* a2) {
  const int kk = blockIdx.x * blockDim.x + threadIdx.x;
  const int ii = blockIdx.y;
  if (kk >= g.nz + 4) return;
  const int i = ii - 2, k = kk - 2;
  if (i < 0 || k < 0 || i >= g.nr || k >= g.nz) {
    long long p = (long long)ii * g.ld + kk;
    a0[p] = 0; a1[p] = 0; a2[p] = 0;
  }
}

__global__ void vb_azimuthal_kernel(GridGeom g, FieldsF64 fd, SpeciesF64 sp) {
  size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= sp.n || sp.r[j] < 0) return;
  Sink s{{fd.J[0], fd.J[1], fd.J[2]}, nullptr, 0, &g, false};
  vb_azimuthal(s, sp.charge * sp.w[j], sp.r[j], sp.z[j], sp.r_old[j], sp.z_old[j], sp.vphi[j],
               sp.cell_r[j], sp.cell_z[j]);
}

__global__ void vb_rz_kernel(GridGeom g, FieldsF64 fd, SpeciesF64 sp, int slot, int fixed,
                             const unsigned long long* reset, DevStatus* st) {
  size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= sp.n || sp.r[j] < 0) return;
  Sink s{{fd.J[0], fd.J[1], fd.J[2]}, reset, particle_order(slot, j) + 1, &g, false};
  if (!vb_rz(s, fixed, sp.charge * sp.w[j], sp.r[j], sp.z[j], sp.r_old[j], sp.z_old[j],
             sp.cell_r[j], sp.cell_z[j]))
    atomicAdd(&st->move_errors, 1ull);
}

__global__ void zigzag_kernel(GridGeom g, FieldsF64 fd, SpeciesF64 sp) {
  size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= sp.n || sp.r[j] < 0) return;
  Sink s{{fd.J[0], fd.J[1], fd.J[2]}, nullptr, 0, &g, false};
  zigzag(s, sp.charge, sp.w[j], sp.vphi[j], sp.r[j], sp.z[j], sp.r_old[j], sp.z_old[j]);
}

// ---------------------------------------------------------------------------
// Fused step, kernel 1: push, move, rotate, reflect, rotate back, bind and
// the runaway test in registers; stores new and old positions and marks the
// strict-axial J_r overwrites.  Without do_push the velocities are taken as
// pushed already (the step of a run with collisions, which act between the
// push and the move).
template <bool EXT>
__global__ void __launch_bounds__(kThreads) advance_kernel(GridGeom g, FieldsF64 fd, SpeciesF64 sp,
                                                           int slot, int pusher, int fixed,
                                                           int current, unsigned long long* reset,
                                                           DevStatus* st, int do_push) {
  const size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= sp.n) return;
  double r = sp.r[j];
  if (r < 0) return;
  double z = sp.z[j];
  Fields f = make_fields(fd);
  double v[3] = {sp.vr[j], sp.vphi[j], sp.vz[j]};
  if (do_push && !gather_push<EXT>(g, f, pusher, fixed, sp.c2m, r, z, v, st)) return;
  const double r_old = r, z_old = z;                 // dump_position_to_old (phi = 0)
  const double X = r + v[0] * g.dt;                  // mover_cylindrical
  const double Y = 0 + v[1] * g.dt;
  z = z + v[2] * g.dt;
  const double rr = sqrt(X * X + Y * Y);             // back_position_to_rz
  const double sn = Y / rr;
  r = rr;
  if (sp.is_beam) reflect_beam(g, &r, &v[0]);        // reflect
  else if (!reflect_one(g, fixed, &r, &z, r_old, z_old, &v[0], &v[2])) raise_error(st, kErrReflectLoop);
  const double cs = sqrt(1 - sn * sn);               // back_velocity_to_rz
  const double u2 = cs * v[0] - sn * v[1];
  const double v2 = sn * v[0] + cs * v[1];
  v[0] = u2; v[1] = v2;
  const int cr = cell_number(r, g.dr), cz = cell_number(z, g.dz);  // bind
  sp.vr[j] = v[0]; sp.vphi[j] = v[1]; sp.vz[j] = v[2];
  sp.r_old[j] = r_old; sp.z_old[j] = z_old;
  if (cr < 0 || cz < 0 || cr >= g.nr || cz >= g.nz) {  // runaway collector
    sp.r[j] = -1.0;
    atomicAdd(&st->removed, 1ull);
    atomicAdd(&st->dead_slots, 1ull);
    return;
  }
  sp.r[j] = r; sp.z[j] = z;
  if (current == 0) {
    int i_n, k_n;
    if (vb_strict_axial_nodes(g, fixed, r, z, r_old, z_old, cr, &i_n, &k_n)) {
      const unsigned long long o1 = particle_order(slot, j) + 1;
      atomicMax(reset + gidx(g, i_n, k_n), o1);
      atomicMax(reset + gidx(g, i_n, k_n + 1), o1);
    }
  }
}

// Fused step, kernel 2: the particle's current, after all overwrites are known.
__global__ void __launch_bounds__(kThreads) deposit_kernel(GridGeom g, FieldsF64 fd, SpeciesF64 sp,
                                                           int slot, int fixed, int current,
                                                           const unsigned long long* reset,
                                                           DevStatus* st) {
  const size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= sp.n) return;
  const double r = sp.r[j];
  if (r < 0) return;
  const double z = sp.z[j], ro = sp.r_old[j], zo = sp.z_old[j];
  const double q = sp.charge * sp.w[j];
  if (current == 1) {
    Sink s{{fd.J[0], fd.J[1], fd.J[2]}, nullptr, 0, &g, false};
    zigzag(s, sp.charge, sp.w[j], sp.vphi[j], r, z, ro, zo);
    return;
  }
  const int cr = cell_number(r, g.dr), cz = cell_number(z, g.dz);
  Sink s{{fd.J[0], fd.J[1], fd.J[2]}, reset, particle_order(slot, j) + 1, &g, true};
  vb_azimuthal(s, q, r, z, ro, zo, sp.vphi[j], cr, cz);
  if (!vb_rz(s, fixed, q, r, z, ro, zo, cr, cz)) atomicAdd(&st->move_errors, 1ull);
}

// BeamP::inject (beamP.cpp:100-145) for `count` particles starting at slot
// n0, with Philox uniforms in place of std::mt19937.
__global__ void inject_kernel(GridGeom g, SpeciesF64 sp, size_t n0, unsigned count,
                              BeamInject b) {
  unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const double dr = g.dr, dz = g.dz;
  double u[2];
  philox_uniform2(b.seed, b.stream, b.step, i, u);
  double pos_r, pos_z, w;
  beam_particle(b, dr, dz, u, &pos_r, &pos_z, &w);
  size_t j = n0 + i;
  sp.r[j] = pos_r;
  sp.z[j] = pos_z;
  sp.vr[j] = 0; sp.vphi[j] = 0; sp.vz[j] = b.velocity;
  sp.w[j] = w;
  sp.r_old[j] = 0; sp.z_old[j] = 0;
  if (sp.phi) { sp.phi[j] = 0; sp.phi_old[j] = 0; sp.sn[j] = 0; }
  if (sp.cell_r) { sp.cell_r[j] = cell_number(pos_r, dr); sp.cell_z[j] = cell_number(pos_r, dz); }
}

// Host doubles -> device state, with the cell binding of SpecieP.
__global__ void import_kernel(GridGeom g, SpeciesF64 sp, size_t n0, size_t n, const double* src) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  size_t j = n0 + i;
  const double r = src[i], z = src[n + i];
  sp.r[j] = r; sp.z[j] = z;
  sp.vr[j] = src[2 * n + i]; sp.vphi[j] = src[3 * n + i]; sp.vz[j] = src[4 * n + i];
  sp.w[j] = src[5 * n + i];
  sp.r_old[j] = 0; sp.z_old[j] = 0;
  if (sp.phi) { sp.phi[j] = 0; sp.phi_old[j] = 0; sp.sn[j] = 0; }
  if (sp.cell_r) { sp.cell_r[j] = cell_number(r, g.dr); sp.cell_z[j] = cell_number(z, g.dz); }
}

template <typename T>
__global__ void compact_gather_kernel(const T* src, T* dst, const unsigned* idx, size_t n) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[idx[i]];
}

}  // namespace

// ---------------------------------------------------------------------------
// Host launchers

void launch_yee_e_f64(const YeeArgs<double>& a, cudaStream_t s) {
  dim3 grid((a.g.nz + 4 + kThreads - 1) / kThreads, a.g.nr + 4);
  yee_e_kernel<double><<<grid, kThreads, 0, s>>>(a);
}

void launch_yee_h_f64(const YeeArgs<double>& a, int fixed, cudaStream_t s) {
  dim3 grid((a.g.nz + 4 + kThreads - 1) / kThreads, a.g.nr + 4);
  yee_h_kernel<double><<<grid, kThreads, 0, s>>>(a, fixed);
}

void launch_stage_f64(int stage, const GridGeom& g, const FieldsF64& f, const SpeciesF64& sp,
                      int slot, int pusher, int fixed, DevStatus* st, cudaStream_t s) {
  if (sp.n == 0) return;
  unsigned nb = blocks_for(sp.n);
  switch (stage) {
    case 3:
      if (f.ext) push_kernel<true><<<nb, kThreads, 0, s>>>(g, f, sp, pusher, fixed, st);
      else push_kernel<false><<<nb, kThreads, 0, s>>>(g, f, sp, pusher, fixed, st);
      break;
    case 4: dump_old_kernel<<<nb, kThreads, 0, s>>>(sp); break;
    case 5: move_kernel<<<nb, kThreads, 0, s>>>(sp, g.dt); break;
    case 6: pos_rz_kernel<<<nb, kThreads, 0, s>>>(sp); break;
    case 7: reflect_kernel<<<nb, kThreads, 0, s>>>(g, sp, fixed, st); break;
    case 8: vel_rz_kernel<<<nb, kThreads, 0, s>>>(sp); break;
    case 9: bind_kernel<<<nb, kThreads, 0, s>>>(g, sp); break;
    case 10: collect_mark_kernel<<<nb, kThreads, 0, s>>>(g, sp, st); break;
    default: break;
  }
  (void)slot;
}

void launch_current_stage_f64(const GridGeom& g, const FieldsF64& f, const SpeciesF64* sp,
                              int nsp, int fixed, int current, unsigned long long* reset,
                              DevStatus* st, cudaStream_t s) {
  dim3 hgrid((g.nz + 4 + kThreads - 1) / kThreads, g.nr + 4);
  const long long nodes = (long long)(g.nr + 4) * g.ld;
  if (current == 1) {  // CurrentZigZag::current_distribution :22-136
    halo_zero_kernel<<<hgrid, kThreads, 0, s>>>(g, f.J[0], f.J[1], f.J[2]);
    for (int t = 0; t < nsp; ++t)
      if (sp[t].n) zigzag_kernel<<<blocks_for(sp[t].n), kThreads, 0, s>>>(g, f, sp[t]);
    return;
  }
  // CurrentVB::current_distribution :731-735: azimuthal, then rz, each
  // starting with overlay_set(0) on J.
  halo_zero_kernel<<<hgrid, kThreads, 0, s>>>(g, f.J[0], f.J[1], f.J[2]);
  for (int t = 0; t < nsp; ++t)
    if (sp[t].n) vb_azimuthal_kernel<<<blocks_for(sp[t].n), kThreads, 0, s>>>(g, f, sp[t]);
  halo_zero_kernel<<<hgrid, kThreads, 0, s>>>(g, f.J[0], f.J[1], f.J[2]);
  cudaMemsetAsync(reset, 0, sizeof(unsigned long long) * nodes, s);
  for (int t = 0; t < nsp; ++t)
    if (sp[t].n) vb_reset_kernel<<<blocks_for(sp[t].n), kThreads, 0, s>>>(g, sp[t], t, fixed, reset);
  zero_reset_nodes_kernel<<<(unsigned)((nodes + kThreads - 1) / kThreads), kThreads, 0, s>>>(nodes, reset, f.J[0]);
  for (int t = 0; t < nsp; ++t)
    if (sp[t].n) vb_rz_kernel<<<blocks_for(sp[t].n), kThreads, 0, s>>>(g, f, sp[t], t, fixed, reset, st);
}

void launch_advance_f64(const GridGeom& g, const FieldsF64& f, const SpeciesF64& sp, int slot,
                        int pusher, int fixed, int current, unsigned long long* reset,
                        DevStatus* st, cudaStream_t s, int do_push) {
  if (sp.n == 0) return;
  auto k = f.ext ? advance_kernel<true> : advance_kernel<false>;
  k<<<blocks_for(sp.n), kThreads, 0, s>>>(g, f, sp, slot, pusher, fixed, current, reset, st,
                                                       do_push);
}

void launch_deposit_f64(const GridGeom& g, const FieldsF64& f, const SpeciesF64& sp, int slot,
                        int fixed, int current, const unsigned long long* reset, DevStatus* st,
                        cudaStream_t s) {
  if (sp.n == 0) return;
  deposit_kernel<<<blocks_for(sp.n), kThreads, 0, s>>>(g, f, sp, slot, fixed, current, reset, st);
}

void launch_halo_zero_f64(const GridGeom& g, double* a0, double* a1, double* a2, cudaStream_t s) {
  dim3 hgrid((g.nz + 4 + kThreads - 1) / kThreads, g.nr + 4);
  halo_zero_kernel<<<hgrid, kThreads, 0, s>>>(g, a0, a1, a2);
}

void launch_inject_f64(const GridGeom& g, const SpeciesF64& sp, size_t n0, unsigned count,
                       const BeamInject& b, cudaStream_t s) {
  if (count == 0) return;
  inject_kernel<<<(count + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, sp, n0, count, b);
}

void launch_import_f64(const GridGeom& g, const SpeciesF64& sp, size_t n0, size_t n,
                       const double* src, cudaStream_t s) {
  if (n == 0) return;
  import_kernel<<<blocks_for(n), kThreads, 0, s>>>(g, sp, n0, n, src);
}

void launch_gather_f64(const double* src, double* dst, const unsigned* idx, size_t n, cudaStream_t s) {
  if (n) compact_gather_kernel<double><<<blocks_for(n), kThreads, 0, s>>>(src, dst, idx, n);
}

void launch_gather_i32(const int* src, int* dst, const unsigned* idx, size_t n, cudaStream_t s) {
  if (n) compact_gather_kernel<int><<<blocks_for(n), kThreads, 0, s>>>(src, dst, idx, n);
}

}  // namespace pcg
