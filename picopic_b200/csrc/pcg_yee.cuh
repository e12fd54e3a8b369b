// pcg_yee.cuh — Yee FDTD update of E and H on the r-z grid with the 2-cell
// halo, one thread per node, for double (reference arithmetic) and float.
//
// MaxwellSolverYee::calc_field_e (maxwellSolverYee.cpp:161-257) and
// calc_field_h (:111-159) for one domain with all walls on: r_begin =
// z_begin = 1, r_end = nr-1, z_end = nz-1.  Every node's update reads only
// neighbours of the other field, so nodes are independent.
#pragma once

#include "pcg_common.cuh"

namespace pcg {

template <typename Real>
struct YeeArgs {
  GridGeom g;
  Real* E[3];
  Real* H[3];
  Real* Hat[3];
  Real* J[3];            // read by the E update
  const Real* sig_r;     // PML sigma per radial cell (r=R wall)
  const Real* sig_z0;    // per axial cell (z=0 wall)
  const Real* sig_zl;    // per axial cell (z=L wall)
  int zero_j;            // the fused step clears J after E consumed it
  DevStatus* st;
};

// E update over the whole (nr+4) x (nz+4) array: halo nodes are set to zero
// (Grid::overlay_set, grid.hpp:87-97), interior nodes follow the axis,
// z=0-wall and regular branches of calc_field_e.
template <typename Real>
__global__ void __launch_bounds__(256) yee_e_kernel(YeeArgs<Real> a) {
  const GridGeom& g = a.g;
  const int kk = blockIdx.x * blockDim.x + threadIdx.x;  // 0 .. nz+3
  const int ii = blockIdx.y;                              // 0 .. nr+3
  if (kk >= g.nz + 4) return;
  const int i = ii - 2, k = kk - 2;
  const long long p = (long long)ii * g.ld + kk;
  const bool halo = i < 0 || k < 0 || i >= g.nr || k >= g.nz;
  if (halo) {
    a.E[0][p] = 0; a.E[1][p] = 0; a.E[2][p] = 0;
    if (a.zero_j) { a.J[0][p] = 0; a.J[1][p] = 0; a.J[2][p] = 0; }
    return;
  }
  const bool axis = (i == 0) && (k >= 1) && (k < g.nz - 1);
  const bool wall = (k == 0) && (i >= 1) && (i < g.nr - 1);
  const bool reg = (i >= 1) && (i < g.nr - 1) && (k >= 1) && (k < g.nz - 1);
  if (axis || wall || reg) {
    const Real dr = (Real)g.dr, dz = (Real)g.dz, dt = (Real)g.dt;
    Real sigma = 0;
    sigma += a.sig_r[i];
    sigma += a.sig_z0[k];
    sigma += a.sig_zl[k];
    const Real epsx2 = (Real)(2 * kEpsilon0);
    const Real sigma_t = sigma * dt;
    const Real koef_e = (epsx2 - sigma_t) / (epsx2 + sigma_t);
    const Real koef_h = 2 * dt / (epsx2 + sigma_t);
    const long long pkm = p - 1, pim = p - g.ld;
    const Real *Hr = a.Hat[0], *Hp = a.Hat[1], *Hz = a.Hat[2];
    Real er = a.E[0][p], ep = a.E[1][p], ez = a.E[2][p];
    const Real jr = a.J[0][p], jp = a.J[1][p], jz = a.J[2][p];
    if (axis) {  // :170-194
      er *= koef_e;
      er -= (jr + (Hp[p] - Hp[pkm]) / dz) * koef_h;
      ez *= koef_e;
      ez -= (jz - Hp[p] * (Real)4. / dr) * koef_h;
    } else if (wall) {  // :196-218
      ez *= koef_e;
      ez -= (jz - (Hp[p] - Hp[pim]) / dr - (Hp[p] + Hp[pim]) / ((Real)2. * dr * (Real)i)) * koef_h;
    } else {  // :220-256
      er *= koef_e;
      er -= (jr + (Hp[p] - Hp[pkm]) / dz) * koef_h;
      ep *= koef_e;
      ep -= (jp - (Hr[p] - Hr[pkm]) / dz + (Hz[p] - Hz[pim]) / dr) * koef_h;
      ez *= koef_e;
      ez -= (jz - (Hp[p] - Hp[pim]) / dr - (Hp[p] + Hp[pim]) / ((Real)2. * dr * (Real)i)) * koef_h;
      if (isnan(er) || isnan(ep) || isnan(ez)) raise_error(a.st, kErrNanField);
    }
    a.E[0][p] = er; a.E[1][p] = ep; a.E[2][p] = ez;
  }
  if (a.zero_j) { a.J[0][p] = 0; a.J[1][p] = 0; a.J[2][p] = 0; }
}

// H update: halo of H and H_at_et set to zero, interior nodes follow
// calc_field_h including the reference's second H_r update on the outer
// row i = nr-1 (:119-130 then :133-141) unless `fixed`.
template <typename Real>
__global__ void __launch_bounds__(256) yee_h_kernel(YeeArgs<Real> a, int fixed) {
  const GridGeom& g = a.g;
  const int kk = blockIdx.x * blockDim.x + threadIdx.x;
  const int ii = blockIdx.y;
  if (kk >= g.nz + 4) return;
  const int i = ii - 2, k = kk - 2;
  const long long p = (long long)ii * g.ld + kk;
  if (i < 0 || k < 0 || i >= g.nr || k >= g.nz) {
    for (int c = 0; c < 3; ++c) { a.H[c][p] = 0; a.Hat[c][p] = 0; }
    return;
  }
  const Real dr = (Real)g.dr, dz = (Real)g.dz, dt = (Real)g.dt, mu = (Real)kMagnConst;
  const long long pk = p + 1, pi = p + g.ld;
  const Real *Er = a.E[0], *Ep = a.E[1], *Ez = a.E[2];
  Real hat_r = a.Hat[0][p];
  const Real a_r = dt * (Ep[pk] - Ep[p]) / (dz * mu);
  if (!fixed && i == g.nr - 1) hat_r += a_r;  // outer-wall loop, then the regular loop again
  a.H[0][p] = hat_r + a_r / 2;
  a.Hat[0][p] = hat_r + a_r;
  const Real a_phi = dt * ((Ez[pi] - Ez[p]) / dr - (Er[pk] - Er[p]) / dz) / mu;
  const Real hat_p = a.Hat[1][p];
  a.H[1][p] = hat_p + a_phi / 2;
  a.Hat[1][p] = hat_p + a_phi;
  const Real a_z = dt * ((Ep[pi] + Ep[p]) / ((Real)2. * dr * ((Real)i + (Real)0.5 + (Real)0.0)) +
                         (Ep[pi] - Ep[p]) / dr) / mu;
  const Real hat_z = a.Hat[2][p];
  a.H[2][p] = hat_z - a_z / 2;
  a.Hat[2][p] = hat_z - a_z;
}

}  // namespace pcg
