// pcg_f64.cuh — the reference arithmetic in double precision, on the device.
//
// Every expression keeps the operation order of the reference source it
// cites, so that with FMA contraction off (the translation units that
// include this header are built with --fmad=false) the results equal the
// reference up to the last bit of log/pow and the order of atomic sums.
#pragma once

#include "pcg_common.cuh"

namespace pcg {
namespace f64 {

struct Fields {
  double* E[3];
  double* H[3];
  double* Hat[3];
  double* J[3];
  const double* sig_r;   // PML sigma contribution of the r=R wall, per radial cell
  const double* sig_z0;  // of the z=0 wall, per axial cell
  const double* sig_zl;  // of the z=L wall, per axial cell
  const double* ext;     // external E (3 planes) then H (3 planes), or null
};

__device__ __forceinline__ int cell_number(double pos, double dx) {  // geometry.hpp:198
  return (int)floor(pos / dx);
}

// CELL_VOLUME(i, dr, dz) with the reference's unparenthesised argument:
// the caller passes the already expanded factor (e.g. 2.0*i + 1 + 1).
__device__ __forceinline__ double cell_volume(double factor, double dr, double dz) {
  return kPi * dz * dr * dr * factor;
}

// field * CYL_RNG_VOL(dz_, ra, rb) / vol, expanded left to right.
__device__ __forceinline__ double ring_term(double f, double dzz, double ra, double rb, double vol) {
  return f * kPi * dzz * (rb * rb - ra * ra) / vol;
}

// PML sigma at an interior node, summed in the order of set_pml
// (maxwellSolverYee.cpp:57-109): r=R wall, then z=0, then z=L.
__device__ __forceinline__ double pml_sigma(const Fields& f, int i, int k) {
  double s = 0.0;
  s += f.sig_r[i];
  s += f.sig_z0[k];
  s += f.sig_zl[k];
  return s;
}

// ---------------------------------------------------------------------------
// Gather: MaxwellSolver::get_field_h / get_field_e (maxwellSolver.hpp:101-316)

// The fixed mode divides each ring term by the volume of the particle's
// cloud, pi dz (r3^2 - r1^2), so that a component's weights sum to 1; the
// reference divides by cell volumes, which weights a uniform field by about
// 1 - 1/(2i) at row i and lowers the plasma frequency by half that.
__device__ __forceinline__ void gather_h(const GridGeom& g, const Fields& f, bool fixed, double radius,
                                         double longitude, double cmp[3]) {
  const double dr = g.dr, dz = g.dz;
  const double *Hr = f.H[0], *Hp = f.H[1], *Hz = f.H[2];
  const double r1 = radius - 0.5 * dr, r3 = radius + 0.5 * dr;
  const double cloud = kPi * dz * (r3 * r3 - r1 * r1);
  double r2, dz1, dz2, v1, v2;
  int i, k;
  cmp[0] = cmp[1] = cmp[2] = 0;
  i = cell_number(radius - 0.5 * dr, dr);  // H_z :120-147
  k = cell_number(longitude, dz);
  v1 = cell_volume(2.0 * i + 1 + 1, dr, dz);
  v2 = cell_volume(2.0 * i + 3 + 1, dr, dz);
  if (fixed) v1 = v2 = cloud;
  dz1 = (k + 1) * dz - longitude;
  dz2 = longitude - k * dz;
  r2 = (i + 1) * dr;
  cmp[2] += ring_term(Hz[gidx(g, i, k)], dz1, r1, r2, v1);
  cmp[2] += ring_term(Hz[gidx(g, i + 1, k)], dz1, r2, r3, v2);
  cmp[2] += ring_term(Hz[gidx(g, i, k + 1)], dz2, r1, r2, v1);
  cmp[2] += ring_term(Hz[gidx(g, i + 1, k + 1)], dz2, r2, r3, v2);
  i = cell_number(radius, dr);  // H_r :149-177
  k = cell_number(longitude - 0.5 * dz, dz);
  v1 = cell_volume(2.0 * i + 1, dr, dz);
  v2 = cell_volume(2.0 * i + 2 + 1, dr, dz);
  if (fixed) v1 = v2 = cloud;
  r2 = (i + 0.5) * dr;
  dz1 = (k + 1.5) * dz - longitude;
  dz2 = longitude - (k + 0.5) * dz;
  cmp[0] += ring_term(Hr[gidx(g, i, k)], dz1, r1, r2, v1);
  cmp[0] += ring_term(Hr[gidx(g, i + 1, k)], dz1, r2, r3, v2);
  cmp[0] += ring_term(Hr[gidx(g, i, k + 1)], dz2, r1, r2, v1);
  cmp[0] += ring_term(Hr[gidx(g, i + 1, k + 1)], dz2, r2, r3, v2);
  i = cell_number(radius - 0.5 * dr, dr);  // H_phi :179-206
  k = cell_number(longitude - 0.5 * dz, dz);
  r2 = (i + 1) * dr;
  v1 = cell_volume(2.0 * i + 1 + 1, dr, dz);
  v2 = cell_volume(2.0 * i + 3 + 1, dr, dz);
  if (fixed) v1 = v2 = cloud;
  dz1 = (k + 1.5) * dz - longitude;
  dz2 = longitude - (k + 0.5) * dz;
  cmp[1] += ring_term(Hp[gidx(g, i, k)], dz1, r1, r2, v1);
  cmp[1] += ring_term(Hp[gidx(g, i + 1, k)], dz1, r2, r3, v2);
  cmp[1] += ring_term(Hp[gidx(g, i, k + 1)], dz2, r1, r2, v1);
  cmp[1] += ring_term(Hp[gidx(g, i + 1, k + 1)], dz2, r2, r3, v2);
}

__device__ __forceinline__ void gather_e(const GridGeom& g, const Fields& f, bool fixed,
                                         double radius, double longitude, double cmp[3]) {
  const double dr = g.dr, dz = g.dz;
  const double *Er = f.E[0], *Ep = f.E[1], *Ez = f.E[2];
  const double r1 = radius - 0.5 * dr, r3 = radius + 0.5 * dr;
  const double cloud = kPi * dz * (r3 * r3 - r1 * r1);
  double r2, dz1, dz2, v1, v2;
  int i, k;
  cmp[0] = cmp[1] = cmp[2] = 0;
  i = cell_number(radius - 0.5 * dr, dr);  // E_r :231-257
  k = cell_number(longitude, dz);
  v1 = cell_volume(2.0 * i + 1 + 1, dr, dz);
  v2 = cell_volume(2.0 * i + 3 + 1, dr, dz);
  if (fixed) v1 = v2 = cloud;
  dz1 = (k + 1) * dz - longitude;
  dz2 = longitude - k * dz;
  r2 = (i + 1) * dr;
  cmp[0] += ring_term(Er[gidx(g, i, k)], dz1, r1, r2, v1);
  cmp[0] += ring_term(Er[gidx(g, i + 1, k)], dz1, r2, r3, v2);
  cmp[0] += ring_term(Er[gidx(g, i, k + 1)], dz2, r1, r2, v1);
  cmp[0] += ring_term(Er[gidx(g, i + 1, k + 1)], dz2, r2, r3, v2);
  i = cell_number(radius, dr);  // E_z :259-283
  k = cell_number(longitude - 0.5 * dz, dz);
  v1 = cell_volume(2.0 * i + 1, dr, dz);
  v2 = cell_volume(2.0 * i + 2 + 1, dr, dz);
  if (fixed) v1 = v2 = cloud;
  r2 = (i + 0.5) * dr;
  dz1 = (k + 1.5) * dz - longitude;
  dz2 = longitude - (k + 0.5) * dz;
  cmp[2] += ring_term(Ez[gidx(g, i, k)], dz1, r1, r2, v1);
  cmp[2] += ring_term(Ez[gidx(g, i + 1, k)], dz1, r2, r3, v2);
  cmp[2] += ring_term(Ez[gidx(g, i, k + 1)], dz2, r1, r2, v1);
  cmp[2] += ring_term(Ez[gidx(g, i + 1, k + 1)], dz2, r2, r3, v2);
  i = cell_number(radius, dr);  // E_phi :285-313
  k = cell_number(longitude, dz);
  v1 = cell_volume(2.0 * i + 1, dr, dz);
  v2 = cell_volume(2.0 * i + 2 + 1, dr, dz);
  if (fixed) v1 = v2 = cloud;
  r2 = (i + 0.5) * dr;
  dz1 = (k + 1) * dz - longitude;
  dz2 = longitude - k * dz;
  cmp[1] += ring_term(Ep[gidx(g, i, k)], dz1, r1, r2, v1);
  cmp[1] += ring_term(Ep[gidx(g, i + 1, k)], dz1, r2, r3, v2);
  cmp[1] += ring_term(Ep[gidx(g, i, k + 1)], dz2, r1, r2, v1);
  // the reference adds the [i+1][k+1] E_phi term to E_z (:313)
  double t = ring_term(Ep[gidx(g, i + 1, k + 1)], dz2, r2, r3, v2);
  if (fixed) cmp[1] += t; else cmp[2] += t;
}

// ---------------------------------------------------------------------------
// Relativity (rel.cpp:24-55) and pushers

__device__ __forceinline__ double len2(const double v[3]) {
  return v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
}

__device__ __forceinline__ bool lorenz_factor(double sq, double* gamma, DevStatus* st) {
  double beta = sq / kLightVel2;
  if (beta > 1) {
    raise_error(st, kErrSuperluminal);
    return false;
  }
  double gm = 1 / sqrt(1.0 - beta);
  if (isinf(gm)) gm = 1e100;
  *gamma = gm;
  return true;
}

__device__ __forceinline__ double lorenz_factor_inv(double sq) {
  return pow(1.0 + sq / kLightVel2, -0.5);
}

// PusherBoris::operator() (pusherBoris.cpp:23-151); mode: 0 classic,
// 1 adaptive (relativistic above REL_LIMIT), 2 relativistic.
__device__ __forceinline__ bool push_boris(int mode, double c2m, const double e_in[3],
                                           const double b_in[3], double v[3], DevStatus* st) {
  double e[3] = {e_in[0] * c2m, e_in[1] * c2m, e_in[2] * c2m};
  const double bk = c2m * kMagnConst;
  double b[3] = {b_in[0] * bk, b_in[1] * bk, b_in[2] * bk};
  double gamma = 1;
  bool use_rel = (mode == 2) ||
                 (mode == 1 && pow(v[0], 2) + pow(v[1], 2) + pow(v[2], 2) > kRelLimit2);
  if (use_rel) {
    if (!lorenz_factor(len2(v), &gamma, st)) return false;
    for (int c = 0; c < 3; ++c) v[c] *= gamma;
  }
  for (int c = 0; c < 3; ++c) v[c] += e[c];
  if (use_rel) {
    gamma = lorenz_factor_inv(len2(v));
    for (int c = 0; c < 3; ++c) b[c] *= gamma;
  }
  const double const2 = 2. / (1. + len2(b));
  const double t0 = v[0], t1 = v[1], t2 = v[2];
  v[0] = t0 + const2 * ((t1 - t0 * b[2] + t2 * b[0]) * b[2] - (t2 + t0 * b[1] - t1 * b[0]) * b[1]);
  v[1] = t1 + const2 * (-(t0 + t1 * b[2] - t2 * b[1]) * b[2] + (t2 + t0 * b[1] - t1 * b[0]) * b[0]);
  v[2] = t2 + const2 * ((t0 + t1 * b[2] - t2 * b[1]) * b[1] - (t1 - t0 * b[2] + t2 * b[0]) * b[0]);
  for (int c = 0; c < 3; ++c) v[c] += e[c];
  if (use_rel) {
    gamma = lorenz_factor_inv(len2(v));
    for (int c = 0; c < 3; ++c) v[c] *= gamma;
  }
  return true;
}

__device__ __forceinline__ double dot3(const double a[3], const double b[3]) {
  double r = 0;
  for (int c = 0; c < 3; ++c) r += a[c] * b[c];
  return r;
}

// PusherVay::operator() (pusherVay.cpp:22-114).  `fixed` normalises u by c,
// which the reference omits (:81).
__device__ __forceinline__ bool push_vay(bool fixed, double c2m, const double e_in[3],
                                         const double b_in[3], double v[3], DevStatus* st) {
  double e[3] = {e_in[0], e_in[1], e_in[2]}, b[3] = {b_in[0], b_in[1], b_in[2]};
  double up[3], psm[3], gamma, s, us2, alpha, B2;
  if (!lorenz_factor(len2(v), &gamma, st)) return false;
  for (int c = 0; c < 3; ++c) v[c] *= gamma;
  if (fixed)
    for (int c = 0; c < 3; ++c) v[c] /= kLightVel;
  for (int c = 0; c < 3; ++c) up[c] = v[c];
  const double ek = 2. * c2m;
  for (int c = 0; c < 3; ++c) e[c] *= ek;
  if (fixed)
    for (int c = 0; c < 3; ++c) e[c] /= kLightVel;
  for (int c = 0; c < 3; ++c) up[c] += e[c];
  const double bk = c2m * kMagnConst;
  for (int c = 0; c < 3; ++c) b[c] *= bk;
  gamma = fixed ? 1. / sqrt(1. + len2(v)) : lorenz_factor_inv(len2(v));
  up[0] += gamma * (v[1] * b[2] - v[2] * b[1]);
  up[1] += gamma * (v[2] * b[0] - v[0] * b[2]);
  up[2] += gamma * (v[0] * b[1] - v[1] * b[0]);
  alpha = 1. + len2(up);
  B2 = len2(b);
  s = alpha - B2;
  us2 = pow(dot3(up, b), 2);
  alpha = 1. / sqrt(0.5 * (s + sqrt(s * s + 4. * (B2 + us2))));
  for (int c = 0; c < 3; ++c) b[c] *= alpha;
  s = 1. / (1. + len2(b));
  alpha = dot3(up, b);
  psm[0] = s * (up[0] + alpha * b[0] + b[2] * up[1] - b[1] * up[2]);
  psm[1] = s * (up[1] + alpha * b[1] + b[0] * up[2] - b[2] * up[0]);
  psm[2] = s * (up[2] + alpha * b[2] + b[1] * up[0] - b[0] * up[1]);
  if (fixed) {
    gamma = 1. / sqrt(1. + len2(psm));
    for (int c = 0; c < 3; ++c) psm[c] *= gamma * kLightVel;
  } else {
    gamma = lorenz_factor_inv(len2(psm));
    for (int c = 0; c < 3; ++c) psm[c] *= gamma;
  }
  v[0] = psm[0]; v[1] = psm[1]; v[2] = psm[2];
  return true;
}

// PusherHC::operator() (pusherHC.cpp:23-117).  The reference omits the
// normalisation by c (:75), uses b2[0] twice in inv_det_B (:94) and b[2]
// for b[1] in the last term of up[0] (:97); `fixed` corrects all three.
__device__ __forceinline__ bool push_hc(bool fixed, double c2m, const double e_in[3],
                                        const double b_in[3], double v[3], DevStatus* st) {
  double e[3] = {e_in[0], e_in[1], e_in[2]}, b[3] = {b_in[0], b_in[1], b_in[2]};
  double psm[3], um[3], upv[3], b2[3], bx[3], gamma, B2;
  if (!lorenz_factor(len2(v), &gamma, st)) return false;
  for (int c = 0; c < 3; ++c) v[c] *= gamma;
  if (fixed)
    for (int c = 0; c < 3; ++c) v[c] /= kLightVel;
  for (int c = 0; c < 3; ++c) e[c] *= c2m;
  if (fixed)
    for (int c = 0; c < 3; ++c) e[c] /= kLightVel;
  for (int c = 0; c < 3; ++c) psm[c] = e[c];
  for (int c = 0; c < 3; ++c) um[c] = v[c] + psm[c];
  const double gfm2 = (1. + len2(um));
  const double bk = c2m * kMagnConst;
  for (int c = 0; c < 3; ++c) b[c] *= bk;
  B2 = len2(b);
  gamma = 1. / sqrt(0.5 * (gfm2 - B2 + sqrt(pow(gfm2 - B2, 2) +
                                            4.0 * (B2 + pow(b[0] * um[0] + b[1] * um[1] + b[2] * um[2], 2)))));
  for (int c = 0; c < 3; ++c) b[c] *= gamma;
  for (int c = 0; c < 3; ++c) b2[c] = b[c] * b[c];
  bx[0] = b[0] * b[1];
  bx[1] = b[1] * b[2];
  bx[2] = b[2] * b[0];
  const double inv_det_B = fixed ? 1.0 / (1.0 + b2[0] + b2[1] + b2[2])
                                 : 1.0 / (1.0 + b2[0] + b2[1] + b2[0]);
  upv[0] = ((1.0 + b2[0] - b2[1] - b2[2]) * um[0] + 2. * (bx[0] + b[2]) * um[1] +
            2. * (bx[2] - (fixed ? b[1] : b[2])) * um[2]) * inv_det_B;
  upv[1] = (2. * (bx[0] - b[2]) * um[0] + (1. - b2[0] + b2[1] - b2[2]) * um[1] +
            2. * (bx[1] + b[0]) * um[2]) * inv_det_B;
  upv[2] = (2. * (bx[2] + b[1]) * um[0] + 2. * (bx[1] - b[0]) * um[1] +
            (1. - b2[0] - b2[1] + b2[2]) * um[2]) * inv_det_B;
  for (int c = 0; c < 3; ++c) psm[c] += upv[c];
  if (fixed) {
    gamma = 1. / sqrt(1. + len2(psm));
    for (int c = 0; c < 3; ++c) psm[c] *= gamma * kLightVel;
  } else {
    gamma = lorenz_factor_inv(len2(psm));
    for (int c = 0; c < 3; ++c) psm[c] *= gamma;
  }
  v[0] = psm[0]; v[1] = psm[1]; v[2] = psm[2];
  return true;
}

// e += external_fields->get_field_e(pos_r, pos_z), b += ...get_field_h
// (pusherBoris.cpp:62-65): the external planes gathered as the fields are.
__device__ __forceinline__ void add_external(const GridGeom& g, const Fields& f, bool fixed, double r, double z,
                                          double e[3], double b[3]) {
  const size_t pl = (size_t)(g.nr + 4) * g.ld;
  Fields x = f;
  for (int c = 0; c < 3; ++c) {
    x.E[c] = const_cast<double*>(f.ext) + c * pl;
    x.H[c] = const_cast<double*>(f.ext) + (3 + c) * pl;
  }
  double ex[3], bx[3];
  gather_e(g, x, fixed, r, z, ex);
  gather_h(g, x, fixed, r, z, bx);
  for (int c = 0; c < 3; ++c) {
    e[c] += ex[c];
    b[c] += bx[c];
  }
}

// Gather at (r, z) and push one particle; pusher numbering as pcg.h.  EXT:
// add the external fields (f.ext); the kernels are instantiated with and
// without, so that runs without keep the push's registers.
template <bool EXT = false>
__device__ __forceinline__ bool gather_push(const GridGeom& g, const Fields& f, int pusher,
                                            bool fixed, double c2m, double r, double z,
                                            double v[3], DevStatus* st) {
  if (isnan(r) || isinf(r) || isnan(z) || isinf(z)) {  // pusherBoris.cpp:51-57
    raise_error(st, kErrNanPosition);
    return false;
  }
  // The gather reads nodes floor(r/dr - 1/2) .. floor(r/dr) + 1; outside the
  // halo that would be out of bounds, so such a particle stops the step.
  if (!(r >= -1.5 * g.dr && r < (g.nr + 1) * g.dr && z >= -1.5 * g.dz && z < (g.nz + 1) * g.dz)) {
    raise_error(st, kErrOutOfGrid);
    return false;
  }
  double e[3], b[3];
  gather_e(g, f, fixed, r, z, e);
  gather_h(g, f, fixed, r, z, b);
  if (EXT) add_external(g, f, fixed, r, z, e, b);
  if (pusher == 3) return push_vay(fixed, c2m, e, b, v, st);
  if (pusher == 4) return push_hc(fixed, c2m, e, b, v, st);
  return push_boris(pusher, c2m, e, b, v, st);
}

// ---------------------------------------------------------------------------
// Kinematics (specieP.cpp:482-663, beamP.cpp:159-177)

// std::isnormal for doubles: finite, non-zero and not subnormal.  Written out
// because the device build does not provide a usable isnormal.
__device__ __forceinline__ bool is_normal(double x) {
  const double a = fabs(x);
  return a >= 2.2250738585072014e-308 && a <= 1.7976931348623157e308;
}

// SpecieP::reflect for one particle of a domain at the origin
// (specieP.cpp:493-607).  Only positions and velocities leave the loop.
__device__ __forceinline__ bool reflect_one(const GridGeom& g, bool fixed, double* r, double* z,
                                            double r_old, double z_old, double* vr, double* vz) {
  const double dr = g.dr, dz = g.dz;
  const double half_dr = dr / 2., half_dz = dz / 2.;
  const double radius_wall = g.R - dr / 2.;
  const double longitude_wall = g.L - dz / 2.;
  const double radius_wallX2 = radius_wall * 2.;
  const double longitude_wallX2 = longitude_wall * 2.;
  double pos_r = *r - 0.0, pos_z = *z - 0.0;
  double pos_old_r = r_old - 0.0, pos_old_z = z_old - 0.0;
  double pdr = pos_r - pos_old_r, pdz = pos_z - pos_old_z;
  int guard = 0;
  while (is_normal(pos_r) && is_normal(pos_z) &&
         (pos_r > radius_wall || pos_z > longitude_wall || pos_r < half_dr || pos_z < half_dz)) {
    if (++guard > 64) return false;
    if (pos_r > radius_wall) {
      *vr = -*vr;
      double dr_small = radius_wall - pos_old_r;
      double dz_small = dr_small * pdz / pdr;
      pos_r = radius_wallX2 - pos_r;
      pdr = pdr - dr_small;
      pdz = pdz - dz_small;
      pos_old_r = radius_wall;
      pos_old_z = pos_old_z - dz_small;
    }
    if (pos_z > longitude_wall) {
      *vz = -*vz;
      double dz_small = longitude_wall - pos_old_z;
      double dr_small = dz_small * pdr / pdz;
      pos_z = longitude_wallX2 - pos_z;
      pdr = pdr - dr_small;
      pdz = pdz - dz_small;
      pos_old_z = longitude_wall;
      pos_old_r = pos_old_r - dr_small;
    }
    if (pos_r < half_dr) {
      *vr = -*vr;
      double dr_small = half_dr - pos_old_r;
      double dz_small = dr_small * pdz / pdr;
      pos_r = dr - pos_r;
      pdr = pdr - dr_small;
      pdz = pdz - dz_small;
      pos_old_r = half_dr;
      pos_old_z = pos_old_z - dz_small;
      if (pos_r < half_dr) pos_r = half_dr;
    }
    if (pos_z < half_dz) {
      *vz = -*vz;
      double dz_small = half_dz - pos_old_z;
      double dr_small = dz_small * pdr / pdz;
      pos_z = dz - pos_z;
      pdr = pdr - dr_small;
      pdz = pdz - dz_small;
      pos_old_z = fixed ? half_dz : dz;
      pos_old_r = pos_old_r - dr_small;
      if (pos_z < half_dz) pos_z = half_dz;
    }
  }
  *r = pos_r + 0.0;
  *z = pos_z + 0.0;
  return true;
}

// BeamP::reflect (beamP.cpp:159-177): the axis only.
__device__ __forceinline__ void reflect_beam(const GridGeom& g, double* r, double* vr) {
  const double half_dr = g.dr / 2.;
  double pos_r = *r - 0.0;
  if (pos_r < half_dr) {
    *r = g.dr - pos_r + 0.0;
    *vr = -*vr;
  }
}

// ---------------------------------------------------------------------------
// Villasenor-Buneman current (currentVB.cpp:22-735)

// Where a particle's current goes.  J_r adds are dropped for particles that
// come before the last strict-axial particle at that node (reset > order+1),
// which reproduces the J_r overwrite of currentVB.cpp:545-546.
struct Sink {
  double* J[3];
  const unsigned long long* reset;  // may be null
  unsigned long long ord1;          // particle order + 1
  const GridGeom* g;
  bool jphi_interior_only;          // fused path: the halo of J_phi is zeroed (currentVB.cpp:177)

  __device__ __forceinline__ void add_r(int i, int k, double v) const {
    long long n = gidx(*g, i, k);
    if (reset && ord1 < reset[n]) return;
    atomicAdd(J[0] + n, v);
  }
  __device__ __forceinline__ void add_phi(int i, int k, double v) const {
    if (jphi_interior_only && (i < 0 || k < 0 || i >= g->nr || k >= g->nz)) return;
    atomicAdd(J[1] + gidx(*g, i, k), v);
  }
  __device__ __forceinline__ void add_z(int i, int k, double v) const {
    atomicAdd(J[2] + gidx(*g, i, k), v);
  }
};

__device__ __forceinline__ double ssd_r(double q, double r, double dr, double dz, double dt) {
  return q / (2. * kPi * r * dr * dz * dt * 2. * dr);
}
__device__ __forceinline__ double ssd_z(double q, double r, double dr, double dz, double dt) {
  return q / (2. * kPi * r * dr * dz * dt * dz);
}
__device__ __forceinline__ double ssd_strict(double q, double r, double dr, double dz, double dt) {
  return q / (kPi * 4. * r * dz * dz * dr * dt);
}

// log1p(e) / e, 1 at e = 0.
__device__ __forceinline__ double log1p_ratio(double e) { return e == 0.0 ? 1.0 : log1p(e) / e; }

// The fixed mode's form of simple_current_distribution: the same integrals
// with k dz = dr and k log((r_o + dr) / r_o) = -(dz / r_o) log1p(e) / e
// substituted (e = dr / r_o), so that no term divides by dr or dz.  The
// reference's form loses a nearly axial or nearly radial segment's digits
// in 1/k and k, and drops every segment with |dr| or |dz| below 1e-15 m
// (:45-46) -- its whole J_z with it when a nearly axial particle crosses a
// cell face.  On the axis row (i_n = 0) the factor 4 r0^2 - dr^2 is
// exactly 0 and its 1/r_o terms are left out.
__device__ inline void vb_simple_fixed(const Sink& s, double rn, double zn, double ro, double zo, int i_n,
                                       int k_n, double q) {
  const GridGeom& g = *s.g;
  const double dr = g.dr, dz = g.dz, dt = g.dt;
  const double delta_r = rn - ro, delta_z = zn - zo;
  if (delta_r == 0.0 && delta_z == 0.0) return;
  const double lr = i_n >= 1 ? log1p_ratio(delta_r / ro) : 0.0;
  double sd, wj;
  if (i_n >= 1) {
    const double t = dr * dr * ((i_n + 0.5) * (i_n + 0.5) - 0.25) * (delta_z / ro) * lr;
    sd = ssd_r(q, i_n * dr, dr, dz, dt);
    wj = sd * (dr * delta_z - delta_r * delta_z / 2. - delta_z * ro + t);
    s.add_z(i_n, k_n, wj);
    sd = ssd_r(q, (i_n + 1) * dr, dr, dz, dt);
    wj = sd * (delta_r * delta_z / 2. + delta_z * ro + delta_z * dr - t);
    s.add_z(i_n + 1, k_n, wj);
  } else {
    sd = q / (2. * kPi * dr / 4. * dr * dz * dt * dr);
    wj = sd * (dr * delta_z - delta_r * delta_z / 2. - delta_z * ro);
    s.add_z(i_n, k_n, wj);
    sd = ssd_r(q, dr, dr, dz, dt);
    wj = sd * (delta_r * delta_z / 2. + delta_z * dr + delta_z * ro);
    s.add_z(i_n + 1, k_n, wj);
  }
  const double r0 = (i_n + 0.5) * dr, r1 = ro;
  const double p8 = 4 * r0 * r0 - dr * dr;  // 8 (r0^2 / 2 - dr^2 / 8)
  sd = ssd_z(q, r0, dr, dz, dt);
  double b = (k_n + 1.) * dz - zo;
  wj = -r0 * delta_z - delta_z / 2. * (ro + delta_r / 2.) + 0.5 * (delta_r * b + delta_z * (2 * r0 + r1));
  if (p8 != 0.0)
    wj += (delta_r * b + delta_z * r1) * p8 / (8 * ro * (ro + delta_r)) - delta_z / ro * (p8 / 8.) * lr;
  s.add_r(i_n, k_n, sd * wj);
  b = zo - k_n * dz;
  wj = r0 * delta_z + delta_z / 2. * (ro + delta_r / 2.) + 0.5 * (delta_r * b - delta_z * (2 * r0 + r1));
  if (p8 != 0.0)
    wj += (delta_r * b - delta_z * r1) * p8 / (8 * ro * (ro + delta_r)) + delta_z / ro * (p8 / 8.) * lr;
  s.add_r(i_n, k_n + 1, sd * wj);
}

// simple_current_distribution :22-173
__device__ inline void vb_simple(const Sink& s, bool fixed, double rn, double zn, double ro, double zo,
                                 int i_n, int k_n, double q) {
  if (fixed) {
    vb_simple_fixed(s, rn, zn, ro, zo, i_n, k_n, q);
    return;
  }
  const GridGeom& g = *s.g;
  const double dr = g.dr, dz = g.dz, dt = g.dt;
  double wj, k, b, r0, r1, sd;
  const double delta_r = rn - ro, delta_z = zn - zo;
  if ((fabs(delta_r) < kMnzl) || (fabs(delta_z) < kMnzl)) return;
  if (i_n >= 1) {
    k = delta_r / delta_z;
    b = ro;
    sd = ssd_r(q, i_n * dr, dr, dz, dt);
    wj = sd * (dr * delta_z - k * delta_z * delta_z / 2. - delta_z * b +
               dr * dr / k * ((i_n + 0.5) * (i_n + 0.5) - 0.25) * log((k * delta_z + b) / b));
    s.add_z(i_n, k_n, wj);
    sd = ssd_r(q, (i_n + 1) * dr, dr, dz, dt);
    wj = sd * (k * delta_z * delta_z / 2. + delta_z * b + delta_z * dr +
               dr * dr / k * (0.25 - (i_n + 0.5) * (i_n + 0.5)) * log((k * delta_z + b) / b));
    s.add_z(i_n + 1, k_n, wj);
  } else {
    k = delta_r / delta_z;
    b = ro;
    sd = q / (2. * kPi * dr / 4. * dr * dz * dt * dr);
    wj = sd * (dr * delta_z - k * delta_z * delta_z / 2. - delta_z * b);
    s.add_z(i_n, k_n, wj);
    sd = ssd_r(q, dr, dr, dz, dt);
    wj = sd * (k * delta_z * delta_z / 2. + delta_z * dr + delta_z * b);
    s.add_z(i_n + 1, k_n, wj);
  }
  k = -delta_z / delta_r;
  r0 = (i_n + 0.5) * dr;
  r1 = ro;
  b = (k_n + 1.) * dz - zo;
  sd = ssd_z(q, r0, dr, dz, dt);
  wj = sd * (r0 * k * delta_r + k / 2. * delta_r * (ro + delta_r / 2.) +
             0.5 * delta_r * (b - k * (2 * r0 + r1)) +
             delta_r * (b - k * r1) * (4 * r0 * r0 - dr * dr) / (8 * ro * (ro + delta_r)) +
             (k * (r0 * r0 / 2. - dr * dr / 8.)) * log((ro + delta_r) / ro));
  s.add_r(i_n, k_n, wj);
  b = zo - k_n * dz;
  wj = sd * (-r0 * k * delta_r - k / 2. * delta_r * (ro + delta_r / 2.) +
             0.5 * delta_r * (b + k * (2 * r0 + r1)) +
             delta_r * (b + k * r1) * (4 * r0 * r0 - dr * dr) / (8 * ro * (ro + delta_r)) -
             (k * (r0 * r0 / 2. - dr * dr / 8.)) * log((ro + delta_r) / ro));
  s.add_r(i_n, k_n + 1, wj);
}

// strict_motion_distribution :500-729.  The J_r overwrite of the axial
// branch is applied by the caller through Sink::reset.
__device__ inline void vb_strict(const Sink& s, bool fixed, double rn, double zn, double ro, double zo,
                          double q) {
  const GridGeom& g = *s.g;
  const double dr = g.dr, dz = g.dz, dt = g.dt;
  const int i_n = cell_number(rn, dr), k_n = cell_number(zn, dz);
  const int i_o = cell_number(ro, dr), k_o = cell_number(zo, dz);
  if ((fabs(rn - ro) < kMnzl) && (fabs(zn - zo) < kMnzl)) return;
  if (fabs(rn - ro) < kMnzl) {
    double delta_z, lo, up;
    const double value_part = 2. * kPi * rn * dr * dz;
    const double r1 = rn - 0.5 * dr, r2 = (i_n + 0.5) * dr, r3 = rn + 0.5 * dr;
    if (i_n == 0)
      lo = q / (dt * kPi * dr * dr / 4.) * kPi * (r2 * r2 - r1 * r1) / value_part;
    else
      lo = q / (dt * 2. * kPi * i_n * dr * dr) * kPi * (r2 * r2 - r1 * r1) / value_part;
    up = q / (dt * 2 * kPi * (i_n + 1) * dr * dr) * kPi * (r3 * r3 - r2 * r2) / value_part;
    switch (k_n - k_o) {
      case 0:
        delta_z = zn - zo;
        s.add_z(i_n, k_n, lo * delta_z);
        s.add_z(i_n + 1, k_n, up * delta_z);
        break;
      case 1:
        delta_z = k_n * dz - zo;
        s.add_z(i_n, k_n - 1, lo * delta_z);
        s.add_z(i_n + 1, k_n - 1, up * delta_z);
        delta_z = zn - k_n * dz;
        s.add_z(i_n, k_n, lo * delta_z);
        s.add_z(i_n + 1, k_n, up * delta_z);
        break;
      case -1:
        delta_z = (k_n + 1) * dz - zo;
        s.add_z(i_n, k_n + 1, lo * delta_z);
        s.add_z(i_n + 1, k_n + 1, up * delta_z);
        delta_z = zn - (k_n + 1) * dz;
        s.add_z(i_n, k_n, lo * delta_z);
        s.add_z(i_n + 1, k_n, up * delta_z);
        break;
      default: break;
    }
  } else if (fabs(zn - zo) < kMnzl) {
    double wj, delta_r, ldz, rdz, r0, sd;
    switch (i_n - i_o) {
      case 0:
        delta_r = rn - ro;
        ldz = (k_n + 1) * dz - zn;
        rdz = zn - k_n * dz;
        r0 = (i_n + 0.5) * dr;
        sd = ssd_strict(q, r0, dr, dz, dt);
        wj = sd * (delta_r - r0 * r0 / (ro + delta_r) + r0 * r0 / ro +
                   dr * dr / (4. * (ro + delta_r)) - dr * dr / (4. * ro));
        s.add_r(i_n, k_n, wj * ldz);
        s.add_r(i_n, k_n + 1, wj * rdz);
        break;
      case 1:
        delta_r = (i_n) * dr - ro;
        ldz = (k_n + 1) * dz - zn;
        rdz = zn - k_n * dz;
        r0 = (i_n - 0.5) * dr;
        sd = ssd_strict(q, r0, dr, dz, dt);
        wj = sd * (delta_r - r0 * r0 / (ro + delta_r) + r0 * r0 / ro +
                   dr * dr / (4. * (ro + delta_r)) - dr * dr / (4. * ro));
        s.add_r(i_n - 1, k_n, wj * ldz);
        s.add_r(i_n - 1, k_n + 1, wj * rdz);
        delta_r = rn - i_n * dr;
        r0 = (i_n + 0.5) * dr;
        sd = ssd_strict(q, r0, dr, dz, dt);
        if (fixed)
          wj = sd * (delta_r - r0 * r0 / (i_n * dr + delta_r) + r0 * r0 / (i_n * dr) +
                     dr * dr / (4. * (i_n * dr + delta_r)) - dr * dr / (4. * i_n * dr));
        else  // precedence of r0*r0/i_n*dr as written at :673
          wj = sd * (delta_r - r0 * r0 / (i_n * dr + delta_r) + r0 * r0 / i_n * dr +
                     dr * dr / (4. * (i_n * dr + delta_r)) - dr * dr / (4. * i_n * dr));
        s.add_r(i_n, k_n, wj * ldz);
        s.add_r(i_n, k_n + 1, wj * rdz);
        break;
      case -1:
        delta_r = (i_n + 1) * dr - ro;
        ldz = (k_n + 1) * dz - zn;
        rdz = zn - k_n * dz;
        r0 = (i_n + 1.5) * dr;
        sd = ssd_strict(q, r0, dr, dz, dt);
        wj = sd * (delta_r - r0 * r0 / (ro + delta_r) + r0 * r0 / ro +
                   dr * dr / (4. * (ro + delta_r)) - dr * dr / (4. * ro));
        s.add_r(i_n + 1, k_n, wj * ldz);
        s.add_r(i_n + 1, k_n + 1, wj * rdz);
        delta_r = rn - (i_n + 1) * dr;
        r0 = (i_n + 0.5) * dr;
        sd = ssd_strict(q, r0, dr, dz, dt);
        if (fixed)
          wj = sd * (delta_r - r0 * r0 / ((i_n + 1) * dr + delta_r) + r0 * r0 / ((i_n + 1) * dr) +
                     dr * dr / (4. * ((i_n + 1) * dr + delta_r)) - dr * dr / (4. * (i_n + 1) * dr));
        else  // :714
          wj = sd * (delta_r - r0 * r0 / ((i_n + 1) * dr + delta_r) + r0 * r0 / (i_n + 1) * dr +
                     dr * dr / (4. * ((i_n + 1) * dr + delta_r)) - dr * dr / (4. * (i_n + 1) * dr));
        s.add_r(i_n, k_n, wj * ldz);
        s.add_r(i_n, k_n + 1, wj * rdz);
        break;
      default: break;
    }
  }
}

// azimuthal_current_distribution :398-498 for one particle.
__device__ __forceinline__ void vb_azimuthal(const Sink& s, double q, double r, double z,
                                             double ro, double zo, double vphi, int r_i, int z_k) {
  const GridGeom& g = *s.g;
  const double dr = g.dr, dz = g.dz;
  const double v_1 = cell_volume(2.0 * r_i + 1, dr, dz);
  const double v_2 = cell_volume(2.0 * r_i + 1 + 1, dr, dz);
  const double pos_r = (r + ro) / 2;
  const double pos_z = (z + zo) / 2;
  const double r1 = pos_r - 0.5 * dr, r2 = (r_i + 0.5) * dr, r3 = pos_r + 0.5 * dr;
  const double ro_v = q / (2. * kPi * dz * dr * pos_r);
  const double dz1 = (z_k + 0.5) * dz - (pos_z - 0.5 * dz);
  const double dz2 = (pos_z + 0.5 * dz) - (z_k + 0.5) * dz;
  double rho;
  rho = ro_v * kPi * dz1 * (r2 * r2 - r1 * r1) / v_1; s.add_phi(r_i, z_k, rho * vphi);
  rho = ro_v * kPi * dz1 * (r3 * r3 - r2 * r2) / v_2; s.add_phi(r_i + 1, z_k, rho * vphi);
  rho = ro_v * kPi * dz2 * (r2 * r2 - r1 * r1) / v_1; s.add_phi(r_i, z_k + 1, rho * vphi);
  rho = ro_v * kPi * dz2 * (r3 * r3 - r2 * r2) / v_2; s.add_phi(r_i + 1, z_k + 1, rho * vphi);
}

// The strict-axial test of rz_current_distribution (:182-213) and
// strict_motion_distribution (:511-546): true when this particle overwrites
// J_r at (i_n, k_n) and (i_n, k_n+1).
__device__ __forceinline__ bool vb_strict_axial_nodes(const GridGeom& g, bool fixed, double R,
                                                      double Z, double RO, double ZO, int cell_r,
                                                      int* i_out, int* k_out) {
  if (fixed) return false;
  const double dr = g.dr, dz = g.dz;
  int i_n = cell_r;
  int i_o = cell_number(RO, dr);
  if (RO == (i_o + 1) * dr) i_o = i_n;
  if (R == (i_n + 1) * dr) i_n = i_o;
  if (abs(i_n - i_o) > 1) return false;  // logged and skipped (:199-204)
  const bool r_strict = fabs(R - RO) < kMnzl, z_strict = fabs(Z - ZO) < kMnzl;
  if (!(r_strict && !z_strict)) return false;
  *i_out = cell_number(R, dr);
  *k_out = cell_number(Z, dz);
  return true;
}

// rz_current_distribution :175-396 for one particle.  Returns false when
// the particle moved more than one cell (logged as ERROR, no current).
__device__ inline bool vb_rz(const Sink& s, bool fixed, double q, double R, double Z, double RO,
                      double ZO, int cell_r, int cell_z) {
  const GridGeom& g = *s.g;
  const double dr = g.dr, dz = g.dz;
  int i_n = cell_r, k_n = cell_z;
  int i_o = cell_number(RO, dr), k_o = cell_number(ZO, dz);
  if (RO == (i_o + 1) * dr) i_o = i_n;
  if (ZO == (k_o + 1) * dz) k_o = k_n;
  if (R == (i_n + 1) * dr) i_n = i_o;
  if (Z == (k_n + 1) * dz) k_n = k_o;
  const int res_cell = abs(i_n - i_o) + abs(k_n - k_o);
  const bool too_far = fixed ? (abs(i_n - i_o) > 1 || abs(k_n - k_o) > 1) : (abs(i_n - i_o) > 1);
  if (too_far) return false;
  if ((fabs(R - RO) < kMnzl) || (fabs(Z - ZO) < kMnzl)) {
    vb_strict(s, fixed, R, Z, RO, ZO, q);
    return true;
  }
  if (res_cell == 0) {
    vb_simple(s, fixed, R, Z, RO, ZO, i_n, k_n, q);
  } else if (res_cell == 1) {
    if ((i_n != i_o) && (k_n == k_o)) {
      if (RO > (i_n + 1) * dr) {
        const double a = (RO - R) / (ZO - Z);
        const double r_b = (i_n + 1) * dr;
        const double delta_r = r_b - R;
        const double z_b = Z + delta_r / a;
        vb_simple(s, fixed, r_b, z_b, RO, ZO, i_n + 1, k_n, q);
        vb_simple(s, fixed, R, Z, r_b, z_b, i_n, k_n, q);
      } else {
        const double a = (R - RO) / (Z - ZO);
        const double r_b = (i_n) * dr;
        const double delta_r = r_b - RO;
        const double z_b = ZO + delta_r / a;
        vb_simple(s, fixed, r_b, z_b, RO, ZO, i_n - 1, k_n, q);
        vb_simple(s, fixed, R, Z, r_b, z_b, i_n, k_n, q);
      }
    } else if ((i_n == i_o) && (k_n != k_o)) {
      if (ZO < k_n * dz) {
        const double z_b = k_n * dz;
        const double delta_z = z_b - ZO;
        const double a = (R - RO) / (Z - ZO);
        const double r_b = RO + a * delta_z;
        vb_simple(s, fixed, r_b, z_b, RO, ZO, i_n, k_n - 1, q);
        vb_simple(s, fixed, R, Z, r_b, z_b, i_n, k_n, q);
      } else {
        const double z_b = (k_n + 1) * dz;
        const double delta_z = z_b - Z;
        const double a = (RO - R) / (ZO - Z);
        const double r_b = R + a * delta_z;
        vb_simple(s, fixed, r_b, z_b, RO, ZO, i_n, k_n + 1, q);
        vb_simple(s, fixed, R, Z, r_b, z_b, i_n, k_n, q);
      }
    }
  } else if (res_cell == 2) {
    if (i_o < i_n) {
      if (k_o < k_n) {
        const double a = (R - RO) / (Z - ZO);
        const double r1 = i_n * dr;
        const double delta_z1 = (r1 - RO) / a;
        const double z1 = ZO + delta_z1;
        const double z2 = k_n * dz;
        const double delta_r2 = (z2 - ZO) * a;
        const double r2 = RO + delta_r2;
        if (z1 < k_n * dz) {
          vb_simple(s, fixed, r1, z1, RO, ZO, i_n - 1, k_n - 1, q);
          vb_simple(s, fixed, r2, z2, r1, z1, i_n, k_n - 1, q);
          vb_simple(s, fixed, R, Z, r2, z2, i_n, k_n, q);
        } else if (z1 > k_n * dz) {
          vb_simple(s, fixed, r2, z2, RO, ZO, i_n - 1, k_n - 1, q);
          vb_simple(s, fixed, r1, z1, r2, z2, i_n - 1, k_n, q);
          vb_simple(s, fixed, R, Z, r1, z1, i_n, k_n, q);
        }
      } else {
        const double a = (R - RO) / (Z - ZO);
        const double r1 = i_n * dr;
        const double delta_z1 = (r1 - RO) / a;
        const double z1 = ZO + delta_z1;
        const double z2 = (k_n + 1) * dz;
        const double delta_r2 = -(ZO - z2) * a;
        const double r2 = RO + delta_r2;
        if (z1 > (k_n + 1) * dz) {
          vb_simple(s, fixed, r1, z1, RO, ZO, i_n - 1, k_n + 1, q);
          vb_simple(s, fixed, r2, z2, r1, z1, i_n, k_n + 1, q);
          vb_simple(s, fixed, R, Z, r2, z2, i_n, k_n, q);
        } else if (z1 < (k_n + 1) * dz) {
          vb_simple(s, fixed, r2, z2, RO, ZO, i_n - 1, k_n + 1, q);
          vb_simple(s, fixed, r1, z1, r2, z2, i_n - 1, k_n, q);
          vb_simple(s, fixed, R, Z, r1, z1, i_n, k_n, q);
        }
      }
    } else if (i_o > i_n) {
      if (k_o < k_n) {
        const double a = (R - RO) / (Z - ZO);
        const double r1 = (i_n + 1) * dr;
        const double delta_z1 = -(RO - r1) / a;
        const double z1 = ZO + delta_z1;
        const double z2 = k_n * dz;
        const double delta_r2 = -(z2 - ZO) * a;
        const double r2 = RO - delta_r2;
        if (z1 < (k_n) * dz) {
          vb_simple(s, fixed, r1, z1, RO, ZO, i_n + 1, k_n - 1, q);
          vb_simple(s, fixed, r2, z2, r1, z1, i_n, k_n - 1, q);
          vb_simple(s, fixed, R, Z, r2, z2, i_n, k_n, q);
        } else if (z1 > (k_n) * dz) {
          vb_simple(s, fixed, r2, z2, RO, ZO, i_n + 1, k_n - 1, q);
          vb_simple(s, fixed, r1, z1, r2, z2, i_n + 1, k_n, q);
          vb_simple(s, fixed, R, Z, r1, z1, i_n, k_n, q);
        }
      } else if (k_o > k_n) {
        const double a = (RO - R) / (ZO - Z);
        const double r1 = (i_n + 1) * dr;
        const double delta_z1 = (r1 - R) / a;
        const double z1 = Z + delta_z1;
        const double z2 = (k_n + 1) * dz;
        const double delta_r2 = (z2 - Z) * a;
        const double r2 = R + delta_r2;
        if (z1 > (k_n + 1) * dz) {
          vb_simple(s, fixed, r1, z1, RO, ZO, i_n + 1, k_n + 1, q);
          vb_simple(s, fixed, r2, z2, r1, z1, i_n, k_n + 1, q);
          vb_simple(s, fixed, R, Z, r2, z2, i_n, k_n, q);
        } else if (z1 < (k_n + 1) * dz) {
          vb_simple(s, fixed, r2, z2, RO, ZO, i_n + 1, k_n + 1, q);
          vb_simple(s, fixed, r1, z1, r2, z2, i_n + 1, k_n, q);
          vb_simple(s, fixed, R, Z, r1, z1, i_n, k_n, q);
        }
      }
    }
  }
  return true;
}

// ---------------------------------------------------------------------------
// ZigZag current (currentZigZag.cpp:22-136, RELAY_POINT currentZigZag.hpp:28-30)

__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double relay_point(int i1, int i2, double x1, double x2, double dx) {
  return dmin(dmin(i1 * dx, i2 * dx) + dx, dmax(dmax(i1 * dx, i2 * dx), (x1 + x2) / 2.));
}

__device__ __forceinline__ void zigzag(const Sink& s, double charge, double w, double vphi,
                                       double rn, double zn, double ro, double zo) {
  const GridGeom& g = *s.g;
  const double dr = g.dr, dz = g.dz, dt = g.dt;
  const double cod = charge * w / dt;
  const int i_n = cell_number(rn, dr), i_o = cell_number(ro, dr);
  const int k_n = cell_number(zn, dz), k_o = cell_number(zo, dz);
  const int i_mid = cell_number((rn + ro) / 2., dr);
  const double oov = 1 / (cell_volume(2.0 * i_mid + 1, dr, dz));
  const double F_phi = charge * w * vphi;
  const double W_phi = vphi * dt / (2. * kPi * (ro + rn));
  const double rr = relay_point(i_o, i_n, ro, rn, dr), zr = relay_point(k_o, k_n, zo, zn, dz);
  const double F_r1 = cod * (rr - ro), F_r2 = cod * (rn - rr);
  const double F_z1 = cod * (zr - zo), F_z2 = cod * (zn - zr);
  const double W_r1 = (ro + rr) / 2 - i_o * dr, W_r2 = (rn + rr) / 2 - i_n * dr;
  const double W_z1 = (zo + zr) / 2 - k_o * dz, W_z2 = (zn + zr) / 2 - k_n * dz;
  const double mWr1 = 1 - W_r1, mWr2 = 1 - W_r2, mWz1 = 1 - W_z1, mWz2 = 1 - W_z2, mWp = 1 - W_phi;
  s.add_r(i_o, k_o, oov * F_r1 * mWp * mWz1 + oov * F_r1 * W_phi * mWz1);
  s.add_r(i_o, k_o + 1, oov * F_r1 * mWp * W_z1 + oov * F_r1 * W_phi * W_z1);
  s.add_r(i_n, k_n, oov * F_r2 * mWp * mWz2 + oov * F_r2 * W_phi * mWz2);
  s.add_r(i_n, k_n + 1, oov * F_r2 * mWp * W_z2 + oov * F_r2 * W_phi * W_z2);
  s.add_phi(i_n, k_n, oov * F_phi * mWr2 * mWz2);
  s.add_phi(i_n, k_n + 1, oov * F_phi * mWr2 * W_z1);
  s.add_phi(i_n + 1, k_n, oov * F_phi * W_r2 * mWz2);
  s.add_phi(i_n + 1, k_n + 1, oov * F_phi * W_r2 * W_z2);
  s.add_z(i_o, k_o, oov * F_z1 * mWr1 * mWp + oov * F_z1 * mWr1 * W_phi);
  s.add_z(i_o + 1, k_o, oov * F_z1 * W_r1 * mWp + oov * F_z1 * W_r1 * W_phi);
  s.add_z(i_n, k_n, oov * F_z2 * mWr2 * mWp + oov * F_z2 * mWr2 * W_phi);
  s.add_z(i_n + 1, k_n, oov * F_z2 * W_r2 * mWp + oov * F_z2 * W_r2 * W_phi);
}

}  // namespace f64
}  // namespace pcg
