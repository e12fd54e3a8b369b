// pcg_collide_pair.cuh — the pair collisions of the binary collision pass
// (Perez 2012, Takizuka-Abe, SK98) on staged FP64 cell lists, shared by the
// pass's two pair kernels: collide_cells_kernel (pcg_collide.cu, a cell per
// thread) and collide_kernel (pcg_collide_crowded.cu, a warp per crowded
// cell), in separate translation units so that each has its own inlining of
// these functions (not inlined, p12_single made the per-thread kernel's
// pass 24 % slower).
#pragma once

#include <cuda_runtime.h>

#include "pcg_collide.h"
#include "pcg_philox.cuh"

// How the pair functions are declared: the per-cell kernel's unit inlines
// them (it defines PCG_PAIR_FN as __device__ __forceinline__ before this
// header; left to the compiler, small changes to that kernel flipped its
// inlining decision and the pass's speed with it), the crowded unit, with
// many call sites, leaves the choice to the compiler.
#ifndef PCG_PAIR_FN
#define PCG_PAIR_FN __device__
#endif

namespace pcg {
namespace {

constexpr int kThreads = 256;
constexpr double kPi = 3.1415926535897932;
constexpr double kC = 3.0e8, kC2 = kC * kC;
constexpr double kEps0 = 8.85e-12, kElCharge = 1.6e-19, kMnzl = 1e-15;
constexpr double kRelLimit2 = 5e7 * 5e7;
constexpr double kPlankBar = 6.6261e-34 / (2. * kPi);
constexpr uint32_t kCollTag = 0x636f6c6cu, kShufTag = 0x73687566u;

inline unsigned blocks_for(size_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

struct SpeciesTable {
  CollSpecies s[kCollMaxSpecies];
  int n;
};

constexpr unsigned long long kStaged = 1ull << 63;
constexpr unsigned long long kRefMask = (1ull << 40) - 1;

// The staged lists alone: what the moments, pair and correction kernels
// read and write (their references are all staged), so that they index no
// species table at run time.
struct Staged {
  double4* stage[2];
};

// std::isnormal: neither zero, subnormal, infinite nor NaN
__device__ __forceinline__ bool normal(double x) {
  const double a = fabs(x);
  return a >= 2.2250738585072014e-308 && a <= 1.7976931348623157e308;
}

__device__ __forceinline__ double u53(uint32_t a, uint32_t b) {
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

// A staged entry (reference = kStaged | list << 40 | position; list 1 = ions).
__device__ __forceinline__ void load_v(const Staged& L, unsigned long long ref, double v[3], double* w) {
  const double4 e = L.stage[(ref >> 40) & 1][ref & kRefMask];
  v[0] = e.x; v[1] = e.y; v[2] = e.z;
  *w = e.w;
}
__device__ __forceinline__ double load_w(const Staged& L, unsigned long long ref) {
  return L.stage[(ref >> 40) & 1][ref & kRefMask].w;
}
__device__ __forceinline__ void store_v(const Staged& L, unsigned long long ref, const double v[3]) {
  double4* e = L.stage[(ref >> 40) & 1] + (ref & kRefMask);
  e->x = v[0]; e->y = v[1]; e->z = v[2];
}
__device__ __forceinline__ int list_of(const Staged&, unsigned long long ref) { return (int)((ref >> 40) & 1); }

// ---------------------------------------------------------------------------
// 5. the pair collision (collisionsP12.cpp:29-328)

__device__ __forceinline__ double len2(const double a[3]) { return a[0] * a[0] + a[1] * a[1] + a[2] * a[2]; }
__device__ __forceinline__ double dot3(const double a[3], const double b[3]) {
  double r = 0;
  for (int c = 0; c < 3; ++c) r += a[c] * b[c];
  return r;
}

// phys::rel::lorenz_factor (rel.cpp:24-45); false when beta > 1
__device__ __forceinline__ bool lorenz(double v2, double* g) {
  const double beta = v2 / kC2;
  if (beta > 1) return false;
  double gm = 1 / sqrt(1.0 - beta);
  if (isinf(gm)) gm = 1e100;
  *g = gm;
  return true;
}

struct PairCtx {
  const Staged* tab;
  const CollParams* p;
  uint32_t cell;
  uint32_t m;      // collision number in the cell
  double* expect;  // the cell's 12 expected moment changes (expectation mode)
};

// Mean of cos(chi) and cos(chi)^2 over the P12 scattering-angle draw for
// s12 (collisionsP12.cpp:215-240): 1 + s ln U for s < 0.1 (E ln U = -1,
// E ln^2 U = 2); the density exp(A cos) / (2 sinh(A) / A) for s < 6
// (E cos = coth A - 1/A, E cos^2 = 1 - 2 E[cos] / A); isotropic beyond.
__device__ __forceinline__ void angle_moments(double s12, double* ec, double* ec2) {
  double A;
  if (s12 < 0.1) {
    *ec = 1 - s12;
    *ec2 = 1 - 2 * s12 + 2 * s12 * s12;
    return;
  } else if (s12 < 3) {
    const double A_inv = 0.00569578 + 0.9560202 * s12 - 0.508139 * (s12 * s12) +
                         0.47913906 * pow(s12, 3) - 0.12788975 * pow(s12, 4) + 0.02389567 * pow(s12, 5);
    A = 1. / A_inv;
  } else if (s12 < 6.) {
    A = 3. * exp(-s12);
  } else {
    *ec = 0;
    *ec2 = 1. / 3.;
    return;
  }
  if (A < 1e-4) {  // near isotropic: coth A - 1/A = A/3 - A^3/45
    *ec = A / 3 - A * A * A / 45;
  } else {
    *ec = 1 / tanh(A) - 1 / A;
  }
  *ec2 = A < 1e-4 ? 1. / 3. + 2 * A * A / 45 : 1 - 2 * *ec / A;
}

// Expected change of sum w v and sum w v^2 of a particle of weight w and
// mass m whose CM momentum sign * p is rotated by the drawn angle (lab
// velocity vcm + p'/m, deflected with probability prob).  The change is
// formed directly, (Ec - 1) p / m and (1 - Ec2)(p^2 - 3 p_k^2) / (2 m^2),
// so that it vanishes exactly without scattering.
__device__ __forceinline__ void expect_add(double* acc, const double vcm[3], const double p[3], double sign,
                                           double m, double w, double prob, double ec, double ec2) {
  const double p2 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
  for (int k = 0; k < 3; ++k) {
    const double d1 = sign * (ec - 1) * p[k] / m;
    const double d2 = 2 * vcm[k] * d1 + (1 - ec2) * (p2 - 3 * p[k] * p[k]) / (2 * m * m);
    acc[k] += prob * w * d1;
    acc[3 + k] += prob * w * d2;
  }
}

PCG_PAIR_FN void p12_single(PairCtx& x, double m_real_a, double m_real_b, double q_real_a,
                           double q_real_b, unsigned long long ra, unsigned long long rb,
                           double density_a_in, double density_b_in, double debye_in) {
  const CollParams& P = *x.p;
  const int fixed = P.fixed;
  double va0[3], vb0[3], wa0, wb0;
  load_v(*x.tab, ra, va0, &wa0);
  load_v(*x.tab, rb, vb0, &wb0);
  const double w_ratio = wa0 / wb0;
  const bool swap = !(w_ratio <= 1);
  const double charge_a = swap ? q_real_b : q_real_a, mass_a = swap ? m_real_b : m_real_a;
  const double charge_b = swap ? q_real_a : q_real_b, mass_b = swap ? m_real_a : m_real_b;
  const double density_a = swap ? density_b_in : density_a_in;
  const double density_b = swap ? density_a_in : density_b_in;
  const double* v_a = swap ? vb0 : va0;
  const double* v_b = swap ? va0 : vb0;
  const double w_a = swap ? wb0 : wa0, w_b = swap ? wa0 : wb0;

  if (v_a[0] == v_b[0] && v_a[1] == v_b[1] && v_a[2] == v_b[2]) return;

  double gamma_a, gamma_b;
  if (!lorenz(len2(v_a), &gamma_a) || !lorenz(len2(v_b), &gamma_b)) { raise_error(x.p->status, kErrSuperluminal); return; }
  const double p0_a = gamma_a * mass_a * kC, p0_b = gamma_b * mass_b * kC;
  double p_a[3], p_b[3], beta_cm[3], t[3];
  for (int c = 0; c < 3; ++c) { p_a[c] = v_a[c] * gamma_a; p_a[c] *= mass_a; }
  for (int c = 0; c < 3; ++c) { p_b[c] = v_b[c] * gamma_b; p_b[c] *= mass_b; }
  for (int c = 0; c < 3; ++c) beta_cm[c] = p_a[c] + p_b[c];
  const double p0_sum = p0_a + p0_b;
  for (int c = 0; c < 3; ++c) beta_cm[c] /= p0_sum;

  double gamma_cm;
  if (!lorenz(len2(beta_cm) * kC2, &gamma_cm)) { raise_error(x.p->status, kErrSuperluminal); return; }
  const double p0_a_cm = gamma_cm * (p0_a - dot3(beta_cm, p_a));
  const double p0_b_cm = gamma_cm * (p0_b - dot3(beta_cm, p_b));

  double p_a_cm[3];
  for (int c = 0; c < 3; ++c) p_a_cm[c] = p_a[c];
  {
    const double d = dot3(beta_cm, p_a), l2 = len2(beta_cm);
    for (int c = 0; c < 3; ++c) { t[c] = beta_cm[c] * d; t[c] *= (gamma_cm - 1); t[c] /= l2; }
    for (int c = 0; c < 3; ++c) p_a_cm[c] += t[c];
    for (int c = 0; c < 3; ++c) { t[c] = beta_cm[c] * gamma_cm; t[c] *= p0_a; }
    for (int c = 0; c < 3; ++c) p_a_cm[c] -= t[c];
  }
  double p_b_cm[3], v_cm[3];
  for (int c = 0; c < 3; ++c) p_b_cm[c] = -p_a_cm[c];
  for (int c = 0; c < 3; ++c) v_cm[c] = beta_cm[c] * kC;
  const double gamma_a_cm = (1 - dot3(v_a, v_cm) / kC2) * gamma_a * gamma_cm;
  const double gamma_b_cm = (1 - dot3(v_b, v_cm) / kC2) * gamma_b * gamma_cm;
  double v_a_cm[3], v_b_cm[3];
  const double da = mass_a * gamma_a_cm, db = mass_b * gamma_b_cm;
  for (int c = 0; c < 3; ++c) { v_a_cm[c] = p_a_cm[c] / da; v_b_cm[c] = p_b_cm[c] / db; }
  const double la = sqrt(len2(v_a_cm)), lb = sqrt(len2(v_b_cm));
  // the reference subtracts the CM speeds (:139-140); fixed adds them
  const double v_rel_abs = (fixed ? la + lb : la - lb) / (1 - dot3(v_a_cm, v_b_cm) / kC2);

  double gamma_rel;
  if (!lorenz(v_rel_abs * v_rel_abs, &gamma_rel)) { raise_error(x.p->status, kErrSuperluminal); return; }
  const double p_rel_abs = gamma_rel * mass_b * v_rel_abs;
  if (p_rel_abs == 0) return;
  if (v_rel_abs < kMnzl) return;
  if (!normal(density_a)) return;
  if (!normal(density_b)) return;

  const bool rel = len2(v_a) > kRelLimit2 || len2(v_b) > kRelLimit2;
  const double debye = rel ? debye_in * gamma_rel : debye_in;
  const double m_red = mass_a * mass_b / (mass_a + mass_b);
  const double cl = log(debye * m_red * v_rel_abs / kPlankBar);  // plasma.cpp:42-52
  const double L_coulomb = 2. < cl ? cl : 2.;
  const double density_w = density_a * density_b / (density_a < density_b ? density_a : density_b);
  const double mass_ab = mass_a * mass_b / (mass_a + mass_b);
  double s12;
  if (rel) {
    const double qq = charge_a * charge_b;
    const double ec = kEps0 * kC2;
    const double f = mass_a * gamma_a_cm * mass_b * gamma_b_cm * kC2 / len2(p_a_cm) + 1;
    s12 = density_w * P.dt * L_coulomb * (qq * qq) /
          (4 * kPi * (ec * ec) * mass_a * gamma_a * mass_b * gamma_b) * gamma_cm * sqrt(len2(p_a)) /
          (mass_a * gamma_a + mass_b * gamma_b) * (f * f);
  } else {
    const double qq = charge_a * charge_b;
    const double em = kEps0 * mass_ab;
    s12 = density_w * P.dt * L_coulomb * (qq * qq) / (4 * kPi * (em * em) * pow(v_rel_abs, 3));
  }
  if (v_rel_abs < 1e6 && density_w > 7e13) {  // low-temperature cap :203-213
    const double na = mass_a * pow(density_a, 2. / 3.), nb = mass_b * pow(density_b, 2. / 3.);
    const double s12max = pow(4. / 3. * kPi, 1. / 3.) * density_w * P.dt * (mass_a + mass_b) /
                          (na > nb ? na : nb) * v_rel_abs;
    if (s12max < s12) s12 = s12max;
  }
  if (x.expect) {  // record this collision's mean change given the velocities it meets
    double ec, ec2;
    angle_moments(s12, &ec, &ec2);
    const double pb_prob = fixed ? w_a / w_b : 1.0;
    const int la = list_of(*x.tab, swap ? rb : ra), lb = list_of(*x.tab, swap ? ra : rb);
    expect_add(x.expect + 6 * la, v_cm, p_a_cm, 1.0, mass_a, w_a, 1.0, ec, ec2);
    expect_add(x.expect + 6 * lb, v_cm, p_a_cm, -1.0, mass_b, w_b, pb_prob, ec, ec2);
  }

  uint32_t o[4], o2[4];
  philox4x32_10(x.cell, 2u * x.m, P.pass, kCollTag, (uint32_t)P.seed, (uint32_t)(P.seed >> 32), o);
  philox4x32_10(x.cell, 2u * x.m + 1u, P.pass, kCollTag, (uint32_t)P.seed, (uint32_t)(P.seed >> 32), o2);
  const double U = u53(o[0], o[1]);
  double cos_xi_cm;
  if (s12 < 0.1) {
    cos_xi_cm = 1 + s12 * log(U);
  } else if (s12 < 3) {
    const double A_inv = 0.00569578 + 0.9560202 * s12 - 0.508139 * (s12 * s12) +
                         0.47913906 * pow(s12, 3) - 0.12788975 * pow(s12, 4) + 0.02389567 * pow(s12, 5);
    const double A = 1. / A_inv;
    cos_xi_cm = A_inv * log(exp(-A) + 2. * U * sinh(A));
  } else if (s12 < 6.) {
    const double A = 3. * exp(-s12);
    const double A_inv = 1. / A;
    cos_xi_cm = A_inv * log(exp(-A) + 2. * U * sinh(A));
  } else {
    cos_xi_cm = 2 * U - 1;
  }
  const double sin_xi_cm = sqrt(1 - cos_xi_cm * cos_xi_cm);
  const double phi_cm = (2 * kPi) * u53(o[2], o[3]);
  double sin_phi_cm, cos_phi_cm;
  sincos(phi_cm, &sin_phi_cm, &cos_phi_cm);

  double p_a_prime_cm[3];
  const double p_a_cm_abs = sqrt(len2(p_a_cm));
  const double p_cm_prp = sqrt(p_a_cm[0] * p_a_cm[0] + p_a_cm[1] * p_a_cm[1]);
  p_a_prime_cm[0] = p_a_cm[0] * p_a_cm[2] / p_cm_prp * sin_xi_cm * cos_phi_cm -
                    p_a_cm[1] * p_a_cm_abs / p_cm_prp * sin_xi_cm * sin_phi_cm + p_a_cm[0] * cos_xi_cm;
  p_a_prime_cm[1] = p_a_cm[1] * p_a_cm[2] / p_cm_prp * sin_xi_cm * cos_phi_cm +
                    p_a_cm[0] * p_a_cm_abs / p_cm_prp * sin_xi_cm * sin_phi_cm + p_a_cm[1] * cos_xi_cm;
  p_a_prime_cm[2] = -p_cm_prp * sin_xi_cm * cos_phi_cm + p_a_cm[2] * cos_xi_cm;

  const double U_defl = u53(o2[0], o2[1]);
  const bool defl_a = fixed ? true : U_defl < w_a;
  const bool defl_b = fixed ? U_defl < w_a / w_b : U_defl < w_b;
  double v_a_prime[3] = {0, 0, 0}, v_b_prime[3] = {0, 0, 0};
  const double l2b = len2(beta_cm);
  if (defl_a) {
    double pp[3];
    for (int c = 0; c < 3; ++c) pp[c] = p_a_prime_cm[c];
    const double d = dot3(beta_cm, p_a_prime_cm);
    for (int c = 0; c < 3; ++c) { t[c] = beta_cm[c] * d; t[c] *= (gamma_cm - 1); t[c] /= l2b; }
    for (int c = 0; c < 3; ++c) pp[c] += t[c];
    for (int c = 0; c < 3; ++c) { t[c] = beta_cm[c] * gamma_cm; t[c] *= p0_a_cm; }
    for (int c = 0; c < 3; ++c) pp[c] += t[c];
    for (int c = 0; c < 3; ++c) v_a_prime[c] = pp[c] / mass_a;
    const double gi = pow(1.0 + len2(v_a_prime) / kC2, -0.5);  // rel.cpp:47-55
    for (int c = 0; c < 3; ++c) v_a_prime[c] *= gi;
  }
  if (defl_b) {
    double pbp[3], pp[3];
    for (int c = 0; c < 3; ++c) pbp[c] = -p_a_prime_cm[c];
    for (int c = 0; c < 3; ++c) pp[c] = pbp[c];
    const double d = dot3(beta_cm, pbp);
    for (int c = 0; c < 3; ++c) { t[c] = beta_cm[c] * d; t[c] *= (gamma_cm - 1); t[c] /= l2b; }
    for (int c = 0; c < 3; ++c) pp[c] += t[c];
    for (int c = 0; c < 3; ++c) { t[c] = beta_cm[c] * gamma_cm; t[c] *= p0_b_cm; }
    for (int c = 0; c < 3; ++c) pp[c] += t[c];
    for (int c = 0; c < 3; ++c) v_b_prime[c] = pp[c] / mass_b;
    const double gi = pow(1.0 + len2(v_b_prime) / kC2, -0.5);
    for (int c = 0; c < 3; ++c) v_b_prime[c] *= gi;
  }
  // write back (:279-310): the reference tests U < w_a for pa and U < w_b
  // for pb whichever is lighter; fixed deflects a always, b as drawn
  const double* to_pa = swap ? v_b_prime : v_a_prime;
  const double* to_pb = swap ? v_a_prime : v_b_prime;
  const bool set_pa = fixed ? (swap ? defl_b : defl_a) : U_defl < wa0;
  const bool set_pb = fixed ? (swap ? defl_a : defl_b) : U_defl < wb0;
  if (set_pa) store_v(*x.tab, ra, to_pa);
  if (set_pb) store_v(*x.tab, rb, to_pb);
}

// ---------------------------------------------------------------------------
// 5'. the Takizuka-Abe pair collision (collisionsTA77S.cpp:33-208): a normal
// delta of variance q_a^2 q_b^2 n L dt / (8 pi eps0^2 m_ab^2 u^3) (Box-Muller
// on draws 0 and 1 of the collision's two Philox blocks), the angle Phi
// (draw 2) and dzeta (draw 3) of the weighted second angle.  The reference
// adds m_ab/m_b du2 to b (:191-193) where the scheme subtracts it; the
// fixed mode subtracts.

PCG_PAIR_FN void ta77s_single(PairCtx& x, double m_real_a, double m_real_b, double q_real_a,
                             double q_real_b, unsigned long long ra, unsigned long long rb,
                             double density_a_in, double density_b_in, double debye) {
  const CollParams& P = *x.p;
  double va[3], vb[3], wa, wb;
  load_v(*x.tab, ra, va, &wa);
  load_v(*x.tab, rb, vb, &wb);
  double w_ratio = wa / wb;
  const bool swap = !(w_ratio <= 1);
  if (swap) w_ratio = 1 / w_ratio;
  const double charge_a = swap ? q_real_b : q_real_a, mass_a = swap ? m_real_b : m_real_a;
  const double charge_b = swap ? q_real_a : q_real_b, mass_b = swap ? m_real_a : m_real_b;
  const double density_a = swap ? density_b_in : density_a_in;
  const double density_b = swap ? density_a_in : density_b_in;
  const double* v_a = swap ? vb : va;
  const double* v_b = swap ? va : vb;
  const double density_lowest = density_a < density_b ? density_a : density_b;
  const double m_ab = mass_a * mass_b / (mass_a + mass_b);
  const double ux = v_a[0] - v_b[0], uy = v_a[1] - v_b[1], uz = v_a[2] - v_b[2];
  const double u = sqrt(ux * ux + uy * uy + uz * uz);
  if (u == 0) return;
  const double cl = log(debye * m_ab * u / kPlankBar);  // plasma.cpp:42-52
  const double lambda = cl > 2. ? cl : 2.;
  const double u_p = sqrt(ux * ux + uy * uy);
  const double variance_d = charge_a * charge_a * (charge_b * charge_b) * density_lowest * lambda /
                            (8 * kPi * (kEps0 * kEps0) * (m_ab * m_ab) * pow(u, 3.0)) * P.dt;
  uint32_t o[4], o2[4];
  philox4x32_10(x.cell, 2u * x.m, P.pass, kCollTag, (uint32_t)P.seed, (uint32_t)(P.seed >> 32), o);
  philox4x32_10(x.cell, 2u * x.m + 1u, P.pass, kCollTag, (uint32_t)P.seed, (uint32_t)(P.seed >> 32), o2);
  const double u0 = u53(o[0], o[1]), u1 = u53(o[2], o[3]);
  const double delta = sqrt(-2.0 * log(1.0 - u0)) * cos(2.0 * kPi * u1) * sqrt(variance_d);
  const double sin_T = 2 * delta / (1 + delta * delta);
  const double cos_T = 1 - 2 * (delta * delta) / (1 + delta * delta);
  double sin_T2 = sqrt(w_ratio * (sin_T * sin_T) + w_ratio * (1 - w_ratio) * ((1 - cos_T) * (1 - cos_T)));
  const double cos_T2 = 1 - w_ratio * (1 - cos_T);
  if (sin_T2 * sin_T < 0) sin_T2 = -sin_T2;
  const double phi = u53(o2[0], o2[1]) * (2 * kPi) + 0.0;
  const double dzeta = u53(o2[2], o2[3]);
  const double phi2 = phi + 2 * kPi * (1 - sqrt(w_ratio)) * (1 - dzeta);
  double sin_P, cos_P, sin_P2, cos_P2;
  sincos(phi, &sin_P, &cos_P);
  sincos(phi2, &sin_P2, &cos_P2);
  double du[3], du2[3];
  if (u_p == 0) {
    du[0] = u * sin_T * cos_P; du[1] = u * sin_T * sin_P; du[2] = -u * (1 - cos_T);
    du2[0] = u * sin_T2 * cos_P2; du2[1] = u * sin_T2 * sin_P2; du2[2] = -u * (1 - cos_T2);
  } else {
    du[0] = (ux / u_p) * uz * sin_T * cos_P - (uy / u_p) * u * sin_T * sin_P - ux * (1 - cos_T);
    du[1] = (uy / u_p) * uz * sin_T * cos_P + (ux / u_p) * u * sin_T * sin_P - uy * (1 - cos_T);
    du[2] = u_p * sin_T * cos_P - uz * (1 - cos_T);
    du2[0] = (ux / u_p) * uz * sin_T2 * cos_P2 - (uy / u_p) * u * sin_T2 * sin_P2 - ux * (1 - cos_T2);
    du2[1] = (uy / u_p) * uz * sin_T2 * cos_P2 + (ux / u_p) * u * sin_T2 * sin_P2 - uy * (1 - cos_T2);
    du2[2] = u_p * sin_T2 * cos_P2 - uz * (1 - cos_T2);
  }
  const double ka = m_ab / mass_a, kb = P.fixed ? -(m_ab / mass_b) : m_ab / mass_b;
  const double na[3] = {v_a[0] + ka * du[0], v_a[1] + ka * du[1], v_a[2] + ka * du[2]};
  const double nb[3] = {v_b[0] + kb * du2[0], v_b[1] + kb * du2[1], v_b[2] + kb * du2[2]};
  store_v(*x.tab, swap ? rb : ra, na);
  store_v(*x.tab, swap ? ra : rb, nb);
}

// ---------------------------------------------------------------------------
// 5''. the relativistic centre-of-mass scheme of CollisionsSK98
// (collisionsSK98.cpp:29-244): a normal delta whose variance is the
// collision frequency (plasma.cpp:54-63) times dt (Box-Muller on draws 0 and
// 1), the CM deflection tan theta_cm = sin theta / (gamma_cm (cos theta -
// v_cm / v_rel)), the azimuth Phi (draw 2); the CM momentum is rotated and
// both particles boosted back, with no weight rejection and no correction
// pass.  The reference subtracts the CM speeds of two particles moving apart
// (:131-132); the fixed mode adds them, as for P12.

PCG_PAIR_FN void sk98_single(PairCtx& x, double m_real_a, double m_real_b, double q_real_a,
                            double q_real_b, unsigned long long ra, unsigned long long rb,
                            double density_a_in, double density_b_in, double debye) {
  const CollParams& P = *x.p;
  double va0[3], vb0[3], wa0, wb0;
  load_v(*x.tab, ra, va0, &wa0);
  load_v(*x.tab, rb, vb0, &wb0);
  const bool swap = !(wa0 / wb0 <= 1);
  const double charge_a = swap ? q_real_b : q_real_a, mass_a = swap ? m_real_b : m_real_a;
  const double charge_b = swap ? q_real_a : q_real_b, mass_b = swap ? m_real_a : m_real_b;
  const double density_a = swap ? density_b_in : density_a_in;
  const double density_b = swap ? density_a_in : density_b_in;
  const double* v_a = swap ? vb0 : va0;
  const double* v_b = swap ? va0 : vb0;
  if (v_a[0] == v_b[0] && v_a[1] == v_b[1] && v_a[2] == v_b[2]) return;

  double gamma_a, gamma_b;
  if (!lorenz(len2(v_a), &gamma_a) || !lorenz(len2(v_b), &gamma_b)) { raise_error(P.status, kErrSuperluminal); return; }
  const double p0_a = gamma_a * mass_a * kC, p0_b = gamma_b * mass_b * kC;
  double p_a[3], p_b[3], beta_cm[3], t[3];
  for (int c = 0; c < 3; ++c) { p_a[c] = v_a[c] * gamma_a; p_a[c] *= mass_a; }
  for (int c = 0; c < 3; ++c) { p_b[c] = v_b[c] * gamma_b; p_b[c] *= mass_b; }
  for (int c = 0; c < 3; ++c) beta_cm[c] = p_a[c] + p_b[c];
  const double p0_sum = p0_a + p0_b;
  for (int c = 0; c < 3; ++c) beta_cm[c] /= p0_sum;
  double gamma_cm;
  const double v_cm_2 = len2(beta_cm) * kC2;
  if (!lorenz(v_cm_2, &gamma_cm)) { raise_error(P.status, kErrSuperluminal); return; }
  const double p0_a_cm = gamma_cm * (p0_a - dot3(beta_cm, p_a));
  const double p0_b_cm = gamma_cm * (p0_b - dot3(beta_cm, p_b));
  const double l2 = len2(beta_cm);

  double p_a_cm[3], p_b_cm[3];
  {
    const double d = dot3(beta_cm, p_a);
    for (int c = 0; c < 3; ++c) p_a_cm[c] = p_a[c];
    for (int c = 0; c < 3; ++c) { t[c] = beta_cm[c] * d; t[c] *= (gamma_cm - 1); t[c] /= l2; }
    for (int c = 0; c < 3; ++c) p_a_cm[c] += t[c];
    for (int c = 0; c < 3; ++c) { t[c] = beta_cm[c] * gamma_cm; t[c] *= p0_a; }
    for (int c = 0; c < 3; ++c) p_a_cm[c] -= t[c];
  }
  for (int c = 0; c < 3; ++c) p_b_cm[c] = -p_a_cm[c];
  const double gamma_a_cm = p0_a_cm / mass_a / kC;
  const double gamma_b_cm = p0_b_cm / mass_b / kC;
  double v_a_cm[3], v_b_cm[3];
  const double da = mass_a * gamma_a_cm, db = mass_b * gamma_b_cm;
  for (int c = 0; c < 3; ++c) { v_a_cm[c] = p_a_cm[c] / da; v_b_cm[c] = p_b_cm[c] / db; }
  const double la = sqrt(len2(v_a_cm)), lb = sqrt(len2(v_b_cm));
  const double v_rel_abs = (P.fixed ? la + lb : la - lb) / (1 - dot3(v_a_cm, v_b_cm) / kC2);
  double gamma_rel;
  if (!lorenz(v_rel_abs * v_rel_abs, &gamma_rel)) { raise_error(P.status, kErrSuperluminal); return; }
  const double p_rel_abs = gamma_rel * mass_b * v_rel_abs;
  const double density_lowest = density_b < density_a ? density_b : density_a;
  if (p_rel_abs == 0) return;
  if (v_rel_abs < kMnzl) return;
  const double m_red = mass_a * mass_b / (mass_a + mass_b);
  const double cl = log(debye * m_red * v_rel_abs / kPlankBar);  // plasma.cpp:42-52
  const double L_coulomb = cl > 2. ? cl : 2.;
  const double qq = charge_a * charge_b;
  const double coll_freq = (qq * qq) * density_lowest * L_coulomb /
                           (8 * kPi * (kEps0 * kEps0) * (p_rel_abs * p_rel_abs) * v_rel_abs);
  const double std_dev_d = sqrt(coll_freq * P.dt);
  uint32_t o[4], o2[4];
  philox4x32_10(x.cell, 2u * x.m, P.pass, kCollTag, (uint32_t)P.seed, (uint32_t)(P.seed >> 32), o);
  philox4x32_10(x.cell, 2u * x.m + 1u, P.pass, kCollTag, (uint32_t)P.seed, (uint32_t)(P.seed >> 32), o2);
  const double u0 = u53(o[0], o[1]), u1 = u53(o[2], o[3]);
  const double delta = sqrt(-2.0 * log(1.0 - u0)) * cos(2.0 * kPi * u1) * std_dev_d;
  const double sin_theta = 2 * delta / (1 + delta * delta);
  const double cos_theta = 1 - 2 * (delta * delta) / (1 + delta * delta);
  const double tg_theta_cm = sin_theta / (gamma_cm * (cos_theta - sqrt(v_cm_2) / v_rel_abs));
  double sin_theta_cm, cos_theta_cm;
  sincos(atan(tg_theta_cm), &sin_theta_cm, &cos_theta_cm);
  const double phi_angle = u53(o2[0], o2[1]) * (2 * kPi) + 0.0;
  double sin_phi, cos_phi;
  sincos(phi_angle, &sin_phi, &cos_phi);

  const double* p_cm = p_a_cm;
  const double p_cm_abs = sqrt(len2(p_cm));
  const double p_cm_prp = sqrt(p_cm[0] * p_cm[0] + p_cm[1] * p_cm[1]);
  double d_p[3];
  d_p[0] = p_cm[0] * p_cm[2] / p_cm_prp * sin_theta_cm * cos_phi -
           p_cm[1] * p_cm_abs / p_cm_prp * sin_theta_cm * sin_phi - p_cm[0] * (1 - cos_theta_cm);
  d_p[1] = p_cm[1] * p_cm[2] / p_cm_prp * sin_theta_cm * cos_phi +
           p_cm[0] * p_cm_abs / p_cm_prp * sin_theta_cm * sin_phi - p_cm[1] * (1 - cos_theta_cm);
  d_p[2] = -p_cm_prp * sin_theta_cm * cos_phi - p_cm[2] * (1 - cos_theta_cm);

  // back to the LAB frame: p' + beta (beta.p')(gamma_cm - 1)/beta^2 + beta gamma_cm p0_cm
  double v_new[2][3];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    double q[3];
    for (int c = 0; c < 3; ++c) q[c] = k == 0 ? p_a_cm[c] + d_p[c] : p_b_cm[c] - d_p[c];
    const double d = dot3(beta_cm, q);
    for (int c = 0; c < 3; ++c) { t[c] = beta_cm[c] * d; t[c] *= (gamma_cm - 1); t[c] /= l2; }
    for (int c = 0; c < 3; ++c) q[c] += t[c];
    const double p0k = k == 0 ? p0_a_cm : p0_b_cm;
    for (int c = 0; c < 3; ++c) { t[c] = beta_cm[c] * gamma_cm; t[c] *= p0k; }
    for (int c = 0; c < 3; ++c) q[c] += t[c];
    const double mk = k == 0 ? mass_a : mass_b;
    for (int c = 0; c < 3; ++c) v_new[k][c] = q[c] / mk;
    const double gi = pow(1.0 + len2(v_new[k]) / kC2, -0.5);  // rel.cpp:47-55
    for (int c = 0; c < 3; ++c) v_new[k][c] *= gi;
  }
  store_v(*x.tab, swap ? rb : ra, v_new[0]);
  store_v(*x.tab, swap ? ra : rb, v_new[1]);
}

}  // namespace
}  // namespace pcg
