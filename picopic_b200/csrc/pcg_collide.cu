// pcg_collide.cu — one pass of binary Coulomb collisions, the Perez et al.
// 2012 scheme of CollisionsP12 (collisionsP12.cpp:29-569 over
// collisions.cpp:87-236), in double precision on the GPU.
//
// Steps, each a kernel:
//  1. keys: every live particle in the grid (in the selected cells) gets a
//     64-bit key (cell, species, insertion id), appended to the electron or
//     ion list (ions: species named "ions"/"Ions"; every other species goes
//     to the electron list, as sort_to_cells does), and counts per cell;
//  2. a radix sort of each list by key gives the reference's cell lists
//     (species order, then particle order) and an exclusive scan the starts;
//  3. optionally a Fisher-Yates shuffle of every cell list (Philox draws
//     (cell, i) of this pass);
//  3b. the lists' velocities and weights are copied, in list order, into
//     contiguous FP64 staging (the particle arrays are in the step's tile
//     order, so a cell's particles lie far apart); steps 4-5 read and write
//     the copy and a last kernel writes the velocities back;
//  4. per cell: weight, energy and density sums in list order (the
//     reference's collect pass), the temperatures and the row stop of the
//     reference's `break` on a non-normal value (:351-354);
//  5. per cell, one thread runs the reference's pairing sequence (ion pairs,
//     electron pairs, the odd-count triples, then electron-ion pairing with
//     the c_i/c_r grouping) and collides each pair in that order, collision m
//     drawing from Philox blocks (cell, 2m) and (cell, 2m+1) of this pass.
//
// Arithmetic follows the reference's operation order (the unit is compiled
// without FMA contraction); log/exp/pow/sin/cos are CUDA's, so results
// agree with the CPU oracle to a few ulp rather than bit for bit.
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>

#include "pcg_collide.h"
#include "pcg_f32.h"
#include "pcg_philox.cuh"

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

// ---------------------------------------------------------------------------
// 1. keys

__global__ void key_kernel(GridGeom g, SpeciesTable tab, int t, unsigned long long* keys,
                           unsigned long long* vals, unsigned* count, unsigned* n_valid,
                           const unsigned char* only, unsigned char only_value) {
  const size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const CollSpecies& sp = tab.s[t];
  int ci = -1, ck = -1;
  unsigned id = 0;
  if (j < sp.n) {
    if (sp.cell) {
      const int c = sp.cell[j];
      ci = c < 0 ? -1 : cell_r_of(c);
      ck = c < 0 ? -1 : cell_z_of(c);
      id = sp.id[j];
    } else {
      const double r = sp.r[j];
      ci = r >= 0.0 ? (int)floor(r / g.dr) : -1;  // CELL_NUMBER geometry.hpp:198; dead slots have r < 0
      ck = (int)floor(sp.z[j] / g.dz);
      id = (unsigned)j;
    }
  }
  bool valid = ci >= 0 && ck >= 0 && ci < g.nr && ck < g.nz;
  const unsigned long long c = valid ? (unsigned long long)ci * g.nz + ck : 0ull;
  if (valid && only && only[c] != only_value) valid = false;
  // valid entries are appended (keys are unique, so the sort fixes the order)
  const unsigned mask = __ballot_sync(0xffffffffu, valid);
  const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
  unsigned base = 0;
  if (mask && lane == leader) base = atomicAdd(n_valid, (unsigned)__popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader < 0 ? 0 : leader);
  if (!valid) return;
  const unsigned pos = base + __popc(mask & ((1u << lane) - 1u));
  keys[pos] = (c << 36) | ((unsigned long long)t << 32) | id;
  vals[pos] = ((unsigned long long)t << 40) | j;
  atomicAdd(count + c, 1u);
}

// ---------------------------------------------------------------------------
// 3. shuffle

__global__ void shuffle_kernel(size_t cells, const unsigned* start, const unsigned* count,
                               unsigned long long* vals, uint64_t seed, uint32_t pass, uint32_t list) {
  const size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (c >= cells) return;
  unsigned long long* L = vals + start[c];
  const unsigned n = count[c];
  for (unsigned i = 1; i < n; ++i) {
    uint32_t o[4];
    philox4x32_10((uint32_t)c, i, pass, kShufTag + list, (uint32_t)seed, (uint32_t)(seed >> 32), o);
    unsigned j = (unsigned)(u53(o[0], o[1]) * (double)(i + 1));
    if (j > i) j = i;
    const unsigned long long tmp = L[i];
    L[i] = L[j];
    L[j] = tmp;
  }
}

// ---------------------------------------------------------------------------
// accessors

// A particle of the lists before staging (reference = species << 40 | slot).
__device__ __forceinline__ void load_v(const SpeciesTable& tab, unsigned long long ref, double v[3],
                                       double* w) {
  const CollSpecies& sp = tab.s[ref >> 40];
  const size_t j = ref & kRefMask;
  if (sp.vr64) {
    v[0] = sp.vr64[j]; v[1] = sp.vphi64[j]; v[2] = sp.vz64[j];
    *w = sp.w64[j];
  } else {
    v[0] = sp.vr32[j]; v[1] = sp.vphi32[j]; v[2] = sp.vz32[j];
    *w = sp.w32[j];
  }
}

__device__ __forceinline__ void store_v(const SpeciesTable& tab, unsigned long long ref, const double v[3]) {
  const CollSpecies& sp = tab.s[ref >> 40];
  const size_t j = ref & kRefMask;
  if (sp.vr64) {
    sp.vr64[j] = v[0]; sp.vphi64[j] = v[1]; sp.vz64[j] = v[2];
  } else {
    sp.vr32[j] = (float)v[0]; sp.vphi32[j] = (float)v[1]; sp.vz32[j] = (float)v[2];
  }
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

// 3b. staging: entry q of list `list` is copied to stage[q] and referenced
// by staged[q]; the write-back stores the (possibly scattered) velocities
// through the original reference.  A float velocity that no collision
// touched returns unchanged, (float)(double)x == x.
__global__ void stage_kernel(SpeciesTable tab, const unsigned long long* refs, unsigned n, int list,
                             double4* stage, unsigned long long* staged) {
  const unsigned q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  double v[3], w;
  load_v(tab, refs[q], v, &w);
  stage[q] = make_double4(v[0], v[1], v[2], w);
  staged[q] = kStaged | ((unsigned long long)list << 40) | q;
}

__global__ void unstage_kernel(SpeciesTable tab, const unsigned long long* refs, unsigned n,
                               const double4* stage) {
  const unsigned q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const double4 e = stage[q];
  const double v[3] = {e.x, e.y, e.z};
  store_v(tab, refs[q], v);
}

// ---------------------------------------------------------------------------
// 4. per-cell moments (collisions.cpp:169-221, 123-156)

__global__ void moments_kernel(GridGeom g, Staged tab, CollParams p, const unsigned* st_e,
                               const unsigned* n_e, const unsigned long long* le, const unsigned* st_i,
                               const unsigned* n_i, const unsigned long long* li, double* mom,
                               int* row_stop, double* totals) {
  const size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (c >= (size_t)g.nr * g.nz) return;
  const int i = (int)(c / g.nz), k = (int)(c - (size_t)i * g.nz);
  double e_tot_e = 0, amount_e = 0, e_tot_i = 0, amount_i = 0, v[3], w;
  double pm_e[3] = {0, 0, 0}, pm_i[3] = {0, 0, 0};  // sum w m v (TA77S)
  for (unsigned q = 0; q < n_i[c]; ++q) {
    load_v(tab, li[st_i[c] + q], v, &w);
    const double v_sq = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    const double wm = w * p.m_ion;
    for (int d = 0; d < 3; ++d) pm_i[d] += wm * v[d];
    amount_i += w;
    e_tot_i += wm * v_sq / 2;
  }
  for (unsigned q = 0; q < n_e[c]; ++q) {
    load_v(tab, le[st_e[c] + q], v, &w);
    const double v_sq = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    const double wm = w * p.m_el;
    for (int d = 0; d < 3; ++d) pm_e[d] += wm * v[d];
    amount_e += w;
    e_tot_e += wm * v_sq / 2;
  }
  if (totals) {
    double* t = totals + 10 * c;
    t[0] = amount_e; t[1] = pm_e[0]; t[2] = pm_e[1]; t[3] = pm_e[2]; t[4] = e_tot_e;
    t[5] = amount_i; t[6] = pm_i[0]; t[7] = pm_i[1]; t[8] = pm_i[2]; t[9] = e_tot_i;
  }
  const double vol = kPi * g.dz * g.dr * g.dr * (2.0 * i + 1);  // CELL_VOLUME(i)
  const double T_el = e_tot_e / amount_e * (1. / kElCharge);
  const double T_ion = e_tot_i / amount_i * (1. / kElCharge);
  double n_el = 0, n_ion = 0;
  for (unsigned q = 0; q < n_e[c]; ++q) n_el += load_w(tab, le[st_e[c] + q]);
  for (unsigned q = 0; q < n_i[c]; ++q) n_ion += load_w(tab, li[st_i[c] + q]);
  n_el /= vol;
  n_ion /= vol;
  mom[4 * c + 0] = T_el;
  mom[4 * c + 1] = T_ion;
  mom[4 * c + 2] = n_el;
  mom[4 * c + 3] = n_ion;
  if (!normal(T_ion) || !normal(T_el) || !normal(n_ion) || !normal(n_el))
    atomicMin(row_stop + i, k);
}

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

__device__ void p12_single(PairCtx& x, double m_real_a, double m_real_b, double q_real_a,
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

__device__ void ta77s_single(PairCtx& x, double m_real_a, double m_real_b, double q_real_a,
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

__device__ void sk98_single(PairCtx& x, double m_real_a, double m_real_b, double q_real_a,
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

// correct_velocities (collisionsTA77S.cpp:419-566) of one list of one cell:
// remove the list's momentum change and scale its thermal velocities by
// sqrt(alpha) so that momentum and kinetic energy return to the totals t
// (sum w, sum w m v, sum w m v^2/2) collected before the pass.  The
// reference takes |alpha| for alpha < 0 and 1 for alpha == 0; the fixed
// mode leaves such a list as it is.
__device__ void ta77s_correct(const Staged& tab, const unsigned long long* L, unsigned n, double mass,
                              const double* t, int fixed) {
  double m3[3] = {0, 0, 0}, e_new = 0, v[3], w;
  for (unsigned q = 0; q < n; ++q) {
    load_v(tab, L[q], v, &w);
    const double v_sq = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    const double mass_m = mass * w;
    for (int d = 0; d < 3; ++d) m3[d] += mass_m * v[d];
    e_new += mass_m * v_sq / 2;
  }
  const double mass_tot = t[0] * mass;
  double dv[3], v0[3];
  for (int d = 0; d < 3; ++d) {
    dv[d] = (m3[d] - t[1 + d]) / mass_tot;
    v0[d] = t[1 + d] / mass_tot;
  }
  const double d_e = e_new - t[4];
  const double v0_sq = v0[0] * v0[0] + v0[1] * v0[1] + v0[2] * v0[2];
  double alpha = (t[4] - mass_tot * v0_sq / 2) /
                 (t[4] + d_e - mass_tot * ((v0[0] + dv[0]) * (v0[0] + dv[0]) + (v0[1] + dv[1]) * (v0[1] + dv[1]) +
                                           (v0[2] + dv[2]) * (v0[2] + dv[2])) / 2);
  if (!normal(alpha)) return;
  if (fixed) {
    if (alpha < 0) return;
  } else {
    if (alpha < 0) alpha = -alpha;
  }
  alpha = sqrt(alpha);
  for (unsigned q = 0; q < n; ++q) {
    load_v(tab, L[q], v, &w);
    const double c[3] = {v0[0] + alpha * (v[0] - v0[0] - dv[0]), v0[1] + alpha * (v[1] - v0[1] - dv[1]),
                         v0[2] + alpha * (v[2] - v0[2] - dv[2])};
    store_v(tab, L[q], c);
  }
}

__global__ void ta77s_correct_kernel(GridGeom g, Staged tab, CollParams p, const unsigned* st_e,
                                     const unsigned* n_e, const unsigned long long* le, const unsigned* st_i,
                                     const unsigned* n_i, const unsigned long long* li, const double* totals) {
  const size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (c >= (size_t)g.nr * g.nz) return;
  if (p.only && p.only[c] != p.only_value) return;
  ta77s_correct(tab, li + st_i[c], n_i[c], p.m_ion, totals + 10 * c + 5, p.fixed);
  ta77s_correct(tab, le + st_e[c], n_e[c], p.m_el, totals + 10 * c, p.fixed);
}

// ---------------------------------------------------------------------------
// 5. the per-cell pairing sequence (collisionsP12.cpp:338-548), one kernel
// instance per scheme (SCHEME = CollParams::scheme: 0 P12, 1 TA77S, 2 SK98)
// so that each is compiled, and given registers, for its own pair function.

template <int SCHEME>
__global__ void collide_kernel(GridGeom g, Staged tab, CollParams p, const unsigned* st_e,
                               const unsigned* n_e, const unsigned long long* le, const unsigned* st_i,
                               const unsigned* n_i, const unsigned long long* li, const double* mom,
                               const int* row_stop, unsigned long long* calls) {
  const size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (c >= (size_t)g.nr * g.nz) return;
  if (p.only && p.only[c] != p.only_value) return;
  const int i = (int)(c / g.nz), k = (int)(c - (size_t)i * g.nz);
  const double T_el = mom[4 * c], T_ion = mom[4 * c + 1], n_el = mom[4 * c + 2], n_ion = mom[4 * c + 3];
  if (p.fixed) {
    if (!normal(T_ion) || !normal(T_el) || !normal(n_ion) || !normal(n_el)) return;
  } else if (k >= row_stop[i]) {
    return;  // `break` out of the row at its first non-normal cell
  }
  const double debye = 7433.944 / sqrt(n_el / T_el + n_ion / T_ion);  // plasma.cpp:24-33
  const unsigned long long* E = le + st_e[c];
  const unsigned long long* I = li + st_i[c];
  const unsigned ne = n_e[c], ni = n_i[c];
  const double me = p.m_el, mi = p.m_ion, qe = p.q_el, qi = p.q_ion;
  double expect[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  PairCtx x{&tab, &p, (uint32_t)c, 0u, p.expect ? expect : nullptr};
#define COLL(MA, MB, QA, QB, A, B, NA, NB)                                       \
  do {                                                                           \
    if (SCHEME == 1) ta77s_single(x, MA, MB, QA, QB, A, B, NA, NB, debye);        \
    else if (SCHEME == 2) sk98_single(x, MA, MB, QA, QB, A, B, NA, NB, debye);    \
    else p12_single(x, MA, MB, QA, QB, A, B, NA, NB, debye);                     \
    ++x.m;                                                                       \
  } while (0)
  if (ni % 2 == 0)
    for (unsigned q = 0; q < ni; q += 2) COLL(mi, mi, qi, qi, I[q], I[q + 1], n_ion, n_ion);
  if (ne % 2 == 0)
    for (unsigned q = 0; q < ne; q += 2) COLL(me, me, qe, qe, E[q], E[q + 1], n_el, n_el);
  if (ni % 2 != 0) {
    if (ni >= 3) {
      COLL(mi, mi, qi, qi, I[0], I[1], n_ion, n_ion);
      COLL(mi, mi, qi, qi, I[1], I[2], n_ion, n_ion);
      COLL(mi, mi, qi, qi, I[2], I[0], n_ion, n_ion);
    }
    if (ni >= 5)
      for (unsigned q = 3; q < ni; q += 2) COLL(mi, mi, qi, qi, I[q], I[q + 1], n_ion, n_ion);
  }
  if (ne % 2 != 0) {
    if (ne >= 3) {
      COLL(me, me, qe, qe, E[0], E[1], n_el, n_el);
      COLL(me, me, qe, qe, E[1], E[2], n_el, n_el);
      COLL(me, me, qe, qe, E[2], E[0], n_el, n_el);
    }
    if (ne >= 5)
      for (unsigned q = 3; q < ne; q += 2) COLL(me, me, qe, qe, E[q], E[q + 1], n_el, n_el);
  }
  if (ni == ne)
    for (unsigned q = 0; q < ne; ++q) COLL(me, mi, qe, qi, E[q], I[q], n_el, n_ion);
  if (ni > ne && ne > 0 && ni > 0) {
    const unsigned c_i = (unsigned)floorf((float)ni / (float)ne);
    const double c_r = (double)((float)ni / (float)ne - (float)c_i);
    const unsigned ions_1st = (unsigned)((double)(c_i + 1) * c_r * ne);
    const unsigned els_1st = (unsigned)(c_r * ne);
    const unsigned ions_2nd = (unsigned)((double)c_i * (1 - c_r) * ne);
    for (unsigned fgi = 0; fgi < ions_1st; ++fgi) {
      const int fge = (int)floorf((float)fgi / (float)(c_i + 1));
      COLL(me, mi, qe, qi, E[fge], I[fgi], n_el, n_ion);
    }
    for (unsigned fgi = 0; fgi < ions_2nd; ++fgi) {
      const int fge = (int)floorf((float)fgi / (float)c_i);
      COLL(me, mi, qe, qi, E[fge + els_1st], I[fgi + ions_1st], n_el, n_ion);
    }
  }
  if (ni < ne && ne > 0 && ni > 0) {
    const double c_i = (double)floorf((float)ne / (float)ni);
    const double c_r = (double)((float)ne / (float)ni) - c_i;
    const unsigned els_1st = (unsigned)((c_i + 1) * c_r * ni);
    const unsigned ions_1st = (unsigned)(c_r * ni);
    const unsigned els_2nd = (unsigned)(c_i * (1 - c_r) * ni);
    for (unsigned fge = 0; fge < els_1st; ++fge) {
      const int fgi = (int)floorf((float)fge / (float)(c_i + 1));
      COLL(me, mi, qe, qi, E[fge], I[fgi], n_el, n_ion);
    }
    for (unsigned fge = 0; fge < els_2nd; ++fge) {
      const int fgi = (int)floorf((float)fge / (float)c_i);
      COLL(me, mi, qe, qi, E[fge + els_1st], I[fgi + ions_1st], n_el, n_ion);
    }
  }
#undef COLL
  if (x.m) atomicAdd(calls, (unsigned long long)x.m);
  if (p.expect)
    for (int q = 0; q < 12; ++q) p.expect[c * 12 + q] = expect[q];
}

template <typename T>
int grow(T** p, size_t n) {
  cudaFree(*p);
  *p = nullptr;
  return cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T)) == cudaSuccess ? 0 : -1;
}

}  // namespace

void collide_free(CollWork& w) {
  for (int l = 0; l < 2; ++l) {
    cudaFree(w.keys[l]); cudaFree(w.keys2[l]); cudaFree(w.vals[l]); cudaFree(w.vals2[l]);
    cudaFree(w.count[l]); cudaFree(w.start[l]); cudaFree(w.stage[l]);
  }
  cudaFree(w.moments); cudaFree(w.row_stop); cudaFree(w.calls); cudaFree(w.valid); cudaFree(w.tmp);
  cudaFree(w.totals);
  w = CollWork();
}

int collide_p12(const GridGeom& g, const CollSpecies* sp, int nsp, const CollParams& p, CollWork& w,
                unsigned long long* pair_calls, cudaStream_t s) {
  if (nsp > kCollMaxSpecies) return -1;
  SpeciesTable tab{};
  tab.n = nsp;
  size_t total[2] = {0, 0};
  for (int t = 0; t < nsp; ++t) {
    tab.s[t] = sp[t];
    total[sp[t].is_ion ? 1 : 0] += sp[t].n;
  }
  const size_t cells = (size_t)g.nr * g.nz;
  const size_t need = std::max(total[0], total[1]);
  if (w.cap < need || w.cells != cells) {
    for (int l = 0; l < 2; ++l) {
      if (grow(&w.keys[l], need) || grow(&w.keys2[l], need) || grow(&w.vals[l], need) ||
          grow(&w.vals2[l], need) || grow(&w.count[l], cells + 1) || grow(&w.start[l], cells + 1) ||
          grow(&w.stage[l], need))
        return -1;
    }
    if (grow(&w.moments, 4 * cells) || grow(&w.row_stop, (size_t)g.nr) || grow(&w.calls, 1) ||
        grow(&w.valid, 2))
      return -1;
    size_t b1 = 0, b2 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, b1, w.keys[0], w.keys2[0], w.vals[0], w.vals2[0], (int)need);
    cub::DeviceScan::ExclusiveSum(nullptr, b2, w.count[0], w.start[0], (int)(cells + 1));
    w.tmp_bytes = std::max(b1, b2);
    if (grow((char**)&w.tmp, w.tmp_bytes)) return -1;
    w.cap = need;
    w.cells = cells;
  }
  if (p.scheme == 1 && w.totals_cells != cells) {
    if (grow(&w.totals, 10 * cells)) return -1;
    w.totals_cells = cells;
  }
  cudaMemsetAsync(w.calls, 0, sizeof(unsigned long long), s);
  cudaMemsetAsync(w.valid, 0, 2 * sizeof(unsigned), s);
  w.launches = 2;  // moments and the pairs
  for (int l = 0; l < 2; ++l) {
    cudaMemsetAsync(w.count[l], 0, (cells + 1) * sizeof(unsigned), s);
    for (int t = 0; t < nsp; ++t) {
      if ((sp[t].is_ion ? 1 : 0) != l || !sp[t].n) continue;
      key_kernel<<<blocks_for(sp[t].n), kThreads, 0, s>>>(g, tab, t, w.keys[l], w.vals[l], w.count[l],
                                                          w.valid + l, p.only, p.only_value);
      ++w.launches;
    }
  }
  unsigned valid[2] = {0, 0};
  if (cudaMemcpyAsync(valid, w.valid, 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return -1;
  for (int l = 0; l < 2; ++l) {
    if (valid[l]) {
      size_t b = w.tmp_bytes;
      int bits = 36;  // the key is cell << 36 | species << 32 | id, cell < 2^28
      while (bits < 64 && (1ull << (bits - 36)) < cells) ++bits;
      cub::DeviceRadixSort::SortPairs(w.tmp, b, w.keys[l], w.keys2[l], w.vals[l], w.vals2[l],
                                      (int)valid[l], 0, std::min(bits + 1, 64), s);
    }
    size_t b = w.tmp_bytes;
    cub::DeviceScan::ExclusiveSum(w.tmp, b, w.count[l], w.start[l], (int)(cells + 1), s);
    if (p.shuffle && valid[l]) {
      shuffle_kernel<<<blocks_for(cells), kThreads, 0, s>>>(cells, w.start[l], w.count[l], w.vals2[l],
                                                             p.seed, p.pass, (uint32_t)l);
      ++w.launches;
    }
    // the sorted keys are spent: keys2 now holds the staged references
    if (valid[l]) {
      stage_kernel<<<blocks_for(valid[l]), kThreads, 0, s>>>(tab, w.vals2[l], valid[l], l, w.stage[l],
                                                             w.keys2[l]);
      w.launches += 2;  // and its write-back
    }
  }
  const Staged staged{{w.stage[0], w.stage[1]}};
  // 0x7f7f7f7f in every row: no stop unless a non-normal cell sets one
  cudaMemsetAsync(w.row_stop, 0x7f, (size_t)g.nr * sizeof(int), s);
  moments_kernel<<<blocks_for(cells), kThreads, 0, s>>>(g, staged, p, w.start[0], w.count[0], w.keys2[0],
                                                        w.start[1], w.count[1], w.keys2[1], w.moments,
                                                        w.row_stop, p.scheme == 1 ? w.totals : nullptr);
  auto collide = p.scheme == 1 ? collide_kernel<1> : p.scheme == 2 ? collide_kernel<2> : collide_kernel<0>;
  collide<<<blocks_for(cells), kThreads, 0, s>>>(g, staged, p, w.start[0], w.count[0], w.keys2[0], w.start[1],
                                                 w.count[1], w.keys2[1], w.moments, w.row_stop, w.calls);
  if (p.scheme == 1) {
    ta77s_correct_kernel<<<blocks_for(cells), kThreads, 0, s>>>(g, staged, p, w.start[0], w.count[0], w.keys2[0],
                                                                w.start[1], w.count[1], w.keys2[1], w.totals);
    ++w.launches;
  }
  for (int l = 0; l < 2; ++l)
    if (valid[l])
      unstage_kernel<<<blocks_for(valid[l]), kThreads, 0, s>>>(tab, w.vals2[l], valid[l], w.stage[l]);
  if (cudaMemcpyAsync(pair_calls, w.calls, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return -1;
  if (cudaStreamSynchronize(s) != cudaSuccess) return -1;
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace pcg
