/*
 * pic_oracle.c — CPU restatement of PiCoPiC's per-timestep PIC loop.
 *
 * TEST INFRASTRUCTURE ONLY (see pic_oracle.h).  Every function cites the
 * reference file:line it restates.  The operation order of every floating
 * point expression follows the reference source exactly, including the
 * reference's arithmetic defects, so that with -ffp-contract=off the
 * results are bit-identical to the compiled reference (oracle/_ref).
 *
 * Constants are the reference's rounded SI values (constant.hpp:35-57).
 */
#include "pic_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define K_PI 3.1415926535897932
#define K_EPSILON0 8.85E-12
#define K_EL_MASS 9.1E-31
#define K_EL_CHARGE 1.6E-19
#define K_LIGHT_VEL 3.0E8
#define K_LIGHT_VEL_POW_2 (K_LIGHT_VEL * K_LIGHT_VEL)
#define K_MAGN_CONST 1.26E-6
#define K_MNZL 1e-15
#define K_REL_LIMIT 5e7
#define K_REL_LIMIT_POW_2 (K_REL_LIMIT * K_REL_LIMIT)
#define MAX_SPECIES 16

/* Status codes shared with the product ABI. */
#define ST_OK 0
#define ST_ARG (-1)
#define ST_FATAL (-10)

typedef struct {
  int id, is_beam;
  char name[64];
  double charge, mass; /* SI: SpecieP ctor specieP.cpp:37-38 */
  size_t n, cap;
  double *r, *phi, *z, *r_old, *phi_old, *z_old, *vr, *vphi, *vz, *w, *sn;
  long long *cell_r, *cell_z;
  double* abs_map; /* SpecieP::momentum_abs_map_w as the last energy map left it (NULL: zeros) */
  /* BeamP state (beamP.cpp:22-69) */
  unsigned macro_amount, bunches_amount, current_bunch;
  double start_time, radius, density, bunch_length, bunches_distance, velocity;
  double finish_time, domain_radius, bunch_macro_amount, macro_per_step;
} species_t;

typedef struct {
  uint32_t mt[624];
  int idx;
} mt19937_t;

struct orc_sim {
  int nr, nz, ld;
  double R, L, dr, dz, dt, t;
  int pml[4];
  double pml_sigma[2];
  size_t gcr, gcz; /* Geometry::global_cell_amount (geometry.hpp:70-71) */
  int pusher, current, quirks;
  double *E[3], *H[3], *Hat[3], *J[3], *sigma;
  double *Eext[3], *Hext[3]; /* ExternalFields' field_e, field_h (NULL: none) */
  int nsp;
  species_t sp[MAX_SPECIES];
  int rng_kind;
  uint64_t seed, step_index;
  uint32_t coll_pass; /* collision passes so far: the Philox counter of their draws */
  mt19937_t mt;
  long errors, removed;
};

/* ------------------------------------------------------------------ */
/* Grid<T> indexing with the 2-cell halo (grid.hpp:46-58, 165-168).     */
#define IDX(s, i, k) ((size_t)((i) + 2) * (size_t)(s)->ld + (size_t)((k) + 2))

static void halo_set(orc_sim* s, double* a, double v) { /* Grid::overlay_set grid.hpp:87-97 */
  int xr = s->nr + 4, yr = s->nz + 4;
  for (int i = 0; i < xr; ++i)
    for (int j = 0; j < yr; ++j)
      if (i < 2 || j < 2 || i >= xr - 2 || j >= yr - 2) a[(size_t)i * yr + j] = v;
}

/* ------------------------------------------------------------------ */
/* Random sources                                                       */

static void mt_seed(mt19937_t* g, uint32_t s) {
  g->mt[0] = s;
  for (int i = 1; i < 624; ++i)
    g->mt[i] = 1812433253u * (g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) + (uint32_t)i;
  g->idx = 624;
}

static uint32_t mt_next(mt19937_t* g) {
  if (g->idx >= 624) {
    for (int i = 0; i < 624; ++i) {
      uint32_t x = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
      uint32_t xa = x >> 1;
      if (x & 1u) xa ^= 0x9908b0dfu;
      g->mt[i] = g->mt[(i + 397) % 624] ^ xa;
    }
    g->idx = 0;
  }
  uint32_t y = g->mt[g->idx++];
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}

/* std::uniform_real_distribution<double>(0, 1) over std::mt19937 as
 * libstdc++ implements it: generate_canonical<double, 53> draws two 32-bit
 * words, sum = w0 + w1 * 2^32 (rounded to double), result = sum / 2^64,
 * clamped below 1. */
static double mt_uniform(mt19937_t* g) {
  double sum = 0.0, tmp = 1.0;
  for (int k = 0; k < 2; ++k) {
    sum += (double)mt_next(g) * tmp;
    tmp *= 4294967296.0;
  }
  double r = sum / tmp;
  if (r >= 1.0) r = nextafter(1.0, 0.0);
  return r;
}

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int round = 0; round < 10; ++round) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Two 53-bit uniforms in [0,1) per Philox block: which = 0 or 1. */
double orc_philox_uniform(uint64_t seed, uint32_t stream, uint64_t step, uint32_t index,
                          int which) {
  uint32_t ctr[4] = {index, (uint32_t)step, (uint32_t)(step >> 32), stream};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t o[4];
  orc_philox4x32_10(ctr, key, o);
  uint32_t a = which ? o[2] : o[0], b = which ? o[3] : o[1];
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

/* ------------------------------------------------------------------ */
/* Relativity: phys::rel (rel.cpp:24-55)                                */

static int lorenz_factor(double sq_velocity, double* gamma_out) {
  double beta = sq_velocity / K_LIGHT_VEL_POW_2;
  if (beta > 1) return ST_FATAL; /* LOG_S(FATAL) rel.cpp:33-34 */
  double gamma = 1 / sqrt(1.0 - beta);
  if (isinf(gamma)) gamma = 1e100; /* rel.cpp:38-42 */
  *gamma_out = gamma;
  return ST_OK;
}

static double lorenz_factor_inv(double sq_velocity) {
  return pow(1.0 + sq_velocity / K_LIGHT_VEL_POW_2, -0.5);
}

/* ------------------------------------------------------------------ */
/* Geometry macros (geometry.hpp:186-198), keeping the reference's        */
/* unparenthesised macro argument: CELL_VOLUME(i+1) expands to            */
/* PI*dz*dr*dr*(2.0*i + 1 + 1).                                           */

static inline double cell_volume_expr(double two_i_plus_rest, double dr, double dz) {
  return K_PI * dz * dr * dr * two_i_plus_rest;
}
#define CELL_NUMBER(pos, dx) ((int)floor((pos) / (dx)))

/* ------------------------------------------------------------------ */
/* PML: MaxwellSolverYee::set_pml (maxwellSolverYee.cpp:57-109)          */

static void set_pml(orc_sim* s) {
  double dr = s->dr, dz = s->dz;
  double l_left = dz * (double)s->pml[1];
  double l_right = dz * (double)s->pml[3];
  double l_ext = dr * (double)s->pml[2];
  double r_off = 0.0 * dr, z_off = 0.0 * dz;
  double sys_r = s->R, sys_l = s->L;
  double dsig = s->pml_sigma[1] - s->pml_sigma[0];
  if (s->pml[2] != 0)
    for (int i = 0; i < s->nr; i++)
      for (int k = 0; k < s->nz; k++) {
        double dist = (double)(s->gcr - 0 - (size_t)i) * dr; /* Geometry::dist_x_to_end */
        if (dist < l_ext)
          s->sigma[IDX(s, i, k)] += s->pml_sigma[0] + dsig / pow(l_ext, 2) *
                                                          pow(dr * (i + 1) + r_off - sys_r + l_ext, 2);
      }
  if (s->pml[1] != 0)
    for (int k = 0; k < s->nz; k++)
      for (int i = 0; i < s->nr; i++)
        if (dz * k + z_off < l_left)
          s->sigma[IDX(s, i, k)] += s->pml_sigma[0] + dsig / pow(l_left, 2) *
                                                          pow(l_left - dz * k - z_off, 2);
  if (s->pml[3] != 0)
    for (int k = 0; k < s->nz; k++)
      for (int i = 0; i < s->nr; i++) {
        double dist = (double)(s->gcz - 0 - (size_t)k) * dz; /* Geometry::dist_y_to_end */
        if (dist < l_right)
          s->sigma[IDX(s, i, k)] += s->pml_sigma[0] + dsig / pow(l_right, 2) *
                                                          pow(dz * (k + 1) + z_off - sys_l + l_right, 2);
      }
}

/* ------------------------------------------------------------------ */
/* Yee solver                                                            */

/* MaxwellSolverYee::calc_field_e (maxwellSolverYee.cpp:161-257); one
 * domain: walls on, r_begin = z_begin = 1, r_end = nr-1, z_end = nz-1. */
static int field_e(orc_sim* s) {
  double *Er = s->E[0], *Ep = s->E[1], *Ez = s->E[2];
  double *Jr = s->J[0], *Jp = s->J[1], *Jz = s->J[2];
  double *Hr = s->Hat[0], *Hp = s->Hat[1], *Hz = s->Hat[2];
  for (int c = 0; c < 3; ++c) halo_set(s, s->E[c], 0.0);
  double dr = s->dr, dz = s->dz, dt = s->dt;
  int r_begin = 1, z_begin = 1, r_end = s->nr - 1, z_end = s->nz - 1;

  for (int k = z_begin; k < z_end; ++k) { /* axis r = 0, :170-194 */
    int i = 0;
    double epsx2 = 2 * K_EPSILON0;
    double sigma_t = s->sigma[IDX(s, i, k)] * dt;
    double koef_e = (epsx2 - sigma_t) / (epsx2 + sigma_t);
    double koef_h = 2 * dt / (epsx2 + sigma_t);
    size_t p = IDX(s, i, k);
    Er[p] *= koef_e;
    Er[p] -= (Jr[p] + (Hp[p] - Hp[IDX(s, i, k - 1)]) / dz) * koef_h;
    Ez[p] *= koef_e;
    Ez[p] -= (Jz[p] - Hp[p] * 4. / dr) * koef_h;
  }
  for (int i = r_begin; i < r_end; ++i) { /* z = 0 wall, :196-218 */
    int k = 0;
    double epsx2 = 2 * K_EPSILON0;
    double sigma_t = s->sigma[IDX(s, i, k)] * dt;
    double koef_e = (epsx2 - sigma_t) / (epsx2 + sigma_t);
    double koef_h = 2 * dt / (epsx2 + sigma_t);
    size_t p = IDX(s, i, k), pm = IDX(s, i - 1, k);
    Ez[p] *= koef_e;
    Ez[p] -= (Jz[p] - (Hp[p] - Hp[pm]) / dr - (Hp[p] + Hp[pm]) / (2. * dr * (double)i)) * koef_h;
  }
  for (int i = r_begin; i < r_end; i++) /* regular, :220-256 */
    for (int k = z_begin; k < z_end; k++) {
      double epsx2 = 2 * K_EPSILON0;
      double sigma_t = s->sigma[IDX(s, i, k)] * dt;
      double koef_e = (epsx2 - sigma_t) / (epsx2 + sigma_t);
      double koef_h = 2 * dt / (epsx2 + sigma_t);
      size_t p = IDX(s, i, k), pkm = IDX(s, i, k - 1), pim = IDX(s, i - 1, k);
      Er[p] *= koef_e;
      Er[p] -= (Jr[p] + (Hp[p] - Hp[pkm]) / dz) * koef_h;
      Ep[p] *= koef_e;
      Ep[p] -= (Jp[p] - (Hr[p] - Hr[pkm]) / dz + (Hz[p] - Hz[pim]) / dr) * koef_h;
      Ez[p] *= koef_e;
      Ez[p] -= (Jz[p] - (Hp[p] - Hp[pim]) / dr - (Hp[p] + Hp[pim]) / (2. * dr * (double)i)) * koef_h;
      if (isnan(Er[p]) || isnan(Ep[p]) || isnan(Ez[p])) return ST_FATAL; /* :253-255 */
    }
  return ST_OK;
}

/* MaxwellSolverYee::calc_field_h (maxwellSolverYee.cpp:111-159). */
static int field_h(orc_sim* s) {
  double *Er = s->E[0], *Ep = s->E[1], *Ez = s->E[2];
  for (int c = 0; c < 3; ++c) {
    halo_set(s, s->H[c], 0.0);
    halo_set(s, s->Hat[c], 0.0);
  }
  double dr = s->dr, dz = s->dz, dt = s->dt;
  int fix = s->quirks == ORC_QUIRKS_FIXED;
  if (!fix) /* outer-wall H_r loop :119-130, updated again by the regular loop */
    for (int k = 0; k < s->nz; k++) {
      int i = s->nr - 1;
      size_t p = IDX(s, i, k);
      double alpha_t = dt * (Ep[IDX(s, i, k + 1)] - Ep[p]) / (dz * K_MAGN_CONST);
      s->H[0][p] = s->Hat[0][p] + alpha_t / 2;
      s->Hat[0][p] += alpha_t;
    }
  for (int i = 0; i < s->nr; i++)
    for (int k = 0; k < s->nz; k++) {
      size_t p = IDX(s, i, k), pk = IDX(s, i, k + 1), pi = IDX(s, i + 1, k);
      double a_r = dt * (Ep[pk] - Ep[p]) / (dz * K_MAGN_CONST);
      s->H[0][p] = s->Hat[0][p] + a_r / 2;
      s->Hat[0][p] += a_r;
      double a_phi = dt * ((Ez[pi] - Ez[p]) / dr - (Er[pk] - Er[p]) / dz) / K_MAGN_CONST;
      s->H[1][p] = s->Hat[1][p] + a_phi / 2;
      s->Hat[1][p] += a_phi;
      double a_z = dt * ((Ep[pi] + Ep[p]) / (2. * dr * (i + 0.5 + 0.0)) + (Ep[pi] - Ep[p]) / dr) / K_MAGN_CONST;
      s->H[2][p] = s->Hat[2][p] - a_z / 2;
      s->Hat[2][p] -= a_z;
    }
  return ST_OK;
}

/* ------------------------------------------------------------------ */
/* Field gather: MaxwellSolver::get_field_h / get_field_e                */
/* (maxwellSolver.hpp:101-209, 211-316).  Each term is                   */
/*   field * PI * dz_ * (rb*rb - ra*ra) / vol                            */
/* evaluated left to right, as the macro expansion of CYL_RNG_VOL gives.  */

static inline double term(double f, double dzz, double ra, double rb, double vol) {
  return f * K_PI * dzz * (rb * rb - ra * ra) / vol;
}

/* The fixed mode divides each ring term by the volume of the particle's
 * cloud, pi dz (r3^2 - r1^2), so that the weights of a component sum to 1;
 * the reference divides by cell volumes, which weights a uniform field by
 * about 1 - 1/(2i) at row i (a density-deposit formula used to interpolate). */
#define GATHER_VOLUMES(s, a, b)                                            \
  do {                                                                     \
    if ((s)->quirks == ORC_QUIRKS_FIXED) (a) = (b) = cloud;                \
  } while (0)

static void gather_h(const orc_sim* s, double* const H[3], double radius, double longitude, double cmp[3]) {
  const double dr = s->dr, dz = s->dz;
  const double *Hr = H[0], *Hp = H[1], *Hz = H[2];
  double r1 = radius - 0.5 * dr, r3 = radius + 0.5 * dr, r2, dz1, dz2, v1, v2;
  const double cloud = K_PI * dz * (r3 * r3 - r1 * r1);
  int i, k;
  cmp[0] = cmp[1] = cmp[2] = 0;
  /* H_z :120-147 */
  i = CELL_NUMBER(radius - 0.5 * dr, dr);
  k = CELL_NUMBER(longitude, dz);
  v1 = cell_volume_expr(2.0 * i + 1 + 1, dr, dz);
  v2 = cell_volume_expr(2.0 * i + 3 + 1, dr, dz);
  GATHER_VOLUMES(s, v1, v2);
  dz1 = (k + 1) * dz - longitude;
  dz2 = longitude - k * dz;
  r2 = (i + 1) * dr;
  cmp[2] += term(Hz[IDX(s, i, k)], dz1, r1, r2, v1);
  cmp[2] += term(Hz[IDX(s, i + 1, k)], dz1, r2, r3, v2);
  cmp[2] += term(Hz[IDX(s, i, k + 1)], dz2, r1, r2, v1);
  cmp[2] += term(Hz[IDX(s, i + 1, k + 1)], dz2, r2, r3, v2);
  /* H_r :149-177 */
  i = CELL_NUMBER(radius, dr);
  k = CELL_NUMBER(longitude - 0.5 * dz, dz);
  v1 = cell_volume_expr(2.0 * i + 1, dr, dz);
  v2 = cell_volume_expr(2.0 * i + 2 + 1, dr, dz);
  GATHER_VOLUMES(s, v1, v2);
  r2 = (i + 0.5) * dr;
  dz1 = (k + 1.5) * dz - longitude;
  dz2 = longitude - (k + 0.5) * dz;
  cmp[0] += term(Hr[IDX(s, i, k)], dz1, r1, r2, v1);
  cmp[0] += term(Hr[IDX(s, i + 1, k)], dz1, r2, r3, v2);
  cmp[0] += term(Hr[IDX(s, i, k + 1)], dz2, r1, r2, v1);
  cmp[0] += term(Hr[IDX(s, i + 1, k + 1)], dz2, r2, r3, v2);
  /* H_phi :179-206 */
  i = CELL_NUMBER(radius - 0.5 * dr, dr);
  k = CELL_NUMBER(longitude - 0.5 * dz, dz);
  r2 = (i + 1) * dr;
  v1 = cell_volume_expr(2.0 * i + 1 + 1, dr, dz);
  v2 = cell_volume_expr(2.0 * i + 3 + 1, dr, dz);
  GATHER_VOLUMES(s, v1, v2);
  dz1 = (k + 1.5) * dz - longitude;
  dz2 = longitude - (k + 0.5) * dz;
  cmp[1] += term(Hp[IDX(s, i, k)], dz1, r1, r2, v1);
  cmp[1] += term(Hp[IDX(s, i + 1, k)], dz1, r2, r3, v2);
  cmp[1] += term(Hp[IDX(s, i, k + 1)], dz2, r1, r2, v1);
  cmp[1] += term(Hp[IDX(s, i + 1, k + 1)], dz2, r2, r3, v2);
}

static void gather_e(const orc_sim* s, double* const E[3], double radius, double longitude, double cmp[3]) {
  const double dr = s->dr, dz = s->dz;
  const double *Er = E[0], *Ep = E[1], *Ez = E[2];
  double r1 = radius - 0.5 * dr, r3 = radius + 0.5 * dr, r2, dz1, dz2, v1, v2;
  const double cloud = K_PI * dz * (r3 * r3 - r1 * r1);
  int i, k;
  cmp[0] = cmp[1] = cmp[2] = 0;
  /* E_r :231-257 */
  i = CELL_NUMBER(radius - 0.5 * dr, dr);
  k = CELL_NUMBER(longitude, dz);
  v1 = cell_volume_expr(2.0 * i + 1 + 1, dr, dz);
  v2 = cell_volume_expr(2.0 * i + 3 + 1, dr, dz);
  GATHER_VOLUMES(s, v1, v2);
  dz1 = (k + 1) * dz - longitude;
  dz2 = longitude - k * dz;
  r2 = (i + 1) * dr;
  cmp[0] += term(Er[IDX(s, i, k)], dz1, r1, r2, v1);
  cmp[0] += term(Er[IDX(s, i + 1, k)], dz1, r2, r3, v2);
  cmp[0] += term(Er[IDX(s, i, k + 1)], dz2, r1, r2, v1);
  cmp[0] += term(Er[IDX(s, i + 1, k + 1)], dz2, r2, r3, v2);
  /* E_z :259-283 */
  i = CELL_NUMBER(radius, dr);
  k = CELL_NUMBER(longitude - 0.5 * dz, dz);
  v1 = cell_volume_expr(2.0 * i + 1, dr, dz);
  v2 = cell_volume_expr(2.0 * i + 2 + 1, dr, dz);
  GATHER_VOLUMES(s, v1, v2);
  r2 = (i + 0.5) * dr;
  dz1 = (k + 1.5) * dz - longitude;
  dz2 = longitude - (k + 0.5) * dz;
  cmp[2] += term(Ez[IDX(s, i, k)], dz1, r1, r2, v1);
  cmp[2] += term(Ez[IDX(s, i + 1, k)], dz1, r2, r3, v2);
  cmp[2] += term(Ez[IDX(s, i, k + 1)], dz2, r1, r2, v1);
  cmp[2] += term(Ez[IDX(s, i + 1, k + 1)], dz2, r2, r3, v2);
  /* E_phi :285-313; the reference adds the [i+1][k+1] E_phi term to E_z */
  i = CELL_NUMBER(radius, dr);
  k = CELL_NUMBER(longitude, dz);
  v1 = cell_volume_expr(2.0 * i + 1, dr, dz);
  v2 = cell_volume_expr(2.0 * i + 2 + 1, dr, dz);
  GATHER_VOLUMES(s, v1, v2);
  r2 = (i + 0.5) * dr;
  dz1 = (k + 1) * dz - longitude;
  dz2 = longitude - k * dz;
  cmp[1] += term(Ep[IDX(s, i, k)], dz1, r1, r2, v1);
  cmp[1] += term(Ep[IDX(s, i + 1, k)], dz1, r2, r3, v2);
  cmp[1] += term(Ep[IDX(s, i, k + 1)], dz2, r1, r2, v1);
  if (s->quirks == ORC_QUIRKS_FIXED)
    cmp[1] += term(Ep[IDX(s, i + 1, k + 1)], dz2, r2, r3, v2);
  else
    cmp[2] += term(Ep[IDX(s, i + 1, k + 1)], dz2, r2, r3, v2);
}

/* ------------------------------------------------------------------ */
/* Pushers                                                               */

static double len2(const double v[3]) { return v[0] * v[0] + v[1] * v[1] + v[2] * v[2]; }

/* PusherBoris::operator() (pusherBoris.cpp:23-151) for one particle.
 * ADAPTIVE uses v^2 > REL_LIMIT^2 as the (intended) switch; the reference
 * leaves `use_rel` uninitialised otherwise (:38). */
static int push_boris(int mode, double charge, double mass, double dt, const double e_in[3],
                      const double b_in[3], double v[3]) {
  double e[3] = {e_in[0], e_in[1], e_in[2]}, b[3] = {b_in[0], b_in[1], b_in[2]}, vt[3];
  double c2m = charge * dt / (2 * mass);
  double gamma = 1;
  for (int c = 0; c < 3; ++c) e[c] *= c2m;
  double bk = c2m * K_MAGN_CONST;
  for (int c = 0; c < 3; ++c) b[c] *= bk;
  int use_rel = (mode == ORC_PUSHER_BORIS_RELATIVISTIC) ||
                (mode == ORC_PUSHER_BORIS_ADAPTIVE &&
                 pow(v[0], 2) + pow(v[1], 2) + pow(v[2], 2) > K_REL_LIMIT_POW_2);
  if (use_rel) {
    if (lorenz_factor(len2(v), &gamma) != ST_OK) return ST_FATAL;
    for (int c = 0; c < 3; ++c) v[c] *= gamma;
  }
  for (int c = 0; c < 3; ++c) v[c] += e[c];
  if (use_rel) {
    gamma = lorenz_factor_inv(len2(v));
    for (int c = 0; c < 3; ++c) b[c] *= gamma;
  }
  double const2 = 2. / (1. + len2(b));
  vt[0] = v[0]; vt[1] = v[1]; vt[2] = v[2];
  v[0] = vt[0] + const2 * ((vt[1] - vt[0] * b[2] + vt[2] * b[0]) * b[2] -
                           (vt[2] + vt[0] * b[1] - vt[1] * b[0]) * b[1]);
  v[1] = vt[1] + const2 * (-(vt[0] + vt[1] * b[2] - vt[2] * b[1]) * b[2] +
                           (vt[2] + vt[0] * b[1] - vt[1] * b[0]) * b[0]);
  v[2] = vt[2] + const2 * ((vt[0] + vt[1] * b[2] - vt[2] * b[1]) * b[1] -
                           (vt[1] - vt[0] * b[2] + vt[2] * b[0]) * b[0]);
  for (int c = 0; c < 3; ++c) v[c] += e[c];
  if (use_rel) {
    gamma = lorenz_factor_inv(len2(v));
    for (int c = 0; c < 3; ++c) v[c] *= gamma;
  }
  return ST_OK;
}

static double dot3(const double a[3], const double b[3]) {
  double r = 0;
  for (int c = 0; c < 3; ++c) r += a[c] * b[c];
  return r;
}

/* PusherVay::operator() (pusherVay.cpp:22-114).  quirks=reference keeps
 * the reference's use of u in m/s where the scheme expects u/c. */
static int push_vay(int fixed, double charge, double mass, double dt, const double e_in[3],
                    const double b_in[3], double v[3]) {
  double e[3] = {e_in[0], e_in[1], e_in[2]}, b[3] = {b_in[0], b_in[1], b_in[2]};
  double up[3], psm[3], gamma, s, us2, alpha, B2;
  double c2m = charge * dt / (2 * mass);
  if (lorenz_factor(len2(v), &gamma) != ST_OK) return ST_FATAL;
  for (int c = 0; c < 3; ++c) v[c] *= gamma;
  if (fixed) /* work in units of c */
    for (int c = 0; c < 3; ++c) v[c] /= K_LIGHT_VEL;
  up[0] = v[0]; up[1] = v[1]; up[2] = v[2];
  double ek = 2. * c2m;
  for (int c = 0; c < 3; ++c) e[c] *= ek;
  if (fixed)
    for (int c = 0; c < 3; ++c) e[c] /= K_LIGHT_VEL;
  for (int c = 0; c < 3; ++c) up[c] += e[c];
  double bk = c2m * K_MAGN_CONST;
  for (int c = 0; c < 3; ++c) b[c] *= bk;
  if (fixed) {
    gamma = 1. / sqrt(1. + len2(v));
  } else {
    gamma = lorenz_factor_inv(len2(v));
  }
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
    for (int c = 0; c < 3; ++c) psm[c] *= gamma * K_LIGHT_VEL;
  } else {
    gamma = lorenz_factor_inv(len2(psm));
    for (int c = 0; c < 3; ++c) psm[c] *= gamma;
  }
  v[0] = psm[0]; v[1] = psm[1]; v[2] = psm[2];
  return ST_OK;
}

/* PusherHC::operator() (pusherHC.cpp:23-117).  quirks=reference keeps the
 * m/s-as-normalised defect and inv_det_B = 1/(1+b2[0]+b2[1]+b2[0]) (:94). */
static int push_hc(int fixed, double charge, double mass, double dt, const double e_in[3],
                   const double b_in[3], double v[3]) {
  double e[3] = {e_in[0], e_in[1], e_in[2]}, b[3] = {b_in[0], b_in[1], b_in[2]};
  double psm[3], um[3], upv[3], b2[3], bx[3], gamma, B2;
  double c2m = charge * dt / (2 * mass);
  if (lorenz_factor(len2(v), &gamma) != ST_OK) return ST_FATAL;
  for (int c = 0; c < 3; ++c) v[c] *= gamma;
  if (fixed)
    for (int c = 0; c < 3; ++c) v[c] /= K_LIGHT_VEL;
  for (int c = 0; c < 3; ++c) e[c] *= c2m;
  if (fixed)
    for (int c = 0; c < 3; ++c) e[c] /= K_LIGHT_VEL;
  psm[0] = e[0]; psm[1] = e[1]; psm[2] = e[2];
  for (int c = 0; c < 3; ++c) um[c] = v[c] + psm[c];
  double gfm2 = (1. + len2(um));
  double bk = c2m * K_MAGN_CONST;
  for (int c = 0; c < 3; ++c) b[c] *= bk;
  B2 = len2(b);
  gamma = 1. / sqrt(0.5 * (gfm2 - B2 +
                           sqrt(pow(gfm2 - B2, 2) +
                                4.0 * (B2 + pow(b[0] * um[0] + b[1] * um[1] + b[2] * um[2], 2)))));
  for (int c = 0; c < 3; ++c) b[c] *= gamma;
  for (int c = 0; c < 3; ++c) b2[c] = b[c] * b[c];
  bx[0] = b[0] * b[1];
  bx[1] = b[1] * b[2];
  bx[2] = b[2] * b[0];
  double inv_det_B = fixed ? 1.0 / (1.0 + b2[0] + b2[1] + b2[2]) : 1.0 / (1.0 + b2[0] + b2[1] + b2[0]);
  /* the reference uses b[2] in the last term of up[0] (:97); Higuera-Cary has b[1] */
  upv[0] = ((1.0 + b2[0] - b2[1] - b2[2]) * um[0] + 2. * (bx[0] + b[2]) * um[1] +
            2. * (bx[2] - (fixed ? b[1] : b[2])) * um[2]) * inv_det_B;
  upv[1] = (2. * (bx[0] - b[2]) * um[0] + (1. - b2[0] + b2[1] - b2[2]) * um[1] +
            2. * (bx[1] + b[0]) * um[2]) * inv_det_B;
  upv[2] = (2. * (bx[2] + b[1]) * um[0] + 2. * (bx[1] - b[0]) * um[1] +
            (1. - b2[0] - b2[1] + b2[2]) * um[2]) * inv_det_B;
  for (int c = 0; c < 3; ++c) psm[c] += upv[c];
  if (fixed) {
    gamma = 1. / sqrt(1. + len2(psm));
    for (int c = 0; c < 3; ++c) psm[c] *= gamma * K_LIGHT_VEL;
  } else {
    gamma = lorenz_factor_inv(len2(psm));
    for (int c = 0; c < 3; ++c) psm[c] *= gamma;
  }
  v[0] = psm[0]; v[1] = psm[1]; v[2] = psm[2];
  return ST_OK;
}

/* ------------------------------------------------------------------ */
/* Particle kinematics (specieP.cpp:482-663, beamP.cpp:159-177)          */

static void stage_dump_old(species_t* p) { /* dump_position_to_old :642-650 */
  for (size_t j = 0; j < p->n; ++j) {
    p->r_old[j] = p->r[j];
    p->phi_old[j] = p->phi[j];
    p->z_old[j] = p->z[j];
  }
}

static void stage_move(species_t* p, double dt) { /* mover_cylindrical :482-491 */
  for (size_t j = 0; j < p->n; ++j) {
    p->r[j] = p->r[j] + p->vr[j] * dt;
    p->phi[j] = p->phi[j] + p->vphi[j] * dt;
    p->z[j] = p->z[j] + p->vz[j] * dt;
  }
}

static void stage_pos_rz(species_t* p) { /* back_position_to_rz :609-622 */
  for (size_t j = 0; j < p->n; ++j) {
    double pr = p->r[j], pp = p->phi[j];
    double r = sqrt(pr * pr + pp * pp);
    p->sn[j] = pp / r;
    p->r[j] = r;
    p->phi[j] = 0;
  }
}

static void stage_vel_rz(species_t* p) { /* back_velocity_to_rz :624-640 */
  for (size_t j = 0; j < p->n; ++j) {
    double sn = p->sn[j];
    double cs = sqrt(1 - sn * sn);
    double vr = p->vr[j], vp = p->vphi[j];
    double u2 = cs * vr - sn * vp;
    double v2 = sn * vr + cs * vp;
    p->vr[j] = u2;
    p->vphi[j] = v2;
  }
}

static void stage_bind(species_t* p, double dr, double dz) { /* bind_cell_numbers :652-663 */
  for (size_t j = 0; j < p->n; ++j) {
    p->cell_r[j] = CELL_NUMBER(p->r[j], dr);
    p->cell_z[j] = CELL_NUMBER(p->z[j], dz);
  }
}

/* SpecieP::reflect (specieP.cpp:493-607) for one domain at the origin. */
static int reflect_one(const orc_sim* s, int fixed, double* r, double* z, double r_old,
                       double z_old, double* vr, double* vz) {
  double dr = s->dr, dz = s->dz;
  double half_dr = dr / 2., half_dz = dz / 2.;
  double radius_wall = s->R - dr / 2.;
  double longitude_wall = s->L - dz / 2.;
  double radius_wallX2 = radius_wall * 2.;
  double longitude_wallX2 = longitude_wall * 2.;
  double pos_r = *r - 0.0, pos_z = *z - 0.0;
  double pos_old_r = r_old - 0.0, pos_old_z = z_old - 0.0;
  double pdr = pos_r - pos_old_r, pdz = pos_z - pos_old_z;
  int guard = 0;
  while (isnormal(pos_r) && isnormal(pos_z) &&
         (pos_r > radius_wall || pos_z > longitude_wall || pos_r < half_dr || pos_z < half_dz)) {
    if (++guard > 1000) return ST_FATAL;
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
      pos_old_z = fixed ? half_dz : dz; /* the reference resets to dz (:592) */
      pos_old_r = pos_old_r - dr_small;
      if (pos_z < half_dz) pos_z = half_dz;
    }
  }
  *r = pos_r + 0.0;
  *z = pos_z + 0.0;
  return ST_OK;
}

static int stage_reflect(orc_sim* s, species_t* p) {
  if (p->is_beam) { /* BeamP::reflect beamP.cpp:159-177: the axis only */
    double half_dr = s->dr / 2.;
    for (size_t j = 0; j < p->n; ++j) {
      double pos_r = p->r[j] - 0.0;
      if (pos_r < half_dr) {
        p->r[j] = s->dr - pos_r + 0.0;
        p->vr[j] = -p->vr[j];
      }
    }
    return ST_OK;
  }
  int fixed = s->quirks == ORC_QUIRKS_FIXED;
  for (size_t j = 0; j < p->n; ++j)
    if (reflect_one(s, fixed, &p->r[j], &p->z[j], p->r_old[j], p->z_old[j], &p->vr[j],
                    &p->vz[j]) != ST_OK)
      return ST_FATAL;
  return ST_OK;
}

/* SMB::particles_runaway_collector for one domain (SMB.cpp:232-345):
 * stable removal of particles bound outside [0,nr) x [0,nz). */
static void stage_collect(orc_sim* s, species_t* p) {
  size_t o = 0;
  for (size_t j = 0; j < p->n; ++j) {
    long long cr = p->cell_r[j], cz = p->cell_z[j];
    int gone = cr < 0 || cz < 0 || cr >= s->nr || cz >= s->nz;
    if (gone) {
      ++s->removed;
      continue;
    }
    if (o != j) {
      p->r[o] = p->r[j]; p->phi[o] = p->phi[j]; p->z[o] = p->z[j];
      p->r_old[o] = p->r_old[j]; p->phi_old[o] = p->phi_old[j]; p->z_old[o] = p->z_old[j];
      p->vr[o] = p->vr[j]; p->vphi[o] = p->vphi[j]; p->vz[o] = p->vz[j];
      p->w[o] = p->w[j]; p->sn[o] = p->sn[j];
      p->cell_r[o] = p->cell_r[j]; p->cell_z[o] = p->cell_z[j];
    }
    ++o;
  }
  p->n = o;
}

/* ------------------------------------------------------------------ */
/* Villasenor-Buneman current (currentVB.cpp:22-735)                     */

static inline double ssd_r(double q, double r, double dr, double dz, double dt) {
  return q / (2. * K_PI * r * dr * dz * dt * 2. * dr); /* SOME_SHIT_DENSITY_R */
}
static inline double ssd_z(double q, double r, double dr, double dz, double dt) {
  return q / (2. * K_PI * r * dr * dz * dt * dz); /* SOME_SHIT_DENSITY_Z */
}
static inline double ssd_strict(double q, double r, double dr, double dz, double dt) {
  return q / (K_PI * 4. * r * dz * dz * dr * dt); /* SOME_SHIT_DENSITY_STRICT */
}

static inline double log1p_ratio(double e) { return e == 0.0 ? 1.0 : log1p(e) / e; }

/* The fixed mode's form of simple_current_distribution: the same integrals
 * with k dz = dr and k log((r_o + dr) / r_o) = -(dz / r_o) log1p(e) / e
 * substituted (e = dr / r_o), so that no term divides by dr or dz; the
 * reference's form loses a nearly axial or nearly radial segment's digits
 * and drops every segment with |dr| or |dz| below MNZL (:45-46).  On the
 * axis row the factor 4 r0^2 - dr^2 is exactly 0 and its 1/r_o terms are
 * left out. */
static void vb_simple_fixed(orc_sim* s, double rn, double zn, double ro, double zo, int i_n,
                            int k_n, double q) {
  double *Jr = s->J[0], *Jz = s->J[2];
  double dr = s->dr, dz = s->dz, dt = s->dt, sd, wj, b;
  double delta_r = rn - ro, delta_z = zn - zo;
  if (delta_r == 0.0 && delta_z == 0.0) return;
  double lr = i_n >= 1 ? log1p_ratio(delta_r / ro) : 0.0;
  if (i_n >= 1) {
    double t = dr * dr * ((i_n + 0.5) * (i_n + 0.5) - 0.25) * (delta_z / ro) * lr;
    sd = ssd_r(q, i_n * dr, dr, dz, dt);
    Jz[IDX(s, i_n, k_n)] += sd * (dr * delta_z - delta_r * delta_z / 2. - delta_z * ro + t);
    sd = ssd_r(q, (i_n + 1) * dr, dr, dz, dt);
    Jz[IDX(s, i_n + 1, k_n)] += sd * (delta_r * delta_z / 2. + delta_z * ro + delta_z * dr - t);
  } else {
    sd = q / (2. * K_PI * dr / 4. * dr * dz * dt * dr);
    Jz[IDX(s, i_n, k_n)] += sd * (dr * delta_z - delta_r * delta_z / 2. - delta_z * ro);
    sd = ssd_r(q, dr, dr, dz, dt);
    Jz[IDX(s, i_n + 1, k_n)] += sd * (delta_r * delta_z / 2. + delta_z * dr + delta_z * ro);
  }
  double r0 = (i_n + 0.5) * dr, r1 = ro;
  double p8 = 4 * r0 * r0 - dr * dr;
  sd = ssd_z(q, r0, dr, dz, dt);
  b = (k_n + 1.) * dz - zo;
  wj = -r0 * delta_z - delta_z / 2. * (ro + delta_r / 2.) + 0.5 * (delta_r * b + delta_z * (2 * r0 + r1));
  if (p8 != 0.0)
    wj += (delta_r * b + delta_z * r1) * p8 / (8 * ro * (ro + delta_r)) - delta_z / ro * (p8 / 8.) * lr;
  Jr[IDX(s, i_n, k_n)] += sd * wj;
  b = zo - k_n * dz;
  wj = r0 * delta_z + delta_z / 2. * (ro + delta_r / 2.) + 0.5 * (delta_r * b - delta_z * (2 * r0 + r1));
  if (p8 != 0.0)
    wj += (delta_r * b - delta_z * r1) * p8 / (8 * ro * (ro + delta_r)) + delta_z / ro * (p8 / 8.) * lr;
  Jr[IDX(s, i_n, k_n + 1)] += sd * wj;
}

/* simple_current_distribution :22-173 — a segment inside cell (i_n, k_n). */
static void vb_simple(orc_sim* s, double rn, double zn, double ro, double zo, int i_n, int k_n,
                      double q) {
  double *Jr = s->J[0], *Jz = s->J[2];
  if (s->quirks == ORC_QUIRKS_FIXED) {
    vb_simple_fixed(s, rn, zn, ro, zo, i_n, k_n, q);
    return;
  }
  double dr = s->dr, dz = s->dz, dt = s->dt, wj, k, b, r0, r1, sd;
  double delta_r = rn - ro, delta_z = zn - zo;
  if ((fabs(delta_r) < K_MNZL) || (fabs(delta_z) < K_MNZL)) return;
  if (i_n >= 1) {
    k = delta_r / delta_z;
    b = ro;
    sd = ssd_r(q, i_n * dr, dr, dz, dt);
    wj = sd * (dr * delta_z - k * delta_z * delta_z / 2. - delta_z * b +
               dr * dr / k * ((i_n + 0.5) * (i_n + 0.5) - 0.25) * log((k * delta_z + b) / b));
    Jz[IDX(s, i_n, k_n)] += wj;
    sd = ssd_r(q, (i_n + 1) * dr, dr, dz, dt);
    wj = sd * (k * delta_z * delta_z / 2. + delta_z * b + delta_z * dr +
               dr * dr / k * (0.25 - (i_n + 0.5) * (i_n + 0.5)) * log((k * delta_z + b) / b));
    Jz[IDX(s, i_n + 1, k_n)] += wj;
  } else {
    k = delta_r / delta_z;
    b = ro;
    sd = q / (2. * K_PI * dr / 4. * dr * dz * dt * dr);
    wj = sd * (dr * delta_z - k * delta_z * delta_z / 2. - delta_z * b);
    Jz[IDX(s, i_n, k_n)] += wj;
    sd = ssd_r(q, dr, dr, dz, dt);
    wj = sd * (k * delta_z * delta_z / 2. + delta_z * dr + delta_z * b);
    Jz[IDX(s, i_n + 1, k_n)] += wj;
  }
  /* J_r, identical in both branches :78-108 and :135-171 */
  k = -delta_z / delta_r;
  r0 = (i_n + 0.5) * dr;
  r1 = ro;
  b = (k_n + 1.) * dz - zo;
  sd = ssd_z(q, r0, dr, dz, dt);
  wj = sd * (r0 * k * delta_r + k / 2. * delta_r * (ro + delta_r / 2.) +
             0.5 * delta_r * (b - k * (2 * r0 + r1)) +
             delta_r * (b - k * r1) * (4 * r0 * r0 - dr * dr) / (8 * ro * (ro + delta_r)) +
             (k * (r0 * r0 / 2. - dr * dr / 8.)) * log((ro + delta_r) / ro));
  Jr[IDX(s, i_n, k_n)] += wj;
  b = zo - k_n * dz;
  wj = sd * (-r0 * k * delta_r - k / 2. * delta_r * (ro + delta_r / 2.) +
             0.5 * delta_r * (b + k * (2 * r0 + r1)) +
             delta_r * (b + k * r1) * (4 * r0 * r0 - dr * dr) / (8 * ro * (ro + delta_r)) -
             (k * (r0 * r0 / 2. - dr * dr / 8.)) * log((ro + delta_r) / ro));
  Jr[IDX(s, i_n, k_n + 1)] += wj;
}

/* strict_motion_distribution :500-729 — purely axial or radial motion. */
static void vb_strict(orc_sim* s, double rn, double zn, double ro, double zo, double q) {
  double *Jr = s->J[0], *Jz = s->J[2];
  double dr = s->dr, dz = s->dz, dt = s->dt;
  int fixed = s->quirks == ORC_QUIRKS_FIXED;
  int i_n = CELL_NUMBER(rn, dr), k_n = CELL_NUMBER(zn, dz);
  int i_o = CELL_NUMBER(ro, dr), k_o = CELL_NUMBER(zo, dz);
  if ((fabs(rn - ro) < K_MNZL) && (fabs(zn - zo) < K_MNZL)) return;
  if (fabs(rn - ro) < K_MNZL) { /* axial :524-604 */
    double delta_z = 0., wj, lo, up;
    double value_part = 2. * K_PI * rn * dr * dz;
    double r1 = rn - 0.5 * dr, r2 = (i_n + 0.5) * dr, r3 = rn + 0.5 * dr;
    if (i_n == 0)
      lo = q / (dt * K_PI * dr * dr / 4.) * K_PI * (r2 * r2 - r1 * r1) / value_part;
    else
      lo = q / (dt * 2. * K_PI * i_n * dr * dr) * K_PI * (r2 * r2 - r1 * r1) / value_part;
    up = q / (dt * 2 * K_PI * (i_n + 1) * dr * dr) * K_PI * (r3 * r3 - r2 * r2) / value_part;
    if (!fixed) { /* :545-546 overwrite J_r at two nodes */
      Jr[IDX(s, i_n, k_n)] = 0.;
      Jr[IDX(s, i_n, k_n + 1)] = 0.;
    }
    switch (k_n - k_o) {
      case 0:
        delta_z = zn - zo;
        wj = lo * delta_z; Jz[IDX(s, i_n, k_n)] += wj;
        wj = up * delta_z; Jz[IDX(s, i_n + 1, k_n)] += wj;
        break;
      case 1:
        delta_z = k_n * dz - zo;
        wj = lo * delta_z; Jz[IDX(s, i_n, k_n - 1)] += wj;
        wj = up * delta_z; Jz[IDX(s, i_n + 1, k_n - 1)] += wj;
        delta_z = zn - k_n * dz;
        wj = lo * delta_z; Jz[IDX(s, i_n, k_n)] += wj;
        wj = up * delta_z; Jz[IDX(s, i_n + 1, k_n)] += wj;
        break;
      case -1:
        delta_z = (k_n + 1) * dz - zo;
        wj = lo * delta_z; Jz[IDX(s, i_n, k_n + 1)] += wj;
        wj = up * delta_z; Jz[IDX(s, i_n + 1, k_n + 1)] += wj;
        delta_z = zn - (k_n + 1) * dz;
        wj = lo * delta_z; Jz[IDX(s, i_n, k_n)] += wj;
        wj = up * delta_z; Jz[IDX(s, i_n + 1, k_n)] += wj;
        break;
      default: break;
    }
  } else if (fabs(zn - zo) < K_MNZL) { /* radial :607-728 */
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
        Jr[IDX(s, i_n, k_n)] += wj * ldz;
        Jr[IDX(s, i_n, k_n + 1)] += wj * rdz;
        break;
      case 1:
        delta_r = (i_n) * dr - ro;
        ldz = (k_n + 1) * dz - zn;
        rdz = zn - k_n * dz;
        r0 = (i_n - 0.5) * dr;
        sd = ssd_strict(q, r0, dr, dz, dt);
        wj = sd * (delta_r - r0 * r0 / (ro + delta_r) + r0 * r0 / ro +
                   dr * dr / (4. * (ro + delta_r)) - dr * dr / (4. * ro));
        Jr[IDX(s, i_n - 1, k_n)] += wj * ldz;
        Jr[IDX(s, i_n - 1, k_n + 1)] += wj * rdz;
        delta_r = rn - i_n * dr;
        r0 = (i_n + 0.5) * dr;
        sd = ssd_strict(q, r0, dr, dz, dt);
        if (fixed) /* (r0*r0)/(i_n*dr), where the reference has r0*r0/i_n*dr (:673) */
          wj = sd * (delta_r - r0 * r0 / (i_n * dr + delta_r) + r0 * r0 / (i_n * dr) +
                     dr * dr / (4. * (i_n * dr + delta_r)) - dr * dr / (4. * i_n * dr));
        else
          wj = sd * (delta_r - r0 * r0 / (i_n * dr + delta_r) + r0 * r0 / i_n * dr +
                     dr * dr / (4. * (i_n * dr + delta_r)) - dr * dr / (4. * i_n * dr));
        Jr[IDX(s, i_n, k_n)] += wj * ldz;
        Jr[IDX(s, i_n, k_n + 1)] += wj * rdz;
        break;
      case -1:
        delta_r = (i_n + 1) * dr - ro;
        ldz = (k_n + 1) * dz - zn;
        rdz = zn - k_n * dz;
        r0 = (i_n + 1.5) * dr;
        sd = ssd_strict(q, r0, dr, dz, dt);
        wj = sd * (delta_r - r0 * r0 / (ro + delta_r) + r0 * r0 / ro +
                   dr * dr / (4. * (ro + delta_r)) - dr * dr / (4. * ro));
        Jr[IDX(s, i_n + 1, k_n)] += wj * ldz;
        Jr[IDX(s, i_n + 1, k_n + 1)] += wj * rdz;
        delta_r = rn - (i_n + 1) * dr;
        r0 = (i_n + 0.5) * dr;
        sd = ssd_strict(q, r0, dr, dz, dt);
        if (fixed)
          wj = sd * (delta_r - r0 * r0 / ((i_n + 1) * dr + delta_r) + r0 * r0 / ((i_n + 1) * dr) +
                     dr * dr / (4. * ((i_n + 1) * dr + delta_r)) - dr * dr / (4. * (i_n + 1) * dr));
        else
          wj = sd * (delta_r - r0 * r0 / ((i_n + 1) * dr + delta_r) + r0 * r0 / (i_n + 1) * dr +
                     dr * dr / (4. * ((i_n + 1) * dr + delta_r)) - dr * dr / (4. * (i_n + 1) * dr));
        Jr[IDX(s, i_n, k_n)] += wj * ldz;
        Jr[IDX(s, i_n, k_n + 1)] += wj * rdz;
        break;
      default: break;
    }
  }
}

/* azimuthal_current_distribution :398-498 for one particle. */
static void vb_azimuthal_one(orc_sim* s, double q, double r, double z, double ro, double zo,
                             double vphi, int r_i, int z_k) {
  double *Jp = s->J[1];
  double dr = s->dr, dz = s->dz;
  double v_1 = cell_volume_expr(2.0 * r_i + 1, dr, dz);
  double v_2 = cell_volume_expr(2.0 * r_i + 1 + 1, dr, dz);
  double pos_r = (r + ro) / 2;
  double pos_z = (z + zo) / 2;
  /* both branches of :418-496 evaluate the same expressions */
  double r1 = pos_r - 0.5 * dr, r2 = (r_i + 0.5) * dr, r3 = pos_r + 0.5 * dr;
  double ro_v = q / (2. * K_PI * dz * dr * pos_r);
  double dz1 = (z_k + 0.5) * dz - (pos_z - 0.5 * dz);
  double dz2 = (pos_z + 0.5 * dz) - (z_k + 0.5) * dz;
  double rho, wj;
  rho = ro_v * K_PI * dz1 * (r2 * r2 - r1 * r1) / v_1; wj = rho * vphi; Jp[IDX(s, r_i, z_k)] += wj;
  rho = ro_v * K_PI * dz1 * (r3 * r3 - r2 * r2) / v_2; wj = rho * vphi; Jp[IDX(s, r_i + 1, z_k)] += wj;
  rho = ro_v * K_PI * dz2 * (r2 * r2 - r1 * r1) / v_1; wj = rho * vphi; Jp[IDX(s, r_i, z_k + 1)] += wj;
  rho = ro_v * K_PI * dz2 * (r3 * r3 - r2 * r2) / v_2; wj = rho * vphi; Jp[IDX(s, r_i + 1, z_k + 1)] += wj;
}

/* rz_current_distribution :175-396 for one particle. */
static void vb_rz_one(orc_sim* s, double q, double R, double Z, double RO, double ZO,
                      long long cell_r, long long cell_z) {
  double dr = s->dr, dz = s->dz;
  int fixed = s->quirks == ORC_QUIRKS_FIXED;
  int i_n = (int)cell_r, k_n = (int)cell_z;
  int i_o = CELL_NUMBER(RO, dr), k_o = CELL_NUMBER(ZO, dz);
  if (RO == (i_o + 1) * dr) i_o = i_n;
  if (ZO == (k_o + 1) * dz) k_o = k_n;
  if (R == (i_n + 1) * dr) i_n = i_o;
  if (Z == (k_n + 1) * dz) k_n = k_o;
  int res_cell = abs(i_n - i_o) + abs(k_n - k_o);
  int too_far = fixed ? (abs(i_n - i_o) > 1 || abs(k_n - k_o) > 1) : (abs(i_n - i_o) > 1);
  if (too_far) {
    ++s->errors; /* LOG_S(ERROR) :199-204 */
    return;
  }
  if ((fabs(R - RO) < K_MNZL) || (fabs(Z - ZO) < K_MNZL)) {
    vb_strict(s, R, Z, RO, ZO, q);
    return;
  }
  if (res_cell == 0) {
    vb_simple(s, R, Z, RO, ZO, i_n, k_n, q);
  } else if (res_cell == 1) {
    if ((i_n != i_o) && (k_n == k_o)) {
      if (RO > (i_n + 1) * dr) {
        double a = (RO - R) / (ZO - Z);
        double r_b = (i_n + 1) * dr;
        double delta_r = r_b - R;
        double z_b = Z + delta_r / a;
        vb_simple(s, r_b, z_b, RO, ZO, i_n + 1, k_n, q);
        vb_simple(s, R, Z, r_b, z_b, i_n, k_n, q);
      } else {
        double a = (R - RO) / (Z - ZO);
        double r_b = (i_n) * dr;
        double delta_r = r_b - RO;
        double z_b = ZO + delta_r / a;
        vb_simple(s, r_b, z_b, RO, ZO, i_n - 1, k_n, q);
        vb_simple(s, R, Z, r_b, z_b, i_n, k_n, q);
      }
    } else if ((i_n == i_o) && (k_n != k_o)) {
      if (ZO < k_n * dz) {
        double z_b = k_n * dz;
        double delta_z = z_b - ZO;
        double a = (R - RO) / (Z - ZO);
        double r_b = RO + a * delta_z;
        vb_simple(s, r_b, z_b, RO, ZO, i_n, k_n - 1, q);
        vb_simple(s, R, Z, r_b, z_b, i_n, k_n, q);
      } else {
        double z_b = (k_n + 1) * dz;
        double delta_z = z_b - Z;
        double a = (RO - R) / (ZO - Z);
        double r_b = R + a * delta_z;
        vb_simple(s, r_b, z_b, RO, ZO, i_n, k_n + 1, q);
        vb_simple(s, R, Z, r_b, z_b, i_n, k_n, q);
      }
    }
  } else if (res_cell == 2) {
    if (i_o < i_n) {
      if (k_o < k_n) {
        double a = (R - RO) / (Z - ZO);
        double r1 = i_n * dr;
        double delta_z1 = (r1 - RO) / a;
        double z1 = ZO + delta_z1;
        double z2 = k_n * dz;
        double delta_r2 = (z2 - ZO) * a;
        double r2 = RO + delta_r2;
        if (z1 < k_n * dz) {
          vb_simple(s, r1, z1, RO, ZO, i_n - 1, k_n - 1, q);
          vb_simple(s, r2, z2, r1, z1, i_n, k_n - 1, q);
          vb_simple(s, R, Z, r2, z2, i_n, k_n, q);
        } else if (z1 > k_n * dz) {
          vb_simple(s, r2, z2, RO, ZO, i_n - 1, k_n - 1, q);
          vb_simple(s, r1, z1, r2, z2, i_n - 1, k_n, q);
          vb_simple(s, R, Z, r1, z1, i_n, k_n, q);
        }
      } else {
        double a = (R - RO) / (Z - ZO);
        double r1 = i_n * dr;
        double delta_z1 = (r1 - RO) / a;
        double z1 = ZO + delta_z1;
        double z2 = (k_n + 1) * dz;
        double delta_r2 = -(ZO - z2) * a;
        double r2 = RO + delta_r2;
        if (z1 > (k_n + 1) * dz) {
          vb_simple(s, r1, z1, RO, ZO, i_n - 1, k_n + 1, q);
          vb_simple(s, r2, z2, r1, z1, i_n, k_n + 1, q);
          vb_simple(s, R, Z, r2, z2, i_n, k_n, q);
        } else if (z1 < (k_n + 1) * dz) {
          vb_simple(s, r2, z2, RO, ZO, i_n - 1, k_n + 1, q);
          vb_simple(s, r1, z1, r2, z2, i_n - 1, k_n, q);
          vb_simple(s, R, Z, r1, z1, i_n, k_n, q);
        }
      }
    } else if (i_o > i_n) {
      if (k_o < k_n) {
        double a = (R - RO) / (Z - ZO);
        double r1 = (i_n + 1) * dr;
        double delta_z1 = -(RO - r1) / a;
        double z1 = ZO + delta_z1;
        double z2 = k_n * dz;
        double delta_r2 = -(z2 - ZO) * a;
        double r2 = RO - delta_r2;
        if (z1 < (k_n) * dz) {
          vb_simple(s, r1, z1, RO, ZO, i_n + 1, k_n - 1, q);
          vb_simple(s, r2, z2, r1, z1, i_n, k_n - 1, q);
          vb_simple(s, R, Z, r2, z2, i_n, k_n, q);
        } else if (z1 > (k_n) * dz) {
          vb_simple(s, r2, z2, RO, ZO, i_n + 1, k_n - 1, q);
          vb_simple(s, r1, z1, r2, z2, i_n + 1, k_n, q);
          vb_simple(s, R, Z, r1, z1, i_n, k_n, q);
        }
      } else if (k_o > k_n) {
        double a = (RO - R) / (ZO - Z);
        double r1 = (i_n + 1) * dr;
        double delta_z1 = (r1 - R) / a;
        double z1 = Z + delta_z1;
        double z2 = (k_n + 1) * dz;
        double delta_r2 = (z2 - Z) * a;
        double r2 = R + delta_r2;
        if (z1 > (k_n + 1) * dz) {
          vb_simple(s, r1, z1, RO, ZO, i_n + 1, k_n + 1, q);
          vb_simple(s, r2, z2, r1, z1, i_n, k_n + 1, q);
          vb_simple(s, R, Z, r2, z2, i_n, k_n, q);
        } else if (z1 < (k_n + 1) * dz) {
          vb_simple(s, r2, z2, RO, ZO, i_n + 1, k_n + 1, q);
          vb_simple(s, r1, z1, r2, z2, i_n + 1, k_n, q);
          vb_simple(s, R, Z, r1, z1, i_n, k_n, q);
        }
      }
    }
  }
}

static void current_vb(orc_sim* s) { /* current_distribution :731-735 */
  for (int c = 0; c < 3; ++c) halo_set(s, s->J[c], 0.0);
  for (int t = 0; t < s->nsp; ++t) {
    species_t* p = &s->sp[t];
    for (size_t j = 0; j < p->n; ++j)
      vb_azimuthal_one(s, p->charge * p->w[j], p->r[j], p->z[j], p->r_old[j], p->z_old[j],
                       p->vphi[j], (int)p->cell_r[j], (int)p->cell_z[j]);
  }
  for (int c = 0; c < 3; ++c) halo_set(s, s->J[c], 0.0);
  for (int t = 0; t < s->nsp; ++t) {
    species_t* p = &s->sp[t];
    for (size_t j = 0; j < p->n; ++j)
      vb_rz_one(s, p->charge * p->w[j], p->r[j], p->z[j], p->r_old[j], p->z_old[j],
                p->cell_r[j], p->cell_z[j]);
  }
}

/* ------------------------------------------------------------------ */
/* ZigZag current (currentZigZag.cpp:22-136, RELAY_POINT currentZigZag.hpp:28-30) */

static inline double dmin(double a, double b) { return (b < a) ? b : a; } /* std::min */
static inline double dmax(double a, double b) { return (a < b) ? b : a; } /* std::max */
static inline double relay(int i1, int i2, double x1, double x2, double dx) {
  return dmin(dmin(i1 * dx, i2 * dx) + dx, dmax(dmax(i1 * dx, i2 * dx), (x1 + x2) / 2.));
}

static void current_zigzag(orc_sim* s) {
  for (int c = 0; c < 3; ++c) halo_set(s, s->J[c], 0.0);
  double *Jr = s->J[0], *Jp = s->J[1], *Jz = s->J[2];
  double dr = s->dr, dz = s->dz, dt = s->dt;
  for (int t = 0; t < s->nsp; ++t) {
    species_t* p = &s->sp[t];
    for (size_t j = 0; j < p->n; ++j) {
      double ro = p->r_old[j], zo = p->z_old[j], rn = p->r[j], zn = p->z[j];
      double cod = p->charge * p->w[j] / dt;
      int i_n = CELL_NUMBER(rn, dr), i_o = CELL_NUMBER(ro, dr);
      int k_n = CELL_NUMBER(zn, dz), k_o = CELL_NUMBER(zo, dz);
      int i_mid = CELL_NUMBER((rn + ro) / 2., dr);
      double oov = 1 / (cell_volume_expr(2.0 * i_mid + 1, dr, dz));
      double F_phi = p->charge * p->w[j] * p->vphi[j];
      double W_phi = p->vphi[j] * dt / (2. * K_PI * (ro + rn));
      double rr = relay(i_o, i_n, ro, rn, dr), zr = relay(k_o, k_n, zo, zn, dz);
      double F_r1 = cod * (rr - ro), F_r2 = cod * (rn - rr);
      double F_z1 = cod * (zr - zo), F_z2 = cod * (zn - zr);
      double W_r1 = (ro + rr) / 2 - i_o * dr, W_r2 = (rn + rr) / 2 - i_n * dr;
      double W_z1 = (zo + zr) / 2 - k_o * dz, W_z2 = (zn + zr) / 2 - k_n * dz;
      double mWr1 = 1 - W_r1, mWr2 = 1 - W_r2, mWz1 = 1 - W_z1, mWz2 = 1 - W_z2, mWp = 1 - W_phi;
      double Jr_a = oov * F_r1 * mWp * mWz1, Jr_b = oov * F_r2 * mWp * mWz2;
      double Jr_c = oov * F_r1 * W_phi * mWz1, Jr_d = oov * F_r2 * W_phi * mWz2;
      double Jr_e = oov * F_r1 * mWp * W_z1, Jr_f = oov * F_r2 * mWp * W_z2;
      double Jr_g = oov * F_r1 * W_phi * W_z1, Jr_h = oov * F_r2 * W_phi * W_z2;
      double Jp_a = oov * F_phi * mWr2 * mWz2, Jp_b = oov * F_phi * mWr2 * W_z1;
      double Jp_c = oov * F_phi * W_r2 * mWz2, Jp_d = oov * F_phi * W_r2 * W_z2;
      double Jz_a = oov * F_z1 * mWr1 * mWp, Jz_b = oov * F_z2 * mWr2 * mWp;
      double Jz_c = oov * F_z1 * mWr1 * W_phi, Jz_d = oov * F_z2 * mWr2 * W_phi;
      double Jz_e = oov * F_z1 * W_r1 * mWp, Jz_f = oov * F_z2 * W_r2 * mWp;
      double Jz_g = oov * F_z1 * W_r1 * W_phi, Jz_h = oov * F_z2 * W_r2 * W_phi;
      Jr[IDX(s, i_o, k_o)] += Jr_a + Jr_c;
      Jr[IDX(s, i_o, k_o + 1)] += Jr_e + Jr_g;
      Jr[IDX(s, i_n, k_n)] += Jr_b + Jr_d;
      Jr[IDX(s, i_n, k_n + 1)] += Jr_f + Jr_h;
      Jp[IDX(s, i_n, k_n)] += Jp_a;
      Jp[IDX(s, i_n, k_n + 1)] += Jp_b;
      Jp[IDX(s, i_n + 1, k_n)] += Jp_c;
      Jp[IDX(s, i_n + 1, k_n + 1)] += Jp_d;
      Jz[IDX(s, i_o, k_o)] += Jz_a + Jz_c;
      Jz[IDX(s, i_o + 1, k_o)] += Jz_e + Jz_g;
      Jz[IDX(s, i_n, k_n)] += Jz_b + Jz_d;
      Jz[IDX(s, i_n + 1, k_n)] += Jz_f + Jz_h;
    }
  }
}

/* ------------------------------------------------------------------ */
/* Beam injection: BeamP::inject (beamP.cpp:71-157)                      */

static int grow(species_t* p, size_t need) {
  if (need <= p->cap) return ST_OK;
  size_t cap = p->cap ? p->cap : 64;
  while (cap < need) cap *= 2;
  double** arrs[] = {&p->r, &p->phi, &p->z, &p->r_old, &p->phi_old, &p->z_old,
                     &p->vr, &p->vphi, &p->vz, &p->w, &p->sn};
  for (size_t a = 0; a < sizeof(arrs) / sizeof(arrs[0]); ++a) {
    double* q = (double*)realloc(*arrs[a], cap * sizeof(double));
    if (!q) return ST_ARG;
    memset(q + p->cap, 0, (cap - p->cap) * sizeof(double));
    *arrs[a] = q;
  }
  long long* cr = (long long*)realloc(p->cell_r, cap * sizeof(long long));
  if (!cr) return ST_ARG;
  p->cell_r = cr;
  long long* cz = (long long*)realloc(p->cell_z, cap * sizeof(long long));
  if (!cz) return ST_ARG;
  p->cell_z = cz;
  p->cap = cap;
  return ST_OK;
}

static double draw(orc_sim* s, int slot, uint32_t idx, int which) {
  if (s->rng_kind == ORC_RNG_PHILOX)
    return orc_philox_uniform(s->seed, 0x6265616du + (uint32_t)slot, s->step_index, idx, which);
  return mt_uniform(&s->mt);
}

static int stage_inject(orc_sim* s, int slot) {
  species_t* p = &s->sp[slot];
  if (!p->is_beam) return ST_OK; /* SpecieP::inject is empty (specieP.cpp:480) */
  double t = s->t;
  if (p->current_bunch < p->bunches_amount) {
    double bunch_start = p->start_time + (p->bunch_length + p->bunches_distance) / p->velocity * p->current_bunch;
    double bunch_finish = bunch_start + p->bunch_length / p->velocity;
    if (0.0 * s->dr < p->radius && t >= bunch_start && t < bunch_finish) {
      double dr = s->dr, dz = s->dz;
      double dl = p->velocity * s->dt;
      double half_z = dz / 2.;
      double v_macro_avg = K_PI * p->radius * dr * dz;
      double N_total = K_PI * p->radius * p->radius * p->bunch_length * p->bunches_amount * p->density;
      double n_per_macro_avg = N_total / p->macro_amount;
      for (unsigned i = 0; i < p->macro_per_step; ++i) {
        double rand_r = draw(s, slot, i, 0);
        double rand_z = draw(s, slot, i, 1);
        double pos_r = p->domain_radius * rand_r + dr / 2 + 0.0 * dr;
        if (grow(p, p->n + 1) != ST_OK) return ST_ARG;
        size_t j = p->n++;
        p->r[j] = pos_r; p->phi[j] = 0; p->z[j] = dl * rand_z + half_z;
        p->vr[j] = 0; p->vphi[j] = 0; p->vz[j] = p->velocity;
        p->r_old[j] = p->phi_old[j] = p->z_old[j] = 0; p->sn[j] = 0;
        double norm;
        if (pos_r > dr / 2)
          norm = 2 * K_PI * pos_r * dr * dz / v_macro_avg;
        else
          norm = K_PI * (pos_r * pos_r + pos_r * dr + dr * dr / 4.) * dz / v_macro_avg;
        p->w[j] = n_per_macro_avg * norm;
        p->cell_r[j] = CELL_NUMBER(p->r[j], dr);
        p->cell_z[j] = CELL_NUMBER(p->r[j], dz); /* :137 binds z from pos_r */
      }
    }
    if (t > bunch_finish) ++p->current_bunch;
  }
  return ST_OK;
}

/* ------------------------------------------------------------------ */
/* API                                                                   */

orc_sim* orc_create(int nr, int nz, double radius, double longitude, double dt, double t_start,
                    const int* pml_size, const double* pml_sigma, int pusher, int current,
                    int quirks) {
  if (nr < 2 || nz < 2) return NULL;
  orc_sim* s = (orc_sim*)calloc(1, sizeof(orc_sim));
  s->nr = nr; s->nz = nz; s->ld = nz + 4;
  s->R = radius; s->L = longitude;
  s->dr = radius / nr; s->dz = longitude / nz; /* Geometry ctor geometry.hpp:67-68 */
  s->gcr = (size_t)(radius / s->dr);          /* geometry.hpp:70-71 */
  s->gcz = (size_t)(longitude / s->dz);
  s->dt = dt; s->t = t_start;
  for (int i = 0; i < 4; ++i) s->pml[i] = pml_size ? pml_size[i] : 0;
  s->pml_sigma[0] = pml_sigma ? pml_sigma[0] : 0; s->pml_sigma[1] = pml_sigma ? pml_sigma[1] : 0;
  s->pusher = pusher; s->current = current; s->quirks = quirks;
  size_t ng = (size_t)(nr + 4) * (size_t)(nz + 4);
  for (int c = 0; c < 3; ++c) {
    s->E[c] = (double*)calloc(ng, sizeof(double));
    s->H[c] = (double*)calloc(ng, sizeof(double));
    s->Hat[c] = (double*)calloc(ng, sizeof(double));
    s->J[c] = (double*)calloc(ng, sizeof(double));
  }
  s->sigma = (double*)calloc(ng, sizeof(double));
  set_pml(s);
  mt_seed(&s->mt, 5489u);
  s->rng_kind = ORC_RNG_MT19937;
  return s;
}

static int add_common(orc_sim* s, int id, const char* name, double charge_e, double mass_e) {
  if (s->nsp >= MAX_SPECIES) return ST_ARG;
  species_t* p = &s->sp[s->nsp];
  memset(p, 0, sizeof(*p));
  p->id = id;
  strncpy(p->name, name ? name : "", sizeof(p->name) - 1);
  p->charge = charge_e * K_EL_CHARGE;
  p->mass = mass_e * K_EL_MASS;
  return s->nsp++;
}

int orc_add_species(orc_sim* s, int id, const char* name, double charge_e, double mass_e) {
  return add_common(s, id, name, charge_e, mass_e);
}

int orc_add_beam(orc_sim* s, int id, const char* name, double charge_e, double mass_e,
                 unsigned macro_amount, double start_time, double b_radius, double density,
                 double amount, double length, double distance, double velocity) {
  int slot = add_common(s, id, name, charge_e, mass_e);
  if (slot < 0) return slot;
  species_t* p = &s->sp[slot];
  p->is_beam = 1;
  p->macro_amount = macro_amount; /* BeamP ctor beamP.cpp:22-69 */
  p->radius = b_radius; p->density = density; p->velocity = velocity;
  p->start_time = start_time; p->bunches_amount = (unsigned)amount;
  p->bunch_length = length; p->bunches_distance = distance;
  p->finish_time = p->start_time + p->bunch_length / p->velocity * p->bunches_amount +
                   p->bunches_distance / p->velocity * (p->bunches_amount - 1);
  if (b_radius > (double)s->nr * s->dr) p->domain_radius = s->R;
  else if (b_radius > 0.0 * s->dr) p->domain_radius = b_radius - 0.0 * s->dr;
  else p->domain_radius = 0;
  double macro_normalizer = p->domain_radius / p->radius;
  p->bunch_macro_amount = (double)(p->macro_amount / p->bunches_amount) * macro_normalizer;
  p->macro_per_step = p->bunch_macro_amount * p->velocity * s->dt / p->bunch_length;
  return slot;
}

void orc_set_rng(orc_sim* s, int kind, uint64_t seed) {
  s->rng_kind = kind;
  s->seed = seed;
  if (kind == ORC_RNG_MT19937) mt_seed(&s->mt, (uint32_t)seed);
}

int orc_set_particles(orc_sim* s, int sid, size_t n, const double* r, const double* z,
                      const double* vr, const double* vphi, const double* vz, const double* w) {
  if (sid < 0 || sid >= s->nsp) return ST_ARG;
  species_t* p = &s->sp[sid];
  if (grow(p, n) != ST_OK) return ST_ARG;
  p->n = n;
  for (size_t j = 0; j < n; ++j) {
    p->r[j] = r[j]; p->z[j] = z[j]; p->phi[j] = 0;
    p->vr[j] = vr[j]; p->vphi[j] = vphi[j]; p->vz[j] = vz[j]; p->w[j] = w[j];
    p->r_old[j] = p->phi_old[j] = p->z_old[j] = 0; p->sn[j] = 0;
    p->cell_r[j] = CELL_NUMBER(r[j], s->dr);
    p->cell_z[j] = CELL_NUMBER(z[j], s->dz);
  }
  return ST_OK;
}

long orc_count(orc_sim* s, int sid) {
  if (sid < 0 || sid >= s->nsp) return -1;
  return (long)s->sp[sid].n;
}

int orc_get_particles(orc_sim* s, int sid, size_t cap, double* r, double* z, double* vr,
                      double* vphi, double* vz, double* w, double* r_old, double* z_old,
                      long long* cell_r, long long* cell_z) {
  if (sid < 0 || sid >= s->nsp) return ST_ARG;
  species_t* p = &s->sp[sid];
  if (cap < p->n) return -4;
  for (size_t j = 0; j < p->n; ++j) {
    r[j] = p->r[j]; z[j] = p->z[j]; vr[j] = p->vr[j]; vphi[j] = p->vphi[j]; vz[j] = p->vz[j];
    w[j] = p->w[j];
    if (r_old) r_old[j] = p->r_old[j];
    if (z_old) z_old[j] = p->z_old[j];
    if (cell_r) cell_r[j] = p->cell_r[j];
    if (cell_z) cell_z[j] = p->cell_z[j];
  }
  return ST_OK;
}

static double* field_ptr(orc_sim* s, int which) {
  if (which >= 0 && which < 3) return s->E[which];
  if (which >= 3 && which < 6) return s->H[which - 3];
  if (which >= 6 && which < 9) return s->Hat[which - 6];
  if (which >= 9 && which < 12) return s->J[which - 9];
  if (which == 12) return s->sigma;
  return NULL;
}

int orc_set_field(orc_sim* s, int which, const double* src) {
  double* a = field_ptr(s, which);
  if (!a || which == 12) return ST_ARG;
  memcpy(a, src, sizeof(double) * (size_t)(s->nr + 4) * (size_t)(s->nz + 4));
  return ST_OK;
}

int orc_get_field(orc_sim* s, int which, double* dst) {
  double* a = field_ptr(s, which);
  if (!a) return ST_ARG;
  memcpy(dst, a, sizeof(double) * (size_t)(s->nr + 4) * (size_t)(s->nz + 4));
  return ST_OK;
}

int orc_stage(orc_sim* s, int stage) {
  int st = ST_OK;
  switch (stage) {
    case ORC_STAGE_INJECT:
      for (int t = 0; t < s->nsp && st == ST_OK; ++t) st = stage_inject(s, t);
      return st;
    case ORC_STAGE_FIELD_E: return field_e(s);
    case ORC_STAGE_FIELD_H: return field_h(s);
    case ORC_STAGE_PUSH:
      for (int t = 0; t < s->nsp; ++t) {
        species_t* p = &s->sp[t];
        for (size_t j = 0; j < p->n; ++j) {
          double pr = p->r[j], pz = p->z[j], e[3], b[3];
          double v[3] = {p->vr[j], p->vphi[j], p->vz[j]};
          if (isnan(pr) || isinf(pr) || isnan(pz) || isinf(pz)) return ST_FATAL; /* :51-57 */
          gather_e(s, s->E, pr, pz, e);
          gather_h(s, s->H, pr, pz, b);
          if (s->Eext[0]) { /* e += external_fields->get_field_e(pos_r, pos_z), pusherBoris.cpp:62-65 */
            double ex[3], bx[3];
            gather_e(s, s->Eext, pr, pz, ex);
            gather_h(s, s->Hext, pr, pz, bx);
            for (int c = 0; c < 3; ++c) {
              e[c] += ex[c];
              b[c] += bx[c];
            }
          }
          int fixed = s->quirks == ORC_QUIRKS_FIXED;
          if (s->pusher == ORC_PUSHER_VAY) st = push_vay(fixed, p->charge, p->mass, s->dt, e, b, v);
          else if (s->pusher == ORC_PUSHER_HC) st = push_hc(fixed, p->charge, p->mass, s->dt, e, b, v);
          else st = push_boris(s->pusher, p->charge, p->mass, s->dt, e, b, v);
          if (st != ST_OK) return st;
          p->vr[j] = v[0]; p->vphi[j] = v[1]; p->vz[j] = v[2];
        }
      }
      return ST_OK;
    case ORC_STAGE_DUMP_OLD:
      for (int t = 0; t < s->nsp; ++t) stage_dump_old(&s->sp[t]);
      return ST_OK;
    case ORC_STAGE_MOVE:
      for (int t = 0; t < s->nsp; ++t) stage_move(&s->sp[t], s->dt);
      return ST_OK;
    case ORC_STAGE_POS_RZ:
      for (int t = 0; t < s->nsp; ++t) stage_pos_rz(&s->sp[t]);
      return ST_OK;
    case ORC_STAGE_REFLECT:
      for (int t = 0; t < s->nsp && st == ST_OK; ++t) st = stage_reflect(s, &s->sp[t]);
      return st;
    case ORC_STAGE_VEL_RZ:
      for (int t = 0; t < s->nsp; ++t) stage_vel_rz(&s->sp[t]);
      return ST_OK;
    case ORC_STAGE_BIND:
      for (int t = 0; t < s->nsp; ++t) stage_bind(&s->sp[t], s->dr, s->dz);
      return ST_OK;
    case ORC_STAGE_COLLECT:
      for (int t = 0; t < s->nsp; ++t) stage_collect(s, &s->sp[t]);
      return ST_OK;
    case ORC_STAGE_RESET_CURRENT: { /* Domain::reset_current domain.cpp:135-139 */
      size_t ng = (size_t)(s->nr + 4) * (size_t)(s->nz + 4);
      for (int c = 0; c < 3; ++c) memset(s->J[c], 0, ng * sizeof(double));
      return ST_OK;
    }
    case ORC_STAGE_CURRENT:
      if (s->current == ORC_CURRENT_ZIGZAG) current_zigzag(s);
      else current_vb(s);
      return ST_OK;
    case ORC_STAGE_ADVANCE_TIME:
      s->t += s->dt;
      s->step_index += 1;
      return ST_OK;
    default: return ST_ARG;
  }
}

int orc_step(orc_sim* s, int nsteps) {
  for (int n = 0; n < nsteps; ++n)
    for (int st = 0; st < ORC_STAGE_COUNT; ++st) {
      int rc = orc_stage(s, st);
      if (rc != ST_OK) return rc;
    }
  return ST_OK;
}

double orc_time(orc_sim* s) { return s->t; }
long orc_removed(orc_sim* s) { return s->removed; }
long orc_error_count(orc_sim* s) { return s->errors; }

/* ExternalFields (externalFields.cpp): the profile named by each formfactor
 * (:51-79), applied after every H update (operator(), :351-436; SMB.cpp:
 * 1253-1262) and constant, so set here once.  The reference's electric name
 * test maps every name but "none" to code 0 and "none" to 1 (const_r), and
 * neither sets a field; of the magnetic codes only 3 (const_z) sets one,
 * set_magn_field_homogenous_z (:298-348): H_z = params[0] on the cells
 * r_begin <= i < r_end, z_begin <= k < z_end, which for one domain with its
 * four walls are 1 <= i < nr-1, 1 <= k < nz-1 (:29-47), zero elsewhere.  The
 * fixed mode applies const_r, const_phi and const_z of both fields to the
 * named component on the same cells; linerad_* has no defined parameters. */
static int extf_code(const char* name) {
  static const char* names[6] = {"none", "const_r", "const_phi", "const_z", "linerad_r", "linerad_z"};
  if (!name) return 0;
  for (int c = 0; c < 6; ++c)
    if (!strcmp(name, names[c])) return c;
  return -1;
}

int orc_set_external_fields(orc_sim* s, const char* electric, const double* e_params, int n_e,
                            const char* magnetic, const double* m_params, int n_m) {
  const int fixed = s->quirks == ORC_QUIRKS_FIXED;
  int ec = extf_code(electric), mc = extf_code(magnetic);
  if (mc < 0 || (fixed && ec < 0)) return ST_ARG;
  if (!fixed) {
    ec = 0;
    if (mc != 3) mc = 0;
  }
  if (ec >= 4 || mc >= 4) return -13; /* PCG_ERR_UNSUPPORTED */
  if ((ec && (!e_params || n_e < 1)) || (mc && (!m_params || n_m < 1))) return ST_ARG;
  size_t ng = (size_t)(s->nr + 4) * (size_t)(s->nz + 4);
  for (int c = 0; c < 3; ++c) {
    free(s->Eext[c]); free(s->Hext[c]);
    s->Eext[c] = s->Hext[c] = NULL;
  }
  if (!ec && !mc) return ST_OK;
  for (int c = 0; c < 3; ++c) {
    s->Eext[c] = (double*)calloc(ng, sizeof(double));
    s->Hext[c] = (double*)calloc(ng, sizeof(double));
  }
  if (ec)
    for (int i = 1; i < s->nr - 1; ++i)
      for (int k = 1; k < s->nz - 1; ++k) s->Eext[ec - 1][IDX(s, i, k)] = e_params[0];
  if (mc)
    for (int i = 1; i < s->nr - 1; ++i)
      for (int k = 1; k < s->nz - 1; ++k) s->Hext[mc - 1][IDX(s, i, k)] = m_params[0];
  return ST_OK;
}

void orc_destroy(orc_sim* s) {
  if (!s) return;
  for (int c = 0; c < 3; ++c) {
    free(s->E[c]); free(s->H[c]); free(s->Hat[c]); free(s->J[c]);
    free(s->Eext[c]); free(s->Hext[c]);
  }
  free(s->sigma);
  for (int t = 0; t < s->nsp; ++t) {
    species_t* p = &s->sp[t];
    free(p->r); free(p->phi); free(p->z); free(p->r_old); free(p->phi_old); free(p->z_old);
    free(p->vr); free(p->vphi); free(p->vz); free(p->w); free(p->sn);
    free(p->cell_r); free(p->cell_z); free(p->abs_map);
  }
  free(s);
}

/* ------------------------------------------------------------------ */
/* Binary Coulomb collisions, Perez et al. 2012 (the reference's default */
/* scheme): Collisions::operator() (collisions.cpp:230-236) over         */
/* CollisionsP12::collide (collisionsP12.cpp:330-548) and ::collide_single */
/* (:29-328).                                                            */
/*                                                                       */
/* quirks=reference keeps: the relative speed as the difference of the   */
/* CM speeds (:139-140; equal masses then give a round-off speed), the    */
/* deflection test U < w against the macroparticle weight (:255, :268),   */
/* and `break` out of the cell row on a non-normal temperature or density */
/* (:351-354).  quirks=fixed uses the sum of the CM speeds, deflects the  */
/* lighter-weight particle always and the other with probability w_a/w_b, */
/* and skips only the cell.                                              */
/*                                                                       */
/* Random numbers: with ORC_RNG_MT19937 the reference's sequence (U, phi, */
/* U_defl per collision that passes the early returns) and no shuffle of  */
/* the cell lists (the reference shuffles with std::srand(time(0)), which */
/* no run can repeat); with ORC_RNG_PHILOX the GPU's counter scheme:      */
/* collision m of cell c draws from blocks (c, 2m) and (c, 2m+1), and the */
/* cell lists are shuffled by Fisher-Yates with draws (c, i); the third  */
/* counter word is the pass number (one pass per collision call).        */

#define K_PLANK_BAR (6.6261e-34 / (2. * K_PI))
#define COLL_TAG 0x636f6c6cu
#define SHUF_TAG 0x73687566u

typedef struct {
  orc_sim* s;
  uint32_t cell, m; /* Philox counters of the current collision */
} coll_rng;

static double coll_draw(coll_rng* g, int q) {
  orc_sim* s = g->s;
  if (s->rng_kind != ORC_RNG_PHILOX) return mt_uniform(&s->mt);
  uint32_t ctr[4] = {g->cell, 2u * g->m + (uint32_t)(q >> 1), s->coll_pass, COLL_TAG};
  uint32_t key[2] = {(uint32_t)s->seed, (uint32_t)(s->seed >> 32)};
  uint32_t o[4];
  orc_philox4x32_10(ctr, key, o);
  uint32_t a = (q & 1) ? o[2] : o[0], b = (q & 1) ? o[3] : o[1];
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

static double shuffle_draw(orc_sim* s, uint32_t cell, uint32_t i, uint32_t list) {
  uint32_t ctr[4] = {cell, i, s->coll_pass, SHUF_TAG + list};
  uint32_t key[2] = {(uint32_t)s->seed, (uint32_t)(s->seed >> 32)};
  uint32_t o[4];
  orc_philox4x32_10(ctr, key, o);
  return ((double)(o[0] >> 5) * 67108864.0 + (double)(o[1] >> 6)) * (1.0 / 9007199254740992.0);
}

typedef struct {
  species_t* sp;
  size_t j;
} pref; /* a particle: species and index */

static int lorenz_or_flag(orc_sim* s, double v2, double* g) {
  if (lorenz_factor(v2, g) != ST_OK) { s->errors++; return 0; }
  return 1;
}

/* CollisionsP12::collide_single (collisionsP12.cpp:29-328). */
static void p12_single(orc_sim* s, coll_rng* g, double m_real_a, double m_real_b, double q_real_a,
                       double q_real_b, pref pa, pref pb, double density_a_in,
                       double density_b_in, double debye_in) {
  const int fixed = s->quirks == ORC_QUIRKS_FIXED;
  double charge_a, mass_a, charge_b, mass_b, w_a, w_b, density_a, density_b;
  double v_a[3], v_b[3];
  int swap = 0;
  double w_ratio = pa.sp->w[pa.j] / pb.sp->w[pb.j];
  pref A = pa, B = pb;
  if (w_ratio <= 1) {
    charge_a = q_real_a; mass_a = m_real_a; density_a = density_a_in;
    charge_b = q_real_b; mass_b = m_real_b; density_b = density_b_in;
  } else {
    A = pb; B = pa;
    charge_a = q_real_b; mass_a = m_real_b; density_a = density_b_in;
    charge_b = q_real_a; mass_b = m_real_a; density_b = density_a_in;
    swap = 1;
  }
  v_a[0] = A.sp->vr[A.j]; v_a[1] = A.sp->vphi[A.j]; v_a[2] = A.sp->vz[A.j];
  v_b[0] = B.sp->vr[B.j]; v_b[1] = B.sp->vphi[B.j]; v_b[2] = B.sp->vz[B.j];
  w_a = A.sp->w[A.j];
  w_b = B.sp->w[B.j];

  if (v_a[0] == v_b[0] && v_a[1] == v_b[1] && v_a[2] == v_b[2]) return;

  double gamma_a, gamma_b;
  if (!lorenz_or_flag(s, len2(v_a), &gamma_a) || !lorenz_or_flag(s, len2(v_b), &gamma_b)) return;
  const double ga0 = gamma_a, gb0 = gamma_b; /* momentum_0 / momentum recompute the same gamma */
  const double p0_a = ga0 * mass_a * K_LIGHT_VEL, p0_b = gb0 * mass_b * K_LIGHT_VEL; /* rel.cpp:57-64 */
  double p_a[3], p_b[3], beta_cm[3];
  for (int c = 0; c < 3; ++c) { p_a[c] = v_a[c] * ga0; p_a[c] *= mass_a; } /* rel.cpp:66-72 */
  for (int c = 0; c < 3; ++c) { p_b[c] = v_b[c] * gb0; p_b[c] *= mass_b; }
  for (int c = 0; c < 3; ++c) beta_cm[c] = p_a[c] + p_b[c];
  const double p0_sum = p0_a + p0_b;
  for (int c = 0; c < 3; ++c) beta_cm[c] /= p0_sum;

  double gamma_cm;
  const double v_cm_2 = len2(beta_cm) * K_LIGHT_VEL_POW_2;
  if (!lorenz_or_flag(s, v_cm_2, &gamma_cm)) return;

  const double p0_a_cm = gamma_cm * (p0_a - dot3(beta_cm, p_a));
  const double p0_b_cm = gamma_cm * (p0_b - dot3(beta_cm, p_b));

  double p_a_cm[3], p_b_cm[3], t[3];
  for (int c = 0; c < 3; ++c) p_a_cm[c] = p_a[c];
  {
    const double d = dot3(beta_cm, p_a), l2 = len2(beta_cm);
    for (int c = 0; c < 3; ++c) { t[c] = beta_cm[c] * d; t[c] *= (gamma_cm - 1); t[c] /= l2; }
    for (int c = 0; c < 3; ++c) p_a_cm[c] += t[c];
    for (int c = 0; c < 3; ++c) { t[c] = beta_cm[c] * gamma_cm; t[c] *= p0_a; }
    for (int c = 0; c < 3; ++c) p_a_cm[c] -= t[c];
  }
  for (int c = 0; c < 3; ++c) p_b_cm[c] = -p_a_cm[c];

  double v_cm[3];
  for (int c = 0; c < 3; ++c) v_cm[c] = beta_cm[c] * K_LIGHT_VEL;
  const double gamma_a_cm = (1 - dot3(v_a, v_cm) / K_LIGHT_VEL_POW_2) * gamma_a * gamma_cm;
  const double gamma_b_cm = (1 - dot3(v_b, v_cm) / K_LIGHT_VEL_POW_2) * gamma_b * gamma_cm;

  double v_a_cm[3], v_b_cm[3];
  const double da = mass_a * gamma_a_cm, db = mass_b * gamma_b_cm;
  for (int c = 0; c < 3; ++c) { v_a_cm[c] = p_a_cm[c] / da; v_b_cm[c] = p_b_cm[c] / db; }

  const double la = sqrt(len2(v_a_cm)), lb = sqrt(len2(v_b_cm));
  const double v_rel_abs = (fixed ? la + lb : la - lb) / (1 - dot3(v_a_cm, v_b_cm) / K_LIGHT_VEL_POW_2);

  double gamma_rel;
  if (!lorenz_or_flag(s, v_rel_abs * v_rel_abs, &gamma_rel)) return;
  const double p_rel_abs = gamma_rel * mass_b * v_rel_abs;

  if (p_rel_abs == 0) return;
  if (v_rel_abs < K_MNZL) return;
  if (!isnormal(density_a)) return;
  if (!isnormal(density_b)) return;

  const int rel = len2(v_a) > K_REL_LIMIT_POW_2 || len2(v_b) > K_REL_LIMIT_POW_2;
  const double debye = rel ? debye_in * gamma_rel : debye_in;

  /* phys::plasma::coulomb_logarithm (plasma.cpp:42-52) */
  const double m_red = mass_a * mass_b / (mass_a + mass_b);
  const double cl = log(debye * m_red * v_rel_abs / K_PLANK_BAR);
  const double L_coulomb = 2. < cl ? cl : 2.; /* std::max(2., cl) */

  const double density_w = density_a * density_b / (density_a < density_b ? density_a : density_b);
  const double mass_ab = mass_a * mass_b / (mass_a + mass_b);

  double s12;
  if (rel) {
    const double qq = charge_a * charge_b;
    const double ec = K_EPSILON0 * K_LIGHT_VEL_POW_2;
    const double f = mass_a * gamma_a_cm * mass_b * gamma_b_cm * K_LIGHT_VEL_POW_2 / len2(p_a_cm) + 1;
    s12 = density_w * s->dt * L_coulomb * (qq * qq)
          / (4 * K_PI * (ec * ec) * mass_a * gamma_a * mass_b * gamma_b)
          * gamma_cm * sqrt(len2(p_a)) / (mass_a * gamma_a + mass_b * gamma_b)
          * (f * f);
  } else {
    const double qq = charge_a * charge_b;
    const double em = K_EPSILON0 * mass_ab;
    s12 = density_w * s->dt * L_coulomb * (qq * qq)
          / (4 * K_PI * (em * em) * pow(v_rel_abs, 3));
  }

  if (v_rel_abs < 1e6 && density_w > 7e13) { /* low-temperature cap :203-213 */
    const double na = mass_a * pow(density_a, 2. / 3.), nb = mass_b * pow(density_b, 2. / 3.);
    const double s12max = pow(4. / 3. * K_PI, 1. / 3.) * density_w * s->dt * (mass_a + mass_b)
                          / (na > nb ? na : nb) * v_rel_abs;
    if (s12max < s12) s12 = s12max;
  }

  const double U = coll_draw(g, 0);
  double cos_xi_cm;
  if (s12 < 0.1) {
    cos_xi_cm = 1 + s12 * log(U);
  } else if (s12 < 3) {
    const double A_inv = 0.00569578 + 0.9560202 * s12 - 0.508139 * pow(s12, 2)
                         + 0.47913906 * pow(s12, 3) - 0.12788975 * pow(s12, 4)
                         + 0.02389567 * pow(s12, 5);
    const double A = 1. / A_inv;
    cos_xi_cm = A_inv * log(exp(-A) + 2. * U * sinh(A));
  } else if (s12 < 6.) {
    const double A = 3. * exp(-s12);
    const double A_inv = 1. / A;
    cos_xi_cm = A_inv * log(exp(-A) + 2. * U * sinh(A));
  } else {
    cos_xi_cm = 2 * U - 1;
  }
  const double sin_xi_cm = sqrt(1 - pow(cos_xi_cm, 2));

  const double phi_cm = (2 * K_PI) * coll_draw(g, 1); /* uniform_distribution_angle rand.cpp:45-49 */
  const double sin_phi_cm = sin(phi_cm), cos_phi_cm = cos(phi_cm);

  double p_a_prime_cm[3];
  const double p_a_cm_abs = sqrt(len2(p_a_cm));
  const double p_cm_prp = sqrt(p_a_cm[0] * p_a_cm[0] + p_a_cm[1] * p_a_cm[1]);
  p_a_prime_cm[0] = p_a_cm[0] * p_a_cm[2] / p_cm_prp * sin_xi_cm * cos_phi_cm
                    - p_a_cm[1] * p_a_cm_abs / p_cm_prp * sin_xi_cm * sin_phi_cm
                    + p_a_cm[0] * cos_xi_cm;
  p_a_prime_cm[1] = p_a_cm[1] * p_a_cm[2] / p_cm_prp * sin_xi_cm * cos_phi_cm
                    + p_a_cm[0] * p_a_cm_abs / p_cm_prp * sin_xi_cm * sin_phi_cm
                    + p_a_cm[1] * cos_xi_cm;
  p_a_prime_cm[2] = -p_cm_prp * sin_xi_cm * cos_phi_cm + p_a_cm[2] * cos_xi_cm;

  const double U_defl = coll_draw(g, 2);
  /* which of v_a', v_b' are computed (the others stay zero, vector3d()) */
  const int defl_a = fixed ? 1 : U_defl < w_a;
  const int defl_b = fixed ? U_defl < w_a / w_b : U_defl < w_b;

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
    const double gi = pow(1.0 + len2(v_a_prime) / K_LIGHT_VEL_POW_2, -0.5); /* rel.cpp:47-55 */
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
    const double gi = pow(1.0 + len2(v_b_prime) / K_LIGHT_VEL_POW_2, -0.5);
    for (int c = 0; c < 3; ++c) v_b_prime[c] *= gi;
  }
  /* write back (:279-310).  A is the lighter-weight particle (pa unless
   * swapped); the reference tests U < w_a for pa and U < w_b for pb in
   * both orders, so a swapped pair can receive a zero vector when a
   * weight is below 1. */
  const double* to_pa = swap ? v_b_prime : v_a_prime;
  const double* to_pb = swap ? v_a_prime : v_b_prime;
  int set_pa, set_pb;
  if (fixed) {
    set_pa = swap ? defl_b : defl_a;
    set_pb = swap ? defl_a : defl_b;
  } else {
    set_pa = U_defl < w_a;
    set_pb = U_defl < w_b;
  }
  if (set_pa) { pa.sp->vr[pa.j] = to_pa[0]; pa.sp->vphi[pa.j] = to_pa[1]; pa.sp->vz[pa.j] = to_pa[2]; }
  if (set_pb) { pb.sp->vr[pb.j] = to_pb[0]; pb.sp->vphi[pb.j] = to_pb[1]; pb.sp->vz[pb.j] = to_pb[2]; }
}

/* std::normal_distribution<double>(0, stddev) as libstdc++ implements it
 * (Marsaglia's polar method; a fresh distribution object per call, as
 * math::random::normal makes one, so the second value of each accepted
 * pair is discarded).  Philox mode: Box-Muller on draws 0 and 1. */
static double coll_normal(coll_rng* g, double stddev) {
  orc_sim* s = g->s;
  double y, mult;
  if (s->rng_kind == ORC_RNG_PHILOX) {
    const double u0 = coll_draw(g, 0), u1 = coll_draw(g, 1);
    y = sqrt(-2.0 * log(1.0 - u0)) * cos(2.0 * K_PI * u1);
    return y * stddev;
  }
  double x, r2;
  do {
    x = 2.0 * mt_uniform(&s->mt) - 1.0;
    y = 2.0 * mt_uniform(&s->mt) - 1.0;
    r2 = x * x + y * y;
  } while (r2 > 1.0 || r2 == 0.0);
  mult = sqrt(-2 * log(r2) / r2);
  return y * mult * stddev + 0.0;
}

/* phys::plasma::coulomb_logarithm (plasma.cpp:42-52) */
static double coulomb_log(double m_a, double m_b, double debye, double v_rel) {
  const double m_ab = m_a * m_b / (m_a + m_b);
  const double cl = log(debye * m_ab * v_rel / K_PLANK_BAR);
  return cl > 2. ? cl : 2.;
}

/* CollisionsTA77S::collide_single (collisionsTA77S.cpp:33-208): Takizuka-Abe
 * scattering by a normal delta of variance q_a^2 q_b^2 n L dt /
 * (8 pi eps0^2 m_ab^2 u^3), with the weighted second angle for the heavier-
 * weight particle.  Draws: delta (normal), Phi (uniform angle), dzeta.
 * The reference adds m_ab/m_b du2 to b (:191-193), where the scheme
 * subtracts it; the fixed mode subtracts. */
static void ta77s_single(orc_sim* s, coll_rng* g, double m_real_a, double m_real_b, double q_real_a,
                         double q_real_b, pref pa, pref pb, double density_a_in, double density_b_in,
                         double debye) {
  const int fixed = s->quirks == ORC_QUIRKS_FIXED;
  double w_ratio = pa.sp->w[pa.j] / pb.sp->w[pb.j];
  pref A = pa, B = pb;
  double charge_a, mass_a, density_a, charge_b, mass_b, density_b;
  if (w_ratio <= 1) {
    charge_a = q_real_a; mass_a = m_real_a; density_a = density_a_in;
    charge_b = q_real_b; mass_b = m_real_b; density_b = density_b_in;
  } else {
    A = pb; B = pa;
    charge_a = q_real_b; mass_a = m_real_b; density_a = density_b_in;
    charge_b = q_real_a; mass_b = m_real_a; density_b = density_a_in;
    w_ratio = 1 / w_ratio;
  }
  const double vr_a = A.sp->vr[A.j], vphi_a = A.sp->vphi[A.j], vz_a = A.sp->vz[A.j];
  const double vr_b = B.sp->vr[B.j], vphi_b = B.sp->vphi[B.j], vz_b = B.sp->vz[B.j];
  const double density_lowest = density_a < density_b ? density_a : density_b;
  const double m_ab = mass_a * mass_b / (mass_a + mass_b);
  const double ux = vr_a - vr_b, uy = vphi_a - vphi_b, uz = vz_a - vz_b;
  const double u = sqrt(ux * ux + uy * uy + uz * uz);
  if (u == 0) return;
  const double lambda = coulomb_log(mass_a, mass_b, debye, u);
  const double u_p = sqrt(ux * ux + uy * uy);
  const double variance_d = charge_a * charge_a * (charge_b * charge_b) * density_lowest * lambda /
                            (8 * K_PI * (K_EPSILON0 * K_EPSILON0) * (m_ab * m_ab) * pow(u, 3)) * s->dt;
  const double delta = coll_normal(g, sqrt(variance_d));
  const double sin_T = 2 * delta / (1 + delta * delta);
  const double cos_T = 1 - 2 * (delta * delta) / (1 + delta * delta);
  double sin_T2 = sqrt(w_ratio * (sin_T * sin_T) + w_ratio * (1 - w_ratio) * ((1 - cos_T) * (1 - cos_T)));
  const double cos_T2 = 1 - w_ratio * (1 - cos_T);
  if (sin_T2 * sin_T < 0) sin_T2 = -sin_T2;
  const double phi = (s->rng_kind == ORC_RNG_PHILOX ? coll_draw(g, 2) : mt_uniform(&s->mt)) * (2 * K_PI) + 0.0;
  const double dzeta = s->rng_kind == ORC_RNG_PHILOX ? coll_draw(g, 3) : mt_uniform(&s->mt);
  const double phi2 = phi + 2 * K_PI * (1 - sqrt(w_ratio)) * (1 - dzeta);
  const double sin_P = sin(phi), cos_P = cos(phi), sin_P2 = sin(phi2), cos_P2 = cos(phi2);
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
  const double kb = fixed ? -(m_ab / mass_b) : m_ab / mass_b;
  A.sp->vr[A.j] = vr_a + m_ab / mass_a * du[0];
  A.sp->vphi[A.j] = vphi_a + m_ab / mass_a * du[1];
  A.sp->vz[A.j] = vz_a + m_ab / mass_a * du[2];
  B.sp->vr[B.j] = vr_b + kb * du2[0];
  B.sp->vphi[B.j] = vphi_b + kb * du2[1];
  B.sp->vz[B.j] = vz_b + kb * du2[2];
}

/* CollisionsSK98::collide_single (collisionsSK98.cpp:29-244): relativistic
 * scattering in the centre-of-mass frame by a normal delta whose variance is
 * the collision frequency (plasma.cpp:54-63) times dt; the CM deflection
 * angle follows from tan theta_cm = sin theta / (gamma_cm (cos theta -
 * v_cm / v_rel)), the azimuth is uniform.  Both particles always take the
 * new velocities (no weight rejection, no correction pass).  Draws: delta
 * (normal), Phi (uniform angle).  The reference's relative speed subtracts
 * the CM speeds of two particles moving apart (:131-132); the fixed mode
 * adds them, as for P12. */
static void sk98_single(orc_sim* s, coll_rng* g, double m_real_a, double m_real_b, double q_real_a,
                        double q_real_b, pref pa, pref pb, double density_a_in, double density_b_in,
                        double debye) {
  const int fixed = s->quirks == ORC_QUIRKS_FIXED;
  double charge_a, mass_a, charge_b, mass_b, density_a, density_b;
  int swap = 0;
  const double w_ratio = pa.sp->w[pa.j] / pb.sp->w[pb.j];
  pref A = pa, B = pb;
  if (w_ratio <= 1) {
    charge_a = q_real_a; mass_a = m_real_a; density_a = density_a_in;
    charge_b = q_real_b; mass_b = m_real_b; density_b = density_b_in;
  } else {
    A = pb; B = pa;
    charge_a = q_real_b; mass_a = m_real_b; density_a = density_b_in;
    charge_b = q_real_a; mass_b = m_real_a; density_b = density_a_in;
    swap = 1;
  }
  double v_a[3], v_b[3];
  v_a[0] = A.sp->vr[A.j]; v_a[1] = A.sp->vphi[A.j]; v_a[2] = A.sp->vz[A.j];
  v_b[0] = B.sp->vr[B.j]; v_b[1] = B.sp->vphi[B.j]; v_b[2] = B.sp->vz[B.j];
  if (v_a[0] == v_b[0] && v_a[1] == v_b[1] && v_a[2] == v_b[2]) return;

  double gamma_a, gamma_b;
  if (!lorenz_or_flag(s, len2(v_a), &gamma_a) || !lorenz_or_flag(s, len2(v_b), &gamma_b)) return;
  const double p0_a = gamma_a * mass_a * K_LIGHT_VEL, p0_b = gamma_b * mass_b * K_LIGHT_VEL; /* rel.cpp:57-64 */
  double p_a[3], p_b[3], beta_cm[3];
  for (int c = 0; c < 3; ++c) { p_a[c] = v_a[c] * gamma_a; p_a[c] *= mass_a; } /* rel.cpp:66-72 */
  for (int c = 0; c < 3; ++c) { p_b[c] = v_b[c] * gamma_b; p_b[c] *= mass_b; }
  for (int c = 0; c < 3; ++c) beta_cm[c] = p_a[c] + p_b[c];
  const double p0_sum = p0_a + p0_b;
  for (int c = 0; c < 3; ++c) beta_cm[c] /= p0_sum;

  double gamma_cm;
  const double v_cm_2 = len2(beta_cm) * K_LIGHT_VEL_POW_2;
  if (!lorenz_or_flag(s, v_cm_2, &gamma_cm)) return;
  const double p0_a_cm = gamma_cm * (p0_a - dot3(beta_cm, p_a));
  const double p0_b_cm = gamma_cm * (p0_b - dot3(beta_cm, p_b));

  /* Lorentz boost of a 3-momentum: p + beta (beta.p)(gamma - 1)/beta^2 + sign beta gamma p0 */
  double p_a_cm[3], p_b_cm[3], t[3];
  const double l2 = len2(beta_cm);
  {
    const double d = dot3(beta_cm, p_a);
    for (int c = 0; c < 3; ++c) p_a_cm[c] = p_a[c];
    for (int c = 0; c < 3; ++c) { t[c] = beta_cm[c] * d; t[c] *= (gamma_cm - 1); t[c] /= l2; }
    for (int c = 0; c < 3; ++c) p_a_cm[c] += t[c];
    for (int c = 0; c < 3; ++c) { t[c] = beta_cm[c] * gamma_cm; t[c] *= p0_a; }
    for (int c = 0; c < 3; ++c) p_a_cm[c] -= t[c];
  }
  for (int c = 0; c < 3; ++c) p_b_cm[c] = -p_a_cm[c];

  const double gamma_a_cm = p0_a_cm / mass_a / K_LIGHT_VEL;
  const double gamma_b_cm = p0_b_cm / mass_b / K_LIGHT_VEL;
  double v_a_cm[3], v_b_cm[3];
  const double da = mass_a * gamma_a_cm, db = mass_b * gamma_b_cm;
  for (int c = 0; c < 3; ++c) { v_a_cm[c] = p_a_cm[c] / da; v_b_cm[c] = p_b_cm[c] / db; }
  double p_cm[3];
  for (int c = 0; c < 3; ++c) p_cm[c] = p_a_cm[c];

  const double la = sqrt(len2(v_a_cm)), lb = sqrt(len2(v_b_cm));
  const double v_rel_abs = (fixed ? la + lb : la - lb) / (1 - dot3(v_a_cm, v_b_cm) / K_LIGHT_VEL_POW_2);
  double gamma_rel;
  if (!lorenz_or_flag(s, v_rel_abs * v_rel_abs, &gamma_rel)) return;
  const double p_rel_abs = gamma_rel * mass_b * v_rel_abs;
  const double density_lowest = density_b < density_a ? density_b : density_a; /* std::min */
  if (p_rel_abs == 0) return;
  if (v_rel_abs < K_MNZL) return;
  const double L_coulomb = coulomb_log(mass_a, mass_b, debye, v_rel_abs);
  if (L_coulomb <= 0) return;
  /* phys::plasma::collision_freqency (plasma.cpp:54-63) */
  const double coll_freq = pow(charge_a * charge_b, 2) * density_lowest * L_coulomb /
                           (8 * K_PI * pow(K_EPSILON0, 2) * pow(p_rel_abs, 2) * v_rel_abs);
  const double variance_d = coll_freq * s->dt;
  const double std_dev_d = sqrt(variance_d);
  const double delta = coll_normal(g, std_dev_d);
  const double sin_theta = 2 * delta / (1 + pow(delta, 2));
  const double cos_theta = 1 - 2 * pow(delta, 2) / (1 + pow(delta, 2));
  const double tg_theta_cm = sin_theta / (gamma_cm * (cos_theta - sqrt(v_cm_2) / v_rel_abs));
  const double sin_theta_cm = sin(atan(tg_theta_cm));
  const double cos_theta_cm = cos(atan(tg_theta_cm));
  const double phi_angle = (s->rng_kind == ORC_RNG_PHILOX ? coll_draw(g, 2) : mt_uniform(&s->mt)) * (2 * K_PI) + 0.0;
  const double sin_phi = sin(phi_angle), cos_phi = cos(phi_angle);

  const double p_cm_abs = sqrt(len2(p_cm));
  const double p_cm_prp = sqrt(p_cm[0] * p_cm[0] + p_cm[1] * p_cm[1]);
  double d_p[3];
  d_p[0] = p_cm[0] * p_cm[2] / p_cm_prp * sin_theta_cm * cos_phi
         - p_cm[1] * p_cm_abs / p_cm_prp * sin_theta_cm * sin_phi
         - p_cm[0] * (1 - cos_theta_cm);
  d_p[1] = p_cm[1] * p_cm[2] / p_cm_prp * sin_theta_cm * cos_phi
         + p_cm[0] * p_cm_abs / p_cm_prp * sin_theta_cm * sin_phi
         - p_cm[1] * (1 - cos_theta_cm);
  d_p[2] = -p_cm_prp * sin_theta_cm * cos_phi - p_cm[2] * (1 - cos_theta_cm);

  double pa_prime[3], pb_prime[3];
  for (int c = 0; c < 3; ++c) { pa_prime[c] = p_a_cm[c] + d_p[c]; pb_prime[c] = p_b_cm[c] - d_p[c]; }
  /* back to the LAB frame: + beta (beta.p')(gamma - 1)/beta^2 + beta gamma p0_cm */
  double* outs[2] = {pa_prime, pb_prime};
  const double p0s[2] = {p0_a_cm, p0_b_cm};
  for (int k = 0; k < 2; ++k) {
    double* q = outs[k];
    const double d = dot3(beta_cm, q);
    for (int c = 0; c < 3; ++c) { t[c] = beta_cm[c] * d; t[c] *= (gamma_cm - 1); t[c] /= l2; }
    for (int c = 0; c < 3; ++c) q[c] += t[c];
    for (int c = 0; c < 3; ++c) { t[c] = beta_cm[c] * gamma_cm; t[c] *= p0s[k]; }
    for (int c = 0; c < 3; ++c) q[c] += t[c];
  }
  double v_a_prime[3], v_b_prime[3];
  for (int c = 0; c < 3; ++c) { v_a_prime[c] = pa_prime[c] / mass_a; v_b_prime[c] = pb_prime[c] / mass_b; }
  const double gia = pow(1.0 + len2(v_a_prime) / K_LIGHT_VEL_POW_2, -0.5); /* lorenz_factor_inv */
  const double gib = pow(1.0 + len2(v_b_prime) / K_LIGHT_VEL_POW_2, -0.5);
  for (int c = 0; c < 3; ++c) { v_a_prime[c] *= gia; v_b_prime[c] *= gib; }
  const double* to_pa = swap ? v_b_prime : v_a_prime;
  const double* to_pb = swap ? v_a_prime : v_b_prime;
  pa.sp->vr[pa.j] = to_pa[0]; pa.sp->vphi[pa.j] = to_pa[1]; pa.sp->vz[pa.j] = to_pa[2];
  pb.sp->vr[pb.j] = to_pb[0]; pb.sp->vphi[pb.j] = to_pb[1]; pb.sp->vz[pb.j] = to_pb[2];
}

static int name_is(const char* n, const char* lower, const char* cap) {
  return strcmp(n, lower) == 0 || strcmp(n, cap) == 0;
}

/* Per cell and list (0 electrons, 1 ions): the sums of
 * collect_weighted_params_tot_grid (collisions.cpp:172-221). */
typedef struct {
  double amount, mom[3], energy;
} coll_tot;

static void ta77s_correct(orc_sim* s, pref* L, unsigned n, double mass, const coll_tot* t);

/* One collision pass over all cells (scheme 0: CollisionsP12, 1:
 * CollisionsTA77S with its correct_velocities, 2: CollisionsSK98, whose
 * collide() pairs as P12's does, collisionsSK98.cpp:246-440).  shuffle: Philox
 * Fisher-Yates of the cell lists (ORC_RNG_PHILOX only).  Returns the number
 * of collide_single calls, or a negative status. */
static long collide_pass(orc_sim* s, int shuffle, int scheme) {
  int el = -1, ion = -1;
  for (int t = 0; t < s->nsp; ++t) { /* collisions.cpp:28-48: the last match wins */
    if (name_is(s->sp[t].name, "electrons", "Electrons")) el = t;
    if (name_is(s->sp[t].name, "ions", "Ions")) ion = t;
  }
  if (el < 0 || ion < 0) return ST_ARG;
  const int fixed = s->quirks == ORC_QUIRKS_FIXED;
  const size_t ncell = (size_t)s->nr * s->nz;
  /* sort_to_cells (collisions.cpp:87-108): counting sort, stable in species
   * then particle order; ions to the ion lists, every other species to the
   * electron lists */
  size_t *cnt_e = calloc(ncell + 1, sizeof(size_t)), *cnt_i = calloc(ncell + 1, sizeof(size_t));
  size_t tot_e = 0, tot_i = 0;
  for (int t = 0; t < s->nsp; ++t) {
    species_t* p = &s->sp[t];
    const int is_ion = name_is(p->name, "ions", "Ions");
    for (size_t j = 0; j < p->n; ++j) {
      long long ci = p->cell_r[j], ck = p->cell_z[j];
      if (ci < 0 || ck < 0 || ci >= s->nr || ck >= s->nz) continue;
      size_t c = (size_t)ci * s->nz + (size_t)ck;
      if (is_ion) { cnt_i[c + 1]++; tot_i++; } else { cnt_e[c + 1]++; tot_e++; }
    }
  }
  for (size_t c = 0; c < ncell; ++c) { cnt_e[c + 1] += cnt_e[c]; cnt_i[c + 1] += cnt_i[c]; }
  pref *le = malloc((tot_e + 1) * sizeof(pref)), *li = malloc((tot_i + 1) * sizeof(pref));
  size_t *fe = malloc((ncell + 1) * sizeof(size_t)), *fi = malloc((ncell + 1) * sizeof(size_t));
  memcpy(fe, cnt_e, (ncell + 1) * sizeof(size_t));
  memcpy(fi, cnt_i, (ncell + 1) * sizeof(size_t));
  for (int t = 0; t < s->nsp; ++t) {
    species_t* p = &s->sp[t];
    const int is_ion = name_is(p->name, "ions", "Ions");
    for (size_t j = 0; j < p->n; ++j) {
      long long ci = p->cell_r[j], ck = p->cell_z[j];
      if (ci < 0 || ck < 0 || ci >= s->nr || ck >= s->nz) continue;
      size_t c = (size_t)ci * s->nz + (size_t)ck;
      pref r = {p, j};
      if (is_ion) li[fi[c]++] = r; else le[fe[c]++] = r;
    }
  }
  free(fe); free(fi);
  if (shuffle && s->rng_kind == ORC_RNG_PHILOX) {
    for (size_t c = 0; c < ncell; ++c) {
      pref* L[2] = {le + cnt_e[c], li + cnt_i[c]};
      size_t n[2] = {cnt_e[c + 1] - cnt_e[c], cnt_i[c + 1] - cnt_i[c]};
      for (int l = 0; l < 2; ++l)
        for (size_t i = 1; i < n[l]; ++i) {
          size_t j = (size_t)(shuffle_draw(s, (uint32_t)c, (uint32_t)i, (uint32_t)l) * (double)(i + 1));
          if (j > i) j = i;
          pref tmp = L[l][i]; L[l][i] = L[l][j]; L[l][j] = tmp;
        }
    }
  }
  const double m_el = s->sp[el].mass, m_ion = s->sp[ion].mass;
  const double q_el = s->sp[el].charge, q_ion = s->sp[ion].charge;
  /* collect_weighted_params_tot_grid (collisions.cpp:172-221), every cell
   * before any collision: ions, then electrons, in list order */
  coll_tot* tot = calloc(2 * ncell, sizeof(coll_tot));
  for (size_t c = 0; c < ncell; ++c) {
    for (int l = 1; l >= 0; --l) {
      pref* L = l ? li + cnt_i[c] : le + cnt_e[c];
      const size_t n = l ? cnt_i[c + 1] - cnt_i[c] : cnt_e[c + 1] - cnt_e[c];
      const double mass = l ? m_ion : m_el;
      coll_tot* t = &tot[2 * c + l];
      for (size_t k = 0; k < n; ++k) {
        const species_t* p = L[k].sp; size_t q = L[k].j;
        double vr = p->vr[q], vphi = p->vphi[q], vz = p->vz[q];
        double v_sq = vr * vr + vphi * vphi + vz * vz;
        double wm = p->w[q] * mass;
        t->mom[0] += wm * vr;
        t->mom[1] += wm * vphi;
        t->mom[2] += wm * vz;
        t->amount += p->w[q];
        t->energy += wm * v_sq / 2;
      }
    }
  }
  long calls = 0;
  for (int i = 0; i < s->nr; ++i) {
    for (int j = 0; j < s->nz; ++j) {
      const size_t c = (size_t)i * s->nz + j;
      pref* E = le + cnt_e[c];
      pref* I = li + cnt_i[c];
      const unsigned ne = (unsigned)(cnt_e[c + 1] - cnt_e[c]), ni = (unsigned)(cnt_i[c + 1] - cnt_i[c]);
      const double vol = K_PI * s->dz * s->dr * s->dr * (2.0 * i + 1); /* CELL_VOLUME(i) */
      const double T_el = tot[2 * c].energy / tot[2 * c].amount * (1. / K_EL_CHARGE);
      const double T_ion = tot[2 * c + 1].energy / tot[2 * c + 1].amount * (1. / K_EL_CHARGE);
      double n_el = 0, n_ion = 0;
      for (unsigned k = 0; k < ne; ++k) n_el += E[k].sp->w[E[k].j];
      for (unsigned k = 0; k < ni; ++k) n_ion += I[k].sp->w[I[k].j];
      n_el /= vol;
      n_ion /= vol;
      if (!isnormal(T_ion) || !isnormal(T_el) || !isnormal(n_ion) || !isnormal(n_el)) {
        if (fixed) continue;
        break; /* collisionsP12.cpp:351-354 */
      }
      /* phys::plasma::debye_length (plasma.cpp:24-33) */
      const double debye = 7433.944 / sqrt(n_el / T_el + n_ion / T_ion);
      coll_rng g = {s, (uint32_t)c, 0};
#define COLL(MA, MB, QA, QB, PA, PB, NA, NB) \
      do {                                                                          \
        if (scheme == 1) ta77s_single(s, &g, MA, MB, QA, QB, PA, PB, NA, NB, debye);    \
        else if (scheme == 2) sk98_single(s, &g, MA, MB, QA, QB, PA, PB, NA, NB, debye);\
        else p12_single(s, &g, MA, MB, QA, QB, PA, PB, NA, NB, debye);                  \
        g.m++;                                                                      \
        calls++;                                                                    \
      } while (0)
      if (ni % 2 == 0)
        for (unsigned k = 0; k < ni; k += 2) COLL(m_ion, m_ion, q_ion, q_ion, I[k], I[k + 1], n_ion, n_ion);
      if (ne % 2 == 0)
        for (unsigned k = 0; k < ne; k += 2) COLL(m_el, m_el, q_el, q_el, E[k], E[k + 1], n_el, n_el);
      if (ni % 2 != 0) {
        if (ni >= 3) {
          COLL(m_ion, m_ion, q_ion, q_ion, I[0], I[1], n_ion, n_ion);
          COLL(m_ion, m_ion, q_ion, q_ion, I[1], I[2], n_ion, n_ion);
          COLL(m_ion, m_ion, q_ion, q_ion, I[2], I[0], n_ion, n_ion);
        }
        if (ni >= 5)
          for (unsigned k = 3; k < ni; k += 2) COLL(m_ion, m_ion, q_ion, q_ion, I[k], I[k + 1], n_ion, n_ion);
      }
      if (ne % 2 != 0) {
        if (ne >= 3) {
          COLL(m_el, m_el, q_el, q_el, E[0], E[1], n_el, n_el);
          COLL(m_el, m_el, q_el, q_el, E[1], E[2], n_el, n_el);
          COLL(m_el, m_el, q_el, q_el, E[2], E[0], n_el, n_el);
        }
        if (ne >= 5)
          for (unsigned k = 3; k < ne; k += 2) COLL(m_el, m_el, q_el, q_el, E[k], E[k + 1], n_el, n_el);
      }
      if (ni == ne)
        for (unsigned k = 0; k < ne; ++k) COLL(m_el, m_ion, q_el, q_ion, E[k], I[k], n_el, n_ion);
      if (ni > ne && ne > 0 && ni > 0) {
        const unsigned c_i = (unsigned)floor((float)ni / (float)ne);
        const double c_r = (double)((float)ni / (float)ne - (float)c_i);
        const unsigned ions_1st = (unsigned)((double)(c_i + 1) * c_r * ne);
        const unsigned els_1st = (unsigned)(c_r * ne);
        const unsigned ions_2nd = (unsigned)((double)c_i * (1 - c_r) * ne);
        for (unsigned fgi = 0; fgi < ions_1st; ++fgi) {
          int fge = (int)floor((float)fgi / (float)(c_i + 1));
          COLL(m_el, m_ion, q_el, q_ion, E[fge], I[fgi], n_el, n_ion);
        }
        for (unsigned fgi = 0; fgi < ions_2nd; ++fgi) {
          int fge = (int)floor((float)fgi / (float)c_i);
          COLL(m_el, m_ion, q_el, q_ion, E[fge + els_1st], I[fgi + ions_1st], n_el, n_ion);
        }
      }
      if (ni < ne && ne > 0 && ni > 0) {
        const double c_i = floor((float)ne / (float)ni);
        const double c_r = (double)((float)ne / (float)ni) - c_i;
        const unsigned els_1st = (unsigned)((c_i + 1) * c_r * ni);
        const unsigned ions_1st = (unsigned)(c_r * ni);
        const unsigned els_2nd = (unsigned)(c_i * (1 - c_r) * ni);
        for (unsigned fge = 0; fge < els_1st; ++fge) {
          int fgi = (int)floor((float)fge / (float)(c_i + 1));
          COLL(m_el, m_ion, q_el, q_ion, E[fge], I[fgi], n_el, n_ion);
        }
        for (unsigned fge = 0; fge < els_2nd; ++fge) {
          int fgi = (int)floor((float)fge / (float)c_i);
          COLL(m_el, m_ion, q_el, q_ion, E[fge + els_1st], I[fgi + ions_1st], n_el, n_ion);
        }
      }
#undef COLL
    }
  }
  if (scheme == 1) /* correct_velocities (collisionsTA77S.cpp:419-566), every cell */
    for (size_t c = 0; c < ncell; ++c) {
      ta77s_correct(s, li + cnt_i[c], (unsigned)(cnt_i[c + 1] - cnt_i[c]), m_ion, &tot[2 * c + 1]);
      ta77s_correct(s, le + cnt_e[c], (unsigned)(cnt_e[c + 1] - cnt_e[c]), m_el, &tot[2 * c]);
    }
  free(tot);
  free(cnt_e); free(cnt_i); free(le); free(li);
  s->coll_pass++;
  return calls;
}

/* TA77S correct_velocities for one list of one cell: the list's momentum
 * change is removed and its thermal velocities scaled by sqrt(alpha) so
 * that momentum and kinetic energy return to the totals `t` collected
 * before the pass.  The reference takes |alpha| when alpha < 0 and 1 when
 * alpha == 0 (:494-498, :518-522); the fixed mode leaves such a list
 * uncorrected. */
static void ta77s_correct(orc_sim* s, pref* L, unsigned n, double mass, const coll_tot* t) {
  double mr = 0, mp = 0, mz = 0, e_new = 0;
  for (unsigned k = 0; k < n; ++k) {
    const species_t* p = L[k].sp; size_t q = L[k].j;
    double vr = p->vr[q], vphi = p->vphi[q], vz = p->vz[q];
    double v_sq = vr * vr + vphi * vphi + vz * vz;
    double mass_m = mass * p->w[q];
    mr += mass_m * vr;
    mp += mass_m * vphi;
    mz += mass_m * vz;
    e_new += mass_m * v_sq / 2;
  }
  const double mass_tot = t->amount * mass;
  const double dvr = (mr - t->mom[0]) / mass_tot, dvp = (mp - t->mom[1]) / mass_tot,
               dvz = (mz - t->mom[2]) / mass_tot;
  const double v0r = t->mom[0] / mass_tot, v0p = t->mom[1] / mass_tot, v0z = t->mom[2] / mass_tot;
  const double d_e = e_new - t->energy;
  const double v0_sq = v0r * v0r + v0p * v0p + v0z * v0z;
  double alpha = (t->energy - mass_tot * v0_sq / 2) /
                 (t->energy + d_e -
                  mass_tot * ((v0r + dvr) * (v0r + dvr) + (v0p + dvp) * (v0p + dvp) + (v0z + dvz) * (v0z + dvz)) / 2);
  if (!isnormal(alpha)) return;
  if (s->quirks == ORC_QUIRKS_FIXED) {
    if (alpha < 0) return;
  } else {
    if (alpha < 0) alpha = -alpha;
    if (alpha == 0) alpha = 1;
  }
  alpha = sqrt(alpha);
  for (unsigned k = 0; k < n; ++k) {
    species_t* p = L[k].sp; size_t q = L[k].j;
    const double vr = p->vr[q], vphi = p->vphi[q], vz = p->vz[q];
    p->vr[q] = v0r + alpha * (vr - v0r - dvr);
    p->vphi[q] = v0p + alpha * (vphi - v0p - dvp);
    p->vz[q] = v0z + alpha * (vz - v0z - dvz);
  }
}

long orc_collide(orc_sim* s, int shuffle) { return collide_pass(s, shuffle, 0); }
long orc_collide_ta77s(orc_sim* s, int shuffle) { return collide_pass(s, shuffle, 1); }
long orc_collide_sk98(orc_sim* s, int shuffle) { return collide_pass(s, shuffle, 2); }


/* ------------------------------------------------------------------ */
/* Species diagnostic maps: SpecieP::calc_density / calc_temperature /   */
/* calc_energy / calc_momentum (specieP.cpp:665-839) over                */
/* weight_cylindrical (weighter.hpp:27-130).                              */

static void grid_inc(const orc_sim* s, double* g, unsigned i, unsigned k, double v) {
  g[IDX(s, (int)i, (int)k)] += v;
}

/* weight_cylindrical: the cloud [r - dr/2, r + dr/2] x [z - dz/2, z + dz/2]
 * split at (i + 1/2) dr and (k + 1/2) dz, each part's ring volume over the
 * node's CELL_VOLUME (macro argument unparenthesised: 2i + 1 + 1 for i + 1),
 * times value / cloud volume; on the axis the cloud is cut at r = 0. */
static void weight_cyl(const orc_sim* s, double* g, double pos_r, double pos_z, double weight_value) {
  const double dr = s->dr, dz = s->dz;
  unsigned r_i = (unsigned)CELL_NUMBER(pos_r, dr);
  const unsigned z_k = (unsigned)CELL_NUMBER(pos_z, dz);
  const unsigned ri_s = r_i, zk_s = z_k;
  double v_1 = K_PI * dz * dr * dr * (2.0 * r_i + 1);
  double v_2 = K_PI * dz * dr * dr * (2.0 * r_i + 1 + 1);
  double r1, r2, r3, dz1, dz2, v_0, rho, value;
  if (pos_r > dr) {
    r1 = pos_r - 0.5 * dr;
    r2 = (r_i + 0.5) * dr;
    r3 = pos_r + 0.5 * dr;
    v_0 = 2. * K_PI * dz * dr * pos_r;
    dz1 = (z_k + 0.5) * dz - (pos_z - 0.5 * dz);
    dz2 = (pos_z + 0.5 * dz) - (z_k + 0.5) * dz;
    rho = weight_value / v_0;
    value = K_PI * dz1 * (r2 * r2 - r1 * r1) / v_1; grid_inc(s, g, ri_s, zk_s, rho * value);
    value = K_PI * dz1 * (r3 * r3 - r2 * r2) / v_2; grid_inc(s, g, ri_s + 1, zk_s, rho * value);
    value = K_PI * dz2 * (r2 * r2 - r1 * r1) / v_1; grid_inc(s, g, ri_s, zk_s + 1, rho * value);
    value = K_PI * dz2 * (r3 * r3 - r2 * r2) / v_2; grid_inc(s, g, ri_s + 1, zk_s + 1, rho * value);
  } else if (pos_r <= dr / 2.) {
    r_i = 0;
    r2 = (r_i + 0.5) * dr;
    r3 = pos_r + 0.5 * dr;
    dz1 = (z_k + 0.5) * dz - (pos_z - 0.5 * dz);
    dz2 = (pos_z + 0.5 * dz) - (z_k + 0.5) * dz;
    v_0 = K_PI * dz * (2. * pos_r * pos_r + dr * dr / 2.);
    rho = weight_value / v_0;
    value = K_PI * dz1 * (dr * dr / 2. - pos_r * dr + pos_r * pos_r) / v_1; grid_inc(s, g, ri_s, zk_s, rho * value);
    value = K_PI * dz1 * (r3 * r3 - r2 * r2) / v_2; grid_inc(s, g, ri_s + 1, zk_s, rho * value);
    value = K_PI * dz2 * (dr * dr / 2. - pos_r * dr + pos_r * pos_r) / v_1; grid_inc(s, g, ri_s, zk_s + 1, rho * value);
    value = K_PI * dz2 * (r3 * r3 - r2 * r2) / v_2; grid_inc(s, g, ri_s + 1, zk_s + 1, rho * value);
  } else {
    r1 = pos_r - 0.5 * dr;
    r2 = (r_i + 0.5) * dr;
    r3 = pos_r + 0.5 * dr;
    dz1 = (z_k + 0.5) * dz - (pos_z - 0.5 * dz);
    dz2 = (pos_z + 0.5 * dz) - (z_k + 0.5) * dz;
    v_0 = 2. * K_PI * dz * dr * pos_r;
    v_1 = K_PI * dz * dr * dr; /* CYL_VOL(dz, dr) */
    v_2 = K_PI * dz * dr * dr * (2.0 * r_i + 1 + 1);
    rho = weight_value / v_0;
    value = K_PI * dz1 * (r2 * r2 - r1 * r1) / v_1; grid_inc(s, g, ri_s, zk_s, rho * value);
    value = K_PI * dz1 * (r3 * r3 - r2 * r2) / v_2; grid_inc(s, g, ri_s + 1, zk_s, rho * value);
    value = K_PI * dz2 * (r2 * r2 - r1 * r1) / v_1; grid_inc(s, g, ri_s, zk_s + 1, rho * value);
    value = K_PI * dz2 * (r3 * r3 - r2 * r2) / v_2; grid_inc(s, g, ri_s + 1, zk_s + 1, rho * value);
  }
}

/* phys::rel::energy_m (rel.cpp:88-101) */
static double energy_m(double mass, double momentum_2) {
  if (momentum_2 > K_REL_LIMIT_POW_2 * mass * mass) {
    double e_rest = mass * K_LIGHT_VEL_POW_2;
    return sqrt(momentum_2 * K_LIGHT_VEL_POW_2 + e_rest * e_rest) - e_rest;
  }
  return 0.5 * momentum_2 / mass;
}

/* calc_momentum_w (:740-782) into m[3], calc_momentum_abs_w (:714-738) into
 * a; gamma is applied below REL_LIMIT only (the reference's test), at every
 * speed in the fixed mode.  Returns nonzero when a speed exceeds c. */
static int momentum_maps(orc_sim* s, const species_t* p, double* m[3], double* a) {
  const int fixed = s->quirks == ORC_QUIRKS_FIXED;
  for (size_t j = 0; j < p->n; ++j) {
    if (!(p->r[j] >= 0.0)) continue;
    const double v_r = p->vr[j], v_phi = p->vphi[j], v_z = p->vz[j];
    if (m) {
      const double m_weighted = p->mass * p->w[j];
      double p_r = m_weighted * v_r, p_phi = m_weighted * v_phi, p_z = m_weighted * v_z;
      const double v_abs_2 = v_r * v_r + v_phi * v_phi + v_z * v_z;
      if (fixed || v_abs_2 < K_REL_LIMIT_POW_2) {
        double gamma;
        if (lorenz_factor(v_abs_2, &gamma) != ST_OK) return -1;
        p_r *= gamma; p_phi *= gamma; p_z *= gamma;
      }
      weight_cyl(s, m[0], p->r[j], p->z[j], p_r);
      weight_cyl(s, m[1], p->r[j], p->z[j], p_phi);
      weight_cyl(s, m[2], p->r[j], p->z[j], p_z);
    }
    if (a) {
      const double v_abs = sqrt(v_r * v_r + v_phi * v_phi + v_z * v_z);
      double p_abs = p->mass * p->w[j] * v_abs;
      if (fixed || v_abs < K_REL_LIMIT) {
        double gamma;
        if (lorenz_factor(v_abs * v_abs, &gamma) != ST_OK) return -1;
        p_abs *= gamma;
      }
      weight_cyl(s, a, p->r[j], p->z[j], p_abs);
    }
  }
  return 0;
}

/* One map of species sid into out ((nr+4) x (nz+4) doubles, 3 of them for
 * ORC_MAP_MOMENTUM: r, phi, z).  which: 0 density, 1 temperature (eV),
 * 2 energy (eV), 3 momentum.  The temperature of the reference reads the
 * absolute-momentum map the last energy map left (calc_momentum_w does not
 * fill it, :681-683); before any it reads a grid never initialised, where
 * this takes zeros.  The fixed mode makes the map afresh. */
int orc_species_map(orc_sim* s, int sid, int which, double* out) {
  if (sid < 0 || sid >= s->nsp || which < 0 || which > 3) return ST_ARG;
  species_t* p = &s->sp[sid];
  const size_t nodes = (size_t)(s->nr + 4) * (size_t)(s->nz + 4);
  double* dens = calloc(nodes, sizeof(double));
  for (size_t j = 0; j < p->n; ++j)
    if (p->r[j] >= 0.0) weight_cyl(s, dens, p->r[j], p->z[j], p->w[j]);
  if (which == 0) {
    memcpy(out, dens, nodes * sizeof(double));
    free(dens);
    return ST_OK;
  }
  if (!p->abs_map) p->abs_map = calloc(nodes, sizeof(double));
  double* mw[3] = {NULL, NULL, NULL};
  int rc = 0;
  if (which == 1 || which == 3) {
    for (int c = 0; c < 3; ++c) mw[c] = calloc(nodes, sizeof(double));
    rc = momentum_maps(s, p, mw, NULL);
  }
  if (rc == 0 && (which == 2 || (which == 1 && s->quirks == ORC_QUIRKS_FIXED))) {
    memset(p->abs_map, 0, nodes * sizeof(double));
    rc = momentum_maps(s, p, NULL, p->abs_map);
  }
  if (rc == 0) {
    const int ncomp = which == 3 ? 3 : 1;
    memset(out, 0, ncomp * nodes * sizeof(double));
    for (int r = 0; r < s->nr; ++r)
      for (int z = 0; z < s->nz; ++z) {
        const size_t q = IDX(s, r, z);
        const double dl = dens[q];
        if (dl == 0) continue;
        if (which == 3) {
          for (int c = 0; c < 3; ++c) out[c * nodes + q] = mw[c][q] / dl;
        } else {
          double p2;
          if (which == 1) {
            const double p_vec_sum_2 = mw[0][q] * mw[0][q] + mw[1][q] * mw[1][q] + mw[2][q] * mw[2][q];
            p2 = p->abs_map[q] * p->abs_map[q] - p_vec_sum_2;
          } else {
            p2 = p->abs_map[q] * p->abs_map[q];
          }
          p2 /= dl * dl;
          out[q] = energy_m(p->mass, p2) * (1. / K_EL_CHARGE);
        }
      }
  }
  for (int c = 0; c < 3; ++c) free(mw[c]);
  free(dens);
  return rc == 0 ? ST_OK : ST_FATAL;
}
