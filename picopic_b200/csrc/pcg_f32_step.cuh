// pcg_f32_step.cuh — the fused single-precision particle step.
//
// One thread per macroparticle does, in registers: field gather, push,
// move in the local Cartesian frame, rotation back to r-z, wall reflection,
// velocity rotation, cell binding, the runaway test and the particle's
// charge-conserving current.  Positions are kept as an integer cell and a
// float offset in [0, 1) (units of dr, dz), so that per-step displacements
// of 1e-4..1e-1 cells keep ~1e-7 relative precision far from the axis.
//
// Every formula is the reference's, rewritten in these normalised
// coordinates (citations at each function); where the reference's form
// cancels (the logarithms of the Villasenor-Buneman weights), the same
// quantity is evaluated by a series in t = dx/x.  Arithmetic quirks of the
// reference are kept (PCG_QUIRKS_REFERENCE) except the order-dependent J_r
// overwrite of strict axial motion (currentVB.cpp:545-546), which has no
// order-free meaning for a parallel deposit; the double-precision path
// reproduces that one.
#pragma once

#include "pcg_f32.h"

namespace pcg {
namespace f32 {

constexpr int kThreads = 256;

struct StepArgs {
  GridGeom g;
  float *Er, *Ep, *Ez, *Hr, *Hp, *Hz;  // fields; H is field_h (time-centred)
  float *Jr, *Jp, *Jz;
  int nr, nz, ld;
  int plane;                   // Ep = Er + plane, ..., Hz = Er + 5 * plane
  float dt_dr, dt_dz;          // dt/dr, dt/dz
  float c2m;                   // charge*dt/(2*mass), pusherBoris.cpp:67
  float bk;                    // c2m * MAGN_CONST
  float qz, qr, qp;            // per unit weight: q/(4 pi dr^2 dt), q/(2 pi dr dz dt), q/(2 pi dz dr^2)
  float mnzl_r, mnzl_z;        // MNZL/dr, MNZL/dz
  float dr_m, dz_m, dt_s;      // dr, dz, dt in SI (ZigZag keeps metre-valued weights)
  float zz_vol;                // 1/(PI dz dr^2)
  int pusher, current, fixed, is_beam;
  int pushed;  // the velocities were pushed already (the push half of a step with collisions)
  // with pushed: the learned collision step's per-cell transforms, applied
  // to a particle before its move when its cell's flag is 1 (v' = u + (v -
  // u) s per axis, u = xform[12 c + xoff ..], s = xform[12 c + xoff + 3 ..])
  const double* xform;
  const unsigned char* xflag;
  int xoff;
  // per radial node i (row i + 2): {1/(2i+1), 1/(2i+2), 1/(2i+3), 1/(2i+4)},
  // {1/i, 1/(i+1), 1/(i+1/2), 0}; a zero where the denominator is zero
  const float4* rt;
  DevStatus* st;
};


// Shared-memory windows of a tile block, fixed by the tile geometry: the
// fields over the tile plus kHalo + 1 nodes per side, the current over the
// tile plus kHalo nodes per side.
constexpr int kFWR = kTileR + 2 * kHalo + 2, kFWZ = kTileZ + 2 * kHalo + 2;
constexpr int kJWR = kTileR + 2 * kHalo, kJWZ = kTileZ + 2 * kHalo;
// Row stride of the field window in shared memory.  A multiple of the 32
// banks would spare the half-cell staggered reads of adjacent rows (rows
// ci-1 and ci) their bank conflicts, measured at 1 % of the step, but costs
// 9 KB per block and with it the fourth resident block of the plasma step.
constexpr int kFWS = kFWZ;
static_assert(kFWS >= kFWZ, "field window rows hold the window");

// Grids are far below 2^31 nodes, so node indices are 32-bit.
__device__ __forceinline__ int node(const StepArgs& a, int i, int k) {
  return (i + 2) * a.ld + (k + 2);
}

// ---------------------------------------------------------------------------
// Gather (maxwellSolver.hpp:101-316) in normalised coordinates.  With
// x = r/dr, a component staggered by s_r in r has i = floor(x - s_r),
// u = x - s_r - i, and the ring-volume weights reduce to
//   s_r = 1/2: (1-u)(2i+1+u)/(2i+2),  u(2i+2+u)/(2i+4)
//   s_r = 0  : (1-u)(2i+u)/(2i+1),    u(2i+1+u)/(2i+3)
// (the denominators are the reference's CELL_VOLUME arguments after macro
// expansion); along z the weights are 1-v and v.

struct Stagger {
  int i;
  float u;
};

__device__ __forceinline__ Stagger half_shift(int c, float f) {  // floor(x - 1/2)
  Stagger s;
  if (f >= 0.5f) { s.i = c; s.u = f - 0.5f; } else { s.i = c - 1; s.u = f + 0.5f; }
  return s;
}

// Six field components (E_r, E_phi, E_z, H_r, H_phi, H_z) seen through a
// window: component c at node (i, k) is at(c, i, k).  GlobalFields is the
// grid itself (i0 = k0 = -2, ld = nz + 4, the allocation's plane stride);
// SharedFields a block's copy around its tile, whose strides are constants.
// Each also serves the radial reciprocal rows (recip_row / recip_int).
struct GlobalFields {
  const float* base;
  int plane, ld, i0, k0;
  const float4* rt;  // the global table, row i at rt[2 * (i + 2)]
  __device__ __forceinline__ const float* at(int c, int i, int k) const {
    return base + c * plane + (i - i0) * ld + (k - k0);
  }
  __device__ __forceinline__ int stride() const { return ld; }
  __device__ __forceinline__ float4 row(int i) const { return __ldg(rt + 2 * (i + 2)); }
  __device__ __forceinline__ float4 row_int(int i) const { return __ldg(rt + 2 * (i + 2) + 1); }
};

struct SharedFields {
  static constexpr int kLd = kFWS, kPlane = kFWR * kFWS;
  const float* base;
  int i0, k0;
  const float4* rt;  // the window's rows of the table, row i at rt[2 * (i - i0)]
  __device__ __forceinline__ const float* at(int c, int i, int k) const {
    return base + c * kPlane + (i - i0) * kLd + (k - k0);
  }
  __device__ __forceinline__ int stride() const { return kLd; }
  __device__ __forceinline__ float4 row(int i) const { return rt[2 * (i - i0)]; }
  __device__ __forceinline__ float4 row_int(int i) const { return rt[2 * (i - i0) + 1]; }
};

template <class V>
__device__ __forceinline__ float interp4(const V& fv, int c, int i, int k, float w0, float w1, float v) {
  const float* F = fv.at(c, i, k);
  const int ld = fv.stride();
  const float f00 = F[0], f10 = F[ld];
  const float f01 = F[1], f11 = F[ld + 1];
  return (f00 * w0 + f10 * w1) * (1.f - v) + (f01 * w0 + f11 * w1) * v;
}

template <class V>
__device__ __forceinline__ void gather(const StepArgs& a, const V& fv, int ci, float fr, int ck,
                                       float fz, float e[3], float b[3]) {
  const Stagger rh = half_shift(ci, fr), zh = half_shift(ck, fz);
  // ring-volume weights; the reciprocals of their denominators come from
  // the table (row ci: 1/(2ci+1), 1/(2ci+3); row rh.i: 1/(2i+2), 1/(2i+4)),
  // or in the fixed mode all are 1/(2x), the particle's cloud volume, so
  // that each component's weights sum to 1
  const float fi = (float)ci, fh = (float)rh.i, u = rh.u;
  float sn0, sn1, sh0, sh1;
  if (a.fixed) {
    sn0 = sn1 = sh0 = sh1 = 0.5f / (fi + fr);
  } else {
    const float4 tn = fv.row(ci), th = fv.row(rh.i);
    sn0 = tn.x; sn1 = tn.z; sh0 = th.y; sh1 = th.w;
  }
  const float n0 = (1.f - fr) * (2.f * fi + fr) * sn0, n1 = fr * (2.f * fi + 1.f + fr) * sn1;
  const float h0 = (1.f - u) * (2.f * fh + 1.f + u) * sh0, h1 = u * (2.f * fh + 2.f + u) * sh1;
  // E_r: (1/2, 0); E_z: (0, 1/2); E_phi: (0, 0)
  e[0] = interp4(fv, 0, rh.i, ck, h0, h1, fz);
  e[2] = interp4(fv, 2, ci, zh.i, n0, n1, zh.u);
  {
    const float* F = fv.at(1, ci, ck);
    const int ld = fv.stride();
    const float f00 = F[0], f10 = F[ld];
    const float f01 = F[1], f11 = F[ld + 1];
    const float t11 = f11 * n1 * fz;
    e[1] = (f00 * n0 + f10 * n1) * (1.f - fz) + f01 * n0 * fz;
    if (a.fixed) e[1] += t11; else e[2] += t11;  // maxwellSolver.hpp:313
  }
  // H_z: (1/2, 0); H_r: (0, 1/2); H_phi: (1/2, 1/2)
  b[2] = interp4(fv, 5, rh.i, ck, h0, h1, fz);
  b[0] = interp4(fv, 3, ci, zh.i, n0, n1, zh.u);
  b[1] = interp4(fv, 4, rh.i, zh.i, h0, h1, zh.u);
}

// ---------------------------------------------------------------------------
// Pushers (pusherBoris.cpp:23-151, pusherVay.cpp:22-114, pusherHC.cpp:23-117)

constexpr float kC2 = 9.0e16f;  // LIGHT_VEL^2

__device__ __forceinline__ float len2(const float v[3]) { return v[0] * v[0] + v[1] * v[1] + v[2] * v[2]; }

__device__ __forceinline__ bool gamma_of_v(float v2, float* g, DevStatus* st) {  // rel.cpp:24-45
  const float beta = v2 / kC2;
  if (beta > 1.f) { raise_error(st, kErrSuperluminal); return false; }
  *g = rsqrtf(1.f - beta);
  return true;
}

__device__ __forceinline__ float gamma_inv_of_u(float u2) { return rsqrtf(1.f + u2 / kC2); }  // rel.cpp:47-55

__device__ __forceinline__ bool push(const StepArgs& a, const float ein[3], const float bin[3],
                                     float v[3]) {
  float e[3], b[3];
  for (int c = 0; c < 3; ++c) b[c] = bin[c] * a.bk;
  if (a.pusher <= 2) {  // Boris: classic, adaptive, relativistic
    for (int c = 0; c < 3; ++c) e[c] = ein[c] * a.c2m;
    const bool rel = a.pusher == 2 || (a.pusher == 1 && len2(v) > (float)kRelLimit2);
    float gm = 1.f;
    if (rel) {
      if (!gamma_of_v(len2(v), &gm, a.st)) return false;
      for (int c = 0; c < 3; ++c) v[c] *= gm;
    }
    for (int c = 0; c < 3; ++c) v[c] += e[c];
    if (rel) {
      gm = gamma_inv_of_u(len2(v));
      for (int c = 0; c < 3; ++c) b[c] *= gm;
    }
    const float k2 = 2.f / (1.f + len2(b));
    const float t0 = v[0], t1 = v[1], t2 = v[2];
    v[0] = t0 + k2 * ((t1 - t0 * b[2] + t2 * b[0]) * b[2] - (t2 + t0 * b[1] - t1 * b[0]) * b[1]);
    v[1] = t1 + k2 * (-(t0 + t1 * b[2] - t2 * b[1]) * b[2] + (t2 + t0 * b[1] - t1 * b[0]) * b[0]);
    v[2] = t2 + k2 * ((t0 + t1 * b[2] - t2 * b[1]) * b[1] - (t1 - t0 * b[2] + t2 * b[0]) * b[0]);
    for (int c = 0; c < 3; ++c) v[c] += e[c];
    if (rel) {
      gm = gamma_inv_of_u(len2(v));
      for (int c = 0; c < 3; ++c) v[c] *= gm;
    }
    return true;
  }
  // Vay and Higuera-Cary work on u = gamma v; `fixed` measures u in units of c.
  const float cn = a.fixed ? 1.f / 3.0e8f : 1.f;
  float gm;
  if (!gamma_of_v(len2(v), &gm, a.st)) return false;
  float u[3] = {v[0] * gm * cn, v[1] * gm * cn, v[2] * gm * cn};
  float psm[3];
  if (a.pusher == 3) {
    const float ek = 2.f * a.c2m * cn;
    float up[3] = {u[0] + ein[0] * ek, u[1] + ein[1] * ek, u[2] + ein[2] * ek};
    const float gi = a.fixed ? rsqrtf(1.f + len2(u)) : gamma_inv_of_u(len2(u));
    up[0] += gi * (u[1] * b[2] - u[2] * b[1]);
    up[1] += gi * (u[2] * b[0] - u[0] * b[2]);
    up[2] += gi * (u[0] * b[1] - u[1] * b[0]);
    const float alpha0 = 1.f + len2(up), B2 = len2(b);
    const float s0 = alpha0 - B2;
    const float ub = up[0] * b[0] + up[1] * b[1] + up[2] * b[2];
    const float al = rsqrtf(0.5f * (s0 + sqrtf(s0 * s0 + 4.f * (B2 + ub * ub))));
    for (int c = 0; c < 3; ++c) b[c] *= al;
    const float s = 1.f / (1.f + len2(b));
    const float ab = up[0] * b[0] + up[1] * b[1] + up[2] * b[2];
    psm[0] = s * (up[0] + ab * b[0] + b[2] * up[1] - b[1] * up[2]);
    psm[1] = s * (up[1] + ab * b[1] + b[0] * up[2] - b[2] * up[0]);
    psm[2] = s * (up[2] + ab * b[2] + b[1] * up[0] - b[0] * up[1]);
  } else {
    const float ek = a.c2m * cn;
    for (int c = 0; c < 3; ++c) psm[c] = ein[c] * ek;
    float um[3] = {u[0] + psm[0], u[1] + psm[1], u[2] + psm[2]};
    const float gfm2 = 1.f + len2(um), B2 = len2(b);
    const float bu = b[0] * um[0] + b[1] * um[1] + b[2] * um[2];
    const float gi = rsqrtf(0.5f * (gfm2 - B2 + sqrtf((gfm2 - B2) * (gfm2 - B2) + 4.f * (B2 + bu * bu))));
    for (int c = 0; c < 3; ++c) b[c] *= gi;
    const float b2x = b[0] * b[0], b2y = b[1] * b[1], b2z = b[2] * b[2];
    const float bxy = b[0] * b[1], byz = b[1] * b[2], bzx = b[2] * b[0];
    const float idet = a.fixed ? 1.f / (1.f + b2x + b2y + b2z) : 1.f / (1.f + b2x + b2y + b2x);
    const float upx = ((1.f + b2x - b2y - b2z) * um[0] + 2.f * (bxy + b[2]) * um[1] +
                       2.f * (bzx - (a.fixed ? b[1] : b[2])) * um[2]) * idet;
    const float upy = (2.f * (bxy - b[2]) * um[0] + (1.f - b2x + b2y - b2z) * um[1] +
                       2.f * (byz + b[0]) * um[2]) * idet;
    const float upz = (2.f * (bzx + b[1]) * um[0] + 2.f * (byz - b[0]) * um[1] +
                       (1.f - b2x - b2y + b2z) * um[2]) * idet;
    psm[0] += upx; psm[1] += upy; psm[2] += upz;
  }
  if (a.fixed) {
    const float gi = rsqrtf(1.f + len2(psm)) * 3.0e8f;
    for (int c = 0; c < 3; ++c) v[c] = psm[c] * gi;
  } else {
    const float gi = gamma_inv_of_u(len2(psm));
    for (int c = 0; c < 3; ++c) v[c] = psm[c] * gi;
  }
  return true;
}

// ---------------------------------------------------------------------------
// Positions

__device__ __forceinline__ void renorm(int* c, float* f) {
  const float fl = floorf(*f);
  *c += (int)fl;
  *f -= fl;
  if (*f >= 1.f) { *f -= 1.f; *c += 1; }  // f just below an integer rounded up
}

// Mirror (c, f) about the wall at cell cw, offset 1/2: x' = 2 w - x.
__device__ __forceinline__ void mirror(int* c, float* f, int cw) {
  const float d = (float)(*c - cw) + (*f - 0.5f);
  float t = 0.5f - d;
  int nc = cw;
  renorm(&nc, &t);
  *c = nc;
  *f = t;
}

// SpecieP::reflect (specieP.cpp:493-607): the walls sit half a cell inside
// the domain; the reference's old-position bookkeeping inside the loop does
// not reach its outputs and is omitted.
__device__ __forceinline__ bool reflect(const StepArgs& a, int* ci, float* fr, int* ck, float* fz,
                                        float* vr, float* vz) {
  for (int guard = 0; guard < 64; ++guard) {
    const bool out_r = *ci > a.nr - 1 || (*ci == a.nr - 1 && *fr > 0.5f);
    const bool out_z = *ck > a.nz - 1 || (*ck == a.nz - 1 && *fz > 0.5f);
    const bool in_r = *ci < 0 || (*ci == 0 && *fr < 0.5f);
    const bool in_z = *ck < 0 || (*ck == 0 && *fz < 0.5f);
    if (!(out_r || out_z || in_r || in_z)) return true;
    if (out_r) { *vr = -*vr; mirror(ci, fr, a.nr - 1); }
    if (*ck > a.nz - 1 || (*ck == a.nz - 1 && *fz > 0.5f)) { *vz = -*vz; mirror(ck, fz, a.nz - 1); }
    if (*ci < 0 || (*ci == 0 && *fr < 0.5f)) {
      *vr = -*vr;
      mirror(ci, fr, 0);
      if (*ci == 0 && *fr < 0.5f) *fr = 0.5f;
    }
    if (*ck < 0 || (*ck == 0 && *fz < 0.5f)) {
      *vz = -*vz;
      mirror(ck, fz, 0);
      if (*ck == 0 && *fz < 0.5f) *fz = 0.5f;
    }
  }
  return false;
}

// ---------------------------------------------------------------------------
// Villasenor-Buneman current (currentVB.cpp:22-735) in normalised form.
//
// For a segment inside cell (i, k) from (i+ao, k+bo) to (i+an, k+bn), with
// dx = an-ao, dy = bn-bo, xo = i+ao, xn = i+an, t = dx/xo,
//   g(t) = ln(1+t)/t, h(t) = g - 1 + t/2, m(t) = 1/(1+t) - g,
// the reference's J_z and J_r increments (:46-108, :110-172) become
//   Jz[i]   += Qz dy A/i,      A = (1-ao)(2i+ao)/xo - dx/2 (1 + i(i+1)/xo^2) + i(i+1) h/xo
//   Jz[i+1] += Qz dy B/(i+1),  B = ao(2i+1+ao)/xo + dx/2 (1 + i(i+1)/xo^2) - i(i+1) h/xo
//   (i = 0: Jz[0] += 8 Qz dy (1 - ao - dx/2), Jz[1] += Qz dy (1 + ao + dx/2))
//   Jr[k]   += Qr/(i+1/2) [dx (b/2 - dy/4) + c/xo (dx b/xn + dy m)],      b = 1 - bo
//   Jr[k+1] += Qr/(i+1/2) [dx (bo/2 + dy/4) + c/xo (dx bo/xn - dy m)],   c = i(i+1)/2
// with Qz = q/(4 pi dr^2 dt) and Qr = q/(2 pi dr dz dt).

__device__ __forceinline__ void g_terms(float t, float* h, float* m) {
  if (fabsf(t) < 0.1f) {
    const float t2 = t * t;
    *h = t2 * (1.f / 3.f + t * (-0.25f + t * (0.2f + t * (-1.f / 6.f + t * (1.f / 7.f + t * (-0.125f))))));
    *m = t * (-0.5f + t * (2.f / 3.f + t * (-0.75f + t * (0.8f + t * (-5.f / 6.f + t * (6.f / 7.f + t * (-0.875f)))))));
  } else {
    const float g = log1pf(t) / t;
    *h = g - 1.f + 0.5f * t;
    *m = 1.f / (1.f + t) - g;
  }
}

// Where the current goes.  comp: 0 J_r, 1 J_phi, 2 J_z.
//
// SharedDep: the block's shared-memory window over nodes [i0, i0+kJWR) x
// [k0, k0+kJWZ); the caller has checked that every node the particle's
// deposit touches lies in it.
struct SharedDep {
  static constexpr int kPlane = kJWR * kJWZ;
  float* s;  // 3 planes of kJWR x kJWZ floats
  int i0, k0;
  // shared-window address of J_r at node (i, k)
  __device__ __forceinline__ unsigned addr(int i, int k) const {
    return (unsigned)__cvta_generic_to_shared(s + (i - i0) * kJWZ + (k - k0));
  }
  // a native shared-memory reduction at addr + OFF bytes
  template <int OFF>
  __device__ __forceinline__ static void red(unsigned addr, float v) {
    asm volatile("red.shared.add.f32 [%0+%1], %2;" ::"r"(addr), "n"(OFF), "f"(v) : "memory");
  }
  // byte offset of component comp at node (i + di, k + dk) from addr(i, k)
  template <int COMP, int DI, int DK>
  __device__ __forceinline__ static void red_at(unsigned addr, float v) {
    red<4 * (COMP * kPlane + DI * kJWZ + DK)>(addr, v);
  }
  __device__ __forceinline__ void add(int comp, int i, int k, float v) const {
    const unsigned p = (unsigned)__cvta_generic_to_shared(s + comp * kPlane + (i - i0) * kJWZ + (k - k0));
    asm volatile("red.shared.add.f32 [%0], %1;" ::"r"(p), "f"(v) : "memory");
  }
};

// GlobalDep: the grids themselves (J_r, J_phi, J_z are consecutive planes).
struct GlobalDep {
  float* J;
  int plane, ld;
  __device__ __forceinline__ void add(int comp, int i, int k, float v) const {
    atomicAdd(J + comp * plane + (i + 2) * ld + (k + 2), v);
  }
};

// simple_current_distribution for cell (i, k): start point (ao, bo) relative
// to that cell and the displacement (dx, dy).  Displacements are carried
// exactly (from the velocity, split by path fractions), never differenced
// from rounded offsets, so the MNZL test below means what it means in the
// reference's double arithmetic.  The terms below have no 1/dx or 1/dy
// (g_terms carries the logarithm as a series near 0), so the fixed mode
// deposits the segments the reference drops.
template <class D>
__device__ __forceinline__ void vb_simple(const StepArgs& a, const D& d, float q, int i, int k,
                                          float ao, float bo, float dx, float dy) {
  if (!a.fixed && (fabsf(dx) < a.mnzl_r || fabsf(dy) < a.mnzl_z)) return;  // currentVB.cpp:45-46
  const float fi = (float)i;
  const float xo = fi + ao, xn = xo + dx;
  const float ixo = 1.f / xo, ixn = 1.f / xn;
  float h, m;
  g_terms(dx * ixo, &h, &m);
  const float qz = q * a.qz * dy;
  const float cc = fi * (fi + 1.f);
  if (i >= 1) {
    const float lin = 0.5f * dx * (1.f + cc * ixo * ixo);
    const float hh = cc * h * ixo;
    const float A = (1.f - ao) * (2.f * fi + ao) * ixo - lin + hh;
    const float B = ao * (2.f * fi + 1.f + ao) * ixo + lin - hh;
    d.add(2, i, k, qz * A / fi);
    d.add(2, i + 1, k, qz * B / (fi + 1.f));
  } else {
    d.add(2, i, k, 8.f * qz * (1.f - ao - 0.5f * dx));
    d.add(2, i + 1, k, qz * (1.f + ao + 0.5f * dx));
  }
  const float qr = q * a.qr / (fi + 0.5f);
  const float bb = 1.f - bo;
  const float cx = 0.5f * cc * ixo;
  d.add(0, i, k, qr * (dx * (0.5f * bb - 0.25f * dy) + cx * (dx * bb * ixn + dy * m)));
  d.add(0, i, k + 1, qr * (dx * (0.5f * bo + 0.25f * dy) + cx * (dx * bo * ixn - dy * m)));
}

// strict_motion_distribution (:500-729).  (Xo, Yo) is the old point relative
// to the new cell, (dX, dY) the exact displacement, (Xn, Yn) the new offsets.
template <class D>
__device__ __forceinline__ void vb_strict(const StepArgs& a, const D& d, float q, int in, int kn,
                                          float Xo, float Yo, float dX, float dY, float Xn,
                                          float Yn) {
  const bool sr = fabsf(dX) < a.mnzl_r, sz = fabsf(dY) < a.mnzl_z;
  if (sr && sz) return;
  const float fi = (float)in;
  const float xn = fi + Xn;
  const int ko = kn + (int)floorf(Yo), io = in + (int)floorf(Xo);
  if (sr) {  // axial motion :524-604 (the J_r overwrite is not reproduced here)
    const float qz = q * a.qz;
    const float lo = (in == 0) ? 8.f * qz * Xn * (1.f - Xn) / xn
                               : qz * (1.f - Xn) * (2.f * fi + Xn) / (fi * xn);
    const float up = qz * Xn * (2.f * fi + 1.f + Xn) / ((fi + 1.f) * xn);
    switch (kn - ko) {
      case 0:
        d.add(2,in, kn, lo * dY);
        d.add(2,in + 1, kn, up * dY);
        break;
      case 1: {  // crossed y = kn: first part in row kn-1
        const float d1 = 0.f - Yo, d2 = dY - d1;
        d.add(2,in, kn - 1, lo * d1);
        d.add(2,in + 1, kn - 1, up * d1);
        d.add(2,in, kn, lo * d2);
        d.add(2,in + 1, kn, up * d2);
        break;
      }
      case -1: {  // crossed y = kn+1: first part in row kn+1
        const float d1 = 1.f - Yo, d2 = dY - d1;
        d.add(2,in, kn + 1, lo * d1);
        d.add(2,in + 1, kn + 1, up * d1);
        d.add(2,in, kn, lo * d2);
        d.add(2,in + 1, kn, up * d2);
        break;
      }
      default: break;
    }
    return;
  }
  if (!sz) return;
  // radial motion :607-728; bracket/dr in normalised units, wj = q Qr/(2(i+1/2)) * bracket
  const float xo = fi + Xo;
  const float ldz = 1.f - Yn, rdz = Yn;
  auto put = [&](int i, float br) {
    const float wj = q * a.qr * 0.5f / ((float)i + 0.5f) * br;
    d.add(0,i, kn, wj * ldz);
    d.add(0,i, kn + 1, wj * rdz);
  };
  const float dr2 = a.dr_m * a.dr_m;
  switch (in - io) {
    case 0:
      put(in, dX * (1.f + fi * (fi + 1.f) / (xo * xn)));
      break;
    case 1: {
      const float d1 = 0.f - Xo, d2 = dX - d1;  // to and from the boundary x = in
      put(in - 1, d1 * (1.f + (fi - 1.f) / xo));
      const float r0 = fi + 0.5f;
      const float br = a.fixed ? d2 * (1.f + (fi + 1.f) / xn)
                               : d2 - r0 * r0 / xn + r0 * r0 * dr2 / fi + 0.25f / xn - 0.25f / fi;  // :673
      put(in, br);
      break;
    }
    case -1: {
      const float d1 = 1.f - Xo, d2 = dX - d1;  // to and from the boundary x = in+1
      put(in + 1, d1 * (1.f + (fi + 2.f) / xo));
      const float r0 = fi + 0.5f;
      const float br = a.fixed ? d2 * (1.f + fi / xn)
                               : d2 - r0 * r0 / xn + r0 * r0 * dr2 / (fi + 1.f) + 0.25f / xn - 0.25f / (fi + 1.f);  // :714
      put(in, br);
      break;
    }
    default: break;
  }
}

// azimuthal_current_distribution (:398-498): J_phi from the mid-point, in
// the cell of the new position (a, b may lie outside [0, 1)).
template <class D>
__device__ __forceinline__ void vb_azimuthal(const StepArgs& a, const D& d, float q, float vphi,
                                             int in, int kn, float Xm, float Ym) {
  const float fi = (float)in;
  const float xm = fi + Xm;
  const float qp = q * a.qp * vphi / xm;
  const float w0 = (1.f - Xm) * (2.f * fi + Xm) / (2.f * fi + 1.f);
  const float w1 = Xm * (2.f * fi + 1.f + Xm) / (2.f * fi + 2.f);
  const bool i0 = in >= 0 && in < a.nr, i1 = in + 1 < a.nr;
  const bool k0 = kn >= 0 && kn < a.nz, k1 = kn + 1 < a.nz;
  // the halo of J_phi is cleared before the rz deposit (currentVB.cpp:177)
  if (i0 && k0) d.add(1,in, kn, qp * w0 * (1.f - Ym));
  if (i1 && k0) d.add(1,in + 1, kn, qp * w1 * (1.f - Ym));
  if (i0 && k1) d.add(1,in, kn + 1, qp * w0 * Ym);
  if (i1 && k1) d.add(1,in + 1, kn + 1, qp * w1 * Ym);
}

// rz_current_distribution (:175-396).  (Xo, Yo): old point relative to the
// new cell (in, kn); (dX, dY): the exact displacement; (Xn, Yn): the new
// offsets.  Crossings split the displacement by path fractions.
template <class D>
__device__ __forceinline__ bool vb_rz(const StepArgs& a, const D& d, float q, int in, int kn,
                                      float Xo, float Yo, float dX, float dY, float Xn, float Yn) {
  const int di = (int)floorf(Xo), dk = (int)floorf(Yo);  // old cell - new cell
  if (abs(di) > 1 || (a.fixed && abs(dk) > 1)) return false;
  if (fabsf(dX) < a.mnzl_r || fabsf(dY) < a.mnzl_z) {
    vb_strict(a, d, q, in, kn, Xo, Yo, dX, dY, Xn, Yn);
    return true;
  }
  const int res = abs(di) + abs(dk);
  if (res > 2 || (res == 2 && di == 0)) return true;  // the reference deposits nothing
  // The path is cut at its cell-boundary crossings into nseg <= 3 parts, part
  // s running over path fractions [f[s], f[s+1]] inside cell (in+ci[s], kn+ck[s]).
  float f[4] = {0.f, 1.f, 1.f, 1.f};
  int ci[3] = {0, 0, 0}, ck[3] = {0, 0, 0};
  int nseg = 1;
  if (res == 1) {
    // radial crossing at x = in+1 (from outside) or x = in; axial likewise
    f[1] = (di != 0) ? ((di > 0 ? 1.f : 0.f) - Xo) / dX : ((dk > 0 ? 1.f : 0.f) - Yo) / dY;
    ci[0] = di; ck[0] = dk;
    nseg = 2;
  } else if (res == 2) {
    const float xb = di > 0 ? 1.f : 0.f, yb = dk > 0 ? 1.f : 0.f;
    const float fx = (xb - Xo) / dX, fy = (yb - Yo) / dY;  // path fractions of the two crossings
    if (fx == fy) return true;  // through the corner: the reference deposits nothing (:278-300)
    ci[0] = di; ck[0] = dk;
    if (fx < fy) { f[1] = fx; f[2] = fy; ci[1] = 0; ck[1] = dk; }   // radial boundary first
    else         { f[1] = fy; f[2] = fx; ci[1] = di; ck[1] = 0; }   // axial boundary first
    nseg = 3;
  }
  for (int s = 0; s < nseg; ++s) {
    const float f0 = f[s], f1 = f[s + 1];
    vb_simple(a, d, q, in + ci[s], kn + ck[s], Xo + f0 * dX - ci[s], Yo + f0 * dY - ck[s],
              (f1 - f0) * dX, (f1 - f0) * dY);
  }
  return true;
}

// ---------------------------------------------------------------------------

// ---------------------------------------------------------------------------
// ZigZag current (currentZigZag.cpp:22-136) with the reference's metre-valued
// weights W = (mean position - cell edge) in metres.

template <class D>
__device__ __forceinline__ void zigzag(const StepArgs& a, const D& d, float qw, float vphi,
                                       int in, int kn, float Xo, float Yo, float Xn, float Yn) {
  const int io = (int)floorf(Xo), ko = (int)floorf(Yo);  // relative to the new cell
  const int imid = in + (int)floorf(0.5f * (Xo + Xn));
  const float oov = a.zz_vol / (2.f * (float)imid + 1.f);
  const float ro = ((float)in + Xo) * a.dr_m, rn = ((float)in + Xn) * a.dr_m;
  const float F_phi = qw * vphi;
  const float W_phi = vphi * a.dt_s / (2.f * 3.14159265f * (ro + rn));
  const float xr = fminf((float)min(io, 0) + 1.f, fmaxf((float)max(io, 0), 0.5f * (Xo + Xn)));
  const float yr = fminf((float)min(ko, 0) + 1.f, fmaxf((float)max(ko, 0), 0.5f * (Yo + Yn)));
  const float cod = qw / a.dt_s;
  const float F_r1 = cod * a.dr_m * (xr - Xo), F_r2 = cod * a.dr_m * (Xn - xr);
  const float F_z1 = cod * a.dz_m * (yr - Yo), F_z2 = cod * a.dz_m * (Yn - yr);
  const float W_r1 = a.dr_m * (0.5f * (Xo + xr) - (float)io), W_r2 = a.dr_m * (0.5f * (Xn + xr));
  const float W_z1 = a.dz_m * (0.5f * (Yo + yr) - (float)ko), W_z2 = a.dz_m * (0.5f * (Yn + yr));
  const float mWr1 = 1.f - W_r1, mWr2 = 1.f - W_r2, mWz1 = 1.f - W_z1, mWz2 = 1.f - W_z2, mWp = 1.f - W_phi;
  const int ia = in + io, ka = kn + ko;
  d.add(0,ia, ka, oov * F_r1 * mWp * mWz1 + oov * F_r1 * W_phi * mWz1);
  d.add(0,ia, ka + 1, oov * F_r1 * mWp * W_z1 + oov * F_r1 * W_phi * W_z1);
  d.add(0,in, kn, oov * F_r2 * mWp * mWz2 + oov * F_r2 * W_phi * mWz2);
  d.add(0,in, kn + 1, oov * F_r2 * mWp * W_z2 + oov * F_r2 * W_phi * W_z2);
  d.add(1,in, kn, oov * F_phi * mWr2 * mWz2);
  d.add(1,in, kn + 1, oov * F_phi * mWr2 * W_z1);
  d.add(1,in + 1, kn, oov * F_phi * W_r2 * mWz2);
  d.add(1,in + 1, kn + 1, oov * F_phi * W_r2 * W_z2);
  d.add(2,ia, ka, oov * F_z1 * mWr1 * mWp + oov * F_z1 * mWr1 * W_phi);
  d.add(2,ia + 1, ka, oov * F_z1 * W_r1 * mWp + oov * F_z1 * W_r1 * W_phi);
  d.add(2,in, kn, oov * F_z2 * mWr2 * mWp + oov * F_z2 * mWr2 * W_phi);
  d.add(2,in + 1, kn, oov * F_z2 * W_r2 * mWp + oov * F_z2 * W_r2 * W_phi);
}

// ---------------------------------------------------------------------------

// What the current deposit of one moved particle needs: the new cell and
// offsets, the old point relative to the new cell, the exact displacement.
struct Moved {
  int ci, ck;      // new cell
  int ci0, ck0;    // old cell
  float fr, fz;    // new offsets
  float Xo, Yo;    // old point relative to the new cell
  float dX, dY;    // displacement (straight line to the mirrored point after a reflection)
  float w, vphi;
};

// One macroparticle after its gather: push, move, reflect, bind and the
// runaway test (pusher*.cpp, specieP.cpp:482-491, 609-640, beamP.cpp:159-177,
// SMB.cpp:252-337).  Writes the particle back; returns false if it left the
// domain (no current) and fills `m` otherwise.
// One particle's slot contents, loaded ahead of its turn.
struct Slot {
  int cell;
  float fr, fz, vr, vphi, vz, w;
};

__device__ __forceinline__ Slot load_slot(const SpeciesF32Buffers& b, size_t j) {
  return Slot{b.cell[j], b.off_r[j], b.off_z[j], b.vr[j], b.vphi[j], b.vz[j], b.w[j]};
}

__device__ __forceinline__ bool advance_one(const StepArgs& a, const SpeciesF32Buffers& b,
                                            size_t j, const Slot& p, const float e[3],
                                            const float bb[3], Moved* m) {
  const int ci0 = cell_r_of(p.cell), ck0 = cell_z_of(p.cell);
  const float fr0 = p.fr, fz0 = p.fz;
  float v[3] = {p.vr, p.vphi, p.vz};
  if (!a.pushed && !push(a, e, bb, v)) return false;
  if (a.pushed && a.xform && ci0 >= 0 && ck0 >= 0 && ci0 < a.nr && ck0 < a.nz) {
    const size_t c = (size_t)ci0 * a.nz + ck0;
    if (a.xflag[c] == 1) {  // the learned collision step's transform of the cell
      const double* t = a.xform + c * 12 + a.xoff;
      for (int q = 0; q < 3; ++q) v[q] = (float)(t[q] + ((double)v[q] - t[q]) * t[3 + q]);
    }
  }
  // mover_cylindrical + back_position_to_rz: x' = sqrt((x+dx)^2 + dy^2),
  // taken as dx + dy^2/(X + x') to keep the displacement's precision.
  const float dx = v[0] * a.dt_dr, dyp = v[1] * a.dt_dr, dzz = v[2] * a.dt_dz;
  const float X = (float)ci0 + fr0 + dx;
  const float xn = sqrtf(X * X + dyp * dyp);
  const float sn = dyp / xn;
  int ci = ci0, ck = ck0;
  // far from the axis x' - x = dx + dy^2/(X + x'); near it (or across it,
  // X < 0) x' itself is small and exact enough
  float dX = (X > 0.5f) ? dx + dyp * dyp / (X + xn) : xn - ((float)ci0 + fr0);  // exact displacement
  float dY = dzz;
  float fr = fr0 + dX;
  float fz = fz0 + dY;
  renorm(&ci, &fr);
  renorm(&ck, &fz);
  bool reflected = false;
  if (a.is_beam) {  // BeamP::reflect beamP.cpp:159-177
    if (ci < 0 || (ci == 0 && fr < 0.5f)) { mirror(&ci, &fr, 0); v[0] = -v[0]; reflected = true; }
  } else if (ci < 1 || ci > a.nr - 2 || ck < 1 || ck > a.nz - 2) {
    // only cells next to a wall can cross one (walls at x = 1/2 and nr - 1/2)
    const int c0 = ci, k0 = ck;
    const float f0 = fr, g0 = fz;
    if (!reflect(a, &ci, &fr, &ck, &fz, &v[0], &v[2])) raise_error(a.st, kErrReflectLoop);
    reflected = ci != c0 || ck != k0 || fr != f0 || fz != g0;
  }
  // After a reflection the deposit follows the straight line to the mirrored
  // point.  In the fixed mode every deposit takes its displacement from the
  // stored (rounded) offsets, so that the charge its current moves is the
  // charge the new position holds (the difference of two close offsets is
  // exact), not the unrounded move.
  if (reflected || a.fixed) {
    dX = (float)(ci - ci0) + (fr - fr0);
    dY = (float)(ck - ck0) + (fz - fz0);
  }
  const float cs = sqrtf(1.f - sn * sn);  // back_velocity_to_rz :624-640
  const float vr2 = cs * v[0] - sn * v[1];
  const float vp2 = sn * v[0] + cs * v[1];
  b.vr[j] = vr2;
  b.vphi[j] = vp2;
  b.vz[j] = v[2];
  if (ci < 0 || ck < 0 || ci >= a.nr || ck >= a.nz) {  // runaway collector SMB.cpp:252-337
    b.cell[j] = kDeadCell;
    atomicAdd(&a.st->removed, 1ull);
    atomicAdd(&a.st->dead_slots, 1ull);
    return false;
  }
  b.cell[j] = pack_cell(ci, ck);
  b.off_r[j] = fr;
  b.off_z[j] = fz;
  m->ci = ci; m->ck = ck; m->ci0 = ci0; m->ck0 = ck0;
  m->fr = fr; m->fz = fz;
  m->Xo = (float)(ci0 - ci) + fr0;
  m->Yo = (float)(ck0 - ck) + fz0;
  m->dX = dX; m->dY = dY;
  m->w = p.w;
  m->vphi = vp2;
  return true;
}

// The current of one moved particle (CUR: 0 Villasenor-Buneman, 1 ZigZag).
template <int CUR, class D>
__device__ __forceinline__ void deposit(const StepArgs& a, const D& d, const Moved& m) {
  if (CUR == 1) {
    zigzag(a, d, m.w, m.vphi, m.ci, m.ck, m.Xo, m.Yo, m.fr, m.fz);
  } else {
    vb_azimuthal(a, d, m.w, m.vphi, m.ci, m.ck, m.Xo + 0.5f * m.dX, m.Yo + 0.5f * m.dY);
    if (!vb_rz(a, d, m.w, m.ci, m.ck, m.Xo, m.Yo, m.dX, m.dY, m.fr, m.fz))
      atomicAdd(&a.st->move_errors, 1ull);
  }
}

// The Villasenor-Buneman deposit of the common case: the particle stayed in
// an interior cell (1 <= i <= nr-2, k <= nz-2) and moved more than MNZL both
// ways.  It is vb_azimuthal + vb_rz (one segment, vb_simple) with the row
// reciprocals from the table and every address an offset from one base.
__device__ __forceinline__ void vb_fast(const StepArgs& a, const SharedFields& sv, const SharedDep& d,
                                        float q, float vphi, int in, int kn, float Xo, float Yo,
                                        float dX, float dY) {
  const float fi = (float)in;
  const float4 tr = sv.row(in), ti = sv.row_int(in);
  const unsigned p = d.addr(in, kn);
  // J_phi from the mid-point (currentVB.cpp:398-498)
  const float Xm = Xo + 0.5f * dX, Ym = Yo + 0.5f * dY;
  const float qp = q * a.qp * vphi / (fi + Xm);
  const float w0 = (1.f - Xm) * (2.f * fi + Xm) * tr.x;
  const float w1 = Xm * (2.f * fi + 1.f + Xm) * tr.y;
  SharedDep::red_at<1, 0, 0>(p, qp * w0 * (1.f - Ym));
  SharedDep::red_at<1, 1, 0>(p, qp * w1 * (1.f - Ym));
  SharedDep::red_at<1, 0, 1>(p, qp * w0 * Ym);
  SharedDep::red_at<1, 1, 1>(p, qp * w1 * Ym);
  // J_z and J_r of the segment (currentVB.cpp:22-173)
  const float xo = fi + Xo, xn = xo + dX;
  const float ixo = 1.f / xo, ixn = 1.f / xn;
  float h, m;
  g_terms(dX * ixo, &h, &m);
  const float qz = q * a.qz * dY;
  const float cc = fi * (fi + 1.f);
  const float lin = 0.5f * dX * (1.f + cc * ixo * ixo);
  const float hh = cc * h * ixo;
  const float A = (1.f - Xo) * (2.f * fi + Xo) * ixo - lin + hh;
  const float B = Xo * (2.f * fi + 1.f + Xo) * ixo + lin - hh;
  SharedDep::red_at<2, 0, 0>(p, qz * A * ti.x);
  SharedDep::red_at<2, 1, 0>(p, qz * B * ti.y);
  const float qr = q * a.qr * ti.z;
  const float bb = 1.f - Yo, cx = 0.5f * cc * ixo;
  SharedDep::red_at<0, 0, 0>(p, qr * (dX * (0.5f * bb - 0.25f * dY) + cx * (dX * bb * ixn + dY * m)));
  SharedDep::red_at<0, 0, 1>(p, qr * (dX * (0.5f * Yo + 0.25f * dY) + cx * (dX * Yo * ixn - dY * m)));
}

__device__ __forceinline__ bool cell_in_halo(const StepArgs& a, int cell) {
  const int ci = cell_r_of(cell), ck = cell_z_of(cell);
  if (ci < -1 || ci > a.nr || ck < -1 || ck > a.nz) {  // the gather would leave the halo
    raise_error(a.st, kErrOutOfGrid);
    return false;
  }
  return true;
}

__device__ __forceinline__ GlobalFields global_fields(const StepArgs& a) {
  return GlobalFields{a.Er, a.plane, a.ld, -2, -2, a.rt};
}

__device__ __forceinline__ GlobalDep global_dep(const StepArgs& a) {
  return GlobalDep{a.Jr, a.plane, a.ld};
}

// Particles [j0, j1), one per thread, fields and current on the global grid
// (particles appended since the last tile sort).
template <int CUR>
__global__ void __launch_bounds__(kThreads) step_flat_kernel(StepArgs a, SpeciesF32Buffers b,
                                                             size_t j0, size_t j1) {
  const size_t j = j0 + blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= j1) return;
  const Slot p = load_slot(b, j);
  if (p.cell < 0 || !cell_in_halo(a, p.cell)) return;
  float e[3] = {0.f, 0.f, 0.f}, bb[3] = {0.f, 0.f, 0.f};
  if (!a.pushed) gather(a, global_fields(a), cell_r_of(p.cell), p.fr, cell_z_of(p.cell), p.fz, e, bb);
  Moved m;
  if (advance_one(a, b, j, p, e, bb, &m)) deposit<CUR>(a, global_dep(a), m);
}

// The push alone, one thread per slot, fields from the global grid: the first half of a step whose collisions act between the push and
// the move (SMB::advance_particles, SMB.cpp:1289-1293); the step kernels
// then run with StepArgs::pushed set.
__device__ __forceinline__ void push_slot(const StepArgs& a, const SpeciesF32Buffers& b, size_t j, const Slot& p) {
  if (p.cell < 0 || !cell_in_halo(a, p.cell)) return;
  float e[3], bb[3];
  gather(a, global_fields(a), cell_r_of(p.cell), p.fr, cell_z_of(p.cell), p.fz, e, bb);
  float v[3] = {p.vr, p.vphi, p.vz};
  if (!push(a, e, bb, v)) return;
  b.vr[j] = v[0];
  b.vphi[j] = v[1];
  b.vz[j] = v[2];
}

// Slots [j0, n).
__global__ void __launch_bounds__(kThreads) push_flat_kernel(StepArgs a, SpeciesF32Buffers b, size_t j0, size_t n) {
  const size_t j = j0 + blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= n) return;
  push_slot(a, b, j, load_slot(b, j));
}

// One particle of a tile block: gather from the shared window (or the grid
// when it drifted out), push and move, deposit into the shared current
// window (or the grid when a node it touches lies outside).
template <int CUR>
__device__ __forceinline__ void tile_particle(const StepArgs& a, const SpeciesF32Buffers& b,
                                              unsigned j, const Slot& p, const SharedFields& sv,
                                              const SharedDep& sd) {
  if (p.cell < 0) return;
  const int ci0 = cell_r_of(p.cell), ck0 = cell_z_of(p.cell);
  // the gather reads nodes ci-1 .. ci+1, ck-1 .. ck+1
  const bool inside = ci0 - 1 >= sv.i0 && ci0 + 2 < sv.i0 + kFWR && ck0 - 1 >= sv.k0 &&
                      ck0 + 2 < sv.k0 + kFWZ;
  if (!inside && !cell_in_halo(a, p.cell)) return;
  bool slow = !inside;
  float ef[3] = {0.f, 0.f, 0.f}, bf[3] = {0.f, 0.f, 0.f};
  if (a.pushed) {
  } else if (inside) {
    gather(a, sv, ci0, p.fr, ck0, p.fz, ef, bf);
  } else {
    gather(a, global_fields(a), ci0, p.fr, ck0, p.fz, ef, bf);
  }
  Moved m;
  if (!advance_one(a, b, j, p, ef, bf, &m)) {
    if (slow) atomicAdd(b.drift, 1u);
    return;
  }
  // every node a deposit touches lies in [min(old, new) cell, max + 1] per axis
  const int lo_r = min(m.ci0, m.ci), hi_r = max(m.ci0, m.ci) + 1;
  const int lo_z = min(m.ck0, m.ck), hi_z = max(m.ck0, m.ck) + 1;
  if (lo_r >= sd.i0 && hi_r < sd.i0 + kJWR && lo_z >= sd.k0 && hi_z < sd.k0 + kJWZ) {
    if (CUR == 0 && m.ci == m.ci0 && m.ck == m.ck0 && m.ci >= 1 && m.ci <= a.nr - 2 &&
        m.ck <= a.nz - 2 && fabsf(m.dX) >= a.mnzl_r && fabsf(m.dY) >= a.mnzl_z)
      vb_fast(a, sv, sd, m.w, m.vphi, m.ci, m.ck, m.Xo, m.Yo, m.dX, m.dY);
    else
      deposit<CUR>(a, sd, m);
  } else {
    deposit<CUR>(a, global_dep(a), m);
    slow = true;
  }
  if (slow) atomicAdd(b.drift, 1u);
}

// Shared memory of a tile block: the field window, then the current window.
constexpr size_t kTileSmemBytes = sizeof(float) * (6 * kFWR * kFWS + 3 * kJWR * kJWZ) + sizeof(float4) * 2 * kFWR;
static_assert((6 * kFWR * kFWS + 3 * kJWR * kJWZ) % 4 == 0, "the table rows need 16-byte alignment");

// One block per tile (or gridDim.y blocks sharing a crowded tile): the
// tile's particles (grouped by the last sort) gather from a shared copy of
// the fields around the tile and deposit into a shared current window that
// is added to the global grid once at the end.  Particles that drifted
// beyond the windows use the global grid.
// PUSH, BEAM, FIX >= 0 fix a.pusher, a.is_beam, a.fixed at compile time
// (the local copy's constant fields fold every test of them away); -1
// leaves them to the arguments.  The specialised ZigZag instance fits 48
// registers without spilling and runs 5 blocks per SM (shared memory allows
// 5); the others keep 64 registers and 4 blocks.
// PUSH = kMoveOnly: the instance for steps whose push ran already (with
// collisions), the pusher's code left out.
constexpr int kMoveOnly = -2;
template <int CUR, int PUSH = -1, int BEAM = -1, int FIX = -1>
__global__ void __launch_bounds__(kThreads, (CUR == 1 && PUSH != -1) ? 5 : 4)
    step_tiled_kernel(StepArgs args, SpeciesF32Buffers b,
                                                                 TileGrid tg) {
  StepArgs a = args;
  if (PUSH >= 0) {  // the specialised instances run whole steps only
    a.pusher = PUSH;
    a.pushed = 0;
    a.xform = nullptr;
  }
  if (PUSH == kMoveOnly) a.pushed = 1;
  if (BEAM >= 0) a.is_beam = BEAM;
  if (FIX >= 0) a.fixed = FIX;
  extern __shared__ float smem[];
  const int t = blockIdx.x;
  // blockIdx.y of the np blocks sharing the tile (the blocks per tile of the
  // last sort, on the device, up to the gridDim.y launched) takes every
  // np-th run of blockDim.x
  const unsigned np = max(1u, min(b.sort_info[2], gridDim.y));
  if (blockIdx.y >= np) return;
  const unsigned s = b.tile_start[t] + blockIdx.y * blockDim.x, e = b.tile_start[t + 1];
  if (s >= e) return;
  const int tr = t / tg.ntz, tz = t - tr * tg.ntz;
  const int r0 = tr * kTileR, z0 = tz * kTileZ;  // first cell of the tile
  const int fi0 = r0 - kHalo - 1, fk0 = z0 - kHalo - 1;  // field window origin (node)
  const int ji0 = r0 - kHalo, jk0 = z0 - kHalo;          // current window origin (node)
  float* sF = smem;
  float* sJ = smem + 6 * kFWR * kFWS;
  // load the field window, one row of one component per warp pass (nodes
  // outside the halo-padded grid read as 0)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int row = warp; row < 6 * kFWR; row += kThreads / 32) {
    const int c = row / kFWR, i = fi0 + (row - c * kFWR);
    const bool row_ok = i >= -2 && i < a.nr + 2;
    const float* src = a.Er + c * a.plane + (i + 2) * a.ld + 2;
    for (int q = lane; q < kFWZ; q += 32) {
      const int k = fk0 + q;
      sF[row * kFWS + q] = (row_ok && k >= -2 && k < a.nz + 2) ? __ldg(src + k) : 0.f;
    }
  }
  for (int q = threadIdx.x; q < 3 * kJWR * kJWZ; q += kThreads) sJ[q] = 0.f;
  // the window's rows of the radial reciprocal table (rows -2 .. nr+2 exist)
  float4* sR = reinterpret_cast<float4*>(sJ + 3 * kJWR * kJWZ);
  if (threadIdx.x < 2 * kFWR) {
    const int i = fi0 + (int)(threadIdx.x >> 1);
    sR[threadIdx.x] = (i >= -2 && i <= a.nr + 2) ? __ldg(a.rt + 2 * (i + 2) + (threadIdx.x & 1))
                                                 : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __syncthreads();
  const SharedFields sv{sF, fi0, fk0, sR};
  const SharedDep sd{sJ, ji0, jk0};
  // each thread walks its slots with the next slot's loads in flight
  const unsigned stride = np * blockDim.x;
  unsigned j = s + threadIdx.x;
  Slot cur{};
  if (j < e) cur = load_slot(b, j);
  while (j < e) {
    const unsigned jn = j + stride;
    Slot nxt{};
    if (jn < e) nxt = load_slot(b, jn);
    tile_particle<CUR>(a, b, j, cur, sv, sd);
    cur = nxt;
    j = jn;
  }
  __syncthreads();
  // add the window to the grid, one row of one component per warp pass
  for (int row = warp; row < 3 * kJWR; row += kThreads / 32) {
    const int c = row / kJWR, i = ji0 + (row - c * kJWR);
    float* dst = a.Jr + c * a.plane + (i + 2) * a.ld + 2;  // J_r, J_phi, J_z are consecutive planes
    for (int q = lane; q < kJWZ; q += 32) {
      const float v = sJ[row * kJWZ + q];
      if (v != 0.f) atomicAdd(dst + jk0 + q, v);
    }
  }
}

}  // namespace f32

inline f32::StepArgs f32_step_args(const F32Step& st, double charge, double mass, int is_beam) {
  const GridGeom& g = st.g;
  f32::StepArgs a;
  a.g = g;
  a.Er = st.fld[0]; a.Ep = st.fld[1]; a.Ez = st.fld[2];
  a.Hr = st.fld[3]; a.Hp = st.fld[4]; a.Hz = st.fld[5];
  a.Jr = st.fld[9]; a.Jp = st.fld[10]; a.Jz = st.fld[11];
  a.nr = g.nr; a.nz = g.nz; a.ld = g.ld;
  a.plane = st.plane;
  a.dt_dr = (float)(g.dt / g.dr);
  a.dt_dz = (float)(g.dt / g.dz);
  const double c2m = charge * g.dt / (2 * mass);
  a.c2m = (float)c2m;
  a.bk = (float)(c2m * kMagnConst);
  a.qz = (float)(charge / (4.0 * kPi * g.dr * g.dr * g.dt));
  a.qr = (float)(charge / (2.0 * kPi * g.dr * g.dz * g.dt));
  a.qp = (float)(charge / (2.0 * kPi * g.dz * g.dr * g.dr));
  a.mnzl_r = (float)(kMnzl / g.dr);
  a.mnzl_z = (float)(kMnzl / g.dz);
  a.dr_m = (float)g.dr; a.dz_m = (float)g.dz; a.dt_s = (float)g.dt;
  // ZigZag: 1/(PI dz dr^2) with the species charge folded in
  a.zz_vol = (float)(charge / (kPi * g.dz * g.dr * g.dr));
  a.pusher = st.pusher; a.current = st.current; a.fixed = st.fixed; a.is_beam = is_beam;
  a.pushed = st.pushed;
  a.xform = st.pushed ? st.xform : nullptr;
  a.xflag = st.xflag;
  a.xoff = 0;
  a.rt = st.recip;
  a.st = st.status;
  return a;
}

}  // namespace pcg
