// pcg_f32_pair.cuh — the plasma step of the single-precision path, two
// macroparticles per thread in Blackwell's packed FP32 pairs.
//
// Two instances: the relativistic Boris pusher with the Villasenor-Buneman
// current, and the Vay pusher with the ZigZag current.
//
// The common case of a sorted plasma tile is a particle that stays in an
// interior cell during the step: no wall, no cell crossing, a single
// Villasenor-Buneman segment.  For that case each thread takes two slots of
// its tile (j and j + stride) and runs gather, relativistic Boris push,
// move, rotation and the in-cell deposit with every add, multiply and
// fused multiply-add on a float2 {particle 0, particle 1} (FADD2, FMUL2,
// FFMA2: one instruction for both).  Reciprocals and square roots are the
// hardware approximations (rcp/rsqrt/sqrt.approx, about 1 ulp).  A pair of
// which either particle leaves that case (dead slot, a cell next to a wall
// or outside the block's windows, a cell crossing, motion below the
// reference's 1e-15 m threshold, a long in-cell step) is handed whole to
// the scalar tile_particle of pcg_f32_step.cuh, which covers every case.
//
// Formulas are those of pcg_f32_step.cuh (gather, push, vb_fast) with the
// in-cell identities Xo = fr0, Yo = fz0 substituted: the gather's radial
// weight numerators (1-x)(2i+x) and x(2i+1+x) are also the numerators of
// the deposit's J_z terms, and 1/(i+1/2) = 2/(2i+1).  References:
// maxwellSolver.hpp:101-316 (gather), pusherBoris.cpp:23-151 (push),
// specieP.cpp:482-491, 609-640 (move, rotation), currentVB.cpp:22-173,
// 398-498 (deposit).
#pragma once

#include "pcg_f32_step.cuh"


namespace pcg {
namespace f32 {
namespace pk {

// packed FP32 pair arithmetic (sm_100: one instruction for both lanes).
// Subtraction is a fused multiply-add by -1 so that no operand needs a
// separate negation.
__device__ __forceinline__ float2 bc(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sub(float2 a, float2 b) { return __ffma2_rn(b, bc(-1.f), a); }
__device__ __forceinline__ float2 one_minus(float2 a) { return __ffma2_rn(a, bc(-1.f), bc(1.f)); }

__device__ __forceinline__ float rcp(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rsq(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float sqr(float x) {
  float y;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float2 rcp(float2 x) { return make_float2(rcp(x.x), rcp(x.y)); }
__device__ __forceinline__ float2 rsq(float2 x) { return make_float2(rsq(x.x), rsq(x.y)); }
__device__ __forceinline__ float2 sqr(float2 x) { return make_float2(sqr(x.x), sqr(x.y)); }

// Shared-memory access at a byte offset from a 32-bit shared address.  The
// loads read the field window and the tables, which no thread writes while
// particles are processed.
template <int OFF>
__device__ __forceinline__ float lds(unsigned addr) {
  float v;
  asm("ld.shared.f32 %0, [%1+%2];" : "=f"(v) : "r"(addr), "n"(OFF));
  return v;
}
__device__ __forceinline__ float4 lds4(unsigned addr) {
  float4 v;
  asm("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(addr));
  return v;
}
__device__ __forceinline__ float2 lds2(unsigned addr) {
  float2 v;
  asm("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr));
  return v;
}
template <int OFF>
__device__ __forceinline__ void red(unsigned addr, float v) {
  asm volatile("red.shared.add.f32 [%0+%1], %2;" ::"r"(addr), "n"(OFF), "f"(v) : "memory");
}

}  // namespace pk

// Radial reciprocals of the pair kernel, per window row i: N = {1/(2i+1),
// 1/(2i+3), 1/i, 1/(i+1)} (gather weights of unstaggered components, the
// deposit's 1/i), H = {1/(2i+2), 1/(2i+4)} (weights of components staggered
// by half a cell).
struct PairTable {
  float4 N[kFWR];
  float2 H[kFWR];
};
constexpr int kQueue = 128;  // per-warp ring of slots left to the scalar path

static_assert(sizeof(PairTable) % 16 == 0, "the scalar rows after the table need 16-byte alignment");

// Shared-memory layout of a pair block, as 32-bit shared addresses.
struct PairWindow {
  unsigned F;    // field window: 6 planes of kFWR x kFWZ
  unsigned J;    // current window: 3 planes of kJWR x kJWZ
  unsigned N, H; // the PairTable arrays
  int fi0, fk0;  // field window origin (node)
  int rlo, rhi, zlo, zhi;  // the cells whose particles may take the pair path
};

// The in-cell ZigZag currents of a pair (currentZigZag.cpp:22-136) as the
// scalar zigzag computes them: relay point at the mid-point, weights in
// metres.  J: J_phi at (i, k), (i+1, k), (i, k+1), (i+1, k+1); J_z at (i, k),
// (i+1, k); J_r at (i, k), (i, k+1).
__device__ __forceinline__ void zigzag_pair(const StepArgs& a, float2 fi, float2 fr, float2 fz, float2 frn,
                                            float2 fzn, float2 w, float2 vp2, float2 J[8]) {
  using namespace pk;
  const float2 x0 = add(fi, fr);
  const float2 oov = mul(bc(a.zz_vol), rcp(fma(bc(2.f), fi, bc(1.f))));
  const float2 ro = mul(x0, bc(a.dr_m)), rn = mul(add(fi, frn), bc(a.dr_m));
  const float2 Fp = mul(w, vp2);
  const float2 Wp = mul(mul(vp2, bc(a.dt_s)), rcp(mul(bc(2.f * 3.14159265f), add(ro, rn))));
  const float2 xr = mul(bc(0.5f), add(fr, frn)), yr = mul(bc(0.5f), add(fz, fzn));
  const float2 cod = mul(w, bc(1.f / a.dt_s));
  const float2 cr = mul(cod, bc(a.dr_m)), cz = mul(cod, bc(a.dz_m));
  const float2 Fr1 = mul(cr, sub(xr, fr)), Fr2 = mul(cr, sub(frn, xr));
  const float2 Fz1 = mul(cz, sub(yr, fz)), Fz2 = mul(cz, sub(fzn, yr));
  const float2 Wr1 = mul(bc(a.dr_m), mul(bc(0.5f), add(fr, xr))), Wr2 = mul(bc(a.dr_m), mul(bc(0.5f), add(frn, xr)));
  const float2 Wz1 = mul(bc(a.dz_m), mul(bc(0.5f), add(fz, yr))), Wz2 = mul(bc(a.dz_m), mul(bc(0.5f), add(fzn, yr)));
  const float2 mWr1 = one_minus(Wr1), mWr2 = one_minus(Wr2), mWz1 = one_minus(Wz1), mWz2 = one_minus(Wz2);
  const float2 op = mul(oov, add(one_minus(Wp), Wp));  // the reference's (1 - W_phi) + W_phi split
  const float2 of = mul(oov, Fp);
  J[0] = mul(of, mul(mWr2, mWz2));
  J[1] = mul(of, mul(Wr2, mWz2));
  J[2] = mul(of, mul(mWr2, Wz1));  // W_z1, as the reference has it (currentZigZag.cpp:104)
  J[3] = mul(of, mul(Wr2, Wz2));
  J[4] = mul(op, fma(Fz2, mWr2, mul(Fz1, mWr1)));
  J[5] = mul(op, fma(Fz2, Wr2, mul(Fz1, Wr1)));
  J[6] = mul(op, fma(Fr2, mWz2, mul(Fr1, mWz1)));
  J[7] = mul(op, fma(Fr2, Wz2, mul(Fr1, Wz1)));
}

// The completed particles of a pair written back.
__device__ __forceinline__ void pair_store(const SpeciesF32Buffers& b, unsigned ja, unsigned jb, bool okA, bool okB,
                                           float2 frn, float2 fzn, float2 vr2, float2 vp2, float2 v2) {
  if (okA) {
    b.off_r[ja] = frn.x; b.off_z[ja] = fzn.x;
    b.vr[ja] = vr2.x; b.vphi[ja] = vp2.x; b.vz[ja] = v2.x;
  }
  if (okB) {
    b.off_r[jb] = frn.y; b.off_z[jb] = fzn.y;
    b.vr[jb] = vr2.y; b.vphi[jb] = vp2.y; b.vz[jb] = v2.y;
  }
}

// The currents of a pair added to the block's window (two particles of one
// cell add theirs first and reduce once).
__device__ __forceinline__ void pair_reduce(const PairWindow& W, bool okA, bool okB, int rowA, int rowB, int ckA,
                                            int ckB, bool same_cell, float2 J[8]) {
  using namespace pk;
  constexpr int JP = kJWR * kJWZ;
  const bool same = okA && okB && same_cell;
  if (same) {
#pragma unroll
    for (int q = 0; q < 8; ++q) J[q].x += J[q].y;
  }
  // J_r of the cell's node in the current window, which starts one node
  // after the field window on each axis
  if (okA) {
    const unsigned p = W.J + 4u * (unsigned)((rowA - 1) * kJWZ + (ckA - W.fk0 - 1));
    red<4 * JP>(p, J[0].x);                   red<4 * (JP + kJWZ)>(p, J[1].x);
    red<4 * (JP + 1)>(p, J[2].x);             red<4 * (JP + kJWZ + 1)>(p, J[3].x);
    red<4 * (2 * JP)>(p, J[4].x);             red<4 * (2 * JP + kJWZ)>(p, J[5].x);
    red<0>(p, J[6].x);                        red<4>(p, J[7].x);
  }
  if (okB && !same) {
    const unsigned p = W.J + 4u * (unsigned)((rowB - 1) * kJWZ + (ckB - W.fk0 - 1));
    red<4 * JP>(p, J[0].y);                   red<4 * (JP + kJWZ)>(p, J[1].y);
    red<4 * (JP + 1)>(p, J[2].y);             red<4 * (JP + kJWZ + 1)>(p, J[3].y);
    red<4 * (2 * JP)>(p, J[4].y);             red<4 * (2 * JP + kJWZ)>(p, J[5].y);
    red<0>(p, J[6].y);                        red<4>(p, J[7].y);
  }
}

// The fast path of one pair of slots.  okA / okB come back true for each
// particle it completed (slot written, current deposited); a live particle
// it did not complete is left untouched for the scalar path.  A particle in
// a cell outside [rlo, rhi] x [zlo, zhi], or a dead slot, never enters: its
// lane computes on the other particle's cell and is discarded.
template <int FIX, int KIND>
__device__ __forceinline__ void pair_particles(const StepArgs& a, const SpeciesF32Buffers& b, unsigned ja,
                                               unsigned jb, const Slot& A, const Slot& B, bool hasA, bool hasB,
                                               const PairWindow& W, bool& okA, bool& okB) {
  using namespace pk;
  okA = okB = false;
  int ciA = cell_r_of(A.cell), ckA = cell_z_of(A.cell);
  int ciB = cell_r_of(B.cell), ckB = cell_z_of(B.cell);
  const bool preA = hasA && A.cell >= 0 && (unsigned)(ciA - W.rlo) <= (unsigned)(W.rhi - W.rlo) &&
                    (unsigned)(ckA - W.zlo) <= (unsigned)(W.zhi - W.zlo);
  const bool preB = hasB && B.cell >= 0 && (unsigned)(ciB - W.rlo) <= (unsigned)(W.rhi - W.rlo) &&
                    (unsigned)(ckB - W.zlo) <= (unsigned)(W.zhi - W.zlo);
  if (!preA && !preB) return;
  if (!preA) { ciA = ciB; ckA = ckB; }
  if (!preB) { ciB = ciA; ckB = ckA; }
  const float2 fr = make_float2(A.fr, B.fr), fz = make_float2(A.fz, B.fz);
  const float2 fi = make_float2((float)ciA, (float)ciB);

  // ---- gather (maxwellSolver.hpp:101-316) from the shared window ----
  const bool rA = A.fr >= 0.5f, rB = B.fr >= 0.5f, zA = A.fz >= 0.5f, zB = B.fz >= 0.5f;
  const float2 u = add(fr, make_float2(rA ? -0.5f : 0.5f, rB ? -0.5f : 0.5f));   // r stagger offset
  const float2 zu = add(fz, make_float2(zA ? -0.5f : 0.5f, zB ? -0.5f : 0.5f));  // z stagger offset
  const float2 fh = add(fi, make_float2(rA ? 0.f : -1.f, rB ? 0.f : -1.f));      // staggered row
  // byte address of the particle's cell node in plane 0, and of its
  // staggered rows / columns
  constexpr int P = kFWR * kFWS, L = kFWS;
  const int rowA = ciA - W.fi0, rowB = ciB - W.fi0;
  const unsigned nA = W.F + 4u * (unsigned)(rowA * L + (ckA - W.fk0));
  const unsigned nB = W.F + 4u * (unsigned)(rowB * L + (ckB - W.fk0));
  const unsigned hnA = nA - (rA ? 0u : 4u * L), hnB = nB - (rB ? 0u : 4u * L);
  const unsigned nhA = nA - (zA ? 0u : 4u), nhB = nB - (zB ? 0u : 4u);
  const unsigned hhA = hnA - (zA ? 0u : 4u), hhB = hnB - (zB ? 0u : 4u);
  const float4 NA = lds4(W.N + 16u * rowA), NB = lds4(W.N + 16u * rowB);
  const float2 sn0 = make_float2(NA.x, NB.x);
  // radial weight numerators, shared with the deposit's J_z terms
  const float2 t2f = fma(bc(2.f), fi, fr);                    // 2i + x
  const float2 nn0 = mul(one_minus(fr), t2f);                 // (1-x)(2i+x)
  const float2 nn1 = mul(fr, add(t2f, bc(1.f)));              // x(2i+1+x)
  const float2 t2h = fma(bc(2.f), fh, u);
  const float2 hh0 = mul(one_minus(u), add(t2h, bc(1.f)));    // (1-u)(2h+1+u)
  const float2 hh1 = mul(u, add(t2h, bc(2.f)));               // u(2h+2+u)
  float2 n0, n1, h0, h1;
  if (FIX) {  // the particle's cloud volume: every weight over 2x
    const float2 s = mul(bc(0.5f), rcp(add(fi, fr)));
    n0 = mul(nn0, s);
    n1 = mul(nn1, s);
    h0 = mul(hh0, s);
    h1 = mul(hh1, s);
  } else {  // the reference's CELL_VOLUME denominators
    const float2 HA = lds2(W.H + 8u * (rowA - (rA ? 0 : 1))), HB = lds2(W.H + 8u * (rowB - (rB ? 0 : 1)));
    n0 = mul(nn0, sn0);
    n1 = mul(nn1, make_float2(NA.y, NB.y));
    h0 = mul(hh0, make_float2(HA.x, HB.x));
    h1 = mul(hh1, make_float2(HA.y, HB.y));
  }
  // ((f00 w0 + f10 w1) (1-v) + (f01 w0 + f11 w1) v) of component C at the
  // nodes from qa / qb
#define PCG_PAIR_LERP(C, qa, qb, w0, w1, v, ov)                                                   \
  fma(fma(make_float2(lds<4 * (C * P + L + 1)>(qa), lds<4 * (C * P + L + 1)>(qb)), w1,             \
          mul(make_float2(lds<4 * (C * P + 1)>(qa), lds<4 * (C * P + 1)>(qb)), w0)),               \
      v,                                                                                          \
      mul(fma(make_float2(lds<4 * (C * P + L)>(qa), lds<4 * (C * P + L)>(qb)), w1,                 \
              mul(make_float2(lds<4 * (C * P)>(qa), lds<4 * (C * P)>(qb)), w0)),                   \
          ov))
  const float2 ofz = one_minus(fz), ozu = one_minus(zu);
  float2 E0 = PCG_PAIR_LERP(0, hnA, hnB, h0, h1, fz, ofz);   // E_r   (1/2, 0)
  float2 B2 = PCG_PAIR_LERP(5, hnA, hnB, h0, h1, fz, ofz);   // H_z   (1/2, 0)
  float2 E2 = PCG_PAIR_LERP(2, nhA, nhB, n0, n1, zu, ozu);   // E_z   (0, 1/2)
  float2 B0 = PCG_PAIR_LERP(3, nhA, nhB, n0, n1, zu, ozu);   // H_r   (0, 1/2)
  float2 B1 = PCG_PAIR_LERP(4, hhA, hhB, h0, h1, zu, ozu);   // H_phi (1/2, 1/2)
#undef PCG_PAIR_LERP
  float2 E1;                                                  // E_phi (0, 0)
  {
    const float2 f00 = make_float2(lds<4 * P>(nA), lds<4 * P>(nB));
    const float2 f10 = make_float2(lds<4 * (P + L)>(nA), lds<4 * (P + L)>(nB));
    const float2 f01 = make_float2(lds<4 * (P + 1)>(nA), lds<4 * (P + 1)>(nB));
    const float2 f11 = make_float2(lds<4 * (P + L + 1)>(nA), lds<4 * (P + L + 1)>(nB));
    const float2 t11 = mul(mul(f11, n1), fz);
    E1 = fma(mul(f01, n0), fz, mul(fma(f10, n1, mul(f00, n0)), ofz));
    if (FIX) E1 = add(E1, t11); else E2 = add(E2, t11);  // maxwellSolver.hpp:313
  }

  float2 v0 = make_float2(A.vr, B.vr), v1 = make_float2(A.vphi, B.vphi), v2 = make_float2(A.vz, B.vz);
  const float2 ic2 = bc(1.f / kC2);
  const float2 beta = mul(fma(v2, v2, fma(v1, v1, mul(v0, v0))), ic2);
  const bool subA = beta.x < 1.f, subB = beta.y < 1.f;  // superluminal or NaN: the scalar path reports it
  if constexpr (KIND == 1 || KIND == 3) {
    // ---- Vay push (pusherVay.cpp:22-114), as the scalar push computes it: u =
    // gamma v, in units of c in the fixed mode and in m/s as the reference has it ----
    const float cn = FIX ? 1.f / 3.0e8f : 1.f;
    const float2 g0 = rsq(one_minus(beta));
    const float2 gc = FIX ? mul(g0, bc(cn)) : g0;
    const float2 u0 = mul(v0, gc), u1 = mul(v1, gc), u2 = mul(v2, gc);
    const float2 ek = bc(2.f * a.c2m * cn), bk = bc(a.bk);
    B0 = mul(B0, bk); B1 = mul(B1, bk); B2 = mul(B2, bk);
    const float2 uu = fma(u2, u2, fma(u1, u1, mul(u0, u0)));
    const float2 gi = FIX ? rsq(add(bc(1.f), uu)) : rsq(fma(uu, ic2, bc(1.f)));
    const float2 up0 = fma(gi, fma(u1, B2, mul(mul(u2, B1), bc(-1.f))), fma(E0, ek, u0));
    const float2 up1 = fma(gi, fma(u2, B0, mul(mul(u0, B2), bc(-1.f))), fma(E1, ek, u1));
    const float2 up2 = fma(gi, fma(u0, B1, mul(mul(u1, B0), bc(-1.f))), fma(E2, ek, u2));
    const float2 Bsq = fma(B2, B2, fma(B1, B1, mul(B0, B0)));
    const float2 s0 = sub(fma(up2, up2, fma(up1, up1, fma(up0, up0, bc(1.f)))), Bsq);
    const float2 ub = fma(up2, B2, fma(up1, B1, mul(up0, B0)));
    const float2 al = rsq(mul(bc(0.5f), add(s0, sqr(fma(s0, s0, mul(bc(4.f), fma(ub, ub, Bsq)))))));
    B0 = mul(B0, al); B1 = mul(B1, al); B2 = mul(B2, al);
    const float2 sc = rcp(fma(B2, B2, fma(B1, B1, fma(B0, B0, bc(1.f)))));
    const float2 ab = fma(up2, B2, fma(up1, B1, mul(up0, B0)));
    const float2 p0 = mul(sc, fma(ab, B0, fma(B2, up1, fma(mul(B1, up2), bc(-1.f), up0))));
    const float2 p1 = mul(sc, fma(ab, B1, fma(B0, up2, fma(mul(B2, up0), bc(-1.f), up1))));
    const float2 p2 = mul(sc, fma(ab, B2, fma(B1, up0, fma(mul(B0, up1), bc(-1.f), up2))));
    const float2 pp = fma(p2, p2, fma(p1, p1, mul(p0, p0)));
    const float2 go = FIX ? mul(rsq(add(bc(1.f), pp)), bc(3.0e8f)) : rsq(fma(pp, ic2, bc(1.f)));
    v0 = mul(p0, go); v1 = mul(p1, go); v2 = mul(p2, go);
  } else {
  // ---- relativistic Boris push (pusherBoris.cpp:33-149) ----
  const float2 ck = bc(a.c2m);
  E0 = mul(E0, ck); E1 = mul(E1, ck); E2 = mul(E2, ck);
  float2 gm = rsq(one_minus(beta));
  v0 = fma(v0, gm, E0); v1 = fma(v1, gm, E1); v2 = fma(v2, gm, E2);
  gm = mul(rsq(fma(fma(v2, v2, fma(v1, v1, mul(v0, v0))), ic2, bc(1.f))), bc(a.bk));
  B0 = mul(B0, gm); B1 = mul(B1, gm); B2 = mul(B2, gm);
  const float2 nB0 = mul(B0, bc(-1.f)), nB1 = mul(B1, bc(-1.f)), nB2 = mul(B2, bc(-1.f));
  const float2 k2 = mul(bc(2.f), rcp(fma(B2, B2, fma(B1, B1, fma(B0, B0, bc(1.f))))));
  {
    const float2 s0 = fma(v2, B0, fma(v0, nB2, v1));   // t1 - t0 b2 + t2 b0
    const float2 s1 = fma(v1, nB0, fma(v0, B1, v2));   // t2 + t0 b1 - t1 b0
    const float2 s2 = fma(v2, nB1, fma(v1, B2, v0));   // t0 + t1 b2 - t2 b1
    const float2 w0 = fma(s1, nB1, mul(s0, B2));
    const float2 w1 = fma(s2, nB2, mul(s1, B0));
    const float2 w2 = fma(s0, nB0, mul(s2, B1));
    v0 = add(fma(k2, w0, v0), E0);
    v1 = add(fma(k2, w1, v1), E1);
    v2 = add(fma(k2, w2, v2), E2);
  }
  gm = rsq(fma(fma(v2, v2, fma(v1, v1, mul(v0, v0))), ic2, bc(1.f)));
  v0 = mul(v0, gm); v1 = mul(v1, gm); v2 = mul(v2, gm);
  }
  if constexpr (KIND == 3) {  // the push half of a collisional step: the velocities alone
    okA = preA && subA;
    okB = preB && subB;
    if (okA) { b.vr[ja] = v0.x; b.vphi[ja] = v1.x; b.vz[ja] = v2.x; }
    if (okB) { b.vr[jb] = v0.y; b.vphi[jb] = v1.y; b.vz[jb] = v2.y; }
    return;
  }

  // ---- move in the local Cartesian frame and back to r-z (specieP.cpp:482-491, 609-640) ----
  const float2 dx = mul(v0, bc(a.dt_dr)), dyp = mul(v1, bc(a.dt_dr)), dYv = mul(v2, bc(a.dt_dz));
  const float2 x0 = add(fi, fr);
  const float2 X = add(x0, dx);
  const float2 dy2 = mul(dyp, dyp);
  const float2 xn2 = fma(X, X, dy2);
  const float2 rxn = rsq(xn2);                          // 1/x'
  const float2 xn = mul(xn2, rxn);                      // x' = sqrt(X^2 + dy^2)
  const float2 sn = mul(dyp, rxn);
  const float2 dXv = fma(dy2, rcp(add(X, xn)), dx);      // x' - x = dx + dy^2/(X + x')
  const float2 frn = add(fr, dXv), fzn = add(fz, dYv);
  // the deposit's displacement: the move itself, or in the fixed mode the
  // difference of the stored offsets (exact for close offsets), so that the
  // current carries the charge the rounded new position holds
  const float2 dX = FIX ? sub(frn, fr) : dXv, dY = FIX ? sub(fzn, fz) : dYv;
  const float2 ixo = rcp(x0);
  const float2 t = mul(dX, ixo);
  if constexpr (KIND == 1) {  // the in-cell case
    okA = preA && subA && frn.x >= 0.f && frn.x < 1.f && fzn.x >= 0.f && fzn.x < 1.f && X.x > 0.5f;
    okB = preB && subB && frn.y >= 0.f && frn.y < 1.f && fzn.y >= 0.f && fzn.y < 1.f && X.y > 0.5f;
  } else {
    // the in-cell case with the logarithm's series valid (|t| < 0.02); motion
    // below 1e-15 m on an axis takes the strict-motion branch (currentVB.cpp:500-729)
    okA = preA && subA && frn.x >= 0.f && frn.x < 1.f && fzn.x >= 0.f && fzn.x < 1.f && X.x > 0.5f &&
          fabsf(t.x) < 0.02f && fabsf(dX.x) >= a.mnzl_r && fabsf(dY.x) >= a.mnzl_z;
    okB = preB && subB && frn.y >= 0.f && frn.y < 1.f && fzn.y >= 0.f && fzn.y < 1.f && X.y > 0.5f &&
          fabsf(t.y) < 0.02f && fabsf(dX.y) >= a.mnzl_r && fabsf(dY.y) >= a.mnzl_z;
  }
  if (!okA && !okB) return;
  const float2 cs = sqr(fma(sn, mul(sn, bc(-1.f)), bc(1.f)));
  const float2 vr2 = fma(cs, v0, mul(mul(sn, v1), bc(-1.f)));
  const float2 vp2 = fma(sn, v0, mul(cs, v1));
  const float2 w = make_float2(A.w, B.w);
  // the eight node currents of each particle: J_phi at (i, k), (i+1, k),
  // (i, k+1), (i+1, k+1); J_z at (i, k), (i+1, k); J_r at (i, k), (i, k+1)
  float2 J[8];
  if constexpr (KIND == 1) {
    zigzag_pair(a, fi, fr, fz, frn, fzn, w, vp2, J);
  } else {
  // ---- in-cell Villasenor-Buneman deposit (currentVB.cpp:22-173, 398-498) ----
  const float2 inv_i = make_float2(NA.z, NB.z), inv_i1 = make_float2(NA.w, NB.w);
  // J_phi from the mid-point
  const float2 Xm = fma(bc(0.5f), dX, fr), Ym = fma(bc(0.5f), dY, fz);
  const float2 t2m = fma(bc(2.f), fi, Xm);
  const float2 qp = mul(mul(w, bc(a.qp)), mul(vp2, rcp(add(fi, Xm))));
  const float2 a0 = mul(qp, mul(mul(one_minus(Xm), t2m), sn0));
  const float2 a1 = mul(qp, mul(mul(Xm, add(t2m, bc(1.f))), mul(bc(0.5f), inv_i1)));
  const float2 oYm = one_minus(Ym);
  // J_z and J_r of the segment
  const float2 t2 = mul(t, t);
  const float2 h = mul(t2, fma(t, fma(t, fma(t, fma(t, bc(1.f / 7.f), bc(-1.f / 6.f)), bc(0.2f)), bc(-0.25f)),
                               bc(1.f / 3.f)));
  const float2 m = mul(t, fma(t, fma(t, fma(t, fma(t, bc(-5.f / 6.f), bc(0.8f)), bc(-0.75f)), bc(2.f / 3.f)),
                              bc(-0.5f)));
  const float2 ixn = rcp(add(x0, dX));
  const float2 cc = fma(fi, fi, fi);                         // i(i+1)
  const float2 lin = mul(mul(bc(0.5f), dX), fma(cc, mul(ixo, ixo), bc(1.f)));
  const float2 d = sub(mul(mul(cc, h), ixo), lin);           // hh - lin
  const float2 qz = mul(mul(w, bc(a.qz)), dY);
  const float2 jz0 = mul(mul(qz, fma(nn0, ixo, d)), inv_i);
  const float2 jz1 = mul(mul(qz, sub(mul(nn1, ixo), d)), inv_i1);
  const float2 qr = mul(mul(w, bc(2.f * a.qr)), sn0);        // q Qr / (i + 1/2)
  const float2 bb = one_minus(fz);
  const float2 cx = mul(mul(bc(0.5f), cc), ixo);
  const float2 dm = mul(dY, m);
  const float2 q4v = mul(bc(0.25f), dY);
  const float2 dXi = mul(dX, ixn);
  const float2 jr0 = mul(qr, fma(dX, sub(mul(bc(0.5f), bb), q4v), mul(cx, fma(dXi, bb, dm))));
  const float2 jr1 = mul(qr, fma(dX, fma(bc(0.5f), fz, q4v), mul(cx, sub(mul(dXi, fz), dm))));
  pair_store(b, ja, jb, okA, okB, frn, fzn, vr2, vp2, v2);
  J[0] = mul(a0, oYm); J[1] = mul(a1, oYm); J[2] = mul(a0, Ym); J[3] = mul(a1, Ym);
  J[4] = jz0; J[5] = jz1; J[6] = jr0; J[7] = jr1;
  }
  if constexpr (KIND != 0) pair_store(b, ja, jb, okA, okB, frn, fzn, vr2, vp2, v2);
  pair_reduce(W, okA, okB, rowA, rowB, ckA, ckB, ciA == ciB && ckA == ckB, J);
}


// The fast path of a pair in the move half of a collisional step (the
// velocities were pushed before the collisions): the learned collision
// step's transform of the particle's cell, v' = u + (v - u) s per axis in
// FP32 from the block's table of its window cells (the identity where the
// cell's flag is not 1; the float store rounds as the FP64 form of the
// scalar path does, to within an ulp), then the move and the in-cell ZigZag
// currents of pair_particles.
template <int FIX>
__device__ __forceinline__ void pair_move_particles(const StepArgs& a, const SpeciesF32Buffers& b, unsigned ja,
                                                    unsigned jb, const Slot& A, const Slot& B, bool hasA, bool hasB,
                                                    const PairWindow& W, bool& okA, bool& okB) {
  using namespace pk;
  okA = okB = false;
  int ciA = cell_r_of(A.cell), ckA = cell_z_of(A.cell);
  int ciB = cell_r_of(B.cell), ckB = cell_z_of(B.cell);
  const bool preA = hasA && A.cell >= 0 && (unsigned)(ciA - W.rlo) <= (unsigned)(W.rhi - W.rlo) &&
                    (unsigned)(ckA - W.zlo) <= (unsigned)(W.zhi - W.zlo);
  const bool preB = hasB && B.cell >= 0 && (unsigned)(ciB - W.rlo) <= (unsigned)(W.rhi - W.rlo) &&
                    (unsigned)(ckB - W.zlo) <= (unsigned)(W.zhi - W.zlo);
  if (!preA && !preB) return;
  if (!preA) { ciA = ciB; ckA = ckB; }
  if (!preB) { ciB = ciA; ckB = ckA; }
  float2 v0 = make_float2(A.vr, B.vr), v1 = make_float2(A.vphi, B.vphi), v2 = make_float2(A.vz, B.vz);
  if (a.xform) {  // the table: {u_r, u_phi, u_z, s_r} per window cell, then {s_phi, s_z}
    constexpr unsigned kXS = 16u * kFWR * kFWS;
    const unsigned qA = (unsigned)((ciA - W.fi0) * kFWS + (ckA - W.fk0));
    const unsigned qB = (unsigned)((ciB - W.fi0) * kFWS + (ckB - W.fk0));
    const float4 UA = lds4(W.F + 16u * qA), UB = lds4(W.F + 16u * qB);
    const float2 SA = lds2(W.F + kXS + 8u * qA), SB = lds2(W.F + kXS + 8u * qB);
    const float2 u0 = make_float2(UA.x, UB.x), u1 = make_float2(UA.y, UB.y), u2 = make_float2(UA.z, UB.z);
    v0 = fma(sub(v0, u0), make_float2(UA.w, UB.w), u0);
    v1 = fma(sub(v1, u1), make_float2(SA.x, SB.x), u1);
    v2 = fma(sub(v2, u2), make_float2(SA.y, SB.y), u2);
  }
  const float2 fr = make_float2(A.fr, B.fr), fz = make_float2(A.fz, B.fz);
  const float2 fi = make_float2((float)ciA, (float)ciB);
  // the move of pair_particles (specieP.cpp:482-491, 609-640)
  const float2 dx = mul(v0, bc(a.dt_dr)), dyp = mul(v1, bc(a.dt_dr)), dYv = mul(v2, bc(a.dt_dz));
  const float2 x0 = add(fi, fr);
  const float2 X = add(x0, dx);
  const float2 dy2 = mul(dyp, dyp);
  const float2 xn2 = fma(X, X, dy2);
  const float2 rxn = rsq(xn2);
  const float2 sn = mul(dyp, rxn);
  const float2 dXv = fma(dy2, rcp(add(X, mul(xn2, rxn))), dx);
  const float2 frn = add(fr, dXv), fzn = add(fz, dYv);
  okA = preA && frn.x >= 0.f && frn.x < 1.f && fzn.x >= 0.f && fzn.x < 1.f && X.x > 0.5f;
  okB = preB && frn.y >= 0.f && frn.y < 1.f && fzn.y >= 0.f && fzn.y < 1.f && X.y > 0.5f;
  if (!okA && !okB) return;
  const float2 cs = sqr(fma(sn, mul(sn, bc(-1.f)), bc(1.f)));
  const float2 vr2 = fma(cs, v0, mul(mul(sn, v1), bc(-1.f)));
  const float2 vp2 = fma(sn, v0, mul(cs, v1));
  float2 J[8];
  zigzag_pair(a, fi, fr, fz, frn, fzn, make_float2(A.w, B.w), vp2, J);
  pair_store(b, ja, jb, okA, okB, frn, fzn, vr2, vp2, v2);
  pair_reduce(W, okA, okB, ciA - W.fi0, ciB - W.fi0, ckA, ckB, ciA == ciB && ckA == ckB, J);
}


// ---------------------------------------------------------------------------
// Slot staging.  A block's particles are a contiguous range of its tile.  It
// reads them in chunks of kChunk slots (two per thread), each chunk's seven
// slot arrays copied by the tensor memory accelerator (cp.async.bulk, one
// issuing thread) into one of kStages shared-memory buffers and completed on
// the buffer's "full" mbarrier; the warps release a buffer on its "empty"
// mbarrier.  A bulk copy moves whole 16-byte units from 16-byte aligned
// addresses, so a chunk's copy starts at the slot index rounded down to a
// multiple of 4 and ends rounded up (the slot arrays have kSlotPad spare
// elements); slot c of the chunk sits at index c - c0 + lead in the buffer.
constexpr int kChunk = 2 * kThreads;
constexpr int kStageArr = kChunk + 8;                 // elements per staged array (with the rounding)
constexpr int kStageBytes = 7 * kStageArr * 4;        // cell, off_r, off_z, vr, vphi, vz, w
constexpr int kStages = 2;
constexpr uint32_t kStageWaitLimit = 1u << 20;        // try_wait rounds before a wait gives up
static_assert(kStageArr * 4 % 16 == 0, "staged arrays keep 16-byte alignment");

namespace tma {

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
// Waits for the phase of the given parity to complete; false after
// kStageWaitLimit unsuccessful rounds.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity) {
  for (uint32_t i = 0; i < kStageWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
// bytes (a multiple of 16) from 16-byte aligned global src to 16-byte aligned shared dst
__device__ __forceinline__ void bulk_load(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

}  // namespace tma

// Issues the bulk copies of chunk k of the block's range [bs, be) into
// stage buffer `buf` (byte address), completing on mbarrier `bar`.
__device__ __forceinline__ void stage_chunk(const SpeciesF32Buffers& b, unsigned bs, unsigned be, unsigned k,
                                            unsigned buf, unsigned bar) {
  const unsigned c0 = bs + k * kChunk, c1 = min(c0 + kChunk, be);
  const unsigned a0 = c0 & ~3u, a1 = (c1 + 3u) & ~3u;
  const unsigned bytes = 4u * (a1 - a0);
  tma::mbar_expect_tx(bar, 7u * bytes);
  tma::bulk_load(buf + 0 * (4u * kStageArr), b.cell + a0, bytes, bar);
  tma::bulk_load(buf + 1 * (4u * kStageArr), b.off_r + a0, bytes, bar);
  tma::bulk_load(buf + 2 * (4u * kStageArr), b.off_z + a0, bytes, bar);
  tma::bulk_load(buf + 3 * (4u * kStageArr), b.vr + a0, bytes, bar);
  tma::bulk_load(buf + 4 * (4u * kStageArr), b.vphi + a0, bytes, bar);
  tma::bulk_load(buf + 5 * (4u * kStageArr), b.vz + a0, bytes, bar);
  tma::bulk_load(buf + 6 * (4u * kStageArr), b.w + a0, bytes, bar);
}

// Slot i of a staged chunk (buffer byte address buf).
__device__ __forceinline__ Slot staged_slot(unsigned buf, unsigned i) {
  using pk::lds;
  const unsigned p = buf + 4u * i;
  Slot q;
  q.cell = __float_as_int(lds<0>(p));
  q.fr = lds<4 * kStageArr>(p);
  q.fz = lds<8 * kStageArr>(p);
  q.vr = lds<12 * kStageArr>(p);
  q.vphi = lds<16 * kStageArr>(p);
  q.vz = lds<20 * kStageArr>(p);
  q.w = lds<24 * kStageArr>(p);
  return q;
}

// fields, current, the pair table, the scalar path's rows (2 float4 per
// row), the per-warp queues, then (1 KB aligned) the slot stages and their
// mbarriers
constexpr size_t kPairFixedBytes = sizeof(float) * (6 * kFWR * kFWS + 3 * kJWR * kJWZ) + sizeof(PairTable) +
                                   sizeof(float4) * 2 * kFWR + sizeof(unsigned) * kQueue * (kThreads / 32);
constexpr size_t kPairSmemBytes = kPairFixedBytes + 1024 + (size_t)kStages * kStageBytes + 2 * kStages * 8;

// One block per part of a tile (up to gridDim.y blocks share a crowded tile,
// each a contiguous part of its slots), for a plasma species under the
// relativistic Boris pusher and the Villasenor-Buneman current.  The slots
// arrive through the staged chunks above; each thread takes two per chunk
// (i and i + kThreads) through pair_particles.  Live particles the pair path
// leaves go to the warp's queue in shared memory; whenever 32 have gathered
// (and once at the end) the warp runs them through the scalar tile_particle
// one per lane (reading them from global memory), so that the rare cases do
// not stall the warp's other lanes.  A wait for a chunk that runs out sets
// kErrTimeout, waits (bounded) for the copies in flight and ends the block.
// KIND 0: the relativistic Boris pusher and the Villasenor-Buneman current;
// KIND 1: the Vay pusher and the ZigZag current; KIND 2: the move half of
// a collisional step with the ZigZag current (no field window); KIND 3:
// the push half of a collisional step with the Vay pusher (gather and push
// from the field window, velocities stored, no current).
template <int FIX, int KIND = 0>
// Four resident blocks per SM (64 registers) measured faster than three
// with 80 registers and no spill.
__global__ void __launch_bounds__(kThreads, 4)
    step_pair_kernel(StepArgs args, SpeciesF32Buffers b, TileGrid tg) {
  StepArgs a = args;
  a.pusher = KIND == 0 ? PCG_PUSHER_BORIS_RELATIVISTIC : PCG_PUSHER_VAY;
  a.is_beam = 0;
  a.fixed = FIX;
  a.pushed = KIND == 2 ? 1 : 0;  // whole steps, or the move half of one
  if (KIND != 2) a.xform = nullptr;
  extern __shared__ __align__(16) float smem[];
  const int t = blockIdx.x;
  // the tile's parts: the blocks per tile of the last sort (on the device),
  // up to the gridDim.y launched
  const unsigned np = max(1u, min(b.sort_info[2], gridDim.y));
  if (blockIdx.y >= np) return;
  const unsigned ts = b.tile_start[t], te = b.tile_start[t + 1];
  const unsigned part = (te - ts + np - 1) / np;
  const unsigned bs = ts + blockIdx.y * part, be = min(bs + part, te);
  if (bs >= be) return;
  const unsigned nchunks = (be - bs + kChunk - 1) / kChunk;
  const int tr = t / tg.ntz, tz = t - tr * tg.ntz;
  const int r0 = tr * kTileR, z0 = tz * kTileZ;
  const int fi0 = r0 - kHalo - 1, fk0 = z0 - kHalo - 1;
  const int ji0 = r0 - kHalo, jk0 = z0 - kHalo;
  float* sF = smem;
  float* sJ = smem + 6 * kFWR * kFWS;
  PairTable* tb = reinterpret_cast<PairTable*>(sJ + 3 * kJWR * kJWZ);
  float4* sR = reinterpret_cast<float4*>(tb + 1);  // the scalar path's rows (2 float4 per row)
  unsigned* queue = reinterpret_cast<unsigned*>(sR + 2 * kFWR);
  const unsigned sbase = (unsigned)__cvta_generic_to_shared(smem);
  const unsigned stage0 = (sbase + (unsigned)kPairFixedBytes + 1023u) & ~1023u;
  const unsigned full0 = stage0 + kStages * kStageBytes, empty0 = full0 + 8 * kStages;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    for (int q = 0; q < kStages; ++q) {
      tma::mbar_init(full0 + 8 * q, 1);
      tma::mbar_init(empty0 + 8 * q, kThreads / 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (unsigned k = 0; k < (unsigned)kStages && k < nchunks; ++k)
      stage_chunk(b, bs, be, k, stage0 + k * kStageBytes, full0 + 8 * k);
  }
  // the field window, each thread's loads issued before its shared stores
  // (the move half of a collisional step gathers nothing)
  if constexpr (KIND != 2) {
    constexpr int kRows = 6 * kFWR, kPer = (kRows + kThreads / 32 - 1) / (kThreads / 32);
    constexpr int kCols = (kFWZ + 31) / 32;
    float v[kPer][kCols];
#pragma unroll
    for (int r = 0; r < kPer; ++r) {
      const int row = warp + r * (kThreads / 32);
      const int c = row / kFWR, i = fi0 + (row - c * kFWR);
      const bool row_ok = row < kRows && i >= -2 && i < a.nr + 2;
      const float* src = a.Er + (size_t)c * a.plane + (i + 2) * a.ld + 2;
#pragma unroll
      for (int q = 0; q < kCols; ++q) {
        const int col = lane + 32 * q, k = fk0 + col;
        v[r][q] = (row_ok && col < kFWZ && k >= -2 && k < a.nz + 2) ? __ldg(src + k) : 0.f;
      }
    }
#pragma unroll
    for (int r = 0; r < kPer; ++r) {
      const int row = warp + r * (kThreads / 32);
#pragma unroll
      for (int q = 0; q < kCols; ++q) {
        const int col = lane + 32 * q;
        if (row < kRows && col < kFWZ) sF[row * kFWS + col] = v[r][q];
      }
    }
  }
  if constexpr (KIND == 2) {
    // the learned transforms of the window's cells, in the field window's
    // place (the move gathers nothing): {u_r, u_phi, u_z, s_r}, then
    // {s_phi, s_z}; the identity where a cell's flag is not 1
    static_assert(6 * kFWR * kFWS * sizeof(float) == (sizeof(float4) + sizeof(float2)) * kFWR * kFWS,
                  "the transform table fills the field window");
    if (a.xform) {
      float4* XU = reinterpret_cast<float4*>(sF);
      float2* XS = reinterpret_cast<float2*>(XU + kFWR * kFWS);
      for (int q = threadIdx.x; q < kFWR * kFWS; q += kThreads) {
        const int i = fi0 + q / kFWS, k = fk0 + q % kFWS;
        float4 u = make_float4(0.f, 0.f, 0.f, 1.f);
        float2 v = make_float2(1.f, 1.f);
        if (i >= 0 && i < a.nr && k >= 0 && k < a.nz) {
          const size_t c = (size_t)i * a.nz + k;
          if (a.xflag[c] == 1) {
            const double* t = a.xform + c * 12 + a.xoff;
            u = make_float4((float)t[0], (float)t[1], (float)t[2], (float)t[3]);
            v = make_float2((float)t[4], (float)t[5]);
          }
        }
        XU[q] = u;
        XS[q] = v;
      }
    }
  }
  for (int q = threadIdx.x; q < 3 * kJWR * kJWZ; q += kThreads) sJ[q] = 0.f;
  if (KIND != 2 && threadIdx.x < 2 * kFWR) {
    const int i = fi0 + (int)(threadIdx.x >> 1);
    sR[threadIdx.x] = (i >= -2 && i <= a.nr + 2) ? __ldg(a.rt + 2 * (i + 2) + (threadIdx.x & 1))
                                                 : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __syncthreads();
  if (KIND != 2 && threadIdx.x < kFWR) {
    const float4 p = sR[2 * threadIdx.x], q = sR[2 * threadIdx.x + 1];
    tb->N[threadIdx.x] = make_float4(p.x, p.z, q.x, q.y);
    tb->H[threadIdx.x] = make_float2(p.y, p.w);
  }
  __syncthreads();
  const SharedFields sv{sF, fi0, fk0, sR};
  const SharedDep sd{sJ, ji0, jk0};
  PairWindow W;
  W.F = sbase;
  W.J = (unsigned)__cvta_generic_to_shared(sJ);
  W.N = (unsigned)__cvta_generic_to_shared(tb->N);
  W.H = (unsigned)__cvta_generic_to_shared(tb->H);
  W.fi0 = fi0;
  W.fk0 = fk0;
  // cells whose particles may take the pair path: interior, and one cell
  // inside the field window on each side (the gather reads ci-1 .. ci+2)
  W.rlo = max(1, fi0 + 1); W.rhi = min(a.nr - 2, fi0 + kFWR - 3);
  W.zlo = max(1, fk0 + 1); W.zhi = min(a.nz - 2, fk0 + kFWZ - 3);
  if (W.rhi < W.rlo || W.zhi < W.zlo) W.rlo = W.rhi = W.zlo = W.zhi = 1 << 20;  // a grid of 1-2 cells
  unsigned* myq = queue + warp * kQueue;
  unsigned qhead = 0, qtail = 0;  // the warp's ring, the same in every lane
  const unsigned below = (1u << lane) - 1u;
  unsigned failed = ~0u;  // the chunk whose wait ran out, if one did
  for (unsigned k = 0; k <= nchunks; ++k) {
    const bool more = k < nchunks;
    if (more) {
      const unsigned st = k % kStages, par = (k / kStages) & 1u;
      const unsigned buf = stage0 + st * kStageBytes;
      if (!__all_sync(0xffffffffu, tma::mbar_wait(full0 + 8 * st, par))) {
        failed = k;
        break;
      }
      const unsigned c0 = bs + k * kChunk, c1 = min(c0 + kChunk, be), lead = c0 & 3u;
      const unsigned ja = c0 + threadIdx.x, jb = ja + kThreads;
      const bool hasA = ja < c1, hasB = jb < c1;
      Slot A{}, B{};
      A.cell = B.cell = kDeadCell;
      if (hasA) A = staged_slot(buf, threadIdx.x + lead);
      if (hasB) B = staged_slot(buf, threadIdx.x + kThreads + lead);
      __syncwarp();
      if (lane == 0) tma::mbar_arrive(empty0 + 8 * st);  // this warp is done reading the buffer
      bool okA, okB;
      if constexpr (KIND == 2) pair_move_particles<FIX>(a, b, ja, jb, A, B, hasA, hasB, W, okA, okB);
      else pair_particles<FIX, KIND>(a, b, ja, jb, A, B, hasA, hasB, W, okA, okB);
      const bool needA = hasA && A.cell >= 0 && !okA, needB = hasB && B.cell >= 0 && !okB;
      const unsigned mA = __ballot_sync(0xffffffffu, needA), mB = __ballot_sync(0xffffffffu, needB);
      if (needA) myq[(qtail + __popc(mA & below)) & (kQueue - 1)] = ja;
      qtail += __popc(mA);
      if (needB) myq[(qtail + __popc(mB & below)) & (kQueue - 1)] = jb;
      qtail += __popc(mB);
      // the buffer's next chunk, once every warp has released it
      if (threadIdx.x == 0 && k + kStages < nchunks && tma::mbar_wait(empty0 + 8 * st, par))
        stage_chunk(b, bs, be, k + kStages, buf, full0 + 8 * st);
      // (a buffer not refilled leaves the later wait for its chunk to run out)
    }
    // the queued slots, 32 at a time (all that is left after the last chunk)
    while (qtail - qhead >= 32u || (!more && qtail != qhead)) {
      __syncwarp();
      const unsigned n = min(32u, qtail - qhead);
      const unsigned jj = myq[(qhead + lane) & (kQueue - 1)];
      qhead += n;
      if ((unsigned)lane < n) {
        if constexpr (KIND == 3) push_slot(a, b, jj, load_slot(b, jj));
        else tile_particle<KIND == 0 ? 0 : 1>(a, b, jj, load_slot(b, jj), sv, sd);
      }
      __syncwarp();
    }
  }
  if (failed != ~0u) {
    // the copies that may still be in flight (the failed chunk and the next
    // kStages - 1) land before the block's shared memory is released, each
    // wait bounded again; then report
    for (unsigned k = failed; k < failed + kStages && k < nchunks; ++k)
      if (!tma::mbar_wait(full0 + 8 * (k % kStages), (k / kStages) & 1u)) break;
    if (lane == 0) raise_error(a.st, kErrTimeout);
  }
  __syncthreads();
  if constexpr (KIND == 3) return;  // a push deposits nothing
  for (int row = warp; row < 3 * kJWR; row += kThreads / 32) {
    const int c = row / kJWR, i = ji0 + (row - c * kJWR);
    float* dst = a.Jr + c * a.plane + (i + 2) * a.ld + 2;
    for (int q = lane; q < kJWZ; q += 32) {
      const float v = sJ[row * kJWZ + q];
      if (v != 0.f) atomicAdd(dst + jk0 + q, v);
    }
  }
}

}  // namespace f32
}  // namespace pcg
