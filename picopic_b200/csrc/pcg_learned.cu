// pcg_learned.cu — the learned collision step.
//
// Per cell and per list (electrons: every species not named ions; ions),
// the moment sums N, W = sum w, W u = sum w v, sum w v^2 (per axis r, phi,
// z) give the mean velocity u and the axis temperatures
// T_a = m (sum w v_a^2 / W - u_a^2) / e (eV).  The 13 features are
//   0-2   T_e,a / T_e - 1            (electron anisotropy, T_e the axis mean)
//   3-5   T_i,a / T_i - 1            (ion anisotropy)
//   6     ln(T_i / T_e)
//   7-9   log10 of s_ee, s_ei, s_ii  (collision numbers of the step)
//   10    |u_e - u_i| / sqrt(3 e T_e / m_e)
//   11    ln(n_i / n_e)
//   12    1 / sqrt(N_e + N_i)        (macroparticle noise)
// with s_ab = max(n_a, n_b) dt L (q_a q_b)^2 / (4 pi eps0^2 m_ab^2 v_ab^3),
// v_ab^2 = 3 e (T_a/m_a + T_b/m_b), L = 10: the P12 scattering parameter
// (collisionsP12.cpp:193-201) at the thermal relative speed.  The network
// predicts y, the change of the axis temperatures over one step in units of
// T_s S, S = s_ee + s_ei + s_ii:
//   T'_s,a = T_s,a + T_s S y_s,a.
// The new temperatures are scaled by one factor per cell so that the
// cell's thermal energy sum_s W_s sum_a T_s,a is unchanged, and every
// particle of the cell moves to v_a' = u_a + (v_a - u_a) sqrt(T'_a / T_a):
// the species' momentum and the new second moments hold exactly in FP64.
// The network itself runs on tcgen05 (pcg_mlp_tc.cuh) in a kernel of its
// own between the per-cell input and transform kernels; training keeps the
// mma.sync kernels of pcg_mlp.cu.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "pcg_f32.h"
#include "pcg_learned.h"
#include "pcg_mlp.cuh"
#include "pcg_mlp_tc.cuh"
#include "pcg_tile_walk.cuh"

namespace pcg {

namespace {

constexpr int kThreads = 256;
constexpr double kPi = 3.1415926535897932, kEps0 = 8.85e-12, kE = 1.6e-19, kLogL = 10.0;
constexpr int kStateWords = 17;  // T_e[3], T_i[3], Tm_e, Tm_i, W_e, W_i, u_e[3], u_i[3], S
// the training box is widened by this fraction of each feature's span
constexpr float kBoxMargin = 0.25f;

inline unsigned blocks_for(size_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

// cell and velocity of slot j of a species; false for dead slots or cells off the grid
__device__ __forceinline__ bool slot_of(const GridGeom& g, const CollSpecies& sp, size_t j, size_t* c,
                                        double v[3]) {
  int ci, ck;
  if (sp.cell) {
    const int p = sp.cell[j];
    if (p < 0) return false;
    ci = cell_r_of(p);
    ck = cell_z_of(p);
    v[0] = sp.vr32[j]; v[1] = sp.vphi32[j]; v[2] = sp.vz32[j];
  } else {
    const double r = sp.r[j];
    if (!(r >= 0.0)) return false;
    ci = (int)floor(r / g.dr);
    ck = (int)floor(sp.z[j] / g.dz);
    v[0] = sp.vr64[j]; v[1] = sp.vphi64[j]; v[2] = sp.vz64[j];
  }
  if (ci < 0 || ck < 0 || ci >= g.nr || ck >= g.nz) return false;
  *c = (size_t)ci * g.nz + ck;
  return true;
}

// Per-cell moment sums.  Lanes of a warp that share a cell and list add
// their values with a warp reduction first (whole-warp groups, the usual
// case for particles stored cell by cell) or one after another through the
// group's leader, so that one atomic per word and group reaches memory.
__global__ void moments_kernel(GridGeom g, CollSpecies sp, double* mom, size_t j0) {
  const size_t j = j0 + blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  size_t c = 0;
  double v[3] = {0, 0, 0}, w = 0;
  const bool valid = j < sp.n && slot_of(g, sp, j, &c, v);
  if (valid) w = sp.w64 ? sp.w64[j] : (double)sp.w32[j];
  double val[8] = {valid ? 1.0 : 0.0, w, w * v[0], w * v[1], w * v[2], w * v[0] * v[0], w * v[1] * v[1],
                   w * v[2] * v[2]};
  const long long key = valid ? (long long)c : -1;
  const unsigned group = __match_any_sync(0xffffffffu, key);
  const int lane = threadIdx.x & 31, leader = __ffs(group) - 1;
  if (group == 0xffffffffu) {
    for (int q = 0; q < 8; ++q)
      for (int o = 16; o > 0; o >>= 1) val[q] += __shfl_xor_sync(0xffffffffu, val[q], o);
  } else {
    // the leader gathers its group's values lane by lane
    unsigned rest = group & ~(1u << leader);
    while (__any_sync(0xffffffffu, rest != 0)) {
      const int src = rest ? __ffs(rest) - 1 : lane;
      for (int q = 0; q < 8; ++q) {
        const double x = __shfl_sync(0xffffffffu, val[q], src);
        if (lane == leader && rest) val[q] += x;
      }
      if (rest) rest &= rest - 1;
    }
  }
  if (!valid || lane != leader) return;
  double* m = mom + c * kMomWords + (sp.is_ion ? 8 : 0);
  for (int q = 0; q < 8; ++q) atomicAdd(m + q, val[q]);
}

constexpr int kWalk = 4;  // layers a tile walk loads at once

// The same sums for the tile-sorted slots of a float species, a block per
// tile and a thread per tile cell (pcg_tile_walk.cuh): thread lc walks the
// particles the last sort put in its cell, kWalk layers at a time, sums in
// registers and adds the sums to the grid with one atomic per word.  A
// particle that has left its cell since the sort, and the run beyond
// kLayerCap layers, add to the grid directly.  The sums equal
// moments_kernel's up to the order of the FP64 additions.
__global__ void __launch_bounds__(kTileCells) tile_moments_kernel(GridGeom g, TileGrid tg, CollSpecies sp,
                                                                  double* mom) {
  __shared__ TileWalk tw;
  const int off = sp.is_ion ? 8 : 0, lc = threadIdx.x;
  for (int t = blockIdx.x; t < tg.ntiles; t += gridDim.x) {
    const size_t base = sp.tile_start[t], end = sp.tile_start[t + 1];
    if (base >= end) continue;  // the same for every thread of the block
    const unsigned cnt = sp.cell_count[(size_t)t * kTileCells + lc];
    tile_walk_begin(tw, sp.layer_start, sp.layer_prefix, t, cnt);
    const int ti = t / tg.ntz, tk = t - ti * tg.ntz;
    const int ci = ti * tg.tr + lc / tg.tz, ck = tk * tg.tz + lc % tg.tz;
    const size_t mine = (size_t)ci * g.nz + ck;
    const unsigned my_n = min(cnt, (unsigned)kLayerCap), wn = tile_walk_layers(cnt);
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (unsigned q0 = 0; q0 < wn; q0 += kWalk) {
      size_t j[kWalk];
      int cell[kWalk];
      float vr[kWalk], vp[kWalk], vz[kWalk], ww[kWalk];
#pragma unroll
      for (int u = 0; u < kWalk; ++u) {
        const unsigned bal = __ballot_sync(0xffffffffu, my_n > q0 + u);
        j[u] = my_n > q0 + u ? base + tile_walk_slot(tw, q0 + u, bal) : ~(size_t)0;
      }
#pragma unroll
      for (int u = 0; u < kWalk; ++u) {
        cell[u] = j[u] != ~(size_t)0 ? sp.cell[j[u]] : kDeadCell;
        if (cell[u] >= 0) { vr[u] = sp.vr32[j[u]]; vp[u] = sp.vphi32[j[u]]; vz[u] = sp.vz32[j[u]]; ww[u] = sp.w32[j[u]]; }
      }
#pragma unroll
      for (int u = 0; u < kWalk; ++u) {
        if (cell[u] < 0) continue;
        const int pi = cell_r_of(cell[u]), pk = cell_z_of(cell[u]);
        if (pi < 0 || pi >= g.nr || pk >= g.nz) continue;
        const size_t c = (size_t)pi * g.nz + pk;
        const double w = ww[u], v0 = vr[u], v1 = vp[u], v2 = vz[u];
        const double val[8] = {1.0, w, w * v0, w * v1, w * v2, w * v0 * v0, w * v1 * v1, w * v2 * v2};
        if (c == mine) {
          for (int k = 0; k < 8; ++k) acc[k] += val[k];
        } else {
          double* m = mom + c * kMomWords + off;
          for (int k = 0; k < 8; ++k) atomicAdd(m + k, val[k]);
        }
      }
    }
    for (size_t j = base + tw.ls[kLayerCap] + threadIdx.x; j < end; j += blockDim.x) {
      size_t c;
      double v[3];
      if (!slot_of(g, sp, j, &c, v)) continue;
      const double w = sp.w32[j];
      const double val[8] = {1.0, w, w * v[0], w * v[1], w * v[2], w * v[0] * v[0], w * v[1] * v[1],
                             w * v[2] * v[2]};
      double* m = mom + c * kMomWords + off;
      for (int k = 0; k < 8; ++k) atomicAdd(m + k, val[k]);
    }
    if (acc[0] != 0.0) {
      double* m = mom + mine * kMomWords + off;
      for (int k = 0; k < 8; ++k) atomicAdd(m + k, acc[k]);
    }
  }
}

// The state of cell c (row i) from its moment sums (st: axis temperatures,
// their means, weights, mean velocities, S), its list densities n, list
// counts N and collision numbers s_ee, s_ei, s_ii; false when the cell has
// fewer than two particles in a list or no positive temperature.
__device__ bool cell_state(const GridGeom& g, const LearnedPhys& ph, const double* m, int i,
                           double st[kStateWords], double n[2], double N[2], double s3[3]) {
  const double mass[2] = {ph.m_el, ph.m_ion}, q[2] = {ph.q_el, ph.q_ion};
  const double vol = kPi * g.dz * g.dr * g.dr * (2.0 * i + 1);
  for (int l = 0; l < 2; ++l) {
    const double* ml = m + 8 * l;
    N[l] = ml[0];
    const double W = ml[1];
    if (N[l] < 2.0 || !(W > 0.0)) return false;
    double tm = 0.0;
    for (int a = 0; a < 3; ++a) {
      const double u = ml[2 + a] / W;
      const double T = mass[l] * (ml[5 + a] / W - u * u) / kE;
      st[3 * l + a] = T;
      st[10 + 3 * l + a] = u;
      tm += T;
    }
    tm /= 3.0;
    if (!(tm > 0.0)) return false;
    st[6 + l] = tm;
    st[8 + l] = W;
    n[l] = W / vol;
  }
  auto s_of = [&](int a, int b) {
    const double mab = mass[a] * mass[b] / (mass[a] + mass[b]);
    const double v2 = 3.0 * kE * (st[6 + a] / mass[a] + st[6 + b] / mass[b]);
    const double qq = q[a] * q[b];
    const double em = kEps0 * mab;
    return fmax(n[a], n[b]) * ph.dt * kLogL * (qq * qq) / (4.0 * kPi * em * em * v2 * sqrt(v2));
  };
  s3[0] = s_of(0, 0);
  s3[1] = s_of(0, 1);
  s3[2] = s_of(1, 1);
  st[16] = s3[0] + s3[1] + s3[2];
  return true;
}

// The state and raw features of cell c (row i); false as cell_state.
__device__ bool cell_features(const GridGeom& g, const LearnedPhys& ph, const double* m, int i,
                              double st[kStateWords], float x[kFeatures]) {
  double n[2], N[2], s3[3];
  if (!cell_state(g, ph, m, i, st, n, N, s3)) return false;
  const double see = s3[0], sei = s3[1], sii = s3[2];
  for (int a = 0; a < 3; ++a) {
    x[a] = (float)(st[a] / st[6] - 1.0);
    x[3 + a] = (float)(st[3 + a] / st[7] - 1.0);
  }
  x[6] = (float)log(st[7] / st[6]);
  x[7] = (float)log10(see);
  x[8] = (float)log10(sei);
  x[9] = (float)log10(sii);
  double du2 = 0.0;
  for (int a = 0; a < 3; ++a) {
    const double d = st[10 + a] - st[13 + a];
    du2 += d * d;
  }
  x[10] = (float)sqrt(du2 / (3.0 * kE * st[6] / ph.m_el));
  x[11] = (float)log(n[1] / n[0]);
  x[12] = (float)(1.0 / sqrt(N[0] + N[1]));
  return true;
}

__global__ void features_kernel(GridGeom g, LearnedPhys ph, const double* mom, float* x, double* scale) {
  const size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (c >= (size_t)g.nr * g.nz) return;
  double st[kStateWords];
  float f[kFeatures];
  const bool ok = cell_features(g, ph, mom + c * kMomWords, (int)(c / g.nz), st, f);
  for (int k = 0; k < kFeatures; ++k) x[c * kFeatures + k] = ok ? f[k] : __int_as_float(0x7fc00000);
  scale[c] = ok ? st[16] : 0.0;
}

// The learned step's cells in three passes, so that the FP64 state and
// feature arithmetic runs at full occupancy and the tensor-core pass only
// moves operands:
//   learned_input_kernel: a thread per cell: features, the training-box
//     test (flag: 0 no collision, 1 learned, 2 binary fallback) and the
//     normalised BF16 network input (16 values, 32 bytes per cell);
//   learned_mlp_kernel: blocks take tiles of 128 cells in turn (weights
//     staged once per block), thread r the tile's cell r: the MLP on the
//     fifth-generation tensor cores (tcgen05.mma into tensor memory,
//     pcg_mlp_tc.cuh) for tiles with a learned cell, the 6 outputs stored;
//     a wait that times out sets count[2] and ends the block;
//   learned_xform_kernel: a thread per cell: the state again from the
//     moments, the new temperatures and the cell's transform.

__global__ void __launch_bounds__(kThreads) learned_input_kernel(GridGeom g, LearnedPhys ph, const double* mom,
                                                                 LearnedNorm nm, uint4* xin, unsigned char* flag,
                                                                 unsigned long long* count) {
  const size_t cells = (size_t)g.nr * g.nz;
  const size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  unsigned char stt = 0;
  float x[kFeatures];
  if (c < cells) {
    double st[kStateWords];
    if (cell_features(g, ph, mom + c * kMomWords, (int)(c / g.nz), st, x)) {
      stt = 1;
      for (int k = 0; k < kFeatures; ++k) {
        const float span = nm.x_hi[k] - nm.x_lo[k];
        if (!(x[k] >= nm.x_lo[k] - kBoxMargin * span && x[k] <= nm.x_hi[k] + kBoxMargin * span)) stt = 2;
      }
    }
    uint32_t pk[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      float v[2];
      for (int h = 0; h < 2; ++h) {
        const int k = 2 * q + h;
        v[h] = stt == 1 && k < kFeatures ? (x[k] - nm.x_mean[k]) / nm.x_std[k] : 0.f;
      }
      pk[q] = mlp::pack2(__float2bfloat16_rn(v[0]), __float2bfloat16_rn(v[1]));
    }
    xin[2 * c] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    xin[2 * c + 1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
    flag[c] = stt;
  }
  const int nl = __syncthreads_count(stt == 1), nf = __syncthreads_count(stt == 2);
  if (threadIdx.x == 0) {
    if (nl) atomicAdd(count, (unsigned long long)nl);
    if (nf) atomicAdd(count + 1, (unsigned long long)nf);
  }
}

__global__ void __launch_bounds__(mlp::tc::kThreads) learned_mlp_kernel(size_t cells, const float* P,
                                                                        const uint4* xin,
                                                                        const unsigned char* flag, float* yout,
                                                                        unsigned long long* count) {
  extern __shared__ __align__(16) unsigned char raw[];
  mlp::tc::Smem& sm = *reinterpret_cast<mlp::tc::Smem*>((reinterpret_cast<uintptr_t>(raw) + 1023) &
                                                        ~uintptr_t(1023));
  const size_t tiles = (cells + mlp::tc::kRows - 1) / mlp::tc::kRows;
  const int r = threadIdx.x;
  mlp::tc::load_weights(sm, P);
  mlp::tc::begin(sm);
  uint32_t phase = 0;
  unsigned char* a1 = reinterpret_cast<unsigned char*>(sm.A1);
  for (size_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const size_t c = tile * mlp::tc::kRows + r;
    const bool on = c < cells && flag[c] == 1;
    if (!__syncthreads_or(on)) continue;  // no learned cell in the tile (the same in every thread)
    const uint4 lo = on ? xin[2 * c] : make_uint4(0, 0, 0, 0), hi = on ? xin[2 * c + 1] : make_uint4(0, 0, 0, 0);
    *reinterpret_cast<uint4*>(a1 + mlp::tc::canon(r, 0, mlp::kInPad)) = lo;
    *reinterpret_cast<uint4*>(a1 + mlp::tc::canon(r, 8, mlp::kInPad)) = hi;
    float y[mlp::kOut];
    if (!mlp::tc::forward_tile(sm, phase, y)) {
      if (r == 0) atomicAdd(count + 2, 1ull);
      break;
    }
    if (on)
      for (int q = 0; q < mlp::kOut; ++q) yout[c * mlp::kOut + q] = y[q];
  }
  mlp::tc::end(sm, phase);
}

__global__ void __launch_bounds__(kThreads) learned_xform_kernel(GridGeom g, LearnedPhys ph, const double* mom,
                                                                 LearnedNorm nm, const float* yout,
                                                                 const unsigned char* flag, double* xform,
                                                                 const unsigned long long* count) {
  const size_t cells = (size_t)g.nr * g.nz;
  const size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (c >= cells || count[2]) return;
  double xf[12] = {0, 0, 0, 1, 1, 1, 0, 0, 0, 1, 1, 1};
  double st[kStateWords], n[2], N[2], s3[3];
  if (flag[c] == 1 && cell_state(g, ph, mom + c * kMomWords, (int)(c / g.nz), st, n, N, s3)) {
    double Tn[2][3], e0 = 0.0, e1 = 0.0;
    for (int l = 0; l < 2; ++l)
      for (int a = 0; a < 3; ++a) {
        const double yv = (double)yout[c * kTargets + 3 * l + a] * nm.y_std[3 * l + a] + nm.y_mean[3 * l + a];
        Tn[l][a] = st[3 * l + a] + st[6 + l] * st[16] * yv;
        e0 += st[8 + l] * st[3 * l + a];
        e1 += st[8 + l] * Tn[l][a];
      }
    const double f = e1 > 0.0 ? e0 / e1 : 1.0;  // the cell's thermal energy is kept
    for (int l = 0; l < 2; ++l)
      for (int a = 0; a < 3; ++a) {
        const double T = st[3 * l + a], T1 = fmax(Tn[l][a] * f, 1e-6 * st[6 + l]);
        xf[6 * l + a] = st[10 + 3 * l + a];
        xf[6 * l + 3 + a] = T > 0.0 ? sqrt(T1 / T) : 1.0;
      }
  }
  for (int q = 0; q < 12; ++q) xform[c * 12 + q] = xf[q];
}

// Applies the per-cell transforms; after a tensor-core time-out (count[2])
// the transforms are incomplete and nothing is applied.
__global__ void transform_kernel(GridGeom g, CollSpecies sp, const double* xform, const unsigned char* flag,
                                 const unsigned long long* count, size_t j0) {
  const size_t j = j0 + blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= sp.n || count[2]) return;
  size_t c;
  double v[3];
  if (!slot_of(g, sp, j, &c, v) || flag[c] != 1) return;
  const double* t = xform + c * 12 + (sp.is_ion ? 6 : 0);
  for (int a = 0; a < 3; ++a) v[a] = t[a] + (v[a] - t[a]) * t[3 + a];
  if (sp.cell) {
    sp.vr32[j] = (float)v[0]; sp.vphi32[j] = (float)v[1]; sp.vz32[j] = (float)v[2];
  } else {
    sp.vr64[j] = v[0]; sp.vphi64[j] = v[1]; sp.vz64[j] = v[2];
  }
}

// transform_kernel over the tile-sorted slots of a float species, walked
// as tile_moments_kernel walks them: thread lc reads its cell's transform
// once; a particle that has left its cell since the sort, and the run
// beyond kLayerCap layers, read their cell's from the grid.
__device__ __forceinline__ void apply_transform(const CollSpecies& sp, size_t j, double v[3], const double tr[6]) {
  for (int a = 0; a < 3; ++a) v[a] = tr[a] + (v[a] - tr[a]) * tr[3 + a];
  sp.vr32[j] = (float)v[0]; sp.vphi32[j] = (float)v[1]; sp.vz32[j] = (float)v[2];
}

__global__ void __launch_bounds__(kTileCells) tile_transform_kernel(GridGeom g, TileGrid tg, CollSpecies sp,
                                                                    const double* xform,
                                                                    const unsigned char* flag,
                                                                    const unsigned long long* count) {
  __shared__ TileWalk tw;
  if (count[2]) return;
  const int off = sp.is_ion ? 6 : 0, lc = threadIdx.x;
  for (int t = blockIdx.x; t < tg.ntiles; t += gridDim.x) {
    const size_t base = sp.tile_start[t], end = sp.tile_start[t + 1];
    if (base >= end) continue;  // the same for every thread of the block
    const unsigned cnt = sp.cell_count[(size_t)t * kTileCells + lc];
    tile_walk_begin(tw, sp.layer_start, sp.layer_prefix, t, cnt);
    const int ti = t / tg.ntz, tk = t - ti * tg.ntz;
    const int ci = ti * tg.tr + lc / tg.tz, ck = tk * tg.tz + lc % tg.tz;
    const size_t mine = (size_t)ci * g.nz + ck;
    const unsigned my_n = min(cnt, (unsigned)kLayerCap), wn = tile_walk_layers(cnt);
    double my_tr[6];
    const bool my_on = my_n > 0 && flag[mine] == 1;
    if (my_on)
      for (int k = 0; k < 6; ++k) my_tr[k] = xform[mine * 12 + off + k];
    for (unsigned q0 = 0; q0 < wn; q0 += kWalk) {
      size_t j[kWalk];
      int cell[kWalk];
      float vr[kWalk], vp[kWalk], vz[kWalk];
#pragma unroll
      for (int u = 0; u < kWalk; ++u) {
        const unsigned bal = __ballot_sync(0xffffffffu, my_n > q0 + u);
        j[u] = my_n > q0 + u ? base + tile_walk_slot(tw, q0 + u, bal) : ~(size_t)0;
      }
#pragma unroll
      for (int u = 0; u < kWalk; ++u) {
        cell[u] = j[u] != ~(size_t)0 ? sp.cell[j[u]] : kDeadCell;
        if (cell[u] >= 0) { vr[u] = sp.vr32[j[u]]; vp[u] = sp.vphi32[j[u]]; vz[u] = sp.vz32[j[u]]; }
      }
#pragma unroll
      for (int u = 0; u < kWalk; ++u) {
        if (cell[u] < 0) continue;
        const int pi = cell_r_of(cell[u]), pk = cell_z_of(cell[u]);
        if (pi < 0 || pi >= g.nr || pk >= g.nz) continue;
        const size_t c = (size_t)pi * g.nz + pk;
        double v[3] = {vr[u], vp[u], vz[u]};
        if (c == mine) {
          if (my_on) apply_transform(sp, j[u], v, my_tr);
        } else if (flag[c] == 1) {
          double tr[6];
          for (int k = 0; k < 6; ++k) tr[k] = xform[c * 12 + off + k];
          apply_transform(sp, j[u], v, tr);
        }
      }
    }
    for (size_t j = base + tw.ls[kLayerCap] + threadIdx.x; j < end; j += blockDim.x) {
      size_t c;
      double v[3];
      if (!slot_of(g, sp, j, &c, v) || flag[c] != 1) continue;
      double tr[6];
      for (int k = 0; k < 6; ++k) tr[k] = xform[c * 12 + off + k];
      apply_transform(sp, j, v, tr);
    }
  }
}

template <typename T>
int grow(T** p, size_t n) {
  cudaFree(*p);
  *p = nullptr;
  return cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T)) == cudaSuccess ? 0 : -1;
}

// a float species whose first slots are grouped by tile (the tile kernels' input)
bool tiled(const CollSpecies& sp) {
  return sp.cell && sp.tile_start && sp.cell_count && sp.layer_mask && sp.layer_prefix && sp.layer_start &&
         sp.sorted > 0 && sp.sorted <= sp.n;
}

unsigned tile_grid_blocks(const TileGrid& tg) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return (unsigned)std::max(1, std::min(tg.ntiles, sms * 8));
}

int ensure(const GridGeom& g, LearnedWork& w) {
  const size_t cells = (size_t)g.nr * g.nz;
  if (w.cells == cells && w.mom) return 0;
  if (grow(&w.mom, cells * kMomWords) || grow(&w.xform, cells * 12) || grow(&w.flag, cells) ||
      grow(&w.count, 3) || grow(&w.xin, 2 * cells) || grow(&w.yout, cells * kTargets))
    return -1;
  w.cells = cells;
  return 0;
}

}  // namespace

int learned_moments(const GridGeom& g, const CollSpecies* sp, int nsp, LearnedWork& w, cudaStream_t s) {
  if (ensure(g, w)) return -1;
  cudaMemsetAsync(w.mom, 0, w.cells * kMomWords * sizeof(double), s);
  const TileGrid tg = f32_tile_grid(g);
  const unsigned tile_blocks = tile_grid_blocks(tg);
  w.launches = 0;
  // the passes are latency-bound walks that only add to the sums: the
  // odd-numbered species' run on the second stream beside the others
  const bool fork = nsp >= 2 && w.aux && w.ev_fork && w.ev_join;
  if (fork && (cudaEventRecord(w.ev_fork, s) != cudaSuccess || cudaStreamWaitEvent(w.aux, w.ev_fork, 0) != cudaSuccess))
    return -1;
  for (int t = 0; t < nsp; ++t) {
    const cudaStream_t st = fork && (t & 1) ? w.aux : s;
    const size_t j0 = tiled(sp[t]) ? sp[t].sorted : 0;
    if (j0) tile_moments_kernel<<<tile_blocks, kTileCells, 0, st>>>(g, tg, sp[t], w.mom);
    if (sp[t].n > j0) moments_kernel<<<blocks_for(sp[t].n - j0), kThreads, 0, st>>>(g, sp[t], w.mom, j0);
    w.launches += (j0 ? 1 : 0) + (sp[t].n > j0 ? 1 : 0);
  }
  if (fork && (cudaEventRecord(w.ev_join, w.aux) != cudaSuccess || cudaStreamWaitEvent(s, w.ev_join, 0) != cudaSuccess))
    return -1;
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int learned_features(const GridGeom& g, const CollSpecies* sp, int nsp, const LearnedPhys& ph, LearnedWork& w,
                     float* x, double* scale, cudaStream_t s) {
  if (learned_moments(g, sp, nsp, w, s)) return -1;
  features_kernel<<<blocks_for(w.cells), kThreads, 0, s>>>(g, ph, w.mom, x, scale);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int learned_step(const GridGeom& g, const CollSpecies* sp, int nsp, const LearnedPhys& ph, LearnedWork& w,
                 unsigned long long counts[2], cudaStream_t s, bool apply) {
  if (!w.model) return -1;
  if (learned_moments(g, sp, nsp, w, s)) return -1;
  const size_t smem = sizeof(mlp::tc::Smem) + 1024;
  static const bool attr = cudaFuncSetAttribute(learned_mlp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)smem) == cudaSuccess;
  if (!attr) return -1;
  cudaMemsetAsync(w.count, 0, 3 * sizeof(unsigned long long), s);
  learned_input_kernel<<<blocks_for(w.cells), kThreads, 0, s>>>(g, ph, w.mom, w.norm, w.xin, w.flag, w.count);
  const size_t tiles = (w.cells + mlp::tc::kRows - 1) / mlp::tc::kRows;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const unsigned blocks = (unsigned)std::min<size_t>(tiles, (size_t)sms * 2);
  learned_mlp_kernel<<<blocks, mlp::tc::kThreads, smem, s>>>(w.cells, w.params, w.xin, w.flag, w.yout, w.count);
  learned_xform_kernel<<<blocks_for(w.cells), kThreads, 0, s>>>(g, ph, w.mom, w.norm, w.yout, w.flag, w.xform,
                                                                  w.count);
  w.launches += 3;
  const TileGrid tg = f32_tile_grid(g);
  const unsigned tile_blocks = tile_grid_blocks(tg);
  for (int t = 0; apply && t < nsp; ++t) {
    const size_t j0 = tiled(sp[t]) ? sp[t].sorted : 0;
    if (j0) tile_transform_kernel<<<tile_blocks, kTileCells, 0, s>>>(g, tg, sp[t], w.xform, w.flag, w.count);
    if (sp[t].n > j0)
      transform_kernel<<<blocks_for(sp[t].n - j0), kThreads, 0, s>>>(g, sp[t], w.xform, w.flag, w.count, j0);
    w.launches += (j0 ? 1 : 0) + (sp[t].n > j0 ? 1 : 0);
  }
  unsigned long long c3[3] = {0, 0, 0};
  if (cudaMemcpyAsync(c3, w.count, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return -1;
  if (c3[2]) return kLearnedTimeout;  // a wait for the tensor cores timed out; no velocity was changed
  counts[0] = c3[0];
  counts[1] = c3[1];
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int learned_set_model(LearnedWork& w, const float* params_host, const float* norm_host, cudaStream_t s) {
  if (!w.params && grow(&w.params, (size_t)mlp::kParams)) return -1;
  if (cudaMemcpyAsync(w.params, params_host, mlp::kParams * sizeof(float), cudaMemcpyHostToDevice, s) !=
          cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return -1;
  static_assert(sizeof(LearnedNorm) == kNormFloats * sizeof(float), "normalisation block");
  std::memcpy(&w.norm, norm_host, sizeof(LearnedNorm));
  w.model = true;
  return 0;
}

void learned_free(LearnedWork& w) {
  cudaFree(w.mom); cudaFree(w.xform); cudaFree(w.flag); cudaFree(w.count); cudaFree(w.params);
  cudaFree(w.xin); cudaFree(w.yout);
  w = LearnedWork();
}

}  // namespace pcg
