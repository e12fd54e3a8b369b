// pcg_collide_crowded.cu — the pairing sequence of crowded cells (more than
// CollParams::crowded particles), one warp per cell, for the binary collision pass of
// pcg_collide.cu.  Built with --fmad=false like the other FP64 kernels.
#include <cuda_runtime.h>

#include <algorithm>

#include "pcg_collide_pair.cuh"

namespace pcg {
namespace {

template <int SCHEME>
__device__ __forceinline__ void collide_pair(PairCtx& x, double ma, double mb, double qa, double qb,
                                             unsigned long long a, unsigned long long b, double na, double nb,
                                             double debye) {
  if (SCHEME == 1) ta77s_single(x, ma, mb, qa, qb, a, b, na, nb, debye);
  else if (SCHEME == 2) sk98_single(x, ma, mb, qa, qb, a, b, na, nb, debye);
  else p12_single(x, ma, mb, qa, qb, a, b, na, nb, debye);
}

// The pairing sequence of one crowded cell (collisionsP12.cpp:359-529;
// TA77S and SK98 repeat it), one warp per cell.  The reference runs the collisions of
// a cell one after another, numbered m = 0, 1, ... in its order: like pairs
// of ions, then of electrons (an odd list starts with the triangle (0,1),
// (1,2), (2,0)), then electron-ion pairs, where with unequal counts one
// electron meets several ions in turn (or one ion several electrons).  Here
// each collision keeps its number m, and with it its Philox draws, and the
// collisions that touch disjoint particles run on different lanes: the like
// pairs of a list, the triangle on one lane; the electron-ion pairs after
// all like pairs, one lane per electron (or ion) walking its partners in
// order, the two groups of unequal counts one after the other.  Every
// collision therefore sees the velocities it sees in the reference order
// and the results are the same.
template <int SCHEME>
__device__ void crowded_cell(size_t c, unsigned lane, const GridGeom& g, const Staged& tab, const CollParams& p,
                             const unsigned* st_e, const unsigned* n_e, const unsigned long long* le,
                             const unsigned* st_i, const unsigned* n_i, const unsigned long long* li,
                             const double* mom, const int* row_stop, unsigned long long* calls) {
  if (c >= (size_t)g.nr * g.nz) return;
  if (p.only && p.only[c] != p.only_value) return;
  if (n_e[c] + n_i[c] <= p.crowded) return;  // collide_cells_kernel takes the others
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
  unsigned m = 0;  // collisions of the cell before the current group
  auto coll = [&](double ma, double mb, double qa, double qb, unsigned long long a, unsigned long long b,
                  double na, double nb, unsigned mm) {
    x.m = mm;
    collide_pair<SCHEME>(x, ma, mb, qa, qb, a, b, na, nb, debye);
  };
  // like pairs of a list L of n: (0,1), (2,3), ... for even n; the triangle
  // and (3,4), (5,6), ... for odd n
  auto like = [&](const unsigned long long* L, unsigned n, double ms, double qs, double ns, bool odd) {
    if (!odd) {
      for (unsigned q = lane; q < n / 2; q += 32) coll(ms, ms, qs, qs, L[2 * q], L[2 * q + 1], ns, ns, m + q);
      m += n / 2;
      return;
    }
    if (n >= 3) {
      if (lane == 0) {
        coll(ms, ms, qs, qs, L[0], L[1], ns, ns, m);
        coll(ms, ms, qs, qs, L[1], L[2], ns, ns, m + 1);
        coll(ms, ms, qs, qs, L[2], L[0], ns, ns, m + 2);
      }
      m += 3;
    }
    if (n >= 5) {
      const unsigned np = (n - 3 + 1) / 2;  // q = 3, 5, ... < n
      for (unsigned q = lane; q < np; q += 32)
        coll(ms, ms, qs, qs, L[3 + 2 * q], L[4 + 2 * q], ns, ns, m + q);
      m += np;
    }
  };
  if (ni % 2 == 0) like(I, ni, mi, qi, n_ion, false);
  if (ne % 2 == 0) like(E, ne, me, qe, n_el, false);
  if (ni % 2 != 0) like(I, ni, mi, qi, n_ion, true);
  if (ne % 2 != 0) like(E, ne, me, qe, n_el, true);
  __syncwarp();  // the electron-ion pairs see every like collision's result
  if (ni == ne) {
    for (unsigned q = lane; q < ne; q += 32) coll(me, mi, qe, qi, E[q], I[q], n_el, n_ion, m + q);
    m += ne;
  }
  // One particle of the less numerous species meets `group` (or group + 1)
  // of the other in turn: lane per particle r of the first list, partners
  // s = 0 .. count-1 of the second whose index floor(s / d) (in float, as
  // the reference computes it) is r, collision number m + s.
  auto chains = [&](const unsigned long long* A, unsigned a_off, const unsigned long long* B, unsigned b_off,
                    unsigned count, float d, bool a_is_el) {
    if (!count) return;
    const unsigned owners = (unsigned)floorf((float)(count - 1) / d) + 1;
    for (unsigned r = lane; r < owners; r += 32) {
      // the partners of owner r form a run of s; start a little early for
      // the float rounding of s / d and keep those whose owner is r
      unsigned s0 = (unsigned)fmaxf(0.f, floorf((float)r * d) - 2.f);
      for (unsigned s = s0; s < count; ++s) {
        const unsigned own = (unsigned)(int)floorf((float)s / d);
        if (own < r) continue;
        if (own > r) break;
        if (a_is_el) coll(me, mi, qe, qi, A[own + a_off], B[s + b_off], n_el, n_ion, m + s);
        else coll(me, mi, qe, qi, B[s + b_off], A[own + a_off], n_el, n_ion, m + s);
      }
    }
    m += count;
  };
  if (ni > ne && ne > 0 && ni > 0) {
    const unsigned c_i = (unsigned)floorf((float)ni / (float)ne);
    const double c_r = (double)((float)ni / (float)ne - (float)c_i);
    const unsigned ions_1st = (unsigned)((double)(c_i + 1) * c_r * ne);
    const unsigned els_1st = (unsigned)(c_r * ne);
    const unsigned ions_2nd = (unsigned)((double)c_i * (1 - c_r) * ne);
    chains(E, 0, I, 0, ions_1st, (float)(c_i + 1), true);
    __syncwarp();  // the second group's first electron may be the first group's last
    chains(E, els_1st, I, ions_1st, ions_2nd, (float)c_i, true);
  }
  if (ni < ne && ne > 0 && ni > 0) {
    const double c_i = (double)floorf((float)ne / (float)ni);
    const double c_r = (double)((float)ne / (float)ni) - c_i;
    const unsigned els_1st = (unsigned)((c_i + 1) * c_r * ni);
    const unsigned ions_1st = (unsigned)(c_r * ni);
    const unsigned els_2nd = (unsigned)(c_i * (1 - c_r) * ni);
    chains(I, 0, E, 0, els_1st, (float)(c_i + 1), false);
    __syncwarp();
    chains(I, ions_1st, E, els_1st, els_2nd, (float)c_i, false);
  }
  if (lane == 0 && m) atomicAdd(calls, (unsigned long long)m);
  if (p.expect) {
#pragma unroll
    for (int q = 0; q < 12; ++q) {
      double v = expect[q];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) p.expect[c * 12 + q] = v;
    }
  }
}

// The crowded cells listed by the moments pass (list[0] cells in list[1..]),
// a warp per cell over a grid of fixed size: with no crowded cell the
// launch costs nothing in proportion to the grid.
template <int SCHEME>
__global__ void collide_kernel(GridGeom g, Staged tab, CollParams p, const unsigned* st_e,
                               const unsigned* n_e, const unsigned long long* le, const unsigned* st_i,
                               const unsigned* n_i, const unsigned long long* li, const double* mom,
                               const int* row_stop, unsigned long long* calls, const unsigned* list) {
  const unsigned lane = threadIdx.x & 31;
  const unsigned warps = (gridDim.x * blockDim.x) >> 5;
  const unsigned n = list[0];
  for (unsigned q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < n; q += warps)
    crowded_cell<SCHEME>(list[1 + q], lane, g, tab, p, st_e, n_e, le, st_i, n_i, li, mom, row_stop, calls);
}

}  // namespace

void collide_crowded(const GridGeom& g, double4* const stage[2], const CollParams& p, const unsigned* st_e,
                     const unsigned* n_e, const unsigned long long* le, const unsigned* st_i, const unsigned* n_i,
                     const unsigned long long* li, const double* mom, const int* row_stop, unsigned long long* calls,
                     const unsigned* list, cudaStream_t s) {
  const size_t cells = (size_t)g.nr * g.nz;
  const Staged tab{{stage[0], stage[1]}};
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // up to 8 blocks of kThreads / 32 warps per SM, no more warps than cells
  const size_t blocks = std::min<size_t>(blocks_for(32 * cells), (size_t)sms * 8);
  auto k = p.scheme == 1 ? collide_kernel<1> : p.scheme == 2 ? collide_kernel<2> : collide_kernel<0>;
  k<<<(unsigned)blocks, kThreads, 0, s>>>(g, tab, p, st_e, n_e, le, st_i, n_i, li, mom, row_stop, calls, list);
}

}  // namespace pcg
