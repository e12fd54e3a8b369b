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
#define PCG_PAIR_FN __device__ __forceinline__
#include "pcg_collide_pair.cuh"

namespace pcg {

namespace {

// ---------------------------------------------------------------------------
// 1. keys

// (the species comes by value: a run-time index into the by-value species
// table would copy the whole table to each thread's local memory)
// The key cell << cs | species << ts | id orders a list by cell, then
// species, then id (insertion order), in as few bits as the list needs.
__global__ void key_kernel(GridGeom g, CollSpecies sp, int t, unsigned long long* keys,
                           unsigned long long* vals, unsigned* n_valid,
                           const unsigned char* only, unsigned char only_value, int cs, int ts) {
  const size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  int ci = -1, ck = -1;
  unsigned id = 0;
  if (j < sp.n) {
    if (sp.cell) {
      const int c = sp.cell[j];
      ci = c < 0 ? -1 : cell_r_of(c);
      ck = c < 0 ? -1 : cell_z_of(c);
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
  // valid entries are appended (keys are unique, so the sort fixes the
  // order), one counter increment per block: per warp, the counter is one
  // address that every warp of the grid would wait on in turn
  __shared__ unsigned warp_n[kThreads / 32], block_base;
  const unsigned mask = __ballot_sync(0xffffffffu, valid);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) warp_n[wid] = __popc(mask);
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned tot = 0;
    for (int q = 0; q < kThreads / 32; ++q) {
      const unsigned v = warp_n[q];
      warp_n[q] = tot;
      tot += v;
    }
    block_base = tot ? atomicAdd(n_valid, tot) : 0u;
  }
  __syncthreads();
  const unsigned base = block_base + warp_n[wid];
  if (!valid) return;
  if (sp.cell) id = sp.id[j];
  const unsigned pos = base + __popc(mask & ((1u << lane) - 1u));
  keys[pos] = (c << cs) | ((unsigned long long)t << ts) | id;
  vals[pos] = ((unsigned long long)t << 40) | j;
}

// Each cell's run in the sorted keys: start[c] its first entry, end[c] one
// past its last (both 0 for a cell without entries, cleared before).
__global__ void bounds_kernel(const unsigned long long* keys, unsigned n, int cs, unsigned* start, unsigned* end) {
  const size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (e >= n) return;
  const unsigned long long c = keys[e] >> cs;
  if (e == 0 || (keys[e - 1] >> cs) != c) start[c] = (unsigned)e;
  if (e + 1 == n || (keys[e + 1] >> cs) != c) end[c] = (unsigned)e + 1;
}

// count[c] = end[c] - start[c], in place of end
__global__ void run_count_kernel(size_t cells, const unsigned* start, unsigned* count) {
  const size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (c < cells) count[c] -= start[c];
}

// ---------------------------------------------------------------------------
// 3. shuffle

// The partner of position i in the Fisher-Yates pass of cell c.
__device__ __forceinline__ unsigned shuffle_partner(size_t c, unsigned i, uint64_t seed, uint32_t pass,
                                                    uint32_t list) {
  uint32_t o[4];
  philox4x32_10((uint32_t)c, i, pass, kShufTag + list, (uint32_t)seed, (uint32_t)(seed >> 32), o);
  const unsigned j = (unsigned)(u53(o[0], o[1]) * (double)(i + 1));
  return j > i ? i : j;
}

// A warp per cell: the lanes draw every position's partner at once and
// stage the list in shared memory, one lane makes the swaps in order (the
// same permutation as one thread drawing and swapping in turn), and the
// lanes write the list back.  A list longer than kShufCap is shuffled by
// one lane in place.
constexpr unsigned kShufCap = 256;
__global__ void shuffle_kernel(size_t cells, const unsigned* start, const unsigned* count,
                               unsigned long long* vals, uint64_t seed, uint32_t pass, uint32_t list) {
  __shared__ unsigned long long buf[kThreads / 32][kShufCap];
  __shared__ unsigned short part[kThreads / 32][kShufCap];
  const unsigned lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  // a warp reads the counts of 32 cells at once and takes the ones with a
  // list of two or more in turn (a pass over chosen cells leaves most empty)
  const size_t stride = (size_t)gridDim.x * (kThreads / 32) * 32;
  for (size_t c0 = (blockIdx.x * (size_t)(kThreads / 32) + w) * 32; c0 < cells; c0 += stride) {
    const unsigned nl = c0 + lane < cells ? count[c0 + lane] : 0u;
    unsigned todo = __ballot_sync(0xffffffffu, nl >= 2);
    while (todo) {
    const int b = __ffs(todo) - 1;
    todo &= todo - 1;
    const size_t c = c0 + b;
    const unsigned n = __shfl_sync(0xffffffffu, nl, b);
    unsigned long long* L = vals + start[c];
    if (n > kShufCap) {
      if (lane == 0)
        for (unsigned i = 1; i < n; ++i) {
          const unsigned j = shuffle_partner(c, i, seed, pass, list);
          const unsigned long long tmp = L[i];
          L[i] = L[j];
          L[j] = tmp;
        }
      __syncwarp();
      continue;
    }
    for (unsigned i = lane; i < n; i += 32) {
      buf[w][i] = L[i];
      part[w][i] = i ? (unsigned short)shuffle_partner(c, i, seed, pass, list) : 0;
    }
    __syncwarp();
    if (lane == 0)
      for (unsigned i = 1; i < n; ++i) {
        const unsigned j = part[w][i];
        const unsigned long long tmp = buf[w][i];
        buf[w][i] = buf[w][j];
        buf[w][j] = tmp;
      }
    __syncwarp();
    for (unsigned i = lane; i < n; i += 32) L[i] = buf[w][i];
    __syncwarp();
    }
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
                               int* row_stop, double* totals, unsigned* crowded, unsigned* active) {
  const size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (c >= (size_t)g.nr * g.nz) return;
  // a pass over chosen cells: the others are neither collided nor stop a row
  if (p.only && p.only[c] != p.only_value) return;
  if (n_e[c] + n_i[c] > p.crowded) crowded[1 + atomicAdd(crowded, 1u)] = (unsigned)c;
  else if (p.only) active[1 + atomicAdd(active, 1u)] = (unsigned)c;
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

// Cells of up to p.crowded particles run their pairing sequence on one
// thread (collide_cells_kernel): with the whole grid's cells in flight that
// keeps the FP64 units busier than spreading a cell over a warp (measured
// 79 ms against 120 ms per pass at 100 + 100 per cell).  Crowded cells (a
// dense bunch) take a warp each (collide_kernel), so one cell's serial
// sequence no longer sets the pass's duration.  Both give the same result.
// (The threshold is a CollParams field, 256 by default.)

// The pairing sequence of a cell (collisionsP12.cpp:359-529; TA77S and SK98
// repeat it), as the collision numbers m = 0, 1, ... of the reference's
// order: like pairs of an even list of ions, of an even list of electrons,
// then of an odd ion list (the triangle (0,1), (1,2), (2,0), then (3,4),
// (5,6), ...) and of an odd electron list, then electron-ion pairs, where
// with unequal counts one particle of the less numerous list meets several
// of the other in turn, in two groups (the split the reference computes in
// float).
struct PairPlan {
  unsigned seg[3];  // collisions of the first like list, the second, then electron-ion
  int first_ion;    // the first like list is the ions'
  unsigned total;
  // electron-ion groups (unequal counts)
  unsigned g1, g2, off_few, off_many;  // group sizes; index offsets of the second group
  float d1, d2;                        // partners per particle of each group, as floats
};

__device__ __forceinline__ unsigned like_count(unsigned n) { return n % 2 == 0 ? n / 2 : (n >= 3 ? 3 + (n - 3) / 2 : 0); }

__device__ __forceinline__ PairPlan pair_plan(unsigned ne, unsigned ni) {
  PairPlan q{};
  // even lists first, ions before electrons in each parity
  q.first_ion = (ni % 2 == 0) || (ne % 2 != 0);
  q.seg[0] = like_count(q.first_ion ? ni : ne);
  q.seg[1] = like_count(q.first_ion ? ne : ni);
  if (ni == ne) {
    q.seg[2] = ne;
  } else if (ne > 0 && ni > 0 && ni > ne) {
    const unsigned c_i = (unsigned)floorf((float)ni / (float)ne);
    const double c_r = (double)((float)ni / (float)ne - (float)c_i);
    q.g1 = (unsigned)((double)(c_i + 1) * c_r * ne);  // ions of the first group
    q.off_few = (unsigned)(c_r * ne);                  // electrons of the first group
    q.g2 = (unsigned)((double)c_i * (1 - c_r) * ne);
    q.off_many = q.g1;
    q.d1 = (float)(c_i + 1);
    q.d2 = (float)c_i;
    q.seg[2] = q.g1 + q.g2;
  } else if (ne > 0 && ni > 0 && ni < ne) {
    const double c_i = (double)floorf((float)ne / (float)ni);
    const double c_r = (double)((float)ne / (float)ni) - c_i;
    q.g1 = (unsigned)((c_i + 1) * c_r * ni);  // electrons of the first group
    q.off_few = (unsigned)(c_r * ni);         // ions of the first group
    q.g2 = (unsigned)(c_i * (1 - c_r) * ni);
    q.off_many = q.g1;
    q.d1 = (float)(c_i + 1);
    q.d2 = (float)c_i;
    q.seg[2] = q.g1 + q.g2;
  }
  q.total = q.seg[0] + q.seg[1] + q.seg[2];
  return q;
}

struct PairRef {
  int kind;  // 0: ion-ion, 1: electron-electron, 2: electron (a) - ion (b)
  unsigned a, b;
};

__device__ __forceinline__ void like_pair(unsigned n, unsigned k, unsigned* a, unsigned* b) {
  if (n % 2 == 0) { *a = 2 * k; *b = 2 * k + 1; return; }
  if (k < 3) { *a = k; *b = k == 2 ? 0 : k + 1; return; }
  *a = 3 + 2 * (k - 3);
  *b = *a + 1;
}

__device__ __forceinline__ PairRef pair_of(const PairPlan& q, unsigned m, unsigned ne, unsigned ni) {
  PairRef r;
  if (m < q.seg[0] + q.seg[1]) {
    const bool first = m < q.seg[0];
    const bool ion = first ? q.first_ion : !q.first_ion;
    r.kind = ion ? 0 : 1;
    like_pair(ion ? ni : ne, first ? m : m - q.seg[0], &r.a, &r.b);
    return r;
  }
  const unsigned k = m - q.seg[0] - q.seg[1];
  r.kind = 2;
  if (ni == ne) { r.a = k; r.b = k; return r; }
  // the many-list index s, the few-list owner floor(s / d) (float, as in the reference)
  unsigned few, many;
  if (k < q.g1) {
    many = k;
    few = (unsigned)(int)floorf((float)k / q.d1);
  } else {
    const unsigned s2 = k - q.g1;
    many = s2 + q.off_many;
    few = (unsigned)(int)floorf((float)s2 / q.d2) + q.off_few;
  }
  if (ni > ne) { r.a = few; r.b = many; } else { r.a = many; r.b = few; }
  return r;
}

// One cell's pairing sequence (collisionsP12.cpp:359-529) on one thread.
template <int SCHEME>
__global__ void __launch_bounds__(kThreads, 2) collide_cells_kernel(GridGeom g, Staged tab, CollParams p, const unsigned* st_e,
                               const unsigned* n_e, const unsigned long long* le, const unsigned* st_i,
                               const unsigned* n_i, const unsigned long long* li, const double* mom,
                               const int* row_stop, unsigned long long* calls, const unsigned* list) {
  // a pass over chosen cells takes them from the list the moments pass
  // made (the chosen cells packed into whole warps), else thread c, cell c
  const size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (list && tid >= list[0]) return;
  const size_t c = list ? list[1 + tid] : tid;
  if (c >= (size_t)g.nr * g.nz) return;
  if (p.only && p.only[c] != p.only_value) return;
  if (n_e[c] + n_i[c] > p.crowded) return;  // collide_kernel takes the crowded cells
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
  // The sequence as one loop over the collision number m with a single
  // call of the pair function: cells of different counts in a warp then
  // run the same code and diverge only in their trip counts.
  const PairPlan plan = pair_plan(ne, ni);
  for (unsigned m = 0; m < plan.total; ++m) {
    const PairRef r = pair_of(plan, m, ne, ni);
    const bool ion_a = r.kind == 0, el_b = r.kind == 1;
    const unsigned long long A = ion_a ? I[r.a] : E[r.a];
    const unsigned long long B = el_b ? E[r.b] : I[r.b];
    const double ma = ion_a ? mi : me, qa = ion_a ? qi : qe, na = ion_a ? n_ion : n_el;
    const double mb = el_b ? me : mi, qb = el_b ? qe : qi, nb = el_b ? n_el : n_ion;
    x.m = m;
    if (SCHEME == 1) ta77s_single(x, ma, mb, qa, qb, A, B, na, nb, debye);
    else if (SCHEME == 2) sk98_single(x, ma, mb, qa, qb, A, B, na, nb, debye);
    else p12_single(x, ma, mb, qa, qb, A, B, na, nb, debye);
  }
  x.m = plan.total;
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
  cudaFree(w.crowded); cudaFree(w.active);
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
  size_t need = std::max(total[0], total[1]);
  if (w.cap < need || w.cells != cells) {
    need += need / 4 + 4096;  // headroom: an injected beam grows the lists every step
    for (int l = 0; l < 2; ++l) {
      if (grow(&w.keys[l], need) || grow(&w.keys2[l], need) || grow(&w.vals[l], need) ||
          grow(&w.vals2[l], need) || grow(&w.count[l], cells + 1) || grow(&w.start[l], cells + 1) ||
          grow(&w.stage[l], need))
        return -1;
    }
    if (grow(&w.moments, 4 * cells) || grow(&w.row_stop, (size_t)g.nr) || grow(&w.calls, 1) ||
        grow(&w.valid, 2) || grow(&w.crowded, cells + 1) || grow(&w.active, cells + 1))
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
  cudaMemsetAsync(w.crowded, 0, sizeof(unsigned), s);
  cudaMemsetAsync(w.active, 0, sizeof(unsigned), s);
  w.launches = 3;  // moments and the pairs of ordinary and of crowded cells
  // bits of the sort keys: id (below the largest id bound of a species), species, cell
  auto width = [](unsigned long long v) { int b = 0; while (b < 64 && (v >> b) != 0) ++b; return b; };
  unsigned long long max_id = 0;
  for (int t = 0; t < nsp; ++t)
    max_id = std::max<unsigned long long>(max_id, sp[t].cell ? sp[t].id_bound : sp[t].n);
  const int id_bits = std::max(1, width(max_id)), sp_bits = std::max(1, width((unsigned long long)(nsp - 1)));
  const int key_ts = id_bits, key_cs = id_bits + sp_bits, key_bits = key_cs + std::max(1, width(cells - 1));
  if (key_bits > 64) return -1;
  for (int l = 0; l < 2; ++l) {
    for (int t = 0; t < nsp; ++t) {
      if ((sp[t].is_ion ? 1 : 0) != l || !sp[t].n) continue;
      key_kernel<<<blocks_for(sp[t].n), kThreads, 0, s>>>(g, sp[t], t, w.keys[l], w.vals[l], w.valid + l, p.only,
                                                          p.only_value, key_cs, key_ts);
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
      cub::DeviceRadixSort::SortPairs(w.tmp, b, w.keys[l], w.keys2[l], w.vals[l], w.vals2[l],
                                      (int)valid[l], 0, key_bits, s);
    }
    // per cell the run of its entries in the sorted list (count = end - start)
    cudaMemsetAsync(w.start[l], 0, (cells + 1) * sizeof(unsigned), s);
    cudaMemsetAsync(w.count[l], 0, (cells + 1) * sizeof(unsigned), s);
    if (valid[l]) {
      bounds_kernel<<<blocks_for(valid[l]), kThreads, 0, s>>>(w.keys2[l], valid[l], key_cs, w.start[l], w.count[l]);
      run_count_kernel<<<blocks_for(cells), kThreads, 0, s>>>(cells, w.start[l], w.count[l]);
      w.launches += 2;
    }
    if (p.shuffle && valid[l]) {
      int dev = 0, sms = 148;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      const size_t blocks = std::min<size_t>((cells + kThreads / 32 - 1) / (kThreads / 32), (size_t)sms * 16);
      shuffle_kernel<<<(unsigned)blocks, kThreads, 0, s>>>(cells, w.start[l], w.count[l], w.vals2[l], p.seed,
                                                          p.pass, (uint32_t)l);
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
                                                        w.row_stop, p.scheme == 1 ? w.totals : nullptr,
                                                        w.crowded, w.active);
  auto cells_k = p.scheme == 1 ? collide_cells_kernel<1>
                 : p.scheme == 2 ? collide_cells_kernel<2> : collide_cells_kernel<0>;
  cells_k<<<blocks_for(cells), kThreads, 0, s>>>(g, staged, p, w.start[0], w.count[0], w.keys2[0], w.start[1],
                                                 w.count[1], w.keys2[1], w.moments, w.row_stop, w.calls,
                                                 p.only ? w.active : nullptr);
  collide_crowded(g, staged.stage, p, w.start[0], w.count[0], w.keys2[0], w.start[1], w.count[1], w.keys2[1],
                  w.moments, w.row_stop, w.calls, w.crowded, s);
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
