// pcg_kernels_f32.cu — the single-precision production path: float Yee
// update, species buffers in (cell, offset) form, import/export, beam
// injection, the tile sort and the fused particle step.
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "pcg.h"
#include "pcg_f32.h"
#include "pcg_f32_pair.cuh"
#include "pcg_f32_step.cuh"
#include "pcg_philox.cuh"
#include "pcg_yee.cuh"

namespace pcg {

namespace {

constexpr int kThreads = 256;

inline unsigned blocks_for(size_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

// Position in metres -> (cell, offset) with 0 <= offset < 1.
// The cell is the reference's CELL_NUMBER (floor(pos / cell size) in
// double, geometry.hpp:198); an offset that rounds up to 1 in float stays
// the largest float below 1, so that the cell never differs from it.
__device__ __forceinline__ void split_position(double x_m, double d, int* cell, float* off) {
  const double x = x_m / d;
  const double c = floor(x);
  float f = (float)(x - c);
  if (f >= 1.0f) f = 0x1.fffffep-1f;
  *cell = (int)c;
  *off = f;
}

// The float layout's cell word of a position.  A position outside the
// grid becomes a dead slot, counted as removed, as the runaway collector
// removes such particles (SMB.cpp:252-337: r < 0, z < 0, r >= R, z >= L):
// the cell of such a position has no tile to be sorted into.  The double
// layout stops a step at positions more than a cell beyond the grid
// (kErrOutOfGrid) and at positions that are not finite numbers
// (kErrNanPosition, the reference's fatal error, pusherBoris.cpp:51-57);
// both are raised here too, and the particle dropped.
__device__ __forceinline__ int place(const GridGeom& g, double r, double z, float* fr, float* fz, DevStatus* st) {
  bool dead = false;
  if (!(isfinite(r) && isfinite(z))) {
    raise_error(st, kErrNanPosition);
    dead = true;
  } else if (!(r >= 0.0 && z >= 0.0 && r / g.dr < (double)g.nr && z / g.dz < (double)g.nz)) {
    if (!(r >= -1.5 * g.dr && r < (g.nr + 1) * g.dr && z >= -1.5 * g.dz && z < (g.nz + 1) * g.dz))
      raise_error(st, kErrOutOfGrid);
    dead = true;
  }
  int ci = 0, ck = 0;
  if (!dead) {
    split_position(r, g.dr, &ci, fr);
    split_position(z, g.dz, &ck, fz);
    dead = ci < 0 || ck < 0 || ci >= g.nr || ck >= g.nz;
  }
  if (dead) {
    *fr = *fz = 0.f;
    atomicAdd(&st->removed, 1ull);
    atomicAdd(&st->dead_slots, 1ull);
    return kDeadCell;
  }
  return pack_cell(ci, ck);
}

__global__ void import_kernel(GridGeom g, SpeciesF32Buffers b, size_t n0, size_t n,
                              const double* src, DevStatus* st) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  size_t j = n0 + i;
  float fr, fz;
  b.cell[j] = place(g, src[i], src[n + i], &fr, &fz, st);
  b.off_r[j] = fr;
  b.off_z[j] = fz;
  b.vr[j] = (float)src[2 * n + i];
  b.vphi[j] = (float)src[3 * n + i];
  b.vz[j] = (float)src[4 * n + i];
  b.w[j] = (float)src[5 * n + i];
  b.id[j] = b.next_id + (unsigned)i;
}

// BeamP::inject (beamP.cpp:100-145), or the Gaussian bunch, with the same
// Philox stream as the double path; positions are computed in double.
__global__ void inject_kernel(GridGeom g, SpeciesF32Buffers b, size_t n0, unsigned count,
                              BeamInject bi, DevStatus* st) {
  unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const double dr = g.dr, dz = g.dz;
  double u[2];
  philox_uniform2(bi.seed, bi.stream, bi.step, i, u);
  double pos_r, pos_z, wgt;
  beam_particle(bi, dr, dz, u, &pos_r, &pos_z, &wgt);
  const size_t j = n0 + i;
  float fr, fz;
  b.cell[j] = place(g, pos_r, pos_z, &fr, &fz, st);  // a bunch wider than the domain loses its edge
  b.off_r[j] = fr;
  b.off_z[j] = fz;
  b.vr[j] = 0.f;
  b.vphi[j] = 0.f;
  b.vz[j] = (float)bi.velocity;
  b.w[j] = (float)wgt;
  b.id[j] = b.next_id + i;
}

__global__ void alive_kernel(const int* cell, unsigned char* flags, size_t n) {
  size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j < n) flags[j] = cell[j] >= 0 ? 1 : 0;
}

template <typename T>
__global__ void gather_kernel(const T* src, T* dst, const unsigned* idx, size_t n) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[idx[i]];
}

__global__ void iota_kernel(unsigned* a, size_t n) {
  size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j < n) a[j] = (unsigned)j;
}

// Export in insertion order: perm[m] is the slot of the m-th smallest id.
__global__ void export_kernel(GridGeom g, SpeciesF32Buffers b, size_t n, const unsigned* perm,
                              double* out, int* cells) {
  size_t m = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (m >= n) return;
  const size_t j = perm[m];
  const int c = b.cell[j];
  const int ci = cell_r_of(c), ck = cell_z_of(c);
  out[m] = ((double)ci + (double)b.off_r[j]) * g.dr;
  out[n + m] = ((double)ck + (double)b.off_z[j]) * g.dz;
  out[2 * n + m] = b.vr[j];
  out[3 * n + m] = b.vphi[j];
  out[4 * n + m] = b.vz[j];
  out[5 * n + m] = b.w[j];
  cells[m] = ci;
  cells[n + m] = ck;
}

// ---------------------------------------------------------------------------
// Tile sort: live particles grouped by tile, and inside a tile in layered
// order: layer q holds the particles of rank q in their cell (the q-th to
// arrive there), one per occupied cell, in cell order (z fastest).  A warp
// then takes 32 particles of 32 neighbouring cells, so its gathers from and
// deposits to the block's shared windows hit distinct addresses and banks.

static_assert(kTileCells % 32 == 0, "layer masks hold whole 32-cell words");

// tile of a packed cell and the cell's index inside the tile (z fastest)
__device__ __forceinline__ int tile_key(int cell, const TileGrid& tg, int* lc) {
  if (cell < 0) return -1;
  const int ci = cell_r_of(cell), ck = cell_z_of(cell);
  const int tr = ci / tg.tr, tz = ck / tg.tz;
  *lc = (ci - tr * tg.tr) * tg.tz + (ck - tz * tg.tz);
  return tr * tg.ntz + tz;
}

// rank of each particle in its cell (warp-aggregated counter increments)
__global__ void cell_rank_kernel(const int* cell, size_t n, TileGrid tg, unsigned* cell_count,
                                 unsigned* rank) {
  const size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  int lc = 0;
  const int t = j < n ? tile_key(cell[j], tg, &lc) : -1;
  const int key = t < 0 ? -1 : t * kTileCells + lc;
  const unsigned mask = __match_any_sync(0xffffffffu, key);
  const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
  unsigned base = 0;
  if (lane == leader && key >= 0) base = atomicAdd(cell_count + key, (unsigned)__popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (j < n) rank[j] = key < 0 ? ~0u : base + __popc(mask & ((1u << lane) - 1u));
}

// One block per tile: the tile's particle count and its layer tables.
__global__ void __launch_bounds__(kThreads) tile_layers_kernel(TileGrid tg, SpeciesF32Buffers b,
                                                               unsigned* tile_count) {
  __shared__ unsigned cnt[kTileCells];
  __shared__ unsigned layer_size[kLayerCap];
  __shared__ unsigned red_max[kThreads / 32], red_sum[kThreads / 32];
  const int t = blockIdx.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned mx = 0, sum = 0;
  for (int c = threadIdx.x; c < kTileCells; c += blockDim.x) {
    const unsigned v = b.cell_count[(size_t)t * kTileCells + c];
    cnt[c] = v;
    mx = max(mx, v);
    sum += v;
  }
  for (int o = 16; o > 0; o >>= 1) {
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    sum += __shfl_xor_sync(0xffffffffu, sum, o);
  }
  if (lane == 0) { red_max[wid] = mx; red_sum[wid] = sum; }
  __syncthreads();
  mx = 0; sum = 0;
  for (int w = 0; w < kThreads / 32; ++w) { mx = max(mx, red_max[w]); sum += red_sum[w]; }
  if (threadIdx.x == 0) {
    tile_count[t] = sum;
    b.overflow[t] = 0;
    if (sum) { atomicMax(b.sort_info, sum); atomicAdd(b.sort_info + 1, 1u); }
  }
  const int nq = (int)min(mx, (unsigned)kLayerCap);
  // layer q: word w of the mask has bit l set when cell 32 w + l holds more than q
  for (int q = wid; q < nq; q += kThreads / 32) {
    unsigned mine = 0;
    for (int w = 0; w < kTileWords; ++w) {
      const unsigned m = __ballot_sync(0xffffffffu, cnt[w * 32 + lane] > (unsigned)q);
      if (lane == w) mine = m;
    }
    // exclusive prefix of the set bits over the words (lanes 0..15)
    const unsigned pc = lane < kTileWords ? __popc(mine) : 0u;
    unsigned incl = pc;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    const size_t at = ((size_t)t * kLayerCap + q) * kTileWords + lane;
    if (lane < kTileWords) {
      b.layer_mask[at] = mine;
      b.layer_prefix[at] = (unsigned short)(incl - pc);
    }
    if (lane == 31) layer_size[q] = incl;
  }
  __syncthreads();
  if (wid == 0) {  // layer starts: exclusive scan of the layer sizes, 4 per lane
    unsigned v[kLayerCap / 32], tot = 0;
    for (int r = 0; r < kLayerCap / 32; ++r) {
      const int q = lane * (kLayerCap / 32) + r;
      v[r] = q < nq ? layer_size[q] : 0u;
      tot += v[r];
    }
    unsigned incl = tot;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned x = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += x;
    }
    unsigned run = incl - tot;
    unsigned* ls = b.layer_start + (size_t)t * (kLayerCap + 1);
    for (int r = 0; r < kLayerCap / 32; ++r) {
      ls[lane * (kLayerCap / 32) + r] = run;
      run += v[r];
    }
    if (lane == 31) ls[kLayerCap] = run;  // the overflow run starts after all kept layers
  }
}

__global__ void tile_scatter_kernel(SpeciesF32Buffers b, size_t n, TileGrid tg) {
  const size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= n) return;
  int lc = 0;
  const int t = tile_key(b.cell[j], tg, &lc);
  if (t < 0) return;
  const unsigned q = b.rank[j];
  unsigned pos = b.tile_start[t];
  if (q < (unsigned)kLayerCap) {
    const size_t at = ((size_t)t * kLayerCap + q) * kTileWords + (lc >> 5);
    pos += b.layer_start[(size_t)t * (kLayerCap + 1) + q] + b.layer_prefix[at] +
           __popc(b.layer_mask[at] & ((1u << (lc & 31)) - 1u));
  } else {
    pos += b.layer_start[(size_t)t * (kLayerCap + 1) + kLayerCap] + atomicAdd(b.overflow + t, 1u);
  }
  b.cell2[pos] = b.cell[j];
  b.off_r2[pos] = b.off_r[j];
  b.off_z2[pos] = b.off_z[j];
  b.vr2[pos] = b.vr[j];
  b.vphi2[pos] = b.vphi[j];
  b.vz2[pos] = b.vz[j];
  b.w2[pos] = b.w[j];
  b.id2[pos] = b.id[j];
}

void swap_buffers(SpeciesF32Buffers& b) {
  std::swap(b.cell, b.cell2);
  std::swap(b.off_r, b.off_r2);
  std::swap(b.off_z, b.off_z2);
  std::swap(b.vr, b.vr2);
  std::swap(b.vphi, b.vphi2);
  std::swap(b.vz, b.vz2);
  std::swap(b.w, b.w2);
  std::swap(b.id, b.id2);
}

// Blocks per tile for the step: enough that about target_blocks blocks run
// when few tiles are occupied (a narrow beam), each with at least min_split
// particles (F32Step; the defaults 148 x 16 and 1024 suit one run on the GPU).
// Computed on the device after a sort into info[2] (info[0] the largest
// tile, info[1] the occupied tiles), with info[3] the live slots.
__global__ void sort_finish_kernel(unsigned* info, const unsigned* live, unsigned target_blocks, unsigned min_split,
                                   unsigned* epoch) {
  *epoch += 1;  // drift[1]: the sorts so far, copied to the host with each step's drift count
  const unsigned largest = info[0], occupied = info[1];
  unsigned splits = 1;
  if (occupied) {
    splits = max(1u, min((target_blocks + occupied - 1) / occupied, (largest + min_split - 1) / min_split));
    splits = min(splits, 65535u);
  }
  info[2] = splits;
  info[3] = *live;
}

// The slots from the live count on (the dead slots the sort dropped) read
// as dead in the sorted buffer.
__global__ void fill_dead_kernel(int* cell, const unsigned* live, size_t n) {
  const size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j < n && j >= *live) cell[j] = kDeadCell;
}

// A tile sort of the species' n slots.  With `wait` the host reads the
// outcome (the live count becomes n, the blocks per tile exact); without,
// nothing waits for the stream: n stays, the dropped dead slots remain as
// dead slots after the tiles, and the step's launch takes the blocks per
// tile of the last sort the host has seen (the kernels use the device's
// value, up to that many).
int tile_sort(const TileGrid& tg, unsigned target_blocks, unsigned min_split, SpeciesF32Buffers& b,
              size_t* n, cudaStream_t s, bool wait) {
  const size_t nt = (size_t)tg.ntiles;
  unsigned* counts = b.tile_cursor;
  cudaMemsetAsync(b.cell_count, 0, nt * kTileCells * sizeof(unsigned), s);
  cudaMemsetAsync(counts + nt, 0, sizeof(unsigned), s);
  cudaMemsetAsync(b.sort_info, 0, 4 * sizeof(unsigned), s);
  if (*n) cell_rank_kernel<<<blocks_for(*n), kThreads, 0, s>>>(b.cell, *n, tg, b.cell_count, b.rank);
  tile_layers_kernel<<<(unsigned)nt, kThreads, 0, s>>>(tg, b, counts);
  size_t tmp = b.scan_tmp_bytes;
  cub::DeviceScan::ExclusiveSum(b.scan_tmp, tmp, counts, b.tile_start, (int)(nt + 1), s);
  if (*n) tile_scatter_kernel<<<blocks_for(*n), kThreads, 0, s>>>(b, *n, tg);
  sort_finish_kernel<<<1, 1, 0, s>>>(b.sort_info, b.tile_start + nt, target_blocks, min_split, b.drift + 1);
  if (*n) fill_dead_kernel<<<blocks_for(*n), kThreads, 0, s>>>(b.cell2, b.tile_start + nt, *n);
  b.launches += (*n ? 4 : 0) + 2 + 2;  // rank, scatter, dead fill; layers, finish; the scan's two kernels
  const unsigned hint = b.host_info[2];  // the blocks per tile of an earlier sort
  cudaMemcpyAsync(b.host_info, b.sort_info, 4 * sizeof(unsigned), cudaMemcpyDeviceToHost, s);
  swap_buffers(b);
  // a sort inside a stream capture (an ensemble's graph) cannot wait: the
  // first sort of a species then launches with the earlier hint (one block
  // per tile unless an earlier sort said more; the kernels take what runs)
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  const bool capturing = cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone;
  if (wait && capturing) return -1;
  if (wait || (b.sorts == 0 && !capturing)) {
    if (cudaStreamSynchronize(s) != cudaSuccess) return -1;
    if (wait) *n = b.host_info[3];
    b.splits = (int)std::max(1u, b.host_info[2]);
  } else {
    b.splits = (int)std::max(1u, std::min(hint, 65535u));
  }
  b.sorts += 1;
  b.sorted_n = *n;
  b.steps_since_sort = 0;
  return 0;
}

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double part[kThreads / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) part[wid] = v;
  __syncthreads();
  v = threadIdx.x < kThreads / 32 ? part[threadIdx.x] : 0.0;
  if (wid == 0)
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

struct Fld12 {
  const float* f[12];
};

__global__ void energy_kernel(GridGeom g, Fld12 fl, double* out) {
  double ee = 0, eh = 0;
  const long long total = (long long)g.nr * g.nz;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q / g.nz), k = (int)(q % g.nz);
    const long long p = gidx(g, i, k);
    const double vol = kPi * g.dz * g.dr * g.dr * (2.0 * i + 1);
    double e2 = 0, h2 = 0;
    for (int c = 0; c < 3; ++c) {
      const double e = fl.f[c][p], hh = fl.f[3 + c][p];
      e2 += e * e;
      h2 += hh * hh;
    }
    ee += 0.5 * kEpsilon0 * e2 * vol;
    eh += 0.5 * kMagnConst * h2 * vol;
  }
  ee = block_sum(ee);
  __syncthreads();
  eh = block_sum(eh);
  if (threadIdx.x == 0) {
    atomicAdd(out, ee);
    atomicAdd(out + 1, eh);
  }
}

__global__ void kinetic_kernel(SpeciesF32Buffers b, size_t n, double mass, double* out) {
  double ek = 0;
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < n;
       j += (size_t)gridDim.x * blockDim.x) {
    if (b.cell[j] < 0) continue;
    const double vr = b.vr[j], vp = b.vphi[j], vz = b.vz[j];
    const double v2 = vr * vr + vp * vp + vz * vz;
    const double gm = 1.0 / sqrt(1.0 - v2 / kLightVel2);
    ek += (double)b.w[j] * mass * v2 * gm * gm / (gm + 1.0);
  }
  ek = block_sum(ek);
  if (threadIdx.x == 0) atomicAdd(out, ek);
}

}  // namespace

namespace {

// Per tile t, the particles [tile_start[t], tile_start[t+1]): each counted
// in its cell, and counted as misplaced when its cell is not in tile t (or
// not in the grid, or the slot is dead).
__global__ void tile_check_kernel(TileGrid tg, SpeciesF32Buffers b, int nr, int nz, unsigned* counts,
                                  unsigned long long* misplaced) {
  const int t = blockIdx.x;
  for (unsigned p = b.tile_start[t] + threadIdx.x; p < b.tile_start[t + 1]; p += blockDim.x) {
    const int c = b.cell[p];
    const int ci = cell_r_of(c), ck = cell_z_of(c);
    if (c < 0 || ci < 0 || ck < 0 || ci >= nr || ck >= nz) {
      atomicAdd(misplaced, 1ull);
      continue;
    }
    if ((ci / tg.tr) * tg.ntz + ck / tg.tz != t) atomicAdd(misplaced, 1ull);
    atomicAdd(counts + (size_t)ci * nz + ck, 1u);
  }
}

}  // namespace

int f32_tile_check(const TileGrid& tg, unsigned target_blocks, unsigned min_split, int nr, int nz,
                   SpeciesF32Buffers& b, size_t* n, unsigned* counts, unsigned long long* misplaced,
                   cudaStream_t s) {
  if (tile_sort(tg, target_blocks, min_split, b, n, s, true) != 0) return -1;
  cudaMemsetAsync(counts, 0, (size_t)nr * nz * sizeof(unsigned), s);
  cudaMemsetAsync(misplaced, 0, sizeof(unsigned long long), s);
  tile_check_kernel<<<(unsigned)tg.ntiles, kThreads, 0, s>>>(tg, b, nr, nz, counts, misplaced);
  b.launches += 1;
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

TileGrid f32_tile_grid(const GridGeom& g) {
  TileGrid t;
  t.tr = kTileR;  // grids smaller than a tile get one partly empty tile
  t.tz = kTileZ;
  t.ntr = (g.nr + t.tr - 1) / t.tr;
  t.ntz = (g.nz + t.tz - 1) / t.tz;
  t.ntiles = t.ntr * t.ntz;
  t.halo = kHalo;
  return t;
}

int f32_alloc_species(SpeciesF32Buffers& b, size_t cap, const TileGrid& tg) {
  if (cap == 0) cap = 1;
  b.cap = cap;
  // the slot arrays have kSlotPad spare elements: the step's bulk copies
  // round the end of a range up to 16 bytes
  int** ints[] = {&b.cell, &b.cell2};
  for (int** a : ints)
    if (cudaMalloc((void**)a, (cap + kSlotPad) * sizeof(int)) != cudaSuccess) return -1;
  float** arrs[] = {&b.off_r, &b.off_z, &b.vr, &b.vphi, &b.vz, &b.w,
                    &b.off_r2, &b.off_z2, &b.vr2, &b.vphi2, &b.vz2, &b.w2};
  for (float** a : arrs)
    if (cudaMalloc((void**)a, (cap + kSlotPad) * sizeof(float)) != cudaSuccess) return -1;
  if (cudaMalloc((void**)&b.id, cap * sizeof(unsigned)) != cudaSuccess) return -1;
  if (cudaMalloc((void**)&b.id2, cap * sizeof(unsigned)) != cudaSuccess) return -1;
  if (cudaMalloc((void**)&b.tile_start, (tg.ntiles + 1) * sizeof(unsigned)) != cudaSuccess) return -1;
  if (cudaMalloc((void**)&b.tile_cursor, (tg.ntiles + 1) * sizeof(unsigned)) != cudaSuccess) return -1;
  const size_t nt = (size_t)tg.ntiles;
  if (cudaMalloc((void**)&b.rank, cap * sizeof(unsigned)) != cudaSuccess) return -1;
  if (cudaMalloc((void**)&b.cell_count, nt * kTileCells * sizeof(unsigned)) != cudaSuccess) return -1;
  if (cudaMalloc((void**)&b.layer_mask, nt * kLayerCap * kTileWords * sizeof(unsigned)) != cudaSuccess) return -1;
  if (cudaMalloc((void**)&b.layer_prefix, nt * kLayerCap * kTileWords * sizeof(unsigned short)) != cudaSuccess)
    return -1;
  if (cudaMalloc((void**)&b.layer_start, nt * (kLayerCap + 1) * sizeof(unsigned)) != cudaSuccess) return -1;
  if (cudaMalloc((void**)&b.overflow, nt * sizeof(unsigned)) != cudaSuccess) return -1;
  if (cudaMalloc((void**)&b.sort_info, 4 * sizeof(unsigned)) != cudaSuccess) return -1;
  if (cudaMallocHost((void**)&b.host_info, 4 * sizeof(unsigned)) != cudaSuccess) return -1;
  b.host_info[0] = b.host_info[1] = b.host_info[3] = 0;
  b.host_info[2] = 1;
  if (cudaMalloc((void**)&b.drift, 2 * sizeof(unsigned)) != cudaSuccess) return -1;
  if (cudaMallocHost((void**)&b.drift_host, 2 * sizeof(unsigned)) != cudaSuccess) return -1;
  cudaMemset(b.drift, 0, 2 * sizeof(unsigned));
  b.drift_host[0] = b.drift_host[1] = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, b.scan_tmp_bytes, b.tile_cursor, b.tile_start, (int)(nt + 1));
  if (cudaMalloc(&b.scan_tmp, std::max<size_t>(b.scan_tmp_bytes, 16)) != cudaSuccess) return -1;
  return 0;
}

void f32_free_species(SpeciesF32Buffers& b) {
  void* arrs[] = {b.cell, b.off_r, b.off_z, b.vr, b.vphi, b.vz, b.w, b.id,
                  b.cell2, b.off_r2, b.off_z2, b.vr2, b.vphi2, b.vz2, b.w2, b.id2,
                  b.tile_start, b.tile_cursor, b.rank, b.cell_count, b.layer_mask, b.layer_prefix,
                  b.layer_start, b.overflow, b.sort_info, b.scan_tmp, b.drift};
  for (void* a : arrs) cudaFree(a);
  cudaFreeHost(b.host_info);
  cudaFreeHost(b.drift_host);
  b = SpeciesF32Buffers();
}

__global__ void add_planes_kernel(float* dst, const float* a, const float* b, size_t n) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    dst[q] = a[q] + b[q];
}

void f32_add_planes(float* dst, const float* a, const float* b, size_t n, cudaStream_t s) {
  add_planes_kernel<<<(unsigned)std::min<size_t>(blocks_for(n), 148 * 16), kThreads, 0, s>>>(dst, a, b, n);
}

void f32_launch_yee_e(const YeeArgs<float>& a, cudaStream_t s) {
  dim3 grid((a.g.nz + 4 + kThreads - 1) / kThreads, a.g.nr + 4);
  yee_e_kernel<float><<<grid, kThreads, 0, s>>>(a);
}

void f32_launch_yee_h(const YeeArgs<float>& a, int fixed, cudaStream_t s) {
  dim3 grid((a.g.nz + 4 + kThreads - 1) / kThreads, a.g.nr + 4);
  yee_h_kernel<float><<<grid, kThreads, 0, s>>>(a, fixed);
}

void f32_launch_inject(const GridGeom& g, SpeciesF32Buffers& b, size_t n0, unsigned count,
                       const BeamInject& bi, DevStatus* st, cudaStream_t s) {
  if (!count) return;
  inject_kernel<<<(count + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, b, n0, count, bi, st);
  b.next_id += count;
}

void f32_launch_import(const GridGeom& g, SpeciesF32Buffers& b, size_t n0, size_t n,
                       const double* src, DevStatus* st, cudaStream_t s) {
  if (n0 == 0) {  // a replacement: ids restart, no tile grouping yet
    b.next_id = 0;
    b.sorted_n = 0;
    b.steps_since_sort = 1 << 30;
  }
  if (n) import_kernel<<<blocks_for(n), kThreads, 0, s>>>(g, b, n0, n, src, st);
  b.next_id += (unsigned)n;
}

int f32_step_species(const F32Step& st, SpeciesF32Buffers& b, size_t* n, double charge,
                     double mass, int is_beam, cudaStream_t s, int xoff) {
  if (*n == 0) return 0;
  // a recent step's count (a hint), if that step came after the last sort
  const volatile unsigned* dh = b.drift_host;
  const size_t drifted = dh[1] == (unsigned)b.sorts ? dh[0] : 0;
  if (b.sorted_n == 0 || b.steps_since_sort >= st.sort_interval || (*n - b.sorted_n) * 4 > *n ||
      drifted * 100 > b.sorted_n) {
    // waits for nothing (the first sort of a species excepted)
    if (tile_sort(st.tiles, st.target_blocks, st.min_split, b, n, s, false) != 0) return -1;
  }
  cudaMemsetAsync(b.drift, 0, sizeof(unsigned), s);
  f32::StepArgs a = f32_step_args(st, charge, mass, is_beam);
  a.xoff = xoff;
  const TileGrid& tg = st.tiles;
  if (b.sorted_n) {
    const size_t smem = f32::kTileSmemBytes;
    const dim3 grid(tg.ntiles, b.splits);
    if (st.current == PCG_CURRENT_ZIGZAG && st.pusher == PCG_PUSHER_VAY && !is_beam && !st.fixed && !st.pushed) {
      auto kern = f32::step_pair_kernel<0, 1>;  // the plasma of the large Vay + ZigZag runs
      if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)f32::kPairSmemBytes) !=
          cudaSuccess)
        return -1;
      kern<<<grid, f32::kThreads, f32::kPairSmemBytes, s>>>(a, b, tg);
    }
    else if (st.current == PCG_CURRENT_ZIGZAG && st.pushed && !is_beam && !st.fixed) {
      auto kern = f32::step_pair_kernel<0, 2>;  // the move half of a collisional step
      if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)f32::kPairSmemBytes) !=
          cudaSuccess)
        return -1;
      kern<<<grid, f32::kThreads, f32::kPairSmemBytes, s>>>(a, b, tg);
    }
    else if (st.current == PCG_CURRENT_ZIGZAG)
      f32::step_tiled_kernel<1><<<grid, f32::kThreads, smem, s>>>(a, b, tg);
    else if (st.pushed)
      f32::step_tiled_kernel<0><<<grid, f32::kThreads, smem, s>>>(a, b, tg);
    else if (st.pusher == PCG_PUSHER_BORIS_RELATIVISTIC && !is_beam) {  // the plasma of the common runs
      auto kern = st.fixed ? f32::step_pair_kernel<1> : f32::step_pair_kernel<0>;
      if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)f32::kPairSmemBytes) !=
          cudaSuccess)
        return -1;
      kern<<<grid, f32::kThreads, f32::kPairSmemBytes, s>>>(a, b, tg);
    }
    else
      f32::step_tiled_kernel<0><<<grid, f32::kThreads, smem, s>>>(a, b, tg);
  }
  if (*n > b.sorted_n) {
    const unsigned nb = blocks_for(*n - b.sorted_n);
    if (st.current == PCG_CURRENT_ZIGZAG)
      f32::step_flat_kernel<1><<<nb, f32::kThreads, 0, s>>>(a, b, b.sorted_n, *n);
    else
      f32::step_flat_kernel<0><<<nb, f32::kThreads, 0, s>>>(a, b, b.sorted_n, *n);
  }
  b.launches += (b.sorted_n ? 1 : 0) + (*n > b.sorted_n ? 1 : 0);
  cudaMemcpyAsync(b.drift_host, b.drift, 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, s);
  b.steps_since_sort += 1;
  return 0;
}

void f32_push_species(const F32Step& st, SpeciesF32Buffers& b, size_t n, double charge, double mass,
                      int is_beam, cudaStream_t s) {
  if (n == 0) return;
  f32::StepArgs a = f32_step_args(st, charge, mass, is_beam);
  a.pushed = 0;
  size_t j0 = 0;
  if (b.sorted_n && st.pusher == PCG_PUSHER_VAY && !is_beam && !st.fixed) {
    // the tile-sorted slots through the pair kernel's push (field window, two per thread)
    auto kern = f32::step_pair_kernel<0, 3>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)f32::kPairSmemBytes) !=
        cudaSuccess)
      return;
    kern<<<dim3(st.tiles.ntiles, b.splits), f32::kThreads, f32::kPairSmemBytes, s>>>(a, b, st.tiles);
    b.launches += 1;
    j0 = std::min(n, b.sorted_n);
  }
  if (n > j0) {
    f32::push_flat_kernel<<<blocks_for(n - j0), f32::kThreads, 0, s>>>(a, b, j0, n);
    b.launches += 1;
  }
}

void f32_alive_flags(const SpeciesF32Buffers& b, unsigned char* flags, size_t n, cudaStream_t s) {
  if (n) alive_kernel<<<blocks_for(n), kThreads, 0, s>>>(b.cell, flags, n);
}

int f32_compact(SpeciesF32Buffers& b, const unsigned* idx, size_t kept, cudaStream_t s) {
  if (kept) {
    gather_kernel<int><<<blocks_for(kept), kThreads, 0, s>>>(b.cell, b.cell2, idx, kept);
    gather_kernel<float><<<blocks_for(kept), kThreads, 0, s>>>(b.off_r, b.off_r2, idx, kept);
    gather_kernel<float><<<blocks_for(kept), kThreads, 0, s>>>(b.off_z, b.off_z2, idx, kept);
    gather_kernel<float><<<blocks_for(kept), kThreads, 0, s>>>(b.vr, b.vr2, idx, kept);
    gather_kernel<float><<<blocks_for(kept), kThreads, 0, s>>>(b.vphi, b.vphi2, idx, kept);
    gather_kernel<float><<<blocks_for(kept), kThreads, 0, s>>>(b.vz, b.vz2, idx, kept);
    gather_kernel<float><<<blocks_for(kept), kThreads, 0, s>>>(b.w, b.w2, idx, kept);
    gather_kernel<unsigned><<<blocks_for(kept), kThreads, 0, s>>>(b.id, b.id2, idx, kept);
    swap_buffers(b);
  }
  b.sorted_n = 0;  // the grouping by tile no longer holds
  b.steps_since_sort = 1 << 30;
  return cudaStreamSynchronize(s) == cudaSuccess ? 0 : -1;
}

int f32_export(const GridGeom& g, SpeciesF32Buffers& b, size_t n, double* r, double* z,
               double* vr, double* vphi, double* vz, double* w, int32_t* cell_r, int32_t* cell_z,
               cudaStream_t s) {
  double* d = nullptr;
  int* c = nullptr;
  unsigned *keys = nullptr, *perm = nullptr;
  void* tmp = nullptr;
  size_t tmpb = 0;
  int rc = 0;
  if (cudaMalloc((void**)&d, 6 * n * sizeof(double)) != cudaSuccess ||
      cudaMalloc((void**)&c, 2 * n * sizeof(int)) != cudaSuccess ||
      cudaMalloc((void**)&keys, 2 * n * sizeof(unsigned)) != cudaSuccess ||
      cudaMalloc((void**)&perm, 2 * n * sizeof(unsigned)) != cudaSuccess) {
    rc = -1;
  } else {
    iota_kernel<<<blocks_for(n), kThreads, 0, s>>>(perm, n);
    cub::DeviceRadixSort::SortPairs(nullptr, tmpb, b.id, keys, perm, perm + n, (int)n, 0, 32, s);
    if (cudaMalloc(&tmp, tmpb) != cudaSuccess) {
      rc = -1;
    } else {
      cub::DeviceRadixSort::SortPairs(tmp, tmpb, b.id, keys, perm, perm + n, (int)n, 0, 32, s);
      export_kernel<<<blocks_for(n), kThreads, 0, s>>>(g, b, n, perm + n, d, c);
      double* dst[6] = {r, z, vr, vphi, vz, w};
      for (int a = 0; a < 6; ++a)
        if (dst[a]) cudaMemcpyAsync(dst[a], d + a * n, n * sizeof(double), cudaMemcpyDeviceToHost, s);
      if (cell_r) cudaMemcpyAsync(cell_r, c, n * sizeof(int), cudaMemcpyDeviceToHost, s);
      if (cell_z) cudaMemcpyAsync(cell_z, c + n, n * sizeof(int), cudaMemcpyDeviceToHost, s);
      if (cudaStreamSynchronize(s) != cudaSuccess) rc = -1;
    }
  }
  cudaFree(tmp);
  cudaFree(d);
  cudaFree(c);
  cudaFree(keys);
  cudaFree(perm);
  return rc;
}

int f32_energies(const GridGeom& g, float* const fld[12], double* ee, double* eh, cudaStream_t s) {
  double* d = nullptr;
  if (cudaMalloc((void**)&d, 2 * sizeof(double)) != cudaSuccess) return -1;
  cudaMemsetAsync(d, 0, 2 * sizeof(double), s);
  Fld12 fl;
  for (int c = 0; c < 12; ++c) fl.f[c] = fld[c];
  energy_kernel<<<296, kThreads, 0, s>>>(g, fl, d);
  double hbuf[2];
  cudaMemcpyAsync(hbuf, d, sizeof(hbuf), cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaStreamSynchronize(s);
  cudaFree(d);
  *ee = hbuf[0];
  *eh = hbuf[1];
  return e == cudaSuccess ? 0 : -1;
}

int f32_kinetic(const SpeciesF32Buffers& b, size_t n, double mass, double* out, cudaStream_t s) {
  *out = 0;
  if (n == 0) return 0;
  double* d = nullptr;
  if (cudaMalloc((void**)&d, sizeof(double)) != cudaSuccess) return -1;
  cudaMemsetAsync(d, 0, sizeof(double), s);
  kinetic_kernel<<<296, kThreads, 0, s>>>(b, n, mass, d);
  cudaMemcpyAsync(out, d, sizeof(double), cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaStreamSynchronize(s);
  cudaFree(d);
  return e == cudaSuccess ? 0 : -1;
}

}  // namespace pcg
