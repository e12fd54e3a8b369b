// pcg_f32.h — the single-precision production particle path: positions as a
// packed int16 (cell_r, cell_z) pair plus float in-cell offsets, velocities
// and weights in float, float field grids.  Particles are kept grouped by
// tile (a rectangle of cells) so that one thread block deposits a tile's
// current in shared memory.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "pcg_common.cuh"
#include "pcg_kernels.h"

namespace pcg {

template <typename Real>
struct YeeArgs;

// Tiles of tr x tz cells; a block's shared window adds `halo` cells per side.
// every tile is kTileR x kTileZ cells: 256 cells, one per thread of a step
// block in a full layer, and 32 along z so that a warp's 32 cells share a row
constexpr int kTileR = 8, kTileZ = 32, kHalo = 3;
constexpr int kTileCells = kTileR * kTileZ;
constexpr int kTileWords = kTileCells / 32;  // 32-cell words of a tile's layer mask
constexpr int kLayerCap = 128;              // layers kept in order; deeper ranks go to an overflow run
constexpr int kSlotPad = 4;                 // spare elements after each slot array (16 bytes)
struct TileGrid {
  int tr, tz, ntr, ntz, ntiles, halo;
};

// cell = (uint16)cell_r | cell_z << 16; a dead slot has cell < 0.
struct SpeciesF32Buffers {
  int* cell = nullptr;
  float *off_r = nullptr, *off_z = nullptr;  // in-cell offsets in [0, 1), units of dr and dz
  float *vr = nullptr, *vphi = nullptr, *vz = nullptr;  // m/s
  float* w = nullptr;                                    // real particles per macroparticle
  unsigned* id = nullptr;  // insertion order, to export in the reference's particle order
  // second buffer set, the target of the tile sort
  int* cell2 = nullptr;
  float *off_r2 = nullptr, *off_z2 = nullptr, *vr2 = nullptr, *vphi2 = nullptr, *vz2 = nullptr,
        *w2 = nullptr;
  unsigned* id2 = nullptr;
  unsigned* tile_start = nullptr;   // ntiles + 1: particles of tile t are [start[t], start[t+1])
  unsigned* tile_cursor = nullptr;  // ntiles + 1, per-tile counts before the scan
  // layered order inside a tile (see tile_sort): per particle its rank in its
  // cell, per tile cell counts and, per layer q, which cells hold more than q
  unsigned* rank = nullptr;            // cap
  unsigned* cell_count = nullptr;      // ntiles * kTileCells
  unsigned* layer_mask = nullptr;      // ntiles * kLayerCap * kTileWords
  unsigned short* layer_prefix = nullptr;  // same shape: set bits in the words before
  unsigned* layer_start = nullptr;     // ntiles * (kLayerCap + 1); entry kLayerCap: overflow run
  unsigned* overflow = nullptr;        // ntiles, cursors of the overflow runs
  // device: largest tile, occupied tiles, blocks per tile, live slots of
  // the last sort (the step kernels read the blocks per tile here)
  unsigned* sort_info = nullptr;
  unsigned* host_info = nullptr;       // pinned: the same, copied after each sort (a hint)
  void* scan_tmp = nullptr;            // the tile-count scan's workspace
  size_t scan_tmp_bytes = 0;
  int splits = 1;                      // blocks per tile launched (the largest tile's share)
  int sorts = 0;                       // sorts issued
  // particles of a step that left their tile's shared windows (and took the
  // slow global path): counted on the device in drift[0], copied with the
  // device's count of sorts (drift[1]) to pinned memory after every step
  // and read by the host, possibly steps late, to decide a sort
  unsigned* drift = nullptr;
  unsigned* drift_host = nullptr;
  uint64_t launches = 0;  // kernels launched for this species (sorts and steps)
  size_t cap = 0;
  size_t sorted_n = 0;       // [0, sorted_n) are grouped by tile; later slots were appended
  int steps_since_sort = 1 << 30;
  unsigned next_id = 0;
};

struct F32Step {
  GridGeom g;
  float* fld[12];  // planes of one allocation: fld[c] = fld[0] + c * plane
  int plane;
  const float4* recip;  // radial reciprocal table, 2 float4 per node row from i = -2
  int pusher, current, fixed;
  DevStatus* status;
  TileGrid tiles;
  int sort_interval;  // most steps between tile sorts
  // a sort splits each occupied tile over enough blocks that about
  // target_blocks run, each with at least min_split particles
  unsigned target_blocks = 148 * 16, min_split = 1024;
  // the velocities were pushed by f32_push_species already (collisions act
  // between the push and the move): the step moves and deposits only
  int pushed = 0;
  // with pushed, the learned collision transforms to apply before the move
  // (12 doubles and a flag per cell; see f32_step_species)
  const double* xform = nullptr;
  const unsigned char* xflag = nullptr;
};

__host__ __device__ __forceinline__ int pack_cell(int ci, int ck) {
  return (int)(((unsigned)ci & 0xffffu) | ((unsigned)ck << 16));
}
__host__ __device__ __forceinline__ int cell_r_of(int cell) { return (int)(short)(cell & 0xffff); }
__host__ __device__ __forceinline__ int cell_z_of(int cell) { return cell >> 16; }
constexpr int kDeadCell = (int)0x80000000u;

TileGrid f32_tile_grid(const GridGeom& g);
// A tile sort of the species now, then per cell (nr x nz, device) the
// particles the sorted tiles hold and, in *misplaced (device), those whose
// cell is outside their tile.
int f32_tile_check(const TileGrid& tg, unsigned target_blocks, unsigned min_split, int nr, int nz,
                   SpeciesF32Buffers& b, size_t* n, unsigned* counts, unsigned long long* misplaced,
                   cudaStream_t s);
int f32_alloc_species(SpeciesF32Buffers& b, size_t cap, const TileGrid& tg);
void f32_free_species(SpeciesF32Buffers& b);
void f32_launch_yee_e(const YeeArgs<float>& a, cudaStream_t s);
// dst[q] = a[q] + b[q], q < n (the external fields added to the step's gather planes)
void f32_add_planes(float* dst, const float* a, const float* b, size_t n, cudaStream_t s);
void f32_launch_yee_h(const YeeArgs<float>& a, int fixed, cudaStream_t s);
// Positions outside the grid (or not finite: kErrNanPosition) become dead
// slots counted in st->removed and st->dead_slots.
void f32_launch_inject(const GridGeom& g, SpeciesF32Buffers& b, size_t n0, unsigned count,
                       const BeamInject& bi, DevStatus* st, cudaStream_t s);
void f32_launch_import(const GridGeom& g, SpeciesF32Buffers& b, size_t n0, size_t n,
                       const double* src, DevStatus* st, cudaStream_t s);
// One step of a species; returns the new slot count (a tile sort drops dead
// particles).  Sorts when the species has no tile grouping, when appended
// particles exceed 1/4 of the slots, when more than 1 % of the particles
// left their tile's windows in a recent step, or after `sort_interval` steps.
// xoff: the species' half of the learned transforms (0 electron list, 6 ions).
int f32_step_species(const F32Step& st, SpeciesF32Buffers& b, size_t* n, double charge,
                     double mass, int is_beam, cudaStream_t s, int xoff = 0);
// The push alone of a species' particles (fields from the global grid),
// for a step with collisions between the push and the move.
void f32_push_species(const F32Step& st, SpeciesF32Buffers& b, size_t n, double charge, double mass,
                      int is_beam, cudaStream_t s);
void f32_alive_flags(const SpeciesF32Buffers& b, unsigned char* flags, size_t n, cudaStream_t s);
int f32_compact(SpeciesF32Buffers& b, const unsigned* idx, size_t kept, cudaStream_t s);
int f32_export(const GridGeom& g, SpeciesF32Buffers& b, size_t n, double* r, double* z,
               double* vr, double* vphi, double* vz, double* w, int32_t* cell_r, int32_t* cell_z,
               cudaStream_t s);
int f32_energies(const GridGeom& g, float* const fld[12], double* ee, double* eh, cudaStream_t s);
int f32_kinetic(const SpeciesF32Buffers& b, size_t n, double mass, double* out, cudaStream_t s);

}  // namespace pcg
