// pcg_collide.h — binary Coulomb collisions (Perez et al. 2012, the
// reference's default scheme) on the GPU, in double precision for either
// particle layout.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "pcg_common.cuh"

namespace pcg {

constexpr int kCollMaxSpecies = 8;

// One species as the collision pass sees it.  Exactly one of the two
// layouts is set: double (r, z: cells from floor(r/dr), floor(z/dz); ids are
// slot indices) or float (packed cell, insertion ids).
struct CollSpecies {
  size_t n = 0;
  int is_ion = 0;  // ion lists take "ions"/"Ions", electron lists every other species
  const double* r = nullptr;
  const double* z = nullptr;
  double *vr64 = nullptr, *vphi64 = nullptr, *vz64 = nullptr;
  const double* w64 = nullptr;
  const int* cell = nullptr;
  const unsigned* id = nullptr;
  unsigned long long id_bound = 0;  // float layout: every id is below it
  float *vr32 = nullptr, *vphi32 = nullptr, *vz32 = nullptr;
  const float* w32 = nullptr;
  // float layout: slots [0, sorted) are grouped by tile, tile t holding
  // [tile_start[t], tile_start[t+1]) (the step's tile sort; sorted = 0 when
  // not), in layers: layer q holds, in cell order, the q-th particle of each
  // tile cell whose count at the sort (cell_count) exceeds q, from
  // layer_start[t][q] with the cell's place given by layer_mask and
  // layer_prefix; the particles beyond kLayerCap layers follow in a run
  const unsigned* tile_start = nullptr;
  const unsigned* cell_count = nullptr;
  const unsigned* layer_mask = nullptr;
  const unsigned short* layer_prefix = nullptr;
  const unsigned* layer_start = nullptr;
  size_t sorted = 0;
};

struct CollParams {
  double m_el, q_el, m_ion, q_ion;  // SI, of the species named electrons / ions
  double dt;
  int fixed;         // PCG_QUIRKS_FIXED
  int shuffle;       // Fisher-Yates of the cell lists with Philox draws
  uint64_t seed;
  uint32_t pass;     // counter of collision passes: the Philox stream of this one
  DevStatus* status; // superluminal pairs raise the error word (rel.cpp:33-34 is fatal)
  const unsigned char* only = nullptr;  // when set, collide only cells c with only[c] == only_value
  unsigned char only_value = 1;
  // when set, per cell the sum over the pass's collisions of each
  // collision's mean change over its scattering draw, given the velocities
  // it meets (the pass itself runs as usual): 12 doubles, sum w v (3) then
  // sum w v^2 (3) of the electron list, then of the ion list
  // (non-relativistic kinematics of the mean)
  double* expect = nullptr;
  int scheme = 0;  // 0: Perez 2012 (CollisionsP12), 1: Takizuka-Abe with correction (CollisionsTA77S)
  // cells of more than `crowded` particles take the warp-per-cell pair
  // kernel (pcg_collide_crowded.cu), the others a thread each
  unsigned crowded = 256;
};

// Scratch of a collision pass, grown on demand and kept by the handle.
struct CollWork {
  size_t cap = 0;  // entries per list
  unsigned long long *keys[2] = {}, *keys2[2] = {}, *vals[2] = {}, *vals2[2] = {};
  unsigned *count[2] = {}, *start[2] = {};  // per cell
  double4* stage[2] = {};                   // per list entry: v (3), w, in list order
  double* moments = nullptr;                // per cell: T_el, T_ion, n_el, n_ion
  double* totals = nullptr;                 // TA77S, per cell and list: sum w, sum w m v (3), sum w m v^2/2
  size_t totals_cells = 0;
  int* row_stop = nullptr;                  // per row: first cell that stops the row
  unsigned long long* calls = nullptr;      // device counter of pair calls
  unsigned* valid = nullptr;                // device: entries appended to each list
  unsigned* crowded = nullptr;              // device: [0] crowded cells listed in [1..]
  unsigned* active = nullptr;               // device: [0] other chosen cells (CollParams::only) in [1..]
  void* tmp = nullptr;
  size_t tmp_bytes = 0;
  size_t cells = 0;
  unsigned launches = 0;                    // this library's kernels launched by the last pass
};

// One collision pass over all cells; returns 0 or -1 (allocation/launch).
// *pair_calls receives the number of collide_single calls.
int collide_p12(const GridGeom& g, const CollSpecies* sp, int nsp, const CollParams& p,
                CollWork& w, unsigned long long* pair_calls, cudaStream_t s);
void collide_free(CollWork& w);
// The pairs of the cells holding more than p.crowded particles, one warp per
// cell (pcg_collide_crowded.cu); the per-cell kernel of collide_p12 skips them.
// list[0] is the number of such cells, list[1..] the cells (device memory).
void collide_crowded(const GridGeom& g, double4* const stage[2], const CollParams& p, const unsigned* st_e,
                     const unsigned* n_e, const unsigned long long* le, const unsigned* st_i, const unsigned* n_i,
                     const unsigned long long* li, const double* mom, const int* row_stop, unsigned long long* calls,
                     const unsigned* list, cudaStream_t s);

}  // namespace pcg
