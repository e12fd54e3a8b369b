// pcg_tile_walk.cuh — walking the tile-sorted slots of a float species a
// thread per tile cell.
//
// The tile sort leaves tile t's slots in layers: layer q holds, in cell
// order, the q-th particle of each of the tile's cells whose count at the
// sort exceeds q, from layer_start[t][q]; layer_prefix[t][q][w] counts the
// layer's particles in the 32-cell words before word w; the particles
// beyond kLayerCap layers follow in one run.  A block of kTileCells threads
// takes a tile, thread lc its cell lc: warp w holds the cells of word w, so
// a ballot of "my count exceeds q" is the layer's mask word and the slot of
// thread lc in layer q is start + prefix + the set bits below its lane.  The
// block stages the tile's starts and prefixes in shared memory once; in the
// walk only the slots themselves are read from global memory, a layer's in
// one coalesced sweep per warp.
#pragma once

#include <cuda_runtime.h>

#include "pcg_f32.h"

namespace pcg {

struct TileWalk {
  unsigned ls[kLayerCap + 1];                    // layer starts, then the overflow run's
  unsigned short pre[kLayerCap][kTileWords];     // per layer and word: particles in the words before
  unsigned nq_max;                               // layers of the tile's fullest cell (<= kLayerCap)
};

// Stage tile t's layer tables (every thread of the block calls this; it
// ends with a barrier).  `count` is the tile cell's count of this thread.
__device__ __forceinline__ void tile_walk_begin(TileWalk& w, const unsigned* layer_start,
                                                const unsigned short* layer_prefix, int t, unsigned count) {
  __syncthreads();  // the previous tile's tables are no longer read
  if (threadIdx.x == 0) w.nq_max = 0;
  __syncthreads();
  unsigned mine = min(count, (unsigned)kLayerCap);
  for (int o = 16; o > 0; o >>= 1) mine = max(mine, __shfl_xor_sync(0xffffffffu, mine, o));
  if ((threadIdx.x & 31) == 0) atomicMax(&w.nq_max, mine);
  for (int q = threadIdx.x; q <= kLayerCap; q += blockDim.x) w.ls[q] = layer_start[(size_t)t * (kLayerCap + 1) + q];
  __syncthreads();
  const unsigned nq = w.nq_max;
  for (unsigned e = threadIdx.x; e < nq * kTileWords; e += blockDim.x)
    w.pre[e / kTileWords][e % kTileWords] = layer_prefix[(size_t)t * kLayerCap * kTileWords + e];
  __syncthreads();
}

// Tile-relative slot of this thread's particle in layer q, given the warp's
// ballot of (count > q); valid only where this thread's count exceeds q.
__device__ __forceinline__ unsigned tile_walk_slot(const TileWalk& w, unsigned q, unsigned ballot) {
  const unsigned lane = threadIdx.x & 31;
  return w.ls[q] + w.pre[q][threadIdx.x >> 5] + __popc(ballot & ((1u << lane) - 1u));
}

// Layers this thread's warp walks (the warp's fullest cell, <= kLayerCap).
__device__ __forceinline__ unsigned tile_walk_layers(unsigned count) {
  unsigned m = min(count, (unsigned)kLayerCap);
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  return m;
}

}  // namespace pcg
