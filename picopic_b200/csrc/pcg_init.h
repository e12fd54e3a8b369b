// pcg_init.h — device initialisers of synthetic plasmas.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "pcg_kernels.h"

namespace pcg {

struct SpeciesF32Buffers;

struct PlasmaSeed {
  uint64_t seed;
  uint32_t stream;
  double sigma_v;  // sqrt(T e / m), m/s
  double weight;   // real particles per macroparticle
};

void launch_seed_f64(const GridGeom& g, const PlasmaSeed& p, const SpeciesF64& sp, size_t n0,
                     size_t n, cudaStream_t s);
void launch_seed_f32(const GridGeom& g, const PlasmaSeed& p, const SpeciesF32Buffers& b,
                     size_t n0, size_t n, cudaStream_t s);

}  // namespace pcg
