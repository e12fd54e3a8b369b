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
  double sigma_v;  // sqrt(T e / m), m/s (sigma_v_par along z when per_cell)
  double weight;   // real particles per macroparticle (whole-cylinder mode)
  // per-cell mode: per_cell particles in every cell, uniform in its volume,
  // weights density * V_cell / per_cell, T_perp on r and phi
  unsigned per_cell = 0;
  double density = 0.0;
  double sigma_v_perp = 0.0;
};

void launch_seed_f64(const GridGeom& g, const PlasmaSeed& p, const SpeciesF64& sp, size_t n0,
                     size_t n, cudaStream_t s);
void launch_seed_f32(const GridGeom& g, const PlasmaSeed& p, const SpeciesF32Buffers& b,
                     size_t n0, size_t n, cudaStream_t s);

}  // namespace pcg
