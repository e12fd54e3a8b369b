// pcg_diag.h — double-precision node charges and flux divergences (the
// continuity and Gauss acceptance diagnostics of the deposit).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

#include "pcg_common.cuh"

namespace pcg {

struct SpeciesF32Buffers;

// Add charge * w of every live particle to the node charges q (C, halo layout).
int diag_node_charge_f64(const GridGeom& g, const double* r, const double* z, const double* w,
                         size_t n, double charge, double* q, cudaStream_t s);
int diag_node_charge_f32(const GridGeom& g, const SpeciesF32Buffers& b, size_t n, double charge,
                         double* q, cudaStream_t s);
// out(i, k) = F_r(i,k) A_r(i) - F_r(i-1,k) A_r(i-1) + (F_z(i,k) - F_z(i,k-1)) S(i).
int diag_divergence(const GridGeom& g, const void* fr, const void* fz, int is_double, double* out,
                    cudaStream_t s);

}  // namespace pcg
