// pcg_region.h — band-of-z particle selection (pcg_region.cu), shared by
// pcg_export_species_range and pcg_keep_species_range.  Exactly one of b32
// (float layout) and s64 (double layout) is non-null.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

#include "pcg_common.cuh"
#include "pcg_f32.h"
#include "pcg_kernels.h"

namespace pcg {

// Scratch bytes of region_select over n slots (at least those of any smaller n).
size_t region_select_bytes(size_t n);
// The indices of the live slots j < n with lo <= z < hi, in slot order, into
// out and their count into *count (device memory); one pass over the
// slots' positions.  Nonzero on a CUDA error.
int region_select(const GridGeom& g, const SpeciesF32Buffers* b32, const SpeciesF64* s64, size_t n, double lo,
                  double hi, void* temp, size_t temp_bytes, unsigned* out, unsigned* count, cudaStream_t s);
// out: r, z - zshift, v_r, v_phi, v_z, w of the slots idx[0..m), m doubles apart
void region_gather(const GridGeom& g, const SpeciesF32Buffers* b32, const SpeciesF64* s64, const unsigned* idx,
                   size_t m, double zshift, double* out, cudaStream_t s);
// marks the live slots outside [lo, hi) dead and counts them in st->dead_slots
void region_keep(const GridGeom& g, const SpeciesF32Buffers* b32, const SpeciesF64* s64, size_t n, double lo,
                 double hi, DevStatus* st, cudaStream_t s);

// rows x w values of a float plane (row length ld, columns from c0) from
// (set) or to device doubles, row-major
void region_columns_f32(float* plane, int ld, int c0, int w, int rows, double* buf, bool set, cudaStream_t s);

}  // namespace pcg
