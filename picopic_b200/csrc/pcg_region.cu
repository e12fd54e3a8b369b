// pcg_region.cu — particles of a species within a band of z: selected,
// copied out, or all others removed.  The exchange of a run split into
// z-slabs (picopic_b200/slabs.py) moves only the particles near a slab's
// ends this way, in place of the reference's particle hand-over between
// domains (SMB::particles_runaway_collector, SMB.cpp:194-564).
#include <cuda_runtime.h>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "pcg_f32.h"
#include "pcg_kernels.h"
#include "pcg_region.h"

namespace pcg {
namespace {

constexpr int kThreads = 256;
inline unsigned blocks_for(size_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

// z of slot j (float layout: cell and offset, as an export computes it)
__device__ __forceinline__ bool slot_z(const GridGeom& g, const SpeciesF32Buffers* b, const SpeciesF64* s,
                                       size_t j, double* z) {
  if (b) {
    const int c = b->cell[j];
    if (c < 0) return false;
    *z = ((double)cell_z_of(c) + (double)b->off_z[j]) * g.dz;
    return true;
  }
  if (!(s->r[j] >= 0.0)) return false;
  *z = s->z[j];
  return true;
}

// lo <= z < hi for a live slot j, z as slot_z computes it (the selection
// predicate of a band; keep_kernel's complement)
struct BandTest {
  GridGeom g;
  const int* cell;
  const float* off_z;
  const double* r;
  const double* z;
  int f32;
  double lo, hi;
  __device__ __forceinline__ bool operator()(const unsigned& j) const {
    double zz;
    if (f32) {
      const int c = cell[j];
      if (c < 0) return false;
      zz = ((double)cell_z_of(c) + (double)off_z[j]) * g.dz;
    } else {
      if (!(r[j] >= 0.0)) return false;
      zz = z[j];
    }
    return zz >= lo && zz < hi;
  }
};

BandTest band_test(const GridGeom& g, const SpeciesF32Buffers* b32, const SpeciesF64* s64, double lo, double hi) {
  BandTest t{};
  t.g = g;
  t.f32 = b32 ? 1 : 0;
  if (b32) {
    t.cell = b32->cell;
    t.off_z = b32->off_z;
  } else {
    t.r = s64->r;
    t.z = s64->z;
  }
  t.lo = lo;
  t.hi = hi;
  return t;
}

// out: 6 x m doubles (r, z - zshift, v_r, v_phi, v_z, w) of the slots idx[0..m)
__global__ void gather_kernel(GridGeom g, SpeciesF32Buffers b32, SpeciesF64 s64, int f32, const unsigned* idx,
                              size_t m, double zshift, double* out) {
  const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (q >= m) return;
  const size_t j = idx[q];
  if (f32) {
    const int c = b32.cell[j];
    out[q] = ((double)cell_r_of(c) + (double)b32.off_r[j]) * g.dr;
    out[m + q] = ((double)cell_z_of(c) + (double)b32.off_z[j]) * g.dz - zshift;
    out[2 * m + q] = b32.vr[j];
    out[3 * m + q] = b32.vphi[j];
    out[4 * m + q] = b32.vz[j];
    out[5 * m + q] = b32.w[j];
  } else {
    out[q] = s64.r[j];
    out[m + q] = s64.z[j] - zshift;
    out[2 * m + q] = s64.vr[j];
    out[3 * m + q] = s64.vphi[j];
    out[4 * m + q] = s64.vz[j];
    out[5 * m + q] = s64.w[j];
  }
}

// Live slots outside [lo, hi) become dead slots (counted as dead, not as
// removed by the runaway collector).
__global__ void keep_kernel(GridGeom g, SpeciesF32Buffers b32, SpeciesF64 s64, int f32, size_t n, double lo,
                            double hi, DevStatus* st) {
  const size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  double z;
  const bool drop = j < n && slot_z(g, f32 ? &b32 : nullptr, &s64, j, &z) && !(z >= lo && z < hi);
  if (drop) {
    if (f32) b32.cell[j] = kDeadCell;
    else s64.r[j] = -1.0;
  }
  const unsigned m = __ballot_sync(0xffffffffu, drop);
  if ((threadIdx.x & 31) == 0 && m) atomicAdd(&st->dead_slots, (unsigned long long)__popc(m));
}

// rows x w block of a float plane (row length ld, from column c0) to or
// from doubles in buf (row-major, w per row)
__global__ void columns_f32_kernel(float* plane, int ld, int c0, int w, int rows, double* buf, int set) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= w * rows) return;
  const int row = q / w, col = q - row * w;
  float* f = plane + (size_t)row * ld + c0 + col;
  if (set) *f = (float)buf[q];
  else buf[q] = *f;
}

}  // namespace

size_t region_select_bytes(size_t n) {
  size_t bytes = 0;
  BandTest t{};
  cub::DeviceSelect::If(nullptr, bytes, thrust::counting_iterator<unsigned>(0u), (unsigned*)nullptr,
                        (unsigned*)nullptr, (int)n, t, (cudaStream_t)0);
  return bytes;
}

int region_select(const GridGeom& g, const SpeciesF32Buffers* b32, const SpeciesF64* s64, size_t n, double lo,
                  double hi, void* temp, size_t temp_bytes, unsigned* out, unsigned* count, cudaStream_t s) {
  if (n == 0) return cudaMemsetAsync(count, 0, sizeof(unsigned), s) == cudaSuccess ? 0 : -1;
  return cub::DeviceSelect::If(temp, temp_bytes, thrust::counting_iterator<unsigned>(0u), out, count, (int)n,
                               band_test(g, b32, s64, lo, hi), s) == cudaSuccess
             ? 0
             : -1;
}

void region_columns_f32(float* plane, int ld, int c0, int w, int rows, double* buf, bool set, cudaStream_t s) {
  const int n = w * rows;
  if (n > 0) columns_f32_kernel<<<blocks_for((size_t)n), kThreads, 0, s>>>(plane, ld, c0, w, rows, buf, set ? 1 : 0);
}

void region_gather(const GridGeom& g, const SpeciesF32Buffers* b32, const SpeciesF64* s64, const unsigned* idx,
                   size_t m, double zshift, double* out, cudaStream_t s) {
  if (!m) return;
  gather_kernel<<<blocks_for(m), kThreads, 0, s>>>(g, b32 ? *b32 : SpeciesF32Buffers{}, s64 ? *s64 : SpeciesF64{},
                                                    b32 ? 1 : 0, idx, m, zshift, out);
}

void region_keep(const GridGeom& g, const SpeciesF32Buffers* b32, const SpeciesF64* s64, size_t n, double lo,
                 double hi, DevStatus* st, cudaStream_t s) {
  if (!n) return;
  keep_kernel<<<blocks_for(n), kThreads, 0, s>>>(g, b32 ? *b32 : SpeciesF32Buffers{}, s64 ? *s64 : SpeciesF64{},
                                                  b32 ? 1 : 0, n, lo, hi, st);
}

}  // namespace pcg
