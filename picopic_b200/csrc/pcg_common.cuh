// pcg_common.cuh — constants, grid parameters and device error reporting
// shared by every kernel of the PIC step.
#pragma once

#include <cstdint>

namespace pcg {

// The reference's rounded SI constants (constant.hpp:35-57); parity with the
// reference needs these exact values, not CODATA ones.
constexpr double kPi = 3.1415926535897932;
constexpr double kEpsilon0 = 8.85E-12;
constexpr double kElMass = 9.1E-31;
constexpr double kElCharge = 1.6E-19;
constexpr double kLightVel = 3.0E8;
constexpr double kLightVel2 = kLightVel * kLightVel;
constexpr double kMagnConst = 1.26E-6;
constexpr double kMnzl = 1e-15;         // MNZL, constant.hpp:57
constexpr double kRelLimit = 5e7;       // REL_LIMIT, configure.ac:224
constexpr double kRelLimit2 = kRelLimit * kRelLimit;

// Device error word bits; the host maps them to PCG_ERR_* status codes.
enum ErrBits : unsigned {
  kErrNanPosition = 1u << 0,   // pusherBoris.cpp:51-57
  kErrSuperluminal = 1u << 1,  // rel.cpp:33-34
  kErrNanField = 1u << 2,      // maxwellSolverYee.cpp:253-255
  kErrReflectLoop = 1u << 3,   // reflection did not converge
  kErrCapacity = 1u << 4,      // species buffer full
  kErrOutOfGrid = 1u << 5,     // a particle outside the grid and its halo
  kErrUnsupported = 1u << 6,   // a switch combination this path does not implement
  kErrTimeout = 1u << 7,       // a bounded wait in a kernel ran out (its results are invalid)
};

// Device-side counters and the error word, one block per handle.
struct DevStatus {
  unsigned error;
  unsigned pad;
  unsigned long long move_errors;  // currentVB.cpp:199-204 (LOG_S(ERROR), skipped)
  unsigned long long removed;      // runaway collector
  unsigned long long dead_slots;   // slots marked dead since the last compaction
};

// Grid geometry for one domain at the origin with all four walls on
// (cfg.cpp:398-429), in the units of the reference.
struct GridGeom {
  int nr, nz;   // cells
  int ld;       // row length with halo: nz + 4
  double R, L;  // domain size, m
  double dr, dz, dt;
  int pml_r, pml_z0, pml_zl;  // PML present on r=R, z=0, z=L
};

// Grid<T> node (i, k) with the 2-cell halo, grid.hpp:165-168.
__host__ __device__ __forceinline__ long long gidx(const GridGeom& g, int i, int k) {
  return (long long)(i + 2) * g.ld + (k + 2);
}

__device__ __forceinline__ void raise_error(DevStatus* st, unsigned bits) {
  atomicOr(&st->error, bits);
}

// Reference processing order of a particle: species slot, then index.  Used
// to reproduce the order-dependent J_r overwrite of strict axial motion
// (currentVB.cpp:545-546).  Stored +1 so that 0 means "no reset".
__host__ __device__ __forceinline__ unsigned long long particle_order(int slot,
                                                                     unsigned long long idx) {
  return ((unsigned long long)slot << 40) | idx;
}

}  // namespace pcg
