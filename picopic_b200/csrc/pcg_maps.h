// pcg_maps.h — the species diagnostic maps of SpecieP (calc_density,
// calc_temperature, calc_energy, calc_momentum; specieP.cpp:665-839) on the
// GPU, in double precision for either particle layout.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

#include "pcg_common.cuh"

namespace pcg {

// One species as the maps see it: the double layout (r, z, v, w) or the
// float one (packed cell, offsets, v, w); dead slots have r < 0 or cell < 0.
struct MapSpecies {
  size_t n = 0;
  double mass = 0;  // SI
  const double *r = nullptr, *z = nullptr, *vr = nullptr, *vphi = nullptr, *vz = nullptr, *w = nullptr;
  const int* cell = nullptr;
  const float *off_r = nullptr, *off_z = nullptr, *vr32 = nullptr, *vphi32 = nullptr, *vz32 = nullptr,
              *w32 = nullptr;
};

// Map `which` (0 density, 1 temperature in eV, 2 energy in eV, 3 momentum:
// three grids r, phi, z) into out, (nr+4) x (nz+4) device doubles per grid.
// scratch: 4 grids.  abs_map: the species' absolute-momentum map, kept
// between calls (the reference's temperature reads the one its last energy
// map left); fixed: gamma at every speed and a fresh absolute-momentum map
// for the temperature.  Returns 0 or -1.
int species_map(const GridGeom& g, const MapSpecies& sp, int which, int fixed, double* abs_map,
                double* scratch, double* out, cudaStream_t s);

}  // namespace pcg
