// pcg_learned.h — the learned collision step: per-cell moments, the
// 13 features of the collision MLP, its forward pass on the tensor cores
// and a moment-matching velocity transform in FP64.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "pcg_collide.h"
#include "pcg_common.cuh"

namespace pcg {

constexpr int kMomWords = 16;  // per cell: for the electron then the ion list N, W, W u (3), W v^2 (3)
constexpr int kFeatures = 13, kTargets = 6;

// Normalisation and the training box of the features (all FP32):
// x_norm = (x - x_mean) / x_std, y = y_norm * y_std + y_mean; a cell whose
// features leave [x_lo, x_hi] widened by 25 % of the span takes the binary
// operator instead.
struct LearnedNorm {
  float x_mean[kFeatures], x_std[kFeatures], y_mean[kTargets], y_std[kTargets];
  float x_lo[kFeatures], x_hi[kFeatures];
};
constexpr int kNormFloats = 4 * kFeatures + 2 * kTargets;  // 64

struct LearnedPhys {
  double m_el, q_el, m_ion, q_ion, dt;
};

struct LearnedWork {
  size_t cells = 0;
  double* mom = nullptr;          // cells x kMomWords
  double* xform = nullptr;        // cells x 12: u_e (3), s_e (3), u_i (3), s_i (3)
  unsigned char* flag = nullptr;  // cells: 0 no collision, 1 learned, 2 binary fallback
  unsigned long long* count = nullptr;  // learned cells, fallback cells, tensor-core time-outs
  uint4* xin = nullptr;           // cells x 2: the network's normalised BF16 inputs
  float* yout = nullptr;          // cells x kTargets: its outputs
  float* params = nullptr;        // the model's FP32 parameters
  LearnedNorm norm{};
  bool model = false;
  unsigned launches = 0;  // kernels launched by the last learned_moments / learned_step
  // a second stream and two events of the caller (all or none): the moment
  // passes of odd-numbered species run there, concurrently with the others
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
};

// Per-cell moment sums of the species (electron list: every species not
// named ions; ion list: ions) into w.mom.
int learned_moments(const GridGeom& g, const CollSpecies* sp, int nsp, LearnedWork& w, cudaStream_t s);
// The raw features of every cell (x: cells x 13, NaN where a cell has no
// collisions) and the collision scale S = s_ee + s_ei + s_ii (cells).
int learned_features(const GridGeom& g, const CollSpecies* sp, int nsp, const LearnedPhys& ph,
                     LearnedWork& w, float* x, double* scale, cudaStream_t s);
// One learned collision step: moments, features, MLP, transform.  Cells
// outside the training box are flagged 2 in w.flag (the caller runs the
// binary operator on them); counts[0] learned cells, counts[1] fallback.
// Returns 0, -1 on a CUDA error, or kLearnedTimeout when a wait for the
// tensor cores timed out (no velocity changed; the kernel's TMEM may still
// be held, so the caller stops using the device work of this handle).
// Without apply the transforms stay in w.xform and w.flag for the caller
// to apply (the float step applies them in its move).
constexpr int kLearnedTimeout = 1;
int learned_step(const GridGeom& g, const CollSpecies* sp, int nsp, const LearnedPhys& ph, LearnedWork& w,
                 unsigned long long counts[2], cudaStream_t s, bool apply = true);
int learned_set_model(LearnedWork& w, const float* params_host, const float* norm_host, cudaStream_t s);
void learned_free(LearnedWork& w);

}  // namespace pcg
