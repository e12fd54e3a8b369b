// pcg_ensemble.cu — many independent runs advanced together (the batched
// configuration: runs of uneven grids and beams), over the public C ABI.
//
// Each run is a pcg_handle with its own stream.  A step of the ensemble
// spreads the runs over a few host threads; each thread issues one step of
// each of its runs in turn, so the GPU overlaps all runs' kernels, and the
// tile sort of one run (the only part of a step that waits for its stream)
// holds up only its own thread.  The device time of a batch runs from an
// event all run streams wait on to an event that waits on all of them.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include "pcg.h"
#include "pcg_device.h"

struct pcg_ensemble {
  std::vector<pcg_handle*> runs;
  std::vector<cudaStream_t> streams;
  int threads = 1;
  int device = 0;
  cudaStream_t join = nullptr;  // the batch's timing stream
  cudaEvent_t start = nullptr, stop = nullptr;
  std::vector<cudaEvent_t> done;
};

namespace {

// The autotuner's candidates: target blocks and minimum particles per block
// of each run, from the run's share f of the ensemble's particles.  A run
// alone fills the GPU with one to two thousand blocks; in an ensemble that
// many per run oversubscribe it, so some candidates scale the target by f.
struct Tiling {
  double blocks;  // target blocks (absolute, or times f when shared)
  bool shared;
  int min_split;
};
const Tiling kCandidates[6] = {{1184, false, 1024}, {148, false, 2048}, {1184, true, 1024},
                               {4736, true, 512},   {592, false, 512},  {2368, false, 512}};
constexpr int kNumCandidates = 6;

int apply(pcg_ensemble* e, const Tiling& t, const std::vector<double>& share) {
  for (size_t i = 0; i < e->runs.size(); ++i) {
    const double b = t.shared ? t.blocks * share[i] : t.blocks;
    const int rc = pcg_set_tiling(e->runs[i], 0, std::max(1, (int)(b + 0.5)), t.min_split);
    if (rc != PCG_OK) return rc;
  }
  return PCG_OK;
}

}  // namespace

extern "C" {

int pcg_ensemble_create(pcg_handle* const* runs, int n, int threads, pcg_ensemble** out) {
  if (!runs || n <= 0 || !out) return PCG_ERR_ARG;
  *out = nullptr;
  int dev = -1;
  for (int i = 0; i < n; ++i) {  // the runs share one GPU
    int d = -1;
    if (!runs[i] || pcg_get_device(runs[i], &d) != PCG_OK || (i > 0 && d != dev)) return PCG_ERR_ARG;
    dev = d;
  }
  pcg::DeviceScope device_scope(dev);
  pcg_ensemble* e = new pcg_ensemble();
  e->device = dev;
  e->threads = std::max(1, std::min(threads > 0 ? threads : 8, n));
  for (int i = 0; i < n; ++i) {
    void* st = nullptr;
    if (!runs[i] || pcg_get_stream(runs[i], &st) != PCG_OK) {
      delete e;
      return PCG_ERR_ARG;
    }
    e->runs.push_back(runs[i]);
    e->streams.push_back((cudaStream_t)st);
  }
  bool ok = cudaStreamCreateWithFlags(&e->join, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreate(&e->start) == cudaSuccess && cudaEventCreate(&e->stop) == cudaSuccess;
  e->done.assign(n, nullptr);
  for (int i = 0; ok && i < n; ++i) ok = cudaEventCreateWithFlags(&e->done[i], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    pcg_ensemble_destroy(e);
    return PCG_ERR_CUDA;
  }
  *out = e;
  return PCG_OK;
}

int pcg_ensemble_step(pcg_ensemble* e, int nsteps, float* device_ms) {
  pcg::DeviceScope device_scope(e ? e->device : -1);
  if (!e || nsteps < 0) return PCG_ERR_ARG;
  const int n = (int)e->runs.size();
  if (cudaEventRecord(e->start, e->join) != cudaSuccess) return PCG_ERR_CUDA;
  for (int i = 0; i < n; ++i)
    if (cudaStreamWaitEvent(e->streams[i], e->start, 0) != cudaSuccess) return PCG_ERR_CUDA;
  std::atomic<int> status(PCG_OK);
  auto work = [&](int t) {
    cudaSetDevice(e->device);
    for (int step = 0; step < nsteps && status.load() == PCG_OK; ++step)
      for (int i = t; i < n; i += e->threads) {
        const int rc = pcg_step(e->runs[i], 1);
        if (rc != PCG_OK) {
          int expect = PCG_OK;
          status.compare_exchange_strong(expect, rc);
          return;
        }
      }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < e->threads; ++t) pool.emplace_back(work, t);
  work(0);
  for (std::thread& th : pool) th.join();
  for (int i = 0; i < n; ++i) {
    if (cudaEventRecord(e->done[i], e->streams[i]) != cudaSuccess ||
        cudaStreamWaitEvent(e->join, e->done[i], 0) != cudaSuccess)
      return PCG_ERR_CUDA;
  }
  if (cudaEventRecord(e->stop, e->join) != cudaSuccess || cudaEventSynchronize(e->stop) != cudaSuccess)
    return PCG_ERR_CUDA;
  if (device_ms && cudaEventElapsedTime(device_ms, e->start, e->stop) != cudaSuccess) return PCG_ERR_CUDA;
  if (status.load() != PCG_OK) return status.load();
  for (pcg_handle* h : e->runs) {  // device-side errors (NaN, capacity, ...) of any run
    const int rc = pcg_synchronize(h);
    if (rc != PCG_OK) return rc;
  }
  return PCG_OK;
}

int pcg_ensemble_autotune(pcg_ensemble* e, int trial_steps, int* choice) {
  pcg::DeviceScope device_scope(e ? e->device : -1);
  if (!e || trial_steps <= 0) return PCG_ERR_ARG;
  std::vector<double> share;
  double total = 0;
  for (pcg_handle* h : e->runs) {
    pcg_diagnostics d;
    const int rc = pcg_diag(h, &d);
    if (rc != PCG_OK) return rc;
    share.push_back((double)d.particles);
    total += (double)d.particles;
  }
  for (double& f : share) f = total > 0 ? f / total : 1.0 / (double)share.size();
  float best = 0;
  int best_c = 0;
  for (int c = 0; c < kNumCandidates; ++c) {
    int rc = apply(e, kCandidates[c], share);
    if (rc == PCG_OK) rc = pcg_ensemble_step(e, 1, nullptr);  // the sorts under this tiling
    float ms = 0;
    if (rc == PCG_OK) rc = pcg_ensemble_step(e, trial_steps, &ms);
    if (rc != PCG_OK) return rc;
    if (c == 0 || ms < best) { best = ms; best_c = c; }
  }
  if (choice) *choice = best_c;
  return apply(e, kCandidates[best_c], share);
}

int pcg_ensemble_destroy(pcg_ensemble* e) {
  pcg::DeviceScope device_scope(e ? e->device : -1);
  if (!e) return PCG_ERR_ARG;
  for (cudaEvent_t ev : e->done)
    if (ev) cudaEventDestroy(ev);
  if (e->start) cudaEventDestroy(e->start);
  if (e->stop) cudaEventDestroy(e->stop);
  if (e->join) cudaStreamDestroy(e->join);
  delete e;
  return PCG_OK;
}

}  // extern "C"
