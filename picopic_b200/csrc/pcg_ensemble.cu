// pcg_ensemble.cu — many independent runs advanced together (the batched
// configuration: runs of uneven grids and beams), over the public C ABI.
//
// Each run is a pcg_handle with its own stream.  A step of the ensemble
// spreads the runs over a few host threads; each thread issues one step of
// each of its runs in turn, so the GPU overlaps all runs' kernels.  The
// device time of a batch runs from an event all run streams wait on to an
// event that waits on all of them.
//
// In graph mode (pcg_ensemble_set_graph) a batch of steps of all runs is
// captured from one host thread into one CUDA graph (the runs' streams
// forked from and joined to the ensemble's stream, so the graph holds every
// run's kernels for every step of the batch as parallel branches) and
// issued as one graph launch.  The host decisions of a step (beam particle
// counts, when to re-sort) are taken at capture, as a direct step takes
// them; the graph of the previous batch is updated in place when the new
// one has the same shape, and instantiated anew otherwise.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
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
  // graph mode
  bool graph = false;
  bool stepped = false;   // a batch has run: every species with particles has had its first sort
  bool broken = false;    // a capture failed after some runs had advanced their host state
  cudaGraphExec_t exec = nullptr;
  size_t graph_nodes = 0;
  float capture_ms = 0;   // host time of the last capture and instantiation or update
  cudaEvent_t fork = nullptr;
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
            cudaEventCreate(&e->start) == cudaSuccess && cudaEventCreate(&e->stop) == cudaSuccess &&
            cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) == cudaSuccess;
  e->done.assign(n, nullptr);
  for (int i = 0; ok && i < n; ++i) ok = cudaEventCreateWithFlags(&e->done[i], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    pcg_ensemble_destroy(e);
    return PCG_ERR_CUDA;
  }
  *out = e;
  return PCG_OK;
}

}  // extern "C"

namespace {

// nsteps steps of every run captured into one graph and launched once on
// the ensemble's stream.
int graph_step(pcg_ensemble* e, int nsteps, float* device_ms) {
  const int n = (int)e->runs.size();
  const auto t0 = std::chrono::steady_clock::now();
  if (cudaStreamBeginCapture(e->join, cudaStreamCaptureModeRelaxed) != cudaSuccess) return PCG_ERR_CUDA;
  int rc = PCG_OK;
  if (cudaEventRecord(e->fork, e->join) != cudaSuccess) rc = PCG_ERR_CUDA;
  for (int i = 0; rc == PCG_OK && i < n; ++i)
    if (cudaStreamWaitEvent(e->streams[i], e->fork, 0) != cudaSuccess) rc = PCG_ERR_CUDA;
  for (int step = 0; rc == PCG_OK && step < nsteps; ++step)
    for (int i = 0; rc == PCG_OK && i < n; ++i) {
      rc = pcg_step(e->runs[i], 1);
      if (rc != PCG_OK) e->broken = true;  // earlier runs advanced their host state without their kernels
    }
  for (int i = 0; rc == PCG_OK && i < n; ++i)
    if (cudaEventRecord(e->done[i], e->streams[i]) != cudaSuccess ||
        cudaStreamWaitEvent(e->join, e->done[i], 0) != cudaSuccess)
      rc = PCG_ERR_CUDA;
  cudaGraph_t g = nullptr;
  const cudaError_t end = cudaStreamEndCapture(e->join, &g);
  if (rc != PCG_OK || end != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    e->broken = true;
    return rc != PCG_OK ? rc : PCG_ERR_CUDA;
  }
  if (e->exec) {  // same shape as the last batch: update its executable graph in place
    cudaGraphExecUpdateResultInfo info;
    if (cudaGraphExecUpdate(e->exec, g, &info) != cudaSuccess) {
      cudaGetLastError();
      cudaGraphExecDestroy(e->exec);
      e->exec = nullptr;
    }
  }
  if (!e->exec && cudaGraphInstantiate(&e->exec, g, 0) != cudaSuccess) {
    cudaGraphDestroy(g);
    e->exec = nullptr;
    e->broken = true;
    return PCG_ERR_CUDA;
  }
  size_t nodes = 0;
  cudaGraphGetNodes(g, nullptr, &nodes);
  cudaGraphDestroy(g);
  e->graph_nodes = nodes;
  e->capture_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (cudaEventRecord(e->start, e->join) != cudaSuccess || cudaGraphLaunch(e->exec, e->join) != cudaSuccess ||
      cudaEventRecord(e->stop, e->join) != cudaSuccess || cudaEventSynchronize(e->stop) != cudaSuccess)
    return PCG_ERR_CUDA;
  if (device_ms && cudaEventElapsedTime(device_ms, e->start, e->stop) != cudaSuccess) return PCG_ERR_CUDA;
  for (pcg_handle* h : e->runs) {  // device-side errors (NaN, capacity, ...) of any run
    const int rs = pcg_synchronize(h);
    if (rs != PCG_OK) return rs;
  }
  return PCG_OK;
}

}  // namespace

extern "C" {

int pcg_ensemble_set_graph(pcg_ensemble* e, int on) {
  if (!e) return PCG_ERR_ARG;
  e->graph = on != 0;
  return PCG_OK;
}

int pcg_ensemble_graph_info(pcg_ensemble* e, unsigned long long* nodes, float* capture_ms) {
  if (!e) return PCG_ERR_ARG;
  if (nodes) *nodes = e->graph_nodes;
  if (capture_ms) *capture_ms = e->capture_ms;
  return PCG_OK;
}

int pcg_ensemble_step(pcg_ensemble* e, int nsteps, float* device_ms) {
  pcg::DeviceScope device_scope(e ? e->device : -1);
  if (!e || nsteps < 0) return PCG_ERR_ARG;
  if (e->broken) return PCG_ERR_STATE;
  if (e->graph && e->stepped && nsteps > 0) return graph_step(e, nsteps, device_ms);
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
  if (nsteps > 0) e->stepped = true;
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
  if (e->exec) cudaGraphExecDestroy(e->exec);
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->start) cudaEventDestroy(e->start);
  if (e->stop) cudaEventDestroy(e->stop);
  if (e->join) cudaStreamDestroy(e->join);
  delete e;
  return PCG_OK;
}

}  // extern "C"
