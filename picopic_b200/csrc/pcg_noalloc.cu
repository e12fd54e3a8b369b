// pcg_noalloc.cu — the Villasenor-Buneman current deposit of one species
// from caller-owned device arrays, without allocating device memory.
//
// Some hosts cannot let a library call cudaMalloc: codes coupled to another
// solver that owns and pre-partitions the device memory, and hosts that
// must avoid cudaMalloc's implicit device synchronisation inside a timed
// loop.  For them this entry point keeps its only scratch (the per-node
// record of the strict-axial J_r overwrite, and a move-error counter) in a
// file-scope device array of fixed size, which every GPU that loads the
// library holds until the process exits.
//
// Built with --fmad=false, like the other double-precision kernels.
#include <cuda_runtime.h>

#include <mutex>

#include "pcg.h"
#include "pcg_f64.cuh"

namespace {

using namespace pcg;
using namespace pcg::f64;

constexpr int kThreads = 256;

// Scratch shared by every call on a device: one word per grid node (with
// halo) plus the move-error counter.  2 MiB.
constexpr long long kNoallocMaxNodes = PCG_NOALLOC_MAX_NODES;
static __device__ __align__(256) unsigned long long g_reset[kNoallocMaxNodes];
static __device__ __align__(256) unsigned long long g_move_errors;

struct Scratch {
  unsigned long long* reset = nullptr;
  unsigned long long* move_errors = nullptr;
};

// Host code must not use g_reset's name as a device address; the address is
// looked up with the device current, once per device and context.  The
// context's id is part of the key: after a cudaDeviceReset the runtime loads
// the module again, possibly elsewhere, in a new primary context, and a
// cached address from the old one would point at freed memory.
constexpr int kMaxDevices = 64;
struct Cached {
  unsigned long long ctx_id = 0;
  bool ready = false;
  Scratch s;
};
Cached g_cache[kMaxDevices];
std::mutex g_lock;

typedef int (*CtxGetCurrentFn)(void**);
typedef int (*CtxGetIdFn)(void*, unsigned long long*);

// The current context's id through the driver's entry points (the runtime
// has no call for it); 0 when the driver cannot say.
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool looked = false;
  if (!looked) {
    looked = true;
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", (void**)&get_current, cudaEnableDefault, &q1) != cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess)
      get_current = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", (void**)&get_id, cudaEnableDefault, &q2) != cudaSuccess ||
        q2 != cudaDriverEntryPointSuccess)
      get_id = nullptr;
  }
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

int scratch_for_current_device(Scratch* out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return PCG_ERR_CUDA;
  std::lock_guard<std::mutex> guard(g_lock);
  Cached& c = g_cache[dev];
  // once looked up, the context exists; a reset context reads as another id
  // (or none), and a driver without context ids makes every call look up again
  const unsigned long long ctx = c.ready ? current_context_id() : 0;
  if (!c.ready || ctx == 0 || ctx != c.ctx_id) {
    Scratch s;
    c.ready = false;
    if (cudaGetSymbolAddress((void**)&s.reset, g_reset) != cudaSuccess) return PCG_ERR_CUDA;
    if (cudaGetSymbolAddress((void**)&s.move_errors, g_move_errors) != cudaSuccess) return PCG_ERR_CUDA;
    c.s = s;
    c.ctx_id = current_context_id();  // the lookup made the device's primary context current
    c.ready = true;
  }
  *out = c.s;
  return PCG_OK;
}

struct Particles {
  size_t n;
  const double *r, *z, *r_old, *z_old, *vphi, *w;
  double charge;  // SI
};

__global__ void halo_zero(GridGeom g, double* a0, double* a1, double* a2) {
  const int kk = blockIdx.x * blockDim.x + threadIdx.x;
  const int ii = blockIdx.y;
  if (kk >= g.nz + 4) return;
  const int i = ii - 2, k = kk - 2;
  if (i < 0 || k < 0 || i >= g.nr || k >= g.nz) {
    const long long p = (long long)ii * g.ld + kk;
    a0[p] = 0; a1[p] = 0; a2[p] = 0;
  }
}

__global__ void azimuthal(GridGeom g, Particles p, double* jr, double* jp, double* jz) {
  const size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= p.n || p.r[j] < 0) return;
  Sink s{{jr, jp, jz}, nullptr, 0, &g, false};
  vb_azimuthal(s, p.charge * p.w[j], p.r[j], p.z[j], p.r_old[j], p.z_old[j], p.vphi[j],
               cell_number(p.r[j], g.dr), cell_number(p.z[j], g.dz));
}

__global__ void mark_overwrites(GridGeom g, Particles p, int fixed, unsigned long long* reset) {
  const size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= p.n || p.r[j] < 0) return;
  int i_n, k_n;
  if (vb_strict_axial_nodes(g, fixed, p.r[j], p.z[j], p.r_old[j], p.z_old[j],
                            cell_number(p.r[j], g.dr), &i_n, &k_n)) {
    const unsigned long long o1 = (unsigned long long)j + 1;
    atomicMax(reset + gidx(g, i_n, k_n), o1);
    atomicMax(reset + gidx(g, i_n, k_n + 1), o1);
  }
}

__global__ void clear_overwritten(long long nodes, const unsigned long long* reset, double* jr) {
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q < nodes && reset[q] != 0) jr[q] = 0.0;
}

__global__ void rz(GridGeom g, Particles p, int fixed, const unsigned long long* reset,
                   unsigned long long* move_errors, double* jr, double* jp, double* jz) {
  const size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= p.n || p.r[j] < 0) return;
  Sink s{{jr, jp, jz}, reset, (unsigned long long)j + 1, &g, false};
  if (!vb_rz(s, fixed, p.charge * p.w[j], p.r[j], p.z[j], p.r_old[j], p.z_old[j],
             cell_number(p.r[j], g.dr), cell_number(p.z[j], g.dz)))
    atomicAdd(move_errors, 1ull);
}

}  // namespace

extern "C" int pcg_current_vb_f64_noalloc(int nr, int nz, double radius, double longitude,
                                          double dt, size_t n, double charge_e, const double* r,
                                          const double* z, const double* r_old,
                                          const double* z_old, const double* vphi,
                                          const double* w, double* j_r, double* j_phi,
                                          double* j_z, int quirks, void* stream,
                                          unsigned long long* move_errors) {
  if (nr < 2 || nz < 2 || !(radius > 0) || !(longitude > 0) || !(dt > 0)) return PCG_ERR_ARG;
  if (quirks != PCG_QUIRKS_REFERENCE && quirks != PCG_QUIRKS_FIXED) return PCG_ERR_ARG;
  if (!j_r || !j_phi || !j_z || (n && !(r && z && r_old && z_old && vphi && w))) return PCG_ERR_ARG;
  const long long nodes = (long long)(nr + 4) * (long long)(nz + 4);
  if (nodes > kNoallocMaxNodes) return PCG_ERR_CAPACITY;  // (nr+4)*(nz+4) above the fixed scratch
  cudaStream_t s = (cudaStream_t)stream;
  if (move_errors) {  // the count's read-back synchronises the stream, which a capture forbids
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) return PCG_ERR_CUDA;
    if (cs != cudaStreamCaptureStatusNone) return PCG_ERR_STATE;
  }
  Scratch sc;
  int rc = scratch_for_current_device(&sc);
  if (rc != PCG_OK) return rc;
  GridGeom g{};
  g.nr = nr; g.nz = nz; g.ld = nz + 4;
  g.R = radius; g.L = longitude;
  g.dr = radius / nr; g.dz = longitude / nz; g.dt = dt;
  Particles p{n, r, z, r_old, z_old, vphi, w, charge_e * kElCharge};
  const int fixed = quirks == PCG_QUIRKS_FIXED;
  // the scratch keeps the previous call's contents: clear it first
  if (cudaMemsetAsync(sc.reset, 0, sizeof(unsigned long long) * nodes, s) != cudaSuccess) return PCG_ERR_CUDA;
  if (cudaMemsetAsync(sc.move_errors, 0, sizeof(unsigned long long), s) != cudaSuccess) return PCG_ERR_CUDA;
  const dim3 hgrid((g.nz + 4 + kThreads - 1) / kThreads, g.nr + 4);
  const unsigned pb = (unsigned)((n + kThreads - 1) / kThreads);
  // CurrentVB::current_distribution (currentVB.cpp:731-735): azimuthal, then
  // rz, each starting with overlay_set(0) on J.
  halo_zero<<<hgrid, kThreads, 0, s>>>(g, j_r, j_phi, j_z);
  if (n) azimuthal<<<pb, kThreads, 0, s>>>(g, p, j_r, j_phi, j_z);
  halo_zero<<<hgrid, kThreads, 0, s>>>(g, j_r, j_phi, j_z);
  if (n) mark_overwrites<<<pb, kThreads, 0, s>>>(g, p, fixed, sc.reset);
  clear_overwritten<<<(unsigned)((nodes + kThreads - 1) / kThreads), kThreads, 0, s>>>(nodes, sc.reset, j_r);
  if (n) rz<<<pb, kThreads, 0, s>>>(g, p, fixed, sc.reset, sc.move_errors, j_r, j_phi, j_z);
  if (cudaGetLastError() != cudaSuccess) return PCG_ERR_CUDA;
  if (move_errors) {
    if (cudaMemcpyAsync(move_errors, sc.move_errors, sizeof(unsigned long long),
                        cudaMemcpyDeviceToHost, s) != cudaSuccess)
      return PCG_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return PCG_ERR_CUDA;
  }
  return PCG_OK;
}
