// pcg_api.cu — host implementation of the C ABI declared in include/pcg.h.
//
// A handle owns one domain: the field grids (Grid<double> layout with the
// 2-cell halo), the PML profile, the species buffers, one CUDA stream and a
// device status block.  Work is queued on the stream; calls that return
// data (export, diag, synchronize) wait for it and turn the device error
// word into a status code.
#include <cuda_runtime.h>
#include <cub/device/device_select.cuh>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pcg.h"
#include "pcg_collide.h"
#include "pcg_device.h"
#include "pcg_diag.h"
#include "pcg_f32.h"
#include "pcg_init.h"
#include "pcg_learned.h"
#include "pcg_maps.h"
#include "pcg_kernels.h"
#include "pcg_region.h"
#include "pcg_yee.cuh"

using namespace pcg;

namespace {

struct Species {
  int id = 0;
  std::string name;
  double charge_e = 0, mass_e = 0, charge = 0, mass = 0;
  bool beam = false;
  size_t cap = 0, n = 0;
  unsigned long long order_base = 0;  // unused slots are never reused before compaction
  // BeamP state (beamP.cpp:22-69)
  unsigned macro_amount = 0, bunches_amount = 0, current_bunch = 0;
  double start_time = 0, radius = 0, density = 0, bunch_length = 0, bunches_distance = 0,
         velocity = 0, finish_time = 0, domain_radius = 0, bunch_macro_amount = 0,
         macro_per_step = 0;
  // PCG_PROFILE_GAUSSIAN
  int profile = PCG_PROFILE_RECTANGLE;
  double sigma_z = 0, gauss_mps = 0;
  // double layout
  double *r = nullptr, *z = nullptr, *vr = nullptr, *vphi = nullptr, *vz = nullptr,
         *w = nullptr, *r_old = nullptr, *z_old = nullptr;
  double *phi = nullptr, *phi_old = nullptr, *sn = nullptr;
  int *cell_r = nullptr, *cell_z = nullptr;
  // float layout
  SpeciesF32Buffers f32;
  double* abs_map = nullptr;  // momentum_abs_map_w as the last energy map left it (pcg_species_map)
};

const char* kFieldNames[12] = {"E_r", "E_phi", "E_z", "H_r", "H_phi", "H_z",
                               "Hat_r", "Hat_phi", "Hat_z", "J_r", "J_phi", "J_z"};

}  // namespace

struct pcg_handle {
  pcg_config cfg{};
  GridGeom g{};
  cudaStream_t stream = nullptr;
  cudaStream_t aux = nullptr;     // float steps: the second stream of the species' step kernels
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // host particle uploads: copies on their own stream, so that the caller
  // waits for its copies only, not for the steps queued before them
  cudaStream_t copy = nullptr;
  cudaEvent_t ev_copied = nullptr, ev_staging_free = nullptr;
  // pcg_step_status: the status block of the last step, copied without waiting
  DevStatus* h_status_lag = nullptr;
  cudaEvent_t ev_status = nullptr;
  // device-to-device hand-over between handles: orders the two streams
  cudaEvent_t ev_region = nullptr;
  bool status_pending = false;
  DevStatus* d_status = nullptr;
  DevStatus* h_status = nullptr;  // pinned mirror
  size_t nodes = 0;               // (nr+4)*(nz+4)
  double* f64[12] = {};
  float* f32[12] = {};            // planes of one allocation, f32_plane floats apart
  size_t f32_plane = 0;
  float4* recip32 = nullptr;      // radial reciprocal table of the float step
  uint64_t dead_dropped = 0;      // dead slots the float tile sorts dropped since the last compaction
  double* map_work = nullptr;     // pcg_species_map: 4 scratch grids and 3 output grids
  uint64_t launches = 0;          // kernels launched by steps and stages
  double* diag = nullptr;         // node-value scratch of the diagnostics
  CollWork coll;                  // scratch of the collision passes
  LearnedWork learned;            // the learned collision step: model and scratch
  uint32_t coll_pass = 0;         // collision passes so far (their Philox counter)
  int collisions = PCG_COLLISIONS_NONE;  // collision operator of every pcg_step
  int coll_scheme = PCG_COLLIDE_P12;     // binary operator of pcg_collide and binary steps
  unsigned coll_crowded = 256;           // particles above which a cell's pairs take a warp
  // external fields (pcg_set_external_fields): E_r, E_phi, E_z, H_r, H_phi,
  // H_z planes of nodes doubles (double path) and floats (float path), and
  // the float step's gather planes E + E_ext, H + H_ext, f32_plane apart
  double* ext64 = nullptr;
  float* ext32 = nullptr;
  float* push32 = nullptr;
  double* sig64[3] = {};          // r, z0, zl profiles
  float* sig32[3] = {};
  unsigned long long* reset = nullptr;
  std::vector<Species> sp;
  double t = 0;
  uint64_t steps = 0, particle_steps = 0;
  bool staged = false;   // stage-by-stage buffers allocated
  bool started = false;  // particles imported or stepped: species list frozen
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  // pcg_export_species_range: selection scratch and the gathered particles
  unsigned char* region = nullptr;
  size_t region_bytes = 0;
  double* region_out = nullptr;
  size_t region_out_n = 0;
  unsigned* h_count = nullptr;  // pinned: the band counts of a selection
  int h_count_n = 0;
  double* staging = nullptr;  // host-to-device particle staging, reused
  size_t staging_n = 0;
  // kernel timers: event pairs per class, recycled after each query
  TileGrid tiles{};       // float path: tile sort geometry
  int sort_interval = 64;  // float path: most steps between tile sorts
  // float path: blocks per tile (pcg_set_tiling).  148 x 16 blocks: with
  // 4 resident blocks per SM one block per occupied tile of a 256 x 4096
  // grid (2048 tiles) runs 3.5 waves and leaves the last half empty; two
  // per tile run 6.9
  unsigned target_blocks = 148 * 16, min_split = 1024;
  bool timers = false;
  // set when a tensor-core wait timed out: the kernel's TMEM may still be in
  // use, so the handle refuses further steps and collisions
  bool halted = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_used;
  std::string err;
};

namespace {

int fail(pcg_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

#define CUDA_TRY(h, expr)                                                        \
  do {                                                                           \
    cudaError_t e_ = (expr);                                                     \
    if (e_ != cudaSuccess)                                                       \
      return fail((h), PCG_ERR_CUDA, std::string(#expr ": ") + cudaGetErrorString(e_)); \
  } while (0)

template <typename T>
int dalloc(pcg_handle* h, T** p, size_t count) {
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
  if (e != cudaSuccess) return fail(h, PCG_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  return PCG_OK;
}

bool is_f64(const pcg_handle* h) { return h->cfg.precision == PCG_PRECISION_F64; }

// True for memory the GPU addresses directly (a device or managed
// allocation): the particle and column calls then copy device to device.
bool device_memory(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // plain host memory on older drivers
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}


// PML profiles of MaxwellSolverYee::set_pml (maxwellSolverYee.cpp:57-109):
// each wall adds a quadratic ramp that depends on i alone (r=R) or k alone
// (z=0, z=L), so sigma(i,k) = sig_r[i] + sig_z0[k] + sig_zl[k].
void pml_profiles(const pcg_config& c, const GridGeom& g, std::vector<double>& sr,
                  std::vector<double>& s0, std::vector<double>& sl) {
  sr.assign(g.nr, 0.0);
  s0.assign(g.nz, 0.0);
  sl.assign(g.nz, 0.0);
  const double dr = g.dr, dz = g.dz;
  const double l_left = dz * (double)c.pml_size[1];
  const double l_right = dz * (double)c.pml_size[3];
  const double l_ext = dr * (double)c.pml_size[2];
  const double dsig = c.pml_sigma[1] - c.pml_sigma[0];
  const size_t gcr = (size_t)(g.R / dr), gcz = (size_t)(g.L / dz);  // geometry.hpp:70-71
  if (c.pml_size[2] != 0)
    for (int i = 0; i < g.nr; i++) {
      double dist = (double)(gcr - 0 - (size_t)i) * dr;
      if (dist < l_ext)
        sr[i] = c.pml_sigma[0] + dsig / pow(l_ext, 2) * pow(dr * (i + 1) + 0.0 * dr - g.R + l_ext, 2);
    }
  if (c.pml_size[1] != 0)
    for (int k = 0; k < g.nz; k++)
      if (dz * k + 0.0 * dz < l_left)
        s0[k] = c.pml_sigma[0] + dsig / pow(l_left, 2) * pow(l_left - dz * k - 0.0 * dz, 2);
  if (c.pml_size[3] != 0)
    for (int k = 0; k < g.nz; k++) {
      double dist = (double)(gcz - 0 - (size_t)k) * dz;
      if (dist < l_right)
        sl[k] = c.pml_sigma[0] + dsig / pow(l_right, 2) * pow(dz * (k + 1) + 0.0 * dz - g.L + l_right, 2);
    }
}

FieldsF64 fields64(pcg_handle* h) {
  FieldsF64 f;
  for (int c = 0; c < 3; ++c) {
    f.E[c] = h->f64[c]; f.H[c] = h->f64[3 + c]; f.Hat[c] = h->f64[6 + c]; f.J[c] = h->f64[9 + c];
  }
  f.sig_r = h->sig64[0]; f.sig_z0 = h->sig64[1]; f.sig_zl = h->sig64[2];
  f.ext = h->ext64;
  return f;
}

template <typename Real>
YeeArgs<Real> yee_args(pcg_handle* h, Real* const* fld, Real* const* sig, int zero_j) {
  YeeArgs<Real> a;
  a.g = h->g;
  for (int c = 0; c < 3; ++c) {
    a.E[c] = fld[c]; a.H[c] = fld[3 + c]; a.Hat[c] = fld[6 + c]; a.J[c] = fld[9 + c];
  }
  a.sig_r = sig[0]; a.sig_z0 = sig[1]; a.sig_zl = sig[2];
  a.zero_j = zero_j;
  a.st = h->d_status;
  return a;
}

SpeciesF64 view64(pcg_handle* h, Species& s) {
  SpeciesF64 v;
  v.n = s.n;
  v.r = s.r; v.z = s.z; v.vr = s.vr; v.vphi = s.vphi; v.vz = s.vz; v.w = s.w;
  v.r_old = s.r_old; v.z_old = s.z_old;
  v.phi = s.phi; v.phi_old = s.phi_old; v.sn = s.sn;
  v.cell_r = s.cell_r; v.cell_z = s.cell_z;
  v.charge = s.charge; v.mass = s.mass;
  v.c2m = s.charge * h->cfg.dt / (2 * s.mass);
  v.is_beam = s.beam ? 1 : 0;
  return v;
}

int alloc_species(pcg_handle* h, Species& s) {
  int rc;
  if (is_f64(h)) {
    double** arrs[] = {&s.r, &s.z, &s.vr, &s.vphi, &s.vz, &s.w, &s.r_old, &s.z_old};
    for (double** a : arrs)
      if ((rc = dalloc(h, a, s.cap)) != PCG_OK) return rc;
  } else {
    if ((rc = f32_alloc_species(s.f32, s.cap, h->tiles)) != 0)
      return fail(h, PCG_ERR_NOMEM, "cudaMalloc of a float species failed");
  }
  return PCG_OK;
}

int ensure_staged(pcg_handle* h) {
  if (h->staged) return PCG_OK;
  if (!is_f64(h)) return fail(h, PCG_ERR_UNSUPPORTED, "stage-by-stage calls need PCG_PRECISION_F64");
  for (Species& s : h->sp) {
    int rc;
    double** arrs[] = {&s.phi, &s.phi_old, &s.sn};
    for (double** a : arrs) {
      if ((rc = dalloc(h, a, s.cap)) != PCG_OK) return rc;
      CUDA_TRY(h, cudaMemsetAsync(*a, 0, sizeof(double) * s.cap, h->stream));
    }
    if ((rc = dalloc(h, &s.cell_r, s.cap)) != PCG_OK) return rc;
    if ((rc = dalloc(h, &s.cell_z, s.cap)) != PCG_OK) return rc;
    // bind the current positions, as after SpecieP::bind_cell_numbers
    SpeciesF64 v = view64(h, s);
    launch_stage_f64(PCG_STAGE_BIND, h->g, fields64(h), v, 0, 0, 0, h->d_status, h->stream);
  }
  h->staged = true;
  return PCG_OK;
}

int status_code(pcg_handle* h, const DevStatus* st);

int check_status(pcg_handle* h) {
  CUDA_TRY(h, cudaMemcpyAsync(h->h_status, h->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost,
                              h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  CUDA_TRY(h, cudaGetLastError());
  return status_code(h, h->h_status);
}

// The error word of a status block as a PCG_ERR_* code.
int status_code(pcg_handle* h, const DevStatus* st) {
  unsigned e = st->error;
  if (e & kErrNanPosition) return fail(h, PCG_ERR_NAN, "particle position is not a finite number");
  if (e & kErrNanField) return fail(h, PCG_ERR_NAN, "electric field became NaN");
  if (e & kErrSuperluminal) return fail(h, PCG_ERR_SUPERLUMINAL, "particle speed above c");
  if (e & kErrReflectLoop) return fail(h, PCG_ERR_STATE, "wall reflection did not converge");
  if (e & kErrOutOfGrid) return fail(h, PCG_ERR_STATE, "particle outside the grid");
  if (e & kErrCapacity) return fail(h, PCG_ERR_CAPACITY, "species capacity exceeded");
  if (e & kErrUnsupported) return fail(h, PCG_ERR_UNSUPPORTED, "switch combination not implemented");
  if (e & kErrTimeout) return fail(h, PCG_ERR_TIMEOUT, "a bounded wait in a kernel ran out");
  return PCG_OK;
}

// BeamP::inject timing (beamP.cpp:73-156), evaluated on the host in the
// reference's double arithmetic: returns how many particles to add now.
unsigned beam_count(pcg_handle* h, Species& s, BeamInject* b, int slot) {
  unsigned count = 0;
  if (s.profile == PCG_PROFILE_GAUSSIAN) {
    // 6 sigma_z of bunch pass z = 0 starting at start_time; the number of
    // macroparticles entering during step m is floor((m+1) a) - floor(m a).
    const double since = h->t - s.start_time;
    const double window = 6.0 * s.sigma_z / s.velocity;
    if (since < 0 || since >= window) return 0;
    const double m = floor(since / h->cfg.dt + 0.5);
    count = (unsigned)(floor((m + 1) * s.gauss_mps) - floor(m * s.gauss_mps));
    const double dr = h->g.dr, dz = h->g.dz;
    b->seed = h->cfg.seed;
    b->stream = 0x6265616du + (uint32_t)slot;
    b->step = h->steps;
    b->dl = s.velocity * h->cfg.dt;
    b->half_z = dz / 2.;
    b->velocity = s.velocity;
    b->profile = 1;
    b->r_min = 0.5 * dr;
    b->radius = s.radius;
    b->sigma = s.sigma_z;
    b->head_dist = (m + 1) * b->dl;
    // equal-volume macroparticles: the slab volume of one step over its count
    const double slab = kPi * (s.radius * s.radius - b->r_min * b->r_min) * b->dl;
    b->w0 = s.density * slab / s.gauss_mps;
    return count;
  }
  if (s.current_bunch < s.bunches_amount) {
    double bunch_start = s.start_time + (s.bunch_length + s.bunches_distance) / s.velocity * s.current_bunch;
    double bunch_finish = bunch_start + s.bunch_length / s.velocity;
    if (0.0 * h->g.dr < s.radius && h->t >= bunch_start && h->t < bunch_finish) {
      const double dr = h->g.dr, dz = h->g.dz;
      b->seed = h->cfg.seed;
      b->stream = 0x6265616du + (uint32_t)slot;
      b->step = h->steps;
      b->domain_radius = s.domain_radius;
      b->dl = s.velocity * h->cfg.dt;
      b->half_z = dz / 2.;
      b->velocity = s.velocity;
      b->v_macro_avg = kPi * s.radius * dr * dz;
      double N_total = kPi * s.radius * s.radius * s.bunch_length * s.bunches_amount * s.density;
      b->n_per_macro_avg = N_total / s.macro_amount;
      for (unsigned i = 0; i < s.macro_per_step; ++i) ++count;
    }
    if (h->t > bunch_finish) ++s.current_bunch;
  }
  return count;
}

// Kernel timers: an event pair around each timed launch group.
cudaEvent_t timer_event(pcg_handle* h) {
  if (!h->ev_pool.empty()) {
    cudaEvent_t e = h->ev_pool.back();
    h->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

struct TimerScope {
  pcg_handle* h;
  int cls;
  cudaEvent_t a = nullptr, b = nullptr;
  TimerScope(pcg_handle* hh, int c) : h(hh), cls(c) {
    if (!h->timers) return;
    a = timer_event(h);
    b = timer_event(h);
    cudaEventRecord(a, h->stream);
  }
  ~TimerScope() {
    if (!h->timers) return;
    cudaEventRecord(b, h->stream);
    h->ev_used.push_back({cls, {a, b}});
  }
};

int compact(pcg_handle* h);

int stage_inject(pcg_handle* h) {
  TimerScope ts(h, PCG_TIMER_INJECT);
  for (size_t t = 0; t < h->sp.size(); ++t) {
    Species& s = h->sp[t];
    if (!s.beam) continue;
    BeamInject b{};
    unsigned count = beam_count(h, s, &b, (int)t);
    if (count == 0) continue;
    if (s.n + count > s.cap && !is_f64(h)) {
      // the dead slots that the float sorts left behind still count in n:
      // remove them (this waits for the stream) before giving up
      int rc = check_status(h);
      if (rc != PCG_OK) return rc;
      if (h->h_status->dead_slots > h->dead_dropped && (rc = compact(h)) != PCG_OK) return rc;
    }
    if (s.n + count > s.cap) return fail(h, PCG_ERR_CAPACITY, "beam '" + s.name + "' capacity exceeded");
    if (is_f64(h)) {
      launch_inject_f64(h->g, view64(h, s), s.n, count, b, h->stream);
    } else {
      f32_launch_inject(h->g, s.f32, s.n, count, b, h->d_status, h->stream);
    }
    s.n += count;
    h->launches += 1;
  }
  return PCG_OK;
}

// Stable removal of dead slots (the erase of std::remove_if, SMB.cpp:216-345).
int compact(pcg_handle* h) {
  for (Species& s : h->sp) {
    if (s.n == 0) continue;
    size_t n = s.n;
    unsigned* idx = nullptr;
    unsigned* nsel = nullptr;
    unsigned char* flags = nullptr;
    int rc;
    if ((rc = dalloc(h, &idx, 2 * n + 1)) != PCG_OK) return rc;
    nsel = idx + 2 * n;
    if ((rc = dalloc(h, &flags, n)) != PCG_OK) return rc;
    if (is_f64(h)) f64_alive_flags(s.r, flags, n, h->stream);
    else f32_alive_flags(s.f32, flags, n, h->stream);
    iota_u32(idx + n, n, h->stream);
    size_t tmp = 0;
    cub::DeviceSelect::Flagged(nullptr, tmp, idx + n, flags, idx, nsel, (int)n, h->stream);
    if (tmp > h->scratch_bytes) {
      cudaFree(h->scratch);
      h->scratch = nullptr;
      if ((rc = dalloc(h, (unsigned char**)&h->scratch, tmp)) != PCG_OK) return rc;
      h->scratch_bytes = tmp;
    }
    cub::DeviceSelect::Flagged(h->scratch, tmp, idx + n, flags, idx, nsel, (int)n, h->stream);
    unsigned kept = 0;
    CUDA_TRY(h, cudaMemcpyAsync(&kept, nsel, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    if (kept != n) {
      if (is_f64(h)) {
        double* tmpd = nullptr;
        if ((rc = dalloc(h, &tmpd, kept)) != PCG_OK) return rc;
        double* arrs[] = {s.r, s.z, s.vr, s.vphi, s.vz, s.w, s.r_old, s.z_old, s.phi, s.phi_old, s.sn};
        for (double* a : arrs) {
          if (!a) continue;
          launch_gather_f64(a, tmpd, idx, kept, h->stream);
          CUDA_TRY(h, cudaMemcpyAsync(a, tmpd, sizeof(double) * kept, cudaMemcpyDeviceToDevice, h->stream));
        }
        int* arri[] = {s.cell_r, s.cell_z};
        for (int* a : arri) {
          if (!a) continue;
          launch_gather_i32(a, (int*)tmpd, idx, kept, h->stream);
          CUDA_TRY(h, cudaMemcpyAsync(a, tmpd, sizeof(int) * kept, cudaMemcpyDeviceToDevice, h->stream));
        }
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
        cudaFree(tmpd);
      } else {
        if (f32_compact(s.f32, idx, kept, h->stream) != 0) return fail(h, PCG_ERR_NOMEM, "compaction");
      }
      s.n = kept;
    }
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    cudaFree(idx);
    cudaFree(flags);
  }
  CUDA_TRY(h, cudaMemsetAsync(&h->d_status->dead_slots, 0, sizeof(unsigned long long), h->stream));
  h->dead_dropped = 0;
  return PCG_OK;
}

int run_stage(pcg_handle* h, int stage) {
  int rc;
  const int fixed = h->cfg.quirks == PCG_QUIRKS_FIXED;
  // Stage-by-stage mode keeps every Particle field of the reference on the
  // device (phi, old phi, sin, bound cells), from the first stage on.
  if (is_f64(h) && (rc = ensure_staged(h)) != PCG_OK) return rc;
  if (stage == PCG_STAGE_INJECT) return stage_inject(h);
  if (stage == PCG_STAGE_ADVANCE_TIME) {
    h->t += h->cfg.dt;
    h->steps += 1;
    return PCG_OK;
  }
  if (stage == PCG_STAGE_FIELD_E || stage == PCG_STAGE_FIELD_H) {
    if (is_f64(h)) {
      YeeArgs<double> a = yee_args<double>(h, h->f64, h->sig64, 0);
      if (stage == PCG_STAGE_FIELD_E) launch_yee_e_f64(a, h->stream);
      else launch_yee_h_f64(a, fixed, h->stream);
    } else {
      YeeArgs<float> a = yee_args<float>(h, h->f32, h->sig32, 0);
      if (stage == PCG_STAGE_FIELD_E) f32_launch_yee_e(a, h->stream);
      else f32_launch_yee_h(a, fixed, h->stream);
    }
    return PCG_OK;
  }
  if (stage == PCG_STAGE_RESET_CURRENT) {  // Domain::reset_current domain.cpp:135-139
    for (int c = 9; c < 12; ++c) {
      if (is_f64(h)) CUDA_TRY(h, cudaMemsetAsync(h->f64[c], 0, sizeof(double) * h->nodes, h->stream));
      else CUDA_TRY(h, cudaMemsetAsync(h->f32[c], 0, sizeof(float) * h->nodes, h->stream));
    }
    return PCG_OK;
  }
  if ((rc = ensure_staged(h)) != PCG_OK) return rc;
  FieldsF64 f = fields64(h);
  if (stage == PCG_STAGE_CURRENT) {
    std::vector<SpeciesF64> v;
    for (Species& s : h->sp) v.push_back(view64(h, s));
    launch_current_stage_f64(h->g, f, v.data(), (int)v.size(), fixed, h->cfg.current, h->reset,
                             h->d_status, h->stream);
    return PCG_OK;
  }
  if (stage < PCG_STAGE_PUSH || stage > PCG_STAGE_COLLECT) return fail(h, PCG_ERR_ARG, "unknown stage");
  for (size_t t = 0; t < h->sp.size(); ++t)
    launch_stage_f64(stage, h->g, f, view64(h, h->sp[t]), (int)t, h->cfg.pusher, fixed,
                     h->d_status, h->stream);
  return PCG_OK;
}

// One fused step (PiCoPiC.cpp:326-347).
// The collision list of a species: ions ("ions" or "Ions"), electrons every
// other species (collisions.cpp:87-108).
bool is_ion_list(const Species& s) { return s.name == "ions" || s.name == "Ions"; }

// The species as the collision passes see them, and the masses and charges
// of the species named electrons and ions (collisions.cpp:28-48: the last
// match wins).  False when either is missing.
bool collision_species(pcg_handle* h, std::vector<CollSpecies>& v, CollParams& p) {
  int el = -1, ion = -1;
  v.assign(h->sp.size(), CollSpecies());
  for (size_t t = 0; t < h->sp.size(); ++t) {
    Species& s = h->sp[t];
    if (s.name == "electrons" || s.name == "Electrons") el = (int)t;
    if (s.name == "ions" || s.name == "Ions") ion = (int)t;
    CollSpecies& c = v[t];
    c.n = s.n;
    c.is_ion = is_ion_list(s);
    if (is_f64(h)) {
      c.r = s.r; c.z = s.z; c.vr64 = s.vr; c.vphi64 = s.vphi; c.vz64 = s.vz; c.w64 = s.w;
    } else {
      c.cell = s.f32.cell; c.id = s.f32.id; c.id_bound = s.f32.next_id;
      c.vr32 = s.f32.vr; c.vphi32 = s.f32.vphi; c.vz32 = s.f32.vz; c.w32 = s.f32.w;
      c.tile_start = s.f32.tile_start;
      c.cell_count = s.f32.cell_count;
      c.layer_mask = s.f32.layer_mask;
      c.layer_prefix = s.f32.layer_prefix;
      c.layer_start = s.f32.layer_start;
      c.sorted = std::min(s.f32.sorted_n, s.n);
    }
  }
  if (el < 0 || ion < 0) return false;
  p.m_el = h->sp[el].mass; p.q_el = h->sp[el].charge;
  p.m_ion = h->sp[ion].mass; p.q_ion = h->sp[ion].charge;
  p.dt = h->cfg.dt;
  p.fixed = h->cfg.quirks == PCG_QUIRKS_FIXED;
  p.shuffle = 1;
  p.seed = h->cfg.seed;
  p.status = h->d_status;
  return true;
}

LearnedPhys learned_phys(const CollParams& p) {
  return LearnedPhys{p.m_el, p.q_el, p.m_ion, p.q_ion, p.dt};
}

// One binary collision pass (no status check).
int run_collide(pcg_handle* h, unsigned long long* pair_calls) {
  if (h->sp.size() > (size_t)kCollMaxSpecies) return fail(h, PCG_ERR_UNSUPPORTED, "too many species for collisions");
  CollParams p{};
  std::vector<CollSpecies> v;
  if (!collision_species(h, v, p))
    return fail(h, PCG_ERR_STATE, "collisions need species named 'electrons' and 'ions'");
  p.pass = h->coll_pass++;
  p.scheme = h->coll_scheme;
  p.crowded = h->coll_crowded;
  unsigned long long calls = 0;
  if (collide_p12(h->g, v.data(), (int)v.size(), p, h->coll, &calls, h->stream) != 0)
    return fail(h, PCG_ERR_CUDA, "collision pass");
  h->launches += h->coll.launches;
  if (pair_calls) *pair_calls = calls;
  return PCG_OK;
}

// One learned collision step with the binary fallback (no status check).
// In a fused float step (in_step) the move applies the transforms.
int run_collide_learned(pcg_handle* h, unsigned long long* learned_cells, unsigned long long* fallback_cells,
                        bool in_step = false) {
  if (!h->learned.model) return fail(h, PCG_ERR_STATE, "no collision model: call pcg_set_collision_model");
  if (h->sp.size() > (size_t)kCollMaxSpecies) return fail(h, PCG_ERR_UNSUPPORTED, "too many species for collisions");
  CollParams p{};
  std::vector<CollSpecies> v;
  if (!collision_species(h, v, p))
    return fail(h, PCG_ERR_STATE, "collisions need species named 'electrons' and 'ions'");
  unsigned long long counts[2] = {0, 0};
  h->learned.aux = h->aux;
  h->learned.ev_fork = h->aux ? h->ev_fork : nullptr;
  h->learned.ev_join = h->aux ? h->ev_join : nullptr;
  const int lr = learned_step(h->g, v.data(), (int)v.size(), learned_phys(p), h->learned, counts, h->stream,
                              !in_step);
  if (lr == kLearnedTimeout) {
    h->halted = true;
    return fail(h, PCG_ERR_TIMEOUT, "learned collision step: a tensor-core wait timed out; the handle is halted");
  }
  if (lr != 0) return fail(h, PCG_ERR_CUDA, "learned collision step");
  h->launches += h->learned.launches;
  if (counts[1]) {  // the binary operator on the cells outside the training box
    p.pass = h->coll_pass++;
    p.only = h->learned.flag;
    p.only_value = 2;
    // few cells, often the fullest (a bunch's): a warp per cell from 32
    // particles on (the same collisions and results as a thread per cell)
    p.crowded = std::min(p.crowded, 32u);
    unsigned long long calls = 0;
    if (collide_p12(h->g, v.data(), (int)v.size(), p, h->coll, &calls, h->stream) != 0)
      return fail(h, PCG_ERR_CUDA, "collision fallback");
    h->launches += h->coll.launches;
  }
  if (learned_cells) *learned_cells = counts[0];
  if (fallback_cells) *fallback_cells = counts[1];
  return PCG_OK;
}

// The collision operator of pcg_step, between the push and the move.
int step_collide(pcg_handle* h) {
  if (h->collisions == PCG_COLLISIONS_BINARY) return run_collide(h, nullptr);
  if (h->collisions == PCG_COLLISIONS_LEARNED) return run_collide_learned(h, nullptr, nullptr, !is_f64(h));
  return PCG_OK;
}

// One step in the order of PiCoPiC's main loop (PiCoPiC.cpp:326-347 over
// SMB.cpp:1231-1322): beam injection, E, H, then per species the push, the
// collisions (SMB::advance_particles collides after the push and before the
// move), the move with reflection and binding, and the current.  Without
// collisions the push and the move are one kernel; with them the push runs
// first for every species, then the collision operator, then the move.
int fused_step(pcg_handle* h) {
  int rc;
  const int fixed = h->cfg.quirks == PCG_QUIRKS_FIXED;
  const bool collide = h->collisions != PCG_COLLISIONS_NONE;
  if ((rc = stage_inject(h)) != PCG_OK) return rc;
  uint64_t live = 0;
  for (Species& s : h->sp) live += s.n;
  if (is_f64(h)) {
    // E consumes J of the previous step, then clears it for this step's deposit.
    { TimerScope ts(h, PCG_TIMER_FIELD_E); launch_yee_e_f64(yee_args<double>(h, h->f64, h->sig64, 1), h->stream); }
    { TimerScope ts(h, PCG_TIMER_FIELD_H); launch_yee_h_f64(yee_args<double>(h, h->f64, h->sig64, 0), fixed, h->stream); }
    h->launches += 2;
    FieldsF64 f = fields64(h);
    if (collide) {
      {
        TimerScope ts(h, PCG_TIMER_PARTICLES);
        for (size_t t = 0; t < h->sp.size(); ++t) {
          launch_stage_f64(PCG_STAGE_PUSH, h->g, f, view64(h, h->sp[t]), (int)t, h->cfg.pusher, fixed,
                           h->d_status, h->stream);
          h->launches += h->sp[t].n ? 1 : 0;
        }
      }
      if ((rc = step_collide(h)) != PCG_OK) return rc;
    }
    {
      TimerScope ts(h, PCG_TIMER_PARTICLES);
      if (h->cfg.current == PCG_CURRENT_VB)
        CUDA_TRY(h, cudaMemsetAsync(h->reset, 0, sizeof(unsigned long long) * h->nodes, h->stream));
      for (size_t t = 0; t < h->sp.size(); ++t) {
        launch_advance_f64(h->g, f, view64(h, h->sp[t]), (int)t, h->cfg.pusher, fixed,
                           h->cfg.current, h->reset, h->d_status, h->stream, collide ? 0 : 1);
        h->launches += h->sp[t].n ? 1 : 0;
      }
    }
    {
      TimerScope ts(h, PCG_TIMER_DEPOSIT);
      for (size_t t = 0; t < h->sp.size(); ++t) {
        launch_deposit_f64(h->g, f, view64(h, h->sp[t]), (int)t, fixed, h->cfg.current, h->reset,
                           h->d_status, h->stream);
        h->launches += h->sp[t].n ? 1 : 0;
      }
    }
  } else {
    { TimerScope ts(h, PCG_TIMER_FIELD_E); f32_launch_yee_e(yee_args<float>(h, h->f32, h->sig32, 1), h->stream); }
    { TimerScope ts(h, PCG_TIMER_FIELD_H); f32_launch_yee_h(yee_args<float>(h, h->f32, h->sig32, 0), fixed, h->stream); }
    h->launches += 2;
    F32Step st;
    st.g = h->g;
    for (int c = 0; c < 12; ++c) st.fld[c] = h->f32[c];
    if (h->ext32) {  // the step gathers E + E_ext and H + H_ext
      f32_add_planes(h->push32, h->f32[0], h->ext32, 6 * h->f32_plane, h->stream);
      h->launches += 1;
      for (int c = 0; c < 6; ++c) st.fld[c] = h->push32 + c * h->f32_plane;
    }
    st.plane = (int)h->f32_plane;
    st.recip = h->recip32;
    st.pusher = h->cfg.pusher;
    st.current = h->cfg.current;
    st.fixed = fixed;
    st.status = h->d_status;
    st.tiles = h->tiles;
    st.sort_interval = h->sort_interval;
    st.target_blocks = h->target_blocks;
    st.min_split = h->min_split;
    const bool learned = h->collisions == PCG_COLLISIONS_LEARNED;
    if (collide) {
      {
        TimerScope ts(h, PCG_TIMER_PARTICLES);
        const bool fork = h->sp.size() >= 2 && h->aux;
        if (fork) {
          CUDA_TRY(h, cudaEventRecord(h->ev_fork, h->stream));
          CUDA_TRY(h, cudaStreamWaitEvent(h->aux, h->ev_fork, 0));
        }
        for (size_t t = 0; t < h->sp.size(); ++t) {
          Species& s = h->sp[t];
          const uint64_t k0 = s.f32.launches;
          f32_push_species(st, s.f32, s.n, s.charge, s.mass, s.beam ? 1 : 0, fork && (t & 1) ? h->aux : h->stream);
          h->launches += s.f32.launches - k0;
        }
        if (fork) {
          CUDA_TRY(h, cudaEventRecord(h->ev_join, h->aux));
          CUDA_TRY(h, cudaStreamWaitEvent(h->stream, h->ev_join, 0));
        }
      }
      if ((rc = step_collide(h)) != PCG_OK) return rc;
      st.pushed = 1;
      if (learned) {  // the move applies the learned transforms
        st.xform = h->learned.xform;
        st.xflag = h->learned.flag;
      }
    }
    TimerScope ts(h, PCG_TIMER_PARTICLES);
    // Species are independent until their currents meet in J (atomics), so
    // the odd-numbered ones run on a second stream: one species' last blocks
    // overlap the next one's first instead of the GPU draining between them
    // (the push of a step with collisions is split the same way).
    const bool fork = h->sp.size() >= 2 && h->aux;
    if (fork) {
      CUDA_TRY(h, cudaEventRecord(h->ev_fork, h->stream));
      CUDA_TRY(h, cudaStreamWaitEvent(h->aux, h->ev_fork, 0));
    }
    for (size_t t = 0; t < h->sp.size(); ++t) {
      Species& s = h->sp[t];
      const size_t n0 = s.n;
      const uint64_t k0 = s.f32.launches;
      cudaStream_t stream = fork && (t & 1) ? h->aux : h->stream;
      if (f32_step_species(st, s.f32, &s.n, s.charge, s.mass, s.beam ? 1 : 0, stream,
                           is_ion_list(s) ? 6 : 0) != 0)
        return fail(h, PCG_ERR_CUDA, "tile sort of species '" + s.name + "' failed");
      h->dead_dropped += n0 - s.n;  // a sort drops the species' dead slots
      h->launches += s.f32.launches - k0;
    }
    if (fork) {
      CUDA_TRY(h, cudaEventRecord(h->ev_join, h->aux));
      CUDA_TRY(h, cudaStreamWaitEvent(h->stream, h->ev_join, 0));
    }
  }
  h->t += h->cfg.dt;
  h->steps += 1;
  h->particle_steps += live;
  return PCG_OK;
}

}  // namespace

extern "C" {

int pcg_abi_version(void) { return PCG_ABI_VERSION; }

int pcg_create(const pcg_config* cfg, pcg_handle** out) {
  if (!cfg || !out) return PCG_ERR_ARG;
  *out = nullptr;
  if (cfg->nr < 2 || cfg->nz < 2 || cfg->nr > 32000 || cfg->nz > 32000 || !(cfg->radius > 0) ||
      !(cfg->longitude > 0) || !(cfg->dt > 0))
    return PCG_ERR_ARG;
  if (cfg->pusher < 0 || cfg->pusher > 4 || cfg->current < 0 || cfg->current > 1 ||
      cfg->precision < 0 || cfg->precision > 1 || cfg->quirks < 0 || cfg->quirks > 1)
    return PCG_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return PCG_ERR_CUDA;
  if (cfg->device < 0 || cfg->device >= ndev) return PCG_ERR_ARG;
  int prev_device = 0;
  if (cudaGetDevice(&prev_device) != cudaSuccess) return PCG_ERR_CUDA;
  if (cudaSetDevice(cfg->device) != cudaSuccess) return PCG_ERR_CUDA;
  struct Restore {  // the caller's device is current again on return
    int d;
    ~Restore() { cudaSetDevice(d); }
  } restore{prev_device};
  pcg_handle* h = new pcg_handle();
  h->cfg = *cfg;
  GridGeom& g = h->g;
  g.nr = cfg->nr; g.nz = cfg->nz; g.ld = cfg->nz + 4;
  g.R = cfg->radius; g.L = cfg->longitude;
  g.dr = cfg->radius / cfg->nr;  // Geometry ctor geometry.hpp:67-68
  g.dz = cfg->longitude / cfg->nz;
  g.dt = cfg->dt;
  g.pml_r = cfg->pml_size[2] != 0; g.pml_z0 = cfg->pml_size[1] != 0; g.pml_zl = cfg->pml_size[3] != 0;
  h->t = cfg->t_start;
  h->nodes = (size_t)(g.nr + 4) * (size_t)g.ld;
  h->tiles = f32_tile_grid(g);
  int rc = PCG_OK;
  auto bail = [&](int code) { pcg_destroy(h); return code; };
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(PCG_ERR_CUDA);
  if (cudaStreamCreateWithFlags(&h->copy, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_copied, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_staging_free, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_status, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_region, cudaEventDisableTiming) != cudaSuccess ||
      cudaMallocHost((void**)&h->h_status_lag, sizeof(DevStatus)) != cudaSuccess)
    return bail(PCG_ERR_CUDA);
  if (cfg->precision == PCG_PRECISION_F32 &&
      (cudaStreamCreateWithFlags(&h->aux, cudaStreamNonBlocking) != cudaSuccess ||
       cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
       cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming) != cudaSuccess))
    return bail(PCG_ERR_CUDA);
  if ((rc = dalloc(h, &h->d_status, 1)) != PCG_OK) return bail(rc);
  if (cudaMallocHost((void**)&h->h_status, sizeof(DevStatus)) != cudaSuccess) return bail(PCG_ERR_NOMEM);
  cudaMemsetAsync(h->d_status, 0, sizeof(DevStatus), h->stream);
  std::vector<double> sr, s0, sl;
  pml_profiles(*cfg, g, sr, s0, sl);
  if (is_f64(h)) {
    for (int c = 0; c < 12; ++c) {
      if ((rc = dalloc(h, &h->f64[c], h->nodes)) != PCG_OK) return bail(rc);
      cudaMemsetAsync(h->f64[c], 0, sizeof(double) * h->nodes, h->stream);
    }
    const std::vector<double>* prof[3] = {&sr, &s0, &sl};
    for (int c = 0; c < 3; ++c) {
      if ((rc = dalloc(h, &h->sig64[c], prof[c]->size())) != PCG_OK) return bail(rc);
      cudaMemcpyAsync(h->sig64[c], prof[c]->data(), sizeof(double) * prof[c]->size(),
                      cudaMemcpyHostToDevice, h->stream);
    }
    if ((rc = dalloc(h, &h->reset, h->nodes)) != PCG_OK) return bail(rc);
    cudaMemsetAsync(h->reset, 0, sizeof(unsigned long long) * h->nodes, h->stream);
  } else {
    // one allocation: a particle kernel reaches component c at base + c * plane
    h->f32_plane = (h->nodes + 63) / 64 * 64;
    if ((rc = dalloc(h, &h->f32[0], 12 * h->f32_plane)) != PCG_OK) return bail(rc);
    cudaMemsetAsync(h->f32[0], 0, sizeof(float) * 12 * h->f32_plane, h->stream);
    for (int c = 1; c < 12; ++c) h->f32[c] = h->f32[0] + c * h->f32_plane;
    // rows i = -2 .. nr+2: {1/(2i+1), 1/(2i+2), 1/(2i+3), 1/(2i+4)}, {1/i, 1/(i+1), 1/(i+1/2), 0},
    // each correctly rounded from double, 0 where the denominator is 0
    const int rows = h->g.nr + 5;
    std::vector<float4> rt(2 * (size_t)rows);
    auto inv = [](double d) { return d == 0.0 ? 0.f : (float)(1.0 / d); };
    for (int r = 0; r < rows; ++r) {
      const double i = r - 2;
      rt[2 * r] = make_float4(inv(2 * i + 1), inv(2 * i + 2), inv(2 * i + 3), inv(2 * i + 4));
      rt[2 * r + 1] = make_float4(inv(i), inv(i + 1), inv(i + 0.5), 0.f);
    }
    if ((rc = dalloc(h, &h->recip32, rt.size())) != PCG_OK) return bail(rc);
    cudaMemcpyAsync(h->recip32, rt.data(), sizeof(float4) * rt.size(), cudaMemcpyHostToDevice, h->stream);
    std::vector<float> prof[3];
    const std::vector<double>* src[3] = {&sr, &s0, &sl};
    for (int c = 0; c < 3; ++c) {
      prof[c].assign(src[c]->begin(), src[c]->end());
      if ((rc = dalloc(h, &h->sig32[c], prof[c].size())) != PCG_OK) return bail(rc);
      cudaMemcpyAsync(h->sig32[c], prof[c].data(), sizeof(float) * prof[c].size(),
                      cudaMemcpyHostToDevice, h->stream);
    }
  }
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return bail(PCG_ERR_CUDA);
  *out = h;
  return PCG_OK;
}

int pcg_destroy(pcg_handle* h) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h) return PCG_OK;
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (int c = 0; c < 12; ++c) cudaFree(h->f64[c]);
  cudaFree(h->f32[0]);
  cudaFree(h->recip32);
  cudaFree(h->diag);
  collide_free(h->coll);
  learned_free(h->learned);
  for (int c = 0; c < 3; ++c) { cudaFree(h->sig64[c]); cudaFree(h->sig32[c]); }
  cudaFree(h->ext64);
  cudaFree(h->ext32);
  cudaFree(h->push32);
  cudaFree(h->reset);
  cudaFree(h->scratch);
  cudaFree(h->region);
  cudaFree(h->region_out);
  cudaFree(h->staging);
  for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
  for (auto& u : h->ev_used) { cudaEventDestroy(u.second.first); cudaEventDestroy(u.second.second); }
  for (Species& s : h->sp) {
    void* arrs[] = {s.r, s.z, s.vr, s.vphi, s.vz, s.w, s.r_old, s.z_old, s.phi, s.phi_old, s.sn,
                    s.cell_r, s.cell_z};
    for (void* a : arrs) cudaFree(a);
    f32_free_species(s.f32);
    cudaFree(s.abs_map);
  }
  cudaFree(h->map_work);
  cudaFree(h->d_status);
  if (h->h_status) cudaFreeHost(h->h_status);
  if (h->aux) cudaStreamSynchronize(h->aux);
  if (h->copy) cudaStreamSynchronize(h->copy);
  if (h->copy) cudaStreamDestroy(h->copy);
  if (h->ev_copied) cudaEventDestroy(h->ev_copied);
  if (h->ev_staging_free) cudaEventDestroy(h->ev_staging_free);
  if (h->ev_status) cudaEventDestroy(h->ev_status);
  if (h->ev_region) cudaEventDestroy(h->ev_region);
  if (h->h_status_lag) cudaFreeHost(h->h_status_lag);
  if (h->h_count) cudaFreeHost(h->h_count);
  if (h->stream) cudaStreamDestroy(h->stream);
  if (h->aux) cudaStreamDestroy(h->aux);
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->ev_join) cudaEventDestroy(h->ev_join);
  delete h;
  return PCG_OK;
}

const char* pcg_last_error(const pcg_handle* h) { return h ? h->err.c_str() : "null handle"; }

static int add_common(pcg_handle* h, int id, const char* name, double charge_e, double mass_e,
                      size_t capacity, int* slot, Species** out) {
  if (!h || !slot) return PCG_ERR_ARG;
  if (h->started) return fail(h, PCG_ERR_STATE, "species must be added before particles are imported");
  if (!(mass_e > 0) || capacity == 0) return fail(h, PCG_ERR_ARG, "mass must be positive and capacity non-zero");
  if (h->sp.size() >= 255) return fail(h, PCG_ERR_ARG, "too many species");
  h->sp.emplace_back();
  Species& s = h->sp.back();
  s.id = id;
  s.name = name ? name : "";
  s.charge_e = charge_e; s.mass_e = mass_e;
  s.charge = charge_e * kElCharge;  // SpecieP ctor specieP.cpp:37-38
  s.mass = mass_e * kElMass;
  s.cap = capacity;
  int rc = alloc_species(h, s);
  if (rc != PCG_OK) { h->sp.pop_back(); return rc; }
  *slot = (int)h->sp.size() - 1;
  *out = &s;
  return PCG_OK;
}

int pcg_add_species(pcg_handle* h, int id, const char* name, double charge_e, double mass_e,
                    size_t capacity, int* slot) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  Species* s = nullptr;
  return add_common(h, id, name, charge_e, mass_e, capacity, slot, &s);
}

int pcg_add_beam(pcg_handle* h, int id, const char* name, double charge_e, double mass_e,
                 size_t capacity, unsigned macro_amount, double start_time, double bunch_radius,
                 double density, double bunches_amount, double bunch_length,
                 double bunches_distance, double velocity, int* slot) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!(velocity > 0) || !(bunch_length > 0) || !(bunch_radius > 0) || bunches_amount < 1)
    return fail(h, PCG_ERR_ARG, "beam velocity, length, radius and bunch count must be positive");
  Species* s = nullptr;
  int rc = add_common(h, id, name, charge_e, mass_e, capacity, slot, &s);
  if (rc != PCG_OK) return rc;
  // BeamP ctor (beamP.cpp:22-69) for a domain at the origin
  s->beam = true;
  s->macro_amount = macro_amount;
  s->radius = bunch_radius; s->density = density; s->velocity = velocity;
  s->start_time = start_time; s->bunches_amount = (unsigned)bunches_amount;
  s->bunch_length = bunch_length; s->bunches_distance = bunches_distance;
  s->finish_time = s->start_time + s->bunch_length / s->velocity * s->bunches_amount +
                   s->bunches_distance / s->velocity * (s->bunches_amount - 1);
  if (bunch_radius > (double)h->g.nr * h->g.dr) s->domain_radius = h->g.R;
  else if (bunch_radius > 0.0 * h->g.dr) s->domain_radius = bunch_radius - 0.0 * h->g.dr;
  else s->domain_radius = 0;
  double macro_normalizer = s->domain_radius / s->radius;
  s->bunch_macro_amount = (double)(s->macro_amount / s->bunches_amount) * macro_normalizer;
  s->macro_per_step = s->bunch_macro_amount * s->velocity * h->cfg.dt / s->bunch_length;
  return PCG_OK;
}

static int put_particles(pcg_handle* h, int slot, size_t n, const double* r, const double* z,
                         const double* vr, const double* vphi, const double* vz, const double* w,
                         bool append) {
  if (!h || slot < 0 || slot >= (int)h->sp.size()) return PCG_ERR_ARG;
  if (n && !(r && z && vr && vphi && vz && w)) return fail(h, PCG_ERR_ARG, "null particle array");
  Species& s = h->sp[slot];
  if (append && s.n + n > s.cap) {  // reclaim the dead slots first
    int rc = check_status(h);
    if (rc != PCG_OK) return rc;
    if (h->h_status->dead_slots > h->dead_dropped && (rc = compact(h)) != PCG_OK) return rc;
  }
  size_t n0 = append ? s.n : 0;
  if (n0 + n > s.cap) return fail(h, PCG_ERR_CAPACITY, "species '" + s.name + "' capacity exceeded");
  h->started = true;
  if (n) {
    if (h->staging_n < n) {  // grow the reusable staging buffer
      CUDA_TRY(h, cudaStreamSynchronize(h->stream));
      cudaFree(h->staging);
      h->staging = nullptr;
      h->staging_n = 0;
      int rc = dalloc(h, &h->staging, 6 * n);
      if (rc != PCG_OK) return rc;
      h->staging_n = n;
    }
    double* stage = h->staging;
    const double* src[6] = {r, z, vr, vphi, vz, w};
    // the copies wait for the last import's read of the staging buffer only,
    // and the import for the copies; the steps queued before run on
    CUDA_TRY(h, cudaStreamWaitEvent(h->copy, h->ev_staging_free, 0));
    for (int a = 0; a < 6; ++a)
      CUDA_TRY(h, cudaMemcpyAsync(stage + a * n, src[a], sizeof(double) * n, cudaMemcpyDefault, h->copy));
    CUDA_TRY(h, cudaEventRecord(h->ev_copied, h->copy));
    CUDA_TRY(h, cudaStreamWaitEvent(h->stream, h->ev_copied, 0));
    if (is_f64(h)) launch_import_f64(h->g, view64(h, s), n0, n, stage, h->stream);
    else f32_launch_import(h->g, s.f32, n0, n, stage, h->d_status, h->stream);
    CUDA_TRY(h, cudaEventRecord(h->ev_staging_free, h->stream));
    // the caller may reuse its host arrays once this call returns
    CUDA_TRY(h, cudaEventSynchronize(h->ev_copied));
  }
  s.n = n0 + n;
  return PCG_OK;
}

int pcg_import_species(pcg_handle* h, int slot, size_t n, const double* r, const double* z,
                       const double* vr, const double* vphi, const double* vz, const double* w) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  return put_particles(h, slot, n, r, z, vr, vphi, vz, w, false);
}

int pcg_append_species(pcg_handle* h, int slot, size_t n, const double* r, const double* z,
                       const double* vr, const double* vphi, const double* vz, const double* w) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  return put_particles(h, slot, n, r, z, vr, vphi, vz, w, true);
}

int pcg_count(pcg_handle* h, int slot, size_t* n) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || !n || slot < 0 || slot >= (int)h->sp.size()) return PCG_ERR_ARG;
  int rc = check_status(h);
  if (rc != PCG_OK) return rc;
  if (h->h_status->dead_slots > h->dead_dropped && (rc = compact(h)) != PCG_OK) return rc;
  *n = h->sp[slot].n;
  return PCG_OK;
}

int pcg_export_species(pcg_handle* h, int slot, size_t cap, double* r, double* z, double* vr,
                       double* vphi, double* vz, double* w, int32_t* cell_r, int32_t* cell_z,
                       size_t* n) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  size_t cnt = 0;
  int rc = pcg_count(h, slot, &cnt);
  if (rc != PCG_OK) return rc;
  if (n) *n = cnt;
  if (cap < cnt) return fail(h, PCG_ERR_CAPACITY, "export buffer too small");
  if (cnt == 0) return PCG_OK;
  Species& s = h->sp[slot];
  if (is_f64(h)) {
    double* dst[6] = {r, z, vr, vphi, vz, w};
    double* src[6] = {s.r, s.z, s.vr, s.vphi, s.vz, s.w};
    for (int a = 0; a < 6; ++a)
      if (dst[a]) CUDA_TRY(h, cudaMemcpyAsync(dst[a], src[a], sizeof(double) * cnt, cudaMemcpyDeviceToHost, h->stream));
    if (s.cell_r) {  // stage-by-stage mode keeps the bound cells (they may lag the positions)
      if (cell_r) CUDA_TRY(h, cudaMemcpyAsync(cell_r, s.cell_r, sizeof(int) * cnt, cudaMemcpyDeviceToHost, h->stream));
      if (cell_z) CUDA_TRY(h, cudaMemcpyAsync(cell_z, s.cell_z, sizeof(int) * cnt, cudaMemcpyDeviceToHost, h->stream));
      CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    } else {
      CUDA_TRY(h, cudaStreamSynchronize(h->stream));
      if ((cell_r || cell_z) && !(r && z)) return fail(h, PCG_ERR_ARG, "cells need r and z");
      for (size_t j = 0; cell_r && j < cnt; ++j) cell_r[j] = (int32_t)floor(r[j] / h->g.dr);
      for (size_t j = 0; cell_z && j < cnt; ++j) cell_z[j] = (int32_t)floor(z[j] / h->g.dz);
    }
  } else {
    if (f32_export(h->g, s.f32, cnt, r, z, vr, vphi, vz, w, cell_r, cell_z, h->stream) != 0)
      return fail(h, PCG_ERR_CUDA, "float export failed");
  }
  return PCG_OK;
}

int pcg_set_field(pcg_handle* h, int which, const double* src) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || !src || which < 0 || which >= 12) return PCG_ERR_ARG;
  if (is_f64(h)) {
    CUDA_TRY(h, cudaMemcpyAsync(h->f64[which], src, sizeof(double) * h->nodes, cudaMemcpyHostToDevice, h->stream));
  } else {
    std::vector<float> tmp(src, src + h->nodes);
    CUDA_TRY(h, cudaMemcpyAsync(h->f32[which], tmp.data(), sizeof(float) * h->nodes, cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  }
  return PCG_OK;
}

int pcg_export_field(pcg_handle* h, int which, double* dst) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || !dst || which < 0 || which >= 12) return PCG_ERR_ARG;
  int rc = check_status(h);
  if (rc != PCG_OK) return rc;
  if (is_f64(h)) {
    CUDA_TRY(h, cudaMemcpyAsync(dst, h->f64[which], sizeof(double) * h->nodes, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  } else {
    std::vector<float> tmp(h->nodes);
    CUDA_TRY(h, cudaMemcpyAsync(tmp.data(), h->f32[which], sizeof(float) * h->nodes, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    for (size_t p = 0; p < h->nodes; ++p) dst[p] = tmp[p];
  }
  (void)kFieldNames;
  return PCG_OK;
}

namespace {

// Columns [c0, c1) of every row of a field grid to or from the host.
int field_columns(pcg_handle* h, int which, int c0, int c1, double* host, bool set) {
  if (!h || !host || which < 0 || which >= 12) return PCG_ERR_ARG;
  const int ld = h->g.ld, rows = h->g.nr + 4;
  if (c0 < 0 || c1 > ld || c0 >= c1) return fail(h, PCG_ERR_ARG, "field columns out of range");
  const size_t w = (size_t)(c1 - c0);
  if (!set) {
    int rc = check_status(h);
    if (rc != PCG_OK) return rc;
  }
  if (is_f64(h)) {
    double* dev = h->f64[which] + c0;
    if (set)
      CUDA_TRY(h, cudaMemcpy2DAsync(dev, sizeof(double) * ld, host, sizeof(double) * w, sizeof(double) * w, rows,
                                    cudaMemcpyDefault, h->stream));
    else
      CUDA_TRY(h, cudaMemcpy2DAsync(host, sizeof(double) * w, dev, sizeof(double) * ld, sizeof(double) * w, rows,
                                    cudaMemcpyDefault, h->stream));
    // a read, or a write from device memory the caller may reuse on return
    if (!set || device_memory(host)) CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  } else if (device_memory(host)) {  // doubles in device memory: converted by a kernel
    region_columns_f32(h->f32[which], ld, c0, (int)w, rows, host, set, h->stream);
    CUDA_TRY(h, cudaGetLastError());
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  } else {
    float* dev = h->f32[which] + c0;
    std::vector<float> tmp(w * rows);
    if (set) {
      for (size_t p = 0; p < tmp.size(); ++p) tmp[p] = (float)host[p];
      CUDA_TRY(h, cudaMemcpy2DAsync(dev, sizeof(float) * ld, tmp.data(), sizeof(float) * w, sizeof(float) * w, rows,
                                    cudaMemcpyHostToDevice, h->stream));
      CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    } else {
      CUDA_TRY(h, cudaMemcpy2DAsync(tmp.data(), sizeof(float) * w, dev, sizeof(float) * ld, sizeof(float) * w, rows,
                                    cudaMemcpyDeviceToHost, h->stream));
      CUDA_TRY(h, cudaStreamSynchronize(h->stream));
      for (size_t p = 0; p < tmp.size(); ++p) host[p] = tmp[p];
    }
  }
  return PCG_OK;
}

// The species' layout view for the band kernels (one of the two is set).
void region_views(pcg_handle* h, Species& s, SpeciesF64* v64, const SpeciesF32Buffers** b32,
                  const SpeciesF64** s64) {
  if (is_f64(h)) {
    *v64 = view64(h, s);
    *s64 = v64;
    *b32 = nullptr;
  } else {
    *s64 = nullptr;
    *b32 = &s.f32;
  }
}

}  // namespace

int pcg_get_field_columns(pcg_handle* h, int which, int c0, int c1, double* dst) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  return field_columns(h, which, c0, c1, dst, false);
}

int pcg_set_field_columns(pcg_handle* h, int which, int c0, int c1, const double* src) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  return field_columns(h, which, c0, c1, const_cast<double*>(src), true);
}

namespace {

// One band of a selection: the live slots of species `slot` with lo <= z < hi.
struct Band {
  int slot;
  double lo, hi;
};

// Selects every band (one pass over its species' slots each), then waits
// once for the counts and the status of the work queued before: m[b] and
// the indices sel[b] (the handle's selection scratch, valid until the next
// selection).
int select_bands(pcg_handle* h, const Band* bands, int nb, unsigned* m, const unsigned** sel) {
  size_t tmp = 0, idx = 0;
  for (int b = 0; b < nb; ++b) {
    const size_t ns = h->sp[bands[b].slot].n;
    if (ns > 0x7fffffffu) return fail(h, PCG_ERR_UNSUPPORTED, "a band selection of more than 2^31 slots");
    tmp = std::max(tmp, region_select_bytes(ns));
    idx += (ns + 63) & ~(size_t)63;
  }
  const size_t o_cnt = 0, o_idx = 256 + (((size_t)nb * sizeof(unsigned) + 255) & ~(size_t)255),
               o_tmp = o_idx + ((4 * idx + 255) & ~(size_t)255), bytes = o_tmp + tmp;
  int rc;
  if (bytes > h->region_bytes) {  // grown with headroom: species counts creep up between exchanges
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    cudaFree(h->region);
    h->region = nullptr;
    h->region_bytes = 0;
    const size_t grown = bytes + bytes / 4;
    if ((rc = dalloc(h, &h->region, grown)) != PCG_OK) return rc;
    h->region_bytes = grown;
  }
  if (nb > h->h_count_n) {
    if (h->h_count) cudaFreeHost(h->h_count);
    h->h_count = nullptr;
    h->h_count_n = 0;
    if (cudaMallocHost((void**)&h->h_count, sizeof(unsigned) * nb) != cudaSuccess)
      return fail(h, PCG_ERR_NOMEM, "pinned band counts");
    h->h_count_n = nb;
  }
  unsigned* cnt = (unsigned*)(h->region + o_cnt);
  unsigned* out = (unsigned*)(h->region + o_idx);
  for (int b = 0; b < nb; ++b) {
    Species& s = h->sp[bands[b].slot];
    SpeciesF64 v64{};
    const SpeciesF32Buffers* b32;
    const SpeciesF64* s64;
    region_views(h, s, &v64, &b32, &s64);
    if (region_select(h->g, b32, s64, s.n, bands[b].lo, bands[b].hi, h->region + o_tmp, tmp, out, cnt + b,
                      h->stream) != 0)
      return fail(h, PCG_ERR_CUDA, "band selection");
    sel[b] = out;
    out += (s.n + 63) & ~(size_t)63;
  }
  // the counts and the status of the steps queued before, in one wait
  CUDA_TRY(h, cudaMemcpyAsync(h->h_count, cnt, sizeof(unsigned) * nb, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaMemcpyAsync(h->h_status, h->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  CUDA_TRY(h, cudaGetLastError());
  if ((rc = status_code(h, h->h_status)) != PCG_OK) return rc;
  for (int b = 0; b < nb; ++b) m[b] = h->h_count[b];
  return PCG_OK;
}

// Room for `total` gathered particles (6 doubles each) in region_out.
int region_room(pcg_handle* h, size_t total) {
  if (h->region_out_n >= total) return PCG_OK;
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  cudaFree(h->region_out);
  h->region_out = nullptr;
  h->region_out_n = 0;
  const size_t grown = total + total / 4 + 1024;
  int rc = dalloc(h, &h->region_out, 6 * grown);
  if (rc != PCG_OK) return rc;
  h->region_out_n = grown;
  return PCG_OK;
}

// The m selected particles as 6 x m doubles (r, z - zshift, v_r, v_phi,
// v_z, w) at out, queued on the handle's stream.
void gather_band(pcg_handle* h, Species& s, const unsigned* sel, unsigned m, double zshift, double* out) {
  if (m == 0) return;
  SpeciesF64 v64{};
  const SpeciesF32Buffers* b32;
  const SpeciesF64* s64;
  region_views(h, s, &v64, &b32, &s64);
  region_gather(h->g, b32, s64, sel, m, zshift, out, h->stream);
}

// Appends (or, append = 0, imports in place of the species' particles) m
// particles that lie as 6 x m doubles in src's device memory at data, on
// dst's stream after src's ev_region; src's later work waits for the copy.
int import_band(pcg_handle* src, const double* data, unsigned m, pcg_handle* dst, int dst_slot, int append) {
  DeviceScope on_dst(dst->cfg.device);
  Species& d = dst->sp[dst_slot];
  int rc;
  if (append && d.n + m > d.cap) {  // reclaim the dead slots first
    if ((rc = check_status(dst)) != PCG_OK) return rc;
    if (dst->h_status->dead_slots > dst->dead_dropped && (rc = compact(dst)) != PCG_OK) return rc;
  }
  const size_t n0 = append ? d.n : 0;
  if (n0 + m > d.cap) return fail(dst, PCG_ERR_CAPACITY, "species '" + d.name + "' capacity exceeded");
  dst->started = true;
  if (m) {
    if (dst->staging_n < m) {
      CUDA_TRY(dst, cudaStreamSynchronize(dst->stream));
      CUDA_TRY(dst, cudaStreamSynchronize(dst->copy));
      cudaFree(dst->staging);
      dst->staging = nullptr;
      dst->staging_n = 0;
      const size_t grown = (size_t)m + m / 4 + 1024;
      if ((rc = dalloc(dst, &dst->staging, 6 * grown)) != PCG_OK) return rc;
      dst->staging_n = grown;
    }
    CUDA_TRY(dst, cudaStreamWaitEvent(dst->stream, src->ev_region, 0));
    // the staging buffer's last host upload has landed (put_particles waits for it)
    const size_t bytes = sizeof(double) * 6 * (size_t)m;
    if (src->cfg.device == dst->cfg.device)
      CUDA_TRY(dst, cudaMemcpyAsync(dst->staging, data, bytes, cudaMemcpyDeviceToDevice, dst->stream));
    else
      CUDA_TRY(dst, cudaMemcpyPeerAsync(dst->staging, dst->cfg.device, data, src->cfg.device, bytes, dst->stream));
  }
  // a replacement with no particles still resets the species (ids, tile grouping)
  if (m || !append) {
    if (is_f64(dst)) launch_import_f64(dst->g, view64(dst, d), n0, m, dst->staging, dst->stream);
    else f32_launch_import(dst->g, d.f32, n0, m, dst->staging, dst->d_status, dst->stream);
  }
  d.n = n0 + m;
  CUDA_TRY(dst, cudaEventRecord(dst->ev_staging_free, dst->stream));
  CUDA_TRY(dst, cudaEventRecord(dst->ev_region, dst->stream));
  CUDA_TRY(dst, cudaGetLastError());
  DeviceScope on_src(src->cfg.device);
  CUDA_TRY(src, cudaStreamWaitEvent(src->stream, dst->ev_region, 0));  // region_out is read
  return PCG_OK;
}

}  // namespace

int pcg_export_species_range(pcg_handle* h, int slot, double lo, double hi, size_t cap, double* r,
                             double* z, double* vr, double* vphi, double* vz, double* w, size_t* n) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || !n || slot < 0 || slot >= (int)h->sp.size()) return PCG_ERR_ARG;
  if (std::isnan(lo) || std::isnan(hi)) return fail(h, PCG_ERR_ARG, "NaN band limit");
  *n = 0;
  Species& s = h->sp[slot];
  const Band band{slot, lo, hi};
  unsigned m = 0;
  const unsigned* sel = nullptr;
  int rc = select_bands(h, &band, 1, &m, &sel);
  if (rc != PCG_OK) return rc;
  *n = m;
  if (cap < m) return fail(h, PCG_ERR_CAPACITY, "export buffer too small");
  if (m == 0) return PCG_OK;
  if ((rc = region_room(h, m)) != PCG_OK) return rc;
  gather_band(h, s, sel, m, 0.0, h->region_out);
  CUDA_TRY(h, cudaGetLastError());
  double* dst[6] = {r, z, vr, vphi, vz, w};
  for (int a = 0; a < 6; ++a)
    if (dst[a])
      CUDA_TRY(h, cudaMemcpyAsync(dst[a], h->region_out + (size_t)a * m, sizeof(double) * m, cudaMemcpyDefault,
                                  h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return PCG_OK;
}

int pcg_transfer_species_bands(pcg_handle* src, int nbands, const pcg_band* bands, size_t* counts) {
  if (!src || nbands < 0 || (nbands && !bands)) return PCG_ERR_ARG;
  for (int b = 0; b < nbands; ++b) {
    const pcg_band& q = bands[b];
    if (q.slot < 0 || q.slot >= (int)src->sp.size() || !q.dst || q.dst == src || q.dst_slot < 0 ||
        q.dst_slot >= (int)q.dst->sp.size())
      return fail(src, PCG_ERR_ARG, "band " + std::to_string(b) + ": bad species slot or destination");
    if (std::isnan(q.lo) || std::isnan(q.hi) || !std::isfinite(q.shift))
      return fail(src, PCG_ERR_ARG, "band " + std::to_string(b) + ": bad limits or shift");
  }
  if (nbands == 0) return PCG_OK;
  std::vector<Band> sb(nbands);
  for (int b = 0; b < nbands; ++b) sb[b] = Band{bands[b].slot, bands[b].lo, bands[b].hi};
  std::vector<unsigned> m(nbands);
  std::vector<const unsigned*> sel(nbands);
  std::vector<size_t> off(nbands + 1, 0);
  int rc;
  {  // select all bands (one wait) and gather them on the source's GPU
    DeviceScope on_src(src->cfg.device);
    if ((rc = select_bands(src, sb.data(), nbands, m.data(), sel.data())) != PCG_OK) return rc;
    for (int b = 0; b < nbands; ++b) off[b + 1] = off[b] + m[b];
    if ((rc = region_room(src, off[nbands])) != PCG_OK) return rc;
    for (int b = 0; b < nbands; ++b)
      gather_band(src, src->sp[bands[b].slot], sel[b], m[b], bands[b].shift, src->region_out + 6 * off[b]);
    CUDA_TRY(src, cudaGetLastError());
    CUDA_TRY(src, cudaEventRecord(src->ev_region, src->stream));
  }
  for (int b = 0; b < nbands; ++b) {  // copy and import on each destination's GPU, in band order
    if ((rc = import_band(src, src->region_out + 6 * off[b], m[b], bands[b].dst, bands[b].dst_slot,
                          bands[b].append)) != PCG_OK)
      return rc;
    if (counts) counts[b] = m[b];
  }
  return PCG_OK;
}

int pcg_transfer_species_range(pcg_handle* src, int slot, double lo, double hi, double shift, pcg_handle* dst,
                               int dst_slot, int append, size_t* n) {
  if (!n) return PCG_ERR_ARG;
  *n = 0;
  const pcg_band band{slot, lo, hi, shift, dst, dst_slot, append};
  return pcg_transfer_species_bands(src, 1, &band, n);
}

int pcg_copy_field_columns(pcg_handle* src, int which, int c0, int c1, pcg_handle* dst, int g0) {
  if (!src || !dst || which < PCG_FIELD_ALL || which >= 12) return PCG_ERR_ARG;
  if (src->cfg.precision != dst->cfg.precision || src->g.nr != dst->g.nr)
    return fail(dst, PCG_ERR_ARG, "field columns between handles of another precision or radial size");
  if (c0 < 0 || c1 > src->g.ld || c0 >= c1 || g0 < 0 || g0 + (c1 - c0) > dst->g.ld)
    return fail(dst, PCG_ERR_ARG, "field columns out of range");
  {
    DeviceScope on_src(src->cfg.device);
    CUDA_TRY(src, cudaEventRecord(src->ev_region, src->stream));
  }
  {
    DeviceScope on_dst(dst->cfg.device);
    CUDA_TRY(dst, cudaStreamWaitEvent(dst->stream, src->ev_region, 0));
    const size_t es = is_f64(dst) ? sizeof(double) : sizeof(float);
    const size_t w = (size_t)(c1 - c0), rows = (size_t)dst->g.nr + 4;
    const int f0 = which == PCG_FIELD_ALL ? 0 : which, f1 = which == PCG_FIELD_ALL ? 12 : which + 1;
    for (int f = f0; f < f1; ++f) {
      char* d = is_f64(dst) ? (char*)(dst->f64[f] + g0) : (char*)(dst->f32[f] + g0);
      const char* s = is_f64(src) ? (const char*)(src->f64[f] + c0) : (const char*)(src->f32[f] + c0);
      if (src->cfg.device == dst->cfg.device) {
        CUDA_TRY(dst, cudaMemcpy2DAsync(d, es * dst->g.ld, s, es * src->g.ld, es * w, rows, cudaMemcpyDeviceToDevice,
                                        dst->stream));
      } else {
        cudaMemcpy3DPeerParms p{};
        p.srcPtr = make_cudaPitchedPtr(const_cast<char*>(s), es * src->g.ld, es * w, rows);
        p.srcDevice = src->cfg.device;
        p.dstPtr = make_cudaPitchedPtr(d, es * dst->g.ld, es * w, rows);
        p.dstDevice = dst->cfg.device;
        p.extent = make_cudaExtent(es * w, rows, 1);
        CUDA_TRY(dst, cudaMemcpy3DPeerAsync(&p, dst->stream));
      }
    }
    CUDA_TRY(dst, cudaEventRecord(dst->ev_region, dst->stream));
  }
  {
    DeviceScope on_src(src->cfg.device);
    CUDA_TRY(src, cudaStreamWaitEvent(src->stream, dst->ev_region, 0));
  }
  return PCG_OK;
}

int pcg_keep_species_range(pcg_handle* h, int slot, double lo, double hi) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || slot < 0 || slot >= (int)h->sp.size()) return PCG_ERR_ARG;
  if (std::isnan(lo) || std::isnan(hi)) return fail(h, PCG_ERR_ARG, "NaN band limit");
  Species& s = h->sp[slot];
  SpeciesF64 v64{};
  const SpeciesF32Buffers* b32;
  const SpeciesF64* s64;
  region_views(h, s, &v64, &b32, &s64);
  region_keep(h->g, b32, s64, s.n, lo, hi, h->d_status, h->stream);
  CUDA_TRY(h, cudaGetLastError());
  return PCG_OK;
}

namespace {
// A device array of node values for the diagnostics, allocated on first use.
int diag_buffer(pcg_handle* h, double** out) {
  if (!h->diag) {
    int rc = dalloc(h, &h->diag, h->nodes);
    if (rc != PCG_OK) return rc;
  }
  *out = h->diag;
  return PCG_OK;
}
}  // namespace

int pcg_node_charge(pcg_handle* h, double* q) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || !q) return PCG_ERR_ARG;
  int rc = check_status(h);
  if (rc != PCG_OK) return rc;
  double* d = nullptr;
  if ((rc = diag_buffer(h, &d)) != PCG_OK) return rc;
  CUDA_TRY(h, cudaMemsetAsync(d, 0, sizeof(double) * h->nodes, h->stream));
  for (Species& s : h->sp) {
    const int e = is_f64(h) ? diag_node_charge_f64(h->g, s.r, s.z, s.w, s.n, s.charge, d, h->stream)
                            : diag_node_charge_f32(h->g, s.f32, s.n, s.charge, d, h->stream);
    if (e != 0) return fail(h, PCG_ERR_CUDA, "node charge");
  }
  CUDA_TRY(h, cudaMemcpyAsync(q, d, sizeof(double) * h->nodes, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return PCG_OK;
}

int pcg_divergence(pcg_handle* h, int which, double* out) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || !out || (which != PCG_FIELD_E_R && which != PCG_FIELD_J_R)) return PCG_ERR_ARG;
  int rc = check_status(h);
  if (rc != PCG_OK) return rc;
  double* d = nullptr;
  if ((rc = diag_buffer(h, &d)) != PCG_OK) return rc;
  const int zc = which + 2;  // the z component of the same field
  const int e = is_f64(h) ? diag_divergence(h->g, h->f64[which], h->f64[zc], 1, d, h->stream)
                          : diag_divergence(h->g, h->f32[which], h->f32[zc], 0, d, h->stream);
  if (e != 0) return fail(h, PCG_ERR_CUDA, "divergence");
  CUDA_TRY(h, cudaMemcpyAsync(out, d, sizeof(double) * h->nodes, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return PCG_OK;
}


int pcg_collide(pcg_handle* h, unsigned long long* pair_calls) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h) return PCG_ERR_ARG;
  int rc = check_status(h);
  if (rc != PCG_OK) return rc;
  if ((rc = run_collide(h, pair_calls)) != PCG_OK) return rc;
  return check_status(h);
}

int pcg_collide_expectation(pcg_handle* h, double* out) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || !out) return PCG_ERR_ARG;
  int rc = check_status(h);
  if (rc != PCG_OK) return rc;
  if (h->sp.size() > (size_t)kCollMaxSpecies) return fail(h, PCG_ERR_UNSUPPORTED, "too many species for collisions");
  CollParams p{};
  std::vector<CollSpecies> v;
  if (!collision_species(h, v, p))
    return fail(h, PCG_ERR_STATE, "collisions need species named 'electrons' and 'ions'");
  const size_t cells = (size_t)h->g.nr * h->g.nz;
  double* d = nullptr;
  if (cudaMalloc((void**)&d, cells * 12 * sizeof(double)) != cudaSuccess) return fail(h, PCG_ERR_NOMEM, "expectation");
  cudaMemsetAsync(d, 0, cells * 12 * sizeof(double), h->stream);
  p.pass = h->coll_pass++;
  p.expect = d;
  unsigned long long calls = 0;
  int e = collide_p12(h->g, v.data(), (int)v.size(), p, h->coll, &calls, h->stream);
  if (e == 0 && (cudaMemcpyAsync(out, d, cells * 12 * sizeof(double), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
                 cudaStreamSynchronize(h->stream) != cudaSuccess))
    e = -1;
  cudaFree(d);
  return e == 0 ? check_status(h) : fail(h, PCG_ERR_CUDA, "expectation pass");
}

int pcg_set_collision_model(pcg_handle* h, const float* params, const float* norm) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || !params || !norm) return PCG_ERR_ARG;
  if (learned_set_model(h->learned, params, norm, h->stream) != 0) return fail(h, PCG_ERR_NOMEM, "collision model");
  return PCG_OK;
}

int pcg_collide_learned(pcg_handle* h, unsigned long long* learned_cells, unsigned long long* fallback_cells) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h) return PCG_ERR_ARG;
  if (h->halted) return fail(h, PCG_ERR_TIMEOUT, "halted after a tensor-core time-out");
  int rc = check_status(h);
  if (rc != PCG_OK) return rc;
  if ((rc = run_collide_learned(h, learned_cells, fallback_cells)) != PCG_OK) return rc;
  return check_status(h);
}

// ExternalFields (externalFields.cpp:22-95, 298-348, 351-436): the profile
// codes 0 none, 1 const_r, 2 const_phi, 3 const_z, 4 linerad_r, 5 linerad_z.
int extf_code(const char* name) {
  static const char* names[6] = {"none", "const_r", "const_phi", "const_z", "linerad_r", "linerad_z"};
  if (!name) return 0;
  for (int c = 0; c < 6; ++c)
    if (!strcmp(name, names[c])) return c;
  return -1;
}

int pcg_set_external_fields(pcg_handle* h, const char* electric, const double* e_params, int n_e,
                            const char* magnetic, const double* m_params, int n_m) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h) return PCG_ERR_ARG;
  const bool fixed = h->cfg.quirks == PCG_QUIRKS_FIXED;
  int ec = extf_code(electric), mc = extf_code(magnetic);
  if (mc < 0) return fail(h, PCG_ERR_ARG, std::string("unknown magnetic field profile ") + magnetic);
  if (fixed && ec < 0) return fail(h, PCG_ERR_ARG, std::string("unknown electric field profile ") + electric);
  if (!fixed) ec = 0;  // the reference's electric name test never selects a profile that sets a field
  if (!fixed && mc != 3) mc = 0;  // of the magnetic profiles only const_z sets one
  if (ec >= 4 || mc >= 4) return fail(h, PCG_ERR_UNSUPPORTED, "linerad external field profiles are not defined");
  if ((ec && (!e_params || n_e < 1)) || (mc && (!m_params || n_m < 1)))
    return fail(h, PCG_ERR_ARG, "an external field profile needs its amplitude in params[0]");
  int rc;
  if (!ec && !mc) {  // no external fields
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    cudaFree(h->ext64); cudaFree(h->ext32); cudaFree(h->push32);
    h->ext64 = nullptr; h->ext32 = nullptr; h->push32 = nullptr;
    return PCG_OK;
  }
  // component c of E (0..2) or H (3..5) = amplitude on 1 <= i < nr-1, 1 <= k < nz-1
  const size_t nodes = h->nodes;
  std::vector<double> host(6 * nodes, 0.0);
  const int comp[2] = {ec ? ec - 1 : -1, mc ? 3 + mc - 1 : -1};
  const double amp[2] = {ec ? e_params[0] : 0.0, mc ? m_params[0] : 0.0};
  for (int f = 0; f < 2; ++f) {
    if (comp[f] < 0) continue;
    double* plane = host.data() + (size_t)comp[f] * nodes;
    for (int i = 1; i < h->g.nr - 1; ++i)
      for (int k = 1; k < h->g.nz - 1; ++k) plane[(size_t)(i + 2) * h->g.ld + (k + 2)] = amp[f];
  }
  if (is_f64(h)) {
    if (!h->ext64 && (rc = dalloc(h, &h->ext64, 6 * nodes)) != PCG_OK) return rc;
    CUDA_TRY(h, cudaMemcpyAsync(h->ext64, host.data(), 6 * nodes * sizeof(double), cudaMemcpyHostToDevice,
                                h->stream));
  } else {
    std::vector<float> hf(6 * h->f32_plane, 0.f);
    for (int c = 0; c < 6; ++c)
      for (size_t q = 0; q < nodes; ++q) hf[c * h->f32_plane + q] = (float)host[c * nodes + q];
    if (!h->ext32 && (rc = dalloc(h, &h->ext32, 6 * h->f32_plane)) != PCG_OK) return rc;
    if (!h->push32 && (rc = dalloc(h, &h->push32, 6 * h->f32_plane)) != PCG_OK) return rc;
    CUDA_TRY(h, cudaMemcpyAsync(h->ext32, hf.data(), hf.size() * sizeof(float), cudaMemcpyHostToDevice,
                                h->stream));
  }
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));  // the host arrays go out of scope
  return PCG_OK;
}

int pcg_set_collision_crowding(pcg_handle* h, unsigned threshold) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h) return PCG_ERR_ARG;
  h->coll_crowded = threshold;
  return PCG_OK;
}

int pcg_set_collision_scheme(pcg_handle* h, int scheme) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || (scheme != PCG_COLLIDE_P12 && scheme != PCG_COLLIDE_TA77S && scheme != PCG_COLLIDE_SK98))
    return PCG_ERR_ARG;
  h->coll_scheme = scheme;
  return PCG_OK;
}

int pcg_set_collisions(pcg_handle* h, int mode) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || mode < PCG_COLLISIONS_NONE || mode > PCG_COLLISIONS_LEARNED) return PCG_ERR_ARG;
  if (mode == PCG_COLLISIONS_LEARNED && !h->learned.model)
    return fail(h, PCG_ERR_STATE, "no collision model: call pcg_set_collision_model");
  h->collisions = mode;
  return PCG_OK;
}

int pcg_set_tiling(pcg_handle* h, int sort_interval, int target_blocks, int min_split) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || sort_interval < 0 || target_blocks < 0 || min_split < 0) return PCG_ERR_ARG;
  if (sort_interval) h->sort_interval = sort_interval;
  if (target_blocks) h->target_blocks = (unsigned)target_blocks;
  if (min_split) h->min_split = (unsigned)min_split;
  for (Species& s : h->sp) s.f32.steps_since_sort = 1 << 30;  // the next step sorts with these
  return PCG_OK;
}

int pcg_tile_sort(pcg_handle* h, int slot, unsigned* counts, unsigned long long* misplaced) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || !counts || !misplaced || slot < 0 || slot >= (int)h->sp.size()) return PCG_ERR_ARG;
  if (is_f64(h)) return fail(h, PCG_ERR_UNSUPPORTED, "the tile sort belongs to the float layout");
  int rc = check_status(h);
  if (rc != PCG_OK) return rc;
  Species& s = h->sp[slot];
  const size_t cells = (size_t)h->g.nr * h->g.nz;
  unsigned* dc = nullptr;
  unsigned long long* dm = nullptr;
  if ((rc = dalloc(h, &dc, cells)) != PCG_OK) return rc;
  if ((rc = dalloc(h, &dm, 1)) != PCG_OK) { cudaFree(dc); return rc; }
  const size_t n0 = s.n;
  const uint64_t k0 = s.f32.launches;
  if (f32_tile_check(h->tiles, h->target_blocks, h->min_split, h->g.nr, h->g.nz, s.f32, &s.n, dc, dm,
                     h->stream) == 0) {
    h->dead_dropped += n0 - s.n;
    h->launches += s.f32.launches - k0;
    cudaMemcpyAsync(counts, dc, cells * sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream);
    cudaMemcpyAsync(misplaced, dm, sizeof(unsigned long long), cudaMemcpyDeviceToHost, h->stream);
    rc = cudaStreamSynchronize(h->stream) == cudaSuccess ? PCG_OK : fail(h, PCG_ERR_CUDA, "tile sort");
  } else {
    rc = fail(h, PCG_ERR_CUDA, "tile sort");
  }
  cudaFree(dc);
  cudaFree(dm);
  return rc;
}

int pcg_species_map(pcg_handle* h, int slot, int which, double* out) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || !out || slot < 0 || slot >= (int)h->sp.size() || which < PCG_MAP_DENSITY || which > PCG_MAP_MOMENTUM)
    return PCG_ERR_ARG;
  int rc = check_status(h);
  if (rc != PCG_OK) return rc;
  Species& s = h->sp[slot];
  const size_t plane = (size_t)(h->g.nr + 4) * h->g.ld;
  if (!h->map_work && (rc = dalloc(h, &h->map_work, 7 * plane)) != PCG_OK) return rc;
  if (!s.abs_map) {
    if ((rc = dalloc(h, &s.abs_map, plane)) != PCG_OK) return rc;
    CUDA_TRY(h, cudaMemsetAsync(s.abs_map, 0, plane * sizeof(double), h->stream));
  }
  MapSpecies m;
  m.n = s.n;
  m.mass = s.mass;
  if (is_f64(h)) {
    m.r = s.r; m.z = s.z; m.vr = s.vr; m.vphi = s.vphi; m.vz = s.vz; m.w = s.w;
  } else {
    m.cell = s.f32.cell; m.off_r = s.f32.off_r; m.off_z = s.f32.off_z;
    m.vr32 = s.f32.vr; m.vphi32 = s.f32.vphi; m.vz32 = s.f32.vz; m.w32 = s.f32.w;
  }
  double* dev_out = h->map_work + 4 * plane;
  if (species_map(h->g, m, which, h->cfg.quirks == PCG_QUIRKS_FIXED, s.abs_map, h->map_work, dev_out,
                  h->stream) != 0)
    return fail(h, PCG_ERR_CUDA, "species map");
  h->launches += 2;
  const size_t count = (which == PCG_MAP_MOMENTUM ? 3 : 1) * plane;
  CUDA_TRY(h, cudaMemcpyAsync(out, dev_out, count * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return PCG_OK;
}

int pcg_cell_moments(pcg_handle* h, double* out) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || !out) return PCG_ERR_ARG;
  int rc = check_status(h);
  if (rc != PCG_OK) return rc;
  CollParams p{};
  std::vector<CollSpecies> v;
  collision_species(h, v, p);
  if (learned_moments(h->g, v.data(), (int)v.size(), h->learned, h->stream) != 0)
    return fail(h, PCG_ERR_CUDA, "cell moments");
  CUDA_TRY(h, cudaMemcpyAsync(out, h->learned.mom, h->learned.cells * kMomWords * sizeof(double),
                              cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return PCG_OK;
}

int pcg_cell_features(pcg_handle* h, float* x, double* scale) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || !x || !scale) return PCG_ERR_ARG;
  int rc = check_status(h);
  if (rc != PCG_OK) return rc;
  CollParams p{};
  std::vector<CollSpecies> v;
  if (!collision_species(h, v, p))
    return fail(h, PCG_ERR_STATE, "collisions need species named 'electrons' and 'ions'");
  const size_t cells = (size_t)h->g.nr * h->g.nz;
  float* dx = nullptr;
  double* ds = nullptr;
  if (cudaMalloc((void**)&dx, cells * kFeatures * sizeof(float)) != cudaSuccess ||
      cudaMalloc((void**)&ds, cells * sizeof(double)) != cudaSuccess) {
    cudaFree(dx);
    return fail(h, PCG_ERR_NOMEM, "feature export");
  }
  int e = learned_features(h->g, v.data(), (int)v.size(), learned_phys(p), h->learned, dx, ds, h->stream);
  if (e == 0 && (cudaMemcpyAsync(x, dx, cells * kFeatures * sizeof(float), cudaMemcpyDeviceToHost, h->stream) !=
                     cudaSuccess ||
                 cudaMemcpyAsync(scale, ds, cells * sizeof(double), cudaMemcpyDeviceToHost, h->stream) !=
                     cudaSuccess ||
                 cudaStreamSynchronize(h->stream) != cudaSuccess))
    e = -1;
  cudaFree(dx);
  cudaFree(ds);
  return e == 0 ? PCG_OK : fail(h, PCG_ERR_CUDA, "feature export");
}

int pcg_stage(pcg_handle* h, int stage) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h) return PCG_ERR_ARG;
  if (stage < 0 || stage > PCG_STAGE_ADVANCE_TIME) return fail(h, PCG_ERR_ARG, "unknown stage");
  h->started = true;
  int rc = run_stage(h, stage);
  if (rc != PCG_OK) return rc;
  if (stage == PCG_STAGE_COLLECT) return pcg_synchronize(h);
  return PCG_OK;
}

int pcg_step(pcg_handle* h, int nsteps) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || nsteps < 0) return PCG_ERR_ARG;
  if (h->halted) return fail(h, PCG_ERR_TIMEOUT, "halted after a tensor-core time-out");
  h->started = true;
  for (int n = 0; n < nsteps; ++n) {
    int rc = fused_step(h);
    if (rc != PCG_OK) return rc;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(h, PCG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return PCG_OK;
}

int pcg_synchronize(pcg_handle* h) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h) return PCG_ERR_ARG;
  return check_status(h);
}

int pcg_step_status(pcg_handle* h) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h) return PCG_ERR_ARG;
  int rc = PCG_OK;
  if (h->status_pending) {  // the block copied after the step before: that step has ended
    CUDA_TRY(h, cudaEventSynchronize(h->ev_status));
    h->status_pending = false;
    rc = status_code(h, h->h_status_lag);
  }
  CUDA_TRY(h, cudaMemcpyAsync(h->h_status_lag, h->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost,
                              h->stream));
  CUDA_TRY(h, cudaEventRecord(h->ev_status, h->stream));
  h->status_pending = true;
  return rc;
}

int pcg_seed_plasma_cells(pcg_handle* h, int slot, unsigned per_cell, double density, double t_par_ev,
                          double t_perp_ev, uint64_t seed) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || slot < 0 || slot >= (int)h->sp.size() || per_cell == 0) return PCG_ERR_ARG;
  if (!(density >= 0) || !(t_par_ev >= 0) || !(t_perp_ev >= 0))
    return fail(h, PCG_ERR_ARG, "negative density or temperature");
  Species& s = h->sp[slot];
  const size_t n = (size_t)h->g.nr * h->g.nz * per_cell;
  if (s.n + n > s.cap) return fail(h, PCG_ERR_CAPACITY, "species '" + s.name + "' capacity exceeded");
  h->started = true;
  PlasmaSeed p;
  p.seed = seed;
  p.stream = 0x706c6300u + (uint32_t)slot;
  p.sigma_v = sqrt(t_par_ev * kElCharge / s.mass);
  p.sigma_v_perp = sqrt(t_perp_ev * kElCharge / s.mass);
  p.weight = 0.0;
  p.per_cell = per_cell;
  p.density = density;
  if (is_f64(h)) launch_seed_f64(h->g, p, view64(h, s), s.n, n, h->stream);
  else {
    if (s.n == 0) { s.f32.next_id = 0; s.f32.sorted_n = 0; }
    launch_seed_f32(h->g, p, s.f32, s.n, n, h->stream);
    s.f32.next_id += (unsigned)n;
  }
  s.n += n;
  CUDA_TRY(h, cudaGetLastError());
  return PCG_OK;
}

int pcg_seed_plasma(pcg_handle* h, int slot, size_t n, double density, double temperature_ev,
                    uint64_t seed) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || slot < 0 || slot >= (int)h->sp.size()) return PCG_ERR_ARG;
  if (!(density >= 0) || !(temperature_ev >= 0)) return fail(h, PCG_ERR_ARG, "negative density or temperature");
  Species& s = h->sp[slot];
  if (s.n + n > s.cap) return fail(h, PCG_ERR_CAPACITY, "species '" + s.name + "' capacity exceeded");
  h->started = true;
  const GridGeom& g = h->g;
  const double r0 = 0.5 * g.dr, r1 = g.R - 0.5 * g.dr;
  const double volume = kPi * (r1 * r1 - r0 * r0) * (g.L - g.dz);
  PlasmaSeed p;
  p.seed = seed;
  p.stream = 0x706c6100u + (uint32_t)slot;
  p.sigma_v = sqrt(temperature_ev * kElCharge / s.mass);
  p.weight = n ? density * volume / (double)n : 0.0;
  if (is_f64(h)) launch_seed_f64(g, p, view64(h, s), s.n, n, h->stream);
  else {
    if (s.n == 0) { s.f32.next_id = 0; s.f32.sorted_n = 0; }
    launch_seed_f32(g, p, s.f32, s.n, n, h->stream);
    s.f32.next_id += (unsigned)n;
  }
  s.n += n;
  CUDA_TRY(h, cudaGetLastError());
  return PCG_OK;
}

int pcg_set_beam_profile(pcg_handle* h, int slot, int profile, double sigma_z,
                         double macro_per_cell) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || slot < 0 || slot >= (int)h->sp.size()) return PCG_ERR_ARG;
  Species& s = h->sp[slot];
  if (!s.beam) return fail(h, PCG_ERR_ARG, "not a beam");
  if (profile == PCG_PROFILE_RECTANGLE) {
    s.profile = profile;
    return PCG_OK;
  }
  if (profile != PCG_PROFILE_GAUSSIAN || !(sigma_z > 0) || !(macro_per_cell > 0))
    return fail(h, PCG_ERR_ARG, "unknown profile or non-positive sigma/macro count");
  s.profile = profile;
  s.sigma_z = sigma_z;
  // macroparticles per step: per cell of the bunch cylinder times the cells
  // its cross-section covers times the cells it advances per step
  s.gauss_mps = macro_per_cell * (s.radius / h->g.dr) * (s.velocity * h->cfg.dt / h->g.dz);
  return PCG_OK;
}

int pcg_enable_timers(pcg_handle* h, int on) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h) return PCG_ERR_ARG;
  h->timers = on != 0;
  return PCG_OK;
}

int pcg_kernel_times(pcg_handle* h, double* ms, int* launches, int n) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || !ms || n < 0) return PCG_ERR_ARG;
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  for (int c = 0; c < n; ++c) { ms[c] = 0; if (launches) launches[c] = 0; }
  for (auto& u : h->ev_used) {
    float t = 0;
    CUDA_TRY(h, cudaEventElapsedTime(&t, u.second.first, u.second.second));
    if (u.first < n) {
      ms[u.first] += t;
      if (launches) launches[u.first] += 1;
    }
    h->ev_pool.push_back(u.second.first);
    h->ev_pool.push_back(u.second.second);
  }
  h->ev_used.clear();
  return PCG_OK;
}

int pcg_get_stream(pcg_handle* h, void** stream) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || !stream) return PCG_ERR_ARG;
  *stream = (void*)h->stream;
  return PCG_OK;
}

int pcg_get_device(pcg_handle* h, int* device) {
  if (!h || !device) return PCG_ERR_ARG;
  *device = h->cfg.device;
  return PCG_OK;
}

int pcg_diag(pcg_handle* h, pcg_diagnostics* out) {
  DeviceScope device_scope(h ? h->cfg.device : -1);
  if (!h || !out) return PCG_ERR_ARG;
  int rc = check_status(h);
  if (rc != PCG_OK) return rc;
  std::memset(out, 0, sizeof(*out));
  out->time = h->t;
  out->steps = h->steps;
  out->removed = h->h_status->removed;
  out->move_errors = h->h_status->move_errors;
  out->particle_steps = h->particle_steps;
  uint64_t slots = 0;
  for (Species& s : h->sp) slots += s.n;
  const uint64_t dead = h->h_status->dead_slots;
  out->particles = slots - (dead > h->dead_dropped ? dead - h->dead_dropped : 0);
  out->kernel_launches = h->launches;
  double ee = 0, eh = 0, ek = 0;
  if (is_f64(h)) {
    if ((rc = f64_energies(h->g, fields64(h), &ee, &eh, h->stream)) != 0) return fail(h, PCG_ERR_CUDA, "energy reduction");
    for (Species& s : h->sp) {
      double e = 0;
      if ((rc = f64_kinetic(s.vr, s.vphi, s.vz, s.w, s.r, s.n, s.mass, &e, h->stream)) != 0) return fail(h, PCG_ERR_CUDA, "kinetic");
      ek += e;
    }
  } else {
    float* fl[12];
    for (int c = 0; c < 12; ++c) fl[c] = h->f32[c];
    if (f32_energies(h->g, fl, &ee, &eh, h->stream) != 0) return fail(h, PCG_ERR_CUDA, "energy reduction");
    for (Species& s : h->sp) {
      double e = 0;
      if (f32_kinetic(s.f32, s.n, s.mass, &e, h->stream) != 0) return fail(h, PCG_ERR_CUDA, "kinetic");
      ek += e;
    }
  }
  out->field_energy_e = ee;
  out->field_energy_h = eh;
  out->kinetic_energy = ek;
  return PCG_OK;
}

}  // extern "C"
