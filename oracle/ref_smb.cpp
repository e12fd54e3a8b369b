/*
 * TEST AND MEASUREMENT INFRASTRUCTURE ONLY — never linked into the product.
 *
 * A C-ABI driver around the reference's own scheduler, the unmodified
 * `SMB` of src/SMB.cpp, compiled by oracle/Makefile.ref together with the
 * reference's hot-path sources into oracle/_ref/libpicopic_ref_smb_<pusher>_<current>.so
 * with the reference's release flags and OpenMP.  It is the CPU arm the GPU
 * path is timed against: the reference's own domain decomposition, its
 * OpenMP loops over domains and its field, current and particle overlays.
 *
 *   smb_new         Cfg::init_geometry (cfg.cpp:379-429): the grid with all
 *                   four walls, its PML and its domains
 *   smb_add_species, smb_add_beam
 *                   the configuration's plasma species and beams
 *   smb_build       SMB::SMB (SMB.cpp:28-192)
 *   smb_distribute  SMB::distribute (SMB.cpp:1324-1334): every domain's own
 *                   flat placement and thermal velocities
 *   smb_step        the main loop body (PiCoPiC.cpp:326-347): inject_beam,
 *                   solve_maxvell, advance_particles, solve_current, then
 *                   time += step
 *
 * Cfg's JSON constructor lives in cfg.cpp, which needs picojson (absent
 * here); the driver defines it as an empty constructor and fills the
 * public fields SMB reads (particle_species, particle_beams).
 */
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "SMB.hpp"

namespace math::random {
extern std::mt19937 gen;  // rand.cpp:25
}

Cfg::Cfg(const std::string) {
  log_file = nullptr;
  macro_amount = 0;
  beam_macro_ratio = 1;
  geometry = nullptr;
  time = nullptr;
  output_data = nullptr;
}

Cfg::~Cfg(void) {}

namespace pcg_ref_log {
static long g_errors = 0;
static long g_warnings = 0;
static bool g_fatal = false;
static std::string g_last;
static std::mutex g_lock;  // SMB logs from inside its OpenMP loops over domains
void record(int level, const std::string& msg) {
  std::lock_guard<std::mutex> hold(g_lock);
  if (level == LVL_ERROR) ++g_errors;
  if (level == LVL_WARNING) ++g_warnings;
  if (level == LVL_FATAL) g_fatal = true;
  if (level >= LVL_WARNING) g_last = msg;
}
}  // namespace pcg_ref_log

namespace {

struct SmbRun {
  Cfg* cfg = nullptr;
  Geometry* geometry = nullptr;
  TimeSim* time = nullptr;
  SMB* smb = nullptr;
};

}  // namespace

extern "C" {

// Cfg::init_geometry (cfg.cpp:379-429): all four walls, PML cells
// {0, left, outer, right} and its two conductivities.  r_domains and
// z_domains must each be 1 or even (cfg.cpp:582-585), and the domains
// square in cells for the overlays (grid.hpp:141-145).
void* smb_new(int nr, int nz, double radius, double longitude, double dt, int r_domains,
              int z_domains, const int* pml_size, const double* pml_sigma) {
  if (nr < 2 || nz < 2 || r_domains < 1 || z_domains < 1) return nullptr;
  if ((r_domains != 1 && r_domains % 2) || (z_domains != 1 && z_domains % 2)) return nullptr;
  SmbRun* s = new SmbRun();
  s->cfg = new Cfg(std::string());
  std::vector<size_t> pml = {0, 0, 0, 0};
  std::vector<double> sigma = {0.0, 0.0};
  if (pml_size)
    for (int i = 0; i < 4; ++i) pml[i] = (size_t)pml_size[i];
  if (pml_sigma) sigma = {pml_sigma[0], pml_sigma[1]};
  s->geometry = new Geometry({radius, longitude}, {0, 0, (size_t)nr, (size_t)nz}, pml, sigma,
                             {true, true, true, true});
  s->geometry->domains_amount = {(size_t)r_domains, (size_t)z_domains};
  s->time = new TimeSim();
  s->time->start = 0;
  s->time->current = 0;
  s->time->end = 1e300;
  s->time->step = dt;
  s->time->print_header_counter = 0;
  s->cfg->geometry = s->geometry;
  s->cfg->time = s->time;
  return s;
}

// A plasma species of the configuration (cfg.cpp particles section): its
// total macroparticle count, which SMB splits evenly over the domains.
int smb_add_species(void* h, unsigned id, const char* name, int charge, unsigned mass,
                    double macro_amount, double density, double temperature) {
  SmbRun* s = (SmbRun*)h;
  if (s->smb) return -3;
  particle_specie p;
  p.id = id;
  p.name = name;
  p.mass = mass;
  p.charge = charge;
  p.macro_amount = macro_amount;
  p.left_density = density;
  p.right_density = density;
  p.temperature = temperature;
  s->cfg->macro_amount += macro_amount;
  s->cfg->particle_species.push_back(p);
  return 0;
}

// A beam of the configuration (cfg.cpp beams section); every domain gets a
// BeamP with these parameters (SMB.cpp:148-164).
int smb_add_beam(void* h, unsigned id, const char* name, int charge, unsigned mass,
                 double macro_amount, double start_time, double bunch_radius, double density,
                 int bunches_amount, double bunch_length, double bunches_distance, double velocity) {
  SmbRun* s = (SmbRun*)h;
  if (s->smb) return -3;
  particle_beam b;
  b.id = id;
  b.name = name;
  b.mass = mass;
  b.charge = charge;
  b.macro_amount = macro_amount;
  b.left_density = density;
  b.right_density = density;
  b.temperature = 0;
  b.velocity = velocity;
  b.density = density;
  b.bunches_amount = bunches_amount;
  b.start_time = start_time;
  b.bunches_distance = bunches_distance;
  b.bunch_length = bunch_length;
  b.bunch_radius = bunch_radius;
  b.current_bunch_number = 0;
  b.radial_profile = "rectangle";
  b.longitudinal_profile = "rectangle";
  s->cfg->particle_beams.push_back(b);
  return 0;
}

// SMB::SMB (SMB.cpp:28-192): the domains, their species and beams.
int smb_build(void* h) {
  SmbRun* s = (SmbRun*)h;
  if (s->smb) return -3;
  pcg_ref_log::g_fatal = false;
  s->smb = new SMB(s->cfg, s->geometry, s->time, 0, 1);
  return pcg_ref_log::g_fatal ? -10 : 0;
}

int smb_distribute(void* h) {
  SmbRun* s = (SmbRun*)h;
  if (!s->smb) return -3;
  pcg_ref_log::g_fatal = false;
  s->smb->distribute();
  return pcg_ref_log::g_fatal ? -10 : 0;
}

int smb_step(void* h, int nsteps) {
  SmbRun* s = (SmbRun*)h;
  if (!s->smb) return -3;
  pcg_ref_log::g_fatal = false;
  for (int n = 0; n < nsteps; ++n) {
    s->smb->inject_beam();
    s->smb->solve_maxvell();
    s->smb->advance_particles();
    s->smb->solve_current();
    s->time->current += s->time->step;
    if (pcg_ref_log::g_fatal) return -10;
  }
  return 0;
}

long smb_particles(void* h) {
  SmbRun* s = (SmbRun*)h;
  if (!s->smb) return -1;
  long n = 0;
  for (unsigned i = 0; i < s->smb->r_domains; ++i)
    for (unsigned j = 0; j < s->smb->z_domains; ++j)
      for (SpecieP* sp : s->smb->domains(i, j)->species_p) n += (long)sp->particles.size();
  return n;
}

// One field of the whole grid, (nr + 4) x (nz + 4) doubles in the Grid
// layout, 0 in the outer halo: each domain's interior nodes, as the
// writers read them after the overlays (outController.cpp:151-297).
// which: 0-2 E, 3-5 H_at_et, 6-8 J (r, phi, z).
int smb_get_field(void* h, int which, double* dst) {
  SmbRun* s = (SmbRun*)h;
  if (!s->smb || which < 0 || which > 8) return -1;
  const size_t ld = s->geometry->cell_amount[1] + 4;
  std::memset(dst, 0, sizeof(double) * (s->geometry->cell_amount[0] + 4) * ld);
  for (unsigned i = 0; i < s->smb->r_domains; ++i)
    for (unsigned j = 0; j < s->smb->z_domains; ++j) {
      Domain* d = s->smb->domains(i, j);
      Grid<double>* g = which < 3   ? &d->maxwell_solver->field_e[which]
                        : which < 6 ? &d->maxwell_solver->field_h_at_et[which - 3]
                                    : &d->current->current[which - 6];
      const size_t r0 = d->geometry.cell_dims[0], z0 = d->geometry.cell_dims[1];
      const size_t nr = d->geometry.cell_amount[0], nz = d->geometry.cell_amount[1];
      double** a = g->get_grid();
      for (size_t r = 0; r < nr; ++r)
        for (size_t z = 0; z < nz; ++z) dst[(r0 + r + 2) * ld + (z0 + z + 2)] = a[r + 2][z + 2];
    }
  return 0;
}

int smb_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

long smb_error_count(void) { return pcg_ref_log::g_errors; }

// Seed the reference's global generator (rand.cpp:25, a non-static global).
void smb_seed(unsigned seed) { math::random::gen.seed(seed); }

}  // extern "C"
