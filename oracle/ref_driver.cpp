/*
 * TEST INFRASTRUCTURE ONLY — never linked into the product.
 *
 * A C-ABI driver around the reference's OWN hot-path objects (Domain,
 * SpecieP, BeamP, MaxwellSolverYee, Pusher*, Current*), compiled together
 * with the unmodified reference sources by oracle/Makefile.ref into
 * oracle/_ref/libpicopic_ref_<pusher>_<current>.so.  It reproduces the
 * per-step order of the reference main loop for one domain:
 *
 *   PiCoPiC.cpp:326-347  inject_beam -> solve_maxvell -> advance_particles
 *                        -> solve_current, then time += step
 *   SMB.cpp:1231-1259    weight_field_e, weight_field_h
 *   SMB.cpp:1280-1306    push, [collide], dump old, move, back_position_to_rz,
 *                        reflect, back_velocity_to_rz, bind_cell_numbers,
 *                        particles_runaway_collector
 *   SMB.cpp:1266-1278    reset_current, weight_current
 *
 * The runaway collector (SMB.cpp:194-349) is restated for a single domain
 * because SMB needs the JSON config object: a particle is removed when its
 * bound cell is < 0 or >= the grid size in r or z; the survivors keep their
 * order (std::remove_if, SMB.cpp:216-345).
 */
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "domain.hpp"
#include "collisions/collisionsP12.hpp"
#include "collisions/collisionsTA77S.hpp"
#include "collisions/collisionsSK98.hpp"

namespace math::random {
extern std::mt19937 gen;  // rand.cpp:25, a non-static global
}

namespace pcg_ref_log {
static long g_errors = 0;
static long g_warnings = 0;
static bool g_fatal = false;
static std::string g_last;
void record(int level, const std::string& msg) {
  if (level == LVL_ERROR) ++g_errors;
  if (level == LVL_WARNING) ++g_warnings;
  if (level == LVL_FATAL) g_fatal = true;
  if (level >= LVL_WARNING) g_last = msg;
}
}  // namespace pcg_ref_log

namespace {

struct RefSim {
  Geometry* geometry = nullptr;
  TimeSim time{};
  std::vector<SpecieP*> species;
  Domain* domain = nullptr;
  size_t removed = 0;
  // ExternalFields' formfactors and params (the ENABLE_EXTERNAL_FIELDS build)
  std::string e_form = "none", m_form = "none";
  std::vector<double> e_params, m_params;
};

// CollisionsP12 with its protected steps reachable: the pass without
// Collisions::random_sort (which reseeds std::rand from time(0) and so can
// never be repeated) is clear, sort_to_cells, collect, collide
// (collisions.cpp:230-236 minus the shuffle).
class P12Pass : public CollisionsP12 {
 public:
  P12Pass(Geometry* g, TimeSim* t, std::vector<SpecieP*> sp) : CollisionsP12(g, t, sp) {}
  void run_unshuffled() {
    clear();
    sort_to_cells();
    collect_weighted_params_tot_grid();
    collide();
  }
};

// CollisionsTA77S::operator() (collisionsTA77S.cpp:568-576) without its
// random_sort, which reseeds std::srand from time(0).
class TA77SPass : public CollisionsTA77S {
 public:
  TA77SPass(Geometry* g, TimeSim* t, std::vector<SpecieP*> sp) : CollisionsTA77S(g, t, sp) {}
  void run_unshuffled() {
    clear();
    sort_to_cells();
    collect_weighted_params_tot_grid();
    collide();
    correct_velocities();
  }
};

// CollisionsSK98::operator() (collisionsSK98.cpp:442-450) without its
// random_sort; it has no correction pass.
class SK98Pass : public CollisionsSK98 {
 public:
  SK98Pass(Geometry* g, TimeSim* t, std::vector<SpecieP*> sp) : CollisionsSK98(g, t, sp) {}
  void run_unshuffled() {
    clear();
    sort_to_cells();
    collect_weighted_params_tot_grid();
    collide();
  }
};

Domain* domain_of(RefSim* s) {
#ifdef ENABLE_EXTERNAL_FIELDS
  // SMB.cpp:164-171 passes the configuration's formfactors and params
  if (!s->domain)
    s->domain = new Domain(*s->geometry, s->species, &s->time, s->e_form, s->m_form, s->e_params, s->m_params);
#else
  if (!s->domain) s->domain = new Domain(*s->geometry, s->species, &s->time);
#endif
  return s->domain;
}

Grid<double>* field_of(RefSim* s, int which) {
  Domain* d = domain_of(s);
  int comp = which % 3;
  switch (which / 3) {
    case 0: return &d->maxwell_solver->field_e[comp];
    case 1: return &d->maxwell_solver->field_h[comp];
    case 2: return &d->maxwell_solver->field_h_at_et[comp];
    case 3: return &d->current->current[comp];
    default: return nullptr;
  }
}

// Restatement of SMB::particles_runaway_collector for one domain (SMB.cpp:232-345).
void collect_runaways(RefSim* s) {
  const long nr = (long)s->geometry->cell_dims[2];
  const long nz = (long)s->geometry->cell_dims[3];
  for (SpecieP* sp : s->species) {
    auto& v = sp->particles;
    auto keep_end = std::remove_if(v.begin(), v.end(), [&](Particle*& o) {
      int r_cell = (int)P_CELL_R((*o));
      int z_cell = (int)P_CELL_Z((*o));
      if (r_cell < 0 || z_cell < 0) return true;
      if (r_cell >= nr) return true;
      if (z_cell >= nz) return true;
      return false;
    });
    for (auto it = keep_end; it != v.end(); ++it) {
      delete *it;
      ++s->removed;
    }
    v.erase(keep_end, v.end());
  }
}

int run_stage(RefSim* s, int stage) {
  Domain* d = domain_of(s);
  switch (stage) {
    case 0: d->manage_beam(); break;                      // inject
    case 1: d->weight_field_e(); break;                   // E
    case 2:                                               // H
      d->weight_field_h();
#ifdef ENABLE_EXTERNAL_FIELDS
      d->apply_external_fields();  // after the H update, SMB.cpp:1253-1262
#endif
      break;
    case 3: d->push_particles(); break;                   // gather + push
    case 4: d->dump_particle_positions_to_old(); break;
    case 5: d->update_particles_coords(); break;          // mover_cylindrical
    case 6: d->particles_back_position_to_rz(); break;
    case 7: d->reflect(); break;
    case 8: d->particles_back_velocity_to_rz(); break;
    case 9: d->bind_cell_numbers(); break;
    case 10: collect_runaways(s); break;
    case 11: d->reset_current(); break;
    case 12: d->weight_current(); break;
    case 13: s->time.current += s->time.step; break;
    default: return -2;
  }
  return 0;
}

}  // namespace

extern "C" {

void* ref_create(int nr, int nz, double radius, double longitude, double dt, double t_start,
                 const int* pml_size, const double* pml_sigma) {
  RefSim* s = new RefSim();
  std::vector<size_t> pml = {0, 0, 0, 0};
  std::vector<double> sigma = {0.0, 0.0};
  if (pml_size)
    for (int i = 0; i < 4; ++i) pml[i] = (size_t)pml_size[i];
  if (pml_sigma) sigma = {pml_sigma[0], pml_sigma[1]};
  // One domain: cfg.cpp:398-429 sets all four walls; SMB.cpp:49-120 keeps the
  // global PML sizes for a single domain.
  s->geometry = new Geometry({radius, longitude}, {radius, longitude},
                             {0, 0, (size_t)nr, (size_t)nz}, pml, sigma,
                             {true, true, true, true});
  s->geometry->domains_amount = {1, 1};
  s->time.start = t_start;
  s->time.current = t_start;
  s->time.end = 1e300;
  s->time.step = dt;
  return s;
}

// ExternalFields of the domain (before it is built: its constructor takes them).
int ref_set_external_fields(void* h, const char* electric, const double* e_params, int n_e,
                            const char* magnetic, const double* m_params, int n_m) {
  RefSim* s = (RefSim*)h;
  if (s->domain) return -3;
  s->e_form = electric ? electric : "none";
  s->m_form = magnetic ? magnetic : "none";
  s->e_params.assign(e_params, e_params + (e_params ? n_e : 0));
  s->m_params.assign(m_params, m_params + (m_params ? n_m : 0));
  return 0;
}

int ref_add_species(void* h, int id, const char* name, double charge_e, double mass_e) {
  RefSim* s = (RefSim*)h;
  if (s->domain) return -3;
  s->species.push_back(new SpecieP((unsigned)id, name, charge_e, mass_e, 0, 0.0, 0.0, 0.0,
                                   s->geometry, &s->time));
  return (int)s->species.size() - 1;
}

// A plasma species that the reference initialises itself: SpecieP with its
// macroparticle count, density and temperature (SMB.cpp:129-146 for one
// domain); its particles appear at ref_distribute.
int ref_add_plasma(void* h, int id, const char* name, double charge_e, double mass_e,
                   unsigned macro_amount, double density, double temperature) {
  RefSim* s = (RefSim*)h;
  if (s->domain) return -3;
  s->species.push_back(new SpecieP((unsigned)id, name, charge_e, mass_e, macro_amount, density,
                                   density, temperature, s->geometry, &s->time));
  return (int)s->species.size() - 1;
}

// Domain::distribute (domain.cpp:86-94): every species' own spatial
// placement (flat: the radical-inverse sequences of specieP.cpp:127-189 and
// the weights of :280-331), cell binding, then its thermal velocities
// (Maxwell-Juettner energies and uniform2 directions, :346-384) drawn from
// math::random::gen.  Beams place nothing here (beamP.hpp:63-64).
int ref_distribute(void* h) {
  RefSim* s = (RefSim*)h;
  pcg_ref_log::g_fatal = false;
  domain_of(s)->distribute();
  return pcg_ref_log::g_fatal ? -10 : 0;
}

int ref_add_beam(void* h, int id, const char* name, double charge_e, double mass_e,
                 unsigned macro_amount, double start_time, double b_radius, double density,
                 double amount, double length, double distance, double velocity) {
  RefSim* s = (RefSim*)h;
  if (s->domain) return -3;
  s->species.push_back(new BeamP((unsigned)id, name, charge_e, mass_e, macro_amount, start_time,
                                 b_radius, density, amount, length, distance, velocity,
                                 s->geometry, &s->time));
  return (int)s->species.size() - 1;
}

int ref_set_particles(void* h, int sid, size_t n, const double* r, const double* z,
                      const double* vr, const double* vphi, const double* vz, const double* w) {
  RefSim* s = (RefSim*)h;
  if (sid < 0 || sid >= (int)s->species.size()) return -1;
  SpecieP* sp = s->species[sid];
  for (Particle* p : sp->particles) delete p;
  sp->particles.clear();
  sp->particles.reserve(n);
  double dr = s->geometry->cell_size[0], dz = s->geometry->cell_size[1];
  for (size_t i = 0; i < n; ++i) {
    Particle* p = new Particle();
    p->specie_id = sp->id;
    p->pos_r = r[i];
    p->pos_z = z[i];
    p->vel_r = vr[i];
    p->vel_phi = vphi[i];
    p->vel_z = vz[i];
    p->weight = w[i];
    p->cell_r = CELL_NUMBER(p->pos_r, dr);   // as SpecieP::bind_cell_numbers
    p->cell_z = CELL_NUMBER(p->pos_z, dz);
    sp->particles.push_back(p);
  }
  return 0;
}

long ref_count(void* h, int sid) {
  RefSim* s = (RefSim*)h;
  if (sid < 0 || sid >= (int)s->species.size()) return -1;
  return (long)s->species[sid]->particles.size();
}

int ref_get_particles(void* h, int sid, size_t cap, double* r, double* z, double* vr,
                      double* vphi, double* vz, double* w, double* r_old, double* z_old,
                      long long* cell_r, long long* cell_z) {
  RefSim* s = (RefSim*)h;
  if (sid < 0 || sid >= (int)s->species.size()) return -1;
  auto& v = s->species[sid]->particles;
  if (cap < v.size()) return -4;
  for (size_t i = 0; i < v.size(); ++i) {
    const Particle* p = v[i];
    r[i] = p->pos_r; z[i] = p->pos_z;
    vr[i] = p->vel_r; vphi[i] = p->vel_phi; vz[i] = p->vel_z;
    w[i] = p->weight;
    if (r_old) r_old[i] = p->pos_old_r;
    if (z_old) z_old[i] = p->pos_old_z;
    if (cell_r) cell_r[i] = (long long)(int)p->cell_r;
    if (cell_z) cell_z[i] = (long long)(int)p->cell_z;
  }
  return 0;
}

int ref_set_field(void* h, int which, const double* src) {
  RefSim* s = (RefSim*)h;
  Grid<double>* g = field_of(s, which);
  if (!g) return -1;
  double** a = g->get_grid();
  for (unsigned i = 0; i < g->x_real_size; ++i)
    std::memcpy(a[i], src + (size_t)i * g->y_real_size, sizeof(double) * g->y_real_size);
  return 0;
}

int ref_get_field(void* h, int which, double* dst) {
  RefSim* s = (RefSim*)h;
  Grid<double>* g = field_of(s, which);
  if (!g) return -1;
  double** a = g->get_grid();
  for (unsigned i = 0; i < g->x_real_size; ++i)
    std::memcpy(dst + (size_t)i * g->y_real_size, a[i], sizeof(double) * g->y_real_size);
  return 0;
}

int ref_stage(void* h, int stage) {
  pcg_ref_log::g_fatal = false;
  int rc = run_stage((RefSim*)h, stage);
  return pcg_ref_log::g_fatal ? -10 : rc;
}

int ref_step(void* h, int nsteps) {
  for (int n = 0; n < nsteps; ++n)
    for (int st = 0; st <= 13; ++st) {
      int rc = ref_stage(h, st);
      if (rc != 0) return rc;
    }
  return 0;
}

// One P12 collision pass over the current particles (cells from the last
// binding), without the time-seeded shuffle; returns the pair count.
long ref_collide(void* h) {
  RefSim* s = (RefSim*)h;
  pcg_ref_log::g_fatal = false;
  P12Pass c(s->geometry, &s->time, s->species);
  c.run_unshuffled();
  return pcg_ref_log::g_fatal ? -10 : (long)c.ncol;
}

long ref_collide_ta77s(void* h) {
  RefSim* s = (RefSim*)h;
  pcg_ref_log::g_fatal = false;
  TA77SPass c(s->geometry, &s->time, s->species);
  c.run_unshuffled();
  return pcg_ref_log::g_fatal ? -10 : 0;
}

long ref_collide_sk98(void* h) {
  RefSim* s = (RefSim*)h;
  pcg_ref_log::g_fatal = false;
  SK98Pass c(s->geometry, &s->time, s->species);
  c.run_unshuffled();
  return pcg_ref_log::g_fatal ? -10 : 0;
}

// SpecieP's diagnostic maps (specieP.cpp:665-839): which 0 density, 1
// temperature, 2 energy, 3 momentum (3 grids r, phi, z).
int ref_species_map(void* h, int sid, int which, double* dst) {
  RefSim* s = (RefSim*)h;
  if (sid < 0 || sid >= (int)s->species.size()) return -1;
  SpecieP* sp = s->species[sid];
  pcg_ref_log::g_fatal = false;
  std::vector<Grid<double>*> grids;
  switch (which) {
    case 0: sp->calc_density(); grids.push_back(&sp->density_map); break;
    case 1: sp->calc_temperature(); grids.push_back(&sp->temperature_map); break;
    case 2: sp->calc_energy(); grids.push_back(&sp->energy_map); break;
    case 3:
      sp->calc_momentum();
      for (int c = 0; c < 3; ++c) grids.push_back(&sp->momentum_map[c]);
      break;
    default: return -1;
  }
  size_t off = 0;
  for (Grid<double>* g : grids) {
    double** a = g->get_grid();
    for (unsigned i = 0; i < g->x_real_size; ++i)
      std::memcpy(dst + off + (size_t)i * g->y_real_size, a[i], sizeof(double) * g->y_real_size);
    off += (size_t)g->x_real_size * g->y_real_size;
  }
  return pcg_ref_log::g_fatal ? -10 : 0;
}

double ref_time(void* h) { return ((RefSim*)h)->time.current; }
long ref_removed(void* h) { return (long)((RefSim*)h)->removed; }
void ref_seed(unsigned seed) { math::random::gen.seed(seed); }
long ref_error_count(void) { return pcg_ref_log::g_errors; }
long ref_warning_count(void) { return pcg_ref_log::g_warnings; }
const char* ref_last_message(void) { return pcg_ref_log::g_last.c_str(); }

void ref_destroy(void* h) {
  RefSim* s = (RefSim*)h;
  for (SpecieP* sp : s->species) delete sp;  // SpecieP deletes its particles (specieP.cpp:72-77)
  // Domain, solvers and geometry are leaked as in the reference (domain.cpp:35-83).
  delete s;
}

}  // extern "C"
