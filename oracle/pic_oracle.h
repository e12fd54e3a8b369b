/*
 * pic_oracle.h — CPU restatement of PiCoPiC's per-timestep PIC loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker for the CUDA path: only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * it.  The product (picopic_b200/libpcg.so) never links or calls it.
 *
 * Parity is pinned: tests/test_oracle_vs_reference.py compares every stage
 * bit-for-bit with the reference's own sources compiled by
 * oracle/Makefile.ref, and tests/golden/ holds fixtures generated from that
 * compiled reference (tests/golden/make_golden.py).
 *
 * Arithmetic is IEEE double in the same operation order as the reference
 * (compile with -ffp-contract=off).  Indices follow Grid<T> (grid.hpp:25-58):
 * field arrays are (nr+4) x (nz+4) doubles, z-contiguous, and node (i, k)
 * lives at [(i+2)*(nz+4) + (k+2)].
 */
#ifndef PIC_ORACLE_H
#define PIC_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Pusher / current switches (configure.ac:226-275), quirk modes. */
enum { ORC_PUSHER_BORIS = 0, ORC_PUSHER_BORIS_ADAPTIVE = 1, ORC_PUSHER_BORIS_RELATIVISTIC = 2,
       ORC_PUSHER_VAY = 3, ORC_PUSHER_HC = 4 };
enum { ORC_CURRENT_VB = 0, ORC_CURRENT_ZIGZAG = 1 };
enum { ORC_QUIRKS_REFERENCE = 0, ORC_QUIRKS_FIXED = 1 };
/* Beam-injection random source: the reference's std::mt19937 +
 * uniform_real_distribution (rand.cpp:24-31), or counter-based Philox4x32-10
 * keyed by (seed, species id) with counter (step, particle), as the GPU. */
enum { ORC_RNG_MT19937 = 0, ORC_RNG_PHILOX = 1 };

/* Stages: the Domain methods in the order SMB and main call them. */
enum { ORC_STAGE_INJECT = 0, ORC_STAGE_FIELD_E, ORC_STAGE_FIELD_H, ORC_STAGE_PUSH,
       ORC_STAGE_DUMP_OLD, ORC_STAGE_MOVE, ORC_STAGE_POS_RZ, ORC_STAGE_REFLECT,
       ORC_STAGE_VEL_RZ, ORC_STAGE_BIND, ORC_STAGE_COLLECT, ORC_STAGE_RESET_CURRENT,
       ORC_STAGE_CURRENT, ORC_STAGE_ADVANCE_TIME, ORC_STAGE_COUNT };

typedef struct orc_sim orc_sim;

orc_sim* orc_create(int nr, int nz, double radius, double longitude, double dt, double t_start,
                    const int* pml_size, const double* pml_sigma, int pusher, int current,
                    int quirks);
int orc_add_species(orc_sim* s, int id, const char* name, double charge_e, double mass_e);
int orc_add_beam(orc_sim* s, int id, const char* name, double charge_e, double mass_e,
                 unsigned macro_amount, double start_time, double b_radius, double density,
                 double amount, double length, double distance, double velocity);
void orc_set_rng(orc_sim* s, int kind, uint64_t seed);
int orc_set_particles(orc_sim* s, int sid, size_t n, const double* r, const double* z,
                      const double* vr, const double* vphi, const double* vz, const double* w);
long orc_count(orc_sim* s, int sid);
int orc_get_particles(orc_sim* s, int sid, size_t cap, double* r, double* z, double* vr,
                      double* vphi, double* vz, double* w, double* r_old, double* z_old,
                      long long* cell_r, long long* cell_z);
/* which: 0-2 E(r,phi,z), 3-5 H, 6-8 H_at_et, 9-11 J, 12 sigma (read only) */
int orc_set_field(orc_sim* s, int which, const double* src);
int orc_get_field(orc_sim* s, int which, double* dst);
/* ExternalFields (externalFields.cpp): formfactor names and params as
 * pcg_set_external_fields takes them. */
int orc_set_external_fields(orc_sim* s, const char* electric, const double* e_params, int n_e,
                            const char* magnetic, const double* m_params, int n_m);
int orc_stage(orc_sim* s, int stage);
int orc_step(orc_sim* s, int nsteps);
double orc_time(orc_sim* s);
long orc_removed(orc_sim* s);
long orc_error_count(orc_sim* s);
void orc_destroy(orc_sim* s);

/* One pass of the binary Coulomb collisions (Perez 2012 scheme,
 * collisions.cpp:230-236 + collisionsP12.cpp) on the current velocities,
 * cells from the last binding.  shuffle: Philox shuffle of the cell lists
 * (ORC_RNG_PHILOX).  Returns the number of pair calls or a negative status. */
long orc_collide(orc_sim* s, int shuffle);
/* One CollisionsTA77S pass (collisionsTA77S.cpp:568-576 without its
 * random_sort): Takizuka-Abe pairs, then the per-cell velocity correction. */
long orc_collide_ta77s(orc_sim* s, int shuffle);
long orc_collide_sk98(orc_sim* s, int shuffle);
/* SpecieP's diagnostic maps (specieP.cpp:665-839): which 0 density, 1
 * temperature, 2 energy, 3 momentum (3 grids); out holds (nr+4) x (nz+4)
 * doubles per grid. */
int orc_species_map(orc_sim* s, int sid, int which, double* out);

/* Building blocks exported for known-answer tests. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
double orc_philox_uniform(uint64_t seed, uint32_t stream, uint64_t step, uint32_t index,
                          int which);

#ifdef __cplusplus
}
#endif
#endif
