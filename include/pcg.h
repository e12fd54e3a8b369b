/*
 * pcg.h — C ABI of the B200-native PiCoPiC per-timestep PIC loop.
 *
 * One handle = one simulation domain (the whole r-z grid on one GPU) with
 * its particle species and beams, owning its device memory and one CUDA
 * stream.  A handle is not thread-safe; use one host thread per handle.
 *
 * The entry points replace the per-domain façade that the reference's
 * scheduler (SMB) drives every step.  Reference interfaces (file:line in
 * the PiCoPiC sources):
 *
 *   pcg_create            Domain::Domain                 src/domain.cpp:26-84
 *                         (Geometry from Cfg::init_geometry src/cfg.cpp:379-429,
 *                          TimeSim from Cfg::init_time     src/cfg.cpp:430-440)
 *   pcg_add_species       SpecieP::SpecieP               src/specieP.cpp:23-70
 *   pcg_add_beam          BeamP::BeamP                   src/beamP.cpp:22-69
 *   pcg_import_species    SpecieP::particles (vector<Particle*>)
 *                                                        include/specieP.hpp:74-163
 *   pcg_export_species    same, read back
 *   pcg_set_field /       MaxwellSolver::field_e, field_h include/maxwellSolver.hpp:39-40,
 *   pcg_export_field      MaxwellSolverYee::field_h_at_et include/maxwellSolver/maxwellSolverYee.hpp:29,
 *                         Current::current                include/current.hpp:41
 *                         (Grid<double> with a 2-cell halo include/algo/grid.hpp:25-58)
 *   pcg_stage             one Domain method:
 *                           PCG_STAGE_INJECT        Domain::manage_beam        src/domain.cpp:180-186
 *                           PCG_STAGE_FIELD_E       Domain::weight_field_e     src/domain.cpp:123-126
 *                           PCG_STAGE_FIELD_H       Domain::weight_field_h     src/domain.cpp:118-121
 *                           PCG_STAGE_PUSH          Domain::push_particles     src/domain.cpp:141-144
 *                           PCG_STAGE_DUMP_OLD      Domain::dump_particle_positions_to_old src/domain.cpp:193-197
 *                           PCG_STAGE_MOVE          Domain::update_particles_coords src/domain.cpp:146-151
 *                           PCG_STAGE_POS_RZ        Domain::particles_back_position_to_rz src/domain.cpp:168-172
 *                           PCG_STAGE_REFLECT       Domain::reflect            src/domain.cpp:160-165
 *                           PCG_STAGE_VEL_RZ        Domain::particles_back_velocity_to_rz src/domain.cpp:174-178
 *                           PCG_STAGE_BIND          Domain::bind_cell_numbers  src/domain.cpp:153-158
 *                           PCG_STAGE_COLLECT       SMB::particles_runaway_collector src/SMB.cpp:194-349
 *                           PCG_STAGE_RESET_CURRENT Domain::reset_current      src/domain.cpp:135-139
 *                           PCG_STAGE_CURRENT       Domain::weight_current     src/domain.cpp:188-191
 *                           PCG_STAGE_ADVANCE_TIME  main loop time += step     src/PiCoPiC.cpp:347
 *   pcg_step              one full step in the order of src/PiCoPiC.cpp:326-347 and
 *                         SMB::inject_beam/solve_maxvell/advance_particles/solve_current
 *                         src/SMB.cpp:1231-1322, as fused device kernels.
 *
 * Errors: every call returns a status (PCG_OK = 0, negative on error).  The
 * reference aborts on LOG_S(FATAL) (NaN positions pusherBoris.cpp:51-57,
 * NaN fields maxwellSolverYee.cpp:253-255, v > c rel.cpp:33-34); here the
 * device raises an error word and the call returns PCG_ERR_NAN or
 * PCG_ERR_SUPERLUMINAL.  The reference's LOG_S(ERROR) on a particle moving
 * more than one cell (currentVB.cpp:199-204) skips that particle's current,
 * as in the reference, and is counted in pcg_diagnostics.move_errors.
 *
 * Layout conventions of the host arrays: fields are (nr+4) x (nz+4) doubles,
 * row i (radius) major, z contiguous, node (i, k) at [(i+2)*(nz+4) + k+2],
 * as Grid<double> stores them.  Particle arrays are structure-of-arrays of
 * doubles in SI units (m, m/s, real particles per macroparticle).
 */
#ifndef PCG_H
#define PCG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PCG_ABI_VERSION 1

/* status codes */
#define PCG_OK 0
#define PCG_ERR_ARG (-1)
#define PCG_ERR_CUDA (-2)
#define PCG_ERR_NOMEM (-3)
#define PCG_ERR_STATE (-4)
#define PCG_ERR_CAPACITY (-5)
#define PCG_ERR_NAN (-10)
#define PCG_ERR_SUPERLUMINAL (-11)
#define PCG_ERR_TIMEOUT (-12)
#define PCG_ERR_UNSUPPORTED (-13)

/* pusher switch (configure.ac:96-98, 226-239) */
#define PCG_PUSHER_BORIS 0
#define PCG_PUSHER_BORIS_ADAPTIVE 1
#define PCG_PUSHER_BORIS_RELATIVISTIC 2
#define PCG_PUSHER_VAY 3
#define PCG_PUSHER_HC 4

/* charge-conserving current scheme (configure.ac:108-110, 268-275) */
#define PCG_CURRENT_VB 0
#define PCG_CURRENT_ZIGZAG 1

/* arithmetic of the particle path */
#define PCG_PRECISION_F64 0 /* positions in double, the reference arithmetic */
#define PCG_PRECISION_F32 1 /* int32 cell + float offset, float fields */

/* PCG_QUIRKS_REFERENCE reproduces the reference's arithmetic defects;
 * PCG_QUIRKS_FIXED corrects them where a correction is defined. */
#define PCG_QUIRKS_REFERENCE 0
#define PCG_QUIRKS_FIXED 1

/* stages, numbered as the oracle's */
#define PCG_STAGE_INJECT 0
#define PCG_STAGE_FIELD_E 1
#define PCG_STAGE_FIELD_H 2
#define PCG_STAGE_PUSH 3
#define PCG_STAGE_DUMP_OLD 4
#define PCG_STAGE_MOVE 5
#define PCG_STAGE_POS_RZ 6
#define PCG_STAGE_REFLECT 7
#define PCG_STAGE_VEL_RZ 8
#define PCG_STAGE_BIND 9
#define PCG_STAGE_COLLECT 10
#define PCG_STAGE_RESET_CURRENT 11
#define PCG_STAGE_CURRENT 12
#define PCG_STAGE_ADVANCE_TIME 13

/* field slots */
#define PCG_FIELD_E_R 0
#define PCG_FIELD_E_PHI 1
#define PCG_FIELD_E_Z 2
#define PCG_FIELD_H_R 3
#define PCG_FIELD_H_PHI 4
#define PCG_FIELD_H_Z 5
#define PCG_FIELD_HAT_R 6 /* field_h_at_et */
#define PCG_FIELD_HAT_PHI 7
#define PCG_FIELD_HAT_Z 8
#define PCG_FIELD_J_R 9
#define PCG_FIELD_J_PHI 10
#define PCG_FIELD_J_Z 11

typedef struct pcg_handle pcg_handle;

typedef struct pcg_config {
  int nr, nz;                /* grid cells in r and z */
  double radius, longitude;  /* domain size, m (dr = radius/nr, dz = longitude/nz) */
  double dt, t_start;        /* time step and start time, s */
  int pml_size[4];           /* PML cells on the walls r=0 (unused), z=0, r=R, z=L */
  double pml_sigma[2];       /* PML sigma_1, sigma_2 */
  int pusher, current, precision, quirks;
  int device;                /* CUDA device ordinal */
  uint64_t seed;             /* beam-injection random stream (Philox4x32-10) */
} pcg_config;

typedef struct pcg_diagnostics {
  double time;                  /* simulation time, s */
  uint64_t steps;               /* steps taken by pcg_step / PCG_STAGE_ADVANCE_TIME */
  uint64_t particles;           /* live macroparticles, all species */
  uint64_t removed;             /* removed by the runaway collector */
  uint64_t move_errors;         /* >1-cell moves whose current was skipped */
  uint64_t particle_steps;      /* sum over steps of live particles pushed */
  double field_energy_e;        /* sum over interior nodes of eps0/2 E^2 * cell volume, J */
  double field_energy_h;        /* sum of mu0/2 H^2 * cell volume, J */
  double kinetic_energy;        /* sum of (gamma-1) m c^2 * weight, J */
  uint64_t kernel_launches;     /* kernels launched by pcg_step and pcg_stage so far */
} pcg_diagnostics;

int pcg_abi_version(void);
int pcg_create(const pcg_config* cfg, pcg_handle** out);
int pcg_destroy(pcg_handle* h);
const char* pcg_last_error(const pcg_handle* h);

/* Species are added before the first particle import; `slot` returns the
 * index used by the calls below (species are processed in slot order, as
 * the reference processes its species vector). */
int pcg_add_species(pcg_handle* h, int id, const char* name, double charge_e, double mass_e,
                    size_t capacity, int* slot);
int pcg_add_beam(pcg_handle* h, int id, const char* name, double charge_e, double mass_e,
                 size_t capacity, unsigned macro_amount, double start_time, double bunch_radius,
                 double density, double bunches_amount, double bunch_length,
                 double bunches_distance, double velocity, int* slot);

/* Replace (import) or extend (append) a species' particles from host SoA.
 * An append that would exceed the capacity first reclaims the species'
 * dead slots (a compaction, which waits for the stream).  The float layout
 * drops a position outside the grid at once (counted in
 * pcg_diagnostics.removed, as the runaway collector counts it); one more
 * than a cell beyond the grid, or not a number, also makes the next call
 * that reads the status return PCG_ERR_STATE or PCG_ERR_NAN, which the
 * double layout returns from the step that meets such a particle. */
int pcg_import_species(pcg_handle* h, int slot, size_t n, const double* r, const double* z,
                       const double* vr, const double* vphi, const double* vz, const double* w);
int pcg_append_species(pcg_handle* h, int slot, size_t n, const double* r, const double* z,
                       const double* vr, const double* vphi, const double* vz, const double* w);
int pcg_count(pcg_handle* h, int slot, size_t* n);
/* Copy a species back (live particles in reference order).  cell_r/cell_z
 * may be NULL.  Fails with PCG_ERR_CAPACITY if cap < count. */
int pcg_export_species(pcg_handle* h, int slot, size_t cap, double* r, double* z, double* vr,
                       double* vphi, double* vz, double* w, int32_t* cell_r, int32_t* cell_z,
                       size_t* n);

/* Seed a species on the device with `n` macroparticles of a uniform
 * plasma filling the region between the reflecting walls: r^2 uniform in
 * [(dr/2)^2, (R-dr/2)^2], z uniform in [dz/2, L-dz/2], Maxwellian velocity
 * components of variance T*e/m, equal weights density*volume/n.  The
 * random numbers are Philox4x32-10 keyed by `seed` and the species slot.
 * Replaces SpecieP::fullyfill_spatial_distribution + velocity_distribution
 * (specieP.cpp:79-478) as the source of synthetic initial conditions. */
int pcg_seed_plasma(pcg_handle* h, int slot, size_t n, double density, double temperature_ev,
                    uint64_t seed);
/* The same with `per_cell` macroparticles in every cell (nr*nz*per_cell
 * in all), uniform in the cell's ring volume, weights density*V_cell/
 * per_cell (the reference's equal-count cell filling, specieP.cpp:127-189),
 * and a bi-Maxwellian: temperature t_par_ev along z, t_perp_ev along r and
 * phi. */
int pcg_seed_plasma_cells(pcg_handle* h, int slot, unsigned per_cell, double density, double t_par_ev,
                          double t_perp_ev, uint64_t seed);

/* Longitudinal bunch profile of a beam.  PCG_PROFILE_RECTANGLE is BeamP
 * (beamP.cpp:71-157).  PCG_PROFILE_GAUSSIAN injects a bunch of density
 * density*exp(-(s-3 sigma_z)^2/(2 sigma_z^2)) over 6 sigma_z behind its
 * head s = 0, with macro_per_cell macroparticles per cell of the bunch
 * cylinder; the reference parses a `profile` key but only injects
 * rectangles (cfg.cpp:366-367). */
#define PCG_PROFILE_RECTANGLE 0
#define PCG_PROFILE_GAUSSIAN 1
int pcg_set_beam_profile(pcg_handle* h, int slot, int profile, double sigma_z,
                         double macro_per_cell);

/* Device time per kernel class, measured with CUDA events on the handle's
 * stream while enabled; pcg_kernel_times returns milliseconds and launch
 * counts accumulated since the last call and resets them. */
#define PCG_TIMER_FIELD_E 0
#define PCG_TIMER_FIELD_H 1
#define PCG_TIMER_INJECT 2
#define PCG_TIMER_PARTICLES 3 /* fused push/move/reflect/bind(/deposit) */
#define PCG_TIMER_DEPOSIT 4   /* separate deposit kernel of the double path */
#define PCG_TIMER_COUNT 5
int pcg_enable_timers(pcg_handle* h, int on);
int pcg_kernel_times(pcg_handle* h, double* ms, int* launches, int n);

/* Acceptance diagnostics of the deposit, double precision; no counterpart
 * in the reference.  pcg_node_charge fills q ((nr+4) x (nz+4), C) with the
 * particles' node charges in the shape the Villasenor-Buneman deposit
 * conserves: a particle at x = r/dr in cell i gives node i the radial share
 * 1/2 + i(i+1)/(2x) - x/2, node i+1 the rest, times linear axial shares.
 * pcg_divergence fills out with the flux divergence of J (which =
 * PCG_FIELD_J_R) or E (PCG_FIELD_E_R):
 *   F_r(i,k) A(i) - F_r(i-1,k) A(i-1) + (F_z(i,k) - F_z(i,k-1)) S(i),
 * A(i) = 2 pi (i+1/2) dr dz, S(i) = 2 pi i dr^2 (pi dr^2 / 4 on the axis),
 * the face areas of the reference's Yee update.  Charge continuity over one
 * step is then Q(n+1) - Q(n) + dt div J = 0, and the Gauss residual is
 * eps0 div E - Q. */
int pcg_node_charge(pcg_handle* h, double* q);
int pcg_divergence(pcg_handle* h, int which, double* out);

/* One pass of binary Coulomb collisions, the Perez et al. 2012 scheme of
 * CollisionsP12::operator() (collisions.cpp:230-236, collisionsP12.cpp:29-569),
 * in double precision on the current velocities, with the cells of the last
 * binding: the reference calls it between the push and the move
 * (SMB.cpp:1289-1293, Domain::collide domain.cpp:199-204).  Electron lists
 * take every species except those named "ions"/"Ions"; masses and charges
 * come from the species named "electrons"/"Electrons" and "ions"/"Ions".
 * Cell lists are shuffled and collisions draw from Philox keyed by the
 * handle seed and a pass counter (the reference shuffles with
 * std::srand(time(0)) and draws from its global mt19937).
 * PCG_QUIRKS_REFERENCE keeps the reference's relative speed (difference of
 * the centre-of-mass speeds), its deflection test against the macroparticle
 * weight and its `break` out of a cell row at a non-normal temperature or
 * density; PCG_QUIRKS_FIXED corrects them.  *pair_calls (may be NULL)
 * receives the number of pair collisions attempted. */
int pcg_collide(pcg_handle* h, unsigned long long* pair_calls);

/* The binary operator of pcg_collide and of PCG_COLLISIONS_BINARY steps;
 * replaces the compile-time choice of collisions scheme
 * (Domain::Domain domain.cpp:55-60: CollisionsP12, CollisionsTA77S or
 * CollisionsSK98).
 * PCG_COLLIDE_TA77S is collisionsTA77S.cpp: Takizuka-Abe pairs with the
 * weighted second angle (:33-208) in the same pairing sequence, then
 * correct_velocities (:419-566), which gives each species of each cell back
 * its momentum and kinetic energy from before the pass.
 * PCG_QUIRKS_REFERENCE keeps its sign of b's velocity change (+m_ab/m_b du2,
 * :191-193) and its |alpha| for a negative correction factor; the fixed mode
 * subtracts and leaves such a species uncorrected.  PCG_COLLIDE_SK98 is
 * collisionsSK98.cpp:29-244: the CM momentum of each pair rotated by a
 * normal delta of variance (collision frequency) x dt and both particles
 * boosted back, no weight rejection, no correction; the reference subtracts
 * the CM speeds in the relative velocity (:131-132), the fixed mode adds
 * them.  The learned step's
 * fallback is always P12, the operator its model was trained on. */
#define PCG_COLLIDE_P12 0
#define PCG_COLLIDE_TA77S 1
#define PCG_COLLIDE_SK98 2
int pcg_set_collision_scheme(pcg_handle* h, int scheme);

/* External fields: ExternalFields (src/maxwellSolver/externalFields.cpp),
 * whose E and H the pushers gather at each particle and add to the field
 * solver's (pusherBoris.cpp:62-65, pusherVay.cpp:48-50, pusherHC.cpp:51-54), set
 * after the H update of every step (SMB.cpp:1253-1262) and constant in time.
 * The reference builds it only with ENABLE_EXTERNAL_FIELDS (configure.ac:
 * 215-222, a development option); without this call there are none.
 * `electric` and `magnetic` are the formfactor names of PiCoPiC.json's
 * external_fields section (cfg.cpp:454-487): "none", "const_r",
 * "const_phi", "const_z", "linerad_r", "linerad_z"; params[0] is the
 * amplitude (V/m, A/m).  The fields live on the cells 1 <= i < nr-1,
 * 1 <= k < nz-1 (the wall rows and the halo stay 0, externalFields.cpp:
 * 298-348).  PCG_QUIRKS_REFERENCE: the electric name test
 * (externalFields.cpp:51-62) maps every name but "none" to "none" and
 * "none" to "const_r", and neither sets a field, so no electric field
 * applies; of the magnetic names only "const_z" sets one, H_z = params[0];
 * an unknown magnetic name is PCG_ERR_ARG (the reference's FATAL).
 * PCG_QUIRKS_FIXED: "const_r", "const_phi" and "const_z" of either field
 * set that component to params[0]; "linerad_*", whose parameters the
 * reference leaves undefined, is PCG_ERR_UNSUPPORTED.  NULL or "none" for
 * both removes the fields. */
int pcg_set_external_fields(pcg_handle* h, const char* electric, const double* e_params, int n_e,
                            const char* magnetic, const double* m_params, int n_m);

/* Work split of the binary pass (no counterpart in the reference, which
 * runs every cell's pairing sequence in turn): cells holding more than
 * `threshold` particles (256 by default) run their sequence on a warp, the
 * collisions touching disjoint particles on different lanes in the
 * reference's order and with the same draws; the others on one thread
 * each.  The result does not depend on the threshold. */
int pcg_set_collision_crowding(pcg_handle* h, unsigned threshold);

/* The per-cell collision MLP of the learned collision step (no counterpart
 * in the reference): 13 inputs -> 128 -> 128 -> 6 outputs, ReLU, BF16
 * operands on the tensor cores with FP32 accumulation.  Parameters are FP32,
 * row-major [in][out] per layer in the order W1, b1, W2, b2, W3, b3.
 * pcg_mlp_create draws He-uniform weights from Philox(seed) on `device`;
 * pcg_mlp_forward runs rows x 13 host inputs to rows x 6 host outputs;
 * pcg_mlp_gradient returns the full-batch gradient (and value) of the loss
 * mean((y - t)^2) over rows and outputs; pcg_mlp_set_data makes a training
 * set resident and pcg_mlp_train takes Adam steps (beta 0.9, 0.999, eps
 * 1e-8) on minibatches of `batch` rows drawn with Philox. */
typedef struct pcg_mlp pcg_mlp;
#define PCG_MLP_INPUTS 13
#define PCG_MLP_HIDDEN 128
#define PCG_MLP_OUTPUTS 6
#define PCG_MLP_PARAMS 19078
int pcg_mlp_create(int device, uint64_t seed, pcg_mlp** out);
int pcg_mlp_destroy(pcg_mlp* m);
int pcg_mlp_get_params(pcg_mlp* m, float* params);
int pcg_mlp_set_params(pcg_mlp* m, const float* params);
int pcg_mlp_forward(pcg_mlp* m, const float* x, size_t rows, float* y);
/* The same forward pass on the fifth-generation tensor cores (tcgen05.mma,
 * accumulators in tensor memory, 128 rows per CTA; no reference
 * counterpart): the same BF16 operands and FP32 accumulation, so outputs
 * agree with pcg_mlp_forward to the order of the FP32 sums.  *device_ms
 * (may be NULL) receives the kernel's device time.  PCG_ERR_TIMEOUT if a
 * wait for the tensor cores timed out (the kernel then stops and frees its
 * tensor memory). */
int pcg_mlp_forward_tc(pcg_mlp* m, const float* x, size_t rows, float* y, float* device_ms);
int pcg_mlp_gradient(pcg_mlp* m, const float* x, const float* t, size_t rows, float* grad, float* loss);
int pcg_mlp_set_data(pcg_mlp* m, const float* x, const float* t, size_t rows);
int pcg_mlp_train(pcg_mlp* m, int steps, int batch, float lr, float* last_loss);

/* The learned collision step (no counterpart in the reference).  Per cell,
 * the moment sums of the electron list (every species not named ions) and
 * the ion list give 13 features; the collision MLP (pcg_mlp_*) maps them to
 * the change of the six axis temperatures over one step, and every particle
 * of the cell moves to v' = u + (v - u) sqrt(T'/T) per axis in FP64, so each
 * species keeps its momentum, the cell its thermal energy, and the new
 * second moments hold exactly.  Cells whose features leave the model's
 * training box (widened by 25 % of each feature's span) take the binary
 * operator (pcg_collide) instead.
 * pcg_set_collision_model loads PCG_MLP_PARAMS parameters and
 * PCG_LEARNED_NORM floats: feature mean[13], std[13], target mean[6],
 * std[6], feature low[13], high[13].  pcg_collide_learned reports the cells
 * that took the learned and the binary path (either pointer may be NULL).
 * pcg_cell_moments fills nr*nz x 16 doubles (per cell, electron list then
 * ion list: N, sum w, sum w v_r, v_phi, v_z, sum w v_r^2, v_phi^2, v_z^2);
 * pcg_cell_features fills nr*nz x 13 raw features (NaN where a cell has
 * fewer than two particles in a list) and the per-cell collision scale
 * S = s_ee + s_ei + s_ii that the targets are measured in. */
#define PCG_LEARNED_NORM 64
/* One binary collision pass (as pcg_collide) that also returns, per cell,
 * the sum over its collisions of each collision's mean change over its
 * scattering-angle draw given the velocities that collision meets
 * (non-relativistic kinematics of the mean): an unbiased estimate of the
 * pass's expected moment change with far less Monte Carlo noise than the
 * change itself.  nr*nz x 12 doubles: the change of sum w v (3) and sum w
 * v^2 (3) of the electron list, then of the ion list.  The training
 * targets of the collision MLP. */
int pcg_collide_expectation(pcg_handle* h, double* out);
int pcg_set_collision_model(pcg_handle* h, const float* params, const float* norm);
int pcg_collide_learned(pcg_handle* h, unsigned long long* learned_cells, unsigned long long* fallback_cells);
int pcg_cell_moments(pcg_handle* h, double* moments);
int pcg_cell_features(pcg_handle* h, float* features, double* scale);

/* Tiling of the float step (no reference counterpart: its particles are not
 * tiled).  Species are re-sorted into 8 x 32-cell tiles at most every
 * sort_interval steps (default 64; sooner when particles drift out of their
 * tile's windows), and a sort spreads each occupied tile over enough blocks
 * that about target_blocks blocks run (default 148 x 16), each with at least
 * min_split particles (default 1024).  0 keeps a value; the next step
 * re-sorts.  pcg_ensemble_autotune picks these per run. */
int pcg_set_tiling(pcg_handle* h, int sort_interval, int target_blocks, int min_split);

/* Sort species `slot` of a float-layout handle into its tiles now (as a
 * step does when its particles have drifted; dead slots are dropped) and
 * report the result: counts[c] (host, nr x nz, cell c = i * nz + k) the
 * particles the sorted tiles hold in cell c, *misplaced those whose cell is
 * outside their tile (0 unless the sort is wrong).  The reference groups
 * particles per cell only for collisions (Collisions::sort_to_cells,
 * collisions.cpp:87-108); this is the float step's replacement, exposed
 * for checking.  PCG_ERR_UNSUPPORTED for the double layout. */
int pcg_tile_sort(pcg_handle* h, int slot, unsigned* counts, unsigned long long* misplaced);

/* An ensemble: independent runs (handles, each with its own grid, species
 * and stream; the batched configuration of many small runs) advanced
 * together.  No reference counterpart: the reference runs one simulation
 * per process.  pcg_ensemble_create groups handles it does not own (all on
 * one device); pcg_ensemble_step advances every run by nsteps, the runs
 * spread over `threads` host threads that each issue their runs' steps in
 * turn, so that the GPU overlaps the runs' kernels; *device_ms (may
 * be NULL) receives the device time from the first to the last of the
 * batch's kernels (events on the runs' streams, joined on one stream).
 * pcg_ensemble_autotune times trial_steps ensemble steps under each of six
 * candidate tilings applied to every run (target blocks 1184, 148, 592 or
 * 2368 per run, or 1184 or 4736 times the run's share of the ensemble's
 * particles; 512 to 2048 particles per block at least), in context, with
 * all runs on the GPU together, and keeps the fastest; *choice (may be
 * NULL) receives its index.  It advances every run by 6 x (trial_steps + 1)
 * steps. */
typedef struct pcg_ensemble pcg_ensemble;
int pcg_ensemble_create(pcg_handle* const* runs, int n, int threads, pcg_ensemble** out);
int pcg_ensemble_step(pcg_ensemble* e, int nsteps, float* device_ms);
int pcg_ensemble_autotune(pcg_ensemble* e, int trial_steps, int* choice);
int pcg_ensemble_destroy(pcg_ensemble* e);

/* Graph mode of an ensemble (no reference counterpart).  With on != 0, each
 * later pcg_ensemble_step(e, nsteps, ...) captures nsteps steps of every run
 * from the calling thread into one CUDA graph, the runs as parallel
 * branches forked from and joined to the ensemble's own stream, and issues
 * it as one graph launch; *device_ms is then the device time of that
 * launch.  A call before the ensemble's first batch steps directly (the
 * first tile sort of a float species waits for its stream, which a capture
 * cannot).  Each step's host decisions (beam particle counts, re-sorts) are
 * taken at capture as a direct step takes them; the graph of the previous
 * batch is updated in place when the new one has the same nodes, and
 * instantiated anew otherwise.  A step that would wait for the device
 * inside the capture (a species at its capacity, dropping dead slots) fails
 * the capture: the call returns its error, the runs' host state has moved
 * on without their kernels, and every later call returns PCG_ERR_STATE.
 * pcg_ensemble_graph_info reports the last graph's node count and the host
 * time (ms) of its capture and instantiation or update; either pointer may
 * be NULL. */
int pcg_ensemble_set_graph(pcg_ensemble* e, int on);
int pcg_ensemble_graph_info(pcg_ensemble* e, unsigned long long* nodes, float* capture_ms);

/* SpecieP's diagnostic maps of species `slot` (specieP.cpp:665-839:
 * calc_density, calc_temperature, calc_energy, calc_momentum) into host
 * `out`: (nr+4) x (nz+4) doubles laid out as the fields, three such grids
 * (r, phi, z) for PCG_MAP_MOMENTUM.  Values spread over the nodes as
 * weight_cylindrical does (weighter.hpp:27-130); temperature and energy are
 * in eV on the interior nodes, momentum is p / n there.  Under
 * PCG_QUIRKS_REFERENCE gamma enters a particle's momentum only below
 * REL_LIMIT = 5e7 m/s (specieP.cpp:729, 764) and the temperature reads the
 * absolute-momentum map of this species' last PCG_MAP_ENERGY call (its
 * calc_momentum_w does not make one; before any call the reference reads
 * an uninitialised grid, here zeros); PCG_QUIRKS_FIXED applies gamma at
 * every speed and makes the map afresh. */
#define PCG_MAP_DENSITY 0
#define PCG_MAP_TEMPERATURE 1
#define PCG_MAP_ENERGY 2
#define PCG_MAP_MOMENTUM 3
int pcg_species_map(pcg_handle* h, int slot, int which, double* out);

/* Collisions inside pcg_step: every step then runs one pass of the chosen
 * operator between the push and the move, as SMB::advance_particles does
 * (SMB.cpp:1289-1293, Domain::collide): the step pushes every species,
 * collides, then moves, reflects, binds and deposits.  The same order by
 * stages: PCG_STAGE_PUSH, pcg_collide (or pcg_collide_learned), then
 * PCG_STAGE_DUMP_OLD onwards. */
#define PCG_COLLISIONS_NONE 0
#define PCG_COLLISIONS_BINARY 1
#define PCG_COLLISIONS_LEARNED 2
int pcg_set_collisions(pcg_handle* h, int mode);

/* Villasenor-Buneman current of one species, double precision, that
 * allocates no device memory.  No counterpart in the reference: it exists
 * for callers that may not call cudaMalloc (a host code that owns and
 * pre-partitions the device memory, or one that cannot afford cudaMalloc's
 * device synchronisation inside its step loop).  All arrays are the
 * caller's device memory: positions r, z (new) and r_old, z_old (before the
 * move), v_phi and weights of n particles, and the three J grids of
 * (nr+4) x (nz+4) doubles with the 2-cell halo, which receive the deposit
 * exactly as PCG_STAGE_CURRENT does for a single species (the halo is
 * cleared, the interior accumulates).  Work is queued on `stream`
 * (cudaStream_t, 0 for the default stream); when move_errors is not NULL
 * the call waits for the stream and stores the number of particles whose
 * current was skipped for moving more than one cell.
 * Scratch lives in a fixed device array shared by every call on a device:
 * grids with (nr+4)*(nz+4) > PCG_NOALLOC_MAX_NODES return PCG_ERR_CAPACITY;
 * each call clears the scratch first, so calls that overlap on the GPU
 * (different streams, no ordering) race.  The first call on each device
 * (and the first after a cudaDeviceReset) looks up the scratch address;
 * under lazy module loading (the CUDA default) that lookup also loads the
 * library's device code, which reserves the 2 MiB array and may
 * synchronise.  So make one warm-up call on each device before the region
 * that must not allocate, and before any stream capture on that device, or
 * run with CUDA_MODULE_LOADING=EAGER.  A non-NULL move_errors while
 * `stream` is being captured returns PCG_ERR_STATE: its read-back would
 * synchronise the stream. */
#define PCG_NOALLOC_MAX_NODES 262144
int pcg_current_vb_f64_noalloc(int nr, int nz, double radius, double longitude, double dt,
                               size_t n, double charge_e, const double* r, const double* z,
                               const double* r_old, const double* z_old, const double* vphi,
                               const double* w, double* j_r, double* j_phi, double* j_z,
                               int quirks, void* stream, unsigned long long* move_errors);

int pcg_set_field(pcg_handle* h, int which, const double* src);
int pcg_export_field(pcg_handle* h, int which, double* dst);

/* Array columns [c0, c1) of a field grid, 0 <= c0 < c1 <= nz+4 (column
 * c holds the nodes of cell k = c - 2 along z): (nr+4) x (c1-c0) doubles,
 * row-major, copied from or to the device without touching the other
 * columns.  These replace whole-array copies in an exchange of ghost
 * columns between domains split along z, the counterpart of the
 * reference's overlap copies (SMB::field_e_overlay, field_h_overlay,
 * current_overlay, SMB.cpp:566-1229). */
int pcg_get_field_columns(pcg_handle* h, int which, int c0, int c1, double* dst);
/* (dst and src, and the particle arrays of pcg_import_species,
 * pcg_append_species and pcg_export_species_range, may also be device
 * memory on the handle's GPU: the copies then stay on the device.  Device
 * arrays must be complete when the call is made, and are free for reuse
 * when it returns.) */
int pcg_set_field_columns(pcg_handle* h, int which, int c0, int c1, const double* src);

/* The live particles of a species with lo <= z < hi (z in m, the domain's
 * coordinates; -inf and +inf are allowed), in slot order:
 * pcg_export_species_range writes their r, z, v_r, v_phi, v_z, w (a null
 * array is skipped) and *n = their count; with cap < count it writes
 * nothing else and returns PCG_ERR_CAPACITY.  pcg_keep_species_range
 * removes every live particle outside [lo, hi); its slots become dead and
 * are reclaimed by the next compaction.  The two use the same z of a
 * particle (the float layout's cell and offset in double), so one band's
 * export and the complementary keep split the particles exactly.  With
 * pcg_append_species they hand particles between domains split along z,
 * the counterpart of SMB::particles_runaway_collector (SMB.cpp:194-564). */
int pcg_export_species_range(pcg_handle* h, int slot, double lo, double hi, size_t cap, double* r,
                             double* z, double* vr, double* vphi, double* vz, double* w, size_t* n);
int pcg_keep_species_range(pcg_handle* h, int slot, double lo, double hi);

/* The same hand-over from one handle to another on the device, with only
 * counts crossing to the host; the handles may be on one GPU or on two (a
 * peer copy, over NVLink where the GPUs reach each other).
 * pcg_transfer_species_range selects src's live particles of `slot` with
 * lo <= z < hi as pcg_export_species_range does, subtracts `shift` from
 * their z (dst's coordinates), and appends them to dst's species dst_slot
 * (append = 1; dead slots are reclaimed first as pcg_append_species does)
 * or replaces that species' particles with them (append = 0); *n = their
 * count.  It waits for src's queued work (the selection's count), not for
 * dst's.  pcg_copy_field_columns copies the array columns [c0, c1) of
 * src's field `which` (PCG_FIELD_ALL: all twelve) into dst's columns
 * [g0, g0 + c1 - c0); both handles need the same precision and nr.  In
 * both, the copy runs after the work queued on both handles before the
 * call, and the work queued on either after the call runs after the copy;
 * the host does not wait for it. */
#define PCG_FIELD_ALL (-1)
int pcg_transfer_species_range(pcg_handle* src, int slot, double lo, double hi, double shift,
                               pcg_handle* dst, int dst_slot, int append, size_t* n);
/* Several bands of src at once, with one wait for all their counts: every
 * band is selected from src's particles as they are at the call, then the
 * bands are appended or imported in order (a destination slot that gets
 * two bands takes the first with append = 0 to replace, the second with
 * append = 1).  counts (may be NULL) receives each band's count.  A band's
 * destination must not be src itself. */
typedef struct pcg_band {
  int slot;           /* src species */
  double lo, hi;      /* lo <= z < hi, src coordinates */
  double shift;       /* subtracted from z: dst coordinates */
  pcg_handle* dst;
  int dst_slot;
  int append;
} pcg_band;
int pcg_transfer_species_bands(pcg_handle* src, int nbands, const pcg_band* bands, size_t* counts);
int pcg_copy_field_columns(pcg_handle* src, int which, int c0, int c1, pcg_handle* dst, int g0);

int pcg_stage(pcg_handle* h, int stage);
int pcg_step(pcg_handle* h, int nsteps);
int pcg_synchronize(pcg_handle* h);
/* The status of the steps queued before the last call of pcg_step_status,
 * read without waiting for the steps queued since (no reference counterpart:
 * the reference aborts inside the step).  Each call queues a copy of the
 * device status block to pinned host memory and returns the block the
 * previous call queued, waiting for that copy only; a loop of pcg_step +
 * pcg_step_status therefore reads every step's status, one step late, while
 * the GPU keeps a step queued.  pcg_synchronize reads the current one.
 * pcg_import_species and pcg_append_species likewise wait for their own
 * host-to-device copies, not for the steps queued before them. */
int pcg_step_status(pcg_handle* h);
int pcg_diag(pcg_handle* h, pcg_diagnostics* out);
/* The handle's cudaStream_t, for callers that time or order work on it. */
int pcg_get_stream(pcg_handle* h, void** stream);
/* The handle's GPU (pcg_config.device).  Every call on a handle runs with
 * that GPU current and restores the caller's current device on return, so
 * one host thread may drive handles on several GPUs. */
int pcg_get_device(pcg_handle* h, int* device);

#ifdef __cplusplus
}
#endif
#endif
