/*
 * samos_gpu.h -- C ABI of the B200 (sm_100a) SAMoS particle-dynamics engine.
 *
 * One handle owns a packed ensemble of R independent replicas (R = 1 for an
 * ordinary `samos` run) resident in HBM as structure-of-arrays FP64 buffers.
 * Components are configured with the same kinds, parameter meanings and
 * ordering rules as SAMoS's class factories; every entry point below names
 * the reference interface it replaces (paths relative to the SAMoS tree).
 *
 * Conventions: every call returns SG_OK (0) or a negative SG_ERR_* code; no
 * exception crosses the ABI; sg_last_error() gives a one-line reason.  All
 * pointers are host pointers unless the name says _device.  A handle is not
 * thread-safe (the reference is single-threaded, src/samos.cpp:878-970).
 */
#ifndef SAMOS_GPU_H
#define SAMOS_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define SG_OK               0
#define SG_ERR_ARG         -1   /* bad argument / unknown field or kind      */
#define SG_ERR_CUDA        -2   /* CUDA runtime error                        */
#define SG_ERR_NOMEM       -3   /* device allocation failed                  */
#define SG_ERR_STATE       -4   /* call out of order (e.g. run before nlist) */
#define SG_ERR_OVERFLOW    -5   /* neighbour capacity exceeded after regrow  */
#define SG_ERR_NONFINITE   -6   /* NaN/Inf detected in the particle state    */
#define SG_ERR_UNSUPPORTED -7   /* configuration outside the GPU path        */
#define SG_ERR_TIMEOUT     -8   /* a bounded device wait gave up             */

/* ---- component kinds (factory names of src/utils/register_*.cpp) -------- */
enum { SG_PAIR_SOFT = 0, SG_PAIR_LJ = 1, SG_PAIR_MORSE = 2, SG_PAIR_GAUSSIAN = 3 };
enum { SG_ALIGN_POLAR = 0, SG_ALIGN_NEMATIC = 1, SG_ALIGN_VICSEK = 2 };
enum { SG_EXT_SELF_PROPULSION = 0 };
enum { SG_CONS_NONE = 0, SG_CONS_PLANE = 1, SG_CONS_SPHERE = 2, SG_CONS_CYLINDER = 3, SG_CONS_TORUS = 4,
       SG_CONS_ELLIPSOID = 5, SG_CONS_PEANUT = 6, SG_CONS_GYROID = 7, SG_CONS_HOURGLASS = 8,
       SG_CONS_GAUSSIAN_BUMP = 9, SG_CONS_SLAB = 10, SG_CONS_PLANE_WALLS = 11, SG_CONS_TETRAHEDRON = 12 };
enum { SG_INT_BROWNIAN = 0, SG_INT_BROWNIAN_POS = 1, SG_INT_BROWNIAN_ALIGN = 2,
       SG_INT_LANGEVIN = 3, SG_INT_FIRE = 4, SG_INT_NVE = 5, SG_INT_VICSEK = 6 };
enum { SG_VALUE_CONSTANT = 0, SG_VALUE_LINEAR = 1 };
enum { SG_LANGEVIN_BAOAB = 0, SG_LANGEVIN_SPV = 1, SG_LANGEVIN_BBK = 2 };

#define SG_PAIR_NPARAM 8
#define SG_INT_NPARAM 16
#define SG_MAX_TYPES 16

typedef struct sg_system sg_system;

typedef struct {
  int64_t steps_done;      /* integration steps executed by the last sg_run  */
  int64_t nlist_builds;    /* neighbour-list builds during the last sg_run   */
  int64_t kernel_launches; /* engine kernels launched during the last sg_run */
  int32_t max_neighbours;  /* largest full-list neighbour count seen         */
  int32_t status;          /* device status word (0 = clean)                 */
  double  device_ms;       /* CUDA-event time of the whole call on its stream */
  double  step_kernel_ms;  /* summed event time of the dominant step kernel   */
  int64_t step_kernels;    /* launches timed in step_kernel_ms (profiling on) */
  double  rebuild_ms;      /* CUDA-event time spent in neighbour-list rebuilds */
} sg_run_stats;

/* ---- lifetime ------------------------------------------------------------
 * Replaces System::System (src/system/system.cpp:64-452) as the owner of the
 * particle store: n_particles[r] particles of ntypes types per replica.     */
int  sg_create(int n_replicas, const int32_t* n_particles, int ntypes, sg_system** out);
/* Select the CUDA device that the next sg_create binds (per calling thread);
 * a handle keeps its device for all later calls.                           */
int  sg_set_device(int device);
int  sg_destroy(sg_system* s);
const char* sg_error_string(int code);
const char* sg_last_error(const sg_system* s);

/* Box(lx,ly,lz) centred at the origin, src/system/box.hpp:56-62; periodic
 * flag of `box periodic|fixed` (src/samos.cpp:205-230).                      */
int  sg_set_box(sg_system* s, int replica, double lx, double ly, double lz, int periodic);
/* `timestep dt` -> System::set_integrator_step (src/samos.cpp:1348)          */
int  sg_set_timestep(sg_system* s, double dt);

/* ---- particle data -------------------------------------------------------
 * Field names follow Particle (src/system/particle.hpp:257-306): doubles
 * "x","y","z","vx","vy","vz","fx","fy","fz","tau_x","tau_y","tau_z","nx",
 * "ny","nz","Nx","Ny","Nz","omega","age","radius","mass"; int32 "type",
 * "ix","iy","iz".  Arrays are in particle-id order (length n_particles[r]). */
int  sg_upload(sg_system* s, int replica, const char* field, const void* host);
int  sg_download(sg_system* s, int replica, const char* field, void* host);
/* Several fields of one replica in one call (System's reader / a dump's
 * loop over Particle fields, src/system/system.cpp:76-450,
 * src/dump/dump.cpp:504-708): the same as one sg_upload / sg_download per
 * field, but every copy is enqueued back to back and the call waits once.
 * From page-locked host arrays (sg_host_alloc) the copies run at the link's
 * bandwidth.                                                                */
int  sg_upload_fields(sg_system* s, int replica, int nfields, const char* const* fields,
                      const void* const* hosts);
int  sg_download_fields(sg_system* s, int replica, int nfields, const char* const* fields,
                        void* const* hosts);
/* Page-locked host memory for the arrays given to sg_upload / sg_download:
 * copies from and to it run at the link's speed, where pageable arrays go
 * through the driver's staging buffers (and a fresh pageable destination is
 * faulted in page by page during the copy).  Plain cudaMallocHost /
 * cudaFreeHost; no reference counterpart (host plumbing).                   */
int  sg_host_alloc(int64_t bytes, void** ptr);
int  sg_host_free(void* ptr);

/* ---- neighbour list ------------------------------------------------------
 * NeighbourList(sys, msg, rcut, pad) (src/system/neighbour_list.hpp:124-217)
 * including the immediate build; build() / build_cell() / build_nsq()
 * (src/system/neighbour_list.cpp:117-273).                                  */
int  sg_set_nlist(sg_system* s, double rcut, double pad);
int  sg_build_nlist(sg_system* s);
/* Half list of replica r as (i<j) id pairs in the reference's list order
 * (NeighbourList::get_neighbours, neighbour_list.hpp:237).                  */
int  sg_get_pairs(sg_system* s, int replica, int32_t* out_i, int32_t* out_j,
                  int64_t cap, int64_t* n_pairs);

/* ---- components ----------------------------------------------------------
 * Pair potential (factory pair_potentials[name], register_pair_potentials.cpp
 * :35-69; parameters pair_soft/lj/morse/gaussian_potential.hpp).  `global`
 * holds the conf-level parameters, `table` (ntypes*ntypes*SG_PAIR_NPARAM,
 * may be NULL) the per-type-pair values of set_pair_parameters (pair_param
 * command).  phase_value = {kind, min_val, max_val, steps} of the phase-in
 * Value object.  Parameter slots: soft {k,a}; lj {epsilon,sigma,rcut};
 * morse {D,a,re,rcut}; gaussian {A,B,alpha,beta,rA,rB,rcut}.               */
int  sg_add_pair(sg_system* s, int kind, const double* global, const double* table,
                 int use_particle_radii, int phase_in, int shifted, int has_pair_params,
                 const double* phase_value);
/* Pair aligner (register_pair_aligners.cpp:35-41): polar / nematic / vicsek
 * with global J and rcut; table = ntypes*ntypes*{J, rcut} of align_param.   */
int  sg_add_align(sg_system* s, int kind, double J, double rcut, const double* table,
                  int has_pair_params);
/* External potential self_propulsion {alpha} with optional per-type alpha
 * (external_self_propulsion.cpp:33-50).                                     */
int  sg_add_external(sg_system* s, int kind, double alpha, const double* type_alpha,
                     int has_params);
/* Constraint (register_constraints.cpp:35-61): params =
 * {plane: zpos | sphere: r | cylinder: r | torus: c | ellipsoid: a |
 *  peanut: a | hourglass: R | gaussian_bump: A | slab: z_lo | walls: l |
 *  tetrahedron: scale,
 *  plane: unlimited, maxiter, tol, rescale, rescale_steps, rescale_freq,
 *  torus: a | ellipsoid: b | peanut: b | hourglass: A | gaussian_bump: a^2 |
 *  slab: z_hi | tetrahedron: value, ellipsoid: c | hourglass: n |
 *  gaussian_bump: b^2} (9 values; the bump's widths squared, as its
 *  constructor stores them, constraint_gaussian_bump.hpp;
 * gyroid takes none, its period is the box; a walls l beyond the box
 * is moved to its edge, constraint_plane_walls.hpp:64-71).  The implicit surfaces (torus and after)
 * project with Constraint::enforce's SHAKE iteration, constraint.cpp:40-87.
 * Peanut needs b > a (constraint_peanut.hpp:84-88; rejected here), an
 * explicitly given hourglass A at most R (constraint_hourglass.hpp:85; the
 * hosts check it).  Enforced on every particle at once like
 * src/samos.cpp:518-522.  rescale / rescale_steps / rescale_freq scale the
 * sphere and cylinder radius and the tetrahedron scale by
 * rescale^(freq/steps) every freq global steps (constraint_sphere.cpp:87-104,
 * constraint_cylinder.cpp:79-96, constraint_tetrahedron.cpp:88-109), at the
 * top of the step, then rebuild the lists (samos.cpp:882-886); a run with a
 * rescaling constraint allows no second constraint.  The plane's box
 * rescale is refused (SG_ERR_UNSUPPORTED); the other kinds ignore the
 * parameters, as the base class's rescale does (constraint.hpp:144).        */
int  sg_add_constraint(sg_system* s, int kind, const double* params);
/* As sg_add_constraint, with params[0] (plane zpos / sphere r) given per
 * replica in value0[n_replicas] before the immediate enforce, so each
 * replica is projected exactly as its own single-system run would be.      */
int  sg_add_constraint_per_replica(sg_system* s, int kind, const double* params, const double* value0);
/* Integrator (register_integrators.cpp:35-55).  params[SG_INT_NPARAM]:
 *  brownian       : 0 dt, 1 v0, 2 nu, 3 mu, 4 mur, 5 seed, 6 nematic, 7 tau, 8 velocity_align
 *  brownian_pos   : 0 dt, 3 mu, 5 seed
 *  brownian_align : 0 dt, 2 nu, 4 mur, 5 seed, 6 nematic, 7 tau
 *  langevin       : 0 dt, 5 seed, 9 gamma, 10 method
 *  fire           : 0 dt, 1 alpha, 2 alpha_scale, 3 f_tolerance, 4 e_tolerance,
 *                   6 dt_inc, 7 dt_dec, 8 dt_max, 9 min_neg_steps, 11 fmax_tolerance
 *  nve            : 0 dt, 12 has_limit, 13 limit, 14 has_angle_limit, 15 angle_limit
 *                   (integrator_nve.hpp:59-75)
 *  vicsek         : 0 dt, 1 v0, 2 eta, 3 mu, 5 seed (integrator_vicsek.hpp:55-105)
 * temperature_value = {kind, min_val, max_val, steps} (Value, value.hpp).
 * Integrators must be added in std::map key order (type + "_" + group).     */
int  sg_add_integrator(sg_system* s, int kind, const double* params,
                       const double* temperature_value);

/* Multi-segment conf files (src/samos.cpp:864-972 runs once per `run`
 * command with whatever the plugin maps hold at that point).
 * sg_insert_integrator: like sg_add_integrator, at position `pos` of the
 *   integrator sequence, so the host can keep std::map key order
 *   (samos.cpp:899-900) when integrators are added between runs.
 * sg_disable_integrator: the `disable` command (samos.cpp, "disable"
 *   branch: the integrator is erased from the map); later integrators keep
 *   their noise streams.
 * sg_clear_forces: drop every pair potential, aligner and external
 *   potential (they hold no state); the host re-adds the current set in map
 *   order before a run.                                                   */
int  sg_insert_integrator(sg_system* s, int pos, int kind, const double* params, const double* temperature_value);
int  sg_disable_integrator(sg_system* s, int index);
/* `group <name> {...}` (samos.cpp:1108-1140, System::make_group,
 * system.cpp:462-572): group index 1..7 of replica r gets the particles with
 * member[id] != 0 (the host evaluates type / not_type / r_* / x_*... on its
 * particles); their order in the group is their index order.               */
int  sg_define_group(sg_system* s, int replica, int group, const uint8_t* member);
/* An integrator's `group = <name>` (integrator.hpp:67-109): the integrator at
 * map position `index` moves only the members of `group` (0 = all), drawing
 * its noise in group order.  brownian, brownian_pos, brownian_align and
 * vicsek take groups here; the others act on "all".                         */
int  sg_set_integrator_group(sg_system* s, int index, int group);
int  sg_clear_forces(sg_system* s);

/* Per-replica override of one numeric parameter (batched ensembles):
 * cls 0 pair global, 1 aligner {0:J,1:rcut}, 2 external alpha,
 * 3 constraint {0: zpos|r}, 4 integrator params[] (slot 5 = seed).          */
int  sg_set_replica_param(sg_system* s, int replica, int cls, int comp, int slot, double value);

/* ---- execution -----------------------------------------------------------
 * sg_compute: reset_forces/reset_torques + Potential::compute(dt) +
 * Aligner::compute() (potential.cpp:36-52, aligner.cpp:35-45) on the current
 * state, no integration.                                                    */
int  sg_compute(sg_system* s, double dt);
/* Constrainer::enforce on every particle (constrainer.hpp:73-77).           */
int  sg_enforce(sg_system* s);
/* `run steps` (src/samos.cpp:864-972): steps+1 integration steps with the
 * skin-triggered neighbour-list rebuilds of samos.cpp:944-966.              */
int  sg_run(sg_system* s, int64_t steps, sg_run_stats* stats);
/* `steps` (>= 1) further integration steps of the current run, with the
 * run-step counter (Value schedules, samos.cpp:881) continuing: a host that
 * reads the state every k steps (dumps, logs: samos.cpp:905-940) splits a
 * `run` into sg_run(k - 1) followed by sg_run_continue(k) calls, with the
 * same results as one sg_run.                                               */
int  sg_run_continue(sg_system* s, int64_t steps, sg_run_stats* stats);
/* The top of the next step up to the dumps and logs (samos.cpp:887-896):
 * the start-of-step constraint enforce is applied now (and not again by the
 * next sg_run / sg_run_continue), so downloads see what the reference's
 * dumps see.  Follow with sg_compute for energies at that point.           */
int  sg_begin_step(sg_system* s);
/* FIRE minimisation driver: run until every replica's FIRE integrator has
 * converged or max_steps integration steps; converged[r] (may be NULL) gets
 * the step count per replica or -1.                                         */
int  sg_minimize(sg_system* s, int64_t max_steps, int64_t* converged, sg_run_stats* stats);
/* Energy of component `comp` of class cls (0 pair, 1 aligner) for replica r
 * from the last force evaluation (PairPotential::get_potential_energy).     */
int  sg_energy(sg_system* s, int replica, int cls, int comp, double* out);
/* FIRE scalars of replica r: {dt, alpha, last_neg, converged, old_energy}.  */
int  sg_fire_state(sg_system* s, int replica, double* out5);
/* Cumulative kernel launches of this handle (for launch accounting).       */
int64_t sg_kernel_launches(const sg_system* s);
/* Time every launch of the dominant per-step kernel with CUDA events on the
 * handle's stream (reported in sg_run_stats.step_kernel_ms).  No reference
 * counterpart (instrumentation).                                            */
int  sg_set_profiling(sg_system* s, int on);
/* Execution path: 0 = automatic (packed hot kernels for a periodic plane or
 * a sphere, specialised when the program is the active-Brownian one),
 * 1 = always the generic structure-of-arrays kernels, 2 = packed kernels
 * without the specialisation.  All give the same results; the switch exists
 * so tests can compare them.  No reference counterpart.                     */
int  sg_set_path(sg_system* s, int path);
/* Kernel variant of the specialised active-Brownian step (0..31: per-particle
 * neighbour sweeps that differ in how far ahead neighbour records are
 * fetched, one or two neighbours per iteration, resident blocks per SM, lane
 * order, where the Gaussian draws are taken and, for a one-replica system,
 * whether the parameters are read from kernel parameter space or a
 * shared-memory copy; a flattened warp-wide sweep; shared-memory staged and
 * tiled sweeps); all variants compute the same bits.  By default the engine's autotuner times every variant on the
 * first steps of a run and keeps the fastest; sg_set_variant pins one
 * (-1 re-enables tuning), sg_get_variant reports the choice (-1 = not yet
 * tuned).  No reference counterpart.                                        */
int  sg_set_variant(sg_system* s, int variant);
int  sg_get_variant(const sg_system* s);
/* Neighbour-list build kernel: 0 = automatic (lanes of a team share one
 * particle's 27-cell stencil when fewer than 2^16 particles are rebuilt,
 * one thread per particle otherwise), 1 = always one thread per particle,
 * 2 = always teams, 3 = cell tiles staged in shared memory for quasi-2-D
 * replicas (cell path, at least 3 cells along x and y, exactly 3 along z;
 * one thread per particle elsewhere; slower than 1 on the plane workloads
 * measured).  All build the same lists.  No reference counterpart.         */
int  sg_set_build(sg_system* s, int mode);
/* Order of FIRE's sums P = sum v.F, |F|^2 and |v|^2 (integrator_fire.cpp:
 * 79-94), whose values steer dt, alpha and the velocity mixing:
 * 0 (default, throughput) = a fixed tree over blocks, deterministic and the
 * same for a replica alone or in an ensemble, but not the reference's order,
 * so iteration counts can differ from the reference's by a few percent;
 * 1 (parity) = one particle at a time in particle-id order, the reference's
 * order, so with fmax_tolerance set FIRE takes the reference's iterations
 * bit for bit (the energy in the reference's own convergence test stays a
 * tree sum).  Costs a sequential pass over each replica per iteration.      */
int  sg_set_fire_order(sg_system* s, int ordered);
/* Generic fused step kernel (programs outside the specialised plane /
 * sphere Brownian kernels: vicsek, curved and implicit constraints, groups,
 * phase-in): the blocks per SM its registers are bounded for, 6 or 8; 0
 * (default) times both on the run's first steps and keeps the faster.
 * Same bits either way.  sg_get_generic_occupancy reports the choice (0 =
 * not yet tuned).  No reference counterpart.                                */
int  sg_set_generic_occupancy(sg_system* s, int blocks_per_sm);
int  sg_get_generic_occupancy(const sg_system* s);

/* ---- device view (for kernels that work on the engine's state) -----------
 * No reference counterpart.  Device pointers into the handle's current
 * structure-of-arrays store (slot order) and neighbour lists, valid until the
 * next call that runs, rebuilds or reconfigures.  Replica r owns slots
 * [offset[r], offset[r] + n[r]); slot k holds particle id[k].  Neighbour q of
 * slot k is slot nb[q * nb_stride + k] for q < nb_cnt[k].  After writing
 * positions through the view call sg_positions_changed(), which rebuilds the
 * neighbour lists before the next step.                                     */
typedef struct {
  double *x_device, *y_device, *z_device, *nx_device, *ny_device, *nz_device;
  double *vx_device, *vy_device, *vz_device, *fx_device, *fy_device, *fz_device;
  const double* radius_device;
  const int32_t *id_device, *nb_device, *nb_cnt_device;
  int32_t *ix_device, *iy_device;
  int32_t nb_stride, slots;
} sg_view;
int  sg_get_view(sg_system* s, sg_view* out);
int  sg_replica_slots(const sg_system* s, int replica, int32_t* offset, int32_t* n);
int  sg_positions_changed(sg_system* s);
/* Particle::coordination after the last list build (neighbour_list.cpp:
 * 185-206, 229-268): the listed neighbours within the sum of the radii at
 * the build positions, per particle id (n_particles[replica] values).     */
int  sg_coordination(sg_system* s, int replica, int32_t* out);
/* cudaMemcpy with direction inferred from the pointers (helper for callers
 * that hold device pointers from a view).                                   */
int  sg_memcpy(void* dst, const void* src, int64_t bytes);

/* ---- learned FIRE warm start (no reference counterpart) ------------------
 * Message-passing network over the engine's neighbour lists (see
 * samos_b200/csrc/sg_ml.cu for the architecture).  All buffers are device
 * memory owned by the caller; box[2*slot] = (Lx, Ly) of the slot's replica,
 * 0 for slots that are not part of the current batch.                      */
int  sg_mlp_param_count(void);
int  sg_mlp_edge_blocks(void);
int  sg_mlp_part_floats(void);
int  sg_mlp_prepare(const float* params, void* W1b16, void* W1bT16, void* Wpq16, void* WpqT16, void* stream);
int  sg_mlp_forward(const sg_view* v, const double* box, double rc, const float* params, const void* W1bT16,
                    const void* WpqT16, void* s16, void* h16, float* PQ, float* disp, void* stream);
int  sg_mlp_backward(const sg_view* v, const double* box, double rc, const float* params, const void* W1b16,
                     const void* Wpq16, const void* s16, const void* h16, const float* PQ, const float* disp,
                     const float* target, float inv_n, float* gPQ, void* gPQ16, float* gh, void* gpre16, float* gs,
                     float* part, float* red, float* loss_part, float* grad, void* stream);
int  sg_mlp_adam(float* params, const float* grad, float* m, float* v, int n, float lr, float beta1, float beta2,
                 float eps, int step, void* stream);
int  sg_mlp_apply(const sg_view* v, const double* box, const float* disp, int32_t* ix, int32_t* iy, void* stream);

/* ---- evaluation without allocation -------------------------------------
 * No counterpart in the reference: an addition of this library for callers
 * that cannot call cudaMalloc -- code running inside another framework's
 * memory pool or under a no-allocation policy, plugins that only receive
 * device pointers from their host application.  Computes the same forces
 * and torques as sg_compute for a single-type program made of one `soft`
 * pair potential {k, a, use_particle_radii} and at most one aligner
 * (align_kind SG_ALIGN_POLAR or SG_ALIGN_NEMATIC, or -1 for none; J and
 * rcut as in pair_align), with neighbours within rcut+pad taken from a cell
 * list in the reference's list order, bit for bit equal to sg_compute.
 * All pointers are DEVICE pointers of n doubles; positions must lie inside
 * the box.  Nothing is allocated: every intermediate array lives in one
 * fixed file-scope device array of sg_compute_static_scratch_bytes() bytes
 * (about 4 MB) that every GPU loading this library holds until exit.  Limits:
 * n <= SG_STATIC_MAX_PARTICLES and int(lx/(rcut+pad))*int(ly/(rcut+pad))*
 * int(lz/(rcut+pad)) <= SG_STATIC_MAX_CELLS, else SG_ERR_ARG.  A particle
 * with more than 64 neighbours on one side of its id gets NaN outputs, and
 * the call counts it: sg_compute_static_overflow reports the count of the
 * last call.  The call is asynchronous on `stream` (NULL = default stream).
 * The first call on a device (and in each further CUDA context a host makes
 * on it) looks up the scratch address there (cudaGetSymbolAddress); make that
 * first call before any stream capture.  All calls share the one scratch
 * array, which keeps the last call's contents: calls whose work overlaps on
 * the GPU (different streams or host threads) race and must be serialised. */
#define SG_STATIC_MAX_PARTICLES 65536
#define SG_STATIC_MAX_CELLS 262144
int  sg_compute_static(int n, double lx, double ly, double lz, int periodic, double rcut, double pad,
                       const double* x_device, const double* y_device, const double* z_device,
                       const double* nx_device, const double* ny_device, const double* nz_device,
                       const double* radius_device, double k_soft, double a_soft,
                       int use_particle_radii, int align_kind, double J, double align_rcut,
                       double* fx_device, double* fy_device, double* fz_device,
                       double* tau_x_device, double* tau_y_device, double* tau_z_device, void* stream);
int64_t sg_compute_static_scratch_bytes(void);
/* Companion of sg_compute_static (no counterpart in the reference either):
 * writes to *count (host memory) how many particles of the last
 * sg_compute_static call on this device had too many neighbours (and NaN
 * outputs); waits for `stream`.  Allocates nothing.                        */
int  sg_compute_static_overflow(int* count, void* stream);

#ifdef __cplusplus
}
#endif
#endif
