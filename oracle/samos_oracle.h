/*
 * samos_oracle.h -- CPU oracle for the SAMoS particle-dynamics hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * C++ loops (SAMoS, src/...) in the reference's own order of operations.  It
 * is the checker for the CUDA path: only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load it.  The product never calls it.
 *
 * Parity status: PARITY UNPINNED.  The reference cannot be compiled here (it
 * needs Boost, GSL and CGAL, none of which are installed) and its tree holds
 * no tests or golden vectors, so no reference output exists to pin against.
 * The oracle is checked against hand-derived known answers instead
 * (tests/test_oracle_cpu.py).
 *
 * Noise: the reference draws from GSL's default generator, which is not
 * available.  Both this oracle and the CUDA path read one project-defined
 * counter-based Gaussian stream (Philox-4x32-10, Salmon et al. SC'11, one
 * block per draw, Box-Muller transform with project-written log and cos),
 * consumed in the reference's draw order: RNG object = (seed, counter),
 * one counter value per draw.
 *
 * Build: oracle/build.sh (gcc -O2 -ffp-contract=off, no fast-math).
 */
#ifndef SAMOS_ORACLE_H
#define SAMOS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* component kinds (same numbering as include/samos_gpu.h) */
enum { OR_PAIR_SOFT = 0, OR_PAIR_LJ = 1, OR_PAIR_MORSE = 2, OR_PAIR_GAUSSIAN = 3 };
enum { OR_ALIGN_POLAR = 0, OR_ALIGN_NEMATIC = 1, OR_ALIGN_VICSEK = 2 };
enum { OR_EXT_SELF_PROPULSION = 0 };
enum { OR_CONS_NONE = 0, OR_CONS_PLANE = 1, OR_CONS_SPHERE = 2, OR_CONS_CYLINDER = 3, OR_CONS_TORUS = 4,
       OR_CONS_ELLIPSOID = 5, OR_CONS_PEANUT = 6, OR_CONS_GYROID = 7, OR_CONS_HOURGLASS = 8,
       OR_CONS_GAUSSIAN_BUMP = 9, OR_CONS_SLAB = 10, OR_CONS_PLANE_WALLS = 11, OR_CONS_TETRAHEDRON = 12 };
enum { OR_INT_BROWNIAN = 0, OR_INT_BROWNIAN_POS = 1, OR_INT_BROWNIAN_ALIGN = 2,
       OR_INT_LANGEVIN = 3, OR_INT_FIRE = 4, OR_INT_NVE = 5, OR_INT_VICSEK = 6 };
enum { OR_VALUE_CONSTANT = 0, OR_VALUE_LINEAR = 1 };
enum { OR_LANGEVIN_BAOAB = 0, OR_LANGEVIN_SPV = 1, OR_LANGEVIN_BBK = 2 };

/* number of parameters per type pair in a pair-potential table */
#define OR_PAIR_NPARAM 8
/* integrator parameter vector (index meaning per kind, see samos_oracle.c) */
#define OR_INT_NPARAM 16

typedef struct or_system or_system;

/* noise stream (shared definition with the CUDA path) */
double or_noise_gauss(uint32_t seed, uint64_t counter);
double or_noise_uniform(uint32_t seed, uint64_t counter);
void   or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
double or_noise_log(double x);
double or_noise_cos2pi(double u);

or_system* or_create(int n, int ntypes);
void       or_destroy(or_system* s);
int        or_size(const or_system* s);
double*    or_field(or_system* s, const char* name);
int*       or_ifield(or_system* s, const char* name);

void   or_set_box(or_system* s, double lx, double ly, double lz, int periodic);
void   or_set_timestep(or_system* s, double dt);

/* neighbour list: created and built at once, like NeighbourList's ctor */
int    or_set_nlist(or_system* s, double rcut, double pad);
int    or_build_nlist(or_system* s);
int    or_nlist_uses_cells(const or_system* s);
/* copy the half list in the reference's storage order; returns pair count
   (or -count if cap is too small) */
int    or_get_pairs(const or_system* s, int* out_i, int* out_j, int cap);
int    or_nlist_builds(const or_system* s);

/* value object: kind, min_val, max_val, steps */
int    or_add_pair(or_system* s, int kind, const double* global_params,
                   const double* table, int use_particle_radii, int phase_in,
                   int shifted, int has_pair_params, const double* phase_value);
int    or_add_align(or_system* s, int kind, double J, double rcut,
                    const double* table, int has_pair_params);
int    or_add_external(or_system* s, int kind, double alpha,
                       const double* type_alpha, int has_params);
/* params: plane {zpos, unlimited}, sphere {r}, cylinder {r}, torus {c, -, .., a
   in [7]}, ellipsoid {a, -, .., b in [7], c in [8]}, peanut {a, .., b in [7]},
   gyroid {} (the box is its period), hourglass {R, .., A in [7], n in [8]},
   gaussian_bump {A, .., a in [7], b in [8]}, slab {z_lo, .., z_hi in [7]},
   plane_walls {l, moved to the box edge if beyond it}, tetrahedron {scale, ..,
   value in [7]}; base {maxiter, tol, rescale,
   rescale_steps, rescale_freq} in params[2..6].  Returns -1 for parameters
   the reference constructor rejects (peanut b <= a). */
int    or_add_constraint(or_system* s, int kind, const double* params);
int    or_add_integrator(or_system* s, int kind, const double* params,
                         const double* temperature_value);
int    or_integrator_state(or_system* s, int idx, double* out /* 8 */);
/* particle groups: group 1..OR_MAX_GROUPS-1 gets the particles with
   member[i] != 0 (index order); an integrator then moves only its group */
#define OR_MAX_GROUPS 8
int    or_define_group(or_system* s, int group, const unsigned char* member);
int    or_set_integrator_group(or_system* s, int idx, int group);

/* one force + torque evaluation (reset, potentials, aligners) */
void   or_compute(or_system* s, double dt);
void   or_enforce_all(or_system* s);
/* `run steps` of samos.cpp: steps+1 integration steps */
int    or_run(or_system* s, int steps);
/* run until every FIRE integrator reports convergence or max_steps */
int    or_run_until_converged(or_system* s, int max_steps);
double or_pair_energy(const or_system* s, int idx);
double or_align_energy(const or_system* s, int idx);
double or_total_potential_energy(const or_system* s);

#ifdef __cplusplus
}
#endif
#endif
