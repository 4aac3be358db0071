// sg_device.cuh -- device-side data model and per-particle physics of the
// SAMoS hot path on sm_100a.
//
// Every routine restates one reference routine (paths relative to the SAMoS
// source tree).  The translation unit is compiled with -fmad=false so that no
// a*b+c is contracted into an FMA: together with IEEE-rounded division and
// square root this reproduces the reference's arithmetic term by term (CUDA
// exp/sin/cos aside, which differ from glibc by at most a few ulp).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>
#include <math.h>

namespace sg {

constexpr int MAX_PAIR = 4;
constexpr int MAX_ALIGN = 3;
constexpr int MAX_EXT = 2;
constexpr int MAX_CONS = 4;
constexpr int MAX_INTEG = 5;
constexpr int PAIR_NPARAM = 8;
constexpr int INT_NPARAM = 16;
constexpr int BLOCK = 128;          // particle slots per block; replicas are padded to it

enum { PAIR_SOFT = 0, PAIR_LJ = 1, PAIR_MORSE = 2, PAIR_GAUSSIAN = 3 };
enum { ALIGN_POLAR = 0, ALIGN_NEMATIC = 1, ALIGN_VICSEK = 2 };
enum { CONS_NONE = 0, CONS_PLANE = 1, CONS_SPHERE = 2, CONS_CYLINDER = 3, CONS_TORUS = 4, CONS_ELLIPSOID = 5,
       CONS_PEANUT = 6, CONS_GYROID = 7, CONS_HOURGLASS = 8, CONS_GAUSSIAN_BUMP = 9, CONS_SLAB = 10,
       CONS_PLANE_WALLS = 11, CONS_TETRAHEDRON = 12 };
// surfaces given by an implicit function g = 0 and projected by the base
// class's SHAKE iteration (no enforce of their own in the reference)
__host__ __device__ __forceinline__ bool cons_implicit(int kind) {
  return (kind >= CONS_TORUS && kind <= CONS_GAUSSIAN_BUMP) || kind == CONS_TETRAHEDRON;
}

// ConstraintTetrahedron's four unit charges (constraint_tetrahedron.hpp:42-45),
// scaled by the constraint's scale; the surface is an equipotential of
// sum 1/|r - a_i| (constraint_tetrahedron.cpp:47-80)
__host__ __device__ __forceinline__ void tetra_charge(int i, double s, double& ax, double& ay, double& az) {
  const double h = 0.7071067811865475;
  const double cx = i == 0 ? 1.0 : i == 1 ? -1.0 : 0.0;
  const double cy = i == 2 ? 1.0 : i == 3 ? -1.0 : 0.0;
  const double cz = i < 2 ? -h : h;
  ax = s * cx; ay = s * cy; az = s * cz;
}
enum { INT_BROWNIAN = 0, INT_BROWNIAN_POS = 1, INT_BROWNIAN_ALIGN = 2, INT_LANGEVIN = 3, INT_FIRE = 4, INT_NVE = 5, INT_VICSEK = 6 };
enum { LANGEVIN_BAOAB = 0, LANGEVIN_SPV = 1, LANGEVIN_BBK = 2 };

// device status word bits
enum { ST_OVERFLOW = 1, ST_NONFINITE = 2, ST_TIMEOUT = 4 };

// Value objects, system/value.hpp:115-178
struct Value { int kind; int steps; double min_val, max_val, dv; };

__host__ __device__ inline double value_get(const Value& v, int step) {
  if (v.kind == 0) return v.min_val;
  if (step > v.steps) return v.max_val;
  return v.min_val + (double)step * v.dv;
}

struct PairComp { int kind, use_radii, phase_in, shifted, has_pp; Value phase; const double* table; };
struct AlignComp { int kind, has_pp; const double* table; };
struct ExtComp { int kind, has_params; const double* type_alpha; };
// b2, b3: torus tube radius a; ellipsoid b, c (the first shape parameter is
// per replica, Replica::cons_p); max_iter, tol: the SHAKE projection
struct ConsComp { int kind, unlimited, max_iter, pad; double b2, b3, tol; };
// group: 0 = "all", else the index of a particle group (System::make_group)
// whose members alone the integrator moves, in group order
struct IntegComp { int kind, method, nematic, velocity, group, pad_g; Value temp; };
constexpr int MAX_GROUPS = 8;  // "all" and up to seven defined groups

// The configured component program, passed by value to every kernel.
struct Program {
  int ntypes;
  int npair, nalign, next, ncons, ninteg;
  PairComp pair[MAX_PAIR];
  AlignComp align[MAX_ALIGN];
  ExtComp ext[MAX_EXT];
  ConsComp cons[MAX_CONS];
  IntegComp integ[MAX_INTEG];
};

// Per-replica numeric parameters and geometry (device array).
struct Replica {
  int off, n;                  // first slot, particle count
  int cell_off, ncell;         // cell range in the packed cell arrays
  int cnx, cny, cnz, use_cell; // grid; use_cell = reference cell path, else N^2 order
  int periodic, pad_i;
  double Lx, Ly, Lz, xlo, xhi, ylo, yhi, zlo, zhi;
  double cwx, cwy, cwz;
  double cut2, pad;
  double pair_g[MAX_PAIR][PAIR_NPARAM];
  double align_J[MAX_ALIGN], align_rcut[MAX_ALIGN];
  double ext_alpha[MAX_EXT];
  double cons_p[MAX_CONS];     // plane: zpos; sphere: r
  double integ_p[MAX_INTEG][INT_NPARAM];
  uint32_t seed[MAX_INTEG];
  int gsize[MAX_GROUPS];       // members of each defined group
};

// Per-replica evolving scalars (device array, updated by the tail kernels).
struct Clock {
  int run_step, time_step;
  uint64_t ctr[MAX_INTEG];     // noise counter base per integrator
  double fire_dt, fire_alpha, fire_old_e;
  int fire_last_neg, fire_converged, fire_conv_step;
  int halt;  // batched stepping: set after a step that flagged a rebuild; later step kernels return at once
  double fire_P, fire_F, fire_V, fire_E, fire_Fmax2;
};

// Particle arrays of one buffer set.
struct Dyn {
  double *x, *y, *z, *vx, *vy, *vz, *nx, *ny, *nz;
  double *fx, *fy, *fz, *tx, *ty, *tz, *omega, *age;
  int *ix, *iy, *iz;
};
struct Stat { double *r, *mass; int *type, *id; };
struct NbList { int *nb, *cnt, *lo; int cap; int stride; double *ox, *oy, *oz; };

// 32-byte record (packed particle data of the step kernels, candidate
// records of the list build), moved with one 256-bit access
struct __align__(32) D4 { double x, y, z, w; };

__device__ __forceinline__ D4 ldg4(const D4* p) {
  D4 v;
  asm volatile("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];"
               : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w) : "l"(p));
  return v;
}
__device__ __forceinline__ void stg4(D4* p, const D4& v) {
  asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(v.x), "d"(v.y), "d"(v.z), "d"(v.w)
               : "memory");
}

struct Part {
  double x, y, z, vx, vy, vz, nx, ny, nz, fx, fy, fz, tx, ty, tz, omega, age, r, mass;
  int ix, iy, iz, type, id;
};

__device__ __forceinline__ void load_dyn(const Dyn& d, int k, Part& p) {
  p.x = d.x[k]; p.y = d.y[k]; p.z = d.z[k];
  p.vx = d.vx[k]; p.vy = d.vy[k]; p.vz = d.vz[k];
  p.nx = d.nx[k]; p.ny = d.ny[k]; p.nz = d.nz[k];
  p.fx = d.fx[k]; p.fy = d.fy[k]; p.fz = d.fz[k];
  p.tx = d.tx[k]; p.ty = d.ty[k]; p.tz = d.tz[k];
  p.omega = d.omega[k]; p.age = d.age[k];
  p.ix = d.ix[k]; p.iy = d.iy[k]; p.iz = d.iz[k];
}
// store of a per-particle pass that leaves the torques as they were (the
// constraint enforce and the Langevin / NVE halves), omega and age only when
// the pass writes them: the loads the pass never uses then drop out too
template <bool OMEGA, bool AGE>
__device__ __forceinline__ void store_dyn_moved(const Dyn& d, int k, const Part& p) {
  d.x[k] = p.x; d.y[k] = p.y; d.z[k] = p.z;
  d.vx[k] = p.vx; d.vy[k] = p.vy; d.vz[k] = p.vz;
  d.nx[k] = p.nx; d.ny[k] = p.ny; d.nz[k] = p.nz;
  d.fx[k] = p.fx; d.fy[k] = p.fy; d.fz[k] = p.fz;
  if (OMEGA) d.omega[k] = p.omega;
  if (AGE) d.age[k] = p.age;
  d.ix[k] = p.ix; d.iy[k] = p.iy; d.iz[k] = p.iz;
}
__device__ __forceinline__ void store_dyn(const Dyn& d, int k, const Part& p) {
  d.x[k] = p.x; d.y[k] = p.y; d.z[k] = p.z;
  d.vx[k] = p.vx; d.vy[k] = p.vy; d.vz[k] = p.vz;
  d.nx[k] = p.nx; d.ny[k] = p.ny; d.nz[k] = p.nz;
  d.fx[k] = p.fx; d.fy[k] = p.fy; d.fz[k] = p.fz;
  d.tx[k] = p.tx; d.ty[k] = p.ty; d.tz[k] = p.tz;
  d.omega[k] = p.omega; d.age[k] = p.age;
  d.ix[k] = p.ix; d.iy[k] = p.iy; d.iz[k] = p.iz;
}

// ---------------------------------------------------------------------------
// noise stream: Philox-4x32-10 (Salmon et al., SC'11), one block per draw,
// Box-Muller transform; one counter value per draw.  The same stream is
// restated independently by the CPU oracle.
// ---------------------------------------------------------------------------
constexpr uint32_t NOISE_KEY1 = 0x53414D4Fu;

__host__ __device__ __forceinline__ uint32_t mulhi32(uint32_t a, uint32_t b) {
  return (uint32_t)(((uint64_t)a * (uint64_t)b) >> 32);
}

__host__ __device__ __forceinline__ void philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                uint32_t k0, uint32_t k1, uint32_t out[4]) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint32_t lo0 = 0xD2511F53u * c0, hi0 = mulhi32(0xD2511F53u, c0);
    uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = mulhi32(0xCD9E8D57u, c2);
    uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

__host__ __device__ __forceinline__ double u53(uint32_t a, uint32_t b) {
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

__host__ __device__ __forceinline__ uint64_t dbits(double x) {
#ifdef __CUDA_ARCH__
  return (uint64_t)__double_as_longlong(x);
#else
  uint64_t u; memcpy(&u, &x, sizeof(u)); return u;
#endif
}
__host__ __device__ __forceinline__ double bitsd(uint64_t u) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)u);
#else
  double x; memcpy(&x, &u, sizeof(x)); return x;
#endif
}

// log(x) from log(m) = 2 atanh((m-1)/(m+1)), x = m 2^e, m in [sqrt(1/2), sqrt(2));
// fixed operation order, no FMA (see the oracle's or_noise_log).
__host__ __device__ __forceinline__ double noise_log(double x) {
  uint64_t u = dbits(x);
  int e = (int)((u >> 52) & 0x7ff) - 1023;
  u = (u & 0x000fffffffffffffull) | 0x3ff0000000000000ull;
  double m = bitsd(u);
  if (m > 1.4142135623730951) { m = m * 0.5; e = e + 1; }
  double z = (m - 1.0) / (m + 1.0);
  double z2 = z * z;
  double p = 1.0 / 23.0;
  p = p * z2 + 1.0 / 21.0;
  p = p * z2 + 1.0 / 19.0;
  p = p * z2 + 1.0 / 17.0;
  p = p * z2 + 1.0 / 15.0;
  p = p * z2 + 1.0 / 13.0;
  p = p * z2 + 1.0 / 11.0;
  p = p * z2 + 1.0 / 9.0;
  p = p * z2 + 1.0 / 7.0;
  p = p * z2 + 1.0 / 5.0;
  p = p * z2 + 1.0 / 3.0;
  double lm = 2.0 * z + 2.0 * z * (z2 * p);
  double de = (double)e;
  const double LN2_HI = 6.93147180369123816490e-01;
  const double LN2_LO = 1.90821492927058770002e-10;
  return (de * LN2_HI + lm) + de * LN2_LO;
}

// cos(2 pi u), u in [0,1) to 53 bits: exact quadrant split of 4u, exact
// reflection to g in [0,1/2], Taylor polynomials of sin (to x^15) / cos (to
// x^16) at x = g pi/2 (same sequence as the oracle's cos2pi).
__host__ __device__ __forceinline__ double noise_cos2pi(double u) {
  double t = u * 4.0;
  int q = (int)t;
  double f = t - (double)q;
  int use_sin = q & 1;
  double g = f;
  if (f > 0.5) { g = 1.0 - f; use_sin = !use_sin; }
  double x = g * 1.5707963267948966;
  double x2 = x * x;
  double v;
  if (use_sin) {
    double p = -1.0 / 1307674368000.0;
    p = p * x2 + 1.0 / 6227020800.0;
    p = p * x2 - 1.0 / 39916800.0;
    p = p * x2 + 1.0 / 362880.0;
    p = p * x2 - 1.0 / 5040.0;
    p = p * x2 + 1.0 / 120.0;
    p = p * x2 - 1.0 / 6.0;
    v = x + x * (x2 * p);
  } else {
    double p = 1.0 / 20922789888000.0;
    p = p * x2 - 1.0 / 87178291200.0;
    p = p * x2 + 1.0 / 479001600.0;
    p = p * x2 - 1.0 / 3628800.0;
    p = p * x2 + 1.0 / 40320.0;
    p = p * x2 - 1.0 / 720.0;
    p = p * x2 + 1.0 / 24.0;
    p = p * x2 - 0.5;
    v = 1.0 + x2 * p;
  }
  return (q == 1 || q == 2) ? -v : v;
}

// standard normal draw `counter` of stream `seed`: Box-Muller on one Philox
// block, g = sqrt(-2 ln u1) cos(2 pi u2), u1 in (0,1], u2 in [0,1)
__host__ __device__ __forceinline__ double noise_gauss(uint32_t seed, uint64_t counter) {
  uint32_t r[4];
  philox((uint32_t)counter, (uint32_t)(counter >> 32), 0u, 0u, seed, NOISE_KEY1, r);
  const double u1 = u53(r[0], r[1]) + (1.0 / 9007199254740992.0);
  const double u2 = u53(r[2], r[3]);
  return sqrt(-2.0 * noise_log(u1)) * noise_cos2pi(u2);
}

__host__ __device__ __forceinline__ double noise_uniform(uint32_t seed, uint64_t counter) {
  uint32_t r[4];
  philox((uint32_t)counter, (uint32_t)(counter >> 32), 0u, 1u, seed, NOISE_KEY1, r);
  return u53(r[0], r[1]);
}

// ---------------------------------------------------------------------------
// periodic box, system/system.cpp:1083-1154
// ---------------------------------------------------------------------------
__device__ __forceinline__ void apply_periodic(const Replica& R, double& dx, double& dy, double& dz) {
  if (R.periodic) {
    if (dx > R.xhi) dx -= R.Lx; else if (dx < R.xlo) dx += R.Lx;
    if (dy > R.yhi) dy -= R.Ly; else if (dy < R.ylo) dy += R.Ly;
    if (dz > R.zhi) dz -= R.Lz; else if (dz < R.zlo) dz += R.Lz;
  }
}

__device__ __forceinline__ void enforce_periodic(const Replica& R, Part& p) {
  if (R.periodic) {
    if (p.x <= R.xlo) { p.x += R.Lx; p.ix--; } else if (p.x > R.xhi) { p.x -= R.Lx; p.ix++; }
    if (p.y <= R.ylo) { p.y += R.Ly; p.iy--; } else if (p.y > R.yhi) { p.y -= R.Ly; p.iy++; }
    if (p.z <= R.zlo) { p.z += R.Lz; p.iz--; } else if (p.z > R.zhi) { p.z -= R.Lz; p.iz++; }
  }
}

// ---------------------------------------------------------------------------
// constraints
// ---------------------------------------------------------------------------
// ConstraintPlane::enforce, constraints/constraint_plane.cpp:36-89
__device__ __forceinline__ void plane_enforce(const Replica& R, double zpos, int unlimited, Part& p) {
  double xlo = -0.5 * R.Lx, xhi = 0.5 * R.Lx;
  double ylo = -0.5 * R.Ly, yhi = 0.5 * R.Ly;
  p.z = zpos; p.vz = 0.0; p.fz = 0.0;
  if (R.periodic) enforce_periodic(R, p);
  else if (!unlimited) {
    if (p.x < xlo) { p.x = xlo; p.vx = -p.vx; } else if (p.x > xhi) { p.x = xhi; p.vx = -p.vx; }
    if (p.y < ylo) { p.y = ylo; p.vy = -p.vy; } else if (p.y > yhi) { p.y = yhi; p.vy = -p.vy; }
  }
  p.nz = 0.0;
  double len_n = sqrt(p.nx * p.nx + p.ny * p.ny);
  double inv_len = 1.0;
  if (len_n != 0.0) inv_len = 1.0 / len_n;  // the reference recomputes the same sqrt
  p.nx *= inv_len; p.ny *= inv_len;
}

// ConstraintSphere::enforce, constraints/constraint_sphere.cpp:38-81
__device__ __forceinline__ void sphere_enforce(double Rs, Part& p) {
  double R = sqrt(p.x * p.x + p.y * p.y + p.z * p.z);
  double s = Rs / R;
  p.x *= s; p.y *= s; p.z *= s;
  double Nx = p.x / Rs, Ny = p.y / Rs, Nz = p.z / Rs;
  double v_dot_N = p.vx * Nx + p.vy * Ny + p.vz * Nz;
  double n_dot_N = p.nx * Nx + p.ny * Ny + p.nz * Nz;
  p.vx -= v_dot_N * Nx; p.vy -= v_dot_N * Ny; p.vz -= v_dot_N * Nz;
  p.nx -= n_dot_N * Nx; p.ny -= n_dot_N * Ny; p.nz -= n_dot_N * Nz;
  double inv_len = 1.0 / sqrt(p.nx * p.nx + p.ny * p.ny + p.nz * p.nz);
  p.nx *= inv_len; p.ny *= inv_len; p.nz *= inv_len;
}

// ConstraintCylinder::enforce, constraints/constraint_cylinder.cpp:38-71 (its
// own periodic wrap in z, without image flags)
__device__ __forceinline__ void cylinder_enforce(const Replica& R, double rc, Part& p) {
  double x = p.x, y = p.y;
  double Rr = sqrt(x * x + y * y);
  double sc = rc / Rr;
  p.x *= sc; p.y *= sc;
  double Nx = p.x / rc, Ny = p.y / rc;
  double v_dot_N = p.vx * Nx + p.vy * Ny;
  double n_dot_N = p.nx * Nx + p.ny * Ny;
  p.vx -= v_dot_N * Nx; p.vy -= v_dot_N * Ny;
  p.nx -= n_dot_N * Nx; p.ny -= n_dot_N * Ny;
  double inv_len = 1.0 / sqrt(p.nx * p.nx + p.ny * p.ny + p.nz * p.nz);
  p.nx *= inv_len; p.ny *= inv_len; p.nz *= inv_len;
  if (R.periodic) {
    if (p.z > R.zhi) p.z -= R.Lz;
    else if (p.z < R.zlo) p.z += R.Lz;
  }
}

// implicit surfaces, gradient and value in the reference's operation order:
// ConstraintTorus ((c - sqrt(x^2+y^2))^2 + z^2 - a^2, constraint_torus.cpp),
// ConstraintEllipsoid (x^2/a^2 + y^2/b^2 + z^2/c^2 - 1, constraint_ellipsoid.cpp),
// ConstraintPeanut (a^4 - b^4 - 2a^2 (x^2 - y^2 - z^2) + (x^2+y^2+z^2)^2,
// constraint_peanut.cpp:47-66), ConstraintGyroid (periodic in the box,
// constraint_gyroid.cpp:61-80), ConstraintHourglass (x^2 + y^2 - (R + A
// sin(2 pi n z / lz))^2, constraint_hourglass.cpp:47-68) and
// ConstraintGaussianBump (A exp(-x^2/a - y^2/b) - z, constraint_gaussian_bump.cpp:58-75).
// a0 is the replica's first shape parameter (torus c, ellipsoid a, peanut a,
// hourglass R, bump A), C.b2 / C.b3 the second and third.
__host__ __device__ __forceinline__ void implicit_gradient(const ConsComp& C, const Replica& R, double a0, double x,
                                                           double y, double z, double& gx, double& gy, double& gz) {
  if (C.kind == CONS_TORUS) {
    double sqr_xy = sqrt(x * x + y * y);
    double fact = -2.0 * (a0 - sqr_xy) / sqr_xy;
    gx = x * fact; gy = y * fact; gz = 2.0 * z;
  } else if (C.kind == CONS_ELLIPSOID) {
    gx = 2.0 * x / a0 / a0; gy = 2.0 * y / C.b2 / C.b2; gz = 2.0 * z / C.b3 / C.b3;
  } else if (C.kind == CONS_PEANUT) {
    double fact_1 = 4.0 * a0 * a0;
    double fact_2 = 4.0 * (x * x + y * y + z * z);
    gx = (-fact_1 + fact_2) * x;
    gy = (fact_1 + fact_2) * y;
    gz = (fact_1 + fact_2) * z;
  } else if (C.kind == CONS_GYROID) {
    const double lx = R.Lx, ly = R.Ly, lz = R.Lz;
    gx = (2.0 * M_PI * (cos((2.0 * M_PI * x) / lx) * cos((2.0 * M_PI * z) / lz) -
                        sin((2.0 * M_PI * x) / lx) * sin((2.0 * M_PI * y) / ly))) / lx;
    gy = (2.0 * M_PI * (cos((2.0 * M_PI * x) / lx) * cos((2.0 * M_PI * y) / ly) -
                        sin((2.0 * M_PI * y) / ly) * sin((2.0 * M_PI * z) / lz))) / ly;
    gz = (2.0 * M_PI * (cos((2.0 * M_PI * y) / ly) * cos((2.0 * M_PI * z) / lz) -
                        sin((2.0 * M_PI * x) / lx) * sin((2.0 * M_PI * z) / lz))) / lz;
  } else if (C.kind == CONS_TETRAHEDRON) {
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int i = 0; i < 4; i++) {
      double ax, ay, az;
      tetra_charge(i, a0, ax, ay, az);
      const double px = x - ax, py = y - ay, pz = z - az;
      const double l = sqrt(px * px + py * py + pz * pz);
      const double l3 = l * l * l;
      sx += px / l3; sy += py / l3; sz += pz / l3;
    }
    gx = -sx; gy = -sy; gz = -sz;
  } else if (C.kind == CONS_HOURGLASS) {
    const double lz = R.Lz, A = C.b2, n = C.b3;
    gx = 2.0 * x;
    gy = 2.0 * y;
    gz = (-4.0 * A * n * M_PI * cos((2.0 * n * M_PI * z) / lz) * (a0 + A * sin((2.0 * n * M_PI * z) / lz))) / lz;
  } else {  // gaussian bump
    double fact = exp(-x * x / C.b2 - y * y / C.b3);
    gx = -2.0 * a0 * x * fact / C.b2;
    gy = -2.0 * a0 * y * fact / C.b3;
    gz = -1.0;
  }
}
__host__ __device__ __forceinline__ double implicit_value(const ConsComp& C, const Replica& R, double a0, double x,
                                                          double y, double z) {
  if (C.kind == CONS_TORUS) {
    double ft = a0 - sqrt(x * x + y * y);
    return ft * ft + z * z - C.b2 * C.b2;
  }
  if (C.kind == CONS_ELLIPSOID) return x * x / a0 / a0 + y * y / C.b2 / C.b2 + z * z / C.b3 / C.b3 - 1.0;
  if (C.kind == CONS_PEANUT) {
    const double b = C.b2;
    double tr = x * x + y * y + z * z;
    return a0 * a0 * a0 * a0 - b * b * b * b - 2.0 * a0 * a0 * (x * x - y * y - z * z) + tr * tr;
  }
  if (C.kind == CONS_GYROID) {
    const double lx = R.Lx, ly = R.Ly, lz = R.Lz;
    return cos((2.0 * M_PI * z) / lz) * sin((2.0 * M_PI * x) / lx) + cos((2.0 * M_PI * x) / lx) * sin((2.0 * M_PI * y) / ly) +
           cos((2.0 * M_PI * y) / ly) * sin((2.0 * M_PI * z) / lz);
  }
  if (C.kind == CONS_TETRAHEDRON) {
    double g = 0.0;
    for (int i = 0; i < 4; i++) {
      double ax, ay, az;
      tetra_charge(i, a0, ax, ay, az);
      const double px = x - ax, py = y - ay, pz = z - az;
      g += 1.0 / sqrt(px * px + py * py + pz * pz);
    }
    return g - C.b2;
  }
  if (C.kind == CONS_HOURGLASS) {
    double zfact = a0 + C.b2 * sin(2.0 * M_PI / R.Lz * C.b3 * z);
    return x * x + y * y - zfact * zfact;
  }
  return a0 * exp(-x * x / C.b2 - y * y / C.b3) - z;
}

// compute_normal of the curved surfaces (sphere x/R; cylinder x/r, y/r, 0,
// constraint_cylinder.hpp:76-80; implicit: the normalised gradient)
__host__ __device__ __forceinline__ void surface_normal(const ConsComp& C, const Replica& R, double a0, const Part& p,
                                                        double& Nx, double& Ny, double& Nz) {
  if (C.kind == CONS_SPHERE) { Nx = p.x / a0; Ny = p.y / a0; Nz = p.z / a0; }
  else if (C.kind == CONS_CYLINDER) { Nx = p.x / a0; Ny = p.y / a0; Nz = 0.0; }
  else {
    implicit_gradient(C, R, a0, p.x, p.y, p.z, Nx, Ny, Nz);
    double len_N = sqrt(Nx * Nx + Ny * Ny + Nz * Nz);
    Nx /= len_N; Ny /= len_N; Nz /= len_N;
  }
}

// ConstraintSlab::enforce (constraint_slab.cpp:35-61): z kept in [z_lo, z_hi]
// by reflection (vz, nz reversed), then the system's periodic wrap
__device__ __forceinline__ void slab_enforce(const Replica& R, double z_lo, double z_hi, Part& p) {
  if (p.z < z_lo) { p.z = z_lo; p.vz = -p.vz; p.nz = -p.nz; }
  if (p.z > z_hi) { p.z = z_hi; p.vz = -p.vz; p.nz = -p.nz; }
  enforce_periodic(R, p);
}

// ConstraintPlaneWalls::enforce (constraint_plane_walls.cpp:38-70): z = 0,
// vz = fz = 0, y wrapped when periodic (no image flag), walls at x = +-l that
// stop the particle and reverse vx
__device__ __forceinline__ void plane_walls_enforce(const Replica& R, double l, Part& p) {
  p.z = 0.0; p.vz = 0.0; p.fz = 0.0;
  if (R.periodic) {
    if (p.y <= R.ylo) p.y += R.Ly;
    else if (p.y >= R.yhi) p.y -= R.Ly;
  }
  if (p.x >= l) { p.x = l; p.vx = -p.vx; }
  else if (p.x <= -l) { p.x = -l; p.vx = -p.vx; }
}

// Constraint::enforce, constraints/constraint.cpp:40-87 (SHAKE along the
// gradient at the start point, then the tangent projections)
__device__ __forceinline__ void implicit_enforce(const ConsComp& C, const Replica& R, double a0, Part& p) {
  double ref_gx, ref_gy, ref_gz;
  implicit_gradient(C, R, a0, p.x, p.y, p.z, ref_gx, ref_gy, ref_gz);
  int iter = 0;
  while (iter++ < C.max_iter) {
    double gx, gy, gz;
    implicit_gradient(C, R, a0, p.x, p.y, p.z, gx, gy, gz);
    double sv = gx * ref_gx + gy * ref_gy + gz * ref_gz;
    double g = implicit_value(C, R, a0, p.x, p.y, p.z);
    double lambda = g / sv;
    if (!(fabs(g) > C.tol)) break;
    p.x -= lambda * ref_gx;
    p.y -= lambda * ref_gy;
    p.z -= lambda * ref_gz;
  }
  double Nx, Ny, Nz;
  surface_normal(C, R, a0, p, Nx, Ny, Nz);
  double v_dot_N = p.vx * Nx + p.vy * Ny + p.vz * Nz;
  double n_dot_N = p.nx * Nx + p.ny * Ny + p.nz * Nz;
  p.vx -= v_dot_N * Nx; p.vy -= v_dot_N * Ny; p.vz -= v_dot_N * Nz;
  p.nx -= n_dot_N * Nx; p.ny -= n_dot_N * Ny; p.nz -= n_dot_N * Nz;
  double inv_len = 1.0 / sqrt(p.nx * p.nx + p.ny * p.ny + p.nz * p.nz);
  p.nx *= inv_len; p.ny *= inv_len; p.nz *= inv_len;
  enforce_periodic(R, p);
}

// Constrainer::enforce (constrainer.hpp:73-77); ConstraintNone::enforce
// (constraint_none.hpp:58-62)
__device__ __forceinline__ void enforce_all(const Program& P, const Replica& R, Part& p) {
  for (int c = 0; c < P.ncons; c++) {
    int kind = P.cons[c].kind;
    if (kind == CONS_PLANE) plane_enforce(R, R.cons_p[c], P.cons[c].unlimited, p);
    else if (kind == CONS_SPHERE) sphere_enforce(R.cons_p[c], p);
    else if (kind == CONS_CYLINDER) cylinder_enforce(R, R.cons_p[c], p);
    else if (cons_implicit(kind)) implicit_enforce(P.cons[c], R, R.cons_p[c], p);
    else if (kind == CONS_SLAB) slab_enforce(R, R.cons_p[c], P.cons[c].b2, p);
    else if (kind == CONS_PLANE_WALLS) plane_walls_enforce(R, R.cons_p[c], p);
    else enforce_periodic(R, p);
  }
}

// Constrainer::project_torque (constrainer.hpp:93-99) over
// Constraint::project_torque (constraint.cpp:158-173, sphere normal
// constraint_sphere.hpp:76) and ConstraintPlane::project_torque
// (constraint_plane.cpp:150-162)
__device__ __forceinline__ double project_torque(const Program& P, const Replica& R, const Part& p) {
  double val = 0.0;
  for (int c = 0; c < P.ncons; c++) {
    int kind = P.cons[c].kind;
    if (kind == CONS_PLANE || kind == CONS_PLANE_WALLS) val += p.tz;
    else if (kind == CONS_SLAB) val += 0.0;  // constraint_slab.hpp:91
    else if (kind != CONS_NONE) {
      double Nx, Ny, Nz;
      surface_normal(P.cons[c], R, R.cons_p[c], p, Nx, Ny, Nz);
      val += p.tx * Nx + p.ty * Ny + p.tz * Nz;
    } else val += 0.0;
  }
  return val;
}

// Constraint::rotate_director (Rodrigues, constraint.cpp:96-119) and
// ConstraintPlane::rotate_director (constraint_plane.cpp:97-114)
__device__ __forceinline__ void rotate_director(const Program& P, const Replica& R, Part& p, double phi) {
  for (int c = 0; c < P.ncons; c++) {
    int kind = P.cons[c].kind;
    if (kind == CONS_PLANE || kind == CONS_PLANE_WALLS) {
      double cs = cos(phi), sn = sin(phi);
      double Rxx = cs, Rxy = -sn, Ryx = sn, Ryy = cs;
      double nx = Rxx * p.nx + Rxy * p.ny;
      double ny = Ryx * p.nx + Ryy * p.ny;
      double len = sqrt(nx * nx + ny * ny);
      p.nx = nx / len; p.ny = ny / len;
    } else if (kind != CONS_NONE && kind != CONS_SLAB) {  // the slab does not rotate (constraint_slab.hpp:85-88)
      double U, V, W;
      surface_normal(P.cons[c], R, R.cons_p[c], p, U, V, W);
      double cs = cos(phi), sn = sin(phi);
      double dot = U * p.nx + V * p.ny + W * p.nz;
      double nx = U * dot * (1.0 - cs) + p.nx * cs + (-W * p.ny + V * p.nz) * sn;
      double ny = V * dot * (1.0 - cs) + p.ny * cs + (W * p.nx - U * p.nz) * sn;
      double nz = W * dot * (1.0 - cs) + p.nz * cs + (-V * p.nx + U * p.ny) * sn;
      double len = sqrt(nx * nx + ny * ny + nz * nz);
      p.nx = nx / len; p.ny = ny / len; p.nz = nz / len;
    }
  }
}

// Constraint::rotate_velocity (constraint.cpp:128-150) and the plane
// variant (constraint_plane.cpp:122-143)
__device__ __forceinline__ void rotate_velocity(const Program& P, const Replica& R, Part& p, double phi) {
  for (int c = 0; c < P.ncons; c++) {
    int kind = P.cons[c].kind;
    if (kind == CONS_PLANE || kind == CONS_PLANE_WALLS) {
      double cs = cos(phi), sn = sin(phi);
      double Rxx = cs, Rxy = -sn, Ryx = sn, Ryy = cs;
      double vx = Rxx * p.vx + Rxy * p.vy;
      double vy = Ryx * p.vx + Ryy * p.vy;
      p.vx = vx; p.vy = vy;
    } else if (kind != CONS_NONE && kind != CONS_SLAB) {  // the slab does not rotate (constraint_slab.hpp:85-88)
      double U, V, W;
      surface_normal(P.cons[c], R, R.cons_p[c], p, U, V, W);
      double cs = cos(phi), sn = sin(phi);
      double dot = U * p.vx + V * p.vy + W * p.vz;
      double vx = U * dot * (1.0 - cs) + p.vx * cs + (-W * p.vy + V * p.vz) * sn;
      double vy = V * dot * (1.0 - cs) + p.vy * cs + (W * p.vx - U * p.vz) * sn;
      double vz = W * dot * (1.0 - cs) + p.vz * cs + (-V * p.vx + U * p.vy) * sn;
      p.vx = vx; p.vy = vy; p.vz = vz;
    }
  }
}

// ---------------------------------------------------------------------------
// pair terms.  With d = x_other - x_self (minimum image), every reference pair
// potential gives the force on the particle at hand as  -ff * d  and every
// polar/nematic aligner its torque as  +J' (n_self x n_other), bit for bit in
// either role of the pair (IEEE negation is exact and the box is centred).
// ---------------------------------------------------------------------------
struct Nb { double x, y, z, r, nx, ny, nz, vx, vy, vz, age; int type; };

__device__ __forceinline__ double phase_factor(const PairComp& C, double age, double dt) {
  return 0.5 * (1.0 + value_get(C.phase, (int)(age / dt)));
}
__device__ __forceinline__ double phase_pair(double ai, double aj) {
  if (ai < 1.0 && aj < 1.0) return ai + aj - 1.0;
  return ai * aj;
}

// Returns ff (force factor) and adds the pair energy to *pe if in range.
// soft: pair_soft_potential.cpp:57-117; lj: pair_lj_potential.cpp:54-122;
// morse: pair_morse_potential.cpp:52-120; gaussian:
// pair_gaussian_potential.cpp:55-126.
__device__ __forceinline__ bool pair_term(const PairComp& C, const double* g, int ntypes,
                                          const Part& me, const Nb& o, double r_sq,
                                          double alpha, double& ff, double& pe) {
  const double* t = C.table + ((size_t)(me.type - 1) * ntypes + (size_t)(o.type - 1)) * PAIR_NPARAM;
  switch (C.kind) {
    case PAIR_SOFT: {
      double k = t[0];
      double r = sqrt(r_sq);
      double ai_p_aj = C.use_radii ? me.r + o.r : t[1];
      if (r < ai_p_aj) {
        double diff = ai_p_aj - r;
        pe = 0.5 * k * alpha * diff * diff;
        if (r > 0.0) ff = k * alpha * diff / r; else ff = k * diff;
        return true;
      }
      return false;
    }
    case PAIR_LJ: {
      double rcut = C.has_pp ? t[2] : g[2];
      double rcut_sq = rcut * rcut;
      if (r_sq <= rcut_sq) {
        double sigma = C.has_pp ? t[1] : g[1];
        double eps = C.has_pp ? t[0] : g[0];
        if (C.use_radii) sigma = me.r + o.r;
        double sigma_sq = sigma * sigma;
        double inv_r_sq = sigma_sq / r_sq;
        double inv_r_6 = inv_r_sq * inv_r_sq * inv_r_sq;
        double e = 4.0 * eps * alpha * inv_r_6 * (inv_r_6 - 1.0);
        if (C.shifted) {
          double ic = sigma_sq / rcut_sq;
          double ic6 = ic * ic * ic;
          e -= 4.0 * eps * alpha * ic6 * (ic6 - 1.0);
        }
        pe = e;
        ff = 48.0 * eps * alpha * inv_r_6 * (inv_r_6 - 0.5) * inv_r_sq;
        return true;
      }
      return false;
    }
    case PAIR_MORSE: {
      double rcut = C.has_pp ? t[3] : g[3];
      double rcut_sq = rcut * rcut;
      if (r_sq <= rcut_sq) {
        double D = C.has_pp ? t[0] : g[0];
        double a = C.has_pp ? t[1] : g[1];
        double re = C.has_pp ? t[2] : g[2];
        if (C.use_radii) re = me.r + o.r;
        double r = sqrt(r_sq);
        double exp_fact = exp(-a * (r - re));
        double pot_fact = exp_fact - 1.0;
        double e = D * alpha * (pot_fact * pot_fact - 1.0);
        if (C.shifted) {
          double sf = exp(-a * (rcut - re)) - 1.0;
          e -= D * alpha * (sf * sf - 1.0);
        }
        pe = e;
        ff = 2.0 * D * a * alpha * exp_fact * pot_fact / r;
        return true;
      }
      return false;
    }
    default: {  // PAIR_GAUSSIAN
      double rcut = C.has_pp ? t[6] : g[6];
      double rcut_sq = rcut * rcut;
      if (r_sq <= rcut_sq) {
        double A = C.has_pp ? t[0] : g[0];
        double B = C.has_pp ? t[1] : g[1];
        double al = C.has_pp ? t[2] : g[2];
        double be = C.has_pp ? t[3] : g[3];
        double rA = C.has_pp ? t[4] : g[4];
        double rB = C.has_pp ? t[5] : g[5];
        if (C.use_radii) rB = me.r + o.r;
        double r = sqrt(r_sq);
        double r_m_rA = r - rA, r_m_rB = r - rB;
        double e = A * alpha * exp(-al * r_m_rA * r_m_rA) + B * exp(-be * r_m_rB * r_m_rB);
        if (C.shifted) {
          double ca = rcut - rA, cb = rcut - rB;
          e -= A * alpha * exp(-al * ca * ca) + B * exp(-be * cb * cb);
        }
        pe = e;
        ff = (2.0 / r) * alpha * (A * al * r_m_rA * exp(-al * r_m_rA * r_m_rA) +
                                  B * be * r_m_rB * exp(-be * r_m_rB * r_m_rB));
        return true;
      }
      return false;
    }
  }
}

}  // namespace sg
