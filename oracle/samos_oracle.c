/*
 * samos_oracle.c -- CPU oracle (test infrastructure) for the SAMoS hot path.
 *
 * Every function below restates one reference routine; the citation next to
 * it names the reference file and lines (paths relative to the SAMoS tree).
 * Operation order, comparison operators and the order in which floating-point
 * terms are accumulated follow the reference so that, compiled with
 * -ffp-contract=off and without fast-math, the oracle reproduces the
 * reference's arithmetic bit for bit (libm exp/sin/cos aside).
 *
 * Deliberate differences, each documented where it occurs:
 *  - cell indices are clamped into the grid (the reference indexes out of
 *    range when a coordinate equals the upper box edge);
 *  - GSL's generator is replaced by the project noise stream (see header);
 *  - particle groups other than "all", exclusions, stress, per-particle
 *    energy maps and coordination counts are not modelled.
 */
#include "samos_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI  /* strict C11 <math.h> does not define it */
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------------ */
/* noise stream                                                              */
/* ------------------------------------------------------------------------ */

/* Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
   easy as 1, 2, 3", SC'11): 10 rounds of the 4x32 S-box with the published
   multipliers and Weyl key increments. */
void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * (uint64_t)c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * (uint64_t)c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n1 = lo1;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    uint32_t n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

#define OR_NOISE_KEY1 0x53414D4Fu /* "SAMO" */

/* 53-bit uniform in [0,1) from two 32-bit words */
static double u53(uint32_t a, uint32_t b)
{
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

/* Natural logarithm written from the series log(m) = 2 atanh(z),
   z = (m-1)/(m+1), after splitting x = m 2^e with m in [sqrt(1/2), sqrt(2)).
   Only +,-,*,/ in a fixed order, so any IEEE double machine that does not
   contract a*b+c into an FMA gets the same bits.  Accuracy ~1 ulp for the
   noise transform's argument range (0,1). */
double or_noise_log(double x)
{
  union { double d; uint64_t u; } v;
  v.d = x;
  int e = (int)((v.u >> 52) & 0x7ff) - 1023;
  v.u = (v.u & 0x000fffffffffffffull) | 0x3ff0000000000000ull; /* m in [1,2) */
  double m = v.d;
  if (m > 1.4142135623730951) { m = m * 0.5; e = e + 1; }
  double z = (m - 1.0) / (m + 1.0);
  double z2 = z * z;
  /* Horner in z^2 over 1/(2k+1), k = 0..11 */
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
  /* ln 2 split so that de*LN2_HI is exact for |e| < 2^11 */
  const double LN2_HI = 6.93147180369123816490e-01;
  const double LN2_LO = 1.90821492927058770002e-10;
  return (de * LN2_HI + lm) + de * LN2_LO;
}

/* cos(2 pi u) for u in [0,1) given to 53 bits.  4u splits exactly into a
   quadrant q and a fraction f, and the reflection f -> 1-f is exact, so the
   polynomial only sees theta = g pi/2 with g in [0, 1/2]: Taylor series of
   sin to x^15 and cos to x^16 (truncation < 5e-17 on [0, pi/4]). */
static double cos2pi(double u)
{
  double t = u * 4.0;
  int q = (int)t;
  double f = t - (double)q;
  int use_sin = q & 1;            /* q=1,3 need sin(pi f/2) */
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
  /* cos(pi/2 (q + f)): q=0 +cos, q=1 -sin, q=2 -cos, q=3 +sin */
  return (q == 1 || q == 2) ? -v : v;
}

/* Standard normal draw number `counter` of stream `seed`: Box-Muller
   (Box & Muller 1958) on one Philox block, u1 in (0,1] from words 0-1 and
   u2 in [0,1) from words 2-3: g = sqrt(-2 ln u1) cos(2 pi u2). */
double or_noise_gauss(uint32_t seed, uint64_t counter)
{
  uint32_t key[2] = { seed, OR_NOISE_KEY1 };
  uint32_t ctr[4] = { (uint32_t)counter, (uint32_t)(counter >> 32), 0u, 0u };
  uint32_t r[4];
  or_philox4x32_10(ctr, key, r);
  double u1 = u53(r[0], r[1]) + (1.0 / 9007199254740992.0);
  double u2 = u53(r[2], r[3]);
  return sqrt(-2.0 * or_noise_log(u1)) * cos2pi(u2);
}

double or_noise_cos2pi(double u) { return cos2pi(u); }

/* Uniform [0,1) draw number `counter` of stream `seed` */
double or_noise_uniform(uint32_t seed, uint64_t counter)
{
  uint32_t key[2] = { seed, OR_NOISE_KEY1 };
  uint32_t ctr[4] = { (uint32_t)counter, (uint32_t)(counter >> 32), 0u, 1u };
  uint32_t r[4];
  or_philox4x32_10(ctr, key, r);
  return u53(r[0], r[1]);
}

/* RNG object of one integrator (utils/rng.cpp:34-69): one counter value per
   draw, shared between gauss_rng and drnd like GSL's generator state. */
typedef struct { uint32_t seed; uint64_t counter; } or_rng;
static double rng_gauss(or_rng* r, double sigma) { return sigma * or_noise_gauss(r->seed, r->counter++); }
static double rng_drnd(or_rng* r) { return or_noise_uniform(r->seed, r->counter++); }

/* ------------------------------------------------------------------------ */
/* data model                                                                */
/* ------------------------------------------------------------------------ */

/* Value objects, system/value.hpp:115-178 */
typedef struct { int kind; double min_val, max_val; int steps; double dv; } or_value;

static or_value make_value(const double* v)
{
  or_value r;
  if (!v) { r.kind = OR_VALUE_CONSTANT; r.min_val = 0.0; r.max_val = 1.0; r.steps = 1000; r.dv = 0.0; return r; }
  r.kind = (int)v[0]; r.min_val = v[1]; r.max_val = v[2]; r.steps = (int)v[3];
  r.dv = (r.max_val - r.min_val) / (double)r.steps;
  return r;
}

static double value_get(const or_value* v, int step)
{
  if (v->kind == OR_VALUE_CONSTANT) return v->min_val;          /* value.hpp:129 */
  if (step > v->steps) return v->max_val;                        /* value.hpp:166-171 */
  return v->min_val + (double)step * v->dv;
}

typedef struct {
  int kind, use_radii, phase_in, shifted, has_pp;
  double g[OR_PAIR_NPARAM];
  double* table;
  or_value phase;
  double energy;
} or_pair;

typedef struct {
  int kind, has_pp;
  double J, rcut;
  double* table; /* [t1][t2][2] = J, rcut */
  double energy;
} or_align;

typedef struct {
  int kind, has_params;
  double alpha;
  double* type_alpha;
} or_ext;

typedef struct {
  int kind;
  double zpos; int unlimited;      /* plane */
  double r;                        /* sphere; cylinder r; torus c; ellipsoid a; peanut a; hourglass R; bump A */
  double b2, b3;                   /* torus a; ellipsoid b, c; peanut b; hourglass A, n; bump a^2, b^2 */
  int max_iter; double tol;
  double rescale; int rescale_steps, rescale_freq; double scale;
} or_cons;

typedef struct {
  int kind;
  double dt;
  double p[OR_INT_NPARAM];
  or_value temp;
  or_rng rng;
  /* FIRE state */
  double alpha, alpha_init, old_energy; int last_neg, converged;
  /* BBK noise vectors */
  double *Rx, *Ry, *Rz;
  int group;  /* 0 = all, else a group defined by or_define_group */
} or_integ;

#define OR_MAX_COMP 8

struct or_system {
  int N, ntypes;
  double *x, *y, *z, *vx, *vy, *vz, *fx, *fy, *fz, *tx, *ty, *tz;
  double *nx, *ny, *nz, *Nx, *Ny, *Nz, *omega, *age, *radius, *mass;
  int *type, *ix, *iy, *iz;
  double xlo, xhi, ylo, yhi, zlo, zhi, Lx, Ly, Lz; int periodic;
  double dt_global; int time_step, run_step;
  /* neighbour list */
  int has_nlist; double cut, pad; int use_cell;
  int cnx, cny, cnz, ncell; double cwx, cwy, cwz;
  int *cell_nb, *cell_start, *cell_idx, *cell_cnt;
  int *nl_start, *nl_idx, nl_cap; double *ox, *oy, *oz;
  int nlist_builds;
  or_pair pairs[OR_MAX_COMP]; int npairs;
  or_align aligns[OR_MAX_COMP]; int naligns;
  or_ext exts[OR_MAX_COMP]; int nexts;
  or_cons cons[OR_MAX_COMP]; int ncons;
  or_integ integ[OR_MAX_COMP]; int ninteg;
  int* glist[OR_MAX_GROUPS]; int gsize[OR_MAX_GROUPS];  /* group members in particle-index order */
};

#define NFIELDS 22
static const char* FIELD_NAMES[NFIELDS] = {
  "x","y","z","vx","vy","vz","fx","fy","fz","tau_x","tau_y","tau_z",
  "nx","ny","nz","Nx","Ny","Nz","omega","age","radius","mass" };

or_system* or_create(int n, int ntypes)
{
  or_system* s = (or_system*)calloc(1, sizeof(or_system));
  s->N = n; s->ntypes = ntypes;
  double** f[NFIELDS] = { &s->x,&s->y,&s->z,&s->vx,&s->vy,&s->vz,&s->fx,&s->fy,&s->fz,
    &s->tx,&s->ty,&s->tz,&s->nx,&s->ny,&s->nz,&s->Nx,&s->Ny,&s->Nz,&s->omega,&s->age,
    &s->radius,&s->mass };
  for (int k = 0; k < NFIELDS; k++) *f[k] = (double*)calloc(n > 0 ? n : 1, sizeof(double));
  for (int i = 0; i < n; i++) { s->radius[i] = 1.0; s->mass[i] = 1.0; }
  s->type = (int*)calloc(n > 0 ? n : 1, sizeof(int));
  s->ix = (int*)calloc(n > 0 ? n : 1, sizeof(int));
  s->iy = (int*)calloc(n > 0 ? n : 1, sizeof(int));
  s->iz = (int*)calloc(n > 0 ? n : 1, sizeof(int));
  for (int i = 0; i < n; i++) s->type[i] = 1;
  s->Lx = s->Ly = s->Lz = 10.0;
  s->xlo = s->ylo = s->zlo = -5.0; s->xhi = s->yhi = s->zhi = 5.0;
  return s;
}

void or_destroy(or_system* s)
{
  if (!s) return;
  double* f[NFIELDS] = { s->x,s->y,s->z,s->vx,s->vy,s->vz,s->fx,s->fy,s->fz,s->tx,s->ty,s->tz,
    s->nx,s->ny,s->nz,s->Nx,s->Ny,s->Nz,s->omega,s->age,s->radius,s->mass };
  for (int k = 0; k < NFIELDS; k++) free(f[k]);
  free(s->type); free(s->ix); free(s->iy); free(s->iz);
  free(s->cell_nb); free(s->cell_start); free(s->cell_idx); free(s->cell_cnt);
  free(s->nl_start); free(s->nl_idx); free(s->ox); free(s->oy); free(s->oz);
  for (int k = 0; k < s->npairs; k++) free(s->pairs[k].table);
  for (int k = 0; k < s->naligns; k++) free(s->aligns[k].table);
  for (int k = 0; k < s->nexts; k++) free(s->exts[k].type_alpha);
  for (int k = 0; k < s->ninteg; k++) { free(s->integ[k].Rx); free(s->integ[k].Ry); free(s->integ[k].Rz); }
  for (int k = 0; k < OR_MAX_GROUPS; k++) free(s->glist[k]);
  free(s);
}

int or_size(const or_system* s) { return s->N; }

double* or_field(or_system* s, const char* name)
{
  double* f[NFIELDS] = { s->x,s->y,s->z,s->vx,s->vy,s->vz,s->fx,s->fy,s->fz,s->tx,s->ty,s->tz,
    s->nx,s->ny,s->nz,s->Nx,s->Ny,s->Nz,s->omega,s->age,s->radius,s->mass };
  for (int k = 0; k < NFIELDS; k++) if (strcmp(name, FIELD_NAMES[k]) == 0) return f[k];
  return NULL;
}

int* or_ifield(or_system* s, const char* name)
{
  if (strcmp(name, "type") == 0) return s->type;
  if (strcmp(name, "ix") == 0) return s->ix;
  if (strcmp(name, "iy") == 0) return s->iy;
  if (strcmp(name, "iz") == 0) return s->iz;
  return NULL;
}

/* Box(lx,ly,lz), system/box.hpp:56-62: centred at the origin */
void or_set_box(or_system* s, double lx, double ly, double lz, int periodic)
{
  s->Lx = lx; s->Ly = ly; s->Lz = lz;
  s->xlo = -0.5 * lx; s->xhi = 0.5 * lx;
  s->ylo = -0.5 * ly; s->yhi = 0.5 * ly;
  s->zlo = -0.5 * lz; s->zhi = 0.5 * lz;
  s->periodic = periodic;
}

void or_set_timestep(or_system* s, double dt) { s->dt_global = dt; }

/* System::apply_periodic, system/system.cpp:1083-1094 */
static inline void apply_periodic(const or_system* s, double* dx, double* dy, double* dz)
{
  if (s->periodic) {
    if (*dx > s->xhi) *dx -= s->Lx;
    else if (*dx < s->xlo) *dx += s->Lx;
    if (*dy > s->yhi) *dy -= s->Ly;
    else if (*dy < s->ylo) *dy += s->Ly;
    if (*dz > s->zhi) *dz -= s->Lz;
    else if (*dz < s->zlo) *dz += s->Lz;
  }
}

/* System::enforce_periodic, system/system.cpp:1119-1154 */
static inline void enforce_periodic(or_system* s, int i)
{
  if (s->periodic) {
    if (s->x[i] <= s->xlo) { s->x[i] += s->Lx; s->ix[i]--; }
    else if (s->x[i] > s->xhi) { s->x[i] -= s->Lx; s->ix[i]++; }
    if (s->y[i] <= s->ylo) { s->y[i] += s->Ly; s->iy[i]--; }
    else if (s->y[i] > s->yhi) { s->y[i] -= s->Ly; s->iy[i]++; }
    if (s->z[i] <= s->zlo) { s->z[i] += s->Lz; s->iz[i]--; }
    else if (s->z[i] > s->zhi) { s->z[i] -= s->Lz; s->iz[i]++; }
  }
}

/* ------------------------------------------------------------------------ */
/* cell list + neighbour list                                                */
/* ------------------------------------------------------------------------ */

/* CellList ctor, system/cell_list.cpp:37-65: n_d = int(L_d/cut), 27-cell
   stencil in (ix,iy,iz) = -1..1 order with periodic wrap (duplicates when a
   dimension has 2 cells, as in the reference). */
static void cell_list_init(or_system* s, double cutoff)
{
  s->cnx = (int)(s->Lx / cutoff);
  s->cny = (int)(s->Ly / cutoff);
  s->cnz = (int)(s->Lz / cutoff);
  s->ncell = s->cnx * s->cny * s->cnz;
  s->cwx = s->Lx / (double)s->cnx;
  s->cwy = s->Ly / (double)s->cny;
  s->cwz = s->Lz / (double)s->cnz;
  free(s->cell_nb);
  s->cell_nb = (int*)malloc(sizeof(int) * 27 * (size_t)s->ncell);
  for (int i = 0; i < s->cnx; i++)
    for (int j = 0; j < s->cny; j++)
      for (int k = 0; k < s->cnz; k++) {
        int idx = s->cny * s->cnz * i + s->cnz * j + k;
        int m = 0;
        for (int ix = -1; ix <= 1; ix++)
          for (int iy = -1; iy <= 1; iy++)
            for (int iz = -1; iz <= 1; iz++) {
              int iix = i + ix, iiy = j + iy, iiz = k + iz;
              if (iix < 0) iix = s->cnx - 1; else if (iix == s->cnx) iix = 0;
              if (iiy < 0) iiy = s->cny - 1; else if (iiy == s->cny) iiy = 0;
              if (iiz < 0) iiz = s->cnz - 1; else if (iiz == s->cnz) iiz = 0;
              s->cell_nb[27 * idx + m++] = s->cny * s->cnz * iix + s->cnz * iiy + iiz;
            }
      }
  free(s->cell_start); free(s->cell_cnt);
  s->cell_start = (int*)malloc(sizeof(int) * ((size_t)s->ncell + 1));
  s->cell_cnt = (int*)malloc(sizeof(int) * (size_t)s->ncell);
}

static inline int clampi(int v, int n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); }

/* CellList::get_cell_idx, system/cell_list.cpp:72-79 (clamped, see top) */
static int cell_idx(const or_system* s, int i)
{
  int a = (int)((s->x[i] - s->xlo) / s->cwx);
  int b = (int)((s->y[i] - s->ylo) / s->cwy);
  int c = (int)((s->z[i] - s->zlo) / s->cwz);
  a = clampi(a, s->cnx); b = clampi(b, s->cny); c = clampi(c, s->cnz);
  return s->cny * s->cnz * a + s->cnz * b + c;
}

/* CellList::populate, system/cell_list.cpp:82-104: single wrap of positions
   (no image-flag update), particles appended in ascending id */
static void cell_list_populate(or_system* s)
{
  int N = s->N;
  if (s->periodic) {
    for (int i = 0; i < N; i++) {
      if (s->x[i] < s->xlo) s->x[i] += s->Lx; else if (s->x[i] > s->xhi) s->x[i] -= s->Lx;
      if (s->y[i] < s->ylo) s->y[i] += s->Ly; else if (s->y[i] > s->yhi) s->y[i] -= s->Ly;
      if (s->z[i] < s->zlo) s->z[i] += s->Lz; else if (s->z[i] > s->zhi) s->z[i] -= s->Lz;
    }
  }
  memset(s->cell_cnt, 0, sizeof(int) * (size_t)s->ncell);
  int* ci = (int*)malloc(sizeof(int) * (size_t)(N > 0 ? N : 1));
  for (int i = 0; i < N; i++) { ci[i] = cell_idx(s, i); s->cell_cnt[ci[i]]++; }
  s->cell_start[0] = 0;
  for (int c = 0; c < s->ncell; c++) s->cell_start[c + 1] = s->cell_start[c] + s->cell_cnt[c];
  free(s->cell_idx);
  s->cell_idx = (int*)malloc(sizeof(int) * (size_t)(N > 0 ? N : 1));
  memset(s->cell_cnt, 0, sizeof(int) * (size_t)s->ncell);
  for (int i = 0; i < N; i++) { int c = ci[i]; s->cell_idx[s->cell_start[c] + s->cell_cnt[c]++] = i; }
  free(ci);
}

static void nl_push(or_system* s, int* cnt_total, int v)
{
  if (*cnt_total >= s->nl_cap) {
    s->nl_cap = s->nl_cap ? 2 * s->nl_cap : 1024;
    s->nl_idx = (int*)realloc(s->nl_idx, sizeof(int) * (size_t)s->nl_cap);
  }
  s->nl_idx[(*cnt_total)++] = v;
}

/* NeighbourList::build / build_cell / build_nsq,
   system/neighbour_list.cpp:117-149, 216-273, 178-213.  The half list is
   stored CSR: entries of list[i] are nl_idx[nl_start[i] .. nl_start[i+1]). */
int or_build_nlist(or_system* s)
{
  int N = s->N;
  double cut = s->cut + s->pad;
  double cut2 = cut * cut;
  free(s->nl_start);
  s->nl_start = (int*)malloc(sizeof(int) * ((size_t)N + 1));
  int total = 0;
  free(s->ox); free(s->oy); free(s->oz);
  s->ox = (double*)malloc(sizeof(double) * (size_t)(N > 0 ? N : 1));
  s->oy = (double*)malloc(sizeof(double) * (size_t)(N > 0 ? N : 1));
  s->oz = (double*)malloc(sizeof(double) * (size_t)(N > 0 ? N : 1));
  if (s->use_cell) {
    cell_list_populate(s);
    for (int i = 0; i < N; i++) {
      s->nl_start[i] = total;
      int c = cell_idx(s, i);
      for (int m = 0; m < 27; m++) {
        int cc = s->cell_nb[27 * c + m];
        for (int q = s->cell_start[cc]; q < s->cell_start[cc + 1]; q++) {
          int j = s->cell_idx[q];
          if (j > i) {
            double dx = s->x[i] - s->x[j];
            double dy = s->y[i] - s->y[j];
            double dz = s->z[i] - s->z[j];
            apply_periodic(s, &dx, &dy, &dz);
            double d2 = dx * dx + dy * dy + dz * dz;
            if (d2 < cut2) nl_push(s, &total, j);
          }
        }
      }
      s->ox[i] = s->x[i]; s->oy[i] = s->y[i]; s->oz[i] = s->z[i];
    }
    s->nl_start[N] = total;
  } else {
    /* build_nsq(i) appends i to list[j] for every j < i within the cutoff;
       list[j] therefore holds all i > j in ascending order. */
    int* cnt = (int*)calloc((size_t)(N > 0 ? N : 1), sizeof(int));
    for (int i = 0; i < N; i++)
      for (int j = 0; j < i; j++) {
        double dx = s->x[i] - s->x[j];
        double dy = s->y[i] - s->y[j];
        double dz = s->z[i] - s->z[j];
        apply_periodic(s, &dx, &dy, &dz);
        double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 < cut2) cnt[j]++;
      }
    for (int i = 0; i < N; i++) { s->nl_start[i] = total; total += cnt[i]; }
    s->nl_start[N] = total;
    if (total > s->nl_cap) {
      s->nl_cap = total;
      s->nl_idx = (int*)realloc(s->nl_idx, sizeof(int) * (size_t)(total > 0 ? total : 1));
    }
    memset(cnt, 0, sizeof(int) * (size_t)(N > 0 ? N : 1));
    for (int i = 0; i < N; i++) {
      for (int j = 0; j < i; j++) {
        double dx = s->x[i] - s->x[j];
        double dy = s->y[i] - s->y[j];
        double dz = s->z[i] - s->z[j];
        apply_periodic(s, &dx, &dy, &dz);
        double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 < cut2) s->nl_idx[s->nl_start[j] + cnt[j]++] = i;
      }
      s->ox[i] = s->x[i]; s->oy[i] = s->y[i]; s->oz[i] = s->z[i];
    }
    free(cnt);
  }
  s->nlist_builds++;
  return 0;
}

/* NeighbourList ctor, system/neighbour_list.hpp:124-150,216: cell list only
   when every box side exceeds 2(rcut+pad); builds immediately. */
int or_set_nlist(or_system* s, double rcut, double pad)
{
  s->has_nlist = 1;
  s->cut = rcut; s->pad = pad;
  if (s->Lx > 2.0 * (rcut + pad) && s->Ly > 2.0 * (rcut + pad) && s->Lz > 2.0 * (rcut + pad)) {
    s->use_cell = 1;
    cell_list_init(s, rcut + pad);
  } else {
    s->use_cell = 0;
  }
  s->nlist_builds = 0;
  return or_build_nlist(s);
}

int or_nlist_uses_cells(const or_system* s) { return s->use_cell; }
int or_nlist_builds(const or_system* s) { return s->nlist_builds; }

int or_get_pairs(const or_system* s, int* out_i, int* out_j, int cap)
{
  int total = s->nl_start[s->N];
  if (total > cap) return -total;
  for (int i = 0; i < s->N; i++)
    for (int q = s->nl_start[i]; q < s->nl_start[i + 1]; q++) { out_i[q] = i; out_j[q] = s->nl_idx[q]; }
  return total;
}

/* NeighbourList::need_update, system/neighbour_list.cpp:278-302 */
static int need_update(const or_system* s, int id)
{
  double dx = s->ox[id] - s->x[id];
  double dy = s->oy[id] - s->y[id];
  double dz = s->oz[id] - s->z[id];
  if (s->periodic) {
    if (dx > s->xhi) dx -= s->Lx; else if (dx < s->xlo) dx += s->Lx;
    if (dy > s->yhi) dy -= s->Ly; else if (dy < s->ylo) dy += s->Ly;
    if (dz > s->zhi) dz -= s->Lz; else if (dz < s->zlo) dz += s->Lz;
  }
  if (dx * dx + dy * dy + dz * dz < 0.25 * s->pad * s->pad) return 0;
  return 1;
}

/* ------------------------------------------------------------------------ */
/* pair potentials                                                           */
/* ------------------------------------------------------------------------ */

int or_add_pair(or_system* s, int kind, const double* g, const double* table,
                int use_radii, int phase_in, int shifted, int has_pp, const double* phase_value)
{
  if (s->npairs >= OR_MAX_COMP) return -1;
  or_pair* p = &s->pairs[s->npairs++];
  memset(p, 0, sizeof(*p));
  p->kind = kind; p->use_radii = use_radii; p->phase_in = phase_in; p->shifted = shifted; p->has_pp = has_pp;
  for (int k = 0; k < OR_PAIR_NPARAM; k++) p->g[k] = g ? g[k] : 0.0;
  size_t nt = (size_t)s->ntypes * (size_t)s->ntypes * OR_PAIR_NPARAM;
  p->table = (double*)malloc(sizeof(double) * nt);
  for (size_t k = 0; k < nt; k++) p->table[k] = table ? table[k] : p->g[k % OR_PAIR_NPARAM];
  p->phase = make_value(phase_value);
  return s->npairs - 1;
}

static inline const double* ptab(const or_pair* p, int nt, int ti, int tj)
{
  return p->table + ((size_t)ti * (size_t)nt + (size_t)tj) * OR_PAIR_NPARAM;
}

/* phase-in factor of one pair, e.g. pair_soft_potential.cpp:60-76 */
static inline double phase_i(const or_pair* p, double age, double dt)
{
  return 0.5 * (1.0 + value_get(&p->phase, (int)(age / dt)));
}
static inline double phase_pair(double ai, double aj)
{
  if (ai < 1.0 && aj < 1.0) return ai + aj - 1.0;
  return ai * aj;
}

/* PairSoftPotential::compute, potentials/pair/pair_soft_potential.cpp:33-119 */
static void pair_soft(or_system* s, or_pair* P, double dt)
{
  int N = s->N, nt = s->ntypes;
  double alpha_i = 1.0, alpha_j = 1.0, alpha = 1.0;
  double tot_pot = 0.0;
  for (int i = 0; i < N; i++) {
    if (P->phase_in) alpha_i = phase_i(P, s->age[i], dt);
    double ai = s->radius[i];
    for (int q = s->nl_start[i]; q < s->nl_start[i + 1]; q++) {
      int j = s->nl_idx[q];
      if (P->phase_in) { alpha_j = phase_i(P, s->age[j], dt); alpha = phase_pair(alpha_i, alpha_j); }
      const double* t = ptab(P, nt, s->type[i] - 1, s->type[j] - 1);
      double k = t[0];
      double aj = s->radius[j];
      double dx = s->x[j] - s->x[i], dy = s->y[j] - s->y[i], dz = s->z[j] - s->z[i];
      apply_periodic(s, &dx, &dy, &dz);
      double r_sq = dx * dx + dy * dy + dz * dz;
      double r = sqrt(r_sq);
      double ai_p_aj = P->use_radii ? ai + aj : t[1];
      if (r < ai_p_aj) {
        double diff = ai_p_aj - r;
        double pot_eng = 0.5 * k * alpha * diff * diff;
        tot_pot += pot_eng;
        double ff;
        if (r > 0.0) ff = k * alpha * diff / r;
        else ff = k * diff;
        s->fx[i] -= ff * dx; s->fy[i] -= ff * dy; s->fz[i] -= ff * dz;
        s->fx[j] += ff * dx; s->fy[j] += ff * dy; s->fz[j] += ff * dz;
      }
    }
  }
  P->energy = tot_pot;
}

/* PairLJPotential::compute, potentials/pair/pair_lj_potential.cpp:32-124.
   Note the reference's force factor multiplies by sigma^2/r^2 (inv_r_sq),
   not 1/r^2; reproduced as written. */
static void pair_lj(or_system* s, or_pair* P, double dt)
{
  int N = s->N, nt = s->ntypes;
  double sigma = P->g[1], eps = P->g[0], rcut = P->g[2];
  double sigma_sq = sigma * sigma, rcut_sq = rcut * rcut;
  double alpha_i = 1.0, alpha_j = 1.0, alpha = 1.0;
  P->energy = 0.0;
  for (int i = 0; i < N; i++) {
    if (P->phase_in) alpha_i = phase_i(P, s->age[i], dt);
    double ai = s->radius[i];
    for (int q = s->nl_start[i]; q < s->nl_start[i + 1]; q++) {
      int j = s->nl_idx[q];
      if (P->phase_in) { alpha_j = phase_i(P, s->age[j], dt); alpha = phase_pair(alpha_i, alpha_j); }
      const double* t = ptab(P, nt, s->type[i] - 1, s->type[j] - 1);
      if (P->has_pp) { rcut = t[2]; rcut_sq = rcut * rcut; }
      double dx = s->x[i] - s->x[j], dy = s->y[i] - s->y[j], dz = s->z[i] - s->z[j];
      apply_periodic(s, &dx, &dy, &dz);
      double r_sq = dx * dx + dy * dy + dz * dz;
      if (r_sq <= rcut_sq) {
        if (P->has_pp) { sigma = t[1]; eps = t[0]; sigma_sq = sigma * sigma; }
        if (P->use_radii) { sigma = ai + s->radius[j]; sigma_sq = sigma * sigma; }
        double inv_r_sq = sigma_sq / r_sq;
        double inv_r_6 = inv_r_sq * inv_r_sq * inv_r_sq;
        double pe = 4.0 * eps * alpha * inv_r_6 * (inv_r_6 - 1.0);
        if (P->shifted) {
          double inv_r_cut_sq = sigma_sq / rcut_sq;
          double inv_r_cut_6 = inv_r_cut_sq * inv_r_cut_sq * inv_r_cut_sq;
          pe -= 4.0 * eps * alpha * inv_r_cut_6 * (inv_r_cut_6 - 1.0);
        }
        P->energy += pe;
        double ff = 48.0 * eps * alpha * inv_r_6 * (inv_r_6 - 0.5) * inv_r_sq;
        s->fx[i] += ff * dx; s->fy[i] += ff * dy; s->fz[i] += ff * dz;
        s->fx[j] -= ff * dx; s->fy[j] -= ff * dy; s->fz[j] -= ff * dz;
      }
    }
  }
}

/* PairMorsePotential::compute, potentials/pair/pair_morse_potential.cpp:32-122 */
static void pair_morse(or_system* s, or_pair* P, double dt)
{
  int N = s->N, nt = s->ntypes;
  double D = P->g[0], a = P->g[1], re = P->g[2], rcut = P->g[3];
  double rcut_sq = rcut * rcut;
  double alpha_i = 1.0, alpha_j = 1.0, alpha = 1.0;
  P->energy = 0.0;
  for (int i = 0; i < N; i++) {
    if (P->phase_in) alpha_i = phase_i(P, s->age[i], dt);
    double ai = s->radius[i];
    for (int q = s->nl_start[i]; q < s->nl_start[i + 1]; q++) {
      int j = s->nl_idx[q];
      if (P->phase_in) { alpha_j = phase_i(P, s->age[j], dt); alpha = phase_pair(alpha_i, alpha_j); }
      const double* t = ptab(P, nt, s->type[i] - 1, s->type[j] - 1);
      if (P->has_pp) { rcut = t[3]; rcut_sq = rcut * rcut; }
      double dx = s->x[i] - s->x[j], dy = s->y[i] - s->y[j], dz = s->z[i] - s->z[j];
      apply_periodic(s, &dx, &dy, &dz);
      double r_sq = dx * dx + dy * dy + dz * dz;
      if (r_sq <= rcut_sq) {
        if (P->has_pp) { D = t[0]; a = t[1]; re = t[2]; }
        if (P->use_radii) re = ai + s->radius[j];
        double r = sqrt(r_sq);
        double exp_fact = exp(-a * (r - re));
        double pot_fact = exp_fact - 1.0;
        double pe = D * alpha * (pot_fact * pot_fact - 1.0);
        if (P->shifted) {
          double shift_fact = exp(-a * (rcut - re)) - 1.0;
          pe -= D * alpha * (shift_fact * shift_fact - 1.0);
        }
        P->energy += pe;
        double ff = 2.0 * D * a * alpha * exp_fact * pot_fact / r;
        s->fx[i] += ff * dx; s->fy[i] += ff * dy; s->fz[i] += ff * dz;
        s->fx[j] -= ff * dx; s->fy[j] -= ff * dy; s->fz[j] -= ff * dz;
      }
    }
  }
}

/* PairGaussianPotential::compute, potentials/pair/pair_gaussian_potential.cpp:32-128.
   The shift subtracts (A-term + B-term) at rcut; the per-type default table
   carries B = A (pair_gaussian_potential.hpp:174) and is only read when
   has_pair_params is set -- both reproduced by the caller's table. */
static void pair_gaussian(or_system* s, or_pair* P, double dt)
{
  int N = s->N, nt = s->ntypes;
  double A = P->g[0], B = P->g[1], alpha = P->g[2], beta = P->g[3], rA = P->g[4], rB = P->g[5], rcut = P->g[6];
  double rcut_sq = rcut * rcut;
  double pf_i = 1.0, pf_j = 1.0, pf = 1.0;
  P->energy = 0.0;
  for (int i = 0; i < N; i++) {
    if (P->phase_in) pf_i = phase_i(P, s->age[i], dt);
    for (int q = s->nl_start[i]; q < s->nl_start[i + 1]; q++) {
      int j = s->nl_idx[q];
      if (P->phase_in) { pf_j = phase_i(P, s->age[j], dt); pf = phase_pair(pf_i, pf_j); }
      double ai = s->radius[i];
      const double* t = ptab(P, nt, s->type[i] - 1, s->type[j] - 1);
      if (P->has_pp) { rcut = t[6]; rcut_sq = rcut * rcut; }
      double dx = s->x[i] - s->x[j], dy = s->y[i] - s->y[j], dz = s->z[i] - s->z[j];
      apply_periodic(s, &dx, &dy, &dz);
      double r_sq = dx * dx + dy * dy + dz * dz;
      if (r_sq <= rcut_sq) {
        if (P->has_pp) { A = t[0]; B = t[1]; alpha = t[2]; beta = t[3]; rA = t[4]; rB = t[5]; }
        if (P->use_radii) rB = ai + s->radius[j];
        double r = sqrt(r_sq);
        double r_m_rA = r - rA, r_m_rB = r - rB;
        double pe = A * pf * exp(-alpha * r_m_rA * r_m_rA) + B * exp(-beta * r_m_rB * r_m_rB);
        if (P->shifted) {
          double rcut_m_rA = rcut - rA, rcut_m_rB = rcut - rB;
          pe -= A * pf * exp(-alpha * rcut_m_rA * rcut_m_rA) + B * exp(-beta * rcut_m_rB * rcut_m_rB);
        }
        P->energy += pe;
        double ff = (2.0 / r) * pf * (A * alpha * r_m_rA * exp(-alpha * r_m_rA * r_m_rA) +
                                      B * beta * r_m_rB * exp(-beta * r_m_rB * r_m_rB));
        s->fx[i] += ff * dx; s->fy[i] += ff * dy; s->fz[i] += ff * dz;
        s->fx[j] -= ff * dx; s->fy[j] -= ff * dy; s->fz[j] -= ff * dz;
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* aligners                                                                  */
/* ------------------------------------------------------------------------ */

int or_add_align(or_system* s, int kind, double J, double rcut, const double* table, int has_pp)
{
  if (s->naligns >= OR_MAX_COMP) return -1;
  or_align* a = &s->aligns[s->naligns++];
  memset(a, 0, sizeof(*a));
  a->kind = kind; a->J = J; a->rcut = rcut; a->has_pp = has_pp;
  size_t nt = (size_t)s->ntypes * (size_t)s->ntypes * 2;
  a->table = (double*)malloc(sizeof(double) * nt);
  for (size_t k = 0; k < nt; k++) a->table[k] = table ? table[k] : ((k & 1) ? rcut : J);
  return s->naligns - 1;
}

/* inline min-image used by the aligners (same as apply_periodic) */
#define ALIGN_WRAP(s, dx, dy, dz) apply_periodic((s), &(dx), &(dy), &(dz))

/* PairPolarAlign::compute, aligner/pair/pair_polar_aligner.cpp:32-107 */
static void align_polar(or_system* s, or_align* A)
{
  int N = s->N, nt = s->ntypes;
  double J = A->J, rcut = A->rcut;
  double tot_pot = 0.0;
  for (int i = 0; i < N; i++) {
    for (int q = s->nl_start[i]; q < s->nl_start[i + 1]; q++) {
      int j = s->nl_idx[q];
      if (A->has_pp) {
        const double* t = A->table + ((size_t)(s->type[i] - 1) * nt + (size_t)(s->type[j] - 1)) * 2;
        J = t[0]; rcut = t[1];
      }
      double dx = s->x[j] - s->x[i], dy = s->y[j] - s->y[i], dz = s->z[j] - s->z[i];
      ALIGN_WRAP(s, dx, dy, dz);
      double r_sq = dx * dx + dy * dy + dz * dz;
      if (r_sq <= rcut * rcut) {
        double tau_x = s->ny[i] * s->nz[j] - s->nz[i] * s->ny[j];
        double tau_y = s->nz[i] * s->nx[j] - s->nx[i] * s->nz[j];
        double tau_z = s->nx[i] * s->ny[j] - s->ny[i] * s->nx[j];
        s->tx[i] += J * tau_x; s->ty[i] += J * tau_y; s->tz[i] += J * tau_z;
        s->tx[j] += -J * tau_x; s->ty[j] += -J * tau_y; s->tz[j] += -J * tau_z;
        double pe = -2.0 * J * (s->nx[i] * s->nx[j] + s->ny[i] * s->ny[j] + s->nz[i] * s->nz[j]);
        tot_pot += pe;
      }
    }
  }
  A->energy = tot_pot;
}

/* PairNematicAlign::compute, aligner/pair/pair_nematic_aligner.cpp:32-96:
   J doubled by default, taken verbatim from align_param */
static void align_nematic(or_system* s, or_align* A)
{
  int N = s->N, nt = s->ntypes;
  double J = 2.0 * A->J, rcut = A->rcut;
  A->energy = 0.0;
  for (int i = 0; i < N; i++) {
    for (int q = s->nl_start[i]; q < s->nl_start[i + 1]; q++) {
      int j = s->nl_idx[q];
      if (A->has_pp) {
        const double* t = A->table + ((size_t)(s->type[i] - 1) * nt + (size_t)(s->type[j] - 1)) * 2;
        J = t[0]; rcut = t[1];
      }
      double dx = s->x[j] - s->x[i], dy = s->y[j] - s->y[i], dz = s->z[j] - s->z[i];
      ALIGN_WRAP(s, dx, dy, dz);
      double r_sq = dx * dx + dy * dy + dz * dz;
      if (r_sq <= rcut * rcut) {
        double c = s->nx[i] * s->nx[j] + s->ny[i] * s->ny[j] + s->nz[i] * s->nz[j];
        double tau_x = s->ny[i] * s->nz[j] - s->nz[i] * s->ny[j];
        double tau_y = s->nz[i] * s->nx[j] - s->nx[i] * s->nz[j];
        double tau_z = s->nx[i] * s->ny[j] - s->ny[i] * s->nx[j];
        s->tx[i] += J * c * tau_x; s->ty[i] += J * c * tau_y; s->tz[i] += J * c * tau_z;
        s->tx[j] += -J * c * tau_x; s->ty[j] += -J * c * tau_y; s->tz[j] += -J * c * tau_z;
        double pe = -2.0 * J * (2.0 * c * c - 1.0);
        A->energy += pe;
      }
    }
  }
}

/* PairVicsekAlign::compute, aligner/pair/pair_vicsek_aligner.cpp:32-83 */
static void align_vicsek(or_system* s, or_align* A)
{
  int N = s->N;
  double rcut = A->rcut;
  for (int i = 0; i < N; i++) {
    for (int q = s->nl_start[i]; q < s->nl_start[i + 1]; q++) {
      int j = s->nl_idx[q];
      double dx = s->x[j] - s->x[i], dy = s->y[j] - s->y[i], dz = s->z[j] - s->z[i];
      ALIGN_WRAP(s, dx, dy, dz);
      double r_sq = dx * dx + dy * dy + dz * dz;
      if (r_sq <= rcut * rcut) {
        s->tx[i] += s->vx[j]; s->ty[i] += s->vy[j]; s->tz[i] += s->vz[j];
        s->tx[j] += s->vx[i]; s->ty[j] += s->vy[i]; s->tz[j] += s->vz[i];
      }
    }
    s->tx[i] += s->vx[i]; s->ty[i] += s->vy[i]; s->tz[i] += s->vz[i];
  }
  for (int i = 0; i < N; i++) {
    double v = sqrt(s->tx[i] * s->tx[i] + s->ty[i] * s->ty[i] + s->tz[i] * s->tz[i]);
    if (v == 0.0) v = 1.0;
    double inv_v = 1.0 / v;
    s->tx[i] *= inv_v; s->ty[i] *= inv_v; s->tz[i] *= inv_v;
  }
  A->energy = 0.0;
}

/* ------------------------------------------------------------------------ */
/* external potentials                                                       */
/* ------------------------------------------------------------------------ */

int or_add_external(or_system* s, int kind, double alpha, const double* type_alpha, int has_params)
{
  if (s->nexts >= OR_MAX_COMP) return -1;
  or_ext* e = &s->exts[s->nexts++];
  memset(e, 0, sizeof(*e));
  e->kind = kind; e->alpha = alpha; e->has_params = has_params;
  e->type_alpha = (double*)malloc(sizeof(double) * (size_t)s->ntypes);
  for (int t = 0; t < s->ntypes; t++) e->type_alpha[t] = type_alpha ? type_alpha[t] : alpha;
  return s->nexts - 1;
}

/* ExternalSelfPropulsion::compute, potentials/external/external_self_propulsion.cpp:33-50 */
static void ext_self_propulsion(or_system* s, or_ext* e)
{
  double alpha = e->alpha;
  for (int i = 0; i < s->N; i++) {
    if (e->has_params) alpha = e->type_alpha[s->type[i] - 1];
    s->fx[i] += alpha * s->nx[i];
    s->fy[i] += alpha * s->ny[i];
    s->fz[i] += alpha * s->nz[i];
  }
}

/* ------------------------------------------------------------------------ */
/* constraints                                                               */
/* ------------------------------------------------------------------------ */

/* Constraint base ctor, constraints/constraint.hpp:56-120 (tol is parsed
   as an int, constraint.hpp:82, so the caller passes the truncated value) */
int or_add_constraint(or_system* s, int kind, const double* p)
{
  if (s->ncons >= OR_MAX_COMP) return -1;
  if (kind == OR_CONS_PEANUT) {  /* constraint_peanut.hpp:84-88, on the defaults too (a 10, b 8) */
    const double a = p ? p[0] : 10.0, b = p ? p[7] : 8.0;
    if (b <= a) return -1;
  }
  or_cons* c = &s->cons[s->ncons++];
  memset(c, 0, sizeof(*c));
  c->kind = kind;
  c->zpos = p ? p[0] : 0.0; c->unlimited = p ? (int)p[1] : 0;
  c->r = p ? p[0]
           : (kind == OR_CONS_PEANUT || kind == OR_CONS_HOURGLASS || kind == OR_CONS_TETRAHEDRON ? 10.0
              : kind == OR_CONS_SLAB ? 0.0 : 1.0);
  if (kind == OR_CONS_PLANE_WALLS && c->r > s->xhi) c->r = s->xhi;  /* constraint_plane_walls.hpp:64-71 */
  if (kind >= OR_CONS_TORUS) {  /* params[7], params[8] */
    c->b2 = p ? p[7] : (kind == OR_CONS_TORUS ? 0.5 : kind == OR_CONS_PEANUT ? 8.0 : 1.0);
    c->b3 = p ? p[8] : 1.0;
  }
  c->max_iter = p ? (int)p[2] : 100;
  c->tol = p ? p[3] : 1e-6;
  c->rescale = p ? p[4] : 1.0;
  c->rescale_steps = p ? (int)p[5] : 1000;
  c->rescale_freq = p ? (int)p[6] : 10;
  c->scale = pow(c->rescale, (double)c->rescale_freq / (double)c->rescale_steps);
  /* the reference enforces the new constraint on every particle at once
     (samos.cpp:518-522) */
  return s->ncons - 1;
}

/* ConstraintPlane::enforce, constraints/constraint_plane.cpp:36-89 */
static void plane_enforce(or_system* s, const or_cons* c, int i)
{
  double Lx = s->Lx, Ly = s->Ly;
  double xlo = -0.5 * Lx, xhi = 0.5 * Lx;
  double ylo = -0.5 * Ly, yhi = 0.5 * Ly;
  s->z[i] = c->zpos;
  s->vz[i] = 0.0;
  s->fz[i] = 0.0;
  s->Nx[i] = 0.0; s->Ny[i] = 0.0; s->Nz[i] = 1.0;
  if (s->periodic) enforce_periodic(s, i);
  else if (!c->unlimited) {
    if (s->x[i] < xlo) { s->x[i] = xlo; s->vx[i] = -s->vx[i]; }
    else if (s->x[i] > xhi) { s->x[i] = xhi; s->vx[i] = -s->vx[i]; }
    if (s->y[i] < ylo) { s->y[i] = ylo; s->vy[i] = -s->vy[i]; }
    else if (s->y[i] > yhi) { s->y[i] = yhi; s->vy[i] = -s->vy[i]; }
  }
  s->nz[i] = 0.0;
  double len_n = sqrt(s->nx[i] * s->nx[i] + s->ny[i] * s->ny[i]);
  double inv_len = 1.0;
  if (len_n != 0.0) inv_len = 1.0 / sqrt(s->nx[i] * s->nx[i] + s->ny[i] * s->ny[i]);
  s->nx[i] *= inv_len; s->ny[i] *= inv_len;
}

/* ConstraintSphere::enforce, constraints/constraint_sphere.cpp:38-81 */
static void sphere_enforce(or_system* s, const or_cons* c, int i)
{
  double x = s->x[i], y = s->y[i], z = s->z[i];
  double R = sqrt(x * x + y * y + z * z);
  double sc = c->r / R;
  s->x[i] *= sc; s->y[i] *= sc; s->z[i] *= sc;
  double Nx = s->x[i] / c->r, Ny = s->y[i] / c->r, Nz = s->z[i] / c->r;
  double v_dot_N = s->vx[i] * Nx + s->vy[i] * Ny + s->vz[i] * Nz;
  double n_dot_N = s->nx[i] * Nx + s->ny[i] * Ny + s->nz[i] * Nz;
  s->vx[i] -= v_dot_N * Nx; s->vy[i] -= v_dot_N * Ny; s->vz[i] -= v_dot_N * Nz;
  s->nx[i] -= n_dot_N * Nx; s->ny[i] -= n_dot_N * Ny; s->nz[i] -= n_dot_N * Nz;
  double inv_len = 1.0 / sqrt(s->nx[i] * s->nx[i] + s->ny[i] * s->ny[i] + s->nz[i] * s->nz[i]);
  s->nx[i] *= inv_len; s->ny[i] *= inv_len; s->nz[i] *= inv_len;
  s->Nx[i] = Nx; s->Ny[i] = Ny; s->Nz[i] = Nz;
}

/* Constrainer::enforce, constraints/constrainer.hpp:73-77; ConstraintNone,
   constraints/constraint_none.hpp:58-62 */
/* ConstraintCylinder::enforce, constraints/constraint_cylinder.cpp:38-71:
   radial projection onto radius r; the periodic wrap in z is the
   constraint's own (no image-flag update). */
static void cylinder_enforce(or_system* s, const or_cons* c, int i)
{
  double x = s->x[i], y = s->y[i];
  double R = sqrt(x * x + y * y);
  double sc = c->r / R;
  s->x[i] *= sc; s->y[i] *= sc;
  double Nx = s->x[i] / c->r, Ny = s->y[i] / c->r;
  double v_dot_N = s->vx[i] * Nx + s->vy[i] * Ny;
  double n_dot_N = s->nx[i] * Nx + s->ny[i] * Ny;
  s->vx[i] -= v_dot_N * Nx; s->vy[i] -= v_dot_N * Ny;
  s->nx[i] -= n_dot_N * Nx; s->ny[i] -= n_dot_N * Ny;
  double inv_len = 1.0 / sqrt(s->nx[i] * s->nx[i] + s->ny[i] * s->ny[i] + s->nz[i] * s->nz[i]);
  s->nx[i] *= inv_len; s->ny[i] *= inv_len; s->nz[i] *= inv_len;
  if (s->periodic) {
    if (s->z[i] > 0.5 * s->Lz) s->z[i] -= s->Lz;
    else if (s->z[i] < -0.5 * s->Lz) s->z[i] += s->Lz;
  }
}

/* ConstraintTetrahedron's unit charges (constraint_tetrahedron.hpp:42-45),
   scaled by the constraint's scale; the surface is an equipotential of
   sum 1/|r - a_i| (constraint_tetrahedron.cpp:47-80) */
static const double TETRA[4][3] = {{1.0, 0.0, -0.7071067811865475}, {-1.0, 0.0, -0.7071067811865475},
                                   {0.0, 1.0, 0.7071067811865475}, {0.0, -1.0, 0.7071067811865475}};

/* compute_gradient / constraint_value of the implicit surfaces, in the
   reference's operation order: ConstraintTorus (constraint_torus.cpp:
   (c - sqrt(x^2+y^2))^2 + z^2 - a^2), ConstraintEllipsoid
   (constraint_ellipsoid.cpp: x^2/a^2 + y^2/b^2 + z^2/c^2 - 1),
   ConstraintPeanut (constraint_peanut.cpp:47-66), ConstraintGyroid
   (constraint_gyroid.cpp:61-80, periodic in the box), ConstraintHourglass
   (constraint_hourglass.cpp:47-68) and ConstraintGaussianBump
   (constraint_gaussian_bump.cpp:58-75) */
static void implicit_gradient(const or_system* s, const or_cons* c, double x, double y, double z, double* gx,
                              double* gy, double* gz)
{
  if (c->kind == OR_CONS_TORUS) {
    double sqr_xy = sqrt(x * x + y * y);
    double fact = -2.0 * (c->r - sqr_xy) / sqr_xy;
    *gx = x * fact; *gy = y * fact; *gz = 2.0 * z;
  } else if (c->kind == OR_CONS_ELLIPSOID) {
    *gx = 2.0 * x / c->r / c->r; *gy = 2.0 * y / c->b2 / c->b2; *gz = 2.0 * z / c->b3 / c->b3;
  } else if (c->kind == OR_CONS_PEANUT) {
    double fact_1 = 4.0 * c->r * c->r;
    double fact_2 = 4.0 * (x * x + y * y + z * z);
    *gx = (-fact_1 + fact_2) * x;
    *gy = (fact_1 + fact_2) * y;
    *gz = (fact_1 + fact_2) * z;
  } else if (c->kind == OR_CONS_GYROID) {
    double lx = s->Lx, ly = s->Ly, lz = s->Lz;
    *gx = (2.0 * M_PI * (cos((2.0 * M_PI * x) / lx) * cos((2.0 * M_PI * z) / lz) -
                         sin((2.0 * M_PI * x) / lx) * sin((2.0 * M_PI * y) / ly))) / lx;
    *gy = (2.0 * M_PI * (cos((2.0 * M_PI * x) / lx) * cos((2.0 * M_PI * y) / ly) -
                         sin((2.0 * M_PI * y) / ly) * sin((2.0 * M_PI * z) / lz))) / ly;
    *gz = (2.0 * M_PI * (cos((2.0 * M_PI * y) / ly) * cos((2.0 * M_PI * z) / lz) -
                         sin((2.0 * M_PI * x) / lx) * sin((2.0 * M_PI * z) / lz))) / lz;
  } else if (c->kind == OR_CONS_TETRAHEDRON) {
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int k = 0; k < 4; k++) {
      double px = x - c->r * TETRA[k][0], py = y - c->r * TETRA[k][1], pz = z - c->r * TETRA[k][2];
      double l = sqrt(px * px + py * py + pz * pz);
      double l3 = l * l * l;
      sx += px / l3; sy += py / l3; sz += pz / l3;
    }
    *gx = -sx; *gy = -sy; *gz = -sz;
  } else if (c->kind == OR_CONS_HOURGLASS) {
    double lz = s->Lz, A = c->b2, n = c->b3;
    *gx = 2.0 * x;
    *gy = 2.0 * y;
    *gz = (-4.0 * A * n * M_PI * cos((2.0 * n * M_PI * z) / lz) * (c->r + A * sin((2.0 * n * M_PI * z) / lz))) / lz;
  } else {
    double fact = exp(-x * x / c->b2 - y * y / c->b3);
    *gx = -2.0 * c->r * x * fact / c->b2;
    *gy = -2.0 * c->r * y * fact / c->b3;
    *gz = -1.0;
  }
}

static double implicit_value(const or_system* s, const or_cons* c, double x, double y, double z)
{
  if (c->kind == OR_CONS_TORUS) {
    double ft = c->r - sqrt(x * x + y * y);
    return ft * ft + z * z - c->b2 * c->b2;
  }
  if (c->kind == OR_CONS_ELLIPSOID) return x * x / c->r / c->r + y * y / c->b2 / c->b2 + z * z / c->b3 / c->b3 - 1.0;
  if (c->kind == OR_CONS_PEANUT) {
    double a = c->r, b = c->b2;
    double tr = x * x + y * y + z * z;
    return a * a * a * a - b * b * b * b - 2.0 * a * a * (x * x - y * y - z * z) + tr * tr;
  }
  if (c->kind == OR_CONS_GYROID) {
    double lx = s->Lx, ly = s->Ly, lz = s->Lz;
    return cos((2.0 * M_PI * z) / lz) * sin((2.0 * M_PI * x) / lx) + cos((2.0 * M_PI * x) / lx) * sin((2.0 * M_PI * y) / ly) +
           cos((2.0 * M_PI * y) / ly) * sin((2.0 * M_PI * z) / lz);
  }
  if (c->kind == OR_CONS_TETRAHEDRON) {
    double g = 0.0;
    for (int k = 0; k < 4; k++) {
      double px = x - c->r * TETRA[k][0], py = y - c->r * TETRA[k][1], pz = z - c->r * TETRA[k][2];
      g += 1.0 / sqrt(px * px + py * py + pz * pz);
    }
    return g - c->b2;
  }
  if (c->kind == OR_CONS_HOURGLASS) {
    double zfact = c->r + c->b2 * sin(2.0 * M_PI / s->Lz * c->b3 * z);
    return x * x + y * y - zfact * zfact;
  }
  return c->r * exp(-x * x / c->b2 - y * y / c->b3) - z;
}

/* compute_normal of each non-plane surface (the gradient normalised for the
   implicit ones, constraint_torus.cpp / constraint_ellipsoid.cpp; x/r, y/r, 0
   for the cylinder, constraint_cylinder.hpp:76-80) */
static void surface_normal(or_system* s, const or_cons* c, int i, double* Nx, double* Ny, double* Nz)
{
  if (c->kind == OR_CONS_SPHERE) { *Nx = s->x[i] / c->r; *Ny = s->y[i] / c->r; *Nz = s->z[i] / c->r; }
  else if (c->kind == OR_CONS_CYLINDER) { *Nx = s->x[i] / c->r; *Ny = s->y[i] / c->r; *Nz = 0.0; }
  else {
    implicit_gradient(s, c, s->x[i], s->y[i], s->z[i], Nx, Ny, Nz);
    double len_N = sqrt(*Nx * *Nx + *Ny * *Ny + *Nz * *Nz);
    *Nx /= len_N; *Ny /= len_N; *Nz /= len_N;
  }
  s->Nx[i] = *Nx; s->Ny[i] = *Ny; s->Nz[i] = *Nz;
}

/* Constraint::enforce, constraints/constraint.cpp:40-87: SHAKE iterations
   along the gradient at the start point until |g| <= tol, then the tangent
   projections of v and n, n normalised, and the periodic wrap. */
static void implicit_enforce(or_system* s, const or_cons* c, int i)
{
  double ref_gx, ref_gy, ref_gz;
  implicit_gradient(s, c, s->x[i], s->y[i], s->z[i], &ref_gx, &ref_gy, &ref_gz);
  int iter = 0;
  while (iter++ < c->max_iter) {
    double gx, gy, gz;
    implicit_gradient(s, c, s->x[i], s->y[i], s->z[i], &gx, &gy, &gz);
    double sv = gx * ref_gx + gy * ref_gy + gz * ref_gz;
    double g = implicit_value(s, c, s->x[i], s->y[i], s->z[i]);
    double lambda = g / sv;
    if (!(fabs(g) > c->tol)) break;
    s->x[i] -= lambda * ref_gx;
    s->y[i] -= lambda * ref_gy;
    s->z[i] -= lambda * ref_gz;
  }
  double Nx, Ny, Nz;
  surface_normal(s, c, i, &Nx, &Ny, &Nz);
  double v_dot_N = s->vx[i] * Nx + s->vy[i] * Ny + s->vz[i] * Nz;
  double n_dot_N = s->nx[i] * Nx + s->ny[i] * Ny + s->nz[i] * Nz;
  s->vx[i] -= v_dot_N * Nx; s->vy[i] -= v_dot_N * Ny; s->vz[i] -= v_dot_N * Nz;
  s->nx[i] -= n_dot_N * Nx; s->ny[i] -= n_dot_N * Ny; s->nz[i] -= n_dot_N * Nz;
  double inv_len = 1.0 / sqrt(s->nx[i] * s->nx[i] + s->ny[i] * s->ny[i] + s->nz[i] * s->nz[i]);
  s->nx[i] *= inv_len; s->ny[i] *= inv_len; s->nz[i] *= inv_len;
  if (s->periodic) enforce_periodic(s, i);
}

/* ConstraintSlab::enforce (constraint_slab.cpp:35-61): reflect z into
   [z_lo, z_hi] (vz and nz reversed), then the periodic wrap; its normal is
   zero (constraint_slab.hpp:94) */
static void slab_enforce(or_system* s, const or_cons* c, int i)
{
  if (s->z[i] < c->r) { s->z[i] = c->r; s->vz[i] = -s->vz[i]; s->nz[i] = -s->nz[i]; }
  if (s->z[i] > c->b2) { s->z[i] = c->b2; s->vz[i] = -s->vz[i]; s->nz[i] = -s->nz[i]; }
  s->Nx[i] = 0.0; s->Ny[i] = 0.0; s->Nz[i] = 0.0;
  if (s->periodic) enforce_periodic(s, i);
}

/* ConstraintPlaneWalls::enforce (constraint_plane_walls.cpp:38-70): z = 0,
   vz = fz = 0, y wrapped without image flag, walls at x = +-l; normal
   (0, 0, 1) (constraint_plane_walls.hpp:90) */
static void plane_walls_enforce(or_system* s, const or_cons* c, int i)
{
  double ylo = s->ylo, yhi = s->yhi, ly = yhi - ylo;
  s->z[i] = 0.0; s->vz[i] = 0.0; s->fz[i] = 0.0;
  s->Nx[i] = 0.0; s->Ny[i] = 0.0; s->Nz[i] = 1.0;
  if (s->periodic) {
    if (s->y[i] <= ylo) s->y[i] += ly;
    else if (s->y[i] >= yhi) s->y[i] -= ly;
  }
  if (s->x[i] >= c->r) { s->x[i] = c->r; s->vx[i] = -s->vx[i]; }
  else if (s->x[i] <= -c->r) { s->x[i] = -c->r; s->vx[i] = -s->vx[i]; }
}

static void enforce_one(or_system* s, int i)
{
  for (int k = 0; k < s->ncons; k++) {
    const or_cons* c = &s->cons[k];
    if (c->kind == OR_CONS_PLANE) plane_enforce(s, c, i);
    else if (c->kind == OR_CONS_SPHERE) sphere_enforce(s, c, i);
    else if (c->kind == OR_CONS_CYLINDER) cylinder_enforce(s, c, i);
    else if ((c->kind >= OR_CONS_TORUS && c->kind <= OR_CONS_GAUSSIAN_BUMP) || c->kind == OR_CONS_TETRAHEDRON)
      implicit_enforce(s, c, i);
    else if (c->kind == OR_CONS_SLAB) slab_enforce(s, c, i);
    else if (c->kind == OR_CONS_PLANE_WALLS) plane_walls_enforce(s, c, i);
    else if (s->periodic) enforce_periodic(s, i);
  }
}

void or_enforce_all(or_system* s)
{
  for (int i = 0; i < s->N; i++) enforce_one(s, i);
}

/* Constrainer::project_torque, constrainer.hpp:93-99, with
   Constraint::project_torque (constraint.cpp:158-173, sphere normal
   constraint_sphere.hpp:76) and ConstraintPlane::project_torque
   (constraint_plane.cpp:150-162) */
static double project_torque(or_system* s, int i)
{
  double val = 0.0;
  for (int k = 0; k < s->ncons; k++) {
    const or_cons* c = &s->cons[k];
    if (c->kind == OR_CONS_PLANE || c->kind == OR_CONS_PLANE_WALLS) val += s->tz[i];
    else if (c->kind == OR_CONS_SLAB) val += 0.0;  /* constraint_slab.hpp:91 */
    else if (c->kind != OR_CONS_NONE) {
      double Nx, Ny, Nz;
      surface_normal(s, c, i, &Nx, &Ny, &Nz);
      val += s->tx[i] * Nx + s->ty[i] * Ny + s->tz[i] * Nz;
    } else val += 0.0;
  }
  return val;
}

/* Constraint::rotate_director (Rodrigues about the normal,
   constraint.cpp:96-119) for the sphere; ConstraintPlane::rotate_director
   (constraint_plane.cpp:97-114); none: no-op */
static void rotate_director(or_system* s, int i, double phi)
{
  for (int k = 0; k < s->ncons; k++) {
    const or_cons* c = &s->cons[k];
    if (c->kind == OR_CONS_PLANE || c->kind == OR_CONS_PLANE_WALLS) {
      double cs = cos(phi), sn = sin(phi);
      double Rxx = cs, Rxy = -sn, Ryx = sn, Ryy = cs;
      double nx = Rxx * s->nx[i] + Rxy * s->ny[i];
      double ny = Ryx * s->nx[i] + Ryy * s->ny[i];
      double len = sqrt(nx * nx + ny * ny);
      s->nx[i] = nx / len; s->ny[i] = ny / len;
    } else if (c->kind != OR_CONS_NONE && c->kind != OR_CONS_SLAB) {  /* the slab does not rotate */
      double U, V, W;
      surface_normal(s, c, i, &U, &V, &W);
      double cs = cos(phi), sn = sin(phi);
      double pnx = s->nx[i], pny = s->ny[i], pnz = s->nz[i];
      double nx = U * (U * pnx + V * pny + W * pnz) * (1.0 - cs) + pnx * cs + (-W * pny + V * pnz) * sn;
      double ny = V * (U * pnx + V * pny + W * pnz) * (1.0 - cs) + pny * cs + (W * pnx - U * pnz) * sn;
      double nz = W * (U * pnx + V * pny + W * pnz) * (1.0 - cs) + pnz * cs + (-V * pnx + U * pny) * sn;
      double len = sqrt(nx * nx + ny * ny + nz * nz);
      s->nx[i] = nx / len; s->ny[i] = ny / len; s->nz[i] = nz / len;
    }
  }
}

/* Constraint::rotate_velocity (constraint.cpp:128-150) and the plane
   variant (constraint_plane.cpp:122-143) */
static void rotate_velocity(or_system* s, int i, double phi)
{
  for (int k = 0; k < s->ncons; k++) {
    const or_cons* c = &s->cons[k];
    if (c->kind == OR_CONS_PLANE || c->kind == OR_CONS_PLANE_WALLS) {
      double cs = cos(phi), sn = sin(phi);
      double Rxx = cs, Rxy = -sn, Ryx = sn, Ryy = cs;
      double vx = Rxx * s->vx[i] + Rxy * s->vy[i];
      double vy = Ryx * s->vx[i] + Ryy * s->vy[i];
      s->vx[i] = vx; s->vy[i] = vy;
    } else if (c->kind != OR_CONS_NONE && c->kind != OR_CONS_SLAB) {  /* the slab does not rotate */
      double U, V, W;
      surface_normal(s, c, i, &U, &V, &W);
      double cs = cos(phi), sn = sin(phi);
      double pvx = s->vx[i], pvy = s->vy[i], pvz = s->vz[i];
      double vx = U * (U * pvx + V * pvy + W * pvz) * (1.0 - cs) + pvx * cs + (-W * pvy + V * pvz) * sn;
      double vy = V * (U * pvx + V * pvy + W * pvz) * (1.0 - cs) + pvy * cs + (W * pvx - U * pvz) * sn;
      double vz = W * (U * pvx + V * pvy + W * pvz) * (1.0 - cs) + pvz * cs + (-V * pvx + U * pvy) * sn;
      s->vx[i] = vx; s->vy[i] = vy; s->vz[i] = vz;
    }
  }
}

/* Constraint::rescale per kind, OR-ed by Constrainer::rescale
   (constrainer.hpp:117-123): ConstraintSphere::rescale
   (constraint_sphere.cpp:87-104) and ConstraintTetrahedron::rescale
   (constraint_tetrahedron.cpp:88-109) scale r / s on steps below
   rescale_steps, ConstraintCylinder::rescale (constraint_cylinder.cpp:79-96)
   up to and including it, ConstraintPlane::rescale
   (constraint_plane.cpp:168-188) scales the box and every position; the
   other constraints keep the base class's no-op (constraint.hpp:144) */
static int constraints_rescale(or_system* s)
{
  int res = 0;
  for (int k = 0; k < s->ncons; k++) {
    or_cons* c = &s->cons[k];
    int r = 0;
    if (res) continue; /* `res || rescale()` short-circuits */
    if (c->rescale != 1.0) {
      int step = s->time_step;
      int due = step % c->rescale_freq == 0 &&
                (c->kind == OR_CONS_CYLINDER ? step <= c->rescale_steps : step < c->rescale_steps);
      if (!due) {
      } else if (c->kind == OR_CONS_SPHERE || c->kind == OR_CONS_CYLINDER || c->kind == OR_CONS_TETRAHEDRON) {
        c->r *= c->scale;
        for (int i = 0; i < s->N; i++) {
          if (c->kind == OR_CONS_SPHERE) sphere_enforce(s, c, i);
          else if (c->kind == OR_CONS_CYLINDER) cylinder_enforce(s, c, i);
          else implicit_enforce(s, c, i);
        }
        r = 1;
      } else if (c->kind == OR_CONS_PLANE) {
        double a = c->scale;
        s->Lx *= a; s->Ly *= a; s->Lz *= a;
        s->xlo *= a; s->ylo *= a; s->zlo *= a;
        s->xhi *= a; s->yhi *= a; s->zhi *= a;
        for (int i = 0; i < s->N; i++) {
          s->x[i] *= a; s->y[i] *= a; s->z[i] *= a;
          plane_enforce(s, c, i);
        }
        r = 1;
      }
    }
    res = res || r;
  }
  return res;
}

/* ------------------------------------------------------------------------ */
/* force / torque evaluation                                                 */
/* ------------------------------------------------------------------------ */

/* System::reset_forces / reset_torques, system/system.hpp:136-157 */
static void reset_forces(or_system* s)
{
  for (int i = 0; i < s->N; i++) { s->fx[i] = 0.0; s->fy[i] = 0.0; s->fz[i] = 0.0; }
}
static void reset_torques(or_system* s)
{
  for (int i = 0; i < s->N; i++) { s->tx[i] = 0.0; s->ty[i] = 0.0; s->tz[i] = 0.0; }
}

/* Potential::compute, potentials/potential.cpp:36-52: pair potentials then
   external ones, each list in the caller's (std::map key) order */
static void potential_compute(or_system* s, double dt)
{
  for (int k = 0; k < s->npairs; k++) {
    or_pair* P = &s->pairs[k];
    switch (P->kind) {
      case OR_PAIR_SOFT: pair_soft(s, P, dt); break;
      case OR_PAIR_LJ: pair_lj(s, P, dt); break;
      case OR_PAIR_MORSE: pair_morse(s, P, dt); break;
      case OR_PAIR_GAUSSIAN: pair_gaussian(s, P, dt); break;
    }
  }
  for (int k = 0; k < s->nexts; k++) ext_self_propulsion(s, &s->exts[k]);
}

/* Aligner::compute, aligner/aligner.cpp:35-45 */
static void aligner_compute(or_system* s)
{
  for (int k = 0; k < s->naligns; k++) {
    or_align* A = &s->aligns[k];
    switch (A->kind) {
      case OR_ALIGN_POLAR: align_polar(s, A); break;
      case OR_ALIGN_NEMATIC: align_nematic(s, A); break;
      case OR_ALIGN_VICSEK: align_vicsek(s, A); break;
    }
  }
}

/* Potential::compute_potential_energy, potentials/potential.cpp:57-75 */
double or_total_potential_energy(const or_system* s)
{
  double e = 0.0;
  for (int k = 0; k < s->npairs; k++) e += s->pairs[k].energy;
  for (int k = 0; k < s->nexts; k++) e += 0.0;
  return e;
}

double or_pair_energy(const or_system* s, int idx) { return s->pairs[idx].energy; }
double or_align_energy(const or_system* s, int idx) { return s->aligns[idx].energy; }

void or_compute(or_system* s, double dt)
{
  reset_forces(s);
  reset_torques(s);
  if (s->npairs + s->nexts) potential_compute(s, dt);
  if (s->naligns) aligner_compute(s);
}

/* ------------------------------------------------------------------------ */
/* integrators                                                               */
/* ------------------------------------------------------------------------ */

/* Parameter vector layouts (p[]):
 *  brownian       : 0 dt, 1 v0, 2 nu, 3 mu, 4 mur, 5 seed, 6 nematic, 7 tau, 8 velocity_align
 *  brownian_pos   : 0 dt, 3 mu, 5 seed
 *  brownian_align : 0 dt, 2 nu, 4 mur, 5 seed, 6 nematic, 7 tau
 *  langevin       : 0 dt, 5 seed, 9 gamma, 10 method
 *  fire           : 0 dt, 1 alpha, 2 alpha_scale, 3 f_tol, 4 e_tol, 6 dt_inc,
 *                   7 dt_dec, 8 dt_max, 9 min_neg_steps, 11 fmax_tol (<=0: off)
 *  nve            : 0 dt, 12 has_limit, 13 limit, 14 has_angle_limit, 15 angle_limit
 *  vicsek         : 0 dt, 1 v0, 2 eta, 3 mu, 5 seed
 * `tau` is the conf value; the flip probability dt/tau is formed here as in
 * integrator_brownian.hpp:139-147.
 */
int or_add_integrator(or_system* s, int kind, const double* p, const double* temp)
{
  if (s->ninteg >= OR_MAX_COMP) return -1;
  or_integ* g = &s->integ[s->ninteg++];
  memset(g, 0, sizeof(*g));
  g->kind = kind;
  for (int k = 0; k < OR_INT_NPARAM; k++) g->p[k] = p[k];
  g->dt = p[0];
  g->temp = make_value(temp);
  g->rng.seed = (uint32_t)(int32_t)p[5];
  g->rng.counter = 0;
  if (kind == OR_INT_FIRE) {
    g->alpha = p[1]; g->alpha_init = p[1];
    g->old_energy = 1e15; g->last_neg = 0; g->converged = 0;
    g->rng.seed = 0;
  }
  if (kind == OR_INT_LANGEVIN && (int)p[10] == OR_LANGEVIN_BBK) {
    /* integrator_langevin.hpp:103-111: 3 draws per particle at construction */
    int N = s->N;
    g->Rx = (double*)malloc(sizeof(double) * (size_t)(N > 0 ? N : 1));
    g->Ry = (double*)malloc(sizeof(double) * (size_t)(N > 0 ? N : 1));
    g->Rz = (double*)malloc(sizeof(double) * (size_t)(N > 0 ? N : 1));
    for (int i = 0; i < N; i++) {
      g->Rx[i] = rng_gauss(&g->rng, 1.0);
      g->Ry[i] = rng_gauss(&g->rng, 1.0);
      g->Rz[i] = rng_gauss(&g->rng, 1.0);
    }
  }
  return s->ninteg - 1;
}

/* System::make_group (system.cpp:462-572): members in particle-index order */
int or_define_group(or_system* s, int group, const unsigned char* member)
{
  if (group < 1 || group >= OR_MAX_GROUPS) return -1;
  free(s->glist[group]);
  s->glist[group] = (int*)malloc(sizeof(int) * (size_t)(s->N > 0 ? s->N : 1));
  int n = 0;
  for (int i = 0; i < s->N; i++)
    if (member[i]) s->glist[group][n++] = i;
  s->gsize[group] = n;
  return 0;
}

/* an integrator's `group` parameter (integrator.hpp:67-109) */
int or_set_integrator_group(or_system* s, int idx, int group)
{
  if (idx < 0 || idx >= s->ninteg || group < 0 || group >= OR_MAX_GROUPS) return -1;
  if (group && !s->glist[group]) return -1;
  s->integ[idx].group = group;
  return 0;
}

int or_integrator_state(or_system* s, int idx, double* out)
{
  or_integ* g = &s->integ[idx];
  out[0] = g->dt; out[1] = g->alpha; out[2] = (double)g->last_neg; out[3] = (double)g->converged;
  out[4] = g->old_energy; out[5] = (double)g->rng.counter; out[6] = 0.0; out[7] = 0.0;
  return 0;
}

/* IntegratorBrownian::integrate, integrators/integrator_brownian.cpp:42-124 */
static void integ_brownian(or_system* s, or_integ* g)
{
  int N = s->N;
  double dt = g->dt, v0 = g->p[1], nu = g->p[2], mu = g->p[3], mur = g->p[4];
  int nematic = (int)g->p[6], velocity = (int)g->p[8];
  double flip = nematic ? dt / g->p[7] : 0.0;
  double stoch_coeff = sqrt(nu * dt);
  double T = value_get(&g->temp, s->run_step);
  double B = sqrt(2.0 * mu * T);
  double sqrt_dt = sqrt(dt);
  const int M = g->group ? s->gsize[g->group] : N;  /* the integrator's group, in index order */
  if (nematic)
    for (int q = 0; q < M; q++) {
      const int i = g->group ? s->glist[g->group][q] : q;
      if (rng_drnd(&g->rng) < flip) {
        s->nx[i] = -s->nx[i]; s->ny[i] = -s->ny[i]; s->nz[i] = -s->nz[i];
        if (velocity) { s->vx[i] = -s->vx[i]; s->vy[i] = -s->vy[i]; s->vz[i] = -s->vz[i]; }
      }
    }
  for (int q = 0; q < M; q++) {
    const int i = g->group ? s->glist[g->group][q] : q;
    double fd_x = v0 * s->nx[i] + mu * s->fx[i];
    double fd_y = v0 * s->ny[i] + mu * s->fy[i];
    double fd_z = v0 * s->nz[i] + mu * s->fz[i];
    s->vx[i] = fd_x; s->vy[i] = fd_y; s->vz[i] = fd_z;
    s->x[i] += dt * fd_x; s->y[i] += dt * fd_y; s->z[i] += dt * fd_z;
    if (T > 0.0) {
      double fr_x = B * rng_gauss(&g->rng, 1.0);
      double fr_y = B * rng_gauss(&g->rng, 1.0);
      double fr_z = B * rng_gauss(&g->rng, 1.0);
      s->vx[i] += fr_x; s->vy[i] += fr_y; s->vz[i] += fr_z;
      s->x[i] += sqrt_dt * fr_x; s->y[i] += sqrt_dt * fr_y; s->z[i] += sqrt_dt * fr_z;
    }
    enforce_one(s, i);
    s->omega[i] = mur * project_torque(s, i);
    double dtheta = dt * s->omega[i] + stoch_coeff * rng_gauss(&g->rng, 1.0);
    rotate_director(s, i, dtheta);
    if (velocity) rotate_velocity(s, i, dtheta);
    s->age[i] += dt;
  }
}

/* IntegratorBrownianPos::integrate, integrators/integrator_brownian_pos.cpp:37-84 */
static void integ_brownian_pos(or_system* s, or_integ* g)
{
  int N = s->N;
  double dt = g->dt, mu = g->p[3];
  double T = value_get(&g->temp, s->run_step);
  double B = sqrt(2.0 * mu * T);
  double sqrt_dt = sqrt(dt);
  const int M = g->group ? s->gsize[g->group] : N;
  for (int q = 0; q < M; q++) {
    const int i = g->group ? s->glist[g->group][q] : q;
    s->vx[i] = mu * s->fx[i]; s->vy[i] = mu * s->fy[i]; s->vz[i] = mu * s->fz[i];
    s->x[i] += dt * s->vx[i]; s->y[i] += dt * s->vy[i]; s->z[i] += dt * s->vz[i];
    if (T > 0.0) {
      double fr_x = B * rng_gauss(&g->rng, 1.0);
      double fr_y = B * rng_gauss(&g->rng, 1.0);
      double fr_z = B * rng_gauss(&g->rng, 1.0);
      s->vx[i] += fr_x; s->vy[i] += fr_y; s->vz[i] += fr_z;
      s->x[i] += sqrt_dt * fr_x; s->y[i] += sqrt_dt * fr_y; s->z[i] += sqrt_dt * fr_z;
    }
    enforce_one(s, i);
    s->age[i] += dt;
  }
}

/* IntegratorBrownianAlign::integrate, integrators/integrator_brownian_align.cpp:41-76 */
static void integ_brownian_align(or_system* s, or_integ* g)
{
  int N = s->N;
  double dt = g->dt, nu = g->p[2], mur = g->p[4];
  int nematic = (int)g->p[6];
  double flip = nematic ? dt / g->p[7] : 0.0;
  double stoch_coeff = sqrt(nu * dt);
  const int M = g->group ? s->gsize[g->group] : N;
  if (nematic)
    for (int q = 0; q < M; q++) {
      const int i = g->group ? s->glist[g->group][q] : q;
      if (rng_drnd(&g->rng) < flip) { s->nx[i] = -s->nx[i]; s->ny[i] = -s->ny[i]; s->nz[i] = -s->nz[i]; }
    }
  for (int q = 0; q < M; q++) {
    const int i = g->group ? s->glist[g->group][q] : q;
    s->omega[i] = mur * project_torque(s, i);
    double dtheta = dt * s->omega[i] + stoch_coeff * rng_gauss(&g->rng, 1.0);
    rotate_director(s, i, dtheta);
  }
}

/* IntegratorLangevin::integrate_baoab, integrators/integrator_langevin.cpp:55-114 */
static void integ_langevin_baoab(or_system* s, or_integ* g)
{
  int N = s->N;
  double dt = g->dt, gamma = g->p[9];
  double T = value_get(&g->temp, s->run_step);
  double B = sqrt(T * (1.0 - exp(-2.0 * gamma * dt)));
  double exp_dt = exp(-gamma * dt);
  double dt2 = 0.5 * dt;
  for (int i = 0; i < N; i++) {
    double fact = dt2 / s->mass[i];
    s->vx[i] += fact * s->fx[i]; s->vy[i] += fact * s->fy[i]; s->vz[i] += fact * s->fz[i];
    s->x[i] += dt2 * s->vx[i]; s->y[i] += dt2 * s->vy[i]; s->z[i] += dt2 * s->vz[i];
    enforce_one(s, i);
    s->vx[i] *= exp_dt; s->vy[i] *= exp_dt; s->vz[i] *= exp_dt;
    if (B != 0.0) {
      double stoch_fact = B / sqrt(s->mass[i]);
      s->vx[i] += stoch_fact * rng_gauss(&g->rng, 1.0);
      s->vy[i] += stoch_fact * rng_gauss(&g->rng, 1.0);
      s->vz[i] += stoch_fact * rng_gauss(&g->rng, 1.0);
    }
    s->x[i] += dt2 * s->vx[i]; s->y[i] += dt2 * s->vy[i]; s->z[i] += dt2 * s->vz[i];
    enforce_one(s, i);
  }
  reset_forces(s);
  if (s->npairs + s->nexts) potential_compute(s, dt);
  for (int i = 0; i < N; i++) {
    double fact = dt2 / s->mass[i];
    s->vx[i] += fact * s->fx[i]; s->vy[i] += fact * s->fy[i]; s->vz[i] += fact * s->fz[i];
    s->age[i] += dt;
  }
}

/* IntegratorLangevin::integrate_spv, integrators/integrator_langevin.cpp:124-184 */
static void integ_langevin_spv(or_system* s, or_integ* g)
{
  int N = s->N;
  double dt = g->dt, gamma = g->p[9];
  double T = value_get(&g->temp, s->run_step);
  double zeta = sqrt(T * (1.0 - exp(-2.0 * gamma * dt)));
  double eta = (gamma == 0.0) ? 0.0 : (1.0 - exp(-dt * gamma)) / gamma;
  double exp_dt = exp(-dt * gamma);
  double dt2 = 0.5 * dt;
  for (int i = 0; i < N; i++) {
    s->x[i] += dt2 * s->vx[i]; s->y[i] += dt2 * s->vy[i]; s->z[i] += dt2 * s->vz[i];
    enforce_one(s, i);
  }
  reset_forces(s);
  if (s->npairs + s->nexts) potential_compute(s, dt);
  for (int i = 0; i < N; i++) {
    double fact = eta / s->mass[i];
    s->vx[i] = exp_dt * s->vx[i] + fact * s->fx[i];
    s->vy[i] = exp_dt * s->vy[i] + fact * s->fy[i];
    s->vz[i] = exp_dt * s->vz[i] + fact * s->fz[i];
    if (zeta != 0.0) {
      double stoch_fact = zeta / sqrt(s->mass[i]);
      s->vx[i] += stoch_fact * rng_gauss(&g->rng, 1.0);
      s->vy[i] += stoch_fact * rng_gauss(&g->rng, 1.0);
      s->vz[i] += stoch_fact * rng_gauss(&g->rng, 1.0);
    }
    s->x[i] += dt2 * s->vx[i]; s->y[i] += dt2 * s->vy[i]; s->z[i] += dt2 * s->vz[i];
    enforce_one(s, i);
    s->age[i] += dt;
  }
}

/* IntegratorLangevin::integrate_bbk, integrators/integrator_langevin.cpp:194-253
   (age advances only when B != 0, as in the reference) */
static void integ_langevin_bbk(or_system* s, or_integ* g)
{
  int N = s->N;
  double dt = g->dt, gamma = g->p[9];
  double T = value_get(&g->temp, s->run_step);
  double B = sqrt(2.0 * T * dt * gamma);
  double dt2 = 0.5 * dt;
  double one_m_dt2 = 1.0 - gamma * dt2;
  double one_div_one_p_dt2 = 1.0 / (1.0 + gamma * dt2);
  for (int i = 0; i < N; i++) {
    double dt2_over_mass = dt2 / s->mass[i];
    s->vx[i] = one_m_dt2 * s->vx[i] + dt2_over_mass * s->fx[i];
    s->vy[i] = one_m_dt2 * s->vy[i] + dt2_over_mass * s->fy[i];
    s->vz[i] = one_m_dt2 * s->vz[i] + dt2_over_mass * s->fz[i];
    if (B != 0.0) {
      double stoch_fact = 0.5 * B / sqrt(s->mass[i]);
      s->vx[i] += stoch_fact * g->Rx[i];
      s->vy[i] += stoch_fact * g->Ry[i];
      s->vz[i] += stoch_fact * g->Rz[i];
    }
    s->x[i] += dt * s->vx[i]; s->y[i] += dt * s->vy[i]; s->z[i] += dt * s->vz[i];
    enforce_one(s, i);
  }
  reset_forces(s);
  if (s->npairs + s->nexts) potential_compute(s, dt);
  for (int i = 0; i < N; i++) {
    double dt2_over_mass = dt2 / s->mass[i];
    s->vx[i] = one_div_one_p_dt2 * (s->vx[i] + dt2_over_mass * s->fx[i]);
    s->vy[i] = one_div_one_p_dt2 * (s->vy[i] + dt2_over_mass * s->fy[i]);
    s->vz[i] = one_div_one_p_dt2 * (s->vz[i] + dt2_over_mass * s->fz[i]);
    if (B != 0.0) {
      double stoch_fact = 0.5 * B * one_div_one_p_dt2 / sqrt(s->mass[i]);
      g->Rx[i] = rng_gauss(&g->rng, 1.0);
      g->Ry[i] = rng_gauss(&g->rng, 1.0);
      g->Rz[i] = rng_gauss(&g->rng, 1.0);
      s->vx[i] += stoch_fact * g->Rx[i];
      s->vy[i] += stoch_fact * g->Ry[i];
      s->vz[i] += stoch_fact * g->Rz[i];
      s->age[i] += dt;
    }
  }
}

/* IntegratorFIRE::integrate, integrators/integrator_fire.cpp:34-148.  With
   fmax_tol > 0 (a parameter added by this project) convergence is
   max_i |F_i| < fmax_tol instead of the reference's RMS-force + energy test. */
static void integ_fire(or_system* s, or_integ* g)
{
  int N = s->N;
  double P = 0.0, E, Fnorm = 0.0, Vnorm = 0.0, Fmax2 = 0.0;
  double sqrt_ndof = sqrt((double)(3 * N));
  double dt_2 = 0.5 * g->dt;
  for (int i = 0; i < N; i++) {
    s->vx[i] += dt_2 * s->fx[i]; s->vy[i] += dt_2 * s->fy[i]; s->vz[i] += dt_2 * s->fz[i];
    s->x[i] += g->dt * s->vx[i]; s->y[i] += g->dt * s->vy[i]; s->z[i] += g->dt * s->vz[i];
    enforce_one(s, i);
    s->omega[i] += dt_2 * project_torque(s, i);
    double dtheta = g->dt * s->omega[i];
    rotate_director(s, i, dtheta);
  }
  reset_forces(s);
  reset_torques(s);
  if (s->npairs + s->nexts) potential_compute(s, g->dt);
  if (s->naligns) aligner_compute(s);
  for (int i = 0; i < N; i++) {
    s->vx[i] += dt_2 * s->fx[i]; s->vy[i] += dt_2 * s->fy[i]; s->vz[i] += dt_2 * s->fz[i];
    P += s->vx[i] * s->fx[i] + s->vy[i] * s->fy[i] + s->vz[i] * s->fz[i];
    double f2 = s->fx[i] * s->fx[i] + s->fy[i] * s->fy[i] + s->fz[i] * s->fz[i];
    Fnorm += f2;
    if (f2 > Fmax2) Fmax2 = f2;
    Vnorm += s->vx[i] * s->vx[i] + s->vy[i] * s->vy[i] + s->vz[i] * s->vz[i];
    enforce_one(s, i);
    s->omega[i] += dt_2 * project_torque(s, i);
  }
  Fnorm = sqrt(Fnorm);
  Vnorm = sqrt(Vnorm);
  E = or_total_potential_energy(s);
  double fmax_tol = g->p[11];
  int conv = (fmax_tol > 0.0) ? (sqrt(Fmax2) < fmax_tol)
                              : (Fnorm / sqrt_ndof < g->p[3] && fabs(E - g->old_energy) < g->p[4]);
  if (conv) { g->converged = 1; return; }
  double inv_Fnorm = 1.0 / Fnorm;
  double fact_1 = 1.0 - g->alpha;
  double fact_2 = g->alpha * inv_Fnorm * Vnorm;
  for (int i = 0; i < N; i++) {
    s->vx[i] = fact_1 * s->vx[i] + fact_2 * s->fx[i];
    s->vy[i] = fact_1 * s->vy[i] + fact_2 * s->fy[i];
    s->vz[i] = fact_1 * s->vz[i] + fact_2 * s->fz[i];
  }
  if (P > 0.0) {
    g->last_neg++;
    if (g->last_neg > (int)g->p[9]) {
      double ndt = g->dt * g->p[6];
      g->dt = ndt < g->p[8] ? ndt : g->p[8];
      g->alpha *= g->p[2];
    }
  } else {
    g->dt *= g->p[7];
    g->alpha = g->alpha_init;
    g->last_neg = 0;
    for (int i = 0; i < N; i++) { s->vx[i] = 0.0; s->vy[i] = 0.0; s->vz[i] = 0.0; }
  }
  g->converged = 0;
  g->old_energy = E;
}

/* IntegratorNVE::integrate, integrators/integrator_nve.cpp:37-141.  The
 * reference leaves m_has_limit / m_has_theta_limit / m_theta_limit
 * uninitialised when `limit` / `angle_limit` are absent (integrator_nve.hpp
 * constructor); here an absent limit is off, and the omega clamp of the last
 * loop (guarded there by m_has_limit but reading m_theta_limit) applies only
 * when both limits are given. */
static void integ_nve(or_system* s, or_integ* g)
{
  int N = s->N;
  double dt = g->dt, dt_2 = 0.5 * dt;
  int has_limit = g->p[12] != 0.0, has_theta = g->p[14] != 0.0;
  double limit = g->p[13], theta_limit = g->p[15];
  for (int i = 0; i < N; i++) {
    s->vx[i] += dt_2 * s->fx[i]; s->vy[i] += dt_2 * s->fy[i]; s->vz[i] += dt_2 * s->fz[i];
    enforce_one(s, i);
    s->omega[i] += dt_2 * project_torque(s, i);
  }
  for (int i = 0; i < N; i++) {
    double dx = dt * s->vx[i], dy = dt * s->vy[i], dz = dt * s->vz[i];
    if (has_limit) {
      double dr = sqrt(dx * dx + dy * dy + dz * dz);
      if (dr > limit) { dx = limit * dx / dr; dy = limit * dy / dr; dz = limit * dz / dr; }
    }
    s->x[i] += dx; s->y[i] += dy; s->z[i] += dz;
    enforce_one(s, i);
  }
  for (int i = 0; i < N; i++) {
    double dtheta = dt * s->omega[i];
    if (has_theta && fabs(dtheta) > theta_limit) dtheta = (dtheta >= 0.0 ? 1.0 : -1.0) * theta_limit;  /* SIGN, integrator_nve.hpp:38 */
    rotate_director(s, i, dtheta);
  }
  reset_forces(s);
  reset_torques(s);
  if (s->npairs + s->nexts) potential_compute(s, dt);
  if (s->naligns) aligner_compute(s);
  for (int i = 0; i < N; i++) {
    s->vx[i] += dt_2 * s->fx[i]; s->vy[i] += dt_2 * s->fy[i]; s->vz[i] += dt_2 * s->fz[i];
    if (has_limit) {
      double v = sqrt(s->vx[i] * s->vx[i] + s->vy[i] * s->vy[i] + s->vz[i] * s->vz[i]);
      if (v * dt > limit) {
        s->vx[i] = s->vx[i] / v * limit / dt;
        s->vy[i] = s->vy[i] / v * limit / dt;
        s->vz[i] = s->vz[i] / v * limit / dt;
      }
    }
    enforce_one(s, i);
    s->omega[i] += dt_2 * project_torque(s, i);
    if (has_limit && has_theta && fabs(s->omega[i]) * dt > theta_limit)
      s->omega[i] = (s->omega[i] >= 0.0 ? 1.0 : -1.0) * theta_limit / dt;
    s->age[i] += dt;
  }
}

/* IntegratorVicsek::integrate, integrators/integrator_vicsek.cpp:44-82:
 * velocity along the aligner's (normalised) torque vector plus mobility
 * times force, a uniform random rotation of the velocity in the tangent plane
 * of width eta*sqrt(dt), then the position update. */
static void integ_vicsek(or_system* s, or_integ* g)
{
  int N = s->N;
  double dt = g->dt, v0 = g->p[1], eta = g->p[2], mu = g->p[3];
  double noise = eta * sqrt(dt);
  const int M = g->group ? s->gsize[g->group] : N;
  for (int q = 0; q < M; q++) {
    const int i = g->group ? s->glist[g->group][q] : q;
    s->vx[i] = v0 * s->tx[i] + mu * s->fx[i];
    s->vy[i] = v0 * s->ty[i] + mu * s->fy[i];
    s->vz[i] = v0 * s->tz[i] + mu * s->fz[i];
    enforce_one(s, i);
    double theta = 2.0 * noise * 3.14159265358979323846 * (rng_drnd(&g->rng) - 0.5);
    rotate_velocity(s, i, theta);
    s->x[i] += dt * s->vx[i];
    s->y[i] += dt * s->vy[i];
    s->z[i] += dt * s->vz[i];
    enforce_one(s, i);
    s->age[i] += dt;
  }
}

static void integrate(or_system* s, or_integ* g)
{
  switch (g->kind) {
    case OR_INT_BROWNIAN: integ_brownian(s, g); break;
    case OR_INT_BROWNIAN_POS: integ_brownian_pos(s, g); break;
    case OR_INT_BROWNIAN_ALIGN: integ_brownian_align(s, g); break;
    case OR_INT_LANGEVIN:
      switch ((int)g->p[10]) {
        case OR_LANGEVIN_SPV: integ_langevin_spv(s, g); break;
        case OR_LANGEVIN_BBK: integ_langevin_bbk(s, g); break;
        default: integ_langevin_baoab(s, g); break;
      }
      break;
    case OR_INT_FIRE: integ_fire(s, g); break;
    case OR_INT_NVE: integ_nve(s, g); break;
    case OR_INT_VICSEK: integ_vicsek(s, g); break;
  }
}

/* ------------------------------------------------------------------------ */
/* run loop, src/samos.cpp:864-972                                           */
/* ------------------------------------------------------------------------ */

static void one_step(or_system* s, int t)
{
  s->run_step = t;
  if (constraints_rescale(s)) or_build_nlist(s);
  for (int i = 0; i < s->N; i++) enforce_one(s, i);
  reset_forces(s);
  reset_torques(s);
  if (s->npairs + s->nexts) potential_compute(s, s->dt_global);
  if (s->naligns) aligner_compute(s);
  for (int k = 0; k < s->ninteg; k++) integrate(s, &s->integ[k]);
  if (s->has_nlist && (s->npairs + s->naligns) > 0) {
    int rebuild = 0;
    for (int i = 0; i < s->N; i++)
      if (need_update(s, i)) { rebuild = 1; break; }
    if (rebuild) or_build_nlist(s);
  }
  s->time_step++;
}

int or_run(or_system* s, int steps)
{
  if (s->npairs + s->nexts) potential_compute(s, s->dt_global);
  if (s->naligns) aligner_compute(s);
  for (int t = 0; t <= steps; t++) one_step(s, t);
  return 0;
}

int or_run_until_converged(or_system* s, int max_steps)
{
  if (s->npairs + s->nexts) potential_compute(s, s->dt_global);
  if (s->naligns) aligner_compute(s);
  for (int t = 0; t <= max_steps; t++) {
    one_step(s, t);
    int all = 1;
    for (int k = 0; k < s->ninteg; k++)
      if (s->integ[k].kind == OR_INT_FIRE && !s->integ[k].converged) all = 0;
    if (all) return t + 1;
  }
  return -1;
}
