// sg_hot.cuh -- the hot step kernels (sm_100a) for the two shapes the
// benchmarks run: active Brownian particles on a periodic plane and on a
// sphere, integrated by brownian / brownian_pos / brownian_align.
//
// The fields a neighbour sweep reads are packed into one 32-byte record per
// particle and moved with 256-bit loads/stores (ld.global.nc.v4.f64):
//   plane : G[k] = {x, y, nx, ny}             (+ radius from the SoA array)
//   sphere: G[k] = {x, y, z, r}, H[k] = {nx, ny, nz, 0}
// so one neighbour costs two 32-byte sectors.  G/H are double-buffered
// (step t reads buffer b, writes 1-b); every other per-particle field stays
// in the structure-of-arrays store and is updated in place by its owner.
// The arithmetic is the same sequence as the generic kernels (sg_kernels.cuh),
// specialised: on the plane z = zpos, n_z = v_z = f_z = 0 exactly after the
// start-of-step enforce, so those terms are dropped without changing a bit.
#pragma once
#include "sg_kernels.cuh"

namespace sg {

// hot-shape eligibility (host side)
enum { HOT_NONE = 0, HOT_PLANE = 1, HOT_SPHERE = 2 };

// ---------------------------------------------------------------------------
// pack / unpack between the SoA store and the packed records
// ---------------------------------------------------------------------------
template <int SHAPE>
__global__ void k_hot_pack(const Replica* __restrict__ reps, const int* __restrict__ blk_rep, Dyn d, Stat st,
                           D4* __restrict__ G, D4* __restrict__ H, const int* __restrict__ blist = nullptr) {
  const int bid_ = blist ? blist[blockIdx.x] : (int)blockIdx.x;  // block of the packed layout
  const Replica& R = reps[blk_rep[bid_]];
  const int k = bid_ * BLOCK + threadIdx.x;
  if (k - R.off >= R.n) return;
  if (SHAPE == HOT_PLANE) {
    stg4(G + k, D4{d.x[k], d.y[k], d.nx[k], d.ny[k]});
  } else {
    stg4(G + k, D4{d.x[k], d.y[k], d.z[k], st.r[k]});
    stg4(H + k, D4{d.nx[k], d.ny[k], d.nz[k], 0.0});
  }
}

template <int SHAPE>
__global__ void k_hot_unpack(const Replica* __restrict__ reps, const int* __restrict__ blk_rep, Dyn d,
                             const D4* __restrict__ G, const D4* __restrict__ H, const int* __restrict__ blist = nullptr) {
  const int bid_ = blist ? blist[blockIdx.x] : (int)blockIdx.x;  // block of the packed layout
  const Replica& R = reps[blk_rep[bid_]];
  const int k = bid_ * BLOCK + threadIdx.x;
  if (k - R.off >= R.n) return;
  const D4 g = ldg4(G + k);
  d.x[k] = g.x; d.y[k] = g.y;
  if (SHAPE == HOT_PLANE) {
    d.nx[k] = g.z; d.ny[k] = g.w;
  } else {
    d.z[k] = g.z;
    const D4 h = ldg4(H + k);
    d.nx[k] = h.x; d.ny[k] = h.y; d.nz[k] = h.z;
  }
}

// The start-of-step Constrainer::enforce of a run's first step (samos.cpp:
// 887-888) fused with the packing: the plane or sphere enforce on the fields
// it reads and writes only (the generic enforce pass moves every field of
// the particle), then the packed records.  Plane: z = zpos, vz = fz = nz = 0,
// periodic wrap with image flags, director normalised; sphere: projection of
// position, velocity and director.
template <int SHAPE>
__global__ void k_hot_pack_enforce(const Replica* __restrict__ reps, const int* __restrict__ blk_rep, Dyn d,
                                   Stat st, D4* __restrict__ G, D4* __restrict__ H, int unlimited) {
  const Replica& R = reps[blk_rep[blockIdx.x]];
  const int k = blockIdx.x * BLOCK + threadIdx.x;
  if (k - R.off >= R.n) return;
  Part p;
  if (SHAPE == HOT_PLANE) {
    p.x = d.x[k]; p.y = d.y[k]; p.z = 0.0; p.vz = 0.0; p.fz = 0.0;
    p.nx = d.nx[k]; p.ny = d.ny[k]; p.nz = 0.0;
    p.ix = d.ix[k]; p.iy = d.iy[k]; p.iz = 0;
    const int ix0 = p.ix, iy0 = p.iy;
    plane_enforce(R, R.cons_p[0], unlimited, p);  // zpos inside the box: z never wraps
    if (p.ix != ix0) { d.x[k] = p.x; d.ix[k] = p.ix; }
    if (p.iy != iy0) { d.y[k] = p.y; d.iy[k] = p.iy; }
    d.z[k] = p.z; d.vz[k] = 0.0; d.fz[k] = 0.0; d.nz[k] = 0.0;
    d.nx[k] = p.nx; d.ny[k] = p.ny;
    stg4(G + k, D4{p.x, p.y, p.nx, p.ny});
  } else {
    p.x = d.x[k]; p.y = d.y[k]; p.z = d.z[k];
    p.vx = d.vx[k]; p.vy = d.vy[k]; p.vz = d.vz[k];
    p.nx = d.nx[k]; p.ny = d.ny[k]; p.nz = d.nz[k];
    sphere_enforce(R.cons_p[0], p);
    d.x[k] = p.x; d.y[k] = p.y; d.z[k] = p.z;
    d.vx[k] = p.vx; d.vy[k] = p.vy; d.vz[k] = p.vz;
    d.nx[k] = p.nx; d.ny[k] = p.ny; d.nz[k] = p.nz;
    stg4(G + k, D4{p.x, p.y, p.z, st.r[k]});
    stg4(H + k, D4{p.nx, p.ny, p.nz, 0.0});
  }
}

// ---------------------------------------------------------------------------
// per-particle pieces specialised to the shapes
// ---------------------------------------------------------------------------
struct Hp {  // hot particle registers
  double x, y, z, nx, ny, nz, vx, vy, vz, fx, fy, fz, tx, ty, tz, omega, r;
  int type, id;
};

// ConstraintPlane::enforce on a periodic box (constraint_plane.cpp:36-89);
// z = zpos, vz = fz = nz = 0 are implicit in the planar registers.
__device__ __forceinline__ void hot_plane_enforce(double xlo, double xhi, double Lx, double ylo, double yhi,
                                                  double Ly, Hp& p, int& dix, int& diy) {
  if (p.x <= xlo) { p.x += Lx; dix--; } else if (p.x > xhi) { p.x -= Lx; dix++; }
  if (p.y <= ylo) { p.y += Ly; diy--; } else if (p.y > yhi) { p.y -= Ly; diy++; }
  double len_n = sqrt(p.nx * p.nx + p.ny * p.ny);
  double inv_len = 1.0;
  if (len_n != 0.0) inv_len = 1.0 / len_n;
  p.nx *= inv_len; p.ny *= inv_len;
}

// ConstraintPlane::rotate_director (constraint_plane.cpp:97-114)
__device__ __forceinline__ void hot_plane_rotate(Hp& p, double phi, bool velocity) {
  double cs, sn;
  sincos(phi, &sn, &cs);
  double nx = cs * p.nx + -sn * p.ny;
  double ny = sn * p.nx + cs * p.ny;
  double len = sqrt(nx * nx + ny * ny);
  p.nx = nx / len; p.ny = ny / len;
  if (velocity) {  // ConstraintPlane::rotate_velocity (122-143)
    double vx = cs * p.vx + -sn * p.vy;
    double vy = sn * p.vx + cs * p.vy;
    p.vx = vx; p.vy = vy;
  }
}

// ConstraintSphere::enforce (constraint_sphere.cpp:38-81)
__device__ __forceinline__ void hot_sphere_enforce(double Rs, Hp& p) {
  double Rr = sqrt(p.x * p.x + p.y * p.y + p.z * p.z);
  double s = Rs / Rr;
  p.x *= s; p.y *= s; p.z *= s;
  double Nx = p.x / Rs, Ny = p.y / Rs, Nz = p.z / Rs;
  double v_dot_N = p.vx * Nx + p.vy * Ny + p.vz * Nz;
  double n_dot_N = p.nx * Nx + p.ny * Ny + p.nz * Nz;
  p.vx -= v_dot_N * Nx; p.vy -= v_dot_N * Ny; p.vz -= v_dot_N * Nz;
  p.nx -= n_dot_N * Nx; p.ny -= n_dot_N * Ny; p.nz -= n_dot_N * Nz;
  double inv_len = 1.0 / sqrt(p.nx * p.nx + p.ny * p.ny + p.nz * p.nz);
  p.nx *= inv_len; p.ny *= inv_len; p.nz *= inv_len;
}

// Constraint::rotate_director / rotate_velocity about the sphere normal
// (constraint.cpp:96-150)
__device__ __forceinline__ void hot_sphere_rotate(double Rs, Hp& p, double phi, bool velocity) {
  double U = p.x / Rs, V = p.y / Rs, W = p.z / Rs;
  double cs, sn;
  sincos(phi, &sn, &cs);
  double dot = U * p.nx + V * p.ny + W * p.nz;
  double nx = U * dot * (1.0 - cs) + p.nx * cs + (-W * p.ny + V * p.nz) * sn;
  double ny = V * dot * (1.0 - cs) + p.ny * cs + (W * p.nx - U * p.nz) * sn;
  double nz = W * dot * (1.0 - cs) + p.nz * cs + (-V * p.nx + U * p.ny) * sn;
  double len = sqrt(nx * nx + ny * ny + nz * nz);
  p.nx = nx / len; p.ny = ny / len; p.nz = nz / len;
  if (velocity) {
    double dv = U * p.vx + V * p.vy + W * p.vz;
    double vx = U * dv * (1.0 - cs) + p.vx * cs + (-W * p.vy + V * p.vz) * sn;
    double vy = V * dv * (1.0 - cs) + p.vy * cs + (W * p.vx - U * p.vz) * sn;
    double vz = W * dv * (1.0 - cs) + p.vz * cs + (-V * p.vx + U * p.vy) * sn;
    p.vx = vx; p.vy = vy; p.vz = vz;
  }
}

// Box/constraint scalars the shape routines read (plane: box; sphere: Rs).
struct ShapeGeom { double xlo, xhi, Lx, ylo, yhi, Ly, Rs; };

__device__ __forceinline__ ShapeGeom geom_of(const Replica& R) {
  return ShapeGeom{R.xlo, R.xhi, R.Lx, R.ylo, R.yhi, R.Ly, R.cons_p[0]};
}

template <int SHAPE>
__device__ __forceinline__ void hot_enforce(const ShapeGeom& G, Hp& p, int& dix, int& diy) {
  if (SHAPE == HOT_PLANE) hot_plane_enforce(G.xlo, G.xhi, G.Lx, G.ylo, G.yhi, G.Ly, p, dix, diy);
  else hot_sphere_enforce(G.Rs, p);
}

template <int SHAPE>
__device__ __forceinline__ double hot_project_torque(const ShapeGeom& G, const Hp& p) {
  if (SHAPE == HOT_PLANE) return 0.0 + p.tz;
  const double Rs = G.Rs;
  double Nx = p.x / Rs, Ny = p.y / Rs, Nz = p.z / Rs;
  return 0.0 + (p.tx * Nx + p.ty * Ny + p.tz * Nz);
}

template <int SHAPE>
__device__ __forceinline__ void hot_rotate(const ShapeGeom& G, Hp& p, double phi, bool velocity) {
  if (SHAPE == HOT_PLANE) hot_plane_rotate(p, phi, velocity);
  else hot_sphere_rotate(G.Rs, p, phi, velocity);
}

// ---------------------------------------------------------------------------
// the hot step kernel
// ---------------------------------------------------------------------------
template <int SHAPE, bool ENERGY>
__global__ void __launch_bounds__(BLOCK, 4)
k_hot_step(Program P, const Replica* __restrict__ reps, const int* __restrict__ blk_rep,
           const Clock* __restrict__ clk, const D4* __restrict__ Gin, D4* __restrict__ Gout,
           const D4* __restrict__ Hin, D4* __restrict__ Hout, Dyn d, Stat st, NbList nl,
           int* __restrict__ rebuild, int* __restrict__ status, double dt_global, int apply_e1, int last,
           double* epart, int nblocks) {
  const int r = my_replica(blk_rep);
  if (clk[r].halt) return;  // batched stepping: a rebuild is pending
  const Replica& R = reps[r];
  const int k = blockIdx.x * BLOCK + threadIdx.x;
  double e[MAX_PAIR + MAX_ALIGN];
#pragma unroll
  for (int i = 0; i < MAX_PAIR + MAX_ALIGN; i++) e[i] = 0.0;
  if (k - R.off < R.n) {
    Hp p;
    {
      const D4 g = ldg4(Gin + k);
      p.x = g.x; p.y = g.y;
      if (SHAPE == HOT_PLANE) { p.z = 0.0; p.nx = g.z; p.ny = g.w; p.nz = 0.0; p.r = st.r[k]; }
      else {
        p.z = g.z; p.r = g.w;
        const D4 h = ldg4(Hin + k);
        p.nx = h.x; p.ny = h.y; p.nz = h.z;
      }
    }
    p.id = st.id[k];
    p.type = P.ntypes > 1 ? st.type[k] : 1;
    p.fx = 0.0; p.fy = 0.0; p.fz = 0.0; p.tx = 0.0; p.ty = 0.0; p.tz = 0.0;
    p.vx = 0.0; p.vy = 0.0; p.vz = 0.0;

    // ---- forces and torques (pair c and aligner c share sweep c) ----------
    const int cnt = nl.cnt[k], lo = nl.lo[k];
    const int nloops = P.npair > P.nalign ? P.npair : P.nalign;
    bool need_r = false;
    for (int c = 0; c < P.npair; c++) need_r = need_r || P.pair[c].use_radii;
    Part me;  // view for pair_term
    me.r = p.r; me.type = p.type;
    for (int c = 0; c < nloops; c++) {
      const bool hp = c < P.npair, ha = c < P.nalign;
      const PairComp pc = P.pair[hp ? c : 0];
      const int akind = ha ? P.align[c].kind : -1;
      const bool app = ha && P.align[c].has_pp;
      double Jg = ha ? R.align_J[c] : 0.0;
      if (akind == ALIGN_NEMATIC) Jg = 2.0 * Jg;
      const double rcg = ha ? R.align_rcut[c] : 0.0;
      const double* g = R.pair_g[hp ? c : 0];
#pragma unroll 2
      for (int q = 0; q < cnt; q++) {
        const int j = __ldg(nl.nb + (size_t)q * nl.stride + k);
        Nb o;
        double dx, dy, dz;
        const D4 gj = ldg4(Gin + j);
        if (SHAPE == HOT_PLANE) {
          o.x = gj.x; o.y = gj.y; o.nx = gj.z; o.ny = gj.w; o.nz = 0.0;
          o.r = need_r ? __ldg(st.r + j) : 1.0;
          dx = o.x - p.x; dy = o.y - p.y; dz = 0.0;
          if (dx > R.xhi) dx -= R.Lx; else if (dx < R.xlo) dx += R.Lx;
          if (dy > R.yhi) dy -= R.Ly; else if (dy < R.ylo) dy += R.Ly;
        } else {
          o.x = gj.x; o.y = gj.y; o.z = gj.z; o.r = gj.w;
          if (ha) { const D4 hj = ldg4(Hin + j); o.nx = hj.x; o.ny = hj.y; o.nz = hj.z; }
          dx = o.x - p.x; dy = o.y - p.y; dz = o.z - p.z;
          apply_periodic(R, dx, dy, dz);
        }
        o.type = (P.ntypes > 1) ? __ldg(st.type + j) : 1;
        const double r_sq = (SHAPE == HOT_PLANE) ? dx * dx + dy * dy : dx * dx + dy * dy + dz * dz;
        const bool upper = q >= lo;
        if (hp) {
          double ff, pe;
          if (pair_term(pc, g, P.ntypes, me, o, r_sq, 1.0, ff, pe)) {
            p.fx -= ff * dx; p.fy -= ff * dy;
            if (SHAPE != HOT_PLANE) p.fz -= ff * dz;
            if (ENERGY && upper) e[c] += pe;
          }
        }
        if (ha) {
          double J = Jg, rcut = rcg;
          if (app) {
            const double* t = P.align[c].table + ((size_t)(p.type - 1) * P.ntypes + (size_t)(o.type - 1)) * 2;
            J = t[0]; rcut = t[1];
          }
          if (r_sq <= rcut * rcut) {
            if (SHAPE == HOT_PLANE) {
              const double tau_z = p.nx * o.ny - p.ny * o.nx;
              if (akind == ALIGN_POLAR) {
                p.tz += J * tau_z;
                if (ENERGY && upper) e[MAX_PAIR + c] += -2.0 * J * (p.nx * o.nx + p.ny * o.ny);
              } else {
                const double cdot = p.nx * o.nx + p.ny * o.ny;
                p.tz += J * cdot * tau_z;
                if (ENERGY && upper) e[MAX_PAIR + c] += -2.0 * J * (2.0 * cdot * cdot - 1.0);
              }
            } else {
              const double tau_x = p.ny * o.nz - p.nz * o.ny;
              const double tau_y = p.nz * o.nx - p.nx * o.nz;
              const double tau_z = p.nx * o.ny - p.ny * o.nx;
              if (akind == ALIGN_POLAR) {
                p.tx += J * tau_x; p.ty += J * tau_y; p.tz += J * tau_z;
                if (ENERGY && upper) e[MAX_PAIR + c] += -2.0 * J * (p.nx * o.nx + p.ny * o.ny + p.nz * o.nz);
              } else {
                const double cdot = p.nx * o.nx + p.ny * o.ny + p.nz * o.nz;
                p.tx += J * cdot * tau_x; p.ty += J * cdot * tau_y; p.tz += J * cdot * tau_z;
                if (ENERGY && upper) e[MAX_PAIR + c] += -2.0 * J * (2.0 * cdot * cdot - 1.0);
              }
            }
          }
        }
      }
    }
    for (int c = 0; c < P.next; c++) {  // external_self_propulsion.cpp:33-50
      double alpha = R.ext_alpha[c];
      if (P.ext[c].has_params) alpha = P.ext[c].type_alpha[p.type - 1];
      p.fx += alpha * p.nx; p.fy += alpha * p.ny;
      if (SHAPE != HOT_PLANE) p.fz += alpha * p.nz;
    }
    const double fx0 = p.fx, fy0 = p.fy, fz0 = p.fz, tx0 = p.tx, ty0 = p.ty, tz0 = p.tz;

    // ---- integrators in map order -----------------------------------------
    const int run_step = clk[r].run_step;
    const ShapeGeom Gm = geom_of(R);
    int dix = 0, diy = 0;
    bool aged = false, vset = false, wset = false;
    double age = 0.0;
    for (int c = 0; c < P.ninteg; c++) {
      const IntegComp ic = P.integ[c];
      const double* ip = R.integ_p[c];
      const uint32_t seed = R.seed[c];
      uint64_t base = clk[r].ctr[c];
      const uint64_t gid = (uint64_t)p.id;
      const double dt = ip[0];
      if (ic.kind == INT_BROWNIAN_ALIGN || ic.kind == INT_BROWNIAN) {
        if (ic.nematic) {
          if (noise_uniform(seed, base + gid) < dt / ip[7]) {
            p.nx = -p.nx; p.ny = -p.ny; p.nz = -p.nz;
            if (ic.kind == INT_BROWNIAN && ic.velocity) { p.vx = -p.vx; p.vy = -p.vy; p.vz = -p.vz; }
          }
          base += (uint64_t)R.n;
        }
      }
      if (ic.kind == INT_BROWNIAN) {  // integrator_brownian.cpp:72-121
        const double v0 = ip[1], nu = ip[2], mu = ip[3], mur = ip[4];
        const double T = value_get(ic.temp, run_step);
        const int D = T > 0.0 ? 4 : 1;
        const uint64_t c0 = base + gid * (uint64_t)D;
        double fd_x = v0 * p.nx + mu * p.fx;
        double fd_y = v0 * p.ny + mu * p.fy;
        double fd_z = v0 * p.nz + mu * p.fz;
        p.vx = fd_x; p.vy = fd_y; p.vz = fd_z;
        vset = true; wset = true;
        p.x += dt * fd_x; p.y += dt * fd_y;
        if (SHAPE != HOT_PLANE) p.z += dt * fd_z;
        if (T > 0.0) {
          const double B = sqrt(2.0 * mu * T), sqrt_dt = sqrt(dt);
          double fr_x = B * noise_gauss(seed, c0 + 0);
          double fr_y = B * noise_gauss(seed, c0 + 1);
          p.vx += fr_x; p.vy += fr_y;
          p.x += sqrt_dt * fr_x; p.y += sqrt_dt * fr_y;
          if (SHAPE != HOT_PLANE) {
            double fr_z = B * noise_gauss(seed, c0 + 2);
            p.vz += fr_z; p.z += sqrt_dt * fr_z;
          }
        }
        hot_enforce<SHAPE>(Gm, p, dix, diy);
        if (SHAPE == HOT_PLANE) p.vz = 0.0;
        p.omega = mur * hot_project_torque<SHAPE>(Gm, p);
        double dtheta = dt * p.omega + sqrt(nu * dt) * noise_gauss(seed, c0 + (uint64_t)(D - 1));
        hot_rotate<SHAPE>(Gm, p, dtheta, ic.velocity != 0);
        if (!aged) { age = d.age[k]; aged = true; }
        age += dt;
      } else if (ic.kind == INT_BROWNIAN_POS) {  // integrator_brownian_pos.cpp:52-81
        const double mu = ip[3];
        const double T = value_get(ic.temp, run_step);
        p.vx = mu * p.fx; p.vy = mu * p.fy; p.vz = mu * p.fz;
        vset = true;
        p.x += dt * p.vx; p.y += dt * p.vy;
        if (SHAPE != HOT_PLANE) p.z += dt * p.vz;
        if (T > 0.0) {
          const uint64_t c0 = base + gid * 3u;
          const double B = sqrt(2.0 * mu * T), sqrt_dt = sqrt(dt);
          double fr_x = B * noise_gauss(seed, c0 + 0);
          double fr_y = B * noise_gauss(seed, c0 + 1);
          p.vx += fr_x; p.vy += fr_y;
          p.x += sqrt_dt * fr_x; p.y += sqrt_dt * fr_y;
          if (SHAPE != HOT_PLANE) {
            double fr_z = B * noise_gauss(seed, c0 + 2);
            p.vz += fr_z; p.z += sqrt_dt * fr_z;
          }
        }
        hot_enforce<SHAPE>(Gm, p, dix, diy);
        if (SHAPE == HOT_PLANE) p.vz = 0.0;
        if (!aged) { age = d.age[k]; aged = true; }
        age += dt;
      } else if (ic.kind == INT_BROWNIAN_ALIGN) {  // integrator_brownian_align.cpp:63-75
        const double nu = ip[2], mur = ip[4];
        p.omega = mur * hot_project_torque<SHAPE>(Gm, p);
        wset = true;
        double dtheta = dt * p.omega + sqrt(nu * dt) * noise_gauss(seed, base + gid);
        hot_rotate<SHAPE>(Gm, p, dtheta, false);
      }
    }

    // ---- skin test on the post-integration position ------------------------
    {
      double ddx = nl.ox[k] - p.x, ddy = nl.oy[k] - p.y, ddz = 0.0;
      if (SHAPE != HOT_PLANE) ddz = nl.oz[k] - p.z;
      if (R.periodic) {
        if (ddx > R.xhi) ddx -= R.Lx; else if (ddx < R.xlo) ddx += R.Lx;
        if (ddy > R.yhi) ddy -= R.Ly; else if (ddy < R.ylo) ddy += R.Ly;
        if (SHAPE != HOT_PLANE) { if (ddz > R.zhi) ddz -= R.Lz; else if (ddz < R.zlo) ddz += R.Lz; }
      }
      const double d2 = (SHAPE == HOT_PLANE) ? ddx * ddx + ddy * ddy : ddx * ddx + ddy * ddy + ddz * ddz;
      if (!(d2 < 0.25 * R.pad * R.pad)) {
        if (rebuild[r] == 0) atomicOr(&rebuild[r], 1);
      }
    }
    if (!(isfinite(p.x) && isfinite(p.y) && isfinite(p.z))) atomicOr(status, ST_NONFINITE);
    if (apply_e1) hot_enforce<SHAPE>(Gm, p, dix, diy);  // next step's Constrainer::enforce

    // ---- stores -------------------------------------------------------------
    if (SHAPE == HOT_PLANE) {
      stg4(Gout + k, D4{p.x, p.y, p.nx, p.ny});
      if (vset) { d.vx[k] = p.vx; d.vy[k] = p.vy; }
    } else {
      stg4(Gout + k, D4{p.x, p.y, p.z, p.r});
      stg4(Hout + k, D4{p.nx, p.ny, p.nz, 0.0});
      if (vset) { d.vx[k] = p.vx; d.vy[k] = p.vy; d.vz[k] = p.vz; }
    }
    if (aged) d.age[k] = age;
    if (dix) d.ix[k] += dix;
    if (diy) d.iy[k] += diy;
    if (last) {
      if (wset) d.omega[k] = p.omega;
      d.fx[k] = fx0; d.fy[k] = fy0; d.fz[k] = SHAPE == HOT_PLANE ? 0.0 : fz0;
      d.tx[k] = tx0; d.ty[k] = ty0; d.tz[k] = tz0;
    }
  }
  if (ENERGY) block_reduce_store<MAX_PAIR + MAX_ALIGN>(e, epart, nblocks);
}

}  // namespace sg
