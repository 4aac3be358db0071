// sg_kernels.cuh -- sm_100a kernels of the SAMoS hot path.
//
// Layout: particles of all replicas live in one packed slot range; replica r
// owns slots [off_r, off_r + n_r) padded to BLOCK, so a thread block never
// straddles two replicas and finds its replica through blk_rep[].  Inside a
// replica the slots are kept in cell order (rebuilt with the neighbour list)
// and Stat::id maps a slot back to the particle id of the reference.
//
// Neighbour lists are full lists stored slot-major (nb[q * stride + k]) so a
// warp reads 32 consecutive ints per neighbour rank.  For particle k the list
// holds first its lower-id neighbours in ascending id, then its higher-id
// neighbours in the reference's list[k] order (27-cell stencil order, or
// ascending id on the N^2 path).  Gathering in that order reproduces the
// summation order of the reference's half-list scatter loops exactly.
#pragma once
#include "sg_device.cuh"

namespace sg {

__device__ __forceinline__ int my_replica(const int* blk_rep) { return blk_rep[blockIdx.x]; }

// ---------------------------------------------------------------------------
// neighbour data fetch (only the fields the program needs)
// ---------------------------------------------------------------------------
struct Need { bool r, type, n, v, age; };

__device__ __forceinline__ void fetch_nb(const Dyn& d, const Stat& st, int j, const Need& nd, Nb& o) {
  o.x = d.x[j]; o.y = d.y[j]; o.z = d.z[j];
  if (nd.r) o.r = st.r[j];
  o.type = nd.type ? st.type[j] : 1;
  if (nd.n) { o.nx = d.nx[j]; o.ny = d.ny[j]; o.nz = d.nz[j]; }
  if (nd.v) { o.vx = d.vx[j]; o.vy = d.vy[j]; o.vz = d.vz[j]; }
  if (nd.age) o.age = d.age[j];
}

__device__ __forceinline__ Need program_needs(const Program& P) {
  Need nd{false, P.ntypes > 1, false, false, false};
  for (int c = 0; c < P.npair; c++) {
    if (P.pair[c].use_radii) nd.r = true;
    if (P.pair[c].phase_in) nd.age = true;
  }
  for (int c = 0; c < P.nalign; c++) {
    if (P.align[c].kind == ALIGN_VICSEK) nd.v = true; else nd.n = true;
    if (P.align[c].has_pp) nd.type = true;
  }
  return nd;
}

// ---------------------------------------------------------------------------
// force + torque gather for one particle.  Component loop c handles pair
// potential c and aligner c (std::map order each); forces and torques are
// separate accumulators, so sharing the neighbour sweep keeps each one's
// summation order.  Pair energies are counted once, on the lower id.
// ---------------------------------------------------------------------------
template <bool ENERGY>
__device__ void compute_ft(const Program& P, const Replica& R, const Dyn& d, const Stat& st,
                           const NbList& nl, int k, Part& me, double dt, bool with_pair,
                           bool with_align, double* epair, double* ealign) {
  me.fx = 0.0; me.fy = 0.0; me.fz = 0.0;
  me.tx = 0.0; me.ty = 0.0; me.tz = 0.0;
  const Need nd = program_needs(P);
  const int cnt = nl.cnt[k], lo = nl.lo[k];
  const int npair = with_pair ? P.npair : 0;
  const int nalign = with_align ? P.nalign : 0;
  const int nloops = npair > nalign ? npair : nalign;
  for (int c = 0; c < nloops; c++) {
    const bool hp = c < npair, ha = c < nalign;
    PairComp pc; AlignComp ac;
    double a_i = 1.0, Jg = 0.0, rcg = 0.0;
    int akind = -1;
    if (hp) { pc = P.pair[c]; if (pc.phase_in) a_i = phase_factor(pc, me.age, dt); }
    if (ha) {
      ac = P.align[c]; akind = ac.kind;
      Jg = R.align_J[c]; rcg = R.align_rcut[c];
      if (akind == ALIGN_NEMATIC) Jg = 2.0 * Jg;  // pair_nematic_aligner.cpp:37
    }
    const double* g = R.pair_g[hp ? c : 0];
    for (int q = 0; q < cnt; q++) {
      const int j = nl.nb[(size_t)q * nl.stride + k];
      Nb o;
      fetch_nb(d, st, j, nd, o);
      double dx = o.x - me.x, dy = o.y - me.y, dz = o.z - me.z;
      apply_periodic(R, dx, dy, dz);
      const double r_sq = dx * dx + dy * dy + dz * dz;
      const bool upper = q >= lo;
      if (hp) {
        double alpha = 1.0;
        if (pc.phase_in) alpha = phase_pair(a_i, phase_factor(pc, o.age, dt));
        double ff, pe;
        if (pair_term(pc, g, P.ntypes, me, o, r_sq, alpha, ff, pe)) {
          me.fx -= ff * dx; me.fy -= ff * dy; me.fz -= ff * dz;
          if (ENERGY && upper) epair[c] += pe;
        }
      }
      if (ha) {
        double J = Jg, rcut = rcg;
        if (ac.has_pp) {
          const double* t = ac.table + ((size_t)(me.type - 1) * P.ntypes + (size_t)(o.type - 1)) * 2;
          J = t[0]; rcut = t[1];
        }
        if (r_sq <= rcut * rcut) {
          if (akind == ALIGN_VICSEK) {
            me.tx += o.vx; me.ty += o.vy; me.tz += o.vz;
          } else {
            double tau_x = me.ny * o.nz - me.nz * o.ny;
            double tau_y = me.nz * o.nx - me.nx * o.nz;
            double tau_z = me.nx * o.ny - me.ny * o.nx;
            if (akind == ALIGN_POLAR) {
              me.tx += J * tau_x; me.ty += J * tau_y; me.tz += J * tau_z;
              if (ENERGY && upper) ealign[c] += -2.0 * J * (me.nx * o.nx + me.ny * o.ny + me.nz * o.nz);
            } else {
              double cdot = me.nx * o.nx + me.ny * o.ny + me.nz * o.nz;
              me.tx += J * cdot * tau_x; me.ty += J * cdot * tau_y; me.tz += J * cdot * tau_z;
              if (ENERGY && upper) ealign[c] += -2.0 * J * (2.0 * cdot * cdot - 1.0);
            }
          }
        }
      }
    }
    if (ha && akind == ALIGN_VICSEK) {  // pair_vicsek_aligner.cpp:72-82
      me.tx += me.vx; me.ty += me.vy; me.tz += me.vz;
      double v = sqrt(me.tx * me.tx + me.ty * me.ty + me.tz * me.tz);
      if (v == 0.0) v = 1.0;
      double inv_v = 1.0 / v;
      me.tx *= inv_v; me.ty *= inv_v; me.tz *= inv_v;
    }
  }
  if (with_pair) {
    for (int c = 0; c < P.next; c++) {  // external_self_propulsion.cpp:33-50
      double alpha = R.ext_alpha[c];
      if (P.ext[c].has_params) alpha = P.ext[c].type_alpha[me.type - 1];
      me.fx += alpha * me.nx; me.fy += alpha * me.ny; me.fz += alpha * me.nz;
    }
  }
}

// block reduction of up to NV doubles into out[v * nblocks + blockIdx.x]
template <int NV>
__device__ __forceinline__ void block_reduce_store(double (&v)[NV], double* out, int nblocks, int slot = -1) {
  __shared__ double sh[NV][BLOCK / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; i++) {
    double x = v[i];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sh[i][w] = x;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0.0;
    for (int i = 0; i < BLOCK / 32; i++) s += sh[threadIdx.x][i];
    out[(size_t)threadIdx.x * nblocks + (slot < 0 ? (int)blockIdx.x : slot)] = s;
  }
}

// ---------------------------------------------------------------------------
// integrators (per particle).  `g` is the particle's position in its group
// (the particle id for group "all"); noise counters follow the reference's
// draw order: optional nematic flip draws for every particle first, then per
// particle the translational draws followed by the rotational one.
// ---------------------------------------------------------------------------

// IntegratorBrownian::integrate, integrators/integrator_brownian.cpp:42-124
__device__ __forceinline__ void integ_brownian(const Program& P, const Replica& R, const IntegComp& ic,
                                               const double* ip, uint32_t seed, uint64_t base,
                                               int run_step, int n, uint64_t g, Part& p) {
  const double dt = ip[0], v0 = ip[1], nu = ip[2], mu = ip[3], mur = ip[4];
  if (ic.nematic) {
    double flip = dt / ip[7];
    if (noise_uniform(seed, base + g) < flip) {
      p.nx = -p.nx; p.ny = -p.ny; p.nz = -p.nz;
      if (ic.velocity) { p.vx = -p.vx; p.vy = -p.vy; p.vz = -p.vz; }
    }
    base += (uint64_t)n;
  }
  const double T = value_get(ic.temp, run_step);
  const int D = T > 0.0 ? 4 : 1;
  const uint64_t c0 = base + g * (uint64_t)D;
  double fd_x = v0 * p.nx + mu * p.fx;
  double fd_y = v0 * p.ny + mu * p.fy;
  double fd_z = v0 * p.nz + mu * p.fz;
  p.vx = fd_x; p.vy = fd_y; p.vz = fd_z;
  p.x += dt * fd_x; p.y += dt * fd_y; p.z += dt * fd_z;
  if (T > 0.0) {
    const double B = sqrt(2.0 * mu * T);
    const double sqrt_dt = sqrt(dt);
    double fr_x = B * noise_gauss(seed, c0 + 0);
    double fr_y = B * noise_gauss(seed, c0 + 1);
    double fr_z = B * noise_gauss(seed, c0 + 2);
    p.vx += fr_x; p.vy += fr_y; p.vz += fr_z;
    p.x += sqrt_dt * fr_x; p.y += sqrt_dt * fr_y; p.z += sqrt_dt * fr_z;
  }
  enforce_all(P, R, p);
  p.omega = mur * project_torque(P, R, p);
  const double stoch = sqrt(nu * dt);
  double dtheta = dt * p.omega + stoch * noise_gauss(seed, c0 + (uint64_t)(D - 1));
  rotate_director(P, R, p, dtheta);
  if (ic.velocity) rotate_velocity(P, R, p, dtheta);
  p.age += dt;
}

// IntegratorBrownianPos::integrate, integrators/integrator_brownian_pos.cpp:37-84
__device__ __forceinline__ void integ_brownian_pos(const Program& P, const Replica& R, const IntegComp& ic,
                                                   const double* ip, uint32_t seed, uint64_t base,
                                                   int run_step, uint64_t g, Part& p) {
  const double dt = ip[0], mu = ip[3];
  const double T = value_get(ic.temp, run_step);
  p.vx = mu * p.fx; p.vy = mu * p.fy; p.vz = mu * p.fz;
  p.x += dt * p.vx; p.y += dt * p.vy; p.z += dt * p.vz;
  if (T > 0.0) {
    const uint64_t c0 = base + g * 3u;
    const double B = sqrt(2.0 * mu * T);
    const double sqrt_dt = sqrt(dt);
    double fr_x = B * noise_gauss(seed, c0 + 0);
    double fr_y = B * noise_gauss(seed, c0 + 1);
    double fr_z = B * noise_gauss(seed, c0 + 2);
    p.vx += fr_x; p.vy += fr_y; p.vz += fr_z;
    p.x += sqrt_dt * fr_x; p.y += sqrt_dt * fr_y; p.z += sqrt_dt * fr_z;
  }
  enforce_all(P, R, p);
  p.age += dt;
}

// IntegratorBrownianAlign::integrate, integrators/integrator_brownian_align.cpp:41-76
__device__ __forceinline__ void integ_brownian_align(const Program& P, const Replica& R, const IntegComp& ic,
                                                     const double* ip, uint32_t seed, uint64_t base,
                                                     int n, uint64_t g, Part& p) {
  const double dt = ip[0], nu = ip[2], mur = ip[4];
  if (ic.nematic) {
    double flip = dt / ip[7];
    if (noise_uniform(seed, base + g) < flip) { p.nx = -p.nx; p.ny = -p.ny; p.nz = -p.nz; }
    base += (uint64_t)n;
  }
  p.omega = mur * project_torque(P, R, p);
  const double stoch = sqrt(nu * dt);
  double dtheta = dt * p.omega + stoch * noise_gauss(seed, base + g);
  rotate_director(P, R, p, dtheta);
}

// IntegratorVicsek::integrate, integrators/integrator_vicsek.cpp:44-82: the
// velocity follows the (normalised) Vicsek torque vector, v0 tau + mu F, and
// is turned by a uniform angle of width eta sqrt(dt); one uniform draw per
// particle.
__device__ __forceinline__ void integ_vicsek(const Program& P, const Replica& R, const double* ip, uint32_t seed,
                                             uint64_t base, uint64_t g, Part& p) {
  const double dt = ip[0], v0 = ip[1], eta = ip[2], mu = ip[3];
  const double noise = eta * sqrt(dt);
  p.vx = v0 * p.tx + mu * p.fx;
  p.vy = v0 * p.ty + mu * p.fy;
  p.vz = v0 * p.tz + mu * p.fz;
  enforce_all(P, R, p);
  const double theta = 2.0 * noise * 3.14159265358979323846 * (noise_uniform(seed, base + g) - 0.5);
  rotate_velocity(P, R, p, theta);
  p.x += dt * p.vx; p.y += dt * p.vy; p.z += dt * p.vz;
  enforce_all(P, R, p);
  p.age += dt;
}

// noise draws consumed per call by integrator c of a replica of n particles
__host__ __device__ inline uint64_t draws_per_call(const IntegComp& ic, int run_step, int n) {
  double T = value_get(ic.temp, run_step);
  switch (ic.kind) {
    case INT_BROWNIAN: return (uint64_t)n * ((ic.nematic ? 1u : 0u) + (T > 0.0 ? 4u : 1u));
    case INT_BROWNIAN_POS: return T > 0.0 ? (uint64_t)n * 3u : 0u;
    case INT_BROWNIAN_ALIGN: return (uint64_t)n * ((ic.nematic ? 1u : 0u) + 1u);
    case INT_VICSEK: return (uint64_t)n;
    default: return 0u;
  }
}

// ---------------------------------------------------------------------------
// skin test, NeighbourList::need_update (neighbour_list.cpp:278-302)
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool need_update(const Replica& R, const NbList& nl, int k, const Part& p) {
  double dx = nl.ox[k] - p.x, dy = nl.oy[k] - p.y, dz = nl.oz[k] - p.z;
  if (R.periodic) {
    if (dx > R.xhi) dx -= R.Lx; else if (dx < R.xlo) dx += R.Lx;
    if (dy > R.yhi) dy -= R.Ly; else if (dy < R.ylo) dy += R.Ly;
    if (dz > R.zhi) dz -= R.Lz; else if (dz < R.zlo) dz += R.Lz;
  }
  return !(dx * dx + dy * dy + dz * dz < 0.25 * R.pad * R.pad);
}

__device__ __forceinline__ bool finite3(double a, double b, double c) {
  return isfinite(a) && isfinite(b) && isfinite(c);
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

// Constrainer::enforce on every particle (samos.cpp:887-888)
__global__ void k_enforce(Program P, const Replica* __restrict__ reps, const int* __restrict__ blk_rep,
                          Dyn d, Stat st, const Clock* __restrict__ frozen, const int* __restrict__ blist = nullptr) {
  const int bid_ = blist ? blist[blockIdx.x] : (int)blockIdx.x;  // block of the packed layout
  const int r = blk_rep[bid_];
  const Replica& R = reps[r];
  const int k = bid_ * BLOCK + threadIdx.x;
  if (k - R.off >= R.n) return;
  if (frozen && (frozen[r].fire_conv_step >= 0 || frozen[r].halt)) return;  // minimiser stopped / batch halted
  Part p;
  load_dyn(d, k, p);
  p.id = st.id[k]; p.type = st.type[k]; p.r = st.r[k]; p.mass = st.mass[k];
  enforce_all(P, R, p);
  store_dyn_moved<false, false>(d, k, p);  // the enforce writes no torque, omega or age
}

// reset + Potential::compute + Aligner::compute, storing F, tau and the
// per-block energy partials (pair c at row c, aligner c at row MAX_PAIR + c)
template <bool ENERGY>
__global__ void k_force(Program P, const Replica* __restrict__ reps, const int* __restrict__ blk_rep,
                        const Clock* __restrict__ clk, Dyn d, Stat st, NbList nl, double dt,
                        int use_fire_dt, int with_pair, int with_align, double* epart, int nblocks, const int* __restrict__ blist = nullptr) {
  const int bid_ = blist ? blist[blockIdx.x] : (int)blockIdx.x;  // block of the packed layout
  const int r = blk_rep[bid_];
  if (clk[r].halt) return;  // batched iterations: a rebuild is pending
  const Replica& R = reps[r];
  if (use_fire_dt) {
    if (clk[r].fire_conv_step >= 0) return;  // converged replica: whole block exits (partials kept)
    dt = clk[r].fire_dt;
  }
  const int k = bid_ * BLOCK + threadIdx.x;
  double e[MAX_PAIR + MAX_ALIGN];
#pragma unroll
  for (int i = 0; i < MAX_PAIR + MAX_ALIGN; i++) e[i] = 0.0;
  if (k - R.off < R.n) {
    Part me;
    me.x = d.x[k]; me.y = d.y[k]; me.z = d.z[k];
    me.nx = d.nx[k]; me.ny = d.ny[k]; me.nz = d.nz[k];
    me.vx = d.vx[k]; me.vy = d.vy[k]; me.vz = d.vz[k];
    me.age = d.age[k]; me.r = st.r[k]; me.type = st.type[k];
    compute_ft<ENERGY>(P, R, d, st, nl, k, me, dt, with_pair != 0, with_align != 0, e, e + MAX_PAIR);
    if (with_pair) { d.fx[k] = me.fx; d.fy[k] = me.fy; d.fz[k] = me.fz; }
    if (with_align) { d.tx[k] = me.tx; d.ty[k] = me.ty; d.tz[k] = me.tz; }
  }
  if (ENERGY) block_reduce_store<MAX_PAIR + MAX_ALIGN>(e, epart, nblocks, bid_);
}

// Fused Brownian-family step: F, tau from the current buffer, integrators in
// map order, skin test, then (apply_e1) the next step's start-of-step
// Constrainer::enforce; result into the next buffer.
// MINB: blocks per SM the register allocation is bounded for (8: 64
// registers with some spills, 6: 80); the engine times both on a run's first
// steps and keeps the faster, since which one wins depends on the program.
template <bool ENERGY, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB)
k_step_brownian(Program P, const Replica* __restrict__ reps, const int* __restrict__ blk_rep,
                const Clock* __restrict__ clk, Dyn cur, Dyn nxt, Stat st, NbList nl,
                int* __restrict__ rebuild, int* __restrict__ status, double dt_global, int apply_e1,
                double* epart, int nblocks, const uint8_t* __restrict__ gmask, const int* __restrict__ grank,
                int slots) {
  const int r = my_replica(blk_rep);
  if (clk[r].halt) return;  // batched stepping: a rebuild is pending, this step does not run
  const Replica& R = reps[r];
  const int k = blockIdx.x * BLOCK + threadIdx.x;
  double e[MAX_PAIR + MAX_ALIGN];
#pragma unroll
  for (int i = 0; i < MAX_PAIR + MAX_ALIGN; i++) e[i] = 0.0;
  if (k - R.off < R.n) {
    Part p;
    load_dyn(cur, k, p);
    p.id = st.id[k]; p.type = st.type[k]; p.r = st.r[k]; p.mass = st.mass[k];
    compute_ft<ENERGY>(P, R, cur, st, nl, k, p, dt_global, true, true, e, e + MAX_PAIR);
    const int run_step = clk[r].run_step;
    for (int c = 0; c < P.ninteg; c++) {
      const IntegComp ic = P.integ[c];
      const uint64_t base = clk[r].ctr[c];
      // a grouped integrator moves its members only, drawing in group order
      // (IntegratorBrownian::integrate loops over the group's particles)
      uint64_t g = (uint64_t)p.id;
      int n = R.n;
      if (ic.group) {
        if (!((gmask[R.off + p.id] >> ic.group) & 1u)) continue;
        g = (uint64_t)grank[(size_t)ic.group * slots + R.off + p.id];
        n = R.gsize[ic.group];
      }
      if (ic.kind == INT_BROWNIAN)
        integ_brownian(P, R, ic, R.integ_p[c], R.seed[c], base, run_step, n, g, p);
      else if (ic.kind == INT_BROWNIAN_POS)
        integ_brownian_pos(P, R, ic, R.integ_p[c], R.seed[c], base, run_step, g, p);
      else if (ic.kind == INT_BROWNIAN_ALIGN)
        integ_brownian_align(P, R, ic, R.integ_p[c], R.seed[c], base, n, g, p);
      else if (ic.kind == INT_VICSEK)
        integ_vicsek(P, R, R.integ_p[c], R.seed[c], base, g, p);
    }
    if (need_update(R, nl, k, p)) {
      if (rebuild[r] == 0) atomicOr(&rebuild[r], 1);
    }
    if (!finite3(p.x, p.y, p.z)) atomicOr(status, ST_NONFINITE);
    if (apply_e1) enforce_all(P, R, p);
    store_dyn(nxt, k, p);
  }
  if (ENERGY) block_reduce_store<MAX_PAIR + MAX_ALIGN>(e, epart, nblocks);
}

// Skin test over all particles of the current buffer (unfused path)
__global__ void k_skin(Program P, const Replica* __restrict__ reps, const int* __restrict__ blk_rep,
                       Dyn d, NbList nl, int* __restrict__ rebuild, int* __restrict__ status, const int* __restrict__ blist = nullptr) {
  const int bid_ = blist ? blist[blockIdx.x] : (int)blockIdx.x;  // block of the packed layout
  const int r = blk_rep[bid_];
  const Replica& R = reps[r];
  const int k = bid_ * BLOCK + threadIdx.x;
  if (k - R.off >= R.n) return;
  Part p;
  p.x = d.x[k]; p.y = d.y[k]; p.z = d.z[k];
  if (need_update(R, nl, k, p)) {
    if (rebuild[r] == 0) atomicOr(&rebuild[r], 1);
  }
  if (!finite3(p.x, p.y, p.z)) atomicOr(status, ST_NONFINITE);
}

// noise draws consumed per call by a Langevin integrator
__host__ __device__ inline uint64_t langevin_draws(const IntegComp& ic, const double* ip, int run_step, int n) {
  const double T = value_get(ic.temp, run_step);
  const double dt = ip[0], gamma = ip[9];
  if (ic.method == LANGEVIN_SPV) return sqrt(T * (1.0 - exp(-2.0 * gamma * dt))) != 0.0 ? (uint64_t)n * 3u : 0u;
  if (ic.method == LANGEVIN_BBK) return sqrt(2.0 * T * dt * gamma) != 0.0 ? (uint64_t)n * 3u : 0u;
  return sqrt(T * (1.0 - exp(-2.0 * gamma * dt))) != 0.0 ? (uint64_t)n * 3u : 0u;
}

// per-replica clock advance after one integration step
// end-of-step bookkeeping of replica r: noise counters and step counters
__device__ __forceinline__ void tail_one(const Program& P, const Replica& R, Clock& C) {
  for (int c = 0; c < P.ninteg; c++) {
    const IntegComp& ic = P.integ[c];
    if (ic.kind == INT_LANGEVIN) C.ctr[c] += langevin_draws(ic, R.integ_p[c], C.run_step, R.n);
    else C.ctr[c] += draws_per_call(ic, C.run_step, ic.group ? R.gsize[ic.group] : R.n);
  }
  C.run_step++;
  C.time_step++;
}

__global__ void k_tail(Program P, const Replica* __restrict__ reps, Clock* clk, int nrep) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrep) return;
  tail_one(P, reps[r], clk[r]);
}

// Tail of one step of a batch enqueued without host synchronisation (one
// block).  If an earlier step of the batch flagged a rebuild, the step just
// enqueued did nothing (its kernel saw the halt) and neither does this.
// Otherwise the step counts as executed, and if it flagged a rebuild every
// replica is halted until the host has rebuilt the lists.
__global__ void k_tail_batch(Program P, const Replica* __restrict__ reps, Clock* clk, int nrep,
                             const int* __restrict__ rebuild, int* __restrict__ executed) {
  __shared__ int halted, any;
  if (threadIdx.x == 0) { halted = clk[0].halt; any = 0; }
  __syncthreads();
  if (halted) return;
  for (int r = threadIdx.x; r < nrep; r += blockDim.x) {
    tail_one(P, reps[r], clk[r]);
    if (rebuild[r]) atomicOr(&any, 1);
  }
  __syncthreads();
  if (any)
    for (int r = threadIdx.x; r < nrep; r += blockDim.x) clk[r].halt = 1;
  if (threadIdx.x == 0) (*executed)++;
}

__global__ void k_set_halt(Clock* clk, int nrep, int v) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < nrep) clk[r].halt = v;
}

// ---------------------------------------------------------------------------
// Langevin (integrators/integrator_langevin.cpp): phase A before and phase B
// after the integrator's own force evaluation.
// ---------------------------------------------------------------------------
// pre_enforce: the start-of-step enforce (samos.cpp:887-888) folded in, when
// no force pass comes between it and this half (forces reused)
__global__ void k_langevin_a(Program P, const Replica* __restrict__ reps, const int* __restrict__ blk_rep,
                             const Clock* __restrict__ clk, Dyn d, Stat st, int c, const double* Rn, int pre_enforce) {
  const int r = my_replica(blk_rep);
  if (clk[r].halt) return;  // batched stepping: a rebuild is pending
  const Replica& R = reps[r];
  const int k = blockIdx.x * BLOCK + threadIdx.x;
  if (k - R.off >= R.n) return;
  Part p;
  load_dyn(d, k, p);
  p.id = st.id[k]; p.type = st.type[k]; p.r = st.r[k]; p.mass = st.mass[k];
  if (pre_enforce) enforce_all(P, R, p);
  const IntegComp ic = P.integ[c];
  const double* ip = R.integ_p[c];
  const double dt = ip[0], gamma = ip[9];
  const double T = value_get(ic.temp, clk[r].run_step);
  const double dt2 = 0.5 * dt;
  const uint32_t seed = R.seed[c];
  const uint64_t base = clk[r].ctr[c];
  if (ic.method == LANGEVIN_SPV) {  // integrator_langevin.cpp:136-146
    p.x += dt2 * p.vx; p.y += dt2 * p.vy; p.z += dt2 * p.vz;
    enforce_all(P, R, p);
  } else if (ic.method == LANGEVIN_BBK) {  // integrator_langevin.cpp:203-223
    const double B = sqrt(2.0 * T * dt * gamma);
    const double one_m_dt2 = 1.0 - gamma * dt2;
    const double dt2_over_mass = dt2 / p.mass;
    p.vx = one_m_dt2 * p.vx + dt2_over_mass * p.fx;
    p.vy = one_m_dt2 * p.vy + dt2_over_mass * p.fy;
    p.vz = one_m_dt2 * p.vz + dt2_over_mass * p.fz;
    if (B != 0.0) {
      const double stoch_fact = 0.5 * B / sqrt(p.mass);
      const size_t gi = (size_t)R.off + (size_t)p.id;
      p.vx += stoch_fact * Rn[3 * gi + 0];
      p.vy += stoch_fact * Rn[3 * gi + 1];
      p.vz += stoch_fact * Rn[3 * gi + 2];
    }
    p.x += dt * p.vx; p.y += dt * p.vy; p.z += dt * p.vz;
    enforce_all(P, R, p);
  } else {  // BAOAB, integrator_langevin.cpp:63-95
    const double B = sqrt(T * (1.0 - exp(-2.0 * gamma * dt)));
    const double exp_dt = exp(-gamma * dt);
    const double fact = dt2 / p.mass;
    p.vx += fact * p.fx; p.vy += fact * p.fy; p.vz += fact * p.fz;
    p.x += dt2 * p.vx; p.y += dt2 * p.vy; p.z += dt2 * p.vz;
    enforce_all(P, R, p);
    p.vx *= exp_dt; p.vy *= exp_dt; p.vz *= exp_dt;
    if (B != 0.0) {
      const double stoch_fact = B / sqrt(p.mass);
      const uint64_t c0 = base + (uint64_t)p.id * 3u;
      p.vx += stoch_fact * noise_gauss(seed, c0 + 0);
      p.vy += stoch_fact * noise_gauss(seed, c0 + 1);
      p.vz += stoch_fact * noise_gauss(seed, c0 + 2);
    }
    p.x += dt2 * p.vx; p.y += dt2 * p.vy; p.z += dt2 * p.vz;
    enforce_all(P, R, p);
  }
  store_dyn_moved<false, false>(d, k, p);
}

// skin: the step's skin test (neighbour_list.cpp:278-302) on the final
// positions, folded in
__global__ void k_langevin_b(Program P, const Replica* __restrict__ reps, const int* __restrict__ blk_rep,
                             const Clock* __restrict__ clk, Dyn d, Stat st, int c, double* Rn, NbList nl,
                             int* __restrict__ rebuild, int* __restrict__ status, int skin) {
  const int r = my_replica(blk_rep);
  if (clk[r].halt) return;  // batched stepping: a rebuild is pending
  const Replica& R = reps[r];
  const int k = blockIdx.x * BLOCK + threadIdx.x;
  if (k - R.off >= R.n) return;
  Part p;
  load_dyn(d, k, p);
  p.id = st.id[k]; p.type = st.type[k]; p.r = st.r[k]; p.mass = st.mass[k];
  const IntegComp ic = P.integ[c];
  const double* ip = R.integ_p[c];
  const double dt = ip[0], gamma = ip[9];
  const double T = value_get(ic.temp, clk[r].run_step);
  const double dt2 = 0.5 * dt;
  const uint32_t seed = R.seed[c];
  const uint64_t base = clk[r].ctr[c];
  if (ic.method == LANGEVIN_SPV) {  // integrator_langevin.cpp:158-183
    const double zeta = sqrt(T * (1.0 - exp(-2.0 * gamma * dt)));
    const double eta = (gamma == 0.0) ? 0.0 : (1.0 - exp(-dt * gamma)) / gamma;
    const double exp_dt = exp(-dt * gamma);
    const double fact = eta / p.mass;
    p.vx = exp_dt * p.vx + fact * p.fx;
    p.vy = exp_dt * p.vy + fact * p.fy;
    p.vz = exp_dt * p.vz + fact * p.fz;
    if (zeta != 0.0) {
      const double stoch_fact = zeta / sqrt(p.mass);
      const uint64_t c0 = base + (uint64_t)p.id * 3u;
      p.vx += stoch_fact * noise_gauss(seed, c0 + 0);
      p.vy += stoch_fact * noise_gauss(seed, c0 + 1);
      p.vz += stoch_fact * noise_gauss(seed, c0 + 2);
    }
    p.x += dt2 * p.vx; p.y += dt2 * p.vy; p.z += dt2 * p.vz;
    enforce_all(P, R, p);
    p.age += dt;
  } else if (ic.method == LANGEVIN_BBK) {  // integrator_langevin.cpp:232-252
    const double B = sqrt(2.0 * T * dt * gamma);
    const double one_div_one_p_dt2 = 1.0 / (1.0 + gamma * dt2);
    const double dt2_over_mass = dt2 / p.mass;
    p.vx = one_div_one_p_dt2 * (p.vx + dt2_over_mass * p.fx);
    p.vy = one_div_one_p_dt2 * (p.vy + dt2_over_mass * p.fy);
    p.vz = one_div_one_p_dt2 * (p.vz + dt2_over_mass * p.fz);
    if (B != 0.0) {
      const double stoch_fact = 0.5 * B * one_div_one_p_dt2 / sqrt(p.mass);
      const uint64_t c0 = base + (uint64_t)p.id * 3u;
      const size_t gi = (size_t)R.off + (size_t)p.id;
      double rx = noise_gauss(seed, c0 + 0), ry = noise_gauss(seed, c0 + 1), rz = noise_gauss(seed, c0 + 2);
      Rn[3 * gi + 0] = rx; Rn[3 * gi + 1] = ry; Rn[3 * gi + 2] = rz;
      p.vx += stoch_fact * rx; p.vy += stoch_fact * ry; p.vz += stoch_fact * rz;
      p.age += dt;
    }
  } else {  // BAOAB final B step, integrator_langevin.cpp:104-111
    const double fact = dt2 / p.mass;
    p.vx += fact * p.fx; p.vy += fact * p.fy; p.vz += fact * p.fz;
    p.age += dt;
  }
  store_dyn_moved<false, true>(d, k, p);
  if (skin) {
    if (need_update(R, nl, k, p) && rebuild[r] == 0) atomicOr(&rebuild[r], 1);
    if (!finite3(p.x, p.y, p.z)) atomicOr(status, ST_NONFINITE);
  }
}

// ---------------------------------------------------------------------------
// NVE (integrators/integrator_nve.cpp:37-141).  The first three loops act on
// each particle alone, so one thread runs them in sequence; then the force
// pass; then the last loop.  Limits: params 12 has_limit, 13 limit,
// 14 has_angle_limit, 15 angle_limit (absent limits are off; the omega clamp
// of the last loop needs both, the reference reading an unset angle limit
// there).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double sign_of(double x) { return x >= 0.0 ? 1.0 : -1.0; }  // integrator_nve.hpp:38

__global__ void k_nve_a(Program P, const Replica* __restrict__ reps, const int* __restrict__ blk_rep,
                        const Clock* __restrict__ clk, Dyn d, Stat st, int c, int pre_enforce) {
  const int r = my_replica(blk_rep);
  if (clk[r].halt) return;  // batched stepping: a rebuild is pending
  const Replica& R = reps[r];
  const int k = blockIdx.x * BLOCK + threadIdx.x;
  if (k - R.off >= R.n) return;
  Part p;
  load_dyn(d, k, p);
  p.id = st.id[k]; p.type = st.type[k]; p.r = st.r[k]; p.mass = st.mass[k];
  if (pre_enforce) enforce_all(P, R, p);  // as in k_langevin_a
  const double* ip = R.integ_p[c];
  const double dt = ip[0], dt_2 = 0.5 * dt;
  const bool has_limit = ip[12] != 0.0, has_theta = ip[14] != 0.0;
  const double limit = ip[13], theta_limit = ip[15];
  p.vx += dt_2 * p.fx; p.vy += dt_2 * p.fy; p.vz += dt_2 * p.fz;  // nve.cpp:49-55
  enforce_all(P, R, p);
  p.omega += dt_2 * project_torque(P, R, p);
  double dx = dt * p.vx, dy = dt * p.vy, dz = dt * p.vz;  // nve.cpp:57-76
  if (has_limit) {
    const double dr = sqrt(dx * dx + dy * dy + dz * dz);
    if (dr > limit) { dx = limit * dx / dr; dy = limit * dy / dr; dz = limit * dz / dr; }
  }
  p.x += dx; p.y += dy; p.z += dz;
  enforce_all(P, R, p);
  double dtheta = dt * p.omega;  // nve.cpp:78-86
  if (has_theta && fabs(dtheta) > theta_limit) dtheta = sign_of(dtheta) * theta_limit;
  rotate_director(P, R, p, dtheta);
  store_dyn_moved<true, false>(d, k, p);
}

__global__ void k_nve_b(Program P, const Replica* __restrict__ reps, const int* __restrict__ blk_rep,
                        const Clock* __restrict__ clk, Dyn d, Stat st, int c, NbList nl, int* __restrict__ rebuild,
                        int* __restrict__ status, int skin) {
  const int r = my_replica(blk_rep);
  if (clk[r].halt) return;  // batched stepping: a rebuild is pending
  const Replica& R = reps[r];
  const int k = blockIdx.x * BLOCK + threadIdx.x;
  if (k - R.off >= R.n) return;
  Part p;
  load_dyn(d, k, p);
  p.id = st.id[k]; p.type = st.type[k]; p.r = st.r[k]; p.mass = st.mass[k];
  const double* ip = R.integ_p[c];
  const double dt = ip[0], dt_2 = 0.5 * dt;
  const bool has_limit = ip[12] != 0.0, has_theta = ip[14] != 0.0;
  const double limit = ip[13], theta_limit = ip[15];
  p.vx += dt_2 * p.fx; p.vy += dt_2 * p.fy; p.vz += dt_2 * p.fz;  // nve.cpp:93-120
  if (has_limit) {
    const double v = sqrt(p.vx * p.vx + p.vy * p.vy + p.vz * p.vz);
    if (v * dt > limit) {
      p.vx = p.vx / v * limit / dt;
      p.vy = p.vy / v * limit / dt;
      p.vz = p.vz / v * limit / dt;
    }
  }
  enforce_all(P, R, p);
  p.omega += dt_2 * project_torque(P, R, p);
  if (has_limit && has_theta && fabs(p.omega) * dt > theta_limit) p.omega = sign_of(p.omega) * theta_limit / dt;
  p.age += dt;
  store_dyn_moved<true, true>(d, k, p);
  if (skin) {  // as in k_langevin_b
    if (need_update(R, nl, k, p) && rebuild[r] == 0) atomicOr(&rebuild[r], 1);
    if (!finite3(p.x, p.y, p.z)) atomicOr(status, ST_NONFINITE);
  }
}

// ---------------------------------------------------------------------------
// FIRE (integrators/integrator_fire.cpp:34-148)
// ---------------------------------------------------------------------------
// first half: half kick, drift, enforce, omega, director rotation (49-66)
__global__ void k_fire_a(Program P, const Replica* __restrict__ reps, const int* __restrict__ blk_rep,
                         const Clock* __restrict__ clk, Dyn d, Stat st, int pre_enforce,
                         const int* __restrict__ blist = nullptr) {
  const int bid_ = blist ? blist[blockIdx.x] : (int)blockIdx.x;  // block of the packed layout
  const int r = blk_rep[bid_];
  const Replica& R = reps[r];
  const int k = bid_ * BLOCK + threadIdx.x;
  if (k - R.off >= R.n) return;
  if (clk[r].fire_conv_step >= 0 || clk[r].halt) return;  // frozen after convergence / batch halted
  Part p;
  load_dyn(d, k, p);
  p.id = st.id[k]; p.type = st.type[k]; p.r = st.r[k]; p.mass = st.mass[k];
  // the step's start-of-step enforce (k_enforce), when no force pass lies
  // between them (the forces of the previous iteration are reused)
  if (pre_enforce) enforce_all(P, R, p);
  const double dt = clk[r].fire_dt;
  const double dt_2 = 0.5 * dt;
  p.vx += dt_2 * p.fx; p.vy += dt_2 * p.fy; p.vz += dt_2 * p.fz;
  p.x += dt * p.vx; p.y += dt * p.vy; p.z += dt * p.vz;
  enforce_all(P, R, p);
  p.omega += dt_2 * project_torque(P, R, p);
  double dtheta = dt * p.omega;
  rotate_director(P, R, p, dtheta);
  store_dyn_moved<true, false>(d, k, p);
}

// The per-replica sums of the block partials, taken by all threads of the
// replica's last block: thread t sums blocks b0 + t, b0 + t + BLOCK, ... in
// order, then a fixed tree over the threads (the same bits for a replica run
// alone or inside an ensemble).  Returns P, |F|^2, |v|^2, max |F_i|^2, E on
// thread 0.
__device__ void fire_sums(const Program& P, const double* part, const double* epart, int nblocks, int b0, int nb,
                          double out[5]) {
  __shared__ double red[5][BLOCK];
  const int t = threadIdx.x;
  double Ps = 0.0, Fn = 0.0, Vn = 0.0, Fm = 0.0, E = 0.0;
  for (int b = b0 + t; b < b0 + nb; b += BLOCK) {  // other blocks' partials, so past L1
    Ps += __ldcg(part + b); Fn += __ldcg(part + (size_t)nblocks + b); Vn += __ldcg(part + (size_t)2 * nblocks + b);
    Fm = fmax(Fm, __ldcg(part + (size_t)3 * nblocks + b));
  }
  for (int pc = 0; pc < P.npair; pc++)
    for (int b = b0 + t; b < b0 + nb; b += BLOCK) E += __ldcg(epart + (size_t)pc * nblocks + b);
  red[0][t] = Ps; red[1][t] = Fn; red[2][t] = Vn; red[3][t] = Fm; red[4][t] = E;
  __syncthreads();
  for (int h = BLOCK / 2; h > 0; h >>= 1) {
    if (t < h) {
      red[0][t] += red[0][t + h]; red[1][t] += red[1][t + h]; red[2][t] += red[2][t + h];
      red[3][t] = fmax(red[3][t], red[3][t + h]); red[4][t] += red[4][t + h];
    }
    __syncthreads();
  }
  if (t == 0)
    for (int i = 0; i < 5; i++) out[i] = red[i][0];
}

// FIRE's convergence test and dt / alpha control on the replica's sums
// (integrator_fire.cpp:96-147).  alpha_mix[r] keeps the alpha the mixing step
// must use (the value before this update).
__device__ void fire_control(const Replica& R, Clock& C, int r, int c, const double sums[5], int driver,
                             double* alpha_mix) {
  if (C.fire_conv_step >= 0 || C.halt) return;
  const double* ip = R.integ_p[c];
  double Ps = sums[0], Fn = sums[1], Vn = sums[2], Fm = sums[3], E = sums[4];
  Fn = sqrt(Fn);
  Vn = sqrt(Vn);
  C.fire_P = Ps; C.fire_F = Fn; C.fire_V = Vn; C.fire_E = E; C.fire_Fmax2 = Fm;
  const double sqrt_ndof = sqrt((double)(3 * R.n));
  const double fmax_tol = ip[11];
  const bool conv = (fmax_tol > 0.0) ? (sqrt(Fm) < fmax_tol)
                                     : (Fn / sqrt_ndof < ip[3] && fabs(E - C.fire_old_e) < ip[4]);
  if (conv) {
    C.fire_converged = 1;
    if (driver) C.fire_conv_step = C.run_step;
    return;
  }
  alpha_mix[r] = C.fire_alpha;
  if (Ps > 0.0) {
    C.fire_last_neg++;
    if (C.fire_last_neg > (int)ip[9]) {
      double ndt = C.fire_dt * ip[6];
      C.fire_dt = ndt < ip[8] ? ndt : ip[8];
      C.fire_alpha *= ip[2];
    }
  } else {
    C.fire_dt *= ip[7];
    C.fire_alpha = ip[1];
    C.fire_last_neg = 0;
  }
  C.fire_converged = 0;
  C.fire_old_e = E;
}

// second half kick + P, |F|^2, |v|^2, max|F|^2 partials (79-94)
// ... and, in the replica's last block to finish, the per-replica sums, the
// convergence test and the dt / alpha control (96-147) of fire_control: the
// blocks of a replica count themselves done on fire_cnt[r] after their
// partials are visible, so the last one sees them all.
// Reference-order sums (the parity mode): P, |F|^2 and |v|^2 accumulated one
// particle at a time in particle-id order, as the reference's loop over the
// group does (integrator_fire.cpp:79-94), from the per-particle terms in
// `terms` (three arrays of `stride` doubles, indexed by replica offset + id).
// One warp: 32 terms loaded at a time, then added in order through shuffles,
// so every lane holds the same sequential sums.
__device__ void fire_ordered_sums(const double* __restrict__ terms, int stride, int off, int n, double out[3]) {
  const int lane = threadIdx.x & 31;
  double sP = 0.0, sF = 0.0, sV = 0.0;
  for (int base = 0; base < n; base += 32) {
    const int i = base + lane;
    const double a = i < n ? __ldcg(terms + off + i) : 0.0;
    const double b = i < n ? __ldcg(terms + (size_t)stride + off + i) : 0.0;
    const double v = i < n ? __ldcg(terms + (size_t)2 * stride + off + i) : 0.0;
    const int m = n - base < 32 ? n - base : 32;
    for (int u = 0; u < m; u++) {
      sP += __shfl_sync(0xffffffffu, a, u);
      sF += __shfl_sync(0xffffffffu, b, u);
      sV += __shfl_sync(0xffffffffu, v, u);
    }
  }
  out[0] = sP; out[1] = sF; out[2] = sV;
}

__global__ void k_fire_b(Program P, const Replica* __restrict__ reps, const int* __restrict__ blk_rep,
                         Clock* __restrict__ clk, Dyn d, Stat st, double* part, int nblocks, const int* rep_blk0,
                         const int* rep_nblk, const double* epart, int c, int driver, double* alpha_mix,
                         int* __restrict__ fire_cnt, const int* __restrict__ blist = nullptr,
                         double* __restrict__ terms = nullptr, int terms_stride = 0) {
  const int bid_ = blist ? blist[blockIdx.x] : (int)blockIdx.x;  // block of the packed layout
  const int r = blk_rep[bid_];
  const Replica& R = reps[r];
  const int k = bid_ * BLOCK + threadIdx.x;
  double v[3] = {0.0, 0.0, 0.0};
  double fmax2 = 0.0;
  if (clk[r].halt) return;  // batched iterations: a rebuild is pending (k_fire_c skips too)
  const bool frozen = clk[r].fire_conv_step >= 0;
  if (k - R.off < R.n && !frozen) {
    Part p;
    load_dyn(d, k, p);
    p.id = st.id[k]; p.type = st.type[k]; p.r = st.r[k]; p.mass = st.mass[k];
    const double dt_2 = 0.5 * clk[r].fire_dt;
    p.vx += dt_2 * p.fx; p.vy += dt_2 * p.fy; p.vz += dt_2 * p.fz;
    v[0] = p.vx * p.fx + p.vy * p.fy + p.vz * p.fz;
    double f2 = p.fx * p.fx + p.fy * p.fy + p.fz * p.fz;
    v[1] = f2;
    fmax2 = f2;
    v[2] = p.vx * p.vx + p.vy * p.vy + p.vz * p.vz;
    if (terms) {  // parity mode: the per-particle terms, by particle id
      const size_t q = (size_t)R.off + (size_t)p.id;
      terms[q] = v[0]; terms[(size_t)terms_stride + q] = v[1]; terms[(size_t)2 * terms_stride + q] = v[2];
    }
    enforce_all(P, R, p);
    p.omega += dt_2 * project_torque(P, R, p);
    store_dyn_moved<true, false>(d, k, p);
  }
  block_reduce_store<3>(v, part, nblocks, bid_);
  // max reduction (exact in any order)
  for (int o = 16; o > 0; o >>= 1) fmax2 = fmax(fmax2, __shfl_down_sync(0xffffffffu, fmax2, o));
  __shared__ double shm[BLOCK / 32];
  if ((threadIdx.x & 31) == 0) shm[threadIdx.x >> 5] = fmax2;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int i = 0; i < BLOCK / 32; i++) m = fmax(m, shm[i]);
    part[(size_t)3 * nblocks + bid_] = m;
  }
  if (frozen) return;  // whole block: a frozen replica takes no control step
  __shared__ int amlast;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) amlast = atomicAdd(&fire_cnt[r], 1) == rep_nblk[r] - 1;
  __syncthreads();
  if (amlast) {  // block-uniform
    __threadfence();
    double sums[5];
    fire_sums(P, part, epart, nblocks, rep_blk0[r], rep_nblk[r], sums);
    if (terms && threadIdx.x < 32) {  // parity mode: P, |F|^2, |v|^2 in the reference's order
      double o[3];
      fire_ordered_sums(terms, terms_stride, R.off, R.n, o);
      if (threadIdx.x == 0) { sums[0] = o[0]; sums[1] = o[1]; sums[2] = o[2]; }
    }
    if (threadIdx.x == 0) {
      fire_control(R, clk[r], r, c, sums, driver, alpha_mix);
      fire_cnt[r] = 0;
    }
  }
}

// FIRE velocity mixing (110-121) with the pre-update alpha, then the
// P <= 0 restart that zeroes the velocities (131-142).
__global__ void k_fire_d(Program P, const Replica* __restrict__ reps, const int* __restrict__ blk_rep,
                         const Clock* __restrict__ clk, Dyn d, const double* alpha_mix, NbList nl, int skin,
                         int* __restrict__ rebuild, int* __restrict__ status, const int* __restrict__ blist = nullptr) {
  const int bid_ = blist ? blist[blockIdx.x] : (int)blockIdx.x;  // block of the packed layout
  const int r = blk_rep[bid_];
  const Replica& R = reps[r];
  const int k = bid_ * BLOCK + threadIdx.x;
  if (k - R.off >= R.n) return;
  const Clock& C = clk[r];
  if (C.fire_conv_step >= 0 || C.halt) return;  // frozen or halted: positions as the last skin test saw them
  if (!C.fire_converged) {
    const double a = alpha_mix[r];
    const double inv_Fnorm = 1.0 / C.fire_F;
    const double fact_1 = 1.0 - a;
    const double fact_2 = a * inv_Fnorm * C.fire_V;
    double vx = fact_1 * d.vx[k] + fact_2 * d.fx[k];
    double vy = fact_1 * d.vy[k] + fact_2 * d.fy[k];
    double vz = fact_1 * d.vz[k] + fact_2 * d.fz[k];
    if (!(C.fire_P > 0.0)) { vx = 0.0; vy = 0.0; vz = 0.0; }
    d.vx[k] = vx; d.vy[k] = vy; d.vz[k] = vz;
  }
  if (skin) {  // the step's skin test (neighbour_list.cpp:278-302), fused
    Part p;
    p.x = d.x[k]; p.y = d.y[k]; p.z = d.z[k];
    if (need_update(R, nl, k, p)) {
      if (rebuild[r] == 0) atomicOr(&rebuild[r], 1);
    }
    if (!finite3(p.x, p.y, p.z)) atomicOr(status, ST_NONFINITE);
  }
}

// ---------------------------------------------------------------------------
// neighbour-list rebuild: counting-sort cell binning + ordered list build
// (CellList::populate, cell_list.cpp:82-104; NeighbourList::build_cell /
// build_nsq, neighbour_list.cpp:178-273)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int cell_of(const Replica& R, double x, double y, double z, int& a, int& b, int& c) {
  a = (int)((x - R.xlo) / R.cwx);
  b = (int)((y - R.ylo) / R.cwy);
  c = (int)((z - R.zlo) / R.cwz);
  a = a < 0 ? 0 : (a >= R.cnx ? R.cnx - 1 : a);
  b = b < 0 ? 0 : (b >= R.cny ? R.cny - 1 : b);
  c = c < 0 ? 0 : (c >= R.cnz ? R.cnz - 1 : c);
  return R.cny * R.cnz * a + R.cnz * b + c;
}

// populate wrap (no image update) + cell index + count
__global__ void k_rb_bin(const Replica* __restrict__ reps, const int* __restrict__ blk_rep,
                         const int* __restrict__ rebuild, Dyn d, int* __restrict__ pcell,
                         int* __restrict__ cell_cnt, const int* __restrict__ blist = nullptr) {
  const int bid_ = blist ? blist[blockIdx.x] : (int)blockIdx.x;  // block of the packed layout
  const int r = blk_rep[bid_];
  if (!rebuild[r]) return;
  const Replica& R = reps[r];
  const int k = bid_ * BLOCK + threadIdx.x;
  if (k - R.off >= R.n) return;
  double x = d.x[k], y = d.y[k], z = d.z[k];
  if (R.periodic) {
    bool ch = false;
    if (x < R.xlo) { x += R.Lx; ch = true; } else if (x > R.xhi) { x -= R.Lx; ch = true; }
    if (y < R.ylo) { y += R.Ly; ch = true; } else if (y > R.yhi) { y -= R.Ly; ch = true; }
    if (z < R.zlo) { z += R.Lz; ch = true; } else if (z > R.zhi) { z -= R.Lz; ch = true; }
    if (ch) { d.x[k] = x; d.y[k] = y; d.z[k] = z; }
  }
  int a, b, c;
  const int cl = cell_of(R, x, y, z, a, b, c);
  pcell[k] = cl;
  atomicAdd(&cell_cnt[R.cell_off + cl], 1);
}

// exclusive scan of the packed cell counts: A) block sums, B) scan of block
// sums (one block), C) block-local scan plus block prefix
constexpr int SCAN_T = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_T * SCAN_ITEMS;

// The scan runs over the cells of the replicas being rebuilt only: their
// cell ranges, concatenated, form a virtual array (CellSeg.vbase = offset of
// the range in it).  Offsets within one replica's range are what the list
// build uses, and those are the same as in a scan over every cell.
struct CellSeg { int cell_off, ncell, vbase, pad; };

__device__ __forceinline__ int seg_cell(const CellSeg* __restrict__ segs, int nseg, int v) {
  int lo = 0, hi = nseg - 1;  // last segment with vbase <= v
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (segs[mid].vbase <= v) lo = mid; else hi = mid - 1;
  }
  return segs[lo].cell_off + (v - segs[lo].vbase);
}

__global__ void k_seg_zero(const CellSeg* __restrict__ segs, int nseg, int n, int* __restrict__ a, int* __restrict__ b) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const int g = seg_cell(segs, nseg, v);
    a[g] = 0; b[g] = 0;
  }
}

__global__ void k_scan_a(const int* __restrict__ in, int n, const CellSeg* __restrict__ segs, int nseg,
                         int* __restrict__ bsum) {
  __shared__ int sh[SCAN_T / 32];
  const int base = blockIdx.x * SCAN_TILE;
  int s = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++) {
    int idx = base + threadIdx.x * SCAN_ITEMS + i;
    if (idx < n) s += in[seg_cell(segs, nseg, idx)];
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    int v = sh[threadIdx.x];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) bsum[blockIdx.x] = v;
  }
}

__device__ __forceinline__ int block_excl_scan(int v, int* sh_warp, int& total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh_warp[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = lane < (blockDim.x >> 5) ? sh_warp[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    sh_warp[lane] = s;
  }
  __syncthreads();
  total = sh_warp[(blockDim.x >> 5) - 1];
  const int wp = w > 0 ? sh_warp[w - 1] : 0;
  __syncthreads();
  return wp + x - v;
}

__global__ void k_scan_b(int* bsum, int nb) {
  __shared__ int shw[32];
  int carry = 0;
  for (int base = 0; base < nb; base += SCAN_T) {
    int idx = base + threadIdx.x;
    int v = idx < nb ? bsum[idx] : 0;
    int tot;
    int ex = block_excl_scan(v, shw, tot);
    if (idx < nb) bsum[idx] = carry + ex;
    carry += tot;
    __syncthreads();
  }
}

__global__ void k_scan_c(const int* __restrict__ in, int n, const CellSeg* __restrict__ segs, int nseg,
                         const int* __restrict__ bsum, int* __restrict__ out) {
  __shared__ int shw[32];
  const int base = blockIdx.x * SCAN_TILE;
  int v[SCAN_ITEMS], g[SCAN_ITEMS];
  int s = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++) {
    int idx = base + threadIdx.x * SCAN_ITEMS + i;
    g[i] = idx < n ? seg_cell(segs, nseg, idx) : 0;
    v[i] = idx < n ? in[g[i]] : 0;
    s += v[i];
  }
  int tot;
  int ex = block_excl_scan(s, shw, tot) + bsum[blockIdx.x];
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++) {
    int idx = base + threadIdx.x * SCAN_ITEMS + i;
    if (idx < n) out[g[i]] = ex;
    ex += v[i];
  }
}

// unordered placement into the cell segments
__global__ void k_rb_scatter(const Replica* __restrict__ reps, const int* __restrict__ blk_rep,
                             const int* __restrict__ rebuild, const int* __restrict__ pcell,
                             const int* __restrict__ cstart, int* __restrict__ cfill, int* __restrict__ tmp, const int* __restrict__ blist = nullptr) {
  const int bid_ = blist ? blist[blockIdx.x] : (int)blockIdx.x;  // block of the packed layout
  const int r = blk_rep[bid_];
  if (!rebuild[r]) return;
  const Replica& R = reps[r];
  const int k = bid_ * BLOCK + threadIdx.x;
  if (k - R.off >= R.n) return;
  const int cg = R.cell_off + pcell[k];
  const int pos = cstart[cg] - cstart[R.cell_off] + atomicAdd(&cfill[cg], 1);
  tmp[R.off + pos] = k;
}

// rank inside the cell by particle id -> deterministic ascending-id order;
// with `cand`, also the particle's candidate record at its cell-ordered
// position: position, and id and slot packed in the fourth word (the slot it
// will occupy once a re-sort, rebuild[r] == 2, has moved it there)
__device__ __forceinline__ double pack_id_slot(int id, int slot) {
  return __longlong_as_double((long long)(((unsigned long long)(unsigned)id << 32) | (unsigned)slot));
}
__global__ void k_rb_rank(const Replica* __restrict__ reps, const int* __restrict__ blk_rep,
                          const int* __restrict__ rebuild, const int* __restrict__ pcell,
                          const int* __restrict__ cstart, const int* __restrict__ ccnt,
                          const int* __restrict__ tmp, const int* __restrict__ id, int* __restrict__ perm,
                          const int* __restrict__ blist = nullptr, Dyn d = Dyn{}, D4* __restrict__ cand = nullptr) {
  const int bid_ = blist ? blist[blockIdx.x] : (int)blockIdx.x;  // block of the packed layout
  const int r = blk_rep[bid_];
  if (!rebuild[r]) return;
  const Replica& R = reps[r];
  const int k = bid_ * BLOCK + threadIdx.x;
  if (k - R.off >= R.n) return;
  const int cg = R.cell_off + pcell[k];
  const int s0 = R.off + cstart[cg] - cstart[R.cell_off];
  const int n = ccnt[cg];
  const int myid = id[k];
  int rank = 0;
  for (int q = 0; q < n; q++) rank += id[tmp[s0 + q]] < myid ? 1 : 0;
  perm[s0 + rank] = k;
  if (cand)
    stg4(cand + s0 + rank, D4{d.x[k], d.y[k], d.z[k], pack_id_slot(myid, rebuild[r] == 2 ? s0 + rank : k)});
}

// gather all particle arrays into the permuted order (dst = src[perm])
__global__ void k_rb_gather(const Replica* __restrict__ reps, const int* __restrict__ blk_rep,
                            const int* __restrict__ rebuild, const int* __restrict__ perm,
                            Dyn src, Dyn dst, Stat ssrc, Stat sdst, const int* __restrict__ blist = nullptr) {
  const int bid_ = blist ? blist[blockIdx.x] : (int)blockIdx.x;  // block of the packed layout
  const int r = blk_rep[bid_];
  if (rebuild[r] != 2) return;
  const Replica& R = reps[r];
  const int k = bid_ * BLOCK + threadIdx.x;
  if (k - R.off >= R.n) return;
  const int o = perm[k];
  Part p;
  load_dyn(src, o, p);
  store_dyn(dst, k, p);
  sdst.r[k] = ssrc.r[o]; sdst.mass[k] = ssrc.mass[o];
  sdst.type[k] = ssrc.type[o]; sdst.id[k] = ssrc.id[o];
}

// copy back (dst -> src) for the rebuilt replicas
__global__ void k_rb_copyback(const Replica* __restrict__ reps, const int* __restrict__ blk_rep,
                              const int* __restrict__ rebuild, Dyn tmpd, Dyn d, Stat tmps, Stat st, const int* __restrict__ blist = nullptr) {
  const int bid_ = blist ? blist[blockIdx.x] : (int)blockIdx.x;  // block of the packed layout
  const int r = blk_rep[bid_];
  if (rebuild[r] != 2) return;
  const Replica& R = reps[r];
  const int k = bid_ * BLOCK + threadIdx.x;
  if (k - R.off >= R.n) return;
  Part p;
  load_dyn(tmpd, k, p);
  store_dyn(d, k, p);
  st.r[k] = tmps.r[k]; st.mass[k] = tmps.mass[k]; st.type[k] = tmps.type[k]; st.id[k] = tmps.id[k];
}

constexpr int NB_LOCAL = 48;  // lower-id (or, on the N^2 path, each side's) neighbours staged per thread

// Ordered full-list build.  Cell path: the reference's 27-cell stencil with
// periodic index wrap (duplicates kept when a dimension has 2 cells, as in
// cell_list.cpp:52-63); higher-id neighbours are written in visiting order by
// a second sweep.  N^2 path: each distinct neighbour cell once, higher ids
// sorted ascending (build_nsq appends in ascending i).  Lower-id neighbours
// ascending in both.  rebuild[r] == 2: the particle arrays were just put in
// cell order, so cell c's q-th particle sits at its segment slot directly;
// rebuild[r] == 1: the slot comes from the cell-ordered index `cslot`.
__device__ __forceinline__ int build_stencil(const Replica& R, int a, int b, int c, int* cells) {
  int ncells = 0;
  for (int ox = -1; ox <= 1; ox++)
    for (int oy = -1; oy <= 1; oy++)
      for (int oz = -1; oz <= 1; oz++) {
        int ia = a + ox, ib = b + oy, ic = c + oz;
        if (ia < 0) ia = R.cnx - 1; else if (ia == R.cnx) ia = 0;
        if (ib < 0) ib = R.cny - 1; else if (ib == R.cny) ib = 0;
        if (ic < 0) ic = R.cnz - 1; else if (ic == R.cnz) ic = 0;
        const int cl = R.cny * R.cnz * ia + R.cnz * ib + ic;
        bool dup = false;
        if (!R.use_cell)
          for (int q = 0; q < ncells; q++) dup = dup || (cells[q] == cl);
        if (!dup) cells[ncells++] = cl;
      }
  return ncells;
}

// The list of slot k, built by one thread (the reference algorithm as it stands).
__device__ __forceinline__ void build_particle(const Replica& R, int mode, int k, Dyn d, Stat st, NbList nl,
                                              const int* __restrict__ cslot, const int* __restrict__ cstart,
                                              const int* __restrict__ ccnt, int* __restrict__ status,
                                              int* __restrict__ maxnb) {
  const double x = d.x[k], y = d.y[k], z = d.z[k];
  const int myid = st.id[k];
  int a, b, c;
  cell_of(R, x, y, z, a, b, c);
  int cells[27];
  const int ncells = build_stencil(R, a, b, c, cells);
  const int base0 = cstart[R.cell_off];
  unsigned long long lo[NB_LOCAL], up[NB_LOCAL];  // (id << 32) | slot
  int nlo = 0, nup = 0;
  bool overflow = false;
  // One sweep: lower-id neighbours as (id, slot) keys, sorted below; on the
  // cell path the higher-id ones are kept in stencil visiting order (the
  // reference's list[i] order), on the N^2 path as keys sorted by id.
  for (int m = 0; m < ncells; m++) {
    const int cg = R.cell_off + cells[m];
    const int s0 = R.off + cstart[cg] - base0, n = ccnt[cg];
    for (int q = 0; q < n; q++) {
      const int j = mode == 2 ? s0 + q : cslot[s0 + q];
      const int jid = st.id[j];
      if (jid == myid) continue;
      double dx, dy, dz;
      if (myid < jid) { dx = x - d.x[j]; dy = y - d.y[j]; dz = z - d.z[j]; }
      else { dx = d.x[j] - x; dy = d.y[j] - y; dz = d.z[j] - z; }
      apply_periodic(R, dx, dy, dz);
      if (dx * dx + dy * dy + dz * dz < R.cut2) {
        const unsigned long long key = ((unsigned long long)(unsigned)jid << 32) | (unsigned)j;
        if (jid < myid) { if (nlo < NB_LOCAL) lo[nlo] = key; nlo++; }
        else { if (nup < NB_LOCAL) up[nup] = key; nup++; }
      }
    }
  }
  if (nlo > NB_LOCAL || (!R.use_cell && nup > NB_LOCAL)) overflow = true;
  const int total = nlo + nup;
  atomicMax(maxnb, total);
  if (total > nl.cap || overflow) {
    atomicOr(status, ST_OVERFLOW);
    nl.cnt[k] = 0; nl.lo[k] = 0;
  } else {
    for (int i = 1; i < nlo; i++) {  // insertion sort by id (stable: equal ids keep their order)
      const unsigned long long v = lo[i];
      int m = i - 1;
      while (m >= 0 && (lo[m] >> 32) > (v >> 32)) { lo[m + 1] = lo[m]; m--; }
      lo[m + 1] = v;
    }
    for (int q = 0; q < nlo; q++) nl.nb[(size_t)q * nl.stride + k] = (int)(unsigned)(lo[q] & 0xffffffffull);
    if (!R.use_cell) {
      for (int i = 1; i < nup; i++) {
        const unsigned long long v = up[i];
        int m = i - 1;
        while (m >= 0 && (up[m] >> 32) > (v >> 32)) { up[m + 1] = up[m]; m--; }
        up[m + 1] = v;
      }
      for (int q = 0; q < nup; q++)
        nl.nb[(size_t)(nlo + q) * nl.stride + k] = (int)(unsigned)(up[q] & 0xffffffffull);
    } else if (nup <= NB_LOCAL) {
      for (int q = 0; q < nup; q++)
        nl.nb[(size_t)(nlo + q) * nl.stride + k] = (int)(unsigned)(up[q] & 0xffffffffull);
    } else {
      // more higher-id neighbours than the local array holds: a second sweep
      // writes them in stencil visiting order straight into the list
      int w = nlo;
      for (int m = 0; m < ncells; m++) {
        const int cg = R.cell_off + cells[m];
        const int s0 = R.off + cstart[cg] - base0, n = ccnt[cg];
        for (int q = 0; q < n; q++) {
          const int j = mode == 2 ? s0 + q : cslot[s0 + q];
          const int jid = st.id[j];
          if (jid <= myid) continue;
          double dx = x - d.x[j], dy = y - d.y[j], dz = z - d.z[j];
          apply_periodic(R, dx, dy, dz);
          if (dx * dx + dy * dy + dz * dz < R.cut2) nl.nb[(size_t)(w++) * nl.stride + k] = j;
        }
      }
    }
    nl.cnt[k] = total; nl.lo[k] = nlo;
  }
  nl.ox[k] = x; nl.oy[k] = y; nl.oz[k] = z;
}

// build_particle over the candidate records k_rb_rank wrote in cell order:
// each candidate is one 32-byte record read straight from its cell's range
// (position, id, slot) instead of a slot index followed by four loads from
// the particle arrays.  Same candidates, order and arithmetic: same lists.
__device__ __forceinline__ void build_particle_packed(const Replica& R, int k, Dyn d, Stat st, NbList nl,
                                                     const D4* __restrict__ cand, const int* __restrict__ cstart,
                                                     const int* __restrict__ ccnt, int* __restrict__ status,
                                                     int* __restrict__ maxnb) {
  const double x = d.x[k], y = d.y[k], z = d.z[k];
  const int myid = st.id[k];
  int a, b, c;
  cell_of(R, x, y, z, a, b, c);
  const int base0 = cstart[R.cell_off];
  // the stencil's cells in visiting order as runs of consecutive candidate
  // records: runs that meet in the record array merge, empty ones drop out.
  // Away from the z faces the three z-cells of one (x, y) column are
  // consecutive (a-major numbering, z innermost): nine runs, and with three
  // z-cells (a quasi-2-D box) the three columns of one x offset meet as well.
  int rs[27], rn[27], nr = 0;
  if (R.use_cell && c >= 1 && c + 1 < R.cnz) {
    for (int ox = -1; ox <= 1; ox++) {
      int ia = a + ox;
      if (ia < 0) ia = R.cnx - 1; else if (ia == R.cnx) ia = 0;
      for (int oy = -1; oy <= 1; oy++) {
        int ib = b + oy;
        if (ib < 0) ib = R.cny - 1; else if (ib == R.cny) ib = 0;
        const int f = R.cell_off + R.cny * R.cnz * ia + R.cnz * ib + (c - 1);
        const int s0 = R.off + cstart[f] - base0, n = cstart[f + 2] + ccnt[f + 2] - cstart[f];
        if (n == 0) continue;
        if (nr > 0 && rs[nr - 1] + rn[nr - 1] == s0) rn[nr - 1] += n;
        else { rs[nr] = s0; rn[nr] = n; nr++; }
      }
    }
  } else {
    int cells[27];
    const int ncells = build_stencil(R, a, b, c, cells);
    for (int m = 0; m < ncells; m++) {
      const int cg = R.cell_off + cells[m];
      const int s0 = R.off + cstart[cg] - base0, n = ccnt[cg];
      if (n == 0) continue;
      if (nr > 0 && rs[nr - 1] + rn[nr - 1] == s0) rn[nr - 1] += n;
      else { rs[nr] = s0; rn[nr] = n; nr++; }
    }
  }
  unsigned long long lo[NB_LOCAL], up[NB_LOCAL];  // (id << 32) | slot
  int nlo = 0, nup = 0;
  bool overflow = false;
  int total = 0;
  for (int i = 0; i < nr; i++) total += rn[i];
  // one flat sweep over the runs' records (lanes of a warp stay together
  // across cell boundaries); each record requested one candidate ahead
  int ri = 0, pos = nr > 0 ? rs[0] : 0, end = nr > 0 ? rs[0] + rn[0] : 0;
  D4 nxt = total > 0 ? ldg4(cand + pos) : D4{0.0, 0.0, 0.0, 0.0};
  for (int t = 0; t < total; t++) {
    const D4 cr = nxt;
    if (t + 1 < total) {
      if (++pos == end) { ri++; pos = rs[ri]; end = pos + rn[ri]; }
      nxt = ldg4(cand + pos);
    }
    {
      const unsigned long long key = (unsigned long long)__double_as_longlong(cr.w);
      const int jid = (int)(unsigned)(key >> 32);
      if (jid == myid) continue;
      double dx, dy, dz;
      if (myid < jid) { dx = x - cr.x; dy = y - cr.y; dz = z - cr.z; }
      else { dx = cr.x - x; dy = cr.y - y; dz = cr.z - z; }
      apply_periodic(R, dx, dy, dz);
      if (dx * dx + dy * dy + dz * dz < R.cut2) {
        if (jid < myid) { if (nlo < NB_LOCAL) lo[nlo] = key; nlo++; }
        else { if (nup < NB_LOCAL) up[nup] = key; nup++; }
      }
    }
  }
  if (nlo > NB_LOCAL || (!R.use_cell && nup > NB_LOCAL)) overflow = true;
  const int found = nlo + nup;
  atomicMax(maxnb, found);
  if (found > nl.cap || overflow) {
    atomicOr(status, ST_OVERFLOW);
    nl.cnt[k] = 0; nl.lo[k] = 0;
  } else {
    for (int i = 1; i < nlo; i++) {  // insertion sort by id (stable: equal ids keep their order)
      const unsigned long long v = lo[i];
      int m = i - 1;
      while (m >= 0 && (lo[m] >> 32) > (v >> 32)) { lo[m + 1] = lo[m]; m--; }
      lo[m + 1] = v;
    }
    for (int q = 0; q < nlo; q++) nl.nb[(size_t)q * nl.stride + k] = (int)(unsigned)(lo[q] & 0xffffffffull);
    if (!R.use_cell) {
      for (int i = 1; i < nup; i++) {
        const unsigned long long v = up[i];
        int m = i - 1;
        while (m >= 0 && (up[m] >> 32) > (v >> 32)) { up[m + 1] = up[m]; m--; }
        up[m + 1] = v;
      }
      for (int q = 0; q < nup; q++)
        nl.nb[(size_t)(nlo + q) * nl.stride + k] = (int)(unsigned)(up[q] & 0xffffffffull);
    } else if (nup <= NB_LOCAL) {
      for (int q = 0; q < nup; q++)
        nl.nb[(size_t)(nlo + q) * nl.stride + k] = (int)(unsigned)(up[q] & 0xffffffffull);
    } else {
      // more higher-id neighbours than the local array holds: a second sweep
      // over the same runs writes them in visiting order straight into the list
      int w = nlo;
      for (int i = 0; i < nr; i++)
        for (int q = rs[i]; q < rs[i] + rn[i]; q++) {
          const D4 cr = ldg4(cand + q);
          const unsigned long long key = (unsigned long long)__double_as_longlong(cr.w);
          if ((int)(unsigned)(key >> 32) <= myid) continue;
          double dx = x - cr.x, dy = y - cr.y, dz = z - cr.z;
          apply_periodic(R, dx, dy, dz);
          if (dx * dx + dy * dy + dz * dz < R.cut2) nl.nb[(size_t)(w++) * nl.stride + k] = (int)(unsigned)key;
        }
    }
    nl.cnt[k] = found; nl.lo[k] = nlo;
  }
  nl.ox[k] = x; nl.oy[k] = y; nl.oz[k] = z;
}

__global__ void k_rb_build(const Replica* __restrict__ reps, const int* __restrict__ blk_rep,
                           const int* __restrict__ rebuild, Dyn d, Stat st, NbList nl,
                           const D4* __restrict__ cand, const int* __restrict__ cstart,
                           const int* __restrict__ ccnt, int* __restrict__ status, int* __restrict__ maxnb, const int* __restrict__ blist = nullptr) {
  const int bid_ = blist ? blist[blockIdx.x] : (int)blockIdx.x;  // block of the packed layout
  const int r = blk_rep[bid_];
  const int mode = rebuild[r];
  if (!mode) return;
  const Replica& R = reps[r];
  const int k = bid_ * BLOCK + threadIdx.x;
  if (k - R.off >= R.n) return;
  build_particle_packed(R, k, d, st, nl, cand, cstart, ccnt, status, maxnb);
}

// Cell m (0..26) of the 27-cell stencil of (a, b, c), in the visiting order
// of build_stencil (x offset outermost, z innermost), with periodic wrap.
__device__ __forceinline__ int stencil_cell(const Replica& R, int a, int b, int c, int m) {
  int ia = a + m / 9 - 1, ib = b + (m / 3) % 3 - 1, ic = c + m % 3 - 1;
  if (ia < 0) ia = R.cnx - 1; else if (ia == R.cnx) ia = 0;
  if (ib < 0) ib = R.cny - 1; else if (ib == R.cny) ib = 0;
  if (ic < 0) ic = R.cnz - 1; else if (ic == R.cnz) ic = 0;
  return R.cny * R.cnz * ia + R.cnz * ib + ic;
}

// Team list build: TEAM lanes per particle, lane t sweeping its own run of
// consecutive stencil cells, so a rebuild of a few small replicas is not
// bound by one thread's chain of dependent loads.  Concatenated in lane order
// the lanes' finds are in stencil visiting order; the lower-id ones are then
// ranked by id (ties by position, i.e. a stable sort) and the higher-id ones
// written in that order: the lists are those of k_rb_build.  The N^2 path and
// a lane with more finds than it stages fall back to build_particle.
constexpr int TEAM = 8;
constexpr int TEAM_PARTS = 32;  // particles per block of TEAM * TEAM_PARTS threads
constexpr int TEAM_SUB = BLOCK / TEAM_PARTS;  // blocks per packed block
constexpr int NB_TEAM = 16;     // finds staged per lane and side

__global__ void __launch_bounds__(TEAM * TEAM_PARTS)
k_rb_build_team(const Replica* __restrict__ reps, const int* __restrict__ blk_rep, const int* __restrict__ rebuild,
                Dyn d, Stat st, NbList nl, const int* __restrict__ cslot, const int* __restrict__ cstart,
                const int* __restrict__ ccnt, int* __restrict__ status, int* __restrict__ maxnb,
                const int* __restrict__ blist = nullptr) {
  __shared__ unsigned long long lokeys[TEAM_PARTS][NB_LOCAL];
  const int bid_ = blist ? blist[blockIdx.x / TEAM_SUB] : (int)(blockIdx.x / TEAM_SUB);
  const int r = blk_rep[bid_];
  const int mode = rebuild[r];
  if (!mode) return;
  const Replica& R = reps[r];
  const int pl = threadIdx.x / TEAM, t = threadIdx.x % TEAM;
  const int k = bid_ * BLOCK + (blockIdx.x % TEAM_SUB) * TEAM_PARTS + pl;
  if (k - R.off >= R.n) return;  // the whole team leaves together
  const unsigned tmask = 0xffu << ((threadIdx.x & 31) & ~(TEAM - 1));
  if (!R.use_cell) {
    if (t == 0) build_particle(R, mode, k, d, st, nl, cslot, cstart, ccnt, status, maxnb);
    return;
  }
  const double x = d.x[k], y = d.y[k], z = d.z[k];
  const int myid = st.id[k];
  int a, b, c;
  cell_of(R, x, y, z, a, b, c);
  const int base0 = cstart[R.cell_off];
  unsigned long long lo[NB_TEAM];  // (id << 32) | slot
  int up[NB_TEAM];
  int nlo = 0, nup = 0;
  const int m1 = (t + 1) * 27 / TEAM;
  for (int m = t * 27 / TEAM; m < m1; m++) {
    const int cg = R.cell_off + stencil_cell(R, a, b, c, m);
    const int s0 = R.off + cstart[cg] - base0, n = ccnt[cg];
    for (int q = 0; q < n; q++) {
      const int j = mode == 2 ? s0 + q : cslot[s0 + q];
      const int jid = st.id[j];
      if (jid == myid) continue;
      double dx, dy, dz;
      if (myid < jid) { dx = x - d.x[j]; dy = y - d.y[j]; dz = z - d.z[j]; }
      else { dx = d.x[j] - x; dy = d.y[j] - y; dz = d.z[j] - z; }
      apply_periodic(R, dx, dy, dz);
      if (dx * dx + dy * dy + dz * dz < R.cut2) {
        if (jid < myid) { if (nlo < NB_TEAM) lo[nlo] = ((unsigned long long)(unsigned)jid << 32) | (unsigned)j; nlo++; }
        else { if (nup < NB_TEAM) up[nup] = j; nup++; }
      }
    }
  }
  if (__any_sync(tmask, nlo > NB_TEAM || nup > NB_TEAM)) {
    if (t == 0) build_particle(R, mode, k, d, st, nl, cslot, cstart, ccnt, status, maxnb);
    return;
  }
  int plo = nlo, pup = nup;  // inclusive scans over the team
  for (int o = 1; o < TEAM; o <<= 1) {
    const int u = __shfl_up_sync(tmask, plo, o, TEAM), v = __shfl_up_sync(tmask, pup, o, TEAM);
    if (t >= o) { plo += u; pup += v; }
  }
  const int tot_lo = __shfl_sync(tmask, plo, TEAM - 1, TEAM), tot_up = __shfl_sync(tmask, pup, TEAM - 1, TEAM);
  plo -= nlo; pup -= nup;
  const int total = tot_lo + tot_up;
  if (t == 0) {
    atomicMax(maxnb, total);
    nl.ox[k] = x; nl.oy[k] = y; nl.oz[k] = z;
  }
  if (tot_lo > NB_LOCAL || total > nl.cap) {  // the one-thread build's overflow rule
    if (t == 0) { atomicOr(status, ST_OVERFLOW); nl.cnt[k] = 0; nl.lo[k] = 0; }
    return;
  }
  for (int i = 0; i < nlo; i++) lokeys[pl][plo + i] = lo[i];
  __syncwarp(tmask);
  for (int i = t; i < tot_lo; i += TEAM) {
    const unsigned long long v = lokeys[pl][i];
    const unsigned vid = (unsigned)(v >> 32);
    int rank = 0;
    for (int m = 0; m < tot_lo; m++) {
      const unsigned mid = (unsigned)(lokeys[pl][m] >> 32);
      rank += (mid < vid || (mid == vid && m < i)) ? 1 : 0;
    }
    nl.nb[(size_t)rank * nl.stride + k] = (int)(unsigned)(v & 0xffffffffull);
  }
  for (int i = 0; i < nup; i++) nl.nb[(size_t)(tot_lo + pup + i) * nl.stride + k] = up[i];
  if (t == 0) { nl.cnt[k] = total; nl.lo[k] = tot_lo; }
}

// ---------------------------------------------------------------------------
// Cell-tile list build for large quasi-2-D replicas (cell path, cnx, cny >= 3,
// cnz == 3, so the 27-cell stencil holds no cell twice).  A block takes a
// tile: TILE_B consecutive (a, b) cell columns along b at one a, every z
// layer.  It stages the particles of the tile and its halo (columns a-1..a+1,
// b0-1..b0+TILE_B, with periodic wrap) in shared memory once -- position, id
// and slot, in each cell's own order -- and every particle of the tile then
// sweeps its stencil there.  The candidates, their order and the arithmetic
// are build_particle's, so the lists are identical; only the global loads
// (one dependent chain per candidate in the one-thread build) are replaced by
// one staging pass whose loads are all independent.  A tile whose halo holds
// more than TILE_CAP particles builds its own particles with build_particle.
// ---------------------------------------------------------------------------
constexpr int TILE_B = 64;
constexpr int TILE_HB = TILE_B + 2;
constexpr int TILE_CZ = 3;
constexpr int TILE_HCELLS = 3 * TILE_HB * TILE_CZ;
constexpr int TILE_CAP = 640;

struct TileRef { int rep, a, b0, nb; };  // nb: own columns (TILE_B, fewer at the end of a row)

__host__ __device__ constexpr bool tile_eligible(int use_cell, int cnx, int cny, int cnz) {
  return use_cell && cnx >= 3 && cny >= 3 && cnz == TILE_CZ;
}

__global__ void __launch_bounds__(BLOCK)
k_rb_build_tile(const Replica* __restrict__ reps, const TileRef* __restrict__ tiles, const int* __restrict__ rebuild,
                Dyn d, Stat st, NbList nl, const int* __restrict__ cslot, const int* __restrict__ cstart,
                const int* __restrict__ ccnt, int* __restrict__ status, int* __restrict__ maxnb) {
  __shared__ int hstart[TILE_HCELLS + 1];  // local first particle of each halo cell; [nh]: total
  __shared__ int hgs[TILE_HCELLS];         // slot-index position of each halo cell's first particle
  __shared__ double sx[TILE_CAP], sy[TILE_CAP], sz[TILE_CAP];
  __shared__ int sid[TILE_CAP], sslot[TILE_CAP];
  __shared__ short scell[TILE_CAP];
  __shared__ int shw[32];
  __shared__ int wmax[BLOCK / 32];
  const TileRef T = tiles[blockIdx.x];
  const int mode = rebuild[T.rep];
  if (!mode) return;
  const Replica& R = reps[T.rep];
  const int base0 = cstart[R.cell_off];
  const int HB = T.nb + 2;
  const int nh = 3 * HB * TILE_CZ;  // halo cells of this tile, ordered (ha, hb, c), c innermost
  // counts and starts of the halo cells (each thread a run of consecutive cells)
  constexpr int CPT = (TILE_HCELLS + BLOCK - 1) / BLOCK;
  int cntv[CPT];
  int run = 0;
  {
    const int h0 = threadIdx.x * CPT;
    int hb = (h0 / TILE_CZ) % HB, ha = h0 / (TILE_CZ * HB), c = h0 % TILE_CZ;
#pragma unroll
    for (int u = 0; u < CPT; u++) {
      const int h = h0 + u;
      cntv[u] = 0;
      if (h < nh) {
        int ia = T.a + ha - 1, ib = T.b0 + hb - 1;
        if (ia < 0) ia += R.cnx; else if (ia >= R.cnx) ia -= R.cnx;
        if (ib < 0) ib += R.cny; else if (ib >= R.cny) ib -= R.cny;
        const int cg = R.cell_off + R.cny * R.cnz * ia + R.cnz * ib + c;
        cntv[u] = ccnt[cg];
        hgs[h] = R.off + cstart[cg] - base0;
      }
      run += cntv[u];
      if (++c == TILE_CZ) { c = 0; if (++hb == HB) { hb = 0; ha++; } }
    }
  }
  int total;
  int ex = block_excl_scan(run, shw, total);
#pragma unroll
  for (int u = 0; u < CPT; u++) {
    const int h = threadIdx.x * CPT + u;
    if (h < nh) hstart[h] = ex;
    ex += cntv[u];
  }
  if (threadIdx.x == 0) hstart[nh] = total;
  __syncthreads();
  // own cells: ha = 1, hb = 1..nb, every c -- contiguous in halo order
  const int own0 = (HB + 1) * TILE_CZ, own1 = (HB + T.nb + 1) * TILE_CZ;
  if (total > TILE_CAP) {  // too dense to stage: the one-thread build for this tile's own particles
    for (int h = own0; h < own1; h++) {
      const int s0 = hgs[h], n = hstart[h + 1] - hstart[h];
      for (int q = threadIdx.x; q < n; q += BLOCK)
        build_particle(R, mode, mode == 2 ? s0 + q : cslot[s0 + q], d, st, nl, cslot, cstart, ccnt, status, maxnb);
    }
    return;
  }
  // stage every halo particle, one per thread at a time: its cell by binary
  // search over the starts, then one slot-index load and the record
  for (int li = threadIdx.x; li < total; li += BLOCK) {
    int lo = 0, hi = nh - 1;  // last cell h with hstart[h] <= li (empty cells share their start)
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (hstart[mid] <= li) lo = mid; else hi = mid - 1;
    }
    const int s = hgs[lo] + (li - hstart[lo]);
    const int j = mode == 2 ? s : cslot[s];
    sx[li] = d.x[j]; sy[li] = d.y[j]; sz[li] = d.z[j];
    sid[li] = st.id[j]; sslot[li] = j; scell[li] = (short)lo;
  }
  __syncthreads();
  // every own particle sweeps its stencil in the staged cells, in the
  // visiting order of build_stencil: x offset outermost, then y, then z.  A
  // particle in the middle layer (c = 1) visits the layers 0, 1, 2 of each
  // column: one contiguous run of staged particles per column.
  const int p0 = hstart[own0], p1 = hstart[own1];
  int mymax = 0;  // longest list of this thread: one atomicMax per block below
  for (int li = p0 + threadIdx.x; li < p1; li += BLOCK) {
    const double x = sx[li], y = sy[li], z = sz[li];
    const int myid = sid[li], k = sslot[li];
    const int h = scell[li];
    const int c = h % TILE_CZ, hb = (h / TILE_CZ) % HB;
    unsigned long long lo[NB_LOCAL];  // (id << 32) | slot
    int nlo = 0, nup = 0;
    // pass 1: lower-id keys and the count of higher-id neighbours
    for (int ox = 0; ox < 3; ox++)
      for (int oy = -1; oy <= 1; oy++) {
        const int col = (ox * HB + hb + oy) * TILE_CZ;
        for (int oz = -1; oz <= 1; oz++) {
          int qa, qb;
          if (c == 1) {  // the whole column at once
            qa = hstart[col]; qb = hstart[col + TILE_CZ]; oz = 1;
          } else {
            int c2 = c + oz;
            c2 += c2 < 0 ? TILE_CZ : 0;
            c2 -= c2 >= TILE_CZ ? TILE_CZ : 0;
            qa = hstart[col + c2]; qb = hstart[col + c2 + 1];
          }
          for (int q = qa; q < qb; q++) {
            const int jid = sid[q];
            if (jid == myid) continue;
            double dx, dy, dz;
            if (myid < jid) { dx = x - sx[q]; dy = y - sy[q]; dz = z - sz[q]; }
            else { dx = sx[q] - x; dy = sy[q] - y; dz = sz[q] - z; }
            apply_periodic(R, dx, dy, dz);
            if (dx * dx + dy * dy + dz * dz < R.cut2) {
              if (jid < myid) {
                if (nlo < NB_LOCAL) lo[nlo] = ((unsigned long long)(unsigned)jid << 32) | (unsigned)sslot[q];
                nlo++;
              } else {
                nup++;
              }
            }
          }
        }
      }
    const int tot = nlo + nup;
    mymax = tot > mymax ? tot : mymax;
    nl.ox[k] = x; nl.oy[k] = y; nl.oz[k] = z;
    if (nlo > NB_LOCAL || tot > nl.cap) {  // build_particle's overflow rule
      atomicOr(status, ST_OVERFLOW);
      nl.cnt[k] = 0; nl.lo[k] = 0;
      continue;
    }
    for (int i = 1; i < nlo; i++) {  // insertion sort by id
      const unsigned long long v = lo[i];
      int m = i - 1;
      while (m >= 0 && (lo[m] >> 32) > (v >> 32)) { lo[m + 1] = lo[m]; m--; }
      lo[m + 1] = v;
    }
    for (int q = 0; q < nlo; q++) nl.nb[(size_t)q * nl.stride + k] = (int)(unsigned)(lo[q] & 0xffffffffull);
    // pass 2: the higher-id neighbours, written in visiting order
    int w = nlo;
    for (int ox = 0; ox < 3; ox++)
      for (int oy = -1; oy <= 1; oy++) {
        const int col = (ox * HB + hb + oy) * TILE_CZ;
        for (int oz = -1; oz <= 1; oz++) {
          int qa, qb;
          if (c == 1) {
            qa = hstart[col]; qb = hstart[col + TILE_CZ]; oz = 1;
          } else {
            int c2 = c + oz;
            c2 += c2 < 0 ? TILE_CZ : 0;
            c2 -= c2 >= TILE_CZ ? TILE_CZ : 0;
            qa = hstart[col + c2]; qb = hstart[col + c2 + 1];
          }
          for (int q = qa; q < qb; q++) {
            const int jid = sid[q];
            if (jid <= myid) continue;
            double dx = x - sx[q], dy = y - sy[q], dz = z - sz[q];
            apply_periodic(R, dx, dy, dz);
            if (dx * dx + dy * dy + dz * dz < R.cut2) nl.nb[(size_t)(w++) * nl.stride + k] = sslot[q];
          }
        }
      }
    nl.cnt[k] = tot; nl.lo[k] = nlo;
  }
  // block maximum of the list lengths, then one atomic
  mymax = __reduce_max_sync(0xffffffffu, mymax);
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = mymax;
  __syncthreads();
  if (threadIdx.x == 0) {
    int m = 0;
    for (int w = 0; w < BLOCK / 32; w++) m = wmax[w] > m ? wmax[w] : m;
    atomicMax(maxnb, m);
  }
}

}  // namespace sg
