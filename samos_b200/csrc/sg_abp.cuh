// sg_abp.cuh -- specialised step kernel for the active-Brownian programs the
// benchmarks run: one `soft` pair potential (single particle type), at most
// one polar or nematic aligner, optional self_propulsion, one `brownian`
// integrator, on a periodic plane or a sphere.
//
// Compared with k_hot_step the component kinds are template parameters, the
// replica's parameters are staged once per block in shared memory, and the
// neighbour sweep fetches four neighbour records before using any of them.
// The arithmetic per term is the reference's (see sg_kernels.cuh), so results
// are bit-identical to the generic kernels.
#pragma once
#include <climits>
#include <cstddef>

#include "sg_hot.cuh"

namespace sg {

enum { ABP_ALIGN_NONE = -1 };

// per-replica constants of the specialised program (host-built)
struct AbpParams {
  double xlo, xhi, ylo, yhi, zlo, zhi, Lx, Ly, Lz;
  double pad2q;           // 0.25*pad*pad  (neighbour_list.cpp:298)
  double k, a;            // soft: table [1][1] (pair_soft_potential.cpp:77,85)
  double J, rc2;          // aligner: effective J (nematic: 2J unless align_param), rcut*rcut
  double alpha;           // self_propulsion alpha
  double dt, v0, nu, mu, mur, stoch, flip;  // brownian; stoch = sqrt(nu*dt), flip = dt/tau
  double Rs;              // sphere radius
  Value temp;
  int off, n, periodic, use_radii, nematic, velocity;
  uint32_t seed, pad0;
};

// Tuning variants (chunk of neighbour records fetched ahead, min blocks/SM):
// the engine's autotuner times them on the live system and keeps the fastest.
// 0-4 per-particle sweep, 5 flattened, 6-7 staged (cp.async), 8 shared-memory
// tile, 9-10 per-particle sweep with lanes assigned in neighbour-count order,
// 11-14 ordered with the Gaussian draws taken before the sweep (fewer live
// registers inside it), at rising occupancy; 15-20 the same with each
// neighbour record fetched one iteration before it is used, at 6-12 blocks/SM;
// 21-27 twins of 18 / 17 / 19 / 11 / 3 / 12 / 13 that read the parameters of
// a one-replica system from the kernel's own parameter space (constant-bank
// operands of the FP64 instructions) instead of a shared-memory copy, whose
// per-neighbour loads otherwise sit on the sweep's dependency chains; 30-31
// pipelined with two neighbours per iteration (both records requested one
// iteration ahead, the two pair terms independent chains the scheduler can
// interleave, added in list order) at 6 and 5 blocks per SM, and 28-29 their
// by-value twins.
constexpr int ABP_NVARIANT = 32;
__host__ __device__ constexpr bool abp_byval(int v) { return v >= 21 && v <= 29; }
// the shared-memory twin of a by-value variant (taken when several replicas
// share the launch); every other property of a by-value variant is its twin's
__host__ __device__ constexpr int abp_twin(int v) {
  return v == 21 ? 18 : v == 22 ? 17 : v == 23 ? 19 : v == 24 ? 11 : v == 25 ? 3 : v == 26 ? 12 : v == 27 ? 13
       : v == 28 ? 30 : v == 29 ? 31 : v;
}
__host__ __device__ constexpr int abp_chunk(int v0) {
  const int v = abp_twin(v0);
  return v == 0 ? 4 : v == 1 ? 4 : v == 2 ? 2 : v == 3 ? 2 : v == 9 ? 2 : v == 10 ? 4 : v >= 15 ? 1 : v >= 11 ? 2 : 8;
}
__host__ __device__ constexpr int abp_minb(int v0) {
  const int v = abp_twin(v0);
  return v == 0 ? 5 : v == 1 ? 4 : v == 2 ? 6 : v == 3 ? 4 : v == 9 ? 6 : v == 10 ? 5 : v == 11 ? 6 : v == 12 ? 7
       : v == 13 ? 8 : v == 14 ? 10 : v == 15 ? 7 : v == 16 ? 6 : v == 17 ? 8 : v == 18 ? 9 : v == 19 ? 10 : v == 20 ? 12
       : v == 30 ? 6 : v == 31 ? 5 : 3;
}
__host__ __device__ constexpr bool abp_ordered(int v) { return abp_twin(v) >= 9; }
__host__ __device__ constexpr bool abp_prenoise(int v) { return abp_twin(v) >= 11; }
__host__ __device__ constexpr bool abp_pipelined(int v) { return abp_twin(v) >= 15; }
__host__ __device__ constexpr bool abp_pair2(int v) { return abp_twin(v) >= 30; }

// The variants the autotuner times (every one can still be pinned): those
// that never won on the plane, sphere or replica workloads are left out.
constexpr int ABP_TUNED[] = {0, 1, 2, 3, 8, 9, 10, 11, 12, 13, 15, 16, 17, 18, 21, 22, 23, 24, 25, 26, 27, 28, 29,
                             30, 31};
constexpr int ABP_NTUNED = (int)(sizeof(ABP_TUNED) / sizeof(ABP_TUNED[0]));

// Lane order of a block for the ordered variants: its particles sorted by
// neighbour count, largest first (ties by slot), so each warp's 32 lanes have
// similar list lengths and the warp's sweep is not set by one long list.
// Padding slots go last.  Each particle's own arithmetic is unchanged.
constexpr int LO_KEYS = 128;  // distinct sort keys the counting sort handles (list lengths 0..126 + padding)
static_assert(BLOCK == LO_KEYS, "k_lane_order scans one key per thread");

__global__ void __launch_bounds__(BLOCK)
k_lane_order(const Replica* __restrict__ reps, const int* __restrict__ blk_rep, NbList nl,
             uint8_t* __restrict__ order, const int* __restrict__ blist = nullptr) {
  constexpr int NW = BLOCK / 32;
  __shared__ int hist[NW][LO_KEYS];  // per warp: lanes holding each key
  __shared__ int wsum[NW];
  __shared__ int sc[BLOCK];
  const int b = blist ? blist[blockIdx.x] : (int)blockIdx.x, t = threadIdx.x, k = b * BLOCK + t;
  const Replica& R = reps[blk_rep[b]];
  const int c = (k - R.off < R.n) ? nl.cnt[k] : -1;
  if (nl.cap + 2 > LO_KEYS) {  // long lists (same branch for the whole grid): rank by comparison
    sc[t] = c;
    __syncthreads();
    int rank = 0;
    for (int u = 0; u < BLOCK; u++) {
      const int cu = sc[u];
      rank += (cu > c || (cu == c && u < t)) ? 1 : 0;
    }
    order[(size_t)b * BLOCK + rank] = (uint8_t)t;
    return;
  }
  // stable counting sort on key = count + 1 (padding 0), largest key first
  const int key = c + 1, w = t >> 5, lane = t & 31;
  for (int i = t; i < NW * LO_KEYS; i += BLOCK) (&hist[0][0])[i] = 0;
  __syncthreads();
  const unsigned same = __match_any_sync(0xffffffffu, key);
  const int below = __popc(same & ((1u << lane) - 1u));  // same key, lower lane
  if (below == 0) hist[w][key] = __popc(same);
  __syncthreads();
  // thread t holds key 127 - t: an inclusive scan over t sums the keys >= that key
  const int rk = LO_KEYS - 1 - t;
  int tot = 0;
  for (int u = 0; u < NW; u++) tot += hist[u][rk];
  int inc = tot;
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += v;
  }
  if (lane == 31) wsum[w] = inc;
  __syncthreads();
  for (int u = 0; u < w; u++) inc += wsum[u];
  sc[rk] = inc - tot;  // lanes with a larger key than rk
  __syncthreads();
  int rank = sc[key] + below;
  for (int u = 0; u < w; u++) rank += hist[u][key];
  order[(size_t)b * BLOCK + rank] = (uint8_t)t;
}

// One neighbour's pair term of the specialised program: soft repulsion
// (PairSoftPotential::compute, pair_soft_potential.cpp:79-104) and the polar /
// nematic torque (pair_polar_aligner.cpp, pair_nematic_aligner.cpp), gathered
// from the particle's side: F -= ff d, tau += J' (n_i x n_j).  `count_e`: the
// neighbour has the higher id, so the half-list energy counts this pair here.
template <int SHAPE, int ALIGN, bool ENERGY>
__device__ __forceinline__ void abp_pair_term(const AbpParams& S, double x, double y, double z, double nx, double ny,
                                              double nz, double ri, const D4& g, const D4& h, double rj, bool count_e,
                                              double& fx, double& fy, double& fz, double& tx, double& ty, double& tz,
                                              double& epair, double& ealign) {
  constexpr bool PLANE = SHAPE == HOT_PLANE;
    double dx = g.x - x, dy = g.y - y, dz = 0.0;
    if (!PLANE) dz = g.z - z;
    if (S.periodic) {
      if (dx > S.xhi) dx -= S.Lx; else if (dx < S.xlo) dx += S.Lx;
      if (dy > S.yhi) dy -= S.Ly; else if (dy < S.ylo) dy += S.Ly;
      if (!PLANE) { if (dz > S.zhi) dz -= S.Lz; else if (dz < S.zlo) dz += S.Lz; }
    }
    const double r_sq = PLANE ? dx * dx + dy * dy : dx * dx + dy * dy + dz * dz;
    // PairSoftPotential::compute, pair_soft_potential.cpp:79-104
    const double sig = S.use_radii ? ri + rj : S.a;
    // r_sq >= sig^2 (1 + 2^-40) implies sqrt(r_sq) >= sig after rounding:
    // no contact, so the square root can be skipped without changing a bit
    const double rd = r_sq < sig * sig * (1.0 + 0x1p-40) ? sqrt(r_sq) : sig;
    if (rd < sig) {
      const double diff = sig - rd;
      double ff;
      if (rd > 0.0) ff = S.k * diff / rd; else ff = S.k * diff;
      fx -= ff * dx; fy -= ff * dy;
      if (!PLANE) fz -= ff * dz;
      if (ENERGY && count_e) epair += 0.5 * S.k * diff * diff;
    }
    if (ALIGN != ABP_ALIGN_NONE && r_sq <= S.rc2) {
      double onx, ony, onz;
      if (PLANE) { onx = g.z; ony = g.w; onz = 0.0; }
      else { onx = h.x; ony = h.y; onz = h.z; }
      if (PLANE) {
        const double tau_z = nx * ony - ny * onx;
        if (ALIGN == ALIGN_POLAR) {
          tz += S.J * tau_z;
          if (ENERGY && count_e) ealign += -2.0 * S.J * (nx * onx + ny * ony);
        } else {
          const double cd = nx * onx + ny * ony;
          tz += S.J * cd * tau_z;
          if (ENERGY && count_e) ealign += -2.0 * S.J * (2.0 * cd * cd - 1.0);
        }
      } else {
        const double tau_x = ny * onz - nz * ony;
        const double tau_y = nz * onx - nx * onz;
        const double tau_z = nx * ony - ny * onx;
        if (ALIGN == ALIGN_POLAR) {
          tx += S.J * tau_x; ty += S.J * tau_y; tz += S.J * tau_z;
          if (ENERGY && count_e) ealign += -2.0 * S.J * (nx * onx + ny * ony + nz * onz);
        } else {
          const double cd = nx * onx + ny * ony + nz * onz;
          tx += S.J * cd * tau_x; ty += S.J * cd * tau_y; tz += S.J * cd * tau_z;
          if (ENERGY && count_e) ealign += -2.0 * S.J * (2.0 * cd * cd - 1.0);
        }
      }
    }
}

// Integration tail of the specialised program: self-propulsion, the
// Brownian update (integrator_brownian.cpp:57-121), enforce, torque
// projection, rotation, skin test (neighbour_list.cpp:278-302), the next
// step's enforce, and the stores.
template <int SHAPE, bool SP>
__device__ __forceinline__ void abp_finish(const AbpParams& S, int r, int k, double x, double y, double z, double nx,
                                           double ny, double nz, double ri, double fx, double fy, double fz, double tx,
                                           double ty, double tz, double g_rot, double g_x, double g_y, double g_z,
                                           double T, uint64_t gid, uint64_t s_base, double ox, double oy, double oz,
                                           double age0, D4* __restrict__ Gout, D4* __restrict__ Hout, Dyn& d,
                                           int* __restrict__ rebuild, int* __restrict__ status, int apply_e1,
                                           int last) {
  constexpr bool PLANE = SHAPE == HOT_PLANE;
  if (SP) { fx += S.alpha * nx; fy += S.alpha * ny; if (!PLANE) fz += S.alpha * nz; }

  // ---- IntegratorBrownian::integrate (integrator_brownian.cpp:57-121) ----
  Hp p;
  p.x = x; p.y = y; p.z = z; p.nx = nx; p.ny = ny; p.nz = nz;
  p.vx = 0.0; p.vy = 0.0; p.vz = 0.0;
  if (S.nematic) {
    // the velocity flip of velocity_align is overwritten below (v = fd)
    if (noise_uniform(S.seed, s_base + gid) < S.flip) { p.nx = -p.nx; p.ny = -p.ny; p.nz = -p.nz; }
  }
  double fd_x = S.v0 * p.nx + S.mu * fx;
  double fd_y = S.v0 * p.ny + S.mu * fy;
  double fd_z = S.v0 * p.nz + S.mu * fz;
  p.vx = fd_x; p.vy = fd_y; p.vz = fd_z;
  p.x += S.dt * fd_x; p.y += S.dt * fd_y;
  if (!PLANE) p.z += S.dt * fd_z;
  if (T > 0.0) {
    const double B = sqrt(2.0 * S.mu * T), sqrt_dt = sqrt(S.dt);
    const double fr_x = B * g_x, fr_y = B * g_y;
    p.vx += fr_x; p.vy += fr_y;
    p.x += sqrt_dt * fr_x; p.y += sqrt_dt * fr_y;
    if (!PLANE) { const double fr_z = B * g_z; p.vz += fr_z; p.z += sqrt_dt * fr_z; }
  }
  int dix = 0, diy = 0;
  const ShapeGeom Rb{S.xlo, S.xhi, S.Lx, S.ylo, S.yhi, S.Ly, S.Rs};
  hot_enforce<SHAPE>(Rb, p, dix, diy);
  if (PLANE) p.vz = 0.0;
  p.tx = tx; p.ty = ty; p.tz = tz;
  p.omega = S.mur * hot_project_torque<SHAPE>(Rb, p);
  const double dtheta = S.dt * p.omega + S.stoch * g_rot;
  hot_rotate<SHAPE>(Rb, p, dtheta, S.velocity != 0);
  const double age = age0 + S.dt;

  // ---- skin test, NeighbourList::need_update (neighbour_list.cpp:278-302)
  {
    double ddx = ox - p.x, ddy = oy - p.y, ddz = PLANE ? 0.0 : oz - p.z;
    if (S.periodic) {
      if (ddx > S.xhi) ddx -= S.Lx; else if (ddx < S.xlo) ddx += S.Lx;
      if (ddy > S.yhi) ddy -= S.Ly; else if (ddy < S.ylo) ddy += S.Ly;
      if (!PLANE) { if (ddz > S.zhi) ddz -= S.Lz; else if (ddz < S.zlo) ddz += S.Lz; }
    }
    const double d2 = PLANE ? ddx * ddx + ddy * ddy : ddx * ddx + ddy * ddy + ddz * ddz;
    if (!(d2 < S.pad2q)) {
      if (rebuild[r] == 0) atomicOr(&rebuild[r], 1);
    }
  }
  if (!(isfinite(p.x) && isfinite(p.y) && isfinite(p.z))) atomicOr(status, ST_NONFINITE);
  if (apply_e1) hot_enforce<SHAPE>(Rb, p, dix, diy);

  // ---- stores ---------------------------------------------------------------
  if (PLANE) {
    stg4(Gout + k, D4{p.x, p.y, p.nx, p.ny});
    d.vx[k] = p.vx; d.vy[k] = p.vy;
  } else {
    stg4(Gout + k, D4{p.x, p.y, p.z, ri});
    stg4(Hout + k, D4{p.nx, p.ny, p.nz, 0.0});
    d.vx[k] = p.vx; d.vy[k] = p.vy; d.vz[k] = p.vz;
  }
  d.age[k] = age;
  if (dix) d.ix[k] += dix;
  if (diy) d.iy[k] += diy;
  if (last) {
    d.omega[k] = p.omega;
    d.fx[k] = fx; d.fy[k] = fy; d.fz[k] = PLANE ? 0.0 : fz;
    d.tx[k] = tx; d.ty[k] = ty; d.tz[k] = tz;
  }
}

template <bool BYVAL>
__device__ __forceinline__ const AbpParams& abp_params(const AbpParams& pv, const AbpParams& staged) {
  if constexpr (BYVAL) return pv;
  else return staged;
}

template <int SHAPE, int ALIGN, bool SP, bool ENERGY, int VAR>
__global__ void __launch_bounds__(BLOCK, abp_minb(VAR))
k_abp_step(const AbpParams* __restrict__ prm, const int* __restrict__ blk_rep, const Clock* __restrict__ clk,
           const D4* __restrict__ Gin, D4* __restrict__ Gout, const D4* __restrict__ Hin, D4* __restrict__ Hout,
           Dyn d, Stat st, NbList nl, int* __restrict__ rebuild, int* __restrict__ status, int apply_e1, int last,
           double* epart, int nblocks, const uint8_t* __restrict__ lane_order,
           const __grid_constant__ AbpParams pv) {
  constexpr bool PLANE = SHAPE == HOT_PLANE;
  __shared__ AbpParams S_sh;
  __shared__ uint64_t s_base;
  __shared__ int s_step;
  // by-value variants serve a one-replica system: its replica is 0, and a
  // halted launch's blocks return after one load instead of two dependent ones
  const int r = abp_byval(VAR) ? 0 : blk_rep[blockIdx.x];
  if (clk[r].halt) return;  // batched stepping: a rebuild is pending (same value for the whole block)
  {
    constexpr int NW = (int)(sizeof(AbpParams) / 8);
    static_assert(sizeof(AbpParams) % 8 == 0, "AbpParams must be 8-byte granular");
    static_assert(NW <= BLOCK, "AbpParams too large for one-word-per-thread staging");
    if (!abp_byval(VAR) && threadIdx.x < NW)
      reinterpret_cast<unsigned long long*>(&S_sh)[threadIdx.x] =
          reinterpret_cast<const unsigned long long*>(prm + r)[threadIdx.x];
    if (threadIdx.x == 0) { s_base = clk[r].ctr[0]; s_step = clk[r].run_step; }
  }
  __syncthreads();
  // by-value variants: the one replica's parameters, read from parameter space
  const AbpParams& S = abp_params<abp_byval(VAR)>(pv, S_sh);
  static_assert(!abp_pipelined(VAR) || abp_prenoise(VAR), "the pipelined sweep takes the draws first");
  const int k = blockIdx.x * BLOCK +
                (abp_ordered(VAR) ? (int)lane_order[(size_t)blockIdx.x * BLOCK + threadIdx.x] : (int)threadIdx.x);
  double epair = 0.0, ealign = 0.0;
  if (k - S.off < S.n) {
    // ---- own state ----------------------------------------------------------
    double x, y, z, nx, ny, nz, ri;
    {
      const D4 g = ldg4(Gin + k);
      x = g.x; y = g.y;
      if (PLANE) { z = 0.0; nx = g.z; ny = g.w; nz = 0.0; ri = st.r[k]; }
      else { z = g.z; ri = g.w; const D4 h = ldg4(Hin + k); nx = h.x; ny = h.y; nz = h.z; }
    }
    const int cnt = nl.cnt[k], lo = nl.lo[k];
    const uint64_t gid = (uint64_t)st.id[k];

    // ---- forces and torques ---------------------------------------------------
    double fx = 0.0, fy = 0.0, fz = 0.0, tx = 0.0, ty = 0.0, tz = 0.0;
    constexpr int CH = abp_chunk(VAR);
    bool noise_done = false;
    double g_rot = 0.0, g_x = 0.0, g_y = 0.0, g_z = 0.0;
    const double T = value_get(S.temp, s_step);
    uint64_t base = s_base;
    if (S.nematic) base += (uint64_t)S.n;
    const int D = T > 0.0 ? 4 : 1;
    const uint64_t c0 = base + gid * (uint64_t)D;
    if (abp_prenoise(VAR)) {
      g_rot = noise_gauss(S.seed, c0 + (uint64_t)(D - 1));
      if (T > 0.0) {
        g_x = noise_gauss(S.seed, c0 + 0);
        g_y = noise_gauss(S.seed, c0 + 1);
        if (!PLANE) g_z = noise_gauss(S.seed, c0 + 2);
      }
      noise_done = true;
    }
    // list entries of the first chunk; each iteration then fetches the next
    // chunk's entries while its own records are in flight (index -> record
    // would otherwise be two dependent memory latencies per chunk)
    if constexpr (abp_pair2(VAR)) {
      // two neighbours per iteration, both records requested during the
      // previous iteration and the list entries two iterations ahead.  Past
      // the end of the list a lane reads its own record: that term is an
      // exact zero (d = 0, n x n = 0), so adding it changes no bit, and both
      // terms stay unconditional, free to interleave.
      int jn0 = 2 < cnt ? __ldg(nl.nb + (size_t)2 * nl.stride + k) : k;
      int jn1 = 3 < cnt ? __ldg(nl.nb + (size_t)3 * nl.stride + k) : k;
      const int j0 = 0 < cnt ? __ldg(nl.nb + k) : k;
      const int j1 = 1 < cnt ? __ldg(nl.nb + (size_t)1 * nl.stride + k) : k;
      D4 ga = ldg4(Gin + j0), gb = ldg4(Gin + j1), ha{0.0, 0.0, 0.0, 0.0}, hb{0.0, 0.0, 0.0, 0.0};
      double ra = PLANE ? (S.use_radii ? __ldg(st.r + j0) : 1.0) : 0.0;
      double rb = PLANE ? (S.use_radii ? __ldg(st.r + j1) : 1.0) : 0.0;
      if (!PLANE && ALIGN != ABP_ALIGN_NONE) { ha = ldg4(Hin + j0); hb = ldg4(Hin + j1); }
      for (int q = 0; q < cnt; q += 2) {
        const D4 g0 = ga, g1 = gb, h0 = ha, h1 = hb;
        const double r0 = PLANE ? ra : g0.w, r1 = PLANE ? rb : g1.w;
        if (q + 2 < cnt) {
          ga = ldg4(Gin + jn0);
          gb = ldg4(Gin + jn1);
          if (PLANE) { ra = S.use_radii ? __ldg(st.r + jn0) : 1.0; rb = S.use_radii ? __ldg(st.r + jn1) : 1.0; }
          if (!PLANE && ALIGN != ABP_ALIGN_NONE) { ha = ldg4(Hin + jn0); hb = ldg4(Hin + jn1); }
          jn0 = q + 4 < cnt ? __ldg(nl.nb + (size_t)(q + 4) * nl.stride + k) : k;
          jn1 = q + 5 < cnt ? __ldg(nl.nb + (size_t)(q + 5) * nl.stride + k) : k;
        }
        abp_pair_term<SHAPE, ALIGN, ENERGY>(S, x, y, z, nx, ny, nz, ri, g0, h0, r0, q >= lo, fx, fy, fz, tx, ty, tz,
                                            epair, ealign);
        abp_pair_term<SHAPE, ALIGN, ENERGY>(S, x, y, z, nx, ny, nz, ri, g1, h1, r1, q + 1 >= lo, fx, fy, fz, tx, ty,
                                            tz, epair, ealign);
      }
    } else if constexpr (abp_pipelined(VAR)) {
      // one neighbour per iteration: its record was requested during the
      // previous iteration, the entry after it two iterations ahead
      int jnext = 1 < cnt ? __ldg(nl.nb + (size_t)1 * nl.stride + k) : k;
      const int j0 = 0 < cnt ? __ldg(nl.nb + k) : k;
      D4 gcur = ldg4(Gin + j0), hcur{0.0, 0.0, 0.0, 0.0};
      double rcur = PLANE ? (S.use_radii ? __ldg(st.r + j0) : 1.0) : 0.0;
      if (!PLANE && ALIGN != ABP_ALIGN_NONE) hcur = ldg4(Hin + j0);
      for (int q = 0; q < cnt; q++) {
        const D4 g = gcur, h = hcur;
        const double rj = PLANE ? rcur : g.w;
        if (q + 1 < cnt) {
          gcur = ldg4(Gin + jnext);
          if (PLANE) rcur = S.use_radii ? __ldg(st.r + jnext) : 1.0;
          if (!PLANE && ALIGN != ABP_ALIGN_NONE) hcur = ldg4(Hin + jnext);
          jnext = q + 2 < cnt ? __ldg(nl.nb + (size_t)(q + 2) * nl.stride + k) : k;
        }
        abp_pair_term<SHAPE, ALIGN, ENERGY>(S, x, y, z, nx, ny, nz, ri, g, h, rj, q >= lo, fx, fy, fz, tx, ty, tz,
                                            epair, ealign);
      }
    } else {
    int jn[CH];
#pragma unroll
    for (int u = 0; u < CH; u++) jn[u] = u < cnt ? __ldg(nl.nb + (size_t)u * nl.stride + k) : k;
    for (int q0 = 0; q0 < cnt || !noise_done; q0 += CH) {
      int jj[CH];
      D4 gg[CH], hh[CH];
      double rr[CH];
#pragma unroll
      for (int u = 0; u < CH; u++) jj[u] = jn[u];
#pragma unroll
      for (int u = 0; u < CH; u++) {
        gg[u] = ldg4(Gin + jj[u]);
        if (PLANE) rr[u] = S.use_radii ? __ldg(st.r + jj[u]) : 1.0;
        if (!PLANE && ALIGN != ABP_ALIGN_NONE) hh[u] = ldg4(Hin + jj[u]);
      }
#pragma unroll
      for (int u = 0; u < CH; u++) {
        const int q = q0 + CH + u;
        jn[u] = q < cnt ? __ldg(nl.nb + (size_t)q * nl.stride + k) : k;
      }
      if (!noise_done) {  // independent of the loads above: overlaps their latency
        g_rot = noise_gauss(S.seed, c0 + (uint64_t)(D - 1));
        if (T > 0.0) {
          g_x = noise_gauss(S.seed, c0 + 0);
          g_y = noise_gauss(S.seed, c0 + 1);
          if (!PLANE) g_z = noise_gauss(S.seed, c0 + 2);
        }
        noise_done = true;
      }
#pragma unroll
      for (int u = 0; u < CH; u++) {
        const int q = q0 + u;
        if (q < cnt) {
          abp_pair_term<SHAPE, ALIGN, ENERGY>(S, x, y, z, nx, ny, nz, ri, gg[u], hh[u], PLANE ? rr[u] : gg[u].w,
                                              q >= lo, fx, fy, fz, tx, ty, tz, epair, ealign);
        }
      }
    }
    }
    // read only now: values the sweep does not need stay out of its registers
    const double ox = nl.ox[k], oy = nl.oy[k], oz = PLANE ? 0.0 : nl.oz[k];
    const double age0 = d.age[k];
    abp_finish<SHAPE, SP>(S, r, k, x, y, z, nx, ny, nz, ri, fx, fy, fz, tx, ty, tz, g_rot, g_x, g_y, g_z, T, gid,
                          s_base, ox, oy, oz, age0, Gout, Hout, d, rebuild, status, apply_e1, last);
  }
  if (ENERGY) {
    if constexpr (abp_ordered(VAR)) {
      // lanes in neighbour-count order: the block's sums are taken in slot
      // order all the same, so every variant stores the same partial sums
      __shared__ double s_ep[BLOCK], s_ea[BLOCK];
      s_ep[k - blockIdx.x * BLOCK] = epair;
      s_ea[k - blockIdx.x * BLOCK] = ealign;
      __syncthreads();
      epair = s_ep[threadIdx.x];
      ealign = s_ea[threadIdx.x];
    }
    double ev[MAX_PAIR + MAX_ALIGN];
#pragma unroll
    for (int i = 0; i < MAX_PAIR + MAX_ALIGN; i++) ev[i] = 0.0;
    ev[0] = epair;
    ev[MAX_PAIR] = ealign;
    block_reduce_store<MAX_PAIR + MAX_ALIGN>(ev, epart, nblocks);
  }
}


// ---------------------------------------------------------------------------
// Staged variant: each thread's neighbour records are copied into shared
// memory with cp.async (no registers held by loads in flight), CH records per
// stage, two stages in flight, while the previous stage is evaluated.  The
// pair term and the integration tail are the same functions as above, so the
// bits are those of k_abp_step.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// One stage: per record slot u, 16-byte chunks laid out lane-consecutive
// ([chunk][thread]), so a warp's shared loads are conflict-free.
template <int SHAPE, int ALIGN, int CH>
struct StagedBuf {
  static constexpr int NCHUNK = SHAPE == HOT_PLANE ? 2 : (ALIGN != ABP_ALIGN_NONE ? 4 : 2);
  double2 c[2][CH][NCHUNK][BLOCK];
  double r[SHAPE == HOT_PLANE ? 2 : 1][SHAPE == HOT_PLANE ? CH : 1][BLOCK];
};

template <int SHAPE, int ALIGN, bool SP, bool ENERGY, int CH, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB)
k_abp_staged(const AbpParams* __restrict__ prm, const int* __restrict__ blk_rep, const Clock* __restrict__ clk,
             const D4* __restrict__ Gin, D4* __restrict__ Gout, const D4* __restrict__ Hin, D4* __restrict__ Hout,
             Dyn d, Stat st, NbList nl, int* __restrict__ rebuild, int* __restrict__ status, int apply_e1, int last,
             double* epart, int nblocks) {
  constexpr bool PLANE = SHAPE == HOT_PLANE;
  using SB = StagedBuf<SHAPE, ALIGN, CH>;
  extern __shared__ __align__(16) unsigned char staged_smem[];
  SB& B = *reinterpret_cast<SB*>(staged_smem);
  __shared__ AbpParams S;
  __shared__ uint64_t s_base;
  __shared__ int s_step;
  const int r = blk_rep[blockIdx.x];
  if (clk[r].halt) return;  // batched stepping: a rebuild is pending (same value for the whole block)
  {
    constexpr int NW = (int)(sizeof(AbpParams) / 8);
    if (threadIdx.x < NW)
      reinterpret_cast<unsigned long long*>(&S)[threadIdx.x] =
          reinterpret_cast<const unsigned long long*>(prm + r)[threadIdx.x];
    if (threadIdx.x == 0) { s_base = clk[r].ctr[0]; s_step = clk[r].run_step; }
  }
  __syncthreads();
  const int t = threadIdx.x;
  const int k = blockIdx.x * BLOCK + t;
  double epair = 0.0, ealign = 0.0;
  if (k - S.off < S.n) {
    double x, y, z, nx, ny, nz, ri;
    {
      const D4 g = ldg4(Gin + k);
      x = g.x; y = g.y;
      if (PLANE) { z = 0.0; nx = g.z; ny = g.w; nz = 0.0; ri = st.r[k]; }
      else { z = g.z; ri = g.w; const D4 h = ldg4(Hin + k); nx = h.x; ny = h.y; nz = h.z; }
    }
    const int cnt = nl.cnt[k], lo = nl.lo[k];
    const uint64_t gid = (uint64_t)st.id[k];
    const double ox = nl.ox[k], oy = nl.oy[k], oz = PLANE ? 0.0 : nl.oz[k];
    const double age0 = d.age[k];
    const double* rr_src = st.r;
    auto issue = [&](int stage, int q0) {
#pragma unroll
      for (int u = 0; u < CH; u++) {
        const int q = q0 + u;
        if (q < cnt) {
          const int j = __ldg(nl.nb + (size_t)q * nl.stride + k);
          const double2* gsrc = reinterpret_cast<const double2*>(Gin + j);
          cp_async16(&B.c[stage][u][0][t], gsrc);
          cp_async16(&B.c[stage][u][1][t], gsrc + 1);
          if (PLANE) {
            if (S.use_radii) cp_async8(&B.r[stage][u][t], rr_src + j);
          } else if (ALIGN != ABP_ALIGN_NONE) {
            const double2* hsrc = reinterpret_cast<const double2*>(Hin + j);
            cp_async16(&B.c[stage][u][2][t], hsrc);
            cp_async16(&B.c[stage][u][3][t], hsrc + 1);
          }
        }
      }
      cp_async_commit();
    };

    double fx = 0.0, fy = 0.0, fz = 0.0, tx = 0.0, ty = 0.0, tz = 0.0;
    const double T = value_get(S.temp, s_step);
    uint64_t base = s_base;
    if (S.nematic) base += (uint64_t)S.n;
    const int D = T > 0.0 ? 4 : 1;
    const uint64_t c0 = base + gid * (uint64_t)D;
    issue(0, 0);
    // the noise is pure ALU work: it runs while the first stage is in flight
    double g_rot = noise_gauss(S.seed, c0 + (uint64_t)(D - 1)), g_x = 0.0, g_y = 0.0, g_z = 0.0;
    if (T > 0.0) {
      g_x = noise_gauss(S.seed, c0 + 0);
      g_y = noise_gauss(S.seed, c0 + 1);
      if (!PLANE) g_z = noise_gauss(S.seed, c0 + 2);
    }
    int stage = 0;
    for (int q0 = 0; q0 < cnt; q0 += CH) {
      issue(stage ^ 1, q0 + CH);  // next stage (an empty group past the end)
      cp_async_wait<1>();         // this thread's copies of `stage` have landed
#pragma unroll
      for (int u = 0; u < CH; u++) {
        const int q = q0 + u;
        if (q < cnt) {
          const double2 a = B.c[stage][u][0][t], b = B.c[stage][u][1][t];
          D4 g{a.x, a.y, b.x, b.y}, h{0.0, 0.0, 0.0, 0.0};
          double rj;
          if (PLANE) rj = S.use_radii ? B.r[stage][u][t] : 1.0;
          else {
            rj = g.w;
            if (ALIGN != ABP_ALIGN_NONE) {
              const double2 c = B.c[stage][u][2][t], e = B.c[stage][u][3][t];
              h = D4{c.x, c.y, e.x, e.y};
            }
          }
          abp_pair_term<SHAPE, ALIGN, ENERGY>(S, x, y, z, nx, ny, nz, ri, g, h, rj, q >= lo, fx, fy, fz, tx, ty, tz,
                                              epair, ealign);
        }
      }
      stage ^= 1;
    }
    cp_async_wait<0>();
    abp_finish<SHAPE, SP>(S, r, k, x, y, z, nx, ny, nz, ri, fx, fy, fz, tx, ty, tz, g_rot, g_x, g_y, g_z, T, gid,
                          s_base, ox, oy, oz, age0, Gout, Hout, d, rebuild, status, apply_e1, last);
  }
  if (ENERGY) {
    double ev[MAX_PAIR + MAX_ALIGN];
#pragma unroll
    for (int i = 0; i < MAX_PAIR + MAX_ALIGN; i++) ev[i] = 0.0;
    ev[0] = epair;
    ev[MAX_PAIR] = ealign;
    block_reduce_store<MAX_PAIR + MAX_ALIGN>(ev, epart, nblocks);
  }
}

template <int SHAPE, int ALIGN, int CH>
constexpr size_t staged_smem_bytes() { return sizeof(StagedBuf<SHAPE, ALIGN, CH>); }
using StagedBufSphere4 = StagedBuf<HOT_SPHERE, ALIGN_POLAR, 4>;
static_assert(offsetof(StagedBufSphere4, c) == 0, "16-byte cp.async targets come first");

// ---------------------------------------------------------------------------
// Tile variant: slots are in cell order, so the neighbours of a block's 128
// particles are a few hundred records from a handful of nearby cells.  After
// every neighbour-list build, k_tile_prep lists each block's distinct
// neighbour slots (ascending) and rewrites the lists as positions in that
// set (16-bit); the step kernel then copies the block's records into shared
// memory once (cp.async, while the Gaussian draws are computed) and every
// pair term reads shared memory.  Blocks whose neighbour slots span more than
// TILE_WIN slots or hold more than TILE_MAX distinct records (periodic wrap,
// unsorted lists) keep the global gather (tile_n = -1).  The pair term and
// the tail are the functions above, in list order: same bits.
// ---------------------------------------------------------------------------
constexpr int TILE_WIN = 16384;  // slot window per block (bitmap bits)
constexpr int TILE_MAX = 640;    // distinct neighbour records staged per block
constexpr int TILE_QMAX = 24;    // list ranks whose positions are staged (deeper ranks read global memory)

__global__ void __launch_bounds__(BLOCK)
k_tile_prep(const Replica* __restrict__ reps, const int* __restrict__ blk_rep, NbList nl, int* __restrict__ tile_n,
            int* __restrict__ tile_slot, uint16_t* __restrict__ nbpos, const int* __restrict__ blist = nullptr) {
  __shared__ uint32_t bm[TILE_WIN / 32];
  __shared__ int woff[TILE_WIN / 32];
  __shared__ int s_min, s_max, s_total;
  __shared__ int wsum[BLOCK / 32];
  const int b = blist ? blist[blockIdx.x] : (int)blockIdx.x, t = threadIdx.x, k = b * BLOCK + t;
  const Replica& R = reps[blk_rep[b]];
  const int cnt = (k - R.off < R.n) ? nl.cnt[k] : 0;
  if (t == 0) { s_min = INT_MAX; s_max = -1; }
  __syncthreads();
  int mn = INT_MAX, mx = -1;
  for (int q = 0; q < cnt; q++) {
    const int j = nl.nb[(size_t)q * nl.stride + k];
    mn = min(mn, j); mx = max(mx, j);
  }
  if (mx >= 0) { atomicMin(&s_min, mn); atomicMax(&s_max, mx); }
  __syncthreads();
  const int lo = s_min, hi = s_max;
  if (hi < 0) { if (t == 0) tile_n[b] = 0; return; }
  if (hi - lo + 1 > TILE_WIN) { if (t == 0) tile_n[b] = -1; return; }
  constexpr int WPT = TILE_WIN / 32 / BLOCK;  // bitmap words per thread
  for (int w = 0; w < WPT; w++) bm[t * WPT + w] = 0u;
  __syncthreads();
  for (int q = 0; q < cnt; q++) {
    const int d = nl.nb[(size_t)q * nl.stride + k] - lo;
    atomicOr(&bm[d >> 5], 1u << (d & 31));
  }
  __syncthreads();
  int pc[WPT], mine = 0;
  for (int w = 0; w < WPT; w++) { pc[w] = __popc(bm[t * WPT + w]); mine += pc[w]; }
  // exclusive scan of `mine` over the block
  const int lane = t & 31, warp = t >> 5;
  int incl = mine;
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  int base = incl - mine;
  for (int w = 0; w < warp; w++) base += wsum[w];
  if (t == BLOCK - 1) s_total = base + mine;
  for (int w = 0; w < WPT; w++) { woff[t * WPT + w] = base; base += pc[w]; }
  __syncthreads();
  const int total = s_total;
  if (total > TILE_MAX) { if (t == 0) tile_n[b] = -1; return; }
  for (int w = 0; w < WPT; w++) {
    uint32_t bits = bm[t * WPT + w];
    int pos = woff[t * WPT + w];
    while (bits) {
      const int l = __ffs(bits) - 1;
      tile_slot[(size_t)b * TILE_MAX + pos++] = lo + (t * WPT + w) * 32 + l;
      bits &= bits - 1u;
    }
  }
  for (int q = 0; q < cnt; q++) {
    const size_t at = (size_t)q * nl.stride + k;
    const int d = nl.nb[at] - lo, w = d >> 5;
    nbpos[at] = (uint16_t)(woff[w] + __popc(bm[w] & ((1u << (d & 31)) - 1u)));
  }
  if (t == 0) tile_n[b] = total;
}

template <int SHAPE, int ALIGN>
struct TileBuf {
  static constexpr int NCHUNK = SHAPE == HOT_PLANE ? 2 : (ALIGN != ABP_ALIGN_NONE ? 4 : 2);
  double2 c[NCHUNK][TILE_MAX];
  double r[SHAPE == HOT_PLANE ? TILE_MAX : 2];     // even count: keeps `pos` 16-byte aligned
  uint16_t pos[TILE_QMAX][BLOCK];  // the block's list positions, rank-major (16-byte cp.async targets)
};
using TileBufPlane = TileBuf<HOT_PLANE, ALIGN_POLAR>;
using TileBufSphere = TileBuf<HOT_SPHERE, ALIGN_POLAR>;
using TileBufSphereNoAlign = TileBuf<HOT_SPHERE, ABP_ALIGN_NONE>;
static_assert(offsetof(TileBufPlane, pos) % 16 == 0, "tile positions must be 16-byte aligned");
static_assert(offsetof(TileBufSphere, pos) % 16 == 0, "tile positions must be 16-byte aligned");
static_assert(offsetof(TileBufSphereNoAlign, pos) % 16 == 0, "tile positions must be 16-byte aligned");
template <int SHAPE, int ALIGN>
constexpr size_t tile_smem_bytes() { return sizeof(TileBuf<SHAPE, ALIGN>); }

template <int SHAPE, int ALIGN, bool SP, bool ENERGY, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB)
k_abp_tile(const AbpParams* __restrict__ prm, const int* __restrict__ blk_rep, const Clock* __restrict__ clk,
           const D4* __restrict__ Gin, D4* __restrict__ Gout, const D4* __restrict__ Hin, D4* __restrict__ Hout,
           Dyn d, Stat st, NbList nl, int* __restrict__ rebuild, int* __restrict__ status, int apply_e1, int last,
           double* epart, int nblocks, const int* __restrict__ tile_n, const int* __restrict__ tile_slot,
           const uint16_t* __restrict__ nbpos) {
  constexpr bool PLANE = SHAPE == HOT_PLANE;
  using TB = TileBuf<SHAPE, ALIGN>;
  extern __shared__ __align__(16) unsigned char tile_smem[];
  TB& B = *reinterpret_cast<TB*>(tile_smem);
  __shared__ AbpParams S;
  __shared__ uint64_t s_base;
  __shared__ int s_step;
  const int r = blk_rep[blockIdx.x];
  if (clk[r].halt) return;  // batched stepping: a rebuild is pending (same value for the whole block)
  {
    constexpr int NW = (int)(sizeof(AbpParams) / 8);
    if (threadIdx.x < NW)
      reinterpret_cast<unsigned long long*>(&S)[threadIdx.x] =
          reinterpret_cast<const unsigned long long*>(prm + r)[threadIdx.x];
    if (threadIdx.x == 0) { s_base = clk[r].ctr[0]; s_step = clk[r].run_step; }
  }
  __syncthreads();
  const int t = threadIdx.x;
  const int k = blockIdx.x * BLOCK + t;
  const int nt = tile_n[blockIdx.x];
  __shared__ int s_qmax;
  const bool active = k - S.off < S.n;
  const int cnt = active ? nl.cnt[k] : 0;
  if (t == 0) s_qmax = 0;
  __syncthreads();
  if (cnt > 0) atomicMax(&s_qmax, cnt);
  __syncthreads();
  const int qst = min(s_qmax, TILE_QMAX);  // list ranks staged
  if (nt > 0) {  // stage the block's distinct neighbour records and list positions
    const uint16_t* prow = nbpos + (size_t)blockIdx.x * BLOCK;
    for (int c = t; c < qst * (BLOCK / 8); c += BLOCK) {  // 16-byte pieces: 8 positions
      const int q = c / (BLOCK / 8), piece = c % (BLOCK / 8);
      cp_async16(&B.pos[q][piece * 8], prow + (size_t)q * nl.stride + piece * 8);
    }
    const int* slots = tile_slot + (size_t)blockIdx.x * TILE_MAX;
    for (int u = t; u < nt; u += BLOCK) {
      const int j = slots[u];
      const double2* gs = reinterpret_cast<const double2*>(Gin + j);
      cp_async16(&B.c[0][u], gs);
      cp_async16(&B.c[1][u], gs + 1);
      if (PLANE) {
        if (S.use_radii) cp_async8(&B.r[u], st.r + j);
      } else if (ALIGN != ABP_ALIGN_NONE) {
        const double2* hs = reinterpret_cast<const double2*>(Hin + j);
        cp_async16(&B.c[2][u], hs);
        cp_async16(&B.c[3][u], hs + 1);
      }
    }
    cp_async_commit();
  }
  double x = 0.0, y = 0.0, z = 0.0, nx = 0.0, ny = 0.0, nz = 0.0, ri = 0.0, ox = 0.0, oy = 0.0, oz = 0.0, age0 = 0.0;
  int lo = 0;
  uint64_t gid = 0;
  double g_rot = 0.0, g_x = 0.0, g_y = 0.0, g_z = 0.0;
  const double T = value_get(S.temp, s_step);
  if (active) {
    const D4 g = ldg4(Gin + k);
    x = g.x; y = g.y;
    if (PLANE) { nx = g.z; ny = g.w; ri = st.r[k]; }
    else { z = g.z; ri = g.w; const D4 h = ldg4(Hin + k); nx = h.x; ny = h.y; nz = h.z; }
    lo = nl.lo[k];
    gid = (uint64_t)st.id[k];
    ox = nl.ox[k]; oy = nl.oy[k];
    if (!PLANE) oz = nl.oz[k];
    age0 = d.age[k];
    // the Gaussian draws: pure ALU work while the records are in flight
    uint64_t base = s_base;
    if (S.nematic) base += (uint64_t)S.n;
    const int D = T > 0.0 ? 4 : 1;
    const uint64_t c0 = base + gid * (uint64_t)D;
    g_rot = noise_gauss(S.seed, c0 + (uint64_t)(D - 1));
    if (T > 0.0) {
      g_x = noise_gauss(S.seed, c0 + 0);
      g_y = noise_gauss(S.seed, c0 + 1);
      if (!PLANE) g_z = noise_gauss(S.seed, c0 + 2);
    }
  }
  if (nt > 0) cp_async_wait<0>();
  __syncthreads();
  double epair = 0.0, ealign = 0.0;
  if (active) {
    double fx = 0.0, fy = 0.0, fz = 0.0, tx = 0.0, ty = 0.0, tz = 0.0;
    for (int q = 0; q < cnt; q++) {
      const size_t at = (size_t)q * nl.stride + k;
      D4 g, h{0.0, 0.0, 0.0, 0.0};
      double rj;
      if (nt >= 0) {
        const int u = q < TILE_QMAX ? B.pos[q][t] : nbpos[at];
        const double2 a = B.c[0][u], c = B.c[1][u];
        g = D4{a.x, a.y, c.x, c.y};
        if (PLANE) rj = S.use_radii ? B.r[u] : 1.0;
        else {
          rj = g.w;
          if (ALIGN != ABP_ALIGN_NONE) {
            const double2 e = B.c[2][u], f = B.c[3][u];
            h = D4{e.x, e.y, f.x, f.y};
          }
        }
      } else {
        const int j = __ldg(nl.nb + at);
        g = ldg4(Gin + j);
        if (PLANE) rj = S.use_radii ? __ldg(st.r + j) : 1.0;
        else {
          rj = g.w;
          if (ALIGN != ABP_ALIGN_NONE) h = ldg4(Hin + j);
        }
      }
      abp_pair_term<SHAPE, ALIGN, ENERGY>(S, x, y, z, nx, ny, nz, ri, g, h, rj, q >= lo, fx, fy, fz, tx, ty, tz,
                                          epair, ealign);
    }
    abp_finish<SHAPE, SP>(S, r, k, x, y, z, nx, ny, nz, ri, fx, fy, fz, tx, ty, tz, g_rot, g_x, g_y, g_z, T, gid,
                          s_base, ox, oy, oz, age0, Gout, Hout, d, rebuild, status, apply_e1, last);
  }
  if (ENERGY) {
    double ev[MAX_PAIR + MAX_ALIGN];
#pragma unroll
    for (int i = 0; i < MAX_PAIR + MAX_ALIGN; i++) ev[i] = 0.0;
    ev[0] = epair;
    ev[MAX_PAIR] = ealign;
    block_reduce_store<MAX_PAIR + MAX_ALIGN>(ev, epart, nblocks);
  }
}

// ---------------------------------------------------------------------------
// Flattened variant: a warp's (particle, neighbour) items are laid out
// contiguously in shared memory (exclusive scan of the list lengths) and the
// expensive part of every pair term (sqrt, IEEE divide, cross products) is
// evaluated with all 32 lanes busy, whatever the spread of list lengths.
// Each lane then folds its own particle's terms in list order, so forces and
// torques are summed exactly as in the per-particle kernels.
// ---------------------------------------------------------------------------
template <int SHAPE>
struct FlatCfg {
  static constexpr int ITEMS = SHAPE == HOT_PLANE ? 192 : 128;  // item slots per warp
};

template <int SHAPE, bool ENERGY>
struct FlatWarp {
  static constexpr int W = FlatCfg<SHAPE>::ITEMS;
  static constexpr bool PL = SHAPE == HOT_PLANE;
  double ox[32], oy[32], oz[PL ? 1 : 32], onx[32], ony[32], onz[PL ? 1 : 32], orr[32];
  double tfx[W], tfy[W], tfz[PL ? 1 : W];
  double ttx[PL ? 1 : W], tty[PL ? 1 : W], ttz[W];
  double tep[ENERGY ? W : 1], tea[ENERGY ? W : 1];
  int idx[W];
  unsigned char own[W], valid[W];
};

template <int SHAPE, int ALIGN, bool SP, bool ENERGY>
__global__ void __launch_bounds__(BLOCK, 4)
k_abp_flat(const AbpParams* __restrict__ prm, const int* __restrict__ blk_rep, const Clock* __restrict__ clk,
           const D4* __restrict__ Gin, D4* __restrict__ Gout, const D4* __restrict__ Hin, D4* __restrict__ Hout,
           Dyn d, Stat st, NbList nl, int* __restrict__ rebuild, int* __restrict__ status, int apply_e1, int last,
           double* epart, int nblocks) {
  constexpr bool PLANE = SHAPE == HOT_PLANE;
  using FW = FlatWarp<SHAPE, ENERGY>;
  constexpr int W = FW::W;
  extern __shared__ __align__(16) unsigned char flat_smem[];
  FW& F = reinterpret_cast<FW*>(flat_smem)[threadIdx.x >> 5];
  __shared__ AbpParams S;
  __shared__ uint64_t s_base;
  __shared__ int s_step;
  const int r = blk_rep[blockIdx.x];
  if (clk[r].halt) return;  // batched stepping: a rebuild is pending (same value for the whole block)
  {
    constexpr int NW = (int)(sizeof(AbpParams) / 8);
    if (threadIdx.x < NW)
      reinterpret_cast<unsigned long long*>(&S)[threadIdx.x] =
          reinterpret_cast<const unsigned long long*>(prm + r)[threadIdx.x];
    if (threadIdx.x == 0) { s_base = clk[r].ctr[0]; s_step = clk[r].run_step; }
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int k = blockIdx.x * BLOCK + threadIdx.x;
  const bool active = k - S.off < S.n;

  // ---- own state into registers and the warp's shared table -------------------
  double x = 0.0, y = 0.0, z = 0.0, nx = 0.0, ny = 0.0, nz = 0.0, ri = 1.0;
  int cnt = 0, lo = 0;
  uint64_t gid = 0;
  double oxr = 0.0, oyr = 0.0, ozr = 0.0, age0 = 0.0;
  if (active) {
    const D4 g = ldg4(Gin + k);
    x = g.x; y = g.y;
    if (PLANE) { nx = g.z; ny = g.w; ri = st.r[k]; }
    else { z = g.z; ri = g.w; const D4 h = ldg4(Hin + k); nx = h.x; ny = h.y; nz = h.z; }
    cnt = nl.cnt[k]; lo = nl.lo[k];
    gid = (uint64_t)st.id[k];
    oxr = nl.ox[k]; oyr = nl.oy[k];
    if (!PLANE) ozr = nl.oz[k];
    age0 = d.age[k];
  }
  F.ox[lane] = x; F.oy[lane] = y; F.onx[lane] = nx; F.ony[lane] = ny; F.orr[lane] = ri;
  if (!PLANE) { F.oz[lane] = z; F.onz[lane] = nz; }
  // exclusive scan of list lengths over the warp
  int incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  const int excl = incl - cnt;
  const int total = __shfl_sync(0xffffffffu, incl, 31);

  // rotational (and translational) noise: pure ALU, independent of the sweep
  const double T = value_get(S.temp, s_step);
  uint64_t base = s_base;
  if (S.nematic) base += (uint64_t)S.n;
  const int D = T > 0.0 ? 4 : 1;
  const uint64_t c0 = base + gid * (uint64_t)D;
  double g_rot = 0.0, g_x = 0.0, g_y = 0.0, g_z = 0.0;

  double fx = 0.0, fy = 0.0, fz = 0.0, tx = 0.0, ty = 0.0, tz = 0.0;
  double epair = 0.0, ealign = 0.0;
  bool noise_done = false;
  for (int b0 = 0; b0 < total || !noise_done; b0 += W) {
    // stage this batch's neighbour slots (coalesced per list rank)
    for (int q = 0; q < cnt; q++) {
      const int it = excl + q - b0;
      if (it >= 0 && it < W) { F.idx[it] = __ldg(nl.nb + (size_t)q * nl.stride + k); F.own[it] = (unsigned char)lane; }
    }
    if (!noise_done) {
      if (active) {
        g_rot = noise_gauss(S.seed, c0 + (uint64_t)(D - 1));
        if (T > 0.0) {
          g_x = noise_gauss(S.seed, c0 + 0);
          g_y = noise_gauss(S.seed, c0 + 1);
          if (!PLANE) g_z = noise_gauss(S.seed, c0 + 2);
        }
      }
      noise_done = true;
    }
    __syncwarp();
    const int nit = min(W, total - b0);
    // evaluate the batch's items with every lane busy
    for (int it = lane; it < nit; it += 32) {
      const int p = F.own[it];
      const int j = F.idx[it];
      const D4 gj = ldg4(Gin + j);
      double rj, onx, ony, onz = 0.0;
      if (PLANE) { rj = S.use_radii ? __ldg(st.r + j) : 1.0; onx = gj.z; ony = gj.w; }
      else {
        rj = gj.w;
        if (ALIGN != ABP_ALIGN_NONE) { const D4 hj = ldg4(Hin + j); onx = hj.x; ony = hj.y; onz = hj.z; }
        else { onx = 0.0; ony = 0.0; }
      }
      const double px = F.ox[p], py = F.oy[p], pz = PLANE ? 0.0 : F.oz[p];
      double dx = gj.x - px, dy = gj.y - py, dz = 0.0;
      if (!PLANE) dz = gj.z - pz;
      if (S.periodic) {
        if (dx > S.xhi) dx -= S.Lx; else if (dx < S.xlo) dx += S.Lx;
        if (dy > S.yhi) dy -= S.Ly; else if (dy < S.ylo) dy += S.Ly;
        if (!PLANE) { if (dz > S.zhi) dz -= S.Lz; else if (dz < S.zlo) dz += S.Lz; }
      }
      const double r_sq = PLANE ? dx * dx + dy * dy : dx * dx + dy * dy + dz * dz;
      unsigned char v = 0;
      // PairSoftPotential::compute, pair_soft_potential.cpp:79-104
      const double sig = S.use_radii ? F.orr[p] + rj : S.a;
      const double rd = r_sq < sig * sig * (1.0 + 0x1p-40) ? sqrt(r_sq) : sig;  // see k_abp_step
      if (rd < sig) {
        const double diff = sig - rd;
        double ff;
        if (rd > 0.0) ff = S.k * diff / rd; else ff = S.k * diff;
        F.tfx[it] = ff * dx; F.tfy[it] = ff * dy;
        if (!PLANE) F.tfz[it] = ff * dz;
        if (ENERGY) F.tep[it] = 0.5 * S.k * diff * diff;
        v |= 1;
      }
      if (ALIGN != ABP_ALIGN_NONE && r_sq <= S.rc2) {
        const double pnx = F.onx[p], pny = F.ony[p], pnz = PLANE ? 0.0 : F.onz[p];
        if (PLANE) {
          const double tau_z = pnx * ony - pny * onx;
          if (ALIGN == ALIGN_POLAR) {
            F.ttz[it] = S.J * tau_z;
            if (ENERGY) F.tea[it] = -2.0 * S.J * (pnx * onx + pny * ony);
          } else {
            const double cd = pnx * onx + pny * ony;
            F.ttz[it] = S.J * cd * tau_z;
            if (ENERGY) F.tea[it] = -2.0 * S.J * (2.0 * cd * cd - 1.0);
          }
        } else {
          const double tau_x = pny * onz - pnz * ony;
          const double tau_y = pnz * onx - pnx * onz;
          const double tau_z = pnx * ony - pny * onx;
          if (ALIGN == ALIGN_POLAR) {
            F.ttx[it] = S.J * tau_x; F.tty[it] = S.J * tau_y; F.ttz[it] = S.J * tau_z;
            if (ENERGY) F.tea[it] = -2.0 * S.J * (pnx * onx + pny * ony + pnz * onz);
          } else {
            const double cd = pnx * onx + pny * ony + pnz * onz;
            const double Jc = S.J * cd;
            F.ttx[it] = Jc * tau_x; F.tty[it] = Jc * tau_y; F.ttz[it] = Jc * tau_z;
            if (ENERGY) F.tea[it] = -2.0 * S.J * (2.0 * cd * cd - 1.0);
          }
        }
        v |= 2;
      }
      F.valid[it] = v;
    }
    __syncwarp();
    // ordered fold of this particle's terms (reference summation order)
    for (int q = 0; q < cnt; q++) {
      const int it = excl + q - b0;
      if (it >= 0 && it < W) {
        const unsigned char v = F.valid[it];
        if (v & 1) {
          fx -= F.tfx[it]; fy -= F.tfy[it];
          if (!PLANE) fz -= F.tfz[it];
          if (ENERGY && q >= lo) epair += F.tep[it];
        }
        if (v & 2) {
          if (!PLANE) { tx += F.ttx[it]; ty += F.tty[it]; }
          tz += F.ttz[it];
          if (ENERGY && q >= lo) ealign += F.tea[it];
        }
      }
    }
    __syncwarp();
  }

  if (active) {
    if (SP) { fx += S.alpha * nx; fy += S.alpha * ny; if (!PLANE) fz += S.alpha * nz; }
    // ---- IntegratorBrownian::integrate (integrator_brownian.cpp:57-121) ----
    Hp p;
    p.x = x; p.y = y; p.z = z; p.nx = nx; p.ny = ny; p.nz = nz;
    if (S.nematic) {
      // the velocity flip of velocity_align is overwritten below (v = fd)
      if (noise_uniform(S.seed, s_base + gid) < S.flip) { p.nx = -p.nx; p.ny = -p.ny; p.nz = -p.nz; }
    }
    double fd_x = S.v0 * p.nx + S.mu * fx;
    double fd_y = S.v0 * p.ny + S.mu * fy;
    double fd_z = S.v0 * p.nz + S.mu * fz;
    p.vx = fd_x; p.vy = fd_y; p.vz = fd_z;
    p.x += S.dt * fd_x; p.y += S.dt * fd_y;
    if (!PLANE) p.z += S.dt * fd_z;
    if (T > 0.0) {
      const double B = sqrt(2.0 * S.mu * T), sqrt_dt = sqrt(S.dt);
      const double fr_x = B * g_x, fr_y = B * g_y;
      p.vx += fr_x; p.vy += fr_y;
      p.x += sqrt_dt * fr_x; p.y += sqrt_dt * fr_y;
      if (!PLANE) { const double fr_z = B * g_z; p.vz += fr_z; p.z += sqrt_dt * fr_z; }
    }
    int dix = 0, diy = 0;
    const ShapeGeom Rb{S.xlo, S.xhi, S.Lx, S.ylo, S.yhi, S.Ly, S.Rs};
    hot_enforce<SHAPE>(Rb, p, dix, diy);
    if (PLANE) p.vz = 0.0;
    p.tx = tx; p.ty = ty; p.tz = tz;
    p.omega = S.mur * hot_project_torque<SHAPE>(Rb, p);
    const double dtheta = S.dt * p.omega + S.stoch * g_rot;
    hot_rotate<SHAPE>(Rb, p, dtheta, S.velocity != 0);
    const double age = age0 + S.dt;
    {
      double ddx = oxr - p.x, ddy = oyr - p.y, ddz = PLANE ? 0.0 : ozr - p.z;
      if (S.periodic) {
        if (ddx > S.xhi) ddx -= S.Lx; else if (ddx < S.xlo) ddx += S.Lx;
        if (ddy > S.yhi) ddy -= S.Ly; else if (ddy < S.ylo) ddy += S.Ly;
        if (!PLANE) { if (ddz > S.zhi) ddz -= S.Lz; else if (ddz < S.zlo) ddz += S.Lz; }
      }
      const double d2 = PLANE ? ddx * ddx + ddy * ddy : ddx * ddx + ddy * ddy + ddz * ddz;
      if (!(d2 < S.pad2q)) {
        if (rebuild[r] == 0) atomicOr(&rebuild[r], 1);
      }
    }
    if (!(isfinite(p.x) && isfinite(p.y) && isfinite(p.z))) atomicOr(status, ST_NONFINITE);
    if (apply_e1) hot_enforce<SHAPE>(Rb, p, dix, diy);
    if (PLANE) {
      stg4(Gout + k, D4{p.x, p.y, p.nx, p.ny});
      d.vx[k] = p.vx; d.vy[k] = p.vy;
    } else {
      stg4(Gout + k, D4{p.x, p.y, p.z, ri});
      stg4(Hout + k, D4{p.nx, p.ny, p.nz, 0.0});
      d.vx[k] = p.vx; d.vy[k] = p.vy; d.vz[k] = p.vz;
    }
    d.age[k] = age;
    if (dix) d.ix[k] += dix;
    if (diy) d.iy[k] += diy;
    if (last) {
      d.omega[k] = p.omega;
      d.fx[k] = fx; d.fy[k] = fy; d.fz[k] = PLANE ? 0.0 : fz;
      d.tx[k] = tx; d.ty[k] = ty; d.tz[k] = tz;
    }
  }
  if (ENERGY) {
    double ev[MAX_PAIR + MAX_ALIGN];
#pragma unroll
    for (int i = 0; i < MAX_PAIR + MAX_ALIGN; i++) ev[i] = 0.0;
    ev[0] = epair;
    ev[MAX_PAIR] = ealign;
    block_reduce_store<MAX_PAIR + MAX_ALIGN>(ev, epart, nblocks);
  }
}

template <int SHAPE, bool ENERGY>
constexpr size_t flat_smem_bytes() { return sizeof(FlatWarp<SHAPE, ENERGY>) * (BLOCK / 32); }

}  // namespace sg
