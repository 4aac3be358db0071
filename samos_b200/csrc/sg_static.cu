// sg_static.cu -- force/torque evaluation that allocates no memory.
//
// Who needs it: callers that cannot call cudaMalloc -- code running inside
// another framework's memory pool or a strict allocator policy, plugins that
// only receive device pointers from their host application, and callers that
// must not allocate while a device graph is being recorded elsewhere.  They
// pass device pointers for inputs and outputs; every intermediate buffer lives
// in one file-scope device array of fixed size (kScratchBytes) that each GPU
// loading this library holds until the process exits.
//
// What it computes: the same as sg_compute for a single-type program with a
// `soft` pair potential and optionally one `polar` or `nematic` aligner --
// reset, PairSoftPotential::compute, Pair{Polar,Nematic}Align::compute
// (pair_soft_potential.cpp:33-119, pair_polar_aligner.cpp:32-107,
// pair_nematic_aligner.cpp:32-96) -- with neighbours taken directly from a
// cell list of width >= rcut+pad and visited in the reference's list order,
// so results match sg_compute bit for bit.
#include "samos_gpu.h"

#include <cuda.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <mutex>

namespace {

constexpr int kMaxParticles = SG_STATIC_MAX_PARTICLES;
constexpr int kMaxCells = SG_STATIC_MAX_CELLS;
constexpr int kScanTile = 1024;
constexpr int kMaxBlocks = (kMaxCells + kScanTile - 1) / kScanTile;
// int32 slots: pcell, tmp, slots (per particle); cnt, start, fill (per cell); block sums;
// one word counting the particles of the last call that had too many neighbours
constexpr size_t kScratchInts = (size_t)3 * kMaxParticles + (size_t)3 * kMaxCells + kMaxBlocks + 1;
constexpr size_t kScratchBytes = kScratchInts * sizeof(int);

// The scratch.  Host code must not use its name as an address: the address
// is obtained per device and context with cudaGetSymbolAddress (see
// scratch_on_device).
static __device__ __align__(256) int g_scratch[kScratchInts];

// Scratch addresses already looked up, keyed by device and CUDA context: an
// address is valid only in the context it was looked up in, and a host that
// creates its own driver-API context, or resets the device, gets a new one.
constexpr int kMaxCached = 64;
struct CachedAddress {
  int device;
  CUcontext context;
  int* address;
};
CachedAddress g_cache[kMaxCached];
int g_cached = 0;
std::mutex g_cache_mutex;

struct Geo {
  int n, cnx, cny, cnz, use_cell, periodic;
  double Lx, Ly, Lz, xlo, xhi, ylo, yhi, zlo, zhi, cwx, cwy, cwz, cut2;
};

__device__ __forceinline__ void wrap(const Geo& G, double& dx, double& dy, double& dz) {
  if (G.periodic) {
    if (dx > G.xhi) dx -= G.Lx; else if (dx < G.xlo) dx += G.Lx;
    if (dy > G.yhi) dy -= G.Ly; else if (dy < G.ylo) dy += G.Ly;
    if (dz > G.zhi) dz -= G.Lz; else if (dz < G.zlo) dz += G.Lz;
  }
}

__device__ __forceinline__ int cell3(const Geo& G, double x, double y, double z, int& a, int& b, int& c) {
  if (G.periodic) {  // CellList::populate's single wrap (cell_list.cpp:92-100)
    if (x < G.xlo) x += G.Lx; else if (x > G.xhi) x -= G.Lx;
    if (y < G.ylo) y += G.Ly; else if (y > G.yhi) y -= G.Ly;
    if (z < G.zlo) z += G.Lz; else if (z > G.zhi) z -= G.Lz;
  }
  a = (int)((x - G.xlo) / G.cwx);
  b = (int)((y - G.ylo) / G.cwy);
  c = (int)((z - G.zlo) / G.cwz);
  a = a < 0 ? 0 : (a >= G.cnx ? G.cnx - 1 : a);
  b = b < 0 ? 0 : (b >= G.cny ? G.cny - 1 : b);
  c = c < 0 ? 0 : (c >= G.cnz ? G.cnz - 1 : c);
  return G.cny * G.cnz * a + G.cnz * b + c;
}

__global__ void k_st_bin(Geo G, const double* __restrict__ x, const double* __restrict__ y,
                         const double* __restrict__ z, int* pcell, int* cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= G.n) return;
  int a, b, c;
  const int cl = cell3(G, x[i], y[i], z[i], a, b, c);
  pcell[i] = cl;
  atomicAdd(&cnt[cl], 1);
}

// exclusive scan of cnt[0..m) into start[0..m) (block sums then one block)
__global__ void k_st_scan_blocks(const int* __restrict__ cnt, int m, int* bsum) {
  __shared__ int sh[32];
  const int i = blockIdx.x * kScanTile + threadIdx.x;
  int v = i < m ? cnt[i] : 0;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int w = 0; w < kScanTile / 32; w++) s += sh[w];
    bsum[blockIdx.x] = s;
  }
}

__global__ void k_st_scan_final(const int* __restrict__ cnt, int m, const int* __restrict__ bsum, int nb,
                                int* start) {
  __shared__ int sh[kScanTile];
  __shared__ int base;
  if (threadIdx.x == 0) {
    int s = 0;
    for (int b = 0; b < (int)blockIdx.x && b < nb; b++) s += bsum[b];
    base = s;
  }
  const int i = blockIdx.x * kScanTile + threadIdx.x;
  sh[threadIdx.x] = i < m ? cnt[i] : 0;
  __syncthreads();
  for (int o = 1; o < kScanTile; o <<= 1) {
    int t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
    __syncthreads();
    sh[threadIdx.x] += t;
    __syncthreads();
  }
  if (i < m) start[i] = base + sh[threadIdx.x] - (i < m ? cnt[i] : 0);
}

__global__ void k_st_scatter(int n, const int* __restrict__ pcell, const int* __restrict__ start, int* fill,
                             int* tmp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = pcell[i];
  tmp[start[c] + atomicAdd(&fill[c], 1)] = i;
}

// particles of a cell in ascending id (= index) order, as CellList::populate
__global__ void k_st_rank(int n, const int* __restrict__ pcell, const int* __restrict__ start,
                          const int* __restrict__ cnt, const int* __restrict__ tmp, int* slots) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = pcell[i], s0 = start[c], m = cnt[c];
  int rank = 0;
  for (int q = 0; q < m; q++) rank += tmp[s0 + q] < i ? 1 : 0;
  slots[s0 + rank] = i;
}

constexpr int kLocal = 64;

// one particle: lower-id neighbours in ascending id, then higher-id ones in
// the reference's list order (27-cell stencil; ascending id on the N^2 path)
__global__ void k_st_forces(Geo G, const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z, const double* __restrict__ nx,
                            const double* __restrict__ ny, const double* __restrict__ nz,
                            const double* __restrict__ rad, const int* __restrict__ start,
                            const int* __restrict__ cnt, const int* __restrict__ slots, double k_soft,
                            double a_soft, int use_radii, int align_kind, double Jeff, double rc,
                            double* fx, double* fy, double* fz, double* tx, double* ty, double* tz,
                            int* overflow) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= G.n) return;
  const double xi = x[i], yi = y[i], zi = z[i];
  const double nxi = nx[i], nyi = ny[i], nzi = nz[i], ri = rad[i];
  int a, b, c;
  cell3(G, xi, yi, zi, a, b, c);
  int cells[27];
  int ncells = 0;
  for (int ox = -1; ox <= 1; ox++)
    for (int oy = -1; oy <= 1; oy++)
      for (int oz = -1; oz <= 1; oz++) {
        int ia = a + ox, ib = b + oy, ic = c + oz;
        if (ia < 0) ia = G.cnx - 1; else if (ia == G.cnx) ia = 0;
        if (ib < 0) ib = G.cny - 1; else if (ib == G.cny) ib = 0;
        if (ic < 0) ic = G.cnz - 1; else if (ic == G.cnz) ic = 0;
        const int cl = G.cny * G.cnz * ia + G.cnz * ib + ic;
        bool dup = false;
        if (!G.use_cell)
          for (int q = 0; q < ncells; q++) dup = dup || cells[q] == cl;
        if (!dup) cells[ncells++] = cl;
      }
  int lo[kLocal], up[kLocal];
  int nlo = 0, nup = 0;
  bool over = false;
  for (int m = 0; m < ncells; m++) {
    const int cl = cells[m], s0 = start[cl], e = s0 + cnt[cl];
    for (int s = s0; s < e; s++) {
      const int j = slots[s];
      if (j == i) continue;
      double dx, dy, dz;
      if (i < j) { dx = xi - x[j]; dy = yi - y[j]; dz = zi - z[j]; }
      else { dx = x[j] - xi; dy = y[j] - yi; dz = z[j] - zi; }
      wrap(G, dx, dy, dz);
      if (dx * dx + dy * dy + dz * dz < G.cut2) {
        if (j < i) { if (nlo < kLocal) lo[nlo++] = j; else over = true; }
        else { if (nup < kLocal) up[nup++] = j; else over = true; }
      }
    }
  }
  if (over) {  // more than kLocal neighbours on one side: flag this particle
    const double bad = nan("");
    fx[i] = bad; fy[i] = bad; fz[i] = bad; tx[i] = bad; ty[i] = bad; tz[i] = bad;
    atomicAdd(overflow, 1);
    return;
  }
  for (int p = 1; p < nlo; p++) {  // stable insertion sort by id
    int v = lo[p], q = p - 1;
    while (q >= 0 && lo[q] > v) { lo[q + 1] = lo[q]; q--; }
    lo[q + 1] = v;
  }
  if (!G.use_cell)
    for (int p = 1; p < nup; p++) {
      int v = up[p], q = p - 1;
      while (q >= 0 && up[q] > v) { up[q + 1] = up[q]; q--; }
      up[q + 1] = v;
    }
  double Fx = 0.0, Fy = 0.0, Fz = 0.0, Tx = 0.0, Ty = 0.0, Tz = 0.0;
  for (int t = 0; t < nlo + nup; t++) {
    const int j = t < nlo ? lo[t] : up[t - nlo];
    double dx = x[j] - xi, dy = y[j] - yi, dz = z[j] - zi;
    wrap(G, dx, dy, dz);
    const double r_sq = dx * dx + dy * dy + dz * dz;
    const double rd = sqrt(r_sq);
    const double sig = use_radii ? ri + rad[j] : a_soft;
    if (rd < sig) {
      const double diff = sig - rd;
      double ff;
      if (rd > 0.0) ff = k_soft * diff / rd; else ff = k_soft * diff;
      Fx -= ff * dx; Fy -= ff * dy; Fz -= ff * dz;
    }
    if (align_kind >= 0 && r_sq <= rc * rc) {
      const double onx = nx[j], ony = ny[j], onz = nz[j];
      const double tau_x = nyi * onz - nzi * ony;
      const double tau_y = nzi * onx - nxi * onz;
      const double tau_z = nxi * ony - nyi * onx;
      if (align_kind == SG_ALIGN_POLAR) {
        Tx += Jeff * tau_x; Ty += Jeff * tau_y; Tz += Jeff * tau_z;
      } else {
        const double cd = nxi * onx + nyi * ony + nzi * onz;
        Tx += Jeff * cd * tau_x; Ty += Jeff * cd * tau_y; Tz += Jeff * cd * tau_z;
      }
    }
  }
  fx[i] = Fx; fy[i] = Fy; fz[i] = Fz;
  tx[i] = Tx; ty[i] = Ty; tz[i] = Tz;
}

// The CUDA context current on this host thread (driver entry point fetched
// through the runtime, so the library does not link the driver library).
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);

CUcontext current_context() {
  static CtxGetCurrentFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<CtxGetCurrentFn>(f);
  }();
  CUcontext c = nullptr;
  if (!fn || fn(&c) != CUDA_SUCCESS) return nullptr;
  return c;
}

// Set-up once per device and context, with that device current: the
// host-side name of g_scratch is a stand-in, not a device address, so the
// address is looked up here (cudaGetSymbolAddress) and cached.  Without a
// context handle to key on, the address is looked up on every call.
int scratch_on_device(int** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return SG_ERR_CUDA;
  // null until the runtime has made a context current on this thread (the
  // lookup below does): such a call looks the address up without caching it
  const CUcontext ctx = current_context();
  std::lock_guard<std::mutex> lock(g_cache_mutex);
  if (ctx)
    for (int k = 0; k < g_cached; k++)
      if (g_cache[k].device == dev && g_cache[k].context == ctx) {
        *out = g_cache[k].address;
        return SG_OK;
      }
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || p == nullptr) return SG_ERR_CUDA;
  if (ctx) {
    // a full table starts over: addresses of earlier contexts are then looked up again
    if (g_cached == kMaxCached) g_cached = 0;
    g_cache[g_cached++] = CachedAddress{dev, ctx, static_cast<int*>(p)};
  }
  *out = static_cast<int*>(p);
  return SG_OK;
}

}  // namespace

extern "C" int sg_compute_static(int n, double lx, double ly, double lz, int periodic, double rcut, double pad,
                                 const double* x, const double* y, const double* z, const double* nx,
                                 const double* ny, const double* nz, const double* radius, double k_soft,
                                 double a_soft, int use_particle_radii, int align_kind, double J,
                                 double align_rcut, double* fx, double* fy, double* fz, double* tau_x,
                                 double* tau_y, double* tau_z, void* stream) {
  if (n < 0 || n > kMaxParticles) return SG_ERR_ARG;
  if (!(lx > 0.0 && ly > 0.0 && lz > 0.0 && rcut > 0.0 && pad >= 0.0)) return SG_ERR_ARG;
  if (align_kind != -1 && align_kind != SG_ALIGN_POLAR && align_kind != SG_ALIGN_NEMATIC) return SG_ERR_ARG;
  if (n == 0) return SG_OK;
  if (!x || !y || !z || !nx || !ny || !nz || !radius || !fx || !fy || !fz || !tau_x || !tau_y || !tau_z)
    return SG_ERR_ARG;
  const double cut = rcut + pad;
  // the cell counts are cast to int below: reject any side too long for the
  // scratch's cells first (this also rejects infinite and NaN sizes)
  if (!(lx / cut <= (double)kMaxCells && ly / cut <= (double)kMaxCells && lz / cut <= (double)kMaxCells))
    return SG_ERR_ARG;
  Geo G;
  G.n = n;
  G.periodic = periodic ? 1 : 0;
  G.Lx = lx; G.Ly = ly; G.Lz = lz;
  G.xlo = -0.5 * lx; G.xhi = 0.5 * lx; G.ylo = -0.5 * ly; G.yhi = 0.5 * ly; G.zlo = -0.5 * lz; G.zhi = 0.5 * lz;
  G.use_cell = (lx > 2.0 * cut && ly > 2.0 * cut && lz > 2.0 * cut) ? 1 : 0;  // neighbour_list.hpp:138
  G.cnx = (int)(lx / cut); G.cny = (int)(ly / cut); G.cnz = (int)(lz / cut);
  if (G.cnx < 1) G.cnx = 1;
  if (G.cny < 1) G.cny = 1;
  if (G.cnz < 1) G.cnz = 1;
  const long long ncell = (long long)G.cnx * G.cny * G.cnz;
  if (ncell > kMaxCells) return SG_ERR_ARG;
  G.cwx = lx / (double)G.cnx; G.cwy = ly / (double)G.cny; G.cwz = lz / (double)G.cnz;
  G.cut2 = cut * cut;
  int* base = nullptr;
  int rc = scratch_on_device(&base);
  if (rc != SG_OK) return rc;
  int* pcell = base;
  int* tmp = pcell + kMaxParticles;
  int* slots = tmp + kMaxParticles;
  int* cnt = slots + kMaxParticles;
  int* start = cnt + kMaxCells;
  int* fill = start + kMaxCells;
  int* bsum = fill + kMaxCells;
  int* overflow = bsum + kMaxBlocks;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int m = (int)ncell;
  // every call reuses the same scratch: clear what has to start at zero
  if (cudaMemsetAsync(cnt, 0, sizeof(int) * m, st) != cudaSuccess) return SG_ERR_CUDA;
  if (cudaMemsetAsync(fill, 0, sizeof(int) * m, st) != cudaSuccess) return SG_ERR_CUDA;
  if (cudaMemsetAsync(overflow, 0, sizeof(int), st) != cudaSuccess) return SG_ERR_CUDA;
  const int tb = 128, nbk = (n + tb - 1) / tb, nsc = (m + kScanTile - 1) / kScanTile;
  k_st_bin<<<nbk, tb, 0, st>>>(G, x, y, z, pcell, cnt);
  k_st_scan_blocks<<<nsc, kScanTile, 0, st>>>(cnt, m, bsum);
  k_st_scan_final<<<nsc, kScanTile, 0, st>>>(cnt, m, bsum, nsc, start);
  k_st_scatter<<<nbk, tb, 0, st>>>(n, pcell, start, fill, tmp);
  k_st_rank<<<nbk, tb, 0, st>>>(n, pcell, start, cnt, tmp, slots);
  const double Jeff = align_kind == SG_ALIGN_NEMATIC ? 2.0 * J : J;  // pair_nematic_aligner.cpp:37
  k_st_forces<<<nbk, tb, 0, st>>>(G, x, y, z, nx, ny, nz, radius, start, cnt, slots, k_soft, a_soft,
                                  use_particle_radii, align_kind, Jeff, align_rcut, fx, fy, fz, tau_x, tau_y,
                                  tau_z, overflow);
  return cudaGetLastError() == cudaSuccess ? SG_OK : SG_ERR_CUDA;
}

extern "C" int64_t sg_compute_static_scratch_bytes(void) { return (int64_t)kScratchBytes; }

extern "C" int sg_compute_static_overflow(int* count, void* stream) {
  if (!count) return SG_ERR_ARG;
  int* base = nullptr;
  int rc = scratch_on_device(&base);
  if (rc != SG_OK) return rc;
  const int* overflow = base + (kScratchInts - 1);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemcpyAsync(count, overflow, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return SG_ERR_CUDA;
  return cudaStreamSynchronize(st) == cudaSuccess ? SG_OK : SG_ERR_CUDA;
}
