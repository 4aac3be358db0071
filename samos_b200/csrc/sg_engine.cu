// sg_engine.cu -- host side of the B200 SAMoS engine: the C ABI declared in
// include/samos_gpu.h.  One stream per handle; device buffers are allocated
// once per configuration and reused by every step.
#include "samos_gpu.h"
#include "sg_abp.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace sg;

namespace {

struct DevBuf {
  std::vector<void*> ptrs;
  cudaError_t err = cudaSuccess;
  template <class T> T* alloc(size_t n) {
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, (n ? n : 1) * sizeof(T));
    if (e != cudaSuccess) { err = e; return nullptr; }
    cudaMemset(p, 0, (n ? n : 1) * sizeof(T));
    cudaDeviceSynchronize();
    ptrs.push_back(p);
    return (T*)p;
  }
  void release(void* p) {
    if (!p) return;
    auto it = std::find(ptrs.begin(), ptrs.end(), p);
    if (it != ptrs.end()) { cudaFree(p); ptrs.erase(it); }
  }
  void free_all() { for (void* p : ptrs) cudaFree(p); ptrs.clear(); }
};

const char* kDoubleFields[] = {"x", "y", "z", "vx", "vy", "vz", "nx", "ny", "nz",
                               "fx", "fy", "fz", "tau_x", "tau_y", "tau_z", "omega", "age"};
const int kNumDynDouble = 17;

}  // namespace

struct sg_system {
  int device = 0;
  int nrep = 0, ntypes = 1;
  std::vector<int> n, off;
  int slots = 0, nblocks = 0;
  int* blk_rep = nullptr;
  std::vector<int> blk_rep_h, rep_blk0_h, rep_nblk_h;
  std::vector<int64_t> rep_builds;  // neighbour-list builds per replica
  int *rep_blk0 = nullptr, *rep_nblk = nullptr;
  std::vector<Replica> reps_h;
  Replica* reps = nullptr;
  std::vector<Clock> clk_h;
  Clock* clk = nullptr;
  Program prog{};
  std::vector<double*> tables;
  Dyn cur{}, alt{};
  Stat st{}, st_alt{};
  NbList nl{};
  bool has_nlist = false;
  double rcut = 0.0, pad = 0.0;
  int ncell_total = 0;
  int *pcell = nullptr, *cell_cnt = nullptr, *cell_start = nullptr, *cell_fill = nullptr;
  int *tmp = nullptr, *perm = nullptr, *scan_bsum = nullptr;
  D4* cand = nullptr;                 // cell-ordered candidate records of the list build (k_rb_rank)
  CellSeg* segs = nullptr;            // cell ranges of the replicas being rebuilt
  int* blist = nullptr;               // blocks of the replicas being rebuilt (null: every block)
  // pinned staging of the small per-rebuild uploads (block list, cell
  // segments) and of the build's status readback; ev_pin marks the last copy
  // out of the staging, which must have run before the staging is rewritten
  int* pin_blist = nullptr;
  CellSeg* pin_segs = nullptr;
  int* pin_res = nullptr;
  cudaEvent_t ev_pin = nullptr;
  bool b_pending = false;  // ev_b0 / ev_b1 bracket a rebuild not yet added to the run's rebuild time
  int nblist = 0;
  // minimiser: blocks of the replicas that have not converged (null: every block)
  int* act = nullptr;
  std::vector<int> act_h;
  int nact = 0;
  int *rebuild = nullptr, *status = nullptr, *maxnb = nullptr;
  int *bstatus = nullptr;   // list-build status (overflow), separate from the run's status word
  void* xfer = nullptr;     // staging for host transfers in particle-id order (largest replica)
  int* xerr = nullptr;      // set by the transfer kernels on an id outside the replica
  int *exec_cnt = nullptr;  // steps executed in a batch (batched stepping)
  int *fire_cnt = nullptr;  // per replica: blocks of k_fire_b done (the last one runs the FIRE control)
  int64_t since_rebuild = 0, last_gap = 8;  // batch length follows the steps between rebuilds
  int* rebuild_h = nullptr;  // pinned
  double *epart = nullptr, *fire_part = nullptr, *alpha_mix = nullptr, *Rn = nullptr;
  // FIRE sums in the reference's particle order (sg_set_fire_order): the
  // per-particle terms by replica offset + id, 3 arrays of `slots` doubles
  int fire_ordered = 0;
  double* fire_terms = nullptr;
  // multi-field transfers: staging for several fields of one replica at once
  double* xfer_multi = nullptr;
  size_t xfer_multi_cap = 0;  // doubles
  double dt_global = 0.0;
  bool e1_applied = false;
  bool forces_fresh = false;  // forces equal those the next start-of-step pass would compute
  bool configured_nlist_once = false;
  int64_t launches = 0;
  int64_t builds_run = 0;
  int profile = 0;
  int maxnb_seen = 0;
  cudaEvent_t ev_run0 = nullptr, ev_run1 = nullptr, ev_k0 = nullptr, ev_k1 = nullptr;
  cudaEvent_t ev_b0 = nullptr, ev_b1 = nullptr;
  cudaStream_t stream = nullptr;
  DevBuf mem;
  std::string last_error;
  std::vector<double> uploaded_N[3];
  D4 *G[2] = {nullptr, nullptr}, *H[2] = {nullptr, nullptr};
  std::vector<std::vector<double>> pair_tab_h, align_tab_h, ext_tab_h;
  AbpParams* abp = nullptr;
  AbpParams abp0_h{};  // replica 0's parameters, passed by value to the by-value variants
  bool abp_on = false;
  // shared-memory tile variant: per-block distinct neighbour slots and the
  // lists rewritten as positions in them (k_tile_prep), valid until the next
  // list build
  int* tile_n = nullptr;
  int* tile_slot = nullptr;
  uint16_t* nbpos = nullptr;
  int nbpos_cap = 0;
  // particle groups (System::make_group): per slot-of-id a bit per group, and
  // each member's position in its group (ids are fixed, so both are indexed
  // by replica offset + particle id and never move with the slots)
  uint8_t* gmask = nullptr;
  int* grank = nullptr;
  std::vector<uint8_t> gmask_h;
  // ConstraintSphere::rescale settings per constraint (rescale, rescale_steps,
  // rescale_freq, and the per-event factor rescale^(freq/steps), constraint.hpp:97-104)
  struct Rescale { double rescale = 1.0, scale = 1.0; int steps = 1000, freq = 10; };
  std::vector<Rescale> cons_rescale;
  int64_t rescaled_at = -1;  // global step whose rescale sg_begin_step already applied
  int build_mode = 0;        // list build: 0 automatic, 1 one thread per particle, 2 teams of TEAM lanes, 3 cell tiles
  // cell-tile build: the tiles of the flagged replicas (rebuilt when the flagged set changes)
  TileRef* tiles = nullptr;
  int tiles_cap = 0, ntiles = 0;
  std::vector<int> tiles_for;
  bool tile_valid = false;
  // ordered variants: per-block lane order by neighbour count (k_lane_order)
  uint8_t* lane_order = nullptr;
  bool order_valid = false;
  int abp_variant = 1;
  // generic fused kernel: blocks per SM of its launch bounds (8 or 6), timed
  // on the run's first steps unless pinned (sg_set_generic_occupancy)
  int gen_minb = 8, gen_pin = 0, gen_trial = 0;
  bool gen_tuned = false;
  double gen_ms[2] = {0.0, 0.0};
  int gen_n[2] = {0, 0};
  // autotuner: every variant yields the same bits, so candidates are timed on
  // the run's own first steps (CUDA events around the step kernel)
  bool tuned = false;
  int tune_trial = 0;
  double tune_ms[ABP_NVARIANT] = {0};
  int tune_n[ABP_NVARIANT] = {0};
  cudaEvent_t ev_t0 = nullptr, ev_t1 = nullptr;
  int hot_buf = 0;
  int force_generic = 0;  // testing aid: keep the generic SoA kernels
};

static int fail(sg_system* s, int code, const std::string& msg) {
  if (s) s->last_error = msg;
  return code;
}

#define CU(s, call)                                                                  \
  do {                                                                               \
    cudaError_t e__ = (call);                                                        \
    if (e__ != cudaSuccess)                                                          \
      return fail((s), SG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e__)); \
  } while (0)

#define LAUNCH_CHECK(s)                                                              \
  do {                                                                               \
    (s)->launches++;                                                                 \
    cudaError_t e__ = cudaGetLastError();                                            \
    if (e__ != cudaSuccess)                                                          \
      return fail((s), SG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e__)); \
  } while (0)

static double* dyn_field(Dyn& d, int i) {
  double* f[kNumDynDouble] = {d.x, d.y, d.z, d.vx, d.vy, d.vz, d.nx, d.ny, d.nz,
                              d.fx, d.fy, d.fz, d.tx, d.ty, d.tz, d.omega, d.age};
  return f[i];
}

static bool alloc_dyn(DevBuf& m, Dyn& d, size_t n) {
  d.x = m.alloc<double>(n); d.y = m.alloc<double>(n); d.z = m.alloc<double>(n);
  d.vx = m.alloc<double>(n); d.vy = m.alloc<double>(n); d.vz = m.alloc<double>(n);
  d.nx = m.alloc<double>(n); d.ny = m.alloc<double>(n); d.nz = m.alloc<double>(n);
  d.fx = m.alloc<double>(n); d.fy = m.alloc<double>(n); d.fz = m.alloc<double>(n);
  d.tx = m.alloc<double>(n); d.ty = m.alloc<double>(n); d.tz = m.alloc<double>(n);
  d.omega = m.alloc<double>(n); d.age = m.alloc<double>(n);
  d.ix = m.alloc<int>(n); d.iy = m.alloc<int>(n); d.iz = m.alloc<int>(n);
  return m.err == cudaSuccess;
}

static bool alloc_stat(DevBuf& m, Stat& s, size_t n) {
  s.r = m.alloc<double>(n); s.mass = m.alloc<double>(n);
  s.type = m.alloc<int>(n); s.id = m.alloc<int>(n);
  return m.err == cudaSuccess;
}

static int push_reps(sg_system* s) {
  CU(s, cudaMemcpyAsync(s->reps, s->reps_h.data(), sizeof(Replica) * s->nrep, cudaMemcpyHostToDevice, s->stream));
  return SG_OK;
}
static int push_clk(sg_system* s) {
  CU(s, cudaMemcpyAsync(s->clk, s->clk_h.data(), sizeof(Clock) * s->nrep, cudaMemcpyHostToDevice, s->stream));
  return SG_OK;
}
static int pull_clk(sg_system* s) {
  CU(s, cudaMemcpyAsync(s->clk_h.data(), s->clk, sizeof(Clock) * s->nrep, cudaMemcpyDeviceToHost, s->stream));
  CU(s, cudaStreamSynchronize(s->stream));
  return SG_OK;
}

extern "C" {

const char* sg_error_string(int code) {
  switch (code) {
    case SG_OK: return "ok";
    case SG_ERR_ARG: return "invalid argument";
    case SG_ERR_CUDA: return "CUDA error";
    case SG_ERR_NOMEM: return "device out of memory";
    case SG_ERR_STATE: return "call out of order";
    case SG_ERR_OVERFLOW: return "neighbour capacity exceeded";
    case SG_ERR_NONFINITE: return "non-finite particle state";
    case SG_ERR_UNSUPPORTED: return "configuration not supported by the GPU path";
    case SG_ERR_TIMEOUT: return "bounded device wait gave up";
    default: return "unknown error";
  }
}

const char* sg_last_error(const sg_system* s) { return s ? s->last_error.c_str() : "null handle"; }

int sg_set_device(int device) {
  return cudaSetDevice(device) == cudaSuccess ? SG_OK : SG_ERR_CUDA;
}
int64_t sg_kernel_launches(const sg_system* s) { return s ? s->launches : 0; }

int sg_create(int n_replicas, const int32_t* n_particles, int ntypes, sg_system** out) {
  if (!out || n_replicas <= 0 || !n_particles || ntypes <= 0 || ntypes > SG_MAX_TYPES) return SG_ERR_ARG;
  for (int r = 0; r < n_replicas; r++)
    if (n_particles[r] < 0) return SG_ERR_ARG;
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) return SG_ERR_CUDA;
  sg_system* s = new sg_system();
  cudaGetDevice(&s->device);
  s->nrep = n_replicas;
  s->ntypes = ntypes;
  s->n.assign(n_particles, n_particles + n_replicas);
  s->off.resize(n_replicas);
  int slot = 0;
  for (int r = 0; r < n_replicas; r++) {
    s->off[r] = slot;
    int padded = ((s->n[r] + BLOCK - 1) / BLOCK) * BLOCK;
    if (padded == 0) padded = BLOCK;
    s->rep_blk0_h.push_back(slot / BLOCK);
    s->rep_nblk_h.push_back(padded / BLOCK);
    for (int b = 0; b < padded / BLOCK; b++) s->blk_rep_h.push_back(r);
    slot += padded;
  }
  s->slots = slot;
  s->nblocks = slot / BLOCK;
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) { delete s; return SG_ERR_CUDA; }
  DevBuf& m = s->mem;
  s->blk_rep = m.alloc<int>(s->nblocks);
  s->rep_blk0 = m.alloc<int>(n_replicas);
  s->rep_nblk = m.alloc<int>(n_replicas);
  s->reps = m.alloc<Replica>(n_replicas);
  s->clk = m.alloc<Clock>(n_replicas);
  bool ok = alloc_dyn(m, s->cur, s->slots) && alloc_dyn(m, s->alt, s->slots) &&
            alloc_stat(m, s->st, s->slots) && alloc_stat(m, s->st_alt, s->slots);
  s->rebuild = m.alloc<int>(n_replicas);
  s->status = m.alloc<int>(1);
  s->bstatus = m.alloc<int>(1);
  s->exec_cnt = m.alloc<int>(1);
  s->fire_cnt = m.alloc<int>(n_replicas);
  s->maxnb = m.alloc<int>(1);
  s->epart = m.alloc<double>((size_t)(MAX_PAIR + MAX_ALIGN) * s->nblocks);
  s->fire_part = m.alloc<double>((size_t)4 * s->nblocks);
  s->alpha_mix = m.alloc<double>(n_replicas);
  s->pcell = m.alloc<int>(s->slots);
  s->tmp = m.alloc<int>(s->slots);
  s->perm = m.alloc<int>(s->slots);
  s->cand = m.alloc<D4>(s->slots);
  if (!ok || m.err != cudaSuccess) { m.free_all(); cudaStreamDestroy(s->stream); delete s; return SG_ERR_NOMEM; }
  cudaMallocHost((void**)&s->rebuild_h, sizeof(int) * n_replicas);
  cudaMallocHost((void**)&s->pin_blist, sizeof(int) * std::max(1, s->nblocks));
  cudaMallocHost((void**)&s->pin_segs, sizeof(CellSeg) * n_replicas);
  cudaMallocHost((void**)&s->pin_res, sizeof(int) * 2);
  cudaEventCreateWithFlags(&s->ev_pin, cudaEventDisableTiming);
  if (!s->rebuild_h || !s->pin_blist || !s->pin_segs || !s->pin_res) {
    for (void* h : {(void*)s->rebuild_h, (void*)s->pin_blist, (void*)s->pin_segs, (void*)s->pin_res})
      if (h) cudaFreeHost(h);
    if (s->ev_pin) cudaEventDestroy(s->ev_pin);
    m.free_all(); cudaStreamDestroy(s->stream); delete s; return SG_ERR_NOMEM;
  }
  cudaEventCreate(&s->ev_run0); cudaEventCreate(&s->ev_run1);
  cudaEventCreate(&s->ev_k0); cudaEventCreate(&s->ev_k1);
  cudaEventCreate(&s->ev_t0); cudaEventCreate(&s->ev_t1);
  cudaEventCreate(&s->ev_b0); cudaEventCreate(&s->ev_b1);
  cudaMemcpy(s->blk_rep, s->blk_rep_h.data(), sizeof(int) * s->nblocks, cudaMemcpyHostToDevice);
  cudaMemcpy(s->rep_blk0, s->rep_blk0_h.data(), sizeof(int) * n_replicas, cudaMemcpyHostToDevice);
  cudaMemcpy(s->rep_nblk, s->rep_nblk_h.data(), sizeof(int) * n_replicas, cudaMemcpyHostToDevice);
  // defaults of Particle's ctor (particle.hpp:68-90) and of the input reader
  std::vector<double> ones(s->slots, 1.0);
  std::vector<int> ids(s->slots, 0), types(s->slots, 1);
  for (int r = 0; r < n_replicas; r++)
    for (int i = 0; i < s->n[r]; i++) ids[s->off[r] + i] = i;
  cudaMemcpy(s->st.r, ones.data(), sizeof(double) * s->slots, cudaMemcpyHostToDevice);
  cudaMemcpy(s->st.mass, ones.data(), sizeof(double) * s->slots, cudaMemcpyHostToDevice);
  cudaMemcpy(s->st.id, ids.data(), sizeof(int) * s->slots, cudaMemcpyHostToDevice);
  cudaMemcpy(s->st.type, types.data(), sizeof(int) * s->slots, cudaMemcpyHostToDevice);
  // the alternate store becomes the store after a full re-sort: same padding
  cudaMemcpy(s->st_alt.r, ones.data(), sizeof(double) * s->slots, cudaMemcpyHostToDevice);
  cudaMemcpy(s->st_alt.mass, ones.data(), sizeof(double) * s->slots, cudaMemcpyHostToDevice);
  cudaMemcpy(s->st_alt.id, ids.data(), sizeof(int) * s->slots, cudaMemcpyHostToDevice);
  cudaMemcpy(s->st_alt.type, types.data(), sizeof(int) * s->slots, cudaMemcpyHostToDevice);
  s->reps_h.assign(n_replicas, Replica{});
  s->rep_builds.assign(n_replicas, 0);
  s->clk_h.assign(n_replicas, Clock{});
  for (int r = 0; r < n_replicas; r++) {
    Replica& R = s->reps_h[r];
    std::memset(&R, 0, sizeof(R));
    R.off = s->off[r]; R.n = s->n[r];
    R.Lx = R.Ly = R.Lz = 10.0;
    R.xlo = R.ylo = R.zlo = -5.0; R.xhi = R.yhi = R.zhi = 5.0;
    R.cnx = R.cny = R.cnz = 1; R.cwx = R.cwy = R.cwz = 10.0;
    Clock& C = s->clk_h[r];
    std::memset(&C, 0, sizeof(C));
    C.fire_conv_step = -1;
  }
  s->prog.ntypes = ntypes;
  for (int k = 0; k < 3; k++) s->uploaded_N[k].assign((size_t)s->slots, 0.0);
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) { m.free_all(); cudaStreamDestroy(s->stream); delete s; return SG_ERR_CUDA; }
  if (push_reps(s) != SG_OK || push_clk(s) != SG_OK) { m.free_all(); delete s; return SG_ERR_CUDA; }
  *out = s;
  return SG_OK;
}

int sg_destroy(sg_system* s) {
  if (!s) return SG_ERR_ARG;
  cudaStreamSynchronize(s->stream);
  s->mem.free_all();
  for (double* t : s->tables) cudaFree(t);
  for (void* h : {(void*)s->rebuild_h, (void*)s->pin_blist, (void*)s->pin_segs, (void*)s->pin_res})
    if (h) cudaFreeHost(h);
  if (s->ev_pin) cudaEventDestroy(s->ev_pin);
  for (cudaEvent_t ev : {s->ev_run0, s->ev_run1, s->ev_k0, s->ev_k1, s->ev_t0, s->ev_t1, s->ev_b0, s->ev_b1})
    if (ev) cudaEventDestroy(ev);
  cudaStreamDestroy(s->stream);
  delete s;
  return SG_OK;
}

int sg_set_box(sg_system* s, int replica, double lx, double ly, double lz, int periodic) {
  if (!s || replica < 0 || replica >= s->nrep || !(lx > 0.0) || !(ly > 0.0) || !(lz > 0.0))
    return fail(s, SG_ERR_ARG, "sg_set_box: bad replica or box size");
  if (s->has_nlist) return fail(s, SG_ERR_STATE, "sg_set_box: box must be set before the neighbour list");
  Replica& R = s->reps_h[replica];
  R.Lx = lx; R.Ly = ly; R.Lz = lz;
  R.xlo = -0.5 * lx; R.xhi = 0.5 * lx;
  R.ylo = -0.5 * ly; R.yhi = 0.5 * ly;
  R.zlo = -0.5 * lz; R.zhi = 0.5 * lz;
  R.periodic = periodic ? 1 : 0;
  return push_reps(s);
}

int sg_set_timestep(sg_system* s, double dt) {
  if (!s || !(dt > 0.0)) return fail(s, SG_ERR_ARG, "sg_set_timestep: dt must be > 0");
  s->dt_global = dt;
  return SG_OK;
}

// host-side id -> slot map of one replica (slots are permuted by rebuilds)
static int slot_map(sg_system* s, int replica, std::vector<int>& slot_of_id) {
  const int n = s->n[replica], off = s->off[replica];
  std::vector<int> ids(n);
  CU(s, cudaMemcpyAsync(ids.data(), s->st.id + off, sizeof(int) * n, cudaMemcpyDeviceToHost, s->stream));
  CU(s, cudaStreamSynchronize(s->stream));
  slot_of_id.assign(n, -1);
  for (int k = 0; k < n; k++) {
    if (ids[k] < 0 || ids[k] >= n) return fail(s, SG_ERR_STATE, "corrupt id map");
    slot_of_id[ids[k]] = k;
  }
  return SG_OK;
}

}  // extern "C"

// Host arrays are in particle-id order, device slots in cell order: uploads
// copy the array as it is into a staging buffer and gather it into slot order
// on the device (slot k holds particle id[k]); downloads scatter slots into
// id order on the device and copy the staging buffer back as it is.
template <class T>
__global__ void k_gather_ids(T* __restrict__ dst, const T* __restrict__ src, const int* __restrict__ id, int n,
                             int* err) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int i = id[k];
  if ((unsigned)i < (unsigned)n) dst[k] = src[i];
  else atomicOr(err, 1);
}

template <class T>
__global__ void k_scatter_ids(T* __restrict__ dst, const T* __restrict__ src, const int* __restrict__ id, int n,
                              int* err) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int i = id[k];
  if ((unsigned)i < (unsigned)n) dst[i] = src[k];
  else atomicOr(err, 1);
}

static int xfer_ready(sg_system* s) {
  if (s->xfer) return SG_OK;
  int maxn = 0;
  for (int v : s->n) maxn = std::max(maxn, v);
  s->xfer = s->mem.alloc<double>(std::max(1, maxn));
  s->xerr = s->mem.alloc<int>(1);
  if (s->mem.err != cudaSuccess) { s->mem.err = cudaSuccess; return fail(s, SG_ERR_NOMEM, "transfer staging allocation failed"); }
  return SG_OK;
}

// Copies n values of T between host (id order) and the replica's slots.
template <class T>
static int xfer_field(sg_system* s, int replica, T* dev, T* host, bool to_device) {
  int rc = xfer_ready(s);
  if (rc) return rc;
  const int n = s->n[replica], off = s->off[replica];
  if (n == 0) return SG_OK;
  T* stage = (T*)s->xfer;
  const int g = (n + 255) / 256;
  CU(s, cudaMemsetAsync(s->xerr, 0, sizeof(int), s->stream));
  if (to_device) {
    CU(s, cudaMemcpyAsync(stage, host, sizeof(T) * n, cudaMemcpyHostToDevice, s->stream));
    k_gather_ids<T><<<g, 256, 0, s->stream>>>(dev + off, stage, s->st.id + off, n, s->xerr);
  } else {
    k_scatter_ids<T><<<g, 256, 0, s->stream>>>(stage, dev + off, s->st.id + off, n, s->xerr);
    CU(s, cudaMemcpyAsync(host, stage, sizeof(T) * n, cudaMemcpyDeviceToHost, s->stream));
  }
  CU(s, cudaGetLastError());
  int bad = 0;
  CU(s, cudaMemcpyAsync(&bad, s->xerr, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  CU(s, cudaStreamSynchronize(s->stream));
  if (bad) return fail(s, SG_ERR_STATE, "corrupt id map");
  return SG_OK;
}

extern "C" {

static int field_ptr(sg_system* s, const char* field, void** p, bool* is_int, int* nfield) {
  *nfield = -1;
  for (int i = 0; i < kNumDynDouble; i++)
    if (std::strcmp(field, kDoubleFields[i]) == 0) { *p = dyn_field(s->cur, i); *is_int = false; *nfield = i; return SG_OK; }
  if (!std::strcmp(field, "radius")) { *p = s->st.r; *is_int = false; return SG_OK; }
  if (!std::strcmp(field, "mass")) { *p = s->st.mass; *is_int = false; return SG_OK; }
  if (!std::strcmp(field, "type")) { *p = s->st.type; *is_int = true; return SG_OK; }
  if (!std::strcmp(field, "ix")) { *p = s->cur.ix; *is_int = true; return SG_OK; }
  if (!std::strcmp(field, "iy")) { *p = s->cur.iy; *is_int = true; return SG_OK; }
  if (!std::strcmp(field, "iz")) { *p = s->cur.iz; *is_int = true; return SG_OK; }
  if (!std::strcmp(field, "Nx") || !std::strcmp(field, "Ny") || !std::strcmp(field, "Nz")) {
    *p = nullptr; *is_int = false; return SG_OK;
  }
  return fail(s, SG_ERR_ARG, std::string("unknown particle field '") + field + "'");
}

// Staging for `nf` fields of a replica (grown on demand, kept).
static int xfer_multi_ready(sg_system* s, int nf) {
  int rc = xfer_ready(s);
  if (rc) return rc;
  int maxn = 0;
  for (int v : s->n) maxn = std::max(maxn, v);
  const size_t need = (size_t)nf * (size_t)std::max(1, maxn);
  if (need <= s->xfer_multi_cap) return SG_OK;
  s->mem.release(s->xfer_multi);
  s->xfer_multi = s->mem.alloc<double>(need);
  if (!s->xfer_multi) { s->mem.err = cudaSuccess; s->xfer_multi_cap = 0; return fail(s, SG_ERR_NOMEM, "transfer staging"); }
  s->xfer_multi_cap = need;
  return SG_OK;
}

// Several fields in one go: every copy is enqueued back to back on the
// engine stream (the DMA engine streams them without gaps), then the id-order
// gathers or scatters, and one synchronisation at the end instead of one per
// field.  Surface normals (kept on the host) go through the one-field path.
static int xfer_fields(sg_system* s, int replica, int nf, const char* const* fields, void* const* hosts,
                       bool to_device) {
  if (!s || replica < 0 || replica >= s->nrep || nf < 1 || !fields || !hosts)
    return fail(s, SG_ERR_ARG, "multi-field transfer: bad argument");
  std::vector<void*> dps(nf);
  std::vector<char> ints(nf), staged(nf);
  for (int i = 0; i < nf; i++) {
    if (!fields[i] || !hosts[i]) return fail(s, SG_ERR_ARG, "multi-field transfer: null field or buffer");
    bool is_int; int nfld;
    int rc = field_ptr(s, fields[i], &dps[i], &is_int, &nfld);
    if (rc) return rc;
    ints[i] = is_int;
    staged[i] = dps[i] != nullptr;
    if (to_device && !std::strcmp(fields[i], "type")) {
      const int* h = (const int*)hosts[i];
      for (int k = 0; k < s->n[replica]; k++)
        if (h[k] < 1 || h[k] > s->ntypes) return fail(s, SG_ERR_ARG, "particle type outside 1..ntypes");
    }
  }
  int rc = xfer_multi_ready(s, nf);
  if (rc) return rc;
  const int n = s->n[replica], off = s->off[replica];
  if (n == 0) return SG_OK;
  const int g = (n + 255) / 256;
  const size_t slice = (size_t)std::max(1, n);
  CU(s, cudaMemsetAsync(s->xerr, 0, sizeof(int), s->stream));
  if (to_device) {
    for (int i = 0; i < nf; i++)
      if (staged[i])
        CU(s, cudaMemcpyAsync(s->xfer_multi + i * slice, hosts[i], (ints[i] ? sizeof(int) : sizeof(double)) * n,
                              cudaMemcpyHostToDevice, s->stream));
    for (int i = 0; i < nf; i++) {
      if (!staged[i]) continue;
      if (ints[i])
        k_gather_ids<int><<<g, 256, 0, s->stream>>>((int*)dps[i] + off, (const int*)(s->xfer_multi + i * slice),
                                                   s->st.id + off, n, s->xerr);
      else
        k_gather_ids<double><<<g, 256, 0, s->stream>>>((double*)dps[i] + off, s->xfer_multi + i * slice,
                                                      s->st.id + off, n, s->xerr);
    }
  } else {
    for (int i = 0; i < nf; i++) {
      if (!staged[i]) continue;
      if (ints[i])
        k_scatter_ids<int><<<g, 256, 0, s->stream>>>((int*)(s->xfer_multi + i * slice), (const int*)dps[i] + off,
                                                    s->st.id + off, n, s->xerr);
      else
        k_scatter_ids<double><<<g, 256, 0, s->stream>>>(s->xfer_multi + i * slice, (const double*)dps[i] + off,
                                                       s->st.id + off, n, s->xerr);
    }
    for (int i = 0; i < nf; i++)
      if (staged[i])
        CU(s, cudaMemcpyAsync(hosts[i], s->xfer_multi + i * slice, (ints[i] ? sizeof(int) : sizeof(double)) * n,
                              cudaMemcpyDeviceToHost, s->stream));
  }
  CU(s, cudaGetLastError());
  int bad = 0;
  CU(s, cudaMemcpyAsync(&bad, s->xerr, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  CU(s, cudaStreamSynchronize(s->stream));
  if (bad) return fail(s, SG_ERR_STATE, "corrupt id map");
  for (int i = 0; i < nf; i++)  // surface normals: the one-field path
    if (!staged[i]) {
      rc = to_device ? sg_upload(s, replica, fields[i], hosts[i]) : sg_download(s, replica, fields[i], hosts[i]);
      if (rc) return rc;
    }
  if (to_device) {
    s->e1_applied = false;
    s->forces_fresh = false;
  }
  return SG_OK;
}

int sg_upload_fields(sg_system* s, int replica, int nfields, const char* const* fields, const void* const* hosts) {
  return xfer_fields(s, replica, nfields, fields, const_cast<void* const*>(hosts), true);
}

int sg_download_fields(sg_system* s, int replica, int nfields, const char* const* fields, void* const* hosts) {
  return xfer_fields(s, replica, nfields, fields, hosts, false);
}

int sg_upload(sg_system* s, int replica, const char* field, const void* host) {
  if (!s || !field || !host || replica < 0 || replica >= s->nrep) return fail(s, SG_ERR_ARG, "sg_upload: bad argument");
  void* dp; bool is_int; int nf;
  int rc = field_ptr(s, field, &dp, &is_int, &nf);
  if (rc) return rc;
  const int n = s->n[replica], off = s->off[replica];
  if (!dp) {  // surface normal: kept on the host, used where no constraint sets it
    std::vector<int> slot_of_id;
    if ((rc = slot_map(s, replica, slot_of_id))) return rc;
    int c = field[1] - 'x';
    const double* h = (const double*)host;
    for (int i = 0; i < n; i++) s->uploaded_N[c][off + i] = h[i];
    return SG_OK;
  }
  if (is_int) {
    const int* h = (const int*)host;
    if (!std::strcmp(field, "type"))
      for (int i = 0; i < n; i++)
        if (h[i] < 1 || h[i] > s->ntypes) return fail(s, SG_ERR_ARG, "particle type outside 1..ntypes");
    rc = xfer_field<int>(s, replica, (int*)dp, (int*)host, true);
  } else {
    rc = xfer_field<double>(s, replica, (double*)dp, (double*)host, true);
  }
  if (rc) return rc;
  s->e1_applied = false;
  s->forces_fresh = false;
  return SG_OK;
}

int sg_download(sg_system* s, int replica, const char* field, void* host) {
  if (!s || !field || !host || replica < 0 || replica >= s->nrep) return fail(s, SG_ERR_ARG, "sg_download: bad argument");
  void* dp; bool is_int; int nf;
  int rc = field_ptr(s, field, &dp, &is_int, &nf);
  if (rc) return rc;
  const int n = s->n[replica], off = s->off[replica];
  if (!dp) {
    std::vector<int> ids(n);
    CU(s, cudaMemcpyAsync(ids.data(), s->st.id + off, sizeof(int) * n, cudaMemcpyDeviceToHost, s->stream));
    // surface normal of the last constraint that sets one (plane: (0,0,1),
    // sphere: x/R as in constraint_sphere.hpp:76)
    const int comp = field[1] - 'x';
    std::vector<double> X(n), Y(n), Z(n);
    CU(s, cudaMemcpyAsync(X.data(), s->cur.x + off, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
    CU(s, cudaMemcpyAsync(Y.data(), s->cur.y + off, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
    CU(s, cudaMemcpyAsync(Z.data(), s->cur.z + off, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
    CU(s, cudaStreamSynchronize(s->stream));
    double* h = (double*)host;
    for (int i = 0; i < n; i++) h[i] = s->uploaded_N[comp][off + i];
    for (int c = 0; c < s->prog.ncons; c++) {
      const int kind = s->prog.cons[c].kind;
      if (kind == CONS_PLANE || kind == CONS_PLANE_WALLS)
        for (int i = 0; i < n; i++) h[i] = comp == 2 ? 1.0 : 0.0;
      else if (kind == CONS_SLAB)  // constraint_slab.hpp:94
        for (int i = 0; i < n; i++) h[i] = 0.0;
      else if (kind != CONS_NONE) {  // compute_normal of the curved surfaces
        const ConsComp& C = s->prog.cons[c];
        const double a0 = s->reps_h[replica].cons_p[c];
        for (int k = 0; k < n; k++) {
          Part q;
          q.x = X[k]; q.y = Y[k]; q.z = Z[k];
          double N[3];
          surface_normal(C, s->reps_h[replica], a0, q, N[0], N[1], N[2]);
          h[ids[k]] = N[comp];
        }
      }
    }
    return SG_OK;
  }
  if (is_int) return xfer_field<int>(s, replica, (int*)dp, (int*)host, false);
  return xfer_field<double>(s, replica, (double*)dp, (double*)host, false);
}

// ---------------------------------------------------------------------------
// neighbour list
// ---------------------------------------------------------------------------
static int nlist_alloc(sg_system* s, int cap) {
  DevBuf& m = s->mem;
  m.release(s->nl.nb); m.release(s->nl.cnt); m.release(s->nl.lo);
  s->nl.cap = cap;
  s->nl.stride = s->slots;
  s->nl.nb = m.alloc<int>((size_t)cap * s->slots);
  s->nl.cnt = m.alloc<int>(s->slots);
  s->nl.lo = m.alloc<int>(s->slots);
  if (!s->nl.ox) { s->nl.ox = m.alloc<double>(s->slots); s->nl.oy = m.alloc<double>(s->slots); s->nl.oz = m.alloc<double>(s->slots); }
  if (m.err != cudaSuccess) { m.err = cudaSuccess; return fail(s, SG_ERR_NOMEM, "neighbour list allocation failed"); }
  return SG_OK;
}

// Rebuilds the lists of the replicas flagged in s->rebuild_h (host copy of
// the device flags).  A replica's particle arrays are also re-sorted into
// cell order on its first build and every kSortEvery-th one after (flag 2);
// otherwise only the lists are rebuilt through the cell-ordered slot index
// (flag 1).  Lists, and so results, are identical either way; the schedule
// depends only on the replica's own history.  Sets *sorted if any replica
// was re-sorted.
static constexpr int kSortEvery = 8;

// Blocks of the flagged replicas (s->rebuild_h): the particle passes of a
// rebuild launch over these only.  When every replica is flagged the list is
// left null and the passes cover the whole grid.
static int prepare_blist(sg_system* s) {
  CU(s, cudaEventSynchronize(s->ev_pin));
  int nb = 0;
  bool all = true;
  for (int r = 0; r < s->nrep; r++) {
    if (!s->rebuild_h[r]) { all = false; continue; }
    for (int b = 0; b < s->rep_nblk_h[r]; b++) s->pin_blist[nb++] = s->rep_blk0_h[r] + b;
  }
  s->nblist = all ? s->nblocks : nb;
  if (all || s->nblist == 0) return SG_OK;
  if (!s->blist) {
    s->blist = s->mem.alloc<int>(s->nblocks);
    if (!s->blist) { s->mem.err = cudaSuccess; return fail(s, SG_ERR_NOMEM, "block list"); }
  }
  CU(s, cudaMemcpyAsync(s->blist, s->pin_blist, sizeof(int) * s->nblist, cudaMemcpyHostToDevice, s->stream));
  CU(s, cudaEventRecord(s->ev_pin, s->stream));
  return SG_OK;
}
static const int* blist_of(const sg_system* s) { return s->nblist == s->nblocks ? nullptr : s->blist; }

// Team list build below this many rebuilt particles: one thread per particle
// leaves most of the GPU idle there (65,536-particle sphere: 8x the threads
// in flight); from a few 10^5 particles on, the team's extra instructions
// cost more than its shorter chains save (4,194,304 disks: 2.8 vs 1.3 ms).
static constexpr int64_t kTeamBelow = 1 << 16;

// The cell-tile build (k_rb_build_tile) applies when it is asked for (mode 3)
// and every flagged replica is quasi-2-D on the cell path (tile_eligible).
// Automatic mode does not take it: on 4,194,304 disks it measured 1.87 ms per
// rebuild against 1.22 ms for the one-thread build (its staging pass and
// block barriers cost more than the dependent loads they replace).
static bool use_tiles(const sg_system* s, int64_t nflag) {
  (void)nflag;
  if (s->build_mode != 3) return false;
  for (int r = 0; r < s->nrep; r++) {
    if (!s->rebuild_h[r]) continue;
    const Replica& R = s->reps_h[r];
    if (!tile_eligible(R.use_cell, R.cnx, R.cny, R.cnz)) return false;
  }
  return true;
}

// Tile list of the flagged replicas: per replica, per a, runs of TILE_B
// columns along b.  Reused while the flagged set is unchanged.
static int prepare_tiles(sg_system* s) {
  std::vector<int> flagged;
  for (int r = 0; r < s->nrep; r++)
    if (s->rebuild_h[r]) flagged.push_back(r);
  if (flagged == s->tiles_for && s->tiles) return SG_OK;
  std::vector<TileRef> t;
  for (int r : flagged) {
    const Replica& R = s->reps_h[r];
    for (int a = 0; a < R.cnx; a++)
      for (int b0 = 0; b0 < R.cny; b0 += TILE_B) t.push_back(TileRef{r, a, b0, std::min(TILE_B, R.cny - b0)});
  }
  if ((int)t.size() > s->tiles_cap) {
    s->mem.release(s->tiles);
    s->tiles = s->mem.alloc<TileRef>(t.size());
    if (!s->tiles) { s->mem.err = cudaSuccess; s->tiles_cap = 0; return fail(s, SG_ERR_NOMEM, "tile list"); }
    s->tiles_cap = (int)t.size();
  }
  CU(s, cudaMemcpyAsync(s->tiles, t.data(), sizeof(TileRef) * t.size(), cudaMemcpyHostToDevice, s->stream));
  CU(s, cudaStreamSynchronize(s->stream));  // t is freed on return
  s->ntiles = (int)t.size();
  s->tiles_for = flagged;
  return SG_OK;
}

static int rebuild_flagged(sg_system* s, bool* sorted, bool blist_ready = false) {
  s->forces_fresh = false;
  bool any_sort = false;
  for (int r = 0; r < s->nrep; r++) {
    if (!s->rebuild_h[r]) continue;
    const bool srt = (s->rep_builds[r] % kSortEvery) == 0;
    s->rebuild_h[r] = srt ? 2 : 1;
    any_sort = any_sort || srt;
  }
  if (sorted) *sorted = any_sort;
  CU(s, cudaMemcpyAsync(s->rebuild, s->rebuild_h, sizeof(int) * s->nrep, cudaMemcpyHostToDevice, s->stream));
  if (!blist_ready) {
    int rc = prepare_blist(s);
    if (rc) return rc;
  }
  const int* bl = blist_of(s);
  const int ng = s->nblist;
  // cell ranges of the flagged replicas (the cell passes touch only these)
  CU(s, cudaEventSynchronize(s->ev_pin));
  int nvirt = 0, nseg = 0;
  for (int r = 0; r < s->nrep; r++) {
    if (!s->rebuild_h[r]) continue;
    const Replica& R = s->reps_h[r];
    s->pin_segs[nseg++] = CellSeg{R.cell_off, R.ncell, nvirt, 0};
    nvirt += R.ncell;
  }
  if (nseg == 0) return SG_OK;
  int64_t nflag = 0;  // particles of the flagged replicas
  for (int r = 0; r < s->nrep; r++)
    if (s->rebuild_h[r]) nflag += s->n[r];
  CU(s, cudaMemcpyAsync(s->segs, s->pin_segs, sizeof(CellSeg) * nseg, cudaMemcpyHostToDevice, s->stream));
  CU(s, cudaEventRecord(s->ev_pin, s->stream));
  for (int attempt = 0; attempt < 4; attempt++) {
    k_seg_zero<<<std::min((nvirt + 255) / 256, 148 * 16), 256, 0, s->stream>>>(s->segs, nseg, nvirt, s->cell_cnt,
                                                                                  s->cell_fill);
    LAUNCH_CHECK(s);
    CU(s, cudaMemsetAsync(s->bstatus, 0, sizeof(int), s->stream));
    CU(s, cudaMemsetAsync(s->maxnb, 0, sizeof(int), s->stream));
    k_rb_bin<<<ng, BLOCK, 0, s->stream>>>(s->reps, s->blk_rep, s->rebuild, s->cur, s->pcell, s->cell_cnt, bl);
    LAUNCH_CHECK(s);
    const int nscan = (nvirt + SCAN_TILE - 1) / SCAN_TILE;
    k_scan_a<<<nscan, SCAN_T, 0, s->stream>>>(s->cell_cnt, nvirt, s->segs, nseg, s->scan_bsum);
    LAUNCH_CHECK(s);
    k_scan_b<<<1, SCAN_T, 0, s->stream>>>(s->scan_bsum, nscan);
    LAUNCH_CHECK(s);
    k_scan_c<<<nscan, SCAN_T, 0, s->stream>>>(s->cell_cnt, nvirt, s->segs, nseg, s->scan_bsum, s->cell_start);
    LAUNCH_CHECK(s);
    k_rb_scatter<<<ng, BLOCK, 0, s->stream>>>(s->reps, s->blk_rep, s->rebuild, s->pcell, s->cell_start, s->cell_fill, s->tmp,
                                            bl);
    LAUNCH_CHECK(s);
    k_rb_rank<<<ng, BLOCK, 0, s->stream>>>(s->reps, s->blk_rep, s->rebuild, s->pcell, s->cell_start, s->cell_cnt,
                                          s->tmp, s->st.id, s->perm, bl, s->cur, s->cand);
    LAUNCH_CHECK(s);
    if (any_sort) {
      k_rb_gather<<<ng, BLOCK, 0, s->stream>>>(s->reps, s->blk_rep, s->rebuild, s->perm, s->cur, s->alt, s->st,
                                               s->st_alt, bl);
      LAUNCH_CHECK(s);
      // every replica re-sorted: the gathered arrays become the store (the
      // others are scratch between steps); otherwise copy the re-sorted
      // replicas back
      bool all = true;
      for (int r = 0; r < s->nrep; r++) all = all && (s->n[r] == 0 || s->rebuild_h[r] == 2);
      if (all) {
        std::swap(s->cur, s->alt);
        std::swap(s->st, s->st_alt);
      } else {
        k_rb_copyback<<<ng, BLOCK, 0, s->stream>>>(s->reps, s->blk_rep, s->rebuild, s->alt, s->cur, s->st_alt, s->st,
                                                   bl);
        LAUNCH_CHECK(s);
      }
    }
    // a rebuild of few particles is latency bound: split each particle's
    // stencil over a team of lanes; a large quasi-2-D one stages cell tiles in
    // shared memory; any other large one: one thread per particle
    if (use_tiles(s, nflag)) {
      int trc = prepare_tiles(s);
      if (trc) return trc;
      k_rb_build_tile<<<s->ntiles, BLOCK, 0, s->stream>>>(s->reps, s->tiles, s->rebuild, s->cur, s->st, s->nl,
                                                          s->perm, s->cell_start, s->cell_cnt, s->bstatus, s->maxnb);
    } else if (s->build_mode == 2 || (s->build_mode == 0 && nflag < kTeamBelow))
      k_rb_build_team<<<ng * TEAM_SUB, TEAM * TEAM_PARTS, 0, s->stream>>>(s->reps, s->blk_rep, s->rebuild, s->cur,
                                                                          s->st, s->nl, s->perm, s->cell_start,
                                                                          s->cell_cnt, s->bstatus, s->maxnb, bl);
    else
      k_rb_build<<<ng, BLOCK, 0, s->stream>>>(s->reps, s->blk_rep, s->rebuild, s->cur, s->st, s->nl, s->cand,
                                             s->cell_start, s->cell_cnt, s->bstatus, s->maxnb, bl);
    LAUNCH_CHECK(s);
    CU(s, cudaMemcpyAsync(s->pin_res, s->bstatus, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    CU(s, cudaMemcpyAsync(s->pin_res + 1, s->maxnb, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    CU(s, cudaStreamSynchronize(s->stream));
    const int st = s->pin_res[0], mx = s->pin_res[1];
    if (!(st & ST_OVERFLOW)) {
      // tile data: re-derived for the rebuilt blocks (the others keep theirs);
      // a grown list capacity invalidates every block's positions
      // (dropped once the tuner has settled on a variant that does not read
      // them; taking such a variant later re-derives them in full)
      if (s->lane_order && s->order_valid) {
        if (s->tuned && !abp_ordered(s->abp_variant)) s->order_valid = false;
        else {
          k_lane_order<<<ng, BLOCK, 0, s->stream>>>(s->reps, s->blk_rep, s->nl, s->lane_order, bl);
          LAUNCH_CHECK(s);
        }
      }
      if (s->tile_n && s->tile_valid) {
        if (s->nbpos_cap < s->nl.cap || (s->tuned && s->abp_variant != 8)) s->tile_valid = false;
        else {
          k_tile_prep<<<ng, BLOCK, 0, s->stream>>>(s->reps, s->blk_rep, s->nl, s->tile_n, s->tile_slot, s->nbpos, bl);
          LAUNCH_CHECK(s);
        }
      }
      s->builds_run++;
      s->maxnb_seen = std::max(s->maxnb_seen, mx);
      for (int r = 0; r < s->nrep; r++)
        if (s->rebuild_h[r]) s->rep_builds[r]++;
      return SG_OK;
    }
    if (any_sort) {  // arrays are now sorted: retry as list-only rebuilds of the same replicas
      for (int r = 0; r < s->nrep; r++)
        if (s->rebuild_h[r] == 2) s->rebuild_h[r] = 1;
      any_sort = false;
      CU(s, cudaMemcpyAsync(s->rebuild, s->rebuild_h, sizeof(int) * s->nrep, cudaMemcpyHostToDevice, s->stream));
    }
    if (mx > 2 * NB_LOCAL)
      return fail(s, SG_ERR_OVERFLOW, "more than " + std::to_string(NB_LOCAL) + " neighbours on one side within rcut+pad");
    int cap = std::max(mx + 8, s->nl.cap * 2);
    int rc = nlist_alloc(s, cap);
    if (rc) return rc;
  }
  return fail(s, SG_ERR_OVERFLOW, "neighbour list did not fit after regrowth");
}

int sg_set_nlist(sg_system* s, double rcut, double pad) {
  if (!s || !(rcut > 0.0) || !(pad >= 0.0)) return fail(s, SG_ERR_ARG, "sg_set_nlist: rcut must be > 0, pad >= 0");
  const double cut = rcut + pad;
  s->rcut = rcut; s->pad = pad;
  int cell_off = 0;
  for (int r = 0; r < s->nrep; r++) {
    Replica& R = s->reps_h[r];
    // NeighbourList ctor, neighbour_list.hpp:138-150
    R.use_cell = (R.Lx > 2.0 * cut && R.Ly > 2.0 * cut && R.Lz > 2.0 * cut) ? 1 : 0;
    R.cnx = std::max(1, (int)(R.Lx / cut));
    R.cny = std::max(1, (int)(R.Ly / cut));
    R.cnz = std::max(1, (int)(R.Lz / cut));
    R.cwx = R.Lx / (double)R.cnx; R.cwy = R.Ly / (double)R.cny; R.cwz = R.Lz / (double)R.cnz;
    R.ncell = R.cnx * R.cny * R.cnz;
    R.cell_off = cell_off;
    cell_off += R.ncell;
    R.cut2 = cut * cut;
    R.pad = pad;
  }
  s->ncell_total = cell_off;
  DevBuf& m = s->mem;
  m.release(s->cell_cnt); m.release(s->cell_start); m.release(s->cell_fill); m.release(s->scan_bsum);
  s->cell_cnt = m.alloc<int>(cell_off);
  s->cell_start = m.alloc<int>(cell_off);
  s->cell_fill = m.alloc<int>(cell_off);
  s->scan_bsum = m.alloc<int>((cell_off + SCAN_TILE - 1) / SCAN_TILE + 1);
  if (!s->segs) s->segs = m.alloc<CellSeg>(s->nrep);
  if (m.err != cudaSuccess) { m.err = cudaSuccess; return fail(s, SG_ERR_NOMEM, "cell list allocation failed"); }
  int rc = push_reps(s);
  if (rc) return rc;
  if (!s->nl.nb && (rc = nlist_alloc(s, 32))) return rc;
  s->has_nlist = true;
  return sg_build_nlist(s);
}

int sg_build_nlist(sg_system* s) {
  if (!s) return SG_ERR_ARG;
  if (!s->has_nlist) return fail(s, SG_ERR_STATE, "no neighbour list configured");
  for (int r = 0; r < s->nrep; r++) s->rebuild_h[r] = 1;
  int rc = rebuild_flagged(s, nullptr);
  if (rc) return rc;
  CU(s, cudaMemsetAsync(s->rebuild, 0, sizeof(int) * s->nrep, s->stream));
  CU(s, cudaStreamSynchronize(s->stream));
  return SG_OK;
}

// Particle::coordination as NeighbourList::build_cell / build_nsq leave it
// (neighbour_list.cpp:185-206, 229-268): for every listed pair, both
// particles count it when their distance at the build, minimum image, is
// below the sum of their radii.  Output indexed by particle id.
int sg_coordination(sg_system* s, int replica, int32_t* out) {
  if (!s || !out || replica < 0 || replica >= s->nrep) return fail(s, SG_ERR_ARG, "sg_coordination: bad argument");
  if (!s->has_nlist) return fail(s, SG_ERR_STATE, "no neighbour list");
  const int n = s->n[replica], off = s->off[replica], C = s->nl.cap;
  const Replica& R = s->reps_h[replica];
  std::vector<int> cnt(n), lo(n), ids(n), nb((size_t)C * n);
  std::vector<double> X(n), Y(n), Z(n), rad(n);
  CU(s, cudaMemcpyAsync(cnt.data(), s->nl.cnt + off, sizeof(int) * n, cudaMemcpyDeviceToHost, s->stream));
  CU(s, cudaMemcpyAsync(lo.data(), s->nl.lo + off, sizeof(int) * n, cudaMemcpyDeviceToHost, s->stream));
  CU(s, cudaMemcpyAsync(ids.data(), s->st.id + off, sizeof(int) * n, cudaMemcpyDeviceToHost, s->stream));
  CU(s, cudaMemcpyAsync(X.data(), s->nl.ox + off, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
  CU(s, cudaMemcpyAsync(Y.data(), s->nl.oy + off, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
  CU(s, cudaMemcpyAsync(Z.data(), s->nl.oz + off, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
  CU(s, cudaMemcpyAsync(rad.data(), s->st.r + off, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
  for (int q = 0; q < C; q++)
    CU(s, cudaMemcpyAsync(nb.data() + (size_t)q * n, s->nl.nb + (size_t)q * s->nl.stride + off, sizeof(int) * n,
                          cudaMemcpyDeviceToHost, s->stream));
  CU(s, cudaStreamSynchronize(s->stream));
  for (int i = 0; i < n; i++) out[i] = 0;
  for (int k = 0; k < n; k++)
    for (int q = lo[k]; q < cnt[k]; q++) {  // each pair once: from its lower-id end
      const int m = nb[(size_t)q * n + k] - off;
      double dx = X[k] - X[m], dy = Y[k] - Y[m], dz = Z[k] - Z[m];
      if (R.periodic) {  // System::apply_periodic, system.cpp:1083-1094
        if (dx > R.xhi) dx -= R.Lx; else if (dx < R.xlo) dx += R.Lx;
        if (dy > R.yhi) dy -= R.Ly; else if (dy < R.ylo) dy += R.Ly;
        if (dz > R.zhi) dz -= R.Lz; else if (dz < R.zlo) dz += R.Lz;
      }
      const double d2 = dx * dx + dy * dy + dz * dz;
      const double r = rad[k] + rad[m];
      if (d2 < r * r) { out[ids[k]]++; out[ids[m]]++; }
    }
  return SG_OK;
}

int sg_get_pairs(sg_system* s, int replica, int32_t* out_i, int32_t* out_j, int64_t cap, int64_t* n_pairs) {
  if (!s || replica < 0 || replica >= s->nrep || !n_pairs) return fail(s, SG_ERR_ARG, "sg_get_pairs: bad argument");
  if (!s->has_nlist) return fail(s, SG_ERR_STATE, "no neighbour list");
  const int n = s->n[replica], off = s->off[replica], C = s->nl.cap;
  std::vector<int> cnt(n), lo(n), ids(n), nb((size_t)C * n);
  CU(s, cudaMemcpyAsync(cnt.data(), s->nl.cnt + off, sizeof(int) * n, cudaMemcpyDeviceToHost, s->stream));
  CU(s, cudaMemcpyAsync(lo.data(), s->nl.lo + off, sizeof(int) * n, cudaMemcpyDeviceToHost, s->stream));
  CU(s, cudaMemcpyAsync(ids.data(), s->st.id + off, sizeof(int) * n, cudaMemcpyDeviceToHost, s->stream));
  for (int q = 0; q < C; q++)
    CU(s, cudaMemcpyAsync(nb.data() + (size_t)q * n, s->nl.nb + (size_t)q * s->nl.stride + off, sizeof(int) * n,
                          cudaMemcpyDeviceToHost, s->stream));
  CU(s, cudaStreamSynchronize(s->stream));
  // emit list[i] for i ascending: the upper part of particle i's list
  std::vector<int> slot_of_id(n);
  for (int k = 0; k < n; k++) slot_of_id[ids[k]] = k;
  int64_t total = 0;
  for (int i = 0; i < n; i++) {
    int k = slot_of_id[i];
    for (int q = lo[k]; q < cnt[k]; q++) {
      if (total < cap && out_i && out_j) { out_i[total] = i; out_j[total] = ids[nb[(size_t)q * n + k] - off]; }
      total++;
    }
  }
  *n_pairs = total;
  return total > cap ? fail(s, SG_ERR_ARG, "sg_get_pairs: capacity too small") : SG_OK;
}

// ---------------------------------------------------------------------------
// components
// ---------------------------------------------------------------------------
static Value make_value(const double* v) {
  Value r{};
  if (!v) { r.kind = 0; r.min_val = 0.0; r.max_val = 1.0; r.steps = 1000; r.dv = 0.0; return r; }
  r.kind = (int)v[0]; r.min_val = v[1]; r.max_val = v[2]; r.steps = (int)v[3];
  r.dv = (r.max_val - r.min_val) / (double)r.steps;
  return r;
}

static double* upload_table(sg_system* s, const std::vector<double>& t) {
  double* d = nullptr;
  if (cudaMalloc(&d, sizeof(double) * std::max<size_t>(1, t.size())) != cudaSuccess) return nullptr;
  cudaMemcpy(d, t.data(), sizeof(double) * t.size(), cudaMemcpyHostToDevice);
  s->tables.push_back(d);
  return d;
}

int sg_add_pair(sg_system* s, int kind, const double* global, const double* table, int use_radii,
                int phase_in, int shifted, int has_pp, const double* phase_value) {
  if (!s || kind < SG_PAIR_SOFT || kind > SG_PAIR_GAUSSIAN || !global) return fail(s, SG_ERR_ARG, "sg_add_pair: bad kind");
  Program& P = s->prog;
  if (P.npair >= MAX_PAIR) return fail(s, SG_ERR_ARG, "too many pair potentials");
  for (int c = 0; c < P.npair; c++)
    if (P.pair[c].kind == kind) return fail(s, SG_ERR_ARG, "pair potential already defined");
  const size_t nt = (size_t)s->ntypes * s->ntypes * PAIR_NPARAM;
  std::vector<double> t(nt);
  for (size_t i = 0; i < nt; i++) t[i] = table ? table[i] : global[i % PAIR_NPARAM];
  PairComp& C = P.pair[P.npair];
  C.kind = kind; C.use_radii = use_radii; C.phase_in = phase_in; C.shifted = shifted; C.has_pp = has_pp;
  C.phase = make_value(phase_value);
  C.table = upload_table(s, t);
  if (!C.table) return fail(s, SG_ERR_NOMEM, "table allocation failed");
  s->pair_tab_h.push_back(t);
  for (int r = 0; r < s->nrep; r++)
    for (int i = 0; i < PAIR_NPARAM; i++) s->reps_h[r].pair_g[P.npair][i] = global[i];
  P.npair++;
  return push_reps(s);
}

int sg_add_align(sg_system* s, int kind, double J, double rcut, const double* table, int has_pp) {
  if (!s || kind < SG_ALIGN_POLAR || kind > SG_ALIGN_VICSEK) return fail(s, SG_ERR_ARG, "sg_add_align: bad kind");
  Program& P = s->prog;
  if (P.nalign >= MAX_ALIGN) return fail(s, SG_ERR_ARG, "too many aligners");
  const size_t nt = (size_t)s->ntypes * s->ntypes * 2;
  std::vector<double> t(nt);
  for (size_t i = 0; i < nt; i++) t[i] = table ? table[i] : ((i & 1) ? rcut : J);
  AlignComp& C = P.align[P.nalign];
  C.kind = kind; C.has_pp = has_pp;
  C.table = upload_table(s, t);
  if (!C.table) return fail(s, SG_ERR_NOMEM, "table allocation failed");
  s->align_tab_h.push_back(t);
  for (int r = 0; r < s->nrep; r++) { s->reps_h[r].align_J[P.nalign] = J; s->reps_h[r].align_rcut[P.nalign] = rcut; }
  P.nalign++;
  return push_reps(s);
}

int sg_add_external(sg_system* s, int kind, double alpha, const double* type_alpha, int has_params) {
  if (!s || kind != SG_EXT_SELF_PROPULSION) return fail(s, SG_ERR_ARG, "sg_add_external: bad kind");
  Program& P = s->prog;
  if (P.next >= MAX_EXT) return fail(s, SG_ERR_ARG, "too many external potentials");
  std::vector<double> t(s->ntypes);
  for (int i = 0; i < s->ntypes; i++) t[i] = type_alpha ? type_alpha[i] : alpha;
  ExtComp& C = P.ext[P.next];
  C.kind = kind; C.has_params = has_params;
  C.type_alpha = upload_table(s, t);
  s->ext_tab_h.push_back(t);
  for (int r = 0; r < s->nrep; r++) s->reps_h[r].ext_alpha[P.next] = alpha;
  P.next++;
  return push_reps(s);
}

// Program-level part of a constraint: kind, plane flag, the second and third
// shape parameters (params[7], params[8]: torus a; ellipsoid b, c; peanut b;
// hourglass A, n; gaussian bump a, b) and the SHAKE settings of the implicit
// surfaces (maxiter params[2], tol params[3]).  Without params the
// reference's defaults (peanut: a 10, b 8, which its b > a check rejects).
static void set_cons(ConsComp& C, int kind, const double* params) {
  C.kind = kind;
  C.unlimited = (kind == CONS_PLANE && params) ? (int)params[1] : 0;
  C.max_iter = params ? (int)params[2] : 100;
  C.tol = params ? params[3] : 1e-6;
  double d2 = 0.0, d3 = 0.0;
  if (kind == CONS_TORUS) d2 = 0.5;
  else if (kind == CONS_ELLIPSOID) { d2 = 1.0; d3 = 1.0; }
  else if (kind == CONS_PEANUT) d2 = 8.0;
  else if (kind == CONS_HOURGLASS) { d2 = 1.0; d3 = 1.0; }
  else if (kind == CONS_GAUSSIAN_BUMP) { d2 = 1.0; d3 = 1.0; }
  else if (kind == CONS_SLAB) d2 = 1.0;  // z_hi (constraint_slab.hpp:68-78)
  else if (kind == CONS_TETRAHEDRON) d2 = 1.0;  // value (constraint_tetrahedron.hpp:78-88)
  C.b2 = params ? params[7] : d2;
  C.b3 = params ? params[8] : d3;
}

static bool rescales(int kind) { return kind == CONS_SPHERE || kind == CONS_CYLINDER || kind == CONS_TETRAHEDRON; }

static void set_rescale(sg_system* s, int c, const double* params) {
  if ((int)s->cons_rescale.size() <= c) s->cons_rescale.resize(c + 1);
  sg_system::Rescale& q = s->cons_rescale[c];
  q = sg_system::Rescale();
  // the other constraints take the parameters and keep the base class's
  // no-op rescale (constraint.hpp:144)
  if (!params || params[4] == 0.0 || !rescales(s->prog.cons[c].kind)) return;
  q.rescale = params[4];
  q.steps = (int)params[5];
  q.freq = (int)params[6];
  q.scale = std::pow(q.rescale, (double)q.freq / (double)q.steps);
}

static bool rescaling(const sg_system* s) {
  for (int c = 0; c < s->prog.ncons && c < (int)s->cons_rescale.size(); c++)
    if (s->cons_rescale[c].rescale != 1.0) return true;
  return false;
}

// Constrainer::rescale (constrainer.hpp:117-123) at global step `step`: the
// first constraint due scales its size (every replica) and projects every
// particle onto the new surface; true when one did (the caller then rebuilds
// the lists).  Sphere radius (constraint_sphere.cpp:87-104) and tetrahedron
// scale (constraint_tetrahedron.cpp:88-109) on steps below rescale_steps,
// cylinder radius (constraint_cylinder.cpp:79-96) up to and including it.
static int apply_rescale(sg_system* s, int64_t step, bool* done) {
  *done = false;
  for (int c = 0; c < s->prog.ncons && c < (int)s->cons_rescale.size(); c++) {
    const sg_system::Rescale& q = s->cons_rescale[c];
    const bool in_range = s->prog.cons[c].kind == CONS_CYLINDER ? step <= q.steps : step < q.steps;
    if (q.rescale == 1.0 || step % q.freq != 0 || !in_range) continue;
    for (int r = 0; r < s->nrep; r++) s->reps_h[r].cons_p[c] *= q.scale;
    int rc = push_reps(s);
    if (rc) return rc;
    k_enforce<<<s->nblocks, BLOCK, 0, s->stream>>>(s->prog, s->reps, s->blk_rep, s->cur, s->st, nullptr);
    LAUNCH_CHECK(s);
    *done = true;
    return SG_OK;
  }
  return SG_OK;
}

static double cons_first_default(int kind) {
  return kind == CONS_PLANE || kind == CONS_NONE || kind == CONS_GYROID || kind == CONS_SLAB ? 0.0
       : kind == CONS_PEANUT || kind == CONS_HOURGLASS || kind == CONS_TETRAHEDRON ? 10.0 : 1.0;
}

// a wall position beyond the box is moved to its edge
// (constraint_plane_walls.hpp:64-71)
static double cons_first_of(const sg_system* s, int kind, double first, int r) {
  return kind == CONS_PLANE_WALLS && first > s->reps_h[r].xhi ? s->reps_h[r].xhi : first;
}

// the peanut constructor's check (constraint_peanut.hpp:84-88); the
// hourglass one applies only to an amplitude given explicitly, so the hosts
// make it where they parse the parameters
static int check_cons(sg_system* s, const ConsComp& C, double first) {
  if (C.kind == CONS_PEANUT && C.b2 <= first)
    return fail(s, SG_ERR_ARG, "Parameter b has to be larger than parameter a. Otherwise the surface will be disconnected.");
  return SG_OK;
}

int sg_add_constraint_per_replica(sg_system* s, int kind, const double* params, const double* value0) {
  if (!s || !value0 || kind < SG_CONS_NONE || kind > SG_CONS_TETRAHEDRON) return fail(s, SG_ERR_ARG, "bad constraint");
  Program& P = s->prog;
  if (P.ncons >= MAX_CONS) return fail(s, SG_ERR_ARG, "too many constraints");
  if (params && params[4] != 0.0 && params[4] != 1.0 && kind == CONS_PLANE)
    return fail(s, SG_ERR_UNSUPPORTED, "constraint rescale of the plane's box is not part of the GPU path");
  set_cons(P.cons[P.ncons], kind, params);
  for (int r = 0; r < s->nrep; r++) {
    int rc = check_cons(s, P.cons[P.ncons], value0[r]);
    if (rc) return rc;
  }
  set_rescale(s, P.ncons, params);
  for (int r = 0; r < s->nrep; r++) s->reps_h[r].cons_p[P.ncons] = cons_first_of(s, kind, value0[r], r);
  P.ncons++;
  int rc = push_reps(s);
  if (rc) return rc;
  return sg_enforce(s);
}

int sg_add_constraint(sg_system* s, int kind, const double* params) {
  if (!s || kind < SG_CONS_NONE || kind > SG_CONS_TETRAHEDRON) return fail(s, SG_ERR_ARG, "sg_add_constraint: bad kind");
  Program& P = s->prog;
  if (P.ncons >= MAX_CONS) return fail(s, SG_ERR_ARG, "too many constraints");
  if (params && params[4] != 0.0 && params[4] != 1.0 && kind == CONS_PLANE)
    return fail(s, SG_ERR_UNSUPPORTED, "constraint rescale of the plane's box is not part of the GPU path");
  set_cons(P.cons[P.ncons], kind, params);
  const double first = params ? params[0] : cons_first_default(kind);
  if (int rc = check_cons(s, P.cons[P.ncons], first)) return rc;
  set_rescale(s, P.ncons, params);
  for (int r = 0; r < s->nrep; r++) s->reps_h[r].cons_p[P.ncons] = cons_first_of(s, kind, first, r);
  P.ncons++;
  int rc = push_reps(s);
  if (rc) return rc;
  return sg_enforce(s);  // samos.cpp:518-522
}

int sg_add_integrator(sg_system* s, int kind, const double* params, const double* temp) {
  if (!s || !params || kind < SG_INT_BROWNIAN || kind > SG_INT_VICSEK) return fail(s, SG_ERR_ARG, "sg_add_integrator: bad kind");
  Program& P = s->prog;
  if (P.ninteg >= MAX_INTEG) return fail(s, SG_ERR_ARG, "too many integrators");
  if (!(params[0] > 0.0)) return fail(s, SG_ERR_ARG, "integrator step size has to be larger than 0");
  IntegComp& C = P.integ[P.ninteg];
  C.kind = kind;
  C.method = kind == INT_LANGEVIN ? (int)params[10] : 0;
  C.nematic = (kind == INT_BROWNIAN || kind == INT_BROWNIAN_ALIGN) ? (params[6] != 0.0) : 0;
  C.velocity = kind == INT_BROWNIAN ? (params[8] != 0.0) : 0;
  C.group = 0;
  C.temp = make_value(temp);
  const int c = P.ninteg;
  for (int r = 0; r < s->nrep; r++) {
    for (int i = 0; i < INT_NPARAM; i++) s->reps_h[r].integ_p[c][i] = params[i];
    s->reps_h[r].seed[c] = (uint32_t)(int32_t)params[5];
    s->clk_h[r].ctr[c] = 0;
  }
  P.ninteg++;
  int rc = push_reps(s);
  if (rc) return rc;
  if (kind == INT_FIRE) {
    for (int r = 0; r < s->nrep; r++) {
      Clock& K = s->clk_h[r];
      K.fire_dt = params[0]; K.fire_alpha = params[1]; K.fire_old_e = 1e15;
      K.fire_last_neg = 0; K.fire_converged = 0; K.fire_conv_step = -1;
    }
  }
  if (kind == INT_LANGEVIN && C.method == LANGEVIN_BBK) {
    // integrator_langevin.hpp:103-111: 3 draws per particle at construction
    if (!s->Rn) s->Rn = s->mem.alloc<double>((size_t)3 * s->slots);
    std::vector<double> h((size_t)3 * s->slots, 0.0);
    for (int r = 0; r < s->nrep; r++) {
      uint32_t seed = s->reps_h[r].seed[c];
      for (int i = 0; i < s->n[r]; i++)
        for (int d = 0; d < 3; d++) {
          // same stream as the device: counter = 3 i + d
          h[(size_t)3 * (s->off[r] + i) + d] = noise_gauss(seed, (uint64_t)3 * i + d);
        }
      s->clk_h[r].ctr[c] = (uint64_t)3 * s->n[r];
    }
    CU(s, cudaMemcpy(s->Rn, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice));
  }
  return push_clk(s);
}

// Move integrator `from` to position `to` (program entry, per-replica
// parameters, seed and noise counter move together).
static void move_integrator(sg_system* s, int from, int to) {
  Program& P = s->prog;
  while (from != to) {
    const int a = from, b = from < to ? from + 1 : from - 1;
    std::swap(P.integ[a], P.integ[b]);
    for (int r = 0; r < s->nrep; r++) {
      Replica& R = s->reps_h[r];
      for (int i = 0; i < INT_NPARAM; i++) std::swap(R.integ_p[a][i], R.integ_p[b][i]);
      std::swap(R.seed[a], R.seed[b]);
      std::swap(s->clk_h[r].ctr[a], s->clk_h[r].ctr[b]);
    }
    from = b;
  }
}

int sg_insert_integrator(sg_system* s, int pos, int kind, const double* params, const double* temp) {
  if (!s) return SG_ERR_ARG;
  if (pos < 0 || pos > s->prog.ninteg) return fail(s, SG_ERR_ARG, "sg_insert_integrator: bad position");
  int rc = pull_clk(s);
  if (rc) return rc;
  if ((rc = sg_add_integrator(s, kind, params, temp))) return rc;
  move_integrator(s, s->prog.ninteg - 1, pos);
  if ((rc = push_reps(s))) return rc;
  return push_clk(s);
}

int sg_define_group(sg_system* s, int replica, int group, const uint8_t* member) {
  if (!s || !member || replica < 0 || replica >= s->nrep || group < 1 || group >= MAX_GROUPS)
    return fail(s, SG_ERR_ARG, "sg_define_group: bad replica, group index or member array");
  CU(s, cudaStreamSynchronize(s->stream));
  if (!s->gmask) {
    s->gmask = s->mem.alloc<uint8_t>(s->slots);
    s->grank = s->mem.alloc<int>((size_t)MAX_GROUPS * s->slots);
    if (!s->gmask || !s->grank) { s->mem.err = cudaSuccess; return fail(s, SG_ERR_NOMEM, "group tables"); }
    s->gmask_h.assign(s->slots, 0);
    CU(s, cudaMemsetAsync(s->gmask, 0, s->slots, s->stream));
  }
  const int n = s->n[replica], off = s->off[replica];
  std::vector<int> rank(n, -1);
  int size = 0;
  for (int i = 0; i < n; i++) {  // members in particle-index order (System::make_group, system.cpp:558-567)
    const uint8_t bit = (uint8_t)(1u << group);
    if (member[i]) { rank[i] = size++; s->gmask_h[off + i] |= bit; }
    else s->gmask_h[off + i] &= (uint8_t)~bit;
  }
  s->reps_h[replica].gsize[group] = size;
  CU(s, cudaMemcpyAsync(s->gmask + off, s->gmask_h.data() + off, n, cudaMemcpyHostToDevice, s->stream));
  CU(s, cudaMemcpyAsync(s->grank + (size_t)group * s->slots + off, rank.data(), sizeof(int) * n,
                        cudaMemcpyHostToDevice, s->stream));
  CU(s, cudaStreamSynchronize(s->stream));
  return push_reps(s);
}

int sg_set_integrator_group(sg_system* s, int index, int group) {
  if (!s || index < 0 || index >= s->prog.ninteg || group < 0 || group >= MAX_GROUPS)
    return fail(s, SG_ERR_ARG, "sg_set_integrator_group: bad integrator or group index");
  const int kind = s->prog.integ[index].kind;
  if (group && kind != INT_BROWNIAN && kind != INT_BROWNIAN_POS && kind != INT_BROWNIAN_ALIGN && kind != INT_VICSEK)
    return fail(s, SG_ERR_UNSUPPORTED, "integrator groups other than 'all' are supported for brownian, brownian_pos, "
                                       "brownian_align and vicsek");
  if (group && !s->gmask) return fail(s, SG_ERR_STATE, "sg_set_integrator_group: group not defined");
  s->prog.integ[index].group = group;
  return SG_OK;
}

int sg_disable_integrator(sg_system* s, int index) {
  if (!s) return SG_ERR_ARG;
  if (index < 0 || index >= s->prog.ninteg) return fail(s, SG_ERR_ARG, "sg_disable_integrator: no such integrator");
  int rc = pull_clk(s);
  if (rc) return rc;
  move_integrator(s, index, s->prog.ninteg - 1);
  s->prog.ninteg--;
  s->e1_applied = false;
  s->forces_fresh = false;
  if ((rc = push_reps(s))) return rc;
  return push_clk(s);
}

int sg_clear_forces(sg_system* s) {
  if (!s) return SG_ERR_ARG;
  CU(s, cudaStreamSynchronize(s->stream));
  Program& P = s->prog;
  P.npair = P.nalign = P.next = 0;
  s->pair_tab_h.clear(); s->align_tab_h.clear(); s->ext_tab_h.clear();
  s->forces_fresh = false;
  return SG_OK;
}

int sg_set_replica_param(sg_system* s, int replica, int cls, int comp, int slot, double value) {
  if (!s || replica < 0 || replica >= s->nrep) return fail(s, SG_ERR_ARG, "sg_set_replica_param: bad replica");
  Replica& R = s->reps_h[replica];
  switch (cls) {
    case 0: if (comp >= s->prog.npair || slot < 0 || slot >= PAIR_NPARAM) return SG_ERR_ARG; R.pair_g[comp][slot] = value; break;
    case 1:
      if (comp >= s->prog.nalign || slot < 0 || slot > 1) return SG_ERR_ARG;
      if (slot == 0) R.align_J[comp] = value; else R.align_rcut[comp] = value;
      break;
    case 2: if (comp >= s->prog.next) return SG_ERR_ARG; R.ext_alpha[comp] = value; break;
    case 3: if (comp >= s->prog.ncons) return SG_ERR_ARG; R.cons_p[comp] = value; break;
    case 4:
      if (comp >= s->prog.ninteg || slot < 0 || slot >= INT_NPARAM) return SG_ERR_ARG;
      R.integ_p[comp][slot] = value;
      if (slot == 5) R.seed[comp] = (uint32_t)(int32_t)value;
      if (slot == 0 && s->prog.integ[comp].kind == INT_FIRE) { s->clk_h[replica].fire_dt = value; push_clk(s); }
      if (slot == 1 && s->prog.integ[comp].kind == INT_FIRE) { s->clk_h[replica].fire_alpha = value; push_clk(s); }
      break;
    default: return fail(s, SG_ERR_ARG, "sg_set_replica_param: bad class");
  }
  return push_reps(s);
}

// ---------------------------------------------------------------------------
// execution
// ---------------------------------------------------------------------------
static int rebuild_pending(sg_system* s, int shape, bool last, double* rebuild_ms);

int sg_begin_step(sg_system* s) {
  if (!s) return SG_ERR_ARG;
  if (!s->e1_applied && rescaling(s) && s->rescaled_at < 0) {
    // a rescale due at this step comes before its enforce (samos.cpp:882-888)
    int rc = pull_clk(s);
    if (rc) return rc;
    const int64_t step = s->clk_h[0].time_step;
    bool scaled = false;
    if ((rc = apply_rescale(s, step, &scaled))) return rc;
    s->rescaled_at = step;  // the run continuing from here skips it
    if (scaled && s->has_nlist) {
      for (int r = 0; r < s->nrep; r++) s->rebuild_h[r] = 1;
      double ms = 0.0;
      if ((rc = rebuild_pending(s, HOT_NONE, false, &ms))) return rc;
    }
  }
  if (!s->e1_applied) {
    k_enforce<<<s->nblocks, BLOCK, 0, s->stream>>>(s->prog, s->reps, s->blk_rep, s->cur, s->st, nullptr);
    LAUNCH_CHECK(s);
    s->e1_applied = true;
  }
  CU(s, cudaStreamSynchronize(s->stream));
  return SG_OK;
}

int sg_enforce(sg_system* s) {
  if (!s) return SG_ERR_ARG;
  k_enforce<<<s->nblocks, BLOCK, 0, s->stream>>>(s->prog, s->reps, s->blk_rep, s->cur, s->st, nullptr);
  LAUNCH_CHECK(s);
  CU(s, cudaStreamSynchronize(s->stream));
  return SG_OK;
}

static int launch_force(sg_system* s, double dt, bool fire_dt, bool with_pair, bool with_align, bool energy,
                        int ng = -1, const int* bl = nullptr) {
  if (ng < 0) ng = s->nblocks;
  if (energy)
    k_force<true><<<ng, BLOCK, 0, s->stream>>>(s->prog, s->reps, s->blk_rep, s->clk, s->cur, s->st, s->nl, dt,
                                               fire_dt, with_pair, with_align, s->epart, s->nblocks, bl);
  else
    k_force<false><<<ng, BLOCK, 0, s->stream>>>(s->prog, s->reps, s->blk_rep, s->clk, s->cur, s->st, s->nl, dt,
                                                fire_dt, with_pair, with_align, s->epart, s->nblocks, bl);
  LAUNCH_CHECK(s);
  return SG_OK;
}

int sg_compute(sg_system* s, double dt) {
  if (!s) return SG_ERR_ARG;
  if (!s->has_nlist && (s->prog.npair + s->prog.nalign) > 0) return fail(s, SG_ERR_STATE, "pair terms need a neighbour list");
  if (!s->nl.nb) { int rc = nlist_alloc(s, 1); if (rc) return rc; }
  int rc = launch_force(s, dt, false, true, true, true);
  if (rc) return rc;
  CU(s, cudaStreamSynchronize(s->stream));
  return SG_OK;
}

static bool fused_program(const Program& P) {
  for (int c = 0; c < P.ninteg; c++)
    if (P.integ[c].kind != INT_BROWNIAN && P.integ[c].kind != INT_BROWNIAN_POS && P.integ[c].kind != INT_BROWNIAN_ALIGN &&
        P.integ[c].kind != INT_VICSEK)
      return false;
  return true;
}

// one unfused integration step (reference phase order, in place)
// True when the start-of-step force pass would reproduce the forces of the
// previous step's FIRE pass bit for bit: periodic plane only (the enforce
// leaves positions unchanged), no aligners or external potentials (forces
// then depend on positions alone) and no neighbour-list rebuild in between.
static bool fire_forces_reusable(const sg_system* s) {
  const Program& P = s->prog;
  if (P.nalign || P.next || P.ncons != 1 || P.cons[0].kind != CONS_PLANE) return false;
  for (int c = 0; c < P.ninteg; c++)
    if (P.integ[c].kind != INT_FIRE) return false;
  for (const Replica& R : s->reps_h)
    if (!R.periodic || !(R.cons_p[0] > R.zlo && R.cons_p[0] <= R.zhi)) return false;
  return true;
}

// The same for one Langevin (BAOAB or BBK: no position change after their
// force pass, integrator_langevin.cpp:100-116, 228-252) or NVE integrator
// (after its pass only velocities, omega and ages change, integrator_nve.cpp:
// 104-140): periodic plane with zpos in the box, no external potentials, no
// phase-in (ages advance after the pass).  Their start-of-step torques are
// never read (Langevin ignores torques; NVE recomputes them in its own pass
// before project_torque), so aligners do not stop the reuse; a step that
// reports energies recomputes everything.
static bool integ_forces_reusable(const sg_system* s) {
  const Program& P = s->prog;
  if (P.next || P.ncons != 1 || P.cons[0].kind != CONS_PLANE || P.ninteg != 1) return false;
  const IntegComp& ic = P.integ[0];
  if (!(ic.kind == INT_NVE || (ic.kind == INT_LANGEVIN && ic.method != LANGEVIN_SPV))) return false;
  for (int c = 0; c < P.npair; c++)
    if (P.pair[c].phase_in) return false;
  for (const Replica& R : s->reps_h)
    if (!R.periodic || !(R.cons_p[0] > R.zlo && R.cons_p[0] <= R.zhi)) return false;
  return true;
}

static int step_unfused(sg_system* s, bool energy, bool driver) {
  const int nb = s->nblocks;
  // the minimiser launches the per-particle passes over the blocks of the
  // replicas still running (converged replicas are frozen, their blocks would
  // only return)
  const int* al = driver && s->nact < nb ? s->act : nullptr;
  const int na = driver ? s->nact : nb;
  const bool reuse_forces =
      s->forces_fresh && (fire_forces_reusable(s) || (!energy && integ_forces_reusable(s)));
  // FIRE alone with reused forces: the start-of-step enforce runs inside the
  // first FIRE pass
  // (and the first half of a Langevin / NVE step likewise)
  const bool fuse_enforce = !s->e1_applied && reuse_forces && s->prog.ninteg == 1 &&
                            (s->prog.integ[0].kind == INT_FIRE || s->prog.integ[0].kind == INT_LANGEVIN ||
                             s->prog.integ[0].kind == INT_NVE);
  // the skin test runs inside the last pass of a step that has one integrator
  const int skin_in = s->has_nlist && s->prog.ninteg == 1 ? 1 : 0;
  if (!s->e1_applied && !fuse_enforce) {  // samos.cpp:887-888 (already applied by sg_begin_step)
    k_enforce<<<na, BLOCK, 0, s->stream>>>(s->prog, s->reps, s->blk_rep, s->cur, s->st, driver ? s->clk : nullptr, al);
    LAUNCH_CHECK(s);
  }
  int rc = SG_OK;
  bool skin_done = false;  // FIRE runs the skin test inside its last pass
  if (!reuse_forces)
    if ((rc = launch_force(s, s->dt_global, false, true, true, energy, na, al))) return rc;
  s->forces_fresh = false;
  for (int c = 0; c < s->prog.ninteg; c++) {
    const IntegComp& ic = s->prog.integ[c];
    if (ic.kind == INT_LANGEVIN) {
      k_langevin_a<<<nb, BLOCK, 0, s->stream>>>(s->prog, s->reps, s->blk_rep, s->clk, s->cur, s->st, c, s->Rn,
                                                fuse_enforce ? 1 : 0);
      LAUNCH_CHECK(s);
      if ((rc = launch_force(s, s->reps_h[0].integ_p[c][0], false, true, false, energy))) return rc;
      k_langevin_b<<<nb, BLOCK, 0, s->stream>>>(s->prog, s->reps, s->blk_rep, s->clk, s->cur, s->st, c, s->Rn, s->nl,
                                                s->rebuild, s->status, skin_in);
      LAUNCH_CHECK(s);
      s->forces_fresh = true;
      skin_done = skin_in != 0;
    } else if (ic.kind == INT_NVE) {
      k_nve_a<<<nb, BLOCK, 0, s->stream>>>(s->prog, s->reps, s->blk_rep, s->clk, s->cur, s->st, c, fuse_enforce ? 1 : 0);
      LAUNCH_CHECK(s);
      if ((rc = launch_force(s, s->reps_h[0].integ_p[c][0], false, true, true, energy))) return rc;
      k_nve_b<<<nb, BLOCK, 0, s->stream>>>(s->prog, s->reps, s->blk_rep, s->clk, s->cur, s->st, c, s->nl, s->rebuild,
                                           s->status, skin_in);
      LAUNCH_CHECK(s);
      s->forces_fresh = true;
      skin_done = skin_in != 0;
    } else if (ic.kind == INT_FIRE) {
      k_fire_a<<<na, BLOCK, 0, s->stream>>>(s->prog, s->reps, s->blk_rep, s->clk, s->cur, s->st, fuse_enforce ? 1 : 0,
                                            al);
      LAUNCH_CHECK(s);
      if ((rc = launch_force(s, 0.0, true, true, true, true, na, al))) return rc;
      s->forces_fresh = true;
      if (s->fire_ordered && !s->fire_terms) {
        s->fire_terms = s->mem.alloc<double>((size_t)3 * s->slots);
        if (!s->fire_terms) { s->mem.err = cudaSuccess; return fail(s, SG_ERR_NOMEM, "FIRE term arrays"); }
      }
      k_fire_b<<<na, BLOCK, 0, s->stream>>>(s->prog, s->reps, s->blk_rep, s->clk, s->cur, s->st, s->fire_part, nb,
                                            s->rep_blk0, s->rep_nblk, s->epart, c, driver ? 1 : 0, s->alpha_mix,
                                            s->fire_cnt, al, s->fire_ordered ? s->fire_terms : nullptr, s->slots);
      LAUNCH_CHECK(s);
      k_fire_d<<<na, BLOCK, 0, s->stream>>>(s->prog, s->reps, s->blk_rep, s->clk, s->cur, s->alpha_mix, s->nl,
                                            s->has_nlist ? 1 : 0, s->rebuild, s->status, al);
      LAUNCH_CHECK(s);
      skin_done = true;
    } else {
      return fail(s, SG_ERR_UNSUPPORTED, "mixing Brownian-family integrators with Langevin/FIRE is not supported");
    }
  }
  if (s->has_nlist && !skin_done) {
    k_skin<<<na, BLOCK, 0, s->stream>>>(s->prog, s->reps, s->blk_rep, s->cur, s->nl, s->rebuild, s->status, al);
    LAUNCH_CHECK(s);
  }
  return SG_OK;
}

static constexpr int kGenMinb[2] = {8, 6};
static constexpr int kGenTuneReps = 3;  // timed steps per candidate (after one untimed)

extern "C++" {
template <bool ENERGY>
static void launch_generic(sg_system* s, int minb, bool apply_e1) {
  const int nb = s->nblocks;
  if (minb == 6)
    k_step_brownian<ENERGY, 6><<<nb, BLOCK, 0, s->stream>>>(s->prog, s->reps, s->blk_rep, s->clk, s->cur, s->alt,
                                                            s->st, s->nl, s->rebuild, s->status, s->dt_global,
                                                            apply_e1 ? 1 : 0, s->epart, nb, s->gmask, s->grank,
                                                            s->slots);
  else
    k_step_brownian<ENERGY, 8><<<nb, BLOCK, 0, s->stream>>>(s->prog, s->reps, s->blk_rep, s->clk, s->cur, s->alt,
                                                            s->st, s->nl, s->rebuild, s->status, s->dt_global,
                                                            apply_e1 ? 1 : 0, s->epart, nb, s->gmask, s->grank,
                                                            s->slots);
}
}  // extern "C++"

// One generic fused step.  `may_tune`: a step launched on its own (not in a
// batch, whose halted kernels would time as empty), which may serve as one
// of the occupancy tuner's timed trials.
static int step_fused(sg_system* s, bool apply_e1, bool energy, bool may_tune = false) {
  const bool tuning = may_tune && !energy && !s->gen_pin && !s->gen_tuned;
  int cand = 0;
  if (tuning) {
    cand = (s->gen_trial / (kGenTuneReps + 1)) % 2;
    s->gen_minb = kGenMinb[cand];
    CU(s, cudaEventRecord(s->ev_t0, s->stream));
  }
  const int minb = s->gen_pin ? s->gen_pin : s->gen_minb;
  if (s->profile) CU(s, cudaEventRecord(s->ev_k0, s->stream));
  if (energy) launch_generic<true>(s, minb, apply_e1);
  else launch_generic<false>(s, minb, apply_e1);
  LAUNCH_CHECK(s);
  if (s->profile) CU(s, cudaEventRecord(s->ev_k1, s->stream));
  std::swap(s->cur, s->alt);
  if (tuning) {
    CU(s, cudaEventRecord(s->ev_t1, s->stream));
    CU(s, cudaEventSynchronize(s->ev_t1));
    float ms = 0.f;
    CU(s, cudaEventElapsedTime(&ms, s->ev_t0, s->ev_t1));
    if (s->gen_trial % (kGenTuneReps + 1) != 0) { s->gen_ms[cand] += ms; s->gen_n[cand]++; }
    s->gen_trial++;
    if (s->gen_trial >= 2 * (kGenTuneReps + 1)) {
      s->gen_minb = s->gen_ms[1] / s->gen_n[1] < s->gen_ms[0] / s->gen_n[0] ? kGenMinb[1] : kGenMinb[0];
      s->gen_tuned = true;
    }
  }
  return SG_OK;
}

// The two packed shapes: one plane constraint on a periodic box with zpos
// inside it, or one sphere constraint; Brownian-family integrators; no
// vicsek aligner (needs neighbour velocities) and no phase-in (needs ages).
static int hot_shape(const sg_system* s) {
  const Program& P = s->prog;
  if (s->force_generic == 1 || !fused_program(P) || P.ncons != 1) return HOT_NONE;
  for (int c = 0; c < P.ninteg; c++)
    if (P.integ[c].group) return HOT_NONE;  // grouped integrators: the generic fused kernel
  if (rescaling(s)) return HOT_NONE;        // the rescale acts between steps, before their enforce
  for (int c = 0; c < P.nalign; c++)
    if (P.align[c].kind == ALIGN_VICSEK) return HOT_NONE;
  for (int c = 0; c < P.ninteg; c++)
    if (P.integ[c].kind == INT_VICSEK) return HOT_NONE;  // generic fused kernel only
  for (int c = 0; c < P.npair; c++)
    if (P.pair[c].phase_in) return HOT_NONE;
  if (P.cons[0].kind == CONS_PLANE) {
    for (const Replica& R : s->reps_h)
      if (!R.periodic || !(R.cons_p[0] > R.zlo && R.cons_p[0] <= R.zhi)) return HOT_NONE;
    return HOT_PLANE;
  }
  if (P.cons[0].kind == CONS_SPHERE) return HOT_SPHERE;
  return HOT_NONE;
}

static int hot_alloc(sg_system* s, int shape) {
  for (int b = 0; b < 2; b++) {
    if (!s->G[b]) s->G[b] = s->mem.alloc<D4>(s->slots);
    if (shape == HOT_SPHERE && !s->H[b]) s->H[b] = s->mem.alloc<D4>(s->slots);
  }
  if (s->mem.err != cudaSuccess) { s->mem.err = cudaSuccess; return fail(s, SG_ERR_NOMEM, "hot buffers"); }
  return SG_OK;
}

// whole grid, or (flagged = true) the blocks of the replicas being rebuilt
static int hot_pack(sg_system* s, int shape, bool flagged = false) {
  const int ng = flagged ? s->nblist : s->nblocks;
  const int* bl = flagged ? blist_of(s) : nullptr;
  if (ng == 0) return SG_OK;
  if (shape == HOT_PLANE)
    k_hot_pack<HOT_PLANE><<<ng, BLOCK, 0, s->stream>>>(s->reps, s->blk_rep, s->cur, s->st, s->G[s->hot_buf], nullptr, bl);
  else
    k_hot_pack<HOT_SPHERE><<<ng, BLOCK, 0, s->stream>>>(s->reps, s->blk_rep, s->cur, s->st, s->G[s->hot_buf],
                                                        s->H[s->hot_buf], bl);
  LAUNCH_CHECK(s);
  return SG_OK;
}

// whole grid: the run's first start-of-step enforce and the packing in one pass
static int hot_pack_enforce(sg_system* s, int shape) {
  if (s->nblocks == 0) return SG_OK;
  if (shape == HOT_PLANE)
    k_hot_pack_enforce<HOT_PLANE><<<s->nblocks, BLOCK, 0, s->stream>>>(s->reps, s->blk_rep, s->cur, s->st,
                                                                      s->G[s->hot_buf], nullptr,
                                                                      s->prog.cons[0].unlimited);
  else
    k_hot_pack_enforce<HOT_SPHERE><<<s->nblocks, BLOCK, 0, s->stream>>>(s->reps, s->blk_rep, s->cur, s->st,
                                                                       s->G[s->hot_buf], s->H[s->hot_buf],
                                                                       s->prog.cons[0].unlimited);
  LAUNCH_CHECK(s);
  return SG_OK;
}

static int hot_unpack(sg_system* s, int shape, bool flagged = false) {
  const int ng = flagged ? s->nblist : s->nblocks;
  const int* bl = flagged ? blist_of(s) : nullptr;
  if (ng == 0) return SG_OK;
  if (shape == HOT_PLANE)
    k_hot_unpack<HOT_PLANE><<<ng, BLOCK, 0, s->stream>>>(s->reps, s->blk_rep, s->cur, s->G[s->hot_buf], nullptr, bl);
  else
    k_hot_unpack<HOT_SPHERE><<<ng, BLOCK, 0, s->stream>>>(s->reps, s->blk_rep, s->cur, s->G[s->hot_buf],
                                                          s->H[s->hot_buf], bl);
  LAUNCH_CHECK(s);
  return SG_OK;
}

}  // extern "C"

template <int SHAPE>
static void launch_hot(sg_system* s, bool apply_e1, bool last, bool energy) {
  const int b = s->hot_buf;
  D4 *Gi = s->G[b], *Go = s->G[1 - b], *Hi = s->H[b], *Ho = s->H[1 - b];
  if (energy)
    k_hot_step<SHAPE, true><<<s->nblocks, BLOCK, 0, s->stream>>>(
        s->prog, s->reps, s->blk_rep, s->clk, Gi, Go, Hi, Ho, s->cur, s->st, s->nl, s->rebuild, s->status,
        s->dt_global, apply_e1 ? 1 : 0, last ? 1 : 0, s->epart, s->nblocks);
  else
    k_hot_step<SHAPE, false><<<s->nblocks, BLOCK, 0, s->stream>>>(
        s->prog, s->reps, s->blk_rep, s->clk, Gi, Go, Hi, Ho, s->cur, s->st, s->nl, s->rebuild, s->status,
        s->dt_global, apply_e1 ? 1 : 0, last ? 1 : 0, s->epart, s->nblocks);
}

extern "C" {

// The specialised active-Brownian program: single type, soft (+ polar or
// nematic) (+ self_propulsion), one brownian integrator.
static bool abp_program(const sg_system* s) {
  const Program& P = s->prog;
  if (P.ntypes != 1 || P.npair != 1 || P.pair[0].kind != PAIR_SOFT || P.pair[0].phase_in) return false;
  if (P.nalign > 1 || (P.nalign == 1 && P.align[0].kind == ALIGN_VICSEK)) return false;
  if (P.next > 1 || P.ninteg != 1 || P.integ[0].kind != INT_BROWNIAN) return false;
  return true;
}

static int abp_upload(sg_system* s) {
  const Program& P = s->prog;
  std::vector<AbpParams> h(s->nrep);
  for (int r = 0; r < s->nrep; r++) {
    const Replica& R = s->reps_h[r];
    AbpParams& A = h[r];
    std::memset(&A, 0, sizeof(A));
    A.xlo = R.xlo; A.xhi = R.xhi; A.ylo = R.ylo; A.yhi = R.yhi; A.zlo = R.zlo; A.zhi = R.zhi;
    A.Lx = R.Lx; A.Ly = R.Ly; A.Lz = R.Lz;
    A.pad2q = 0.25 * R.pad * R.pad;
    A.k = s->pair_tab_h[0][0];
    A.a = s->pair_tab_h[0][1];
    if (P.nalign == 1) {
      double J, rc;
      if (P.align[0].has_pp) { J = s->align_tab_h[0][0]; rc = s->align_tab_h[0][1]; }
      else { J = R.align_J[0]; rc = R.align_rcut[0]; if (P.align[0].kind == ALIGN_NEMATIC) J = 2.0 * J; }
      A.J = J; A.rc2 = rc * rc;
    }
    if (P.next == 1) A.alpha = P.ext[0].has_params ? s->ext_tab_h[0][0] : R.ext_alpha[0];
    const double* ip = R.integ_p[0];
    A.dt = ip[0]; A.v0 = ip[1]; A.nu = ip[2]; A.mu = ip[3]; A.mur = ip[4];
    A.stoch = std::sqrt(ip[2] * ip[0]);
    A.flip = P.integ[0].nematic ? ip[0] / ip[7] : 0.0;
    A.Rs = R.cons_p[0];
    A.temp = P.integ[0].temp;
    A.off = R.off; A.n = R.n; A.periodic = R.periodic; A.use_radii = P.pair[0].use_radii;
    A.nematic = P.integ[0].nematic; A.velocity = P.integ[0].velocity;
    A.seed = R.seed[0];
  }
  if (!s->abp) s->abp = s->mem.alloc<AbpParams>(s->nrep);
  if (!s->abp) { s->mem.err = cudaSuccess; return fail(s, SG_ERR_NOMEM, "abp params"); }
  CU(s, cudaMemcpyAsync(s->abp, h.data(), sizeof(AbpParams) * s->nrep, cudaMemcpyHostToDevice, s->stream));
  s->abp0_h = h[0];
  return SG_OK;
}

}  // extern "C"

template <int SHAPE, int ALIGN, bool SP, bool ENERGY, int VAR>
static void launch_abp_v(sg_system* s, bool apply_e1, bool last) {
  const int b = s->hot_buf;
  k_abp_step<SHAPE, ALIGN, SP, ENERGY, VAR><<<s->nblocks, BLOCK, 0, s->stream>>>(
      s->abp, s->blk_rep, s->clk, s->G[b], s->G[1 - b], s->H[b], s->H[1 - b], s->cur, s->st, s->nl, s->rebuild,
      s->status, apply_e1 ? 1 : 0, last ? 1 : 0, s->epart, s->nblocks, s->lane_order, s->abp0_h);
}

// cudaFuncSetAttribute is per device: remember, per kernel, the devices it
// has been raised on.
template <typename K>
static void raise_smem(K kernel, size_t smem, unsigned* done_mask, int device) {
  const unsigned bit = 1u << (device & 31);
  if (!(*done_mask & bit)) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    *done_mask |= bit;
  }
}

template <int SHAPE, int ALIGN, bool SP, bool ENERGY>
static void launch_abp_flat(sg_system* s, bool apply_e1, bool last) {
  const int b = s->hot_buf;
  constexpr size_t smem = flat_smem_bytes<SHAPE, ENERGY>();
  static unsigned done = 0;
  raise_smem(k_abp_flat<SHAPE, ALIGN, SP, ENERGY>, smem, &done, s->device);
  k_abp_flat<SHAPE, ALIGN, SP, ENERGY><<<s->nblocks, BLOCK, smem, s->stream>>>(
      s->abp, s->blk_rep, s->clk, s->G[b], s->G[1 - b], s->H[b], s->H[1 - b], s->cur, s->st, s->nl, s->rebuild,
      s->status, apply_e1 ? 1 : 0, last ? 1 : 0, s->epart, s->nblocks);
}

template <int SHAPE, int ALIGN, bool SP, bool ENERGY, int CH, int MINB>
static void launch_abp_staged(sg_system* s, bool apply_e1, bool last) {
  const int b = s->hot_buf;
  constexpr size_t smem = staged_smem_bytes<SHAPE, ALIGN, CH>();
  static unsigned done = 0;
  raise_smem(k_abp_staged<SHAPE, ALIGN, SP, ENERGY, CH, MINB>, smem, &done, s->device);
  k_abp_staged<SHAPE, ALIGN, SP, ENERGY, CH, MINB><<<s->nblocks, BLOCK, smem, s->stream>>>(
      s->abp, s->blk_rep, s->clk, s->G[b], s->G[1 - b], s->H[b], s->H[1 - b], s->cur, s->st, s->nl, s->rebuild,
      s->status, apply_e1 ? 1 : 0, last ? 1 : 0, s->epart, s->nblocks);
}

// (Re)derive the tile data from the current lists (after any list build).
static int tile_prep(sg_system* s) {
  DevBuf& m = s->mem;
  if (!s->tile_n) {
    s->tile_n = m.alloc<int>(s->nblocks);
    s->tile_slot = m.alloc<int>((size_t)s->nblocks * TILE_MAX);
  }
  if (s->nbpos_cap < s->nl.cap) {
    m.release(s->nbpos);
    s->nbpos = m.alloc<uint16_t>((size_t)s->nl.cap * s->nl.stride);
    s->nbpos_cap = s->nl.cap;
  }
  if (m.err != cudaSuccess) { m.err = cudaSuccess; return fail(s, SG_ERR_NOMEM, "tile buffers"); }
  k_tile_prep<<<s->nblocks, BLOCK, 0, s->stream>>>(s->reps, s->blk_rep, s->nl, s->tile_n, s->tile_slot, s->nbpos);
  LAUNCH_CHECK(s);
  s->tile_valid = true;
  return SG_OK;
}

template <int SHAPE, int ALIGN, bool SP, bool ENERGY, int MINB>
static void launch_abp_tile(sg_system* s, bool apply_e1, bool last) {
  const int b = s->hot_buf;  // tile data prepared by step_hot
  constexpr size_t smem = tile_smem_bytes<SHAPE, ALIGN>();
  static unsigned done = 0;
  raise_smem(k_abp_tile<SHAPE, ALIGN, SP, ENERGY, MINB>, smem, &done, s->device);
  k_abp_tile<SHAPE, ALIGN, SP, ENERGY, MINB><<<s->nblocks, BLOCK, smem, s->stream>>>(
      s->abp, s->blk_rep, s->clk, s->G[b], s->G[1 - b], s->H[b], s->H[1 - b], s->cur, s->st, s->nl, s->rebuild,
      s->status, apply_e1 ? 1 : 0, last ? 1 : 0, s->epart, s->nblocks, s->tile_n, s->tile_slot, s->nbpos);
}

template <int SHAPE, int ALIGN, bool SP>
static void launch_abp3(sg_system* s, bool apply_e1, bool last, bool energy) {
  // energy-reporting steps: the pipelined kernel (by value for one replica)
  if (energy) {
    if (s->nrep > 1) launch_abp_v<SHAPE, ALIGN, SP, true, 17>(s, apply_e1, last);
    else launch_abp_v<SHAPE, ALIGN, SP, true, 22>(s, apply_e1, last);
    return;
  }
  // by-value variants carry one replica's parameters: several replicas take the twin
  switch (s->nrep > 1 ? abp_twin(s->abp_variant) : s->abp_variant) {
    case 5: launch_abp_flat<SHAPE, ALIGN, SP, false>(s, apply_e1, last); break;
    case 6: launch_abp_staged<SHAPE, ALIGN, SP, false, 4, 4>(s, apply_e1, last); break;
    case 7: launch_abp_staged<SHAPE, ALIGN, SP, false, 4, 5>(s, apply_e1, last); break;
    case 8: launch_abp_tile<SHAPE, ALIGN, SP, false, 5>(s, apply_e1, last); break;
    case 9: launch_abp_v<SHAPE, ALIGN, SP, false, 9>(s, apply_e1, last); break;
    case 10: launch_abp_v<SHAPE, ALIGN, SP, false, 10>(s, apply_e1, last); break;
    case 11: launch_abp_v<SHAPE, ALIGN, SP, false, 11>(s, apply_e1, last); break;
    case 12: launch_abp_v<SHAPE, ALIGN, SP, false, 12>(s, apply_e1, last); break;
    case 13: launch_abp_v<SHAPE, ALIGN, SP, false, 13>(s, apply_e1, last); break;
    case 14: launch_abp_v<SHAPE, ALIGN, SP, false, 14>(s, apply_e1, last); break;
    case 15: launch_abp_v<SHAPE, ALIGN, SP, false, 15>(s, apply_e1, last); break;
    case 16: launch_abp_v<SHAPE, ALIGN, SP, false, 16>(s, apply_e1, last); break;
    case 17: launch_abp_v<SHAPE, ALIGN, SP, false, 17>(s, apply_e1, last); break;
    case 18: launch_abp_v<SHAPE, ALIGN, SP, false, 18>(s, apply_e1, last); break;
    case 19: launch_abp_v<SHAPE, ALIGN, SP, false, 19>(s, apply_e1, last); break;
    case 20: launch_abp_v<SHAPE, ALIGN, SP, false, 20>(s, apply_e1, last); break;
    case 21: launch_abp_v<SHAPE, ALIGN, SP, false, 21>(s, apply_e1, last); break;
    case 22: launch_abp_v<SHAPE, ALIGN, SP, false, 22>(s, apply_e1, last); break;
    case 23: launch_abp_v<SHAPE, ALIGN, SP, false, 23>(s, apply_e1, last); break;
    case 24: launch_abp_v<SHAPE, ALIGN, SP, false, 24>(s, apply_e1, last); break;
    case 25: launch_abp_v<SHAPE, ALIGN, SP, false, 25>(s, apply_e1, last); break;
    case 26: launch_abp_v<SHAPE, ALIGN, SP, false, 26>(s, apply_e1, last); break;
    case 27: launch_abp_v<SHAPE, ALIGN, SP, false, 27>(s, apply_e1, last); break;
    case 28: launch_abp_v<SHAPE, ALIGN, SP, false, 28>(s, apply_e1, last); break;
    case 29: launch_abp_v<SHAPE, ALIGN, SP, false, 29>(s, apply_e1, last); break;
    case 30: launch_abp_v<SHAPE, ALIGN, SP, false, 30>(s, apply_e1, last); break;
    case 31: launch_abp_v<SHAPE, ALIGN, SP, false, 31>(s, apply_e1, last); break;
    case 0: launch_abp_v<SHAPE, ALIGN, SP, false, 0>(s, apply_e1, last); break;
    case 1: launch_abp_v<SHAPE, ALIGN, SP, false, 1>(s, apply_e1, last); break;
    case 2: launch_abp_v<SHAPE, ALIGN, SP, false, 2>(s, apply_e1, last); break;
    case 3: launch_abp_v<SHAPE, ALIGN, SP, false, 3>(s, apply_e1, last); break;
    default: launch_abp_v<SHAPE, ALIGN, SP, false, 4>(s, apply_e1, last); break;
  }
}

template <int SHAPE>
static void launch_abp(sg_system* s, bool apply_e1, bool last, bool energy) {
  const Program& P = s->prog;
  const int al = P.nalign == 0 ? ABP_ALIGN_NONE : P.align[0].kind;
  const bool sp = P.next == 1;
  if (al == ABP_ALIGN_NONE) { if (sp) launch_abp3<SHAPE, ABP_ALIGN_NONE, true>(s, apply_e1, last, energy);
                              else launch_abp3<SHAPE, ABP_ALIGN_NONE, false>(s, apply_e1, last, energy); }
  else if (al == ALIGN_POLAR) { if (sp) launch_abp3<SHAPE, ALIGN_POLAR, true>(s, apply_e1, last, energy);
                                else launch_abp3<SHAPE, ALIGN_POLAR, false>(s, apply_e1, last, energy); }
  else { if (sp) launch_abp3<SHAPE, ALIGN_NEMATIC, true>(s, apply_e1, last, energy);
         else launch_abp3<SHAPE, ALIGN_NEMATIC, false>(s, apply_e1, last, energy); }
}

extern "C" {

static constexpr int TUNE_REPS = 3;  // timed steps per candidate (after one untimed)

static int step_hot(sg_system* s, int shape, bool apply_e1, bool last, bool energy) {
  const bool tuning = s->abp_on && !s->tuned && !energy;
  if (tuning) {
    s->abp_variant = ABP_TUNED[(s->tune_trial / (TUNE_REPS + 1)) % ABP_NTUNED];
    CU(s, cudaEventRecord(s->ev_t0, s->stream));
  }
  if (s->abp_on && !energy && s->abp_variant == 8 && !s->tile_valid) {
    int rc = tile_prep(s);
    if (rc) return rc;
  }
  if (s->abp_on && (energy || abp_ordered(s->abp_variant)) && !s->order_valid) {  // energy steps run ordered
    if (!s->lane_order) {
      s->lane_order = s->mem.alloc<uint8_t>((size_t)s->nblocks * BLOCK);
      if (!s->lane_order) { s->mem.err = cudaSuccess; return fail(s, SG_ERR_NOMEM, "lane order"); }
    }
    k_lane_order<<<s->nblocks, BLOCK, 0, s->stream>>>(s->reps, s->blk_rep, s->nl, s->lane_order);
    LAUNCH_CHECK(s);
    s->order_valid = true;
  }
  if (s->profile) CU(s, cudaEventRecord(s->ev_k0, s->stream));
  if (s->abp_on) {
    if (shape == HOT_PLANE) launch_abp<HOT_PLANE>(s, apply_e1, last, energy);
    else launch_abp<HOT_SPHERE>(s, apply_e1, last, energy);
  } else if (shape == HOT_PLANE) launch_hot<HOT_PLANE>(s, apply_e1, last, energy);
  else launch_hot<HOT_SPHERE>(s, apply_e1, last, energy);
  LAUNCH_CHECK(s);
  if (s->profile) CU(s, cudaEventRecord(s->ev_k1, s->stream));
  s->hot_buf = 1 - s->hot_buf;
  if (tuning) {
    CU(s, cudaEventRecord(s->ev_t1, s->stream));
    CU(s, cudaEventSynchronize(s->ev_t1));
    float ms = 0.f;
    CU(s, cudaEventElapsedTime(&ms, s->ev_t0, s->ev_t1));
    const int v = s->abp_variant;
    if (s->tune_trial % (TUNE_REPS + 1) != 0) { s->tune_ms[v] += ms; s->tune_n[v]++; }
    s->tune_trial++;
    if (s->tune_trial >= ABP_NTUNED * (TUNE_REPS + 1)) {
      int best = ABP_TUNED[0];
      for (int i = 1; i < ABP_NTUNED; i++) {
        const int c = ABP_TUNED[i];
        if (s->tune_ms[c] / s->tune_n[c] < s->tune_ms[best] / s->tune_n[best]) best = c;
      }
      s->abp_variant = best;
      s->tuned = true;
    }
  }
  return SG_OK;
}

// Rebuild the lists of the replicas flagged in s->rebuild_h (already read
// back), keeping the packed records in step (mid-run: unpack / re-pack the
// rebuilt replicas around the build).
// Adds the device time of the last rebuild to *rebuild_ms (its end event has
// normally run by the time this is called, so no wait).
static int flush_rebuild_time(sg_system* s, double* rebuild_ms) {
  if (!s->b_pending) return SG_OK;
  s->b_pending = false;
  CU(s, cudaEventSynchronize(s->ev_b1));
  float bms = 0.f;
  CU(s, cudaEventElapsedTime(&bms, s->ev_b0, s->ev_b1));
  *rebuild_ms += bms;
  return SG_OK;
}

static int rebuild_pending(sg_system* s, int shape, bool last, double* rebuild_ms) {
  bool any = false;
  for (int r = 0; r < s->nrep; r++) any = any || s->rebuild_h[r];
  if (!any) return SG_OK;
  s->last_gap = std::max<int64_t>(1, s->since_rebuild);
  s->since_rebuild = 0;
  int rc;
  if ((rc = flush_rebuild_time(s, rebuild_ms))) return rc;
  CU(s, cudaEventRecord(s->ev_b0, s->stream));
  if ((rc = prepare_blist(s))) return rc;
  if (shape != HOT_NONE && !last && (rc = hot_unpack(s, shape, true))) return rc;
  bool sorted = false;
  if ((rc = rebuild_flagged(s, &sorted, true))) return rc;
  if (shape != HOT_NONE && !last && sorted && (rc = hot_pack(s, shape, true))) return rc;
  CU(s, cudaMemsetAsync(s->rebuild, 0, sizeof(int) * s->nrep, s->stream));
  CU(s, cudaEventRecord(s->ev_b1, s->stream));
  s->b_pending = true;  // read once the stream has passed it (next rebuild or run end)
  return SG_OK;
}

// K non-final steps on the packed path, enqueued without waiting (the caller
// keeps K at or below half the last gap between rebuilds, since a longer
// batch would mostly enqueue halted launches, and steps one at a time when
// that is 1): each
// step kernel returns at once when an earlier step of the batch flagged a
// rebuild (Clock::halt, set by k_tail_batch), so the host learns after the
// batch how many steps ran, puts the double-buffer index right, rebuilds and
// goes on from there.  Results are those of stepping one at a time.
static constexpr int64_t kBatch = 32;

static int run_batch(sg_system* s, int shape, int64_t K, bool needs_nl, int64_t* executed, double* rebuild_ms) {
  const int b0 = s->hot_buf;
  CU(s, cudaMemsetAsync(s->exec_cnt, 0, sizeof(int), s->stream));
  for (int64_t i = 0; i < K; i++) {
    int rc = step_hot(s, shape, true, false, false);
    if (rc) return rc;
    k_tail_batch<<<1, 256, 0, s->stream>>>(s->prog, s->reps, s->clk, s->nrep, s->rebuild, s->exec_cnt);
    LAUNCH_CHECK(s);
  }
  int ex = 0;
  CU(s, cudaMemcpyAsync(&ex, s->exec_cnt, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  if (needs_nl)
    CU(s, cudaMemcpyAsync(s->rebuild_h, s->rebuild, sizeof(int) * s->nrep, cudaMemcpyDeviceToHost, s->stream));
  CU(s, cudaStreamSynchronize(s->stream));
  if (ex < 1 || ex > K) return fail(s, SG_ERR_CUDA, "batched stepping: inconsistent step count");
  s->hot_buf = b0 ^ (int)(ex & 1);
  s->e1_applied = true;
  *executed = ex;
  s->since_rebuild += ex;
  if (!needs_nl) return SG_OK;
  bool any = false;
  for (int r = 0; r < s->nrep; r++) any = any || s->rebuild_h[r];
  if (!any) return SG_OK;
  k_set_halt<<<(s->nrep + 127) / 128, 128, 0, s->stream>>>(s->clk, s->nrep, 0);
  LAUNCH_CHECK(s);
  return rebuild_pending(s, shape, false, rebuild_ms);
}

// The generic fused step (k_step_brownian), K steps enqueued without a host
// round trip like run_batch: the halted steps' kernels return at once and
// write nothing, so the buffer holding the state is the one after the
// executed steps' swaps; the host swapped once per enqueued step and undoes
// the swaps of the halted ones.
static int run_batch_generic(sg_system* s, int64_t K, bool needs_nl, int64_t* executed, double* rebuild_ms) {
  CU(s, cudaMemsetAsync(s->exec_cnt, 0, sizeof(int), s->stream));
  if (!s->e1_applied) {  // the first step's start-of-step enforce (samos.cpp:887-888)
    k_enforce<<<s->nblocks, BLOCK, 0, s->stream>>>(s->prog, s->reps, s->blk_rep, s->cur, s->st, nullptr);
    LAUNCH_CHECK(s);
  }
  for (int64_t i = 0; i < K; i++) {
    int rc = step_fused(s, true, false);
    if (rc) return rc;
    k_tail_batch<<<1, 256, 0, s->stream>>>(s->prog, s->reps, s->clk, s->nrep, s->rebuild, s->exec_cnt);
    LAUNCH_CHECK(s);
  }
  int ex = 0;
  CU(s, cudaMemcpyAsync(&ex, s->exec_cnt, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  if (needs_nl)
    CU(s, cudaMemcpyAsync(s->rebuild_h, s->rebuild, sizeof(int) * s->nrep, cudaMemcpyDeviceToHost, s->stream));
  CU(s, cudaStreamSynchronize(s->stream));
  if (ex < 1 || ex > K) return fail(s, SG_ERR_CUDA, "batched stepping: inconsistent step count");
  if ((K - ex) & 1) std::swap(s->cur, s->alt);
  s->e1_applied = true;
  *executed = ex;
  s->since_rebuild += ex;
  if (!needs_nl) return SG_OK;
  bool any = false;
  for (int r = 0; r < s->nrep; r++) any = any || s->rebuild_h[r];
  if (!any) return SG_OK;
  k_set_halt<<<(s->nrep + 127) / 128, 128, 0, s->stream>>>(s->clk, s->nrep, 0);
  LAUNCH_CHECK(s);
  return rebuild_pending(s, HOT_NONE, false, rebuild_ms);
}

// Langevin / NVE steps with reusable forces, K enqueued without a host round
// trip like run_batch: after the first step (which may recompute the forces
// and enforce on its own, and is never halted) a step is the two integrator
// halves around one force pass, each returning at once while a rebuild is
// pending; the steps run in place, so nothing is left to fix afterwards.
static int run_batch_unfused(sg_system* s, int64_t K, bool needs_nl, int64_t* executed, double* rebuild_ms) {
  CU(s, cudaMemsetAsync(s->exec_cnt, 0, sizeof(int), s->stream));
  for (int64_t i = 0; i < K; i++) {
    int rc = step_unfused(s, false, false);
    if (rc) return rc;
    k_tail_batch<<<1, 256, 0, s->stream>>>(s->prog, s->reps, s->clk, s->nrep, s->rebuild, s->exec_cnt);
    LAUNCH_CHECK(s);
  }
  int ex = 0;
  CU(s, cudaMemcpyAsync(&ex, s->exec_cnt, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  if (needs_nl)
    CU(s, cudaMemcpyAsync(s->rebuild_h, s->rebuild, sizeof(int) * s->nrep, cudaMemcpyDeviceToHost, s->stream));
  CU(s, cudaStreamSynchronize(s->stream));
  if (ex < 1 || ex > K) return fail(s, SG_ERR_CUDA, "batched stepping: inconsistent step count");
  s->e1_applied = false;
  *executed = ex;
  s->since_rebuild += ex;
  if (!needs_nl) return SG_OK;
  bool any = false;
  for (int r = 0; r < s->nrep; r++) any = any || s->rebuild_h[r];
  if (!any) return SG_OK;
  k_set_halt<<<(s->nrep + 127) / 128, 128, 0, s->stream>>>(s->clk, s->nrep, 0);
  LAUNCH_CHECK(s);
  return rebuild_pending(s, HOT_NONE, false, rebuild_ms);
}

// Blocks of the replicas whose minimiser has not converged (from clk_h).
static int refresh_active(sg_system* s) {
  s->act_h.clear();
  for (int r = 0; r < s->nrep; r++)
    if (s->clk_h[r].fire_conv_step < 0)
      for (int b = 0; b < s->rep_nblk_h[r]; b++) s->act_h.push_back(s->rep_blk0_h[r] + b);
  s->nact = (int)s->act_h.size();
  if (s->nact == s->nblocks || s->nact == 0) return SG_OK;
  if (!s->act) {
    s->act = s->mem.alloc<int>(s->nblocks);
    if (!s->act) { s->mem.err = cudaSuccess; return fail(s, SG_ERR_NOMEM, "active block list"); }
  }
  CU(s, cudaMemcpyAsync(s->act, s->act_h.data(), sizeof(int) * s->nact, cudaMemcpyHostToDevice, s->stream));
  return SG_OK;
}

// The minimiser's iterations, K at a time with no host round trip between
// them (same halt mechanism as run_batch: an iteration whose skin test flags a
// rebuild halts the ones enqueued after it).  Afterwards the host rebuilds if
// needed and polls convergence; *all_done reports that every replica has
// converged.
static int run_fire_batch(sg_system* s, int64_t K, bool needs_nl, int64_t* executed, double* rebuild_ms,
                          bool* all_done) {
  CU(s, cudaMemsetAsync(s->exec_cnt, 0, sizeof(int), s->stream));
  for (int64_t i = 0; i < K; i++) {
    int rc = step_unfused(s, false, true);
    if (rc) return rc;
    k_tail_batch<<<1, 256, 0, s->stream>>>(s->prog, s->reps, s->clk, s->nrep, s->rebuild, s->exec_cnt);
    LAUNCH_CHECK(s);
  }
  int ex = 0;
  CU(s, cudaMemcpyAsync(&ex, s->exec_cnt, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  if (needs_nl)
    CU(s, cudaMemcpyAsync(s->rebuild_h, s->rebuild, sizeof(int) * s->nrep, cudaMemcpyDeviceToHost, s->stream));
  CU(s, cudaStreamSynchronize(s->stream));
  if (ex < 1 || ex > K) return fail(s, SG_ERR_CUDA, "batched iterations: inconsistent step count");
  *executed = ex;
  s->since_rebuild += ex;
  s->e1_applied = false;
  int rc;
  if (needs_nl) {
    bool any = false;
    for (int r = 0; r < s->nrep; r++) any = any || s->rebuild_h[r];
    if (any) {
      k_set_halt<<<(s->nrep + 127) / 128, 128, 0, s->stream>>>(s->clk, s->nrep, 0);
      LAUNCH_CHECK(s);
      if ((rc = rebuild_pending(s, HOT_NONE, false, rebuild_ms))) return rc;
    }
  }
  if ((rc = pull_clk(s))) return rc;
  bool all = true;
  for (int r = 0; r < s->nrep; r++) all = all && s->clk_h[r].fire_conv_step >= 0;
  *all_done = all;
  return all ? SG_OK : refresh_active(s);
}

static int run_impl(sg_system* s, int64_t steps, sg_run_stats* stats, bool driver, int64_t* conv_out,
                    bool cont = false) {
  if (!s || steps < 0) return SG_ERR_ARG;
  if (s->prog.ninteg == 0) return fail(s, SG_ERR_STATE, "Integrator has not been defined");
  if (s->prog.ncons == 0) return fail(s, SG_ERR_STATE, "Constraint has not been defined");
  // Every integrator has its own step (checked when it is added); the global
  // one defaults to 0 as in System (system.cpp:71) and is read only by the
  // phase-in factor, age / dt (pair_soft_potential.cpp:60-76): refuse that
  // division by a zero step, which the reference leaves undefined.
  for (int c = 0; c < s->prog.npair; c++)
    if (s->prog.pair[c].phase_in && !(s->dt_global > 0.0))
      return fail(s, SG_ERR_STATE, "timestep has not been set (phase_in divides the age by it)");
  const bool needs_nl = (s->prog.npair + s->prog.nalign) > 0;
  if (needs_nl && !s->has_nlist) return fail(s, SG_ERR_STATE, "pair terms need a neighbour list");
  if (!s->nl.nb) { int rc = nlist_alloc(s, 1); if (rc) return rc; }
  const bool fused = fused_program(s->prog);
  const int shape = fused ? hot_shape(s) : HOT_NONE;
  s->forces_fresh = false;
  if (shape != HOT_NONE) { int rc = hot_alloc(s, shape); if (rc) return rc; }
  s->abp_on = shape != HOT_NONE && abp_program(s) && s->force_generic == 0;
  if (s->abp_on) { int rc = abp_upload(s); if (rc) return rc; }
  const int64_t launches0 = s->launches, builds0 = s->builds_run;
  double kernel_ms = 0.0, rebuild_ms = 0.0;
  int64_t kernels_timed = 0;
  s->b_pending = false;
  CU(s, cudaEventRecord(s->ev_run0, s->stream));
  CU(s, cudaMemsetAsync(s->status, 0, sizeof(int), s->stream));
  // run-step counters restart with every `run` (samos.cpp:881); a
  // continued segment keeps counting
  if (!cont) {
    int rc = pull_clk(s);
    if (rc) return rc;
    for (int r = 0; r < s->nrep; r++) { s->clk_h[r].run_step = 0; s->clk_h[r].halt = 0; }
    if ((rc = push_clk(s))) return rc;
  }
  // constraint rescaling acts at the top of a step, before its enforce
  // (samos.cpp:882-888): such runs go one step at a time, e1 never pre-applied
  const bool resc = rescaling(s);
  if (resc && s->prog.ncons != 1)
    return fail(s, SG_ERR_UNSUPPORTED, "constraint rescale needs a single constraint on the GPU path");
  int64_t step0 = 0;
  if (resc) {
    int rcp = pull_clk(s);
    if (rcp) return rcp;
    step0 = s->clk_h[0].time_step;
  }
  int64_t done = 0;
  for (int64_t t = 0; t <= steps; t++) {
    const bool last = (t == steps);
    int rc;
    if (resc && s->rescaled_at == step0 + t) {
      s->rescaled_at = -1;  // applied by sg_begin_step before this segment
    } else if (resc) {
      bool scaled = false;
      if ((rc = apply_rescale(s, step0 + t, &scaled))) return rc;
      if (scaled && needs_nl) {  // nlist->build() after a rescale
        for (int r = 0; r < s->nrep; r++) s->rebuild_h[r] = 1;
        if ((rc = rebuild_pending(s, shape, false, &rebuild_ms))) return rc;
      }
    }
    // batched stepping: steps enqueued kBatch at a time with no host round
    // trip, the first step that flags a rebuild halting the rest (same bits)
    const int64_t K = std::min<int64_t>(needs_nl ? std::min<int64_t>(kBatch, s->last_gap / 2) : kBatch, steps - t);
    if (driver && t > 0 && !last && K > 1 && !s->profile && !resc) {
      int64_t ex = 0;
      bool all = false;
      if ((rc = run_fire_batch(s, std::min<int64_t>(K, 16), needs_nl, &ex, &rebuild_ms, &all))) return rc;
      done += ex;
      t += ex - 1;
      if (all) break;
      continue;
    }
    if (shape != HOT_NONE && t > 0 && !last && K > 1 && !driver && !s->profile && (!s->abp_on || s->tuned)) {
      int64_t ex = 0;
      if ((rc = run_batch(s, shape, K, needs_nl, &ex, &rebuild_ms))) return rc;
      done += ex;
      t += ex - 1;
      continue;
    }
    if (!fused && !driver && !resc && t > 0 && !last && K > 1 && !s->profile && integ_forces_reusable(s)) {
      int64_t ex = 0;
      if ((rc = run_batch_unfused(s, K, needs_nl, &ex, &rebuild_ms))) return rc;
      done += ex;
      t += ex - 1;
      continue;
    }
    if (shape == HOT_NONE && fused && !resc && t > 0 && !last && K > 1 && !s->profile && (s->gen_tuned || s->gen_pin)) {
      int64_t ex = 0;
      if ((rc = run_batch_generic(s, K, needs_nl, &ex, &rebuild_ms))) return rc;
      done += ex;
      t += ex - 1;
      continue;
    }
    if (shape != HOT_NONE) {
      if (t == 0) {
        if (!s->e1_applied) rc = hot_pack_enforce(s, shape);
        else rc = hot_pack(s, shape);
        if (rc) return rc;
      }
      rc = step_hot(s, shape, !last, last, last);
      s->e1_applied = !last;
    } else if (fused) {
      if (!s->e1_applied) {
        k_enforce<<<s->nblocks, BLOCK, 0, s->stream>>>(s->prog, s->reps, s->blk_rep, s->cur, s->st, nullptr);
        LAUNCH_CHECK(s);
      }
      rc = step_fused(s, !last && !resc, last, true);
      s->e1_applied = !last && !resc;
    } else {
      rc = step_unfused(s, last, driver);
      s->e1_applied = false;
    }
    if (rc) return rc;
    k_tail<<<(s->nrep + 127) / 128, 128, 0, s->stream>>>(s->prog, s->reps, s->clk, s->nrep);
    LAUNCH_CHECK(s);
    done++;
    if (shape != HOT_NONE && last && (rc = hot_unpack(s, shape))) return rc;
    if (s->profile && fused) {
      CU(s, cudaEventSynchronize(s->ev_k1));
      float ms = 0.f;
      CU(s, cudaEventElapsedTime(&ms, s->ev_k0, s->ev_k1));
      kernel_ms += ms;
      kernels_timed++;
    }
    s->since_rebuild++;
    if (needs_nl) {
      CU(s, cudaMemcpyAsync(s->rebuild_h, s->rebuild, sizeof(int) * s->nrep, cudaMemcpyDeviceToHost, s->stream));
      CU(s, cudaStreamSynchronize(s->stream));
      if ((rc = rebuild_pending(s, shape, last, &rebuild_ms))) return rc;
    }
    if (driver && ((t & 15) == 15 || t == steps)) {  // converged replicas are frozen on the device
      if ((rc = pull_clk(s))) return rc;
      bool all = true;
      for (int r = 0; r < s->nrep; r++) all = all && s->clk_h[r].fire_conv_step >= 0;
      if (all) break;
      if ((rc = refresh_active(s))) return rc;
    }
  }
  CU(s, cudaEventRecord(s->ev_run1, s->stream));
  int st = 0;
  CU(s, cudaMemcpyAsync(&st, s->status, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  CU(s, cudaStreamSynchronize(s->stream));
  float run_ms = 0.f;
  CU(s, cudaEventElapsedTime(&run_ms, s->ev_run0, s->ev_run1));
  if (int rcb = flush_rebuild_time(s, &rebuild_ms)) return rcb;
  int rc = pull_clk(s);
  if (rc) return rc;
  if (conv_out)
    for (int r = 0; r < s->nrep; r++) conv_out[r] = s->clk_h[r].fire_conv_step >= 0 ? s->clk_h[r].fire_conv_step + 1 : -1;
  if (stats) {
    stats->steps_done = done;
    stats->nlist_builds = s->builds_run - builds0;
    stats->kernel_launches = s->launches - launches0;
    stats->max_neighbours = s->maxnb_seen;
    stats->status = st;
    stats->device_ms = run_ms;
    stats->step_kernel_ms = kernel_ms;
    stats->step_kernels = kernels_timed;
    stats->rebuild_ms = rebuild_ms;
  }
  if (st & ST_NONFINITE) return fail(s, SG_ERR_NONFINITE, "non-finite particle position detected");
  return SG_OK;
}

int sg_run(sg_system* s, int64_t steps, sg_run_stats* stats) { return run_impl(s, steps, stats, false, nullptr); }

int sg_run_continue(sg_system* s, int64_t steps, sg_run_stats* stats) {
  if (!s || steps < 1) return SG_ERR_ARG;
  return run_impl(s, steps - 1, stats, false, nullptr, true);
}

int sg_minimize(sg_system* s, int64_t max_steps, int64_t* converged, sg_run_stats* stats) {
  if (!s) return SG_ERR_ARG;
  bool has_fire = false;
  for (int c = 0; c < s->prog.ninteg; c++) has_fire = has_fire || s->prog.integ[c].kind == INT_FIRE;
  if (!has_fire) return fail(s, SG_ERR_STATE, "sg_minimize needs a FIRE integrator");
  int rc = pull_clk(s);
  if (rc) return rc;
  for (int r = 0; r < s->nrep; r++) s->clk_h[r].fire_conv_step = -1;
  rc = push_clk(s);
  if (rc) return rc;
  s->nact = s->nblocks;
  return run_impl(s, max_steps, stats, true, converged);
}

int sg_get_view(sg_system* s, sg_view* v) {
  if (!s || !v) return SG_ERR_ARG;
  if (!s->nl.nb) { int rc = nlist_alloc(s, 1); if (rc) return rc; }
  v->x_device = s->cur.x; v->y_device = s->cur.y; v->z_device = s->cur.z;
  v->nx_device = s->cur.nx; v->ny_device = s->cur.ny; v->nz_device = s->cur.nz;
  v->vx_device = s->cur.vx; v->vy_device = s->cur.vy; v->vz_device = s->cur.vz;
  v->fx_device = s->cur.fx; v->fy_device = s->cur.fy; v->fz_device = s->cur.fz;
  v->radius_device = s->st.r;
  v->id_device = s->st.id; v->nb_device = s->nl.nb; v->nb_cnt_device = s->nl.cnt;
  v->ix_device = s->cur.ix; v->iy_device = s->cur.iy;
  v->nb_stride = s->nl.stride; v->slots = s->slots;
  CU(s, cudaStreamSynchronize(s->stream));
  return SG_OK;
}

int sg_replica_slots(const sg_system* s, int replica, int32_t* offset, int32_t* n) {
  if (!s || replica < 0 || replica >= s->nrep || !offset || !n) return SG_ERR_ARG;
  *offset = s->off[replica];
  *n = s->n[replica];
  return SG_OK;
}

int sg_host_alloc(int64_t bytes, void** ptr) {
  if (!ptr || bytes < 0) return SG_ERR_ARG;
  *ptr = nullptr;
  if (bytes == 0) return SG_OK;
  if (cudaMallocHost(ptr, (size_t)bytes) != cudaSuccess) {
    cudaGetLastError();
    *ptr = nullptr;
    return SG_ERR_NOMEM;
  }
  return SG_OK;
}

int sg_host_free(void* ptr) {
  if (!ptr) return SG_OK;
  return cudaFreeHost(ptr) == cudaSuccess ? SG_OK : SG_ERR_CUDA;
}

int sg_memcpy(void* dst, const void* src, int64_t bytes) {
  if (bytes < 0 || (!dst && bytes) || (!src && bytes)) return SG_ERR_ARG;
  return cudaMemcpy(dst, src, (size_t)bytes, cudaMemcpyDefault) == cudaSuccess ? SG_OK : SG_ERR_CUDA;
}

int sg_positions_changed(sg_system* s) {
  if (!s) return SG_ERR_ARG;
  CU(s, cudaDeviceSynchronize());
  s->e1_applied = false;
  s->forces_fresh = false;
  return s->has_nlist ? sg_build_nlist(s) : SG_OK;
}

int sg_set_variant(sg_system* s, int variant) {
  if (!s || variant < -1 || variant >= ABP_NVARIANT) return SG_ERR_ARG;
  if (variant < 0) {  // re-tune on the next run
    s->tuned = false; s->tune_trial = 0;
    for (int v = 0; v < ABP_NVARIANT; v++) { s->tune_ms[v] = 0.0; s->tune_n[v] = 0; }
    return SG_OK;
  }
  s->abp_variant = variant;
  s->tuned = true;
  return SG_OK;
}

int sg_get_variant(const sg_system* s) { return s ? (s->tuned ? s->abp_variant : -1) : SG_ERR_ARG; }

int sg_set_generic_occupancy(sg_system* s, int blocks_per_sm) {
  if (!s || !(blocks_per_sm == 0 || blocks_per_sm == 6 || blocks_per_sm == 8)) return SG_ERR_ARG;
  s->gen_pin = blocks_per_sm;
  if (blocks_per_sm == 0) {  // re-tune on the next run
    s->gen_tuned = false; s->gen_trial = 0;
    s->gen_ms[0] = s->gen_ms[1] = 0.0; s->gen_n[0] = s->gen_n[1] = 0;
  }
  return SG_OK;
}

int sg_get_generic_occupancy(const sg_system* s) {
  if (!s) return SG_ERR_ARG;
  if (s->gen_pin) return s->gen_pin;
  return s->gen_tuned ? s->gen_minb : 0;
}

int sg_set_fire_order(sg_system* s, int ordered) {
  if (!s || ordered < 0 || ordered > 1) return SG_ERR_ARG;
  s->fire_ordered = ordered;
  return SG_OK;
}

int sg_set_build(sg_system* s, int mode) {
  if (!s || mode < 0 || mode > 3) return SG_ERR_ARG;
  s->build_mode = mode;
  return SG_OK;
}

int sg_set_path(sg_system* s, int path) {
  if (!s || path < 0 || path > 2) return SG_ERR_ARG;
  s->force_generic = path;
  return SG_OK;
}

int sg_set_profiling(sg_system* s, int on) {
  if (!s) return SG_ERR_ARG;
  s->profile = on ? 1 : 0;
  return SG_OK;
}

int sg_energy(sg_system* s, int replica, int cls, int comp, double* out) {
  if (!s || !out || replica < 0 || replica >= s->nrep || cls < 0 || cls > 1) return fail(s, SG_ERR_ARG, "sg_energy: bad argument");
  if ((cls == 0 && comp >= s->prog.npair) || (cls == 1 && comp >= s->prog.nalign) || comp < 0)
    return fail(s, SG_ERR_ARG, "sg_energy: no such component");
  const int row = cls == 0 ? comp : MAX_PAIR + comp;
  const int b0 = s->rep_blk0_h[replica], nb = s->rep_nblk_h[replica];
  std::vector<double> h(nb);
  CU(s, cudaMemcpyAsync(h.data(), s->epart + (size_t)row * s->nblocks + b0, sizeof(double) * nb, cudaMemcpyDeviceToHost,
                        s->stream));
  CU(s, cudaStreamSynchronize(s->stream));
  double e = 0.0;
  for (int b = 0; b < nb; b++) e += h[b];
  *out = e;
  return SG_OK;
}

int sg_fire_state(sg_system* s, int replica, double* out5) {
  if (!s || !out5 || replica < 0 || replica >= s->nrep) return SG_ERR_ARG;
  int rc = pull_clk(s);
  if (rc) return rc;
  const Clock& C = s->clk_h[replica];
  out5[0] = C.fire_dt; out5[1] = C.fire_alpha; out5[2] = C.fire_last_neg;
  out5[3] = C.fire_converged; out5[4] = C.fire_old_e;
  return SG_OK;
}

}  // extern "C"
