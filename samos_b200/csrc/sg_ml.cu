// sg_ml.cu -- learned FIRE warm start: a two-layer message-passing network
// over the engine's neighbour lists that predicts each particle's
// displacement to its relaxed position.  No reference counterpart (this is
// the learned part of the project).
//
// Network (width 64, edges with r < rc; e_ij = (r, a_i, a_j, a_i + a_j - r),
// d_ij the minimum-image vector from i to j):
//   s_i  = sum_j relu(W1a e_ij + b1a)                       edge kernel, FP32
//   h_i  = relu(s_i W1b + b1b)                              BF16 tensor cores
//   [P|Q] = h Wpq                                           BF16 tensor cores
//   z_ij = relu(P_i + Q_j + W2e e_ij + b2),  w_ij = z_ij . w2 + c
//   disp_i = sum_j w_ij d_ij / r_ij                         edge kernel, FP32
// The 64-wide products are node-level (the first edge layer is summed before
// W1b, the second is split into P_i + Q_j), so the tensor-core GEMMs are
// [slots x 64] x [64 x 64|128] with FP32 accumulation (k_ml_gemm_tc), and the
// weight gradients are reductions over every slot ([64 x slots] x [slots x
// 64|128], k_ml_wgrad_tc); both run on the 5th-generation tensor cores: TMA
// tiles in the 128-byte swizzle, tcgen05.mma with the accumulator in tensor
// memory, tcgen05.ld epilogues.
// Activations s, h and the GEMM operands of the backward pass are BF16.
#include "samos_gpu.h"

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace {

constexpr int F = 64;          // hidden width
constexpr int NP_W1A = 0, NP_B1A = 256, NP_W1B = 320, NP_B1B = 4416, NP_WPQ = 4480, NP_B2 = 12672,
              NP_W2E = 12736, NP_W2 = 12992, NP_C = 13056, NP_TOTAL = 13057;
constexpr int EDGE_WARPS = 8;  // warps per block in the edge kernels
constexpr int EDGE_BLOCKS = 148 * 8;

__device__ __forceinline__ float bf(const __nv_bfloat16 v) { return __bfloat162float(v); }

__device__ __forceinline__ bool edge_vec(const sg_view& V, const double* box, int i, int j, double rc, float* e,
                                         float& ux, float& uy, float ai) {
  const double Lx = box[2 * i], Ly = box[2 * i + 1];
  double dx = V.x_device[j] - V.x_device[i], dy = V.y_device[j] - V.y_device[i];
  if (dx > 0.5 * Lx) dx -= Lx; else if (dx < -0.5 * Lx) dx += Lx;
  if (dy > 0.5 * Ly) dy -= Ly; else if (dy < -0.5 * Ly) dy += Ly;
  const double r = sqrt(dx * dx + dy * dy);
  if (!(r < rc) || r == 0.0) return false;
  const float aj = (float)V.radius_device[j];
  e[0] = (float)r; e[1] = ai; e[2] = aj; e[3] = ai + aj - (float)r;
  ux = (float)(dx / r); uy = (float)(dy / r);
  return true;
}

// ---- layer 1 edges: s_i = sum_j relu(W1a e + b1a), stored BF16 ----------------
__global__ void k_ml_l1(sg_view V, const double* __restrict__ box, double rc, const float* __restrict__ P,
                        __nv_bfloat16* __restrict__ s16) {
  const int lane = threadIdx.x & 31;
  const int nw = gridDim.x * (blockDim.x >> 5);
  float w[2][4], b[2];
  for (int h = 0; h < 2; h++) {
    const int f = lane + 32 * h;
    for (int d = 0; d < 4; d++) w[h][d] = P[NP_W1A + 4 * f + d];
    b[h] = P[NP_B1A + f];
  }
  for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < V.slots; i += nw) {
    float acc[2] = {0.f, 0.f};
    if (box[2 * i] > 0.0) {
      const float ai = (float)V.radius_device[i];
      const int cnt = V.nb_cnt_device[i];
      for (int q = 0; q < cnt; q++) {
        const int j = V.nb_device[(size_t)q * V.nb_stride + i];
        float e[4], ux, uy;
        if (!edge_vec(V, box, i, j, rc, e, ux, uy, ai)) continue;
        for (int h = 0; h < 2; h++) {
          const float z = w[h][0] * e[0] + w[h][1] * e[1] + w[h][2] * e[2] + w[h][3] * e[3] + b[h];
          acc[h] += fmaxf(z, 0.f);
        }
      }
    }
    s16[(size_t)i * F + lane] = __float2bfloat16_rn(acc[0]);
    s16[(size_t)i * F + lane + 32] = __float2bfloat16_rn(acc[1]);
  }
}

// ---- weight gradient on tcgen05: W[k][n] = sum_m X[m][k] G[m][n] ----------------
// The reduction runs over all slots, so it is the MMA's K dimension: per
// 64-row chunk, D[128 x 64] += G_chunk^T (A: M = G's features, zero rows
// above NF) x X_chunk (B: N = X's 64 features), four K = 16 steps.  Both
// operands are the tiles exactly as TMA lands them with the 128-byte swizzle
// (rows of 64 BF16 features = 128 B; "MN-major" in the MMA's terms, 8-row
// groups 1024 B apart).  One CTA per SM owns a contiguous run of chunks and a
// private [64 x NF] FP32 partial (deterministic: chunks in order, partials
// summed in block order by k_ml_reduce).  Thread 0 issues the TMA loads (four
// stages) and the MMAs; tcgen05.commit releases a stage; the accumulator is
// read back with tcgen05.ld by the four warps, one 32-lane quarter each.
// Every mbarrier wait is bounded: on a timeout the kernel records it in
// *err, drains what it issued, frees its tensor memory and returns.
constexpr int WG_STAGES = 4;
constexpr int WG_ROWS = 64;                     // slots per chunk (4 MMA K steps)
constexpr int WG_A_BYTES = 2 * WG_ROWS * 128;   // G^T: two 128-B feature groups
constexpr int WG_B_BYTES = WG_ROWS * 128;       // X: one 128-B feature group
constexpr int WG_STAGE_BYTES = WG_A_BYTES + WG_B_BYTES;
constexpr int WG_SMEM = 1024 + WG_STAGES * WG_STAGE_BYTES + 128;
constexpr uint32_t WG_TMEM_COLS = 64;
__device__ int g_ml_tc_err;  // set by a tcgen05 kernel of this file whose bounded wait ran out
constexpr long long WG_SPIN_LIMIT = 1ll << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
  for (long long it = 0; it < WG_SPIN_LIMIT; it++) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok) : "r"(bar), "r"(phase) : "memory");
    if (ok) return true;
  }
  return false;
}

// shared-memory matrix descriptor of a 128-B-swizzled tile (layout type 2,
// descriptor version 1): start address, leading byte offset (between 64-wide
// feature groups), stride byte offset (between 8-row groups), all >> 4
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46) | (2ull << 61);
}

// instruction descriptor: D FP32, A and B BF16, both MN-major, N = 64, M = 128
constexpr uint32_t WG_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((64u >> 3) << 17) |
                              ((128u >> 4) << 24);

template <int NF>
__global__ void __launch_bounds__(128, 1)
k_ml_wgrad_tc(const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmG, int M,
              int chunks_per_block, float* __restrict__ partial, int* __restrict__ err) {
  static_assert(NF == 64 || NF == 128, "G has 64 or 128 features");
  extern __shared__ uint8_t wg_smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(wg_smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + WG_STAGES * WG_STAGE_BYTES);  // full[S], empty[S], done
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * WG_STAGES + 1);
  __shared__ int abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nchunks = (M + WG_ROWS - 1) / WG_ROWS;
  const int c0 = blockIdx.x * chunks_per_block;
  const int n = max(0, min(nchunks, c0 + chunks_per_block) - c0);

  if (threadIdx.x == 0) {
    abort_flag = 0;
    for (int i = 0; i < 2 * WG_STAGES + 1; i++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bars + i)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (NF == 64) {  // the A tiles' second feature group stays zero (rows 64..127 of D)
    for (int s = 0; s < WG_STAGES; s++)
      for (int i = threadIdx.x; i < WG_ROWS * 128 / 16; i += blockDim.x)
        reinterpret_cast<uint4*>(smem + s * WG_STAGE_BYTES + WG_ROWS * 128)[i] = make_uint4(0u, 0u, 0u, 0u);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                 ::"r"(smem_u32(tmem_slot)), "r"(WG_TMEM_COLS) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + WG_STAGES), done = smem_u32(bars + 2 * WG_STAGES);

  if (threadIdx.x == 0 && n > 0) {
    const uint64_t mapX = reinterpret_cast<uint64_t>(&tmX), mapG = reinterpret_cast<uint64_t>(&tmG);
    constexpr uint32_t tx_bytes = (NF == 128 ? WG_A_BYTES : WG_ROWS * 128) + WG_B_BYTES;
    auto issue = [&](int i) {  // TMA loads of chunk i into stage i % S
      const int s = i % WG_STAGES;
      const uint32_t a = smem_u32(smem + s * WG_STAGE_BYTES), b = a + WG_A_BYTES, bar = full0 + 8 * s;
      const int row = (c0 + i) * WG_ROWS;
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(tx_bytes) : "memory");
      asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
                   ::"r"(a), "l"(mapG), "r"(0), "r"(row), "r"(bar) : "memory");
      if (NF == 128)
        asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
                     ::"r"(a + WG_ROWS * 128), "l"(mapG), "r"(64), "r"(row), "r"(bar) : "memory");
      asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
                   ::"r"(b), "l"(mapX), "r"(0), "r"(row), "r"(bar) : "memory");
    };
    const int pre = min(WG_STAGES, n);
    for (int i = 0; i < pre; i++) issue(i);
    int issued = pre, consumed = 0;
    bool ok = true;
    for (int i = 0; i < n && ok; i++) {
      const int s = i % WG_STAGES;
      const uint32_t phase = (uint32_t)((i / WG_STAGES) & 1);
      if (!mbar_wait(full0 + 8 * s, phase)) { ok = false; break; }
      consumed = i + 1;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const uint32_t a = smem_u32(smem + s * WG_STAGE_BYTES), b = a + WG_A_BYTES;
#pragma unroll
      for (int k = 0; k < WG_ROWS / 16; k++) {  // 16 slots per MMA: two 8-row groups, 2048 B
        const uint64_t da = umma_desc_sw128(a + k * 2048, WG_ROWS * 128, 1024);
        const uint64_t db = umma_desc_sw128(b + k * 2048, WG_ROWS * 128, 1024);
        const uint32_t acc = (i > 0 || k > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
            ::"r"(tmem), "l"(da), "l"(db), "r"(WG_IDESC), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                   ::"r"(empty0 + 8 * s) : "memory");
      if (i + WG_STAGES < n) {  // refill this stage once its MMAs have read it
        if (!mbar_wait(empty0 + 8 * s, phase)) { ok = false; break; }
        issue(i + WG_STAGES);
        issued++;
      }
    }
    if (!ok) {  // timed out: drain the loads still in flight before leaving
      atomicExch(err, 1);
      abort_flag = 1;
      for (int i = consumed; i < issued; i++) mbar_wait(full0 + 8 * (i % WG_STAGES), (uint32_t)((i / WG_STAGES) & 1));
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(done)
                 : "memory");
  }
  __syncthreads();
  bool have = n > 0 && !abort_flag;
  if (n > 0 && !mbar_wait(done, 0)) {  // every MMA of this CTA has completed
    if (lane == 0) atomicExch(err, 1);
    have = false;
  }
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  // D row m (G feature) is TMEM lane m, column j (X feature) is column j
  float* out = partial + (size_t)blockIdx.x * F * NF;
  const int m = warp * 32 + lane;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    uint32_t r[16];
    if (n > 0) {
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(q * 16);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
    }
    if (m < NF)
#pragma unroll
      for (int j = 0; j < 16; j++) out[(size_t)(q * 16 + j) * NF + m] = have ? __uint_as_float(r[j]) : 0.f;
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(WG_TMEM_COLS) : "memory");
}

// 2-D row-major BF16 tensor map [rows x cols] with boxes of 64 columns x
// box_rows rows and the 128-byte swizzle (cuTensorMapEncodeTiled, fetched through the runtime so
// the library does not link the driver library)
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

bool make_bf16_map(CUtensorMap* map, const void* base, int rows, int cols, int box_rows = WG_ROWS) {
  static EncodeTiledFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<EncodeTiledFn>(f);
  }();
  if (!fn || (reinterpret_cast<uintptr_t>(base) & 15) || rows < 1) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
  const cuuint32_t box[2] = {64, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// partial[b] = X^T G over block b's chunks, for X [M x 64], G [M x NF] (BF16)
template <int NF>
int launch_wgrad_tc(const void* X, const void* G, int M, int blocks, float* partial, int* err, cudaStream_t st) {
  CUtensorMap mx, mg;
  if (!make_bf16_map(&mx, X, M, F) || !make_bf16_map(&mg, G, M, NF)) return SG_ERR_CUDA;
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_ml_wgrad_tc<NF>, cudaFuncAttributeMaxDynamicSharedMemorySize, WG_SMEM) != cudaSuccess)
      return SG_ERR_CUDA;
    attr = true;
  }
  const int nchunks = (M + WG_ROWS - 1) / WG_ROWS;
  const int per = (nchunks + blocks - 1) / blocks;
  k_ml_wgrad_tc<NF><<<blocks, 128, WG_SMEM, st>>>(mx, mg, M, per, partial, err);
  return cudaGetLastError() == cudaSuccess ? SG_OK : SG_ERR_CUDA;
}

// ---- activation GEMM on tcgen05: C[m][n] = act(sum_k A[m][k] Bt[n][k] + bias[n]) ------
// One CTA per 128-row tile of A: the tile (K/64 groups of 128 rows x 128 B)
// and all of Bt (K/64 groups of N rows x 128 B) arrive by TMA in the 128-byte
// swizzle, K-major for both operands; one thread issues K/16 tcgen05.mma
// (M = 128, N) into tensor memory; the four warps read their 32 rows back
// with tcgen05.ld and apply bias, relu and the slot mask (box <= 0: padding,
// written as 0) in the epilogue, storing FP32 and / or BF16.  Waits bounded
// as in k_ml_wgrad_tc.
template <int K, int N>
__global__ void __launch_bounds__(128)
k_ml_gemm_tc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int M,
             const float* __restrict__ bias, int relu, const double* __restrict__ box, float* __restrict__ C32,
             __nv_bfloat16* __restrict__ C16, int* __restrict__ err) {
  static_assert((K == 64 || K == 128) && (N == 64 || N == 128), "K, N in {64, 128}");
  constexpr int KG = K / 64;                      // 128-B K groups
  constexpr int A_GROUP = 128 * 128, B_GROUP = N * 128;
  constexpr uint32_t TX = KG * (A_GROUP + B_GROUP);
  constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((128u >> 4) << 24);
  extern __shared__ uint8_t gm_smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(gm_smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* sA = smem;
  uint8_t* sB = smem + KG * A_GROUP;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sB + KG * B_GROUP);  // full, done
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2);
  __shared__ int ok_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row0 = blockIdx.x * 128;
  if (threadIdx.x == 0) {
    ok_flag = 1;
    for (int i = 0; i < 2; i++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bars + i)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                 ::"r"(smem_u32(tmem_slot)), "r"((uint32_t)N) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t full = smem_u32(bars), done = smem_u32(bars + 1);
  if (threadIdx.x == 0) {
    const uint64_t mapA = reinterpret_cast<uint64_t>(&tmA), mapB = reinterpret_cast<uint64_t>(&tmB);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(full), "r"(TX) : "memory");
#pragma unroll
    for (int g = 0; g < KG; g++) {
      asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
                   ::"r"(smem_u32(sA + g * A_GROUP)), "l"(mapA), "r"(g * 64), "r"(row0), "r"(full) : "memory");
      asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
                   ::"r"(smem_u32(sB + g * B_GROUP)), "l"(mapB), "r"(g * 64), "r"(0), "r"(full) : "memory");
    }
    if (mbar_wait(full, 0)) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
#pragma unroll
      for (int ks = 0; ks < K / 16; ks++) {  // K-major: 16 elements = 32 B along each 128-B row
        const int g = ks / 4, off = (ks % 4) * 32;
        const uint64_t da = umma_desc_sw128(smem_u32(sA + g * A_GROUP) + off, 16, 1024);
        const uint64_t db = umma_desc_sw128(smem_u32(sB + g * B_GROUP) + off, 16, 1024);
        const uint32_t acc = ks > 0 ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
            ::"r"(tmem), "l"(da), "l"(db), "r"(IDESC), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u) : "memory");
      }
    } else {
      atomicExch(err, 1);
      ok_flag = 0;
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(done)
                 : "memory");
  }
  __syncthreads();
  bool have = ok_flag != 0;
  if (!mbar_wait(done, 0)) {
    if (lane == 0) atomicExch(err, 1);
    have = false;
  }
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const int row = row0 + warp * 32 + lane;
  const bool inside = row < M;
  const bool valid = inside && box[2 * (size_t)row] > 0.0;
#pragma unroll
  for (int q = 0; q < N / 16; q++) {
    uint32_t r[16];
    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(q * 16);
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
    if (!inside) continue;
    float v[16];
#pragma unroll
    for (int j = 0; j < 16; j++) {
      float t = have ? __uint_as_float(r[j]) : 0.f;
      if (bias) t += bias[q * 16 + j];
      if (relu) t = fmaxf(t, 0.f);
      v[j] = valid ? t : 0.f;
    }
    if (C32) {
      float4* o = reinterpret_cast<float4*>(C32 + (size_t)row * N + q * 16);
#pragma unroll
      for (int j = 0; j < 4; j++) o[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
    }
    if (C16) {
      __align__(16) __nv_bfloat16 h[16];
#pragma unroll
      for (int j = 0; j < 16; j++) h[j] = __float2bfloat16_rn(v[j]);
      uint4* o = reinterpret_cast<uint4*>(C16 + (size_t)row * N + q * 16);
      o[0] = reinterpret_cast<const uint4*>(h)[0];
      o[1] = reinterpret_cast<const uint4*>(h)[1];
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"((uint32_t)N) : "memory");
}

template <int K, int N>
int launch_gemm_tc(const void* A, const void* Bt, int M, const float* bias, int relu, const double* box, float* C32,
                   void* C16, int* err, cudaStream_t st) {
  // at most 512 / N CTAs may share an SM's 512 tensor-memory columns: the
  // shared-memory request is padded so that no more fit (an allocation
  // beyond them would wait for another CTA's release)
  constexpr int NEED = 1024 + (K / 64) * (128 * 128 + N * 128) + 64;
  constexpr int CAP = (N == 128 ? 48 : 26) * 1024;
  constexpr int SMEM = NEED > CAP ? NEED : CAP;
  CUtensorMap ma, mb;
  if (!make_bf16_map(&ma, A, M, K, 128) || !make_bf16_map(&mb, Bt, N, K, N)) return SG_ERR_CUDA;
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_ml_gemm_tc<K, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM) != cudaSuccess)
      return SG_ERR_CUDA;
    attr = true;
  }
  k_ml_gemm_tc<K, N><<<(M + 127) / 128, 128, SMEM, st>>>(ma, mb, M, bias, relu, box, C32, (__nv_bfloat16*)C16, err);
  return cudaGetLastError() == cudaSuccess ? SG_OK : SG_ERR_CUDA;
}

// out[i] += sum_b partial[b][i]   (fixed order)
__global__ void k_ml_reduce(const float* __restrict__ partial, int nblk, int len, float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= len) return;
  float s = 0.f;
  for (int b = 0; b < nblk; b++) s += partial[(size_t)b * len + i];
  out[i] += s;
}

// ---- layer 2 edges (forward): disp_i --------------------------------------------
__global__ void k_ml_l2(sg_view V, const double* __restrict__ box, double rc, const float* __restrict__ P,
                        const float* __restrict__ PQ, float* __restrict__ disp) {
  const int lane = threadIdx.x & 31;
  const int nw = gridDim.x * (blockDim.x >> 5);
  float we[2][4], b2[2], w2[2];
  for (int h = 0; h < 2; h++) {
    const int f = lane + 32 * h;
    for (int d = 0; d < 4; d++) we[h][d] = P[NP_W2E + 4 * f + d];
    b2[h] = P[NP_B2 + f];
    w2[h] = P[NP_W2 + f];
  }
  const float c = P[NP_C];
  for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < V.slots; i += nw) {
    float dx = 0.f, dy = 0.f;
    if (box[2 * i] > 0.0) {
      const float ai = (float)V.radius_device[i];
      const float Pi0 = PQ[(size_t)i * 2 * F + lane], Pi1 = PQ[(size_t)i * 2 * F + lane + 32];
      const int cnt = V.nb_cnt_device[i];
      for (int q = 0; q < cnt; q++) {
        const int j = V.nb_device[(size_t)q * V.nb_stride + i];
        float e[4], ux, uy;
        if (!edge_vec(V, box, i, j, rc, e, ux, uy, ai)) continue;
        const float Qj0 = PQ[(size_t)j * 2 * F + F + lane], Qj1 = PQ[(size_t)j * 2 * F + F + lane + 32];
        const float z0 = Pi0 + Qj0 + we[0][0] * e[0] + we[0][1] * e[1] + we[0][2] * e[2] + we[0][3] * e[3] + b2[0];
        const float z1 = Pi1 + Qj1 + we[1][0] * e[0] + we[1][1] * e[1] + we[1][2] * e[2] + we[1][3] * e[3] + b2[1];
        float part = fmaxf(z0, 0.f) * w2[0] + fmaxf(z1, 0.f) * w2[1];
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        const float w = part + c;
        dx += w * ux; dy += w * uy;
      }
    }
    if (lane == 0) { disp[2 * i] = dx; disp[2 * i + 1] = dy; }
  }
}

// ---- layer 2 edges (backward) -------------------------------------------------
// gPQ must be zero on entry: the P half of row i is written by i's warp, the Q
// half of row j receives atomic contributions from every i that has j as a
// neighbour.  Per-block partials of (gW2e, gb2, gw2, gc) go to part[block].
constexpr int L2_GRAD = 256 + 64 + 64 + 1;  // W2e, b2, w2, c
__global__ void k_ml_l2_bwd(sg_view V, const double* __restrict__ box, double rc, const float* __restrict__ P,
                            const float* __restrict__ PQ, const float* __restrict__ disp,
                            const float* __restrict__ target, float inv_n, float* __restrict__ gPQ,
                            float* __restrict__ part, float* __restrict__ loss_part) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = gridDim.x * (blockDim.x >> 5);
  float we[2][4], b2[2], w2[2];
  for (int h = 0; h < 2; h++) {
    const int f = lane + 32 * h;
    for (int d = 0; d < 4; d++) we[h][d] = P[NP_W2E + 4 * f + d];
    b2[h] = P[NP_B2 + f];
    w2[h] = P[NP_W2 + f];
  }
  float gWe[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}}, gb2[2] = {0.f, 0.f}, gw2[2] = {0.f, 0.f};
  float gc = 0.f, lsum = 0.f;
  for (int i = blockIdx.x * (blockDim.x >> 5) + warp; i < V.slots; i += nw) {
    if (!(box[2 * i] > 0.0)) continue;
    const float ddx = disp[2 * i] - target[2 * i], ddy = disp[2 * i + 1] - target[2 * i + 1];
    if (lane == 0) lsum += ddx * ddx + ddy * ddy;
    const float gdx = 2.f * ddx * inv_n, gdy = 2.f * ddy * inv_n;
    const float ai = (float)V.radius_device[i];
    const float Pi0 = PQ[(size_t)i * 2 * F + lane], Pi1 = PQ[(size_t)i * 2 * F + lane + 32];
    float gP0 = 0.f, gP1 = 0.f;
    const int cnt = V.nb_cnt_device[i];
    for (int q = 0; q < cnt; q++) {
      const int j = V.nb_device[(size_t)q * V.nb_stride + i];
      float e[4], ux, uy;
      if (!edge_vec(V, box, i, j, rc, e, ux, uy, ai)) continue;
      const float Qj0 = PQ[(size_t)j * 2 * F + F + lane], Qj1 = PQ[(size_t)j * 2 * F + F + lane + 32];
      const float z0 = Pi0 + Qj0 + we[0][0] * e[0] + we[0][1] * e[1] + we[0][2] * e[2] + we[0][3] * e[3] + b2[0];
      const float z1 = Pi1 + Qj1 + we[1][0] * e[0] + we[1][1] * e[1] + we[1][2] * e[2] + we[1][3] * e[3] + b2[1];
      const float a0 = fmaxf(z0, 0.f), a1 = fmaxf(z1, 0.f);
      const float gw = gdx * ux + gdy * uy;  // d loss / d w_ij
      gw2[0] += gw * a0; gw2[1] += gw * a1;
      if (lane == 0) gc += gw;
      const float gz0 = z0 > 0.f ? gw * w2[0] : 0.f, gz1 = z1 > 0.f ? gw * w2[1] : 0.f;
      gb2[0] += gz0; gb2[1] += gz1;
      for (int d = 0; d < 4; d++) { gWe[0][d] += gz0 * e[d]; gWe[1][d] += gz1 * e[d]; }
      gP0 += gz0; gP1 += gz1;
      atomicAdd(&gPQ[(size_t)j * 2 * F + F + lane], gz0);
      atomicAdd(&gPQ[(size_t)j * 2 * F + F + lane + 32], gz1);
    }
    gPQ[(size_t)i * 2 * F + lane] = gP0;
    gPQ[(size_t)i * 2 * F + lane + 32] = gP1;
  }
  // block reduction of the weight-gradient partials (fixed order over warps)
  __shared__ float sp[EDGE_WARPS][L2_GRAD];
  for (int h = 0; h < 2; h++) {
    const int f = lane + 32 * h;
    for (int d = 0; d < 4; d++) sp[warp][4 * f + d] = gWe[h][d];
    sp[warp][256 + f] = gb2[h];
    sp[warp][320 + f] = gw2[h];
  }
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if (lane == 0) sp[warp][384] = gc;
  __shared__ float sl[EDGE_WARPS];
  if (lane == 0) sl[warp] = lsum;
  __syncthreads();
  for (int idx = threadIdx.x; idx < L2_GRAD; idx += blockDim.x) {
    float s = 0.f;
    for (int w = 0; w < EDGE_WARPS; w++) s += sp[w][idx];
    part[(size_t)blockIdx.x * L2_GRAD + idx] = s;
  }
  if (threadIdx.x == 0) {
    float s = 0.f;
    for (int w = 0; w < EDGE_WARPS; w++) s += sl[w];
    loss_part[blockIdx.x] = s;
  }
}

// gpre = gh * (h > 0) (BF16) and per-block column partials of gpre (gb1b)
__global__ void k_ml_relu_bwd(int M, const float* __restrict__ gh, const __nv_bfloat16* __restrict__ h16,
                              __nv_bfloat16* __restrict__ gpre16, float* __restrict__ part) {
  const int f = threadIdx.x & 63, rsub = threadIdx.x >> 6;  // 256 threads: 4 rows per pass
  float acc = 0.f;
  const int rows_per_block = (M + gridDim.x - 1) / gridDim.x;
  const int m0 = blockIdx.x * rows_per_block, m1 = min(M, m0 + rows_per_block);
  for (int m = m0 + rsub; m < m1; m += 4) {
    const float g = bf(h16[(size_t)m * F + f]) > 0.f ? gh[(size_t)m * F + f] : 0.f;
    const __nv_bfloat16 gb = __float2bfloat16_rn(g);
    gpre16[(size_t)m * F + f] = gb;
    acc += bf(gb);
  }
  __shared__ float s[4][64];
  s[rsub][f] = acc;
  __syncthreads();
  if (threadIdx.x < 64) part[(size_t)blockIdx.x * 64 + threadIdx.x] = s[0][f] + s[1][f] + s[2][f] + s[3][f];
}

// ---- layer 1 edges (backward): gW1a, gb1a partials ------------------------------
constexpr int L1_GRAD = 256 + 64;
__global__ void k_ml_l1_bwd(sg_view V, const double* __restrict__ box, double rc, const float* __restrict__ P,
                            const float* __restrict__ gs, float* __restrict__ part) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = gridDim.x * (blockDim.x >> 5);
  float w[2][4], b[2];
  for (int h = 0; h < 2; h++) {
    const int f = lane + 32 * h;
    for (int d = 0; d < 4; d++) w[h][d] = P[NP_W1A + 4 * f + d];
    b[h] = P[NP_B1A + f];
  }
  float gW[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}}, gb[2] = {0.f, 0.f};
  for (int i = blockIdx.x * (blockDim.x >> 5) + warp; i < V.slots; i += nw) {
    if (!(box[2 * i] > 0.0)) continue;
    const float ai = (float)V.radius_device[i];
    const float gs0 = gs[(size_t)i * F + lane], gs1 = gs[(size_t)i * F + lane + 32];
    const int cnt = V.nb_cnt_device[i];
    for (int q = 0; q < cnt; q++) {
      const int j = V.nb_device[(size_t)q * V.nb_stride + i];
      float e[4], ux, uy;
      if (!edge_vec(V, box, i, j, rc, e, ux, uy, ai)) continue;
      const float z0 = w[0][0] * e[0] + w[0][1] * e[1] + w[0][2] * e[2] + w[0][3] * e[3] + b[0];
      const float z1 = w[1][0] * e[0] + w[1][1] * e[1] + w[1][2] * e[2] + w[1][3] * e[3] + b[1];
      const float g0 = z0 > 0.f ? gs0 : 0.f, g1 = z1 > 0.f ? gs1 : 0.f;
      gb[0] += g0; gb[1] += g1;
      for (int d = 0; d < 4; d++) { gW[0][d] += g0 * e[d]; gW[1][d] += g1 * e[d]; }
    }
  }
  __shared__ float sp[EDGE_WARPS][L1_GRAD];
  for (int h = 0; h < 2; h++) {
    const int f = lane + 32 * h;
    for (int d = 0; d < 4; d++) sp[warp][4 * f + d] = gW[h][d];
    sp[warp][256 + f] = gb[h];
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < L1_GRAD; idx += blockDim.x) {
    float s = 0.f;
    for (int ww = 0; ww < EDGE_WARPS; ww++) s += sp[ww][idx];
    part[(size_t)blockIdx.x * L1_GRAD + idx] = s;
  }
}

// add the reduced small-gradient vectors into the flat gradient buffer
__global__ void k_ml_place(const float* __restrict__ src, int len, float* __restrict__ dst, int off_d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < len) dst[off_d + i] += src[i];
}

__global__ void k_ml_to_bf16(const float* __restrict__ a, __nv_bfloat16* __restrict__ b, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = __float2bfloat16_rn(a[i]);
}

__global__ void k_ml_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                          float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi; v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// BF16 copies of the GEMM weights: W1b [64x64], W1b^T, Wpq [64x128], Wpq^T
__global__ void k_ml_bf16_weights(const float* __restrict__ p, __nv_bfloat16* W1b, __nv_bfloat16* W1bT,
                                  __nv_bfloat16* Wpq, __nv_bfloat16* WpqT) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < F * F) {
    const int k = i / F, n = i % F;
    const __nv_bfloat16 v = __float2bfloat16_rn(p[NP_W1B + i]);
    W1b[i] = v;
    W1bT[n * F + k] = v;
  }
  if (i < F * 2 * F) {
    const int k = i / (2 * F), n = i % (2 * F);
    const __nv_bfloat16 v = __float2bfloat16_rn(p[NP_WPQ + i]);
    Wpq[i] = v;
    WpqT[n * F + k] = v;
  }
}

}  // namespace

extern "C" {

int sg_mlp_param_count(void) { return NP_TOTAL; }
int sg_mlp_edge_blocks(void) { return EDGE_BLOCKS; }
int sg_mlp_part_floats(void) { return 148 * F * 2 * F > EDGE_BLOCKS * L2_GRAD ? 148 * F * 2 * F : EDGE_BLOCKS * L2_GRAD; }

int sg_mlp_prepare(const float* params, void* W1b16, void* W1bT16, void* Wpq16, void* WpqT16, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_ml_bf16_weights<<<(F * 2 * F + 255) / 256, 256, 0, st>>>(
      params, (__nv_bfloat16*)W1b16, (__nv_bfloat16*)W1bT16, (__nv_bfloat16*)Wpq16, (__nv_bfloat16*)WpqT16);
  return cudaGetLastError() == cudaSuccess ? SG_OK : SG_ERR_CUDA;
}

int sg_mlp_forward(const sg_view* V, const double* box, double rc, const float* params, const void* W1bT16,
                   const void* WpqT16, void* s16, void* h16, float* PQ, float* disp, void* stream) {
  if (!V || !box || !params) return SG_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int M = V->slots;
  k_ml_l1<<<EDGE_BLOCKS, 32 * EDGE_WARPS, 0, st>>>(*V, box, rc, params, (__nv_bfloat16*)s16);
  int* gerr = nullptr;
  if (cudaGetSymbolAddress((void**)&gerr, g_ml_tc_err) != cudaSuccess) return SG_ERR_CUDA;
  cudaMemsetAsync(gerr, 0, sizeof(int), st);
  int grc = launch_gemm_tc<F, F>(s16, W1bT16, M, params + NP_B1B, 1, box, nullptr, h16, gerr, st);
  if (grc) return grc;
  grc = launch_gemm_tc<F, 2 * F>(h16, WpqT16, M, nullptr, 0, box, PQ, nullptr, gerr, st);
  if (grc) return grc;
  k_ml_l2<<<EDGE_BLOCKS, 32 * EDGE_WARPS, 0, st>>>(*V, box, rc, params, PQ, disp);
  if (cudaGetLastError() != cudaSuccess) return SG_ERR_CUDA;
  int timed_out = 0;
  if (cudaMemcpyAsync(&timed_out, gerr, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return SG_ERR_CUDA;
  return timed_out ? SG_ERR_TIMEOUT : SG_OK;
}

// Gradients are ADDED to grad[NP_TOTAL] (zero it first).  work: gPQ [M x 128]
// fp32, gPQ16 [M x 128] bf16, gh [M x 64] fp32, gpre16 [M x 64] bf16, gs
// [M x 64] fp32, part >= sg_mlp_part_floats() floats, red >= 512 floats,
// loss_part >= sg_mlp_edge_blocks() floats (per-block partial sums of
// |disp - target|^2).
int sg_mlp_backward(const sg_view* V, const double* box, double rc, const float* params, const void* W1b16,
                    const void* Wpq16, const void* s16, const void* h16, const float* PQ, const float* disp,
                    const float* target, float inv_n, float* gPQ, void* gPQ16, float* gh, void* gpre16, float* gs,
                    float* part, float* red, float* loss_part, float* grad, void* stream) {
  if (!V || !box || !params || !grad) return SG_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int M = V->slots;
  cudaMemsetAsync(gPQ, 0, sizeof(float) * (size_t)M * 2 * F, st);
  // layer 2 edges
  k_ml_l2_bwd<<<EDGE_BLOCKS, 32 * EDGE_WARPS, 0, st>>>(*V, box, rc, params, PQ, disp, target, inv_n, gPQ, part,
                                                       loss_part);
  cudaMemsetAsync(red, 0, sizeof(float) * L2_GRAD, st);
  k_ml_reduce<<<(L2_GRAD + 255) / 256, 256, 0, st>>>(part, EDGE_BLOCKS, L2_GRAD, red);
  k_ml_place<<<1, 256, 0, st>>>(red, 256, grad, NP_W2E);
  k_ml_place<<<1, 64, 0, st>>>(red + 256, 64, grad, NP_B2);
  k_ml_place<<<1, 64, 0, st>>>(red + 320, 64, grad, NP_W2);
  k_ml_place<<<1, 1, 0, st>>>(red + 384, 1, grad, NP_C);
  // gPQ -> bf16 for the GEMMs
  {
    const size_t len = (size_t)M * 2 * F;
    k_ml_to_bf16<<<(unsigned)((len + 255) / 256), 256, 0, st>>>(gPQ, (__nv_bfloat16*)gPQ16, len);
  }
  // gWpq = h^T gPQ (tensor cores, one CTA per SM)
  constexpr int WG_BLOCKS = 148;
  int* werr = nullptr;
  if (cudaGetSymbolAddress((void**)&werr, g_ml_tc_err) != cudaSuccess) return SG_ERR_CUDA;
  cudaMemsetAsync(werr, 0, sizeof(int), st);
  int wrc = launch_wgrad_tc<2 * F>(h16, gPQ16, M, WG_BLOCKS, part, werr, st);
  if (wrc) return wrc;
  k_ml_reduce<<<(F * 2 * F + 255) / 256, 256, 0, st>>>(part, WG_BLOCKS, F * 2 * F, grad + NP_WPQ);
  // gh = gPQ Wpq^T
  wrc = launch_gemm_tc<2 * F, F>(gPQ16, Wpq16, M, nullptr, 0, box, gh, nullptr, werr, st);
  if (wrc) return wrc;
  // through relu(s W1b + b1b)
  k_ml_relu_bwd<<<WG_BLOCKS, 256, 0, st>>>(M, gh, (const __nv_bfloat16*)h16, (__nv_bfloat16*)gpre16, part);
  k_ml_reduce<<<1, 64, 0, st>>>(part, WG_BLOCKS, F, grad + NP_B1B);
  wrc = launch_wgrad_tc<F>(s16, gpre16, M, WG_BLOCKS, part, werr, st);
  if (wrc) return wrc;
  k_ml_reduce<<<(F * F + 255) / 256, 256, 0, st>>>(part, WG_BLOCKS, F * F, grad + NP_W1B);
  // gs = gpre W1b^T
  wrc = launch_gemm_tc<F, F>(gpre16, W1b16, M, nullptr, 0, box, gs, nullptr, werr, st);
  if (wrc) return wrc;
  // layer 1 edges
  k_ml_l1_bwd<<<EDGE_BLOCKS, 32 * EDGE_WARPS, 0, st>>>(*V, box, rc, params, gs, part);
  cudaMemsetAsync(red, 0, sizeof(float) * L1_GRAD, st);
  k_ml_reduce<<<(L1_GRAD + 255) / 256, 256, 0, st>>>(part, EDGE_BLOCKS, L1_GRAD, red);
  k_ml_place<<<1, 256, 0, st>>>(red, 256, grad, NP_W1A);
  k_ml_place<<<1, 64, 0, st>>>(red + 256, 64, grad, NP_B1A);
  if (cudaGetLastError() != cudaSuccess) return SG_ERR_CUDA;
  int timed_out = 0;
  if (cudaMemcpyAsync(&timed_out, werr, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return SG_ERR_CUDA;
  return timed_out ? SG_ERR_TIMEOUT : SG_OK;
}

// x += dx, y += dy for the slots with box > 0 (scale 1), wrapped back into
// the periodic box with the image flags updated, as enforce_periodic would.
__global__ void k_ml_apply(sg_view V, const double* __restrict__ box, const float* __restrict__ disp,
                           int* __restrict__ ix, int* __restrict__ iy) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V.slots) return;
  const double Lx = box[2 * i], Ly = box[2 * i + 1];
  if (!(Lx > 0.0)) return;
  double x = V.x_device[i] + (double)disp[2 * i], y = V.y_device[i] + (double)disp[2 * i + 1];
  if (x <= -0.5 * Lx) { x += Lx; ix[i]--; } else if (x > 0.5 * Lx) { x -= Lx; ix[i]++; }
  if (y <= -0.5 * Ly) { y += Ly; iy[i]--; } else if (y > 0.5 * Ly) { y -= Ly; iy[i]++; }
  V.x_device[i] = x;
  V.y_device[i] = y;
}

int sg_mlp_adam(float* params, const float* grad, float* m, float* v, int n, float lr, float beta1, float beta2,
                float eps, int step, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  k_ml_adam<<<(n + 255) / 256, 256, 0, st>>>(params, grad, m, v, n, lr, beta1, beta2, eps, c1, c2);
  return cudaGetLastError() == cudaSuccess ? SG_OK : SG_ERR_CUDA;
}

int sg_mlp_apply(const sg_view* V, const double* box, const float* disp, int* ix, int* iy, void* stream) {
  if (!V || !box || !disp) return SG_ERR_ARG;
  k_ml_apply<<<(V->slots + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(*V, box, disp, ix, iy);
  return cudaGetLastError() == cudaSuccess ? SG_OK : SG_ERR_CUDA;
}

}  // extern "C"

