// Element-batched form of the fine-level elastic operator on the tensor cores,
// kept to measure it against the matrix-free stencil kernel (k_apply_fine).
//
// The reference applies K(rho) element by element: u_e (24 x R) gathered from
// the element's 8 nodes, Ke_e u_e with Ke_e = rho_e Ke0 by torch.bmm, then
// scattered back with index_add_ (utils/EBE_GMG.py:412-430).  Here the same
// contraction is one GEMM for all elements and load cases of a batch:
//   Y (rows (cell, element, load case) x 24) = U (rows x 24) * Ke0 (24 x 24)
// (Ke0 is symmetric), run by tcgen05.mma kind::tf32 (M = 128 rows per MMA,
// N = 32 with Ke0's 24 columns zero-padded, K = 24 in three K = 8 steps, FP32
// accumulator in tensor memory),
// with rho_e and the operator scale applied in the epilogue.  Three kernels:
//   k_ebe_gather   u [B][6][3][N] -> U rows, written straight into the
//                  tensor-core operand layout (128-row tiles of 12 KB),
//   k_ebe_gemm_tc  U tiles -> Y rows ([rows][24] FP32), a persistent loop
//                  over tiles with double-buffered cp.async staging,
//   k_ebe_scatter  Y rows -> y [B][6][3][N], each node summing the blocks of
//                  its 8 elements.
// Operands are TF32 (10-bit mantissa), which suffices for a multigrid
// preconditioner but not for the FP32 smoother the solver uses; the point
// of the kernels is the cost comparison.
#pragma once

#include "tcgen05.cuh"

namespace maple {

constexpr int EBE_ROWS = 128;                 // rows per tile (one MMA's M)
constexpr int EBE_K = 24;                     // 8 corners x 3 components
constexpr int EBE_N = 32;                     // MMA N: Ke0's 24 columns and 8 zero columns
constexpr int EBE_TILE_BYTES = EBE_ROWS * EBE_K * 4;  // 12 KB
constexpr int EBE_SBO = (EBE_K / 4) * 128;    // 8-row group stride of the K-major TF32 layout
constexpr long long kEbePolls = 1LL << 24;

// byte offset of (row rr, k) inside a 128-row tile: core matrices of 8 rows x
// 16 bytes (4 TF32 values along K), K-chunks 128 bytes apart, 8-row groups
// EBE_SBO apart
__host__ __device__ constexpr int ebe_offset(int rr, int k) {
  return (rr >> 3) * EBE_SBO + (k >> 2) * 128 + (rr & 7) * 16 + (k & 3) * 4;
}

__host__ __device__ constexpr uint32_t idesc_tf32_f32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// one thread per (cell, load case, element): row (cell * N + e) * 6 + r
__global__ void k_ebe_gather(const float* __restrict__ u, float* __restrict__ rows, int n, int B) {
  const int N = n * n * n;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)B * 6 * N) return;
  const int e = (int)(t % N), r = (int)((t / N) % 6), b = (int)(t / ((long long)6 * N));
  const int x = e / (n * n), y = (e / n) % n, z = e % n;
  const long long row = ((long long)b * N + e) * 6 + r;
  char* tile = reinterpret_cast<char*>(rows) + (row / EBE_ROWS) * EBE_TILE_BYTES;
  const int rr = (int)(row % EBE_ROWS);
  const float* ub = u + ((size_t)b * 6 + r) * 3 * N;
  float v[EBE_K];
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int nx = x + corner_x(a), ny = y + corner_y(a), nz = z + corner_z(a);
    const int node = ((nx == n ? 0 : nx) * n + (ny == n ? 0 : ny)) * n + (nz == n ? 0 : nz);
#pragma unroll
    for (int c = 0; c < 3; ++c) v[a * 3 + c] = __ldg(ub + (size_t)c * N + node);
  }
#pragma unroll
  for (int j = 0; j < EBE_K / 4; ++j)
    *reinterpret_cast<float4*>(tile + ebe_offset(rr, 4 * j)) = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
}

// Y rows = U rows * Ke0, scaled by kscale * rho_e; persistent over tiles
__global__ void __launch_bounds__(EBE_ROWS) k_ebe_gemm_tc(const float* __restrict__ rows, const float* __restrict__ rho,
                                                          float* __restrict__ out, long long ntiles, int N,
                                                          float kscale, int* err) {
  using namespace maple_tc;
  __shared__ __align__(1024) uint8_t sA[2][EBE_TILE_BYTES];
  __shared__ __align__(1024) uint8_t sB[EBE_N * EBE_K * 4];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // B = Ke0 rows (N = 32 rows, the last 8 zero, of K = 24), K-major in the same layout
  for (int i = tid; i < EBE_N * EBE_K; i += EBE_ROWS) {
    const int nn = i / EBE_K, k = i % EBE_K;
    *reinterpret_cast<float*>(sB + ebe_offset(nn, k)) = nn < EBE_K ? c_Ke3f[nn * 24 + k] : 0.0f;
  }
  if (warp == 0) tmem_alloc(&tslot, 64);  // two accumulators of 32 columns (at 0 and 32)
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
  }
  fence_async_smem();
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = tslot;
  const uint32_t idesc = idesc_tf32_f32(EBE_ROWS, EBE_N);
  const uint32_t bdesc0 = smem_u32(sB);
  int it = 0;
  bool bad = false;
  long long prev_tile = -1;
  for (long long tile = blockIdx.x;; tile += gridDim.x, ++it) {
    const bool have = tile < ntiles;
    const int buf = it & 1;
    if (have) {
      // stage the tile (12 KB, already in operand layout) with cp.async
      const char* src = reinterpret_cast<const char*>(rows) + tile * EBE_TILE_BYTES;
      for (int i = tid; i < EBE_TILE_BYTES / 16; i += EBE_ROWS) {
        const unsigned sa = smem_u32(sA[buf] + 16 * i);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(src + 16 * i) : "memory");
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    fence_async_smem();
    __syncthreads();
    if (have && tid == 0) {
      fence_after_sync();
      const uint32_t a0 = smem_u32(sA[buf]);
      for (int j = 0; j < EBE_K / 8; ++j)
        mma_tf32(tmem + 32 * buf, smem_desc(a0 + j * 256, 128, EBE_SBO), smem_desc(bdesc0 + j * 256, 128, EBE_SBO),
                 idesc, j > 0 ? 1u : 0u);
      mma_commit(&bar[buf]);
    }
    // epilogue of the previous tile overlaps this tile's MMA
    if (prev_tile >= 0) {
      const int pb = (it - 1) & 1;
      const bool ok = mbar_wait(&bar[pb], (uint32_t)(((it - 1) >> 1) & 1), kEbePolls);
      if (__syncthreads_or(!ok)) {
        bad = true;
        break;
      }
      fence_after_sync();
      float y[EBE_K];
#pragma unroll
      for (int c = 0; c < EBE_K; c += 8) {
        float v[8];
        tmem_ld8(tmem + 32 * pb + ((uint32_t)(32 * warp) << 16) + c, v);
#pragma unroll
        for (int j = 0; j < 8; ++j) y[c + j] = v[j];
      }
      const long long row = prev_tile * EBE_ROWS + 32 * warp + lane;
      const long long cell_e = row / 6;  // cell * N + e
      const float s = kscale * __ldg(rho + cell_e);
      float* o = out + row * EBE_K;
#pragma unroll
      for (int j = 0; j < EBE_K / 4; ++j)
        reinterpret_cast<float4*>(o)[j] = make_float4(s * y[4 * j], s * y[4 * j + 1], s * y[4 * j + 2], s * y[4 * j + 3]);
      fence_before_sync();
      __syncthreads();
    }
    if (!have) break;
    prev_tile = tile;
  }
  if (bad && tid == 0) atomicExch(err, 1);
  // every committed MMA is complete before the tensor memory is freed
  if (tid == 0) mma_commit(&bar[it & 1]);
  mbar_wait(&bar[it & 1], (uint32_t)((it >> 1) & 1), kEbePolls);
  fence_before_sync();
  __syncthreads();
  if (warp == 0) tmem_free(tmem, 64);
}

// y[b][r][c][node] = sum over the 8 elements e with node at their corner a
// of Y[(b * N + e) * 6 + r][3a + c]
__global__ void k_ebe_scatter(const float* __restrict__ Y, float* __restrict__ y, int n, int B) {
  const int N = n * n * n;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)B * 6 * N) return;
  const int node = (int)(t % N), r = (int)((t / N) % 6), b = (int)(t / ((long long)6 * N));
  const int x = node / (n * n), yy = (node / n) % n, z = node % n;
  float acc[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int ex = x - corner_x(a), ey = yy - corner_y(a), ez = z - corner_z(a);
    const int e = ((ex < 0 ? ex + n : ex) * n + (ey < 0 ? ey + n : ey)) * n + (ez < 0 ? ez + n : ez);
    const float* row = Y + (((size_t)b * N + e) * 6 + r) * EBE_K + 3 * a;
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[c] += __ldg(row + c);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) y[(((size_t)b * 6 + r) * 3 + c) * N + node] = acc[c];
}

}  // namespace maple
