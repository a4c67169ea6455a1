// Periodic 3-D convolution network kernels (BF16 storage, FP32 accumulation)
// for the learned initial guess of the homogenization solves.
//
// Activations are channels-last [cell][voxel][channel] BF16 on an n^3
// periodic grid (voxel id x*n*n + y*n + z).  Convolution weights are
// [tap][cin][cout] BF16, tap = 9*(dx+1) + 3*(dy+1) + (dz+1) for a 3x3x3
// kernel (a single tap for 1x1x1).  A convolution is an implicit GEMM on the
// tensor cores (16x16x16 BF16 fragments, FP32 accumulators): rows are output
// voxels, columns output channels, and the reduction runs over (tap, input
// channel) with periodic neighbour gathers (circular padding).
//
// Training uses the same kernel for the data gradient (weights flipped and
// transposed), a tiled weight-gradient GEMM whose reduction runs over
// (cell, voxel), and elementwise kernels for pooling, upsampling, ReLU, the
// MSE loss and Adam.  Conversion kernels move solver fields ([B][R][D][N]
// FP64) to and from network channels.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <mma.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>

#include "../../include/maple_b200.h"
#include "tcgen05.cuh"

namespace maple_nn {

using namespace nvcuda;
using bf16 = __nv_bfloat16;

static thread_local std::string g_nn_err;

constexpr int BM = 64, BN = 64, BK = 16;
constexpr int NT = 128;  // 4 warps; warp w owns rows [16w, 16w+16) of the tile
constexpr int APAD = 8, BPAD = 8, CPAD = 4;

__device__ __forceinline__ int wrapc(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

__device__ __forceinline__ int neighbour(int v, int n, int dx, int dy, int dz) {
  const int z = v % n, y = (v / n) % n, x = v / (n * n);
  return (wrapc(x + dx, n) * n + wrapc(y + dy, n)) * n + wrapc(z + dz, n);
}

// q = v / n and r = v % n for 0 <= v < 2^24 with rn = 1/n (float): one
// multiply and a correction instead of an integer division by a runtime value
__device__ __forceinline__ void divmod_n(int v, int n, float rn, int& q, int& r) {
  q = __float2int_rz((float)v * rn);
  r = v - q * n;
  if (r < 0) {
    --q;
    r += n;
  } else if (r >= n) {
    ++q;
    r -= n;
  }
}

// coordinates of node v (id x n^2 + y n + z)
__device__ __forceinline__ void node_xyz(int v, int n, float rn, int& x, int& y, int& z) {
  int t;
  divmod_n(v, n, rn, t, z);
  divmod_n(t, n, rn, x, y);
}

// neighbour with zero padding outside the grid: -1 there
__device__ __forceinline__ int neighbour_zp(int v, int n, int dx, int dy, int dz) {
  const int z = v % n + dz, y = (v / n) % n + dy, x = v / (n * n) + dx;
  if (x < 0 || x >= n || y < 0 || y >= n || z < 0 || z >= n) return -1;
  return (x * n + y) * n + z;
}

__device__ __forceinline__ void tap_offsets(int tap, int taps, int& dx, int& dy, int& dz) {
  if (taps == 1) {
    dx = dy = dz = 0;
  } else {
    dx = tap / 9 - 1;
    dy = (tap / 3) % 3 - 1;
    dz = tap % 3 - 1;
  }
}

// out[b][v][co] = act( sum_{tap,ci} in[b][nbr(v,tap)][ci] * W[tap][ci][co] + bias[co] + res[b][v][co] )
// act = ReLU when relu != 0; BF16 and/or FP32 outputs.  Neighbours wrap
// (circular padding) unless zero_pad, where taps outside the grid read zero.
// res may alias out (gradient accumulation): each element is read, then written, by one thread.
__global__ void __launch_bounds__(NT) k_conv3d(const bf16* __restrict__ in, const bf16* __restrict__ W,
                                               const float* __restrict__ bias, const bf16* res, bf16* out,
                                               float* __restrict__ out_f32, int n, int cin, int cout, int taps,
                                               int relu, int zero_pad) {
  __shared__ __align__(32) bf16 sA[BM][BK + APAD];
  __shared__ __align__(32) bf16 sB[BK][BN + BPAD];
  __shared__ __align__(32) float sC[BM][BN + CPAD];
  const int N = n * n * n;
  const int b = blockIdx.z;
  const int v0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int warp = threadIdx.x >> 5;
  const bf16* inb = in + (size_t)b * N * cin;
  wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[BN / 16];
#pragma unroll
  for (int j = 0; j < BN / 16; ++j) wmma::fill_fragment(acc[j], 0.0f);
  const bool vec = (cin % 8) == 0;
  for (int tap = 0; tap < taps; ++tap) {
    int dx, dy, dz;
    tap_offsets(tap, taps, dx, dy, dz);
    for (int c0 = 0; c0 < cin; c0 += BK) {
      if (vec) {  // 16-byte gathers: 8 channels of one neighbour voxel
        for (int t = threadIdx.x; t < BM * (BK / 8); t += NT) {
          const int m = t / (BK / 8), h = t % (BK / 8);
          const int v = v0 + m;
          uint4 val = make_uint4(0, 0, 0, 0);
          if (v < N && c0 + 8 * h < cin) {
            const int q = zero_pad ? neighbour_zp(v, n, dx, dy, dz) : neighbour(v, n, dx, dy, dz);
            if (q >= 0) val = *reinterpret_cast<const uint4*>(inb + (size_t)q * cin + c0 + 8 * h);
          }
          *reinterpret_cast<uint4*>(&sA[m][8 * h]) = val;
        }
      } else {
        for (int t = threadIdx.x; t < BM * BK; t += NT) {
          const int m = t / BK, k = t % BK;
          const int v = v0 + m;
          bf16 val = __float2bfloat16(0.0f);
          if (v < N && c0 + k < cin) {
            const int q = zero_pad ? neighbour_zp(v, n, dx, dy, dz) : neighbour(v, n, dx, dy, dz);
            if (q >= 0) val = inb[(size_t)q * cin + c0 + k];
          }
          sA[m][k] = val;
        }
      }
      for (int t = threadIdx.x; t < BK * BN; t += NT) {
        const int k = t / BN, j = t % BN;
        bf16 val = __float2bfloat16(0.0f);
        if (c0 + k < cin && n0 + j < cout) val = W[((size_t)tap * cin + c0 + k) * cout + n0 + j];
        sB[k][j] = val;
      }
      __syncthreads();
      wmma::fragment<wmma::matrix_a, 16, 16, 16, bf16, wmma::row_major> fa;
      wmma::load_matrix_sync(fa, &sA[warp * 16][0], BK + APAD);
#pragma unroll
      for (int j = 0; j < BN / 16; ++j) {
        wmma::fragment<wmma::matrix_b, 16, 16, 16, bf16, wmma::row_major> fb;
        wmma::load_matrix_sync(fb, &sB[0][16 * j], BN + BPAD);
        wmma::mma_sync(acc[j], fa, fb, acc[j]);
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int j = 0; j < BN / 16; ++j)
    wmma::store_matrix_sync(&sC[warp * 16][16 * j], acc[j], BN + CPAD, wmma::mem_row_major);
  __syncthreads();
  for (int t = threadIdx.x; t < BM * BN; t += NT) {
    const int m = t / BN, j = t % BN;
    const int v = v0 + m, co = n0 + j;
    if (v >= N || co >= cout) continue;
    const size_t o = ((size_t)b * N + v) * cout + co;
    float val = sC[m][j];
    if (bias) val += bias[co];
    if (res) val += __bfloat162float(res[o]);
    if (relu) val = fmaxf(val, 0.0f);
    if (out) out[o] = __float2bfloat16(val);
    if (out_f32) out_f32[o] = val;
  }
}

// ---------------------------------------------------------------------------
// The same convolution on the fifth-generation tensor cores (tcgen05):
// an implicit GEMM whose rows are 128 output voxels, columns the output
// channels (one tile of up to 256, zero-padded to a multiple of 16) and
// reduction steps of (tap, KC input channels), KC = the input channel count
// rounded up to 16, at most TC_KC_MAX.  (With TC_KC_MAX 64 the larger stages
// left room for fewer CTAs per SM and the kernel ran slower on B200: 131 vs
// 159 TFLOP/s at 128 channels, 68 vs 74 at 32; so the steps are 16 wide.)  Per step, the 128 threads
// gather the A tile (each thread one voxel row: the tap's periodic or
// zero-padded neighbour, KC/8 chunks of 8 channels, K-major) and the B tile
// (weights, output channel contiguous: MN-major) with cp.async into one of
// TC_STAGES shared-memory stages; one thread issues the step's KC/16
// tcgen05.mma (M = 128, K = 16 each) into an FP32 accumulator in tensor
// memory and commits them to the stage's mbarrier, which releases the stage
// for the load TC_STAGES steps later.  The epilogue reads the accumulator
// rows back (tcgen05.ld, warp w lanes 32w..32w+31) and applies bias,
// residual and ReLU as k_conv3d.  Every mbarrier wait is bounded; a wait that
// runs out sets g_nn_wait_err, waits (bounded) for the issued MMAs and frees
// the tensor memory.  Requires cin % 8 == 0 (16-byte channel chunks).
// ---------------------------------------------------------------------------
constexpr int TC_BM = 128, TC_THREADS = 128, TC_STAGES = 4, TC_BN_MAX = 256, TC_KC_MAX = 16;
constexpr long long kTcPolls = 1LL << 24;
__device__ int g_nn_wait_err;

__host__ __device__ inline int tc_bn(int cout_left) {
  const int c = cout_left < TC_BN_MAX ? cout_left : TC_BN_MAX;
  return (c + 15) / 16 * 16;
}
__host__ __device__ inline int tc_kc(int cin) {
  const int c = (cin + 15) / 16 * 16;
  return c < TC_KC_MAX ? c : TC_KC_MAX;
}
__host__ __device__ inline int tc_tmem_cols(int bn) {
  int c = 32;
  while (c < bn) c <<= 1;
  return c;
}
// one stage: A (128 x KC) and B (BN x KC) BF16
__host__ __device__ inline size_t tc_stage_bytes(int bn, int kc) { return (size_t)(TC_BM + bn) * kc * 2; }

__device__ __forceinline__ void cp_async16_zfill(void* sdst, const void* gsrc, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gsrc), "r"(n) : "memory");
}

__global__ void __launch_bounds__(TC_THREADS) k_conv3d_tc(const bf16* __restrict__ in, const bf16* __restrict__ W,
                                                          const float* __restrict__ bias, const bf16* res, bf16* out,
                                                          float* __restrict__ out_f32, int n, int cin, int cout,
                                                          int taps, int relu, int zero_pad) {
  using namespace maple_tc;
  extern __shared__ __align__(1024) uint8_t tc_smem[];
  __shared__ __align__(8) uint64_t mma_bar[TC_STAGES];
  __shared__ __align__(8) uint64_t done_bar;
  __shared__ uint32_t tslot;
  const int N = n * n * n;
  const int b = blockIdx.z;
  const int v0 = blockIdx.x * TC_BM, n0 = blockIdx.y * TC_BN_MAX;
  const int BN = tc_bn(cout - n0), KC = tc_kc(cin), KB = KC / 8;
  const uint32_t ncols = (uint32_t)tc_tmem_cols(BN);
  const size_t stage = tc_stage_bytes(BN, KC);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int kc = (cin + KC - 1) / KC, KS = taps * kc;
  const bf16* inb = in + (size_t)b * N * cin;
  const bool wvec = (cout % 8) == 0;
  if (warp == 0) tmem_alloc(&tslot, ncols);
  if (tid == 0) {
    for (int i = 0; i < TC_STAGES; ++i) mbar_init(&mma_bar[i], 1);
    mbar_init(&done_bar, 1);
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = tslot;
  const uint32_t idesc = idesc_bf16_f32(TC_BM, BN, 1);
  // A: K-major, 8-row groups KB*128 bytes apart; B: MN-major, K-groups 128
  // bytes apart, 8-column groups KC*16 bytes apart; each MMA takes 16 of K
  const uint32_t sbo_a = (uint32_t)KB * 128, sbo_b = (uint32_t)KC * 16;
  const int m = tid;  // this thread's A row
  const int v = v0 + m;
  // the row's coordinates, once (the taps only shift them)
  int vx = 0, vy = 0, vz = 0;
  if (v < N) node_xyz(v, n, 1.0f / (float)n, vx, vy, vz);
  int issued = 0;     // MMA steps issued (thread 0)
  bool timed_out = false;
  int tap = 0, chunk = 0;  // step t = tap * kc + chunk
  for (int t = 0; t <= KS; ++t) {
    if (t < KS) {
      const int st = t % TC_STAGES;
      if (t >= TC_STAGES) {
        const bool ok = mbar_wait(&mma_bar[st], (uint32_t)((t / TC_STAGES - 1) & 1), kTcPolls);
        if (__syncthreads_or(!ok)) {
          timed_out = true;
          break;
        }
      }
      uint8_t* sA = tc_smem + st * stage;
      uint8_t* sB = sA + TC_BM * KC * 2;
      const int c0 = chunk * KC;
      int dx, dy, dz;
      tap_offsets(tap, taps, dx, dy, dz);
      int q = -1;
      if (v < N) {
        int x = vx + dx, y = vy + dy, z = vz + dz;
        if (zero_pad) {
          if (x >= 0 && x < n && y >= 0 && y < n && z >= 0 && z < n) q = (x * n + y) * n + z;
        } else {
          q = (wrapc(x, n) * n + wrapc(y, n)) * n + wrapc(z, n);
        }
      }
      const bf16* rowp = inb + (size_t)(q < 0 ? 0 : q) * cin + c0;
      for (int h = 0; h < KB; ++h) {
        const bool ok = q >= 0 && c0 + 8 * h < cin;
        cp_async16_zfill(sA + (m >> 3) * sbo_a + h * 128 + (m & 7) * 16, ok ? rowp + 8 * h : inb, ok);
      }
      const int groups = BN / 8;
      if (wvec) {
        for (int i = tid; i < KC * groups; i += TC_THREADS) {
          const int k = i / groups, g = i - k * groups;
          const int ci = c0 + k, co = n0 + 8 * g;
          const bool ok = ci < cin && co < cout;
          const bf16* src = ok ? W + ((size_t)tap * cin + ci) * cout + co : W;
          cp_async16_zfill(sB + mnmajor_offset(8 * g, k, 128, sbo_b), src, ok);
        }
      } else {
        for (int i = tid; i < KC * BN; i += TC_THREADS) {
          const int k = i / BN, j = i - k * BN;
          const int ci = c0 + k, co = n0 + j;
          bf16 val = __float2bfloat16(0.0f);
          if (ci < cin && co < cout) val = W[((size_t)tap * cin + ci) * cout + co];
          *reinterpret_cast<bf16*>(sB + mnmajor_offset(j, k, 128, sbo_b)) = val;
        }
      }
      if (++chunk == kc) {
        chunk = 0;
        ++tap;
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    if (t >= 1) {
      asm volatile("cp.async.wait_group 1;\n" ::: "memory");
      fence_async_smem();
      __syncthreads();
      if (tid == 0) {
        fence_after_sync();
        const int s = t - 1, st = s % TC_STAGES;
        const uint32_t a = smem_u32(tc_smem + st * stage), bb = a + TC_BM * KC * 2;
        for (int j = 0; j < KC / 16; ++j)
          mma_bf16(tmem, smem_desc(a + j * 256, 128, sbo_a), smem_desc(bb + j * 256, 128, sbo_b), idesc,
                   (s > 0 || j > 0) ? 1u : 0u);
        mma_commit(&mma_bar[st]);
        issued = s + 1;
      }
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  // every issued MMA has completed once done_bar flips (also after a timeout)
  if (tid == 0) {
    if (issued == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&done_bar)) : "memory");
    else mma_commit(&done_bar);
  }
  const bool fin = mbar_wait(&done_bar, 0, kTcPolls);
  const bool bad = __syncthreads_or(timed_out || !fin);
  if (bad) {
    if (tid == 0) atomicExch(&g_nn_wait_err, 1);
  } else {
    fence_after_sync();
    for (int c = 0; c < BN; c += 8) {
      float acc[8];
      tmem_ld8(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c, acc);
      const int vv = v0 + 32 * warp + lane;
      if (vv < N) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int co = n0 + c + j;
          if (co >= cout) continue;
          const size_t o = ((size_t)b * N + vv) * cout + co;
          float val = acc[j];
          if (bias) val += bias[co];
          if (res) val += __bfloat162float(res[o]);
          if (relu) val = fmaxf(val, 0.0f);
          if (out) out[o] = __float2bfloat16(val);
          if (out_f32) out_f32[o] = val;
        }
      }
    }
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) tmem_free(tmem, ncols);
}

// Weight gradient on the tcgen05 tensor cores:
//   dW[tap][ci][co] += sum over (cell, voxel) of in[cell][nbr(v, tap)][ci] * dz[cell][v][co].
// The rows of dW, r = tap * cin + ci, are one flat M dimension: a CTA owns 128
// consecutive rows (16 groups of 8 channels, each group inside one tap, so
// narrow layers put several taps in one tile), up to 256 output channels (N)
// and a chunk of (cell, voxel) pairs, the reduction.  Both operands come
// MN-major straight from the channels-last activations: per stage the 256
// threads gather 64 pairs x 16 channel groups of the input (each group's own
// periodic neighbour) and 64 rows of dz with cp.async into a 4-stage ring, in
// four 16-pair slabs, and one thread issues the four K = 16 MMAs of the stage
// into an FP32 accumulator in tensor memory while the next two stages load.
// The epilogue adds the CTA's partial dW to global memory with FP32 atomics.
// Waits are bounded as in k_conv3d_tc.  Requires cin % 8 == 0, cout % 8 == 0
// and 64 <= n^3 < 2^24 (a stage's pairs cross at most one cell boundary; the
// coordinates come from a float reciprocal).
constexpr int WG_CI = 128;     // dW rows per CTA
constexpr int WG_KP = 64;      // (cell, voxel) pairs per stage: four MMAs of K = 16
constexpr int WG_STAGES = 4;   // ring depth; loads run WG_STAGES - 2 stages ahead
constexpr int WG_THREADS = 256;
__host__ __device__ inline size_t wg_stage_bytes(int bn) { return (size_t)(WG_CI + bn) * WG_KP * 2; }

__global__ void __launch_bounds__(WG_THREADS) k_conv3d_wgrad_tc(const bf16* __restrict__ in,
                                                                const bf16* __restrict__ dz, float* __restrict__ dW,
                                                                int B, int n, int cin, int cout, int taps,
                                                                long long chunk) {
  using namespace maple_tc;
  constexpr int LA = WG_STAGES - 2;
  extern __shared__ __align__(1024) uint8_t wg_smem[];
  __shared__ __align__(8) uint64_t mma_bar[WG_STAGES];
  __shared__ __align__(8) uint64_t done_bar;
  __shared__ uint32_t tslot;
  const int N = n * n * n;
  const int R = taps * cin;
  const int r0 = blockIdx.x * WG_CI;
  const int n0 = blockIdx.y * TC_BN_MAX;
  const int BN = tc_bn(cout - n0);
  const uint32_t ncols = (uint32_t)tc_tmem_cols(BN);
  const size_t stage = wg_stage_bytes(BN);
  const uint32_t slab_a = WG_CI * 32, slab_b = (uint32_t)BN * 32;  // one 16-pair slab of each operand
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // this thread's input group: dW rows ra .. ra + 7 = tap ra / cin, channels cia .. cia + 7
  const int g = tid & 15, ra = r0 + 8 * g;
  const bool row_ok = ra < R;
  int ox = 0, oy = 0, oz = 0, cia = 0;
  if (row_ok) {
    const int tp = ra / cin;
    cia = ra - tp * cin;
    tap_offsets(tp, taps, ox, oy, oz);
  }
  const long long total = (long long)B * N;
  const long long kbeg = (long long)blockIdx.z * chunk, kend = kbeg + chunk < total ? kbeg + chunk : total;
  const int KS = (int)((kend - kbeg + WG_KP - 1) / WG_KP);
  const float rn = 1.0f / (float)n;
  if (warp == 0) tmem_alloc(&tslot, ncols);
  if (tid == 0) {
    for (int i = 0; i < WG_STAGES; ++i) mbar_init(&mma_bar[i], 1);
    mbar_init(&done_bar, 1);
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = tslot;
  // A (M = dW rows) and B (N = output channels) both MN-major: 8-row groups
  // 256 bytes apart, the two 8-pair K-groups of a slab 128 bytes apart
  const uint32_t idesc = idesc_bf16_f32(WG_CI, BN, 1, 1);
  const int groups = BN / 8;
  int issued = 0;
  bool timed_out = false;
  for (int t = 0; t < KS + LA; ++t) {
    if (t < KS) {
      const int st = t % WG_STAGES;
      if (t >= WG_STAGES) {
        const bool ok = mbar_wait(&mma_bar[st], (uint32_t)((t / WG_STAGES - 1) & 1), kTcPolls);
        if (__syncthreads_or(!ok)) {
          timed_out = true;
          break;
        }
      }
      uint8_t* sA = wg_smem + st * stage;
      uint8_t* sB = sA + (WG_KP / 16) * slab_a;
      const long long k0 = kbeg + (long long)WG_KP * t;
      // the stage's first (cell, voxel) pair, once per stage; its 64 pairs
      // wrap into the next cell at most once (N >= 64)
      const int b0 = (int)(k0 / N), v0 = (int)(k0 - (long long)b0 * N);
#pragma unroll
      for (int j = 0; j < WG_KP / 16; ++j) {
        const int k = (tid >> 4) + 16 * j;
        const long long kk = k0 + k;
        const bool ok = row_ok && kk < kend;
        const bf16* src = in;
        if (ok) {
          int b = b0, v = v0 + k;
          if (v >= N) {
            v -= N;
            ++b;
          }
          int x, y, z;
          node_xyz(v, n, rn, x, y, z);
          const int q = (wrapc(x + ox, n) * n + wrapc(y + oy, n)) * n + wrapc(z + oz, n);
          src = in + ((size_t)b * N + q) * cin + cia;
        }
        cp_async16_zfill(sA + j * slab_a + mnmajor_offset(8 * g, k & 15, 128, 256), src, ok);
      }
      for (int i = tid; i < WG_KP * groups; i += WG_THREADS) {
        const int k = i / groups, h = i - k * groups;
        const long long kk = k0 + k;
        const bool ok = kk < kend && n0 + 8 * h < cout;
        cp_async16_zfill(sB + (k >> 4) * slab_b + mnmajor_offset(8 * h, k & 15, 128, 256),
                         ok ? dz + (size_t)kk * cout + n0 + 8 * h : dz, ok);
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    const int s = t - LA;
    if (s >= 0) {
      asm volatile("cp.async.wait_group %0;\n" ::"n"(LA) : "memory");
      fence_async_smem();
      __syncthreads();
      if (tid == 0) {
        fence_after_sync();
        const int st = s % WG_STAGES;
        const uint32_t a = smem_u32(wg_smem + st * stage), bb = a + (WG_KP / 16) * slab_a;
#pragma unroll
        for (int j = 0; j < WG_KP / 16; ++j)
          mma_bf16(tmem, smem_desc(a + j * slab_a, 128, 256), smem_desc(bb + j * slab_b, 128, 256), idesc,
                   (s > 0 || j > 0) ? 1u : 0u);
        mma_commit(&mma_bar[st]);
        issued = s + 1;
      }
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  if (tid == 0) {
    if (issued == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&done_bar)) : "memory");
    else mma_commit(&done_bar);
  }
  const bool fin = mbar_wait(&done_bar, 0, kTcPolls);
  const bool bad = __syncthreads_or(timed_out || !fin);
  if (bad) {
    if (tid == 0) atomicExch(&g_nn_wait_err, 1);
  } else if (KS > 0) {
    fence_after_sync();
    // warp w reads TMEM lanes 32 (w % 4) .. + 31 (its rows), columns of half w / 4
    const int q = warp & 3, r = r0 + 32 * q + lane;
    const int cb = (warp >> 2) * (BN / 2);
    for (int c = cb; c < cb + BN / 2; c += 8) {
      float acc[8];
      tmem_ld8(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)c, acc);
      if (r < R) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int co = n0 + c + j;
          if (co < cout) atomicAdd(&dW[(size_t)r * cout + co], acc[j]);
        }
      }
    }
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) tmem_free(tmem, ncols);
}

// dW[tap][ci][co] += sum_{b,v} in[b][nbr(v,tap)][ci] * dz[b][v][co]  (FP32 atomics)
// The reduction index kk runs over (b, v) flattened; CTA (x, y, z) owns
// tap x / (cin tiles), a 64x64 (ci, co) tile and the z-th slice of kk.
constexpr int WK = 32;
__global__ void __launch_bounds__(NT) k_conv3d_wgrad(const bf16* __restrict__ in, const bf16* __restrict__ dz,
                                                     float* __restrict__ dW, int B, int n, int cin, int cout, int taps,
                                                     long long chunk) {
  __shared__ __align__(32) bf16 sX[WK][BM + APAD];  // [kk][ci]: A = X^T is col-major
  __shared__ __align__(32) bf16 sD[WK][BN + BPAD];  // [kk][co]
  __shared__ __align__(32) float sC[BM][BN + CPAD];
  const int N = n * n * n;
  const int mt = (cin + BM - 1) / BM;
  const int tap = blockIdx.x / mt, c0 = (blockIdx.x % mt) * BM;
  const int n0 = blockIdx.y * BN;
  int ox, oy, oz;
  tap_offsets(tap, taps, ox, oy, oz);
  const int warp = threadIdx.x >> 5;
  const long long total = (long long)B * N;
  const long long kbeg = (long long)blockIdx.z * chunk, kend = kbeg + chunk < total ? kbeg + chunk : total;
  wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[BN / 16];
#pragma unroll
  for (int j = 0; j < BN / 16; ++j) wmma::fill_fragment(acc[j], 0.0f);
  const bool vec = (cin % 8) == 0;
  for (long long k0 = kbeg; k0 < kend; k0 += WK) {
    if (vec) {
      for (int t = threadIdx.x; t < WK * (BM / 8); t += NT) {
        const int k = t / (BM / 8), h = t % (BM / 8);
        const long long kk = k0 + k;
        uint4 val = make_uint4(0, 0, 0, 0);
        if (kk < kend && c0 + 8 * h < cin) {
          const long long b = kk / N;
          const int v = (int)(kk - b * N);
          val = *reinterpret_cast<const uint4*>(in + ((size_t)b * N + neighbour(v, n, ox, oy, oz)) * cin + c0 + 8 * h);
        }
        *reinterpret_cast<uint4*>(&sX[k][8 * h]) = val;
      }
    } else {
      for (int t = threadIdx.x; t < WK * BM; t += NT) {
        const int k = t / BM, m = t % BM;
        const long long kk = k0 + k;
        bf16 val = __float2bfloat16(0.0f);
        if (kk < kend && c0 + m < cin) {
          const long long b = kk / N;
          const int v = (int)(kk - b * N);
          val = in[((size_t)b * N + neighbour(v, n, ox, oy, oz)) * cin + c0 + m];
        }
        sX[k][m] = val;
      }
    }
    if ((cout % 8) == 0) {
      for (int t = threadIdx.x; t < WK * (BN / 8); t += NT) {
        const int k = t / (BN / 8), h = t % (BN / 8);
        const long long kk = k0 + k;
        uint4 val = make_uint4(0, 0, 0, 0);
        if (kk < kend && n0 + 8 * h < cout) val = *reinterpret_cast<const uint4*>(dz + (size_t)kk * cout + n0 + 8 * h);
        *reinterpret_cast<uint4*>(&sD[k][8 * h]) = val;
      }
    } else {
      for (int t = threadIdx.x; t < WK * BN; t += NT) {
        const int k = t / BN, j = t % BN;
        const long long kk = k0 + k;
        bf16 val = __float2bfloat16(0.0f);
        if (kk < kend && n0 + j < cout) val = dz[(size_t)kk * cout + n0 + j];
        sD[k][j] = val;
      }
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < WK; ks += 16) {
      wmma::fragment<wmma::matrix_a, 16, 16, 16, bf16, wmma::col_major> fa;
      wmma::load_matrix_sync(fa, &sX[ks][16 * warp], BM + APAD);
#pragma unroll
      for (int j = 0; j < BN / 16; ++j) {
        wmma::fragment<wmma::matrix_b, 16, 16, 16, bf16, wmma::row_major> fb;
        wmma::load_matrix_sync(fb, &sD[ks][16 * j], BN + BPAD);
        wmma::mma_sync(acc[j], fa, fb, acc[j]);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < BN / 16; ++j)
    wmma::store_matrix_sync(&sC[warp * 16][16 * j], acc[j], BN + CPAD, wmma::mem_row_major);
  __syncthreads();
  for (int t = threadIdx.x; t < BM * BN; t += NT) {
    const int m = t / BN, j = t % BN;
    if (c0 + m < cin && n0 + j < cout) atomicAdd(&dW[((size_t)tap * cin + c0 + m) * cout + n0 + j], sC[m][j]);
  }
}

// db[co] += sum_rows dz[row][co]
__global__ void k_bias_grad(const bf16* __restrict__ dz, float* __restrict__ db, long long rows, int cout) {
  const int co = blockIdx.y * 32 + (threadIdx.x & 31);
  if (co >= cout) return;
  float s = 0;
  const int wpb = blockDim.x / 32;
  for (long long r = (long long)blockIdx.x * wpb + (threadIdx.x >> 5); r < rows; r += (long long)gridDim.x * wpb)
    s += __bfloat162float(dz[r * cout + co]);
  atomicAdd(&db[co], s);
}

// data-gradient weights: Wt[taps-1-tap][co][ci] = W[tap][ci][co]
__global__ void k_flip_weights(const bf16* __restrict__ W, bf16* __restrict__ Wt, int cin, int cout, int taps) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t total = (size_t)taps * cin * cout;
  if (i >= total) return;
  const int co = i % cout, ci = (i / cout) % cin, tap = i / ((size_t)cout * cin);
  Wt[((size_t)(taps - 1 - tap) * cout + co) * cin + ci] = W[i];
}

__device__ __forceinline__ size_t fine_of(size_t b, int X, int Y, int Z, int o, int nf) {
  const int x = 2 * X + (o >> 2), y = 2 * Y + ((o >> 1) & 1), z = 2 * Z + (o & 1);
  return b * nf * nf * nf + ((size_t)x * nf + y) * nf + z;
}

// fine -> coarse: w * (sum of the 8 children) [+ c]
// (w = 1/8: average pooling; w = 1: adjoint of nearest upsampling)
__global__ void k_fine_to_coarse(const bf16* __restrict__ f, bf16* __restrict__ c, int nc, int C, int B, float w,
                                 int add) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t Nc = (size_t)nc * nc * nc, total = (size_t)B * Nc * C;
  if (i >= total) return;
  const int ch = i % C;
  const size_t vc = (i / C) % Nc, b = i / (C * Nc);
  const int Z = vc % nc, Y = (vc / nc) % nc, X = vc / ((size_t)nc * nc);
  float s = 0;
#pragma unroll
  for (int o = 0; o < 8; ++o) s += __bfloat162float(f[fine_of(b, X, Y, Z, o, 2 * nc) * C + ch]);
  s *= w;
  if (add) s += __bfloat162float(c[i]);
  c[i] = __float2bfloat16(s);
}

// coarse -> fine: w * parent [+ base] [+ f]
// (w = 1: nearest upsampling, base = skip connection; w = 1/8: adjoint of pooling)
__global__ void k_coarse_to_fine(const bf16* __restrict__ c, const bf16* __restrict__ base, bf16* __restrict__ f,
                                 int nc, int C, int B, float w, int add) {
  const int nf = 2 * nc;
  const size_t Nf = (size_t)nf * nf * nf, total = (size_t)B * Nf * C;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int ch = i % C;
  const size_t vf = (i / C) % Nf, b = i / (C * Nf);
  const int z = vf % nf, y = (vf / nf) % nf, x = vf / ((size_t)nf * nf);
  float v = w * __bfloat162float(c[((b * nc * nc * nc) + ((size_t)(x >> 1) * nc + (y >> 1)) * nc + (z >> 1)) * C + ch]);
  if (base) v += __bfloat162float(base[i]);
  if (add) v += __bfloat162float(f[i]);
  f[i] = __float2bfloat16(v);
}

// dst = src (+ dst when add)
__global__ void k_accumulate(bf16* __restrict__ dst, const bf16* __restrict__ src, size_t total, int add) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  float v = __bfloat162float(src[i]);
  if (add) v += __bfloat162float(dst[i]);
  dst[i] = __float2bfloat16(v);
}

// g <- g * [y > 0]
__global__ void k_relu_mask(const bf16* __restrict__ y, bf16* __restrict__ g, size_t total) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  if (!(__bfloat162float(y[i]) > 0.0f)) g[i] = __float2bfloat16(0.0f);
}

// mean squared error of an FP32 prediction against a BF16 target: loss +=
// sum (p - t)^2 / total, grad = 2 (p - t) / total * gscale (BF16).
__global__ void k_mse(const float* __restrict__ pred, const bf16* __restrict__ target, bf16* __restrict__ grad,
                      float* __restrict__ loss, size_t total, float gscale) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0;
  if (i < total) {
    const float d = pred[i] - __bfloat162float(target[i]);
    if (grad) grad[i] = __float2bfloat16(2.0f * d / (float)total * gscale);
    l = d * d / (float)total;
  }
  for (int off = 16; off > 0; off >>= 1) l += __shfl_down_sync(0xffffffffu, l, off);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
}

// Stiffness weights of the nodes of a cell: w[b][v] = (mean of rho over the 8
// elements sharing node v) / (mean of rho over the cell), so that the weights
// average to 1 in every cell.  Element e = (x,y,z) has nodes (x+a, y+b, z+c),
// a,b,c in {0,1}, periodically.  One block per cell.
__global__ void k_node_weights(const double* __restrict__ rho, float* __restrict__ w, int n) {
  __shared__ double red[32];
  const int N = n * n * n;
  const double* r = rho + (size_t)blockIdx.x * N;
  double s = 0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) s += r[i];
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if (threadIdx.x == 0) red[0] = s / N;
  }
  __syncthreads();
  const double inv = red[0] > 0 ? 1.0 / red[0] : 0.0;
  for (int v = threadIdx.x; v < N; v += blockDim.x) {
    double acc = 0;
#pragma unroll
    for (int o = 0; o < 8; ++o) acc += r[neighbour(v, n, -(o >> 2), -((o >> 1) & 1), -(o & 1))];
    w[(size_t)blockIdx.x * N + v] = (float)(0.125 * acc * inv);
  }
}

// ebar[b][c] += sum_v w[b][v] * (pred - target)[b][v][c] / N  (weights average to 1)
// grid (chunks, B); C <= 64 channels
__global__ void k_weighted_error_mean(const float* __restrict__ pred, const bf16* __restrict__ target,
                                      const float* __restrict__ w, float* __restrict__ ebar, int N, int C) {
  __shared__ float acc[64];
  for (int c = threadIdx.x; c < C; c += blockDim.x) acc[c] = 0.0f;
  __syncthreads();
  const size_t b = blockIdx.y, NC = (size_t)N * C;
  const size_t per = (NC + gridDim.x - 1) / gridDim.x;
  const size_t beg = blockIdx.x * per, end = beg + per < NC ? beg + per : NC;
  for (size_t i = beg + threadIdx.x; i < end; i += blockDim.x) {
    const size_t g = b * NC + i;
    const float ww = w ? w[b * N + i / C] : 1.0f;
    atomicAdd(&acc[i % C], ww * (pred[g] - __bfloat162float(target[g])));
  }
  __syncthreads();
  for (int c = threadIdx.x; c < C; c += blockDim.x) atomicAdd(&ebar[b * C + c], acc[c] / N);
}

// loss += sum w (e - ebar)^2 / total, grad = 2 w (e - ebar) / total * gscale,
// e = pred - target: the node-weighted squared error with the per-(cell,
// channel) weighted mean error removed (a constant field is free).
__global__ void k_mse_weighted(const float* __restrict__ pred, const bf16* __restrict__ target,
                               const float* __restrict__ w, const float* __restrict__ ebar, bf16* __restrict__ grad,
                               float* __restrict__ loss, int N, int C, size_t total, float gscale) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0;
  if (i < total) {
    const size_t row = i / C;
    const int c = i % C;
    const size_t b = row / N;
    const float ww = w ? w[row] : 1.0f;
    const float e = pred[i] - __bfloat162float(target[i]) - (ebar ? ebar[b * C + c] : 0.0f);
    if (grad) grad[i] = __float2bfloat16(2.0f * ww * e / (float)total * gscale);
    l = ww * e * e / (float)total;
  }
  for (int off = 16; off > 0; off >>= 1) l += __shfl_down_sync(0xffffffffu, l, off);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
}

// e[b][f][v] = scale[f] * (pred - target)[b][v][c0 + f]: the prediction error of
// F fields as a solver field [B][F][N] (FP64)
__global__ void k_error_fields(const float* __restrict__ pred, const bf16* __restrict__ target,
                               const double* __restrict__ scale, double* __restrict__ e, int N, int F, int C, int c0,
                               size_t total) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int v = i % N;
  const size_t bf = i / N;
  const int f = bf % F;
  const size_t b = bf / F;
  const size_t o = (b * N + v) * C + c0 + f;
  e[i] = (scale ? scale[f] : 1.0) * (double)(pred[o] - __bfloat162float(target[o]));
}

// out[k] = sum_j a[k][j] * b[k][j] over blocks of L contiguous doubles (one CTA per block)
__global__ void k_block_dot(const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out,
                            size_t L) {
  __shared__ double red[32];
  const double* pa = a + blockIdx.x * L;
  const double* pb = b + blockIdx.x * L;
  double s = 0;
  for (size_t i = threadIdx.x; i < L; i += blockDim.x) s += pa[i] * pb[i];
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if (threadIdx.x == 0) out[blockIdx.x] = s;
  }
}

// grad[b][v][c0 + r*D + d] = coef * scale[r*D + d] * y[b][r][d][v] / norm[b][r]  (BF16):
// the gradient of sum_{b,r} e_r^T K e_r / norm[b][r] with y = K e, through e = scale * channels
__global__ void k_energy_grad(const double* __restrict__ y, const double* __restrict__ norm,
                              const double* __restrict__ scale, bf16* __restrict__ grad, int N, int R, int D, int C,
                              int c0, double coef, size_t total) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;  // over B*R*D*N, node fastest
  if (i >= total) return;
  const int v = i % N;
  const size_t bf = i / N;
  const int f = bf % (R * D);
  const size_t b = bf / (R * D);
  const int r = f / D;
  const double g = coef * (scale ? scale[f] : 1.0) * y[i] / norm[b * R + r];
  grad[(b * N + v) * C + c0 + f] = __float2bfloat16((float)g);
}

// out += sum g^2 (FP64 accumulation across blocks)
__global__ void k_sumsq(const float* __restrict__ g, size_t n, double* __restrict__ out) {
  __shared__ double red[32];
  double s = 0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    s += (double)g[i] * g[i];
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if (threadIdx.x == 0) atomicAdd(out, s);
  }
}

// Adam on FP32 master weights (bias-corrected, decoupled weight decay),
// refreshing the BF16 copy; the gradient is divided by gscale first.
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       bf16* __restrict__ wb, size_t total, float lr, float b1, float b2, float eps, float c1, float c2,
                       float inv_gscale, float wd) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const float gi = g[i] * inv_gscale;
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  float wi = w[i] * (1.0f - lr * wd);
  wi -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  if (wb) wb[i] = __float2bfloat16(wi);
}

__global__ void k_f32_to_bf16(const float* __restrict__ a, bf16* __restrict__ b, size_t total) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < total) b[i] = __float2bfloat16(a[i]);
}

// input features from the element density: ch0 = rho^(1/3), ch1 = rho, rest 0
__global__ void k_features(const double* __restrict__ rho, bf16* __restrict__ out, size_t total, int C) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const double r = rho[i];
  bf16* o = out + i * C;
  o[0] = __float2bfloat16((float)cbrt(r > 0 ? r : 0.0));
  if (C > 1) o[1] = __float2bfloat16((float)r);
  for (int c = 2; c < C; ++c) o[c] = __float2bfloat16(0.0f);
}

// per-(cell, field) mean over the N nodes of an SoA field [B*F][N]
__global__ void k_field_mean(const double* __restrict__ u, double* __restrict__ mean, int N) {
  __shared__ double red[32];
  const double* p = u + (size_t)blockIdx.x * N;
  double s = 0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) s += p[i];
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if (threadIdx.x == 0) mean[blockIdx.x] = s / N;
  }
}

// out[b][v][c0 + f] = scale[f] * (u[b][f][v] - mean[b][f])  for f < F  (BF16)
__global__ void k_fields_to_channels(const double* __restrict__ u, const double* __restrict__ mean,
                                     bf16* __restrict__ out, int N, int F, int C, int c0,
                                     const double* __restrict__ scale, size_t total) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;  // over B*F*N, node fastest
  if (i >= total) return;
  const int v = i % N;
  const size_t bf = i / N;
  const int f = bf % F;
  const size_t b = bf / F;
  const double m = mean ? mean[bf] : 0.0;
  const double sc = scale ? scale[f] : 1.0;
  out[(b * N + v) * C + c0 + f] = __float2bfloat16((float)(sc * (u[i] - m)));
}

// u[b][f][v] = scale[f] * in[b][v][c0 + f]  (FP32 channels -> FP64 field)
__global__ void k_channels_to_fields(const float* __restrict__ in, double* __restrict__ u, int N, int F, int C, int c0,
                                     const double* __restrict__ scale, size_t total) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int v = i % N;
  const size_t bf = i / N;
  const int f = bf % F;
  const size_t b = bf / F;
  u[i] = (scale ? scale[f] : 1.0) * (double)in[(b * N + v) * C + c0 + f];
}

// trilinear prolongation of periodic nodal fields [BF][nc^3] -> [BF][nf^3],
// nf = s * nc: fine node j lies at coarse coordinate j / s.
__global__ void k_prolong_fields(const double* __restrict__ uc, double* __restrict__ uf, int nc, int s, size_t total) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int nf = nc * s;
  const size_t Nf = (size_t)nf * nf * nf, Nc = (size_t)nc * nc * nc;
  const size_t bf = i / Nf;
  const int vf = i % Nf;
  const int z = vf % nf, y = (vf / nf) % nf, x = vf / (nf * nf);
  const int X = x / s, Y = y / s, Z = z / s;
  const double fx = (double)(x - X * s) / s, fy = (double)(y - Y * s) / s, fz = (double)(z - Z * s) / s;
  const double* c = uc + bf * Nc;
  double acc = 0;
#pragma unroll
  for (int o = 0; o < 8; ++o) {
    const int ax = o >> 2, ay = (o >> 1) & 1, az = o & 1;
    const double w = (ax ? fx : 1 - fx) * (ay ? fy : 1 - fy) * (az ? fz : 1 - fz);
    const int cx = (X + ax) % nc, cy = (Y + ay) % nc, cz = (Z + az) % nc;
    acc += w * c[((size_t)cx * nc + cy) * nc + cz];
  }
  uf[i] = acc;
}

// periodic average of element densities over s^3 blocks: [B][nf^3] -> [B][nc^3]
__global__ void k_restrict_density(const double* __restrict__ rf, double* __restrict__ rc, int nc, int s,
                                   size_t total) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int nf = nc * s;
  const size_t Nc = (size_t)nc * nc * nc;
  const size_t b = i / Nc;
  const int vc = i % Nc;
  const int Z = vc % nc, Y = (vc / nc) % nc, X = vc / (nc * nc);
  const double* f = rf + b * (size_t)nf * nf * nf;
  double acc = 0;
  for (int a = 0; a < s; ++a)
    for (int c = 0; c < s; ++c)
      for (int d = 0; d < s; ++d) acc += f[((size_t)(X * s + a) * nf + (Y * s + c)) * nf + (Z * s + d)];
  rc[i] = acc / ((double)s * s * s);
}

static inline unsigned blocks(size_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

template <typename F>
static int nn_guard(F&& f) {
  const char* msg = f();
  if (msg) {
    g_nn_err = msg;
    return MAPLE_E_BADARG;
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    g_nn_err = std::string("CUDA error: ") + cudaGetErrorString(e);
    return MAPLE_E_CUDA;
  }
  return MAPLE_OK;
}

static unsigned long long g_nn_launches = 0;

}  // namespace maple_nn

using namespace maple_nn;
static cudaStream_t Sx(maple_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }
#define NNL(launch)  \
  do {               \
    launch;          \
    ++g_nn_launches; \
  } while (0)

#define CKN(call)                                    \
  do {                                               \
    const cudaError_t e_ = (call);                   \
    if (e_ != cudaSuccess) return cudaGetErrorString(e_); \
  } while (0)

extern "C" {

const char* maple_nn_last_error_string(void) { return g_nn_err.c_str(); }
unsigned long long maple_nn_launch_count(void) { return g_nn_launches; }

int maple_nn_conv3d_padded(const void* in, const void* W, const float* bias, const void* res, void* out,
                           float* out_f32, int B, int n, int cin, int cout, int ksize, int relu, int padding,
                           maple_stream_t s) {
  return nn_guard([&]() -> const char* {
    if (!in || !W || (!out && !out_f32)) return "NULL argument";
    if (B < 1 || n < 1 || cin < 1 || cout < 1) return "bad sizes";
    if (ksize != 1 && ksize != 3) return "kernel size must be 1 or 3";
    if (padding != MAPLE_NN_PAD_CIRCULAR && padding != MAPLE_NN_PAD_ZEROS) return "unknown padding mode";
    if ((cin % 8) == 0 && (reinterpret_cast<uintptr_t>(in) & 15) != 0) return "input must be 16-byte aligned";
    const int N = n * n * n;
    const int taps = ksize == 3 ? 27 : 1, zp = padding == MAPLE_NN_PAD_ZEROS ? 1 : 0;
    if ((cin % 8) == 0 && (reinterpret_cast<uintptr_t>(W) & 15) == 0 && (long long)n * n * n < (1 << 24)) {
      // tensor-core (tcgen05) implicit GEMM
      const size_t smem = TC_STAGES * tc_stage_bytes(tc_bn(cout), tc_kc(cin));
      static bool attr_set[128] = {};
      int dev = 0;
      CKN(cudaGetDevice(&dev));
      if (dev >= 0 && dev < 128 && !attr_set[dev]) {
        CKN(cudaFuncSetAttribute(k_conv3d_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(TC_STAGES * tc_stage_bytes(TC_BN_MAX, TC_KC_MAX))));
        attr_set[dev] = true;
      }
      dim3 g((N + TC_BM - 1) / TC_BM, (cout + TC_BN_MAX - 1) / TC_BN_MAX, B);
      NNL((k_conv3d_tc<<<g, TC_THREADS, smem, Sx(s)>>>((const bf16*)in, (const bf16*)W, bias, (const bf16*)res,
                                                        (bf16*)out, out_f32, n, cin, cout, taps, relu, zp)));
      return nullptr;
    }
    // other channel counts: the warp-level MMA kernel
    dim3 g((N + BM - 1) / BM, (cout + BN - 1) / BN, B);
    NNL((k_conv3d<<<g, NT, 0, Sx(s)>>>((const bf16*)in, (const bf16*)W, bias, (const bf16*)res, (bf16*)out, out_f32,
                                       n, cin, cout, taps, relu, zp)));
    return nullptr;
  });
}

int maple_nn_conv3d(const void* in, const void* W, const float* bias, const void* res, void* out, float* out_f32,
                    int B, int n, int cin, int cout, int ksize, int relu, maple_stream_t s) {
  return maple_nn_conv3d_padded(in, W, bias, res, out, out_f32, B, n, cin, cout, ksize, relu, MAPLE_NN_PAD_CIRCULAR, s);
}

int maple_nn_wait_status(int* timed_out_host, maple_stream_t s) {
  return nn_guard([&]() -> const char* {
    if (!timed_out_host) return "NULL argument";
    int v = 0;
    CKN(cudaMemcpyFromSymbolAsync(&v, g_nn_wait_err, sizeof(int), 0, cudaMemcpyDeviceToHost, Sx(s)));
    CKN(cudaStreamSynchronize(Sx(s)));
    const int zero = 0;
    if (v) CKN(cudaMemcpyToSymbolAsync(g_nn_wait_err, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, Sx(s)));
    CKN(cudaStreamSynchronize(Sx(s)));
    *timed_out_host = v;
    return nullptr;
  });
}

int maple_nn_conv3d_wgrad(const void* in, const void* dz, float* dW, float* db, int B, int n, int cin, int cout,
                          int ksize, maple_stream_t s) {
  return nn_guard([&]() -> const char* {
    if (!in || !dz || !dW) return "NULL argument";
    if (B < 1 || n < 1 || cin < 1 || cout < 1) return "bad sizes";
    if (ksize != 1 && ksize != 3) return "kernel size must be 1 or 3";
    if ((cin % 8) == 0 && (reinterpret_cast<uintptr_t>(in) & 15) != 0) return "input must be 16-byte aligned";
    if ((cout % 8) == 0 && (reinterpret_cast<uintptr_t>(dz) & 15) != 0) return "gradient must be 16-byte aligned";
    const int N = n * n * n, taps = ksize == 3 ? 27 : 1;
    const long long total = (long long)B * N;
    if ((cin % 8) == 0 && (cout % 8) == 0 && n >= 4 && N < (1 << 24)) {
      // tensor-core (tcgen05) GEMM over the flat (tap, input channel) rows.
      // The reduction is split so that the CTAs fill whole waves of the 148
      // SMs (at the occupancy shared memory allows), each CTA reducing at
      // least 4096 (cell, voxel) pairs.
      const long long tiles = (long long)((taps * cin + WG_CI - 1) / WG_CI) * ((cout + TC_BN_MAX - 1) / TC_BN_MAX);
      const size_t smem = WG_STAGES * wg_stage_bytes(tc_bn(cout));
      const long long slots = 148LL * std::max(1, std::min(4, (int)(220 * 1024 / smem)));
      const long long smax = std::max(1LL, std::min(total / 4096, 8 * slots));
      long long splits = 1;
      double best = -1.0;
      for (long long sp = 1; sp <= smax; ++sp) {
        const long long ctas = tiles * sp, waves = (ctas + slots - 1) / slots;
        // fraction of the SM slots the last wave keeps busy, and whether the machine is full at all
        const double eff = (double)ctas / (double)(waves * slots) - (ctas < slots ? 1.0 : 0.0);
        if (eff > best + 0.05) {
          best = eff;
          splits = sp;
        }
      }
      long long chunk = (total + splits - 1) / splits;
      chunk = (chunk + WG_KP - 1) / WG_KP * WG_KP;
      splits = (total + chunk - 1) / chunk;
      static bool attr_set[128] = {};
      int dev = 0;
      CKN(cudaGetDevice(&dev));
      if (dev >= 0 && dev < 128 && !attr_set[dev]) {
        CKN(cudaFuncSetAttribute(k_conv3d_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(WG_STAGES * wg_stage_bytes(TC_BN_MAX))));
        attr_set[dev] = true;
      }
      dim3 g((unsigned)((taps * cin + WG_CI - 1) / WG_CI), (cout + TC_BN_MAX - 1) / TC_BN_MAX, (unsigned)splits);
      NNL((k_conv3d_wgrad_tc<<<g, WG_THREADS, smem, Sx(s)>>>((const bf16*)in, (const bf16*)dz, dW, B, n, cin, cout,
                                                             taps, chunk)));
      if (db) {
        dim3 gb((unsigned)std::min<long long>(512, (total + 7) / 8), (cout + 31) / 32);
        NNL((k_bias_grad<<<gb, 256, 0, Sx(s)>>>((const bf16*)dz, db, total, cout)));
      }
      return nullptr;
    }
    // other channel counts: the warp-level MMA kernel
    const long long tiles = (long long)taps * ((cin + BM - 1) / BM) * ((cout + BN - 1) / BN);
    // about 8 CTAs per SM, each reducing at least 1024 (cell, voxel) pairs
    long long splits = std::max(1LL, std::min((148LL * 8 + tiles - 1) / tiles, total / 1024));
    long long chunk = (total + splits - 1) / splits;
    chunk = (chunk + WK - 1) / WK * WK;
    splits = (total + chunk - 1) / chunk;
    dim3 g(taps * ((cin + BM - 1) / BM), (cout + BN - 1) / BN, (unsigned)splits);
    NNL((k_conv3d_wgrad<<<g, NT, 0, Sx(s)>>>((const bf16*)in, (const bf16*)dz, dW, B, n, cin, cout, taps, chunk)));
    if (db) {
      dim3 gb((unsigned)std::min<long long>(512, (total + 7) / 8), (cout + 31) / 32);
      NNL((k_bias_grad<<<gb, 256, 0, Sx(s)>>>((const bf16*)dz, db, total, cout)));
    }
    return nullptr;
  });
}

int maple_nn_flip_weights(const void* W, void* Wt, int cin, int cout, int ksize, maple_stream_t s) {
  return nn_guard([&]() -> const char* {
    if (!W || !Wt) return "NULL argument";
    if (ksize != 1 && ksize != 3) return "kernel size must be 1 or 3";
    const int taps = ksize == 3 ? 27 : 1;
    const size_t total = (size_t)taps * cin * cout;
    NNL((k_flip_weights<<<blocks(total), 256, 0, Sx(s)>>>((const bf16*)W, (bf16*)Wt, cin, cout, taps)));
    return nullptr;
  });
}

int maple_nn_resample(int op, const void* src, const void* base, void* dst, int B, int nc, int C, int add,
                      maple_stream_t s) {
  return nn_guard([&]() -> const char* {
    if (!src || !dst) return "NULL argument";
    if (B < 1 || nc < 1 || C < 1) return "bad sizes";
    const size_t Nc = (size_t)nc * nc * nc, Nf = Nc * 8;
    const bf16 *a = (const bf16*)src, *bs = (const bf16*)base;
    bf16* o = (bf16*)dst;
    switch (op) {
      case MAPLE_NN_POOL:
        NNL((k_fine_to_coarse<<<blocks((size_t)B * Nc * C), 256, 0, Sx(s)>>>(a, o, nc, C, B, 0.125f, add)));
        break;
      case MAPLE_NN_UPSAMPLE:
        NNL((k_coarse_to_fine<<<blocks((size_t)B * Nf * C), 256, 0, Sx(s)>>>(a, bs, o, nc, C, B, 1.0f, add)));
        break;
      case MAPLE_NN_UPSAMPLE_ADJ:
        NNL((k_fine_to_coarse<<<blocks((size_t)B * Nc * C), 256, 0, Sx(s)>>>(a, o, nc, C, B, 1.0f, add)));
        break;
      case MAPLE_NN_POOL_ADJ:
        NNL((k_coarse_to_fine<<<blocks((size_t)B * Nf * C), 256, 0, Sx(s)>>>(a, bs, o, nc, C, B, 0.125f, add)));
        break;
      default: return "unknown resample op";
    }
    return nullptr;
  });
}

int maple_nn_accumulate(void* dst, const void* src, size_t total, int add, maple_stream_t s) {
  return nn_guard([&]() -> const char* {
    if (!dst || !src) return "NULL argument";
    NNL((k_accumulate<<<blocks(total), 256, 0, Sx(s)>>>((bf16*)dst, (const bf16*)src, total, add)));
    return nullptr;
  });
}

int maple_nn_relu_mask(const void* y, void* g, size_t total, maple_stream_t s) {
  return nn_guard([&]() -> const char* {
    if (!y || !g) return "NULL argument";
    NNL((k_relu_mask<<<blocks(total), 256, 0, Sx(s)>>>((const bf16*)y, (bf16*)g, total)));
    return nullptr;
  });
}

int maple_nn_mse(const float* pred, const void* target, void* grad, float* loss, size_t total, float gscale,
                 maple_stream_t s) {
  return nn_guard([&]() -> const char* {
    if (!pred || !target || !loss) return "NULL argument";
    NNL((k_mse<<<blocks(total), 256, 0, Sx(s)>>>(pred, (const bf16*)target, (bf16*)grad, loss, total, gscale)));
    return nullptr;
  });
}

int maple_nn_node_weights(const double* rho, float* w, int B, int n, maple_stream_t s) {
  return nn_guard([&]() -> const char* {
    if (!rho || !w) return "NULL argument";
    if (B < 1 || n < 1) return "bad sizes";
    NNL((k_node_weights<<<B, 512, 0, Sx(s)>>>(rho, w, n)));
    return nullptr;
  });
}

int maple_nn_mse_weighted(const float* pred, const void* target, const float* w, float* ebar, void* grad, float* loss,
                          int B, int N, int C, float gscale, maple_stream_t s) {
  return nn_guard([&]() -> const char* {
    if (!pred || !target || !loss) return "NULL argument";
    if (B < 1 || N < 1 || C < 1 || C > 64) return "bad sizes (1 <= C <= 64)";
    if (ebar) {
      CKN(cudaMemsetAsync(ebar, 0, sizeof(float) * B * C, Sx(s)));
      const unsigned chunks = (unsigned)std::max<size_t>(1, std::min<size_t>(256, ((size_t)N * C) / 8192));
      NNL((k_weighted_error_mean<<<dim3(chunks, B), 256, 0, Sx(s)>>>(pred, (const bf16*)target, w, ebar, N, C)));
    }
    const size_t total = (size_t)B * N * C;
    NNL((k_mse_weighted<<<blocks(total), 256, 0, Sx(s)>>>(pred, (const bf16*)target, w, ebar, (bf16*)grad, loss, N, C,
                                                         total, gscale)));
    return nullptr;
  });
}

int maple_nn_error_fields(const float* pred, const void* target, const double* scale, double* e, int B, int N, int F,
                          int C, int c0, maple_stream_t s) {
  return nn_guard([&]() -> const char* {
    if (!pred || !target || !e) return "NULL argument";
    if (B < 1 || N < 1 || F < 1 || c0 < 0 || c0 + F > C) return "bad sizes";
    const size_t total = (size_t)B * F * N;
    NNL((k_error_fields<<<blocks(total), 256, 0, Sx(s)>>>(pred, (const bf16*)target, scale, e, N, F, C, c0, total)));
    return nullptr;
  });
}

int maple_nn_block_dot(const double* a, const double* b, double* out, int nblocks, size_t len, maple_stream_t s) {
  return nn_guard([&]() -> const char* {
    if (!a || !b || !out) return "NULL argument";
    if (nblocks < 1 || len < 1) return "bad sizes";
    NNL((k_block_dot<<<nblocks, 256, 0, Sx(s)>>>(a, b, out, len)));
    return nullptr;
  });
}

int maple_nn_energy_grad(const double* y, const double* norm, const double* scale, void* grad, int B, int N, int R,
                         int D, int C, int c0, double coef, maple_stream_t s) {
  return nn_guard([&]() -> const char* {
    if (!y || !norm || !grad) return "NULL argument";
    if (B < 1 || N < 1 || R < 1 || D < 1 || c0 < 0 || c0 + R * D > C) return "bad sizes";
    const size_t total = (size_t)B * R * D * N;
    NNL((k_energy_grad<<<blocks(total), 256, 0, Sx(s)>>>(y, norm, scale, (bf16*)grad, N, R, D, C, c0, coef, total)));
    return nullptr;
  });
}

int maple_nn_sumsq(const float* g, size_t n, double* out, maple_stream_t s) {
  return nn_guard([&]() -> const char* {
    if (!g || !out) return "NULL argument";
    CKN(cudaMemsetAsync(out, 0, sizeof(double), Sx(s)));
    const unsigned nb = (unsigned)std::max<size_t>(1, std::min<size_t>(1184, (n + 255) / 256));
    NNL((k_sumsq<<<nb, 256, 0, Sx(s)>>>(g, n, out)));
    return nullptr;
  });
}

int maple_nn_adam(float* w, const float* g, float* m, float* v, void* wb, size_t total, float lr, float b1, float b2,
                  float eps, float weight_decay, float gscale, int step, maple_stream_t s) {
  return nn_guard([&]() -> const char* {
    if (!w || !g || !m || !v) return "NULL argument";
    if (step < 1) return "step must be >= 1";
    if (!(gscale > 0)) return "gscale must be > 0";
    const float c1 = 1.0f - std::pow(b1, (float)step), c2 = 1.0f - std::pow(b2, (float)step);
    NNL((k_adam<<<blocks(total), 256, 0, Sx(s)>>>(w, g, m, v, (bf16*)wb, total, lr, b1, b2, eps, c1, c2,
                                                  1.0f / gscale, weight_decay)));
    return nullptr;
  });
}

int maple_nn_to_bf16(const float* src, void* dst, size_t total, maple_stream_t s) {
  return nn_guard([&]() -> const char* {
    if (!src || !dst) return "NULL argument";
    NNL((k_f32_to_bf16<<<blocks(total), 256, 0, Sx(s)>>>(src, (bf16*)dst, total)));
    return nullptr;
  });
}

int maple_nn_features(const double* rho, void* out, int B, int N, int C, maple_stream_t s) {
  return nn_guard([&]() -> const char* {
    if (!rho || !out) return "NULL argument";
    if (B < 1 || N < 1 || C < 1) return "bad sizes";
    const size_t total = (size_t)B * N;
    NNL((k_features<<<blocks(total), 256, 0, Sx(s)>>>(rho, (bf16*)out, total, C)));
    return nullptr;
  });
}

int maple_nn_fields_to_channels(const double* u, double* mean_work, void* out, int B, int N, int F, int C, int c0,
                                const double* scale, maple_stream_t s) {
  return nn_guard([&]() -> const char* {
    if (!u || !out) return "NULL argument";
    if (B < 1 || N < 1 || F < 1 || c0 < 0 || c0 + F > C) return "bad sizes";
    if (mean_work) NNL((k_field_mean<<<B * F, 256, 0, Sx(s)>>>(u, mean_work, N)));
    const size_t total = (size_t)B * F * N;
    NNL((k_fields_to_channels<<<blocks(total), 256, 0, Sx(s)>>>(u, mean_work, (bf16*)out, N, F, C, c0, scale,
                                                                 total)));
    return nullptr;
  });
}

int maple_nn_channels_to_fields(const float* in, double* u, int B, int N, int F, int C, int c0, const double* scale,
                                maple_stream_t s) {
  return nn_guard([&]() -> const char* {
    if (!in || !u) return "NULL argument";
    if (B < 1 || N < 1 || F < 1 || c0 < 0 || c0 + F > C) return "bad sizes";
    const size_t total = (size_t)B * F * N;
    NNL((k_channels_to_fields<<<blocks(total), 256, 0, Sx(s)>>>(in, u, N, F, C, c0, scale, total)));
    return nullptr;
  });
}

int maple_nn_prolong_fields(const double* uc, double* uf, int BF, int nc, int factor, maple_stream_t s) {
  return nn_guard([&]() -> const char* {
    if (!uc || !uf) return "NULL argument";
    if (BF < 1 || nc < 1 || factor < 1) return "bad sizes";
    const size_t nf = (size_t)nc * factor, total = (size_t)BF * nf * nf * nf;
    NNL((k_prolong_fields<<<blocks(total), 256, 0, Sx(s)>>>(uc, uf, nc, factor, total)));
    return nullptr;
  });
}

int maple_nn_restrict_density(const double* rf, double* rc, int B, int nc, int factor, maple_stream_t s) {
  return nn_guard([&]() -> const char* {
    if (!rf || !rc) return "NULL argument";
    if (B < 1 || nc < 1 || factor < 1) return "bad sizes";
    const size_t total = (size_t)B * nc * nc * nc;
    NNL((k_restrict_density<<<blocks(total), 256, 0, Sx(s)>>>(rf, rc, nc, factor, total)));
    return nullptr;
  });
}

}  // extern "C"
