// Inference kernels of the Stage-II conditional density generator
// (core/stage2/density_generator.py:123-197) and of the warm-start
// post-processing of the Pareto dataset worker
// (pareto/densify_pareto_property_network_32.py:1031-1053).
//
// The generator is condition MLP -> fc -> 4^3 x 128 seed volume -> three
// (trilinear x2 upsample, ConvBlock3d) levels -> 1x1 conv -> sigmoid.  Its
// 3x3x3 convolutions run on the BF16 tensor-core implicit GEMM of convnet.cu
// (maple_nn_conv3d_padded, zero padding); everything else is here, in FP32
// with FP64 reductions for the normalisation statistics:
//   k_linear          y = x W^T + b (nn.Linear, weight [out][in]), optional SiLU
//   k_layernorm       nn.LayerNorm over the last dim, optional SiLU
//   k_upsample2       nn.Upsample(scale 2, trilinear, align_corners=False),
//                     any input strides -> channels-last BF16 (the conv input)
//   k_group_stats /   nn.GroupNorm + SiLU on channels-last FP32 conv outputs,
//   k_group_apply     BF16 and/or FP32 results
//   k_head_sigmoid    1x1x1 conv to one channel + sigmoid
//   k_binomial_axis   one axis of the periodic [1 4 6 4 1]/16 smoothing, in
//                     the reference's operation order (bit-identical in FP32)
//   k_match_mean      the clamped mean correction, one CTA per cell
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>

#include "../../include/maple_b200.h"

namespace maple_gen {

using bf16 = __nv_bfloat16;

static thread_local std::string g_err;
static unsigned long long g_launches = 0;

__device__ __forceinline__ float silu(float v) { return v / (1.0f + expf(-v)); }

__device__ __forceinline__ double block_sum(double v, double* sm) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  __syncthreads();  // sm may still be read from a previous call
  if ((threadIdx.x & 31) == 0) sm[w] = v;
  __syncthreads();
  double s = 0.0;
  for (int i = 0; i < nw; ++i) s += sm[i];
  return s;  // every thread gets the sum
}

// one warp per (output feature, group of kRows rows): the weight row stays in L1
constexpr int kRows = 8;
__global__ void k_linear(const float* __restrict__ x, const float* __restrict__ W, const float* __restrict__ b,
                         float* __restrict__ y, int rows, int in, int out, int act) {
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int groups = (rows + kRows - 1) / kRows;
  if (warp >= (long long)out * groups) return;
  const int o = (int)(warp % out), r0 = (int)(warp / out) * kRows;
  const float* wr = W + (size_t)o * in;
  for (int r = r0; r < min(rows, r0 + kRows); ++r) {
    const float* xr = x + (size_t)r * in;
    float acc = 0.0f;
    for (int i = lane; i < in; i += 32) acc = fmaf(xr[i], wr[i], acc);
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if (lane == 0) {
      float v = acc + (b ? b[o] : 0.0f);
      if (act) v = silu(v);
      y[(size_t)r * out + o] = v;
    }
  }
}

// one CTA per row
__global__ void k_layernorm(const float* __restrict__ x, const float* __restrict__ g, const float* __restrict__ beta,
                            float* __restrict__ y, int dim, float eps, int act) {
  __shared__ double sm[32];
  const float* xr = x + (size_t)blockIdx.x * dim;
  float* yr = y + (size_t)blockIdx.x * dim;
  double s = 0.0;
  for (int i = threadIdx.x; i < dim; i += blockDim.x) s += xr[i];
  const double mean = block_sum(s, sm) / dim;
  double q = 0.0;
  for (int i = threadIdx.x; i < dim; i += blockDim.x) {
    const double d = xr[i] - mean;
    q += d * d;
  }
  const double var = block_sum(q, sm) / dim;
  const float rstd = (float)(1.0 / sqrt(var + (double)eps)), m = (float)mean;
  for (int i = threadIdx.x; i < dim; i += blockDim.x) {
    float v = (xr[i] - m) * rstd;
    if (g) v = v * g[i];
    if (beta) v = v + beta[i];
    if (act) v = silu(v);
    yr[i] = v;
  }
}

// source index and weights of align_corners=False linear interpolation at
// scale 2: src = max(0, (o + 0.5) / 2 - 0.5)
__device__ __forceinline__ void lin_src(int o, int n, int& i0, int& step, float& l0, float& l1) {
  float src = 0.5f * ((float)o + 0.5f) - 0.5f;
  if (src < 0.0f) src = 0.0f;
  i0 = min((int)floorf(src), n - 1);
  step = i0 < n - 1 ? 1 : 0;
  l1 = fminf(fmaxf(src - (float)i0, 0.0f), 1.0f);
  l0 = 1.0f - l1;
}

// out[b][vo][c] (fine grid 2n, channels-last BF16) from in[b*cs_b + v*vs + c*cs]
__global__ void k_upsample2(const float* __restrict__ in, long long bs, long long vs, long long cs,
                            bf16* __restrict__ out, int n, int C, long long total) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int m = 2 * n;
  const long long No = (long long)m * m * m;
  const int c = (int)(i % C);
  const long long vo = (i / C) % No;
  const long long b = i / (C * No);
  const int oz = (int)(vo % m), oy = (int)((vo / m) % m), ox = (int)(vo / ((long long)m * m));
  int x0, xs, y0, ys, z0, zs;
  float tx0, tx1, ty0, ty1, tz0, tz1;
  lin_src(ox, n, x0, xs, tx0, tx1);
  lin_src(oy, n, y0, ys, ty0, ty1);
  lin_src(oz, n, z0, zs, tz0, tz1);
  const float* p = in + b * bs + (long long)c * cs;
  auto at = [&](int x, int y, int z) { return p[((long long)(x * n + y) * n + z) * vs]; };
  const float v = tx0 * (ty0 * (tz0 * at(x0, y0, z0) + tz1 * at(x0, y0, z0 + zs)) +
                         ty1 * (tz0 * at(x0, y0 + ys, z0) + tz1 * at(x0, y0 + ys, z0 + zs))) +
                  tx1 * (ty0 * (tz0 * at(x0 + xs, y0, z0) + tz1 * at(x0 + xs, y0, z0 + zs)) +
                         ty1 * (tz0 * at(x0 + xs, y0 + ys, z0) + tz1 * at(x0 + xs, y0 + ys, z0 + zs)));
  out[i] = __float2bfloat16(v);
}

// stats[(b*G+g)*2 + {0,1}] = mean, 1/sqrt(var + eps) of the group's channels over all voxels
__global__ void k_group_stats(const float* __restrict__ x, double* __restrict__ stats, long long N, int C, int G,
                              double eps) {
  __shared__ double sm[32];
  const int b = blockIdx.x / G, g = blockIdx.x % G, cg = C / G;
  const float* xb = x + (size_t)b * N * C + (size_t)g * cg;
  const long long cnt = N * cg;
  double s = 0.0;
  for (long long e = threadIdx.x; e < cnt; e += blockDim.x) s += xb[(e / cg) * C + e % cg];
  const double mean = block_sum(s, sm) / (double)cnt;
  double q = 0.0;
  for (long long e = threadIdx.x; e < cnt; e += blockDim.x) {
    const double d = xb[(e / cg) * C + e % cg] - mean;
    q += d * d;
  }
  const double var = block_sum(q, sm) / (double)cnt;
  if (threadIdx.x == 0) {
    stats[2 * blockIdx.x] = mean;
    stats[2 * blockIdx.x + 1] = 1.0 / sqrt(var + eps);
  }
}

__global__ void k_group_apply(const float* __restrict__ x, const double* __restrict__ stats,
                              const float* __restrict__ gamma, const float* __restrict__ beta, bf16* __restrict__ ob,
                              float* __restrict__ of, long long N, int C, int G, int act, long long total) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int c = (int)(i % C);
  const long long b = i / (N * C);
  const int g = c / (C / G);
  const double* st = stats + 2 * (b * G + g);
  float v = (x[i] - (float)st[0]) * (float)st[1];
  if (gamma) v = v * gamma[c];
  if (beta) v = v + beta[c];
  if (act) v = silu(v);
  if (ob) ob[i] = __float2bfloat16(v);
  if (of) of[i] = v;
}

__global__ void k_head_sigmoid(const float* __restrict__ x, const float* __restrict__ w, float bias,
                               float* __restrict__ out, int C, long long total) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const float* xr = x + i * C;
  float acc = 0.0f;
  for (int c = 0; c < C; ++c) acc = fmaf(w[c], xr[c], acc);
  out[i] = 1.0f / (1.0f + expf(-(acc + bias)));
}

// out = sum_k w_k * roll(in, s_k, axis) for s = -2..2, w = [1 4 6 4 1] / 16,
// accumulated from zero in that order with separately rounded products and
// sums (roll(in, s)[i] = in[i - s], periodic)
__global__ void k_binomial_axis(const float* __restrict__ in, float* __restrict__ out, int n, int axis,
                                long long total) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const long long N = (long long)n * n * n;
  const long long v = i % N;
  const int z = (int)(v % n), y = (int)((v / n) % n), x = (int)(v / ((long long)n * n));
  const int c = axis == 0 ? x : (axis == 1 ? y : z);
  const long long stride = axis == 0 ? (long long)n * n : (axis == 1 ? n : 1);
  const float* row = in + (i - (long long)c * stride);
  const float w[5] = {0.0625f, 0.25f, 0.375f, 0.25f, 0.0625f};
  float acc = 0.0f;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const int s = k - 2;
    const int src = ((c - s) % n + n) % n;
    acc = __fadd_rn(acc, __fmul_rn(w[k], row[(long long)src * stride]));
  }
  out[i] = acc;
}

// per cell: iters times x <- clamp(x - mean(x) + target, lo, hi), FP32 values, FP64 mean
__global__ void k_match_mean(float* __restrict__ x, const double* __restrict__ target, long long N, float lo,
                             float hi, int iters) {
  __shared__ double sm[32];
  float* xb = x + (size_t)blockIdx.x * N;
  const float t = (float)fmin(fmax(target[blockIdx.x], (double)lo), (double)hi);
  for (int it = 0; it < iters; ++it) {
    double s = 0.0;
    for (long long e = threadIdx.x; e < N; e += blockDim.x) s += xb[e];
    const float m = (float)(block_sum(s, sm) / (double)N);
    for (long long e = threadIdx.x; e < N; e += blockDim.x)
      xb[e] = fminf(fmaxf(__fadd_rn(__fsub_rn(xb[e], m), t), lo), hi);
    __syncthreads();
  }
}

template <typename F>
static int guard(F&& f) {
  const char* msg = f();
  if (msg) {
    g_err = msg;
    return MAPLE_E_BADARG;
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    g_err = std::string("CUDA error: ") + cudaGetErrorString(e);
    return MAPLE_E_CUDA;
  }
  return MAPLE_OK;
}

static inline unsigned nblk(long long n, int t = 256) { return (unsigned)((n + t - 1) / t); }
static inline cudaStream_t S(maple_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

}  // namespace maple_gen

using namespace maple_gen;
#define GL(launch) \
  do {             \
    launch;        \
    ++g_launches;  \
  } while (0)

extern "C" {

const char* maple_gen_last_error_string(void) { return g_err.c_str(); }
unsigned long long maple_gen_launch_count(void) { return g_launches; }

int maple_gen_linear(const float* x, const float* W, const float* b, float* y, int rows, int in, int out, int act,
                     maple_stream_t s) {
  return guard([&]() -> const char* {
    if (!x || !W || !y) return "NULL argument";
    if (rows < 1 || in < 1 || out < 1) return "bad sizes";
    const long long warps = (long long)out * ((rows + kRows - 1) / kRows);
    GL((k_linear<<<nblk(warps * 32), 256, 0, S(s)>>>(x, W, b, y, rows, in, out, act ? 1 : 0)));
    return nullptr;
  });
}

int maple_gen_layernorm(const float* x, const float* gamma, const float* beta, float* y, int rows, int dim, float eps,
                        int act, maple_stream_t s) {
  return guard([&]() -> const char* {
    if (!x || !y) return "NULL argument";
    if (rows < 1 || dim < 1 || !(eps > 0.0f)) return "bad sizes";
    GL((k_layernorm<<<rows, 256, 0, S(s)>>>(x, gamma, beta, y, dim, eps, act ? 1 : 0)));
    return nullptr;
  });
}

int maple_gen_upsample2(const float* in, long long cell_stride, long long voxel_stride, long long channel_stride,
                        void* out, int B, int n, int C, maple_stream_t s) {
  return guard([&]() -> const char* {
    if (!in || !out) return "NULL argument";
    if (B < 1 || n < 1 || C < 1 || voxel_stride < 1 || channel_stride < 1 || cell_stride < 1) return "bad sizes";
    const long long total = (long long)B * 8LL * n * n * n * C;
    GL((k_upsample2<<<nblk(total), 256, 0, S(s)>>>(in, cell_stride, voxel_stride, channel_stride, (bf16*)out, n, C,
                                                     total)));
    return nullptr;
  });
}

int maple_gen_groupnorm(const float* x, const float* gamma, const float* beta, int groups, float eps, int act,
                        void* out_bf16, float* out_f32, double* stats, int B, long long N, int C, maple_stream_t s) {
  return guard([&]() -> const char* {
    if (!x || !stats || (!out_bf16 && !out_f32)) return "NULL argument";
    if (B < 1 || N < 1 || C < 1 || groups < 1 || C % groups != 0 || !(eps > 0.0f)) return "bad sizes";
    GL((k_group_stats<<<B * groups, 512, 0, S(s)>>>(x, stats, N, C, groups, (double)eps)));
    const long long total = (long long)B * N * C;
    GL((k_group_apply<<<nblk(total), 256, 0, S(s)>>>(x, stats, gamma, beta, (bf16*)out_bf16, out_f32, N, C, groups,
                                                       act ? 1 : 0, total)));
    return nullptr;
  });
}

int maple_gen_head_sigmoid(const float* x, const float* w, float bias, float* out, int B, long long N, int C,
                           maple_stream_t s) {
  return guard([&]() -> const char* {
    if (!x || !w || !out) return "NULL argument";
    if (B < 1 || N < 1 || C < 1) return "bad sizes";
    const long long total = (long long)B * N;
    GL((k_head_sigmoid<<<nblk(total), 256, 0, S(s)>>>(x, w, bias, out, C, total)));
    return nullptr;
  });
}

int maple_gen_binomial_smooth(const float* in, float* out, float* work, int B, int n, int passes, maple_stream_t s) {
  return guard([&]() -> const char* {
    if (!in || !out) return "NULL argument";
    if (B < 1 || n < 1 || passes < 0) return "bad sizes";
    const long long total = (long long)B * n * n * n;
    if (passes == 0) {
      if (in != out) {
        const cudaError_t e = cudaMemcpyAsync(out, in, (size_t)total * sizeof(float), cudaMemcpyDeviceToDevice, S(s));
        if (e != cudaSuccess) return cudaGetErrorString(e);
      }
      return nullptr;
    }
    if (!work) return "NULL work buffer";
    if (in == out || in == work || out == work) return "in, out and work must be distinct buffers";
    const int L = 3 * passes;
    const float* src = in;
    for (int k = 0; k < L; ++k) {
      float* dst = ((L - 1 - k) % 2 == 0) ? out : work;
      GL((k_binomial_axis<<<nblk(total), 256, 0, S(s)>>>(src, dst, n, k % 3, total)));
      src = dst;
    }
    return nullptr;
  });
}

int maple_gen_match_mean(float* x, const double* target, int B, long long N, float lo, float hi, int iters,
                         maple_stream_t s) {
  return guard([&]() -> const char* {
    if (!x || !target) return "NULL argument";
    if (B < 1 || N < 1 || !(lo <= hi)) return "bad sizes";
    GL((k_match_mean<<<B, 1024, 0, S(s)>>>(x, target, N, lo, hi, std::max(1, iters))));
    return nullptr;
  });
}

}  // extern "C"
