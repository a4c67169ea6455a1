// sm_100a kernels for the periodic voxel homogenization path.
//
// Data layout (one "cell" = one periodic r^3 unit cell; B cells per context):
//   * element / node id  x*n*n + y*n + z (maple/core/main_IHD_v3.py:175-186)
//   * vectors: [cell][rhs][comp][node]  (component-major: a warp's accesses to
//     consecutive nodes are contiguous for every load case and component)
//   * coarse stencils: [cell][27][D*D][node]  (node fastest: coalesced)
//   * element matrices of coarse levels: [cell][elem][8D][8D]  (FP64)
// The element stiffness of the fine level lives in __constant__ memory for a
// voxel of edge 1; every kernel multiplies by the context's scale factor.
#pragma once
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <utility>

namespace maple {

constexpr int kThreads = 256;
constexpr int TX = 4, TY = 8, TZ = 8;  // fine-level node tile per CTA (z fastest)
constexpr int kFineThreads = TX * TY * TZ;

__constant__ double c_Ke3d[576];
__constant__ float c_Ke3f[576];
__constant__ double c_Ke1d[64];
__constant__ float c_Ke1f[64];
__constant__ double c_Fe3[144];
__constant__ double c_X03[144];
__constant__ double c_KX3[144];
__constant__ double c_Fe1[24];
__constant__ double c_X01[24];
__constant__ double c_KX1[24];
__constant__ double c_W[512];

template <typename T, int D>
__device__ __forceinline__ T ke(int i, int j);
template <>
__device__ __forceinline__ double ke<double, 3>(int i, int j) { return c_Ke3d[i * 24 + j]; }
template <>
__device__ __forceinline__ float ke<float, 3>(int i, int j) { return c_Ke3f[i * 24 + j]; }
template <>
__device__ __forceinline__ double ke<double, 1>(int i, int j) { return c_Ke1d[i * 8 + j]; }
template <>
__device__ __forceinline__ float ke<float, 1>(int i, int j) { return c_Ke1f[i * 8 + j]; }

template <int D>
__device__ __forceinline__ double fe(int i, int r) { return D == 3 ? c_Fe3[i * 6 + r] : c_Fe1[i * 3 + r]; }
template <int D>
__device__ __forceinline__ double x0(int i, int r) { return D == 3 ? c_X03[i * 6 + r] : c_X01[i * 3 + r]; }
template <int D>
__device__ __forceinline__ double kx(int i, int r) { return D == 3 ? c_KX3[i * 6 + r] : c_KX1[i * 3 + r]; }

// element-local corner index of corner bits (cx,cy,cz): 000,100,110,010,001,101,111,011
__host__ __device__ constexpr int lidx(int cx, int cy, int cz) { return cz * 4 + (cy ? (cx ? 2 : 3) : (cx ? 1 : 0)); }
__host__ __device__ constexpr int corner_x(int a) { return (a == 1 || a == 2 || a == 5 || a == 6) ? 1 : 0; }
__host__ __device__ constexpr int corner_y(int a) { return (a == 2 || a == 3 || a == 6 || a == 7) ? 1 : 0; }
__host__ __device__ constexpr int corner_z(int a) { return a >= 4 ? 1 : 0; }

__device__ __forceinline__ int wrapn(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// Programmatic dependent launch (sm_90+).  A kernel launched with the
// programmatic-serialization attribute may start while its predecessor in the
// stream still runs; griddep_wait() returns once every prerequisite grid has
// completed and its memory operations are visible.  Kernels that use these
// call griddep_wait() in every thread before reading anything an earlier
// kernel of the solve wrote, and before returning, so completion stays
// transitive along the stream; only data written before the solve (stencils,
// block inverses, bounds) is read before it, and data written during the
// solve is read with coherent (not read-only-path) loads.  griddep_launch(),
// called after the wait, lets the next launch begin its own prologue, so at
// most two kernels of a stream overlap.  Without the attribute both are
// no-ops.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Explicitly rounded arithmetic (CUDA's _rn intrinsics): the compiler may not
// contract or split these, so two kernels written with them round alike.  The
// coarse-level nine-thread kernel, the grid transfers, the coarsest solve and
// the fused V-cycle tail use them, and the tail reproduces the separate
// launches bit for bit.
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

// ----------------------------------------------------------------------------
// block reductions (deterministic: fixed shuffle tree + fixed warp order)
// ----------------------------------------------------------------------------
template <int K, int NWARP = kThreads / 32>
__device__ __forceinline__ void block_sum_store(double (&v)[K], double* out) {
  __shared__ double sm[NWARP][K];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], off);
  }
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) sm[warp][k] = v[k];
  }
  __syncthreads();
  if (threadIdx.x < K) {
    double s = 0;
#pragma unroll
    for (int w = 0; w < NWARP; ++w) s += sm[w][threadIdx.x];
    out[threadIdx.x] = s;
  }
}

__device__ __forceinline__ double block_max(double v) {
  __shared__ double sm[kThreads / 32];
  __shared__ double res;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
  if (lane == 0) sm[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = sm[0];
    for (int w = 1; w < kThreads / 32; ++w) m = fmax(m, sm[w]);
    res = m;
  }
  __syncthreads();
  return res;
}

// sum part[cell][0..nblk)[K] -> out[cell][K]; one block per cell, fixed order
template <int K>
__global__ void k_reduce_partials(const double* __restrict__ part, int nblk, double* __restrict__ out) {
  const int b = blockIdx.x;
  double v[K];
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = 0;
  for (int i = threadIdx.x; i < nblk; i += kThreads) {
    const double* p = part + ((size_t)b * nblk + i) * K;
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] += p[k];
  }
  block_sum_store<K>(v, out + (size_t)b * K);
}

// ----------------------------------------------------------------------------
// small dense helpers
// ----------------------------------------------------------------------------
template <typename T, int D>
__device__ __forceinline__ void block_inverse(const T (&A)[D][D], T (&Ai)[D][D]) {
  if constexpr (D == 1) {
    Ai[0][0] = A[0][0] != T(0) ? T(1) / A[0][0] : T(1);
  } else {
    T c00 = A[1][1] * A[2][2] - A[1][2] * A[2][1];
    T c01 = A[1][2] * A[2][0] - A[1][0] * A[2][2];
    T c02 = A[1][0] * A[2][1] - A[1][1] * A[2][0];
    T det = A[0][0] * c00 + A[0][1] * c01 + A[0][2] * c02;
    if (det == T(0)) {
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Ai[i][j] = (i == j) ? T(1) : T(0);
      return;
    }
    T id = T(1) / det;
    Ai[0][0] = c00 * id;
    Ai[1][0] = c01 * id;
    Ai[2][0] = c02 * id;
    Ai[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) * id;
    Ai[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) * id;
    Ai[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) * id;
    Ai[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) * id;
    Ai[1][2] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) * id;
    Ai[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) * id;
  }
}

// Chebyshev step coefficients on [hi/ratio, hi]: step 0 -> (0, 1/theta);
// step k -> (rho_k rho_{k-1}, 2 rho_k / delta).
__device__ __forceinline__ void cheb_coeffs(double hi, double ratio, int step, double& alpha, double& beta) {
  const double lo = hi / ratio;
  const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo);
  const double sigma = theta / delta;
  if (step == 0) {
    alpha = 0.0;
    beta = 1.0 / theta;
    return;
  }
  double rp = 1.0 / sigma, rk = rp;
  for (int k = 1; k <= step; ++k) {
    rk = 1.0 / (2.0 * sigma - rp);
    if (k < step) rp = rk;
  }
  alpha = rk * rp;
  beta = 2.0 * rk / delta;
}

// ----------------------------------------------------------------------------
// operator application: fine level (matrix-free from rho) and coarse levels
// (stored 27-point stencils)
// ----------------------------------------------------------------------------
enum ApplyMode { M_MV = 0, M_RES = 1, M_CHEB = 2, M_JAC0 = 3, M_POWER = 4 };

// 16-byte vector type of T and its width (vectorised vector kernels)
template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
  using type = float4;
  static constexpr int n = 4;
};
template <>
struct Vec16<double> {
  using type = double2;
  static constexpr int n = 2;
};

template <typename T>
struct ApplyArgs {
  int n, N;
  T scale;                 // fine level: stiffness scale (E/r or kappa/r)
  const T* rho;            // fine level densities [B][N]
  const T* S;              // coarse stencils [B][27][D*D][N]
  const T* Dinv;           // coarse block-diagonal inverses [B][D*D][N]
  const T* u;              // input iterate
  const T* f;              // right-hand side (RES, CHEB, JAC0)
  const T* din;            // Chebyshev direction in (may alias dout)
  T* dout;                 // Chebyshev direction out
  T* out;                  // MV/RES/POWER output, CHEB/JAC0 new iterate
  const double* hi;        // per-cell Chebyshev upper bound (CHEB, JAC0)
  double cheb_al, cheb_be; // this block's step coefficients (set inside the kernels)
  double ratio;            // Chebyshev interval ratio hi/lo
  int step;                // Chebyshev step index
  double* part;            // per-block partial dots [B][nblk][R or 2] (nullable)
  int dot_f_out;           // CHEB: partial sum of f.out (PCG r.z) instead of nothing
  const int* active;       // per-cell flag (nullable)
};

// Loads the 8 element densities around node (x,y,z): element q = 4qx+2qy+qz at
// offset (qx-1, qy-1, qz-1).
template <typename T>
__device__ __forceinline__ void load_rho8(const T* __restrict__ rho, int n, int x, int y, int z, T (&rq)[8]) {
  const int xs[2] = {wrapn(x - 1, n), x}, ys[2] = {wrapn(y - 1, n), y}, zs[2] = {wrapn(z - 1, n), z};
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int qx = (q >> 2) & 1, qy = (q >> 1) & 1, qz = q & 1;
    rq[q] = __ldg(rho + ((size_t)xs[qx] * n + ys[qy]) * n + zs[qz]);
  }
}

// Assembled 3x3 (or 1x1) coupling block between node n and n+o on the fine
// level: sum over the elements sharing both nodes of rho_e * Ke0 block.
template <typename T, int D, int O>
__device__ __forceinline__ void fine_block(const T (&rq)[8], T (&C)[D][D]) {
  constexpr int ox = O / 9 - 1, oy = (O / 3) % 3 - 1, oz = O % 3 - 1;
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) C[i][j] = T(0);
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int qx = (q >> 2) & 1, qy = (q >> 1) & 1, qz = q & 1;
    const int cx = 1 - qx, cy = 1 - qy, cz = 1 - qz;
    const int nx = cx + ox, ny = cy + oy, nz = cz + oz;
    if (nx < 0 || nx > 1 || ny < 0 || ny > 1 || nz < 0 || nz > 1) continue;
    const int a = lidx(cx, cy, cz), bb = lidx(nx, ny, nz);
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) C[i][j] += rq[q] * ke<T, D>(D * a + i, D * bb + j);
  }
}

template <typename T, int D, int R, int O>
__device__ __forceinline__ void fine_accumulate(const T (&rq)[8], const T* __restrict__ u, size_t cell_off, int n,
                                                const int (&xs)[3], const int (&ys)[3], const int (&zs)[3],
                                                T (&acc)[R][D], T (&C0)[D][D]) {
  T C[D][D];
  fine_block<T, D, O>(rq, C);
  constexpr int ox = O / 9, oy = (O / 3) % 3, oz = O % 3;
  const T* __restrict__ un = u + (cell_off + ((size_t)xs[ox] * n + ys[oy]) * n + zs[oz]) * (R * D);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    T uv[D];
#pragma unroll
    for (int j = 0; j < D; ++j) uv[j] = __ldg(un + r * D + j);
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) acc[r][i] += C[i][j] * uv[j];
  }
  if constexpr (O == 13) {
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) C0[i][j] = C[i][j];
  }
}

template <typename T, int D, int R, int... Os>
__device__ __forceinline__ void fine_all(std::integer_sequence<int, Os...>, const T (&rq)[8], const T* __restrict__ u,
                                         size_t cell_off, int n, const int (&xs)[3], const int (&ys)[3],
                                         const int (&zs)[3], T (&acc)[R][D], T (&C0)[D][D]) {
  (fine_accumulate<T, D, R, Os>(rq, u, cell_off, n, xs, ys, zs, acc, C0), ...);
}

template <typename T, int RD>
struct FineTile {
  // Vector width (elements of T) of shared-memory reads and async copies:
  // pairs (8 B for float, 16 B for double) when a node holds an even count.
  static constexpr int VW = (RD % 2 == 0) ? 2 : 1;
  static constexpr int NS = RD;                            // node stride (T)
  static constexpr int ROW0 = (TZ + 2) * NS;
  // Row stride: warp lanes are (tz 0..7, ty 0..3).  Scalar reads need
  // RW = 8*NS (mod 32 banks, 16 for double) with NS odd; float2 reads are
  // issued per half-warp and need RW = 8*NS (mod 32); double2 reads per
  // quarter-warp are conflict-free for any even RW.
  static constexpr int MOD = (VW == 2 && sizeof(T) == 8) ? 2 : (sizeof(T) == 8 ? 16 : 32);
  static constexpr int WANT = (VW == 2 && sizeof(T) == 8) ? 0 : (8 * NS) % MOD;
  static constexpr int RW = ROW0 + ((WANT - ROW0 % MOD) % MOD + MOD) % MOD;
  static constexpr int HALO_NODES = (TX + 2) * (TY + 2) * (TZ + 2);
  static constexpr int U_WORDS = (TX + 2) * (TY + 2) * RW;
  static constexpr int RHO_WORDS = (TX + 1) * (TY + 1) * (TZ + 1);
  static constexpr int RHO_OFF = (U_WORDS + 1) / 2 * 2;     // keep rho 8/16-byte aligned
  static constexpr size_t BYTES = (size_t)(RHO_OFF + RHO_WORDS) * sizeof(T);
  static_assert(RW % MOD == WANT, "row padding");
  static_assert(VW == 1 || (NS % 2 == 0 && RW % 2 == 0), "vector alignment");
};

template <typename T>
struct Vec2;
template <>
struct Vec2<float> {
  using type = float2;
};
template <>
struct Vec2<double> {
  using type = double2;
};

// asynchronous global -> shared copy of BYTES (4, 8 or 16) bytes
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem_dst, const void* gsrc) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(sa), "l"(gsrc), "n"(BYTES));
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n" ::);
  asm volatile("cp.async.wait_group 0;\n" ::);
}

template <typename T, int RD, int VW>
__device__ __forceinline__ void lds_node(const T* __restrict__ p, T (&v)[RD]) {
  if constexpr (VW == 2) {
    using V = typename Vec2<T>::type;
#pragma unroll
    for (int i = 0; i < RD / 2; ++i) {
      const V t = reinterpret_cast<const V*>(p)[i];
      v[2 * i] = t.x;
      v[2 * i + 1] = t.y;
    }
  } else {
#pragma unroll
    for (int i = 0; i < RD; ++i) v[i] = p[i];
  }
}

// Packed FP32 pairs (two lanes of one 64-bit register) for fma.rn.f32x2: each
// lane is rounded exactly like a scalar fma.rn.f32.
__device__ __forceinline__ unsigned long long pk2(float a, float b) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void upk2(unsigned long long v, float& a, float& b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ unsigned long long ffma2(unsigned long long a, unsigned long long b, unsigned long long c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// The FP32 elastic operator (D = 3, R = 6) stages a node's values
// component-major ([j][r]) so that load cases 2m, 2m+1 of one component are
// adjacent: one 64-bit shared load gives a packed pair, and one fma.rn.f32x2
// applies a coupling entry to both.  Every accumulator sums its terms in the
// same (offset, j) order as the scalar form, so the results are identical.
template <typename T, int D, int R>
__host__ __device__ constexpr bool fine_packed() {
  return sizeof(T) == 4 && D == 3 && R == 6;
}

template <int RW, int NS, int O>
__device__ __forceinline__ void fine_tile_accumulate_pk(const float (&rq)[8], const float* __restrict__ base,
                                                        unsigned long long (&acc2)[3][3], float (&C0)[3][3]) {
  float C[3][3];
  fine_block<float, 3, O>(rq, C);
  constexpr int ox = O / 9, oy = (O / 3) % 3, oz = O % 3;
  const float* un = base + (ox * (TY + 2) + oy) * RW + oz * NS;
  unsigned long long u2[3][3];  // [j][m]: load cases 2m, 2m+1 of component j
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int m = 0; m < 3; ++m) u2[j][m] = reinterpret_cast<const unsigned long long*>(un + j * 6)[m];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const unsigned long long cc = pk2(C[i][j], C[i][j]);
#pragma unroll
      for (int m = 0; m < 3; ++m) acc2[m][i] = ffma2(cc, u2[j][m], acc2[m][i]);
    }
  if constexpr (O == 13) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) C0[i][j] = C[i][j];
  }
}

template <int RW, int NS, int... Os>
__device__ __forceinline__ void fine_tile_all_pk(std::integer_sequence<int, Os...>, const float (&rq)[8],
                                                 const float* __restrict__ base, unsigned long long (&acc2)[3][3],
                                                 float (&C0)[3][3]) {
  (fine_tile_accumulate_pk<RW, NS, Os>(rq, base, acc2, C0), ...);
}

template <typename T, int D, int R, int RW, int NS, int O>
__device__ __forceinline__ void fine_tile_accumulate(const T (&rq)[8], const T* __restrict__ base, T (&acc)[R][D],
                                                     T (&C0)[D][D]) {
  T C[D][D];
  fine_block<T, D, O>(rq, C);
  constexpr int ox = O / 9, oy = (O / 3) % 3, oz = O % 3;
  const T* un = base + (ox * (TY + 2) + oy) * RW + oz * NS;
  T uv[R * D];
  lds_node<T, R * D, (R * D) % 2 == 0 ? 2 : 1>(un, uv);
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) acc[r][i] += C[i][j] * uv[r * D + j];
  if constexpr (O == 13) {
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) C0[i][j] = C[i][j];
  }
}

template <typename T, int D, int R, int RW, int NS, int... Os>
__device__ __forceinline__ void fine_tile_all(std::integer_sequence<int, Os...>, const T (&rq)[8],
                                              const T* __restrict__ base, T (&acc)[R][D], T (&C0)[D][D]) {
  (fine_tile_accumulate<T, D, R, RW, NS, Os>(rq, base, acc, C0), ...);
}

// Shared epilogue of both apply kernels.
// vo = cell*R*D*N + node; component (r, i) lives at vo + (r*D + i) * N.
// uown (nullable) holds the node's own values at uown[(r*D + i) * uown_stride],
// or at uown[(i*R + r) * uown_stride] when CM (component-major staging).
template <typename T, int D, int R, int MODE, int NWARP = kThreads / 32, bool CM = false>
__device__ __forceinline__ void apply_epilogue(const ApplyArgs<T>& a, int b, size_t vo, bool valid, T (&acc)[R][D],
                                               const T (&Di)[D][D], const T* uown = nullptr, size_t uown_stride = 0) {
  const size_t NN = (size_t)a.N;
  auto own = [&](int r, int i) { return uown[(CM ? i * R + r : r * D + i) * uown_stride]; };
  constexpr int K = R;
  double dots[K];
#pragma unroll
  for (int k = 0; k < K; ++k) dots[k] = 0;
  if (valid) {
    if constexpr (MODE == M_MV) {
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int i = 0; i < D; ++i) {
          const T y = a.scale * acc[r][i];
          a.out[vo + (size_t)(r * D + i) * NN] = y;
          if (a.part)
            dots[r] += (double)y * (double)(uown ? own(r, i) : a.u[vo + (size_t)(r * D + i) * NN]);
        }
    } else if constexpr (MODE == M_RES) {
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int i = 0; i < D; ++i) {
          const T y = a.f[vo + (size_t)(r * D + i) * NN] - a.scale * acc[r][i];
          a.out[vo + (size_t)(r * D + i) * NN] = y;
          dots[r] += (double)y * (double)y;
        }
    } else if constexpr (MODE == M_CHEB || MODE == M_JAC0) {
      const double al = a.cheb_al, be = a.cheb_be;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        T res[D];
#pragma unroll
        for (int i = 0; i < D; ++i) {
          if constexpr (MODE == M_JAC0)
            res[i] = a.f[vo + (size_t)(r * D + i) * NN];
          else
            res[i] = a.f[vo + (size_t)(r * D + i) * NN] - a.scale * acc[r][i];
        }
#pragma unroll
        for (int i = 0; i < D; ++i) {
          T z = 0;
#pragma unroll
          for (int j = 0; j < D; ++j) z += Di[i][j] * res[j];
          T d = T(be) * z;
          if (MODE == M_CHEB && al != 0.0) d += T(al) * a.din[vo + (size_t)(r * D + i) * NN];
          a.dout[vo + (size_t)(r * D + i) * NN] = d;
          const T uo = uown ? own(r, i) : a.u[vo + (size_t)(r * D + i) * NN];
          const T un = (MODE == M_JAC0) ? d : uo + d;
          a.out[vo + (size_t)(r * D + i) * NN] = un;
          if (a.dot_f_out) dots[r] += (double)a.f[vo + (size_t)(r * D + i) * NN] * (double)un;
        }
      }
    }
  }
  if (a.part && (MODE != M_CHEB || a.dot_f_out)) {
    block_sum_store<K, NWARP>(dots, a.part + ((size_t)b * gridDim.x + blockIdx.x) * K);
  }
}

// ---------------------------------------------------------------------------
// Fine-level tile geometry: a CTA owns TX x TY x TZ nodes (z fastest, 256
// threads) and stages the (TX+2)(TY+2)(TZ+2) halo'd nodes' R*D values in
// shared memory.  Node stride NS is odd and each (x,y) row is padded so that
// the 32 lanes of a warp (tz 0..7, ty 0..3) hit 32 distinct banks.
// ---------------------------------------------------------------------------
static_assert(kFineThreads % 32 == 0 && TZ * 4 == 32, "a warp spans tz 0..7 x ty 0..3");

__host__ __device__ inline int ceil_div(int a, int b) { return (a + b - 1) / b; }
__host__ __device__ inline int fine_tiles(int n) { return ceil_div(n, TX) * ceil_div(n, TY) * ceil_div(n, TZ); }

// CTAs per SM the register allocation must allow (256-thread tiles): 4 for
// the FP32 elastic operator (64 registers, no spills), 2 for its FP64 form
// (128 registers), 4 or 6 for the small ones.  4x8x8-node tiles measured
// faster than 4x4x8 (FP64 K p 65 vs 76 us at 64^3, OC step +4%) and than
// 8x4x8.
template <typename T, int RD>
constexpr int fine_min_blocks() {
  return RD == 18 ? (sizeof(T) == 4 ? 4 : 2) : (RD == 3 && sizeof(T) == 8 ? 4 : 6);
}

template <typename T, int D, int R, int MODE, bool PDL = false>
__global__ void __launch_bounds__(kFineThreads, fine_min_blocks<T, R * D>()) k_apply_fine(ApplyArgs<T> a) {
  using G = FineTile<T, R * D>;
  constexpr int RD = R * D;
  constexpr bool PK = fine_packed<T, D, R>() && MODE != M_POWER;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* su = reinterpret_cast<T*>(smem_raw);
  T* srho = su + G::RHO_OFF;
  if constexpr (PDL) {
    griddep_wait();
    griddep_launch();
  }
  const int b = blockIdx.y;
  if (a.active && !a.active[b]) return;
  const int n = a.n;
  const size_t NN = (size_t)a.N;
  const int ntz = ceil_div(n, TZ), nty = ceil_div(n, TY);
  const int tile = blockIdx.x;
  const int z0 = (tile % ntz) * TZ, y0 = ((tile / ntz) % nty) * TY, x0 = (tile / (ntz * nty)) * TX;
  const int tz = threadIdx.x % TZ, ty = (threadIdx.x / TZ) % TY, tx = threadIdx.x / (TZ * TY);
  const int x = x0 + tx, y = y0 + ty, z = z0 + tz;
  const bool valid = x < n && y < n && z < n;
  const size_t cell = (size_t)b * NN;
  // ---- stage densities of the (TX+1)(TY+1)(TZ+1) elements touching the tile
  //      and the halo'd node values (component-major in global memory,
  //      node-major in shared memory), all as asynchronous copies in flight
  const int xm = x0 - 1, ym = y0 - 1, zm = z0 - 1;
  for (int w = threadIdx.x; w < G::RHO_WORDS; w += kFineThreads) {
    const int iz = w % (TZ + 1), iy = (w / (TZ + 1)) % (TY + 1), ix = w / ((TZ + 1) * (TY + 1));
    int gx = xm + ix, gy = ym + iy, gz = zm + iz;
    gx += gx < 0 ? n : (gx >= n ? -n : 0);
    gy += gy < 0 ? n : (gy >= n ? -n : 0);
    gz += gz < 0 ? n : (gz >= n ? -n : 0);
    cp_async<sizeof(T)>(srho + w, a.rho + cell + ((size_t)gx * n + gy) * n + gz);
  }
  if constexpr (MODE != M_JAC0) {
    // 25 groups of 10 lanes: a group copies whole halo rows (10 nodes along z),
    // lane iz owning one z position; the R*D components of a row then follow
    // with incremental addresses (component-major global, node-major shared).
    constexpr int ROWS = (TX + 2) * (TY + 2);
    constexpr int GROUPS = kFineThreads / (TZ + 2);
    const T* __restrict__ ub = a.u + cell * RD;
    const int g = threadIdx.x / (TZ + 2), iz = threadIdx.x - g * (TZ + 2);
    if (g < GROUPS) {
      int gz = zm + iz;
      gz += gz < 0 ? n : (gz >= n ? -n : 0);
      for (int row = g; row < ROWS; row += GROUPS) {
        const int ix = row / (TY + 2), iy = row - ix * (TY + 2);
        int gx = xm + ix, gy = ym + iy;
        gx += gx < 0 ? n : (gx >= n ? -n : 0);
        gy += gy < 0 ? n : (gy >= n ? -n : 0);
        const T* src = ub + ((size_t)gx * n + gy) * n + gz;
        T* dst = su + row * G::RW + iz * G::NS;
#pragma unroll 6
        for (int k = 0; k < RD; ++k) {
          // global component k = r*D + j; shared slot j*R + r when packed
          const int sk = PK ? (k % D) * R + k / D : k;
          cp_async<sizeof(T)>(dst + sk, src + (size_t)k * NN);
        }
      }
    }
  }
  cp_async_wait_all();
  __syncthreads();
  T rq[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int qx = (q >> 2) & 1, qy = (q >> 1) & 1, qz = q & 1;
    rq[q] = srho[((tx + qx) * (TY + 1) + (ty + qy)) * (TZ + 1) + (tz + qz)];
  }
  T acc[R][D];
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int i = 0; i < D; ++i) acc[r][i] = T(0);
  T C0[D][D];
  if constexpr (MODE == M_JAC0) {
    fine_block<T, D, 13>(rq, C0);
  } else if constexpr (PK) {
    const T* base = su + (tx * (TY + 2) + ty) * G::RW + tz * G::NS;
    unsigned long long acc2[3][3];
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
      for (int i = 0; i < 3; ++i) acc2[m][i] = 0ull;
    fine_tile_all_pk<G::RW, G::NS>(std::make_integer_sequence<int, 27>{}, rq, base, acc2, C0);
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
      for (int i = 0; i < 3; ++i) upk2(acc2[m][i], acc[2 * m][i], acc[2 * m + 1][i]);
  } else {
    const T* base = su + (tx * (TY + 2) + ty) * G::RW + tz * G::NS;
    fine_tile_all<T, D, R, G::RW, G::NS>(std::make_integer_sequence<int, 27>{}, rq, base, acc, C0);
  }
  T Di[D][D];
  T C0s[D][D];
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) C0s[i][j] = a.scale * C0[i][j];
  block_inverse<T, D>(C0s, Di);
  const int id = valid ? (x * n + y) * n + z : 0;
  const size_t vo = cell * RD + id;
  if constexpr (MODE == M_POWER) {
    double dots[2] = {0, 0};
    if (valid) {
      T Au[D];
      for (int i = 0; i < D; ++i) Au[i] = a.scale * acc[0][i];
      for (int i = 0; i < D; ++i) {
        T w = 0;
        for (int j = 0; j < D; ++j) w += Di[i][j] * Au[j];
        a.out[vo + i * NN] = w;
        dots[0] += (double)a.u[vo + i * NN] * (double)Au[i];
        for (int j = 0; j < D; ++j) dots[1] += (double)a.u[vo + i * NN] * (double)C0s[i][j] * (double)a.u[vo + j * NN];
      }
    }
    block_sum_store<2, kFineThreads / 32>(dots, a.part + ((size_t)b * gridDim.x + blockIdx.x) * 2);
  } else {
    if constexpr (MODE == M_CHEB || MODE == M_JAC0) {
      __shared__ double s_coef[2];
      if (threadIdx.x == 0) cheb_coeffs(a.hi[b], a.ratio, MODE == M_JAC0 ? 0 : a.step, s_coef[0], s_coef[1]);
      __syncthreads();
      a.cheb_al = s_coef[0];
      a.cheb_be = s_coef[1];
    }
    // the node's own values are the centre of the staged tile (stride 1)
    const T* uown = (MODE == M_JAC0) ? nullptr : su + ((tx + 1) * (TY + 2) + (ty + 1)) * G::RW + (tz + 1) * G::NS;
    apply_epilogue<T, D, R, MODE, kFineThreads / 32, PK>(a, b, vo, valid, acc, Di, uown, 1);
  }
}

// Fine-level block-Jacobi inverse, stored once per hierarchy build: for each
// node the inverse of scale * (its 3x3 (or 1x1) diagonal block), formed from
// the eight surrounding element densities with the operations k_apply_fine
// uses for it, so the stored values are the ones it forms on the fly.
// Layout [cell][D*D][node].
template <typename T, int D>
__global__ void k_fine_dinv(const T* __restrict__ rho, T* __restrict__ Dinv, int n, T scale, const int* active) {
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const int N = n * n * n;
  const int id = blockIdx.x * kThreads + threadIdx.x;
  if (id >= N) return;
  const int z = id % n, y = (id / n) % n, x = id / (n * n);
  const T* rb = rho + (size_t)b * N;
  T rq[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int qx = (q >> 2) & 1, qy = (q >> 1) & 1, qz = q & 1;
    rq[q] = rb[((size_t)wrapn(x - 1 + qx, n) * n + wrapn(y - 1 + qy, n)) * n + wrapn(z - 1 + qz, n)];
  }
  T C0[D][D], C0s[D][D], Di[D][D];
  fine_block<T, D, 13>(rq, C0);
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) C0s[i][j] = scale * C0[i][j];
  block_inverse<T, D>(C0s, Di);
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) Dinv[((size_t)b * D * D + i * D + j) * N + id] = Di[i][j];
}

// The first Chebyshev step from zero on the fine level with the stored block
// inverse: d = beta * Dinv f, u = d (k_apply_fine's M_JAC0 epilogue, without
// forming the diagonal block again).  A vector kernel: reads f and Dinv,
// writes u and d.
template <typename T, int D, int R, bool PDL = false>
__global__ void __launch_bounds__(kThreads) k_fine_jac0(ApplyArgs<T> a) {
  if constexpr (PDL) {
    griddep_wait();
    griddep_launch();
  }
  const int b = blockIdx.y;
  if (a.active && !a.active[b]) return;
  const int N = a.N;
  const size_t NN = (size_t)N;
  const int id = blockIdx.x * kThreads + threadIdx.x;
  if (id >= N) return;
  double al, be;
  cheb_coeffs(a.hi[b], a.ratio, 0, al, be);
  T Di[D][D];
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) Di[i][j] = a.Dinv[((size_t)b * D * D + i * D + j) * NN + id];
  const size_t vo = (size_t)b * N * R * D + id;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    T res[D];
#pragma unroll
    for (int i = 0; i < D; ++i) res[i] = a.f[vo + (size_t)(r * D + i) * NN];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      T zz = 0;
#pragma unroll
      for (int j = 0; j < D; ++j) zz += Di[i][j] * res[j];
      const T d = T(be) * zz;
      a.dout[vo + (size_t)(r * D + i) * NN] = d;
      a.out[vo + (size_t)(r * D + i) * NN] = d;
    }
  }
}

// The same on 16-byte vectors: W = 16 / sizeof(T) consecutive nodes per thread
// (the node count a multiple of W, every array 16-byte aligned).
template <typename T, int D, int R, bool PDL = false>
__global__ void __launch_bounds__(kThreads) k_fine_jac0_vec(ApplyArgs<T> a) {
  using V = typename Vec16<T>::type;
  constexpr int W = Vec16<T>::n;
  if constexpr (PDL) {
    griddep_wait();
    griddep_launch();
  }
  const int b = blockIdx.y;
  if (a.active && !a.active[b]) return;
  const int NG = a.N / W;
  const int g = blockIdx.x * kThreads + threadIdx.x;
  if (g >= NG) return;
  double al, be;
  cheb_coeffs(a.hi[b], a.ratio, 0, al, be);
  const T tb = T(be);
  V Di[D][D];
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j)
      Di[i][j] = reinterpret_cast<const V*>(a.Dinv)[((size_t)b * D * D + i * D + j) * NG + g];
  const size_t vo = (size_t)b * NG * R * D + g;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    V res[D];
#pragma unroll
    for (int i = 0; i < D; ++i) res[i] = reinterpret_cast<const V*>(a.f)[vo + (size_t)(r * D + i) * NG];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      V dv;
      T* ds = reinterpret_cast<T*>(&dv);
#pragma unroll
      for (int k = 0; k < W; ++k) {
        T zz = 0;
#pragma unroll
        for (int j = 0; j < D; ++j) zz += reinterpret_cast<const T*>(&Di[i][j])[k] * reinterpret_cast<const T*>(&res[j])[k];
        ds[k] = tb * zz;
      }
      reinterpret_cast<V*>(a.dout)[vo + (size_t)(r * D + i) * NG] = dv;
      reinterpret_cast<V*>(a.out)[vo + (size_t)(r * D + i) * NG] = dv;
    }
  }
}

// Coarse levels: one thread per (node, load case) so that the small grids of
// the deep levels still fill the machine; consecutive threads are consecutive
// nodes of one load case (coalesced stencil and field loads).
template <typename T, int D, int R, int MODE>
__global__ void __launch_bounds__(kThreads) k_apply_stencil(ApplyArgs<T> a) {
  static_assert(MODE != M_POWER, "power iterations use k_apply_stencil_power");
  const int b = blockIdx.y;
  if (a.active && !a.active[b]) return;
  const int n = a.n, N = a.N;
  const size_t NN = (size_t)N;
  const int t = blockIdx.x * kThreads + threadIdx.x;
  if (t >= N * R) return;
  const int r = t / N, id = t - r * N;
  const int z = id % n, y = (id / n) % n, x = id / (n * n);
  const size_t cell = (size_t)b * N;
  T acc[D];
#pragma unroll
  for (int i = 0; i < D; ++i) acc[i] = T(0);
  const T* __restrict__ S = a.S + (size_t)b * 27 * D * D * N + id;
  if constexpr (MODE != M_JAC0) {
    const int xs[3] = {wrapn(x - 1, n), x, wrapn(x + 1, n)};
    const int ys[3] = {wrapn(y - 1, n), y, wrapn(y + 1, n)};
    const int zs[3] = {wrapn(z - 1, n), z, wrapn(z + 1, n)};
    const T* __restrict__ ub = a.u + (cell * R + (size_t)r * N) * D;
#pragma unroll 9
    for (int o = 0; o < 27; ++o) {
      const int ox = o / 9, oy = (o / 3) % 3, oz = o % 3;
      const int nb = (xs[ox] * n + ys[oy]) * n + zs[oz];
      T uv[D];
#pragma unroll
      for (int j = 0; j < D; ++j) uv[j] = __ldg(ub + (size_t)j * NN + nb);
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) acc[i] += __ldg(S + ((size_t)o * D * D + i * D + j) * N) * uv[j];
    }
  }
  T Di[D][D];
  const T* __restrict__ Dp = a.Dinv + (size_t)b * D * D * N + id;
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) Di[i][j] = __ldg(Dp + (size_t)(i * D + j) * N);
  const size_t vo = (cell * R + (size_t)r * N) * D + id;  // component i at vo + i*N
  if constexpr (MODE == M_MV) {
#pragma unroll
    for (int i = 0; i < D; ++i) a.out[vo + i * NN] = acc[i];
  } else if constexpr (MODE == M_RES) {
#pragma unroll
    for (int i = 0; i < D; ++i) a.out[vo + i * NN] = a.f[vo + i * NN] - acc[i];
  } else {
    double al, be;
    cheb_coeffs(a.hi[b], a.ratio, MODE == M_JAC0 ? 0 : a.step, al, be);
    T res[D];
#pragma unroll
    for (int i = 0; i < D; ++i) res[i] = (MODE == M_JAC0) ? a.f[vo + i * NN] : a.f[vo + i * NN] - acc[i];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      T zz = 0;
#pragma unroll
      for (int j = 0; j < D; ++j) zz += Di[i][j] * res[j];
      T d = T(be) * zz;
      if (MODE == M_CHEB && al != 0.0) d += T(al) * a.din[vo + i * NN];
      a.dout[vo + i * NN] = d;
      a.out[vo + i * NN] = (MODE == M_JAC0) ? d : a.u[vo + i * NN] + d;
    }
  }
}

// ---------------------------------------------------------------------------
// Coarse levels, tiled: a CTA owns a 4x4x4 node tile and runs one thread per
// (tile node, load case).  The tile's stencils, block-diagonal inverses and
// the halo'd field values are staged into shared memory with asynchronous
// copies that are all in flight together, which removes the dependent-load
// latency chains that dominate small grids.  Requires n % 4 == 0.
// ---------------------------------------------------------------------------
constexpr int CT = 4;                         // tile edge
constexpr int CT_NODES = CT * CT * CT;        // 64
constexpr int CT_HALO = (CT + 2) * (CT + 2) * (CT + 2);  // 216

template <typename T, int D, int R>
struct CoarseTile {
  static constexpr int RD = R * D;
  static constexpr int NS = RD % 2 ? RD : RD + 1;   // odd node stride
  static constexpr int S_WORDS = 27 * D * D * CT_NODES;
  static constexpr int DI_WORDS = D * D * CT_NODES;
  static constexpr int U_WORDS = CT_HALO * NS;
  static constexpr size_t BYTES = (size_t)(S_WORDS + DI_WORDS + U_WORDS) * sizeof(T);
  static constexpr int THREADS = CT_NODES * R;
};

template <typename T, int D, int R, int MODE>
__global__ void __launch_bounds__(CT_NODES * 6) k_apply_stencil_tile(ApplyArgs<T> a) {
  using G = CoarseTile<T, D, R>;
  constexpr int RD = R * D;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sS = reinterpret_cast<T*>(smem_raw);          // [27*D*D][64]
  T* sDi = sS + G::S_WORDS;                         // [D*D][64]
  T* sU = sDi + G::DI_WORDS;                        // [216][NS]
  const int b = blockIdx.y;
  if (a.active && !a.active[b]) return;
  const int n = a.n, N = a.N;
  const size_t NN = (size_t)N;
  const int nt = n / CT;
  const int tile = blockIdx.x;
  const int z0 = (tile % nt) * CT, y0 = ((tile / nt) % nt) * CT, x0 = (tile / (nt * nt)) * CT;
  const int tid = threadIdx.x;
  // ---- stage: stencil rows and Dinv of the 64 tile nodes (16-byte chunks of
  //      4 consecutive z nodes), and the halo'd field values (scalar copies)
  {
    constexpr int CH = CT / (16 / (int)sizeof(T) < CT ? 16 / (int)sizeof(T) : CT);  // chunks per z-run
    constexpr int CW = CT / CH;                     // elements per chunk (4 floats or 2 doubles)
    const T* Sb = a.S + (size_t)b * 27 * D * D * N;
    const T* Db = a.Dinv + (size_t)b * D * D * N;
    constexpr int RUNS = CT * CT;                   // (x,y) runs per tile
    constexpr int K0 = MODE == M_JAC0 ? 27 * D * D : 0;  // JAC0 needs only the inverses
    for (int w = tid + K0 * RUNS * CH; w < (27 * D * D + D * D) * RUNS * CH; w += G::THREADS) {
      const int ch = w % CH, run = (w / CH) % RUNS, k = w / (CH * RUNS);
      const int ix = run / CT, iy = run % CT;
      const size_t gofs = ((size_t)(x0 + ix) * n + (y0 + iy)) * n + z0 + ch * CW;
      const int sofs = (ix * CT + iy) * CT + ch * CW;
      if (k < 27 * D * D)
        cp_async<CW * sizeof(T)>(sS + k * CT_NODES + sofs, Sb + (size_t)k * N + gofs);
      else
        cp_async<CW * sizeof(T)>(sDi + (k - 27 * D * D) * CT_NODES + sofs, Db + (size_t)(k - 27 * D * D) * N + gofs);
    }
    if constexpr (MODE != M_JAC0) {
      const T* ub = a.u + (size_t)b * RD * N;
      for (int w = tid; w < CT_HALO * RD; w += G::THREADS) {
        const int k = w / CT_HALO, h = w - k * CT_HALO;
        const int iz = h % (CT + 2), iy = (h / (CT + 2)) % (CT + 2), ix = h / ((CT + 2) * (CT + 2));
        int gx = x0 - 1 + ix, gy = y0 - 1 + iy, gz = z0 - 1 + iz;
        gx += gx < 0 ? n : (gx >= n ? -n : 0);
        gy += gy < 0 ? n : (gy >= n ? -n : 0);
        gz += gz < 0 ? n : (gz >= n ? -n : 0);
        cp_async<sizeof(T)>(sU + h * G::NS + k, ub + (size_t)k * N + ((size_t)gx * n + gy) * n + gz);
      }
    }
    cp_async_wait_all();
    __syncthreads();
  }
  const int tn = tid % CT_NODES, r = tid / CT_NODES;
  const int tz = tn % CT, ty = (tn / CT) % CT, tx = tn / (CT * CT);
  T acc[D];
#pragma unroll
  for (int i = 0; i < D; ++i) acc[i] = T(0);
  if constexpr (MODE != M_JAC0) {
#pragma unroll
    for (int o = 0; o < 27; ++o) {
      const int ox = o / 9, oy = (o / 3) % 3, oz = o % 3;
      const T* un = sU + (((tx + ox) * (CT + 2) + (ty + oy)) * (CT + 2) + (tz + oz)) * G::NS + r * D;
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) acc[i] += sS[((o * D + i) * D + j) * CT_NODES + tn] * un[j];
    }
  }
  T Di[D][D];
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) Di[i][j] = sDi[(i * D + j) * CT_NODES + tn];
  const int id = ((x0 + tx) * n + (y0 + ty)) * n + (z0 + tz);
  const size_t vo = ((size_t)b * R + r) * D * NN + id;   // component i at vo + i*N
  if constexpr (MODE == M_MV) {
#pragma unroll
    for (int i = 0; i < D; ++i) a.out[vo + i * NN] = acc[i];
  } else if constexpr (MODE == M_RES) {
#pragma unroll
    for (int i = 0; i < D; ++i) a.out[vo + i * NN] = a.f[vo + i * NN] - acc[i];
  } else {
    __shared__ double s_coef[2];
    if (tid == 0) cheb_coeffs(a.hi[b], a.ratio, MODE == M_JAC0 ? 0 : a.step, s_coef[0], s_coef[1]);
    __syncthreads();
    const double al = s_coef[0], be = s_coef[1];
    T res[D];
#pragma unroll
    for (int i = 0; i < D; ++i) res[i] = (MODE == M_JAC0) ? a.f[vo + i * NN] : a.f[vo + i * NN] - acc[i];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      T zz = 0;
#pragma unroll
      for (int j = 0; j < D; ++j) zz += Di[i][j] * res[j];
      T d = T(be) * zz;
      if (MODE == M_CHEB && al != 0.0) d += T(al) * a.din[vo + i * NN];
      a.dout[vo + i * NN] = d;
      a.out[vo + i * NN] = (MODE == M_JAC0) ? d : a.u[vo + i * NN] + d;
    }
  }
}

// Coarse-level stencil apply with the 27-offset reduction split over three
// threads per node: thread (node, px) sums the 9 offsets of x-offset plane
// px - 1 for all R load cases, reading its 9 D x D stencil blocks straight from
// global memory (coalesced: a warp is one 8 x 4 (z, y) slab of nodes; each
// stencil entry is read once, by one thread).  The neighbour values come from
// a halo'd shared-memory tile of the iterate; after the sums, the same shared
// memory holds the three partial sums, which thread (node, g) adds in plane
// order for load cases [g R/3, (g+1) R/3) and finishes (MV / RES / CHEB / JAC0
// as in k_apply_stencil_tile).  Requires n % 8 == 0 and R % 3 == 0.
constexpr int ST_Z = 8, ST_Y = 4, ST_X = 4;
constexpr int ST_NODES = ST_Z * ST_Y * ST_X;                       // 128
constexpr int ST_HALO = (ST_Z + 2) * (ST_Y + 2) * (ST_X + 2);      // 360
constexpr int ST_THREADS = 3 * ST_NODES;                           // 384

template <typename T, int D, int R>
struct SplitTile {
  static constexpr int RD = R * D;
  static constexpr int NS = RD % 2 ? RD : RD + 1;  // odd node stride: conflict-free halo reads
  static constexpr size_t HALO_BYTES = (size_t)ST_HALO * NS * sizeof(T);
  static constexpr size_t RED_BYTES = (size_t)3 * RD * ST_NODES * sizeof(T);
  static constexpr size_t BYTES = HALO_BYTES > RED_BYTES ? HALO_BYTES : RED_BYTES;
};

template <typename T, int D, int R, int MODE>
__global__ void __launch_bounds__(ST_THREADS) k_apply_stencil_split(ApplyArgs<T> a) {
  using G = SplitTile<T, D, R>;
  constexpr int RD = R * D, R3 = R / 3;
  static_assert(R % 3 == 0, "three threads per node share the load cases");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sU = reinterpret_cast<T*>(smem_raw);   // [ST_HALO][NS], then the partial sums [3][RD][ST_NODES]
  const int b = blockIdx.y;
  if (a.active && !a.active[b]) return;
  const int n = a.n, N = a.N;
  const size_t NN = (size_t)N;
  const int ntz = n / ST_Z, nty = n / ST_Y;
  const int tile = blockIdx.x;
  const int z0 = (tile % ntz) * ST_Z, y0 = ((tile / ntz) % nty) * ST_Y, x0 = (tile / (ntz * nty)) * ST_X;
  const int tid = threadIdx.x;
  const int tn = tid % ST_NODES, px = tid / ST_NODES;
  const int tz = tn % ST_Z, ty = (tn / ST_Z) % ST_Y, tx = tn / (ST_Z * ST_Y);
  const int id = ((x0 + tx) * n + (y0 + ty)) * n + (z0 + tz);
  T acc[R][D];
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int i = 0; i < D; ++i) acc[r][i] = T(0);
  if constexpr (MODE != M_JAC0) {
    const T* ub = a.u + (size_t)b * RD * N;
    for (int w = tid; w < ST_HALO * RD; w += ST_THREADS) {
      const int k = w / ST_HALO, h = w - k * ST_HALO;
      const int iz = h % (ST_Z + 2), iy = (h / (ST_Z + 2)) % (ST_Y + 2), ix = h / ((ST_Z + 2) * (ST_Y + 2));
      int gx = x0 - 1 + ix, gy = y0 - 1 + iy, gz = z0 - 1 + iz;
      gx += gx < 0 ? n : (gx >= n ? -n : 0);
      gy += gy < 0 ? n : (gy >= n ? -n : 0);
      gz += gz < 0 ? n : (gz >= n ? -n : 0);
      cp_async<sizeof(T)>(sU + h * G::NS + k, ub + (size_t)k * N + ((size_t)gx * n + gy) * n + gz);
    }
    cp_async_wait_all();
    __syncthreads();
    const T* Sb = a.S + (size_t)b * 27 * D * D * N + id;
#pragma unroll 1
    for (int q = 0; q < 9; ++q) {
      const int oy = q / 3, oz = q % 3, o = px * 9 + q;
      T sv[D][D];
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) sv[i][j] = Sb[(size_t)((o * D + i) * D + j) * N];
      const T* un = sU + (((tx + px) * (ST_Y + 2) + (ty + oy)) * (ST_Z + 2) + (tz + oz)) * G::NS;
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int j = 0; j < D; ++j) {
          const T uv = un[r * D + j];
#pragma unroll
          for (int i = 0; i < D; ++i) acc[r][i] += sv[i][j] * uv;
        }
    }
    __syncthreads();  // the halo is consumed: its space takes the partial sums
    T* red = sU;
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int i = 0; i < D; ++i) red[(px * RD + r * D + i) * ST_NODES + tn] = acc[r][i];
    __syncthreads();
  }
  // finish load cases [px R3, (px+1) R3) of node tn
  const int g = px;
  T tot[R3][D];
  if constexpr (MODE != M_JAC0) {
    const T* red = sU;
#pragma unroll
    for (int rr = 0; rr < R3; ++rr)
#pragma unroll
      for (int i = 0; i < D; ++i) {
        const int k = (g * R3 + rr) * D + i;
        tot[rr][i] = (red[k * ST_NODES + tn] + red[(RD + k) * ST_NODES + tn]) + red[(2 * RD + k) * ST_NODES + tn];
      }
  }
  const size_t cellv = (size_t)b * R * D * NN + id;
  if constexpr (MODE == M_MV || MODE == M_RES) {
#pragma unroll
    for (int rr = 0; rr < R3; ++rr)
#pragma unroll
      for (int i = 0; i < D; ++i) {
        const size_t o = cellv + ((size_t)(g * R3 + rr) * D + i) * NN;
        a.out[o] = MODE == M_MV ? tot[rr][i] : a.f[o] - tot[rr][i];
      }
  } else {
    __shared__ double s_coef[2];
    if (tid == 0) cheb_coeffs(a.hi[b], a.ratio, MODE == M_JAC0 ? 0 : a.step, s_coef[0], s_coef[1]);
    __syncthreads();
    const double al = s_coef[0], be = s_coef[1];
    T Di[D][D];
    const T* Db = a.Dinv + (size_t)b * D * D * N + id;
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) Di[i][j] = Db[(size_t)(i * D + j) * N];
#pragma unroll
    for (int rr = 0; rr < R3; ++rr) {
      const size_t vo = cellv + (size_t)(g * R3 + rr) * D * NN;
      T res[D];
#pragma unroll
      for (int i = 0; i < D; ++i) res[i] = (MODE == M_JAC0) ? a.f[vo + i * NN] : a.f[vo + i * NN] - tot[rr][i];
#pragma unroll
      for (int i = 0; i < D; ++i) {
        T zz = 0;
#pragma unroll
        for (int j = 0; j < D; ++j) zz += Di[i][j] * res[j];
        T d = T(be) * zz;
        if (MODE == M_CHEB && al != 0.0) d += T(al) * a.din[vo + i * NN];
        a.dout[vo + i * NN] = d;
        a.out[vo + i * NN] = (MODE == M_JAC0) ? d : a.u[vo + i * NN] + d;
      }
    }
  }
}

// Small coarse levels: nine threads per node, one per (x, y) offset pair, each
// summing its 3 z offsets for all R load cases straight from global memory
// (the whole level sits in L2), 32 nodes per CTA (a warp is 32 consecutive
// nodes of one offset pair: coalesced stencil reads).  The nine partial sums
// meet in shared memory, added in (x, y) offset order; thread (node, q < R)
// finishes load case q (MV / RES / CHEB / JAC0 as in k_apply_stencil_tile).
constexpr int NINE_NODES = 32;
constexpr int NINE_THREADS = 9 * NINE_NODES;

template <typename T, int D, int R, int MODE, bool PDL = false>
__global__ void __launch_bounds__(NINE_THREADS) k_apply_stencil_nine(ApplyArgs<T> a) {
  constexpr int RD = R * D;
  static_assert(R <= 9, "one finishing thread per load case");
  __shared__ T red[9][RD][NINE_NODES];
  const int b = blockIdx.y;
  if constexpr (PDL) {
    griddep_wait();
    griddep_launch();
  }
  if (a.active && !a.active[b]) return;
  const int n = a.n, N = a.N;
  const size_t NN = (size_t)N;
  const int tn = threadIdx.x % NINE_NODES, q = threadIdx.x / NINE_NODES;  // q = 3 ox + oy
  const int id = blockIdx.x * NINE_NODES + tn;
  const bool valid = id < N;
  const int z = id % n, y = (id / n) % n, x = id / (n * n);
  if constexpr (MODE != M_JAC0) {
    T acc[R][D];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int i = 0; i < D; ++i) acc[r][i] = T(0);
    if (valid) {
      const int ox = q / 3, oy = q % 3;
      const int xx = wrapn(x + ox - 1, n), yy = wrapn(y + oy - 1, n);
      const T* ub = a.u + (size_t)b * RD * NN;
      const T* __restrict__ S = a.S + (size_t)b * 27 * D * D * NN + id;
#pragma unroll
      for (int oz = 0; oz < 3; ++oz) {
        const int o = q * 3 + oz;
        const int nb = (xx * n + yy) * n + wrapn(z + oz - 1, n);
        T sv[D][D];
#pragma unroll
        for (int i = 0; i < D; ++i)
#pragma unroll
          for (int j = 0; j < D; ++j) sv[i][j] = __ldg(S + (size_t)((o * D + i) * D + j) * NN);
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
          for (int j = 0; j < D; ++j) {
            // under PDL the iterate was written during this grid's lifetime:
            // a coherent load, not the read-only path
            const T uv = PDL ? ub[(size_t)(r * D + j) * NN + nb] : __ldg(ub + (size_t)(r * D + j) * NN + nb);
#pragma unroll
            for (int i = 0; i < D; ++i) acc[r][i] = fma_rn(sv[i][j], uv, acc[r][i]);
          }
      }
    }
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int i = 0; i < D; ++i) red[q][r * D + i][tn] = acc[r][i];
  }
  __shared__ double s_coef[2];
  if constexpr (MODE == M_CHEB || MODE == M_JAC0) {
    if (threadIdx.x == 0) cheb_coeffs(a.hi[b], a.ratio, MODE == M_JAC0 ? 0 : a.step, s_coef[0], s_coef[1]);
  }
  __syncthreads();
  if (q >= R || !valid) return;
  const int r = q;
  T tot[D];
#pragma unroll
  for (int i = 0; i < D; ++i) {
    T t = T(0);
    if constexpr (MODE != M_JAC0) {
#pragma unroll
      for (int k = 0; k < 9; ++k) t = add_rn(t, red[k][r * D + i][tn]);
    }
    tot[i] = t;
  }
  const size_t vo = ((size_t)b * R + r) * D * NN + id;  // component i at vo + i*N
  if constexpr (MODE == M_MV) {
#pragma unroll
    for (int i = 0; i < D; ++i) a.out[vo + i * NN] = tot[i];
  } else if constexpr (MODE == M_RES) {
#pragma unroll
    for (int i = 0; i < D; ++i) a.out[vo + i * NN] = sub_rn(a.f[vo + i * NN], tot[i]);
  } else {
    const double al = s_coef[0], be = s_coef[1];
    T Di[D][D];
    const T* __restrict__ Dp = a.Dinv + (size_t)b * D * D * NN + id;
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) Di[i][j] = __ldg(Dp + (size_t)(i * D + j) * NN);
    T res[D];
#pragma unroll
    for (int i = 0; i < D; ++i) res[i] = (MODE == M_JAC0) ? a.f[vo + i * NN] : sub_rn(a.f[vo + i * NN], tot[i]);
#pragma unroll
    for (int i = 0; i < D; ++i) {
      T zz = mul_rn(Di[i][0], res[0]);
#pragma unroll
      for (int j = 1; j < D; ++j) zz = fma_rn(Di[i][j], res[j], zz);
      T d = mul_rn(T(be), zz);
      if (MODE == M_CHEB && al != 0.0) d = fma_rn(T(al), a.din[vo + i * NN], d);
      a.dout[vo + i * NN] = d;
      a.out[vo + i * NN] = (MODE == M_JAC0) ? d : add_rn(a.u[vo + i * NN], d);
    }
  }
}

// power iteration step on a coarse level: w = Dinv A u and the Rayleigh terms.
// One thread per (node, row i): a CTA covers kPowerNodes<D> nodes, rows
// i-major so that consecutive threads read consecutive stencil entries; the
// D row sums meet in shared memory for the Dinv product.
template <int D>
constexpr int kPowerNodes = D == 1 ? 256 : 64;

template <typename T, int D>
__global__ void __launch_bounds__(D * kPowerNodes<D>) k_apply_stencil_power(ApplyArgs<T> a) {
  constexpr int NB = kPowerNodes<D>;
  __shared__ T sacc[D][NB];
  const int b = blockIdx.y;
  if (a.active && !a.active[b]) return;
  const int n = a.n, N = a.N;
  const size_t NN = (size_t)N;
  const int i = threadIdx.x / NB, ln = threadIdx.x - i * NB;
  const int idx = blockIdx.x * NB + ln;
  const bool valid = idx < N;
  const int id = valid ? idx : 0;
  const int z = id % n, y = (id / n) % n, x = id / (n * n);
  const size_t cell = (size_t)b * N;
  const T* __restrict__ S = a.S + (size_t)b * 27 * D * D * N + id;
  const int xs[3] = {wrapn(x - 1, n), x, wrapn(x + 1, n)};
  const int ys[3] = {wrapn(y - 1, n), y, wrapn(y + 1, n)};
  const int zs[3] = {wrapn(z - 1, n), z, wrapn(z + 1, n)};
  const T* __restrict__ ub = a.u + cell * D;
  T acc = T(0);
#pragma unroll 9
  for (int o = 0; o < 27; ++o) {
    const int ox = o / 9, oy = (o / 3) % 3, oz = o % 3;
    const int nb = (xs[ox] * n + ys[oy]) * n + zs[oz];
#pragma unroll
    for (int j = 0; j < D; ++j) acc += __ldg(S + ((size_t)o * D * D + i * D + j) * N) * __ldg(ub + j * NN + nb);
  }
  sacc[i][ln] = acc;
  __syncthreads();
  double dots[2] = {0, 0};
  if (valid) {
    const size_t vo = cell * D + id;
    T w = 0;
    double diag = 0;
#pragma unroll
    for (int j = 0; j < D; ++j) {
      w += __ldg(a.Dinv + (size_t)b * D * D * N + (size_t)(i * D + j) * N + id) * sacc[j][ln];
      diag += (double)__ldg(S + ((size_t)13 * D * D + i * D + j) * N) * (double)a.u[vo + j * NN];
    }
    a.out[vo + i * NN] = w;
    const double ui = (double)a.u[vo + i * NN];
    dots[0] = ui * (double)acc;
    dots[1] = ui * diag;
  }
  block_sum_store<2, D * NB / 32>(dots, a.part + ((size_t)b * gridDim.x + blockIdx.x) * 2);
}

template <typename T>
__global__ void k_fill(T* __restrict__ p, size_t n, T v) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

// two consecutive values loaded or stored as one vector access
template <typename T>
struct alignas(2 * sizeof(T)) Pair {
  T lo, hi;
};

// ----------------------------------------------------------------------------
// grid transfer: periodic trilinear P (EBE_GMG.py:38-79, 531-647)
// ----------------------------------------------------------------------------
// rc = P^T rf : coarse node gathers its 27 fine neighbours 2X+d, weight
// prod(1-|d|/2).  One thread per (coarse node, component).
template <typename T, int K, bool PDL = false>
__global__ void k_restrict(const T* rf, T* rc, int nc, const int* active) {
  const int b = blockIdx.y;
  if constexpr (PDL) {
    griddep_wait();
    griddep_launch();
  }
  if (active && !active[b]) return;
  const int Nc = nc * nc * nc, nf = 2 * nc, Nf = Nc * 8;
  const int t = blockIdx.x * kThreads + threadIdx.x;
  if (t >= Nc * K) return;
  const int k = t / Nc, idx = t - k * Nc;
  const int Z = idx % nc, Y = (idx / nc) % nc, X = idx / (nc * nc);
  const T* base = rf + ((size_t)b * K + k) * Nf;
  const int fx[3] = {wrapn(2 * X - 1, nf), 2 * X, 2 * X + 1};
  const int fy[3] = {wrapn(2 * Y - 1, nf), 2 * Y, 2 * Y + 1};
  const int fz[3] = {wrapn(2 * Z - 1, nf), 2 * Z, 2 * Z + 1};
  T acc = 0;
#pragma unroll
  for (int dx = 0; dx < 3; ++dx)
#pragma unroll
    for (int dy = 0; dy < 3; ++dy) {
      // the z-run 2Z-1, 2Z, 2Z+1 of this (x, y) row: one scalar and one pair load
      const T* row = base + ((size_t)fx[dx] * nf + fy[dy]) * nf;
      const Pair<T> p = *reinterpret_cast<const Pair<T>*>(row + fz[1]);
      const T v[3] = {PDL ? row[fz[0]] : __ldg(row + fz[0]), p.lo, p.hi};
#pragma unroll
      for (int dz = 0; dz < 3; ++dz) {
        const T w = T((dx != 1 ? 0.5 : 1.0) * (dy != 1 ? 0.5 : 1.0) * (dz != 1 ? 0.5 : 1.0));
        acc = fma_rn(w, v[dz], acc);
      }
    }
  rc[((size_t)b * K + k) * Nc + idx] = acc;
}

// uf += P uc, one thread per (coarse node, component): the thread reads the 8
// coarse values of its coarse cell once and updates the 2 x 2 x 2 fine nodes
// (2X + rx, 2Y + ry, 2Z + rz), the two z neighbours as one vector access.  A
// fine coordinate that is even takes weight 1 from its own coarse node and 0
// from the next one, an odd one 1/2 from each; each fine value is the sum over
// the 8 corners in (x, y, z) order of weight x value.
template <typename T, int K, bool PDL = false>
__global__ void k_prolong_add(const T* uc, T* uf, int nc, const int* active) {
  const int b = blockIdx.y;
  if constexpr (PDL) {
    griddep_wait();
    griddep_launch();
  }
  if (active && !active[b]) return;
  const int nf = 2 * nc, Nc = nc * nc * nc;
  const size_t Nf = (size_t)Nc * 8;
  const int t = blockIdx.x * kThreads + threadIdx.x;
  if (t >= Nc * K) return;
  const int k = t / Nc, idx = t - k * Nc;
  const int Z = idx % nc, Y = (idx / nc) % nc, X = idx / (nc * nc);
  const T* base = uc + ((size_t)b * K + k) * Nc;
  const int cx[2] = {X, X + 1 == nc ? 0 : X + 1};
  const int cy[2] = {Y, Y + 1 == nc ? 0 : Y + 1};
  const int cz[2] = {Z, Z + 1 == nc ? 0 : Z + 1};
  T cv[8];
#pragma unroll
  for (int o = 0; o < 8; ++o)
    cv[o] = PDL ? base[((size_t)cx[(o >> 2) & 1] * nc + cy[(o >> 1) & 1]) * nc + cz[o & 1]]
                : __ldg(base + ((size_t)cx[(o >> 2) & 1] * nc + cy[(o >> 1) & 1]) * nc + cz[o & 1]);
  T* fb = uf + ((size_t)b * K + k) * Nf;
#pragma unroll
  for (int rx = 0; rx < 2; ++rx)
#pragma unroll
    for (int ry = 0; ry < 2; ++ry) {
      const T wx[2] = {T(rx ? 0.5 : 1.0), T(rx ? 0.5 : 0.0)};
      const T wy[2] = {T(ry ? 0.5 : 1.0), T(ry ? 0.5 : 0.0)};
      T acc[2];
#pragma unroll
      for (int rz = 0; rz < 2; ++rz) {
        const T wz[2] = {T(rz ? 0.5 : 1.0), T(rz ? 0.5 : 0.0)};
        T a = 0;
#pragma unroll
        for (int o = 0; o < 8; ++o) a = fma_rn(wx[(o >> 2) & 1] * wy[(o >> 1) & 1] * wz[o & 1], cv[o], a);
        acc[rz] = a;
      }
      Pair<T>* dst = reinterpret_cast<Pair<T>*>(fb + ((size_t)(2 * X + rx) * nf + (2 * Y + ry)) * nf + 2 * Z);
      Pair<T> v = *dst;
      v.lo = add_rn(v.lo, acc[0]);
      v.hi = add_rn(v.hi, acc[1]);
      *dst = v;
    }
}

// coarsest level: u = Ainv f with the FP64 (regularised) inverse, per cell;
// one warp per row, lanes over the columns.
template <typename T, int R>
__global__ void k_coarse_solve(const double* __restrict__ Ainv, const T* __restrict__ f, T* __restrict__ u, int ndof,
                               int D, const int* active) {
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const int lane = threadIdx.x & 31;
  const int row = blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5);
  if (row >= ndof) return;
  const int Nc = ndof / D;
  const double* A = Ainv + ((size_t)b * ndof + row) * ndof;
  const T* fb = f + (size_t)b * ndof * R;  // [rhs][comp][node]; dof = node*D + comp
  double acc[R];
#pragma unroll
  for (int r = 0; r < R; ++r) acc[r] = 0;
  for (int col = lane; col < ndof; col += 32) {
    const int node = col / D, c = col - node * D;
    const double a = A[col];
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = fma_rn(a, (double)fb[(size_t)(r * D + c) * Nc + node], acc[r]);
  }
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc[r] = add_rn(acc[r], __shfl_down_sync(0xffffffffu, acc[r], off));
  if (lane == 0) {
    const int node = row / D, c = row - node * D;
    T* ub = u + (size_t)b * ndof * R;
#pragma unroll
    for (int r = 0; r < R; ++r) ub[(size_t)(r * D + c) * Nc + node] = (T)acc[r];
  }
}

// ----------------------------------------------------------------------------
// Fused bottom of the V-cycle (FP32): the 8^3-node level above a 4^3-node
// coarsest level -- Chebyshev pre-smoothing, residual, restriction, coarsest
// solve, prolongation, post-smoothing -- in one launch, one cluster of 8 CTAs
// per cell.  CTA p owns the x = p plane (64 nodes): its stencils, block
// inverses, right-hand side, iterate, direction and residual stay in shared
// memory for the whole cycle.  A sweep copies the x-1 and x+1 planes of the
// iterate from the neighbouring CTAs' shared memory (distributed shared
// memory) after a cluster barrier.  The iterate is double-buffered, so one
// barrier per sweep suffices: a CTA overwrites a buffer two barriers after
// its neighbours last copied it.  The restricted right-hand side and the
// coarsest solution are written into every CTA of the cluster.  Every sum
// keeps the operand order and the explicit rounding of the separate kernels
// (k_apply_stencil_nine, k_restrict, k_coarse_solve, k_prolong_add), so the
// cycle reproduces their launch sequence bit for bit.  Cluster barriers are
// hardware barriers:
// no thread of a cluster returns before the last one, and a cell's cluster
// either runs all of them or (inactive cell) none.
// ----------------------------------------------------------------------------
constexpr int TAIL_N = 8, TAIL_NC = 4, TAIL_CTAS = 8, TAIL_P = 64, TAIL_THREADS = 9 * TAIL_P;
constexpr int kTailMaxDegree = 8;

struct TailArgs {
  const float* S;      // level stencils [B][27][D*D][512]
  const float* Dinv;   // block-diagonal inverses [B][D*D][512]
  const float* f;      // level right-hand side [B][R][D][512]
  float* u;            // resulting iterate [B][R][D][512]
  const double* Ainv;  // coarsest inverse [B][64 D][64 D]
  const double* hi;    // per-cell Chebyshev upper bound of the level
  double ratio;        // Chebyshev interval ratio
  int deg;             // Chebyshev steps per smoothing, 1..kTailMaxDegree
  const int* active;   // per-cell flag (nullable)
};

template <int D, int R>
struct TailSmem {
  static constexpr int RD = R * D, P = TAIL_P, NCN = TAIL_NC * TAIL_NC * TAIL_NC;
  static constexpr int S = 0;                    // [27 D D][P]
  static constexpr int DI = S + 27 * D * D * P;  // [D D][P]
  static constexpr int F = DI + D * D * P;       // [RD][P]
  static constexpr int U = F + RD * P;           // [2][RD][P] iterate
  static constexpr int H = U + 2 * RD * P;       // [2][RD][P] planes x-1, x+1
  static constexpr int DD = H + 2 * RD * P;      // [RD][P] Chebyshev direction
  static constexpr int RS = DD + RD * P;         // [RD][P] residual
  static constexpr int RED = RS + RD * P;        // [9][RD][P] partial sums
  static constexpr int FC = RED + 9 * RD * P;    // [RD][NCN] coarsest right-hand side
  static constexpr int UC = FC + RD * NCN;       // [RD][NCN] coarsest solution
  static constexpr int FLOATS = UC + RD * NCN;
  static constexpr size_t BYTES = (size_t)FLOATS * sizeof(float) + 2 * kTailMaxDegree * sizeof(double);
  static_assert(FLOATS % 4 == 0 && U % 4 == 0 && H % 4 == 0 && (RD * P) % 4 == 0, "16-byte aligned planes");
};

template <int D, int R, bool PDL = false>
__global__ void __cluster_dims__(TAIL_CTAS, 1, 1) __launch_bounds__(TAIL_THREADS) k_tail_cycle(TailArgs a) {
  namespace cg = cooperative_groups;
  using L = TailSmem<D, R>;
  constexpr int RD = R * D, P = TAIL_P, n = TAIL_N, nc = TAIL_NC, N = n * n * n, NCN = L::NCN, ndof = NCN * D;
  constexpr int V4 = RD * P / 4;  // float4 per plane of the iterate
  extern __shared__ __align__(16) float tsm[];
  float* sS = tsm + L::S;
  float* sDi = tsm + L::DI;
  float* sF = tsm + L::F;
  float* sU = tsm + L::U;
  float* sH = tsm + L::H;
  float* sDd = tsm + L::DD;
  float* sRs = tsm + L::RS;
  float* red = tsm + L::RED;
  float* sFc = tsm + L::FC;
  float* sUc = tsm + L::UC;
  double* s_al = reinterpret_cast<double*>(tsm + L::FLOATS);
  double* s_be = s_al + kTailMaxDegree;

  const int b = blockIdx.y;
  // the whole cluster belongs to cell b: an inactive cell's CTAs all return
  // (under PDL only after the wait, which also covers the flag itself)
  if (!PDL && a.active && !a.active[b]) return;
  cg::cluster_group cl = cg::this_cluster();
  const int px = (int)cl.block_rank();
  const int tid = threadIdx.x;
  const int tn = tid % P, q = tid / P;  // node of the plane, (x, y) offset pair 3 ox + oy
  const int deg = a.deg;

  // stencils, inverses and bounds were built before the solve (under PDL they
  // are staged before the wait); the right-hand side comes from the previous
  // launch and is read coherently under PDL
  auto stage = [&](float* dst, const float* src, int rows, bool coherent) {
    for (int t = tid; t < rows * (P / 4); t += TAIL_THREADS) {
      const int k = t / (P / 4), m = t - k * (P / 4);
      const float4* g = reinterpret_cast<const float4*>(src + (size_t)k * N) + m;
      reinterpret_cast<float4*>(dst)[t] = coherent ? *g : __ldg(g);
    }
  };
  stage(sS, a.S + (size_t)b * 27 * D * D * N + px * P, 27 * D * D, false);
  stage(sDi, a.Dinv + (size_t)b * D * D * N + px * P, D * D, false);
  if (tid < deg) cheb_coeffs(a.hi[b], a.ratio, tid, s_al[tid], s_be[tid]);
  if constexpr (PDL) {
    griddep_wait();
    griddep_launch();
    if (a.active && !a.active[b]) return;
  }
  stage(sF, a.f + (size_t)b * RD * N + px * P, RD, PDL);
  __syncthreads();

  // copy the x-1 and x+1 planes of iterate buffer `cur` from the neighbours
  auto halo = [&](int cur) {
    const float4* lo = reinterpret_cast<const float4*>(cl.map_shared_rank(sU + cur * RD * P, (px + TAIL_CTAS - 1) % TAIL_CTAS));
    const float4* hi = reinterpret_cast<const float4*>(cl.map_shared_rank(sU + cur * RD * P, (px + 1) % TAIL_CTAS));
    float4* h = reinterpret_cast<float4*>(sH);
    for (int t = tid; t < 2 * V4; t += TAIL_THREADS) h[t] = t < V4 ? lo[t] : hi[t - V4];
  };
  // thread (tn, q): the 3 z offsets of offset pair q for all load cases
  auto partials = [&](const float* own) {
    const int ox = q / 3, oy = q % 3;
    const float* plane = ox == 1 ? own : sH + (ox >> 1) * RD * P;
    const int y = tn / n, z = tn % n;
    const int yy = wrapn(y + oy - 1, n);
    float acc[R][D];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int i = 0; i < D; ++i) acc[r][i] = 0.f;
#pragma unroll
    for (int oz = 0; oz < 3; ++oz) {
      const int o = q * 3 + oz;
      const int nb = yy * n + wrapn(z + oz - 1, n);
      float sv[D][D];
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) sv[i][j] = sS[((o * D + i) * D + j) * P + tn];
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int j = 0; j < D; ++j) {
          const float uv = plane[(r * D + j) * P + nb];
#pragma unroll
          for (int i = 0; i < D; ++i) acc[r][i] = fma_rn(sv[i][j], uv, acc[r][i]);
        }
    }
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int i = 0; i < D; ++i) red[(q * RD + r * D + i) * P + tn] = acc[r][i];
  };
  // thread (tn, r = q < R): residual, or one Chebyshev step from buffer cur
  // into buffer 1 - cur (the last one also to global memory)
  auto finish = [&](int mode, int st, int cur, bool last) {
    if (q >= R) return;
    const int r = q;
    float tot[D];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      float t = 0.f;
      if (mode != M_JAC0) {
#pragma unroll
        for (int k = 0; k < 9; ++k) t = add_rn(t, red[(k * RD + r * D + i) * P + tn]);
      }
      tot[i] = t;
    }
    if (mode == M_RES) {
#pragma unroll
      for (int i = 0; i < D; ++i) sRs[(r * D + i) * P + tn] = sub_rn(sF[(r * D + i) * P + tn], tot[i]);
      return;
    }
    const double al = s_al[st], be = s_be[st];
    float Di[D][D];
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) Di[i][j] = sDi[(i * D + j) * P + tn];
    float res[D];
#pragma unroll
    for (int i = 0; i < D; ++i) res[i] = mode == M_JAC0 ? sF[(r * D + i) * P + tn] : sub_rn(sF[(r * D + i) * P + tn], tot[i]);
#pragma unroll
    for (int i = 0; i < D; ++i) {
      float zz = mul_rn(Di[i][0], res[0]);
#pragma unroll
      for (int j = 1; j < D; ++j) zz = fma_rn(Di[i][j], res[j], zz);
      const int e = (r * D + i) * P + tn;
      float d = mul_rn(float(be), zz);
      if (mode == M_CHEB && al != 0.0) d = fma_rn(float(al), sDd[e], d);
      sDd[e] = d;
      const float un = mode == M_JAC0 ? d : add_rn(sU[cur * RD * P + e], d);
      sU[(1 - cur) * RD * P + e] = un;
      if (last) a.u[((size_t)b * RD + r * D + i) * N + px * P + tn] = un;
    }
  };
  auto sweep = [&](int mode, int st, int cur, bool last) {
    cl.sync();  // every plane's buffer `cur` is complete
    halo(cur);
    __syncthreads();
    partials(sU + cur * RD * P);
    __syncthreads();
    finish(mode, st, cur, last);
  };

  // pre-smoothing: a step from the zero iterate into buffer 0, then deg - 1 steps
  finish(M_JAC0, 0, 1, false);
  int cur = 0;
  for (int st = 1; st < deg; ++st, cur ^= 1) sweep(M_CHEB, st, cur, false);
  sweep(M_RES, 0, cur, false);
  cl.sync();  // every plane's residual is complete

  // restriction: CTA p forms half of coarse plane X = p / 2, written to every CTA
  {
    constexpr int HALF = 8 * RD;  // 16 (Y, Z) x RD entries per coarse plane
    const int X = px >> 1;
    const int fx[3] = {wrapn(2 * X - 1, n), 2 * X, 2 * X + 1};
    for (int t = tid; t < HALF; t += TAIL_THREADS) {
      const int e = (px & 1) * HALF + t;
      const int k = e / 16, Y = (e % 16) / nc, Z = e % nc;
      const int fy[3] = {wrapn(2 * Y - 1, n), 2 * Y, 2 * Y + 1};
      const int fz[3] = {wrapn(2 * Z - 1, n), 2 * Z, 2 * Z + 1};
      float acc = 0.f;
#pragma unroll
      for (int dx = 0; dx < 3; ++dx) {
        const float* pl = cl.map_shared_rank(sRs, fx[dx]) + k * P;
#pragma unroll
        for (int dy = 0; dy < 3; ++dy) {
          const float* row = pl + fy[dy] * n;
          const float v[3] = {row[fz[0]], row[fz[1]], row[fz[2]]};
#pragma unroll
          for (int dz = 0; dz < 3; ++dz) {
            const float w = float((dx != 1 ? 0.5 : 1.0) * (dy != 1 ? 0.5 : 1.0) * (dz != 1 ? 0.5 : 1.0));
            acc = fma_rn(w, v[dz], acc);
          }
        }
      }
      const int ci = k * NCN + (X * nc + Y) * nc + Z;
#pragma unroll
      for (int rk = 0; rk < TAIL_CTAS; ++rk) cl.map_shared_rank(sFc, rk)[ci] = acc;
    }
  }
  cl.sync();

  // coarsest solve u_c = Ainv f_c: CTA p takes rows [p ndof/8, (p+1) ndof/8),
  // one warp per row, lanes over the columns (FP64 accumulation)
  {
    constexpr int ROWS = ndof / TAIL_CTAS;
    static_assert(ndof % TAIL_CTAS == 0, "rows split evenly over the cluster");
    const int warp = tid >> 5, lane = tid & 31;
    for (int rr = warp; rr < ROWS; rr += TAIL_THREADS / 32) {
      const int row = px * ROWS + rr;
      const double* A = a.Ainv + ((size_t)b * ndof + row) * ndof;
      double acc[R];
#pragma unroll
      for (int r = 0; r < R; ++r) acc[r] = 0;
      for (int col = lane; col < ndof; col += 32) {
        const int node = col / D, c = col - node * D;
        const double av = __ldg(A + col);
#pragma unroll
        for (int r = 0; r < R; ++r) acc[r] = fma_rn(av, (double)sFc[(r * D + c) * NCN + node], acc[r]);
      }
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc[r] = add_rn(acc[r], __shfl_down_sync(0xffffffffu, acc[r], off));
      if (lane == 0) {
        const int node = row / D, c = row - node * D;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const float v = (float)acc[r];
#pragma unroll
          for (int rk = 0; rk < TAIL_CTAS; ++rk) cl.map_shared_rank(sUc, rk)[(r * D + c) * NCN + node] = v;
        }
      }
    }
  }
  cl.sync();

  // prolongation into this plane of buffer cur
  {
    const int X = px >> 1, rx = px & 1;
    const int cx[2] = {X, (X + 1) % nc};
    const float wx[2] = {rx ? 0.5f : 1.0f, rx ? 0.5f : 0.0f};
    for (int t = tid; t < RD * P; t += TAIL_THREADS) {
      const int k = t / P, m = t - k * P, y = m / n, z = m % n;
      const int Y = y >> 1, ry = y & 1, Z = z >> 1, rz = z & 1;
      const int cy[2] = {Y, (Y + 1) % nc};
      const int cz[2] = {Z, (Z + 1) % nc};
      const float wy[2] = {ry ? 0.5f : 1.0f, ry ? 0.5f : 0.0f};
      const float wz[2] = {rz ? 0.5f : 1.0f, rz ? 0.5f : 0.0f};
      float s = 0.f;
#pragma unroll
      for (int o = 0; o < 8; ++o) {
        const float cv = sUc[k * NCN + (cx[(o >> 2) & 1] * nc + cy[(o >> 1) & 1]) * nc + cz[o & 1]];
        s = fma_rn(wx[(o >> 2) & 1] * wy[(o >> 1) & 1] * wz[o & 1], cv, s);
      }
      sU[cur * RD * P + t] = add_rn(sU[cur * RD * P + t], s);
    }
  }

  // post-smoothing; the last step also writes the iterate to global memory
  for (int st = 0; st < deg; ++st, cur ^= 1) sweep(M_CHEB, st, cur, st == deg - 1);
  cl.sync();  // no CTA leaves while a neighbour may still read its shared memory
}

// ----------------------------------------------------------------------------
// hierarchy construction (FP64)
// ----------------------------------------------------------------------------
// level-1 element matrices: K_E = sum_c rho_c M_c  (exact Galerkin of rho*Ke0)
template <int D>
__global__ void k_level1_elements(const double* __restrict__ rho, const double* __restrict__ M, double* __restrict__ KE,
                                  int nc, double scale, const int* active) {
  constexpr int k = 8 * D, kk = k * k;
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const int Nc = nc * nc * nc, nf = 2 * nc;
  const size_t t = (size_t)blockIdx.x * kThreads + threadIdx.x;
  if (t >= (size_t)Nc * kk) return;
  const int e = (int)(t / kk), ij = (int)(t % kk);
  const int Z = e % nc, Y = (e / nc) % nc, X = e / (nc * nc);
  const double* rb = rho + (size_t)b * nf * nf * nf;
  double s = 0;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int cx = (c >> 2) & 1, cy = (c >> 1) & 1, cz = c & 1;
    const double r = rb[((size_t)(2 * X + cx) * nf + (2 * Y + cy)) * nf + (2 * Z + cz)];
    s = fma(r, M[c * kk + ij], s);
  }
  KE[((size_t)b * Nc + e) * kk + ij] = __dmul_rn(scale, s);
}

// Level-1 node stencils straight from the fine densities, without forming
// the level-1 element matrices: the D x D block of node n and offset o sums,
// over the level-1 elements holding both nodes, scale * sum_c rho_c M_c of
// that element (the matrix k_level1_elements forms, with the same operations
// in the same order, so these are the stencils k_stencil_from_elements builds
// from its output); block-diagonal inverse at o = 13.  Consecutive threads are
// consecutive nodes of one offset, so the table entries they read coincide.
template <typename T, int D>
__global__ void k_level1_stencils(const double* __restrict__ rho, const double* __restrict__ M, T* __restrict__ S,
                                  T* __restrict__ Dinv, int n, double scale, const int* active) {
  constexpr int k = 8 * D, kk = k * k;
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const int N = n * n * n, nf = 2 * n;
  const int t = blockIdx.x * kThreads + threadIdx.x;
  if (t >= N * 27) return;
  const int node = t % N, o = t / N;
  const int z = node % n, y = (node / n) % n, x = node / (n * n);
  const int ox = o / 9 - 1, oy = (o / 3) % 3 - 1, oz = o % 3 - 1;
  const double* rb = rho + (size_t)b * nf * nf * nf;
  double C[D][D] = {};
  for (int q = 0; q < 8; ++q) {
    const int qx = (q >> 2) & 1, qy = (q >> 1) & 1, qz = q & 1;
    const int cx = 1 - qx, cy = 1 - qy, cz = 1 - qz;
    const int nx = cx + ox, ny = cy + oy, nz = cz + oz;
    if (nx < 0 || nx > 1 || ny < 0 || ny > 1 || nz < 0 || nz > 1) continue;
    const int ex = wrapn(x + qx - 1, n), ey = wrapn(y + qy - 1, n), ez = wrapn(z + qz - 1, n);
    double rc[8];
#pragma unroll
    for (int ch = 0; ch < 8; ++ch) {
      const int hx = (ch >> 2) & 1, hy = (ch >> 1) & 1, hz = ch & 1;
      rc[ch] = rb[((size_t)(2 * ex + hx) * nf + (2 * ey + hy)) * nf + (2 * ez + hz)];
    }
    const int aa = lidx(cx, cy, cz), bb = lidx(nx, ny, nz);
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) {
        const int ij = (D * aa + i) * k + D * bb + j;
        double sum = 0;
#pragma unroll
        for (int ch = 0; ch < 8; ++ch) sum = fma(rc[ch], __ldg(M + ch * kk + ij), sum);
        C[i][j] = __dadd_rn(C[i][j], __dmul_rn(scale, sum));
      }
  }
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) S[(((size_t)b * 27 + o) * D * D + i * D + j) * N + node] = (T)C[i][j];
  if (o == 13) {
    double Ci[D][D];
    block_inverse<double, D>(C, Ci);
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) Dinv[((size_t)b * D * D + i * D + j) * N + node] = (T)Ci[i][j];
  }
}

// Level-2 element matrices straight from the fine densities:
// K_2[E] = scale * sum over the 4^3 fine elements f of E of rho_f G_f, with
// G_f the exact two-level Galerkin product of one fine element of unit
// density (host table, f = (4 fx + fy) 4 + fz).  A block owns kL2Elems
// elements, its threads the matrix entries: each G_f entry is read once per
// block and used for all of them.
constexpr int kL2Elems = 8;
template <int D>
__global__ void __launch_bounds__(kThreads) k_level2_elements(const double* __restrict__ rho,
                                                              const double* __restrict__ G, double* __restrict__ KE,
                                                              int nc, double scale, const int* active) {
  constexpr int k = 8 * D, kk = k * k;
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const int Nc = nc * nc * nc, nf = 4 * nc;
  const int e0 = blockIdx.x * kL2Elems;
  __shared__ double sr[64][kL2Elems];
  for (int t = threadIdx.x; t < 64 * kL2Elems; t += kThreads) {
    const int f = t / kL2Elems, el = t - f * kL2Elems, e = e0 + el;
    double v = 0;
    if (e < Nc) {
      const int Z = e % nc, Y = (e / nc) % nc, X = e / (nc * nc);
      const int fx = f >> 4, fy = (f >> 2) & 3, fz = f & 3;
      v = rho[(size_t)b * nf * nf * nf + ((size_t)(4 * X + fx) * nf + (4 * Y + fy)) * nf + (4 * Z + fz)];
    }
    sr[f][el] = v;
  }
  __syncthreads();
  for (int ij = threadIdx.x; ij < kk; ij += kThreads) {
    double acc[kL2Elems];
#pragma unroll
    for (int el = 0; el < kL2Elems; ++el) acc[el] = 0;
#pragma unroll 4
    for (int f = 0; f < 64; ++f) {
      const double g = __ldg(G + (size_t)f * kk + ij);
#pragma unroll
      for (int el = 0; el < kL2Elems; ++el) acc[el] = fma(sr[f][el], g, acc[el]);
    }
#pragma unroll
    for (int el = 0; el < kL2Elems; ++el)
      if (e0 + el < Nc) KE[((size_t)b * Nc + e0 + el) * kk + ij] = scale * acc[el];
  }
}

// K_{l+1}[E] = sum_c (W_c (x) I)^T K_l[child c] (W_c (x) I), one block per coarse element
template <int D>
__global__ void k_coarsen_elements(const double* __restrict__ Kf, double* __restrict__ Kc, int nc, const int* active) {
  constexpr int k = 8 * D, kk = k * k;
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  extern __shared__ double smem_c[];
  double(*sK)[kk] = reinterpret_cast<double(*)[kk]>(smem_c);
  double(*sT)[kk] = reinterpret_cast<double(*)[kk]>(smem_c + 8 * kk);
  const int e = blockIdx.x;
  const int Z = e % nc, Y = (e / nc) % nc, X = e / (nc * nc);
  const int nf = 2 * nc, Nf = nf * nf * nf, Nc = nc * nc * nc;
  for (int t = threadIdx.x; t < 8 * kk; t += blockDim.x) {
    const int c = t / kk, ij = t % kk;
    const int cx = (c >> 2) & 1, cy = (c >> 1) & 1, cz = c & 1;
    const size_t fe = ((size_t)(2 * X + cx) * nf + (2 * Y + cy)) * nf + (2 * Z + cz);
    sK[c][ij] = Kf[((size_t)b * Nf + fe) * kk + ij];
  }
  __syncthreads();
  // stage 1: T_c[(a',al)][(bb,be)] = sum_b' K_c[(a',al)][(b',be)] W_c[b'][bb]
  for (int t = threadIdx.x; t < 8 * kk; t += blockDim.x) {
    const int c = t / kk, ij = t % kk, row = ij / k, col = ij % k;
    const int bb = col / D, be = col % D;
    double s = 0;
#pragma unroll
    for (int b2 = 0; b2 < 8; ++b2) s += sK[c][row * k + D * b2 + be] * c_W[(c * 8 + b2) * 8 + bb];
    sT[c][ij] = s;
  }
  __syncthreads();
  // stage 2: out[(a,al)][col] = sum_c sum_a' W_c[a'][a] T_c[(a',al)][col]
  for (int t = threadIdx.x; t < kk; t += blockDim.x) {
    const int row = t / k, col = t % k, aa = row / D, al = row % D;
    double s = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c)
#pragma unroll
      for (int a2 = 0; a2 < 8; ++a2) s += c_W[(c * 8 + a2) * 8 + aa] * sT[c][(D * a2 + al) * k + col];
    Kc[((size_t)b * Nc + e) * kk + t] = s;
  }
}

// node stencils from element matrices; block-diagonal inverse at o = 13.
template <typename T, int D>
__global__ void k_stencil_from_elements(const double* __restrict__ KE, T* __restrict__ S, T* __restrict__ Dinv,
                                        double* __restrict__ S64, int n, const int* active) {
  constexpr int k = 8 * D, kk = k * k;
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const int N = n * n * n;
  const int t = blockIdx.x * kThreads + threadIdx.x;
  if (t >= N * 27) return;
  const int node = t % N, o = t / N;
  const int z = node % n, y = (node / n) % n, x = node / (n * n);
  const int ox = o / 9 - 1, oy = (o / 3) % 3 - 1, oz = o % 3 - 1;
  double C[D][D] = {};
  for (int q = 0; q < 8; ++q) {
    const int qx = (q >> 2) & 1, qy = (q >> 1) & 1, qz = q & 1;
    const int cx = 1 - qx, cy = 1 - qy, cz = 1 - qz;
    const int nx = cx + ox, ny = cy + oy, nz = cz + oz;
    if (nx < 0 || nx > 1 || ny < 0 || ny > 1 || nz < 0 || nz > 1) continue;
    const int ex = wrapn(x + qx - 1, n), ey = wrapn(y + qy - 1, n), ez = wrapn(z + qz - 1, n);
    const double* K = KE + ((size_t)b * N + ((size_t)ex * n + ey) * n + ez) * kk;
    const int aa = lidx(cx, cy, cz), bb = lidx(nx, ny, nz);
    for (int i = 0; i < D; ++i)
      for (int j = 0; j < D; ++j) C[i][j] += K[(D * aa + i) * k + D * bb + j];
  }
  for (int i = 0; i < D; ++i)
    for (int j = 0; j < D; ++j) {
      const size_t si = (((size_t)b * 27 + o) * D * D + i * D + j) * N + node;
      if (S) S[si] = (T)C[i][j];
      if (S64) S64[si] = C[i][j];
    }
  if (o == 13 && Dinv) {
    double Ci[D][D];
    block_inverse<double, D>(C, Ci);
    for (int i = 0; i < D; ++i)
      for (int j = 0; j < D; ++j) Dinv[((size_t)b * D * D + i * D + j) * N + node] = (T)Ci[i][j];
  }
}

// dense coarsest matrix from the FP64 stencil (n >= 3: the 27 neighbours are
// distinct), plus alpha * Z Z^T on the D translation modes.
template <int D>
__global__ void k_dense_from_stencil(const double* __restrict__ S64, double* __restrict__ A, int n, const int* active) {
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const int N = n * n * n, ndof = N * D;
  const int t = blockIdx.x * kThreads + threadIdx.x;
  if (t >= N * 27) return;
  const int node = t % N, o = t / N;
  const int z = node % n, y = (node / n) % n, x = node / (n * n);
  const int ox = o / 9 - 1, oy = (o / 3) % 3 - 1, oz = o % 3 - 1;
  const int m = (wrapn(x + ox, n) * n + wrapn(y + oy, n)) * n + wrapn(z + oz, n);
  double* Ab = A + (size_t)b * ndof * ndof;
  for (int i = 0; i < D; ++i)
    for (int j = 0; j < D; ++j)
      Ab[(size_t)(node * D + i) * ndof + m * D + j] = S64[(((size_t)b * 27 + o) * D * D + i * D + j) * N + node];
}

// In-place inverse of the SPD matrix A + alpha Z Z^T (one block per cell).
// Cholesky (lower) then inverse via L^-1; A is ndof x ndof FP64 in global memory,
// work holds ndof x ndof scratch.
__global__ void k_chol_inverse(double* __restrict__ A, double* __restrict__ work, int ndof, int D, const int* active,
                               int* status) {
  const int b = blockIdx.x;
  if (active && !active[b]) return;
  double* M = A + (size_t)b * ndof * ndof;
  double* Li = work + (size_t)b * ndof * ndof;
  __shared__ double s_alpha;
  // regularise: alpha = mean diagonal, Z columns = unit translation per component / sqrt(N)
  if (threadIdx.x == 0) {
    double s = 0;
    for (int i = 0; i < ndof; ++i) s += M[(size_t)i * ndof + i];
    s_alpha = s / ndof;
  }
  __syncthreads();
  const double alpha = s_alpha;
  const int Nn = ndof / D;
  for (int t = threadIdx.x; t < ndof * ndof; t += blockDim.x) {
    const int i = t / ndof, j = t % ndof;
    if ((i % D) == (j % D)) M[t] += alpha / Nn;
  }
  __syncthreads();
  // Cholesky, right-looking, lower triangle
  for (int kcol = 0; kcol < ndof; ++kcol) {
    __shared__ double s_piv;
    if (threadIdx.x == 0) {
      double d = M[(size_t)kcol * ndof + kcol];
      if (!(d > 0)) {
        if (status) status[b] = 1;
        d = 1e-300;
      }
      s_piv = sqrt(d);
      M[(size_t)kcol * ndof + kcol] = s_piv;
    }
    __syncthreads();
    const double piv = s_piv;
    for (int i = kcol + 1 + threadIdx.x; i < ndof; i += blockDim.x) M[(size_t)i * ndof + kcol] /= piv;
    __syncthreads();
    const int m = ndof - kcol - 1;
    for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
      const int i = kcol + 1 + t / m, j = kcol + 1 + t % m;
      if (j <= i) M[(size_t)i * ndof + j] -= M[(size_t)i * ndof + kcol] * M[(size_t)j * ndof + kcol];
    }
    __syncthreads();
  }
  // Li = L^-1 (lower), column by column: thread per column
  for (int j = threadIdx.x; j < ndof; j += blockDim.x) {
    for (int i = 0; i < ndof; ++i) {
      double s = (i == j) ? 1.0 : 0.0;
      for (int p = j; p < i; ++p) s -= M[(size_t)i * ndof + p] * Li[(size_t)p * ndof + j];
      Li[(size_t)i * ndof + j] = (i < j) ? 0.0 : s / M[(size_t)i * ndof + i];
    }
  }
  __syncthreads();
  // A^-1 = Li^T Li
  for (int t = threadIdx.x; t < ndof * ndof; t += blockDim.x) {
    const int i = t / ndof, j = t % ndof;
    const int p0 = i > j ? i : j;
    double s = 0;
    for (int p = p0; p < ndof; ++p) s += Li[(size_t)p * ndof + i] * Li[(size_t)p * ndof + j];
    M[t] = s;
  }
}

// Same result for ndof <= kCholSmemMax, with the packed lower triangle of the
// regularised matrix held in shared memory (one block of 1024 threads per cell).
constexpr int kCholSmemMax = 192;
constexpr int kCholThreads = 512;
constexpr int kCholPanel = 8;  // columns per panel of the blocked factorisation and inversion
// packed lower triangle of L (then of L^-1) and one panel of saved columns
__host__ __device__ constexpr size_t chol_smem_bytes(int ndof) {
  return ((size_t)ndof * (ndof + 1) / 2 + (size_t)kCholPanel * ndof) * sizeof(double);
}

// A <- (A + reg * I_blocks)^-1 for one cell per CTA, A symmetric positive
// (semi-)definite of order ndof <= kCholSmemMax: Cholesky factor L in shared
// memory, its inverse X = L^{-1} in place, then A^{-1} = X^T X.  The
// factorisation and the inversion run by panels of kCholPanel columns with
// three block barriers each: one warp factors the panel's diagonal block in
// registers, then every row below it is an independent triangular solve (one
// thread per row), and the rest of the matrix takes the panel as one
// rank-kCholPanel update.  The inversion mirrors it (the panel rows' columns
// are independent triangular solves, then a rank-kCholPanel update of the rows
// below).  A zero or negative pivot sets status[b] (nullable) and continues
// with a tiny pivot.
__global__ void __launch_bounds__(kCholThreads) k_chol_inverse_smem(double* __restrict__ A, int ndof, int D,
                                                                    const int* active, int* status) {
  constexpr int NB = kCholPanel;
  const int b = blockIdx.x;
  if (active && !active[b]) return;
  extern __shared__ double Lp[];  // packed lower triangle, row i starts at i(i+1)/2
  double* M = A + (size_t)b * ndof * ndof;
  const int tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nth >> 5;
  double* P = Lp + (size_t)ndof * (ndof + 1) / 2;  // panel columns of the rows below: P[q * ndof + i]
  // (column-major, so that lanes reading consecutive rows hit distinct banks)
  auto at = [&](int i, int j) -> double& { return Lp[(size_t)i * (i + 1) / 2 + j]; };
  __shared__ double sL[NB][NB];  // the panel's diagonal block of L
  __shared__ double sR[NB];      // reciprocals of its diagonal
  __shared__ double s_alpha;
  __shared__ int s_bad;
  if (warp == 0) {
    double t = 0;
    for (int i = lane; i < ndof; i += 32) t += M[(size_t)i * ndof + i];
    for (int off = 16; off > 0; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
    if (lane == 0) {
      s_alpha = t / ndof;
      s_bad = 0;
    }
  }
  __syncthreads();
  const double reg = s_alpha / (ndof / D);
  for (int i = warp; i < ndof; i += nw)
    for (int j = lane; j <= i; j += 32)
      Lp[(size_t)i * (i + 1) / 2 + j] = M[(size_t)i * ndof + j] + (((i - j) % D) == 0 ? reg : 0.0);
  __syncthreads();
  // ---- factorisation A = L L^T
  for (int k0 = 0; k0 < ndof; k0 += NB) {
    const int kb = min(NB, ndof - k0), k1 = k0 + kb;
    if (warp == 0) {
      // diagonal block, lane i holding row i, right-looking over its columns
      double a[NB];
#pragma unroll
      for (int q = 0; q < NB; ++q) a[q] = (lane < kb && q <= lane) ? at(k0 + lane, k0 + q) : 0.0;
      bool bad = false;
#pragma unroll
      for (int j = 0; j < NB; ++j) {
        if (j < kb) {
          double d = __shfl_sync(0xffffffffu, a[j], j);
          if (!(d > 0)) {
            bad = true;
            d = 1e-300;
          }
          const double piv = sqrt(d), rp = 1.0 / piv;
          if (lane == j) a[j] = piv;
          if (lane > j) a[j] *= rp;
#pragma unroll
          for (int q = j + 1; q < NB; ++q) {
            const double lqj = __shfl_sync(0xffffffffu, a[j], q);
            if (q < kb && lane >= q) a[q] -= a[j] * lqj;
          }
          if (lane == 0) sR[j] = rp;
        }
      }
      if (lane < NB)
#pragma unroll
        for (int q = 0; q < NB; ++q) sL[lane][q] = a[q];
      if (bad && lane == 0) s_bad = 1;
    }
    __syncthreads();
    // rows below the panel: L21 row i = A21 row i L11^{-T}
    for (int i = k1 + tid; i < ndof; i += nth) {
      double l[NB];
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        double v = q < kb ? at(i, k0 + q) : 0.0;
#pragma unroll
        for (int t = 0; t < q; ++t) v -= l[t] * sL[q][t];
        l[q] = q < kb ? v * sR[q] : 0.0;
      }
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        if (q < kb) at(i, k0 + q) = l[q];
        P[(size_t)q * ndof + i] = l[q];
      }
    }
    if (tid < NB * NB) {
      const int i = tid / NB, j = tid % NB;
      if (i < kb && j <= i) at(k0 + i, k0 + j) = sL[i][j];
    }
    __syncthreads();
    // trailing update: L[i][j] -= sum_q L[i][k0+q] L[j][k0+q], k1 <= j <= i
    for (int i = k1 + warp; i < ndof; i += nw) {
      double li[NB];
#pragma unroll
      for (int q = 0; q < NB; ++q) li[q] = P[(size_t)q * ndof + i];
      double* row = Lp + (size_t)i * (i + 1) / 2;
      for (int j = k1 + lane; j <= i; j += 32) {
        double sum = 0;
#pragma unroll
        for (int q = 0; q < NB; ++q) sum = fma(li[q], P[(size_t)q * ndof + j], sum);
        row[j] -= sum;
      }
    }
    __syncthreads();
  }
  if (status && tid == 0 && s_bad) status[b] = 1;
  // ---- X = L^{-1} in place of L.  Before panel p0, entry (i, j), j < p0 <= i,
  // holds b_ij = -sum_{p<p0} L_ip x_pj; the entries j >= p0 still hold L.
  for (int p0 = 0; p0 < ndof; p0 += NB) {
    const int pb = min(NB, ndof - p0), p1 = p0 + pb;
    if (tid < NB * NB) {
      const int i = tid / NB, j = tid % NB;
      sL[i][j] = (i < pb && j <= i) ? at(p0 + i, p0 + j) : 0.0;
      if (j == 0) sR[i] = i < pb ? 1.0 / at(p0 + i, p0 + i) : 0.0;
    }
    for (int i = p1 + tid; i < ndof; i += nth)
#pragma unroll
      for (int q = 0; q < NB; ++q) P[(size_t)q * ndof + i] = q < pb ? at(i, p0 + q) : 0.0;
    __syncthreads();
    // the panel rows: column j < p0 is x = L11^{-1} b (forward substitution);
    // column p0 + c of the diagonal block is L11^{-1} e_c
    for (int j = tid; j < p1; j += nth) {
      double x[NB];
      const int c = j - p0;  // >= 0 inside the diagonal block
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        double v;
        if (c < 0)
          v = q < pb ? at(p0 + q, j) : 0.0;
        else
          v = q == c ? 1.0 : 0.0;
#pragma unroll
        for (int t = 0; t < q; ++t) v -= sL[q][t] * x[t];
        x[q] = q < pb ? v * sR[q] : 0.0;
      }
#pragma unroll
      for (int q = 0; q < NB; ++q)
        if (q < pb && (c < 0 || q >= c)) at(p0 + q, j) = x[q];
    }
    __syncthreads();
    // rows below: entry (i, j), j < p1, becomes
    // (j < p0 ? b_ij : 0) - sum_q L_i,p0+q x_p0+q,j   (x_pj = 0 for j > p)
    for (int i = p1 + warp; i < ndof; i += nw) {
      double li[NB];
#pragma unroll
      for (int q = 0; q < NB; ++q) li[q] = P[(size_t)q * ndof + i];
      double* row = Lp + (size_t)i * (i + 1) / 2;
      for (int j = lane; j < p1; j += 32) {
        double sum = 0;
#pragma unroll
        for (int q = 0; q < NB; ++q) {
          const int p = p0 + q;
          if (q < pb && j <= p) sum = fma(li[q], at(p, j), sum);
        }
        row[j] = (j < p0 ? row[j] : 0.0) - sum;
      }
    }
    __syncthreads();
  }
  // A^{-1} = X^T X: entry (i, j) is sum_k X_ki X_kj over k >= max(i, j)
  // (X_kj = 0 for j > k).  A thread owns a 4 x 4 block (I, J), I <= J, of the
  // upper triangle and writes it and its mirror.
  const int nb = (ndof + 3) / 4, nblocks = nb * (nb + 1) / 2;
  for (int t = tid; t < nblocks; t += nth) {
    int I = 0, rem = t;  // t-th block of the packed upper block triangle, row-major
    while (rem >= nb - I) {
      rem -= nb - I;
      ++I;
    }
    const int J = I + rem;
    const int i0 = 4 * I, j0 = 4 * J;
    double acc[4][4] = {};
    size_t rk = (size_t)j0 * (j0 + 1) / 2;
    for (int k = j0; k < ndof; ++k) {
      double xi[4], xj[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        xi[a] = (i0 + a <= k && i0 + a < ndof) ? Lp[rk + i0 + a] : 0.0;
        xj[a] = (j0 + a <= k && j0 + a < ndof) ? Lp[rk + j0 + a] : 0.0;
      }
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[a][c] += xi[a] * xj[c];
      rk += k + 1;
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int i = i0 + a, j = j0 + c;
        if (i < ndof && j < ndof) {
          M[(size_t)i * ndof + j] = acc[a][c];
          M[(size_t)j * ndof + i] = acc[a][c];
        }
      }
  }
}

// ----------------------------------------------------------------------------
// right-hand sides, vectors, PCG scalars
// ----------------------------------------------------------------------------
// F = sum_e rho_e Fe0 gathered at nodes (utils/_utils.py:453-507)
template <int D, int R>
__global__ void k_assemble_F(const double* __restrict__ rho, double* __restrict__ F, int n, double scale,
                             const int* active) {
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const int N = n * n * n;
  const int idx = blockIdx.x * kThreads + threadIdx.x;
  if (idx >= N) return;
  const int z = idx % n, y = (idx / n) % n, x = idx / (n * n);
  double rq[8];
  load_rho8<double>(rho + (size_t)b * N, n, x, y, z, rq);
  double acc[R][D] = {};
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int qx = (q >> 2) & 1, qy = (q >> 1) & 1, qz = q & 1;
    const int aa = lidx(1 - qx, 1 - qy, 1 - qz);
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int i = 0; i < D; ++i) acc[r][i] += rq[q] * fe<D>(D * aa + i, r);
  }
  double* o = F + (size_t)b * N * R * D + idx;
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int i = 0; i < D; ++i) o[(size_t)(r * D + i) * N] = scale * acc[r][i];
}

// rho = rho_min + (1-rho_min) clamp(x,xmin,1)^p, FP64 and FP32 copies
__global__ void k_simp(const double* __restrict__ x, double* __restrict__ rho64, float* __restrict__ rho32, size_t total,
                       int N, double xmin, double penal, double rho_min, const int* active) {
  const size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x;
  if (i >= total) return;
  if (active && !active[i / N]) return;
  double xc = fmin(fmax(x[i], xmin), 1.0);
  double r = rho_min + (1.0 - rho_min) * pow(xc, penal);
  rho64[i] = r;
  if (rho32) rho32[i] = (float)r;
}

__global__ void k_copy_rho(const double* __restrict__ rho, double* __restrict__ rho64, float* __restrict__ rho32,
                           size_t total) {
  const size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x;
  if (i >= total) return;
  rho64[i] = rho[i];
  if (rho32) rho32[i] = (float)rho[i];
}

// partial dots x.y per rhs over [cell][node][R][D]
template <typename T, int R, int D>
__global__ void k_dot(const T* __restrict__ x, const T* __restrict__ y, double* __restrict__ part, int N,
                      const int* active) {
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const int idx = blockIdx.x * kThreads + threadIdx.x;
  double v[R] = {};
  if (idx < N) {
    const size_t o = (size_t)b * N * R * D + idx;
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int i = 0; i < D; ++i) {
        const size_t j = o + (size_t)(r * D + i) * N;
        v[r] += (double)x[j] * (double)y[j];
      }
  }
  block_sum_store<R>(v, part + ((size_t)b * gridDim.x + blockIdx.x) * R);
}

// x += alpha p ; r -= alpha q ; partial r.r   (alpha per cell/rhs)
template <typename T, int R, int D>
__global__ void k_pcg_update(T* __restrict__ x, T* __restrict__ r, const T* __restrict__ p, const T* __restrict__ q,
                             const double* __restrict__ alpha, double* __restrict__ part, int N, const int* active) {
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const int idx = blockIdx.x * kThreads + threadIdx.x;
  double v[R] = {};
  if (idx < N) {
    const size_t o = (size_t)b * N * R * D + idx;
#pragma unroll
    for (int c = 0; c < R; ++c) {
      const T a = (T)alpha[b * R + c];
#pragma unroll
      for (int i = 0; i < D; ++i) {
        const size_t j = o + (size_t)(c * D + i) * N;
        x[j] += a * p[j];
        const T rn = r[j] - a * q[j];
        r[j] = rn;
        v[c] += (double)rn * (double)rn;
      }
    }
  }
  block_sum_store<R>(v, part + ((size_t)b * gridDim.x + blockIdx.x) * R);
}

// The same two updates on 16-byte vectors (4 FP32 or 2 FP64 nodes per thread
// and load): twice to four times the bytes in flight per load instruction, which
// the FP32 update needs to reach the HBM roofline.  Requires N % W == 0; the
// partial sums are per block of kThreads vectors.


template <typename T, int R, int D, bool PDL = false>
__global__ void k_pcg_direction_vec(T* __restrict__ p, const T* __restrict__ z, const double* __restrict__ beta, int N,
                                    const int* active) {
  using V = typename Vec16<T>::type;
  constexpr int W = Vec16<T>::n;
  if constexpr (PDL) {
    griddep_wait();
    griddep_launch();
  }
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const int g = blockIdx.x * kThreads + threadIdx.x;
  const int NG = N / W;
  if (g >= NG) return;
  const size_t o = (size_t)b * NG * R * D + g;
#pragma unroll
  for (int c = 0; c < R; ++c) {
    const T be = (T)beta[b * R + c];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const size_t j = o + (size_t)(c * D + i) * NG;
      V pv = reinterpret_cast<const V*>(p)[j];
      const V zv = reinterpret_cast<const V*>(z)[j];
      T* ps = reinterpret_cast<T*>(&pv);
      const T* zs = reinterpret_cast<const T*>(&zv);
#pragma unroll
      for (int k = 0; k < W; ++k) ps[k] = zs[k] + be * ps[k];
      reinterpret_cast<V*>(p)[j] = pv;
    }
  }
}

// p = z + beta p
template <typename T, int R, int D>
__global__ void k_pcg_direction(T* __restrict__ p, const T* __restrict__ z, const double* __restrict__ beta, int N,
                                const int* active) {
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const int idx = blockIdx.x * kThreads + threadIdx.x;
  if (idx >= N) return;
  const size_t o = (size_t)b * N * R * D + idx;
#pragma unroll
  for (int c = 0; c < R; ++c) {
    const T be = (T)beta[b * R + c];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const size_t j = o + (size_t)(c * D + i) * N;
      p[j] = z[j] + be * p[j];
    }
  }
}

// Mixed-precision direction update from the FP32 preconditioner output:
// p = z + beta p with z = ||r|| z32 formed on the fly (the same explicitly
// rounded product as k_precond_back), so z is never stored in FP64.  FIRST:
// p = z (the first direction; p may hold anything before).
template <int R, int D, bool FIRST>
__global__ void k_pcg_direction_f32(double* __restrict__ p, const float* __restrict__ z32,
                                    const double* __restrict__ inv, const double* __restrict__ beta, int N,
                                    const int* active) {
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const int idx = blockIdx.x * kThreads + threadIdx.x;
  if (idx >= N) return;
  const size_t o = (size_t)b * N * R * D + idx;
#pragma unroll
  for (int c = 0; c < R; ++c) {
    const double s = inv[b * R + c];
    const double be = FIRST ? 0.0 : beta[b * R + c];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const size_t j = o + (size_t)(c * D + i) * N;
      const double zv = mul_rn(s, (double)z32[j]);
      p[j] = FIRST ? zv : fma_rn(be, p[j], zv);
    }
  }
}

// per-(cell,rhs) PCG scalar logic, one thread per (cell, rhs)
struct PcgScalars {
  double* rz;      // r.z
  double* rz_new;  // reduced r.z of the new z
  double* pq;      // reduced p.q
  double* rr;      // reduced r.r
  double* bnorm2;  // ||b||^2 of the system being solved
  double* alpha;
  double* beta;
  int* done;       // per (cell,rhs)
  int* cell_done;  // per cell
  int* iters;      // per cell
};

// convert an FP64 vector to FP32 with a per-(cell,rhs) scale; and back (add)
template <int R, int D>
__global__ void k_to_f32_scaled(const double* __restrict__ src, float* __restrict__ dst, const double* __restrict__ inv_scale,
                                int N, const int* active) {
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const int idx = blockIdx.x * kThreads + threadIdx.x;
  if (idx >= N) return;
  const size_t o = (size_t)b * N * R * D + idx;
#pragma unroll
  for (int c = 0; c < R; ++c) {
    const double s = inv_scale[b * R + c];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const size_t j = o + (size_t)(c * D + i) * N;
      dst[j] = (float)(src[j] * s);
    }
  }
}

template <int R, int D>
__global__ void k_add_f32_scaled(double* __restrict__ dst, const float* __restrict__ src, const double* __restrict__ scale,
                                 int N, const int* active) {
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const int idx = blockIdx.x * kThreads + threadIdx.x;
  if (idx >= N) return;
  const size_t o = (size_t)b * N * R * D + idx;
#pragma unroll
  for (int c = 0; c < R; ++c) {
    const double s = scale[b * R + c];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const size_t j = o + (size_t)(c * D + i) * N;
      dst[j] += s * (double)src[j];
    }
  }
}

// Reliable updates of the mixed-precision PCG (the iteration in FP32 on a
// residual scaled to unit norm, FP64 residual replacement).  Cells with
// flag[b] set fold the FP32 correction into the FP64 iterate,
// x += inv * x32 (inv: the column's residual norm at the last replacement),
// and restart the correction, x32 = 0.
template <int R, int D>
__global__ void k_flush_f32(double* __restrict__ x, float* __restrict__ x32, const double* __restrict__ inv, int N,
                            const int* flag) {
  const int b = blockIdx.y;
  if (flag && !flag[b]) return;
  const int idx = blockIdx.x * kThreads + threadIdx.x;
  if (idx >= N) return;
  const size_t o = (size_t)b * N * R * D + idx;
#pragma unroll
  for (int c = 0; c < R; ++c) {
    const double s = inv[b * R + c];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const size_t j = o + (size_t)(c * D + i) * N;
      x[j] = fma(s, (double)x32[j], x[j]);
      x32[j] = 0.0f;
    }
  }
}

// After the FP64 residual r of the flushed iterate: r32 = scale * r
// (scale = 1 / ||r||), and the direction and its image rescaled to the new
// unit, p32 *= t, q32 *= t (t = old ||r|| / new ||r||).  Cells with flag[b].
template <int R, int D>
__global__ void k_rel_rescale(const double* __restrict__ r, float* __restrict__ r32, float* __restrict__ p32,
                              float* __restrict__ q32, const double* __restrict__ scale, const double* __restrict__ t,
                              int N, const int* flag) {
  const int b = blockIdx.y;
  if (flag && !flag[b]) return;
  const int idx = blockIdx.x * kThreads + threadIdx.x;
  if (idx >= N) return;
  const size_t o = (size_t)b * N * R * D + idx;
#pragma unroll
  for (int c = 0; c < R; ++c) {
    const double sc = scale[b * R + c];
    const float tc = (float)t[b * R + c];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const size_t j = o + (size_t)(c * D + i) * N;
      r32[j] = (float)(r[j] * sc);
      p32[j] *= tc;
      q32[j] *= tc;
    }
  }
}

// partial dots r.z and (optionally) q.z of z = inv * z32, formed in FP64 and
// not stored (k_pcg_direction_f32 forms it again for the direction update)
template <int R, int D>
__global__ void k_precond_back(const float* __restrict__ z32, const double* __restrict__ inv,
                               const double* __restrict__ r, const double* __restrict__ q, double* __restrict__ part,
                               int N, const int* active) {
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const int idx = blockIdx.x * kThreads + threadIdx.x;
  double v[2 * R] = {};
  if (idx < N) {
    const size_t o = (size_t)b * N * R * D + idx;
#pragma unroll
    for (int c = 0; c < R; ++c) {
      const double s = inv[b * R + c];
#pragma unroll
      for (int i = 0; i < D; ++i) {
        const size_t j = o + (size_t)(c * D + i) * N;
        const double zv = mul_rn(s, (double)z32[j]);
        v[c] += r[j] * zv;
        if (q) v[R + c] += q[j] * zv;
      }
    }
  }
  block_sum_store<2 * R>(v, part + ((size_t)b * gridDim.x + blockIdx.x) * 2 * R);
}

// A block per cell reduces that cell's partial sums (as k_reduce_partials) and
// then its first R lanes (one per load case) apply the PCG scalar step that
// consumes them, one launch instead of two:
//   ALPHA      alpha = rz / p.q, or freeze the column (done = 2) on a breakdown
//              (p.q <= 0 or non-finite)
//   CHECK      advance the iteration count (count), mark columns with
//              ||r||^2 <= rtol^2 ||b||^2 done, the cell done when all are, clear
//              its run flag, and (scale != NULL) the column scales 1/||r||, ||r||
//   BETA       beta = rz_new / rz, rz = rz_new
//   BETA_FLEX  flexible beta = -alpha (q.z) / rz, rz = r.z (first: beta = 0)
//   SET_RZ     rz = rz_new
//   RELCHECK   (reliable updates) advance the iteration count and flag the cell
//              for a residual replacement (rel) when a live column's recurrence
//              residual, in units of its last replaced residual (inv), fell
//              below delta2 (squared) or passes the tolerance test; no column is
//              marked done here
//   RELSET     (flagged cells) the true residual norms of the replacement: mark
//              columns with ||r||^2 <= rtol^2 ||b||^2 done (the cell done when
//              all are, its run flag cleared), set scale = 1/||r||, t = old
//              ||r|| / new ||r||, inv = ||r||, and rz *= t^2
enum { RED_PLAIN = 0, RED_ALPHA = 1, RED_CHECK = 2, RED_BETA = 3, RED_BETA_FLEX = 4, RED_SET_RZ = 5,
       RED_RELCHECK = 6, RED_RELSET = 7 };
struct RedOp {
  PcgScalars s;
  int R = 0;
  int* breakdown = nullptr;  // ALPHA
  double rtol2 = 0;          // CHECK (used when rtol2_dev is NULL)
  const double* rtol2_dev = nullptr;  // CHECK: rtol^2 read on device, so captured graphs serve any tolerance
  int count = 0;             // CHECK: advance the iteration counter
  int* run = nullptr;        // CHECK: run flags cleared for finished cells
  double* scale = nullptr;   // CHECK: column scales 1/||r|| and ||r|| (nullable)
  double* inv = nullptr;
  int first = 0;             // BETA_FLEX
  int* rel = nullptr;        // RELCHECK, RELSET: per cell, a residual replacement is due
  double delta2 = 0;         // RELCHECK: squared reduction per FP32 segment
  double* t = nullptr;       // RELSET: rescaling of the direction
  // Inside a captured graph: the conditional IF handle around the residual
  // replacement (0: none), cleared by ALPHA and set by RELCHECK when a cell has
  // a replacement due; RELSET inside the IF body counts its executions.
  cudaGraphConditionalHandle cond = 0;
  int* cond_count = nullptr;
};

// The body of k_reduce_op for cell b, run by a whole block of kThreads
// threads (the partials are read through L2: the last block of the grid that
// wrote them may run it, see k_pcg_update_vec).
template <int K, int OP>
__device__ __forceinline__ void reduce_op_cell(const double* __restrict__ part, int nblk, double* __restrict__ out,
                                               RedOp& op, int b) {
  double v[K];
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = 0;
  for (int i = threadIdx.x; i < nblk; i += kThreads) {
    const double* p = part + ((size_t)b * nblk + i) * K;
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] += __ldcg(p + k);
  }
  block_sum_store<K>(v, out + (size_t)b * K);
  if constexpr (OP == RED_PLAIN) return;
  __syncthreads();
  if (threadIdx.x >= 32) return;
  // lane c < R handles load case c (the cell-level test is a warp vote)
  PcgScalars& s = op.s;
  const int R = op.R, c = threadIdx.x;
  const bool col = c < R;
  const int i = b * R + c;
  if constexpr (OP == RED_ALPHA) {
    if (op.cond && b == 0 && c == 0) cudaGraphSetConditional(op.cond, 0u);
    if (col) {
      double a = 0.0;
      if (!s.done[i]) {
        const double pq = s.pq[i];
        if (pq > 0.0 && isfinite(pq)) {
          a = s.rz[i] / pq;
        } else {
          s.done[i] = 2;  // breakdown: freeze this column
          if (op.breakdown) atomicOr(op.breakdown, 1);
        }
      }
      s.alpha[i] = a;
    }
  } else if constexpr (OP == RED_CHECK) {
    const int was_done = s.cell_done[b];
    int dn = 1;
    if (col) {
      dn = s.done[i];
      const double rt2 = op.rtol2_dev ? *op.rtol2_dev : op.rtol2;
      if (!was_done && !dn && s.rr[i] <= rt2 * s.bnorm2[i]) {
        dn = 1;
        s.done[i] = 1;
      }
    }
    const bool all = __all_sync(0xffffffffu, dn != 0);
    if (c == 0) {
      if (!was_done) {
        if (op.count) s.iters[b] += 1;
        if (all) s.cell_done[b] = 1;
      }
      if (was_done || all) op.run[b] = 0;
    }
    if (col && op.scale) {
      const double nrm = sqrt(fmax(s.rr[i], 0.0));
      op.scale[i] = nrm > 0 ? 1.0 / nrm : 0.0;
      op.inv[i] = nrm;
    }
  } else if constexpr (OP == RED_BETA) {
    if (col) {
      double be = 0.0;
      if (!s.done[i] && s.rz[i] != 0.0) be = s.rz_new[i] / s.rz[i];
      s.beta[i] = be;
      s.rz[i] = s.rz_new[i];
    }
  } else if constexpr (OP == RED_BETA_FLEX) {
    if (col) {
      const double* red = out + (size_t)b * K;
      const double rz_new = red[c], zq = red[R + c];
      double be = 0.0;
      if (!op.first && !s.done[i] && s.rz[i] != 0.0) be = -s.alpha[i] * zq / s.rz[i];
      s.beta[i] = be;
      s.rz[i] = rz_new;
    }
  } else if constexpr (OP == RED_SET_RZ) {
    if (col) s.rz[i] = s.rz_new[i];
  } else if constexpr (OP == RED_RELCHECK) {
    const int was_done = s.cell_done[b];
    int due = 0;
    if (col && !was_done && !s.done[i]) {
      const double rt2 = op.rtol2_dev ? *op.rtol2_dev : op.rtol2;
      const double rr = s.rr[i], nrm = op.inv[i];
      due = rr <= op.delta2 || rr * nrm * nrm <= rt2 * s.bnorm2[i];
    }
    const bool any = __any_sync(0xffffffffu, due != 0);
    if (c == 0) {
      if (!was_done && op.count) s.iters[b] += 1;
      op.rel[b] = any ? 1 : 0;
      if (op.cond && any) cudaGraphSetConditional(op.cond, 1u);
    }
  } else if constexpr (OP == RED_RELSET) {
    if (op.cond_count && b == 0 && c == 0) atomicAdd(op.cond_count, 1);
    if (!op.rel[b]) return;
    int dn = 1;
    if (col) {
      const double rr = out[(size_t)b * K + c];
      const double rt2 = op.rtol2_dev ? *op.rtol2_dev : op.rtol2;
      dn = s.done[i];
      if (!dn && rr <= rt2 * s.bnorm2[i]) {
        dn = 1;
        s.done[i] = 1;
      }
      const double nrm = sqrt(fmax(rr, 0.0));
      const double tt = nrm > 0 ? op.inv[i] / nrm : 0.0;
      op.scale[i] = nrm > 0 ? 1.0 / nrm : 0.0;
      op.t[i] = tt;
      op.inv[i] = nrm;
      s.rz[i] *= tt * tt;
    }
    const bool all = __all_sync(0xffffffffu, dn != 0);
    if (c == 0 && all) {
      s.cell_done[b] = 1;
      op.run[b] = 0;
    }
  }
}

template <int K, int OP, bool PDL = false>
__global__ void k_reduce_op(const double* __restrict__ part, int nblk, double* __restrict__ out, RedOp op) {
  if constexpr (PDL) {
    griddep_wait();
    griddep_launch();
  }
  reduce_op_cell<K, OP>(part, nblk, out, op, blockIdx.x);
}

// FIN (RED_CHECK or RED_RELCHECK; 0: none): the last block of a cell to
// finish runs that reduction of the cell's partial sums itself (the block
// count and summation order of k_reduce_op), so the step needs no separate
// reduction launch; fin_count[cell] counts the finished blocks and is reset
// by the last one.
template <typename T, int R, int D, bool PDL = false, int FIN = 0>
__global__ void k_pcg_update_vec(T* __restrict__ x, T* __restrict__ r, const T* __restrict__ p,
                                 const T* __restrict__ q, const double* __restrict__ alpha, double* __restrict__ part,
                                 int N, const int* active, unsigned* fin_count, double* fin_out, RedOp fin_op) {
  using V = typename Vec16<T>::type;
  constexpr int W = Vec16<T>::n;
  if constexpr (PDL) {
    griddep_wait();
    griddep_launch();
  }
  const int b = blockIdx.y;
  if (active && !active[b]) {
    // a finished or inactive cell: what the reduction would have left it
    if constexpr (FIN == RED_RELCHECK) {
      if (blockIdx.x == 0 && threadIdx.x == 0) fin_op.rel[b] = 0;
    }
    return;
  }
  const int g = blockIdx.x * kThreads + threadIdx.x;
  const int NG = N / W;
  double v[R] = {};
  if (g < NG) {
    const size_t o = (size_t)b * NG * R * D + g;
#pragma unroll
    for (int c = 0; c < R; ++c) {
      const T a = (T)alpha[b * R + c];
#pragma unroll
      for (int i = 0; i < D; ++i) {
        const size_t j = o + (size_t)(c * D + i) * NG;
        V xv = reinterpret_cast<const V*>(x)[j], rv = reinterpret_cast<const V*>(r)[j];
        const V pv = reinterpret_cast<const V*>(p)[j], qv = reinterpret_cast<const V*>(q)[j];
        T* xs = reinterpret_cast<T*>(&xv);
        T* rs = reinterpret_cast<T*>(&rv);
        const T* ps = reinterpret_cast<const T*>(&pv);
        const T* qs = reinterpret_cast<const T*>(&qv);
#pragma unroll
        for (int k = 0; k < W; ++k) {
          xs[k] += a * ps[k];
          const T rn = rs[k] - a * qs[k];
          rs[k] = rn;
          v[c] += (double)rn * (double)rn;
        }
        reinterpret_cast<V*>(x)[j] = xv;
        reinterpret_cast<V*>(r)[j] = rv;
      }
    }
  }
  block_sum_store<R>(v, part + ((size_t)b * gridDim.x + blockIdx.x) * R);
  if constexpr (FIN != 0) {
    __shared__ int s_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(fin_count + b, 1u) == gridDim.x - 1;
    __syncthreads();
    if (s_last) {
      __threadfence();
      reduce_op_cell<R, FIN>(part, gridDim.x, fin_out, fin_op, b);
      if (threadIdx.x == 0) fin_count[b] = 0;
    }
  }
}


// deterministic pseudo-random start vector for power iterations
template <typename T>
__global__ void k_power_init(T* __restrict__ v, size_t total) {
  const size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x;
  if (i >= total) return;
  unsigned h = (unsigned)(i * 2654435761u) ^ 0x9e3779b9u;
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  v[i] = (T)(((h & 0xffffff) / 8388608.0) - 1.0);
}

// hi[cell] = safety * (u.Au)/(u.Du) from the reduced Rayleigh terms
__global__ void k_power_finish(const double* __restrict__ red, double* __restrict__ hi, int B, double safety) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  const double num = red[2 * b], den = red[2 * b + 1];
  double lam = (den > 0 && num > 0) ? num / den : 2.0;
  hi[b] = safety * lam;
}

// ----------------------------------------------------------------------------
// homogenization, sensitivity, objective, filter, OC
// ----------------------------------------------------------------------------
// per element (X0-u_e)^T Ke0 (X0-u_e) -> energy[cell][e][R][R]; partial sums of
// rho_e * energy for C^H / kappa^H (model.py:33-95)
template <int D, int R>
__global__ void __launch_bounds__(kThreads) k_homogenize(const double* __restrict__ u, const double* __restrict__ rho,
                                                         double* __restrict__ energy, double* __restrict__ part, int n,
                                                         double kscale, double xscale, const int* active) {
  constexpr int k = 8 * D;
  constexpr int K = R * (R + 1) / 2;
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const int N = n * n * n;
  const int e = blockIdx.x * kThreads + threadIdx.x;
  const bool valid = e < N;
  const int ee = valid ? e : 0;
  const int z = ee % n, y = (ee / n) % n, x = ee / (n * n);
  int nodes[8];
#pragma unroll
  for (int a = 0; a < 8; ++a)
    nodes[a] = (wrapn(x + corner_x(a), n) * n + wrapn(y + corner_y(a), n)) * n + wrapn(z + corner_z(a), n);
  const double* __restrict__ ub = u + (size_t)b * N * R * D;
  const double re = valid ? rho[(size_t)b * N + ee] : 0.0;
  double* eo = energy + (size_t)b * R * R * N + ee;  // [cell][r][s][elem]
  double v[K];
#pragma unroll
  for (int s = 0; s < R; ++s) {
    double KL[k];
    {
      double L[k];
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int i = 0; i < D; ++i)
          L[D * a + i] = xscale * x0<D>(D * a + i, s) - __ldg(ub + (size_t)(s * D + i) * N + nodes[a]);
#pragma unroll
      for (int p = 0; p < k; ++p) {
        double acc = 0;
#pragma unroll
        for (int q = 0; q < k; ++q) acc += ke<double, D>(p, q) * L[q];
        KL[p] = kscale * acc;
      }
    }
#pragma unroll
    for (int r = 0; r <= s; ++r) {
      double acc = 0;
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int i = 0; i < D; ++i)
          acc += (xscale * x0<D>(D * a + i, r) - __ldg(ub + (size_t)(r * D + i) * N + nodes[a])) * KL[D * a + i];
      // index of (r,s), r <= s, in the packed upper triangle
      v[r * R - r * (r - 1) / 2 + (s - r)] = re * acc;
      if (valid) {
        eo[(size_t)(r * R + s) * N] = acc;
        eo[(size_t)(s * R + r) * N] = acc;
      }
    }
  }
  block_sum_store<K>(v, part + ((size_t)b * gridDim.x + blockIdx.x) * K);
}

// The elastic form (D = 3, R = 6) with the same energies, register-lean:
// warp s of a 192-thread block owns load case s of 32 consecutive elements,
// eight such groups per block (256 elements: the generic kernel's partial-sum
// count).  The six fields X0 - u_e of a group meet in shared memory, so a
// thread holds only its K (X0 - u_e) column (the generic kernel held both
// vectors of every pair and ran at one block per SM).  Energies are formed
// with the generic kernel's operations in its order (bit-identical); the
// block partial sums of C^H add in a different order.
constexpr int kHomWarps = 6, kHomGroups = 8;
__global__ void __launch_bounds__(32 * kHomWarps) k_homogenize_elastic(const double* __restrict__ u,
                                                                      const double* __restrict__ rho,
                                                                      double* __restrict__ energy,
                                                                      double* __restrict__ part, int n,
                                                                      double kscale, double xscale,
                                                                      const int* active) {
  constexpr int D = 3, R = 6, k = 24, K = 21;
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const int N = n * n * n;
  const int s = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __shared__ double sL[R][k][33];
  __shared__ double sv[K];
  const double* __restrict__ ub = u + (size_t)b * N * R * D;
  double vacc[R];
#pragma unroll
  for (int r = 0; r < R; ++r) vacc[r] = 0;
  for (int grp = 0; grp < kHomGroups; ++grp) {
    const int e = (blockIdx.x * kHomGroups + grp) * 32 + lane;
    const bool valid = e < N;
    const int ee = valid ? e : 0;
    const int z = ee % n, y = (ee / n) % n, x = ee / (n * n);
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const int node = (wrapn(x + corner_x(a), n) * n + wrapn(y + corner_y(a), n)) * n + wrapn(z + corner_z(a), n);
#pragma unroll
      for (int i = 0; i < D; ++i)
        sL[s][D * a + i][lane] = xscale * x0<D>(D * a + i, s) - __ldg(ub + (size_t)(s * D + i) * N + node);
    }
    __syncthreads();
    double KL[k];
#pragma unroll
    for (int p = 0; p < k; ++p) KL[p] = 0;
#pragma unroll
    for (int q = 0; q < k; ++q) {
      const double lq = sL[s][q][lane];
#pragma unroll
      for (int p = 0; p < k; ++p) KL[p] += ke<double, D>(p, q) * lq;
    }
#pragma unroll
    for (int p = 0; p < k; ++p) KL[p] = kscale * KL[p];
    const double re = valid ? rho[(size_t)b * N + ee] : 0.0;
    double* eo = energy + (size_t)b * R * R * N + ee;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (r <= s) {
        double acc = 0;
#pragma unroll
        for (int q = 0; q < k; ++q) acc += sL[r][q][lane] * KL[q];
        vacc[r] += re * acc;
        if (valid) {
          eo[(size_t)(r * R + s) * N] = acc;
          eo[(size_t)(s * R + r) * N] = acc;
        }
      }
    }
    __syncthreads();
  }
  // pair (r, s), r <= s: warp s, component r; packed upper-triangle index
#pragma unroll
  for (int r = 0; r < R; ++r) {
    double v = vacc[r];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0 && r <= s) sv[r * R - r * (r - 1) / 2 + (s - r)] = v;
  }
  __syncthreads();
  if (threadIdx.x < K) part[((size_t)b * gridDim.x + blockIdx.x) * K + threadIdx.x] = sv[threadIdx.x];
}

// unpack reduced upper triangles into full symmetric matrices H[cell][R][R]
__global__ void k_unpack_sym(const double* __restrict__ red, double* __restrict__ H, int B, int R) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  const int K = R * (R + 1) / 2;
  int m = 0;
  for (int r = 0; r < R; ++r)
    for (int s = r; s < R; ++s) {
      const double v = red[b * K + m++];
      H[(b * R + r) * R + s] = v;
      H[(b * R + s) * R + r] = v;
    }
}

// objective J = wE*E + wG*G + wK*trace(kappa) and its gradients
// (maple/core/utils/objective.py:11-41, 180-251), one thread per cell.
__device__ void inv6(const double (&A)[6][6], double (&Ai)[6][6]) {
  double M[6][12];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      M[i][j] = A[i][j];
      M[i][6 + j] = (i == j) ? 1.0 : 0.0;
    }
  for (int k = 0; k < 6; ++k) {
    int p = k;
    for (int i = k + 1; i < 6; ++i)
      if (fabs(M[i][k]) > fabs(M[p][k])) p = i;
    if (p != k)
      for (int j = 0; j < 12; ++j) {
        double t = M[k][j];
        M[k][j] = M[p][j];
        M[p][j] = t;
      }
    const double d = M[k][k];
    for (int j = 0; j < 12; ++j) M[k][j] /= d;
    for (int i = 0; i < 6; ++i)
      if (i != k) {
        const double f = M[i][k];
        for (int j = 0; j < 12; ++j) M[i][j] -= f * M[k][j];
      }
  }
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) Ai[i][j] = M[i][6 + j];
}

__global__ void k_objective(const double* __restrict__ CH, const double* __restrict__ KAP, const double* __restrict__ w,
                            double* __restrict__ J, double* __restrict__ terms, double* __restrict__ G3,
                            double* __restrict__ G1, int B, int need_ch, int need_k, const int* active) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  if (active && !active[b]) return;
  const double wE = w[3 * b], wG = w[3 * b + 1], wK = w[3 * b + 2];
  double j = 0, tE = 0, tG = 0, tK = 0;
  double g3[6][6] = {};
  if (need_ch) {
    double C[6][6], S[6][6];
    for (int r = 0; r < 6; ++r)
      for (int s = 0; s < 6; ++s) C[r][s] = 0.5 * (CH[(b * 6 + r) * 6 + s] + CH[(b * 6 + s) * 6 + r]) + (r == s ? 1e-9 : 0.0);
    inv6(C, S);
    for (int t = 0; t < 2; ++t) {
      const double wt = t == 0 ? wE : wG;
      double val = 0;
      for (int ii = 0; ii < 3; ++ii) {
        const int i = 3 * t + ii;
        val += 1.0 / S[i][i];
        if (wt != 0.0) {
          const double f = wt / 3.0 / (S[i][i] * S[i][i]);
          for (int r = 0; r < 6; ++r)
            for (int s = 0; s < 6; ++s) g3[r][s] += f * S[r][i] * S[i][s];
        }
      }
      val /= 3.0;
      if (t == 0) tE = val; else tG = val;
      j += wt * val;
    }
  }
  if (need_k) {
    tK = KAP[b * 9 + 0] + KAP[b * 9 + 4] + KAP[b * 9 + 8];
    j += wK * tK;
  }
  J[b] = j;
  terms[3 * b] = tE;
  terms[3 * b + 1] = tG;
  terms[3 * b + 2] = tK;
  for (int r = 0; r < 6; ++r)
    for (int s = 0; s < 6; ++s) G3[(b * 6 + r) * 6 + s] = 0.5 * (g3[r][s] + g3[s][r]);
  for (int r = 0; r < 3; ++r)
    for (int s = 0; s < 3; ++s) G1[(b * 3 + r) * 3 + s] = (r == s) ? wK : 0.0;
}

// dJ/dx_e = p (1-rho_min) xc^(p-1) * (G3 : E3_e + G1 : E1_e)
// dJ/drho_e = sum_ij G_ij dH_ij/drho_e (energies E) - lp dPp/drho_e - lc dPc/drho_e
// (penalty gradients nullable), and dJ/dx_e through the SIMP map
__global__ void k_sensitivity(const double* __restrict__ x, const double* __restrict__ E3, const double* __restrict__ E1,
                              const double* __restrict__ G3, const double* __restrict__ G1, double* __restrict__ dJdx,
                              double* __restrict__ dJdrho, int N, double xmin, double penal, double rho_min,
                              const int* active, const double* __restrict__ dPp = nullptr, double lp = 0.0,
                              const double* __restrict__ dPc = nullptr, double lc = 0.0) {
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const int e = blockIdx.x * kThreads + threadIdx.x;
  if (e >= N) return;
  const size_t i = (size_t)b * N + e;
  double s = 0;
  if (E3) {
    const double* Ee = E3 + (size_t)b * 36 * N + e;
    const double* G = G3 + (size_t)b * 36;
#pragma unroll
    for (int k = 0; k < 36; ++k) s += G[k] * Ee[(size_t)k * N];
  }
  if (E1) {
    const double* Ee = E1 + (size_t)b * 9 * N + e;
    const double* G = G1 + (size_t)b * 9;
#pragma unroll
    for (int k = 0; k < 9; ++k) s += G[k] * Ee[(size_t)k * N];
  }
  if (dPp) s -= lp * dPp[i];
  if (dPc) s -= lc * dPc[i];
  if (dJdrho) dJdrho[i] = s;
  if (dJdx) {
    const double xv = x[i];
    const double xc = fmin(fmax(xv, xmin), 1.0);
    const double inside = (xv >= xmin && xv <= 1.0) ? 1.0 : 0.0;
    dJdx[i] = inside * s * penal * (1.0 - rho_min) * pow(xc, penal - 1.0);
  }
}

// out[b][e] (+)= sum_k g[b][k] * energy[b][e][k]
__global__ void k_energy_contract(const double* __restrict__ energy, const double* __restrict__ g,
                                  double* __restrict__ out, int N, int RR, int accumulate) {
  const int b = blockIdx.y;
  const int e = blockIdx.x * kThreads + threadIdx.x;
  if (e >= N) return;
  const size_t i = (size_t)b * N + e;
  const double* Ee = energy + (size_t)b * RR * N + e;
  const double* gb = g + (size_t)b * RR;
  double s = 0;
  for (int k = 0; k < RR; ++k) s += gb[k] * Ee[(size_t)k * N];
  out[i] = accumulate ? out[i] + s : s;
}

// Symmetry projection of element fields (main_IHD_v3.py:259-337): the mean of
// the field over a group of cube maps, voxel index i reflecting to n-1-i.
// kind 1 (mirror): the reflections about the centre planes of the axes in
// mask (bit 0 = x, 1 = y, 2 = z); kind 2 (cubic): all 48 axis permutations and
// reflections.  With clamp, inputs are clamped to [lo, hi] before averaging
// and the mean after it (the clamps around the projection of the OC loop).
enum { SYM_NONE = 0, SYM_MIRROR = 1, SYM_CUBIC = 2 };

__global__ void k_symmetrize(const double* __restrict__ in, double* __restrict__ out, int n, int kind, int mask,
                             int clamp, double lo, double hi, const int* active) {
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const int N = n * n * n;
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= N) return;
  const int c[3] = {v / (n * n), (v / n) % n, v % n};
  const double* src = in + (size_t)b * N;
  auto at = [&](int a0, int a1, int a2) {
    const double t = src[(a0 * n + a1) * n + a2];
    return clamp ? fmin(fmax(t, lo), hi) : t;
  };
  double acc = 0.0;
  int cnt = 0;
  if (kind == SYM_MIRROR) {
    for (int f = 0; f < 8; ++f) {
      if (f & ~mask) continue;
      acc += at((f & 1) ? n - 1 - c[0] : c[0], (f & 2) ? n - 1 - c[1] : c[1], (f & 4) ? n - 1 - c[2] : c[2]);
      ++cnt;
    }
  } else if (kind == SYM_CUBIC) {
    constexpr int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
#pragma unroll 1
    for (int p = 0; p < 6; ++p) {
      const int q0 = c[perm[p][0]], q1 = c[perm[p][1]], q2 = c[perm[p][2]];
#pragma unroll
      for (int f = 0; f < 8; ++f)
        acc += at((f & 1) ? n - 1 - q0 : q0, (f & 2) ? n - 1 - q1 : q1, (f & 4) ? n - 1 - q2 : q2);
    }
    cnt = 48;
  } else {
    acc = at(c[0], c[1], c[2]);
    cnt = 1;
  }
  double r = acc / cnt;
  if (clamp) r = fmin(fmax(r, lo), hi);
  out[(size_t)b * N + v] = r;
}

// per-cell max |x1 - x0| and mean |x1 - x0| into stats [B][2]; one CTA per cell
__global__ void __launch_bounds__(1024) k_dx_stats(const double* __restrict__ x0, const double* __restrict__ x1,
                                                   double* __restrict__ stats, int N, const int* active) {
  const int b = blockIdx.x;
  if (active && !active[b]) return;
  __shared__ double smax[32], ssum[32];
  double mx = 0.0, sm = 0.0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const double d = fabs(x1[(size_t)b * N + i] - x0[(size_t)b * N + i]);
    mx = fmax(mx, d);
    sm += d;
  }
  for (int off = 16; off > 0; off >>= 1) {
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
    sm += __shfl_down_sync(0xffffffffu, sm, off);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    smax[warp] = mx;
    ssum[warp] = sm;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0, t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      m = fmax(m, smax[w]);
      t += ssum[w];
    }
    stats[2 * b] = m;
    stats[2 * b + 1] = t / N;
  }
}

// periodic k^3 box mean (main_IHD_v3.py:342-359)
__global__ void k_box_filter(const double* __restrict__ in, double* __restrict__ out, int n, int kf, const int* active) {
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const int N = n * n * n;
  const int e = blockIdx.x * kThreads + threadIdx.x;
  if (e >= N) return;
  const int z = e % n, y = (e / n) % n, x = e / (n * n);
  const int p = kf / 2;
  const double* ib = in + (size_t)b * N;
  double s = 0;
  for (int dx = -p; dx <= p; ++dx) {
    const int xx = ((x + dx) % n + n) % n;
    for (int dy = -p; dy <= p; ++dy) {
      const int yy = ((y + dy) % n + n) % n;
      for (int dz = -p; dz <= p; ++dz) {
        const int zz = ((z + dz) % n + n) % n;
        s += ib[((size_t)xx * n + yy) * n + zz];
      }
    }
  }
  out[(size_t)b * N + e] = s / (double)(kf * kf * kf);
}

// Bounded grid barrier for co-resident (cooperatively launched) blocks.  A
// block whose wait runs past `limit` polls, or that finds another block has
// already given up, raises *err and returns false; the caller then returns at
// once, so a barrier that cannot complete ends the kernel instead of hanging it
// (and every later barrier of the launch gives up immediately).  `nblocks` is
// the number of blocks expected to arrive.
__device__ __forceinline__ bool grid_barrier(unsigned* count, unsigned* gen, unsigned nblocks, int* err,
                                             long long limit) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = gen;
    volatile int* verr = err;
    int ok = 1;
    if (*verr) {
      ok = 0;
    } else {
      const unsigned g = *vgen;
      __threadfence();
      const unsigned arrived = atomicAdd(count, 1u);
      if (arrived == nblocks - 1) {
        atomicExch(count, 0u);
        __threadfence();
        atomicAdd(gen, 1u);
      } else {
        long long polls = 0;
        while (*vgen == g) {
          if (++polls > limit || *verr) {
            atomicExch(err, 1);
            ok = 0;
            break;
          }
          if (polls > 4096) __nanosleep(32);
        }
      }
      __threadfence();
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// default poll limit of grid_barrier: the OC kernel's blocks arrive within
// microseconds of each other; 2^24 polls (several seconds) only bound a wait
// that can never end
constexpr long long kBarrierPolls = 1LL << 24;

// OC update with 60 bisection steps on lambda in [1e-12, 1e6]
// (main_IHD_v3.py:362-380).  Grid (G, B): G co-resident blocks per cell.
// The returned x is that of the last bisection step, as in the reference.
struct OcArgs {
  const double* x;
  const double* dJ;
  double* xnew;
  const double* volfrac;  // [B]
  double move, xmin;
  int N;
  double* part;       // [B][4][G]: bisection sums (double-buffered) + |dx| sum/max
  double* stats;      // [B][2]: dx_max, dx_mean
  double* lam_out;    // [B]
  unsigned* bar;      // [2] barrier counter, generation
  int* err;           // set when a grid barrier gave up (the kernel then returns early)
  const int* active;
  long long poll_limit;  // grid_barrier poll limit
  unsigned phantom;      // extra blocks the barrier waits for (0; more only to test the bounded wait)
  int cache_chunk;       // k_oc_update_tree: elements per block its dynamic shared memory caches (0: none)
};

__global__ void __launch_bounds__(kThreads) k_oc_update(OcArgs a) {
  const int G = gridDim.x, g = blockIdx.x, b = blockIdx.y;
  const unsigned nblocks = gridDim.x * gridDim.y + a.phantom;
  const bool act = !a.active || a.active[b];
  const int N = a.N;
  const int chunk = (N + G - 1) / G;
  const int lo = g * chunk, hi = min(N, lo + chunk);
  const double* xb = a.x + (size_t)b * N;
  const double* db = a.dJ + (size_t)b * N;
  const double vf = act ? a.volfrac[b] : 0.0;
  double l1 = 1e-12, l2 = 1e6, lam = 0;
  for (int it = 0; it < 60; ++it) {
    lam = 0.5 * (l1 + l2);
    double s = 0;
    if (act) {
      for (int i = lo + threadIdx.x; i < hi; i += kThreads) {
        const double xv = xb[i];
        const double dj = fmax(db[i], 1e-12);
        double xn = xv * sqrt(dj / lam);
        xn = fmin(fmax(xn, xv - a.move), xv + a.move);
        xn = fmin(fmax(xn, a.xmin), 1.0);
        s += xn;
      }
    }
    double v[1] = {s};
    block_sum_store<1>(v, a.part + ((size_t)b * 4 + (it & 1)) * G + g);
    if (!grid_barrier(a.bar, a.bar + 1, nblocks, a.err, a.poll_limit)) return;
    if (act) {
      __shared__ double s_tot;
      if (threadIdx.x < 32) {
        const double* pp = a.part + ((size_t)b * 4 + (it & 1)) * G;
        double t = 0;
        for (int k = threadIdx.x; k < G; k += 32) t += __ldcg(pp + k);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
        if (threadIdx.x == 0) s_tot = t;
      }
      __syncthreads();
      const double tot = s_tot;
      __syncthreads();
      if (tot / (double)N > vf)
        l1 = lam;
      else
        l2 = lam;
    }
  }
  // final x (that of the last step) and |dx| statistics
  double dmax = 0, dsum = 0;
  if (act) {
    double* xo = a.xnew + (size_t)b * N;
    for (int i = lo + threadIdx.x; i < hi; i += kThreads) {
      const double xv = xb[i];
      const double dj = fmax(db[i], 1e-12);
      double xn = xv * sqrt(dj / lam);
      xn = fmin(fmax(xn, xv - a.move), xv + a.move);
      xn = fmin(fmax(xn, a.xmin), 1.0);
      xo[i] = xn;
      const double d = fabs(xn - xv);
      dmax = fmax(dmax, d);
      dsum += d;
    }
  }
  dmax = block_max(dmax);
  double v[1] = {dsum};
  __syncthreads();
  block_sum_store<1>(v, a.part + ((size_t)b * 4 + 2) * G + g);
  if (threadIdx.x == 0) a.part[((size_t)b * 4 + 3) * G + g] = dmax;
  if (!grid_barrier(a.bar, a.bar + 1, nblocks, a.err, a.poll_limit)) return;
  if (act && g == 0 && threadIdx.x == 0) {
    double m = 0, t = 0;
    for (int k = 0; k < G; ++k) {
      t += __ldcg(a.part + ((size_t)b * 4 + 2) * G + k);
      m = fmax(m, __ldcg(a.part + ((size_t)b * 4 + 3) * G + k));
    }
    a.stats[2 * b] = m;
    a.stats[2 * b + 1] = t / (double)N;
    if (a.lam_out) a.lam_out[b] = lam;
  }
}

// The same OC update resolving LV bisection steps per grid barrier: each pass
// evaluates the volume at the 2^LV - 1 midpoints the next LV steps can visit
// (the bisection tree below the current [l1, l2], each midpoint formed as
// 0.5 (lo + hi) exactly as the step that would reach it), with the per-block
// sums and their reduction over blocks in the order k_oc_update uses, then
// walks the tree with those volumes, taking k_oc_update's branches; the
// launch waits at 60 / LV + 1 barriers instead of 61.  Partial sums:
// [cells][2][G][2^LV - 1], then the |dx| statistics [cells][2][G].
constexpr int kOcMaxG = 160;  // blocks per cell k_oc_update_tree supports
template <int LV>
__global__ void __launch_bounds__(kThreads) k_oc_update_tree(OcArgs a) {
  constexpr int NC = (1 << LV) - 1;
  static_assert(60 % LV == 0, "LV must divide the 60 bisection steps");
  const int G = gridDim.x, g = blockIdx.x, b = blockIdx.y;
  const unsigned nblocks = gridDim.x * gridDim.y + a.phantom;
  const bool act = !a.active || a.active[b];
  const int N = a.N;
  const int chunk = (N + G - 1) / G;
  const int lo_i = g * chunk, hi_i = min(N, lo_i + chunk);
  const double* xb = a.x + (size_t)b * N;
  const double* db = a.dJ + (size_t)b * N;
  const double vf = act ? a.volfrac[b] : 0.0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __shared__ double s_tot[NC], s_rl[NC];
  // the block's x sqrt(dJ) and move bounds, formed once when the dynamic
  // shared memory holds them (3 doubles per element of the chunk)
  extern __shared__ double s_oc[];
  const bool cached = a.cache_chunk >= chunk;
  if (cached && act)
    for (int i = lo_i + threadIdx.x; i < hi_i; i += kThreads) {
      const double xv = xb[i];
      const int j = i - lo_i;
      s_oc[3 * j] = xv * sqrt(fmax(db[i], 1e-12));
      s_oc[3 * j + 1] = fmax(xv - a.move, a.xmin);
      s_oc[3 * j + 2] = fmin(xv + a.move, 1.0);
    }
  __syncthreads();
  double l1 = 1e-12, l2 = 1e6, lam = 0;
  for (int pass = 0; pass < 60 / LV; ++pass) {
    double lamc[NC];
    {
      double lo[NC], hi[NC];
      lo[0] = l1;
      hi[0] = l2;
#pragma unroll
      for (int h = 0; h < NC; ++h) {
        const double m = 0.5 * (lo[h] + hi[h]);
        lamc[h] = m;
        if (2 * h + 2 < NC) {
          lo[2 * h + 1] = lo[h];  // volume <= vf: l2 = m
          hi[2 * h + 1] = m;
          lo[2 * h + 2] = m;      // volume > vf: l1 = m
          hi[2 * h + 2] = hi[h];
        }
      }
    }
    // sqrt(dJ / lambda) as sqrt(dJ) / sqrt(lambda): one square root per
    // element and pass instead of a division and a root per candidate.  The
    // volumes differ from k_oc_update's by rounding, which can only change a
    // branch whose volume is within rounding of vf, i.e. at a midpoint within
    // rounding of the root, so lambda agrees to rounding.
    // 1 / sqrt(lambda) of the candidates, formed once per block
    if (threadIdx.x < NC) {
      double m = lamc[0];
#pragma unroll
      for (int h = 1; h < NC; ++h)
        if (threadIdx.x == h) m = lamc[h];
      s_rl[threadIdx.x] = 1.0 / sqrt(m);
    }
    __syncthreads();
    double rl[NC], sc[NC];
#pragma unroll
    for (int h = 0; h < NC; ++h) {
      rl[h] = s_rl[h];
      sc[h] = 0;
    }
    if (act) {
      for (int i = lo_i + threadIdx.x; i < hi_i; i += kThreads) {
        double xs, lo, hi;
        if (cached) {
          const int j = i - lo_i;
          xs = s_oc[3 * j];
          lo = s_oc[3 * j + 1];
          hi = s_oc[3 * j + 2];
        } else {
          const double xv = xb[i];
          xs = xv * sqrt(fmax(db[i], 1e-12));
          lo = fmax(xv - a.move, a.xmin);
          hi = fmin(xv + a.move, 1.0);
        }
#pragma unroll
        for (int h = 0; h < NC; ++h) sc[h] += fmin(fmax(xs * rl[h], lo), hi);
      }
    }
    double* pp = a.part + (((size_t)b * 2 + (pass & 1)) * G) * NC;
    block_sum_store<NC>(sc, pp + (size_t)g * NC);
    if (!grid_barrier(a.bar, a.bar + 1, nblocks, a.err, a.poll_limit)) return;
    if (act) {
      // the volumes over the G blocks, summed in k_oc_update's order (lane
      // strided, then the shuffle tree); every load of a warp's candidates is
      // issued before the first sum (G <= kOcMaxG)
      constexpr int NW = kThreads / 32, KM = kOcMaxG / 32, HM = (NC + NW - 1) / NW;
      double vals[HM][KM];
#pragma unroll
      for (int r = 0; r < HM; ++r)
#pragma unroll
        for (int m = 0; m < KM; ++m) {
          const int h = warp + r * NW, k = lane + 32 * m;
          vals[r][m] = (h < NC && k < G) ? __ldcg(pp + (size_t)k * NC + h) : 0.0;
        }
#pragma unroll
      for (int r = 0; r < HM; ++r) {
        const int h = warp + r * NW;
        double t = 0;
#pragma unroll
        for (int m = 0; m < KM; ++m)
          if (lane + 32 * m < G) t += vals[r][m];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
        if (lane == 0 && h < NC) s_tot[h] = t;
      }
      __syncthreads();
      int h = 0;
#pragma unroll
      for (int lev = 0; lev < LV; ++lev) {
        lam = lamc[h];
        if (s_tot[h] / (double)N > vf) {
          l1 = lam;
          h = 2 * h + 2;
        } else {
          l2 = lam;
          h = 2 * h + 1;
        }
      }
      __syncthreads();
    }
  }
  double dmax = 0, dsum = 0;
  if (act) {
    double* xo = a.xnew + (size_t)b * N;
    for (int i = lo_i + threadIdx.x; i < hi_i; i += kThreads) {
      const double xv = xb[i];
      const double dj = fmax(db[i], 1e-12);
      double xn = xv * sqrt(dj / lam);
      xn = fmin(fmax(xn, xv - a.move), xv + a.move);
      xn = fmin(fmax(xn, a.xmin), 1.0);
      xo[i] = xn;
      const double d = fabs(xn - xv);
      dmax = fmax(dmax, d);
      dsum += d;
    }
  }
  dmax = block_max(dmax);
  double v[1] = {dsum};
  __syncthreads();
  double* st = a.part + (size_t)gridDim.y * 2 * G * NC;
  block_sum_store<1>(v, st + ((size_t)b * 2 + 0) * G + g);
  if (threadIdx.x == 0) st[((size_t)b * 2 + 1) * G + g] = dmax;
  if (!grid_barrier(a.bar, a.bar + 1, nblocks, a.err, a.poll_limit)) return;
  if (act && g == 0 && threadIdx.x == 0) {
    double m = 0, t = 0;
    for (int k = 0; k < G; ++k) {
      t += __ldcg(st + ((size_t)b * 2 + 0) * G + k);
      m = fmax(m, __ldcg(st + ((size_t)b * 2 + 1) * G + k));
    }
    a.stats[2 * b] = m;
    a.stats[2 * b + 1] = t / (double)N;
    if (a.lam_out) a.lam_out[b] = lam;
  }
}

}  // namespace maple
