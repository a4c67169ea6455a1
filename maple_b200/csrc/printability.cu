// Manufacturability penalties and their gradients (see printability.h).
//
// Overhang: one CTA per cell sweeps the layers z = 1..r-1 (each layer's
// lateral max-pool needs the whole previous layer), recording the pooled
// support and its argmax per voxel; the backward sweep runs the layers in
// reverse.  Cavity: the (super)cell is materialised once, then every opening
// and flood-fill step is one grid-wide kernel (one thread per supercell voxel),
// each flood-fill step recording its dilation and argmax for the backward
// pass.  Pool adjoints are gathers: a voxel sums the gradients of the windows
// whose argmax it is, so no atomics are needed and results are deterministic.
#include "printability.h"

#include <algorithm>
#include <atomic>
#include <utility>
#include <cmath>
#include <stdexcept>
#include <string>

namespace maple_pr {

static std::atomic<unsigned long long> g_launches{0};
unsigned long long launches() { return g_launches.load(); }

#define PR_LAUNCH(...)                                                                               \
  do {                                                                                               \
    __VA_ARGS__;                                                                                     \
    const cudaError_t e_ = cudaGetLastError();                                                       \
    if (e_ != cudaSuccess) throw std::runtime_error(std::string("penalty kernel: ") + cudaGetErrorString(e_)); \
    g_launches.fetch_add(1);                                                                         \
  } while (0)

constexpr int kT = 256;
static inline unsigned nb(size_t n) { return (unsigned)((n + kT - 1) / kT); }
static inline size_t al(size_t b) { return (b + 255) / 256 * 256; }

__device__ __forceinline__ int wrapi(int i, int n) { return ((i % n) + n) % n; }

// gradient of torch.minimum(a, b) w.r.t. a for upstream g: g where a < b, g/2 where equal
__device__ __forceinline__ double min_grad(double a, double b, double g) {
  return a < b ? g : (a == b ? 0.5 * g : 0.0);
}

// block sum of v (blockDim.x <= 1024) returned to thread 0
__device__ double block_sum(double v) {
  __shared__ double sm[32];
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) s += sm[w];
  __syncthreads();
  return s;
}

// ---------------------------------------------------------------------------
// overhang
// ---------------------------------------------------------------------------
struct OverhangWork {
  double* tape_s;  // [B][r-1][r^2] pooled support of layer z-1
  int* tape_src;   // [B][r-1][r^2] its argmax (layer index, -1 = padding)
  double* buf;     // [B][3][r^2] two support / gradient layers and one scratch layer
};

static OverhangWork overhang_parts(const OverhangPlan& p, void* work) {
  const size_t L = (size_t)p.r * p.r, T = (size_t)p.B * (p.r - 1) * L;
  char* w = static_cast<char*>(work);
  OverhangWork o;
  o.tape_s = reinterpret_cast<double*>(w);
  o.tape_src = reinterpret_cast<int*>(w + al(T * sizeof(double)));
  o.buf = reinterpret_cast<double*>(w + al(T * sizeof(double)) + al(T * sizeof(int)));
  return o;
}

size_t OverhangPlan::bytes() const {
  const size_t L = (size_t)r * r, T = (size_t)B * (r - 1) * L;
  return al(T * sizeof(double)) + al(T * sizeof(int)) + al((size_t)B * 3 * L * sizeof(double));
}

__global__ void __launch_bounds__(1024) k_overhang_fwd(const double* __restrict__ rho, int r, int rad, int periodic,
                                                       OverhangWork w, double* __restrict__ P) {
  const int b = blockIdx.x;
  const int L = r * r;
  const double* g = rho + (size_t)b * L * r;
  double* cur = w.buf + (size_t)b * 3 * L;
  double* nxt = cur + L;
  for (int q = threadIdx.x; q < L; q += blockDim.x) cur[q] = g[(size_t)q * r];
  __syncthreads();
  double acc = 0.0;
  for (int z = 1; z < r; ++z) {
    double* ts = w.tape_s + ((size_t)b * (r - 1) + (z - 1)) * L;
    int* tsrc = w.tape_src + ((size_t)b * (r - 1) + (z - 1)) * L;
    for (int q = threadIdx.x; q < L; q += blockDim.x) {
      const int x = q / r, y = q % r;
      double best = -INFINITY;
      int bsrc = -1;
      for (int dx = -rad; dx <= rad; ++dx)
        for (int dy = -rad; dy <= rad; ++dy) {
          int xx = x + dx, yy = y + dy;
          double v;
          int src;
          if (periodic) {
            xx = wrapi(xx, r);
            yy = wrapi(yy, r);
            src = xx * r + yy;
            v = cur[src];
          } else if (xx < 0 || xx >= r || yy < 0 || yy >= r) {
            src = -1;
            v = 0.0;
          } else {
            src = xx * r + yy;
            v = cur[src];
          }
          if (v > best) {
            best = v;
            bsrc = src;
          }
        }
      ts[q] = best;
      tsrc[q] = bsrc;
      const double rz = g[(size_t)q * r + z];
      acc += fmax(rz - best, 0.0);
      nxt[q] = fmin(rz, best);
    }
    __syncthreads();
    double* t = cur;
    cur = nxt;
    nxt = t;
  }
  const double s = block_sum(acc);
  if (threadIdx.x == 0) P[b] = s / ((double)L * (r > 1 ? r - 1 : 1));
}

__global__ void __launch_bounds__(1024) k_overhang_bwd(const double* __restrict__ rho, int r, int rad, int periodic,
                                                       OverhangWork w, double* __restrict__ grad) {
  const int b = blockIdx.x;
  const int L = r * r;
  const double den = (double)L * (r > 1 ? r - 1 : 1);
  const double* g = rho + (size_t)b * L * r;
  double* out = grad + (size_t)b * L * r;
  double* gsup = w.buf + (size_t)b * 3 * L;  // gradient arriving at support(z)
  double* gnew = gsup + L;
  double* gs = gnew + L;                     // gradient at the pooled support of layer z
  for (int q = threadIdx.x; q < L; q += blockDim.x) gsup[q] = 0.0;
  __syncthreads();
  for (int z = r - 1; z >= 1; --z) {
    const double* ts = w.tape_s + ((size_t)b * (r - 1) + (z - 1)) * L;
    const int* tsrc = w.tape_src + ((size_t)b * (r - 1) + (z - 1)) * L;
    for (int q = threadIdx.x; q < L; q += blockDim.x) {
      const double rz = g[(size_t)q * r + z], s = ts[q], up = gsup[q];
      const double act = (rz - s) > 0.0 ? 1.0 / den : 0.0;
      out[(size_t)q * r + z] = min_grad(rz, s, up) + act;
      gs[q] = min_grad(s, rz, up) - act;
    }
    __syncthreads();
    // pool adjoint: voxel p collects the windows whose argmax it is
    for (int p = threadIdx.x; p < L; p += blockDim.x) {
      const int x = p / r, y = p % r;
      double acc = 0.0;
      for (int dx = -rad; dx <= rad; ++dx)
        for (int dy = -rad; dy <= rad; ++dy) {
          int xx = x + dx, yy = y + dy;
          if (periodic) {
            xx = wrapi(xx, r);
            yy = wrapi(yy, r);
          } else if (xx < 0 || xx >= r || yy < 0 || yy >= r) {
            continue;
          }
          const int q = xx * r + yy;
          if (tsrc[q] == p) acc += gs[q];
        }
      gnew[p] = acc;
    }
    __syncthreads();
    double* t = gsup;
    gsup = gnew;
    gnew = t;
  }
  for (int q = threadIdx.x; q < L; q += blockDim.x) out[(size_t)q * r] = gsup[q];
}

void overhang(const double* rho, const OverhangPlan& p, double* P, double* grad, void* work, cudaStream_t s) {
  if (p.r < 2 || p.B < 1 || p.rad < 1) throw std::runtime_error("overhang penalty: bad sizes");
  if (p.periodic && 2 * p.rad + 1 > p.r) throw std::runtime_error("overhang penalty: support window wider than the cell");
  const OverhangWork w = overhang_parts(p, work);
  PR_LAUNCH(k_overhang_fwd<<<p.B, 1024, 0, s>>>(rho, p.r, p.rad, p.periodic, w, P));
  if (grad) PR_LAUNCH(k_overhang_bwd<<<p.B, 1024, 0, s>>>(rho, p.r, p.rad, p.periodic, w, grad));
}

// ---------------------------------------------------------------------------
// cavity
// ---------------------------------------------------------------------------
struct CavGeo {
  int r, X, Y, Z;  // cell size and supercell dims
  size_t M;
  int periodic;
  __device__ void coords(size_t v, int& x, int& y, int& z) const {
    z = (int)(v % Z);
    y = (int)((v / Z) % Y);
    x = (int)(v / ((size_t)Y * Z));
  }
  __device__ size_t index(int x, int y, int z) const { return ((size_t)x * Y + y) * Z + z; }
  // neighbour at offset, or false (outside a non-periodic supercell)
  __device__ bool shift(int x, int y, int z, int dx, int dy, int dz, size_t& out) const {
    int a = x + dx, bb = y + dy, c = z + dz;
    if (periodic) {
      a = wrapi(a, X);
      bb = wrapi(bb, Y);
      c = wrapi(c, Z);
    } else if (a < 0 || a >= X || bb < 0 || bb >= Y || c < 0 || c >= Z) {
      return false;
    }
    out = index(a, bb, c);
    return true;
  }
};

struct CavWork {
  double *void_uc, *vsc, *er, *vconn, *reach0, *reach1, *t1, *t2, *dil, *gr0, *gr1, *g1, *g2, *gvconn, *gvoid, *part;
  signed char *er_off, *di_off, *off;  // per-pass argmax offsets: [3][B][M] (opening) and [steps][3][B][M]
  unsigned char* tape;                 // flood-fill radius 1: one packed byte per voxel and step [steps][B][M]
};

constexpr signed char kPadOff = 127;  // the pass picked a padding cell

static size_t cav_parts(const CavityPlan& p, void* work, CavWork* o) {
  const size_t B = p.B, M = p.M(), N = (size_t)p.r * p.r * p.r, S = (size_t)std::max(p.nsteps, 0);
  const size_t nparts = (M + kT - 1) / kT;
  size_t off = 0;
  char* w = static_cast<char*>(work);
  auto take = [&](size_t bytes) {
    char* q = w ? w + off : nullptr;
    off += al(bytes);
    return q;
  };
  CavWork c{};
  c.void_uc = reinterpret_cast<double*>(take(B * N * 8));
  c.vsc = reinterpret_cast<double*>(take(B * M * 8));
  if (p.min_channel_rad > 0) {
    c.er = reinterpret_cast<double*>(take(B * M * 8));
    c.vconn = reinterpret_cast<double*>(take(B * M * 8));
    c.er_off = reinterpret_cast<signed char*>(take(3 * B * M));
    c.di_off = reinterpret_cast<signed char*>(take(3 * B * M));
  }
  c.reach0 = reinterpret_cast<double*>(take(B * M * 8));
  c.reach1 = reinterpret_cast<double*>(take(B * M * 8));
  c.t1 = reinterpret_cast<double*>(take(B * M * 8));
  c.t2 = reinterpret_cast<double*>(take(B * M * 8));
  if (p.rad == 1) {
    c.tape = reinterpret_cast<unsigned char*>(take(B * M * S));
  } else {
    c.dil = reinterpret_cast<double*>(take(B * M * S * 8));
    c.off = reinterpret_cast<signed char*>(take(3 * B * M * S));
  }
  c.gr0 = reinterpret_cast<double*>(take(B * M * 8));
  c.gr1 = reinterpret_cast<double*>(take(B * M * 8));
  c.g1 = reinterpret_cast<double*>(take(B * M * 8));
  c.g2 = reinterpret_cast<double*>(take(B * M * 8));
  c.gvconn = reinterpret_cast<double*>(take(B * M * 8));
  c.gvoid = reinterpret_cast<double*>(take(B * M * 8));
  c.part = reinterpret_cast<double*>(take(B * nparts * 8));
  if (o) *o = c;
  return off;
}

size_t CavityPlan::bytes() const { return cav_parts(*this, nullptr, nullptr); }

__global__ void k_cav_void(const double* __restrict__ rho, double* __restrict__ void_uc, size_t N, double thresh,
                           double beta) {
  const size_t i = (size_t)blockIdx.x * kT + threadIdx.x + (size_t)blockIdx.y * N;
  if ((size_t)blockIdx.x * kT + threadIdx.x >= N) return;
  void_uc[i] = 1.0 / (1.0 + exp(-beta * (thresh - rho[i])));
}

__global__ void k_cav_tile(const double* __restrict__ void_uc, double* __restrict__ vsc, CavGeo G) {
  const size_t v = (size_t)blockIdx.x * kT + threadIdx.x;
  if (v >= G.M) return;
  const int b = blockIdx.y;
  int x, y, z;
  G.coords(v, x, y, z);
  const int r = G.r;
  vsc[(size_t)b * G.M + v] = void_uc[(size_t)b * r * r * r + ((size_t)(x % r) * r + (y % r)) * r + (z % r)];
}

// One axis of a separable (2 rad + 1)^3 max pool:
//   out(v) = so * max_{d=-rad..rad} (v + d e_axis inside ? si * in(v + d e_axis) : pad)
// keeping the first maximum (strict >); off(v) = its d, or kPadOff for padding.
// Passes along z, then y, then x reproduce the first maximum of the 3-D window
// in (x, y, z) scan order: it is the lexicographically smallest (dx, dy, dz)
// among the maxima, and each pass keeps the smallest offset of its axis.
// With fuse_min, the result also gives min_out = min(vmin, out) (a flood-fill step).
__global__ void k_cav_pass(const double* __restrict__ in, double* __restrict__ out, signed char* __restrict__ off,
                           CavGeo G, int axis, int rad, double si, double so, double pad,
                           const double* __restrict__ vmin, double* __restrict__ min_out) {
  const size_t v = (size_t)blockIdx.x * kT + threadIdx.x;
  if (v >= G.M) return;
  const size_t base = (size_t)blockIdx.y * G.M;
  int x, y, z;
  G.coords(v, x, y, z);
  double best = -INFINITY;
  int bd = kPadOff;
  for (int d = -rad; d <= rad; ++d) {
    size_t q;
    const bool inside = G.shift(x, y, z, axis == 0 ? d : 0, axis == 1 ? d : 0, axis == 2 ? d : 0, q);
    const double val = inside ? si * in[base + q] : pad;
    if (val > best) {
      best = val;
      bd = inside ? d : kPadOff;
    }
  }
  const double res = so * best;
  out[base + v] = res;
  off[base + v] = (signed char)bd;
  if (min_out) min_out[base + v] = fmin(vmin[base + v], res);
}

// Adjoint of one pass: gin(p) (+)= sum over the outputs q = p - d e_axis that
// picked p (off(q) == d) of their gradient; with vmin, the output gradient is
// first taken through min(vmin, out): the dil branch of min_grad.
__global__ void k_cav_pass_adj(const double* __restrict__ gout, const signed char* __restrict__ off,
                               double* __restrict__ gin, CavGeo G, int axis, int rad, int accumulate,
                               const double* __restrict__ vmin, const double* __restrict__ outv) {
  const size_t v = (size_t)blockIdx.x * kT + threadIdx.x;
  if (v >= G.M) return;
  const size_t base = (size_t)blockIdx.y * G.M;
  int x, y, z;
  G.coords(v, x, y, z);
  double acc = 0.0;
  for (int d = -rad; d <= rad; ++d) {
    size_t q;
    if (!G.shift(x, y, z, axis == 0 ? -d : 0, axis == 1 ? -d : 0, axis == 2 ? -d : 0, q)) continue;
    if (off[base + q] != d) continue;
    const double g = gout[base + q];
    acc += vmin ? min_grad(outv[base + q], vmin[base + q], g) : g;
  }
  gin[base + v] = accumulate ? gin[base + v] + acc : acc;
}

// ---------------------------------------------------------------------------
// Flood-fill steps of radius 1, fused: one CTA per 8^3 tile runs the z, y and
// x passes of the step's 3^3 max pool in shared memory (the z pass over the
// tile and its x/y halo, the y pass over the tile and its x halo, the x pass
// over the tile), with the same candidate order and padding rules as
// k_cav_pass, so the dilation, its argmax offsets and reach = min(void_conn,
// dil) are those of the three separate passes.  The step's tape is one byte per
// voxel: bits 0-1, 2-3, 4-5 the z, y, x argmax codes (offset + 1; 3 = padding)
// and bits 6-7 the comparison of void_conn with dil (0: <, 1: ==, 2: >), which
// is all the backward step needs.  The backward kernel gathers through the x,
// then y, then z adjoints over the same tile and halo, summing in the order of
// k_cav_pass_adj.
// ---------------------------------------------------------------------------
constexpr int FT = 8, FH = FT + 2, FTHREADS = FT * FT * FT;

struct FillTile {
  int x0, y0, z0;
  __device__ FillTile(const CavGeo& G) {
    const int ntz = (G.Z + FT - 1) / FT, nty = (G.Y + FT - 1) / FT;
    const int t = blockIdx.x;
    z0 = (t % ntz) * FT;
    y0 = ((t / ntz) % nty) * FT;
    x0 = (t / (ntz * nty)) * FT;
  }
};

__device__ __forceinline__ bool in_grid(const CavGeo& G, int x, int y, int z) {
  return G.periodic || (x >= 0 && x < G.X && y >= 0 && y < G.Y && z >= 0 && z < G.Z);
}

__device__ __forceinline__ unsigned enc_off(int d) { return d == kPadOff ? 3u : (unsigned)(d + 1); }

__global__ void __launch_bounds__(FTHREADS) k_cav_fill_fwd(const double* __restrict__ reach,
                                                          const double* __restrict__ vconn,
                                                          double* __restrict__ reach_out,
                                                          unsigned char* __restrict__ tape, CavGeo G) {
  __shared__ double s_in[FH][FH][FH];
  __shared__ double t1[FH][FH][FT];
  __shared__ double t2[FH][FT][FT];
  __shared__ unsigned char cz[FT][FT][FT], cy[FT][FT][FT];
  const FillTile T(G);
  const size_t base = (size_t)blockIdx.y * G.M;
  const int tid = threadIdx.x;
  for (int w = tid; w < FH * FH * FH; w += FTHREADS) {
    const int iz = w % FH, iy = (w / FH) % FH, ix = w / (FH * FH);
    size_t q;
    s_in[ix][iy][iz] = G.shift(T.x0 - 1 + ix, T.y0 - 1 + iy, T.z0 - 1 + iz, 0, 0, 0, q) ? reach[base + q] : 0.0;
  }
  __syncthreads();
  for (int w = tid; w < FH * FH * FT; w += FTHREADS) {  // z pass
    const int iz = w % FT, iy = (w / FT) % FH, ix = w / (FT * FH);
    const int gx = T.x0 - 1 + ix, gy = T.y0 - 1 + iy, gz = T.z0 + iz;
    double best = -INFINITY;
    int bd = kPadOff;
#pragma unroll
    for (int d = -1; d <= 1; ++d) {
      const bool inside = in_grid(G, gx, gy, gz + d);
      const double v = inside ? s_in[ix][iy][iz + 1 + d] : 0.0;
      if (v > best) {
        best = v;
        bd = inside ? d : kPadOff;
      }
    }
    t1[ix][iy][iz] = best;
    if (ix >= 1 && ix <= FT && iy >= 1 && iy <= FT) cz[ix - 1][iy - 1][iz] = (unsigned char)enc_off(bd);
  }
  __syncthreads();
  for (int w = tid; w < FH * FT * FT; w += FTHREADS) {  // y pass
    const int iz = w % FT, iy = (w / FT) % FT, ix = w / (FT * FT);
    const int gx = T.x0 - 1 + ix, gy = T.y0 + iy, gz = T.z0 + iz;
    double best = -INFINITY;
    int bd = kPadOff;
#pragma unroll
    for (int d = -1; d <= 1; ++d) {
      const bool inside = in_grid(G, gx, gy + d, gz);
      const double v = inside ? t1[ix][iy + 1 + d][iz] : 0.0;
      if (v > best) {
        best = v;
        bd = inside ? d : kPadOff;
      }
    }
    t2[ix][iy][iz] = best;
    if (ix >= 1 && ix <= FT) cy[ix - 1][iy][iz] = (unsigned char)enc_off(bd);
  }
  __syncthreads();
  const int tz = tid % FT, ty = (tid / FT) % FT, tx = tid / (FT * FT);  // x pass, one thread per voxel
  const int gx = T.x0 + tx, gy = T.y0 + ty, gz = T.z0 + tz;
  if (gx >= G.X || gy >= G.Y || gz >= G.Z) return;
  double best = -INFINITY;
  int bd = kPadOff;
#pragma unroll
  for (int d = -1; d <= 1; ++d) {
    const bool inside = in_grid(G, gx + d, gy, gz);
    const double v = inside ? t2[tx + 1 + d][ty][tz] : 0.0;
    if (v > best) {
      best = v;
      bd = inside ? d : kPadOff;
    }
  }
  const size_t i = base + G.index(gx, gy, gz);
  const double vc = vconn[i];
  reach_out[i] = fmin(vc, best);
  const unsigned cmp = vc < best ? 0u : (vc == best ? 1u : 2u);
  tape[i] = (unsigned char)(cz[tx][ty][tz] | (cy[tx][ty][tz] << 2) | (enc_off(bd) << 4) | (cmp << 6));
}

// adjoint of k_cav_fill_fwd: gin = gradient at reach (overwritten), gvconn +=
// the void_conn branch of the min, from gout = gradient at reach_out
__global__ void __launch_bounds__(FTHREADS) k_cav_fill_bwd(const double* __restrict__ gout,
                                                          const unsigned char* __restrict__ tape,
                                                          double* __restrict__ gin, double* __restrict__ gvconn,
                                                          CavGeo G) {
  __shared__ double sg[FH][FH][FH];    // the dil branch of the min's gradient
  __shared__ unsigned char st[FH][FH][FH];
  __shared__ double ax[FT][FH][FH];    // after the x adjoint
  __shared__ double ay[FT][FT][FH];    // after the y adjoint
  const FillTile T(G);
  const size_t base = (size_t)blockIdx.y * G.M;
  const int tid = threadIdx.x;
  for (int w = tid; w < FH * FH * FH; w += FTHREADS) {
    const int iz = w % FH, iy = (w / FH) % FH, ix = w / (FH * FH);
    size_t q;
    unsigned char code = 0xFF;  // outside the grid: every code reads as padding
    double g = 0.0;
    if (G.shift(T.x0 - 1 + ix, T.y0 - 1 + iy, T.z0 - 1 + iz, 0, 0, 0, q)) {
      code = tape[base + q];
      const unsigned cmp = code >> 6;
      const double go = gout[base + q];
      g = cmp == 2 ? go : (cmp == 1 ? 0.5 * go : 0.0);
    }
    sg[ix][iy][iz] = g;
    st[ix][iy][iz] = code;
  }
  __syncthreads();
  for (int w = tid; w < FT * FH * FH; w += FTHREADS) {  // x adjoint
    const int iz = w % FH, iy = (w / FH) % FH, jx = w / (FH * FH), ix = jx + 1;
    double acc = 0.0;
#pragma unroll
    for (int d = -1; d <= 1; ++d) {
      const unsigned code = (st[ix - d][iy][iz] >> 4) & 3u;
      if (code == (unsigned)(d + 1)) acc += sg[ix - d][iy][iz];
    }
    ax[jx][iy][iz] = acc;
  }
  __syncthreads();
  for (int w = tid; w < FT * FT * FH; w += FTHREADS) {  // y adjoint
    const int iz = w % FH, jy = (w / FH) % FT, jx = w / (FH * FT), iy = jy + 1;
    double acc = 0.0;
#pragma unroll
    for (int d = -1; d <= 1; ++d) {
      const unsigned code = (st[jx + 1][iy - d][iz] >> 2) & 3u;
      if (code == (unsigned)(d + 1)) acc += ax[jx][iy - d][iz];
    }
    ay[jx][jy][iz] = acc;
  }
  __syncthreads();
  const int tz = tid % FT, ty = (tid / FT) % FT, tx = tid / (FT * FT);  // z adjoint, one thread per voxel
  const int gx = T.x0 + tx, gy = T.y0 + ty, gz = T.z0 + tz;
  if (gx >= G.X || gy >= G.Y || gz >= G.Z) return;
  double acc = 0.0;
#pragma unroll
  for (int d = -1; d <= 1; ++d) {
    const unsigned code = st[tx + 1][ty + 1][tz + 1 - d] & 3u;
    if (code == (unsigned)(d + 1)) acc += ay[tx][ty][tz + 1 - d];
  }
  const size_t i = base + G.index(gx, gy, gz);
  gin[i] = acc;
  const unsigned cmp = st[tx + 1][ty + 1][tz + 1] >> 6;
  if (cmp < 2) gvconn[i] += cmp == 0 ? gout[i] : 0.5 * gout[i];
}

__device__ __forceinline__ bool is_seed(const CavGeo& G, int seed, int x, int y, int z) {
  const bool fx = x == 0 || x == G.X - 1, fy = y == 0 || y == G.Y - 1, fz = z == 0 || z == G.Z - 1;
  switch (seed) {
    case SEED_ALL: return fx || fy || fz;
    case SEED_X: return fx;
    case SEED_Y: return fy;
    default: return fz;  // SEED_Z, SEED_XY
  }
}

__global__ void k_cav_seed(const double* __restrict__ vconn, double* __restrict__ reach, CavGeo G, int seed) {
  const size_t v = (size_t)blockIdx.x * kT + threadIdx.x;
  if (v >= G.M) return;
  const size_t i = (size_t)blockIdx.y * G.M + v;
  int x, y, z;
  G.coords(v, x, y, z);
  reach[i] = is_seed(G, seed, x, y, z) ? vconn[i] : 0.0;
}

__device__ __forceinline__ bool in_region(const CavGeo& G, int focus, int x, int y, int z) {
  if (!focus) return true;
  const int r = G.r, cx = (G.X / r) / 2, cy = (G.Y / r) / 2, cz = (G.Z / r) / 2;
  return x / r == cx && y / r == cy && z / r == cz;
}

// per-block partial sums of relu(void - reach) over the penalty region
__global__ void k_cav_trapped(const double* __restrict__ vsc, const double* __restrict__ reach,
                              double* __restrict__ part, CavGeo G, int focus) {
  const size_t v = (size_t)blockIdx.x * kT + threadIdx.x;
  double t = 0.0;
  if (v < G.M) {
    const size_t i = (size_t)blockIdx.y * G.M + v;
    int x, y, z;
    G.coords(v, x, y, z);
    if (in_region(G, focus, x, y, z)) t = fmax(vsc[i] - reach[i], 0.0);
  }
  const double s = block_sum(t);
  if (threadIdx.x == 0) part[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = s;
}

__global__ void k_cav_total(const double* __restrict__ part, int nparts, double* __restrict__ P, double count) {
  const int b = blockIdx.x;
  double s = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) s += part[(size_t)b * nparts + i];
  s = block_sum(s);
  if (threadIdx.x == 0) P[b] = s / count;
}

// upstream gradient of the mean of relu(void - reach) over the region
__global__ void k_cav_bwd_init(const double* __restrict__ vsc, const double* __restrict__ reach,
                               double* __restrict__ gvoid, double* __restrict__ greach, double* __restrict__ gvconn,
                               CavGeo G, int focus, double inv_count) {
  const size_t v = (size_t)blockIdx.x * kT + threadIdx.x;
  if (v >= G.M) return;
  const size_t i = (size_t)blockIdx.y * G.M + v;
  int x, y, z;
  G.coords(v, x, y, z);
  const double g = (in_region(G, focus, x, y, z) && vsc[i] - reach[i] > 0.0) ? inv_count : 0.0;
  gvoid[i] = g;
  greach[i] = -g;
  gvconn[i] = 0.0;
}

// gvconn += the vconn branch of min(vconn, dil) for upstream gout
__global__ void k_cav_min_vconn(const double* __restrict__ gout, const double* __restrict__ vconn,
                                const double* __restrict__ dil, double* __restrict__ gvconn, size_t M) {
  const size_t v = (size_t)blockIdx.x * kT + threadIdx.x;
  if (v >= M) return;
  const size_t i = (size_t)blockIdx.y * M + v;
  gvconn[i] += min_grad(vconn[i], dil[i], gout[i]);
}

// g_out += seed * g_reach (the seeded start of the flood fill)
__global__ void k_cav_bwd_seed(const double* __restrict__ greach, double* __restrict__ gvconn, CavGeo G, int seed) {
  const size_t v = (size_t)blockIdx.x * kT + threadIdx.x;
  if (v >= G.M) return;
  const size_t i = (size_t)blockIdx.y * G.M + v;
  int x, y, z;
  G.coords(v, x, y, z);
  if (is_seed(G, seed, x, y, z)) gvconn[i] += greach[i];
}

__global__ void k_cav_add(double* __restrict__ a, const double* __restrict__ b, size_t n) {
  const size_t i = (size_t)blockIdx.x * kT + threadIdx.x + (size_t)blockIdx.y * n;
  if ((size_t)blockIdx.x * kT + threadIdx.x < n) a[i] += b[i];
}

// dP/drho of the cell: the tile copies summed, times d sigmoid / d rho
__global__ void k_cav_untile(const double* __restrict__ gvoid, const double* __restrict__ void_uc,
                             double* __restrict__ grad, CavGeo G, double beta) {
  const int r = G.r;
  const size_t N = (size_t)r * r * r;
  const size_t i = (size_t)blockIdx.x * kT + threadIdx.x;
  if (i >= N) return;
  const int b = blockIdx.y;
  const int x = (int)(i / ((size_t)r * r)), y = (int)((i / r) % r), z = (int)(i % r);
  double acc = 0.0;
  for (int a = 0; a < G.X / r; ++a)
    for (int c = 0; c < G.Y / r; ++c)
      for (int d = 0; d < G.Z / r; ++d) acc += gvoid[(size_t)b * G.M + G.index(a * r + x, c * r + y, d * r + z)];
  const double s = void_uc[(size_t)b * N + i];
  grad[(size_t)b * N + i] = acc * (-beta) * s * (1.0 - s);
}

void cavity(const double* rho, const CavityPlan& p, double* P, double* grad, void* work, cudaStream_t s) {
  if (p.r < 2 || p.B < 1 || p.rad < 0 || p.min_channel_rad < 0 || p.nsteps < 0)
    throw std::runtime_error("cavity penalty: bad sizes");
  if (p.rad > 100 || p.min_channel_rad > 100) throw std::runtime_error("cavity penalty: radius too large");
  for (int a = 0; a < 3; ++a)
    if (p.tiles[a] < 1) throw std::runtime_error("cavity penalty: tiles must be >= 1");
  const bool array = p.tiles[0] > 1 || p.tiles[1] > 1 || p.tiles[2] > 1;
  CavGeo G{p.r, p.dims(0), p.dims(1), p.dims(2), p.M(), (p.periodic && !array) ? 1 : 0};
  if (G.periodic) {
    const int mn = std::min(G.X, std::min(G.Y, G.Z));
    if (2 * p.rad + 1 > mn || 2 * p.min_channel_rad + 1 > mn)
      throw std::runtime_error("cavity penalty: window wider than the periodic cell");
  }
  if (G.M > (size_t)INT32_MAX) throw std::runtime_error("cavity penalty: supercell too large");
  CavWork w;
  cav_parts(p, work, &w);
  const size_t N = (size_t)p.r * p.r * p.r, BM = (size_t)p.B * G.M;
  const dim3 gN(nb(N), p.B), gM(nb(G.M), p.B);
  const int focus = p.focused() ? 1 : 0;
  const double count = focus ? (double)N : (double)G.M;
  const int mcr = p.min_channel_rad;
  // three passes z, y, x of a separable pool: in -> out, offsets off[0..2]
  auto pool3 = [&](const double* in, double* out, signed char* off, int rad, double sign, double pad,
                   const double* vmin, double* min_out) {
    PR_LAUNCH(k_cav_pass<<<gM, kT, 0, s>>>(in, w.t1, off, G, 2, rad, sign, 1.0, pad, nullptr, nullptr));
    PR_LAUNCH(k_cav_pass<<<gM, kT, 0, s>>>(w.t1, w.t2, off + BM, G, 1, rad, 1.0, 1.0, pad, nullptr, nullptr));
    PR_LAUNCH(k_cav_pass<<<gM, kT, 0, s>>>(w.t2, out, off + 2 * BM, G, 0, rad, 1.0, sign, pad, vmin, min_out));
  };
  // adjoint of pool3: gout at the output -> gin (x, y, z passes in reverse)
  auto pool3_adj = [&](const double* gout, const signed char* off, double* gin, int rad, int accumulate,
                       const double* vmin, const double* outv) {
    PR_LAUNCH(k_cav_pass_adj<<<gM, kT, 0, s>>>(gout, off + 2 * BM, w.g2, G, 0, rad, 0, vmin, outv));
    PR_LAUNCH(k_cav_pass_adj<<<gM, kT, 0, s>>>(w.g2, off + BM, w.g1, G, 1, rad, 0, nullptr, nullptr));
    PR_LAUNCH(k_cav_pass_adj<<<gM, kT, 0, s>>>(w.g1, off, gin, G, 2, rad, accumulate, nullptr, nullptr));
  };
  PR_LAUNCH(k_cav_void<<<gN, kT, 0, s>>>(rho, w.void_uc, N, p.void_thresh, p.beta));
  PR_LAUNCH(k_cav_tile<<<gM, kT, 0, s>>>(w.void_uc, w.vsc, G));
  const double* vconn = w.vsc;
  if (mcr > 0) {  // opening: erosion -maxpool(-x) with pad 1, then dilation with pad 0
    pool3(w.vsc, w.er, w.er_off, mcr, -1.0, -1.0, nullptr, nullptr);
    pool3(w.er, w.vconn, w.di_off, mcr, 1.0, 0.0, nullptr, nullptr);
    vconn = w.vconn;
  }
  PR_LAUNCH(k_cav_seed<<<gM, kT, 0, s>>>(vconn, w.reach0, G, p.seed));
  double* reach = w.reach0;
  double* other = w.reach1;
  const int steps = p.rad > 0 ? p.nsteps : 0;
  const dim3 gF((unsigned)(((G.X + FT - 1) / FT) * ((G.Y + FT - 1) / FT) * ((G.Z + FT - 1) / FT)), p.B);
  for (int t = 0; t < steps; ++t) {
    if (p.rad == 1)
      PR_LAUNCH(k_cav_fill_fwd<<<gF, FTHREADS, 0, s>>>(reach, vconn, other, w.tape + (size_t)t * BM, G));
    else
      pool3(reach, w.dil + (size_t)t * BM, w.off + (size_t)t * 3 * BM, p.rad, 1.0, 0.0, vconn, other);
    std::swap(reach, other);
  }
  PR_LAUNCH(k_cav_trapped<<<gM, kT, 0, s>>>(w.vsc, reach, w.part, G, focus));
  PR_LAUNCH(k_cav_total<<<p.B, kT, 0, s>>>(w.part, (int)gM.x, P, count));
  if (!grad) return;
  double* gr = w.gr0;
  double* gr_other = w.gr1;
  PR_LAUNCH(k_cav_bwd_init<<<gM, kT, 0, s>>>(w.vsc, reach, w.gvoid, gr, w.gvconn, G, focus, 1.0 / count));
  for (int t = steps - 1; t >= 0; --t) {
    if (p.rad == 1) {
      PR_LAUNCH(k_cav_fill_bwd<<<gF, FTHREADS, 0, s>>>(gr, w.tape + (size_t)t * BM, gr_other, w.gvconn, G));
    } else {
      const double* dil = w.dil + (size_t)t * BM;
      PR_LAUNCH(k_cav_min_vconn<<<gM, kT, 0, s>>>(gr, vconn, dil, w.gvconn, G.M));
      pool3_adj(gr, w.off + (size_t)t * 3 * BM, gr_other, p.rad, 0, vconn, dil);
    }
    std::swap(gr, gr_other);
  }
  PR_LAUNCH(k_cav_bwd_seed<<<gM, kT, 0, s>>>(gr, w.gvconn, G, p.seed));
  if (mcr > 0) {
    pool3_adj(w.gvconn, w.di_off, gr_other, mcr, 0, nullptr, nullptr);  // through the dilation
    pool3_adj(gr_other, w.er_off, w.gvoid, mcr, 1, nullptr, nullptr);   // through the erosion (signs cancel)
  } else {
    PR_LAUNCH(k_cav_add<<<gM, kT, 0, s>>>(w.gvoid, w.gvconn, G.M));
  }
  PR_LAUNCH(k_cav_untile<<<gN, kT, 0, s>>>(w.gvoid, w.void_uc, grad, G, p.beta));
}

}  // namespace maple_pr
