// maple_b200 runtime: context, operator hierarchy, MG-PCG driver, OC step and
// the C ABI declared in include/maple_b200.h.
#include "../../include/maple_b200.h"
#include "kernels.cuh"
#include "ebe_tc.cuh"
#include "printability.h"
#include "tables.h"

#include <nvtx3/nvToolsExt.h>

#include <cmath>
#include <memory>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <map>
#include <set>
#include <exception>
#include <mutex>
#include <thread>
#include <type_traits>
#include <stdexcept>
#include <string>
#include <vector>

namespace maple {

static thread_local std::string g_err;

struct Failure {
  int code;
  std::string msg;
};

#define CK(call)                                                                                  \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess)                                                                        \
      throw Failure{MAPLE_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_) + " at " +   \
                                      std::string(__FILE__) + ":" + std::to_string(__LINE__)};    \
  } while (0)
static std::atomic<unsigned long long> g_launches{0};
static thread_local unsigned long long tl_launches = 0;  // this thread's launches (graph capture accounting)
// kernels captured into the bodies of conditional IF nodes during the current
// capture (they run only when the condition is set; counted apart)
static thread_local unsigned long long tl_cond_kernels = 0;
#define CKL()                         \
  do {                                \
    CK(cudaGetLastError());           \
    g_launches.fetch_add(1);          \
    ++tl_launches;                    \
  } while (0)

static void require(bool ok, const std::string& msg) {
  if (!ok) throw Failure{MAPLE_E_BADARG, msg};
}

constexpr int kMaxLevels = 8;

// ---------------------------------------------------------------------------
// per-device constant tables (unit voxel; one Poisson ratio per process)
// ---------------------------------------------------------------------------
static std::mutex g_mu;
static double g_nu = -1.0;
static bool g_dev_ready[128];
static ElementTables g_tab;

static void ensure_tables(double nu) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_nu < 0) {
    element_tables(1.0, nu, 1.0, &g_tab);
    g_nu = nu;
  } else {
    require(g_nu == nu, "all contexts of a process must share one Poisson ratio");
  }
  int dev = 0;
  CK(cudaGetDevice(&dev));
  require(dev >= 0 && dev < 128, "device index out of range");
  if (!g_dev_ready[dev]) {
    float f3[576], f1[64];
    for (int i = 0; i < 576; ++i) f3[i] = (float)g_tab.Ke3[i];
    for (int i = 0; i < 64; ++i) f1[i] = (float)g_tab.Ke1[i];
    CK(cudaMemcpyToSymbol(c_Ke3d, g_tab.Ke3, sizeof(g_tab.Ke3)));
    CK(cudaMemcpyToSymbol(c_Ke3f, f3, sizeof(f3)));
    CK(cudaMemcpyToSymbol(c_Ke1d, g_tab.Ke1, sizeof(g_tab.Ke1)));
    CK(cudaMemcpyToSymbol(c_Ke1f, f1, sizeof(f1)));
    CK(cudaMemcpyToSymbol(c_Fe3, g_tab.Fe3, sizeof(g_tab.Fe3)));
    CK(cudaMemcpyToSymbol(c_X03, g_tab.X03, sizeof(g_tab.X03)));
    CK(cudaMemcpyToSymbol(c_KX3, g_tab.KX3, sizeof(g_tab.KX3)));
    CK(cudaMemcpyToSymbol(c_Fe1, g_tab.Fe1, sizeof(g_tab.Fe1)));
    CK(cudaMemcpyToSymbol(c_X01, g_tab.X01, sizeof(g_tab.X01)));
    CK(cudaMemcpyToSymbol(c_KX1, g_tab.KX1, sizeof(g_tab.KX1)));
    CK(cudaMemcpyToSymbol(c_W, g_tab.W, sizeof(g_tab.W)));
    g_dev_ready[dev] = true;
  }
}

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
template <typename T>
struct Ops {
  bool alloc = false, vectors = false;  // density copy / solver vectors allocated
  T* rho = nullptr;                      // fine densities [B][N0]
  T* S[kMaxLevels] = {};                 // stencils (1 <= l < L-1)
  T* Dinv[kMaxLevels] = {};
  T* F[kMaxLevels] = {};                 // level RHS (l >= 1)
  T* U[kMaxLevels][2] = {};              // iterate ping-pong; result in U[l][1]
  T* Dd[kMaxLevels] = {};                // Chebyshev direction
  T* Res[kMaxLevels] = {};               // residual
  double* hi[kMaxLevels] = {};           // per-cell Chebyshev upper bound
  bool dinv0 = false;                    // Dinv[0] holds the fine-level block inverse of the current density
  T *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr;  // PCG (level 0)
};

struct Phys {
  int D = 0, R = 0;
  double kscale = 0, fscale = 0, xscale = 0;  // stiffness, load and X0 scale at resolution r
  bool alloc = false, built = false, solved = false, energies = false;
  bool current = false;  // the solution belongs to the current density
  int built_prec = -1;
  double* KE[kMaxLevels] = {};   // FP64 element matrices of level l >= 1
  bool ke1_formed = false;       // KE[1] holds this density's level-1 element matrices
  double* S64c = nullptr;        // FP64 coarsest stencil
  double* Ainv = nullptr;        // FP64 coarsest inverse [B][ndof][ndof]
  double* cwork = nullptr;
  double* F64 = nullptr;         // RHS [B][N][R][D]
  double* u64 = nullptr;         // solution
  double* r64 = nullptr;         // residual (FP64)
  double *p64 = nullptr, *q64 = nullptr;  // mixed-precision PCG vectors (z stays FP32)
  float* b32 = nullptr;          // right-hand side of the FP32 inner solve (refinement mode)
  double* u_prev = nullptr;      // the solution of the OC step before the last (extrapolated warm start)
  bool prev_valid = false;       // u_prev holds the previous OC step's solution of every active cell
  bool from_oc = false;          // u64 is the solution of the last maple_oc_step
  double* energy = nullptr;      // [B][N][R][R]
  double* H = nullptr;           // [B][R][R]
  Ops<double> o64;
  Ops<float> o32;
};

struct Scalars {
  double *rz, *rz_new, *pq, *rr, *bnorm2, *alpha, *beta;
  double* rtol2;  // [1] the tolerance of the running solve, squared
  int *done, *cell_done, *iters, *run;
};

// Per-solve scratch: the partial sums, PCG scalars, refinement scalars, pinned
// convergence flags and capture stream of one solve in flight.  A context has
// one lane per physics so that the elastic and thermal solves of an OC step
// can run at the same time (from two host threads, on two streams).
// NVTX range for profilers (nsys, ncu --nvtx): a no-op unless a tool is attached
struct Range {
  explicit Range(const char* name) { nvtxRangePushA(name); }
  ~Range() { nvtxRangePop(); }
  Range(const Range&) = delete;
  Range& operator=(const Range&) = delete;
};

struct Lane {
  double* part = nullptr;  // partial sums [B][nblk0][32]
  double* red = nullptr;   // reduced values [B][32]
  Scalars sc{};            // inner PCG scalars
  double *o_rr = nullptr, *o_bn = nullptr, *o_scale = nullptr, *o_inv = nullptr;  // outer refinement
  int *o_done = nullptr, *o_run = nullptr;
  int* o_live = nullptr;   // refinement: cells still refined (active, not broken down)
  int* rel = nullptr;      // reliable updates: per cell, a residual replacement is due
  unsigned* fin_count = nullptr;  // per cell: blocks of a fused update-and-reduce launch that finished
  double* o_t = nullptr;   // reliable updates: per (cell, rhs) rescaling of the direction
  int* h_flags = nullptr;  // pinned host [B + 2]: convergence flags, the device loop's count, IF executions
  int* loop = nullptr;     // device [3]: iterations run by the device-side loop, its limit, IF-node executions
  int* breakdown = nullptr;
  cudaStream_t cap_stream = nullptr;
  cudaStream_t cap_stream2 = nullptr;  // captures the body of a conditional node inside a capture
  // the coarsest-level inverse of a hierarchy build runs here, beside the
  // power iterations of the other levels
  cudaStream_t side = nullptr;
  cudaEvent_t side_fork = nullptr, side_join = nullptr;
  // power iterations of the levels below 1, concurrent: a stream, events and
  // partial sums per level
  cudaStream_t pw[kMaxLevels] = {};
  cudaEvent_t pw_fork = nullptr, pw_join[kMaxLevels] = {};
  double* pw_part[kMaxLevels] = {};
  double* pw_red[kMaxLevels] = {};
  int* fb_mask = nullptr;  // cells re-solved in FP64 after a mixed-precision breakdown
  int* fb_bad = nullptr;   // per cell: the iterate holds a non-finite value
};

// lane of the calling thread: set by LaneScope around each physics' work
static thread_local int tl_lane = 0;
struct LaneScope {
  int prev;
  explicit LaneScope(int lane) : prev(tl_lane) { tl_lane = lane; }
  ~LaneScope() { tl_lane = prev; }
};

}  // namespace maple

struct maple_ctx {
  int dev = 0;
  int r = 0, B = 0, L = 0;
  int n[maple::kMaxLevels] = {};
  double E = 1, nu = 0.3, kappa = 1;
  maple::Phys ph[2];
  std::vector<void*> allocs;
  size_t bytes = 0;
  int* active = nullptr;          // device [B]
  std::vector<int> h_active;
  maple::Lane lanes[2];           // per-solve scratch, one lane per physics
  // OC step buffers
  double *x_sym = nullptr, *dJdx = nullptr, *dJf = nullptr, *Jv = nullptr, *terms = nullptr, *G3 = nullptr,
         *G1 = nullptr, *stats = nullptr, *ocpart = nullptr, *ocvf = nullptr;
  unsigned* bar = nullptr;
  int* err = nullptr;             // device: an OC grid barrier gave up
  int* h_err = nullptr;           // pinned host copy of err
  int oc_G = 0;
  // captured PCG iteration bodies: [physics][precision]
  struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
    unsigned long long kernels = 0;  // kernel nodes per replay (for launch counting)
    // the same body inside a conditional WHILE node (the whole solve in one replay)
    cudaGraphExec_t loop_exec = nullptr;
    unsigned long long loop_kernels = 0;  // kernels per loop iteration
    bool loop_failed = false;             // the runtime refused the conditional graph
    unsigned long long cond_kernels = 0;  // kernels of the IF-node body per execution (not in the counts above)
  } graphs[2][4];  // [physics][FP64 PCG, flexible mixed PCG, FP32 inner PCG of refinement, reliable updates]
  cudaStream_t aux_stream = nullptr;  // second physics of a concurrent OC step
  cudaEvent_t aux_fork = nullptr, aux_join = nullptr;
  // the elastic solve of a concurrent OC step runs on a stream of the highest
  // priority: its chain is the longer one, the thermal solve fills the SMs it
  // leaves free
  cudaStream_t hi_stream = nullptr;
  cudaEvent_t hi_fork = nullptr, hi_join = nullptr;
  bool use_graphs = true;
  bool concurrent = true;  // elastic and thermal solves of an OC step on two streams
  int split_min_n = 32;    // coarse levels with n >= this (n % 8 == 0) use k_apply_stencil_split; 0: never
  int nine_max_n = 64;     // coarse levels with n <= this use k_apply_stencil_nine; 0: never
  bool tail_fused = true;  // FP32 8^3 level + 4^3 coarsest solve as one cluster launch (k_tail_cycle)
  bool pdl = true;         // coarse-level launches with programmatic dependent launch
  bool device_loop = true; // conditional graph nodes: PCG iterations looped on device, IF node of the replacement
  bool fused_reduce = true; // the PCG update's last block per cell runs the convergence reduction
  int sym_kind = 0, sym_mask = 0;  // symmetry projection of the OC step (SYM_*)
  // manufacturability penalties of the OC objective (maple_set_penalties)
  double lambda_print = 0, lambda_cavity = 0;
  bool print_set = false, cavity_set = false;
  maple_pr::OverhangPlan oplan;
  maple_pr::CavityPlan cplan;
  void* pen_work = nullptr;
  size_t pen_bytes = 0;
  double *pen_rho = nullptr, *P_print = nullptr, *P_cav = nullptr, *dP_print = nullptr, *dP_cav = nullptr,
         *J_raw = nullptr;
  // per-kernel-class event timing of fine-level launches (bench instrumentation)
  bool profiling = false;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  struct Rec {
    std::string name;
    double bytes;
    size_t ev;
  };
  std::vector<Rec> recs;
  // options
  int cheb_degree = 1;         // levels 0 and 1 (level 1 of at most 16^3 nodes: see cheb_degree_coarse)
  int cheb_degree_coarse = 0;  // levels >= 2; 0: automatic
  double cheb_ratio = 10.0;
  int power_iters = 12;
  double power_safety = 1.15;
  double inner_rtol = 1e-5;
  int check_every = 1;
  int mixed_mode = 0;  // MAPLE_MIXED_FLEXIBLE (default), MAPLE_MIXED_REFINE or MAPLE_MIXED_RELIABLE
  double rel_delta = 1e-3;  // reliable updates: residual reduction per FP32 segment
  int rel_handover = 120;   // reliable updates: iterations before an unconverged cell moves to the flexible form
  double extrap = 0.0;  // warm start of maple_oc_step: u + extrap * (u - u_prev)
};

#define LN(c) ((c)->lanes[maple::tl_lane])

namespace maple {

// Optional event bracketing of every launch (bench instrumentation).
static bool prof_on(maple_ctx* c) { return c->profiling && c->ev_used + 2 <= c->ev_pool.size(); }
static void prof_begin(maple_ctx* c, cudaStream_t s) {
  if (prof_on(c)) CK(cudaEventRecord(c->ev_pool[c->ev_used], s));
}
static void prof_end(maple_ctx* c, cudaStream_t s, const char* text, double bytes) {
  if (!prof_on(c)) return;
  CK(cudaEventRecord(c->ev_pool[c->ev_used + 1], s));
  std::string name(text);
  const size_t cut = name.find("<<<");
  if (cut != std::string::npos) name = name.substr(0, cut);
  name.erase(std::remove(name.begin(), name.end(), ' '), name.end());
  const std::string pdl = "launch_pdl(";  // launch_pdl(kernel<...>, grid, ...)
  if (name.rfind(pdl, 0) == 0) name = name.substr(pdl.size(), name.find(",gt,") - pdl.size());
  c->recs.push_back({name, bytes, c->ev_used});
  c->ev_used += 2;
}
#define KL(ctx, stream, ...)                \
  do {                                      \
    prof_begin(ctx, stream);                \
    __VA_ARGS__;                            \
    CKL();                                  \
    prof_end(ctx, stream, #__VA_ARGS__, 0); \
  } while (0)

static void* dalloc(maple_ctx* c, size_t bytes) {
  void* p = nullptr;
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) throw Failure{MAPLE_E_NOMEM, std::string("cudaMalloc failed: ") + cudaGetErrorString(e)};
  c->allocs.push_back(p);
  c->bytes += bytes;
  return p;
}
template <typename T>
static T* dnew(maple_ctx* c, size_t count) {
  return reinterpret_cast<T*>(dalloc(c, count * sizeof(T)));
}

// Opt a kernel into `bytes` of dynamic shared memory on device `dev`, once per
// (kernel, device): the attribute is per device, and several host threads
// (the two physics lanes, or contexts of different threads) may launch the
// same kernel for the first time together.
static std::mutex g_attr_mu;
static std::set<std::pair<const void*, int>> g_attr_done;
template <typename K>
static void smem_attr(K* kernel, size_t bytes, int dev) {
  std::lock_guard<std::mutex> lk(g_attr_mu);
  const std::pair<const void*, int> key{reinterpret_cast<const void*>(kernel), dev};
  if (g_attr_done.count(key)) return;
  CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  g_attr_done.insert(key);
}

// Programmatic dependent launch pays where a launch is a wave or two of
// blocks: its prologue overlaps the previous kernel's drain.  On large grids
// the per-block griddepcontrol.wait costs more than it saves (256 cells of
// 32^3: +15% step time with it on every coarse launch), so only launches of
// at most kPdlMaxBlocks blocks (the fused tail: one wave of clusters) use the
// PDL instantiation of their kernel; the others launch the plain one.
constexpr size_t kPdlMaxBlocks = 8 * 148;
static bool use_pdl(const maple_ctx* c, dim3 grid, size_t max_blocks = kPdlMaxBlocks) {
  return c->pdl && (size_t)grid.x * grid.y * grid.z <= max_blocks;
}

// Launch the PDL instantiation of a kernel (it calls griddep_wait before
// reading its predecessors' output) with the programmatic-serialization
// attribute: it may start while the previous kernel in the stream drains.
template <typename... KArgs, typename... Args>
static void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  CK(cudaLaunchKernelEx(&cfg, kernel, args...));  // counted by the caller's CKL
}

static inline unsigned nblk(size_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }
// 16-byte alignment of a pointer (vector accesses; a caller's buffer may be only element-aligned)
static inline bool al16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }
static inline dim3 g2(size_t n, int B) { return dim3(nblk(n), (unsigned)B); }

static int nodes(int n) { return n * n * n; }

template <typename T>
static void alloc_ops(maple_ctx* c, Phys& p, Ops<T>& o, bool vectors) {
  const int B = c->B, RD = p.R * p.D, DD = p.D * p.D;
  const size_t N0 = nodes(c->n[0]);
  if (!o.alloc) o.rho = dnew<T>(c, (size_t)B * N0);
  o.alloc = true;
  // the FP64 operator of a mixed-precision solve needs only the density copy;
  // its solver vectors are added when the same context is first used in FP64
  if (vectors && !o.vectors) {
    o.vectors = true;
    for (int l = 0; l < c->L; ++l) {
      const size_t Nl = nodes(c->n[l]);
      if (l >= 1 && l < c->L - 1) {
        o.S[l] = dnew<T>(c, (size_t)B * 27 * DD * Nl);
        o.Dinv[l] = dnew<T>(c, (size_t)B * DD * Nl);
      }
      if (l >= 1) o.F[l] = dnew<T>(c, (size_t)B * Nl * RD);
      o.U[l][0] = dnew<T>(c, (size_t)B * Nl * RD);
      o.U[l][1] = dnew<T>(c, (size_t)B * Nl * RD);
      o.Dd[l] = dnew<T>(c, (size_t)B * Nl * RD);
      o.Res[l] = dnew<T>(c, (size_t)B * Nl * RD);
      o.hi[l] = dnew<double>(c, B);
    }
    o.Dinv[0] = dnew<T>(c, (size_t)B * N0 * DD);  // fine-level block inverse (k_fine_dinv)
    o.x = dnew<T>(c, (size_t)B * N0 * RD);
    o.r = dnew<T>(c, (size_t)B * N0 * RD);
    o.p = dnew<T>(c, (size_t)B * N0 * RD);
    o.q = dnew<T>(c, (size_t)B * N0 * RD);
  }
}

static void alloc_phys(maple_ctx* c, int phys) {
  Phys& p = c->ph[phys];
  if (p.alloc) return;
  const int B = c->B, D = p.D, R = p.R, k = 8 * D;
  const size_t N0 = nodes(c->n[0]);
  for (int l = 1; l < c->L; ++l) p.KE[l] = dnew<double>(c, (size_t)B * nodes(c->n[l]) * k * k);
  const int nc = c->n[c->L - 1], ndof = nodes(nc) * D;
  p.S64c = dnew<double>(c, (size_t)B * 27 * D * D * nodes(nc));
  p.Ainv = dnew<double>(c, (size_t)B * ndof * ndof);
  p.cwork = dnew<double>(c, (size_t)B * ndof * ndof);
  p.F64 = dnew<double>(c, (size_t)B * N0 * R * D);
  p.u64 = dnew<double>(c, (size_t)B * N0 * R * D);
  p.r64 = dnew<double>(c, (size_t)B * N0 * R * D);
  p.energy = dnew<double>(c, (size_t)B * N0 * R * R);
  p.H = dnew<double>(c, (size_t)B * R * R);
  CK(cudaMemset(p.u64, 0, (size_t)B * N0 * R * D * sizeof(double)));
  if (c->extrap > 0) p.u_prev = dnew<double>(c, (size_t)B * N0 * R * D);
  p.alloc = true;
}

template <typename T>
static Ops<T>& ops(Phys& p);
template <>
Ops<double>& ops<double>(Phys& p) { return p.o64; }
template <>
Ops<float>& ops<float>(Phys& p) { return p.o32; }

// ---------------------------------------------------------------------------
// operator application dispatch
// ---------------------------------------------------------------------------
template <typename T, int D, int R, int MODE>
static void apply(maple_ctx* c, Phys& p, Ops<T>& o, int l, ApplyArgs<T> a, const int* act, cudaStream_t s) {
  a.n = c->n[l];
  a.N = nodes(a.n);
  // the fine level applies the unit-voxel Ke0 and scales it; coarse stencils
  // were built from scaled element matrices already
  a.scale = l == 0 ? (T)p.kscale : (T)1;
  a.active = act;
  a.ratio = c->cheb_ratio;
  const dim3 g = g2(a.N, c->B);
  if (l == 0) {
    a.rho = o.rho;
    if constexpr (MODE == M_JAC0) {
      if (o.dinv0) {
        a.Dinv = o.Dinv[0];
        prof_begin(c, s);
        constexpr int W = Vec16<T>::n;
        const bool vec = a.N % W == 0 && al16(a.Dinv) && al16(a.f) && al16(a.out) && al16(a.dout);
        const dim3 grid(nblk(vec ? a.N / W : a.N), c->B);
        if (vec) {
          if (use_pdl(c, grid) && !prof_on(c))
            launch_pdl(k_fine_jac0_vec<T, D, R, true>, grid, dim3(kThreads), 0, s, a);
          else
            k_fine_jac0_vec<T, D, R><<<grid, kThreads, 0, s>>>(a);
        } else if (use_pdl(c, grid) && !prof_on(c)) {
          launch_pdl(k_fine_jac0<T, D, R, true>, grid, dim3(kThreads), 0, s, a);
        } else {
          k_fine_jac0<T, D, R><<<grid, kThreads, 0, s>>>(a);
        }
        CKL();
        if (prof_on(c)) {
          const double bytes = (double)c->B * a.N * ((double)D * D + 3.0 * R * D) * sizeof(T);
          prof_end(c, s, (std::string("k_fine_jac0<") + (sizeof(T) == 8 ? "f64," : "f32,") + std::to_string(D) +
                          "," + std::to_string(R) + ">").c_str(), bytes);
        }
        return;
      }
    }
    using G = FineTile<T, R * D>;
    smem_attr(k_apply_fine<T, D, R, MODE>, G::BYTES, c->dev);
    smem_attr(k_apply_fine<T, D, R, MODE, true>, G::BYTES, c->dev);
    prof_begin(c, s);
    const dim3 grid(fine_tiles(a.n), c->B);
    if (use_pdl(c, grid) && !prof_on(c))
      launch_pdl(k_apply_fine<T, D, R, MODE, true>, grid, dim3(kFineThreads), G::BYTES, s, a);
    else
      k_apply_fine<T, D, R, MODE><<<grid, kFineThreads, G::BYTES, s>>>(a);
    CKL();
    if (prof_on(c)) {
      static const char* mname[] = {"MV", "RES", "CHEB", "JAC0", "POWER"};
      // algorithmic bytes: rho once, each vector read or written once
      const int nvec = MODE == M_MV ? 2 : MODE == M_RES ? 3 : MODE == M_CHEB ? 5 : MODE == M_JAC0 ? 3 : 2;
      const double bytes = (double)c->B * a.N * ((double)sizeof(T) + (double)nvec * R * D * sizeof(T));
      const std::string nm = std::string("k_apply_fine<") + (sizeof(T) == 8 ? "f64," : "f32,") + std::to_string(D) +
                             "," + std::to_string(R) + "," + mname[MODE] + ">";
      prof_end(c, s, nm.c_str(), bytes);
    }
    return;
  } else {
    a.S = o.S[l];
    a.Dinv = o.Dinv[l];
    prof_begin(c, s);
    if constexpr (MODE == M_POWER) {
      static_assert(R == 1, "power iterations run on one column");
      k_apply_stencil_power<T, D>
          <<<dim3(ceil_div(a.N, kPowerNodes<D>), c->B), D * kPowerNodes<D>, 0, s>>>(a);
    } else {
      require(a.part == nullptr, "coarse-level applies produce no partial sums");
      bool split = false;
      if (c->nine_max_n > 0 && a.n <= c->nine_max_n) {
        const dim3 grid(ceil_div(a.N, NINE_NODES), c->B);
        if (use_pdl(c, grid))
          launch_pdl(k_apply_stencil_nine<T, D, R, MODE, true>, grid, dim3(NINE_THREADS), 0, s, a);
        else
          k_apply_stencil_nine<T, D, R, MODE><<<grid, NINE_THREADS, 0, s>>>(a);
        split = true;
      }
      if constexpr (R % 3 == 0) {
        if (!split && c->split_min_n > 0 && a.n >= c->split_min_n && a.n % ST_Z == 0) {
          using G = SplitTile<T, D, R>;
          smem_attr(k_apply_stencil_split<T, D, R, MODE>, G::BYTES, c->dev);
          const int tiles = (a.n / ST_Z) * (a.n / ST_Y) * (a.n / ST_X);
          k_apply_stencil_split<T, D, R, MODE><<<dim3(tiles, c->B), ST_THREADS, G::BYTES, s>>>(a);
          split = true;
        }
      }
      if (split) {
      } else if (a.n % CT == 0) {
        using G = CoarseTile<T, D, R>;
        smem_attr(k_apply_stencil_tile<T, D, R, MODE>, G::BYTES, c->dev);
        const int nt = a.n / CT;
        k_apply_stencil_tile<T, D, R, MODE><<<dim3(nt * nt * nt, c->B), G::THREADS, G::BYTES, s>>>(a);
      } else {
        k_apply_stencil<T, D, R, MODE><<<g2((size_t)a.N * R, c->B), kThreads, 0, s>>>(a);
      }
    }
    CKL();
    if (prof_on(c)) {
      static const char* mname[] = {"MV", "RES", "CHEB", "JAC0", "POWER"};
      const std::string nm = std::string("k_apply_stencil<") + (sizeof(T) == 8 ? "f64," : "f32,") +
                             std::to_string(D) + "," + std::to_string(R) + "," + mname[MODE] + ">@L" + std::to_string(l);
      // algorithmic bytes per node: the stencil (not for JAC0), the block
      // inverse (CHEB, JAC0, POWER), each vector read or written once
      const double es = sizeof(T), dd = D * D, rd = R * D;
      const double per_node = MODE == M_MV     ? (27 * dd + 2 * rd) * es
                              : MODE == M_RES  ? (27 * dd + 3 * rd) * es
                              : MODE == M_CHEB ? (27 * dd + dd + 5 * rd) * es
                              : MODE == M_JAC0 ? (dd + 3 * rd) * es
                                               : (27 * dd + dd + 2 * D) * es;
      prof_end(c, s, nm.c_str(), (double)c->B * a.N * per_node);
    }
  }
}

template <int K>
static void reduce(maple_ctx* c, const double* part, unsigned nb, double* out, cudaStream_t s) {
  KL(c, s, k_reduce_partials<K><<<c->B, kThreads, 0, s>>>(part, (int)nb, out));
}

// reduce a cell's partial sums and apply the PCG scalar step OP in one launch
template <int K, int OP>
static void reduce_op(maple_ctx* c, const double* part, unsigned nb, double* out, const RedOp& op, cudaStream_t s) {
  if (use_pdl(c, dim3(c->B)))
    KL(c, s, launch_pdl(k_reduce_op<K, OP, true>, dim3(c->B), dim3(kThreads), 0, s, part, (int)nb, out, op));
  else
    KL(c, s, k_reduce_op<K, OP><<<c->B, kThreads, 0, s>>>(part, (int)nb, out, op));
}

// ---------------------------------------------------------------------------
// hierarchy
// ---------------------------------------------------------------------------
template <typename T, int D>
static void power_bounds(maple_ctx* c, Phys& p, Ops<T>& o, cudaStream_t s, const int* act) {
  // level 0: the element bound holds for every density
  KL(c, s, k_fill<double><<<nblk(c->B), kThreads, 0, s>>>(o.hi[0], c->B, g_tab.lam_elem[D == 3 ? 0 : 1]));
  // Levels are independent: level 1 (the longest chain) runs on the
  // caller's stream, the deeper levels each on a stream of their own with
  // their own partial sums, joined back before the build returns.
  Lane& ln = LN(c);
  CK(cudaEventRecord(ln.pw_fork, s));
  for (int l = 1; l < c->L - 1; ++l) {
    const int Nl = nodes(c->n[l]);
    const size_t len = (size_t)c->B * Nl * D;
    cudaStream_t st = s;
    if (l > 1) {
      st = ln.pw[l];
      CK(cudaStreamWaitEvent(st, ln.pw_fork, 0));
    }
    double* part = ln.pw_part[l];
    double* red = ln.pw_red[l];
    T* v = o.U[l][0];
    T* w = o.U[l][1];
    KL(c, st, k_power_init<T><<<nblk(len), kThreads, 0, st>>>(v, len));
    for (int it = 0; it < c->power_iters; ++it) {
      ApplyArgs<T> a{};
      a.u = v;
      a.out = w;
      a.part = part;
      apply<T, D, 1, M_POWER>(c, p, o, l, a, act, st);
      std::swap(v, w);
    }
    reduce<2>(c, part, ceil_div(Nl, kPowerNodes<D>), red, st);
    KL(c, st, k_power_finish<<<nblk(c->B), kThreads, 0, st>>>(red, o.hi[l], c->B, c->power_safety));
    if (l > 1) {
      CK(cudaEventRecord(ln.pw_join[l], st));
      CK(cudaStreamWaitEvent(s, ln.pw_join[l], 0));
    }
  }
}

// Per-device copies of the host coarsening tables (M: level-1 child
// matrices, G: level-2 fine-element matrices), uploaded once and kept for the
// process; looked up under the lock (contexts may build on several threads).
enum { TAB_M = 0, TAB_G = 1 };
static const double* device_table(maple_ctx* c, int D, int which) {
  static double* slots[128][2][2] = {};
  std::lock_guard<std::mutex> lk(g_mu);
  double*& slot = slots[c->dev][D == 3 ? 0 : 1][which];
  if (!slot) {
    const int k = 8 * D;
    const double* src = which == TAB_M ? (D == 3 ? g_tab.M3 : g_tab.M1) : (D == 3 ? g_tab.G3 : g_tab.G1);
    const size_t bytes = (size_t)(which == TAB_M ? 8 : 64) * k * k * sizeof(double);
    double* m = nullptr;
    CK(cudaMalloc(&m, bytes));
    CK(cudaMemcpy(m, src, bytes, cudaMemcpyHostToDevice));
    slot = m;
  }
  return slot;
}

// level-1 element matrices into p.KE[1] (the direct build does not form them)
template <int D>
static void level1_elements(maple_ctx* c, Phys& p, cudaStream_t s, const int* act) {
  const int nc = c->n[1], k = 8 * D;
  const size_t tot = (size_t)nodes(nc) * k * k;
  KL(c, s, k_level1_elements<D><<<g2(tot, c->B), kThreads, 0, s>>>(p.o64.rho, device_table(c, D, TAB_M), p.KE[1], nc,
                                                                      p.kscale, act));
}

template <int D>
static void build_hierarchy(maple_ctx* c, int phys, int prec, cudaStream_t s, const int* mask = nullptr) {
  Range range(D == 3 ? "maple:build elastic" : "maple:build thermal");
  Phys& p = c->ph[phys];
  bool side_inverse = false;
  const int B = c->B, k = 8 * D, L = c->L;
  const int* act = mask ? mask : c->active;
  // With a level 2, the level-1 stencils and the level-2 element matrices
  // come straight from the fine densities (the level-1 element matrices,
  // 4.6 KB per level-1 element, are never formed); otherwise level 1 is the
  // coarsest and its element matrices are formed as before.
  const bool direct = L >= 3;
  if (direct) {
    const int n1 = c->n[1], N1 = nodes(n1), n2 = c->n[2], N2 = nodes(n2);
    const double* M = device_table(c, D, TAB_M);
    if (prec == MAPLE_FP64)
      KL(c, s, k_level1_stencils<double, D><<<g2((size_t)N1 * 27, B), kThreads, 0, s>>>(
                   p.o64.rho, M, p.o64.S[1], p.o64.Dinv[1], n1, p.kscale, act));
    else
      KL(c, s, k_level1_stencils<float, D><<<g2((size_t)N1 * 27, B), kThreads, 0, s>>>(
                   p.o64.rho, M, p.o32.S[1], p.o32.Dinv[1], n1, p.kscale, act));
    KL(c, s, k_level2_elements<D><<<dim3((unsigned)ceil_div(N2, kL2Elems), B), kThreads, 0, s>>>(
                 p.o64.rho, device_table(c, D, TAB_G), p.KE[2], n2, p.kscale, act));
    p.ke1_formed = false;
  } else {
    level1_elements<D>(c, p, s, act);
    p.ke1_formed = true;
  }
  for (int l = direct ? 2 : 1; l < L; ++l) {
    const int n = c->n[l], N = nodes(n);
    if (l < L - 1) {
      if (prec == MAPLE_FP64) {
        KL(c, s, k_stencil_from_elements<double, D><<<g2((size_t)N * 27, B), kThreads, 0, s>>>(
                     p.KE[l], p.o64.S[l], p.o64.Dinv[l], nullptr, n, act));
      } else {
        KL(c, s, k_stencil_from_elements<float, D><<<g2((size_t)N * 27, B), kThreads, 0, s>>>(
                     p.KE[l], p.o32.S[l], p.o32.Dinv[l], nullptr, n, act));
      }
      // coarsen to the next level
      const int nc = c->n[l + 1];
      const size_t smem = (size_t)2 * 8 * k * k * sizeof(double);
      CK(cudaFuncSetAttribute(k_coarsen_elements<D>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      KL(c, s, k_coarsen_elements<D><<<dim3(nodes(nc), B), 256, smem, s>>>(p.KE[l], p.KE[l + 1], nc, act));
    } else {
      const int ndof = N * D;
      KL(c, s, k_stencil_from_elements<double, D><<<g2((size_t)N * 27, B), kThreads, 0, s>>>(p.KE[l], (double*)nullptr,
                                                                                    (double*)nullptr, p.S64c, n, act));
      CK(cudaMemsetAsync(p.Ainv, 0, (size_t)B * ndof * ndof * sizeof(double), s));
      KL(c, s, k_dense_from_stencil<D><<<g2((size_t)N * 27, B), kThreads, 0, s>>>(p.S64c, p.Ainv, n, act));
      if (ndof <= kCholSmemMax) {
        const size_t sm = chol_smem_bytes(ndof);
        smem_attr(k_chol_inverse_smem, chol_smem_bytes(kCholSmemMax), c->dev);
        Lane& ln = LN(c);
        if (!ln.side) {
          int least = 0, greatest = 0;
          CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
          CK(cudaStreamCreateWithPriority(&ln.side, cudaStreamNonBlocking, tl_lane == 0 ? greatest : least));
          CK(cudaEventCreateWithFlags(&ln.side_fork, cudaEventDisableTiming));
          CK(cudaEventCreateWithFlags(&ln.side_join, cudaEventDisableTiming));
        }
        CK(cudaEventRecord(ln.side_fork, s));
        CK(cudaStreamWaitEvent(ln.side, ln.side_fork, 0));
        KL(c, ln.side, k_chol_inverse_smem<<<B, kCholThreads, sm, ln.side>>>(p.Ainv, ndof, D, act, nullptr));
        CK(cudaEventRecord(ln.side_join, ln.side));
        side_inverse = true;
      } else {
        KL(c, s, k_chol_inverse<<<B, 512, 0, s>>>(p.Ainv, p.cwork, ndof, D, act, nullptr));
      }
    }
  }
  // the fine level's block inverse, for the first smoothing step
  {
    const int n0 = c->n[0];
    const dim3 g(nblk(nodes(n0)), B);
    if (prec == MAPLE_FP64) {
      KL(c, s, k_fine_dinv<double, D><<<g, kThreads, 0, s>>>(p.o64.rho, p.o64.Dinv[0], n0, (double)p.kscale, act));
      p.o64.dinv0 = true;
    } else {
      KL(c, s, k_fine_dinv<float, D><<<g, kThreads, 0, s>>>(p.o32.rho, p.o32.Dinv[0], n0, (float)p.kscale, act));
      p.o32.dinv0 = true;
    }
  }
  if (prec == MAPLE_FP64)
    power_bounds<double, D>(c, p, p.o64, s, act);
  else
    power_bounds<float, D>(c, p, p.o32, s, act);
  if (side_inverse) CK(cudaStreamWaitEvent(s, LN(c).side_join, 0));
  p.built = true;
  p.built_prec = prec;
  // the current solution (if any) stays: it is the warm start for this density
  p.current = false;
  p.energies = false;
}

// ---------------------------------------------------------------------------
// V-cycle (symmetric: Chebyshev pre/post, exact FP64 coarsest solve)
// ---------------------------------------------------------------------------
// Whether the FP32 V-cycle runs level l (8^3 nodes, above the 4^3-node
// coarsest level) as one k_tail_cycle launch.  The first call per (D, R,
// device) opts the kernel in to its shared memory and asks the occupancy
// calculator whether one 8-CTA cluster of it fits on the device.
template <int D, int R>
static bool tail_fused_ok(maple_ctx* c, int l, int deg) {
  if (!c->tail_fused || l < 1 || l != c->L - 2 || c->n[l] != TAIL_N || c->n[l + 1] != TAIL_NC ||
      deg < 1 || deg > kTailMaxDegree)
    return false;
  static std::mutex mu;
  static std::map<int, bool> fits;
  std::lock_guard<std::mutex> lk(mu);
  auto it = fits.find(c->dev);
  if (it != fits.end()) return it->second;
  const size_t bytes = TailSmem<D, R>::BYTES;
  bool ok = cudaFuncSetAttribute(k_tail_cycle<D, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) ==
                cudaSuccess &&
            cudaFuncSetAttribute(k_tail_cycle<D, R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) ==
                cudaSuccess;
  if (ok) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(TAIL_CTAS, 1, 1);
    cfg.blockDim = dim3(TAIL_THREADS, 1, 1);
    cfg.dynamicSmemBytes = bytes;
    int clusters = 0;
    ok = cudaOccupancyMaxActiveClusters(&clusters, k_tail_cycle<D, R>, &cfg) == cudaSuccess && clusters > 0;
  }
  (void)cudaGetLastError();  // a refused query leaves the separate launches in use
  fits[c->dev] = ok;
  return ok;
}

template <typename T, int D, int R>
static void vcycle(maple_ctx* c, Phys& p, Ops<T>& o, int l, const T* f, const int* act, double* rz_part,
                   cudaStream_t s) {
  const int B = c->B;
  if (l == c->L - 1) {
    const int ndof = nodes(c->n[l]) * D;
    KL(c, s, k_coarse_solve<T, R><<<dim3((ndof + 7) / 8, B), kThreads, 0, s>>>(p.Ainv, f, o.U[l][1], ndof, D, act));
    return;
  }
  // Chebyshev degree per level.  Automatic (cheb_degree_coarse == 0): 3 on
  // every level below level 1 and on a level 1 of at most 16^3 nodes, where
  // the extra cheap sweeps save more PCG iterations than they cost; the fine
  // level and a larger level 1 keep the common degree.  An explicit
  // cheb_degree_coarse applies to levels 2 and deeper.
  int deg = c->cheb_degree;
  if (l >= 1) {
    if (c->cheb_degree_coarse > 0) {
      if (l >= 2) deg = c->cheb_degree_coarse;
    } else if (l >= 2 || c->n[l] <= 16) {
      deg = std::max(3, deg);
    }
  }
  if constexpr (std::is_same<T, float>::value) {
    if (tail_fused_ok<D, R>(c, l, deg)) {
      // smoothing, residual, restriction, coarsest solve and prolongation of
      // this level in one launch; the result lands in U[l][1] as below
      TailArgs ta{o.S[l], o.Dinv[l], f, o.U[l][1], p.Ainv, o.hi[l], c->cheb_ratio, deg, act};
      prof_begin(c, s);
      const dim3 grid(TAIL_CTAS, c->B);
      if (use_pdl(c, grid, 148))
        launch_pdl(k_tail_cycle<D, R, true>, grid, dim3(TAIL_THREADS), TailSmem<D, R>::BYTES, s, ta);
      else
        k_tail_cycle<D, R><<<grid, TAIL_THREADS, TailSmem<D, R>::BYTES, s>>>(ta);
      CKL();
      if (prof_on(c)) {
        // algorithmic bytes per cell: the level's stencils, block inverses,
        // right-hand side and result once, and the coarsest inverse
        const double N = nodes(TAIL_N), ndof = nodes(TAIL_NC) * D;
        const double cell = (27.0 * D * D + D * D + 2.0 * R * D) * N * sizeof(float) + ndof * ndof * sizeof(double);
        prof_end(c, s, ("k_tail_cycle<" + std::to_string(D) + "," + std::to_string(R) + ">").c_str(), c->B * cell);
      }
      return;
    }
  }
  int cur = 0;
  {
    ApplyArgs<T> a{};
    a.f = f;
    a.u = nullptr;
    a.out = o.U[l][0];
    a.din = o.Dd[l];
    a.dout = o.Dd[l];
    a.hi = o.hi[l];
    a.step = 0;
    apply<T, D, R, M_JAC0>(c, p, o, l, a, act, s);
  }
  for (int st = 1; st < deg; ++st) {
    ApplyArgs<T> a{};
    a.f = f;
    a.u = o.U[l][cur];
    a.out = o.U[l][1 - cur];
    a.din = o.Dd[l];
    a.dout = o.Dd[l];
    a.hi = o.hi[l];
    a.step = st;
    apply<T, D, R, M_CHEB>(c, p, o, l, a, act, s);
    cur ^= 1;
  }
  {
    ApplyArgs<T> a{};
    a.f = f;
    a.u = o.U[l][cur];
    a.out = o.Res[l];
    apply<T, D, R, M_RES>(c, p, o, l, a, act, s);
  }
  const int nc = c->n[l + 1];
  const dim3 gt = g2((size_t)nodes(nc) * R * D, B);
  if (use_pdl(c, gt))
    KL(c, s, launch_pdl(k_restrict<T, R * D, true>, gt, dim3(kThreads), 0, s, (const T*)o.Res[l], o.F[l + 1], nc, act));
  else
    KL(c, s, k_restrict<T, R * D><<<gt, kThreads, 0, s>>>(o.Res[l], o.F[l + 1], nc, act));
  vcycle<T, D, R>(c, p, o, l + 1, o.F[l + 1], act, nullptr, s);
  if (use_pdl(c, gt))
    KL(c, s, launch_pdl(k_prolong_add<T, R * D, true>, gt, dim3(kThreads), 0, s, (const T*)o.U[l + 1][1], o.U[l][cur],
                        nc, act));
  else
    KL(c, s, k_prolong_add<T, R * D><<<gt, kThreads, 0, s>>>(o.U[l + 1][1], o.U[l][cur], nc, act));
  for (int st = 0; st < deg; ++st) {
    ApplyArgs<T> a{};
    a.f = f;
    a.u = o.U[l][cur];
    a.out = o.U[l][1 - cur];
    a.din = o.Dd[l];
    a.dout = o.Dd[l];
    a.hi = o.hi[l];
    a.step = st;
    if (st == deg - 1 && rz_part) {
      a.part = rz_part;
      a.dot_f_out = 1;
    }
    apply<T, D, R, M_CHEB>(c, p, o, l, a, act, s);
    cur ^= 1;
  }
}

// ---------------------------------------------------------------------------
// PCG on level 0 in precision T
// ---------------------------------------------------------------------------
static bool all_done(maple_ctx* c, const int* cell_done, const int* run_ref, cudaStream_t s) {
  CK(cudaMemcpyAsync(LN(c).h_flags, cell_done, c->B * sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  for (int b = 0; b < c->B; ++b)
    if (!LN(c).h_flags[b] && c->h_active[b]) return false;
  return true;
}

__global__ void k_init_flags(const int* active, const int* outer_run, int* done, int* cell_done, int* run, int* iters,
                             int B, int R) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  const int a = (active ? active[b] : 1) && (outer_run ? outer_run[b] : 1);
  run[b] = a;
  cell_done[b] = a ? 0 : 1;
  iters[b] = 0;
  for (int r = 0; r < R; ++r) done[b * R + r] = a ? 0 : 1;
}

// Ends one iteration of the device-side PCG loop: counts it and keeps the
// loop running while an active cell has not converged and fewer than
// loop[1] iterations ran.  One CTA.
__global__ void k_loop_next(cudaGraphConditionalHandle h, const int* __restrict__ cell_done, int B, int* loop) {
  int open = 0;
  for (int b = threadIdx.x; b < B; b += blockDim.x) open |= cell_done[b] == 0;
  open = __syncthreads_or(open);
  if (threadIdx.x == 0) {
    const int n = loop[0] + 1;
    loop[0] = n;
    cudaGraphSetConditional(h, (open && n < loop[1]) ? 1u : 0u);
  }
}

__global__ void k_loop_arm(int* loop, int limit) {
  loop[0] = 0;
  loop[1] = limit;
}

// Captures the iteration body, followed by k_loop_next, as the body of a
// conditional WHILE node, so that one replay runs a whole solve with no host
// round trip between iterations.  Returns false (and the caller keeps the
// per-iteration graphs) when the runtime refuses any part of it.
template <typename Body>
static bool loop_graph(maple_ctx* c, maple_ctx::GraphEntry& ge, Body& body) {
  if (ge.loop_exec) return true;
  if (ge.loop_failed) return false;
  Lane& ln = LN(c);
  if (!ln.cap_stream) CK(cudaStreamCreateWithFlags(&ln.cap_stream, cudaStreamNonBlocking));
  cudaGraph_t g = nullptr;
  CK(cudaGraphCreate(&g, 0));
  bool ok = false;
  const unsigned long long before = tl_launches;
  tl_cond_kernels = 0;
  cudaGraphConditionalHandle h{};
  cudaGraphNodeParams np{};
  cudaGraphNode_t node{};
  if (cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) == cudaSuccess) {
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    if (cudaGraphAddNode(&node, g, nullptr, 0, &np) == cudaSuccess &&
        cudaStreamBeginCaptureToGraph(ln.cap_stream, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      bool captured = true;
      try {
        body(ln.cap_stream);
        KL(c, ln.cap_stream, k_loop_next<<<1, 256, 0, ln.cap_stream>>>(h, ln.sc.cell_done, c->B, ln.loop));
      } catch (const Failure&) {
        captured = false;
      }
      cudaGraph_t out = nullptr;
      const bool ended = cudaStreamEndCapture(ln.cap_stream, &out) == cudaSuccess;
      ok = captured && ended && cudaGraphInstantiate(&ge.loop_exec, g, 0) == cudaSuccess;
    }
  }
  (void)cudaGetLastError();  // a refused step leaves the per-iteration graphs in use
  cudaGraphDestroy(g);
  const unsigned long long captured = tl_launches - before;
  ge.loop_kernels = captured - tl_cond_kernels;
  ge.cond_kernels = tl_cond_kernels;
  g_launches.fetch_sub(captured);  // captured, not launched
  tl_launches -= captured;
  if (!ok) {
    if (ge.loop_exec) cudaGraphExecDestroy(ge.loop_exec);
    ge.loop_exec = nullptr;
    ge.loop_failed = true;
  }
  return ok;
}

// Runs the PCG iteration body until every active cell has converged or maxit
// iterations ran.  The first iteration of a solve always runs eagerly, which
// also performs the one-time kernel attribute setup outside of any capture.
// With graphs, the rest runs as one replay of the device-side loop
// (loop_graph) and the host waits once per solve; where that is off or
// refused, the body is captured once into a CUDA graph per (physics, solve
// form) and replayed per iteration, the convergence flags read back after
// every check_every replays.  Either graph serves every tolerance (it is read
// on device); cells that converged skip all further work on device.
template <typename Body>
static void run_iterations(maple_ctx* c, maple_ctx::GraphEntry& ge, int maxit, Body& body,
                           cudaStream_t s) {
  const bool graphs = c->use_graphs && !c->profiling;
  int first = 1;
  if (graphs && c->device_loop && maxit > 1) {
    body(s);
    if (all_done(c, LN(c).sc.cell_done, nullptr, s)) return;
    if (loop_graph(c, ge, body)) {
      Lane& ln = LN(c);
      KL(c, s, k_loop_arm<<<1, 1, 0, s>>>(ln.loop, maxit - 1));
      CK(cudaGraphLaunch(ge.loop_exec, s));
      CK(cudaMemcpyAsync(ln.h_flags + c->B, ln.loop, sizeof(int), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      const unsigned long long n = (unsigned long long)std::max(ln.h_flags[c->B], 0) * ge.loop_kernels;
      g_launches.fetch_add(n);
      tl_launches += n;
      return;
    }
    first = 2;
  }
  for (int it = first; it <= maxit; ++it) {
    if (!graphs || it == 1) {
      body(s);
    } else {
      if (ge.exec == nullptr) {
        if (!LN(c).cap_stream) CK(cudaStreamCreateWithFlags(&LN(c).cap_stream, cudaStreamNonBlocking));
        cudaGraph_t graph = nullptr;
        const unsigned long long before = tl_launches;
        tl_cond_kernels = 0;
        CK(cudaStreamBeginCapture(LN(c).cap_stream, cudaStreamCaptureModeThreadLocal));
        try {
          body(LN(c).cap_stream);
        } catch (...) {
          cudaStreamEndCapture(LN(c).cap_stream, &graph);
          if (graph) cudaGraphDestroy(graph);
          throw;
        }
        CK(cudaStreamEndCapture(LN(c).cap_stream, &graph));
        CK(cudaGraphInstantiate(&ge.exec, graph, 0));
        CK(cudaGraphDestroy(graph));
        const unsigned long long captured = tl_launches - before;
        ge.kernels = captured - tl_cond_kernels;
        ge.cond_kernels = tl_cond_kernels;
        g_launches.fetch_sub(captured);  // captured, not launched
        tl_launches -= captured;
      }
      CK(cudaGraphLaunch(ge.exec, s));
      g_launches.fetch_add(ge.kernels);
    }
    if (it % c->check_every == 0 || it == maxit) {
      if (all_done(c, LN(c).sc.cell_done, nullptr, s)) break;
    }
  }
}

static void drop_graphs(maple_ctx* c) {
  for (auto& row : c->graphs)
    for (auto& ge : row) {
      if (ge.exec) cudaGraphExecDestroy(ge.exec);
      if (ge.loop_exec) cudaGraphExecDestroy(ge.loop_exec);
      ge.exec = nullptr;
      ge.loop_exec = nullptr;
      ge.loop_failed = false;
    }
}


// x += alpha p, r -= alpha q with the partial sums of r.r (16-byte vectors
// when the node count and every pointer allow: a caller's buffer may be only
// element-aligned); returns the number of partial blocks
template <typename T, int R, int D>
static unsigned pcg_update(maple_ctx* c, T* x, T* r, const T* p, const T* q, const double* alpha, double* part,
                           int N, int B, const int* run, cudaStream_t s) {
  constexpr int W = Vec16<T>::n;
  if (N % W == 0 && al16(x) && al16(r) && al16(p) && al16(q)) {
    const unsigned nb = nblk((size_t)(N / W));
    const dim3 grid(nb, B);
    const RedOp none{};
    if (use_pdl(c, grid))
      KL(c, s, launch_pdl(k_pcg_update_vec<T, R, D, true>, grid, dim3(kThreads), 0, s, x, r, p, q, alpha, part, N,
                          run, (unsigned*)nullptr, (double*)nullptr, none));
    else
      KL(c, s, k_pcg_update_vec<T, R, D><<<grid, kThreads, 0, s>>>(x, r, p, q, alpha, part, N, run, nullptr, nullptr,
                                                                   none));
    return nb;
  }
  KL(c, s, k_pcg_update<T, R, D><<<g2(N, B), kThreads, 0, s>>>(x, r, p, q, alpha, part, N, run));
  return nblk(N);
}

// The update followed by the reduction OP of its partial sums (RED_CHECK or
// RED_RELCHECK into out): with the vector kernel, its last block per cell runs
// the reduction (one launch instead of two); otherwise the separate launch.
template <typename T, int R, int D, int OP>
static void pcg_update_reduce(maple_ctx* c, T* x, T* r, const T* p, const T* q, const double* alpha, double* part,
                              int N, int B, const int* run, double* out, const RedOp& op, cudaStream_t s) {
  constexpr int W = Vec16<T>::n;
  if (c->fused_reduce && N % W == 0 && al16(x) && al16(r) && al16(p) && al16(q)) {
    const unsigned nb = nblk((size_t)(N / W));
    const dim3 grid(nb, B);
    unsigned* cnt = LN(c).fin_count;
    if (use_pdl(c, grid))
      KL(c, s, launch_pdl(k_pcg_update_vec<T, R, D, true, OP>, grid, dim3(kThreads), 0, s, x, r, p, q, alpha, part, N,
                          run, cnt, out, op));
    else
      KL(c, s, k_pcg_update_vec<T, R, D, false, OP><<<grid, kThreads, 0, s>>>(x, r, p, q, alpha, part, N, run, cnt,
                                                                              out, op));
    return;
  }
  const unsigned nbu = pcg_update<T, R, D>(c, x, r, p, q, alpha, part, N, B, run, s);
  reduce_op<R, OP>(c, part, nbu, out, op, s);
}

// p = z + beta p
template <typename T, int R, int D>
static void pcg_direction(maple_ctx* c, T* p, const T* z, const double* beta, int N, int B, const int* run,
                          cudaStream_t s) {
  constexpr int W = Vec16<T>::n;
  if (N % W == 0 && al16(p) && al16(z)) {
    const dim3 grid(nblk((size_t)(N / W)), B);
    if (use_pdl(c, grid))
      KL(c, s, launch_pdl(k_pcg_direction_vec<T, R, D, true>, grid, dim3(kThreads), 0, s, p, z, beta, N, run));
    else
      KL(c, s, k_pcg_direction_vec<T, R, D><<<grid, kThreads, 0, s>>>(p, z, beta, N, run));
  } else
    KL(c, s, k_pcg_direction<T, R, D><<<g2(N, B), kThreads, 0, s>>>(p, z, beta, N, run));
}

template <typename T, int D, int R>
static void pcg(maple_ctx* c, Phys& p, Ops<T>& o, const T* b, bool x_zero, double rtol, int maxit,
                const int* outer_run, cudaStream_t s) {
  const int B = c->B, N = nodes(c->n[0]);
  const size_t vbytes = (size_t)B * N * R * D * sizeof(T);
  Scalars& sc = LN(c).sc;
  const unsigned nb = nblk(N);                    // partials of the vector kernels
  const unsigned nbf = (unsigned)fine_tiles(c->n[0]);  // partials of the fine-level operator
  PcgScalars ps{sc.rz, sc.rz_new, sc.pq, sc.rr, sc.bnorm2, sc.alpha, sc.beta, sc.done, sc.cell_done, sc.iters};
  KL(c, s, k_init_flags<<<nblk(B), kThreads, 0, s>>>(c->active, outer_run, sc.done, sc.cell_done, sc.run, sc.iters, B, R));
  const int* run = sc.run;
  // r = b - A x
  if (x_zero) {
    CK(cudaMemsetAsync(o.x, 0, vbytes, s));
    CK(cudaMemcpyAsync(o.r, b, vbytes, cudaMemcpyDeviceToDevice, s));
  } else {
    ApplyArgs<T> a{};
    a.u = o.x;
    a.f = b;
    a.out = o.r;
    apply<T, D, R, M_RES>(c, p, o, 0, a, run, s);
  }
  KL(c, s, k_dot<T, R, D><<<g2(N, B), kThreads, 0, s>>>(b, b, LN(c).part, N, run));
  reduce<R>(c, LN(c).part, nb, sc.bnorm2, s);
  KL(c, s, k_dot<T, R, D><<<g2(N, B), kThreads, 0, s>>>(o.r, o.r, LN(c).part, N, run));
  RedOp op{};
  op.s = ps;
  op.R = R;
  op.breakdown = LN(c).breakdown;
  op.rtol2 = rtol * rtol;
  op.rtol2_dev = sc.rtol2;
  KL(c, s, k_fill<double><<<1, 32, 0, s>>>(sc.rtol2, 1, rtol * rtol));
  op.run = sc.run;
  RedOp op0 = op;  // before the loop: no iteration counted
  reduce_op<R, RED_CHECK>(c, LN(c).part, nb, sc.rr, op0, s);
  if (all_done(c, sc.cell_done, run, s)) return;
  // z = M r ; rz ; p = z
  vcycle<T, D, R>(c, p, o, 0, o.r, run, LN(c).part, s);
  reduce_op<R, RED_SET_RZ>(c, LN(c).part, nbf, sc.rz_new, op, s);
  CK(cudaMemcpyAsync(o.p, o.U[0][1], vbytes, cudaMemcpyDeviceToDevice, s));
  op.count = 1;
  auto body = [&](cudaStream_t st) {
    {
      ApplyArgs<T> a{};
      a.u = o.p;
      a.out = o.q;
      a.part = LN(c).part;
      apply<T, D, R, M_MV>(c, p, o, 0, a, run, st);
    }
    reduce_op<R, RED_ALPHA>(c, LN(c).part, nbf, sc.pq, op, st);
    pcg_update_reduce<T, R, D, RED_CHECK>(c, o.x, o.r, o.p, o.q, sc.alpha, LN(c).part, N, B, run, sc.rr, op, st);
    vcycle<T, D, R>(c, p, o, 0, o.r, run, LN(c).part, st);
    reduce_op<R, RED_BETA>(c, LN(c).part, nbf, sc.rz_new, op, st);
    pcg_direction<T, R, D>(c, o.p, o.U[0][1], sc.beta, N, B, run, st);
  };
  run_iterations(c, c->graphs[&p == &c->ph[0] ? 0 : 1][std::is_same<T, float>::value ? 2 : MAPLE_FP64], maxit,
                 body, s);
}

// ---------------------------------------------------------------------------
// Mixed precision: FP64 flexible PCG (FP64 fine operator, residuals and dots)
// preconditioned by the FP32 V-cycle; the coarsest solve stays FP64.
// ---------------------------------------------------------------------------
// z = M r with the column scales of r already in place (set by the fused
// convergence check), then r.z, q.z and the flexible beta in one reduction
template <int D, int R>
static void precondition_f32(maple_ctx* c, Phys& p, const double* r, const double* q, const int* run,
                             const RedOp& op, cudaStream_t s) {
  const int B = c->B, N = nodes(c->n[0]);
  Ops<float>& o = p.o32;
  KL(c, s, k_to_f32_scaled<R, D><<<g2(N, B), kThreads, 0, s>>>(r, o.r, LN(c).o_scale, N, run));
  vcycle<float, D, R>(c, p, o, 0, o.r, run, nullptr, s);
  KL(c, s, k_precond_back<R, D><<<g2(N, B), kThreads, 0, s>>>(o.U[0][1], LN(c).o_inv, r, q, LN(c).part, N, run));
  reduce_op<2 * R, RED_BETA_FLEX>(c, LN(c).part, nblk(N), LN(c).red, op, s);
}

template <int D, int R>
static void pcg_mixed(maple_ctx* c, Phys& p, const double* b, double* x, bool x_zero, double rtol, int maxit,
                      cudaStream_t s, const int* mask = nullptr) {
  const int B = c->B, N = nodes(c->n[0]);
  const size_t vbytes = (size_t)B * N * R * D * sizeof(double);
  Scalars& sc = LN(c).sc;
  const unsigned nb = nblk(N), nbf = (unsigned)fine_tiles(c->n[0]);
  PcgScalars ps{sc.rz, sc.rz_new, sc.pq, sc.rr, sc.bnorm2, sc.alpha, sc.beta, sc.done, sc.cell_done, sc.iters};
  Ops<double>& o64 = p.o64;
  double *r = p.r64, *pv = p.p64, *q = p.q64;
  const float* z32 = p.o32.U[0][1];  // preconditioner output; z = ||r|| z32 is formed where it is used
  KL(c, s, k_init_flags<<<nblk(B), kThreads, 0, s>>>(c->active, mask, sc.done, sc.cell_done, sc.run, sc.iters, B, R));
  const int* run = sc.run;
  if (x_zero) {
    CK(cudaMemsetAsync(x, 0, vbytes, s));
    CK(cudaMemcpyAsync(r, b, vbytes, cudaMemcpyDeviceToDevice, s));
  } else {
    ApplyArgs<double> a{};
    a.u = x;
    a.f = b;
    a.out = r;
    apply<double, D, R, M_RES>(c, p, o64, 0, a, run, s);
  }
  KL(c, s, k_dot<double, R, D><<<g2(N, B), kThreads, 0, s>>>(b, b, LN(c).part, N, run));
  reduce<R>(c, LN(c).part, nb, sc.bnorm2, s);
  KL(c, s, k_dot<double, R, D><<<g2(N, B), kThreads, 0, s>>>(r, r, LN(c).part, N, run));
  RedOp op{};
  op.s = ps;
  op.R = R;
  op.breakdown = LN(c).breakdown;
  op.rtol2 = rtol * rtol;
  op.rtol2_dev = sc.rtol2;
  KL(c, s, k_fill<double><<<1, 32, 0, s>>>(sc.rtol2, 1, rtol * rtol));
  op.run = sc.run;
  op.scale = LN(c).o_scale;
  op.inv = LN(c).o_inv;
  RedOp op0 = op;  // before the loop: no iteration counted, first flexible beta
  op0.first = 1;
  reduce_op<R, RED_CHECK>(c, LN(c).part, nb, sc.rr, op0, s);
  if (all_done(c, sc.cell_done, run, s)) return;
  precondition_f32<D, R>(c, p, r, nullptr, run, op0, s);
  KL(c, s, k_pcg_direction_f32<R, D, true><<<g2(N, B), kThreads, 0, s>>>(pv, z32, LN(c).o_inv, nullptr, N, run));
  op.count = 1;
  auto body = [&](cudaStream_t st) {
    {
      ApplyArgs<double> a{};
      a.u = pv;
      a.out = q;
      a.part = LN(c).part;
      apply<double, D, R, M_MV>(c, p, o64, 0, a, run, st);
    }
    reduce_op<R, RED_ALPHA>(c, LN(c).part, nbf, sc.pq, op, st);
    pcg_update_reduce<double, R, D, RED_CHECK>(c, x, r, pv, q, sc.alpha, LN(c).part, N, B, run, sc.rr, op, st);
    precondition_f32<D, R>(c, p, r, q, run, op, st);
    KL(c, st, k_pcg_direction_f32<R, D, false><<<g2(N, B), kThreads, 0, st>>>(pv, z32, LN(c).o_inv, sc.beta, N, run));
  };
  run_iterations(c, c->graphs[&p == &c->ph[0] ? 0 : 1][MAPLE_MIXED], maxit, body, s);
}

// ---------------------------------------------------------------------------
// Mixed precision, reliable-update form: the whole PCG iteration in FP32 (FP32
// fine operator, FP32 vectors, FP64-accumulated dots) on the residual scaled
// to unit norm, with the FP64 iterate and residual replaced from time to time
// instead of restarting.  A cell is flagged when a live column's recurrence
// residual fell by delta since the last replacement, or passes the tolerance
// test; its FP32 correction is folded into the FP64 iterate, the residual
// b - A x is computed in FP64, tested (only this test marks a column
// converged), scaled to unit norm and continues the iteration with the same
// (rescaled) direction, so the Krylov space is kept.
// ---------------------------------------------------------------------------
constexpr int MIXED_RELIABLE_GRAPH = 3;

template <int D, int R>
static void pcg_reliable(maple_ctx* c, Phys& p, const double* b, double* x, bool x_zero, double rtol, int maxit,
                         cudaStream_t s) {
  const int B = c->B, N = nodes(c->n[0]);
  const size_t vbytes = (size_t)B * N * R * D * sizeof(double), v32 = (size_t)B * N * R * D * sizeof(float);
  Lane& ln = LN(c);
  Scalars& sc = ln.sc;
  const unsigned nb = nblk(N), nbf = (unsigned)fine_tiles(c->n[0]);
  PcgScalars ps{sc.rz, sc.rz_new, sc.pq, sc.rr, sc.bnorm2, sc.alpha, sc.beta, sc.done, sc.cell_done, sc.iters};
  Ops<double>& o64 = p.o64;
  Ops<float>& o = p.o32;
  double* r = p.r64;
  const float* z = o.U[0][1];  // preconditioner output
  KL(c, s, k_init_flags<<<nblk(B), kThreads, 0, s>>>(c->active, nullptr, sc.done, sc.cell_done, sc.run, sc.iters, B, R));
  const int* run = sc.run;
  if (x_zero) {
    CK(cudaMemsetAsync(x, 0, vbytes, s));
    CK(cudaMemcpyAsync(r, b, vbytes, cudaMemcpyDeviceToDevice, s));
  } else {
    ApplyArgs<double> a{};
    a.u = x;
    a.f = b;
    a.out = r;
    apply<double, D, R, M_RES>(c, p, o64, 0, a, run, s);
  }
  KL(c, s, k_dot<double, R, D><<<g2(N, B), kThreads, 0, s>>>(b, b, ln.part, N, run));
  reduce<R>(c, ln.part, nb, sc.bnorm2, s);
  KL(c, s, k_dot<double, R, D><<<g2(N, B), kThreads, 0, s>>>(r, r, ln.part, N, run));
  RedOp op{};
  op.s = ps;
  op.R = R;
  op.breakdown = ln.breakdown;
  op.rtol2 = rtol * rtol;
  op.rtol2_dev = sc.rtol2;
  KL(c, s, k_fill<double><<<1, 32, 0, s>>>(sc.rtol2, 1, rtol * rtol));
  op.run = sc.run;
  op.scale = ln.o_scale;
  op.inv = ln.o_inv;
  op.rel = ln.rel;
  op.t = ln.o_t;
  op.delta2 = c->rel_delta * c->rel_delta;
  RedOp op0 = op;  // before the loop: no iteration counted; column scales of the first residual
  reduce_op<R, RED_CHECK>(c, ln.part, nb, sc.rr, op0, s);
  if (all_done(c, sc.cell_done, run, s)) return;
  CK(cudaMemsetAsync(o.x, 0, v32, s));
  CK(cudaMemsetAsync(ln.loop + 2, 0, sizeof(int), s));  // IF-node executions of this solve
  KL(c, s, k_to_f32_scaled<R, D><<<g2(N, B), kThreads, 0, s>>>(r, o.r, ln.o_scale, N, run));
  vcycle<float, D, R>(c, p, o, 0, o.r, run, ln.part, s);
  reduce_op<R, RED_SET_RZ>(c, ln.part, nbf, sc.rz_new, op, s);
  CK(cudaMemcpyAsync(o.p, z, v32, cudaMemcpyDeviceToDevice, s));
  op.count = 1;
  auto body = [&](cudaStream_t st) {
    // In a captured graph the residual replacement below sits in a
    // conditional IF node (handle h), so iterations without one launch none
    // of it; ALPHA clears the condition, RELCHECK sets it.
    cudaGraphConditionalHandle h = 0;
    cudaGraph_t cg = nullptr;
    if (c->device_loop) {
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      if (cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg) != cudaSuccess || cs != cudaStreamCaptureStatusActive ||
          cudaGraphConditionalHandleCreate(&h, cg, 0, cudaGraphCondAssignDefault) != cudaSuccess)
        h = 0;
      (void)cudaGetLastError();
    }
    RedOp opc = op;
    opc.cond = h;
    {
      ApplyArgs<float> a{};
      a.u = o.p;
      a.out = o.q;
      a.part = ln.part;
      apply<float, D, R, M_MV>(c, p, o, 0, a, run, st);
    }
    reduce_op<R, RED_ALPHA>(c, ln.part, nbf, sc.pq, opc, st);
    pcg_update_reduce<float, R, D, RED_RELCHECK>(c, o.x, o.r, o.p, o.q, sc.alpha, ln.part, N, B, run, sc.rr, opc, st);
    // residual replacement of the flagged cells (every launch skips the others)
    auto replace = [&](cudaStream_t sr, bool in_if) {
      KL(c, sr, k_flush_f32<R, D><<<g2(N, B), kThreads, 0, sr>>>(x, o.x, ln.o_inv, N, ln.rel));
      ApplyArgs<double> a{};
      a.u = x;
      a.f = b;
      a.out = r;
      apply<double, D, R, M_RES>(c, p, o64, 0, a, ln.rel, sr);
      KL(c, sr, k_dot<double, R, D><<<g2(N, B), kThreads, 0, sr>>>(r, r, ln.part, N, ln.rel));
      RedOp ops = op;
      if (in_if) ops.cond_count = ln.loop + 2;  // launches of the IF body are counted by executions
      reduce_op<R, RED_RELSET>(c, ln.part, nb, ln.o_rr, ops, sr);
      KL(c, sr, k_rel_rescale<R, D><<<g2(N, B), kThreads, 0, sr>>>(r, o.r, o.p, o.q, ln.o_scale, ln.o_t, N, ln.rel));
    };
    bool nested = false;
    if (h) {
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      const cudaGraphNode_t* deps = nullptr;
      size_t nd = 0;
      cudaGraphNodeParams np{};
      np.type = cudaGraphNodeTypeConditional;
      np.conditional.handle = h;
      np.conditional.type = cudaGraphCondTypeIf;
      np.conditional.size = 1;
      cudaGraphNode_t node{};
      if (!ln.cap_stream2) CK(cudaStreamCreateWithFlags(&ln.cap_stream2, cudaStreamNonBlocking));
      // the capture of st goes on after the IF node; its body is captured on
      // the second stream
      nested = cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, &deps, &nd) == cudaSuccess &&
               cudaGraphAddNode(&node, cg, deps, nd, &np) == cudaSuccess &&
               cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies) == cudaSuccess &&
               cudaStreamBeginCaptureToGraph(ln.cap_stream2, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                             cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      (void)cudaGetLastError();
      if (nested) {
        const unsigned long long before = tl_launches;
        try {
          replace(ln.cap_stream2, true);
          tl_cond_kernels += tl_launches - before;
        } catch (...) {
          cudaGraph_t tmp = nullptr;
          cudaStreamEndCapture(ln.cap_stream2, &tmp);
          throw;
        }
        cudaGraph_t tmp = nullptr;
        CK(cudaStreamEndCapture(ln.cap_stream2, &tmp));
      }
    }
    // without the IF node (eager, or refused: an IF node left with an empty
    // body does nothing) the predicated launches run in line
    if (!nested) replace(st, false);
    // z = M r, r.z fused into the last smoothing step; p = z + beta p
    vcycle<float, D, R>(c, p, o, 0, o.r, run, ln.part, st);
    reduce_op<R, RED_BETA>(c, ln.part, nbf, sc.rz_new, op, st);
    pcg_direction<float, R, D>(c, o.p, z, sc.beta, N, B, run, st);
  };
  maple_ctx::GraphEntry& ge = c->graphs[&p == &c->ph[0] ? 0 : 1][MIXED_RELIABLE_GRAPH];
  run_iterations(c, ge, maxit, body, s);
  // cells stopped by the iteration limit keep their last FP32 correction
  KL(c, s, k_flush_f32<R, D><<<g2(N, B), kThreads, 0, s>>>(x, o.x, ln.o_inv, N, c->active));
  if (ge.cond_kernels) {  // launches of the replacements that ran inside graphs
    CK(cudaMemcpyAsync(ln.h_flags + B + 1, ln.loop + 2, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const unsigned long long n = (unsigned long long)std::max(ln.h_flags[B + 1], 0) * ge.cond_kernels;
    g_launches.fetch_add(n);
    tl_launches += n;
  }
}

// Extrapolated warm start of an OC step: u <- u + theta (u - prev), prev <- u
// (the solution this step starts from becomes the next step's "previous");
// with theta = 0 only prev <- u.  Cells with active[b] == 0 are skipped.
__global__ void k_extrapolate(double* __restrict__ u, double* __restrict__ prev, double theta, size_t len,
                              const int* active) {
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  double* ub = u + (size_t)b * len;
  double* pb = prev + (size_t)b * len;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (size_t)gridDim.x * blockDim.x) {
    const double uv = ub[i];
    if (theta != 0.0) ub[i] = fma(theta, uv - pb[i], uv);
    pb[i] = uv;
  }
}

// outer refinement bookkeeping: per (cell, rhs) residual scale and cell done
__global__ void k_outer_check(const double* rr, const double* bn, double rtol2, double* scale, double* inv, int* done,
                              int* run, const int* active, int B, int R) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  if (active && !active[b]) {
    done[b] = 1;
    run[b] = 0;
    return;
  }
  int all = 1;
  for (int r = 0; r < R; ++r) {
    const double v = rr[b * R + r];
    all &= (v <= rtol2 * bn[b * R + r]);
    const double nrm = sqrt(v);
    scale[b * R + r] = nrm > 0 ? 1.0 / nrm : 0.0;
    inv[b * R + r] = nrm;
  }
  done[b] = all;
  run[b] = !all;
}

// ---------------------------------------------------------------------------
// Mixed precision, refinement form: FP32 MG-PCG (FP32 fine operator, FP32
// vectors, FP64-accumulated dots) on the scaled FP64 residual, inside FP64
// iterative refinement.  Per outer pass: r = b - A x in FP64, convergence test
// ||r|| <= rtol ||b|| per load case, the inner FP32 solve of A e = r/||r|| to
// the inner tolerance (tightened in the last pass to what the tolerance still
// needs), then x += ||r|| e in FP64.  FP64 work per pass is one fine-level
// residual and the vector updates; all per-iteration work is FP32.
// ---------------------------------------------------------------------------
constexpr int kMaxOuter = 12;

template <int D, int R>
static void pcg_refine(maple_ctx* c, Phys& p, const double* b, double* x, bool x_zero, double rtol, int maxit,
                       std::vector<int>& iters, std::vector<int>& status, cudaStream_t s) {
  const int B = c->B, N = nodes(c->n[0]);
  const size_t vbytes = (size_t)B * N * R * D * sizeof(double);
  Lane& ln = LN(c);
  Ops<double>& o64 = p.o64;
  Ops<float>& o32 = p.o32;
  double* r = p.r64;
  const unsigned nb = nblk(N);
  iters.assign(B, 0);
  status.assign(B, MAPLE_CELL_MAXIT);
  std::vector<int> broken(B, 0), act(B, 1), done(B, 0), it_in(B), dn((size_t)B * R);
  std::vector<double> rr((size_t)B * R), bn((size_t)B * R);
  for (int b = 0; b < B; ++b) {
    act[b] = c->h_active.empty() || c->h_active[b];
    if (!act[b]) status[b] = MAPLE_CELL_CONVERGED;  // as read_outcome reports skipped cells
  }
  // cells still refined: active and not broken down (uploaded when it changes)
  int* live = ln.o_live;
  CK(cudaMemcpyAsync(live, act.data(), B * sizeof(int), cudaMemcpyHostToDevice, s));
  if (x_zero) {
    CK(cudaMemsetAsync(x, 0, vbytes, s));
    CK(cudaMemcpyAsync(r, b, vbytes, cudaMemcpyDeviceToDevice, s));
  } else {
    ApplyArgs<double> a{};
    a.u = x;
    a.f = b;
    a.out = r;
    apply<double, D, R, M_RES>(c, p, o64, 0, a, c->active, s);
  }
  KL(c, s, k_dot<double, R, D><<<g2(N, B), kThreads, 0, s>>>(b, b, ln.part, N, c->active));
  reduce<R>(c, ln.part, nb, ln.o_bn, s);
  CK(cudaMemcpyAsync(bn.data(), ln.o_bn, (size_t)B * R * sizeof(double), cudaMemcpyDeviceToHost, s));
  int used = 0;
  for (int outer = 0;; ++outer) {
    KL(c, s, k_dot<double, R, D><<<g2(N, B), kThreads, 0, s>>>(r, r, ln.part, N, live));
    reduce<R>(c, ln.part, nb, ln.o_rr, s);
    KL(c, s, k_outer_check<<<nblk(B), kThreads, 0, s>>>(ln.o_rr, ln.o_bn, rtol * rtol, ln.o_scale, ln.o_inv,
                                                        ln.o_done, ln.o_run, live, B, R));
    CK(cudaMemcpyAsync(rr.data(), ln.o_rr, (size_t)B * R * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(done.data(), ln.o_done, B * sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    // the inner tolerance: the default, or looser when every unfinished load
    // case needs less (0.5 x the reduction that reaches rtol)
    double need = 1.0;
    bool any = false;
    for (int b = 0; b < B; ++b) {
      if (!act[b] || broken[b]) continue;
      if (done[b]) {
        status[b] = MAPLE_CELL_CONVERGED;
        continue;
      }
      any = true;
      for (int k = 0; k < R; ++k) {
        const double v = rr[(size_t)b * R + k];
        if (v > rtol * rtol * bn[(size_t)b * R + k] && v > 0) need = std::min(need, rtol * std::sqrt(bn[(size_t)b * R + k] / v));
      }
    }
    if (!any || used >= maxit || outer >= kMaxOuter) break;
    const double tol = std::max(c->inner_rtol, 0.5 * need);
    KL(c, s, k_to_f32_scaled<R, D><<<g2(N, B), kThreads, 0, s>>>(r, p.b32, ln.o_scale, N, ln.o_run));
    pcg<float, D, R>(c, p, o32, p.b32, true, tol, maxit - used, ln.o_run, s);
    CK(cudaMemcpyAsync(it_in.data(), ln.sc.iters, B * sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(dn.data(), ln.sc.done, (size_t)B * R * sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    bool newly_broken = false;
    int most = 0;
    for (int b = 0; b < B; ++b) {
      if (!act[b] || broken[b] || done[b]) continue;
      iters[b] += it_in[b];
      most = std::max(most, it_in[b]);
      for (int k = 0; k < R; ++k)
        if (dn[(size_t)b * R + k] == 2) {
          broken[b] = 1;
          status[b] = MAPLE_CELL_BREAKDOWN;
          newly_broken = true;
        }
    }
    used += std::max(most, 1);
    if (newly_broken) {
      std::vector<int> lv(B);
      for (int b = 0; b < B; ++b) lv[b] = act[b] && !broken[b];
      CK(cudaMemcpyAsync(live, lv.data(), B * sizeof(int), cudaMemcpyHostToDevice, s));
      CK(cudaMemcpyAsync(ln.o_run, lv.data(), B * sizeof(int), cudaMemcpyHostToDevice, s));
      // lv is read by the copies above before it goes out of scope
      CK(cudaStreamSynchronize(s));
    }
    // x += ||r|| e ; r = b - A x (FP64)
    KL(c, s, k_add_f32_scaled<R, D><<<g2(N, B), kThreads, 0, s>>>(x, o32.x, ln.o_inv, N, ln.o_run));
    ApplyArgs<double> a{};
    a.u = x;
    a.f = b;
    a.out = r;
    apply<double, D, R, M_RES>(c, p, o64, 0, a, ln.o_run, s);
  }
}

static void ensure_prec(maple_ctx* c, int phys, int prec);

// per-cell outcome of the last PCG run of this lane: BREAKDOWN when a column was
// frozen by a breakdown (p.Ap <= 0 or non-finite), else CONVERGED or MAXIT
static void read_outcome(maple_ctx* c, int R, std::vector<int>& iters, std::vector<int>& status, cudaStream_t s) {
  const int B = c->B;
  std::vector<int> cd(B), dn((size_t)B * R);
  iters.assign(B, 0);
  status.assign(B, 0);
  CK(cudaMemcpyAsync(iters.data(), LN(c).sc.iters, B * sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(cd.data(), LN(c).sc.cell_done, B * sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(dn.data(), LN(c).sc.done, (size_t)B * R * sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  for (int b = 0; b < B; ++b) {
    bool brk = false;
    for (int r = 0; r < R; ++r) brk |= dn[(size_t)b * R + r] == 2;
    status[b] = brk ? MAPLE_CELL_BREAKDOWN : (cd[b] ? MAPLE_CELL_CONVERGED : MAPLE_CELL_MAXIT);
  }
}

// flags[b] = 1 if cell b of x (B cells of len values) holds a non-finite value
__global__ void k_nonfinite_cells(const double* __restrict__ x, size_t len, const int* mask, int* flags) {
  const int b = blockIdx.y;
  if (mask && !mask[b]) return;
  const double* xb = x + (size_t)b * len;
  bool bad = false;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (size_t)gridDim.x * blockDim.x)
    bad |= !isfinite(xb[i]);
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flags + b, 1);
}

template <int D, int R>
static void solve_phys(maple_ctx* c, int phys, int prec, const double* F, double* x64, bool x_zero, double rtol,
                       int maxit, int* iters_host, int* status_host, cudaStream_t s) {
  Range range(D == 3 ? (prec == MAPLE_FP64 ? "maple:solve elastic fp64" : "maple:solve elastic mixed")
                     : (prec == MAPLE_FP64 ? "maple:solve thermal fp64" : "maple:solve thermal mixed"));
  Phys& p = c->ph[phys];
  const int B = c->B, N = nodes(c->n[0]);
  const size_t vb64 = (size_t)B * N * R * D * sizeof(double), cell_len = (size_t)N * R * D;
  std::vector<int> it, st;
  if (prec == MAPLE_FP64) {
    Ops<double>& o = p.o64;
    if (!x_zero) CK(cudaMemcpyAsync(o.x, x64, vb64, cudaMemcpyDeviceToDevice, s));
    pcg<double, D, R>(c, p, o, F, x_zero, rtol, maxit, nullptr, s);
    CK(cudaMemcpyAsync(x64, o.x, vb64, cudaMemcpyDeviceToDevice, s));
    read_outcome(c, R, it, st, s);
  } else {
    if (c->mixed_mode == MAPLE_MIXED_REFINE) {
      pcg_refine<D, R>(c, p, F, x64, x_zero, rtol, maxit, it, st, s);
    } else if (c->mixed_mode == MAPLE_MIXED_RELIABLE) {
      // FP32 recurrences lose orthogonality on badly conditioned cells (near
      // void, floating stiff islands), where the flexible form, with FP64
      // recurrences, still converges: a cell still unconverged after
      // rel_handover iterations continues in the flexible form from its
      // iterate, within the same iteration limit.
      const int cap = std::min(maxit, c->rel_handover);
      pcg_reliable<D, R>(c, p, F, x64, x_zero, rtol, cap, s);
      read_outcome(c, R, it, st, s);
      if (cap < maxit) {
        std::vector<int> ho(B, 0);
        bool any = false;
        for (int b = 0; b < B; ++b)
          if (st[b] == MAPLE_CELL_MAXIT && (c->h_active.empty() || c->h_active[b])) ho[b] = 1, any = true;
        if (any) {
          Lane& ln = LN(c);
          CK(cudaMemcpyAsync(ln.o_live, ho.data(), B * sizeof(int), cudaMemcpyHostToDevice, s));
          pcg_mixed<D, R>(c, p, F, x64, false, rtol, maxit - cap, s, ln.o_live);
          std::vector<int> it2, st2;
          read_outcome(c, R, it2, st2, s);  // synchronises: ho is read before it goes out of scope
          for (int b = 0; b < B; ++b)
            if (ho[b]) {
              it[b] += it2[b];
              st[b] = st2[b];
            }
        }
      }
    } else {
      pcg_mixed<D, R>(c, p, F, x64, x_zero, rtol, maxit, s);
      read_outcome(c, R, it, st, s);
    }
    // Fallback: a cell whose mixed-precision solve broke down is solved again
    // in plain FP64 MG-PCG (FP64 hierarchy built for those cells only) from its
    // last iterate, or from zero when that iterate is not finite or when the
    // FP64 solve from it breaks down too.  The other
    // cells and the FP32 hierarchy are untouched; the second host thread of
    // an OC step never sees this lane's masks.
    std::vector<int> fb(B, 0);
    bool any = false;
    for (int b = 0; b < B; ++b)
      if (st[b] == MAPLE_CELL_BREAKDOWN && (c->h_active.empty() || c->h_active[b])) fb[b] = 1, any = true;
    if (any) {
      Lane& ln = LN(c);
      if (!ln.fb_mask) {
        ln.fb_mask = dnew<int>(c, B);
        ln.fb_bad = dnew<int>(c, B);
      }
      CK(cudaMemcpyAsync(ln.fb_mask, fb.data(), B * sizeof(int), cudaMemcpyHostToDevice, s));
      CK(cudaMemsetAsync(ln.fb_bad, 0, B * sizeof(int), s));
      KL(c, s, k_nonfinite_cells<<<dim3(64, B), kThreads, 0, s>>>(x64, cell_len, ln.fb_mask, ln.fb_bad));
      std::vector<int> bad(B, 0);
      CK(cudaMemcpyAsync(bad.data(), ln.fb_bad, B * sizeof(int), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      ensure_prec(c, phys, MAPLE_FP64);
      build_hierarchy<D>(c, phys, MAPLE_FP64, s, ln.fb_mask);
      Ops<double>& o = p.o64;
      for (int b = 0; b < B; ++b) {
        if (!fb[b]) continue;
        double* xo = o.x + (size_t)b * cell_len;
        if (bad[b])
          CK(cudaMemsetAsync(xo, 0, cell_len * sizeof(double), s));
        else
          CK(cudaMemcpyAsync(xo, x64 + (size_t)b * cell_len, cell_len * sizeof(double), cudaMemcpyDeviceToDevice, s));
      }
      std::vector<int> it2, st2;
      // attempt 1 from the last iterate; attempt 2 from zero for the cells whose
      // last iterate led into a breakdown again (e.g. a finite but wild guess,
      // whose size puts the tolerance beyond reach)
      for (int attempt = 0; attempt < 2 && any; ++attempt) {
        if (attempt == 1) {
          any = false;
          for (int b = 0; b < B; ++b) {
            fb[b] = fb[b] && st2[b] == MAPLE_CELL_BREAKDOWN && !bad[b];
            if (fb[b]) {
              any = true;
              CK(cudaMemsetAsync(o.x + (size_t)b * cell_len, 0, cell_len * sizeof(double), s));
            }
          }
          if (!any) break;
          CK(cudaMemcpyAsync(ln.fb_mask, fb.data(), B * sizeof(int), cudaMemcpyHostToDevice, s));
        }
        pcg<double, D, R>(c, p, o, F, false, rtol, maxit, ln.fb_mask, s);
        for (int b = 0; b < B; ++b)
          if (fb[b])
            CK(cudaMemcpyAsync(x64 + (size_t)b * cell_len, o.x + (size_t)b * cell_len, cell_len * sizeof(double),
                               cudaMemcpyDeviceToDevice, s));
        read_outcome(c, R, it2, st2, s);
        for (int b = 0; b < B; ++b)
          if (fb[b]) {
            it[b] += it2[b];
            st[b] = st2[b] | MAPLE_CELL_FALLBACK;
          }
      }
      p.built_prec = MAPLE_MIXED;  // the FP32 hierarchy still serves the next mixed solves
    }
  }
  for (int b = 0; b < B; ++b) {
    if (iters_host) iters_host[b] = it[b];
    if (status_host) status_host[b] = st[b];
  }
}

static void dispatch_solve(maple_ctx* c, int phys, int prec, const double* F, double* x64, bool x_zero, double rtol,
                           int maxit, int* iters, int* status, cudaStream_t s) {
  if (phys == MAPLE_ELASTIC)
    solve_phys<3, 6>(c, phys, prec, F, x64, x_zero, rtol, maxit, iters, status, s);
  else
    solve_phys<1, 3>(c, phys, prec, F, x64, x_zero, rtol, maxit, iters, status, s);
}

static void ensure_prec(maple_ctx* c, int phys, int prec) {
  Phys& p = c->ph[phys];
  alloc_phys(c, phys);
  alloc_ops<double>(c, p, p.o64, prec == MAPLE_FP64);
  if (prec == MAPLE_MIXED) {
    alloc_ops<float>(c, p, p.o32, true);
    if (!p.p64) {
      const size_t n = (size_t)c->B * nodes(c->n[0]) * p.R * p.D;
      p.p64 = dnew<double>(c, n);
      p.q64 = dnew<double>(c, n);
      p.b32 = dnew<float>(c, n);
    }
  }
}

static void load_density(maple_ctx* c, int phys, const double* rho, int prec, cudaStream_t s) {
  Phys& p = c->ph[phys];
  const size_t tot = (size_t)c->B * nodes(c->n[0]);
  KL(c, s, k_copy_rho<<<nblk(tot), kThreads, 0, s>>>(rho, p.o64.rho, prec == MAPLE_MIXED ? p.o32.rho : nullptr, tot));
}

static void build(maple_ctx* c, int phys, int prec, cudaStream_t s) {
  if (phys == MAPLE_ELASTIC)
    build_hierarchy<3>(c, phys, prec, s);
  else
    build_hierarchy<1>(c, phys, prec, s);
}

static void assemble_rhs(maple_ctx* c, int phys, const double* rho, double* F, cudaStream_t s) {
  Phys& p = c->ph[phys];
  const int N = nodes(c->n[0]);
  if (phys == MAPLE_ELASTIC)
    KL(c, s, k_assemble_F<3, 6><<<g2(N, c->B), kThreads, 0, s>>>(rho, F, c->n[0], p.fscale, c->active));
  else
    KL(c, s, k_assemble_F<1, 3><<<g2(N, c->B), kThreads, 0, s>>>(rho, F, c->n[0], p.fscale, c->active));
}

static void homogenize(maple_ctx* c, int phys, cudaStream_t s) {
  Range range("maple:homogenize");
  Phys& p = c->ph[phys];
  const int N = nodes(c->n[0]);
  const unsigned nb = nblk(N);
  if (phys == MAPLE_ELASTIC) {
    const unsigned nbe = (unsigned)ceil_div(N, 32 * kHomGroups);
    KL(c, s, k_homogenize_elastic<<<dim3(nbe, c->B), 32 * kHomWarps, 0, s>>>(p.u64, p.o64.rho, p.energy, LN(c).part,
                                                                            c->n[0], p.kscale, p.xscale, c->active));
    reduce<21>(c, LN(c).part, nbe, LN(c).red, s);
    KL(c, s, k_unpack_sym<<<nblk(c->B), kThreads, 0, s>>>(LN(c).red, p.H, c->B, 6));
  } else {
    KL(c, s, k_homogenize<1, 3><<<g2(N, c->B), kThreads, 0, s>>>(p.u64, p.o64.rho, p.energy, LN(c).part, c->n[0], p.kscale,
                                                        p.xscale, c->active));
    reduce<6>(c, LN(c).part, nb, LN(c).red, s);
    KL(c, s, k_unpack_sym<<<nblk(c->B), kThreads, 0, s>>>(LN(c).red, p.H, c->B, 3));
  }
  p.energies = true;
}

// Poll limit and phantom block count of the OC kernel's grid barriers for
// launches from this thread (maple_test_wait_limit); the defaults are the
// normal bound and no phantom blocks.
static thread_local long long tl_wait_polls = kBarrierPolls;
static thread_local unsigned tl_wait_phantom = 0;

// The context's OC update resolves four bisection steps per grid barrier
// (k_oc_update_tree: lambda and x as k_oc_update to rounding, 16 barriers instead
// of 61); the allocation-free entry point keeps k_oc_update and its scratch
// layout.
constexpr int kOcLevels = 4;
constexpr int kOcPartPerBlock = 2 * ((1 << kOcLevels) - 1) + 2;  // doubles per (cell, block)
constexpr int kOcCacheElems = 2048;                                 // elements per block cached in shared memory
constexpr size_t kOcCacheBytes = (size_t)3 * kOcCacheElems * sizeof(double);

static void oc_update(maple_ctx* c, const double* x, const double* dJ, const double* vf, double move, double xmin,
                      double* xnew, double* stats, cudaStream_t s) {
  const int N = nodes(c->n[0]);
  int per_sm = 0, sms = 0;
  smem_attr(k_oc_update_tree<kOcLevels>, kOcCacheBytes, c->dev);
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_oc_update_tree<kOcLevels>, kThreads, kOcCacheBytes));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->dev));
  const int maxres = per_sm * sms;
  require(maxres >= 1, "OC kernel cannot be resident");
  // cells per launch and blocks per cell
  const int want_G = std::max(1, std::min(sms, (N + 4 * kThreads - 1) / (4 * kThreads)));
  int cells_per_launch = std::max(1, std::min(c->B, maxres / want_G));
  // cleared once per update: a launch that finds it set (an earlier launch's
  // barrier gave up) returns at its first barrier
  CK(cudaMemsetAsync(c->err, 0, sizeof(int), s));
  for (int c0 = 0; c0 < c->B; c0 += cells_per_launch) {
    const int nb = std::min(cells_per_launch, c->B - c0);
    const int G = std::max(1, std::min({want_G, maxres / nb, kOcMaxG}));
    OcArgs a{};
    a.x = x + (size_t)c0 * N;
    a.dJ = dJ + (size_t)c0 * N;
    a.xnew = xnew + (size_t)c0 * N;
    a.volfrac = vf + c0;
    a.move = move;
    a.xmin = xmin;
    a.N = N;
    a.part = c->ocpart;
    a.stats = stats ? stats + 2 * c0 : c->stats + 2 * c0;
    a.lam_out = nullptr;
    a.bar = c->bar;
    a.err = c->err;
    a.active = c->active ? c->active + c0 : nullptr;
    a.poll_limit = tl_wait_polls;
    a.phantom = tl_wait_phantom;
    a.cache_chunk = kOcCacheElems;
    CK(cudaMemsetAsync(c->bar, 0, 2 * sizeof(unsigned), s));
    void* args[] = {&a};
    prof_begin(c, s);
    CK(cudaLaunchCooperativeKernel((void*)k_oc_update_tree<kOcLevels>, dim3(G, nb), dim3(kThreads), args,
                                   kOcCacheBytes, s));
    g_launches.fetch_add(1);
    prof_end(c, s, "k_oc_update", 0);
  }
}

// Waits for the stream and raises MAPLE_E_TIMEOUT if a grid barrier of the
// last oc_update gave up (its outputs are then incomplete).
static void check_oc_barrier(maple_ctx* c, cudaStream_t s) {
  CK(cudaMemcpyAsync(c->h_err, c->err, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (*c->h_err)
    throw Failure{MAPLE_E_TIMEOUT, "OC update: a grid barrier wait ran out (not every block of the cooperative "
                                   "launch arrived); x_next and the statistics are incomplete"};
}

// ---------------------------------------------------------------------------
// Allocation-free OC update.
//
// Some host applications own every byte of device memory through their own
// allocator and do not let a library call cudaMalloc (which also synchronises
// the whole device and so stalls their other streams).  For them the OC
// bisection kernel can run with its scratch (per-block partial sums, per-cell
// |dx| statistics when the caller passes none, and the grid-barrier counters)
// in one fixed, file-scope device array instead of context workspace.
//
// * The array is 256 KiB (kNoAllocScratch doubles) and every GPU that loads
//   this library holds it until the process exits.
// * Host code cannot use the array's name as a device address: its address is
//   fetched once per device with cudaGetSymbolAddress.  The first call on a
//   device does that set-up, so make that first call before any stream capture.
// * All calls share the array and it keeps the last call's contents; the
//   barrier counters are cleared at the start of every call.  Calls whose
//   kernels overlap on the GPU (for example on two streams) race on it.
// ---------------------------------------------------------------------------
// J = J_raw - lp P_print - lc P_cavity per cell
__global__ void k_penalise_J(double* J, const double* Pp, double lp, const double* Pc, double lc, int B) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  double j = J[b];
  if (Pp) j -= lp * Pp[b];
  if (Pc) j -= lc * Pc[b];
  J[b] = j;
}

// the configured penalties of rho [B][N] and their gradients into the context
static void run_penalties(maple_ctx* c, const double* rho, bool print, bool cavity, cudaStream_t s) {
  Range range("maple:penalties");
  try {
    if (print) maple_pr::overhang(rho, c->oplan, c->P_print, c->dP_print, c->pen_work, s);
    if (cavity) maple_pr::cavity(rho, c->cplan, c->P_cav, c->dP_cav, c->pen_work, s);
  } catch (const std::runtime_error& e) {
    throw Failure{MAPLE_E_CUDA, e.what()};
  }
}

static constexpr int kNoAllocScratch = 32768;  // doubles
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratch];
static std::mutex g_noalloc_mu;
static double* g_noalloc_addr[128] = {};

static double* noalloc_scratch_address() {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  require(dev >= 0 && dev < 128, "device index out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      throw Failure{MAPLE_E_CUDA, std::string("cudaGetSymbolAddress of the OC scratch array failed: ") +
                                      cudaGetErrorString(e)};
    g_noalloc_addr[dev] = static_cast<double*>(p);
  }
  return g_noalloc_addr[dev];
}

}  // namespace maple

using namespace maple;

template <typename F>
static int guarded(F&& f) {
  try {
    f();
    return MAPLE_OK;
  } catch (const Failure& e) {
    g_err = e.msg;
    return e.code;
  } catch (const std::exception& e) {
    g_err = e.what();
    return MAPLE_E_CUDA;
  }
}

static cudaStream_t S(maple_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

extern "C" {

const char* maple_last_error_string(void) { return g_err.c_str(); }
int maple_version(void) { return 100; }

int maple_element_matrices(int r, double E, double nu, double kappa, double* Ke3, double* Fe3, double* X03,
                           double* Ke1, double* Fe1, double* X01) {
  return guarded([&] {
    require(r >= 1, "resolution must be positive");
    std::unique_ptr<ElementTables> tp(new ElementTables);  // about 0.4 MB: not on the stack
    ElementTables& t = *tp;
    element_tables(E, nu, kappa, &t);
    const double h = 1.0 / r;
    for (int i = 0; i < 576; ++i) if (Ke3) Ke3[i] = t.Ke3[i] * h;
    for (int i = 0; i < 144; ++i) {
      if (Fe3) Fe3[i] = t.Fe3[i] * h * h;
      if (X03) X03[i] = t.X03[i] * h;
    }
    for (int i = 0; i < 64; ++i) if (Ke1) Ke1[i] = t.Ke1[i] * h;
    for (int i = 0; i < 24; ++i) {
      if (Fe1) Fe1[i] = t.Fe1[i] * h * h;
      if (X01) X01[i] = t.X01[i] * h;
    }
  });
}

int maple_ctx_create(int r, int ncells, int levels, double E, double nu, double kappa, maple_ctx** out) {
  return guarded([&] {
    require(out != nullptr, "out is NULL");
    *out = nullptr;
    require(r >= 6 && r % 2 == 0, "resolution must be even and >= 6");
    require(ncells >= 1 && ncells <= 65535, "ncells must be in [1, 65535]");
    require((size_t)r * r * r * 27 < (size_t)1 << 31, "resolution too large");
    require(E > 0 && kappa > 0 && nu > -1.0 && nu < 0.5, "invalid material constants");
    ensure_tables(nu);
    maple_ctx* c = new maple_ctx();
    try {
      CK(cudaGetDevice(&c->dev));
      c->r = r;
      c->B = ncells;
      c->E = E;
      c->nu = nu;
      c->kappa = kappa;
      // levels: coarsen while the grid stays even and the coarse grid has n >= 3
      int n = r, L = 1;
      c->n[0] = r;
      const int maxL = levels > 0 ? std::min(levels, kMaxLevels) : kMaxLevels;
      while (L < maxL && n % 2 == 0 && n / 2 >= 3 && (levels > 0 || n > 4)) {
        n /= 2;
        c->n[L++] = n;
      }
      require(L >= 2, "resolution admits no coarse level");
      require(nodes(n) * 3 <= 1536, "coarsest grid too large for the dense FP64 solve; use more levels");
      c->L = L;
      const double h = 1.0 / r;
      c->ph[0].D = 3;
      c->ph[0].R = 6;
      c->ph[0].kscale = E * h;
      c->ph[0].fscale = E * h * h;
      c->ph[0].xscale = h;
      c->ph[1].D = 1;
      c->ph[1].R = 3;
      c->ph[1].kscale = kappa * h;
      c->ph[1].fscale = kappa * h * h;
      c->ph[1].xscale = h;
      const int B = ncells;
      const size_t N0 = nodes(r);
      for (Lane& L : c->lanes) {
        L.part = dnew<double>(c, (size_t)B * std::max<size_t>(nblk(N0), fine_tiles(r)) * 32);
        L.red = dnew<double>(c, (size_t)B * 32);
        L.sc.rz = dnew<double>(c, B * 6);
        L.sc.rz_new = dnew<double>(c, B * 6);
        L.sc.pq = dnew<double>(c, B * 6);
        L.sc.rr = dnew<double>(c, B * 6);
        L.sc.bnorm2 = dnew<double>(c, B * 6);
        L.sc.alpha = dnew<double>(c, B * 6);
        L.sc.beta = dnew<double>(c, B * 6);
        L.sc.rtol2 = dnew<double>(c, 1);
        L.sc.done = dnew<int>(c, B * 6);
        L.sc.cell_done = dnew<int>(c, B);
        L.sc.iters = dnew<int>(c, B);
        L.sc.run = dnew<int>(c, B);
        L.o_rr = dnew<double>(c, B * 6);
        L.o_bn = dnew<double>(c, B * 6);
        L.o_scale = dnew<double>(c, B * 6);
        L.o_inv = dnew<double>(c, B * 6);
        L.o_done = dnew<int>(c, B);
        L.o_run = dnew<int>(c, B);
        L.o_live = dnew<int>(c, B);
        L.rel = dnew<int>(c, B);
        L.fin_count = dnew<unsigned>(c, B);
        CK(cudaMemset(L.fin_count, 0, B * sizeof(unsigned)));
        L.o_t = dnew<double>(c, B * 6);
        CK(cudaEventCreateWithFlags(&L.pw_fork, cudaEventDisableTiming));
        // the elastic lane's streams take the highest priority (see hi_stream)
        int least = 0, greatest = 0;
        CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        const int prio = (&L == &c->lanes[0]) ? greatest : least;
        for (int l = 1; l + 1 < c->L; ++l) {
          L.pw_part[l] = dnew<double>(c, (size_t)B * nodes(c->n[l]) * 2);
          L.pw_red[l] = dnew<double>(c, (size_t)B * 2);
          if (l > 1) {
            CK(cudaStreamCreateWithPriority(&L.pw[l], cudaStreamNonBlocking, prio));
            CK(cudaEventCreateWithFlags(&L.pw_join[l], cudaEventDisableTiming));
          }
        }
        L.breakdown = dnew<int>(c, 1);
        CK(cudaMemset(L.breakdown, 0, sizeof(int)));
        L.loop = dnew<int>(c, 3);
        CK(cudaMallocHost(&L.h_flags, (B + 2) * sizeof(int)));
      }
      c->active = dnew<int>(c, B);
      c->h_active.assign(B, 1);
      CK(cudaMemcpy(c->active, c->h_active.data(), B * sizeof(int), cudaMemcpyHostToDevice));
      c->x_sym = dnew<double>(c, (size_t)B * N0);  // projected design of a symmetric OC step
      c->dJdx = dnew<double>(c, (size_t)B * N0);
      c->dJf = dnew<double>(c, (size_t)B * N0);
      c->Jv = dnew<double>(c, B);
      c->J_raw = dnew<double>(c, B);
      c->terms = dnew<double>(c, B * 3);
      c->G3 = dnew<double>(c, B * 36);
      c->G1 = dnew<double>(c, B * 9);
      c->stats = dnew<double>(c, B * 2);
      c->ocvf = dnew<double>(c, B);
      int sms = 0;
      CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->dev));
      c->ocpart = dnew<double>(c, (size_t)kOcPartPerBlock * std::max(B, 1) * std::max(sms, 1) * 8);
      c->bar = dnew<unsigned>(c, 2);
      c->err = dnew<int>(c, 1);
      CK(cudaMemset(c->err, 0, sizeof(int)));
      CK(cudaMallocHost(&c->h_err, sizeof(int)));
    } catch (...) {
      for (void* p : c->allocs) cudaFree(p);
      for (Lane& L : c->lanes) {
        if (L.h_flags) cudaFreeHost(L.h_flags);
        if (L.pw_fork) cudaEventDestroy(L.pw_fork);
        for (int l = 0; l < kMaxLevels; ++l) {
          if (L.pw[l]) cudaStreamDestroy(L.pw[l]);
          if (L.pw_join[l]) cudaEventDestroy(L.pw_join[l]);
        }
      }
      if (c->h_err) cudaFreeHost(c->h_err);
      delete c;
      throw;
    }
    *out = c;
  });
}

unsigned long long maple_launch_count(void) { return g_launches.load() + maple_pr::launches(); }

int maple_profile_enable(maple_ctx* c, int enable, int max_launches) {
  return guarded([&] {
    require(c != nullptr, "ctx is NULL");
    if (enable) {
      require(max_launches >= 1 && max_launches <= (1 << 20), "max_launches out of range");
      const size_t want = (size_t)2 * max_launches;
      while (c->ev_pool.size() < want) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        c->ev_pool.push_back(e);
      }
    }
    c->ev_used = 0;
    c->recs.clear();
    c->profiling = enable != 0;
  });
}

int maple_profile_read(maple_ctx* c, char* buf, int buflen) {
  return guarded([&] {
    require(c != nullptr && buf != nullptr && buflen > 0, "NULL argument");
    for (auto& e : c->ev_pool) (void)e;
    if (!c->recs.empty()) CK(cudaEventSynchronize(c->ev_pool[c->recs.back().ev + 1]));
    struct Acc {
      long n = 0;
      double ms = 0, bytes = 0;
    };
    std::map<std::string, Acc> acc;
    for (const auto& r : c->recs) {
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, c->ev_pool[r.ev], c->ev_pool[r.ev + 1]));
      Acc& a = acc[r.name];
      a.n += 1;
      a.ms += ms;
      a.bytes = r.bytes;
    }
    std::string out = "{";
    bool first = true;
    for (const auto& kv : acc) {
      char tmp[512];
      snprintf(tmp, sizeof(tmp), "%s\"%s\": {\"launches\": %ld, \"total_ms\": %.6f, \"bytes_per_launch\": %.1f}",
               first ? "" : ", ", kv.first.c_str(), kv.second.n, kv.second.ms, kv.second.bytes);
      out += tmp;
      first = false;
    }
    out += "}";
    require((int)out.size() < buflen, "profile buffer too small");
    memcpy(buf, out.c_str(), out.size() + 1);
  });
}

int maple_ctx_destroy(maple_ctx* c) {
  return guarded([&] {
    if (!c) return;
    for (auto& e : c->ev_pool) cudaEventDestroy(e);
    drop_graphs(c);
    for (Lane& L : c->lanes) {
      if (L.cap_stream) cudaStreamDestroy(L.cap_stream);
      if (L.cap_stream2) cudaStreamDestroy(L.cap_stream2);
      if (L.side) cudaStreamDestroy(L.side);
      if (L.side_fork) cudaEventDestroy(L.side_fork);
      if (L.side_join) cudaEventDestroy(L.side_join);
      if (L.h_flags) cudaFreeHost(L.h_flags);
      if (L.pw_fork) cudaEventDestroy(L.pw_fork);
      for (int l = 0; l < kMaxLevels; ++l) {
        if (L.pw[l]) cudaStreamDestroy(L.pw[l]);
        if (L.pw_join[l]) cudaEventDestroy(L.pw_join[l]);
      }
    }
    if (c->pen_work) cudaFree(c->pen_work);
    if (c->h_err) cudaFreeHost(c->h_err);
    if (c->aux_stream) cudaStreamDestroy(c->aux_stream);
    if (c->aux_fork) cudaEventDestroy(c->aux_fork);
    if (c->aux_join) cudaEventDestroy(c->aux_join);
    if (c->hi_stream) cudaStreamDestroy(c->hi_stream);
    if (c->hi_fork) cudaEventDestroy(c->hi_fork);
    if (c->hi_join) cudaEventDestroy(c->hi_join);
    for (void* p : c->allocs) cudaFree(p);
    delete c;
  });
}

int maple_ctx_info(const maple_ctx* c, int* levels, int* coarsest, size_t* bytes) {
  return guarded([&] {
    require(c != nullptr, "ctx is NULL");
    if (levels) *levels = c->L;
    if (coarsest) *coarsest = c->n[c->L - 1];
    if (bytes) *bytes = c->bytes;
  });
}

int maple_set_symmetry(maple_ctx* c, int kind, int axes_mask) {
  return guarded([&] {
    require(c != nullptr, "ctx is NULL");
    require(kind == MAPLE_SYM_NONE || kind == MAPLE_SYM_MIRROR || kind == MAPLE_SYM_CUBIC, "unknown symmetry kind");
    require(kind != MAPLE_SYM_MIRROR || (axes_mask > 0 && axes_mask < 8), "mirror symmetry needs axes (mask 1..7)");
    c->sym_kind = kind;
    c->sym_mask = kind == MAPLE_SYM_MIRROR ? axes_mask : (kind == MAPLE_SYM_CUBIC ? 7 : 0);
  });
}

int maple_symmetrize(int r, int ncells, int kind, int axes_mask, const double* in, double* out, maple_stream_t s) {
  return guarded([&] {
    require(in != nullptr && out != nullptr, "NULL argument");
    require(in != out, "out must not alias in");
    require(r >= 1 && ncells >= 1, "bad sizes");
    require(kind == MAPLE_SYM_NONE || kind == MAPLE_SYM_MIRROR || kind == MAPLE_SYM_CUBIC, "unknown symmetry kind");
    require(kind != MAPLE_SYM_MIRROR || (axes_mask > 0 && axes_mask < 8), "mirror symmetry needs axes (mask 1..7)");
    const size_t N = (size_t)r * r * r;
    k_symmetrize<<<g2(N, ncells), kThreads, 0, S(s)>>>(in, out, r, kind, axes_mask, 0, 0.0, 0.0, nullptr);
    CKL();
  });
}

int maple_set_penalties(maple_ctx* c, double lambda_print, double overhang_deg, int overhang_periodic,
                        double lambda_cavity, double void_thresh, double beta, int min_channel_rad, int rad, int iters,
                        int tiles_x, int tiles_y, int tiles_z, int focus_center, int seed_faces, int periodic) {
  return guarded([&] {
    require(c != nullptr, "ctx is NULL");
    require(lambda_print >= 0 && lambda_cavity >= 0, "penalty weights must be >= 0");
    require(seed_faces >= MAPLE_SEED_ALL && seed_faces <= MAPLE_SEED_XY, "unknown seed faces");
    require(tiles_x >= 1 && tiles_y >= 1 && tiles_z >= 1, "tiles must be >= 1");
    require(min_channel_rad >= 0 && rad >= 0 && iters >= 0, "radii and iterations must be >= 0");
    require(std::isfinite(overhang_deg) && std::isfinite(void_thresh) && std::isfinite(beta), "non-finite parameter");
    const int r = c->r, B = c->B;
    maple_pr::OverhangPlan op;
    op.r = r;
    op.B = B;
    {  // lateral support radius for the overhang angle (utils/printability.py:76-90)
      const double od = std::min(89.0, std::max(1.0, overhang_deg));
      op.rad = std::max(1, (int)std::ceil(std::tan((90.0 - od) * M_PI / 180.0)));
    }
    op.periodic = overhang_periodic ? 1 : 0;
    if (op.periodic) require(2 * op.rad + 1 <= r, "overhang support window wider than the cell");
    maple_pr::CavityPlan cp;
    cp.r = r;
    cp.B = B;
    cp.tiles[0] = tiles_x;
    cp.tiles[1] = tiles_y;
    cp.tiles[2] = tiles_z;
    const bool array = tiles_x > 1 || tiles_y > 1 || tiles_z > 1;
    cp.periodic = (periodic && !array) ? 1 : 0;
    cp.min_channel_rad = min_channel_rad;
    cp.rad = rad;
    cp.nsteps = iters > 0 ? iters : (array ? std::max(cp.dims(0), std::max(cp.dims(1), cp.dims(2))) : r);
    cp.seed = seed_faces;
    cp.focus_center = focus_center ? 1 : 0;
    cp.void_thresh = void_thresh;
    cp.beta = beta;
    if (cp.periodic) require(2 * std::max(rad, min_channel_rad) + 1 <= r, "cavity window wider than the cell");
    const bool want_p = lambda_print > 0, want_c = lambda_cavity > 0;
    const size_t bytes = std::max(want_p ? op.bytes() : 0, want_c ? cp.bytes() : 0);
    if (bytes > c->pen_bytes) {
      if (c->pen_work) CK(cudaFree(c->pen_work));
      c->pen_work = nullptr;
      c->pen_bytes = 0;
      cudaError_t e = cudaMalloc(&c->pen_work, bytes);
      if (e != cudaSuccess) throw Failure{MAPLE_E_NOMEM, std::string("penalty workspace: ") + cudaGetErrorString(e)};
      c->pen_bytes = bytes;
    }
    if (!c->pen_rho) {
      const size_t N = (size_t)nodes(r);
      c->pen_rho = dnew<double>(c, (size_t)B * N);
      c->dP_print = dnew<double>(c, (size_t)B * N);
      c->dP_cav = dnew<double>(c, (size_t)B * N);
      c->P_print = dnew<double>(c, B);
      c->P_cav = dnew<double>(c, B);
      CK(cudaMemset(c->P_print, 0, B * sizeof(double)));
      CK(cudaMemset(c->P_cav, 0, B * sizeof(double)));
    }
    c->oplan = op;
    c->cplan = cp;
    c->lambda_print = lambda_print;
    c->lambda_cavity = lambda_cavity;
    c->print_set = want_p;
    c->cavity_set = want_c;
  });
}

int maple_penalties(maple_ctx* c, const double* rho, double* P_print, double* dP_print, double* P_cavity,
                    double* dP_cavity, maple_stream_t s) {
  return guarded([&] {
    require(c != nullptr && rho != nullptr, "NULL argument");
    require(!P_print || c->print_set, "the overhang penalty is not configured (maple_set_penalties)");
    require(!P_cavity || c->cavity_set, "the cavity penalty is not configured (maple_set_penalties)");
    require(!dP_print || P_print, "dP_print needs P_print");
    require(!dP_cavity || P_cavity, "dP_cavity needs P_cavity");
    try {
      if (P_print) maple_pr::overhang(rho, c->oplan, P_print, dP_print, c->pen_work, S(s));
      if (P_cavity) maple_pr::cavity(rho, c->cplan, P_cavity, dP_cavity, c->pen_work, S(s));
    } catch (const std::runtime_error& e) {
      throw Failure{MAPLE_E_CUDA, e.what()};
    }
  });
}

int maple_get_oc_terms(maple_ctx* c, double* J_raw, double* P_print, double* P_cavity, maple_stream_t s) {
  return guarded([&] {
    require(c != nullptr, "ctx is NULL");
    const size_t nb = (size_t)c->B * sizeof(double);
    if (J_raw) CK(cudaMemcpyAsync(J_raw, c->J_raw, nb, cudaMemcpyDeviceToDevice, S(s)));
    if (P_print) {
      if (c->P_print)
        CK(cudaMemcpyAsync(P_print, c->P_print, nb, cudaMemcpyDeviceToDevice, S(s)));
      else
        CK(cudaMemsetAsync(P_print, 0, nb, S(s)));
    }
    if (P_cavity) {
      if (c->P_cav)
        CK(cudaMemcpyAsync(P_cavity, c->P_cav, nb, cudaMemcpyDeviceToDevice, S(s)));
      else
        CK(cudaMemsetAsync(P_cavity, 0, nb, S(s)));
    }
  });
}

int maple_set_concurrency(maple_ctx* c, int enable) {
  return guarded([&] {
    require(c != nullptr, "ctx is NULL");
    c->concurrent = enable != 0;
  });
}

int maple_set_graphs(maple_ctx* c, int enable) {
  return guarded([&] {
    require(c != nullptr, "ctx is NULL");
    drop_graphs(c);
    c->use_graphs = enable != 0;
  });
}

int maple_set_stencil_split(maple_ctx* c, int min_n) {
  return guarded([&] {
    require(c != nullptr, "ctx is NULL");
    require(min_n >= 0, "min_n must be >= 0");
    drop_graphs(c);
    c->split_min_n = min_n;
  });
}

int maple_set_stencil_nine(maple_ctx* c, int max_n) {
  return guarded([&] {
    require(c != nullptr, "ctx is NULL");
    require(max_n >= 0, "max_n must be >= 0");
    drop_graphs(c);
    c->nine_max_n = max_n;
  });
}

int maple_set_pdl(maple_ctx* c, int enable) {
  return guarded([&] {
    require(c != nullptr, "ctx is NULL");
    drop_graphs(c);
    c->pdl = enable != 0;
  });
}

int maple_set_device_loop(maple_ctx* c, int enable) {
  return guarded([&] {
    require(c != nullptr, "ctx is NULL");
    drop_graphs(c);
    c->device_loop = enable != 0;
  });
}

int maple_get_device_loop(maple_ctx* c, int* state) {
  return guarded([&] {
    require(c != nullptr && state != nullptr, "NULL argument");
    int st = 0;
    for (auto& row : c->graphs)
      for (auto& ge : row) {
        if (ge.loop_failed) st = -1;
        else if (ge.loop_exec && st == 0) st = 1;
      }
    *state = st;
  });
}

int maple_set_tail_fused(maple_ctx* c, int enable) {
  return guarded([&] {
    require(c != nullptr, "ctx is NULL");
    drop_graphs(c);
    c->tail_fused = enable != 0;
  });
}

int maple_set_extrapolation(maple_ctx* c, double theta) {
  return guarded([&] {
    require(c != nullptr, "ctx is NULL");
    require(theta >= 0 && theta <= 2, "theta must be in [0, 2]");
    c->extrap = theta;
    for (Phys& p : c->ph) {
      if (theta > 0 && p.alloc && !p.u_prev) p.u_prev = dnew<double>(c, (size_t)c->B * nodes(c->n[0]) * p.R * p.D);
      p.prev_valid = false;
    }
  });
}

int maple_set_mixed_mode(maple_ctx* c, int mode) {
  return guarded([&] {
    require(c != nullptr, "ctx is NULL");
    require(mode == MAPLE_MIXED_FLEXIBLE || mode == MAPLE_MIXED_REFINE || mode == MAPLE_MIXED_RELIABLE,
            "unknown mixed-precision mode");
    c->mixed_mode = mode;
  });
}

int maple_set_reliable_options(maple_ctx* c, double delta, int handover) {
  return guarded([&] {
    require(c != nullptr, "ctx is NULL");
    require(delta > 0.0 && delta < 1.0, "delta must be in (0, 1)");
    require(handover >= 1, "handover must be >= 1");
    c->rel_delta = delta;
    c->rel_handover = handover;
  });
}

int maple_set_coarse_degree(maple_ctx* c, int deg) {
  return guarded([&] {
    require(c != nullptr, "ctx is NULL");
    require(deg >= 0 && deg <= 8, "chebyshev degree must be in [0, 8] (0: automatic)");
    drop_graphs(c);
    c->cheb_degree_coarse = deg;
  });
}

int maple_set_solver_options(maple_ctx* c, int deg, double ratio, int piters, double inner_rtol, int check_every) {
  return guarded([&] {
    require(c != nullptr, "ctx is NULL");
    require(deg >= 1 && deg <= 8, "chebyshev degree must be in [1, 8]");
    require(ratio > 1.0, "chebyshev ratio must exceed 1");
    require(piters >= 1 && piters <= 100, "power iterations must be in [1, 100]");
    require(inner_rtol > 0 && inner_rtol < 1, "inner tolerance must be in (0, 1)");
    require(check_every >= 1, "check_every must be >= 1");
    drop_graphs(c);  // captured launches embed these settings
    c->cheb_degree = deg;
    c->cheb_ratio = ratio;
    c->power_iters = piters;
    c->inner_rtol = inner_rtol;
    c->check_every = check_every;
  });
}

int maple_set_active(maple_ctx* c, const int* act, maple_stream_t s) {
  return guarded([&] {
    require(c != nullptr, "ctx is NULL");
    for (int b = 0; b < c->B; ++b) c->h_active[b] = act ? (act[b] != 0) : 1;
    CK(cudaMemcpyAsync(c->active, c->h_active.data(), c->B * sizeof(int), cudaMemcpyHostToDevice, S(s)));
    CK(cudaStreamSynchronize(S(s)));
  });
}

int maple_set_density(maple_ctx* c, int phys, const double* rho, int prec, maple_stream_t s) {
  return guarded([&] {
    LaneScope lane(phys == MAPLE_THERMAL ? 1 : 0);
    require(c != nullptr && rho != nullptr, "NULL argument");
    require(phys == MAPLE_ELASTIC || phys == MAPLE_THERMAL, "unknown physics");
    require(prec == MAPLE_FP64 || prec == MAPLE_MIXED, "unknown precision");
    ensure_prec(c, phys, prec);
    load_density(c, phys, rho, prec, S(s));
    build(c, phys, prec, S(s));
  });
}

int maple_solve(maple_ctx* c, int phys, int prec, double rtol, int maxit, int warm, int* iters, int* status,
                maple_stream_t s) {
  return guarded([&] {
    LaneScope lane(phys == MAPLE_THERMAL ? 1 : 0);
    require(c != nullptr, "ctx is NULL");
    require(phys == MAPLE_ELASTIC || phys == MAPLE_THERMAL, "unknown physics");
    Phys& p = c->ph[phys];
    require(p.built, "maple_set_density must be called before maple_solve");
    require(p.built_prec == prec, "precision differs from the one the hierarchy was built for");
    require(rtol > 0 && maxit >= 1, "rtol must be > 0 and maxit >= 1");
    assemble_rhs(c, phys, p.o64.rho, p.F64, S(s));
    dispatch_solve(c, phys, prec, p.F64, p.u64, !(warm && p.solved), rtol, maxit, iters, status, S(s));
    p.solved = true;
    p.current = true;
    p.energies = false;
    p.from_oc = false;
  });
}

int maple_solve_rhs(maple_ctx* c, int phys, int prec, const double* F, const double* x0, double rtol, int maxit,
                    double* u_out, double* r_out, int* iters, int* status, maple_stream_t s) {
  return guarded([&] {
    LaneScope lane(phys == MAPLE_THERMAL ? 1 : 0);
    require(c != nullptr && F != nullptr && u_out != nullptr, "NULL argument");
    require(phys == MAPLE_ELASTIC || phys == MAPLE_THERMAL, "unknown physics");
    Phys& p = c->ph[phys];
    require(p.built && p.built_prec == prec, "maple_set_density (same precision) must precede maple_solve_rhs");
    const size_t vb = (size_t)c->B * nodes(c->n[0]) * p.R * p.D * sizeof(double);
    if (x0) CK(cudaMemcpyAsync(u_out, x0, vb, cudaMemcpyDeviceToDevice, S(s)));
    dispatch_solve(c, phys, prec, F, u_out, x0 == nullptr, rtol, maxit, iters, status, S(s));
    if (r_out) {
      ApplyArgs<double> a{};
      a.u = u_out;
      a.f = F;
      a.out = r_out;
      if (phys == MAPLE_ELASTIC)
        apply<double, 3, 6, M_RES>(c, p, p.o64, 0, a, c->active, S(s));
      else
        apply<double, 1, 3, M_RES>(c, p, p.o64, 0, a, c->active, S(s));
    }
  });
}

int maple_get_solution(maple_ctx* c, int phys, double* u_out, maple_stream_t s) {
  return guarded([&] {
    require(c != nullptr && u_out != nullptr, "NULL argument");
    Phys& p = c->ph[phys];
    require(p.solved, "no solution available");
    const size_t vb = (size_t)c->B * nodes(c->n[0]) * p.R * p.D * sizeof(double);
    CK(cudaMemcpyAsync(u_out, p.u64, vb, cudaMemcpyDeviceToDevice, S(s)));
  });
}

int maple_set_solution(maple_ctx* c, int phys, const double* u, maple_stream_t s) {
  return guarded([&] {
    require(c != nullptr && u != nullptr, "NULL argument");
    require(phys == MAPLE_ELASTIC || phys == MAPLE_THERMAL, "unknown physics");
    Phys& p = c->ph[phys];
    alloc_phys(c, phys);
    const size_t vb = (size_t)c->B * nodes(c->n[0]) * p.R * p.D * sizeof(double);
    CK(cudaMemcpyAsync(p.u64, u, vb, cudaMemcpyDeviceToDevice, S(s)));
    p.solved = true;
    p.current = false;
    p.energies = false;
    p.from_oc = false;
  });
}

int maple_homogenize(maple_ctx* c, int phys, double* H_out, double* energy_out, maple_stream_t s) {
  return guarded([&] {
    LaneScope lane(phys == MAPLE_THERMAL ? 1 : 0);
    require(c != nullptr, "ctx is NULL");
    require(phys == MAPLE_ELASTIC || phys == MAPLE_THERMAL, "unknown physics");
    Phys& p = c->ph[phys];
    require(p.current, "maple_solve must follow maple_set_density before maple_homogenize");
    homogenize(c, phys, S(s));
    if (H_out) CK(cudaMemcpyAsync(H_out, p.H, (size_t)c->B * p.R * p.R * sizeof(double), cudaMemcpyDeviceToDevice, S(s)));
    if (energy_out)
      CK(cudaMemcpyAsync(energy_out, p.energy, (size_t)c->B * nodes(c->n[0]) * p.R * p.R * sizeof(double),
                         cudaMemcpyDeviceToDevice, S(s)));
  });
}

int maple_energy_contract(int ncells, int N, int RR, const double* energy, const double* g, int accumulate,
                          double* out, maple_stream_t s) {
  return guarded([&] {
    require(energy && g && out, "NULL argument");
    require(ncells >= 1 && N >= 1 && (RR == 36 || RR == 9), "bad sizes");
    k_energy_contract<<<g2(N, ncells), kThreads, 0, S(s)>>>(energy, g, out, N, RR, accumulate);
    CKL();
  });
}

int maple_sensitivity(maple_ctx* c, const double* gC, const double* gK, double* dJdrho, maple_stream_t s) {
  return guarded([&] {
    require(c != nullptr && dJdrho != nullptr, "NULL argument");
    require(gC || gK, "at least one of gC, gK is required");
    if (gC) require(c->ph[0].energies, "elastic energies missing: call maple_homogenize first");
    if (gK) require(c->ph[1].energies, "thermal energies missing: call maple_homogenize first");
    const int N = nodes(c->n[0]);
    KL(c, S(s), k_sensitivity<<<g2(N, c->B), kThreads, 0, S(s)>>>(nullptr, gC ? c->ph[0].energy : nullptr,
                                                       gK ? c->ph[1].energy : nullptr, gC, gK, nullptr, dJdrho, N, 0, 1,
                                                       0, c->active));
  });
}

int maple_assemble_rhs(maple_ctx* c, int phys, const double* rho, double* F, maple_stream_t s) {
  return guarded([&] {
    require(c != nullptr && rho != nullptr && F != nullptr, "NULL argument");
    require(phys == MAPLE_ELASTIC || phys == MAPLE_THERMAL, "unknown physics");
    assemble_rhs(c, phys, rho, F, S(s));
  });
}

int maple_matvec(maple_ctx* c, int phys, const double* rho, const double* u, double* y, maple_stream_t s) {
  return guarded([&] {
    require(c != nullptr && rho != nullptr && u != nullptr && y != nullptr, "NULL argument");
    require(phys == MAPLE_ELASTIC || phys == MAPLE_THERMAL, "unknown physics");
    Phys& p = c->ph[phys];
    Ops<double> o{};
    o.rho = const_cast<double*>(rho);
    ApplyArgs<double> a{};
    a.u = u;
    a.out = y;
    if (phys == MAPLE_ELASTIC)
      apply<double, 3, 6, M_MV>(c, p, o, 0, a, c->active, S(s));
    else
      apply<double, 1, 3, M_MV>(c, p, o, 0, a, c->active, S(s));
  });
}

int maple_get_level_elements(maple_ctx* c, int phys, int level, double* out, maple_stream_t s) {
  return guarded([&] {
    require(c != nullptr && out != nullptr, "NULL argument");
    require(phys == MAPLE_ELASTIC || phys == MAPLE_THERMAL, "unknown physics");
    require(level >= 1 && level < c->L, "level must be in [1, levels)");
    Phys& p = c->ph[phys];
    require(p.built, "no hierarchy built for this physics (call maple_set_density first)");
    const size_t k = 8 * (size_t)p.D;
    if (level == 1 && !p.ke1_formed) {
      if (p.D == 3)
        level1_elements<3>(c, p, S(s), c->active);
      else
        level1_elements<1>(c, p, S(s), c->active);
      p.ke1_formed = true;
    }
    CK(cudaMemcpyAsync(out, p.KE[level], (size_t)c->B * nodes(c->n[level]) * k * k * sizeof(double),
                       cudaMemcpyDeviceToDevice, S(s)));
  });
}

int maple_matvec_ebe_tc(maple_ctx* c, const float* u, float* y, float* rows_work, float* out_work, maple_stream_t s) {
  return guarded([&] {
    require(c != nullptr && u && y && rows_work && out_work, "NULL argument");
    Phys& p = c->ph[MAPLE_ELASTIC];
    require(p.built && p.o32.alloc && p.o32.rho, "build the elastic hierarchy in mixed precision first");
    const int n = c->n[0], N = nodes(n), B = c->B;
    const long long rows = (long long)B * N * 6;
    require(rows % EBE_ROWS == 0, "the cell size must be a multiple of 4");
    cudaStream_t st = S(s);
    CK(cudaMemsetAsync(c->err, 0, sizeof(int), st));
    const long long tot = (long long)B * 6 * N;
    k_ebe_gather<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(u, rows_work, n, B);
    CKL();
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->dev));
    const long long ntiles = rows / EBE_ROWS;
    const unsigned grid = (unsigned)std::min<long long>(ntiles, (long long)sms * 4);
    k_ebe_gemm_tc<<<grid, EBE_ROWS, 0, st>>>(rows_work, p.o32.rho, out_work, ntiles, N, (float)p.kscale, c->err);
    CKL();
    k_ebe_scatter<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(out_work, y, n, B);
    CKL();
    CK(cudaMemcpyAsync(c->h_err, c->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (*c->h_err) throw Failure{MAPLE_E_TIMEOUT, "maple_matvec_ebe_tc: a tensor-core pipeline wait ran out"};
  });
}

int maple_transfer(int op, int nc, int K, int ncells, const double* in, double* out, maple_stream_t s) {
  return guarded([&] {
    require(in && out && in != out, "in and out must be distinct non-NULL pointers");
    require(op == MAPLE_RESTRICT || op == MAPLE_PROLONG_ADD, "unknown transfer");
    require(nc >= 2 && ncells >= 1 && ncells <= 65535, "nc must be >= 2 and ncells in [1, 65535]");
    require(K == 3 || K == 18, "K must be 3 (thermal fields) or 18 (elastic fields)");
    cudaStream_t st = S(s);
    const dim3 g = g2((size_t)nodes(nc) * K, ncells);
    if (op == MAPLE_RESTRICT) {
      if (K == 3)
        k_restrict<double, 3><<<g, kThreads, 0, st>>>(in, out, nc, nullptr);
      else
        k_restrict<double, 18><<<g, kThreads, 0, st>>>(in, out, nc, nullptr);
    } else {
      if (K == 3)
        k_prolong_add<double, 3><<<g, kThreads, 0, st>>>(in, out, nc, nullptr);
      else
        k_prolong_add<double, 18><<<g, kThreads, 0, st>>>(in, out, nc, nullptr);
    }
    CKL();
  });
}

int maple_box_filter(int r, int ncells, int k, const double* in, double* out, maple_stream_t s) {
  return guarded([&] {
    require(in != nullptr && out != nullptr, "NULL argument");
    require(k > 0 && k % 2 == 1, "filter size must be a positive odd integer");
    require(r >= 1 && ncells >= 1, "bad sizes");
    require(in != out, "in-place filtering is not supported");
    k_box_filter<<<g2((size_t)r * r * r, ncells), kThreads, 0, S(s)>>>(in, out, r, k, nullptr);
    CKL();
  });
}

int maple_oc_update(maple_ctx* c, const double* x, const double* dJdx, const double* vf, double move, double xmin,
                    double* xnew, double* stats, maple_stream_t s) {
  return guarded([&] {
    require(c != nullptr && x && dJdx && vf && xnew, "NULL argument");
    require(xnew != x, "xnew must not alias x");
    oc_update(c, x, dJdx, vf, move, xmin, xnew, stats, S(s));
    check_oc_barrier(c, S(s));
  });
}

int maple_oc_update_noalloc(int N, int ncells, const double* x, const double* dJdx, const double* vf, double move,
                            double xmin, double* xnew, double* stats, maple_stream_t s) {
  return guarded([&] {
    require(x && dJdx && vf && xnew, "NULL argument");
    require(xnew != x, "xnew must not alias x");
    require(N >= 1 && ncells >= 1, "N and ncells must be positive");
    // layout of the array per launch: [4*nb*G partial sums][2*nb statistics if
    // the caller passes none] ... [4 doubles: barrier count, generation, error]
    constexpr int kTail = 4;
    const int per_cell_min = 4 + (stats ? 0 : 2);  // G = 1
    const int max_cells = (kNoAllocScratch - kTail) / per_cell_min;
    require(ncells <= max_cells, "maple_oc_update_noalloc: " + std::to_string(ncells) + " cells exceed the " +
                                     std::to_string(max_cells) + " cells its fixed 256 KiB scratch array holds");
    double* scratch = noalloc_scratch_address();
    cudaStream_t st = S(s);
    int dev = 0, per_sm = 0, sms = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_oc_update, kThreads, 0));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int maxres = per_sm * sms;
    require(maxres >= 1, "OC kernel cannot be resident");
    const int want_G = std::max(1, std::min(sms, (N + 4 * kThreads - 1) / (4 * kThreads)));
    const int cells_per_launch = std::max(1, std::min(ncells, maxres / want_G));
    unsigned* bar = reinterpret_cast<unsigned*>(scratch + kNoAllocScratch - kTail);
    int* err = reinterpret_cast<int*>(scratch + kNoAllocScratch - kTail + 2);
    // the error word is cleared once per call and read after its last launch;
    // the barrier words before every launch
    CK(cudaMemsetAsync(err, 0, sizeof(int), st));
    for (int c0 = 0; c0 < ncells; c0 += cells_per_launch) {
      const int nb = std::min(cells_per_launch, ncells - c0);
      const int stats_words = stats ? 0 : 2 * nb;
      const int G = std::max(1, std::min({want_G, maxres / nb, (kNoAllocScratch - kTail - stats_words) / (4 * nb)}));
      OcArgs a{};
      a.x = x + (size_t)c0 * N;
      a.dJ = dJdx + (size_t)c0 * N;
      a.xnew = xnew + (size_t)c0 * N;
      a.volfrac = vf + c0;
      a.move = move;
      a.xmin = xmin;
      a.N = N;
      a.part = scratch;
      a.stats = stats ? stats + 2 * c0 : scratch + (size_t)4 * nb * G;
      a.lam_out = nullptr;
      a.bar = bar;
      a.err = err;
      a.active = nullptr;
      a.poll_limit = tl_wait_polls;
      a.phantom = tl_wait_phantom;
      CK(cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), st));
      void* args[] = {&a};
      CK(cudaLaunchCooperativeKernel((void*)k_oc_update, dim3(G, nb), dim3(kThreads), args, 0, st));
      g_launches.fetch_add(1);
    }
    // a barrier that gave up is reported here: copying the word into host
    // (stack) memory waits for the stream
    int h_err = 0;
    CK(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (h_err)
      throw Failure{MAPLE_E_TIMEOUT, "maple_oc_update_noalloc: a grid barrier wait ran out (not every block of the "
                                     "cooperative launch arrived); xnew and the statistics are incomplete"};
  });
}

int maple_oc_step(maple_ctx* c, const double* x, const double* w, const double* vf, double penal, double rho_min,
                  double move, double xmin, int filter_k, int prec, double rtol, int maxit, int warm, double* x_next,
                  double* J, double* terms, double* CH, double* kappa, double* stats, int* iters, maple_stream_t s) {
  return guarded([&] {
    Range range("maple:oc_step");
    require(c != nullptr && x && w && vf && x_next, "NULL argument");
    require(x_next != x, "x_next must not alias x");
    require(prec == MAPLE_FP64 || prec == MAPLE_MIXED, "unknown precision");
    cudaStream_t st = S(s);
    const int B = c->B, N = nodes(c->n[0]);
    std::vector<double> hw(3 * B);
    CK(cudaMemcpyAsync(hw.data(), w, 3 * B * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    bool need_ch = false, need_k = false;
    for (int b = 0; b < B; ++b) {
      if (!c->h_active[b]) continue;
      need_ch |= (hw[3 * b] != 0.0 || hw[3 * b + 1] != 0.0);
      need_k |= (hw[3 * b + 2] != 0.0);
    }
    // symmetric designs: the solves see clamp(P(clamp(x))) (main_IHD_v3.py:625-626)
    const bool sym = c->sym_kind != SYM_NONE;
    const double* xu = x;
    if (sym) {
      KL(c, st, k_symmetrize<<<g2(N, B), kThreads, 0, st>>>(x, c->x_sym, c->n[0], c->sym_kind, c->sym_mask, 1, xmin,
                                                           1.0, c->active));
      xu = c->x_sym;
    }
    // manufacturability penalties at the solves' densities (main_IHD_v3.py:649-686)
    const bool pen_p = c->lambda_print > 0 && c->print_set, pen_c = c->lambda_cavity > 0 && c->cavity_set;
    auto run_pen = [&](cudaStream_t ps) {
      KL(c, ps, k_simp<<<nblk((size_t)B * N), kThreads, 0, ps>>>(xu, c->pen_rho, nullptr, (size_t)B * N, N, xmin,
                                                               penal, rho_min, c->active));
      run_penalties(c, c->pen_rho, pen_p, pen_c, ps);
    };
    // one physics: SIMP map, hierarchy, RHS, MG-PCG solve, energies
    auto run_phys = [&](int phys, cudaStream_t ps, int* it_out) {
      LaneScope lane(phys);
      Phys& p = c->ph[phys];
      const size_t tot = (size_t)B * N;
      KL(c, ps, k_simp<<<nblk(tot), kThreads, 0, ps>>>(xu, p.o64.rho, prec == MAPLE_MIXED ? p.o32.rho : nullptr,
                                                       tot, N, xmin, penal, rho_min, c->active));
      build(c, phys, prec, ps);
      assemble_rhs(c, phys, p.o64.rho, p.F64, ps);
      const bool was_solved = p.solved;
      if (warm && was_solved && p.from_oc && c->extrap > 0 && p.u_prev) {
        // start from the previous solution extrapolated along the OC trajectory
        const size_t len = (size_t)nodes(c->n[0]) * p.R * p.D;
        KL(c, ps, k_extrapolate<<<dim3(64, B), kThreads, 0, ps>>>(p.u64, p.u_prev, p.prev_valid ? c->extrap : 0.0,
                                                                  len, c->active));
        p.prev_valid = true;
      } else {
        p.prev_valid = false;
      }
      dispatch_solve(c, phys, prec, p.F64, p.u64, !(warm && was_solved), rtol, maxit, it_out, nullptr, ps);
      p.solved = true;
      p.current = true;
      p.from_oc = true;
      homogenize(c, phys, ps);
    };
    std::vector<int> it_el(B, 0), it_th(B, 0), it_sum(B, 0);
    if (!need_ch) c->ph[0].energies = false;
    if (!need_k) c->ph[1].energies = false;
    if (need_ch) ensure_prec(c, 0, prec);  // all allocation happens here, on this thread
    if (need_k) ensure_prec(c, 1, prec);
    // work of the caller's stream and of the second stream: with concurrency,
    // the penalties and (when both physics are needed) the thermal solve run
    // on the second stream, driven by a second host thread (each solve waits
    // on its own convergence checks)
    const bool pen = pen_p || pen_c;
    const bool conc = c->concurrent && !c->profiling;
    const bool aux_thermal = conc && need_ch && need_k, aux_pen = conc && pen && (need_ch || need_k);
    if (aux_thermal || aux_pen) {
      if (!c->aux_stream) {
        int least = 0, greatest = 0;
        CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        CK(cudaStreamCreateWithPriority(&c->aux_stream, cudaStreamNonBlocking, least));
        CK(cudaEventCreateWithFlags(&c->aux_fork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c->aux_join, cudaEventDisableTiming));
        CK(cudaStreamCreateWithPriority(&c->hi_stream, cudaStreamNonBlocking, greatest));
        CK(cudaEventCreateWithFlags(&c->hi_fork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c->hi_join, cudaEventDisableTiming));
      }
      CK(cudaEventRecord(c->aux_fork, st));
      CK(cudaStreamWaitEvent(c->aux_stream, c->aux_fork, 0));
      // the caller's stream hands its work to the high-priority stream and
      // takes it back after the solves
      cudaStream_t sm = aux_thermal ? c->hi_stream : st;
      if (aux_thermal) CK(cudaStreamWaitEvent(c->hi_stream, c->aux_fork, 0));
      std::exception_ptr thermal_err;
      const int dev = c->dev;
      std::thread worker([&] {
        try {
          CK(cudaSetDevice(dev));
          if (aux_pen) run_pen(c->aux_stream);
          if (aux_thermal) run_phys(1, c->aux_stream, it_th.data());
        } catch (...) {
          thermal_err = std::current_exception();
        }
      });
      try {
        if (need_ch) run_phys(0, sm, it_el.data());
        if (need_k && !aux_thermal) run_phys(1, sm, it_th.data());
      } catch (...) {
        worker.join();
        throw;
      }
      worker.join();
      if (thermal_err) std::rethrow_exception(thermal_err);
      CK(cudaEventRecord(c->aux_join, c->aux_stream));
      CK(cudaStreamWaitEvent(st, c->aux_join, 0));
      if (aux_thermal) {
        CK(cudaEventRecord(c->hi_join, c->hi_stream));
        CK(cudaStreamWaitEvent(st, c->hi_join, 0));
      }
    } else {
      if (pen) run_pen(st);
      if (need_ch) run_phys(0, st, it_el.data());
      if (need_k) run_phys(1, st, it_th.data());
    }
    for (int b = 0; b < B; ++b) it_sum[b] = it_el[b] + it_th[b];
    KL(c, st, k_objective<<<nblk(B), kThreads, 0, st>>>(c->ph[0].H, c->ph[1].H, w, c->Jv, c->terms, c->G3, c->G1, B,
                                              need_ch ? 1 : 0, need_k ? 1 : 0, c->active));
    CK(cudaMemcpyAsync(c->J_raw, c->Jv, B * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (pen_p || pen_c)
      KL(c, st, k_penalise_J<<<nblk(B), kThreads, 0, st>>>(c->Jv, pen_p ? c->P_print : nullptr, c->lambda_print,
                                                          pen_c ? c->P_cav : nullptr, c->lambda_cavity, B));
    KL(c, st, k_sensitivity<<<g2(N, B), kThreads, 0, st>>>(xu, need_ch ? c->ph[0].energy : nullptr,
                                                 need_k ? c->ph[1].energy : nullptr, c->G3, c->G1, c->dJdx, nullptr, N,
                                                 xmin, penal, rho_min, c->active, pen_p ? c->dP_print : nullptr,
                                                 c->lambda_print, pen_c ? c->dP_cav : nullptr, c->lambda_cavity));
    double *dJ = c->dJdx, *spare = c->dJf;
    if (sym) {  // the gradient through the (self-adjoint) projection
      KL(c, st, k_symmetrize<<<g2(N, B), kThreads, 0, st>>>(dJ, spare, c->n[0], c->sym_kind, c->sym_mask, 0, 0.0,
                                                           0.0, c->active));
      std::swap(dJ, spare);
    }
    if (filter_k > 1) {
      require(filter_k % 2 == 1, "filter size must be odd");
      KL(c, st, k_box_filter<<<g2(N, B), kThreads, 0, st>>>(dJ, spare, c->n[0], filter_k, c->active));
      std::swap(dJ, spare);
    }
    oc_update(c, x, dJ, vf, move, xmin, x_next, c->stats, st);
    if (sym) {  // x_next = clamp(P(x_new)), statistics of x_next - x (main_IHD_v3.py:695-700)
      KL(c, st, k_symmetrize<<<g2(N, B), kThreads, 0, st>>>(x_next, c->x_sym, c->n[0], c->sym_kind, c->sym_mask, 1,
                                                           xmin, 1.0, c->active));
      CK(cudaMemcpyAsync(x_next, c->x_sym, (size_t)B * N * sizeof(double), cudaMemcpyDeviceToDevice, st));
      KL(c, st, k_dx_stats<<<B, 1024, 0, st>>>(x, x_next, c->stats, N, c->active));
    }
    if (J) CK(cudaMemcpyAsync(J, c->Jv, B * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (terms) CK(cudaMemcpyAsync(terms, c->terms, 3 * B * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (CH && need_ch) CK(cudaMemcpyAsync(CH, c->ph[0].H, 36 * B * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (kappa && need_k) CK(cudaMemcpyAsync(kappa, c->ph[1].H, 9 * B * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (stats) CK(cudaMemcpyAsync(stats, c->stats, 2 * B * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (iters)
      for (int b = 0; b < B; ++b) iters[b] = it_sum[b];
    check_oc_barrier(c, st);
  });
}

int maple_test_wait_limit(long long max_polls, int phantom_blocks) {
  return guarded([&] {
    require(max_polls >= 0 && phantom_blocks >= 0, "max_polls and phantom_blocks must be >= 0");
    tl_wait_polls = max_polls > 0 ? max_polls : kBarrierPolls;
    tl_wait_phantom = (unsigned)phantom_blocks;
  });
}

}  // extern "C"
