/*
 * maple_b200 — C ABI of the B200-native inverse-homogenization inner loop.
 *
 * Every entry point takes plain pointers and sizes (device pointers unless a
 * name says "host"), enqueues its work on the caller's CUDA stream and returns
 * an int status (MAPLE_OK = 0).  On failure maple_last_error_string() returns a
 * thread-local message.  Per-cell solver outcomes are returned in arrays and
 * never raised, so one bad cell does not abort a batch.
 *
 * Layouts: a batch holds B periodic cells of r^3 voxels; element / node id is
 * x*r*r + y*r + z.  Design variables, densities and sensitivities are [B][N]
 * FP64; solution fields are [B][R][D][N] FP64 (R load cases of D components,
 * component-major so that consecutive nodes are contiguous).
 *
 * Each declaration names the reference interface (xing-yuu/MAPLE, paths under
 * src/maple/core) whose role it takes over.
 */
#ifndef MAPLE_B200_H
#define MAPLE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct maple_ctx maple_ctx;
typedef void* maple_stream_t; /* cudaStream_t */

enum {
  MAPLE_OK = 0,
  MAPLE_E_BADARG = 1,
  MAPLE_E_CUDA = 2,
  MAPLE_E_NOT_CONVERGED = 3,
  MAPLE_E_BREAKDOWN = 4,
  MAPLE_E_TIMEOUT = 5,
  MAPLE_E_NOMEM = 6
};

enum { MAPLE_ELASTIC = 0, MAPLE_THERMAL = 1 };
enum { MAPLE_FP64 = 0, MAPLE_MIXED = 1 };

/* Per-cell solver status (maple_solve / maple_solve_rhs status_out): CONVERGED,
 * BREAKDOWN (a load case's PCG hit p.Ap <= 0 or a non-finite value and was
 * frozen at its last iterate) or MAXIT, plus the FALLBACK bit when a
 * mixed-precision breakdown was solved again in plain FP64 (the status is then
 * that solve's outcome, e.g. CONVERGED | FALLBACK). */
enum { MAPLE_CELL_CONVERGED = 1, MAPLE_CELL_BREAKDOWN = 2, MAPLE_CELL_MAXIT = 4, MAPLE_CELL_FALLBACK = 8 };

const char* maple_last_error_string(void);
int maple_version(void);

/* Element tables for a voxel of edge 1/r (FP64, host memory).
 * Replaces utils/_utils.py:39-48 isotropic_elastic_tensor,
 * utils/_utils.py:49-109 hexahedron and utils/_utils.py:116-196
 * hexahedron_scalar.  Ke3 24x24, Fe3 24x6, X03 24x6, Ke1 8x8, Fe1 8x3,
 * X01 8x3, all row-major.  C has the float32 entries of the reference. */
int maple_element_matrices(int r, double E, double nu, double kappa, double* Ke3_host, double* Fe3_host,
                           double* X03_host, double* Ke1_host, double* Fe1_host, double* X01_host);

/* Context: B cells of r^3 voxels, `levels` multigrid levels (0 = automatic:
 * coarsen until the coarsest grid is 4^3).  All device workspace is allocated
 * here and on first use of a precision; no allocation happens inside solves.
 * Replaces the per-call hierarchy build of utils/EBE_GMG.py:790-849 and
 * utils/EBE_GMG_scalar.py:650-698, and the IHD module state of
 * utils/model.py:12-32. */
int maple_ctx_create(int r, int ncells, int levels, double E, double nu, double kappa, maple_ctx** out);
int maple_ctx_destroy(maple_ctx* ctx);
int maple_ctx_info(const maple_ctx* ctx, int* levels_out, int* coarsest_n_out, size_t* bytes_out);

/* Solver tuning (defaults: chebyshev degree 1 on the fine level and on level 1
 * (when it has more than 16^3 nodes; coarser levels: maple_set_coarse_degree),
 * interval ratio 10, 12 power iterations, inner FP32 tolerance 1e-5,
 * convergence check every iteration). */
int maple_set_solver_options(maple_ctx* ctx, int cheb_degree, double cheb_ratio, int power_iters, double inner_rtol,
                             int check_every);

/* Form of the mixed-precision (MAPLE_MIXED) solve:
 *   MAPLE_MIXED_FLEXIBLE  (default) flexible FP64 PCG (FP64 fine operator, residuals and
 *                         dot products every iteration) preconditioned by the
 *                         FP32 V-cycle;
 *   MAPLE_MIXED_REFINE    FP32 MG-PCG (FP32 fine operator and vectors, FP64
 *                         accumulated dots) on the scaled FP64 residual inside
 *                         FP64 iterative refinement: per outer pass one FP64
 *                         residual r = b - A x, the convergence test, the inner
 *                         solve to the inner tolerance of
 *                         maple_set_solver_options, and x += ||r|| e in FP64.
 *   MAPLE_MIXED_RELIABLE  FP32 MG-PCG (FP32 fine operator and vectors, FP64
 *                         accumulated dots) on the residual scaled to unit
 *                         norm, with reliable updates: when a load case's
 *                         recurrence residual fell by the factor of
 *                         maple_set_reliable_delta, or passes the tolerance
 *                         test, the FP32 correction is folded into the FP64
 *                         iterate and the residual is recomputed as b - A x in
 *                         FP64 and continues the iteration (the direction is
 *                         kept, not restarted).  Faster where the cells are
 *                         well conditioned (64^3 benchmark cell: same PCG
 *                         iterations, 7% less time); on badly conditioned ones
 *                         the FP32 recurrences need up to twice the iterations
 *                         (128^3, vf 0.15), so the autotuner chooses per workload.
 * All stop at the same FP64 residual test ||b - A x|| <= rtol ||b|| per load
 * case.  The reference solves in one precision (utils/EBE_GMG.py:758-885,
 * dtype argument). */
enum { MAPLE_MIXED_FLEXIBLE = 0, MAPLE_MIXED_REFINE = 1, MAPLE_MIXED_RELIABLE = 2 };
int maple_set_mixed_mode(maple_ctx* ctx, int mode);

/* MAPLE_MIXED_RELIABLE options: delta, the residual reduction per FP32
 * segment, in (0, 1) (default 1e-3); handover, the iterations after which a
 * cell that has not converged continues in the MAPLE_MIXED_FLEXIBLE form from
 * its iterate, within the same iteration limit (default 120: FP32
 * recurrences lose orthogonality on badly conditioned cells, e.g. near-void
 * designs with floating stiff islands, where FP64 recurrences still
 * converge). */
int maple_set_reliable_options(maple_ctx* ctx, double delta, int handover);

/* Warm start of the solves of maple_oc_step (with warm = 1) along the OC
 * trajectory: from u_k + theta (u_k - u_{k-1}), the last two steps'
 * solutions, instead of u_k (theta = 0, the default).  Only the initial
 * iterate changes; every solve still stops at its tolerance.  The reference
 * starts every solve from zero (utils/EBE_GMG.py:851-858). */
int maple_set_extrapolation(maple_ctx* ctx, double theta);

/* CUDA-graph replay of the PCG iteration body (default on).  Off runs every
 * launch eagerly (same results). */
int maple_set_graphs(maple_ctx* ctx, int enable);

/* Coarse multigrid levels with n >= min_n nodes per axis (and n % 8 == 0)
 * apply their stencils with the split-offset kernel (three threads per node,
 * one per x-offset plane); the others with the shared-memory tile kernel.
 * 0 disables the split kernel.  Default 32 (on B200 the tile kernel is
 * faster below 32^3 nodes).  Results differ only by FP summation order. */
int maple_set_stencil_split(maple_ctx* ctx, int min_n);

/* Coarse multigrid levels with n <= max_n nodes per axis apply their stencils
 * with the nine-thread kernel (one thread per node and (x, y) offset pair;
 * taken before the split kernel); 0 disables it.  Default 64: on B200 it is
 * faster than the tile kernel on 8^3 and 16^3 levels and than the split
 * kernel on 32^3 and 64^3 levels.  Results differ only by FP summation order. */
int maple_set_stencil_nine(maple_ctx* ctx, int max_n);

/* FP32 V-cycles whose second-coarsest level has 8^3 nodes above a 4^3-node
 * coarsest level run that level's smoothing, residual, restriction, the
 * coarsest solve and the prolongation as one launch: a cluster of 8 CTAs per
 * cell, each holding one x plane of the level in shared memory.  Default on;
 * 0 runs the separate launches.  Same operand order, so the same results.
 * The reference's V-cycle (utils/EBE_GMG.py:886-970, _v_cycle) recurses one
 * level at a time; this changes only how the bottom two levels are launched. */
int maple_set_tail_fused(maple_ctx* ctx, int enable);

/* Launch the coarse-level stencil sweeps, the grid transfers and the fused
 * V-cycle tail with programmatic dependent launch: each may start, and load
 * the stencils built before the solve, while the previous kernel in the
 * stream drains; it reads the previous kernel's output only after
 * griddepcontrol.wait.  Default on; 0 launches them plainly.  Results are
 * identical either way. */
int maple_set_pdl(maple_ctx* ctx, int enable);

/* Run the PCG iterations of a solve as a loop on the device: the captured
 * iteration body sits in a conditional WHILE graph node, whose last kernel
 * counts the iteration and ends the loop once every active cell has converged
 * or the iteration limit is reached, so the host waits once per solve instead
 * of once per iteration (check_every of maple_set_solver_options then has no
 * effect); the residual replacement of MAPLE_MIXED_RELIABLE sits in a
 * conditional IF node of the captured iteration.  Default on; 0, or a runtime
 * that refuses conditional graph nodes, replays one graph per iteration with
 * the replacement's launches predicated on device flags (profilers that do
 * not support conditional graphs see every kernel this way).  Results and
 * iteration counts are identical either way.  The reference's loop (utils/EBE_GMG.py:858-885,
 * GMGSolver.solve) tests the residual on the host after every cycle. */
int maple_set_device_loop(maple_ctx* ctx, int enable);

/* *state = 1 when a device-side loop graph of this context is built and in
 * use, 0 when none has been built (no graph solve yet, or the loop is off),
 * -1 when the runtime refused one and per-iteration graphs run instead. */
int maple_get_device_loop(maple_ctx* ctx, int* state);

/* Chebyshev degree of the smoother on multigrid levels 2 and deeper (level 0
 * and 1 use the degree of maple_set_solver_options).  0 (default): automatic,
 * 3 on every level below level 1 and on a level 1 of at most 16^3 nodes,
 * never below the common degree. */
int maple_set_coarse_degree(maple_ctx* ctx, int deg);

/* Elastic and thermal solves of maple_oc_step at the same time (default on):
 * the thermal build and solve run on a second stream driven by a second host
 * thread of the library.  Off runs them one after the other on the caller's
 * stream (same results).  maple_oc_step replaces the two TO_homo calls of
 * main_IHD_v3.py:639-645, which the reference makes one after the other. */
int maple_set_concurrency(maple_ctx* ctx, int enable);

/* Symmetry projection (main_IHD_v3.py:221-337): kind MAPLE_SYM_MIRROR averages
 * over the reflections about the centre planes of the axes in axes_mask
 * (bit 0 = x, 1 = y, 2 = z; voxel i reflects to r-1-i); MAPLE_SYM_CUBIC over
 * all 48 axis permutations and reflections.  maple_set_symmetry makes
 * maple_oc_step solve at clamp(P(x)), project the gradient and return
 * clamp(P(x_new)) (main_IHD_v3.py:625-626, 695-700; default none);
 * maple_symmetrize applies P to [ncells][r^3] fields (symmetrize_vec,
 * main_IHD_v3.py:329-337).  out must not alias in. */
enum { MAPLE_SYM_NONE = 0, MAPLE_SYM_MIRROR = 1, MAPLE_SYM_CUBIC = 2 };
int maple_set_symmetry(maple_ctx* ctx, int kind, int axes_mask);
int maple_symmetrize(int r, int ncells, int kind, int axes_mask, const double* in, double* out,
                     maple_stream_t stream);

/* Manufacturability penalties of the OC objective (utils/printability.py,
 * main_IHD_v3.py:649-686): J = J_raw - lambda_print * P_overhang -
 * lambda_cavity * P_cavity, differentiated with the tie rules of the
 * reference's autograd.  Overhang: build direction +z, lateral support radius
 * ceil(tan(90 - overhang_deg)), periodic in x and y if overhang_periodic
 * (printability_penalty_overhang; the optimizer uses periodic).  Cavity: soft void sigmoid(beta (thresh -
 * rho)), optional opening of radius min_channel_rad, flood fill of `iters`
 * steps (0: the supercell's largest dimension) with windows of radius rad
 * from the seed faces; tiles 1,1,1 = cavity_penalty_closed_void (periodic as
 * given), more tiles = cavity_penalty_periodic_array (non-periodic supercell,
 * focus_center: the centre tile only when every count >= 3).  Workspace is
 * allocated here (the cavity tape grows with iters x supercell size).  A
 * weight of 0 disables that penalty in maple_oc_step. */
enum { MAPLE_SEED_ALL = 0, MAPLE_SEED_X = 1, MAPLE_SEED_Y = 2, MAPLE_SEED_Z = 3, MAPLE_SEED_XY = 4 };
int maple_set_penalties(maple_ctx* ctx, double lambda_print, double overhang_deg, int overhang_periodic,
                        double lambda_cavity, double void_thresh, double beta, int min_channel_rad, int rad, int iters,
                        int tiles_x, int tiles_y, int tiles_z, int focus_center, int seed_faces, int periodic);

/* The configured penalties of densities rho [B][N] (device): P [B] and dP/drho
 * [B][N] (each nullable; a gradient needs its value).  A penalty must have
 * been enabled (weight > 0) by maple_set_penalties. */
int maple_penalties(maple_ctx* ctx, const double* rho, double* P_print, double* dP_print, double* P_cavity,
                    double* dP_cavity, maple_stream_t stream);

/* Terms of the last maple_oc_step per cell (device [B], nullable): the
 * objective before penalties and both penalty values (0 when disabled). */
int maple_get_oc_terms(maple_ctx* ctx, double* J_raw, double* P_print, double* P_cavity, maple_stream_t stream);

/* Per-cell active mask (host int[B], nonzero = active). Inactive cells are
 * skipped by every kernel.  NULL = all active. */
int maple_set_active(maple_ctx* ctx, const int* active_host, maple_stream_t stream);

/* Load element densities rho [B][N] (FP64 device) and build the operator
 * hierarchy of one physics: Galerkin coarse element matrices
 * (utils/EBE_GMG.py:226-337, utils/EBE_GMG_scalar.py:135-230), node stencils,
 * Chebyshev bounds and the FP64 coarsest inverse.  `precision` selects which
 * operator copies are built (MAPLE_FP64 or MAPLE_MIXED). */
int maple_set_density(maple_ctx* ctx, int physics, const double* rho, int precision, maple_stream_t stream);

/* Solve K(rho) u = F(rho) for all R load cases of all cells by MG-PCG
 * (plain FP64, or FP32 PCG inside FP64 iterative refinement).  `warm` = 1
 * starts from the previous solution of this physics, 0 from zero.  Replaces
 * utils/EBE_GMG.py:758-885 GMGSolver.solve (and the scalar
 * utils/EBE_GMG_scalar.py:617-725) as called by utils/model.py:111-124 and
 * 140-152.  iters_out/status_out: host int[B] (nullable). */
int maple_solve(maple_ctx* ctx, int physics, int precision, double rtol, int maxit, int warm, int* iters_out_host,
                int* status_out_host, maple_stream_t stream);

/* Solve with a caller-provided RHS F [B][R][D][N] and initial guess x0
 * (nullable) on the density of the last maple_set_density: the
 * GMGSolver.solve(fine_ke, global_f, ...) surface of utils/EBE_GMG.py:758.
 * The solution is written to u_out [B][R][D][N] and the final residual
 * F - K u to r_out (nullable). */
int maple_solve_rhs(maple_ctx* ctx, int physics, int precision, const double* F, const double* x0, double rtol,
                    int maxit, double* u_out, double* r_out, int* iters_out_host, int* status_out_host,
                    maple_stream_t stream);

/* Copy the current solution [B][R][D][N] of a physics into u_out. */
int maple_get_solution(maple_ctx* ctx, int physics, double* u_out, maple_stream_t stream);

/* Homogenized tensor H [B][R][R] = sum_e (X0-u_e)^T rho_e Ke0 (X0-u_e) and the
 * per-element energies kept for maple_sensitivity.  Replaces
 * utils/model.py:33-44 homogenized_batch_3d and 47-95
 * homogenized_batch_thermal.  energy_out [B][R][R][N] (nullable) receives a
 * copy of the per-element energies. */
int maple_homogenize(maple_ctx* ctx, int physics, double* H_out, double* energy_out, maple_stream_t stream);

/* out[b][e] (+)= sum_{r,s} g[b][r][s] * energy[b][r][s][e]: the contraction of
 * saved per-element energies [B][RR][N] (RR = R*R) with dJ/dH [B][RR]; the
 * backward pass of the homogenization (main_IHD_v3.py:688).  accumulate != 0
 * adds to out. */
int maple_energy_contract(int ncells, int N, int RR, const double* energy, const double* g, int accumulate,
                          double* out, maple_stream_t stream);

/* dJ/drho_e = sum_ij gC_ij dC_ij/drho_e + sum_ij gK_ij dkappa_ij/drho_e from
 * the energies of the last homogenization (the analytic adjoint of the
 * autograd call at main_IHD_v3.py:688).  gC [B][6][6], gK [B][3][3] (either
 * nullable), dJdrho [B][N]. */
int maple_sensitivity(maple_ctx* ctx, const double* gC, const double* gK, double* dJdrho, maple_stream_t stream);

/* RHS assembly F = sum_e rho_e Fe0 [B][R][D][N] (utils/_utils.py:453-507,
 * assemble_F_fast / assemble_F_fast_scalar). */
int maple_assemble_rhs(maple_ctx* ctx, int physics, const double* rho, double* F_out, maple_stream_t stream);

/* y = K(rho) u on the fine level, FP64 (utils/EBE_GMG.py:412-430
 * EBEOperator.matvec with Ke_e = rho_e Ke0). */
int maple_matvec(maple_ctx* ctx, int physics, const double* rho, const double* u, double* y, maple_stream_t stream);

/* Galerkin element matrices of multigrid level `level` (1 <= level < levels)
 * of the hierarchy the last maple_set_density built for `physics`: out
 * [B][N_l][8D][8D] FP64, row-major, element id x*n*n + y*n + z of the level's
 * n^3 grid, local index corner*D + component with the element-local corner
 * order 000,100,110,010,001,101,111,011.  The coarse Ke of
 * utils/EBE_GMG.py:226-337 sparse_coarsen_ke (scalar:
 * utils/EBE_GMG_scalar.py:135-230). */
int maple_get_level_elements(maple_ctx* ctx, int physics, int level, double* out, maple_stream_t stream);

/* Periodic trilinear grid transfer between a (2 nc)^3 fine and an nc^3 coarse
 * grid for ncells x K fields (K = 3 or 18), FP64, layout [ncells][K][nodes]:
 * MAPLE_RESTRICT out = P^T in (fine in, coarse out); MAPLE_PROLONG_ADD
 * out += P in (coarse in, fine out).  P interpolates a fine node at an even
 * coordinate from its own coarse node and at an odd one half-and-half from
 * the two neighbours, per axis.  ProlongStencil.prolong / restrict_PT
 * (utils/EBE_GMG.py:38-79; weights of _build_prolongation_operator_robust,
 * EBE_GMG.py:531-647). */
enum { MAPLE_RESTRICT = 0, MAPLE_PROLONG_ADD = 1 };
int maple_transfer(int op, int nc, int K, int ncells, const double* in, double* out, maple_stream_t stream);

/* The fine-level elastic operator in element-batched form on the tensor
 * cores, kept to measure it against the stencil form the solver uses:
 * y = K(rho) u for FP32 u, y [B][6][3][N] of the density of the last mixed
 * maple_set_density of the elastic physics, as the reference applies it
 * (utils/EBE_GMG.py:412-430: gather u_e, Ke_e u_e by bmm, scatter back) but
 * with the contraction of all elements and load cases as one tcgen05 GEMM,
 * rows (cell, element, load case) x Ke0, TF32 operands with FP32
 * accumulation (about 1e-3 relative).  rows_work and out_work hold
 * B * N * 6 * 24 floats each (the gathered rows and the GEMM result).  N
 * must make B * N * 6 a multiple of 128 (cell size a multiple of 4).  Waits
 * for its stream; MAPLE_E_TIMEOUT if a pipeline wait ran out. */
int maple_matvec_ebe_tc(maple_ctx* ctx, const float* u, float* y, float* rows_work, float* out_work,
                        maple_stream_t stream);

/* Periodic k^3 box filter of [B][N] (main_IHD_v3.py:342-359). */
int maple_box_filter(int r, int ncells, int k, const double* in, double* out, maple_stream_t stream);

/* OC update: 60 bisection steps on lambda in [1e-12, 1e6] per cell
 * (main_IHD_v3.py:362-380).  volfrac [B] device, xnew [B][N]; stats [B][2]
 * = (max|dx|, mean|dx|) (nullable).  The bisection runs in one cooperative
 * launch whose blocks meet at grid barriers; every wait there is bounded.  The
 * call waits for its stream and returns MAPLE_E_TIMEOUT if a wait ran out
 * (xnew and stats are then incomplete); the context stays usable. */
int maple_oc_update(maple_ctx* ctx, const double* x, const double* dJdx, const double* volfrac, double move, double xmin,
                    double* xnew, double* stats, maple_stream_t stream);

/* The OC update of maple_oc_update without a context and without allocating
 * anything: for host applications that manage all device memory themselves
 * and cannot let a library call cudaMalloc.  Its scratch (partial sums,
 * statistics when stats is NULL, barrier counters) lives in one fixed 256 KiB
 * device array per GPU, held until the process exits.  N = elements per cell;
 * at most 8191 cells per call with stats given (5460 with stats NULL); larger
 * batches are rejected.  The first call on a device looks up the array's
 * address and keeps it for the life of the process: make that first call
 * before any stream capture, and do not use the library across a reset of the
 * device (cudaDeviceReset), which would leave the kept address stale.  Calls
 * share the array, so calls whose kernels overlap on the GPU race.  Like
 * maple_oc_update it waits for its stream at the end and returns
 * MAPLE_E_TIMEOUT if a grid-barrier wait ran out.  This entry point has no
 * counterpart in the reference. */
int maple_oc_update_noalloc(int N, int ncells, const double* x, const double* dJdx, const double* volfrac, double move,
                            double xmin, double* xnew, double* stats, maple_stream_t stream);

/* Testing aid for the bounded waits of the OC update: later OC updates
 * launched from the calling thread (maple_oc_update, maple_oc_update_noalloc,
 * maple_oc_step) give up a grid-barrier wait after max_polls polls (0 = the
 * default bound of 2^24 polls) and wait for phantom_blocks more blocks than
 * they launch, which never arrive.  With phantom_blocks > 0 every such call
 * returns MAPLE_E_TIMEOUT after its bounded waits; (0, 0) restores the normal
 * behaviour.  No counterpart in the reference. */
int maple_test_wait_limit(long long max_polls, int phantom_blocks);

/* One full OC iteration on device for every active cell (main_IHD_v3.py:
 * 620-716 with symmetry "none" and no manufacturing penalties): SIMP map,
 * both solves (as needed by the weights), C^H / kappa^H, objective
 * J = wE*E + wG*G + wK*trace(kappa) (utils/objective.py:11-41, 180-251),
 * analytic sensitivities, k^3 sensitivity filter and OC update.
 * x [B][N] in, x_next [B][N] out; weights [B][3] and volfrac [B] device.
 * Per-cell outputs (device, nullable): J [B], terms [B][3] (E, G, trace k),
 * CH [B][6][6], kappa [B][3][3], stats [B][2] (max|dx|, mean|dx|).  Waits
 * for its stream at the end; MAPLE_E_TIMEOUT as for maple_oc_update. */
int maple_oc_step(maple_ctx* ctx, const double* x, const double* weights, const double* volfrac, double penal,
                  double rho_min, double move, double xmin, int filter_k, int precision, double rtol, int maxit,
                  int warm, double* x_next, double* J, double* terms, double* CH, double* kappa, double* stats,
                  int* iters_out_host, maple_stream_t stream);

/* Initial iterate for the next warm-started solve: copies u [B][R][D][N]
 * (device, FP64) into the context's solution of `physics`, so that
 * maple_solve / maple_oc_step with warm = 1 start from it.  Takes the role of
 * GMGSolver.solve(init_list=...) (EBE_GMG.py:648-757, 851-858), where the
 * reference aligns network-predicted fields to the node order as initial u. */
int maple_set_solution(maple_ctx* ctx, int physics, const double* u, maple_stream_t stream);

/* Number of kernels this library has launched in this process (all
 * contexts); used to count device launches inside a timed region. */
unsigned long long maple_launch_count(void);

/* ---------------------------------------------------------------------------
 * Learned initial guess: periodic 3-D convolution network kernels.
 * No counterpart in the reference's FE path (its network-initialisation hook,
 * EBE_GMG.py:733-757, is fed by no network on the live path).
 *
 * Activations are channels-last [B][n^3][C] BF16 (voxel id x*n*n + y*n + z);
 * weights [taps][cin][cout] BF16, taps = 27 (3x3x3, tap = 9(dx+1)+3(dy+1)+dz+1)
 * or 1; bias [cout] FP32.  The guess network's convolutions are periodic
 * (circular padding); maple_nn_conv3d_padded also takes zero padding
 * (nn.Conv3d(padding=1), the Stage-II density generator's convolutions).
 * Errors: maple_nn_last_error_string().
 * ------------------------------------------------------------------------- */
enum { MAPLE_NN_POOL = 0, MAPLE_NN_UPSAMPLE = 1, MAPLE_NN_UPSAMPLE_ADJ = 2, MAPLE_NN_POOL_ADJ = 3 };
enum { MAPLE_NN_PAD_CIRCULAR = 0, MAPLE_NN_PAD_ZEROS = 1 };

const char* maple_nn_last_error_string(void);
unsigned long long maple_nn_launch_count(void);

/* out = act(conv(in, W) + bias + res); act = ReLU if relu.  out (BF16) and/or
 * out_f32 (FP32, same layout); bias and res nullable (res may alias out).
 * BF16 products with FP32 accumulation on the tensor cores. */
int maple_nn_conv3d(const void* in, const void* W, const float* bias, const void* res, void* out, float* out_f32,
                    int B, int n, int cin, int cout, int ksize, int relu, maple_stream_t stream);

/* maple_nn_conv3d with the padding mode MAPLE_NN_PAD_CIRCULAR or MAPLE_NN_PAD_ZEROS. */
int maple_nn_conv3d_padded(const void* in, const void* W, const float* bias, const void* res, void* out,
                           float* out_f32, int B, int n, int cin, int cout, int ksize, int relu, int padding,
                           maple_stream_t stream);

/* The convolutions of maple_nn_conv3d(_padded) run as an implicit GEMM on the
 * fifth-generation tensor cores (tcgen05.mma, FP32 accumulator in tensor
 * memory) when cin is a multiple of 8 and in / W are 16-byte aligned, else on
 * warp-level MMA.  Their pipeline waits are bounded: a wait that runs out
 * ends the kernel and sets a device flag.  maple_nn_wait_status waits for the
 * stream, returns that flag in *timed_out_host (0: no wait ran out since the
 * last call) and clears it.  No counterpart in the reference. */
int maple_nn_wait_status(int* timed_out_host, maple_stream_t stream);

/* dW += sum over cells and voxels of in(shifted by tap) x dz (FP32 [taps][cin][cout]);
 * db += sum of dz (nullable). */
int maple_nn_conv3d_wgrad(const void* in, const void* dz, float* dW, float* db, int B, int n, int cin, int cout,
                          int ksize, maple_stream_t stream);

/* Wt[taps-1-tap][co][ci] = W[tap][ci][co]: the weights whose forward
 * convolution of dz is the data gradient. */
int maple_nn_flip_weights(const void* W, void* Wt, int cin, int cout, int ksize, maple_stream_t stream);

/* 2x resampling between nc^3 and (2nc)^3 grids of C channels:
 * POOL (fine src -> coarse dst, mean of 8), UPSAMPLE (coarse src -> fine dst,
 * plus base if given), UPSAMPLE_ADJ (fine -> coarse, sum of 8), POOL_ADJ
 * (coarse -> fine, 1/8 each).  add != 0 accumulates into dst. */
int maple_nn_resample(int op, const void* src, const void* base, void* dst, int B, int nc, int C, int add,
                      maple_stream_t stream);

/* dst = src (+ dst when add) elementwise (BF16). */
int maple_nn_accumulate(void* dst, const void* src, size_t total, int add, maple_stream_t stream);

/* g = g * [y > 0] elementwise (BF16). */
int maple_nn_relu_mask(const void* y, void* g, size_t total, maple_stream_t stream);

/* loss += mean (pred - target)^2; grad = gscale * d loss / d pred (BF16, nullable). */
int maple_nn_mse(const float* pred, const void* target, void* grad, float* loss, size_t total, float gscale,
                 maple_stream_t stream);

/* Node weights w [B][n^3] FP32 of densities rho [B][n^3]: the mean density of
 * the 8 elements sharing a node over the cell's mean density (mean 1 per cell). */
int maple_nn_node_weights(const double* rho, float* w, int B, int n, maple_stream_t stream);

/* Weighted, offset-free squared error of pred [B][N][C] FP32 against target
 * (BF16): e = pred - target - ebar[b][c], ebar = weighted mean of pred - target
 * per cell and channel (computed into ebar [B][C] FP32; NULL: not removed);
 * loss += sum w e^2 / (B N C); grad = gscale * d loss / d pred (BF16,
 * nullable).  w [B][N] (NULL: 1).  C <= 64. */
int maple_nn_mse_weighted(const float* pred, const void* target, const float* w, float* ebar, void* grad, float* loss,
                          int B, int N, int C, float gscale, maple_stream_t stream);

/* Energy-norm training loss, in three steps around maple_matvec:
 * maple_nn_error_fields: e[b][f][v] = scale[f] * (pred - target)[b][v][c0+f]
 *   as an FP64 solver field [B][F][N] (scale device [F], NULL: 1);
 * maple_nn_block_dot: out[k] = sum_j a[k*len + j] * b[k*len + j], k < nblocks
 *   (with len = D*N: the per-(cell, load case) products e_r^T (K e)_r);
 * maple_nn_energy_grad: grad[b][v][c0 + r*D + d] = coef * scale[r*D+d] *
 *   y[b][r][d][v] / norm[b][r] (BF16), the gradient of
 *   coef/2 * sum e_r^T K e_r / norm[b][r] for y = K e. */
int maple_nn_error_fields(const float* pred, const void* target, const double* scale, double* e, int B, int N, int F,
                          int C, int c0, maple_stream_t stream);
int maple_nn_block_dot(const double* a, const double* b, double* out, int nblocks, size_t len, maple_stream_t stream);
int maple_nn_energy_grad(const double* y, const double* norm, const double* scale, void* grad, int B, int N, int R,
                         int D, int C, int c0, double coef, maple_stream_t stream);

/* *out = sum of g[i]^2 over n FP32 values (FP64 result, device). */
int maple_nn_sumsq(const float* g, size_t n, double* out, maple_stream_t stream);

/* One Adam step (bias-corrected, decoupled weight decay) on FP32 weights w
 * with gradient g / gscale; refreshes the BF16 copy wb (nullable). */
int maple_nn_adam(float* w, const float* g, float* m, float* v, void* wb, size_t total, float lr, float beta1,
                  float beta2, float eps, float weight_decay, float gscale, int step, maple_stream_t stream);

int maple_nn_to_bf16(const float* src, void* dst, size_t total, maple_stream_t stream);

/* Network input [B][N][C] BF16 from densities rho [B][N] FP64:
 * channel 0 = rho^(1/3), channel 1 = rho, others 0. */
int maple_nn_features(const double* rho, void* out, int B, int N, int C, maple_stream_t stream);

/* Training targets: out[b][v][c0+f] = scale[f] * (u[b][f][v] - mean_v u[b][f][.])
 * for F fields of a solver layout [B][F][N] (F = R*D).  mean_work [B*F] FP64
 * (NULL: no mean removal); scale [F] FP64 device (NULL: 1). */
int maple_nn_fields_to_channels(const double* u, double* mean_work, void* out, int B, int N, int F, int C, int c0,
                                const double* scale, maple_stream_t stream);

/* Initial iterates: u[b][f][v] = scale[f] * in[b][v][c0+f] (FP32 -> FP64);
 * scale [F] FP64 device (NULL: 1). */
int maple_nn_channels_to_fields(const float* in, double* u, int B, int N, int F, int C, int c0, const double* scale,
                                maple_stream_t stream);

/* Trilinear prolongation of periodic nodal fields [BF][nc^3] -> [BF][(factor*nc)^3]. */
int maple_nn_prolong_fields(const double* uc, double* uf, int BF, int nc, int factor, maple_stream_t stream);

/* Block average of element densities [B][(factor*nc)^3] -> [B][nc^3]. */
int maple_nn_restrict_density(const double* rf, double* rc, int B, int nc, int factor, maple_stream_t stream);

/* ---------------------------------------------------------------------------
 * Stage-II density generator inference and warm-start post-processing of the
 * Pareto dataset worker.  The generator is core/stage2/density_generator.py:
 * 123-197 (Stage2DensityGenerator.encode_latent / decode_latent); its 3x3x3
 * convolutions are maple_nn_conv3d_padded(..., MAPLE_NN_PAD_ZEROS).  FP32
 * unless stated.  Errors: maple_gen_last_error_string().
 * ------------------------------------------------------------------------- */
const char* maple_gen_last_error_string(void);
unsigned long long maple_gen_launch_count(void);

/* y[rows][out] = x[rows][in] W^T + b (nn.Linear; W [out][in]; b nullable);
 * SiLU after it when act. */
int maple_gen_linear(const float* x, const float* W, const float* b, float* y, int rows, int in, int out, int act,
                     maple_stream_t stream);

/* nn.LayerNorm(dim, eps) of each row (gamma, beta nullable); SiLU after it when act. */
int maple_gen_layernorm(const float* x, const float* gamma, const float* beta, float* y, int rows, int dim, float eps,
                        int act, maple_stream_t stream);

/* nn.Upsample(scale_factor=2, mode="trilinear", align_corners=False) of an
 * n^3 grid of C channels read at in[b*cell_stride + v*voxel_stride +
 * c*channel_stride] (v = x*n*n + y*n + z) into channels-last BF16
 * out[B][(2n)^3][C]. */
int maple_gen_upsample2(const float* in, long long cell_stride, long long voxel_stride, long long channel_stride,
                        void* out, int B, int n, int C, maple_stream_t stream);

/* nn.GroupNorm(groups, C, eps) of channels-last x[B][N][C] (gamma, beta
 * nullable), SiLU after it when act, into out_bf16 (BF16) and/or out_f32.
 * stats: B*groups*2 doubles of workspace. */
int maple_gen_groupnorm(const float* x, const float* gamma, const float* beta, int groups, float eps, int act,
                        void* out_bf16, float* out_f32, double* stats, int B, long long N, int C,
                        maple_stream_t stream);

/* out[B][N] = sigmoid(bias + sum_c w[c] x[B][N][c]) (1x1x1 conv to one channel). */
int maple_gen_head_sigmoid(const float* x, const float* w, float bias, float* out, int B, long long N, int C,
                           maple_stream_t stream);

/* binomial_smooth_periodic_torch (pareto/densify_pareto_property_network_32.py:
 * 1040-1052): `passes` times, along x, y, z, the periodic [1 4 6 4 1]/16
 * filter, bit-identical to the reference's FP32 operation order.  in, out and
 * work ([B][n^3] each) distinct; passes = 0 copies in to out. */
int maple_gen_binomial_smooth(const float* in, float* out, float* work, int B, int n, int passes,
                              maple_stream_t stream);

/* match_mean_clamped_torch (same file, 1031-1037), per cell in place:
 * max(1, iters) times x <- clamp(x - mean(x) + clamp(target[b], lo, hi), lo, hi)
 * (target FP64 device array [B]; the mean is summed in FP64). */
int maple_gen_match_mean(float* x, const double* target, int B, long long N, float lo, float hi, int iters,
                         maple_stream_t stream);

/* Instrumentation: when enabled, every fine-level operator launch of this
 * context is bracketed by CUDA events (at most max_launches are kept).
 * maple_profile_read writes a JSON object {kernel class: {launches, total_ms,
 * bytes_per_launch}} into buf, bytes_per_launch being the algorithmic bytes
 * (each input read once, each output written once). */
int maple_profile_enable(maple_ctx* ctx, int enable, int max_launches);
int maple_profile_read(maple_ctx* ctx, char* buf, int buflen);

#ifdef __cplusplus
}
#endif

#endif /* MAPLE_B200_H */
