// Manufacturability penalties of the OC objective (utils/printability.py):
// the overhang penalty and the trapped-void (cavity) penalty of a single
// periodic cell or of a finite periodic array, with their gradients w.r.t. the
// element densities.  The gradients follow the tie rules of the autograd the
// reference differentiates them with: a max-pool window passes its gradient to
// its first maximum in scan order, torch.minimum splits it in half between
// equal arguments, relu passes nothing at 0.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace maple_pr {

// utils/printability.py:91-134; build direction +z, lateral support radius rad
struct OverhangPlan {
  int r = 0, B = 0, rad = 1, periodic = 1;
  size_t bytes() const;  // workspace
};

// utils/printability.py:139-323
enum SeedFaces { SEED_ALL = 0, SEED_X = 1, SEED_Y = 2, SEED_Z = 3, SEED_XY = 4 };
struct CavityPlan {
  int r = 0, B = 0;
  int tiles[3] = {1, 1, 1};
  int periodic = 1;         // flood fill wraps around (single cell only)
  int min_channel_rad = 0;  // opening radius before the flood fill
  int rad = 1;              // flood-fill window radius (0: no flood fill)
  int nsteps = 0;           // flood-fill steps
  int seed = SEED_ALL;
  int focus_center = 1;     // arrays of >= 3 tiles per axis: penalty over the centre tile only
  double void_thresh = 0.5, beta = 20.0;
  int dims(int a) const { return tiles[a] * r; }
  size_t M() const { return (size_t)dims(0) * dims(1) * dims(2); }
  bool focused() const { return focus_center && tiles[0] >= 3 && tiles[1] >= 3 && tiles[2] >= 3; }
  size_t bytes() const;  // workspace
};

// P [B] (device) and, if grad != nullptr, dP/drho [B][r^3] (device).
// work: a device buffer of plan.bytes(); launches on s; throws std::runtime_error
// on invalid plans.
void overhang(const double* rho, const OverhangPlan& plan, double* P, double* grad, void* work, cudaStream_t s);
void cavity(const double* rho, const CavityPlan& plan, double* P, double* grad, void* work, cudaStream_t s);

// kernels launched by the two calls above (for launch accounting)
unsigned long long launches();

}  // namespace maple_pr
