// Triangular-solve workspace and entry point (solve.cu).
#pragma once
#include "engine.hpp"

namespace mpir {

struct SolveWorkspace {
  DeviceBuffer zbuf;      // front vectors, zofs layout (doubles)
  DeviceBuffer part;      // backward partial sums (doubles)
  DeviceBuffer counters;  // backward completion counters, one per step desc
  void allocate(const Plan &P);
};

// Phases of the solve, combinable as bits.
enum SolvePhase : int { kForward = 1, kDiagonal = 2, kBackward = 4, kAllPhases = 7 };

// x (permuted order, float64, device) <- (L D L^T)^{-1} x, or the phases
// selected: (L+I)^{-1} x, Dinv .* x, (L+I)^{-T} x (qdldl.hpp:362-432).
void ldlt_solve(const Plan &P, const Numeric &F, double *x, SolveWorkspace &ws,
                cudaStream_t s, int phases = kAllPhases);

}  // namespace mpir
