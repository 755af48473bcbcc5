// Types shared by the host code and the kernels.
#pragma once
#include <cstdint>

#include "../../include/ecogen_b200.h"

namespace ecg {

// EOS parameters as the kernels use them (same fields as ecg_eos).
struct EosParams {
  int type;
  double gamma, pinf, b, cv, eref, sref;
};

// Geometry of a uniform Cartesian mesh, precomputed on the host with the reference's formulas
// (MeshCartesian::meshStretching src/Meshes/MeshCartesian.cpp:168 and
// initializeGeometrieMonoCpu :212-558) so that the kernels see the same doubles.
struct Geometry {
  int n[3];           // cells per axis
  int dim;            // number of axes with more than one cell
  double coefA[3];    // face surface / cell volume for faces normal to each axis
  double lcfl;        // CFL length of every cell (min of used sizes, x0.6 when dim > 1)
  // Distances used by the MUSCL reconstruction, per axis and face position (indexed by the
  // left cell i of face (i, i+1)): centre-to-centre, face-to-left-centre, face-to-right-centre.
  const double* dcc[3];
  const double* dfl[3];
  const double* dfr[3];
};

// Device counters filled by the step kernels.
struct DevStats {
  unsigned long long relax_calls, newton_evals, newton_fallback, seeded, seed_rejected, ptmu_errors, nonfinite;
  unsigned long long newton_max;
  unsigned long long hist[16];
};

}  // namespace ecg
