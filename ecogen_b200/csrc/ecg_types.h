// Types shared by the host code and the kernels.
#pragma once
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/ecogen_b200.h"

namespace ecg {

// EOS parameters as the kernels use them (same fields as ecg_eos).
struct EosParams {
  int type;
  double gamma, pinf, b, cv, eref, sref;
  // sendSpecialMixtureEos constants (src/Eos/EosSG.cpp:196): gamma*pInf/(gamma-1) (0 for IG) and
  // 1/(gamma-1), evaluated once on the host (IEEE division, the same value as in the kernels).
  double gpi, ig;
};

inline EosParams make_eos_params(const ecg_eos& e) {
  EosParams q{e.type, e.gamma, e.pinf, e.b, e.cv, e.eref, e.sref, 0., 0.};
  q.gpi = (e.type == ECG_EOS_IG) ? 0. : e.gamma * e.pinf / (e.gamma - 1.);
  q.ig = 1. / (e.gamma - 1.);
  return q;
}

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
  // Sides Xm, Xp, Ym, Yp, Zm, Zp (index 2*axis + plus): boundary condition, centre-minus-face
  // coordinate along the axis (Element::distanceX(Face*), divisor of a symmetry side's velocity
  // slope) and the signed centre-to-face distance of the MUSCL extrapolation towards that side
  // (negative on the minus sides, BoundCondWallO2Cartesian::solveRiemann).
  int bc[6];
  double wslope[6];
  double wdist[6];
  // Stretched meshes (mesh.xml meshStretching): cell sizes per axis and index; the kernels then take
  // each cell's own lCFL and surface / volume (cell_lcfl, cell_coefA) instead of lcfl and coefA.
  int stretched;
  const double* dsz[3];
};

// Fills the side fields of a Geometry with the reference's mesh arithmetic (cell centres and sizes of
// each axis as MeshCartesian::meshStretching computes them, minus faces at 0, plus faces at the last
// centre + its half size, src/Meshes/MeshCartesian.cpp:168, :402, :426).  sz / ctr: per axis, the cell
// sizes and centres.
inline void side_geometry(const ecg_case& c, const std::vector<double>* sz, const std::vector<double>* ctr,
                          Geometry& g) {
  for (int a = 0; a < 3; a++) {
    double p0 = ctr[a][0], pn = ctr[a][c.ncells[a] - 1];
    double fm = 0., fp = pn + 0.5 * sz[a][c.ncells[a] - 1];
    for (int side = 0; side < 2; side++) {
      double cen = side ? pn : p0, face = side ? fp : fm;
      double x = face - cen;
      double dist = std::sqrt(x * x + 0. * 0. + 0. * 0.);
      g.bc[2 * a + side] = c.bc[2 * a + side];
      g.wslope[2 * a + side] = cen - face;
      g.wdist[2 * a + side] = side ? dist : -dist;
    }
  }
}

// Device counters filled by the step kernels.
struct DevStats {
  unsigned long long relax_calls, newton_evals, newton_fallback, seeded, seed_rejected, ptmu_errors, nonfinite;
  unsigned long long newton_max;
  unsigned long long hist[16];
  // p-T-mu relaxation: saturation solves, their p* iterations (sum, max, histogram), T_sat solves and
  // their iterations (sum, max)
  unsigned long long ptmu_solves, ptmu_outer, ptmu_outer_max, ptmu_tsat_calls, ptmu_tsat_iters, ptmu_tsat_max;
  unsigned long long ptmu_hist[16];
  unsigned long long ptmu_seeded, ptmu_seed_rejected;
  unsigned long long bounds_violations;  // bounds-checked builds: accesses outside their buffer (skipped)
  unsigned long long staging_timeouts;   // face-kernel warps whose TMA staging wait ran out
};

}  // namespace ecg
