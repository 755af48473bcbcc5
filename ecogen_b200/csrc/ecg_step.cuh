// Fused Kapila (PUEq) step kernels for uniform Cartesian meshes.
//
// One kernel launch performs one face-flux pass plus the cell update that follows it:
//   PASS_O1   first order: fluxes on S^n, U^{n+1} = U^n + dt*sum F, buildPrim, relaxation,
//             energy correction                           (Run::solveHyperbolic + solveRelaxations)
//   PASS_PRED MUSCL predictor: fluxes of the reconstructed S^n, U^{n+1/2} = U^n + dt/2*sum F,
//             buildPrim, relaxation, energy correction     (CellO2::predictionOrdre2, src/Order2/CellO2.cpp:111)
//   PASS_CORR MUSCL corrector: fluxes of the reconstructed S^{n+1/2}, U^{n+1} = U^n + dt*sum F,
//             buildPrim, relaxation, energy correction     (Run::solveHyperbolicO2 steps 6-8 + solveRelaxations)
//
// Work decomposition.  A block owns a tile of cells (TX x TY x TZ, one thread per cell).  For
// each axis in turn it stages the tile plus a halo of H cells along that axis in shared
// memory (H = 1 first order, 2 MUSCL), computes every face slope once, then every face flux of
// the tile once (one thread per face), and each cell thread accumulates its two faces of that
// axis in the reference order (left face added, right face subtracted,
// CellInterface::addFlux/subtractFlux src/Order1/CellInterface.cpp:267-297).  Boundary faces
// come last in the order Xm, Xp, Ym, Yp, Zm, Zp, as MeshCartesian enumerates them
// (src/Meshes/MeshCartesian.cpp:384-557).  Accumulation therefore happens in exactly the
// reference's order, with no atomics: each cell is written by one thread.
#pragma once
#include "ecg_device.cuh"


namespace ecg {

enum { PASS_O1 = 0, PASS_PRED = 1, PASS_CORR = 2 };

// Cells of a block's tile and threads of the block.  Face fluxes are computed one per thread, so
// the tiles are shaped for every axis to have at most THREADS faces ((X+1)*Y*Z, X*(Y+1)*Z,
// X*Y*(Z+1)): each face pass then takes a single round and no warp waits at the following barrier
// for a partial second round.  MINB is the number of resident blocks per SM asked of the compiler
// (__launch_bounds__), which caps registers at 65536 / (THREADS * MINB): the kernels are bound by
// FP64 latency, and more resident warps beat the spills this costs.  Measured on the 2048^2
// two-phase MUSCL step (cell-updates/s): 16x15 / 256 threads / 2 blocks (128 registers) 652 M;
// 16x15 / 256 / 3 (80) 825 M; 16x15 / 256 / 4 (64) 790 M; 8x14 / 128 / 6 (80) 849 M;
// 8x14 / 128 / 7 (72) 949 M; 8x14 / 128 / 8 (64) 883 M; 16x7 / 128 / 7 868 M; 8x7 / 64 / 14 719 M.
// 1D single cases (the 1000-cell tube of the reference's CPU-sized configuration) run a few blocks
// and are latency-bound: fewer spills matter more than resident warps.  Measured on that tube
// (cell-updates/s): 3 blocks per SM (80 registers) 48.6 M, 2 (128 registers) 51.8 M, 1 52.8 M.
#ifndef ECG_TILE1D_MINB
#define ECG_TILE1D_MINB 2
#endif
#ifndef ECG_TILE2D_X
#define ECG_TILE2D_X 8
#define ECG_TILE2D_Y 14
#define ECG_TILE2D_THREADS 128
#endif
#ifndef ECG_TILE2D_MINB
#define ECG_TILE2D_MINB 7
#endif
#ifndef ECG_TILE3D_X
#define ECG_TILE3D_X 6
#define ECG_TILE3D_Y 6
#define ECG_TILE3D_Z 6
#define ECG_TILE3D_THREADS 256
#endif
#ifndef ECG_TILE3D_MINB
#define ECG_TILE3D_MINB 2
#endif
// Resident blocks asked for the 2D p-T-mu kernels (0: the tile shape's MINB).  Their saturation
// solve makes them larger than the other Kapila kernels: at 7 blocks (72 registers) they spilled
// 1.4 KB a thread and wrote 4-6x the algorithmic bytes to DRAM.  Measured on the 1024^2 expansion
// (cell-updates/s): 7 blocks 360 M, 6 370 M, 5 388 M, 4 (128 registers) 389 M.
#ifndef ECG_PTMU_MINB
#define ECG_PTMU_MINB 4
#endif
template <int DIM>
struct TileShape;
template <>
struct TileShape<1> { static constexpr int X = 255, Y = 1, Z = 1, THREADS = 256, MINB = ECG_TILE1D_MINB; };
template <>
struct TileShape<2> {
  static constexpr int X = ECG_TILE2D_X, Y = ECG_TILE2D_Y, Z = 1, THREADS = ECG_TILE2D_THREADS, MINB = ECG_TILE2D_MINB;
};
template <>
struct TileShape<3> {
  static constexpr int X = ECG_TILE3D_X, Y = ECG_TILE3D_Y, Z = ECG_TILE3D_Z, THREADS = ECG_TILE3D_THREADS,
                       MINB = ECG_TILE3D_MINB;
};

// Field indices of a state array (stride = ncells):
//   alpha_k [0,NP), rho_k [NP,2NP), p 2NP, u_d 2NP+1+d, E 2NP+1+DIM
template <int NP, int DIM>
struct Fields {
  static constexpr int A = 0, R = NP, P = 2 * NP, U = 2 * NP + 1, E = 2 * NP + 1 + DIM;
  static constexpr int NQ = 2 * NP + 1 + DIM;    // primitive fields used by fluxes
  static constexpr int NS = NQ + 1;              // full state (with E)
  static constexpr int NSL = 3 * NP + DIM;       // slope components: alpha_k, rho_k, p_k, u_d
  static constexpr int NFL = 3 * NP + DIM + 3;   // flux components: a_k, m_k, e_k, mom_d, E, sM, uStar
};

// Device scalars of a context's time loop (Run::solver src/Run.cpp:385-490).
struct DevScalars {
  double dt;                       // step being taken (1e-15 before the first step, src/Run.cpp:38)
  double t;                        // physical time
  double cfl;
  double t_end;
  unsigned long long dtmax_bits;   // min over faces of lCFL/|s|, as ordered bits of a positive double
  long long it, max_it;
  int mode;                        // 0: free stepping, 1: stop after max_it, 2: stop once t >= t_end
  int done;                        // set once the stop condition holds; later steps are no-ops
};

struct StepParams {
  const int* done;      // device flag: skip the launch when set
  const double* q;      // primitives the fluxes are built from (S^n, or S^{n+1/2} in the corrector)
  const double* sn;     // S^n (U^n, non-conservative terms, time-n alpha_0 of neighbours)
  double* out;          // S^{n+1/2} (predictor) or S^{n+1}
  int64_t n;            // cells
  const double* dt;     // device scalar: current time step
  unsigned long long* dtmax_bits;  // device scalar: min over faces of lCFL/|s| as ordered bits
  DevStats* stats;
  int lim[4];
  int newton_cap;
  int newton_accept;  // 1: a relaxation that reaches the cap keeps its last iterate (no fallback)
  // learned seed (optional)
  const struct MlpDev* mlp;  // installed model (nullptr = plain start)
  // recording of (features, converged pressure) pairs of relaxations with at least rec_min_evals
  // Newton evaluations
  float* rec_x;
  float* rec_y;
  unsigned long long* rec_count;
  unsigned long long rec_max;
  int rec_min_evals;
  // p-T-mu relaxation
  int ptmu, ptmu_liq, ptmu_vap;
  double pcrit;
  int ptmu_seed_p;  // seeded p-T-mu: 1 = the network's p* starts the saturation Newton too (else T only)
  double* tsat_hist;  // p-T-mu warm start: per-cell T_sat of the cell's last saturation solve (nullptr: off)
  // THINC reconstruction of alpha (a volume-fraction limiter is THINC): cosh and tanh of the
  // sharpness beta = 1.6, evaluated once on the host like the reference does
  int thinc;
  double thinc_cosh, thinc_tanh;
  // passive transports: stored after the NS fields of a state (at NS + j), j < ntr
  int ntr;
  // analytic pressure-temperature relaxation after the pressure one (two phases)
  int pt;
  // split form of a 2D / 3D pass (ecg_kapila_split.cuh): face-flux arrays per axis (nullptr: the fused
  // kernels run), and optional events recorded after each axis' face kernel (profiling)
  double* flux[3];
  cudaEvent_t* split_ev;
  // host side: tensor maps of the face kernels' TMA staging (nullptr: the kernels load their tiles)
  const struct FaceMaps* fmaps;
};

// Host side of the THINC parameters (CellInterfaceO2Cartesian::solveRiemann's beta = 1.6).
inline void set_thinc(StepParams& P, const ecg_case& c) {
  P.thinc = (c.order == 2 && (c.limiter[2] == ECG_LIM_THINC || c.limiter[3] == ECG_LIM_THINC)) ? 1 : 0;
  P.thinc_cosh = std::cosh(1.6);
  P.thinc_tanh = std::tanh(1.6);
}

// CFL length of cell (i, j, k): the smallest size along the used axes, x 0.6 beyond 1D
// (MeshCartesian::initializeGeometrieMonoCpu src/Meshes/MeshCartesian.cpp:232-238); the same for every
// cell of a uniform mesh.
__device__ __forceinline__ double cell_lcfl(const Geometry& G, int i, int j, int k) {
  if (!G.stretched) return G.lcfl;
  double l = 1.e10;
  if (G.n[0] != 1) l = dmin(l, G.dsz[0][i]);
  if (G.n[1] != 1) l = dmin(l, G.dsz[1][j]);
  if (G.n[2] != 1) l = dmin(l, G.dsz[2][k]);
  if (G.dim > 1) l *= 0.6;
  return l;
}

// Face surface over cell volume for the faces of cell (i, j, k) normal to axis ax: the coefA of
// CellInterface::addFlux / subtractFlux (src/Order1/CellInterface.cpp:269, :287), surface dY dZ (X
// faces), dX dZ (Y faces) or dX dY (Z faces) over the volume dX dY dZ (:226, :287, :320, :353).
__device__ __forceinline__ double cell_coefA(const Geometry& G, int ax, int i, int j, int k) {
  if (!G.stretched) return G.coefA[ax];
  const double dx = G.dsz[0][i], dy = G.dsz[1][j], dz = G.dsz[2][k];
  const double vol = dx * dy * dz;
  const double s = (ax == 0) ? dy * dz : ((ax == 1) ? dx * dz : dx * dy);
  return ddiv(s, vol) * 1.;
}

// Bounds-checked builds (-DECG_BOUNDS_CHECK, libecg_bounds.so): every state, face-array and output
// access of the step kernels checks its linear index against its buffer; an index outside is counted
// in DevStats::bounds_violations and the access is skipped -- never a trap.  Regular builds compile the
// checks away.
#ifdef ECG_BOUNDS_CHECK
__device__ __forceinline__ bool ecg_in_bounds(DevStats* st, int64_t i, int64_t n) {
  if (i >= 0 && i < n) return true;
  atomicAdd(&st->bounds_violations, 1ull);
  return false;
}
#define ECG_IN_BOUNDS(st, i, n) ecg_in_bounds((st), (int64_t)(i), (int64_t)(n))
#else
#define ECG_IN_BOUNDS(st, i, n) true
#endif

// Faces normal to axis ax of a mesh of n cells per axis, the two domain sides of every line included
// (the face arrays of the split form).
__host__ __device__ inline int64_t split_nfaces(const int n[3], int ax) {
  return (int64_t)(n[0] + (ax == 0)) * (n[1] + (ax == 1)) * (n[2] + (ax == 2));
}

__device__ __forceinline__ void atomic_min_pos_double(unsigned long long* addr, double v) {
  // positive doubles order like their bit patterns
  atomicMin(addr, (unsigned long long)__double_as_longlong(v));
}


// Reduces the per-thread relaxation counters of a block (warp reductions, then shared atomics)
// and adds them to the device counters with one global atomic per counter and block.
// Every thread of the block must call it.
__device__ __forceinline__ void block_counters(DevStats* st, unsigned int relax, unsigned int iters,
                                               unsigned int fallback, unsigned int seeded, unsigned int rejected,
                                               unsigned int nonfinite, unsigned int ptmu, unsigned int max_iters,
                                               bool hist) {
  __shared__ unsigned int sc[24];
  const int tid = threadIdx.x;
  if (tid < 24) sc[tid] = 0u;
  __syncthreads();
  const unsigned full = 0xffffffffu;
  unsigned int v[7] = {relax, iters, fallback, seeded, rejected, nonfinite, ptmu};
#pragma unroll
  for (int i = 0; i < 7; i++) {
    unsigned int w = __reduce_add_sync(full, v[i]);
    if ((tid & 31) == 0 && w) atomicAdd(&sc[i], w);
  }
  unsigned int mx = __reduce_max_sync(full, max_iters);
  if ((tid & 31) == 0 && mx) atomicMax(&sc[7], mx);
  if (hist && relax) atomicAdd(&sc[8 + (iters < 16 ? (iters >= 1 ? iters - 1 : 0) : 15)], 1u);
  __syncthreads();
  if (tid < 24 && sc[tid]) {
    unsigned long long x = sc[tid];
    switch (tid) {
      case 0: atomicAdd(&st->relax_calls, x); break;
      case 1: atomicAdd(&st->newton_evals, x); break;
      case 2: atomicAdd(&st->newton_fallback, x); break;
      case 3: atomicAdd(&st->seeded, x); break;
      case 4: atomicAdd(&st->seed_rejected, x); break;
      case 5: atomicAdd(&st->nonfinite, x); break;
      case 6: atomicAdd(&st->ptmu_errors, x); break;
      case 7: atomicMax(&st->newton_max, x); break;
      default: atomicAdd(&st->hist[tid - 8], x); break;
    }
  }
}

// Reduces the p-T-mu iteration counts of a block (kernels with p-T-mu relaxation only) and adds them to
// the device counters, one global atomic per counter and block.  Every thread of the block must call it.
__device__ __forceinline__ void block_ptmu_counters(DevStats* st, unsigned int solve, unsigned int outer,
                                                    unsigned int tsat_calls, unsigned int tsat_iters,
                                                    unsigned int tsat_max, unsigned int seeded,
                                                    unsigned int rejected) {
  __shared__ unsigned int sp[24];
  const int tid = threadIdx.x;
  if (tid < 24) sp[tid] = 0u;
  __syncthreads();
  const unsigned full = 0xffffffffu;
  const unsigned int v[4] = {solve, outer, tsat_calls, tsat_iters};
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const unsigned int w = __reduce_add_sync(full, v[i]);
    if ((tid & 31) == 0 && w) atomicAdd(&sp[i], w);
  }
  const unsigned int ws = __reduce_add_sync(full, seeded), wr = __reduce_add_sync(full, rejected);
  if ((tid & 31) == 0 && ws) atomicAdd(&sp[22], ws);
  if ((tid & 31) == 0 && wr) atomicAdd(&sp[23], wr);
  const unsigned int mo = __reduce_max_sync(full, solve ? outer : 0u), mt = __reduce_max_sync(full, tsat_max);
  if ((tid & 31) == 0) {
    if (mo) atomicMax(&sp[4], mo);
    if (mt) atomicMax(&sp[5], mt);
  }
  if (solve) atomicAdd(&sp[6 + (outer < 16 ? (outer >= 1 ? outer - 1 : 0) : 15)], 1u);
  __syncthreads();
  if (tid < 24 && sp[tid]) {
    const unsigned long long x = sp[tid];
    switch (tid) {
      case 22: atomicAdd(&st->ptmu_seeded, x); break;
      case 23: atomicAdd(&st->ptmu_seed_rejected, x); break;
      case 0: atomicAdd(&st->ptmu_solves, x); break;
      case 1: atomicAdd(&st->ptmu_outer, x); break;
      case 2: atomicAdd(&st->ptmu_tsat_calls, x); break;
      case 3: atomicAdd(&st->ptmu_tsat_iters, x); break;
      case 4: atomicMax(&st->ptmu_outer_max, x); break;
      case 5: atomicMax(&st->ptmu_tsat_max, x); break;
      default: atomicAdd(&st->ptmu_hist[tid - 6], x); break;
    }
  }
}

}  // namespace ecg
