// One time step on caller-owned device buffers without allocating any device memory.
//
// Who needs it: codes that own every byte of device memory through their own allocator or memory
// pool (and forbid the CUDA runtime allocator), codes that must not allocate inside their time loop
// (allocation can synchronise the device and stall other streams), and codes that record the step
// into work that may not contain allocations.  ecg_create allocates a context (states, half-step
// buffer, tables, counters); this entry point instead keeps its scratch — the MUSCL half-step
// state, the distance tables, dt / dtMax scalars and counters — in one file-scope __device__ array
// of fixed size, so a call allocates nothing.  Every GPU that loads the library holds that array
// (sizeof(NoallocScratch), about 10 MB) until the process exits.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "ecg_internal.h"
#include "ecg_step.cuh"

namespace ecg {

cudaError_t kapila_launch(int np, int dim, bool ptmu, int pass, const StepParams& P, const Geometry& G,
                          const ecg_eos* eos, double eps, cudaStream_t s, bool prepare);
cudaError_t euler_launch(int dim, int pass, const StepParams& P, const Geometry& G, const ecg_eos* eos, double eps,
                         cudaStream_t s, bool prepare);
__global__ void k_finalize(DevScalars* s);

namespace {

constexpr int64_t kMaxCells = ECG_NOALLOC_MAX_CELLS;
constexpr int kMaxFields = 2 * ECG_MAX_PHASES + 1 + 3;  // primitive fields of the half-step state

struct NoallocScratch {
  DevScalars scal;
  DevStats stats;
  int done;
  int pad;
  double dist[9 * kMaxCells];           // per axis: centre-centre, face-left, face-right distances
  double half[kMaxFields * kMaxCells];  // MUSCL half-step primitives
};

}  // namespace

// The scratch.  In host code this name is only a handle: its device address comes from
// cudaGetSymbolAddress, once per device (noalloc_scratch below).
static __device__ __align__(256) NoallocScratch g_noalloc_scratch;

namespace {

std::mutex g_mu;
NoallocScratch* g_addr[64] = {};

// Device address of the scratch on the current device (looked up on the first call per device).
ecg_status noalloc_scratch(NoallocScratch** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    return ECG_ERR_CUDA;
  }
  if (dev < 0 || dev >= 64) {
    set_error("device index above 63");
    return ECG_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      set_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return ECG_ERR_CUDA;
    }
    g_addr[dev] = static_cast<NoallocScratch*>(p);
  }
  *out = g_addr[dev];
  return ECG_OK;
}

// Starts a call: scalars of this step, counters and stop flag cleared, and the distance tables of
// the case computed on the device with the same arithmetic as the host tables of ecg_create.
__global__ void k_noalloc_begin(NoallocScratch* S, double dt, double cfl, int n0, int n1, int n2, double l0, double l1,
                                double l2) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid == 0) {
    S->scal.dt = dt;
    S->scal.t = 0.;
    S->scal.cfl = cfl;
    S->scal.t_end = 0.;
    S->scal.dtmax_bits = (unsigned long long)__double_as_longlong(1.e10);
    S->scal.it = 0;
    S->scal.max_it = 0;
    S->scal.mode = 0;
    S->scal.done = 0;
    S->done = 0;
    S->stats = DevStats{};
  }
  const int n[3] = {n0, n1, n2};
  const double l[3] = {l0, l1, l2};
  int nmax = max(n0, max(n1, n2));
  for (int a = 0; a < 3; a++) {
    double d = l[a] / (double)n[a];
    for (int i = tid; i + 1 < n[a]; i += gridDim.x * blockDim.x) {
      double pl = (i + 0.5) * d, pr = (i + 1 + 0.5) * d, pf = pl + 0.5 * d;
      double x = pl - pr, y = pf - pl, z = pf - pr;
      S->dist[(3 * a + 0) * nmax + i] = sqrt(x * x);
      S->dist[(3 * a + 1) * nmax + i] = sqrt(y * y);
      S->dist[(3 * a + 2) * nmax + i] = sqrt(z * z);
    }
  }
}

}  // namespace
}  // namespace ecg

using namespace ecg;

extern "C" ecg_status ecg_step_noalloc(const ecg_case* c, const double* state_in, double* state_out, double dt,
                                       double* dt_next, ecg_step_stats* stats, void* stream) {
  // the cases ecg_create accepts, less the ones this entry point has no scratch or kernels for
  ecg_status vs = validate_case(c);
  if (vs != ECG_OK) return vs;
  if (c->model == ECG_MODEL_PTUEQ) {
    set_error("ecg_step_noalloc runs the Kapila and Euler models; use ecg_create / ecg_step for PTUEq");
    return ECG_ERR_UNSUPPORTED;
  }
  if (c->ntransports != 0) {
    set_error("ecg_step_noalloc runs without passive transports");
    return ECG_ERR_UNSUPPORTED;
  }
  if (case_stretched(*c)) {
    set_error("ecg_step_noalloc runs uniform meshes; use ecg_create / ecg_step for a stretched mesh");
    return ECG_ERR_UNSUPPORTED;
  }
  const int64_t n = (int64_t)c->ncells[0] * c->ncells[1] * c->ncells[2];
  if (n > kMaxCells) {
    set_error("ecg_step_noalloc: more than ECG_NOALLOC_MAX_CELLS (65536) cells; use ecg_create / ecg_step");
    return ECG_ERR_TOO_LARGE;
  }
  // the two states, nstate fields of n doubles each (the layout of ecg_create), must not overlap: the
  // kernels read neighbours of the input while they write the output
  const int dim0 = (c->ncells[0] != 1) + (c->ncells[1] != 1) + (c->ncells[2] != 1);
  const int64_t nstate = c->model == ECG_MODEL_EULER ? 3 + dim0 : 2 * c->nphases + 2 + dim0;
  const uintptr_t ib = reinterpret_cast<uintptr_t>(state_in), ob = reinterpret_cast<uintptr_t>(state_out);
  const uintptr_t bytes = (uintptr_t)(nstate * n) * sizeof(double);
  if (!state_in || !state_out || (ib < ob + bytes && ob < ib + bytes)) {
    set_error("ecg_step_noalloc: null or overlapping state buffers");
    return ECG_ERR_INVALID;
  }
  NoallocScratch* S = nullptr;
  ecg_status st = noalloc_scratch(&S);
  if (st != ECG_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int dim = (c->ncells[0] != 1) + (c->ncells[1] != 1) + (c->ncells[2] != 1);
  const bool euler = c->model == ECG_MODEL_EULER;
  const double eps = c->alpha_null ? 1.e-15 : 0.;
  // geometry: same formulas as ecg_create
  Geometry G{};
  const int nmax = std::max({c->ncells[0], c->ncells[1], c->ncells[2]});
  for (int a = 0; a < 3; a++) {
    G.n[a] = c->ncells[a];
    G.dcc[a] = S->dist + (size_t)(3 * a + 0) * nmax;
    G.dfl[a] = S->dist + (size_t)(3 * a + 1) * nmax;
    G.dfr[a] = S->dist + (size_t)(3 * a + 2) * nmax;
  }
  G.dim = dim;
  {
    std::vector<double> sz[3], ctr[3];  // uniform cells (stretched meshes are refused above)
    for (int a = 0; a < 3; a++) axis_cells(*c, a, sz[a], ctr[a]);
    side_geometry(*c, sz, ctr, G);
  }
  double dX = c->length[0] / (double)c->ncells[0], dY = c->length[1] / (double)c->ncells[1],
         dZ = c->length[2] / (double)c->ncells[2];
  double vol = dX * dY * dZ;
  G.coefA[0] = (dY * dZ) / vol;
  G.coefA[1] = (dX * dZ) / vol;
  G.coefA[2] = (dX * dY) / vol;
  double l = 1.e10;
  if (c->ncells[0] != 1) l = std::min(l, dX);
  if (c->ncells[1] != 1) l = std::min(l, dY);
  if (c->ncells[2] != 1) l = std::min(l, dZ);
  if (dim > 1) l *= 0.6;
  G.lcfl = l;

  StepParams P{};
  P.done = &S->done;
  P.n = n;
  P.dt = &S->scal.dt;
  P.dtmax_bits = &S->scal.dtmax_bits;
  P.stats = &S->stats;
  for (int i = 0; i < 4; i++) P.lim[i] = c->limiter[i];
  P.newton_cap = 100;
  set_thinc(P, *c);
  P.pt = c->pt_relaxation;
  P.ptmu = c->ptmu;
  P.ptmu_liq = c->ptmu_liquid;
  P.ptmu_vap = c->ptmu_vapor;
  if (c->ptmu) {
    const ecg_eos& L = c->eos[c->ptmu_liquid];
    const ecg_eos& V = c->eos[c->ptmu_vapor];
    double piL = L.type == ECG_EOS_IG ? 0. : L.pinf, piV = V.type == ECG_EOS_IG ? 0. : V.pinf;
    double pc = piL * (V.gamma - 1.) * V.cv - piV * (L.gamma - 1.) * L.cv;
    P.pcrit = pc / ((L.gamma - 1.) * L.cv - (V.gamma - 1.) * V.cv);
  }
  auto run = [&](int pass, bool prepare) -> cudaError_t {
    if (euler) return euler_launch(dim, pass, P, G, c->eos, eps, s, prepare);
    return kapila_launch(c->nphases, dim, c->ptmu != 0, pass, P, G, c->eos, eps, s, prepare);
  };
  for (int pass = 0; pass < 3; pass++) {
    cudaError_t e = run(pass, true);
    if (e == cudaErrorNotSupported) {
      set_error("no kernel built for this model / phases / dimension");
      return ECG_ERR_UNSUPPORTED;
    }
    if (e != cudaSuccess) {
      set_error(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
      return ECG_ERR_CUDA;
    }
  }
  k_noalloc_begin<<<64, 256, 0, s>>>(S, dt, c->cfl, c->ncells[0], c->ncells[1], c->ncells[2], c->length[0],
                                     c->length[1], c->length[2]);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    if (c->order == 1) {
      P.q = state_in;
      P.sn = state_in;
      P.out = state_out;
      e = run(PASS_O1, false);
    } else {
      P.q = state_in;
      P.sn = state_in;
      P.out = S->half;
      e = run(PASS_PRED, false);
      if (e == cudaSuccess) {
        P.q = S->half;
        P.out = state_out;
        e = run(PASS_CORR, false);
      }
    }
  }
  if (e == cudaSuccess) {
    k_finalize<<<1, 1, 0, s>>>(&S->scal);
    e = cudaGetLastError();
  }
  DevScalars r{};
  DevStats ds{};
  if (e == cudaSuccess) e = cudaMemcpyAsync(&r, &S->scal, sizeof(r), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&ds, &S->stats, sizeof(ds), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    set_error(std::string("ecg_step_noalloc: ") + cudaGetErrorString(e));
    return ECG_ERR_CUDA;
  }
  if (dt_next) *dt_next = r.dt;
  if (stats) stats_out(ds, n, stats);
  if (ds.ptmu_errors) {
    set_error("p-T-mu relaxation exceeded 50 iterations");
    return ECG_ERR_PHYSICS;
  }
  return ECG_OK;
}
