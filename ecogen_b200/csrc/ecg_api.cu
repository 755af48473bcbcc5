// C ABI: contexts, device state, the time loop and CUDA-graph capture of step sequences.
//
// A context owns, on one GPU, two copies of the state S (ping-pong: a step reads S^n and writes
// S^{n+1}), the MUSCL half-step state, the mesh distance tables, device scalars (dt, t, dtMax,
// stop flag) and counters, and one stream.  Every step is a fixed launch sequence
//   first order : step(O1) -> finalize
//   MUSCL       : step(PRED) -> step(CORR) -> finalize
// whose only data-dependent quantity (dt) lives in device memory, so sequences of steps are
// captured once as CUDA graphs and replayed without host round trips.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "ecg_internal.h"
#include "ecg_mlp_device.cuh"
#include "ecg_step.cuh"
#include "ecg_tma.cuh"

namespace ecg {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }

cudaError_t kapila_launch(int np, int dim, bool ptmu, int pass, const StepParams& P, const Geometry& G,
                          const ecg_eos* eos, double eps, cudaStream_t s, bool prepare);
cudaError_t euler_launch(int dim, int pass, const StepParams& P, const Geometry& G, const ecg_eos* eos, double eps,
                         cudaStream_t s, bool prepare);
cudaError_t ptueq_launch(int dim, int pass, const StepParams& P, const Geometry& G, const ecg_eos* eos, cudaStream_t s,
                         bool prepare);

__global__ void k_finalize(DevScalars* s) {
  // Run::solver src/Run.cpp:417-440: t += dt, iteration++, stop test, dt = cfl * dtMax
  if (s->done) return;
  double dtmax = __longlong_as_double((long long)s->dtmax_bits);
  s->t += s->dt;
  s->it += 1;
  if (s->mode == 1 && s->it >= s->max_it) s->done = 1;
  if (s->mode == 2 && s->t >= s->t_end) s->done = 1;
  s->dt = s->cfl * dtmax;
  s->dtmax_bits = (unsigned long long)__double_as_longlong(1.e10);
}

// Mixture pressure sum_k alpha_k p_k of the stored state (what the reference writes as
// Pressure_Mixture after fulfillState), optionally per-phase temperature and mass fraction.
__global__ void k_derived(const double* __restrict__ S, int64_t n, int np, int dim, ecg_eos e0, ecg_eos e1, ecg_eos e2,
                          double eps, double* pmix, double* T, double* Y) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const ecg_eos eos[3] = {e0, e1, e2};
  double p = S[(int64_t)(2 * np) * n + i];
  double a[ECG_MAX_PHASES], r[ECG_MAX_PHASES], pk[ECG_MAX_PHASES];
  double rho = 0., pm = 0.;
  for (int k = 0; k < np; k++) {
    a[k] = S[(int64_t)k * n + i];
    r[k] = S[(int64_t)(np + k) * n + i];
    EosParams q{eos[k].type, eos[k].gamma, eos[k].pinf, eos[k].b, eos[k].cv, eos[k].eref, eos[k].sref};
    pk[k] = eos_fix_p(q, p);
    rho += a[k] * r[k];
    pm += a[k] * pk[k];
  }
  if (pmix) pmix[i] = pm;
  for (int k = 0; k < np; k++) {
    EosParams q{eos[k].type, eos[k].gamma, eos[k].pinf, eos[k].b, eos[k].cv, eos[k].eref, eos[k].sref};
    if (T) T[(int64_t)k * n + i] = eos_T(q, eps, r[k], pk[k]);
    if (Y) Y[(int64_t)k * n + i] = a[k] * r[k] / dmax(rho, eps);
  }
}

// Temperature-pressure equilibrium model: phase densities computeDensity(p, T) (EosIG.cpp:85, EosSG.cpp:87),
// every phase's temperature (the mixture's) and mass fractions, from the state alpha_0, alpha_1, p, T, ...
__global__ void k_ptueq_derived(const double* __restrict__ S, int64_t n, ecg_eos e0, ecg_eos e1, double* rho,
                                double* T, double* Y) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const ecg_eos eos[2] = {e0, e1};
  const double p = S[2 * n + i], Tm = S[3 * n + i];
  double r[2], mix = 0.;
  for (int k = 0; k < 2; k++) {
    const double den = dmax(((eos[k].gamma - 1.) * eos[k].cv * Tm), 0.);
    r[k] = eos[k].type == ECG_EOS_IG ? p / den : (p + eos[k].pinf) / den;
    mix += S[(int64_t)k * n + i] * r[k];
  }
  for (int k = 0; k < 2; k++) {
    if (rho) rho[(int64_t)k * n + i] = r[k];
    if (T) T[(int64_t)k * n + i] = Tm;
    if (Y) Y[(int64_t)k * n + i] = S[(int64_t)k * n + i] * r[k] / mix;
  }
}

__global__ void k_euler_derived(const double* __restrict__ S, int64_t n, ecg_eos e0, double eps, double* T) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  EosParams q{e0.type, e0.gamma, e0.pinf, e0.b, e0.cv, e0.eref, e0.sref};
  T[i] = eos_T(q, eps, S[i], S[n + i]);
}

}  // namespace ecg

using namespace ecg;

struct ecg_ctx {
  ecg_case c;
  int dim = 1, np = 2, nstate = 0, nq = 0;
  int64_t n = 0;
  double eps = 0.;
  int device = 0;
  cudaStream_t stream = nullptr;
  double* state[2] = {nullptr, nullptr};
  double* half = nullptr;     // MUSCL half-step primitives
  double* dist = nullptr;     // distance tables (3 axes x 3 tables)
  double* tmp = nullptr;      // download scratch (mixture pressure)
  double* flux[3] = {nullptr, nullptr, nullptr};  // face arrays of the split form (Kapila 2D / 3D)
  bool split = false;         // step passes in split form (face kernels + cell kernel)
  FaceMaps fmaps{};           // tensor maps of the face kernels' TMA staging (fmaps.ok = 0: none)
  int staging = ECG_STAGING_TMA;
  DevScalars* scal = nullptr;
  DevStats* stats = nullptr;
  // pinned host staging of the scalars and counters an ecg_step call exchanges (asynchronous copies,
  // one synchronisation per call)
  DevScalars* h_scal = nullptr;
  DevStats* h_stats = nullptr;
  int cur = 0;
  int newton_cap = 100;
  int newton_accept = 0;
  int ptmu_seed_p = 0;  // ECG_PTMU_SEED_P_T: the network's p* starts the saturation Newton too
  double* tsat_hist = nullptr;  // p-T-mu warm start (ecg_set_ptmu_warm_start): T_sat of each cell's last solve
  MlpDev* mlp = nullptr;
  float* rec_x = nullptr;
  float* rec_y = nullptr;
  unsigned long long* rec_count = nullptr;
  unsigned long long rec_max = 0;
  int rec_min_evals = 1;
  double pcrit = 0.;
  Geometry geo{};
  cudaGraphExec_t graph[2] = {nullptr, nullptr};  // two-step sequences starting from state[0] / state[1]
  bool graph_dirty = true;
};

namespace {

ecg_status cuda_fail(cudaError_t e, const char* what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return ECG_ERR_CUDA;
}
#define ECG_CUDA(call)                                    \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);   \
  } while (0)

}  // namespace

namespace ecg {

}  // namespace ecg

namespace ecg {

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled() {
  static const EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

// The two maps (all primitive fields; field 0 alone) of buffer b for the face kernels of axis AX.
template <int AX>
static bool encode_axis(EncodeTiledFn enc, FaceMaps& m, int b, int dim, const cuuint64_t* gdim, const cuuint64_t* gstr,
                        int nq) {
  using FT = FaceTile<AX>;
  const cuuint32_t rank = (cuuint32_t)(dim + 1);
  cuuint32_t box[4], es[4] = {1, 1, 1, 1};
  for (int d = 0; d < dim; d++) box[d] = (cuuint32_t)FT::box(d);
  void* base = const_cast<double*>(m.buf[b]);
  for (int which = 0; which < 2; which++) {
    box[dim] = which == 0 ? (cuuint32_t)nq : 1u;
    CUtensorMap* out = which == 0 ? &m.q[b][AX] : &m.a0[b][AX];
    if (enc(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, rank, base, gdim, gstr, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
        CUDA_SUCCESS)
      return false;
  }
  return true;
}

bool build_face_maps(FaceMaps& m, const double* const bufs[3], int dim, const int n[3], int nq) {
  std::memset(&m, 0, sizeof(m));
  // 2D meshes are x-y meshes; a row of x cells must be a multiple of 16 bytes (tensor strides)
  if (dim < 2 || dim > 3 || (dim == 2 && n[2] != 1) || (n[0] & 1)) return false;
  const EncodeTiledFn enc = encode_tiled();
  if (!enc) return false;
  cuuint64_t gdim[4], gstr[3];
  gdim[0] = (cuuint64_t)n[0];
  gdim[1] = (cuuint64_t)n[1];
  if (dim == 3) gdim[2] = (cuuint64_t)n[2];
  gdim[dim] = (cuuint64_t)nq;
  gstr[0] = (cuuint64_t)n[0] * sizeof(double);
  if (dim == 3) gstr[1] = (cuuint64_t)n[0] * n[1] * sizeof(double);
  gstr[dim - 1] = (cuuint64_t)n[0] * n[1] * n[2] * sizeof(double);
  for (int b = 0; b < 3; b++) {
    m.buf[b] = bufs[b];
    if (!bufs[b]) continue;
    if (!encode_axis<0>(enc, m, b, dim, gdim, gstr, nq) || !encode_axis<1>(enc, m, b, dim, gdim, gstr, nq) ||
        (dim == 3 && !encode_axis<2>(enc, m, b, dim, gdim, gstr, nq))) {
      std::memset(&m, 0, sizeof(m));
      return false;
    }
  }
  m.ok = 1;
  return true;
}

}  // namespace ecg

namespace {

// Distances of the MUSCL reconstruction per axis, with the reference's arithmetic: cell centres
// (i + 0.5) * d, face position centre + 0.5 * d, lengths as Coord::norm of a difference
// (src/Meshes/Element.cpp:77-113, src/Maths/Coord.cpp:82).
// Then, per axis, the cell sizes (stretched meshes).
void distance_tables(const ecg_case& c, const std::vector<double>* sz, const std::vector<double>* ctr,
                     std::vector<double>& h) {
  int nmax = std::max({c.ncells[0], c.ncells[1], c.ncells[2]});
  h.assign(12 * (size_t)nmax, 0.);
  for (int a = 0; a < 3; a++) {
    for (int i = 0; i < c.ncells[a]; i++) h[(size_t)(9 + a) * nmax + i] = sz[a][i];
    for (int i = 0; i + 1 < c.ncells[a]; i++) {
      double pl = ctr[a][i], pr = ctr[a][i + 1], pf = pl + 0.5 * sz[a][i];
      double x = pl - pr, y = pf - pl, z = pf - pr;
      h[(size_t)(3 * a + 0) * nmax + i] = std::sqrt(x * x + 0. * 0. + 0. * 0.);
      h[(size_t)(3 * a + 1) * nmax + i] = std::sqrt(y * y + 0. * 0. + 0. * 0.);
      h[(size_t)(3 * a + 2) * nmax + i] = std::sqrt(z * z + 0. * 0. + 0. * 0.);
    }
  }
}

ecg_status launch_step(ecg_ctx* x, int parity, cudaEvent_t* ev = nullptr) {
  StepParams P{};
  P.done = &x->scal->done;
  P.n = x->n;
  P.dt = &x->scal->dt;
  P.dtmax_bits = &x->scal->dtmax_bits;
  P.stats = x->stats;
  for (int i = 0; i < 4; i++) P.lim[i] = x->c.limiter[i];
  P.newton_cap = x->newton_cap;
  P.newton_accept = x->newton_accept;
  P.mlp = x->mlp;
  P.rec_x = x->rec_x;
  P.rec_y = x->rec_y;
  P.rec_count = x->rec_count;
  P.rec_max = x->rec_max;
  P.rec_min_evals = x->rec_min_evals;
  P.ntr = x->c.ntransports;
  P.pt = x->c.pt_relaxation;
  set_thinc(P, x->c);
  P.ptmu = x->c.ptmu;
  P.ptmu_liq = x->c.ptmu_liquid;
  P.ptmu_vap = x->c.ptmu_vapor;
  P.pcrit = x->pcrit;
  P.ptmu_seed_p = x->ptmu_seed_p;
  P.tsat_hist = x->tsat_hist;
  for (int a = 0; a < 3; a++) P.flux[a] = x->split ? x->flux[a] : nullptr;
  P.fmaps = (x->split && x->staging == ECG_STAGING_TMA && x->fmaps.ok) ? &x->fmaps : nullptr;
  double* sn = x->state[parity];
  double* s1 = x->state[1 - parity];
  const bool euler = x->c.model == ECG_MODEL_EULER;
  const bool ptueq = x->c.model == ECG_MODEL_PTUEQ;
  auto run = [&](int pass) -> cudaError_t {
    if (euler) return euler_launch(x->dim, pass, P, x->geo, x->c.eos, x->eps, x->stream, false);
    if (ptueq) return ptueq_launch(x->dim, pass, P, x->geo, x->c.eos, x->stream, false);
    return kapila_launch(x->np, x->dim, x->c.ptmu != 0, pass, P, x->geo, x->c.eos, x->eps, x->stream, false);
  };
  cudaError_t e;
  if (ev) cudaEventRecord(ev[0], x->stream);
  if (x->c.order == 1) {
    P.q = sn;
    P.sn = sn;
    P.out = s1;
    P.split_ev = (ev && x->split) ? ev + 4 : nullptr;
    e = run(PASS_O1);
    if (e != cudaSuccess) return cuda_fail(e, "step kernel");
    if (ev) cudaEventRecord(ev[1], x->stream);
  } else {
    P.q = sn;
    P.sn = sn;
    P.out = x->half;
    P.split_ev = (ev && x->split) ? ev + 4 : nullptr;  // after each axis' face kernel (profiling)
    e = run(PASS_PRED);
    if (e != cudaSuccess) return cuda_fail(e, "predictor kernel");
    if (ev) cudaEventRecord(ev[1], x->stream);
    P.q = x->half;
    P.out = s1;
    P.split_ev = (ev && x->split) ? ev + 7 : nullptr;
    e = run(PASS_CORR);
    if (e != cudaSuccess) return cuda_fail(e, "corrector kernel");
  }
  if (ev) cudaEventRecord(ev[2], x->stream);
  k_finalize<<<1, 1, 0, x->stream>>>(x->scal);
  if (ev) cudaEventRecord(ev[3], x->stream);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "finalize kernel");
  return ECG_OK;
}

void drop_graphs(ecg_ctx* x) {
  for (int i = 0; i < 2; i++)
    if (x->graph[i]) {
      cudaGraphExecDestroy(x->graph[i]);
      x->graph[i] = nullptr;
    }
  x->graph_dirty = false;
}

// Captures two consecutive steps starting from state[parity] (the pair returns to state[parity]).
ecg_status build_graph(ecg_ctx* x, int parity) {
  cudaGraph_t g = nullptr;
  ECG_CUDA(cudaStreamBeginCapture(x->stream, cudaStreamCaptureModeThreadLocal));
  ecg_status s1 = launch_step(x, parity);
  ecg_status s2 = (s1 == ECG_OK) ? launch_step(x, 1 - parity) : s1;
  cudaError_t e = cudaStreamEndCapture(x->stream, &g);
  if (s2 != ECG_OK) {
    if (g) cudaGraphDestroy(g);
    return s2;
  }
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(&x->graph[parity], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
  return ECG_OK;
}

ecg_status advance(ecg_ctx* x, int nsteps) {
  if (x->graph_dirty) drop_graphs(x);
  while (nsteps >= 2) {
    if (!x->graph[x->cur]) {
      ecg_status s = build_graph(x, x->cur);
      if (s != ECG_OK) return s;
    }
    ECG_CUDA(cudaGraphLaunch(x->graph[x->cur], x->stream));
    nsteps -= 2;
  }
  if (nsteps == 1) {
    ecg_status s = launch_step(x, x->cur);
    if (s != ECG_OK) return s;
    x->cur = 1 - x->cur;
  }
  return ECG_OK;
}

}  // namespace

namespace ecg {
void stats_out(const DevStats& d, int64_t updates, ecg_step_stats* st) {
  std::memset(st, 0, sizeof(*st));
  st->cell_updates = updates;
  st->relax_calls = (int64_t)d.relax_calls;
  st->newton_evals = (int64_t)d.newton_evals;
  st->newton_fallback = (int64_t)d.newton_fallback;
  st->newton_max = (int64_t)d.newton_max;
  st->seeded = (int64_t)d.seeded;
  st->seed_rejected = (int64_t)d.seed_rejected;
  st->ptmu_errors = (int64_t)d.ptmu_errors;
  st->nonfinite_cells = (int64_t)d.nonfinite;
  for (int i = 0; i < 16; i++) st->newton_hist[i] = (int64_t)d.hist[i];
  st->ptmu_solves = (int64_t)d.ptmu_solves;
  st->ptmu_outer_iters = (int64_t)d.ptmu_outer;
  st->ptmu_outer_max = (int64_t)d.ptmu_outer_max;
  st->ptmu_tsat_calls = (int64_t)d.ptmu_tsat_calls;
  st->ptmu_tsat_iters = (int64_t)d.ptmu_tsat_iters;
  st->ptmu_tsat_max = (int64_t)d.ptmu_tsat_max;
  for (int i = 0; i < 16; i++) st->ptmu_outer_hist[i] = (int64_t)d.ptmu_hist[i];
  st->ptmu_seeded = (int64_t)d.ptmu_seeded;
  st->ptmu_seed_rejected = (int64_t)d.ptmu_seed_rejected;
  st->bounds_violations = (int64_t)d.bounds_violations;
  st->staging_timeouts = (int64_t)d.staging_timeouts;
}
}  // namespace ecg

namespace {

}  // namespace

namespace ecg {

// B fragments of the seed model's two hidden layers (layout of MlpDev, ecg_mlp_device.cuh).  Packed
// parameters: w1 b1 w2 b2 w3 b3 in_shift in_scale out_shift out_scale, then for a second output
// w3b b3b out_shift_1 out_scale_1.
__global__ void k_mlp_pack(const float* __restrict__ W, int nin, int nout, MlpDev* out) {
  const int H = MLP_H;
  const float* w1 = W;
  const float* b1 = w1 + H * nin;
  const float* w2 = b1 + H;
  const float* b2 = w2 + H * H;
  const float* w3 = b2 + H;
  const float* b3 = w3 + H;
  const float* ish = b3 + 1;
  const float* isc = ish + nin;
  const float* w3b = isc + nin + 2;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  for (int i = tid; i < 8 * 32; i += nth) {
    const int nt = i / 32, lane = i % 32, g = lane >> 2, t = lane & 3, n = 8 * nt + g;
    auto word = [&](int j) {
      const float lo = (2 * j < nin) ? w1[n * nin + 2 * j] : 0.f, hi = (2 * j + 1 < nin) ? w1[n * nin + 2 * j + 1] : 0.f;
      return pack_bf16(lo, hi);
    };
    out->w1[nt][lane] = make_uint2(word(t), word(t + 4));
  }
  for (int i = tid; i < 8 * 4 * 32; i += nth) {
    const int nt = i / 128, kc = (i / 32) % 4, lane = i % 32, g = lane >> 2, t = lane & 3, n = 8 * nt + g;
    const int j0 = kc * 8 + t, j1 = j0 + 4;
    out->w2[nt][kc][lane] = make_uint2(pack_bf16(w2[n * H + 2 * j0], w2[n * H + 2 * j0 + 1]),
                                       pack_bf16(w2[n * H + 2 * j1], w2[n * H + 2 * j1 + 1]));
  }
  for (int i = tid; i < H; i += nth) {
    out->b1[i] = b1[i];
    out->b2[i] = b2[i];
    out->w3[i] = w3[i];
    out->w3b[i] = nout > 1 ? w3b[i] : 0.f;
  }
  for (int i = tid; i < 16; i += nth) {
    out->ish[i] = i < nin ? ish[i] : 0.f;
    out->isc[i] = i < nin ? isc[i] : 0.f;
  }
  if (tid == 0) {
    out->b3 = b3[0];
    out->osh = isc[nin];
    out->osc = isc[nin + 1];
    out->pad = 0.f;
    out->b3b = nout > 1 ? w3b[H] : 0.f;
    out->osh2 = nout > 1 ? w3b[H + 1] : 0.f;
    out->osc2 = nout > 1 ? w3b[H + 2] : 0.f;
    out->pad2 = 0.f;
  }
}

cudaError_t mlp_install(const float* d_params, int nin, int nout, MlpDev* d_out, cudaStream_t stream) {
  k_mlp_pack<<<4, 256, 0, stream>>>(d_params, nin, nout, d_out);
  return cudaGetLastError();
}

ecg_status mlp_upload(const ecg_mlp* m, int np, bool ptmu, MlpDev** dev, cudaStream_t stream) {
  const int nout = m->n_out > 1 ? m->n_out : 1;
  if (ptmu ? (m->hidden != ECG_MLP_HIDDEN || m->n_in != PTMU_NIN || nout != 2)
           : (m->hidden != ECG_MLP_HIDDEN || m->n_in != 3 * np || nout != 1)) {
    set_error(ptmu ? "p-T-mu seed model shape must be 8 -> 64 -> 64 -> 2"
                   : "seed model shape must be 3*nphases -> 64 -> 64 -> 1");
    return ECG_ERR_INVALID;
  }
  const int nin = m->n_in, H = ECG_MLP_HIDDEN;
  std::vector<float> pk((size_t)mlp_packed_size(nin) + (nout > 1 ? H + 3 : 0));
  float* q = pk.data();
  std::memcpy(q, m->w1, sizeof(float) * H * nin); q += H * nin;
  std::memcpy(q, m->b1, sizeof(float) * H); q += H;
  std::memcpy(q, m->w2, sizeof(float) * H * H); q += H * H;
  std::memcpy(q, m->b2, sizeof(float) * H); q += H;
  std::memcpy(q, m->w3, sizeof(float) * H); q += H;
  *q++ = m->b3;
  for (int i = 0; i < nin; i++) *q++ = m->in_shift[i];
  for (int i = 0; i < nin; i++) *q++ = m->in_scale[i];
  *q++ = m->out_shift;
  *q++ = m->out_scale;
  if (nout > 1) {
    std::memcpy(q, m->w3 + H, sizeof(float) * H); q += H;
    *q++ = m->b3_1;
    *q++ = m->out_shift_1;
    *q++ = m->out_scale_1;
  }
  float* tmp = nullptr;
  cudaError_t e = cudaMalloc(&tmp, sizeof(float) * pk.size());
  if (e == cudaSuccess && !*dev) e = cudaMalloc(dev, sizeof(MlpDev));
  if (e == cudaSuccess) e = cudaMemcpyAsync(tmp, pk.data(), sizeof(float) * pk.size(), cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = mlp_install(tmp, nin, nout, *dev, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  cudaFree(tmp);
  if (e != cudaSuccess) {
    set_error(std::string("seed model upload: ") + cudaGetErrorString(e));
    return ECG_ERR_CUDA;
  }
  return ECG_OK;
}

}  // namespace ecg

extern "C" const char* ecg_status_str(ecg_status s) {
  switch (s) {
    case ECG_OK: return "ok";
    case ECG_ERR_INVALID: return "invalid argument";
    case ECG_ERR_UNSUPPORTED: return "unsupported case";
    case ECG_ERR_CUDA: return "CUDA error";
    case ECG_ERR_XML: return "case input error";
    case ECG_ERR_PHYSICS: return "physics check failed";
    case ECG_ERR_NOMEM: return "out of memory";
    case ECG_ERR_TOO_LARGE: return "size above the stated maximum";
    case ECG_ERR_TIMEOUT: return "device wait timed out";
  }
  return "unknown status";
}

extern "C" const char* ecg_last_error(void) { return g_last_error.c_str(); }
extern "C" int ecg_version(void) { return 10000; }

extern "C" ecg_status ecg_create(const ecg_case* c, ecg_ctx** out) {
  if (!out) { set_error("null out"); return ECG_ERR_INVALID; }
  *out = nullptr;
  ecg_status vs = validate_case(c);
  if (vs != ECG_OK) return vs;
  auto x = new ecg_ctx();
  x->c = *c;
  x->dim = (c->ncells[0] != 1) + (c->ncells[1] != 1) + (c->ncells[2] != 1);
  x->np = c->nphases;
  x->n = (int64_t)c->ncells[0] * c->ncells[1] * c->ncells[2];
  x->eps = c->alpha_null ? 1.e-15 : 0.;
  const bool euler = c->model == ECG_MODEL_EULER;
  const bool ptueq = c->model == ECG_MODEL_PTUEQ;
  // Euler: rho, p, u, E ; PTUEq: alpha_0, alpha_1, p, T, u, E ; Kapila: alpha_k, rho_k, p, u, E
  x->nstate = euler ? (3 + x->dim) : (ptueq ? 5 + x->dim : 2 * x->np + 2 + x->dim);
  x->nq = x->nstate - 1;
  auto fail_free = [&](ecg_status s) {
    ecg_destroy(x);
    return s;
  };
  cudaError_t e = cudaGetDevice(&x->device);
  if (e != cudaSuccess) return fail_free(cuda_fail(e, "cudaGetDevice"));
  e = cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return fail_free(cuda_fail(e, "cudaStreamCreate"));
  // state: the 2N + 2 + d (Euler 3 + d) fields, then the passive transports
  size_t sbytes = sizeof(double) * (size_t)(x->nstate + c->ntransports) * (size_t)x->n;
  for (int i = 0; i < 2; i++) {
    e = cudaMalloc(&x->state[i], sbytes);
    if (e != cudaSuccess) return fail_free(cuda_fail(e, "cudaMalloc(state)"));
    cudaMemsetAsync(x->state[i], 0, sbytes, x->stream);
  }
  if (c->order == 2) {
    e = cudaMalloc(&x->half, sizeof(double) * (size_t)(x->nstate + c->ntransports) * (size_t)x->n);
    if (e != cudaSuccess) return fail_free(cuda_fail(e, "cudaMalloc(half)"));
  }
  e = cudaMalloc(&x->tmp, sizeof(double) * (size_t)(ptueq ? 2 : 1) * (size_t)x->n);  // download scratch
  if (e != cudaSuccess) return fail_free(cuda_fail(e, "cudaMalloc(tmp)"));
  if (!euler && !ptueq && x->dim >= 2 && c->ntransports == 0) {
    // face arrays of the split form: 3N + d + 3 flux components per face, faces of each axis including
    // the domain sides
    const int nfl = 3 * x->np + x->dim + 3;
    for (int a = 0; a < x->dim; a++) {
      e = cudaMalloc(&x->flux[a], sizeof(double) * (size_t)nfl * (size_t)split_nfaces(c->ncells, a));
      if (e != cudaSuccess) return fail_free(cuda_fail(e, "cudaMalloc(face fluxes)"));
    }
    x->split = true;
#ifndef ECG_BOUNDS_CHECK
    // TMA staging of the face kernels' tiles where the layout allows it (the bounds-checked build
    // checks the kernels' own loads, so it stages them that way)
    const double* bufs[3] = {x->state[0], x->state[1], x->half};
    build_face_maps(x->fmaps, bufs, x->dim, c->ncells, x->nq);
#endif
  }
  std::vector<double> h, sz[3], ctr[3];
  for (int a = 0; a < 3; a++) axis_cells(*c, a, sz[a], ctr[a]);
  distance_tables(*c, sz, ctr, h);
  e = cudaMalloc(&x->dist, sizeof(double) * h.size());
  if (e != cudaSuccess) return fail_free(cuda_fail(e, "cudaMalloc(dist)"));
  cudaMemcpy(x->dist, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice);
  int nmax = std::max({c->ncells[0], c->ncells[1], c->ncells[2]});
  for (int a = 0; a < 3; a++) {
    x->geo.n[a] = c->ncells[a];
    x->geo.dcc[a] = x->dist + (size_t)(3 * a + 0) * nmax;
    x->geo.dfl[a] = x->dist + (size_t)(3 * a + 1) * nmax;
    x->geo.dfr[a] = x->dist + (size_t)(3 * a + 2) * nmax;
    x->geo.dsz[a] = x->dist + (size_t)(9 + a) * nmax;
  }
  x->geo.dim = x->dim;
  x->geo.stretched = case_stretched(*c) ? 1 : 0;
  side_geometry(*c, sz, ctr, x->geo);
  // MeshCartesian::initializeGeometrieMonoCpu :228-236 and face surfaces :287, :320, :353
  double dX = c->length[0] / (double)c->ncells[0], dY = c->length[1] / (double)c->ncells[1],
         dZ = c->length[2] / (double)c->ncells[2];
  double vol = dX * dY * dZ;
  x->geo.coefA[0] = (dY * dZ) / vol;
  x->geo.coefA[1] = (dX * dZ) / vol;
  x->geo.coefA[2] = (dX * dY) / vol;
  double l = 1.e10;
  if (c->ncells[0] != 1) l = std::min(l, dX);
  if (c->ncells[1] != 1) l = std::min(l, dY);
  if (c->ncells[2] != 1) l = std::min(l, dZ);
  if (x->dim > 1) l *= 0.6;
  x->geo.lcfl = l;
  if (c->ptmu) {  // Mixture::computeCriticalPressure src/Models/Mixture.cpp:146
    const ecg_eos& L = c->eos[c->ptmu_liquid];
    const ecg_eos& V = c->eos[c->ptmu_vapor];
    double piL = L.type == ECG_EOS_IG ? 0. : L.pinf, piV = V.type == ECG_EOS_IG ? 0. : V.pinf;
    double pc = piL * (V.gamma - 1.) * V.cv - piV * (L.gamma - 1.) * L.cv;
    pc /= (L.gamma - 1.) * L.cv - (V.gamma - 1.) * V.cv;
    x->pcrit = pc;
  }
  e = cudaMalloc(&x->scal, sizeof(DevScalars));
  if (e != cudaSuccess) return fail_free(cuda_fail(e, "cudaMalloc(scalars)"));
  e = cudaMalloc(&x->stats, sizeof(DevStats));
  if (e == cudaSuccess) e = cudaMallocHost(&x->h_scal, sizeof(DevScalars));
  if (e == cudaSuccess) e = cudaMallocHost(&x->h_stats, sizeof(DevStats));
  if (e != cudaSuccess) return fail_free(cuda_fail(e, "cudaMalloc(stats)"));
  DevScalars s0{};
  s0.dt = 1.e-15;
  s0.cfl = c->cfl;
  s0.dtmax_bits = (unsigned long long)0;
  double big = 1.e10;
  std::memcpy(&s0.dtmax_bits, &big, sizeof(double));
  cudaMemcpy(x->scal, &s0, sizeof(s0), cudaMemcpyHostToDevice);
  cudaMemset(x->stats, 0, sizeof(DevStats));
  // kernel attributes (dynamic shared memory) for every pass of this case shape
  for (int pass = 0; pass < 3; pass++) {
    StepParams P{};
    P.ntr = c->ntransports;
    cudaError_t pe = euler   ? euler_launch(x->dim, pass, P, x->geo, c->eos, x->eps, x->stream, true)
                     : ptueq ? ptueq_launch(x->dim, pass, P, x->geo, c->eos, x->stream, true)
                             : kapila_launch(x->np, x->dim, c->ptmu != 0, pass, P, x->geo, c->eos, x->eps, x->stream, true);
    if (pe == cudaErrorNotSupported) {
      set_error("no kernel built for this model / phases / dimension");
      ecg_destroy(x);
      return ECG_ERR_UNSUPPORTED;
    }
    if (pe != cudaSuccess) return fail_free(cuda_fail(pe, "cudaFuncSetAttribute"));
  }
  e = cudaStreamSynchronize(x->stream);
  if (e != cudaSuccess) return fail_free(cuda_fail(e, "create"));
  *out = x;
  return ECG_OK;
}

extern "C" void ecg_destroy(ecg_ctx* x) {
  if (!x) return;
  if (x->stream) cudaStreamSynchronize(x->stream);
  drop_graphs(x);
  cudaFree(x->state[0]);
  cudaFree(x->state[1]);
  cudaFree(x->half);
  cudaFree(x->dist);
  cudaFree(x->tmp);
  for (int a = 0; a < 3; a++) cudaFree(x->flux[a]);
  cudaFree(x->scal);
  cudaFree(x->stats);
  cudaFreeHost(x->h_scal);
  cudaFreeHost(x->h_stats);
  cudaFree(x->mlp);
  cudaFree(x->rec_x);
  cudaFree(x->rec_y);
  cudaFree(x->rec_count);
  cudaFree(x->tsat_hist);
  if (x->stream) cudaStreamDestroy(x->stream);
  delete x;
}

extern "C" int64_t ecg_ncells(const ecg_ctx* x) { return x ? x->n : 0; }
extern "C" void* ecg_stream(const ecg_ctx* x) { return x ? (void*)x->stream : nullptr; }

extern "C" ecg_status ecg_set_step_form(ecg_ctx* x, int32_t form) {
  if (!x || (form != ECG_FORM_FUSED && form != ECG_FORM_SPLIT)) { set_error("bad step form"); return ECG_ERR_INVALID; }
  if (form == ECG_FORM_SPLIT && !x->flux[0]) { set_error("no split form for this case (1D, Euler, PTUEq or transports)"); return ECG_ERR_UNSUPPORTED; }
  x->split = form == ECG_FORM_SPLIT;
  x->graph_dirty = true;
  return ECG_OK;
}

extern "C" int32_t ecg_step_form(const ecg_ctx* x) { return (x && x->split) ? ECG_FORM_SPLIT : ECG_FORM_FUSED; }

extern "C" ecg_status ecg_set_face_staging(ecg_ctx* x, int32_t staging) {
  if (!x || (staging != ECG_STAGING_PLAIN && staging != ECG_STAGING_TMA)) { set_error("bad staging"); return ECG_ERR_INVALID; }
  x->staging = staging;
  x->graph_dirty = true;
  return ECG_OK;
}

extern "C" int32_t ecg_face_staging(const ecg_ctx* x) {
  return (x && x->split && x->staging == ECG_STAGING_TMA && x->fmaps.ok) ? ECG_STAGING_TMA : ECG_STAGING_PLAIN;
}

extern "C" ecg_status ecg_set_newton_cap(ecg_ctx* x, int32_t cap) {
  if (!x || cap < 1 || cap > 100000) { set_error("bad Newton cap"); return ECG_ERR_INVALID; }
  x->newton_cap = cap;
  x->graph_dirty = true;
  return ECG_OK;
}

extern "C" ecg_status ecg_set_newton_cap_mode(ecg_ctx* x, int32_t mode) {
  if (!x || (mode != ECG_CAP_FALLBACK && mode != ECG_CAP_ACCEPT)) { set_error("bad Newton cap mode"); return ECG_ERR_INVALID; }
  x->newton_accept = mode == ECG_CAP_ACCEPT ? 1 : 0;
  x->graph_dirty = true;
  return ECG_OK;
}

static ecg_status upload_impl(ecg_ctx* x, const double* const* f, int64_t ncells, cudaMemcpyKind kind) {
  if (!x || !f) { set_error("null argument"); return ECG_ERR_INVALID; }
  if (ncells != x->n) { set_error("ncells does not match the context"); return ECG_ERR_INVALID; }
  const int nf = abi_nfields(x->c);
  for (int i = 0; i < nf; i++)
    if (!f[i]) { set_error("null field pointer"); return ECG_ERR_INVALID; }
  const int64_t n = x->n;
  const size_t fb = sizeof(double) * (size_t)n;
  double* S = x->state[x->cur];
  const bool euler = x->c.model == ECG_MODEL_EULER;
  // a new state: the p-T-mu warm start forgets the previous state's T_sat values
  if (x->tsat_hist) ECG_CUDA(cudaMemsetAsync(x->tsat_hist, 0, fb, x->stream));
  if (x->c.model == ECG_MODEL_PTUEQ) {
    // ABI: alpha_0 alpha_1 rho_0 rho_1 p u_x u_y u_z E T -> device: alpha_0 alpha_1 p T u_0..u_{dim-1} E
    // (the phase densities are computeDensity(p, T); the uploaded ones are not read)
    for (int i = 0; i < 2; i++) ECG_CUDA(cudaMemcpyAsync(S + (size_t)i * n, f[i], fb, kind, x->stream));
    ECG_CUDA(cudaMemcpyAsync(S + (size_t)2 * n, f[4], fb, kind, x->stream));
    ECG_CUDA(cudaMemcpyAsync(S + (size_t)3 * n, f[9], fb, kind, x->stream));
    for (int d = 0; d < x->dim; d++) ECG_CUDA(cudaMemcpyAsync(S + (size_t)(4 + d) * n, f[5 + d], fb, kind, x->stream));
    ECG_CUDA(cudaMemcpyAsync(S + (size_t)(4 + x->dim) * n, f[8], fb, kind, x->stream));
    if (kind == cudaMemcpyHostToDevice)
      for (int d = x->dim; d < 3; d++)
        for (int64_t i = 0; i < n; i++)
          if (f[5 + d][i] != 0.) {
            set_error("non-zero velocity component along an axis with one cell is not supported");
            return ECG_ERR_UNSUPPORTED;
          }
    return ECG_OK;
  }
  // ABI: [alpha_k, rho_k] p u_x u_y u_z E  -> device: [alpha_k, rho_k] p u_0..u_{dim-1} E
  const int pre = euler ? 2 : 2 * x->np + 1;  // fields up to and including p
  for (int i = 0; i < pre; i++) ECG_CUDA(cudaMemcpyAsync(S + (size_t)i * n, f[i], fb, kind, x->stream));
  for (int d = 0; d < x->dim; d++) ECG_CUDA(cudaMemcpyAsync(S + (size_t)(pre + d) * n, f[pre + d], fb, kind, x->stream));
  ECG_CUDA(cudaMemcpyAsync(S + (size_t)(pre + x->dim) * n, f[pre + 3], fb, kind, x->stream));
  // passive transports follow E on both sides
  for (int j = 0; j < x->c.ntransports; j++)
    ECG_CUDA(cudaMemcpyAsync(S + (size_t)(x->nstate + j) * n, f[pre + 4 + j], fb, kind, x->stream));
  if (kind == cudaMemcpyHostToDevice) {
    // transverse velocity components of a lower-dimensional case must be zero (they are not stored)
    for (int d = x->dim; d < 3; d++)
      for (int64_t i = 0; i < n; i++)
        if (f[pre + d][i] != 0.) {
          set_error("non-zero velocity component along an axis with one cell is not supported");
          return ECG_ERR_UNSUPPORTED;
        }
  }
  return ECG_OK;
}

extern "C" ecg_status ecg_upload_prim(ecg_ctx* x, const double* const* f, int64_t ncells) {
  ecg_status s = upload_impl(x, f, ncells, cudaMemcpyHostToDevice);
  if (s != ECG_OK) return s;
  ECG_CUDA(cudaStreamSynchronize(x->stream));
  return ECG_OK;
}

extern "C" ecg_status ecg_upload_prim_device(ecg_ctx* x, const double* const* f, int64_t ncells) {
  return upload_impl(x, f, ncells, cudaMemcpyDeviceToDevice);
}

static ecg_status download_impl(ecg_ctx* x, double* const* f, int64_t ncells, cudaMemcpyKind kind) {
  if (!x || !f) { set_error("null argument"); return ECG_ERR_INVALID; }
  if (ncells != x->n) { set_error("ncells does not match the context"); return ECG_ERR_INVALID; }
  const int nf = abi_nfields(x->c);
  for (int i = 0; i < nf; i++)
    if (!f[i]) { set_error("null field pointer"); return ECG_ERR_INVALID; }
  const int64_t n = x->n;
  const size_t fb = sizeof(double) * (size_t)n;
  const double* S = x->state[x->cur];
  const bool euler = x->c.model == ECG_MODEL_EULER;
  if (x->c.model == ECG_MODEL_PTUEQ) {
    k_ptueq_derived<<<(unsigned)((n + 255) / 256), 256, 0, x->stream>>>(S, n, x->c.eos[0], x->c.eos[1], x->tmp,
                                                                       nullptr, nullptr);
    ECG_CUDA(cudaGetLastError());
    for (int i = 0; i < 2; i++) {
      ECG_CUDA(cudaMemcpyAsync(f[i], S + (size_t)i * n, fb, kind, x->stream));
      ECG_CUDA(cudaMemcpyAsync(f[2 + i], x->tmp + (size_t)i * n, fb, kind, x->stream));
    }
    ECG_CUDA(cudaMemcpyAsync(f[4], S + (size_t)2 * n, fb, kind, x->stream));
    for (int d = 0; d < 3; d++) {
      if (d < x->dim) ECG_CUDA(cudaMemcpyAsync(f[5 + d], S + (size_t)(4 + d) * n, fb, kind, x->stream));
      else if (kind == cudaMemcpyDeviceToHost) {
        ECG_CUDA(cudaStreamSynchronize(x->stream));
        std::memset(f[5 + d], 0, fb);
      } else ECG_CUDA(cudaMemsetAsync(f[5 + d], 0, fb, x->stream));
    }
    ECG_CUDA(cudaMemcpyAsync(f[8], S + (size_t)(4 + x->dim) * n, fb, kind, x->stream));
    ECG_CUDA(cudaMemcpyAsync(f[9], S + (size_t)3 * n, fb, kind, x->stream));
    return ECG_OK;
  }
  if (euler) {
    for (int i = 0; i < 2; i++) ECG_CUDA(cudaMemcpyAsync(f[i], S + (size_t)i * n, fb, kind, x->stream));
  } else {
    k_derived<<<(unsigned)((n + 255) / 256), 256, 0, x->stream>>>(S, n, x->np, x->dim, x->c.eos[0], x->c.eos[1],
                                                                 x->c.eos[2], x->eps, x->tmp, nullptr, nullptr);
    ECG_CUDA(cudaGetLastError());
    for (int i = 0; i < 2 * x->np; i++) ECG_CUDA(cudaMemcpyAsync(f[i], S + (size_t)i * n, fb, kind, x->stream));
    ECG_CUDA(cudaMemcpyAsync(f[2 * x->np], x->tmp, fb, kind, x->stream));
  }
  const int pre = euler ? 2 : 2 * x->np + 1;
  for (int d = 0; d < 3; d++) {
    if (d < x->dim) ECG_CUDA(cudaMemcpyAsync(f[pre + d], S + (size_t)(pre + d) * n, fb, kind, x->stream));
    else if (kind == cudaMemcpyDeviceToHost) {
      ECG_CUDA(cudaStreamSynchronize(x->stream));
      std::memset(f[pre + d], 0, fb);
    } else ECG_CUDA(cudaMemsetAsync(f[pre + d], 0, fb, x->stream));
  }
  ECG_CUDA(cudaMemcpyAsync(f[pre + 3], S + (size_t)(pre + x->dim) * n, fb, kind, x->stream));
  for (int j = 0; j < x->c.ntransports; j++)
    ECG_CUDA(cudaMemcpyAsync(f[pre + 4 + j], S + (size_t)(x->nstate + j) * n, fb, kind, x->stream));
  return ECG_OK;
}

extern "C" ecg_status ecg_download_prim(ecg_ctx* x, double* const* f, int64_t ncells) {
  ecg_status s = download_impl(x, f, ncells, cudaMemcpyDeviceToHost);
  if (s != ECG_OK) return s;
  ECG_CUDA(cudaStreamSynchronize(x->stream));
  return ECG_OK;
}

extern "C" ecg_status ecg_download_prim_device(ecg_ctx* x, double* const* f, int64_t ncells) {
  return download_impl(x, f, ncells, cudaMemcpyDeviceToDevice);
}

extern "C" ecg_status ecg_download_derived(ecg_ctx* x, double* T, double* Y, int64_t ncells) {
  if (!x || !T || !Y) { set_error("null argument"); return ECG_ERR_INVALID; }
  if (ncells != x->n) { set_error("ncells does not match the context"); return ECG_ERR_INVALID; }
  const int64_t n = x->n;
  const int np = x->np;
  double *dT = nullptr, *dY = nullptr;
  ECG_CUDA(cudaMalloc(&dT, sizeof(double) * (size_t)np * n));
  cudaError_t e = cudaMalloc(&dY, sizeof(double) * (size_t)np * n);
  if (e != cudaSuccess) {
    cudaFree(dT);
    return cuda_fail(e, "cudaMalloc");
  }
  const double* S = x->state[x->cur];
  if (x->c.model == ECG_MODEL_EULER) {
    k_euler_derived<<<(unsigned)((n + 255) / 256), 256, 0, x->stream>>>(S, n, x->c.eos[0], x->eps, dT);
    cudaMemsetAsync(dY, 0, sizeof(double) * n, x->stream);
  } else if (x->c.model == ECG_MODEL_PTUEQ) {
    k_ptueq_derived<<<(unsigned)((n + 255) / 256), 256, 0, x->stream>>>(S, n, x->c.eos[0], x->c.eos[1], nullptr, dT,
                                                                       dY);
  } else {
    k_derived<<<(unsigned)((n + 255) / 256), 256, 0, x->stream>>>(S, n, np, x->dim, x->c.eos[0], x->c.eos[1],
                                                                 x->c.eos[2], x->eps, nullptr, dT, dY);
  }
  cudaMemcpyAsync(T, dT, sizeof(double) * (size_t)np * n, cudaMemcpyDeviceToHost, x->stream);
  cudaMemcpyAsync(Y, dY, sizeof(double) * (size_t)np * n, cudaMemcpyDeviceToHost, x->stream);
  e = cudaStreamSynchronize(x->stream);
  cudaFree(dT);
  cudaFree(dY);
  if (e != cudaSuccess) return cuda_fail(e, "download_derived");
  if (x->c.model == ECG_MODEL_EULER)
    for (int64_t i = 0; i < n; i++) Y[i] = 1.;
  return ECG_OK;
}

// kernel_ms (profiled steps, every kernel launched separately): with nms = 3 the pass-1, pass-2 and
// update times; with nms = 9 per kernel: pass 1 X, Y, Z face kernels and cell kernel (the whole pass
// in fused form), pass 2 the same, update.
static ecg_status step_common(ecg_ctx* x, int mode, int32_t nsteps, double* dt, double* t, int32_t* iterations,
                              ecg_step_stats* stats, double* kernel_ms = nullptr, int nms = 3) {
  // host values of dt and t seed the device scalars (the caller owns the time loop state)
  DevScalars h{};
  h.dt = *dt;
  h.t = *t;
  h.cfl = x->c.cfl;
  h.t_end = x->c.total_time;
  double big = 1.e10;
  std::memcpy(&h.dtmax_bits, &big, sizeof(double));
  h.it = iterations ? *iterations : 0;
  h.max_it = x->c.max_iterations;
  h.mode = mode;
  h.done = (mode == 1 && h.it >= h.max_it) || (mode == 2 && h.t >= h.t_end);
  *x->h_scal = h;  // the previous call synchronised, so the staging buffer is free
  ECG_CUDA(cudaMemcpyAsync(x->scal, x->h_scal, sizeof(h), cudaMemcpyHostToDevice, x->stream));
  ECG_CUDA(cudaMemsetAsync(x->stats, 0, sizeof(DevStats), x->stream));
  const int cur0 = x->cur;  // a step that finds the stop flag set writes nothing, so the state that
                            // holds the result is decided by the number of steps actually taken
  int64_t done_steps = 0;
  if (kernel_ms) {
    // ev[0..3]: step start, after pass 1, after pass 2, after the update; ev[4..6] / ev[7..9]: after
    // the X, Y, Z face kernels of pass 1 / pass 2 (split form)
    cudaEvent_t ev[10];
    for (int i = 0; i < 10; i++) ECG_CUDA(cudaEventCreate(&ev[i]));
    auto ms = [&](int a, int b) {
      float v = 0.f;
      cudaEventElapsedTime(&v, ev[a], ev[b]);
      return (double)v;
    };
    const bool two = x->c.order == 2;
    for (int i = 0; i < nsteps; i++) {
      ecg_status s = launch_step(x, x->cur, ev);
      if (s != ECG_OK) return s;
      x->cur = 1 - x->cur;
      ECG_CUDA(cudaEventSynchronize(ev[3]));
      if (nms < 9) {
        kernel_ms[0] += ms(0, 1);
        kernel_ms[1] += ms(1, 2);
        kernel_ms[2] += ms(2, 3);
        continue;
      }
      for (int pass = 0; pass < (two ? 2 : 1); pass++) {
        const int start = pass == 0 ? 0 : 1, end = pass == 0 ? 1 : 2, base = pass == 0 ? 4 : 7;
        double* o = kernel_ms + 4 * pass;
        if (x->split) {
          int prev = start;
          for (int a = 0; a < x->dim; a++) {
            o[a] += ms(prev, base + a);
            prev = base + a;
          }
          o[3] += ms(prev, end);
        } else {
          o[3] += ms(start, end);
        }
      }
      kernel_ms[8] += ms(2, 3);
    }
    for (int i = 0; i < 10; i++) cudaEventDestroy(ev[i]);
  } else if (mode == 0) {
    ecg_status s = advance(x, nsteps);
    if (s != ECG_OK) return s;
  } else {
    // chunks of captured steps; steps after the stop condition are no-ops on the device
    const int chunk = 64;
    for (;;) {
      ecg_status s = advance(x, chunk);
      if (s != ECG_OK) return s;
      DevScalars r{};
      ECG_CUDA(cudaMemcpyAsync(&r, x->scal, sizeof(r), cudaMemcpyDeviceToHost, x->stream));
      ECG_CUDA(cudaStreamSynchronize(x->stream));
      if (r.done) break;
    }
  }
  ECG_CUDA(cudaMemcpyAsync(x->h_scal, x->scal, sizeof(DevScalars), cudaMemcpyDeviceToHost, x->stream));
  ECG_CUDA(cudaMemcpyAsync(x->h_stats, x->stats, sizeof(DevStats), cudaMemcpyDeviceToHost, x->stream));
  ECG_CUDA(cudaStreamSynchronize(x->stream));
  const DevScalars r = *x->h_scal;
  const DevStats ds = *x->h_stats;
  done_steps = r.it - h.it;
  x->cur = cur0 ^ (int)(done_steps & 1);
  *dt = r.dt;
  *t = r.t;
  if (iterations) *iterations = (int32_t)r.it;
  if (stats) stats_out(ds, done_steps * x->n, stats);
  if (ds.staging_timeouts) {
    set_error("a face kernel's TMA staging copy did not complete");
    return ECG_ERR_CUDA;
  }
  if (ds.ptmu_errors) {
    set_error("p-T-mu relaxation exceeded 50 iterations");
    return ECG_ERR_PHYSICS;
  }
  return ECG_OK;
}

extern "C" ecg_status ecg_step(ecg_ctx* x, int32_t nsteps, double* dt, double* t, ecg_step_stats* stats) {
  if (!x || !dt || !t || nsteps < 0) { set_error("bad argument"); return ECG_ERR_INVALID; }
  return step_common(x, 0, nsteps, dt, t, nullptr, stats);
}

extern "C" ecg_status ecg_step_profiled(ecg_ctx* x, int32_t nsteps, double* dt, double* t, ecg_step_stats* stats,
                                        double* kernel_ms) {
  if (!x || !dt || !t || nsteps < 0 || !kernel_ms) { set_error("bad argument"); return ECG_ERR_INVALID; }
  return step_common(x, 0, nsteps, dt, t, nullptr, stats, kernel_ms, 3);
}

extern "C" ecg_status ecg_step_profiled_kernels(ecg_ctx* x, int32_t nsteps, double* dt, double* t,
                                                ecg_step_stats* stats, double* kernel_ms) {
  if (!x || !dt || !t || nsteps < 0 || !kernel_ms) { set_error("bad argument"); return ECG_ERR_INVALID; }
  return step_common(x, 0, nsteps, dt, t, nullptr, stats, kernel_ms, 9);
}

extern "C" ecg_status ecg_run(ecg_ctx* x, double* dt, double* t, int32_t* iterations, ecg_step_stats* stats) {
  if (!x || !dt || !t || !iterations) { set_error("bad argument"); return ECG_ERR_INVALID; }
  return step_common(x, x->c.time_iterations ? 1 : 2, 0, dt, t, iterations, stats);
}

extern "C" ecg_status ecg_set_seed_model(ecg_ctx* x, const ecg_mlp* m) {
  if (!x) { set_error("null context"); return ECG_ERR_INVALID; }
  x->graph_dirty = true;
  if (!m) {
    cudaFree(x->mlp);
    x->mlp = nullptr;
    return ECG_OK;
  }
  if (x->c.model != ECG_MODEL_KAPILA) { set_error("the seed model applies to Kapila relaxation"); return ECG_ERR_UNSUPPORTED; }
  if (x->c.ntransports > 0) { set_error("the seeded kernels run without passive transports"); return ECG_ERR_UNSUPPORTED; }
  return mlp_upload(m, x->np, x->c.ptmu != 0, &x->mlp, x->stream);
}

extern "C" ecg_status ecg_set_ptmu_warm_start(ecg_ctx* x, int32_t on) {
  if (!x || (on != 0 && on != 1)) { set_error("bad argument"); return ECG_ERR_INVALID; }
  if (on && !x->c.ptmu) { set_error("the warm start applies to p-T-mu relaxation"); return ECG_ERR_UNSUPPORTED; }
  x->graph_dirty = true;
  if (!on) {
    if (x->stream) cudaStreamSynchronize(x->stream);
    cudaFree(x->tsat_hist);
    x->tsat_hist = nullptr;
    return ECG_OK;
  }
  if (!x->tsat_hist) {
    ECG_CUDA(cudaMalloc(&x->tsat_hist, sizeof(double) * (size_t)x->n));
    ECG_CUDA(cudaMemsetAsync(x->tsat_hist, 0, sizeof(double) * (size_t)x->n, x->stream));  // 0: no solve yet
  }
  return ECG_OK;
}

extern "C" ecg_status ecg_set_ptmu_seed(ecg_ctx* x, int32_t mode) {
  if (!x || (mode != ECG_PTMU_SEED_T && mode != ECG_PTMU_SEED_P_T)) { set_error("bad p-T-mu seed mode"); return ECG_ERR_INVALID; }
  x->ptmu_seed_p = mode == ECG_PTMU_SEED_P_T ? 1 : 0;
  x->graph_dirty = true;
  return ECG_OK;
}

extern "C" ecg_status ecg_record_pairs(ecg_ctx* x, int64_t max_pairs, int32_t min_evals) {
  if (!x || max_pairs < 0 || min_evals < 1) { set_error("bad argument"); return ECG_ERR_INVALID; }
  x->graph_dirty = true;
  x->rec_min_evals = min_evals;
  cudaFree(x->rec_x);
  cudaFree(x->rec_y);
  cudaFree(x->rec_count);
  x->rec_x = x->rec_y = nullptr;
  x->rec_count = nullptr;
  x->rec_max = 0;
  if (max_pairs == 0) return ECG_OK;
  const int nin = x->c.ptmu ? PTMU_NIN : 3 * x->np, nout = x->c.ptmu ? 2 : 1;
  ECG_CUDA(cudaMalloc(&x->rec_x, sizeof(float) * nin * (size_t)max_pairs));
  ECG_CUDA(cudaMalloc(&x->rec_y, sizeof(float) * nout * (size_t)max_pairs));
  ECG_CUDA(cudaMalloc(&x->rec_count, sizeof(unsigned long long)));
  ECG_CUDA(cudaMemset(x->rec_count, 0, sizeof(unsigned long long)));
  x->rec_max = (unsigned long long)max_pairs;
  return ECG_OK;
}

extern "C" ecg_status ecg_fetch_pairs(ecg_ctx* x, float* features, float* targets, int64_t* count) {
  if (!x || !count) { set_error("bad argument"); return ECG_ERR_INVALID; }
  if (!x->rec_count) { *count = 0; return ECG_OK; }
  unsigned long long c = 0;
  ECG_CUDA(cudaMemcpyAsync(&c, x->rec_count, sizeof(c), cudaMemcpyDeviceToHost, x->stream));
  ECG_CUDA(cudaStreamSynchronize(x->stream));
  if (c > x->rec_max) c = x->rec_max;
  *count = (int64_t)c;
  const int nin = x->c.ptmu ? PTMU_NIN : 3 * x->np, nout = x->c.ptmu ? 2 : 1;
  if (features && c) ECG_CUDA(cudaMemcpy(features, x->rec_x, sizeof(float) * nin * c, cudaMemcpyDeviceToHost));
  if (targets && c) ECG_CUDA(cudaMemcpy(targets, x->rec_y, sizeof(float) * nout * c, cudaMemcpyDeviceToHost));
  return ECG_OK;
}
