// Batched independent 1D cases: one persistent kernel per pass pulls (case, tile) work items from
// a device queue.
//
// The reference runs independent cases one after the other (src/main.cpp:82-133), each with its
// own time loop.  Here all cases live in one concatenated structure-of-arrays state (case c owns
// cells [off_c, off_c + n_c)), every pass (first order, or MUSCL predictor then corrector) is one
// launch of #SM x occupancy blocks that loop over the work items, and each case keeps its own dt:
// the min of lCFL/|s| over a case's faces is reduced per work item and merged into the case's slot
// with one atomicMin (a segmented min-reduction), then a per-case update sets dt_c = cfl_c dtMax_c.
// The step sequence is captured once as a CUDA graph.  Tile size and block size are picked by a
// small autotuner that times each candidate on a copy of the state.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "ecg_internal.h"
#include "ecg_kapila_cell.cuh"

// Register budget of the batched kernels: ECG_BATCH_SM_THREADS > 0 asks the compiler to fit
// ECG_BATCH_SM_THREADS / TB blocks of TB threads on an SM (more resident warps, fewer registers a
// thread); 0 leaves the register count to the compiler.  Measured on 4096 batched two-phase tubes
// (cell-updates/s, tile chosen by the autotuner): no budget (168 registers, 12 warps per SM) 1168 M;
// 512 threads 1448 M; 640: 1464 M; 896 (85 registers at 256-cell tiles, 24 warps) 1628-1658 M;
// 1024: 1599 M; 1152: 1602 M.
#ifndef ECG_BATCH_SM_THREADS
#define ECG_BATCH_SM_THREADS 896
#endif
// Cells of one work item for TB threads: TB - ECG_BATCH_ITEM_TRIM.  With a trim of 1 the item's
// TB faces take one round of the block; with 0 the item has TB + 1 faces and one warp computes two
// while the block waits at the next barrier.  Measured on 4096 batched tubes: trim 0 1657 M, trim 1
// 2066 M cell-updates/s.
#ifndef ECG_BATCH_ITEM_TRIM
#define ECG_BATCH_ITEM_TRIM 1
#endif
#if ECG_BATCH_SM_THREADS > 0
#define ECG_BATCH_BOUNDS(TB) __launch_bounds__(TB, (ECG_BATCH_SM_THREADS / (TB) > 0 ? ECG_BATCH_SM_THREADS / (TB) : 1))
#else
#define ECG_BATCH_BOUNDS(TB) __launch_bounds__(TB)
#endif

namespace ecg {

struct BatchCase {
  int64_t off;
  int n;
  double dx, coefA, lcfl, cfl;
};

struct BatchScalars {
  double dt, t;
  unsigned long long dtmax_bits;
  long long it;
};

struct BatchParams {
  StepParams P;              // q / sn / out point at the concatenated state (stride = total cells)
  const BatchCase* cases;
  BatchScalars* scal;
  const int2* items;         // (case, first cell)
  int nitems;
  unsigned int* queue;       // work counter of this pass
};

template <int NP, int TB, int PASS>
struct BatchTile {
  static constexpr int TC = TB - ECG_BATCH_ITEM_TRIM;  // cells of one work item
  static constexpr int H = (PASS == PASS_O1) ? 1 : 2;
  static constexpr int RL = TC + 2 * H;
  static constexpr int NQ = Fields<NP, 1>::NQ + ((PASS == PASS_CORR) ? 1 : 0);
  static constexpr int NS = (PASS == PASS_O1) ? 0 : TC + 3;
  static constexpr size_t smem_bytes() {
    return sizeof(double) * ((size_t)RL * NQ + (size_t)NS * Fields<NP, 1>::NSL + (size_t)(TC + 1) * Fields<NP, 1>::NFL);
  }
};

template <int NP, int TB, int PASS, int TYPES>
__global__ void ECG_BATCH_BOUNDS(TB) k_batch(BatchParams B, Model<NP> M0) {
  const Model<NP> M = specialize_eos<NP, TYPES>(M0);  // EOS types compiled in for the shipped workload
  using FL = Fields<NP, 1>;
  using K = BatchTile<NP, TB, PASS>;
  constexpr bool O2 = (PASS != PASS_O1);
  constexpr int TC = K::TC;
  constexpr int RS = K::RL;
  constexpr int SS = O2 ? K::NS : 1;
  constexpr int FS = TC + 1;
  extern __shared__ double smem[];
  double* sq = smem;
  double* sa0 = sq + (size_t)FL::NQ * RS;
  double* ssl = sq + (size_t)K::NQ * RS;
  double* sfl = ssl + (O2 ? (size_t)FL::NSL * SS : 0);
  __shared__ int s_item;
  __shared__ double red[32];
  const StepParams& P = B.P;
  const int64_t nn = P.n;
  const int tid = threadIdx.x;
  CellCounters total;
  unsigned int max_iters = 0;

  for (;;) {
    if (tid == 0) s_item = (int)atomicAdd(B.queue, 1u);
    __syncthreads();
    const int item = s_item;
    __syncthreads();
    if (item >= B.nitems) break;
    const int c = B.items[item].x;
    const int org = B.items[item].y;
    const BatchCase C = B.cases[c];
    const int n = C.n;
    // ---- stage the tile and its halo of this case
    for (int e = tid; e < RS; e += TB) {
      int g = org + e - K::H;
      if (g >= 0 && g < n) {
        int64_t gi = C.off + g;
#pragma unroll
        for (int f = 0; f < FL::NQ; f++) sq[f * RS + e] = P.q[(int64_t)f * nn + gi];
        if (PASS == PASS_CORR) sa0[e] = P.sn[(int64_t)FL::A * nn + gi];
      }
    }
    __syncthreads();
    if (O2) {
      for (int e = tid; e < SS; e += TB) {
        int j = e - 1;
        int gl = org + j - 1;
        if (gl < 0 || gl + 1 >= n) continue;
        int rl = j - 1 + K::H, rr = rl + 1;
        // centre-to-centre distance with the reference's arithmetic (Element::distance)
        double pl = (gl + 0.5) * C.dx, pr = (gl + 1 + 0.5) * C.dx, x = pl - pr;
        double d = dsqrt(x * x);
#pragma unroll
        for (int k = 0; k < NP; k++) {
          ssl[k * SS + e] = ddiv(sq[(FL::A + k) * RS + rr] - sq[(FL::A + k) * RS + rl], d);
          ssl[(NP + k) * SS + e] = ddiv(sq[(FL::R + k) * RS + rr] - sq[(FL::R + k) * RS + rl], d);
          double pR = eos_fix_p(M.eos[k], sq[FL::P * RS + rr]), pL = eos_fix_p(M.eos[k], sq[FL::P * RS + rl]);
          ssl[(2 * NP + k) * SS + e] = ddiv(pR - pL, d);
        }
        ssl[(3 * NP) * SS + e] = ddiv(sq[FL::U * RS + rr] - sq[FL::U * RS + rl], d);
      }
      __syncthreads();
    }
    double dtmax = 1.e10;
    for (int j = tid; j <= TC; j += TB) {
      int gl = org + j - 1;
      if (gl < 0 || gl + 1 >= n) continue;
      int rl = j - 1 + K::H, rr = rl + 1;
      Thermo<NP> tl, tr;
      double ug[3], vg[3];
      if (!O2) {
        cell_thermo<NP, 1>(M, sq, RS, rl, tl, ug);
        cell_thermo<NP, 1>(M, sq, RS, rr, tr, vg);
      } else {
        const int f1 = j + 1;
        const bool hasL = (gl - 1 >= 0), hasR = (gl + 2 < n);
        const double* a0 = (PASS == PASS_CORR) ? sa0 : sq;
        double aL = sq[FL::A * RS + rl], aR = sq[FL::A * RS + rr];
        double aLL = hasL ? a0[rl - 1] : 0., aRR = hasR ? a0[rr + 1] : 0.;
        double pl = (gl + 0.5) * C.dx, pf = pl + 0.5 * C.dx, pr = (gl + 1 + 0.5) * C.dx;
        double y = pf - pl, z = pf - pr;
        constexpr bool kThinc = (TYPES == EOS_DYNAMIC);
        constexpr int kLim = code_limiter(TYPES);
        reconstruct_side<NP, 1, kThinc, kLim>(M, P, sq, RS, rl, ssl, SS, f1, hasL ? j : -1, aL, aR, aLL, dsqrt(y * y), 1.,
                                              tl, ug);
        reconstruct_side<NP, 1, kThinc, kLim>(M, P, sq, RS, rr, ssl, SS, f1, hasR ? j + 2 : -1, aR, aL, aRR, dsqrt(z * z),
                                              -1.,
                                tr, vg);
      }
      double Fn[3];
      Flux<NP> F;
      hllc<NP>(M, tl, ug, tr, vg, C.lcfl, C.lcfl, dtmax, Fn, F);
      F.mom[0] = Fn[0];
#pragma unroll
      for (int k = 0; k < NP; k++) {
        sfl[k * FS + j] = F.a[k];
        sfl[(NP + k) * FS + j] = F.m[k];
        sfl[(2 * NP + k) * FS + j] = F.en[k];
      }
      sfl[(3 * NP) * FS + j] = F.mom[0];
      sfl[(3 * NP + 1) * FS + j] = F.E;
      sfl[(3 * NP + 2) * FS + j] = F.sM;
      sfl[(3 * NP + 3) * FS + j] = F.uStar;
    }
    __syncthreads();
    const int g = org + tid;
    const bool own = tid < TC && g < n;  // this thread's cell of the item
    CellPrim<NP, 1> cp;
    if (own) {
      const int64_t cell = C.off + g;
      double an[NP], rn[NP], pn[NP], aa[NP], am[NP], ae[NP], amom[1] = {0.}, aE = 0.;
      double p0 = P.sn[(int64_t)FL::P * nn + cell];
#pragma unroll
      for (int k = 0; k < NP; k++) {
        an[k] = P.sn[(int64_t)(FL::A + k) * nn + cell];
        rn[k] = P.sn[(int64_t)(FL::R + k) * nn + cell];
        pn[k] = eos_fix_p(M.eos[k], p0);
        aa[k] = am[k] = ae[k] = 0.;
      }
#pragma unroll
      for (int side = 0; side < 2; side++) {
        int j = tid + side;
        int gl = org + j - 1;
        if (gl < 0 || gl + 1 >= n) continue;
        Flux<NP> F;
#pragma unroll
        for (int k = 0; k < NP; k++) {
          F.a[k] = sfl[k * FS + j];
          F.m[k] = sfl[(NP + k) * FS + j];
          F.en[k] = sfl[(2 * NP + k) * FS + j];
        }
        F.mom[0] = sfl[(3 * NP) * FS + j];
        F.E = sfl[(3 * NP + 1) * FS + j];
        F.sM = sfl[(3 * NP + 2) * FS + j];
        F.uStar = sfl[(3 * NP + 3) * FS + j];
        acc_face<NP, 1>(C.coefA, side == 0, F, an, pn, aa, am, ae, amom, aE);
      }
      if (g == 0) boundary_face<NP, 1>(M, P.q, nn, cell, 0, true, C.lcfl, C.coefA, dtmax, an, pn, aa, am, ae, amom, aE);
      if (g == n - 1)
        boundary_face<NP, 1>(M, P.q, nn, cell, 0, false, C.lcfl, C.coefA, dtmax, an, pn, aa, am, ae, amom, aE);
      kapila_rebuild<NP, 1, PASS>(P, M, nn, cell, B.scal[c].dt, an, rn, pn, aa, am, ae, amom, aE, cp);
    }
    SeedGate<NP> sg;
    const bool seeded = P.mlp != nullptr;  // uniform over the launch
    if (seeded) seed_gate<NP, 1>(P, M, own, cp, sg);
    if (own) {
      const int64_t cell = C.off + g;
      CellCounters cc;
      if (seeded)
        kapila_finish<NP, 1, PASS, false, true, (TYPES == EOS_DYNAMIC)>(P, M, nn, cell, cp, sg, cc);
      else
        kapila_finish<NP, 1, PASS, false, false, (TYPES == EOS_DYNAMIC)>(P, M, nn, cell, cp, sg, cc);
      total.relax += cc.relax;
      total.iters += cc.iters;
      total.fallback += cc.fallback;
      total.seeded += cc.seeded;
      total.rejected += cc.rejected;
      total.nonfinite += cc.nonfinite;
      max_iters = max_iters > cc.iters ? max_iters : cc.iters;
    }
    // ---- segmented min: this item's faces belong to case c only
    double v = dtmax;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = dmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((tid & 31) == 0) red[tid >> 5] = v;
    __syncthreads();
    if (tid < 32) {
      v = (tid < TB / 32) ? red[tid] : 1.e10;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v = dmin(v, __shfl_xor_sync(0xffffffffu, v, o));
      if (tid == 0) atomic_min_pos_double(&B.scal[c].dtmax_bits, v);
    }
    __syncthreads();
  }
  // per-thread totals of all items this block processed; the per-bin histogram is not kept in
  // batched mode (relax_calls / newton_evals / newton_max are)
  block_counters(P.stats, total.relax, total.iters, total.fallback, total.seeded, total.rejected, total.nonfinite, 0u,
                 max_iters, false);
}

__global__ void k_batch_finalize(BatchScalars* s, const BatchCase* cases, int ncases, unsigned int* queue, int nq) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c == 0)
    for (int i = 0; i < nq; i++) queue[i] = 0u;
  if (c >= ncases) return;
  double dtmax = __longlong_as_double((long long)s[c].dtmax_bits);
  s[c].t += s[c].dt;
  s[c].it += 1;
  s[c].dt = cases[c].cfl * dtmax;
  s[c].dtmax_bits = (unsigned long long)__double_as_longlong(1.e10);
}

template <int NP, int TB, int PASS, int TYPES>
static cudaError_t batch_one(const BatchParams& B, const ecg_eos* eos, double eps, int grid, cudaStream_t s,
                             bool prepare, int* max_blocks) {
  auto kern = k_batch<NP, TB, PASS, TYPES>;
  const size_t base = BatchTile<NP, TB, PASS>::smem_bytes();
  const size_t sm = base;
  if (prepare) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)base);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(max_blocks, kern, TB, base);
  }
  Model<NP> M;
  for (int k = 0; k < NP; k++) M.eos[k] = make_eos_params(eos[k]);
  M.eps = eps;
  kern<<<grid, TB, sm, s>>>(B, M);
  return cudaGetLastError();
}

template <int NP, int TB, int TYPES = EOS_DYNAMIC>
static cudaError_t batch_tb(int pass, const BatchParams& B, const ecg_eos* eos, double eps, int grid, cudaStream_t s,
                            bool prepare, int* mb) {
  if (pass == PASS_O1) return batch_one<NP, TB, PASS_O1, TYPES>(B, eos, eps, grid, s, prepare, mb);
  if (pass == PASS_PRED) return batch_one<NP, TB, PASS_PRED, TYPES>(B, eos, eps, grid, s, prepare, mb);
  return batch_one<NP, TB, PASS_CORR, TYPES>(B, eos, eps, grid, s, prepare, mb);
}

// fast: two phases, SG liquid then ideal gas, no THINC -- the kernels with the EOS types compiled in
static cudaError_t batch_launch(int np, int tb, int pass, const BatchParams& B, const ecg_eos* eos, double eps,
                                int grid, cudaStream_t s, bool prepare, int* mb, bool fast) {
  // the batched workload's configuration: SG liquid, IG gas, van Leer everywhere
  constexpr int kSgIg = fast_code(eos_types_code<2>(ECG_EOS_SG, ECG_EOS_IG), ECG_LIM_VANLEER);
  if (np == 2 && fast) {
    if (tb == 64) return batch_tb<2, 64, kSgIg>(pass, B, eos, eps, grid, s, prepare, mb);
    if (tb == 128) return batch_tb<2, 128, kSgIg>(pass, B, eos, eps, grid, s, prepare, mb);
    return batch_tb<2, 256, kSgIg>(pass, B, eos, eps, grid, s, prepare, mb);
  }
  if (np == 2) {
    if (tb == 64) return batch_tb<2, 64>(pass, B, eos, eps, grid, s, prepare, mb);
    if (tb == 128) return batch_tb<2, 128>(pass, B, eos, eps, grid, s, prepare, mb);
    return batch_tb<2, 256>(pass, B, eos, eps, grid, s, prepare, mb);
  }
  if (tb == 64) return batch_tb<3, 64>(pass, B, eos, eps, grid, s, prepare, mb);
  if (tb == 128) return batch_tb<3, 128>(pass, B, eos, eps, grid, s, prepare, mb);
  return batch_tb<3, 256>(pass, B, eos, eps, grid, s, prepare, mb);
}

}  // namespace ecg

using namespace ecg;

struct ecg_batch {
  ecg_case c0;
  bool fast = false;  // kernels with the EOS types compiled in apply
  int ncases = 0, np = 2, order = 1, nstate = 0, nq = 0;
  int64_t total = 0;
  double eps = 0.;
  cudaStream_t stream = nullptr;
  std::vector<BatchCase> hcases;
  BatchCase* cases = nullptr;
  BatchScalars* scal = nullptr;
  double* state[2] = {nullptr, nullptr};
  double* half = nullptr;
  double* tmp = nullptr;
  int* done = nullptr;
  unsigned long long* dummy_dtmax = nullptr;
  double* dummy_dt = nullptr;
  DevStats* stats = nullptr;
  unsigned int* queue = nullptr;
  int2* items = nullptr;
  int nitems = 0;
  int tile = 0, threads = 0;
  int grid = 0;
  int cur = 0;
  int newton_cap = 100;
  MlpDev* mlp = nullptr;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
};

namespace {

ecg_status bfail(cudaError_t e, const char* what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return ECG_ERR_CUDA;
}
#define BCUDA(call)                                    \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return bfail(e_, #call);    \
  } while (0)

void drop_graphs(ecg_batch* b) {
  for (int i = 0; i < 2; i++)
    if (b->graph[i]) {
      cudaGraphExecDestroy(b->graph[i]);
      b->graph[i] = nullptr;
    }
}

ecg_status build_items(ecg_batch* b, int tile) {
  std::vector<int2> it;
  for (int c = 0; c < b->ncases; c++)
    for (int s = 0; s < b->hcases[c].n; s += tile - ECG_BATCH_ITEM_TRIM) it.push_back(make_int2(c, s));
  cudaFree(b->items);
  b->items = nullptr;
  BCUDA(cudaMalloc(&b->items, sizeof(int2) * it.size()));
  BCUDA(cudaMemcpy(b->items, it.data(), sizeof(int2) * it.size(), cudaMemcpyHostToDevice));
  b->nitems = (int)it.size();
  return ECG_OK;
}

ecg_status set_shape(ecg_batch* b, int tile) {
  if (tile != 64 && tile != 128 && tile != 256) {
    set_error("tile must be 64, 128 or 256 cells");
    return ECG_ERR_INVALID;
  }
  int sms = 0, dev = 0;
  BCUDA(cudaGetDevice(&dev));
  BCUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  int occ = 1 << 30;
  BatchParams B{};
  for (int pass = 0; pass < 3; pass++) {
    int mb = 0;
    BCUDA(batch_launch(b->np, tile, pass, B, b->c0.eos, b->eps, 0, b->stream, true, &mb, b->fast));
    if ((b->order == 1 && pass == PASS_O1) || (b->order == 2 && pass != PASS_O1)) occ = std::min(occ, std::max(mb, 1));
  }
  b->tile = tile;
  b->threads = tile;
  b->grid = sms * occ;
  drop_graphs(b);
  return build_items(b, tile);
}

ecg_status launch_pass(ecg_batch* b, int pass, double* q, double* sn, double* out, unsigned int* queue) {
  BatchParams B{};
  B.P.done = b->done;
  B.P.q = q;
  B.P.sn = sn;
  B.P.out = out;
  B.P.n = b->total;
  B.P.dt = b->dummy_dt;
  B.P.dtmax_bits = b->dummy_dtmax;
  B.P.stats = b->stats;
  for (int i = 0; i < 4; i++) B.P.lim[i] = b->c0.limiter[i];
  B.P.newton_cap = b->newton_cap;
  set_thinc(B.P, b->c0);
  B.P.pt = b->c0.pt_relaxation;
  B.P.mlp = b->mlp;
  B.cases = b->cases;
  B.scal = b->scal;
  B.items = b->items;
  B.nitems = b->nitems;
  B.queue = queue;
  BCUDA(batch_launch(b->np, b->tile, pass, B, b->c0.eos, b->eps, b->grid, b->stream, false, nullptr, b->fast));
  return ECG_OK;
}

ecg_status launch_step(ecg_batch* b, int parity) {
  double* sn = b->state[parity];
  double* s1 = b->state[1 - parity];
  ecg_status s;
  if (b->order == 1) {
    s = launch_pass(b, PASS_O1, sn, sn, s1, b->queue);
  } else {
    s = launch_pass(b, PASS_PRED, sn, sn, b->half, b->queue);
    if (s == ECG_OK) s = launch_pass(b, PASS_CORR, b->half, sn, s1, b->queue + 1);
  }
  if (s != ECG_OK) return s;
  k_batch_finalize<<<(b->ncases + 255) / 256, 256, 0, b->stream>>>(b->scal, b->cases, b->ncases, b->queue, 2);
  BCUDA(cudaGetLastError());
  return ECG_OK;
}

ecg_status advance(ecg_batch* b, int nsteps) {
  while (nsteps >= 2) {
    if (!b->graph[b->cur]) {
      cudaGraph_t g = nullptr;
      BCUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      ecg_status s1 = launch_step(b, b->cur);
      ecg_status s2 = (s1 == ECG_OK) ? launch_step(b, 1 - b->cur) : s1;
      cudaError_t e = cudaStreamEndCapture(b->stream, &g);
      if (s2 != ECG_OK) {
        if (g) cudaGraphDestroy(g);
        return s2;
      }
      if (e != cudaSuccess) return bfail(e, "cudaStreamEndCapture");
      e = cudaGraphInstantiate(&b->graph[b->cur], g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return bfail(e, "cudaGraphInstantiate");
    }
    BCUDA(cudaGraphLaunch(b->graph[b->cur], b->stream));
    nsteps -= 2;
  }
  if (nsteps == 1) {
    ecg_status s = launch_step(b, b->cur);
    if (s != ECG_OK) return s;
    b->cur = 1 - b->cur;
  }
  return ECG_OK;
}

}  // namespace

extern "C" ecg_status ecg_batch_create(const ecg_case* cs, int32_t ncases, ecg_batch** out) {
  if (!cs || !out || ncases < 1) {
    set_error("bad argument");
    return ECG_ERR_INVALID;
  }
  *out = nullptr;
  const ecg_case& c0 = cs[0];
  if (c0.model != ECG_MODEL_KAPILA || c0.nphases < 2 || c0.nphases > 3 || c0.ptmu) {
    set_error("batched mode runs Kapila cases of 2 or 3 phases without p-T-mu relaxation");
    return ECG_ERR_UNSUPPORTED;
  }
  for (int c = 0; c < ncases; c++) {
    const ecg_case& x = cs[c];
    if (x.ncells[1] != 1 || x.ncells[2] != 1 || x.ncells[0] < 2) {
      set_error("batched mode runs 1D cases");
      return ECG_ERR_UNSUPPORTED;
    }
    if (x.ntransports != 0) {
      set_error("batched mode runs without passive transports");
      return ECG_ERR_UNSUPPORTED;
    }
    if (case_stretched(x)) {
      set_error("batched mode runs uniform meshes");
      return ECG_ERR_UNSUPPORTED;
    }
    if (x.bc[0] != ECG_BC_NONREFLECTING || x.bc[1] != ECG_BC_NONREFLECTING) {
      set_error("batched mode runs non-reflecting sides only");
      return ECG_ERR_UNSUPPORTED;
    }
    if (x.model != c0.model || x.nphases != c0.nphases || x.order != c0.order || x.alpha_null != c0.alpha_null ||
        std::memcmp(x.limiter, c0.limiter, sizeof(x.limiter)) != 0 || std::memcmp(x.eos, c0.eos, sizeof(x.eos)) != 0 ||
        x.pt_relaxation != c0.pt_relaxation) {
      set_error("all cases of a batch share model, phases, EOS, order, limiters and alphaNull");
      return ECG_ERR_INVALID;
    }
  }
  auto b = new ecg_batch();
  b->c0 = c0;
  b->fast = c0.nphases == 2 && c0.eos[0].type == ECG_EOS_SG && c0.eos[1].type == ECG_EOS_IG && !c0.pt_relaxation &&
            c0.order == 2 && c0.limiter[0] == ECG_LIM_VANLEER && c0.limiter[1] == ECG_LIM_VANLEER &&
            c0.limiter[2] == ECG_LIM_VANLEER && c0.limiter[3] == ECG_LIM_VANLEER;
  b->ncases = ncases;
  b->np = c0.nphases;
  b->order = c0.order;
  b->eps = c0.alpha_null ? 1.e-15 : 0.;
  b->nstate = 2 * b->np + 3;  // alpha_k, rho_k, p, u, E
  b->nq = b->nstate - 1;
  int64_t off = 0;
  for (int c = 0; c < ncases; c++) {
    const ecg_case& x = cs[c];
    BatchCase h{};
    h.off = off;
    h.n = x.ncells[0];
    double dX = x.length[0] / (double)x.ncells[0], dY = x.length[1] / (double)x.ncells[1],
           dZ = x.length[2] / (double)x.ncells[2];
    h.dx = dX;
    h.coefA = (dY * dZ) / (dX * dY * dZ);
    h.lcfl = std::min(1.e10, dX);
    h.cfl = x.cfl;
    b->hcases.push_back(h);
    off += h.n;
  }
  b->total = off;
  auto fail = [&](ecg_status s) {
    ecg_batch_destroy(b);
    return s;
  };
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return fail(bfail(e, "cudaStreamCreate"));
  const size_t sb = sizeof(double) * (size_t)b->nstate * (size_t)b->total;
  for (int i = 0; i < 2; i++)
    if ((e = cudaMalloc(&b->state[i], sb)) != cudaSuccess) return fail(bfail(e, "cudaMalloc(state)"));
  if (b->order == 2 && (e = cudaMalloc(&b->half, sizeof(double) * (size_t)b->nq * b->total)) != cudaSuccess)
    return fail(bfail(e, "cudaMalloc(half)"));
  if ((e = cudaMalloc(&b->tmp, sizeof(double) * (size_t)b->total)) != cudaSuccess) return fail(bfail(e, "cudaMalloc"));
  if ((e = cudaMalloc(&b->cases, sizeof(BatchCase) * ncases)) != cudaSuccess) return fail(bfail(e, "cudaMalloc"));
  if ((e = cudaMalloc(&b->scal, sizeof(BatchScalars) * ncases)) != cudaSuccess) return fail(bfail(e, "cudaMalloc"));
  if ((e = cudaMalloc(&b->done, sizeof(int))) != cudaSuccess) return fail(bfail(e, "cudaMalloc"));
  if ((e = cudaMalloc(&b->dummy_dtmax, sizeof(unsigned long long))) != cudaSuccess) return fail(bfail(e, "cudaMalloc"));
  if ((e = cudaMalloc(&b->dummy_dt, sizeof(double))) != cudaSuccess) return fail(bfail(e, "cudaMalloc"));
  if ((e = cudaMalloc(&b->stats, sizeof(DevStats))) != cudaSuccess) return fail(bfail(e, "cudaMalloc"));
  if ((e = cudaMalloc(&b->queue, 2 * sizeof(unsigned int))) != cudaSuccess) return fail(bfail(e, "cudaMalloc"));
  cudaMemcpy(b->cases, b->hcases.data(), sizeof(BatchCase) * ncases, cudaMemcpyHostToDevice);
  std::vector<BatchScalars> hs(ncases);
  double big = 1.e10;
  for (auto& s : hs) {
    s.dt = 1.e-15;
    s.t = 0.;
    std::memcpy(&s.dtmax_bits, &big, sizeof(double));
    s.it = 0;
  }
  cudaMemcpy(b->scal, hs.data(), sizeof(BatchScalars) * ncases, cudaMemcpyHostToDevice);
  cudaMemset(b->done, 0, sizeof(int));
  cudaMemset(b->queue, 0, 2 * sizeof(unsigned int));
  cudaMemset(b->stats, 0, sizeof(DevStats));
  cudaMemset(b->state[0], 0, sb);
  cudaMemset(b->state[1], 0, sb);
  ecg_status s = set_shape(b, 128);
  if (s != ECG_OK) return fail(s);
  *out = b;
  return ECG_OK;
}

extern "C" void ecg_batch_destroy(ecg_batch* b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graphs(b);
  cudaFree(b->state[0]);
  cudaFree(b->state[1]);
  cudaFree(b->half);
  cudaFree(b->tmp);
  cudaFree(b->cases);
  cudaFree(b->scal);
  cudaFree(b->done);
  cudaFree(b->dummy_dtmax);
  cudaFree(b->dummy_dt);
  cudaFree(b->stats);
  cudaFree(b->queue);
  cudaFree(b->items);
  cudaFree(b->mlp);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

extern "C" int64_t ecg_batch_total_cells(const ecg_batch* b) { return b ? b->total : 0; }
extern "C" void* ecg_batch_stream(const ecg_batch* b) { return b ? (void*)b->stream : nullptr; }

extern "C" ecg_status ecg_batch_upload_prim(ecg_batch* b, const double* const* f, int64_t total) {
  if (!b || !f || total != b->total) {
    set_error("bad argument");
    return ECG_ERR_INVALID;
  }
  const int np = b->np;
  const size_t fb = sizeof(double) * (size_t)total;
  double* S = b->state[b->cur];
  for (int i = 0; i < 2 * np + 1; i++) BCUDA(cudaMemcpyAsync(S + (size_t)i * total, f[i], fb, cudaMemcpyHostToDevice, b->stream));
  BCUDA(cudaMemcpyAsync(S + (size_t)(2 * np + 1) * total, f[2 * np + 1], fb, cudaMemcpyHostToDevice, b->stream));
  BCUDA(cudaMemcpyAsync(S + (size_t)(2 * np + 2) * total, f[2 * np + 4], fb, cudaMemcpyHostToDevice, b->stream));
  BCUDA(cudaStreamSynchronize(b->stream));
  return ECG_OK;
}

namespace ecg {
__global__ void k_derived(const double* __restrict__ S, int64_t n, int np, int dim, ecg_eos e0, ecg_eos e1, ecg_eos e2,
                          double eps, double* pmix, double* T, double* Y);
}

extern "C" ecg_status ecg_batch_download_prim(ecg_batch* b, double* const* f, int64_t total) {
  if (!b || !f || total != b->total) {
    set_error("bad argument");
    return ECG_ERR_INVALID;
  }
  const int np = b->np;
  const size_t fb = sizeof(double) * (size_t)total;
  const double* S = b->state[b->cur];
  k_derived<<<(unsigned)((total + 255) / 256), 256, 0, b->stream>>>(S, total, np, 1, b->c0.eos[0], b->c0.eos[1],
                                                                     b->c0.eos[2], b->eps, b->tmp, nullptr, nullptr);
  BCUDA(cudaGetLastError());
  for (int i = 0; i < 2 * np; i++) BCUDA(cudaMemcpyAsync(f[i], S + (size_t)i * total, fb, cudaMemcpyDeviceToHost, b->stream));
  BCUDA(cudaMemcpyAsync(f[2 * np], b->tmp, fb, cudaMemcpyDeviceToHost, b->stream));
  BCUDA(cudaMemcpyAsync(f[2 * np + 1], S + (size_t)(2 * np + 1) * total, fb, cudaMemcpyDeviceToHost, b->stream));
  BCUDA(cudaMemcpyAsync(f[2 * np + 4], S + (size_t)(2 * np + 2) * total, fb, cudaMemcpyDeviceToHost, b->stream));
  BCUDA(cudaStreamSynchronize(b->stream));
  std::memset(f[2 * np + 2], 0, fb);
  std::memset(f[2 * np + 3], 0, fb);
  return ECG_OK;
}

extern "C" ecg_status ecg_batch_step(ecg_batch* b, int32_t nsteps, double* dt, double* t, ecg_step_stats* stats) {
  if (!b || nsteps < 0) {
    set_error("bad argument");
    return ECG_ERR_INVALID;
  }
  const int nc = b->ncases;
  if (dt || t) {
    // the caller's per-case dt / t seed the device scalars
    std::vector<BatchScalars> hs(nc);
    BCUDA(cudaMemcpy(hs.data(), b->scal, sizeof(BatchScalars) * nc, cudaMemcpyDeviceToHost));
    for (int c = 0; c < nc; c++) {
      if (dt) hs[c].dt = dt[c];
      if (t) hs[c].t = t[c];
    }
    BCUDA(cudaMemcpyAsync(b->scal, hs.data(), sizeof(BatchScalars) * nc, cudaMemcpyHostToDevice, b->stream));
  }
  BCUDA(cudaMemsetAsync(b->stats, 0, sizeof(DevStats), b->stream));
  ecg_status s = advance(b, nsteps);
  if (s != ECG_OK) return s;
  DevStats ds{};
  BCUDA(cudaMemcpyAsync(&ds, b->stats, sizeof(ds), cudaMemcpyDeviceToHost, b->stream));
  if (dt || t) {
    std::vector<BatchScalars> hs(nc);
    BCUDA(cudaMemcpyAsync(hs.data(), b->scal, sizeof(BatchScalars) * nc, cudaMemcpyDeviceToHost, b->stream));
    BCUDA(cudaStreamSynchronize(b->stream));
    for (int c = 0; c < nc; c++) {
      if (dt) dt[c] = hs[c].dt;
      if (t) t[c] = hs[c].t;
    }
  }
  BCUDA(cudaStreamSynchronize(b->stream));
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->cell_updates = (int64_t)nsteps * b->total;
    stats->relax_calls = (int64_t)ds.relax_calls;
    stats->newton_evals = (int64_t)ds.newton_evals;
    stats->newton_fallback = (int64_t)ds.newton_fallback;
    stats->newton_max = (int64_t)ds.newton_max;
    stats->seeded = (int64_t)ds.seeded;
    stats->seed_rejected = (int64_t)ds.seed_rejected;
    stats->nonfinite_cells = (int64_t)ds.nonfinite;
    for (int i = 0; i < 16; i++) stats->newton_hist[i] = (int64_t)ds.hist[i];
  }
  return ECG_OK;
}

extern "C" ecg_status ecg_batch_set_seed_model(ecg_batch* b, const ecg_mlp* m) {
  if (!b) {
    set_error("null batch");
    return ECG_ERR_INVALID;
  }
  drop_graphs(b);
  if (!m) {
    cudaFree(b->mlp);
    b->mlp = nullptr;
    return ECG_OK;
  }
  return mlp_upload(m, b->np, false, &b->mlp, b->stream);
}

extern "C" ecg_status ecg_batch_set_shape(ecg_batch* b, int32_t tile, int32_t threads) {
  if (!b) {
    set_error("null batch");
    return ECG_ERR_INVALID;
  }
  if (tile == 0) {
    int32_t t2 = 0, th = 0;
    return ecg_batch_autotune(b, &t2, &th);
  }
  if (threads != 0 && threads != tile) {
    set_error("one thread per cell of a tile: threads must equal tile");
    return ECG_ERR_INVALID;
  }
  return set_shape(b, tile);
}

// Times two steps of every candidate tile on a copy of the current state and keeps the fastest.
extern "C" ecg_status ecg_batch_autotune(ecg_batch* b, int32_t* tile, int32_t* threads) {
  if (!b) {
    set_error("null batch");
    return ECG_ERR_INVALID;
  }
  const size_t sb = sizeof(double) * (size_t)b->nstate * (size_t)b->total;
  double* save = nullptr;
  BatchScalars* ssave = nullptr;
  BCUDA(cudaMalloc(&save, sb));
  cudaError_t e = cudaMalloc(&ssave, sizeof(BatchScalars) * b->ncases);
  if (e != cudaSuccess) {
    cudaFree(save);
    return bfail(e, "cudaMalloc");
  }
  const int cur0 = b->cur;
  cudaMemcpyAsync(save, b->state[cur0], sb, cudaMemcpyDeviceToDevice, b->stream);
  cudaMemcpyAsync(ssave, b->scal, sizeof(BatchScalars) * b->ncases, cudaMemcpyDeviceToDevice, b->stream);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int best = 128;
  float best_ms = 1e30f;
  ecg_status st = ECG_OK;
  for (int cand : {64, 128, 256}) {
    st = set_shape(b, cand);
    if (st != ECG_OK) break;
    b->cur = cur0;
    st = advance(b, 2);  // warm-up / graph capture
    if (st != ECG_OK) break;
    cudaMemcpyAsync(b->state[cur0], save, sb, cudaMemcpyDeviceToDevice, b->stream);
    cudaMemcpyAsync(b->scal, ssave, sizeof(BatchScalars) * b->ncases, cudaMemcpyDeviceToDevice, b->stream);
    b->cur = cur0;
    cudaEventRecord(e0, b->stream);
    st = advance(b, 2);
    cudaEventRecord(e1, b->stream);
    if (st != ECG_OK) break;
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best_ms) {
      best_ms = ms;
      best = cand;
    }
    cudaMemcpyAsync(b->state[cur0], save, sb, cudaMemcpyDeviceToDevice, b->stream);
    cudaMemcpyAsync(b->scal, ssave, sizeof(BatchScalars) * b->ncases, cudaMemcpyDeviceToDevice, b->stream);
  }
  cudaStreamSynchronize(b->stream);
  b->cur = cur0;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(save);
  cudaFree(ssave);
  cudaMemsetAsync(b->stats, 0, sizeof(DevStats), b->stream);
  if (st != ECG_OK) return st;
  st = set_shape(b, best);
  if (st != ECG_OK) return st;
  if (tile) *tile = best;
  if (threads) *threads = best;
  return ECG_OK;
}
