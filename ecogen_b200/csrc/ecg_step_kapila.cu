// Kapila (PUEq) step kernels: first-order step, MUSCL predictor and MUSCL corrector.
// See ecg_step.cuh for the work decomposition.
#include <cuda_runtime.h>

#include "ecg_mlp_device.cuh"
#include "ecg_step.cuh"

namespace ecg {

template <int NP, int DIM, int PASS>
struct KapilaStep {
  using FL = Fields<NP, DIM>;
  using TS = TileShape<DIM>;
  static constexpr int H = (PASS == PASS_O1) ? 1 : 2;
  static constexpr int NTH = TS::X * TS::Y * TS::Z;
  static constexpr bool O2 = (PASS != PASS_O1);

  __host__ __device__ static constexpr int ext(int a) { return a == 0 ? TS::X : (a == 1 ? TS::Y : TS::Z); }
  __host__ __device__ static constexpr int lines(int a) { return NTH / ext(a); }
  __host__ __device__ static constexpr int rlen(int a) { return ext(a) + 2 * H; }
  __host__ __device__ static constexpr int region(int a) { return rlen(a) * lines(a); }
  __host__ __device__ static constexpr int nslope(int a) { return O2 ? (ext(a) + 3) * lines(a) : 0; }
  __host__ __device__ static constexpr int nface(int a) { return (ext(a) + 1) * lines(a); }
  __host__ __device__ static constexpr int cmax(int a, int b) { return a > b ? a : b; }
  __host__ __device__ static constexpr int RMAX() {
    return cmax(region(0), cmax(DIM > 1 ? region(1) : 0, DIM > 2 ? region(2) : 0));
  }
  __host__ __device__ static constexpr int SMAX() {
    return cmax(nslope(0), cmax(DIM > 1 ? nslope(1) : 0, DIM > 2 ? nslope(2) : 0));
  }
  __host__ __device__ static constexpr int FMAX() {
    return cmax(nface(0), cmax(DIM > 1 ? nface(1) : 0, DIM > 2 ? nface(2) : 0));
  }
  static constexpr int NA0 = (PASS == PASS_CORR) ? 1 : 0;  // separate time-n alpha_0 plane
  static constexpr size_t smem_bytes() {
    return sizeof(double) * ((size_t)RMAX() * (FL::NQ + NA0) + (size_t)SMAX() * FL::NSL + (size_t)FMAX() * FL::NFL);
  }
};

// Reconstructs one side of an internal face (CellInterfaceO2Cartesian::solveRiemann
// src/Order2/CellInterfaceO2Cartesian.cpp:101-160 with CellO2Cartesian::computeLocalSlopes
// src/Order2/CellO2Cartesian.cpp:23-171 on a Cartesian mesh): the limited slope combines the slope
// of this face (s1) and of the face on the opposite side of the cell along the same axis (s2, zero
// when that face is a boundary); the interface detector decides between the global and interface
// limiters; the state is extrapolated by `sign * slope * dist` and clamped.
template <int NP, int DIM>
__device__ __forceinline__ void reconstruct_side(const Model<NP>& M, const int lim[4], const double* sq, int RS, int rc,
                                                 const double* ssl, int SS, int f1, int f2, double alphaCell,
                                                 double alphaOther, double alphaAfter, double dist, double sign,
                                                 Thermo<NP>& t, double u[3]) {
  using FL = Fields<NP, DIM>;
  const bool iface = (alphaCell >= 1.e-4) && (alphaCell <= 1. - 1.e-4) &&
                     ((alphaOther - alphaCell) * (alphaCell - alphaAfter) >= 1.e-8);
  const int lg = iface ? lim[1] : lim[0];
  const int lv = iface ? lim[3] : lim[2];
#pragma unroll
  for (int k = 0; k < NP; k++) {
    double s1a = ssl[(k)*SS + f1], s1r = ssl[(NP + k) * SS + f1], s1p = ssl[(2 * NP + k) * SS + f1];
    double s2a = 0., s2r = 0., s2p = 0.;
    if (f2 >= 0) {
      s2a = ssl[(k)*SS + f2];
      s2r = ssl[(NP + k) * SS + f2];
      s2p = ssl[(2 * NP + k) * SS + f2];
    }
    double la = limiter(lv, s1a, s2a), lr = limiter(lg, s1r, s2r), lp = limiter(lg, s1p, s2p);
    double a = sq[(FL::A + k) * RS + rc], r = sq[(FL::R + k) * RS + rc];
    double p = eos_fix_p(M.eos[k], sq[FL::P * RS + rc]);  // phase pressure of the cell
    a += (sign * la) * dist;
    r += (sign * lr) * dist;
    p += (sign * lp) * dist;
    phase_fix_ar(M.eps, a, r);
    p = eos_fix_p(M.eos[k], p);
    eos_rho_max(M.eos[k], r);
    t.a[k] = a;
    t.r[k] = r;
    t.p[k] = p;
  }
  u[0] = u[1] = u[2] = 0.;
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    double s1 = ssl[(3 * NP + d) * SS + f1];
    double s2 = (f2 >= 0) ? ssl[(3 * NP + d) * SS + f2] : 0.;
    double l = limiter(lg, s1, s2);
    u[d] = sq[(FL::U + d) * RS + rc] + (sign * l) * dist;
  }
  fulfill<NP>(M, t);
}

template <int NP, int DIM>
__device__ __forceinline__ void cell_thermo(const Model<NP>& M, const double* sq, int RS, int rc, Thermo<NP>& t,
                                            double u[3]) {
  using FL = Fields<NP, DIM>;
#pragma unroll
  for (int k = 0; k < NP; k++) {
    t.a[k] = sq[(FL::A + k) * RS + rc];
    t.r[k] = sq[(FL::R + k) * RS + rc];
    t.p[k] = eos_fix_p(M.eos[k], sq[FL::P * RS + rc]);
  }
  u[0] = u[1] = u[2] = 0.;
#pragma unroll
  for (int d = 0; d < DIM; d++) u[d] = sq[(FL::U + d) * RS + rc];
  fulfill<NP>(M, t);
}

template <int NP, int DIM>
__device__ __forceinline__ void acc_face(double cA, bool add, const Flux<NP>& F, const double an[NP],
                                         const double pn[NP], double aa[NP], double am[NP], double ae[NP],
                                         double amom[DIM], double& aE) {
  // FluxUEq::addFlux/subtractFlux src/Models/UEq/FluxUEq.cpp:61,85 then
  // FluxPUEq::addNonCons/subtractNonCons src/Models/PUEq/FluxPUEq.cpp:44,56 (time-n alpha_k, p_k).
  if (add) {
#pragma unroll
    for (int k = 0; k < NP; k++) {
      aa[k] += cA * F.a[k];
      am[k] += cA * F.m[k];
      ae[k] += cA * F.en[k];
    }
#pragma unroll
    for (int d = 0; d < DIM; d++) amom[d] += cA * F.mom[d];
    aE += cA * F.E;
#pragma unroll
    for (int k = 0; k < NP; k++) {
      aa[k] += -cA * an[k] * F.sM;
      ae[k] += cA * an[k] * pn[k] * F.uStar;
    }
  } else {
#pragma unroll
    for (int k = 0; k < NP; k++) {
      aa[k] -= cA * F.a[k];
      am[k] -= cA * F.m[k];
      ae[k] -= cA * F.en[k];
    }
#pragma unroll
    for (int d = 0; d < DIM; d++) amom[d] -= cA * F.mom[d];
    aE -= cA * F.E;
#pragma unroll
    for (int k = 0; k < NP; k++) {
      aa[k] -= -cA * an[k] * F.sM;
      ae[k] -= cA * an[k] * pn[k] * F.uStar;
    }
  }
}

template <int NP, int DIM, int PASS, bool PTMU>
__global__ void __launch_bounds__(KapilaStep<NP, DIM, PASS>::NTH)
    k_kapila_step(StepParams P, Geometry G, Model<NP> M) {
  using K = KapilaStep<NP, DIM, PASS>;
  using FL = Fields<NP, DIM>;
  using TS = TileShape<DIM>;
  extern __shared__ double smem[];
  constexpr int RS = K::RMAX();
  constexpr int SS = (K::SMAX() > 0) ? K::SMAX() : 1;
  constexpr int FS = K::FMAX();
  double* sq = smem;                                       // [NQ][RS]
  double* sa0 = sq + (size_t)FL::NQ * RS;                  // [NA0][RS]
  double* ssl = sa0 + (size_t)K::NA0 * RS;                 // [NSL][SS]
  double* sfl = ssl + (K::O2 ? (size_t)FL::NSL * SS : 0);  // [NFL][FS]

  if (*P.done) return;  // stop condition reached earlier in a captured step sequence
  const int tid = threadIdx.x;
  const int org[3] = {(int)blockIdx.x * TS::X, (int)blockIdx.y * TS::Y, (int)blockIdx.z * TS::Z};
  const int lc[3] = {tid % TS::X, (tid / TS::X) % TS::Y, tid / (TS::X * TS::Y)};
  const int gc[3] = {org[0] + lc[0], org[1] + lc[1], org[2] + lc[2]};
  const bool active = gc[0] < G.n[0] && gc[1] < G.n[1] && gc[2] < G.n[2];
  const int64_t nn = P.n;
  const int64_t cell = (int64_t)gc[0] + (int64_t)gc[1] * G.n[0] + (int64_t)gc[2] * G.n[0] * G.n[1];

  // time-n state of the own cell: non-conservative terms and U^n
  double an[NP], rn[NP], pn[NP];
  double aa[NP], am[NP], ae[NP], amom[DIM], aE = 0.;
#pragma unroll
  for (int k = 0; k < NP; k++) {
    an[k] = rn[k] = pn[k] = 0.;
    aa[k] = am[k] = ae[k] = 0.;
  }
#pragma unroll
  for (int d = 0; d < DIM; d++) amom[d] = 0.;
  if (active) {
    double p0 = P.sn[(int64_t)FL::P * nn + cell];
#pragma unroll
    for (int k = 0; k < NP; k++) {
      an[k] = P.sn[(int64_t)(FL::A + k) * nn + cell];
      rn[k] = P.sn[(int64_t)(FL::R + k) * nn + cell];
      pn[k] = eos_fix_p(M.eos[k], p0);
    }
  }
  double dtmax = 1.e10;

#pragma unroll 1
  for (int ax = 0; ax < DIM; ax++) {
    const int T = K::ext(ax), RL = K::rlen(ax), NL = K::lines(ax);
    const int b1 = (ax == 0) ? 1 : 0, b2 = (ax == 2) ? 1 : 2;  // the two other axes
    const int e1 = K::ext(b1);
    const int nax = G.n[ax];
    // ---- stage tile + halo along ax
    for (int e = tid; e < K::region(ax); e += K::NTH) {
      int la = e % RL - K::H, line = e / RL;
      int l1 = line % e1, l2 = line / e1;
      int g[3];
      g[ax] = org[ax] + la;
      g[b1] = org[b1] + l1;
      g[b2] = org[b2] + l2;
      bool in = g[ax] >= 0 && g[ax] < nax && g[b1] < G.n[b1] && g[b2] < G.n[b2];
      if (in) {
        int64_t c = (int64_t)g[0] + (int64_t)g[1] * G.n[0] + (int64_t)g[2] * G.n[0] * G.n[1];
#pragma unroll
        for (int f = 0; f < FL::NQ; f++) sq[f * RS + e] = P.q[(int64_t)f * nn + c];
        if (K::NA0) sa0[e] = P.sn[(int64_t)FL::A * nn + c];
      }
    }
    __syncthreads();
    // ---- face slopes (MUSCL): face j between local cells j-1 and j, j in [-1, T+1]
    if (K::O2) {
      for (int e = tid; e < K::nslope(ax); e += K::NTH) {
        int j = e % (T + 3) - 1, line = e / (T + 3);
        int gl = org[ax] + j - 1;
        if (gl < 0 || gl + 1 >= nax) continue;  // not an internal face
        int rl = line * RL + (j - 1 + K::H), rr = rl + 1;
        double d = G.dcc[ax][gl];
#pragma unroll
        for (int k = 0; k < NP; k++) {
          ssl[k * SS + e] = (sq[(FL::A + k) * RS + rr] - sq[(FL::A + k) * RS + rl]) / d;
          ssl[(NP + k) * SS + e] = (sq[(FL::R + k) * RS + rr] - sq[(FL::R + k) * RS + rl]) / d;
          double pr = eos_fix_p(M.eos[k], sq[FL::P * RS + rr]), pl = eos_fix_p(M.eos[k], sq[FL::P * RS + rl]);
          ssl[(2 * NP + k) * SS + e] = (pr - pl) / d;
        }
#pragma unroll
        for (int dd = 0; dd < DIM; dd++)
          ssl[(3 * NP + dd) * SS + e] = (sq[(FL::U + dd) * RS + rr] - sq[(FL::U + dd) * RS + rl]) / d;
      }
      __syncthreads();
    }
    // ---- face fluxes: face j between local cells j-1 and j, j in [0, T]
    for (int e = tid; e < K::nface(ax); e += K::NTH) {
      int j = e % (T + 1), line = e / (T + 1);
      int l1 = line % e1, l2 = line / e1;
      int gl = org[ax] + j - 1;
      if (gl < 0 || gl + 1 >= nax || org[b1] + l1 >= G.n[b1] || org[b2] + l2 >= G.n[b2]) continue;
      int rl = line * RL + (j - 1 + K::H), rr = rl + 1;
      Thermo<NP> tl, tr;
      double ug[3], vg[3];
      if (!K::O2) {
        cell_thermo<NP, DIM>(M, sq, RS, rl, tl, ug);
        cell_thermo<NP, DIM>(M, sq, RS, rr, tr, vg);
      } else {
        const int fs = line * (T + 3);
        const int f1 = fs + j + 1;                         // this face
        const bool hasL = (gl - 1 >= 0), hasR = (gl + 2 < nax);
        const int f2l = hasL ? fs + j : -1;                // face (j-2, j-1)
        const int f2r = hasR ? fs + j + 2 : -1;            // face (j, j+1)
        const double* a0 = K::NA0 ? sa0 : sq;              // time-n alpha_0 planes
        double aL = sq[FL::A * RS + rl], aR = sq[FL::A * RS + rr];
        double aLL = hasL ? a0[rl - 1] : 0., aRR = hasR ? a0[rr + 1] : 0.;
        reconstruct_side<NP, DIM>(M, P.lim, sq, RS, rl, ssl, SS, f1, f2l, aL, aR, aLL, G.dfl[ax][gl], 1., tl, ug);
        reconstruct_side<NP, DIM>(M, P.lim, sq, RS, rr, ssl, SS, f1, f2r, aR, aL, aRR, G.dfr[ax][gl], -1., tr, vg);
      }
      double ul[3], ur[3], Fn[3];
      to_local(ax, false, ug, ul);
      to_local(ax, false, vg, ur);
      Flux<NP> F;
      hllc<NP>(M, tl, ul, tr, ur, G.lcfl, G.lcfl, dtmax, Fn, F);
      to_global(ax, false, Fn, F.mom);
#pragma unroll
      for (int k = 0; k < NP; k++) {
        sfl[k * FS + e] = F.a[k];
        sfl[(NP + k) * FS + e] = F.m[k];
        sfl[(2 * NP + k) * FS + e] = F.en[k];
      }
#pragma unroll
      for (int d = 0; d < DIM; d++) sfl[(3 * NP + d) * FS + e] = F.mom[d];
      sfl[(3 * NP + DIM) * FS + e] = F.E;
      sfl[(3 * NP + DIM + 1) * FS + e] = F.sM;
      sfl[(3 * NP + DIM + 2) * FS + e] = F.uStar;
    }
    __syncthreads();
    // ---- accumulate the two faces of this axis into the own cell (left +, right -)
    if (active) {
      int la = lc[ax];
      int line = lc[b1] + lc[b2] * e1;
      const double cA = G.coefA[ax];
#pragma unroll
      for (int side = 0; side < 2; side++) {
        int j = la + side;
        int gl = org[ax] + j - 1;
        if (gl < 0 || gl + 1 >= nax) continue;  // boundary face: handled below
        int e = line * (T + 1) + j;
        Flux<NP> F;
#pragma unroll
        for (int k = 0; k < NP; k++) {
          F.a[k] = sfl[k * FS + e];
          F.m[k] = sfl[(NP + k) * FS + e];
          F.en[k] = sfl[(2 * NP + k) * FS + e];
        }
#pragma unroll
        for (int d = 0; d < DIM; d++) F.mom[d] = sfl[(3 * NP + d) * FS + e];
        F.E = sfl[(3 * NP + DIM) * FS + e];
        F.sM = sfl[(3 * NP + DIM + 1) * FS + e];
        F.uStar = sfl[(3 * NP + DIM + 2) * FS + e];
        acc_face<NP, DIM>(cA, side == 0, F, an, pn, aa, am, ae, amom, aE);
      }
    }
    __syncthreads();
  }

  // per-thread counters, reduced per block at the end
  unsigned int c_relax = 0, c_iters = 0, c_fallback = 0, c_seeded = 0, c_rejected = 0, c_nonfinite = 0, c_ptmu = 0;
  if (active) {
    // ---- boundary faces (non-reflecting: HLLC(cell, cell), BoundCondNonReflecting::solveRiemannBoundary
    //      src/BoundConds/BoundCondNonReflecting.cpp:62), subtracted from the cell (BoundCond::computeFlux :61)
#pragma unroll 1
    for (int bf = 0; bf < 2 * DIM; bf++) {
      int ax = bf >> 1;
      bool neg = (bf & 1) == 0;
      if (neg ? (gc[ax] != 0) : (gc[ax] != G.n[ax] - 1)) continue;
      Thermo<NP> t;
      double ug[3], ul[3], Fn[3];
#pragma unroll
      for (int k = 0; k < NP; k++) {
        t.a[k] = P.q[(int64_t)(FL::A + k) * nn + cell];
        t.r[k] = P.q[(int64_t)(FL::R + k) * nn + cell];
        t.p[k] = eos_fix_p(M.eos[k], P.q[(int64_t)FL::P * nn + cell]);
      }
      ug[0] = ug[1] = ug[2] = 0.;
#pragma unroll
      for (int d = 0; d < DIM; d++) ug[d] = P.q[(int64_t)(FL::U + d) * nn + cell];
      fulfill<NP>(M, t);
      to_local(ax, neg, ug, ul);
      Flux<NP> F;
      hllc<NP>(M, t, ul, t, ul, G.lcfl, G.lcfl, dtmax, Fn, F);
      to_global(ax, neg, Fn, F.mom);
      acc_face<NP, DIM>(G.coefA[ax], false, F, an, pn, aa, am, ae, amom, aE);
    }

    // ---- U^n (FluxUEq::buildCons src/Models/UEq/FluxUEq.cpp:147) and time evolution
    //      (Cell::timeEvolution src/Order1/Cell.cpp:286: m_cons*dt then + U^n)
    const double dt = *P.dt;
    const double scale = (PASS == PASS_PRED) ? 0.5 * dt : dt;
    double rhon = 0.;
#pragma unroll
    for (int k = 0; k < NP; k++) rhon += an[k] * rn[k];
#pragma unroll
    for (int k = 0; k < NP; k++) {
      double Uk_m = an[k] * rn[k];
      double Uk_e = an[k] * rn[k] * eos_e(M.eos[k], M.eps, rn[k], pn[k]);
      aa[k] = aa[k] * scale + 1. * an[k];
      am[k] = am[k] * scale + 1. * Uk_m;
      ae[k] = ae[k] * scale + 1. * Uk_e;
    }
    double un[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      un[d] = P.sn[(int64_t)(FL::U + d) * nn + cell];
      amom[d] = amom[d] * scale + 1. * (rhon * un[d]);
    }
    double En = P.sn[(int64_t)FL::E * nn + cell];
    aE = aE * scale + 1. * (rhon * En);

    // ---- buildPrim (FluxUEq::buildPrim src/Models/UEq/FluxUEq.cpp:161-209)
    double un_sum = 0.;
    if (M.eps > 1.e-20) {
#pragma unroll
      for (int k = 0; k < NP; k++) {
        if (aa[k] < 0.) aa[k] = 0.;
        if (aa[k] > 1.) aa[k] = 1.;
        un_sum += aa[k];
      }
    } else {
#pragma unroll
      for (int k = 0; k < NP; k++) {
        if (aa[k] <= 1.e-15) aa[k] = 1e-15;
        if (aa[k] >= 1. - 1.e-15) aa[k] = 1.0 - 1e-15;
        un_sum += aa[k];
      }
    }
    double a[NP], r[NP], pk[NP];
    double rhoMel = 0.;
#pragma unroll
    for (int k = 0; k < NP; k++) {
      aa[k] /= un_sum;
      rhoMel += am[k];
      a[k] = aa[k];
      r[k] = am[k] / dmax(aa[k], M.eps);
      if (M.eos[k].type == ECG_EOS_NASG && r[k] > 1. / M.eos[k].b - 1.) {  // verifyAndCorrectDensityMax(mass)
        r[k] = 1. / M.eos[k].b - 1.;
        a[k] = am[k] / r[k];
      }
      double ek = ae[k] / dmax(am[k], M.eps);
      pk[k] = eos_p(M.eos[k], M.eps, r[k], ek);
      phase_fix_ar(M.eps, a[k], r[k]);
      pk[k] = eos_fix_p(M.eos[k], pk[k]);
    }
    double u[DIM], usq = 0.;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      u[d] = amom[d] / rhoMel;
      if (fabs(u[d]) < 1.e-8) u[d] = 0.;
      usq += u[d] * u[d];
    }
    double E = aE / rhoMel;
    // mixture density (and internal energy for p-T-mu) of the rebuilt state
    double rhomix = 0.;
#pragma unroll
    for (int k = 0; k < NP; k++) rhomix += a[k] * r[k];

    // ---- relaxations (Model::relaxations src/Models/Model.cpp:74): pressure, then p-T-mu
    RelaxStats rs;
    double seed = 0.;
    bool use_seed = false;
    if (P.mlp != nullptr) {
      seed = mlp_seed<NP>(P.mlp, P.mlp_nin, a, r, pk);
      use_seed = true;
    }
    double a0[NP], r0[NP], p0[NP];
#pragma unroll
    for (int k = 0; k < NP; k++) { a0[k] = a[k]; r0[k] = r[k]; p0[k] = pk[k]; }
    double pstar = 0.;
    bool relaxed = relax_pinf<NP>(M, a, r, pk, pstar, rs, seed, use_seed, P.newton_cap);
    if (relaxed) {
#pragma unroll
      for (int k = 0; k < NP; k++) pk[k] = pstar;
      if (P.rec_x != nullptr && !rs.fallback) record_pair<NP>(P.rec_x, P.rec_y, P.rec_count, P.rec_max, a0, r0, p0, pstar);
    }
    if (PTMU) {
      // mixture internal energy of the rebuilt state (MixUEq::computeMixtureVariables :136), which
      // RelaxationPTMu reads before any fulfillState
      double emix = 0.;
#pragma unroll
      for (int k = 0; k < NP; k++) {
        double Y = a0[k] * r0[k] / dmax(rhomix, M.eps);
        emix += Y * eos_e(M.eos[k], M.eps, r0[k], p0[k]);
      }
      bool err = false;
      if (relax_ptmu<NP>(M, P.ptmu_liq, P.ptmu_vap, P.pcrit, a, r, pk, rhomix, emix, err)) {
        rhomix = 0.;
#pragma unroll
        for (int k = 0; k < NP; k++) rhomix += a[k] * r[k];
      }
      if (err) c_ptmu = 1;
    }

    // ---- energy correction (FluxPUEq::correctionEnergy) and clamps
    double p = correction_pressure<NP>(M, a, r, rhomix, E, usq);
#pragma unroll
    for (int k = 0; k < NP; k++) phase_fix_ar(M.eps, a[k], r[k]);

    // ---- store
    bool finite = isfinite(p) && isfinite(E);
#pragma unroll
    for (int k = 0; k < NP; k++) {
      P.out[(int64_t)(FL::A + k) * nn + cell] = a[k];
      P.out[(int64_t)(FL::R + k) * nn + cell] = r[k];
      finite = finite && isfinite(a[k]) && isfinite(r[k]);
    }
    P.out[(int64_t)FL::P * nn + cell] = p;
#pragma unroll
    for (int d = 0; d < DIM; d++) P.out[(int64_t)(FL::U + d) * nn + cell] = u[d];
    if (PASS != PASS_PRED) P.out[(int64_t)FL::E * nn + cell] = E;

    // ---- counters
    if (relaxed) {
      c_relax = 1;
      c_iters = (unsigned int)rs.iters;
      c_fallback = rs.fallback ? 1u : 0u;
      c_seeded = rs.seeded ? 1u : 0u;
      c_rejected = rs.rejected ? 1u : 0u;
    }
    c_nonfinite = finite ? 0u : 1u;
  }
  block_counters(P.stats, c_relax, c_iters, c_fallback, c_seeded, c_rejected, c_nonfinite, c_ptmu);

  // ---- dtMax: block min, one atomic per block
  __shared__ double red[32];
  double v = dtmax;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = dmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((tid & 31) == 0) red[tid >> 5] = v;
  __syncthreads();
  if (tid < 32) {
    v = (tid < K::NTH / 32) ? red[tid] : 1.e10;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = dmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (tid == 0) atomic_min_pos_double(P.dtmax_bits, v);
  }
}

}  // namespace ecg

// ------------------------------------------------------------------------------- host launchers
namespace ecg {

template <int NP, int DIM, int PASS, bool PTMU>
static cudaError_t launch_one(const StepParams& P, const Geometry& G, const ecg_eos* eos, double eps, cudaStream_t s,
                              bool prepare) {
  using K = KapilaStep<NP, DIM, PASS>;
  using TS = TileShape<DIM>;
  auto kern = k_kapila_step<NP, DIM, PASS, PTMU>;
  const size_t sm = K::smem_bytes();
  if (prepare) return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  Model<NP> M;
  for (int k = 0; k < NP; k++) {
    M.eos[k].type = eos[k].type;
    M.eos[k].gamma = eos[k].gamma;
    M.eos[k].pinf = eos[k].pinf;
    M.eos[k].b = eos[k].b;
    M.eos[k].cv = eos[k].cv;
    M.eos[k].eref = eos[k].eref;
    M.eos[k].sref = eos[k].sref;
  }
  M.eps = eps;
  dim3 grid((G.n[0] + TS::X - 1) / TS::X, (G.n[1] + TS::Y - 1) / TS::Y, (G.n[2] + TS::Z - 1) / TS::Z);
  kern<<<grid, K::NTH, sm, s>>>(P, G, M);
  return cudaGetLastError();
}

template <int NP, int DIM, bool PTMU>
static cudaError_t launch_pass(int pass, const StepParams& P, const Geometry& G, const ecg_eos* eos, double eps,
                               cudaStream_t s, bool prepare) {
  switch (pass) {
    case PASS_O1: return launch_one<NP, DIM, PASS_O1, PTMU>(P, G, eos, eps, s, prepare);
    case PASS_PRED: return launch_one<NP, DIM, PASS_PRED, PTMU>(P, G, eos, eps, s, prepare);
    default: return launch_one<NP, DIM, PASS_CORR, PTMU>(P, G, eos, eps, s, prepare);
  }
}

// Launches (or, with prepare, configures) one pass of the Kapila step for a case shape.
cudaError_t kapila_launch(int np, int dim, bool ptmu, int pass, const StepParams& P, const Geometry& G,
                          const ecg_eos* eos, double eps, cudaStream_t s, bool prepare) {
  if (np == 2) {
    if (ptmu) {
      if (dim == 1) return launch_pass<2, 1, true>(pass, P, G, eos, eps, s, prepare);
      if (dim == 2) return launch_pass<2, 2, true>(pass, P, G, eos, eps, s, prepare);
      return cudaErrorNotSupported;
    }
    if (dim == 1) return launch_pass<2, 1, false>(pass, P, G, eos, eps, s, prepare);
    if (dim == 2) return launch_pass<2, 2, false>(pass, P, G, eos, eps, s, prepare);
    return launch_pass<2, 3, false>(pass, P, G, eos, eps, s, prepare);
  }
  if (np == 3 && !ptmu) {
    if (dim == 1) return launch_pass<3, 1, false>(pass, P, G, eos, eps, s, prepare);
    if (dim == 2) return launch_pass<3, 2, false>(pass, P, G, eos, eps, s, prepare);
    return launch_pass<3, 3, false>(pass, P, G, eos, eps, s, prepare);
  }
  return cudaErrorNotSupported;
}

size_t kapila_smem_bytes(int np, int dim, int pass) {
#define ECG_SM(NPV, DV)                                                         \
  if (np == NPV && dim == DV) {                                                 \
    if (pass == PASS_O1) return KapilaStep<NPV, DV, PASS_O1>::smem_bytes();     \
    if (pass == PASS_PRED) return KapilaStep<NPV, DV, PASS_PRED>::smem_bytes(); \
    return KapilaStep<NPV, DV, PASS_CORR>::smem_bytes();                        \
  }
  ECG_SM(2, 1) ECG_SM(2, 2) ECG_SM(2, 3) ECG_SM(3, 1) ECG_SM(3, 2) ECG_SM(3, 3)
#undef ECG_SM
  return 0;
}

}  // namespace ecg
