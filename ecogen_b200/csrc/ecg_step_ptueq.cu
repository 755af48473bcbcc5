// Temperature-pressure-velocity equilibrium model (ECOGEN's PTUEq, src/Models/PTUEq) step kernels:
// first-order step, MUSCL predictor and corrector, with the tile / per-axis halo staging of the
// other models (see ecg_step.cuh).
//
// The model carries two phases at one pressure, temperature and velocity.  Its conservative
// variables are the phase masses alpha_k rho_k, the momentum and the total energy; no volume-fraction
// equation, no non-conservative term, no relaxation.  State fields (stride = ncells):
//   alpha_0 0, alpha_1 1, p 2, T 3, u_d 4+d, E 4+DIM.
// Phase densities are rho_k = computeDensity(p, T) of each EOS (EosIG.cpp:85, EosSG.cpp:87): the
// reference stores exactly that after every FluxPTUEq::buildPrim, so the kernels recompute them.
// Every derived quantity (e_k, c_k, mixture rho, e and frozen sound speed) follows from the state as
// ModPTUEq::fulfillState (src/Models/PTUEq/ModPTUEq.cpp:99-108) and
// MixPTUEq::computeMixtureVariables (src/Models/PTUEq/MixPTUEq.cpp:293-313) compute them.
#include <cuda_runtime.h>

#include "ecg_step.cuh"

namespace ecg {

template <int DIM, int PASS>
struct PtStep {
  using TS = TileShape<DIM>;
  static constexpr int H = (PASS == PASS_O1) ? 1 : 2;
  static constexpr int NTH = TS::THREADS;
  static constexpr int NCELL = TS::X * TS::Y * TS::Z;
  static constexpr bool O2 = (PASS != PASS_O1);
  static_assert(NCELL <= NTH, "one thread per cell of the tile");
  static_assert(NTH % 32 == 0 && NTH <= 1024, "whole warps");
  static constexpr int NS = 5 + DIM;      // stored fields
  static constexpr int NQ = 4 + DIM;      // staged: alpha_0, alpha_1, p, T, u_d
  static constexpr int NSL = 4 + DIM;     // slopes of the same
  static constexpr int NFL = 3 + DIM;     // fluxes: mass_0, mass_1, mom_d, E
  static constexpr int NA0 = (PASS == PASS_CORR) ? 1 : 0;  // time-n alpha_0 plane of the corrector
  __host__ __device__ static constexpr int ext(int a) { return a == 0 ? TS::X : (a == 1 ? TS::Y : TS::Z); }
  __host__ __device__ static constexpr int lines(int a) { return NCELL / ext(a); }
  __host__ __device__ static constexpr int rlen(int a) { return ext(a) + 2 * H; }
  __host__ __device__ static constexpr int region(int a) { return rlen(a) * lines(a); }
  __host__ __device__ static constexpr int nslope(int a) { return O2 ? (ext(a) + 3) * lines(a) : 0; }
  __host__ __device__ static constexpr int nface(int a) { return (ext(a) + 1) * lines(a); }
  __host__ __device__ static constexpr int cmax(int a, int b) { return a > b ? a : b; }
  __host__ __device__ static constexpr int RMAX() { return cmax(region(0), cmax(DIM > 1 ? region(1) : 0, DIM > 2 ? region(2) : 0)); }
  __host__ __device__ static constexpr int SMAX() { return cmax(nslope(0), cmax(DIM > 1 ? nslope(1) : 0, DIM > 2 ? nslope(2) : 0)); }
  __host__ __device__ static constexpr int FMAX() { return cmax(nface(0), cmax(DIM > 1 ? nface(1) : 0, DIM > 2 ? nface(2) : 0)); }
  static constexpr size_t smem_bytes() {
    return sizeof(double) * ((size_t)RMAX() * (NQ + NA0) + (size_t)SMAX() * NSL + (size_t)FMAX() * NFL);
  }
};

struct PtEos {
  EosParams e[2];
};

// Eos::getPInf: the ideal gas has none (Errors::defaultDouble = 0).
__device__ __forceinline__ double pt_pinf(const EosParams& q) { return q.type == ECG_EOS_IG ? 0. : q.pinf; }

// computeDensity(p, T) of an IG or SG phase (EosIG.cpp:85, EosSG.cpp:87).
__device__ __forceinline__ double pt_rho(const EosParams& q, double p, double T) {
  const double den = dmax(((q.gamma - 1.) * q.cv * T), 0.);
  return q.type == ECG_EOS_IG ? ddiv(p, den) : ddiv(p + q.pinf, den);
}

// One side of a face (or a cell) with its derived quantities.
struct PtSide {
  double a[2], r[2];
  double p, T, rho, e, c;
  double u[3];
};

// ModPTUEq::fulfillState + MixPTUEq::computeMixtureVariables (mass fractions without a floor).
__device__ __forceinline__ void pt_complete(const PtEos& M, PtSide& s) {
  double ek[2], ck[2];
#pragma unroll
  for (int k = 0; k < 2; k++) {
    s.r[k] = pt_rho(M.e[k], s.p, s.T);
    ek[k] = eos_e(M.e[k], 0., s.r[k], s.p);
    ck[k] = eos_c(M.e[k], 0., s.r[k], s.p);
  }
  s.rho = 0.;
#pragma unroll
  for (int k = 0; k < 2; k++) s.rho += s.a[k] * s.r[k];
  double Y[2];
#pragma unroll
  for (int k = 0; k < 2; k++) Y[k] = ddiv(s.a[k] * s.r[k], s.rho);
  s.e = 0.;
  s.c = 0.;
#pragma unroll
  for (int k = 0; k < 2; k++) {
    s.e += Y[k] * ek[k];
    s.c += Y[k] * ck[k] * ck[k];
  }
  s.c = dsqrt(s.c);
}

// ModPTUEq::solveRiemannIntern src/Models/PTUEq/ModPTUEq.cpp:113-227 on face-frame velocities;
// the total energy uses the face-frame squared norm, as the reference's projected buffer cells do.
__device__ __forceinline__ void hllc_pt(const PtSide& L, const double ul[3], const PtSide& R, const double ur[3],
                                        double dxL, double dxR, double& dtmax, double Fm[2], double Fn[3],
                                        double& FE) {
  const double uL = ul[0], cL = L.c, pL = L.p, rhoL = L.rho;
  const double uR = ur[0], cR = R.c, pR = R.p, rhoR = R.rho;
  const double sL = dmin(uL - cL, uR - cR);
  const double sR = dmax(uR + cR, uL + cL);
  if (fabs(sL) > 1.e-3) dtmax = dmin(dtmax, ddiv(dxL, fabs(sL)));
  if (fabs(sR) > 1.e-3) dtmax = dmin(dtmax, ddiv(dxR, fabs(sR)));
  const double mL = rhoL * (sL - uL), mR = rhoR * (sR - uR);
  double sM = ddiv(pR - pL + mL * uL - mR * uR, mL - mR);
  if (fabs(sM) < 1.e-8) sM = 0.;
  if (sL >= 0.) {
#pragma unroll
    for (int k = 0; k < 2; k++) Fm[k] = L.a[k] * L.r[k] * uL;
    const double Et = L.e + 0.5 * (ul[0] * ul[0] + ul[1] * ul[1] + ul[2] * ul[2]);
    Fn[0] = rhoL * uL * uL + pL;
    Fn[1] = rhoL * ul[1] * uL;
    Fn[2] = rhoL * ul[2] * uL;
    FE = (rhoL * Et + pL) * uL;
  } else if (sR <= 0.) {
#pragma unroll
    for (int k = 0; k < 2; k++) Fm[k] = R.a[k] * R.r[k] * uR;
    const double Et = R.e + 0.5 * (ur[0] * ur[0] + ur[1] * ur[1] + ur[2] * ur[2]);
    Fn[0] = rhoR * uR * uR + pR;
    Fn[1] = rhoR * ur[1] * uR;
    Fn[2] = rhoR * ur[2] * uR;
    FE = (rhoR * Et + pR) * uR;
  } else if (sM >= 0.) {
    const double Et = L.e + 0.5 * (ul[0] * ul[0] + ul[1] * ul[1] + ul[2] * ul[2]);
    const double rhoStar = ddiv(mL, sL - sM);
    const double EStar = Et + (sM - uL) * (sM + ddiv(pL, mL));
    const double pStar = mL * (sM - uL) + pL;
#pragma unroll
    for (int k = 0; k < 2; k++) Fm[k] = ddiv(L.a[k] * L.r[k] * (sL - uL), sL - sM) * sM;
    Fn[0] = rhoStar * sM * sM + pStar;
    Fn[1] = rhoStar * ul[1] * sM;
    Fn[2] = rhoStar * ul[2] * sM;
    FE = (rhoStar * EStar + pStar) * sM;
  } else {
    const double Et = R.e + 0.5 * (ur[0] * ur[0] + ur[1] * ur[1] + ur[2] * ur[2]);
    const double rhoStar = ddiv(mR, sR - sM);
    const double EStar = Et + (sM - uR) * (sM + ddiv(pR, mR));
    const double pStar = mR * (sM - uR) + pR;
#pragma unroll
    for (int k = 0; k < 2; k++) Fm[k] = ddiv(R.a[k] * R.r[k] * (sR - uR), sR - sM) * sM;
    Fn[0] = rhoStar * sM * sM + pStar;
    Fn[1] = rhoStar * ur[1] * sM;
    Fn[2] = rhoStar * ur[2] * sM;
    FE = (rhoStar * EStar + pStar) * sM;
  }
}

// Register budget: the resident-block target of the tile shape (TileShape::MINB), as the Kapila
// kernels, with 8 blocks in 2D (ECG_PTUEQ_MINB2D); ECG_PTUEQ_NO_MINB leaves the register count to the
// compiler.  Measured on the 2D bubble at 2048^2 (MUSCL + van Leer, cell-updates/s): compiler's choice
// (94 registers, 20 warps per SM) 1170 M; blocks of 128 threads per SM: 5 1182 M, 6 1362 M,
// 7 (72 registers) 1540 M, 8 (64 registers, 32 warps) 1572 M, 9 1468 M, 10 1385 M.
#ifndef ECG_PTUEQ_MINB2D
#define ECG_PTUEQ_MINB2D 8
#endif
#ifndef ECG_PTUEQ_NO_MINB
#define ECG_PTUEQ_BOUNDS(DIM, PASS) \
  __launch_bounds__(PtStep<DIM, PASS>::NTH, DIM == 2 ? ECG_PTUEQ_MINB2D : TileShape<DIM>::MINB)
#else
#define ECG_PTUEQ_BOUNDS(DIM, PASS) __launch_bounds__(PtStep<DIM, PASS>::NTH)
#endif

template <int DIM, int PASS>
__global__ void ECG_PTUEQ_BOUNDS(DIM, PASS) k_ptueq_step(StepParams P, Geometry G, PtEos M) {
  using K = PtStep<DIM, PASS>;
  using TS = TileShape<DIM>;
  if (*P.done) return;
  extern __shared__ double smem[];
  constexpr int RS = K::RMAX();
  constexpr int SS = (K::SMAX() > 0) ? K::SMAX() : 1;
  constexpr int FS = K::FMAX();
  constexpr int NQ = K::NQ;
  constexpr int FA = 0, FP = 2, FT = 3, FU = 4;  // field indices of the state and of the staged planes
  double* sq = smem;                                      // [NQ][RS]
  double* sa0 = sq + (size_t)NQ * RS;                     // [NA0][RS]
  double* ssl = sa0 + (size_t)K::NA0 * RS;                // [NSL][SS]
  double* sfl = ssl + (K::O2 ? (size_t)K::NSL * SS : 0);  // [NFL][FS]
  const int tid = threadIdx.x;
  const int org[3] = {(int)blockIdx.x * TS::X, (int)blockIdx.y * TS::Y, (int)blockIdx.z * TS::Z};
  const int lc[3] = {tid % TS::X, (tid / TS::X) % TS::Y, tid / (TS::X * TS::Y)};
  const int gc[3] = {org[0] + lc[0], org[1] + lc[1], org[2] + lc[2]};
  const bool active = tid < K::NCELL && gc[0] < G.n[0] && gc[1] < G.n[1] && gc[2] < G.n[2];
  const int64_t nn = P.n;
  const int64_t cell = (int64_t)gc[0] + (int64_t)gc[1] * G.n[0] + (int64_t)gc[2] * G.n[0] * G.n[1];
  double am[2] = {0., 0.}, amom[DIM], aE = 0.;
#pragma unroll
  for (int d = 0; d < DIM; d++) amom[d] = 0.;
  double dtmax = 1.e10;

#pragma unroll
  for (int ax = 0; ax < DIM; ax++) {
    const int T = K::ext(ax), RL = K::rlen(ax);
    const int b1 = (ax == 0) ? 1 : 0, b2 = (ax == 2) ? 1 : 2;
    const int e1 = K::ext(b1);
    const int nax = G.n[ax];
    // ---- stage tile + halo along ax
    for (int e = tid; e < K::region(ax); e += K::NTH) {
      int la = e % RL - K::H, line = e / RL;
      int g[3];
      g[ax] = org[ax] + la;
      g[b1] = org[b1] + line % e1;
      g[b2] = org[b2] + line / e1;
      if (g[ax] >= 0 && g[ax] < nax && g[b1] < G.n[b1] && g[b2] < G.n[b2]) {
        int64_t c = (int64_t)g[0] + (int64_t)g[1] * G.n[0] + (int64_t)g[2] * G.n[0] * G.n[1];
#pragma unroll
        for (int f = 0; f < NQ; f++) sq[f * RS + e] = P.q[(int64_t)f * nn + c];
        if (K::NA0) sa0[e] = P.sn[c];
      }
    }
    __syncthreads();
    // ---- face slopes (PhasePTUEq::computeSlopesPhase :233, MixPTUEq::computeSlopesMixture :347);
    // a side of the domain has none (non-reflecting; MUSCL symmetry sides are refused)
    if (K::O2) {
      for (int e = tid; e < K::nslope(ax); e += K::NTH) {
        int j = e % (T + 3) - 1, line = e / (T + 3);
        int gl = org[ax] + j - 1;
        if (gl < 0 || gl + 1 >= nax) continue;
        int rl = line * RL + (j - 1 + K::H), rr = rl + 1;
        double d = G.dcc[ax][gl];
#pragma unroll
        for (int f = 0; f < K::NSL; f++) ssl[f * SS + e] = ddiv(sq[f * RS + rr] - sq[f * RS + rl], d);
      }
      __syncthreads();
    }
    // ---- face fluxes: face j between local cells j-1 and j, j in [0, T]
    for (int e = tid; e < K::nface(ax); e += K::NTH) {
      int j = e % (T + 1), line = e / (T + 1);
      int gl = org[ax] + j - 1;
      if (gl < 0 || gl + 1 >= nax || org[b1] + line % e1 >= G.n[b1] || org[b2] + line / e1 >= G.n[b2]) continue;
      int rl = line * RL + (j - 1 + K::H), rr = rl + 1;
      PtSide S[2];
#pragma unroll
      for (int side = 0; side < 2; side++) {
        const int rc = side ? rr : rl;
        PtSide& s = S[side];
        s.a[0] = sq[(FA + 0) * RS + rc];
        s.a[1] = sq[(FA + 1) * RS + rc];
        s.p = sq[FP * RS + rc];
        s.T = sq[FT * RS + rc];
        s.u[0] = s.u[1] = s.u[2] = 0.;
#pragma unroll
        for (int d = 0; d < DIM; d++) s.u[d] = sq[(FU + d) * RS + rc];
      }
      if (K::O2) {
        // CellInterfaceO2Cartesian::solveRiemann src/Order2/CellInterfaceO2Cartesian.cpp:101-226:
        // CellO2Cartesian::computeLocalSlopes limiters (interface detector on alpha_0; the opposite
        // face of a cell next to a side has no slope), extrapolation, PhasePTUEq::verifyAndCorrectPhase
        // (alpha in [1e-10, 1 - 1e-10]), optional THINC, then fulfillState
        const int fs = line * (T + 3), f1 = fs + j + 1;
        const bool hasL = (gl - 1 >= 0), hasR = (gl + 2 < nax);
        const double* a0 = K::NA0 ? sa0 : sq;
        const double aL = S[0].a[0], aR = S[1].a[0];
        const double aLL = hasL ? a0[rl - 1] : 0., aRR = hasR ? a0[rr + 1] : 0.;
#pragma unroll
        for (int side = 0; side < 2; side++) {
          PtSide& s = S[side];
          const int f2 = side ? (hasR ? fs + j + 2 : -1) : (hasL ? fs + j : -1);
          const double aCell = side ? aR : aL, aOther = side ? aL : aR, aAfter = side ? aRR : aLL;
          const bool iface = (aCell >= 1.e-4) && (aCell <= 1. - 1.e-4) && ((aOther - aCell) * (aCell - aAfter) >= 1.e-8);
          const int lg = iface ? P.lim[1] : P.lim[0];
          const int lv = iface ? P.lim[3] : P.lim[2];
          const double sign = side ? -1. : 1.;
          const double dist = side ? G.dfr[ax][gl] : G.dfl[ax][gl];
#pragma unroll
          for (int k = 0; k < 2; k++) {
            const double l = limiter(lv, ssl[(FA + k) * SS + f1], f2 >= 0 ? ssl[(FA + k) * SS + f2] : 0.);
            double a = s.a[k] + (sign * l) * dist;
            if (a < 1e-10) a = 1e-10;
            if (a > 1. - 1e-10) a = 1. - 1e-10;
            s.a[k] = a;
          }
          s.p += (sign * limiter(lg, ssl[FP * SS + f1], f2 >= 0 ? ssl[FP * SS + f2] : 0.)) * dist;
          s.T += (sign * limiter(lg, ssl[FT * SS + f1], f2 >= 0 ? ssl[FT * SS + f2] : 0.)) * dist;
#pragma unroll
          for (int d = 0; d < DIM; d++)
            s.u[d] = s.u[d] + (sign * limiter(lg, ssl[(FU + d) * SS + f1], f2 >= 0 ? ssl[(FU + d) * SS + f2] : 0.)) * dist;
          if (P.thinc && iface) {  // THINC alpha_0 (left: :132-150, right: :164-181; different final expressions)
            const double beta = 1.6, eps = 1.e-4;
            const bool right = side == 1;
            const double hi = right ? aAfter : aOther, lo = right ? aOther : aAfter;
            const double sg = (hi - lo > 0.) ? 1. : -1.;
            const double qmin = dmin(hi, lo);
            const double qmax = dmax(hi, lo) - qmin;
            const double C = ddiv(aCell - qmin + 1.e-20, qmax + 1.e-20);
            const double B = exp(sg * beta * (2. * C - 1.));
            const double A = ddiv(ddiv(B, P.thinc_cosh) - 1., P.thinc_tanh);
            double na = right ? qmin + 0.5 * qmax * (1. + sg * A)
                              : qmin + 0.5 * qmax * (1. + ddiv(sg * (P.thinc_tanh + A), 1. + A * P.thinc_tanh));
            if (na < eps) na = eps;
            if (na > 1. - eps) na = 1. - eps;
            s.a[0] = na;
            s.a[1] = 1. - na;
          }
        }
      }
      pt_complete(M, S[0]);
      pt_complete(M, S[1]);
      double ul[3], ur[3], Fn[3], Fg[3], Fm[2], FE;
      to_local(ax, false, S[0].u, ul);
      to_local(ax, false, S[1].u, ur);
      int gf[3];  // the face's left cell, then its right cell: their CFL lengths
      gf[ax] = gl;
      gf[b1] = org[b1] + line % e1;
      gf[b2] = org[b2] + line / e1;
      const double lL = cell_lcfl(G, gf[0], gf[1], gf[2]);
      gf[ax] = gl + 1;
      const double lR = cell_lcfl(G, gf[0], gf[1], gf[2]);
      hllc_pt(S[0], ul, S[1], ur, lL, lR, dtmax, Fm, Fn, FE);
      to_global(ax, false, Fn, Fg);
      sfl[0 * FS + e] = Fm[0];
      sfl[1 * FS + e] = Fm[1];
#pragma unroll
      for (int d = 0; d < DIM; d++) sfl[(2 + d) * FS + e] = Fg[d];
      sfl[(2 + DIM) * FS + e] = FE;
    }
    __syncthreads();
    // ---- accumulate the two faces of this axis into the own cell (FluxPTUEq::addFlux / subtractFlux)
    if (active) {
      const int la = lc[ax];
      const int line = lc[b1] + lc[b2] * e1;
      const double cA = cell_coefA(G, ax, gc[0], gc[1], gc[2]);
#pragma unroll
      for (int side = 0; side < 2; side++) {
        const int j = la + side;
        const int gl = org[ax] + j - 1;
        if (gl < 0 || gl + 1 >= nax) continue;
        const int e = line * (T + 1) + j;
        const double sg = side ? -1. : 1.;
        if (side == 0) {
          am[0] += cA * sfl[0 * FS + e];
          am[1] += cA * sfl[1 * FS + e];
#pragma unroll
          for (int d = 0; d < DIM; d++) amom[d] += cA * sfl[(2 + d) * FS + e];
          aE += cA * sfl[(2 + DIM) * FS + e];
        } else {
          am[0] -= cA * sfl[0 * FS + e];
          am[1] -= cA * sfl[1 * FS + e];
#pragma unroll
          for (int d = 0; d < DIM; d++) amom[d] -= cA * sfl[(2 + d) * FS + e];
          aE -= cA * sfl[(2 + DIM) * FS + e];
        }
        (void)sg;
      }
    }
    __syncthreads();
  }

  if (active) {
    // ---- sides of the domain, in face order Xm, Xp, Ym, Yp, Zm, Zp (BoundCond::computeFlux)
#pragma unroll
    for (int bf = 0; bf < 2 * DIM; bf++) {
      const int ax = bf >> 1;
      const bool neg = (bf & 1) == 0;
      if (neg ? (gc[ax] != 0) : (gc[ax] != G.n[ax] - 1)) continue;
      PtSide s;
      s.a[0] = P.q[cell];
      s.a[1] = P.q[nn + cell];
      s.p = P.q[(int64_t)FP * nn + cell];
      s.T = P.q[(int64_t)FT * nn + cell];
      s.u[0] = s.u[1] = s.u[2] = 0.;
#pragma unroll
      for (int d = 0; d < DIM; d++) s.u[d] = P.q[(int64_t)(FU + d) * nn + cell];
      pt_complete(M, s);  // BoundCond::solveRiemann calls fulfillState on its buffer
      double ul[3], Fn[3], Fg[3];
      to_local(ax, neg, s.u, ul);
      const double cA = cell_coefA(G, ax, gc[0], gc[1], gc[2]);
      const double lc = cell_lcfl(G, gc[0], gc[1], gc[2]);
      if (G.bc[bf] == ECG_BC_SYMMETRY) {
        // ModPTUEq::solveRiemannWall src/Models/PTUEq/ModPTUEq.cpp:233-265 (first order only)
        const double uL = ul[0];
        const double sL = dmin(uL - s.c, -uL - s.c);
        if (fabs(sL) > 1.e-3) dtmax = dmin(dtmax, ddiv(lc, fabs(sL)));
        Fn[0] = s.rho * (uL - sL) * uL + s.p;
        Fn[1] = Fn[2] = 0.;
        to_global(ax, neg, Fn, Fg);
#pragma unroll
        for (int d = 0; d < DIM; d++) amom[d] -= cA * Fg[d];
        continue;
      }
      double Fm[2], FE;
      hllc_pt(s, ul, s, ul, lc, lc, dtmax, Fm, Fn, FE);
      to_global(ax, neg, Fn, Fg);
      am[0] -= cA * Fm[0];
      am[1] -= cA * Fm[1];
#pragma unroll
      for (int d = 0; d < DIM; d++) amom[d] -= cA * Fg[d];
      aE -= cA * FE;
    }
    // ---- FluxPTUEq::buildCons (time-n state), Cell::timeEvolution, FluxPTUEq::buildPrim (:125-160) with
    // MixPTUEq::computePressure (:93-122, Le Martelot's analytic p of two IG/SG phases) and
    // computeTemperature (:126-145)
    const double dt = *P.dt;
    const double scale = (PASS == PASS_PRED) ? 0.5 * dt : dt;
    PtSide n0;
    n0.a[0] = P.sn[cell];
    n0.a[1] = P.sn[nn + cell];
    n0.p = P.sn[(int64_t)FP * nn + cell];
    n0.T = P.sn[(int64_t)FT * nn + cell];
    const double En = P.sn[(int64_t)(FU + DIM) * nn + cell];
    double rhon = 0.;
#pragma unroll
    for (int k = 0; k < 2; k++) {
      n0.r[k] = pt_rho(M.e[k], n0.p, n0.T);
      rhon += n0.a[k] * n0.r[k];
    }
    double m[2];
#pragma unroll
    for (int k = 0; k < 2; k++) m[k] = am[k] * scale + 1. * (n0.a[k] * n0.r[k]);
    double mom[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) mom[d] = amom[d] * scale + 1. * (rhon * P.sn[(int64_t)(FU + d) * nn + cell]);
    const double rE = aE * scale + 1. * (rhon * En);
    const double rhoMel = 0. + m[0] + m[1];
    double u[3] = {0., 0., 0.};
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      u[d] = ddiv(mom[d], rhoMel);
      if (fabs(u[d]) < 1.e-8) u[d] = 0.;
    }
    const double ie = ddiv(rE, rhoMel) - 0.5 * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    const EosParams& E1 = M.e[0];
    const EosParams& E2 = M.e[1];
    const double pInf1 = pt_pinf(E1), pInf2 = pt_pinf(E2);
    const double Y1 = ddiv(m[0], rhoMel), Y2 = ddiv(m[1], rhoMel);
    const double q = Y1 * E1.eref + Y2 * E2.eref;
    const double cvMel = Y1 * E1.cv + Y2 * E2.cv;
    const double A1 = ddiv(Y1 * (E1.gamma - 1.) * E1.cv, cvMel) * (rhoMel * (ie - q) - pInf1);
    const double A2 = ddiv(Y2 * (E2.gamma - 1.) * E2.cv, cvMel) * (rhoMel * (ie - q) - pInf2);
    const double p = 0.5 * (A1 + A2 - (pInf1 + pInf2)) +
                     dsqrt(0.25 * (A2 - A1 - (pInf2 - pInf1)) * (A2 - A1 - (pInf2 - pInf1)) + A1 * A2);
    double Tm = 0.;
    Tm += ddiv(ddiv(m[0], rhoMel) * (E1.gamma - 1.) * E1.cv, p + pInf1);
    Tm += ddiv(ddiv(m[1], rhoMel) * (E2.gamma - 1.) * E2.cv, p + pInf2);
    Tm = ddiv(1., Tm * rhoMel);
    P.out[cell] = ddiv(m[0], pt_rho(E1, p, Tm));
    P.out[nn + cell] = ddiv(m[1], pt_rho(E2, p, Tm));
    P.out[(int64_t)FP * nn + cell] = p;
    P.out[(int64_t)FT * nn + cell] = Tm;
#pragma unroll
    for (int d = 0; d < DIM; d++) P.out[(int64_t)(FU + d) * nn + cell] = u[d];
    if (PASS != PASS_PRED) P.out[(int64_t)(FU + DIM) * nn + cell] = ddiv(rE, rhoMel);
  }
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

template <int DIM, int PASS>
static cudaError_t ptueq_one(const StepParams& P, const Geometry& G, const ecg_eos* eos, cudaStream_t s,
                             bool prepare) {
  using K = PtStep<DIM, PASS>;
  using TS = TileShape<DIM>;
  auto kern = k_ptueq_step<DIM, PASS>;
  const size_t sm = K::smem_bytes();
  if (prepare) return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  PtEos M;
  for (int k = 0; k < 2; k++)
    M.e[k] = EosParams{eos[k].type, eos[k].gamma, eos[k].pinf, eos[k].b, eos[k].cv, eos[k].eref, eos[k].sref};
  dim3 grid((G.n[0] + TS::X - 1) / TS::X, (G.n[1] + TS::Y - 1) / TS::Y, (G.n[2] + TS::Z - 1) / TS::Z);
  kern<<<grid, K::NTH, sm, s>>>(P, G, M);
  return cudaGetLastError();
}

template <int DIM>
static cudaError_t ptueq_dim(int pass, const StepParams& P, const Geometry& G, const ecg_eos* eos, cudaStream_t s,
                             bool prepare) {
  if (pass == PASS_O1) return ptueq_one<DIM, PASS_O1>(P, G, eos, s, prepare);
  if (pass == PASS_PRED) return ptueq_one<DIM, PASS_PRED>(P, G, eos, s, prepare);
  return ptueq_one<DIM, PASS_CORR>(P, G, eos, s, prepare);
}

cudaError_t ptueq_launch(int dim, int pass, const StepParams& P, const Geometry& G, const ecg_eos* eos, cudaStream_t s,
                         bool prepare) {
  if (P.ntr != 0) return cudaErrorNotSupported;  // the model has no transport Riemann solver
  if (dim == 1) return ptueq_dim<1>(pass, P, G, eos, s, prepare);
  if (dim == 2) return ptueq_dim<2>(pass, P, G, eos, s, prepare);
  return ptueq_dim<3>(pass, P, G, eos, s, prepare);
}

}  // namespace ecg
