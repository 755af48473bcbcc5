// Euler (single-phase) step kernels: first-order step, MUSCL predictor and corrector, with the
// same tile / per-axis halo staging as the Kapila kernels (see ecg_step.cuh).
//
// State fields (stride = ncells): rho 0, p 1, u_d 2+d, E 2+DIM.  The stored E is the specific total
// energy rebuilt by FluxEuler::buildPrim (src/Models/Euler/FluxEuler.cpp:124, E = (rho E)/rho);
// wherever the reference calls fulfillState (boundary faces, reconstructed face states, the MUSCL
// half step) E is recomputed from (rho, p, u) by PhaseEuler::extendedCalculusPhase
// (src/Models/Euler/PhaseEuler.cpp:105), and so it is here.
#include <cuda_runtime.h>

#include "ecg_step.cuh"

namespace ecg {

template <int DIM, int PASS, int NTM = 0>
struct EulerStep {
  using TS = TileShape<DIM>;
  static constexpr int H = (PASS == PASS_O1) ? 1 : 2;
  static constexpr int NTH = TS::THREADS;
  static constexpr int NCELL = TS::X * TS::Y * TS::Z;
  static constexpr bool O2 = (PASS != PASS_O1);
  static_assert(NCELL <= NTH, "one thread per cell of the tile");
  static_assert(NTH % 32 == 0 && NTH <= 1024, "whole warps");
  static constexpr int NQ = 3 + DIM;      // rho, p, u_d, E
  static constexpr int NSL = 2 + DIM;     // rho, p, u_d
  static constexpr int NFL = 2 + DIM;     // mass, mom_d, E
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
  // passive transports (up to NTM): staged planes, slopes, and per face sM plus the transport fluxes
  static constexpr int NFT = NTM > 0 ? NTM + 1 : 0;
  static constexpr size_t smem_bytes() {
    return sizeof(double) * ((size_t)RMAX() * (NQ + NTM) + (size_t)SMAX() * (NSL + NTM) + (size_t)FMAX() * (NFL + NFT));
  }
};

struct EulerSide {
  double rho, p, c, E;
  double u[3];  // absolute frame
};

__device__ __forceinline__ void euler_complete(const EosParams& q, double eps, EulerSide& s) {
  // PhaseEuler::extendedCalculusPhase: e, c, E = e + |u|^2 / 2 (absolute frame)
  double e = eos_e(q, eps, s.rho, s.p);
  s.c = eos_c(q, eps, s.rho, s.p);
  s.E = e + 0.5 * (s.u[0] * s.u[0] + s.u[1] * s.u[1] + s.u[2] * s.u[2]);
}

// ModEuler::solveRiemannIntern src/Models/Euler/ModEuler.cpp:105-225 (strict sL > 0 / sR < 0).
__device__ __forceinline__ void hllc_euler(const EulerSide& L, const double ul[3], const EulerSide& R,
                                           const double ur[3], double dxL, double dxR, double& dtmax, double& Fm,
                                           double Fn[3], double& FE, double* sM_out = nullptr) {
  double uL = ul[0], vL = ul[1], wL = ul[2], pL = L.p, rhoL = L.rho, cL = L.c, EL = L.E;
  double uR = ur[0], vR = ur[1], wR = ur[2], pR = R.p, rhoR = R.rho, cR = R.c, ER = R.E;
  double sL = dmin(uL - cL, uR - cR);
  double sR = dmax(uR + cR, uL + cL);
  if (fabs(sL) > 1.e-3) dtmax = dmin(dtmax, ddiv(1. * dxL, fabs(sL)));
  if (fabs(sR) > 1.e-3) dtmax = dmin(dtmax, ddiv(1. * dxR, fabs(sR)));
  double mL = rhoL * (sL - uL), mR = rhoR * (sR - uR);
  double sM = ddiv(pR - pL + mL * uL - mR * uR, mL - mR);
  if (fabs(sM) < 1.e-8) sM = 0.;
  if (sM_out) *sM_out = sM;
  if (sL > 0.) {
    Fm = rhoL * uL;
    Fn[0] = rhoL * uL * uL + pL;
    Fn[1] = rhoL * vL * uL;
    Fn[2] = rhoL * wL * uL;
    FE = (rhoL * EL + pL) * uL;
  } else if (sR < 0.) {
    Fm = rhoR * uR;
    Fn[0] = rhoR * uR * uR + pR;
    Fn[1] = rhoR * vR * uR;
    Fn[2] = rhoR * wR * uR;
    FE = (rhoR * ER + pR) * uR;
  } else if (sM >= 0.) {
    double pStar = mL * (sM - uL) + pL;
    double rhoStar = ddiv(mL, sL - sM);
    double Estar = EL + (sM - uL) * (sM + ddiv(pL, mL));
    Fm = rhoStar * sM;
    Fn[0] = rhoStar * sM * sM + pStar;
    Fn[1] = rhoStar * sM * vL;
    Fn[2] = rhoStar * sM * wL;
    FE = (rhoStar * Estar + pStar) * sM;
  } else {
    double pStar = mR * (sM - uR) + pR;
    double rhoStar = ddiv(mR, sR - sM);
    double Estar = ER + (sM - uR) * (sM + ddiv(pR, mR));
    Fm = rhoStar * sM;
    Fn[0] = rhoStar * sM * sM + pStar;
    Fn[1] = rhoStar * sM * vR;
    Fn[2] = rhoStar * sM * wR;
    FE = (rhoStar * Estar + pStar) * sM;
  }
}

// Register budget: ECG_EULER_MINB2D > 0 asks the compiler for that many resident blocks per SM in 2D;
// 0 leaves the register count to the compiler.  Measured on a 2048^2 blast (MUSCL + van Leer,
// cell-updates/s): compiler's choice (80 registers, 6 blocks of 128 threads) 2449 M; 6 blocks 2721 M;
// 7 (72 registers) 2909 M; 8 (64 registers) 2754 M.
#ifndef ECG_EULER_MINB2D
#define ECG_EULER_MINB2D 7
#endif

template <int DIM, int PASS, int NTM = 0>
__global__ void __launch_bounds__(EulerStep<DIM, PASS, NTM>::NTH,
                                  (DIM == 2 && ECG_EULER_MINB2D > 0) ? ECG_EULER_MINB2D : 1)
    k_euler_step(StepParams P, Geometry G, EosParams q, double eps) {
  using K = EulerStep<DIM, PASS, NTM>;
  using TS = TileShape<DIM>;
  if (*P.done) return;
  extern __shared__ double smem[];
  constexpr int RS = K::RMAX();
  constexpr int SS = (K::SMAX() > 0) ? K::SMAX() : 1;
  constexpr int FS = K::FMAX();
  constexpr int NQ = K::NQ;
  double* sq = smem;
  double* str = sq + (size_t)NQ * RS;                           // [NTM][RS] transports
  double* ssl = str + (size_t)NTM * RS;                         // [NSL + NTM][SS]
  double* sfl = ssl + (K::O2 ? (size_t)(K::NSL + NTM) * SS : 0);  // [NFL + NFT][FS]
  constexpr int NTA = NTM > 0 ? NTM : 1;
  constexpr int NS = 3 + DIM;  // fields of the Euler state; transports at NS + j
  const int tid = threadIdx.x;
  const int org[3] = {(int)blockIdx.x * TS::X, (int)blockIdx.y * TS::Y, (int)blockIdx.z * TS::Z};
  const int lc[3] = {tid % TS::X, (tid / TS::X) % TS::Y, tid / (TS::X * TS::Y)};
  const int gc[3] = {org[0] + lc[0], org[1] + lc[1], org[2] + lc[2]};
  const bool active = tid < K::NCELL && gc[0] < G.n[0] && gc[1] < G.n[1] && gc[2] < G.n[2];
  const int64_t nn = P.n;
  const int64_t cell = (int64_t)gc[0] + (int64_t)gc[1] * G.n[0] + (int64_t)gc[2] * G.n[0] * G.n[1];
  double am = 0., amom[DIM], aE = 0.;
#pragma unroll
  for (int d = 0; d < DIM; d++) amom[d] = 0.;
  double tn[NTA], at[NTA];  // transports: time-n values, accumulated fluxes
#pragma unroll
  for (int t = 0; t < NTA; t++) tn[t] = at[t] = 0.;
  if (NTM > 0 && active) {
#pragma unroll
    for (int t = 0; t < NTM; t++)
      if (t < P.ntr) tn[t] = P.sn[(int64_t)(NS + t) * nn + cell];
  }
  double dtmax = 1.e10;
  double wallp[DIM];  // normal momentum flux of the cell's symmetry sides, per axis
#pragma unroll
  for (int d = 0; d < DIM; d++) wallp[d] = 0.;

#pragma unroll
  for (int ax = 0; ax < DIM; ax++) {
    const int T = K::ext(ax), RL = K::rlen(ax);
    const int b1 = (ax == 0) ? 1 : 0, b2 = (ax == 2) ? 1 : 2;
    const int e1 = K::ext(b1);
    const int nax = G.n[ax];
    for (int e = tid; e < K::region(ax); e += K::NTH) {
      int la = e % RL - K::H, line = e / RL;
      int g[3];
      g[ax] = org[ax] + la;
      g[b1] = org[b1] + line % e1;
      g[b2] = org[b2] + line / e1;
      if (g[ax] >= 0 && g[ax] < nax && g[b1] < G.n[b1] && g[b2] < G.n[b2]) {
        int64_t c = (int64_t)g[0] + (int64_t)g[1] * G.n[0] + (int64_t)g[2] * G.n[0] * G.n[1];
#pragma unroll
        for (int f = 0; f < NQ; f++) sq[f * RS + e] = (f < NQ - 1 || !K::O2) ? P.q[(int64_t)f * nn + c] : 0.;
#pragma unroll
        for (int t = 0; t < NTM; t++)
          if (t < P.ntr) str[t * RS + e] = P.q[(int64_t)(NS + t) * nn + c];
      }
    }
    __syncthreads();
    if (K::O2) {
      for (int e = tid; e < K::nslope(ax); e += K::NTH) {
        int j = e % (T + 3) - 1, line = e / (T + 3);
        int gl = org[ax] + j - 1;
        int rl = line * RL + (j - 1 + K::H), rr = rl + 1;
        if (gl < 0 || gl + 1 >= nax) {
          // symmetry side: velocity slope along the axis (BoundCondWallO2Cartesian::computeSlopes :84-108,
          // PhaseEuler::setU)
          const int sd = (gl == -1) ? 0 : ((gl == nax - 1) ? 1 : -1);
          if (sd < 0 || G.bc[2 * ax + sd] != ECG_BC_SYMMETRY) continue;
          if (org[b1] + line % e1 >= G.n[b1] || org[b2] + line / e1 >= G.n[b2]) continue;
#pragma unroll
          for (int f = 0; f < K::NSL + NTM; f++) ssl[f * SS + e] = 0.;
          const double wd = G.wslope[2 * ax + sd];
          if (fabs(wd) > 1.e-8) ssl[(2 + ax) * SS + e] = ddiv(sq[(2 + ax) * RS + (sd ? rl : rr)], wd);
          continue;
        }
        double d = G.dcc[ax][gl];
#pragma unroll
        for (int f = 0; f < K::NSL; f++) ssl[f * SS + e] = ddiv(sq[f * RS + rr] - sq[f * RS + rl], d);
#pragma unroll
        for (int t = 0; t < NTM; t++)  // Transport::computeSlopeTransport
          if (t < P.ntr) ssl[(K::NSL + t) * SS + e] = ddiv(str[t * RS + rr] - str[t * RS + rl], d);
      }
      __syncthreads();
    }
    for (int e = tid; e < K::nface(ax); e += K::NTH) {
      int j = e % (T + 1), line = e / (T + 1);
      int l1 = line % e1, l2 = line / e1;
      int gl = org[ax] + j - 1;
      if (gl < 0 || gl + 1 >= nax || org[b1] + l1 >= G.n[b1] || org[b2] + l2 >= G.n[b2]) continue;
      int rl = line * RL + (j - 1 + K::H), rr = rl + 1;
      EulerSide L, R;
      double xs[2][NTA];  // transports of the two sides
#pragma unroll
      for (int side = 0; side < 2; side++) {
        EulerSide& S = side ? R : L;
        int rc = side ? rr : rl;
#pragma unroll
        for (int t = 0; t < NTM; t++) xs[side][t] = str[t * RS + rc];
        S.rho = sq[0 * RS + rc];
        S.p = sq[1 * RS + rc];
        S.u[0] = S.u[1] = S.u[2] = 0.;
#pragma unroll
        for (int d = 0; d < DIM; d++) S.u[d] = sq[(2 + d) * RS + rc];
        if (!K::O2) {
          S.c = eos_c(q, eps, S.rho, S.p);
          S.E = sq[(2 + DIM) * RS + rc];  // stored total energy (no fulfillState on interior first-order faces)
        } else {
          const int fs = line * (T + 3), f1 = fs + j + 1;
          const bool has = side ? (gl + 2 < nax) : (gl - 1 >= 0);
          const bool wall = !has && G.bc[2 * ax + side] == ECG_BC_SYMMETRY;  // opposite slope of a symmetry side
          const int f2 = (has || wall) ? (side ? fs + j + 2 : fs + j) : -1;
          const double sign = side ? -1. : 1.;
          const double dist = side ? G.dfr[ax][gl] : G.dfl[ax][gl];
          // PhaseEuler::limitSlopes (global limiter: the interface detector never fires for Euler),
          // extrapolate, verifyAndCorrectPhase, verifyAndCorrectDensityMax, then fulfillState
          double lr = limiter(P.lim[0], ssl[0 * SS + f1], f2 >= 0 ? ssl[0 * SS + f2] : 0.);
          double lp = limiter(P.lim[0], ssl[1 * SS + f1], f2 >= 0 ? ssl[1 * SS + f2] : 0.);
          S.rho += (sign * lr) * dist;
          S.p += (sign * lp) * dist;
#pragma unroll
          for (int t = 0; t < NTM; t++) {  // global volume-fraction limiter (no interface detection for Euler)
            double lt = limiter(P.lim[2], ssl[(K::NSL + t) * SS + f1], f2 >= 0 ? ssl[(K::NSL + t) * SS + f2] : 0.);
            xs[side][t] += (sign * lt) * dist;
          }
#pragma unroll
          for (int d = 0; d < DIM; d++) {
            double l = limiter(P.lim[0], ssl[(2 + d) * SS + f1], f2 >= 0 ? ssl[(2 + d) * SS + f2] : 0.);
            S.u[d] = S.u[d] + (sign * l) * dist;
          }
          if (S.rho < 1.e-10) S.rho = 1.e-10;
          S.p = eos_fix_p(q, S.p);
          eos_rho_max(q, S.rho);
          euler_complete(q, eps, S);
        }
      }
      double ul[3], ur[3], Fn[3], Fm, FE, Fg[3];
      to_local(ax, false, L.u, ul);
      to_local(ax, false, R.u, ur);
      double sM = 0.;
      int gf[3];  // the face's left cell, then its right cell: their CFL lengths
      gf[ax] = gl;
      gf[b1] = org[b1] + l1;
      gf[b2] = org[b2] + l2;
      const double lL = cell_lcfl(G, gf[0], gf[1], gf[2]);
      gf[ax] = gl + 1;
      const double lR = cell_lcfl(G, gf[0], gf[1], gf[2]);
      hllc_euler(L, ul, R, ur, lL, lR, dtmax, Fm, Fn, FE, &sM);
      to_global(ax, false, Fn, Fg);
      sfl[0 * FS + e] = Fm;
#pragma unroll
      for (int d = 0; d < DIM; d++) sfl[(1 + d) * FS + e] = Fg[d];
      sfl[(1 + DIM) * FS + e] = FE;
      if (NTM > 0) {
        sfl[K::NFL * FS + e] = sM;
#pragma unroll
        for (int t = 0; t < NTM; t++)  // Transport::solveRiemann: upwind by sM
          sfl[(K::NFL + 1 + t) * FS + e] = (sM > 0.) ? xs[0][t] * sM : xs[1][t] * sM;
      }
    }
    __syncthreads();
    if (active) {
      int la = lc[ax];
      int line = lc[b1] + lc[b2] * e1;
      const double cA = cell_coefA(G, ax, gc[0], gc[1], gc[2]);
#pragma unroll
      for (int side = 0; side < 2; side++) {
        int j = la + side;
        int gl = org[ax] + j - 1;
        if (gl < 0 || gl + 1 >= nax) continue;
        int e = line * (T + 1) + j;
        double Fm = sfl[0 * FS + e], FE = sfl[(1 + DIM) * FS + e];
        if (side == 0) {
          am += cA * Fm;
#pragma unroll
          for (int d = 0; d < DIM; d++) amom[d] += cA * sfl[(1 + d) * FS + e];
          aE += cA * FE;
        } else {
          am -= cA * Fm;
#pragma unroll
          for (int d = 0; d < DIM; d++) amom[d] -= cA * sfl[(1 + d) * FS + e];
          aE -= cA * FE;
        }
        if (NTM > 0) {  // Transport::addFlux / addNonCons (time-n value), or subtract
          const double sM = sfl[K::NFL * FS + e];
#pragma unroll
          for (int t = 0; t < NTM; t++) {
            if (t >= P.ntr) continue;
            const double ft = sfl[(K::NFL + 1 + t) * FS + e];
            if (side == 0) {
              at[t] += cA * ft;
              at[t] += -cA * tn[t] * sM;
            } else {
              at[t] -= cA * ft;
              at[t] -= -cA * tn[t] * sM;
            }
          }
        }
      }
      // symmetry side along ax: flux now (slopes of this axis staged), subtracted below in face order
      const int sd = (gc[ax] == 0) ? 0 : ((gc[ax] == nax - 1) ? 1 : -1);
      if (sd >= 0 && G.bc[2 * ax + sd] == ECG_BC_SYMMETRY) {
        const int rc = line * RL + la + K::H;
        EulerSide S;
        S.rho = sq[0 * RS + rc];
        S.p = sq[1 * RS + rc];
        S.u[0] = S.u[1] = S.u[2] = 0.;
#pragma unroll
        for (int d = 0; d < DIM; d++) S.u[d] = sq[(2 + d) * RS + rc];
        if (K::O2) {
          // BoundCondWallO2Cartesian::solveRiemann :111-141: limited slopes (global limiter), extrapolation
          // by the signed distance without clamps
          const int fs = line * (T + 3), fw = fs + la + 1 + sd, fo = fs + la + 2 - sd;
          const double dist = G.wdist[2 * ax + sd];
          S.rho = S.rho + limiter(P.lim[0], ssl[0 * SS + fw], ssl[0 * SS + fo]) * dist;
          S.p = S.p + limiter(P.lim[0], ssl[1 * SS + fw], ssl[1 * SS + fo]) * dist;
#pragma unroll
          for (int d = 0; d < DIM; d++)
            S.u[d] = S.u[d] + limiter(P.lim[0], ssl[(2 + d) * SS + fw], ssl[(2 + d) * SS + fo]) * dist;
        }
        euler_complete(q, eps, S);
        double ul[3];
        to_local(ax, sd == 0, S.u, ul);
        // ModEuler::solveRiemannWall src/Models/Euler/ModEuler.cpp:368-409
        const double uL = ul[0], cL = S.c, pL = S.p, rhoL = S.rho;
        const double sL = dmin(uL - cL, -uL - cL);
        if (fabs(sL) > 1.e-3) dtmax = dmin(dtmax, ddiv(1. * cell_lcfl(G, gc[0], gc[1], gc[2]), fabs(sL)));
        wallp[ax] = rhoL * uL * (uL - sL) + pL;
      }
    }
    __syncthreads();
  }

  if (active) {
#pragma unroll
    for (int bf = 0; bf < 2 * DIM; bf++) {
      int ax = bf >> 1;
      bool neg = (bf & 1) == 0;
      if (neg ? (gc[ax] != 0) : (gc[ax] != G.n[ax] - 1)) continue;
      if (G.bc[bf] == ECG_BC_SYMMETRY) {
        const double Fn[3] = {wallp[ax], 0., 0.};
        double Fg[3];
        to_global(ax, neg, Fn, Fg);
        const double cA = cell_coefA(G, ax, gc[0], gc[1], gc[2]);
        am -= cA * 0.;
#pragma unroll
        for (int d = 0; d < DIM; d++) amom[d] -= cA * Fg[d];
        aE -= cA * 0.;
#pragma unroll
        for (int t = 0; t < NTM; t++) {  // no transport flux through a symmetry side, sM = 0
          if (t >= P.ntr) continue;
          at[t] -= cA * 0.;
          at[t] -= -cA * tn[t] * 0.;
        }
        continue;
      }
      EulerSide S;
      S.rho = P.q[cell];
      S.p = P.q[nn + cell];
      S.u[0] = S.u[1] = S.u[2] = 0.;
#pragma unroll
      for (int d = 0; d < DIM; d++) S.u[d] = P.q[(int64_t)(2 + d) * nn + cell];
      euler_complete(q, eps, S);  // BoundCond::solveRiemann calls fulfillState on its buffer
      double ul[3], Fn[3], Fm, FE, Fg[3];
      to_local(ax, neg, S.u, ul);
      double sMb = 0.;
      const double lc = cell_lcfl(G, gc[0], gc[1], gc[2]);
      hllc_euler(S, ul, S, ul, lc, lc, dtmax, Fm, Fn, FE, &sMb);
      to_global(ax, neg, Fn, Fg);
      const double cA = cell_coefA(G, ax, gc[0], gc[1], gc[2]);
      am -= cA * Fm;
#pragma unroll
      for (int d = 0; d < DIM; d++) amom[d] -= cA * Fg[d];
      aE -= cA * FE;
#pragma unroll
      for (int t = 0; t < NTM; t++) {  // non-reflecting side: T sM of the cell
        if (t >= P.ntr) continue;
        const double ft = P.q[(int64_t)(NS + t) * nn + cell] * sMb;
        at[t] -= cA * ft;
        at[t] -= -cA * tn[t] * sMb;
      }
    }
    // FluxEuler::buildCons, Cell::timeEvolution, FluxEuler::buildPrim
    const double dt = *P.dt;
    const double scale = (PASS == PASS_PRED) ? 0.5 * dt : dt;
    double rn = P.sn[cell];
    double En = P.sn[(int64_t)(2 + DIM) * nn + cell];
    am = am * scale + 1. * rn;
    double u[DIM], usq = 0.;
#pragma unroll
    for (int d = 0; d < DIM; d++) amom[d] = amom[d] * scale + 1. * (rn * P.sn[(int64_t)(2 + d) * nn + cell]);
    aE = aE * scale + 1. * (rn * En);
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      u[d] = ddiv(amom[d], am);
      if (fabs(u[d]) < 1.e-8) u[d] = 0.;
      usq += u[d] * u[d];
    }
    double E = ddiv(aE, am);
    double e = E - 0.5 * usq;
    double p = eos_p(q, eps, am, e);
    P.out[cell] = am;
    P.out[nn + cell] = p;
#pragma unroll
    for (int d = 0; d < DIM; d++) P.out[(int64_t)(2 + d) * nn + cell] = u[d];
    if (PASS != PASS_PRED) P.out[(int64_t)(2 + DIM) * nn + cell] = E;
#pragma unroll
    for (int t = 0; t < NTM; t++)  // Cell::timeEvolution / CellO2::predictionOrdre2
      if (t < P.ntr) P.out[(int64_t)(NS + t) * nn + cell] = tn[t] + at[t] * scale;
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

template <int DIM, int PASS, int NTM>
static cudaError_t euler_one(const StepParams& P, const Geometry& G, const ecg_eos* eos, double eps, cudaStream_t s,
                             bool prepare) {
  using K = EulerStep<DIM, PASS, NTM>;
  using TS = TileShape<DIM>;
  auto kern = k_euler_step<DIM, PASS, NTM>;
  const size_t sm = K::smem_bytes();
  if (prepare) return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  EosParams q{eos[0].type, eos[0].gamma, eos[0].pinf, eos[0].b, eos[0].cv, eos[0].eref, eos[0].sref};
  dim3 grid((G.n[0] + TS::X - 1) / TS::X, (G.n[1] + TS::Y - 1) / TS::Y, (G.n[2] + TS::Z - 1) / TS::Z);
  kern<<<grid, K::NTH, sm, s>>>(P, G, q, eps);
  return cudaGetLastError();
}

template <int DIM, int NTM>
static cudaError_t euler_dim_tr(int pass, const StepParams& P, const Geometry& G, const ecg_eos* eos, double eps,
                                cudaStream_t s, bool prepare) {
  if (pass == PASS_O1) return euler_one<DIM, PASS_O1, NTM>(P, G, eos, eps, s, prepare);
  if (pass == PASS_PRED) return euler_one<DIM, PASS_PRED, NTM>(P, G, eos, eps, s, prepare);
  return euler_one<DIM, PASS_CORR, NTM>(P, G, eos, eps, s, prepare);
}

template <int DIM>
static cudaError_t euler_dim(int pass, const StepParams& P, const Geometry& G, const ecg_eos* eos, double eps,
                             cudaStream_t s, bool prepare) {
  if (P.ntr > 2) return cudaErrorNotSupported;
  if (P.ntr > 0) return euler_dim_tr<DIM, 2>(pass, P, G, eos, eps, s, prepare);  // up to two passive transports
  return euler_dim_tr<DIM, 0>(pass, P, G, eos, eps, s, prepare);
}

cudaError_t euler_launch(int dim, int pass, const StepParams& P, const Geometry& G, const ecg_eos* eos, double eps,
                         cudaStream_t s, bool prepare) {
  if (dim == 1) return euler_dim<1>(pass, P, G, eos, eps, s, prepare);
  if (dim == 2) return euler_dim<2>(pass, P, G, eos, eps, s, prepare);
  return euler_dim<3>(pass, P, G, eos, eps, s, prepare);
}

}  // namespace ecg
