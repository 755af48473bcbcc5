// Per-cell pieces of the Kapila step shared by the single-case kernels (ecg_step_kapila.cu) and
// the batched kernel (ecg_batch.cu): face reconstruction, flux accumulation and the cell update
// (U^n, time evolution, buildPrim, relaxations, energy correction, store).
#pragma once
#include "ecg_mlp_device.cuh"
#include "ecg_step.cuh"

namespace ecg {

struct CellCounters {
  unsigned int relax = 0, iters = 0, fallback = 0, seeded = 0, rejected = 0, nonfinite = 0, ptmu = 0;
  PtmuCount pc;  // p-T-mu iteration counts (kernels with p-T-mu relaxation)
};

// Reconstructs one side of an internal face (CellInterfaceO2Cartesian::solveRiemann
// src/Order2/CellInterfaceO2Cartesian.cpp:101-160 with CellO2Cartesian::computeLocalSlopes
// src/Order2/CellO2Cartesian.cpp:23-171 on a Cartesian mesh): the limited slope combines the slope
// of this face (s1) and of the face on the opposite side of the cell along the same axis (s2, zero
// when that face is a boundary); the interface detector decides between the global and interface
// limiters; the state is extrapolated by `sign * slope * dist` and clamped.  With THINC
// (CellInterfaceO2Cartesian.cpp:132-150 left side, :164-181 right side, whose final expressions
// differ and are kept as they are) alpha_0 and alpha_1 = 1 - alpha_0 of an interface cell are then
// replaced by the hyperbolic-tangent reconstruction.
template <int NP, int DIM, bool THINC = true, int LIMC = -1>
__device__ ECG_RECON_INLINE void reconstruct_side(const Model<NP>& M, const StepParams& P, const double* sq, int RS,
                                                 int rc, const double* ssl, int SS, int f1, int f2, double alphaCell,
                                                 double alphaOther, double alphaAfter, double dist, double sign,
                                                 Thermo<NP>& t, double u[3]) {
  const int* lim = P.lim;
  using FL = Fields<NP, DIM>;
  const bool iface = (alphaCell >= 1.e-4) && (alphaCell <= 1. - 1.e-4) &&
                     ((alphaOther - alphaCell) * (alphaCell - alphaAfter) >= 1.e-8);
  // LIMC >= 0: one limiter compiled in for all four slots
  const int lg = LIMC >= 0 ? LIMC : (iface ? lim[1] : lim[0]);
  const int lv = LIMC >= 0 ? LIMC : (iface ? lim[3] : lim[2]);
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
  if (THINC && NP >= 2 && P.thinc && iface) {
    const double beta = 1.6, eps = 1.e-4;
    const bool right = sign < 0.;
    // neighbours: (right cell, left-left cell) for a left side, (right-right cell, left cell) for a right side
    const double hi = right ? alphaAfter : alphaOther, lo = right ? alphaOther : alphaAfter;
    const double sg = (hi - lo > 0.) ? 1. : -1.;
    const double qmin = dmin(hi, lo);
    const double qmax = dmax(hi, lo) - qmin;
    const double C = ddiv(alphaCell - qmin + 1.e-20, qmax + 1.e-20);
    const double B = exp(sg * beta * (2. * C - 1.));
    const double A = ddiv(ddiv(B, P.thinc_cosh) - 1., P.thinc_tanh);
    double na = right ? qmin + 0.5 * qmax * (1. + sg * A)
                      : qmin + 0.5 * qmax * (1. + ddiv(sg * (P.thinc_tanh + A), 1. + A * P.thinc_tanh));
    if (na < eps) na = eps;
    if (na > 1. - eps) na = 1. - eps;
    t.a[0] = na;
    t.a[1] = 1. - na;
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


// Non-reflecting boundary face of a cell: HLLC(cell, cell) in the face frame, subtracted from the
// cell (BoundCondNonReflecting::solveRiemannBoundary src/BoundConds/BoundCondNonReflecting.cpp:62,
// BoundCond::computeFlux src/BoundConds/BoundCond.cpp:61; the buffer cell is fulfilled first, :84).
template <int NP, int DIM>
__device__ __forceinline__ void boundary_face(const Model<NP>& M, const double* q, int64_t nn, int64_t cell, int ax,
                                              bool neg, double lcfl, double coefA, double& dtmax, const double an[NP],
                                              const double pn[NP], double aa[NP], double am[NP], double ae[NP],
                                              double amom[DIM], double& aE, double* sM_out = nullptr) {
  using FL = Fields<NP, DIM>;
  Thermo<NP> t;
  double ug[3], ul[3], Fn[3];
#pragma unroll
  for (int k = 0; k < NP; k++) {
    t.a[k] = q[(int64_t)(FL::A + k) * nn + cell];
    t.r[k] = q[(int64_t)(FL::R + k) * nn + cell];
    t.p[k] = eos_fix_p(M.eos[k], q[(int64_t)FL::P * nn + cell]);
  }
  ug[0] = ug[1] = ug[2] = 0.;
#pragma unroll
  for (int d = 0; d < DIM; d++) ug[d] = q[(int64_t)(FL::U + d) * nn + cell];
  fulfill<NP>(M, t);
  to_local(ax, neg, ug, ul);
  Flux<NP> F;
  hllc<NP>(M, t, ul, t, ul, lcfl, lcfl, dtmax, Fn, F);
  to_global(ax, neg, Fn, F.mom);
  acc_face<NP, DIM>(coefA, false, F, an, pn, aa, am, ae, amom, aE);
  if (sM_out) *sM_out = F.sM;
}

// Buffer cell of a symmetry side in a MUSCL pass (BoundCondWallO2Cartesian::solveRiemann
// src/BoundConds/BoundCondWallO2Cartesian.cpp:111-141 with CellO2Cartesian::computeLocalSlopesLimite
// src/Order2/CellO2Cartesian.cpp:173-272): slope 1 is the side's own slope (fw), slope 2 the slope of the
// internal face on the opposite side (fo); the interface detector only tests the cell's time-n alpha;
// the state is extrapolated by slope * dist (dist signed) without the clamps of the internal faces.
template <int NP, int DIM>
__device__ __forceinline__ void wall_side(const Model<NP>& M, const int lim[4], const double* sq, int RS, int rc,
                                          const double* ssl, int SS, int fw, int fo, double alphaN, double dist,
                                          Thermo<NP>& t, double u[3]) {
  using FL = Fields<NP, DIM>;
  const bool iface = (alphaN >= 1.e-4) && (alphaN <= 1. - 1.e-4);
  const int lg = iface ? lim[1] : lim[0];
  const int lv = iface ? lim[3] : lim[2];
#pragma unroll
  for (int k = 0; k < NP; k++) {
    double la = limiter(lv, ssl[k * SS + fw], ssl[k * SS + fo]);
    double lr = limiter(lg, ssl[(NP + k) * SS + fw], ssl[(NP + k) * SS + fo]);
    double lp = limiter(lg, ssl[(2 * NP + k) * SS + fw], ssl[(2 * NP + k) * SS + fo]);
    t.a[k] = sq[(FL::A + k) * RS + rc] + la * dist;
    t.r[k] = sq[(FL::R + k) * RS + rc] + lr * dist;
    t.p[k] = eos_fix_p(M.eos[k], sq[FL::P * RS + rc]) + lp * dist;
  }
  u[0] = u[1] = u[2] = 0.;
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    double l = limiter(lg, ssl[(3 * NP + d) * SS + fw], ssl[(3 * NP + d) * SS + fo]);
    u[d] = sq[(FL::U + d) * RS + rc] + l * dist;
  }
  fulfill<NP>(M, t);
}

// Symmetry side (also an inviscid wall): ModUEq::solveRiemannWall src/Models/UEq/ModUEq.cpp:452-492 on the
// fulfilled buffer cell t with face-frame velocity ul.  Returns the normal momentum flux pStar; every other
// flux component, sM and uStar are zero.
template <int NP>
__device__ __forceinline__ double wall_pstar(const Thermo<NP>& t, const double ul[3], double lcfl, double& dtmax) {
  const double uL = ul[0], cL = t.cF, pL = t.pm, rhoL = t.rho;
  const double sL = dmin(uL - cL, -uL - cL);
  if (fabs(sL) > 1.e-3) dtmax = dmin(dtmax, ddiv(1. * lcfl, fabs(sL)));
  return rhoL * (uL - sL) * uL + pL;
}

// Subtracts a symmetry side's flux (zero but for the normal momentum pStar) from the cell
// (BoundCond::computeFlux src/BoundConds/BoundCond.cpp:61).
template <int NP, int DIM>
__device__ __forceinline__ void wall_acc(int ax, bool neg, double pstar, double coefA, const double an[NP],
                                         const double pn[NP], double aa[NP], double am[NP], double ae[NP],
                                         double amom[DIM], double& aE) {
  Flux<NP> F;
#pragma unroll
  for (int k = 0; k < NP; k++) F.a[k] = F.m[k] = F.en[k] = 0.;
  F.E = 0.;
  F.sM = 0.;
  F.uStar = 0.;
  const double Fn[3] = {pstar, 0., 0.};
  to_global(ax, neg, Fn, F.mom);
  acc_face<NP, DIM>(coefA, false, F, an, pn, aa, am, ae, amom, aE);
}

// State of a cell after buildPrim, handed from kapila_rebuild to kapila_finish (the learned seed, when
// installed, is evaluated between the two by the whole warp).
template <int NP, int DIM>
struct CellPrim {
  double a[NP], r[NP], pk[NP];
  double u[DIM];
  double usq, E, rhomix;
};

// The cell update that follows the flux accumulation of one pass (everything after the face loop
// of solveHyperbolic for one cell), first half: U^n, time evolution and buildPrim.  aa/am/ae/amom/aE
// hold sum_faces coefA*F (+ the non-conservative terms); an/rn/pn are the time-n alpha_k, rho_k, p_k.
template <int NP, int DIM, int PASS>
__device__ __forceinline__ void kapila_rebuild(const StepParams& P, const Model<NP>& M, int64_t nn, int64_t cell,
                                               double dt, const double an[NP], const double rn[NP],
                                               const double pn[NP], double aa[NP], double am[NP], double ae[NP],
                                               double amom[DIM], double aE, CellPrim<NP, DIM>& cp) {
  using FL = Fields<NP, DIM>;
  // ---- U^n (FluxUEq::buildCons src/Models/UEq/FluxUEq.cpp:147) and time evolution
  //      (Cell::timeEvolution src/Order1/Cell.cpp:286: m_cons*dt then + U^n)
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
  double* a = cp.a;
  double* r = cp.r;
  double* pk = cp.pk;
  double rhoMel = 0.;
#pragma unroll
  for (int k = 0; k < NP; k++) {
    aa[k] = ddiv(aa[k], un_sum);
    rhoMel += am[k];
    a[k] = aa[k];
    r[k] = ddiv(am[k], dmax(aa[k], M.eps));
    if (M.eos[k].type == ECG_EOS_NASG && r[k] > ddiv(1., M.eos[k].b) - 1.) {  // verifyAndCorrectDensityMax(mass)
      r[k] = ddiv(1., M.eos[k].b) - 1.;
      a[k] = ddiv(am[k], r[k]);
    }
    double ek = ddiv(ae[k], dmax(am[k], M.eps));
    pk[k] = eos_p(M.eos[k], M.eps, r[k], ek);
    phase_fix_ar(M.eps, a[k], r[k]);
    pk[k] = eos_fix_p(M.eos[k], pk[k]);
  }
  double* u = cp.u;
  double usq = 0.;
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    u[d] = ddiv(amom[d], rhoMel);
    if (fabs(u[d]) < 1.e-8) u[d] = 0.;
    usq += u[d] * u[d];
  }
  cp.usq = usq;
  cp.E = ddiv(aE, rhoMel);
  // mixture density (and internal energy for p-T-mu) of the rebuilt state
  double rhomix = 0.;
#pragma unroll
  for (int k = 0; k < NP; k++) rhomix += a[k] * r[k];
  cp.rhomix = rhomix;
}


// The learned seed of a seeded kernel, gated on the plain start: the first Newton evaluation at
// sum_k alpha_k p_k is made for every cell (the plain iteration's first step); only cells it leaves
// unconverged ("hard") take the network's seed, which the warp evaluates when any of its lanes needs it.
template <int NP>
struct SeedGate {
  NewtonState ns;        // state after the first evaluation
  double aS[NP], rS[NP];
  double seed;
  bool applies, hard;
  // p-T-mu relaxation: the network's (p*, T) start and the features it was evaluated on
  double ptmu_p = -1., ptmu_T = -1.;
  float ptmu_x[PTMU_NIN];
};

// Mixture internal energy of the rebuilt state, sum_k Y_k e_k(rho_k, p_k) (MixUEq::computeMixtureVariables
// :136), which RelaxationPTMu reads before any fulfillState.
template <int NP>
__device__ __forceinline__ double rebuilt_emix(const Model<NP>& M, const double a[NP], const double r[NP],
                                               const double p[NP], double rhomix) {
  double emix = 0.;
#pragma unroll
  for (int k = 0; k < NP; k++) {
    double Y = ddiv(a[k] * r[k], dmax(rhomix, M.eps));
    emix += Y * eos_e(M.eos[k], M.eps, r[k], p[k]);
  }
  return emix;
}

// The learned (p*, T) start of the p-T-mu relaxation of every cell of the warp (all lanes call it;
// `active` marks a cell): features of the rebuilt state, the network, then the checks that keep a seed
// (finite, positive, p* below the critical pressure); a rejected seed leaves the plain start.
template <int NP, int DIM>
__device__ __forceinline__ void ptmu_seed_gate(const StepParams& P, const Model<NP>& M, bool active,
                                               const CellPrim<NP, DIM>& cp, SeedGate<NP>& g, CellCounters& cc) {
  if (active) {
    const double emix = rebuilt_emix<NP>(M, cp.a, cp.r, cp.pk, cp.rhomix);
    ptmu_features<NP>(M, P.ptmu_liq, P.ptmu_vap, cp.a, cp.r, cp.pk, cp.rhomix, emix, g.ptmu_x);
  }
  double ps = -1., Ts = -1.;
  mlp_ptmu_seed_warp(P.mlp, active, g.ptmu_x, ps, Ts);
  g.ptmu_p = g.ptmu_T = -1.;
  if (!active) return;
  // the T start is used when finite and positive; the p* start (ECG_PTMU_SEED_P_T only) when finite,
  // positive and below the critical pressure as well
  const bool okT = isfinite(Ts) && Ts > 0.;
  const bool okP = !P.ptmu_seed_p || (isfinite(ps) && ps > 0. && ps < P.pcrit);
  if (okT && okP) {
    g.ptmu_p = P.ptmu_seed_p ? ps : -1.;
    g.ptmu_T = Ts;
  } else {
    cc.pc.rejected = 1;
  }
}

// First evaluation and the warp-wide seed (all lanes of the warp call it; `active` marks a cell).
template <int NP, int DIM>
__device__ __forceinline__ void seed_gate(const StepParams& P, const Model<NP>& M, bool active,
                                          const CellPrim<NP, DIM>& cp, SeedGate<NP>& g) {
  g.applies = active && pinf_applies<NP>(M, cp.a);
  g.hard = false;
  if (g.applies) {
    pinf_first<NP>(M, cp.a, cp.r, cp.pk, g.ns, g.aS, g.rS);
    g.hard = fabs(g.ns.f) > 1e-10 && g.ns.it < P.newton_cap;
  }
  g.seed = 0.;
  if (__any_sync(0xffffffffu, g.hard)) g.seed = mlp_seed_warp<NP>(P.mlp, g.hard, cp.a, cp.r, cp.pk);
}

// Relaxations, energy correction, clamps and store of one rebuilt cell.  SEED: the pressure
// relaxation continues from the seed gate (see seed_gate); a hard cell restarts Newton from the
// network's seed when it is finite and inside the bracket of the phase pressures, otherwise it
// continues the plain iteration.  Newton still stops at |f| <= 1e-10 either way.
// RelaxationPT::relaxation src/Relaxations/RelaxationPT.cpp:43-140: analytic pressure-temperature
// equilibrium of two IG/SG phases (Le Martelot 2013) from the mixture energy and density of the rebuilt
// state (emix, rho0) and its mass fractions, then rho_k = computeDensity(p*, T*).
template <int NP>
__device__ __forceinline__ void relax_pt(const Model<NP>& M, double a[NP], double r[NP], double pk[NP],
                                         const double Y[NP], double emix, double rho0) {
  if (M.eps > 1.e-20) {
#pragma unroll
    for (int k = 0; k < NP; k++)
      if (a[k] > (1. - 1.e-5)) return;
  }
  const EosParams& E1 = M.eos[0];
  const EosParams& E2 = M.eos[1];
  const double pInf1 = (E1.type == ECG_EOS_IG) ? 0. : E1.pinf, pInf2 = (E2.type == ECG_EOS_IG) ? 0. : E2.pinf;
  const double q = Y[0] * E1.eref + Y[1] * E2.eref;
  const double cvMel = Y[0] * E1.cv + Y[1] * E2.cv;
  const double A1 = ddiv(Y[0] * (E1.gamma - 1.) * E1.cv, cvMel) * (rho0 * (emix - q) - pInf1);
  const double A2 = ddiv(Y[1] * (E2.gamma - 1.) * E2.cv, cvMel) * (rho0 * (emix - q) - pInf2);
  const double pressure = 0.5 * (A1 + A2 - (pInf1 + pInf2)) +
                          dsqrt(0.25 * (A2 - A1 - (pInf2 - pInf1)) * (A2 - A1 - (pInf2 - pInf1)) + A1 * A2);
  double temperature = 0.;
  temperature += ddiv(Y[0] * (E1.gamma - 1.) * E1.cv, pressure + pInf1);
  temperature += ddiv(Y[1] * (E2.gamma - 1.) * E2.cv, pressure + pInf2);
  temperature = ddiv(1., temperature * rho0);
  double rS[2], aS[2];
#pragma unroll
  for (int k = 0; k < 2; k++) {
    const EosParams& E = M.eos[k];
    const double den = dmax((E.gamma - 1.) * E.cv * temperature, M.eps);
    rS[k] = (E.type == ECG_EOS_IG) ? ddiv(pressure, den) : ddiv(pressure + E.pinf, den);
    aS[k] = ddiv(a[k] * r[k], rS[k]);
  }
#pragma unroll
  for (int k = 0; k < 2; k++) {
    a[k] = aS[k];
    r[k] = rS[k];
    pk[k] = pressure;
  }
}

// SEED: with PTMU, the learned (p*, T) start of the p-T-mu relaxation (ptmu_seed_gate), the pressure
// relaxation plain; without, the learned start of the pressure relaxation (seed_gate).
template <int NP, int DIM, int PASS, bool PTMU, bool SEED = false, bool XPT = true>
__device__ __forceinline__ void kapila_finish(const StepParams& P, const Model<NP>& M, int64_t nn, int64_t cell,
                                              CellPrim<NP, DIM>& cp, const SeedGate<NP>& g, CellCounters& cc) {
  constexpr bool kPinfSeed = SEED && !PTMU;
  using FL = Fields<NP, DIM>;
  double* a = cp.a;
  double* r = cp.r;
  double* pk = cp.pk;
  const double* u = cp.u;
  const double usq = cp.usq, E = cp.E;
  double rhomix = cp.rhomix;
  // ---- relaxations (Model::relaxations src/Models/Model.cpp:74): pressure, then p-T-mu
  RelaxStats rs;
  double a0[NP], r0[NP], p0[NP];
#pragma unroll
  for (int k = 0; k < NP; k++) { a0[k] = a[k]; r0[k] = r[k]; p0[k] = pk[k]; }
  double pstar = 0.;
  bool relaxed;
  if (kPinfSeed) {
    rs.iters = 0;
    rs.fallback = rs.seeded = rs.rejected = false;
    relaxed = g.applies;
    if (relaxed) {
      NewtonState s = g.ns;
      double aS[NP], rS[NP];
#pragma unroll
      for (int k = 0; k < NP; k++) { aS[k] = g.aS[k]; rS[k] = g.rS[k]; }
      if (g.hard) {
        double lo = pk[0], hi = pk[0];
#pragma unroll
        for (int k = 1; k < NP; k++) { lo = dmin(lo, pk[k]); hi = dmax(hi, pk[k]); }
        if (isfinite(g.seed) && g.seed >= lo && g.seed <= hi) {
          s.ps = g.seed - 0. / 1.;
          s.it += 1;
          pinf_eval<NP>(M, a, r, s, pk, aS, rS);
          rs.seeded = true;
        } else {
          rs.rejected = true;
        }
      }
      pinf_finish<NP>(M, a, r, pk, s, aS, rS, pstar, rs, P.newton_cap, P.newton_accept != 0);
    }
  } else {
    relaxed = relax_pinf<NP>(M, a, r, pk, pstar, rs, 0., false, P.newton_cap, P.newton_accept != 0);
  }
  if (relaxed) {
#pragma unroll
    for (int k = 0; k < NP; k++) pk[k] = pstar;
    if (!PTMU && P.rec_x != nullptr && !rs.fallback && rs.iters >= P.rec_min_evals)
      record_pair<NP>(P.rec_x, P.rec_y, P.rec_count, P.rec_max, a0, r0, p0, pstar);
  }
  if (PTMU) {
    // mixture internal energy of the rebuilt state (MixUEq::computeMixtureVariables :136), which
    // RelaxationPTMu reads before any fulfillState
    const double emix = rebuilt_emix<NP>(M, a0, r0, p0, rhomix);
    bool err = false;
    const double ps = SEED ? g.ptmu_p : -1.;
    // T_sat start: the network's (seeded kernels), else the cell's previous converged T_sat when the
    // warm start is on (a value <= 0: no solve yet, cold start), else the reference's cold start
    const double Ts = SEED ? g.ptmu_T : (P.tsat_hist != nullptr ? P.tsat_hist[cell] : -1.);
    if (relax_ptmu<NP>(M, P.ptmu_liq, P.ptmu_vap, P.pcrit, a, r, pk, rhomix, emix, err, &cc.pc, ps, Ts)) {
      rhomix = 0.;
#pragma unroll
      for (int k = 0; k < NP; k++) rhomix += a[k] * r[k];
    }
    if (cc.pc.solve && Ts > 0.) cc.pc.seeded = 1;
    if (P.tsat_hist != nullptr && cc.pc.solve && !err) P.tsat_hist[cell] = cc.pc.tsat;
    if (P.rec_x != nullptr && cc.pc.solve && !err && (int)cc.pc.outer >= P.rec_min_evals) {
      float x[PTMU_NIN];
      if (SEED) {
#pragma unroll
        for (int j = 0; j < PTMU_NIN; j++) x[j] = g.ptmu_x[j];
      } else {
        ptmu_features<NP>(M, P.ptmu_liq, P.ptmu_vap, a0, r0, p0, cp.rhomix, emix, x);
      }
      record_ptmu_pair(P.rec_x, P.rec_y, P.rec_count, P.rec_max, x, cc.pc.pstar, cc.pc.tsat);
    }
    if (err) cc.ptmu = 1;
  }
  if (XPT && !PTMU && NP == 2 && P.pt) {
    // RelaxationPT reads the mass fractions and mixture energy of the rebuilt state
    double Y[NP], emix = 0.;
#pragma unroll
    for (int k = 0; k < NP; k++) {
      Y[k] = ddiv(a0[k] * r0[k], dmax(rhomix, M.eps));
      emix += Y[k] * eos_e(M.eos[k], M.eps, r0[k], p0[k]);
    }
    relax_pt<NP>(M, a, r, pk, Y, emix, rhomix);
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
    cc.relax = 1;
    cc.iters = (unsigned int)rs.iters;
    cc.fallback = rs.fallback ? 1u : 0u;
    cc.seeded = rs.seeded ? 1u : 0u;
    cc.rejected = rs.rejected ? 1u : 0u;
  }
  cc.nonfinite = finite ? 0u : 1u;
}

}  // namespace ecg
