// Device-side physics of the ECOGEN Cartesian FV step, in FP64.
//
// Every routine restates a reference routine (file:line relative to the ECOGEN
// tree) with the same operation order, so that results agree with the CPU code
// to the last bits except where a math function's result differs from glibc's by
// an ulp (epow, ecg_pow.cuh: in about 0.1 % of the calls, where glibc's pow is
// not correctly rounded; exp of the THINC reconstruction).  Divisions and square
// roots go through ddiv / dsqrt (ecg_ieee.cuh), which return the IEEE quotient and
// root bit for bit without a branch.  Kernels are built with --fmad=false so that
// no multiply-add is contracted, as in the reference's x86-64 SSE2 build.
//
// Compact state.  The reference keeps per phase (alpha, rho, p, T, e, c, Y) and per
// cell a mixture record (rho, p, u, e, E, cF, cWood).  After each full step every
// phase pressure equals the mixture-EOS pressure p clamped by that phase's EOS floor
// (FluxPUEq::correctionEnergy src/Models/PUEq/FluxPUEq.cpp:68-112 sets p_k = p then
// PhaseUEq::verifyAndCorrectPhase clamps it), and T, e, c, Y and the mixture record
// are pure functions of (alpha_k, rho_k, p_k, u).  So the state that defines a step is
// (alpha_k, rho_k)_k, p, u (DIM components) and E, and everything else is recomputed.
#pragma once
#include <cstdint>

#include "ecg_ieee.cuh"
#include "ecg_pow.cuh"
#include "ecg_types.h"

// Inlining of the two largest face routines (HLLC and the MUSCL side reconstruction).  Inlined, the
// fused pass holds one copy per axis and side; as calls, one copy each (smaller instruction
// footprint, call overhead).  Build-time choice, measured by the benchmark.
#ifndef ECG_HLLC_INLINE
#define ECG_HLLC_INLINE __forceinline__
#endif
#ifndef ECG_RECON_INLINE
#define ECG_RECON_INLINE __forceinline__
#endif

namespace ecg {

// std::max / std::min with libstdc++'s argument order (NaN behaviour included)
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }

// ----------------------------------------------------------------------------------------- EOS
// src/Eos/EosIG.cpp:64-257, src/Eos/EosSG.cpp:66-257, src/Eos/EosNASG.cpp:68-280

__device__ __forceinline__ double eos_T(const EosParams& q, double eps, double rho, double p) {
  if (q.type == ECG_EOS_IG) return ddiv(ddiv(ddiv(p, q.gamma - 1.), dmax(rho, eps)), q.cv);
  if (q.type == ECG_EOS_SG) return ddiv(ddiv(ddiv(p + q.pinf, q.gamma - 1.), dmax(rho, eps)), q.cv);
  return ddiv(ddiv(ddiv((p + q.pinf) * dmax(1. - rho * q.b, eps), q.gamma - 1.), q.cv), dmax(rho, eps));
}

__device__ __forceinline__ double eos_e(const EosParams& q, double eps, double rho, double p) {
  if (q.type == ECG_EOS_IG) return ddiv(ddiv(p, q.gamma - 1.), dmax(rho, eps)) + q.eref;
  if (q.type == ECG_EOS_SG) return ddiv(ddiv(p + q.gamma * q.pinf, q.gamma - 1.), dmax(rho, eps)) + q.eref;
  return ddiv(ddiv((p + q.gamma * q.pinf) * dmax(1. - rho * q.b, eps), q.gamma - 1.), dmax(rho, eps)) + q.eref;
}

__device__ __forceinline__ double eos_p(const EosParams& q, double eps, double rho, double e) {
  if (q.type == ECG_EOS_IG) return (q.gamma - 1.) * rho * (e - q.eref);
  if (q.type == ECG_EOS_SG) return (q.gamma - 1.) * rho * (e - q.eref) - q.gamma * q.pinf;
  return (ddiv(rho * (q.gamma - 1.) * (e - q.eref), dmax(1. - rho * q.b, eps)) - q.gamma * q.pinf);
}

__device__ __forceinline__ double eos_c(const EosParams& q, double eps, double rho, double p) {
  if (q.type == ECG_EOS_IG) return dsqrt(ddiv(q.gamma * p, dmax(rho, eps)));
  if (q.type == ECG_EOS_SG) return dsqrt(ddiv(q.gamma * (p + q.pinf), dmax(rho, eps)));
  return dsqrt(ddiv(q.gamma * (p + q.pinf), dmax(rho * (1. - rho * q.b), eps)));
}

__device__ __forceinline__ double nonzero(double a, double eps) {  // Tools::returnNonZeroValue src/Tools.cpp:134
  if (a > eps || a < -eps) return a;
  int sg = (0. < a) - (a < 0.);
  return sg * eps;
}

__device__ __forceinline__ double eos_p_isentropic(const EosParams& q, double eps, double p0, double rho0,
                                                   double rho1) {
  if (q.type == ECG_EOS_IG) return p0 * epow(ddiv(rho1, dmax(rho0, eps)), q.gamma);
  if (q.type == ECG_EOS_SG) return (p0 + q.pinf) * epow(ddiv(rho1, dmax(rho0, eps)), q.gamma) - q.pinf;
  return (p0 + q.pinf) * epow(ddiv(rho1, dmax(rho0, eps)), q.gamma) * epow(ddiv(1. - rho0 * q.b, 1. - rho1 * q.b), q.gamma) -
         q.pinf;
}

__device__ __forceinline__ double eos_rho_pfinal(const EosParams& q, double eps, double p0, double rho0, double p1,
                                                 double* drhodp) {
  double num, denom, rho1;
  if (q.type == ECG_EOS_IG) {
    num = q.gamma * p1;
    denom = num + p0 - p1;
    rho1 = ddiv(rho0 * num, dmax(denom, eps));
    *drhodp = ddiv(rho0 * q.gamma * p0, dmax(denom * denom, eps));
    return rho1;
  }
  if (q.type == ECG_EOS_SG) {
    num = q.gamma * (p1 + q.pinf);
    denom = num + p0 - p1;
    rho1 = ddiv(rho0 * num, nonzero(denom, eps));
    *drhodp = ddiv(rho0 * q.gamma * (p0 + q.pinf), dmax(denom * denom, eps));
    return rho1;
  }
  num = q.gamma * (p1 + q.pinf);
  denom = num + p0 - p1 + q.b * rho0 * (p1 - p0);
  rho1 = ddiv(rho0 * num, nonzero(denom, eps));
  *drhodp = ddiv(rho0 * q.gamma * (p0 + q.pinf - q.b * rho0 * (p0 + q.pinf)), nonzero(denom * denom, eps));
  return rho1;
}

// verifyAndModifyPressure (EosIG.cpp:250, EosSG.cpp:252, EosNASG.cpp:268)
__device__ __forceinline__ double eos_fix_p(const EosParams& q, double p) {
  if (q.type == ECG_EOS_IG) return (p < 1.e-8) ? 1.e-8 : p;
  double floor = -(1. - 1.e-15) * q.pinf + 1.e-15;
  return (p <= floor) ? floor : p;
}

__device__ __forceinline__ void eos_rho_max(const EosParams& q, double& rho) {  // verifyAndCorrectDensityMax(density)
  if (q.type == ECG_EOS_NASG && rho > ddiv(1., q.b) - 1.) rho = ddiv(1., q.b) - 1.;
}

// ------------------------------------------------------------------------------ model parameters

template <int NP>
struct Model {
  EosParams eos[NP];
  double eps;  // epsilonAlphaNull: 1e-15 with alphaNull, else 0 (src/Eos/Eos.cpp:88-97)
};

// Kernel configuration known at compile time ("fast" kernels): the type of phase k in bits
// 2k..2k+1 (ECG_EOS_IG 0, SG 1, NASG 2) and, in bits 8 and up, one more than a limiter used for all
// four limiter slots (0: limiters read at run time).  EOS_DYNAMIC marks the generic kernels.  With
// known types and limiter every EOS and limiter branch folds away (the arithmetic is unchanged),
// which shrinks the fused kernels' code.
constexpr int EOS_DYNAMIC = -1;
template <int NP>
__host__ __device__ constexpr int eos_types_code(int t0, int t1, int t2 = 0) {
  return NP == 2 ? (t0 | (t1 << 2)) : (t0 | (t1 << 2) | (t2 << 4));
}
__host__ __device__ constexpr int fast_code(int types, int limiter) { return types | ((limiter + 1) << 8); }
__host__ __device__ constexpr int code_limiter(int code) { return code == EOS_DYNAMIC ? -1 : (code >> 8) - 1; }
template <int NP, int TYPES>
__device__ __forceinline__ Model<NP> specialize_eos(const Model<NP>& M0) {
  Model<NP> M = M0;
  if (TYPES != EOS_DYNAMIC) {
#pragma unroll
    for (int k = 0; k < NP; k++) M.eos[k].type = (TYPES >> (2 * k)) & 3;
  }
  return M;
}

// PhaseUEq::verifyAndCorrectPhase src/Models/UEq/PhaseUEq.cpp:348 (alpha / density clamps)
__device__ __forceinline__ void phase_fix_ar(double eps, double& a, double& r) {
  if (eps > 1.e-20) {
    if (a < 0.) a = 0.;
    if (a > 1.) a = 1.;
    if (r <= 1.e-15) r = 1.e-15;
  } else {
    if (a < 1e-15) a = 1e-14;
    if (a > 1. - 1e-15) a = 1. - 1e-14;
    if (r < 1.e-15) r = 1.e-14;
  }
}

// Thermodynamic closure of one side of a face or of a cell: what fulfillState computes
// (ModUEq::fulfillState src/Models/UEq/ModUEq.cpp:99 -> PhaseUEq::extendedCalculusPhase :97,
// MixUEq::computeMixtureVariables src/Models/UEq/MixUEq.cpp:136).
// The phase internal energies e_k and the mixture energy sum_k Y_k e_k are needed only on the side
// the HLLC solution is sampled from, so hllc() evaluates them once the side is known
// (hllc_side_energy); the values are the ones fulfillState would have produced.
template <int NP>
struct Thermo {
  double a[NP], r[NP], p[NP], Y[NP];
  double rho, pm, cF;
};

template <int NP>
__device__ __forceinline__ void fulfill(const Model<NP>& M, Thermo<NP>& t) {
  double c[NP];
#pragma unroll
  for (int k = 0; k < NP; k++) c[k] = eos_c(M.eos[k], M.eps, t.r[k], t.p[k]);
  t.rho = 0.;
  t.pm = 0.;
#pragma unroll
  for (int k = 0; k < NP; k++) {
    t.rho += t.a[k] * t.r[k];
    t.pm += t.a[k] * t.p[k];
  }
  double cF = 0.;
#pragma unroll
  for (int k = 0; k < NP; k++) {
    t.Y[k] = ddiv(t.a[k] * t.r[k], dmax(t.rho, M.eps));
    cF += t.Y[k] * c[k] * c[k];
  }
  t.cF = dsqrt(cF);
}

// PhaseUEq::extendedCalculusPhase energies and MixUEq::computeMixtureVariables' e = sum_k Y_k e_k.
template <int NP>
__device__ __forceinline__ double side_energy(const Model<NP>& M, const Thermo<NP>& t, double e[NP]) {
  double em = 0.;
#pragma unroll
  for (int k = 0; k < NP; k++) {
    e[k] = eos_e(M.eos[k], M.eps, t.r[k], t.p[k]);
    em += t.Y[k] * e[k];
  }
  return em;
}

// Face-frame projection of a Cartesian face (src/Maths/Coord.cpp:133-151 with the frames of
// src/Meshes/MeshCartesian.cpp:281-557).  axis 0/1/2; neg = true for the Xm/Ym/Zm boundary frames.
__device__ __forceinline__ void to_local(int axis, bool neg, const double u[3], double l[3]) {
  if (axis == 0) {
    if (!neg) { l[0] = u[0]; l[1] = u[1]; l[2] = u[2]; }
    else { l[0] = -u[0]; l[1] = -u[1]; l[2] = u[2]; }
  } else if (axis == 1) {
    if (!neg) { l[0] = u[1]; l[1] = -u[0]; l[2] = u[2]; }
    else { l[0] = -u[1]; l[1] = u[0]; l[2] = u[2]; }
  } else {
    if (!neg) { l[0] = u[2]; l[1] = u[0]; l[2] = u[1]; }
    else { l[0] = -u[2]; l[1] = -u[0]; l[2] = u[1]; }
  }
}
__device__ __forceinline__ void to_global(int axis, bool neg, const double f[3], double g[3]) {
  if (axis == 0) {
    if (!neg) { g[0] = f[0]; g[1] = f[1]; g[2] = f[2]; }
    else { g[0] = -f[0]; g[1] = -f[1]; g[2] = f[2]; }
  } else if (axis == 1) {
    if (!neg) { g[0] = -f[1]; g[1] = f[0]; g[2] = f[2]; }
    else { g[0] = f[1]; g[1] = -f[0]; g[2] = f[2]; }
  } else {
    if (!neg) { g[0] = f[1]; g[1] = f[2]; g[2] = f[0]; }
    else { g[0] = -f[1]; g[1] = f[2]; g[2] = -f[0]; }
  }
}

// Face flux of the Kapila / UEq system, in the absolute frame.
template <int NP>
struct Flux {
  double a[NP], m[NP], en[NP];
  double mom[3];
  double E;
  double sM, uStar;
};

// HLLC: ModUEq::solveRiemannIntern src/Models/UEq/ModUEq.cpp:113-267.  L and R carry local-frame
// velocities ul/ur (normal first).  dtmax is min-updated with lCFL/|s|.
template <int NP>
__device__ ECG_HLLC_INLINE void hllc(const Model<NP>& M, const Thermo<NP>& L, const double ul[3],
                                     const Thermo<NP>& R, const double ur[3], double dxL, double dxR,
                                     double& dtmax, double Fn[3], Flux<NP>& F) {
  double uL = ul[0], cL = L.cF, pL = L.pm, rhoL = L.rho;
  double uR = ur[0], cR = R.cF, pR = R.pm, rhoR = R.rho;
  double sL = dmin(uL - cL, uR - cR);
  double sR = dmax(uR + cR, uL + cL);
  if (fabs(sL) > 1.e-3) dtmax = dmin(dtmax, ddiv(1. * dxL, fabs(sL)));
  if (fabs(sR) > 1.e-3) dtmax = dmin(dtmax, ddiv(1. * dxR, fabs(sR)));
  double mL = rhoL * (sL - uL), mR = rhoR * (sR - uR);
  double sM = ddiv(pR - pL + mL * uL - mR * uR, mL - mR);
  if (fabs(sM) < 1.e-8) sM = 0.;
  F.sM = sM;
  if (sL >= 0. || sR <= 0.) {
    const bool left = (sL >= 0.);
    const Thermo<NP>& S = left ? L : R;
    const double* us = left ? ul : ur;
    double un = us[0], rhoS = S.rho, pS = S.pm;
    double e[NP];
    const double em = side_energy<NP>(M, S, e);
#pragma unroll
    for (int k = 0; k < NP; k++) {
      F.a[k] = S.a[k] * sM;
      F.m[k] = S.a[k] * S.r[k] * un;
      F.en[k] = S.a[k] * S.r[k] * e[k] * un;
    }
    double Et = em + 0.5 * (us[0] * us[0] + us[1] * us[1] + us[2] * us[2]);
    Fn[0] = rhoS * un * un + pS;
    Fn[1] = rhoS * us[1] * un;
    Fn[2] = rhoS * us[2] * un;
    F.E = (rhoS * Et + pS) * un;
    F.uStar = un;
  } else {
    const bool left = (sM >= 0.);
    const Thermo<NP>& S = left ? L : R;
    const double* us = left ? ul : ur;
    double sK = left ? sL : sR;
    double mK = left ? mL : mR;
    double uK = us[0], pK = S.pm;
    double e[NP];
    const double em = side_energy<NP>(M, S, e);
    double Et = em + 0.5 * (us[0] * us[0] + us[1] * us[1] + us[2] * us[2]);
    double rhoStar = ddiv(mK, sK - sM);
    double EStar = Et + (sM - uK) * (sM + ddiv(pK, mK));
    double pStar = mK * (sM - uK) + pK;
#pragma unroll
    for (int k = 0; k < NP; k++) {
      double mk = S.r[k] * (sK - uK);
      double rks = ddiv(mk, sK - sM);
      eos_rho_max(M.eos[k], rks);
      double pks = eos_p_isentropic(M.eos[k], M.eps, S.p[k], S.r[k], rks);
      double eks = eos_e(M.eos[k], M.eps, rks, pks);
      F.a[k] = S.a[k] * sM;
      F.m[k] = S.a[k] * rks * sM;
      F.en[k] = S.a[k] * rks * eks * sM;
    }
    Fn[0] = rhoStar * sM * sM + pStar;
    Fn[1] = rhoStar * us[1] * sM;
    Fn[2] = rhoStar * us[2] * sM;
    F.E = (rhoStar * EStar + pStar) * sM;
    F.uStar = sM;
  }
}

// Limiters src/Order2/Limiter{Minmod,VanLeer,VanAlbada,SuperBee,MC,THINC}.cpp:43-55
__device__ __forceinline__ double limiter(int kind, double s1, double s2) {
  double slope = 0., prod = s1 * s2;
  switch (kind) {
    case ECG_LIM_MINMOD:
    case ECG_LIM_THINC:
      if (prod > 1e-9) {
        slope = dmin(fabs(s1), fabs(s2));
        if (s1 < 0) slope = -slope;
      }
      return slope;
    case ECG_LIM_VANLEER: {
      double sum = s1 + s2;
      if ((fabs(sum) > 1e-6) && (prod > 1e-6)) slope = ddiv(2. * prod, sum);
      return slope;
    }
    case ECG_LIM_VANALBADA: {
      double sum = s1 + s2;
      if ((fabs(s1) > 1e-6) && (fabs(s2) > 1e-6) && (fabs(sum) > 1e-6) && (prod > 1e-6))
        slope = ddiv(prod * sum, s1 * s1 + s2 * s2);
      return slope;
    }
    case ECG_LIM_SUPERBEE:
      if (prod > 1e-6) slope = dmax(dmin(2. * fabs(s1), fabs(s2)), dmin(fabs(s1), 2. * fabs(s2)));
      if (s1 < 0.) slope = -slope;
      return slope;
    case ECG_LIM_MC:
      if (prod > 1e-9) {
        slope = dmin(2. * fabs(s1), 2. * fabs(s2));
        slope = dmin(slope, 0.5 * (fabs(s1) + fabs(s2)));
      }
      if (s1 < 0.) slope = -slope;
      return slope;
    default:
      return 0.;
  }
}

// ------------------------------------------------------------------------ relaxation (pressure)

struct RelaxStats {
  int iters;      // Newton evaluations of this cell (0 if skipped)
  bool fallback;  // reached 100 iterations -> interface pressure
  bool seeded;    // a learned seed was used
  bool rejected;  // the learned seed was rejected (plain start used)
};

// RelaxationPInfinite::relaxation src/Relaxations/RelaxationPInfinite.cpp:43-97 with
// RelaxationP::NewtonRaphson src/Relaxations/RelaxationP.cpp:43-68.  a/r/p are the phase state
// after buildPrim (p per phase); the phase sound speeds of that state are needed only by the
// interface-pressure fallback, RelaxationP::computeInterfacePressure :72, recomputed there from
// the same rho_k, p_k as PhaseUEq::extendedCalculusPhase does).  On return a/r hold
// the relaxed state and pstar the relaxed pressure; returns false if the relaxation was skipped.
template <int NP>
__device__ __forceinline__ bool relax_pinf(const Model<NP>& M, double a[NP], double r[NP], const double p[NP],
                                           double& pstar, RelaxStats& st, double seed, bool use_seed,
                                           int max_iter, bool accept = false) {
  st.iters = 0;
  st.fallback = false;
  st.seeded = false;
  st.rejected = false;
  if (M.eps > 1.e-20) {
    bool relax = true;
#pragma unroll
    for (int k = 0; k < NP; k++)
      if (a[k] > (1. - 1.e-5)) relax = false;
    if (!relax) return false;
  }
  double ps = 0.;
#pragma unroll
  for (int k = 0; k < NP; k++) ps += a[k] * p[k];
  if (use_seed) {
    // A learned initial guess replaces sum_k alpha_k p_k only when it is finite and inside the
    // bracket of the phase pressures; otherwise it is rejected and the plain start is kept.
    double lo = p[0], hi = p[0];
#pragma unroll
    for (int k = 1; k < NP; k++) { lo = dmin(lo, p[k]); hi = dmax(hi, p[k]); }
    if (isfinite(seed) && seed >= lo && seed <= hi) { ps = seed; st.seeded = true; }
    else st.rejected = true;
  }
  double aS[NP], rS[NP];
  double f = 0., df = 1., drhodp = 0.;
  int iteration = 0;
  do {
    iteration++;
    ps -= ddiv(f, df);
#pragma unroll
    for (int k = 0; k < NP; k++) ps = eos_fix_p(M.eos[k], ps);
    f = -1.;
    df = 0.;
#pragma unroll
    for (int k = 0; k < NP; k++) {
      rS[k] = eos_rho_pfinal(M.eos[k], M.eps, p[k], r[k], ps, &drhodp);
      aS[k] = ddiv(a[k] * r[k], rS[k]);
      double dalpha = ddiv(a[k] * r[k] * drhodp, rS[k] * rS[k]);
      f += aS[k];
      df -= dalpha;
    }
  } while (fabs(f) > 1e-10 && iteration < max_iter);
  st.iters = iteration;
  if (iteration < max_iter || accept) {  // accept: a capped iteration keeps its last iterate
#pragma unroll
    for (int k = 0; k < NP; k++) { a[k] = aS[k]; r[k] = rS[k]; }
    pstar = ps;
    return true;
  }
  st.fallback = true;
  double zk[NP], pI = 0., sumZk = 0.;
#pragma unroll
  for (int k = 0; k < NP; k++) zk[k] = r[k] * eos_c(M.eos[k], M.eps, r[k], p[k]);
#pragma unroll
  for (int k = 0; k < NP; k++) {
    sumZk += zk[k];
    double sumZj = 0.;
#pragma unroll
    for (int j = 0; j < NP; j++)
      if (j != k) sumZj += zk[j];
    pI += sumZj * (p[k] - 0.);
  }
  pI = ddiv(pI, sumZk * (NP - 1));
#pragma unroll
  for (int k = 0; k < NP; k++) pI = eos_fix_p(M.eos[k], pI);
#pragma unroll
  for (int k = 0; k < NP; k++) {
    double rr = eos_rho_pfinal(M.eos[k], M.eps, p[k], r[k], pI, &drhodp);
    a[k] = ddiv(a[k] * r[k], rr);
    r[k] = rr;
  }
  pstar = pI;
  return true;
}


// ------------------------------------------------------------------ logarithm of the saturation solve
// The saturation temperature solve (Mixture::computeTsat) branches on tight tests (pure-phase
// hypotheses, |f| > 1e-10), so a last-ulp difference between the device's log and the host libm's can
// change a cell's path.  It takes its logarithms from elog (ecg_pow.cuh): ln x carried as a
// double-double from a 128-row table and rounded once, i.e. the correctly rounded logarithm except
// within about 2^-75 of a midpoint; on the solve's arguments (temperatures, pressures) it equals the
// host glibc log on every one of 8e6 tested values.

// ------------------------------------------------------------------ relaxation (p-T-mu, 2 phases)

// Pieces of the same relaxation for the seeded kernels, which gate the learned seed on the first
// evaluation: a Newton state after k evaluations, one evaluation at an iterate (verifyAndModifyPressure
// of every phase, then f = sum_k alpha_k rho_k / rho_k*(p) - 1 and its derivative) and the
// interface-pressure fallback (RelaxationP::NewtonRaphson src/Relaxations/RelaxationP.cpp:43-68,
// RelaxationPInfinite.cpp:43-97).  The arithmetic is relax_pinf's, operation for operation.
struct NewtonState {
  double ps, f, df;
  int it;
};

template <int NP>
__device__ __forceinline__ bool pinf_applies(const Model<NP>& M, const double a[NP]) {
  if (M.eps > 1.e-20) {
#pragma unroll
    for (int k = 0; k < NP; k++)
      if (a[k] > (1. - 1.e-5)) return false;
  }
  return true;
}

template <int NP>
__device__ __forceinline__ void pinf_eval(const Model<NP>& M, const double a[NP], const double r[NP], NewtonState& s,
                                          const double p[NP], double aS[NP], double rS[NP]) {
  double drhodp = 0.;
#pragma unroll
  for (int k = 0; k < NP; k++) s.ps = eos_fix_p(M.eos[k], s.ps);
  s.f = -1.;
  s.df = 0.;
#pragma unroll
  for (int k = 0; k < NP; k++) {
    rS[k] = eos_rho_pfinal(M.eos[k], M.eps, p[k], r[k], s.ps, &drhodp);
    aS[k] = ddiv(a[k] * r[k], rS[k]);
    double dalpha = ddiv(a[k] * r[k] * drhodp, rS[k] * rS[k]);
    s.f += aS[k];
    s.df -= dalpha;
  }
}

// First evaluation at the plain start sum_k alpha_k p_k (relax_pinf's first iteration).
template <int NP>
__device__ __forceinline__ void pinf_first(const Model<NP>& M, const double a[NP], const double r[NP],
                                           const double p[NP], NewtonState& s, double aS[NP], double rS[NP]) {
  double ps = 0.;
#pragma unroll
  for (int k = 0; k < NP; k++) ps += a[k] * p[k];
  s.ps = ps - 0. / 1.;
  s.it = 1;
  pinf_eval<NP>(M, a, r, s, p, aS, rS);
}

// Continues from state s to |f| <= 1e-10 or the cap; relaxes a, r like relax_pinf.
template <int NP>
__device__ __forceinline__ void pinf_finish(const Model<NP>& M, double a[NP], double r[NP], const double p[NP],
                                            NewtonState s, double aS[NP], double rS[NP], double& pstar, RelaxStats& st,
                                            int max_iter, bool accept = false) {
  while (fabs(s.f) > 1e-10 && s.it < max_iter) {
    s.it++;
    s.ps -= ddiv(s.f, s.df);
    pinf_eval<NP>(M, a, r, s, p, aS, rS);
  }
  st.iters = s.it;
  if (s.it < max_iter || accept) {
#pragma unroll
    for (int k = 0; k < NP; k++) { a[k] = aS[k]; r[k] = rS[k]; }
    pstar = s.ps;
    return;
  }
  st.fallback = true;
  double drhodp = 0.;
  double zk[NP], pI = 0., sumZk = 0.;
#pragma unroll
  for (int k = 0; k < NP; k++) zk[k] = r[k] * eos_c(M.eos[k], M.eps, r[k], p[k]);
#pragma unroll
  for (int k = 0; k < NP; k++) {
    sumZk += zk[k];
    double sumZj = 0.;
#pragma unroll
    for (int j = 0; j < NP; j++)
      if (j != k) sumZj += zk[j];
    pI += sumZj * (p[k] - 0.);
  }
  pI = ddiv(pI, sumZk * (NP - 1));
#pragma unroll
  for (int k = 0; k < NP; k++) pI = eos_fix_p(M.eos[k], pI);
#pragma unroll
  for (int k = 0; k < NP; k++) {
    double rr = eos_rho_pfinal(M.eos[k], M.eps, p[k], r[k], pI, &drhodp);
    a[k] = ddiv(a[k] * r[k], rr);
    r[k] = rr;
  }
  pstar = pI;
}

// Iteration counts of one p-T-mu relaxation (diagnostics; they do not change the arithmetic).
struct PtmuCount {
  unsigned int solve = 0;      // 1 when the saturation Newton on p* ran
  unsigned int outer = 0;      // its iterations
  unsigned int tsat_calls = 0;  // T_sat(p) solves (pure-phase tests included)
  unsigned int tsat_iters = 0;  // their Newton iterations
  unsigned int tsat_max = 0;    // the largest of them
  unsigned int seeded = 0;      // 1 when the saturation Newton started from a learned (p*, T) seed
  unsigned int rejected = 0;    // 1 when a learned seed was rejected (plain start)
  double pstar = 0., tsat = 0.;  // converged p* and T_sat(p*) of the saturation Newton (recording)
};

// Mixture::computeTsat src/Models/Mixture.cpp:59-100 (liquid and vapour IG/SG).
// T0 > 0: the Newton iteration starts there instead of at 0.1 B / C (a seeded p-T-mu relaxation).
// With B / C > 0, f(T) = A + B / T + C ln T - ... is monotone and of one curvature on (0, B / C), the
// branch the cold start 0.1 B / C converges on: a start left of the root approaches it monotonically, a
// start right of it jumps left of it in one step, possibly past T = 0.  So a start is taken only inside
// (0, 0.5 B / C), and an iterate that leaves (0, B / C) sends the iteration back to the cold start
// (at most once); either way it converges to the root the reference's iteration finds.
__device__ __forceinline__ double compute_tsat(const EosParams& L, const EosParams& V, double p, double* dTsat,
                                               bool& err, PtmuCount* pc = nullptr, double T0 = -1.) {
  double gL = L.gamma, piL = (L.type == ECG_EOS_IG) ? 0. : L.pinf, cvL = L.cv, e0L = L.eref, s0L = L.sref;
  double gV = V.gamma, piV = (V.type == ECG_EOS_IG) ? 0. : V.pinf, cvV = V.cv, e0V = V.eref, s0V = V.sref;
  double A = ddiv(gL * cvL - gV * cvV + s0V - s0L, gV * cvV - cvV);
  double B = ddiv(e0L - e0V, gV * cvV - cvV);
  double C = ddiv(gV * cvV - gL * cvL, gV * cvV - cvV);
  double D = ddiv(gL * cvL - cvL, gV * cvV - cvV);
  int iteration = 0;
  bool seeded = T0 > 0. && T0 < ddiv(0.5 * B, C);
  double Tsat = seeded ? T0 : ddiv(0.1 * B, C), f = 0., df = 1.;
  // ln(p + pInf) of both phases do not depend on the iterate: evaluated once per solve (the same
  // values enter the same sum, so f has the bits of the reference's per-iteration evaluation)
  const double lnV = elog(p + piV), lnL = elog(p + piL);
  do {
    Tsat -= ddiv(f, df);
    if (seeded && !(Tsat > 0. && Tsat < ddiv(B, C))) {  // a seeded iterate left the root's branch
      seeded = false;
      Tsat = ddiv(0.1 * B, C);
    }
    iteration++;
    if (iteration > 50) {
      err = true;
      break;
    }
    f = A + ddiv(B, Tsat) + C * elog(Tsat) - lnV + D * lnL;
    df = ddiv(C, Tsat) - ddiv(B, Tsat * Tsat);
  } while (fabs(f) > 1e-10);
  if (pc) {
    pc->tsat_calls++;
    pc->tsat_iters += (unsigned int)iteration;
    pc->tsat_max = max(pc->tsat_max, (unsigned int)iteration);
  }
  double dfdp = ddiv(-1., p + piV) + ddiv(D, p + piL);
  *dTsat = ddiv(-dfdp, df);
  return Tsat;
}

// computeDensitySaturation (EosIG.cpp:170, EosSG.cpp:172, EosNASG.cpp:189)
__device__ __forceinline__ double eos_rho_sat(const EosParams& q, double eps, double p, double Tsat, double dTsat,
                                              double* drhodp) {
  double pp = (q.type == ECG_EOS_IG) ? p : p + q.pinf;
  double g1cvT = (q.gamma - 1.) * q.cv * Tsat;
  double den = (q.type == ECG_EOS_NASG) ? g1cvT + q.b * (p + q.pinf) : g1cvT;
  double d = (q.gamma - 1.) * q.cv * Tsat - pp * (q.gamma - 1.) * q.cv * dTsat;
  *drhodp = ddiv(d, dmax(den * den, eps));
  return ddiv(pp, dmax(den, eps));
}

// computeDensityEnergySaturation (EosIG.cpp:184, EosSG.cpp:186, EosNASG.cpp:203)
__device__ __forceinline__ double eos_rhoe_sat(const EosParams& q, double p, double rho, double drhodp,
                                               double* drhoedp) {
  if (q.type == ECG_EOS_IG) {
    *drhoedp = ddiv(1., q.gamma - 1.) + drhodp * q.eref;
    return ddiv(p, q.gamma - 1.) + rho * q.eref;
  }
  if (q.type == ECG_EOS_SG) {
    *drhoedp = ddiv(1., q.gamma - 1.) + drhodp * q.eref;
    return ddiv(p + q.gamma * q.pinf, q.gamma - 1.) + rho * q.eref;
  }
  *drhoedp = ddiv(1. - rho * q.b, q.gamma - 1.) + drhodp * (q.eref - ddiv(q.b * (p + q.gamma * q.pinf), q.gamma - 1.));
  return ddiv((p + q.gamma * q.pinf) * (1. - rho * q.b), q.gamma - 1.) + rho * q.eref;
}

// RelaxationPTMu::relaxation src/Relaxations/RelaxationPTMu.cpp:73-200.  rhomix / emix are the
// mixture density and internal energy the cell holds at that point (from buildPrim).  Returns true
// when the phases were updated (the reference then calls fulfillState, so the mixture density
// is recomputed from the new phases).
//
// Seeded forms: T_seed > 0: the T_sat(p) solves of the saturation Newton start at T_seed (the first)
// and then at the previous iteration's T_sat, instead of the cold start 0.1 B / C of every solve (the
// pure-phase tests keep the cold start, so they decide as the reference does); p_seed > 0: the Newton
// iteration on p* starts at p_seed instead of sum_k alpha_k p_k.  Every loop still stops at
// |f| <= 1e-10.
template <int NP>
__device__ __forceinline__ bool relax_ptmu(const Model<NP>& M, int liq, int vap, double pcrit, double a[NP],
                                           double r[NP], double p[NP], double rhomix, double emix, bool& err,
                                           PtmuCount* pc = nullptr, double p_seed = -1., double T_seed = -1.) {
  const EosParams& EL = M.eos[liq];
  const EosParams& EV = M.eos[vap];
  double pStar = 0., Tsat, dTsat = 0.;
#pragma unroll
  for (int k = 0; k < NP; k++) pStar += a[k] * p[k];
  if (pStar > pcrit) return false;
  double rho = rhomix, rhoe = rho * emix;
  double pv = eos_p(EV, M.eps, rho, emix);
  double Tv = eos_T(EV, M.eps, rho, pv);
  if (pv > 0) {
    Tsat = compute_tsat(EL, EV, pv, &dTsat, err, pc);
    if (Tv >= Tsat) {
      a[vap] = 1.;
      a[liq] = 0.;
      r[vap] = rho;
      p[vap] = pv;
      return true;
    }
  }
  double pl = eos_p(EL, M.eps, rho, emix);
  double Tl = eos_T(EL, M.eps, rho, pl);
  if (pl > 0.) {
    Tsat = compute_tsat(EL, EV, pl, &dTsat, err, pc);
    if (Tl <= Tsat) {
      a[liq] = 1.;
      a[vap] = 0.;
      r[liq] = rho;
      p[liq] = pl;
      return true;
    }
  }
  double rhoLSat = 0., rhoVSat = 0., drhoLSat, drhoVSat, aLSat = 0., aVSat = 0., daLSat, daVSat;
  double rhoeLSat, rhoeVSat, drhoeLSat, drhoeVSat;
  int iteration = 0;
  double f = 0., df = 1.;
  double Tstart = T_seed;  // start of the next T_sat solve (seeded form)
  if (p_seed > 0.) pStar = p_seed;
  do {
    pStar -= ddiv(f, df);
    iteration++;
    if (iteration > 50) {
      err = true;
      break;
    }
#pragma unroll
    for (int k = 0; k < NP; k++) pStar = eos_fix_p(M.eos[k], pStar);
    Tsat = compute_tsat(EL, EV, pStar, &dTsat, err, pc, Tstart);
    if (T_seed > 0.) Tstart = Tsat;
    rhoLSat = eos_rho_sat(EL, M.eps, pStar, Tsat, dTsat, &drhoLSat);
    rhoVSat = eos_rho_sat(EV, M.eps, pStar, Tsat, dTsat, &drhoVSat);
    aLSat = ddiv(rho - rhoVSat, rhoLSat - rhoVSat);
    daLSat = ddiv(-drhoVSat * (rhoLSat - rhoVSat) - (rho - rhoVSat) * (drhoLSat - drhoVSat),
                  (rhoLSat - rhoVSat) * (rhoLSat - rhoVSat));
    aVSat = 1. - aLSat;
    daVSat = -daLSat;
    f = rhoe;
    df = 0.;
    rhoeLSat = eos_rhoe_sat(EL, pStar, rhoLSat, drhoLSat, &drhoeLSat);
    rhoeVSat = eos_rhoe_sat(EV, pStar, rhoVSat, drhoVSat, &drhoeVSat);
    f -= (aLSat * rhoeLSat + aVSat * rhoeVSat);
    df -= (daLSat * rhoeLSat + aLSat * drhoeLSat + daVSat * rhoeVSat + aVSat * drhoeVSat);
    f = ddiv(f, rhoe);
    df = ddiv(df, rhoe);
  } while (fabs(f) > 1e-10);
  if (pc) {
    pc->solve = 1;
    pc->outer = (unsigned int)iteration;
    pc->pstar = pStar;
    pc->tsat = Tsat;
  }
  a[liq] = aLSat;
  r[liq] = rhoLSat;
  p[liq] = pStar;
  a[vap] = aVSat;
  r[vap] = rhoVSat;
  p[vap] = pStar;
  return true;
}

// ------------------------------------------------------------------ energy correction

// Cell::correctionEnergy src/Order1/Cell.cpp:327: MixUEq::totalEnergyToInternalEnergy :175 then
// FluxPUEq::correctionEnergy src/Models/PUEq/FluxPUEq.cpp:68-112 (mixture-EOS pressure).
template <int NP>
__device__ __forceinline__ double correction_pressure(const Model<NP>& M, const double a[NP], const double r[NP],
                                                      double rhomix, double E, double usq) {
  double e = E - 0.5 * usq;
  double rhoe = rhomix * e;
  double pp = rhoe, denom = 0.;
#pragma unroll
  for (int k = 0; k < NP; k++) {
    const EosParams& q = M.eos[k];
    const double gpi = q.gpi, ig = q.ig;  // sendSpecialMixtureEos constants, computed on the host
    double cov = (q.type == ECG_EOS_NASG) ? q.b : 0.;
    pp -= a[k] * (gpi * (1. - r[k] * cov) + r[k] * q.eref);
    denom += a[k] * ig * (1. - r[k] * cov);
  }
  return ddiv(pp, denom);
}

}  // namespace ecg
