/*
 * CPU restatement of ECOGEN's Cartesian explicit FV step — TEST INFRASTRUCTURE.
 *
 * The oracle the CUDA kernels are checked against.  It keeps the reference's
 * data model (one phase record per phase and one mixture record per cell, a
 * second set for the MUSCL predictor, one flux accumulator per cell) and walks
 * faces in the reference's order, so that each floating-point operation
 * happens in the same order and with the same rounding as in the reference
 * build (compile with -ffp-contract=off, see oracle/Makefile).  Every function
 * names the reference file:line it restates (paths relative to the ECOGEN tree).
 */
#include "ecg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ln of the saturation solve: the host libm's, as the reference (the default build), or a correctly
 * rounded one (the sensitivity variant libecg_oracle_crlog.so, -DECGO_CR_LOG; see ecg_crlog.h). */
#ifdef ECGO_CR_LOG
#include "ecg_crlog.h"
#define ECGO_LOG ecgo_cr_log
#else
#define ECGO_LOG log
#endif
/* pow of the isentropic star pressure: the host libm's (the default build), or with last-ulp changes in
 * 1 call in 100 (the sensitivity variant libecg_oracle_powulp.so, -DECGO_POW_ULP; see ecg_powulp.h). */
#ifdef ECGO_POW_ULP
#include "ecg_powulp.h"
#define ECGO_POW ecgo_pow_ulp
#else
#define ECGO_POW pow
#endif

#define NP_MAX 3
#define NT_MAX 4   /* passive transports (model.xml numberTransports) */

/* std::max / std::min exactly as libstdc++ defines them (NaN handling included) */
static inline double omax(double a, double b) { return (a < b) ? b : a; }
static inline double omin(double a, double b) { return (b < a) ? b : a; }

/* --------------------------------------------------------------------------------------------- data */

typedef struct {
  double alpha, rho, p, Y, T, e, c;  /* PhaseUEq (src/Models/UEq/PhaseUEq.h) */
  double u[3], E;                    /* PhaseEuler velocity and total energy (src/Models/Euler/PhaseEuler.h) */
} OPh;

typedef struct {
  double rho, p, u[3], e, E, cF, cW; /* MixUEq (src/Models/UEq/MixUEq.h) */
  double T;                          /* MixPTUEq temperature (src/Models/PTUEq/MixPTUEq.h) */
} OMix;

typedef struct {
  OPh ph[NP_MAX];
  OMix m;
  double tr[NT_MAX];  /* Transport values (src/Transport/Transport.h) */
} OSt;

typedef struct {
  double alpha[NP_MAX], mass[NP_MAX], energ[NP_MAX], mom[3], energMix; /* FluxUEq / FluxEuler */
  double tr[NT_MAX];  /* transport fluxes / accumulated m_consTransports */
  double sM, uStar;
} OFlux;

typedef struct {
  double alpha[NP_MAX], rho[NP_MAX], p[NP_MAX];
  double u[3];
  double pm, Tm;      /* MixPTUEq pressure and temperature slopes */
  double tr[NT_MAX];
} OSlope; /* PhaseUEq/PhaseEuler/PhasePTUEq slopes + MixUEq/MixPTUEq slopes */

typedef struct {
  int L, R;           /* R < 0 for a boundary face */
  int axis;           /* 0,1,2 */
  int bc;             /* -1 internal face, else ECGO_BC_* of its side */
  double n[3], t[3], b[3];
  double surface;
  double pos[3];
} OFace;

struct ecgo_sim {
  ecgo_case c;
  double eps;         /* epsilonAlphaNull (src/Eos/Eos.cpp:88-97) */
  int np, dim, n;
  OSt* s;             /* vecPhases */
  OSt* s2;            /* vecPhasesO2 */
  OFlux* cons;        /* m_cons */
  OFlux* save;        /* m_consSauvegarde */
  double* pos;        /* 3 per cell */
  double* vol;
  double* lcfl;
  OFace* faces;
  int nfaces, ninner;
  int* cellface;      /* per cell, per axis, [minus, plus] face index (-1 none) : 6 ints */
  OSlope* slopes;     /* per face */
  double pcrit;
  int thinc;          /* a volume-fraction limiter is THINC */
  ecgo_stats st;
};

/* ------------------------------------------------------------------------------------------ EOS */
/* src/Eos/EosIG.cpp:64-257, src/Eos/EosSG.cpp:66-257, src/Eos/EosNASG.cpp:68-280 */

static double eos_T(const ecgo_eos* q, double eps, double rho, double p) {
  switch (q->type) {
    case ECGO_EOS_IG: return p / (q->gamma - 1.) / omax(rho, eps) / q->cv;
    case ECGO_EOS_SG: return (p + q->pinf) / (q->gamma - 1.) / omax(rho, eps) / q->cv;
    default: return (p + q->pinf) * omax(1. - rho * q->b, eps) / (q->gamma - 1.) / q->cv / omax(rho, eps);
  }
}

static double eos_e(const ecgo_eos* q, double eps, double rho, double p) {
  switch (q->type) {
    case ECGO_EOS_IG: return p / (q->gamma - 1.) / omax(rho, eps) + q->eref;
    case ECGO_EOS_SG: return (p + q->gamma * q->pinf) / (q->gamma - 1.) / omax(rho, eps) + q->eref;
    default:
      return (p + q->gamma * q->pinf) * omax(1. - rho * q->b, eps) / (q->gamma - 1.) / omax(rho, eps) + q->eref;
  }
}

static double eos_p(const ecgo_eos* q, double eps, double rho, double e) {
  switch (q->type) {
    case ECGO_EOS_IG: return (q->gamma - 1.) * rho * (e - q->eref);
    case ECGO_EOS_SG: return (q->gamma - 1.) * rho * (e - q->eref) - q->gamma * q->pinf;
    default: return (rho * (q->gamma - 1.) * (e - q->eref) / omax(1. - rho * q->b, eps) - q->gamma * q->pinf);
  }
}

static double eos_c(const ecgo_eos* q, double eps, double rho, double p) {
  switch (q->type) {
    case ECGO_EOS_IG: return sqrt(q->gamma * p / omax(rho, eps));
    case ECGO_EOS_SG: return sqrt(q->gamma * (p + q->pinf) / omax(rho, eps));
    default: return sqrt(q->gamma * (p + q->pinf) / omax(rho * (1. - rho * q->b), eps));
  }
}

static double nonzero(double a, double eps) { /* Tools::returnNonZeroValue, src/Tools.cpp:134 */
  if (a > eps || a < -eps) return a;
  int sg = (0. < a) - (a < 0.);
  return sg * eps;
}

static double eos_p_isentropic(const ecgo_eos* q, double eps, double p0, double rho0, double rho1) {
  switch (q->type) {
    case ECGO_EOS_IG: return p0 * ECGO_POW(rho1 / omax(rho0, eps), q->gamma);
    case ECGO_EOS_SG: return (p0 + q->pinf) * ECGO_POW(rho1 / omax(rho0, eps), q->gamma) - q->pinf;
    default:
      return (p0 + q->pinf) * ECGO_POW(rho1 / omax(rho0, eps), q->gamma) *
                 ECGO_POW((1. - rho0 * q->b) / (1. - rho1 * q->b), q->gamma) - q->pinf;
  }
}

static double eos_rho_pfinal(const ecgo_eos* q, double eps, double p0, double rho0, double p1, double* drhodp) {
  double num, denom, rho1;
  switch (q->type) {
    case ECGO_EOS_IG:
      num = q->gamma * p1;
      denom = num + p0 - p1;
      rho1 = rho0 * num / omax(denom, eps);
      if (drhodp) *drhodp = rho0 * q->gamma * p0 / omax(denom * denom, eps);
      return rho1;
    case ECGO_EOS_SG:
      num = q->gamma * (p1 + q->pinf);
      denom = num + p0 - p1;
      rho1 = rho0 * num / nonzero(denom, eps);
      if (drhodp) *drhodp = rho0 * q->gamma * (p0 + q->pinf) / omax(denom * denom, eps);
      return rho1;
    default:
      num = q->gamma * (p1 + q->pinf);
      denom = num + p0 - p1 + q->b * rho0 * (p1 - p0);
      rho1 = rho0 * num / nonzero(denom, eps);
      if (drhodp) *drhodp = rho0 * q->gamma * (p0 + q->pinf - q->b * rho0 * (p0 + q->pinf)) / nonzero(denom * denom, eps);
      return rho1;
  }
}

static void eos_fix_p(const ecgo_eos* q, double* p) { /* verifyAndModifyPressure */
  if (q->type == ECGO_EOS_IG) {
    if (*p < 1.e-8) *p = 1.e-8;
  } else {
    if (*p <= -(1. - 1.e-15) * q->pinf + 1.e-15) *p = -(1. - 1.e-15) * q->pinf + 1.e-15;
  }
}

static void eos_rho_max(const ecgo_eos* q, double* rho) { /* verifyAndCorrectDensityMax(density) */
  if (q->type == ECGO_EOS_NASG && *rho > 1. / q->b - 1.) *rho = 1. / q->b - 1.;
}

static void eos_rho_max_mass(const ecgo_eos* q, double mass, double* alpha, double* rho) {
  if (q->type == ECGO_EOS_NASG && *rho > 1. / q->b - 1.) {
    *rho = 1. / q->b - 1.;
    *alpha = mass / *rho;
  }
}

static void eos_mix(const ecgo_eos* q, double* gpi, double* eref, double* ig, double* cov) { /* sendSpecialMixtureEos */
  *gpi = (q->type == ECGO_EOS_IG) ? 0. : q->gamma * q->pinf / (q->gamma - 1.);
  *eref = q->eref;
  *ig = 1. / (q->gamma - 1.);
  *cov = (q->type == ECGO_EOS_NASG) ? q->b : 0.;
}

static double eos_rho_sat(const ecgo_eos* q, double eps, double p, double Tsat, double dTsat, double* drhodp) {
  /* computeDensitySaturation: EosIG.cpp:170, EosSG.cpp:172, EosNASG.cpp:189 */
  double pp = (q->type == ECGO_EOS_IG) ? p : p + q->pinf;
  double g1cvT = (q->gamma - 1.) * q->cv * Tsat;
  double den = (q->type == ECGO_EOS_NASG) ? g1cvT + q->b * (p + q->pinf) : g1cvT;
  if (drhodp) {
    *drhodp = (q->gamma - 1.) * q->cv * Tsat - pp * (q->gamma - 1.) * q->cv * dTsat;
    *drhodp /= omax(den * den, eps);
  }
  return pp / omax(den, eps);
}

static double eos_rhoe_sat(const ecgo_eos* q, double p, double rho, double drhodp, double* drhoedp) {
  if (q->type == ECGO_EOS_IG) {
    if (drhoedp) *drhoedp = 1. / (q->gamma - 1.) + drhodp * q->eref;
    return p / (q->gamma - 1.) + rho * q->eref;
  }
  if (q->type == ECGO_EOS_SG) {
    if (drhoedp) *drhoedp = 1. / (q->gamma - 1.) + drhodp * q->eref;
    return (p + q->gamma * q->pinf) / (q->gamma - 1.) + rho * q->eref;
  }
  if (drhoedp)
    *drhoedp = (1. - rho * q->b) / (q->gamma - 1.) +
               drhodp * (q->eref - q->b * (p + q->gamma * q->pinf) / (q->gamma - 1.));
  return (p + q->gamma * q->pinf) * (1. - rho * q->b) / (q->gamma - 1.) + rho * q->eref;
}

/* ----------------------------------------------------------------------------------- phase / mixture */

static void phase_extended(const ecgo_sim* S, int k, OPh* ph) { /* PhaseUEq::extendedCalculusPhase :97 */
  const ecgo_eos* q = &S->c.eos[k];
  ph->T = eos_T(q, S->eps, ph->rho, ph->p);
  ph->e = eos_e(q, S->eps, ph->rho, ph->p);
  ph->c = eos_c(q, S->eps, ph->rho, ph->p);
}

static void phase_fix(const ecgo_sim* S, int k, OPh* ph) { /* PhaseUEq::verifyAndCorrectPhase :348 */
  if (S->eps > 1.e-20) {
    if (ph->alpha < 0.) ph->alpha = 0.;
    if (ph->alpha > 1.) ph->alpha = 1.;
    if (ph->rho <= 1.e-15) ph->rho = 1.e-15;
  } else {
    if (ph->alpha < 1e-15) ph->alpha = 1e-14;
    if (ph->alpha > 1. - 1e-15) ph->alpha = 1. - 1e-14;
    if (ph->rho < 1.e-15) ph->rho = 1.e-14;
  }
  eos_fix_p(&S->c.eos[k], &ph->p);
}

static void mixture_vars(const ecgo_sim* S, OSt* st) { /* MixUEq::computeMixtureVariables src/Models/UEq/MixUEq.cpp:136 */
  int np = S->np;
  st->m.rho = 0.;
  st->m.p = 0.;
  for (int k = 0; k < np; k++) {
    st->m.rho += st->ph[k].alpha * st->ph[k].rho;
    st->m.p += st->ph[k].alpha * st->ph[k].p;
  }
  for (int k = 0; k < np; k++) st->ph[k].Y = st->ph[k].alpha * st->ph[k].rho / omax(st->m.rho, S->eps);
  st->m.e = 0.;
  st->m.cF = 0.;
  st->m.cW = 0.;
  for (int k = 0; k < np; k++) {
    OPh* ph = &st->ph[k];
    st->m.e += ph->Y * ph->e;
    st->m.cF += ph->Y * ph->c * ph->c;
    st->m.cW += ph->alpha / omax((ph->rho * ph->c * ph->c), S->eps);
  }
  st->m.cF = sqrt(st->m.cF);
  st->m.cW = 1. / sqrt(st->m.rho * st->m.cW);
}

static void euler_extended(const ecgo_sim* S, OPh* ph) { /* PhaseEuler::extendedCalculusPhase :105 */
  const ecgo_eos* q = &S->c.eos[0];
  ph->e = eos_e(q, S->eps, ph->rho, ph->p);
  ph->c = eos_c(q, S->eps, ph->rho, ph->p);
  ph->E = ph->e + 0.5 * (ph->u[0] * ph->u[0] + ph->u[1] * ph->u[1] + ph->u[2] * ph->u[2]);
  ph->T = eos_T(q, S->eps, ph->rho, ph->p);
}

/* ---- temperature-pressure-velocity equilibrium model (PTUEq, src/Models/PTUEq) ---- */

static double eos_pinf(const ecgo_eos* q) { /* Eos::getPInf: 0 for IG (Errors::defaultDouble) */
  return (q->type == ECGO_EOS_IG) ? 0. : q->pinf;
}

static double eos_rho_pT(const ecgo_eos* q, double eps, double p, double T) {
  /* computeDensity(p, T): EosIG.cpp:85, EosSG.cpp:87 */
  if (q->type == ECGO_EOS_IG) return p / omax(((q->gamma - 1.) * q->cv * T), eps);
  return (p + q->pinf) / omax(((q->gamma - 1.) * q->cv * T), eps);
}

static void ptueq_mixture_vars(const ecgo_sim* S, OSt* st) {
  /* MixPTUEq::computeMixtureVariables src/Models/PTUEq/MixPTUEq.cpp:293-313 (mass fractions without a floor) */
  st->m.rho = 0.;
  for (int k = 0; k < S->np; k++) st->m.rho += st->ph[k].alpha * st->ph[k].rho;
  for (int k = 0; k < S->np; k++) st->ph[k].Y = st->ph[k].alpha * st->ph[k].rho / st->m.rho;
  st->m.e = 0.;
  st->m.cF = 0.;
  for (int k = 0; k < S->np; k++) {
    st->m.e += st->ph[k].Y * st->ph[k].e;
    st->m.cF += st->ph[k].Y * st->ph[k].c * st->ph[k].c;
  }
  st->m.cF = sqrt(st->m.cF);
}

static void ptueq_phase(const ecgo_sim* S, int k, OPh* ph, double p, double T) {
  /* ModPTUEq::fulfillState src/Models/PTUEq/ModPTUEq.cpp:99-108 for one phase:
   * p_k = p, rho_k = computeDensity(p, T), then PhasePTUEq::extendedCalculusPhase (e_k, c_k) */
  const ecgo_eos* q = &S->c.eos[k];
  ph->p = p;
  ph->rho = eos_rho_pT(q, S->eps, p, T);
  ph->T = T;
  ph->e = eos_e(q, S->eps, ph->rho, ph->p);
  ph->c = eos_c(q, S->eps, ph->rho, ph->p);
}

static void ptueq_fulfill(const ecgo_sim* S, OSt* st) {
  for (int k = 0; k < S->np; k++) ptueq_phase(S, k, &st->ph[k], st->m.p, st->m.T);
  ptueq_mixture_vars(S, st);
}

static void fulfill(const ecgo_sim* S, OSt* st) { /* ModUEq::fulfillState :99 ; ModEuler::fulfillState :95 */
  if (S->c.model == ECGO_MODEL_EULER) {
    euler_extended(S, &st->ph[0]);
    return;
  }
  if (S->c.model == ECGO_MODEL_PTUEQ) {
    ptueq_fulfill(S, st);
    return;
  }
  for (int k = 0; k < S->np; k++) phase_extended(S, k, &st->ph[k]);
  mixture_vars(S, st);
}

static double sqnorm(const double* u) { return u[0] * u[0] + u[1] * u[1] + u[2] * u[2]; }

/* ------------------------------------------------------------------------------------ projections */
/* src/Maths/Coord.cpp:133-151 */
static void proj_local(double* v, const double* n, const double* t, const double* b) {
  double x = v[0] * n[0] + v[1] * n[1] + v[2] * n[2];
  double y = v[0] * t[0] + v[1] * t[1] + v[2] * t[2];
  double z = v[0] * b[0] + v[1] * b[1] + v[2] * b[2];
  v[0] = x; v[1] = y; v[2] = z;
}
static void proj_reverse(double* v, const double* n, const double* t, const double* b) {
  double x = n[0] * v[0] + t[0] * v[1] + b[0] * v[2];
  double y = n[1] * v[0] + t[1] * v[1] + b[1] * v[2];
  double z = n[2] * v[0] + t[2] * v[1] + b[2] * v[2];
  v[0] = x; v[1] = y; v[2] = z;
}
static double* vel_of(const ecgo_sim* S, OSt* st) {
  return (S->c.model == ECGO_MODEL_EULER) ? st->ph[0].u : st->m.u;
}

/* ------------------------------------------------------------------------------------------ HLLC */

static void hllc_ueq(const ecgo_sim* S, const OSt* L, const OSt* R, double dxL, double dxR, double* dtMax, OFlux* F) {
  /* ModUEq::solveRiemannIntern src/Models/UEq/ModUEq.cpp:113-267 (inherited by ModPUEq) */
  int np = S->np;
  double sL, sR, pStar = 0., rhoStar = 0., EStar = 0.;
  double uL = L->m.u[0], cL = L->m.cF, pL = L->m.p, rhoL = L->m.rho;
  double uR = R->m.u[0], cR = R->m.cF, pR = R->m.p, rhoR = R->m.rho;
  double machRefMin = 1.;
  sL = omin(uL - cL, uR - cR);
  sR = omax(uR + cR, uL + cL);
  if (fabs(sL) > 1.e-3) *dtMax = omin(*dtMax, machRefMin * dxL / fabs(sL));
  if (fabs(sR) > 1.e-3) *dtMax = omin(*dtMax, machRefMin * dxR / fabs(sR));
  double mL = rhoL * (sL - uL), mR = rhoR * (sR - uR), mkL, mkR;
  double sM = (pR - pL + mL * uL - mR * uR) / (mL - mR);
  if (fabs(sM) < 1.e-8) sM = 0.;

  if (sL >= 0.) {
    for (int k = 0; k < np; k++) {
      const OPh* ph = &L->ph[k];
      F->alpha[k] = ph->alpha * sM;
      F->mass[k] = ph->alpha * ph->rho * uL;
      F->energ[k] = ph->alpha * ph->rho * ph->e * uL;
    }
    double vY = L->m.u[1], vZ = L->m.u[2];
    double Et = L->m.e + 0.5 * sqnorm(L->m.u);
    F->mom[0] = rhoL * uL * uL + pL;
    F->mom[1] = rhoL * vY * uL;
    F->mom[2] = rhoL * vZ * uL;
    F->energMix = (rhoL * Et + pL) * uL;
    F->uStar = uL;
  } else if (sR <= 0.) {
    for (int k = 0; k < np; k++) {
      const OPh* ph = &R->ph[k];
      F->alpha[k] = ph->alpha * sM;
      F->mass[k] = ph->alpha * ph->rho * uR;
      F->energ[k] = ph->alpha * ph->rho * ph->e * uR;
    }
    double vY = R->m.u[1], vZ = R->m.u[2];
    double Et = R->m.e + 0.5 * sqnorm(R->m.u);
    F->mom[0] = rhoR * uR * uR + pR;
    F->mom[1] = rhoR * vY * uR;
    F->mom[2] = rhoR * vZ * uR;
    F->energMix = (rhoR * Et + pR) * uR;
    F->uStar = uR;
  } else if (sM >= 0.) {
    double vY = L->m.u[1], vZ = L->m.u[2];
    double Et = L->m.e + 0.5 * sqnorm(L->m.u);
    rhoStar = mL / (sL - sM);
    EStar = Et + (sM - uL) * (sM + pL / mL);
    pStar = mL * (sM - uL) + pL;
    for (int k = 0; k < np; k++) {
      const OPh* ph = &L->ph[k];
      const ecgo_eos* q = &S->c.eos[k];
      mkL = ph->rho * (sL - uL);
      double rks = mkL / (sL - sM);
      eos_rho_max(q, &rks);
      double pks = eos_p_isentropic(q, S->eps, ph->p, ph->rho, rks);
      double eks = eos_e(q, S->eps, rks, pks);
      F->alpha[k] = ph->alpha * sM;
      F->mass[k] = ph->alpha * rks * sM;
      F->energ[k] = ph->alpha * rks * eks * sM;
    }
    F->mom[0] = rhoStar * sM * sM + pStar;
    F->mom[1] = rhoStar * vY * sM;
    F->mom[2] = rhoStar * vZ * sM;
    F->energMix = (rhoStar * EStar + pStar) * sM;
    F->uStar = sM;
  } else {
    double vY = R->m.u[1], vZ = R->m.u[2];
    double Et = R->m.e + 0.5 * sqnorm(R->m.u);
    rhoStar = mR / (sR - sM);
    EStar = Et + (sM - uR) * (sM + pR / mR);
    pStar = mR * (sM - uR) + pR;
    for (int k = 0; k < np; k++) {
      const OPh* ph = &R->ph[k];
      const ecgo_eos* q = &S->c.eos[k];
      mkR = ph->rho * (sR - uR);
      double rks = mkR / (sR - sM);
      eos_rho_max(q, &rks);
      double pks = eos_p_isentropic(q, S->eps, ph->p, ph->rho, rks);
      double eks = eos_e(q, S->eps, rks, pks);
      F->alpha[k] = ph->alpha * sM;
      F->mass[k] = ph->alpha * rks * sM;
      F->energ[k] = ph->alpha * rks * eks * sM;
    }
    F->mom[0] = rhoStar * sM * sM + pStar;
    F->mom[1] = rhoStar * vY * sM;
    F->mom[2] = rhoStar * vZ * sM;
    F->energMix = (rhoStar * EStar + pStar) * sM;
    F->uStar = sM;
  }
  F->sM = sM;
}

static void hllc_euler(const ecgo_sim* S, const OSt* Ls, const OSt* Rs, double dxL, double dxR, double* dtMax,
                       OFlux* F) {
  /* ModEuler::solveRiemannIntern src/Models/Euler/ModEuler.cpp:105-225 */
  (void)S;
  const OPh* L = &Ls->ph[0];
  const OPh* R = &Rs->ph[0];
  double uL = L->u[0], vL = L->u[1], wL = L->u[2], pL = L->p, rhoL = L->rho, cL = L->c, EL = L->E;
  double uR = R->u[0], vR = R->u[1], wR = R->u[2], pR = R->p, rhoR = R->rho, cR = R->c, ER = R->E;
  double machRefMin = 1.;
  double sL = omin(uL - cL, uR - cR);
  double sR = omax(uR + cR, uL + cL);
  if (fabs(sL) > 1.e-3) *dtMax = omin(*dtMax, machRefMin * dxL / fabs(sL));
  if (fabs(sR) > 1.e-3) *dtMax = omin(*dtMax, machRefMin * dxR / fabs(sR));
  double mL = rhoL * (sL - uL), mR = rhoR * (sR - uR);
  double sM = (pR - pL + mL * uL - mR * uR) / (mL - mR);
  if (fabs(sM) < 1.e-8) sM = 0.;
  if (sL > 0.) {
    F->mass[0] = rhoL * uL;
    F->mom[0] = rhoL * uL * uL + pL;
    F->mom[1] = rhoL * vL * uL;
    F->mom[2] = rhoL * wL * uL;
    F->energMix = (rhoL * EL + pL) * uL;
  } else if (sR < 0.) {
    F->mass[0] = rhoR * uR;
    F->mom[0] = rhoR * uR * uR + pR;
    F->mom[1] = rhoR * vR * uR;
    F->mom[2] = rhoR * wR * uR;
    F->energMix = (rhoR * ER + pR) * uR;
  } else if (sM >= 0.) {
    double pStar = mL * (sM - uL) + pL;
    double rhoStar = mL / (sL - sM);
    double Estar = EL + (sM - uL) * (sM + pL / mL);
    F->mass[0] = rhoStar * sM;
    F->mom[0] = rhoStar * sM * sM + pStar;
    F->mom[1] = rhoStar * sM * vL;
    F->mom[2] = rhoStar * sM * wL;
    F->energMix = (rhoStar * Estar + pStar) * sM;
  } else {
    double pStar = mR * (sM - uR) + pR;
    double rhoStar = mR / (sR - sM);
    double Estar = ER + (sM - uR) * (sM + pR / mR);
    F->mass[0] = rhoStar * sM;
    F->mom[0] = rhoStar * sM * sM + pStar;
    F->mom[1] = rhoStar * sM * vR;
    F->mom[2] = rhoStar * sM * wR;
    F->energMix = (rhoStar * Estar + pStar) * sM;
  }
  F->sM = sM;
  F->uStar = 0.;
}

static void hllc_ptueq(const ecgo_sim* S, const OSt* L, const OSt* R, double dxL, double dxR, double* dtMax,
                       OFlux* F) {
  /* ModPTUEq::solveRiemannIntern src/Models/PTUEq/ModPTUEq.cpp:113-227: mixture HLLC, phase masses
   * carried by the mass fractions of the upwind side */
  int np = S->np;
  double uL = L->m.u[0], cL = L->m.cF, pL = L->m.p, rhoL = L->m.rho;
  double uR = R->m.u[0], cR = R->m.cF, pR = R->m.p, rhoR = R->m.rho;
  double sL = omin(uL - cL, uR - cR);
  double sR = omax(uR + cR, uL + cL);
  if (fabs(sL) > 1.e-3) *dtMax = omin(*dtMax, dxL / fabs(sL));
  if (fabs(sR) > 1.e-3) *dtMax = omin(*dtMax, dxR / fabs(sR));
  double mL = rhoL * (sL - uL), mR = rhoR * (sR - uR);
  double sM = (pR - pL + mL * uL - mR * uR) / (mL - mR);
  if (fabs(sM) < 1.e-8) sM = 0.;
  if (sL >= 0.) {
    for (int k = 0; k < np; k++) F->mass[k] = L->ph[k].alpha * L->ph[k].rho * uL;
    double vY = L->m.u[1], vZ = L->m.u[2];
    double Et = L->m.e + 0.5 * sqnorm(L->m.u);
    F->mom[0] = rhoL * uL * uL + pL;
    F->mom[1] = rhoL * vY * uL;
    F->mom[2] = rhoL * vZ * uL;
    F->energMix = (rhoL * Et + pL) * uL;
  } else if (sR <= 0.) {
    for (int k = 0; k < np; k++) F->mass[k] = R->ph[k].alpha * R->ph[k].rho * uR;
    double vY = R->m.u[1], vZ = R->m.u[2];
    double Et = R->m.e + 0.5 * sqnorm(R->m.u);
    F->mom[0] = rhoR * uR * uR + pR;
    F->mom[1] = rhoR * vY * uR;
    F->mom[2] = rhoR * vZ * uR;
    F->energMix = (rhoR * Et + pR) * uR;
  } else if (sM >= 0.) {
    double vY = L->m.u[1], vZ = L->m.u[2];
    double Et = L->m.e + 0.5 * sqnorm(L->m.u);
    double rhoStar = mL / (sL - sM);
    double EStar = Et + (sM - uL) * (sM + pL / mL);
    double pStar = mL * (sM - uL) + pL;
    for (int k = 0; k < np; k++) {
      double mkL = L->ph[k].alpha * L->ph[k].rho * (sL - uL);
      F->mass[k] = mkL / (sL - sM) * sM;
    }
    F->mom[0] = rhoStar * sM * sM + pStar;
    F->mom[1] = rhoStar * vY * sM;
    F->mom[2] = rhoStar * vZ * sM;
    F->energMix = (rhoStar * EStar + pStar) * sM;
  } else {
    double vY = R->m.u[1], vZ = R->m.u[2];
    double Et = R->m.e + 0.5 * sqnorm(R->m.u);
    double rhoStar = mR / (sR - sM);
    double EStar = Et + (sM - uR) * (sM + pR / mR);
    double pStar = mR * (sM - uR) + pR;
    for (int k = 0; k < np; k++) {
      double mkR = R->ph[k].alpha * R->ph[k].rho * (sR - uR);
      F->mass[k] = mkR / (sR - sM) * sM;
    }
    F->mom[0] = rhoStar * sM * sM + pStar;
    F->mom[1] = rhoStar * vY * sM;
    F->mom[2] = rhoStar * vZ * sM;
    F->energMix = (rhoStar * EStar + pStar) * sM;
  }
  F->sM = sM;
  F->uStar = 0.;
}

/* ------------------------------------------------------------------------------ flux accumulation */
/* FluxUEq::addFlux/subtractFlux src/Models/UEq/FluxUEq.cpp:61,85 ;
 * FluxPUEq::addNonCons/subtractNonCons src/Models/PUEq/FluxPUEq.cpp:44,56 ;
 * FluxEuler add/subtract (no non-conservative terms). */
static void acc_add(const ecgo_sim* S, OFlux* acc, const OFlux* F, double cA, const OSt* cellN) {
  for (int k = 0; k < S->c.ntr; k++) { /* Transport::addFlux, addNonCons (time-n value) */
    acc->tr[k] += cA * F->tr[k];
    acc->tr[k] += -cA * cellN->tr[k] * F->sM;
  }
  if (S->c.model == ECGO_MODEL_EULER) {
    acc->mass[0] += cA * F->mass[0];
    for (int d = 0; d < 3; d++) acc->mom[d] += cA * F->mom[d];
    acc->energMix += cA * F->energMix;
    return;
  }
  if (S->c.model == ECGO_MODEL_PTUEQ) { /* FluxPTUEq::addFlux src/Models/PTUEq/FluxPTUEq.cpp:55 */
    for (int k = 0; k < S->np; k++) acc->mass[k] += cA * F->mass[k];
    for (int d = 0; d < 3; d++) acc->mom[d] += cA * F->mom[d];
    acc->energMix += cA * F->energMix;
    return;
  }
  for (int k = 0; k < S->np; k++) {
    acc->alpha[k] += cA * F->alpha[k];
    acc->mass[k] += cA * F->mass[k];
    acc->energ[k] += cA * F->energ[k];
  }
  for (int d = 0; d < 3; d++) acc->mom[d] += cA * F->mom[d];
  acc->energMix += cA * F->energMix;
  for (int k = 0; k < S->np; k++) {
    const OPh* ph = &cellN->ph[k];
    acc->alpha[k] += -cA * ph->alpha * F->sM;
    acc->energ[k] += cA * ph->alpha * ph->p * F->uStar;
  }
}

static void acc_sub(const ecgo_sim* S, OFlux* acc, const OFlux* F, double cA, const OSt* cellN) {
  for (int k = 0; k < S->c.ntr; k++) { /* Transport::subtractFlux, subtractNonCons */
    acc->tr[k] -= cA * F->tr[k];
    acc->tr[k] -= -cA * cellN->tr[k] * F->sM;
  }
  if (S->c.model == ECGO_MODEL_EULER) {
    acc->mass[0] -= cA * F->mass[0];
    for (int d = 0; d < 3; d++) acc->mom[d] -= cA * F->mom[d];
    acc->energMix -= cA * F->energMix;
    return;
  }
  if (S->c.model == ECGO_MODEL_PTUEQ) { /* FluxPTUEq::subtractFlux :79 */
    for (int k = 0; k < S->np; k++) acc->mass[k] -= cA * F->mass[k];
    for (int d = 0; d < 3; d++) acc->mom[d] -= cA * F->mom[d];
    acc->energMix -= cA * F->energMix;
    return;
  }
  for (int k = 0; k < S->np; k++) {
    acc->alpha[k] -= cA * F->alpha[k];
    acc->mass[k] -= cA * F->mass[k];
    acc->energ[k] -= cA * F->energ[k];
  }
  for (int d = 0; d < 3; d++) acc->mom[d] -= cA * F->mom[d];
  acc->energMix -= cA * F->energMix;
  for (int k = 0; k < S->np; k++) {
    const OPh* ph = &cellN->ph[k];
    acc->alpha[k] -= -cA * ph->alpha * F->sM;
    acc->energ[k] -= cA * ph->alpha * ph->p * F->uStar;
  }
}

/* --------------------------------------------------------------------------- cons <-> prim */

static void build_cons(const ecgo_sim* S, const OSt* st, OFlux* U) { /* FluxUEq::buildCons :147 ; FluxEuler::buildCons */
  if (S->c.model == ECGO_MODEL_EULER) {
    const OPh* ph = &st->ph[0];
    U->mass[0] = ph->rho;
    for (int d = 0; d < 3; d++) U->mom[d] = U->mass[0] * ph->u[d];
    U->energMix = U->mass[0] * ph->E;
    return;
  }
  if (S->c.model == ECGO_MODEL_PTUEQ) { /* FluxPTUEq::buildCons src/Models/PTUEq/FluxPTUEq.cpp:109 */
    for (int k = 0; k < S->np; k++) U->mass[k] = st->ph[k].alpha * st->ph[k].rho;
    for (int d = 0; d < 3; d++) U->mom[d] = st->m.rho * st->m.u[d];
    U->energMix = st->m.rho * st->m.E;
    return;
  }
  for (int k = 0; k < S->np; k++) {
    const OPh* ph = &st->ph[k];
    U->alpha[k] = ph->alpha;
    U->mass[k] = ph->alpha * ph->rho;
    U->energ[k] = ph->alpha * ph->rho * eos_e(&S->c.eos[k], S->eps, ph->rho, ph->p);
  }
  for (int d = 0; d < 3; d++) U->mom[d] = st->m.rho * st->m.u[d];
  U->energMix = st->m.rho * st->m.E;
}

/* m_cons = scale * m_cons + Un  (multiply, then addFlux(1.) of fluxBuff = Un) */
static void time_evolve(const ecgo_sim* S, OFlux* acc, const OFlux* Un, double scale) {
  int np = (S->c.model == ECGO_MODEL_EULER) ? 1 : S->np;
  for (int k = 0; k < np; k++) {
    acc->alpha[k] *= scale;
    acc->mass[k] *= scale;
    acc->energ[k] *= scale;
  }
  for (int d = 0; d < 3; d++) acc->mom[d] *= scale;
  acc->energMix *= scale;
  for (int k = 0; k < np; k++) {
    acc->alpha[k] += 1. * Un->alpha[k];
    acc->mass[k] += 1. * Un->mass[k];
    acc->energ[k] += 1. * Un->energ[k];
  }
  for (int d = 0; d < 3; d++) acc->mom[d] += 1. * Un->mom[d];
  acc->energMix += 1. * Un->energMix;
}

static void build_prim(const ecgo_sim* S, OFlux* U, OSt* st) { /* FluxUEq::buildPrim :161 ; FluxEuler::buildPrim :124 */
  double eps = S->eps;
  if (S->c.model == ECGO_MODEL_EULER) {
    const ecgo_eos* q = &S->c.eos[0];
    OPh* ph = &st->ph[0];
    ph->rho = U->mass[0];
    ph->u[0] = U->mom[0] / U->mass[0];
    ph->u[1] = U->mom[1] / U->mass[0];
    ph->u[2] = U->mom[2] / U->mass[0];
    for (int d = 0; d < 3; d++)
      if (fabs(ph->u[d]) < 1.e-8) ph->u[d] = 0.;
    double Et = U->energMix / U->mass[0];
    ph->E = Et;
    double ei = Et - 0.5 * sqnorm(ph->u);
    ph->e = ei;
    ph->p = eos_p(q, eps, U->mass[0], ei);
    ph->c = eos_c(q, eps, U->mass[0], ph->p);
    ph->T = eos_T(q, eps, U->mass[0], ph->p);
    return;
  }
  if (S->c.model == ECGO_MODEL_PTUEQ) {
    /* FluxPTUEq::buildPrim src/Models/PTUEq/FluxPTUEq.cpp:125-160 with MixPTUEq::computePressure
     * (:93-122, analytic p of two IG/SG phases, Le Martelot 2013) and computeTemperature (:126-145) */
    double rhoMel = 0.;
    for (int k = 0; k < 2; k++) rhoMel += U->mass[k];
    st->m.u[0] = U->mom[0] / rhoMel;
    st->m.u[1] = U->mom[1] / rhoMel;
    st->m.u[2] = U->mom[2] / rhoMel;
    for (int d = 0; d < 3; d++)
      if (fabs(st->m.u[d]) < 1.e-8) st->m.u[d] = 0.;
    double ie = U->energMix / rhoMel - 0.5 * (st->m.u[0] * st->m.u[0] + st->m.u[1] * st->m.u[1] + st->m.u[2] * st->m.u[2]);
    const ecgo_eos* E1 = &S->c.eos[0];
    const ecgo_eos* E2 = &S->c.eos[1];
    double gamma1 = E1->gamma, pInf1 = eos_pinf(E1), cv1 = E1->cv, e01 = E1->eref, Y1 = U->mass[0] / rhoMel;
    double gamma2 = E2->gamma, pInf2 = eos_pinf(E2), cv2 = E2->cv, e02 = E2->eref, Y2 = U->mass[1] / rhoMel;
    double q = Y1 * e01 + Y2 * e02;
    double cvMel = Y1 * cv1 + Y2 * cv2;
    double A1 = Y1 * (gamma1 - 1.) * cv1 / cvMel * (rhoMel * (ie - q) - pInf1);
    double A2 = Y2 * (gamma2 - 1.) * cv2 / cvMel * (rhoMel * (ie - q) - pInf2);
    double pressure = 0.5 * (A1 + A2 - (pInf1 + pInf2)) +
                      sqrt(0.25 * (A2 - A1 - (pInf2 - pInf1)) * (A2 - A1 - (pInf2 - pInf1)) + A1 * A2);
    double temperature = 0.;
    for (int k = 0; k < 2; k++) {
      const ecgo_eos* E = &S->c.eos[k];
      temperature += U->mass[k] / rhoMel * (E->gamma - 1.) * E->cv / (pressure + eos_pinf(E));
    }
    temperature = 1. / (temperature * rhoMel);
    st->m.p = pressure;
    st->m.T = temperature;
    for (int k = 0; k < 2; k++) {
      OPh* ph = &st->ph[k];
      ph->p = pressure;
      ph->rho = eos_rho_pT(&S->c.eos[k], eps, pressure, temperature);
      ph->alpha = U->mass[k] / ph->rho;
      ph->T = temperature;
      ph->e = eos_e(&S->c.eos[k], eps, ph->rho, ph->p);
      ph->c = eos_c(&S->c.eos[k], eps, ph->rho, ph->p);
    }
    ptueq_mixture_vars(S, st);
    st->m.E = U->energMix / rhoMel;
    return;
  }
  int np = S->np;
  double un = 0., rhoMel = 0.;
  if (eps > 1.e-20) {
    for (int k = 0; k < np; k++) {
      if (U->alpha[k] < 0.) U->alpha[k] = 0.;
      if (U->alpha[k] > 1.) U->alpha[k] = 1.;
      un += U->alpha[k];
    }
  } else {
    for (int k = 0; k < np; k++) {
      if (U->alpha[k] <= 1.e-15) U->alpha[k] = 1e-15;
      if (U->alpha[k] >= 1. - 1.e-15) U->alpha[k] = 1.0 - 1e-15;
      un += U->alpha[k];
    }
  }
  for (int k = 0; k < np; k++) U->alpha[k] /= un;
  for (int k = 0; k < np; k++) {
    const ecgo_eos* q = &S->c.eos[k];
    OPh* ph = &st->ph[k];
    rhoMel += U->mass[k];
    ph->alpha = U->alpha[k];
    ph->rho = U->mass[k] / omax(U->alpha[k], eps);
    eos_rho_max_mass(q, U->mass[k], &ph->alpha, &ph->rho);
    double ek = U->energ[k] / omax(U->mass[k], eps);
    ph->p = eos_p(q, eps, ph->rho, ek);
    phase_fix(S, k, ph);
  }
  st->m.u[0] = U->mom[0] / rhoMel;
  st->m.u[1] = U->mom[1] / rhoMel;
  st->m.u[2] = U->mom[2] / rhoMel;
  for (int d = 0; d < 3; d++)
    if (fabs(st->m.u[d]) < 1.e-8) st->m.u[d] = 0.;
  for (int k = 0; k < np; k++) phase_extended(S, k, &st->ph[k]);
  mixture_vars(S, st);
  st->m.E = U->energMix / rhoMel;
}

/* ----------------------------------------------------------------------------------- relaxations */

static int newton_p(const ecgo_sim* S, double* pStar, const double* ak, const double* pk, const double* rhok,
                    double* akS, double* rhokS) {
  /* RelaxationP::NewtonRaphson src/Relaxations/RelaxationP.cpp:43-68 */
  int np = S->np, iteration = 0;
  double f = 0., df = 1., drhodp = 0., dalpha = 0.;
  do {
    iteration++;
    *pStar -= f / df;
    for (int k = 0; k < np; k++) eos_fix_p(&S->c.eos[k], pStar);
    f = -1.;
    df = 0.;
    for (int k = 0; k < np; k++) {
      rhokS[k] = eos_rho_pfinal(&S->c.eos[k], S->eps, pk[k], rhok[k], *pStar, &drhodp);
      akS[k] = ak[k] * rhok[k] / rhokS[k];
      dalpha = ak[k] * rhok[k] * drhodp / (rhokS[k] * rhokS[k]);
      f += akS[k];
      df -= dalpha;
    }
  } while (fabs(f) > 1e-10 && iteration < 100);
  return iteration;
}

static void relax_pinf(ecgo_sim* S, OSt* st) {
  /* RelaxationPInfinite::relaxation src/Relaxations/RelaxationPInfinite.cpp:43-97 */
  int np = S->np;
  int relax = 1;
  if (S->eps > 1.e-20) {
    for (int k = 0; k < np; k++)
      if (st->ph[k].alpha > (1. - 1.e-5)) relax = 0;
  }
  if (!relax) return;
  double ak[NP_MAX], pk[NP_MAX], rhok[NP_MAX], akS[NP_MAX], rhokS[NP_MAX];
  double pStar = 0.;
  for (int k = 0; k < np; k++) {
    ak[k] = st->ph[k].alpha;
    pk[k] = st->ph[k].p;
    rhok[k] = st->ph[k].rho;
    pStar += ak[k] * pk[k];
  }
  int it = newton_p(S, &pStar, ak, pk, rhok, akS, rhokS);
  S->st.relax_calls++;
  S->st.newton_evals += it;
  if (it > S->st.newton_max) S->st.newton_max = it;
  if (it < 100) {
    for (int k = 0; k < np; k++) {
      st->ph[k].alpha = akS[k];
      st->ph[k].rho = rhokS[k];
      st->ph[k].p = pStar;
    }
    st->m.p = pStar;
  } else {
    S->st.newton_fallback++;
    /* RelaxationP::computeInterfacePressure src/Relaxations/RelaxationP.cpp:72 */
    double zk[NP_MAX], pI = 0., sumZk = 0., sumZj = 0., drhodp = 0.;
    for (int k = 0; k < np; k++) zk[k] = st->ph[k].rho * st->ph[k].c;
    for (int k = 0; k < np; k++) {
      sumZk += zk[k];
      sumZj = 0.;
      for (int j = 0; j < np; j++)
        if (j != k) sumZj += zk[j];
      pI += sumZj * (st->ph[k].p - 0.);
    }
    pI /= sumZk * (np - 1);
    for (int k = 0; k < np; k++) eos_fix_p(&S->c.eos[k], &pI);
    for (int k = 0; k < np; k++) {
      rhokS[k] = eos_rho_pfinal(&S->c.eos[k], S->eps, pk[k], rhok[k], pI, &drhodp);
      akS[k] = ak[k] * rhok[k] / rhokS[k];
      st->ph[k].alpha = akS[k];
      st->ph[k].rho = rhokS[k];
      st->ph[k].p = pI;
    }
    st->m.p = pI;
  }
}

static double compute_tsat(const ecgo_eos* L, const ecgo_eos* V, double p, double* dTsat, int* err) {
  /* Mixture::computeTsat src/Models/Mixture.cpp:59-100 (IG/SG only) */
  double gL = L->gamma, piL = (L->type == ECGO_EOS_IG) ? 0. : L->pinf, cvL = L->cv, e0L = L->eref, s0L = L->sref;
  double gV = V->gamma, piV = (V->type == ECGO_EOS_IG) ? 0. : V->pinf, cvV = V->cv, e0V = V->eref, s0V = V->sref;
  double A = (gL * cvL - gV * cvV + s0V - s0L) / (gV * cvV - cvV);
  double B = (e0L - e0V) / (gV * cvV - cvV);
  double C = (gV * cvV - gL * cvL) / (gV * cvV - cvV);
  double D = (gL * cvL - cvL) / (gV * cvV - cvV);
  int iteration = 0;
  double Tsat = 0.1 * B / C, f = 0., df = 1.;
  do {
    Tsat -= f / df;
    iteration++;
    if (iteration > 50) {
      *err = 1;
      break;
    }
    f = A + B / Tsat + C * ECGO_LOG(Tsat) - ECGO_LOG(p + piV) + D * ECGO_LOG(p + piL);
    df = C / Tsat - B / (Tsat * Tsat);
  } while (fabs(f) > 1e-10);
  double dfdp = -1. / (p + piV) + D / (p + piL);
  if (dTsat) *dTsat = -dfdp / df;
  return Tsat;
}

static void relax_ptmu(ecgo_sim* S, OSt* st) {
  /* RelaxationPTMu::relaxation src/Relaxations/RelaxationPTMu.cpp:73-200 */
  int liq = S->c.ptmu_liq, vap = S->c.ptmu_vap, err = 0;
  const ecgo_eos* EL = &S->c.eos[liq];
  const ecgo_eos* EV = &S->c.eos[vap];
  double pStar = 0., Tsat, dTsat = 0.;
  for (int k = 0; k < S->np; k++) pStar += st->ph[k].alpha * st->ph[k].p;
  if (pStar > S->pcrit) return;
  double rho = st->m.rho;
  double rhoe = rho * st->m.e;
  double rhov = st->m.rho, ev = st->m.e;
  double pv = eos_p(EV, S->eps, rhov, ev);
  double Tv = eos_T(EV, S->eps, rhov, pv);
  if (pv > 0) {
    Tsat = compute_tsat(EL, EV, pv, &dTsat, &err);
    if (Tv >= Tsat) {
      st->ph[vap].alpha = 1.;
      st->ph[liq].alpha = 0.;
      st->ph[vap].rho = rhov;
      st->ph[vap].e = ev;
      st->ph[vap].p = pv;
      fulfill(S, st);
      if (err) S->st.ptmu_errors++;
      return;
    }
  }
  double rhol = st->m.rho, el = st->m.e;
  double pl = eos_p(EL, S->eps, rhol, el);
  double Tl = eos_T(EL, S->eps, rhol, pl);
  if (pl > 0.) {
    Tsat = compute_tsat(EL, EV, pl, &dTsat, &err);
    if (Tl <= Tsat) {
      st->ph[liq].alpha = 1.;
      st->ph[vap].alpha = 0.;
      st->ph[liq].rho = rhol;
      st->ph[liq].e = el;
      st->ph[liq].p = pl;
      fulfill(S, st);
      if (err) S->st.ptmu_errors++;
      return;
    }
  }
  double rhoLSat = 0., rhoVSat = 0., drhoLSat, drhoVSat, aLSat = 0., aVSat = 0., daLSat, daVSat;
  double rhoeLSat, rhoeVSat, drhoeLSat, drhoeVSat;
  int iteration = 0;
  double f = 0., df = 1.;
  do {
    pStar -= f / df;
    iteration++;
    if (iteration > 50) {
      err = 1;
      break;
    }
    for (int k = 0; k < S->np; k++) eos_fix_p(&S->c.eos[k], &pStar);
    Tsat = compute_tsat(EL, EV, pStar, &dTsat, &err);
    rhoLSat = eos_rho_sat(EL, S->eps, pStar, Tsat, dTsat, &drhoLSat);
    rhoVSat = eos_rho_sat(EV, S->eps, pStar, Tsat, dTsat, &drhoVSat);
    aLSat = (rho - rhoVSat) / (rhoLSat - rhoVSat);
    daLSat = (-drhoVSat * (rhoLSat - rhoVSat) - (rho - rhoVSat) * (drhoLSat - drhoVSat)) /
             ((rhoLSat - rhoVSat) * (rhoLSat - rhoVSat));
    aVSat = 1. - aLSat;
    daVSat = -daLSat;
    f = rhoe;
    df = 0.;
    rhoeLSat = eos_rhoe_sat(EL, pStar, rhoLSat, drhoLSat, &drhoeLSat);
    rhoeVSat = eos_rhoe_sat(EV, pStar, rhoVSat, drhoVSat, &drhoeVSat);
    f -= (aLSat * rhoeLSat + aVSat * rhoeVSat);
    df -= (daLSat * rhoeLSat + aLSat * drhoeLSat + daVSat * rhoeVSat + aVSat * drhoeVSat);
    f /= rhoe;
    df /= rhoe;
  } while (fabs(f) > 1e-10);
  if (err) S->st.ptmu_errors++;
  st->ph[liq].alpha = aLSat;
  st->ph[liq].rho = rhoLSat;
  st->ph[liq].p = pStar;
  st->ph[vap].alpha = aVSat;
  st->ph[vap].rho = rhoVSat;
  st->ph[vap].p = pStar;
  fulfill(S, st);
}

/* RelaxationPT::relaxation src/Relaxations/RelaxationPT.cpp:43-140: analytic pressure-temperature
 * equilibrium of two IG/SG phases (Le Martelot 2013) from the mixture energy and density and the
 * mass fractions of the rebuilt state, then rho_k = computeDensity(p*, T*). */
static void relax_pt(ecgo_sim* S, OSt* st) {
  if (S->eps > 1.e-20)
    for (int k = 0; k < S->np; k++)
      if (st->ph[k].alpha > (1. - 1.e-5)) return;
  const ecgo_eos* E1 = &S->c.eos[0];
  const ecgo_eos* E2 = &S->c.eos[1];
  double e0 = st->m.e, rho0 = st->m.rho;
  double gamma1 = E1->gamma, pInf1 = (E1->type == ECGO_EOS_IG) ? 0. : E1->pinf, cv1 = E1->cv, e01 = E1->eref;
  double gamma2 = E2->gamma, pInf2 = (E2->type == ECGO_EOS_IG) ? 0. : E2->pinf, cv2 = E2->cv, e02 = E2->eref;
  double Y1 = st->ph[0].Y, Y2 = st->ph[1].Y;
  double q = Y1 * e01 + Y2 * e02;
  double cvMel = Y1 * cv1 + Y2 * cv2;
  double A1 = Y1 * (gamma1 - 1.) * cv1 / cvMel * (rho0 * (e0 - q) - pInf1);
  double A2 = Y2 * (gamma2 - 1.) * cv2 / cvMel * (rho0 * (e0 - q) - pInf2);
  double pressure = 0.5 * (A1 + A2 - (pInf1 + pInf2)) +
                    sqrt(0.25 * (A2 - A1 - (pInf2 - pInf1)) * (A2 - A1 - (pInf2 - pInf1)) + A1 * A2);
  double temperature = 0.;
  for (int k = 0; k < 2; k++) {
    const ecgo_eos* E = &S->c.eos[k];
    double pInfk = (E->type == ECGO_EOS_IG) ? 0. : E->pinf;
    temperature += st->ph[k].Y * (E->gamma - 1.) * E->cv / (pressure + pInfk);
  }
  temperature = 1. / (temperature * rho0);
  double rhoS[2], aS[2];
  for (int k = 0; k < 2; k++) {
    const ecgo_eos* E = &S->c.eos[k];
    double den = omax(((E->gamma - 1.) * E->cv * temperature), S->eps);
    rhoS[k] = (E->type == ECGO_EOS_IG) ? pressure / den : (pressure + E->pinf) / den;
    aS[k] = st->ph[k].alpha * st->ph[k].rho / rhoS[k];
  }
  for (int k = 0; k < 2; k++) {
    st->ph[k].alpha = aS[k];
    st->ph[k].rho = rhoS[k];
    st->ph[k].p = pressure;
  }
  st->m.p = pressure;
}

static void relaxations(ecgo_sim* S, OSt* st) { /* Model::relaxations src/Models/Model.cpp:74 */
  if (S->c.model != ECGO_MODEL_KAPILA) return;
  relax_pinf(S, st);
  if (S->c.ptmu) relax_ptmu(S, st);
  if (S->c.pt) relax_pt(S, st);
}

static void correction_energy(ecgo_sim* S, OSt* st) {
  /* Cell::correctionEnergy src/Order1/Cell.cpp:327 -> MixUEq::totalEnergyToInternalEnergy :175
   * -> FluxPUEq::correctionEnergy src/Models/PUEq/FluxPUEq.cpp:68-112 */
  st->m.e = st->m.E - 0.5 * sqnorm(st->m.u);
  double rhoe = st->m.rho * st->m.e;
  double p = rhoe, denom = 0., gpi, eref, ig, cov;
  for (int k = 0; k < S->np; k++) {
    eos_mix(&S->c.eos[k], &gpi, &eref, &ig, &cov);
    p -= st->ph[k].alpha * (gpi * (1. - st->ph[k].rho * cov) + st->ph[k].rho * eref);
    denom += st->ph[k].alpha * ig * (1. - st->ph[k].rho * cov);
  }
  p /= denom;
  for (int k = 0; k < S->np; k++) {
    st->ph[k].p = p;
    phase_fix(S, k, &st->ph[k]);
  }
  st->m.p = p;
}

/* ------------------------------------------------------------------------------------- limiters */
/* src/Order2/Limiter{Minmod,VanLeer,VanAlbada,SuperBee,MC,THINC}.cpp */
double ecgo_limiter(int kind, double s1, double s2) {
  double slope = 0., prod = s1 * s2, sum = s1 + s2;
  switch (kind) {
    case ECGO_LIM_MINMOD:
    case ECGO_LIM_THINC:
      if (prod > 1e-9) {
        slope = omin(fabs(s1), fabs(s2));
        if (s1 < 0) slope = -slope;
      }
      return slope;
    case ECGO_LIM_VANLEER:
      if ((fabs(sum) > 1e-6) && (prod > 1e-6)) slope = 2. * prod / sum;
      return slope;
    case ECGO_LIM_VANALBADA:
      if ((fabs(s1) > 1e-6) && (fabs(s2) > 1e-6) && (fabs(sum) > 1e-6) && (prod > 1e-6))
        slope = prod * sum / (s1 * s1 + s2 * s2);
      return slope;
    case ECGO_LIM_SUPERBEE:
      if (prod > 1e-6) slope = omax(omin(2. * fabs(s1), fabs(s2)), omin(fabs(s1), 2. * fabs(s2)));
      if (s1 < 0.) slope = -slope;
      return slope;
    case ECGO_LIM_MC:
      if (prod > 1e-9) {
        slope = omin(2. * fabs(s1), 2. * fabs(s2));
        slope = omin(slope, 0.5 * (fabs(s1) + fabs(s2)));
      }
      if (s1 < 0.) slope = -slope;
      return slope;
    default:
      return 0.;
  }
}

/* ----------------------------------------------------------------------------------------- mesh */

/* Cell sizes and centres along one axis: MeshCartesian::meshStretching src/Meshes/MeshCartesian.cpp:168-210
 * (uniform: l / n and (i + 0.5) d) with stretchZone::stretching src/Meshes/stretchZone.cpp:45-66 for
 * each zone in turn (geometric progression of ratio `factor`, or uniform when |factor - 1| < 1e-6). */
static void axis_cells(const ecgo_case* c, int ax, int n, double l, double* d, double* pos) {
  if (c->nstretch[ax] == 0 || n == 1) {
    const double dd = l / (double)n;
    for (int i = 0; i < n; i++) {
      d[i] = dd;
      pos[i] = (i + 0.5) * dd;
    }
    return;
  }
  int m = 0;
  for (int z = 0; z < c->nstretch[ax]; z++) {
    const ecgo_stretch* st = &c->stretch[ax][z];
    double dX0 = (st->end - st->start) / st->ncells;
    if (fabs(st->factor - 1.) < 1e-6) {
      for (int i = 0; i < st->ncells; i++, m++) {
        d[m] = dX0;
        pos[m] = st->start + (i + 0.5) * dX0;
      }
    } else {
      dX0 = (st->end - st->start) * (1. - st->factor) / (1. - pow(st->factor, st->ncells));
      d[m] = dX0;
      pos[m] = st->start + 0.5 * dX0;
      m++;
      for (int i = 1; i < st->ncells; i++, m++) {
        d[m] = dX0 * pow(st->factor, i);
        pos[m] = pos[m - 1] + 0.5 * (d[m - 1] + d[m]);
      }
    }
  }
}

static void build_mesh(ecgo_sim* S) {
  /* MeshCartesian::meshStretching :168 and initializeGeometrieMonoCpu :212-558 */
  const ecgo_case* c = &S->c;
  int nx = c->nx, ny = c->ny, nz = c->nz, n = nx * ny * nz;
  double* dX = (double*)malloc(sizeof(double) * (size_t)nx);
  double* dY = (double*)malloc(sizeof(double) * (size_t)ny);
  double* dZ = (double*)malloc(sizeof(double) * (size_t)nz);
  double* pX = (double*)malloc(sizeof(double) * (size_t)nx);
  double* pY = (double*)malloc(sizeof(double) * (size_t)ny);
  double* pZ = (double*)malloc(sizeof(double) * (size_t)nz);
  axis_cells(c, 0, nx, c->lx, dX, pX);
  axis_cells(c, 1, ny, c->ly, dY, pY);
  axis_cells(c, 2, nz, c->lz, dZ, pZ);
  S->pos = (double*)calloc((size_t)3 * n, sizeof(double));
  S->vol = (double*)calloc((size_t)n, sizeof(double));
  S->lcfl = (double*)calloc((size_t)n, sizeof(double));
  S->cellface = (int*)malloc(sizeof(int) * 6 * (size_t)n);
  for (int i = 0; i < 6 * n; i++) S->cellface[i] = -1;
  for (int i = 0; i < n; i++) {
    int iz = i / (nx * ny), r = i % (nx * ny), iy = r / nx, ix = r % nx;
    S->vol[i] = dX[ix] * dY[iy] * dZ[iz];
    double l = 1.e10;
    if (nx != 1) l = omin(l, dX[ix]);
    if (ny != 1) l = omin(l, dY[iy]);
    if (nz != 1) l = omin(l, dZ[iz]);
    if (S->dim > 1) l *= 0.6;
    S->lcfl[i] = l;
    S->pos[3 * i + 0] = pX[ix];
    S->pos[3 * i + 1] = pY[iy];
    S->pos[3 * i + 2] = pZ[iz];
  }
  int maxf = 3 * n + 2 * (ny * nz + nx * nz + nx * ny);
  S->faces = (OFace*)calloc((size_t)maxf, sizeof(OFace));
  int f = 0;
#define IDX(a, b, cc) ((nx != 1 ? (a) : 0) + (ny != 1 ? (b) * nx : 0) + (nz != 1 ? (cc) * nx * ny : 0))
#define SETV(v, x, y, z) (v)[0] = (x), (v)[1] = (y), (v)[2] = (z)
  /* X faces */
  for (int ix = 0; ix < nx - 1; ix++)
    for (int iy = 0; iy < ny; iy++)
      for (int iz = 0; iz < nz; iz++) {
        OFace* F = &S->faces[f];
        F->L = IDX(ix, iy, iz); F->R = IDX(ix + 1, iy, iz); F->axis = 0; F->bc = -1;
        SETV(F->n, 1., 0., 0.); SETV(F->t, 0., 1., 0.); SETV(F->b, 0., 0., 1.);
        F->surface = dY[iy] * dZ[iz];
        SETV(F->pos, S->pos[3 * F->L] + 0.5 * dX[ix], S->pos[3 * F->L + 1], S->pos[3 * F->L + 2]);
        S->cellface[6 * F->L + 1] = f; S->cellface[6 * F->R + 0] = f;
        f++;
      }
  for (int ix = 0; ix < nx; ix++)
    for (int iy = 0; iy < ny - 1; iy++)
      for (int iz = 0; iz < nz; iz++) {
        OFace* F = &S->faces[f];
        F->L = IDX(ix, iy, iz); F->R = IDX(ix, iy + 1, iz); F->axis = 1; F->bc = -1;
        SETV(F->n, 0., 1., 0.); SETV(F->t, -1., 0., 0.); SETV(F->b, 0., 0., 1.);
        F->surface = dX[ix] * dZ[iz];
        SETV(F->pos, S->pos[3 * F->L], S->pos[3 * F->L + 1] + 0.5 * dY[iy], S->pos[3 * F->L + 2]);
        S->cellface[6 * F->L + 3] = f; S->cellface[6 * F->R + 2] = f;
        f++;
      }
  for (int ix = 0; ix < nx; ix++)
    for (int iy = 0; iy < ny; iy++)
      for (int iz = 0; iz < nz - 1; iz++) {
        OFace* F = &S->faces[f];
        F->L = IDX(ix, iy, iz); F->R = IDX(ix, iy, iz + 1); F->axis = 2; F->bc = -1;
        SETV(F->n, 0., 0., 1.); SETV(F->t, 1., 0., 0.); SETV(F->b, 0., 1., 0.);
        F->surface = dX[ix] * dY[iy];
        SETV(F->pos, S->pos[3 * F->L], S->pos[3 * F->L + 1], S->pos[3 * F->L + 2] + 0.5 * dZ[iz]);
        S->cellface[6 * F->L + 5] = f; S->cellface[6 * F->R + 4] = f;
        f++;
      }
  S->ninner = f;
  /* boundary faces: Xm, Xp, Ym, Yp, Zm, Zp (src/Meshes/MeshCartesian.cpp:384-557); positions 0 on the
   * minus sides and last centre + half size on the plus sides; each side takes the boundary condition
   * of its index in the case file (MeshCartesian::assignLimits :86) */
  const int nn3[3] = {nx, ny, nz};
  for (int ax = 0; ax < 3; ax++) {
    if (nn3[ax] == 1) continue;
    int o1 = (ax == 0) ? 1 : 0, o2 = (ax == 2) ? 1 : 2;
    for (int side = 0; side < 2; side++) {
      for (int a = 0; a < nn3[o1]; a++)
        for (int b2 = 0; b2 < nn3[o2]; b2++) {
          int ijk[3];
          ijk[ax] = side ? nn3[ax] - 1 : 0;
          ijk[o1] = a;
          ijk[o2] = b2;
          OFace* F = &S->faces[f];
          F->L = IDX(ijk[0], ijk[1], ijk[2]); F->R = -1; F->axis = ax;
          F->bc = c->bc[2 * ax + side];
          double sg = side ? 1. : -1.;
          const double sx = dX[ijk[0]], sy = dY[ijk[1]], sz = dZ[ijk[2]];
          if (ax == 0) { SETV(F->n, sg, 0., 0.); SETV(F->t, 0., sg, 0.); SETV(F->b, 0., 0., 1.); F->surface = sy * sz; }
          if (ax == 1) { SETV(F->n, 0., sg, 0.); SETV(F->t, -sg, 0., 0.); SETV(F->b, 0., 0., 1.); F->surface = sx * sz; }
          if (ax == 2) { SETV(F->n, 0., 0., sg); SETV(F->t, sg, 0., 0.); SETV(F->b, 0., 1., 0.); F->surface = sx * sy; }
          const double dd[3] = {sx, sy, sz};
          for (int d = 0; d < 3; d++) F->pos[d] = S->pos[3 * F->L + d];
          F->pos[ax] = side ? S->pos[3 * F->L + ax] + 0.5 * dd[ax] : 0.;
          S->cellface[6 * F->L + 2 * ax + side] = f;
          f++;
        }
    }
  }
#undef IDX
#undef SETV
  S->nfaces = f;
  free(dX); free(dY); free(dZ); free(pX); free(pY); free(pZ);
}

static double vnorm_diff(const double* a, const double* b) { /* Element::distance / Face::distance */
  double x = a[0] - b[0], y = a[1] - b[1], z = a[2] - b[2];
  return sqrt(x * x + y * y + z * z);
}

/* ------------------------------------------------------------------------------------ face fluxes */

static void riemann(ecgo_sim* S, OSt* L, OSt* R, const OFace* F, double dxL, double dxR, double* dtMax, OFlux* out) {
  /* projections + model Riemann solver + flux reverse projection (CellInterface::solveRiemann :154) */
  OSt l = *L, r = *R;
  proj_local(vel_of(S, &l), F->n, F->t, F->b);
  proj_local(vel_of(S, &r), F->n, F->t, F->b);
  if (S->c.model == ECGO_MODEL_EULER) hllc_euler(S, &l, &r, dxL, dxR, dtMax, out);
  else if (S->c.model == ECGO_MODEL_PTUEQ) hllc_ptueq(S, &l, &r, dxL, dxR, dtMax, out);
  else hllc_ueq(S, &l, &r, dxL, dxR, dtMax, out);
  for (int k = 0; k < S->c.ntr; k++) /* Transport::solveRiemann src/Transport/Transport.cpp: upwind by sM */
    out->tr[k] = (out->sM > 0.) ? l.tr[k] * out->sM : r.tr[k] * out->sM;
  proj_reverse(out->mom, F->n, F->t, F->b);
}

static void compute_slopes(ecgo_sim* S, OSt* st) {
  /* CellInterfaceO2Cartesian::computeSlopes src/Order2/CellInterfaceO2Cartesian.cpp:77 */
  for (int f = 0; f < S->ninner; f++) {
    OFace* F = &S->faces[f];
    OSlope* sl = &S->slopes[f];
    double dist = vnorm_diff(&S->pos[3 * F->L], &S->pos[3 * F->R]);
    OSt* L = &st[F->L];
    OSt* R = &st[F->R];
    for (int k = 0; k < S->c.ntr; k++) sl->tr[k] = (R->tr[k] - L->tr[k]) / dist; /* computeSlopeTransport */
    if (S->c.model == ECGO_MODEL_EULER) {
      sl->rho[0] = (R->ph[0].rho - L->ph[0].rho) / dist;
      sl->p[0] = (R->ph[0].p - L->ph[0].p) / dist;
      for (int d = 0; d < 3; d++) sl->u[d] = (R->ph[0].u[d] - L->ph[0].u[d]) / dist;
      continue;
    }
    if (S->c.model == ECGO_MODEL_PTUEQ) { /* PhasePTUEq::computeSlopesPhase :233, MixPTUEq::computeSlopesMixture :347 */
      for (int k = 0; k < S->np; k++) sl->alpha[k] = (R->ph[k].alpha - L->ph[k].alpha) / dist;
      sl->pm = (R->m.p - L->m.p) / dist;
      sl->Tm = (R->m.T - L->m.T) / dist;
      for (int d = 0; d < 3; d++) sl->u[d] = (R->m.u[d] - L->m.u[d]) / dist;
      continue;
    }
    for (int k = 0; k < S->np; k++) {
      sl->alpha[k] = (R->ph[k].alpha - L->ph[k].alpha) / dist;
      sl->rho[k] = (R->ph[k].rho - L->ph[k].rho) / dist;
      sl->p[k] = (R->ph[k].p - L->ph[k].p) / dist;
    }
    for (int d = 0; d < 3; d++) sl->u[d] = (R->m.u[d] - L->m.u[d]) / dist;
  }
  /* symmetry sides: BoundCondWallO2Cartesian::computeSlopes src/BoundConds/BoundCondWallO2Cartesian.cpp:84-108.
   * Only the velocity slope along each axis whose centre-to-face distance exceeds 1e-8 is set (the phase
   * slopes of PUEq have no velocity and stay zero). */
  for (int f = S->ninner; f < S->nfaces; f++) {
    OFace* F = &S->faces[f];
    if (F->bc != ECGO_BC_SYMMETRY) continue;
    OSlope* sl = &S->slopes[f];
    memset(sl, 0, sizeof(*sl));
    const double* u = (S->c.model == ECGO_MODEL_EULER) ? st[F->L].ph[0].u : st[F->L].m.u;
    for (int d = 0; d < 3; d++) {
      double dd = S->pos[3 * F->L + d] - F->pos[d]; /* Element::distanceX(Face*) src/Meshes/Element.cpp:117 */
      if (fabs(dd) > 1.e-8) sl->u[d] = u[d] / dd;
    }
  }
}

/* CellO2Cartesian::computeLocalSlopes src/Order2/CellO2Cartesian.cpp:23-171 for a Cartesian mesh without
 * AMR: slope 1 is the reference face's slope, slope 2 the slope of the face on the opposite side along the
 * same axis (zero if that side is a boundary); the neighbour across that face gives alphaCellAfterOppositeSide
 * (time-n volume fraction of phase 0). */
static void local_slopes(ecgo_sim* S, int cell, int face, double alphaCell, double alphaOther, OSlope* out,
                         double* alphaAfterOut) {
  const OFace* F = &S->faces[face];
  int side_plus = (F->L == cell);  /* reference face is on the + side of the cell */
  int opp = S->cellface[6 * cell + 2 * F->axis + (side_plus ? 0 : 1)];
  OSlope s1 = S->slopes[face], s2;
  double alphaAfter = 0.;
  memset(&s2, 0, sizeof(s2));
  if (opp >= 0 && S->faces[opp].bc != ECGO_BC_NONREFLECTING) {
    /* a non-reflecting side has no slopes and is skipped; a symmetry side gives its slopes and, as
     * alphaCellAfterOppositeSide, the cell's own alpha (its left cell, CellO2Cartesian.cpp:68-71) */
    s2 = S->slopes[opp];
    const OFace* G = &S->faces[opp];
    int nb = (G->R < 0) ? cell : ((G->L == cell) ? G->R : G->L);
    alphaAfter = (S->c.model == ECGO_MODEL_EULER) ? 0. : S->s[nb].ph[0].alpha;
  }
  int np = S->np;
  double eps = 1.e-4;
  *alphaAfterOut = alphaAfter;
  int interface = (alphaCell >= eps) && (alphaCell <= 1. - eps) &&
                  ((alphaOther - alphaCell) * (alphaCell - alphaAfter) >= 1.e-8);
  int lim = interface ? S->c.lim[1] : S->c.lim[0];
  int limv = interface ? S->c.lim[3] : S->c.lim[2];
  for (int k = 0; k < S->c.ntr; k++) out->tr[k] = ecgo_limiter(limv, s1.tr[k], s2.tr[k]);
  if (S->c.model == ECGO_MODEL_EULER) {
    out->rho[0] = ecgo_limiter(lim, s1.rho[0], s2.rho[0]);
    out->p[0] = ecgo_limiter(lim, s1.p[0], s2.p[0]);
    for (int d = 0; d < 3; d++) out->u[d] = ecgo_limiter(lim, s1.u[d], s2.u[d]);
    return;
  }
  if (S->c.model == ECGO_MODEL_PTUEQ) { /* PhasePTUEq::limitSlopes :256, MixPTUEq::limitSlopes :376 */
    for (int k = 0; k < np; k++) out->alpha[k] = ecgo_limiter(limv, s1.alpha[k], s2.alpha[k]);
    out->pm = ecgo_limiter(lim, s1.pm, s2.pm);
    out->Tm = ecgo_limiter(lim, s1.Tm, s2.Tm);
    for (int d = 0; d < 3; d++) out->u[d] = ecgo_limiter(lim, s1.u[d], s2.u[d]);
    return;
  }
  for (int k = 0; k < np; k++) {
    out->alpha[k] = ecgo_limiter(limv, s1.alpha[k], s2.alpha[k]);
    out->rho[k] = ecgo_limiter(lim, s1.rho[k], s2.rho[k]);
    out->p[k] = ecgo_limiter(lim, s1.p[k], s2.p[k]);
  }
  for (int d = 0; d < 3; d++) out->u[d] = ecgo_limiter(lim, s1.u[d], s2.u[d]);
}

/* CellO2Cartesian::computeLocalSlopesLimite src/Order2/CellO2Cartesian.cpp:173-272 for a symmetry side:
 * slope 1 is the side's own slope, slope 2 the slope of the internal face on the opposite side; the
 * interface detector only tests the cell's time-n alpha against 1e-4. */
static void local_slopes_side(ecgo_sim* S, int cell, int face, OSlope* out) {
  const OFace* F = &S->faces[face];
  int plus = (S->cellface[6 * cell + 2 * F->axis + 1] == face);
  int opp = S->cellface[6 * cell + 2 * F->axis + (plus ? 0 : 1)];
  OSlope s1 = S->slopes[face], s2;
  memset(&s2, 0, sizeof(s2));
  if (opp >= 0 && S->faces[opp].bc != ECGO_BC_NONREFLECTING) s2 = S->slopes[opp];
  double eps = 1.e-4;
  int interface = 0;
  if (S->c.model != ECGO_MODEL_EULER) {
    double a = S->s[cell].ph[0].alpha;
    interface = (a >= eps) && (a <= 1. - eps);
  }
  int lim = interface ? S->c.lim[1] : S->c.lim[0];
  int limv = interface ? S->c.lim[3] : S->c.lim[2];
  if (S->c.model == ECGO_MODEL_EULER) {
    out->rho[0] = ecgo_limiter(lim, s1.rho[0], s2.rho[0]);
    out->p[0] = ecgo_limiter(lim, s1.p[0], s2.p[0]);
    for (int d = 0; d < 3; d++) out->u[d] = ecgo_limiter(lim, s1.u[d], s2.u[d]);
    return;
  }
  for (int k = 0; k < S->np; k++) {
    out->alpha[k] = ecgo_limiter(limv, s1.alpha[k], s2.alpha[k]);
    out->rho[k] = ecgo_limiter(lim, s1.rho[k], s2.rho[k]);
    out->p[k] = ecgo_limiter(lim, s1.p[k], s2.p[k]);
  }
  for (int d = 0; d < 3; d++) out->u[d] = ecgo_limiter(lim, s1.u[d], s2.u[d]);
}

/* Reflecting boundary: ModUEq::solveRiemannWall src/Models/UEq/ModUEq.cpp:452-492 and
 * ModEuler::solveRiemannWall src/Models/Euler/ModEuler.cpp:368-409 on the face-frame state. */
static void riemann_wall(ecgo_sim* S, const OSt* b, double dxL, double* dtMax, OFlux* out) {
  double uL, cL, pL, rhoL;
  int euler = (S->c.model == ECGO_MODEL_EULER);
  if (euler) {
    uL = b->ph[0].u[0]; pL = b->ph[0].p; rhoL = b->ph[0].rho; cL = b->ph[0].c;
  } else {
    uL = b->m.u[0]; cL = b->m.cF; pL = b->m.p; rhoL = b->m.rho;
  }
  double sL = omin(uL - cL, -uL - cL);
  if (fabs(sL) > 1.e-3) *dtMax = omin(*dtMax, 1. * dxL / fabs(sL));
  double pStar = euler ? rhoL * uL * (uL - sL) + pL : rhoL * (uL - sL) * uL + pL;
  memset(out, 0, sizeof(*out));
  out->mom[0] = pStar;
}

static void extrapolate_side(ecgo_sim* S, OSt* b, const OSlope* sl, double dist) {
  /* Phase::extrapolate / MixUEq::extrapolate without the clamps of the internal faces
   * (BoundCondWallO2Cartesian::solveRiemann src/BoundConds/BoundCondWallO2Cartesian.cpp:120-131) */
  if (S->c.model == ECGO_MODEL_EULER) {
    OPh* ph = &b->ph[0];
    ph->rho += sl->rho[0] * dist;
    ph->p += sl->p[0] * dist;
    for (int d = 0; d < 3; d++) ph->u[d] = ph->u[d] + sl->u[d] * dist;
    return;
  }
  for (int k = 0; k < S->np; k++) {
    OPh* ph = &b->ph[k];
    ph->alpha += sl->alpha[k] * dist;
    ph->rho += sl->rho[k] * dist;
    ph->p += sl->p[k] * dist;
  }
  for (int d = 0; d < 3; d++) b->m.u[d] = b->m.u[d] + sl->u[d] * dist;
}

static void extrapolate(ecgo_sim* S, OSt* b, const OSlope* sl, double dist, double sign) {
  /* Phase::extrapolate + verifyAndCorrectPhase + verifyAndCorrectDensityMax, MixUEq::extrapolate,
   * Transport::extrapolate */
  for (int k = 0; k < S->c.ntr; k++) b->tr[k] += (sign * sl->tr[k]) * dist;
  if (S->c.model == ECGO_MODEL_EULER) {
    OPh* ph = &b->ph[0];
    ph->rho += (sign * sl->rho[0]) * dist;
    ph->p += (sign * sl->p[0]) * dist;
    for (int d = 0; d < 3; d++) ph->u[d] = ph->u[d] + (sign * sl->u[d]) * dist;
    if (ph->rho < 1.e-10) ph->rho = 1.e-10;
    eos_fix_p(&S->c.eos[0], &ph->p);
    eos_rho_max(&S->c.eos[0], &ph->rho);
    return;
  }
  if (S->c.model == ECGO_MODEL_PTUEQ) {
    /* PhasePTUEq::extrapolate + verifyAndCorrectPhase (:291: alpha in [1e-10, 1 - 1e-10]; its density and
     * pressure corrections act on values fulfillState overwrites), MixPTUEq::extrapolate (:366) */
    for (int k = 0; k < S->np; k++) {
      OPh* ph = &b->ph[k];
      ph->alpha += (sign * sl->alpha[k]) * dist;
      if (ph->alpha < 1e-10) ph->alpha = 1e-10;
      if (ph->alpha > 1. - 1e-10) ph->alpha = 1. - 1e-10;
    }
    b->m.p += (sign * sl->pm) * dist;
    b->m.T += (sign * sl->Tm) * dist;
    for (int d = 0; d < 3; d++) b->m.u[d] = b->m.u[d] + (sign * sl->u[d]) * dist;
    return;
  }
  for (int k = 0; k < S->np; k++) {
    OPh* ph = &b->ph[k];
    ph->alpha += (sign * sl->alpha[k]) * dist;
    ph->rho += (sign * sl->rho[k]) * dist;
    ph->p += (sign * sl->p[k]) * dist;
    phase_fix(S, k, ph);
    eos_rho_max(&S->c.eos[k], &ph->rho);
  }
  for (int d = 0; d < 3; d++) b->m.u[d] = b->m.u[d] + (sign * sl->u[d]) * dist;
}

/* THINC reconstruction of alpha_0 (and alpha_1 = 1 - alpha_0) at an interface cell, after the MUSCL
 * extrapolation of that side (CellInterfaceO2Cartesian::solveRiemann
 * src/Order2/CellInterfaceO2Cartesian.cpp:132-150 for the left side, :164-181 for the right side;
 * the two sides use different final expressions there, kept as they are). */
static void thinc(OSt* b, double aCell, double aOther, double aAfter, int right) {
  const double beta = 1.6, eps = 1.e-4;
  if (!((aCell >= eps) && (aCell <= 1. - eps) && ((aOther - aCell) * (aCell - aAfter) >= 1.e-8))) return;
  /* left side: neighbours (right cell, left-left cell); right side: (right-right cell, left cell) */
  double hi = right ? aAfter : aOther, lo = right ? aOther : aAfter;
  double sign = (hi - lo > 0.) ? 1. : -1.;
  double qmin = omin(hi, lo);
  double qmax = omax(hi, lo) - qmin;
  double C = (aCell - qmin + 1.e-20) / (qmax + 1.e-20);
  double B = exp(sign * beta * (2. * C - 1.));
  double A = (B / cosh(beta) - 1.) / tanh(beta);
  double na = right ? qmin + 0.5 * qmax * (1. + sign * A)
                    : qmin + 0.5 * qmax * (1. + sign * (tanh(beta) + A) / (1. + A * tanh(beta)));
  if (na < eps) na = eps;
  if (na > 1. - eps) na = 1. - eps;
  b->ph[0].alpha = na;
  b->ph[1].alpha = 1. - na;
}

static void flux_pass(ecgo_sim* S, OSt* prim, int o2, double* dtMax) {
  /* face loop of Run::solveHyperbolic :696 / solveHyperbolicO2 :627 (steps 2 and 7) */
  for (int f = 0; f < S->nfaces; f++) {
    OFace* F = &S->faces[f];
    OFlux fl;
    memset(&fl, 0, sizeof(fl));
    if (F->R < 0) {
      /* BoundCond::computeFlux / solveRiemann src/BoundConds/BoundCond.cpp:61-98 */
      OSt b = prim[F->L];
      if (F->bc == ECGO_BC_SYMMETRY) {
        if (o2) {
          /* BoundCondWallO2Cartesian::solveRiemann :111-141: extrapolate by the signed distance */
          double dG = vnorm_diff(F->pos, &S->pos[3 * F->L]);
          if (F->n[0] < 0. || F->n[1] < 0. || F->n[2] < 0.) dG = -dG;
          OSlope sl;
          memset(&sl, 0, sizeof(sl));
          local_slopes_side(S, F->L, f, &sl);
          extrapolate_side(S, &b, &sl, dG);
        }
        fulfill(S, &b);
        proj_local(vel_of(S, &b), F->n, F->t, F->b);
        riemann_wall(S, &b, S->lcfl[F->L], dtMax, &fl);
        proj_reverse(fl.mom, F->n, F->t, F->b);
      } else {
        fulfill(S, &b);
        riemann(S, &b, &b, F, S->lcfl[F->L], S->lcfl[F->L], dtMax, &fl);
      }
      double cA = F->surface / S->vol[F->L];
      acc_sub(S, &S->cons[F->L], &fl, cA, &S->s[F->L]);
      continue;
    }
    if (!o2) {
      riemann(S, &prim[F->L], &prim[F->R], F, S->lcfl[F->L], S->lcfl[F->R], dtMax, &fl);
    } else {
      /* CellInterfaceO2Cartesian::solveRiemann src/Order2/CellInterfaceO2Cartesian.cpp:101-226 */
      OSt bl = prim[F->L], br = prim[F->R];
      double dG = vnorm_diff(F->pos, &S->pos[3 * F->L]);
      double dD = vnorm_diff(F->pos, &S->pos[3 * F->R]);
      double aL = (S->c.model == ECGO_MODEL_EULER) ? 0. : bl.ph[0].alpha;
      double aR = (S->c.model == ECGO_MODEL_EULER) ? 0. : br.ph[0].alpha;
      OSlope sl;
      double aLL = 0., aRR = 0.;
      memset(&sl, 0, sizeof(sl));
      local_slopes(S, F->L, f, aL, aR, &sl, &aLL);
      extrapolate(S, &bl, &sl, dG, 1.);
      if (S->thinc) thinc(&bl, aL, aR, aLL, 0);
      memset(&sl, 0, sizeof(sl));
      local_slopes(S, F->R, f, aR, aL, &sl, &aRR);
      extrapolate(S, &br, &sl, dD, -1.);
      if (S->thinc) thinc(&br, aR, aL, aRR, 1);
      fulfill(S, &bl);
      fulfill(S, &br);
      riemann(S, &bl, &br, F, S->lcfl[F->L], S->lcfl[F->R], dtMax, &fl);
    }
    double cR = F->surface / S->vol[F->R];
    acc_add(S, &S->cons[F->R], &fl, cR, &S->s[F->R]);
    double cL = F->surface / S->vol[F->L];
    acc_sub(S, &S->cons[F->L], &fl, cL, &S->s[F->L]);
  }
}

static void solve_relaxations(ecgo_sim* S) { /* Run::solveRelaxations src/Run.cpp:771 */
  if (S->c.model != ECGO_MODEL_KAPILA) return; /* Euler and PTUEq have no relaxation (advancingProcedure :596) */
  for (int i = 0; i < S->n; i++) relaxations(S, &S->s[i]);
  for (int i = 0; i < S->n; i++) {
    correction_energy(S, &S->s[i]);
    fulfill(S, &S->s[i]);
  }
}

static void step_o1(ecgo_sim* S, double dt, double* dtMax) {
  memset(S->cons, 0, sizeof(OFlux) * (size_t)S->n);
  flux_pass(S, S->s, 0, dtMax);
  for (int i = 0; i < S->n; i++) { /* Cell::timeEvolution :286 + buildPrim :313 */
    OFlux Un;
    memset(&Un, 0, sizeof(Un));
    build_cons(S, &S->s[i], &Un);
    time_evolve(S, &S->cons[i], &Un, dt);
    build_prim(S, &S->cons[i], &S->s[i]);
    for (int k = 0; k < S->c.ntr; k++) S->s[i].tr[k] += S->cons[i].tr[k] * dt; /* Cell::timeEvolution :294-298 */
  }
  solve_relaxations(S);
}

static void step_o2(ecgo_sim* S, double dt, double* dtMax) {
  /* Run::solveHyperbolicO2 src/Run.cpp:627-692 */
  memset(S->cons, 0, sizeof(OFlux) * (size_t)S->n);
  compute_slopes(S, S->s);
  flux_pass(S, S->s, 1, dtMax);
  for (int i = 0; i < S->n; i++) { /* CellO2::predictionOrdre2 src/Order2/CellO2.cpp:111 */
    OFlux Un;
    memset(&Un, 0, sizeof(Un));
    build_cons(S, &S->s[i], &Un);
    time_evolve(S, &S->cons[i], &Un, 0.5 * dt);
    S->s2[i] = S->s[i];
    build_prim(S, &S->cons[i], &S->s2[i]);
    for (int k = 0; k < S->c.ntr; k++) /* CellO2::predictionOrdre2 :121-125 */
      S->s2[i].tr[k] = S->s[i].tr[k] + S->cons[i].tr[k] * (0.5 * dt);
    relaxations(S, &S->s2[i]);
    if (S->c.model == ECGO_MODEL_KAPILA) correction_energy(S, &S->s2[i]);
    fulfill(S, &S->s2[i]);
  }
  memset(S->cons, 0, sizeof(OFlux) * (size_t)S->n);
  compute_slopes(S, S->s2);
  flux_pass(S, S->s2, 1, dtMax);
  for (int i = 0; i < S->n; i++) {
    OFlux Un;
    memset(&Un, 0, sizeof(Un));
    build_cons(S, &S->s[i], &Un);
    time_evolve(S, &S->cons[i], &Un, dt);
    build_prim(S, &S->cons[i], &S->s[i]);
    for (int k = 0; k < S->c.ntr; k++) S->s[i].tr[k] += S->cons[i].tr[k] * dt;
  }
  solve_relaxations(S);
}

/* -------------------------------------------------------------------------------------------- API */

static ecgo_sim* create_impl(const ecgo_case* c, const double* alpha, const double* rho, const double* T,
                             const double* p, const double* u, const double* tr) {
  if (c->ntr < 0 || c->ntr > NT_MAX || (c->ntr > 0 && !tr)) return NULL;
  if ((c->model == ECGO_MODEL_PTUEQ) != (T != NULL)) return NULL;
  if (c->model == ECGO_MODEL_PTUEQ && c->nphases != 2) return NULL;
  /* ModPTUEq has no transport Riemann solver: the reference reports "solveRiemannTransportIntern not
   * available for required model" (src/Models/Model.h:185) at every face */
  if (c->model == ECGO_MODEL_PTUEQ && c->ntr > 0) return NULL;
  /* MUSCL symmetry sides set phase velocity slopes (BoundCondWallO2Cartesian::computeSlopes :92-112), which
   * PhasePTUEq does not have: the reference stops there (Phase::setU, src/Models/Phase.h:159) */
  if (c->model == ECGO_MODEL_PTUEQ && c->order == 2)
    for (int i = 0; i < 6; i++)
      if (c->bc[i] == ECGO_BC_SYMMETRY) return NULL;
  ecgo_sim* S = (ecgo_sim*)calloc(1, sizeof(ecgo_sim));
  S->c = *c;
  S->np = (c->model == ECGO_MODEL_EULER) ? 1 : c->nphases;
  S->eps = c->alpha_null ? 1.e-15 : 0.;
  S->dim = (c->nx != 1) + (c->ny != 1) + (c->nz != 1);
  S->n = c->nx * c->ny * c->nz;
  build_mesh(S);
  int n = S->n;
  S->s = (OSt*)calloc((size_t)n, sizeof(OSt));
  S->s2 = (OSt*)calloc((size_t)n, sizeof(OSt));
  S->cons = (OFlux*)calloc((size_t)n, sizeof(OFlux));
  S->slopes = (OSlope*)calloc((size_t)(S->nfaces > 0 ? S->nfaces : 1), sizeof(OSlope));
  for (int i = 0; i < n; i++) {
    OSt* st = &S->s[i];
    for (int k = 0; k < c->ntr; k++) st->tr[k] = tr[(size_t)k * n + i];
    if (c->model == ECGO_MODEL_EULER) {
      st->ph[0].rho = rho[i];
      st->ph[0].p = p[i];
      st->ph[0].alpha = 1.;
      for (int d = 0; d < 3; d++) st->ph[0].u[d] = u[d * n + i];
      euler_extended(S, &st->ph[0]);
    } else if (c->model == ECGO_MODEL_PTUEQ) {
      /* PhasePTUEq / MixPTUEq states (alpha_k; p, T, u), then Cell::completeFulfillState */
      for (int k = 0; k < S->np; k++) st->ph[k].alpha = alpha[k * n + i];
      st->m.p = p[i];
      st->m.T = T[i];
      for (int d = 0; d < 3; d++) st->m.u[d] = u[d * n + i];
      fulfill(S, st);
      st->m.E = st->m.e + 0.5 * sqnorm(st->m.u); /* MixPTUEq::computeTotalEnergy :316 */
    } else {
      for (int k = 0; k < S->np; k++) {
        st->ph[k].alpha = alpha[k * n + i];
        st->ph[k].rho = rho[k * n + i];
        st->ph[k].p = p[i];
      }
      st->m.p = p[i];
      for (int d = 0; d < 3; d++) st->m.u[d] = u[d * n + i];
      fulfill(S, st);
      st->m.E = st->m.e + 0.5 * sqnorm(st->m.u); /* MixUEq::computeTotalEnergy :166 */
    }
  }
  S->thinc = (c->order == 2) && (c->lim[2] == ECGO_LIM_THINC || c->lim[3] == ECGO_LIM_THINC);
  if (c->ptmu) { /* Mixture::computeCriticalPressure src/Models/Mixture.cpp:146 */
    const ecgo_eos* L = &c->eos[c->ptmu_liq];
    const ecgo_eos* V = &c->eos[c->ptmu_vap];
    double piL = (L->type == ECGO_EOS_IG) ? 0. : L->pinf, piV = (V->type == ECGO_EOS_IG) ? 0. : V->pinf;
    double pc = piL * (V->gamma - 1.) * V->cv - piV * (L->gamma - 1.) * L->cv;
    pc /= (L->gamma - 1.) * L->cv - (V->gamma - 1.) * V->cv;
    S->pcrit = pc;
  }
  return S;
}

ecgo_sim* ecgo_create(const ecgo_case* c, const double* alpha, const double* rho, const double* p, const double* u,
                      const double* tr) {
  return create_impl(c, alpha, rho, NULL, p, u, tr);
}

ecgo_sim* ecgo_create_ptueq(const ecgo_case* c, const double* alpha, const double* T, const double* p,
                            const double* u, const double* tr) {
  return create_impl(c, alpha, NULL, T, p, u, tr);
}

void ecgo_destroy(ecgo_sim* S) {
  if (!S) return;
  free(S->s); free(S->s2); free(S->cons); free(S->slopes);
  free(S->pos); free(S->vol); free(S->lcfl); free(S->faces); free(S->cellface);
  free(S);
}

int ecgo_step(ecgo_sim* S, int nsteps, double* dt, double* t, ecgo_stats* st) {
  for (int it = 0; it < nsteps; it++) {
    double dtMax = 1.e10; /* src/Run.cpp:406 */
    if (S->c.order == 2) step_o2(S, *dt, &dtMax);
    else step_o1(S, *dt, &dtMax);
    *t += *dt;
    *dt = S->c.cfl * dtMax; /* src/Run.cpp:439 */
  }
  if (st) *st = S->st;
  return 0;
}

void ecgo_get_transports(const ecgo_sim* S, double* tr) {
  for (int k = 0; k < S->c.ntr; k++)
    for (int i = 0; i < S->n; i++) tr[(size_t)k * S->n + i] = S->s[i].tr[k];
}

void ecgo_get(const ecgo_sim* S, double* alpha, double* rho, double* T, double* Y, double* rho_mix, double* p,
              double* E, double* u) {
  int n = S->n;
  for (int i = 0; i < n; i++) {
    const OSt* st = &S->s[i];
    if (S->c.model == ECGO_MODEL_EULER) {
      if (alpha) alpha[i] = 1.;
      if (rho) rho[i] = st->ph[0].rho;
      if (T) T[i] = st->ph[0].T;
      if (Y) Y[i] = 1.;
      if (rho_mix) rho_mix[i] = st->ph[0].rho;
      if (p) p[i] = st->ph[0].p;
      if (E) E[i] = st->ph[0].E;
      if (u)
        for (int d = 0; d < 3; d++) u[d * n + i] = st->ph[0].u[d];
      continue;
    }
    for (int k = 0; k < S->np; k++) {
      if (alpha) alpha[k * n + i] = st->ph[k].alpha;
      if (rho) rho[k * n + i] = st->ph[k].rho;
      if (T) T[k * n + i] = st->ph[k].T;
      if (Y) Y[k * n + i] = st->ph[k].Y;
    }
    if (rho_mix) rho_mix[i] = st->m.rho;
    if (p) p[i] = st->m.p;
    if (E) E[i] = st->m.E;
    if (u)
      for (int d = 0; d < 3; d++) u[d * n + i] = st->m.u[d];
  }
}

void ecgo_get_phase_pressure(const ecgo_sim* S, double* pk) {
  for (int i = 0; i < S->n; i++)
    for (int k = 0; k < S->np; k++) pk[k * S->n + i] = S->s[i].ph[k].p;
}

int ecgo_relax_pinf(const ecgo_case* c, double* alpha, double* rho, double* pk, double* pmix, int* iterations) {
  ecgo_sim S;
  memset(&S, 0, sizeof(S));
  S.c = *c;
  S.np = c->nphases;
  S.eps = c->alpha_null ? 1.e-15 : 0.;
  OSt st;
  memset(&st, 0, sizeof(st));
  for (int k = 0; k < S.np; k++) {
    st.ph[k].alpha = alpha[k];
    st.ph[k].rho = rho[k];
    st.ph[k].p = pk[k];
  }
  fulfill(&S, &st);
  relax_pinf(&S, &st);
  for (int k = 0; k < S.np; k++) {
    alpha[k] = st.ph[k].alpha;
    rho[k] = st.ph[k].rho;
    pk[k] = st.ph[k].p;
  }
  *pmix = st.m.p;
  if (iterations) *iterations = (int)S.st.newton_evals;
  return 0;
}

double ecgo_pressure_isentropic(const ecgo_eos* e, double p0, double rho0, double rho1, int alpha_null) {
  return eos_p_isentropic(e, alpha_null ? 1.e-15 : 0., p0, rho0, rho1);
}

double ecgo_density_pfinal(const ecgo_eos* e, double p0, double rho0, double p1, double* drhodp, int alpha_null) {
  return eos_rho_pfinal(e, alpha_null ? 1.e-15 : 0., p0, rho0, p1, drhodp);
}
