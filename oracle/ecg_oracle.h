/*
 * CPU restatement of ECOGEN's explicit finite-volume time step on Cartesian
 * meshes (Euler and Kapila/PUEq models, HLLC, first order or MUSCL-Hancock,
 * IG/SG/NASG EOS, infinite pressure relaxation and p-T-mu relaxation).
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA path is checked
 * against; it is never linked into the product library.  Its parity with the
 * reference itself is pinned by tests that run the reference binary built from
 * the reference sources (oracle/Makefile, oracle/refrun.py) on the same cases.
 *
 * (The temperature-pressure-velocity equilibrium model, PTUEq, is restated too.)
 *
 * Layout of state arrays passed across this interface (n = number of cells,
 * cell index i + j*nx + k*nx*ny, reference src/Meshes/MeshCartesian.cpp:141):
 *   alpha[k*n + c], rho[k*n + c] for k < nphases, p[c], u[d*n + c] (d < 3), E[c], tr[k*n + c] (k < ntr)
 */
#ifndef ECG_ORACLE_H
#define ECG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ECGO_EOS_IG = 0, ECGO_EOS_SG = 1, ECGO_EOS_NASG = 2 };
enum { ECGO_LIM_NONE = 0, ECGO_LIM_MINMOD = 1, ECGO_LIM_VANLEER = 2, ECGO_LIM_VANALBADA = 3,
       ECGO_LIM_SUPERBEE = 4, ECGO_LIM_MC = 5, ECGO_LIM_THINC = 6 };
enum { ECGO_MODEL_KAPILA = 0, ECGO_MODEL_EULER = 1, ECGO_MODEL_PTUEQ = 2 };
/* Boundary conditions per side Xm, Xp, Ym, Yp, Zm, Zp: non-reflecting, or symmetry (also an
 * inviscid "wall", src/InputOutput/Input.cpp:1146-1180). */
enum { ECGO_BC_NONREFLECTING = 0, ECGO_BC_SYMMETRY = 1 };

typedef struct {
  int type;
  double gamma, pinf, b, cv, eref, sref;
} ecgo_eos;

/* One zone of mesh.xml meshStretching (stretchZone, src/Meshes/stretchZone.h). */
#define ECGO_MAX_STRETCH 8
typedef struct {
  double start, end, factor;
  int ncells;
} ecgo_stretch;

typedef struct {
  int model;       /* ECGO_MODEL_* */
  int nphases;     /* 1 for Euler, 2..3 for Kapila */
  int alpha_null;  /* model.xml alphaNull */
  int order;       /* 1 = first order, 2 = MUSCL-Hancock */
  int nx, ny, nz;
  double lx, ly, lz;
  double cfl;
  int lim[4];      /* global, interface, global volume-fraction, interface volume-fraction */
  int ptmu, ptmu_liq, ptmu_vap;
  ecgo_eos eos[3];
  int bc[6];       /* ECGO_BC_* per side */
  int ntr;         /* passive transports (0..4) */
  int pt;          /* model.xml <relaxation type="PT">: analytic p-T relaxation after the pressure one */
  int nstretch[3]; /* stretch zones per axis (0: uniform cells of l / n) */
  ecgo_stretch stretch[3][ECGO_MAX_STRETCH];
} ecgo_case;

typedef struct {
  long long relax_calls;      /* PInfinite relaxations performed (not skipped) */
  long long newton_evals;     /* Newton evaluations summed over calls */
  long long newton_fallback;  /* calls that reached 100 iterations */
  long long newton_max;       /* largest evaluation count of one call */
  long long ptmu_errors;      /* p-T-mu loops that exceeded 50 iterations */
} ecgo_stats;

typedef struct ecgo_sim ecgo_sim;

/* Build a simulation from the initial primitive state (per-phase alpha, rho,
 * mixture pressure given to every phase, mixture velocity); total energy is
 * completed as in Cell::completeFulfillState (src/Order1/Cell.cpp:344). */
ecgo_sim* ecgo_create(const ecgo_case* c, const double* alpha, const double* rho, const double* p, const double* u,
                      const double* tr);
/* Temperature-pressure-velocity equilibrium model (ModPTUEq, two IG/SG phases): the initial state is
 * alpha_k and the mixture p, T and velocity (src/Models/PTUEq/PhasePTUEq.cpp:42, MixPTUEq.cpp:44); phase
 * densities follow from (p, T).  ecgo_get returns the mixture temperature as every phase's T. */
ecgo_sim* ecgo_create_ptueq(const ecgo_case* c, const double* alpha, const double* T, const double* p,
                            const double* u, const double* tr);
void ecgo_destroy(ecgo_sim* s);
/* Advance nsteps time steps.  *dt is the step to take first (1e-15 at start,
 * src/Run.cpp:38); on return it holds the next step cfl*dtMax (src/Run.cpp:439). */
int ecgo_step(ecgo_sim* s, int nsteps, double* dt, double* t, ecgo_stats* st);
/* Output fields as the reference writes them: alpha_k, rho_k, T_k, Y_k,
 * mixture density, mixture pressure (sum alpha_k p_k), total energy, velocity. */
void ecgo_get(const ecgo_sim* s, double* alpha, double* rho, double* T, double* Y, double* rho_mix, double* p,
              double* E, double* u);
/* Passive transport values tr[k*n + c]. */
void ecgo_get_transports(const ecgo_sim* s, double* tr);
/* Per-phase pressures and the mixture internal energy (diagnostics). */
void ecgo_get_phase_pressure(const ecgo_sim* s, double* pk);

/* Single-cell kernels exposed for function-level tests. */
int ecgo_relax_pinf(const ecgo_case* c, double* alpha, double* rho, double* pk, double* pmix, int* iterations);
double ecgo_pressure_isentropic(const ecgo_eos* e, double p0, double rho0, double rho1, int alpha_null);
double ecgo_density_pfinal(const ecgo_eos* e, double p0, double rho0, double p1, double* drhodp, int alpha_null);
double ecgo_limiter(int kind, double s1, double s2);

#ifdef __cplusplus
}
#endif
#endif
