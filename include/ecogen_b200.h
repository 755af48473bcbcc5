/*
 * ecogen_b200 — C ABI of the B200 (sm_100a) explicit finite-volume step of ECOGEN.
 *
 * The library replaces, for Cartesian non-AMR Euler / Kapila (PUEq) / PTUEq cases, the part of the
 * reference CPU run loop that advances the solution by one time step:
 *   Run::solveHyperbolic / Run::solveHyperbolicO2 + Run::solveRelaxations
 *   (src/Run.cpp:696, :627, :771) and the dt update of Run::solver (src/Run.cpp:406-440).
 * The entry points below take plain host pointers and sizes; device memory, streams and
 * CUDA graphs belong to a context.  Calls on one context are not reentrant; independent
 * contexts may be used from different threads.
 *
 * Field layout used by upload/download (n = number of cells, cell index i + j*nx + k*nx*ny as
 * src/Meshes/MeshCartesian.cpp:141 orders cells): a caller passes an array of pointers, one per
 * field, in the order
 *   alpha_0 .. alpha_{N-1}, rho_0 .. rho_{N-1}, p, u_x, u_y, u_z, E, T_0 .. T_{M-1}  (Kapila, N phases)
 *   rho, p, u_x, u_y, u_z, E, T_0 .. T_{M-1}                                       (Euler)
 *   alpha_0, alpha_1, rho_0, rho_1, p, u_x, u_y, u_z, E, temperature               (PTUEq)
 * each pointing at n doubles, M = ecg_case.ntransports.  For Kapila, p is the mixture pressure
 * sum_k alpha_k p_k as the reference writes it ("Pressure_Mixture", src/Models/UEq/MixUEq.cpp:201);
 * E is the specific total energy ("Total_energy_Mixture"); T_j are the passive transports.  The
 * temperature-pressure-velocity equilibrium model (PTUEq, src/Models/PTUEq) has one pressure and one
 * temperature; its phase densities are computeDensity(p, temperature) of each EOS, so an upload reads
 * alpha_k, p, u, E and the temperature and a download returns the densities it derives.
 */
#ifndef ECOGEN_B200_H
#define ECOGEN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  ECG_OK = 0,
  ECG_ERR_INVALID = 1,      /* bad argument (null pointer, size mismatch, bad enum) */
  ECG_ERR_UNSUPPORTED = 2,  /* case outside this library's scope (AMR, unstructured, add-phys, ...) */
  ECG_ERR_CUDA = 3,         /* a CUDA runtime call failed; see ecg_last_error() */
  ECG_ERR_XML = 4,          /* malformed or incomplete case input (reference: ErrorXML*) */
  ECG_ERR_PHYSICS = 5,      /* a physics check failed during the step (reference: errors vector) */
  ECG_ERR_NOMEM = 6,        /* device or host allocation failed */
  ECG_ERR_TOO_LARGE = 7,    /* size above a stated maximum */
  ECG_ERR_TIMEOUT = 8       /* a bounded device-side wait gave up */
} ecg_status;

/* Flow models: Kapila = PressureVelocityEq (ModPUEq), Euler (ModEuler), PTUEq =
 * TemperaturePressureVelocityEq (ModPTUEq: two IG/SG phases, no transports, first-order symmetry sides). */
enum { ECG_MODEL_KAPILA = 0, ECG_MODEL_EULER = 1, ECG_MODEL_PTUEQ = 2 };
enum { ECG_EOS_IG = 0, ECG_EOS_SG = 1, ECG_EOS_NASG = 2 };
enum {
  ECG_LIM_NONE = 0, ECG_LIM_MINMOD = 1, ECG_LIM_VANLEER = 2, ECG_LIM_VANALBADA = 3,
  ECG_LIM_SUPERBEE = 4, ECG_LIM_MC = 5, ECG_LIM_THINC = 6
};
/* Boundary condition of one side of the domain (initialConditions.xml <boundCond type=...>):
 * nonReflecting (BoundCondNonReflecting), or symmetry -- also what an inviscid "wall" is
 * (BoundCondSymmetry / BoundCondSymmetryO2Cartesian, src/InputOutput/Input.cpp:1146-1180). */
enum { ECG_BC_NONREFLECTING = 0, ECG_BC_SYMMETRY = 1 };
#define ECG_MAX_PHASES 3

/* One EOS (src/Eos/EosIG.h, EosSG.h, EosNASG.h parameters). */
typedef struct {
  int32_t type;                 /* ECG_EOS_* */
  double gamma, pinf, b, cv, eref, sref;
} ecg_eos;

/* One zone of mesh.xml <meshStretching> along an axis (stretchZone, src/Meshes/stretchZone.cpp:45-66):
 * ncells cells from start to end whose sizes grow geometrically by factor (uniform when |factor - 1| <
 * 1e-6).  The zones of an axis follow one another from 0 to the axis length. */
#define ECG_MAX_STRETCH_ZONES 8
typedef struct {
  double start, end, factor;
  int32_t ncells;
} ecg_stretch_zone;

/* A case as the four ECOGEN XML files describe it (Input::readInputXML src/InputOutput/Input.cpp:54). */
typedef struct {
  int32_t model;                /* ECG_MODEL_* */
  int32_t nphases;              /* Kapila: 2..3 ; Euler: 1 ; PTUEq: 2 */
  int32_t alpha_null;           /* model.xml alphaNull */
  int32_t order;                /* 1 first order, 2 MUSCL-Hancock (secondOrder) */
  int32_t limiter[4];           /* global, interface, global vol.-fraction, interface vol.-fraction */
  int32_t ncells[3];            /* nx, ny, nz (mesh.xml numberCells) */
  double length[3];             /* lx, ly, lz (mesh.xml dimensions) */
  double cfl;                   /* main.xml computationControl CFL */
  int32_t time_iterations;      /* 1: stop after max_iterations ; 0: stop at total_time */
  int32_t max_iterations;
  double total_time;
  int32_t ptmu;                 /* p-T-mu relaxation (model.xml <relaxation type="PTMu">) */
  int32_t ptmu_liquid, ptmu_vapor;
  ecg_eos eos[ECG_MAX_PHASES];
  int32_t bc[6];                /* ECG_BC_* of the sides Xm, Xp, Ym, Yp, Zm, Zp (MeshCartesian::assignLimits) */
  int32_t ntransports;          /* passive transports (model.xml numberTransports, src/Transport), 0..2 */
  int32_t pt_relaxation;        /* model.xml <relaxation type="PT">: analytic p-T relaxation (RelaxationPT) */
  int32_t nstretch[3];          /* mesh.xml meshStretching zones per axis (0: cells of length / ncells);
                                   the zones' cells add up to ncells[axis] */
  ecg_stretch_zone stretch[3][ECG_MAX_STRETCH_ZONES];
} ecg_case;

/* Counters of one ecg_step call (replace the reference's errors / warnings vectors). */
typedef struct {
  int64_t cell_updates;         /* cells x steps advanced */
  int64_t relax_calls;          /* pressure relaxations performed (not skipped) */
  int64_t newton_evals;         /* Newton evaluations summed over relaxations */
  int64_t newton_fallback;      /* relaxations that hit the iteration cap (interface pressure used) */
  int64_t newton_max;           /* largest Newton evaluation count of one relaxation */
  int64_t seeded;               /* relaxations started from the learned seed */
  int64_t seed_rejected;        /* learned seeds rejected (plain start used) */
  int64_t ptmu_errors;          /* p-T-mu solves above 50 iterations (reference: error, run stops) */
  int64_t nonfinite_cells;      /* cells whose state became NaN/inf */
  int64_t newton_hist[16];      /* histogram of Newton evaluations: bins 1..15, 16+ in [15] */
  /* p-T-mu relaxation (RelaxationPTMu::relaxation): solves that ran the saturation Newton on p*, their
   * Newton iterations (sum, largest, histogram as newton_hist), and the T_sat(p) solves of
   * Mixture::computeTsat they made (pure-phase tests included) with those solves' iterations */
  int64_t ptmu_solves;
  int64_t ptmu_outer_iters;
  int64_t ptmu_outer_max;
  int64_t ptmu_tsat_calls;
  int64_t ptmu_tsat_iters;
  int64_t ptmu_tsat_max;
  int64_t ptmu_outer_hist[16];
  int64_t ptmu_seeded;          /* saturation solves whose T_sat Newton started from a seed (the learned
                                   network's, or the cell's previous solve with the warm start) */
  int64_t ptmu_seed_rejected;   /* learned (p*, T) seeds rejected (plain start) */
  int64_t bounds_violations;    /* bounds-checked builds (-DECG_BOUNDS_CHECK) only: device accesses outside
                                   their buffer, counted and skipped; always 0 in the regular build */
  int64_t staging_timeouts;     /* face-kernel warps whose wait for a TMA staging copy ran out (the step
                                   then returns ECG_ERR_CUDA); 0 in a healthy run */
} ecg_step_stats;

typedef struct ecg_ctx ecg_ctx;
typedef struct ecg_input ecg_input;

/* ------------------------------------------------------------------ status / version */
const char* ecg_status_str(ecg_status s);
/* Text of the last error seen on this thread (CUDA error string, XML path, ...). */
const char* ecg_last_error(void);
int ecg_version(void);

/* ------------------------------------------------------------------ case input (XML) */
/* Reads <case_dir>/{main,mesh,model,initialConditions}.xml and the EOS files they name from
 * <eos_dir> (ECOGEN reads them from <work>/libEOS, Input::inputEOS src/InputOutput/Input.cpp:865).
 * Replaces Input::readInputXML for the Cartesian Euler / Kapila cases this library runs. */
ecg_status ecg_input_read(const char* case_dir, const char* eos_dir, ecg_input** out);
void ecg_input_free(ecg_input* in);
ecg_status ecg_input_case(const ecg_input* in, ecg_case* out);
/* Run name (main.xml <run>) and output format; strings are owned by the input. */
const char* ecg_input_run_name(const ecg_input* in);
/* Print control of main.xml: iterFreq (iteration mode) or timeFreq (physical-time mode). */
ecg_status ecg_input_print_control(const ecg_input* in, int32_t* iter_freq, double* time_freq);
/* Output and restart control of main.xml: <outputMode binary precision> (precision 0 = the stream
 * default of 6 significant digits) and <restartSimulation restartFileNumber> (0 = no restart). */
ecg_status ecg_input_output_control(const ecg_input* in, int32_t* binary, int32_t* precision, int32_t* restart_file);
/* EOS file name of phase k (model.xml <EOS name>), used for output field names. */
const char* ecg_input_eos_name(const ecg_input* in, int32_t k);
/* Fills the initial primitive fields on the host, domain by domain in document order
 * (GeometricalDomain::fillIn src/Geometries/GeometricalDomain.cpp:64).  Field layout as above. */
ecg_status ecg_input_fill(const ecg_input* in, double* const* fields, int64_t ncells);

/* Completes fields read from a result file the way a restart does (Run::restartSimulation src/Run.cpp:345):
 * Kapila: every phase takes the mixture pressure and is corrected (ModPUEq::fulfillStateRestart
 * src/Models/PUEq/ModPUEq.cpp:76, PhaseUEq::verifyAndCorrectPhase), then the total energy is rebuilt
 * (Cell::completeFulfillState src/Order1/Cell.cpp:344); Euler: the total energy only.  alpha_k and rho_k
 * are corrected in place and E is overwritten; p and u are kept.  PTUEq: the phase densities are recomputed
 * from p and the temperature (ModPTUEq::fulfillState) and E is rebuilt.  Host-only, no GPU work. */
ecg_status ecg_restart_fill(const ecg_case* c, double* const* fields, int64_t ncells);

/* ------------------------------------------------------------------ one case on one GPU */
/* Creates a context on the current CUDA device: device state, stream, dt accumulator.
 * Replaces Run::initialize's mesh and cell allocation (src/Run.cpp:69-160). */
ecg_status ecg_create(const ecg_case* c, ecg_ctx** out);
void ecg_destroy(ecg_ctx* ctx);
/* Host -> device copy of the primitive fields (initial condition or restart); completes the
 * thermodynamic state like Cell::completeFulfillState (src/Order1/Cell.cpp:344). */
ecg_status ecg_upload_prim(ecg_ctx* ctx, const double* const* fields, int64_t ncells);
/* Device -> host copy of the fields as the reference writes them. */
ecg_status ecg_download_prim(ecg_ctx* ctx, double* const* fields, int64_t ncells);
/* Per-phase temperature and mass fraction (reference output "F<k>_Temperature" / "F<k>_Mass fraction");
 * T and Y each receive nphases*n doubles, phase-major. */
ecg_status ecg_download_derived(ecg_ctx* ctx, double* T, double* Y, int64_t ncells);
/* Advances nsteps time steps.  *dt is the step to take first (1e-15 before the first step,
 * src/Run.cpp:38) and on return the next one, cfl*dtMax (src/Run.cpp:439); *t accumulates.
 * stats may be NULL.  Returns ECG_ERR_PHYSICS if a physics check failed (the state is kept). */
ecg_status ecg_step(ecg_ctx* ctx, int32_t nsteps, double* dt, double* t, ecg_step_stats* stats);
/* Diagnostic form of ecg_step: launches every kernel separately (no graph) and adds each one's
 * device time, measured with CUDA events on the context's stream, to kernel_ms[0..2]:
 * [0] first-order or MUSCL predictor pass, [1] MUSCL corrector pass, [2] time-step update. */
ecg_status ecg_step_profiled(ecg_ctx* ctx, int32_t nsteps, double* dt, double* t, ecg_step_stats* stats,
                             double* kernel_ms);
/* The same per kernel, kernel_ms[0..8]: pass 1's X, Y and Z face kernels and its cell kernel, pass 2's
 * (MUSCL corrector) the same, then the time-step update.  In fused form a pass is one kernel, whose
 * time goes to its cell-kernel slot ([3] or [7]); entries of kernels that do not run stay 0. */
ecg_status ecg_step_profiled_kernels(ecg_ctx* ctx, int32_t nsteps, double* dt, double* t, ecg_step_stats* stats,
                                     double* kernel_ms);
/* Form of the Kapila step passes on 2D and 3D meshes.  ECG_FORM_SPLIT (the default where it applies):
 * per axis a face-flux kernel writing every face's flux to a face array of the context, then one cell
 * kernel accumulating them in the reference's face order; ECG_FORM_FUSED: one kernel per pass that
 * stages a tile per axis in shared memory.  Both compute every flux with the same arithmetic and
 * accumulate in the same order, so they give the same bits.  1D cases, passive transports and the Euler
 * and PTUEq models run fused only (ECG_ERR_UNSUPPORTED for ECG_FORM_SPLIT). */
enum { ECG_FORM_FUSED = 0, ECG_FORM_SPLIT = 1 };
ecg_status ecg_set_step_form(ecg_ctx* ctx, int32_t form);
int32_t ecg_step_form(const ecg_ctx* ctx);
/* How the split form's face kernels stage their cell tiles in shared memory.  ECG_STAGING_TMA (the
 * default): one tensor copy (cp.async.bulk.tensor through a tensor map of the state) per block, where
 * the layout allows one (an even number of cells along x); elsewhere, and with ECG_STAGING_PLAIN, the
 * threads load the tiles themselves.  Both give the same bits. */
enum { ECG_STAGING_PLAIN = 0, ECG_STAGING_TMA = 1 };
ecg_status ecg_set_face_staging(ecg_ctx* ctx, int32_t staging);
/* The staging the next split-form step uses: ECG_STAGING_TMA only where the maps exist. */
int32_t ecg_face_staging(const ecg_ctx* ctx);
/* Runs the reference time loop to its stop condition (iterations or total time), in chunks
 * captured as CUDA graphs. */
ecg_status ecg_run(ecg_ctx* ctx, double* dt, double* t, int32_t* iterations, ecg_step_stats* stats);
/* Number of cells, phases and the CUDA stream of a context. */
int64_t ecg_ncells(const ecg_ctx* ctx);
void* ecg_stream(const ecg_ctx* ctx);
/* Newton iteration cap (default 100, RelaxationP::NewtonRaphson src/Relaxations/RelaxationP.cpp:66);
 * a lower cap forces the interface-pressure fallback and is used to test that path. */
ecg_status ecg_set_newton_cap(ecg_ctx* ctx, int32_t cap);
/* What a pressure relaxation that reaches the Newton cap does: ECG_CAP_FALLBACK (the reference's
 * interface pressure, the default) or ECG_CAP_ACCEPT (keep the last Newton iterate).  A measurement aid:
 * with ECG_CAP_ACCEPT and a cap of 1 every relaxation costs one evaluation, what it would cost if started
 * at p*, so the step time is the ceiling of any seed's gain (the fields then differ from the plain
 * iteration's by the unconverged cells' residuals). */
enum { ECG_CAP_FALLBACK = 0, ECG_CAP_ACCEPT = 1 };
ecg_status ecg_set_newton_cap_mode(ecg_ctx* ctx, int32_t mode);
/* Device-resident variants for callers that keep their own device buffers: fields[] point at
 * device memory laid out as above.  Run on the context's stream. */
ecg_status ecg_upload_prim_device(ecg_ctx* ctx, const double* const* dfields, int64_t ncells);
ecg_status ecg_download_prim_device(ecg_ctx* ctx, double* const* dfields, int64_t ncells);

/* One time step on device buffers the caller owns, allocating no device memory.  This entry point
 * has no counterpart in the reference (whose CPU run loop owns its memory): it is for callers that
 * cannot call cudaMalloc, e.g. codes whose device memory all comes from their own allocator or pool,
 * or that must not allocate inside their time loop.  Instead of a context it uses one fixed
 * __device__ scratch array of the library (about 10 MB per GPU that loads the library, held until
 * the process exits) for the MUSCL half-step state, distance tables, dt scalars and counters.
 *   - At most ECG_NOALLOC_MAX_CELLS cells; larger cases return ECG_ERR_TOO_LARGE.
 *   - state_in / state_out: device arrays in the library's device layout, fields of ncells doubles
 *     back to back: alpha_0..alpha_{N-1}, rho_0..rho_{N-1}, p, u_0..u_{dim-1}, E (Kapila) or
 *     rho, p, u_0..u_{dim-1}, E (Euler), where dim counts the axes with more than one cell; this is
 *     what ecg_upload_prim stores.  The two ranges must not overlap (ECG_ERR_INVALID).
 *   - The case is checked as ecg_create checks it; PTUEq cases and passive transports are refused
 *     with ECG_ERR_UNSUPPORTED.
 *   - dt: the step to take; *dt_next (optional) receives cfl * dtMax.  stats may be NULL.
 *   - stream: a cudaStream_t (NULL = legacy default stream); the call returns after the step ran.
 *   - The first call on a device does the set-up: it looks up the scratch's device address, and with
 *     CUDA's lazy module loading (the default) that first touch also loads the library's device code,
 *     which is when the scratch array itself is allocated.  Make that first call before the time loop
 *     and before any stream capture (or set CUDA_MODULE_LOADING=EAGER); later calls allocate nothing.
 *     All calls share the scratch and the last call's contents stay in it; every call re-initialises
 *     what must start at zero.  Calls that overlap on the GPU (other streams, other host threads)
 *     race on the scratch and must be serialised by the caller. */
#define ECG_NOALLOC_MAX_CELLS 65536
ecg_status ecg_step_noalloc(const ecg_case* c, const double* state_in, double* state_out, double dt, double* dt_next,
                            ecg_step_stats* stats, void* stream);

/* ------------------------------------------------------------------ learned relaxation seed */
/* A 9 -> 64 -> 64 -> 1 (or nin -> h -> h -> 1) GELU MLP whose output seeds the pressure-relaxation
 * Newton iteration (RelaxationP::NewtonRaphson start, src/Relaxations/RelaxationPInfinite.cpp:58-63).
 * Newton still iterates to |f| <= 1e-10, so the plain iteration remains the judge. */
#define ECG_MLP_MAX_IN 16
#define ECG_MLP_HIDDEN 64
typedef struct {
  int32_t n_in;                 /* input features (<= ECG_MLP_MAX_IN) */
  int32_t hidden;               /* must be ECG_MLP_HIDDEN */
  const float* w1;              /* [hidden][n_in] */
  const float* b1;              /* [hidden] */
  const float* w2;              /* [hidden][hidden] */
  const float* b2;              /* [hidden] */
  const float* w3;              /* [n_out][hidden] */
  float b3;
  float in_shift[ECG_MLP_MAX_IN], in_scale[ECG_MLP_MAX_IN]; /* feature normalisation */
  float out_shift, out_scale;   /* target de-normalisation */
  /* A second output (n_out = 2; 0 reads as 1): its bias and de-normalisation.  The two-output network
   * (8 -> 64 -> 64 -> 2) seeds the p-T-mu saturation solve with (p*, T_sat(p*)). */
  int32_t n_out;
  float b3_1, out_shift_1, out_scale_1;
} ecg_mlp;
/* Installs (copies) the weights; NULL restores the plain starts.
 * Pressure relaxation (n_in = 3 N, n_out = 1): the step makes the plain iteration's first Newton
 * evaluation for every cell and starts the cells it leaves unconverged again from the network's seed
 * (kept only when finite and inside the bracket of the phase pressures); Newton still stops at
 * |f| <= 1e-10.
 * p-T-mu relaxation (a case with ptmu; n_in = 8, n_out = 2): what the network starts is set by
 * ecg_set_ptmu_seed; a seed that is not finite and positive (a p* at or above the critical pressure)
 * is rejected (plain start, counted).  Both Newton loops still stop at |f| <= 1e-10, so the plain
 * iteration remains the judge; the pressure relaxation runs plain. */
ecg_status ecg_set_seed_model(ecg_ctx* ctx, const ecg_mlp* mlp);
/* What the learned seed of a p-T-mu case starts.  ECG_PTMU_SEED_T (the default): the T_sat(p) Newton
 * solves (Mixture::computeTsat, cold start 0.1 B / C at src/Models/Mixture.cpp:85) -- the first from
 * the network's T_sat(p*), each later one from the previous solve's result -- while the saturation
 * Newton on p* starts at sum_k alpha_k p_k as in the reference (RelaxationPTMu.cpp:129).
 * ECG_PTMU_SEED_P_T: the saturation Newton starts from the network's p* as well. */
enum { ECG_PTMU_SEED_T = 0, ECG_PTMU_SEED_P_T = 1 };
ecg_status ecg_set_ptmu_seed(ecg_ctx* ctx, int32_t mode);
/* p-T-mu warm start (no network): with on = 1 the context keeps, per cell, the T_sat of the cell's last
 * saturation solve, and the next solve of that cell starts its T_sat(p) Newton there (then at the previous
 * iteration's T_sat) instead of at the cold start 0.1 B / C; the saturation Newton on p* keeps the
 * reference's start.  Every loop still stops at |f| <= 1e-10: the fields agree with the plain solve to
 * that residual, not bit for bit.  A seed model, when installed, takes precedence.  An upload clears the
 * record (the next solves start cold).  on = 0 (the default) frees the per-cell record and restores the
 * reference's starts. */
ecg_status ecg_set_ptmu_warm_start(ecg_ctx* ctx, int32_t on);
/* Records up to max_pairs (features, targets) pairs from the relaxations of the next ecg_step calls
 * into an internal device buffer; ecg_fetch_pairs copies them out.  Pressure relaxation: 3 N features,
 * one target (the relaxed pressure's place in the bracket of the phase pressures), relaxations that
 * took at least min_evals Newton evaluations (1 = all).  p-T-mu relaxation: 8 features, two targets
 * (ln p*, T_sat(p*)) of every saturation solve (min_evals: at least that many p* iterations). */
ecg_status ecg_record_pairs(ecg_ctx* ctx, int64_t max_pairs, int32_t min_evals);
ecg_status ecg_fetch_pairs(ecg_ctx* ctx, float* features, float* targets, int64_t* count);

/* ------------------------------------------------------------------ MLP training on the GPU */
typedef struct ecg_trainer ecg_trainer;
ecg_status ecg_trainer_create(int32_t n_in, int32_t hidden, uint64_t seed, ecg_trainer** out);
/* The same with n_out outputs (1 or 2): targets y are then n x n_out, the loss sums the outputs' mean
 * squared errors, and ecg_trainer_grad's gw3 / gb3 hold n_out x hidden and n_out values. */
ecg_status ecg_trainer_create_n(int32_t n_in, int32_t n_out, int32_t hidden, uint64_t seed, ecg_trainer** out);
void ecg_trainer_destroy(ecg_trainer* tr);
/* One AdamW epoch over (x, y) (host arrays, n rows), minibatches of `batch`; returns mean loss. */
ecg_status ecg_trainer_epoch(ecg_trainer* tr, const float* x, const float* y, int64_t n, int32_t batch, float lr,
                             float weight_decay, float* mean_loss);
/* Forward + backward of one batch: loss and the gradients of every parameter (for gradient checks). */
ecg_status ecg_trainer_grad(ecg_trainer* tr, const float* x, const float* y, int32_t n, float* loss, float* gw1,
                            float* gb1, float* gw2, float* gb2, float* gw3, float* gb3);
ecg_status ecg_trainer_forward(ecg_trainer* tr, const float* x, int32_t n, float* yhat);
/* Current parameters (host copies owned by the trainer) in ecg_mlp form, with normalisation fields
 * set from the last ecg_trainer_set_norm call. */
ecg_status ecg_trainer_export(ecg_trainer* tr, ecg_mlp* out);
ecg_status ecg_trainer_import(ecg_trainer* tr, const ecg_mlp* in);
ecg_status ecg_trainer_set_norm(ecg_trainer* tr, const float* in_shift, const float* in_scale, float out_shift,
                                float out_scale);
/* De-normalisation of the second output of a two-output trainer (out_shift_1 / out_scale_1). */
ecg_status ecg_trainer_set_norm_out1(ecg_trainer* tr, float out_shift, float out_scale);

/* ------------------------------------------------------------------ batched independent cases */
/* Many independent 1D cases of uneven cell counts advanced together by one persistent kernel per
 * pass that pulls (case, tile) work items from a device queue; each case keeps its own dt
 * (segmented min-reduction) and time.  All cases must share model, phases, EOS, order and
 * limiters; their cell counts, lengths, CFL and initial states differ.  The reference runs such
 * cases one after another (src/main.cpp:82-133). */
typedef struct ecg_batch ecg_batch;
ecg_status ecg_batch_create(const ecg_case* cases, int32_t ncases, ecg_batch** out);
void ecg_batch_destroy(ecg_batch* b);
/* fields[f] points at sum(ncells) doubles: case 0's cells, then case 1's, ... */
ecg_status ecg_batch_upload_prim(ecg_batch* b, const double* const* fields, int64_t total_cells);
ecg_status ecg_batch_download_prim(ecg_batch* b, double* const* fields, int64_t total_cells);
/* Advance every case nsteps steps (each with its own dt); dt/t arrays of ncases (may be NULL). */
ecg_status ecg_batch_step(ecg_batch* b, int32_t nsteps, double* dt, double* t, ecg_step_stats* stats);
ecg_status ecg_batch_set_seed_model(ecg_batch* b, const ecg_mlp* mlp);
/* Tile = threads per block (64, 128 or 256; 0 = autotuned); a work item covers tile - 1 cells of one
 * case, so its tile faces take one round of the block.  threads must be 0 or equal to tile. */
ecg_status ecg_batch_set_shape(ecg_batch* b, int32_t tile, int32_t threads);
ecg_status ecg_batch_autotune(ecg_batch* b, int32_t* tile, int32_t* threads);
int64_t ecg_batch_total_cells(const ecg_batch* b);
/* The cudaStream_t every batch operation is ordered on (for events around ecg_batch_step). */
void* ecg_batch_stream(const ecg_batch* b);

#ifdef __cplusplus
}
#endif
#endif
