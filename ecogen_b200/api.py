"""Python binding of the C ABI in ``include/ecogen_b200.h`` (ctypes over ``ecogen_b200/libecg.so``).

The library is the product; this module only marshals arguments.  Loading fails loudly when the
shared library has not been built (``python -m ecogen_b200.build``) — there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("ECG_LIB", os.path.join(HERE, "libecg.so"))

ECG_OK = 0
STATUS = {0: "ok", 1: "invalid argument", 2: "unsupported case", 3: "CUDA error", 4: "case input error",
          5: "physics check failed", 6: "out of memory", 7: "size above the stated maximum", 8: "device wait timed out"}
MODEL_KAPILA, MODEL_EULER, MODEL_PTUEQ = 0, 1, 2
FORM_FUSED, FORM_SPLIT = 0, 1
STAGING_PLAIN, STAGING_TMA = 0, 1
PTMU_SEED_T, PTMU_SEED_P_T = 0, 1
CAP_FALLBACK, CAP_ACCEPT = 0, 1
EOS_CODE = {"IG": 0, "SG": 1, "NASG": 2}
BC_CODE = {"NONREFLECTING": 0, "SYMMETRY": 1, "WALL": 1}
LIM_CODE = {None: 0, "NONE": 0, "MINMOD": 1, "VANLEER": 2, "VANALBADA": 3, "SUPERBEE": 4, "MC": 5, "THINC": 6}


class EcgError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str):
        super().__init__(f"{where}: {STATUS.get(status, status)}: {detail}")
        self.status = status


class Eos(C.Structure):
    _fields_ = [("type", C.c_int32), ("gamma", C.c_double), ("pinf", C.c_double), ("b", C.c_double),
                ("cv", C.c_double), ("eref", C.c_double), ("sref", C.c_double)]


MAX_STRETCH_ZONES = 8


class StretchZone(C.Structure):
    _fields_ = [("start", C.c_double), ("end", C.c_double), ("factor", C.c_double), ("ncells", C.c_int32)]


class Case(C.Structure):
    _fields_ = [("model", C.c_int32), ("nphases", C.c_int32), ("alpha_null", C.c_int32), ("order", C.c_int32),
                ("limiter", C.c_int32 * 4), ("ncells", C.c_int32 * 3), ("length", C.c_double * 3),
                ("cfl", C.c_double), ("time_iterations", C.c_int32), ("max_iterations", C.c_int32),
                ("total_time", C.c_double), ("ptmu", C.c_int32), ("ptmu_liquid", C.c_int32),
                ("ptmu_vapor", C.c_int32), ("eos", Eos * 3), ("bc", C.c_int32 * 6), ("ntransports", C.c_int32),
                ("pt_relaxation", C.c_int32), ("nstretch", C.c_int32 * 3),
                ("stretch", (StretchZone * MAX_STRETCH_ZONES) * 3)]


class StepStats(C.Structure):
    _fields_ = [("cell_updates", C.c_int64), ("relax_calls", C.c_int64), ("newton_evals", C.c_int64),
                ("newton_fallback", C.c_int64), ("newton_max", C.c_int64), ("seeded", C.c_int64),
                ("seed_rejected", C.c_int64), ("ptmu_errors", C.c_int64), ("nonfinite_cells", C.c_int64),
                ("newton_hist", C.c_int64 * 16), ("ptmu_solves", C.c_int64), ("ptmu_outer_iters", C.c_int64),
                ("ptmu_outer_max", C.c_int64), ("ptmu_tsat_calls", C.c_int64), ("ptmu_tsat_iters", C.c_int64),
                ("ptmu_tsat_max", C.c_int64), ("ptmu_outer_hist", C.c_int64 * 16), ("ptmu_seeded", C.c_int64),
                ("ptmu_seed_rejected", C.c_int64), ("bounds_violations", C.c_int64),
                ("staging_timeouts", C.c_int64)]

    def as_dict(self) -> Dict[str, object]:
        d = {f: getattr(self, f) for f, _ in self._fields_ if f not in ("newton_hist", "ptmu_outer_hist")}
        d["newton_hist"] = list(self.newton_hist)
        d["ptmu_outer_hist"] = list(self.ptmu_outer_hist)
        return d


MLP_MAX_IN = 16
MLP_HIDDEN = 64


class Mlp(C.Structure):
    _fields_ = [("n_in", C.c_int32), ("hidden", C.c_int32), ("w1", C.POINTER(C.c_float)),
                ("b1", C.POINTER(C.c_float)), ("w2", C.POINTER(C.c_float)), ("b2", C.POINTER(C.c_float)),
                ("w3", C.POINTER(C.c_float)), ("b3", C.c_float), ("in_shift", C.c_float * MLP_MAX_IN),
                ("in_scale", C.c_float * MLP_MAX_IN), ("out_shift", C.c_float), ("out_scale", C.c_float),
                ("n_out", C.c_int32), ("b3_1", C.c_float), ("out_shift_1", C.c_float), ("out_scale_1", C.c_float)]


_lib = None


def lib():
    """Load libecg.so (fails loudly when it is missing: no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is not built; run `python -m ecogen_b200.build`")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    vp, dp, fp = C.c_void_p, P(C.c_double), P(C.c_float)
    L.ecg_status_str.restype = C.c_char_p
    L.ecg_status_str.argtypes = [C.c_int]
    L.ecg_last_error.restype = C.c_char_p
    L.ecg_version.restype = C.c_int
    L.ecg_input_read.argtypes = [C.c_char_p, C.c_char_p, P(vp)]
    L.ecg_input_free.argtypes = [vp]
    L.ecg_input_case.argtypes = [vp, P(Case)]
    L.ecg_input_run_name.restype = C.c_char_p
    L.ecg_input_run_name.argtypes = [vp]
    L.ecg_input_fill.argtypes = [vp, P(dp), C.c_int64]
    L.ecg_create.argtypes = [P(Case), P(vp)]
    L.ecg_destroy.argtypes = [vp]
    L.ecg_upload_prim.argtypes = [vp, P(dp), C.c_int64]
    L.ecg_download_prim.argtypes = [vp, P(dp), C.c_int64]
    L.ecg_download_derived.argtypes = [vp, dp, dp, C.c_int64]
    L.ecg_upload_prim_device.argtypes = [vp, P(dp), C.c_int64]
    L.ecg_download_prim_device.argtypes = [vp, P(dp), C.c_int64]
    L.ecg_step.argtypes = [vp, C.c_int32, dp, dp, P(StepStats)]
    L.ecg_run.argtypes = [vp, dp, dp, P(C.c_int32), P(StepStats)]
    L.ecg_step_profiled.argtypes = [vp, C.c_int32, dp, dp, P(StepStats), dp]
    L.ecg_step_profiled_kernels.argtypes = [vp, C.c_int32, dp, dp, P(StepStats), dp]
    L.ecg_set_step_form.argtypes = [vp, C.c_int32]
    L.ecg_step_form.restype = C.c_int32
    L.ecg_step_form.argtypes = [vp]
    L.ecg_set_face_staging.argtypes = [vp, C.c_int32]
    L.ecg_face_staging.restype = C.c_int32
    L.ecg_face_staging.argtypes = [vp]
    L.ecg_set_ptmu_seed.argtypes = [vp, C.c_int32]
    L.ecg_set_ptmu_warm_start.argtypes = [vp, C.c_int32]
    L.ecg_step_noalloc.argtypes = [P(Case), vp, vp, C.c_double, dp, P(StepStats), vp]
    L.ecg_ncells.restype = C.c_int64
    L.ecg_ncells.argtypes = [vp]
    L.ecg_stream.restype = vp
    L.ecg_stream.argtypes = [vp]
    L.ecg_set_newton_cap.argtypes = [vp, C.c_int32]
    L.ecg_set_newton_cap_mode.argtypes = [vp, C.c_int32]
    L.ecg_set_seed_model.argtypes = [vp, P(Mlp)]
    L.ecg_record_pairs.argtypes = [vp, C.c_int64, C.c_int32]
    L.ecg_fetch_pairs.argtypes = [vp, fp, fp, P(C.c_int64)]
    for name in ("ecg_trainer_create", "ecg_trainer_destroy", "ecg_trainer_epoch", "ecg_trainer_grad",
                 "ecg_trainer_forward", "ecg_trainer_export", "ecg_trainer_import", "ecg_trainer_set_norm",
                 "ecg_batch_create", "ecg_batch_destroy", "ecg_batch_upload_prim", "ecg_batch_download_prim",
                 "ecg_batch_step", "ecg_batch_set_seed_model", "ecg_batch_set_shape", "ecg_batch_autotune",
                 "ecg_batch_total_cells"):
        getattr(L, name)  # every symbol the header declares must be exported
    L.ecg_trainer_create.argtypes = [C.c_int32, C.c_int32, C.c_uint64, P(vp)]
    L.ecg_trainer_create_n.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_uint64, P(vp)]
    L.ecg_trainer_set_norm_out1.argtypes = [vp, C.c_float, C.c_float]
    L.ecg_trainer_destroy.argtypes = [vp]
    L.ecg_trainer_epoch.argtypes = [vp, fp, fp, C.c_int64, C.c_int32, C.c_float, C.c_float, fp]
    L.ecg_trainer_grad.argtypes = [vp, fp, fp, C.c_int32, fp, fp, fp, fp, fp, fp, fp]
    L.ecg_trainer_forward.argtypes = [vp, fp, C.c_int32, fp]
    L.ecg_trainer_export.argtypes = [vp, P(Mlp)]
    L.ecg_trainer_import.argtypes = [vp, P(Mlp)]
    L.ecg_trainer_set_norm.argtypes = [vp, fp, fp, C.c_float, C.c_float]
    L.ecg_batch_create.argtypes = [P(Case), C.c_int32, P(vp)]
    L.ecg_batch_destroy.argtypes = [vp]
    L.ecg_batch_upload_prim.argtypes = [vp, P(dp), C.c_int64]
    L.ecg_batch_download_prim.argtypes = [vp, P(dp), C.c_int64]
    L.ecg_batch_step.argtypes = [vp, C.c_int32, dp, dp, P(StepStats)]
    L.ecg_batch_set_seed_model.argtypes = [vp, P(Mlp)]
    L.ecg_batch_set_shape.argtypes = [vp, C.c_int32, C.c_int32]
    L.ecg_batch_autotune.argtypes = [vp, P(C.c_int32), P(C.c_int32)]
    L.ecg_batch_total_cells.restype = C.c_int64
    L.ecg_batch_total_cells.argtypes = [vp]
    L.ecg_input_output_control.argtypes = [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    L.ecg_restart_fill.argtypes = [C.POINTER(Case), C.POINTER(C.POINTER(C.c_double)), C.c_int64]
    L.ecg_batch_stream.restype = vp
    L.ecg_batch_stream.argtypes = [vp]
    _lib = L
    return L


def check(status: int, where: str):
    if status != ECG_OK:
        raise EcgError(status, where, lib().ecg_last_error().decode())


def _field_ptrs(arrs: Sequence[np.ndarray]):
    ptrs = (C.POINTER(C.c_double) * len(arrs))()
    for i, a in enumerate(arrs):
        ptrs[i] = a.ctypes.data_as(C.POINTER(C.c_double))
    return ptrs


def nfields(case: Case) -> int:
    if case.model == MODEL_EULER:
        return 6 + case.ntransports
    if case.model == MODEL_PTUEQ:  # + the mixture temperature
        return 2 * case.nphases + 6 + case.ntransports
    return 2 * case.nphases + 5 + case.ntransports


def case_from_spec(spec) -> Case:
    """ABI case record of an ``ecogen_b200.cases.Case`` description."""
    c = Case()
    euler = spec.model.upper() == "EULER"
    c.model = MODEL_EULER if euler else (MODEL_PTUEQ if getattr(spec, "ptueq", False) else MODEL_KAPILA)
    c.nphases = spec.nphases
    c.alpha_null = 1 if spec.alpha_null else 0
    c.order = 2 if spec.second_order else 1
    g = (spec.second_order or "NONE").upper()
    il = (spec.interface_limiter or g).upper()
    gv = (spec.vf_limiter or g).upper()
    iv = (spec.interface_vf_limiter or il).upper()
    for i, name in enumerate((g, il, gv, iv)):
        c.limiter[i] = LIM_CODE[name]
    for i in range(3):
        c.ncells[i] = int(spec.cells[i])
        c.length[i] = float(spec.lengths[i])
    c.cfl = spec.cfl
    c.time_iterations = 1 if spec.iterations is not None else 0
    c.max_iterations = int(spec.iterations or 0)
    c.total_time = float(spec.total_time or 0.0)
    if spec.ptmu is not None:
        c.ptmu, c.ptmu_liquid, c.ptmu_vapor = 1, spec.ptmu[0], spec.ptmu[1]
    for k, e in enumerate(spec.eos):
        c.eos[k] = Eos(EOS_CODE[e.kind], e.gamma, e.pinf, e.b, e.cv, e.eref, e.sref)
    for i, b in enumerate(spec.boundary_types()):
        c.bc[i] = BC_CODE[b.upper()]
    c.ntransports = len(spec.transports or [])
    c.pt_relaxation = 1 if getattr(spec, "pt_relaxation", False) else 0
    for a, ax in enumerate("xyz"):
        zones = (getattr(spec, "stretch", None) or {}).get(ax) or []
        if int(spec.cells[a]) <= 1:
            zones = []
        c.nstretch[a] = len(zones)
        for z, (s0, s1, f, m) in enumerate(zones):
            c.stretch[a][z] = StretchZone(float(s0), float(s1), float(f), int(m))
    return c


class Input:
    """A case read from its ECOGEN XML files (``ecg_input_read``)."""

    def __init__(self, case_dir: str, eos_dir: str):
        h = C.c_void_p()
        check(lib().ecg_input_read(case_dir.encode(), eos_dir.encode(), C.byref(h)), "ecg_input_read")
        self.h = h
        self.case = Case()
        check(lib().ecg_input_case(self.h, C.byref(self.case)), "ecg_input_case")
        self.run_name = lib().ecg_input_run_name(self.h).decode()

    @property
    def ncells(self) -> int:
        return int(self.case.ncells[0]) * int(self.case.ncells[1]) * int(self.case.ncells[2])

    def fill(self) -> List[np.ndarray]:
        arrs = [np.zeros(self.ncells) for _ in range(nfields(self.case))]
        check(lib().ecg_input_fill(self.h, _field_ptrs(arrs), self.ncells), "ecg_input_fill")
        return arrs

    def __del__(self):
        if getattr(self, "h", None):
            lib().ecg_input_free(self.h)
            self.h = None


class Context:
    """One case on the current GPU: device state, stream and time-loop scalars."""

    def __init__(self, case: Case):
        self.case = case
        h = C.c_void_p()
        check(lib().ecg_create(C.byref(case), C.byref(h)), "ecg_create")
        self.h = h
        self.n = int(lib().ecg_ncells(self.h))
        self.dt = C.c_double(1e-15)
        self.t = C.c_double(0.0)
        self.iteration = 0
        self.stats = StepStats()

    def upload(self, fields: Sequence[np.ndarray]):
        arrs = [np.ascontiguousarray(f, dtype=np.float64) for f in fields]
        self._keep = arrs
        check(lib().ecg_upload_prim(self.h, _field_ptrs(arrs), self.n), "ecg_upload_prim")

    def download(self) -> List[np.ndarray]:
        arrs = [np.zeros(self.n) for _ in range(nfields(self.case))]
        check(lib().ecg_download_prim(self.h, _field_ptrs(arrs), self.n), "ecg_download_prim")
        return arrs

    def download_dict(self) -> Dict[str, np.ndarray]:
        f = self.download()
        nt = self.case.ntransports
        if self.case.model == MODEL_EULER:
            return {"alpha": np.ones((1, self.n)), "rho": f[0][None, :], "p": f[1], "u": np.stack(f[2:5]),
                    "E": f[5], "tr": np.array(f[6:6 + nt]).reshape(nt, self.n)}
        k = self.case.nphases
        out = {"alpha": np.stack(f[:k]), "rho": np.stack(f[k:2 * k]), "p": f[2 * k],
               "u": np.stack(f[2 * k + 1:2 * k + 4]), "E": f[2 * k + 4]}
        if self.case.model == MODEL_PTUEQ:
            out["Tm"] = f[2 * k + 5]
            out["tr"] = np.zeros((0, self.n))
        else:
            out["tr"] = np.array(f[2 * k + 5:2 * k + 5 + nt]).reshape(nt, self.n)
        return out

    def derived(self):
        k = self.case.nphases
        T = np.zeros(k * self.n)
        Y = np.zeros(k * self.n)
        check(lib().ecg_download_derived(self.h, T.ctypes.data_as(C.POINTER(C.c_double)),
                                         Y.ctypes.data_as(C.POINTER(C.c_double)), self.n), "ecg_download_derived")
        return T.reshape(k, self.n), Y.reshape(k, self.n)

    def step(self, nsteps: int = 1) -> StepStats:
        st = StepStats()
        check(lib().ecg_step(self.h, nsteps, C.byref(self.dt), C.byref(self.t), C.byref(st)), "ecg_step")
        self.iteration += nsteps
        self.stats = st
        return st

    def step_profiled(self, nsteps: int = 1):
        """Steps with every kernel timed separately: returns (stats, [pass1_ms, pass2_ms, update_ms])."""
        st = StepStats()
        ms = (C.c_double * 3)(0.0, 0.0, 0.0)
        check(lib().ecg_step_profiled(self.h, nsteps, C.byref(self.dt), C.byref(self.t), C.byref(st), ms),
              "ecg_step_profiled")
        self.iteration += nsteps
        return st, list(ms)

    def step_profiled_kernels(self, nsteps: int = 1):
        """Steps with every kernel timed separately: (stats, 9 times in ms) -- pass 1 X / Y / Z face
        kernels and cell kernel, pass 2 the same, update (ecg_step_profiled_kernels)."""
        st = StepStats()
        ms = (C.c_double * 9)(*([0.0] * 9))
        check(lib().ecg_step_profiled_kernels(self.h, nsteps, C.byref(self.dt), C.byref(self.t), C.byref(st), ms),
              "ecg_step_profiled_kernels")
        self.iteration += nsteps
        return st, list(ms)

    def set_step_form(self, form: int):
        """FORM_FUSED or FORM_SPLIT (ecg_set_step_form)."""
        check(lib().ecg_set_step_form(self.h, form), "ecg_set_step_form")

    @property
    def step_form(self) -> int:
        return int(lib().ecg_step_form(self.h))

    def set_face_staging(self, staging: int):
        """STAGING_TMA (default where the mesh allows) or STAGING_PLAIN (ecg_set_face_staging)."""
        check(lib().ecg_set_face_staging(self.h, staging), "ecg_set_face_staging")

    @property
    def face_staging(self) -> int:
        """The staging the next split-form step uses (ecg_face_staging)."""
        return int(lib().ecg_face_staging(self.h))

    def set_ptmu_warm_start(self, on: bool):
        """Start each cell's T_sat solves from its previous solve (ecg_set_ptmu_warm_start)."""
        check(lib().ecg_set_ptmu_warm_start(self.h, 1 if on else 0), "ecg_set_ptmu_warm_start")

    def set_ptmu_seed(self, mode: int):
        """PTMU_SEED_T (default) or PTMU_SEED_P_T: what a p-T-mu seed model starts (ecg_set_ptmu_seed)."""
        check(lib().ecg_set_ptmu_seed(self.h, mode), "ecg_set_ptmu_seed")

    def run(self) -> StepStats:
        st = StepStats()
        it = C.c_int32(self.iteration)
        check(lib().ecg_run(self.h, C.byref(self.dt), C.byref(self.t), C.byref(it), C.byref(st)), "ecg_run")
        self.iteration = it.value
        self.stats = st
        return st

    def set_newton_cap(self, cap: int):
        check(lib().ecg_set_newton_cap(self.h, cap), "ecg_set_newton_cap")

    def set_newton_cap_mode(self, mode: int):
        """CAP_FALLBACK (interface pressure at the cap, the reference's) or CAP_ACCEPT (keep the iterate)."""
        check(lib().ecg_set_newton_cap_mode(self.h, mode), "ecg_set_newton_cap_mode")

    def set_seed_model(self, mlp: Optional["Mlp"]):
        check(lib().ecg_set_seed_model(self.h, C.byref(mlp) if mlp is not None else None), "ecg_set_seed_model")

    def record_pairs(self, max_pairs: int, min_evals: int = 1):
        check(lib().ecg_record_pairs(self.h, max_pairs, min_evals), "ecg_record_pairs")

    def fetch_pairs(self):
        """Recorded (features, targets): pressure relaxation 3N features and one target; p-T-mu
        relaxation 8 features and two targets (ln p*, T_sat(p*)), targets then an (n, 2) array."""
        cnt = C.c_int64(0)
        check(lib().ecg_fetch_pairs(self.h, None, None, C.byref(cnt)), "ecg_fetch_pairs")
        ptmu = bool(self.case.ptmu)
        nin = 8 if ptmu else 3 * self.case.nphases
        x = np.zeros((cnt.value, nin), dtype=np.float32)
        y = np.zeros((cnt.value, 2) if ptmu else cnt.value, dtype=np.float32)
        if cnt.value:
            check(lib().ecg_fetch_pairs(self.h, x.ctypes.data_as(C.POINTER(C.c_float)),
                                        y.ctypes.data_as(C.POINTER(C.c_float)), C.byref(cnt)), "ecg_fetch_pairs")
        return x, y

    def close(self):
        if getattr(self, "h", None):
            lib().ecg_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()
