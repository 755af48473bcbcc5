"""ctypes binding of the C restatement (``oracle/ecg_oracle.c``) — TEST INFRASTRUCTURE.

Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use this
module, and only as the checker.  ``initial_fields`` fills the initial state
of a case the way the reference does (src/Geometries/GeometricalDomain.cpp:64
fillIn, domains applied in document order, each one overwriting the cells it
contains; phase states from src/Models/PUEq/PhasePUEq.cpp:41).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from typing import Dict, Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libecg_oracle.so")
# Sensitivity variants of the same restatement, which measure how far last-ulp changes of the math
# library travel through a run: "crlog", a correctly rounded ln in the saturation solve (ecg_crlog.h);
# "powulp", pow of the isentropic star pressure moved by one ulp in 1 call in 100 (ecg_powulp.h).
VARIANT_PATHS = {"crlog": os.path.join(HERE, "_ref", "libecg_oracle_crlog.so"),
                 "powulp": os.path.join(HERE, "_ref", "libecg_oracle_powulp.so")}

EOS_CODE = {"IG": 0, "SG": 1, "NASG": 2}
BC_CODE = {"NONREFLECTING": 0, "SYMMETRY": 1, "WALL": 1}
LIM_CODE = {None: 0, "NONE": 0, "MINMOD": 1, "VANLEER": 2, "VANALBADA": 3, "SUPERBEE": 4, "MC": 5, "THINC": 6}


class Eos(C.Structure):
    _fields_ = [("type", C.c_int), ("gamma", C.c_double), ("pinf", C.c_double), ("b", C.c_double),
                ("cv", C.c_double), ("eref", C.c_double), ("sref", C.c_double)]


MAX_STRETCH = 8


class Stretch(C.Structure):
    _fields_ = [("start", C.c_double), ("end", C.c_double), ("factor", C.c_double), ("ncells", C.c_int)]


class Case(C.Structure):
    _fields_ = [("model", C.c_int), ("nphases", C.c_int), ("alpha_null", C.c_int), ("order", C.c_int),
                ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double), ("cfl", C.c_double),
                ("lim", C.c_int * 4), ("ptmu", C.c_int), ("ptmu_liq", C.c_int), ("ptmu_vap", C.c_int),
                ("eos", Eos * 3), ("bc", C.c_int * 6), ("ntr", C.c_int), ("pt", C.c_int),
                ("nstretch", C.c_int * 3), ("stretch", (Stretch * MAX_STRETCH) * 3)]


class Stats(C.Structure):
    _fields_ = [("relax_calls", C.c_longlong), ("newton_evals", C.c_longlong), ("newton_fallback", C.c_longlong),
                ("newton_max", C.c_longlong), ("ptmu_errors", C.c_longlong)]


_lib = None
_libs = {}


def build() -> str:
    """Compile the C restatement into oracle/_ref/libecg_oracle.so (gcc, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", HERE, "lib"], check=True)
    return LIB_PATH


def lib(variant: Optional[str] = None):
    """The oracle library, or one of its sensitivity variants ("crlog", "powulp")."""
    global _lib
    if variant:
        if variant not in _libs:
            path = VARIANT_PATHS[variant]
            src = os.path.join(HERE, "ecg_oracle.c")
            if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
                build()
            _libs[variant] = _declare(C.CDLL(path))
        return _libs[variant]
    if _lib is None:
        src = os.path.join(HERE, "ecg_oracle.c")
        if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
            build()
        _lib = _declare(C.CDLL(LIB_PATH))
    return _lib


def _declare(L):
    """Declares the C signatures of an oracle library."""
    dp = C.POINTER(C.c_double)
    L.ecgo_create.restype = C.c_void_p
    L.ecgo_create.argtypes = [C.POINTER(Case), dp, dp, dp, dp, dp]
    L.ecgo_create_ptueq.restype = C.c_void_p
    L.ecgo_create_ptueq.argtypes = [C.POINTER(Case), dp, dp, dp, dp, dp]
    L.ecgo_get_transports.argtypes = [C.c_void_p, dp]
    L.ecgo_destroy.argtypes = [C.c_void_p]
    L.ecgo_step.argtypes = [C.c_void_p, C.c_int, dp, dp, C.POINTER(Stats)]
    L.ecgo_get.argtypes = [C.c_void_p] + [dp] * 8
    L.ecgo_get_phase_pressure.argtypes = [C.c_void_p, dp]
    L.ecgo_relax_pinf.argtypes = [C.POINTER(Case), dp, dp, dp, dp, C.POINTER(C.c_int)]
    L.ecgo_pressure_isentropic.restype = C.c_double
    L.ecgo_pressure_isentropic.argtypes = [C.POINTER(Eos), C.c_double, C.c_double, C.c_double, C.c_int]
    L.ecgo_density_pfinal.restype = C.c_double
    L.ecgo_density_pfinal.argtypes = [C.POINTER(Eos), C.c_double, C.c_double, C.c_double, dp, C.c_int]
    L.ecgo_limiter.restype = C.c_double
    L.ecgo_limiter.argtypes = [C.c_int, C.c_double, C.c_double]
    return L


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def make_case(case) -> Case:
    """Convert an ``ecogen_b200.cases.Case`` into the oracle's case record."""
    c = Case()
    euler = case.model.upper() == "EULER"
    c.model = 1 if euler else (2 if getattr(case, "ptueq", False) else 0)
    c.nphases = case.nphases
    c.alpha_null = 1 if case.alpha_null else 0
    c.order = 2 if case.second_order else 1
    c.nx, c.ny, c.nz = (int(v) for v in case.cells)
    c.lx, c.ly, c.lz = (float(v) for v in case.lengths)
    c.cfl = case.cfl
    g = (case.second_order or "NONE").upper()
    il = (case.interface_limiter or g).upper()
    gv = (case.vf_limiter or g).upper()
    iv = (case.interface_vf_limiter or il).upper()
    for i, name in enumerate((g, il, gv, iv)):
        c.lim[i] = LIM_CODE[name]
    if case.ptmu is not None:
        c.ptmu, c.ptmu_liq, c.ptmu_vap = 1, case.ptmu[0], case.ptmu[1]
    for k, e in enumerate(case.eos):
        c.eos[k] = Eos(EOS_CODE[e.kind], e.gamma, e.pinf, e.b, e.cv, e.eref, e.sref)
    for i, b in enumerate(case.boundary_types()):
        c.bc[i] = BC_CODE[b.upper()]
    c.ntr = len(case.transports or [])
    c.pt = 1 if getattr(case, "pt_relaxation", False) else 0
    for a, ax in enumerate("xyz"):
        zones = (getattr(case, "stretch", None) or {}).get(ax) or []
        if int(case.cells[a]) <= 1:
            zones = []
        c.nstretch[a] = len(zones)
        for z, (s0, s1, f, m) in enumerate(zones):
            c.stretch[a][z] = Stretch(float(s0), float(s1), float(f), int(m))
    return c


def cell_centres(case) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Cell centres per axis -- (i+0.5)*d, or the stretched centres -- in cell index order
    (src/Meshes/MeshCartesian.cpp:168-210)."""
    xs, ys, zs = (case.axis_cells(a)[1] for a in range(3))
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    return X.ravel(), Y.ravel(), Z.ravel()


def _belongs(d, X, Y, Z) -> np.ndarray:
    ax = {"x": X, "y": Y, "z": Z}
    k = d.kind
    if k == "entireDomain":
        return np.ones_like(X, dtype=bool)
    if k == "halfSpace":
        v = ax[d.data["axis"].lower()]
        return v >= d.data["origin"] if d.data["direction"] == "positive" else v <= d.data["origin"]
    if k == "disc":
        c = d.data["center"]
        cc = {"x": c[0], "y": c[1], "z": c[2]}
        s = np.zeros_like(X)
        for a in (d.data["axis1"].lower(), d.data["axis2"].lower()):
            s = s + (ax[a] - cc[a]) ** 2
        return s <= d.data["radius"] * d.data["radius"]
    if k == "sphere":
        c = d.data["center"]
        s = (X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2
        return s <= d.data["radius"] * d.data["radius"]
    if k == "rectangle":
        c = d.data["corner"]
        cc = {"x": c[0], "y": c[1], "z": c[2]}
        m = np.ones_like(X, dtype=bool)
        for a, l in ((d.data["axis1"].lower(), d.data["l1"]), (d.data["axis2"].lower(), d.data["l2"])):
            m &= ~((ax[a] - cc[a]) < 0) & ~((ax[a] - cc[a]) > l)
        return m
    if k == "cuboid":
        c = d.data["corner"]
        m = np.ones_like(X, dtype=bool)
        for v, o, l in ((X, c[0], d.data["lx"]), (Y, c[1], d.data["ly"]), (Z, c[2], d.data["lz"])):
            m &= ~((v - o) < 0) & ~((v - o) > l)
        return m
    raise ValueError(k)


def initial_fields(case) -> Dict[str, np.ndarray]:
    """Initial (alpha_k, rho_k, p, u) of a case, filled domain by domain like the reference; the
    temperature-pressure equilibrium model adds the mixture temperature "T" (phase densities from (p, T))."""
    X, Y, Z = cell_centres(case)
    n = X.size
    npf = case.nphases
    alpha = np.zeros((npf, n))
    rho = np.zeros((npf, n))
    p = np.zeros(n)
    T = np.zeros(n)
    u = np.zeros((3, n))
    names = list(case.transports or [])
    tr = np.zeros((len(names), n))
    states = {s.name: s for s in case.states}
    for d in case.domains:
        m = _belongs(d, X, Y, Z)
        st = states[d.state]
        for k, ph in enumerate(st.phases):
            e = case.eos[k]
            if getattr(case, "ptueq", False):
                r = e.density_from_pT(st.pressure, st.temperature)
            elif ph.temperature is not None:
                r = e.density_from_pT(st.pressure, ph.temperature)
            else:
                r = ph.density
            alpha[k, m] = ph.alpha
            rho[k, m] = r
        p[m] = st.pressure
        if getattr(st, "temperature", None) is not None:
            T[m] = st.temperature
        for dd in range(3):
            u[dd, m] = st.velocity[dd]
        for j, name in enumerate(names):  # a state without the transport leaves 0 (Input.cpp:1034-1050)
            tr[j, m] = (st.transports or {}).get(name, 0.0)
    out = {"alpha": alpha, "rho": rho, "p": p, "u": u, "tr": tr}
    if getattr(case, "ptueq", False):
        out["T"] = T
    return out


class Sim:
    """One oracle simulation; mirrors the reference run loop (dt starts at 1e-15, src/Run.cpp:38)."""

    def __init__(self, case, fields: Optional[Dict[str, np.ndarray]] = None, variant: Optional[str] = None):
        self.case = case
        self._L = lib(variant)
        self.c = make_case(case)
        f = fields or initial_fields(case)
        self.n = case.ncells
        self.np = case.nphases
        a = np.ascontiguousarray(f["alpha"], dtype=np.float64)
        r = np.ascontiguousarray(f["rho"], dtype=np.float64)
        p = np.ascontiguousarray(f["p"], dtype=np.float64)
        u = np.ascontiguousarray(f["u"], dtype=np.float64)
        self.ntr = self.c.ntr
        tr = np.ascontiguousarray(f.get("tr", np.zeros((self.ntr, self.n))), dtype=np.float64)
        self._tr = tr
        if self.c.model == 2:
            T = np.ascontiguousarray(f["T"], dtype=np.float64)
            self._T = T
            self.h = self._L.ecgo_create_ptueq(C.byref(self.c), _p(a), _p(T), _p(p), _p(u), _p(tr) if self.ntr else None)
        else:
            self.h = self._L.ecgo_create(C.byref(self.c), _p(a), _p(r), _p(p), _p(u), _p(tr) if self.ntr else None)
        if not self.h:
            raise ValueError("ecgo_create refused the case")
        self.dt = C.c_double(1e-15)
        self.t = C.c_double(0.0)
        self.iteration = 0
        self.stats = Stats()

    def step(self, nsteps: int = 1):
        self._L.ecgo_step(self.h, nsteps, C.byref(self.dt), C.byref(self.t), C.byref(self.stats))
        self.iteration += nsteps

    def run_to_time(self, t_end: float, max_steps: int = 10 ** 9):
        """Physical-time mode: step until t >= t_end, no clipping of the last step (src/Run.cpp:421-428)."""
        while self.t.value < t_end and self.iteration < max_steps:
            self.step(1)

    def fields(self) -> Dict[str, np.ndarray]:
        n, k = self.n, self.np
        out = {"alpha": np.zeros((k, n)), "rho": np.zeros((k, n)), "T": np.zeros((k, n)), "Y": np.zeros((k, n)),
               "rho_mix": np.zeros(n), "p": np.zeros(n), "E": np.zeros(n), "u": np.zeros((3, n))}
        self._L.ecgo_get(self.h, _p(out["alpha"]), _p(out["rho"]), _p(out["T"]), _p(out["Y"]), _p(out["rho_mix"]),
                       _p(out["p"]), _p(out["E"]), _p(out["u"]))
        out["tr"] = np.zeros((self.ntr, n))
        if self.ntr:
            self._L.ecgo_get_transports(self.h, _p(out["tr"]))
        return out

    def phase_pressures(self) -> np.ndarray:
        pk = np.zeros((self.np, self.n))
        self._L.ecgo_get_phase_pressure(self.h, _p(pk))
        return pk

    def __del__(self):
        if getattr(self, "h", None):
            self._L.ecgo_destroy(self.h)
            self.h = None
