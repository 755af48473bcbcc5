"""Writers for ECOGEN-format case inputs (main / mesh / model / initialConditions + libEOS).

ECOGEN reads a case as four XML files in one folder plus EOS parameter files in
``<work>/libEOS`` (reference: src/InputOutput/Input.cpp:40-48 for the file names,
:77 inputMain, :319 inputMesh, :566 inputModel, :865 inputEOS, :917
inputInitialConditions).  This module writes exactly that layout so that the
same folder drives both the reference CPU solver and this library's C++ host
(``ecg_input_read``).

The named workloads are built here as seeded synthetic cases:

* ``shock_tube_1d``      1D two-phase water/air shock tube, Kapila, first order
* ``shock_bubble_2d``    2D planar water shock hitting an air bubble, MUSCL + van Leer
* ``cavity_collapse_3d`` 3D three-phase liquid with 64 spherical gas inclusions, MUSCL + minmod
* ``batch_shock_tubes``  many independent 1D shock tubes of uneven length (batched mode)
* ``expansion_tube_2d``  2D liquid/vapour expansion with p-T-mu relaxation

Every function takes the mesh size as an argument so that the parity tests can
run the same physics at sizes the CPU oracle finishes in seconds.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np


# ----------------------------------------------------------------------------- EOS


@dataclass
class Eos:
    """One EOS parameter file (reference src/Eos/EosIG.cpp:36, EosSG.cpp:36, EosNASG.cpp:36)."""

    name: str  # file name inside libEOS, e.g. "SG_water.xml"
    kind: str  # "IG" | "SG" | "NASG"
    gamma: float
    cv: float
    pinf: float = 0.0
    b: float = 0.0
    eref: float = 0.0
    sref: float = 0.0

    def xml(self) -> str:
        if self.kind == "IG":
            params = f'gamma="{self.gamma!r}" cv="{self.cv!r}" energyRef="{self.eref!r}" entropyRef="{self.sref!r}"'
        elif self.kind == "SG":
            params = (f'gamma="{self.gamma!r}" pInf="{self.pinf!r}" cv="{self.cv!r}" '
                      f'energyRef="{self.eref!r}" entropyRef="{self.sref!r}"')
        elif self.kind == "NASG":
            params = (f'gamma="{self.gamma!r}" pInf="{self.pinf!r}" b="{self.b!r}" cv="{self.cv!r}" '
                      f'energyRef="{self.eref!r}" entropyRef="{self.sref!r}"')
        else:
            raise ValueError(self.kind)
        return ('<?xml version = "1.0" encoding = "UTF-8" standalone = "yes"?>\n'
                f'<parametersEOS>\n  <EOS type="{self.kind}"/>\n  <parameters {params}/>\n</parametersEOS>\n')

    # thermodynamics used by the case builders (host-side, not the hot path)
    def density_from_pT(self, p: float, T: float) -> float:
        if self.kind == "IG":
            return p / ((self.gamma - 1.0) * self.cv * T)
        if self.kind == "SG":
            return (p + self.pinf) / ((self.gamma - 1.0) * self.cv * T)
        return (p + self.pinf) / ((self.gamma - 1.0) * self.cv * T + self.b * (p + self.pinf))


WATER_SG = Eos("SG_water.xml", "SG", gamma=4.4, pinf=6.0e8, cv=1000.0)
AIR_IG = Eos("IG_air.xml", "IG", gamma=1.4, cv=800.0)
GAS_B_IG = Eos("IG_gasB.xml", "IG", gamma=1.67, cv=3116.0)
LIQ_PC = Eos("SG_liquidPC.xml", "SG", gamma=2.35, pinf=1.0e9, cv=1816.0, eref=-1167.0e3, sref=0.0)
VAP_PC = Eos("SG_vapourPC.xml", "SG", gamma=1.43, pinf=0.0, cv=1040.0, eref=2030.0e3, sref=-23.0e3)
PTUEQ = "TemperaturePressureVelocityEq"
WATER_SG300 = Eos("SG_water300K.xml", "SG", gamma=2.955, pinf=7.22e8, cv=1231.2)
WATER_NASG = Eos("NASG_water.xml", "NASG", gamma=1.19, pinf=7.028e8, b=6.61e-4, cv=3610.0, eref=-1177788.0)


# ----------------------------------------------------------------------------- case description


@dataclass
class PhaseState:
    alpha: float
    density: Optional[float] = None
    temperature: Optional[float] = None


@dataclass
class State:
    name: str
    phases: List[PhaseState]
    pressure: float
    velocity: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    transports: Optional[Dict[str, float]] = None  # value of each passive transport in this state
    temperature: Optional[float] = None  # mixture temperature (temperature-pressure equilibrium model)


@dataclass
class Domain:
    """A geometrical domain (reference src/Geometries/GD*.cpp); later domains overwrite earlier ones."""

    name: str
    state: str
    kind: str  # entireDomain | halfSpace | disc | sphere | rectangle | cuboid
    data: Dict[str, object] = field(default_factory=dict)

    def xml(self) -> str:
        head = f'<domain name="{self.name}" state="{self.state}" type="{self.kind}"'
        d = self.data
        if self.kind == "entireDomain":
            return head + "/>"
        if self.kind == "halfSpace":
            return (head + f'>\n      <dataHalfSpace axis="{d["axis"]}" origin="{d["origin"]!r}" '
                    f'direction="{d["direction"]}"/>\n    </domain>')
        if self.kind == "disc":
            c = d["center"]
            return (head + f'>\n      <dataDisc axis1="{d["axis1"]}" axis2="{d["axis2"]}" radius="{d["radius"]!r}">\n'
                    f'        <center x="{c[0]!r}" y="{c[1]!r}" z="{c[2]!r}"/>\n      </dataDisc>\n    </domain>')
        if self.kind == "sphere":
            c = d["center"]
            return (head + f'>\n      <dataSphere radius="{d["radius"]!r}">\n'
                    f'        <center x="{c[0]!r}" y="{c[1]!r}" z="{c[2]!r}"/>\n      </dataSphere>\n    </domain>')
        if self.kind == "rectangle":
            c = d["corner"]
            return (head + f'>\n      <dataRectangle axis1="{d["axis1"]}" axis2="{d["axis2"]}" '
                    f'lAxis1="{d["l1"]!r}" lAxis2="{d["l2"]!r}">\n'
                    f'        <posInferiorVertex x="{c[0]!r}" y="{c[1]!r}" z="{c[2]!r}"/>\n'
                    f'      </dataRectangle>\n    </domain>')
        if self.kind == "cuboid":
            c = d["corner"]
            return (head + f'>\n      <dataCuboid lAxisX="{d["lx"]!r}" lAxisY="{d["ly"]!r}" lAxisZ="{d["lz"]!r}">\n'
                    f'        <posInferiorVertex x="{c[0]!r}" y="{c[1]!r}" z="{c[2]!r}"/>\n'
                    f'      </dataCuboid>\n    </domain>')
        raise ValueError(self.kind)


@dataclass
class Case:
    """Everything the four ECOGEN case files hold for one run."""

    name: str
    eos: List[Eos]
    lengths: Tuple[float, float, float]
    cells: Tuple[int, int, int]
    states: List[State]
    domains: List[Domain]
    model: str = "PressureVelocityEq"
    alpha_null: bool = False
    cfl: float = 0.8
    iterations: Optional[int] = None      # iteration mode (timeControlMode iterations="true")
    total_time: Optional[float] = None    # physical-time mode
    second_order: Optional[str] = None    # global limiter name, None = first order
    interface_limiter: Optional[str] = None
    vf_limiter: Optional[str] = None
    interface_vf_limiter: Optional[str] = None
    ptmu: Optional[Tuple[int, int]] = None  # (liquid phase, vapour phase)
    boundaries: Optional[List[str]] = None  # boundCond types Xm, Xp, Ym, Yp, Zm, Zp (default nonReflecting)
    transports: Optional[List[str]] = None  # names of passive transports (model.xml <transport>)
    pt_relaxation: bool = False             # model.xml <relaxation type="PT"> (analytic p-T relaxation)
    output_format: str = "XML"
    output_binary: bool = True
    output_precision: Optional[int] = None  # outputMode precision (ASCII values, infoCalcul.out)
    print_freq: Optional[int] = None        # iterFreq (iteration mode; default: print at the end only)
    restart_file: Optional[int] = None      # restartSimulation restartFileNumber
    # mesh.xml meshStretching: per axis ("x", "y", "z") a list of zones (startAt, endAt, factor, numberCells)
    stretch: Optional[Dict[str, List[Tuple[float, float, float, int]]]] = None
    extra: Dict[str, object] = field(default_factory=dict)

    def boundary_types(self) -> List[str]:
        """boundCond type of each side Xm, Xp, Ym, Yp, Zm, Zp (sides of unused axes included)."""
        b = list(self.boundaries or [])
        return b + ["nonReflecting"] * (6 - len(b))

    @property
    def ptueq(self) -> bool:
        """Temperature-pressure-velocity equilibrium model (ModPTUEq, src/Models/PTUEq)."""
        return self.model.upper() == PTUEQ.upper()

    @property
    def ncells(self) -> int:
        return int(self.cells[0]) * int(self.cells[1]) * int(self.cells[2])

    @property
    def nphases(self) -> int:
        return len(self.eos)

    @property
    def dim(self) -> int:
        return sum(1 for n in self.cells if n != 1)

    # -- XML -----------------------------------------------------------------
    def main_xml(self) -> str:
        if self.iterations is not None:
            tc = (f'<timeControlMode iterations="true">\n    <iterations number="{self.iterations}" '
                  f'iterFreq="{self.print_freq or self.iterations}"/>\n  </timeControlMode>')
        else:
            tc = (f'<timeControlMode iterations="false">\n    <physicalTime totalTime="{self.total_time!r}" '
                  f'timeFreq="{self.total_time!r}"/>\n  </timeControlMode>')
        so = ""
        if self.second_order:
            so = f"  <secondOrder>\n    <globalLimiter>{self.second_order}</globalLimiter>\n"
            if self.interface_limiter:
                so += f"    <interfaceLimiter>{self.interface_limiter}</interfaceLimiter>\n"
            if self.vf_limiter:
                so += f"    <globalVolumeFractionLimiter>{self.vf_limiter}</globalVolumeFractionLimiter>\n"
            if self.interface_vf_limiter:
                so += (f"    <interfaceVolumeFractionLimiter>{self.interface_vf_limiter}"
                       f"</interfaceVolumeFractionLimiter>\n")
            so += "  </secondOrder>\n"
        binary = "true" if self.output_binary else "false"
        prec = ' precision="17"' if self.output_format == "GNU" else ""
        if self.output_precision is not None:
            prec = f' precision="{self.output_precision}"'
        rs = ""
        if self.restart_file is not None:
            rs = f'  <restartSimulation restartFileNumber="{self.restart_file}" AMRsaveFreq="0"/>\n'
        return ('<?xml version = "1.0" encoding = "UTF-8" standalone = "yes"?>\n<computationParam>\n'
                f'  <run>{self.name}</run>\n'
                f'  <outputMode format="{self.output_format}" binary="{binary}"{prec}/>\n'
                f'  {tc}\n  <computationControl CFL="{self.cfl!r}"/>\n{so}{rs}</computationParam>\n')

    def mesh_xml(self) -> str:
        lx, ly, lz = self.lengths
        nx, ny, nz = self.cells
        st = ""
        if self.stretch:  # Input::inputMesh src/InputOutput/Input.cpp:460-520
            st = "    <meshStretching>\n"
            for ax in ("x", "y", "z"):
                zones = self.stretch.get(ax)
                if not zones:
                    continue
                st += f"      <{ax.upper()}Stretching>\n"
                for a, b, f, n in zones:
                    st += f'        <stretch startAt="{a!r}" endAt="{b!r}" factor="{f!r}" numberCells="{n}"/>\n'
                st += f"      </{ax.upper()}Stretching>\n"
            st += "    </meshStretching>\n"
        return ('<?xml version = "1.0" encoding = "UTF-8" standalone = "yes"?>\n<mesh>\n'
                '  <type structure="cartesian"/>\n  <cartesianMesh>\n'
                f'    <dimensions x="{lx!r}" y="{ly!r}" z="{lz!r}"/>\n'
                f'    <numberCells x="{nx}" y="{ny}" z="{nz}"/>\n{st}  </cartesianMesh>\n</mesh>\n')

    def axis_cells(self, axis: int) -> Tuple[np.ndarray, np.ndarray]:
        """Cell sizes and centres along one axis (MeshCartesian::meshStretching
        src/Meshes/MeshCartesian.cpp:168-210, stretchZone::stretching src/Meshes/stretchZone.cpp:45-66)."""
        n, l = int(self.cells[axis]), float(self.lengths[axis])
        zones = (self.stretch or {}).get("xyz"[axis]) if n > 1 else None
        if not zones:
            d = l / float(n)
            return np.full(n, d), (np.arange(n) + 0.5) * d
        ds, ps = [], []
        for a, b, f, m in zones:
            d0 = (b - a) / m
            if abs(f - 1.0) < 1e-6:
                for i in range(m):
                    ds.append(d0)
                    ps.append(a + (i + 0.5) * d0)
            else:
                d0 = (b - a) * (1.0 - f) / (1.0 - math.pow(f, m))
                ds.append(d0)
                ps.append(a + 0.5 * d0)
                for i in range(1, m):
                    ds.append(d0 * math.pow(f, i))
                    ps.append(ps[-1] + 0.5 * (ds[-2] + ds[-1]))
        return np.array(ds), np.array(ps)

    def model_xml(self) -> str:
        s = '<?xml version = "1.0" encoding = "UTF-8" standalone = "yes"?>\n<model>\n'
        nt = len(self.transports or [])
        ntr = f' numberTransports="{nt}"' if nt else ""
        if self.model.upper() == "EULER":
            s += f'  <flowModel name="Euler"{ntr}/>\n'
        elif self.ptueq:  # Input::inputModel src/InputOutput/Input.cpp:642 (no alphaNull attribute)
            s += f'  <flowModel name="{self.model}" numberPhases="{self.nphases}"{ntr}/>\n'
        else:
            an = "true" if self.alpha_null else "false"
            s += f'  <flowModel name="{self.model}" numberPhases="{self.nphases}"{ntr} alphaNull="{an}"/>\n'
        for e in self.eos:
            s += f'  <EOS name="{e.name}"/>\n'
        for name in self.transports or []:
            s += f'  <transport name="{name}"/>\n'
        if self.ptmu is not None:
            liq, vap = self.ptmu
            s += ('  <relaxation type="PTMu">\n'
                  f'    <dataPTMu liquid="{self.eos[liq].name}" vapor="{self.eos[vap].name}"/>\n'
                  '  </relaxation>\n')
        if self.pt_relaxation:
            s += '  <relaxation type="PT"/>\n'
        return s + "</model>\n"

    def ic_xml(self) -> str:
        s = '<?xml version = "1.0" encoding = "UTF-8" standalone = "yes"?>\n<CI>\n  <physicalDomains>\n'
        for d in self.domains:
            s += "    " + d.xml() + "\n"
        s += "  </physicalDomains>\n  <boundaryConditions>\n"
        names = ["CLXm", "CLXp", "CLYm", "CLYp", "CLZm", "CLZp"]
        types = self.boundary_types()
        for i in range(2 * self.dim):
            s += f'    <boundCond name="{names[i]}" type="{types[i]}" number="{i + 1}"/>\n'
        s += "  </boundaryConditions>\n"
        euler = self.model.upper() == "EULER"
        for st in self.states:
            s += f'  <state name="{st.name}">\n'
            for k, ph in enumerate(st.phases):
                s += f'    <material type="fluid" EOS="{self.eos[k].name}">\n'
                if euler:
                    s += f'      <dataFluid density="{ph.density!r}" pressure="{st.pressure!r}">\n'
                    u = st.velocity
                    s += f'        <velocity x="{u[0]!r}" y="{u[1]!r}" z="{u[2]!r}"/>\n      </dataFluid>\n'
                elif self.ptueq:  # PhasePTUEq::PhasePTUEq: alpha only
                    s += f'      <dataFluid alpha="{ph.alpha!r}"/>\n'
                else:
                    attr = f'alpha="{ph.alpha!r}"'
                    if ph.temperature is not None:
                        attr += f' temperature="{ph.temperature!r}"'
                    else:
                        attr += f' density="{ph.density!r}"'
                    s += f"      <dataFluid {attr}/>\n"
                s += "    </material>\n"
            if self.ptueq:  # MixPTUEq::MixPTUEq src/Models/PTUEq/MixPTUEq.cpp:44: pressure and temperature
                u = st.velocity
                s += (f'    <mixture>\n      <dataMix pressure="{st.pressure!r}" temperature="{st.temperature!r}"/>\n'
                      f'      <velocity x="{u[0]!r}" y="{u[1]!r}" z="{u[2]!r}"/>\n    </mixture>\n')
            elif not euler:
                u = st.velocity
                s += (f'    <mixture>\n      <dataMix pressure="{st.pressure!r}"/>\n'
                      f'      <velocity x="{u[0]!r}" y="{u[1]!r}" z="{u[2]!r}"/>\n    </mixture>\n')
            for name, v in (st.transports or {}).items():
                s += f'    <transport name="{name}" value="{v!r}"/>\n'
            s += "  </state>\n"
        return s + "</CI>\n"

    def write(self, work: str, subdir: Optional[str] = None) -> str:
        """Write the case under ``work/<subdir>/`` and its EOS files under ``work/libEOS``.

        Returns the case folder path (with a trailing separator, as ECOGEN expects).
        """
        subdir = subdir or self.name
        cdir = os.path.join(work, subdir)
        os.makedirs(cdir, exist_ok=True)
        os.makedirs(os.path.join(work, "libEOS"), exist_ok=True)
        for e in self.eos:
            with open(os.path.join(work, "libEOS", e.name), "w") as f:
                f.write(e.xml())
        for fname, txt in (("main.xml", self.main_xml()), ("mesh.xml", self.mesh_xml()),
                           ("model.xml", self.model_xml()), ("initialConditions.xml", self.ic_xml())):
            with open(os.path.join(cdir, fname), "w") as f:
                f.write(txt)
        return cdir + os.sep


def write_ecogen_list(work: str, case_dirs: Sequence[str]) -> str:
    """Write ``work/ECOGEN.xml`` listing case folders (relative to work), as src/main.cpp:82 reads it."""
    s = "<?xml version='1.0' encoding='UTF-8' standalone='yes'?>\n<ecogen>\n"
    for d in case_dirs:
        rel = os.path.relpath(d, work).rstrip(os.sep) + "/"
        s += f"  <testCase>{rel}</testCase>\n"
    s += "</ecogen>\n"
    path = os.path.join(work, "ECOGEN.xml")
    with open(path, "w") as f:
        f.write(s)
    return path


# ----------------------------------------------------------------------------- named workloads


def shock_tube_1d(ncells: int = 1000, iterations: Optional[int] = None, total_time: Optional[float] = 240e-6,
                  order: Optional[str] = None, p_left: float = 1e9, x_interface: float = 0.7,
                  alpha_floor: float = 1e-6, name: str = "shockTube1D", liquid: Eos = WATER_SG,
                  alpha_null: bool = False) -> Case:
    """1D two-phase water/air shock tube on [0,1] m (Kapila, CFL 0.8, transmissive ends).

    Left of ``x_interface``: water-rich (alpha_water = 1-floor), p = ``p_left``;
    right: air-rich (alpha_water = floor), p = 1e5 Pa.  rho_water 1000, rho_air 50.
    """
    a = alpha_floor
    states = [
        State("airSide", [PhaseState(a, 1000.0), PhaseState(1.0 - a, 50.0)], 1.0e5),
        State("waterSide", [PhaseState(1.0 - a, 1000.0), PhaseState(a, 50.0)], p_left),
    ]
    domains = [Domain("base", "airSide", "entireDomain"),
               Domain("HP", "waterSide", "halfSpace", {"axis": "x", "origin": x_interface, "direction": "negative"})]
    if iterations is not None:
        total_time = None
    return Case(name, [liquid, AIR_IG], (1.0, 0.1, 0.1), (ncells, 1, 1), states, domains, alpha_null=alpha_null,
                cfl=0.8, iterations=iterations, total_time=total_time, second_order=order)


def sg_hugoniot_post_shock(eos: Eos, rho0: float, p0: float, p1: float) -> Tuple[float, float]:
    """Post-shock (rho1, u1) of a stiffened-gas shock running into fluid at rest.

    Rankine-Hugoniot for SG: rho1/rho0 = ((g+1)(p1+pinf) + (g-1)(p0+pinf)) / ((g-1)(p1+pinf) + (g+1)(p0+pinf));
    the piston velocity is u1 = sqrt((p1-p0)(1/rho0 - 1/rho1)).
    """
    g, pi = eos.gamma, eos.pinf
    ratio = ((g + 1) * (p1 + pi) + (g - 1) * (p0 + pi)) / ((g - 1) * (p1 + pi) + (g + 1) * (p0 + pi))
    rho1 = rho0 * ratio
    u1 = math.sqrt((p1 - p0) * (1.0 / rho0 - 1.0 / rho1))
    return rho1, u1


def shock_bubble_2d(n: int = 2048, iterations: int = 2000, limiter: str = "vanleer", alpha_floor: float = 1e-6,
                    length: float = 0.01, bubble_radius: float = 1e-3, shock_x: float = 2e-3,
                    name: str = "shockBubble2D") -> Case:
    """2D shock-bubble interaction: water at rest with one air bubble, hit by a planar water shock.

    n x n cells on a ``length`` square; bubble of ``bubble_radius`` at the centre; the post-shock
    region x <= ``shock_x`` holds the Rankine-Hugoniot state for p = 1e9 Pa (Kapila, MUSCL, CFL 0.6).
    """
    a = alpha_floor
    rho1, u1 = sg_hugoniot_post_shock(WATER_SG, 1000.0, 1.0e5, 1.0e9)
    states = [
        State("water", [PhaseState(1.0 - a, 1000.0), PhaseState(a, 1.2)], 1.0e5),
        State("bubble", [PhaseState(a, 1000.0), PhaseState(1.0 - a, 1.2)], 1.0e5),
        State("shocked", [PhaseState(1.0 - a, rho1), PhaseState(a, 1.2)], 1.0e9, (u1, 0.0, 0.0)),
    ]
    c = length / 2
    domains = [Domain("base", "water", "entireDomain"),
               Domain("bubble", "bubble", "disc", {"axis1": "x", "axis2": "y", "radius": bubble_radius,
                                                  "center": (c, c, 0.0)}),
               Domain("shock", "shocked", "halfSpace", {"axis": "x", "origin": shock_x, "direction": "negative"})]
    return Case(name, [WATER_SG, AIR_IG], (length, length, 1.0), (n, n, 1), states, domains,
                cfl=0.6, iterations=iterations, second_order=limiter)


def cavity_collapse_3d(n: int = 256, iterations: int = 100, seed: int = 12345, ninclusions: int = 64,
                       limiter: str = "minmod", alpha_floor: float = 1e-6, length: float = 0.01,
                       radius_cells: Tuple[float, float] = (3.0, 10.0), name: str = "cavityCollapse3D") -> Case:
    """3D three-phase collapse: liquid at 5e7 Pa with ``ninclusions`` gas spheres (gas A or B, 1e5 Pa).

    Radii are uniform in ``radius_cells`` (in cells), centres uniform in the box, drawn from ``seed``.
    """
    rng = np.random.default_rng(seed)
    a = alpha_floor
    dx = length / n
    states = [
        State("liquid", [PhaseState(1.0 - 2 * a, 1000.0), PhaseState(a, 1.2), PhaseState(a, 0.16)], 5.0e7),
        State("gasA", [PhaseState(a, 1000.0), PhaseState(1.0 - 2 * a, 1.2), PhaseState(a, 0.16)], 1.0e5),
        State("gasB", [PhaseState(a, 1000.0), PhaseState(a, 1.2), PhaseState(1.0 - 2 * a, 0.16)], 1.0e5),
    ]
    domains = [Domain("base", "liquid", "entireDomain")]
    for i in range(ninclusions):
        r = float(rng.uniform(*radius_cells)) * dx
        cx, cy, cz = (float(v) for v in rng.uniform(0.0, length, size=3))
        gas = "gasA" if rng.uniform() < 0.5 else "gasB"
        domains.append(Domain(f"inc{i}", gas, "sphere", {"radius": r, "center": (cx, cy, cz)}))
    return Case(name, [WATER_SG, AIR_IG, GAS_B_IG], (length, length, length), (n, n, n), states, domains,
                cfl=0.6, iterations=iterations, second_order=limiter, extra={"seed": seed})


def batch_shock_tubes(ncases: int = 4096, seed: int = 2024, cells_range: Tuple[int, int] = (200, 8000),
                      iterations: int = 1000, limiter: Optional[str] = "vanleer", alpha_floor: float = 1e-6
                      ) -> List[Case]:
    """Independent 1D water/air shock tubes with seeded uneven sizes and loads (batched mode).

    Cells log-uniform in ``cells_range``; interface uniform in [0.3, 0.7]; left pressure
    log-uniform in [1e6, 1e9] Pa; right 1e5 Pa; per-case CFL 0.8.
    """
    rng = np.random.default_rng(seed)
    lo, hi = cells_range
    cases = []
    for c in range(ncases):
        n = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        xi = float(rng.uniform(0.3, 0.7))
        pl = float(math.exp(rng.uniform(math.log(1e6), math.log(1e9))))
        case = shock_tube_1d(ncells=max(n, 2), iterations=iterations, order=limiter, p_left=pl, x_interface=xi,
                             alpha_floor=alpha_floor, name=f"tube{c:05d}")
        cases.append(case)
    return cases


def expansion_tube_2d(n: int = 1024, iterations: int = 100, limiter: str = "vanleer", alpha_vap: float = 1e-2,
                      velocity: float = 500.0, length: float = 1.0, name: str = "expansionTube2D") -> Case:
    """2D liquid/vapour expansion with pressure + thermal + chemical (p-T-mu) relaxation.

    Liquid with alpha_vap = 1e-2 at 1e5 Pa and 355 K everywhere; inside the centre strip
    |y - L/2| <= L/4 the left half moves at -``velocity`` and the right half at +``velocity``.
    """
    T = 355.0
    states = [
        State("rest", [PhaseState(1.0 - alpha_vap, temperature=T), PhaseState(alpha_vap, temperature=T)], 1.0e5),
        State("left", [PhaseState(1.0 - alpha_vap, temperature=T), PhaseState(alpha_vap, temperature=T)], 1.0e5,
              (-velocity, 0.0, 0.0)),
        State("right", [PhaseState(1.0 - alpha_vap, temperature=T), PhaseState(alpha_vap, temperature=T)], 1.0e5,
              (velocity, 0.0, 0.0)),
    ]
    L = length
    domains = [Domain("base", "rest", "entireDomain"),
               Domain("left", "left", "rectangle", {"axis1": "x", "axis2": "y", "l1": L / 2, "l2": L / 2,
                                                   "corner": (0.0, L / 4, 0.0)}),
               Domain("right", "right", "rectangle", {"axis1": "x", "axis2": "y", "l1": L / 2, "l2": L / 2,
                                                     "corner": (L / 2, L / 4, 0.0)})]
    return Case(name, [LIQ_PC, VAP_PC], (L, L, 1.0), (n, n, 1), states, domains, alpha_null=True,
                cfl=0.5, iterations=iterations, second_order=limiter, ptmu=(0, 1))


def euler_shock_tube(ncells: int = 400, iterations: int = 50, order: Optional[str] = None,
                     name: str = "eulerShockTube") -> Case:
    """Single-phase air shock tube (Euler model; reference src/Models/Euler)."""
    states = [State("low", [PhaseState(1.0, 1.0)], 1.0e5), State("high", [PhaseState(1.0, 10.0)], 1.0e6)]
    domains = [Domain("base", "low", "entireDomain"),
               Domain("HP", "high", "halfSpace", {"axis": "x", "origin": 0.5, "direction": "negative"})]
    return Case(name, [AIR_IG], (1.0, 0.1, 0.1), (ncells, 1, 1), states, domains, model="Euler",
                cfl=0.8, iterations=iterations, second_order=order)


def ptueq_shock_tube_1d(ncells: int = 400, iterations: Optional[int] = 50, total_time: Optional[float] = None,
                        order: Optional[str] = "vanleer", p_left: float = 1.0e8, x_interface: float = 0.7,
                        alpha_floor: float = 1e-6, name: str = "ptueqShockTube1D",
                        boundaries: Optional[List[str]] = None, transports: Optional[List[str]] = None) -> Case:
    """1D water/air shock tube in temperature-pressure-velocity equilibrium (PTUEq model).

    Air (IG) and water (SG) phases; left of ``x_interface`` water-rich at ``p_left`` and 341.5 K,
    right of it air-rich at 1e5 Pa and 300 K, at rest (the layout of the reference's PTUEq
    water/air shock tube, without its AMR).  With ``transports`` each side carries 0 / 1.
    """
    a = alpha_floor
    tr_w = {t: 1.0 for t in transports or []}
    tr_a = {t: 0.0 for t in transports or []}
    states = [
        State("water", [PhaseState(a), PhaseState(1.0 - a)], p_left, temperature=341.5, transports=tr_w or None),
        State("air", [PhaseState(1.0 - a), PhaseState(a)], 1.0e5, temperature=300.0, transports=tr_a or None),
    ]
    domains = [Domain("left", "water", "entireDomain"),
               Domain("right", "air", "halfSpace", {"axis": "x", "origin": x_interface, "direction": "positive"})]
    return Case(name, [AIR_IG, WATER_SG300], (1.0, 0.1, 0.1), (ncells, 1, 1), states, domains, model=PTUEQ,
                cfl=0.8, iterations=iterations, total_time=total_time if iterations is None else None,
                second_order=order, boundaries=boundaries, transports=transports)


def ptueq_bubble_2d(n: int = 64, iterations: int = 20, limiter: Optional[str] = "vanleer", alpha_floor: float = 1e-6,
                    name: str = "ptueqBubble2D", ny: Optional[int] = None, nz: int = 1,
                    boundaries: Optional[List[str]] = None) -> Case:
    """2D air bubble in water hit by a planar pressure wave, PTUEq model, on a 1 cm square
    (with ``nz`` > 1, a 1 cm cube crossed by an air cylinder along z).

    Water at 1e5 Pa / 300 K with an air disc (radius 2 mm) at the centre; the water left of
    x = 2 mm is at 1e8 Pa / 320 K and moves at +50 m/s.
    """
    a = alpha_floor
    states = [
        State("water", [PhaseState(a), PhaseState(1.0 - a)], 1.0e5, temperature=300.0),
        State("hp", [PhaseState(a), PhaseState(1.0 - a)], 1.0e8, (50.0, 0.0, 0.0), temperature=320.0),
        State("air", [PhaseState(1.0 - a), PhaseState(a)], 1.0e5, temperature=300.0),
    ]
    L = 0.01
    domains = [Domain("base", "water", "entireDomain"),
               Domain("bubble", "air", "disc", {"axis1": "x", "axis2": "y", "radius": 0.002,
                                                "center": (0.5 * L, 0.5 * L, 0.0)}),
               Domain("HP", "hp", "halfSpace", {"axis": "x", "origin": 0.002, "direction": "negative"})]
    return Case(name, [AIR_IG, WATER_SG300], (L, L, L if nz > 1 else 1.0), (n, ny or n, nz), states, domains,
                model=PTUEQ,
                cfl=0.6, iterations=iterations, second_order=limiter, boundaries=boundaries)


def euler_blast_2d(n: int = 64, ny: Optional[int] = None, nz: int = 1, iterations: int = 20,
                   order: Optional[str] = "vanleer", name: str = "eulerBlast2D",
                   boundaries: Optional[List[str]] = None) -> Case:
    """Single-phase air (Euler model) on a 1 m square (a 1 m cube with ``nz`` > 1): a dense,
    high-pressure disc (a cylinder along z in 3D) off the centre, moving air left of x = 0.2 m."""
    states = [State("ambient", [PhaseState(1.0, 1.0)], 1.0e5),
              State("blast", [PhaseState(1.0, 5.0)], 1.0e6),
              State("inflow", [PhaseState(1.0, 1.5)], 2.0e5, (80.0, 20.0, 0.0))]
    domains = [Domain("base", "ambient", "entireDomain"),
               Domain("blast", "blast", "disc", {"axis1": "x", "axis2": "y", "radius": 0.15,
                                                "center": (0.55, 0.45, 0.5)}),
               Domain("inflow", "inflow", "halfSpace", {"axis": "x", "origin": 0.2, "direction": "negative"})]
    return Case(name, [AIR_IG], (1.0, 1.0, 1.0 if nz > 1 else 0.1), (n, ny or n, nz), states, domains,
                model="Euler", cfl=0.6, iterations=iterations, second_order=order, boundaries=boundaries)
