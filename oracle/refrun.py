"""Runs the reference ECOGEN binary built by ``oracle/Makefile`` and reads its results.

Test infrastructure only.  The reference writes its fields as VTK rectilinear
files with base64 Float64 payloads when ``outputMode format="XML"
binary="true"`` (reference src/InputOutput/OutputXML.cpp:320 writeResultsXML,
src/InputOutput/Output.cpp:372 writeDataset, src/InputOutput/IO.cpp:40
writeb64Chaine: a base64 4-byte length header followed by the base64 data).
Cells are written in k, j, i order, which is the cell index order
i + j*Nx + k*Nx*Ny (src/Meshes/MeshCartesian.cpp:1820 getData).
"""
from __future__ import annotations

import base64
import glob
import os
import re
import subprocess
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BINARY = os.path.join(HERE, "_ref", "ECOGEN")

_ARRAY_RE = re.compile(r'<DataArray type="Float64" Name="([^"]+)"(?: NumberOfComponents="(\d)")? format="binary">\s*'
                       r'([A-Za-z0-9+/=]+)\s*</DataArray>')


def _decode(payload: str) -> np.ndarray:
    head = base64.b64decode(payload[:8])
    nbytes = int(np.frombuffer(head, dtype="<i4")[0])
    data = base64.b64decode(payload[8:])
    return np.frombuffer(data[:nbytes], dtype="<f8").copy()


_ASCII_RE = re.compile(r'<DataArray type="Float64" Name="([^"]+)"(?: NumberOfComponents="(\d)")? format="ascii">'
                       r'([^<]*)</DataArray>')


def read_vtr(path: str) -> Dict[str, np.ndarray]:
    """Read every named Float64 cell array of one reference ``.vtr`` result file (base64 or ASCII)."""
    with open(path) as f:
        txt = f.read()
    out: Dict[str, np.ndarray] = {}
    for name, ncomp, payload in _ARRAY_RE.findall(txt):
        arr = _decode(payload)
        if ncomp:
            arr = arr.reshape(-1, int(ncomp))
        out[name] = arr
    for name, ncomp, payload in _ASCII_RE.findall(txt):
        arr = np.array([float(x) for x in payload.split()], dtype=np.float64)
        if ncomp:
            arr = arr.reshape(-1, int(ncomp))
        out[name] = arr
    return out


def read_vtr_ordered(path: str):
    """(name, array) of every cell array in document order (the order a restart reads them in)."""
    with open(path) as f:
        txt = f.read()
    body = txt[txt.index("<CellData>"):]
    items = []
    for m in re.finditer(r'<DataArray type="Float64" Name="([^"]+)"(?: NumberOfComponents="(\d)")? '
                         r'format="(ascii|binary)">([^<]*)</DataArray>', body):
        name, ncomp, fmt, payload = m.groups()
        arr = _decode(payload.strip()) if fmt == "binary" else np.array([float(x) for x in payload.split()])
        items.append((name, arr.reshape(-1, int(ncomp)) if ncomp else arr))
    return items


def result_file(work: str, run_name: str, number: int, binary: bool = True) -> str:
    """Path of result file ``number`` (OutputXML::createFilenameXML: result[B64]_CPU0_TIME<k>.vtr)."""
    return os.path.join(work, "results", run_name, "datasets",
                        f"result{'B64' if binary else ''}_CPU0_TIME{number}.vtr")


def available() -> bool:
    return os.path.isfile(REF_BINARY) and os.access(REF_BINARY, os.X_OK)


def run(work: str, binary: Optional[str] = None, timeout: float = 3600.0) -> subprocess.CompletedProcess:
    """Run the reference on ``work/ECOGEN.xml`` (its only argument is the work folder, src/main.cpp:66)."""
    binary = binary or REF_BINARY
    work = os.path.abspath(work) + os.sep
    return subprocess.run([binary, work], cwd=work, capture_output=True, text=True, timeout=timeout)


def result_files(work: str, run_name: str):
    files = glob.glob(os.path.join(work, "results", run_name, "datasets", "resultB64_CPU0_TIME*.vtr"))
    return sorted(files, key=lambda p: int(re.search(r"TIME(\d+)\.vtr$", p).group(1)))


def final_fields(work: str, run_name: str) -> Dict[str, np.ndarray]:
    files = result_files(work, run_name)
    if not files:
        raise FileNotFoundError(f"no reference results for {run_name} under {work}")
    return read_vtr(files[-1])


def info(work: str, run_name: str):
    """Last (iteration, time, dt) line of infoCalcul.out (6 significant digits)."""
    with open(os.path.join(work, "results", run_name, "infoCalcul.out")) as f:
        rows = [ln.split() for ln in f if ln.strip()]
    last = rows[-1]
    return int(last[1]), float(last[2]), float(last[3])


def _transports(fields: Dict[str, np.ndarray]):
    """Passive transports, written as T1, T2, ... (OutputXML::writePhysicalDataXML)."""
    out, k = [], 1
    while f"T{k}" in fields:
        out.append(fields[f"T{k}"])
        k += 1
    return np.stack(out) if out else None


def reference_prim(fields: Dict[str, np.ndarray], nphases: int):
    """Map reference output names to (alpha[k], rho[k], p, u[3], E, tr) arrays (PUEq, PTUEq or Euler output)."""
    if "Pressure_Mixture" not in fields:  # Euler: PhaseEuler scalars + velocity (no total energy written)
        get = lambda pre: [v for n, v in fields.items() if n.startswith(pre)][0]
        rho = get("F0_Density")
        return {"alpha": np.ones((1, rho.size)), "rho": rho[None, :], "p": get("F0_Pressure"),
                "u": get("F0_Velocity").T.copy(), "E": None, "rho_mix": rho, "T": get("F0_Temperature")[None, :],
                "tr": _transports(fields)}
    if "Temperature_Mixture" in fields:  # PTUEq: PhasePTUEq (Alpha, Density), MixPTUEq (rho, p, T, velocity)
        alpha = np.stack([[v for n, v in fields.items() if n.startswith(f"F{k}_Alpha")][0] for k in range(nphases)])
        rho = np.stack([[v for n, v in fields.items() if n.startswith(f"F{k}_Density")][0] for k in range(nphases)])
        Tm = fields["Temperature_Mixture"]
        return {"alpha": alpha, "rho": rho, "p": fields["Pressure_Mixture"],
                "u": fields["Velocity_Mixture_norm"].T.copy(), "E": None, "rho_mix": fields["Density_Mixture"],
                "T": np.stack([Tm] * nphases), "Tm": Tm, "tr": _transports(fields)}
    alpha, rho = [], []
    for k in range(nphases):
        a = [v for n, v in fields.items() if n.startswith(f"F{k}_Alpha")]
        r = [v for n, v in fields.items() if n.startswith(f"F{k}_Density")]
        alpha.append(a[0])
        rho.append(r[0])
    return {
        "alpha": np.stack(alpha),
        "rho": np.stack(rho),
        "p": fields["Pressure_Mixture"],
        "u": fields["Velocity_Mixture"].T.copy(),
        "E": fields["Total_energy_Mixture"],
        "rho_mix": fields["Density_Mixture"],
        "T": np.stack([[v for n, v in fields.items() if n.startswith(f"F{k}_Temperature")][0] for k in range(nphases)]),
        "tr": _transports(fields),
    }
