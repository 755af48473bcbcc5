"""Benchmark: cell-updates/s of the ECOGEN Cartesian FV step on one B200 (or N replicas).

Default workload (the largest single-GPU configuration of the metric, the one the learned-seed target
is quoted on): 3D three-phase cavity collapse, Kapila model, MUSCL-Hancock + minmod, FP64, 256^3 cells,
64 seeded spherical gas inclusions (two ideal gases in a stiffened-gas liquid), CFL 0.6 -- seeded
synthetic input generated by ecogen_b200.cases.cavity_collapse_3d and read through the library's own
XML reader.  The line reports the plain FP64 path (`value`) and the same workload with the learned
pressure-relaxation seed installed (`mlp_seeded`; c5: the (p*, T) seed of the p-T-mu saturation
solve), and beside it the ceiling of any pressure seed: the plain step with Newton stopped after one
(three) evaluations (`mlp_seeded.ceiling`); c5 also reports the p-T-mu warm start without a network
(`ptmu_warm_start`).  One "step" is one full time step of the whole
grid (predictor + corrector + relaxations + dt update).  The state (256^3 x 11 doubles = 1.48 GB per
copy) is larger than L2, so no L2 flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config c3|c2|c1|c4|c5|p2|e2]

c2 is the 2D shock-bubble (Kapila 2-phase, MUSCL + van Leer, 2048^2), c1 the 1000-cell first-order
tube, c4 4096 batched 1D tubes, c5 the 1024^2 p-T-mu expansion, p2 / e2 the PTUEq and Euler models.
Other workloads' lines say in config.l2 whether their data exceeds L2 (the 1D tube of 1000 cells is
L2-resident: a latency-bound configuration, not a bandwidth measurement).

Two rooflines are reported for the dominant kernel: HBM (algorithmic bytes over the measured copy
bandwidth) and FP64 (FP64 thread instructions per cell, counted by ncu on one launch, over the FP64
pipe rate measured live by a DFMA-throughput probe).

Multi-GPU: the path does not shard (one case per GPU; a single large domain would need halo
exchange, which this workload does not use), so N ranks run N independent replicas ("replicas
only"); value = total cell-updates of all ranks / max-over-ranks device time.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s on 1 B200: plain FP64 vs MLP-seeded relaxation, same residual"


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def make_case(config: str, size: int | None):
    from ecogen_b200 import cases
    if config == "c1":
        return cases.shock_tube_1d(ncells=size or 1000, iterations=10 ** 6)
    if config == "c3":
        return cases.cavity_collapse_3d(n=size or 256, iterations=10 ** 6)
    if config == "c5":
        return cases.expansion_tube_2d(n=size or 1024, iterations=10 ** 6)
    if config == "p2":
        return cases.ptueq_bubble_2d(n=size or 2048, iterations=10 ** 6)
    if config == "e2":
        return cases.euler_blast_2d(n=size or 2048, iterations=10 ** 6)
    if config == "c4":
        # one case of the batched workload (its per-case reference timing)
        return cases.shock_tube_1d(ncells=1000, iterations=10 ** 6, order="vanleer")
    return cases.shock_bubble_2d(n=size or 2048, iterations=10 ** 6)


def seed_model_path(config: str, nphases: int) -> str:
    """The shipped seed model of a workload family (1D tubes have their own)."""
    models = os.path.join(ROOT, "ecogen_b200", "models")
    if config == "c5":  # the (p*, T) seed of the p-T-mu saturation solve
        return os.path.join(models, "seed_ptmu.npz")
    if config in ("c1", "c4"):
        p = os.path.join(models, "seed_np2_tube1d.npz")
        if os.path.exists(p):
            return p
    return os.path.join(models, f"seed_np{nphases}.npz")


def state_fields(case) -> int:
    """Doubles per cell of the stored state: (alpha_k, rho_k)_k, p, u (d components), E; for the
    temperature-pressure equilibrium model alpha_k, p, T, u, E."""
    if getattr(case, "ptueq", False):
        return case.nphases + 3 + case.dim
    per_phase = 1 if case.model.upper() == "EULER" else 2
    return per_phase * case.nphases + 2 + case.dim


L2_BYTES = 126 * 2 ** 20


def l2_note(case) -> str:
    """Whether one step's data (the state read, the state written, the MUSCL half-step state) exceeds L2."""
    state = 8 * state_fields(case) * case.ncells
    ws = state * (3 if case.second_order else 2)
    if state > L2_BYTES:
        return f"state {state / 1e6:.0f} MB per copy, larger than the 126 MB L2 (no flush needed)"
    if ws > L2_BYTES:
        return (f"state {state / 1e6:.0f} MB per copy, {ws / 1e6:.0f} MB touched per step, more than the 126 MB L2; "
                "no flush between steps (part of the state stays L2-resident)")
    return (f"state {state / 1e6:.2f} MB: L2-resident, no flush between steps (a latency-bound configuration, "
            "not a bandwidth measurement)")


def bytes_per_cell_update(case) -> int:
    """Minimal algorithmic bytes of one step: read and write the state once."""
    return 16 * state_fields(case)


def pass_bytes_per_cell(case) -> dict:
    """Algorithmic bytes per cell of each step kernel.

    MUSCL predictor: reads S^n (NS doubles), writes S^{n+1/2} without E (NS - 1).
    MUSCL corrector: reads S^{n+1/2} (NS - 1) and S^n (NS), writes S^{n+1} (NS).
    First order: reads S^n, writes S^{n+1}.
    """
    ns = state_fields(case)
    if case.second_order:
        return {"pass1": 8 * (2 * ns - 1), "pass2": 8 * (3 * ns - 1)}
    return {"pass1": 16 * ns}


# Per-kernel slots of ecg_step_profiled_kernels: pass 1 (first order or MUSCL predictor) X / Y / Z face
# kernels and cell kernel, pass 2 (MUSCL corrector) the same, time-step update.  In fused form a
# pass is one kernel, timed in its cell-kernel slot.
KERNEL_SLOTS = ["pass1_faces_x", "pass1_faces_y", "pass1_faces_z", "pass1_cells",
                "pass2_faces_x", "pass2_faces_y", "pass2_faces_z", "pass2_cells", "update"]


def kernel_bytes_per_cell(case, form: str, slot: str) -> int:
    """Algorithmic bytes per cell of one launch of a step kernel.

    Fused form: the pass's bytes (pass_bytes_per_cell).  Split form, face kernel of one axis: read the
    pass's input state (NS - 1 fields; the corrector also the time-n alpha_0), write one flux
    (3N + d + 3 doubles) per face; cell kernel: read the d faces' fluxes per cell, S^n (NS), write the
    output state (NS, the predictor NS - 1)."""
    ns = state_fields(case)
    pb = pass_bytes_per_cell(case)
    if form != "split" or case.dim < 2:
        return pb["pass2" if slot.startswith("pass2") else "pass1"]
    nfl = 3 * case.nphases + case.dim + 3
    corr = slot.startswith("pass2")
    pred = slot.startswith("pass1") and case.second_order
    if "_faces_" in slot:
        return 8 * ((ns - 1) + (1 if corr else 0) + nfl)
    return 8 * (case.dim * nfl + ns + (ns - 1 if pred else ns))


def kernel_label(case, form: str, slot: str) -> str:
    euler, ptueq = case.model.upper() == "EULER", getattr(case, "ptueq", False)
    base = "k_euler_step" if euler else ("k_ptueq_step" if ptueq else "k_kapila_step")
    pas = ("MUSCL corrector" if slot.startswith("pass2") else
           ("MUSCL predictor" if case.second_order else "first-order step"))
    if form == "split" and case.dim >= 2 and not euler and not ptueq:
        if "_faces_" in slot:
            return f"k_kapila_faces, {slot[-1].upper()} faces ({pas})"
        return f"k_kapila_cells ({pas})"
    return f"{base} ({pas})"


def launches_per_step(case, form: str) -> int:
    passes = 2 if case.second_order else 1
    per_pass = (case.dim + 1) if (form == "split" and case.dim >= 2) else 1
    return passes * per_pass + 1


# DRAM bytes per cell of the step kernels measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum
# of one launch / cells: 2D two-phase MUSCL at 1536^2, 3D three-phase MUSCL at 128^3, 2D PTUEq MUSCL at
# 1536^2, 2D p-T-mu at 1536^2, 2D Euler at 2048^2).  The kernels stream the state once, so traffic
# scales with the cell count.
NCU_TRAFFIC_PER_CELL = {("kapila", 2, 2, True, "fused", "pass2_cells"): 190.96,
                        ("kapila", 2, 2, True, "fused", "pass1_cells"): 125.14,
                        ("kapila", 3, 3, True, "fused", "pass2_cells"): 250.27,
                        ("kapila", 3, 3, True, "fused", "pass1_cells"): 155.89,
                        ("ptueq", 2, 2, True, "fused", "pass2_cells"): 150.78,
                        ("ptueq", 2, 2, True, "fused", "pass1_cells"): 91.56,
                        ("kapila_ptmu", 2, 2, True, "fused", "pass2_cells"): 181.05,
                        ("kapila_ptmu", 2, 2, True, "fused", "pass1_cells"): 112.08,
                        ("euler", 1, 2, True, "fused", "pass2_cells"): 98.52,
                        ("euler", 1, 2, True, "fused", "pass1_cells"): 64.92}
# Split form: DRAM bytes per unit of the kernel (faces of its axis for a face kernel, cells for the cell
# kernel), ncu on one launch at 1536^2 (2D two-phase), 128^3 (3D three-phase) and 1024^2 (p-T-mu); the
# traffic of a launch grows with its units, so a full-size launch is the per-unit figure times its units.
_SPLIT_NCU = {  # (model, phases, dim): {slot: (FP64 thread instructions per unit, DRAM bytes per unit)}
    ("kapila", 2, 2): {"pass1_faces_x": (742, 124), "pass1_faces_y": (751, 123), "pass1_cells": (498, 290),
                       "pass2_faces_x": (742, 133), "pass2_faces_y": (751, 132), "pass2_cells": (498, 297)},
    ("kapila", 3, 3): {"pass1_faces_x": (988, 184), "pass1_faces_y": (1003, 183), "pass1_faces_z": (997, 181),
                       "pass1_cells": (879, 534), "pass2_faces_x": (982, 191), "pass2_faces_y": (1005, 191),
                       "pass2_faces_z": (999, 190), "pass2_cells": (899, 542)},
    ("kapila_ptmu", 2, 2): {"pass1_faces_x": (753, 96), "pass1_faces_y": (763, 95), "pass1_cells": (1722, 303),
                            "pass2_faces_x": (753, 105), "pass2_faces_y": (763, 106), "pass2_cells": (1731, 310)},
}
for (_m, _np, _d), _slots in _SPLIT_NCU.items():
    for _slot, (_fp, _dram) in _slots.items():
        NCU_TRAFFIC_PER_CELL[(_m, _np, _d, True, "split", _slot)] = float(_dram)
# Batched tubes (2048 cases): predictor + corrector DRAM bytes per cell-update.
NCU_BATCH_BYTES_PER_CELL_UPDATE = 98.05 + 157.17


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while the timed region runs."""

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t0 = time.time()
            while not self.rows and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.02)  # the timed region starts once sampling runs
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def fp64_pipe_peak(device_index: int):
    """FP64 pipe rate of this GPU in thread instructions per second, measured live by the DFMA
    throughput probe (ecogen_b200/libecg_probe.so), with the SM clock sampled meanwhile."""
    import ctypes as C
    path = os.path.join(ROOT, "ecogen_b200", "libecg_probe.so")
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    lib.ecg_probe_fp64.argtypes = [C.c_int, C.c_longlong, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    rate, ms = C.c_double(), C.c_double()
    with ClockSampler(device_index) as clk:
        rc = lib.ecg_probe_fp64(8, 1 << 19, 5, C.byref(rate), C.byref(ms))
    if rc != 0:
        return None
    return {"dfma_per_s": rate.value, "launch_ms": ms.value, "clocks": clk.summary(),
            "how": "148 SMs x 8 blocks x 256 threads, 8 independent DFMA chains per thread, best of 5 launches"}


# FP64 thread instructions per unit (face or cell) of one launch of a step kernel, counted by ncu
# (smsp__sass_thread_inst_executed_op_fp64_pred_on.sum / units), keyed like NCU_TRAFFIC_PER_CELL.  The
# count does not depend on the mesh size beyond boundary cells (measured at 1536^2 in 2D, 128^3 in 3D,
# 1024^2 for the p-T-mu workload).
NCU_FP64_PER_CELL: dict = {(_m, _np, _d, True, "split", _slot): float(_fp)
                           for (_m, _np, _d), _slots in _SPLIT_NCU.items() for _slot, (_fp, _dram) in _slots.items()}


def kernel_units(case, form: str, slot: str) -> int:
    """Units one launch of a step kernel processes: faces of its axis for a split-form face kernel
    (n_AX + 1 times the other two), cells otherwise."""
    if form == "split" and "_faces_" in slot:
        ax = "xyz".index(slot[-1])
        n = list(case.cells)
        n[ax] += 1
        return n[0] * n[1] * n[2]
    return case.ncells


def max_over_ranks(value: float, device: str) -> float:
    """Max of a per-rank device time over all ranks of the default process group (if any)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ----------------------------------------------------------------------------------- reference arm


# Per-process mesh of the reference sample of each workload: large enough that the step dominates the
# reference's set-up, small enough that a sample of a few iterations takes seconds on one core
# (reference, one core: 2D 256^2 MUSCL ~0.9 s per step, 3D 32^3 three-phase MUSCL ~0.7 s per step).
REF_SAMPLE_SIZE = {"c1": 1000, "c3": 32, "c4": None}
# iterations of a sample's long run (the 1D tubes take milliseconds per step)
REF_SAMPLE_ITERS = {"c1": 200, "c4": 200}
REF_SAMPLE_BUDGET_S = 150.0


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_sample(steps: int, warmup: int, iters: int | None = None, procs: int | None = None,
                     config: str = "c3", budget_s: float = REF_SAMPLE_BUDGET_S):
    """Time the reference CPU solver (oracle/_ref/ECOGEN, built from the reference sources).

    Each sample runs `procs` independent reference processes concurrently (one per host core; the
    reference has no threads and no MPI exists on the box) on a reduced mesh of the workload
    (REF_SAMPLE_SIZE) for `iters` iterations, and once for 1 iteration; the difference removes
    initialisation and output, giving cell-updates/s over all cores.  Samples stop after
    `warmup + steps` or once `budget_s` seconds have passed with at least one timed sample.
    """
    from ecogen_b200 import cases
    from oracle import refrun
    if not refrun.available():
        return None
    procs = procs or len(os.sched_getaffinity(0))
    size = REF_SAMPLE_SIZE.get(config, 256)
    iters = iters or REF_SAMPLE_ITERS.get(config, 4)
    base = tempfile.mkdtemp(prefix="ecg_ref_")

    def prepare(nit):
        dirs = []
        for p in range(procs):
            w = os.path.join(base, f"n{nit}_p{p}")
            c = make_case(config, size)
            c.iterations = nit
            c.name = f"refsample{p}"
            d = c.write(w)
            cases.write_ecogen_list(w, [d])
            dirs.append(w)
        return dirs

    def run_all(dirs):
        t0 = time.perf_counter()
        ps = [subprocess.Popen([refrun.REF_BINARY, os.path.abspath(w) + os.sep], cwd=w, stdout=subprocess.DEVNULL,
                               stderr=subprocess.DEVNULL) for w in dirs]
        for p in ps:
            p.wait()
        return time.perf_counter() - t0

    d1, dn = prepare(1), prepare(iters)
    c = make_case(config, size)
    cells = c.ncells
    samples = []
    start = time.perf_counter()
    for i in range(warmup + steps):
        t1 = run_all(d1)
        tn = run_all(dn)
        if i >= warmup:
            samples.append(procs * cells * (iters - 1) / max(tn - t1, 1e-9))
        if samples and time.perf_counter() - start > budget_s:
            break
    shutil.rmtree(base, ignore_errors=True)
    mesh = "x".join(str(n) for n in c.cells if n > 1)
    return {"value": statistics.median(samples), "cores": procs, "cpu": cpu_model(),
            "sample": f"{procs} concurrent reference processes (one per core of a {cpu_model()}), {mesh} cells each, "
                      f"{iters}-1 iterations (time of an {iters}-iteration run minus a 1-iteration run); "
                      f"{len(samples)} timed samples, median", "samples": samples}


# ------------------------------------------------------------------------------------ batched mode


def bench_batch(args, rank, world, local):
    """Batched independent 1D shock tubes (persistent work-queue kernel, per-case dt)."""
    import ctypes as C

    import torch
    from ecogen_b200 import api, cases
    torch.cuda.set_device(local if world > 1 else 0)
    ncases = args.size or 4096
    specs = cases.batch_shock_tubes(ncases=ncases, seed=2024 + rank, iterations=1000)
    work = tempfile.mkdtemp(prefix=f"ecg_batch_{rank}_")
    recs, fields = [], []
    for i, c in enumerate(specs):
        d = c.write(work, subdir=f"c{i}")
        inp = api.Input(d, os.path.join(work, "libEOS"))
        recs.append(inp.case)
        fields.append(inp.fill())
    shutil.rmtree(work, ignore_errors=True)
    arr = (api.Case * len(recs))(*recs)
    cat = [np.ascontiguousarray(np.concatenate([f[k] for f in fields])) for k in range(len(fields[0]))]
    h = C.c_void_p()
    api.check(api.lib().ecg_batch_create(arr, len(recs), C.byref(h)), "ecg_batch_create")
    total = int(api.lib().ecg_batch_total_cells(h))
    api.check(api.lib().ecg_batch_upload_prim(h, api._field_ptrs(cat), total), "upload")
    tile, th = C.c_int32(), C.c_int32()
    api.check(api.lib().ecg_batch_autotune(h, C.byref(tile), C.byref(th)), "autotune")
    st = api.StepStats()
    api.check(api.lib().ecg_batch_step(h, args.warmup, None, None, C.byref(st)), "warmup")
    stream = torch.cuda.ExternalStream(api.lib().ecg_batch_stream(h))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        api.check(api.lib().ecg_batch_step(h, args.steps, None, None, C.byref(st)), "step")
        e1.record(stream)
        e1.synchronize()
    dt_s = max_over_ranks(e0.elapsed_time(e1), "cuda") * 1e-3
    value = total * args.steps / dt_s
    api.lib().ecg_batch_destroy(h)

    # the same batch with the learned seed installed (fresh copy of the initial state)
    seeded = None
    model_path = seed_model_path("c4", recs[0].nphases)
    if not args.no_seeded and os.path.exists(model_path):
        from ecogen_b200 import seed as seedmod
        model = seedmod.SeedModel.load(model_path)
        h2 = C.c_void_p()
        api.check(api.lib().ecg_batch_create(arr, len(recs), C.byref(h2)), "ecg_batch_create")
        api.check(api.lib().ecg_batch_upload_prim(h2, api._field_ptrs(cat), total), "upload")
        api.check(api.lib().ecg_batch_set_shape(h2, tile, th), "set_shape")
        model.install_batch(h2)
        st2 = api.StepStats()
        api.check(api.lib().ecg_batch_step(h2, args.warmup, None, None, C.byref(st2)), "warmup")
        stream2 = torch.cuda.ExternalStream(api.lib().ecg_batch_stream(h2))
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream2)
        api.check(api.lib().ecg_batch_step(h2, args.steps, None, None, C.byref(st2)), "step")
        s1.record(stream2)
        s1.synchronize()
        ms2 = s0.elapsed_time(s1)
        api.lib().ecg_batch_destroy(h2)
        seeded = {"value": total * args.steps / (ms2 * 1e-3), "unit": "cell-updates/s",
                  "speedup_vs_plain": dt_s * 1e3 / ms2,
                  "newton_evals_per_relaxation": st2.newton_evals / max(1, st2.relax_calls),
                  "plain_newton_evals_per_relaxation": st.newton_evals / max(1, st.relax_calls),
                  "seeded": st2.seeded, "seed_rejected": st2.seed_rejected, "model": os.path.relpath(model_path, ROOT)}
    # ---- end to end through the C ABI with host buffers: upload from pinned host memory, one
    #      ecg_batch_step call per step (per-case dt and t read back), download to pinned memory
    nf = len(cat)
    pin_in = [torch.from_numpy(np.ascontiguousarray(f)).pin_memory() for f in cat]
    pin_out = [torch.empty(total, dtype=torch.float64).pin_memory() for _ in range(nf)]
    in_np, out_np = [p.numpy() for p in pin_in], [p.numpy() for p in pin_out]
    dts = torch.empty(len(recs), dtype=torch.float64).pin_memory().numpy()
    ts = torch.empty(len(recs), dtype=torch.float64).pin_memory().numpy()
    h3 = C.c_void_p()
    api.check(api.lib().ecg_batch_create(arr, len(recs), C.byref(h3)), "ecg_batch_create")
    api.check(api.lib().ecg_batch_set_shape(h3, tile, th), "set_shape")
    st3 = api.StepStats()
    api.check(api.lib().ecg_batch_upload_prim(h3, api._field_ptrs(in_np), total), "upload")
    api.check(api.lib().ecg_batch_step(h3, args.warmup, None, None, C.byref(st3)), "warmup")
    torch.cuda.synchronize()
    dp = C.POINTER(C.c_double)
    t0 = time.perf_counter()
    api.check(api.lib().ecg_batch_upload_prim(h3, api._field_ptrs(in_np), total), "upload")
    for _ in range(args.steps):
        api.check(api.lib().ecg_batch_step(h3, 1, dts.ctypes.data_as(dp), ts.ctypes.data_as(dp), C.byref(st3)), "step")
    api.check(api.lib().ecg_batch_download_prim(h3, api._field_ptrs(out_np), total), "download")
    e2e_s = max_over_ranks(time.perf_counter() - t0, "cuda")
    api.lib().ecg_batch_destroy(h3)
    e2e = {"value": total * args.steps * world / e2e_s, "unit": "cell-updates/s",
           "h2d_bytes_per_step": 8.0 * total * nf / args.steps,
           "d2h_bytes_per_step": 8.0 * total * nf / args.steps + 16.0 * len(recs),
           "note": "state uploaded from pinned host memory once and downloaded once per timed run; one "
                   "ecg_batch_step call per step reading back every case's dt and t"}
    if rank == 0:
        peak, kind = measured_peak()
        B = 16 * (2 * 2 + 2 + 1)
        line = {"metric": METRIC, "value": value * world, "unit": "cell-updates/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt_s * 1e3 / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic",
                "config": {"workload": f"batched 1D shock tubes, Kapila 2-phase, MUSCL + van Leer, {len(recs)} cases",
                           "cells": total, "tile": tile.value, "cells_per_item": tile.value - 1,
                           "parallelism": f"replicas{world}"},
                "roofline": {"bound": "hbm", "achieved": B * value / 1e9, "peak": peak, "unit": "GB/s",
                             "frac": B * value / 1e9 / peak, "traffic": None, "peak_kind": kind,
                             "kernel": "k_batch (predictor + corrector of one step)",
                             "ncu_bytes_per_cell_update": NCU_BATCH_BYTES_PER_CELL_UPDATE},
                "e2e": e2e, "gpu_launches": args.steps * 3, "clocks": clk.summary(),
                "newton": {"relax_calls": st.relax_calls, "evals": st.newton_evals, "max": st.newton_max}}
        if seeded is not None:
            line["mlp_seeded"] = seeded
        print(json.dumps(line))


# ------------------------------------------------------------------------------------------- main


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c3", choices=["c1", "c2", "c3", "c4", "c5", "p2", "e2"])
    ap.add_argument("--no-seeded", action="store_true", help="skip the learned-seed measurement")
    ap.add_argument("--size", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--form", default="default", choices=["default", "split", "fused"],
                    help="form of the 2D / 3D Kapila passes (ecg_set_step_form); default: the library's")
    ap.add_argument("--staging", default="default", choices=["default", "tma", "plain"],
                    help="face-kernel tile staging of the split form (default: TMA where the mesh allows)")
    args = ap.parse_args()
    rank, world, local = env_rank()
    case = make_case(args.config, args.size)
    workload = {"c4": "1D water/air shock tube, Kapila, MUSCL + van Leer (one case of the batched workload)",
                "c1": "1D water/air shock tube, Kapila, first order",
                "c2": "2D shock-bubble, Kapila 2-phase, MUSCL + van Leer",
                "c3": "3D three-phase cavity collapse, Kapila, MUSCL + minmod",
                "c5": "2D liquid/vapour expansion, Kapila + p-T-mu relaxation, MUSCL + van Leer",
                "p2": "2D air bubble in water, PTUEq (temperature-pressure-velocity equilibrium), MUSCL + van Leer",
                "e2": "2D blast in air, Euler (single phase), MUSCL + van Leer"}[
        args.config]
    config = {"workload": f"{workload}, {'x'.join(str(n) for n in case.cells if n > 1)} cells, FP64",
              "cells": case.ncells, "phases": case.nphases, "dim": case.dim, "order": 2 if case.second_order else 1,
              "l2": l2_note(case), "parallelism": f"replicas{args.gpus}"}

    if args.impl == "reference":
        if rank != 0:
            return
        r = reference_sample(args.steps, args.warmup, config=args.config)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference binary oracle/_ref/ECOGEN not built"}))
            return
        line = {"metric": METRIC, "value": r["value"], "unit": "cell-updates/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference", "config": config,
                "cpu_baseline": {"value": r["value"], "unit": "cell-updates/s", "cores": r["cores"],
                                 "kind": "reference", "cpu": r["cpu"], "sample": r["sample"]},
                "e2e": {"value": r["value"], "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    if args.config == "c4":
        bench_batch(args, rank, world, local)
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    from ecogen_b200 import api

    work = tempfile.mkdtemp(prefix=f"ecg_bench_{rank}_")
    d = case.write(work)
    inp = api.Input(d, os.path.join(work, "libEOS"))
    fields0 = inp.fill()

    def new_context():
        c = api.Context(inp.case)
        if args.form != "default":
            c.set_step_form(api.FORM_SPLIT if args.form == "split" else api.FORM_FUSED)
        if args.staging != "default":
            c.set_face_staging(api.STAGING_TMA if args.staging == "tma" else api.STAGING_PLAIN)
        return c

    ctx = new_context()
    ctx.upload(fields0)
    ctx.step(args.warmup)
    stream = torch.cuda.ExternalStream(api.lib().ecg_stream(ctx.h))

    # ---- device-timed region: K steps replayed from captured graphs, events on the context stream
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        st = ctx.step(args.steps)
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, "cuda")
    value = case.ncells * args.steps * world / (ms_max * 1e-3)

    # ---- learned seed: same workload, relaxation Newton started from the installed MLP
    seeded = None
    model_path = seed_model_path(args.config, case.nphases)
    if not args.no_seeded and os.path.exists(model_path) and not case.ptueq:  # PTUEq has no relaxation to seed
        from ecogen_b200 import seed as seedmod
        model = seedmod.SeedModel.load(model_path)
        ref_ctx = new_context()
        ref_ctx.upload(fields0)
        ctx3 = new_context()
        ctx3.upload(fields0)
        model.install(ctx3)
        ref_ctx.step(args.warmup)
        ctx3.step(args.warmup)
        stream3 = torch.cuda.ExternalStream(api.lib().ecg_stream(ctx3.h))
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream3)
        st3 = ctx3.step(args.steps)
        s1.record(stream3)
        s1.synchronize()
        ms3 = s0.elapsed_time(s1)
        st_ref = ref_ctx.step(args.steps)
        a, b = ref_ctx.download_dict(), ctx3.download_dict()
        diff = max(float(np.abs(a[k] - b[k]).sum() / max(np.abs(a[k]).sum(), 1e-300)) for k in ("alpha", "rho", "p", "E"))
        seeded = {"value": case.ncells * args.steps / (ms3 * 1e-3), "unit": "cell-updates/s",
                  "speedup_vs_plain": ms_max / ms3,
                  "newton_evals_per_relaxation": st3.newton_evals / max(1, st3.relax_calls),
                  "plain_newton_evals_per_relaxation": st_ref.newton_evals / max(1, st_ref.relax_calls),
                  "seeded": st3.seeded, "seed_rejected": st3.seed_rejected, "fallback": st3.newton_fallback,
                  "nonfinite_cells": st3.nonfinite_cells,
                  "field_rel_l1_vs_plain": diff, "model": os.path.relpath(model_path, ROOT)}
        if case.ptmu is not None:  # the p-T-mu saturation solve: iterations with and without the seed
            seeded.update({"ptmu_seed_mode": "T", "ptmu_seeded": st3.ptmu_seeded,
                           "ptmu_seed_rejected": st3.ptmu_seed_rejected,
                           "ptmu_outer_iters_per_solve": st3.ptmu_outer_iters / max(1, st3.ptmu_solves),
                           "plain_ptmu_outer_iters_per_solve": st_ref.ptmu_outer_iters / max(1, st_ref.ptmu_solves),
                           "tsat_iters_per_solve": st3.ptmu_tsat_iters / max(1, st3.ptmu_solves),
                           "plain_tsat_iters_per_solve": st_ref.ptmu_tsat_iters / max(1, st_ref.ptmu_solves)})
            # the alternative: the network's p* starts the saturation Newton as well
            ctx4 = new_context()
            ctx4.upload(fields0)
            model.install(ctx4)
            ctx4.set_ptmu_seed(api.PTMU_SEED_P_T)
            ctx4.step(args.warmup)
            stream4 = torch.cuda.ExternalStream(api.lib().ecg_stream(ctx4.h))
            torch.cuda.synchronize()
            q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            q0.record(stream4)
            st4 = ctx4.step(args.steps)
            q1.record(stream4)
            q1.synchronize()
            ms4 = q0.elapsed_time(q1)
            d4 = ctx4.download_dict()
            seeded["p_and_T"] = {
                "value": case.ncells * args.steps / (ms4 * 1e-3), "speedup_vs_plain": ms_max / ms4,
                "ptmu_outer_iters_per_solve": st4.ptmu_outer_iters / max(1, st4.ptmu_solves),
                "tsat_iters_per_solve": st4.ptmu_tsat_iters / max(1, st4.ptmu_solves),
                "ptmu_seed_rejected": st4.ptmu_seed_rejected,
                "field_rel_l1_vs_plain": max(float(np.abs(a[k] - d4[k]).sum() / max(np.abs(a[k]).sum(), 1e-300))
                                             for k in ("alpha", "rho", "p", "E"))}
            ctx4.close()
        ref_ctx.close()
        ctx3.close()
        if case.ptmu is None:
            # ceiling of any pressure-relaxation seed: the plain workload with Newton stopped after one
            # (three) evaluations and the last iterate kept (no fallback), i.e. the step time of a seed
            # that always lands on p* (within three iterations); the seeded speed-up is judged against it
            ceil = {}
            for cap in (1, 3):
                cctx = new_context()
                cctx.upload(fields0)
                cctx.set_newton_cap(cap)
                cctx.set_newton_cap_mode(api.CAP_ACCEPT)
                cctx.step(args.warmup)
                cstream = torch.cuda.ExternalStream(api.lib().ecg_stream(cctx.h))
                torch.cuda.synchronize()
                c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                c0.record(cstream)
                stc = cctx.step(args.steps)
                c1.record(cstream)
                c1.synchronize()
                cms = c0.elapsed_time(c1)
                ceil[f"newton_cap_{cap}"] = {"ms_per_step": cms / args.steps, "speedup_vs_plain": ms_max / cms,
                                             "newton_evals_per_relaxation": stc.newton_evals / max(1, stc.relax_calls),
                                             "relaxations_at_cap": int(sum(list(stc.newton_hist)[cap - 1:]))}
                cctx.close()
            seeded["ceiling"] = ceil

    # ---- p-T-mu warm start (no network): each cell's T_sat solves start from its previous solve
    warm = None
    if case.ptmu is not None and not args.no_seeded:
        ref_w = new_context()
        ref_w.upload(fields0)
        ctxw = new_context()
        ctxw.upload(fields0)
        ctxw.set_ptmu_warm_start(True)
        ref_w.step(args.warmup)
        ctxw.step(args.warmup)
        streamw = torch.cuda.ExternalStream(api.lib().ecg_stream(ctxw.h))
        torch.cuda.synchronize()
        w0, w1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0.record(streamw)
        stw = ctxw.step(args.steps)
        w1.record(streamw)
        w1.synchronize()
        msw = w0.elapsed_time(w1)
        st_rw = ref_w.step(args.steps)
        a, b = ref_w.download_dict(), ctxw.download_dict()
        warm = {"value": case.ncells * args.steps / (msw * 1e-3), "unit": "cell-updates/s",
                "speedup_vs_plain": ms_max / msw,
                "tsat_iters_per_solve": stw.ptmu_tsat_iters / max(1, stw.ptmu_solves),
                "plain_tsat_iters_per_solve": st_rw.ptmu_tsat_iters / max(1, st_rw.ptmu_solves),
                "ptmu_outer_iters_per_solve": stw.ptmu_outer_iters / max(1, stw.ptmu_solves),
                "plain_ptmu_outer_iters_per_solve": st_rw.ptmu_outer_iters / max(1, st_rw.ptmu_solves),
                "nonfinite_cells": stw.nonfinite_cells,
                "field_rel_l1_vs_plain": max(float(np.abs(a[k] - b[k]).sum() / max(np.abs(a[k]).sum(), 1e-300))
                                             for k in ("alpha", "rho", "p", "E"))}
        ref_w.close()
        ctxw.close()

    # ---- per-kernel attribution (separate launches, events between kernels)
    nprof = max(2, min(args.steps, 10))
    st_p, kms = ctx.step_profiled_kernels(nprof)
    step_ms = sum(kms) / nprof
    kernel_ms = {name: v / nprof for name, v in zip(KERNEL_SLOTS, kms) if v > 0.0}
    form = "split" if ctx.step_form == api.FORM_SPLIT else "fused"
    config["form"] = form
    if form == "split":
        config["face_staging"] = "tma" if ctx.face_staging == api.STAGING_TMA else "plain"

    # ---- end to end through the C ABI with host buffers: upload from pinned host memory, one
    #      ecg_step call per step (host -> device dt/t, device -> host dt/t/counters), download
    nf = len(fields0)
    pinned_in = [torch.from_numpy(f).pin_memory() for f in fields0]
    pinned_out = [torch.empty(case.ncells, dtype=torch.float64).pin_memory() for _ in range(nf)]
    in_np = [p.numpy() for p in pinned_in]
    out_np = [p.numpy() for p in pinned_out]
    ctx2 = new_context()
    ctx2.upload(in_np)
    ctx2.step(args.warmup)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    ptrs_in = api._field_ptrs(in_np)
    api.check(api.lib().ecg_upload_prim(ctx2.h, ptrs_in, case.ncells), "upload")
    for _ in range(args.steps):
        ctx2.step(1)
    ptrs_out = api._field_ptrs(out_np)
    api.check(api.lib().ecg_download_prim(ctx2.h, ptrs_out, case.ncells), "download")
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], device="cuda")
    if world > 1:
        torch.distributed.all_reduce(te, op=torch.distributed.ReduceOp.MAX)
    e2e_value = case.ncells * args.steps * world / float(te.item())
    state_bytes = 8 * case.ncells * nf
    scal_bytes = 64
    stat_bytes = 8 * 24
    ctx2.close()

    if rank == 0:
        peak, peak_kind = measured_peak()
        B = bytes_per_cell_update(case)
        top = max((k for k in kernel_ms if k != "update"), key=lambda k: kernel_ms[k])
        top_ms = kernel_ms[top]
        top_bytes = kernel_bytes_per_cell(case, form, top)
        units = kernel_units(case, form, top)
        achieved = top_bytes * units / (top_ms * 1e-3) / 1e9
        model_key = "euler" if case.model.upper() == "EULER" else ("ptueq" if case.ptueq else "kapila")
        if model_key == "kapila" and case.ptmu is not None:
            model_key = "kapila_ptmu"
        tkey = (model_key, case.nphases, case.dim, bool(case.second_order), form, top)
        traffic = NCU_TRAFFIC_PER_CELL.get(tkey)
        kname = kernel_label(case, form, top)
        # FP64 roofline of the same kernel: its FP64 thread instructions (ncu count per cell) over the
        # FP64 pipe rate measured now by the DFMA probe
        fp64 = None
        pk64 = fp64_pipe_peak(local)
        if pk64 is not None:
            per_cell = NCU_FP64_PER_CELL.get(tkey)
            ach64 = per_cell * units / (top_ms * 1e-3) if per_cell else None
            fp64 = {"bound": "fp64", "unit": "FP64 thread-instructions/s (one DFMA = 2 flops)",
                    "peak": pk64["dfma_per_s"], "peak_kind": "measured (DFMA probe, this run)",
                    "peak_how": pk64["how"], "peak_clocks": pk64["clocks"],
                    "instructions_per_unit": per_cell, "achieved": ach64,
                    "frac": ach64 / pk64["dfma_per_s"] if ach64 else None}
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = reference_sample(steps=3, warmup=1, config=args.config, budget_s=60.0)
        line = {
            "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config,
            "e2e": {"value": e2e_value, "unit": "cell-updates/s",
                    "h2d_bytes_per_step": state_bytes / args.steps + scal_bytes,
                    "d2h_bytes_per_step": state_bytes / args.steps + scal_bytes + stat_bytes,
                    "note": "state uploaded from pinned host memory once and downloaded once per timed run; "
                            "one ecg_step call per step"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": traffic * units if traffic is not None else None, "units_per_launch": units,
                         "peak_kind": peak_kind, "kernel": kname, "form": form,
                         "algorithmic_bytes_per_unit": top_bytes, "unit_of_work": "face" if (form == "split" and "_faces_" in top) else "cell",
                         "launch_ms": top_ms,
                         "step_bytes_per_cell_update": B,
                         "step_frac": B * case.ncells / (step_ms * 1e-3) / 1e9 / peak,
                         "fp64": fp64},
            "kernels_ms": kernel_ms,
            "gpu_launches": args.steps * launches_per_step(case, form),
            "clocks": clk.summary(),
            "newton": {"relax_calls": st.relax_calls, "evals": st.newton_evals, "max": st.newton_max,
                       "fallback": st.newton_fallback, "hist": list(st.newton_hist)},
            "ptmu": ({"solves": st.ptmu_solves, "outer_iters": st.ptmu_outer_iters, "outer_max": st.ptmu_outer_max,
                      "outer_hist": list(st.ptmu_outer_hist), "tsat_calls": st.ptmu_tsat_calls,
                      "tsat_iters": st.ptmu_tsat_iters, "tsat_max": st.ptmu_tsat_max}
                     if case.ptmu is not None else None),
        }
        if seeded is not None:
            line["mlp_seeded"] = seeded
        if warm is not None:
            line["ptmu_warm_start"] = warm
        if cpu is not None:
            line["cpu_baseline"] = {"value": cpu["value"], "unit": "cell-updates/s", "cores": cpu["cores"],
                                    "kind": "reference", "cpu": cpu["cpu"], "sample": cpu["sample"]}
        print(json.dumps(line))
    ctx.close()
    shutil.rmtree(work, ignore_errors=True)
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
