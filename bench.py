"""Benchmark of the B200 FDTD stepper (one JSON line on rank 0).

Workload (default): the 512^3 single solve with CPML and gain -- 512^3 core cells at
20 nm + 12-cell CPML (536^3 = 154 M total cells), an n = 3.4 slab with a two-level gain
layer, dipole source, Ez probe with a 21-frequency DFT
(3d_fdtd_version008_b200/configs/b512_gain_slab.params).

A bench "step" is one fdtd_run() call that advances the solve by S = --fdtd-steps time
steps (default 10).  The headline is the FP64 mode, the reference's own arithmetic: `value` =
total cell-updates / device time of K bench steps, in Mcell-updates/s, measured with CUDA
events on the library's stream(s) bracketed by barriers and synchronisation, max over ranks.
FP32, BF16 and FP16 storage are measured in the same run (--forms) as blocks of the line, each
with its roofline (per-kernel events of a whole solve) and its accuracy against the FP64 solve
after the same W + K runs from the same state.  The field state (3.7-7.4 GB) is far larger
than L2 (126 MB), so no L2 flush is needed.

Multi-GPU (--gpus N under torchrun): replicas -- every rank runs an independent solve of
the same workload, value = all ranks' cell-updates / max over ranks of the device time.  With
--shard-gpus one process splits one solve along z over the N GPUs instead (strong scaling).

e2e: the same metric through the public C ABI from host buffers: fdtd_create from the host
setup (H2D of the material index and 1-D profiles, layout transpose on the device), K runs of
S steps each followed by a D2H read of that run's probe samples, a D2H read of the final Ez
field, fdtd_destroy -- all inside the timed region (wall clock, synchronised).  It is taken
first in the process, after a warm-up solve of the sample grid (CUDA context, kernel modules).

--impl reference: times the reference's own CPU loop (the reference headers compiled with its
CMake flags, OpenMP on all host cores) on the same 536^3 grid, W untimed and K timed steps;
it falls back to the bounded 216^3 sample when the host lacks the memory for the reference's
full-grid arrays, and to the oracle's C restatement when the reference binary is absent.

--serving, --sweep, --sweep-check and --precision-study print lines of their own.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
PKG = importlib.import_module("3d_fdtd_version008_b200")

WORKLOADS = {
    "b512": ("b512_gain_slab.params", "b512_gain_slab_cpu_sample.params",
             "512^3 core (536^3 total) uniform 20 nm, 12-cell CPML, n=3.4 slab with 200 nm two-level gain layer "
             "(pump 1e9/s), z dipole, Ez probe + 21-freq DFT"),
    "b256": ("b256_gain_slab.params", "b512_gain_slab_cpu_sample.params",
             "256^3 core (280^3 total) uniform 20 nm, 12-cell CPML, n=3.4 slab with 200 nm two-level gain layer "
             "(pump 1e9/s), z dipole, Ez probe + 21-freq DFT"),
    "c2": ("c2_spheres_512.params", "b512_gain_slab_cpu_sample.params",
           "512^3 core (536^3 total) uniform 20 nm, 12-cell CPML, 4000 seeded dielectric spheres (r 3-12 cells, "
           "eps_r 2-12), z dipole, Ez probe + 21-freq DFT"),
    "c1": ("c1_gain_slab.params", "c1_gain_slab.params",
           "C1 non-uniform mesh + gain slab (201x201x69 total)"),
    "c0": ("c0_dipole_sphere.params", "c0_dipole_sphere.params",
           "C0 64^3 + 8-cell CPML (80^3 total), dielectric sphere, dipole"),
}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_bytes(setup, word: int, coef_word: int = 0, material_bytes: int = 0):
    """Compulsory bytes per step of the two-sweep algorithm: fields and psi stored in `word`
    bytes, bE and gain state in `coef_word` bytes (default: the same).

    H sweep: read E(3) H(3), write H(3) = 9 field words/cell; E sweep: read H(3) E(3), write
    E(3) = 9 field words + the material (bE: 3 coefficient words per cell, or `material_bytes`
    per cell when the stepper holds it as a row index -- the small row table stays on chip);
    + 2 field words per active CPML psi (4 per axis, 2 per sweep) in that axis' slab; + gain
    cells: read P^n, P^{n-1}, Nu, Ng and write P^{n+1}, Nu, Ng = 7 coefficient words."""
    cw = coef_word or word
    mat = material_bytes or 3 * cw
    NxT, NyT, NzT = setup.shape
    npml = int(setup.view.npml)
    cells = NxT * NyT * NzT
    slab = sum(2 * npml * (cells // n) for n in (NxT, NyT, NzT))  # cells inside each axis' slab, summed
    gain = int((setup.array("tls_region_map") >= 0).sum()) if setup.view.n_tls_regions else 0
    h = 9 * word * cells + 2 * 2 * word * slab
    e = 9 * word * cells + mat * cells + 2 * 2 * word * slab + 7 * cw * gain
    return {"cells": cells, "h_bytes": h, "e_bytes": e, "step_bytes": h + e,
            "per_cell": (h + e) / cells, "slab_cells": slab, "gain_cells": gain}


def dist_setup(n_gpus: int):
    """Replica ranks under torchrun: one process per GPU (NCCL; gloo where no GPU is visible,
    which is how the multi-rank logic is tested on CPU).  The ranks exchange nothing on the
    data path: only the timing barrier and the max-over-ranks reduction."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=600))
        return rank, local, world, dist
    return rank, local, 1, None


def reduce_max(dist, value: float) -> float:
    if dist is None:
        return value
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(cells: int, steps_total: int, world: int, device_ms_max: float) -> float:
    """Whole-job Mcell-updates/s: every rank advanced its own replica by steps_total steps;
    the job took the slowest rank's device time."""
    return cells * steps_total * world / (device_ms_max * 1e-3) / 1e6


def barrier(dist):
    if dist is not None:
        dist.barrier()


def cpu_reference(sample_cfg: str, steps: int, warmup: int, fdtd_steps: int):
    """Times the reference CPU loop on the bounded sample; returns (Mcell/s, info)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    cores = os.cpu_count() or 1
    n = warmup + steps
    path = PKG.config_path(sample_cfg)
    if oracle.REF_HARNESS_NATIVE.exists():
        r = oracle.run_harness(path, n * fdtd_steps, "--no-fields", native=True, env={"OMP_NUM_THREADS": str(cores)})
        shape = [r["meta"][k] for k in ("NxT", "NyT", "NzT")]
        loop_s = float(r["meta"]["loop_seconds"])
        cells = shape[0] * shape[1] * shape[2]
        exe_p = oracle.native_harness()
        march = "x86-64-v4" if exe_p == oracle.REF_HARNESS_NATIVE_V4 else "x86-64-v3"
        kind, exe = "reference", f"{exe_p.relative_to(ROOT)} (reference headers, -O3 -march={march} -fopenmp)"
    else:
        s = PKG.Setup.from_file(path)
        o = oracle.OracleSolve(s, 0)
        t0 = time.time()
        o.run(n * fdtd_steps, threads=cores)
        loop_s = time.time() - t0
        shape = list(s.shape)
        cells = s.shape[0] * s.shape[1] * s.shape[2]
        kind, exe = "port", "oracle/lib/libfdtd_oracle.so (C restatement, OpenMP)"
    value = cells * n * fdtd_steps / loop_s / 1e6
    sample = (f"{sample_cfg}: {shape[0]}x{shape[1]}x{shape[2]} total cells, {n * fdtd_steps} steps of the "
              f"reference loop (H, CPML-H, E with gain, CPML-E, probe, populations), {exe}, "
              f"{cores} threads, loop wall time {loop_s:.2f} s")
    return value, {"value": round(value, 3), "unit": "Mcell-updates/s", "cores": cores, "kind": kind,
                   "sample": sample}


# ------------------------------------------------------------------ serving (packed engine)
def serving_job_text(core: tuple, steps_hint: int) -> str:
    """A slab microcavity with a two-level gain layer (the 512^3 workload's recipe scaled to
    a core of nx x ny x nz cells at 20 nm, 8-cell CPML), z dipole, Ez probe + DFT."""
    nx, ny, nz = core
    d = 20e-9
    L = [n * d for n in core]
    cx, cy, cz = (0.5 * l for l in L)
    return "\n".join([
        "MESH_MODE = 0", f"NX = {nx}", f"NY = {ny}", f"NZ = {nz}",
        f"DX_UNIFORM = {d}", f"DY_UNIFORM = {d}", f"DZ_UNIFORM = {d}",
        "DOMAIN_X_MIN = 0", f"DOMAIN_X_MAX = {L[0]}", "DOMAIN_Y_MIN = 0", f"DOMAIN_Y_MAX = {L[1]}",
        "DOMAIN_Z_MIN = 0", f"DOMAIN_Z_MAX = {L[2]}",
        "LAMBDA0 = 1550.1264633919338e-9", "CFL_FACTOR = 0.99", f"N_STEPS = {steps_hint}", "SAVE_EVERY = 1",
        "CPML_NPML = 8", "CPML_M = 3.0", "CPML_RERR = 1e-6", "CPML_ALPHA0 = 0.05", "CPML_KAPPA_MAX = 5.0",
        "CPML_ALPHA_LINEAR = true", "BACKGROUND_N = 1.0", "TLS_ENABLED = true", "MESH_OVERRIDE_ENABLED = false",
        "TLS_MATERIALS += gain_1550, 1550.1264633919338e-9, 31415926535897.93, 1e-9, 5e23, 0.0",
        f'STRUCTURES += box, 3.4, {0.1 * L[0]}, {0.9 * L[0]}, {0.1 * L[1]}, {0.9 * L[1]}, {cz - 110e-9}, {cz + 110e-9}, ""',
        f"STRUCTURES += box, 3.4, {0.1 * L[0]}, {0.9 * L[0]}, {0.1 * L[1]}, {0.9 * L[1]}, {cz - 100e-9}, {cz + 100e-9}, gain_1550",
        f"DIPOLE_SOURCES += true, {cx + 10e-9}, {cy + 10e-9}, {cz - 10e-9}, 1e-7, 193.4e12, 0, 0, 50e12, 3.0, 1, 2",
        f"POINT_FIELD_DETECTORS += true, Ez_probe, {cx + 0.1 * L[0]}, {cy + 10e-9}, {cz - 10e-9}, 2",
        "DFT_FREQS = 168e12, 218e12, 21", "PUMP_RATE = 1e9", "PRECISION = fp32", ""])


def serving_bench(args):
    """The serving configuration's stream, bounded to --serving-jobs solves: gain-slab
    microcavities with core edges log-uniform in 32..192 cells (aspect 1..2), steps uniform in
    2000..20000, 8-cell CPML, FP32, admitted by footprint under a 150 GB budget (seed 3).
    Throughput: all jobs queued at once, served by the packed engine, and one at a time by
    fdtd_create/fdtd_run.  Latency: the same jobs arriving as a Poisson stream at 80 % of the
    packed engine's measured throughput (the admission thread prepares arrivals while the
    resident solves step); the one-at-a-time server's latencies are its FIFO queue over its own
    measured service times."""
    import numpy as np
    rng = np.random.default_rng(3)
    lo, hi = args.serving_edges
    s_lo, s_hi = args.serving_steps
    jobs = []
    for _ in range(args.serving_jobs):
        edge = float(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        asp = rng.uniform(1.0, 2.0, size=2)
        core = (int(edge), int(max(16, edge / asp[0])), int(max(16, edge / asp[1])))
        steps = int(rng.integers(s_lo, s_hi + 1))
        jobs.append((core, steps))
    setups = [PKG.Setup.from_text(serving_job_text(c, n)) for c, n in jobs]
    cells = [s.shape[0] * s.shape[1] * s.shape[2] for s in setups]
    work = sum(c * n for c, (_, n) in zip(cells, jobs))
    # warm-up outside the timed phases: CUDA context, module load, both code paths
    w = PKG.Solver(setups[0], precision=PKG.PREC_FP32)
    w.run(20)
    w.close()
    wb = PKG.Batch(budget_bytes=150 << 30)
    wt = wb.submit(setups[0], 20)
    while wb.state(wt)[0] < PKG.JOB_DONE:
        wb.run(20)
    wb.close()
    # one at a time
    service = []
    for s, (_, n) in zip(setups, jobs):
        t0 = time.perf_counter()
        sol = PKG.Solver(s, precision=PKG.PREC_FP32)
        sol.run(n)
        sol.probe_series()
        sol.close()
        service.append(time.perf_counter() - t0)
    plain_s = sum(service)
    # packed, all queued at t = 0
    b = PKG.Batch(budget_bytes=150 << 30)
    t0 = time.perf_counter()
    tickets = [b.submit(s, n) for s, (_, n) in zip(setups, jobs)]
    pending = set(tickets)
    occ = []  # (seconds since start, resident jobs) after every run call
    while pending:
        r, _ = b.run(32)
        occ.append((time.perf_counter() - t0, r))
        for t in list(pending):
            if b.state(t)[0] >= PKG.JOB_DONE:
                b.probe_series(t)
                b.release(t)
                pending.discard(t)
    packed_s = time.perf_counter() - t0
    # time spent with r resident jobs, in bands
    bands = {"1": 0.0, "2-4": 0.0, "5-16": 0.0, "17-64": 0.0}
    prev = 0.0
    for ts, r in occ:
        key = "1" if r <= 1 else "2-4" if r <= 4 else "5-16" if r <= 16 else "17-64"
        bands[key] += ts - prev
        prev = ts
    # Poisson arrivals at 80 % of the packed throughput
    rate = 0.8 * len(jobs) / packed_s
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(jobs)))
    lat_packed = [0.0] * len(jobs)
    t0 = time.perf_counter()
    submitted, pending, tick = 0, {}, {}
    while submitted < len(jobs) or pending:
        now = time.perf_counter() - t0
        while submitted < len(jobs) and arrivals[submitted] <= now:
            pending[b.submit(setups[submitted], jobs[submitted][1])] = submitted
            submitted += 1
        if pending:
            b.run(16)
        else:
            time.sleep(max(0.0, min(arrivals[submitted] - now, 0.01)))
        now = time.perf_counter() - t0
        for t, k in list(pending.items()):
            if b.state(t)[0] >= PKG.JOB_DONE:
                b.release(t)
                lat_packed[k] = now - arrivals[k]
                del pending[t]
    b.close()
    lat_plain, free_at = [], 0.0
    for k in range(len(jobs)):
        start = max(arrivals[k], free_at)
        free_at = start + service[k]
        lat_plain.append(free_at - arrivals[k])
    pct = lambda v, q: round(float(np.percentile(v, q)) * 1e3, 2)
    line = {
        "metric": "solves/s (packed multi-solve engine)", "value": round(len(jobs) / packed_s, 3), "unit": "solves/s",
        "n_gpus": 1, "steps": len(jobs), "warmup": 0, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"serving: stream of gain-slab microcavities, core edge {lo}-{hi} cells log-uniform "
                               f"(aspect 1-2), {s_lo}-{s_hi} steps, 8-cell CPML, FP32, Poisson arrivals at 80 % load",
                   "jobs": len(jobs), "jobs_note": "the first jobs of the seed-3 stream (the full stream is 4000)",
                   "cell_updates": int(work), "budget_GB": 150},
        "packed": {"seconds": round(packed_s, 3), "Mcell_updates_per_s": round(work / packed_s / 1e6, 1),
                   "p50_ms": pct(lat_packed, 50), "p95_ms": pct(lat_packed, 95), "p99_ms": pct(lat_packed, 99)},
        "one_at_a_time": {"seconds": round(plain_s, 3), "Mcell_updates_per_s": round(work / plain_s / 1e6, 1),
                          "p50_ms": pct(lat_plain, 50), "p95_ms": pct(lat_plain, 95), "p99_ms": pct(lat_plain, 99)},
        "throughput_ratio": round(plain_s / packed_s, 2),
        "packed_seconds_by_resident_jobs": {k: round(v, 3) for k, v in bands.items()},
        "arrival_rate_per_s": round(rate, 2),
    }
    print(json.dumps(line))


def c4_setups(pumps, steps: int):
    """The sweep's cavities (configs/c4_cavity.params: the C1 recipe on the auto mesher's graded
    mesh, 96 x 96 x 65 total cells), one per pump rate."""
    text = PKG.config_path("c4_cavity.params").read_text().replace("N_STEPS = 20000", f"N_STEPS = {int(steps)}")
    return [PKG.Setup.from_text(text.replace("PUMP_RATE = 1e9", f"PUMP_RATE = {float(p)!r}")) for p in pumps]


def sweep_bench(args):
    """The batched gain-laser sweep: 256 slab microcavities on the auto mesher's graded mesh
    (96 x 96 x 65 total cells, configs/c4_cavity.params), pump W_p log-uniform in 1e7..1e11
    1/s (seed 4), BF16 field storage with FP32 arithmetic, FP32 populations, FP64 DFT, through
    the packed engine, --sweep-steps steps each (200000 for the full sweep).  The same jobs in
    FP32 storage are timed beside them unless --sweep-forms says otherwise.  Two figures per
    storage form: the whole sweep (all jobs queued at once, admission included) and the packed
    step of 64 resident cavities alone; the BF16 sweep also reports each cavity's end state
    (population inversion, growth of the probe signal) against its pump."""
    import numpy as np
    rng = np.random.default_rng(4)
    pumps = np.exp(rng.uniform(np.log(1e7), np.log(1e11), size=args.sweep_jobs))
    n = args.sweep_steps
    setups = c4_setups(pumps, n)
    cells = setups[0].shape[0] * setups[0].shape[1] * setups[0].shape[2]
    out = {}
    ends = []
    forms = [(f, {"bf16": PKG.PREC_BF16, "fp32": PKG.PREC_FP32, "fp16": PKG.PREC_FP16}[f])
             for f in args.sweep_forms.split(",")]
    for name, prec in forms:
        views = []
        for s in setups:
            v = PKG.SetupV1.from_buffer_copy(s.view)
            v.precision = prec
            views.append(v)
        # warm-up: module load and one packed step of each kernel kind
        b = PKG.Batch(budget_bytes=150 << 30)
        t = b.submit(setups[0], 20, view=views[0])
        while b.state(t)[0] < PKG.JOB_DONE:
            b.run(20)
        b.release(t)
        # the packed step alone: 64 resident cavities
        ts = [b.submit(s, args.sweep_probe_steps + 100, view=v) for s, v in zip(setups[:64], views[:64])]
        b.run(3)
        t0 = time.perf_counter()
        b.run(args.sweep_probe_steps)
        step_s = (time.perf_counter() - t0) / args.sweep_probe_steps
        b.close()
        # the whole sweep, all jobs queued at t = 0
        b = PKG.Batch(budget_bytes=150 << 30)
        t0 = time.perf_counter()
        ts = [b.submit(s, n, view=v) for s, v in zip(setups, views)]
        pending, failed = set(ts), 0
        end = {}
        while pending:
            b.run(64)
            for t in list(pending):
                st = b.state(t)[0]
                if st >= PKG.JOB_DONE:
                    failed += st == PKG.JOB_FAILED
                    b.dft(t)
                    if name == forms[0][0]:
                        d = b.diagnostics(t)
                        ser = b.probe_series(t)[:, 0]
                        end[t] = (d, ser)
                    b.release(t)
                    pending.discard(t)
        wall = time.perf_counter() - t0
        b.close()
        if name == forms[0][0]:
            dt = setups[0].view.dt
            for q, t in enumerate(ts):
                d, ser = end[t]
                nu, ng = d["integrated_Nu"], d["integrated_Ng"]
                # growth of the probe signal over the last half of the run (RMS of the two
                # quarters), in 1/ps: > 0 would mean net gain
                m = len(ser) // 4
                r1 = float(np.sqrt(np.mean(ser[-2 * m:-m] ** 2))) if m else 0.0
                r2 = float(np.sqrt(np.mean(ser[-m:] ** 2))) if m else 0.0
                g = float(np.log(r2 / r1) / (m * dt) * 1e-12) if r1 > 0 and r2 > 0 else None
                ends.append({"pump_per_s": float(pumps[q]), "inversion": round((nu - ng) / (nu + ng), 6),
                             "late_growth_per_ps": round(g, 5) if g is not None else None})
        out[name] = {"sweep_seconds": round(wall, 3),
                     "sweep_Gcell_updates_per_s": round(len(setups) * cells * n / wall / 1e9, 2),
                     "packed_step_ms_64_cavities": round(step_s * 1e3, 4),
                     "packed_Gcell_updates_per_s": round(64 * cells / step_s / 1e9, 2),
                     "failed_jobs": int(failed),
                     "projected_hours_200000_steps": round(len(setups) / 64 * 200000 * step_s / 3600, 3)}
    line = {
        "metric": "Gcell-updates/s (batched BF16 sweep, packed engine)", "value": out[forms[0][0]]["sweep_Gcell_updates_per_s"],
        "unit": "Gcell-updates/s", "n_gpus": 1, "steps": n, "warmup": 1, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16 storage, f32 arithmetic", "data": "synthetic",
        "config": {"workload": f"sweep: {len(setups)} gain-slab microcavities on the auto mesher's graded mesh "
                               f"({'x'.join(map(str, setups[0].shape))} cells, configs/c4_cavity.params), pump "
                               "log-uniform 1e7-1e11 1/s, BF16 fields / FP32 populations / FP64 DFT", "jobs": len(setups),
                   "cells_per_job": cells, "steps_per_job": n, "budget_GB": 150},
        "cavity_end_state": ends,
        "lasing": lasing_summary(ends),
    }
    line.update(out)
    print(json.dumps(line))


def lasing_summary(ends):
    """Lasing threshold from the cavities' end states: the smallest pump whose cavity reached
    population inversion (Nu > Ng) and whose probe signal grew over the last half of the run;
    None when no cavity did, with the largest inversion reached."""
    lasing = [e for e in ends if e["inversion"] > 0 and (e["late_growth_per_ps"] or -1) > 0]
    top = max(ends, key=lambda e: e["inversion"]) if ends else None
    return {"threshold_pump_per_s": min(e["pump_per_s"] for e in lasing) if lasing else None,
            "max_inversion": top["inversion"] if top else None,
            "pump_at_max_inversion": top["pump_per_s"] if top else None,
            "note": "inversion = (int Nu - int Ng) / (int Nu + int Ng) over the gain layer at the end; it starts at -1 "
                    "(all in the ground state) and the pump W_p raises it by about 2 W_p t, so a window of t = "
                    "steps x dt bounds how far any cavity can get"}


def ringdown(series, dt, t_from, band=(100e12, 300e12)):
    """Emission peak frequency (Hz; zero-padded FFT of the probe series after t_from, inside
    `band` -- the source's 193.4 THz +- 25 THz lies well inside; 16-bit storage adds broadband
    rounding noise whose lines elsewhere must not be taken for the emission -- parabolic
    interpolation of the peak bin), amplitude growth rate g (1/s; slope of log RMS over windows
    of one period of the series band-passed around f, E ~ exp(g t): g < 0 decays) and
    Q = pi f / (-g).  A decaying signal is fitted only while it stands 10x above the noise floor
    (the median RMS of the last tenth of the windows) that it decays into."""
    import numpy as np
    x = np.asarray(series, dtype=np.float64)[int(t_from / dt):]
    tt = np.arange(len(x))
    x = x - np.polyval(np.polyfit(tt, x, 1), tt)  # a static or drifting part is not the emission
    nfft = 1 << (int(np.ceil(np.log2(len(x)))) + 3)
    spec = np.abs(np.fft.rfft(x * np.hanning(len(x)), nfft))
    k0 = int(np.ceil(band[0] * nfft * dt))
    k1 = min(len(spec), int(np.floor(band[1] * nfft * dt)) + 1)
    k = int(np.argmax(spec[k0:k1])) + k0
    if 1 <= k < len(spec) - 1:
        a, b, c = np.log(spec[k - 1:k + 2] + 1e-300)
        k = k + 0.5 * (a - c) / (a - 2 * b + c)
    f = k / (nfft * dt)
    # the band around the peak only (a Gaussian of 0.15 f around f): slow drifts and noise do not
    # set the rate.  A Gaussian's time response is about one period long; a brick-wall band
    # leaks the large start of the window into its decayed end through slowly falling sidelobes
    # and flattens a fast decay (5 % at Q 46)
    X = np.fft.rfft(x)
    fr = np.fft.rfftfreq(len(x), dt)
    X *= np.exp(-0.5 * ((fr - f) / (0.15 * f)) ** 2)
    x = np.fft.irfft(X, len(x))
    per = max(4, int(round(1.0 / (f * dt))))
    nw = len(x) // per
    rms = np.sqrt(np.mean(x[:nw * per].reshape(nw, per) ** 2, axis=1))
    t = (np.arange(nw) + 0.5) * per * dt
    cut = nw // 10  # the band-pass rings at both ends of the window
    lo, hi = cut, nw - cut
    if rms[lo] > rms[hi - 1]:  # decaying: stop where it reaches its noise floor
        floor = float(np.median(rms[nw - max(1, nw // 10):]))
        above = np.nonzero(rms[lo:hi] < 10.0 * floor)[0]
        if len(above) and above[0] >= 8:
            hi = lo + int(above[0])
    g = float(np.polyfit(t[lo:hi], np.log(rms[lo:hi] + 1e-300), 1)[0])
    return float(f), g, (float(np.pi * f / -g) if g < 0 else None)


def sweep_check(args):
    """The sweep's fidelity check: 8 of its cavities (indices 0, 32, ..., 224 of the 256, same
    pumps) in the packed engine, in each storage form of --check-forms, against FP64 single
    solves, --check-steps steps each: emission peak frequency, ring-down (growth) rate, Q, and
    the lasing threshold estimated from the growth rate's dependence on the pump (W_p where the
    fitted growth rate reaches 0).  Forms: fp32, fp16, bf16 (round to nearest) and bf16sr
    (BF16 with stochastic rounding of the E and H stores)."""
    import numpy as np
    rng = np.random.default_rng(4)
    pumps = np.exp(rng.uniform(np.log(1e7), np.log(1e11), size=256))
    idx = list(range(0, 256, 32))
    n = args.check_steps
    setups = c4_setups([pumps[q] for q in idx], n)
    dt = setups[0].view.dt
    t_from = 4000 * dt  # after the source pulse (t0 + 3 tau = 64 fs)
    t0 = time.perf_counter()
    ref = []
    for s in setups:
        sol = PKG.Solver(s, precision=PKG.PREC_FP64)
        sol.run(n)
        ref.append((sol.probe_series()[:, 0], sol.dft(0)))
        sol.close()
    seconds = {"fp64_one_at_a_time": round(time.perf_counter() - t0, 2)}
    ref_rd = [ringdown(r[0], dt, t_from) for r in ref]

    def threshold(g):
        w = np.array([float(pumps[q]) for q in idx])
        slope, icpt = np.polyfit(w, np.asarray(g), 1)
        th = -icpt / slope if slope > 0 else None
        return float(th) if th is not None and w.min() <= th <= w.max() else None

    forms = {}
    for form in args.check_forms.split(","):
        prec = {"fp32": PKG.PREC_FP32, "fp16": PKG.PREC_FP16, "bf16": PKG.PREC_BF16, "bf16sr": PKG.PREC_BF16}[form]
        b = PKG.Batch(budget_bytes=150 << 30)
        views = []
        for s in setups:
            v = PKG.SetupV1.from_buffer_copy(s.view)
            v.precision = prec
            v.rounding = 1 if form == "bf16sr" else 0
            views.append(v)
        t0 = time.perf_counter()
        ts = [b.submit(s, n, view=v) for s, v in zip(setups, views)]
        while any(b.state(t)[0] < PKG.JOB_DONE for t in ts):
            b.run(256)
        seconds[form + "_packed"] = round(time.perf_counter() - t0, 2)
        got = [(b.probe_series(t)[:, 0], b.dft(t), b.state(t)[0]) for t in ts]
        b.close()
        rd = [ringdown(g[0], dt, t_from) for g in got]
        forms[form] = {
            "all_done": all(g[2] == PKG.JOB_DONE for g in got),
            "max_peak_shift_THz": round(max(abs(a[0] - b_[0]) for a, b_ in zip(ref_rd, rd)) / 1e12, 5),
            "growth_per_ps": [round(x[1] * 1e-12, 4) for x in rd],
            "Q": [round(x[2], 1) if x[2] else None for x in rd],
            "max_Q_rel_err": (max(abs(x[2] - r[2]) / r[2] for x, r in zip(rd, ref_rd)) if all(x[2] for x in rd) else None),
            "max_dft_rel_err": max(float(np.linalg.norm(g[1] - r[1]) / np.linalg.norm(r[1])) for g, r in zip(got, ref)),
            "threshold_per_s": threshold([x[1] for x in rd]),
        }
    line = {
        "metric": "sweep fidelity: packed 16-bit storage vs FP64 on 8 cavities (max Q rel. error)", "unit": "rel. error",
        "value": forms[args.check_forms.split(",")[0]]["max_Q_rel_err"], "n_gpus": 1, "steps": n, "warmup": 0,
        "higher_is_better": False, "vs_baseline": None, "dtype": "storage forms vs f64", "data": "synthetic",
        "config": {"workload": "8 of the sweep's 256 gain-slab microcavities on the graded mesh, "
                               f"{'x'.join(map(str, setups[0].shape))} cells (indices 0, 32, ..., 224)",
                   "steps_per_job": n, "window_from_step": 4000, "pumps_per_s": [float(pumps[q]) for q in idx]},
        "fp64": {"peak_THz": [round(r[0] / 1e12, 4) for r in ref_rd], "growth_per_ps": [round(r[1] * 1e-12, 4) for r in ref_rd],
                 "Q": [round(r[2], 1) if r[2] else None for r in ref_rd],
                 "threshold_per_s": threshold([r[1] for r in ref_rd])},
        "forms": forms,
        "threshold_note": "null: the growth rate does not reach 0 inside the swept pump range (tau21 = 1 ns >> window)",
        "seconds": seconds,
    }
    print(json.dumps(line))


def precision_study(args):
    """The 512^3 sphere solve (or --workload's) for --study-steps steps as FP64, FP32, FP16 and
    BF16 storage: field L2 (E and H), probe series, DFT and DFT-peak errors against FP64."""
    import numpy as np
    cfg, _, desc = WORKLOADS[args.workload]
    setup = PKG.Setup.from_file(PKG.config_path(cfg))
    n = args.study_steps
    comps = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
    ref, res = {}, {}
    for name, prec in (("fp64", PKG.PREC_FP64), ("fp32", PKG.PREC_FP32), ("fp16", PKG.PREC_FP16),
                       ("bf16", PKG.PREC_BF16)):
        sol = PKG.Solver(setup, precision=prec)
        sol.set_timing(PKG.TIMING_RUN)
        sol.run(n)
        ms = sol.timing()["run_ms"]
        series, dft = sol.probe_series()[:, 0], sol.dft(0)
        if name == "fp64":
            ref = {"f": {c: sol.field(c) for c in comps}, "series": series, "dft": dft}
            res[name] = {"ms": round(ms, 1)}
        else:
            num = {"E": 0.0, "H": 0.0}
            den = {"E": 0.0, "H": 0.0}
            for c in comps:
                f = sol.field(c)
                num[c[0]] += float(np.sum((f - ref["f"][c]) ** 2))
                den[c[0]] += float(np.sum(ref["f"][c] ** 2))
                del f
            res[name] = {"ms": round(ms, 1),
                         "E_L2": float(np.sqrt(num["E"] / den["E"])), "H_L2": float(np.sqrt(num["H"] / den["H"])),
                         "probe": float(np.linalg.norm(series - ref["series"]) / np.linalg.norm(ref["series"])),
                         "dft": float(np.abs(dft - ref["dft"]).max() / np.abs(ref["dft"]).max()),
                         "dft_peak_same": bool(np.argmax(np.abs(dft)) == np.argmax(np.abs(ref["dft"])))}
        sol.close()
    cells = setup.shape[0] * setup.shape[1] * setup.shape[2]
    for v in res.values():
        v["Gcell_per_s"] = round(cells * n / (v["ms"] * 1e-3) / 1e9, 2)
    print(json.dumps({"metric": "precision study (errors against the FP64 solve)", "workload": desc,
                      "config_file": cfg, "steps": n, "results": res}))


PREC = {"fp32": PKG.PREC_FP32, "fp64": PKG.PREC_FP64, "fp16": PKG.PREC_FP16, "bf16": PKG.PREC_BF16}
WORD = {"fp32": 4, "fp64": 8, "fp16": 2, "bf16": 2}
DTYPE = {"fp32": "f32", "fp64": "f64", "fp16": "f32 (fp16 storage)", "bf16": "f32 (bf16 storage)"}


def shards_for(args, form: str) -> int:
    """z shards of the solve on the GPU for a storage form: --shards, else the fastest measured
    on the 536^3 workload (one B200, 20 x 10 steps): FP64 steps fastest whole (37.0 against 36.7
    with 2 shards and 36.5 with 4); FP32, BF16 and FP16 with 4 shards (72.6 / 101.8 / 104.6
    against 72.2 / 97.5 / 100.8 whole), whose sweeps' tails overlap on their streams."""
    if args.shards:
        return args.shards
    return 1 if form == "fp64" else 4


def workload_config(setup, cfg: str, desc: str) -> dict:
    """The workload, identical in both arms' lines (the reference arm runs the same grid)."""
    return {"workload": desc, "config_file": cfg, "grid": list(setup.shape),
            "total_cells": int(setup.shape[0] * setup.shape[1] * setup.shape[2])}


def cpu_model() -> str:
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def host_mem_gb() -> float:
    try:
        for ln in open("/proc/meminfo"):
            if ln.startswith("MemAvailable"):
                return int(ln.split()[1]) / 1e6
    except OSError:
        pass
    return 0.0


def reference_arm(args, cfg: str, sample_cfg: str, desc: str, K: int, W: int) -> dict:
    """--impl reference: the reference's own time loop (src/3D_FDTD_version008.cpp:269-328,
    compiled from its headers with its CMake flags, OpenMP on every host core) on the same
    workload grid as the GPU arm, W untimed then K timed steps; one bench step = one time step
    of the reference (the metric is per cell-update).  It needs the reference's ~41 full-grid
    FP64 arrays in host memory; with less memory than that it times the bounded sample grid
    and says so."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    setup = PKG.Setup.from_file(PKG.config_path(cfg), mesh_only=True)
    cells = setup.shape[0] * setup.shape[1] * setup.shape[2]
    need_gb = 41 * 8 * cells / 1e9 * 1.1
    cores = os.cpu_count() or 1
    use = cfg if host_mem_gb() >= need_gb else sample_cfg
    path = PKG.config_path(use)
    t0 = time.time()
    if oracle.REF_HARNESS_NATIVE.exists():
        exe = oracle.native_harness()
        r = oracle.run_harness(path, W + K, "--no-fields", "--warmup", str(W), native=True,
                               env={"OMP_NUM_THREADS": str(cores)})
        shape = [r["meta"][k] for k in ("NxT", "NyT", "NzT")]
        loop_s = float(r["meta"]["loop_seconds"])
        kind = "reference"
        march = "x86-64-v4" if exe == oracle.REF_HARNESS_NATIVE_V4 else "x86-64-v3"
        what = f"{exe.relative_to(ROOT)} (the reference headers compiled with -O3 -march={march} -fopenmp)"
    else:
        s = PKG.Setup.from_file(path)
        o = oracle.OracleSolve(s, 0)
        o.run(W, threads=cores)
        t1 = time.time()
        o.run(K, threads=cores)
        loop_s = time.time() - t1
        shape = list(s.shape)
        kind = "port"
        what = "oracle/lib/libfdtd_oracle.so (C restatement of the reference loop, OpenMP)"
    total = time.time() - t0
    ncell = shape[0] * shape[1] * shape[2]
    value = ncell * K / loop_s / 1e6
    sample = (f"{use}: {shape[0]}x{shape[1]}x{shape[2]} total cells, {W} untimed + {K} timed steps of the reference "
              f"loop (J clear, source, polarization, H, CPML-H, E with gain, CPML-E, probe, populations), {what}, "
              f"{cores} threads on {cpu_model()}; loop {loop_s:.2f} s, process {total:.1f} s with set-up")
    same = use == cfg
    cfgd = workload_config(setup, cfg, desc) if same else dict(workload_config(setup, cfg, desc),
                                                                 sample_grid=shape, sample_config=use)
    return {"metric": "Mcell-updates/s", "value": round(value, 3), "unit": "Mcell-updates/s", "n_gpus": args.gpus,
            "steps": K, "warmup": W, "ms_per_step": round(loop_s * 1e3 / K, 3), "higher_is_better": True,
            "impl": "reference", "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": cfgd,
            "detail": {"fdtd_steps_per_step": 1, "parallelism": f"OpenMP, {cores} host threads",
                       "cpu_model": cpu_model(), "host_mem_available_gb": round(host_mem_gb(), 1),
                       "same_grid_as_gpu_arm": same},
            "cpu_baseline": {"value": round(value, 3), "unit": "Mcell-updates/s", "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": round(value, 3), "unit": "Mcell-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def e2e_run(setup, sample_cfg: str, prec: int, local: int, K: int, S: int, dist, world: int) -> dict:
    """The metric through the public C ABI from host buffers: fdtd_create from the host setup
    (H2D of the material row index and 1-D profiles, layout transpose on the device), K runs of
    S steps each followed by a D2H read of that run's probe samples, a D2H read of the final Ez
    field, fdtd_destroy -- all inside the timed region (wall clock, synchronised)."""
    import numpy as np
    cells = setup.shape[0] * setup.shape[1] * setup.shape[2]
    coef_word = 8 if prec == PKG.PREC_FP64 else 4
    warm = PKG.Solver(PKG.Setup.from_file(PKG.config_path(sample_cfg)), device=local, precision=prec)
    warm.run(S)
    warm.probe_series()
    warm.field("Ez")
    warm.close()
    del warm
    # bytes fdtd_create copies host -> device: the material (the setup's row index, 2 bytes per
    # cell, and its row table -- or bE as three FP64 idx3 arrays), 1-D spacing / CPML arrays,
    # gain box (counted before the timed region)
    nrows = int(setup.view.n_bE_rows)
    h2d = (2 * cells + 24 * nrows if nrows else 3 * cells * 8) + sum(8 * n for n in setup.shape) * 16
    if setup.view.n_tls_regions:
        m = setup.array("tls_region_map").reshape(setup.shape) >= 0
        box = int(np.prod([np.ptp(np.nonzero(m.any(axis=tuple(x for x in range(3) if x != ax)))[0]) + 1
                           for ax in range(3)]))
        h2d += box * (2 * coef_word + 1)
        del m
    barrier(dist)
    t0 = time.perf_counter()
    s2 = PKG.Solver(setup, device=local, precision=prec)
    d2h = 0
    for _ in range(K):
        s2.run(S)
        series = s2.probe_series()
        d2h += series[-S:].nbytes
    ez = s2.field("Ez")
    d2h += ez.nbytes
    s2.close()
    t_e2e = reduce_max(dist, time.perf_counter() - t0)
    return {"value": round(cells * K * S * world / t_e2e / 1e6, 3), "unit": "Mcell-updates/s",
            "h2d_bytes_per_step": int(h2d / K), "d2h_bytes_per_step": int(d2h / K), "seconds": round(t_e2e, 4)}


def device_run(setup, form: str, shards: int, W: int, K: int, S: int, local: int, dist, devices=None) -> dict:
    """W untimed and K timed runs of S steps, inputs resident; device time from CUDA events on
    the library's stream(s), max over ranks; the solve is returned open.  devices: the shards'
    GPUs (one solve split over several GPUs), else all shards on `local`."""
    sol = PKG.Solver(setup, device=local, precision=PREC[form], shards=shards, devices=devices)
    for _ in range(W):
        sol.run(S)
    sol.synchronize()
    sol.set_timing(PKG.TIMING_RUN)
    barrier(dist)
    clocks = ClockSampler(local)
    clocks.start()
    t_wall = time.perf_counter()
    launches_a = sol.kernel_launches
    for _ in range(K):
        sol.run(S)
    sol.synchronize()
    t_wall = time.perf_counter() - t_wall
    launches = sol.kernel_launches - launches_a
    clk = clocks.stop()
    barrier(dist)
    dev_ms = sol.timing()["run_ms"]
    return {"solve": sol, "dev_ms_max": reduce_max(dist, dev_ms), "wall_ms": t_wall * 1e3, "launches": launches,
            "clocks": clk}


def accuracy(sols: dict, ref) -> dict:
    """Storage forms against the FP64 solve of the same run: relative L2 of the stacked E and
    H components, of the probe series and of the DFT.  Each FP64 component is read once."""
    import numpy as np
    num = {f: {"E": 0.0, "H": 0.0} for f in sols}
    den = {"E": 0.0, "H": 0.0}
    for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        b = ref.field(c)
        den[c[0]] += float(np.dot(b.ravel(), b.ravel()))
        for f, sol in sols.items():
            d = sol.field(c)
            np.subtract(d, b, out=d)
            num[f][c[0]] += float(np.dot(d.ravel(), d.ravel()))
            del d
        del b
    pr, dr = ref.probe_series(), ref.dft(0)

    def rel(x, y):
        return float(np.linalg.norm(np.ravel(x - y)) / np.linalg.norm(np.ravel(y)))
    out = {}
    for f, sol in sols.items():
        ps, ds = sol.probe_series(), sol.dft(0)
        out[f] = {"E_field_rel_l2": float((num[f]["E"] / den["E"]) ** 0.5),
                  "H_field_rel_l2": float((num[f]["H"] / den["H"]) ** 0.5),
                  "probe_rel_l2": rel(ps, pr), "dft_rel_l2": rel(ds, dr),
                  "dft_peak_same_bin": bool(np.argmax(np.abs(ds)) == np.argmax(np.abs(dr)))}
    return out


def kernel_roofline(setup, form: str, S: int, K: int, local: int) -> dict:
    """Per-kernel CUDA events (one synchronisation per step) on a whole solve of the workload:
    the E sweep's algorithmic bytes per launch over its average launch time, against the
    measured copy bandwidth of this pool's B200s."""
    word = WORD[form]
    coef_word = 8 if form == "fp64" else 4
    sol = PKG.Solver(setup, device=local, precision=PREC[form])
    alg = algorithmic_bytes(setup, word, coef_word, 2 if sol.material_rows else 0)
    sol.run(S)
    sol.set_timing(PKG.TIMING_KERNELS)
    for _ in range(min(K, 5)):
        sol.run(S)
    tm = sol.timing()
    sol.close()
    e_ms = tm["e_ms"] / tm["steps"]
    h_ms = tm["h_ms"] / tm["steps"]
    peak, peak_src = peaks()
    achieved = alg["e_bytes"] / (e_ms * 1e-3) / 1e9
    traffic = None
    prof = ROOT / "profiles" / f"k_update_E_b512_{form}_traffic.json"
    if prof.exists():
        traffic = json.loads(prof.read_text()).get("dram_bytes_per_launch")
    return {"roofline": {"bound": "hbm", "kernel": "k_update_E", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_src,
                         "traffic": traffic, "algorithmic_bytes_per_launch": alg["e_bytes"],
                         "avg_launch_ms": round(e_ms, 5), "h_sweep_avg_launch_ms": round(h_ms, 5),
                         "h_sweep_achieved": round(alg["h_bytes"] / (h_ms * 1e-3) / 1e9, 1)},
            "hbm_gbs_step": round(alg["step_bytes"] / ((e_ms + h_ms) * 1e-3) / 1e9, 1),
            "per_cell": round(alg["per_cell"], 2)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="b512", choices=sorted(WORKLOADS))
    ap.add_argument("--fdtd-steps", type=int, default=10, help="time steps per bench step")
    ap.add_argument("--precision", default="fp64", choices=["fp32", "fp64", "fp16", "bf16"],
                    help="the headline's storage: fp64 (the reference's arithmetic), fp32, or fp16/bf16 (E, H, "
                         "psi stored in 16 bits, FP32 arithmetic)")
    ap.add_argument("--forms", default="fp64,fp32,bf16,fp16",
                    help="storage forms measured beside the headline, each with its roofline and its accuracy "
                         "against the FP64 solve (the FP64 solve is needed for the accuracy blocks)")
    ap.add_argument("--serving", action="store_true",
                    help="serving form: a stream of small solves through the packed engine (own JSON line)")
    ap.add_argument("--serving-jobs", type=int, default=48)
    ap.add_argument("--serving-edges", type=int, nargs=2, default=[32, 192], help="core edge range (cells)")
    ap.add_argument("--serving-steps", type=int, nargs=2, default=[2000, 20000], help="step count range")
    ap.add_argument("--sweep", action="store_true",
                    help="the batched BF16 gain-laser sweep through the packed engine (own JSON line)")
    ap.add_argument("--sweep-jobs", type=int, default=256)
    ap.add_argument("--sweep-steps", type=int, default=1000, help="steps per cavity (the full sweep is 200000)")
    ap.add_argument("--sweep-forms", default="bf16,fp32", help="storage forms of the sweep; the first reports end states")
    ap.add_argument("--sweep-probe-steps", type=int, default=200)
    ap.add_argument("--sweep-check", action="store_true",
                    help="the sweep's BF16 cavities against FP64 on 8 of them: peak, ring-down, Q (own JSON line)")
    ap.add_argument("--check-steps", type=int, default=20000)
    ap.add_argument("--check-forms", default="bf16,bf16sr,fp16,fp32")
    ap.add_argument("--precision-study", action="store_true",
                    help="FP64 / FP32 / FP16 / BF16 errors on --workload (own JSON line)")
    ap.add_argument("--study-steps", type=int, default=5000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    # z shards of the solve on one GPU (0: the fastest per storage form, shards_for); results are
    # identical whatever the count.
    ap.add_argument("--shard-gpus", action="store_true",
                    help="with --gpus N > 1: one solve split along z over the N GPUs of this node, driven by one "
                         "process (strong scaling; rank 0 only under torchrun), instead of N replicas")
    ap.add_argument("--shards", type=int, default=0,
                    help="z shards of the solve on this GPU (fdtd_create_sharded; their sweeps overlap)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    cfg, sample_cfg, desc = WORKLOADS[args.workload]
    rank, local, world, dist = dist_setup(args.gpus)
    S, K, W = args.fdtd_steps, args.steps, args.warmup

    if args.precision_study and args.impl != "reference":
        if rank == 0:
            precision_study(args)
        return

    if args.sweep_check and args.impl != "reference":
        if rank == 0:
            sweep_check(args)
        return

    if args.sweep and args.impl != "reference":
        if rank == 0:
            sweep_bench(args)
        return

    if args.serving and args.impl != "reference":
        if rank == 0:
            serving_bench(args)
        return

    if args.impl == "reference":
        if rank != 0:
            return
        print(json.dumps(reference_arm(args, cfg, sample_cfg, desc, K, W)))
        return

    if args.shard_gpus and args.gpus > 1:
        # one process drives the sharded solve on all N GPUs; under torchrun the other ranks
        # have nothing to run
        if rank != 0:
            return
        world, dist = 1, None
    setup = PKG.Setup.from_file(PKG.config_path(cfg))
    cells = setup.shape[0] * setup.shape[1] * setup.shape[2]
    head = args.precision
    forms = [head] + [f for f in args.forms.split(",") if f and f != head]

    # ---------------------------------------------------------------- e2e through the C ABI
    # Measured first, as a user's first solve in a process: after a warm-up solve of the same
    # physics on the small sample grid (CUDA context, kernel modules), before the device-
    # resident runs, whose retired solves would leave the memory pool in their own pieces.
    e2e = None if args.no_e2e else e2e_run(setup, sample_cfg, PREC[head], local, K, S, dist, world)

    # ---------------------------------------------------------------- device-resident values
    # Every storage form steps the same workload from the same state for W + K runs of S
    # steps; the FP64 solve stays open as the accuracy reference of the others.
    runs = {}
    shard_devs = list(range(args.gpus)) if args.shard_gpus and args.gpus > 1 else None
    for f in forms:
        if shard_devs:
            runs[f] = device_run(setup, f, len(shard_devs), W, K, S, 0, None, devices=shard_devs)
        else:
            runs[f] = device_run(setup, f, shards_for(args, f), W, K, S, local, dist)
    ref_sol = runs["fp64"]["solve"] if "fp64" in runs else None
    acc = {}
    if ref_sol is not None:
        acc = accuracy({f: runs[f]["solve"] for f in forms if f != "fp64"}, ref_sol)
    for f in forms:
        runs[f]["solve"].close()
        runs[f]["solve"] = None
    roof = {f: kernel_roofline(setup, f, S, K, local) for f in forms}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        _, cpu = cpu_reference(sample_cfg, 3, 3, 10 if args.workload == "b512" else S)
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    def block(f):
        r = runs[f]
        b = {"value": round(replica_value(cells, K * S, world, r["dev_ms_max"]), 3), "unit": "Mcell-updates/s",
             "ms_per_step": round(r["dev_ms_max"] / K, 4), "dtype": DTYPE[f], "roofline": roof[f]["roofline"],
             "hbm_gbs_step": roof[f]["hbm_gbs_step"], "algorithmic_bytes_per_cell_step": roof[f]["per_cell"]}
        if f in acc:
            b["accuracy_vs_fp64"] = acc[f]
        return b

    h = runs[head]
    line = {
        "metric": "Mcell-updates/s",
        "value": round(replica_value(cells, K * S, world, h["dev_ms_max"]), 3),
        "unit": "Mcell-updates/s",
        "n_gpus": args.gpus if shard_devs else world,
        "steps": K,
        "warmup": W,
        "ms_per_step": round(h["dev_ms_max"] / K, 4),
        "higher_is_better": True,
        "scaling": "strong" if shard_devs else "weak",
        "vs_baseline": None,
        "dtype": DTYPE[head],
        "data": "synthetic",
        "config": workload_config(setup, cfg, desc),
        "detail": {"fdtd_steps_per_step": S,
                   "parallelism": (f"1 solve sharded along z over {args.gpus} GPUs (peer halo copies)" if shard_devs else
                                   ("replicas, one per GPU" if world > 1 else "single GPU")
                                   + (f", {shards_for(args, head)} z-shards of the solve overlapped on the GPU"
                                      if shards_for(args, head) > 1 else "")),
                   "roofline_timing": "whole (unsharded) solve, per-kernel CUDA events on the library's stream",
                   "kernel_path": "separate H and E sweeps",
                   "l2": "state (%.1f GB of fields) larger than L2 (126 MB), no flush" % (cells * WORD[head] * 6 / 1e9),
                   "wall_ms_per_step": round(h["wall_ms"] / K, 4),
                   "accuracy_note": "each form against the FP64 solve after the same W + K runs of S steps "
                                    "from the same initial state: relative L2 of the stacked E and H components, "
                                    "of the probe series and of the 21-frequency DFT",
                   "accuracy_steps": (W + K) * S,
                   "accuracy_window": "the default 230 steps lie in the rise of the dipole's pulse: the FP64 "
                                      "Ez at the probe (50 cells from the source) stays below 2.0e-6 V/m, under "
                                      "FP16's smallest subnormal at the automatic field scale (sE = 64, the "
                                      "source cell's peak stored near 4096: 2^-24 sE = 3.8e-6 V/m), so the FP16 "
                                      "probe and DFT read 0 (error 1.0); BF16 has FP32's range.  The 16-bit "
                                      "forms over a whole pulse: the precision study (--precision-study) and "
                                      "the sweep check (--sweep-check)"},
        "roofline": roof[head]["roofline"],
        "e2e": e2e,
        "cpu_baseline": cpu,
        "gpu_launches": int(h["launches"]),
        "clocks": h["clocks"],
    }
    line["detail"]["hbm_gbs_step"] = roof[head]["hbm_gbs_step"]
    line["detail"]["algorithmic_bytes_per_cell_step"] = roof[head]["per_cell"]
    for f in forms:
        if f != head:
            line[f] = block(f)
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
