#!/usr/bin/env python
"""Benchmark: ns/day and atom-steps/s of CAPS's MD step on the 32,000-atom polystyrene PME melt, on one B200, in the mixed
FP32/fixed-point form against the FP64 form at a stated force error.

Workload (the reference's configuration "All-atom atactic polystyrene melt with PME"): 40 chains x 50 repeat units x 16
atoms = 32,000 atoms, atactic, cubic box at 1.04 g/cm^3, OPLS-AA-style LJ 12-6 with geometric mixing, cut-off 12 Å with a
2 Å Verlet buffer, partial charges (aromatic C -0.115 / H +0.115, backbone neutral), 1-2/1-3 excluded, 1-4 scaled 0.5, PME
(rtol 1e-5, 1.0 Å spacing, order 4), SHAKE on C-H, Nose-Hoover chain NVT at 500 K, dt 1 fs. The cell is synthetic (seeded
growth, device push-off and equilibration: caps_b200/data/make_ps32k.py); the starting positions and velocities are
caps_b200/data/ps32k_start.npz.

A step is one MD step. value: simulated ns/day summed over the replicas of the job (one per GPU, no collective: the
path does not shard; replicas only), from CUDA events around every step on the engine's stream, with a 256 MB L2
flush between steps outside the events. e2e: the same metric through the C ABI call caps_gpu_run with host buffers
(wall clock around the call: setup, first force, host<->device copies included).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl caps_b200|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

REF_SECONDS = 60.0           # bound on the reference arm's timed sample (CPU)
CPU_SAMPLE_SECONDS = 15.0    # bound on the cpu_baseline sample beside the GPU run
# DRAM bytes (read + write) of one k_pair_f32 launch on this workload, from an ncu capture of that kernel (cold L2)
PAIR_DRAM_BYTES = 10.94e6
# FP32 flops of one interacting pair on a force-only step, FMA as 2: separation, r^2 and its inverse powers 11 (the
# reciprocal square root not counted), LJ 12-6 6, the Ewald real-space term through its rational fit 33, force
# components and their sums 9
FLOPS_PER_PAIR = 59
FLUSH_BYTES = 256 << 20      # > 126 MB L2
START = ROOT / "caps_b200" / "data" / "ps32k_start.npz"
WORKLOAD = {"workload": "polystyrene PME melt, 40 chains x 50 units x 16 atoms = 32,000 atoms", "box_A": None, "density_g_cm3": 1.04,
            "cutoff_A": 12.0, "skin_A": 2.0, "pme": "rtol 1e-5, spacing 1.0 Å, order 4", "constraints": "SHAKE on C-H",
            "thermostat": "Nose-Hoover chain 500 K", "dt_fs": 1.0, "l2": "256 MB flush between timed steps"}


# One metric string for both arms (this engine and the reference's CPU path), so that their lines compare directly; the
# arithmetic each arm runs in is its "dtype".
METRIC = "ns/day (32k-atom polystyrene PME melt, MD step)"


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown CPU"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


class Clocks:
    """nvidia-smi sampled every 200 ms during the timed region: median SM clock under load and throttle reasons."""

    def __init__(self, index: int):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        q = "index,clocks.sm,clocks.max.sm,power.draw,utilization.gpu,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
            "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def wait_first(self, seconds: float = 5.0):
        """Waits (a few seconds at most) for nvidia-smi's first sample, so that the sampling covers what follows."""
        t0 = time.perf_counter()
        while self.proc and not self.rows and time.perf_counter() - t0 < seconds:
            time.sleep(0.05)

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        import statistics
        rows = [r for r in self.rows if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        load = [r for r in rows if r[4].isdigit() and int(r[4]) > 10] or rows
        sm = [float(r[1]) for r in load if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in load for k in range(4) if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(load),
                "window": "from the warm-up to the end of the GPU work (timed steps, end-to-end calls, pair-kernel timing, FP64 and "
                          "NVE runs); samples with the GPU busy"}


def workload():
    import numpy as np

    from caps_b200.systems import polystyrene_melt
    z = np.load(START)
    ff, _, cell = polystyrene_melt(40, 50, 1.04, seed=1, grow=False)
    return ff, z["x"].astype(np.float64), z["v"].astype(np.float64), z["cell"].astype(np.float64)


def options(precision: str, steps: int, seed: int, thermostat: str = "nose-hoover", thermo_every: int | None = None):
    from caps_b200 import DynamicsOptions, EnergyOptions
    eo = EnergyOptions(cutoff=12.0, skin=2.0, electrostatics="pme", ewald_rtol=1e-5, pme_spacing=1.0, pme_order=4, tail=True, precision=precision)
    return DynamicsOptions(dt=1.0, steps=steps, temperature=500.0, thermostat=thermostat, tau_t=100.0, constraints="h-bonds", seed=seed,
                           thermo_every=thermo_every or max(steps, 1), energy=eo)


E2E_CALLS = 5


def force_errors(f, f_ref, e, e_ref) -> dict:
    """RMS force error relative to the RMS force, per-atom relative error (RMS and max), relative energy error."""
    import numpy as np
    f, f_ref = np.asarray(f).reshape(-1, 3), np.asarray(f_ref).reshape(-1, 3)
    df = f - f_ref
    per_atom = np.linalg.norm(df, axis=1) / np.maximum(np.linalg.norm(f_ref, axis=1), 1e-12)
    return {"rms_relative": float(np.sqrt((df ** 2).sum(1).mean() / (f_ref ** 2).sum(1).mean())),
            "per_atom_rms": float(np.sqrt(np.mean(per_atom ** 2))), "per_atom_max": float(per_atom.max()),
            "energy_relative": float(abs(e - e_ref) / abs(e_ref))}

# An earlier measurement on B200s of the same kind (HBM copy GB/s, max SM clock), used when no measured-peaks file is present
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "sm_max_mhz": 1965.0}


def measured_peaks() -> dict:
    """The measured denominators (MEASURED_PEAKS.json), else the fallback; "source" says which."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        d.setdefault("source", "measured")
        return d
    return dict(FALLBACK_PEAKS, source="fallback")


# --- the other configurations (python bench.py --config NAME): one JSON line each, beside the headline ---------------
CONFIGS = ("kg", "water", "replicas", "composite")


def _timed(ev, x, cell, opts, v=None) -> tuple[float, dict]:
    """Device ms per step of a run in measurement mode (per-step events, L2 flushed between steps), and its result."""
    ev.set_timing(FLUSH_BYTES)
    out = ev.run(x, cell, opts, v=v)
    ev.set_timing(-1)
    return ev.last_step_ms(), out


def _errors_vs(ff, eo_mixed, eo_fp64, x, cell, oracle: bool) -> dict:
    """Mixed forces against this engine's FP64 forces on one frame, and against the reference's (oracle) when asked."""
    from caps_b200 import Evaluator
    em, ed = Evaluator(ff, eo_mixed), Evaluator(ff, eo_fp64)
    tm, fm = em.compute(x, cell)
    td, fd = ed.compute(x, cell)
    em.close()
    ed.close()
    out = {"vs_fp64": force_errors(fm, fd, tm["total"], td["total"])}
    if oracle:
        try:
            from oracle import ref
            if ref.available():
                tr, fr = ref.compute(ff, eo_fp64, x, cell, threads=os.cpu_count() or 1)
                er = sum(tr[k] for k in ("bond", "angle", "dihedral", "improper", "vdw", "coulomb"))
                out["vs_oracle"] = force_errors(fm, fr, tm["total"], er)
                out["fp64_vs_oracle"] = force_errors(fd, fr, td["total"], er)
        except Exception as e:   # the check is reported, not required
            out["vs_oracle"] = f"failed: {e}"
    return out


def _drift(rows, n) -> float:
    """NVE drift of the conserved energy, kT per ns per atom, from a linear fit over the thermo rows."""
    import numpy as np
    cons = np.array([r["conserved"] for r in rows])
    tps = np.array([r["time_ps"] for r in rows])
    slope = float(np.polyfit(tps, cons, 1)[0]) if len(cons) > 2 else 0.0
    kT = 0.0019872041 * float(np.mean([r["temperature"] for r in rows]))
    return slope * 1000.0 / kT / n


def _line(name: str, n: int, dt: float, ms: float, ms64: float | None, extra: dict) -> dict:
    sps = 1000.0 / ms
    line = {"config": name, "metric": f"ns/day ({name})", "unit": "ns/day", "value": sps * dt * 86400e-6, "ms_per_step": ms,
            "atom_steps_per_s": sps * n, "atoms": n, "dt_fs": dt, "n_gpus": 1, "data": "synthetic",
            "l2": "256 MB flush between timed steps"}
    if ms64:
        line["fp64"] = {"ns_per_day": 1000.0 / ms64 * dt * 86400e-6, "ms_per_step": ms64, "atom_steps_per_s": 1000.0 / ms64 * n,
                        "mixed_speedup": ms64 / ms}
    line.update(extra)
    return line


def run_config(args) -> dict:
    import numpy as np

    from caps_b200 import DynamicsOptions, EnergyOptions, Evaluator, run_batch
    from caps_b200 import systems as S
    t_build = time.perf_counter()
    if args.config == "kg":
        # Kremer-Grest 100 x 50 beads at 0.85 sigma^-3, sigma = 1 Å, eps = 1 kcal/mol, m = 1 g/mol: tau = 48.888 fs,
        # dt = 0.01 tau, T* = 1 is 1/kB K, Langevin gamma = 0.5/tau (tau_t = 2 tau)
        tau = 48.888
        ff, x, cell = S.kg_melt(100, 50, 0.85, seed=1)
        kw = dict(cutoff=2.0 ** (1 / 6), skin=0.4, coulomb=False, tail=False)
        T = 1.0 / 0.0019872041
        x = S.push_off(ff, x, cell, kw, temperature=T, steps=400, log=log)
        dyn = lambda prec, steps, seed: DynamicsOptions(dt=0.01 * tau, steps=steps, temperature=T, thermostat="langevin", tau_t=2 * tau,
                                                        seed=seed, thermo_every=max(steps, 1), energy=EnergyOptions(**kw, precision=prec))
        dt = 0.01 * tau
    elif args.config == "water":
        ff, x, cell = S.spce_water(100000, 0.997, seed=1)
        kw = dict(cutoff=10.0, skin=2.0, electrostatics="pme", ewald_rtol=1e-5, pme_spacing=1.2, pme_order=4, tail=True)
        x = S.push_off(ff, x, cell, kw, temperature=300.0, steps=300, log=log)
        dyn = lambda prec, steps, seed: DynamicsOptions(dt=2.0, steps=steps, temperature=300.0, thermostat="bussi", tau_t=100.0,
                                                        constraints="h-bonds", seed=seed, thermo_every=max(steps, 1),
                                                        energy=EnergyOptions(**kw, precision=prec))
        dt = 2.0
    elif args.config == "composite":
        ff, x, cell = S.rubber_composite(1_000_000, sheets=4, units=200, density=0.91, seed=1)
        kw = dict(cutoff=12.0, skin=2.0, electrostatics="pme", ewald_rtol=1e-5, pme_spacing=1.0, pme_order=4, tail=True)
        x = S.push_off(ff, x, cell, kw, temperature=300.0, steps=300, log=log)
        dyn = lambda prec, steps, seed: DynamicsOptions(dt=1.0, steps=steps, temperature=300.0, thermostat="bussi", tau_t=100.0,
                                                        barostat="c-rescale", pressure=1.0, tau_p=1000.0, barostat_every=10, respa=2,
                                                        respa_split="pme", seed=seed, thermo_every=max(steps, 1),
                                                        energy=EnergyOptions(**kw, precision=prec))
        dt = 1.0
    elif args.config == "replicas":
        return run_replicas(args)
    else:
        raise SystemExit(f"--config takes one of {', '.join(CONFIGS)}")
    n = ff.natoms
    build_s = time.perf_counter() - t_build
    log(f"[bench] {args.config}: {n} atoms built and pushed off in {build_s:.0f} s")
    ev = Evaluator(ff, dyn("mixed", 1, 1).energy)
    out = ev.run(x, cell, dyn("mixed", max(args.warmup, 200), 3))
    x1, v1, c1 = out["x"], out["v"], out["cell"]
    ms, out = _timed(ev, x1, c1, dyn("mixed", args.steps, 5), v1)
    x2, v2, c2 = out["x"], out["v"], out["cell"]
    ev.close()
    e64 = Evaluator(ff, dyn("double", 1, 1).energy)
    e64.run(x1, c1, dyn("double", 20, 3), v=v1)
    ms64, _ = _timed(e64, x1, c1, dyn("double", max(20, args.steps // 4), 5), v1)
    e64.close()
    extra = {"build_s": build_s, "errors_end_frame": _errors_vs(ff, dyn("mixed", 1, 1).energy, dyn("double", 1, 1).energy, x2, c2,
                                                                 oracle=args.config != "composite" or n <= 1_100_000)}
    if args.config == "water":
        # NVE drift of both paths over args.drift_ps picoseconds from the same state (SETTLE, 2 fs)
        nsteps = int(args.drift_ps * 1000 / dt)
        drift = {}
        for prec in ("mixed", "double"):
            o = dyn(prec, nsteps, 9)
            o.thermostat = "none"
            o.thermo_every = max(1, nsteps // 100)
            e = Evaluator(ff, o.energy)
            rows = e.run(x2, c2, o, v=v2)["thermo"]
            e.close()
            drift[prec] = {"kT_per_ns_per_atom": _drift(rows, n), "ps": args.drift_ps}
        extra["nve_drift"] = drift
    if args.config == "composite":
        extra["density_g_cm3_end"] = float(ff.mass.sum() / 6.02214076e23 / (abs(np.linalg.det(c2[3:].reshape(3, 3))) * 1e-24))
        extra["run"] = "Bussi 300 K, c-rescale 1 atm every 10 steps, r-RESPA with PME every 2 steps (PME outer, the rest inner at 0.5 fs)"
    return _line(args.config, n, dt, ms, ms64, extra)


def run_replicas(args) -> dict:
    """64 cis-polyisoprene melts of 4-46 chains x 100 units (5.2k-59.8k atoms), each at its own rung of a 500 -> 150 K
    ladder (replica k at 500 - 10 (k mod 36) K), Langevin, dt 1 fs, in lock step through run_batch, against one system
    of the same total size (one melt of all their chains)."""
    import numpy as np

    from caps_b200 import DynamicsOptions, EnergyOptions, Evaluator, run_batch
    from caps_b200 import systems as S
    rng = np.random.default_rng(2024)
    R = args.replicas_count
    chains = rng.integers(4, 47, size=R)
    kw = dict(cutoff=10.0, skin=2.0, electrostatics="pme", ewald_rtol=1e-5, pme_spacing=1.0, pme_order=4, tail=True)
    t0 = time.perf_counter()
    systems = [S.polyisoprene_melt(int(c), 100, 0.91, seed=100 + r) for r, c in enumerate(chains)]
    ffs = [s_[0] for s_ in systems]
    cells = [s_[2] for s_ in systems]
    xs = S.push_off_batch(ffs, [s_[1] for s_ in systems], cells, kw, temperature=400.0, steps=300, log=log)
    temps = [500.0 - 10.0 * (k % 36) for k in range(R)]
    lang = lambda r, steps, prec="mixed": DynamicsOptions(dt=1.0, steps=steps, temperature=temps[r], thermostat="langevin", tau_t=100.0,
                                                           seed=11 + r, thermo_every=max(steps, 1), energy=EnergyOptions(**kw, precision=prec))
    evs = [Evaluator(ff, lang(r, 1).energy) for r, ff in enumerate(ffs)]
    out = run_batch(evs, xs, cells, [lang(r, max(args.warmup, 100)) for r in range(R)])
    xs, vs = [o["x"] for o in out], [o["v"] for o in out]
    run_batch(evs, xs, cells, [lang(r, args.steps) for r in range(R)], vs=vs)
    batch_sps = evs[0].steps_per_second()
    for e in evs:
        e.close()
    n_total = int(sum(ff.natoms for ff in ffs))
    # one system of the same size: a melt of all the replicas' chains
    fb, xb, cb = S.polyisoprene_melt(int(chains.sum()), 100, 0.91, seed=7)
    xb = S.push_off(fb, xb, cb, kw, temperature=400.0, steps=300, log=log)
    big = DynamicsOptions(dt=1.0, steps=max(args.warmup, 100), temperature=400.0, thermostat="langevin", tau_t=100.0, seed=3,
                          thermo_every=max(args.warmup, 100), energy=EnergyOptions(**kw, precision="mixed"))
    eb = Evaluator(fb, big.energy)
    ob = eb.run(xb, cb, big)
    big.steps, big.thermo_every = args.steps, args.steps
    eb.run(ob["x"], cb, big, v=ob["v"])
    big_sps = eb.steps_per_second()
    eb.close()
    eff = batch_sps * n_total / (big_sps * fb.natoms) if big_sps > 0 else None
    return {"config": "replicas", "metric": "atom-steps/s (64 uneven polyisoprene replicas, one graph per step)", "unit": "atom-steps/s",
            "value": batch_sps * n_total, "replicas": R, "atoms_total": n_total, "atoms_min": int(min(ff.natoms for ff in ffs)),
            "atoms_max": int(max(ff.natoms for ff in ffs)), "ns_per_day_each": batch_sps * 86400e-6, "steps": args.steps,
            "single_system_atoms": fb.natoms, "single_system_atom_steps_per_s": big_sps * fb.natoms, "efficiency": eff,
            "ladder": "replica k at 500 - 10 (k mod 36) K, Langevin, dt 1 fs, mixed", "build_s": time.perf_counter() - t0,
            "timing": "device time over the step loop (CUDA events), L2 not flushed", "data": "synthetic"}


def step_timeline(args) -> dict:
    """Where a mixed MD step's time goes, kernel by kernel, with the concurrency of its graph: the kernel records of
    args.profile_timeline steps (after args.warmup), each kernel's start taken from the step's first kernel (the
    integrator's head). Measurement only: torch.profiler reads the CUDA profiling interface's kernel records, which
    include the kernels of replayed CUDA graphs; no L2 flush between the steps."""
    import bisect
    import re
    import statistics
    import tempfile

    import torch
    from torch.profiler import ProfilerActivity, profile

    from caps_b200 import Evaluator
    torch.zeros(1, device="cuda")
    ff, x, v, cell = workload()
    o = options("mixed", max(args.warmup, 50), 7)
    ev = Evaluator(ff, o.energy)
    if args.tuning:
        ev.pin_tuning([int(t) for t in args.tuning.split(",")])
    out = ev.run(x, cell, o, v=v)
    ev.run(out["x"], cell, options("mixed", 50, 7), v=out["v"])
    b0, p0 = ev.list_counts()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        ev.run(out["x"], cell, options("mixed", args.profile_timeline, 7), v=out["v"])
        torch.cuda.synchronize()
    b1, p1 = ev.list_counts()
    tuning = ev.tuning()
    ev.close()
    with tempfile.NamedTemporaryFile(suffix=".json") as tf:
        prof.export_chrome_trace(tf.name)
        trace = json.load(open(tf.name))
    ks = sorted((e for e in trace["traceEvents"] if e.get("cat") == "kernel"), key=lambda e: e["ts"])
    short = lambda n: re.sub(r"capsb::(\(anonymous namespace\)::)?", "", re.sub(r"^void ", "", n)).split("(")[0]
    starts = [e["ts"] for e in ks if "k_nhc_begin" in e["name"]]
    rows: dict = {}
    for e in ks:
        i = bisect.bisect_right(starts, e["ts"]) - 1
        if 0 <= i < len(starts) - 1:
            r = rows.setdefault(short(e["name"]), {"start": [], "dur": []})
            r["start"].append(e["ts"] - starts[i])
            r["dur"].append(e["dur"])
    period = [b - a for a, b in zip(starts, starts[1:])]
    # median start and duration, and the mean duration (gated kernels that did their work on some steps: the list
    # build, the prune)
    kern = sorted(({"kernel": k, "start_us": statistics.median(r["start"]), "us": statistics.median(r["dur"]),
                    "mean_us": statistics.fmean(r["dur"]), "count": len(r["dur"])} for k, r in rows.items()), key=lambda d: d["start_us"])
    return {"timeline_steps": len(period), "step_period_us": statistics.median(period) if period else None,
            "tuning": ",".join(map(str, tuning)), "list_builds": b1 - b0, "prunes": p1 - p0, "kernels": kern}


def run_reference(args, rank: int) -> dict:
    """The reference's own CPU implementation (oracle/_ref: the reference core built from its sources) on this
    workload: run_dynamics in its fastest form (EnergyOptions::mixed = true), all host threads."""
    from oracle import ref
    if not ref.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libcaps_ref.so is not built (make -C oracle where the reference sources are)"}
    ff, x, v, cell = workload()
    threads = os.cpu_count() or 1
    # warm-up (at most 3 steps), then the timed sample: K steps, bounded to about REF_SECONDS of CPU time
    probe = ref.run(ff, x, cell, options("mixed", max(3, min(args.warmup, 10)), 1), v=v, threads=threads)
    per_step = probe["seconds"] / max(3, min(args.warmup, 10)) if probe["seconds"] > 0 else 0.01
    steps = int(max(1, min(args.steps, REF_SECONDS / max(per_step, 1e-6))))
    t0 = time.perf_counter()
    out = ref.run(ff, x, cell, options("mixed", steps, 1), v=v, threads=threads)
    wall = time.perf_counter() - t0
    nsd = out["ns_per_day"]
    n = ff.natoms
    sps = steps / out["seconds"] if out["seconds"] > 0 else 0.0
    cfg = dict(WORKLOAD, box_A=round(float(cell[3]), 3), parallelism="1 CPU process", sample=f"{steps} MD steps")
    return {"impl": "reference", "metric": METRIC, "value": nsd, "unit": "ns/day", "n_gpus": args.gpus,
            "steps": steps, "warmup": args.warmup, "ms_per_step": 1000.0 / sps if sps else None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 pair kernel, f64 sums (reference mixed)", "data": "synthetic", "config": cfg,
            "atom_steps_per_s": sps * n,
            "cpu_baseline": {"value": nsd, "unit": "ns/day", "cores": threads, "kind": "reference",
                             "sample": f"{steps} steps of the reference's run_dynamics on the same cell, EnergyOptions::mixed = true, {threads} threads "
                                       f"on {cpu_model()}, wall {wall:.1f} s; PME through the C++ restatement of the reference's Fortran k-space "
                                       f"module (no Fortran compiler on the box)"},
            "e2e": {"value": nsd, "unit": "ns/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=200)
    ap.add_argument("--impl", default="caps_b200")
    ap.add_argument("--fp64-steps", type=int, default=None)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--replicas", type=int, default=8, help="batched-replica measurement with this many replicas (0: skip)")
    ap.add_argument("--profile-pair", type=int, default=0, metavar="LAUNCHES",
                    help="only time the pair kernel LAUNCHES times on the start structure (a small case for ncu captures)")
    ap.add_argument("--config", default=None, choices=CONFIGS,
                    help="measure another configuration instead of the headline one: kg (5k-bead Kremer-Grest melt), water (300k-atom "
                         "SPC/E, NVE drift), replicas (64 uneven polyisoprene melts in lock step), composite (1M-atom rubber/graphene)")
    ap.add_argument("--drift-ps", type=float, default=100.0, help="NVE drift run length of --config water (ps)")
    ap.add_argument("--replicas-count", type=int, default=64, help="replicas of --config replicas")
    ap.add_argument("--profile-phases", type=int, default=0, metavar="LAUNCHES",
                    help="only time the force evaluation's branches alone and together, and the MD step, in both precisions")
    ap.add_argument("--profile-md", type=int, default=0, metavar="STEPS",
                    help="only run the mixed MD: --warmup steps, then STEPS steps (the command for ncu launch lists)")
    ap.add_argument("--profile-timeline", type=int, default=0, metavar="STEPS",
                    help="only run the mixed MD and print the concurrent kernel timeline of STEPS steps after --warmup steps (kernel "
                         "records of the CUDA profiling interface through torch.profiler): per kernel its median start within the "
                         "step, median duration and count")
    ap.add_argument("--tuning", default=None, metavar="V1,...,V7",
                    help="with --profile-md or --profile-timeline: pin these launch shapes (as a plain run prints them) instead of "
                         "tuning, so that a run under a profiler, which misleads the tuners, uses the shapes of a plain run")
    args = ap.parse_args()
    rank, world, local = int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))
    if args.warmup < 3:
        args.warmup = 3

    if args.profile_pair:
        from caps_b200 import Evaluator
        ff, x, v, cell = workload()
        for prec in ("mixed", "double"):
            ev = Evaluator(ff, options(prec, 1, 1).energy)
            print(json.dumps({"precision": prec, **ev.pair_timing(x, cell, launches=args.profile_pair)}), flush=True)
            ev.close()
        return

    if args.profile_phases:
        from caps_b200 import Evaluator
        ff, x, v, cell = workload()
        for prec in ("mixed", "double"):
            ev = Evaluator(ff, options(prec, 1, 1).energy)
            ph = ev.phase_timing(x, cell, launches=args.profile_phases, flush_bytes=FLUSH_BYTES)
            pt = ev.pair_timing(x, cell, launches=args.profile_phases, flush_bytes=FLUSH_BYTES)
            o = options(prec, args.warmup, 7)
            out = ev.run(x, cell, o, v=v)
            ev.set_timing(FLUSH_BYTES)
            ev.run(out["x"], cell, options(prec, max(args.steps, 50), 7), v=out["v"])
            print(json.dumps({"precision": prec, **ph, "pair_ms": pt["avg_ms"], "step_ms": ev.last_step_ms(),
                              "step_kernels": ev.step_kernels()}), flush=True)
            ev.close()
        return

    if args.profile_md:
        from caps_b200 import Evaluator
        ff, x, v, cell = workload()
        o = options("mixed", args.warmup, 7)
        ev = Evaluator(ff, o.energy)
        if args.tuning:
            ev.pin_tuning([int(t) for t in args.tuning.split(",")])
        out = ev.run(x, cell, o, v=v)
        out = ev.run(out["x"], cell, options("mixed", args.profile_md, 7), v=out["v"])
        print(json.dumps({"profile_md": args.profile_md, "report": out["report"], "kernels_run": ev.kernels_run(),
                          "tuning": ",".join(map(str, ev.tuning()))}), flush=True)
        ev.close()
        return

    if args.profile_timeline:
        print(json.dumps(step_timeline(args)), flush=True)
        return

    if args.config:
        print(json.dumps(run_config(args)), flush=True)
        return

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args, rank)), flush=True)
        return

    # one process per GPU: this rank sees its own device only (the engine takes the current device)
    if world > 1:
        os.environ["CUDA_VISIBLE_DEVICES"] = str(local)
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(0)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist

    import numpy as np

    from caps_b200 import Evaluator
    ff, x, v, cell = workload()
    n = ff.natoms
    seed = 1 + rank

    def barrier():
        if pg:
            pg.barrier()

    def max_over_ranks(val: float) -> float:
        if not pg:
            return val
        import torch
        t = torch.tensor([val], dtype=torch.float64, device="cuda" if pg.get_backend() == "nccl" else "cpu")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        return float(t.item())

    # Clocks are sampled from before the warm-up to the end of the GPU work (the K timed steps last milliseconds, less
    # than the 200 ms sampling period; the samples under load span the timed steps, the end-to-end calls, the FP64 run
    # and the NVE run)
    clk = Clocks(local).__enter__()
    clk.wait_first()
    # --- mixed FP32/fixed-point: warm-up, then K timed steps (events per step, L2 flushed between steps) ---
    o = options("mixed", args.warmup, seed)
    ev = Evaluator(ff, o.energy)
    out = ev.run(x, cell, o, v=v)
    x1, v1 = out["x"], out["v"]
    ev.set_timing(FLUSH_BYTES)
    barrier()
    b0 = ev.list_builds()
    out = ev.run(x1, cell, options("mixed", args.steps, seed), v=v1)
    barrier()
    builds = ev.list_builds() - b0
    ms_step = max_over_ranks(ev.last_step_ms())
    launches = ev.kernels_run()
    print(f"[bench] timed run: {out['report']} · {ev.step_kernels()} kernel nodes per plain step, {launches} kernels run", file=sys.stderr, flush=True)
    ev.set_timing(-1)
    x2, v2 = out["x"], out["v"]
    sps = 1000.0 / ms_step
    nsd = sps * 1.0 * 86400e-6            # dt = 1 fs
    value = nsd * world                    # whole job: the replicas' simulated time per day
    # --- e2e: the C ABI call with host buffers, wall clock around it; the best of E2E_CALLS calls, since the host is
    # shared and a call's set-up and launches can stall behind other processes ---
    walls = []
    for _ in range(E2E_CALLS):
        t0 = time.perf_counter()
        eo_run = ev.run(x2, cell, options("mixed", args.steps, seed), v=v2)
        walls.append(time.perf_counter() - t0)
        print(f"[bench] e2e run: {eo_run['report']}", file=sys.stderr, flush=True)
    e2e_wall = min(walls)
    e2e_nsd = args.steps * 1.0 * 1e-6 / e2e_wall * 86400 * world
    h2d = (2 * 3 * n * 8 + 12 * 8) / args.steps
    d2h = (2 * 3 * n * 8 + 12 * 8 + 2 * 232) / args.steps
    del eo_run
    # --- the dominant kernel (the pair kernel) timed alone: roofline ---
    pt = ev.pair_timing(x2, cell, launches=max(20, min(args.steps, 200)), flush_bytes=FLUSH_BYTES)
    achieved = pt["pairs_in_cutoff"] * FLOPS_PER_PAIR / (pt["avg_ms"] * 1e-3) / 1e12
    peaks = measured_peaks()
    sm_max = peaks.get("sm_max_mhz") or FALLBACK_PEAKS["sm_max_mhz"]
    fp32_peak = 148 * 128 * 2 * sm_max * 1e6 / 1e12   # FP32 FMA issue peak at the measured max clock (not measured directly)
    # --- forces at the end state: mixed vs FP64 ---
    em = Evaluator(ff, options("mixed", 1, seed).energy)
    tm, fm = em.compute(x2, cell)
    ed = Evaluator(ff, options("double", 1, seed).energy)
    td, fd = ed.compute(x2, cell)
    err_fp64 = force_errors(fm, fd, tm["total"], td["total"])
    em.close()
    ed.close()
    # --- the FP64 path on the same workload ---
    k64 = args.fp64_steps or max(100, args.steps // 4)
    ev64 = Evaluator(ff, options("double", args.warmup, seed).energy)
    ev64.run(x2, cell, options("double", args.warmup, seed), v=v2)
    ev64.set_timing(FLUSH_BYTES)
    ev64.run(x2, cell, options("double", k64, seed), v=v2)
    ms64 = max_over_ranks(ev64.last_step_ms())
    nsd64 = 1000.0 / ms64 * 86400e-6
    ev64.close()
    # --- batched replicas (the 64-replica cooling workload's efficiency target): R replicas of this cell, each at its own Langevin temperature,
    # in lock step (one graph launch per plain step), against one equally large system (the cell tiled 2 x 2 x 2) ---
    batch = None
    if args.replicas > 0:
        from caps_b200 import run_batch
        from caps_b200.systems import tile
        R = args.replicas
        kb = max(50, args.steps // 10)
        lang = [options("mixed", kb, seed + r, thermostat="langevin") for r in range(R)]
        for r, o_ in enumerate(lang):
            o_.temperature = 500.0 - 10.0 * r
        evs = [Evaluator(ff, lang[0].energy) for _ in range(R)]
        warm = [options("mixed", 20, seed + r, thermostat="langevin") for r in range(R)]
        run_batch(evs, [x2] * R, [cell] * R, warm, vs=[v2] * R)
        run_batch(evs, [x2] * R, [cell] * R, lang, vs=[v2] * R)
        batch_sps = evs[0].steps_per_second()
        for e_ in evs:
            e_.close()
        fb, xb, cb = tile(ff, x2, cell, (2, 2, 2))
        vb = np.concatenate([v2] * 8)
        eb = Evaluator(fb, lang[0].energy)
        eb.run(xb, cb, options("mixed", 20, seed, thermostat="langevin"), v=vb)
        eb.run(xb, cb, options("mixed", kb, seed, thermostat="langevin"), v=vb)
        big_sps = eb.steps_per_second()
        eb.close()
        batch = {"replicas": R, "atoms_per_replica": n, "steps": kb, "thermostat": "Langevin, 500 K down in 10 K rungs",
                 "atom_steps_per_s": batch_sps * R * n, "single_system_atoms": 8 * n, "single_system_atom_steps_per_s": big_sps * 8 * n,
                 "efficiency": (batch_sps * R * n) / (big_sps * 8 * n) if big_sps > 0 else None,
                 "note": "replicas of this cell (not the polyisoprene sizes of the config); the single system is the cell tiled 2x2x2; "
                         "device time over the step loop, L2 not flushed"}
    # --- NVE drift of the mixed path (2 ps) ---
    nve = options("mixed", 2000, seed, thermostat="none", thermo_every=100)
    outn = ev.run(x2, cell, nve, v=v2)
    cons = np.array([r["conserved"] for r in outn["thermo"]])
    tps = np.array([r["time_ps"] for r in outn["thermo"]])
    slope = float(np.polyfit(tps, cons, 1)[0]) if len(cons) > 2 else 0.0          # kcal/mol/ps
    kT = 0.0019872041 * float(np.mean([r["temperature"] for r in outn["thermo"]]))
    drift_kt_ns_atom = slope * 1000.0 / kT / n
    ev.close()
    clk.__exit__(None, None, None)
    # --- CPU baseline: the reference's own code on the host cores, bounded samples (rank 0, N = 1): its mixed path
    # (its fastest) and its FP64 path; and the checker: the reference's FP64 forces and energy on the end-state frame,
    # against which the mixed and FP64 device forces are reported ---
    cpu, cpu64, err_oracle = None, None, None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            from oracle import ref
            if ref.available():
                threads = os.cpu_count() or 1
                model = cpu_model()
                pme_note = "PME through the C++ restatement of the reference's Fortran k-space module (no Fortran compiler on the box)"
                t_ref, f_ref = ref.compute(ff, options("double", 1, seed).energy, x2, cell, threads=threads)
                e_ref = sum(t_ref[k] for k in ("bond", "angle", "dihedral", "improper", "vdw", "coulomb"))
                err_oracle = {"reference": "the reference's Evaluator::compute, EnergyOptions::mixed = false (FP64), on the end-state frame",
                              "mixed": force_errors(fm, f_ref, tm["total"], e_ref), "fp64": force_errors(fd, f_ref, td["total"], e_ref)}
                for prec, secs in (("mixed", CPU_SAMPLE_SECONDS), ("double", CPU_SAMPLE_SECONDS / 2)):
                    probe = ref.run(ff, x2, cell, options(prec, 3, seed), v=v2, threads=threads)
                    per_step = probe["seconds"] / 3 if probe["seconds"] > 0 else 0.01
                    steps_cpu = int(max(5, min(5000, secs / max(per_step, 1e-6))))
                    r = ref.run(ff, x2, cell, options(prec, steps_cpu, seed), v=v2, threads=threads)
                    row = {"value": r["ns_per_day"], "unit": "ns/day", "cores": threads, "kind": "reference",
                           "sample": f"{steps_cpu} MD steps of the same cell through the reference's run_dynamics "
                                     f"(EnergyOptions::mixed = {'true, its fastest' if prec == 'mixed' else 'false, FP64'}), {threads} threads on "
                                     f"{model}, {r['seconds']:.1f} s; {pme_note}"}
                    if prec == "mixed":
                        cpu = row
                    else:
                        cpu64 = row
        except Exception as e:   # the baseline is reported, not required
            cpu = {"value": None, "unit": "ns/day", "cores": os.cpu_count(), "kind": "reference", "sample": f"failed: {e}"}
    if rank == 0:
        cfg = dict(WORKLOAD, box_A=round(float(cell[3]), 3), parallelism=f"{world} independent replica(s), one per GPU")
        line = {
            "metric": METRIC, "value": value, "unit": "ns/day", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 pair/PME spread-gather, int64 fixed-point sums, f64 FFT/bonded/integrator", "data": "synthetic", "config": cfg,
            "atom_steps_per_s": sps * n * world,
            "list_builds": builds,
            "fp64": {"ns_per_day": nsd64 * world, "ms_per_step": ms64, "steps": k64, "mixed_speedup": ms64 / ms_step},
            "force_error_vs_oracle": err_oracle,
            "force_error_vs_fp64": dict(err_fp64, reference="this engine's FP64 path on the same frame"),
            "nve_drift_kT_per_ns_per_atom": drift_kt_ns_atom,
            "batched_replicas": batch,
            "e2e": {"value": e2e_nsd, "unit": "ns/day", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "calls_s": [round(w, 4) for w in walls], "taken": f"best of {E2E_CALLS} calls",
                    "call": "caps_gpu_run (C ABI) on host buffers, wall clock"},
            "roofline": {"bound": "fp32", "kernel": "k_pair_f32 (LJ + Ewald real space)", "achieved": achieved,
                         "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                         "peak_note": f"FP32 FMA issue rate, 148 SMs x 128 lanes x 2 at the max SM clock ({sm_max:.0f} MHz, of {peaks['source']})",
                         "work": f"{pt['pairs_in_cutoff']:.0f} pairs inside the cut-off x {FLOPS_PER_PAIR} flops per launch",
                         "pair_ms": pt["avg_ms"], "pairs_listed": pt["pairs_listed"], "entries": pt["entries"],
                         "traffic": PAIR_DRAM_BYTES,
                         "traffic_note": "DRAM bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum, cold L2)",
                         "hbm_view": {"achieved_gbs": PAIR_DRAM_BYTES / (pt["avg_ms"] * 1e-3) / 1e9, "peak_gbs": peaks.get("hbm_gbs"),
                                      "peak_source": peaks["source"],
                                      "frac": (PAIR_DRAM_BYTES / (pt["avg_ms"] * 1e-3) / 1e9) / peaks["hbm_gbs"] if peaks.get("hbm_gbs") else None}},
            "gpu_launches": launches,
            "gpu_launches_note": "kernels launched in the timed step loop, counted by the engine: the step graphs' kernel nodes per replayed step (list-build and prune kernels included; they return at once on steps without a build or prune), plus one kinetic-energy kernel per thermo row",
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "cpu_baseline_fp64": cpu64,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
