"""UVLM time-stepper benchmark on B200 (one JSON line on rank 0).

Workload (the metric's configuration): one flat-plate wing, aspect ratio 8
(chord 1, span 8), 32 x 128 = 4096 bound vortex rings, heave
h = 0.2 sin(wt) and pitch 10 deg sin(wt + 90 deg) about the leading-edge root,
reduced frequency k = wc/2U = 0.5 (w = 1), U = 1, dt = 2 pi / w / 40, RK2 wake
advection.  The run is advanced 400 steps so that the wake holds 400 ring rows
(51,200 rings); --erase_wake_after 400 (EraseOldestWake) then keeps it at that
size while steps are timed.  A "step" is one full MainLoop: kinematics, shed,
influence matrix, RHS, solve, Joukowski loads and RK2 roll-up.

value       steps/s of the mixed-precision form (FP32 N-body and assembly,
            stale-LU-preconditioned GMRES with FP64 residuals), device-timed
            with CUDA events on the library's stream, L2 flushed between steps
plain_fp64  steps/s of the plain FP64 form (fresh FP64 LU every step)
cl_rel_err  max |CL_mixed - CL_fp64| / max |CL_fp64| over the 400-step run
e2e         the same metric through the C-ABI, wall-clock, with the load row
            and the circulation vector copied to host memory every step
roofline    the N-body kernel: 59 FLOP per (target, unique segment) pair of
            every N-body launch of a step over their CUDA-event time, against
            the measured FP32 FMA peak of this GPU
cpu_baseline the FP64 CPU oracle (restated reference) on a bounded sample

--impl reference times that CPU oracle alone (the reference cannot be built
here: its third-party libraries and submodules are absent): one complete
MainLoop at the held-wake state, cut into --steps timed slices.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "UVLM steps/s (4096 panels, 50k wake) mixed+learned vs plain FP64, CL err<=1e-6"
ROWS, COLS, CHORD, SPAN = 32, 128, 1.0, 8.0
OMEGA = 1.0  # k = 0.5, c = 1, U = 1
DT = 2 * math.pi / OMEGA / 40
WAKE_ROWS = 400
FLOP_PER_PAIR = 59
# Bounded CPU sample of one MainLoop (a few seconds of host work): the
# N-body stages on every CPU_STRIDE-th target, the full-pivoting LU on the
# leading CPU_LU_N^2 block, each scaled to the whole step.
CPU_STRIDE, CPU_LU_N = 32, 2048
# DRAM bytes of one advection launch of the N-body kernel at the held wake,
# from an ncu capture of the packed FP32x2 tile with the far-field walker
# (bench.py --profile): about the algorithmic bytes (56,115 source records x
# 64 B + targets + outputs).
NBODY_TRAFFIC = {"heave_pitch": 4899072}


def variant_index(name):
    """Index of an N-body tile variant by name (e.g. "fp32_h3_t2_b128_x2f")."""
    import uvlm_b200 as U

    for v in range(64):
        if U.lib().uvlm_nbody_variant_name(v).decode() == name:
            return v
    raise ValueError(name)


def stage_variant_names(st):
    """The N-body tile each stage ran with in the step whose stats are st."""
    import uvlm_b200 as U

    return {name: U.lib().uvlm_nbody_variant_name(int(st.stage_variant[i])).decode()
            for i, name in enumerate(("rhs", "loads", "advect"))}


def make_mixed(device=0, warm_start=None, wl=None, **kw):
    """The mixed-precision form: FP32 N-body, TF32 tensor-core LU factored
    once and used stale as the GMRES preconditioner (its dense inverse), FP64
    residuals, learned warm start where the workload has trained weights
    (trained on 20k plain-solver steps of seeded variations of the workload,
    uvlm_b200/train_warmstart.py), else the extrapolation 2 g_n - g_{n-1}."""
    wl = wl or _heave_pitch()
    if warm_start is None:
        warm_start = "mlp" if wl.weights and os.path.exists(wl.weights) else "extrapolate"
    sim = wl.build("mixed", device=device, solver="gmres_stale", warm_start=warm_start, **kw)
    if warm_start == "mlp":
        from uvlm_b200.warmstart import MLP

        sim.set_mlp(MLP.load(wl.weights))
    return sim


class Workload:
    """A SimpleSimulator set-up in the reference's terms: wings (RectGenerator
    lattice, Morphing kinematics as closed-form sinusoids), forward flight,
    advection scheme, dt, and the wake length held by erase_wake_after."""

    def __init__(self, name, metric, description, wings, advection, dt, wake_rows, weights=None):
        self.name, self.metric, self.description = name, metric, description
        self.wings, self.advection, self.dt, self.wake_rows, self.weights = wings, advection, dt, wake_rows, weights
        self.num = len(wings)
        self.rows, self.cols = wings[0]["rows"], wings[0]["cols"]

    def config(self):
        return {"workload": self.description, "wings": self.num, "rows": self.rows, "cols": self.cols,
                "wake_rings": self.wake_rows * self.cols * self.num, "dt": self.dt, "advection": self.advection,
                "l2": "flushed between timed steps (256 MiB write)"}

    def build(self, precision, **kw):
        import uvlm_b200 as U

        sim = U.SimpleSimulator(precision=precision, erase_wake_after=self.wake_rows,
                                max_wake_rows=self.wake_rows + 8, **kw)
        for w in self.wings:
            m = U.Morphing()
            k = w["kin"]
            m.set_alpha(k.get("alpha", 0.0))
            m.set_plug(k.get("plug_amp", 0.0), k.get("plug_omega", 0.0), k.get("plug_phase", 0.0))
            m.set_twist(k.get("twist_amp", 0.0), k.get("twist_omega", 0.0), k.get("twist_phase", 0.0))
            m.set_bend(k.get("bend_cx", 0.0), k.get("bend_cy", 0.0), k.get("bend_omega", 0.0),
                       k.get("bend_phase", 0.0))
            sim.AddWing(U.RectGenerator(), m, w["chord"], w["span"], w["rows"], w["cols"], w["origin"])
        sim.set_forward_flight([-1.0, 0.0, 0.0])
        sim.set_advection(self.advection)
        return sim

    def oracle(self):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle as o

        sim = o.Simulator()
        for w in self.wings:
            sim.add_wing(w["chord"], w["span"], w["rows"], w["cols"], origin=w["origin"], kin=o.kinematics(**w["kin"]))
        sim.set_forward_flight([-1.0, 0.0, 0.0])
        sim.set_advection(self.advection)
        return sim

    def advect_pairs(self, ignore_rows=5):
        """(target, unique segment) pairs of the advection stage at the held
        wake: the bound sheets and W ring rows of wake as sources, the wake
        node rows 1..W+1 as targets of each evaluation, except the last one of
        RK2 and RK4, whose targets are the rows past ignore_rows (the others
        take the Euler step)."""
        R, Cc, W = self.rows, self.cols, self.wake_rows
        segs = self.num * ((R + 1) * Cc + R * (Cc + 1) + (W + 1) * Cc + W * (Cc + 1))
        full = {"euler": 1, "RK2": 1, "RK4": 2, "AB2": 1}[self.advection]
        rows = full * (W + 1) + (max(0, W + 1 - ignore_rows) if self.advection in ("RK2", "RK4") else 0)
        return self.num * rows * (Cc + 1) * segs


def _heave_pitch():
    return Workload(
        "heave_pitch", METRIC,
        "single flapping wing 32x128 (4096 rings), heave 0.2 sin(wt) + pitch 10deg sin(wt+90deg), k=0.5, RK2, "
        "wake held at 400 rows (51,200 rings) by erase_wake_after=400",
        [dict(chord=CHORD, span=SPAN, rows=ROWS, cols=COLS, origin=(0.0, 0.0, 0.0),
              kin=dict(plug_amp=0.2, plug_omega=OMEGA, twist_amp=math.radians(10), twist_omega=OMEGA,
                       twist_phase=math.pi / 2))],
        "RK2", DT, WAKE_ROWS,
        weights=os.path.join(ROOT, "uvlm_b200", "weights", "warmstart_heave_pitch_32x128.npz"))


def _tandem4():
    # 2 x 2 tandem/biplane arrangement {x=0,1.5} x {z=0,0.5}: phases 0/90 deg
    # for the front lower/upper wing and 180/270 deg for the rear pair, so
    # biplane partners move a quarter period apart (in anti-phase their
    # trailing edges cross and the core-free Biot-Savart diverges); k = 0.4
    # (w = 0.8), heave 0.15 c, pitch 15 deg (90 deg ahead of the heave)
    w, wings = 0.8, []
    for q, (x, z) in enumerate([(0.0, 0.0), (0.0, 0.5), (1.5, 0.0), (1.5, 0.5)]):
        ph = q * math.pi / 2
        wings.append(dict(chord=1.0, span=4.0, rows=16, cols=64, origin=(x, 0.0, z),
                          kin=dict(plug_amp=0.15, plug_omega=w, plug_phase=ph, twist_amp=math.radians(15),
                                   twist_omega=w, twist_phase=ph + math.pi / 2)))
    return Workload("tandem4", "UVLM steps/s (4 wings x 16x64 = 4096 panels, 77k wake), mixed vs plain FP64",
                    "4 flapping wings 16x64 (chord 1, span 4) in a 2x2 tandem/biplane arrangement "
                    "{x=0,1.5}x{z=0,0.5}, phases 0/90 (front) 180/270 deg (rear), k=0.4, heave 0.15 c, "
                    "pitch 15 deg, RK2, wake held at 300 rows per wing (76,800 rings)", wings, "RK2",
                    2 * math.pi / w / 40, 300)


def _morphing():
    # camber z = 0.05 sin(wt) x(1-x) and span bend 0.1 sin(wt) y^2, k = 0.3
    w = 0.6
    return Workload("morphing", "UVLM steps/s (24x96 morphing wing, 57.6k wake), mixed vs plain FP64",
                    "morphing wing 24x96 (chord 1, span 8), camber 0.05 sin(wt) x(1-x) + span bend "
                    "0.1 sin(wt) y^2, k=0.3, Euler, wake held at 600 rows (57,600 rings)",
                    [dict(chord=1.0, span=8.0, rows=24, cols=96, origin=(0.0, 0.0, 0.0),
                          kin=dict(bend_cx=0.05, bend_cy=0.1, bend_omega=w))],
                    "euler", 2 * math.pi / w / 40, 600,
                    weights=os.path.join(ROOT, "uvlm_b200", "weights", "warmstart_morphing_24x96.npz"))


WORKLOADS = {"heave_pitch": _heave_pitch, "tandem4": _tandem4, "morphing": _morphing}


def workload_config():
    return _heave_pitch().config()


def make_sim(precision, wl=None, **kw):
    return (wl or _heave_pitch()).build(precision, **kw)


class Clocks:
    """SM clock and clock-event (throttle) reasons sampled during a timed region.

    NVML (the nvidia_ml_py bindings; read-only queries) every 10 ms where it
    loads, else nvidia-smi every 200 ms (a short region then gets one or two
    samples).  `nvml` replaces the bindings module (tests)."""

    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_index, nvml=None):
        self.gpu = gpu_index
        self.samples = []  # (sm MHz, max sm MHz, active reason names)
        self._stop = threading.Event()
        self._t = None
        self._nvml = nvml
        self._nvml_open = None
        self.source = None

    def _nvml_reader(self):
        mod = self._nvml
        if mod is None:
            try:
                import pynvml as mod
            except Exception:
                return None
        try:
            mod.nvmlInit()
            self._nvml_open = mod
            h = mod.nvmlDeviceGetHandleByIndex(self.gpu)
            # the clocks-event query of newer drivers, else its older name
            get_reasons = mod.nvmlDeviceGetCurrentClocksThrottleReasons
            newer = getattr(mod, "nvmlDeviceGetCurrentClocksEventReasons", None)
            if newer is not None:
                try:
                    newer(h)
                    get_reasons = newer
                except Exception:
                    pass
            bits = (getattr(mod, "nvmlClocksThrottleReasonHwSlowdown", 0x8),
                    getattr(mod, "nvmlClocksThrottleReasonHwThermalSlowdown", 0x40),
                    getattr(mod, "nvmlClocksThrottleReasonSwThermalSlowdown", 0x20),
                    getattr(mod, "nvmlClocksThrottleReasonSwPowerCap", 0x4))
            mx = float(mod.nvmlDeviceGetMaxClockInfo(h, mod.NVML_CLOCK_SM))

            def read():
                mask = int(get_reasons(h))
                return (float(mod.nvmlDeviceGetClockInfo(h, mod.NVML_CLOCK_SM)), mx,
                        tuple(n for n, b in zip(self.NAMES, bits) if mask & b))

            read()
            return read
        except Exception:
            return None

    def _smi_read(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}", "--format=csv,noheader,nounits"],
                             capture_output=True, text=True, timeout=5).stdout.strip()
        if not out:
            return None
        f = [x.strip() for x in out.split(",")]
        num = lambda x: float(x) if x.replace(".", "").isdigit() else None  # noqa: E731
        return (num(f[0]), num(f[1]), tuple(n for i, n in enumerate(self.NAMES) if f[2 + i] == "Active"))

    def start(self):
        read = self._nvml_reader()
        self.source = "nvml" if read else "nvidia-smi"
        period = 0.01 if read else 0.2
        read = read or self._smi_read

        def run():
            while not self._stop.is_set():
                try:
                    smp = read()
                    if smp:
                        self.samples.append(smp)
                except Exception:
                    pass
                self._stop.wait(period)

        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        if self._nvml_open is not None:
            try:
                self._nvml_open.nvmlShutdown()
            except Exception:
                pass
            self._nvml_open = None
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "source": self.source}
        sm = [x[0] for x in self.samples if x[0] is not None]
        mx = [x[1] for x in self.samples if x[1] is not None]
        reasons = sorted({n for x in self.samples for n in x[2]})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples), "source": self.source}


def oracle_sample(wl, state, stride, lu_n, threads):
    """Time one MainLoop of the FP64 CPU oracle on a bounded sample."""
    sim = wl.oracle()
    sim.set_threads(threads)
    sim.begin()
    wr = state["wake_gamma"].shape[1]
    sim.set_state(wr, state["wing_pos"], state["wake_pos"], state["wing_gamma"], state["wing_gamma_prev"],
                  state["wake_gamma"])
    sec = sim.time_step_sampled(wl.wake_rows + 1, wl.dt, stride, lu_n)
    return float(np.sum(sec)), sec


def synthetic_state_np():
    """The metric's shapes without the solver or the oracle: the whole-wing
    lattice moved by the heave/pitch kinematics, its trailing edge convected at
    U (no roll-up) to form 400 wake rows, smooth circulations."""
    xs = np.linspace(0, CHORD, ROWS + 1)
    ys = np.concatenate([-np.linspace(0, SPAN / 2, COLS // 2 + 1)[::-1], np.linspace(0, SPAN / 2, COLS // 2 + 1)[1:]])
    X, Y = np.meshgrid(xs, ys, indexing="ij")

    def move(x, y, t):
        th = math.radians(10) * math.sin(OMEGA * t + math.pi / 2)
        z = 0.2 * math.sin(OMEGA * t)
        return np.stack([math.cos(th) * x, y, -math.sin(th) * x + z], -1)

    t_now = WAKE_ROWS * DT
    wing = move(X, Y, t_now)[None]
    wake = np.stack([move(np.full(COLS + 1, CHORD), ys, t_now - i * DT) + np.array([i * DT, 0, 0])
                     for i in range(WAKE_ROWS + 1)])[None]
    g = np.sqrt(np.clip(1 - np.linspace(-1, 1, COLS) ** 2, 0, None)) * 0.1
    wing_gamma = (np.tile(g, (ROWS, 1)) * np.linspace(1, 0.2, ROWS)[:, None])[None]
    wake_gamma = np.stack([g * 0.1 * math.sin(OMEGA * (t_now - i * DT)) for i in range(WAKE_ROWS)])[None]
    return dict(wing_pos=wing, wake_pos=wake, wing_gamma=wing_gamma, wing_gamma_prev=wing_gamma * 0.99,
                wake_gamma=wake_gamma)


def run_profile(args):
    """The small, quick workloads used for ncu captures: the heave/pitch
    wing's per-step kernels from a synthesized full-size state (default), its
    step 0 alone (--profile-step0: the first TF32 factorisation and dense
    inverse), or the 256-case sweep (--workload batch256: steps + warmup
    batched MainLoops from the start)."""
    import uvlm_b200 as U

    if args.workload == "batch256":
        from uvlm_b200.batch import draw_cases, make_batch

        sim = make_batch(draw_cases(256, seed=0), precision="mixed", max_steps=150)
        sim.run(args.steps + args.warmup)
        sim.close()
        print(json.dumps({"profile": "ok", "workload": "batch256", "steps": args.steps + args.warmup,
                          "launches": int(U.lib().uvlm_kernel_launch_count())}), flush=True)
        return
    # the library's default tiles, not the autotuner (whose timings a profiler distorts)
    pinned = dict(nbody_variant=variant_index(args.variant) if args.variant else
                  variant_index("fp32_h3_t2_b128_x2f" if args.form == "mixed" else
                                              "fp64_h2_t1_b128_m3"))
    if args.profile_step0:
        sim = make_mixed(warm_start="extrapolate", **pinned)
        sim.begin()
        sim.step(0, DT)
        sim.synchronize()
        sim.close()
        print(json.dumps({"profile": "ok", "step0": True, "launches": int(U.lib().uvlm_kernel_launch_count())}),
              flush=True)
        return
    if args.form == "mixed":
        sim = make_mixed(**pinned)
    else:
        sim = make_sim("fp64", **pinned)
    sim.begin()
    sim.step(0, DT)
    st = synthetic_state_np()
    sim.set_state(WAKE_ROWS, st["wing_pos"], st["wake_pos"], st["wing_gamma"], st["wing_gamma_prev"],
                  st["wake_gamma"])
    for i in range(args.warmup + args.steps):
        sim.step(WAKE_ROWS + 1 + i, DT)
    sim.synchronize()
    print(json.dumps({"profile": "ok", "steps": args.steps, "warmup": args.warmup,
                      "launches": int(U.lib().uvlm_kernel_launch_count())}), flush=True)
    sim.close()


def cpu_threads():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()


def headline_config(wl, world):
    """The `config` of the headline line, shared by both arms."""
    learned = bool(wl.weights and os.path.exists(wl.weights))
    return dict(wl.config(), parallelism=f"replicas x{world}",
                form=("mixed+learned" if learned else "mixed") + ": FP32 N-body, TF32 tcgen05 LU factored once (dense "
                     "inverse as the GMRES preconditioner), FP64 matrix and residuals, " +
                     ("MLP warm start" if learned else "warm start 2 g_n - g_{n-1}"))


def run_reference(args, rank, world):
    """The reference's CPU method (the FP64 oracle restating it; the reference itself cannot be built here),
    timed on one complete, unsampled MainLoop at the held-wake state of the headline workload, with every
    host thread on the loops the reference parallelises and the FullPivLU single-threaded as Eigen's.  The
    MainLoop is cut into --steps consecutive slices of about equal estimated time (every slice runs part of
    the same loop; all of them together are exactly one MainLoop), one slice per timed step, so the whole
    run stays within a few minutes: value = 1 MainLoop / (sum of the slice times).  Warm-up: the first
    --warmup slices of a second MainLoop on a copy of the state, untimed."""
    threads = cpu_threads()
    if rank != 0:
        return
    wl = WORKLOADS[args.workload]()
    state = synthetic_state_np() if wl.name == "heave_pitch" else None
    if state is None:
        raise SystemExit("--impl reference runs the headline workload (heave_pitch)")

    def prepared():
        sim = wl.oracle()
        sim.set_threads(threads)
        sim.set_erase_wake_after(wl.wake_rows)
        sim.begin()
        sim.set_state(wl.wake_rows, state["wing_pos"], state["wake_pos"], state["wing_gamma"],
                      state["wing_gamma_prev"], state["wake_gamma"])
        return sim

    step = wl.wake_rows + 1
    k = max(1, args.steps)
    warm = prepared()
    warm.sliced_begin(step, wl.dt, k, threads)
    for q in range(min(args.warmup, k)):
        warm.sliced_run(q, np.zeros(1 + 2 * wl.num))
    del warm
    sim = prepared()
    sim.sliced_begin(step, wl.dt, k, threads)
    row = np.zeros(1 + 2 * wl.num)
    times = []
    for q in range(k):
        t0 = time.perf_counter()
        sim.sliced_run(q, row)
        times.append(time.perf_counter() - t0)
    total = float(np.sum(times))
    value = 1.0 / total
    sample = (f"one complete FP64 MainLoop (no sampling, no scaling) at the {wl.num * wl.wake_rows * wl.cols:,}-ring "
              f"state, cut into {k} consecutive slices timed as the {k} steps (kinematics+shed, CalcMatrix rows, "
              f"CalcRhs rows, FullPivLU columns single-threaded, load lines, RK2 wake-node ranges); value = 1 "
              f"MainLoop / sum of slice times ({total:.1f} s); OpenMP {threads} threads; synthetic convected wake")
    line = {"impl": "reference", "metric": wl.metric, "value": value, "unit": "steps/s", "n_gpus": world,
            "steps": k, "warmup": args.warmup, "ms_per_step": 1e3 * total / k, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": headline_config(wl, world),
            "mainloop_s": total, "slice_s": [round(t, 3) for t in times], "load_row": [float(x) for x in row],
            "cpu_baseline": {"value": value, "unit": "steps/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def timed_steps(sim, first_step, k, flush_buf, torch, stream):
    """Per-step CUDA-event times on the library's stream, L2 flushed between."""
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(k)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(k)]
    rows = []
    with torch.cuda.stream(stream):
        for i in range(k):
            flush_buf.fill_(float(i))
            ev0[i].record(stream)
            rows.append(sim.step(first_step + i, DT))
            ev1[i].record(stream)
    torch.cuda.synchronize()
    return np.array([a.elapsed_time(b) for a, b in zip(ev0, ev1)]), rows


def run_ours(args, rank, world, local_rank):
    import torch

    import uvlm_b200 as U

    dev = local_rank
    torch.cuda.set_device(dev)
    if world > 1:
        import torch.distributed as dist

    wl = WORKLOADS[args.workload]()
    DT, WAKE_ROWS, ROWS, COLS = wl.dt, wl.wake_rows, wl.rows, wl.cols
    # --- accuracy run: both forms from step 0 to the held wake ----------------
    sim64 = wl.build("fp64", device=dev)
    simmx = make_mixed(dev, wl=wl)
    learned = simmx._cfg.warm_start == 2
    # ablation: the method without the network
    simex = make_mixed(dev, warm_start="extrapolate", wl=wl) if learned else None
    sim64.begin()
    simmx.begin()
    if simex:
        simex.begin()
    cl64, clmx = [], []
    abl = {"mlp": ([], []), "extrapolate": ([], [])}
    t0 = time.time()
    for s in range(WAKE_ROWS + 1):
        cl64.append(sim64.step(s, DT))
        clmx.append(simmx.step(s, DT))
        if simex:
            simex.step(s, DT)
        if s >= 3:
            for name, sm in (("mlp" if learned else "extrapolate", simmx), ("extrapolate", simex)):
                if sm is None:
                    continue
                st_ = sm.stats()
                abl[name][0].append(st_.initial_residual)
                abl[name][1].append(st_.gmres_iters)
    preroll_s = time.time() - t0
    warm_ablation = {k: {"initial_residual_mean": float(np.mean(v[0])), "gmres_iters_total": int(np.sum(v[1])),
                         "steps": len(v[1])} for k, v in abl.items() if v[1]}
    cl64, clmx = np.array(cl64), np.array(clmx)
    CLc, CDc = list(range(2, 1 + 2 * wl.num, 2)), list(range(1, 1 + 2 * wl.num, 2))

    def rel_err(a, b, cols, end=None):
        # max over wings of max_t |a - b| / max_t |b|
        return float(max(np.max(np.abs(a[:end, c] - b[:end, c])) / np.max(np.abs(b[:, c])) for c in cols))

    cl_err = rel_err(clmx, cl64, CLc)
    cd_err = rel_err(clmx, cl64, CDc)
    # rounding floor of the FP64 form itself: the same run with the forward
    # flight perturbed by one ulp (the wake roll-up amplifies any rounding)
    accuracy = {}
    if not args.no_floor:
        simf = wl.build("fp64", device=dev)
        simf.set_forward_flight([-(1.0 + 2.0 ** -52), 0.0, 0.0])
        simf.begin()
        clf = np.array([simf.step(s, DT) for s in range(WAKE_ROWS + 1)])
        simf.close()
        accuracy["fp64_one_ulp_cl_rel_err"] = {}
    accuracy["mixed_cl_rel_err"] = {}
    for end in sorted({e for e in (50, 100, 200, 300, 400, 600) if e < WAKE_ROWS + 1} | {WAKE_ROWS + 1}):
        accuracy["mixed_cl_rel_err"][f"steps_0_{end - 1}"] = rel_err(clmx, cl64, CLc, end)
        if not args.no_floor:
            accuracy["fp64_one_ulp_cl_rel_err"][f"steps_0_{end - 1}"] = rel_err(clf, cl64, CLc, end)

    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{dev}")
    step0 = WAKE_ROWS + 1
    # --- warm-up and timed steps ---------------------------------------------
    s_mx = torch.cuda.ExternalStream(simmx.stream(), device=dev)
    s_64 = torch.cuda.ExternalStream(sim64.stream(), device=dev)
    s_ex = torch.cuda.ExternalStream(simex.stream(), device=dev) if simex else None
    for i in range(args.warmup):
        simmx.step(step0 + i, DT)
        sim64.step(step0 + i, DT)
        if simex:
            simex.step(step0 + i, DT)
    step0 += args.warmup
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(dev)
    clocks.start()
    launches0 = U.lib().uvlm_kernel_launch_count()
    t_mx, _ = timed_steps(simmx, step0, args.steps, flush, torch, s_mx)
    launches = U.lib().uvlm_kernel_launch_count() - launches0
    clk = clocks.stop()
    t_64, _ = timed_steps(sim64, step0, args.steps, flush, torch, s_64)
    # the same steps without the network (warm start 2 g_n - g_{n-1}), timed alike
    t_ex = timed_steps(simex, step0, args.steps, flush, torch, s_ex)[0] if simex else None
    st = simmx.stats()
    total_mx = float(np.sum(t_mx))
    if world > 1:
        tt = torch.tensor([total_mx], device=f"cuda:{dev}", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total_mx = float(tt.item())
        dist.barrier()
    value = world * args.steps / (total_mx * 1e-3)
    plain = args.steps / (float(np.sum(t_64)) * 1e-3)
    step0 += args.steps

    # the warm start's own stage: the solve (with the guess) timed per step with
    # CUDA events, learned network against the extrapolation, the same steps
    warm_stage = None
    if simex:
        def solve_stage(sim):
            sim.set_stage_timing(True)
            v, it = [], []
            for i in range(args.steps):
                sim.step(step0 + i, DT)
                s_ = sim.stats()
                v.append(float(s_.stage_ms[3] + s_.stage_ms[6]))
                it.append(int(s_.gmres_iters))
            sim.set_stage_timing(False)
            return float(np.mean(v)), float(np.mean(it))
        (ms_l, it_l), (ms_e, it_e) = solve_stage(simmx), solve_stage(simex)
        warm_stage = {"learned_solve_ms": ms_l, "extrapolate_solve_ms": ms_e, "learned_gmres_iters": it_l,
                      "extrapolate_gmres_iters": it_e, "stage_speedup": ms_e / ms_l,
                      "note": "solve stage incl. the guess, CUDA events, mean over the steps after the timed ones"}
        simex.close()
        step0 += args.steps

    # --- stage timing + roofline of the N-body advection kernel --------------
    simmx.set_stage_timing(True)
    simmx.step(step0, DT)
    stmx = simmx.stats()
    simmx.set_stage_timing(False)
    step0 += 1
    stage_ms = [float(x) for x in stmx.stage_ms]
    sim64.set_stage_timing(True)
    sim64.step(step0 - 1, DT)
    st64 = sim64.stats()
    stage64 = [float(x) for x in st64.stage_ms]
    nbody_ms64 = float(st64.nbody_ms)
    pairs64 = C.c_double()
    U._capi.check(U.lib().uvlm_get_last_work(sim64._h, C.byref(pairs64), None, None))
    sim64.set_stage_timing(False)

    # roofline of the N-body kernel: the step's algorithmic pairs (RHS, loads,
    # advection) over the device time of its N-body launches (CUDA events
    # around each launch on the library's stream)
    pairs_step = C.c_double()
    U._capi.check(U.lib().uvlm_get_last_work(simmx._h, C.byref(pairs_step), None, None))
    nbody_ms = float(stmx.nbody_ms)
    achieved = FLOP_PER_PAIR * pairs_step.value / (nbody_ms * 1e-3) / 1e12
    pairs_advect = wl.advect_pairs()
    adv_ms = stage_ms[5]
    advect_stage_tflops = FLOP_PER_PAIR * pairs_advect / (adv_ms * 1e-3) / 1e12
    pk = C.c_double()
    U._capi.check(U.lib().uvlm_measure_fp32_peak(dev, C.byref(pk)))
    peak = pk.value
    pk64 = C.c_double()
    U._capi.check(U.lib().uvlm_measure_fp64_peak(dev, C.byref(pk64)))
    achieved64 = FLOP_PER_PAIR * pairs64.value / (nbody_ms64 * 1e-3) / 1e12
    # assembly (CalcMatrix): N collocation points x the wing lattices' unique
    # segments, 59 FLOP each, over the stage's device time; the mixed form
    # assembles its residual matrix in FP64 every step (the FP32 matrix only
    # when it factors), so the FP64 probe is the denominator
    n_panels = wl.num * ROWS * COLS
    asm_pairs = n_panels * wl.num * ((ROWS + 1) * COLS + ROWS * (COLS + 1))
    asm_tflops = FLOP_PER_PAIR * asm_pairs / (stage_ms[1] * 1e-3) / 1e12

    # --- end-to-end through the C-ABI with host buffers ------------------------
    e2e_t = []
    gam = np.zeros((wl.num, ROWS, COLS))
    for i in range(args.steps):
        t1 = time.perf_counter()
        simmx.step(step0 + i, DT)
        U.lib().uvlm_get_state(simmx._h, None, None, None, gam.ctypes.data_as(C.POINTER(C.c_double)), None, None)
        e2e_t.append(time.perf_counter() - t1)
    step0 += args.steps
    e2e_value = world * args.steps / float(np.sum(e2e_t))

    # --- the fine-grained drop-in: advect::Advection::Advect with host sheets ----
    # (the call a reference caller swaps first), at the held wake, mixed form:
    # every call copies the wing and wake sheets in and the advected wake out
    st_adv = simmx.state()
    adv = U.AdvectFactory(wl.advection, precision="mixed")
    nxt = np.empty_like(st_adv["wake_pos"])
    ff = np.array([-1.0, 0.0, 0.0])
    for _ in range(2):
        adv.Advect(st_adv["wing_pos"], st_adv["wing_gamma"], st_adv["wake_pos"], st_adv["wake_gamma"], ff, DT, nxt)
    adv_t = []
    for _ in range(args.steps):
        t1 = time.perf_counter()
        adv.Advect(st_adv["wing_pos"], st_adv["wing_gamma"], st_adv["wake_pos"], st_adv["wake_gamma"], ff, DT, nxt)
        adv_t.append(time.perf_counter() - t1)
    del adv
    adv_in = sum(st_adv[k].nbytes for k in ("wing_pos", "wing_gamma", "wake_pos", "wake_gamma"))
    e2e_advect = {"value": args.steps / float(np.sum(adv_t)), "unit": "Advect calls/s",
                  "h2d_bytes_per_step": int(adv_in), "d2h_bytes_per_step": int(nxt.nbytes),
                  "note": f"advect::Advection::Advect ({wl.advection}, mixed form) through uvlm_advection_advect "
                          f"with host MultipleSheet arrays at the held wake, wall clock per call"}

    # --- CPU baseline (rank 0 only) --------------------------------------------
    cpu = None
    if rank == 0 and not args.no_cpu:
        state = simmx.state()
        threads = cpu_threads()
        stride, lu_n = CPU_STRIDE, CPU_LU_N
        tcpu, secs = oracle_sample(wl, state, stride, lu_n, threads)
        n_panels = wl.num * ROWS * COLS
        cpu = {"value": 1.0 / tcpu, "unit": "steps/s", "cores": threads, "kind": "port",
               "sample": (f"FP64 CPU oracle, one MainLoop at the {wl.num * WAKE_ROWS * COLS:,}-ring state: N-body "
                          f"stages on every {stride}th target scaled x{stride}, FullPivLU on the leading {lu_n}^2 "
                          f"block scaled by ({n_panels}/{lu_n})^3; stage seconds "
                          f"{[round(float(x), 3) for x in secs]}")}

    if rank == 0:
        line = {
            "metric": wl.metric, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_mx / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": headline_config(wl, world),
            "plain_fp64_steps_per_s": plain, "speedup_vs_plain_fp64": value / world / plain,
            "mixed_extrapolate_steps_per_s": (args.steps / (float(np.sum(t_ex)) * 1e-3)) if t_ex is not None else None,
            "learned_warm_start_speedup": ((value / world) / (args.steps / (float(np.sum(t_ex)) * 1e-3))
                                           if t_ex is not None else None),
            "learned_warm_start_solve_stage": warm_stage,
            "cl_rel_err": cl_err, "cd_rel_err": cd_err,
            "cl_err_reference": f"plain FP64 GPU form, same {WAKE_ROWS} steps",
            "accuracy": accuracy, "warm_start_ablation": warm_ablation,
            "gmres_iters_last": int(st.gmres_iters), "solve_path_last": int(st.solve_path),
            "nbody_variant": U.lib().uvlm_nbody_variant_name(int(st.nbody_variant)).decode(),
            "plain_fp64_nbody_variant": U.lib().uvlm_nbody_variant_name(int(st64.nbody_variant)).decode(),
            "nbody_stage_variants": stage_variant_names(st),
            "plain_fp64_nbody_stage_variants": stage_variant_names(st64),
            "stage_ms": {"kin_shed": stage_ms[0], "assembly": stage_ms[1], "rhs": stage_ms[2], "solve": stage_ms[3],
                         "loads": stage_ms[4], "advect": stage_ms[5], "total": stage_ms[7]},
            "plain_fp64_stage_ms": {"kin_shed": stage64[0], "assembly": stage64[1], "rhs": stage64[2],
                                    "solve": stage64[3], "loads": stage64[4], "advect": stage64[5],
                                    "total": stage64[7]},
            "roofline": {"bound": "fp32_simt", "kernel": "nbody_kernel (every N-body launch of a step: RHS, "
                                                              f"loads, {wl.advection} advection)",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         "peak_source": "FP32 FMA probe on this GPU, the larger of scalar FFMA and packed FP32x2 "
                                        "(uvlm_measure_fp32_peak)",
                         "per_unit": f"{FLOP_PER_PAIR} FLOP per (target, unique segment) pair",
                         "units_per_step": pairs_step.value, "nbody_ms_per_step": nbody_ms,
                         "advect_stage_tflops": advect_stage_tflops, "advect_pairs_per_step": pairs_advect,
                         "traffic": NBODY_TRAFFIC.get(wl.name),
                         "traffic_unit": "DRAM bytes per advection launch (ncu dram__bytes_read.sum + "
                                         "dram__bytes_write.sum, one launch at the held wake)"},
            "plain_fp64_roofline": {"bound": "fp64_simt", "kernel": "nbody_kernel<double> (every N-body launch "
                                                                     "of a plain FP64 step)",
                                    "achieved": achieved64, "peak": pk64.value, "unit": "TFLOP/s",
                                    "frac": achieved64 / pk64.value,
                                    "peak_source": "FP64 FMA probe on this GPU (uvlm_measure_fp64_peak)",
                                    "units_per_step": pairs64.value, "nbody_ms_per_step": nbody_ms64},
            "assembly_roofline": {"bound": "fp64_simt", "kernel": "assemble_kernel<double> (the FP64 residual "
                                                                   "matrix, every step)",
                                  "achieved": asm_tflops, "peak": pk64.value, "unit": "TFLOP/s",
                                  "frac": asm_tflops / pk64.value,
                                  "per_unit": f"{FLOP_PER_PAIR} FLOP per (collocation point, unique wing segment) pair",
                                  "units_per_step": asm_pairs, "stage_ms": stage_ms[1],
                                  "note": "each unique segment once per collocation point (a ring's 4 "
                                          "segments combined from its own and its neighbours'); the FP64 "
                                          "reciprocal square roots and divides are instruction sequences"},
            "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 8 * (1 + 2 * wl.num + wl.num * ROWS * COLS),
                    "note": "wall clock per uvlm_step + circulation download; per-step inputs are scalars"},
            "e2e_advect": e2e_advect,
            "gpu_launches": int(launches), "clocks": clk, "preroll_s": preroll_s,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    sim64.close()
    simmx.close()


def run_batch(args, rank=0, world=1, local_rank=0):
    """The 256-case seeded flapping-wing sweep (chordwise 4-16, spanwise 8-64,
    AR 2-10, k 0.1-1, heave 0.05-0.3 c, pitch 0-20 deg, 150 Euler steps per
    case) in one batch: aggregate case-steps/s over steps 1..149, device-timed
    on the batch's stream; the FP64 batch beside it and the CL error of the
    mixed batch against it.  Under torchrun the cases are split over the ranks
    by their N-body work (shard_cases; no data moves while stepping) and the
    time is the maximum over ranks."""
    import torch

    import uvlm_b200 as U
    from uvlm_b200.batch import case_cost, draw_cases, gather_case_rows, make_batch, shard_cases

    all_cases = draw_cases(256, seed=0)
    steps = 150
    mine = shard_cases([case_cost(d, steps) for d in all_cases], world)[rank]
    cases = [all_cases[i] for i in mine]
    torch.cuda.set_device(local_rank)
    warm = make_batch(cases, precision="mixed", max_steps=args.warmup + 1)
    warm.run(args.warmup + 1)  # module load, graph capture, first launches
    warm.close()
    out = {}
    for prec in ("mixed", "fp64"):
        sim = make_batch(cases, precision=prec, max_steps=steps)
        sim.run(1)
        stream = torch.cuda.ExternalStream(sim.stream(), device=local_rank)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
        clocks = Clocks(local_rank) if prec == "mixed" else None
        if clocks:
            clocks.start()
        l0 = U.lib().uvlm_kernel_launch_count()
        e0.record(stream)
        sim.run(steps - 1)
        e1.record(stream)
        torch.cuda.synchronize()
        launches = U.lib().uvlm_kernel_launch_count() - l0
        clk = clocks.stop() if clocks else None
        ms = e0.elapsed_time(e1)
        if world > 1:
            import torch.distributed as dist

            t = torch.tensor([ms], device=f"cuda:{local_rank}", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        dist_mod = None
        if world > 1:
            import torch.distributed as dist_mod
        # every rank's per-case load rows, gathered into case order (no data moves while stepping)
        loads_all = gather_case_rows(sim.loads(), mine, len(all_cases), dist_mod)
        out[prec] = dict(ms=ms, loads=loads_all, launches=launches, per_step=sim.launches_per_step(), clocks=clk,
                         res=sim.solve_stats()[1], factorizations=sim.factorizations())
        sim.close()
    if rank != 0:
        return
    L, L64 = out["mixed"]["loads"], out["fp64"]["loads"]
    cl_err = float(np.max(np.abs(L[:, :, 2] - L64[:, :, 2]).max(axis=0) / np.abs(L64[:, :, 2]).max(axis=0)))
    value = 256 * (steps - 1) / (out["mixed"]["ms"] * 1e-3)
    line = {"metric": "case-steps/s (256 seeded flapping-wing cases x 150 steps, batched, mixed)", "value": value,
            "unit": "case-steps/s", "n_gpus": world, "steps": steps - 1, "warmup": args.warmup,
            "ms_per_step": out["mixed"]["ms"] / (steps - 1), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": "batch256: seed 0 draws, rows U{4..16}, even cols U{8..64}, AR U[2,10], "
                                   "k U[0.1,1], heave U[0.05,0.3] c, pitch U[0,20] deg, phase 90 deg, Euler, "
                                   "150 MainLoops each, all cases in one graph-replayed step",
                       "panels_total": int(sum(d["rows"] * d["cols"] for d in all_cases)),
                       "parallelism": f"cases sharded over {world} GPU(s) by N-body work",
                       "form": "FP32 N-body, per-case FP32 LU (refactored only when refinement from the "
                               "previous step's factors stalls) + FP64 refinement (residual <= 1e-12)"},
            "plain_fp64_case_steps_per_s": 256 * (steps - 1) / (out["fp64"]["ms"] * 1e-3),
            "cl_rel_err_max_over_cases": cl_err, "cl_err_scope": f"all {len(all_cases)} cases, gathered from "
                                                                  f"{world} rank(s)",
            "refinement_residual_max": float(np.max(out["mixed"]["res"])),
            "factorizations": {"mixed": out["mixed"]["factorizations"], "fp64": out["fp64"]["factorizations"],
                               "case_steps": 256 * steps},
            "gpu_launches": int(out["mixed"]["launches"]), "launches_per_step": int(out["mixed"]["per_step"]),
            "clocks": out["mixed"]["clocks"], "cpu_baseline": None}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-floor", action="store_true", help="skip the one-ulp FP64 rounding-floor run")
    ap.add_argument("--profile", action="store_true", help="one form on a synthesized state, for ncu")
    ap.add_argument("--form", default="mixed", choices=["mixed", "fp64"], help="form run by --profile")
    ap.add_argument("--variant", default=None, help="N-body tile pinned by --profile (default: the form's default)")
    ap.add_argument("--profile-step0", action="store_true",
                    help="with --profile: only step 0 of the mixed form (first factorisation and inverse)")
    ap.add_argument("--workload", default="heave_pitch", choices=list(WORKLOADS) + ["batch256"],
                    help="heave_pitch (the metric's configuration, default), tandem4, morphing, batch256")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.profile:
        run_profile(args)
        return
    if args.workload == "batch256":
        if world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            torch.cuda.set_device(local_rank)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        try:
            run_batch(args, rank, world, local_rank)
        finally:
            if world > 1:
                import torch.distributed as dist

                dist.destroy_process_group()
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
