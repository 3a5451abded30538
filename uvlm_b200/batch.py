"""Batched independent wing cases on one GPU (the uvlm_batch_* C-ABI).

The reference steps one ``SimpleSimulator`` per process
(src/simulator/simple_simulator.cpp:240-313).  ``BatchSimulator`` advances
many single-wing cases together: every MainLoop stage is one launch over all
cases and one step is replayed from a CUDA graph.  Each case keeps the
reference's semantics (lattice, Morphing kinematics, shed, matrix, RHS, solve,
Joukowski loads, Euler or RK2 roll-up); cases do not interact.

``draw_cases`` makes the seeded flapping-wing sweep (chordwise panels 4-16,
spanwise 8-64 even, aspect ratio 2-10, reduced frequency 0.1-1, heave
0.05-0.3 chords, pitch 0-20 deg, phase 90 deg) and ``shard_cases`` splits
cases over ranks by their N-body work.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._capi import BatchCase, BatchConfig, check, lib
from . import Morphing, RectGenerator

ADVECTION = {"euler": 0, "RK2": 1}
PRECISION = {"fp64": 0, "mixed": 1}


class BatchError(RuntimeError):
    pass


def _check(code, h):
    if code != 0:
        msg = lib().uvlm_batch_last_error(h) if h else lib().uvlm_global_last_error()
        raise BatchError(f"status {code}: {(msg or b'').decode()}")


class BatchSimulator:
    """Many independent single-wing UVLM cases stepped together."""

    def __init__(self, precision: str = "mixed", advection: str = "euler", max_steps: int = 151, device: int = 0,
                 use_graph: bool = True, refine_tol: float = 1e-12, refine_max_iter: int = 10,
                 rk_ignore_rows: int = 5, stale_factors: bool = True, nbody_tile: int = -1):
        cfg = BatchConfig()
        check(lib().uvlm_batch_config_default(C.byref(cfg)))
        cfg.precision = PRECISION[precision]
        cfg.advection = ADVECTION[advection]
        cfg.max_steps = int(max_steps)
        cfg.device = int(device)
        cfg.use_graph = int(bool(use_graph))
        cfg.refine_tol = float(refine_tol)
        cfg.refine_max_iter = int(refine_max_iter)
        cfg.rk_ignore_rows = int(rk_ignore_rows)
        cfg.stale_factors = int(bool(stale_factors))
        cfg.nbody_tile = int(nbody_tile)  # -1: the tile autotuner chooses at creation
        self._cfg = cfg
        self._cases = []
        self._h = None

    def add_case(self, morphing: Morphing, chord: float, span: float, rows: int, cols: int, dt: float,
                 forward_flight=(-1.0, 0.0, 0.0), origin=(0.0, 0.0, 0.0), generator: RectGenerator | None = None):
        if self._h is not None:
            raise BatchError("cases are added before begin()")
        b = BatchCase()
        b.chord, b.span, b.rows, b.cols, b.dt = float(chord), float(span), int(rows), int(cols), float(dt)
        for d in range(3):
            b.origin[d] = float(origin[d])
            b.forward_flight[d] = float(forward_flight[d])
        b.kin = morphing.k
        gen = generator or RectGenerator()
        b.chebyshev_chord, b.chebyshev_span = int(gen.chebyshev_chord), int(gen.chebyshev_span)
        self._cases.append(b)
        return len(self._cases) - 1

    @property
    def n_cases(self) -> int:
        return len(self._cases)

    def begin(self) -> None:
        arr = (BatchCase * len(self._cases))(*self._cases)
        h = C.c_void_p()
        _check(lib().uvlm_batch_create(C.byref(self._cfg), arr, len(self._cases), C.byref(h)), None)
        self._h = h

    def run(self, n_steps: int) -> None:
        """n_steps more MainLoops of every case."""
        if self._h is None:
            self.begin()
        _check(lib().uvlm_batch_run(self._h, int(n_steps)), self._h)

    def Run(self, steps: int) -> None:  # noqa: N802
        """SimpleSimulator::Run convention: MainLoop(step) for step = 0..steps."""
        self.run(steps + 1)

    def steps_done(self) -> int:
        v = C.c_int64()
        _check(lib().uvlm_batch_steps_done(self._h, C.byref(v)), self._h)
        return v.value

    def nbody_tile(self) -> str:
        """Name of the N-body tile the batch runs (autotuned or pinned)."""
        if self._h is None:
            self.begin()
        return lib().uvlm_batch_nbody_tile_name(self._h).decode()

    def loads(self) -> np.ndarray:
        """[steps_done][n_cases][3] = (t, CD, CL)."""
        out = np.zeros((self.steps_done(), self.n_cases, 3))
        if out.size:
            _check(lib().uvlm_batch_get_loads(self._h, out.ctypes.data_as(C.POINTER(C.c_double))), self._h)
        return out

    def case_state(self, c: int) -> dict:
        b = self._cases[c]
        R, Cc = int(b.rows), int(b.cols)
        rows = max(self.steps_done() - 1, 0)
        s = dict(wing_pos=np.zeros((R + 1, Cc + 1, 3)), wing_gamma=np.zeros((R, Cc)),
                 wake_pos=np.zeros((rows + 1, Cc + 1, 3)), wake_gamma=np.zeros((rows, Cc)))
        wr = C.c_int64()
        P = C.POINTER(C.c_double)
        _check(lib().uvlm_batch_get_case(self._h, int(c), s["wing_pos"].ctypes.data_as(P),
                                         s["wing_gamma"].ctypes.data_as(P), s["wake_pos"].ctypes.data_as(P),
                                         s["wake_gamma"].ctypes.data_as(P), C.byref(wr)), self._h)
        return s

    def solve_stats(self):
        sw = np.zeros(self.n_cases, np.int32)
        res = np.zeros(self.n_cases)
        _check(lib().uvlm_batch_get_solve_stats(self._h, sw.ctypes.data_as(C.POINTER(C.c_int32)),
                                                res.ctypes.data_as(C.POINTER(C.c_double))), self._h)
        return sw, res

    def factorizations(self) -> int:
        """Per-case LU factorisations so far."""
        v = C.c_int64()
        _check(lib().uvlm_batch_factorizations(self._h, C.byref(v)), self._h)
        return v.value

    def launches_per_step(self) -> int:
        v = C.c_int64()
        _check(lib().uvlm_batch_launches_per_step(self._h, C.byref(v)), self._h)
        return v.value

    def stream(self) -> int:
        """The batch's cudaStream_t as an integer handle."""
        return lib().uvlm_batch_stream(self._h)

    def close(self) -> None:
        if self._h is not None:
            lib().uvlm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def draw_cases(n: int = 256, seed: int = 0) -> list[dict]:
    """Seeded flapping-wing sweep: chord 1, U = 1, rows U{4..16}, even cols
    U{8..64}, aspect ratio U[2,10], k U[0.1,1] (w = 2 U k / c), heave
    U[0.05,0.3] c, pitch U[0,20] deg with 90 deg phase, dt = 2 pi / w / 40."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        rows = int(rng.integers(4, 17))
        cols = 2 * int(rng.integers(4, 33))
        ar = float(rng.uniform(2, 10))
        k = float(rng.uniform(0.1, 1.0))
        heave = float(rng.uniform(0.05, 0.3))
        pitch = float(rng.uniform(0, 20))
        w = 2 * k
        out.append(dict(rows=rows, cols=cols, chord=1.0, span=ar, k=k, omega=w, heave=heave, pitch_deg=pitch,
                        dt=2 * math.pi / w / 40))
    return out


def case_morphing(d: dict) -> Morphing:
    return Morphing().set_plug(d["heave"], d["omega"]).set_twist(math.radians(d["pitch_deg"]), d["omega"],
                                                                  math.pi / 2)


def case_cost(d: dict, steps: int) -> float:
    """N-body pairs of the last step (targets x unique segments), the
    dominant work of a case."""
    R, Cc = d["rows"], d["cols"]
    segs = (R + 1) * Cc + R * (Cc + 1) + (steps + 1) * Cc + steps * (Cc + 1)
    return float((steps * (Cc + 1) + R * (2 * Cc + 1)) * segs)


def shard_cases(costs, world: int) -> list[list[int]]:
    """Longest-processing-time split of cases over `world` ranks: cases in
    decreasing cost, each to the least-loaded rank.  No data moves between
    ranks while stepping; rank r runs the cases in element r."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def gather_case_rows(rows, mine, n_cases: int, dist=None):
    """Per-case result rows of every rank in case order.  rows: [steps][len(mine)][...] of this rank's
    cases `mine` (from shard_cases); returns [steps][n_cases][...] on every rank (the all-gather of
    torch.distributed when `dist` is given and initialised, else this rank's rows alone must cover
    every case)."""
    rows = np.asarray(rows)
    parts = [(list(mine), rows)]
    if dist is not None and dist.is_initialized() and dist.get_world_size() > 1:
        got = [None] * dist.get_world_size()
        dist.all_gather_object(got, (list(mine), rows))
        parts = got
    out = np.zeros((rows.shape[0], n_cases) + rows.shape[2:], dtype=rows.dtype)
    seen = np.zeros(n_cases, dtype=bool)
    for idx, r in parts:
        out[:, idx] = r
        seen[idx] = True
    if not seen.all():
        raise ValueError("the gathered shards do not cover every case")
    return out


def make_batch(cases: list[dict], precision: str = "mixed", advection: str = "euler", max_steps: int = 151,
               device: int = 0, use_graph: bool = True, stale_factors: bool = True,
               nbody_tile: int = -1) -> BatchSimulator:
    sim = BatchSimulator(precision=precision, advection=advection, max_steps=max_steps, device=device,
                         use_graph=use_graph, stale_factors=stale_factors, nbody_tile=nbody_tile)
    for d in cases:
        sim.add_case(case_morphing(d), d["chord"], d["span"], d["rows"], d["cols"], d["dt"])
    return sim
