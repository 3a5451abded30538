"""uvlm_b200 -- B200-native UVLM time-stepper behind xeno14/UVLM's interface.

The Python classes mirror the reference's C++ API for the per-step hot path
(names, argument meaning and error behaviour):

  SimpleSimulator  src/simulator/simple_simulator.h:36-108
  Morphing         src/morphing.h:25-108 (closed-form sinusoids instead of
                   std::function; see ``Morphing``)
  RectGenerator, NACA4digitGenerator, NACA00XXGenerator, WholeWing
                   src/wing/* (host-side lattice generators, uvlm_b200.wing)
  AdvectFactory    src/advect_factory.cpp:43-60 -> ``Advection`` objects
                   whose ``Advect`` matches src/advect.h:48-59
  InducedVelocity  src/velocity.h:14-24
  rings.*          the legacy AoS API of src/shed.h and src/linear.h

Every call goes through the C-ABI of include/uvlm_b200.h into the CUDA
library built in-tree for sm_100a; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._capi import (ADVECT, LU_PREC, PRECISION, SOLVER, WARM, Config, Kinematics, StepStats, UVLMError, WingDesc,
                    check, lib)
from .wing import NACA00XXGenerator, NACA4digitGenerator, RectGenerator, WholeWing, WingGenerator

__all__ = ["SimpleSimulator", "Morphing", "WingGenerator", "RectGenerator", "NACA4digitGenerator",
           "NACA00XXGenerator", "WholeWing", "AdvectFactory", "Advection", "InducedVelocity", "UVLMError",
           "dense_solve", "rings", "lib"]

_P = C.POINTER(C.c_double)


def _p(a):
    return None if a is None else a.ctypes.data_as(_P)


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


@dataclass
class Sinusoid:
    """f(t) = amp * sin(omega * t + phase)."""

    amp: float = 0.0
    omega: float = 0.0
    phase: float = 0.0


class Morphing:
    """Wing kinematics (src/morphing.h:25-108).

    The reference takes arbitrary std::function objects; here each motion is a
    closed-form sinusoid so that it can be evaluated on the device:
      plug(t)     = A sin(w t + p)                          set_plug
      flap(t)     = A sin(w t + p)                          set_flap
      twist(x0,t) = (A + slope*|y|) sin(w t + p)            set_twist
      bend(x0,t)  = (cx x(1-x) + cy y^2) sin(w t + p)       set_bend
    The velocity is the reference's FP64 central difference (h = 1e-6).
    """

    def __init__(self):
        self.k = Kinematics()

    def set_alpha(self, alpha: float) -> "Morphing":
        self.k.alpha = float(alpha)
        return self

    def set_plug(self, amp: float, omega: float, phase: float = 0.0) -> "Morphing":
        self.k.plug_amp, self.k.plug_omega, self.k.plug_phase = float(amp), float(omega), float(phase)
        return self

    def set_flap(self, amp: float, omega: float, phase: float = 0.0) -> "Morphing":
        self.k.flap_amp, self.k.flap_omega, self.k.flap_phase = float(amp), float(omega), float(phase)
        return self

    def set_twist(self, amp: float, omega: float, phase: float = 0.0, span_slope: float = 0.0) -> "Morphing":
        self.k.twist_amp, self.k.twist_omega, self.k.twist_phase = float(amp), float(omega), float(phase)
        self.k.twist_span_slope = float(span_slope)
        return self

    def set_bend(self, cx: float, cy: float, omega: float, phase: float = 0.0) -> "Morphing":
        self.k.bend_cx, self.k.bend_cy = float(cx), float(cy)
        self.k.bend_omega, self.k.bend_phase = float(omega), float(phase)
        return self

    def set_origin(self, origin) -> None:
        for i in range(3):
            self.k.origin[i] = float(origin[i])

    def Perfome(self, x0, t: float) -> np.ndarray:  # noqa: N802 (reference name)
        """Morphing::Perfome (src/morphing.cpp:23-43) of reference point(s) x0 ((3,) or (n, 3)), on the GPU."""
        return self._eval(lib().uvlm_kinematics_perfome, x0, t)

    def Velocity(self, x0, t: float) -> np.ndarray:  # noqa: N802 (reference name)
        """Morphing::Velocity (src/morphing.cpp:45-52) of reference point(s) x0, on the GPU."""
        return self._eval(lib().uvlm_kinematics_velocity, x0, t)

    def _eval(self, fn, x0, t):
        x = _f64(x0)
        single = x.ndim == 1
        x = np.ascontiguousarray(x.reshape(-1, 3))
        out = np.zeros_like(x)
        check(fn(C.byref(self.k), _p(x), x.shape[0], float(t), _p(out)))
        return out[0] if single else out

    def Clear(self) -> None:  # noqa: N802 (reference name)
        alpha = self.k.alpha
        origin = tuple(self.k.origin)
        self.k = Kinematics()
        self.k.alpha = alpha
        self.set_origin(origin)


class SimpleSimulator:
    """The UVLM time-stepper (src/simulator/simple_simulator.{h,cpp}) on a B200.

    Extra keyword arguments select the B200 arithmetic:
      precision   "fp64" (plain form) or "mixed" (FP32 N-body/assembly,
                  tensor-core LU, FP64 residuals)
      solver      "lu" (factor every step) or "gmres_stale" (GMRES
                  preconditioned by stale LU factors, fresh-LU fallback)
      warm_start  "previous", "extrapolate" or "mlp"
      preconditioner  "inverse" (dense (LU)^-1 of the stale factors, one
                  matrix-vector product per GMRES iteration) or "triangular"
                  (forward/backward solves with the factors)
      fp64_stages mixed form: N-body stages evaluated in FP64, any of
                  "rhs", "loads", "advect"
      near_fp64   mixed form: the near-field pairs of the FP32 N-body stages
                  in FP64 (FP64 records, FP64 accumulation): True for every
                  stage, or any of "rhs", "loads", "advect"; None (default)
                  takes the library's default, the RHS stage
      lu_pivoting mixed form, the preconditioner's factors: "panel" (pivots
                  over every row of each 64-column panel) or "local" (over
                  the panel's top 256 rows); None takes the library's default
      gmres_refresh_iter  mixed form: refactor the preconditioner after a step
                  whose GMRES took at least this many iterations (0: only on
                  the fallback); None takes the library's default (16)
    """

    def __init__(self, precision: str = "fp64", solver: str | None = None, warm_start: str = "previous",
                 lu_precision: str = "tf32", max_wake_rows: int = 1024, erase_wake_after: int = 0,
                 gmres_tol: float = 1e-12, gmres_max_iter: int = 20, gmres_restart: int = 20, device: int = 0,
                 assembly_fp64: bool | None = None, nbody_variant: int = -1, compute_loads: bool = True,
                 preconditioner: str = "inverse", fp64_stages=(), near_fp64=None, lu_pivoting: str | None = None,
                 gmres_refresh_iter: int | None = None):
        cfg = Config()
        lib().uvlm_config_default(C.byref(cfg))
        cfg.precision = PRECISION[precision]
        if solver is None:
            solver = "lu" if precision == "fp64" else "gmres_stale"
        cfg.solver = SOLVER[solver]
        cfg.warm_start = WARM[warm_start]
        cfg.lu_precision = LU_PREC[lu_precision]
        cfg.max_wake_rows = int(max_wake_rows)
        cfg.erase_wake_after = int(erase_wake_after)
        cfg.gmres_tol = float(gmres_tol)
        cfg.gmres_max_iter = int(gmres_max_iter)
        cfg.gmres_restart = int(gmres_restart)
        cfg.device = int(device)
        # the mixed form forms its FP64 residual matrix in FP64 unless told otherwise
        cfg.assembly_fp64 = int(precision == "mixed" if assembly_fp64 is None else bool(assembly_fp64))
        cfg.nbody_variant = int(nbody_variant)
        cfg.compute_loads = int(bool(compute_loads))
        cfg.preconditioner = {"inverse": 0, "triangular": 1}[preconditioner]
        cfg.nbody_fp64_stages = sum({"rhs": 1, "loads": 2, "advect": 4}[s] for s in set(fp64_stages))
        stages = {"rhs": 1, "loads": 2, "advect": 4}
        if near_fp64 is True:
            near_fp64 = tuple(stages)
        if near_fp64 is not None:
            cfg.nbody_near_fp64 = sum(stages[s] for s in set(near_fp64 or ()))
        if lu_pivoting is not None:
            cfg.lu_pivoting = {"panel": 0, "local": 1}[lu_pivoting]
        if gmres_refresh_iter is not None:
            cfg.gmres_refresh_iter = int(gmres_refresh_iter)
        self._cfg = cfg
        h = C.c_void_p()
        check(lib().uvlm_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self._num = 0
        self._wings = []
        self._load_path = None
        self._built = False

    # -- reference API ------------------------------------------------------
    def AddWing(self, generator: WingGenerator, morphing: Morphing, chord: float, span: float, rows: int,  # noqa: N802
                cols: int, origin=(0.0, 0.0, 0.0)) -> None:
        """SimpleSimulator::AddWing (simple_simulator.cpp:126-140, BuildWing :142-169) with any
        WingGenerator: the half wing (chord, span/2, rows, cols/2) from the generator, mirrored by
        WholeWing, moved to `origin`.  A plain RectGenerator wing is generated by the library itself."""
        gen = generator or RectGenerator()
        if int(cols) % 2:
            raise UVLMError(1, "columns must be even.")
        if type(gen) is RectGenerator:
            w = WingDesc()
            w.chord, w.span, w.rows, w.cols = float(chord), float(span), int(rows), int(cols)
            for i in range(3):
                w.origin[i] = float(origin[i])
            w.chebyshev_chord, w.chebyshev_span = int(gen.chebyshev_chord), int(gen.chebyshev_span)
            check(lib().uvlm_add_wing(self._h, C.byref(w), C.byref(morphing.k)), self._h)
        else:
            nodes = _f64(WholeWing(gen.Generate(float(chord), float(span) / 2, int(rows), int(cols) // 2)))
            check(lib().uvlm_add_wing_nodes(self._h, int(rows), int(cols), _p(nodes), float(chord), float(span),
                                            _p(_f64(origin)), C.byref(morphing.k)), self._h)
        self._num += 1
        self._wings.append((chord, span, rows, cols))

    add_wing = AddWing

    def set_forward_flight(self, v) -> None:
        check(lib().uvlm_set_forward_flight(self._h, _p(_f64(v))), self._h)

    def set_advection(self, advection) -> None:
        name = advection.name if isinstance(advection, Advection) else str(advection)
        check(lib().uvlm_set_advection(self._h, name.encode()), self._h)

    def set_load_path(self, path: str) -> None:
        self._load_path = path or None

    def set_sheet_path(self, path: str) -> None:
        """SimpleSimulator::set_sheet_path (simple_simulator.cpp:61-66): an AllVortexSheets record per step
        (read them with uvlm_b200.output.read_sheets)."""
        self._sheet_path = path or None
        self._set_output()

    def set_result_path(self, path: str) -> None:
        """SimpleSimulator::set_result_path (simple_simulator.cpp:53-59): a Snapshot2 record per step."""
        self._result_path = path or None
        self._set_output()

    def _set_output(self) -> None:
        enc = [p.encode() if p else None for p in (getattr(self, "_sheet_path", None),
                                                     getattr(self, "_result_path", None))]
        check(lib().uvlm_set_output_paths(self._h, enc[0], enc[1]), self._h)

    def flush_output(self) -> None:
        """Wait until every record of the steps run so far is written."""
        check(lib().uvlm_flush_output(self._h), self._h)

    def Run(self, steps: int, dt: float) -> np.ndarray:  # noqa: N802
        """Run(steps, dt): steps+1 MainLoops; returns the load rows."""
        self.begin()
        rows = np.zeros((steps + 1, 1 + 2 * self._num))
        for s in range(steps + 1):
            rows[s] = self.step(s, dt)
        if self._load_path:
            self._write_loads(rows)
        return rows

    run = Run

    # -- stepping and state -------------------------------------------------
    def begin(self) -> None:
        check(lib().uvlm_begin(self._h), self._h)
        self._built = True

    def step(self, step: int, dt: float) -> np.ndarray:
        row = np.zeros(1 + 2 * self._num)
        check(lib().uvlm_step(self._h, int(step), float(dt), _p(row)), self._h)
        return row

    # MainLoop in its six stages (uvlm_stage_*): step() is exactly these calls in this order
    def stage_kinematics(self, step: int, dt: float) -> None:
        """Morphing of every wing, Shed(step), collocation points and normals (simple_simulator.cpp:241-262)."""
        check(lib().uvlm_stage_kinematics(self._h, int(step), float(dt)), self._h)

    def stage_assemble(self) -> None:
        """CalcMatrix (simple_simulator.cpp:76-101)."""
        check(lib().uvlm_stage_assemble(self._h), self._h)

    def stage_rhs(self) -> None:
        """CalcRhs (simple_simulator.cpp:103-124)."""
        check(lib().uvlm_stage_rhs(self._h), self._h)

    def stage_solve(self) -> None:
        """The circulation solve (simple_simulator.cpp:264-268) and the per-step state output."""
        check(lib().uvlm_stage_solve(self._h), self._h)

    def stage_loads(self) -> None:
        """CalcLoad (simple_simulator.cpp:195-233)."""
        check(lib().uvlm_stage_loads(self._h), self._h)

    def stage_advect(self) -> np.ndarray:
        """Advect(dt) (simple_simulator.cpp:284), the optional erase, and the step's load row."""
        row = np.zeros(1 + 2 * self._num)
        check(lib().uvlm_stage_advect(self._h, _p(row)), self._h)
        return row

    def erase_oldest_wake(self) -> None:
        check(lib().uvlm_erase_oldest_wake(self._h), self._h)

    def sizes(self):
        v = [C.c_int64() for _ in range(5)]
        check(lib().uvlm_get_sizes(self._h, *[C.byref(x) for x in v]), self._h)
        return tuple(x.value for x in v)

    def state(self) -> dict:
        num, rows, cols, wr, wn = self.sizes()
        s = dict(wing_pos=np.zeros((num, rows + 1, cols + 1, 3)), wing_pos_init=np.zeros((num, rows + 1, cols + 1, 3)),
                 wake_pos=np.zeros((num, wn, cols + 1, 3)), wing_gamma=np.zeros((num, rows, cols)),
                 wing_gamma_prev=np.zeros((num, rows, cols)), wake_gamma=np.zeros((num, wr, cols)))
        check(lib().uvlm_get_state(self._h, _p(s["wing_pos"]), _p(s["wing_pos_init"]), _p(s["wake_pos"]),
                                   _p(s["wing_gamma"]), _p(s["wing_gamma_prev"]), _p(s["wake_gamma"])), self._h)
        return s

    def set_state(self, wake_rows, wing_pos, wake_pos, wing_gamma, wing_gamma_prev, wake_gamma) -> None:
        check(lib().uvlm_set_state(self._h, int(wake_rows), _p(_f64(wing_pos)), _p(_f64(wake_pos)),
                                   _p(_f64(wing_gamma)), _p(_f64(wing_gamma_prev)), _p(_f64(wake_gamma))), self._h)

    def stats(self) -> StepStats:
        s = StepStats()
        check(lib().uvlm_get_last_stats(self._h, C.byref(s)), self._h)
        return s

    def last_work(self):
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        check(lib().uvlm_get_last_work(self._h, C.byref(a), C.byref(b), C.byref(c)), self._h)
        return a.value, b.value, c.value

    def Velocity(self, x, include_freestream: bool = True) -> np.ndarray:  # noqa: N802
        """SimpleSimulator::Velocity (simple_simulator.h:98-100) at points x
        ((3,) or (T, 3)) for the current state: -ff + U_bound + U_wake."""
        xs = _f64(x)
        single = xs.ndim == 1
        xs = np.ascontiguousarray(xs.reshape(-1, 3))
        out = np.zeros_like(xs)
        check(lib().uvlm_velocity_at(self._h, _p(xs), xs.shape[0], int(bool(include_freestream)), _p(out)), self._h)
        return out[0] if single else out

    def set_mlp(self, mlp) -> None:
        """Network of the learned warm start (keep it alive while in use)."""
        self._mlp = mlp
        check(lib().uvlm_set_mlp(self._h, mlp.handle if mlp is not None else None), self._h)

    def collect_training_data(self, enable: bool, max_samples: int = 0) -> None:
        check(lib().uvlm_collect_training_data(self._h, int(bool(enable)), int(max_samples)), self._h)

    def training_data(self):
        n = C.c_int64()
        check(lib().uvlm_get_training_data(self._h, None, None, C.byref(n)), self._h)
        X = np.zeros((n.value, 8), np.float32)
        T = np.zeros(n.value, np.float32)
        FP = C.POINTER(C.c_float)
        check(lib().uvlm_get_training_data(self._h, X.ctypes.data_as(FP), T.ctypes.data_as(FP), C.byref(n)),
              self._h)
        return X, T

    def set_stage_timing(self, enable: bool) -> None:
        check(lib().uvlm_set_stage_timing(self._h, int(bool(enable))), self._h)

    def synchronize(self) -> None:
        check(lib().uvlm_synchronize(self._h), self._h)

    def stream(self) -> int:
        return lib().uvlm_stream(self._h) or 0

    def close(self) -> None:
        if getattr(self, "_h", None):
            h, self._h = self._h, None
            check(lib().uvlm_destroy(h))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _write_loads(self, rows: np.ndarray) -> None:
        # PrepareOutputLoad + CalcLoad's TSV rows (simple_simulator.cpp:226-232, 334-346)
        names = ["t"] + [f"{k}{n}" for n in range(self._num) for k in ("CD", "CL")]
        with open(self._load_path, "w") as f:
            f.write("\t".join(names) + "\n")
            for r in rows:
                f.write("\t".join("%g" % v for v in r) + "\n")


class Advection:
    """advect::Advection (src/advect.h:48-59) created by ``AdvectFactory``."""

    def __init__(self, name: str, precision: str = "fp64"):
        if name not in ADVECT:
            raise UVLMError(1, "Invalid advection name! Please choose from following: [AB2, RK2, RK4, euler]")
        self.name = name
        h = C.c_void_p()
        check(lib().uvlm_advection_create(name.encode(), PRECISION[precision], C.byref(h)))
        self._h = h

    def Advect(self, wing_pos, wing_gamma, wake_pos, wake_gamma, forward_flight, dt, next=None):  # noqa: N802,A002
        """Returns the advected wake nodes (``next``, which may be wake_pos)."""
        wp = _f64(wing_pos)
        wg = _f64(wing_gamma)
        kp = _f64(wake_pos)
        kg = _f64(wake_gamma)
        num, rows, cols = wg.shape
        wake_rows = kp.shape[1] - 1
        out = next if next is not None else np.empty_like(kp)
        if out is kp or not out.flags.c_contiguous:
            out = np.empty_like(kp)
        check(lib().uvlm_advection_advect(self._h, _p(out), _p(wp), _p(wg), num, rows, cols, _p(kp),
                                          _p(kg) if kg.size else None, wake_rows, _p(_f64(forward_flight)),
                                          float(dt)))
        if next is not None and out is not next:
            next[...] = out
            return next
        return out

    advect = Advect

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                lib().uvlm_advection_destroy(self._h)
            except Exception:
                pass
            self._h = None


def AdvectFactory(name: str, precision: str = "fp64") -> Advection:  # noqa: N802
    """src/advect_factory.cpp:43-60."""
    return Advection(name, precision)


def InducedVelocity(x, pos, gamma, precision: str = "fp64") -> np.ndarray:  # noqa: N802
    """UVLM::InducedVelocity(x, pos, gamma) (src/velocity.h:14-24).

    x: (3,) or (T, 3); pos: (num, rows+1, cols+1, 3); gamma: (num, rows, cols)."""
    pos = _f64(pos)
    gamma = _f64(gamma)
    xs = _f64(x)
    single = xs.ndim == 1
    xs = xs.reshape(-1, 3)
    out = np.zeros_like(xs)
    num, gr, gc = gamma.shape
    check(lib().uvlm_sheet_induced_velocity(_p(pos), _p(gamma) if gamma.size else None, num, gr, gc, _p(xs),
                                            xs.shape[0], _p(out), PRECISION[precision]))
    return out[0] if single else out


def dense_solve(A, b, method: str = "fp64"):
    """x = A^-1 b on the GPU; method "fp64" (LU), "tf32" or "bf16" (LU + GMRES).

    Returns (x, gmres_iterations)."""
    A = _f64(A)
    b = _f64(b)
    x = np.zeros_like(b)
    it = C.c_int32(0)
    m = {"fp64": 0, "tf32": 1, "bf16": 2}[method]
    check(lib().uvlm_dense_solve(_p(A), A.shape[0], _p(b), _p(x), m, C.byref(it)))
    return x, it.value


def lu_factor_f32(A, update: str = "tf32"):
    """FP32 LU with partial pivoting on the GPU; update "simt", "tf32" or
    "bf16" (tcgen05 tensor-core trailing updates).  Returns (LU, ipiv)."""
    A = np.ascontiguousarray(np.asarray(A, dtype=np.float32))
    n = A.shape[0]
    LU = np.zeros_like(A)
    ipiv = np.zeros(n, np.int32)
    FP = C.POINTER(C.c_float)
    check(lib().uvlm_lu_factor_f32(A.ctypes.data_as(FP), n, {"simt": 0, "tf32": 1, "bf16": 2}[update],
                                   LU.ctypes.data_as(FP), ipiv.ctypes.data_as(C.POINTER(C.c_int32))))
    return LU, ipiv


from . import rings  # noqa: E402  (legacy AoS API)
from . import legacy  # noqa: E402  (legacy stepper over the AoS API)
from . import warmstart  # noqa: E402  (learned warm start)


from .batch import BatchSimulator, draw_cases, shard_cases  # noqa: E402,F401
