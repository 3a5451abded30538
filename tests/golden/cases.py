"""Parity cases shared by the fixture generator and the tests.

Each case is a SimpleSimulator set-up in the reference's own terms (wings from
RectGenerator + WholeWing, Morphing kinematics, forward flight, advection
scheme, dt, steps).  ``plunge_euler_8x16_200`` is the reference's CPU-runnable configuration:
one 8 x 16 flat-plate wing (chord 1, span 4), plunge 0.1 sin(2 pi 0.25 t) at
5 degrees, U = 1, dt = 1/8, 200 explicit-Euler steps; its lattice is shifted
1/4 panel downstream so that the ring centroids (the reference's collocation
points) sit at 3/4 of each geometric panel chord.
"""
import math

DEG = math.pi / 180.0

CASES = {
    "plunge_euler_8x16_200": dict(
        wings=[dict(chord=1.0, span=4.0, rows=8, cols=16, origin=(1.0 / 8 / 4, 0.0, 0.0),
                    kin=dict(alpha=5 * DEG, plug_amp=0.1, plug_omega=2 * math.pi * 0.25))],
        ff=(-1.0, 0.0, 0.0), advection="euler", dt=0.125, steps=200),
    "rk2_heave_pitch_4x8": dict(
        wings=[dict(chord=1.0, span=4.0, rows=4, cols=8, origin=(0.0, 0.0, 0.0),
                    kin=dict(plug_amp=0.2, plug_omega=1.0, twist_amp=10 * DEG, twist_omega=1.0,
                             twist_phase=math.pi / 2))],
        ff=(-1.0, 0.0, 0.0), advection="RK2", dt=2 * math.pi / 40, steps=14),
    "rk4_flap_4x8": dict(
        wings=[dict(chord=1.0, span=6.0, rows=4, cols=8, origin=(0.0, 0.0, 0.0),
                    kin=dict(alpha=4 * DEG, flap_amp=15 * DEG, flap_omega=0.2, flap_phase=math.pi / 2,
                             twist_span_slope=4 * DEG / 6.0, twist_omega=0.2, twist_phase=math.pi))],
        ff=(-1.0, 0.0, 0.0), advection="RK4", dt=0.25, steps=10),
    "ab2_plunge_4x8": dict(
        wings=[dict(chord=1.0, span=6.0, rows=4, cols=8, origin=(0.0, 0.0, 0.0),
                    kin=dict(alpha=5 * DEG, plug_amp=0.175, plug_omega=1.0, plug_phase=math.pi / 2))],
        ff=(-1.0, 0.0, 0.0), advection="AB2", dt=2 * math.pi / 40, steps=12),
    "two_wings_euler_3x6": dict(
        wings=[dict(chord=1.0, span=4.0, rows=3, cols=6, origin=(0.0, 0.0, 0.0),
                    kin=dict(alpha=5 * DEG, plug_amp=0.15, plug_omega=0.8)),
               dict(chord=1.0, span=4.0, rows=3, cols=6, origin=(1.5, 0.0, 0.5),
                    kin=dict(alpha=5 * DEG, plug_amp=0.15, plug_omega=0.8, plug_phase=math.pi / 2))],
        ff=(-1.0, 0.0, 0.0), advection="euler", dt=0.2, steps=10),
    "morph_bend_rk2_4x8": dict(
        wings=[dict(chord=1.0, span=4.0, rows=4, cols=8, origin=(0.0, 0.0, 0.0),
                    kin=dict(alpha=3 * DEG, bend_cx=0.05, bend_cy=0.1, bend_omega=0.6))],
        ff=(-1.0, 0.0, 0.0), advection="RK2", dt=0.2, steps=10),
    "erase_euler_4x8": dict(
        wings=[dict(chord=1.0, span=4.0, rows=4, cols=8, origin=(0.0, 0.0, 0.0),
                    kin=dict(alpha=5 * DEG, plug_amp=0.1, plug_omega=1.0))],
        ff=(-1.0, 0.0, 0.0), advection="euler", dt=0.2, steps=14, erase_wake_after=8),
    # the 4-wing tandem/biplane formation at small size: 2 x 2 arrangement
    # {x=0,1.5} x {z=0,0.5}; phases 0/90 deg (front lower/upper) and 180/270
    # deg (rear lower/upper), so biplane partners move a quarter period apart
    # (in anti-phase their trailing edges cross and the core-free kernel
    # diverges); heave 0.15 c + pitch 15 deg
    "tandem4_rk2_3x6": dict(
        wings=[dict(chord=1.0, span=4.0, rows=3, cols=6, origin=(x, 0.0, z),
                    kin=dict(plug_amp=0.15, plug_omega=0.8, plug_phase=q * math.pi / 2, twist_amp=15 * DEG,
                             twist_omega=0.8, twist_phase=q * math.pi / 2 + math.pi / 2))
               for q, (x, z) in enumerate([(0.0, 0.0), (0.0, 0.5), (1.5, 0.0), (1.5, 0.5)])],
        ff=(-1.0, 0.0, 0.0), advection="RK2", dt=2 * math.pi / 0.8 / 40, steps=12,
        wake_pos_tol=1e-7),  # the wakes pass close to the rear wings and amplify rounding
    # the morphing shape at small size: camber 0.05 sin(wt) x(1-x) + span bend
    # 0.1 sin(wt) y^2, k = 0.3, Euler
    "morph_camber_euler_4x8": dict(
        wings=[dict(chord=1.0, span=8.0, rows=4, cols=8, origin=(0.0, 0.0, 0.0),
                    kin=dict(bend_cx=0.05, bend_cy=0.1, bend_omega=0.6))],
        ff=(-1.0, 0.0, 0.0), advection="euler", dt=2 * math.pi / 0.6 / 40, steps=16),
    # src/multiple_flapping_wings_main.cpp:40-73 with its flag defaults: NACA 83 camber lattice
    # (NACA4digitGenerator(83)), AR 6, alpha 5 deg, flap -pi/4 cos(w t) = pi/4 sin(w t - pi/2) with
    # w = 2 U k / c, k = 0.1, --lines 2 (the leading wing and two wings at (3, +-6, 0)), 6 x 20 rings,
    # 40 steps per cycle, Euler; 30 of its 50 steps
    "naca83_flap_3wings_6x20": dict(
        wings=[dict(chord=1.0, span=6.0, rows=6, cols=20, origin=o, generator=("naca4digit", 83),
                    kin=dict(alpha=5 * DEG, flap_amp=math.pi / 4, flap_omega=0.2, flap_phase=-math.pi / 2))
               for o in [(0.0, 0.0, 0.0), (3.0, 6.0, 0.0), (3.0, -6.0, 0.0)]],
        ff=(-1.0, 0.0, 0.0), advection="euler", dt=2 * math.pi / 0.2 / 40, steps=30,
        wake_pos_tol=1e-8),  # the +-45 deg flap sweeps each wake close to its own wing's lattice
    "chebyshev_euler_4x8": dict(
        wings=[dict(chord=1.0, span=4.0, rows=4, cols=8, origin=(0.0, 0.0, 0.0), cheb_chord=True, cheb_span=True,
                    kin=dict(alpha=6 * DEG, plug_amp=0.05, plug_omega=1.5))],
        ff=(-1.0, 0.0, 0.0), advection="euler", dt=0.2, steps=8),
}


def run_oracle(case: dict):
    """Runs a case on the CPU oracle; returns (loads, final state)."""
    import numpy as np
    import pyoracle as o

    sim = o.Simulator()
    for w in case["wings"]:
        gen, digit = w.get("generator", ("rect", 0))
        sim.add_wing_generator(gen, digit, w["chord"], w["span"], w["rows"], w["cols"], origin=w["origin"],
                               kin=o.kinematics(**w["kin"]), cheb_chord=w.get("cheb_chord", False),
                               cheb_span=w.get("cheb_span", False))
    sim.set_forward_flight(case["ff"])
    sim.set_advection(case["advection"])
    if case.get("erase_wake_after"):
        sim.set_erase_wake_after(case["erase_wake_after"])
    loads = sim.run(case["steps"], case["dt"])
    return np.asarray(loads), sim.state()


def make_gpu_sim(case: dict, **kw):
    """The same case on the CUDA library (uvlm_b200.SimpleSimulator)."""
    import uvlm_b200 as U

    sim = U.SimpleSimulator(erase_wake_after=case.get("erase_wake_after", 0), **kw)
    for w in case["wings"]:
        m = U.Morphing()
        k = w["kin"]
        m.set_alpha(k.get("alpha", 0.0))
        m.set_plug(k.get("plug_amp", 0.0), k.get("plug_omega", 0.0), k.get("plug_phase", 0.0))
        m.set_flap(k.get("flap_amp", 0.0), k.get("flap_omega", 0.0), k.get("flap_phase", 0.0))
        m.set_twist(k.get("twist_amp", 0.0), k.get("twist_omega", 0.0), k.get("twist_phase", 0.0),
                    k.get("twist_span_slope", 0.0))
        m.set_bend(k.get("bend_cx", 0.0), k.get("bend_cy", 0.0), k.get("bend_omega", 0.0), k.get("bend_phase", 0.0))
        gen, digit = w.get("generator", ("rect", 0))
        cheb = (w.get("cheb_chord", False), w.get("cheb_span", False))
        g = {"rect": lambda: U.RectGenerator(*cheb), "naca4digit": lambda: U.NACA4digitGenerator(digit, *cheb),
             "naca00xx": lambda: U.NACA00XXGenerator(digit, *cheb)}[gen]()
        sim.AddWing(g, m, w["chord"], w["span"], w["rows"], w["cols"], w["origin"])
    sim.set_forward_flight(case["ff"])
    sim.set_advection(case["advection"])
    return sim


# The benchmark workloads at full size (the same set-ups as bench.py's
# heave_pitch, tandem4 and morphing workloads; tests/test_oracle_golden.py
# checks that they agree), for the oracle-pinned full-size fixtures made by
# tests/golden/make_fullsize.py.  `steps` is the window the fixture covers:
# from step 0 while the FP64 form's own one-ulp sensitivity stays far below
# the tolerances of the parity tests.
def _fullsize():
    hp_w = 1.0
    heave_pitch = dict(
        wings=[dict(chord=1.0, span=8.0, rows=32, cols=128, origin=(0.0, 0.0, 0.0),
                    kin=dict(plug_amp=0.2, plug_omega=hp_w, twist_amp=10 * DEG, twist_omega=hp_w,
                             twist_phase=math.pi / 2))],
        ff=(-1.0, 0.0, 0.0), advection="RK2", dt=2 * math.pi / hp_w / 40, steps=40,
        # the mixed form as configured by default (RHS near field in FP64): CL/CD bound per window end
        mixed=dict(kw={}, windows={40: 1e-6}))
    tw = 0.8
    tandem = dict(
        wings=[dict(chord=1.0, span=4.0, rows=16, cols=64, origin=(x, 0.0, z),
                    kin=dict(plug_amp=0.15, plug_omega=tw, plug_phase=q * math.pi / 2, twist_amp=15 * DEG,
                             twist_omega=tw, twist_phase=q * math.pi / 2 + math.pi / 2))
               for q, (x, z) in enumerate([(0.0, 0.0), (0.0, 0.5), (1.5, 0.0), (1.5, 0.5)])],
        ff=(-1.0, 0.0, 0.0), advection="RK2", dt=2 * math.pi / tw / 40, steps=20,
        # the front wings' wakes pass through the rear wings' lattices: a wake node that
        # passes a bound segment closely amplifies rounding in its own position
        gamma_tol=1e-8, wake_pos_tol=1e-4,
        # the near field of every stage in FP64 (the default's 2.6e-6 misses 1e-6 here)
        mixed=dict(kw=dict(near_fp64=True), windows={20: 1e-6}))
    mw = 0.6
    morphing = dict(
        wings=[dict(chord=1.0, span=8.0, rows=24, cols=96, origin=(0.0, 0.0, 0.0),
                    kin=dict(bend_cx=0.05, bend_cy=0.1, bend_omega=mw))],
        ff=(-1.0, 0.0, 0.0), advection="euler", dt=2 * math.pi / mw / 40, steps=50,
        # the span bend lifts the tips by up to 1.6 chords: the rolled-up tip wake
        # passes its own segments closely, which amplifies rounding in those nodes
        wake_pos_tol=1e-4,
        # near field of every stage in FP64; after step 40 the tip wake's roll-up amplifies
        # the FP32 far field's rounding (the FP64 form's own one-ulp sensitivity grows from
        # 2e-14 to 1.4e-10 between steps 40 and 50)
        mixed=dict(kw=dict(near_fp64=True), windows={40: 1e-6, 50: 1e-5}))
    return {"heave_pitch_32x128": heave_pitch, "tandem4_16x64": tandem, "morphing_24x96": morphing}


FULLSIZE = _fullsize()
