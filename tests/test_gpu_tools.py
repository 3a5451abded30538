"""Velocity-field tools on the GPU N-body against the oracle (B200), on the
records of a short run.  velocity_at evaluates the AllVortexSheets rings in
their stored node order with the AoS law, which gives the negative of the
simulator's sheet velocity (the reference tool's behaviour); the Snapshot2
rings of the grid tools reproduce the sheet velocity."""
import math
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def records(tmp_path_factory):
    import uvlm_b200 as U

    d = tmp_path_factory.mktemp("run")
    sheets, result = str(d / "sheets.rec"), str(d / "result.rec")
    sim = U.SimpleSimulator(precision="fp64")
    sim.AddWing(U.RectGenerator(), U.Morphing().set_plug(0.1, 1.0).set_alpha(0.08), 1.0, 4.0, 4, 8)
    sim.set_forward_flight([-1.0, 0.0, 0.0])
    sim.set_advection("RK2")
    sim.set_sheet_path(sheets)
    sim.set_result_path(result)
    sim.Run(8, 2 * math.pi / 40)
    sim.close()
    return d, sheets, result


def _orc_rings(o, rings, gammas, pts):
    return np.array([o.rings_induced_velocity(rings, gammas, p) for p in pts])


def test_velocity_at_matches_oracle_and_sign(records):
    import pyoracle as o

    from uvlm_b200 import output, tools

    _, sheets, _ = records
    x = np.array([0.6, 0.3, 0.15])
    rows = tools.velocity_at(sheets, x, 0, wing=True, wake=True)
    recs = output.read_sheets(sheets)
    assert rows.shape == (9, 5)
    for r, rec in zip(rows, recs):
        ref = o.rings_induced_velocity(rec["wing"]["rings"], rec["wing"]["gammas"], x)
        if rec["wake"]["rows"]:
            ref = ref + o.rings_induced_velocity(rec["wake"]["rings"], rec["wake"]["gammas"], x)
        np.testing.assert_allclose(r[2:], ref, rtol=0, atol=1e-12 * max(1.0, np.abs(ref).max()))
        pos, g = output.sheet_to_grid(rec["wing"])
        sheet_v = o.sheet_induced_velocity(pos, g, x[None])[0]
        if rec["wake"]["rows"]:
            wpos, wg = output.sheet_to_grid(rec["wake"])
            sheet_v = sheet_v + o.sheet_induced_velocity(wpos, wg, x[None])[0]
        np.testing.assert_allclose(r[2:], -sheet_v, rtol=0, atol=1e-12 * max(1.0, np.abs(sheet_v).max()))


def test_plane_and_volume_velocity_match_oracle(records):
    import pyoracle as o

    from uvlm_b200 import output, tools

    _, sheets, result = records
    snap = output.read_snapshots(result)[-1]
    pts, vel = tools.plane_velocity(snap, "xz", (-0.5, 2.5, -0.6, 0.6), 0.4, 7)
    ref = _orc_rings(o, snap["rings"], snap["gammas"], pts)
    np.testing.assert_allclose(vel, ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    # the Snapshot2 node order reproduces the simulator's sheet velocity
    rec = output.read_sheets(sheets)[-1]
    pos, g = output.sheet_to_grid(rec["wing"])
    wpos, wg = output.sheet_to_grid(rec["wake"])
    sv = o.sheet_induced_velocity(pos, g, pts) + o.sheet_induced_velocity(wpos, wg, pts)
    np.testing.assert_allclose(vel, sv, rtol=0, atol=1e-12 * np.abs(sv).max())
    grid = dict(xmin=-0.5, xmax=2.5, ymin=-2.0, ymax=2.0, zmin=-0.5, zmax=0.5, resolution=4)
    p3, v3 = tools.volume_velocity(snap, **grid)
    ref3 = _orc_rings(o, snap["rings"], snap["gammas"], p3) + np.array([1.0, 0.0, 0.0])
    np.testing.assert_allclose(v3, ref3, rtol=0, atol=1e-12 * np.abs(ref3).max())


def test_command_line_tools(records):
    from uvlm_b200 import tools

    d, sheets, result = records
    out = str(d / "vat.tsv")
    assert tools.main(["velocity_at", "--input", sheets, "--output", out, "--x", "0.5", "--wing", "--wake"]) == 0
    assert len(open(out).read().splitlines()) == 10
    os.makedirs(d / "plane", exist_ok=True)
    assert tools.main(["2d_velocity", "--recordio", "--input", result, "--output", str(d / "plane"),
                       "--resolution", "5", "--filetype", "tsv"]) == 0
    files = sorted(os.listdir(d / "plane"))
    assert len(files) == 9 and files[0] == "v00000000.tsv"
    assert len(open(d / "plane" / files[-1]).read().splitlines()) == 26
    vtk = str(d / "v.vtk")
    assert tools.main(["3d_velocity", "--input", result, "--output", vtk, "--resolution", "3", "--step", "8"]) == 0
    lines = open(vtk).read().splitlines()
    assert lines[4] == "DIMENSIONS 3 3 3" and len(lines) == 9 + 27
    wf = str(d / "front.tsv")
    assert tools.main(["wakefront", "--input", sheets, "--output", wf, "--start", "2"]) == 0
    assert len(open(wf).read().splitlines()) == 9 - 3
