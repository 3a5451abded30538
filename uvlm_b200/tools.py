"""The reference's velocity-field tools (src/tools/*_main.cpp) on the GPU N-body.

They post-process the per-step records of a run (uvlm_b200.output):

* velocity_at  (velocity_at_main.cpp:53-99): the velocity that the wing and/or
  wake sheet of one wing induces at a fixed point, per AllVortexSheets record;
* plane_velocity (2d_velocity_main.cpp:58-174): the velocity induced by every
  ring of a Snapshot2 on a resolution x resolution grid of a coordinate plane;
* volume_velocity (3d_velocity_main.cpp:35-126): the same on a 3-D grid plus
  the freestream (1, 0, 0), written as a VTK structured-points file;
* wakefront (wakefront_main.cpp:17-58): the x of the nodes of one wake row;
* calc_impulse (src/calc_impulse_main.cpp:54-107): per legacy Snapshot2 file,
  the vortex impulse of the first wing, its Lamb-vector term and the vortex
  impulse of the wake (GPU reductions);
* dump_circulation / dump_centroid (dump_circulation_main.cpp:23-57,
  dump_centroid_main.cpp:30-122): gnuplot text of one legacy Snapshot2 file.

Rings are evaluated as the reference's tools evaluate them: AoS rings with
the nodes in the order the record stores them (ProtoToVortexRing,
src/proto_adaptor.h:39-47), summed by UVLM::InducedVelocity
(src/shed.inl:22-33) -- one FP64 N-body launch per record.  As in the
reference, velocity_at reads ToVortexSheet's node order p(i,j), p(i,j+1),
p(i+1,j+1), p(i+1,j), which the AoS segment order traverses opposite to the
simulator's VORING, so its velocities have the opposite sign of the
simulator's own; the Snapshot2 order of the grid tools matches VORING.

Command line: python -m uvlm_b200.tools {velocity_at,2d_velocity,3d_velocity,wakefront,calc_impulse,
dump_circulation,dump_centroid} --flag=value ... with the reference tools' flag names.  The text tables of
the last three use the reference's number format (C++ stream default, printf %g).
"""
from __future__ import annotations

import argparse
import glob
import os
import sys

import numpy as np

from . import output, rings


def velocity_at(sheet_path: str, pos, wing_id: int = 0, wing: bool = False, wake: bool = False) -> np.ndarray:
    """Rows (step, t, vx, vy, vz), one per AllVortexSheets record."""
    if not (wing or wake):
        raise ValueError("At least one of --wing or --wake must be true.")
    if wing_id < 0:
        raise ValueError("id must be >= 0")
    x = np.asarray(pos, dtype=np.float64).reshape(3)
    rows = []
    for count, rec in enumerate(output.read_sheets(sheet_path)):
        v = np.zeros(3)
        for use, sheet in ((wing, rec["wing"]), (wake, rec["wake"])):
            if not use or sheet is None:
                continue
            per = sheet["rows"] * sheet["cols"]
            sel = slice(wing_id * per, (wing_id + 1) * per)  # iterator_at(id, 0, 0) .. iterator_at(id + 1, 0, 0)
            if per:
                v = v + rings.InducedVelocity(x, sheet["rings"][sel], sheet["gammas"][sel])
        rows.append([count, rec["t"], v[0], v[1], v[2]])
    return np.array(rows).reshape(-1, 5)


def plane_points(plane: str = "xz", rng=(-1.0, -1.0, 1.0, 1.0), at: float = 0.0, resolution: int = 100) -> np.ndarray:
    """CreatePoints (2d_velocity_main.cpp:58-89): axis plane[0] over [rng[0], rng[1]], plane[1] over
    [rng[2], rng[3]], the third axis at `at`; nested x, y, z loops (x outermost)."""
    if len(plane) != 2 or plane[0] == plane[1] or any(c not in "xyz" for c in plane):
        raise ValueError("plane must be two different characters of 'xyz'")
    axes = {plane[0]: np.linspace(rng[0], rng[1], resolution), plane[1]: np.linspace(rng[2], rng[3], resolution)}
    (third,) = set("xyz") - set(plane)
    axes[third] = np.array([at], dtype=np.float64)
    X, Y, Z = np.meshgrid(axes["x"], axes["y"], axes["z"], indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], -1)


def plane_velocity(snapshot: dict, plane: str = "xz", rng=(-1.0, -1.0, 1.0, 1.0), at: float = 0.0,
                   resolution: int = 100):
    """Points and induced velocities of every ring of a decoded Snapshot2 (CalcData, :104-123)."""
    pts = plane_points(plane, rng, at, resolution)
    return pts, rings.InducedVelocity(pts, _rings(snapshot), snapshot["gammas"])


def volume_points(xmin=0.0, xmax=8.0, ymin=-4.0, ymax=4.0, zmin=-4.0, zmax=4.0, resolution=100) -> np.ndarray:
    """CreatePoints (3d_velocity_main.cpp:35-51): z outermost, x innermost."""
    xs, ys, zs = (np.linspace(a, b, resolution) for a, b in ((xmin, xmax), (ymin, ymax), (zmin, zmax)))
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], -1)


def volume_velocity(snapshot: dict, **grid) -> tuple[np.ndarray, np.ndarray]:
    """CalcData (3d_velocity_main.cpp:68-83): induced velocity plus the freestream (1, 0, 0)."""
    pts = volume_points(**grid)
    return pts, rings.InducedVelocity(pts, _rings(snapshot), snapshot["gammas"]) + np.array([1.0, 0.0, 0.0])


def write_vtk(path: str, vel: np.ndarray, xmin, xmax, ymin, ymax, zmin, zmax, resolution) -> None:
    """Write (3d_velocity_main.cpp:85-112): VTK legacy STRUCTURED_POINTS with one vector per point."""
    n = resolution
    dx, dy, dz = ((b - a) / (n - 1) for a, b in ((xmin, xmax), (ymin, ymax), (zmin, zmax)))
    with open(path, "w") as f:
        f.write("# vtk DataFile Version 2.0\nHOGE FLOW\nASCII\nDATASET STRUCTURED_POINTS\n")
        f.write(f"DIMENSIONS {n} {n} {n}\nORIGIN {xmin:f} {ymin:f} {zmin:f}\nSPACING {dx:f} {dy:f} {dz:f}\n")
        f.write(f"POINT_DATA {n * n * n}\nVECTORS volume_vectors double\n")
        for u in vel:
            f.write(f"{u[0]:f} {u[1]:f} {u[2]:f}\n")


def wakefront(sheet_path: str, start: int = 0, wing_id: int = 0) -> list[list[float]]:
    """WakeFront (wakefront_main.cpp:17-58): per record, t and the x of node 0 of every ring of wake row
    rows - start - 1 of wing `wing_id`, then node 1 of its last ring; records without that row are skipped."""
    out = []
    for rec in output.read_sheets(sheet_path):
        wk = rec["wake"]
        target = wk["rows"] - start - 1
        if target < 0:
            continue
        r = wk["rings"].reshape(wk["num"], wk["rows"], wk["cols"], 4, 3)[wing_id, target]
        out.append([rec["t"]] + list(r[:, 0, 0]) + [r[-1, 1, 0]])
    return out


def _g(values) -> str:
    """util::join("\t", ...) of doubles with the C++ stream default (src/util.h:67-78)."""
    return "\t".join(f"{v:g}" for v in values)


def _containers(snap: dict):
    return output.snapshot_containers(snap)


def _rings(snap: dict) -> np.ndarray:
    if snap["rings"] is None:
        raise ValueError("snapshot rings carry no nodes")
    return snap["rings"]


def calc_impulse(snap: dict) -> np.ndarray:
    """CalcImpulse (calc_impulse_main.cpp:54-87) of one decoded legacy Snapshot2: [t, impulse (3),
    other_term (3), wake_impulse (3)].  impulse sums VortexRing::Impulse over the first container,
    wake_impulse over the rings after all containers (CountTotalSize), and other_term sums
    CalcLambVectorOnPanel over the first container's rings with morphing record i for ring i and the
    whole pool as the inducing rings (src/calc_impulse.h:15-30)."""
    cs = _containers(snap)
    if not cs:
        raise ValueError("snapshot has no container")
    c0 = cs[0]
    n0 = c0["rows"] * c0["cols"]
    sel = slice(c0["offset"], c0["offset"] + n0)
    n_bound = sum(c["rows"] * c["cols"] for c in cs)
    R, G = _rings(snap), snap["gammas"]
    if sel.stop > len(R) or n0 > len(snap["mv_center"]):
        raise ValueError("snapshot holds fewer rings or morphing records than its first container")
    impulse = rings.CalcVortexImpulse(R[sel], G[sel])
    wake = rings.CalcVortexImpulse(R[n_bound:], G[n_bound:])
    other = rings.CalcLambVector(R[sel], G[sel], snap["mv_nodes"][:n0], snap["mv_freestream"][:n0], R, G)
    return np.concatenate([[snap["t"]], impulse, other, wake])


def glob_result(path: str) -> list[str]:
    """GlobResult (calc_impulse_main.cpp:18-32): the sorted entries of path/*."""
    return sorted(glob.glob(os.path.join(path, "*")))


def dump_circulation(snap: dict) -> str:
    """Dump (dump_circulation_main.cpp:23-57): per container, per ring (i, j) one line
    index, i, j, gamma, the xyz of its nodes; a blank line after each ring row and two after each container."""
    out = []
    R, G = snap["rings"], snap["gammas"]
    for index, c in enumerate(_containers(snap)):
        for i in range(c["rows"]):
            for j in range(c["cols"]):
                k = c["offset"] + j + i * c["cols"]
                nodes = [] if R is None else R[k].ravel()   # rings without nodes: the circulation alone
                out.append(f"{index}\t{i}\t{j}\t" + _g([G[k], *nodes]) + "\n")
            out.append("\n")
        out.append("\n\n")
    return "".join(out)


def dump_centroid(snap: dict) -> tuple[str, str, str]:
    """Dump (dump_centroid_main.cpp:30-100): the (node, centroid, velocity) files' text.  node: per ring
    of every container its nodes and the first again, then two blank lines; centroid: one line per ring
    (VortexRing::Centroid, src/vortex.cpp:98-100); velocity: centroid and morphing-velocity center per ring
    and two blank lines, written only when there is one morphing record per container ring."""
    node, cent, pos = [], [], []
    R = _rings(snap)
    for c in _containers(snap):
        for k in range(c["offset"], c["offset"] + c["rows"] * c["cols"]):
            r = R[k]
            node.extend(_g(p) + "\n" for p in (r[0], r[1], r[2], r[3], r[0]))
            node.append("\n\n")
        for k in range(c["offset"], c["offset"] + c["rows"] * c["cols"]):
            r = R[k]
            x = (r[0] + r[1] + r[2] + r[3]) / 4
            pos.append(x)
            cent.append(_g(x) + "\n")
    vel = ""
    if len(pos) == len(snap["mv_center"]):
        vel = "".join(_g(p) + "\t" + _g(v) + "\n" for p, v in zip(pos, snap["mv_center"])) + "\n\n"
    return "".join(node), "".join(cent), vel


def _write_table(path: str, header, rows, sep: str) -> None:
    with open(path, "w") as f:
        f.write(sep.join(header) + "\n")
        for r in rows:
            f.write(sep.join(f"{v:.17g}" for v in r) + "\n")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m uvlm_b200.tools")
    ap.add_argument("tool", choices=["velocity_at", "2d_velocity", "3d_velocity", "wakefront", "calc_impulse",
                                     "dump_circulation", "dump_centroid"])
    ap.add_argument("--input", default="")
    ap.add_argument("--output", default="")
    ap.add_argument("--x", type=float, default=0.0)
    ap.add_argument("--y", type=float, default=0.0)
    ap.add_argument("--z", type=float, default=0.0)
    ap.add_argument("--id", type=int, default=0)
    ap.add_argument("--wing", action="store_true")
    ap.add_argument("--wake", action="store_true")
    ap.add_argument("--resolution", type=int, default=100)
    ap.add_argument("--filetype", default="csv", choices=["csv", "tsv"])
    ap.add_argument("--plane", default="xz")
    ap.add_argument("--range", default="-1,-1,1,1")
    ap.add_argument("--at", type=float, default=0.0)
    ap.add_argument("--recordio", action="store_true")
    ap.add_argument("--prefix", default="v")
    ap.add_argument("--xmin", type=float, default=0.0)
    ap.add_argument("--xmax", type=float, default=8.0)
    ap.add_argument("--ymin", type=float, default=-4.0)
    ap.add_argument("--ymax", type=float, default=4.0)
    ap.add_argument("--zmin", type=float, default=-4.0)
    ap.add_argument("--zmax", type=float, default=4.0)
    ap.add_argument("--step", type=int, default=0)
    ap.add_argument("--start", type=int, default=0)
    a = ap.parse_args(argv)
    if a.tool == "velocity_at":
        rows = velocity_at(a.input, (a.x, a.y, a.z), a.id, a.wing, a.wake)
        _write_table(a.output, ["step", "t", "x", "y", "z"], [[int(r[0])] + list(r[1:]) for r in rows], "\t")
        print(f"{len(rows)} lines are written.", file=sys.stderr)
    elif a.tool == "2d_velocity":
        rng = tuple(float(s) for s in a.range.split(","))
        if len(rng) != 4:
            raise SystemExit("--range must be min0,max0,min1,max1")
        if a.recordio:
            snaps = output.read_snapshots(a.input)
        else:  # one Snapshot2 per file (the legacy simulator's per-step files)
            snaps = [output.decode_snapshot2(open(p, "rb").read()) for p in sorted(glob.glob(a.input))]
        sep = "," if a.filetype == "csv" else "\t"
        for k, snap in enumerate(snaps):
            pts, vel = plane_velocity(snap, a.plane, rng, a.at, a.resolution)
            _write_table(os.path.join(a.output, f"{a.prefix}{k:08d}.{a.filetype}"), ["x", "y", "z", "u", "v", "w"],
                         np.concatenate([pts, vel], 1), sep)
        print(f"write {len(snaps)} files", file=sys.stderr)
    elif a.tool == "3d_velocity":
        grid = dict(xmin=a.xmin, xmax=a.xmax, ymin=a.ymin, ymax=a.ymax, zmin=a.zmin, zmax=a.zmax,
                    resolution=a.resolution)
        for k, snap in enumerate(output.read_snapshots(a.input)):
            if k == a.step:
                _, vel = volume_velocity(snap, **grid)
                write_vtk(a.output, vel, **grid)
                print(f"write {len(vel)} points", file=sys.stderr)
                break
    elif a.tool == "calc_impulse":
        paths = glob_result(a.input)
        with open(a.output, "w") as f:
            for path in paths:
                f.write(_g(calc_impulse(output.read_snapshot2_file(path))) + "\n")
        print(f"{len(paths)} lines are written.", file=sys.stderr)
    elif a.tool == "dump_circulation":
        text = dump_circulation(output.read_snapshot2_file(a.input))
        with open(a.output, "w") as f:
            f.write(text)
        print(a.output, file=sys.stderr)
    elif a.tool == "dump_centroid":
        name = a.input[a.input.rfind("/") + 1:]  # ResultName (dump_centroid_main.cpp:64-70)
        paths = [f"{a.output}/{name}_{kind}.dat" for kind in ("node", "cent", "vel")]
        for path, text in zip(paths, dump_centroid(output.read_snapshot2_file(a.input))):
            with open(path, "w") as f:
                f.write(text)
        print(f"splot '{paths[1]}' w p, '{paths[0]}' w l, '{paths[2]}' usi 1:2:3:4:5:6 w vec\npause -1")
    else:
        rows = wakefront(a.input, a.start, a.id)
        with open(a.output, "w") as f:
            for r in rows:
                f.write("\t".join(f"{v:.17g}" for v in r) + "\n")
        print(f"{len(rows)} lines are saved", file=sys.stderr)
    return 0


if __name__ == "__main__":
    sys.exit(main())
