"""Per-step state records (no GPU): the library's encoder against the protobuf runtime.

`uvlm_write_state_record` writes AllVortexSheets / Snapshot2 records from
host arrays with the same encoder the time-stepper's writer thread uses.
The records are parsed by google.protobuf with message classes built from a
descriptor restating proto/uvlm.proto (field numbers, types, labels), and
re-serialised: the bytes must be identical (the encoder writes the canonical
field order of the C++ protobuf runtime).  uvlm_b200.output decodes them to
the same arrays.
"""
import numpy as np
import pytest


def _classes():
    from google.protobuf import descriptor_pb2, descriptor_pool, message_factory

    F = descriptor_pb2.FieldDescriptorProto
    fd = descriptor_pb2.FileDescriptorProto(name="uvlm_test.proto", package="UVLM.proto", syntax="proto2")

    def msg(name, flds, parent=None):
        m = (parent.nested_type if parent else fd.message_type).add(name=name)
        for fname, num, typ, label, tname in flds:
            f = m.field.add(name=fname, number=num, type=typ, label=label)
            if tname:
                f.type_name = tname
        return m

    OPT, REP, REQ = F.LABEL_OPTIONAL, F.LABEL_REPEATED, F.LABEL_REQUIRED
    D, U32, U64, M = F.TYPE_DOUBLE, F.TYPE_UINT32, F.TYPE_UINT64, F.TYPE_MESSAGE
    # proto/uvlm.proto:4-100
    msg("Point", [("x", 1, D, OPT, None), ("y", 2, D, OPT, None), ("z", 3, D, OPT, None)])
    msg("VortexRing", [("gamma", 1, D, OPT, None), ("nodes", 2, M, REP, ".UVLM.proto.Point"),
                       ("nodes0", 3, M, REP, ".UVLM.proto.Point")])
    msg("MorphingVelocity", [("center", 1, M, OPT, ".UVLM.proto.Point"), ("nodes", 2, M, REP, ".UVLM.proto.Point"),
                             ("freestream", 3, M, OPT, ".UVLM.proto.Point")])
    s2 = msg("Snapshot2", [("t", 1, D, OPT, None),
                           ("container_shapes", 2, M, REP, ".UVLM.proto.Snapshot2.ContainerShape"),
                           ("vortices", 3, M, REP, ".UVLM.proto.VortexRing"),
                           ("morphing_velocities", 4, M, REP, ".UVLM.proto.MorphingVelocity")])
    msg("ContainerShape", [("rows", 1, U32, REQ, None), ("cols", 2, U32, REQ, None), ("id", 3, U32, OPT, None),
                           ("origin", 4, M, OPT, ".UVLM.proto.Point"), ("chord", 5, D, OPT, None),
                           ("span", 6, D, OPT, None)], parent=s2)
    msg("VortexSheet", [("t", 1, D, OPT, None), ("num", 2, U32, REQ, None), ("rows", 3, U32, REQ, None),
                        ("cols", 4, U32, REQ, None), ("vortices", 5, M, REP, ".UVLM.proto.VortexRing")])
    msg("AllVortexSheets", [("t", 1, D, OPT, None), ("wing", 2, M, OPT, ".UVLM.proto.VortexSheet"),
                            ("wake", 3, M, OPT, ".UVLM.proto.VortexSheet")])
    del U64
    pool = descriptor_pool.DescriptorPool()
    pool.Add(fd)
    get = lambda n: message_factory.GetMessageClass(pool.FindMessageTypeByName("UVLM.proto." + n))  # noqa: E731
    return get("AllVortexSheets"), get("Snapshot2")


def _state(rng, num, rows, cols, wr):
    pos = rng.standard_normal((num, rows + 1, cols + 1, 3))
    g = rng.standard_normal((num, rows, cols))
    wpos = rng.standard_normal((num, wr + 1, cols + 1, 3))
    wg = rng.standard_normal((num, wr, cols))
    return pos, g, wpos, wg


def _write(path, kind, append, st, t):
    import ctypes as C

    from uvlm_b200._capi import check, lib

    pos, g, wpos, wg = [np.ascontiguousarray(a) for a in st]
    P = C.POINTER(C.c_double)
    num, rows, cols = g.shape
    check(lib().uvlm_write_state_record(str(path).encode(), int(append), kind, num, rows, cols, wg.shape[1],
                                        pos.ctypes.data_as(P), g.ctypes.data_as(P), wpos.ctypes.data_as(P),
                                        wg.ctypes.data_as(P) if wg.size else None, float(t)))


@pytest.mark.parametrize("wr", [0, 3])
def test_sheet_records_parse_and_reserialise(tmp_path, wr):
    from uvlm_b200 import output

    AllVortexSheets, Snapshot2 = _classes()
    rng = np.random.default_rng(wr)
    st = _state(rng, 2, 3, 4, wr)
    path = tmp_path / "sheets.rec"
    _write(path, 0, False, st, 0.25)
    _write(path, 0, True, st, 0.5)
    recs = list(output.read_records(str(path)))
    assert len(recs) == 2
    for rec, t in zip(recs, (0.25, 0.5)):
        m = AllVortexSheets()
        m.ParseFromString(rec)
        assert m.t == t and m.wing.num == 2 and m.wing.rows == 3 and m.wing.cols == 4 and m.wake.rows == wr
        assert len(m.wing.vortices) == 24 and len(m.wake.vortices) == 2 * wr * 4
        assert m.SerializeToString() == rec
        pos, g, wpos, wg = st
        v = m.wing.vortices[1 * 12 + 2 * 4 + 3]   # ring (n=1, i=2, j=3): p(i,j), p(i,j+1), p(i+1,j+1), p(i+1,j)
        assert v.gamma == g[1, 2, 3]
        want = [pos[1, 2, 3], pos[1, 2, 4], pos[1, 3, 4], pos[1, 3, 3]]
        assert all([nd.x, nd.y, nd.z] == list(w) for nd, w in zip(v.nodes, want))
        d = output.decode_all_vortex_sheets(rec)
        assert d["t"] == t
        p2, g2 = output.sheet_to_grid(d["wing"])
        np.testing.assert_array_equal(p2, pos)
        np.testing.assert_array_equal(g2, g)
        if wr:
            p3, g3 = output.sheet_to_grid(d["wake"])
            np.testing.assert_array_equal(p3, wpos)
            np.testing.assert_array_equal(g3, wg)


def test_snapshot2_records(tmp_path):
    from uvlm_b200 import output

    _, Snapshot2 = _classes()
    st = _state(np.random.default_rng(5), 1, 2, 3, 2)
    path = tmp_path / "result.rec"
    _write(path, 1, False, st, 1.0)
    (rec,) = list(output.read_records(str(path)))
    m = Snapshot2()
    m.ParseFromString(rec)
    assert not m.HasField("t") and len(m.vortices) == 6 + 6
    assert m.SerializeToString() == rec
    pos, g, wpos, wg = st
    v = m.vortices[6 + 4]  # wake ring (0, 1, 1): SheetToSnapshot order p(i+1,j), p(i+1,j+1), p(i,j+1), p(i,j)
    want = [wpos[0, 2, 1], wpos[0, 2, 2], wpos[0, 1, 2], wpos[0, 1, 1]]
    assert v.gamma == wg[0, 1, 1] and all([nd.x, nd.y, nd.z] == list(w) for nd, w in zip(v.nodes, want))
    d = output.decode_snapshot2(rec)
    np.testing.assert_array_equal(d["gammas"], np.concatenate([g.ravel(), wg.ravel()]))


def _legacy_snapshot(rng, shapes, n_wake):
    n_bound = sum(r * c for r, c, _, _ in shapes)
    n = n_bound + n_wake
    return dict(rings=rng.standard_normal((n, 4, 3)), rings0=rng.standard_normal((n, 4, 3)),
                gammas=rng.standard_normal(n), mv_center=rng.standard_normal((n_bound, 3)),
                mv_nodes=rng.standard_normal((n_bound, 4, 3)), mv_freestream=rng.standard_normal((n_bound, 3)))


@pytest.mark.parametrize("with_nodes0", [True, False])
def test_legacy_snapshot2_file(tmp_path, with_nodes0):
    """OutputSnapshot2 (src/simulator/simulator.cpp:118-160): unframed Snapshot2 with t, shapes, the pool
    with nodes0 and the morphing velocity records, in the C++ runtime's canonical field order."""
    from uvlm_b200 import output

    _, Snapshot2 = _classes()
    shapes = [(2, 4, 1.0, 2.0), (2, 4, 0.5, 1.5)]
    s = _legacy_snapshot(np.random.default_rng(11), shapes, 6)
    r0 = s["rings0"] if with_nodes0 else None
    path = tmp_path / "00000003"
    output.write_legacy_snapshot2(path, 0.75, shapes, s["rings"], r0, s["gammas"], s["mv_center"], s["mv_nodes"],
                                  s["mv_freestream"])
    raw = open(path, "rb").read()
    m = Snapshot2()
    m.ParseFromString(raw)
    assert m.SerializeToString() == raw
    assert m.t == 0.75
    assert [(c.rows, c.cols, c.id, c.chord, c.span) for c in m.container_shapes] == [(2, 4, 0, 1.0, 2.0),
                                                                                     (2, 4, 1, 0.5, 1.5)]
    assert not m.container_shapes[0].HasField("origin")
    assert len(m.vortices) == 22 and len(m.morphing_velocities) == 16
    v = m.vortices[19]
    assert v.gamma == s["gammas"][19]
    assert [[p.x, p.y, p.z] for p in v.nodes] == s["rings"][19].tolist()
    assert [[p.x, p.y, p.z] for p in v.nodes0] == (s["rings0"][19].tolist() if with_nodes0 else [])
    mv = m.morphing_velocities[5]
    assert [mv.center.x, mv.center.y, mv.center.z] == s["mv_center"][5].tolist()
    assert [[p.x, p.y, p.z] for p in mv.nodes] == s["mv_nodes"][5].tolist()
    assert [mv.freestream.x, mv.freestream.y, mv.freestream.z] == s["mv_freestream"][5].tolist()
    d = output.read_snapshot2_file(str(path))
    assert d["t"] == 0.75
    for k in ("rings", "gammas", "mv_center", "mv_nodes", "mv_freestream"):
        np.testing.assert_array_equal(d[k], s[k])
    if with_nodes0:
        np.testing.assert_array_equal(d["rings0"], s["rings0"])
    else:
        assert d["rings0"] is None
    assert [c["offset"] for c in output.snapshot_containers(d)] == [0, 8]


def test_legacy_snapshot2_errors(tmp_path):
    import uvlm_b200 as U
    from uvlm_b200 import output

    s = _legacy_snapshot(np.random.default_rng(1), [(1, 2, 1.0, 1.0)], 0)
    with pytest.raises(ValueError):
        output.write_legacy_snapshot2(tmp_path / "x", 0.0, [(1, 2, 1.0, 1.0)], s["rings"], s["rings0"][:1],
                                      s["gammas"], s["mv_center"], s["mv_nodes"], s["mv_freestream"])
    with pytest.raises(U.UVLMError):
        output.write_legacy_snapshot2(tmp_path / "no_dir" / "x", 0.0, [(1, 2, 1.0, 1.0)], s["rings"], None,
                                      s["gammas"], s["mv_center"], s["mv_nodes"], s["mv_freestream"])
    # an empty snapshot (no containers, rings or records) is a valid message holding only t
    output.write_legacy_snapshot2(tmp_path / "e", 2.5, [], np.zeros((0, 4, 3)), None, [], np.zeros((0, 3)),
                                  np.zeros((0, 4, 3)), np.zeros((0, 3)))
    d = output.read_snapshot2_file(str(tmp_path / "e"))
    assert d["t"] == 2.5 and d["rings"].shape == (0, 4, 3) and d["container_shapes"] == []


def test_snapshot2_to_containers_kat():
    """test/proto_adaptor_test.cpp:7-50 (Snapshot2ToContainers): two shapes {id i, rows 2, cols 1} and four
    rings carrying only their circulations 0..3; container c holds rings 2c, 2c + 1."""
    from uvlm_b200 import output, tools

    _, Snapshot2 = _classes()
    m = Snapshot2()
    for i in range(2):
        sh = m.container_shapes.add()
        sh.id, sh.rows, sh.cols = i, 2, 1
    for i in range(4):
        m.vortices.add().gamma = i
    d = output.decode_snapshot2(m.SerializeToString())
    np.testing.assert_array_equal(d["gammas"], [0, 1, 2, 3])
    assert d["rings"] is None
    cs = output.snapshot_containers(d)
    assert [(c["rows"], c["cols"], c["rows"] * c["cols"]) for c in cs] == [(2, 1, 2), (2, 1, 2)]
    assert [d["gammas"][c["offset"] + k] for c in cs for k in range(2)] == [0, 1, 2, 3]
    # dump_circulation prints the circulation alone for rings without nodes
    assert tools.dump_circulation(d) == "0\t0\t0\t0\n\n0\t1\t0\t1\n\n\n\n1\t0\t0\t2\n\n1\t1\t0\t3\n\n\n\n"
    with pytest.raises(ValueError, match="no nodes"):
        tools.dump_centroid(d)


def test_to_vortex_sheet_kat(tmp_path):
    """test/proto_adaptor_test.cpp:52-79 (ToVortexSheet / FromVortexSheet): a 2 x 2 x 1 sheet set with
    circulations at(n, i, 0) = 2n + i."""
    from uvlm_b200 import output

    pos = np.zeros((2, 3, 2, 3))
    g = np.array([[[0.0], [1.0]], [[2.0], [3.0]]])
    path = tmp_path / "sheet.rec"
    _write(path, 0, False, (pos, g, np.zeros((2, 1, 2, 3)), np.zeros((2, 0, 1))), 0.0)
    (rec,) = output.read_sheets(str(path))
    w = rec["wing"]
    assert (w["num"], w["rows"], w["cols"]) == (2, 2, 1)
    np.testing.assert_array_equal(w["gammas"], [0, 1, 2, 3])
    _, g2 = output.sheet_to_grid(w)
    np.testing.assert_array_equal(g2, g)
