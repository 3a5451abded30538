"""Host logic of the batched sweep: seeded case draws, cost model and the
case sharding over ranks (world size 2, gloo on CPU; no GPU)."""
import os

import numpy as np
import pytest


def test_draw_cases_ranges_and_seed():
    from uvlm_b200.batch import draw_cases

    a = draw_cases(256, seed=0)
    b = draw_cases(256, seed=0)
    assert a == b
    assert draw_cases(256, seed=1) != a
    for d in a:
        assert 4 <= d["rows"] <= 16
        assert 8 <= d["cols"] <= 64 and d["cols"] % 2 == 0
        assert 2 <= d["span"] <= 10
        assert 0.1 <= d["k"] <= 1.0
        assert 0.05 <= d["heave"] <= 0.3
        assert 0 <= d["pitch_deg"] <= 20
        assert abs(d["dt"] - 2 * np.pi / (2 * d["k"]) / 40) < 1e-15


def test_shard_cases_balances_work():
    from uvlm_b200.batch import case_cost, draw_cases, shard_cases

    cases = draw_cases(256, seed=0)
    costs = [case_cost(d, 150) for d in cases]
    for world in (1, 2, 4, 8):
        parts = shard_cases(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(256))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) <= 1.02 * (sum(costs) / world) + max(costs)


def _rank(rank, world, port, out_dir):
    import torch.distributed as dist

    from uvlm_b200.batch import case_cost, draw_cases, gather_case_rows, shard_cases

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    cases = draw_cases(256, seed=0)
    costs = [case_cost(d, 150) for d in cases]
    mine = shard_cases(costs, world)[rank]
    # every rank reports the cases it would step and their work; rank 0 checks
    # the union is the whole sweep exactly once
    got = [None] * world
    dist.all_gather_object(got, (mine, sum(costs[i] for i in mine)))
    # per-case load rows (t, CD, CL) of this rank's cases, as a batch returns
    # them ([steps][cases][3]), gathered into case order on every rank
    steps = 5
    rows = np.array([[[s * 0.1, 1e-3 * c + s, -c - 1e-4 * s] for c in mine] for s in range(steps)])
    full = gather_case_rows(rows, mine, 256, dist)
    if rank == 0:
        seen = sorted(i for m, _ in got for i in m)
        np.save(os.path.join(out_dir, "seen.npy"), np.array(seen))
        np.save(os.path.join(out_dir, "work.npy"), np.array([w for _, w in got]))
        np.save(os.path.join(out_dir, "rows.npy"), full)
    dist.barrier()
    dist.destroy_process_group()


def test_case_sharding_world_size_two(tmp_path):
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_rank, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn")
    seen = np.load(tmp_path / "seen.npy")
    work = np.load(tmp_path / "work.npy")
    assert list(seen) == list(range(256))
    assert abs(work[0] - work[1]) / work.sum() < 0.02
    rows = np.load(tmp_path / "rows.npy")
    c = np.arange(256)
    expect = np.array([np.stack([np.full(256, s * 0.1), 1e-3 * c + s, -c - 1e-4 * s], -1) for s in range(5)])
    np.testing.assert_array_equal(rows, expect)


def test_gather_case_rows_single_process_needs_every_case():
    import pytest

    from uvlm_b200.batch import gather_case_rows

    rows = np.arange(12.0).reshape(2, 2, 3)
    np.testing.assert_array_equal(gather_case_rows(rows, [1, 0], 2), rows[:, ::-1])
    with pytest.raises(ValueError):
        gather_case_rows(rows, [0, 1], 3)


def _batch_create(cfg_changes=None, case_changes=None, n=1):
    import ctypes as C

    from uvlm_b200 import _capi

    L = _capi.lib()
    cfg = _capi.BatchConfig()
    L.uvlm_batch_config_default(C.byref(cfg))
    for k, v in (cfg_changes or {}).items():
        setattr(cfg, k, v)
    cases = (_capi.BatchCase * n)()
    for c in cases:
        c.chord, c.span, c.rows, c.cols, c.dt = 1.0, 4.0, 4, 8, 0.1
        c.forward_flight[0] = -1.0
        for k, v in (case_changes or {}).items():
            setattr(c, k, v)
    out = C.c_void_p(1)
    rc = L.uvlm_batch_create(C.byref(cfg), cases, n, C.byref(out))
    return rc, out.value, L.uvlm_global_last_error().decode()



@pytest.mark.parametrize("field,value", [
    ("precision", 5), ("advection", 2), ("max_steps", 0), ("refine_max_iter", -1), ("refine_tol", 0.0),
    ("nbody_tile", -2), ("nbody_tile", 3),
])
def test_batch_invalid_configuration_is_rejected_before_the_device(field, value):
    """uvlm_batch_create checks its configuration and every case before it
    looks for a device: UVLM_ERR_INVALID on any machine, no handle."""
    rc, h, msg = _batch_create({field: value})
    assert rc == 1 and h is None
    assert "invalid configuration" in msg


@pytest.mark.parametrize("field,value", [
    ("rows", 0), ("rows", 65), ("cols", 7), ("cols", 66), ("cols", 0), ("chord", 0.0), ("span", -1.0), ("dt", 0.0),
])
def test_batch_invalid_case_is_rejected_before_the_device(field, value):
    rc, h, msg = _batch_create(case_changes={field: value}, n=3)
    assert rc == 1 and h is None
    assert "every case needs" in msg


def test_batch_case_size_limit():
    # 32 x 40 = 1280 rings per case is above the one-CTA solve's 1024
    rc, h, msg = _batch_create(case_changes={"rows": 32, "cols": 40})
    assert rc == 1 and h is None
    assert "rows * cols <= 1024" in msg
