"""The allocation-free InducedVelocity entry point (needs a B200).

uvlm_sheet_induced_velocity_noalloc serves callers that cannot call
cudaMalloc: loops in which an allocation would synchronise the device, and
frameworks that own the whole device-memory budget and hand the library only
buffers they allocated.  It takes device pointers and keeps all scratch in a
fixed device array inside the library.  These tests call it through the C-ABI
twice in a row (the array keeps the previous call's contents) and compare each
result with the allocating entry point and with the FP64 CPU oracle, within
the tolerances of the other N-body tests.  This file is collected last so that
a failure here never hides the others.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))

_P = C.POINTER(C.c_double)


def _sheet(rng, num, rows, cols):
    base = np.stack(np.meshgrid(np.linspace(0, 1, rows + 1), np.linspace(-2, 2, cols + 1), indexing="ij"), -1)
    pos = np.zeros((num, rows + 1, cols + 1, 3))
    for n in range(num):
        pos[n, ..., :2] = base + 0.02 * rng.standard_normal(base.shape)
        pos[n, ..., 0] += 1.3 * n
        pos[n, ..., 2] = 0.05 * rng.standard_normal(base.shape[:2]) + 0.2 * n
    return pos, rng.standard_normal((num, rows, cols))


def _noalloc(pos, gamma, targets, precision, fill=float("nan")):
    import torch

    import uvlm_b200 as U

    dev = torch.device("cuda:0")
    d_pos = torch.from_numpy(np.ascontiguousarray(pos)).to(dev)
    d_g = torch.from_numpy(np.ascontiguousarray(gamma)).to(dev)
    d_t = torch.from_numpy(np.ascontiguousarray(targets)).to(dev)
    d_out = torch.full_like(d_t, fill)
    stream = torch.cuda.current_stream()
    num, rows, cols = gamma.shape
    rc = U.lib().uvlm_sheet_induced_velocity_noalloc(
        C.cast(d_pos.data_ptr(), _P), C.cast(d_g.data_ptr(), _P), num, rows, cols, C.cast(d_t.data_ptr(), _P),
        targets.shape[0], C.cast(d_out.data_ptr(), _P), {"fp64": 0, "mixed": 1}[precision],
        C.c_void_p(stream.cuda_stream))
    U._capi.check(rc)
    stream.synchronize()
    return d_out.cpu().numpy()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 2e-5)])
def test_noalloc_matches_allocating_entry_point_and_oracle_twice(precision, tol):
    import pyoracle

    import uvlm_b200 as U

    rng = np.random.default_rng(11)
    calls = [(2, 9, 40, 700), (1, 20, 128, 3000)]  # second call: other shapes, other values
    for num, rows, cols, nt in calls:
        pos, gamma = _sheet(rng, num, rows, cols)
        targets = np.concatenate([rng.uniform(-1, 3, size=(nt, 3)), pos.reshape(-1, 3)[:50]])
        got = _noalloc(pos, gamma, targets, precision)
        ref = U.InducedVelocity(targets, pos, gamma, precision=precision)
        orc = pyoracle.sheet_induced_velocity(pos, gamma, targets)
        scale = np.max(np.abs(orc))
        assert np.all(np.isfinite(got))
        assert np.max(np.abs(got - ref)) <= tol * scale
        assert np.max(np.abs(got - orc)) <= tol * scale


@pytest.mark.parametrize("shape", [(0, 4, 8), (1, 0, 8), (1, 4, 0)])
def test_noalloc_empty_sheet_gives_zeros(shape):
    num, rows, cols = shape
    pos = np.zeros((num, rows + 1, cols + 1, 3))
    gamma = np.zeros((num, rows, cols))
    targets = np.random.default_rng(5).uniform(-1, 1, size=(300, 3))
    got = _noalloc(pos, gamma, targets, "fp64", fill=7.0)
    assert np.array_equal(got, np.zeros_like(targets))


def test_noalloc_rejects_requests_beyond_its_scratch():
    import uvlm_b200 as U

    pos, gamma = _sheet(np.random.default_rng(3), 1, 4, 8)
    targets = np.zeros((2_000_000, 3))  # 6 x 16 MB of SoA vectors alone exceed the 32 MiB array
    with pytest.raises(U.UVLMError) as ei:
        _noalloc(pos, gamma, targets, "fp64")
    assert ei.value.code == 6
    assert "scratch" in str(ei.value)
