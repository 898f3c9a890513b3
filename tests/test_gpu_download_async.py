"""fe_download_async: a field copied out while later frames run equals what
fe_download returned for the same state, bit for bit, for contiguous,
32-byte-record and scalar fields, with the two snapshot slots rotating."""
import numpy as np
import pytest

from fluid_step import _abi, scene
from fluid_step.pipelines import Simulation

pytestmark = pytest.mark.gpu


def _pinned(shape, dtype=np.float32):
    import torch
    t = torch.empty(shape, dtype=torch.float32 if dtype == np.float32 else torch.int32,
                    pin_memory=True)
    return t, t.numpy().view(dtype)


def test_async_downloads_equal_synchronous_ones_across_frames():
    w = scene.workload("dam_break_16k")
    p = _abi.copy_params(w.params)
    p.mode = _abi.FE_MODE_FIXED
    p.solver = _abi.FE_SOLVER_TOLERANCE
    sim = Simulation(w.positions()[:10_001], p)
    d = sim.data
    fields = [_abi.FE_FIELD_POSITION_A, _abi.FE_FIELD_VELOCITY_A, _abi.FE_FIELD_POSITION_B,
              _abi.FE_FIELD_DENSITY]
    keep, pending = [], []
    for frame in range(5):
        sim.step(1)
        expect = {f: d.download(f) for f in fields}
        for f in fields:
            shape = expect[f].shape
            t, buf = _pinned(shape, expect[f].dtype.type)
            keep.append(t)
            pending.append((d.download_async(f, buf), buf, expect[f], frame, f))
        # later frames run while the copies are in flight
    sim.step(1)
    for ticket, buf, exp, frame, f in pending:
        d.download_wait(ticket)
        assert np.array_equal(buf.view(np.uint32), exp.view(np.uint32)), (frame, f)
    sim.close()


def test_async_download_into_pageable_memory_and_bad_tickets():
    w = scene.workload("dam_break_16k")
    sim = Simulation(w.positions()[:2000], w.params)
    sim.step(1)
    d = sim.data
    buf = np.empty((2000, 4), np.float32)
    t = d.download_async(_abi.FE_FIELD_VELOCITY_B, buf)
    d.download_wait(t)
    assert np.array_equal(buf, d.download(_abi.FE_FIELD_VELOCITY_B))
    assert d._lib.fe_download_wait(d.handle, t + 5) == _abi.FE_ERR_INVALID_ARGUMENT
    assert d._lib.fe_download_wait(d.handle, 0) == _abi.FE_ERR_INVALID_ARGUMENT
    sim.close()


def test_async_stats_equal_the_waiting_read_across_frames():
    """fe_read_stats_async captures a frame's stats in stream order: waited
    for a frame later, they equal what fe_step returned for that frame."""
    w = scene.workload("dam_break_16k")
    p = _abi.copy_params(w.params)
    p.mode, p.solver, p.use_cfl, p.dt = (_abi.FE_MODE_FIXED, _abi.FE_SOLVER_TOLERANCE, 1, 0.004)
    ref = Simulation(w.positions()[:8000], p)
    sim = Simulation(w.positions()[:8000], p)
    lib, h = sim.data._lib, sim.data.handle
    expect, tickets = [], []
    for _ in range(6):
        expect.append(ref.step(1))
        assert lib.fe_step(h, 1, 0, None) == 0
        tickets.append(sim.data.read_stats_async())
        if len(tickets) >= 2:   # the previous frame's capture, a frame later
            got = sim.data.stats_wait(tickets[-2])
            _same_stats(got, expect[-2])
    _same_stats(sim.data.stats_wait(tickets[-1]), expect[-1])
    assert lib.fe_stats_wait(h, tickets[-3], None) == _abi.FE_ERR_INVALID_ARGUMENT
    bad = _abi.FeStats()
    import ctypes
    assert lib.fe_stats_wait(h, tickets[-3], ctypes.byref(bad)) == _abi.FE_ERR_INVALID_ARGUMENT
    ref.close()
    sim.close()


def _same_stats(a, b):
    for name, _ in _abi.FeStats._fields_:
        if name in ("reserved",):
            continue
        va, vb = getattr(a, name), getattr(b, name)
        assert va == vb or (va != va and vb != vb), (name, va, vb)
