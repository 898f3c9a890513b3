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
