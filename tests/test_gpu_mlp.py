"""The tensor-core MLP (forward, backward, Adam) against the FP64 reference.

The kernels round operands to BF16 where they store BF16 and accumulate in
FP32 on the tensor cores; the reference (oracle/mlp_ref.py) applies the same
BF16 roundings in FP64.  Tolerances: outputs within 2e-2 absolute on
standardised targets of order 1, gradients within 2 % relative L2 with
cosine similarity above 0.999.
"""
import ctypes

import numpy as np
import pytest

import mlp_ref
from fluid_step import _abi

pytestmark = pytest.mark.gpu


class Model:
    def __init__(self, seed=1):
        self.lib = _abi.load_library()
        self.h = ctypes.c_void_p()
        _abi.check(self.lib, self.lib.fe_model_create(seed, 0, ctypes.byref(self.h)), "create")

    def params(self):
        p = np.empty(_abi.FE_MODEL_PARAMS, np.float32)
        _abi.check(self.lib, self.lib.fe_model_get_parameters(
            self.h, p.ctypes.data_as(ctypes.c_void_p), p.size), "get")
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        _abi.check(self.lib, self.lib.fe_model_set_parameters(
            self.h, p.ctypes.data_as(ctypes.c_void_p), p.size), "set")

    def close(self):
        self.lib.fe_model_destroy(self.h)


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def ptr(t):
    """Device address of a tensor the caller keeps referenced."""
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("n", [1, 127, 128, 129, 1000, 70_000])
def test_forward_matches_reference(n):
    import torch
    m = Model(seed=3)
    rng = np.random.default_rng(n)
    x = rng.normal(0, 1, (n, 12)).astype(np.float32)
    xd, yd = dev(x), torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    _abi.check(m.lib, m.lib.fe_model_forward(m.h, ptr(xd), ptr(yd), n, None), "forward")
    torch.cuda.synchronize()
    ref, _ = mlp_ref.forward(m.params(), x)
    got = yd.cpu().numpy()
    assert np.max(np.abs(got - ref)) < 2e-2, np.max(np.abs(got - ref))
    m.close()


@pytest.mark.parametrize("n", [128, 300, 5000])
def test_gradients_match_reference(n):
    m = Model(seed=5)
    rng = np.random.default_rng(n + 1)
    x = rng.normal(0, 1, (n, 12)).astype(np.float32)
    y = rng.normal(0, 1, (n, 2)).astype(np.float32)
    g = np.empty(_abi.FE_MODEL_PARAMS, np.float32)
    loss = ctypes.c_float()
    xd, yd = dev(x), dev(y)          # keep the device tensors alive across the call
    _abi.check(m.lib, m.lib.fe_model_gradients(m.h, ptr(xd), ptr(yd), n,
                                               g.ctypes.data_as(ctypes.c_void_p),
                                               ctypes.byref(loss)), "gradients")
    ref, ref_loss = mlp_ref.gradients(m.params(), x, y)
    report = {}
    for name, sl in [("w1", slice(0, mlp_ref.W1)), ("w2", slice(mlp_ref.W1, mlp_ref.W1 + mlp_ref.W2)),
                     ("w3", slice(mlp_ref.W1 + mlp_ref.W2, mlp_ref.NW)),
                     ("b1", slice(mlp_ref.NW, mlp_ref.NW + 64)),
                     ("b2", slice(mlp_ref.NW + 64, mlp_ref.NW + 128)),
                     ("b3", slice(mlp_ref.NW + 128, mlp_ref.NP))]:
        a, b = g[sl].astype(np.float64), ref[sl]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30))
        report[name] = (round(rel, 5), round(cos, 6))
    for name, (rel, cos) in report.items():
        assert rel < 2e-2 and cos > 0.999, report
    assert abs(loss.value - ref_loss) <= 2e-2 * ref_loss
    m.close()


def test_training_reduces_loss():
    """Adam on a smooth synthetic regression: the loss falls by 10x."""
    import torch
    m = Model(seed=7)
    rng = np.random.default_rng(9)
    x = rng.normal(0, 1, (65_536, 12)).astype(np.float32)
    y = np.stack([np.tanh(x[:, 0] + 0.5 * x[:, 1] * x[:, 2]),
                  np.sin(x[:, 3]) - 0.3 * x[:, 4]], axis=1).astype(np.float32)
    xd, yd = dev(x), dev(y)
    losses = []
    bs = 4096
    for step in range(400):
        i0 = (step * bs) % x.shape[0]
        loss = ctypes.c_float()
        _abi.check(m.lib, m.lib.fe_model_train_step(
            m.h, ctypes.c_void_p(xd.data_ptr() + i0 * 48), ctypes.c_void_p(yd.data_ptr() + i0 * 8),
            bs, 3e-3, 0.0, None, ctypes.byref(loss)), "train_step")
        losses.append(loss.value)
    flags = ctypes.c_uint32()
    m.lib.fe_model_read_flags(m.h, ctypes.byref(flags))
    assert flags.value == 0
    assert np.mean(losses[-20:]) < 0.1 * np.mean(losses[:5]), (losses[:5], losses[-5:])
    m.close()
