"""The water pass (raymarch.frag) into a headless image, against the
oracle's restatement of the shader.  Tolerance: the device and host
transcendentals (exp, pow, atan2, asin) differ in the last bits, which can
move a ray's surface test across the threshold; so (1) hit/miss (alpha)
agrees on >= 99.5 % of pixels, (2) where both hit, >= 99 % of pixels agree
within 2e-3 in every colour channel and the mean difference is <= 2e-4."""
import numpy as np
import pytest

from fluid_step import _abi, camera, scene
from fluid_step.pipelines import Simulation

pytestmark = pytest.mark.gpu


def _compare(got, ref):
    a_got, a_ref = got[..., 3] > 0, ref[..., 3] > 0
    assert (a_got == a_ref).mean() >= 0.995, (a_got != a_ref).sum()
    both = a_got & a_ref
    assert both.sum() > 100
    d = np.abs(got[..., :3] - ref[..., :3])[both].max(axis=1)
    assert (d <= 2e-3).mean() >= 0.99, np.sort(d)[-10:]
    assert d.mean() <= 2e-4
    assert not np.isnan(got).any()


@pytest.mark.parametrize("eye,size", [((0.0, 2.0, -4.5), (160, 90)),
                                      ((2.5, 3.0, -3.0), (200, 200)),
                                      ((-0.5, 1.5, 0.0), (128, 72))])    # inside the box
def test_raymarch_matches_oracle(oracle_mod, eye, size):
    p, pos, _ = scene.app_scene()
    p.sort_algorithm = _abi.FE_SORT_RADIX
    sim = Simulation(pos, p)
    for _ in range(5):
        sim.step(1)
    grid = sim.data.splat_density()
    sky = camera.gradient_sky()
    sim.data.set_skybox(sky)
    cam = camera.make_camera(eye, (-0.3, 1.2, 0.0), *size)
    got = sim.data.raymarch(cam)
    ref = oracle_mod.raymarch(grid, sky, cam, p.box_min, p.box_max)
    _compare(got, ref)
    sim.close()


def test_raymarch_errors():
    p, pos, _ = scene.app_scene()
    sim = Simulation(pos[:1000], p)
    lib = sim.data._lib
    cam = camera.make_camera((0, 2, -4), (0, 1, 0), 32, 32)
    import ctypes
    assert lib.fe_raymarch(sim.data.handle, ctypes.byref(cam)) == _abi.FE_ERR_INVALID_ARGUMENT
    sim.data.splat_density()
    assert lib.fe_raymarch(sim.data.handle, ctypes.byref(cam)) == _abi.FE_ERR_INVALID_ARGUMENT
    sim.data.set_skybox(camera.gradient_sky(8, 4))
    cam.width = 0
    assert lib.fe_raymarch(sim.data.handle, ctypes.byref(cam)) == _abi.FE_ERR_INVALID_ARGUMENT
    sim.close()
