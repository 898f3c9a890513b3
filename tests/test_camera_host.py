"""The headless camera helper (no GPU): the centre pixel's ray points at the
target and rows run top to bottom."""
import numpy as np

from fluid_step.camera import make_camera


def _ray(cam, px, py):
    m = np.frombuffer(bytes(cam.inv_view_proj), np.float32).reshape(4, 4).T  # column-major
    nx = (px + 0.5) / cam.width * 2 - 1
    ny = (py + 0.5) / cam.height * 2 - 1
    w = m @ np.array([nx, ny, 1.0, 1.0])
    d = w[:3] / w[3] - np.frombuffer(bytes(cam.camera_pos), np.float32)
    return d / np.linalg.norm(d)


def test_centre_ray_points_at_target():
    eye, target = np.array([0.0, 2.0, -4.0]), np.array([0.0, 1.0, 0.0])
    cam = make_camera(eye, target, 101, 51)
    d = _ray(cam, 50, 25)
    want = (target - eye) / np.linalg.norm(target - eye)
    assert np.dot(d, want) > 0.9999


def test_rows_run_top_to_bottom_and_columns_left_to_right():
    cam = make_camera((0.0, 0.0, -5.0), (0.0, 0.0, 0.0), 64, 64)
    assert _ray(cam, 32, 0)[1] > 0 > _ray(cam, 32, 63)[1]        # row 0 looks up
    # looking along +z with y up, screen-right is -x in a right-handed frame
    assert _ray(cam, 63, 32)[0] < 0 < _ray(cam, 0, 32)[0]
