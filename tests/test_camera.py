"""strelka_camera_lookat: the per-job cameras of the batched launch."""
import ctypes as C

import numpy as np
import pytest

from strelka_b200 import abi, scenes


def test_look_at_sets_camera_and_keeps_the_rest():
    s = scenes.cornell(32, 24, sphere_levels=1)
    p = s.look_at(17, 11, (0.3, 0.6, 2.2), (0.5, 0.4, 0.0), 50.0, spp=3, maxDepth=6, frameNumber=9)
    assert (p.dimension[0], p.dimension[1]) == (17, 11)
    assert p.invDimension[0] == np.float32(1 / 17) and p.invDimension[1] == np.float32(1 / 11)
    assert (p.spp, p.maxDepth, p.frameNumber) == (3, 6, 9)
    assert p.numLights == s.camera.numLights
    m = np.array(p.viewToWorld.m, np.float64).reshape(4, 4)  # column-major: column c = m[c]
    eye = m[3, :3]
    assert np.allclose(eye, (0.3, 0.6, 2.2), atol=1e-5)
    assert np.allclose([p.camPos.x, p.camPos.y, p.camPos.z], (0.3, 0.6, 2.2))
    # the camera looks down its -z axis toward the target
    fwd = -m[2, :3]
    d = np.array([0.2, -0.2, -2.2]) / np.linalg.norm([0.2, -0.2, -2.2])
    assert np.allclose(fwd / np.linalg.norm(fwd), d, atol=1e-5)


def test_look_at_rejects_degenerate():
    s = scenes.cornell(8, 8, sphere_levels=1)
    with pytest.raises(abi.StrelkaError):
        s.look_at(8, 8, (1, 1, 1), (1, 1, 1))
    with pytest.raises(abi.StrelkaError):
        s.look_at(0, 8, (0, 0, 1), (0, 0, 0))
