"""The camera builders of the C ABI against the reference's own camera classes: the
description the device receives (Camera::describeGpu, src/camera/camera.h:17-29) is bit-equal to
the reference's for the pinhole, thin-lens (round and polygonal aperture) and orthographic
cameras."""
import pytest


@pytest.mark.parametrize("make", [
    lambda pe: pe.PerspectiveCamera((1.0, 2.0, -5.0), (0.0, 0.5, 0.0), (0.0, 1.0, 0.0), 40.0, 1.5),
    lambda pe: pe.ThinLensCamera((1.0, 2.0, -5.0), (0.0, 0.5, 0.0), (0.0, 1.0, 0.0), 40.0, 1.5, 0.2, 4.5),
    lambda pe: pe.ThinLensCamera((1.0, 2.0, -5.0), (0.0, 0.5, 0.0), (0.0, 1.0, 0.0), 35.0, 1.0, 0.1, 3.0, 6, 15.0),
    lambda pe: pe.OrthographicCamera((1.0, 2.0, -5.0), (0.0, 0.5, 0.0), (0.0, 1.0, 0.0), 3.0, 1.5),
], ids=["pinhole", "thin-lens", "thin-lens-hexagon", "orthographic"])
def test_camera_description_matches_reference(pe, oracle, make):
    cam = make(pe)
    mine = cam.describe_gpu()
    ref = oracle.describe_reference_camera(cam)
    assert bytes(mine) == bytes(ref)
