"""The volume-observer oracle against an affine field (CPU): the reference's
independent check (tests/test_volume.py:13-62) applied to oracle.volume."""

import numpy as np

from oracle.volume import OFFSETS, record_volume


def affine_fields(shape):
    xyz = np.indices(shape).astype(float)
    fields = []
    for c in range(6):
        position = xyz + OFFSETS[c].astype(float)[:, None, None, None]
        fields.append((position[0] + 2 * position[1] - 3 * position[2] + c).astype("f").ravel())
    return np.array(fields[:3]), 4 * np.array(fields[3:]), 2 * np.array(fields[3:])


def test_oracle_affine_sampling_and_time_centering():
    shape = (7, 8, 9)
    e, h, prev = affine_fields(shape)
    points = np.array([[2.1, 3.4, 4.2], [1.3, 2.5, 3.7], [4.8, 5.1, 6.3]], "f")
    weights = np.array([[0, 0], [0.2, 0.3]], "f")
    out = np.zeros((6, len(points)), complex)
    record_volume(e, h, prev, points, weights, 0, out, shape, 1)
    assert not out.any()  # before the window's first step
    record_volume(e, h, prev, points, weights, 1, out, shape, 1)
    for c in range(6):
        v = points[:, 0].astype(float) + 2 * points[:, 1] - 3 * points[:, 2] + c
        np.testing.assert_allclose(out[c], v * (1 if c < 3 else 3) * (0.2 + 0.3j), rtol=2e-6, atol=3e-6)
