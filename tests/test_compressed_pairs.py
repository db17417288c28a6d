"""The compressed OBVH's transformation pairs derived from an OBB tree
(obvh_b200.bvh.compressed_pairs_from_obbs, host code): the axis-angle
columns rebuild each child box's rotation, and they agree with the oracle's
restatement (oracle.bvh.compressed_pairs) wherever that one is defined
(rotations away from pi)."""
import numpy as np

from obvh_b200 import bvh
from oracle import bvh as ref


def _rodrigues(axis, angle):
    k = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    return np.eye(3) + np.sin(angle) * k + (1 - np.cos(angle)) * (k @ k)


def _tree(boxes):
    """A root over two leaves 1 and 2, with the given kr_obb3 rows for nodes 0..2."""
    nodes = np.zeros(3, ref.NODE)
    nodes["left"][0], nodes["right"][0] = 1, 2
    return nodes, np.asarray(boxes, np.float32)


def _box(rot, mid, ext, scale=(1.0, 1.0, 1.0)):
    o = np.zeros(15, np.float32)
    o[0:3] = mid
    o[3:12] = (rot.T * np.asarray(scale)[:, None]).ravel()  # rows: the (scaled) box axes
    o[12:15] = ext
    return o


def test_pairs_rebuild_the_rotation_and_match_the_oracle():
    rng = np.random.default_rng(3)
    for _ in range(200):
        axis = rng.normal(size=3)
        axis /= np.linalg.norm(axis)
        angle = rng.uniform(0.05, 3.0)
        rot = _rodrigues(axis, angle)
        mid, ext = rng.uniform(-5, 5, 3), rng.uniform(0.01, 2, 3)
        scale = (1.0, 1.0, rng.uniform(0.1, 3.0))   # a leaf's third axis is not normalised
        nodes, obbs = _tree([np.zeros(15), _box(rot, mid, ext, scale), _box(np.eye(3), mid, ext)])
        got = bvh.compressed_pairs_from_obbs(nodes, obbs)
        want = ref.compressed_pairs(nodes, obbs)
        assert got.shape == want.shape == (1, 32)
        np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-5)
        a, t = got[0, 0:3].astype(np.float64), float(got[0, 3]) * np.pi
        np.testing.assert_allclose(_rodrigues(a, t), rot, atol=2e-5)
        np.testing.assert_allclose(got[0, 8:11], 2 * ext * np.asarray(scale), rtol=1e-5)


def test_half_turns_keep_their_axis():
    """At an angle of pi the skew part vanishes; the axis comes from R + I."""
    rng = np.random.default_rng(4)
    for _ in range(50):
        axis = rng.normal(size=3)
        axis /= np.linalg.norm(axis)
        rot = _rodrigues(axis, np.pi)
        nodes, obbs = _tree([np.zeros(15), _box(rot, np.zeros(3), np.ones(3)), _box(np.eye(3), np.zeros(3), np.ones(3))])
        got = bvh.compressed_pairs_from_obbs(nodes, obbs)
        a, t = got[0, 0:3].astype(np.float64), float(got[0, 3]) * np.pi
        np.testing.assert_allclose(_rodrigues(a, t), rot, atol=1e-3)


def test_left_handed_frames_become_right_handed():
    rot = _rodrigues(np.array([0.0, 0.0, 1.0]), 0.7)
    mirror = rot.copy()
    mirror[:, 2] *= -1.0   # det -1
    nodes, obbs = _tree([np.zeros(15), _box(mirror, np.zeros(3), np.ones(3)), _box(np.eye(3), np.zeros(3), np.ones(3))])
    got = bvh.compressed_pairs_from_obbs(nodes, obbs)
    a, t = got[0, 0:3].astype(np.float64), float(got[0, 3]) * np.pi
    np.testing.assert_allclose(_rodrigues(a, t), rot, atol=1e-5)
