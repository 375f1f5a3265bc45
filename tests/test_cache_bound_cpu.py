"""The motion bound the DEM graph step's clearance cache relies on (k_cache_skip), checked numerically on
the host: a point v of a rigid body moves by at most |x - x0| + 2 |v| min(|q - q0|, |q + q0|) between two
poses (x0, q0) and (x, q) with unit quaternions, so two bodies whose such bounds add up to less than a
clearance cannot have closed it."""
import numpy as np


def _rot(q, v):
    w, x, y, z = q.T
    R = np.stack([np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
                  np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
                  np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1)], -2)
    return np.einsum("nij,nj->ni", R, v)


def _unit(a):
    return a / np.linalg.norm(a, axis=-1, keepdims=True)


def test_rotation_displacement_bound():
    rng = np.random.default_rng(12)
    n = 200_000
    q0 = _unit(rng.normal(size=(n, 4)))
    # small and large rotations, and the sign-flipped representation of a nearby rotation
    step = rng.normal(size=(n, 4)) * np.where(rng.random((n, 1)) < 0.5, 1e-3, 0.5)
    q = _unit(q0 + step)
    q[::3] *= -1.0
    v = rng.normal(size=(n, 3)) * rng.uniform(0.0, 2e-3, size=(n, 1))
    moved = np.linalg.norm(_rot(q, v) - _rot(q0, v), axis=1)
    qd = np.minimum(np.linalg.norm(q - q0, axis=1), np.linalg.norm(q + q0, axis=1))
    bound = 2.0 * np.linalg.norm(v, axis=1) * qd
    assert np.all(moved <= bound * (1 + 1e-12) + 1e-18)
    # the bound is within a factor of two of the motion for small rotations
    small = qd < 1e-2
    ratio = moved[small] / np.maximum(bound[small], 1e-300)
    assert ratio.max() > 0.9


def test_translation_and_rotation_add():
    rng = np.random.default_rng(13)
    n = 100_000
    q0 = _unit(rng.normal(size=(n, 4)))
    q = _unit(q0 + rng.normal(size=(n, 4)) * 1e-2)
    x0 = rng.normal(size=(n, 3))
    x = x0 + rng.normal(size=(n, 3)) * 1e-4
    v = rng.normal(size=(n, 3)) * 1e-3
    moved = np.linalg.norm((_rot(q, v) + x) - (_rot(q0, v) + x0), axis=1)
    qd = np.minimum(np.linalg.norm(q - q0, axis=1), np.linalg.norm(q + q0, axis=1))
    bound = np.linalg.norm(x - x0, axis=1) + 2.0 * np.linalg.norm(v, axis=1) * qd
    assert np.all(moved <= bound * (1 + 1e-12) + 1e-18)
