"""Host-side pieces of zdemx.autograd: the map from a world-frame rotation-vector gradient to the
gradient of the (normalised in the forward) quaternion, against torch autograd of a plain rotation."""
import numpy as np
import torch


def _rot(q):
    q = q / q.norm()
    w, x, y, z = q
    return torch.stack([torch.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)]),
                        torch.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)]),
                        torch.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)])])


def test_rotation_vector_grad_to_quaternion_grad():
    from zdemx.autograd import _rot_grad_to_quat

    rng = np.random.default_rng(0)
    for _ in range(20):
        q = torch.tensor(rng.normal(size=4) * rng.uniform(0.3, 3.0), dtype=torch.float64, requires_grad=True)
        v = torch.tensor(rng.normal(size=3), dtype=torch.float64)
        w = torch.tensor(rng.normal(size=3), dtype=torch.float64)
        f = w @ (_rot(q) @ v)
        f.backward()
        # d/dtheta of w . (exp(theta) R v) at 0 is (R v) x w
        g_theta = torch.linalg.cross(_rot(q.detach()) @ v, w)
        got = _rot_grad_to_quat(g_theta[None], q.detach()[None])[0]
        np.testing.assert_allclose(got.numpy(), q.grad.numpy(), rtol=1e-12, atol=1e-12)


def test_quat_exp_matches_axis_angle():
    from zdemx.autograd import quat_exp

    th = torch.tensor([[0.3, -0.2, 0.5], [0.0, 0.0, 0.0], [1e-10, 0.0, 0.0]], dtype=torch.float64)
    q = quat_exp(th)
    a = th.norm(dim=1)
    np.testing.assert_allclose(q[:, 0].numpy(), torch.cos(a / 2).numpy(), rtol=1e-15)
    np.testing.assert_allclose(q.norm(dim=1).numpy(), 1.0, rtol=1e-15)
    R = _rot(q[0])
    # rotation by the angle about the axis leaves the axis fixed
    np.testing.assert_allclose((R @ th[0]).numpy(), th[0].numpy(), rtol=1e-14)
