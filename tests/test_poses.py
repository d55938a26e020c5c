"""Quaternion poses to move vectors (gd_poses_from_quaternions), on CPU.

The move vector's angles must rebuild the quaternion's rotation through the
ZYX matrix Move_d uses (move_d.cu:90-105), including at gimbal lock, for any
scale and sign of the quaternion."""
import numpy as np
import pytest

from gpudock_b200 import abi, lib


def _rot_from_move(m):
    """R = Rz(m3) Ry(m4) Rx(m5), element by element as move_d.cu:90-105."""
    s1, c1 = np.sin(m[:, 3]), np.cos(m[:, 3])
    s2, c2 = np.sin(m[:, 4]), np.cos(m[:, 4])
    s3, c3 = np.sin(m[:, 5]), np.cos(m[:, 5])
    return np.stack([c1 * c2, c1 * s2 * s3 - c3 * s1, s1 * s3 + c1 * c3 * s2,
                     c2 * s1, c1 * c3 + s1 * s2 * s3, c3 * s1 * s2 - c1 * s3,
                     -s2, c2 * s3, c2 * c3], axis=1).reshape(-1, 3, 3)


def _rot_from_quat(q):
    q = q / np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
                     2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                     2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)],
                    axis=1).reshape(-1, 3, 3)


def _quat_mul(a, b):
    aw, ax, ay, az = a
    bw, bx, by, bz = b
    return np.array([aw * bw - ax * bx - ay * by - az * bz, aw * bx + ax * bw + ay * bz - az * by,
                     aw * by - ax * bz + ay * bw + az * bx, aw * bz + ax * by - ay * bx + az * bw])


def _axis(ang, k):
    q = np.zeros(4)
    q[0], q[1 + k] = np.cos(ang / 2), np.sin(ang / 2)
    return q


def test_random_rotations():
    rng = np.random.Generator(np.random.PCG64(7))
    n = 4096
    q = rng.normal(size=(n, 4))
    q *= rng.uniform(0.01, 100.0, size=(n, 1)) / np.linalg.norm(q, axis=1, keepdims=True)
    t = rng.uniform(-20, 20, size=(n, 3))
    qp = np.concatenate([t, q], axis=1).astype(np.float32)
    m = lib.poses_from_quaternions(qp)
    assert m.dtype == np.float32 and m.shape == (n, 6)
    assert np.array_equal(m[:, :3], qp[:, :3])
    err = np.abs(_rot_from_move(m.astype(np.float64)) - _rot_from_quat(qp[:, 3:].astype(np.float64)))
    assert err.max() < 1e-6, err.max()
    assert (np.abs(m[:, 4]) <= np.float32(np.pi / 2)).all()
    # q and -q are the same rotation and give the same angles
    qn = qp.copy()
    qn[:, 3:] *= -1
    assert np.array_equal(lib.poses_from_quaternions(qn), m)


@pytest.mark.parametrize("pitch", [np.pi / 2, -np.pi / 2])
def test_gimbal_lock(pitch):
    rows = []
    for yaw, roll in [(0.0, 0.0), (0.3, -1.1), (2.5, 2.9), (-3.0, 0.7)]:
        q = _quat_mul(_quat_mul(_axis(yaw, 2), _axis(pitch, 1)), _axis(roll, 0))
        rows.append(np.concatenate([[1.0, 2.0, 3.0], q]))
    qp = np.asarray(rows, np.float32)
    m = lib.poses_from_quaternions(qp)
    err = np.abs(_rot_from_move(m.astype(np.float64)) - _rot_from_quat(qp[:, 3:].astype(np.float64)))
    assert err.max() < 1e-6, err.max()
    assert np.allclose(m[:, 4], pitch, atol=1e-3)


def test_identity_and_errors():
    m = lib.poses_from_quaternions(np.float32([[0.5, -0.5, 1.0, 1.0, 0.0, 0.0, 0.0]]))
    assert np.array_equal(m, np.float32([[0.5, -0.5, 1.0, 0.0, 0.0, 0.0]]))
    assert lib.poses_from_quaternions(np.zeros((0, 7), np.float32)).shape == (0, 6)
    for bad in ([0, 0, 0, 0, 0, 0, 0], [0, 0, 0, np.nan, 1, 0, 0], [np.inf, 0, 0, 1, 0, 0, 0]):
        with pytest.raises(lib.GdError) as e:
            lib.poses_from_quaternions(np.float32([bad]))
        assert e.value.status == abi.GD_EINVAL
