"""gd_energy_poses_noalloc: pose energies staged in the library's fixed device
array instead of allocated buffers, for callers whose device memory belongs
to another allocator and that therefore cannot allocate on their scoring path.
Called through the C-ABI and compared bit for bit with gd_energy_poses on two
calls in a row (different sizes and conformations, so the second call cannot
lean on what the first left in the shared array), and checked to leave the
device's free memory and its stream-ordered pool untouched. The file sorts
last so that it also runs after every other GPU test in the same process."""
import ctypes as C

import numpy as np
import pytest

from gpudock_b200 import abi, lib, synth

pytestmark = pytest.mark.gpu

MAX_POSES = 16384  # GD_NOALLOC_MAX_POSES in include/gpudock.h


def _noalloc_fn():
    fn = lib.load().gd_energy_poses_noalloc
    P = C.c_void_p
    fn.argtypes = [P, P, C.c_int, C.c_int, C.c_int, abi.f32p, abi.f32p, abi.f64p]
    fn.restype = C.c_int
    return fn


def _noalloc(fn, ctx, d, poses, prt_conf, lig_conf, raw=True):
    poses = np.ascontiguousarray(poses, np.float32).reshape(-1, 6)
    n = poses.shape[0]
    terms = np.full((n, abi.NTERM), np.nan, np.float32)
    rw = np.full((n, abi.NRAW), np.nan, np.float64) if raw else None
    lib.check(fn(ctx.h, d.h, prt_conf, lig_conf, n, abi._ptr(poses, C.c_float),
                 abi._ptr(terms, C.c_float), abi._ptr(rw, C.c_double)),
              "gd_energy_poses_noalloc")
    return terms, rw


def test_noalloc_matches_allocating_entry_point():
    fn = _noalloc_fn()
    ctx = lib.Context(0)
    cx = synth.make_complex(synth.ComplexSpec(pnp=1800, lna=30, n_prt=2, n_lig=3), seed=77)
    d = lib.DeviceComplex(ctx, cx)
    rng = np.random.default_rng(5)
    calls = [(synth.random_poses(rng, 700, box=4.0), 0, 0),
             (synth.random_poses(rng, 133, box=6.0), 1, 2)]
    for poses, pc, lc in calls:
        t_ref, r_ref = d.energy_poses(poses, prt_conf=pc, lig_conf=lc)
        t_na, r_na = _noalloc(fn, ctx, d, poses, pc, lc)
        assert np.array_equal(t_na, t_ref)
        assert np.array_equal(r_na, r_ref)
    # without the raw sums
    poses, pc, lc = calls[1]
    t_na, r_na = _noalloc(fn, ctx, d, poses, pc, lc, raw=False)
    assert r_na is None
    assert np.array_equal(t_na, d.energy_poses(poses, prt_conf=pc, lig_conf=lc)[0])
    d.close()
    ctx.close()


def _memory_state():
    """(free device bytes, default pool's used and reserved bytes) of device 0."""
    from cuda.bindings import runtime as rt
    err, free, _total = rt.cudaMemGetInfo()
    assert err == rt.cudaError_t.cudaSuccess
    err, pool = rt.cudaDeviceGetDefaultMemPool(0)
    assert err == rt.cudaError_t.cudaSuccess
    vals = []
    for attr in (rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent,
                 rt.cudaMemPoolAttr.cudaMemPoolAttrReservedMemCurrent,
                 rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh):
        err, v = rt.cudaMemPoolGetAttribute(pool, attr)
        assert err == rt.cudaError_t.cudaSuccess
        vals.append(int(v))
    return int(free), vals, pool


def test_noalloc_allocates_nothing():
    from cuda.bindings import driver
    from cuda.bindings import runtime as rt
    fn = _noalloc_fn()
    ctx = lib.Context(0)
    cx = synth.make_complex(synth.ComplexSpec(pnp=900, lna=20), seed=79)
    d = lib.DeviceComplex(ctx, cx)
    poses = synth.random_poses(np.random.default_rng(7), 4000, box=3.0)
    t_ref, r_ref = d.energy_poses(poses)  # the allocating path, first
    _noalloc(fn, ctx, d, poses, 0, 0)
    assert rt.cudaDeviceSynchronize()[0] == rt.cudaError_t.cudaSuccess
    free0, (used0, res0, _), pool = _memory_state()
    # the pool's high-water mark from here on shows any allocation, even one
    # freed again before the call returns
    err, = rt.cudaMemPoolSetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh,
                                      driver.cuuint64_t(0))
    assert err == rt.cudaError_t.cudaSuccess
    t_na, r_na = _noalloc(fn, ctx, d, poses, 0, 0)
    assert rt.cudaDeviceSynchronize()[0] == rt.cudaError_t.cudaSuccess
    free1, (used1, res1, high1), _ = _memory_state()
    assert np.array_equal(t_na, t_ref) and np.array_equal(r_na, r_ref)
    assert free1 == free0
    assert (used1, res1) == (used0, res0)
    assert high1 <= used0
    d.close()
    ctx.close()


def test_noalloc_limits():
    fn = _noalloc_fn()
    ctx = lib.Context(0)
    cx = synth.make_complex(synth.ComplexSpec(pnp=600, lna=12), seed=78)
    d = lib.DeviceComplex(ctx, cx)
    # the largest call the array holds
    poses = synth.random_poses(np.random.default_rng(6), MAX_POSES, box=3.0)
    t_na, r_na = _noalloc(fn, ctx, d, poses, 0, 0)
    t_ref, r_ref = d.energy_poses(poses)
    assert np.array_equal(t_na, t_ref) and np.array_equal(r_na, r_ref)
    # one pose more is refused before anything runs
    big = np.zeros((MAX_POSES + 1, 6), np.float32)
    terms = np.zeros((MAX_POSES + 1, abi.NTERM), np.float32)
    st = fn(ctx.h, d.h, 0, 0, MAX_POSES + 1, abi._ptr(big, C.c_float),
            abi._ptr(terms, C.c_float), None)
    assert st == abi.GD_EINVAL
    assert "exceeds" in lib.last_error()
    # an empty call succeeds whatever the indices, as gd_energy_poses does
    assert fn(ctx.h, d.h, 0, 0, 0, None, None, None) == abi.GD_OK
    assert fn(ctx.h, d.h, 5, 7, 0, None, None, None) == abi.GD_OK
    st = fn(ctx.h, d.h, 1, 0, 4, abi._ptr(big, C.c_float), abi._ptr(terms, C.c_float), None)
    assert st == abi.GD_EINVAL
    d.close()
    ctx.close()
