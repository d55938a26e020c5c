"""Failure detection and checkpoint / resume on the GPU.

1. Bounded waits run out: with the persistent schedule a CTA that continues a
   unit waits (bounded) for the CTA that ran the unit's earlier steps.  The
   test hook gd_ctx_set_wait_test makes every such wait target a step that is
   never reached, with a limit of 10^4 polls, so each wait runs out; the
   kernel records the error and finishes, the host sees GD_ETIMEDOUT, the
   error word is cleared, and the context keeps working.  No kernel faults,
   traps or hangs: the waits end by their limit.
2. A run snapshotted at step 50 and restored into a new handle continues
   bit for bit as the same run without the break (the reference keeps no
   random state in its dumps, util_d.cu:85-92, and cannot resume).
3. Device allocations that fail (injected with gd_ctx_set_alloc_fail) give
   GD_ENOMEM, free what the failing call had allocated, and leave the
   context and the server usable (the reference exits on any CUDA error,
   include_cuda/cutil_yeah.h:26-47)."""
import numpy as np
import pytest

from gpudock_b200 import abi, lib, synth

pytestmark = pytest.mark.gpu


def _same(a, b, rec_from=0):
    assert np.array_equal(a.energy, b.energy)
    assert np.array_equal(a.movematrix, b.movematrix)
    assert np.array_equal(a.idx_tmp, b.idx_tmp)
    assert np.array_equal(a.acs_mc, b.acs_mc)
    assert np.array_equal(a.acs_temp_exchg, b.acs_temp_exchg)
    assert a.ac_mc == b.ac_mc and a.ac_temp_exchg == b.ac_temp_exchg
    if a.record is not None:
        assert np.array_equal(a.record[:, rec_from:], b.record[:, rec_from:])


def _complex(case):
    if case == "fused":  # 8 temperatures: exchange inside the kernel
        return synth.make_complex(synth.ComplexSpec(pnp=900, lna=24, n_prt=3, n_lig=8),
                                  seed=901), 8
    return synth.make_complex(synth.ComplexSpec(pnp=700, lna=17, n_prt=2, n_lig=10),
                              seed=902), 6  # exchange kernel, captured interval


def test_bounded_wait_runs_out_and_reports_timeout():
    ctx = lib.Context(0)
    ctx.set_split(1)
    cx, n_tmp = _complex("fused")  # 6 units of 32 replicas
    d = lib.DeviceComplex(ctx, cx)
    _, mb = lib.set_temperature(n_tmp, 0.004, 0.04)
    # 4 persistent CTAs for 6 units x 40 steps: units are cut mid-run, so
    # some pieces wait on another CTA
    ctx.set_schedule(abi.SCHED_PERSISTENT, 4)
    ctx.set_wait_test(10_000, True)
    r = lib.Remc(d, 40, 10, mb, seed=5, flags=abi.MC_EXCHANGE)
    r.init()
    r.run(40)
    with pytest.raises(lib.GdError) as exc:
        r.read()
    assert exc.value.status == abi.GD_ETIMEDOUT
    assert "code 4" in str(exc.value)
    r.close()
    # the error word was cleared by the call that reported it
    ctx.sync()
    # defaults back: the same run completes and equals one on a fresh context
    ctx.set_wait_test(0, False)
    r = lib.Remc(d, 40, 10, mb, seed=5, flags=abi.MC_EXCHANGE)
    r.init()
    r.run(40)
    got = r.read()
    r.close()
    ctx2 = lib.Context(0)
    ctx2.set_split(1)
    ctx2.set_schedule(abi.SCHED_WAVES)
    d2 = lib.DeviceComplex(ctx2, cx)
    r2 = lib.Remc(d2, 40, 10, mb, seed=5, flags=abi.MC_EXCHANGE)
    r2.init()
    r2.run(40)
    _same(got, r2.read())
    r2.close()
    d2.close()
    ctx2.close()
    ctx.set_schedule(abi.SCHED_AUTO)
    d.close()
    ctx.close()


def test_wait_hook_needs_a_limit():
    ctx = lib.Context(0)
    with pytest.raises(lib.GdError) as exc:
        ctx.set_wait_test(0, True)
    assert exc.value.status == abi.GD_EINVAL
    ctx.close()


@pytest.mark.parametrize("case", ["fused", "graph"])
@pytest.mark.parametrize("sched", [abi.SCHED_AUTO, abi.SCHED_PERSISTENT])
def test_snapshot_restore_continues_bit_for_bit(case, sched):
    ctx = lib.Context(0)
    ctx.set_schedule(sched, 3 if sched == abi.SCHED_PERSISTENT else 0)
    if sched == abi.SCHED_PERSISTENT:
        ctx.set_split(1)
    cx, n_tmp = _complex(case)
    d = lib.DeviceComplex(ctx, cx)
    _, mb = lib.set_temperature(n_tmp, 0.004, 0.04)
    flags = abi.MC_EXCHANGE | abi.MC_MOVE_AWAY | abi.MC_RECORD | abi.MC_MCC
    kw = dict(seed=77, stream_id=3, flags=flags)
    # one run of 100 steps without a break
    a = lib.Remc(d, 100, 10, mb, **kw)
    a.init()
    a.run(50)
    a.run(50)
    ref = a.read()
    a.close()
    # the same run, snapshotted at step 50 and continued in a new handle
    b = lib.Remc(d, 100, 10, mb, **kw)
    b.init()
    b.run(50)
    blob = b.snapshot()
    b.close()
    c = lib.Remc(d, 100, 10, mb, **kw)
    c.restore(blob)
    c.run(50)
    got = c.read()
    c.close()
    _same(got, ref, rec_from=50)
    assert not np.any(got.record["step"][:, :50])  # steps before the snapshot: not recorded
    # a snapshot only fits a run of the same shape and random stream
    other = lib.Remc(d, 100, 10, mb, seed=78, stream_id=3, flags=flags)
    with pytest.raises(lib.GdError) as exc:
        other.restore(blob)
    assert exc.value.status == abi.GD_EINVAL
    other.close()
    with pytest.raises(lib.GdError):
        c2 = lib.Remc(d, 100, 10, mb, **kw)
        try:
            c2.restore(blob[:-4])
        finally:
            c2.close()
    ctx.set_schedule(abi.SCHED_AUTO)
    d.close()
    ctx.close()


def test_batch_snapshot_restore():
    ctx = lib.Context(0)
    raw, _, _ = synth.default_ff()
    rng = np.random.Generator(np.random.PCG64(31))
    spec = synth.ComplexSpec(pnp=1200, lna=20, n_prt=2, n_lig=4)
    prt = synth.make_protein(rng, spec, 9.0, raw)
    cxs = [synth.make_complex(synth.ComplexSpec(pnp=1200, lna=n, n_prt=2, n_lig=4),
                              seed=40 + i, protein=prt) for i, n in enumerate((12, 29, 41))]
    base = lib.DeviceComplex(ctx, cxs[0])
    dcxs = [lib.DeviceComplex(ctx, cx, share=base, prt_conf0=i % 2, n_prt=1)
            for i, cx in enumerate(cxs)]
    _, mb = lib.set_temperature(8, 0.004, 0.04)
    params = lambda: [abi.mc_params(60, 10, mb, seed=9, stream_id=i,
                                    flags=abi.MC_EXCHANGE | abi.MC_MOVE_AWAY)
                      for i in range(len(dcxs))]
    a = lib.Batch(ctx, dcxs, params())
    a.init()
    a.run(60)
    ref = [a.read(i) for i in range(len(dcxs))]
    a.close()
    b = lib.Batch(ctx, dcxs, params())
    b.init()
    b.run(30)
    blob = b.snapshot()
    b.close()
    c = lib.Batch(ctx, dcxs, params())
    c.restore(blob)
    c.run(30)
    for i in range(len(dcxs)):
        _same(c.read(i), ref[i])
    c.close()
    for d in dcxs:
        d.close()
    base.close()
    ctx.close()


def _pool_used():
    from cuda.bindings import runtime as rt
    assert rt.cudaDeviceSynchronize()[0] == rt.cudaError_t.cudaSuccess
    err, pool = rt.cudaDeviceGetDefaultMemPool(0)
    err, used = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)
    assert err == rt.cudaError_t.cudaSuccess
    return int(used)


def test_injected_allocation_failures():
    """A device allocation that fails (injected at the library's allocation
    sites, as cudaMallocAsync fails on a full device) makes the call return
    GD_ENOMEM, frees what the call had allocated, and leaves the context,
    and the server, working."""
    ctx = lib.Context(0)
    cx, n_tmp = _complex("fused")
    _, mb = lib.set_temperature(n_tmp, 0.004, 0.04)
    used0 = _pool_used()
    for nth in (1, 3, 7):  # upload: the protein, the tables, the ligand ...
        ctx.set_alloc_fail(nth)
        with pytest.raises(lib.GdError) as exc:
            lib.DeviceComplex(ctx, cx)
        assert exc.value.status == abi.GD_ENOMEM and "injected" in str(exc.value)
        assert _pool_used() == used0
    d = lib.DeviceComplex(ctx, cx)  # the hook is off again
    used1 = _pool_used()
    ctx.set_alloc_fail(2)  # the run's state
    with pytest.raises(lib.GdError) as exc:
        lib.Remc(d, 20, 10, mb, seed=3)
    assert exc.value.status == abi.GD_ENOMEM
    assert _pool_used() == used1
    r = lib.Remc(d, 20, 10, mb, seed=3)
    r.init()
    r.run(20)
    out = r.read()
    assert np.isfinite(out.energy).all()
    r.close()
    d.close()
    ctx.close()
    # a served request whose admission fails, between two that succeed
    srv = lib.Server(0, hbm_budget_bytes=1 << 30, max_active=4, steps_per_launch=10)
    pid = srv.add_protein(cx)
    ok0 = srv.wait(srv.submit(pid, cx, 20, 10, mb, n_prt=cx.n_prt, seed=4))
    srv.set_alloc_fail(1)
    bad = srv.submit(pid, cx, 20, 10, mb, n_prt=cx.n_prt, seed=4)
    with pytest.raises(lib.GdError) as exc:
        srv.wait(bad)
    assert exc.value.status == abi.GD_ENOMEM
    ok1 = srv.wait(srv.submit(pid, cx, 20, 10, mb, n_prt=cx.n_prt, seed=4))
    assert np.array_equal(ok0.energy, ok1.energy)
    srv.close()
