"""Persistent launch schedule on the GPU: the same runs with one CTA per unit
(GD_SCHED_WAVES) and with units cut at MC-step boundaries over a few
persistent CTAs (GD_SCHED_PERSISTENT) must give bit-identical trajectories,
records and counters.  Few CTAs force many cuts, table switches between items
and protein conformations, and pieces that wait on another CTA."""
import numpy as np
import pytest

from gpudock_b200 import abi, lib, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = lib.Context(0)
    c.set_split(1)  # persistent schedules are for unsplit units
    yield c
    c.set_schedule(abi.SCHED_AUTO)
    c.close()


def _same(a, b):
    assert np.array_equal(a.energy, b.energy)
    assert np.array_equal(a.movematrix, b.movematrix)
    assert np.array_equal(a.idx_tmp, b.idx_tmp)
    assert a.ac_mc == b.ac_mc and a.ac_temp_exchg == b.ac_temp_exchg
    if a.record is not None:
        assert np.array_equal(a.record, b.record)


def _remc(ctx, d, mb, steps, spe, flags, chunks, sched, machines=0, tail=2):
    ctx.set_schedule(sched, machines)
    ctx.set_schedule_tail(tail)
    r = lib.Remc(d, steps, spe, mb, seed=21, flags=flags)
    r.init()
    for n in chunks:
        r.run(n)
    out = r.read()
    r.close()
    return out


@pytest.mark.parametrize("case", ["fused", "graph", "streamed", "mcc"])
def test_persistent_equals_waves(ctx, case):
    flags = abi.MC_EXCHANGE | abi.MC_MOVE_AWAY | abi.MC_RECORD
    if case == "fused":      # 8 temperatures: exchange inside the kernel, 6 units
        spec, n_tmp = synth.ComplexSpec(pnp=900, lna=24, n_prt=3, n_lig=8), 8
    elif case == "graph":    # 6 temperatures: exchange kernel, captured interval
        spec, n_tmp = synth.ComplexSpec(pnp=700, lna=17, n_prt=2, n_lig=10), 6
    elif case == "streamed":  # 8,000 points: the protein streams through the ring
        spec, n_tmp = synth.ComplexSpec(pnp=8000, lna=20, n_prt=3, n_lig=4), 8
    else:
        spec, n_tmp = synth.ComplexSpec(pnp=800, lna=30, n_prt=2, n_lig=12), 8
        flags |= abi.MC_MCC
    cx = synth.make_complex(spec, seed=300 + len(case))
    d = lib.DeviceComplex(ctx, cx)
    _, mb = lib.set_temperature(n_tmp, 0.004, 0.04)
    steps, spe = 40, 10
    ref = _remc(ctx, d, mb, steps, spe, flags, [20, 20], abi.SCHED_WAVES)
    # tail > 0: the last steps of every unit go through the shared queue
    for machines, tail in ((1, 2), (2, 0), (2, 1), (3, 2), (5, 5), (5, 0)):
        got = _remc(ctx, d, mb, steps, spe, flags, [20, 20], abi.SCHED_PERSISTENT, machines, tail)
        _same(got, ref)
    ctx.set_schedule(abi.SCHED_AUTO)
    ctx.set_schedule_tail(2)


def test_persistent_batch_of_items(ctx):
    """Several complexes in one plan: pieces switch items (tables) and
    protein conformations (resident tiles) on one CTA."""
    raw, _, _ = synth.default_ff()
    rng = np.random.Generator(np.random.PCG64(7))
    pspec = synth.ComplexSpec(pnp=1000, lna=8, n_prt=2)
    prt = synth.make_protein(rng, pspec, 8.0, raw)
    cxs = [synth.make_complex(synth.ComplexSpec(pnp=1000, lna=n, n_prt=2, n_lig=4),
                              seed=50 + n, protein=prt) for n in (33, 36, 38, 40)]
    _, mb = lib.set_temperature(8, 0.004, 0.04)
    base = lib.DeviceComplex(ctx, cxs[0])
    dcxs = [base] + [lib.DeviceComplex(ctx, cx, share=base, prt_conf0=0, n_prt=2)
                     for cx in cxs[1:]]
    steps, spe = 30, 10
    flags = abi.MC_EXCHANGE | abi.MC_RECORD
    params = [abi.mc_params(steps, spe, mb, seed=4, stream_id=i, flags=flags)
              for i in range(len(cxs))]

    def run(sched, machines=0, tail=2):
        ctx.set_schedule(sched, machines)
        ctx.set_schedule_tail(tail)
        b = lib.Batch(ctx, dcxs, params)
        b.init()
        b.run(steps)
        out = [b.read(i) for i in range(len(cxs))]
        b.close()
        return out

    ref = run(abi.SCHED_WAVES)
    for machines, tail in ((1, 2), (3, 0), (3, 3), (7, 2)):
        for a, b in zip(run(abi.SCHED_PERSISTENT, machines, tail), ref):
            _same(a, b)
    ctx.set_schedule(abi.SCHED_AUTO)
    ctx.set_schedule_tail(2)


def test_schedule_option_checks(ctx):
    with pytest.raises(lib.GdError):
        ctx.set_schedule(7)
    with pytest.raises(lib.GdError):
        ctx.set_schedule(abi.SCHED_PERSISTENT, -1)
    ctx.set_schedule(abi.SCHED_AUTO)
