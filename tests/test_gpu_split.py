"""Split units (thread-block clusters): a 32-replica unit on `split` CTAs that
each evaluate every split-th protein tile and add their partial energies
through distributed shared memory every MC step.

Checked: the energies of recorded states against the oracle at every split,
every Metropolis decision replayed bit-exactly on the oracle from the
recorded totals, a split unit's run identical alone and inside a batch and
inside the server (the split follows from the complex, not from the mix),
streamed and resident proteins, and the size rule of the default."""
import time

import numpy as np
import pytest

from gpudock_b200 import abi, lib, synth
from oracle import oracle as orc
from tests import tolerance as tol

pytestmark = pytest.mark.gpu

FLAGS = abi.MC_EXCHANGE | abi.MC_MOVE_AWAY | abi.MC_RECORD | abi.MC_MCC


def _run(ctx, cx, split, steps=30, spe=10, seed=12, flags=FLAGS):
    ctx.set_split(split)
    _, mb = lib.set_temperature(8, 0.004, 0.04)
    d = lib.DeviceComplex(ctx, cx)
    r = lib.Remc(d, steps, spe, mb, seed=seed, flags=flags)
    r.init()
    r.run(steps)
    out = r.read()
    r.close()
    d.close()
    ctx.set_split(0)
    return out, mb


def _check_records(cx, out, mb, seed=12, steps=(0, -1)):
    rec = out.record
    # decisions: every step of every replica, from the recorded totals
    flat = rec.reshape(-1)
    ref = orc.metropolis(flat["e_prop_total"], flat["e"][:, abi.E_TOTAL],
                         mb[flat["idx_tmp"]], seed, 0, flat["idx_rep"], flat["step"])
    assert np.array_equal(ref, flat["accepted"])
    # energies of recorded states (first and last step) against the oracle
    for s in steps:
        r = rec[:, s]
        for p in range(cx.n_prt):
            for l in range(cx.n_lig):
                sel = (r["idx_prt"] == p) & (r["idx_lig"] == l)
                if not sel.any():
                    continue
                poses = np.ascontiguousarray(r["movematrix"][sel], np.float32)
                terms_r, raw_r, asum = orc.energy_poses(cx, poses, p, l)
                bad, rel = tol.check_terms(r["e"][sel], terms_r, raw_r, asum, cx.ff)
                assert not bad.any(), (s, p, l, np.nanmax(rel, axis=0))


@pytest.mark.parametrize("pnp", [3000, 9000])  # resident; streamed unsplit
def test_split_energies_and_decisions(pnp):
    ctx = lib.Context(0)
    cx = synth.make_complex(synth.ComplexSpec(pnp=pnp, lna=28, n_prt=2, n_lig=4), seed=80)
    base, _ = _run(ctx, cx, 1)
    for split in (2, 4, 8):
        out, mb = _run(ctx, cx, split)
        _check_records(cx, out, mb)
        # the start states (before any decision) agree with the unsplit run
        assert np.allclose(out.record[:, 0]["e"], base.record[:, 0]["e"], rtol=1e-5, atol=1e-5)
        assert 0 < out.ac_mc < out.record.size
    ctx.close()


def test_split_batch_equals_alone():
    raw, _, _ = synth.default_ff()
    rng = np.random.Generator(np.random.PCG64(81))
    spec = synth.ComplexSpec(pnp=2500, lna=8, n_prt=2)
    prt = synth.make_protein(rng, spec, 8.0, raw)
    cxs = [synth.make_complex(synth.ComplexSpec(pnp=2500, lna=n, n_prt=2, n_lig=4), seed=82 + n,
                              protein=prt) for n in (20, 35, 50)]
    _, mb = lib.set_temperature(8, 0.004, 0.04)
    ctx = lib.Context(0)
    ctx.set_split(4)
    base = lib.DeviceComplex(ctx, cxs[0])
    dcxs = [base] + [lib.DeviceComplex(ctx, cx, share=base, prt_conf0=0, n_prt=2)
                     for cx in cxs[1:]]
    steps, spe = 30, 10
    flags = abi.MC_EXCHANGE | abi.MC_MOVE_AWAY
    params = [abi.mc_params(steps, spe, mb, seed=5, stream_id=i, flags=flags) for i in range(3)]
    b = lib.Batch(ctx, dcxs, params)
    b.init()
    b.run(steps)
    for i, d in enumerate(dcxs):
        got = b.read(i)
        r = lib.Remc(d, steps, spe, mb, seed=5, stream_id=i, flags=flags)
        r.init()
        r.run(steps)
        alone = r.read()
        assert np.array_equal(got.energy, alone.energy), i
        assert np.array_equal(got.movematrix, alone.movematrix), i
        assert got.ac_mc == alone.ac_mc and got.ac_temp_exchg == alone.ac_temp_exchg
    b.close()
    ctx.close()


def test_split_default_rule_and_server():
    """A 100-atom ligand against 8,000 points splits 8 ways by default; served
    alone, served among smaller requests and run in the plain form it gives
    the same trajectory."""
    raw, _, _ = synth.default_ff()
    rng = np.random.Generator(np.random.PCG64(83))
    prt = synth.make_protein(rng, synth.ComplexSpec(pnp=8000, lna=8, n_prt=1), 8.0, raw)
    big = synth.make_complex(synth.ComplexSpec(pnp=8000, lna=100, n_prt=1, n_lig=4), seed=84,
                             protein=prt)
    small = [synth.make_complex(synth.ComplexSpec(pnp=8000, lna=n, n_prt=1, n_lig=4),
                                seed=85 + n, protein=prt) for n in (12, 30)]
    _, mb = lib.set_temperature(8, 0.004, 0.04)
    steps, spe = 40, 10
    kw = dict(flags=abi.MC_EXCHANGE | abi.MC_MOVE_AWAY)
    srv = lib.Server(0, hbm_budget_bytes=2 << 30, max_active=8, steps_per_launch=10)
    pid = srv.add_protein(big)
    alone = srv.wait(srv.submit(pid, big, steps, spe, mb, n_prt=1, seed=3, stream_id=0, **kw))
    ids = [srv.submit(pid, c, steps, spe, mb, n_prt=1, seed=3, stream_id=1 + i, **kw)
           for i, c in enumerate(small)]
    time.sleep(0.02)
    rid = srv.submit(pid, big, steps, spe, mb, n_prt=1, seed=3, stream_id=0, **kw)
    mixed = srv.wait(rid)
    for i in ids:
        srv.wait(i)
    srv.close()
    assert np.array_equal(alone.energy, mixed.energy)
    assert np.array_equal(alone.movematrix, mixed.movematrix)
    ctx = lib.Context(0)
    d = lib.DeviceComplex(ctx, big)
    r = lib.Remc(d, steps, spe, mb, seed=3, stream_id=0, **kw)
    r.init()
    r.run(steps)
    plain = r.read()
    assert np.array_equal(alone.energy, plain.energy)
    r.close()
    d.close()
    ctx.close()


def test_split_option_checks():
    ctx = lib.Context(0)
    for bad in (-1, 3, 16):
        with pytest.raises(lib.GdError):
            ctx.set_split(bad)
    ctx.set_split(0)
    ctx.close()
