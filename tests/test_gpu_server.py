"""Serving form: continuous batching with HBM-budget admission.

Requests that arrive while others run are admitted as slots free up and
share launches; each request keeps its own step counter, state and random
stream, so its result is bit-identical alone and in the mix."""
import time

import numpy as np
import pytest

from gpudock_b200 import abi, lib, synth

pytestmark = pytest.mark.gpu


def _protein_and_ligands(pnp, lnas, seed, n_prt=1):
    raw, _, _ = synth.default_ff()
    rng = np.random.Generator(np.random.PCG64(seed))
    prt = synth.make_protein(rng, synth.ComplexSpec(pnp=pnp, lna=8, n_prt=n_prt), 8.0, raw)
    cxs = [synth.make_complex(synth.ComplexSpec(pnp=pnp, lna=lna, n_prt=n_prt, n_lig=4),
                              seed=seed + 11 * i, protein=prt) for i, lna in enumerate(lnas)]
    return cxs


def _run_alone(cx, steps, spe, mb, seed, stream, split=1):
    """The plain-form run of a complex with the split its server request gets
    (these requests are below the server's split threshold: unsplit)."""
    ctx = lib.Context(0)
    ctx.set_split(split)
    d = lib.DeviceComplex(ctx, cx)
    r = lib.Remc(d, steps, spe, mb, seed=seed, stream_id=stream,
                 flags=abi.MC_EXCHANGE | abi.MC_MOVE_AWAY)
    r.init()
    r.run(steps)
    return r.read()


def test_server_alone_equals_mix():
    cxs = _protein_and_ligands(700, [10, 25, 40, 60, 17, 33], seed=50)
    _, mb = lib.set_temperature(8, 0.004, 0.04)
    steps, spe = 60, 10
    kw = dict(flags=abi.MC_EXCHANGE | abi.MC_MOVE_AWAY)
    srv = lib.Server(0, hbm_budget_bytes=1 << 30, max_active=4, steps_per_launch=10)
    pid = srv.add_protein(cxs[0])
    # request 0 alone
    rid = srv.submit(pid, cxs[0], steps, spe, mb, n_prt=1, seed=9, stream_id=0, **kw)
    alone = srv.wait(rid)
    # the same request among others that arrive before and after it
    ids = []
    for i, cx in enumerate(cxs[1:4]):
        ids.append(srv.submit(pid, cx, steps + 20 * i, spe, mb, n_prt=1, seed=9,
                              stream_id=i + 1, **kw))
    time.sleep(0.05)
    rid0 = srv.submit(pid, cxs[0], steps, spe, mb, n_prt=1, seed=9, stream_id=0, **kw)
    for i, cx in enumerate(cxs[4:]):
        ids.append(srv.submit(pid, cx, steps, spe, mb, n_prt=1, seed=9, stream_id=10 + i, **kw))
    mixed = srv.wait(rid0)
    others = [srv.wait(i) for i in ids]
    st = srv.stats()
    srv.close()
    assert np.array_equal(alone.energy, mixed.energy)
    assert np.array_equal(alone.movematrix, mixed.movematrix)
    assert np.array_equal(alone.idx_tmp, mixed.idx_tmp)
    assert alone.ac_mc == mixed.ac_mc and alone.ac_temp_exchg == mixed.ac_temp_exchg
    assert st.completed == 2 + len(others)
    # and equal to the plain form run of the same complex and stream
    plain = _run_alone(cxs[0], steps, spe, mb, 9, 0)
    assert np.array_equal(alone.energy, plain.energy)
    assert alone.log.t_wall > 0 and mixed.log.t_wall >= mixed.log.t_compute


def test_server_errors_and_cancel():
    cxs = _protein_and_ligands(400, [12, 20], seed=51)
    _, mb = lib.set_temperature(8, 0.004, 0.04)
    srv = lib.Server(0, hbm_budget_bytes=64 << 20, max_active=1, steps_per_launch=10)
    pid = srv.add_protein(cxs[0])
    with pytest.raises(lib.GdError) as e:
        srv.submit(pid + 5, cxs[0], 20, 10, mb, n_prt=1)
    assert e.value.status == abi.GD_EINVAL
    with pytest.raises(lib.GdError) as e:
        srv.submit(pid, cxs[0], 25, 10, mb, n_prt=1)  # not a multiple of 10
    assert e.value.status == abi.GD_EINVAL
    long_id = srv.submit(pid, cxs[0], 100000, 10, mb, n_prt=1)
    queued = srv.submit(pid, cxs[1], 20, 10, mb, n_prt=1)  # waits for the slot
    with pytest.raises(lib.GdError) as e:
        srv.wait(queued, timeout_ms=200)
    assert e.value.status == abi.GD_ETIMEDOUT
    srv.cancel(queued)
    with pytest.raises(lib.GdError) as e:
        srv.wait(queued, timeout_ms=10000)
    assert e.value.status == abi.GD_ECANCELLED
    srv.cancel(long_id)
    with pytest.raises(lib.GdError) as e:
        srv.wait(long_id, timeout_ms=20000)
    assert e.value.status == abi.GD_ECANCELLED
    st = srv.stats()
    assert st.active == 0 and st.queued == 0
    srv.close()
    # a request that can never fit the budget
    tiny = lib.Server(0, hbm_budget_bytes=60 << 10, max_active=1, steps_per_launch=10)
    with pytest.raises(lib.GdError) as e:
        pid = tiny.add_protein(cxs[0])
        tiny.submit(pid, cxs[0], 20, 10, mb, n_prt=1)
    assert e.value.status == abi.GD_EBUDGET
    tiny.close()


def test_served_records_replay_on_oracle():
    """Requests recorded through the server (GD_MC_RECORD) while they share
    launches: every Metropolis decision and every exchange round replays
    bit-exactly on the oracle from the request's own record, the state
    follows the decisions, the temperature labels of every exchange group
    stay a permutation, and a seeded sample of recorded states has the
    oracle's energies (per term, 1e-5 relative)."""
    from tests.test_gpu_fullsize import _groups_are_permutations, _sample_energies
    from tests.test_gpu_remc import _replay_checks

    cxs = _protein_and_ligands(900, [14, 30, 47, 22, 61], seed=52)
    _, mb = lib.set_temperature(8, 0.004, 0.04)
    steps, spe, seed = 60, 10, 13
    kw = dict(flags=abi.MC_EXCHANGE | abi.MC_MOVE_AWAY | abi.MC_RECORD)
    srv = lib.Server(0, hbm_budget_bytes=1 << 30, max_active=3, steps_per_launch=20)
    pid = srv.add_protein(cxs[0])
    ids = []
    for i, cx in enumerate(cxs):
        ids.append(srv.submit(pid, cx, steps, spe, mb, n_prt=1, seed=seed, stream_id=i, **kw))
        if i == 2:
            time.sleep(0.02)  # later requests join launches already running
    swaps = 0
    for i, (rid, cx) in enumerate(zip(ids, cxs)):
        out = srv.wait(rid)
        rec = out.record
        assert rec.shape == (cx.n_lig * 8, steps)
        assert np.array_equal(rec["step"][0], np.arange(steps))
        swaps += _replay_checks(cx, mb, rec, seed, spe, 8, stream=i)
        _groups_are_permutations(rec, 1, 8, cx.n_lig)
        assert out.ac_mc == int(rec["accepted"].sum())
        # the final state is the state after the last recorded decision
        last = rec[:, -1]
        e_fin = np.where(last["accepted"] == 1, last["e_prop_total"], last["e"][:, abi.E_TOTAL])
        assert np.array_equal(out.energy[:, abi.E_TOTAL], e_fin)
        _sample_energies(cx, rec, np.random.Generator(np.random.PCG64(i)), n_sample=6)
    assert swaps > 0
    srv.close()
