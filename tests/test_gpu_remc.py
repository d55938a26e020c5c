"""REMC parity: decisions bit-exact against the oracle given the device's own
energies, building blocks (Philox, decision exp, Metropolis) bit-exact, and
per-temperature energy distributions statistically indistinguishable from the
oracle's CPU run."""
import numpy as np
import pytest
import torch
from scipy import stats

from gpudock_b200 import abi, lib, synth
from oracle import oracle as orc
from tests import tolerance as tol

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = lib.Context(0)
    yield c
    c.close()


def test_philox_bitexact(ctx):
    rng = np.random.default_rng(7)
    n = 4096
    ctr = rng.integers(0, 2 ** 32, size=(n, 4), dtype=np.uint64).astype(np.uint32)
    key = rng.integers(0, 2 ** 32, size=(n, 2), dtype=np.uint64).astype(np.uint32)
    ctr[:3] = [[0, 0, 0, 0], [0xFFFFFFFF] * 4, [1, 2, 3, 4]]
    key[:3] = [[0, 0], [0xFFFFFFFF] * 2, [5, 6]]
    dc = torch.from_numpy(ctr.view(np.int32)).cuda()
    dk = torch.from_numpy(key.view(np.int32)).cuda()
    do = torch.zeros_like(dc)
    lib.check(ctx._lib.gd_philox_dev(ctx.h, n, dc.data_ptr(), dk.data_ptr(), do.data_ptr()),
              "philox")
    ctx.sync()
    got = do.cpu().numpy().view(np.uint32)
    ref = orc.philox(ctr[:512], key[:512])
    assert np.array_equal(got[:512], ref)


def test_decision_expf_bitexact(ctx):
    rng = np.random.default_rng(8)
    x = np.concatenate([
        rng.uniform(-100, 100, 20000), rng.uniform(-1, 1, 20000), rng.normal(0, 5, 20000),
        np.array([0.0, -0.0, 88.72, 88.7199, -87.33, -87.3299, 1e-30, -1e-30, np.inf, -np.inf,
                  np.nan]),
    ]).astype(np.float32)
    dx = torch.from_numpy(x).cuda()
    dy = torch.empty_like(dx)
    lib.check(ctx._lib.gd_expf_dev(ctx.h, len(x), dx.data_ptr(), dy.data_ptr()), "expf")
    ctx.sync()
    got = dy.cpu().numpy()
    ref = orc.expf(x)
    same = (got.view(np.uint32) == ref.view(np.uint32)) | (np.isnan(got) & np.isnan(ref))
    assert same.all(), x[~same][:10]
    # and it is an accurate exp (relative error of a few ulp where normal)
    m = (x > -80) & (x < 80)
    rel = np.abs(got[m].astype(np.float64) - np.exp(x[m].astype(np.float64))) / np.exp(
        x[m].astype(np.float64))
    assert rel.max() < 4e-7


def test_metropolis_bitexact(ctx):
    rng = np.random.default_rng(9)
    n = 20000
    e_old = rng.normal(0, 1, n).astype(np.float32)
    e_new = (e_old + rng.normal(0, 0.01, n)).astype(np.float32)
    mb = (-1.0 / rng.uniform(0.004, 0.08, n)).astype(np.float32)
    rep = rng.integers(0, 100000, n).astype(np.int32)
    step = rng.integers(0, 5000, n).astype(np.int32)
    t = [torch.from_numpy(a).cuda() for a in (e_new, e_old, mb, rep, step)]
    acc = torch.zeros(n, dtype=torch.int32, device="cuda")
    seed = 0x1234_5678_9ABC_DEF0
    lib.check(ctx._lib.gd_metropolis_dev(ctx.h, n, *[a.data_ptr() for a in t], seed, 3,
                                         acc.data_ptr()), "metropolis")
    ctx.sync()
    got = acc.cpu().numpy()
    ref = orc.metropolis(e_new[:4000], e_old[:4000], mb[:4000], seed, 3, rep[:4000], step[:4000])
    assert np.array_equal(got[:4000], ref)
    assert 0 < got.mean() < 1


def _replay_checks(cx, mb, rec, seed, spe, n_tmp, stream=0, dump=1000):
    """Decision replay from the device's own trajectory record."""
    n_rep, steps = rec.shape
    n_lig = cx.n_lig
    # Metropolis: same decision from (proposed total, accepted total, beta, u)
    e_old = rec["e"][:, :, abi.E_TOTAL].reshape(-1)
    e_new = rec["e_prop_total"].reshape(-1)
    beta = mb[rec["idx_tmp"].reshape(-1)]
    reps = rec["idx_rep"].reshape(-1)
    st = rec["step"].reshape(-1)
    ref = orc.metropolis(e_new, e_old, beta, seed, stream, reps, st)
    assert np.array_equal(ref, rec["accepted"].reshape(-1)), "Metropolis decisions differ"
    # state transitions follow the decisions
    nxt = rec[:, 1:]
    cur = rec[:, :-1]
    acc = cur["accepted"] == 1
    assert np.array_equal(nxt["e"][..., abi.E_TOTAL][acc], cur["e_prop_total"][acc])
    assert np.array_equal(nxt["e"][..., abi.E_TOTAL][~acc], cur["e"][..., abi.E_TOTAL][~acc])
    # exchanges: replay each round from the totals at its boundary
    params, _ = abi.mc_params(steps, spe, mb, seed=seed, stream_id=stream,
                              flags=abi.MC_EXCHANGE, steps_per_dump=dump)
    n_prt = cx.n_prt
    swaps = 0
    for s0 in range(0, steps - spe, spe):
        last = s0 + spe - 1
        e_after = np.where(rec["accepted"][:, last] == 1, rec["e_prop_total"][:, last],
                           rec["e"][:, last, abi.E_TOTAL]).astype(np.float32)
        before = rec["idx_tmp"][:, last]
        after = rec["idx_tmp"][:, last + 1]
        mode_t = ((s0 % dump) // spe) % 2
        it, _ = orc.exchange(params, n_prt, n_lig, n_tmp, s0 // spe, mode_t, e_after, before)
        assert np.array_equal(it, after), f"exchange round {s0 // spe} differs"
        swaps += int((before != after).sum())
    return swaps


def test_remc_replay_plain(ctx):
    w = synth.WORKLOADS["plain_1500x24"]
    cx = synth.make_complex(w.spec, seed=21)
    _, mb = synth.temperatures(w)
    d = lib.DeviceComplex(ctx, cx)
    steps, spe, seed = 400, w.steps_per_exchange, 77
    r = lib.Remc(d, steps, spe, mb, seed=seed, flags=abi.MC_EXCHANGE | abi.MC_RECORD)
    r.init()
    r.run(steps)
    out = r.read()
    swaps = _replay_checks(cx, mb, out.record, seed, spe, w.n_tmp)
    assert out.ac_mc == int(out.record["accepted"].sum())
    assert swaps > 0
    # the last exchange round follows the last recorded step
    rec = out.record
    e_last = np.where(rec["accepted"][:, -1] == 1, rec["e_prop_total"][:, -1],
                      rec["e"][:, -1, abi.E_TOTAL]).astype(np.float32)
    params, _ = abi.mc_params(steps, spe, mb, seed=seed, flags=abi.MC_EXCHANGE)
    s0 = steps - spe
    it, _ = orc.exchange(params, 1, 1, w.n_tmp, s0 // spe, ((s0 % 1000) // spe) % 2, e_last,
                         rec["idx_tmp"][:, -1])
    assert np.array_equal(it, out.idx_tmp)
    swaps += int((rec["idx_tmp"][:, -1] != out.idx_tmp).sum())
    assert out.ac_temp_exchg == swaps


def test_remc_replay_ensemble(ctx):
    """Several protein and ligand conformations, odd temperature count."""
    spec = synth.ComplexSpec(pnp=600, lna=16, n_prt=3, n_lig=5)
    cx = synth.make_complex(spec, seed=22)
    _, mb = lib.set_temperature(7, 0.004, 0.08)
    d = lib.DeviceComplex(ctx, cx)
    steps, spe, seed = 120, 6, 1234
    r = lib.Remc(d, steps, spe, mb, seed=seed, stream_id=5,
                 flags=abi.MC_EXCHANGE | abi.MC_RECORD | abi.MC_MOVE_AWAY, steps_per_dump=30)
    r.init()
    r.run(steps)
    out = r.read()
    assert out.record.shape == (3 * 5 * 7, steps)
    _replay_checks(cx, mb, out.record, seed, spe, 7, stream=5, dump=30)


def test_remc_init_energies(ctx):
    """MonteCarlo_Init_d: move-away pose energies against the oracle."""
    w = synth.WORKLOADS["plain_1500x24"]
    cx = synth.make_complex(w.spec, seed=23)
    _, mb = synth.temperatures(w)
    d = lib.DeviceComplex(ctx, cx)
    r = lib.Remc(d, 10, 10, mb, flags=abi.MC_EXCHANGE | abi.MC_MOVE_AWAY)
    r.init()
    out = r.read()
    pose = (np.asarray(w.move_scale, np.float32) * np.float32(44.5)).reshape(1, 6)
    terms_r, raw_r, asum = orc.energy_poses(cx, pose)
    bad, rel = tol.check_terms(out.energy, np.repeat(terms_r, len(out.energy), 0),
                               np.repeat(raw_r, len(out.energy), 0),
                               np.repeat(asum, len(out.energy), 0), cx.ff)
    assert not bad.any(), rel.max(axis=0)
    assert np.array_equal(out.movematrix, np.repeat(pose, len(out.energy), 0))
    assert out.ac_mc == 0
    assert np.array_equal(out.idx_tmp, np.arange(w.n_tmp))


def test_remc_resume_matches_single_run(ctx):
    """Counter-based RNG: 2 x 50 steps == 1 x 100 steps, bit for bit."""
    w = synth.WORKLOADS["plain_1500x24"]
    cx = synth.make_complex(w.spec, seed=24)
    _, mb = synth.temperatures(w)
    d = lib.DeviceComplex(ctx, cx)
    a = lib.Remc(d, 100, 10, mb, seed=5)
    a.init()
    a.run(100)
    oa = a.read()
    b = lib.Remc(d, 100, 10, mb, seed=5)
    b.init()
    b.run(50)
    b.run(50)
    ob = b.read()
    assert np.array_equal(oa.energy, ob.energy)
    assert np.array_equal(oa.movematrix, ob.movematrix)
    assert np.array_equal(oa.idx_tmp, ob.idx_tmp)


def test_gd_run_matches_handles(ctx):
    w = synth.WORKLOADS["plain_1500x24"]
    cx = synth.make_complex(w.spec, seed=25)
    _, mb = synth.temperatures(w)
    out = lib.run(cx, 60, 10, mb, seed=9)
    d = lib.DeviceComplex(ctx, cx)
    r = lib.Remc(d, 60, 10, mb, seed=9)
    r.init()
    r.run(60)
    o2 = r.read()
    assert np.array_equal(out.energy, o2.energy)
    assert out.ac_mc == o2.ac_mc
    assert out.log.t_wall > 0.0


def test_remc_distributions_match_oracle(ctx):
    """Per-temperature energy distributions, acceptance rates and exchange
    rates of the GPU run against the CPU oracle run, on independent samples:
    64 exchange groups of identical starting conformations evolve
    independently, so the final state of each group is one independent draw
    of the same law for both implementations; the GPU and CPU runs use
    different random streams.  Two-sample KS per temperature, Welch t on
    per-group acceptance counts, Fisher's exact test on accepted / rejected
    swap attempts; every p-value must exceed 0.01."""
    spec = synth.ComplexSpec(pnp=500, lna=12, n_prt=1, n_lig=1)
    cx = synth.make_complex(spec, seed=26)
    cx.lig_xyz = np.repeat(cx.lig_xyz[:1], 64, axis=0)  # 64 independent groups
    cx._struct = None
    n_tmp, steps, spe = 4, 60, 10
    _, mb = lib.set_temperature(n_tmp, 0.01, 0.05)
    d = lib.DeviceComplex(ctx, cx)
    scale = (0.2, 0.2, 0.2, 0.3, 0.3, 0.3)
    flags = abi.MC_EXCHANGE | abi.MC_MOVE_AWAY
    gpu_e, cpu_e, gpu_a, cpu_a = [], [], [], []
    swaps = {"gpu": 0, "cpu": 0}
    for k in range(4):
        r = lib.Remc(d, steps, spe, mb, scale, seed=2000 + k, flags=flags)
        r.init()
        r.run(steps)
        g = r.read()
        c = orc.remc_run(cx, steps, spe, mb, move_scale=scale, seed=3000 + k, flags=flags)
        for out, es, acs in ((g, gpu_e, gpu_a), (c, cpu_e, cpu_a)):
            es.append((out.energy[:, abi.E_TOTAL], out.idx_tmp.copy()))
            acs.append(out.acs_mc.reshape(n_tmp, 64).sum(axis=0))
        # a swap credits both replica slots of the pair
        swaps["gpu"] += g.ac_temp_exchg // 2
        swaps["cpu"] += c.ac_temp_exchg // 2
    for t in range(n_tmp):
        a = np.concatenate([e[it == t] for e, it in gpu_e])
        b = np.concatenate([e[it == t] for e, it in cpu_e])
        assert len(a) == len(b) == 4 * 64
        p = stats.ks_2samp(a, b).pvalue
        assert p > 0.01, (t, p)
    p = stats.ttest_ind(np.concatenate(gpu_a), np.concatenate(cpu_a), equal_var=False).pvalue
    assert p > 0.01, p
    # attempts: after every interval, in each of the 64 groups, the pairs
    # (2j + mode, 2j + mode + 1) with mode alternating 0, 1 by round
    rounds = steps // spe
    per_mode = [n_tmp // 2, n_tmp // 2 - (n_tmp % 2 == 0)]
    attempts = 4 * 64 * sum(per_mode[k % 2] for k in range(rounds))
    assert 0 < swaps["gpu"] < attempts and 0 < swaps["cpu"] < attempts
    table = [[swaps["gpu"], attempts - swaps["gpu"]], [swaps["cpu"], attempts - swaps["cpu"]]]
    p = stats.fisher_exact(table).pvalue
    assert p > 0.01, (table, p)
