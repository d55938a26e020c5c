"""Statistical parity of the GPU REMC against the CPU oracle on the benchmark's
plain configuration, and the reference's own sanity sweeps on its sample
complex 1a07C1.

Every comparison draws the GPU and the CPU samples from different random
streams and from independent replicas (identical starting conformations
that evolve independently), so each group is one independent draw of the
same law for both implementations.  A family of m tests passes when every
p-value exceeds 0.01 / m (Bonferroni: the family's false-failure rate stays
below 1%).

1. Plain single complex (1,500 points x 24 atoms, 8 temperatures geometric
   from 0.004 to 0.04, exchange every 10 steps, 1,000 MC steps, moves
   0.02 A / 0.08 rad) with 64 independent exchange groups on the CPU and
   256 on the GPU:
   per-temperature distributions of the final total energy (two-sample KS),
   per-temperature Metropolis acceptance rates of the groups (Welch t) and
   per-group swap counts (Welch t), plus Fisher's exact test on the pooled
   swap counts.
2. The sweeps of gpudocksm-rem-1.2/README.org on 1a07C1 (protein
   conformation 0, ligand conformation 0): Metropolis acceptance vs
   temperature at a single temperature (README.org:295-340, the set-up of
   FF_opt/dock_decoy_gen/test/AR_MC_single_temp.sh: moves 0.01 A / 0.04 rad),
   exchange acceptance of two temperatures vs their ratio (README.org:
   380-406) and exchange acceptance vs steps per exchange (README.org:
   414-452): GPU against oracle per point.

    python -m tests.test_gpu_stats     (GPU only: the sweep tables at the
                                        reference's run lengths, markdown)
"""
import numpy as np
import pytest
from scipy import stats

from gpudock_b200 import abi, lib, synth
from oracle import oracle as orc
from tests.golden_fixture import load_complex

pytestmark = pytest.mark.gpu

ALPHA = 0.01


@pytest.fixture(scope="module")
def ctx():
    c = lib.Context(0)
    yield c
    c.close()


def _replicate(cx, n_groups, prt_conf=None, lig_conf=0):
    """The complex with n_groups identical ligand conformations (independent
    exchange groups) and optionally one protein conformation."""
    cx.lig_xyz = np.ascontiguousarray(np.repeat(cx.lig_xyz[lig_conf:lig_conf + 1], n_groups,
                                                axis=0))
    if prt_conf is not None:
        cx.prt_xyz = np.ascontiguousarray(cx.prt_xyz[prt_conf:prt_conf + 1])
    cx._struct = None
    return cx


def _gpu_run(ctx, cx, steps, spe, mb, scale, seed, flags, stream_id=0):
    d = lib.DeviceComplex(ctx, cx)
    r = lib.Remc(d, steps, spe, mb, scale, seed=seed, stream_id=stream_id, flags=flags)
    r.init()
    r.run(steps)
    out = r.read()
    r.close()
    d.close()
    return out


def _cpu_run(cx, steps, spe, mb, scale, seed, flags, stream_id=0):
    return orc.remc_run(cx, steps, spe, mb, move_scale=scale, seed=seed, stream_id=stream_id,
                        flags=flags)


def group_stats(out, n_tmp, n_lig, spe):
    """Per group (one protein conformation): final total energy at each
    temperature [n_lig, n_tmp], Metropolis acceptance rate at each
    temperature [n_lig, n_tmp], and swap count [n_lig] (from the records)."""
    rec = out.record
    n_rep, steps = rec.shape
    grp = np.arange(n_rep) % n_lig               # r = n_lig t + l (one protein conf)
    e_fin = np.zeros((n_lig, n_tmp))
    e_fin[grp, out.idx_tmp] = out.energy[:, abi.E_TOTAL]
    it, acc = rec["idx_tmp"], rec["accepted"].astype(np.float64)
    ar = np.zeros((n_lig, n_tmp))
    cnt = np.zeros((n_lig, n_tmp))
    g2 = np.broadcast_to(grp[:, None], it.shape)
    np.add.at(ar, (g2, it), acc)
    np.add.at(cnt, (g2, it), 1.0)
    ar /= np.maximum(cnt, 1.0)
    # a swap changes the temperature index of two replicas of the group
    # between the last step of an interval and the next step
    moved = (it[:, 1:] != it[:, :-1]).sum(axis=1)
    swaps = np.bincount(grp, weights=moved, minlength=n_lig) / 2.0
    return e_fin, ar, swaps


def exchange_attempts(steps, spe, n_tmp, steps_per_dump=1000):
    """Pair attempts per group in `steps` MC steps (exchangereplicas_d.cu:
    pairs (2j + mode, 2j + mode + 1), mode alternating by round within a
    dump) -- the rounds after the last step included, as the run does."""
    n = 0
    for s0 in range(0, steps, spe):
        mode = ((s0 % steps_per_dump) // spe) % 2 if steps_per_dump > 0 else (s0 // spe) % 2
        n += n_tmp // 2 - (1 if (n_tmp % 2 == 0 and mode == 1) else 0)
    return n


def _family(pvals, what):
    m = len(pvals)
    bad = [(k, p) for k, p in enumerate(pvals) if not p > ALPHA / m]
    assert not bad, (what, bad, pvals)


def test_plain_config_statistics(ctx):
    w = synth.WORKLOADS["plain_1500x24"]
    # 64 groups per run; the GPU side runs 4 times (256 groups), the CPU once
    n_groups = 64
    cx = _replicate(synth.make_complex(w.spec, seed=4001), n_groups)
    _, mb = synth.temperatures(w)
    n_tmp, spe, steps = w.n_tmp, w.steps_per_exchange, w.steps
    flags = abi.MC_EXCHANGE | abi.MC_MOVE_AWAY | abi.MC_RECORD
    side = {"gpu": [], "cpu": []}
    for k in range(4):
        g = _gpu_run(ctx, cx, steps, spe, mb, w.move_scale, 5100 + k, flags)
        side["gpu"].append(group_stats(g, n_tmp, n_groups, spe))
    c = _cpu_run(cx, steps, spe, mb, w.move_scale, 6100, flags)
    side["cpu"].append(group_stats(c, n_tmp, n_groups, spe))
    cat = {k: [np.concatenate([v[i] for v in side[k]]) for i in range(3)] for k in side}
    (ge, ga, gs), (ce, ca, cs) = cat["gpu"], cat["cpu"]
    assert ge.shape == (4 * n_groups, n_tmp) and ce.shape == (n_groups, n_tmp)
    _family([stats.ks_2samp(ge[:, t], ce[:, t]).pvalue for t in range(n_tmp)],
            "final energy per temperature (KS)")
    _family([stats.ttest_ind(ga[:, t], ca[:, t], equal_var=False).pvalue for t in range(n_tmp)],
            "acceptance rate per temperature (Welch)")
    att = exchange_attempts(steps, spe, n_tmp)
    assert 0 < gs.sum() < att * len(gs) and 0 < cs.sum() < att * len(cs)
    p_swap = stats.ttest_ind(gs, cs, equal_var=False).pvalue
    tg, tc = len(gs) * att, len(cs) * att  # attempts of each side
    p_fisher = stats.fisher_exact([[gs.sum(), tg - gs.sum()], [cs.sum(), tc - cs.sum()]]).pvalue
    _family([p_swap, p_fisher], "swaps per group (Welch) and pooled (Fisher)")
    # acceptance rises with the temperature (slot 0 is the lowest)
    assert np.all(np.diff(ga.mean(axis=0)) >= -0.02)


# ---------------------------------------------------------------------------
# The reference's sanity sweeps (README.org) on 1a07C1
# ---------------------------------------------------------------------------
AR_TEMPS = (0.000016, 0.000128, 0.000512, 0.001024, 0.002048, 0.004096, 0.008192, 0.016384,
            0.032768, 0.065536, 0.131072, 0.262144)
SCRIPT_MOVE = (0.01, 0.01, 0.01, 0.04, 0.04, 0.04)  # AR_MC_single_temp.sh: -t 0.01 -r 0.04


def _sample_complex(n_groups):
    cx, _, _ = load_complex("rem")
    return _replicate(cx, n_groups, prt_conf=0)


def ar_vs_temperature(ctx, temps, steps, n_groups, seed, cpu=False, stream_id=0):
    """Metropolis acceptance per replica at fixed temperatures (no exchange):
    [n_groups, len(temps)]."""
    cx = _sample_complex(n_groups)
    mb = (-1.0 / np.asarray(temps, np.float32)).astype(np.float32)
    if cpu:
        out = _cpu_run(cx, steps, steps, mb, SCRIPT_MOVE, seed, 0, stream_id)
    else:
        out = _gpu_run(ctx, cx, steps, steps, mb, SCRIPT_MOVE, seed, 0, stream_id)
    # replica r = n_lig t + l stays at temperature t
    return out.acs_mc.reshape(len(temps), n_groups).T / float(steps)


def exchange_ar(ctx, temps, steps, spe, n_groups, seed, cpu=False, record=True):
    """Swaps per group and attempts per group of a run at the given ladder."""
    cx = _sample_complex(n_groups)
    mb = (-1.0 / np.asarray(temps, np.float32)).astype(np.float32)
    flags = abi.MC_EXCHANGE | (abi.MC_RECORD if record else 0)
    if cpu:
        out = _cpu_run(cx, steps, spe, mb, SCRIPT_MOVE, seed, flags)
    else:
        out = _gpu_run(ctx, cx, steps, spe, mb, SCRIPT_MOVE, seed, flags)
    att = exchange_attempts(steps, spe, len(temps))
    if record:
        _, _, swaps = group_stats(out, len(temps), n_groups, spe)
    else:
        swaps = np.full(n_groups, out.ac_temp_exchg / 2.0 / n_groups)
    return swaps, att


def test_ar_vs_temperature_matches_oracle(ctx):
    n_groups, steps = 16, 1500
    g = ar_vs_temperature(ctx, AR_TEMPS, steps, n_groups, seed=71)
    c = ar_vs_temperature(ctx, AR_TEMPS, steps, n_groups, seed=72, cpu=True)
    _family([stats.ttest_ind(g[:, t], c[:, t], equal_var=False).pvalue
             for t in range(len(AR_TEMPS))], "AR vs temperature (Welch)")
    # the reference's trend: acceptance grows with the temperature
    m = g.mean(axis=0)
    assert m[-1] > m[0] and np.all(np.diff(m) > -0.03), m


RATIO_LOW = (0.0004, 0.0011942, 0.0035656, 0.0106464)


def test_exchange_ar_vs_ratio_matches_oracle(ctx):
    n_groups, steps, spe = 32, 1000, 5
    pv = []
    for k, t0 in enumerate(RATIO_LOW):
        temps = (t0, t0 * 1.2)
        gs, att = exchange_ar(ctx, temps, steps, spe, n_groups, seed=81 + k)
        cs, _ = exchange_ar(ctx, temps, steps, spe, n_groups, seed=91 + k, cpu=True)
        tot = n_groups * att
        pv.append(stats.fisher_exact([[gs.sum(), tot - gs.sum()],
                                      [cs.sum(), tot - cs.sum()]]).pvalue)
    _family(pv, "exchange AR of two temperatures (Fisher)")


def test_exchange_ar_vs_cadence_matches_oracle(ctx):
    w = synth.WORKLOADS["plain_1500x24"]
    _, mb = synth.temperatures(w)
    temps = -1.0 / mb
    n_groups, steps = 16, 1000
    pv = []
    for k, spe in enumerate((10, 20, 50, 100)):
        gs, att = exchange_ar(ctx, temps, steps, spe, n_groups, seed=101 + k)
        cs, _ = exchange_ar(ctx, temps, steps, spe, n_groups, seed=111 + k, cpu=True)
        tot = n_groups * att
        pv.append(stats.fisher_exact([[gs.sum(), tot - gs.sum()],
                                      [cs.sum(), tot - cs.sum()]]).pvalue)
    _family(pv, "exchange AR vs steps per exchange (Fisher)")


# ---------------------------------------------------------------------------
# Tables at the reference's run lengths (GPU only)
# ---------------------------------------------------------------------------
REF_AR = {0.000016: 0.003475, 0.000128: 0.004107, 0.000512: 0.010275, 0.001024: 0.027060,
          0.002048: 0.073684, 0.004096: 0.157058, 0.008192: 0.282580, 0.016384: 0.440276,
          0.032768: 0.581020, 0.065536: 0.706120, 0.131072: 0.866801, 0.262144: 0.960365}
REF_RATIO = {0.0004: 0.310700, 0.0011942: 0.334733, 0.0035656: 0.327690, 0.0106464: 0.330657}


def main():
    ctx = lib.Context(0)
    print("| temperature | AR of MC (this build, 1a07C1, 300,000 steps, 16 replicas) "
          "| AR of MC (README.org:295-340) |")
    print("|---|---|---|")
    g = ar_vs_temperature(ctx, AR_TEMPS, 300_000, 16, seed=1)
    for t, v in zip(AR_TEMPS, g.mean(axis=0)):
        print(f"| {t:.6f} | {v:.6f} | {REF_AR[t]:.6f} |")
    print()
    print("| T1 | T2 | exchange AR (this build, 20,000 steps, spe 5, 32 groups) "
          "| exchange AR (README.org:387-406) |")
    print("|---|---|---|---|")
    for t0 in RATIO_LOW:
        s, att = exchange_ar(ctx, (t0, t0 * 1.2), 20_000, 5, 32, seed=2, record=False)
        print(f"| {t0:.7f} | {t0 * 1.2:.7f} | {s.sum() / (32 * att):.6f} | {REF_RATIO[t0]:.6f} |")
    print()
    w = synth.WORKLOADS["plain_1500x24"]
    _, mb = synth.temperatures(w)
    print("| steps per exchange | exchange AR (this build, 8 T 0.004..0.04, 20,000 steps, "
          "32 groups) |")
    print("|---|---|")
    for spe in (10, 20, 50, 100, 200):
        s, att = exchange_ar(ctx, -1.0 / mb, 20_000, spe, 32, seed=3, record=False)
        print(f"| {spe} | {s.sum() / (32 * att):.6f} |")
    ctx.close()


if __name__ == "__main__":
    main()
