"""Parity at the benchmark's full sizes, through checks whose oracle cost does
not grow with the workload: the headline ensemble (8,800 replicas, 40 atoms x
4,000 points, 11 protein x 50 ligand conformations x 16 temperatures), the
512-ligand batch (16,384 replicas against a 6,000-point protein) and the
1,048,576-pose sweep against 2,000 / 4,000 / 8,000 / 16,000 points.

Checked at those sizes: every Metropolis decision and every exchange round
replayed bit-exactly from the device's own records; the energies of a seeded
sample of recorded states against the oracle; the temperature labels of every
exchange group a permutation at every step; the acceptance counter equal to
the records; pose energies bit-identical whatever the order of the poses, and
a seeded 4,096-pose subset at each protein size against the oracle."""
import dataclasses
import types

import numpy as np
import pytest
import torch

from gpudock_b200 import abi, lib, synth
from oracle import oracle as orc
from tests import tolerance as tol
from tests.test_gpu_remc import _replay_checks

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = lib.Context(0)
    yield c
    c.close()


def _sample_energies(cx, rec, rng, n_sample=24, steps=(0, -1), prt_conf0=0):
    """Recorded states of a seeded replica sample against the oracle
    (record protein conformation p is the complex's prt_conf0 + p)."""
    reps = rng.choice(rec.shape[0], size=min(n_sample, rec.shape[0]), replace=False)
    for s in steps:
        r = rec[reps, s]
        for k in range(len(reps)):
            p, l = prt_conf0 + int(r["idx_prt"][k]), int(r["idx_lig"][k])
            pose = np.ascontiguousarray(r["movematrix"][k:k + 1], np.float32)
            terms_r, raw_r, asum = orc.energy_poses(cx, pose, p, l)
            bad, rel = tol.check_terms(r["e"][k:k + 1], terms_r, raw_r, asum, cx.ff)
            assert not bad.any(), (s, int(reps[k]), np.nanmax(rel, axis=0))


def _groups_are_permutations(rec, n_prt, n_tmp, n_lig):
    it = rec["idx_tmp"].reshape(n_prt, n_tmp, n_lig, -1)
    want = np.arange(n_tmp).reshape(1, n_tmp, 1, 1)
    assert np.array_equal(np.sort(it, axis=1), np.broadcast_to(want, it.shape))


def test_headline_ensemble_full_size(ctx):
    w = synth.WORKLOADS["ensemble_4000x40"]
    cx = synth.make_complex(w.spec, seed=2024)
    _, mb = synth.temperatures(w)
    spe = w.steps_per_exchange
    steps, seed = 2 * spe, 77
    d = lib.DeviceComplex(ctx, cx)
    r = lib.Remc(d, steps, spe, mb, w.move_scale, seed=seed,
                 flags=abi.MC_EXCHANGE | abi.MC_MOVE_AWAY | abi.MC_RECORD)
    r.init()
    r.run(steps)
    out = r.read()
    r.close()
    d.close()
    rec = out.record
    assert rec.shape == (8800, steps)
    swaps = _replay_checks(cx, mb, rec, seed, spe, w.n_tmp)
    assert swaps > 0
    _groups_are_permutations(rec, cx.n_prt, w.n_tmp, cx.n_lig)
    assert out.ac_mc == int(rec["accepted"].sum())
    _sample_energies(cx, rec, np.random.Generator(np.random.PCG64(5)))


def test_batched_512_full_size(ctx):
    w = synth.WORKLOADS["batched_512"]
    raw, _, _ = synth.default_ff()
    rng = np.random.Generator(np.random.PCG64(2025))
    prt = synth.make_protein(rng, w.spec, 9.0, raw)
    lo, hi = w.extra["lna_range"]
    lnas = rng.integers(lo, hi + 1, size=w.extra["n_ligand"])
    cxs = [synth.make_complex(dataclasses.replace(w.spec, lna=int(n)), seed=2124 + i,
                              protein=prt) for i, n in enumerate(lnas)]
    _, mb = synth.temperatures(w)
    spe = w.steps_per_exchange
    steps, seed = 2 * spe, 9
    base = lib.DeviceComplex(ctx, cxs[0])
    dcxs = [lib.DeviceComplex(ctx, cx, share=base, prt_conf0=i % w.spec.n_prt, n_prt=1)
            for i, cx in enumerate(cxs)]
    params = [abi.mc_params(steps, spe, mb, w.move_scale, seed=seed, stream_id=i,
                            flags=abi.MC_EXCHANGE | abi.MC_MOVE_AWAY | abi.MC_RECORD)
              for i in range(len(dcxs))]
    b = lib.Batch(ctx, dcxs, params)
    b.init()
    b.run(steps)
    assert b.n_rep == 16384
    pick = set(np.random.Generator(np.random.PCG64(6)).choice(len(cxs), 8, replace=False))
    swaps = 0
    for i, cx in enumerate(cxs):
        out = b.read(i)
        rec = out.record
        # the item runs one protein conformation (the shared protein's
        # i % n_prt, its own conformation 0)
        shape = types.SimpleNamespace(n_prt=1, n_lig=cx.n_lig)
        swaps += _replay_checks(shape, mb, rec, seed, spe, w.n_tmp, stream=i)
        _groups_are_permutations(rec, 1, w.n_tmp, cx.n_lig)
        assert out.ac_mc == int(rec["accepted"].sum())
        if i in pick:
            _sample_energies(cx, rec, np.random.Generator(np.random.PCG64(i)), n_sample=6,
                             prt_conf0=i % w.spec.n_prt)
    assert swaps > 0
    b.close()
    for d in dcxs:
        d.close()
    base.close()


@pytest.mark.parametrize("pnp", [2000, 4000, 8000, 16000])
def test_poses_full_size(ctx, pnp):
    """The 1,048,576-pose sweep at each protein size: a seeded 4,096-pose
    subset against the oracle, term by term (raw FP64 sums too), and every
    pose's energy bit-identical whatever the order of the poses."""
    w = synth.WORKLOADS["poses_48"]
    n_pose = 1 << 20
    cx = synth.make_complex(dataclasses.replace(w.spec, pnp=pnp), seed=2024 + pnp)
    rng = np.random.default_rng(11 + pnp)
    poses = synth.random_poses(rng, n_pose, box=w.extra["box"])
    perm = rng.permutation(n_pose)
    d = lib.DeviceComplex(ctx, cx)
    pd = torch.from_numpy(poses).cuda()
    pp = torch.from_numpy(np.ascontiguousarray(poses[perm])).cuda()
    t1 = torch.empty((n_pose, abi.NTERM), dtype=torch.float32, device="cuda")
    t2 = torch.empty_like(t1)
    r1 = torch.empty((n_pose, abi.NRAW), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()  # the inputs were copied on torch's stream
    d.energy_poses_dev(n_pose, pd.data_ptr(), t1.data_ptr(), r1.data_ptr())
    d.energy_poses_dev(n_pose, pp.data_ptr(), t2.data_ptr())
    ctx.sync()
    a, b, raw = t1.cpu().numpy(), t2.cpu().numpy(), r1.cpu().numpy()
    d.close()
    assert np.isfinite(a).all()
    assert np.array_equal(a[perm], b)
    idx = rng.choice(n_pose, w.extra["parity_subset"], replace=False)
    terms_r, raw_r, asum = orc.energy_poses(cx, poses[idx])
    bad, rel = tol.check_raw(raw[idx], raw_r, asum)
    assert not bad.any(), np.nanmax(rel, axis=0)
    bad, rel = tol.check_terms(a[idx], terms_r, raw_r, asum, cx.ff)
    assert not bad.any(), np.nanmax(rel, axis=0)
