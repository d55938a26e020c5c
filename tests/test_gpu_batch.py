"""Batched form: many complexes of uneven sizes in one run.

Every complex keeps its own random stream (seed, stream id) and its local
replica numbering, so its trajectory in the batch must be bit-identical to
running it alone in the plain form, whatever else shares the launch."""
import numpy as np
import pytest

from gpudock_b200 import abi, lib, synth
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = lib.Context(0)
    yield c
    c.close()


def _ligand_set(protein_spec, lnas, seed):
    """Complexes of one protein (shared upload) and ligands of uneven sizes."""
    raw, _, _ = synth.default_ff()
    rng = np.random.Generator(np.random.PCG64(seed))
    prt = synth.make_protein(rng, protein_spec, 8.0, raw)
    out = []
    for i, lna in enumerate(lnas):
        spec = synth.ComplexSpec(pnp=protein_spec.pnp, lna=lna, n_prt=protein_spec.n_prt,
                                 n_lig=4)
        out.append(synth.make_complex(spec, seed=seed + 17 * i, protein=prt))
    return out


@pytest.mark.parametrize("n_tmp", [8, 6])
def test_batch_equals_alone(ctx, n_tmp):
    """8 temperatures: whole groups per CTA, exchange inside the kernel;
    6 temperatures: separate exchange kernel replayed from a CUDA graph."""
    pspec = synth.ComplexSpec(pnp=900, lna=8, n_prt=2)
    cxs = _ligand_set(pspec, [12, 33, 57, 96], seed=40)
    _, mb = lib.set_temperature(n_tmp, 0.004, 0.04)
    base = lib.DeviceComplex(ctx, cxs[0])
    dcxs = [lib.DeviceComplex(ctx, cx, share=base, prt_conf0=i % 2, n_prt=1)
            for i, cx in enumerate(cxs)]
    steps, spe = 40, 10
    params = [abi.mc_params(steps, spe, mb, seed=7, stream_id=100 + i,
                            flags=abi.MC_EXCHANGE | abi.MC_MOVE_AWAY) for i in range(len(cxs))]
    b = lib.Batch(ctx, dcxs, params)
    assert b.n_rep == sum(4 * n_tmp for _ in cxs)
    b.init()
    b.run(20)
    b.run(20)
    for i, d in enumerate(dcxs):
        got = b.read(i)
        r = lib.Remc(d, steps, spe, mb, seed=7, stream_id=100 + i,
                     flags=abi.MC_EXCHANGE | abi.MC_MOVE_AWAY)
        r.init()
        r.run(steps)
        alone = r.read()
        assert np.array_equal(got.energy, alone.energy), i
        assert np.array_equal(got.movematrix, alone.movematrix), i
        assert np.array_equal(got.idx_tmp, alone.idx_tmp), i
        assert got.ac_mc == alone.ac_mc and got.ac_temp_exchg == alone.ac_temp_exchg


def test_batch_hbond_mix_equals_alone(ctx):
    """A ligand with an H-bond term on every atom and one with none share a
    launch (same size bucket): the launch evaluates the term for every atom
    pair, the term-free ligand alone skips it; trajectories stay identical."""
    from tests.test_gpu_energy import hbond_types, with_ligand_types
    pspec = synth.ComplexSpec(pnp=900, lna=8, n_prt=1)
    cxs = _ligand_set(pspec, [40, 40], seed=44)
    cap, free = hbond_types(cxs[0])
    with_ligand_types(cxs[0], cap)
    with_ligand_types(cxs[1], free)
    _, mb = lib.set_temperature(8, 0.004, 0.04)
    base = lib.DeviceComplex(ctx, cxs[0])
    dcxs = [base, lib.DeviceComplex(ctx, cxs[1], share=base)]
    steps, spe = 30, 10
    flags = abi.MC_EXCHANGE | abi.MC_MOVE_AWAY
    params = [abi.mc_params(steps, spe, mb, seed=9, stream_id=i, flags=flags) for i in range(2)]
    b = lib.Batch(ctx, dcxs, params)
    b.init()
    b.run(steps)
    for i, d in enumerate(dcxs):
        got = b.read(i)
        r = lib.Remc(d, steps, spe, mb, seed=9, stream_id=i, flags=flags)
        r.init()
        r.run(steps)
        alone = r.read()
        assert np.array_equal(got.energy, alone.energy), i
        assert np.array_equal(got.movematrix, alone.movematrix), i
    # the normalised H-bond term is constant (a * 0 + b) without H-bond atoms
    assert np.unique(b.read(1).energy[..., abi.E_HDB]).size == 1
    assert np.unique(b.read(0).energy[..., abi.E_HDB]).size > 1


def test_batch_replay_against_oracle(ctx):
    """Decisions of a batched complex replay bit-exactly on the oracle."""
    pspec = synth.ComplexSpec(pnp=600, lna=8, n_prt=1)
    cxs = _ligand_set(pspec, [20, 45], seed=41)
    _, mb = lib.set_temperature(8, 0.004, 0.04)
    base = lib.DeviceComplex(ctx, cxs[0])
    dcxs = [base, lib.DeviceComplex(ctx, cxs[1], share=base, prt_conf0=0, n_prt=1)]
    steps, spe = 30, 10
    params = [abi.mc_params(steps, spe, mb, seed=3, stream_id=i,
                            flags=abi.MC_EXCHANGE | abi.MC_RECORD) for i in range(2)]
    b = lib.Batch(ctx, dcxs, params)
    b.init()
    b.run(steps)
    for i in range(2):
        rec = b.read(i).record
        ref = orc.metropolis(rec["e_prop_total"].reshape(-1),
                             rec["e"][..., abi.E_TOTAL].reshape(-1),
                             mb[rec["idx_tmp"].reshape(-1)], 3, i, rec["idx_rep"].reshape(-1),
                             rec["step"].reshape(-1))
        assert np.array_equal(ref, rec["accepted"].reshape(-1))


def test_batch_rejects_mixed_cadence(ctx):
    cxs = _ligand_set(synth.ComplexSpec(pnp=300, lna=8), [10, 11], seed=42)
    _, mb = lib.set_temperature(4, 0.01, 0.05)
    d = [lib.DeviceComplex(ctx, cx) for cx in cxs]
    params = [abi.mc_params(20, 10, mb), abi.mc_params(20, 5, mb)]
    with pytest.raises(lib.GdError) as e:
        lib.Batch(ctx, d, params)
    assert e.value.status == abi.GD_EINVAL


def test_autotune_picks_a_covering_shape(ctx):
    cx = synth.make_complex(synth.ComplexSpec(pnp=1500, lna=40), seed=43)
    d = lib.DeviceComplex(ctx, cx)
    (A, P, NA), ms = d.autotune()
    assert A * NA >= 40 and A * P <= 12 and ms > 0
    # the tuned shape is used afterwards and gives the same energies
    poses = synth.random_poses(np.random.default_rng(0), 64, box=3.0)
    t, raw = d.energy_poses(poses)
    tr, rr, asum = orc.energy_poses(cx, poses)
    from tests import tolerance as tol
    bad, rel = tol.check_terms(t, tr, rr, asum, cx.ff)
    assert not bad.any(), rel.max(axis=0)
