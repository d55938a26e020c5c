"""Pose-energy parity: the sm_100a kernel (through the C-ABI) vs the CPU oracle.

The oracle restates calcenergy_d.cu with FP32 pair arithmetic and FP64 sums;
the kernel must agree per term within the tolerance of tests/tolerance.py
(1e-5 relative, cancellation-aware).
"""
import numpy as np
import pytest

from gpudock_b200 import abi, lib, synth
from oracle import oracle as orc
from tests import tolerance as tol

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = lib.Context(0)
    yield c
    c.close()


def _compare(cx, terms_g, raw_g, poses, prt_conf=0, lig_conf=0):
    terms_r, raw_r, asum = orc.energy_poses(cx, poses, prt_conf, lig_conf)
    bad_raw, rel_raw = tol.check_raw(raw_g, raw_r, asum)
    bad_t, rel_t = tol.check_terms(terms_g, terms_r, raw_r, asum, cx.ff)
    assert not bad_raw.any(), (
        f"raw terms off at {np.argwhere(bad_raw)[:5]}: worst rel {np.nanmax(rel_raw, axis=0)}")
    assert not bad_t.any(), (
        f"terms off at {np.argwhere(bad_t)[:5]}: worst rel {np.nanmax(rel_t, axis=0)}")
    return rel_raw, rel_t


def test_energy_small_complex(ctx):
    cx = synth.make_complex(synth.ComplexSpec(pnp=1500, lna=24, cube=40.0), seed=11)
    d = lib.DeviceComplex(ctx, cx)
    rng = np.random.default_rng(1)
    poses = synth.random_poses(rng, 257, box=3.0)
    poses[0] = 0.0
    terms, raw = d.energy_poses(poses)
    _compare(cx, terms, raw, poses)


def test_energy_streamed_protein(ctx):
    """8,000 points exceed the resident limit: tiles stream through the ring."""
    cx = synth.make_complex(synth.ComplexSpec(pnp=8000, lna=48), seed=12)
    d = lib.DeviceComplex(ctx, cx)
    poses = synth.random_poses(np.random.default_rng(2), 96, box=8.0)
    terms, raw = d.energy_poses(poses)
    _compare(cx, terms, raw, poses)


@pytest.mark.parametrize("lna", [1, 7, 96, 120])
def test_energy_ligand_sizes(ctx, lna):
    cx = synth.make_complex(synth.ComplexSpec(pnp=700, lna=lna), seed=100 + lna)
    d = lib.DeviceComplex(ctx, cx)
    poses = synth.random_poses(np.random.default_rng(lna), 40, box=4.0)
    terms, raw = d.energy_poses(poses)
    _compare(cx, terms, raw, poses)


def hbond_types(cx):
    """Ligand types with an H-bond term for some point type (hdb0 > 0.1), and the rest."""
    hd = np.ctypeslib.as_array(cx.ff.hdb0)[:abi.NLT]
    cap = (hd > 0.1).any(axis=1)
    return np.nonzero(cap)[0].astype(np.int32), np.nonzero(~cap)[0].astype(np.int32)


def with_ligand_types(cx, pick):
    """The complex with its ligand types replaced by draws from `pick`."""
    rng = np.random.default_rng(int(cx.lig_t.sum()))
    cx.lig_t = rng.choice(pick, size=len(cx.lig_t)).astype(np.int32)
    cx._struct = None
    return cx


@pytest.mark.parametrize("which", ["all", "none"])
@pytest.mark.parametrize("lna", [16, 40, 80])
def test_energy_hbond_atom_counts(ctx, which, lna):
    """Every atom with an H-bond term (the launch evaluates it for every atom
    pair) or none (only the term-free chunk body runs)."""
    cx = synth.make_complex(synth.ComplexSpec(pnp=1100, lna=lna), seed=200 + lna)
    cap, free = hbond_types(cx)
    with_ligand_types(cx, cap if which == "all" else free)
    d = lib.DeviceComplex(ctx, cx)
    poses = synth.random_poses(np.random.default_rng(lna), 64, box=3.0)
    terms, raw = d.energy_poses(poses)
    _compare(cx, terms, raw, poses)
    if which == "none":
        assert np.all(raw[:, abi.E_HDB] == 0.0)
    else:
        assert np.any(raw[:, abi.E_HDB] != 0.0)


def test_energy_conformations(ctx):
    cx = synth.make_complex(synth.ComplexSpec(pnp=900, lna=20, n_prt=3, n_lig=4), seed=13)
    d = lib.DeviceComplex(ctx, cx)
    poses = synth.random_poses(np.random.default_rng(3), 33, box=4.0)
    for pc in range(3):
        for lc in (0, 3):
            terms, raw = d.energy_poses(poses, prt_conf=pc, lig_conf=lc)
            _compare(cx, terms, raw, poses, pc, lc)


def test_energy_edge_counts(ctx):
    cx = synth.make_complex(synth.ComplexSpec(pnp=300, lna=10), seed=14)
    d = lib.DeviceComplex(ctx, cx)
    t0, r0 = d.energy_poses(np.zeros((0, 6), np.float32))
    assert t0.shape == (0, 10)
    for n in (1, 31, 32, 33, 65):
        poses = synth.random_poses(np.random.default_rng(n), n, box=4.0)
        terms, raw = d.energy_poses(poses)
        _compare(cx, terms, raw, poses)


def test_energy_no_kde_no_mcs(ctx):
    """pnk = 0 gives ekde = 0; pos = 0 gives log(0/0) = NaN, as the reference."""
    cx = synth.make_complex(synth.ComplexSpec(pnp=400, lna=12), seed=15)
    cx.kde_xyz = np.zeros((0, 3), np.float32)
    cx.kde_t = np.zeros(0, np.int32)
    cx.mcs_xyz = np.zeros((0, cx.mcs_xyz.shape[1], 3), np.float32)
    cx.mcs_tcc = np.zeros(0, np.float32)
    cx._struct = None
    d = lib.DeviceComplex(ctx, cx)
    poses = synth.random_poses(np.random.default_rng(5), 8, box=4.0)
    terms, raw = d.energy_poses(poses)
    terms_r, raw_r, asum = orc.energy_poses(cx, poses)
    assert np.all(raw[:, abi.E_KDE] == 0.0) and np.all(raw_r[:, abi.E_KDE] == 0.0)
    assert np.all(np.isnan(raw[:, abi.E_LHM])) and np.all(np.isnan(raw_r[:, abi.E_LHM]))
    assert np.all(np.isnan(terms[:, abi.E_TOTAL])) and np.all(np.isnan(terms_r[:, abi.E_TOTAL]))
    keep = [0, 1, 2, 3, 4, 5, 6, 8]
    bad, rel = tol.check_raw(raw[:, keep], raw_r[:, keep],
                             np.concatenate([asum, np.zeros((len(asum), 4))], axis=1)[:, keep])
    assert not bad.any(), rel.max(axis=0)


def test_energy_invalid_inputs(ctx):
    cx = synth.make_complex(synth.ComplexSpec(pnp=200, lna=8), seed=16)
    d = lib.DeviceComplex(ctx, cx)
    with pytest.raises(lib.GdError) as e:
        d.energy_poses(np.zeros((4, 6), np.float32), prt_conf=1)
    assert e.value.status == abi.GD_EINVAL
    bad = synth.make_complex(synth.ComplexSpec(pnp=200, lna=8), seed=16)
    bad.lig_t = bad.lig_t.copy()
    bad.lig_t[0] = 99
    bad._struct = None
    with pytest.raises(lib.GdError) as e:
        lib.DeviceComplex(ctx, bad)
    assert e.value.status == abi.GD_EINVAL


def test_golden_line_on_gpu(ctx):
    """The 1a07C1 sample complex (tables from the reference's own loaders):
    the kernel reproduces the published initial-energy line
    (SimilarityMatirxGen/data/report:21-22) to its four decimals, through the
    MonteCarlo_Init_d path (move-away pose, forced accept)."""
    from tests.golden_fixture import golden_lines, load_complex
    cx, _, _ = load_complex("smg")
    g = np.array(golden_lines()["report"])
    d = lib.DeviceComplex(ctx, cx)
    pose = (np.float32([0.02, 0.02, 0.02, 0.08, 0.08, 0.08]) * np.float32(44.5)).reshape(1, 6)
    terms, raw = d.energy_poses(pose)
    assert np.allclose(np.round(terms[0].astype(np.float64), 4), g, atol=1.01e-4), terms[0]
    _, mb = lib.set_temperature(1, 0.044, 0.036)
    r = lib.Remc(d, 10, 10, mb, flags=abi.MC_MOVE_AWAY)
    r.init()
    out = r.read()
    assert np.allclose(np.round(out.energy[0].astype(np.float64), 4), g, atol=1.01e-4)
