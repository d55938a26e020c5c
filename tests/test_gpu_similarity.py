"""Contact-mode similarity matrix on the GPU (gd_similarity_matrix): bit for
bit the oracle's values, on the reference's 100-conformation sample (and so
within print precision of the matrix the reference wrote for it) and on a
larger synthetic trajectory, including conformations without contacts, a
single conformation and the argument checks."""
import numpy as np
import pytest
import torch

from gpudock_b200 import abi, lib, synth
from oracle import oracle as orc
from tests.golden_fixture import load_complex
from tests.test_similarity import golden, printed_tolerance

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = lib.Context(0)
    yield c
    c.close()


def test_reference_sample(ctx):
    cx, _, _ = load_complex("smg")
    confs, want = golden()
    d = lib.DeviceComplex(ctx, cx)
    S = d.similarity_matrix(confs)
    # the device-output entry point writes the same matrix
    out = torch.full((len(confs), len(confs)), -1.0, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    d.similarity_matrix_dev(confs, out.data_ptr())
    d.close()
    assert np.array_equal(out.cpu().numpy(), S)
    assert np.array_equal(S, orc.similarity_matrix(cx, confs))
    assert np.all(np.abs(S - want) <= printed_tolerance(want))


def test_synthetic_trajectory(ctx):
    """600 conformations of a 40-atom ligand against a 4,000-point protein
    with 3 conformations: moves of a few angstroms and tenths of a radian
    about the pocket (overlapping sparse maps), two far away (no contacts)."""
    cx = synth.make_complex(synth.ComplexSpec(pnp=4000, lna=40, n_prt=3, n_lig=6), seed=31)
    rng = np.random.Generator(np.random.PCG64(32))
    n = 600
    confs = np.zeros((n, 8), np.float32)
    confs[:, 0] = rng.integers(0, 3, n)
    confs[:, 1] = rng.integers(0, 6, n)
    confs[:, 2:5] = rng.normal(0.0, 1.5, (n, 3))
    confs[:, 5:8] = rng.normal(0.0, 0.3, (n, 3))
    confs[[17, 400], 2] = 500.0
    d = lib.DeviceComplex(ctx, cx)
    S = d.similarity_matrix(confs)
    ref = orc.similarity_matrix(cx, confs)
    assert np.array_equal(S, ref)
    assert np.all(S[17] == 10000.0) and np.all(S[:, 400] == 10000.0)
    ok = np.delete(np.delete(S, [17, 400], axis=0), [17, 400], axis=1)
    # a map against itself: 1 up to the rounding of the float product of the
    # four sums (the reference's arithmetic)
    assert np.allclose(np.diag(ok), 1.0, rtol=0, atol=2.5e-7)
    assert (ok < 0.99).any() and (ok > 0.0).any()
    # a single conformation, and none
    assert np.array_equal(d.similarity_matrix(confs[:1]), ref[:1, :1])
    assert d.similarity_matrix(np.zeros((0, 8), np.float32)).shape == (0, 0)
    d.close()


def test_argument_checks(ctx):
    cx, _, _ = load_complex("smg")
    confs, _ = golden()
    d = lib.DeviceComplex(ctx, cx)
    for row, col, val in ((0, 0, float(cx.n_prt)), (1, 1, float(cx.n_lig)), (2, 0, -1.0),
                          (3, 5, np.nan)):
        bad = confs[:4].copy()
        bad[row, col] = val
        with pytest.raises(lib.GdError) as e:
            d.similarity_matrix(bad)
        assert e.value.status == abi.GD_EINVAL
    # the context still works afterwards
    assert np.array_equal(d.similarity_matrix(confs[:3]), orc.similarity_matrix(cx, confs[:3]))
    d.close()


def test_ragged_sizes_and_shared_protein(ctx):
    """A 120-atom ligand against 1,000 points (the last word of every atom
    row is part padding), and a complex that uses another's protein
    conformation 1 as its own conformation 0."""
    raw, _, _ = synth.default_ff()
    rng = np.random.Generator(np.random.PCG64(34))
    prt = synth.make_protein(rng, synth.ComplexSpec(pnp=1000, lna=8, n_prt=2), 8.0, raw)
    a = synth.make_complex(synth.ComplexSpec(pnp=1000, lna=120, n_prt=2, n_lig=2), seed=35,
                           protein=prt)
    b = synth.make_complex(synth.ComplexSpec(pnp=1000, lna=33, n_prt=2, n_lig=3), seed=36,
                           protein=prt)
    n = 150
    confs = np.zeros((n, 8), np.float32)
    confs[:, 1] = rng.integers(0, 2, n)
    confs[:, 2:5] = rng.normal(0.0, 1.0, (n, 3))
    confs[:, 5:8] = rng.normal(0.0, 0.2, (n, 3))
    da = lib.DeviceComplex(ctx, a)
    confs[:, 0] = rng.integers(0, 2, n)
    assert np.array_equal(da.similarity_matrix(confs), orc.similarity_matrix(a, confs))
    db = lib.DeviceComplex(ctx, b, share=da, prt_conf0=1, n_prt=1)
    cb = confs.copy()
    cb[:, 0] = 0
    cb[:, 1] = rng.integers(0, 3, n)
    ref = cb.copy()
    ref[:, 0] = 1  # conformation 0 of the shared view is the protein's conformation 1
    assert np.array_equal(db.similarity_matrix(cb), orc.similarity_matrix(b, ref))
    db.close()
    da.close()
