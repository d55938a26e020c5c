"""Bayesian total (GD_MC_BAYES, the reference's IS_BAYE,
calcenergy_d.cu:311-347) on the REMC path against the oracle.

The kernel's total of every recorded accepted state must be the oracle's
Bayesian total of the same nine normalised terms (CUDA's expf / powf /
log10f against the host libm's: a few float32 ulps per density), every
Metropolis decision must replay bit-exactly on the oracle from the recorded
totals, and the terms themselves are those of the weighted-total run.

The densities were fitted to normalised terms of poses in the pocket; far
from it (the move-away start pose, say) they underflow to 0 and the total is
-inf, +inf or NaN, in the reference as here (such a proposal is rejected, a
non-finite current state is left at the first finite proposal).  The runs
start at the crystal pose, where most totals are finite."""
import numpy as np
import pytest

from gpudock_b200 import abi, lib, synth
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _run(ctx, cx, flags, seed=17):
    _, mb = lib.set_temperature(8, 0.004, 0.04)
    d = lib.DeviceComplex(ctx, cx)
    r = lib.Remc(d, 40, 10, mb, seed=seed, flags=flags)
    r.init()
    r.run(40)
    out = r.read()
    r.close()
    return out, mb


def test_bayes_total_matches_oracle_and_decisions_replay():
    ctx = lib.Context(0)
    cx = synth.make_complex(synth.ComplexSpec(pnp=900, lna=26, n_prt=2, n_lig=4), seed=71)
    flags = abi.MC_EXCHANGE | abi.MC_RECORD | abi.MC_BAYES
    out, mb = _run(ctx, cx, flags)
    rec = out.record.reshape(-1)
    e = rec["e"]
    want = orc.bayes_total(e)
    got = e[:, abi.E_TOTAL]
    fin = np.isfinite(got) & np.isfinite(want)
    assert fin.mean() > 0.5
    # non-finite in the same places, up to densities at the edge of underflow
    assert (np.isfinite(got) != np.isfinite(want)).mean() < 0.01
    assert np.allclose(got[fin], want[fin], rtol=1e-5, atol=1e-4), np.abs(got - want)[fin].max()
    # the Bayesian total is not the weighted sum
    w = np.ctypeslib.as_array(cx.ff.w)[:9]
    assert not np.allclose(got[fin], (e[fin, :9] * w).sum(axis=1), atol=1e-3)
    # decisions from the recorded totals
    ref = orc.metropolis(rec["e_prop_total"], got, mb[rec["idx_tmp"]], 17, 0, rec["idx_rep"],
                         rec["step"])
    assert np.array_equal(ref, rec["accepted"])
    assert 0 < rec["accepted"].mean() < 1
    ctx.close()


def test_bayes_keeps_the_terms():
    """Only the total differs: the first step's proposals (same moves, same
    random numbers) have the same nine terms with and without the flag."""
    ctx = lib.Context(0)
    cx = synth.make_complex(synth.ComplexSpec(pnp=600, lna=18, n_prt=1, n_lig=4), seed=72)
    base = abi.MC_EXCHANGE | abi.MC_RECORD
    a, _ = _run(ctx, cx, base)
    b, _ = _run(ctx, cx, base | abi.MC_BAYES)
    # step 0 records the start state, whose terms do not depend on the total
    assert np.array_equal(a.record[:, 0]["e"][:, :9], b.record[:, 0]["e"][:, :9])
    assert not np.array_equal(a.record[:, 0]["e"][:, 9], b.record[:, 0]["e"][:, 9])
    ctx.close()
