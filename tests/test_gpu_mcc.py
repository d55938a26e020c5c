"""Contact-map MCC score (GD_MC_MCC) of the REMC path against the oracle.

The reference computes it every MC step for the new pose and carries it
with the accepted state (calcmcc_d.cu:148-213, accept_d.cu:50); the per-step
record holds the accepted state's value.  Each recorded value is recomputed
on the oracle from the recorded pose.  A contact is d <= pmf0, a step
function of the distance, so a pair within rounding of pmf0 may fall on
different sides on the CPU and the GPU: such flips are rare and move the
score by about one contact's worth."""
import numpy as np
import pytest

from gpudock_b200 import abi, lib, synth
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _run(flags, n_prt=2, n_lig=3, seed=31):
    ctx = lib.Context(0)
    cx = synth.make_complex(synth.ComplexSpec(pnp=600, lna=16, n_prt=n_prt, n_lig=n_lig), seed=seed)
    _, mb = lib.set_temperature(4, 0.004, 0.04)
    d = lib.DeviceComplex(ctx, cx)
    steps = 40
    r = lib.Remc(d, steps, 10, mb, seed=5, flags=flags)
    r.init()
    r.run(steps)
    return cx, r.read()


def test_mcc_record_matches_oracle():
    flags = abi.MC_EXCHANGE | abi.MC_MOVE_AWAY | abi.MC_RECORD | abi.MC_MCC
    cx, out = _run(flags)
    rec = out.record
    got = rec["cmcc"].ravel()
    ref = np.array([orc.mcc(cx, 0, int(p), int(l), m) for p, l, m in
                    zip(rec["idx_prt"].ravel(), rec["idx_lig"].ravel(),
                        rec["movematrix"].reshape(-1, 6))], np.float32)
    assert np.all(np.isfinite(got))
    assert (got != abi.CMCC_INVALID).any() and np.unique(got).size > 5
    exact = got == ref
    assert exact.mean() >= 0.98, f"{(~exact).sum()} of {exact.size} differ"
    assert np.abs(got - ref).max() <= 0.1


def test_mcc_off_records_zero():
    cx, out = _run(abi.MC_EXCHANGE | abi.MC_RECORD, n_prt=1, n_lig=2, seed=32)
    assert np.all(out.record["cmcc"] == 0.0)


def test_mcc_does_not_change_the_trajectory():
    base = abi.MC_EXCHANGE | abi.MC_MOVE_AWAY | abi.MC_RECORD
    _, a = _run(base, seed=33)
    _, b = _run(base | abi.MC_MCC, seed=33)
    assert np.array_equal(a.energy, b.energy)
    assert np.array_equal(a.movematrix, b.movematrix)
    assert np.array_equal(a.record["accepted"], b.record["accepted"])
