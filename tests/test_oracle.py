"""CPU tests: the oracle pinned to the reference's own outputs and to the
independent Philox implementation, and the host side of the library."""
import json
import math
import os

import numpy as np
import pytest

from gpudock_b200 import abi, forcefield, lib, synth
from oracle import oracle as orc
from tests.golden_fixture import HERE as GOLDEN, golden_lines, load_complex


def test_philox_known_answers():
    """Philox4x32-10 of the oracle vs vectors made with the Random123 header
    the reference vendors (tests/golden/make_philox_golden.py)."""
    with open(os.path.join(GOLDEN, "philox4x32_10.json")) as f:
        d = json.load(f)
    got = orc.philox(np.array(d["ctr"], np.uint32), np.array(d["key"], np.uint32))
    assert np.array_equal(got, np.array(d["out"], np.uint32))


def test_decision_exp_accuracy():
    x = np.concatenate([np.linspace(-87, 88, 20001), np.random.default_rng(0).normal(0, 3, 5000)])
    x = x.astype(np.float32)
    got = orc.expf(x).astype(np.float64)
    ref = np.exp(x.astype(np.float64))
    rel = np.abs(got - ref) / ref
    assert rel.max() < 4e-7
    assert orc.expf(np.array([0.0], np.float32))[0] == 1.0
    assert orc.expf(np.array([100.0], np.float32))[0] == np.inf
    assert orc.expf(np.array([-100.0], np.float32))[0] == 0.0
    assert math.isnan(orc.expf(np.array([np.nan], np.float32))[0])


def test_oracle_reproduces_report_line():
    """GeauxDock v0 sample (SimilarityMatirxGen/data/report:21-22): the initial
    energy of replica 0 after MoveAway (perturbation 44.5 x move scale
    0.02 A / 0.08 rad), tables from the reference's own loaders.  All ten terms
    agree to the four printed decimals."""
    cx, _, _ = load_complex("smg")
    g = np.array(golden_lines()["report"])
    pose = (np.float32([0.02, 0.02, 0.02, 0.08, 0.08, 0.08]) * np.float32(44.5)).reshape(1, 6)
    terms, _, _ = orc.energy_poses(cx, pose, prt_conf=0, lig_conf=0)
    assert np.allclose(np.round(terms[0].astype(np.float64), 4), g, atol=1.01e-4), terms[0]


def test_oracle_reproduces_instruction_pair_terms():
    """SimilarityMatirxGen/doc/instructions.txt:156-159: at the crystal pose
    the four pair terms (vdw, ele, pmf, hdb) agree to four decimals.  The
    other six printed terms come from an older normalisation of psp, hpc,
    kde, lhm and dst than the one in the kernels of this path."""
    cx, _, _ = load_complex("smg")
    g = np.array(golden_lines()["instructions"])
    terms, _, _ = orc.energy_poses(cx, np.zeros((1, 6), np.float32))
    for i in (abi.E_VDW, abi.E_ELE, abi.E_PMF, abi.E_HDB):
        assert abs(round(float(terms[0, i]), 4) - g[i]) <= 1.01e-4, (i, terms[0, i], g[i])


def test_fixture_init_coords_match_reference():
    """InitLigCoord's coord_new equals the oracle's placement at m = 0."""
    cx, _, z = load_complex("smg")
    new = z["lig_new_xyz"]
    ref = cx.lig_xyz + cx.lig_center
    assert np.array_equal(new.astype(np.float32), ref.astype(np.float32))


def test_forcefield_parser_matches_reference_loader():
    """The packaged FF (our .ff parser) equals loadEnePara+loadWeight+
    loadNorPara's raw table from the reference fixture (rem test inputs)."""
    _, raw_ref, _ = load_complex("rem")
    mine = forcefield.raw_struct(forcefield.load_raw())
    a = np.frombuffer(bytes(mine), np.float32)
    b = np.frombuffer(bytes(raw_ref), np.float32)
    # w[9], a_para[9], b_para[9] are never read by the energy (9 terms)
    names = [n for n, _ in abi.GdEneparaRaw._fields_]
    for n in names:
        off = getattr(abi.GdEneparaRaw, n).offset // 4
        size = abi.C.sizeof(dict(abi.GdEneparaRaw._fields_)[n]) // 4
        x, y = a[off:off + size], b[off:off + size]
        if n in ("w", "a_para", "b_para"):
            x, y = x[:9], y[:9]
        assert np.array_equal(x, y), n


def test_enepara_optimize_library_equals_oracle_and_reference():
    cx, raw_ref, z = load_complex("rem")
    mine = lib.enepara_optimize(raw_ref)
    theirs = orc.enepara_optimize(raw_ref)
    assert bytes(mine) == bytes(theirs)
    # and equals the reference's own OptimizeEnepara output (hdb2 included)
    ref = np.frombuffer(z["enepara"].tobytes(), np.float32)
    got = np.frombuffer(bytes(mine), np.float32)
    assert np.array_equal(got[:len(ref)], ref[:len(got)])


def test_set_temperature_matches_oracle():
    for n, lo, hi in [(1, 0.3, 0.3), (8, 0.004, 0.04), (16, 0.004, 0.08), (40, 0.001, 1.0)]:
        t1, m1 = lib.set_temperature(n, lo, hi)
        t2, m2 = orc.set_temperature(n, lo, hi)
        assert np.array_equal(m1, m2) and np.array_equal(t1, t2)
    assert np.isclose(lib.set_temperature(8, 0.004, 0.04)[0][-1], 0.04, rtol=1e-5)


def test_oracle_remc_runs_and_counts():
    """The oracle's own REMC driver: counters consistent with the record."""
    cx = synth.make_complex(synth.ComplexSpec(pnp=200, lna=8, n_lig=2), seed=5)
    _, mb = lib.set_temperature(4, 0.01, 0.05)
    out = orc.remc_run(cx, 40, 10, mb, seed=3, flags=abi.MC_EXCHANGE | abi.MC_RECORD)
    rec = out.record
    assert rec.shape == (8, 40)
    assert out.ac_mc == int(rec["accepted"].sum())
    assert sorted(out.idx_tmp[[0, 2, 4, 6]].tolist()) == [0, 1, 2, 3]
    assert (rec["step"] == np.arange(40)).all()


def _bayes_reference_f64(e):
    """IS_BAYE total from scipy's standard densities (float64): normal,
    Cauchy, logistic and Wald (inverse Gaussian with mean 1) in loc/scale
    form, with the parameter sets and pairings of distribution.h and
    calcenergy_d.cu:311-347 (low H-bond: normal with the "logistic"
    parameters; low PSP: logistic with the "Laplace" parameters; a Wald
    argument below loc has density 1e-8).  The parameters are the
    reference's float literals, so they are rounded to float32 first: near
    a Wald location the rounding of loc alone moves log10 by ~1e-4."""
    from scipy import stats as st

    def f32(v):
        return float(np.float32(v))

    def norm(x, loc, scale):
        return st.norm.pdf(x, f32(loc), f32(scale))

    def cauchy(x, loc, scale):
        return st.cauchy.pdf(x, f32(loc), f32(scale))

    def logistic(x, loc, scale):
        return st.logistic.pdf(x, f32(loc), f32(scale))

    def wald(x, loc, scale):
        return st.wald.pdf(x, f32(loc), f32(scale)) if x >= f32(loc) else 1e-8

    vdw, ele, pmf, psp, hdb, hpc, kde, lhm, dst = (float(v) for v in e[:9])
    high = [norm(vdw, 0.05286683, 0.29916642), cauchy(ele, -0.3653806, 0.00681102),
            logistic(pmf, -0.0221777, 0.11847532), wald(hpc, -1.0041231, 0.1151713),
            norm(hdb, 0.60986808, 0.30974999), logistic(dst, -0.8246522, 0.05218529),
            logistic(psp, -0.2346999, 0.09871713), wald(kde, -1.0112055, 0.09882933),
            logistic(lhm, -0.3377100, 0.09282947)]
    low = [norm(vdw, 0.15818486, 0.29032471), cauchy(ele, -0.3647824, 0.00534225),
           logistic(pmf, 0.04257942, 0.08801551), wald(hpc, -1.0019512, 0.10312611),
           norm(hdb, 0.76967708, 0.11224029), logistic(dst, -0.7509618, 0.08757299),
           logistic(psp, -0.2022064, 0.07854212), wald(kde, -1.004605, 0.02967548),
           logistic(lhm, -0.2387023, 0.12134983)]
    lh, ll = np.log10(high), np.log10(low)
    return ll.sum() - lh.sum(), np.abs(lh).sum() + np.abs(ll).sum()


def test_oracle_bayes_total_matches_standard_densities():
    rng = np.random.default_rng(12)
    locs = np.array([0.1, -0.365, 0.0, -0.22, 0.7, -0.95, -0.9, -0.3, -0.8], np.float32)
    e = (locs + rng.normal(0, 0.1, (200, 9))).astype(np.float32)
    e[:5, 5] = -1.2  # Wald below its loc: density 1e-8
    got = orc.bayes_total(e)
    for row, g in zip(e, got):
        ref, mag = _bayes_reference_f64(row)
        assert abs(float(g) - ref) <= 2e-6 * mag + 1e-5, (row, g, ref)


def test_oracle_mcc_bookkeeping():
    """GD_MC_MCC in the oracle's REMC driver: every recorded value is the MCC of
    the recorded (accepted) pose; the start pose of ligand conformation 0 against
    protein conformation 0 is the reference map itself (MCC 1); the score never
    changes the trajectory."""
    cx = synth.make_complex(synth.ComplexSpec(pnp=300, lna=10, n_prt=2, n_lig=2), seed=6)
    _, mb = lib.set_temperature(4, 0.01, 0.05)
    assert orc.mcc(cx, 0, 0, 0, np.zeros(6)) == 1.0
    base = abi.MC_EXCHANGE | abi.MC_RECORD | abi.MC_MOVE_AWAY
    a = orc.remc_run(cx, 20, 5, mb, seed=4, flags=base)
    b = orc.remc_run(cx, 20, 5, mb, seed=4, flags=base | abi.MC_MCC)
    assert np.array_equal(a.energy, b.energy) and np.all(a.record["cmcc"] == 0)
    rec = b.record
    for r in range(0, rec.shape[0], 3):
        for s in (0, 7, 19):
            x = rec[r, s]
            assert x["cmcc"] == orc.mcc(cx, 0, int(x["idx_prt"]), int(x["idx_lig"]),
                                        x["movematrix"])


def test_exchange_rules():
    """Pairing of exchangereplicas_d.cu:43-46: (0,1),(2,3).. for mode 0,
    (1,2),(3,4).. for mode 1; an infinitely favourable swap always happens."""
    n_tmp = 6
    mb = -np.arange(1, n_tmp + 1, dtype=np.float32)
    params, _ = abi.mc_params(10, 10, mb, seed=1)
    # delta = (mb1 - mb2)(E2 - E1) = 10 > 0 for every adjacent pair -> swap
    et = np.array([10.0, 20, 30, 40, 50, 60], np.float32)
    it0 = np.arange(n_tmp, dtype=np.int32)
    it, acs = orc.exchange(params, 1, 1, n_tmp, 0, 0, et, it0)
    assert it.tolist() == [1, 0, 3, 2, 5, 4] and acs.tolist() == [1] * 6
    it, acs = orc.exchange(params, 1, 1, n_tmp, 0, 1, et, it0)
    assert it.tolist() == [0, 2, 1, 4, 3, 5] and acs.tolist() == [0, 1, 1, 1, 1, 0]


def test_library_exports_every_header_symbol():
    hdr = open(os.path.join(os.path.dirname(GOLDEN), "..", "include", "gpudock.h")).read()
    import re
    names = set(re.findall(r"^\s*(?:gd_status|const char \*|uint64_t|size_t|int)\s+(gd_\w+)\(",
                           hdr, re.M))
    assert len(names) > 20
    so = lib.load()
    missing = [n for n in names if not hasattr(so, n)]
    assert not missing, missing


def test_validation_errors_without_gpu():
    cx = synth.make_complex(synth.ComplexSpec(pnp=100, lna=6), seed=2)
    assert lib.validate(cx) == abi.GD_OK
    cx.prt_t = cx.prt_t.copy()
    cx.prt_t[3] = 30
    cx._struct = None
    assert lib.validate(cx) == abi.GD_EINVAL
    assert "type 30" in lib.last_error()
    cx2 = synth.make_complex(synth.ComplexSpec(pnp=100, lna=6), seed=2)
    cx2.prt_seq3r = cx2.prt_seq3r.copy()
    cx2.prt_seq3r[0] = 10 ** 7
    cx2._struct = None
    assert lib.validate(cx2) == abi.GD_EINVAL
    with pytest.raises(lib.GdError):
        lib.set_temperature(0, 0.1, 0.2)
