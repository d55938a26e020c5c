"""Trajectory dump files (the reference's IS_OUTPUT HDF5 dumps, gpusingle.cu:
24-32, hdf5io.C): every completed dump of steps_per_dump MC steps lands in
{dir}/{stem}_NNNN.bin as n_rep LigRecord of steps_per_dump
LigRecordSingleStep, described by {stem}.layout.json.  The files must hold
exactly the records that the in-memory record (GD_MC_RECORD) of the same run
holds, dump by dump."""
import json
import os

import numpy as np
import pytest

from gpudock_b200 import abi, lib, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = lib.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("n_tmp", [8, 6])
def test_dump_files_equal_in_memory_record(ctx, tmp_path, n_tmp):
    """8 temperatures: one launch per segment with the exchange inside;
    6: captured intervals and the exchange kernel.  Runs of 30 steps cross
    dump boundaries (20 steps per dump) in the middle of a call."""
    cx = synth.make_complex(synth.ComplexSpec(pnp=700, lna=21, n_prt=2, n_lig=4), seed=61)
    d = lib.DeviceComplex(ctx, cx)
    _, mb = lib.set_temperature(n_tmp, 0.004, 0.04)
    steps, spe, spd = 90, 10, 20
    flags = abi.MC_EXCHANGE | abi.MC_MOVE_AWAY | abi.MC_MCC
    mem = lib.Remc(d, steps, spe, mb, seed=8, flags=flags | abi.MC_RECORD, steps_per_dump=spd)
    mem.init()
    mem.run(steps)
    ref = mem.read()
    mem.close()

    r = lib.Remc(d, steps, spe, mb, seed=8, flags=flags, steps_per_dump=spd)
    r.set_trajectory(str(tmp_path), "traj")
    r.init()
    for n in (30, 30, 30):
        r.run(n)
    out = r.read()
    r.close()
    # the trajectory does not change the run
    assert np.array_equal(out.energy, ref.energy)
    assert np.array_equal(out.movematrix, ref.movematrix)

    layout = json.load(open(tmp_path / "traj.layout.json"))
    assert layout["dataset"] == "dset" and layout["record"]["bytes"] == 88
    assert layout["shape"] == [ref.record.shape[0]] and layout["steps_per_dump"] == spd
    dumps = lib.read_trajectory(str(tmp_path), "traj")
    assert len(dumps) == steps // spd  # 4 complete dumps; the last 10 steps are not written
    for k, dump in enumerate(dumps):
        assert os.path.getsize(tmp_path / f"traj_{k:04d}.bin") == 88 * spd * len(dump)
        want = ref.record[:, k * spd:(k + 1) * spd]
        assert np.array_equal(dump["step"], want["step"])
        assert np.array_equal(dump["replica.idx_rep"], want["idx_rep"])
        assert np.array_equal(dump["replica.idx_prt"], want["idx_prt"])
        assert np.array_equal(dump["replica.idx_tmp"], want["idx_tmp"])
        assert np.array_equal(dump["replica.idx_lig"], want["idx_lig"])
        assert np.array_equal(dump["energy.e"], want["e"])
        assert np.array_equal(dump["energy.cmcc"], want["cmcc"])
        assert np.array_equal(dump["movematrix"], want["movematrix"])


def test_trajectory_argument_checks(ctx, tmp_path):
    cx = synth.make_complex(synth.ComplexSpec(pnp=300, lna=10), seed=62)
    d = lib.DeviceComplex(ctx, cx)
    _, mb = lib.set_temperature(4, 0.004, 0.04)
    r = lib.Remc(d, 20, 10, mb, steps_per_dump=15)  # not a multiple of the interval
    with pytest.raises(lib.GdError) as e:
        r.set_trajectory(str(tmp_path), "t")
    assert e.value.status == abi.GD_EINVAL
    r.close()
    r = lib.Remc(d, 20, 10, mb, steps_per_dump=10)
    with pytest.raises(lib.GdError) as e:
        r.set_trajectory(str(tmp_path / "missing"), "t")
    assert e.value.status == abi.GD_EIO
    with pytest.raises(lib.GdError):
        r.set_trajectory(str(tmp_path), "a/b")
    r.set_trajectory(str(tmp_path), "t")
    with pytest.raises(lib.GdError):
        r.set_trajectory(str(tmp_path), "t")  # once per run
    r.close()
