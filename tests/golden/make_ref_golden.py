"""Builds the 1a07C1 golden fixture from the reference's own loaders.

    python tests/golden/make_ref_golden.py [REFERENCE_ROOT]

1. builds oracle/_ref/ref_dump (oracle/Makefile.ref) from the reference's
   host sources (load.C, data.C, util.C) -- loaders, OptimizeLigand /
   OptimizeProtein / OptimizePsp / OptimizeKde / OptimizeMcs /
   OptimizeEnepara and InitLigCoord exactly as linear_dock runs them;
2. runs it on the GeauxDock v0 sample complex (SimilarityMatirxGen/data:
   1a07C.pdb, 1a07C1.sdf, 1a07C1-0.8.ff, parameters/{paras,08ff_opt,
   08_nor_a,08_nor_b}) and on the rem test inputs (gpudocksm-rem-1.2/test);
3. stores the kernel-ready tables as tests/golden/1a07C1_{smg,rem}.npz and
   the published initial-energy lines (SimilarityMatirxGen/doc/
   instructions.txt:156-159, SimilarityMatirxGen/data/report:21-22) as
   tests/golden/1a07C1_golden.json.
"""
import json
import os
import re
import struct
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def read_dump(path):
    recs = {}
    with open(path, "rb") as f:
        data = f.read()
    i = 0
    while i < len(data):
        j = data.index(b"\0", i)
        name = data[i:j].decode()
        typ = chr(data[j + 1])
        (n,) = struct.unpack("<Q", data[j + 2:j + 10])
        elem = 1 if typ == "b" else 4
        payload = data[j + 10:j + 10 + n * elem]
        i = j + 10 + n * elem
        arr = {"f": np.frombuffer(payload, "<f4"), "i": np.frombuffer(payload, "<i4"),
               "b": np.frombuffer(payload, np.uint8)}[typ].copy()
        recs.setdefault(name, []).append(arr)
    return recs


def to_npz(recs, out):
    n_lig, n_prt, lna, pnp, pnk, pos = [int(v) for v in recs["sizes"][0][:6]]
    st = lambda k: np.stack(recs[k])  # noqa: E731
    d = dict(
        lig_xyz=np.stack([st("lig_x"), st("lig_y"), st("lig_z")], axis=-1),
        lig_new_xyz=np.stack([st("lig_new_x"), st("lig_new_y"), st("lig_new_z")], axis=-1),
        lig_center=recs["lig_center"][0], lig_t=recs["lig_t"][0], lig_c=recs["lig_c"][0],
        lig_n=recs["lig_n"][0],
        prt_xyz=np.stack([st("prt_x"), st("prt_y"), st("prt_z")], axis=-1),
        prt_t=recs["prt_t"][0], prt_c=recs["prt_c"][0], prt_ele=recs["prt_ele"][0],
        prt_seq3r=recs["prt_seq3r"][0], prt_hpcflag=recs["prt_hpcflag"][0],
        prt_hpp=recs["prt_hpp"][0], pocket_center=recs["pocket_center"][0],
        psp=st("psp_row"),
        kde_xyz=np.stack([recs["kde_x"][0], recs["kde_y"][0], recs["kde_z"][0]], axis=-1),
        kde_t=recs["kde_t"][0],
        mcs_xyz=np.stack([st("mcs_x"), st("mcs_y"), st("mcs_z")], axis=-1) if pos else
        np.zeros((0, 256, 3), np.float32),
        mcs_tcc=np.concatenate(recs["mcs_tcc"]) if pos else np.zeros(0, np.float32),
        enepara=recs["enepara"][0], enepara_raw=recs["enepara_raw"][0],
        sizes=np.array([n_lig, n_prt, lna, pnp, pnk, pos], np.int32))
    np.savez_compressed(out, **d)
    return d


def golden_lines(ref):
    pat = re.compile(r"^\s*0 0 ((?:-?\d+\.\d+\s*){10})$")
    out = {}
    for key, rel in (("instructions", "SimilarityMatirxGen/doc/instructions.txt"),
                     ("report", "SimilarityMatirxGen/data/report")):
        with open(os.path.join(ref, rel)) as f:
            for line in f:
                m = pat.match(line.rstrip("\n"))
                if m:
                    out[key] = [float(v) for v in m.group(1).split()]
    out["order"] = ["vdw", "ele", "pmf", "psp", "hdb", "hpc", "kde", "lhm", "dst", "total"]
    out["report_command"] = ("-ns 1000 -nc 10 -floor_temp 0.044f -ceiling_temp 0.036f -nt 1 "
                             "-t 0.02f -r 0.08f")
    return out


def main(argv):
    ref = argv[1] if len(argv) > 1 else os.environ.get("GD_REFERENCE")
    if not ref:
        sys.exit("usage: give the reference checkout as the argument or in GD_REFERENCE")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "-f", "Makefile.ref",
                    f"REF={ref}"], check=True)
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_dump")
    smg = os.path.join(ref, "SimilarityMatirxGen", "data")
    rem = os.path.join(ref, "gpudocksm-rem-1.2", "test")
    jobs = {
        "smg": [f"{smg}/1a07C1/1a07C.pdb", f"{smg}/1a07C1/1a07C1.sdf",
                f"{smg}/1a07C1/1a07C1-0.8.ff", f"{smg}/parameters/paras",
                f"{smg}/parameters/08ff_opt", f"{smg}/parameters/08_nor_a",
                f"{smg}/parameters/08_nor_b", "1a07C1"],
        "rem": [f"{rem}/1a07C.pdb", f"{rem}/1a07C1.sdf", f"{rem}/1a07C1-0.8.ff",
                f"{rem}/gpudocksm.ff", f"{rem}/08ff_opt", f"{rem}/08_nor_a", f"{rem}/08_nor_b",
                "1a07C1"],
    }
    tmp = os.path.join(ROOT, "oracle", "_ref")
    for name, args in jobs.items():
        b = os.path.join(tmp, f"{name}.bin")
        subprocess.run([exe, *args, b], check=True)
        d = to_npz(read_dump(b), os.path.join(HERE, f"1a07C1_{name}.npz"))
        print(name, d["sizes"])
    with open(os.path.join(HERE, "1a07C1_golden.json"), "w") as f:
        json.dump(golden_lines(ref), f, indent=1)


if __name__ == "__main__":
    main(sys.argv)
