"""Loads the committed 1a07C1 fixtures (tables produced by the reference's own
loaders, see tests/golden/make_ref_golden.py) as an abi.Complex."""
import ctypes as C
import json
import os

import numpy as np

from gpudock_b200 import abi

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_complex(name="smg"):
    z = np.load(os.path.join(HERE, f"1a07C1_{name}.npz"))
    ff = abi.GdEnepara.from_buffer_copy(z["enepara"].tobytes())
    raw = abi.GdEneparaRaw.from_buffer_copy(z["enepara_raw"].tobytes())
    cx = abi.Complex(
        lig_xyz=z["lig_xyz"], lig_t=z["lig_t"], lig_c=z["lig_c"], lig_n=z["lig_n"],
        lig_center=z["lig_center"], prt_xyz=z["prt_xyz"], prt_t=z["prt_t"], prt_c=z["prt_c"],
        prt_ele=z["prt_ele"], prt_seq3r=z["prt_seq3r"], prt_hpcflag=z["prt_hpcflag"],
        prt_hpp=z["prt_hpp"], pocket_center=z["pocket_center"], psp=z["psp"],
        kde_xyz=z["kde_xyz"], kde_t=z["kde_t"], mcs_xyz=z["mcs_xyz"], mcs_tcc=z["mcs_tcc"],
        ff=ff)
    return cx, raw, z


def golden_lines():
    with open(os.path.join(HERE, "1a07C1_golden.json")) as f:
        return json.load(f)
