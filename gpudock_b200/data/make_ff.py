"""Converts the reference force-field files into data/gpudocksm_ff.npz.

Run where the reference project is available, giving its
gpudocksm-rem-1.2/test directory as the argument (or the reference checkout
in GD_REFERENCE):

    python -m gpudock_b200.data.make_ff REFERENCE_TEST_DIR

Inputs: gpudocksm.ff (VDW/PMF/HDB/ELE/HPP/HPL/PLJ/PEL/KDE), 08ff_opt (term
weights), 08_nor_a and 08_nor_b (normalisation a, b), the files the
reference's linear_dock reads by default (util.C:35-62).
"""
import os
import sys

import numpy as np

from gpudock_b200 import forcefield



def main(argv):
    if len(argv) > 1:
        src = argv[1]
    elif os.environ.get("GD_REFERENCE"):
        src = os.path.join(os.environ["GD_REFERENCE"], "gpudocksm-rem-1.2", "test")
    else:
        sys.exit("usage: python -m gpudock_b200.data.make_ff REFERENCE_TEST_DIR")

    def read(name):
        with open(os.path.join(src, name)) as f:
            return f.read()

    raw = forcefield.build_raw(read("gpudocksm.ff"), read("08ff_opt"), read("08_nor_a"),
                               read("08_nor_b"))
    np.savez_compressed(forcefield.DEFAULT_FF, **raw)
    print("wrote", forcefield.DEFAULT_FF, {k: v.shape for k, v in raw.items()})


if __name__ == "__main__":
    main(sys.argv)
