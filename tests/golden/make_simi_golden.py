"""Builds the similarity-matrix golden fixture from the reference's sample run.

    python tests/golden/make_simi_golden.py [REFERENCE_ROOT]

The GeauxDock v0 sample data (SimilarityMatirxGen/data) holds a trace file of
100 near-native conformations of 1a07C1 (1a07C1.tr: protein conf, ligand
conf, move vector per line) and the similarity matrix the reference's
similarity tool wrote for them (correct_simi_matrix.txt, 100 x 100 contact
MCCs printed with 6 significant digits; data/dock.bash is the command line:
the 1a07C1 complex with parameters/{paras,08ff_opt,08_nor_a,08_nor_b}, the
tables of tests/golden/1a07C1_smg.npz).  This script stores both as
tests/golden/1a07C1_simi.npz: the conformations as read2D parses them
(float32) and the matrix as printed (float64).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gpudock_b200 import lib  # noqa: E402


def main(argv):
    ref = argv[1] if len(argv) > 1 else os.environ.get("GD_REFERENCE")
    if not ref:
        sys.exit("usage: give the reference checkout as the argument or in GD_REFERENCE")
    data = os.path.join(ref, "SimilarityMatirxGen", "data")
    confs = lib.read_traces(os.path.join(data, "1a07C1.tr"))
    matrix = np.loadtxt(os.path.join(data, "correct_simi_matrix.txt"), dtype=np.float64)
    assert confs.shape == (100, 8) and matrix.shape == (100, 100)
    out = os.path.join(HERE, "1a07C1_simi.npz")
    np.savez_compressed(out, confs=confs, matrix=matrix)
    print("wrote", out)


if __name__ == "__main__":
    main(sys.argv)
