"""Contact-mode similarity matrix on CPU: the oracle against the matrix the
reference's similarity tool wrote for its 100-conformation sample
(tests/golden/1a07C1_simi.npz, made by tests/golden/make_simi_golden.py),
and the trace / matrix file helpers against the formats of read2D and
SaveSimilarityMatrix (SimilarityMatirxGen util.C:128-144, 211-240)."""
import numpy as np

from gpudock_b200 import lib
from oracle import oracle as orc
from tests.golden_fixture import HERE, load_complex


def printed_tolerance(v):
    """Half a unit in the 6th significant digit of each printed value."""
    v = np.abs(np.asarray(v, np.float64))
    mag = np.floor(np.log10(np.where(v > 0, v, 1.0)))
    return np.where(v > 0, 0.5 * 10.0 ** (mag - 5) * 1.000001, 5e-7)


def golden():
    g = np.load(f"{HERE}/1a07C1_simi.npz")
    return g["confs"], g["matrix"]


def test_oracle_matches_reference_matrix():
    cx, _, _ = load_complex("smg")
    confs, want = golden()
    S = orc.similarity_matrix(cx, confs)
    assert np.all(np.abs(S - want) <= printed_tolerance(want))
    assert np.all(np.diag(S) == 1.0)


def test_oracle_degenerate_maps():
    """A conformation with no contact has an undefined score in its row and
    column (the reference's 10000)."""
    cx, _, _ = load_complex("smg")
    confs, _ = golden()
    c = confs[:5].copy()
    c[2, 2:5] += 1000.0  # far from the protein: no contacts
    S = orc.similarity_matrix(cx, c)
    assert np.all(S[2, :] == 10000.0) and np.all(S[:, 2] == 10000.0)
    keep = [0, 1, 3, 4]
    assert np.array_equal(S[np.ix_(keep, keep)], orc.similarity_matrix(cx, c[keep]))


def test_trace_and_matrix_files(tmp_path):
    p = tmp_path / "t.tr"
    p.write_text("# comment line\n"
                 "0.0 14.0 0.5 -0.25 1e-3 4.66 4.44 3.27\n"
                 " 1.0 2.0 0 0 0 0 0 0\n"          # starts with a space: skipped
                 "2 3 1.5 2.5 3.5 0.1 0.2 0.3 junk 9\n")
    t = lib.read_traces(str(p))
    assert t.shape == (2, 8)
    assert t[0, 1] == 14.0 and t[0, 4] == np.float32(1e-3) and t[1, 7] == np.float32(0.3)
    S = np.float32([[1.0, 0.5], [10000.0, 1e-5]])
    q = tmp_path / "s.txt"
    lib.save_similarity(str(q), S)
    assert q.read_text() == "2\n1 0.5\n10000 1e-05\n"
