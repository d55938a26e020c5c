"""Native input loaders (gd_load, gpudock_b200/csrc/gd_load.cpp) on CPU.

1. The reference's own sample inputs (1a07C1, where the reference checkout
   is present) load to exactly the tables its loaders produce: the golden
   fixtures tests/golden/1a07C1_{rem,smg}.npz were dumped by
   oracle/_ref/ref_dump, which runs load.C / util.C themselves.
2. Small hand-written files check each rule independently of the
   reference: effective points per residue, per-model means, the RMSD
   filter of ligand conformations, KDE / PSP / MCS records, error codes."""
import ctypes
import os

import numpy as np
import pytest

from gpudock_b200 import abi, forcefield, lib
from oracle.oracle import reference_root
from tests.golden_fixture import load_complex

REF = reference_root() or ""
FIELDS = ("lig_xyz", "lig_t", "lig_c", "lig_n", "lig_center", "prt_xyz", "prt_t", "prt_c",
          "prt_ele", "prt_seq3r", "prt_hpcflag", "prt_hpp", "pocket_center", "kde_xyz",
          "kde_t", "mcs_xyz", "mcs_tcc")
SAMPLES = {
    "rem": ("gpudocksm-rem-1.2/test", "1a07C.pdb", "1a07C1.sdf", "1a07C1-0.8.ff"),
    "smg": ("SimilarityMatirxGen/data/1a07C1", "1a07C.pdb", "1a07C1.sdf", "1a07C1-0.8.ff"),
}


@pytest.mark.parametrize("name", sorted(SAMPLES))
def test_sample_inputs_match_reference_loaders(name):
    d, pdb, sdf, ff = SAMPLES[name]
    base = os.path.join(REF, d)
    if not os.path.isdir(base):
        pytest.skip("reference checkout not present")
    ref, raw, _ = load_complex(name)
    cx = lib.load_files(os.path.join(base, pdb), os.path.join(base, sdf), os.path.join(base, ff),
                        "1a07C1", raw=raw)
    assert cx.ligand_id == "1a07C1"
    for k in FIELDS:
        a, b = getattr(cx, k), getattr(ref, k)
        assert a.shape == b.shape and np.array_equal(a, b), k
    assert np.array_equal(cx.psp, ref.psp[:abi.NLT, :cx.psp.shape[1]])
    # the peptide-plane rule in every model changes only peptide points of
    # models after the second
    cf = lib.load_files(os.path.join(base, pdb), os.path.join(base, sdf),
                        os.path.join(base, ff), "1a07C1", raw=raw,
                        flags=lib.LOAD_PEPTIDE_ALL_MODELS)
    diff = np.abs(cf.prt_xyz - cx.prt_xyz).max(axis=2)
    assert (diff[:2] == 0).all() and (diff[:, cx.prt_t != 1] == 0).all()


# ---------------------------------------------------------------------------
# hand-written files
# ---------------------------------------------------------------------------
def _atom(serial, name, res, rseq, x, y, z):
    return (f"ATOM  {serial:5d} {name:<4s} {res:3s} A{rseq:4d}    "
            f"{x:8.3f}{y:8.3f}{z:8.3f}  1.00  0.00")


RESIDUES = [  # residue name, atoms (name, offset)
    ("ALA", [(" N  ", 0.0), (" CA ", 0.5), (" C  ", 1.0), (" O  ", 1.5), (" CB ", 2.0)]),
    ("GLY", [(" N  ", 0.0), (" CA ", 0.5), (" C  ", 1.0), (" O  ", 1.5)]),
    ("ARG", [(" N  ", 0.0), (" CA ", 0.5), (" C  ", 1.0), (" O  ", 1.5), (" CB ", 2.0),
             (" CG ", 2.5), (" CD ", 3.0), (" NE ", 3.5)]),
    ("SER", [(" N  ", 0.0), (" CA ", 0.5), (" C  ", 1.0), (" O  ", 1.5), (" CB ", 2.0),
             (" OG ", 2.5)]),
]


def _write_pdb(path, n_models=3):
    lines, pos = [], {}
    for m in range(n_models):
        lines.append(f"MODEL {m + 1}")
        k = 1
        for i, (res, atoms) in enumerate(RESIDUES):
            for name, off in atoms:
                xyz = (10.0 * i + off + 0.1 * m, 1.0 + 0.25 * off, -2.0 + 0.125 * i * off)
                # as written (3 decimals) and read back (atof into a float)
                pos[(m, i, name)] = np.float32([float(f"{v:8.3f}") for v in xyz])
                lines.append(_atom(k, name, res, i + 1, *xyz))
                k += 1
        lines.append("ENDMDL")
    open(path, "w").write("\n".join(lines) + "\n")
    return pos


def _expected_points():
    """Point rules of loadProtein restated for the hand-written residues:
    (residue index, type, class, atoms averaged in model m, residue code d).
    A peptide-plane point belongs to the previous residue but carries the
    code of the residue whose CA pushed it (load.C:641-643); from the third
    model on it is the N atom alone (see gd_load)."""
    side = {"ALA": [(2, 2, "not_bb")], "GLY": [],
            "ARG": [(21, 2, "not_bb_cbcg"), (22, 3, "cbcg")], "SER": [(23, 2, "not_bb")]}
    bb = {" N  ", " CA ", " C  ", " O  "}
    pts = []
    for i, (res, atoms) in enumerate(RESIDUES):
        names = [a for a, _ in atoms]
        d = forcefield.RES_THREE.index(res)
        pts.append((i, 0, 0, lambda m, i=i: [(m, i, " CA ")], d))
        if i > 1:  # peptide-plane point of residue i - 1, pushed at residue i
            r = i - 1
            pts.append((r, 1, 1, lambda m, r=r: (
                [(m, r, " N  "), (m, r - 1, " C  "), (m, r - 1, " O  ")] if m < 2
                else [(m, r, " N  ")]), d))
        for t, c, rule in side[res]:
            if rule == "not_bb":
                sel = [a for a in names if a not in bb]
            elif rule == "not_bb_cbcg":
                sel = [a for a in names if a not in bb | {" CB ", " CG "}]
            else:
                sel = [a for a in names if a in {" CB ", " CG "}]
            pts.append((i, t, c, lambda m, i=i, sel=sel: [(m, i, a) for a in sel], d))
    return pts


def _file_order(keys):
    """Atoms in the order the PDB lists them (residue, then atom)."""
    order = {(i, a): k for k, (i, a) in enumerate(
        (i, a) for i, (_, atoms) in enumerate(RESIDUES) for a, _ in atoms)}
    return sorted(keys, key=lambda key: order[(key[1], key[2])])


def _write_sdf(path, native, confs, types, charges, molid="LIG7"):
    lna = len(native)
    lines = ["", " hand-written", "", f"{lna:3d}{0:3d}  0  0  0  0  0  0  0  0999 V2000"]
    for x, y, z in native:
        lines.append(f"{x:10.4f}{y:10.4f}{z:10.4f} C   0  0  0  0  0")
    lines += ["M  END", f">  <MOLID> ({molid})", molid, "", f">  <OB_ATOM_TYPES> ({molid})",
              " ".join(types), "", f">  <OB_ATOMIC_CHARGES> ({molid})",
              " ".join(f"{c:.4f}" for c in charges), "", f">  <ENSEMBLE_COORDS> ({molid})"]
    for c in confs:
        lines.append(" ".join(f"{v:.4f}" for v in np.asarray(c).reshape(-1)))
    lines += ["", "$$$$"]
    open(path, "w").write("\n".join(lines) + "\n")


def test_hand_written_complex(tmp_path):
    raw = forcefield.raw_struct(forcefield.load_raw())
    pos = _write_pdb(tmp_path / "p.pdb")
    rng = np.random.default_rng(4)
    native = rng.normal(0, 1.5, (6, 3)).round(4) + np.array([10.0, 2.0, -1.0])
    c0 = native - native.mean(axis=0)
    rot = np.array([[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])
    confs = [c0 + 5.0,                            # a shifted copy: RMSD 0, dropped
             c0 @ rot.T,                          # a rotated copy: RMSD 0, dropped
             c0 + rng.normal(0, 0.5, c0.shape),   # distorted: kept
             c0 + rng.normal(0, 0.01, c0.shape)]  # within 0.1 A: dropped
    types = ["C.3", "C.ar", "N.am", "O.2", "S.3", "C.2"]
    charges = [0.1, -0.2, 0.3, -0.4, 0.05, 0.15]
    _write_sdf(tmp_path / "l.sdf", native, confs, types, charges)
    lhm = ["KDE C.3 1.0 2.0 3.0", "KDE Xx 9.0 9.0 9.0", "KDE O.2 -1.5 0.5 2.25",
           "PSP 3 N.am 0.75", "PSP 2 C.ar 1.25", "PSP 99 C.3 4.0",
           "MCS LIG7 0.25 2 1 0.5 0.5 0.5 4 1.5 -1.5 2.5",
           "MCS OTHER 0.5 1 2 3.0 3.0 3.0"]
    open(tmp_path / "t.ff", "w").write("\n".join(lhm) + "\n")
    paths = [str(tmp_path / f) for f in ("p.pdb", "l.sdf", "t.ff")]

    cx = lib.load_files(*paths, "LIG7", raw=raw)
    assert cx.ligand_id == "LIG7"
    # --- protein points, in push order, with their per-model means
    pts = _expected_points()
    assert cx.pnp == len(pts) and cx.n_prt == 3
    assert list(cx.prt_t) == [pt[1] for pt in pts]
    assert list(cx.prt_c) == [pt[2] for pt in pts]
    assert list(cx.prt_seq3r) == [pt[0] + 1 for pt in pts]
    hpp = np.ctypeslib.as_array(raw.hpp)
    ele = np.ctypeslib.as_array(raw.ele)
    assert np.array_equal(cx.prt_hpp, hpp[[pt[4] for pt in pts]])
    assert np.array_equal(cx.prt_ele, [ele[pt[4] + 30] if pt[1] == 0 else ele[pt[1]]
                                       for pt in pts])
    assert list(cx.prt_hpcflag) == [int((pt[2] == 0 and pt[4] == 12) or pt[2] == 2)
                                    for pt in pts]
    for m in range(3):
        for p, pt in enumerate(pts):
            acc, n = np.zeros(3, np.float32), np.float32(0)
            for key in _file_order(pt[3](m)):  # float sums in file order
                acc = (acc + pos[key]).astype(np.float32)
                n = np.float32(n + 1)
            assert np.array_equal(cx.prt_xyz[m, p], (acc / n).astype(np.float32)), (m, p)
    # --- ligand: default pose + the one distorted conformation
    assert cx.n_lig == 2 and cx.lna == 6
    nat32 = np.float32([[float(f"{v:10.4f}") for v in row] for row in native])
    assert np.allclose(cx.lig_center, nat32.mean(axis=0), atol=1e-5)
    assert np.allclose(cx.lig_xyz[0], nat32 - cx.lig_center, atol=1e-5)
    kept = np.float32([[float(f"{v:.4f}") for v in row] for row in confs[2]])
    assert np.allclose(cx.lig_xyz[1], kept - kept.mean(axis=0), atol=1e-4)
    assert list(cx.lig_t) == [forcefield.LIG_CODE[t] for t in types]
    assert np.allclose(cx.lig_c, charges) and list(cx.lig_n) == list(range(6))
    assert np.array_equal(cx.pocket_center, cx.lig_center)
    # --- pocket template
    assert list(cx.kde_t) == [forcefield.LIG_CODE["C.3"], forcefield.LIG_CODE["O.2"]]
    assert np.array_equal(cx.kde_xyz, np.float32([[1, 2, 3], [-1.5, 0.5, 2.25]]))
    assert cx.psp.shape == (abi.NLT, 5)  # residue serials 1..4
    assert cx.psp[forcefield.LIG_CODE["N.am"], 3] == np.float32(0.75)
    assert cx.psp[forcefield.LIG_CODE["C.ar"], 2] == np.float32(1.25)
    assert np.count_nonzero(cx.psp) == 2
    assert cx.mcs_xyz.shape == (2, 256, 3)
    assert np.array_equal(cx.mcs_tcc, np.float32([0.25, 0.0]))
    assert np.array_equal(cx.mcs_xyz[0, 1], np.float32([0.5, 0.5, 0.5]))
    assert np.array_equal(cx.mcs_xyz[0, 4], np.float32([1.5, -1.5, 2.5]))
    assert (np.delete(cx.mcs_xyz[0], [1, 4], axis=0) == abi.MCS_INVALID_COORD).all()
    assert (cx.mcs_xyz[1] == abi.MCS_INVALID_COORD).all()
    # the complex is valid input to the library
    lib.check(lib.load().gd_complex_validate(ctypes.byref(cx.struct())), "gd_complex_validate")
    # the peptide-plane rule in every model
    cf = lib.load_files(*paths, "LIG7", raw=raw, flags=lib.LOAD_PEPTIDE_ALL_MODELS)
    diff = np.abs(cf.prt_xyz - cx.prt_xyz).max(axis=2)
    assert (diff[:2] == 0).all() and (diff[2][cx.prt_t == 1] > 0).all()
    assert (diff[2][cx.prt_t != 1] == 0).all()


def test_loader_errors(tmp_path):
    raw = forcefield.raw_struct(forcefield.load_raw())
    _write_pdb(tmp_path / "p.pdb")
    _write_sdf(tmp_path / "l.sdf", np.float64([[0, 0, 0], [1, 0, 0], [0, 1, 0]]), [],
               ["C.3"] * 3, [0.0] * 3)
    open(tmp_path / "t.ff", "w").write("KDE C.3 0 0 0\n")
    args = [str(tmp_path / "p.pdb"), str(tmp_path / "l.sdf"), str(tmp_path / "t.ff"), "X"]
    with pytest.raises(lib.GdError) as e:
        lib.load_files(str(tmp_path / "missing.pdb"), *args[1:], raw=raw)
    assert e.value.status == abi.GD_EIO
    open(tmp_path / "nomodel.pdb", "w").write(_atom(1, " CA ", "ALA", 1, 0, 0, 0) + "\n")
    with pytest.raises(lib.GdError) as e:
        lib.load_files(str(tmp_path / "nomodel.pdb"), *args[1:], raw=raw)
    assert e.value.status == abi.GD_EINVAL
    open(tmp_path / "bad.pdb", "w").write(
        "MODEL 1\n" + _atom(1, " CA ", "XYZ", 1, 0, 0, 0) + "\nENDMDL\n")
    with pytest.raises(lib.GdError) as e:
        lib.load_files(str(tmp_path / "bad.pdb"), *args[1:], raw=raw)
    assert e.value.status == abi.GD_EINVAL and "unknown residue" in str(e.value)
    cx = lib.load_files(*args, raw=raw)
    assert cx.n_lig == 1 and cx.pnp > 0


# ---------------------------------------------------------------------------
# force-field parameter files (gd_load_enepara)
# ---------------------------------------------------------------------------
PARAM_FILES = {  # the parameter files each golden fixture was dumped with
    "rem": ("gpudocksm-rem-1.2/test", "gpudocksm.ff", "08ff_opt", "08_nor_a", "08_nor_b"),
    "smg": ("SimilarityMatirxGen/data/parameters", "paras", "08ff_opt", "08_nor_a", "08_nor_b"),
}


@pytest.mark.parametrize("name", sorted(PARAM_FILES))
def test_enepara_files_match_reference_loaders(name):
    d, *files = PARAM_FILES[name]
    base = os.path.join(REF, d)
    if not os.path.isdir(base):
        pytest.skip("reference checkout not present")
    _, _, z = load_complex(name)
    raw = lib.load_enepara(*[os.path.join(base, f) for f in files])
    assert bytes(raw) == z["enepara_raw"].tobytes()
    if name == "rem":  # the packaged parameter set is these files
        assert bytes(raw) == bytes(forcefield.raw_struct(forcefield.load_raw()))


def test_enepara_hand_written(tmp_path):
    ff = ["VDW CA C.3 1.5 0.25", "PMF Y2 S.O2 4.0", "HDB N1 O.2 2.9 0.7",
          "ELE CA 0.5", "ELE KC -1.25", "HPP A 1.8", "HPP R -4.5", "HPP G -0.4",
          "HPL C.ar 0.3 2.5", "PLJ 1 2 3", "PEL 2.0 0.5", "WEI 1 2 3", "KDE 0.25",
          "XYZ ignored line", "VDW", ""]
    (tmp_path / "p.ff").write_text("\n".join(ff) + "\n")
    (tmp_path / "w").write_text("0.5\n\n2.5   trailing text\n")
    (tmp_path / "a").write_text("\n".join(str(v) for v in range(12)) + "\n")
    raw = lib.load_enepara(str(tmp_path / "p.ff"))
    nlt = forcefield.LIG_CODE
    npt = forcefield.PNT_CODE
    assert raw.vdw[npt["CA"]][nlt["C.3"]][0] == np.float32(1.5)
    assert raw.vdw[npt["CA"]][nlt["C.3"]][1] == np.float32(0.25)
    assert raw.pmf[npt["Y2"]][nlt["S.O2"]][0] == np.float32(4.0)
    assert raw.pmf[npt["Y2"]][nlt["S.O2"]][1] == 0.0  # missing value
    assert raw.hdb[npt["N1"]][nlt["O.2"]][1] == np.float32(0.7)
    assert raw.ele[npt["CA"]] == np.float32(0.5)
    assert raw.ele[30 + forcefield.RES_CODE_ONE["K"]] == np.float32(-1.25)
    # hydrophobicity rescaled over all 20 residues (unset ones are 0):
    # min -4.5 -> -1, max 1.8 -> 1
    hpp = np.array(raw.hpp[:], np.float32)
    assert hpp[forcefield.RES_CODE_ONE["A"]] == 1.0 and hpp[forcefield.RES_CODE_ONE["R"]] == -1.0
    lo, hi = np.float32(-4.5), np.float32(1.8)
    want_g = np.float32(np.float64((np.float32(-0.4) - lo) / np.float32(hi - lo)) * 2.0 - 1.0)
    assert hpp[forcefield.RES_CODE_ONE["G"]] == want_g
    assert list(raw.lj) == [1.0, 2.0, 3.0] and list(raw.el) == [2.0, 0.5]
    assert list(raw.w) == [1.0, 2.0, 3.0] + [0.0] * 7 and raw.kde == np.float32(0.25)
    assert list(raw.a_para) == [0.0] * 10 and list(raw.b_para) == [0.0] * 10
    # the same text through the Python parser gives the same table
    py = forcefield.raw_struct(forcefield.parse_ff_text("\n".join(ff)))
    assert bytes(py) == bytes(raw)
    # weight and normalisation columns: first 30 characters of each of the
    # first 10 lines, empty lines 0; w replaces the WEI values line by line
    raw2 = lib.load_enepara(str(tmp_path / "p.ff"), str(tmp_path / "w"), str(tmp_path / "a"),
                            str(tmp_path / "a"))
    assert list(raw2.w) == [0.5, 0.0, 2.5] + [0.0] * 7
    assert list(raw2.a_para) == [float(v) for v in range(10)]
    assert list(raw2.b_para) == list(raw2.a_para)


@pytest.mark.parametrize("line", ["VDW XX C.3 1 1", "PMF CA Q.9 1 1", "HPL Zz 1 1",
                                  "ELE ZC 1", "ELE Q 1", "HPP B 1"])
def test_enepara_unknown_names(tmp_path, line):
    (tmp_path / "p.ff").write_text("PLJ 1 2 3\n" + line + "\n")
    with pytest.raises(lib.GdError) as e:
        lib.load_enepara(str(tmp_path / "p.ff"))
    assert e.value.status == abi.GD_EINVAL


def test_enepara_missing_files(tmp_path):
    (tmp_path / "p.ff").write_text("PLJ 1 2 3\n")
    for args in ([str(tmp_path / "none.ff")],
                 [str(tmp_path / "p.ff"), str(tmp_path / "none")],
                 [str(tmp_path / "p.ff"), None, None, str(tmp_path / "none")]):
        with pytest.raises(lib.GdError) as e:
            lib.load_enepara(*args)
        assert e.value.status == abi.GD_EIO
