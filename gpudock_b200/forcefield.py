"""Force-field parameter files of GeauxDock / gpudocksm.

Parses the text formats the reference reads in ``loadEnePara``,
``loadWeight`` and ``loadNorPara`` (gpudocksm-rem-1.2/src/load.C:1139-1419)
into the raw ``gd_enepara_raw`` table, with the same type codes
(``getPntCode``/``getLigCode``/``getResCodeOne``, data.C:239-600) and the same
hydrophobicity rescaling of HPP to [-1, 1] (load.C:1297-1323).

The packaged parameter set ``data/gpudocksm_ff.npz`` holds the reference's
``gpudocksm.ff`` with the ``08ff_opt`` weights and ``08_nor_a``/``08_nor_b``
normalisation, converted by ``data/make_ff.py``.
"""
from __future__ import annotations

import os
import re

import numpy as np

from . import abi

# getPntCode (data.C:391-460): protein effective-point names, index = code
PNT_NAMES = ("CA", "PP", "A1", "C1", "D1", "E1", "E2", "F1", "F2", "H1", "H2", "I1",
             "K1", "K2", "L1", "M1", "M2", "N1", "P1", "Q1", "Q2", "R1", "R2", "S1",
             "T1", "V1", "W1", "W2", "Y1", "Y2")
# getLigCode (data.C:532-583): ligand (Sybyl) atom types, index = code
LIG_NAMES = ("Br", "C.1", "C.2", "C.3", "C.ar", "C.cat", "Cl", "F", "I", "N.1", "N.2",
             "N.3", "N.4", "N.am", "N.ar", "N.pl3", "O.2", "O.3", "O.co2", "P.3", "S.2",
             "S.3", "S.O", "S.O2")
# getResCode / getResCodeOne (data.C:285-386): residue codes
RES_THREE = ("ALA", "ARG", "CYS", "PRO", "LEU", "ILE", "GLU", "HIS", "TRP", "THR", "MET",
             "ASP", "GLY", "PHE", "LYS", "GLN", "SER", "ASN", "TYR", "VAL")
RES_ONE = ("A", "R", "C", "P", "L", "I", "E", "H", "W", "T", "M", "D", "G", "F", "K", "Q",
           "S", "N", "Y", "V")

PNT_CODE = {n: i for i, n in enumerate(PNT_NAMES)}
LIG_CODE = {n: i for i, n in enumerate(LIG_NAMES)}
RES_CODE_ONE = {n: i for i, n in enumerate(RES_ONE)}

# Side-chain effective points of each residue code, (point type, class),
# as pushed by loadProtein (load.C:648-715); GLY (12) has none.
SIDECHAIN_POINTS = {
    0: ((2, 2),), 1: ((21, 2), (22, 3)), 2: ((3, 2),), 3: ((18, 2),), 4: ((14, 2),),
    5: ((11, 2),), 6: ((5, 2), (6, 3)), 7: ((9, 2), (10, 3)), 8: ((26, 2), (27, 3)),
    9: ((24, 2),), 10: ((15, 2), (16, 3)), 11: ((4, 2),), 12: (),
    13: ((7, 2), (8, 3)), 14: ((12, 2), (13, 3)), 15: ((19, 2), (20, 3)),
    16: ((23, 2),), 17: ((17, 2),), 18: ((28, 2), (29, 3)), 19: ((25, 2),),
}
# point type -> (residue code, class) for side-chain points
SIDECHAIN_OWNER = {t: (d, c) for d, pts in SIDECHAIN_POINTS.items() for (t, c) in pts}

DATA_DIR = os.path.join(os.path.dirname(__file__), "data")
DEFAULT_FF = os.path.join(DATA_DIR, "gpudocksm_ff.npz")


def empty_raw() -> dict:
    return {
        "vdw": np.zeros((abi.NPT, abi.NLT, 2), np.float32),
        "ele": np.zeros(abi.NELE, np.float32),
        "pmf": np.zeros((abi.NPT, abi.NLT, 2), np.float32),
        "hpp": np.zeros(abi.NRES, np.float32),
        "hpl": np.zeros((abi.NLT, 2), np.float32),
        "hdb": np.zeros((abi.NPT, abi.NLT, 2), np.float32),
        "lj": np.zeros(3, np.float32),
        "el": np.zeros(2, np.float32),
        "kde": np.zeros(1, np.float32),
        "w": np.zeros(abi.NTERM, np.float32),
        "a_para": np.zeros(abi.NTERM, np.float32),
        "b_para": np.zeros(abi.NTERM, np.float32),
    }


_NUM = re.compile(r"\s*[+-]?(\d+\.?\d*|\.\d+)([eE][+-]?\d+)?")


def _atof(s: str) -> np.float32:
    """atof stored as a float: the longest leading decimal number, else 0."""
    m = _NUM.match(s)
    return np.float32(float(m.group(0)) if m else 0.0)


def parse_ff_text(text: str, raw: dict | None = None) -> dict:
    """Parses the .ff parameter format (VDW/PLJ/ELE/PEL/PMF/HPP/HPL/HDB/WEI/KDE
    lines) the way loadEnePara does, including the HPP rescaling."""
    raw = empty_raw() if raw is None else raw
    for line in text.splitlines():
        if len(line) <= 3:
            continue
        tag, tok = line[:3], line.split()
        tok += [""] * (abi.NTERM + 1 - len(tok))  # a missing field reads as 0
        f = _atof
        if tag == "VDW":
            raw["vdw"][PNT_CODE[tok[1]], LIG_CODE[tok[2]]] = (f(tok[3]), f(tok[4]))
        elif tag == "PLJ":
            raw["lj"][:] = [f(v) for v in tok[1:4]]
        elif tag == "ELE":
            name = tok[1]
            if name[1:2] != "C":
                raw["ele"][PNT_CODE[name]] = f(tok[2])
            else:
                raw["ele"][RES_CODE_ONE[name[0:1]] + 30] = f(tok[2])
        elif tag == "PEL":
            raw["el"][:] = [f(v) for v in tok[1:3]]
        elif tag == "PMF":
            raw["pmf"][PNT_CODE[tok[1]], LIG_CODE[tok[2]]] = (f(tok[3]), f(tok[4]))
        elif tag == "HPP":
            raw["hpp"][RES_CODE_ONE[tok[1]]] = f(tok[2])
        elif tag == "HPL":
            raw["hpl"][LIG_CODE[tok[1]]] = (f(tok[2]), f(tok[3]))
        elif tag == "HDB":
            raw["hdb"][PNT_CODE[tok[1]], LIG_CODE[tok[2]]] = (f(tok[3]), f(tok[4]))
        elif tag == "WEI":
            raw["w"][:] = [f(v) for v in tok[1:abi.NTERM + 1]]
        elif tag == "KDE":
            raw["kde"][0] = f(tok[1])
    # rescale hydrophobicity to [-1, 1] (load.C:1297-1323): the difference and
    # quotient in single precision, "* 2.0 - 1.0" in double, stored as float
    hpp = raw["hpp"]
    lo = np.float32(min(np.float32(1e6), hpp.min()))
    hi = np.float32(max(np.float32(-1e6), hpp.max()))
    q = ((hpp - lo) / np.float32(hi - lo)).astype(np.float32)
    out = (q.astype(np.float64) * 2.0 - 1.0).astype(np.float32)
    raw["hpp"] = np.clip(out, np.float32(-1.0), np.float32(1.0)).astype(np.float32)
    return raw


def parse_column(text: str) -> np.ndarray:
    """One float per line (first 30 characters), as loadWeight/loadNorPara."""
    vals = []
    for line in text.splitlines():
        s = line[:30].split()
        vals.append(np.float32(s[0]) if s else np.float32(0.0))
    return np.asarray(vals, np.float32)


def build_raw(ff_text: str, weight_text: str, nor_a_text: str, nor_b_text: str) -> dict:
    """Raw table after loadEnePara, loadWeight, loadNorPara (dock.C:43-45)."""
    raw = parse_ff_text(ff_text)
    for key, txt in (("w", weight_text), ("a_para", nor_a_text), ("b_para", nor_b_text)):
        v = parse_column(txt)[: abi.NTERM]
        raw[key][: len(v)] = v
    return raw


def load_raw(path: str = DEFAULT_FF) -> dict:
    with np.load(path) as z:
        return {k: z[k].astype(np.float32) for k in z.files}


def raw_struct(raw: dict) -> abi.GdEneparaRaw:
    d = dict(raw)
    d["kde"] = np.asarray(d["kde"], np.float32).reshape(1)
    return abi.raw_from_arrays(d)
