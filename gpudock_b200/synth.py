"""Seeded synthetic docking complexes with the shapes of the benchmark configs.

No dataset ships with this build; every workload is generated from a numpy
PCG64 seed:

* protein: ``pnp`` effective points by random sequential packing in a cube
  (minimum pair distance 3.0 A) around an empty spherical pocket at the cube
  centre; point types uniform over the 30 force-field point types, with the
  class and residue code that loadProtein gives each type
  (gpudocksm-rem-1.2/src/load.C:648-715), ``ele``/``hpp`` derived as
  CopyProteinResidue does (util.C:253-275); extra conformations add Gaussian
  coordinate noise;
* ligand: a random tree with 1.5 A bonds, centred on the pocket, atom types
  uniform over the 24 ligand types, charges N(0, 0.3) shifted to an integer
  sum; extra conformations rotate random subtrees about their bond;
* pocket template: KDE points near the crystal pose per ligand type present,
  32 PSP entries U(0, 2) on pocket residues, 11 MCS records with
  tcc ~ U(0.1, 0.4) covering at least half of the atoms;
* force field: the reference's gpudocksm.ff with 08ff_opt weights and
  08_nor normalisation (data/gpudocksm_ff.npz).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
from scipy.spatial import cKDTree

from . import abi, forcefield

DENSITY = 1500.0 / 40.0 ** 3  # points per A^3 of the 1,500-point / 40 A workload


@dataclass
class ComplexSpec:
    pnp: int
    lna: int
    n_prt: int = 1
    n_lig: int = 1
    cube: float | None = None      # edge of the packing cube (A); None: fixed density
    prt_noise: float = 0.5         # sigma of the protein-conformation noise (A)
    min_dist: float = 3.0
    n_psp: int = 32
    n_mcs: int = 11
    kde_per_type: int = 20


@dataclass
class Workload:
    """A named benchmark workload: complex spec + MC parameters."""
    name: str
    spec: ComplexSpec
    n_tmp: int = 8
    t_floor: float = 0.004
    t_ceil: float = 0.04
    steps: int = 1000
    steps_per_exchange: int = 10
    move_scale: tuple = (0.02, 0.02, 0.02, 0.08, 0.08, 0.08)
    extra: dict = field(default_factory=dict)


# The five benchmark configurations (sizes from the reference's benchmark
# set-up; the replica grid follows SetReplica's prt x tmp x lig layout).
WORKLOADS = {
    "plain_1500x24": Workload("plain_1500x24", ComplexSpec(pnp=1500, lna=24, cube=40.0),
                              n_tmp=8, t_floor=0.004, t_ceil=0.04, steps=1000,
                              steps_per_exchange=10),
    "ensemble_4000x40": Workload("ensemble_4000x40",
                                 ComplexSpec(pnp=4000, lna=40, n_prt=11, n_lig=50, cube=50.0,
                                             min_dist=2.7),
                                 n_tmp=16, t_floor=0.004, t_ceil=0.08, steps=5000,
                                 steps_per_exchange=20),
    "poses_48": Workload("poses_48", ComplexSpec(pnp=16000, lna=48), extra={
        "pnp_sweep": (2000, 4000, 8000, 16000), "n_pose": 1 << 20, "parity_subset": 4096,
        "box": 8.0}),
    "batched_512": Workload("batched_512", ComplexSpec(pnp=6000, lna=54, n_prt=4, n_lig=4),
                            n_tmp=8, t_floor=0.004, t_ceil=0.04, steps=3000,
                            steps_per_exchange=10, extra={
                                "n_ligand": 512, "lna_range": (12, 96)}),
    "serving": Workload("serving", ComplexSpec(pnp=4000, lna=30, n_prt=1, n_lig=4), n_tmp=8,
                        t_floor=0.004, t_ceil=0.04, steps=2000, steps_per_exchange=10, extra={
                            "proteins": (2000, 4000, 7000, 10000), "n_request": 10000,
                            "lna_median": 30, "lna_clip": (8, 120), "rate": (50, 400),
                            "hbm_budget_gb": 120}),
}


# ---------------------------------------------------------------------------
# force field
# ---------------------------------------------------------------------------
_FF_CACHE = {}


def raw_ff():
    """(raw dict, GdEneparaRaw) of the packaged force field (no library call)."""
    if "raw" not in _FF_CACHE:
        raw = forcefield.load_raw()
        _FF_CACHE["raw"] = (raw, forcefield.raw_struct(raw))
    return _FF_CACHE["raw"]


def default_ff():
    """(raw dict, GdEneparaRaw, optimised GdEnepara) of the packaged force field,
    the kernel tables derived by the library's gd_enepara_optimize."""
    if "ff" not in _FF_CACHE:
        from . import lib
        raw, rs = raw_ff()
        _FF_CACHE["ff"] = (raw, rs, lib.enepara_optimize(rs))
    return _FF_CACHE["ff"]


# ---------------------------------------------------------------------------
# protein
# ---------------------------------------------------------------------------
def pack_points(rng, n, edge, min_dist, center, r_excl, max_rounds=200):
    """Random sequential packing of n points in [0, edge]^3 outside a sphere."""
    pts = np.zeros((0, 3))
    rounds = 0
    while len(pts) < n:
        rounds += 1
        if rounds > max_rounds:
            raise RuntimeError(f"packing stalled at {len(pts)}/{n} points")
        need = n - len(pts)
        # near saturation only a small fraction of the cube is still free, so
        # the candidate batch grows with the number of rounds
        cand = rng.uniform(0.0, edge, size=(max(512, 8 * need, min(100000, 1000 * rounds)), 3))
        cand = cand[np.linalg.norm(cand - center, axis=1) > r_excl]
        if len(pts):
            d, _ = cKDTree(pts).query(cand, k=1)
            cand = cand[d >= min_dist]
        if len(cand) == 0:
            continue
        keep = np.ones(len(cand), bool)
        pairs = cKDTree(cand).query_pairs(min_dist, output_type="ndarray")
        if len(pairs):
            pairs = pairs[np.argsort(pairs[:, 1], kind="stable")]
            for i, j in pairs:
                if keep[i] and keep[j]:
                    keep[j] = False
        cand = cand[keep][:need]
        pts = np.concatenate([pts, cand])
    return pts


def protein_types(rng, pnp, raw):
    t = rng.integers(0, abi.NPT, size=pnp).astype(np.int32)
    d = np.zeros(pnp, np.int32)
    c = np.zeros(pnp, np.int32)
    for i in range(pnp):
        if t[i] == 0:
            c[i], d[i] = 0, rng.integers(0, abi.NRES)
        elif t[i] == 1:
            c[i], d[i] = 1, rng.integers(0, abi.NRES)
        else:
            d[i], c[i] = forcefield.SIDECHAIN_OWNER[int(t[i])]
    dt = np.where(t == 0, d + 30, t)
    ele = raw["ele"][dt].astype(np.float32)
    hpp = raw["hpp"][d].astype(np.float32)
    hflag = (((c == 0) & (d == 12)) | (c == 2)).astype(np.int32)
    seq3r = (1 + np.arange(pnp) // 3).astype(np.int32)
    return t, c, d, ele, hpp, hflag, seq3r


# ---------------------------------------------------------------------------
# ligand
# ---------------------------------------------------------------------------
def ligand_tree(rng, lna, bond=1.5, clash=2.2):
    xyz = np.zeros((lna, 3))
    parent = -np.ones(lna, np.int64)
    deg = np.zeros(lna, np.int64)
    for i in range(1, lna):
        for _ in range(10000):
            j = int(rng.integers(0, i))
            if deg[j] >= 4:
                continue
            v = rng.normal(size=3)
            v /= np.linalg.norm(v)
            p = xyz[j] + bond * v
            others = np.delete(xyz[:i], j, axis=0)
            if len(others) == 0 or np.min(np.linalg.norm(others - p, axis=1)) >= clash:
                xyz[i], parent[i] = p, j
                deg[i] += 1
                deg[j] += 1
                break
        else:
            raise RuntimeError("ligand growth failed")
    return xyz - xyz.mean(axis=0), parent


def _subtree(parent, root):
    kids = {}
    for i, p in enumerate(parent):
        kids.setdefault(int(p), []).append(i)
    out, stack = [], [root]
    while stack:
        k = stack.pop()
        out.append(k)
        stack.extend(kids.get(k, []))
    return np.array(out)


def ligand_conformers(rng, xyz, parent, n_conf, n_torsions=4, clash=2.2):
    confs = [xyz.copy()]
    lna = len(xyz)
    bonded = set()
    for i, p in enumerate(parent):
        if p >= 0:
            bonded.add((i, int(p)))
            bonded.add((int(p), i))
    movable = [i for i in range(1, lna)]
    while len(confs) < n_conf:
        x = confs[0].copy()
        for _ in range(n_torsions):
            for _try in range(50):
                i = int(rng.choice(movable))
                j = int(parent[i])
                sub = _subtree(parent, i)
                axis = x[i] - x[j]
                axis /= np.linalg.norm(axis)
                ang = rng.uniform(0.0, 2.0 * math.pi)
                K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]],
                              [-axis[1], axis[0], 0]])
                Rm = np.eye(3) + math.sin(ang) * K + (1 - math.cos(ang)) * (K @ K)
                y = x.copy()
                y[sub] = (x[sub] - x[j]) @ Rm.T + x[j]
                dm = np.linalg.norm(y[:, None] - y[None], axis=-1)
                ok = True
                for a in range(lna):
                    for b in range(a + 1, lna):
                        if dm[a, b] < clash and (a, b) not in bonded:
                            ok = False
                            break
                    if not ok:
                        break
                if ok:
                    x = y
                    break
        confs.append(x - x.mean(axis=0))
    return np.stack(confs)


# ---------------------------------------------------------------------------
# complex
# ---------------------------------------------------------------------------
def make_protein(rng, spec: ComplexSpec, pocket_radius: float, raw):
    if spec.cube:
        edge = spec.cube
    else:  # fixed point density outside the pocket sphere
        edge = (spec.pnp / DENSITY + 4.0 / 3.0 * math.pi * pocket_radius ** 3) ** (1.0 / 3.0)
    center = np.full(3, edge / 2.0)
    base = pack_points(rng, spec.pnp, edge, spec.min_dist, center, pocket_radius)
    confs = [base]
    for _ in range(spec.n_prt - 1):
        confs.append(base + rng.normal(0.0, spec.prt_noise, size=base.shape))
    t, c, d, ele, hpp, hflag, seq3r = protein_types(rng, spec.pnp, raw)
    return dict(xyz=np.stack(confs).astype(np.float32), t=t, c=c, d=d, ele=ele, hpp=hpp,
                hflag=hflag, seq3r=seq3r, center=center.astype(np.float32), edge=edge)


def make_template(rng, lig_xyz0, lig_t, prt, spec: ComplexSpec, pocket):
    """KDE / PSP / MCS pocket-template terms around the crystal pose."""
    lna = len(lig_t)
    pose = lig_xyz0 + pocket
    kx, kt = [], []
    for lt in np.unique(lig_t):
        atoms = np.nonzero(lig_t == lt)[0]
        for _ in range(spec.kde_per_type):
            a = int(rng.choice(atoms))
            kx.append(pose[a] + rng.normal(0.0, 1.5, size=3))
            kt.append(int(lt))
    kde_xyz = np.asarray(kx, np.float32).reshape(-1, 3)
    kde_t = np.asarray(kt, np.int32)

    n_col = int(prt["seq3r"].max()) + 1
    psp = np.zeros((abi.NLT, n_col), np.float32)
    near = np.linalg.norm(prt["xyz"][0] - pocket, axis=1) < 12.0
    cand_res = np.unique(prt["seq3r"][(prt["c"] == 2) & near])
    if len(cand_res) == 0:
        cand_res = np.unique(prt["seq3r"][prt["c"] == 2])
    types_present = np.unique(lig_t)
    for _ in range(spec.n_psp):
        psp[int(rng.choice(types_present)), int(rng.choice(cand_res))] = rng.uniform(0.0, 2.0)

    n_field = lna + 2
    mcs = np.full((spec.n_mcs, n_field, 3), abi.MCS_INVALID_COORD, np.float32)
    tcc = rng.uniform(0.1, 0.4, size=spec.n_mcs).astype(np.float32)
    for m in range(spec.n_mcs):
        k = int(rng.integers((lna + 1) // 2, lna + 1))
        atoms = rng.choice(lna, size=k, replace=False)
        for a in atoms:
            mcs[m, a + 1] = pose[a] + rng.normal(0.0, 1.0, size=3)
    return kde_xyz, kde_t, psp, mcs, tcc


def make_complex(spec: ComplexSpec, seed: int, protein: dict | None = None,
                 ff: abi.GdEnepara | None = None) -> abi.Complex:
    """A seeded synthetic complex; `protein` reuses an already generated one.
    `ff`: kernel tables to attach (default: the packaged force field through
    the library's gd_enepara_optimize); the generated geometry does not
    depend on it."""
    raw, _ = raw_ff()
    if ff is None:
        ff = default_ff()[2]
    rng = np.random.Generator(np.random.PCG64(seed))
    lig0, parent = ligand_tree(rng, spec.lna)
    r_lig = float(np.max(np.linalg.norm(lig0, axis=1)))
    if protein is None:
        protein = make_protein(rng, spec, r_lig + 2.0, raw)
    pocket = protein["center"]
    lig_xyz = ligand_conformers(rng, lig0, parent, spec.n_lig).astype(np.float32)
    lig_t = rng.integers(0, abi.NLT, size=spec.lna).astype(np.int32)
    q = rng.normal(0.0, 0.3, size=spec.lna)
    q -= (q.sum() - round(q.sum())) / spec.lna
    lig_n = np.arange(spec.lna, dtype=np.int32)
    kde_xyz, kde_t, psp, mcs, tcc = make_template(rng, lig0, lig_t, protein, spec, pocket)
    return abi.Complex(
        lig_xyz=lig_xyz, lig_t=lig_t, lig_c=q.astype(np.float32), lig_n=lig_n,
        lig_center=pocket.copy(), prt_xyz=protein["xyz"], prt_t=protein["t"],
        prt_c=protein["c"], prt_ele=protein["ele"], prt_seq3r=protein["seq3r"],
        prt_hpcflag=protein["hflag"], prt_hpp=protein["hpp"], pocket_center=pocket.copy(),
        psp=psp, kde_xyz=kde_xyz, kde_t=kde_t, mcs_xyz=mcs, mcs_tcc=tcc, ff=ff)


def random_poses(rng, n, box=8.0):
    """Rigid poses as move vectors: uniform rotations (Shoemake quaternions)
    converted to the ZYX angles of move_d.cu, translations uniform in a box."""
    u1, u2, u3 = rng.uniform(size=(3, n))
    qx = np.sqrt(1 - u1) * np.sin(2 * np.pi * u2)
    qy = np.sqrt(1 - u1) * np.cos(2 * np.pi * u2)
    qz = np.sqrt(u1) * np.sin(2 * np.pi * u3)
    qw = np.sqrt(u1) * np.cos(2 * np.pi * u3)
    r00 = 1 - 2 * (qy * qy + qz * qz)
    r10 = 2 * (qx * qy + qz * qw)
    r20 = 2 * (qx * qz - qy * qw)
    r21 = 2 * (qy * qz + qx * qw)
    r22 = 1 - 2 * (qx * qx + qy * qy)
    # R = Rz(a) Ry(b) Rx(c): r00 = cos a cos b, r10 = sin a cos b, r20 = -sin b,
    # r21 = cos b sin c, r22 = cos b cos c
    a = np.arctan2(r10, r00)
    b = -np.arcsin(np.clip(r20, -1.0, 1.0))
    c = np.arctan2(r21, r22)
    t = rng.uniform(-box / 2, box / 2, size=(n, 3))
    return np.concatenate([t, np.stack([a, b, c], axis=1)], axis=1).astype(np.float32)


def temperatures(w: Workload, set_temperature=None):
    """(temperatures, minus_beta) of the workload's geometric ladder, from
    `set_temperature(n, floor, ceiling)` (default: the library's)."""
    if set_temperature is None:
        from . import lib
        set_temperature = lib.set_temperature
    return set_temperature(w.n_tmp, w.t_floor, w.t_ceil)
