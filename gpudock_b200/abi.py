"""ctypes mirror of include/gpudock.h (structs, constants, status codes).

The structures here are byte-for-byte the C structs of the header; the
numpy-backed :class:`Complex` keeps the arrays alive while a ``gd_complex``
struct points into them.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

NPT, NLT, NELE, NRES, NTERM, NRAW = 30, 24, 50, 20, 10, 9
MCS_INVALID_COORD = np.float32(728492.0)

E_VDW, E_ELE, E_PMF, E_PSP, E_HDB, E_HPC, E_KDE, E_LHM, E_DST, E_TOTAL = range(10)
TERM_NAMES = ("vdw", "ele", "pmf", "psp", "hdb", "hpc", "kde", "lhm", "dst", "total")

MC_EXCHANGE = 0x1
MC_MOVE_AWAY = 0x2
MC_RECORD = 0x4
MC_MCC = 0x8
MC_BAYES = 0x10
CMCC_INVALID = 10000.0
# launch schedules (gd_ctx_set_schedule)
SCHED_AUTO, SCHED_WAVES, SCHED_PERSISTENT = 0, 1, 2

STATUS = {
    0: "GD_OK", 1: "GD_EINVAL", 2: "GD_ENOMEM", 3: "GD_EBUDGET", 4: "GD_ECUDA",
    5: "GD_ETIMEDOUT", 6: "GD_ECANCELLED", 7: "GD_ENOTFOUND", 8: "GD_EAGAIN",
    9: "GD_ENODEV", 10: "GD_EIO",
}
GD_OK, GD_EINVAL, GD_ENOMEM, GD_EBUDGET, GD_ECUDA = 0, 1, 2, 3, 4
GD_ETIMEDOUT, GD_ECANCELLED, GD_ENOTFOUND, GD_EAGAIN, GD_ENODEV, GD_EIO = 5, 6, 7, 8, 9, 10

f32p = C.POINTER(C.c_float)
i32p = C.POINTER(C.c_int)
f64p = C.POINTER(C.c_double)


class GdEneparaRaw(C.Structure):
    _fields_ = [
        ("vdw", C.c_float * 2 * NLT * NPT),
        ("ele", C.c_float * NELE),
        ("pmf", C.c_float * 2 * NLT * NPT),
        ("hpp", C.c_float * NRES),
        ("hpl", C.c_float * 2 * NLT),
        ("hdb", C.c_float * 2 * NLT * NPT),
        ("lj", C.c_float * 3),
        ("el", C.c_float * 2),
        ("kde", C.c_float),
        ("w", C.c_float * NTERM),
        ("a_para", C.c_float * NTERM),
        ("b_para", C.c_float * NTERM),
    ]


class GdEnepara(C.Structure):
    _fields_ = [
        ("p1a", C.c_float * NPT * NLT),
        ("p2a", C.c_float * NPT * NLT),
        ("lj0", C.c_float), ("lj1", C.c_float),
        ("el0", C.c_float), ("el1", C.c_float),
        ("ele", C.c_float * NELE),
        ("a1", C.c_float), ("b1", C.c_float),
        ("pmf0", C.c_float * NPT * NLT),
        ("pmf1", C.c_float * NPT * NLT),
        ("hdb0", C.c_float * NPT * NLT),
        ("hdb1", C.c_float * NPT * NLT),
        ("hdb2", C.c_float * NPT * NLT),
        ("hpp", C.c_float * NRES),
        ("hpl0", C.c_float * NLT), ("hpl1", C.c_float * NLT), ("hpl2", C.c_float * NLT),
        ("kde2", C.c_float), ("kde3", C.c_float),
        ("w", C.c_float * NTERM),
        ("a_para", C.c_float * NTERM),
        ("b_para", C.c_float * NTERM),
    ]


class GdProtein(C.Structure):
    _fields_ = [
        ("pnp", C.c_int), ("n_conf", C.c_int),
        ("x", f32p), ("y", f32p), ("z", f32p),
        ("t", i32p), ("c", i32p), ("ele", f32p), ("seq3r", i32p),
        ("c0_and_d12_or_c2", i32p), ("hpp", f32p),
        ("pocket_center", C.c_float * 3),
    ]


class GdLigand(C.Structure):
    _fields_ = [
        ("lna", C.c_int), ("n_conf", C.c_int),
        ("x", f32p), ("y", f32p), ("z", f32p),
        ("t", i32p), ("c", f32p), ("n", i32p),
        ("center", C.c_float * 3),
    ]


class GdPsp(C.Structure):
    _fields_ = [("n_col", C.c_int), ("psp", f32p)]


class GdKde(C.Structure):
    _fields_ = [("pnk", C.c_int), ("x", f32p), ("y", f32p), ("z", f32p), ("t", i32p)]


class GdMcs(C.Structure):
    _fields_ = [
        ("pos", C.c_int), ("n_field", C.c_int),
        ("x", f32p), ("y", f32p), ("z", f32p), ("tcc", f32p),
    ]


class GdComplex(C.Structure):
    _fields_ = [
        ("lig", GdLigand), ("prt", GdProtein), ("psp", GdPsp), ("kde", GdKde),
        ("mcs", GdMcs), ("ff", C.POINTER(GdEnepara)),
    ]


class GdTile(C.Structure):
    _fields_ = [("atom_groups", C.c_int), ("tile_groups", C.c_int), ("atoms_per_warp", C.c_int)]


class GdServerStats(C.Structure):
    _fields_ = [
        ("queued", C.c_int), ("active", C.c_int), ("completed", C.c_uint64),
        ("iterations", C.c_uint64), ("launches", C.c_uint64), ("bytes_in_use", C.c_size_t),
        ("busy_s", C.c_double), ("cta_busy_s", C.c_double), ("host_launch_s", C.c_double),
    ]


class GdMcParams(C.Structure):
    _fields_ = [
        ("steps_total", C.c_int), ("steps_per_exchange", C.c_int),
        ("steps_per_dump", C.c_int), ("n_tmp", C.c_int),
        ("move_scale", C.c_float * 6),
        ("minus_beta", f32p),
        ("seed", C.c_uint64), ("stream_id", C.c_uint32), ("flags", C.c_uint32),
    ]


class GdRecord(C.Structure):
    _fields_ = [
        ("idx_rep", C.c_int), ("idx_prt", C.c_int), ("idx_tmp", C.c_int), ("idx_lig", C.c_int),
        ("e", C.c_float * NTERM), ("cmcc", C.c_float),
        ("movematrix", C.c_float * 6), ("step", C.c_int),
        ("e_prop_total", C.c_float), ("accepted", C.c_int),
    ]


RECORD_DTYPE = np.dtype([
    ("idx_rep", "<i4"), ("idx_prt", "<i4"), ("idx_tmp", "<i4"), ("idx_lig", "<i4"),
    ("e", "<f4", (NTERM,)), ("cmcc", "<f4"), ("movematrix", "<f4", (6,)), ("step", "<i4"),
    ("e_prop_total", "<f4"), ("accepted", "<i4"),
])
assert RECORD_DTYPE.itemsize == C.sizeof(GdRecord)


class GdMcLog(C.Structure):
    _fields_ = [
        ("t_compute", C.c_double), ("t_wall", C.c_double),
        ("ac_mc", C.c_int64), ("ac_temp_exchg", C.c_int64),
        ("acs_mc", i32p), ("acs_temp_exchg", i32p),
        ("energy", f32p), ("movematrix", f32p), ("idx_tmp", i32p),
        ("record", C.POINTER(GdRecord)),
    ]


def _ptr(a: Optional[np.ndarray], ctype):
    if a is None:
        return C.cast(None, C.POINTER(ctype))
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(C.POINTER(ctype))


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


@dataclass
class Complex:
    """A docking complex held as numpy arrays (caller-owned host buffers).

    Shapes: lig_xyz [n_lig, lna, 3] (relative to the ligand centre),
    prt_xyz [n_prt, pnp, 3]; per-point and per-atom vectors as in
    ``gd_protein`` / ``gd_ligand``.
    """

    lig_xyz: np.ndarray
    lig_t: np.ndarray
    lig_c: np.ndarray
    lig_n: np.ndarray
    lig_center: np.ndarray
    prt_xyz: np.ndarray
    prt_t: np.ndarray
    prt_c: np.ndarray
    prt_ele: np.ndarray
    prt_seq3r: np.ndarray
    prt_hpcflag: np.ndarray
    prt_hpp: np.ndarray
    pocket_center: np.ndarray
    psp: np.ndarray            # [NLT, n_col]
    kde_xyz: np.ndarray        # [pnk, 3]
    kde_t: np.ndarray          # [pnk]
    mcs_xyz: np.ndarray        # [pos, n_field, 3]
    mcs_tcc: np.ndarray        # [pos]
    ff: GdEnepara
    _keep: list = field(default_factory=list, repr=False)
    _struct: Optional[GdComplex] = field(default=None, repr=False)

    @property
    def lna(self) -> int:
        return int(self.lig_xyz.shape[1])

    @property
    def n_lig(self) -> int:
        return int(self.lig_xyz.shape[0])

    @property
    def pnp(self) -> int:
        return int(self.prt_xyz.shape[1])

    @property
    def n_prt(self) -> int:
        return int(self.prt_xyz.shape[0])

    @property
    def pnk(self) -> int:
        return int(self.kde_xyz.shape[0])

    @property
    def pos(self) -> int:
        return int(self.mcs_xyz.shape[0])

    def struct(self) -> GdComplex:
        """Builds (once) the gd_complex pointing into this object's arrays."""
        if self._struct is not None:
            return self._struct
        k = self._keep
        k.clear()

        def keep(a):
            k.append(a)
            return a

        lx = keep(_f32(self.lig_xyz[..., 0]))
        ly = keep(_f32(self.lig_xyz[..., 1]))
        lz = keep(_f32(self.lig_xyz[..., 2]))
        lt, lc, ln = keep(_i32(self.lig_t)), keep(_f32(self.lig_c)), keep(_i32(self.lig_n))
        px = keep(_f32(self.prt_xyz[..., 0]))
        py = keep(_f32(self.prt_xyz[..., 1]))
        pz = keep(_f32(self.prt_xyz[..., 2]))
        pt, pc = keep(_i32(self.prt_t)), keep(_i32(self.prt_c))
        pe, ps = keep(_f32(self.prt_ele)), keep(_i32(self.prt_seq3r))
        ph, pp = keep(_i32(self.prt_hpcflag)), keep(_f32(self.prt_hpp))
        psp = keep(_f32(self.psp))
        kx = keep(_f32(self.kde_xyz[:, 0])) if self.pnk else keep(np.zeros(1, np.float32))
        ky = keep(_f32(self.kde_xyz[:, 1])) if self.pnk else keep(np.zeros(1, np.float32))
        kz = keep(_f32(self.kde_xyz[:, 2])) if self.pnk else keep(np.zeros(1, np.float32))
        kt = keep(_i32(self.kde_t)) if self.pnk else keep(np.zeros(1, np.int32))
        nf = int(self.mcs_xyz.shape[1]) if self.mcs_xyz.ndim == 3 else 1
        mx = keep(_f32(self.mcs_xyz[..., 0]).reshape(-1)) if self.pos else keep(np.zeros(1, np.float32))
        my = keep(_f32(self.mcs_xyz[..., 1]).reshape(-1)) if self.pos else keep(np.zeros(1, np.float32))
        mz = keep(_f32(self.mcs_xyz[..., 2]).reshape(-1)) if self.pos else keep(np.zeros(1, np.float32))
        mt = keep(_f32(self.mcs_tcc)) if self.pos else keep(np.zeros(1, np.float32))
        keep(self.ff)

        s = GdComplex()
        s.lig = GdLigand(self.lna, self.n_lig, _ptr(lx, C.c_float), _ptr(ly, C.c_float),
                         _ptr(lz, C.c_float), _ptr(lt, C.c_int), _ptr(lc, C.c_float),
                         _ptr(ln, C.c_int), (C.c_float * 3)(*map(float, self.lig_center)))
        s.prt = GdProtein(self.pnp, self.n_prt, _ptr(px, C.c_float), _ptr(py, C.c_float),
                          _ptr(pz, C.c_float), _ptr(pt, C.c_int), _ptr(pc, C.c_int),
                          _ptr(pe, C.c_float), _ptr(ps, C.c_int), _ptr(ph, C.c_int),
                          _ptr(pp, C.c_float),
                          (C.c_float * 3)(*map(float, self.pocket_center)))
        s.psp = GdPsp(int(self.psp.shape[1]), _ptr(psp, C.c_float))
        s.kde = GdKde(self.pnk, _ptr(kx, C.c_float), _ptr(ky, C.c_float), _ptr(kz, C.c_float),
                      _ptr(kt, C.c_int))
        s.mcs = GdMcs(self.pos, nf, _ptr(mx, C.c_float), _ptr(my, C.c_float),
                      _ptr(mz, C.c_float), _ptr(mt, C.c_float))
        s.ff = C.pointer(self.ff)
        self._struct = s
        return s


def mc_params(steps_total: int, steps_per_exchange: int, minus_beta: np.ndarray,
              move_scale=(0.02, 0.02, 0.02, 0.08, 0.08, 0.08), seed: int = 1,
              stream_id: int = 0, flags: int = MC_EXCHANGE, steps_per_dump: int = 1000):
    """Builds a gd_mc_params; returns (struct, keep-alive array)."""
    mb = np.ascontiguousarray(minus_beta, dtype=np.float32)
    p = GdMcParams()
    p.steps_total = int(steps_total)
    p.steps_per_exchange = int(steps_per_exchange)
    p.steps_per_dump = int(steps_per_dump)
    p.n_tmp = int(mb.shape[0])
    p.move_scale = (C.c_float * 6)(*map(float, move_scale))
    p.minus_beta = _ptr(mb, C.c_float)
    p.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    p.stream_id = int(stream_id) & 0xFFFFFFFF
    p.flags = int(flags)
    return p, mb


class McLogBuffers:
    """Host output buffers of one run, wired into a GdMcLog."""

    def __init__(self, n_rep: int, n_tmp: int, steps_total: int = 0, record: bool = False):
        self.acs_mc = np.zeros(n_rep, np.int32)
        self.acs_temp_exchg = np.zeros(n_tmp, np.int32)
        self.energy = np.zeros((n_rep, NTERM), np.float32)
        self.movematrix = np.zeros((n_rep, 6), np.float32)
        self.idx_tmp = np.zeros(n_rep, np.int32)
        self.record = np.zeros((n_rep, steps_total), RECORD_DTYPE) if record else None
        self.log = GdMcLog()
        self.log.acs_mc = _ptr(self.acs_mc, C.c_int)
        self.log.acs_temp_exchg = _ptr(self.acs_temp_exchg, C.c_int)
        self.log.energy = _ptr(self.energy, C.c_float)
        self.log.movematrix = _ptr(self.movematrix, C.c_float)
        self.log.idx_tmp = _ptr(self.idx_tmp, C.c_int)
        self.log.record = (self.record.ctypes.data_as(C.POINTER(GdRecord))
                           if record else C.cast(None, C.POINTER(GdRecord)))

    @property
    def ac_mc(self) -> int:
        return int(self.log.ac_mc)

    @property
    def ac_temp_exchg(self) -> int:
        return int(self.log.ac_temp_exchg)


def enepara_from_arrays(d: dict) -> GdEnepara:
    """GdEnepara from a dict of numpy arrays keyed by field name."""
    e = GdEnepara()
    buf = np.frombuffer(e, dtype=np.uint8)
    for name, ctype in GdEnepara._fields_:
        off = getattr(GdEnepara, name).offset
        a = np.ascontiguousarray(d[name], dtype=np.float32).reshape(-1)
        buf[off:off + a.nbytes] = a.view(np.uint8)
    return e


def enepara_to_arrays(e) -> dict:
    out = {}
    cls = type(e)
    raw = bytes(e)
    for name, ctype in cls._fields_:
        off = getattr(cls, name).offset
        size = C.sizeof(ctype)
        a = np.frombuffer(raw[off:off + size], dtype=np.float32).copy()
        out[name] = a if a.size > 1 else a[0]
    return out


def raw_from_arrays(d: dict) -> GdEneparaRaw:
    e = GdEneparaRaw()
    buf = np.frombuffer(e, dtype=np.uint8)
    for name, ctype in GdEneparaRaw._fields_:
        off = getattr(GdEneparaRaw, name).offset
        a = np.ascontiguousarray(d[name], dtype=np.float32).reshape(-1)
        assert a.nbytes == C.sizeof(ctype), (name, a.nbytes, C.sizeof(ctype))
        buf[off:off + a.nbytes] = a.view(np.uint8)
    return e
