"""Python wrapper of the CPU oracle (oracle/gd_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by bench.py's CPU-baseline leg, never by the gpudock_b200 package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from gpudock_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libgdoracle.so")
LIB_NATIVE = os.path.join(HERE, "_build", "libgdoracle_native.so")

_libs = {}
_max_threads = {}


def reference_root():
    """The reference checkout the checker reads sample inputs and sources
    from (GD_REFERENCE, else the default of oracle/Makefile.ref), or None
    where it is absent."""
    ref = os.environ.get("GD_REFERENCE")
    if not ref:
        try:
            ref = subprocess.run(["make", "-s", "-f", "Makefile.ref", "print-ref"], cwd=HERE,
                                 capture_output=True, text=True, check=True).stdout.strip()
        except Exception:
            return None
    return ref if ref and os.path.isdir(ref) else None


def build(native: bool = False) -> str:
    target = "native" if native else "all"
    path = LIB_NATIVE if native else LIB
    src = os.path.join(HERE, "gd_oracle.c")
    if os.path.exists(path) and os.path.getmtime(path) >= os.path.getmtime(src):
        return path
    subprocess.run(["make", "-s", "-C", HERE, target], check=True)
    return path


def load(native: bool = False):
    key = "native" if native else "portable"
    if key in _libs:
        return _libs[key]
    path = build(native)
    lib = C.CDLL(path)
    P = C.c_void_p
    lib.orc_philox.argtypes = [P, P, P]
    lib.orc_expf.argtypes = [C.c_float]
    lib.orc_expf.restype = C.c_float
    lib.orc_metropolis.argtypes = [C.c_float, C.c_float, C.c_float, C.c_uint64, C.c_uint32,
                                   C.c_int, C.c_int]
    lib.orc_metropolis.restype = C.c_int
    lib.orc_enepara_optimize.argtypes = [C.POINTER(abi.GdEneparaRaw), C.POINTER(abi.GdEnepara)]
    lib.orc_set_temperature.argtypes = [C.c_int, C.c_float, C.c_float, P, P]
    lib.orc_energy_pose.argtypes = [C.POINTER(abi.GdComplex), C.c_int, C.c_int, P, P, P, P]
    lib.orc_energy_poses.argtypes = [C.POINTER(abi.GdComplex), C.c_int, C.c_int, C.c_int, P, P,
                                     P, P, C.c_int]
    lib.orc_exchange.argtypes = [C.POINTER(abi.GdMcParams), C.c_int, C.c_int, C.c_int, C.c_int,
                                 C.c_int, P, P, P]
    lib.orc_remc_run.argtypes = [C.POINTER(abi.GdComplex), C.POINTER(abi.GdMcParams),
                                 C.POINTER(abi.GdMcLog), C.c_int]
    lib.orc_remc_run.restype = C.c_int
    lib.orc_mc_sample.argtypes = [C.POINTER(abi.GdComplex), C.POINTER(abi.GdMcParams), C.c_int,
                                  C.c_int, C.c_int, C.c_int]
    lib.orc_mc_sample.restype = C.c_longlong
    lib.orc_similarity_matrix.argtypes = [C.POINTER(abi.GdComplex), C.c_int, P, P]
    lib.orc_max_threads.restype = C.c_int
    lib.orc_mcc.argtypes = [C.POINTER(abi.GdComplex), C.c_int, C.c_int, C.c_int, P]
    lib.orc_mcc.restype = C.c_float
    lib.orc_bayes_total.argtypes = [P]
    lib.orc_bayes_total.restype = C.c_float
    _libs[key] = lib
    # OpenMP's thread count is process-wide and a call with n_threads sets
    # it for good: note the host's before any call does
    _max_threads.setdefault("n", int(lib.orc_max_threads()))
    return lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def philox(ctr: np.ndarray, key: np.ndarray) -> np.ndarray:
    lib = load()
    ctr = np.ascontiguousarray(ctr, np.uint32).reshape(-1, 4)
    key = np.ascontiguousarray(key, np.uint32).reshape(-1, 2)
    out = np.zeros_like(ctr)
    for i in range(ctr.shape[0]):
        lib.orc_philox(_p(ctr[i]), _p(key[i]), _p(out[i]))
    return out


def expf(x: np.ndarray) -> np.ndarray:
    lib = load()
    x = np.asarray(x, np.float32).reshape(-1)
    return np.array([lib.orc_expf(float(v)) for v in x], np.float32)


def metropolis(e_new, e_old, mbeta, seed, stream, rep, step) -> np.ndarray:
    lib = load()
    return np.array([lib.orc_metropolis(float(a), float(b), float(m), int(seed), int(stream),
                                        int(r), int(s))
                     for a, b, m, r, s in zip(e_new, e_old, mbeta, rep, step)], np.int32)


def enepara_optimize(raw: abi.GdEneparaRaw) -> abi.GdEnepara:
    out = abi.GdEnepara()
    load().orc_enepara_optimize(C.byref(raw), C.byref(out))
    return out


def set_temperature(n: int, floor_t: float, ceil_t: float):
    t = np.zeros(n, np.float32)
    mb = np.zeros(n, np.float32)
    load().orc_set_temperature(n, floor_t, ceil_t, _p(t), _p(mb))
    return t, mb


def energy_poses(cx: abi.Complex, poses: np.ndarray, prt_conf: int = 0, lig_conf: int = 0,
                 n_threads: int = 0, native: bool = False):
    """terms [n,10] f32, raw [n,9] f64, abs_sum [n,5] f64 (|contribution| sums)."""
    lib = load(native)
    poses = np.ascontiguousarray(poses, np.float32).reshape(-1, 6)
    n = poses.shape[0]
    terms = np.zeros((n, abi.NTERM), np.float32)
    raw = np.zeros((n, abi.NRAW), np.float64)
    asum = np.zeros((n, 5), np.float64)
    lib.orc_energy_poses(C.byref(cx.struct()), prt_conf, lig_conf, n, _p(poses), _p(terms),
                         _p(raw), _p(asum), n_threads or max_threads(native))
    return terms, raw, asum


def exchange(params: abi.GdMcParams, n_prt: int, n_lig: int, n_tmp: int, rnd: int, mode_t: int,
             etotal: np.ndarray, idx_tmp: np.ndarray):
    """One exchange round on given totals; returns (new idx_tmp, slot counters)."""
    et = np.ascontiguousarray(etotal, np.float32)
    it = np.ascontiguousarray(idx_tmp, np.int32).copy()
    acs = np.zeros(n_tmp, np.int32)
    load().orc_exchange(C.byref(params), n_prt, n_lig, n_tmp, rnd, mode_t, _p(et), _p(it),
                        _p(acs))
    return it, acs


def remc_run(cx: abi.Complex, steps_total: int, steps_per_exchange: int, minus_beta,
             n_threads: int = 0, **kw) -> abi.McLogBuffers:
    params, mb = abi.mc_params(steps_total, steps_per_exchange, minus_beta, **kw)
    n_rep = cx.n_prt * cx.n_lig * len(mb)
    buf = abi.McLogBuffers(n_rep, len(mb), steps_total, bool(params.flags & abi.MC_RECORD))
    st = load().orc_remc_run(C.byref(cx.struct()), C.byref(params), C.byref(buf.log),
                             n_threads or max_threads())
    if st != 0:
        raise RuntimeError(f"orc_remc_run: status {st}")
    return buf


def mc_sample(cx: abi.Complex, params: abi.GdMcParams, r0: int, n_rep: int, n_steps: int,
              n_threads: int = 0, native: bool = False) -> int:
    return int(load(native).orc_mc_sample(C.byref(cx.struct()), C.byref(params), r0, n_rep,
                                          n_steps, n_threads or max_threads(native)))


def max_threads(native: bool = False) -> int:
    """Threads an all-cores call uses: OpenMP's default for this process,
    noted when the oracle was first loaded."""
    load(native)
    return _max_threads["n"]


def mcc(cx: abi.Complex, ref_prt: int, prt_conf: int, lig_conf: int, m) -> float:
    """Contact MCC of the pose m (6-vector) against the complex's reference
    map (ligand conformation 0, start pose, protein conformation ref_prt)."""
    mv = np.ascontiguousarray(m, np.float32).reshape(6)
    return float(load().orc_mcc(C.byref(cx.struct()), ref_prt, prt_conf, lig_conf,
                                mv.ctypes.data))


def similarity_matrix(cx: abi.Complex, confs: np.ndarray) -> np.ndarray:
    """Contact-mode similarity matrix [n, n] of trace rows [n, 8]."""
    confs = np.ascontiguousarray(confs, np.float32).reshape(-1, 8)
    n = confs.shape[0]
    out = np.zeros((n, n), np.float32)
    load().orc_similarity_matrix(C.byref(cx.struct()), n, _p(confs), _p(out))
    return out


def bayes_total(e) -> np.ndarray:
    """Bayesian total (IS_BAYE) of normalised terms e[..., :9] (rem order)."""
    e = np.ascontiguousarray(e, np.float32).reshape(-1, np.shape(e)[-1])
    lib = load()
    out = np.empty(len(e), np.float32)
    for i in range(len(e)):
        row = np.ascontiguousarray(e[i, :9])
        out[i] = lib.orc_bayes_total(row.ctypes.data)
    return out
