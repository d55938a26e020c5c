"""ctypes binding of libgpudock.so (the C-ABI of include/gpudock.h).

The library is built in-tree by :mod:`gpudock_b200.build`; loading it never
falls back to anything else: a missing or unloadable library raises.
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libgpudock.so")

_lib = None


class GdError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        self.status = status
        super().__init__(f"{where}: {abi.STATUS.get(status, status)}: {msg}")


def _declare(lib):
    P = C.c_void_p
    i32, u32, u64 = C.c_int, C.c_uint32, C.c_uint64
    sigs = {
        "gd_last_error": ([], C.c_char_p),
        "gd_version": ([], C.c_char_p),
        "gd_enepara_optimize": ([C.POINTER(abi.GdEneparaRaw), C.POINTER(abi.GdEnepara)], i32),
        "gd_set_temperature": ([i32, C.c_float, C.c_float, abi.f32p, abi.f32p], i32),
        "gd_poses_from_quaternions": ([i32, abi.f32p, abi.f32p], i32),
        "gd_similarity_matrix": ([P, P, i32, abi.f32p, abi.f32p], i32),
        "gd_similarity_matrix_dev": ([P, P, i32, abi.f32p, P], i32),
        "gd_complex_validate": ([C.POINTER(abi.GdComplex)], i32),
        "gd_ctx_create": ([i32, P, C.POINTER(P)], i32),
        "gd_ctx_destroy": ([P], i32),
        "gd_ctx_sync": ([P], i32),
        "gd_ctx_launch_count": ([P], u64),
        "gd_complex_upload": ([P, C.POINTER(abi.GdComplex), C.POINTER(P)], i32),
        "gd_complex_upload_shared": ([P, C.POINTER(abi.GdComplex), P, i32, i32, C.POINTER(P)],
                                     i32),
        "gd_autotune": ([P, P, C.POINTER(abi.GdTile), C.POINTER(C.c_double)], i32),
        "gd_ctx_set_tile": ([P, i32, i32, C.POINTER(abi.GdTile)], i32),
        "gd_ctx_set_schedule": ([P, i32, i32], i32),
        "gd_ctx_set_schedule_tail": ([P, i32], i32),
        "gd_ctx_set_split": ([P, i32], i32),
        "gd_ctx_set_wait_test": ([P, C.c_uint, i32], i32),
        "gd_ctx_set_alloc_fail": ([P, i32], i32),
        "gd_remc_snapshot": ([P, P, C.c_size_t, C.POINTER(C.c_size_t)], i32),
        "gd_remc_restore": ([P, P, C.c_size_t], i32),
        "gd_batch_snapshot": ([P, P, C.c_size_t, C.POINTER(C.c_size_t)], i32),
        "gd_batch_restore": ([P, P, C.c_size_t], i32),
        "gd_load": ([C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p,
                     C.POINTER(abi.GdEneparaRaw), C.POINTER(abi.GdEnepara), C.c_uint,
                     C.POINTER(P)], i32),
        "gd_loaded_complex": ([P, C.POINTER(abi.GdComplex)], i32),
        "gd_loaded_ligand_id": ([P], C.c_char_p),
        "gd_loaded_free": ([P], i32),
        "gd_load_enepara": ([C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p,
                             C.POINTER(abi.GdEneparaRaw)], i32),
        "gd_schedule_pieces": ([C.POINTER(C.c_double), C.POINTER(C.c_int), i32, i32,
                                C.POINTER(C.c_int), i32, C.POINTER(C.c_int),
                                C.POINTER(C.c_int)], i32),
        "gd_schedule_queue": ([C.POINTER(C.c_double), C.POINTER(C.c_int), i32, i32, i32,
                               C.POINTER(C.c_int), i32, C.POINTER(C.c_int),
                               C.POINTER(C.c_int)], i32),
        "gd_batch_create": ([P, i32, C.POINTER(P), C.POINTER(abi.GdMcParams), C.POINTER(P)], i32),
        "gd_batch_init": ([P], i32),
        "gd_batch_run": ([P, i32], i32),
        "gd_batch_read": ([P, i32, C.POINTER(abi.GdMcLog)], i32),
        "gd_batch_destroy": ([P], i32),
        "gd_batch_n_rep": ([P], i32),
        "gd_batch_n_launch_shapes": ([P], i32),
        "gd_batch_set_profiling": ([P, i32], i32),
        "gd_batch_kernel_times": ([P, C.POINTER(C.c_double), C.POINTER(C.c_int),
                                   C.POINTER(C.c_double), C.POINTER(C.c_int)], i32),
        "gd_server_create": ([i32, C.c_size_t, i32, i32, C.POINTER(P)], i32),
        "gd_server_add_protein": ([P, C.POINTER(abi.GdComplex), C.POINTER(C.c_int)], i32),
        "gd_server_submit": ([P, i32, C.POINTER(abi.GdComplex), C.POINTER(abi.GdMcParams),
                              C.POINTER(C.c_uint64)], i32),
        "gd_server_poll": ([P, C.c_uint64, C.POINTER(abi.GdMcLog)], i32),
        "gd_server_wait": ([P, C.c_uint64, i32, C.POINTER(abi.GdMcLog)], i32),
        "gd_server_cancel": ([P, C.c_uint64], i32),
        "gd_server_get_stats": ([P, C.POINTER(abi.GdServerStats)], i32),
        "gd_server_destroy": ([P], i32),
        "gd_server_context": ([P], P),
        "gd_complex_free": ([P], i32),
        "gd_complex_device_bytes": ([P], C.c_size_t),
        "gd_energy_poses_dev": ([P, P, i32, i32, i32, P, P, P], i32),
        "gd_energy_poses": ([P, P, i32, i32, i32, abi.f32p, abi.f32p, abi.f64p], i32),
        "gd_remc_create": ([P, P, C.POINTER(abi.GdMcParams), C.POINTER(P)], i32),
        "gd_remc_init": ([P], i32),
        "gd_remc_run": ([P, i32], i32),
        "gd_remc_read": ([P, C.POINTER(abi.GdMcLog)], i32),
        "gd_remc_destroy": ([P], i32),
        "gd_remc_n_rep": ([P], i32),
        "gd_remc_set_profiling": ([P, i32], i32),
        "gd_remc_set_trajectory": ([P, C.c_char_p, C.c_char_p], i32),
        "gd_remc_kernel_times": ([P, C.POINTER(C.c_double), C.POINTER(C.c_int),
                                  C.POINTER(C.c_double), C.POINTER(C.c_int)], i32),
        "gd_run": ([C.POINTER(abi.GdComplex), C.POINTER(abi.GdMcParams), C.POINTER(abi.GdMcLog)], i32),
        "gd_metropolis_dev": ([P, i32, P, P, P, P, P, u64, u32, P], i32),
        "gd_philox_dev": ([P, i32, P, P, P], i32),
        "gd_expf_dev": ([P, i32, P, P], i32),
        "gd_fma_peak": ([P, i32, i32, C.POINTER(C.c_float), C.POINTER(C.c_double)], i32),
    }
    for name, (args, res) in sigs.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.argtypes = args
        fn.restype = res


def load(path: str = LIB_PATH):
    """Loads libgpudock.so (building it first when the sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path) or os.environ.get("GD_REBUILD"):
        from . import build
        build.build()
    lib = C.CDLL(path)
    _declare(lib)
    _lib = lib
    return lib


def last_error() -> str:
    return load().gd_last_error().decode(errors="replace")


def check(status: int, where: str):
    if status != abi.GD_OK:
        raise GdError(status, where, last_error())


# ---------------------------------------------------------------------------
# Host-side helpers (no GPU needed)
# ---------------------------------------------------------------------------
def enepara_optimize(raw: abi.GdEneparaRaw) -> abi.GdEnepara:
    out = abi.GdEnepara()
    check(load().gd_enepara_optimize(C.byref(raw), C.byref(out)), "gd_enepara_optimize")
    return out


def set_temperature(n: int, floor_t: float, ceil_t: float):
    t = np.zeros(n, np.float32)
    mb = np.zeros(n, np.float32)
    check(load().gd_set_temperature(n, floor_t, ceil_t, abi._ptr(t, C.c_float),
                                    abi._ptr(mb, C.c_float)), "gd_set_temperature")
    return t, mb


def poses_from_quaternions(quat_poses: np.ndarray) -> np.ndarray:
    """[n][7] {tx, ty, tz, qw, qx, qy, qz} -> [n][6] move vectors
    (gd_poses_from_quaternions)."""
    q = np.ascontiguousarray(quat_poses, np.float32).reshape(-1, 7)
    out = np.zeros((q.shape[0], 6), np.float32)
    check(load().gd_poses_from_quaternions(q.shape[0], abi._ptr(q, C.c_float),
                                           abi._ptr(out, C.c_float)),
          "gd_poses_from_quaternions")
    return out


def validate(cx: abi.Complex) -> int:
    return load().gd_complex_validate(C.byref(cx.struct()))


# ---------------------------------------------------------------------------
# Device objects
# ---------------------------------------------------------------------------
class Context:
    """A CUDA device + stream bound to the library (gd_ctx)."""

    def __init__(self, device: int = 0, stream: int | None = None):
        self._lib = load()
        h = C.c_void_p()
        check(self._lib.gd_ctx_create(device, C.c_void_p(stream) if stream else None,
                                      C.byref(h)), "gd_ctx_create")
        self.h = h
        self.device = device

    def sync(self):
        check(self._lib.gd_ctx_sync(self.h), "gd_ctx_sync")

    @property
    def launches(self) -> int:
        return int(self._lib.gd_ctx_launch_count(self.h))

    def set_split(self, split: int):
        """CTAs per 32-replica unit of MC launches (0: chosen per complex)."""
        check(self._lib.gd_ctx_set_split(self.h, split), "gd_ctx_set_split")

    def set_schedule(self, mode: int, machines: int = 0):
        """abi.SCHED_AUTO / SCHED_WAVES / SCHED_PERSISTENT (over `machines` CTAs)."""
        check(self._lib.gd_ctx_set_schedule(self.h, mode, machines), "gd_ctx_set_schedule")

    def set_schedule_tail(self, tail: int):
        """MC steps per unit left to a persistent launch's shared queue
        (gd_ctx_set_schedule_tail; default 2, 0: none)."""
        check(self._lib.gd_ctx_set_schedule_tail(self.h, tail), "gd_ctx_set_schedule_tail")

    def set_wait_test(self, wait_limit: int, never_release: bool):
        """Test hook: dependency waits of later MC launches give up after
        `wait_limit` polls; with never_release every one of them runs out
        (gd_ctx_set_wait_test).  set_wait_test(0, False) restores the default."""
        check(self._lib.gd_ctx_set_wait_test(self.h, int(wait_limit), int(never_release)),
              "gd_ctx_set_wait_test")

    def set_alloc_fail(self, nth: int):
        """Test hook: the nth device allocation from now fails with GD_ENOMEM
        (gd_ctx_set_alloc_fail); 0 turns it off."""
        check(self._lib.gd_ctx_set_alloc_fail(self.h, int(nth)), "gd_ctx_set_alloc_fail")

    def close(self):
        if self.h:
            self._lib.gd_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class DeviceComplex:
    """A complex uploaded to the device in the kernel layout (gd_dcomplex).

    With ``share`` the protein arrays of that uploaded complex are reused
    (conformations ``prt_conf0 .. prt_conf0 + n_prt - 1``) instead of copied.
    """

    def __init__(self, ctx: Context, cx: abi.Complex, share: "DeviceComplex | None" = None,
                 prt_conf0: int = 0, n_prt: int = 1):
        self.ctx = ctx
        self.cx = cx
        self.share = share
        h = C.c_void_p()
        self.n_prt_view = cx.n_prt if share is None else n_prt
        if share is None:
            check(ctx._lib.gd_complex_upload(ctx.h, C.byref(cx.struct()), C.byref(h)),
                  "gd_complex_upload")
        else:
            check(ctx._lib.gd_complex_upload_shared(ctx.h, C.byref(cx.struct()), share.h,
                                                    prt_conf0, n_prt, C.byref(h)),
                  "gd_complex_upload_shared")
        self.h = h

    def autotune(self):
        """Autotunes the launch shape of this complex's size class."""
        t = abi.GdTile()
        ms = C.c_double()
        check(self.ctx._lib.gd_autotune(self.ctx.h, self.h, C.byref(t), C.byref(ms)),
              "gd_autotune")
        return (t.atom_groups, t.tile_groups, t.atoms_per_warp), ms.value

    @property
    def size_class(self):
        """(ligand-size bucket, protein tiles): the key of the context's shape cache."""
        return lna_bucket(self.cx.lna), (self.cx.pnp + 127) // 128

    @property
    def device_bytes(self) -> int:
        return int(self.ctx._lib.gd_complex_device_bytes(self.h))

    def energy_poses(self, poses: np.ndarray, prt_conf: int = 0, lig_conf: int = 0,
                     raw: bool = True):
        """Host-buffer call: terms [n, 10] float32 and raw [n, 9] float64."""
        poses = np.ascontiguousarray(poses, np.float32).reshape(-1, 6)
        n = poses.shape[0]
        terms = np.zeros((n, abi.NTERM), np.float32)
        rw = np.zeros((n, abi.NRAW), np.float64) if raw else None
        check(self.ctx._lib.gd_energy_poses(
            self.ctx.h, self.h, prt_conf, lig_conf, n, abi._ptr(poses, C.c_float),
            abi._ptr(terms, C.c_float), abi._ptr(rw, C.c_double)), "gd_energy_poses")
        return terms, rw

    def similarity_matrix(self, confs: np.ndarray) -> np.ndarray:
        """Contact-mode similarity matrix [n, n] of conformations [n, 8]
        (trace-file rows: protein conf, ligand conf, move vector)
        (gd_similarity_matrix)."""
        confs = np.ascontiguousarray(confs, np.float32).reshape(-1, 8)
        n = confs.shape[0]
        out = np.zeros((n, n), np.float32)
        check(self.ctx._lib.gd_similarity_matrix(self.ctx.h, self.h, n,
                                                  abi._ptr(confs, C.c_float),
                                                  abi._ptr(out, C.c_float)),
              "gd_similarity_matrix")
        return out

    def similarity_matrix_dev(self, confs: np.ndarray, out_ptr: int) -> None:
        """The matrix into device memory at out_ptr (n * n floats)
        (gd_similarity_matrix_dev)."""
        confs = np.ascontiguousarray(confs, np.float32).reshape(-1, 8)
        check(self.ctx._lib.gd_similarity_matrix_dev(self.ctx.h, self.h, confs.shape[0],
                                                      abi._ptr(confs, C.c_float),
                                                      C.c_void_p(out_ptr)),
              "gd_similarity_matrix_dev")

    def energy_poses_dev(self, n: int, poses_ptr: int, terms_ptr: int, raw_ptr: int = 0,
                         prt_conf: int = 0, lig_conf: int = 0):
        """Device-pointer call (asynchronous on the context stream)."""
        check(self.ctx._lib.gd_energy_poses_dev(
            self.ctx.h, self.h, prt_conf, lig_conf, n, C.c_void_p(poses_ptr),
            C.c_void_p(terms_ptr), C.c_void_p(raw_ptr) if raw_ptr else None),
            "gd_energy_poses_dev")

    def close(self):
        if self.h:
            self.ctx._lib.gd_complex_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Remc:
    """Replica-exchange Monte Carlo of one uploaded complex (gd_remc)."""

    def __init__(self, dcx: DeviceComplex, steps_total: int, steps_per_exchange: int,
                 minus_beta, move_scale=(0.02, 0.02, 0.02, 0.08, 0.08, 0.08), seed: int = 1,
                 stream_id: int = 0, flags: int = abi.MC_EXCHANGE, steps_per_dump: int = 1000):
        self.dcx = dcx
        self.params, self._mb = abi.mc_params(steps_total, steps_per_exchange, minus_beta,
                                              move_scale, seed, stream_id, flags, steps_per_dump)
        h = C.c_void_p()
        lib = dcx.ctx._lib
        check(lib.gd_remc_create(dcx.ctx.h, dcx.h, C.byref(self.params), C.byref(h)),
              "gd_remc_create")
        self.h = h
        self.n_rep = int(lib.gd_remc_n_rep(h))
        self.n_tmp = int(self.params.n_tmp)
        self.steps_total = int(steps_total)
        self.record = bool(flags & abi.MC_RECORD)

    def init(self):
        check(self.dcx.ctx._lib.gd_remc_init(self.h), "gd_remc_init")

    def run(self, n_steps: int):
        check(self.dcx.ctx._lib.gd_remc_run(self.h, int(n_steps)), "gd_remc_run")

    def set_profiling(self, on: bool = True):
        check(self.dcx.ctx._lib.gd_remc_set_profiling(self.h, int(on)), "gd_remc_set_profiling")

    def set_trajectory(self, directory: str, stem: str):
        """Writes every completed dump of steps_per_dump MC steps to
        {directory}/{stem}_NNNN.bin (see read_trajectory); call before init."""
        check(self.dcx.ctx._lib.gd_remc_set_trajectory(self.h, os.fsencode(directory),
                                                       os.fsencode(stem)),
              "gd_remc_set_trajectory")

    def kernel_times(self):
        """(MC-interval ms, launches, exchange ms, launches) since the last call."""
        a, b = C.c_double(), C.c_double()
        na, nb = C.c_int(), C.c_int()
        check(self.dcx.ctx._lib.gd_remc_kernel_times(self.h, C.byref(a), C.byref(na), C.byref(b),
                                                     C.byref(nb)), "gd_remc_kernel_times")
        return a.value, na.value, b.value, nb.value

    def snapshot(self) -> bytes:
        """The run's state as bytes (gd_remc_snapshot): replica state, counters, step."""
        lib = self.dcx.ctx._lib
        n = C.c_size_t()
        check(lib.gd_remc_snapshot(self.h, None, 0, C.byref(n)), "gd_remc_snapshot")
        buf = C.create_string_buffer(n.value)
        check(lib.gd_remc_snapshot(self.h, buf, n.value, C.byref(n)), "gd_remc_snapshot")
        return buf.raw

    def restore(self, blob: bytes):
        """Loads a snapshot of a run of the same shape (gd_remc_restore)."""
        buf = C.create_string_buffer(bytes(blob), len(blob))
        check(self.dcx.ctx._lib.gd_remc_restore(self.h, buf, len(blob)), "gd_remc_restore")

    def read(self) -> abi.McLogBuffers:
        buf = abi.McLogBuffers(self.n_rep, self.n_tmp, self.steps_total, self.record)
        check(self.dcx.ctx._lib.gd_remc_read(self.h, C.byref(buf.log)), "gd_remc_read")
        return buf

    def close(self):
        if self.h:
            self.dcx.ctx._lib.gd_remc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many complexes advanced together (gd_batch): the batched form."""

    def __init__(self, ctx: Context, dcxs, params):
        self.ctx = ctx
        self.dcxs = list(dcxs)
        self.params = [p for p, _ in params]
        self._keep = [k for _, k in params]
        n = len(self.dcxs)
        arr = (C.c_void_p * n)(*[d.h.value for d in self.dcxs])
        parr = (abi.GdMcParams * n)(*self.params)
        h = C.c_void_p()
        check(ctx._lib.gd_batch_create(ctx.h, n, C.cast(arr, C.POINTER(C.c_void_p)), parr,
                                       C.byref(h)), "gd_batch_create")
        self.h = h
        self.n_rep = int(ctx._lib.gd_batch_n_rep(h))
        self.n_shapes = int(ctx._lib.gd_batch_n_launch_shapes(h))

    def init(self):
        check(self.ctx._lib.gd_batch_init(self.h), "gd_batch_init")

    def run(self, n_steps: int):
        check(self.ctx._lib.gd_batch_run(self.h, int(n_steps)), "gd_batch_run")

    def read(self, i: int) -> abi.McLogBuffers:
        p = self.params[i]
        n_rep = self._n_rep_of(i)
        buf = abi.McLogBuffers(n_rep, p.n_tmp, p.steps_total, bool(p.flags & abi.MC_RECORD))
        check(self.ctx._lib.gd_batch_read(self.h, i, C.byref(buf.log)), "gd_batch_read")
        return buf

    def snapshot(self) -> bytes:
        """The run's state as bytes (gd_batch_snapshot): replica state, counters, step."""
        lib = self.ctx._lib
        n = C.c_size_t()
        check(lib.gd_batch_snapshot(self.h, None, 0, C.byref(n)), "gd_batch_snapshot")
        buf = C.create_string_buffer(n.value)
        check(lib.gd_batch_snapshot(self.h, buf, n.value, C.byref(n)), "gd_batch_snapshot")
        return buf.raw

    def restore(self, blob: bytes):
        """Loads a snapshot of a run of the same shape (gd_batch_restore)."""
        buf = C.create_string_buffer(bytes(blob), len(blob))
        check(self.ctx._lib.gd_batch_restore(self.h, buf, len(blob)), "gd_batch_restore")

    def _n_rep_of(self, i):
        d = self.dcxs[i]
        return d.n_prt_view * d.cx.n_lig * self.params[i].n_tmp

    def set_profiling(self, on: bool = True):
        check(self.ctx._lib.gd_batch_set_profiling(self.h, int(on)), "gd_batch_set_profiling")

    def kernel_times(self):
        a, b = C.c_double(), C.c_double()
        na, nb = C.c_int(), C.c_int()
        check(self.ctx._lib.gd_batch_kernel_times(self.h, C.byref(a), C.byref(na), C.byref(b),
                                                  C.byref(nb)), "gd_batch_kernel_times")
        return a.value, na.value, b.value, nb.value

    def close(self):
        if self.h:
            self.ctx._lib.gd_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """The serving form (gd_server): resident proteins, a request queue with
    HBM-budget admission and continuous batching on a scheduler thread."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 120 << 30, max_active: int = 0,
                 steps_per_launch: int = 10):
        self._lib = load()
        h = C.c_void_p()
        check(self._lib.gd_server_create(device, int(hbm_budget_bytes), int(max_active),
                                         int(steps_per_launch), C.byref(h)), "gd_server_create")
        self.h = h
        self._pending = {}  # request id -> (McLogBuffers, complex, params, keep-alive)

    def add_protein(self, cx: abi.Complex) -> int:
        pid = C.c_int()
        check(self._lib.gd_server_add_protein(self.h, C.byref(cx.struct()), C.byref(pid)),
              "gd_server_add_protein")
        return pid.value

    def submit(self, protein_id: int, cx: abi.Complex, steps_total: int, steps_per_exchange: int,
               minus_beta, n_prt: int, **kw) -> int:
        params, mb = abi.mc_params(steps_total, steps_per_exchange, minus_beta, **kw)
        rid = C.c_uint64()
        check(self._lib.gd_server_submit(self.h, protein_id, C.byref(cx.struct()),
                                         C.byref(params), C.byref(rid)), "gd_server_submit")
        n_rep = n_prt * cx.n_lig * len(mb)
        record = bool(params.flags & abi.MC_RECORD)
        self._pending[rid.value] = abi.McLogBuffers(n_rep, len(mb), steps_total, record)
        return rid.value

    def poll(self, rid: int):
        """None while running; the results when done (raises on failure)."""
        buf = self._pending[rid]
        st = self._lib.gd_server_poll(self.h, C.c_uint64(rid), C.byref(buf.log))
        if st == abi.GD_EAGAIN:
            return None
        del self._pending[rid]
        check(st, "gd_server_poll")
        return buf

    def wait(self, rid: int, timeout_ms: int = 600000):
        buf = self._pending[rid]
        st = self._lib.gd_server_wait(self.h, C.c_uint64(rid), int(timeout_ms), C.byref(buf.log))
        if st != abi.GD_ETIMEDOUT:
            del self._pending[rid]
        check(st, "gd_server_wait")
        return buf

    def cancel(self, rid: int):
        check(self._lib.gd_server_cancel(self.h, C.c_uint64(rid)), "gd_server_cancel")

    def set_alloc_fail(self, nth: int):
        """Test hook on the server's context (gd_ctx_set_alloc_fail)."""
        check(self._lib.gd_ctx_set_alloc_fail(self._lib.gd_server_context(self.h), int(nth)),
              "gd_ctx_set_alloc_fail")

    def set_split(self, split: int):
        """CTAs per request unit for requests admitted from now on (0: the
        server's rule), through the server's own context."""
        check(self._lib.gd_ctx_set_split(self._lib.gd_server_context(self.h), split),
              "gd_ctx_set_split")

    def stats(self) -> abi.GdServerStats:
        s = abi.GdServerStats()
        check(self._lib.gd_server_get_stats(self.h, C.byref(s)), "gd_server_get_stats")
        return s

    def close(self):
        if self.h:
            self._lib.gd_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run(cx: abi.Complex, steps_total: int, steps_per_exchange: int, minus_beta, **kw):
    """gd_run: the one-call counterpart of the reference's Run()."""
    params, mb = abi.mc_params(steps_total, steps_per_exchange, minus_beta, **kw)
    n_rep = cx.n_prt * cx.n_lig * len(mb)
    buf = abi.McLogBuffers(n_rep, len(mb), steps_total, bool(params.flags & abi.MC_RECORD))
    check(load().gd_run(C.byref(cx.struct()), C.byref(params), C.byref(buf.log)), "gd_run")
    return buf


def lna_bucket(lna: int) -> int:
    """Ligand-size bucket of the launch-shape cache (lna rounded up to 8)."""
    return min(((lna + 7) // 8) * 8, 128)


def autotune_buckets(dcxs):
    """Autotunes one launch shape per size class of a batch: the largest
    ligand of each (bucket, protein tiles) class is timed and its shape is
    kept in the context for every ligand of the class.
    Returns {size_class: ((A, P, NA), ms)}."""
    rep = {}
    for d in dcxs:
        k = d.size_class
        if k not in rep or d.cx.lna > rep[k].cx.lna:
            rep[k] = d
    return {k: d.autotune() for k, d in sorted(rep.items())}


def autotune_cadence(ctx: Context, dcxs, minus_beta, candidates=(1, 2, 4, 5, 10, 20, 50),
                     tol: float = 0.02, steps: int = 100, **kw):
    """Exchange-cadence autotuner for a batch.

    Exchanging more often mixes the temperature ladder faster but costs a
    kernel boundary per interval where the exchange cannot run inside the
    MC kernel.  Each candidate steps_per_exchange is timed on the batch
    (about `steps` MC steps after a warm-up); the smallest cadence whose time
    per MC step is within `tol` of the fastest candidate is returned with the
    table {spe: ms per MC step}.  The cadence changes the sampled trajectory,
    so the caller decides whether to adopt it."""
    table = {}
    for spe in candidates:
        n = max(spe, (steps // spe) * spe)
        params = [abi.mc_params(3 * n, spe, minus_beta, stream_id=i, **kw)
                  for i in range(len(dcxs))]
        b = Batch(ctx, dcxs, params)
        b.init()
        b.run(n)
        ctx.sync()
        t0 = time.perf_counter()
        b.run(n)
        ctx.sync()
        table[spe] = (time.perf_counter() - t0) * 1e3 / n
        b.close()
    best = min(table.values())
    chosen = min(s for s, t in table.items() if t <= best * (1.0 + tol))
    return chosen, table


def fma_peak(ctx: Context, n_blocks: int = 148 * 16, iters: int = 4096):
    ms = C.c_float()
    fl = C.c_double()
    check(ctx._lib.gd_fma_peak(ctx.h, n_blocks, iters, C.byref(ms), C.byref(fl)), "gd_fma_peak")
    return fl.value / (ms.value * 1e-3)


def schedule_pieces(cost, steps, machines: int):
    """The persistent schedule of units with per-step `cost` and `steps` MC
    steps over `machines` CTAs: (pieces [n][4] = unit, first step, end step,
    wait; piece_off [used + 1]), pieces of CTA m at piece_off[m]:piece_off[m+1]
    in run order."""
    lib = load()
    cost = np.ascontiguousarray(cost, np.float64)
    steps = np.ascontiguousarray(steps, np.int32)
    n = len(cost)
    cap = 2 * n + machines + 1
    pieces = np.zeros((cap, 4), np.int32)
    off = np.zeros(machines + 1, np.int32)
    used = C.c_int(0)
    check(lib.gd_schedule_pieces(cost.ctypes.data_as(C.POINTER(C.c_double)),
                                 steps.ctypes.data_as(C.POINTER(C.c_int)), n, machines,
                                 pieces.ctypes.data_as(C.POINTER(C.c_int)), cap,
                                 off.ctypes.data_as(C.POINTER(C.c_int)), C.byref(used)),
          "gd_schedule_pieces")
    u = used.value
    return pieces[:off[u]].copy(), off[:u + 1].copy()


def schedule_queue(cost, steps, machines: int, tail: int):
    """The persistent schedule with a shared queue: (pieces [n][4], piece_off
    [machines + 1], n_queue); the queue is the last n_queue pieces."""
    lib = load()
    cost = np.ascontiguousarray(cost, np.float64)
    steps = np.ascontiguousarray(steps, np.int32)
    n = len(cost)
    cap = 2 * n + machines + 1 + n * tail
    pieces = np.zeros((cap, 4), np.int32)
    off = np.zeros(machines + 1, np.int32)
    nq = C.c_int(0)
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
    check(lib.gd_schedule_queue(cost.ctypes.data_as(C.POINTER(C.c_double)), ip(steps), n,
                                machines, tail, ip(pieces), cap, ip(off), C.byref(nq)),
          "gd_schedule_queue")
    return pieces[:off[machines] + nq.value].copy(), off, nq.value


def trajectory_dtype(layout: dict) -> np.dtype:
    """numpy structured dtype of one LigRecordSingleStep from a layout file."""
    rec = layout["record"]
    names, formats, offsets = [], [], []
    for f in rec["fields"]:
        base = {"int32": "<i4", "float32": "<f4"}[f["type"]]
        names.append(f["name"])
        formats.append((base, tuple(f["shape"])) if "shape" in f else base)
        offsets.append(f["offset"])
    return np.dtype({"names": names, "formats": formats, "offsets": offsets,
                     "itemsize": rec["bytes"]})


def read_trajectory(directory: str, stem: str):
    """The dump files of a trajectory: a list of [n_rep][steps_per_dump]
    structured arrays (fields of LigRecordSingleStep), one per dump."""
    import glob
    import json
    with open(os.path.join(directory, stem + ".layout.json")) as f:
        layout = json.load(f)
    dt = trajectory_dtype(layout)
    n_rep, spd = layout["shape"][0], layout["steps_per_dump"]
    out = []
    for path in sorted(glob.glob(os.path.join(directory, stem + "_[0-9][0-9][0-9][0-9].bin"))):
        out.append(np.fromfile(path, dtype=dt).reshape(n_rep, spd))
    return out


LOAD_PEPTIDE_ALL_MODELS = 0x1


def read_traces(path: str) -> np.ndarray:
    """A trace file of the similarity-matrix tool as read2D reads it
    (SimilarityMatirxGen util.C:211-240): lines that start with a digit, one
    conformation each (protein conf, ligand conf, move vector), numbers read
    as floats until the first that does not parse."""
    libc = C.CDLL(None)
    libc.strtof.restype = C.c_float
    libc.strtof.argtypes = [C.c_char_p, C.POINTER(C.c_char_p)]
    rows = []
    with open(path) as f:
        for line in f:
            if not line[:1].isdigit():
                continue
            row = []
            for tok in line.split():
                buf = C.create_string_buffer(tok.encode())
                end = C.c_char_p()
                v = libc.strtof(buf, C.byref(end))
                used = C.cast(end, C.c_void_p).value - C.addressof(buf)
                if used == 0:
                    break
                row.append(v)
                if used < len(tok):  # a number followed by other characters
                    break
            rows.append(row)
    if not rows:
        return np.zeros((0, 8), np.float32)
    return np.asarray(rows, np.float32)


def save_similarity(path: str, S: np.ndarray) -> None:
    """The similarity-matrix file as SaveSimilarityMatrix writes it
    (SimilarityMatirxGen util.C:128-144): the size, then one row per line,
    values in the stream's default format (6 significant digits)."""
    S = np.asarray(S, np.float32)
    with open(path, "w") as f:
        f.write(f"{S.shape[0]}\n")
        for row in S:
            f.write(" ".join(f"{float(v):g}" for v in row) + "\n")


def load_enepara(ff: str, weights: str | None = None, nor_a: str | None = None,
                 nor_b: str | None = None) -> abi.GdEneparaRaw:
    """The raw force field from the reference's parameter files
    (gd_load_enepara: loadEnePara, loadWeight, loadNorPara)."""
    lib = load()
    raw = abi.GdEneparaRaw()
    enc = (lambda v: None if v is None else os.fsencode(v))
    check(lib.gd_load_enepara(enc(ff), enc(weights), enc(nor_a), enc(nor_b), C.byref(raw)),
          "gd_load_enepara")
    return raw


def load_files(pdb: str, sdf: str, lhm: str, ligand_id: str, molid: str = "MOLID",
               raw: "abi.GdEneparaRaw | None" = None, flags: int = 0) -> abi.Complex:
    """A complex from the reference's input files (gd_load: loadProtein,
    loadLigand, loadLHM and the table derivation linear_dock runs), copied
    into numpy arrays.  raw: force field (default: the packaged one);
    flags: LOAD_PEPTIDE_ALL_MODELS (see gd_load)."""
    from . import forcefield
    lib = load()
    if raw is None:
        raw = forcefield.raw_struct(forcefield.load_raw())
    ff = enepara_optimize(raw)
    h = C.c_void_p()
    check(lib.gd_load(os.fsencode(pdb), os.fsencode(sdf), os.fsencode(lhm),
                      ligand_id.encode(), molid.encode(), C.byref(raw), C.byref(ff),
                      int(flags), C.byref(h)), "gd_load")
    try:
        v = abi.GdComplex()
        check(lib.gd_loaded_complex(h, C.byref(v)), "gd_loaded_complex")

        def arr(ptr, n, dt):
            if not n:
                return np.zeros(0, dt)
            return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt, copy=True)

        def xyz(x, y, z, n, shape):
            return np.stack([arr(x, n, np.float32), arr(y, n, np.float32),
                             arr(z, n, np.float32)], axis=-1).reshape(*shape, 3)

        lg, pr, pk, mc = v.lig, v.prt, v.kde, v.mcs
        lna, nl, pnp, npr, nf = lg.lna, lg.n_conf, pr.pnp, pr.n_conf, mc.n_field
        cx = abi.Complex(
            lig_xyz=xyz(lg.x, lg.y, lg.z, nl * lna, (nl, lna)),
            lig_t=arr(lg.t, lna, np.int32), lig_c=arr(lg.c, lna, np.float32),
            lig_n=arr(lg.n, lna, np.int32), lig_center=np.array(lg.center[:], np.float32),
            prt_xyz=xyz(pr.x, pr.y, pr.z, npr * pnp, (npr, pnp)),
            prt_t=arr(pr.t, pnp, np.int32), prt_c=arr(pr.c, pnp, np.int32),
            prt_ele=arr(pr.ele, pnp, np.float32), prt_seq3r=arr(pr.seq3r, pnp, np.int32),
            prt_hpcflag=arr(pr.c0_and_d12_or_c2, pnp, np.int32),
            prt_hpp=arr(pr.hpp, pnp, np.float32),
            pocket_center=np.array(pr.pocket_center[:], np.float32),
            psp=arr(v.psp.psp, abi.NLT * v.psp.n_col, np.float32).reshape(abi.NLT, v.psp.n_col),
            kde_xyz=xyz(pk.x, pk.y, pk.z, pk.pnk, (pk.pnk,)), kde_t=arr(pk.t, pk.pnk, np.int32),
            mcs_xyz=xyz(mc.x, mc.y, mc.z, mc.pos * nf, (mc.pos, nf)),
            mcs_tcc=arr(mc.tcc, mc.pos, np.float32), ff=ff)
        cx.ligand_id = (lib.gd_loaded_ligand_id(h) or b"").decode()
        return cx
    finally:
        lib.gd_loaded_free(h)
