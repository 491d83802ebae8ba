"""Python binding of libbeam_gpu (include/beam_gpu.h) over ctypes.

The product is the C ABI; this module is the thin host-side mirror used by
the tests, the benchmark and Python callers. It mirrors the reference's
estimator interface -- the five command-line values of
``barbie NN NRi UL_k1 LL_k1 BW_k1`` (barbie.c:58-65) plus the constants the
reference hard-codes (barbie.c:67-84) -- and returns the reference's bin
arrays (barbie.c:87) as numpy arrays of shape [n_k1bin][n_mtbin][n_mtbin][16].

There is no CPU fallback: loading fails loudly when libbeam_gpu.so is missing,
and every call that needs a GPU raises BeamError when none is usable.
"""
from __future__ import annotations

import ctypes
import os
import re
import weakref

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbeam_gpu.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "beam_gpu.h")

NPOLES = 16
PREC = {"fp64": 0, "mixed": 1, "int8": 2}
METHOD = {"triangle": 0, "pixel": 1}

BEAM_OK = 0
BEAM_EINVAL = -1
BEAM_ENOMEM = -2
BEAM_EDEVMEM = -3
BEAM_ECUDA = -4
BEAM_ETIMEDOUT = -5
BEAM_EBUSY = -6
BEAM_EBOUNDS = -7
BEAM_ENODEV = -8
BEAM_ENOTFOUND = -9


class BeamError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        detail = _lib.beam_gpu_last_error_detail().decode() if _lib is not None else ""
        msg = _lib.beam_gpu_strerror(code).decode() if _lib is not None else str(code)
        super().__init__(f"{what}: {msg} ({code}){': ' + detail if detail else ''}")


class Cfg(ctypes.Structure):
    _fields_ = [("NN", ctypes.c_long), ("Nmax", ctypes.c_long), ("Nr", ctypes.c_long),
                ("UL_k1", ctypes.c_int), ("LL_k1", ctypes.c_int), ("BW_k1", ctypes.c_int),
                ("n_mtbin", ctypes.c_int), ("LL", ctypes.c_double),
                ("precision", ctypes.c_int), ("method", ctypes.c_int),
                ("shard_index", ctypes.c_int), ("shard_count", ctypes.c_int)]


class Result(ctypes.Structure):
    _fields_ = [("bs", ctypes.POINTER(ctypes.c_double)), ("norm", ctypes.POINTER(ctypes.c_double)),
                ("out", ctypes.POINTER(ctypes.c_double)), ("count", ctypes.POINTER(ctypes.c_int64)),
                ("ana_sum", ctypes.POINTER(ctypes.c_double)), ("ana", ctypes.POINTER(ctypes.c_double))]


class PlanInfo(ctypes.Structure):
    _fields_ = [("n_k1bin", ctypes.c_int), ("n_bins", ctypes.c_long), ("n_closed_triplets", ctypes.c_long),
                ("n_triples", ctypes.c_long), ("n_used_triplets", ctypes.c_long),
                ("n_fourier_terms", ctypes.c_long), ("n_modes", ctypes.c_long), ("n_planes", ctypes.c_int),
                ("device_bytes", ctypes.c_size_t), ("vol", ctypes.c_double),
                ("n_shard_terms", ctypes.c_long), ("launches_last_run", ctypes.c_int),
                ("run_bytes", ctypes.c_size_t), ("n_run_combos", ctypes.c_long), ("build_ms", ctypes.c_float * 5)]


TUNE_MAX, FIELD_TUNE_MAX = 16, 4


class TuneReport(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("best", ctypes.c_int), ("tau0", ctypes.c_longlong * TUNE_MAX),
                ("balance", ctypes.c_double * TUNE_MAX), ("ms", ctypes.c_float * TUNE_MAX),
                ("items", ctypes.c_int * TUNE_MAX)]


class FieldTuneReport(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("best_cols", ctypes.c_int), ("best_rows", ctypes.c_int),
                ("tile", ctypes.c_int * FIELD_TUNE_MAX), ("cols_ms", ctypes.c_float * FIELD_TUNE_MAX),
                ("rows_ms", ctypes.c_float * FIELD_TUNE_MAX)]


_lib = None


def header_symbols() -> list[str]:
    """Every function the public header declares."""
    with open(HEADER) as fh:
        text = fh.read()
    return sorted(set(re.findall(r"^\s*BEAM_API\s+(?:const\s+)?\w+\s*\*?\s*(beam_\w+)\s*\(", text, flags=re.M)))


def load() -> ctypes.CDLL:
    """Load libbeam_gpu.so (built in-tree by ``make -C barbie_b200``)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C barbie_b200` (no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    vp, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
    L.beam_gpu_strerror.argtypes = [ctypes.c_int]
    L.beam_gpu_strerror.restype = ctypes.c_char_p
    L.beam_gpu_last_error_detail.argtypes = []
    L.beam_gpu_last_error_detail.restype = ctypes.c_char_p
    L.beam_cfg_default.argtypes = [ctypes.POINTER(Cfg), ctypes.c_long, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.beam_cfg_default.restype = None
    L.beam_gpu_init.argtypes = [ctypes.c_int, ctypes.POINTER(vp)]
    L.beam_gpu_destroy.argtypes = [vp]
    L.beam_gpu_destroy.restype = None
    L.beam_gpu_plan_create.argtypes = [vp, ctypes.POINTER(Cfg), ctypes.POINTER(vp)]
    L.beam_gpu_plan_destroy.argtypes = [vp]
    L.beam_gpu_plan_destroy.restype = None
    L.beam_gpu_plan_set_triangle_launch.argtypes = [vp, ctypes.c_int]
    L.beam_gpu_plan_get_info.argtypes = [vp, ctypes.POINTER(PlanInfo)]
    L.beam_gpu_run.argtypes = [vp, vp, ctypes.c_int, ctypes.POINTER(Result)]
    L.beam_gpu_run_batch.argtypes = [vp, ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(Result)]
    L.beam_gpu_run_batch_ex.argtypes = [vp, ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(Result), ctypes.c_int]
    L.beam_shard_assign.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.beam_gpu_closed_rings.argtypes = [vp, dp, ctypes.c_long, ctypes.POINTER(ctypes.c_long)]
    L.beam_gpu_plane_rings.argtypes = [vp, vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int), ctypes.c_int, vp, ctypes.c_int]
    L.beam_gpu_triangle_sums.argtypes = [vp, vp, ctypes.c_int, dp]
    L.beam_gpu_stream.argtypes = [vp]
    L.beam_gpu_stream.restype = vp
    L.beam_gpu_plan_last_timings.argtypes = [vp, ctypes.POINTER(ctypes.c_float), ctypes.c_int]
    L.beam_gpu_plan_last_timings.restype = ctypes.c_int
    for name in ("beam_gpu_init", "beam_gpu_plan_create", "beam_gpu_plan_get_info", "beam_gpu_run",
                 "beam_gpu_run_batch", "beam_gpu_run_batch_ex", "beam_shard_assign", "beam_gpu_closed_rings",
                 "beam_gpu_plane_rings", "beam_gpu_triangle_sums"):
        getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def shard_assign(work, shard_count: int) -> np.ndarray:
    """Owner shard of each work unit (beam_shard_assign; host only, no GPU)."""
    L = load()
    w = np.ascontiguousarray(work, dtype=np.float64)
    owner = np.zeros(max(1, w.size), dtype=np.int32)
    _check(L.beam_shard_assign(w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), w.size, shard_count,
                               owner.ctypes.data_as(ctypes.POINTER(ctypes.c_int))), "beam_shard_assign")
    return owner[: w.size]


def _alloc_result(shape):
    """A Result pointing at fresh numpy bin arrays of the given bin shape, and those arrays:
    bs, norm, out, count, ana_sum (sum Biana*Num*bs) and ana (ana_sum/norm, column 5)."""
    arrays = dict(bs=np.zeros(shape), norm=np.zeros(shape), out=np.zeros(shape),
                  count=np.zeros(shape[:3], dtype=np.int64), ana_sum=np.zeros(shape), ana=np.zeros(shape))
    dp = ctypes.POINTER(ctypes.c_double)
    res = Result(arrays["bs"].ctypes.data_as(dp), arrays["norm"].ctypes.data_as(dp), arrays["out"].ctypes.data_as(dp),
                 arrays["count"].ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), arrays["ana_sum"].ctypes.data_as(dp),
                 arrays["ana"].ctypes.data_as(dp))
    return res, arrays


def _check(rc: int, what: str) -> None:
    if rc != BEAM_OK:
        raise BeamError(rc, what)


def _ptr(a):
    """(address, on_device) of a C-contiguous float64 numpy array or torch tensor."""
    if isinstance(a, np.ndarray):
        if a.dtype != np.float64 or not a.flags.c_contiguous:
            raise TypeError("expected a C-contiguous float64 array")
        return a.ctypes.data, 0
    if hasattr(a, "data_ptr"):  # torch tensor
        import torch
        if a.dtype != torch.float64 or not a.is_contiguous():
            raise TypeError("expected a contiguous float64 tensor")
        return a.data_ptr(), 1 if a.is_cuda else 0
    raise TypeError(f"unsupported buffer type {type(a)}")


class Context:
    """One CUDA device and stream (beam_gpu_init)."""

    def __init__(self, device: int = 0):
        L = load()
        h = ctypes.c_void_p()
        _check(L.beam_gpu_init(device, ctypes.byref(h)), "beam_gpu_init")
        self._h = h
        self.device = device
        self._plans = weakref.WeakSet()

    @property
    def stream(self) -> int:
        """cudaStream_t the library launches on (address)."""
        return _lib.beam_gpu_stream(self._h) or 0

    def field_launches(self) -> int:
        """Kernels the last field generate / ingest call launched."""
        _lib.beam_gpu_field_launches.argtypes = [ctypes.c_void_p]
        _lib.beam_gpu_field_launches.restype = ctypes.c_int
        return int(_lib.beam_gpu_field_launches(self._h))

    def close(self) -> None:
        """Destroy the context; plans made on it are destroyed first."""
        if getattr(self, "_h", None):
            for plan in list(self._plans):
                plan.close()
            _lib.beam_gpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Plan:
    """Estimator plan for one configuration (beam_gpu_plan_create)."""

    def __init__(self, ctx: Context, NN: int, UL_k1: int, LL_k1: int, BW_k1: int, *, Nmax: int = 100,
                 Nr: int = 40, n_mtbin: int = 5, LL: float = 1.0, precision: str = "fp64",
                 method: str = "triangle", shard: tuple[int, int] = (0, 1)):
        L = load()
        cfg = Cfg()
        L.beam_cfg_default(ctypes.byref(cfg), NN, UL_k1, LL_k1, BW_k1)
        cfg.Nmax, cfg.Nr, cfg.n_mtbin, cfg.LL = Nmax, Nr, n_mtbin, LL
        cfg.precision, cfg.method = PREC[precision], METHOD[method]
        cfg.shard_index, cfg.shard_count = shard
        h = ctypes.c_void_p()
        _check(L.beam_gpu_plan_create(ctx._h, ctypes.byref(cfg), ctypes.byref(h)), "beam_gpu_plan_create")
        self._h, self.ctx, self.cfg = h, ctx, cfg
        ctx._plans.add(self)
        info = PlanInfo()
        _check(L.beam_gpu_plan_get_info(h, ctypes.byref(info)), "beam_gpu_plan_get_info")
        self.info = {k: (list(getattr(info, k)) if k == "build_ms" else getattr(info, k)) for k, _ in PlanInfo._fields_}
        self.n_k1bin = info.n_k1bin
        self.shape = (info.n_k1bin, n_mtbin, n_mtbin, NPOLES)
        self.NN = NN
        self.precision = precision

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.beam_gpu_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _result(self):
        return _alloc_result(self.shape)

    def run(self, r2c) -> dict:
        """One bispectrum of an r2c buffer (numpy host array or torch CUDA tensor)."""
        addr, dev = _ptr(r2c)
        self._check_size(r2c)
        res, arrays = self._result()
        _check(_lib.beam_gpu_run(self._h, addr, dev, ctypes.byref(res)), "beam_gpu_run")
        return arrays

    def run_batch(self, fields: list, batch: int = 0) -> list[dict]:
        """Several realizations (host numpy arrays) through beam_gpu_run_batch_ex
        (batch = realizations per device batch, 0 = chosen by the library)."""
        addrs = (ctypes.c_void_p * len(fields))()
        results = (Result * len(fields))()
        out = []
        for k, f in enumerate(fields):
            a, dev = _ptr(f)
            if dev:
                raise TypeError("run_batch takes host arrays")
            self._check_size(f)
            addrs[k] = a
            results[k], arrays = self._result()
            out.append(arrays)
        _check(_lib.beam_gpu_run_batch_ex(self._h, addrs, len(fields), results, batch), "beam_gpu_run_batch_ex")
        return out

    def set_triangle_launch(self, mode: str) -> None:
        """'classes' (one launch per tile class, the default) or 'persistent' (one launch for all)."""
        m = {"classes": 0, "persistent": 1}[mode]
        _check(_lib.beam_gpu_plan_set_triangle_launch(self._h, m), "beam_gpu_plan_set_triangle_launch")

    def refresh_info(self) -> dict:
        """Re-read beam_gpu_plan_get_info (device bytes and launch count change as the plan runs)."""
        info = PlanInfo()
        _check(_lib.beam_gpu_plan_get_info(self._h, ctypes.byref(info)), "beam_gpu_plan_get_info")
        self.info = {k: (list(getattr(info, k)) if k == "build_ms" else getattr(info, k)) for k, _ in PlanInfo._fields_}
        return self.info

    def triangle_sums(self, r2c) -> np.ndarray:
        """B per accepted triangle in the reference's loop order."""
        addr, dev = _ptr(r2c)
        self._check_size(r2c)
        B = np.zeros(max(1, self.info["n_triples"]))
        _check(_lib.beam_gpu_triangle_sums(self._h, addr, dev, B.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
               "beam_gpu_triangle_sums")
        return B[: self.info["n_triples"]]

    def closed_rings(self) -> np.ndarray:
        """calCR records {r1, r2, r3, Num = NN^2 * count}."""
        n = ctypes.c_long(0)
        cap = self.info["n_closed_triplets"]
        out = np.zeros((max(cap, 1), 4))
        _check(_lib.beam_gpu_closed_rings(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), cap,
                                          ctypes.byref(n)), "beam_gpu_closed_rings")
        return out[: n.value]

    def plane_rings(self, r2c, planes, rings) -> np.ndarray:
        """Df transforms -> complex128[n][NN][NN] (host)."""
        addr, dev = _ptr(r2c)
        self._check_size(r2c)
        planes = np.ascontiguousarray(planes, dtype=np.int32)
        rings = np.ascontiguousarray(rings, dtype=np.int32)
        n = len(planes)
        out = np.zeros((n, self.NN, self.NN), dtype=np.complex128)
        ip = ctypes.POINTER(ctypes.c_int)
        _check(_lib.beam_gpu_plane_rings(self._h, addr, dev, planes.ctypes.data_as(ip), rings.ctypes.data_as(ip),
                                         n, out.ctypes.data, 0), "beam_gpu_plane_rings")
        return out

    def autotune(self, reps: int = 3) -> dict:
        """Choose the triangle sums' work decomposition by timing (beam_gpu_plan_autotune).

        Returns the candidates (tau0, balance, ms, items) and the kept one."""
        _lib.beam_gpu_plan_autotune.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(TuneReport)]
        _lib.beam_gpu_plan_autotune.restype = ctypes.c_int
        rep = TuneReport()
        _check(_lib.beam_gpu_plan_autotune(self._h, reps, ctypes.byref(rep)), "beam_gpu_plan_autotune")
        self.refresh_info()
        cands = [dict(tau0=rep.tau0[k], balance=rep.balance[k], ms=rep.ms[k], items=rep.items[k])
                 for k in range(rep.n)]
        return dict(candidates=cands, best=cands[rep.best])

    def last_timings(self) -> dict:
        """Device milliseconds of the stages of the last run (CUDA events)."""
        ms = (ctypes.c_float * 4)()
        _check(_lib.beam_gpu_plan_last_timings(self._h, ms, 4), "beam_gpu_plan_last_timings")
        return dict(upload=ms[0], triangle=ms[1], reduce=ms[2], epilogue=ms[3])

    def _check_size(self, r2c) -> None:
        NN = self.NN
        if tuple(r2c.shape) not in ((NN, NN, NN + 2), (NN * NN * (NN + 2),)):
            raise ValueError(f"r2c buffer must be [{NN}][{NN}][{NN + 2}] float64")


PK_COLUMNS = ("k", "P0", "P2", "P4", "P6", "count")


def power_multipoles(ctx: "Context", r2c, NN: int, LL: float = 0.56, Nbin: int = 10) -> dict:
    """Power spectrum multipoles of an r2c buffer (beam_gpu_power_multipoles, the
    reference's calpow_mom): arrays k, P0, P2, P4, P6, count over Nbin log bins."""
    L = load()
    L.beam_gpu_power_multipoles.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_double, ctypes.c_int,
                                            ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.beam_gpu_power_multipoles.restype = ctypes.c_int
    addr, dev = _ptr(r2c)
    if tuple(r2c.shape) not in ((NN, NN, NN + 2), (NN * NN * (NN + 2),)):
        raise ValueError(f"r2c buffer must be [{NN}][{NN}][{NN + 2}] float64")
    out = np.zeros(6 * Nbin)
    _check(L.beam_gpu_power_multipoles(ctx._h, NN, LL, Nbin, addr, dev,
                                       out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
           "beam_gpu_power_multipoles")
    return dict(zip(PK_COLUMNS, out.reshape(6, Nbin)))


def field_autotune(ctx: "Context", NN: int) -> dict:
    """Choose the field FFT staging tiles for NN by timing (beam_gpu_field_autotune)."""
    L = load()
    L.beam_gpu_field_autotune.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.POINTER(FieldTuneReport)]
    L.beam_gpu_field_autotune.restype = ctypes.c_int
    rep = FieldTuneReport()
    _check(L.beam_gpu_field_autotune(ctx._h, NN, ctypes.byref(rep)), "beam_gpu_field_autotune")
    cands = [dict(tile=rep.tile[k], cols_ms=rep.cols_ms[k], rows_ms=rep.rows_ms[k]) for k in range(rep.n)]
    return dict(candidates=cands, cols_tile=rep.tile[rep.best_cols], rows_tile=rep.tile[rep.best_rows])


def field_seed(NRi: int) -> int:
    """The reference generator's seed for realization NRi (generate_field.c:49)."""
    return 100020 + 146 * NRi


def _field_out(NN: int, out):
    if out is None:
        out = np.empty((NN, NN, NN + 2))
    if tuple(out.shape) not in ((NN, NN, NN + 2), (NN * NN * (NN + 2),)):
        raise ValueError(f"r2c buffer must be [{NN}][{NN}][{NN + 2}] float64")
    return out


def generate_field(ctx: "Context", NN: int, seed: int, LL: float = 0.56, ff: float = 0.5, beta: float = 1.0,
                   out=None):
    """The reference's field generator on the device (beam_gpu_field_generate).

    Returns (r2c, sigma): r2c is ``out`` (a float64 numpy array or CUDA tensor of
    shape [NN][NN][NN+2]) or a new numpy array; sigma the Gaussian image's rms.
    A device ``out`` stays on the device, ready for Plan.run."""
    L = load()
    L.beam_gpu_field_generate.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_ulonglong, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_void_p, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_double)]
    L.beam_gpu_field_generate.restype = ctypes.c_int
    out = _field_out(NN, out)
    addr, dev = _ptr(out)
    sigma = ctypes.c_double()
    _check(L.beam_gpu_field_generate(ctx._h, NN, seed, LL, ff, beta, addr, dev, ctypes.byref(sigma)),
           "beam_gpu_field_generate")
    return out, sigma.value


def ingest_field(ctx: "Context", cube, LL: float = 0.56, beta: float = 1.0, out=None):
    """A real-space cube [NN][NN][NN] (numpy or CUDA tensor, float64) to the r2c
    buffer on the device (beam_gpu_field_ingest): x LL^3, 3D r2c, RSD(beta)."""
    L = load()
    L.beam_gpu_field_ingest.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
    L.beam_gpu_field_ingest.restype = ctypes.c_int
    NN = int(cube.shape[0])
    if tuple(cube.shape) != (NN, NN, NN):
        raise ValueError("cube must be [NN][NN][NN]")
    src, src_dev = _ptr(cube)
    out = _field_out(NN, out)
    addr, dev = _ptr(out)
    _check(L.beam_gpu_field_ingest(ctx._h, NN, LL, beta, src, src_dev, addr, dev), "beam_gpu_field_ingest")
    return out


class ServerCfg(ctypes.Structure):
    _fields_ = [("mem_budget", ctypes.c_size_t), ("max_active", ctypes.c_int), ("max_plans", ctypes.c_int)]


class JobInfo(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int), ("error", ctypes.c_int), ("n_k1bin", ctypes.c_int), ("n_mtbin", ctypes.c_int),
                ("n_bins", ctypes.c_long), ("queue_ms", ctypes.c_double), ("run_ms", ctypes.c_double),
                ("total_ms", ctypes.c_double)]


JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED = 0, 1, 2, 3


def _server_protos(L) -> None:
    if getattr(L, "_server_protos", False):
        return
    vp = ctypes.c_void_p
    L.beam_server_cfg_default.argtypes = [ctypes.POINTER(ServerCfg)]
    L.beam_server_cfg_default.restype = None
    L.beam_gpu_server_create.argtypes = [vp, ctypes.POINTER(ServerCfg), ctypes.POINTER(vp)]
    L.beam_gpu_server_destroy.argtypes = [vp]
    L.beam_gpu_server_destroy.restype = None
    L.beam_gpu_server_submit.argtypes = [vp, ctypes.POINTER(Cfg), vp, ctypes.POINTER(ctypes.c_int64)]
    L.beam_gpu_server_wait.argtypes = [vp, ctypes.c_int64, ctypes.c_int, ctypes.POINTER(JobInfo)]
    L.beam_gpu_server_take.argtypes = [vp, ctypes.c_int64, ctypes.POINTER(Result)]
    L.beam_gpu_server_memory.argtypes = [vp, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]
    for name in ("beam_gpu_server_create", "beam_gpu_server_submit", "beam_gpu_server_wait", "beam_gpu_server_take",
                 "beam_gpu_server_memory"):
        getattr(L, name).restype = ctypes.c_int
    L._server_protos = True


class Server:
    """Job server on a context (beam_gpu_server_*): submit realizations of any
    configuration as they arrive; they run concurrently on the device."""

    def __init__(self, ctx: Context, mem_budget: int = 0, max_active: int = 0, max_plans: int = 0):
        L = load()
        _server_protos(L)
        cfg = ServerCfg()
        L.beam_server_cfg_default(ctypes.byref(cfg))
        if mem_budget:
            cfg.mem_budget = mem_budget
        if max_active:
            cfg.max_active = max_active
        if max_plans:
            cfg.max_plans = max_plans
        h = ctypes.c_void_p()
        _check(L.beam_gpu_server_create(ctx._h, ctypes.byref(cfg), ctypes.byref(h)), "beam_gpu_server_create")
        self._h, self.ctx = h, ctx
        self._held = {}  # job -> r2c buffer, kept alive until the job is taken
        ctx._plans.add(self)  # closed with the context, like plans

    def submit(self, r2c, NN: int, UL_k1: int, LL_k1: int, BW_k1: int, *, Nmax: int = 100, Nr: int = 40,
               n_mtbin: int = 5, LL: float = 1.0, precision: str = "fp64") -> int:
        addr, dev = _ptr(r2c)
        if dev:
            raise TypeError("server jobs take host arrays")
        if tuple(r2c.shape) not in ((NN, NN, NN + 2), (NN * NN * (NN + 2),)):
            raise ValueError(f"r2c buffer must be [{NN}][{NN}][{NN + 2}] float64")
        cfg = Cfg()
        _lib.beam_cfg_default(ctypes.byref(cfg), NN, UL_k1, LL_k1, BW_k1)
        cfg.Nmax, cfg.Nr, cfg.n_mtbin, cfg.LL, cfg.precision = Nmax, Nr, n_mtbin, LL, PREC[precision]
        job = ctypes.c_int64()
        _check(_lib.beam_gpu_server_submit(self._h, ctypes.byref(cfg), addr, ctypes.byref(job)), "beam_gpu_server_submit")
        self._held[job.value] = r2c
        return job.value

    def wait(self, job: int, timeout_ms: int = -1) -> dict | None:
        """Job info once it has ended (None if still queued/running at the timeout)."""
        info = JobInfo()
        rc = _lib.beam_gpu_server_wait(self._h, job, timeout_ms, ctypes.byref(info))
        if rc == BEAM_EBUSY:
            return None
        _check(rc, "beam_gpu_server_wait")
        return {k: getattr(info, k) for k, _ in JobInfo._fields_}

    def take(self, job: int) -> dict:
        """Bins of an ended job (raises BeamError for a failed one); forgets the job."""
        info = self.wait(job, 0)
        if info is None:
            raise BeamError(BEAM_EBUSY, "beam_gpu_server_take")
        shape = (info["n_k1bin"], info["n_mtbin"], info["n_mtbin"], NPOLES)
        res, arrays = _alloc_result(shape)
        rc = _lib.beam_gpu_server_take(self._h, job, ctypes.byref(res))
        self._held.pop(job, None)
        _check(rc, "beam_gpu_server_take")
        return dict(arrays, info=info)

    def memory(self) -> tuple[int, int]:
        now, peak = ctypes.c_size_t(), ctypes.c_size_t()
        _check(_lib.beam_gpu_server_memory(self._h, ctypes.byref(now), ctypes.byref(peak)), "beam_gpu_server_memory")
        return now.value, peak.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.beam_gpu_server_destroy(self._h)
            self._h = None
            self._held.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
