"""ctypes binding of the oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py``, to compare against or to time. The GPU
product path never imports this module.

Each wrapper names the reference lines (barbie.c / funcs.c of
sukhdeepsinghgill/BARBIE) its C function restates.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "barbie_ref")

_lib = None

NPOLES = 16


class OrcTriple(ctypes.Structure):
    _fields_ = [
        ("p1", ctypes.c_int32), ("r1", ctypes.c_int32),
        ("p2", ctypes.c_int32), ("r2", ctypes.c_int32),
        ("p3", ctypes.c_int32), ("r3", ctypes.c_int32),
        ("rp", ctypes.c_int32),
        ("k1_bin", ctypes.c_int32), ("t_bin", ctypes.c_int32), ("mu_bin", ctypes.c_int32),
        ("K1", ctypes.c_double), ("T", ctypes.c_double), ("MU", ctypes.c_double),
        ("px", ctypes.c_double), ("pz", ctypes.c_double), ("num", ctypes.c_double),
        ("leg_k", ctypes.c_double * 3), ("leg_p", ctypes.c_double * 3),
    ]


TRIPLE_DTYPE = np.dtype([
    ("p1", "<i4"), ("r1", "<i4"), ("p2", "<i4"), ("r2", "<i4"), ("p3", "<i4"), ("r3", "<i4"),
    ("rp", "<i4"), ("k1_bin", "<i4"), ("t_bin", "<i4"), ("mu_bin", "<i4"),
    ("K1", "<f8"), ("T", "<f8"), ("MU", "<f8"), ("px", "<f8"), ("pz", "<f8"), ("num", "<f8"),
    ("leg_k", "<f8", (3,)), ("leg_p", "<f8", (3,)),
])
assert TRIPLE_DTYPE.itemsize == ctypes.sizeof(OrcTriple)


def build() -> None:
    """Compile liboracle.so (and oracle/_ref/barbie_ref where the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        L.orc_ring_edges.argtypes = [ctypes.c_long, ctypes.c_long, dp, dp, dp]
        L.orc_ring_edges.restype = ctypes.c_int
        L.orc_ring_masks.argtypes = [ctypes.c_long, ctypes.c_long, dp, dp, dp]
        L.orc_closed_rings.argtypes = [ctypes.c_long, ctypes.c_long, dp, dp, dp, dp, ctypes.c_long]
        L.orc_closed_rings.restype = ctypes.c_long
        L.orc_triangle_count_direct.argtypes = [ctypes.c_long, dp, ctypes.c_long, ctypes.c_long, ctypes.c_long]
        L.orc_triangle_count_direct.restype = ctypes.c_int64
        L.orc_plane_ring.argtypes = [ctypes.c_long, ctypes.c_long, ctypes.c_long, dp, dp, dp]
        L.orc_cal_coeff.argtypes = [ctypes.c_double, ctypes.c_double, dp, dp]
        L.orc_enumerate.argtypes = [ctypes.c_long, ctypes.c_long, ctypes.c_long, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int, dp, dp, ctypes.c_long,
                                    ctypes.c_void_p, ctypes.c_long, ctypes.POINTER(ctypes.c_long)]
        L.orc_enumerate.restype = ctypes.c_long
        L.orc_estimate.argtypes = [ctypes.c_long, ctypes.c_long, ctypes.c_long, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_double, dp, dp, dp, dp,
                                   ctypes.POINTER(ctypes.c_int64), dp, ctypes.c_long, ctypes.c_int, dp]
        L.orc_estimate.restype = ctypes.c_int
        L.orc_estimate_ex.argtypes = L.orc_estimate.argtypes + [ctypes.c_int]
        L.orc_estimate_ex.restype = ctypes.c_int
        L.orc_biana.argtypes = [ctypes.c_long, ctypes.c_double, dp, dp]
        L.orc_biana.restype = ctypes.c_double
        L.orc_biana_all.argtypes = [ctypes.c_long, ctypes.c_double, ctypes.c_void_p, ctypes.c_long, dp]
        L.orc_biana_all.restype = None
        L.orc_triple_product.argtypes = [ctypes.c_long, dp, dp, dp, ctypes.c_int, ctypes.c_int]
        L.orc_triple_product.restype = ctypes.c_double
        L.orc_fft2d.argtypes = [ctypes.c_long, ctypes.c_long, ctypes.c_int, dp]
        L.orc_r2c_3d.argtypes = [ctypes.c_long, ctypes.c_long, ctypes.c_long, dp]
        L.orc_c2r_3d.argtypes = [ctypes.c_long, ctypes.c_long, ctypes.c_long, dp]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def ring_edges(Nr: int, Nmax: int):
    """barbie.c:110-130 -> (low, high, avg)."""
    low, high, avg = (np.zeros(Nr) for _ in range(3))
    if lib().orc_ring_edges(Nr, Nmax, _dp(low), _dp(high), _dp(avg)) != 0:
        raise ValueError("Nr must be a positive multiple of 10")
    return low, high, avg


def ring_masks(NN: int, Nr: int, Nmax: int) -> np.ndarray:
    """barbie.c:135-148 -> RR[Nr][NN][NN]."""
    low, high, _ = ring_edges(Nr, Nmax)
    RR = np.zeros((Nr, NN, NN))
    lib().orc_ring_masks(NN, Nr, _dp(low), _dp(high), _dp(RR))
    return RR


def closed_rings(NN: int, Nr: int, Nmax: int) -> np.ndarray:
    """funcs.c:328-424 (calCR) -> rings4[rcount][4] = {r1, r2, r3, Num}."""
    low, high, avg = ring_edges(Nr, Nmax)
    cap = Nr * Nr * Nr
    out = np.zeros((cap, 4))
    n = lib().orc_closed_rings(NN, Nr, _dp(low), _dp(high), _dp(avg), _dp(out), cap)
    if n < 0:
        raise MemoryError("orc_closed_rings failed")
    return out[:n].copy()


def triangle_count_direct(NN: int, RR: np.ndarray, r1: int, r2: int, r3: int) -> int:
    return int(lib().orc_triangle_count_direct(NN, _dp(np.ascontiguousarray(RR)), r1, r2, r3))


def plane_ring(NN: int, p: int, r: int, r2c: np.ndarray, RR: np.ndarray) -> np.ndarray:
    """funcs.c:88-109 (Df, sign=+1) -> complex128[NN][NN]."""
    out = np.zeros((NN, NN, 2))
    lib().orc_plane_ring(NN, p, r, _dp(np.ascontiguousarray(r2c)), _dp(np.ascontiguousarray(RR)), _dp(out))
    return out.view(np.complex128)[..., 0]


def cal_coeff(px: float, pz: float):
    """funcs.c:708-745 -> (bs[16], norm[16])."""
    bs, nm = np.zeros(NPOLES), np.zeros(NPOLES)
    lib().orc_cal_coeff(px, pz, _dp(bs), _dp(nm))
    return bs, nm


def enumerate_triples(NN, Nmax, Nr, UL_k1, LL_k1, BW_k1, n_mtbin=5, rings4=None):
    """barbie.c:247-298 -> (structured array of accepted triangles, loop iterations)."""
    _, _, avg = ring_edges(Nr, Nmax)
    if rings4 is None:
        rings4 = closed_rings(NN, Nr, Nmax)
    rings4 = np.ascontiguousarray(rings4, dtype=np.float64)
    iters = ctypes.c_long(0)
    n = lib().orc_enumerate(NN, Nmax, Nr, UL_k1, LL_k1, BW_k1, n_mtbin, _dp(avg), _dp(rings4),
                            len(rings4), None, 0, ctypes.byref(iters))
    out = np.zeros(n, dtype=TRIPLE_DTYPE)
    lib().orc_enumerate(NN, Nmax, Nr, UL_k1, LL_k1, BW_k1, n_mtbin, _dp(avg), _dp(rings4),
                        len(rings4), out.ctypes.data_as(ctypes.c_void_p), n, None)
    return out, int(iters.value)


def power_multipoles(r2c: np.ndarray, NN: int, LL: float = 0.56, Nbin: int = 10) -> dict:
    """funcs.c:860-1074 (calpow_mom) -> arrays k, P0, P2, P4, P6, count over Nbin bins."""
    L = lib()
    L.orc_power_multipoles.argtypes = [ctypes.c_long, ctypes.c_double, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    L.orc_power_multipoles.restype = ctypes.c_int
    out = np.zeros(6 * Nbin)
    if L.orc_power_multipoles(NN, LL, Nbin, _dp(np.ascontiguousarray(r2c, dtype=np.float64)), _dp(out)) != 0:
        raise ValueError("orc_power_multipoles: invalid arguments")
    return dict(zip(("k", "P0", "P2", "P4", "P6", "count"), out.reshape(6, Nbin)))


def field_seed(NRi: int) -> int:
    """generate_field.c:49: the generator's seed for realization NRi."""
    return 100020 + 146 * NRi


def field_generate(NN: int, seed: int, LL: float = 0.56, ff: float = 0.5, beta: float = 1.0):
    """generate_field.c:81-86 (Fill_Modes .. RSD) -> (r2c double[NN][NN][NN+2], sigma).
    The Gaussian draws are the Philox stream of oracle/philox_normal.h."""
    L = lib()
    L.orc_field_generate.argtypes = [ctypes.c_long, ctypes.c_uint64, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    L.orc_field_generate.restype = ctypes.c_int
    out = np.zeros((NN, NN, NN + 2))
    sigma = ctypes.c_double()
    if L.orc_field_generate(NN, seed, LL, ff, beta, _dp(out), ctypes.byref(sigma)) != 0:
        raise ValueError("orc_field_generate: invalid arguments")
    return out, sigma.value


def field_fill_modes(NN: int, seed: int, LL: float = 0.56) -> np.ndarray:
    """ngrf_2d_funcs.c:341-510 -> the Gaussian half-complex modes, complex [NN][NN][NN/2+1]."""
    L = lib()
    L.orc_field_fill_modes.argtypes = [ctypes.c_long, ctypes.c_uint64, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
    out = np.zeros((NN, NN, NN // 2 + 1), dtype=np.complex128)
    L.orc_field_fill_modes(NN, seed, LL, out.view(np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return out


def field_ingest(cube: np.ndarray, LL: float = 0.56, beta: float = 1.0) -> np.ndarray:
    """Get_Modes + RSD (ngrf_2d_funcs.c:534-550,734-765) of a real cube [NN][NN][NN] -> r2c buffer."""
    cube = np.ascontiguousarray(cube, dtype=np.float64)
    NN = cube.shape[0]
    L = lib()
    L.orc_field_ingest.argtypes = [ctypes.c_long, ctypes.c_double, ctypes.c_double,
                                   ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    L.orc_field_ingest.restype = ctypes.c_int
    out = np.zeros((NN, NN, NN + 2))
    if L.orc_field_ingest(NN, LL, beta, _dp(cube), _dp(out)) != 0:
        raise ValueError("orc_field_ingest: invalid arguments")
    return out


def r2c_3d(cube: np.ndarray) -> np.ndarray:
    """The oracle's in-place 3D r2c transform (FFTW's fftw_plan_dft_r2c_3d definition) of a real cube."""
    cube = np.asarray(cube, dtype=np.float64)
    NN = cube.shape[0]
    buf = np.zeros((NN, NN, NN + 2))
    buf[:, :, :NN] = cube
    lib().orc_r2c_3d(NN, NN, NN, _dp(buf))
    return buf.view(np.complex128)


def c2r_3d(half: np.ndarray) -> np.ndarray:
    """The oracle's 3D c2r transform (FFTW's fftw_plan_dft_c2r_3d definition) of a half spectrum."""
    half = np.ascontiguousarray(half, dtype=np.complex128)
    NN = half.shape[0]
    buf = half.view(np.float64).copy()
    lib().orc_c2r_3d(NN, NN, NN, _dp(buf))
    return buf[:, :, :NN].copy()


def biana(tri: np.ndarray, NN: int, LL: float = 1.0) -> np.ndarray:
    """barbie.c:300-305: analytic bispectrum of each enumerated triangle."""
    tri = np.ascontiguousarray(tri, dtype=TRIPLE_DTYPE)
    out = np.zeros(max(1, len(tri)))
    lib().orc_biana_all(NN, LL, tri.ctypes.data_as(ctypes.c_void_p), len(tri), _dp(out))
    return out[: len(tri)]


def estimate(r2c: np.ndarray, NN, Nmax, Nr, UL_k1, LL_k1, BW_k1, n_mtbin=5, LL=1.0,
             nthreads=None, want_B=False, wide=False):
    """The full estimator (barbie.c:110-397) with the plane-ring cache in RAM.
    wide: accumulate each triangle's pixel sum in long double (orc_estimate_ex).

    Returns dict(bs, norm, out, counts, ana, ana_out[, B]) with bins shaped
    [n_k1bin][n_mtbin][n_mtbin][16] (counts without the pole axis)."""
    n_k1bin = int((UL_k1 - LL_k1) / (1.0 * BW_k1))
    shape = (n_k1bin, n_mtbin, n_mtbin, NPOLES)
    bs, nm, out, ana = np.zeros(shape), np.zeros(shape), np.zeros(shape), np.zeros(shape)
    counts = np.zeros(shape[:3], dtype=np.int64)
    ntri = 0
    B = None
    if want_B:
        ntri = len(enumerate_triples(NN, Nmax, Nr, UL_k1, LL_k1, BW_k1, n_mtbin)[0])
        B = np.zeros(max(ntri, 1))
    nthreads = nthreads or os.cpu_count() or 1
    rc = lib().orc_estimate_ex(NN, Nmax, Nr, UL_k1, LL_k1, BW_k1, n_mtbin, LL,
                               _dp(np.ascontiguousarray(r2c, dtype=np.float64)), _dp(bs), _dp(nm), _dp(out),
                               counts.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                               _dp(B) if B is not None else None, ntri, nthreads, _dp(ana), int(bool(wide)))
    if rc != 0:
        raise RuntimeError(f"orc_estimate failed ({rc})")
    with np.errstate(divide="ignore", invalid="ignore"):
        ana_out = ana / nm  # column 5 of the output files, barbie.c:391
    res = dict(bs=bs, norm=nm, out=out, counts=counts, ana=ana, ana_out=ana_out)
    if want_B:
        res["B"] = B[:ntri]
    return res


def fft2_backward(a: np.ndarray) -> np.ndarray:
    """Unnormalised backward 2D DFT (the FFTW_BACKWARD transform of funcs.c:546)."""
    z = np.ascontiguousarray(a, dtype=np.complex128).copy()
    lib().orc_fft2d(z.shape[0], z.shape[1], +1, z.view(np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return z


def time_sample(r2c, NN, Nmax, Nr, UL_k1, LL_k1, BW_k1, sample, nthreads):
    """CPU timing of a bounded sample of one bispectrum's work (see orc_time_sample)."""
    L = lib()
    L.orc_time_sample.argtypes = [ctypes.c_long, ctypes.c_long, ctypes.c_long, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_long),
                                  ctypes.c_long, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(ctypes.c_double)]
    L.orc_time_sample.restype = ctypes.c_int
    s = np.ascontiguousarray(sample, dtype=np.int64)
    t_fft, t_sum, chk = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    n_fft = ctypes.c_long()
    rc = L.orc_time_sample(NN, Nmax, Nr, UL_k1, LL_k1, BW_k1, _dp(np.ascontiguousarray(r2c, dtype=np.float64)),
                           s.ctypes.data_as(ctypes.POINTER(ctypes.c_long)), len(s), int(nthreads),
                           ctypes.byref(t_fft), ctypes.byref(n_fft), ctypes.byref(t_sum), ctypes.byref(chk))
    if rc != 0:
        raise RuntimeError("orc_time_sample failed")
    return dict(t_fft=t_fft.value, n_fft=n_fft.value, t_sum=t_sum.value, checksum=chk.value)
