"""The library's host-side geometry (ring membership, closed ring triplets, the
accepted triangles of the loop with K1/T/MU/px/pz and bins) against the oracle,
bit for bit. Runs on the CPU: beam_geom_build needs no device."""
import ctypes

import numpy as np
import pytest


class Geom(ctypes.Structure):
    _fields_ = [("NN", ctypes.c_long), ("Nmax", ctypes.c_long), ("Nr", ctypes.c_long),
                ("UL_k1", ctypes.c_int), ("LL_k1", ctypes.c_int), ("BW_k1", ctypes.c_int),
                ("n_mtbin", ctypes.c_int), ("n_k1bin", ctypes.c_int),
                ("LL", ctypes.c_double), ("vol", ctypes.c_double),
                ("low", ctypes.POINTER(ctypes.c_double)), ("high", ctypes.POINTER(ctypes.c_double)),
                ("avg", ctypes.POINTER(ctypes.c_double)), ("ringmap", ctypes.POINTER(ctypes.c_int16)),
                ("nrp", ctypes.c_long), ("rp", ctypes.POINTER(ctypes.c_int32)),
                ("ntri", ctypes.c_long), ("t_rp", ctypes.POINTER(ctypes.c_int32)),
                ("t_p1", ctypes.POINTER(ctypes.c_int32)), ("t_p2", ctypes.POINTER(ctypes.c_int32)),
                ("t_bin", ctypes.POINTER(ctypes.c_int32)),
                ("t_px", ctypes.POINTER(ctypes.c_double)), ("t_pz", ctypes.POINTER(ctypes.c_double)),
                ("t_ana", ctypes.POINTER(ctypes.c_double)), ("iterations", ctypes.c_long)]


def build_geom(beamlib, NN, Nmax, Nr, UL, LL, BW, n_mtbin=5):
    L = beamlib.load()
    L.beam_geom_build.argtypes = [ctypes.POINTER(Geom), ctypes.POINTER(beamlib.Cfg)]
    L.beam_geom_build.restype = ctypes.c_int
    L.beam_geom_free.argtypes = [ctypes.POINTER(Geom)]
    L.beam_geom_free.restype = None
    cfg = beamlib.Cfg()
    L.beam_cfg_default(ctypes.byref(cfg), NN, UL, LL, BW)
    cfg.Nmax, cfg.Nr, cfg.n_mtbin = Nmax, Nr, n_mtbin
    g = Geom()
    rc = L.beam_geom_build(ctypes.byref(g), ctypes.byref(cfg))
    return rc, g, L


def arr(ptr, n, dtype):
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True) if n else np.zeros(0, dtype)


@pytest.mark.parametrize("NN,Nmax,Nr,UL,LL,BW", [
    (64, 16, 10, 11, 1, 1),     # config 1
    (64, 16, 10, 13, 3, 2),
    (96, 32, 20, 21, 1, 1),
    (256, 64, 30, 31, 1, 1),    # config 2
    (384, 100, 40, 51, 1, 1),   # config 3
])
def test_geometry_bit_identical_to_oracle(beamlib, oracle, NN, Nmax, Nr, UL, LL, BW):
    rc, g, L = build_geom(beamlib, NN, Nmax, Nr, UL, LL, BW)
    assert rc == 0
    try:
        low, high, avg = oracle.ring_edges(Nr, Nmax)
        assert np.array_equal(arr(g.low, Nr, np.float64), low)
        assert np.array_equal(arr(g.high, Nr, np.float64), high)
        assert np.array_equal(arr(g.avg, Nr, np.float64), avg)
        rings = oracle.closed_rings(NN, Nr, Nmax)
        assert g.nrp == len(rings)
        assert np.array_equal(arr(g.rp, 3 * g.nrp, np.int32).reshape(-1, 3), rings[:, :3].astype(np.int32))
        if NN <= 96:
            RR = oracle.ring_masks(NN, Nr, Nmax)
            want = np.full(NN * NN, -1, np.int16)
            for r in range(Nr):
                want[RR[r].reshape(-1) != 0] = r
            assert np.array_equal(arr(g.ringmap, NN * NN, np.int16), want)
        tri, iters = oracle.enumerate_triples(NN, Nmax, Nr, UL, LL, BW, rings4=rings)
        assert g.ntri == len(tri) and g.iterations == iters
        assert np.array_equal(arr(g.t_rp, g.ntri, np.int32), tri["rp"])
        assert np.array_equal(arr(g.t_p1, g.ntri, np.int32), tri["p1"])
        assert np.array_equal(arr(g.t_p2, g.ntri, np.int32), tri["p2"])
        bins = (tri["k1_bin"].astype(np.int64) * 5 + tri["t_bin"]) * 5 + tri["mu_bin"]
        assert np.array_equal(arr(g.t_bin, g.ntri, np.int32), bins.astype(np.int32))
        # bit-identical orientation parameters
        assert np.array_equal(arr(g.t_px, g.ntri, np.float64).view(np.int64), tri["px"].view(np.int64))
        assert np.array_equal(arr(g.t_pz, g.ntri, np.float64).view(np.int64), tri["pz"].view(np.int64))
        # bit-identical analytic bispectrum per triangle (barbie.c:300-305)
        ana = oracle.biana(tri, NN)
        assert np.array_equal(arr(g.t_ana, g.ntri, np.float64).view(np.int64), ana.view(np.int64))
        assert g.vol == float(NN) ** 3
    finally:
        L.beam_geom_free(ctypes.byref(g))


@pytest.mark.parametrize("bad", [
    dict(NN=63), dict(Nr=15), dict(BW=0), dict(UL=1), dict(UL=12, BW=2), dict(Nmax=40),
])
def test_geometry_rejects_invalid_configs(beamlib, bad):
    p = dict(NN=64, Nmax=16, Nr=10, UL=11, LL=1, BW=1)
    p.update(bad)
    rc, g, L = build_geom(beamlib, p["NN"], p["Nmax"], p["Nr"], p["UL"], p["LL"], p["BW"])
    assert rc == beamlib.BEAM_EINVAL
