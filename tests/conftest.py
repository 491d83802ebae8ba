import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")

# name: (NN, Nmax, Nr, UL_k1, LL_k1, BW_k1, realization), as in tests/golden/make_golden.py
GOLDEN_CASES = {
    "nn64_cfg1": (64, 16, 10, 11, 1, 1, 1),
    "nn64_bw2": (64, 16, 10, 13, 3, 2, 2),
    "nn96_r20": (96, 32, 20, 21, 1, 1, 3),
    "nn256_cfg2": (256, 64, 30, 31, 1, 1, 1),
}


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (sm_100a) device")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle_py
    if not os.path.exists(oracle_py.LIB_PATH):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)
    oracle_py.lib()
    return oracle_py


@pytest.fixture(scope="session")
def beamlib():
    lib_path = os.path.join(ROOT, "barbie_b200", "libbeam_gpu.so")
    if not os.path.exists(lib_path):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "barbie_b200")], check=True)
    from barbie_b200 import beam
    beam.load()
    return beam


def load_golden(name):
    path = os.path.join(GOLDEN, f"{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"golden fixture {name} not generated")
    z = np.load(path)
    return dict(rows=z["rows"], sha=str(z["field_sha256"]), config=tuple(int(v) for v in z["config"]))


def golden_field(name):
    from barbie_b200.synth import realization_seed, synth_field
    NN = GOLDEN_CASES[name][0]
    return synth_field(NN, realization_seed(GOLDEN_CASES[name][6]))


def compare_to_golden(rows, out, norm, NN, rtol=1e-10, ana=None, ana_rtol=1e-9):
    """Check every printed reference row against out[i,j,l,ii] and norm/NN^2
    (and, when given, the analytic column ana[i,j,l,ii] against column 5), and
    that exactly the reference's rows would be printed. Returns the max
    relative difference of the multipole values.

    Columns 5 and 6 are weighted by each triplet's Num, which the reference
    takes from calCR's FFT (NN^2 x count with round-off that reaches ~1e-10 at
    NN=256) and the library from the exact count: they get the 1e-9 bar."""
    printed = {(int(r[1]), int(r[2]), int(r[3])) for r in rows}
    mine = {tuple(int(v) for v in ijl) for ijl in np.argwhere(norm[..., 0] > 0.1)}
    assert printed == mine, (sorted(printed ^ mine)[:10])
    worst = 0.0
    for r in rows:
        ii, i, j, l = (int(v) for v in r[:4])
        ref, val = r[4], out[i, j, l, ii]
        if np.isnan(ref) or np.isnan(val):
            assert np.isnan(ref) and np.isnan(val), (ii, i, j, l, ref, val)
        else:
            rel = abs(val - ref) / max(abs(ref), 1e-300)
            worst = max(worst, rel)
            assert rel <= rtol, (ii, i, j, l, ref, val, rel)
        nref, nval = r[5], norm[i, j, l, ii] / (NN * NN)
        assert abs(nval - nref) <= 1e-9 * max(1.0, abs(nref)), (ii, i, j, l, nref, nval)
        if ana is not None:
            aref, aval = r[6], ana[i, j, l, ii]
            if np.isnan(aref) or np.isnan(aval):
                assert np.isnan(aref) and np.isnan(aval), (ii, i, j, l, aref, aval)
            else:
                assert abs(aval - aref) <= ana_rtol * max(abs(aref), 1e-300), (ii, i, j, l, aref, aval)
    return worst
