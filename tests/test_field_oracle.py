"""The field generator's oracle (oracle/field_oracle.c) pinned to the reference
generator and to numpy; no GPU.

The fixtures field_<case>.npz are the output files of the reference's
generate_field.c + ngrf_2d_funcs.c, compiled from its own sources against the
FFTW shim and the GSL stand-in (oracle/Makefile); both draw the Philox normal
stream of oracle/philox_normal.h."""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

FIELD_CASES = {"n16_r1": (16, 1), "n24_r3": (24, 3)}  # as in tests/golden/make_golden.py


def load_field(name):
    z = np.load(os.path.join(GOLDEN, f"field_{name}.npz"))
    return z["r2c"], float(z["sigma"])


def rsd_factor(NN, beta):
    """(1 + beta mu^2) of ngrf_2d_funcs.c:743-762 over the half-complex array (1 at k = 0)."""
    i = np.arange(NN)
    f = np.minimum(i, NN - i).astype(np.float64)
    k = np.arange(NN // 2 + 1, dtype=np.float64)
    kk = np.sqrt(f[:, None, None] ** 2 + f[None, :, None] ** 2 + k[None, None, :] ** 2)
    with np.errstate(invalid="ignore", divide="ignore"):
        mu = k[None, None, :] / kk
    out = 1.0 + beta * mu * mu
    out[0, 0, 0] = 1.0
    return out


@pytest.mark.parametrize("name", list(FIELD_CASES))
def test_oracle_field_generate_matches_reference(oracle, name):
    """generate_field.c:81-86 restated: bit for bit the reference generator's
    output file (same normal stream, same transforms, same libm)."""
    NN, r = FIELD_CASES[name]
    ref, sigma_ref = load_field(name)
    got, sigma = oracle.field_generate(NN, oracle.field_seed(r))
    assert np.array_equal(got, ref)
    assert sigma == pytest.approx(sigma_ref, rel=1e-6)  # printed with %e


def test_oracle_field_generate_matches_live_reference(oracle, tmp_path):
    """Where the reference generator was built here, a larger grid too (NN=48: a radix-3 stage)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "field_ref")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/field_ref not built (reference sources absent)")
    NN, r = 48, 2
    (tmp_path / f"ResFiles_N{NN}" / "data_files").mkdir(parents=True)
    subprocess.run([exe, str(NN), str(r)], cwd=tmp_path, check=True, capture_output=True)
    ref = np.fromfile(tmp_path / f"ResFiles_N{NN}" / "data_files" / f"field_N{NN}_R{r}.txt").reshape(NN, NN, NN + 2)
    got, _ = oracle.field_generate(NN, oracle.field_seed(r))
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("NN", [4, 6, 12, 16, 24, 48])
def test_oracle_real_transforms_match_numpy(oracle, NN):
    """The 3D r2c / c2r of the FFTW definitions (fft.c) against numpy's pocketfft."""
    x = np.random.default_rng(NN).standard_normal((NN, NN, NN))
    X = oracle.r2c_3d(x)
    want = np.fft.rfftn(x)
    assert np.abs(X - want).max() <= 1e-13 * np.abs(want).max()
    y = oracle.c2r_3d(want)
    assert np.abs(y - x * NN**3).max() <= 1e-13 * np.abs(x * NN**3).max()


@pytest.mark.parametrize("beta", [0.0, 1.0, 0.37])
def test_oracle_field_ingest_matches_numpy(oracle, beta):
    """Get_Modes + RSD: rfftn(x LL^3) (1 + beta mu^2)."""
    NN, LL = 24, 0.56
    x = np.random.default_rng(7).standard_normal((NN, NN, NN))
    got = oracle.field_ingest(x, LL=LL, beta=beta).view(np.complex128)
    want = np.fft.rfftn(x * LL**3) * rsd_factor(NN, beta)
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()


def test_oracle_fill_modes_structure_and_statistics(oracle):
    """Fill_Modes (ngrf_2d_funcs.c:341-510): every mode written once with the
    amplitude sqrt(vol/2 k^-2) times a unit normal; the k=0 and k=N/2 planes
    Hermitian; the 7 non-zero corner modes real; the deviates N(0, 1)."""
    NN, LL = 32, 0.56
    A = oracle.field_fill_modes(NN, 12345, LL)
    h = NN // 2
    assert A[0, 0, 0] == 0
    for i in (0, h):
        for j in (0, h):
            for k in (0, h):
                assert A[i, j, k].imag == 0
    neg = (-np.arange(NN)) % NN
    for k in (0, h):
        P = A[:, :, k]
        assert np.array_equal(P, np.conj(P[neg][:, neg]))
    f = np.minimum(np.arange(NN), NN - np.arange(NN)).astype(np.float64)
    C = 2 * np.pi / (NN * LL)
    kmag = C * np.sqrt(f[:, None, None] ** 2 + f[None, :, None] ** 2 + np.arange(h + 1)[None, None, :] ** 2.0)
    kmag[0, 0, 0] = 1.0
    amp = np.sqrt((NN * LL) ** 3 / 2 * kmag**-2.0)
    g = (A / amp).ravel()[1:]
    re, im = g.real, g.imag[g.imag != 0]
    assert abs(re.mean()) < 0.01 and abs(re.var() - 1) < 0.02
    assert abs(im.mean()) < 0.01 and abs(im.var() - 1) < 0.02
