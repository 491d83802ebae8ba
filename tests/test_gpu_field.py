"""Field ingestion on the GPU (beam_gpu_field_generate / beam_gpu_field_ingest):
the reference's field generator (generate_field.c:78-88, ngrf_2d_funcs.c) and
its real-space-to-r2c step, against the reference generator's output files,
the oracle and numpy, through the C ABI; the `field` drop-in. Needs an sm_100a
device.

Tolerance: the device transforms are FP64 Stockham FFTs whose rounding differs
from the oracle's, so fields are compared on the scale of the field:
max |got - want| <= 1e-12 max |want|; sigma within 1e-13 relative. Mode
placement, the RSD factor and the amplitudes round as the reference's C."""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, GOLDEN_CASES, ROOT

pytestmark = pytest.mark.gpu

FIELD_CASES = {"n16_r1": (16, 1), "n24_r3": (24, 3)}
TOL = 1e-12


@pytest.fixture(scope="module")
def ctx(beamlib):
    c = beamlib.Context(0)
    yield c
    c.close()


def close(got, want, tol=TOL):
    got, want = np.asarray(got), np.asarray(want)
    err = np.abs(got - want).max()
    assert err <= tol * np.abs(want).max(), err / np.abs(want).max()


def modes(r2c):
    """The r2c buffer's complex values (the padded doubles are the last axis)."""
    return np.ascontiguousarray(r2c).view(np.complex128)


@pytest.mark.parametrize("name", list(FIELD_CASES))
def test_generate_matches_reference_generator(beamlib, ctx, oracle, name):
    NN, r = FIELD_CASES[name]
    z = np.load(os.path.join(GOLDEN, f"field_{name}.npz"))
    got, sigma = beamlib.generate_field(ctx, NN, beamlib.field_seed(r))
    close(modes(got), modes(z["r2c"]))
    _, sigma_o = oracle.field_generate(NN, oracle.field_seed(r))
    assert sigma == pytest.approx(sigma_o, rel=1e-13)


@pytest.mark.parametrize("NN", [4, 6, 12, 32, 48, 96, 128])
def test_generate_matches_oracle(beamlib, ctx, oracle, NN):
    """Radix mixes 4, 2+3, 4+3, 4+4+2, 4+4+3, 4+4+2+3, 4+4+4+2; other ff and beta."""
    seed, LL, ff, beta = 777 + NN, 0.8, 0.3, 0.6
    want, sigma_o = oracle.field_generate(NN, seed, LL=LL, ff=ff, beta=beta)
    got, sigma = beamlib.generate_field(ctx, NN, seed, LL=LL, ff=ff, beta=beta)
    close(modes(got), modes(want))
    assert sigma == pytest.approx(sigma_o, rel=1e-13)


def test_generate_is_deterministic_and_device_output_matches(beamlib, ctx):
    torch = pytest.importorskip("torch")
    NN = 96
    a, sa = beamlib.generate_field(ctx, NN, 5)
    b, sb = beamlib.generate_field(ctx, NN, 5)
    assert np.array_equal(a, b) and sa == sb
    d = torch.empty((NN, NN, NN + 2), dtype=torch.float64, device="cuda")
    c, sc = beamlib.generate_field(ctx, NN, 5, out=d)
    assert c is d and sc == sa
    assert np.array_equal(d.cpu().numpy(), a)


@pytest.mark.parametrize("NN,beta", [(48, 1.0), (64, 0.0), (64, 0.45)])
def test_ingest_matches_oracle_host_and_device(beamlib, ctx, oracle, NN, beta):
    torch = pytest.importorskip("torch")
    x = np.random.default_rng(NN).standard_normal((NN, NN, NN))
    want = modes(oracle.field_ingest(x, LL=0.56, beta=beta))
    got_h = beamlib.ingest_field(ctx, x, LL=0.56, beta=beta)
    close(modes(got_h), want)
    xd = torch.from_numpy(x).cuda()
    out = torch.empty((NN, NN, NN + 2), dtype=torch.float64, device="cuda")
    beamlib.ingest_field(ctx, xd, LL=0.56, beta=beta, out=out)
    got_d = out.cpu().numpy()
    assert np.array_equal(got_d[..., :NN + 2], got_h)  # same kernels, same bits
    pinned = torch.from_numpy(x).pin_memory()
    got_p = beamlib.ingest_field(ctx, pinned, LL=0.56, beta=beta)
    assert np.array_equal(got_p, got_h)


@pytest.mark.parametrize("NN", [384, 512])
def test_ingest_full_size_plane_waves(beamlib, ctx, NN):
    """Size-independent: a sum of two plane waves goes to exactly four modes
    (two and their Hermitian partners on k = 0), N^3/2 LL^3 (1 + beta mu^2)
    each; every other mode is round-off."""
    torch = pytest.importorskip("torch")
    LL, beta = 0.56, 1.0
    waves = [((3, 5, 7), 1.0), ((NN // 2 - 1, 1, 0), 0.5)]
    i = torch.arange(NN, dtype=torch.int64, device="cuda")
    x = torch.zeros((NN, NN, NN), dtype=torch.float64, device="cuda")
    for (a, b, c), w in waves:
        n = (a * i[:, None, None] + b * i[None, :, None] + c * i[None, None, :]) % NN  # exact phase index
        x += w * torch.cos(n.to(torch.float64) * (2 * np.pi / NN))
        del n
    out = torch.empty((NN, NN, NN + 2), dtype=torch.float64, device="cuda")
    beamlib.ingest_field(ctx, x, LL=LL, beta=beta, out=out)
    X = torch.view_as_complex(out.view(NN, NN, NN // 2 + 1, 2))
    expect = torch.zeros_like(X)
    scale = NN**3 / 2 * LL**3
    for (a, b, c), w in waves:
        fa, fb = min(a, NN - a), min(b, NN - b)
        mu = c / np.sqrt(fa * fa + fb * fb + c * c)
        v = w * scale * (1 + beta * mu * mu)
        expect[a, b, c] += v
        if c == 0:
            expect[(NN - a) % NN, (NN - b) % NN, 0] += v
    err = (X - expect).abs().max().item()
    assert err <= 1e-12 * NN**3 * LL**3, err


def test_generate_full_size_gaussian_round_trip(beamlib, ctx, oracle):
    """Size-independent at NN=384: with ff = 0 and beta = 0 the generator's
    c2r then r2c returns the Gaussian modes (x LL^3 / vol x NN^3 = 1), so the
    output is Fill_Modes itself to round-off; with beta = 1 it is Fill_Modes
    times (1 + mu^2)."""
    NN, seed, LL = 384, 99, 0.56
    A = oracle.field_fill_modes(NN, seed, LL)
    got, _ = beamlib.generate_field(ctx, NN, seed, LL=LL, ff=0.0, beta=0.0)
    close(modes(got), A)
    got, _ = beamlib.generate_field(ctx, NN, seed, LL=LL, ff=0.0, beta=1.0)
    i = np.arange(NN)
    f = np.minimum(i, NN - i).astype(np.float64)
    k = np.arange(NN // 2 + 1, dtype=np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        mu2 = k[None, None, :] ** 2 / (f[:, None, None] ** 2 + f[None, :, None] ** 2 + k[None, None, :] ** 2)
    mu2[0, 0, 0] = 0.0
    close(modes(got), A * (1.0 + mu2))


def test_generated_field_runs_through_the_estimator_on_device(beamlib, ctx, oracle):
    """The generator's device buffer goes straight into a bispectrum run; the
    bins match the oracle estimator on the same field."""
    torch = pytest.importorskip("torch")
    NN, Nmax, Nr, UL, LLk, BW, _ = GOLDEN_CASES["nn64_cfg1"]
    d = torch.empty((NN, NN, NN + 2), dtype=torch.float64, device="cuda")
    beamlib.generate_field(ctx, NN, beamlib.field_seed(4), out=d)
    plan = beamlib.Plan(ctx, NN, UL, LLk, BW, Nmax=Nmax, Nr=Nr)
    res = plan.run(d)
    want = oracle.estimate(d.cpu().numpy(), NN, Nmax, Nr, UL, LLk, BW)
    ok = want["norm"][..., 0] > 0.1
    for key, wkey in (("bs", "bs"), ("norm", "norm")):
        a, b = res[key][ok], want[wkey][ok]
        assert np.all(np.abs(a - b) <= 1e-10 * np.abs(b) + 1e-300), key
    assert np.array_equal(res["count"], want["counts"])


def test_invalid_sizes_are_rejected(beamlib, ctx):
    """Sizes other than even 2^a 3^b in [4, 1024] fail before any buffer is touched."""
    L = beamlib.load()
    beamlib.generate_field(ctx, 4, 1)  # sets the prototypes
    tiny = np.zeros(64)
    for NN in (10, 2, 7, 1536, 2048):
        rc = L.beam_gpu_field_generate(ctx._h, NN, 1, 0.56, 0.5, 1.0, tiny.ctypes.data, 0, None)
        assert rc == beamlib.BEAM_EINVAL, NN
    with pytest.raises(beamlib.BeamError):
        beamlib.ingest_field(ctx, np.zeros((20, 20, 20)))
    with pytest.raises(beamlib.BeamError):
        beamlib.generate_field(ctx, 12, 1, LL=0.0)


def test_overlapping_and_misaligned_device_buffers_are_rejected(beamlib, ctx):
    """A device cube that overlaps the r2c output, and a device r2c buffer off a
    16-byte boundary, are refused before any kernel runs."""
    torch = pytest.importorskip("torch")
    NN = 16
    big = torch.zeros(NN * NN * (NN + 2) + NN**3, dtype=torch.float64, device="cuda")
    out = big[: NN * NN * (NN + 2)].view(NN, NN, NN + 2)
    cube = big[8: 8 + NN**3].view(NN, NN, NN)  # starts inside the output
    with pytest.raises(beamlib.BeamError) as e:
        beamlib.ingest_field(ctx, cube, out=out)
    assert e.value.code == beamlib.BEAM_EINVAL
    buf = torch.zeros(NN * NN * (NN + 2) + 1, dtype=torch.float64, device="cuda")
    odd = buf[1:].view(NN, NN, NN + 2)  # 8 bytes past an aligned start
    with pytest.raises(beamlib.BeamError) as e:
        beamlib.power_multipoles(ctx, odd, NN)
    assert e.value.code == beamlib.BEAM_EINVAL


def test_field_cli_matches_reference_generator(tmp_path):
    exe = os.path.join(ROOT, "barbie_b200", "field")
    if not os.path.exists(exe):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "barbie_b200")], check=True)
    NN, r = FIELD_CASES["n24_r3"]
    (tmp_path / f"ResFiles_N{NN}" / "data_files").mkdir(parents=True)
    p = subprocess.run([exe, str(NN), str(r)], cwd=tmp_path, capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
    assert f"Generating field Realization(NRi) = {r} for Grids(NN) = {NN}" in p.stdout
    z = np.load(os.path.join(GOLDEN, "field_n24_r3.npz"))
    assert f"sigma = {float(z['sigma']):e}" in p.stdout
    got = np.fromfile(tmp_path / f"ResFiles_N{NN}" / "data_files" / f"field_N{NN}_R{r}.txt")
    close(modes(got.reshape(NN, NN, NN + 2)), modes(z["r2c"]))
