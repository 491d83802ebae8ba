"""GPU power spectrum multipoles (beam_gpu_power_multipoles, the reference's
calpow_mom, funcs.c:860-1074) against the oracle and the reference program's
own outputs, through the C ABI, and the `calpow_mom` drop-in. Needs an sm_100a
device.

Tolerances: mode counts exact (every mode lands in the reference's bin); mean
|k|, P0 and P2 within 1e-12 relative (they round as the reference's float and
double expressions, only the order of the bin sums differs); P4 and P6 within
1e-8 of themselves plus 1e-8 of the bin's P0 (the reference's libm powf is off
by one float ulp from the correctly rounded mu^4, mu^6 on about 0.06% of modes;
those differences scale with the bin's power, and P4, P6 cancel in the
highest bins)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, GOLDEN_CASES, ROOT, golden_field

pytestmark = pytest.mark.gpu

COLS = ("k", "P0", "P2", "P4", "P6", "count")
RTOL = dict(k=1e-12, P0=1e-12, P2=1e-12, P4=1e-8, P6=1e-8, count=0.0)


@pytest.fixture(scope="module")
def ctx(beamlib):
    c = beamlib.Context(0)
    yield c
    c.close()


def check(got, want, p46_atol=1e-8):
    for col in COLS:
        a, b = np.asarray(got[col]), np.asarray(want[col])
        atol = p46_atol * np.abs(np.asarray(want["P0"])) if col in ("P4", "P6") else 0.0
        assert np.all(np.abs(a - b) <= RTOL[col] * np.abs(b) + atol), (col, a, b)


@pytest.mark.parametrize("name", ["nn64_cfg1", "nn96_r20", "nn256_cfg2"])
def test_power_multipoles_match_reference(beamlib, ctx, name):
    path = os.path.join(GOLDEN, f"pk_{name}.npz")
    if not os.path.exists(path):
        pytest.skip("fixture not generated")
    ref = np.load(path)["pk"]
    NN = GOLDEN_CASES[name][0]
    got = beamlib.power_multipoles(ctx, golden_field(name), NN, LL=0.56, Nbin=10)
    keep = got["count"] > 0
    check({c: got[c][keep] for c in COLS}, {c: ref[:, k] for k, c in enumerate(COLS)})


@pytest.mark.parametrize("Nbin", [7, 24, 100])  # 100: the per-plane kernel (more than 32 bins)
def test_power_multipoles_match_oracle_other_bins(beamlib, ctx, oracle, Nbin):
    torch = pytest.importorskip("torch")
    name = "nn96_r20"
    NN = GOLDEN_CASES[name][0]
    f = golden_field(name)
    want = oracle.power_multipoles(f, NN, LL=1.0, Nbin=Nbin)
    # with many narrow bins a bin holds few modes, so one float ulp of mu^4 or
    # mu^6 on one of them is no longer small beside the bin's P0
    p46 = 1e-8 if Nbin <= 24 else 1e-6
    check(beamlib.power_multipoles(ctx, f, NN, LL=1.0, Nbin=Nbin), want, p46)
    check(beamlib.power_multipoles(ctx, torch.from_numpy(f).cuda(), NN, LL=1.0, Nbin=Nbin), want, p46)


def test_calpow_mom_drop_in(tmp_path):
    """`calpow_mom NN NRi` reads and writes the reference program's files."""
    from barbie_b200.synth import write_field
    name = "nn64_cfg1"
    path = os.path.join(GOLDEN, f"pk_{name}.npz")
    if not os.path.exists(path):
        pytest.skip("fixture not generated")
    ref = np.load(path)["pk"]
    NN, r = GOLDEN_CASES[name][0], GOLDEN_CASES[name][6]
    (tmp_path / f"ResFiles_N{NN}" / "data_files").mkdir(parents=True)
    write_field(str(tmp_path / f"ResFiles_N{NN}" / "data_files" / f"field_N{NN}_R{r}.txt"), golden_field(name))
    exe = os.path.join(ROOT, "barbie_b200", "calpow_mom")
    out = subprocess.run([exe, str(NN), str(r)], cwd=tmp_path, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    mine = np.loadtxt(tmp_path / f"ResFiles_N{NN}" / f"psoutN{NN}_R{r}.dat", ndmin=2)
    assert mine.shape == ref.shape
    assert np.all(np.abs(mine - ref) <= 6e-7 * np.abs(ref))  # %e keeps 7 significant digits
    bad = subprocess.run([exe, str(NN)], cwd=tmp_path, capture_output=True, text=True)
    assert bad.returncode == 1 and "Usage" in bad.stdout


def test_repeated_calls_with_kept_geometry_give_the_same_bits(beamlib, oracle):
    """The first call with a given (NN, Nbin) forms every sum from the modes and
    keeps the geometry; later calls read it and form only the field's sums, in
    the same order: the same bits, for another field too, and again after a
    call with other sizes replaced the kept geometry."""
    from barbie_b200.synth import realization_seed, synth_field
    ctx = beamlib.Context(0)
    name = "nn96_r20"
    NN = GOLDEN_CASES[name][0]
    f, g = golden_field(name), synth_field(NN, realization_seed(9))
    first = beamlib.power_multipoles(ctx, f, NN, LL=0.56, Nbin=10)  # forms everything, keeps the geometry
    second = beamlib.power_multipoles(ctx, f, NN, LL=0.56, Nbin=10)  # from the kept geometry
    other = beamlib.power_multipoles(ctx, g, NN, LL=0.56, Nbin=10)
    beamlib.power_multipoles(ctx, golden_field("nn64_cfg1"), 64, LL=0.56, Nbin=10)  # other sizes replace it
    again = beamlib.power_multipoles(ctx, f, NN, LL=0.56, Nbin=10)
    for col in COLS:
        assert np.array_equal(first[col], second[col]), col
        assert np.array_equal(first[col], again[col]), col
    ctx2 = beamlib.Context(0)  # a fresh context forms the other field's sums from its modes
    fresh = beamlib.power_multipoles(ctx2, g, NN, LL=0.56, Nbin=10)
    for col in COLS:
        assert np.array_equal(other[col], fresh[col]), col
    ctx2.close()
    ctx.close()
