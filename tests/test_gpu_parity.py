"""GPU parity: libbeam_gpu against the reference's own outputs (golden
fixtures) and against the oracle, through the C ABI. Needs an sm_100a device.

Tolerances (FP64 path): multipole values within 1e-10 relative of the
reference per printed bin, normalisations within 1e-9 relative, triangle
counts exact, and exactly the reference's set of printed bins."""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN_CASES, ROOT, compare_to_golden, golden_field, load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(beamlib):
    c = beamlib.Context(0)
    yield c
    c.close()


def make_plan(beamlib, ctx, name, **kw):
    NN, Nmax, Nr, UL, LL, BW, _ = GOLDEN_CASES[name]
    return beamlib.Plan(ctx, NN, UL, LL, BW, Nmax=Nmax, Nr=Nr, **kw)


@pytest.mark.parametrize("name", list(GOLDEN_CASES))
def test_fp64_matches_reference_outputs(beamlib, ctx, name):
    g = load_golden(name)
    plan = make_plan(beamlib, ctx, name)
    res = plan.run(golden_field(name))
    NN = GOLDEN_CASES[name][0]
    worst = compare_to_golden(g["rows"], res["out"], res["norm"], NN, rtol=1e-10, ana=res["ana"])
    for r in g["rows"][g["rows"][:, 0] == 0]:
        assert res["count"][int(r[1]), int(r[2]), int(r[3])] == int(np.rint(r[5]))
    assert np.array_equal(res["norm"][..., 0], res["count"] * float(NN * NN))
    print(f"{name}: max relative difference to the reference {worst:.2e}")


@pytest.mark.parametrize("name", ["nn64_cfg1", "nn96_r20"])
def test_fp64_matches_oracle_arrays_and_triangle_sums(beamlib, ctx, oracle, name):
    NN, Nmax, Nr, UL, LL, BW, _ = GOLDEN_CASES[name]
    f = golden_field(name)
    want = oracle.estimate(f, NN, Nmax, Nr, UL, LL, BW, want_B=True)
    plan = make_plan(beamlib, ctx, name)
    res = plan.run(f)
    ok = want["norm"][..., 0] > 0.1
    for key, wkey in (("bs", "bs"), ("norm", "norm"), ("ana_sum", "ana")):
        a, b = res[key][ok], want[wkey][ok]
        fin = np.isfinite(b)
        assert np.all(np.abs(a[fin] - b[fin]) <= 1e-10 * np.abs(b[fin]) + 1e-300), key
    assert np.array_equal(res["count"], want["counts"])
    B = plan.triangle_sums(f)
    Bo = want["B"]
    assert B.shape == Bo.shape
    assert np.array_equal(B == 0, Bo == 0)  # the B == 0 rule of barbie.c:355-357
    # each B is a sum of many oscillating terms; compare on the scale of the sums
    scale = np.sqrt(np.mean(Bo ** 2))
    assert np.max(np.abs(B - Bo)) <= 1e-12 * scale + 1e-12 * np.max(np.abs(Bo))


@pytest.mark.parametrize("name", ["nn64_cfg1", "nn96_r20"])
def test_closed_ring_counts_exact(beamlib, ctx, oracle, name):
    NN, Nmax, Nr, *_ = GOLDEN_CASES[name]
    plan = make_plan(beamlib, ctx, name)
    got = plan.closed_rings()
    want = oracle.closed_rings(NN, Nr, Nmax)
    assert np.array_equal(got[:, :3], want[:, :3])
    assert np.array_equal(got[:, 3], np.rint(want[:, 3] / NN ** 2) * NN ** 2)


@pytest.mark.parametrize("name", ["nn64_cfg1", "nn96_r20"])
def test_plane_rings_match_oracle(beamlib, ctx, oracle, name):
    NN, Nmax, Nr, *_ = GOLDEN_CASES[name]
    f = golden_field(name)
    RR = oracle.ring_masks(NN, Nr, Nmax)
    planes = [0, 0, 0, 1, 3, Nmax - 1, Nmax // 2, 2]
    rings = [0, 1, Nr - 1, 0, 5, Nr - 1, Nr // 2, 9]
    plan = make_plan(beamlib, ctx, name)
    got = plan.plane_rings(f, planes, rings)
    for k, (p, r) in enumerate(zip(planes, rings)):
        want = oracle.plane_ring(NN, p, r, f, RR)
        scale = max(np.max(np.abs(want)), 1e-300)
        assert np.max(np.abs(got[k] - want)) <= 1e-13 * scale, (p, r)
    assert np.all(got[0] == 0)  # ring 0 on plane 0 is only the zeroed k=0 mode


@pytest.mark.parametrize("name", ["nn64_cfg1", "nn96_r20"])
def test_pixel_method_matches_triangle_method(beamlib, ctx, name):
    f = golden_field(name)
    a = make_plan(beamlib, ctx, name).run(f)
    b = make_plan(beamlib, ctx, name, method="pixel").run(f)
    ok = a["norm"][..., 0] > 0.1
    fin = np.isfinite(a["out"][ok])
    x, y = a["out"][ok][fin], b["out"][ok][fin]
    assert np.all(np.abs(x - y) <= 1e-10 * np.abs(x))
    assert np.array_equal(a["count"], b["count"])


def test_serving_geometry_matches_oracle(beamlib, ctx, oracle):
    """A job shape of the served mix: NN=128 with Nr=20 rings to Nmax=40 and k1
    bins 1..41 of width 2 (neither in the golden cases), FP64 at 1e-10 of the
    oracle per printed bin with exact counts, and the mixed path's counts."""
    from barbie_b200.synth import realization_seed, synth_field
    NN, Nmax, Nr, UL, LL, BW = 128, 40, 20, 41, 1, 2
    f = synth_field(NN, realization_seed(7))
    want = oracle.estimate(f, NN, Nmax, Nr, UL, LL, BW)
    res = beamlib.Plan(ctx, NN, UL, LL, BW, Nmax=Nmax, Nr=Nr).run(f)
    ok = want["norm"][..., 0] > 0.1
    assert np.array_equal(res["norm"][..., 0] > 0.1, ok) and ok.sum() > 100
    for key, wkey in (("bs", "bs"), ("norm", "norm"), ("out", "out")):
        a, b = res[key][ok], want[wkey][ok]
        fin = np.isfinite(b)
        assert np.array_equal(np.isfinite(a), fin), key
        assert np.all(np.abs(a[fin] - b[fin]) <= 1e-10 * np.abs(b[fin]) + 1e-300), key
    assert np.array_equal(res["count"], want["counts"])
    mix = beamlib.Plan(ctx, NN, UL, LL, BW, Nmax=Nmax, Nr=Nr, precision="mixed").run(f)
    assert np.array_equal(mix["count"], want["counts"])


def test_mixed_precision_error_is_bounded(beamlib, ctx):
    name = "nn96_r20"
    f = golden_field(name)
    a = make_plan(beamlib, ctx, name).run(f)
    b = make_plan(beamlib, ctx, name, precision="mixed").run(f)
    assert np.array_equal(a["count"], b["count"])
    ok = (a["norm"][..., 0] > 0.1)[..., None] & np.isfinite(a["out"]) & (a["out"] != 0)
    rel = np.abs(b["out"] - a["out"])[ok] / np.abs(a["out"][ok])
    print(f"mixed vs fp64: median {np.median(rel):.2e} p99 {np.quantile(rel, 0.99):.2e} max {rel.max():.2e}")
    assert np.median(rel) < 1e-5


def test_runs_are_deterministic_and_device_input_matches(beamlib, ctx):
    torch = pytest.importorskip("torch")
    name = "nn96_r20"
    f = golden_field(name)
    plan = make_plan(beamlib, ctx, name)
    a = plan.run(f)
    b = plan.run(f)
    for k in a:
        assert np.array_equal(a[k], b[k], equal_nan=True), k
    c = plan.run(torch.from_numpy(f).cuda())
    for k in a:
        assert np.array_equal(a[k], c[k], equal_nan=True), k


def test_misaligned_buffers(beamlib, ctx):
    """A device r2c buffer off a 16-byte boundary is refused (the kernels read
    it as complex128); a page-locked host one is gathered on the host instead
    of being read in place, with the same bins."""
    torch = pytest.importorskip("torch")
    name = "nn64_cfg1"
    f = golden_field(name)
    plan = make_plan(beamlib, ctx, name)
    a = plan.run(f)
    n = f.size
    dev = torch.zeros(n + 1, dtype=torch.float64, device="cuda")
    dev[1:] = torch.from_numpy(f.ravel()).cuda()
    with pytest.raises(beamlib.BeamError) as e:
        plan.run(dev[1:].view(f.shape))
    assert e.value.code == beamlib.BEAM_EINVAL
    host = torch.zeros(n + 1, dtype=torch.float64).pin_memory()
    host[1:] = torch.from_numpy(f.ravel())
    b = plan.run(host[1:].view(f.shape))
    for k in a:
        assert np.array_equal(a[k], b[k], equal_nan=True), k


def test_page_locked_host_input_matches_pageable(beamlib, ctx):
    """Page-locked host buffers are read in place by the device (no host gather);
    the bins must be the same bit for bit as from a pageable buffer."""
    torch = pytest.importorskip("torch")
    name = "nn96_r20"
    f = golden_field(name)
    plan = make_plan(beamlib, ctx, name)
    a = plan.run(f)
    pinned = torch.from_numpy(f).pin_memory()
    assert pinned.is_pinned()
    b = plan.run(pinned)
    for k in a:
        assert np.array_equal(a[k], b[k], equal_nan=True), k
    B1 = plan.triangle_sums(f)
    B2 = plan.triangle_sums(pinned)
    assert np.array_equal(B1, B2)


def test_zero_field_prints_no_bins(beamlib, ctx):
    name = "nn64_cfg1"
    NN = GOLDEN_CASES[name][0]
    res = make_plan(beamlib, ctx, name).run(np.zeros((NN, NN, NN + 2)))
    assert np.all(res["count"] == 0) and np.all(res["norm"] == 0) and np.all(res["bs"] == 0)
    assert not np.any(res["norm"][..., 0] > 0.1)


def test_batch_matches_single_runs(beamlib, ctx):
    from barbie_b200.synth import realization_seed, synth_field
    NN, Nmax, Nr, UL, LL, BW, _ = GOLDEN_CASES["nn64_cfg1"]
    plan = beamlib.Plan(ctx, NN, UL, LL, BW, Nmax=Nmax, Nr=Nr)
    fields = [synth_field(NN, realization_seed(r)) for r in (4, 5, 6)]
    batch = plan.run_batch(fields)
    for f, got in zip(fields, batch):
        want = plan.run(f)
        for k in want:
            assert np.array_equal(got[k], want[k], equal_nan=True), k


def test_host_drop_in_cli(tmp_path):
    """The `barbie` drop-in on the config-1 input writes the reference's files."""
    from barbie_b200.synth import write_field
    name = "nn64_cfg1"
    g = load_golden(name)
    NN, Nmax, Nr, UL, LL, BW, r = GOLDEN_CASES[name]
    write_field(str(tmp_path / f"field_N{NN}_R{r}.txt"), golden_field(name))
    exe = os.path.join(ROOT, "barbie_b200", "barbie")
    env = dict(os.environ, BEAM_NMAX=str(Nmax), BEAM_NR=str(Nr))
    out = subprocess.run([exe, str(NN), str(r), str(UL), str(LL), str(BW)], cwd=tmp_path, env=env,
                         capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    assert (tmp_path / f"ResFiles_N{NN}" / f"time_{NN}_R{r}.txt").exists()
    rows = []
    for ii in range(16):
        for line in open(tmp_path / f"ResFiles_N{NN}" / f"BS_test_ii{ii}_N{NN}_R{r}.txt"):
            f = line.split()
            rows.append((ii, int(f[0]), int(f[1]), int(f[2]), float(f[3]), float(f[5]), float(f[4])))
    assert len(rows) == len(g["rows"])
    for mine, ref in zip(rows, g["rows"]):
        assert mine[:4] == tuple(int(v) for v in ref[:4])
        if np.isnan(ref[4]):
            assert np.isnan(mine[4])
        else:
            assert abs(mine[4] - ref[4]) <= 6e-7 * abs(ref[4])  # %e keeps 7 significant digits
        assert abs(mine[5] - ref[5]) <= 1e-6 * max(1, abs(ref[5]))
        if np.isnan(ref[6]):  # column 5, the analytic bispectrum
            assert np.isnan(mine[6])
        else:
            assert abs(mine[6] - ref[6]) <= 6e-7 * abs(ref[6])
