"""Per-bin parity at the benchmark size and at served shapes outside the
reference-program fixtures, against the oracle's bins (tests/golden/oracle_*.npz,
made by tests/golden/make_golden.py --oracle: the oracle's pixel sums of
barbie.c:315-337, accumulated in long double, binned and weighted as
barbie.c:343-363, on the case's seeded field).

- nn384_cfg3: `barbie 384 1 51 1 1`, the benchmark workload, on the benchmark's
  first field: 923 printed bins x 16 multipoles.
- nn192_serve: NN=192, 30 rings to 60, k1 bins of width 2 over 1..61.
- nn512_serve: NN=512, 40 rings to 128, k1 bins 1..31.

The plain FP64 path must agree within 1e-10 relative on every printed
(l, m, bin), print the same bins, give the same NaN bins (odd m where every pz
is 0) and exact triangle counts. The CPU tests check each fixture against the
oracle's geometry (accepted triangles and their exact counts)."""
import hashlib
import os

import numpy as np
import pytest

from conftest import GOLDEN

# name: (NN, Nmax, Nr, UL_k1, LL_k1, BW_k1, realization), as ORACLE_CASES in tests/golden/make_golden.py
ORACLE_CASES = {
    "nn384_cfg3": (384, 100, 40, 51, 1, 1, 1),
    "nn192_serve": (192, 60, 30, 61, 1, 2, 4),
    "nn512_serve": (512, 128, 40, 31, 1, 1, 5),
}
RTOL = 1e-10


def load_fixture(name):
    path = os.path.join(GOLDEN, f"oracle_{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"oracle fixture {name} not generated")
    z = np.load(path)
    cfg = tuple(int(v) for v in z["config"])
    assert cfg == ORACLE_CASES[name]
    return {k: z[k] for k in ("bs", "norm", "ana", "counts")} | {"sha": str(z["field_sha256"])}


def fixture_field(name, sha):
    from barbie_b200.synth import realization_seed, synth_field
    NN, r = ORACLE_CASES[name][0], ORACLE_CASES[name][6]
    f = synth_field(NN, realization_seed(r))
    assert hashlib.sha256(f.tobytes()).hexdigest() == sha, "field recipe changed since the fixture was made"
    return f


def compare_bins(got_out, got_norm, fx, NN):
    """Max relative difference over the printed (l, m, bin) of got against the
    fixture; asserts the printed set and the NaN / zero pattern."""
    vol = float(NN) ** 3
    with np.errstate(divide="ignore", invalid="ignore"):
        want = fx["bs"] / (vol * fx["norm"])
    printed = fx["norm"][..., 0] > 0.1
    assert np.array_equal(got_norm[..., 0] > 0.1, printed)
    a, b = got_out[printed], want[printed]
    assert np.array_equal(np.isnan(a), np.isnan(b))
    fin = ~np.isnan(b)
    a, b = a[fin], b[fin]
    assert np.all(a[b == 0] == 0)
    nz = b != 0
    return float(np.max(np.abs(a[nz] - b[nz]) / np.abs(b[nz])))


@pytest.mark.parametrize("name", list(ORACLE_CASES))
def test_fixture_matches_the_oracle_geometry(oracle, name):
    """CPU: the fixture's per-bin counts are the oracle loop's exact triangle
    counts over the bin's accepted triangles with B != 0 (B = 0 exactly where
    a leg is ring 0 on plane 0: the zeroed k = 0 mode, funcs.c:104)."""
    fx = load_fixture(name)
    NN, Nmax, Nr, UL, LL, BW, _ = ORACLE_CASES[name]
    tri, _ = oracle.enumerate_triples(NN, Nmax, Nr, UL, LL, BW)
    dc = np.zeros(len(tri), dtype=bool)
    for k in "123":
        dc |= (tri["p" + k] == 0) & (tri["r" + k] == 0)
    t = tri[~dc]
    want = np.zeros(fx["counts"].shape, dtype=np.int64)
    np.add.at(want, (t["k1_bin"], t["t_bin"], t["mu_bin"]), np.rint(t["num"] / NN**2).astype(np.int64))
    assert np.array_equal(fx["counts"], want)
    # calCR's Num carries FFT round-off (funcs.c:396-399): norm[..][0] is NN^2 x count to ~1e-10
    assert np.allclose(fx["norm"][..., 0], NN**2 * want, rtol=1e-9, atol=0)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(ORACLE_CASES))
def test_fp64_bins_match_the_oracle(beamlib, name):
    fx = load_fixture(name)
    NN, Nmax, Nr, UL, LL, BW, _ = ORACLE_CASES[name]
    field = fixture_field(name, fx["sha"])
    ctx = beamlib.Context(0)
    plan = beamlib.Plan(ctx, NN, UL, LL, BW, Nmax=Nmax, Nr=Nr)
    res = plan.run(field)
    plan.close()
    ctx.close()
    assert np.array_equal(res["count"], fx["counts"])
    worst = compare_bins(res["out"], res["norm"], fx, NN)
    assert worst <= RTOL, worst
    # the analytic column (barbie.c:391): the library weights it by exact counts, the oracle by calCR's Num
    printed = fx["norm"][..., 0] > 0.1
    with np.errstate(divide="ignore", invalid="ignore"):
        want_ana = (fx["ana"] / fx["norm"])[printed]
    got_ana = res["ana"][printed]
    fin = np.isfinite(want_ana) & (want_ana != 0)
    assert np.max(np.abs(got_ana[fin] - want_ana[fin]) / np.abs(want_ana[fin])) <= 1e-9
