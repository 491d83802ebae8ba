"""The int8 path (BEAM_PREC_INT8): mode values cut into five 8-bit slices per
(ring, plane) scale, slice products and each run's sums exact in int32 on the
int8 tensor cores, FP64 from the run's end on. Its bar is the one the
mixed-precision target sets: every printed (l, m, bin) within 1e-5 relative
of the FP64 result -- checked here against the reference program's own
outputs (golden fixtures) and against the oracle's bins at the benchmark
size and the served shapes, with exact triangle counts and the same printed
bins. The sum being replaced is barbie.c:329-337."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, compare_to_golden, golden_field, load_golden
from test_gpu_oracle_large import ORACLE_CASES, compare_bins, fixture_field, load_fixture

pytestmark = pytest.mark.gpu

RTOL = 1e-5


@pytest.fixture(scope="module")
def ctx(beamlib):
    c = beamlib.Context(0)
    yield c
    c.close()


def make_plan(beamlib, ctx, case, **kw):
    NN, Nmax, Nr, UL, LL, BW = case[:6]
    return beamlib.Plan(ctx, NN, UL, LL, BW, Nmax=Nmax, Nr=Nr, **kw)


@pytest.mark.parametrize("name", list(GOLDEN_CASES))
def test_int8_matches_reference_outputs(beamlib, ctx, name):
    g = load_golden(name)
    plan = make_plan(beamlib, ctx, GOLDEN_CASES[name], precision="int8")
    res = plan.run(golden_field(name))
    plan.close()
    NN = GOLDEN_CASES[name][0]
    worst = compare_to_golden(g["rows"], res["out"], res["norm"], NN, rtol=RTOL)
    for r in g["rows"][g["rows"][:, 0] == 0]:
        assert res["count"][int(r[1]), int(r[2]), int(r[3])] == int(np.rint(r[5]))
    print(f"{name}: int8 max relative difference to the reference {worst:.2e}")


@pytest.mark.parametrize("name", list(ORACLE_CASES))
def test_int8_bins_match_the_oracle(beamlib, ctx, name):
    fx = load_fixture(name)
    field = fixture_field(name, fx["sha"])
    plan = make_plan(beamlib, ctx, ORACLE_CASES[name], precision="int8")
    res = plan.run(field)
    plan.close()
    assert np.array_equal(res["count"], fx["counts"])
    worst = compare_bins(res["out"], res["norm"], fx, ORACLE_CASES[name][0])
    print(f"{name}: int8 max relative difference to the oracle {worst:.2e}")
    assert worst <= RTOL, worst


def test_int8_is_deterministic_and_batches_match(beamlib, ctx):
    case = GOLDEN_CASES["nn96_r20"]
    from barbie_b200.synth import realization_seed, synth_field
    fields = [synth_field(case[0], realization_seed(r)) for r in (1, 2, 3)]
    plan = make_plan(beamlib, ctx, case, precision="int8")
    single = [plan.run(f) for f in fields]
    again = plan.run(fields[0])
    assert np.array_equal(single[0]["out"], again["out"], equal_nan=True)
    batch = plan.run_batch(fields)
    for a, b in zip(single, batch):
        assert np.array_equal(a["out"], b["out"], equal_nan=True)
        assert np.array_equal(a["count"], b["count"])
    # the triangle sums run as one launch per tile class only
    with pytest.raises(beamlib.BeamError):
        plan.set_triangle_launch("persistent")
    plan.close()


def test_int8_cubic_scaling(beamlib, ctx):
    """Scales are powers of two per (ring, plane): doubling the field doubles
    every scale and leaves every slice unchanged, so bs and out scale by
    exactly 8 and counts and norms stay put."""
    case = GOLDEN_CASES["nn64_cfg1"]
    f = golden_field("nn64_cfg1")
    plan = make_plan(beamlib, ctx, case, precision="int8")
    a = plan.run(f)
    b = plan.run(2.0 * f)
    plan.close()
    assert np.array_equal(b["count"], a["count"])
    assert np.array_equal(b["norm"], a["norm"])
    assert np.array_equal(b["out"], 8.0 * a["out"], equal_nan=True)


@pytest.mark.parametrize("shards", [2, 3])
def test_int8_shard_partials_add_up(beamlib, ctx, shards):
    """A bispectrum split by ring triplet over shards: each shard's int8 plan
    sums its own triplets (the others' triangles enter as exact zeros), and
    the partial bins add up to the unsharded int8 run up to the rounding of
    the final additions."""
    from barbie_b200 import shard
    case = GOLDEN_CASES["nn96_r20"]
    f = golden_field("nn96_r20")
    whole_plan = make_plan(beamlib, ctx, case, precision="int8")
    whole = whole_plan.run(f)
    parts = []
    for k in range(shards):
        p = make_plan(beamlib, ctx, case, precision="int8", shard=(k, shards))
        parts.append(p.run(f))
        p.close()
    got = shard.sum_partials(parts, whole_plan.info["vol"])
    whole_plan.close()
    assert np.array_equal(got["count"], whole["count"])
    for key in ("bs", "norm"):
        scale = np.maximum(np.abs(whole[key]), sum(np.abs(p[key]) for p in parts))
        assert np.all(np.abs(got[key] - whole[key]) <= 1e-12 * scale), key
