"""GPU tests of the batched and sharded forms of the estimator, through the
C ABI. Needs an sm_100a device.

- Batches (beam_gpu_run_batch_ex): every kernel of a batch covers all of its
  realizations and the batch runs as a replayed CUDA graph; each realization's
  bins must equal a single beam_gpu_run bit for bit, for ragged last batches,
  both alternating batch buffers and both precisions.
- Shards (beam_cfg.shard_index/shard_count): the partial bins of all shards,
  added on the host, must equal the whole estimator -- counts exactly, bs and
  norm to 1e-12 relative (only the order of the final additions differs)."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, golden_field

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(beamlib):
    c = beamlib.Context(0)
    yield c
    c.close()


def make_plan(beamlib, ctx, name, **kw):
    NN, Nmax, Nr, UL, LL, BW, _ = GOLDEN_CASES[name]
    return beamlib.Plan(ctx, NN, UL, LL, BW, Nmax=Nmax, Nr=Nr, **kw)


def fields_for(name, seeds):
    from barbie_b200.synth import realization_seed, synth_field
    return [synth_field(GOLDEN_CASES[name][0], realization_seed(r)) for r in seeds]


def assert_same(got, want):
    for k in want:
        assert np.array_equal(got[k], want[k], equal_nan=True), k


@pytest.mark.parametrize("precision,batch", [("fp64", 2), ("fp64", 0), ("mixed", 3)])
def test_batches_equal_single_runs_bit_for_bit(beamlib, ctx, precision, batch):
    name = "nn96_r20"
    plan = make_plan(beamlib, ctx, name, precision=precision)
    fields = fields_for(name, range(11, 16))  # 5 realizations: batches of 2 -> 2, 2, 1 over both buffers
    got = plan.run_batch(fields, batch=batch)
    for f, g in zip(fields, got):
        assert_same(g, plan.run(f))
    # a second call replays the captured graphs
    again = plan.run_batch(fields, batch=batch)
    for g, h in zip(got, again):
        assert_same(h, g)
    plan.close()


def test_batch_of_golden_field_matches_golden_run(beamlib, ctx):
    name = "nn256_cfg2"
    plan = make_plan(beamlib, ctx, name)
    f = golden_field(name)
    (got,) = plan.run_batch([f], batch=1)
    assert_same(got, plan.run(f))
    plan.close()


@pytest.mark.parametrize("shards", [2, 3])
def test_shard_partials_add_up_to_the_whole_estimator(beamlib, ctx, shards):
    from barbie_b200 import shard
    name = "nn96_r20"
    f = golden_field(name)
    whole_plan = make_plan(beamlib, ctx, name)
    whole = whole_plan.run(f)
    total_terms = whole_plan.info["n_fourier_terms"]
    parts, terms = [], 0
    for k in range(shards):
        p = make_plan(beamlib, ctx, name, shard=(k, shards))
        assert p.info["n_fourier_terms"] == total_terms
        assert 0 < p.info["n_shard_terms"] < total_terms
        terms += p.info["n_shard_terms"]
        parts.append(p.run(f))
        p.close()
    assert terms == total_terms
    got = shard.sum_partials(parts, whole_plan.info["vol"])
    assert np.array_equal(got["count"], whole["count"])
    # Non-owned triangles enter a shard's epilogue as exact zeros, so each
    # partial is the whole estimator's reduction with some terms zeroed; the
    # only new rounding is in adding the partials, bounded by eps * sum |partials|.
    for key in ("bs", "norm"):
        scale = np.maximum(np.abs(whole[key]), sum(np.abs(p[key]) for p in parts))
        assert np.all(np.abs(got[key] - whole[key]) <= 1e-12 * scale), key
    ok = whole["norm"][..., 0] > 0.1
    rel_bs = np.abs(got["bs"] - whole["bs"])[ok] / np.maximum(np.abs(whole["bs"][ok]), 1e-300)
    print(f"{shards} shards: median rel diff of bs {np.median(rel_bs):.1e}, max {rel_bs.max():.1e}")
    whole_plan.close()


def test_shard_arguments_are_checked(beamlib, ctx):
    with pytest.raises(beamlib.BeamError):
        make_plan(beamlib, ctx, "nn64_cfg1", shard=(2, 2))
    with pytest.raises(beamlib.BeamError):
        make_plan(beamlib, ctx, "nn64_cfg1", shard=(0, 2), method="pixel")


def test_launch_count_is_reported(beamlib, ctx):
    plan = make_plan(beamlib, ctx, "nn96_r20")
    plan.run(golden_field("nn96_r20"))
    n = plan.refresh_info()["launches_last_run"]
    # mode build + 1..7 triangle-sum classes + split reduction + 2 epilogue passes
    assert 5 <= n <= 11
    plan.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_persistent_launch_equals_class_launches(beamlib, ctx, precision):
    """One persistent launch of every tile class and realization gives the bins
    of the per-class launches bit for bit, single runs and batches (the same
    units sum the same triangles in the same order), and switching the mode back
    and forth recaptures the batch graphs."""
    name = "nn256_cfg2"
    plan = make_plan(beamlib, ctx, name, precision=precision)
    fields = fields_for(name, range(21, 24))
    want = [plan.run(f) for f in fields]
    want_batch = plan.run_batch(fields, batch=2)
    plan.set_triangle_launch("persistent")
    for f, w in zip(fields, want):
        assert_same(plan.run(f), w)
    for g, w in zip(plan.run_batch(fields, batch=2), want_batch):
        assert_same(g, w)
    assert plan.refresh_info()["launches_last_run"] < 8  # mode build, one triangle launch, reduction, epilogue
    plan.set_triangle_launch("classes")
    for g, w in zip(plan.run_batch(fields, batch=2), want_batch):
        assert_same(g, w)
    plan.close()
