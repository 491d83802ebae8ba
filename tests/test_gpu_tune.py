"""Autotuning (beam_gpu_plan_autotune, beam_gpu_field_autotune) through the C
ABI: the tuned plan still matches the reference's outputs at 1e-10 and the
untuned plan to round-off; tuned field transforms are bit-identical. Needs an
sm_100a device."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, compare_to_golden, golden_field, load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(beamlib):
    c = beamlib.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed", "int8"])
def test_plan_autotune_keeps_parity(beamlib, ctx, precision):
    name = "nn96_r20"
    NN, Nmax, Nr, UL, LL, BW, _ = GOLDEN_CASES[name]
    f = golden_field(name)
    plan = beamlib.Plan(ctx, NN, UL, LL, BW, Nmax=Nmax, Nr=Nr, precision=precision)
    before = plan.run(f)
    rep = plan.autotune(reps=2)
    assert len(rep["candidates"]) == 12
    assert all(c["ms"] > 0 and c["items"] > 0 for c in rep["candidates"])
    assert rep["best"]["ms"] == min(c["ms"] for c in rep["candidates"])
    after = plan.run(f)
    assert np.array_equal(before["count"], after["count"])
    ok = before["norm"][..., 0] > 0.1
    a, b = after["bs"][ok], before["bs"][ok]
    scale = np.abs(b).max()
    tol = 1e-12 if precision == "fp64" else 1e-10  # only the order of FP64 partial sums changes
    assert np.abs(a - b).max() <= tol * scale
    if precision != "mixed":
        g = load_golden(name)
        rtol = 1e-10 if precision == "fp64" else 1e-5  # int8: the 1e-5 bar per printed bin
        compare_to_golden(g["rows"], after["out"], after["norm"], NN, rtol=rtol, ana=after["ana"] if rtol == 1e-10 else None)
    again = plan.run(f)
    for k in after:
        assert np.array_equal(after[k], again[k], equal_nan=True), k
    plan.close()


def test_field_autotune_is_bit_identical(beamlib, ctx):
    NN = 96
    a, sa = beamlib.generate_field(ctx, NN, 3)
    rep = beamlib.field_autotune(ctx, NN)
    assert len(rep["candidates"]) == 3
    assert rep["cols_tile"] in (768, 1536, 3072) and rep["rows_tile"] in (768, 1536, 3072)
    b, sb = beamlib.generate_field(ctx, NN, 3)
    assert np.array_equal(a, b) and sa == sb
