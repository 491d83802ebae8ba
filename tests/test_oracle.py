"""The oracle (CPU restatement of the reference) pinned against the reference's
own outputs (golden fixtures) and against independent definitions."""
import hashlib

import numpy as np
import pytest

from conftest import GOLDEN_CASES, compare_to_golden, golden_field, load_golden


def reference_cal_coeff(px, pz):
    """funcs.c:710-744 written out term by term as the reference states them."""
    s = np.sqrt
    bs = [1.0,
          2. * (3. * pz * pz - 1.),
          -s(2. / 3.) * px * pz,
          2. * s(0.6666666666666666) * (-1. + 2. * px ** 2 + pz ** 2),
          8. * (3. - 30. * pz ** 2 + 35. * pz ** 4),
          (-4. * px * pz * (-3. + 7. * pz ** 2)) / s(5.),
          4. * s(0.4) * (-1 + 2. * px ** 2 + pz ** 2) * (-1. + 7. * pz ** 2),
          (-4. * px * pz * (-3. + 4. * px ** 2 + 3. * pz ** 2)) / s(35.),
          8. * s(0.05714285714285714) * (8. * px ** 4 + 8. * px ** 2 * (-1. + pz ** 2) + (-1. + pz ** 2) ** 2),
          16. * (-5. + 105. * pz ** 2 - 315. * pz ** 4 + 231. * pz ** 6),
          -8. * s(0.09523809523809523) * px * pz * (5. - 30. * pz ** 2 + 33. * pz ** 4),
          (32. * (-1. + 2. * px ** 2 + pz ** 2) * (1. - 18. * pz ** 2 + 33. * pz ** 4)) / s(105.0),
          (-16. * px * pz * (-3. + 4. * px ** 2 + 3. * pz ** 2) * (-3. + 11. * pz ** 2)) / s(105.0),
          (16. * s(0.2857142857142857) * (-1. + 11. * pz ** 2)
           * (8. * px ** 4 + 8. * px ** 2 * (-1. + pz ** 2) + (-1. + pz ** 2) ** 2)) / 3.,
          (-16 * pz * (16 * px ** 5 + 20 * px ** 3 * (-1 + pz ** 2) + 5 * px * (-1 + pz ** 2) ** 2)) / (3. * s(77.0)),
          (32. * (32. * px ** 6 + 48. * px ** 4 * (-1. + pz ** 2) + 18. * px ** 2 * (-1. + pz ** 2) ** 2
                  + (-1. + pz ** 2) ** 3.)) / s(231.)]
    nm = [1.,
          (3. * pz * pz - 1.) ** 2,
          pz * pz * (1. - pz * pz),
          (-1. + pz ** 2) ** 2,
          (3. - 30. * pz ** 2 + 35. * pz ** 4) ** 2,
          (1. - pz ** 2) * (-3. * pz + 7. * pz ** 3) ** 2,
          (-1. + pz ** 2) ** 2 * (-1. + 7. * pz ** 2) ** 2,
          pz ** 2 * (1. - pz ** 2) ** 3,
          (-1. + pz ** 2) ** 4,
          (-5. + 105. * pz ** 2 - 315. * pz ** 4 + 231. * pz ** 6) ** 2,
          (1. - pz ** 2) * (5. * pz - 30. * pz ** 3 + 33. * pz ** 5) ** 2,
          (-1. + pz ** 2) ** 2 * (1. - 18. * pz ** 2 + 33. * pz ** 4) ** 2,
          (1. - pz ** 2) ** 3 * (-3. * pz + 11. * pz ** 3) ** 2,
          (-1 + pz ** 2) ** 4 * (-1 + 11 * pz ** 2) ** 2,
          pz ** 2 * (1 - pz ** 2) ** 5,
          (-1. + pz ** 2) ** 6]
    return np.array(bs), np.array(nm)


def test_cal_coeff_matches_reference_formulas(oracle):
    rng = np.random.default_rng(7)
    for _ in range(500):
        pz = rng.uniform(-1, 1)
        px = rng.uniform(-1, 1) * np.sqrt(1 - pz * pz)
        bs, nm = oracle.cal_coeff(px, pz)
        rbs, rnm = reference_cal_coeff(px, pz)
        # the polynomials have coefficients up to ~1e4, so both evaluations carry
        # absolute rounding errors of a few 1e-12 for |px|, |pz| <= 1
        assert np.all(np.abs(bs - rbs) <= 1e-11 + 1e-13 * np.abs(rbs))
        assert np.all(np.abs(nm - rnm) <= 1e-11 + 1e-13 * np.abs(rnm))


@pytest.mark.parametrize("n0,n1", [(64, 64), (96, 96), (48, 72), (10, 14)])
def test_oracle_fft_is_unnormalised_backward_dft(oracle, n0, n1):
    rng = np.random.default_rng(n0 * 1000 + n1)
    a = rng.standard_normal((n0, n1)) + 1j * rng.standard_normal((n0, n1))
    got = oracle.fft2_backward(a)
    want = np.fft.ifft2(a) * (n0 * n1)
    assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))


def test_ring_edges_reference_values(oracle):
    low, high, avg = oracle.ring_edges(10, 16)
    assert np.allclose(low, [0, .9, 1.9, 2.9, 3.9, 4.9, 5.9, 6.9, 7.9, 8.9], rtol=0, atol=1e-15)
    assert np.allclose(high, [.9, 1.9, 2.9, 3.9, 4.9, 5.9, 6.9, 7.9, 8.9, 16], rtol=0, atol=1e-15)
    low, high, avg = oracle.ring_edges(40, 100)
    assert low[10] == 10 - .1 and low[20] == 30 - .1 and low[30] == 60 - .1
    assert high[39] == 100 and abs(low[39] - 95.9) < 1e-12
    assert np.all(avg == (high + low) / 2.)
    with pytest.raises(ValueError):
        oracle.ring_edges(15, 16)


def test_closed_ring_counts_are_exact_integers(oracle):
    NN, Nmax, Nr = 64, 16, 10
    rings = oracle.closed_rings(NN, Nr, Nmax)
    assert len(rings) == 110  # calCR's rcount at config 1
    c = rings[:, 3] / NN ** 2
    assert np.max(np.abs(c - np.rint(c))) < 1e-6
    RR = oracle.ring_masks(NN, Nr, Nmax)
    for k in range(0, len(rings), 9):
        r1, r2, r3 = (int(v) for v in rings[k, :3])
        assert oracle.triangle_count_direct(NN, RR, r1, r2, r3) == int(np.rint(c[k]))


def test_enumeration_counts(oracle):
    tri, _ = oracle.enumerate_triples(64, 16, 10, 11, 1, 1)
    assert len(tri) == 8340
    assert np.all((tri["t_bin"] >= 0) & (tri["t_bin"] < 5) & (tri["mu_bin"] >= 0) & (tri["mu_bin"] < 5))


@pytest.mark.parametrize("name", ["nn64_cfg1", "nn64_bw2", "nn96_r20"])
def test_field_generator_is_pinned(name):
    g = load_golden(name)
    assert hashlib.sha256(golden_field(name).tobytes()).hexdigest() == g["sha"]


@pytest.mark.parametrize("name", ["nn64_cfg1", "nn64_bw2", "nn96_r20"])
def test_oracle_matches_reference_outputs(oracle, name):
    g = load_golden(name)
    NN, Nmax, Nr, UL, LL, BW, _ = GOLDEN_CASES[name]
    res = oracle.estimate(golden_field(name), NN, Nmax, Nr, UL, LL, BW, nthreads=4)
    # the oracle uses calCR's own Num, so its analytic column meets the 1e-10 bar
    compare_to_golden(g["rows"], res["out"], res["norm"], NN, rtol=1e-10, ana=res["ana_out"], ana_rtol=1e-10)
    rows0 = g["rows"][g["rows"][:, 0] == 0]
    for r in rows0:
        assert res["counts"][int(r[1]), int(r[2]), int(r[3])] == int(np.rint(r[5]))


def load_pk(name):
    import os
    from conftest import GOLDEN
    path = os.path.join(GOLDEN, f"pk_{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"power-spectrum fixture {name} not generated")
    return np.load(path)["pk"]


@pytest.mark.parametrize("name", ["nn64_cfg1", "nn96_r20"])
def test_oracle_power_multipoles_match_reference(oracle, name):
    """The restatement of calpow_mom (funcs.c:860-1074) against the reference
    program's own output on the same field: bit for bit (same libm, same float
    and double types)."""
    NN = GOLDEN_CASES[name][0]
    ref = load_pk(name)
    got = oracle.power_multipoles(golden_field(name), NN, LL=0.56, Nbin=10)
    mine = np.stack([got[c] for c in ("k", "P0", "P2", "P4", "P6", "count")], axis=1)
    mine = mine[mine[:, 5] > 0]
    assert mine.shape == ref.shape
    assert np.array_equal(mine, ref)
