"""The synthetic field recipe (barbie_b200/synth.py), CPU only: the torch form
used to make many fields quickly has the numpy form's layout and spectrum."""
import numpy as np
import pytest

from barbie_b200.synth import realization_seed, synth_field, synth_field_torch


def test_torch_recipe_matches_numpy_recipe_in_distribution():
    torch = pytest.importorskip("torch")
    NN = 48
    a = np.stack([synth_field(NN, realization_seed(r)) for r in (1, 2, 3)]).view(np.complex128)
    b = np.stack([synth_field_torch(NN, realization_seed(r), device="cpu").numpy() for r in (1, 2, 3)])
    assert b.shape == (3, NN, NN, NN + 2) and b.dtype == np.float64
    b = b.view(np.complex128)
    assert np.all(b[:, 0, 0, 0] == 0)
    # a real field's r2c buffer: the round trip through real space returns it
    x = np.fft.irfftn(b[0], s=(NN, NN, NN), axes=(0, 1, 2))
    assert np.abs(np.fft.rfftn(x) - b[0]).max() <= 1e-12 * np.abs(b[0]).max()
    # the same power per |k| shell, to the scatter of three realizations
    i = np.minimum(np.arange(NN), NN - np.arange(NN))
    kz = np.arange(NN // 2 + 1)
    kk = np.rint(np.sqrt(i[:, None, None] ** 2 + i[None, :, None] ** 2 + kz[None, None, :] ** 2)).astype(int)
    for s in (5, 8, 12, 16, 20):
        m = kk == s
        ratio = np.mean(np.abs(b[:, m]) ** 2) / np.mean(np.abs(a[:, m]) ** 2)
        assert 0.8 < ratio < 1.25, (s, ratio)
    # seeded: the same seed gives the same bytes, another seed another field
    again = synth_field_torch(NN, realization_seed(1), device="cpu").numpy().view(np.complex128)
    assert np.array_equal(again, b[0])
    assert not np.array_equal(b[0], b[1])
