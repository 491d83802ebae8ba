"""Seeded synthetic input fields in the estimator's input format.

The reference reads ``field_N<NN>_R<NRi>.txt``: raw native-endian float64 in
the FFTW in-place r2c layout ``double[NN][NN][NN+2]`` =
``complex128[NN][NN][NN/2+1]`` with the last axis (k_z >= 0) along the line of
sight (barbie.c:176-185). No public dataset is involved; this module makes the
non-Gaussian redshift-space test field used by the tests and the benchmark:

* a real Gaussian field delta(x) whose spectrum is P(k) = A k^-1.5 exp(-(k/k_c)^2),
  k_c = 0.5 k_Nyquist, with A set so the real-space cell variance is 1;
* a quadratic term delta -> delta + f (delta^2 - <delta^2>), f = 0.5;
* the r2c transform times the cell volume LL^3 (LL = 0.56);
* Kaiser redshift-space distortion along z: (1 + beta mu_k^2) with beta = 0.5,
  and the k = 0 mode set to zero.

Seeds follow 100020 + 146 * r for realization r. The generator uses numpy's
PCG64 stream and numpy's FFT, so a given (NN, seed) gives the same bytes on any
x86-64 host running this image (the tests pin a checksum of the NN=64 field).
"""
from __future__ import annotations

import numpy as np

DEFAULT_LL = 0.56
DEFAULT_QUAD = 0.5
DEFAULT_KAISER = 0.5
DEFAULT_SLOPE = -1.5


def realization_seed(r: int) -> int:
    return 100020 + 146 * r


def synth_field(NN: int, seed: int, LL: float = DEFAULT_LL, quad: float = DEFAULT_QUAD,
                kaiser: float = DEFAULT_KAISER, slope: float = DEFAULT_SLOPE) -> np.ndarray:
    """Return the float64 r2c buffer of shape (NN, NN, NN+2)."""
    if NN <= 0 or NN % 2:
        raise ValueError("NN must be a positive even integer")
    rng = np.random.Generator(np.random.PCG64(seed))
    white = rng.standard_normal((NN, NN, NN))
    W = np.fft.rfftn(white)
    del white
    kx = 2.0 * np.pi * np.fft.fftfreq(NN, d=LL)
    kz = 2.0 * np.pi * np.fft.rfftfreq(NN, d=LL)
    k2 = kx[:, None, None] ** 2 + kx[None, :, None] ** 2 + kz[None, None, :] ** 2
    k = np.sqrt(k2)
    kc = 0.5 * np.pi / LL
    with np.errstate(divide="ignore"):
        amp = np.where(k > 0, k ** (0.5 * slope) * np.exp(-0.5 * (k / kc) ** 2), 0.0)
    delta = np.fft.irfftn(W * amp, s=(NN, NN, NN), axes=(0, 1, 2))
    del W
    delta /= np.sqrt(np.mean(delta * delta))
    d2 = delta * delta
    delta += quad * (d2 - d2.mean())
    del d2
    D = np.fft.rfftn(delta) * LL ** 3
    del delta
    with np.errstate(invalid="ignore", divide="ignore"):
        mu2 = np.where(k2 > 0, kz[None, None, :] ** 2 / k2, 0.0)
    D *= 1.0 + kaiser * mu2
    D[0, 0, 0] = 0.0
    buf = np.empty((NN, NN, NN + 2), dtype=np.float64)
    buf.view(np.complex128)[...] = D
    return buf


def synth_field_torch(NN: int, seed: int, device="cuda", LL: float = DEFAULT_LL, quad: float = DEFAULT_QUAD,
                      kaiser: float = DEFAULT_KAISER, slope: float = DEFAULT_SLOPE):
    """The same recipe as synth_field with torch (on a GPU, milliseconds per
    field at NN=256 instead of seconds): a torch tensor of shape (NN, NN, NN+2),
    float64, on `device`. The white noise comes from torch's generator seeded
    with `seed`, so the fields differ from synth_field's for the same seed but
    share their spectrum, non-Gaussian term and distortion."""
    import torch
    if NN <= 0 or NN % 2:
        raise ValueError("NN must be a positive even integer")
    dev = torch.device(device)
    g = torch.Generator(device=dev).manual_seed(int(seed))
    W = torch.fft.rfftn(torch.randn((NN, NN, NN), dtype=torch.float64, device=dev, generator=g))
    kx = 2.0 * np.pi * torch.fft.fftfreq(NN, d=LL, dtype=torch.float64, device=dev)
    kz = 2.0 * np.pi * torch.fft.rfftfreq(NN, d=LL, dtype=torch.float64, device=dev)
    k2 = kx[:, None, None] ** 2 + kx[None, :, None] ** 2 + kz[None, None, :] ** 2
    k = torch.sqrt(k2)
    kc = 0.5 * np.pi / LL
    pos = k > 0
    amp = torch.where(pos, torch.where(pos, k, 1.0) ** (0.5 * slope) * torch.exp(-0.5 * (k / kc) ** 2),
                      torch.zeros_like(k))
    delta = torch.fft.irfftn(W * amp, s=(NN, NN, NN))
    del W, amp
    delta /= torch.sqrt(torch.mean(delta * delta))
    d2 = delta * delta
    delta += quad * (d2 - d2.mean())
    del d2
    D = torch.fft.rfftn(delta) * LL ** 3
    del delta
    mu2 = torch.where(pos, kz[None, None, :] ** 2 / torch.where(pos, k2, 1.0), torch.zeros_like(k2))
    D *= 1.0 + kaiser * mu2
    D[0, 0, 0] = 0.0
    return torch.view_as_real(D).reshape(NN, NN, NN + 2).contiguous()


def write_field(path: str, buf: np.ndarray) -> None:
    """Write the buffer as the reference's raw native-double field file."""
    np.ascontiguousarray(buf, dtype=np.float64).tofile(path)


def read_field(path: str, NN: int) -> np.ndarray:
    buf = np.fromfile(path, dtype=np.float64)
    if buf.size != NN * NN * (NN + 2):
        raise ValueError(f"{path}: expected {NN * NN * (NN + 2)} doubles, found {buf.size}")
    return buf.reshape(NN, NN, NN + 2)
