"""Seeded random media for the layered model (the lhm_rmed perturbation).

The reference reads a precomputed random-medium file per layer
(src/swpc_3d/m_vmodel_lhm_rmed.f90:138) generated by gen_rmed3d with the
von Karman power spectral density of src/shared/m_rmedia.f90:667-679,
seeded through the compiler's random_number.  Realisations therefore depend
on the Fortran compiler; here the field is generated once from a numpy seed
by spectral filtering of white noise (FFT on the GPU through torch when one
is present, numpy otherwise) and the same array feeds every consumer.

PSD (3D von Karman): P(m) ~ eps^2 a^3 / (1 + m^2 a^2)^(kappa + 3/2),
m the wavenumber magnitude; the field is scaled to standard deviation eps.
"""
from __future__ import annotations

import numpy as np


def vonkarman_3d(shape_kij: tuple[int, int, int], dx: float, dy: float, dz: float, eps: float, a: float,
                 kappa: float, seed: int, device: str | None = None) -> np.ndarray:
    """Return a float32 field of shape (nj, ni, nk) (numpy view of the
    Fortran (k, i, j) memory box) with zero mean and std ``eps``."""
    nj, ni, nk = shape_kij
    rng = np.random.default_rng(seed)
    white = rng.standard_normal((nj, ni, nk), dtype=np.float32)
    try:
        import torch

        dev = device or ("cuda" if torch.cuda.is_available() else "cpu")
        w = torch.from_numpy(white).to(dev)
        del white
        spec = torch.fft.rfftn(w)
        del w
        mj = torch.fft.fftfreq(nj, d=dy, device=dev) * (2 * np.pi)
        mi = torch.fft.fftfreq(ni, d=dx, device=dev) * (2 * np.pi)
        mk = torch.fft.rfftfreq(nk, d=dz, device=dev) * (2 * np.pi)
        m2 = mj[:, None, None] ** 2 + mi[None, :, None] ** 2 + mk[None, None, :] ** 2
        amp = (1.0 + m2 * (a * a)) ** (-(kappa + 1.5) / 2.0)
        del m2
        spec *= amp
        del amp
        x = torch.fft.irfftn(spec, s=(nj, ni, nk))
        del spec
        x -= x.mean()
        x *= eps / x.std()
        out = x.to(torch.float32).cpu().numpy()
        del x
        if dev.startswith("cuda"):
            torch.cuda.empty_cache()
        return out
    except ImportError:
        spec = np.fft.rfftn(white)
        mj = np.fft.fftfreq(nj, d=dy) * (2 * np.pi)
        mi = np.fft.fftfreq(ni, d=dx) * (2 * np.pi)
        mk = np.fft.rfftfreq(nk, d=dz) * (2 * np.pi)
        m2 = mj[:, None, None] ** 2 + mi[None, :, None] ** 2 + mk[None, None, :] ** 2
        spec *= (1.0 + m2 * (a * a)) ** (-(kappa + 1.5) / 2.0)
        x = np.fft.irfftn(spec, s=(nj, ni, nk))
        x -= x.mean()
        x *= eps / x.std()
        return x.astype(np.float32)
