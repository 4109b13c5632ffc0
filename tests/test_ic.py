"""Seeded spectral initial condition (examples/ssg_example.jl:70-125 recipe)."""
import numpy as np


def test_ic_statistics_and_band_limit(ssg):
    n = 128
    b = ssg.jfm_spectral_buoyancy(n, n, 6, seed=1)
    assert b.shape == (n, n) and b.flags.f_contiguous
    assert abs(b.mean()) < 1e-15
    assert abs(np.sqrt(np.mean(b * b)) - 1.0) < 1e-14
    bh = np.fft.rfft2(b, axes=(0, 1))
    mask = ssg.twothirds_mask(n, n // 2 + 1)
    mask[n // 3, 0] = True  # conjugate partner of (-n/3, 0) in a real field
    assert np.abs(bh[~mask]).max() < 1e-12 * np.abs(bh).max()


def test_ic_spectrum_peaks_at_k0(ssg):
    n, k0 = 256, 10
    b = ssg.jfm_spectral_buoyancy(n, n, k0, seed=3)
    bh = np.fft.rfft2(b, axes=(0, 1))
    kx, ky = ssg.ic.wavenumbers(n, n)
    K = np.sqrt(kx[:, None] ** 2 + ky[None, :] ** 2)
    shells = np.bincount(np.round(K).astype(int).ravel(), weights=(np.abs(bh) ** 2).ravel())
    counts = np.bincount(np.round(K).astype(int).ravel())
    per_mode = shells / np.maximum(counts, 1)
    assert abs(int(np.argmax(per_mode)) - k0) <= 1


def test_ic_deterministic_and_seeded(ssg):
    a = ssg.jfm_spectral_buoyancy(64, 64, 5, seed=9)
    b = ssg.jfm_spectral_buoyancy(64, 64, 5, seed=9)
    c = ssg.jfm_spectral_buoyancy(64, 64, 5, seed=10)
    assert np.array_equal(a, b)
    assert np.abs(a - c).max() > 0.1
