"""Seeded initial conditions for the surface buoyancy.

Restates the spectral recipe of ``initialize_jfm_spectral_buoyancy!``
(examples/ssg_example.jl:70-125 in SSG.jl):

    b_hat(k) = A * |k|^(m/4) / (|k| + k0)^(m/2)   with a random phase per mode,

then the 2/3 mask, the inverse real FFT and mean removal.  Two departures,
both needed to make the fields reproducible and comparable:

* the reference draws each phase from Julia's global RNG re-seeded with
  ``seed + 1000*i + j``; that stream cannot be reproduced without Julia, so
  the phase here is a counter-based SplitMix64 hash of (seed, i, j);
* the field is normalised to unit rms (the reference keeps the raw amplitude
  ``A``, which only sets the scale).

The spectrum peaks exactly at |k| = k0 for any m.
"""
import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix64(x):
    """SplitMix64 finaliser on a uint64 array (wrapping arithmetic)."""
    with np.errstate(over="ignore"):
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def mode_uniform(seed, i, j):
    """Uniform [0, 1) draw keyed by (seed, i, j); i, j are 0-based mode indices."""
    with np.errstate(over="ignore"):
        key = (np.uint64(seed) * np.uint64(0x100000001B3)) ^ (np.asarray(i, dtype=np.uint64) << np.uint64(32)) ^ np.asarray(j, dtype=np.uint64)
    z = _splitmix64(_splitmix64(key))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def wavenumbers(nx, ny, lx=2 * np.pi, ly=2 * np.pi):
    """kx, ky as src/domain.jl:155-162 computes them (2pi * fftfreq, rfftfreq)."""
    dx, dy = lx / nx, ly / ny
    fsx, fsy = 1.0 / dx, 1.0 / dy
    nnx = (nx - 1) // 2 + 1
    i = np.arange(nx)
    kx = 2.0 * np.pi * (np.where(i < nnx, i, i - nx).astype(np.float64) * (fsx / nx))
    ky = 2.0 * np.pi * (np.arange(ny // 2 + 1).astype(np.float64) * (fsy / ny))
    return kx, ky


def twothirds_mask(nx, nyc):
    """twothirds_mask(Nx, Nyc), src/domain.jl:498-514 (0-based)."""
    mask = np.ones((nx, nyc), dtype=bool)
    kxm = nx // 3
    mask[kxm:nx - kxm, :] = False
    mask[:, (2 * nyc) // 3:] = False
    return mask


def jfm_spectral_buoyancy(nx, ny, k0, *, m=20, seed=1234, lx=2 * np.pi, ly=2 * np.pi, rms=1.0):
    """Surface buoyancy (nx, ny), Fortran order, zero mean, given rms."""
    kx, ky = wavenumbers(nx, ny, lx, ly)
    KX, KY = np.meshgrid(kx, ky, indexing="ij")
    K = np.sqrt(KX ** 2 + KY ** 2)
    I, J = np.meshgrid(np.arange(nx), np.arange(ny // 2 + 1), indexing="ij")
    phase = 2.0 * np.pi * mode_uniform(seed, I, J)
    with np.errstate(divide="ignore", invalid="ignore"):
        amp = np.where(K > 1e-14, K ** (m / 4.0) / (K + k0) ** (m / 2.0), 0.0)
    bh = amp * (np.cos(phase) + 1j * np.sin(phase))
    bh *= twothirds_mask(nx, ny // 2 + 1)
    b = np.fft.irfft2(bh, s=(nx, ny), axes=(0, 1))
    b -= b.mean()
    b *= rms / np.sqrt(np.mean(b * b))
    return np.asfortranarray(b)


def perturbed_member(nx, ny, k0, seed, member, amplitude=1e-3, **kw):
    """Base field plus an independent unit-rms field of the same spectrum
    scaled by ``amplitude`` (ensemble members)."""
    base = jfm_spectral_buoyancy(nx, ny, k0, seed=seed, **kw)
    pert = jfm_spectral_buoyancy(nx, ny, k0, seed=seed + 7919 * (member + 1), **kw)
    return np.asfortranarray(base + amplitude * pert)
