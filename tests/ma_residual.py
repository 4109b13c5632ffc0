"""Residual of the Monge-Ampere problem the time step solves, computed on the
host with numpy from a physical 3-D potential Phi (test infrastructure).

The problem (src/poisson.jl:1-12 on the reference's discretisation):
interior planes k = 1 .. nz-2 satisfy, on the modes the solver keeps
(the 2/3 mask of src/domain.jl:498-514 closed under conjugation),

    Phi_xx + Phi_yy + Phi_zz - eps (Phi_xx Phi_yy - Phi_xy^2) = 0,

with horizontal derivatives spectral (src/poisson.jl:150-205) and Phi_zz the
3-point d2dz2! stencil (src/transforms.jl:812-818); the top plane satisfies
the one-sided Neumann row of apply_neumann_surface! with dPhi/dz = b_s and the
bottom plane that of apply_neumann_bottom! with 0 (src/poisson.jl:309-364).
"""
import numpy as np


def _closed_mask(n):
    nyc = n // 2 + 1
    m = np.ones((n, nyc), dtype=bool)
    kxm = n // 3
    m[kxm:n - kxm, :] = False
    m[:, (2 * nyc) // 3:] = False
    if kxm > 0 and m[n - kxm, 0]:
        m[kxm, 0] = True
    return m


def ma_residual(phi, bs, eps, lx=2 * np.pi, lz=1.0, dz=None):
    """Returns (interior, top, bottom): ||r||_2 / ||b_s||_2 of the projected
    interior equation over the interior planes, of the top Neumann row and of
    the bottom Neumann row, each residual taken as a physical field."""
    phi = np.asarray(phi, dtype=np.float64)
    n, _, nz = phi.shape
    if dz is None:
        dz = np.full(nz, lz / (nz - 1))
    k = 2 * np.pi / lx * np.fft.fftfreq(n, 1.0 / n)
    kx = k[:, None]
    ky = (2 * np.pi / lx * np.arange(n // 2 + 1))[None, :]
    mask = _closed_mask(n)
    ph = np.fft.rfft2(phi, axes=(0, 1))
    ph *= mask[:, :, None]
    bsh = np.fft.rfft2(bs) * mask
    bsh[0, 0] = 0.0
    K2 = kx ** 2 + ky ** 2
    rint = []
    for q in range(1, nz - 1):
        dzm, dzp = dz[q - 1], dz[q]
        al, be, ga = 2 / (dzm * (dzm + dzp)), -2 / (dzm * dzp), 2 / (dzp * (dzm + dzp))
        P = ph[:, :, q]
        xx = np.fft.irfft2(-kx ** 2 * P, s=(n, n))
        yy = np.fft.irfft2(-ky ** 2 * P, s=(n, n))
        xy = np.fft.irfft2(-kx * ky * P, s=(n, n))
        F = np.fft.rfft2(xx * yy - xy * xy) * mask
        r = -K2 * P + al * ph[:, :, q - 1] + be * P + ga * ph[:, :, q + 1] - eps * F
        r[0, 0] = 0.0
        rint.append(np.fft.irfft2(r, s=(n, n)))
    h1, h2 = dz[nz - 2], dz[nz - 3]
    a = h1 + h2
    at, bt, ct = (2 * h1 + h2) / (h1 * a), -a / (h1 * h2), h1 / (h2 * a)
    rt = at * ph[:, :, -1] + bt * ph[:, :, -2] + ct * ph[:, :, -3] - bsh
    rt[0, 0] = 0.0
    h1, h2 = dz[0], dz[1]
    a = h1 + h2
    ab, bb, cb = -(2 * h1 + h2) / (h1 * a), a / (h1 * h2), -h1 / (h2 * a)
    rb = ab * ph[:, :, 0] + bb * ph[:, :, 1] + cb * ph[:, :, 2]
    rb[0, 0] = 0.0
    nb = np.linalg.norm(bs)
    return (float(np.linalg.norm(np.array(rint)) / nb), float(np.linalg.norm(np.fft.irfft2(rt, s=(n, n))) / nb),
            float(np.linalg.norm(np.fft.irfft2(rb, s=(n, n))) / nb))
