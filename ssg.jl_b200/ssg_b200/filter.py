"""Spectral filters (src/filter.jl:36-177): the reference's filter types and
transfer functions.  A problem applies one of them every ``filter_freq``
steps inside its fused stage kernel; ``apply_spectral_filter_`` applies it
once.  Every filter reaches the device as a table of transfer values on the
dealiased modes, so a ``CustomFilter`` costs the same as the built-in ones."""
import math

import numpy as np


class AbstractSpectralFilter:
    pass


class ExponentialFilter(AbstractSpectralFilter):
    """exp(-strength * ((k_norm - cutoff)/(1 - cutoff))^order) above cutoff."""

    def __init__(self, strength=1.0, order=4, cutoff=0.65):
        assert strength >= 0, "Filter strength must be non-negative"
        assert order >= 1, "Filter order must be positive"
        assert 0 < cutoff <= 1, "Cutoff must be between 0 and 1"
        self.strength, self.order, self.cutoff = float(strength), int(order), float(cutoff)


class HyperviscosityFilter(AbstractSpectralFilter):
    """exp(-coefficient * |k|^(2 order) * dt)."""

    def __init__(self, coefficient, order=2):
        assert coefficient >= 0, "Hyperviscosity coefficient must be non-negative"
        assert order >= 1, "Hyperviscosity order must be positive"
        self.coefficient, self.order = float(coefficient), int(order)


class CutoffFilter(AbstractSpectralFilter):
    def __init__(self, cutoff=2.0 / 3.0):
        assert 0 < cutoff <= 1, "Cutoff must be between 0 and 1"
        self.cutoff = float(cutoff)


class CesaroFilter(AbstractSpectralFilter):
    def __init__(self, cutoff=0.5, order=2):
        assert 0 < cutoff <= 1, "Cutoff must be between 0 and 1"
        assert order >= 1, "Cesaro order must be positive"
        self.cutoff, self.order = float(cutoff), int(order)


class CustomFilter(AbstractSpectralFilter):
    """transfer_function(k_norm, k_x, k_y, **parameters) -> transfer value."""

    def __init__(self, transfer_function, parameters=None):
        self.transfer_function = transfer_function
        self.parameters = dict(parameters or {})


def exponential_transfer(k_norm, f):
    if k_norm <= f.cutoff:
        return 1.0
    ratio = (k_norm - f.cutoff) / (1.0 - f.cutoff)
    return math.exp(-f.strength * ratio ** f.order)


def hyperviscosity_transfer(k_mag, dt, f):
    return math.exp(-f.coefficient * k_mag ** (2 * f.order) * dt)


def cutoff_transfer(k_norm, f):
    return 1.0 if k_norm <= f.cutoff else 0.0


def cesaro_transfer(k_norm, f):
    if k_norm <= f.cutoff:
        return 1.0
    if k_norm >= 1.0:
        return 0.0
    ratio = (k_norm - f.cutoff) / (1.0 - f.cutoff)
    return (1.0 - ratio) ** f.order


def custom_transfer(k_norm, k_x, k_y, f):
    return f.transfer_function(k_norm, k_x, k_y, **f.parameters)


def transfer_table(domain, f, dt=None):
    """Transfer values on the reference's (Nx, Nyc) spectral grid."""
    KX, KY = np.meshgrid(domain.kx, domain.ky, indexing="ij")
    dx, dy = domain.Lx / domain.Nx, domain.Ly / domain.Ny
    kmax = math.sqrt((math.pi / dx) ** 2 + (math.pi / dy) ** 2)
    kmag = np.sqrt(KX ** 2 + KY ** 2)
    kn = kmag / kmax
    if isinstance(f, ExponentialFilter):
        r = np.clip((kn - f.cutoff) / (1.0 - f.cutoff), 0.0, None) if f.cutoff < 1 else np.zeros_like(kn)
        tab = np.where(kn <= f.cutoff, 1.0, np.exp(-f.strength * r ** f.order))
    elif isinstance(f, HyperviscosityFilter):
        if dt is None:
            raise ValueError("Hyperviscosity filter requires time step dt")
        tab = np.exp(-f.coefficient * kmag ** (2 * f.order) * dt)
    elif isinstance(f, CutoffFilter):
        tab = np.where(kn <= f.cutoff, 1.0, 0.0)
    elif isinstance(f, CesaroFilter):
        r = np.clip((kn - f.cutoff) / (1.0 - f.cutoff), 0.0, 1.0)
        tab = np.where(kn <= f.cutoff, 1.0, np.where(kn >= 1.0, 0.0, (1.0 - r) ** f.order))
    elif isinstance(f, CustomFilter):
        tab = np.vectorize(lambda a, b, c: custom_transfer(a, b, c, f))(kn, KX, KY)
    else:
        raise ValueError(f"Unknown filter type: {type(f)}")
    return np.asfortranarray(tab.astype(np.float64))
