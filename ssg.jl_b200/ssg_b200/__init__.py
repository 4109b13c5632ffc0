"""ssg_b200 -- SSG.jl's time-step path on one NVIDIA B200.

Public names mirror SSG.jl's exports (src/SSG.jl:41-80) with ``!`` spelled
``_``.  The compute runs in libssg_b200.so (hand-written sm_100a kernels, C ABI
in include/ssg_b200.h); this package is the host-side API over it.
"""
from . import _lib, adjoint, filter, ic
from .api import (AB2_LowStorage, RK3, RK3_LowStorage, DiagnosticTimeSeries, Domain, Fields,
                  SemiGeostrophicProblem, TimeParams, TimeState, apply_spectral_filter_,
                  compute_surface_geostrophic_velocities_, create_stretched_grid, diagnostics, install_filter_,
                  load_simulation_state_full, make_domain, make_vertical_grid, save_simulation_state_full, set_b_,
                  solve_monge_ampere_fields_, step_until_, stepforward_, timestep_, update_diagnostics_)
from .filter import (CesaroFilter, CustomFilter, CutoffFilter, ExponentialFilter, HyperviscosityFilter,
                     cesaro_transfer, cutoff_transfer, custom_transfer, exponential_transfer,
                     hyperviscosity_transfer)
from ._lib import SsgError
from .multigrid import SSGMultigrid, solve_ssg_equation
from .ic import jfm_spectral_buoyancy, twothirds_mask

__all__ = [
    "AB2_LowStorage", "RK3", "RK3_LowStorage", "DiagnosticTimeSeries", "Domain", "Fields",
    "SemiGeostrophicProblem", "TimeParams", "TimeState", "compute_surface_geostrophic_velocities_",
    "make_domain", "set_b_", "solve_monge_ampere_fields_", "step_until_", "stepforward_", "timestep_",
    "update_diagnostics_", "SsgError", "jfm_spectral_buoyancy", "twothirds_mask", "ic",
    "apply_spectral_filter_", "install_filter_", "filter", "ExponentialFilter", "HyperviscosityFilter",
    "CutoffFilter", "CesaroFilter", "CustomFilter", "exponential_transfer", "hyperviscosity_transfer",
    "cutoff_transfer", "cesaro_transfer", "custom_transfer", "diagnostics", "save_simulation_state_full",
    "load_simulation_state_full", "SSGMultigrid", "solve_ssg_equation", "adjoint", "make_vertical_grid",
    "create_stretched_grid",
]
