"""Filter types and transfer functions (src/filter.jl), host side.  Restates
the scalar checks of test/test_filter.jl:43-74 and compares the transfer
tables the GPU receives with the oracle's filtering."""
import math

import numpy as np
import pytest


def test_transfer_function_kats(ssg):
    f = ssg.ExponentialFilter(1.0, 2, 0.5)
    assert ssg.exponential_transfer(0.3, f) == 1.0
    assert 0.0 < ssg.exponential_transfer(0.8, f) < 1.0
    h = ssg.HyperviscosityFilter(1e-3, 1)
    assert abs(ssg.hyperviscosity_transfer(2.0, 0.01, h) - math.exp(-1e-3 * 2.0 ** 2 * 0.01)) < 1e-14
    c = ssg.CutoffFilter(0.6)
    assert ssg.cutoff_transfer(0.4, c) == 1.0 and ssg.cutoff_transfer(0.8, c) == 0.0
    ce = ssg.CesaroFilter(0.5, 2)
    assert ssg.cesaro_transfer(0.4, ce) == 1.0 and ssg.cesaro_transfer(1.0, ce) == 0.0
    assert ssg.cesaro_transfer(0.75, ce) == pytest.approx(0.25)


@pytest.mark.parametrize("bad", [lambda s: s.ExponentialFilter(-1.0), lambda s: s.ExponentialFilter(1.0, 0),
                                 lambda s: s.ExponentialFilter(1.0, 4, 1.5), lambda s: s.CutoffFilter(0.0),
                                 lambda s: s.HyperviscosityFilter(-1.0), lambda s: s.CesaroFilter(0.5, 0)])
def test_filter_parameter_checks(ssg, bad):
    with pytest.raises(AssertionError):
        bad(ssg)


@pytest.mark.parametrize("ftype", [0, 1, 2, 3])
def test_transfer_tables_match_oracle(ssg, oracle_mod, ftype):
    n = 32
    dom = ssg.make_domain(n, n, 4)
    dt = 0.01
    objs = {0: (ssg.ExponentialFilter(2.0, 4, 0.3), dict(filter_strength=2.0, filter_order=4, filter_cutoff=0.3)),
            1: (ssg.HyperviscosityFilter(1e-4, 2), dict(filter_strength=1e-4, filter_order=2)),
            2: (ssg.CutoffFilter(0.4), dict(filter_cutoff=0.4)),
            3: (ssg.CesaroFilter(0.2, 3), dict(filter_cutoff=0.2, filter_order=3))}
    f, kw = objs[ftype]
    tab = ssg.filter.transfer_table(dom, f, dt)
    o = oracle_mod.Oracle(n, n, 4, dt=dt, filter_type=ftype, **kw)
    b = np.random.default_rng(1).standard_normal((n, n))
    bh = np.fft.rfft2(b, axes=(0, 1))
    ref = np.fft.irfft2(bh * tab, s=(n, n), axes=(0, 1))
    assert np.abs(o.filter(b) - ref).max() < 1e-12
