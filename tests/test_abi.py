"""CPU-side checks of the C ABI: the library loads, exports every function
include/ssg_b200.h declares, its ctypes structs match the C layout, and
argument validation fails cleanly (no GPU work is attempted here)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ssg_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ssg_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(ssg):
    L = ssg._lib.load()
    names = declared_functions()
    assert len(names) >= 12
    for name in names:
        assert hasattr(L, name), name
    assert sorted(ssg._lib.EXPORTED_SYMBOLS) == names


def test_struct_layouts_match_header(ssg, tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "ssg_b200.h"\n'
        "int main(void){printf(\"%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n\", sizeof(ssg_config), sizeof(ssg_ma_stats),"
        " sizeof(ssg_step_stats), offsetof(ssg_config, eps), offsetof(ssg_config, ma_tol),"
        " offsetof(ssg_config, nmembers), offsetof(ssg_step_stats, step), sizeof(ssg_adjoint_stats),"
        " offsetof(ssg_adjoint_stats, adjoint_update_max), offsetof(ssg_adjoint_stats, device_bytes)); return 0;}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = list(map(int, subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()))
    L = ssg._lib
    want = [ctypes.sizeof(L.SsgConfig), ctypes.sizeof(L.SsgMaStats), ctypes.sizeof(L.SsgStepStats),
            L.SsgConfig.eps.offset, L.SsgConfig.ma_tol.offset, L.SsgConfig.nmembers.offset,
            L.SsgStepStats.step.offset, ctypes.sizeof(L.SsgAdjointStats), L.SsgAdjointStats.adjoint_update_max.offset,
            L.SsgAdjointStats.device_bytes.offset]
    assert got == want


def test_config_defaults(ssg):
    c = ssg._lib.default_config()
    assert c.abi_version == ssg._lib.ABI_VERSION == ssg._lib.load().ssg_abi_version()
    assert c.lx == pytest.approx(2 * np.pi) and c.lz == 1.0
    assert (c.filter_freq, c.filter_order, c.filter_cutoff, c.filter_strength) == (10, 4, 0.65, 0.1)
    assert (c.ma_tol, c.ma_maxiter, c.ma_per_stage, c.ma_rhs_mode, c.precision) == (1e-10, 50, 1, 0, 0)


@pytest.mark.parametrize("field,value,code", [
    ("nx", 48, -6), ("nx", 2048, -6), ("nz", 3, -6), ("nz", 65, -6), ("scheme", 7, -1),
    ("ma_maxiter", 0, -1), ("abi_version", 99, -1), ("precision", 2, -1), ("ma_rhs_mode", 5, -1), ("ma_predictor", 4, -1),
])
def test_invalid_configs_rejected_before_device_work(ssg, field, value, code):
    L = ssg._lib.load()
    c = ssg._lib.default_config()
    c.nx = c.ny = 64
    c.nz = 8
    setattr(c, field, value)
    if field == "nx":
        c.ny = value
    h = ctypes.c_void_p()
    rc = L.ssg_ctx_create(ctypes.byref(c), 0, ctypes.byref(h))
    assert rc == code and not h.value
    assert L.ssg_last_error(None)


def test_null_context_is_an_argument_error(ssg):
    L = ssg._lib.load()
    assert L.ssg_step(None, 1, 0.0, None) == ssg._lib.SSG_ERR_ARG
    assert L.ssg_solve_ma(None, None) == ssg._lib.SSG_ERR_ARG
    assert L.ssg_ctx_destroy(None) == 0


def test_python_api_domain(ssg):
    d = ssg.make_domain(128, 128, 16)
    assert d.kx.shape == (128,) and d.ky.shape == (65,) and d.mask.shape == (128, 65)
    assert d.dz[0] == pytest.approx(1 / 15) and d.z[-1] == 1.0
    with pytest.raises(ValueError):  # stretched without stretch_params (src/domain.jl:251-254)
        ssg.make_domain(64, 64, 8, z_grid="stretched")
    d = ssg.make_domain(64, 64, 8, z_grid="stretched", stretch_params={"type": "tanh"})
    assert d.z[0] == pytest.approx(1.0) and (d.dz < 0).all()
    with pytest.raises(NotImplementedError):
        ssg.TimeParams(0.01, adaptive_dt=True)
