"""Block shapes of the transform passes (ssg_set_tiles / ssg_autotune).

A block shape only regroups whole transforms (rows or column pairs) into
blocks; each transform's operations are the same, but each shape is its own
compiled kernel and may contract a multiply-add differently, so fields agree
to rounding: 1e-14 relative in FP64, 1e-11 in mixed precision (measured: at
most 5e-16 and 4e-13), with identical iteration counts.  Pinned shapes are
reproducible bit for bit.  ssg_autotune times the candidates on the context's
own grid and must leave the state exactly as it found it."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

X_SHAPES = (64, 128, 256)
Y_SHAPES = (128, 256, 512)
TOL = {"fp64": 1e-14, "mixed": 1e-11}


def rel_max(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def make(ssg, n, nz, precision, scheme="AB2"):
    dom = ssg.make_domain(n, n, nz)
    sch = ssg.AB2_LowStorage if scheme == "AB2" else ssg.RK3
    prob = ssg.SemiGeostrophicProblem(dom, scheme=sch, dt=1e-3, filter_freq=4, filter_order=8, precision=precision,
                                      enable_diagnostics=False)
    return dom, prob


def run(ssg, n, nz, precision, tiles=None, steps=8, scheme="AB2"):
    dom, prob = make(ssg, n, nz, precision, scheme)
    if tiles is not None:
        prob._ctx.set_tiles(*tiles)
    ssg.set_b_(prob, ssg.jfm_spectral_buoyancy(n, n, 4, seed=77 + n), dom)
    st = ssg.stepforward_(prob, steps)
    out = (prob.fields.bs, prob.fields.phi, st.ma_iterations)
    prob.close()
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("n,nz", [(64, 8), (128, 12), (256, 8)])
def test_every_shape_agrees_to_rounding(require_gpu, ssg, n, nz, precision):
    ref = run(ssg, n, nz, precision)
    shapes = [(x, 0) for x in X_SHAPES] + [(0, y) for y in Y_SHAPES] + [(X_SHAPES[0], Y_SHAPES[-1])]
    for tiles in shapes:
        out = run(ssg, n, nz, precision, tiles)
        assert out[2] == ref[2], tiles
        assert rel_max(out[0], ref[0]) < TOL[precision], tiles
        assert rel_max(out[1], ref[1]) < TOL[precision], tiles
        # the same pinned shape again: bit for bit
        again = run(ssg, n, nz, precision, tiles)
        assert np.array_equal(again[0], out[0]), tiles


def test_rk3_shapes_agree(require_gpu, ssg):
    ref = run(ssg, 256, 8, "fp64", scheme="RK3", steps=4)
    out = run(ssg, 256, 8, "fp64", (64, 512), scheme="RK3", steps=4)
    assert out[2] == ref[2] and rel_max(out[0], ref[0]) < TOL["fp64"]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_autotune_keeps_the_state(require_gpu, ssg, precision):
    n, nz = 128, 12
    dom, prob = make(ssg, n, nz, precision)
    ssg.set_b_(prob, ssg.jfm_spectral_buoyancy(n, n, 5, seed=5), dom)
    ssg.stepforward_(prob, 3)
    before = (prob.fields.bs, prob.fields.phi, prob._ctx.time())
    x, y = prob.autotune(reps=2)
    assert x in X_SHAPES and y in Y_SHAPES
    assert prob.tiles == (x, y)
    variants = prob.variants
    after = (prob.fields.bs, prob.fields.phi, prob._ctx.time())
    assert np.array_equal(before[0], after[0]) and np.array_equal(before[1], after[1]) and before[2] == after[2]
    # the run continues exactly as one that pins the same shapes and kernels at
    # the same point
    ssg.stepforward_(prob, 5)
    b_tuned = prob.fields.bs
    prob.close()
    dom2, ref = make(ssg, n, nz, precision)
    ssg.set_b_(ref, ssg.jfm_spectral_buoyancy(n, n, 5, seed=5), dom2)
    ssg.stepforward_(ref, 3)
    ref._ctx.set_tiles(x, y)
    ref._ctx.set_variants(*variants)
    ssg.stepforward_(ref, 5)
    assert np.array_equal(ref.fields.bs, b_tuned)
    ref.close()


def test_tile_arguments(require_gpu, ssg):
    L = ssg._lib.load()
    dom, prob = make(ssg, 64, 8, "fp64")
    assert L.ssg_set_tiles(prob._ctx.h, 96, 0) == ssg._lib.SSG_ERR_ARG
    assert L.ssg_set_tiles(prob._ctx.h, 0, 64) == ssg._lib.SSG_ERR_ARG
    assert L.ssg_set_tiles(prob._ctx.h, 64, 512) == ssg._lib.SSG_OK
    assert prob.tiles == (64, 512)
    assert L.ssg_set_tiles(prob._ctx.h, 0, 0) == ssg._lib.SSG_OK
    prob.close()
    dom, prob = make(ssg, 32, 8, "fp64")
    assert L.ssg_set_tiles(prob._ctx.h, 128, 0) == ssg._lib.SSG_ERR_UNSUPPORTED
    x, y = ctypes.c_int32(-1), ctypes.c_int32(-1)
    assert L.ssg_autotune(prob._ctx.h, 1, ctypes.byref(x), ctypes.byref(y)) == ssg._lib.SSG_OK
    assert (x.value, y.value) == (0, 0)  # nothing to tune outside 64..512
    prob.close()


def test_autotuned_ensemble_matches_solo_runs(require_gpu, ssg):
    """Batched members equal solo runs with the same block shapes and kernel
    variants pinned at the same point."""
    from ssg_b200.ensemble import DeviceBatch
    grids = [(64, 8), (64, 8), (128, 8)]
    probs, doms = [], []
    for i, (n, nz) in enumerate(grids):
        dom, p = make(ssg, n, nz, "mixed")
        ssg.set_b_(p, ssg.jfm_spectral_buoyancy(n, n, 4, seed=300 + i), dom)
        probs.append(p)
    batch = DeviceBatch(probs, "threads", autotune=True)
    assert set(batch.tiles) == {(64, 64, 8, 1), (128, 128, 8, 1)}
    assert probs[1].tiles == probs[0].tiles
    batch.step(6)
    outs = [p.fields.bs for p in probs]
    batch_tiles = dict(batch.tiles)
    batch_variants = dict(batch.variants)
    batch.close()
    for i, (n, nz) in enumerate(grids):
        # as in the batch: set_b with the default kernels, then the tuned ones
        dom, p = make(ssg, n, nz, "mixed")
        ssg.set_b_(p, ssg.jfm_spectral_buoyancy(n, n, 4, seed=300 + i), dom)
        p._ctx.set_tiles(*batch_tiles[(n, n, nz, 1)])
        p._ctx.set_variants(*batch_variants[(n, n, nz, 1)])
        ssg.stepforward_(p, 6)
        assert np.array_equal(p.fields.bs, outs[i]), i
        p.close()
    for p in probs:
        p.close()


@pytest.mark.parametrize("precision,n,nz", [("mixed", 1024, 8), ("fp64", 512, 8), ("mixed", 128, 16)])
def test_every_kernel_variant_agrees(require_gpu, ssg, precision, n, nz):
    """ssg_set_variants: every y-pass kernel that exists for the grid and
    precision, and both vertical-solve forms, give the same fields to
    rounding (the warp y-pass bit for bit across warps per block; the
    vertical-solve forms bit for bit); a kernel that does not exist is
    rejected and leaves the context as it was."""
    L = ssg._lib
    outs = {}
    for v in (L.SSG_YPASS_PLAIN, L.SSG_YPASS_TMA, L.SSG_YPASS_WARP2, L.SSG_YPASS_WARP4, L.SSG_YPASS_WARP8):
        for staged in (0, 1):
            dom, prob = make(ssg, n, nz, precision)
            before = prob.variants
            try:
                prob._ctx.set_variants(v, staged)
            except ssg.SsgError as e:
                assert e.status == L.SSG_ERR_UNSUPPORTED and prob.variants == before
                prob.close()
                continue
            assert prob.variants == (v, staged)
            ssg.set_b_(prob, ssg.jfm_spectral_buoyancy(n, n, 8, seed=5), dom)
            st = ssg.stepforward_(prob, 6)
            outs[(v, staged)] = (prob.fields.bs, st.ma_iterations)
            prob.close()
    assert (L.SSG_YPASS_PLAIN, 0) in outs and len(outs) >= 4
    # different transform kernels round differently: FP64 to 1e-12, and the
    # mixed path to its FP32 floor
    tol = {"fp64": 1e-12, "mixed": 1e-6}[precision]
    ref = outs[(L.SSG_YPASS_PLAIN, 0)][0]
    for (v, staged), (b, it) in outs.items():
        assert rel_max(b, ref) < tol, (v, staged)
        assert np.array_equal(b, outs[(v, 0)][0])
        if v in (L.SSG_YPASS_WARP2, L.SSG_YPASS_WARP4):
            assert np.array_equal(b, outs[(L.SSG_YPASS_WARP8, staged)][0])
    if n == 1024 and precision == "mixed":
        assert (L.SSG_YPASS_WARP2, 0) in outs
