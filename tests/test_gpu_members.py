"""Ensemble members held by one context (ssg_config.nmembers).

Every kernel pass covers all members in one launch, and a Monge-Ampere solve
iterates until every member's stop rule has fired, leaving a member whose
solve stopped as it is.  Each member's fields must therefore equal those of
a one-member problem started from the same field, bit for bit: the members'
initial fields differ in amplitude and spectrum so that their solves stop
after different iteration counts."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def member_fields(ssg, n, m, seed):
    # amplitudes over two decades: the members' solves need different
    # iteration counts
    return [ssg.jfm_spectral_buoyancy(n, n, 3 + (i % 4), seed=seed + i) * (0.3 + 0.9 * i) for i in range(m)]


def make(ssg, n, nz, precision, scheme, nmembers=1, **kw):
    dom = ssg.make_domain(n, n, nz)
    sch = ssg.AB2_LowStorage if scheme == "AB2" else ssg.RK3
    prob = ssg.SemiGeostrophicProblem(dom, scheme=sch, dt=1e-3, filter_freq=4, filter_order=8, precision=precision,
                                      enable_diagnostics=False, nmembers=nmembers, **kw)
    return dom, prob


def solo(ssg, n, nz, precision, scheme, b, steps, **kw):
    dom, p = make(ssg, n, nz, precision, scheme, **kw)
    ssg.set_b_(p, b, dom)
    st = ssg.stepforward_(p, steps)
    out = (p.fields.bs, p.fields.phi, p.fields.u, st)
    p.close()
    return out


@pytest.mark.parametrize("precision,scheme,n,nz", [("fp64", "AB2", 64, 8), ("fp64", "RK3", 64, 12),
                                                   ("mixed", "AB2", 128, 16), ("mixed", "RK3", 128, 8),
                                                   ("fp64", "AB2", 512, 8), ("mixed", "AB2", 512, 16)])
def test_members_equal_solo_runs(require_gpu, ssg, precision, scheme, n, nz):
    m, steps = 3, 9
    bs = member_fields(ssg, n, m, 40 + n)
    dom, batch = make(ssg, n, nz, precision, scheme, nmembers=m)
    ssg.set_b_(batch, np.stack(bs, axis=-1), dom)
    st = ssg.stepforward_(batch, steps)
    b_all, phi_all, u_all = batch.fields.bs, batch.fields.phi, batch.fields.u
    assert b_all.shape == (n, n, m) and phi_all.shape == (n, n, nz, m)
    batch.close()
    iters = []
    for i in range(m):
        b, phi, u, sst = solo(ssg, n, nz, precision, scheme, bs[i], steps)
        assert np.array_equal(b_all[..., i], b), i
        assert np.array_equal(phi_all[..., i], phi), i
        assert np.array_equal(u_all[..., i], u), i
        iters.append(sst.ma_iterations)
    # the batch's statistics count every member's solves
    assert st.ma_solves == m * steps * (3 if scheme == "RK3" else 1)
    assert st.ma_iterations == sum(iters)
    assert len(set(iters)) > 1 or precision == "mixed"


def test_members_at_1024_mixed(require_gpu, ssg):
    """The warp-transform y-pass and its tensor maps over two members."""
    n, nz, m, steps = 1024, 8, 2, 5
    bs = member_fields(ssg, n, m, 7)
    dom, batch = make(ssg, n, nz, "mixed", "AB2", nmembers=m)
    ssg.set_b_(batch, np.stack(bs, axis=-1), dom)
    ssg.stepforward_(batch, steps)
    b_all = batch.fields.bs
    batch.close()
    for i in range(m):
        b = solo(ssg, n, nz, "mixed", "AB2", bs[i], steps)[0]
        assert np.array_equal(b_all[..., i], b), i


@pytest.mark.parametrize("graphs", ["1", "0"])
def test_members_host_loop_and_graphs(require_gpu, ssg, monkeypatch, graphs):
    """The solve's host loop (every step, graphs off) and the graph form
    agree bit for bit with one-member runs."""
    monkeypatch.setenv("SSG_B200_GRAPHS", graphs)
    n, nz, m, steps = 64, 8, 4, 6
    bs = member_fields(ssg, n, m, 11)
    dom, batch = make(ssg, n, nz, "fp64", "RK3", nmembers=m)
    ssg.set_b_(batch, np.stack(bs, axis=-1), dom)
    ssg.stepforward_(batch, steps)
    b_all = batch.fields.bs
    batch.close()
    for i in range(m):
        assert np.array_equal(b_all[..., i], solo(ssg, n, nz, "fp64", "RK3", bs[i], steps)[0]), i


def test_members_checkpoint_and_fields(require_gpu, ssg, tmp_path):
    n, nz, m = 64, 8, 3
    bs = member_fields(ssg, n, m, 90)
    dom, batch = make(ssg, n, nz, "fp64", "AB2", nmembers=m)
    ssg.set_b_(batch, np.stack(bs, axis=-1), dom)
    ssg.stepforward_(batch, 4)
    blob = batch._ctx.checkpoint()
    ssg.stepforward_(batch, 5)
    ref = batch.fields.bs
    batch._ctx.restore(blob)
    ssg.stepforward_(batch, 5)
    assert np.array_equal(batch.fields.bs, ref)
    # a member's field written and read back
    old = batch.clock.db_dt_old
    assert old.shape == (n, n, m)
    batch.clock.db_dt_old = old
    assert np.allclose(batch.clock.db_dt_old, old, rtol=0, atol=1e-12 * np.abs(old).max())
    # wrong member count
    with pytest.raises(ValueError):
        ssg.set_b_(batch, bs[0], dom)
    with pytest.raises(ValueError):
        ssg.save_simulation_state_full(str(tmp_path / "m.npz"), batch)
    batch.close()
    # a blob of three members does not restore into two
    _, two = make(ssg, n, nz, "fp64", "AB2", nmembers=2)
    with pytest.raises(ssg.SsgError) as e:
        two._ctx.restore(blob)
    assert e.value.status == ssg._lib.SSG_ERR_ARG
    two.close()


def test_members_reject(require_gpu, ssg):
    L = ssg._lib
    dom, batch = make(ssg, 64, 8, "fp64", "AB2", nmembers=2)
    with pytest.raises(ssg.SsgError) as e:
        ssg.diagnostics(batch)
    assert e.value.status == L.SSG_ERR_UNSUPPORTED
    batch.close()
    with pytest.raises(ssg.SsgError) as e:
        make(ssg, 64, 8, "fp64", "AB2", nmembers=2, ma_rhs="volume")
    assert e.value.status == L.SSG_ERR_UNSUPPORTED
    with pytest.raises(ssg.SsgError) as e:
        make(ssg, 64, 8, "fp64", "AB2", nmembers=2000)
    assert e.value.status == L.SSG_ERR_ARG


def test_device_batch_members_mode(require_gpu, ssg):
    """DeviceBatch "members": problems of the same kind share a context;
    after sync each problem's own context holds exactly the state of a run
    stepped alone, and keeps stepping as that run would."""
    from ssg_b200.ensemble import DeviceBatch
    kinds = [(64, 8, "mixed", "AB2")] * 3 + [(128, 8, "mixed", "AB2")] * 2 + [(64, 8, "fp64", "RK3")]
    fields = [ssg.jfm_spectral_buoyancy(n, n, 3 + i % 3, seed=500 + i) * (0.5 + 0.7 * i)
              for i, (n, _, _, _) in enumerate(kinds)]
    probs = []
    for (n, nz, prec, sch), b in zip(kinds, fields):
        dom, p = make(ssg, n, nz, prec, sch)
        ssg.set_b_(p, b, dom)
        probs.append(p)
    batch = DeviceBatch(probs, "members")
    assert len(batch.groups) == 2 and sorted(len(g[1]) for g in batch.groups) == [2, 3]
    batch.step(4)
    batch.step(3)
    batch.sync()
    for p in probs:
        ssg.stepforward_(p, 2)  # the problems' own contexts continue
    got = [(p.fields.bs, p.fields.phi) for p in probs]
    batch.close()
    for p in probs:
        p.close()
    for i, ((n, nz, prec, sch), b) in enumerate(zip(kinds, fields)):
        bs, phi, _, _ = solo(ssg, n, nz, prec, sch, b, 9)
        assert np.array_equal(got[i][0], bs), i
        assert np.array_equal(got[i][1], phi), i


def test_members_gather_checks(require_gpu, ssg):
    L = ssg._lib.load()
    import ctypes
    dom, batch = make(ssg, 64, 8, "fp64", "AB2", nmembers=2)
    _, a = make(ssg, 64, 8, "fp64", "AB2")
    _, b = make(ssg, 64, 8, "mixed", "AB2")
    _, c = make(ssg, 64, 8, "fp64", "AB2")
    ssg.set_b_(a, ssg.jfm_spectral_buoyancy(64, 64, 4, seed=1), dom)
    ssg.set_b_(c, ssg.jfm_spectral_buoyancy(64, 64, 4, seed=2), dom)
    arr = lambda *ps: (ctypes.c_void_p * len(ps))(*[p._ctx.h.value for p in ps])
    E = ssg._lib
    assert L.ssg_members_gather(batch._ctx.h, arr(a, b), 2) == E.SSG_ERR_ARG   # configurations differ
    assert L.ssg_members_gather(batch._ctx.h, arr(a), 1) == E.SSG_ERR_ARG      # member count
    ssg.stepforward_(c, 1)
    assert L.ssg_members_gather(batch._ctx.h, arr(a, c), 2) == E.SSG_ERR_ARG   # clocks differ
    ssg.stepforward_(a, 1)
    assert L.ssg_members_gather(batch._ctx.h, arr(a, c), 2) == E.SSG_OK
    # a member on another vertical grid (a different operator and pivot table)
    sdom = ssg.make_domain(64, 64, 8, z_grid="stretched",
                           stretch_params={"type": "tanh", "β": 2.0, "surface_concentration": True})
    s = ssg.SemiGeostrophicProblem(sdom, scheme=ssg.AB2_LowStorage, dt=1e-3, filter_freq=4, filter_order=8,
                                   precision="fp64", enable_diagnostics=False)
    ssg.set_b_(s, ssg.jfm_spectral_buoyancy(64, 64, 4, seed=3), sdom)
    ssg.stepforward_(s, 1)
    assert L.ssg_members_gather(batch._ctx.h, arr(a, s), 2) == E.SSG_ERR_ARG
    for p in (batch, a, b, c, s):
        p.close()


def test_device_batch_members_autotuned(require_gpu, ssg):
    """The members mode with tuned kernels: each problem equals a run stepped
    alone with the batched context's block shapes and kernel variants pinned
    (the same compiled kernels)."""
    from ssg_b200.ensemble import DeviceBatch
    n, nz, m = 128, 16, 3
    fields = [ssg.jfm_spectral_buoyancy(n, n, 4, seed=700 + i) * (0.4 + 0.8 * i) for i in range(m)]
    probs = []
    for b in fields:
        dom, p = make(ssg, n, nz, "mixed", "AB2")
        ssg.set_b_(p, b, dom)
        probs.append(p)
    batch = DeviceBatch(probs, "members", autotune=True)
    tiles, variants = batch.tiles[(n, n, nz, 1)], batch.variants[(n, n, nz, 1)]
    batch.step(7)
    batch.close()  # hands the state back
    got = [p.fields.bs for p in probs]
    for p in probs:
        p.close()
    for i, b in enumerate(fields):
        dom, p = make(ssg, n, nz, "mixed", "AB2")
        ssg.set_b_(p, b, dom)
        p._ctx.set_tiles(*tiles)
        p._ctx.set_variants(*variants)
        ssg.stepforward_(p, 7)
        assert np.array_equal(p.fields.bs, got[i]), i
        p.close()
