"""Batched and served forms.

CPU: the native request loop's admission checks and error reporting (no
device is needed to reject an oversize request, and a request that finds no
device fails with THP_E_NO_DEVICE instead of crashing).  GPU: every served
result is the same alone and in the mix (within the CG tolerance), contexts
evicted under a tight budget are re-targeted for new systems and still give
the same answers, and batched solves equal single solves."""
import numpy as np
import pytest

DEBYE = 4.80321


def test_server_rejects_oversize_and_unknown(thp):
    from tinker_hp_b200 import serve, lib
    ws = thp.water.make_water_box(400)
    srv = serve.Server(budget_bytes=1000, workers=1)
    with pytest.raises(lib.ThpError) as e:
        srv.submit("big", ws)
    assert e.value.status == lib.THP_E_OOM_ADMISSION
    import ctypes as C
    t = C.c_ulonglong()
    x = np.zeros(ws.n)
    st = lib.load().thp_server_submit(srv.h, 12345, lib._p(x), lib._p(x), lib._p(x), None, None, C.byref(t))
    assert st == lib.THP_E_INVALID
    srv.close()


def test_server_reports_device_status(thp):
    # on a machine without a GPU the request fails cleanly with NO_DEVICE;
    # on a GPU it is solved
    from tinker_hp_b200 import serve, lib
    ws = thp.water.make_water_box(400)
    srv = serve.Server(workers=2)
    out = srv.run([serve.Request(0, 0.0, "a", ws)], realtime=False)
    assert out[0].status in (lib.THP_OK, lib.THP_E_NO_DEVICE)
    st = srv.stats()
    assert st["completed"] + st["failed"] == 1
    srv.close()


@pytest.mark.gpu
def test_batch_equals_single(thp):
    from tinker_hp_b200 import lib
    systems = thp.water.make_batch(6, seed=4003)
    ctxs = [lib.Context(ws, precision=lib.MIXED, poleps=1e-6) for ws in systems]
    infos = lib.solve_batch(ctxs)
    for ws, ctx, info in zip(systems, ctxs, infos):
        ub, _ = ctx.dipoles()
        single = lib.Context(ws, precision=lib.MIXED, poleps=1e-6)
        r = single.solve()
        us, _ = single.dipoles()
        assert info["converged"] and info["niter"] == r["niter"]
        # same kernels; only the order of the FP32 grid atomics differs
        assert np.sqrt(np.mean(np.sum((ub - us) ** 2, 1))) * DEBYE < 1e-7
        assert abs(info["epol"] - r["epol"]) < 1e-7 * abs(r["epol"])


@pytest.mark.gpu
def test_served_results_same_alone_and_in_mix(thp):
    from tinker_hp_b200 import serve, lib
    reqs = serve.poisson_stream(16, rate=500.0, nmin=1000, nmax=6000, seed=11)
    srv = serve.Server(precision=lib.MIXED, poleps=1e-6, workers=4)
    out = {r.rid: r for r in srv.run(reqs, realtime=True)}
    srv.close()
    assert all(out[q.rid].warm == q.repeat for q in reqs)
    for q in reqs:
        r = out[q.rid]
        assert r.status == lib.THP_OK
        # against the converged FP64 answer: the mixed form's 1e-5 D bound
        exact = lib.Context(q.ws, precision=lib.FP64, poleps=1e-8)
        exact.solve()
        ue, _ = exact.dipoles()
        err = np.sqrt(np.mean(np.sum((r.uind - ue) ** 2, 1))) * DEBYE
        assert err < 1e-5, (q.rid, q.repeat, err)
        if not q.repeat:
            # the same request alone on an idle GPU: same solver path
            alone = lib.Context(q.ws, precision=lib.MIXED, poleps=1e-6)
            alone.solve()
            ua, _ = alone.dipoles()
            assert np.sqrt(np.mean(np.sum((r.uind - ua) ** 2, 1))) * DEBYE < 1e-7
    reps = [out[q.rid].niter for q in reqs if q.repeat]
    fresh = [out[q.rid].niter for q in reqs if not q.repeat]
    if reps:
        assert np.mean(reps) < np.mean(fresh)


@pytest.mark.gpu
def test_server_fills_caller_buffers_in_place(thp):
    # coordinates and dipoles in the caller's own arrays (read and written
    # when the request runs); two overlapping systems, each repeated
    from tinker_hp_b200 import serve, lib
    boxes = [thp.water.make_water_box(2000, cfg=0), thp.water.make_water_box(1500, cfg=1)]
    srv = serve.Server(precision=lib.MIXED, poleps=1e-6, workers=2)
    for k, ws in enumerate(boxes):
        srv.register(f"s{k}", ws)
    rng = np.random.default_rng(3)
    work = []
    for rep in range(3):
        for k, ws in enumerate(boxes):
            moved = ws.with_positions(ws.positions() + rng.normal(0.0, 0.005, size=(ws.n, 3)))
            xyz = [np.ascontiguousarray(a, dtype=np.float64) for a in (moved.x, moved.y, moved.z)]
            uind = np.full((ws.n, 3), np.nan)
            ticket, out = srv.submit(f"s{k}", moved, xyz=xyz, uind=uind)
            assert out is uind
            work.append((ticket, moved, uind, rep > 0))
    for ticket, moved, uind, repeat in work:
        r = srv.wait(ticket)
        assert r.status == lib.THP_OK and bool(r.warm) == repeat
        exact = lib.Context(moved, precision=lib.FP64, poleps=1e-8)
        exact.solve()
        ue, _ = exact.dipoles()
        assert np.sqrt(np.mean(np.sum((uind - ue) ** 2, 1))) * DEBYE < 1e-5
    srv.close()


@pytest.mark.gpu
def test_server_reuses_contexts_under_a_tight_budget(thp):
    from tinker_hp_b200 import serve, lib
    reqs = serve.poisson_stream(24, rate=1000.0, nmin=1000, nmax=8000, repeat_frac=0.3, seed=13)
    biggest = max(lib.footprint(q.ws, lib.MIXED) for q in reqs)
    srv = serve.Server(precision=lib.MIXED, poleps=1e-6, workers=3, budget_bytes=3 * biggest)
    out = {r.rid: r for r in srv.run(reqs, realtime=False)}
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["evicted"] > 0 and st["reused"] > 0, st
    assert st["bytes"] <= 3 * biggest
    for q in reqs:
        alone = lib.Context(q.ws, precision=lib.MIXED, poleps=1e-6)
        alone.solve()
        ua, _ = alone.dipoles()
        d = np.sqrt(np.mean(np.sum((out[q.rid].uind - ua) ** 2, 1))) * DEBYE
        # a warm start converges to the same answer within the CG tolerance
        assert d < (1e-5 if out[q.rid].warm else 1e-7), (q.rid, out[q.rid].warm, d)


@pytest.mark.gpu
def test_context_retarget_matches_fresh_context(thp):
    # one context serves a small, a larger and another small system in turn
    # (thp_ctx_reset grows buffers and re-plans the FFT only when needed)
    from tinker_hp_b200 import lib
    boxes = [thp.water.make_water_box(216, cfg=0), thp.water.make_water_box(648, cfg=1),
             thp.water.make_water_box(300, cfg=2)]
    ctx = lib.Context(boxes[0])
    for k, ws in enumerate(boxes):
        if k:
            ctx.retarget(ws)
        r = ctx.solve()
        u, p = ctx.dipoles()
        fresh = lib.Context(ws)
        rf = fresh.solve()
        uf, pf = fresh.dipoles()
        assert r["niter"] == rf["niter"]
        assert np.abs(u - uf).max() < 1e-12 * np.abs(uf).max() and np.abs(p - pf).max() < 1e-12 * np.abs(pf).max()
        assert abs(r["epol"] - rf["epol"]) < 1e-12 * abs(rf["epol"])
        _, g = ctx.gradient()
        _, gf = fresh.gradient()
        assert np.abs(g - gf).max() < 1e-9 * np.abs(gf).max()
