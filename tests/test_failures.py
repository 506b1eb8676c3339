"""Failure detection in the forms this library can raise without faulting a
GPU: statuses made on the host or by the solver's own flags.

  * a timed wait on the request loop returns THP_E_TIMEOUT when the request
    has not finished (here: held back by a paused queue), leaves the ticket
    valid, and the request completes once the queue resumes (CPU);
  * a non-finite polarizability set on the host reaches the CG reductions,
    whose last block flags the solve THP_E_NAN instead of reporting a
    converged answer (GPU);
  * in a served stream, a request whose coordinates are not finite fails
    alone with THP_E_INVALID while the requests around it, on the same and on
    other systems, give the results they give alone (GPU).
"""
import numpy as np
import pytest

DEBYE = 4.80321


def test_timed_wait_reports_timeout_then_completes(thp):
    from tinker_hp_b200 import serve, lib
    ws = thp.water.make_water_box(400)
    srv = serve.Server(workers=1)
    srv.register("a", ws)
    srv.pause(True)
    ticket, _ = srv.submit("a", ws)
    with pytest.raises(lib.ThpError) as e:
        srv.wait(ticket, timeout_ms=50.0)
    assert e.value.status == lib.THP_E_TIMEOUT
    # still queued, still waitable
    with pytest.raises(lib.ThpError) as e:
        srv.wait(ticket, timeout_ms=0.0)
    assert e.value.status == lib.THP_E_TIMEOUT
    srv.pause(False)
    r = srv.wait(ticket, timeout_ms=600_000.0)
    assert r.status in (lib.THP_OK, lib.THP_E_NO_DEVICE)
    # a finished ticket is gone
    with pytest.raises(lib.ThpError) as e:
        srv.wait(ticket, timeout_ms=10.0)
    assert e.value.status == lib.THP_E_INVALID
    st = srv.stats()
    assert st["completed"] + st["failed"] == 1
    srv.close()


def test_destroy_drains_a_paused_queue(thp):
    from tinker_hp_b200 import serve, lib
    ws = thp.water.make_water_box(400)
    srv = serve.Server(workers=2)
    srv.pause(True)
    tickets = [srv.submit("a", ws)[0] for _ in range(3)]
    assert len(set(tickets)) == 3
    srv.close()  # serves the queue before it returns


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_nan_polarizability_flags_the_solve(thp, precision):
    from tinker_hp_b200 import lib
    ws = thp.water.make_water_box(648, cfg=0)
    pol = np.array(ws.polarity, dtype=np.float64)
    pol[100] = np.nan
    import dataclasses
    bad = dataclasses.replace(ws, polarity=pol)
    prec = lib.FP64 if precision == "fp64" else lib.MIXED
    ctx = lib.Context(bad, precision=prec, poleps=1e-6)
    with pytest.raises(lib.ThpError) as e:
        ctx.solve()
    assert e.value.status == lib.THP_E_NAN
    # the same context solves again once the parameters are finite
    good = lib.Context(ws, precision=prec, poleps=1e-6)
    ref = good.solve()
    ctx.retarget(ws)
    r = ctx.solve()
    assert r["converged"] and r["niter"] == ref["niter"]


@pytest.mark.gpu
def test_served_nonfinite_request_fails_alone(thp):
    from tinker_hp_b200 import serve, lib
    boxes = [thp.water.make_water_box(1000, cfg=0), thp.water.make_water_box(1500, cfg=1)]
    srv = serve.Server(precision=lib.MIXED, poleps=1e-6, workers=2)
    for k, ws in enumerate(boxes):
        srv.register(f"s{k}", ws)
    srv.pause(True)  # queue the whole mix before any of it starts
    work = []
    for rep in range(3):
        for k, ws in enumerate(boxes):
            xyz = [np.array(a, dtype=np.float64) for a in (ws.x, ws.y, ws.z)]
            poisoned = (rep == 1 and k == 0)
            if poisoned:
                xyz[1][17] = np.inf
            uind = np.zeros((ws.n, 3))
            ticket, _ = srv.submit(f"s{k}", ws, xyz=xyz, uind=uind)
            work.append((ticket, k, poisoned, uind))
    srv.pause(False)
    alone = {}
    for k, ws in enumerate(boxes):
        c = lib.Context(ws, precision=lib.MIXED, poleps=1e-6)
        c.solve()
        alone[k] = c.dipoles()[0]
    for ticket, k, poisoned, uind in work:
        r = srv.wait(ticket)
        if poisoned:
            assert r.status == lib.THP_E_INVALID
            continue
        assert r.status == lib.THP_OK
        err = np.sqrt(np.mean(np.sum((uind - alone[k]) ** 2, 1))) * DEBYE
        # repeats start warm from the system's last dipoles: same answer within the CG tolerance
        assert err < (1e-5 if r.warm else 1e-7), (k, r.warm, err)
    st = srv.stats()
    srv.close()
    assert st["failed"] == 1 and st["completed"] == len(work) - 1
