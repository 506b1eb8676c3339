"""Batch plans (thp_batch_*): the CG iterations of many small systems run as
batched persistent kernels, with the convolution as batched cuFFT transforms
per grid shape, checked against the same systems solved alone (one context
each) and against the CPU FP64 oracle's restatement of newinduce_pme2
(newinduce_pme2.f:16-283) on a subset.

Tolerances.  FP64 form: the same CG iteration count as alone and as the
oracle; dipoles within 1e-9 D RMS of the solve alone (batched and single
transforms and reduction tiles round differently), within 1e-6 D of the oracle; Epol within 1e-8 relative of the
oracle.  Mixed form: dipoles within 1e-5 D RMS of the oracle and within
5e-6 D of the mixed solve alone (its FP32 rounding differs), Epol within 6e-7 relative of the oracle.
"""
import dataclasses

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

DEBYE = 4.80321


def rms(a, b):
    return float(np.sqrt(np.mean(np.sum((a - b) ** 2, axis=1))) * DEBYE)


@pytest.fixture(scope="module")
def lib(thp):
    from tinker_hp_b200 import lib as L
    L.load()
    return L


@pytest.fixture(scope="module")
def boxes(thp):
    # eight boxes of 300-6000 atoms (the batched workload's construction)
    return thp.water.make_batch(8, seed=4003)


@pytest.fixture(scope="module")
def oracle_refs(boxes):
    refs = {}
    for q in np.argsort([w.n for w in boxes])[:3]:
        orc = O.Oracle(boxes[q], poleps=1e-6)
        assert orc.mlistcell()[0] == 0
        ref = orc.solve()
        refs[int(q)] = (ref, orc.epolar(ref["uind"])[0])
    return refs


def solve_alone(lib, ws, precision):
    ctx = lib.Context(ws, precision=precision, poleps=1e-6)
    res = ctx.solve()
    return res, ctx.dipoles()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_plan_matches_alone_and_oracle(lib, boxes, oracle_refs, precision):
    prec = lib.FP64 if precision == "fp64" else lib.MIXED
    ctxs = [lib.Context(ws, precision=prec, poleps=1e-6) for ws in boxes]
    plan = lib.Batch(ctxs)
    infos = plan.solve()
    for q, (ws, ctx, info) in enumerate(zip(boxes, ctxs, infos)):
        assert info["converged"], q
        uind, uinp = ctx.dipoles()
        alone, (ua, pa) = solve_alone(lib, ws, prec)
        d = max(rms(uind, ua), rms(uinp, pa))
        if prec == lib.FP64:
            assert info["niter"] == alone["niter"], (q, info["niter"], alone["niter"])
            assert d < 1e-9, (q, d)
        else:
            assert d < 5e-6, (q, d)
        if q in oracle_refs:
            ref, e_ref = oracle_refs[q]
            do = max(rms(uind, ref["uind"]), rms(uinp, ref["uinp"]))
            e_rel = abs(info["epol"] - e_ref) / abs(e_ref)
            if prec == lib.FP64:
                assert info["niter"] == ref["niter"]
                assert do < 1e-6 and e_rel < 1e-8, (q, do, e_rel)
            else:
                assert do < 1e-5 and e_rel < 6e-7, (q, do, e_rel)
    plan.close()


def test_autotuner_keeps_a_shape_and_results_hold(lib, boxes):
    # every candidate of the tuner is a correct schedule: the dipoles agree
    # across the tuning solves, and the kept shape is reported afterwards
    ctxs = [lib.Context(ws, precision=lib.MIXED, poleps=1e-6) for ws in boxes]
    plan = lib.Batch(ctxs)
    first = None
    for _ in range(8):
        plan.solve()
        u = np.concatenate([c.dipoles()[0] for c in ctxs])
        if first is None:
            first = u
        assert rms(u, first) < 1e-6
    t = plan.tuning()
    assert t is not None and t["ms_per_solve"] > 0, t
    assert t["blocks_per_sm"] in (4, 8, 16) and t["matvec_atoms"] in (16, 32)
    # a second plan of the same size class starts with the kept shape
    plan2 = lib.Batch(ctxs)
    assert plan2.tuning() is not None
    plan.close()
    plan2.close()


def test_plan_warm_start(lib, boxes):
    ctxs = [lib.Context(ws, precision=lib.FP64, poleps=1e-6) for ws in boxes]
    plan = lib.Batch(ctxs)
    cold = plan.solve()
    warm = plan.solve(guess=lib.GUESS_PREVIOUS)
    for c, w in zip(cold, warm):
        assert w["converged"] and w["niter"] < c["niter"]
    plan.close()


def test_plan_rejects_what_it_cannot_batch(lib, thp, boxes):
    big = thp.water.make_water_box(10800, cfg=1)  # 32,400 atoms: above the batched kernels' range
    ctxs = [lib.Context(boxes[0], precision=lib.MIXED), lib.Context(big, precision=lib.MIXED)]
    with pytest.raises(lib.ThpError) as e:
        lib.Batch(ctxs)
    assert e.value.status == lib.THP_E_INVALID
    mixed_prec = [lib.Context(boxes[0], precision=lib.MIXED), lib.Context(boxes[1], precision=lib.FP64)]
    with pytest.raises(lib.ThpError):
        lib.Batch(mixed_prec)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_plan_with_an_odd_grid_ahead(lib, boxes, precision):
    # a system with an odd grid (25^3 points) takes the first grid slots; the
    # systems after it still start on 16-byte boundaries (paired reductions,
    # vector gathers) and the batched transforms honour the padded slots
    prec = lib.FP64 if precision == "fp64" else lib.MIXED
    odd = dataclasses.replace(boxes[0], nfft=(25, 25, 25))
    systems = [odd] + list(boxes[1:4])
    ctxs = [lib.Context(ws, precision=prec, poleps=1e-6) for ws in systems]
    plan = lib.Batch(ctxs)
    infos = plan.solve()
    for q, (ws, ctx, info) in enumerate(zip(systems, ctxs, infos)):
        assert info["converged"], q
        uind, uinp = ctx.dipoles()
        alone, (ua, pa) = solve_alone(lib, ws, prec)
        d = max(rms(uind, ua), rms(uinp, pa))
        assert d < (1e-9 if prec == lib.FP64 else 5e-6), (q, d)
    plan.close()
