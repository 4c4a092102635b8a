"""Serving (psb_server_*): continuous batching of solve requests, through the
C ABI. Results against the oracle; each result equal alone and in the mix;
the FIFO baseline equal to the batched server; budget, slots, cancellation
and timeouts."""
import time

import numpy as np
import pytest

import physis_b200 as ps
from oracle import oracle as O
from tests.gpu_util import bits_equal, himeno_inputs

pytestmark = pytest.mark.gpu

COEF = (0.1, 0.1, 0.1, 0.1, 0.1, 0.1, 0.4)
GB = 1 << 30


def _diff_residual(a, b):
    d = a.astype(np.float64) - b.astype(np.float64)
    return float(np.sqrt(np.sum(d * d) / np.sum(a.astype(np.float64) ** 2)))


def _serve(reqs, mode=ps.SERVE_BATCHED, budget=8 * GB, slots=0):
    """Serve the requests (dicts of Server.submit keywords) together; returns
    the records and the output fields in request order."""
    s = ps.Server(budget, slots, mode)
    try:
        outs, ids = [], []
        for r in reqs:
            r = dict(r)
            nx, ny, nz = r["dims"]
            out = np.full((nz, ny, nx), np.nan, np.float32)
            ids.append(s.submit(out=out, **r))
            outs.append(out)
        recs = [s.wait(i, timeout=120.0) for i in ids]
        stats = s.stats()
    finally:
        s.destroy()
    for rec in recs:
        assert rec["status"] == ps.PSB_OK, rec
        assert rec["submit_s"] <= rec["start_s"] <= rec["finish_s"]
    return recs, outs, stats


def _mix():
    """Mixed requests with device-generated inputs and early stops."""
    out = []
    rng = np.random.default_rng(77)
    for i in range(12):
        dims = tuple(int(v) for v in rng.integers(12, 70, size=3))
        kind = (ps.DIFFUSION7, ps.DIFFUSION7_PERIODIC, ps.HIMENO19)[i % 3]
        params = [0.8] if kind == ps.HIMENO19 else list(COEF)
        out.append(dict(kernel=kind, dims=dims, params=params, max_steps=int(rng.integers(20, 90)),
                        tol=(0.0, 2e-3, 0.3)[i % 3] if i % 4 else 0.0, check_every=int(rng.integers(1, 9)),
                        seed=1000 + i))
    return out


@pytest.mark.parametrize("periodic", [False, True])
def test_diffusion_against_oracle_with_stop(periodic):
    nx, ny, nz, ce, max_steps = 24, 20, 36, 5, 60
    u0 = np.random.default_rng(5).random((nz, ny, nx), dtype=np.float32)
    # Oracle residual at every check, and the tolerance between the 4th and 5th.
    states = [u0]
    for _ in range(max_steps):
        states.append(O.diffusion7(states[-1], 1, COEF, periodic=periodic))
    checks = list(range(ce, max_steps + 1, ce))
    res = {n: _diff_residual(states[n], states[n - 1]) for n in checks}
    tol = float(np.sqrt(res[checks[3]] * res[checks[4]]))
    stop = next(n for n in checks if res[n] <= tol)
    kind = ps.DIFFUSION7_PERIODIC if periodic else ps.DIFFUSION7
    reqs = [dict(kernel=kind, dims=(nx, ny, nz), params=list(COEF), max_steps=max_steps, tol=tol,
                 check_every=ce, init=u0),
            dict(kernel=kind, dims=(nx, ny, nz), params=list(COEF), max_steps=13, init=u0)]
    recs, outs, _ = _serve(reqs)
    assert recs[0]["steps_done"] == stop
    assert bits_equal(outs[0], states[stop])
    assert recs[0]["residual"] == pytest.approx(res[stop], rel=1e-9)
    assert recs[1]["steps_done"] == 13 and recs[1]["residual"] == -1.0
    assert bits_equal(outs[1], states[13])


def test_himeno_against_oracle_with_stop():
    shape = (21, 15, 17)
    p, coef = himeno_inputs(shape, 11)
    ce, max_steps = 4, 40
    _, gosa = O.himeno(p, coef, 0.8, max_steps)
    checks = [1] + list(range(ce, max_steps + 1, ce))
    res = {n: float(np.sqrt(gosa[n - 1] / gosa[0])) for n in checks}
    tol = float(np.sqrt(res[checks[3]] * res[checks[4]]))
    stop = next(n for n in checks if res[n] <= tol)
    want, _ = O.himeno(p, coef, 0.8, stop)
    nz, ny, nx = shape
    host_coef = np.ascontiguousarray(np.stack(coef))
    reqs = [dict(kernel=ps.HIMENO19, dims=(nx, ny, nz), params=[0.8], max_steps=max_steps,
                 tol=tol, check_every=ce, init=np.ascontiguousarray(p), coef=host_coef)]
    recs, outs, _ = _serve(reqs)
    assert recs[0]["steps_done"] == stop
    assert bits_equal(outs[0], want)
    assert recs[0]["residual"] == pytest.approx(res[stop], rel=1e-9)


def test_each_result_same_alone_and_in_mix():
    reqs = _mix()
    recs, outs, stats = _serve(reqs)
    assert stats["completed"] == len(reqs)
    stopped = 0
    for r, rec, out in zip(reqs, recs, outs):
        alone_recs, alone_outs, _ = _serve([r])
        assert alone_recs[0]["steps_done"] == rec["steps_done"], r
        assert alone_recs[0]["residual"] == rec["residual"], r
        assert bits_equal(alone_outs[0], out), r
        assert not np.isnan(out).any()
        stopped += rec["steps_done"] < r["max_steps"]
    assert stopped >= 2  # the mix exercises early stops


def test_fifo_baseline_equals_batched():
    reqs = _mix()
    recs, outs, _ = _serve(reqs)
    frecs, fouts, fstats = _serve(reqs, mode=ps.SERVE_FIFO)
    for r, a, b, oa, ob in zip(reqs, recs, frecs, outs, fouts):
        assert a["steps_done"] == b["steps_done"], r
        assert bits_equal(oa, ob), r
        if a["residual"] < 0:
            assert b["residual"] < 0
        else:
            assert b["residual"] == pytest.approx(a["residual"], rel=1e-9)
    # One launch per step (plus residual passes) in the baseline.
    assert fstats["launches"] >= sum(r["steps_done"] for r in frecs)
    # FIFO: requests finish in arrival order.
    fin = [r["finish_s"] for r in frecs]
    assert fin == sorted(fin)


def test_budget_and_slots():
    big = dict(kernel=ps.HIMENO19, dims=(64, 64, 64), params=[0.8], max_steps=30, seed=3)
    one = ps.Server.request_bytes(ps.Server.request(**big))
    assert one >= 14 * 64 ** 3 * 4
    reqs = [dict(big, seed=3 + i) for i in range(5)]
    recs, outs, stats = _serve(reqs, budget=2 * one + one // 2)
    assert stats["peak_bytes"] <= 2 * one + one // 2
    assert stats["peak_bytes"] >= one
    # Same results with one slot at a time.
    recs1, outs1, stats1 = _serve(reqs, slots=1)
    # One request advancing, at most one more whose result is being copied out.
    assert one <= stats1["peak_bytes"] <= 2 * one
    for a, b in zip(outs, outs1):
        assert bits_equal(a, b)
    # A request larger than the whole budget is refused at submit.
    s = ps.Server(one - 1)
    try:
        with pytest.raises(ps.PhysisError) as e:
            s.submit(**big)
        assert e.value.status == ps.PSB_ERR_NOMEM
    finally:
        s.destroy()


def test_invalid_requests_are_refused():
    s = ps.Server(GB)
    try:
        bad = [dict(kernel=ps.DIFFUSION7, dims=(2, 8, 8), params=list(COEF), max_steps=4),
               dict(kernel=ps.DIFFUSION7, dims=(8, 8, 8), params=list(COEF), max_steps=0),
               dict(kernel=ps.DIFFUSION7, dims=(8, 8, 8), params=[0.1], max_steps=4),
               dict(kernel=ps.DIFFUSION7, dims=(8, 8, 8), params=list(COEF), max_steps=4, tol=0.1)]
        for b in bad:
            with pytest.raises(ps.PhysisError) as e:
                s.submit(**b)
            assert e.value.status == ps.PSB_ERR_INVALID
        with pytest.raises(ps.PhysisError) as e:
            s.wait(12345, timeout=0.0)
        assert e.value.status == ps.PSB_ERR_INVALID
    finally:
        s.destroy()


def test_cancel_and_wait_timeout():
    long_req = dict(kernel=ps.HIMENO19, dims=(128, 128, 160), params=[0.8], max_steps=1000)
    s = ps.Server(16 * GB, 1)
    try:
        a = s.submit(seed=1, **long_req)
        b = s.submit(seed=2, **long_req)
        c = s.submit(seed=3, **long_req)
        with pytest.raises(ps.PhysisError) as e:
            s.wait(c, timeout=0.0)
        assert e.value.status == ps.PSB_ERR_TIMEOUT
        s.cancel(c)  # still queued behind a and b (one slot)
        rc = s.wait(c, timeout=5.0)
        assert rc["status"] == ps.PSB_ERR_CANCELLED and rc["steps_done"] == 0
        s.cancel(a)
        ra = s.wait(a, timeout=120.0)
        assert ra["status"] in (ps.PSB_ERR_CANCELLED, ps.PSB_OK)
        rb = s.wait(-1, timeout=120.0)
        assert rb["id"] == b and rb["status"] == ps.PSB_OK and rb["steps_done"] == 1000
    finally:
        s.destroy()


def test_continuous_admission_overlaps_requests():
    """Requests arriving while others run join them: the second request starts
    before the first finishes."""
    s = ps.Server(16 * GB)
    try:
        first = s.submit(kernel=ps.DIFFUSION7, dims=(384, 384, 384), params=list(COEF),
                         max_steps=1000, seed=9)
        time.sleep(0.02)
        second = s.submit(kernel=ps.DIFFUSION7, dims=(64, 64, 64), params=list(COEF),
                          max_steps=50, seed=10)
        r1 = s.wait(first, timeout=120.0)
        r2 = s.wait(second, timeout=120.0)
        assert r2["start_s"] < r1["finish_s"]
        assert r1["steps_done"] == 1000 and r2["steps_done"] == 50
        assert s.stats()["rounds"] >= 2
    finally:
        s.destroy()


def test_large_requests_take_the_wavefront_path():
    """Requests large enough for the batched kernel's per-tile dependencies
    (their steps overlap as a wavefront): a 200^3 clamped diffusion and a
    176x160x144 Himeno solve with a residual stop, served together with the
    small mix. Each equals the oracle, and equals itself served alone."""
    nd = (200, 200, 200)
    u0 = np.random.default_rng(23).random(tuple(reversed(nd)), dtype=np.float32)
    hd = (176, 160, 144)
    p, coef = himeno_inputs(tuple(reversed(hd)), 21)
    ce, max_steps = 5, 40
    _, gosa = O.himeno(p, coef, 0.8, max_steps)
    checks = [1] + list(range(ce, max_steps + 1, ce))
    res = {n: float(np.sqrt(gosa[n - 1] / gosa[0])) for n in checks}
    tol = float(np.sqrt(res[checks[3]] * res[checks[4]]))
    stop = next(n for n in checks if res[n] <= tol)
    big = [dict(kernel=ps.DIFFUSION7, dims=nd, params=list(COEF), max_steps=36, init=u0),
           dict(kernel=ps.HIMENO19, dims=hd, params=[0.8], max_steps=max_steps, tol=tol,
                check_every=ce, init=np.ascontiguousarray(p),
                coef=np.ascontiguousarray(np.stack(coef)))]
    recs, outs, _ = _serve(big + _mix())
    want = [O.diffusion7(u0, 36, np.asarray(COEF, np.float32)), O.himeno(p, coef, 0.8, stop)[0]]
    assert recs[0]["steps_done"] == 36
    assert recs[1]["steps_done"] == stop
    assert recs[1]["residual"] == pytest.approx(res[stop], rel=1e-9)
    for i in range(2):
        assert recs[i]["wave_rounds"] >= 1, recs[i]
        assert bits_equal(outs[i], want[i]), i
        alone_recs, alone_outs, _ = _serve([big[i]])
        assert alone_recs[0]["steps_done"] == recs[i]["steps_done"]
        assert alone_recs[0]["wave_rounds"] >= 1
        assert bits_equal(alone_outs[0], want[i]), i


def test_two_sweep_himeno_requests_match_one_sweep():
    """Himeno requests served on two sweeps per pass (tune entries with
    t_depth 2 for their size buckets) end with the same steps, residuals and
    fields as on the one-sweep kernel (a pass flips which grid holds the
    state; the server tracks it for the copy-out)."""
    def bucket(dims):
        return tuple(1 << max(3, (v - 1).bit_length()) for v in dims)

    reqs = [dict(kernel=ps.HIMENO19, dims=(96, 80, 72), params=[0.8], max_steps=150, tol=0.02,
                 check_every=10, seed=41),
            dict(kernel=ps.HIMENO19, dims=(40, 36, 30), params=[0.8], max_steps=33, seed=42),
            dict(kernel=ps.DIFFUSION7, dims=(50, 40, 30), params=list(COEF), max_steps=40,
                 seed=43)]
    base = _serve(reqs)
    try:
        for r in reqs:
            if r["kernel"] == ps.HIMENO19:
                ps.tune_set(102, ps.PS_FLOAT, bucket(r["dims"]), impl=ps.IMPL_TMA, tile_x=64,
                            tile_y=8, z_chunk=8, stages=6, t_depth=2)
        two = _serve(reqs)
    finally:
        for r in reqs:
            if r["kernel"] == ps.HIMENO19:
                ps.tune_set(102, ps.PS_FLOAT, bucket(r["dims"]), impl=ps.IMPL_TMA, tile_x=64,
                            tile_y=8, z_chunk=8, stages=6, t_depth=1)
    for a, b, oa, ob in zip(base[0], two[0], base[1], two[1]):
        assert a["steps_done"] == b["steps_done"]
        assert b["residual"] == pytest.approx(a["residual"], rel=1e-12)
        assert bits_equal(oa, ob)
