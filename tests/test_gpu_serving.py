"""Serving loop (cps_server_*): continuous batching of jobs that arrive while
others run, admission against a memory budget, per-job failure isolation and
cancellation; every job's result is the same alone and in the mix."""
import numpy as np
import pytest

from cpsfdtd_b200 import decks

pytestmark = pytest.mark.gpu


def _job_decks():
    """Three material mixes (dielectric, Drude-Lorentz + TF/SF, gain) with
    different sizes and step counts, so jobs retire at different chunks."""
    a = decks.config1(n=40, steps=150)
    b = decks.config2(n=36, steps=97, nfreq=3)
    c = decks.config4_member(48, 40, 44, seed=5, steps=130, nfreq=4)
    d = decks.config3(n=34, steps=61, nfreq=2)
    return [(a, 150), (b, 97), (c, 130), (d, 61)]


def _result(g):
    out = {"fields": g.fields(), "step": g.get_step()}
    out["dft"] = [g.port_dft(p, raw=True).copy() for p in range(len(g.ports)) if g.ports[p][2] > 0]
    return out


def _serve(cps, jobs, arrivals, chunk=64, budget=8 * 10 ** 9, max_jobs=16, polls_between=1, tile=None):
    """Submit job n after arrivals[n] polls; returns {index: (status, result)}."""
    srv = cps.Server(cps.FP32, max_jobs=max_jobs, budget_bytes=budget, chunk_steps=chunk, tile=tile)
    res = {}
    order = sorted(range(len(jobs)), key=lambda n: arrivals[n])
    polls = 0
    nxt = 0
    while nxt < len(order) or len(res) < len(jobs):
        while nxt < len(order) and arrivals[order[nxt]] <= polls:
            n = order[nxt]
            dk, steps = jobs[n]

            def done(g, status, n=n):
                res[n] = (status, _result(g) if (g is not None and status == 0) else None)

            srv.submit(lambda dk=dk: cps.Grid.from_deck(dk, cps.FP32), done, steps, cps.footprint(dk))
            nxt += 1
        srv.poll()
        polls += 1
        assert polls < 10000
    st = srv.stats()
    srv.close()
    return res, st


def _same(a, b):
    assert a["step"] == b["step"]
    for c in range(6):
        assert np.array_equal(a["fields"][c], b["fields"][c])
    for x, y in zip(a["dft"], b["dft"]):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("tile", [None, (4, 8, 0)])
def test_alone_equals_mix(tile):
    """Default batch tiling (each member's own sweep launches) and the class
    launches over a shared tile table give the same per-job results."""
    import cpsfdtd_b200 as cps
    jobs = _job_decks()
    alone = {}
    for n, job in enumerate(jobs):
        r, st = _serve(cps, [job], [0], tile=tile)
        assert r[0][0] == 0 and st["jobs_done"] == 1
        alone[n] = r[0][1]
    # the same jobs arriving while others run, with a chunk that splits them
    mix, st = _serve(cps, jobs, [0, 1, 3, 4], chunk=24, tile=tile)
    assert st["jobs_done"] == len(jobs) and st["jobs_failed"] == 0
    assert st["latency_p99_ms"] >= st["latency_p50_ms"] > 0
    for n in range(len(jobs)):
        assert mix[n][0] == 0
        _same(alone[n], mix[n][1])
    # and against a grid stepped on its own, outside the server
    dk, steps = jobs[1]
    g = cps.Grid.from_deck(dk, cps.FP32)
    g.step(steps, cps.FUSED)
    _same(_result(g), mix[1][1])


def test_admission_budget_and_rejection():
    import cpsfdtd_b200 as cps
    jobs = _job_decks()
    fps = [cps.footprint(dk) for dk, _ in jobs]
    budget = max(fps) + min(fps)  # never room for all of them at once
    srv = cps.Server(cps.FP32, max_jobs=8, budget_bytes=budget, chunk_steps=32)
    seen_peak = 0
    done = {}
    for n, (dk, steps) in enumerate(jobs):
        srv.submit(lambda dk=dk: cps.Grid.from_deck(dk, cps.FP32),
                   lambda g, s, n=n: done.__setitem__(n, s), steps, fps[n])
    big = srv.submit(lambda: cps.Grid.from_deck(jobs[0][0], cps.FP32),
                     lambda g, s: done.__setitem__("big", s), 10, budget + 1)
    while len(done) < len(jobs) + 1:
        srv.poll()
        st = srv.stats()
        seen_peak = max(seen_peak, st["bytes_in_use"])
        assert st["bytes_in_use"] <= budget * 1.5  # charged: max(estimate, actual)
    st = srv.stats()
    assert done["big"] == cps.CPS_E_BUDGET and st["jobs_rejected"] == 1
    assert all(done[n] == 0 for n in range(len(jobs)))
    assert st["jobs_done"] == len(jobs)
    assert big > 0 and seen_peak > 0
    srv.close()


def test_failed_build_and_cancel_are_isolated():
    import cpsfdtd_b200 as cps
    jobs = _job_decks()
    srv = cps.Server(cps.FP32, max_jobs=8, budget_bytes=8 * 10 ** 9, chunk_steps=16)
    status = {}

    def bad_build():
        raise ValueError("malformed deck")

    def rec(key):
        return lambda g, s: status.__setitem__(key, s)

    ok = srv.submit(lambda: cps.Grid.from_deck(jobs[0][0], cps.FP32), rec("ok"), 40, 10 ** 8)
    bad = srv.submit(bad_build, rec("bad"), 40, 10 ** 8)
    live_cancel = srv.submit(lambda: cps.Grid.from_deck(jobs[3][0], cps.FP32), rec("live"), 1000, 10 ** 8)
    srv.poll()
    srv.cancel(live_cancel)
    queued = srv.submit(lambda: cps.Grid.from_deck(jobs[2][0], cps.FP32), rec("queued"), 40, 10 ** 8)
    srv.cancel(queued)
    with pytest.raises(cps.CpsError):
        srv.cancel(123456)
    srv.drain()
    assert status["ok"] == 0
    assert status["bad"] == cps.CPS_E_INVALID and "malformed" in srv.errors[bad]
    assert status["live"] == cps.CPS_E_CANCELLED
    assert status["queued"] == cps.CPS_E_CANCELLED
    st = srv.stats()
    assert st["jobs_done"] == 1 and st["jobs_failed"] == 1 and st["jobs_cancelled"] == 2
    assert ok > 0
    srv.close()
