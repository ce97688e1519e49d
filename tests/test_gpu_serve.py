"""The request server (continuous batching) on the GPU.

Checked: a request gives the same bits (solution, IER, iteration count) when
solved alone by the one-shot batch solver, alone through the server, and in a
mix it joins while other requests are already iterating; the FP64 server
equals the FP64 drop-in; a mixed request whose FP32 iteration cannot run
(residual beyond FP32 range) moves to the FP64 batch and equals the one-shot
mixed solve, which hands over the same way; admission never holds more device
memory than the budget; the copy-back / device-pointer flags; submits from
several threads; withdrawing queued requests, wait_any and the counters.
"""
import threading

import numpy as np
import pytest

import oracle as O
from mfix_b200 import leq
from mfix_b200 import systems as S

pytestmark = pytest.mark.gpu


def _true_rel(s, x):
    ref = s.copy()
    O.scale(ref)
    return O.true_resid(ref, x) / O.true_resid(ref, np.zeros(s.n))


def _others():
    sizes = [(18, 22, 16), (30, 14, 12), (12, 40, 10), (24, 24, 24), (9, 31, 20), (26, 12, 30)]
    out = [S.conv_diff(*d, seed=50 + q) for q, d in enumerate(sizes)]
    out += [S.pressure_like(26, 30, 22, seed=60 + q, nspheres=4, rmin=2, rmax=5, itmax=3000) for q in range(3)]
    out.append(S.conv_diff(40, 33, 1, seed=70, do_k=False))
    return out


@pytest.mark.parametrize("precision", [1, 0])
def test_alone_equals_in_mix(cuda, precision):
    target = S.conv_diff(22, 34, 18, seed=101)
    alone = target.copy()
    rc, res = leq.batch_solve([alone], precision=precision)
    assert rc == 0 and res[0].ier == 0, leq.last_error()

    with leq.Server(precision=precision) as srv:
        solo = target.copy()
        r_solo = srv.wait(srv.submit(solo), 120)
    assert r_solo is not None and r_solo["ier"] == 0

    others = _others()
    with leq.Server(precision=precision, check_every=2) as srv:
        tickets = [srv.submit(o) for o in others]
        assert min(tickets) >= 0
        # join the target once the others are iterating
        for _ in range(2000):
            states = [srv.poll(t) for t in tickets[:3]]
            if any(s is not None for s in states):
                break
            c = srv.counters()
            if c["running"] >= len(others) - 2:
                break
            threading.Event().wait(0.001)
        mixed_in = target.copy()
        tt = srv.submit(mixed_in)
        r_mix = srv.wait(tt, 120)
        r_oth = [srv.wait(t, 300) for t in tickets]
        cnt = srv.counters()
    assert r_mix is not None and all(r is not None for r in r_oth)
    assert np.array_equal(alone.x, solo.x)
    assert np.array_equal(alone.x, mixed_in.x)
    assert r_solo["iterations"] == r_mix["iterations"] == res[0].iterations
    assert r_mix["ier"] == 0 and _true_rel(target, mixed_in.x) <= target.tol * 1.01
    # it was a mix: other requests were in the batch while the target iterated
    overlap = [r for r in r_oth if r["t_start"] < r_mix["t_done"] and r["t_done"] > r_mix["t_start"]]
    assert overlap, "no request overlapped the target"
    assert cnt["max_running"] >= 2 and cnt["commits"] >= 2
    for o, r in zip(others, r_oth):
        assert r["ier"] == 0, r
        assert _true_rel(o, o.x) <= o.tol * 1.01


def test_fp64_server_equals_drop_in(cuda):
    systems = [S.conv_diff(15, 19, 13, seed=3), S.known_answer(12, 14, 10, seed=4)[0],
               S.conv_diff(33, 27, 1, seed=5, do_k=False)]
    ref = [s.copy() for s in systems]
    for r in ref:
        assert leq.solve_system(r) == 0
    with leq.Server(precision=0) as srv:
        got = [s.copy() for s in systems]
        ts = [srv.submit(g, write_ab=True) for g in got]
        rs = [srv.wait(t, 60) for t in ts]
    for r, g, res in zip(ref, got, rs):
        assert res["ier"] == 0
        assert np.array_equal(r.x, g.x)
        assert np.array_equal(r.a, g.a) and np.array_equal(r.b, g.b)  # unit-scaled A/B written back


def test_mixed_hands_over_beyond_fp32_range(cuda):
    """A residual beyond FP32 range (B ~ 1e40) makes the FP32 iteration fail;
    the request is re-solved by the FP64 batch from its initial guess."""
    s = S.conv_diff(14, 20, 12, seed=7)
    s.b *= 1e40
    one = s.copy()
    rc, res = leq.batch_solve([one], precision=1)
    assert rc == 0 and res[0].fp64_fallback == 1 and res[0].ier == 0
    ref = s.copy()
    st = O.leq_bicgs(ref)
    assert st["ier"] == 0
    with leq.Server(precision=1) as srv:
        mix = [S.conv_diff(20, 18, 16, seed=8), S.conv_diff(10, 26, 9, seed=9)]
        ts = [srv.submit(m) for m in mix]
        got = s.copy()
        r = srv.wait(srv.submit(got), 120)
        rm = [srv.wait(t, 60) for t in ts]
        cnt = srv.counters()
    assert r["fp64_fallback"] == 1 and r["ier"] == 0 and r["mixed_iterations"] >= 0
    assert np.array_equal(got.x, one.x)
    assert r["iterations"] == res[0].iterations
    assert cnt["fp64_fallbacks"] == 1
    assert all(x["ier"] == 0 and x["fp64_fallback"] == 0 for x in rm)
    assert _true_rel(s, got.x) <= s.tol * 1.01


def test_budget_admission(cuda):
    systems = [S.conv_diff(20, 20, 20, seed=20 + q) for q in range(6)]
    n = systems[0].n
    per = (72 + 110) * n  # inputs plus a generous bound on the work block
    with leq.Server(precision=1, hbm_budget=2.2 * per) as srv:
        big = S.conv_diff(40, 40, 40, seed=1)
        assert srv.submit(big) == leq.IER_NOMEM  # larger than the whole budget
        ts = [srv.submit(s) for s in systems]
        rs = [srv.wait(t, 120) for t in ts]
        c = srv.counters()
    assert all(r["ier"] == 0 for r in rs)
    assert c["peak_reserved_bytes"] <= c["budget_bytes"]
    assert c["max_running"] <= 2
    # the later requests waited for memory: admitted only after earlier ones finished
    assert rs[-1]["t_admit"] >= min(r["t_done"] for r in rs[:2]) - 1e-3


def test_device_pointers_and_zero_guess(cuda):
    torch = cuda
    s = S.conv_diff(16, 18, 14, seed=30)
    host = s.copy()
    with leq.Server(precision=1) as srv:
        r_host = srv.wait(srv.submit(host, zero_guess=True), 60)
        da = torch.from_numpy(s.a.copy()).cuda()
        db = torch.from_numpy(s.b.copy()).cuda()
        dx = torch.full((s.n,), 7.0, dtype=torch.float64, device="cuda")  # ignored: zero guess
        t = srv.submit(s, zero_guess=True, on_device=True,
                       pointers=(da.data_ptr(), db.data_ptr(), dx.data_ptr()))
        r_dev = srv.wait(t, 60)
    assert r_host["ier"] == r_dev["ier"] == 0
    assert np.array_equal(dx.cpu().numpy(), host.x)
    scaled = s.copy()
    O.scale(scaled)
    assert np.array_equal(da.cpu().numpy(), scaled.a)  # solved in place: A scaled on the device


def test_concurrent_submitters(cuda):
    systems = [S.conv_diff(10 + q, 12 + 2 * q, 9 + q, seed=40 + q) for q in range(8)]
    results = {}
    with leq.Server(precision=1, max_systems=4) as srv:
        def client(idx):
            for q in idx:
                results[q] = srv.wait(srv.submit(systems[q]), 120)

        th = [threading.Thread(target=client, args=(list(range(k, 8, 2)),)) for k in range(2)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        c = srv.counters()
    assert sorted(results) == list(range(8))
    assert all(r["ier"] == 0 for r in results.values())
    assert c["completed"] == 8 and c["max_running"] <= 4


def test_batch_mixes_2d_and_3d(cuda):
    systems = [S.conv_diff(21, 19, 1, seed=80, do_k=False), S.conv_diff(11, 13, 9, seed=81),
               S.conv_diff(30, 17, 1, seed=82, do_k=False)]
    alone = [s.copy() for s in systems]
    for a in alone:
        rc, _ = leq.batch_solve([a], precision=0)
        assert rc == 0
    together = [s.copy() for s in systems]
    rc, res = leq.batch_solve(together, precision=0)
    assert rc == 0 and all(r.ier == 0 for r in res)
    for a, t in zip(alone, together):
        assert np.array_equal(a.x, t.x)


def test_cancel_queued_and_wait_any(cuda):
    """Requests not yet admitted can be withdrawn (IER -17); admitted ones finish;
    wait_any hands out every finished request once; the counters add up."""
    systems = [S.conv_diff(30, 30, 30, seed=90 + q) for q in range(10)]
    per = (72 + 110) * systems[0].n
    with leq.Server(precision=1, hbm_budget=1.5 * per) as srv:  # one request on the device at a time
        ts = [srv.submit(s) for s in systems]
        for _ in range(5000):  # withdraw once the first request has been admitted
            c = srv.counters()
            if c["copying"] + c["running"] + c["completed"] >= 1:
                break
            threading.Event().wait(0.001)
        srv.cancel_queued()
        got = {}
        while len(got) < len(ts):
            r = srv.wait_any(60)
            assert r is not None
            t, res = r
            assert t not in got
            got[t] = res
        c = srv.counters()
    iers = [got[t]["ier"] for t in ts]
    assert all(i in (0, leq.IER_CANCELLED) for i in iers)
    assert iers.count(leq.IER_CANCELLED) >= 1 and iers.count(0) >= 1
    for t, s in zip(ts, systems):
        if got[t]["ier"] == 0:
            assert got[t]["t_submit"] <= got[t]["t_admit"] <= got[t]["t_start"] <= got[t]["t_done"]
            assert O.true_resid(_scaled(s), s.x) / O.true_resid(_scaled(s), np.zeros(s.n)) <= s.tol * 1.01
    assert c["completed"] == c["submitted"] == len(ts)
    assert c["queued"] == c["copying"] == c["running"] == 0
    assert c["busy_ms"][0] > 0 and c["iterations"] > 0 and c["kernel_launches"] > 0


def _scaled(s):
    t = s.copy()
    O.scale(t)
    return t
