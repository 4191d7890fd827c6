"""The serving loop (rq_server_*): requests of mixed mesh classes submitted while
others are on the GPU are admitted as slots free up, and each result equals the
same request evaluated alone by ForwardBatch.evaluate. The tolerance is 1e-12
relative on predictions and loglik (the serving kernel runs the same per-solve
code at the same CTA size, so the results are expected to be bitwise equal),
and status and iteration count must match exactly. Failed requests are flagged
(status, sentinel loglik, no predictions), not returned.
"""
import time

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def classes(rq):
    """Three mesh classes: two small channels and a capped bump (never converges)."""
    a = cases.product_batch(rq, cases.small_channel())
    b = cases.product_batch(rq, cases.small_channel(ny=32, max_iter=60000))
    c = cases.product_batch(rq, cases.bump_case(24, 16, max_iter=150))
    return [a, b, c]


def stream(n=24, seed=7):
    """Request mix: class per request, theta, with two out-of-bounds (poisoned) rows."""
    rng = np.random.default_rng(seed)
    cls = rng.choice(3, size=n, p=[0.45, 0.35, 0.20])
    theta = np.column_stack([rng.uniform(0.29, 0.33, n), rng.uniform(0.086, 0.094, n)])
    theta[5] = (0.95, 0.09)   # a1 above its bound 0.8 -> InvalidParameters
    theta[17] = (0.31, 0.5)   # beta* above its bound 0.2 -> InvalidParameters
    return cls, theta


def alone(batches, cls, theta):
    return [batches[c].evaluate(theta[i:i + 1]).rows[0].result for i, c in enumerate(cls)]


def check_same(served, ref):
    assert served.status == ref.status, (served.ticket, served.status, ref.status)
    assert served.iterations == ref.simple_iters
    if ref.status.name == "Converged":
        np.testing.assert_allclose(served.predictions, ref.predictions, rtol=RTOL, atol=0)
        assert abs(served.log_lik - ref.log_lik) <= RTOL * abs(ref.log_lik)
    else:
        assert served.flagged and served.predictions is None
        assert served.log_lik == ref.log_lik  # the reference's sentinels


def test_served_results_equal_alone_results(rq):
    batches = classes(rq)
    cls, theta = stream()
    srv = rq.ForwardServer(batches, capacity=64, idle_timeout=5.0)
    tickets = []
    for i in range(len(cls)):
        tickets.append(srv.submit(int(cls[i]), theta[i]))
        if i % 4 == 3:
            time.sleep(0.05)  # arrivals while earlier requests run
    assert srv.wait(600.0) == len(cls)
    served = [srv.poll(t) for t in tickets]
    info = srv.info()
    srv.destroy()
    ref = alone(batches, cls, theta)
    for s, r in zip(served, ref):
        check_same(s, r)
    assert served[5].status.name == "InvalidParameters" and served[5].log_lik == -1e30
    assert served[17].status.name == "InvalidParameters"
    # the bump class is capped below the solver's 505-iteration start-up: never converged
    assert all(s.flagged and s.predictions is None for s, c in zip(served, cls) if c == 2)
    assert info["completed"] == len(cls) and info["slots"] >= 1
    # requests overlapped on the device: some solve started before another ended
    spans = sorted((s.start_ns, s.end_ns) for s in served if s.iterations > 0)
    assert any(b[0] < a[1] for a, b in zip(spans, spans[1:]))


def test_idle_exit_and_relaunch(rq):
    batches = classes(rq)[:1]
    srv = rq.ForwardServer(batches, capacity=8, idle_timeout=0.2)
    t0 = srv.submit(0, (0.31, 0.09))
    assert srv.wait(300.0) == 1
    time.sleep(1.0)  # the kernel's CTAs leave after 0.2 s without requests
    t1 = srv.submit(0, (0.30, 0.088))
    assert srv.wait(300.0) == 2
    r0, r1 = srv.poll(t0), srv.poll(t1)
    assert srv.info()["launches"] >= 2
    srv.destroy()
    ref = alone(batches, [0, 0], np.array([(0.31, 0.09), (0.30, 0.088)]))
    check_same(r0, ref[0])
    check_same(r1, ref[1])


def test_close_drains_and_rejects_new_requests(rq):
    batches = classes(rq)[:1]
    srv = rq.ForwardServer(batches, capacity=8, idle_timeout=5.0, max_slots=2)
    ts = [srv.submit(0, (0.30 + 0.005 * i, 0.09)) for i in range(4)]
    srv.close()
    with pytest.raises(ValueError):
        srv.submit(0, (0.31, 0.09))
    assert srv.wait(300.0) == 4
    assert srv.info()["slots"] == 2
    assert all(srv.poll(t) is not None for t in ts)
    srv.destroy()


def test_served_far_off_draws_get_the_reference_verdicts(rq):
    """In-bounds draws far from the calibration box (a1 or beta* at the edge of its
    admissible range) do not converge within the cap; served among in-box draws that
    do, every request must come back with the compiled reference's own verdict and
    iteration count for the same draw (tests/golden/serve_failures_ref.json, made by
    tests/golden/make_serve_failures.py from oracle/_ref), the failed ones flagged with
    no predictions returned."""
    import json

    g = json.loads(open(cases.__file__.replace("cases.py", "golden/serve_failures_ref.json")).read())
    batch = cases.product_batch(rq, cases.small_channel(max_iter=g["cap"]))
    srv = rq.ForwardServer([batch], capacity=32, idle_timeout=5.0)
    tickets = [srv.submit(0, r["theta"]) for r in g["rows"]]
    assert srv.wait(600.0) == len(tickets)
    served = [srv.poll(t) for t in tickets]
    srv.destroy()
    assert sum(r["status"] != "Converged" for r in g["rows"]) >= 3
    for s, r in zip(served, g["rows"]):
        assert s.status.name == r["status"], (r["theta"], s.status.name, r["status"])
        if r["status"] == "Converged":
            assert abs(s.iterations - r["iterations"]) <= 0.02 * r["iterations"]
            assert not s.flagged and s.predictions is not None
        else:
            assert s.iterations == r["iterations"] == g["cap"]
            assert s.flagged and s.predictions is None


def test_admission_by_pool_space(rq):
    """A workspace pool that holds two solves of the class: six requests submitted at
    once are admitted two at a time, in submission order, as earlier solves retire and
    return their regions; at no moment do more than two solves run, every result
    equals the same request evaluated alone, and the pool is empty at the end."""
    batch = cases.product_batch(rq, cases.small_channel(max_iter=3000))
    ws = batch._problem.workspace_bytes()
    pool = 2 * ((ws + 255) // 256 * 256)
    srv = rq.ForwardServer([batch], capacity=16, idle_timeout=5.0, pool_bytes=pool)
    theta = np.column_stack([np.linspace(0.29, 0.33, 6), np.linspace(0.086, 0.094, 6)])
    tickets = [srv.submit(0, t) for t in theta]
    mem = srv.memory()
    assert mem["pool_bytes"] == pool
    assert mem["waiting"] >= 3 and mem["in_use_bytes"] <= pool
    assert srv.wait(600.0) == len(tickets)
    served = [srv.poll(t) for t in tickets]
    mem = srv.memory()
    srv.destroy()
    assert mem["waiting"] == 0 and mem["in_use_bytes"] == 0
    ref = alone([batch], [0] * 6, theta)
    for s, r in zip(served, ref):
        check_same(s, r)
    # never more than two solves at once, and starts follow submission order
    ev = sorted([(s.start_ns, 1) for s in served] + [(s.end_ns, -1) for s in served])
    live, peak = 0, 0
    for _, d in ev:
        live += d
        peak = max(peak, live)
    assert peak <= 2


def test_top_up_while_a_long_solve_runs(rq):
    """CTAs that leave after the idle timeout while another CTA is still in a long
    solve are replaced beside it: a request submitted then starts before the long
    solve ends, instead of waiting for the whole kernel to finish."""
    long_batch = cases.product_batch(rq, cases.small_channel(max_iter=60000, tol=1e-14))
    short_batch = cases.product_batch(rq, cases.small_channel(max_iter=200))
    srv = rq.ForwardServer([long_batch, short_batch], capacity=8, idle_timeout=0.2)
    t_long = srv.submit(0, (0.31, 0.09))
    time.sleep(1.5)  # every other CTA leaves after 0.2 s without requests
    t_short = srv.submit(1, (0.30, 0.088))
    assert srv.wait(600.0) == 2
    r_long, r_short = srv.poll(t_long), srv.poll(t_short)
    info = srv.info()
    srv.destroy()
    assert info["launches"] >= 2
    assert r_short.start_ns < r_long.end_ns
    assert r_short.end_ns < r_long.end_ns
