"""GPU: the request server (psg_server_*): continuous batching of count
requests from the serving distribution. Every result equals the per-range
count (psg_count) of the same request, whether the request ran alone on an
idle server or mixed with many others on a loaded one; admission refuses a
request whose bucket storage exceeds the HBM budget."""
import random

import pytest

pytestmark = pytest.mark.gpu


def _requests(psg, n, rate, seed=1):
    # the serving distribution with lengths capped at 2^30 to bound test time
    return psg.serving_workload(n, rate, seed=seed, len_log2=(12.0, 30.0))


def test_server_alone_equals_in_mix(psg, ctx):
    reqs, _ = _requests(psg, 120, 1000.0)
    with psg.Server(ctx) as srv:
        alone = []
        for a, b, k in reqs:
            counts, lat = srv.wait(srv.submit(a, b, k))
            assert lat >= 0
            alone.append(counts)
        # all at once: every request shares steps with the others
        mixed, lats = srv.replay(reqs, [0.0] * len(reqs))
        st = srv.stats()
    assert mixed == alone
    assert st["completed"] == 2 * len(reqs)
    assert st["bucket_requests"] > 0 and st["batch_requests"] > 0
    for (a, b, k), got in random.Random(5).sample(list(zip(reqs, alone)), 25):
        assert got == ctx.count(a, b, k), (a, b, k)


def test_server_poisson_replay(psg, ctx):
    reqs, arrivals = _requests(psg, 200, 2000.0, seed=11)
    with psg.Server(ctx) as srv:
        counts, lats = srv.replay(reqs, arrivals)
    assert len(lats) == len(reqs) and min(lats) > 0
    for (a, b, k), got in list(zip(reqs, counts))[::8]:
        assert got == ctx.count(a, b, k), (a, b, k)


def test_server_trivial_requests(psg, ctx):
    with psg.Server(ctx) as srv:
        cases = [(10, 5, 63), (0, 0, 63), (0, 6, 63), (2, 3, 1), (0, 100, 0), (3, 5, 2),
                 (2 ** 64 - 1, 2 ** 64 - 1, 63), (0, 10 ** 6, 63)]
        ids = [srv.submit(a, b, k) for a, b, k in cases]
        for (a, b, k), i in zip(cases, ids):
            assert srv.wait(i)[0] == ctx.count(a, b, k), (a, b, k)


def test_server_refuses_over_hbm_budget(psg, ctx):
    with psg.Server(ctx, hbm_budget=1 << 20) as srv:
        big = srv.submit(10 ** 18, 10 ** 18 + 10 ** 10, 1)      # needs bucket lists
        small = srv.submit(10 ** 9, 10 ** 9 + 10 ** 6, 1)       # batch kernel only
        with pytest.raises(psg.PsgError) as e:
            srv.wait(big)
        assert e.value.status == 4 and "HBM budget" in str(e.value)
        assert srv.wait(small)[0] == ctx.count(10 ** 9, 10 ** 9 + 10 ** 6, 1)
        assert srv.stats()["refused"] == 1


def test_server_each_id_collected_once(psg, ctx):
    """Two waits for one request, concurrent or one after the other: exactly
    one gets the counts, the other fails with PSG_ERR_ARG (1)."""
    import threading
    a, b = 10 ** 15, 10 ** 15 + 10 ** 10
    want = ctx.count(a, b, 1)
    with psg.Server(ctx) as srv:
        rid = srv.submit(a, b, 1)
        results = []

        def waiter():
            try:
                results.append(srv.wait(rid)[0])
            except psg.PsgError as e:
                results.append(e.status)

        threads = [threading.Thread(target=waiter) for _ in range(2)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        assert sorted(results, key=str) == sorted([want, 1], key=str)
        with pytest.raises(psg.PsgError) as e:
            srv.wait(rid)
        assert e.value.status == 1


def test_closing_the_context_stops_its_server(psg):
    """A server keeps its context alive and closing the context stops the
    server first (its worker thread uses the engine)."""
    c = psg.Context()
    srv = psg.Server(c)
    rid = srv.submit(10 ** 12, 10 ** 12 + 10 ** 8, 1)
    assert srv.wait(rid)[0][0] == c.count(10 ** 12, 10 ** 12 + 10 ** 8, 1)[0]
    c.close()
    assert srv._h is None
    with pytest.raises(psg.PsgError) as e:
        srv.submit(0, 100, 1)      # stopped: a NULL server handle
    assert e.value.status == 1


def test_failed_step_leaves_no_waiter_blocked(psg, ctx):
    """A step that fails while planning its admitted requests (injected on the
    host: the second request planned makes its step fail with
    PSG_ERR_CUDA, 3) completes every request of that step -- the ones it had
    planned and the ones it had not reached -- with the error, and the
    server goes on serving."""
    import threading
    reqs = [(10 ** 12 + i * 10 ** 7, 10 ** 12 + (i + 1) * 10 ** 7, 1) for i in range(8)]
    with psg.Server(ctx) as srv:
        srv.inject_failure(2, 3)
        out = [None] * len(reqs)

        def run():
            try:
                out[:] = srv.replay(reqs, [0.0] * len(reqs))[0]
            except psg.PsgError as e:
                out[:] = [e.status] * len(reqs)

        t = threading.Thread(target=run, daemon=True)
        t.start()
        t.join(timeout=120)
        assert not t.is_alive(), "a waiter stayed blocked after the failed step"
        assert out[0] == 3                   # replay reports the first failure
        st = srv.stats()
        assert st["completed"] + st["refused"] == st["submitted"] == len(reqs)
        assert st["refused"] >= 1
        rid = srv.submit(*reqs[0])
        assert srv.wait(rid)[0] == ctx.count(*reqs[0])
