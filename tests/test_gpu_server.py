"""The query server on the GPU: queries arriving while others run are admitted
into later rounds and share launches with them; every result must equal the
same request computed alone by dd_histogram (bit-exact: integer histograms)."""
import random
import threading
import time

import pytest

import coding_reliability_b200 as dd

pytestmark = pytest.mark.gpu


def mixed_requests(count=40, seed=7):
    rng = random.Random(seed)
    out = []
    for i in range(count):
        A = rng.randrange(129, 1 << 16) | 1
        k = rng.choice([8, 12, 16, 18, 20])
        kind = rng.random()
        if kind < 0.6:
            q = dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, A, k)
        elif kind < 0.8:
            q = dd.Request(dd.CODE_AN, dd.MODE_GRID_1D, A, k, m=1 << max(3, k - 8))
        elif kind < 0.95:
            q = dd.Request(dd.CODE_AN, dd.MODE_MONTE_CARLO, A, k, m=1 << rng.randrange(2, 8), seed=i)
        else:
            q = dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, 16, with_1bit=1)
        q.user_tag = i
        out.append(q)
    return out


def test_server_mix_equals_alone(ctx):
    reqs = mixed_requests()
    alone = [ctx.histogram(q) for q in reqs]
    rng = random.Random(11)
    with dd.Server(0, round_ms=10) as s:
        tickets = []

        def client():
            for q in reqs:
                tickets.append(s.submit(q))
                time.sleep(rng.expovariate(400.0))  # Poisson arrivals, 400/s

        th = threading.Thread(target=client)
        th.start()
        th.join()
        results = [s.wait(t, 120) for t in tickets]
        stats = s.stats()
    for q, (st, r), a in zip(reqs, results, alone):
        assert st == 0, q
        assert r.counts == a.counts and r.raw == a.raw and r.user_tag == q.user_tag, q
    assert stats["completed"] == len(reqs) and stats["rounds"] >= 1
    assert stats["p50_ms"] > 0 and stats["p99_ms"] >= stats["p50_ms"]


def test_server_small_queries_overlap_a_large_one(ctx):
    big = dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 58659, 23)      # 3.5e13 pairs: seconds of device time
    smalls = [dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, A, 14) for A in (641, 1021, 32771, 65521)]
    with dd.Server(0, round_ms=20) as s:
        tb = s.submit(big)
        time.sleep(0.1)
        ts = [s.submit(q) for q in smalls]
        for t, q in zip(ts, smalls):
            st, r = s.wait(t, 60)
            assert st == 0 and r.counts == ctx.histogram(q).counts
        assert s.poll(tb) is None  # the big query is still running while the small ones finished
        st, r = s.wait(tb, 120)
        assert st == 0 and r.counts == ctx.histogram(big).counts


def test_server_large_queries_mix_equals_alone(ctx):
    """The large query classes of the serving mix, each running over many
    rounds beside small queries that arrive meanwhile: the k=24 grid with stride
    2^(k-16) (m = 2^16 lattice points, 2^40 pairs) and Monte Carlo with 2^32
    Philox-drawn pairs at k=24 and k=26.  Every result equals the same request
    run alone."""
    big = [dd.Request(dd.CODE_AN, dd.MODE_GRID_1D, 58659, 24, m=1 << 16),
           dd.Request(dd.CODE_AN, dd.MODE_GRID_1D, 1021, 24, m=1 << 16),
           dd.Request(dd.CODE_AN, dd.MODE_MONTE_CARLO, 32771, 24, m=(1 << 32) >> 24, seed=5),
           dd.Request(dd.CODE_AN, dd.MODE_MONTE_CARLO, 641, 26, m=(1 << 32) >> 26, seed=6)]
    small = [dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, A, k) for A, k in ((641, 12), (58659, 16), (255, 20))]
    reqs = big + small
    for i, q in enumerate(reqs):
        q.user_tag = i
    alone = [ctx.histogram(q) for q in reqs]
    with dd.Server(0, round_ms=10) as s:
        tickets = [s.submit(q) for q in big]
        time.sleep(0.05)
        tickets += [s.submit(q) for q in small]
        results = [s.wait(t, 300) for t in tickets]
        stats = s.stats()
    for q, (st, r), a in zip(reqs, results, alone):
        assert st == 0, q
        assert r.counts == a.counts and r.raw == a.raw and r.user_tag == q.user_tag, q
    assert stats["rounds"] > len(reqs)  # the large queries were split over many rounds
