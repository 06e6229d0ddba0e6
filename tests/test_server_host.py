"""Host logic of the query server, run without a device (dry_run: rounds
advance cursors and take round_ms of simulated device time).  Faults are made
on the host only: an injected allocation failure, a budget below one slot,
malformed requests, a full queue, clients that go away, a shutdown with work
pending."""
import threading
import time

import pytest

import coding_reliability_b200 as dd

SLOT = 64 * 8 + 160 + 16  # bins + job entry + cursor, per query (matches kSlotBytes to within the Job size)


def small(A=641, n=12, **kw):
    return dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, A, n, **kw)


def big():
    return dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 58659, 24)  # ~1700 simulated rounds


def test_injected_allocation_failure(lib):
    with pytest.raises(dd.DDError) as e:
        dd.Server(dry_run=True, inject_alloc_failure=True)
    assert e.value.status == 5


def test_budget_below_one_slot(lib):
    with pytest.raises(dd.DDError) as e:
        dd.Server(dry_run=True, memory_budget_bytes=100)
    assert e.value.status == 5


def test_malformed_requests_refused_at_submit(lib):
    with dd.Server(dry_run=True, round_ms=1) as s:
        for bad, st in ((dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, 12), 2),
                        (dd.Request(dd.CODE_AN, dd.MODE_GRID_1D, 61, 16, m=1), 1),
                        (dd.Request(9, dd.MODE_EXHAUSTIVE, 61, 16), 1)):
            with pytest.raises(dd.DDError) as e:
                s.submit(bad)
            assert e.value.status == st
        assert s.stats()["submitted"] == 0


def until(cond, timeout_s=10.0):
    """Polls cond() until it holds (the scheduler thread runs on its own time)."""
    end = time.monotonic() + timeout_s
    while not cond():
        assert time.monotonic() < end, "condition not reached"
        time.sleep(0.002)


def test_admission_by_slots_and_queue_bound(lib):
    # one slot, queue of two: the big query holds the slot, two wait, the rest are refused
    with dd.Server(dry_run=True, round_ms=5, memory_budget_bytes=1000, max_queue=2) as s:
        assert s.stats()["slots"] == 1
        t_big = s.submit(big())
        until(lambda: s.stats()["active"] == 1)  # admitted into the only slot
        waiting = [s.submit(small()) for _ in range(2)]
        with pytest.raises(dd.DDError) as e:
            s.submit(small())
        assert e.value.status == 6
        st = s.stats()
        assert st["rejected"] == 1 and st["queued"] == 2 and st["active"] == 1
        s.cancel(t_big)  # client of the big query goes away: its slot frees after this round
        for t in waiting:
            assert s.wait(t, 10)[0] == 0
        assert s.wait(t_big, 10)[0] == 9


def test_small_query_overtakes_a_big_one(lib):
    with dd.Server(dry_run=True, round_ms=2) as s:
        t_big = s.submit(big())
        until(lambda: s.stats()["active"] == 1)
        t_small = s.submit(small())
        assert s.wait(t_small, 5)[0] == 0
        assert s.poll(t_big) is None  # still running: both shared the rounds
        s.cancel(t_big)
        assert s.wait(t_big, 5)[0] == 9


def test_cancel_queued_query(lib):
    with dd.Server(dry_run=True, round_ms=5, memory_budget_bytes=1000, max_queue=4) as s:
        t_big = s.submit(big())
        until(lambda: s.stats()["active"] == 1)
        t_q = s.submit(small())
        s.cancel(t_q)
        assert s.wait(t_q, 1)[0] == 9
        assert s.stats()["cancelled"] == 1
        s.cancel(t_big)


def test_unknown_ticket(lib):
    with dd.Server(dry_run=True, round_ms=1) as s:
        with pytest.raises(dd.DDError) as e:
            s.poll(12345)
        assert e.value.status == 8


def test_shutdown_cancels_pending(lib):
    s = dd.Server(dry_run=True, round_ms=5, memory_budget_bytes=1000)
    t_big = s.submit(big())
    t_q = s.submit(small())
    results = {}

    def waiter(t):
        try:
            results[t] = s.wait(t, 10)[0]
        except dd.DDError as e:  # the wait began after close(): the server refuses it
            results[t] = e.status

    th = [threading.Thread(target=waiter, args=(t,), daemon=True) for t in (t_big, t_q)]
    for x in th:
        x.start()
    time.sleep(0.05)
    s.close()
    for x in th:
        x.join(10)
    assert results == {t_big: 9, t_q: 9}
    with pytest.raises(dd.DDError):
        s.submit(small())


def test_close_while_many_threads_wait(lib):
    # waiters woken by the shutdown still hold the server: it is freed only after they return
    for _ in range(20):
        s = dd.Server(dry_run=True, round_ms=1, memory_budget_bytes=1000)
        tickets = [s.submit(big())] + [s.submit(small()) for _ in range(3)]
        results, th = [], []
        for t in tickets:
            for _ in range(4):
                def waiter(t=t):
                    try:
                        results.append(s.wait(t, 10)[0])
                    except dd.DDError as e:
                        results.append(e.status)
                th.append(threading.Thread(target=waiter, daemon=True))
        for x in th:
            x.start()
        s.close()
        for x in th:
            x.join(10)
        assert len(results) == len(th)
        # the small queries may finish before the shutdown; nothing else may happen
        assert set(results) <= {0, 9}


def test_many_clients_latency_stats(lib):
    with dd.Server(dry_run=True, round_ms=1) as s:
        tickets = []

        def client(k):
            for i in range(5):
                tickets.append(s.submit(small(A=2 * (k * 5 + i) + 33, n=10)))

        th = [threading.Thread(target=client, args=(k,)) for k in range(8)]
        for x in th:
            x.start()
        for x in th:
            x.join()
        for t in tickets:
            assert s.wait(t, 10)[0] == 0
        st = s.stats()
        assert st["completed"] == 40 and st["submitted"] == 40
        assert 0 < st["p50_ms"] <= st["p99_ms"]
        assert st["slots_free"] == st["slots"]


def test_release_and_retention(lib):
    """A delivered result stays answerable until 4096 newer ones were delivered,
    then its ticket is unknown; release drops a finished one at once and refuses
    a running one."""
    with dd.Server(dry_run=True, round_ms=1) as s:
        t_big = s.submit(big())
        until(lambda: s.stats()["active"] == 1)
        with pytest.raises(dd.DDError) as e:
            s.release(t_big)  # still running
        assert e.value.status == 6
        t = s.submit(small())
        assert s.wait(t, 10)[0] == 0
        assert s.wait(t, 10)[0] == 0  # delivered results stay answerable
        s.release(t)
        with pytest.raises(dd.DDError) as e:
            s.poll(t)
        assert e.value.status == 8
        tickets = [s.submit(small(A=2 * i + 33, n=8)) for i in range(4100)]
        for x in tickets:
            assert s.wait(x, 10)[0] == 0
        with pytest.raises(dd.DDError) as e:  # the oldest delivered records were dropped
            s.poll(tickets[0])
        assert e.value.status == 8
        assert s.poll(tickets[-1]) is not None
        s.cancel(t_big)
        assert s.wait(t_big, 10)[0] == 9
        st = s.stats()
        assert st["completed"] == 4101 and 0 < st["p50_ms"] <= st["p99_ms"]
