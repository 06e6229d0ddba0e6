"""Checkpoint / resume of one long histogram (run_resumable over dd_histogram_part),
host logic only: a stand-in context adds a known amount per tile, and the fault is
made on the host (the stand-in raises after some parts, as a killed process would
stop between parts)."""
import ctypes as C
import json

import pytest

import coding_reliability_b200 as dd


def per_tile(t, b):
    return (t * 31 + b * 7) % 5


class FakeCtx:
    """Adds per_tile(t, b) to bin b for every tile t of a part; records the parts."""

    def __init__(self, fail_after=None):
        self.parts = []
        self.fail_after = fail_after

    def histogram_part(self, req, tile_begin, tile_count, raw=None):
        if self.fail_after is not None and len(self.parts) >= self.fail_after:
            raise RuntimeError("stopped between parts")
        nb = dd.request_shape(req)[0]
        raw = list(raw or [0] * nb)
        for t in range(tile_begin, tile_begin + tile_count):
            for b in range(nb):
                raw[b] += per_tile(t, b)
        self.parts.append((tile_begin, tile_count))
        return raw, 0.0


def expected(req):
    total = dd.request_plan(req)["tiles"]
    nb = dd.request_shape(req)[0]
    return [sum(per_tile(t, b) for t in range(total)) for b in range(nb)]


REQ = dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 641, 12)  # 80 tiles, 23 bins


def covers_once(parts, total):
    seen = [0] * total
    for b, c in parts:
        for t in range(b, b + c):
            seen[t] += 1
    return all(x == 1 for x in seen)


def test_uninterrupted_run(lib, tmp_path):
    f = tmp_path / "state.json"
    ctx = FakeCtx()
    res = dd.run_resumable(ctx, REQ, f, chunk_tiles=7)
    assert res.raw == expected(REQ)
    assert res.counts == dd.postprocess(REQ, expected(REQ)).counts
    assert covers_once(ctx.parts, 80) and not f.exists()


@pytest.mark.parametrize("stop", [1, 5, 11])
def test_resume_after_a_stop(lib, tmp_path, stop):
    f = tmp_path / "state.json"
    first = FakeCtx(fail_after=stop)
    with pytest.raises(RuntimeError):
        dd.run_resumable(first, REQ, f, chunk_tiles=7)
    st = json.loads(f.read_text())
    assert st["next_tile"] == 7 * stop and st["tiles"] == 80
    second = FakeCtx()
    res = dd.run_resumable(second, REQ, f, chunk_tiles=9)  # another part size on resume
    assert res.raw == expected(REQ)
    assert covers_once(first.parts + second.parts, 80) and not f.exists()


def test_checkpoint_of_another_request_is_refused(lib, tmp_path):
    f = tmp_path / "state.json"
    with pytest.raises(RuntimeError):
        dd.run_resumable(FakeCtx(fail_after=2), REQ, f, chunk_tiles=7)
    other = dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 61, 12)
    with pytest.raises(dd.DDError):
        dd.run_resumable(FakeCtx(), other, f)


def test_damaged_checkpoint_is_refused(lib, tmp_path):
    f = tmp_path / "state.json"
    with pytest.raises(RuntimeError):
        dd.run_resumable(FakeCtx(fail_after=2), REQ, f, chunk_tiles=7)
    st = json.loads(f.read_text())
    st["next_tile"] = 81
    f.write_text(json.dumps(st))
    with pytest.raises(dd.DDError):
        dd.run_resumable(FakeCtx(), REQ, f)


def test_part_entry_point_validates_without_a_device(lib):
    raw = (C.c_uint64 * 64)()
    req = REQ._c()
    assert lib.dd_histogram_part(None, C.byref(req), 0, 1, raw, 64, None) == 1
