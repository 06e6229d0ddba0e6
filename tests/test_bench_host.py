"""Host-side pieces of bench.py that need no GPU: the serving mix covers every
query class of the serving configuration (the k=32 grid included), the latency
percentiles are nearest-rank, and the tcgen05 path's issue-rate roofline is
computed from the ncu figures and tolerates missing ones."""
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402
import coding_reliability_b200 as dd  # noqa: E402


def test_serving_mix_covers_every_class():
    mix = bench.serving_mix(dd)
    assert len(mix) == 48
    seen = set()
    for cls, q in mix:
        assert 129 <= q.A < 1 << 16 and q.A % 2 == 1
        assert q.n in (8, 12, 16, 20, 24, 32)
        if q.n <= 20:
            assert cls == "exhaustive" and q.mode == dd.MODE_EXHAUSTIVE
        elif cls == "grid":
            assert q.mode == dd.MODE_GRID_1D and q.m == 1 << 16  # stride 2^(k-16)
        else:
            assert cls == "monte_carlo" and q.mode == dd.MODE_MONTE_CARLO
            assert 1 << 32 <= (q.m << q.n) <= 1 << 36 or q.m == 1
        seen.add((cls, q.n))
    assert ("grid", 32) in seen and ("grid", 24) in seen
    assert {c for c, _ in seen} == set(bench.SERVING_CLASSES)


def test_percentile_is_nearest_rank():
    v = sorted(float(x) for x in range(1, 49))
    assert bench.percentile(v, 0.50) == 24.0
    assert bench.percentile(v, 0.99) == 48.0
    assert bench.percentile([5.0], 0.99) == 5.0
    assert bench.percentile(sorted(float(x) for x in range(1, 101)), 0.99) == 99.0


class _StandIn:
    """A context stand-in that returns a fixed histogram for either kernel."""
    def __init__(self, raw, counts, differ=False):
        self.raw, self.counts, self.differ = raw, counts, differ

    def histogram(self, req):
        import types
        counts = list(self.counts)
        if self.differ:
            counts[1] += 1
        return types.SimpleNamespace(kernel_used=req.kernel, raw=list(self.raw), counts=counts, kernel_ms=1000.0)


def test_cross_kernel_check_requires_identical_histograms():
    import types
    timed = types.SimpleNamespace(kernel_used=dd.KERNEL_MMA, raw=[0, 3, 5], counts=[8, 6, 10])
    out = bench.cross_kernel_check(_StandIn(timed.raw, timed.counts), dd, 641, 3, timed)
    assert out["cross_kernel"] and out["other_kernel"] == "popc" and out["timed_kernel"] == "mma"
    assert out["sha256_counts"] == bench.counts_digest([8, 6, 10])
    assert out["other_kernel_pairs_per_s"] == bench.pairs_of(3) / 1.0
    import pytest
    with pytest.raises(AssertionError):
        bench.cross_kernel_check(_StandIn(timed.raw, timed.counts, differ=True), dd, 641, 3, timed)


def test_issue_roofline():
    """The tcgen05 path's issue figure: 5,386 warp instructions per 65,536-pair tile
    (the ncu capture) at 9.35e12 pairs/s against 4 per clock on 148 SMs at 1965 MHz
    is about 0.66; a missing clock or instruction count gives None, never an error."""
    r = bench.issue_roofline(9.35e12, "paired", 1965.0, 148)
    assert abs(r["warp_inst_per_pair"] - 5386 / 65536) < 1e-12
    assert abs(r["peak_ginst_s"] - 4 * 148 * 1.965) < 1e-6
    assert abs(r["frac"] - 0.6606) < 1e-3
    assert r["achieved_ginst_s"] < r["peak_ginst_s"]
    none_clock = bench.issue_roofline(9.35e12, "paired", None, 148)
    assert none_clock["peak_ginst_s"] is None and none_clock["frac"] is None
    single = bench.issue_roofline(6.1e12, "single", 1965.0, 148)
    assert single["frac"] is None and single["ncu_issue_active_pct"] == 65.2
