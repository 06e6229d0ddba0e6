"""dd_histogram_noalloc: the entry point for callers that cannot allocate
device memory (its scratch is a fixed __device__ array).  Checked through the
C-ABI against dd_histogram, bit-exact like every histogram here, on two calls
in a row (the second call must not see the first call's counts).  Kept in a
file that pytest collects last; it passes alone and after the other tests."""
import pytest

import coding_reliability_b200 as dd

pytestmark = pytest.mark.gpu


def requests():
    return [
        dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 641, 12),
        dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 58659, 16, convention=dd.CONV_SUPER_A),
        dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 65521, 17),               # codewords above 32 bits
        dd.Request(dd.CODE_AN, dd.MODE_GRID_1D, 61, 20, m=1001),
        dd.Request(dd.CODE_AN, dd.MODE_MONTE_CARLO, 641, 14, m=100, seed=3),
        dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, 16, with_1bit=1),
        dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, 8, with_1bit=1,
                   hamming_method=dd.HAMMING_ALL_PAIRS),
    ]


def test_noalloc_matches_dd_histogram_twice():
    reqs = requests()
    with dd.Context(0) as ctx:
        expected = [ctx.histogram(r) for r in reqs]
    for call in range(2):
        got = dd.histogram_noalloc(reqs, device=0)
        for q, g, e in zip(reqs, got, expected):
            assert g.counts == e.counts, (call, q)
            assert g.raw == e.raw and g.minb == e.minb and g.nbins == e.nbins, (call, q)


def test_noalloc_single_requests_in_a_row():
    with dd.Context(0) as ctx:
        for q in requests()[:3]:
            e = ctx.histogram(q)
            for _ in range(2):
                assert dd.histogram_noalloc([q])[0].counts == e.counts


def test_noalloc_refuses_more_than_its_scratch_holds():
    with pytest.raises(dd.DDError) as err:
        dd.histogram_noalloc([dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 61, 8)] * 33)
    assert err.value.status == 1 and "32" in str(err.value)
