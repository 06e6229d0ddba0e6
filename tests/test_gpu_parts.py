"""dd_histogram_part on the GPU: disjoint tile ranges of one request, with
boundaries inside super tiles and of uneven sizes, sum to the raw histogram of
the whole request, bit for bit, on both kernels; run_resumable (a checkpoint
after every part) gives dd_histogram's result."""
import pytest

import coding_reliability_b200 as dd

pytestmark = pytest.mark.gpu


def bounds(total):
    # uneven parts, most boundaries off the 8-strip super-tile grid
    cuts = sorted({0, 3, total // 7 + 5, total // 2 + 1, total - 11, total} & set(range(total + 1)))
    return list(zip(cuts[:-1], cuts[1:]))


CASES = [
    (dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 58659, 16, kernel=dd.KERNEL_POPC), "popc"),
    (dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 58659, 16, kernel=dd.KERNEL_MMA), "mma"),
    (dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 641, 13, kernel=dd.KERNEL_MMA), "mma"),
    (dd.Request(dd.CODE_AN, dd.MODE_GRID_1D, 58659, 18, m=77, kernel=dd.KERNEL_POPC), "popc"),
    (dd.Request(dd.CODE_AN, dd.MODE_GRID_1D, 58659, 18, m=77, kernel=dd.KERNEL_MMA), "mma"),
    (dd.Request(dd.CODE_AN, dd.MODE_GRID_2D, 61, 14, m=300, m2=129, kernel=dd.KERNEL_POPC), "popc"),
    (dd.Request(dd.CODE_AN, dd.MODE_GRID_2D, 61, 14, m=300, m2=129, kernel=dd.KERNEL_MMA), "mma"),
    (dd.Request(dd.CODE_AN, dd.MODE_MONTE_CARLO, 641, 12, m=16, seed=5, kernel=dd.KERNEL_POPC), "popc"),
    # 256 codewords: 8 tiles of which 6 lie past the last row, so some parts hold no strip at all
    (dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, 8, with_1bit=1,
                hamming_method=dd.HAMMING_ALL_PAIRS, kernel=dd.KERNEL_MMA), "mma"),
    (dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, 16, with_1bit=1, kernel=dd.KERNEL_POPC), "popc"),
]


# the tcgen05 cases run under each epilogue
VARIANTS = [(q, k, e) for q, k in CASES for e in ((dd.MMA_EPILOGUE_PAIRED, dd.MMA_EPILOGUE_SINGLE)
                                                   if k == "mma" else (dd.MMA_EPILOGUE_AUTO,))]


@pytest.mark.parametrize("req,kern,epi", VARIANTS,
                         ids=[f"{c[0].code}-{c[0].mode}-{c[0].A}-{c[0].n}-{c[1]}{c[2] or ''}" for c in VARIANTS])
def test_parts_sum_to_the_whole(ctx, req, kern, epi):
    ctx.set_mma_epilogue(epi)
    full = ctx.histogram(req)
    assert full.kernel_used == (dd.KERNEL_MMA if kern == "mma" else dd.KERNEL_POPC)
    if kern == "mma":
        assert full.mma_epilogue == epi
    total = dd.request_plan(req)["tiles"]
    raw = None
    for b, e in reversed(bounds(total)):  # any order
        raw, _ = ctx.histogram_part(req, b, e - b, raw)
    assert raw == full.raw[:full.nbins]
    assert dd.postprocess(req, raw).counts == full.counts
    ctx.set_mma_epilogue(dd.MMA_EPILOGUE_AUTO)


def test_resumable_equals_one_call(ctx, kernel, tmp_path):
    req = dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 58659, 18, kernel=int(kernel))
    res = dd.run_resumable(ctx, req, tmp_path / "k18.json", chunk_tiles=1001)
    assert res.counts == ctx.histogram(req).counts


def test_part_outside_the_tile_space_is_refused(ctx):
    req = dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 641, 12)
    total = dd.request_plan(req)["tiles"]
    with pytest.raises(dd.DDError) as e:
        ctx.histogram_part(req, total - 1, 2)
    assert e.value.status == 1
    raw, ms = ctx.histogram_part(req, total, 0)  # an empty part adds nothing
    assert raw == [0] * dd.request_shape(req)[0] and ms == 0.0
