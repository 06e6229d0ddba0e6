"""Parity of the tcgen05 kind::i8 bit-plane MMA path with the oracle and with
the popc path (through the C-ABI), under each of its two epilogues (every test
runs twice: paired, where one accumulator holds a packed pair of distances,
and single, one distance per accumulator).  Bit-exact: INT32 accumulation of
0/1 planes is exact, and the accumulator holds the distance(s) themselves."""
import pytest

import coding_reliability_b200 as dd
import oracle
from conftest import golden

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True, params=["paired", "single"])
def epi(request, ctx):
    e = dd.MMA_EPILOGUE_PAIRED if request.param == "paired" else dd.MMA_EPILOGUE_SINGLE
    ctx.set_mma_epilogue(e)
    yield e
    ctx.set_mma_epilogue(dd.MMA_EPILOGUE_AUTO)


def on_mma(res, epi):
    """The result came from the tcgen05 kernel with the epilogue under test."""
    assert res.kernel_used == dd.KERNEL_MMA and res.mma_epilogue == epi, (res.kernel_used, res.mma_epilogue)


def mma_req(A, n, **kw):
    return dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, A, n, kernel=dd.KERNEL_MMA, **kw)


@pytest.mark.parametrize("A,n", [(641, 10), (641, 12), (61, 9), (3, 11), (58659, 12), (65521, 13), (1, 12)])
def test_mma_small_vs_oracle(ctx, epi, A, n):
    req = mma_req(A, n)
    nb, h, Aeff = dd.request_shape(req)
    res = ctx.histogram(req)
    on_mma(res, epi)
    assert res.raw == oracle.an_exhaustive_raw(Aeff, n, nb)


@pytest.mark.parametrize("A,n", [(58659, 16), (61, 16), (641, 16), (58659, 17), (32771, 18)])
def test_mma_vs_popc(ctx, epi, A, n):
    """32-bit and wider (>32-bit) codewords: MMA path equals the popc path."""
    a = ctx.histogram(mma_req(A, n))
    b = ctx.histogram(dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, A, n, kernel=dd.KERNEL_POPC))
    on_mma(a, epi)
    assert b.kernel_used == dd.KERNEL_POPC
    assert a.raw == b.raw and a.counts == b.counts


def test_mma_solutions_h(ctx, epi):
    for A in (61, 641):
        sol = golden("solutions.json")[f"solution_an16_A{A}"]
        res = ctx.histogram(mma_req(A, 16))
        on_mma(res, epi)
        k = min(len(sol), res.nbins)
        assert res.counts[:k] == sol[:k]


def test_mma_batch_super_a(ctx, epi):
    from test_gpu_parity import super_a_set
    As = super_a_set(64)
    reqs = [mma_req(A, 16, convention=dd.CONV_SUPER_A) for A in As]
    out = ctx.batch(reqs, use_graph=True)
    for A, r in list(zip(As, out))[::8]:
        p = ctx.histogram(dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, A, 16, kernel=dd.KERNEL_POPC,
                                     convention=dd.CONV_SUPER_A))
        assert r.counts == p.counts
    for r in out:
        on_mma(r, epi)


# -- grid jobs on the tcgen05 path (lattice rows x codeword / lattice columns) -----
@pytest.mark.parametrize("A,n,m", [(61, 12, 3), (61, 12, 17), (641, 14, 1000), (58659, 16, 4096), (58659, 18, 77),
                                   (3, 10, 1024), (65521, 17, 333), (58659, 20, 1 << 12)])
def test_mma_grid1d_vs_oracle_and_popc(ctx, epi, A, n, m):
    req = dd.Request(dd.CODE_AN, dd.MODE_GRID_1D, A, n, m=m, kernel=dd.KERNEL_MMA)
    nb, h, Aeff = dd.request_shape(req)
    res = ctx.histogram(req)
    on_mma(res, epi)
    popc = ctx.histogram(dd.Request(dd.CODE_AN, dd.MODE_GRID_1D, A, n, m=m, kernel=dd.KERNEL_POPC))
    assert res.raw == popc.raw and res.counts == popc.counts
    if n <= 18:
        raw, _ = oracle.an_grid1d_raw(Aeff, n, h, m, nb)
        assert res.raw == raw


@pytest.mark.parametrize("A,n,m,m2", [(61, 12, 100, 37), (641, 14, 64, 64), (58659, 18, 50, 300), (3, 8, 256, 1),
                                      (61, 40, 1000, 1000), (58659, 40, 4096, 512), (641, 36, 999, 1001)])
def test_mma_grid2d_vs_oracle(ctx, epi, A, n, m, m2):
    req = dd.Request(dd.CODE_AN, dd.MODE_GRID_2D, A, n, m=m, m2=m2, kernel=dd.KERNEL_MMA)
    nb, h, Aeff = dd.request_shape(req)
    res = ctx.histogram(req)
    on_mma(res, epi)
    raw = oracle.an_grid2d_raw(Aeff, n, m, m2, nb, with_bin0=True)
    assert res.raw == raw  # bin 0: the coincident lattice points, which counts[0] leaves out
    ref_raw = [0] + raw[1:]
    assert res.counts == oracle.an_grid_counts(2, n, min(m, 1 << n), min(m2, 1 << n), ref_raw)


def test_mma_grid_archive(ctx, epi):
    """Archived 1-D grid histograms of the reference (results/GridMs, converge/geom)."""
    checked = 0
    for x in golden("an_grid1d.json"):
        if x["n"] > 24 or any(isinstance(c, str) for c in x["counts"]):
            continue
        res = ctx.histogram(dd.Request(dd.CODE_AN, dd.MODE_GRID_1D, x["A"], x["n"], m=x["m"], kernel=dd.KERNEL_MMA))
        on_mma(res, epi)
        assert res.counts == x["counts"], x["file"]
        checked += 1
    assert checked >= 90


# -- Ext-Hamming all-pairs brute force on the tcgen05 path --------------------------
@pytest.mark.parametrize("n", [8, 16])
@pytest.mark.parametrize("method", [dd.HAMMING_ALL_PAIRS, dd.HAMMING_ALL_PAIRS_DISTINCT])
def test_mma_hamming_all_pairs(ctx, epi, n, method):
    for w1 in (0, 1):
        kw = dict(with_1bit=w1, hamming_method=method)
        a = ctx.histogram(dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, n, kernel=dd.KERNEL_MMA, **kw))
        b = ctx.histogram(dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, n, kernel=dd.KERNEL_POPC, **kw))
        on_mma(a, epi)
        assert b.kernel_used == dd.KERNEL_POPC
        assert a.raw == b.raw and a.counts == b.counts
        if n == 8:
            f = oracle.hamming_pairs_distinct_raw if method == dd.HAMMING_ALL_PAIRS_DISTINCT else oracle.hamming_pairs_raw
            assert a.counts == f(n, w1, a.nbins)


def test_mma_hamming_reference_runs(ctx, epi):
    """The reference's own `-e 2/3` stdout tables, on the tcgen05 path."""
    method = {"2": dd.HAMMING_ALL_PAIRS, "3": dd.HAMMING_ALL_PAIRS_DISTINCT, "4": dd.HAMMING_ALL_PAIRS}
    runs = [r for r in golden("ref_runs.json") if r["args"][0] == "-e" and r["args"][1] in method]
    assert runs
    for run in runs:
        args = run["args"]
        res = ctx.histogram(dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, int(args[-1]),
                                       with_1bit=int("-b" in args), hamming_method=method[args[1]],
                                       kernel=dd.KERNEL_MMA))
        on_mma(res, epi)
        assert res.counts == run["counts"], args


def test_mma_batch_mixed_shapes(ctx, epi):
    """One launch over jobs of different widths: windowed jobs (A = 58659, k = 18..20:
    S = 35..37, the joint table holds only part of the d2 rows) beside jobs whose
    window holds every distance (small k), a 1-D grid and an Ext-Hamming all-pairs job.
    The table is folded with each job's own S and window at every job change; every
    histogram equals its popc-kernel run."""
    reqs = [dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 58659, 20, kernel=dd.KERNEL_MMA),
            dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 641, 12, kernel=dd.KERNEL_MMA),
            dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 58659, 18, kernel=dd.KERNEL_MMA),
            dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 61, 14, kernel=dd.KERNEL_MMA),
            dd.Request(dd.CODE_AN, dd.MODE_GRID_1D, 1021, 20, m=4096, kernel=dd.KERNEL_MMA),
            dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 32771, 19, kernel=dd.KERNEL_MMA),
            dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, 16, hamming_method=dd.HAMMING_ALL_PAIRS,
                       kernel=dd.KERNEL_MMA)]
    for graph in (False, True):
        out = ctx.batch(reqs, use_graph=graph, kernel=dd.KERNEL_MMA)
        for q, r in zip(reqs, out):
            on_mma(r, epi)
            p = dd.Request(q.code, q.mode, q.A, q.n, m=q.m, hamming_method=q.hamming_method, kernel=dd.KERNEL_POPC)
            s = ctx.histogram(p)
            assert s.kernel_used == dd.KERNEL_POPC
            assert r.raw == s.raw and r.counts == s.counts, q
