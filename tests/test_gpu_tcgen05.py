"""Parity of the tcgen05 kind::i8 bit-plane MMA path with the oracle and with
the popc path (through the C-ABI).  Bit-exact: INT32 accumulation of 0/1
planes is exact, and the accumulator holds the distance itself."""
import pytest

import coding_reliability_b200 as dd
import oracle
from conftest import golden

pytestmark = pytest.mark.gpu


def mma_req(A, n, **kw):
    return dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, A, n, kernel=dd.KERNEL_MMA, **kw)


@pytest.mark.parametrize("A,n", [(641, 10), (641, 12), (61, 9), (3, 11), (58659, 12), (65521, 13), (1, 12)])
def test_mma_small_vs_oracle(ctx, A, n):
    req = mma_req(A, n)
    nb, h, Aeff = dd.request_shape(req)
    res = ctx.histogram(req)
    assert res.kernel_used == dd.KERNEL_MMA
    assert res.raw == oracle.an_exhaustive_raw(Aeff, n, nb)


@pytest.mark.parametrize("A,n", [(58659, 16), (61, 16), (641, 16), (58659, 17), (32771, 18)])
def test_mma_vs_popc(ctx, A, n):
    """32-bit and wider (>32-bit) codewords: MMA path equals the popc path."""
    a = ctx.histogram(mma_req(A, n))
    b = ctx.histogram(dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, A, n, kernel=dd.KERNEL_POPC))
    assert a.kernel_used == dd.KERNEL_MMA and b.kernel_used == dd.KERNEL_POPC
    assert a.raw == b.raw and a.counts == b.counts


def test_mma_solutions_h(ctx):
    for A in (61, 641):
        sol = golden("solutions.json")[f"solution_an16_A{A}"]
        res = ctx.histogram(mma_req(A, 16))
        k = min(len(sol), res.nbins)
        assert res.counts[:k] == sol[:k]


def test_mma_batch_super_a(ctx):
    from test_gpu_parity import super_a_set
    As = super_a_set(64)
    reqs = [mma_req(A, 16, convention=dd.CONV_SUPER_A) for A in As]
    out = ctx.batch(reqs, use_graph=True)
    for A, r in list(zip(As, out))[::8]:
        p = ctx.histogram(dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, A, 16, kernel=dd.KERNEL_POPC,
                                     convention=dd.CONV_SUPER_A))
        assert r.counts == p.counts
    assert all(r.kernel_used == dd.KERNEL_MMA for r in out)


def test_mma_k24_archive_A63877(ctx):
    """The config-3 shape (40-bit codewords, 41 bins) on the MMA path vs the archive."""
    case = next(c for c in golden("an_exhaustive.json") if c["A"] == 63877 and c["n"] == 24)
    res = ctx.histogram(mma_req(63877, 24))
    assert res.counts == case["counts"]


# -- grid jobs on the tcgen05 path (lattice rows x codeword / lattice columns) -----
@pytest.mark.parametrize("A,n,m", [(61, 12, 3), (61, 12, 17), (641, 14, 1000), (58659, 16, 4096), (58659, 18, 77),
                                   (3, 10, 1024), (65521, 17, 333), (58659, 20, 1 << 12)])
def test_mma_grid1d_vs_oracle_and_popc(ctx, A, n, m):
    req = dd.Request(dd.CODE_AN, dd.MODE_GRID_1D, A, n, m=m, kernel=dd.KERNEL_MMA)
    nb, h, Aeff = dd.request_shape(req)
    res = ctx.histogram(req)
    assert res.kernel_used == dd.KERNEL_MMA
    popc = ctx.histogram(dd.Request(dd.CODE_AN, dd.MODE_GRID_1D, A, n, m=m, kernel=dd.KERNEL_POPC))
    assert res.raw == popc.raw and res.counts == popc.counts
    if n <= 18:
        raw, _ = oracle.an_grid1d_raw(Aeff, n, h, m, nb)
        assert res.raw == raw


@pytest.mark.parametrize("A,n,m,m2", [(61, 12, 100, 37), (641, 14, 64, 64), (58659, 18, 50, 300), (3, 8, 256, 1),
                                      (61, 40, 1000, 1000), (58659, 40, 4096, 512), (641, 36, 999, 1001)])
def test_mma_grid2d_vs_oracle(ctx, A, n, m, m2):
    req = dd.Request(dd.CODE_AN, dd.MODE_GRID_2D, A, n, m=m, m2=m2, kernel=dd.KERNEL_MMA)
    nb, h, Aeff = dd.request_shape(req)
    res = ctx.histogram(req)
    assert res.kernel_used == dd.KERNEL_MMA
    raw = oracle.an_grid2d_raw(Aeff, n, m, m2, nb)
    assert res.raw[1:] == raw[1:] and res.raw[0] == 0
    assert res.counts == oracle.an_grid_counts(2, n, min(m, 1 << n), min(m2, 1 << n), raw)


def test_mma_grid_archive(ctx):
    """Archived 1-D grid histograms of the reference (results/GridMs, converge/geom)."""
    checked = 0
    for x in golden("an_grid1d.json"):
        if x["n"] > 24 or any(isinstance(c, str) for c in x["counts"]):
            continue
        res = ctx.histogram(dd.Request(dd.CODE_AN, dd.MODE_GRID_1D, x["A"], x["n"], m=x["m"], kernel=dd.KERNEL_MMA))
        assert res.counts == x["counts"], x["file"]
        checked += 1
    assert checked >= 90


# -- Ext-Hamming all-pairs brute force on the tcgen05 path --------------------------
@pytest.mark.parametrize("n", [8, 16])
@pytest.mark.parametrize("method", [dd.HAMMING_ALL_PAIRS, dd.HAMMING_ALL_PAIRS_DISTINCT])
def test_mma_hamming_all_pairs(ctx, n, method):
    for w1 in (0, 1):
        kw = dict(with_1bit=w1, hamming_method=method)
        a = ctx.histogram(dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, n, kernel=dd.KERNEL_MMA, **kw))
        b = ctx.histogram(dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, n, kernel=dd.KERNEL_POPC, **kw))
        assert a.kernel_used == dd.KERNEL_MMA and b.kernel_used == dd.KERNEL_POPC
        assert a.raw == b.raw and a.counts == b.counts
        if n == 8:
            f = oracle.hamming_pairs_distinct_raw if method == dd.HAMMING_ALL_PAIRS_DISTINCT else oracle.hamming_pairs_raw
            assert a.counts == f(n, w1, a.nbins)


def test_mma_hamming_reference_runs(ctx):
    """The reference's own `-e 2/3` stdout tables, on the tcgen05 path."""
    method = {"2": dd.HAMMING_ALL_PAIRS, "3": dd.HAMMING_ALL_PAIRS_DISTINCT, "4": dd.HAMMING_ALL_PAIRS}
    runs = [r for r in golden("ref_runs.json") if r["args"][0] == "-e" and r["args"][1] in method]
    assert runs
    for run in runs:
        args = run["args"]
        res = ctx.histogram(dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, int(args[-1]),
                                       with_1bit=int("-b" in args), hamming_method=method[args[1]],
                                       kernel=dd.KERNEL_MMA))
        assert res.kernel_used == dd.KERNEL_MMA
        assert res.counts == run["counts"], args
