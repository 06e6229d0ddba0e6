"""Parity of the GPU path (through the C-ABI) with the oracle and the
reference's golden data.  Bit-exact for every histogram: the arithmetic is
integer, and the grid lattice's double arithmetic is the reference's own.

Every test names the kernel it runs (the `kernel` fixture runs the popc
kernel and the tcgen05 kernel with each of its epilogues where a job allows
them; Monte Carlo and the Hamming weight enumerator run on the popc kernel
only) and asserts kernel_used, so no case depends on the context's autotune
state."""
import random

import pytest

import coding_reliability_b200 as dd
import oracle
from conftest import golden

pytestmark = pytest.mark.gpu


def an_req(A, n, **kw):
    return dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, A, n, **kw)


def ran(res, kernel):
    """The result came from `kernel` (and, on the tcgen05 kernel, its epilogue)."""
    assert res.kernel_used == int(kernel), (res.kernel_used, kernel)
    if res.kernel_used == dd.KERNEL_MMA and getattr(kernel, "epilogue", 0):
        assert res.mma_epilogue == kernel.epilogue, (res.mma_epilogue, kernel.epilogue)


def run(ctx, req, kernel):
    """ctx.histogram(req) on `kernel`, checking that this kernel ran."""
    req.kernel = int(kernel)
    res = ctx.histogram(req)
    ran(res, kernel)
    return res


# -- AN exhaustive --------------------------------------------------------------
@pytest.mark.parametrize("A", [1, 3, 61, 255, 641, 1021, 32771, 58659, 65521])
@pytest.mark.parametrize("n", [1, 2, 3, 5, 7, 9, 10, 11, 12])
def test_an_exhaustive_small(ctx, kernel, A, n):
    req = an_req(A, n)
    nb, h, Aeff = dd.request_shape(req)
    res = run(ctx, req, kernel)
    assert res.raw == oracle.an_exhaustive_raw(Aeff, n, nb)
    assert res.counts == oracle.an_exhaustive_counts(Aeff, n, nb)
    assert sum(res.raw) == (1 << n) * ((1 << n) - 1) // 2


@pytest.mark.parametrize("A,n", [(61, 8), (641, 8), (61, 16), (641, 16)])
def test_an_solutions_h(ctx, kernel, A, n):
    sol = golden("solutions.json")[f"solution_an{n}_A{A}"]
    res = run(ctx, an_req(A, n), kernel)
    k = min(len(sol), res.nbins)
    assert res.counts[:k] == sol[:k]


def consistent(case):
    """An archived exhaustive histogram is usable as a pin only if it passes the
    conservation law sum(counts) = (2^n)^2 (all ordered pairs incl. the diagonal).
    41 archived runs of the reference (6-bit A, n >= 20) fail it: their GPU runs
    lost counts, e.g. A=35 n=22 bin 2 has 21222760 where a direct enumeration of
    the 378 two-bit flips of every codeword finds 37269512."""
    return sum(case["counts"]) == (1 << (2 * case["n"]))


def test_an_results_archive(ctx, kernel):
    """results/As exhaustive histograms n=8..22 (every self-consistent file)."""
    cases = [c for c in golden("an_exhaustive.json") if c["n"] <= 22 and consistent(c)]
    assert len(cases) > 580
    for c in cases:
        res = run(ctx, an_req(c["A"], c["n"]), kernel)
        assert res.h == c["h"], c["file"]
        assert res.counts == c["counts"], c["file"]


def test_an_archive_inconsistent_files_conserve(ctx, kernel):
    """Where the archive fails conservation, our histogram still conserves pairs
    and agrees with an independent count of the distance-2 pairs."""
    bad = [c for c in golden("an_exhaustive.json") if c["n"] <= 22 and not consistent(c)]
    assert bad
    for c in bad[:6]:
        res = run(ctx, an_req(c["A"], c["n"]), kernel)
        assert sum(res.counts) == 1 << (2 * c["n"])
    res = run(ctx, an_req(35, 22), kernel)
    d1, d2 = oracle.an_low_distance(35, 22, 22 + 6)
    assert (res.counts[1], res.counts[2]) == (2 * d1, 2 * d2)


@pytest.mark.parametrize("A,n", [(58659, 13), (58659, 16), (65521, 16), (641, 18), (3, 18)])
def test_an_wide_and_mid(ctx, kernel, A, n):
    """40-bit style codewords (n+h > 32 for n>=17 at 16-bit A) and mid sizes vs the oracle."""
    req = an_req(A, n)
    nb, h, Aeff = dd.request_shape(req)
    res = run(ctx, req, kernel)
    assert res.raw == oracle.an_exhaustive_raw(Aeff, n, nb)


@pytest.mark.parametrize("A,n", [(58659, 18), (32771, 17), (65535, 17)])
def test_an_wide_codewords(ctx, kernel, A, n):
    """Codewords above 32 bits: the high-word segment split of the popc kernel,
    more than 32 operand bit planes on the tcgen05 kernel."""
    req = an_req(A, n)
    nb, h, Aeff = dd.request_shape(req)
    assert (Aeff * ((1 << n) - 1)) >> 32
    res = run(ctx, req, kernel)
    assert res.raw == oracle.an_exhaustive_raw(Aeff, n, nb)


@pytest.mark.parametrize("conv", [dd.CONV_GPU, dd.CONV_CPU, dd.CONV_SUPER_A])
def test_an_conventions(ctx, kernel, conv):
    for A in (64, 58659, 641):
        req = an_req(A, 12, convention=conv)
        nb, h, Aeff = dd.request_shape(req)
        res = run(ctx, req, kernel)
        assert res.counts == oracle.an_exhaustive_counts(Aeff, 12, nb)
        lim = (nb + 1) // 2 if conv == dd.CONV_SUPER_A else nb // 2
        first = next((i for i in range(1, lim) if res.counts[i]), 0xFFFF)
        assert res.minb == first


def test_an_k24_archive_A63877(ctx, kernel):
    """The k=24 exhaustive shape (16-bit A, 40-bit codewords, 41 bins) against
    the reference's archived exhaustive run
    (distance_distribution/results/As/ancoding_gpu_A63877_n24_h16.csv)."""
    case = next(c for c in golden("an_exhaustive.json") if c["A"] == 63877 and c["n"] == 24)
    res = run(ctx, an_req(63877, 24), kernel)
    assert res.counts == case["counts"]


def test_an_k24_solutions_A641(ctx, kernel):
    """A=641, k=24 against the exact table of distance_distribution/src/solutions.h:28-66."""
    sol = golden("solutions.json")["solution_an24_A641"]
    res = run(ctx, an_req(641, 24), kernel)
    assert res.counts == sol[: res.nbins]


# -- AN grid ---------------------------------------------------------------------
def test_an_grid1d_archive(ctx, kernel):
    """Every archived 1-D grid run with n <= 24 (m up to 10^6, non-power-of-two steps)."""
    checked = 0
    for x in golden("an_grid1d.json"):
        if x["n"] > 24 or any(isinstance(c, str) for c in x["counts"]):
            continue
        res = run(ctx, dd.Request(dd.CODE_AN, dd.MODE_GRID_1D, x["A"], x["n"], m=x["m"]), kernel)
        assert res.counts == x["counts"], x["file"]
        checked += 1
    assert checked >= 90


@pytest.mark.parametrize("A,n,m", [(61, 12, 3), (61, 12, 16), (61, 12, 17), (641, 14, 1000), (58659, 16, 4096),
                                   (58659, 18, 77), (3, 10, 1024), (65521, 17, 333)])
def test_an_grid1d_oracle(ctx, kernel, A, n, m):
    req = dd.Request(dd.CODE_AN, dd.MODE_GRID_1D, A, n, m=m)
    nb, h, Aeff = dd.request_shape(req)
    res = run(ctx, req, kernel)
    raw, _ = oracle.an_grid1d_raw(Aeff, n, h, m, nb)
    assert res.raw == raw


@pytest.mark.parametrize("A,n,m,m2", [(61, 12, 100, 37), (641, 14, 64, 64), (58659, 18, 50, 300), (3, 8, 256, 1),
                                      (61, 40, 1000, 1000), (58659, 40, 4096, 512), (61, 48, 2000, 3000),
                                      (255, 48, 1 << 16, 7), (641, 36, 999, 1001)])
def test_an_grid2d_oracle(ctx, kernel, A, n, m, m2):
    """Includes the k=40 and k=48 buckets (an_coding.h:27-29,38-40): 2^(2k)/(m*m2)
    scale factors above 2^64, so the uint128 counts are exercised."""
    req = dd.Request(dd.CODE_AN, dd.MODE_GRID_2D, A, n, m=m, m2=m2)
    nb, h, Aeff = dd.request_shape(req)
    res = run(ctx, req, kernel)
    raw = oracle.an_grid2d_raw(Aeff, n, m, m2, nb, with_bin0=True)
    assert res.raw == raw  # bin 0: the coincident lattice points, which counts[0] leaves out
    ref_raw = [0] + raw[1:]
    assert res.counts == oracle.an_grid_counts(2, n, min(m, 1 << n), min(m2, 1 << n), ref_raw)
    assert res.counts[0] == 0


# -- AN Monte Carlo ----------------------------------------------------------------
@pytest.mark.parametrize("A,n,it,seed", [(61, 10, 100, 1), (641, 12, 257, 99), (58659, 16, 13, 7),
                                         (58659, 18, 4, 2026), (61, 33, 1, 5)])
def test_an_mc_replay(ctx, A, n, it, seed):
    """Exact equality with the CPU replay of the same Philox counter stream."""
    req = dd.Request(dd.CODE_AN, dd.MODE_MONTE_CARLO, A, n, m=it, seed=seed)
    nb, h, Aeff = dd.request_shape(req)
    if n > 24:
        pytest.skip("n=33 replay is too long on the CPU")
    res = run(ctx, req, dd.KERNEL_POPC)
    assert res.raw == oracle.an_mc_raw(Aeff, n, it, seed, nb)
    assert res.counts == oracle.an_mc_counts(n, min(it, 1 << n), res.raw)


@pytest.mark.parametrize("A,n,it", [(61, 40, 1), (641, 36, 2)])
def test_an_mc_wide_buckets(ctx, A, n, it):
    """k=36/40 Monte Carlo (2^k codewords x it samples; too long to replay on the
    CPU): every sample lands in a bin, and the uint128 counts are the host
    post-processing of the device bins."""
    req = dd.Request(dd.CODE_AN, dd.MODE_MONTE_CARLO, A, n, m=it, seed=3)
    nb, h, Aeff = dd.request_shape(req)
    res = run(ctx, req, dd.KERNEL_POPC)
    assert sum(res.raw) == (1 << n) * it
    assert res.counts == oracle.an_mc_counts(n, it, res.raw)
    assert max(res.counts) > (1 << 64)


def test_an_mc_statistical_agreement(ctx):
    """MC estimate vs the exact solutions.h histogram (A=61, n=16): every well-populated
    bin within 5 standard deviations of its binomial sampling noise."""
    sol = golden("solutions.json")["solution_an16_A61"]
    it = 4096
    res = run(ctx, dd.Request(dd.CODE_AN, dd.MODE_MONTE_CARLO, 61, 16, m=it, seed=12345), dd.KERNEL_POPC)
    N = 1 << 16
    total = N * it
    for d in range(1, res.nbins):
        p = sol[d] / (N * N)
        if p * total < 1000:
            continue
        sd = (total * p * (1 - p)) ** 0.5
        assert abs(res.raw[d] - total * p) < 5 * sd, d


# -- Ext-Hamming ------------------------------------------------------------------
@pytest.mark.parametrize("n", [4, 8, 16, 24, 32])
@pytest.mark.parametrize("w1", [0, 1])
def test_hamming_weights(ctx, n, w1):
    req = dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, n, with_1bit=w1)
    nb, h, _ = dd.request_shape(req)
    res = run(ctx, req, dd.KERNEL_POPC)
    if n <= 24:
        assert res.raw == oracle.hamming_weights_raw(n, nb)
    assert res.counts == oracle.hamming_weights_counts(n, w1, res.raw)
    if n in (8, 16, 24, 32):
        sol = golden("solutions.json")[f"sol_hamming_n{n}"]
        for i in range(4, nb, 2):
            assert res.counts[i] == sol[i] << n


@pytest.mark.parametrize("ref", [r for r in golden("ref_runs.json") if r["args"][0] == "-e"],
                         ids=lambda r: " ".join(r["args"]))
def test_hamming_reference_runs(ctx, kernel, ref):
    args = ref["args"]
    n = int(args[-1])
    method = {"1": dd.HAMMING_WEIGHTS, "2": dd.HAMMING_ALL_PAIRS, "3": dd.HAMMING_ALL_PAIRS_DISTINCT,
              "4": dd.HAMMING_ALL_PAIRS}[args[1]]
    if method == dd.HAMMING_WEIGHTS and kernel == dd.KERNEL_MMA:
        pytest.skip("the weight enumerator is a popc-kernel job")
    res = run(ctx, dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, n, with_1bit=int("-b" in args),
                              hamming_method=method), kernel)
    assert res.counts == ref["counts"]


@pytest.mark.parametrize("n", [8, 16, 24])
def test_hamming_all_pairs_vs_weights(ctx, kernel, n):
    """All-pairs brute force (2^2n pairs on the GPU) equals the weight enumerator, with spheres."""
    for w1 in (0, 1):
        a = run(ctx, dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, n, with_1bit=w1,
                                hamming_method=dd.HAMMING_ALL_PAIRS), kernel)
        b = run(ctx, dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, n, with_1bit=w1), dd.KERNEL_POPC)
        assert a.counts == b.counts
        if n == 8:
            assert a.counts == oracle.hamming_pairs_raw(8, w1, a.nbins)


@pytest.mark.parametrize("n,m", [(8, 100), (16, 1000), (16, 4096), (24, 99999), (32, 1 << 20)])
def test_hamming_grid(ctx, n, m):
    for w1 in (0, 1):
        req = dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_GRID_1D, 1, n, m=m, with_1bit=w1)
        nb, h, _ = dd.request_shape(req)
        res = run(ctx, req, dd.KERNEL_POPC)
        raw, _ = oracle.hamming_grid_raw(n, m, nb)
        assert res.raw == raw
        assert res.counts == oracle.hamming_sampled_counts(0, n, w1, min(m, 1 << n), raw)


@pytest.mark.parametrize("n,m,seed", [(8, 100, 1), (16, 5000, 2), (24, 1 << 16, 3), (40, 1 << 16, 4)])
def test_hamming_mc(ctx, n, m, seed):
    req = dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_MONTE_CARLO, 1, n, m=m, seed=seed, with_1bit=1)
    nb, h, _ = dd.request_shape(req)
    res = run(ctx, req, dd.KERNEL_POPC)
    raw, _ = oracle.hamming_mc_raw(n, m, seed, nb)
    assert res.raw == raw
    assert res.counts == oracle.hamming_sampled_counts(1, n, 1, min(m, 1 << n), raw)


# -- batch ---------------------------------------------------------------------------
def super_a_set(count=256, seed=20261203):
    rng = random.Random(seed)
    out = []
    while len(out) < count:
        a = rng.randrange(32768, 65536) | 1
        if a not in out:
            out.append(a)
    return out


def test_batch_equals_single(ctx, kernel):
    reqs = [an_req(A, 12, convention=dd.CONV_SUPER_A) for A in super_a_set(64)]
    reqs += [an_req(641, 12), an_req(61, 9), dd.Request(dd.CODE_AN, dd.MODE_GRID_1D, 61, 14, m=333),
             dd.Request(dd.CODE_AN, dd.MODE_MONTE_CARLO, 58659, 12, m=50, seed=3),
             dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, 16, with_1bit=1)]
    # Monte Carlo and the Hamming weight enumerator are popc-kernel jobs in either batch
    popc_only = {len(reqs) - 2, len(reqs) - 1}
    for graph in (False, True, True):
        out = ctx.batch(reqs, use_graph=graph, kernel=int(kernel))
        for i, (q, r) in enumerate(zip(reqs, out)):
            want = dd.KERNEL_POPC if i in popc_only else kernel
            ran(r, want)
            s = run(ctx, q, want)
            assert r.counts == s.counts and r.raw == s.raw and r.minb == s.minb


def test_graph_cache_after_buffer_growth(kernel):
    """A fresh context replays a graph-captured batch after a larger batch has
    reallocated its bins and job table: the cached graph is rebuilt for the new
    buffers and gives the same histograms as the first run and as single runs."""
    small = [an_req(A, 10) for A in range(33, 33 + 2 * 70, 2)]   # 70 requests: past the initial 64 slots
    large = [an_req(A, 8) for A in range(33, 33 + 2 * 300, 2)]   # 300: grows the buffers again
    with dd.Context(0) as c:
        c.set_mma_epilogue(kernel.epilogue or dd.MMA_EPILOGUE_AUTO)
        first = c.batch(small, use_graph=True, kernel=int(kernel))
        c.batch(large, use_graph=True, kernel=int(kernel))
        again = c.batch(small, use_graph=True, kernel=int(kernel))
        assert [r.raw for r in again] == [r.raw for r in first]
        for q, r in list(zip(small, again))[::7]:
            assert r.raw == run(c, q, kernel).raw


def test_super_a_sweep_k16_batched(ctx, kernel):
    """The 256-candidate k=16 sweep in one launch: every instance equals its own run,
    and the archived sweep pins (results/superAs/superA_n16_h16.txt) hold."""
    As = super_a_set(256)
    reqs = [an_req(A, 16, convention=dd.CONV_SUPER_A) for A in As]
    out = ctx.batch(reqs, use_graph=True, kernel=int(kernel))
    for r in out:
        ran(r, kernel)
    for A, r in list(zip(As, out))[::32]:
        s = run(ctx, an_req(A, 16, convention=dd.CONV_SUPER_A), kernel)
        assert r.counts == s.counts
    pins = next(f for f in golden("super_a.json") if f["n"] == 16 and f["h"] == 16)["pins"]
    pin_reqs = [an_req(A, 16) for A, _, _ in pins]
    for (A, minb, mincb), r in zip(pins, ctx.batch(pin_reqs, kernel=int(kernel))):
        ran(r, kernel)
        assert (r.minb, r.mincb) == (minb, mincb), A
    # one exact oracle check of the batch
    assert out[0].raw == oracle.an_exhaustive_raw(As[0], 16, out[0].nbins)
