"""Monte Carlo continuation (dd_mc_extend): growing the sample count from an
earlier run gives bit-identical histograms to a fresh run, so an error-bound
search never redraws samples (the reference's search restarts each step,
distance_distribution/src/main.cpp:179-202)."""
import re
import subprocess
from pathlib import Path

import pytest

import coding_reliability_b200 as dd

pytestmark = pytest.mark.gpu

BIN = Path(__file__).resolve().parent.parent / "coding_reliability_b200" / "bin"


def mc(A, n, m, seed=16384):
    return dd.Request(dd.CODE_AN, dd.MODE_MONTE_CARLO, A, n, m=m, seed=seed)


def same(a, b):
    assert a.raw == b.raw and a.counts == b.counts and a.minb == b.minb
    assert a.max_rel_error == b.max_rel_error


def test_chain_equals_fresh(ctx):
    A, n = 61, 16
    done, raw = 0, []
    for m in (1, 3, 9, 27, 81):
        r = ctx.mc_extend(mc(A, n, m), done, raw)
        same(r, ctx.histogram(mc(A, n, m)))
        assert r.pairs == (1 << n) * (m - done)
        done, raw = m, r.raw


@pytest.mark.parametrize("A,n,done,m", [(641, 12, 5, 17), (641, 12, 2, 3), (58659, 20, 7, 300),
                                        (61, 33, 3, 5), (255, 24, 1, 2)])
def test_unaligned_and_wide_continuations(ctx, A, n, done, m):
    first = ctx.histogram(mc(A, n, done, seed=99))
    r = ctx.mc_extend(mc(A, n, m, seed=99), done, first.raw)
    same(r, ctx.histogram(mc(A, n, m, seed=99)))


def test_nothing_left_to_draw(ctx):
    first = ctx.histogram(mc(641, 12, 40))
    r = ctx.mc_extend(mc(641, 12, 40), 40, first.raw)
    same(r, first)


def test_refused_requests(ctx):
    first = ctx.histogram(mc(641, 12, 40))
    with pytest.raises(dd.DDError) as e:
        ctx.mc_extend(mc(641, 12, 30), 40, first.raw)
    assert e.value.status == 1
    with pytest.raises(dd.DDError) as e:
        ctx.mc_extend(dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 641, 12), 0, [])
    assert e.value.status == 2
    with pytest.raises(dd.DDError) as e:
        ctx.mc_extend(dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_MONTE_CARLO, 1, 16, m=4), 0, [])
    assert e.value.status == 2


def test_cli_error_bound_search(ctx, tmp_path):
    """codrel -s: the search stops at the first step whose fresh histogram meets
    the bound, and every step reports a fresh run's error."""
    bound = 0.05
    r = subprocess.run([str(BIN / "codrel"), "-a", "61", "-n", "16", "-s", str(bound)], capture_output=True,
                       text=True, cwd=tmp_path, timeout=300)
    assert r.returncode == 0, r.stderr
    steps = [(int(a), float(b)) for a, b in re.findall(r"^(\d+) iterations - max\. rel\. error ([0-9.]+)$",
                                                         r.stdout, re.M)]
    assert steps and all(b[0] == 3 * a[0] for a, b in zip(steps, steps[1:]))
    for it, err in steps:
        fresh = ctx.histogram(mc(61, 16, it))
        assert abs(fresh.max_rel_error - err) < 1e-6
    assert steps[-1][1] <= bound and all(err > bound for _, err in steps[:-1])
    assert f"Achieved error of {steps[-1][1]:f} after {steps[-1][0]} iterations" in r.stdout
    rows = (tmp_path / "ancoding_mc_search.csv").read_text().splitlines()
    assert len(rows) == len(steps) and rows[0].startswith(f"0,16,0.050000,{steps[0][0]},")
