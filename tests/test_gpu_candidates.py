"""The super-A candidate pre-filter on the GPU (dd_an_candidates, bin/ancandidates)
against the reference's ANcandidates tool (golden digests of every cell with A
width 1..17 and data width 1..24) and the oracle; the candidates file feeding
the batched super-A sweep of bin/codrel_supera."""
import hashlib
import json
import subprocess
from pathlib import Path

import pytest

import coding_reliability_b200 as dd
import oracle

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = json.loads((ROOT / "tests" / "golden" / "ancandidates.json").read_text())
BIN = ROOT / "coding_reliability_b200" / "bin"


def digest(lst):
    return hashlib.sha256(",".join(str(a) for a in lst).encode()).hexdigest()


def test_every_golden_cell(ctx):
    for c in GOLDEN:
        info, lst = ctx.an_candidates(c["k"], c["a"])
        assert info["sdr"] == c["sdr"] and info["num_candidates"] == c["count"], c
        assert lst == sorted(lst) and digest(lst) == c["sha256"], (c["k"], c["a"])
        if c["candidates"] is not None:
            assert lst == c["candidates"]
        assert info["num_A"] == (1 << (c["a"] - 2) if c["a"] >= 2 else 0)


@pytest.mark.parametrize("k,a", [(5, 20), (9, 18), (12, 19), (24, 10), (26, 8), (28, 6)])
def test_cells_beyond_the_golden_range_vs_oracle(ctx, k, a):
    info, lst = ctx.an_candidates(k, a)
    assert (info["sdr"], lst) == oracle.an_candidates(k, a)


def test_short_list_returns_the_smallest(ctx):
    info, full = ctx.an_candidates(12, 13)
    assert info["num_candidates"] == len(full) > 10
    info2, part = ctx.an_candidates(12, 13, capacity=10)
    assert info2["num_candidates"] == len(full) and part == full[:10]
    info3, none = ctx.an_candidates(12, 13, capacity=0)
    assert info3["num_candidates"] == len(full) and none == []


@pytest.mark.parametrize("k,a", [(0, 8), (49, 4), (8, 0), (8, 33), (40, 22)])
def test_invalid_widths(ctx, k, a):
    with pytest.raises(dd.DDError) as e:
        ctx.an_candidates(k, a)
    assert e.value.status == 1


def expected_rows(amin, amax, dmin, dmax):
    cells = {(c["k"], c["a"]): c for c in GOLDEN}
    rows = []
    for a in range(amin, amax + 1):
        for k in range(dmin, dmax + 1):
            sdr, lst = oracle.an_candidates(k, a)
            c = cells.get((k, a))
            if c:
                assert (sdr, len(lst), digest(lst)) == (c["sdr"], c["count"], c["sha256"])
            rows.append(f"{k + a}\t{k}\t{a}\t{sdr}\t{len(lst)}\t" + ",".join(map(str, lst)))
    return rows


def test_cli_output_layout(tmp_path):
    out = subprocess.run([str(BIN / "ancandidates"), "-a", "2", "-A", "12", "-d", "2", "-D", "16",
                          "--csv", str(tmp_path / "cand")], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.splitlines()
    assert lines[:3] == ["# bit width data = [2,16]", "# bit width A = [2,12]",
                         "# n=|C|\tk=|D|\t|A|\t|SDR|\t|candidates|\tcandidates"]
    assert lines[3:] == expected_rows(2, 12, 2, 16)
    f = (tmp_path / "cand_k12_a12.csv").read_text().strip()
    assert f == "3349,3365,3493,3691,3737,3997,4051"


def test_candidates_feed_the_super_a_sweep(tmp_path):
    """ancandidates --csv -> codrel_supera -c: the super-A of the k=16, 16-bit
    candidates, checked against the oracle's exact histograms."""
    r = subprocess.run([str(BIN / "ancandidates"), "-a", "16", "-A", "16", "-d", "16", "-D", "16", "--csv", "cand"],
                       capture_output=True, text=True, cwd=tmp_path, timeout=300)
    assert r.returncode == 0, r.stderr
    cand = tmp_path / "cand_k16_a16.csv"
    As = [int(x) for x in cand.read_text().strip().split(",")]
    assert As == [58659, 63157, 63859, 63877]
    r = subprocess.run([str(BIN / "codrel_supera"), "-k", "16", "-c", cand.name, "-f", "sweep"],
                       capture_output=True, text=True, cwd=tmp_path, timeout=300)
    assert r.returncode == 0, r.stderr
    out = tmp_path / "sweep_k16_c_cand_k16_a16.csv.csv"
    assert out.exists(), sorted(p.name for p in tmp_path.iterdir())
    rows = [l.split(",") for l in out.read_text().splitlines() if l and l[0].isdigit() and "," in l]
    rows = [r for r in rows if len(r) > 40]
    assert [int(r[2]) for r in rows] == As
    best = None
    for A in As:
        h = oracle.h_floor1(A)
        counts = oracle.an_exhaustive_counts(A, 16, 16 + h + 1)
        minb, mincb = next((i, c) for i, c in enumerate(counts[1:(16 + h + 2) // 2], 1) if c)
        if best is None or minb > best[0] or (minb == best[0] and mincb < best[1]):
            best = (minb, mincb, A)
    last = rows[-1]
    assert (int(last[-6]), int(last[-5]), int(last[-4])) == best
