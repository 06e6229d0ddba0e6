"""Pins the CPU oracle (oracle/dd_oracle.c) to the reference: its golden
tables (src/solutions.h), its archived result files (results/As, GridMs,
converge, runtimes, superAs) and its own tool run on the CPU path.  Only when
these hold is the oracle trusted as the checker of the GPU path."""
import pytest

import oracle
from conftest import golden


def test_philox_known_answers():
    # Known-answer vectors of Philox4x32-10 published with Random123.
    assert oracle.philox((0, 0, 0, 0), (0, 0)) == (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)
    assert oracle.philox((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2) == (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)
    assert oracle.philox((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0)) == (
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)


@pytest.mark.parametrize("A,n", [(61, 8), (641, 8), (61, 16), (641, 16)])
def test_an_solutions_h(A, n):
    sol = golden("solutions.json")[f"solution_an{n}_A{A}"]
    h = oracle.h_ceil(A)
    got = oracle.an_exhaustive_counts(A, n, n + h + 1)
    k = min(len(got), len(sol))
    assert got[:k] == sol[:k]
    assert all(x == 0 for x in sol[k:]) and all(x == 0 for x in got[k:])


@pytest.mark.parametrize("n", [8, 16, 24])
def test_hamming_weight_table(n):
    sol = golden("solutions.json")[f"sol_hamming_n{n}"]
    h = oracle.hamming_h(n)
    raw = oracle.hamming_weights_raw(n, n + h + 1)
    # extended weight of even i = w[i] + w[i-1] (odd weights gain the overall parity bit)
    ext = [raw[i] + raw[i - 1] if i % 2 == 0 and i >= 2 else 0 for i in range(n + h + 1)]
    assert ext[4:] == sol[4: n + h + 1]


def _as_cases(max_n):
    return [c for c in golden("an_exhaustive.json") if c["n"] <= max_n]


@pytest.mark.parametrize("case", _as_cases(12), ids=lambda c: c["file"].split("/")[-1])
def test_an_results_archive_small(case):
    """results/As exhaustive histograms (GPU runs of the reference), n <= 12."""
    A, n, h = case["A"], case["n"], case["h"]
    assert oracle.h_ceil(A if A & (A - 1) else 1) == h
    got = oracle.an_exhaustive_counts(A if A & (A - 1) else 1, n, n + h + 1)
    assert got == case["counts"]


def test_an_results_archive_n16_sample():
    cases = [c for c in golden("an_exhaustive.json") if c["n"] == 16][::16]
    assert cases
    for c in cases:
        assert oracle.an_exhaustive_counts(c["A"], 16, 16 + c["h"] + 1) == c["counts"], c["file"]


def test_an_grid_archive():
    """results/*grid1d* files: the lattice walk with double stepsize, n <= 24."""
    checked = 0
    for x in golden("an_grid1d.json"):
        if x["n"] > 24 or any(isinstance(c, str) for c in x["counts"]) or (x["n"] == 24 and x["m"] > 103):
            continue  # larger n=24 lattices are checked on the GPU
        A, n, h, m = x["A"], x["n"], x["h"], x["m"]
        A = A if A & (A - 1) else 1
        raw, _ = oracle.an_grid1d_raw(A, n, h, m, len(x["counts"]))
        assert oracle.an_grid_counts(1, n, min(m, 1 << n), 0, raw) == x["counts"], x["file"]
        checked += 1
    assert checked >= 15


def test_super_a_archive_pins_n8():
    """results/superAs/superA_n8_h*.txt: c[minb] of every improving A (exact sweeps)."""
    for f in golden("super_a.json"):
        if f["n"] != 8:
            continue
        for A, minb, mincb in f["pins"]:
            h = oracle.h_ceil(A)
            c = oracle.an_exhaustive_counts(A, 8, 8 + h + 1)
            nb = 8 + h + 1
            first = next((i for i in range(1, nb // 2) if c[i]), None)
            assert (first, c[first]) == (minb, mincb), (f["file"], A)


def test_super_a_archive_pin_58659():
    pins = {p[0]: p for f in golden("super_a.json") if f["n"] == 16 and f["h"] == 16 for p in f["pins"]}
    A, minb, mincb = pins[58659]
    c = oracle.an_exhaustive_counts(A, 16, 16 + 16 + 1)
    assert (minb, c[minb]) == (6, mincb)


@pytest.mark.parametrize("run", golden("ref_runs.json"), ids=lambda r: " ".join(r["args"]))
def test_reference_tool_runs(run):
    """The reference's own CPU path (built from its sources) against the oracle."""
    args = run["args"]
    counts = run["counts"]
    if args[0] == "-a":
        A, n = int(args[1]), int(args[3])
        assert oracle.an_exhaustive_counts(A, n, len(counts)) == counts
    elif args[:2] == ["-e", "1"]:
        n = int(args[-1])
        w1 = "-b" in args
        raw = oracle.hamming_weights_raw(n, len(counts))
        assert oracle.hamming_weights_counts(n, int(w1), raw) == counts
    else:
        n = int(args[-1])
        w1 = "-b" in args
        if n > 8:
            pytest.skip("brute force at n=16 takes a minute; covered on the GPU")
        f = oracle.hamming_pairs_distinct_raw if args[1] == "3" else oracle.hamming_pairs_raw
        assert f(n, int(w1), len(counts)) == counts


def test_hamming_all_pairs_equals_weight_enumerator():
    for n in (8,):
        for w1 in (0, 1):
            nb = n + oracle.hamming_h(n) + 1
            assert oracle.hamming_pairs_raw(n, w1, nb) == oracle.hamming_weights_counts(
                n, w1, oracle.hamming_weights_raw(n, nb))


def test_mc_index_layout():
    # four 32-bit samples per Philox block for n <= 32, top n bits
    seed, idx = 0x1234_5678_9ABC_DEF0, 77
    o = oracle.philox((0, 0, idx, 0), (seed & 0xFFFFFFFF, seed >> 32))
    assert [oracle.mc_index(seed, idx, t, 20) for t in range(4)] == [x >> 12 for x in o]
    o2 = oracle.philox((1, 0, idx, 0), (seed & 0xFFFFFFFF, seed >> 32))
    assert oracle.mc_index(seed, idx, 5, 32) == o2[1]
    # two 64-bit samples per block for n > 32
    assert oracle.mc_index(seed, idx, 1, 40) == ((o[2] << 32) | o[3]) >> 24


def _digest(lst):
    import hashlib
    return hashlib.sha256(",".join(str(a) for a in lst).encode()).hexdigest()


def test_candidates_oracle_vs_reference_golden():
    """ANcandidates cells (A width 1..14, data width 1..20) from the reference's
    own tool, against the oracle's restatement of its worker."""
    n = 0
    for c in golden("ancandidates.json"):
        if c["a"] > 14 or c["k"] > 20:
            continue
        sdr, lst = oracle.an_candidates(c["k"], c["a"])
        assert (sdr, len(lst), _digest(lst)) == (c["sdr"], c["count"], c["sha256"]), (c["k"], c["a"])
        if c["candidates"] is not None:
            assert lst == c["candidates"]
        n += 1
    assert n == 14 * 20


def test_candidates_reference_tool_live():
    if not oracle.ref_ancandidates_available():
        pytest.skip("reference ANcandidates not built")
    cells = oracle.parse_candidates(oracle.ref_ancandidates(2, 11, 1, 14))
    assert len(cells) == 10 * 14
    for (k, a), want in cells.items():
        assert oracle.an_candidates(k, a) == want


def test_naf_weight_early_exit():
    # the worker's early exit returns the running minimum once it is below the floor
    exact = oracle.naf_min(58659, 16)
    assert exact == 6
    assert oracle.naf_min(58659, 16, floor=exact) == exact
    assert oracle.naf_min(58659, 16, floor=exact + 1) < exact + 1
