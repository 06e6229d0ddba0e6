"""Host-side behaviour of the C-ABI that needs no GPU: exported symbols, the
reference drivers' shape rules, post-processing, results-file layout, Philox,
error statuses."""
import random
import re
from pathlib import Path

import pytest

import coding_reliability_b200 as dd
import oracle
from conftest import ROOT, golden


def header_symbols():
    syms = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        syms |= set(re.findall(r"\b(dd_[a-z0-9_]+)\s*\(", text))
    return syms


def test_library_exports_every_declared_symbol(lib):
    syms = header_symbols()
    assert {"dd_histogram", "dd_batch_run", "dd_context_create", "dd_postprocess"} <= syms
    for s in sorted(syms):
        assert hasattr(lib, s), f"{s} declared in include/ but not exported"


def test_version_and_status_strings(lib):
    assert b"sm_100a" in lib.dd_version()
    assert lib.dd_status_string(0) == b"ok"
    assert lib.dd_status_string(7) == b"timeout"


@pytest.mark.parametrize("A", [1, 2, 3, 61, 64, 641, 1021, 32768, 32771, 58659, 65535, 65536, 65537])
def test_shape_rules_an(lib, A):
    n = 16
    nb, h, a = dd.request_shape(dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, A, n))
    Aeff = 1 if A & (A - 1) == 0 else A            # src/an_coding.cu:278-279
    assert (a, h, nb) == (Aeff, oracle.h_ceil(Aeff), n + oracle.h_ceil(Aeff) + 1)
    nb, h, a = dd.request_shape(dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, A, n, convention=dd.CONV_CPU))
    assert (a, h) == (A, oracle.h_ceil(A))          # src/an_coding.cpp:111, no normalisation
    nb, h, a = dd.request_shape(dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, A, n, convention=dd.CONV_SUPER_A))
    assert (a, h) == (Aeff, oracle.h_floor1(A))     # super_a/src/main.cpp:261


@pytest.mark.parametrize("n", [4, 8, 16, 24, 32, 40, 48])
def test_shape_rules_hamming(lib, n):
    nb, h, _ = dd.request_shape(dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, n))
    assert h == oracle.hamming_h(n) and nb == n + h + 1


@pytest.mark.parametrize("req,status", [
    (dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, 12), 2),    # "Unsupported n."
    (dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 65537, 48), 2),        # n+h+1 > 64
    (dd.Request(dd.CODE_AN, dd.MODE_GRID_1D, 61, 16, m=2), 1),         # assert(iterations >= 3)
    (dd.Request(dd.CODE_AN, dd.MODE_MONTE_CARLO, 61, 16, m=0), 1),
    (dd.Request(7, dd.MODE_EXHAUSTIVE, 61, 16), 1),
    (dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 58659, 16, h=3, convention=dd.CONV_SUPER_A), 1),  # h too small
    (dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_GRID_2D, 1, 16, m=5), 1),
    (dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 1 << 33, 8), 2),
])
def test_invalid_requests_return_status(lib, req, status):
    with pytest.raises(dd.DDError) as e:
        dd.request_shape(req)
    assert e.value.status == status


def test_context_without_device_fails_loudly(lib):
    if dd.device_count() > 0:
        pytest.skip("a device is present")
    with pytest.raises(dd.DDError) as e:
        dd.Context(0)
    assert e.value.status == 4


def _rand_raw(nb, rng, scale=1 << 40):
    return [rng.randrange(scale) for _ in range(nb)]


def test_postprocess_an_exhaustive_matches_oracle(lib):
    rng = random.Random(1)
    for A, n in [(641, 12), (58659, 24), (61, 16), (1, 20)]:
        req = dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, A, n)
        nb, _, _ = dd.request_shape(req)
        raw = [0] + _rand_raw(nb - 1, rng)
        got = dd.postprocess(req, raw)
        import ctypes as C
        lo, hi = (C.c_uint64 * 64)(), (C.c_uint64 * 64)()
        oracle.lib().dd_oracle_post_an_exhaustive(n, (C.c_uint64 * 64)(*raw), nb, lo, hi)
        assert got.counts == [(hi[i] << 64) | lo[i] for i in range(nb)]
        # minb: first non-zero in [1, nb/2)
        first = next((i for i in range(1, nb // 2) if got.counts[i]), 0xFFFF)
        assert got.minb == first


def test_postprocess_grid_and_mc_match_oracle(lib):
    rng = random.Random(2)
    for A, n, m, m2 in [(61, 24, 100, 0), (61, 16, 1001, 0), (641, 20, 4096, 0), (61, 16, 333, 77)]:
        for mode in (dd.MODE_GRID_1D, dd.MODE_GRID_2D, dd.MODE_MONTE_CARLO):
            if mode != dd.MODE_GRID_2D and m2:
                continue
            req = dd.Request(dd.CODE_AN, mode, A, n, m=m, m2=m2 or m)
            nb, _, _ = dd.request_shape(req)
            raw = _rand_raw(nb, rng, 1 << 44)
            got = dd.postprocess(req, raw)
            if mode == dd.MODE_MONTE_CARLO:
                exp = oracle.an_mc_counts(n, m, raw)
            else:
                gd = 1 if mode == dd.MODE_GRID_1D else 2
                r2 = list(raw)
                if gd == 2:
                    r2[0] = 0
                exp = oracle.an_grid_counts(gd, n, m, m2 or m, r2)
            assert got.counts == exp, (A, n, m, mode)


def test_postprocess_hamming_matches_oracle(lib):
    for n in (8, 16, 24):
        nb = n + oracle.hamming_h(n) + 1
        raw = oracle.hamming_weights_raw(n, nb)
        for w1 in (0, 1):
            got = dd.postprocess(dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, n, with_1bit=w1), raw)
            assert got.counts == oracle.hamming_weights_counts(n, w1, raw)
    rng = random.Random(3)
    for n, m in [(16, 4096), (24, 1 << 20), (32, 1 << 20)]:
        nb = n + oracle.hamming_h(n) + 1
        raw = _rand_raw(nb, rng, 1 << 30)
        for mode, is_mc in ((dd.MODE_GRID_1D, 0), (dd.MODE_MONTE_CARLO, 1)):
            for w1 in (0, 1):
                got = dd.postprocess(dd.Request(dd.CODE_EXT_HAMMING, mode, 1, n, m=m, with_1bit=w1), raw)
                assert got.counts == oracle.hamming_sampled_counts(is_mc, n, w1, m, raw)


def test_postprocess_hamming_all_pairs_equals_brute_force(lib):
    """raw = unordered pairs; the post-processing must give the `-e 2 [-b]` counts."""
    n = 8
    nb = n + oracle.hamming_h(n) + 1
    # unordered i<j histogram of extended codewords
    cws = [oracle.lib().dd_oracle_hamming_cw_ext(x, n) for x in range(1 << n)]
    raw = [0] * nb
    for i in range(len(cws)):
        for j in range(i + 1, len(cws)):
            raw[bin(cws[i] ^ cws[j]).count("1")] += 1
    for w1 in (0, 1):
        got = dd.postprocess(dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, n, with_1bit=w1,
                                        hamming_method=dd.HAMMING_ALL_PAIRS), raw)
        assert got.counts == oracle.hamming_pairs_raw(n, w1, nb)


def _table_part(text):
    """Rows, blank lines and the Total line; runtime rows masked."""
    out = []
    for line in text.splitlines():
        if "Runtime" in line:
            line = re.sub(r",[0-9.e+-]+,s$", ",<t>,s", line)
        if line.startswith("Sum counts") or line.startswith(" A = ") or line.startswith("Start "):
            break
        out.append(line)
    while out and out[-1] == "":
        out.pop()
    return out


@pytest.mark.parametrize("run", [r for r in golden("ref_runs.json") if r["args"][0] in ("-a", "-e")],
                         ids=lambda r: " ".join(r["args"]))
def test_results_file_layout_matches_reference(lib, run):
    """dd_format_result renders the reference's own output byte for byte (timings masked)."""
    args = run["args"]
    if args[0] == "-a":
        req = dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, int(args[1]), int(args[3]), convention=dd.CONV_CPU)
        nb, _, _ = dd.request_shape(req)
        raw = [0] + [c // 2 for c in run["counts"][1:]]
    else:
        n = int(args[-1])
        w1 = int("-b" in args)
        method = {"1": dd.HAMMING_WEIGHTS, "2": dd.HAMMING_ALL_PAIRS, "3": dd.HAMMING_ALL_PAIRS_DISTINCT,
                  "4": dd.HAMMING_ALL_PAIRS}[args[1]]
        req = dd.Request(dd.CODE_EXT_HAMMING, dd.MODE_EXHAUSTIVE, 1, n, with_1bit=w1, hamming_method=method,
                         convention=dd.CONV_CPU if "-c" in args else dd.CONV_GPU)
        nb, _, _ = dd.request_shape(req)
        if method == dd.HAMMING_WEIGHTS:
            raw = oracle.hamming_weights_raw(n, nb)
        else:
            if n > 8:
                pytest.skip("n > 8 brute force in Python is slow; the GPU tests cover it")
            cws = [oracle.lib().dd_oracle_hamming_cw_ext(x, n) for x in range(1 << n)]
            raw = [0] * nb
            for i in range(len(cws)):
                for j in range(i + 1, len(cws)):
                    raw[bin(cws[i] ^ cws[j]).count("1")] += 1
            if n > 8:
                pytest.skip("n > 8 brute force in Python is slow")
    res = dd.postprocess(req, raw)
    assert res.counts == run["counts"]
    text = dd.format_result(req, res, "")
    ref = run["stdout"]
    ref_lines = [l for l in ref.splitlines() if not l.startswith("Start ")]
    assert _table_part(text) == _table_part("\n".join(ref_lines))


def test_philox_library_matches_oracle(lib):
    rng = random.Random(4)
    for _ in range(200):
        ctr = tuple(rng.randrange(1 << 32) for _ in range(4))
        key = tuple(rng.randrange(1 << 32) for _ in range(2))
        assert dd.philox4x32_10(ctr, key) == oracle.philox(ctr, key)


def _grid_cases():
    cases = []
    for n in (8, 10, 12, 16, 20, 24, 28, 31):
        N = 1 << n
        for m in sorted({3, 4, 7, 13, 16, 17, 64, 100, 127, 128, 129, 1000, 1001, 4096, 65536, 100001,
                         N - 1, N, N + 5, N // 2, N // 3}):
            if 3 <= m:
                cases.append((61, n, m))
    return cases + [(58659, 16, 333), (58659, 24, 65536), (1, 24, 400000), (65533, 24, 400000), (3, 9, 512)]


@pytest.mark.parametrize("A,n,m", _grid_cases())
def test_grid_lattice_points_match_reference_walk(lib, A, n, m):
    """The lattice size comes from a search over k; it must equal the reference's
    sequential walk (an_coding_grid.cu:78-107) for every m, powers of two included."""
    req = dd.Request(dd.CODE_AN, dd.MODE_GRID_1D, A, n, m=m)
    try:
        nb, h, Aeff = dd.request_shape(req)
    except dd.DDError:
        pytest.skip("n+h+1 > 64")
    plan = dd.request_plan(req)
    assert plan["lattice"] == oracle.grid1d_points(Aeff, n, h, m)
    req2 = dd.Request(dd.CODE_AN, dd.MODE_GRID_2D, A, n, m=m, m2=m)
    assert dd.request_plan(req2)["lattice"] == oracle.grid2d_points(Aeff, n, m)
