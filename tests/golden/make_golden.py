"""Generates the golden fixtures under tests/golden/ from the reference.

Sources (all read from the reference checkout: $CODREL_REFERENCE, else the
checkout named `reference` beside this repository):
  * distance_distribution/src/solutions.h           exact AN / Ext-Hamming tables
  * distance_distribution/results/As/*.csv          exhaustive AN histograms (many A, n=8..24)
  * distance_distribution/results/{GridMs,converge/geom,runtimes/0,As}/*grid1d*.csv
                                                   1-D grid histograms (A=61 and others)
  * distance_distribution/results/superAs/*.txt    super-A sweep minima
  * distance_distribution/results/converge/{pseudo,sobol,sobolSinus}/*.csv
                                                   the reference's Monte Carlo runs (A=61)
  * the reference's own tool built from its sources (oracle/_ref/ref_codrel):
    full stdout of CPU-path runs, used for the results-file layout and counts.
  * the reference's ANcandidates tool built from its source
    (oracle/_ref/ref_ancandidates): |SDR|, count and a SHA-256 of the sorted
    candidate list of every cell with A width 1..17 and data width 1..24
    (about 5 minutes on 16 cores for the widths 15..17).

Run from the repo root:  python tests/golden/make_golden.py [fixture.json ...]
"""
from __future__ import annotations

import json
import os
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
# the reference checkout: $CODREL_REFERENCE, else a checkout named `reference`
# beside this repository
REF = Path(os.environ.get("CODREL_REFERENCE", str(ROOT.parent / "reference")))
RES = REF / "distance_distribution" / "results"
sys.path.insert(0, str(ROOT))

ROW = re.compile(r"^\s*(\d+),\s*([0-9.e+]+),\s*([0-9.e+-]+),\s*([0-9.e+-]+)")


def parse_counts(path: Path) -> list:
    counts = []
    for line in path.read_text().splitlines():
        m = ROW.match(line)
        if not m:
            if counts:
                break
            continue
        i = int(m.group(1))
        if i != len(counts):
            break
        tok = m.group(2)
        counts.append(int(tok) if tok.isdigit() else tok)  # long double print for >2^64
    return counts


def kernel_time(path: Path):
    m = re.search(r'"Kernel Runtime",([0-9.e+-]+),s', path.read_text())
    return float(m.group(1)) if m else None


def solutions() -> dict:
    text = (REF / "distance_distribution" / "src" / "solutions.h").read_text()
    out = {}
    for m in re.finditer(r"const uint128_t\s+(\w+)\[\]\s*=\s*\{([^}]*)\}", text):
        out[m.group(1)] = [int(x.strip().rstrip("ull")) for x in m.group(2).replace("\n", " ").split(",") if x.strip()]
    return out


def an_exhaustive() -> list:
    out = []
    for p in sorted((RES / "As").glob("ancoding_gpu_A*_n*_h*.csv")):
        m = re.match(r"ancoding_gpu_A(\d+)_n(\d+)_h(\d+)\.csv", p.name)
        out.append({"file": f"results/As/{p.name}", "A": int(m.group(1)), "n": int(m.group(2)),
                    "h": int(m.group(3)), "counts": parse_counts(p), "kernel_s": kernel_time(p)})
    for p in sorted((RES / "runtimes" / "0").glob("ancoding_gpu_A*_n*_h*.csv")):
        m = re.match(r"ancoding_gpu_A(\d+)_n(\d+)_h(\d+)\.csv", p.name)
        out.append({"file": f"results/runtimes/0/{p.name}", "A": int(m.group(1)), "n": int(m.group(2)),
                    "h": int(m.group(3)), "counts": parse_counts(p), "kernel_s": kernel_time(p)})
    return out


def an_grid() -> list:
    out = []
    pats = [(RES / "GridMs", "ancoding_grid1d_gpu_m*_A*_n*_h*.csv"),
            (RES / "converge" / "geom", "ancoding_grid1d_gpu_m*_A*_n*_h*.csv"),
            (RES / "runtimes" / "0", "ancoding_grid1d_gpu_m*_A*_n*_h*.csv"),
            (RES / "As", "ancoding_grid1d_m*_A*_n*_h*.csv")]
    for d, pat in pats:
        for p in sorted(d.glob(pat)):
            m = re.match(r"ancoding_grid1d_(?:gpu_)?m(\d+)_A(\d+)_n(\d+)_h(\d+)\.csv", p.name)
            out.append({"file": str(p.relative_to(RES.parent)), "m": int(m.group(1)), "A": int(m.group(2)),
                        "n": int(m.group(3)), "h": int(m.group(4)), "counts": parse_counts(p),
                        "kernel_s": kernel_time(p)})
    return out


def an_mc_converge() -> list:
    """The reference's Monte Carlo runs (cuRAND pseudo-random, Sobol and
    scrambled-Sobol draws) of A=61, n=16/24 at many sample counts; the draws
    cannot be replayed, so these pin the Monte Carlo path statistically."""
    out = []
    for kind in ("pseudo", "sobol", "sobolSinus"):
        for p in sorted((RES / "converge" / kind).glob("ancoding_mc_gpu_m*_A*_n*_h*.csv")):
            m = re.match(r"ancoding_mc_gpu_m(\d+)_A(\d+)_n(\d+)_h(\d+)\.csv", p.name)
            out.append({"file": str(p.relative_to(RES.parent)), "kind": kind, "m": int(m.group(1)),
                        "A": int(m.group(2)), "n": int(m.group(3)), "h": int(m.group(4)),
                        "counts": parse_counts(p)})
    return out


def super_a() -> list:
    out = []
    for p in sorted((RES / "superAs").glob("superA_n*_h*.txt")):
        m = re.match(r"superA_n(\d+)_h(\d+)\.txt", p.name)
        n, h = int(m.group(1)), int(m.group(2))
        pins, summary = [], None
        for line in p.read_text().splitlines():
            mm = re.match(r"^(\d+): c\[(\d+)\] = (\d+)$", line.strip())
            if mm:
                pins.append([int(mm.group(1)), int(mm.group(2)), int(mm.group(3))])
            elif line.startswith("n,"):
                summary = line.strip()
        out.append({"file": f"results/superAs/{p.name}", "n": n, "h": h, "pins": pins, "summary": summary})
    return out


REF_CASES = [
    ["-a", "641", "-n", "12", "-c"],
    ["-a", "61", "-n", "8", "-c"],
    ["-a", "61", "-n", "12", "-c"],
    ["-a", "641", "-n", "10", "-c"],
    ["-a", "58659", "-n", "10", "-c"],
    ["-a", "58659", "-n", "12", "-c"],
    ["-a", "64", "-n", "10", "-c"],
    ["-a", "3", "-n", "9", "-c"],
    ["-a", "1", "-n", "8", "-c"],
    ["-a", "255", "-n", "11", "-c"],
    ["-a", "32771", "-n", "8", "-c"],
    ["-a", "65521", "-n", "9", "-c"],
    ["-e", "1", "-c", "-n", "8"],
    ["-e", "1", "-c", "-b", "-n", "8"],
    ["-e", "1", "-c", "-n", "16"],
    ["-e", "1", "-c", "-b", "-n", "16"],
    ["-e", "1", "-c", "-b", "-n", "24"],
    ["-e", "2", "-n", "8"],
    ["-e", "2", "-b", "-n", "8"],
    ["-e", "3", "-b", "-n", "8"],
]


def ref_runs() -> list:
    import oracle
    oracle.build_reference()
    out = []
    for args in REF_CASES:
        text = oracle.ref_run(args)
        out.append({"args": args, "stdout": text, "counts": oracle.parse_table(text)})
    # sizes that take seconds on the CPU path; recorded, not re-run by the tests
    for args in (["-a", "58659", "-n", "16", "-c"], ["-e", "2", "-b", "-n", "16"]):
        text = oracle.ref_run(args, timeout=900)
        out.append({"args": args, "stdout": text, "counts": oracle.parse_table(text)})
    return out


def candidates_digest(lst: list) -> str:
    import hashlib
    return hashlib.sha256(",".join(str(a) for a in sorted(lst)).encode()).hexdigest()


def ancandidates() -> list:
    import oracle
    oracle.build_reference()
    out = []
    for amin, amax in ((1, 14), (15, 17)):
        cells = oracle.parse_candidates(oracle.ref_ancandidates(amin, amax, 1, 24, timeout=3600))
        for (k, a), (sdr, lst) in sorted(cells.items(), key=lambda kv: (kv[0][1], kv[0][0])):
            out.append({"k": k, "a": a, "sdr": sdr, "count": len(lst), "sha256": candidates_digest(lst),
                        "candidates": lst if len(lst) <= 16 else None})
    return out


FIXTURES = {
    "solutions.json": solutions,
    "an_exhaustive.json": an_exhaustive,
    "an_grid1d.json": an_grid,
    "an_mc_converge.json": an_mc_converge,
    "super_a.json": super_a,
    "ref_runs.json": ref_runs,
    "ancandidates.json": ancandidates,
}


def main() -> None:
    names = sys.argv[1:] or list(FIXTURES)
    for name in names:
        data = FIXTURES[name]()
        (HERE / name).write_text(json.dumps(data, indent=0, sort_keys=True))
        print(name, (HERE / name).stat().st_size, "bytes")


if __name__ == "__main__":
    main()
