"""Records the output files of the reference's super-A tool (its GPU path,
oracle/_ref/ref_codrel_supera built from distance_distribution_super_a/src by
oracle/ref.mk) for a few sweeps, as the golden fixture supera_ref.json.

Needs a GPU.  Every case passes `-d 1`, so the tool uses device 0 only.  The
inputs were checked by reading the tool's kernels (an_coding.cu:32-128 of the
super-A fork): data widths k >= 4 (the k < 4 kernel adds 32 bins into an
allocation of k+h+1), and k+h+1 <= 48, so every shared and global bin index
stays inside its array.

Run from the repo root:  python tests/golden/make_supera_golden.py OUT.json
"""
from __future__ import annotations

import json
import subprocess
import sys
import tempfile
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent.parent
EXE = ROOT / "oracle" / "_ref" / "ref_codrel_supera"

CANDIDATES = "58659,63157,63859,63877\n"  # ANcandidates' k=16, 16-bit cell
CASES = [
    ["-k", "8", "-s", "129", "-S", "255", "-d", "1", "-f", "ref"],
    ["-k", "8", "-s", "1", "-S", "63", "-d", "1", "-f", "ref"],
    ["-k", "12", "-s", "1001", "-S", "1101", "-d", "1", "-f", "ref"],
    ["-k", "16", "-c", "cand.csv", "-d", "1", "-f", "ref"],
    ["-k", "16", "-a", "58659", "-d", "1", "-f", "ref"],
    ["-k", "10", "-a", "64", "-d", "1", "-f", "ref"],
]


def run_case(args: list[str]) -> dict:
    with tempfile.TemporaryDirectory() as d:
        (Path(d) / "cand.csv").write_text(CANDIDATES)
        res = subprocess.run([str(EXE)] + args, capture_output=True, text=True, cwd=d, timeout=600)
        if res.returncode != 0:
            raise RuntimeError(f"{args}: rc {res.returncode}: {res.stderr[-400:]}")
        files = sorted(p for p in Path(d).glob("*.csv") if p.name != "cand.csv")
        if len(files) != 1:
            raise RuntimeError(f"{args}: expected one output file, got {[p.name for p in files]}")
        return {"args": args, "file": files[0].name, "content": files[0].read_text()}


def main() -> None:
    out = Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent / "supera_ref.json"
    data = {"candidates_file": CANDIDATES, "cases": [run_case(a) for a in CASES]}
    out.write_text(json.dumps(data, indent=0))
    print(out, out.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
