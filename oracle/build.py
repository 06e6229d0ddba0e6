"""Builds the checker side: the C restatement (oracle/_build/libdd_oracle.so)
and, where the reference's sources are present, the reference's own tool
(oracle/_ref/ref_codrel, ref_codrel_supera, ref_ancandidates) via oracle/ref.mk.

Test infrastructure only; the product never loads anything built here.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_build"
LIB = OUT / "libdd_oracle.so"
REF_OUT = HERE / "_ref"
# The reference checkout: $CODREL_REFERENCE, else a checkout named `reference`
# beside this repository.
REF_SRC = Path(os.environ.get("CODREL_REFERENCE", str(HERE.parent.parent / "reference")))


def build_oracle() -> Path:
    OUT.mkdir(exist_ok=True)
    src = HERE / "dd_oracle.c"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        cmd = ["gcc", "-O3", "-fopenmp", "-shared", "-fPIC", "-o", str(LIB), str(src), "-lm"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError("oracle build failed")
    return LIB


def build_reference() -> bool:
    """Compiles the reference tool when its sources exist; True if available."""
    if all((REF_OUT / b).exists() for b in ("ref_codrel", "ref_codrel_supera", "ref_ancandidates")):
        return True
    if not (REF_SRC / "distance_distribution" / "src" / "main.cpp").exists():
        return False
    cmd = ["make", "-s", "-j8", "-f", str(HERE / "ref.mk"), f"REF={REF_SRC}", f"OUT={REF_OUT}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("reference build failed")
    return True


if __name__ == "__main__":
    print(build_oracle())
    print("reference:", build_reference())
