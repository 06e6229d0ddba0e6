"""In-tree build of the CUDA library and the drop-in command-line tools.

Produces, next to this file:
  libcodrel_b200.so   the C-ABI (include/codrel_b200.h) + C++ drop-in drivers
  bin/codrel          the reference tool's command line (distance_distribution/src/main.cpp)
  bin/codrel_supera   the super-A fork's command line (distance_distribution_super_a/src/main.cpp)
  bin/ancandidates    the candidate pre-filter's command line (ANcandidates/ANcandidates.cpp)

Everything is compiled for sm_100a only.  Run `python -m coding_reliability_b200.build`.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libcodrel_b200.so"
BIN = PKG / "bin"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O3", f"-I{ROOT / 'include'}"]
LIB_SOURCES = ["dd_kernels.cu", "dd_mma.cu", "dd_host.cu", "dd_noalloc.cu", "dd_candidates.cu", "dd_server.cpp",
               "dd_rules.cpp", "dd_dropin.cpp"]
HEADERS = ["dd_device.cuh", "dd_jobs.h", "dd_kernels.h", "dd_host.h", "dd_mma.h"]
TOOLS = {"codrel": "codrel_main.cpp", "codrel_supera": "codrel_supera_main.cpp",
         "ancandidates": "codrel_ancandidates_main.cpp"}


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def _newer(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.exists() and d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd)}")


def build(verbose: bool = False) -> Path:
    """Compiles what is out of date and returns the library path."""
    BUILD.mkdir(exist_ok=True)
    BIN.mkdir(exist_ok=True)
    headers = [CSRC / h for h in HEADERS if (CSRC / h).exists()] + [ROOT / "include" / "codrel_b200.h",
                                                                      ROOT / "include" / "codrel_dropin.h"]
    objs = []
    for src in LIB_SOURCES:
        s = CSRC / src
        if not s.exists():
            continue
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if _newer(o, [s] + headers):
            cmd = [nvcc()] + NVCC_FLAGS + ["-Xptxas", "-v"] * verbose + ["-c", str(s), "-o", str(o)]
            _run(cmd)
    if _newer(LIB, objs):
        _run([nvcc()] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs] + ["-lcudart", "-lpthread"])
    for name, src in TOOLS.items():
        s = CSRC / src
        if not s.exists():
            continue
        exe = BIN / name
        if _newer(exe, [s, LIB] + headers):
            _run([nvcc()] + NVCC_FLAGS + [str(s), "-o", str(exe), f"-L{PKG}", "-lcodrel_b200",
                  f"-Xlinker", f"-rpath,$ORIGIN/..", "-lcudart"])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
