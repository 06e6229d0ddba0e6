"""Checker for the parity tests: ctypes access to the C restatement of the
reference's algorithms (oracle/dd_oracle.c) and to the reference's own tool
built from its sources (oracle/_ref/ref_codrel).

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline / reference legs may import this package, and only as the checker
or the timed CPU baseline; the product never does.
"""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

from .build import LIB, REF_OUT, build_oracle, build_reference

MAXB = 64
_u64p = C.POINTER(C.c_uint64)
_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build_oracle()
        L = C.CDLL(str(LIB))
        u32, u64, i32, dbl = C.c_uint32, C.c_uint64, C.c_int, C.c_double
        L.dd_oracle_an_exhaustive.argtypes = [u64, u32, _u64p, u32]
        L.dd_oracle_an_rows.argtypes = [u64, u32, u64, u64, _u64p, u32]
        L.dd_oracle_an_grid1d.argtypes = [u64, u32, u32, u64, _u64p, u32, _u64p]
        L.dd_oracle_an_grid2d.argtypes = [u64, u32, u64, u64, _u64p, u32]
        L.dd_oracle_an_grid2d.restype = u64
        L.dd_oracle_an_low_distance.argtypes = [u64, u32, u32, _u64p, _u64p]
        L.dd_oracle_grid1d_points.argtypes = [u64, u32, u32, u64]
        L.dd_oracle_grid1d_points.restype = u64
        L.dd_oracle_grid2d_points.argtypes = [u64, u32, u64]
        L.dd_oracle_grid2d_points.restype = u64
        L.dd_oracle_an_mc.argtypes = [u64, u32, u64, u64, _u64p, u32]
        L.dd_oracle_hamming_weights.argtypes = [u32, _u64p, u32]
        L.dd_oracle_hamming_pairs.argtypes = [u32, i32, _u64p, u32]
        L.dd_oracle_hamming_pairs_distinct.argtypes = [u32, i32, _u64p, u32]
        L.dd_oracle_hamming_grid.argtypes = [u32, u64, _u64p, u32, _u64p]
        L.dd_oracle_hamming_mc.argtypes = [u32, u64, u64, _u64p, u32, _u64p]
        L.dd_oracle_philox.argtypes = [C.POINTER(u32), C.POINTER(u32), C.POINTER(u32)]
        L.dd_oracle_mc_index.argtypes = [u64, u64, u64, u32]
        L.dd_oracle_mc_index.restype = u64
        L.dd_oracle_hamming_cw_ext.argtypes = [u64, u32]
        L.dd_oracle_hamming_cw_ext.restype = u64
        L.dd_oracle_hamming_cw_gpu.argtypes = [u64, u32, i32]
        L.dd_oracle_hamming_cw_gpu.restype = u64
        L.dd_oracle_h_ceil.argtypes = [u64]
        L.dd_oracle_h_ceil.restype = u32
        L.dd_oracle_h_floor1.argtypes = [u64]
        L.dd_oracle_h_floor1.restype = u32
        L.dd_oracle_hamming_h.argtypes = [u32]
        L.dd_oracle_hamming_h.restype = u32
        for f in ("dd_oracle_post_an_exhaustive",):
            getattr(L, f).argtypes = [u32, _u64p, u32, _u64p, _u64p]
        L.dd_oracle_post_an_grid.argtypes = [i32, u32, u64, u64, _u64p, u32, _u64p, _u64p]
        L.dd_oracle_post_an_mc.argtypes = [u32, u64, _u64p, u32, _u64p, _u64p]
        L.dd_oracle_post_hamming_weights.argtypes = [u32, i32, _u64p, u32, _u64p, _u64p]
        L.dd_oracle_post_hamming_sampled.argtypes = [i32, u32, i32, u64, _u64p, u32, _u64p, _u64p]
        L.dd_oracle_num_threads.restype = i32
        L.dd_oracle_naf_min.argtypes = [u64, u32, u32]
        L.dd_oracle_naf_min.restype = u32
        L.dd_oracle_an_candidates.argtypes = [u32, u32, _u64p, u64, C.POINTER(u32)]
        L.dd_oracle_an_candidates.restype = u64
        _lib = L
    return _lib


def _buf(n=MAXB):
    return (C.c_uint64 * n)()


def _u128(lo, hi, nb):
    return [(hi[i] << 64) | lo[i] for i in range(nb)]


def h_ceil(A: int) -> int:
    return lib().dd_oracle_h_ceil(A)


def h_floor1(A: int) -> int:
    return lib().dd_oracle_h_floor1(A)


def hamming_h(n: int) -> int:
    return lib().dd_oracle_hamming_h(n)


def an_exhaustive_raw(A: int, n: int, nbins: int) -> list[int]:
    b = _buf()
    lib().dd_oracle_an_exhaustive(A, n, b, nbins)
    return list(b[:nbins])


def an_rows_raw(A: int, n: int, r0: int, r1: int, nbins: int) -> list[int]:
    b = _buf()
    lib().dd_oracle_an_rows(A, n, r0, r1, b, nbins)
    return list(b[:nbins])


def an_exhaustive_counts(A: int, n: int, nbins: int) -> list[int]:
    raw = an_exhaustive_raw(A, n, nbins)
    lo, hi = _buf(), _buf()
    lib().dd_oracle_post_an_exhaustive(n, (C.c_uint64 * MAXB)(*raw), nbins, lo, hi)
    return _u128(lo, hi, nbins)


def an_grid1d_raw(A: int, n: int, h: int, m: int, nbins: int) -> tuple[list[int], int]:
    b, k = _buf(), (C.c_uint64 * 1)()
    lib().dd_oracle_an_grid1d(A, n, h, m, b, nbins, k)
    return list(b[:nbins]), k[0]


def an_low_distance(A: int, n: int, bits: int) -> tuple[int, int]:
    """Unordered pairs at distance 1 and 2 by bit-flip membership tests."""
    d1, d2 = (C.c_uint64 * 1)(), (C.c_uint64 * 1)()
    lib().dd_oracle_an_low_distance(A, n, bits, d1, d2)
    return d1[0], d2[0]


def grid1d_points(A: int, n: int, h: int, m: int) -> int:
    return lib().dd_oracle_grid1d_points(A, n, h, m)


def grid2d_points(A: int, n: int, m: int) -> int:
    return lib().dd_oracle_grid2d_points(A, n, m)


def an_grid2d_raw(A: int, n: int, m: int, m2: int, nbins: int, with_bin0: bool = False) -> list[int]:
    """The reference's raw 2-D grid histogram (bin 0 left at 0), or with
    with_bin0 the device histogram of every pair (bin 0 = coincident points)."""
    b = _buf()
    zero = lib().dd_oracle_an_grid2d(A, n, m, m2, b, nbins)
    out = list(b[:nbins])
    if with_bin0:
        out[0] = zero
    return out


def an_grid_counts(gdim: int, n: int, m: int, m2: int, raw: list[int]) -> list[int]:
    lo, hi = _buf(), _buf()
    lib().dd_oracle_post_an_grid(gdim, n, m, m2, (C.c_uint64 * MAXB)(*raw), len(raw), lo, hi)
    return _u128(lo, hi, len(raw))


def an_mc_raw(A: int, n: int, it: int, seed: int, nbins: int) -> list[int]:
    b = _buf()
    lib().dd_oracle_an_mc(A, n, it, seed, b, nbins)
    return list(b[:nbins])


def an_mc_counts(n: int, it: int, raw: list[int]) -> list[int]:
    lo, hi = _buf(), _buf()
    lib().dd_oracle_post_an_mc(n, it, (C.c_uint64 * MAXB)(*raw), len(raw), lo, hi)
    return _u128(lo, hi, len(raw))


def hamming_weights_raw(n: int, nbins: int) -> list[int]:
    b = _buf()
    lib().dd_oracle_hamming_weights(n, b, nbins)
    return list(b[:nbins])


def hamming_weights_counts(n: int, with_1bit: int, raw: list[int]) -> list[int]:
    lo, hi = _buf(), _buf()
    lib().dd_oracle_post_hamming_weights(n, with_1bit, (C.c_uint64 * MAXB)(*raw), len(raw), lo, hi)
    return _u128(lo, hi, len(raw))


def hamming_pairs_raw(n: int, with_1bit: int, nbins: int) -> list[int]:
    """Ordered pairs incl. the diagonal (+ spheres): the final counts of `-e 2`."""
    b = _buf()
    lib().dd_oracle_hamming_pairs(n, with_1bit, b, nbins)
    return list(b[:nbins])


def hamming_pairs_distinct_raw(n: int, with_1bit: int, nbins: int) -> list[int]:
    """Pairs a<b (+ spheres of b), doubled: the final counts of `-e 3`."""
    b = _buf()
    lib().dd_oracle_hamming_pairs_distinct(n, with_1bit, b, nbins)
    return list(b[:nbins])


def hamming_grid_raw(n: int, m: int, nbins: int) -> tuple[list[int], int]:
    b, s = _buf(), (C.c_uint64 * 1)()
    lib().dd_oracle_hamming_grid(n, m, b, nbins, s)
    return list(b[:nbins]), s[0]


def hamming_mc_raw(n: int, m: int, seed: int, nbins: int) -> tuple[list[int], int]:
    b, s = _buf(), (C.c_uint64 * 1)()
    lib().dd_oracle_hamming_mc(n, m, seed, b, nbins, s)
    return list(b[:nbins]), s[0]


def hamming_sampled_counts(is_mc: int, n: int, with_1bit: int, m: int, raw: list[int]) -> list[int]:
    lo, hi = _buf(), _buf()
    lib().dd_oracle_post_hamming_sampled(is_mc, n, with_1bit, m, (C.c_uint64 * MAXB)(*raw), len(raw), lo, hi)
    return _u128(lo, hi, len(raw))


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().dd_oracle_philox(c, k, o)
    return tuple(o)


def mc_index(seed: int, idx: int, t: int, n: int) -> int:
    return lib().dd_oracle_mc_index(seed, idx, t, n)


def threads() -> int:
    return lib().dd_oracle_num_threads()


def naf_min(A: int, k: int, floor: int = 0) -> int:
    """Smallest signed-digit weight of A*x over x in [1, 2^k) (early exit below floor)."""
    return lib().dd_oracle_naf_min(A, k, floor)


def an_candidates(k: int, a: int) -> tuple[int, list[int]]:
    """(|SDR|, ascending candidates) of one ANcandidates cell."""
    cap = max(1, 1 << max(0, a - 2))
    out = (C.c_uint64 * cap)()
    sdr = C.c_uint32(0)
    n = lib().dd_oracle_an_candidates(k, a, out, cap, C.byref(sdr))
    return sdr.value, list(out[:n])


# -- the reference's own tool --------------------------------------------------------
def ref_available() -> bool:
    return (REF_OUT / "ref_codrel").exists()


def ref_run(args: list[str], cwd: str | None = None, timeout: float = 600) -> str:
    exe = REF_OUT / "ref_codrel"
    if not exe.exists():
        raise FileNotFoundError(exe)
    res = subprocess.run([str(exe)] + args, capture_output=True, text=True, cwd=cwd, timeout=timeout)
    if res.returncode != 0:
        raise RuntimeError(f"ref_codrel {' '.join(args)} failed: {res.stderr[-500:]}")
    return res.stdout


def ref_ancandidates_available() -> bool:
    return (REF_OUT / "ref_ancandidates").exists()


def ref_ancandidates(amin: int, amax: int, dmin: int, dmax: int, timeout: float = 600) -> str:
    """stdout of the reference's ANcandidates tool for the given width ranges."""
    exe = REF_OUT / "ref_ancandidates"
    res = subprocess.run([str(exe), "-a", str(amin), "-A", str(amax), "-d", str(dmin), "-D", str(dmax)],
                         capture_output=True, text=True, timeout=timeout)
    if res.returncode != 0:
        raise RuntimeError(f"ref_ancandidates failed: {res.stderr[-500:]}")
    return res.stdout


def parse_candidates(text: str) -> dict[tuple[int, int], tuple[int, list[int]]]:
    """{(k, a): (|SDR|, sorted candidates)} from ANcandidates' stdout."""
    out = {}
    for line in text.splitlines():
        if not line or line.startswith("#"):
            continue
        f = line.split("\t")
        n, k, a, sdr, cnt = (int(x) for x in f[:5])
        lst = sorted(int(x) for x in f[5].split(",")) if len(f) > 5 and f[5] else []
        assert n == k + a and cnt == len(lst), line
        out[(k, a)] = (sdr, lst)
    return out


_ROW = re.compile(r"^\s*(\d+),\s*([0-9.e+]+),")


def parse_table(text: str) -> list[int]:
    """counts column of a process_result table (rows `i, count, prob, base...`)."""
    out = []
    for line in text.splitlines():
        m = _ROW.match(line)
        if m and '"' not in line:
            i = int(m.group(1))
            if i != len(out):
                break
            out.append(int(float(m.group(2))) if ("e" in m.group(2) or "." in m.group(2)) else int(m.group(2)))
        elif out:
            break
    return out


def ref_total_runtime(text: str) -> float:
    m = re.search(r'"Total Runtime",([0-9.e+-]+),s', text)
    return float(m.group(1)) if m else float("nan")
