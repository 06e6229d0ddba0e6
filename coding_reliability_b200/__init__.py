"""B200-native distance-distribution histograms (AN codes, Extended Hamming).

Python host-side mirror of the C-ABI in include/codrel_b200.h.  The compute
always runs in libcodrel_b200.so on the GPU; there is no Python or CPU
fallback: loading fails loudly if the library is missing, and every call that
needs a device raises when none is present.

The reference's driver names are mirrored by thin functions (run_ancoding,
run_ancoding_grid, run_ancoding_mc, run_hamming, run_hamming_grid,
run_hamming_mc; distance_distribution/src/algorithms.h:20-34) that return the
post-processed uint128 counts[] as Python ints.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import threading
from dataclasses import dataclass, field
from pathlib import Path

__all__ = [
    "CODE_AN", "CODE_EXT_HAMMING", "MODE_EXHAUSTIVE", "MODE_GRID_1D", "MODE_GRID_2D", "MODE_MONTE_CARLO",
    "KERNEL_AUTO", "KERNEL_POPC", "KERNEL_MMA", "HAMMING_WEIGHTS", "HAMMING_ALL_PAIRS", "HAMMING_ALL_PAIRS_DISTINCT",
    "CONV_GPU", "CONV_CPU", "CONV_SUPER_A", "MMA_EPILOGUE_AUTO", "MMA_EPILOGUE_PAIRED",
    "MMA_EPILOGUE_SINGLE", "MAX_BINS", "DDError", "Request", "Result", "Context", "Server",
    "load", "lib_path", "postprocess", "request_plan", "format_result", "request_shape", "philox4x32_10", "device_count",
    "run_ancoding", "run_ancoding_cpu", "run_ancoding_grid", "run_ancoding_mc", "run_hamming",
    "run_hamming_grid", "run_hamming_mc",
]

CODE_AN, CODE_EXT_HAMMING = 0, 1
MODE_EXHAUSTIVE, MODE_GRID_1D, MODE_GRID_2D, MODE_MONTE_CARLO = 0, 1, 2, 3
KERNEL_AUTO, KERNEL_POPC, KERNEL_MMA = 0, 1, 2
HAMMING_WEIGHTS, HAMMING_ALL_PAIRS, HAMMING_ALL_PAIRS_DISTINCT = 0, 1, 2
CONV_GPU, CONV_CPU, CONV_SUPER_A = 0, 1, 2
MMA_EPILOGUE_AUTO, MMA_EPILOGUE_PAIRED, MMA_EPILOGUE_SINGLE = 0, 1, 2
EPILOGUE_NAMES = {0: "none", 1: "paired", 2: "single"}
MAX_BINS = 64

STATUS = {
    0: "ok", 1: "invalid argument", 2: "unsupported", 3: "cuda error", 4: "no device",
    5: "out of memory", 6: "busy", 7: "timeout", 8: "not found", 9: "cancelled",
}

_PKG = Path(__file__).resolve().parent


def lib_path() -> Path:
    return Path(os.environ.get("CODREL_B200_LIB", _PKG / "libcodrel_b200.so"))


class DDError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class _Req(C.Structure):
    _fields_ = [("code", C.c_uint32), ("mode", C.c_uint32), ("A", C.c_uint64), ("n", C.c_uint32),
                ("h", C.c_uint32), ("m", C.c_uint64), ("m2", C.c_uint64), ("seed", C.c_uint64),
                ("with_1bit", C.c_uint32), ("hamming_method", C.c_uint32), ("kernel", C.c_uint32),
                ("convention", C.c_uint32), ("user_tag", C.c_uint64)]


class _Res(C.Structure):
    _fields_ = [("status", C.c_uint32), ("nbins", C.c_uint32), ("h", C.c_uint32), ("kernel_used", C.c_uint32),
                ("A", C.c_uint64), ("iterations", C.c_uint64), ("iterations2", C.c_uint64),
                ("pairs_lo", C.c_uint64), ("pairs_hi", C.c_uint64),
                ("raw", C.c_uint64 * MAX_BINS), ("counts_lo", C.c_uint64 * MAX_BINS),
                ("counts_hi", C.c_uint64 * MAX_BINS), ("minb", C.c_uint64), ("mincb_lo", C.c_uint64),
                ("mincb_hi", C.c_uint64), ("max_rel_error", C.c_double), ("kernel_ms", C.c_double),
                ("total_ms", C.c_double), ("user_tag", C.c_uint64), ("mma_epilogue", C.c_uint32),
                ("reserved", C.c_uint32)]


class _Tuning(C.Structure):
    _fields_ = [("kernel", C.c_uint32), ("hist_mode", C.c_uint32), ("popc_red_pairs_per_s", C.c_double),
                ("popc_ldst_pairs_per_s", C.c_double), ("mma_pairs_per_s", C.c_double),
                ("probe_pairs", C.c_uint64), ("mma_paired_pairs_per_s", C.c_double),
                ("mma_epilogue", C.c_uint32), ("reserved", C.c_uint32)]


class _RedProbe(C.Structure):
    _fields_ = [("warps_per_sm", C.c_uint32), ("pattern", C.c_uint32), ("adds_per_s", C.c_double)]


class _CandRes(C.Structure):
    _fields_ = [("status", C.c_int32), ("k", C.c_uint32), ("a_bits", C.c_uint32), ("sdr", C.c_uint32),
                ("num_A", C.c_uint64), ("num_candidates", C.c_uint64), ("evaluations", C.c_uint64),
                ("kernel_ms", C.c_double),
                ("total_ms", C.c_double)]


class _BatchOpts(C.Structure):
    _fields_ = [("use_graph", C.c_uint32), ("kernel", C.c_uint32), ("ctas_per_sm", C.c_uint32),
                ("reserved", C.c_uint32)]


@dataclass
class Request:
    code: int = CODE_AN
    mode: int = MODE_EXHAUSTIVE
    A: int = 61
    n: int = 8
    h: int = 0
    m: int = 0
    m2: int = 0
    seed: int = 0
    with_1bit: int = 0
    hamming_method: int = HAMMING_WEIGHTS
    kernel: int = KERNEL_AUTO
    convention: int = CONV_GPU
    user_tag: int = 0

    def _c(self) -> _Req:
        return _Req(self.code, self.mode, self.A, self.n, self.h, self.m, self.m2, self.seed, self.with_1bit,
                    self.hamming_method, self.kernel, self.convention, self.user_tag)


@dataclass
class Result:
    nbins: int
    h: int
    A: int
    raw: list[int]
    counts: list[int]
    minb: int
    mincb: int
    max_rel_error: float
    kernel_ms: float
    total_ms: float
    pairs: int
    iterations: int
    iterations2: int
    kernel_used: int
    user_tag: int = 0
    mma_epilogue: int = 0
    _c: object = field(default=None, repr=False)

    @staticmethod
    def _from(r: _Res) -> "Result":
        nb = r.nbins
        return Result(
            nbins=nb, h=r.h, A=r.A, raw=[r.raw[i] for i in range(nb)],
            counts=[(r.counts_hi[i] << 64) | r.counts_lo[i] for i in range(nb)],
            minb=r.minb, mincb=(r.mincb_hi << 64) | r.mincb_lo, max_rel_error=r.max_rel_error,
            kernel_ms=r.kernel_ms, total_ms=r.total_ms, pairs=(r.pairs_hi << 64) | r.pairs_lo,
            iterations=r.iterations, iterations2=r.iterations2, kernel_used=r.kernel_used,
            user_tag=r.user_tag, mma_epilogue=r.mma_epilogue, _c=r)


_lib = None


def load() -> C.CDLL:
    """Loads libcodrel_b200.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    p = lib_path()
    if not p.exists():
        raise RuntimeError(f"{p} is missing: build it with `python -m coding_reliability_b200.build`")
    lib = C.CDLL(str(p))
    vp, i32, u32 = C.c_void_p, C.c_int, C.c_uint32
    lib.dd_version.restype = C.c_char_p
    lib.dd_status_string.restype = C.c_char_p
    lib.dd_last_error.restype = C.c_char_p
    lib.dd_device_count.restype = i32
    lib.dd_context_create.argtypes = [i32, vp, C.POINTER(vp)]
    lib.dd_context_destroy.argtypes = [vp]
    lib.dd_histogram.argtypes = [vp, C.POINTER(_Req), C.POINTER(_Res)]
    lib.dd_histogram_plain.argtypes = [vp, C.POINTER(_Req), C.POINTER(_Res)]
    lib.dd_histogram_part.argtypes = [vp, C.POINTER(_Req), C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64), u32,
                                      C.POINTER(C.c_double)]
    lib.dd_batch_run.argtypes = [vp, C.POINTER(_Req), u32, C.POINTER(_Res), C.POINTER(_BatchOpts)]
    lib.dd_request_shape.argtypes = [C.POINTER(_Req), C.POINTER(u32), C.POINTER(u32), C.POINTER(C.c_uint64)]
    lib.dd_postprocess.argtypes = [C.POINTER(_Req), C.POINTER(C.c_uint64), u32, C.POINTER(_Res)]
    u64p = C.POINTER(C.c_uint64)
    lib.dd_request_plan.argtypes = [C.POINTER(_Req), u64p, u64p, u64p, u64p]
    lib.dd_format_result.argtypes = [C.POINTER(_Req), C.POINTER(_Res), C.c_char_p, C.c_char_p, C.c_size_t,
                                     C.POINTER(C.c_size_t)]
    lib.dd_philox4x32_10.argtypes = [C.POINTER(u32), C.POINTER(u32), C.POINTER(u32)]
    lib.dd_philox4x32_10.restype = None
    lib.dd_measure_popc_peak.argtypes = [vp, C.POINTER(C.c_double)]
    lib.dd_measure_red_peak.argtypes = [vp, C.POINTER(C.c_double)]
    lib.dd_measure_red_sweep.argtypes = [vp, vp, u32, C.POINTER(C.c_uint32)]
    lib.dd_set_wait_timeout.argtypes = [vp, C.c_uint64]
    lib.dd_set_mma_epilogue.argtypes = [vp, u32]
    lib.dd_autotune.argtypes = [vp, C.POINTER(_Tuning)]
    lib.dd_mc_extend.argtypes = [vp, C.POINTER(_Req), C.c_uint64, C.POINTER(C.c_uint64), C.POINTER(_Res)]
    lib.dd_an_candidates.argtypes = [vp, u32, u32, C.POINTER(C.c_uint64), C.c_uint64, C.POINTER(_CandRes)]
    lib.dd_histogram_noalloc.argtypes = [i32, vp, C.POINTER(_Req), u32, C.POINTER(_Res)]
    lib.dd_server_create.argtypes = [i32, C.c_void_p, C.POINTER(vp)]
    lib.dd_server_submit.argtypes = [vp, C.POINTER(_Req), C.POINTER(C.c_uint64)]
    lib.dd_server_poll.argtypes = [vp, C.c_uint64, C.POINTER(_Res), C.POINTER(C.c_int)]
    lib.dd_server_wait.argtypes = [vp, C.c_uint64, C.c_double, C.POINTER(_Res)]
    lib.dd_server_cancel.argtypes = [vp, C.c_uint64]
    lib.dd_server_release.argtypes = [vp, C.c_uint64]
    lib.dd_server_get_stats.argtypes = [vp, C.c_void_p]
    lib.dd_server_shutdown.argtypes = [vp]
    lib.dd_server_destroy.argtypes = [vp]
    _lib = lib
    return lib


def _check(st: int) -> None:
    if st != 0:
        raise DDError(st, load().dd_last_error().decode())


def device_count() -> int:
    return load().dd_device_count()


def request_shape(req: Request) -> tuple[int, int, int]:
    nb, h, a = C.c_uint32(), C.c_uint32(), C.c_uint64()
    _check(load().dd_request_shape(C.byref(req._c()), C.byref(nb), C.byref(h), C.byref(a)))
    return nb.value, h.value, a.value


def request_plan(req: Request) -> dict:
    """Device work a request plans (no device needed): lattice points, tiles, pairs."""
    lat, tiles, lo, hi = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint64()
    _check(load().dd_request_plan(C.byref(req._c()), C.byref(lat), C.byref(tiles), C.byref(lo), C.byref(hi)))
    return {"lattice": lat.value, "tiles": tiles.value, "pairs": (hi.value << 64) | lo.value}


def postprocess(req: Request, raw: list[int]) -> Result:
    """The reference drivers' host post-processing of a raw histogram (no device needed)."""
    arr = (C.c_uint64 * MAX_BINS)(*([int(x) for x in raw] + [0] * (MAX_BINS - len(raw))))
    out = _Res()
    _check(load().dd_postprocess(C.byref(req._c()), arr, MAX_BINS, C.byref(out)))
    return Result._from(out)


def format_result(req: Request, res: Result, device_line: str | None = None) -> str:
    lib = load()
    n = C.c_size_t()
    r = res._c if res._c is not None else _Res()
    dl = device_line.encode() if device_line is not None else None
    _check(lib.dd_format_result(C.byref(req._c()), C.byref(r), dl, None, 0, C.byref(n)))
    buf = C.create_string_buffer(n.value + 1)
    _check(lib.dd_format_result(C.byref(req._c()), C.byref(r), dl, buf, n.value + 1, C.byref(n)))
    return buf.value.decode()


def philox4x32_10(ctr: tuple[int, int, int, int], key: tuple[int, int]) -> tuple[int, int, int, int]:
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    load().dd_philox4x32_10(c, k, o)
    return tuple(o)


def _request_key(req: Request) -> dict:
    return {k: getattr(req, k) for k in ("code", "mode", "A", "n", "h", "m", "m2", "seed", "with_1bit",
                                         "hamming_method", "convention")}


def run_resumable(ctx, req: Request, state_path: str | os.PathLike, chunk_tiles: int = 0) -> Result:
    """One histogram computed in parts with a checkpoint after each: the state
    file holds the request, the next tile and the raw bins so far (JSON, written
    atomically), and a later call with the same request and file resumes where
    the last one stopped.  The file is removed once the result is complete.
    chunk_tiles = 0: about 64 parts.  `ctx` needs `histogram_part`."""
    path = Path(state_path)
    total = request_plan(req)["tiles"]
    nb = request_shape(req)[0]
    key = _request_key(req)
    nxt, raw = 0, [0] * nb
    if path.exists():
        st = json.loads(path.read_text())
        if st.get("request") != key or st.get("tiles") != total:
            raise DDError(1, f"{path}: checkpoint of another request")
        nxt, raw = int(st["next_tile"]), [int(x) for x in st["raw"]]
        if not (0 <= nxt <= total and len(raw) == nb):
            raise DDError(1, f"{path}: damaged checkpoint")
    step = chunk_tiles if chunk_tiles > 0 else max(1, -(-total // 64))
    while nxt < total:
        cnt = min(step, total - nxt)
        raw, _ = ctx.histogram_part(req, nxt, cnt, raw)
        nxt += cnt
        tmp = path.with_name(path.name + ".tmp")
        tmp.write_text(json.dumps({"request": key, "tiles": total, "next_tile": nxt, "raw": raw}))
        os.replace(tmp, path)
    res = postprocess(req, raw)
    res.user_tag = req.user_tag
    if path.exists():
        path.unlink()
    return res


class Context:
    """One device + one CUDA stream (dd_context)."""

    def __init__(self, device: int = 0, stream: int | None = None):
        lib = load()
        h = C.c_void_p()
        _check(lib.dd_context_create(device, C.c_void_p(stream) if stream else None, C.byref(h)))
        self._h = h
        self.device = device

    def close(self) -> None:
        if getattr(self, "_h", None):
            load().dd_context_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def histogram(self, req: Request) -> Result:
        out = _Res()
        _check(load().dd_histogram(self._h, C.byref(req._c()), C.byref(out)))
        return Result._from(out)

    def mc_extend(self, req: Request, it_done: int, raw_done: list[int]) -> Result:
        """dd_mc_extend: `req` (Monte Carlo, req.m samples per codeword) grown
        from an earlier run of it_done samples whose raw bins are raw_done."""
        raw = (C.c_uint64 * 64)(*(list(raw_done) + [0] * (64 - len(raw_done))))
        out = _Res()
        _check(load().dd_mc_extend(self._h, C.byref(req._c()), it_done, raw, C.byref(out)))
        return Result._from(out)

    def histogram_part(self, req: Request, tile_begin: int, tile_count: int,
                       raw: list[int] | None = None) -> tuple[list[int], float]:
        """dd_histogram_part: tiles [tile_begin, tile_begin + tile_count) of the
        request's tile space (request_plan(req)["tiles"]) added to `raw`; returns
        (raw, kernel_ms).  Disjoint parts covering the space sum to the full raw
        histogram; postprocess(req, raw) gives the result."""
        arr = (C.c_uint64 * MAX_BINS)(*([int(x) for x in (raw or [])] + [0] * (MAX_BINS - len(raw or []))))
        ms = C.c_double()
        _check(load().dd_histogram_part(self._h, C.byref(req._c()), tile_begin, tile_count, arr, MAX_BINS,
                                        C.byref(ms)))
        nb = request_shape(req)[0]
        return [int(arr[b]) for b in range(nb)], ms.value

    def histogram_plain(self, req: Request) -> Result:
        """The plain one-launch-per-instance baseline (AN exhaustive only)."""
        out = _Res()
        _check(load().dd_histogram_plain(self._h, C.byref(req._c()), C.byref(out)))
        return Result._from(out)

    def batch(self, reqs: list[Request], use_graph: bool = True, kernel: int = KERNEL_AUTO) -> list[Result]:
        n = len(reqs)
        arr = (_Req * n)(*[r._c() for r in reqs])
        out = (_Res * n)()
        opts = _BatchOpts(1 if use_graph else 0, kernel, 0, 0)
        _check(load().dd_batch_run(self._h, arr, n, out, C.byref(opts)))
        return [Result._from(out[i]) for i in range(n)]

    def autotune(self) -> dict:
        t = _Tuning()
        _check(load().dd_autotune(self._h, C.byref(t)))
        return {"kernel": "mma" if t.kernel == KERNEL_MMA else "popc",
                "hist_mode": "red" if t.hist_mode == 0 else "ldst",
                "mma_epilogue": EPILOGUE_NAMES.get(t.mma_epilogue, str(t.mma_epilogue)),
                "popc_red_pairs_per_s": t.popc_red_pairs_per_s, "popc_ldst_pairs_per_s": t.popc_ldst_pairs_per_s,
                "mma_single_pairs_per_s": t.mma_pairs_per_s, "mma_paired_pairs_per_s": t.mma_paired_pairs_per_s,
                "probe_pairs": t.probe_pairs}

    def set_mma_epilogue(self, epilogue: int) -> None:
        """Epilogue of this context's tcgen05 launches: MMA_EPILOGUE_AUTO (the
        autotuner's choice), MMA_EPILOGUE_PAIRED or MMA_EPILOGUE_SINGLE."""
        _check(load().dd_set_mma_epilogue(self._h, epilogue))

    def popc_peak(self) -> float:
        v = C.c_double()
        _check(load().dd_measure_popc_peak(self._h, C.byref(v)))
        return v.value

    def set_wait_timeout(self, ns: int) -> None:
        """Bound of the tcgen05 kernel's device-side waits (0: the 2 s default)."""
        _check(load().dd_set_wait_timeout(self._h, ns))

    def red_peak(self) -> float:
        """Shared-memory atomic adds per second (the tcgen05 epilogue's bound):
        the maximum of red_sweep()."""
        v = C.c_double()
        _check(load().dd_measure_red_peak(self._h, C.byref(v)))
        return v.value

    def red_sweep(self) -> list[dict]:
        """The shared-memory atomic rate at 8..32 warps per SM for the per-thread
        column pattern (single epilogue) and the shared lane-column pattern
        (paired epilogue)."""
        rows = (_RedProbe * 64)()
        n = C.c_uint32()
        _check(load().dd_measure_red_sweep(self._h, rows, 64, C.byref(n)))
        return [{"warps_per_sm": rows[i].warps_per_sm,
                 "pattern": "per_thread_columns" if rows[i].pattern == 0 else "lane_columns_shared",
                 "adds_per_s": rows[i].adds_per_s} for i in range(n.value)]

    def an_candidates(self, k: int, a_bits: int, capacity: int | None = None) -> tuple[dict, list[int]]:
        """dd_an_candidates: the super-A candidates of (k data bits, A width
        a_bits) as ANcandidates ranks them; returns (summary, ascending A list)."""
        if capacity is None:
            capacity = max(1, 1 << max(0, a_bits - 2)) if a_bits <= 26 else 1 << 24
        buf = (C.c_uint64 * max(1, capacity))()
        r = _CandRes()
        _check(load().dd_an_candidates(self._h, k, a_bits, buf, capacity, C.byref(r)))
        info = {"k": r.k, "a_bits": r.a_bits, "sdr": r.sdr, "num_A": r.num_A, "num_candidates": r.num_candidates,
                "evaluations": r.evaluations, "kernel_ms": r.kernel_ms, "total_ms": r.total_ms}
        return info, list(buf[:min(r.num_candidates, capacity)])


def histogram_noalloc(reqs: list[Request], device: int = 0, stream: int | None = None) -> list[Result]:
    """dd_histogram_noalloc: up to 32 histograms without any device allocation,
    for callers that may not allocate device memory (see include/codrel_b200.h).
    Calls that overlap on the same GPU race on the shared scratch."""
    n = len(reqs)
    arr = (_Req * max(n, 1))(*[r._c() for r in reqs])
    out = (_Res * max(n, 1))()
    _check(load().dd_histogram_noalloc(device, C.c_void_p(stream) if stream else None, arr, n, out))
    return [Result._from(out[i]) for i in range(n)]


class _ServerOpts(C.Structure):
    _fields_ = [("memory_budget_bytes", C.c_uint64), ("max_queue", C.c_uint32), ("round_ms", C.c_uint32),
                ("dry_run", C.c_uint32), ("inject_alloc_failure", C.c_uint32)]


class _ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("admitted", C.c_uint64), ("completed", C.c_uint64),
                ("rejected", C.c_uint64), ("cancelled", C.c_uint64), ("rounds", C.c_uint64),
                ("active", C.c_uint32), ("queued", C.c_uint32), ("slots", C.c_uint32), ("slots_free", C.c_uint32),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("pairs_per_s", C.c_double),
                ("busy_ms", C.c_double), ("pairs_lo", C.c_uint64), ("pairs_hi", C.c_uint64)]


class Server:
    """dd_server: continuous-batching query server on one GPU (dry_run: host logic only)."""

    def __init__(self, device: int = 0, memory_budget_bytes: int = 0, max_queue: int = 0, round_ms: int = 0,
                 dry_run: bool = False, inject_alloc_failure: bool = False):
        lib = load()
        h = C.c_void_p()
        opts = _ServerOpts(memory_budget_bytes, max_queue, round_ms, int(dry_run), int(inject_alloc_failure))
        _check(lib.dd_server_create(device, C.byref(opts), C.byref(h)))
        self._h = h
        # calls in flight: close() frees the server only after they have returned
        self._cv = threading.Condition()
        self._users = 0
        self._closing = False

    def _enter(self):
        with self._cv:
            if self._closing or not self._h:
                raise DDError(9, "server closed")
            self._users += 1
            return self._h

    def _leave(self):
        with self._cv:
            self._users -= 1
            self._cv.notify_all()

    def submit(self, req: Request) -> int:
        t = C.c_uint64()
        h = self._enter()
        try:
            _check(load().dd_server_submit(h, C.byref(req._c()), C.byref(t)))
        finally:
            self._leave()
        return t.value

    def poll(self, ticket: int) -> Result | None:
        out, done = _Res(), C.c_int()
        h = self._enter()
        try:
            _check(load().dd_server_poll(h, ticket, C.byref(out), C.byref(done)))
        finally:
            self._leave()
        return Result._from(out) if done.value else None

    def wait(self, ticket: int, timeout_s: float = -1.0) -> tuple[int, Result]:
        """(status, result): status is the query's dd_status (0 = done; 9 = cancelled,
        also when the server is closed while this call waits)."""
        out = _Res()
        h = self._enter()
        try:
            st = load().dd_server_wait(h, ticket, timeout_s, C.byref(out))
        finally:
            self._leave()
        if st in (7, 8):  # timeout / unknown ticket
            _check(st)
        return st, Result._from(out)

    def cancel(self, ticket: int) -> None:
        h = self._enter()
        try:
            _check(load().dd_server_cancel(h, ticket))
        finally:
            self._leave()

    def release(self, ticket: int) -> None:
        """Drops a finished query's result now (DDError 6 while it runs or is waited on).
        Delivered results are also dropped by themselves once 4096 newer ones were delivered."""
        h = self._enter()
        try:
            _check(load().dd_server_release(h, ticket))
        finally:
            self._leave()

    def stats(self) -> dict:
        s = _ServerStats()
        h = self._enter()
        try:
            _check(load().dd_server_get_stats(h, C.byref(s)))
        finally:
            self._leave()
        d = {k: getattr(s, k) for k, _ in _ServerStats._fields_}
        d["pairs"] = (d.pop("pairs_hi") << 64) | d.pop("pairs_lo")
        return d

    def close(self) -> None:
        """Cancels unfinished queries (their waiters return status 9), waits for the
        calls in flight, then frees the server.  Calls made afterwards raise DDError."""
        cv = getattr(self, "_cv", None)
        if cv is None or not getattr(self, "_h", None):
            return
        with cv:
            if self._closing:
                return
            self._closing = True
        lib = load()
        lib.dd_server_shutdown(self._h)  # wakes every waiter
        with cv:
            cv.wait_for(lambda: self._users == 0)
        lib.dd_server_destroy(self._h)
        self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Context | None = None


def _ctx() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


# -- the reference's driver names -------------------------------------------------
def run_ancoding(n: int, A: int) -> Result:
    """src/an_coding.cu:276 run_ancoding (GPU conventions)."""
    return _ctx().histogram(Request(CODE_AN, MODE_EXHAUSTIVE, A, n, convention=CONV_GPU))


def run_ancoding_cpu(n: int, A: int) -> Result:
    """src/an_coding.cpp:104 run_ancoding_cpu conventions, computed on the GPU."""
    return _ctx().histogram(Request(CODE_AN, MODE_EXHAUSTIVE, A, n, convention=CONV_CPU))


def run_ancoding_grid(gdim: int, n: int, m: int, m2: int, A: int) -> Result:
    """src/an_coding_grid.cu:215 run_ancoding_grid."""
    return _ctx().histogram(Request(CODE_AN, MODE_GRID_2D if gdim == 2 else MODE_GRID_1D, A, n, m=m, m2=m2))


def run_ancoding_mc(n: int, m: int, A: int, seed: int = 16384) -> Result:
    """src/an_coding_mc.cu:205 run_ancoding_mc (Philox draws)."""
    return _ctx().histogram(Request(CODE_AN, MODE_MONTE_CARLO, A, n, m=m, seed=seed))


def run_hamming(n: int, with_1bit: int = 0, method: int = HAMMING_WEIGHTS) -> Result:
    """src/hamming.cu:97 run_hamming (`-e 1`) or the all-pairs brute force (`-e 2/3/4`)."""
    return _ctx().histogram(Request(CODE_EXT_HAMMING, MODE_EXHAUSTIVE, 1, n, with_1bit=with_1bit,
                                    hamming_method=method))


def run_hamming_grid(n: int, with_1bit: int, m: int) -> Result:
    """src/hamming_grid.cu:91 run_hamming_grid."""
    return _ctx().histogram(Request(CODE_EXT_HAMMING, MODE_GRID_1D, 1, n, m=m, with_1bit=with_1bit))


def run_hamming_mc(n: int, with_1bit: int, m: int, seed: int = 1337) -> Result:
    """src/hamming_mc.cu:98 run_hamming_mc (Philox draws)."""
    return _ctx().histogram(Request(CODE_EXT_HAMMING, MODE_MONTE_CARLO, 1, n, m=m, seed=seed,
                                    with_1bit=with_1bit))
