"""Launch-shape autotuner for the tracer and propagator kernels.

The library compiles each kernel in several launch shapes
(``bh_trace_variant``): threads per block, a ``__launch_bounds__`` minimum of
resident blocks (which caps registers per thread), and rays per thread (two
rays per thread run in the halves of packed float32x2 instructions).  Which
shape is fastest depends on the precision policy, the workload and the GPU,
so the tuner times every shape on a probe of the actual workload with CUDA
events and keeps the fastest.

Results are cached per (GPU name, kernel kind, precision, size bucket) in
memory and in a JSON file (``$BH_AUTOTUNE_CACHE``, default
``~/.cache/blackhorizon_b200/autotune.json``).  Launch shapes change
scheduling only: float64 results are bit-identical across shapes, float32
results can differ in rounding (see the kernels' notes).
"""

from __future__ import annotations

import ctypes
import json
import math
import os
import threading

import torch

from . import _lib
from .backend import ptr, stream_handle

_MEM: dict = {}
_LOCK = threading.Lock()


def cache_path() -> str:
    return os.environ.get("BH_AUTOTUNE_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "blackhorizon_b200", "autotune.json")


def _load_file() -> dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _save_file(data: dict) -> None:
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home only loses the on-disk cache


def variants(precision: str) -> list[dict]:
    """The compiled launch shapes of a precision policy."""
    lib = _lib.load()
    code = _lib.PRECISION[precision]
    out = []
    for i in range(lib.bh_trace_variant_count(code)):
        vals = [ctypes.c_int32() for _ in range(5)]
        _lib.check(lib.bh_trace_variant(code, i, *vals))
        block, minb, rpt, regs, occ = (v.value for v in vals)
        out.append({"variant": i, "block": block, "min_blocks": minb,
                    "rays_per_thread": rpt, "registers": regs, "blocks_per_sm": occ})
    return out


def size_bucket(n: int) -> int:
    return int(math.log2(max(n, 1)))


def _key(kind: str, precision: str, bucket: int, extra: str = "") -> str:
    name = torch.cuda.get_device_name(torch.cuda.current_device()).replace(" ", "_")
    return f"{name}|{kind}|{precision}|{bucket}|{extra}"


def lookup(kind: str, precision: str, n: int, extra: str = ""):
    key = _key(kind, precision, size_bucket(n), extra)
    with _LOCK:
        if key in _MEM:
            return _MEM[key]
        disk = _load_file()
        if key in disk:
            _MEM[key] = disk[key]
            return disk[key]
    return None


def store(kind: str, precision: str, n: int, result: dict, extra: str = "") -> None:
    key = _key(kind, precision, size_bucket(n), extra)
    with _LOCK:
        _MEM[key] = result
        disk = _load_file()
        disk[key] = result
        _save_file(disk)


def time_candidates(run, candidates, reps: int = 3) -> list[tuple[float, dict]]:
    """Milliseconds of run(candidate) for each candidate (best of `reps`
    after one untimed run), fastest first."""
    timings = []
    for cand in candidates:
        run(cand)
        best = math.inf
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            run(cand)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        timings.append((best, cand))
    timings.sort(key=lambda t: t[0])
    return timings


def tune_propagate(state0, spins, precision: str, n_steps: int = 200,
                   rtol: float = 1e-8, atol: float = 1e-10, mass: float = 1.0,
                   spin: float = 0.0, max_step: float = 2.0,
                   initial_step: float = 0.1, force: bool = False) -> dict:
    """Fastest launch shape of bh_propagate on (n, 8) device states."""
    from .integrators import make_config

    n = state0.shape[0]
    if not force:
        hit = lookup("propagate", precision, n)
        if hit is not None:
            return hit
    lib = _lib.load()
    work = torch.empty_like(state0)
    h = torch.empty(n, dtype=torch.float64, device=state0.device)
    acc = torch.empty(n, dtype=torch.int64, device=state0.device)
    ws = torch.empty(lib.bh_trace_workspace_bytes(), dtype=torch.uint8, device=state0.device)

    def run(cand):
        work.copy_(state0)
        h.fill_(initial_step)
        cfg = make_config(1, rtol, atol, initial_step, max_step, 0.0, precision, "aos",
                          600.0, cand["variant"], cand.get("blocks_per_sm_cap", 0))
        _lib.check(lib.bh_propagate(cfg, mass, spin, ptr(spins), ptr(work), ptr(h), None,
                                    ptr(acc), n, n_steps, ptr(ws), stream_handle()),
                   "autotune propagate")

    timings = time_candidates(run, variants(precision))
    best_ms, best = timings[0]
    result = {"variant": best["variant"], "blocks_per_sm": 0, "ms": best_ms,
              "probe": f"{n} rays x {n_steps} steps",
              "table": [{"variant": c["variant"], "ms": round(t, 4)} for t, c in timings]}
    store("propagate", precision, n, result)
    return result


def tune_trace(spacetime, state0, escape_radius: float, precision: str,
               max_steps: int = 20000, rtol: float = 1e-9, atol: float = 1e-12,
               capture_margin: float = 1e-3, max_step: float = 2.0,
               sample: int = 1 << 18, force: bool = False) -> dict:
    """Fastest launch shape of bh_trace, timed on an evenly strided sample of
    up to `sample` rays of the workload."""
    from .integrators import make_config

    n = state0.shape[0]
    extra = f"rtol={rtol:.1e}"
    if not force:
        hit = lookup("trace", precision, n, extra)
        if hit is not None:
            return hit
    lib = _lib.load()
    stride = max(1, n // sample)
    probe = state0[::stride].contiguous()
    m = probe.shape[0]
    out = torch.empty_like(probe)
    status = torch.empty(m, dtype=torch.int32, device=probe.device)
    steps = torch.empty(m, dtype=torch.int64, device=probe.device)
    ws = torch.empty(lib.bh_trace_workspace_bytes(), dtype=torch.uint8, device=probe.device)
    scene = _lib.Scene(spacetime.mass, spacetime.spin,
                       spacetime.capture_radius(capture_margin), float(escape_radius))

    def run(cand):
        cfg = make_config(max_steps, rtol, atol, 0.1, max_step, 1e-10, precision, "aos",
                          600.0, cand["variant"], 0)
        _lib.check(lib.bh_trace(cfg, scene, ptr(probe), ptr(out), ptr(status), ptr(steps),
                                m, ptr(ws), stream_handle()), "autotune trace")

    timings = time_candidates(run, variants(precision))
    best_ms, best = timings[0]
    result = {"variant": best["variant"], "blocks_per_sm": 0, "ms": best_ms,
              "probe": f"{m} of {n} rays",
              "table": [{"variant": c["variant"], "ms": round(t, 4)} for t, c in timings]}
    store("trace", precision, n, result, extra)
    return result


def tune_trace_policy(spacetime, state0, escape_radius: float, max_steps: int = 20000,
                      rtol: float = 1e-9, atol: float = 1e-12, capture_margin: float = 1e-3,
                      max_step: float = 2.0, sample: int = 1 << 18, force: bool = False) -> dict:
    """Precision policy and launch shape with the shortest trace time on a
    probe of the workload.  Both policies classify rays alike; which is
    faster depends on the tolerance: float32 stage arithmetic costs half as
    much per step, but its rounding noise in the embedded error estimate
    forces smaller steps as rtol tightens (near rtol 1e-9 the float64 kernel
    needs fewer, costlier steps and finishes first)."""
    n = state0.shape[0]
    extra = f"rtol={rtol:.1e}"
    if not force:
        hit = lookup("trace-policy", "auto", n, extra)
        if hit is not None:
            return hit
    best = None
    table = {}
    for prec in ("mixed", "fp64"):
        r = tune_trace(spacetime, state0, escape_radius, prec, max_steps, rtol, atol,
                       capture_margin, max_step, sample, force)
        table[prec] = {"variant": r["variant"], "ms": r["ms"]}
        if best is None or r["ms"] < best["ms"]:
            best = {"precision": prec, "variant": r["variant"], "ms": r["ms"]}
    best["table"] = table
    store("trace-policy", "auto", n, best, extra)
    return best
