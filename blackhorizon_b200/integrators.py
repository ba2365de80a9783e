"""Batched integrators, b200 backend.

Same signatures as blackhorizon/integrators.py: ``rk4_step``,
``dormand_prince_step``, ``error_ratio``, ``step_factor`` and
``integrate_dense``, each a CUDA kernel.  The RHS argument must be a
``GeodesicRhs`` (or ``functools.partial(geodesic_rhs, spacetime)``);
any other callable raises TypeError because there is no CPU path.

``propagate`` is the no-termination mode of the tracer loop (tracer.py:111-120
without the status cascade): every ray makes exactly ``n_steps`` attempted
DP5(4) steps with its own adaptive step size, optionally with one spin per
ray.  It is the raw-throughput benchmark workload.
"""

from __future__ import annotations

import numpy
import torch

from . import _lib
from .backend import Array, is_device_array, out_like, ptr, stream_handle, to_device_f64
from .geodesics import spacetime_of_rhs

PRECISIONS = ("fp64", "mixed")


def _precision_code(precision: str) -> int:
    try:
        return _lib.PRECISION[precision]
    except KeyError:
        raise ValueError(f"precision must be one of {PRECISIONS}") from None


def _h_vector(h, n, device):
    if is_device_array(h):
        t = h.to(device=device, dtype=torch.float64)
    else:
        t = torch.as_tensor(numpy.asarray(h, dtype=numpy.float64), device=device)
    if t.dim() == 0:
        t = t.expand(n)
    if t.shape != (n,):
        raise ValueError("h must be a scalar or have shape (n,)")
    return t.contiguous()


def rk4_step(rhs, state: Array, h: Array, precision: str = "fp64",
             n_steps: int = 1) -> Array:
    """Classical RK4 (integrators.py:57-73); ``n_steps`` > 1 repeats it in
    registers without leaving the kernel."""
    st = spacetime_of_rhs(rhs)
    s, host = to_device_f64(state, "state")
    if s.dim() != 2 or s.shape[1] != 8:
        raise ValueError("state must have shape (n, 8)")
    hh = _h_vector(h, s.shape[0], s.device)
    out = torch.empty_like(s)
    _lib.check(_lib.load().bh_rk4(st.mass, st.spin, ptr(s), ptr(hh), ptr(out),
                                  s.shape[0], int(n_steps), _precision_code(precision),
                                  stream_handle()), "rk4_step")
    return out_like(out, host, state)


def implicit_midpoint_step(rhs, state: Array, h: Array, iterations: int = 4,
                           n_steps: int = 1) -> Array:
    """One implicit midpoint step (integrators.py:177-207), symplectic for
    the Hamiltonian flow: y1 = y0 + h f((y0 + y1) / 2), solved by
    ``iterations`` fixed-point refinements seeded with an explicit Euler
    half step; float64.  ``n_steps`` > 1 repeats it in registers."""
    st = spacetime_of_rhs(rhs)
    s, host = to_device_f64(state, "state")
    if s.dim() != 2 or s.shape[1] != 8:
        raise ValueError("state must have shape (n, 8)")
    hh = _h_vector(h, s.shape[0], s.device)
    out = torch.empty_like(s)
    _lib.check(_lib.load().bh_implicit_midpoint(st.mass, st.spin, ptr(s), ptr(hh), ptr(out),
                                                s.shape[0], int(iterations), int(n_steps),
                                                stream_handle()), "implicit_midpoint_step")
    return out_like(out, host, state)


def dormand_prince_step(rhs, state: Array, h: Array, precision: str = "fp64"):
    """Embedded Dormand-Prince 5(4) step (integrators.py:76-107): returns
    (new_state, error)."""
    st = spacetime_of_rhs(rhs)
    s, host = to_device_f64(state, "state")
    if s.dim() != 2 or s.shape[1] != 8:
        raise ValueError("state must have shape (n, 8)")
    hh = _h_vector(h, s.shape[0], s.device)
    new = torch.empty_like(s)
    err = torch.empty_like(s)
    _lib.check(_lib.load().bh_dp5_step(st.mass, st.spin, ptr(s), ptr(hh), ptr(new),
                                       ptr(err), s.shape[0], _precision_code(precision),
                                       stream_handle()), "dormand_prince_step")
    return out_like(new, host, state), out_like(err, host, state)


def error_ratio(state: Array, new_state: Array, error: Array, rtol: float,
                atol: float) -> Array:
    """Scaled RMS error per sample (integrators.py:110-117)."""
    s, host = to_device_f64(state, "state")
    sn, _ = to_device_f64(new_state, "new_state")
    e, _ = to_device_f64(error, "error")
    if s.dim() != 2 or s.shape[1] != 8 or sn.shape != s.shape or e.shape != s.shape:
        raise ValueError("state, new_state and error must have shape (n, 8)")
    out = torch.empty(s.shape[0], dtype=torch.float64, device=s.device)
    _lib.check(_lib.load().bh_error_ratio(ptr(s), ptr(sn), ptr(e), float(rtol),
                                          float(atol), ptr(out), s.shape[0],
                                          stream_handle()), "error_ratio")
    return out_like(out, host, state)


def step_factor(ratio: Array) -> Array:
    """clip(0.9 max(ratio, 1e-16)^-0.2, 0.2, 5) (integrators.py:120-124)."""
    r, host = to_device_f64(ratio, "ratio")
    flat = r.reshape(-1).contiguous()
    out = torch.empty_like(flat)
    _lib.check(_lib.load().bh_step_factor(ptr(flat), ptr(out), flat.shape[0],
                                          stream_handle()), "step_factor")
    return out_like(out.reshape(r.shape), host, ratio)


def integrate_dense(rhs, state0: Array, lambda_total: float, rtol: float = 1e-10,
                    atol: float = 1e-12, initial_step: float = 0.05,
                    max_step: float = 2.0, precision: str = "fp64") -> list:
    """Lock-step adaptive integration with one step size for the batch
    (integrators.py:127-174): returns the list of accepted states."""
    st = spacetime_of_rhs(rhs)
    s, host = to_device_f64(state0, "state0")
    n = s.shape[0]
    state = s.clone()
    states = [state.clone()]
    elapsed = 0.0
    h_scalar = float(initial_step)
    while elapsed < lambda_total:
        h_scalar = min(h_scalar, max_step, lambda_total - elapsed)
        h = torch.full((n,), h_scalar, dtype=torch.float64, device=s.device)
        new_state, error = dormand_prince_step(rhs, state, h, precision)
        ratio = float(error_ratio(state, new_state, error, rtol, atol).max())
        if ratio <= 1.0:
            state = new_state
            states.append(state.clone())
            elapsed += h_scalar
        factor = float(min(max(0.9 * max(ratio, 1e-16) ** (-0.2), 0.2), 5.0))
        h_scalar *= factor
        if h_scalar < 1e-14:
            raise RuntimeError("integrate_dense: step size underflow")
    del st
    return [out_like(x, host, state0) for x in states]


def make_config(max_steps: int = 1, rtol: float = 1e-9, atol: float = 1e-12,
                initial_step: float = 0.1, max_step: float = 2.0,
                min_step: float = 1e-10, precision: str = "fp64",
                layout: str = "aos", timeout_s: float = 0.0, variant: int = -1,
                blocks_per_sm: int = 0, project_every: int = 0,
                flags: int = 0, f64_radius: float | str = 0.0) -> "_lib.TraceConfig":
    """The C ABI's bh_trace_config.  ``f64_radius`` (propagate, mixed
    policy): radius in units of M of the float64 band, ``"auto"`` for
    8 u M / rtol (u = 2^-24), 0 for none."""
    if layout not in _lib.LAYOUT:
        raise ValueError("layout must be 'aos' or 'soa'")
    if int(project_every) < 0:
        raise ValueError("project_every must be >= 0")
    return _lib.TraceConfig(
        int(max_steps), float(rtol), float(atol), float(initial_step),
        float(max_step), float(min_step), _precision_code(precision),
        _lib.LAYOUT[layout], int(max(0.0, timeout_s) * 1e9), int(variant),
        int(blocks_per_sm), int(project_every), int(flags), 0, _band_radius(f64_radius))


def _band_radius(f64_radius) -> float:
    if isinstance(f64_radius, str):
        if f64_radius != "auto":
            raise ValueError("f64_radius must be a radius >= 0 or 'auto'")
        return -1.0
    r = float(f64_radius)
    if not r >= 0.0:
        raise ValueError("f64_radius must be a radius >= 0 or 'auto'")
    return r


def propagate(spacetime, state0: Array, n_steps: int, rtol: float = 1e-8,
              atol: float = 1e-10, initial_step: float = 0.1,
              max_step: float = 2.0, precision: str = "fp64", spins=None,
              h0: Array | None = None, layout: str = "aos",
              timeout_s: float = 0.0, variant: int = -1, workspace=None,
              in_place: bool = False, project_every: int = 0, out=None,
              chunks: int = 3, f64_radius: float | str = "auto", order_rays=None):
    """n_steps attempted DP5(4) steps per ray with per-ray accept/reject and
    step update (tracer.py:111-120), no termination.

    Mixed policy: the stage arithmetic runs in float32 except in the float64
    band: while a ray of a warp lies between the outer horizon and
    ``f64_radius`` (units of M), the warp's attempt runs in float64 (with the
    default launch shape).  The default ``"auto"`` puts the band's edge at
    8 u M / rtol (u = 2^-24), where float32 rounding of the curvature terms
    reaches the tolerance; 0 runs float32 stages everywhere.  Ignored by the
    float64 policy and, under ``"auto"``, by projecting calls.

    ``order_rays`` (default: on whenever the band is): the launch takes the
    rays of each segment of ORDER_SEGMENT consecutive rays inward-moving
    first, by impact parameter (bh_propagate_order), so that rays passing the
    hole alike share warps and fewer warps need the band; results come back
    in the caller's order.  Off (and for launches of more than 2^31 - 1
    rays, whose indices the order cannot hold), a warp holds rays
    [64 k, 64 k + 64) of the call.

    Returns (states, h, lam, accepted, stats): ``lam`` is the affine
    parameter each ray advanced (sum of its accepted step sizes, float64).
    ``spins`` (n,) gives each ray its own spin.  With ``in_place`` and a
    device float64 ``state0`` the states are advanced in place.
    ``project_every`` K > 0 projects every ray onto the null constraint in
    float64 after every K-th attempt (not in the reference; off by default).

    Streaming from host memory: with ``state0`` (and ``spins``, if given) a
    float64 CPU tensor in pinned memory and ``out`` a pinned (n, 8) float64
    CPU tensor, the rays go through in ``chunks`` contiguous pieces on
    separate CUDA streams, each piece's host-to-device copy, kernel and
    device-to-host copy of its final states overlapping the other pieces'
    work.  With three or more pieces the first and the last hold n/16 rays,
    so that little copy time stays exposed at either end.  The final
    states land in ``out`` (returned); h, lam and accepted stay on the device,
    as every result of a call with torch input does (only NumPy input gets
    NumPy results back).  The stats sum the pieces' counters.  Results equal
    the single-launch path's."""
    if out is not None:
        if h0 is not None or layout != "aos" or in_place:
            raise ValueError("streaming from host memory takes neither h0, layout 'soa' "
                             "nor in_place")
        return _propagate_streamed(spacetime, state0, n_steps, rtol, atol, initial_step,
                                   max_step, precision, spins, timeout_s, variant,
                                   project_every, out, chunks, f64_radius, order_rays)
    s, host = to_device_f64(state0, "state0")
    n = s.shape[0] if layout == "aos" else s.shape[-1]
    if layout == "aos" and (s.dim() != 2 or s.shape[1] != 8):
        raise ValueError("state0 must have shape (n, 8)")
    if layout == "soa" and (s.dim() != 2 or s.shape[0] != 8):
        raise ValueError("state0 must have shape (8, n) for layout 'soa'")
    states = s if (in_place and host is None and s.data_ptr() == state0.data_ptr()) else s.clone()
    if h0 is None:
        h = torch.full((n,), float(initial_step), dtype=torch.float64, device=s.device)
    else:
        h = _h_vector(h0, n, s.device).clone()
    spin_t = None
    if spins is not None:
        spin_t, _ = to_device_f64(spins, "spins")
        if spin_t.shape != (n,):
            raise ValueError("spins must have shape (n,)")
        if bool((spin_t.abs() > spacetime.mass).any()):
            raise ValueError("Kerr bound violated: |spin| must be <= mass")
    acc = torch.empty(n, dtype=torch.int64, device=s.device)
    lam = torch.zeros(n, dtype=torch.float64, device=s.device)
    lib = _lib.load()
    if variant == "auto":
        from .autotune import tune_propagate

        variant = -1
        if n and layout == "aos":
            variant = tune_propagate(s, spin_t, precision, min(int(n_steps), 200), rtol, atol,
                                     float(spacetime.mass), float(spacetime.spin), max_step,
                                     initial_step)["variant"]
    ws = workspace if workspace is not None else torch.empty(
        lib.bh_trace_workspace_bytes(), dtype=torch.uint8, device=s.device)
    band = _propagate_band(f64_radius, precision, project_every)
    cfg = make_config(1, rtol, atol, initial_step, max_step, 0.0, precision,
                      layout, timeout_s, variant, 0, project_every, f64_radius=band)
    stream = stream_handle()
    order = _ray_order(lib, states, layout, n, order_rays, band) if n else None
    _lib.check(lib.bh_propagate_ordered(cfg, float(spacetime.mass), float(spacetime.spin),
                                        ptr(spin_t), ptr(states), ptr(h), ptr(lam), ptr(acc),
                                        ptr(order), n, int(n_steps), ptr(ws), stream),
               "propagate")
    stats = _lib.TraceStats()
    _lib.check(lib.bh_trace_stats_read(ptr(ws), stats, stream), "propagate")
    return (out_like(states, host, state0), out_like(h, host, state0),
            out_like(lam, host, state0),
            acc.cpu().numpy() if host is not None else acc, stats)


# Rays per segment of bh_propagate_order (include/bh_b200.h): the launch order
# stays within each segment.
ORDER_SEGMENT = 16384


def _ray_order(lib, states, layout: str, n: int, order_rays, band, buffers=None):
    """The launch order of a propagate call's rays (an int32 device tensor),
    or None for the rays' own order.  order_rays None orders whenever the
    float64 band is on.  buffers: (order, workspace) allocated by the caller
    (_order_buffers), else allocated here on the current stream."""
    if order_rays is None:
        order_rays = band != 0.0
    # The order holds int32 ray indices: larger launches take the rays as given.
    if not order_rays or n > _INT32_MAX:
        return None
    order, ws = buffers if buffers is not None else _order_buffers(lib, n, states.device)
    _lib.check(lib.bh_propagate_order(ptr(states), _lib.LAYOUT[layout], n, ptr(order), ptr(ws),
                                      ws.numel(), stream_handle()), "propagate order")
    return order


_INT32_MAX = 2**31 - 1


def _order_buffers(lib, n: int, device):
    """An order array and bh_propagate_order's workspace for n rays (None
    beyond the int32 range, where the launch takes the rays as given)."""
    if n > _INT32_MAX:
        return None
    return (torch.empty(n, dtype=torch.int32, device=device),
            torch.empty(lib.bh_propagate_order_workspace_bytes(n), dtype=torch.uint8,
                        device=device))


# Side streams per device for the streamed path, kept for the process: the
# caching allocator keeps freed blocks per stream, and streams made afresh on
# every call kept missing that cache.
_SIDE_STREAMS: dict = {}


def _side_streams(dev):
    key = dev.index if dev.index is not None else torch.cuda.current_device()
    if key not in _SIDE_STREAMS:
        _SIDE_STREAMS[key] = [torch.cuda.Stream(dev) for _ in range(3)]
    return _SIDE_STREAMS[key]


def _pieces(n: int, k: int, align: int):
    """[a, b) bounds of the streamed path's k pieces, starting at multiples of
    align.  With k >= 3 the first and last pieces hold about n/16 rays: only
    their copies stay exposed, the first's input and the last's output (on
    the headline workload three pieces of 1/16, 7/8 and 1/16 took 60.6 ms, two
    halves 62.2 ms, one piece 61.6 ms)."""
    k = max(1, min(int(k), n))
    if k >= 3:
        edge = max(align, (n // 16) // align * align)
        last = (n - edge) // align * align
        if edge < last:
            inner = [edge + (last - edge) * c // (k - 2) // align * align for c in range(k - 2)]
            cuts = [0] + inner + [last, n]
            return [(a, b) for a, b in zip(cuts[:-1], cuts[1:]) if b > a]
        k = 2
    cuts = [min(n, (n * c // k + align - 1) // align * align) for c in range(k)] + [n]
    return [(a, b) for a, b in zip(cuts[:-1], cuts[1:]) if b > a]


def _propagate_band(f64_radius, precision: str, project_every: int):
    """The band radius a propagate call passes: none for the float64 policy
    and none by default under projection (the two do not combine)."""
    if precision != "mixed" or (int(project_every) > 0 and f64_radius == "auto"):
        return 0.0
    return f64_radius


def _propagate_streamed(spacetime, state0, n_steps, rtol, atol, initial_step, max_step,
                        precision, spins, timeout_s, variant, project_every, out, chunks,
                        f64_radius="auto", order_rays=None):
    def pinned_f64(t, name, shape):
        if not (torch.is_tensor(t) and not t.is_cuda and t.is_pinned()
                and t.dtype == torch.float64 and t.is_contiguous() and tuple(t.shape) == shape):
            raise ValueError(f"{name} must be a contiguous pinned float64 CPU tensor of "
                             f"shape {shape}")

    n = int(state0.shape[0]) if torch.is_tensor(state0) else -1
    pinned_f64(state0, "state0", (n, 8))
    pinned_f64(out, "out", (n, 8))
    if spins is not None:
        # The kernel checks the Kerr bound of each ray's spin (the stats read
        # below raises ValueError): a host pass over the pinned spins costs
        # about 1 ms per million rays.
        pinned_f64(spins, "spins", (n,))
    if int(chunks) < 1:
        raise ValueError("chunks must be >= 1")
    dev = torch.device("cuda", torch.cuda.current_device())
    lib = _lib.load()
    states = torch.empty((n, 8), dtype=torch.float64, device=dev)
    h = torch.full((n,), float(initial_step), dtype=torch.float64, device=dev)
    lam = torch.zeros(n, dtype=torch.float64, device=dev)
    acc = torch.empty(n, dtype=torch.int64, device=dev)
    spin_d = None if spins is None else torch.empty(n, dtype=torch.float64, device=dev)
    k = max(1, min(int(chunks), n))
    band = _propagate_band(f64_radius, precision, project_every)
    ordered = (band != 0.0) if order_rays is None else bool(order_rays)
    # A warp of the mixed propagator decides its float64 band for its 64 rays:
    # pieces that start at multiples of 64 rays (of ORDER_SEGMENT rays when the
    # launch orders its rays within such segments) give every ray the
    # warp-mates, and hence the results, of the single launch.
    align = ORDER_SEGMENT if ordered else 64
    bounds = _pieces(n, k, align)
    ws = [torch.empty(lib.bh_trace_workspace_bytes(), dtype=torch.uint8, device=dev)
          for _ in bounds]
    cfg = make_config(1, rtol, atol, initial_step, max_step, 0.0, precision, "aos", timeout_s,
                      variant, 0, project_every, f64_radius=band)
    main = torch.cuda.current_stream(dev)
    # Every buffer is allocated on the caller's stream before the pieces are
    # enqueued.  An allocation inside a side stream's context could miss the
    # allocator's cache and stall the host in the middle of the pipeline (one
    # call in about ten stalled 16 ms so).  They stay alive until the side
    # streams' work is done (the stats reads below synchronise).
    order_bufs = [_order_buffers(lib, b - a, dev) if ordered else None for a, b in bounds]
    streams = _side_streams(dev)
    for st in streams:
        st.wait_stream(main)  # h, lam and the buffers come from the main stream
    for c, (a, b) in enumerate(bounds):
        st = streams[c % len(streams)]
        with torch.cuda.stream(st):
            states[a:b].copy_(state0[a:b], non_blocking=True)
            if spin_d is not None:
                spin_d[a:b].copy_(spins[a:b], non_blocking=True)
            order = _ray_order(lib, states[a:b], "aos", b - a, ordered, band, order_bufs[c])
            _lib.check(lib.bh_propagate_ordered(cfg, float(spacetime.mass),
                                                float(spacetime.spin),
                                                ptr(None if spin_d is None else spin_d[a:b]),
                                                ptr(states[a:b]), ptr(h[a:b]), ptr(lam[a:b]),
                                                ptr(acc[a:b]), ptr(order), b - a,
                                                int(n_steps), ptr(ws[c]), st.cuda_stream),
                       "propagate")
            out[a:b].copy_(states[a:b], non_blocking=True)
    for st in streams:
        main.wait_stream(st)
    stats = _lib.TraceStats()
    for c in range(len(bounds)):
        part = _lib.TraceStats()
        _lib.check(lib.bh_trace_stats_read(ptr(ws[c]), part, stream_handle()), "propagate")
        stats.attempts += part.attempts
        stats.accepted += part.accepted
        stats.iterations = max(stats.iterations, part.iterations)
        stats.timed_out = stats.timed_out or part.timed_out
        stats.bad_rays += part.bad_rays
    return out, h, lam, acc, stats
