"""Generate the golden fixtures under tests/golden/ from the reference itself.

Run where the reference project (MegaKruk/BlackHorizon) is importable; it is
read from the checkout given by --reference (required).  The fixtures are small
.npz files; MANIFEST.json records the command, the reference files' SHA-256
and the shapes written, so a reader can regenerate and compare.

    python tests/golden/make_golden.py --reference <path of the reference checkout>

Every workload below is built with the reference's own functions
(KerrSpacetime, null_momentum_from_velocity, build_state, PinholeCamera,
trace_rays, dormand_prince_step, error_ratio, step_factor, rk4_step).  The
raw-throughput workload (2^20 photons on the Kerr-Schild sphere r=30, per-ray
spin in [-0.95, 0.95]) is defined in synthetic_inputs() so bench.py and the
tests can rebuild the same rays from the seed without the reference.
"""

from __future__ import annotations

import argparse
import hashlib
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from blackhorizon_b200.workloads import (  # noqa: E402  (host-only, no GPU)
    RAW_SEED,
    raw_throughput_inputs,
)

REF_FILES = [
    "blackhorizon/kerr.py",
    "blackhorizon/geodesics.py",
    "blackhorizon/integrators.py",
    "blackhorizon/tracer.py",
    "blackhorizon/camera.py",
    "blackhorizon/imaging.py",
    "blackhorizon/examples/benchmark.py",
    "blackhorizon/offline/render.py",
    "blackhorizon/realtime/fly_camera.py",
    "blackhorizon/realtime/reference.py",
    "blackhorizon/realtime/settings.py",
    "blackhorizon/frames.py",
    "blackhorizon/vaidya.py",
    "blackhorizon/offline/inflation.py",
    "blackhorizon/emission/novikov_thorne.py",
    "blackhorizon/emission/blackbody.py",
    "blackhorizon/emission/redshift.py",
    "blackhorizon/emission/bluesheet.py",
    "blackhorizon/offline/post.py",
    "blackhorizon/offline/infall.py",
    "blackhorizon/offline/camera_path.py",
    "blackhorizon/offline/video.py",
    "tests/test_kerr.py",
    "tests/test_shadow.py",
    "tests/test_bluesheet.py",
]


def sha256(path: str) -> str:
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def random_points(n, r_min, r_max, seed):
    """Same construction as the reference's tests/test_kerr.py:11-17."""
    rng = np.random.default_rng(seed)
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=-1, keepdims=True)
    radii = rng.uniform(r_min, r_max, size=(n, 1))
    return radii * u


def gen_geometry(ref, out):
    KerrSpacetime = ref["KerrSpacetime"]
    sets = {}
    special = np.array([
        [0.0, 0.0, 1.5], [0.0, 0.0, -7.0], [2.0, 0.0, 0.0], [11.0, 0.0, 0.0],
        [0.5, 0.3, 0.01], [0.95, 0.0, 1e-6], [1.2, 0.9, 0.4], [0.0, 1.5, -0.2],
        [1.44, 0.0, 0.0], [0.3, -0.2, 1.45],
    ])
    for tag, spin, pts in [
        ("a09", 0.9, np.concatenate([random_points(300, 2.2, 60.0, 11), special])),
        ("a095", 0.95, random_points(200, 2.5, 40.0, 3)),
        ("a0", 0.0, random_points(100, 2.5, 40.0, 13)),
        ("am0998", -0.998, random_points(200, 1.1, 30.0, 17)),
    ]:
        st = KerrSpacetime(1.0, spin)
        g = st.geometry(pts[:, 0], pts[:, 1], pts[:, 2], gradients=True)
        sets[f"{tag}_spin"] = np.float64(spin)
        sets[f"{tag}_xyz"] = pts
        sets[f"{tag}_r"] = g.radius
        sets[f"{tag}_h"] = g.h
        sets[f"{tag}_l"] = g.l
        sets[f"{tag}_grad_h"] = g.grad_h
        sets[f"{tag}_grad_l"] = g.grad_l
    np.savez_compressed(os.path.join(out, "geometry.npz"), **sets)


def photon_states(ref, spin, n, seed, r_min=2.5, r_max=40.0):
    """Past-directed null states at random points outside the ergosphere."""
    G = ref["geodesics"]
    st = ref["KerrSpacetime"](1.0, spin)
    rng = np.random.default_rng(seed)
    pos = random_points(n, r_min, r_max, seed)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    mom = G.null_momentum_from_velocity(st, pos, d, "past")
    return st, G.build_state(pos, mom), pos, d


def gen_steps(ref, out):
    G, I = ref["geodesics"], ref["integrators"]
    st, s0, pos, d = photon_states(ref, 0.9, 512, 21)
    rng = np.random.default_rng(22)
    h = np.exp(rng.uniform(np.log(1e-3), np.log(2.0), size=512))

    def rhs(b):
        return G.geodesic_rhs(st, b)

    y_new, err = I.dormand_prince_step(rhs, s0, h)
    ratio = I.error_ratio(s0, y_new, err, 1e-8, 1e-10)
    factor = I.step_factor(ratio)
    rk4 = I.rk4_step(rhs, s0, h)
    np.savez_compressed(
        os.path.join(out, "steps.npz"),
        spin=np.float64(0.9), state=s0, h=h, rhs=G.geodesic_rhs(st, s0),
        dp5_new=y_new, dp5_err=err, ratio=ratio, factor=factor, rk4_new=rk4,
        hamiltonian=G.hamiltonian(st, s0),
        velocity=G.coordinate_velocity(st, s0), rtol=1e-8, atol=1e-10,
    )
    # Null momenta, both time orientations, normalised and not.
    out_nm = {"spin": np.float64(0.9), "pos": pos, "dir": d}
    for tor in ("past", "future"):
        for norm in (True, False):
            out_nm[f"{tor}_{int(norm)}"] = G.null_momentum_from_velocity(
                st, pos, d, tor, norm
            )
    np.savez_compressed(os.path.join(out, "null_momentum.npz"), **out_nm)


def gen_camera(ref, out):
    C = ref["camera"]
    cams = {
        "c1": C.PinholeCamera.from_orbit(50.0, 60.0, fov_degrees=30.0, width=40, height=30),
        "c3": C.PinholeCamera.from_orbit(50.0, 80.0, fov_degrees=25.0, width=32, height=18),
        "pole": C.PinholeCamera.from_orbit(20.0, 0.0, fov_degrees=30.0, width=8, height=6),
        "free": C.PinholeCamera(position=(3.0, -40.0, 7.0), target=(1.0, 2.0, -1.0),
                                up_hint=(0.2, 0.1, 1.0), fov_degrees=45.0, width=17, height=11),
    }
    arrs = {}
    for k, c in cams.items():
        arrs[f"{k}_position"] = np.asarray(c.position, dtype=np.float64)
        arrs[f"{k}_target"] = np.asarray(c.target, dtype=np.float64)
        arrs[f"{k}_up_hint"] = np.asarray(c.up_hint, dtype=np.float64)
        arrs[f"{k}_fov"] = np.float64(c.fov_degrees)
        arrs[f"{k}_wh"] = np.array([c.width, c.height], dtype=np.int64)
        arrs[f"{k}_basis"] = np.stack([c.forward, c.right, c.up])
        arrs[f"{k}_dirs"] = c.ray_directions()
    np.savez_compressed(os.path.join(out, "camera.npz"), **arrs)


def camera_state(ref, spin, distance, inc, fov, w, h):
    C, G = ref["camera"], ref["geodesics"]
    st = ref["KerrSpacetime"](1.0, spin)
    cam = C.PinholeCamera.from_orbit(distance, inc, fov_degrees=fov, width=w, height=h)
    pos = cam.ray_origins()
    d = cam.ray_directions()
    mom = G.null_momentum_from_velocity(st, pos, d, "past")
    return st, G.build_state(pos, mom)


def gen_trace_c1(ref, out):
    T = ref["tracer"]
    kw = dict(escape_radius=100.0, max_steps=5000, rtol=1e-8, atol=1e-10,
              capture_margin=0.01)
    # Full-state golden at 40x30 (same camera geometry as the 160x120 frame).
    st, s_small = camera_state(ref, 0.9, 50.0, 60.0, 30.0, 40, 30)
    res = T.trace_rays(st, s_small, **kw)
    np.savez_compressed(
        os.path.join(out, "trace_c1_40x30.npz"), state0=s_small,
        states=res.states, status=res.status.astype(np.int8),
        steps=res.steps.astype(np.int32), iterations=np.int64(res.iterations),
    )
    # Full 160x120 frame: status and steps for every ray, states for every
    # 8th ray.
    st, s_full = camera_state(ref, 0.9, 50.0, 60.0, 30.0, 160, 120)
    t0 = time.perf_counter()
    res = T.trace_rays(st, s_full, **kw)
    dt = time.perf_counter() - t0
    sub = np.arange(0, s_full.shape[0], 8)
    np.savez_compressed(
        os.path.join(out, "trace_c1_160x120.npz"),
        status=res.status.astype(np.int8), steps=res.steps.astype(np.int16),
        iterations=np.int64(res.iterations), sub_index=sub,
        sub_states=res.states[sub], reference_seconds=np.float64(dt),
    )


def _trace_shard(args):
    spin, state, kw = args
    sys.path.insert(0, _REFERENCE_PATH)
    from blackhorizon.kerr import KerrSpacetime
    from blackhorizon.tracer import trace_rays

    res = trace_rays(KerrSpacetime(1.0, spin), state, **kw)
    return res.status.astype(np.int8), res.steps.astype(np.int16)


def gen_trace_c3(ref, out, procs):
    """Full-HD frame, a=0.9, 80 deg, fov 25: status for every pixel.

    Rays are independent, so tracing contiguous shards in worker processes
    gives the per-ray results of one trace_rays call."""
    st, s = camera_state(ref, 0.9, 50.0, 80.0, 25.0, 1920, 1080)
    kw = dict(escape_radius=100.0, max_steps=10000, rtol=1e-9, atol=1e-12,
              capture_margin=0.01)
    shards = np.array_split(s, procs * 8)
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(procs) as pool:
        parts = pool.map(_trace_shard, [(0.9, x, kw) for x in shards])
    dt = time.perf_counter() - t0
    status = np.concatenate([p[0] for p in parts])
    steps = np.concatenate([p[1] for p in parts])
    np.savez_compressed(
        os.path.join(out, "trace_c3_status.npz"), status=status, steps=steps,
        reference_seconds=np.float64(dt), procs=np.int64(procs),
    )


def gen_fans(ref, out):
    """First-round equatorial fans of the reference's tests/test_shadow.py:22-84
    (camera at D=1000 on +x, escape 1.2 D, max_steps 60000, rtol 1e-10,
    atol 1e-13, max_step 5)."""
    G, T = ref["geodesics"], ref["tracer"]
    D = 1000.0
    arrs = {}
    for tag, spin, lo, hi in [
        ("a0_pos", 0.0, 4.5e-3, 6.5e-3),
        ("a09_pro", 0.9, -4.0e-3, -2.0e-3),
        ("a09_ret", 0.9, 5.5e-3, 8.0e-3),
    ]:
        st = ref["KerrSpacetime"](1.0, spin)
        offsets = np.linspace(lo, hi, 48)
        n = offsets.shape[0]
        pos = np.tile(np.array([[D, 0.0, 0.0]]), (n, 1))
        d = np.stack([-np.ones(n), offsets, np.zeros(n)], axis=-1)
        d /= np.linalg.norm(d, axis=-1, keepdims=True)
        mom = G.null_momentum_from_velocity(st, pos, d, "past")
        s0 = G.build_state(pos, mom)
        res = T.trace_rays(st, s0, escape_radius=1.2 * D, max_steps=60000,
                           rtol=1e-10, atol=1e-13, max_step=5.0)
        arrs[f"{tag}_spin"] = np.float64(spin)
        arrs[f"{tag}_offsets"] = offsets
        arrs[f"{tag}_state0"] = s0
        arrs[f"{tag}_status"] = res.status.astype(np.int8)
        arrs[f"{tag}_steps"] = res.steps.astype(np.int32)
        arrs[f"{tag}_states"] = res.states
    np.savez_compressed(os.path.join(out, "fans.npz"), **arrs)


def gen_raw_throughput(ref, out, n=512, n_steps=2000):
    """First n rays of the raw-throughput workload, n_steps attempted DP5(4)
    steps each with the tracer's accept/reject and step update
    (tracer.py:111-120) and no termination, per-ray spin."""
    G, I = ref["geodesics"], ref["integrators"]
    pos, d, spin = raw_throughput_inputs(n)
    st = object.__new__(ref["KerrSpacetime"])
    st.mass = 1.0
    st.spin = spin
    mom = G.null_momentum_from_velocity(st, pos, d, "past")
    s0 = G.build_state(pos, mom)
    y = s0.copy()
    h = np.full(n, 0.1)
    acc = np.zeros(n, dtype=np.int64)

    def rhs(b):
        return G.geodesic_rhs(st, b)

    with np.errstate(all="ignore"):
        for _ in range(n_steps):
            y_new, err = I.dormand_prince_step(rhs, y, h)
            ratio = I.error_ratio(y, y_new, err, 1e-8, 1e-10)
            ok = ratio <= 1.0
            y = np.where(ok[:, None], y_new, y)
            acc += ok
            h = np.clip(h * I.step_factor(ratio), 0.0, 2.0)
    np.savez_compressed(
        os.path.join(out, "raw_throughput.npz"), seed=np.int64(RAW_SEED),
        pos=pos, dir=d, spin=spin, state0=s0, final=y, h=h, accepted=acc,
        n_steps=np.int64(n_steps), rtol=1e-8, atol=1e-10,
    )


def gen_rk4(ref, out, n=256, n_steps=50):
    """examples/benchmark.py:22-51: inward photons on r=50, a=0.9, seed 7,
    fixed h=0.05."""
    G, I = ref["geodesics"], ref["integrators"]
    st = ref["KerrSpacetime"](1.0, 0.9)
    rng = np.random.default_rng(7)
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=-1, keepdims=True)
    pos = 50.0 * u
    mom = G.null_momentum_from_velocity(st, pos, -u)
    s0 = G.build_state(pos, mom)
    y = s0.copy()
    h = np.full(n, 0.05)
    for _ in range(n_steps):
        y = I.rk4_step(lambda b: G.geodesic_rhs(st, b), y, h)
    np.savez_compressed(os.path.join(out, "rk4.npz"), state0=s0, final=y,
                        h=np.float64(0.05), n_steps=np.int64(n_steps))


def _offline_modules(reference):
    """The offline renderer's module without the real-time package's GL
    initialisation: blackhorizon.realtime is registered as a bare package so
    that only fly_camera (pure NumPy) is imported from it."""
    import types

    if "blackhorizon.realtime" not in sys.modules:
        pkg = types.ModuleType("blackhorizon.realtime")
        pkg.__path__ = [os.path.join(reference, "blackhorizon", "realtime")]
        sys.modules["blackhorizon.realtime"] = pkg
    from blackhorizon.emission.novikov_thorne import disk_inner_radius
    from blackhorizon.offline import render
    from blackhorizon.realtime.fly_camera import FlyCamera

    return render, FlyCamera, disk_inner_radius


def tile_camera_states(ref, render, FlyCamera, spin, distance, inc, az, w, h, fov, ss):
    """render.py:555-599: subpixel directions of a FlyCamera and the
    past-directed null states at its position."""
    G = ref["geodesics"]
    st = ref["KerrSpacetime"](1.0, spin)
    cam = FlyCamera.from_orbit(distance, inc, az)
    d = render.subpixel_directions(cam, w, h, fov, ss)
    pos = np.tile(cam.position[None, :], (d.shape[0], 1))
    mom = G.null_momentum_from_velocity(st, pos, d, time_orientation="past")
    return st, cam, d, G.build_state(pos, mom)


def gen_offline_tile(ref, out):
    """render.py:184-349 on a 32x20 tile of the offline renderer's default
    view (a=0.9, FlyCamera at D=26, inclination 82, fov 70, disk from the
    ISCO to 18 M, escape at 1.3 max(D, 18)): first pass at rtol 1e-9 with
    12000 steps, then the photon-shell pass (render.py:613-630) of the
    saturated non-disk rays at rtol 1e-11 with 48000 steps.  A second tile
    at a=-0.7 (retrograde ISCO) with a 200-step budget makes the
    saturation branch common."""
    render, FlyCamera, disk_inner_radius = _offline_modules(_REFERENCE_PATH)
    arrs = {}
    for tag, spin, inc, az, max_steps in [("a09", 0.9, 82.0, 0.0, 12000),
                                          ("am07", -0.7, 75.0, 40.0, 200)]:
        settings = render.OfflineSettings(spin=spin)
        st, cam, d, s0 = tile_camera_states(ref, render, FlyCamera, spin, 26.0, inc, az,
                                            32, 20, settings.fov_degrees, 1)
        r_in = float(disk_inner_radius(st))
        r_out = max(settings.disk_outer_radius, r_in + 1.0)
        esc = 1.3 * max(cam.distance_from_origin, r_out)
        res = render._trace_tile(st, s0, esc, settings, (r_in, r_out), settings.rtol, max_steps)
        retrace = res.saturated & (res.status != 5)
        idx = np.nonzero(retrace)[0]
        if idx.size:
            ref2 = render._trace_tile(st, s0[idx], esc, settings, (r_in, r_out),
                                      settings.refine_rtol, max_steps * 4)
        arrs[f"{tag}_spin"] = np.float64(spin)
        arrs[f"{tag}_position"] = cam.position
        arrs[f"{tag}_directions"] = d
        arrs[f"{tag}_state0"] = s0
        arrs[f"{tag}_disk"] = np.array([r_in, r_out])
        arrs[f"{tag}_escape_radius"] = np.float64(esc)
        arrs[f"{tag}_max_steps"] = np.int64(max_steps)
        arrs[f"{tag}_status"] = res.status.astype(np.int8)
        arrs[f"{tag}_escape_directions"] = res.escape_directions
        arrs[f"{tag}_hit_positions"] = res.hit_positions
        arrs[f"{tag}_hit_momenta"] = res.hit_momenta
        arrs[f"{tag}_saturated"] = res.saturated.astype(np.int8)
        arrs[f"{tag}_retrace_index"] = idx
        if idx.size:
            arrs[f"{tag}_retrace_status"] = ref2.status.astype(np.int8)
            arrs[f"{tag}_retrace_escape_directions"] = ref2.escape_directions
            arrs[f"{tag}_retrace_hit_positions"] = ref2.hit_positions
            arrs[f"{tag}_retrace_hit_momenta"] = ref2.hit_momenta
    np.savez_compressed(os.path.join(out, "offline_tile.npz"), **arrs)


# Interior cameras of render_hdr (render.py:520-550 with camera_tetrad): the
# rain observer's tetrad, pinhole directions, tetrad momenta, escape radius
# max(100, 1.3 disk_outer).  (tag, spin, position, forward, up, stop, disk);
# stop None is the realistic terminal surface 1.02 r_minus.
INTERIOR_CASES = [
    ("sheet", 0.9, (0.03, 0.03, 0.68), (0.0, 0.0, -1.0), (0.0, 1.0, 0.0), None, False),
    ("ideal", 0.9, (0.03, 0.03, 1.2), (0.0, 0.0, -1.0), (0.0, 1.0, 0.0), 0.02, False),
    ("disk", 0.6, (0.6, 0.3, 1.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0), None, True),
    ("schw", 0.0, (0.0, 0.0, 1.5), (0.0, 0.0, -1.0), (0.0, 1.0, 0.0), 0.05, True),
]


def gen_offline_interior(ref, out):
    """render.py:184-309 in interior-camera mode (interior_stop) on 32x24
    tetrad tiles (fov 80, supersample 1) of cameras inside the horizon,
    as tests/test_bluesheet.py:86-130 sets them up."""
    render, _, disk_inner_radius = _offline_modules(_REFERENCE_PATH)
    from blackhorizon.frames import build_tetrad, rain_four_velocity, tetrad_ray_momenta

    G = ref["geodesics"]
    arrs = {}
    for tag, spin, pos, fwd, up, stop, disk in INTERIOR_CASES:
        st = ref["KerrSpacetime"](1.0, spin)
        stop = st.inner_horizon_radius * 1.02 if stop is None else stop
        pos = np.array(pos)
        vel = rain_four_velocity(st, pos[None, :])[0]
        tet = build_tetrad(st, pos, vel, np.array(fwd), np.array(up))
        settings = render.OfflineSettings(spin=spin, supersample=1, fov_degrees=80.0,
                                          disk_enabled=disk)
        d = render.pinhole_grid(32, 24, settings.fov_degrees, 1)
        mom = tetrad_ray_momenta(st, pos, tet, d)
        s0 = G.build_state(np.tile(pos[None, :], (d.shape[0], 1)), mom)
        r_in = float(disk_inner_radius(st))
        r_out = max(settings.disk_outer_radius, r_in + 1.0)
        esc = max(100.0, 1.3 * r_out)
        radii = (r_in, r_out) if disk else None
        res = render._trace_tile(st, s0, esc, settings, radii, settings.rtol,
                                 settings.max_steps, interior_stop=stop)
        arrs[f"{tag}_spin"] = np.float64(spin)
        arrs[f"{tag}_position"] = pos
        arrs[f"{tag}_forward"] = np.array(fwd)
        arrs[f"{tag}_up"] = np.array(up)
        arrs[f"{tag}_velocity"] = vel
        arrs[f"{tag}_tetrad"] = tet
        arrs[f"{tag}_stop"] = np.float64(stop)
        arrs[f"{tag}_disk"] = np.array([r_in, r_out] if disk else [0.0, 0.0])
        arrs[f"{tag}_escape_radius"] = np.float64(esc)
        arrs[f"{tag}_state0"] = s0
        arrs[f"{tag}_status"] = res.status.astype(np.int8)
        arrs[f"{tag}_escape_directions"] = res.escape_directions
        arrs[f"{tag}_hit_positions"] = res.hit_positions
        arrs[f"{tag}_hit_momenta"] = res.hit_momenta
        arrs[f"{tag}_saturated"] = res.saturated.astype(np.int8)
    np.savez_compressed(os.path.join(out, "offline_interior.npz"), **arrs)


def _reference_frame_rays(render, st, state0, escape_radius, settings, disk_radii,
                          interior_stop):
    """The tracing half of render_hdr (render.py:599-630) for one tile: the
    first pass and the photon-shell retrace merged."""
    res = render._trace_tile(st, state0, escape_radius, settings, disk_radii, settings.rtol,
                             settings.max_steps, interior_stop=interior_stop)
    retrace = res.saturated & (res.status != 5) & (res.status != 6)
    if retrace.any():
        idx = np.nonzero(retrace)[0]
        ref2 = render._trace_tile(st, state0[idx], escape_radius, settings, disk_radii,
                                  settings.refine_rtol, settings.max_steps * 4,
                                  interior_stop=interior_stop)
        for name in ("status", "escape_directions", "hit_positions", "hit_momenta"):
            getattr(res, name)[retrace] = getattr(ref2, name)
    return res


def gen_emission(ref, out):
    """The emission half of render_hdr (render.py:352-484, 630-680) and
    develop (post.py:88-106): the temperature and blackbody tables, the
    starfield and disk radiance per ray, three small frames traced and shaded
    by render_hdr (exterior default view 48x30 supersample 2; interior tetrad
    cameras near the blue sheet (tests/test_bluesheet.py's close observer,
    looking down the spin axis) and inside a=0.6 with the disk), their
    per-ray trace outputs, and developed 8-bit images."""
    render, FlyCamera, disk_inner_radius = _offline_modules(_REFERENCE_PATH)
    from blackhorizon.emission.blackbody import blackbody_lut
    from blackhorizon.emission.bluesheet import (SHEET_COLOR, blueshift_amplification,
                                                 sheet_radiance)
    from blackhorizon.emission.novikov_thorne import temperature_lut
    from blackhorizon.emission.redshift import static_observer_lapse
    from blackhorizon.frames import build_tetrad, rain_four_velocity, tetrad_ray_momenta
    from blackhorizon.offline.post import develop, gaussian_kernel

    G = ref["geodesics"]
    arrs = {}
    for tag, spin in (("a09", 0.9), ("am07", -0.7), ("a0", 0.0)):
        st = ref["KerrSpacetime"](1.0, spin)
        r_in = float(disk_inner_radius(st))
        table, lo, hi = temperature_lut(spin, max(18.0, r_in + 1.0), size=2048)
        arrs[f"temperature_{tag}"] = table
        arrs[f"temperature_{tag}_range"] = np.array([lo, hi])
    bb, bb_lo, bb_hi = blackbody_lut(size=1024)
    arrs["blackbody"] = bb
    arrs["blackbody_log_range"] = np.array([bb_lo, bb_hi])
    for sigma in (6.0, 3.0, 0.2):
        arrs[f"gauss_{sigma}"] = gaussian_kernel(sigma)
    rng = np.random.default_rng(5)
    d = rng.normal(size=(4096, 3))
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    shift = rng.uniform(0.3, 3.0, 4096)
    arrs["star_dirs"] = d
    arrs["star_shift"] = shift
    arrs["star_rgb"] = render._starfield_hdr(d)
    arrs["star_rgb_shift"] = render._starfield_hdr(d, shift=shift)
    frames = [
        ("ext", 0.9, 48, 30, 2, None, None, True),
        ("sheet", 0.9, 48, 32, 1, ((0.03, 0.03, 0.68), (0.0, 0.0, -1.0), (0.0, 1.0, 0.0)),
         "real", False),
        ("indisk", 0.6, 48, 32, 1, ((0.6, 0.3, 1.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0)),
         "real", True),
    ]
    for tag, spin, w, h, ss, tetrad_seed, stop, disk in frames:
        st = ref["KerrSpacetime"](1.0, spin)
        fov = 70.0 if tetrad_seed is None else 80.0
        settings = render.OfflineSettings(spin=spin, supersample=ss, fov_degrees=fov,
                                          disk_enabled=disk)
        r_in = float(disk_inner_radius(st))
        r_out = max(settings.disk_outer_radius, r_in + 1.0)
        radii = (r_in, r_out) if disk else None
        table, _, _ = temperature_lut(spin, r_out, size=2048)
        kw = {}
        if tetrad_seed is None:
            cam = FlyCamera.from_orbit(26.0, 82.0, 0.0)
            dirs = render.subpixel_directions(cam, w, h, fov, ss)
            pos = np.tile(cam.position[None, :], (dirs.shape[0], 1))
            mom = G.null_momentum_from_velocity(st, pos, dirs, time_orientation="past")
            esc = 1.3 * max(cam.distance_from_origin, r_out)
            lapse = static_observer_lapse(st, cam.position)
            energy = None
            interior = None
            sheet = np.zeros(3)
        else:
            position, fwd, up = (np.array(v) for v in tetrad_seed)
            interior = st.inner_horizon_radius * 1.02
            vel = rain_four_velocity(st, position[None, :])[0]
            tet = build_tetrad(st, position, vel, fwd, up)
            cam = FlyCamera(position=position.copy(), yaw=0.0, pitch=0.0)
            dirs = render.pinhole_grid(w, h, fov, ss)
            pos = np.tile(position[None, :], (dirs.shape[0], 1))
            mom = tetrad_ray_momenta(st, position, tet, dirs)
            esc = max(100.0, 1.3 * r_out)
            cam_r = float(st.kerr_schild_radius(position[None, 0], position[None, 1],
                                                position[None, 2])[0])
            lapse = float(blueshift_amplification(st, np.array([cam_r]))[0])
            energy = mom[:, 0]
            sheet = (float(sheet_radiance(np.array([lapse]))[0])
                     * np.array(SHEET_COLOR, dtype=np.float32)) if lapse > 1.0 else np.zeros(3)
            kw = dict(camera_tetrad=tet, interior_stop=interior)
            arrs[f"{tag}_tetrad"] = tet
        s0 = G.build_state(pos, mom)
        res = _reference_frame_rays(render, st, s0, esc, settings, radii, interior)
        rad = np.zeros((s0.shape[0], 3))
        esc_m = res.status == 2
        if esc_m.any():
            shift = None if energy is None else lapse / energy[esc_m]
            rad[esc_m] = render._starfield_hdr(res.escape_directions[esc_m], shift=shift)
        hit = res.status == 5
        if hit.any():
            rad[hit] = render._disk_radiance(st, res.hit_positions[hit], res.hit_momenta[hit],
                                             settings, r_in, r_out, table, lapse, bb, bb_lo,
                                             bb_hi)
        rad[res.status == 6] = sheet
        hdr = render.render_hdr(cam, w, h, settings, progress=False, **kw)
        mean = rad.reshape(h, w, ss * ss, 3).mean(axis=2).astype(np.float32)
        assert np.array_equal(mean, hdr), tag
        for k, v in (("state0", s0), ("status", res.status.astype(np.int8)),
                     ("escape_directions", res.escape_directions),
                     ("hit_positions", res.hit_positions), ("hit_momenta", res.hit_momenta),
                     ("radiance", rad), ("hdr", hdr),
                     ("params", np.array([spin, w, h, ss, fov, esc, lapse, r_in, r_out,
                                          -1.0 if interior is None else interior,
                                          1.0 if disk else 0.0])),
                     ("sheet_rgb", np.asarray(sheet, dtype=np.float64)),
                     ("position", cam.position)):
            arrs[f"{tag}_{k}"] = v
        arrs[f"{tag}_developed"] = develop(hdr)
        arrs[f"{tag}_developed_e2s3"] = develop(hdr, exposure=2.5, bloom_sigma=3.0)
        arrs[f"{tag}_developed_nobloom"] = develop(hdr, exposure=0.7, bloom_strength=0.0)
    np.savez_compressed(os.path.join(out, "emission.npz"), **arrs)


def gen_inflation_frame(ref, out):
    """render_layer_frame (offline/inflation.py:243-346) on small flythrough
    frames of the q = 0.9 surrogate with the shell at v = 6, R = 1.2: rain
    observers at r = 1.3 (looking outward and inward) and at r = 0.8, 24x16
    pixels with supersample 2, fov 90.  The per-ray trace outputs are made
    by the same steps as render_layer_frame and checked against its image."""
    _offline_modules(_REFERENCE_PATH)
    from blackhorizon.frames import build_tetrad, lower_index
    from blackhorizon.offline import inflation as infl
    from blackhorizon.offline.render import OfflineSettings
    from blackhorizon.vaidya import ChargedVaidyaSpacetime

    st = ChargedVaidyaSpacetime(charge=0.9, shell_start_v=6.0, shell_start_radius=1.2)
    settings = OfflineSettings(supersample=2, fov_degrees=90.0)
    w, h, ss = 24, 16, 2
    arrs = {"params": np.array([st.mass, st.charge, st.tail_mass, st.tail_start, st.tail_power,
                                st.shell_energy, st.shell_start_v, st.shell_start_radius,
                                st.shell_width, st.mass_cap]),
            "frame": np.array([w, h, ss, settings.fov_degrees])}
    for tag, radius, look in (("out13", 1.3, "outward"), ("in13", 1.3, "inward"),
                              ("out08", 0.8, "outward")):
        state = infl.rain_state(st, np.array([radius, 0.0, 0.0]), 6.0)[0]
        hdr = infl.render_layer_frame(st, state, w, h, settings, look)
        # The rays of render_layer_frame (inflation.py:252-320), step by step.
        position = state[1:4]
        velocity = infl.camera_four_velocity(st, state[None, :])
        slice_geo = st.frozen(float(state[0]))
        outward = position / max(np.linalg.norm(position), 1e-12)
        up_seed = np.array([0.0, 0.0, 1.0])
        forward = -outward if look == "inward" else outward
        tetrad = build_tetrad(slice_geo, position, velocity, forward, up_seed)
        tan_half = np.tan(np.radians(settings.fov_degrees) / 2.0)
        offsets = (np.arange(ss) + 0.5) / ss
        u = (np.arange(w)[:, None] + offsets[None, :]).reshape(-1) / w * 2.0 - 1.0
        v = 1.0 - (np.arange(h)[:, None] + offsets[None, :]).reshape(-1) / h * 2.0
        ug = np.tile(u.reshape(w, ss)[None, :, None, :], (h, 1, ss, 1)).reshape(-1)
        vg = np.tile(v.reshape(h, ss)[:, None, :, None], (1, w, 1, ss)).reshape(-1)
        local = np.stack([np.ones_like(ug), ug * tan_half, vg * tan_half / (w / h)], axis=-1)
        local /= np.linalg.norm(local, axis=-1, keepdims=True)
        spatial = local[:, 0:1] * tetrad[1] + local[:, 1:2] * tetrad[2] + local[:, 2:3] * tetrad[3]
        positions = np.tile(position[None, :], (local.shape[0], 1))
        momenta = lower_index(slice_geo, positions, -(tetrad[0][None, :] - spatial))
        s0 = np.concatenate([np.full((local.shape[0], 1), float(state[0])), positions, momenta],
                            axis=1)
        esc = max(12.0, 2.5 * float(np.linalg.norm(position)))
        status, edir, mass, _ = infl._trace_vaidya_tile(st, s0, esc,
                                                        st.inner_horizon_radius * 1.001)
        rad = np.zeros((s0.shape[0], 3), dtype=np.float32)
        if (status == 0).any():
            rad[status == 0] = infl._surrogate_sky(edir[status == 0])
        lay = status == 1
        if lay.any():
            excess = np.maximum(mass[lay] - st.mass, 0.0) / st.mass
            glow = 0.35 + 1.2 * np.log1p(excess) ** 2
            rad[lay] = glow[:, None] * np.array(infl.SHEET_COLOR, dtype=np.float32)
        assert np.array_equal(rad.reshape(h, w, ss * ss, 3).mean(axis=2), hdr), tag
        for k, val in (("state", state), ("tetrad", tetrad), ("state0", s0),
                       ("status", status.astype(np.int8)), ("escape_dir", edir),
                       ("end_mass", mass), ("radiance", rad), ("hdr", hdr)):
            arrs[f"{tag}_{k}"] = val
        arrs[f"{tag}_look"] = np.array(look)
    # The flythrough's camera worldline (inflation.py:77-135) with the CLI's
    # defaults: start at r = 1.3, v = 6, stop at 1.001 r_minus.
    taus, states = infl.build_worldline(st, 1.3, 6.0, st.inner_horizon_radius * 1.001)
    arrs["worldline_taus"] = taus
    arrs["worldline_states"] = states
    np.savez_compressed(os.path.join(out, "inflation_frame.npz"), **arrs)


def gen_plunge(ref, out):
    """offline/infall.py:38-262: radial momenta, the plunge worldlines of
    three presets (rain at a = 0.6 from r = 3 to the Cauchy horizon, fast
    E = 1.5 in Schwarzschild from r = 6 to 0.02, maximal E = 0 at a = 0.9
    from just inside r_plus), the camera tetrads at samples of the first, and
    one 32x20 frame of it rendered by render_hdr with the tetrad and stop."""
    render, FlyCamera, _ = _offline_modules(_REFERENCE_PATH)
    from blackhorizon.offline import infall

    arrs = {}
    cases = (("rain06", 0.6, 3.0, 1.0, "real"), ("fast0", 0.0, 6.0, 1.5, 0.02),
             ("max09", 0.9, None, 0.0, "real"))
    for tag, spin, start, energy, stop in cases:
        st = ref["KerrSpacetime"](1.0, spin)
        if start is None:
            start = st.outer_horizon_radius * 0.995
        if stop == "real":
            stop = st.inner_horizon_radius * 1.02
        mom = infall.radial_momentum(st, np.array([start, 0.0, 0.0]), energy)
        taus, states = infall.build_plunge(st, start, energy, stop)
        idx = np.unique(np.concatenate([np.arange(0, taus.size, 25), [taus.size - 1]]))
        arrs[f"{tag}_args"] = np.array([spin, start, energy, stop])
        arrs[f"{tag}_momentum"] = mom
        arrs[f"{tag}_count"] = np.int64(taus.size)
        arrs[f"{tag}_index"] = idx
        arrs[f"{tag}_taus"] = taus[idx]
        arrs[f"{tag}_states"] = states[idx]
        if tag == "rain06":
            samples = [0, taus.size // 2, taus.size - 1]
            for k, look in zip(samples, ("inward", "outward", "side")):
                pos, tet = infall.plunge_tetrad(st, states[k], look)
                arrs[f"tetrad_{look}_sample"] = states[k]
                arrs[f"tetrad_{look}"] = tet
            settings = render.OfflineSettings(spin=spin, supersample=1, fov_degrees=80.0)
            k = taus.size // 2
            pos, tet = infall.plunge_tetrad(st, states[k], "inward")
            cam = FlyCamera(position=pos.copy(), yaw=0.0, pitch=0.0)
            arrs["frame_sample"] = states[k]
            arrs["frame_hdr"] = render.render_hdr(cam, 32, 20, settings, progress=False,
                                                  camera_tetrad=tet, interior_stop=stop)
    np.savez_compressed(os.path.join(out, "plunge.npz"), **arrs)


def gen_video(ref, out):
    """offline/camera_path.py and offline/video.py:33-59: poses and cameras
    along a three-keyframe path and an orbit path, and downsample /
    frame_bloom of a seeded random frame and of a developed offline frame."""
    _offline_modules(_REFERENCE_PATH)
    from blackhorizon.offline import camera_path as cp
    from blackhorizon.offline import video

    keys = [cp.CameraKeyframe(0.0, 30.0, 80.0, 0.0, 60.0),
            cp.CameraKeyframe(2.0, 15.0, 60.0, 90.0, 70.0),
            cp.CameraKeyframe(5.0, 20.0, 85.0, 400.0, 50.0)]
    times = np.array([-1.0, 0.0, 0.7, 2.0, 3.3, 4.99, 5.0, 6.0])
    arrs = {"keys": np.array([[k.time, k.distance, k.inclination_degrees, k.azimuth_degrees,
                               k.fov_degrees] for k in keys]), "times": times}
    for tag, path in (("path", cp.CameraPath(keys)), ("orbit", cp.orbit_path(4.0, 25.0, 70.0, 1.5))):
        poses, positions, bases = [], [], []
        for t in times:
            p = path.pose_at(float(t))
            poses.append([p.time, p.distance, p.inclination_degrees, p.azimuth_degrees,
                          p.fov_degrees])
            cam = path.camera_at(float(t))
            positions.append(cam.position)
            bases.append(np.stack(cam.basis()))
        arrs[f"{tag}_poses"] = np.array(poses)
        arrs[f"{tag}_positions"] = np.array(positions)
        arrs[f"{tag}_bases"] = np.array(bases)
    rng = np.random.default_rng(11)
    frames = {"random": rng.integers(0, 256, size=(67, 97, 3), dtype=np.uint8),
              "developed": np.load(os.path.join(out, "emission.npz"))["ext_developed"]}
    for tag, img in frames.items():
        arrs[f"{tag}_frame"] = img
        for f in (2, 3):
            arrs[f"{tag}_down{f}"] = video.downsample(img, f)
        for st in (0.25, 0.6):
            arrs[f"{tag}_bloom{st}"] = video.frame_bloom(img, st)
    np.savez_compressed(os.path.join(out, "video.npz"), **arrs)


def gen_midpoint(ref, out):
    """implicit_midpoint_step (integrators.py:177-207) from the states and
    steps of steps.npz, with 4 and 6 fixed-point iterations, and 200 steps
    of the bound timelike orbit of tests/test_offline.py:38-44 (h = 0.2)."""
    G, I = ref["geodesics"], ref["integrators"]
    g = np.load(os.path.join(out, "steps.npz"))
    st = ref["KerrSpacetime"](1.0, float(g["spin"]))
    rhs = lambda b: G.geodesic_rhs(st, b)  # noqa: E731
    arrs = {"spin": g["spin"], "state": g["state"], "h": g["h"]}
    for it in (4, 6):
        arrs[f"step_it{it}"] = I.implicit_midpoint_step(rhs, g["state"], g["h"], iterations=it)
    orbit_st = ref["KerrSpacetime"](1.0, 0.9)
    pos = np.array([[14.0, 0.0, 0.0]])
    y = G.build_state(pos, G.timelike_momentum(orbit_st, pos, np.array([[0.0, 0.21, 0.02]])))
    arrs["orbit_state0"] = y.copy()
    orhs = lambda b: G.geodesic_rhs(orbit_st, b)  # noqa: E731
    for _ in range(200):
        y = I.implicit_midpoint_step(orhs, y, np.array([0.2]))
    arrs["orbit_200"] = y
    np.savez_compressed(os.path.join(out, "midpoint.npz"), **arrs)


def gen_images(ref, out):
    """imaging.py:27-91 on the reference's own traces.

    - render_image of the 40x30 and 160x120 frames of the small config;
    - celestial_checkerboard of random directions, directions on cell
      boundaries, and the poles;
    - render_image of random states with every status code (0-5), so that
      each status's colour is pinned."""
    from blackhorizon import imaging

    T = ref["tracer"]
    kw = dict(escape_radius=100.0, max_steps=5000, rtol=1e-8, atol=1e-10,
              capture_margin=0.01)
    arrs = {}
    for w, h in ((40, 30), (160, 120)):
        st, s0 = camera_state(ref, 0.9, 50.0, 60.0, 30.0, w, h)
        res = T.trace_rays(st, s0, **kw)
        arrs[f"image_{w}x{h}"] = imaging.render_image(st, res, w, h)
        if w == 40:
            arrs["states_40x30"] = res.states
            arrs["status_40x30"] = res.status.astype(np.int32)
    rng = np.random.default_rng(31)
    d = rng.normal(size=(4000, 3))
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    # Cell boundaries: polar angles k pi / 12 and azimuths k pi / 12 - pi.
    k = np.arange(0, 25)
    th = np.repeat(k * np.pi / 12.0, 25)
    ph = np.tile(k * np.pi / 12.0 - np.pi, 25)
    edge = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], axis=-1)
    poles = np.array([[0.0, 0.0, 1.0], [0.0, 0.0, -1.0], [1.0, 0.0, 0.0], [-1.0, 0.0, 0.0],
                      [0.0, 1.0, 0.0], [0.0, -1.0, 0.0], [-1.0, -0.0, 0.0]])
    dirs = np.concatenate([d, edge, poles])
    arrs["checker_directions"] = dirs
    arrs["checker_colors_12"] = imaging.celestial_checkerboard(dirs)
    arrs["checker_colors_7"] = imaging.celestial_checkerboard(dirs, cells=7)
    st, s0, _, _ = photon_states(ref, 0.9, 600, 41)
    status = np.arange(600, dtype=np.int32) % 6
    res = T.TraceResult(states=s0, status=status, steps=np.zeros(600, dtype=np.int64),
                        iterations=0)
    arrs["mixed_states"] = s0
    arrs["mixed_status"] = status
    arrs["mixed_image"] = imaging.render_image(st, res, 30, 20)
    np.savez_compressed(os.path.join(out, "images.npz"), **arrs)


def _fibonacci_sphere(n):
    """Nearly uniform unit directions (the construction of the reference's
    tests/test_interior.py:26-39)."""
    i = np.arange(n, dtype=float) + 0.5
    polar = np.arccos(1.0 - 2.0 * i / n)
    az = np.pi * (1.0 + 5.0 ** 0.5) * i
    return np.stack([np.cos(az) * np.sin(polar), np.sin(az) * np.sin(polar), np.cos(polar)],
                    axis=-1)


def gen_realtime(ref, out):
    """realtime/reference.py:41-188 (trace_like_shader), the CPU mirror of the
    real-time fragment shader, on:

    - the equatorial fans of tests/test_realtime_reference.py at D = 30, with
      every quality preset at a = 0.9, MEDIUM at a = 0, HIGH and LOW at
      a = 0.998, and the adaptive tracer's statuses at rtol 1e-10;
    - a 48x36 pinhole frame with the disk (a = 0.9, D = 30, inclination 80);
    - interior rain-observer cameras (frames.py:102-218; the views of
      tests/test_interior.py) at r = 1.9 and 0.5 (a = 0) and inside a = 0.6."""
    _offline_modules(_REFERENCE_PATH)  # registers the bare realtime package
    from blackhorizon import frames
    from blackhorizon.emission.novikov_thorne import disk_inner_radius
    from blackhorizon.realtime.reference import trace_like_shader
    from blackhorizon.realtime.settings import QualityPreset, RenderSettings

    G, T, C = ref["geodesics"], ref["tracer"], ref["camera"]
    K = ref["KerrSpacetime"]
    arrs = {}

    def store(tag, res, state0, settings, esc, extra=None):
        arrs[f"{tag}_state0"] = state0
        arrs[f"{tag}_settings"] = np.array([settings.max_steps, settings.step_scale,
                                            settings.min_step, settings.max_step,
                                            settings.capture_margin, settings.momentum_bailout,
                                            esc])
        arrs[f"{tag}_status"] = res.status.astype(np.int8)
        arrs[f"{tag}_positions"] = res.positions
        arrs[f"{tag}_momenta"] = res.momenta
        if res.hit_radii is not None:
            arrs[f"{tag}_hit_radii"] = res.hit_radii
            arrs[f"{tag}_hit_positions"] = res.hit_positions
            arrs[f"{tag}_hit_momenta"] = res.hit_momenta
        for k, v in (extra or {}).items():
            arrs[f"{tag}_{k}"] = v

    def fan(st, offsets):
        n = offsets.shape[0]
        pos = np.tile([[30.0, 0.0, 0.0]], (n, 1))
        d = np.stack([-np.ones(n), offsets, np.zeros(n)], axis=-1)
        d /= np.linalg.norm(d, axis=-1, keepdims=True)
        return G.build_state(pos, G.null_momentum_from_velocity(st, pos, d, "past"))

    wide = np.linspace(0.03, 0.40, 300)
    wide = np.concatenate([wide, -wide])
    for spin, offsets, presets, tag in (
            (0.9, wide, list(QualityPreset), "a09"),
            (0.0, np.linspace(0.10, 0.25, 600), [QualityPreset.MEDIUM], "a0"),
            (0.998, wide, [QualityPreset.HIGH], "a0998"),
            (0.998, np.linspace(0.001, 0.15, 200), [QualityPreset.LOW], "plunge")):
        st = K(spin=spin)
        s0 = fan(st, offsets)
        truth = T.trace_rays(st, s0, escape_radius=60.0, rtol=1e-10)
        for preset in presets:
            settings = RenderSettings(spin=spin).apply_preset(preset)
            res = trace_like_shader(st, s0, settings, escape_radius=60.0)
            store(f"fan_{tag}_{preset.value}", res, s0, settings, 60.0,
                  {"spin": np.float64(spin), "truth_status": truth.status.astype(np.int8)})
    # Disk frame.
    st = K(spin=0.9)
    cam = C.PinholeCamera.from_orbit(30.0, 80.0, fov_degrees=40.0, width=48, height=36)
    pos = cam.ray_origins()
    s0 = G.build_state(pos, G.null_momentum_from_velocity(st, pos, cam.ray_directions(), "past"))
    settings = RenderSettings(spin=0.9).apply_preset(QualityPreset.MEDIUM)
    radii = (float(disk_inner_radius(st)), 18.0)
    res = trace_like_shader(st, s0, settings, escape_radius=100.0, disk_radii=radii)
    store("disk", res, s0, settings, 100.0, {"spin": np.float64(0.9), "disk": np.array(radii)})
    # Interior rain observers.
    for tag, spin, position in (("in19", 0.0, [1.9, 0.0, 0.0]), ("in05", 0.0, [0.5, 0.0, 0.0]),
                                ("in_a06", 0.6, [1.2, 0.3, 0.4])):
        st = K(spin=spin)
        p = np.array(position)
        u = frames.rain_four_velocity(st, p[None, :])[0]
        tetrad = frames.build_tetrad(st, p, u, -p / np.linalg.norm(p), np.array([0.0, 0.0, 1.0]))
        dirs = _fibonacci_sphere(400)
        mom = frames.tetrad_ray_momenta(st, p, tetrad, dirs)
        s0 = G.build_state(np.tile(p[None, :], (400, 1)), mom)
        settings = RenderSettings(spin=spin, disk_enabled=False).apply_preset(QualityPreset.HIGH)
        res = trace_like_shader(st, s0, settings, escape_radius=400.0, interior_stop=0.02)
        store(tag, res, s0, settings, 400.0,
              {"spin": np.float64(spin), "position": p, "four_velocity": u, "tetrad": tetrad,
               "directions": dirs})
    np.savez_compressed(os.path.join(out, "realtime.npz"), **arrs)


def gen_vaidya(ref, out):
    """vaidya.py (the charged-Vaidya/Ori surrogate) and the tracing loop of
    the mass-inflation renderer (offline/inflation.py:165-240):

    - the shell tables of three spacetimes: the default (q = 0.9), the
      flythrough one of tests/test_vaidya.py (shell at v = 6, R = 1.2) and
      the static limit (no tail, no shell);
    - geometry_t, mass_function / misner_sharp_mass and vaidya_geodesic_rhs
      at random points around the layer;
    - 3000 RK4 steps (h = 0.002) of the two rays of tests/test_vaidya.py;
    - two tiles of flythrough camera rays (rain observer at r = 1.3, v = 6 and
      at r = 0.8 inside the layer) traced by _trace_vaidya_tile."""
    _offline_modules(_REFERENCE_PATH)
    from blackhorizon import frames
    from blackhorizon.offline import inflation
    from blackhorizon.vaidya import ChargedVaidyaSpacetime, vaidya_geodesic_rhs

    I = ref["integrators"]
    arrs = {}
    specs = {"default": {}, "fly": {"shell_start_v": 6.0, "shell_start_radius": 1.2},
             "static": {"tail_mass": 0.0, "shell_energy": 0.0}}
    spaces = {}
    for tag, kw in specs.items():
        st = ChargedVaidyaSpacetime(charge=0.9, **kw)
        spaces[tag] = st
        arrs[f"{tag}_params"] = np.array([st.mass, st.charge, st.tail_mass, st.tail_start,
                                          st.tail_power, st.shell_energy, st.shell_start_v,
                                          st.shell_start_radius, st.shell_width, st.mass_cap])
        if st._shell_v.size <= 100000:
            arrs[f"{tag}_shell_v"] = st._shell_v
            arrs[f"{tag}_shell_r"] = st._shell_r
            arrs[f"{tag}_shell_m2"] = st._shell_m2
        else:
            # The static limit never reaches the mass cap and runs the full
            # 4e6 steps; its increment is zero, so keep the ends only.
            arrs[f"{tag}_shell_size"] = np.int64(st._shell_v.size)
            for k, a in (("v", st._shell_v), ("r", st._shell_r), ("m2", st._shell_m2)):
                arrs[f"{tag}_shell_{k}_ends"] = np.concatenate([a[:50], a[-50:]])
    rng = np.random.default_rng(51)
    n = 2000
    t = rng.uniform(0.0, 40.0, n)
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=-1, keepdims=True)
    pts = u * np.exp(rng.uniform(np.log(0.3), np.log(30.0), n))[:, None]
    p = rng.normal(size=(n, 4))
    states = np.concatenate([t[:, None], pts, p], axis=1)
    states = np.concatenate([states, np.array([[20.0, 0.9, 0.3, 0.2, -1.1, 0.4, -0.7, 0.5]])])
    arrs["sample_states"] = states
    for tag, st in spaces.items():
        g = st.geometry_t(states[:, 0], states[:, 1], states[:, 2], states[:, 3])
        arrs[f"{tag}_geo_h"] = g.h
        arrs[f"{tag}_geo_l"] = g.l
        arrs[f"{tag}_geo_hs"] = g.h_spatial_scale
        arrs[f"{tag}_geo_ht"] = g.h_t
        arrs[f"{tag}_geo_r"] = g.radius
        v = states[:, 0] + np.linalg.norm(states[:, 1:4], axis=-1)
        r = np.linalg.norm(states[:, 1:4], axis=-1)
        arrs[f"{tag}_mass"] = st.mass_function(v, r)
        arrs[f"{tag}_misner_sharp"] = st.misner_sharp_mass(v, r)
        arrs[f"{tag}_rhs"] = vaidya_geodesic_rhs(st, states)
    for tag, st, y0 in (("static", spaces["static"],
                         [[0.0, 5.0, 0.0, 0.0, 1.0, 0.0, 0.55, 0.0]]),
                        ("default", spaces["default"],
                         [[13.0, 3.0, 0.0, 0.5, 1.0, -0.9, 0.2, 0.1]])):
        y = np.array(y0)
        for _ in range(3000):
            y = I.rk4_step(lambda b, st=st: vaidya_geodesic_rhs(st, b), y, np.array([0.002]))
        arrs[f"{tag}_rk4_state0"] = np.array(y0)
        arrs[f"{tag}_rk4_final"] = y
    st = spaces["fly"]
    for tag, radius, time_ in (("tile_out", 1.3, 6.0), ("tile_in", 0.8, 9.0)):
        state = inflation.rain_state(st, np.array([radius, 0.0, 0.0]), time_)
        velocity = inflation.camera_four_velocity(st, state)
        slice_geo = st.frozen(float(state[0, 0]))
        pos = state[0, 1:4]
        outward = pos / np.linalg.norm(pos)
        tetrad = frames.build_tetrad(slice_geo, pos, velocity, outward,
                                     np.array([0.0, 0.0, 1.0]))
        dirs = _fibonacci_sphere(300)
        mom = frames.tetrad_ray_momenta(slice_geo, pos, tetrad, dirs)
        s0 = np.concatenate([np.full((300, 1), float(state[0, 0])), np.tile(pos, (300, 1)), mom],
                            axis=1)
        esc = max(12.0, 2.5 * radius)
        stop = st.inner_horizon_radius * 1.001
        status, edir, mass, v_end = inflation._trace_vaidya_tile(st, s0, esc, stop)
        arrs[f"{tag}_state0"] = s0
        arrs[f"{tag}_radii"] = np.array([esc, stop])
        arrs[f"{tag}_status"] = status.astype(np.int8)
        arrs[f"{tag}_escape_dir"] = edir
        arrs[f"{tag}_end_mass"] = mass
        arrs[f"{tag}_v_end"] = v_end
    np.savez_compressed(os.path.join(out, "vaidya.npz"), **arrs)


_REFERENCE_PATH = ""  # set from --reference


def main():
    global _REFERENCE_PATH
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True,
                    help="path of the reference project checkout (MegaKruk/BlackHorizon)")
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--procs", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--skip-c3", action="store_true")
    ap.add_argument("--only", default="", help="comma-separated step names to regenerate")
    args = ap.parse_args()
    _REFERENCE_PATH = args.reference
    sys.path.insert(0, args.reference)
    from blackhorizon import camera, geodesics, integrators, tracer
    from blackhorizon.kerr import KerrSpacetime

    ref = dict(KerrSpacetime=KerrSpacetime, geodesics=geodesics,
               integrators=integrators, tracer=tracer, camera=camera)
    steps = [
        ("geometry", lambda: gen_geometry(ref, args.out)),
        ("steps", lambda: gen_steps(ref, args.out)),
        ("camera", lambda: gen_camera(ref, args.out)),
        ("rk4", lambda: gen_rk4(ref, args.out)),
        ("fans", lambda: gen_fans(ref, args.out)),
        ("trace_c1", lambda: gen_trace_c1(ref, args.out)),
        ("raw_throughput", lambda: gen_raw_throughput(ref, args.out)),
        ("offline_tile", lambda: gen_offline_tile(ref, args.out)),
        ("offline_interior", lambda: gen_offline_interior(ref, args.out)),
        ("emission", lambda: gen_emission(ref, args.out)),
        ("inflation_frame", lambda: gen_inflation_frame(ref, args.out)),
        ("plunge", lambda: gen_plunge(ref, args.out)),
        ("video", lambda: gen_video(ref, args.out)),
        ("midpoint", lambda: gen_midpoint(ref, args.out)),
        ("images", lambda: gen_images(ref, args.out)),
        ("realtime", lambda: gen_realtime(ref, args.out)),
        ("vaidya", lambda: gen_vaidya(ref, args.out)),
    ]
    if not args.skip_c3:
        steps.append(("trace_c3", lambda: gen_trace_c3(ref, args.out, args.procs)))
    if args.only:
        keep = set(args.only.split(","))
        steps = [s for s in steps if s[0] in keep]
    timings = {}
    mpath = os.path.join(args.out, "MANIFEST.json")
    if args.only and os.path.exists(mpath):
        with open(mpath) as f:
            timings = json.load(f).get("seconds", {})
    for name, fn in steps:
        t0 = time.perf_counter()
        fn()
        timings[name] = round(time.perf_counter() - t0, 2)
        print(f"{name}: {timings[name]} s", flush=True)
    manifest = {
        "command": "python tests/golden/make_golden.py --reference <path>",
        "reference_sha256": {f: sha256(os.path.join(args.reference, f)) for f in REF_FILES},
        "numpy": np.__version__,
        "seconds": timings,
        "files": sorted(f for f in os.listdir(args.out) if f.endswith(".npz")),
    }
    with open(os.path.join(args.out, "MANIFEST.json"), "w") as f:
        json.dump(manifest, f, indent=1)


if __name__ == "__main__":
    main()
