"""The C ABI without a GPU: the library loads, exports every symbol that
include/bh_b200.h declares, its struct layouts match the ctypes mirror, and
argument validation answers before any CUDA call."""

import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "bh_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bh_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported(bhlib):
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(bhlib, n)]
    assert not missing, f"not exported: {missing}"


def test_python_binding_covers_header(bhlib):
    from blackhorizon_b200 import _lib

    assert set(declared_functions()) <= set(_lib.exported_symbols())


def test_struct_layouts_match_header(tmp_path):
    from blackhorizon_b200 import _lib

    probe = tmp_path / "probe.c"
    probe.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "bh_b200.h"\n'
        "int main(void){\n"
        'printf("%zu %zu %zu %zu\\n", sizeof(bh_trace_config), sizeof(bh_camera),'
        " sizeof(bh_scene), sizeof(bh_trace_stats));\n"
        'printf("%zu %zu %zu %zu\\n", offsetof(bh_trace_config, precision),'
        " offsetof(bh_trace_config, timeout_ns), offsetof(bh_camera, scene),"
        " offsetof(bh_trace_stats, bad_rays));\n"
        'printf("%zu %zu\\n", sizeof(bh_tile_stats), offsetof(bh_tile_stats, rounds));\n'
        'printf("%zu\\n", offsetof(bh_trace_config, f64_radius));\n'
        "return 0;}\n"
    )
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(probe), "-o", str(exe)],
                   check=True)
    lines = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    sizes = [int(v) for v in lines[0].split()]
    offs = [int(v) for v in lines[1].split()]
    assert sizes == [ctypes.sizeof(_lib.TraceConfig), ctypes.sizeof(_lib.Camera),
                     ctypes.sizeof(_lib.Scene), ctypes.sizeof(_lib.TraceStats)]
    assert offs == [_lib.TraceConfig.precision.offset, _lib.TraceConfig.timeout_ns.offset,
                    _lib.Camera.scene.offset, _lib.TraceStats.bad_rays.offset]
    tile = [int(v) for v in lines[2].split()]
    assert tile == [ctypes.sizeof(_lib.TileStats), _lib.TileStats.rounds.offset]
    assert int(lines[3]) == _lib.TraceConfig.f64_radius.offset


def test_status_strings(bhlib):
    assert bhlib.bh_abi_version() == 5
    assert bhlib.bh_status_string(0) == b"ok"
    assert b"escape_radius" in bhlib.bh_status_string(-4)
    assert bhlib.bh_trace_workspace_bytes() == 256
    assert bhlib.bh_trace_cameras_workspace_bytes(64) % 256 == 0


@pytest.mark.parametrize("mass,spin", [(1.0, 1.01), (-1.0, 0.0), (0.0, 0.0)])
def test_kerr_bound_rejected_before_launch(bhlib, mass, spin):
    # kerr.py:65-71 raises ValueError; the ABI returns BH_ERR_INVALID_ARGUMENT.
    assert bhlib.bh_geodesic_rhs(mass, spin, None, None, 1, None) == -1
    assert b"Kerr" in bhlib.bh_last_error() or b"mass" in bhlib.bh_last_error()


def test_trace_argument_validation(bhlib):
    from blackhorizon_b200 import _lib

    scene = _lib.Scene(1.0, 0.9, 1.45, 100.0)
    assert bhlib.bh_trace(None, scene, None, None, None, None, 1, None, None) == -1
    cfg = _lib.TraceConfig(5000, 1e-8, 1e-10, 0.1, 2.0, 1e-10, 7, 0, 0, -1, 0)
    assert bhlib.bh_trace(cfg, scene, None, None, None, None, 1, None, None) == -1
    assert b"precision" in bhlib.bh_last_error()
    cfg = _lib.TraceConfig(0, 1e-8, 1e-10, 0.1, 2.0, 1e-10, 0, 0, 0, -1, 0)
    assert bhlib.bh_trace(cfg, scene, None, None, None, None, 1, None, None) == -1
    cfg = _lib.TraceConfig(10, 1e-8, 1e-10, 0.1, 2.0, 1e-10, 0, 0, 0, -1, 0)
    # No workspace: reported before any CUDA call.
    assert bhlib.bh_trace(cfg, scene, None, None, None, None, 1, None, None) == -5


def test_projection_config_validation(bhlib):
    """A negative projection period, and projection on a taped trace (the
    adjoint replays unprojected steps), are rejected before any CUDA call."""
    import ctypes as C

    from blackhorizon_b200 import _lib

    scene = _lib.Scene(1.0, 0.9, 1.45, 100.0)
    cfg = _lib.TraceConfig(5000, 1e-8, 1e-10, 0.1, 2.0, 1e-10, 0, 0, 0, -1, 0, -1, 0)
    assert bhlib.bh_trace(cfg, scene, None, None, None, None, 1, None, None) == -1
    assert b"project_every" in bhlib.bh_last_error()
    cfg.project_every = 4
    fake = C.c_void_p(0x10000)
    assert bhlib.bh_trace_tape(cfg, scene, fake, fake, fake, fake, 1, fake, fake, 16, 8,
                               fake, None) == -1
    assert b"taped" in bhlib.bh_last_error()


def test_trace_tile_argument_validation(bhlib):
    """bh_trace_tile rejects malformed calls before any CUDA call."""
    import ctypes as C

    from blackhorizon_b200 import _lib

    scene = _lib.Scene(1.0, 0.9, 1.44, 34.0)
    cfg = _lib.TraceConfig(12000, 1e-9, 1e-12, 0.1, 2.0, 0.0, 0, 0, 0, -1, 0)
    st = _lib.TileStats()
    fake = C.c_void_p(0x10000)  # never dereferenced: validation fails first
    args = [fake] * 8

    def call(cfg, r_in, r_out, n, ws=None, wsb=0):
        return bhlib.bh_trace_tile(cfg, scene, r_in, r_out, fake, n, *args[:7], ws, wsb, st,
                                   None)

    assert call(None, 2.3, 18.0, 4) == -1
    bad = _lib.TraceConfig(0, 1e-9, 1e-12, 0.1, 2.0, 0.0, 0, 0, 0, -1, 0)
    assert call(bad, 2.3, 18.0, 4) == -1
    assert call(cfg, 20.0, 18.0, 4) == -1  # inner > outer
    assert b"disk" in bhlib.bh_last_error()
    assert call(cfg, 2.3, 18.0, -1) == -1
    assert call(cfg, 2.3, 18.0, 0) == 0  # empty tile: nothing to do
    assert call(cfg, 2.3, 18.0, 4) == -5  # no workspace
    assert call(cfg, 2.3, 18.0, 4, C.c_void_p(0x10000), 100) == -5  # too small
    # Header, resume-sort counters, n parked and min(n / 8 + 1024, n)
    # speculative 176-byte crossing records, two 96-byte resume records, an
    # 8-byte first hit and a 1-byte flag per ray (rounded up to 16 bytes).
    for n in (10, 100_000):
        spec = min(n // 8 + 1024, n)
        assert bhlib.bh_trace_tile_workspace_bytes(n) == (
            256 + 1024 + (n + spec) * 176 + n * (2 * 96 + 8) + (n + 15) // 16 * 16)
    # Config flags: BH_TRACE_INTERIOR only, and only with a stop radius > 0.
    cfg.flags = 2
    assert call(cfg, 2.3, 18.0, 4) == -1
    assert b"flags" in bhlib.bh_last_error()
    cfg.flags = _lib.TRACE_INTERIOR
    scene.capture_radius = 0.0
    assert call(cfg, 2.3, 18.0, 4) == -1
    assert b"stop" in bhlib.bh_last_error()
    scene.capture_radius = 0.02
    assert call(cfg, 2.3, 18.0, 4) == -5  # valid interior call: workspace next
    # The other tracers take no flags.
    assert bhlib.bh_trace(cfg, scene, None, None, None, None, 1, None, None) == -1
    assert b"flags" in bhlib.bh_last_error()


def test_f64_band_config_validation(bhlib):
    """The float64 band radius belongs to bh_propagate: the tracers reject a
    nonzero one, and propagate rejects NaN and the band with projection,
    all before any CUDA call."""
    import ctypes as C

    from blackhorizon_b200 import _lib
    from blackhorizon_b200.integrators import make_config

    scene = _lib.Scene(1.0, 0.9, 1.45, 100.0)
    cfg = make_config(5000, 1e-8, 1e-10, 0.1, 2.0, 1e-10, "mixed", f64_radius=50.0)
    assert cfg.f64_radius == 50.0
    assert bhlib.bh_trace(cfg, scene, None, None, None, None, 1, None, None) == -1
    assert b"f64_radius" in bhlib.bh_last_error()
    fake = C.c_void_p(0x10000)  # never dereferenced: validation fails first
    st = _lib.TileStats()
    assert bhlib.bh_trace_tile(cfg, scene, 2.3, 18.0, fake, 4, *[fake] * 7, None, 0, st,
                               None) == -1
    assert b"f64_radius" in bhlib.bh_last_error()
    assert make_config(f64_radius="auto").f64_radius == -1.0
    with pytest.raises(ValueError):
        make_config(f64_radius=-2.0)
    with pytest.raises(ValueError):
        make_config(f64_radius="inner")
    nan = make_config(1, 1e-8, 1e-10, precision="mixed")
    nan.f64_radius = float("nan")
    assert bhlib.bh_propagate(nan, 1.0, 0.9, None, fake, fake, None, fake, 4, 10, fake,
                              None) == -1
    assert b"NaN" in bhlib.bh_last_error()
    both = make_config(1, 1e-8, 1e-10, precision="mixed", project_every=2, f64_radius=40.0)
    assert bhlib.bh_propagate(both, 1.0, 0.9, None, fake, fake, None, fake, 4, 10, fake,
                              None) == -1
    assert b"project_every" in bhlib.bh_last_error()
    assert bhlib.bh_device_math(3, fake, fake, 4, None) == -1


def test_check_maps_status_to_reference_exceptions(bhlib):
    from blackhorizon_b200 import _lib

    with pytest.raises(ValueError):
        _lib.check(-1)
    with pytest.raises(ValueError):
        _lib.check(-4)
    with pytest.raises(RuntimeError):
        _lib.check(-3)


def test_propagate_order_argument_validation(bhlib):
    """bh_propagate_order checks its layout, size, pointers and workspace
    alignment before any CUDA call; its workspace covers two 64-bit key
    arrays, an int32 index array and the sort's temporary storage."""
    import ctypes as C

    fake = C.c_void_p(0x10000)  # never dereferenced: validation fails first
    assert bhlib.bh_propagate_order(fake, 2, 4, fake, None, 0, None) == -1
    assert b"layout" in bhlib.bh_last_error()
    assert bhlib.bh_propagate_order(fake, 0, -1, fake, None, 0, None) == -1
    assert bhlib.bh_propagate_order(fake, 0, 0, fake, None, 0, None) == 0
    assert bhlib.bh_propagate_order(None, 0, 4, fake, None, 0, None) == -1
    assert bhlib.bh_propagate_order(fake, 0, 4, fake, None, 0, None) == -5
    assert bhlib.bh_propagate_order(fake, 0, 4, fake, C.c_void_p(0x10010), 1 << 20, None) == -5
    # Sizing the sort needs a CUDA device; without one the size is 0.
    need = bhlib.bh_propagate_order_workspace_bytes(100_000)
    if need:
        assert need % 256 == 0 and need >= 100_000 * (8 + 8 + 4)
        assert bhlib.bh_propagate_order(fake, 0, 100_000, fake, fake, need - 1, None) == -5
    assert bhlib.bh_propagate_order_workspace_bytes(1 << 31) == 0

