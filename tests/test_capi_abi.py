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


def test_status_strings(bhlib):
    assert bhlib.bh_abi_version() == 1
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


def test_check_maps_status_to_reference_exceptions(bhlib):
    from blackhorizon_b200 import _lib

    with pytest.raises(ValueError):
        _lib.check(-1)
    with pytest.raises(ValueError):
        _lib.check(-4)
    with pytest.raises(RuntimeError):
        _lib.check(-3)
