"""Struct layouts and the C ABI surface (no GPU needed)."""
import ctypes
import os
import re

from cube_tracing import layouts as L
from cube_tracing import native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_numpy_layouts_match_reference_sizes():
    for name, size in L.SIZES.items():
        assert getattr(L, name).itemsize == size, name


def test_oracle_sees_the_same_layouts(oracle_lib):
    i = oracle_lib.info()
    assert (i.instance, i.aabb, i.primitive, i.material, i.light, i.light_config) == (72, 24, 8, 84, 40, 52)
    assert (i.reservoir, i.di_info, i.velocity, i.path_reservoir) == (36, 60, 8, 92)
    assert (i.camera_view, i.status, i.world, i.restir, i.push_constant) == (264, 96, 96, 72, 88)


def test_ctypes_structs_match_header():
    assert ctypes.sizeof(native.PushConstant) == 88
    assert ctypes.sizeof(native.SceneDesc) == 32
    assert ctypes.sizeof(native.ErrorInfo) == 16
    assert ctypes.sizeof(native.AdjointDesc) == 72
    assert ctypes.sizeof(native.NrcFrame) == 72


def declared_functions():
    src = open(os.path.join(ROOT, "include", "ct.h")).read()
    return sorted(set(re.findall(r"^\s*(?:ct_status|uint32_t|const char \*|void)\s+\*?(ct_\w+)\s*\(", src, re.M)))


def test_library_exports_every_declared_entry_point():
    lib = native.lib()
    names = declared_functions()
    assert "ct_build_accel" in names and "ct_render_frame" in names
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) <= set(native.exported_symbols())


def test_abi_version_and_defaults():
    lib = native.lib()
    assert lib.ct_abi_version() == 1
    p = native.default_params()
    assert p.struct_size == ctypes.sizeof(native.Params)
    # reference constants: defines.glsl:34-48, shared.inl:45, taa.glsl:13
    assert (p.min_ris_cube_samples, p.max_ris_cube_samples) == (4, 32)
    assert (p.min_num_of_neighbors, p.max_num_of_neighbors) == (3, 4)
    assert abs(p.voxel_extent - 0.03125) == 0 and abs(p.taa_alpha - 0.8) < 1e-7
    assert p.spatial_passes == 1
    assert lib.ct_status_string(0) == b"ok"


def test_cpp_host_check_program_is_built():
    """The C++ host side's check program links against libct.so and answers
    a wrong command line without touching a device."""
    import subprocess
    prog = os.path.join(ROOT, "cube-tracing_b200", "host", "ct_host_check")
    assert os.path.exists(prog)
    r = subprocess.run([prog], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "usage" in r.stderr


def test_cpp_host_rejects_an_empty_scene(tmp_path):
    """ct::Renderer checks its scene before any device call: a scene without
    instances is refused with CT_ERR_INVALID_ARG."""
    import subprocess
    import numpy as np
    import hostcpp
    from cases import build_case
    sc, W, H, cams, kw = build_case("grid16")
    sc.instances = sc.instances[:0]
    inp, outp = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    hostcpp.write_input(inp, sc, W, H, cams, native.default_params(voxel_extent=1.0), L.RIS_CUBE_LIGHT_BIT, 3)
    r = subprocess.run([hostcpp.PROGRAM, inp, outp], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and "invalid argument" in r.stderr, r.stderr
    assert not os.path.exists(outp)
