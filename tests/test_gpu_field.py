"""The walk's cell field as the GPU builds it (ct_build_accel: Jacobi sweeps,
the grow pass to 30 cells, 4-bit codes) against the CPU restatement in
fieldref.py, cell by cell for every ray octant.  A field that overstated one
cube would let a walk skip an occupied cell; the traversal tests see that
only where a ray crosses it, this test everywhere."""
import numpy as np
import pytest

import fieldref
from cases import build_case
from cube_tracing import scenes


def _scene(name):
    if name == "terrain40":  # open sky above the surface: edges up to 30
        return scenes.heightfield_scene(40, base=10.0, amplitude=6.0, emissive_fraction=0.02, seed=9)
    if name == "sparse24":  # isolated voxels: every edge class
        return scenes.random_grid_scene(24, 0.02, emissive_fraction=0.1, seed=4)
    return build_case(name)[0]


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["terrain40", "sparse24", "grid16", "instances16"])
def test_field_matches_restatement(name):
    from cube_tracing.frame import SceneBuffers
    sc = _scene(name)
    sb = SceneBuffers(sc)
    assert sb.accel.info().grid_exact == 1
    n_inst = sc.instances.shape[0]
    seen = set()
    for inst in sorted({0, n_inst - 1}):
        for octant in range(8):
            got, gmin = sb.accel.field(inst, octant)
            occ = fieldref.grid_occupancy(sc, inst, gmin, got.shape)
            want = fieldref.coded_edges(occ, octant)
            bad = np.argwhere(got != want)
            assert len(bad) == 0, (f"instance {inst} octant {octant}: {len(bad)} cells differ, first "
                                   f"[z,y,x]={bad[0].tolist()} got {got[tuple(bad[0])]} want {want[tuple(bad[0])]}")
            seen.update(np.unique(got).tolist())
    if name == "terrain40":
        assert 30 in seen and 19 in seen  # the grow pass ran


@pytest.mark.gpu
def test_field_arguments_checked():
    import ctypes
    from cube_tracing import native
    from cube_tracing.frame import SceneBuffers
    sb = SceneBuffers(build_case("instances16")[0])
    lib = native.lib()
    g, c = (ctypes.c_int32 * 3)(), (ctypes.c_uint32 * 3)()
    n = sb.n_instances
    assert lib.ct_accel_field(sb.accel.handle, n - 1, 7, None, ctypes.byref(g), ctypes.byref(c), None) == 0
    assert c[0] % 8 == 0 and c[1] % 8 == 0 and c[2] % 8 == 0
    assert lib.ct_accel_field(sb.accel.handle, n, 0, None, ctypes.byref(g), ctypes.byref(c), None) == 1
    assert lib.ct_accel_field(sb.accel.handle, 0, 8, None, ctypes.byref(g), ctypes.byref(c), None) == 1
    assert lib.ct_accel_field(sb.accel.handle, 0, 0, None, None, ctypes.byref(c), None) == 1
