"""The adjoint's oracle on the CPU (no GPU): its FP64 gradient restatement
(oracle/adjoint_ref.py) against central differences of its own FP64
forward, on paths traced by the reference's shader functions; the paths do
not depend on the number of host threads; and the float32 forward stays
within float rounding of the float64 one."""
import numpy as np

import adjoint_ref as ar
from cube_tracing import adjoint


def _paths(threads=0):
    a = adjoint.adjoint_scene(edge=32, occupancy=0.25, emissive_fraction=0.05, width=64, height=64)
    v = ar.paths(a.scene, a.inv_view, a.inv_proj, 64, 64, 4, 3, 1, (16, 16, 48, 48), threads=threads)
    return a, v


def test_paths_do_not_depend_on_threads(oracle_lib):
    _, v = _paths()
    _, v1 = _paths(threads=1)
    assert np.array_equal(v, v1)
    assert (v[:, :, 0] != ar.NONE).all()          # the camera sees the grid everywhere in the crop
    assert (v[:, :, 1] != ar.NONE).mean() > 0.2   # and bounces find more voxels


def test_fp64_gradient_matches_central_differences(oracle_lib):
    a, v = _paths()
    alb, em = a.albedo_target.astype(np.float64), a.emission_target.astype(np.float64)
    rng = np.random.default_rng(0)
    d_img = rng.standard_normal((v.shape[0], 3))
    ga, ge = ar.backward64(v, alb, em, a.emitter_index, d_img)

    def loss(al, e):
        return float((ar.forward64(v, al, e, a.emitter_index) * d_img).sum())

    eps = 1e-6
    for i in rng.choice(np.nonzero(np.abs(ga).max(1) > 0)[0], 6, replace=False):
        c = int(rng.integers(3))
        p, m = alb.copy(), alb.copy()
        p[i, c] += eps
        m[i, c] -= eps
        fd = (loss(p, em) - loss(m, em)) / (2 * eps)
        assert abs(fd - ga[i, c]) <= 1e-6 * abs(ga[i, c]) + 1e-12
    for i in rng.choice(np.nonzero(np.abs(ge).max(1) > 0)[0], 4, replace=False):
        c = int(rng.integers(3))
        p, m = em.copy(), em.copy()
        p[i, c] += eps
        m[i, c] -= eps
        fd = (loss(alb, p) - loss(alb, m)) / (2 * eps)
        assert abs(fd - ge[i, c]) <= 1e-6 * abs(ge[i, c]) + 1e-12


def test_float32_forward_within_rounding(oracle_lib):
    a, v = _paths()
    f32 = ar.forward32(v, a.albedo_target, a.emission_target, a.emitter_index).astype(np.float64)
    f64 = ar.forward64(v, a.albedo_target, a.emission_target, a.emitter_index)
    assert np.abs(f32 - f64).max() <= 1e-5 * max(np.abs(f64).max(), 1.0)
