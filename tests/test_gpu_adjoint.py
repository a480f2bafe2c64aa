"""The path-replay adjoint (ct_adjoint_forward / ct_adjoint_backward)
through the C ABI, against its oracle, finite differences, and an
optimisation run.

  * forward, bit for bit: the CUDA image of a crop against the oracle's
    float32 restatement on paths the oracle traced with the reference's own
    intersect() / compute_ray_origin / random_cosine_direction
    (oracle/adjoint_ref.py);
  * gradients against the FP64 oracle on the same paths, for a random
    image derivative;
  * the gradient of the L2 image loss on the differentiation workload
    (128^3 grid at 25% occupancy, 1% emitters, 512x512, 64 spp, depth 3)
    against central finite differences (eps 1e-3, image accumulated in
    float64) on 64 parameters of voxels the camera sees, to 1e-3 relative;
  * 200 Adam steps (lr 1e-2) from albedo 0.5 and radiance 5 towards a
    target rendered from hidden parameters with other sample streams: the
    loss must fall.

RenderFn, the torch.autograd.Function below, exists only in this harness:
the library's interface is the C ABI pair."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS = 1e-3
FD_RTOL = 1e-3


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch


def _small():
    from cube_tracing import adjoint
    a = adjoint.adjoint_scene(edge=32, occupancy=0.25, emissive_fraction=0.05, width=64, height=64)
    return a, (12, 10, 52, 50)


def test_forward_matches_oracle_bit_for_bit(oracle_lib):
    torch = _torch()
    import adjoint_ref as ar
    from cube_tracing import adjoint
    a, rect = _small()
    r = adjoint.AdjointRenderer(a, spp=8, max_depth=3, seed=7)
    alb = torch.from_numpy(a.albedo_target).cuda()
    em = torch.from_numpy(a.emission_target).cuda()
    img = r.forward(alb, em, rect=rect).cpu().numpy()
    x0, y0, x1, y1 = rect
    v = ar.paths(a.scene, a.inv_view, a.inv_proj, a.width, a.height, 8, 3, 7, rect)
    want = ar.forward32(v, a.albedo_target, a.emission_target, a.emitter_index).reshape(y1 - y0, x1 - x0, 3)
    got = img[y0:y1, x0:x1]
    assert (want > 0).mean() > 0.05  # some paths reach an emitter
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), \
        f"{int((got != want).any(-1).sum())} pixels differ, max {np.abs(got - want).max()}"
    outside = img.copy()
    outside[y0:y1, x0:x1] = 0
    assert not outside.any()
    r.close()


def test_gradient_matches_fp64_oracle(oracle_lib):
    torch = _torch()
    import adjoint_ref as ar
    from cube_tracing import adjoint
    a, rect = _small()
    r = adjoint.AdjointRenderer(a, spp=8, max_depth=3, seed=7)
    x0, y0, x1, y1 = rect
    rng = np.random.default_rng(5)
    d_img = np.zeros((a.height, a.width, 3), np.float32)
    d_img[y0:y1, x0:x1] = rng.standard_normal((y1 - y0, x1 - x0, 3)).astype(np.float32)
    ga, ge = r.backward(torch.from_numpy(a.albedo_target).cuda(), torch.from_numpy(a.emission_target).cuda(),
                        torch.from_numpy(d_img).cuda(), rect=rect)
    ga, ge = ga.cpu().numpy().astype(np.float64), ge.cpu().numpy().astype(np.float64)
    v = ar.paths(a.scene, a.inv_view, a.inv_proj, a.width, a.height, 8, 3, 7, rect)
    wa, we = ar.backward64(v, a.albedo_target, a.emission_target, a.emitter_index,
                           d_img[y0:y1, x0:x1].reshape(-1, 3))
    for got, want, what in ((ga, wa, "albedo"), (ge, we, "emission")):
        assert np.abs(want).max() > 0, what
        scale = np.abs(want).max()
        bad = np.abs(got - want) > 1e-4 * np.abs(want) + 1e-6 * scale
        assert not bad.any(), f"{what}: {int(bad.sum())} entries off, e.g. {got[bad][:3]} vs {want[bad][:3]}"
        assert np.array_equal(got != 0, want != 0), what
    r.close()


def _render_fn():
    import torch

    class RenderFn(torch.autograd.Function):
        """image = render(albedo, emission); backward by path replay."""

        @staticmethod
        def forward(ctx, albedo, emission, renderer):
            ctx.save_for_backward(albedo, emission)
            ctx.renderer = renderer
            return renderer.forward(albedo.detach(), emission.detach())

        @staticmethod
        def backward(ctx, grad_image):
            albedo, emission = ctx.saved_tensors
            ga, ge = ctx.renderer.backward(albedo.detach(), emission.detach(), grad_image)
            return ga, ge, None

    return RenderFn


@pytest.fixture(scope="module")
def workload():
    torch = _torch()
    from cube_tracing import adjoint
    a = adjoint.adjoint_scene()
    r = adjoint.AdjointRenderer(a, spp=64, max_depth=3, seed=1)
    # the target: hidden parameters, other sample streams
    rt = adjoint.AdjointRenderer(a, spp=64, max_depth=3, seed=1001)
    target = rt.forward(torch.from_numpy(a.albedo_target).cuda(), torch.from_numpy(a.emission_target).cuda())
    rt.close()
    yield a, r, target
    r.close()


def test_gradient_matches_central_differences(workload):
    torch = _torch()
    a, r, target = workload
    RenderFn = _render_fn()
    alb = torch.from_numpy(a.albedo_init).cuda().requires_grad_(True)
    em = torch.from_numpy(a.emission_init).cuda().requires_grad_(True)
    img = RenderFn.apply(alb, em, r)
    loss = ((img - target) ** 2).sum()
    loss.backward()
    ga, ge = alb.grad.cpu().numpy(), em.grad.cpu().numpy()
    rng = np.random.default_rng(11)
    seen_a = np.nonzero(np.abs(ga).max(1) > 0)[0]
    seen_e = np.nonzero(np.abs(ge).max(1) > 0)[0]
    assert seen_a.size > 1000 and seen_e.size > 10
    picks = [("albedo", int(i), int(rng.integers(3))) for i in rng.choice(seen_a, 48, replace=False)]
    picks += [("emission", int(i), int(rng.integers(3))) for i in rng.choice(seen_e, 16, replace=False)]
    tgt = target.double()

    def loss64(al, e):
        im = r.forward(al, e, f64=True)
        return float(((im - tgt) ** 2).sum())

    a0, e0 = alb.detach().clone(), em.detach().clone()
    rel = []
    for what, i, c in picks:
        plus_a, minus_a, plus_e, minus_e = a0.clone(), a0.clone(), e0.clone(), e0.clone()
        if what == "albedo":
            plus_a[i, c] += EPS
            minus_a[i, c] -= EPS
            adj = float(ga[i, c])
        else:
            plus_e[i, c] += EPS
            minus_e[i, c] -= EPS
            adj = float(ge[i, c])
        # the perturbed parameter as the float32 the kernel reads
        h = (float(plus_a[i, c] - minus_a[i, c]) if what == "albedo" else float(plus_e[i, c] - minus_e[i, c]))
        fd = (loss64(plus_a, plus_e) - loss64(minus_a, minus_e)) / h
        rel.append(abs(adj - fd) / max(abs(fd), 1e-30))
    rel = np.array(rel)
    print(f"central differences, 64 parameters: median rel {np.median(rel):.2e}, max {rel.max():.2e}")
    assert (rel <= FD_RTOL).all(), list(zip(picks, rel))


def test_adam_reduces_loss(workload):
    torch = _torch()
    a, r, target = workload
    RenderFn = _render_fn()
    alb = torch.from_numpy(a.albedo_init).cuda().requires_grad_(True)
    em = torch.from_numpy(a.emission_init).cuda().requires_grad_(True)
    opt = torch.optim.Adam([alb, em], lr=1e-2)
    losses = []
    for step in range(200):
        opt.zero_grad()
        img = RenderFn.apply(alb, em, r)
        loss = ((img - target) ** 2).sum()
        loss.backward()
        opt.step()
        with torch.no_grad():
            alb.clamp_(0.0, 1.0)
            em.clamp_(min=0.0)
        losses.append(float(loss))
    print(f"Adam: loss {losses[0]:.4g} -> {losses[-1]:.4g} after 200 steps")
    assert np.isfinite(losses).all()
    assert losses[-1] < 0.5 * losses[0]
