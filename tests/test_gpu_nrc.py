"""The neural radiance cache's fused MLP (ct_nrc_encode / ct_nrc_infer /
ct_nrc_infer_encoded: tcgen05.mma with fp32 accumulators in tensor memory,
bf16 weights and activations) against a plain PyTorch fp32 reference of the
same network, through the C ABI.

  * the encoding against its torch restatement, to bf16 rounding;
  * the network on the kernel's own encoded inputs against the fp32
    reference that rounds inputs, weights and hidden activations to bf16
    where the kernel does (the remaining difference is the summation order
    of fp32 accumulation), on a query count that leaves a partial tile;
  * encoding and network fused against the fp32 reference on torch's
    encoding;
  * a few Adam steps on a fixed target reduce the cache's error.
No tensor-core wait may run out (ct_nrc_status stays 0)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 5000 + 77  # 40 full tiles of 128 and a partial one


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch


def _cache():
    from cube_tracing import nrc
    return nrc.NrcCache((0.0, 0.0, 0.0), (256.0, 128.0, 256.0), seed=3)


def test_encoding_matches_restatement():
    torch = _torch()
    from cube_tracing import nrc
    c = _cache()
    q = nrc.random_queries(N, seed=1)
    got = c.encode_device(q).float()
    want = nrc.encode(q, c.bbox_min, c.bbox_extent)
    err = (got - want).abs()
    # bf16 keeps 8 significant bits: half an ulp of a value up to 1 is 2^-9
    assert err.max().item() <= 2.0 ** -8 + 1e-6, err.max().item()
    assert (got[:, 227:] == 0).all()
    assert nrc.status() == 0


def test_mlp_matches_fp32_reference_on_encoded_inputs():
    torch = _torch()
    from cube_tracing import nrc
    c = _cache()
    q = nrc.random_queries(N, seed=2)
    enc = c.encode_device(q)
    got = c.infer_encoded(enc)
    torch.cuda.synchronize()
    assert nrc.status() == 0
    with torch.no_grad():
        want = c.mlp(enc.float(), round_bf16=True)[:, :3]
    scale = want.abs().max().item()
    assert scale > 1e-3
    err = (got - want).abs()
    # fp32 sums in another order can flip a bf16 rounding of a hidden value
    assert err.max().item() <= 2e-2 * scale, (err.max().item(), scale)
    assert err.mean().item() <= 2e-3 * scale, (err.mean().item(), scale)


def test_fused_encoding_and_mlp_match_fp32_reference():
    torch = _torch()
    from cube_tracing import nrc
    c = _cache()
    q = nrc.random_queries(N, seed=3)
    got = c.infer(q)
    torch.cuda.synchronize()
    assert nrc.status() == 0
    with torch.no_grad():
        want = c.mlp(nrc.encode(q, c.bbox_min, c.bbox_extent))[:, :3]
    scale = want.abs().max().item()
    err = (got - want).abs()
    assert err.max().item() <= 5e-2 * scale, (err.max().item(), scale)
    assert err.mean().item() <= 1e-2 * scale, (err.mean().item(), scale)


def test_training_reduces_the_error():
    torch = _torch()
    from cube_tracing import nrc
    c = _cache()
    q = nrc.random_queries(1 << 14, seed=4)
    # a smooth radiance field of the position and albedo
    target = (q[:, 9:12] * (1.0 + torch.sin(q[:, 0:1] / 40.0))).contiguous()

    def rel_err():
        pred = c.infer(q)
        return float((((pred - target) ** 2).sum(1) / ((target ** 2).sum(1) + 1e-2)).mean())

    before = rel_err()
    for _ in range(200):
        c.train_step(q, target)
    after = rel_err()
    assert after < 0.25 * before, (before, after)
    assert nrc.status() == 0


def _tracer(max_depth=2):
    from cube_tracing import adjoint
    a = adjoint.adjoint_scene(edge=32, occupancy=0.25, emissive_fraction=0.05, width=64, height=48)
    return a, adjoint.AdjointRenderer(a, spp=1, max_depth=max_depth, seed=11)


@pytest.mark.parametrize("cache_vertex", [1, 2])
def test_cache_trace_matches_the_plain_tracer_up_to_the_cache_vertex(cache_vertex):
    """ct_nrc_trace's radiance before the cache vertex v_c is the plain
    tracer's image of c vertices bit for bit (same sample stream, no miss
    light), its throughput is the product of the albedos before v_c, and
    every pixel whose path reaches v_c has a query there."""
    torch = _torch()
    from cube_tracing import nrc
    a, t = _tracer(max_depth=cache_vertex)
    alb = torch.from_numpy(a.albedo_target).cuda()
    em = torch.from_numpy(a.emission_target).cuda()
    cache = nrc.NrcCache((0.0, 0.0, 0.0), (32.0, 32.0, 32.0))
    r = nrc.NrcRenderer(t, cache, train_paths=256, train_bounces=4, cache_vertex=cache_vertex)
    r.trace(11)
    plain2 = t.forward(alb, em, spp=1).reshape(-1, 3)
    torch.cuda.synchronize()
    assert torch.equal(r.base.view(torch.int32), plain2.contiguous().view(torch.int32))
    reached = r.query[:, 9] >= 0.0
    assert 0.05 < float(reached.float().mean()) < 1.0
    assert (r.thp[~reached] == 0).all() and (r.thp[reached] > 0).any()
    assert (r.query[reached, 9:12] <= 1.0).all()
    # training vertices: partial radiance and throughput are finite, unreached ones marked
    assert torch.isfinite(r.tpart).all() and torch.isfinite(r.tthp).all()
    assert (r.tq[:, :, 9] >= 0.0).any()


def test_cache_renderer_trains_online():
    """After 60 frames of online training, the cache's frames are closer to
    a 4096-spp image of the plain tracer than the plain tracer's own
    one-sample frames are (relMSE over pixels and channels)."""
    torch = _torch()
    from cube_tracing import nrc
    a, t = _tracer()
    t.max_depth = 8
    t.miss_radiance = 0.5
    alb = torch.from_numpy(a.albedo_target).cuda()
    em = torch.from_numpy(a.emission_target).cuda()
    t.seed = 90001
    ref = t.forward(alb, em, spp=4096).double()

    def relmse(img):
        return float((((img.double() - ref) ** 2) / (ref * ref + 1e-2)).mean())

    plain = []
    for k in range(10):
        t.seed = 500 + k
        plain.append(relmse(t.forward(alb, em, spp=1)))
    cache = nrc.NrcCache((0.0, 0.0, 0.0), (32.0, 32.0, 32.0), lr=1e-3)
    r = nrc.NrcRenderer(t, cache, train_paths=1024, train_bounces=4, min_frames=20, batch=4096)
    errs = []
    for f in range(60):
        img, (loss, n) = r.render(100 + f)
        assert n > 0 and np.isfinite(loss)
        errs.append(relmse(img))
    torch.cuda.synchronize()
    print(f"relMSE: plain 1 spp {np.mean(plain):.4f}, cache frames {np.mean(errs[-10:]):.4f}; "
          f"{r.fallbacks} plain frames")
    assert torch.isfinite(img).all()
    assert r.fallbacks >= 20 and r.cache_usable()  # plain frames while it warmed up, the cache after
    assert np.mean(errs[-10:]) < np.mean(plain), (np.mean(errs[-10:]), np.mean(plain))
    assert nrc.status() == 0
