"""Host logic of the radiance cache, on the CPU: the encoding's layout and
exactness, and the rule that switches frames between the plain tracer and
the cache (NrcRenderer.cache_usable).  The kernels are tested against these
restatements in test_gpu_nrc.py."""
import math
import types

import numpy as np
import torch

from cube_tracing import nrc


def test_encoding_layout():
    q = nrc.random_queries(64, seed=3, device="cpu")
    e = nrc.encode(q, (0.0, 0.0, 0.0), (256.0, 128.0, 256.0))
    assert e.shape == (64, nrc.IN)
    # sin^2 + cos^2 = 1 for every band of every axis
    s, c = e[:, 0:96:2], e[:, 1:96:2]
    assert torch.allclose(s * s + c * c, torch.ones_like(s), atol=1e-5)
    # one-blob bins lie in [0, 1] (far bins underflow to 0) and peak at the bin of u
    blobs = e[:, 96:224]
    assert (blobs >= 0).all() and (blobs <= 1.0).all()
    u1 = q[:, 4] * 0.5 + 0.5  # the direction's second angle
    peak = blobs[:, 32:64].argmax(1).float()
    assert (peak - torch.clamp(torch.floor(u1 * 32.0), 0, 31)).abs().max() <= 1.0
    assert torch.equal(e[:, 224:227], q[:, 9:12])
    assert (e[:, 227:] == 0).all()


def test_band_phase_is_exact():
    # (x 2^k) mod 2 of the torch restatement equals the kernel's
    # s - 2 floor(s / 2): both are exact in float32
    rng = np.random.default_rng(0)
    x = rng.random(10000).astype(np.float32)
    for k in range(16):
        s = x * np.float32(2 ** k)
        a = torch.remainder(torch.from_numpy(s), 2.0).numpy()
        b = s - np.float32(2.0) * np.floor(s * np.float32(0.5))
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), k


def _renderer(**kw):
    tracer = types.SimpleNamespace(W=4, H=2, device="cpu",
                                   a=types.SimpleNamespace(albedo_target=np.zeros((1, 3), np.float32),
                                                           emission_target=np.zeros((1, 3), np.float32)))
    return nrc.NrcRenderer(tracer, cache=None, train_paths=4, train_bounces=2, **kw)


def test_fallback_until_warm_then_on_divergence():
    r = _renderer(min_frames=3, diverge=4.0)
    assert not r.cache_usable()  # nothing trained yet
    for loss in (20.0, 15.0, 12.0):
        r.trained += 1
        r.ema = loss if r.ema is None else 0.95 * r.ema + 0.05 * loss
        r.best_ema = min(r.best_ema, r.ema)
        assert not r.cache_usable()  # still within the warm-up frames
    r.trained += 1
    assert r.cache_usable()
    # the moving average more than 4x its lowest value: plain frames again
    r.ema = 4.01 * r.best_ema
    assert not r.cache_usable()
    r.ema = r.best_ema
    assert r.cache_usable()
    r.ema = math.inf
    assert not r.cache_usable()
    r.ema = math.nan
    assert not r.cache_usable()
