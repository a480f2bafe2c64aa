"""Neural radiance cache: the network the fused tensor-core kernel evaluates
(ct_nrc_infer, include/ct.h), its input encoding, and its training in torch.

The kernel is the product's inference path; torch holds the fp32 master
weights and trains them (Adam), and every export rounds them to the bf16
buffer the kernel reads.  Both sides compute the same encoding:

  position q = clamp((p - bbox_min) / bbox_extent, 0, 1); per axis c and band
    k < 16, t = (q_c 2^k) mod 2: sin(pi t), cos(pi t)         (96 values)
  direction, then normal: u0 = atan2(v.z, v.x) / 2pi + 1/2, u1 = v.y / 2 + 1/2,
    one-blob in 32 bins: exp(-((u - (i + 1/2) / 32) 32)^2 / 2) (2 x 64 values)
  albedo (3); zeros up to 256.

Network: 256 -> 64 x 5 (ReLU) -> 16, no biases; outputs 0..2 are RGB.
"""
import ctypes
import math

import numpy as np
import torch

from . import native

IN, WIDTH, HIDDEN, OUT = 256, 64, 5, 16
WEIGHT_COUNT = WIDTH * IN + 4 * WIDTH * WIDTH + OUT * WIDTH
QUERY_FLOATS = 12  # position, direction, normal, albedo


class NrcNet(ctypes.Structure):
    _fields_ = [("weights_address", ctypes.c_uint64), ("bbox_min", ctypes.c_float * 3),
                ("bbox_extent", ctypes.c_float * 3)]


_CONSTS = {}


def _consts(device, bbox_min, bbox_extent):
    """The encoding's constant tensors on `device`, made once: a host list
    copied to the device at every call would wait for the stream."""
    key = (str(device), tuple(float(v) for v in bbox_min), tuple(float(v) for v in bbox_extent))
    c = _CONSTS.get(key)
    if c is None:
        c = (torch.tensor(key[1], dtype=torch.float32, device=device),
             torch.tensor(key[2], dtype=torch.float32, device=device),
             torch.tensor([float(2 ** k) for k in range(16)], device=device),
             (torch.arange(32, dtype=torch.float32, device=device) + 0.5) / 32.0)
        _CONSTS[key] = c
    return c


def encode(queries, bbox_min, bbox_extent):
    """The encoding of `queries` (n, 12) float32 -> (n, 256) float32."""
    q = queries
    n = q.shape[0]
    out = torch.zeros((n, IN), dtype=torch.float32, device=q.device)
    bmin, bext, scales, centres = _consts(q.device, bbox_min, bbox_extent)
    x = ((q[:, 0:3] - bmin) / bext).clamp(0.0, 1.0)
    t = torch.remainder(x[:, :, None] * scales, 2.0)  # exact: power-of-two scale, then mod 2
    ang = math.pi * t
    enc = torch.stack([torch.sin(ang), torch.cos(ang)], dim=-1).reshape(n, 96)
    out[:, :96] = enc
    for v, off in ((q[:, 3:6], 96), (q[:, 6:9], 160)):
        u0 = torch.atan2(v[:, 2], v[:, 0]) * (0.5 / math.pi) + 0.5
        u1 = v[:, 1] * 0.5 + 0.5
        for j, u in enumerate((u0, u1)):
            d = (u[:, None] - centres) * 32.0
            out[:, off + 32 * j:off + 32 * j + 32] = torch.exp(-0.5 * d * d)
    out[:, 224:227] = q[:, 9:12]
    return out


class NrcMlp(torch.nn.Module):
    """The fp32 master copy of the network (no biases)."""

    def __init__(self, seed=0):
        super().__init__()
        g = torch.Generator().manual_seed(seed)
        dims = [IN] + [WIDTH] * HIDDEN + [OUT]
        self.weights = torch.nn.ParameterList()
        for i in range(len(dims) - 1):
            w = torch.randn(dims[i + 1], dims[i], generator=g) * math.sqrt(2.0 / dims[i])
            self.weights.append(torch.nn.Parameter(w))

    def forward(self, enc, round_bf16=False):
        """fp32 forward; with round_bf16, inputs, weights and hidden
        activations are rounded to bf16 as the kernel rounds them."""
        h = enc.to(torch.bfloat16).float() if round_bf16 else enc
        for i, w in enumerate(self.weights):
            wt = w.to(torch.bfloat16).float() if round_bf16 else w
            h = h @ wt.t()
            if i < len(self.weights) - 1:
                h = torch.relu(h)
                if round_bf16:
                    h = h.to(torch.bfloat16).float()
        return h

    def packed(self):
        """The kernel's bf16 weight buffer (CT_NRC_WEIGHT_COUNT values)."""
        return torch.cat([w.detach().reshape(-1) for w in self.weights]).to(torch.bfloat16).contiguous()


class NrcCache:
    """The cache on the device: bf16 weights for ct_nrc_infer, an fp32
    NrcMlp trained with Adam on (query, radiance) pairs."""

    def __init__(self, bbox_min, bbox_extent, device="cuda", lr=1e-3, seed=0):
        self.device = device
        self.mlp = NrcMlp(seed).to(device)
        self.opt = torch.optim.Adam(self.mlp.parameters(), lr=lr, fused=torch.device(device).type == "cuda")
        self.bbox_min = [float(v) for v in bbox_min]
        self.bbox_extent = [float(v) for v in bbox_extent]
        self.weights = torch.zeros(WEIGHT_COUNT, dtype=torch.bfloat16, device=device)
        self.export()

    def export(self):
        self.weights.copy_(self.mlp.packed())

    def net(self):
        n = NrcNet()
        n.weights_address = self.weights.data_ptr()
        for i in range(3):
            n.bbox_min[i] = self.bbox_min[i]
            n.bbox_extent[i] = self.bbox_extent[i]
        return n

    @staticmethod
    def _stream():
        return torch.cuda.current_stream().cuda_stream

    def infer(self, queries):
        """RGB (n, 3) of (n, 12) float32 device queries, by the fused kernel."""
        queries = queries.contiguous()
        n = queries.shape[0]
        rgb = torch.empty((n, 3), dtype=torch.float32, device=self.device)
        net = self.net()
        native.check("ct_nrc_infer", native.lib().ct_nrc_infer(ctypes.byref(net), queries.data_ptr(), n,
                                                               rgb.data_ptr(), self._stream()))
        return rgb

    def infer_encoded(self, encoded):
        encoded = encoded.to(torch.bfloat16).contiguous()
        n = encoded.shape[0]
        rgb = torch.empty((n, 3), dtype=torch.float32, device=self.device)
        net = self.net()
        native.check("ct_nrc_infer_encoded", native.lib().ct_nrc_infer_encoded(
            ctypes.byref(net), encoded.data_ptr(), n, rgb.data_ptr(), self._stream()))
        return rgb

    def encode_device(self, queries):
        """The kernel's encoding, bf16 (n, 256)."""
        queries = queries.contiguous()
        n = queries.shape[0]
        enc = torch.empty((n, IN), dtype=torch.bfloat16, device=self.device)
        net = self.net()
        native.check("ct_nrc_encode", native.lib().ct_nrc_encode(ctypes.byref(net), queries.data_ptr(), n,
                                                                 enc.data_ptr(), self._stream()))
        return enc

    def train_step(self, queries, targets, weights=None):
        """One Adam step on the relative L2 loss of the cache's RGB against
        `targets` (n, 3), each query weighted by `weights` (n,) if given;
        the bf16 export follows.  Returns the loss as a device scalar (no
        host synchronisation)."""
        enc = encode(queries, self.bbox_min, self.bbox_extent)
        pred = self.mlp(enc)[:, :3]
        rel = ((pred - targets) ** 2) / (pred.detach() ** 2 + 1e-2)
        if weights is None:
            loss = rel.mean()
        else:
            loss = (rel * weights[:, None]).sum() / (3.0 * weights.sum()).clamp(min=1.0)
        self.opt.zero_grad()
        loss.backward()
        self.opt.step()
        self.export()
        return loss.detach()


def status(reset=True):
    v = ctypes.c_uint32()
    native.check("ct_nrc_status", native.lib().ct_nrc_status(int(reset), ctypes.byref(v)))
    return v.value


def random_queries(n, seed=0, device="cuda", bbox_min=(0.0, 0.0, 0.0), bbox_extent=(256.0, 128.0, 256.0)):
    """n seeded queries inside the box (unit directions and normals)."""
    rng = np.random.default_rng(seed)
    q = np.zeros((n, QUERY_FLOATS), np.float32)
    q[:, 0:3] = np.asarray(bbox_min) + rng.random((n, 3)) * np.asarray(bbox_extent)
    for off in (3, 6):
        v = rng.standard_normal((n, 3))
        q[:, off:off + 3] = v / np.linalg.norm(v, axis=1, keepdims=True)
    q[:, 9:12] = rng.uniform(0.1, 0.9, (n, 3))
    return torch.from_numpy(q).to(device)


class NrcRenderer:
    """One sample per pixel of the adjoint's path tracer (ct_nrc_trace),
    terminated by the cache at surface vertex `cache_vertex` (v0 the primary
    hit; the default 1 is path vertex 2 counting the camera as vertex 0),
    the cache training online on `train_paths` self-training paths per
    frame.  `tracer` is an AdjointRenderer over the scene (its tables,
    camera, miss light)."""

    def __init__(self, tracer, cache, train_paths=1 << 16, train_bounces=4, min_frames=32, diverge=4.0,
                 steps_per_frame=4, batch=1 << 14, cache_vertex=1):
        self.cache_vertex = cache_vertex
        self.t, self.cache = tracer, cache
        # The plain path tracer renders the frame instead of the cache while
        # the cache's error is out of bounds: until it has trained on
        # `min_frames` frames before this one, and whenever the slow moving
        # average of its training loss (relative L2 on single-sample targets,
        # so noisy and well above 0 even for a good cache) is not finite or
        # exceeds `diverge` times its lowest value.
        self.min_frames, self.diverge = min_frames, diverge
        self.steps_per_frame, self.batch = steps_per_frame, batch
        self.ema = None
        self.best_ema = float("inf")
        self.trained = 0
        self.last_loss = float("inf")
        self.fallbacks = 0
        W, H, dev = tracer.W, tracer.H, tracer.device
        self.train_paths, self.train_bounces = train_paths, train_bounces
        px = W * H
        self.base = torch.zeros((px, 3), dtype=torch.float32, device=dev)
        self.thp = torch.zeros((px, 3), dtype=torch.float32, device=dev)
        self.query = torch.zeros((px, QUERY_FLOATS), dtype=torch.float32, device=dev)
        B = train_bounces
        self.tq = torch.zeros((train_paths, B + 1, QUERY_FLOATS), dtype=torch.float32, device=dev)
        self.tpart = torch.zeros((train_paths, B, 3), dtype=torch.float32, device=dev)
        self.tthp = torch.zeros((train_paths, B, 3), dtype=torch.float32, device=dev)
        self.albedo = torch.from_numpy(tracer.a.albedo_target).to(dev)
        self.emission = torch.from_numpy(tracer.a.emission_target).to(dev)
        self.frame = 0

    def trace(self, seed):
        f = native.NrcFrame()
        f.struct_size = ctypes.sizeof(native.NrcFrame)
        f.train_paths = self.train_paths
        f.train_offset = (self.frame * 7919) % max(self.t.W * self.t.H // max(self.train_paths, 1), 1)
        f.train_bounces = self.train_bounces
        f.cache_vertex = self.cache_vertex
        f.base_address = self.base.data_ptr()
        f.query_address = self.query.data_ptr()
        f.throughput_address = self.thp.data_ptr()
        f.train_query_address = self.tq.data_ptr()
        f.train_partial_address = self.tpart.data_ptr()
        f.train_throughput_address = self.tthp.data_ptr()
        d = self.t.desc(spp=1)
        d.seed = seed
        native.check("ct_nrc_trace", native.lib().ct_nrc_trace(
            self.t.accel.handle, ctypes.byref(d), self.albedo.data_ptr(), self.emission.data_ptr(), ctypes.byref(f),
            torch.cuda.current_stream().cuda_stream))

    def train(self):
        """Targets from this frame's self-training paths (partial radiance +
        throughput x the cache at the terminal vertex), then steps_per_frame
        Adam steps on random batches of their vertices (vertices a path did
        not reach weigh 0).  One host synchronisation per frame."""
        B = self.train_bounces
        term = self.tq[:, B]
        with torch.no_grad():
            boot = self.cache.infer(term.contiguous()).clamp(min=0.0)
            boot = torch.where((term[:, 9:10] >= 0.0), boot, torch.zeros_like(boot))
            targets = self.tpart + self.tthp * boot[:, None, :]
            q = self.tq[:, :B].reshape(-1, QUERY_FLOATS)
            tg = targets.reshape(-1, 3)
            valid = (q[:, 9] >= 0.0).float()
        loss = None
        for _ in range(self.steps_per_frame):
            pick = torch.randint(0, q.shape[0], (min(self.batch, q.shape[0]),), device=q.device)
            loss = self.cache.train_step(q[pick], tg[pick], weights=valid[pick])
        loss, n = torch.stack([loss, valid.sum()]).tolist()
        if n == 0:
            return float("inf"), 0
        self.trained += 1
        self.ema = loss if self.ema is None else 0.95 * self.ema + 0.05 * loss
        self.best_ema = min(self.best_ema, self.ema)
        return loss, int(n)

    def cache_usable(self):
        return (self.trained > self.min_frames and self.ema is not None and math.isfinite(self.ema)
                and self.ema <= self.diverge * self.best_ema)

    def render(self, seed, train=True, out=None):
        """One frame: trace, train on its self-training paths, then the image
        base + throughput x cache (H, W, 3), written into `out` if given;
        while the cache is not usable (cache_usable), the frame is the plain
        tracer's (one sample, its own depth) instead."""
        self.trace(seed)
        info = self.train() if train else (self.last_loss, 0)
        self.last_loss = info[0]
        self.frame += 1
        if not self.cache_usable():
            self.fallbacks += 1
            t = self.t
            old = t.seed
            t.seed = seed
            try:
                img = t.forward(self.albedo, self.emission, spp=1)
            finally:
                t.seed = old
            if out is not None:
                out.copy_(img.reshape(out.shape))
                img = out
            return img, info
        rgb = self.cache.infer(self.query).clamp_(min=0.0)
        if out is None:
            return (self.base + self.thp * rgb).reshape(self.t.H, self.t.W, 3), info
        torch.addcmul(self.base, self.thp, rgb, out=out.view(-1, 3))
        return out, info
