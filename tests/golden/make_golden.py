"""Regenerates the golden fixtures: the CPU oracle (the reference's GLSL
compiled as C++, oracle/) rendering the small workloads of tests/cases.py.

    make -C oracle && python tests/golden/make_golden.py

The full-size small workload (cases "config0" and "config0_spec": 256x256,
8 frames) is pinned by per-buffer SHA-256 digests instead
(<case>_digest.json).

Each fixture <case>.npz holds, per frame f: f{f}_<buffer> raw bytes of the
per-pixel buffers (DI info, intermediate and previous reservoirs, velocity;
for the *_pt cases also the output and temporal path reservoirs and the
indirect colour) and f{f}_image, the output image.  The fixtures pin the oracle: the CPU test
suite re-renders them and requires identical bytes."""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "cube-tracing_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import pyoracle  # noqa: E402
from cases import CASES, PT_CASES, build_case, frame_keys  # noqa: E402


def render_case(name, threads=0):
    sc, W, H, cams, kw = build_case(name)
    r = pyoracle.OracleRenderer(sc, W, H, threads=threads, **kw)
    out = {}
    for f, (iv, ip) in enumerate(cams):
        img = r.render(iv, ip)
        for k in frame_keys(name):
            out[f"f{f}_{k}"] = r.buf[k].view(np.uint8).copy()
        out[f"f{f}_image"] = img.copy()
    r.close()
    return out


def digest_case(name, threads=0):
    """SHA-256 of every buffer of every frame (for workloads whose full
    fixture would be too large to commit)."""
    out = render_case(name, threads=threads)
    return {k: hashlib.sha256(np.ascontiguousarray(v).view(np.uint8).tobytes()).hexdigest() for k, v in out.items()}


def main():
    for name in CASES + PT_CASES:
        out = render_case(name)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, {k: v.shape for k, v in out.items() if k.startswith("f0")})
    for name in ("config0", "config0_spec"):
        with open(os.path.join(HERE, f"{name}_digest.json"), "w") as f:
            json.dump(digest_case(name), f, indent=1, sort_keys=True)
        print(f"{name} digests written")


if __name__ == "__main__":
    main()
