"""Input and output files of the C++ host side's check program
(cube-tracing_b200/host/ct_host_check): a scene, a camera path and the
ct_params of a frame sequence in; the last frame's image and RESTIR buffers
out."""
import ctypes
import os
import struct
import subprocess

import numpy as np

from cube_tracing import layouts as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROGRAM = os.path.join(ROOT, "cube-tracing_b200", "host", "ct_host_check")
RESTIR_ORDER = ["previous_reservoir", "intermediate_reservoir", "reservoir", "previous_di", "di", "velocity",
                "output_path_reservoir", "temporal_path_reservoir", "indirect_color"]


def write_input(path, scene, W, H, cams, params, features, max_depth, taa=True, sky_time=1.0, is_afternoon=1):
    arrays = [scene.instances, scene.primitives, scene.aabbs, scene.materials, scene.point_lights,
              scene.cube_lights, scene.env_lights]
    dts = [L.INSTANCE, L.PRIMITIVE, L.AABB, L.MATERIAL, L.LIGHT, L.LIGHT, L.LIGHT]
    with open(path, "wb") as f:
        f.write(b"CTHI")
        f.write(struct.pack("<7I2f", W, H, len(cams), features, max_depth, int(taa), is_afternoon, sky_time,
                            scene.voxel_extent))
        f.write(struct.pack("<7I", *[a.shape[0] for a in arrays]))
        raw = bytes(params)
        f.write(struct.pack("<I", len(raw)))
        f.write(raw)
        f.write(np.ascontiguousarray(scene.light_config, L.LIGHT_CONFIG).tobytes())
        for a, dt in zip(arrays, dts):
            f.write(np.ascontiguousarray(a, dt).tobytes())
        for iv, ip in cams:
            f.write(np.asarray(iv, np.float32).tobytes())
            f.write(np.asarray(ip, np.float32).tobytes())


def read_output(path):
    with open(path, "rb") as f:
        data = f.read()
    assert data[:4] == b"CTHO"
    W, H = struct.unpack("<2I", data[4:12])
    off = 12
    out = {"image": np.frombuffer(data, np.float32, W * H * 4, off).reshape(H, W, 4)}
    off += W * H * 16
    for k in RESTIR_ORDER:
        n = W * H * L.PER_PIXEL_BUFFERS[k].itemsize
        out[k] = np.frombuffer(data, np.uint8, n, off)
        off += n
    assert off == len(data)
    return out


def run(inp, outp):
    return subprocess.run([PROGRAM, inp, outp], capture_output=True, text=True, timeout=300)
