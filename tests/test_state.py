"""Frame history checkpoint (ct_state_size / ct_state_save / ct_state_load)
on the CPU: the blob's size and header, argument checks that need no
device, and the oracle's own save/load in the same format resuming a run
exactly."""
import ctypes

import numpy as np

from cases import build_case, frame_keys
from cube_tracing import layouts as L
from cube_tracing import native


def test_state_size():
    n = ctypes.c_uint64()
    lib = native.lib()
    assert lib.ct_state_size(36, 28, ctypes.byref(n)) == 0
    per_pixel = 3 * 36 + 2 * 60 + 8 + 2 * 92 + 12 + 4 * 16
    assert n.value == native.STATE_HEADER_BYTES + 36 * 28 * per_pixel
    assert lib.ct_state_size(0, 28, ctypes.byref(n)) == 1
    assert lib.ct_state_size(65536, 65536, ctypes.byref(n)) == 2
    assert lib.ct_state_size(4, 4, None) == 1


def test_state_calls_check_their_arguments():
    lib = native.lib()
    pc = native.PushConstant()
    pc.size[0], pc.size[1] = 8, 8
    buf = (ctypes.c_uint8 * 64)()
    # a size other than ct_state_size's, and null pointers: refused before any device work
    assert lib.ct_state_save(ctypes.byref(pc), buf, 64, None) == 1
    assert lib.ct_state_load(ctypes.byref(pc), buf, 64, None) == 1
    assert lib.ct_state_save(None, buf, 64, None) == 1
    assert lib.ct_state_load(ctypes.byref(pc), None, 64, None) == 1


def test_oracle_resumes_from_its_saved_state(oracle_lib):
    name = "grid16_materials_brdf_pt"
    sc, W, H, cams, kw = build_case(name)
    a = oracle_lib.OracleRenderer(sc, W, H, **kw)
    for iv, ip in cams[:2]:
        a.render(iv, ip)
    state = a.save_state()
    blob = state[0]
    head = blob[:24].view(np.uint32)
    assert tuple(head[:5]) == (native.STATE_MAGIC, native.STATE_VERSION, W, H, len(native.STATE_SECTIONS))
    assert blob.size == native.STATE_HEADER_BYTES + int(blob[24:24 + 8 * 13].view(np.uint64).sum())
    b = oracle_lib.OracleRenderer(sc, W, H, **kw)
    b.load_state(state)
    ia = a.render(*cams[2]).copy()
    ib = b.render(*cams[2]).copy()
    assert ia.tobytes() == ib.tobytes()
    for k in frame_keys(name):
        assert a.buf[k].tobytes() == b.buf[k].tobytes(), k
    a.close()
    b.close()
