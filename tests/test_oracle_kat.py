"""Known-answer checks of the oracle's shader primitives against values
computed here from the published algorithms (no GPU needed).

The reference ships no tests or golden vectors; these pin the pieces the
whole parity chain rests on: the TEA seed hash and LCG stream of
random.glsl:26-77, the self-intersection offset of primitives.glsl:233-257
and the ray/box test of primitives.glsl:273-355."""
import ctypes
import math
import struct

import numpy as np
import pytest

M32 = 0xFFFFFFFF


def tea_ref(v0, v1):
    """Zafar, Olano and Curtis, "GPU Random Numbers via the Tiny Encryption
    Algorithm", 16 rounds as random.glsl uses."""
    s0 = 0
    for _ in range(16):
        s0 = (s0 + 0x9E3779B9) & M32
        v0 = (v0 + ((((v1 << 4) & M32) + 0xA341316C) ^ ((v1 + s0) & M32) ^ ((v1 >> 5) + 0xC8013EA4))) & M32
        v1 = (v1 + ((((v0 << 4) & M32) + 0xAD90777D) ^ ((v0 + s0) & M32) ^ ((v0 >> 5) + 0x7E95761E))) & M32
    return v0


def lcg_ref(state):
    state = (1664525 * state + 1013904223) & M32
    return state, state & 0x00FFFFFF


@pytest.mark.parametrize("a,b", [(0, 0), (1, 0), (0, 1), (65535, 7), (123456, 99), (M32, M32), (2073599, 59)])
def test_tea(oracle_lib, a, b):
    assert oracle_lib.lib().oracle_tea(a, b) == tea_ref(a, b)


def test_lcg_stream(oracle_lib):
    seed = ctypes.c_uint32(tea_ref(42, 3))
    state = seed.value
    for _ in range(1000):
        got = oracle_lib.lib().oracle_rnd(ctypes.byref(seed))
        state, bits = lcg_ref(state)
        assert got == np.float32(bits) / np.float32(1 << 24)
        assert seed.value == state
        assert 0.0 <= got < 1.0


def f32_bits(x):
    return struct.unpack("<i", struct.pack("<f", x))[0]


def bits_f32(i):
    return struct.unpack("<f", struct.pack("<i", i))[0]


def compute_ray_origin_ref(pos, n):
    out = []
    for p, c in zip(pos, n):
        p = np.float32(p)
        ioff = int(np.float32(c) * np.float32(256.0))
        ipos = bits_f32(f32_bits(p) + (-ioff if p < 0 else ioff))
        fpos = np.float32(p + np.float32(np.float32(c) * np.float32(1.0 / 65536.0)))
        out.append(np.float32(fpos if abs(p) < np.float32(1.0 / 32.0) else ipos))
    return out


@pytest.mark.parametrize("pos,n", [((10.5, 3.0, -7.25), (0, 1, 0)), ((0.01, -0.02, 5.0), (1, 0, 0)),
                                   ((-33.0, 12.0, 0.0), (0, 0, -1)), ((1e-3, 64.0, 64.0), (-1, 0, 0))])
def test_compute_ray_origin(oracle_lib, pos, n):
    p = (ctypes.c_float * 3)(*pos)
    q = (ctypes.c_float * 3)(*n)
    o = (ctypes.c_float * 3)()
    oracle_lib.lib().oracle_compute_ray_origin(p, q, o)
    assert list(o) == [float(x) for x in compute_ray_origin_ref(pos, n)]


def box(oracle_lib, c, h, o, d, can_start=1, oriented=1):
    t = ctypes.c_float()
    n = (ctypes.c_float * 3)()
    hit = oracle_lib.lib().oracle_intersect_box((ctypes.c_float * 3)(*c), h, (ctypes.c_float * 3)(*o),
                                                (ctypes.c_float * 3)(*d), can_start, oriented, ctypes.byref(t), n)
    return hit, t.value, list(n)


def test_box_axis_hit(oracle_lib):
    hit, t, n = box(oracle_lib, (0.5, 0.5, 0.5), 0.5, (0.5, 0.5, -3.0), (0, 0, 1))
    assert hit == 1 and t == 3.0 and n == [0.0, 0.0, -1.0]


def test_box_oblique_hit(oracle_lib):
    d = np.array([1.0, 0.1, 0.05])
    d /= np.linalg.norm(d)
    hit, t, n = box(oracle_lib, (0.5, 0.5, 0.5), 0.5, (-1.0, 0.3, 0.4), tuple(d))
    assert hit == 1 and abs(t - 1.0 / d[0]) < 1e-5 and n == [-1.0, 0.0, 0.0]


def test_box_corner_is_not_a_hit(oracle_lib):
    # the in-face test is strict, so a ray through a corner misses
    d = np.array([1.0, 1.0, 1.0]) / math.sqrt(3.0)
    assert box(oracle_lib, (0.5, 0.5, 0.5), 0.5, (-1.0, -1.0, -1.0), tuple(d))[0] == 0


def test_box_miss_and_edge(oracle_lib):
    assert box(oracle_lib, (0.5, 0.5, 0.5), 0.5, (0.5, 2.0, -3.0), (0, 0, 1))[0] == 0
    # a ray along a face plane does not hit (strict inequality in the test)
    assert box(oracle_lib, (0.5, 0.5, 0.5), 0.5, (0.5, 1.0, -3.0), (0, 0, 1))[0] == 0


def test_box_inside(oracle_lib):
    # starting inside: exit distance when the ray may start in the box, no hit otherwise
    hit, t, _ = box(oracle_lib, (0.5, 0.5, 0.5), 0.5, (0.5, 0.5, 0.5), (1, 0, 0), can_start=1)
    assert hit == 1 and t == 0.5
    assert box(oracle_lib, (0.5, 0.5, 0.5), 0.5, (0.5, 0.5, 0.5), (1, 0, 0), can_start=0)[0] == 0


def test_box_behind(oracle_lib):
    assert box(oracle_lib, (0.5, 0.5, 0.5), 0.5, (0.5, 0.5, 3.0), (0, 0, 1))[0] == 0
