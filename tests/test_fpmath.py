"""The sine, cosine and integer power of cube-tracing_b200/csrc/ct_fpmath.h
(shared by the CUDA kernels and the oracle's GLSL shim, see the header)
against double precision: a few units in the last place over the range the
path tracer uses, [0, 2*pi), and beyond it."""
import numpy as np


def ulp_error(got, want):
    got = got.astype(np.float64)
    ulp = np.spacing(np.abs(want).astype(np.float32)).astype(np.float64)
    # near zero crossings compare against the scale of the argument range
    ulp = np.maximum(ulp, np.spacing(np.float32(1.0)) * 2.0 ** -24)
    return np.abs(got - want) / ulp


def test_sin_cos_accuracy(oracle_lib):
    rng = np.random.default_rng(7)
    x = np.concatenate([np.linspace(0.0, 2 * np.pi, 200001, dtype=np.float32),
                        rng.uniform(-200.0, 200.0, 100000).astype(np.float32)])
    s, c, _ = oracle_lib.fpmath(x)
    xd = x.astype(np.float64)
    es, ec = np.sin(xd), np.cos(xd)
    # absolute error relative to 1 (the values' scale) stays near float epsilon
    assert np.max(np.abs(s - es)) < 4e-7 and np.max(np.abs(c - ec)) < 4e-7
    # and relative error is a few ulp away from the zeros
    big = np.abs(es) > 1e-2
    assert np.max(ulp_error(s[big], es[big])) <= 4
    big = np.abs(ec) > 1e-2
    assert np.max(ulp_error(c[big], ec[big])) <= 4


def test_integer_power_is_repeated_product(oracle_lib):
    x = np.linspace(-2.0, 2.0, 10001, dtype=np.float32)
    _, _, p = oracle_lib.fpmath(x)
    want = x * x
    want = want * x
    want = want * x
    want = want * x
    assert np.array_equal(p, want)
