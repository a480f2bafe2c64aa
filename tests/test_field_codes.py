"""The cell field's code table and the CPU restatement of the field that
tests/test_gpu_field.py checks the GPU build against."""
import numpy as np
import pytest

import fieldref


def test_header_table_matches():
    assert fieldref.header_edges() == fieldref.FIELD_EDGES


def test_table_shape():
    t = fieldref.FIELD_EDGES
    assert len(t) == 16 and t[0] == 0 and t[1] == 1
    assert all(a < b for a, b in zip(t, t[1:]))
    # the build reaches the largest edge by doubling the Jacobi cap of 15
    cap = 15
    while cap < t[-1]:
        cap *= 2
    assert t[-1] <= cap <= 240


@pytest.mark.parametrize("octant", range(8))
def test_restatement_against_brute_force(octant):
    rng = np.random.default_rng(octant)
    occ = rng.random((7, 6, 9)) < 0.08
    occ[0, 0, 0] = True
    for cap in (5, 30):
        assert np.array_equal(fieldref.exact_edges(occ, octant, cap), fieldref.brute_edges(occ, octant, cap))


def test_coding_rounds_down():
    occ = np.zeros((40, 40, 40), bool)
    occ[39, 39, 39] = True
    got = fieldref.coded_edges(occ, 0)
    k = fieldref.exact_edges(occ, 0, 30)
    assert (got <= k).all() and got.max() == 30 and got[39, 39, 39] == 0
    assert set(np.unique(got)) <= set(fieldref.FIELD_EDGES)
