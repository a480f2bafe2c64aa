"""The oracle reproduces its committed golden fixtures byte for byte,
independent of the number of host threads (no GPU needed)."""
import os

import numpy as np
import pytest

from cases import CASES, FRAME_KEYS
from cube_tracing import layouts as L

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("threads", [1, 0])
def test_oracle_matches_golden(oracle_lib, name, threads):
    from golden.make_golden import render_case
    golden = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    out = render_case(name, threads=threads)
    assert sorted(out) == sorted(golden.files)
    for k in out:
        assert np.array_equal(out[k], golden[k]), k


@pytest.mark.parametrize("name", CASES)
def test_golden_fixtures_are_not_degenerate(name):
    g = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    di = g["f2_di"].view(L.DI_INFO)
    hit = di["distance"] > 0
    assert 0.2 < hit.mean() <= 1.0
    res = g["f2_previous_reservoir"].view(L.RESERVOIR)
    valid = (res["M"] > 0) & (res["Y"] != 0xFFFFFFFF)
    assert valid[hit].mean() > 0.05          # some pixels keep a light sample
    assert (res["W_y"][hit] > 0).any()
    img = g["f2_image"]
    assert np.isfinite(img).all() and img[..., :3].max() > 0
