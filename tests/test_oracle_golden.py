"""The oracle reproduces its committed golden fixtures byte for byte,
independent of the number of host threads (no GPU needed)."""
import json
import os

import numpy as np
import pytest

from cases import CASES, PT_CASES
from cube_tracing import layouts as L

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("name", CASES + PT_CASES)
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


@pytest.mark.parametrize("name", PT_CASES)
def test_pt_golden_fixtures_are_not_degenerate(name):
    g = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    hit = g["f2_di"].view(L.DI_INFO)["distance"] > 0
    out = g["f2_output_path_reservoir"].view(L.PATH_RESERVOIR)
    fin = g["f2_temporal_path_reservoir"].view(L.PATH_RESERVOIR)
    assert (out["M"][hit] > 0).all()                  # every hit pixel built a path
    assert (fin["weight"][hit] > 0).mean() > 0.01     # some carry indirect light
    assert (fin["rc_instance_id"][hit] < L.MAX_INSTANCES).any()
    ind = g["f2_indirect_color"].view(np.float32)
    assert np.isfinite(ind).all()


@pytest.mark.parametrize("name", ["config0", "config0_spec"])
def test_oracle_matches_config0_digest(oracle_lib, name):
    """The 256x256, 8-frame workload with DI and PT, pinned by digests: with
    the reference's reuse parameters and a point light ("config0"), and as
    specified, 5 neighbours in 30 px and no point light ("config0_spec")."""
    from golden.make_golden import digest_case
    with open(os.path.join(HERE, "golden", f"{name}_digest.json")) as f:
        want = json.load(f)
    got = digest_case(name)
    assert sorted(got) == sorted(want)
    bad = [k for k in got if got[k] != want[k]]
    assert not bad, bad[:10]
