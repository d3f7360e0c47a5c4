"""The FP64 oracle against its own pinned config-1 outputs (tests/golden/
make_config1_fixture.py): the whole projection and backprojection are regenerated
and must hash to the committed SHA-256 values, and the committed raw views / slice
must match bit for bit.  This guards the oracle itself against regression."""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_config1_fixture as F  # noqa: E402

GOLD = os.path.join(HERE, "golden")


def test_config1_oracle_outputs_match_pinned_hashes():
    ref = json.load(open(os.path.join(GOLD, "config1_oracle.json")))
    g, vol, prj, back = F.config1_outputs()
    got = F.summary(vol, prj, back)
    assert got["volume_sha256_f32"] == ref["volume_sha256_f32"], "phantom changed"
    views = np.fromfile(os.path.join(GOLD, "config1_proj_views.f64"), "<f8").reshape(len(F.VIEWS), g.DNU, g.DNV)
    np.testing.assert_array_equal(prj[list(F.VIEWS)], views)
    sl = np.fromfile(os.path.join(GOLD, "config1_back_slice.f64"), "<f8").reshape(g.YN, g.XN)
    np.testing.assert_array_equal(back[:, :, F.SLICE], sl)
    assert got["proj_sha256_f64"] == ref["proj_sha256_f64"]
    assert got["back_sha256_f64"] == ref["back_sha256_f64"]
