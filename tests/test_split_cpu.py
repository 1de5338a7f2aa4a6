"""The held-out split (felog_heldout_split, the split felog_synth_generate
applies) against the reference's own gtrain tool (src/tools/gtrain.cpp:293-343)
run on the same edges with the same draws (tests/golden/split_*.npz, made by
oracle/_ref/ref_gtrain through make_fixtures.py): the kept training edges in
the tool's swapped order, the held-out positives and the negatives, exactly.
"""
import numpy as np
import pytest

import felog_b200 as fb
from conftest import load_golden


@pytest.mark.parametrize("name", ["split_rmat300.npz", "split_rmat4096.npz", "split_star_path.npz"])
def test_split_matches_reference_tool(name):
    fx = load_golden(name)
    e = np.zeros(len(fx["src"]), fb.EDGE12)
    e["src"], e["dst"] = fx["src"], fx["dst"]
    tr, ts, td, tl = fb.heldout_split(e, int(fx["v_num"]), float(fx["sample"]), int(fx["seed"]))
    np.testing.assert_array_equal(tr["src"], fx["train_src"])
    np.testing.assert_array_equal(tr["dst"], fx["train_dst"])
    np.testing.assert_array_equal(ts, fx["test_src"])
    np.testing.assert_array_equal(td, fx["test_dst"])
    np.testing.assert_array_equal(tl, fx["test_label"])


def test_synthetic_graphs_use_the_same_split():
    full = fb.synth_graph(seed=9, v_target=2048, e_target=12000, holdout=0.0)
    part = fb.synth_graph(seed=9, v_target=2048, e_target=12000, holdout=0.1)
    assert full["v_num"] == part["v_num"]
    tr, ts, td, tl = fb.heldout_split(full["edges"], full["v_num"], 0.1, 9)
    np.testing.assert_array_equal(part["edges"]["src"], tr["src"])
    np.testing.assert_array_equal(part["edges"]["dst"], tr["dst"])
    np.testing.assert_array_equal(part["edges"]["data"].view(np.uint32), tr["data"].view(np.uint32))
    np.testing.assert_array_equal(part["test_src"], ts)
    np.testing.assert_array_equal(part["test_label"], tl)
