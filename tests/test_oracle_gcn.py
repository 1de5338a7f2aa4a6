"""The common-neighbour oracle (src/tools/gcn.cpp restated) against the
reference tool's own output on the golden edge lists."""
import numpy as np
import pytest

import oracle_binding as ob
from conftest import load_golden


@pytest.mark.parametrize("name", ["gcn_multi64_undirected.npz", "gcn_multi64_directed.npz",
                                  "gcn_rmat4096_undirected.npz"])
def test_oracle_matches_reference_tool(name):
    fx = load_golden(name)
    cn = ob.common_neighbours(fx["src"], fx["dst"], int(fx["v_num"]), bool(fx["undirected"]))
    np.testing.assert_array_equal(cn, fx["cn"])


def test_oracle_small_cases_by_hand():
    # triangle 0-1-2 plus a pendant 3 on 2: every triangle edge has one common neighbour
    src = np.array([0, 1, 0, 2], np.uint32)
    dst = np.array([1, 2, 2, 3], np.uint32)
    np.testing.assert_array_equal(ob.common_neighbours(src, dst, 4), [1, 1, 1, 0])
    # a repeated edge: the repeat shows in both lists, the counts stay
    src2 = np.concatenate([src, [0]]).astype(np.uint32)
    dst2 = np.concatenate([dst, [1]]).astype(np.uint32)
    np.testing.assert_array_equal(ob.common_neighbours(src2, dst2, 4), [1, 1, 1, 0, 1])
