"""GPU common neighbours (felog_common_neighbours) against the reference tool's
golden vectors and the oracle (src/tools/gcn.cpp restated)."""
import numpy as np
import pytest

import felog_b200 as fb
import oracle_binding as ob
from conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    f = fb.Felog(v_num=1, seed=1)
    yield f
    f.close()


@pytest.mark.parametrize("name", ["gcn_multi64_undirected.npz", "gcn_multi64_directed.npz",
                                  "gcn_rmat4096_undirected.npz"])
def test_gpu_matches_reference_tool(ctx, name):
    fx = load_golden(name)
    cn, _ = ctx.common_neighbours(fx["src"], fx["dst"], int(fx["v_num"]), bool(fx["undirected"]))
    np.testing.assert_array_equal(cn, fx["cn"])


@pytest.mark.parametrize("seed,undirected", [(1, True), (2, False), (3, True)])
def test_gpu_matches_oracle_on_multigraphs(ctx, seed, undirected):
    # hubs with long lists (the warp path), repeats, reciprocal pairs, self-loops
    rng = np.random.default_rng(seed)
    V = 3000
    n = 60000
    a = (rng.pareto(1.2, n) * 7).astype(np.int64) % V
    b = rng.integers(0, V, n)
    src = np.concatenate([a, b[:5000], a[:3000], np.arange(0, V, 17)]).astype(np.uint32)
    dst = np.concatenate([b, a[:5000], b[:3000], np.arange(0, V, 17)]).astype(np.uint32)
    if not undirected:  # every vertex keeps an out-edge
        src = np.concatenate([src, np.arange(V)]).astype(np.uint32)
        dst = np.concatenate([dst, (np.arange(V) + 1) % V]).astype(np.uint32)
    cn, ms = ctx.common_neighbours(src, dst, V, undirected)
    ref = ob.common_neighbours(src, dst, V, undirected)
    np.testing.assert_array_equal(cn, ref)
    assert ms > 0


def test_gpu_edge_cases(ctx):
    empty, _ = ctx.common_neighbours(np.zeros(0, np.uint32), np.zeros(0, np.uint32), 4)
    assert empty.shape == (0,)
    one, _ = ctx.common_neighbours(np.array([2], np.uint32), np.array([2], np.uint32), 3)
    np.testing.assert_array_equal(one, ob.common_neighbours([2], [2], 3))
    with pytest.raises(fb.FelogError):
        ctx.common_neighbours(np.array([0, 5], np.uint32), np.array([1, 1], np.uint32), 4)
