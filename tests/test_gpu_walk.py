"""GPU walker engine parity, through the C ABI.

* CSR identical to the oracle's (reference adjacency order).
* Injected draws: corpus bit-exact to the reference's own walker (golden
  fixtures produced by include/walk.hpp under the loopback harness).
* Native Philox draws: corpus bit-exact to the oracle fed the same stream;
  transition frequencies pass a chi-square test.
* Spill path, visit counts, KL, alias tables, and loud errors.
"""
import numpy as np
import pytest

import felog_b200 as fb
import oracle_binding as ob
from conftest import load_golden, walk_draws

pytestmark = pytest.mark.gpu

WALKS = ["walk_rmat512.npz", "walk_rmat512_stop_w2.npz", "walk_rmat512_minl5.npz", "walk_edgecases.npz",
         "walk_rmat4096.npz"]


def ctx_for(fx, **kw):
    V = int(fx["V"])
    f = fb.Felog(v_num=V, walker_num=int(fx["walker_num"]), min_length=int(fx["min_L"]), **kw)
    f.load_graph(fx["edges"], V, undirected=True)
    if "stop" in fx:
        f.set_stop_flags(fx["stop"])
    return f


@pytest.mark.parametrize("name", WALKS)
def test_csr_matches_oracle(name):
    fx = load_golden(name)
    f = ctx_for(fx)
    rp, nb, dt = f.csr()
    c = ob.OracleCsr(fx["edges"], int(fx["V"]))
    np.testing.assert_array_equal(rp, c.row_ptr)
    np.testing.assert_array_equal(nb, c.nbr)
    np.testing.assert_array_equal(dt.view(np.uint32), c.data.view(np.uint32))
    np.testing.assert_array_equal(f.degrees(), c.deg)


@pytest.mark.parametrize("layout", ["entries", "csr"])
@pytest.mark.parametrize("name", WALKS)
def test_walk_injected_bit_exact_to_reference(name, layout):
    """Both walker layouts: the walker entries (the default) and the plain CSR
    (after felog_walk_entries frees the entries, as for graphs above 2^31
    entries)."""
    fx = load_golden(name)
    f = ctx_for(fx)
    if layout == "csr":
        assert f.walk_entries(keep=False) == 0
    else:
        assert f.walk_entries() == 16 * len(f.csr()[1])
    for r in range(int(fx["rounds"])):
        st = f.walk_round(r, draws=walk_draws(fx, r))
        tok, off = f.corpus()
        np.testing.assert_array_equal(off, fx[f"r{r}_off"])
        np.testing.assert_array_equal(tok, fx[f"r{r}_tokens"])
        assert st["n_tokens"] == len(tok)


@pytest.mark.parametrize("name,rounds,slot", [("walk_rmat4096.npz", 3, 64), ("walk_edgecases.npz", 3, 64),
                                              ("walk_rmat512_stop_w2.npz", 2, 8), ("walk_rmat512.npz", 2, 4)])
@pytest.mark.parametrize("layout", ["entries", "csr"])
def test_walk_philox_bit_exact_to_oracle(name, rounds, slot, layout):
    fx = load_golden(name)
    f = ctx_for(fx, seed=1234, slot_len=slot)
    if layout == "csr":
        f.walk_entries(keep=False)
    V = int(fx["V"])
    c = ob.OracleCsr(fx["edges"], V)
    for r in range(rounds):
        st = f.walk_round(r)
        tok, off = f.corpus()
        otok, ooff, _, ost = ob.walk_round(c, int(fx["walker_num"]), int(fx["min_L"]), seed=1234, round_=r,
                                           stop_flags=fx.get("stop"))
        np.testing.assert_array_equal(off, ooff)
        np.testing.assert_array_equal(tok, otok)
        assert st["n_traces"] == ost.n_traces and st["n_iterations"] == ost.n_iterations
        if slot < 22:
            assert st["n_long"] == st["n_sentences"]


def test_walk_long_min_length_spills():
    """min_L 100 makes every walk longer than the 64-token slot."""
    fx = load_golden("walk_rmat512.npz")
    V = int(fx["V"])
    f = fb.Felog(v_num=V, min_length=100, seed=9)
    f.load_graph(fx["edges"], V)
    st = f.walk_round(0)
    tok, off = f.corpus()
    c = ob.OracleCsr(fx["edges"], V)
    otok, ooff, _, _ = ob.walk_round(c, V, 100, seed=9, round_=0)
    np.testing.assert_array_equal(off, ooff)
    np.testing.assert_array_equal(tok, otok)
    assert st["n_long"] == V


def test_first_step_transitions_uniform_chisq():
    """Step-0 candidate draws are uniform over the start's neighbours (walk.hpp:976)."""
    fx = load_golden("walk_rmat512.npz")
    V = int(fx["V"])
    c = ob.OracleCsr(fx["edges"], V)
    hub = int(np.argmax(c.deg))
    R = 200 * int(c.deg[hub])  # walkers per start vertex
    f = fb.Felog(v_num=V, walker_num=V * R, min_length=1, seed=77)
    f.load_graph(fx["edges"], V)
    stop = np.ones(V, np.uint8)
    stop[hub] = 0
    f.set_stop_flags(stop)
    f.walk_round(0)
    tok, off = f.corpus()
    first = tok[off[:-1].astype(np.int64) + 1]
    nbrs = c.nbr[c.row_ptr[hub]:c.row_ptr[hub + 1]]
    expect = np.bincount(nbrs, minlength=V).astype(np.float64)
    expect = expect / expect.sum() * len(first)
    obs = np.bincount(first, minlength=V).astype(np.float64)
    m = expect > 0
    assert obs[~m].sum() == 0
    chi2 = ((obs[m] - expect[m]) ** 2 / expect[m]).sum()
    dof = m.sum() - 1
    assert chi2 < dof + 6 * np.sqrt(2 * dof), (chi2, dof)


def test_visit_freq_and_kl_match_oracle():
    fx = load_golden("walk_rmat4096.npz")
    V = int(fx["V"])
    f = fb.Felog(v_num=V, seed=5)
    f.load_graph(fx["edges"], V)
    total = np.zeros(V, np.uint64)
    for r in range(2):
        st = f.walk_round(r)
        tok, _ = f.corpus()
        total += np.bincount(tok, minlength=V).astype(np.uint64)
        np.testing.assert_array_equal(f.visit_freq(), total)
        kl = ob.round_kl(f.degrees(), total)
        assert abs(st["kl"] - kl) <= 1e-12 * max(1.0, abs(kl))


def test_alias_tables_reproduce_weights():
    g = fb.synth_graph(seed=2, v_target=1024, e_target=4096, abcd=(0.6, 0.15, 0.15, 0.1), lognormal=True)
    V = g["v_num"]
    f = fb.Felog(v_num=V)
    f.load_graph(g["edges"], V)
    f.build_alias()
    prob, alias = f.alias()
    rp, nb, dt = f.csr()
    for v in range(0, V, 7):
        b, e = int(rp[v]), int(rp[v + 1])
        n = e - b
        if n == 0:
            continue
        mass = np.zeros(n)
        for j in range(n):
            mass[j] += prob[b + j]
            mass[alias[b + j]] += 1.0 - prob[b + j]
        w = dt[b:e].astype(np.float64)
        np.testing.assert_allclose(mass / n, w / w.sum(), atol=2e-6)


def test_weighted_walk_follows_alias_distribution():
    g = fb.synth_graph(seed=2, v_target=1024, e_target=4096, abcd=(0.6, 0.15, 0.15, 0.1), lognormal=True)
    V = g["v_num"]
    f = fb.Felog(v_num=V, walker_num=V * 3000, min_length=1, weighted=1, seed=3)
    f.load_graph(g["edges"], V)
    f.build_alias()
    rp, nb, dt = f.csr()
    deg = np.diff(rp)
    v0 = int(np.argsort(deg)[-5])
    stop = np.ones(V, np.uint8)
    stop[v0] = 0
    f.set_stop_flags(stop)
    f.walk_round(0)
    tok, off = f.corpus()
    first = tok[off[:-1].astype(np.int64) + 1]
    b, e = int(rp[v0]), int(rp[v0 + 1])
    w = np.zeros(V)
    np.add.at(w, nb[b:e], dt[b:e].astype(np.float64))
    expect = w / w.sum() * len(first)
    obs = np.bincount(first, minlength=V).astype(np.float64)
    m = expect > 5
    chi2 = ((obs[m] - expect[m]) ** 2 / expect[m]).sum()
    dof = m.sum() - 1
    assert chi2 < dof + 6 * np.sqrt(2 * dof), (chi2, dof)


def test_injected_draws_too_short_is_an_error():
    fx = load_golden("walk_rmat512.npz")
    f = ctx_for(fx)
    idx_off, idx, p_off, p = walk_draws(fx, 0)
    short = idx_off.copy()
    short[1:] = np.minimum(short[1:], short[:-1] + 3)  # every walker gets <= 3 index draws
    with pytest.raises(fb.FelogError) as ei:
        f.walk_round(0, draws=(short, idx, p_off, p))
    assert ei.value.status == 1
    # the context stays usable
    f.walk_round(0, draws=walk_draws(fx, 0))


def test_bad_vertex_is_an_error():
    e = np.zeros(3, fb.EDGE12)
    e["src"] = [0, 1, 5]
    e["dst"] = [1, 2, 0]
    f = fb.Felog(v_num=3)
    with pytest.raises(fb.FelogError) as ei:
        f.load_graph(e, 3)
    assert ei.value.status == 1


def test_walk_ceiling_skeleton_leaves_corpus():
    """felog_walk_ceiling times a memory skeleton of the last round (same walkers
    and token counts) without touching the round's corpus."""
    g = fb.synth_graph(seed=5, v_target=8192, e_target=65536, holdout=0.0)
    V = g["v_num"]
    f = fb.Felog(v_num=V, seed=9)
    f.load_graph(g["edges"], V)
    with pytest.raises(fb.FelogError):
        f.walk_ceiling()  # no walk round yet
    ws = f.walk_round(0)
    tok0, off0 = f.corpus()
    ms, tokens = f.walk_ceiling()
    assert ms > 0 and tokens == ws["n_tokens"]
    tok1, off1 = f.corpus()
    assert np.array_equal(tok0, tok1) and np.array_equal(off0, off1)
    f.close()
