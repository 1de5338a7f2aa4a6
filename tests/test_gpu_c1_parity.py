"""Parity on the C1 benchmark graph itself (seed-0 R-MAT, 16,384 vertex ids,
131,072 undirected edges, 10% held out), not only on the small fixtures:

* the CSR (walk.hpp's adjacency order), two walk rounds with the native
  Philox draws and the round KL against the oracle, bit for bit;
* the batch plan of the round-0 corpus (vocabulary, subsampling, batching,
  per-sentence plan negatives; word2vec.cu:1133-1248) against the oracle;
* the convergence check after two trained rounds against the oracle.
"""
import numpy as np
import pytest

import felog_b200 as fb
import oracle_binding as ob

pytestmark = pytest.mark.gpu

SEED = 2024


@pytest.fixture(scope="module")
def c1():
    return fb.synth_graph(seed=0, v_target=16384, e_target=131072, holdout=0.10)


def test_c1_csr_and_philox_walks_match_oracle(c1):
    e, V = c1["edges"], c1["v_num"]
    f = fb.Felog(v_num=V, seed=SEED)
    f.load_graph(e, V)
    c = ob.OracleCsr(e, V)
    row, nbr, data = f.csr()
    np.testing.assert_array_equal(row, c.row_ptr)
    np.testing.assert_array_equal(nbr, c.nbr)
    np.testing.assert_array_equal(data.view(np.uint32), c.data.view(np.uint32))
    for r in range(2):
        st = f.walk_round(r)
        tok, off = f.corpus()
        otok, ooff, _, ost = ob.walk_round(c, V, 20, seed=SEED, round_=r)
        np.testing.assert_array_equal(off, ooff)
        np.testing.assert_array_equal(tok, otok)
    f.close()


def test_c1_batch_plan_matches_oracle(c1):
    e, V = c1["edges"], c1["v_num"]
    f = fb.Felog(v_num=V, size=128, window=10, negative=5, sample=1e-3, cbow=0, reuse_neg=0, min_count=0, seed=SEED)
    f.load_graph(e, V)
    f.init_model()
    f.walk_round(0)
    tok, off = f.corpus()
    f.train_round(0)
    pl = f.plan()
    c = ob.OracleCsr(e, V)
    vv, vcn, id2, vs, tw = ob.vocab(c.deg, 0)
    np.testing.assert_array_equal(f.vocab()[0], vv)
    thr, used = ob.subsample_thresholds(vcn, 1e-3, tw)
    table = ob.unigram_table(vcn)
    opl = ob.plan_batches(tok, off, id2, thr, used, table, vs, 5)
    np.testing.assert_array_equal(pl["sen"], opl["sen"])
    np.testing.assert_array_equal(pl["sent_start"], opl["sent_start"])
    np.testing.assert_array_equal(pl["batch_first"], opl["batch_first"])
    np.testing.assert_array_equal(pl["negs"], opl["negs"])
    f.close()


def test_c1_convergence_check_matches_oracle(c1):
    e, V = c1["edges"], c1["v_num"]
    f = fb.Felog(v_num=V, size=128, window=10, negative=5, cbow=0, reuse_neg=0, min_count=0, seed=SEED)
    f.load_graph(e, V)
    f.init_model()
    for r in range(2):
        f.walk_round(r)
        f.train_round(r)
    s0, _ = f.embeddings()
    _, id2, _, _ = f.vocab()
    flags0 = np.zeros(V, np.uint8)
    f.set_stop_flags(flags0)
    st = f.budget_check(1)
    c = ob.OracleCsr(e, V)
    eva, oflags, osim = ob.convergence(s0, id2, 128, c, flags0, f.opts.seed, 1)
    np.testing.assert_array_equal(f.stop_flags(), oflags)
    np.testing.assert_array_equal(f.similarity(), osim)
    assert st["unconverged"] == eva and st["evaluated"] == V
    f.close()
