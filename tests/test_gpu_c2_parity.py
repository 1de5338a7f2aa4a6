"""Parity on the C2 benchmark graph itself (seed-1 R-MAT, 2,238,731 vertex ids,
34.7M undirected edges, 5% held out: 1,344,705 vertices and 65.9 M CSR
entries after the split), the mid-scale configuration the bench line is
quoted on:

* the CSR in walk.hpp's adjacency order, bit for bit against the oracle;
* round 0 of the walk (every one of the 1.34 M walkers, native Philox draws)
  bit for bit against the oracle's walker;
* the batch plan of that corpus (vocabulary, subsampling, batching,
  per-sentence plan negatives; word2vec.cu:1133-1248) against the oracle;
* the BF16 skip-gram trainer in the one-warp mode over the first sentences
  of that plan, on the full C2 tables (1.34 M rows, 13,448 FP32 master rows),
  bit for bit against the oracle's restatement.
"""
import numpy as np
import pytest

import felog_b200 as fb
import oracle_binding as ob

pytestmark = pytest.mark.gpu

SEED = 2024


@pytest.fixture(scope="module")
def c2():
    g = fb.synth_graph(seed=1, v_target=2238731, e_target=34_700_000, holdout=0.05)
    V = g["v_num"]
    c = ob.OracleCsr(g["edges"], V)
    tok, off, _, _ = ob.walk_round(c, V, 20, seed=SEED, round_=0, tok_cap=V * 64)
    vv, vcn, id2, vs, tw = ob.vocab(c.deg, 0)
    thr, used = ob.subsample_thresholds(vcn, 1e-3, tw)
    table = ob.unigram_table(vcn)
    plan = ob.plan_batches(tok, off, id2, thr, used, table, vs, 5)
    return dict(g=g, V=V, csr=c, tok=tok, off=off, vocab=(vv, vcn, id2, vs, tw), table=table, plan=plan)


def test_c2_csr_and_round0_walk_match_oracle(c2):
    g, V, c = c2["g"], c2["V"], c2["csr"]
    f = fb.Felog(v_num=V, seed=SEED)
    f.load_graph(g["edges"], V)
    row, nbr, data = f.csr()
    np.testing.assert_array_equal(row, c.row_ptr)
    np.testing.assert_array_equal(nbr, c.nbr)
    np.testing.assert_array_equal(data.view(np.uint32), c.data.view(np.uint32))
    f.walk_round(0)
    tok, off = f.corpus()
    np.testing.assert_array_equal(off, c2["off"])
    np.testing.assert_array_equal(tok, c2["tok"])
    f.close()


def test_c2_round0_plan_matches_oracle(c2):
    g, V = c2["g"], c2["V"]
    f = fb.Felog(v_num=V, size=128, window=10, negative=5, sample=1e-3, cbow=0, reuse_neg=0, min_count=0, seed=SEED)
    f.load_graph(g["edges"], V)
    f.init_model()
    f.walk_round(0)
    f.train_round(0)
    pl = f.plan()
    vv = c2["vocab"][0]
    np.testing.assert_array_equal(f.vocab()[0], vv)
    opl = c2["plan"]
    np.testing.assert_array_equal(pl["sen"], opl["sen"])
    np.testing.assert_array_equal(pl["sent_start"], opl["sent_start"])
    np.testing.assert_array_equal(pl["batch_first"], opl["batch_first"])
    np.testing.assert_array_equal(pl["negs"], opl["negs"])
    f.close()


def test_c2_bf16_skipgram_slice_matches_oracle(c2):
    """The first 3,000 walks of round 0 trained by one warp on the full C2
    tables (BF16 form) equal the oracle's restatement bit for bit."""
    g, V = c2["g"], c2["V"]
    n = 3000
    tok, off = c2["tok"][: int(c2["off"][n])], c2["off"][: n + 1]
    f = fb.Felog(v_num=V, size=128, window=10, negative=5, sample=1e-3, cbow=0, reuse_neg=0, min_count=0,
                 precision=1, deterministic=1, seed=SEED)
    f.load_graph(g["edges"], V)
    f.init_model()
    _, _, vs, _ = f.vocab()
    vv, vcn, id2, ovs, tw = c2["vocab"]
    assert vs == ovs
    nh = max(1, (vs + 99) // 100)
    o0, o1 = ob.init_net(vs, 128)
    m0, m1 = ob.MixedRows(o0, vs, 128, nh), ob.MixedRows(o1, vs, 128, nh)
    f.set_corpus(tok, off)
    alpha = 0.025
    st = f.train_round(0, alpha=alpha)
    assert st["pairs"] > 100_000
    thr, used = ob.subsample_thresholds(vcn, 1e-3, tw)
    pl = ob.plan_batches(tok, off, id2, thr, used, c2["table"], vs, 5)
    bf = pl["batch_first"]
    for b in range(len(bf) - 1):
        ob.skipgram_bf16(m0, m1, ob.round_sr_seed(SEED, 0), ob.exp_table(), c2["table"], vs, pl["sen"],
                         pl["sent_start"], int(bf[b]), int(bf[b + 1] - bf[b]), 10, 128, 5, alpha)
    g0, g1 = f.embeddings()
    exact = np.mean(g0 == m0.full()), np.mean(g1 == m1.full())
    assert exact == (1.0, 1.0), f"fraction bit-exact syn0/syn1: {exact}"
    f.close()
