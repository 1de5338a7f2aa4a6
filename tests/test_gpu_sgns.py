"""GPU trainer parity through the C ABI.

* Batch plan (sentence packing, subsampling draws, per-batch negatives,
  per-sentence seeds) identical to the oracle, which the golden fixtures pin
  to the reference's TrainModelThreadMemory.
* Skip-gram: the one-warp deterministic mode reproduces the oracle's
  sequential restatement of skip_gram_kernel; the tolerance of the path is
  1e-5 relative (FP32), and the dot-product order and FMA placement are the
  reference kernel's, so the expected difference is zero.
* The reference's own skip_gram_kernel (oracle/_ref, run one sentence per
  launch) agrees with the oracle.
"""
import ctypes
import hashlib
import os

import numpy as np
import pytest

import felog_b200 as fb
import oracle_binding as ob
from conftest import ROOT, load_golden
from recipes import pack, synth_corpus

pytestmark = pytest.mark.gpu

RTOL = 1e-5


def graph4096():
    fx = load_golden("walk_rmat4096.npz")
    return fx["edges"], int(fx["V"])


def trainer(dim=128, window=10, negative=5, sample=1e-3, reuse_neg=0, cbow=0, **kw):
    e, V = graph4096()
    f = fb.Felog(v_num=V, size=dim, window=window, negative=negative, sample=sample, cbow=cbow, reuse_neg=reuse_neg,
                 min_count=0, **kw)
    f.load_graph(e, V)
    f.init_model()
    return f, e, V


@pytest.mark.parametrize("name", ["plan_multibatch.npz", "plan_subsample.npz", "plan_nosample_long.npz",
                                  "plan_tokens_sub.npz"])
def test_plan_matches_reference(name):
    fx = load_golden(name)
    f, e, V = trainer(dim=int(fx["dim"]), window=int(fx["window"]), negative=int(fx["negative"]),
                      sample=float(fx["sample"]))
    vv, id2, vs, tw = f.vocab()
    np.testing.assert_array_equal(vv, fx["vocab_vertex"])
    rc = fx["recipe"]
    tok, off = pack(synth_corpus(int(rc[0]), int(rc[1]), int(rc[2]), int(rc[3]), int(rc[4]), int(rc[5])))
    f.set_corpus(tok, off)
    f.train_round(0, alpha=0.0)
    pl = f.plan()
    assert hashlib.sha256(pl["sen"].tobytes()).hexdigest() == fx["sen_sha256"].item().decode()
    assert hashlib.sha256(pl["negs"].tobytes()).hexdigest() == fx["negs_sha256"].item().decode()
    np.testing.assert_array_equal(np.diff(pl["batch_first"]).astype(np.int64), fx["batch_cnt"])
    bf = pl["batch_first"]
    sl = [(pl["sent_start"][bf[b]:bf[b + 1] + 1] - pl["sent_start"][bf[b]]).astype(np.int32)
          for b in range(len(bf) - 1)]
    np.testing.assert_array_equal(np.concatenate(sl), fx["sentence_length"])


def oracle_train(f, e, V, tok, off, dim, window, negative, sample, alpha, rounds=1, cbow=False):
    """The oracle's sequential training of the same corpus, batch after batch."""
    c = ob.OracleCsr(e, V)
    vv, vcn, id2, vs, tw = ob.vocab(c.deg, 0)
    thr, used = ob.subsample_thresholds(vcn, sample, tw)
    table = ob.unigram_table(vcn)
    et = ob.exp_table()
    syn0, syn1 = ob.init_net(vs, dim)
    for _ in range(rounds):
        pl = ob.plan_batches(tok, off, id2, thr, used, table, vs, negative)
        bf = pl["batch_first"]
        for b in range(len(bf) - 1):
            ob.skipgram_batch(syn0, syn1, et, table, vs, pl["sen"], pl["sent_start"], int(bf[b]),
                              int(bf[b + 1] - bf[b]), window, dim, negative, alpha, cbow=cbow)
    return syn0, syn1


def walk_corpus(V, e, seed=21, walker_num=None):
    c = ob.OracleCsr(e, V)
    tok, off, _, _ = ob.walk_round(c, walker_num or V, 20, seed=seed, round_=0)
    return tok, off


@pytest.mark.parametrize("dim", [32, 64, 128, 256])
def test_skipgram_deterministic_matches_oracle(dim):
    f, e, V = trainer(dim=dim, window=10, negative=5, sample=1e-3, deterministic=1)
    tok, off = walk_corpus(V, e)
    n = 400  # sentences
    tok, off = tok[: int(off[n])], off[: n + 1]
    s0_init, _ = f.embeddings()
    o0, o1 = ob.init_net(f.vocab()[2], dim)
    np.testing.assert_array_equal(s0_init, o0)
    f.set_corpus(tok, off)
    f.train_round(0, alpha=0.025)
    g0, g1 = f.embeddings()
    r0, r1 = oracle_train(f, e, V, tok, off, dim, 10, 5, 1e-3, 0.025)
    np.testing.assert_allclose(g0, r0, rtol=RTOL, atol=1e-7)
    np.testing.assert_allclose(g1, r1, rtol=RTOL, atol=1e-7)
    exact = np.mean(g0 == r0), np.mean(g1 == r1)
    assert exact == (1.0, 1.0), f"fraction bit-exact syn0/syn1: {exact}"


def test_skipgram_two_rounds_and_multibatch_deterministic():
    f, e, V = trainer(dim=64, window=5, negative=7, sample=1e-4, deterministic=1)
    tok, off = pack(synth_corpus(V, 16000, 3, 0, 1, 6))  # 2 batches by sentence count
    f.set_corpus(tok, off)
    for r in range(2):
        st = f.train_round(r, alpha=0.02)
        assert st["batches"] == 2
    g0, g1 = f.embeddings()
    r0, r1 = oracle_train(f, e, V, tok, off, 64, 5, 7, 1e-4, 0.02, rounds=2)
    np.testing.assert_allclose(g0, r0, rtol=RTOL, atol=1e-7)
    np.testing.assert_allclose(g1, r1, rtol=RTOL, atol=1e-7)


REF_SO = os.path.join(ROOT, "oracle", "_ref", "libref_sgns_gpu.so")


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference harness not built")
def test_reference_skip_gram_kernel_matches_oracle():
    """The reference's own skip_gram_kernel, one sentence per launch with its
    batch index as blockIdx.x, against the oracle's sequential restatement."""
    e, V = graph4096()
    dim, window, K, alpha = 128, 10, 5, 0.025
    c = ob.OracleCsr(e, V)
    vv, vcn, id2, vs, tw = ob.vocab(c.deg, 0)
    thr, used = ob.subsample_thresholds(vcn, 1e-3, tw)
    table = ob.unigram_table(vcn)
    et = ob.exp_table()
    tok, off = walk_corpus(V, e, seed=5)
    n = 120
    tok, off = tok[: int(off[n])], off[: n + 1]
    pl = ob.plan_batches(tok, off, id2, thr, used, table, vs, K)
    assert len(pl["batch_first"]) == 2
    s0, s1 = ob.init_net(vs, dim)
    # make syn1 non-trivial so every dot product is exercised
    s1[:] = np.sin(np.arange(len(s1), dtype=np.float64)).astype(np.float32) * 0.01
    r0, r1 = s0.copy(), s1.copy()
    L = ctypes.CDLL(REF_SO)
    L.ref_sgns_run_sentencewise.argtypes = [ctypes.c_int] * 4 + [ctypes.c_longlong] + [ctypes.c_void_p] * 3 + \
        [ctypes.c_int64] + [ctypes.c_void_p] * 3 + [ctypes.c_int, ctypes.c_float]
    sen = np.ascontiguousarray(pl["sen"], np.int32)
    ss = np.ascontiguousarray(pl["sent_start"].astype(np.int64))
    rc = L.ref_sgns_run_sentencewise(0, dim, window, K, vs, r0.ctypes.data, r1.ctypes.data, table.ctypes.data,
                                     len(table), et.ctypes.data, sen.ctypes.data, ss.ctypes.data, n, alpha)
    assert rc == 0
    ob.skipgram_batch(s0, s1, et, table, vs, sen, pl["sent_start"], 0, n, window, dim, K, alpha)
    np.testing.assert_allclose(r0, s0, rtol=RTOL, atol=1e-7)
    np.testing.assert_allclose(r1, s1, rtol=RTOL, atol=1e-7)
    exact = np.mean(r0 == s0), np.mean(r1 == s1)
    print("reference kernel vs oracle, fraction bit-exact:", exact)


def link_auc(s0, s1, id2, vs, dim, g):
    """Exact AUC of held-out edges vs non-edges: cosine(syn0, syn0) and syn0 . syn1 scores."""
    e0 = s0.reshape(vs, dim)[id2]
    e1 = s1.reshape(vs, dim)[id2]
    n0 = e0 / np.linalg.norm(e0, axis=1, keepdims=True)
    cos = np.sum(n0[g["test_src"]] * n0[g["test_dst"]], axis=1)
    d01 = np.sum(e0[g["test_src"]] * e1[g["test_dst"]], 1) + np.sum(e0[g["test_dst"]] * e1[g["test_src"]], 1)
    return fb.auc(cos, g["test_label"]), fb.auc(d01, g["test_label"])


def test_hogwild_auc_within_0005_of_sequential_oracle():
    """Hogwild training on the GPU (thousands of warps racing on shared rows)
    against the oracle's strictly sequential training of the same walks: the
    link-prediction AUC agrees within 0.005."""
    g = fb.synth_graph(seed=3, v_target=4096, e_target=32768, holdout=0.1)
    V = g["v_num"]
    f = fb.Felog(v_num=V, size=128, window=10, negative=5, sample=1e-3, cbow=0, reuse_neg=0, min_count=0,
                 seed=17)
    f.load_graph(g["edges"], V)
    f.init_model()
    c = ob.OracleCsr(g["edges"], V)
    vv, vcn, id2o, vs, tw = ob.vocab(c.deg, 0)
    thr, used = ob.subsample_thresholds(vcn, 1e-3, tw)
    table = ob.unigram_table(vcn)
    et = ob.exp_table()
    o0, o1 = ob.init_net(vs, 128)
    for r in range(3):
        f.walk_round(r)
        st = f.train_round(r)
        assert st["kept_words"] > 0
        tok, off, _, _ = ob.walk_round(c, V, 20, seed=17, round_=r)
        gtok, goff = f.corpus()
        assert np.array_equal(tok, gtok)
        pl = ob.plan_batches(tok, off, id2o, thr, used, table, vs, 5)
        bf = pl["batch_first"]
        for b in range(len(bf) - 1):
            ob.skipgram_batch(o0, o1, et, table, vs, pl["sen"], pl["sent_start"], int(bf[b]), int(bf[b + 1] - bf[b]),
                              10, 128, 5, ob.lr(0.025, 0.1, r))
    s0, s1 = f.embeddings()
    _, id2, _, _ = f.vocab()
    assert np.isfinite(s0).all() and np.isfinite(s1).all()
    a_gpu = link_auc(s0, s1, id2, vs, 128, g)
    a_orc = link_auc(o0, o1, id2o, vs, 128, g)
    # the defined metric is the cosine of syn0 rows (the similarity of the
    # convergence check); the syn0 . syn1 score is printed for information
    print("AUC cosine / syn0.syn1: gpu", a_gpu, "oracle", a_orc)
    assert abs(a_gpu[0] - a_orc[0]) < 0.005, (a_gpu, a_orc)


@pytest.mark.parametrize("dim,negative", [(128, 5), (64, 7), (256, 5)])
def test_reuse_neg_deterministic_matches_oracle(dim, negative):
    """-reuse-neg 1 (per-sentence plan negatives, full window) in the one-warp
    mode equals the oracle's restatement of __sgNegReuse with true dots."""
    f, e, V = trainer(dim=dim, window=5, negative=negative, sample=1e-3, deterministic=1, reuse_neg=1)
    tok, off = walk_corpus(V, e, seed=9)
    n = 300
    tok, off = tok[: int(off[n])], off[: n + 1]
    f.set_corpus(tok, off)
    f.train_round(0, alpha=0.025)
    g0, g1 = f.embeddings()
    c = ob.OracleCsr(e, V)
    vv, vcn, id2, vs, tw = ob.vocab(c.deg, 0)
    thr, used = ob.subsample_thresholds(vcn, 1e-3, tw)
    table = ob.unigram_table(vcn)
    et = ob.exp_table()
    syn0, syn1 = ob.init_net(vs, dim)
    pl = ob.plan_batches(tok, off, id2, thr, used, table, vs, negative)
    gp = f.plan()
    assert np.array_equal(gp["negs"], pl["negs"])
    bf = pl["batch_first"]
    for b in range(len(bf) - 1):
        ob.negreuse_batch(syn0, syn1, et, pl["sen"], pl["sent_start"], int(bf[b]), int(bf[b + 1] - bf[b]),
                          pl["negs"], 5, dim, negative, 0.025)
    exact = np.mean(g0 == syn0), np.mean(g1 == syn1)
    assert exact == (1.0, 1.0), f"fraction bit-exact syn0/syn1: {exact}"


@pytest.mark.parametrize("dim,negative", [(128, 5), (64, 3)])
def test_cbow_deterministic_matches_oracle(dim, negative):
    """-cbow 1 (cbow_kernel, word2vec.cu:538-646) in the one-warp mode, FP32
    form, against the oracle's sequential restatement."""
    f, e, V = trainer(dim=dim, window=5, negative=negative, sample=1e-3, deterministic=1, cbow=1)
    tok, off = walk_corpus(V, e, seed=13)
    n = 300
    tok, off = tok[: int(off[n])], off[: n + 1]
    f.set_corpus(tok, off)
    f.train_round(0, alpha=0.05)
    g0, g1 = f.embeddings()
    r0, r1 = oracle_train(f, e, V, tok, off, dim, 5, negative, 1e-3, 0.05, cbow=True)
    np.testing.assert_allclose(g0, r0, rtol=RTOL, atol=1e-7)
    np.testing.assert_allclose(g1, r1, rtol=RTOL, atol=1e-7)
    exact = np.mean(g0 == r0), np.mean(g1 == r1)
    print("cbow fraction bit-exact syn0/syn1:", exact)


def test_pair_row_mix_counts_master_rows():
    """felog_pair_row_mix: row references of the last pair-stream chunk; every
    reference is a master row in the FP32 form, a share of them in BF16."""
    g = fb.synth_graph(seed=6, v_target=8192, e_target=65536, holdout=0.0)
    V = g["v_num"]
    out = {}
    for prec in (0, 1):
        f = fb.Felog(v_num=V, size=128, window=10, negative=5, sample=1e-3, cbow=0, reuse_neg=0, min_count=0,
                     seed=3, precision=prec)
        f.load_graph(g["edges"], V)
        f.init_model()
        with pytest.raises(fb.FelogError):
            f.pair_row_mix()
        f.walk_round(0)
        ts = f.train_round(0)
        out[prec] = f.pair_row_mix()
        f.close()
        pairs, refs, hot = out[prec]
        assert pairs == ts["pairs"] and pairs < refs <= 7 * pairs
    assert out[0][2] == out[0][1]
    assert 0 < out[1][2] < out[1][1]
