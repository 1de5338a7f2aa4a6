"""BF16 storage form through the C ABI.

The form: FP32 master rows for the top 1% of the vocabulary (rows
0..n_hot-1, the vocabulary being sorted by degree), BF16 rows after them,
FP32 arithmetic, stochastically rounded write-back (rule in the oracle,
oracle/felog_oracle.c, orc_skipgram_bf16).

* The one-warp deterministic mode equals the oracle's restatement bit for
  bit (skip-gram through the multi-target path, the any-K path, dim 32, CBOW).
* Hogwild BF16 training reaches a link-prediction AUC within 0.005 of the
  FP32 form on the same walks (the precision bar).
* Precision study: on 1,024 fixed seeded batches the trainer's dots and the
  batch losses from the stored tables are compared with FP64 recomputations
  from the FP32 tables; the error bound is the one BF16 storage implies.
"""
import numpy as np
import pytest

import felog_b200 as fb
import oracle_binding as ob
from conftest import load_golden

pytestmark = pytest.mark.gpu

SEED = 0x5EED0001


def graph4096():
    fx = load_golden("walk_rmat4096.npz")
    return fx["edges"], int(fx["V"])


def n_hot(vocab_size):
    return max(1, (vocab_size + 99) // 100)


def walk_corpus(V, e, n_sent, seed=21):
    c = ob.OracleCsr(e, V)
    tok, off, _, _ = ob.walk_round(c, V, 20, seed=seed, round_=0)
    return tok[: int(off[n_sent])], off[: n_sent + 1]


@pytest.mark.parametrize("dim,negative,cbow", [(128, 5, 0), (64, 5, 0), (256, 7, 0), (128, 3, 0), (32, 5, 0),
                                               (128, 5, 1)])
def test_bf16_deterministic_matches_oracle(dim, negative, cbow):
    e, V = graph4096()
    f = fb.Felog(v_num=V, size=dim, window=10, negative=negative, sample=1e-3, cbow=cbow, reuse_neg=0, min_count=0,
                 precision=1, deterministic=1, seed=SEED)
    f.load_graph(e, V)
    f.init_model()
    _, _, vs, _ = f.vocab()
    nh = n_hot(vs)
    o0, o1 = ob.init_net(vs, dim)
    m0, m1 = ob.MixedRows(o0, vs, dim, nh), ob.MixedRows(o1, vs, dim, nh)
    g0, g1 = f.embeddings()
    np.testing.assert_array_equal(g0, m0.full())  # InitNet, BF16 rows rounded to nearest
    np.testing.assert_array_equal(g1, m1.full())
    tok, off = walk_corpus(V, e, 300)
    f.set_corpus(tok, off)
    alpha = 0.025
    f.train_round(0, alpha=alpha)
    c = ob.OracleCsr(e, V)
    vv, vcn, id2, vs2, tw = ob.vocab(c.deg, 0)
    assert vs2 == vs
    thr, used = ob.subsample_thresholds(vcn, 1e-3, tw)
    table = ob.unigram_table(vcn)
    et = ob.exp_table()
    pl = ob.plan_batches(tok, off, id2, thr, used, table, vs, negative)
    bf = pl["batch_first"]
    for b in range(len(bf) - 1):
        ob.skipgram_bf16(m0, m1, ob.round_sr_seed(SEED, 0), et, table, vs, pl["sen"], pl["sent_start"], int(bf[b]),
                         int(bf[b + 1] - bf[b]), 10, dim, negative, alpha, cbow=bool(cbow))
    g0, g1 = f.embeddings()
    r0, r1 = m0.full(), m1.full()
    assert not np.array_equal(r0, ob.MixedRows(o0, vs, dim, nh).full())  # training moved the rows
    exact = np.mean(g0 == r0), np.mean(g1 == r1)
    assert exact == (1.0, 1.0), f"fraction bit-exact syn0/syn1: {exact}"


@pytest.mark.parametrize("dim", [128, 64])
def test_bf16_reuse_neg_deterministic_matches_oracle(dim):
    e, V = graph4096()
    f = fb.Felog(v_num=V, size=dim, window=5, negative=5, sample=1e-3, cbow=0, reuse_neg=1, min_count=0,
                 precision=1, deterministic=1, seed=SEED)
    f.load_graph(e, V)
    f.init_model()
    _, _, vs, _ = f.vocab()
    nh = n_hot(vs)
    o0, o1 = ob.init_net(vs, dim)
    m0, m1 = ob.MixedRows(o0, vs, dim, nh), ob.MixedRows(o1, vs, dim, nh)
    tok, off = walk_corpus(V, e, 300, seed=4)
    f.set_corpus(tok, off)
    f.train_round(0, alpha=0.025)
    c = ob.OracleCsr(e, V)
    vv, vcn, id2, _, tw = ob.vocab(c.deg, 0)
    thr, used = ob.subsample_thresholds(vcn, 1e-3, tw)
    table = ob.unigram_table(vcn)
    pl = ob.plan_batches(tok, off, id2, thr, used, table, vs, 5)
    bf = pl["batch_first"]
    for b in range(len(bf) - 1):
        ob.negreuse_bf16(m0, m1, ob.round_sr_seed(SEED, 0), ob.exp_table(), pl["sen"], pl["sent_start"], int(bf[b]),
                         int(bf[b + 1] - bf[b]), pl["negs"], 5, dim, 5, 0.025)
    g0, g1 = f.embeddings()
    exact = np.mean(g0 == m0.full()), np.mean(g1 == m1.full())
    assert exact == (1.0, 1.0), f"fraction bit-exact syn0/syn1: {exact}"


@pytest.mark.parametrize("precision,dim,negative", [(0, 128, 5), (1, 128, 5), (0, 64, 7), (1, 256, 5)])
def test_reuse_tile_deterministic_matches_oracle(precision, dim, negative):
    """-reuse-neg 2 (one tile per center) in the one-warp mode, FP32 and BF16
    forms, against the oracle's restatement."""
    e, V = graph4096()
    f = fb.Felog(v_num=V, size=dim, window=5, negative=negative, sample=1e-3, cbow=0, reuse_neg=2, min_count=0,
                 precision=precision, deterministic=1, seed=SEED)
    f.load_graph(e, V)
    f.init_model()
    _, _, vs, _ = f.vocab()
    nh = n_hot(vs) if precision else vs
    o0, o1 = ob.init_net(vs, dim)
    m0, m1 = ob.MixedRows(o0, vs, dim, nh), ob.MixedRows(o1, vs, dim, nh)
    tok, off = walk_corpus(V, e, 300, seed=6)
    f.set_corpus(tok, off)
    f.train_round(0, alpha=0.025)
    c = ob.OracleCsr(e, V)
    vv, vcn, id2, _, tw = ob.vocab(c.deg, 0)
    thr, used = ob.subsample_thresholds(vcn, 1e-3, tw)
    table = ob.unigram_table(vcn)
    pl = ob.plan_batches(tok, off, id2, thr, used, table, vs, negative)
    bf = pl["batch_first"]
    for b in range(len(bf) - 1):
        ob.negreuse_tile(m0, m1, ob.round_sr_seed(SEED, 0), ob.exp_table(), pl["sen"], pl["sent_start"], int(bf[b]),
                         int(bf[b + 1] - bf[b]), pl["negs"], 5, dim, negative, 0.025)
    g0, g1 = f.embeddings()
    exact = np.mean(g0 == m0.full()), np.mean(g1 == m1.full())
    assert exact == (1.0, 1.0), f"fraction bit-exact syn0/syn1: {exact}"


@pytest.mark.parametrize("precision,dim,negative,window", [(0, 128, 5, 10), (1, 128, 5, 10), (1, 64, 7, 5),
                                                            (0, 256, 5, 3)])
def test_window_tile_deterministic_matches_oracle(precision, dim, negative, window):
    """-reuse-neg 4 (window tiles: skip-gram windows, each center's first draws
    shared by its contexts) in the one-warp mode against the oracle."""
    e, V = graph4096()
    f = fb.Felog(v_num=V, size=dim, window=window, negative=negative, sample=1e-3, cbow=0, reuse_neg=4,
                 min_count=0, precision=precision, deterministic=1, seed=SEED)
    f.load_graph(e, V)
    f.init_model()
    _, _, vs, _ = f.vocab()
    nh = n_hot(vs) if precision else vs
    o0, o1 = ob.init_net(vs, dim)
    m0, m1 = ob.MixedRows(o0, vs, dim, nh), ob.MixedRows(o1, vs, dim, nh)
    tok, off = walk_corpus(V, e, 300, seed=8)
    f.set_corpus(tok, off)
    st = f.train_round(0, alpha=0.025)
    c = ob.OracleCsr(e, V)
    vv, vcn, id2, _, tw = ob.vocab(c.deg, 0)
    thr, used = ob.subsample_thresholds(vcn, 1e-3, tw)
    table = ob.unigram_table(vcn)
    pl = ob.plan_batches(tok, off, id2, thr, used, table, vs, negative)
    bf = pl["batch_first"]
    for b in range(len(bf) - 1):
        ob.window_tile(m0, m1, ob.round_sr_seed(SEED, 0), ob.exp_table(), table, vs, pl["sen"], pl["sent_start"],
                       int(bf[b]), int(bf[b + 1] - bf[b]), window, dim, negative, 0.025)
    g0, g1 = f.embeddings()
    assert not np.array_equal(m0.full(), ob.MixedRows(o0, vs, dim, nh).full())  # training moved the rows
    exact = np.mean(g0 == m0.full()), np.mean(g1 == m1.full())
    assert exact == (1.0, 1.0), f"fraction bit-exact syn0/syn1: {exact}"
    # the windows are the skip-gram windows: as many pairs as the pair stream trains
    f2 = fb.Felog(v_num=V, size=dim, window=window, negative=negative, sample=1e-3, cbow=0, reuse_neg=0,
                  min_count=0, precision=precision, deterministic=1, seed=SEED)
    f2.load_graph(e, V)
    f2.init_model()
    f2.set_corpus(tok, off)
    st2 = f2.train_round(0, alpha=0.025)
    assert st["pairs"] == st2["pairs"] > 0
    f.close()
    f2.close()


@pytest.mark.parametrize("dim,negative", [(128, 5), (64, 7)])
def test_reuse_tile_tensor_core_matches_oracle(dim, negative):
    """-reuse-neg 3 (BF16 form, center tiles scored by tcgen05.mma BF16) in the
    one-warp mode against the oracle's restatement with FP64 dots of the same
    BF16 operands.  The tensor core's FP32 accumulation order is unspecified,
    so a score can differ in its last bits and flip a stochastic rounding that
    later centers then read: the tables must agree bit for bit on >= 99% of the
    values, within a few BF16 ulps (2^-5 relative, 1e-6 absolute) on >= 99.9%,
    and within 2^-5 relative plus 1e-3 absolute everywhere (the drift a flipped
    rounding leaves after it has passed through later centers' gradients)."""
    e, V = graph4096()
    f = fb.Felog(v_num=V, size=dim, window=5, negative=negative, sample=1e-3, cbow=0, reuse_neg=3, min_count=0,
                 precision=1, deterministic=1, seed=SEED)
    f.load_graph(e, V)
    f.init_model()
    _, _, vs, _ = f.vocab()
    nh = n_hot(vs)
    o0, o1 = ob.init_net(vs, dim)
    m0, m1 = ob.MixedRows(o0, vs, dim, nh), ob.MixedRows(o1, vs, dim, nh)
    tok, off = walk_corpus(V, e, 300, seed=6)
    f.set_corpus(tok, off)
    st = f.train_round(0, alpha=0.025)
    assert st["pairs"] > 0
    c = ob.OracleCsr(e, V)
    vv, vcn, id2, _, tw = ob.vocab(c.deg, 0)
    thr, used = ob.subsample_thresholds(vcn, 1e-3, tw)
    table = ob.unigram_table(vcn)
    pl = ob.plan_batches(tok, off, id2, thr, used, table, vs, negative)
    bf = pl["batch_first"]
    for b in range(len(bf) - 1):
        ob.negreuse_tile_tc(m0, m1, ob.round_sr_seed(SEED, 0), ob.exp_table(), pl["sen"], pl["sent_start"],
                            int(bf[b]), int(bf[b + 1] - bf[b]), pl["negs"], 5, dim, negative, 0.025)
    g0, g1 = f.embeddings()
    r0, r1 = m0.full(), m1.full()
    for g, r in ((g0, r0), (g1, r1)):
        exact = np.mean(g == r)
        d = np.abs(g - r)
        print(f"tensor-core tile vs oracle: exact {exact:.5f}, max abs diff {d.max():.3e}")
        assert exact >= 0.99
        assert np.mean(d <= 2.0 ** -5 * np.abs(r) + 1e-6) >= 0.999
        assert np.all(d <= 2.0 ** -5 * np.abs(r) + 1e-3)


def link_auc(s0, id2, vs, dim, g):
    e0 = s0.reshape(vs, dim)[id2]
    n0 = e0 / np.maximum(np.linalg.norm(e0, axis=1, keepdims=True), 1e-30)
    cos = np.sum(n0[g["test_src"]] * n0[g["test_dst"]], axis=1)
    return fb.auc(cos, g["test_label"])


def run_form(g, precision, seed=17):
    """End-to-end: felog_run (walk, train, convergence check until the stop-all rule)."""
    V = g["v_num"]
    f = fb.Felog(v_num=V, size=128, window=10, negative=5, sample=1e-3, cbow=0, reuse_neg=0, min_count=0,
                 min_rounds=2, seed=seed, precision=precision)
    f.load_graph(g["edges"], V)
    f.init_model()
    st = f.run()
    s0, _ = f.embeddings()
    _, id2, vs, _ = f.vocab()
    f.close()
    return s0, id2, vs, st


def test_bf16_auc_within_0005_of_fp32():
    """End-to-end embeddings of the BF16 form against the FP32 form on the same
    graph and walk seed, run to completion.  The graph has ~100 k held-out
    pairs, so the AUC estimate itself has a standard error near 0.001; on a
    16 k-vertex graph it is ~0.002 and the forms can also stop after a
    different number of rounds, which makes a 0.005 bar a coin toss there."""
    g = fb.synth_graph(seed=3, v_target=65536, e_target=1048576, holdout=0.1)
    s32, id2, vs, st32 = run_form(g, 0)
    s16, id2b, vsb, st16 = run_form(g, 1)
    assert np.isfinite(s16).all()
    a32, a16 = link_auc(s32, id2, vs, 128, g), link_auc(s16, id2b, vsb, 128, g)
    print(f"AUC fp32 {a32:.4f} ({st32['rounds']} rounds) bf16 {a16:.4f} ({st16['rounds']} rounds) "
          f"delta {a16 - a32:+.4f}")
    assert abs(a16 - a32) < 0.005, (a32, a16)


def test_precision_study_1024_batches():
    """Dots and batch losses on 1,024 fixed seeded batches (64 contexts x
    (1 positive + 5 negatives)) from the stored tables, against FP64 from the
    FP32 tables.  FP32 storage: FP32 accumulation error only.  BF16 storage:
    every stored value carries a relative error <= 2^-9 (round to nearest), so
    |f - f64| <= 2^-8 (1 + 2^-9) sum |x_i y_i| plus the accumulation term."""
    g = fb.synth_graph(seed=0, v_target=16384, e_target=131072, holdout=0.1)
    V = g["v_num"]
    f = fb.Felog(v_num=V, size=128, window=10, negative=5, sample=1e-3, cbow=0, reuse_neg=0, min_count=0,
                 seed=11)
    f.load_graph(g["edges"], V)
    f.init_model()
    for r in range(2):
        f.walk_round(r)
        f.train_round(r)
    s0, s1 = f.embeddings()
    _, _, vs, _ = f.vocab()
    rng = np.random.default_rng(1024)
    nb, per = 1024, 64
    ctx = rng.integers(0, vs, nb * per).astype(np.int32)
    pos = rng.integers(0, vs, nb * per).astype(np.int32)
    neg = rng.integers(0, vs, (nb * per, 5)).astype(np.int32)
    c_all = np.repeat(ctx, 6)
    t_all = np.concatenate([pos[:, None], neg], axis=1).reshape(-1)
    lab = np.tile(np.array([1, 0, 0, 0, 0, 0], np.int8), nb * per)
    bof = np.repeat(np.arange(nb, dtype=np.uint64), per * 6)
    X = s0.reshape(vs, 128).astype(np.float64)
    Y = s1.reshape(vs, 128).astype(np.float64)
    d64 = np.einsum("ij,ij->i", X[c_all], Y[t_all])
    absd = np.einsum("ij,ij->i", np.abs(X[c_all]), np.abs(Y[t_all]))
    z = np.where(lab == 1, d64, -d64)
    l64 = np.bincount(bof.astype(np.int64), weights=np.logaddexp(0.0, -z), minlength=nb)

    d32, L32 = f.score_pairs(c_all, t_all, lab, bof, nb)
    f.close()
    f16 = fb.Felog(v_num=V, size=128, window=10, negative=5, sample=1e-3, cbow=0, reuse_neg=0, min_count=0,
                   seed=11, precision=1)
    f16.load_graph(g["edges"], V)
    f16.init_model()
    f16.set_embeddings(s0, s1)
    d16, L16 = f16.score_pairs(c_all, t_all, lab, bof, nb)
    f16.close()
    u32 = 2.0 ** -24
    e32 = np.abs(d32 - d64)
    e16 = np.abs(d16 - d64)
    assert np.all(e32 <= 130 * u32 * absd + 1e-30)
    assert np.all(e16 <= (2.0 ** -8) * (1 + 2.0 ** -9) * absd + 130 * u32 * absd + 1e-30)
    rl32 = np.abs(L32 - l64) / l64
    rl16 = np.abs(L16 - l64) / l64
    print(f"precision study ({nb} batches x {per * 6} dots): "
          f"FP32 dot abs err max {e32.max():.3e} mean {e32.mean():.3e}, loss rel err max {rl32.max():.3e}; "
          f"BF16 dot abs err max {e16.max():.3e} mean {e16.mean():.3e}, loss rel err max {rl16.max():.3e} "
          f"mean {rl16.mean():.3e}; |f64| mean {np.abs(d64).mean():.3e}")
    assert rl32.max() < 1e-5
    assert rl16.max() < 1e-2


def test_lost_update_count():
    """felog_count_lost_updates: one warp in sentence order never overwrites a
    concurrent update (0 lost, and the trained tables equal an uncounted run's);
    Hogwild over many warps does, the more the fewer rows there are (this
    8k-vertex graph is trained by thousands of warps at once), and the count is
    reported."""
    g = fb.synth_graph(seed=12, v_target=8192, e_target=65536, holdout=0.0)
    V = g["v_num"]
    res = {}
    for det in (1, 0):
        for count in (False, True):
            f = fb.Felog(v_num=V, size=128, window=10, negative=5, cbow=0, reuse_neg=0, min_count=0, seed=3,
                         precision=1, deterministic=det)
            f.load_graph(g["edges"], V)
            f.init_model()
            if count:
                f.count_lost_updates(True)
            f.walk_round(0)
            if det:
                tok, off = f.corpus()
                n = int(np.searchsorted(off, 20000))
                f.set_corpus(tok[: int(off[n])], off[: n + 1])
            f.train_round(0)
            res[(det, count)] = (f.embeddings(), f.lost_updates() if count else None)
            f.close()
    (d0, _), (d1, (nu, nl)) = res[(1, False)], res[(1, True)]
    assert nu > 0 and nl == 0
    for a, b in zip(d0, d1):
        np.testing.assert_array_equal(a, b)
    nu, nl = res[(0, True)][1]
    print(f"Hogwild: {nl} of {nu} BF16-row updates overwritten")
    assert nu > 0 and 0 < nl <= nu
