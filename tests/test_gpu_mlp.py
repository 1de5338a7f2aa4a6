"""Learned walk budget through the C ABI.

* Per-vertex features (degree, weighted degree, transition entropy, 2-hop
  degree sum, visits, first walk length) equal the oracle's FP64 features.
* The backward kernel's mean gradient and loss equal the oracle's FP64
  gradient (FP32 accumulation tolerance).
* Training on labels that the plain criterion produced lowers the loss and
  beats the trivial predictors; on an unseen graph the learned budget check
  decides most vertices without the convergence check, the plain criterion
  overrules few audited predictions, and the end-to-end link-prediction AUC
  stays within 0.005 of the plain run.
"""
import numpy as np
import pytest

import felog_b200 as fb
import oracle_binding as ob

pytestmark = pytest.mark.gpu

TRAIN = dict(size=128, window=10, negative=5, sample=1e-3, cbow=0, reuse_neg=0, min_count=0, min_rounds=2)


def test_features_match_oracle():
    g = fb.synth_graph(seed=0, v_target=4096, e_target=32768, holdout=0.1)
    V = g["v_num"]
    f = fb.Felog(v_num=V, seed=3, **TRAIN)
    f.load_graph(g["edges"], V)
    f.walk_round(0)
    feat = f.budget_features()
    tok, off = f.corpus()
    first_len = np.diff(off).astype(np.uint32)  # round 0: walker k starts at vertex k
    c = ob.OracleCsr(g["edges"], V)
    ref = ob.budget_features(c, f.visit_freq(), first_len)
    np.testing.assert_allclose(feat, ref, rtol=2e-6, atol=1e-6)


def test_mlp_gradient_matches_oracle():
    V = 1000
    f = fb.Felog(v_num=V, **TRAIN)
    rng = np.random.default_rng(5)
    n = 700  # three blocks, the last one partial
    params = (rng.standard_normal(fb.MLP_PARAMS) * 0.15).astype(np.float32)
    X = rng.standard_normal((n, 6)).astype(np.float32)
    count = rng.integers(2, 11, n).astype(np.uint8)
    length = rng.uniform(20, 80, n).astype(np.float32)
    g, loss = f.mlp_gradient(params, X, count, length)
    rg, rloss = ob.mlp_loss_grad(params, X, count, length)
    assert abs(loss - rloss) <= 1e-5 * abs(rloss)
    scale = np.abs(rg).max()
    err = np.abs(g - rg)
    print(f"gradient: max |err| {err.max():.3e} (max |g| {scale:.3e})")
    assert err.max() <= 1e-4 * scale  # FP32 sums over 256-sample blocks


def plain_label_run(g, seed, rounds=10):
    """Plain criterion for a fixed number of rounds (no stop-all), recording
    each vertex's budget labels."""
    V = g["v_num"]
    f = fb.Felog(v_num=V, seed=seed, **TRAIN)
    f.load_graph(g["edges"], V)
    f.init_model()
    for r in range(rounds):
        f.walk_round(r)
        f.train_round(r)
        if r + 1 >= TRAIN["min_rounds"]:
            f.budget_check(r)
    return f


def link_auc(f, g):
    s0, _ = f.embeddings()
    _, id2, vs, _ = f.vocab()
    e0 = s0.reshape(vs, 128)[id2]
    n0 = e0 / np.maximum(np.linalg.norm(e0, axis=1, keepdims=True), 1e-30)
    cos = np.sum(n0[g["test_src"]] * n0[g["test_dst"]], axis=1)
    return fb.auc(cos, g["test_label"])


def run_rounds(f, max_rounds=10):
    """felog_run's loop (stop-all rule included), collecting the budget stats."""
    tot = dict(evaluated=0, predicted=0, audited=0, overruled=0, rounds=0, tokens=0)
    for r in range(max_rounds):
        ws = f.walk_round(r)
        if f.opts.budget_mode == 1 and r == 0:
            f.mlp_predict()
        f.train_round(r)
        tot["tokens"] += ws["n_tokens"]
        tot["rounds"] = r + 1
        if r + 1 >= TRAIN["min_rounds"]:
            bs = f.budget_check(r)
            for k in ("evaluated", "predicted", "audited", "overruled"):
                tot[k] += bs[k]
            if bs["stop_all"]:
                break
    return tot


def test_mlp_trains_and_learned_budget_gains():
    gtrain = fb.synth_graph(seed=2, v_target=16384, e_target=131072, holdout=0.1, abcd=(0.6, 0.15, 0.15, 0.1))
    f = plain_label_run(gtrain, seed=21)
    cnt, ln = f.budget_labels()
    st = f.mlp_train(epochs=40, batch=1024, lr=3e-3, seed=1)
    majority = np.bincount(cnt, minlength=11).max() / len(cnt)
    mae_const = np.abs(ln - np.median(ln)).mean()
    print(f"labels: counts {np.bincount(cnt, minlength=11)[2:]}, length mean {ln.mean():.1f}; train {st}")
    print(f"majority-class accuracy {majority:.3f}, constant-length MAE {mae_const:.2f}")
    assert st["loss_last"] < st["loss_first"]
    assert st["count_accuracy"] >= majority
    # walk lengths are nearly constant on these graphs (the correlation stop
    # fires right after min_L); the length head must stay within a token
    assert st["length_mae"] < mae_const + 1.0
    state = f.mlp_state()
    f.close()

    gtest = fb.synth_graph(seed=3, v_target=16384, e_target=131072, holdout=0.1)
    V = gtest["v_num"]
    res = {}
    for mode in (0, 1):
        h = fb.Felog(v_num=V, seed=17, budget_mode=mode, **TRAIN)
        h.load_graph(gtest["edges"], V)
        h.init_model()
        if mode == 1:
            h.mlp_set_state(state)
        tot = run_rounds(h)
        tot["auc"] = link_auc(h, gtest)
        res[mode] = tot
        h.close()
    plain, learned = res[0], res[1]
    print(f"plain {plain}\nlearned {learned}")
    # most vertices skip the convergence check; few audited predictions are overruled
    assert learned["predicted"] > learned["evaluated"]
    assert learned["evaluated"] < 0.5 * plain["evaluated"]
    assert learned["audited"] > 0
    assert learned["overruled"] / learned["audited"] < 0.25
    assert abs(learned["auc"] - plain["auc"]) < 0.005
