"""Walk-budget (per-vertex convergence) parity and the whole round loop."""
import numpy as np
import pytest

import felog_b200 as fb
import oracle_binding as ob
from conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dim", [64, 128])
def test_convergence_check_matches_oracle(dim):
    fx = load_golden("walk_rmat4096.npz")
    e, V = fx["edges"], int(fx["V"])
    f = fb.Felog(v_num=V, size=dim, window=10, negative=5, cbow=0, reuse_neg=0, min_count=0, seed=99)
    f.load_graph(e, V)
    f.init_model()
    for r in range(3):
        f.walk_round(r)
        f.train_round(r)
    s0, _ = f.embeddings()
    vv, id2, vs, _ = f.vocab()
    flags0 = np.zeros(V, np.uint8)
    flags0[::17] = 1  # already converged vertices are not re-evaluated
    f.set_stop_flags(flags0)
    st = f.budget_check(5)
    c = ob.OracleCsr(e, V)
    eva, oflags, osim = ob.convergence(s0, id2, dim, c, flags0, f.opts.seed, 5)
    np.testing.assert_array_equal(f.stop_flags(), oflags)
    sim = f.similarity()
    ev = flags0 == 0
    np.testing.assert_array_equal(sim[ev], osim[ev])
    assert st["unconverged"] == eva and st["evaluated"] == int(ev.sum())
    assert st["stopped_total"] == int(oflags.sum())


def test_run_loop_terminates_and_writes_reference_format(tmp_path):
    g = fb.synth_graph(seed=3, v_target=4096, e_target=32768, holdout=0.1)
    V = g["v_num"]
    f = fb.Felog(v_num=V, size=128, window=10, negative=5, cbow=0, reuse_neg=0, min_count=0, min_rounds=2,
                 max_rounds=12, seed=3)
    f.load_graph(g["edges"], V)
    rs = f.run()
    assert 2 <= rs["rounds"] <= 12 and rs["walk_tokens"] > 0 and rs["train_words"] > 0
    p = str(tmp_path / "emb.txt")
    f.write_embeddings(p)
    lines = open(p).read().splitlines()
    assert lines[0] == f"{V} 128"  # "%lld %lld\n" (word2vec.cu:2121)
    vv, id2, vs, _ = f.vocab()
    s0, _ = f.embeddings()
    first = lines[1].split(" ")
    assert first[0] == str(vv[0]) and first[-1] == "" and len(first) == 130  # "%s " + 128 x "%lf " (:2123-2125)
    assert first[1] == "%lf" % s0[0]
    assert len(lines) == V + 1
    # the whole file equals a serial printf rendering of every row
    rows = s0.reshape(vs, 128)
    want = f"{V} 128\n" + "".join(f"{vv[a]} " + "".join("%f " % float(x) for x in rows[a]) + "\n" for a in range(vs))
    assert open(p).read() == want


def test_stopped_vertices_spawn_no_walkers():
    fx = load_golden("walk_rmat512.npz")
    V = int(fx["V"])
    f = fb.Felog(v_num=V, seed=1)
    f.load_graph(fx["edges"], V)
    flags = np.zeros(V, np.uint8)
    flags[: V // 2] = 1
    f.set_stop_flags(flags)
    st = f.walk_round(0)
    tok, off = f.corpus()
    assert st["n_sentences"] == V - V // 2
    assert (tok[off[:-1].astype(np.int64)] >= V // 2).all()


def test_async_embedding_copy_equals_sync_copy():
    """felog_copy_embeddings_async snapshots syn0 at the call: after another
    round has run, the host buffer holds the rows of the earlier round, equal
    to a synchronous felog_get_embeddings taken at the same point."""
    import ctypes

    import torch

    g = fb.synth_graph(seed=4, v_target=4096, e_target=32768, holdout=0.0)
    V = g["v_num"]
    f = fb.Felog(v_num=V, size=128, window=5, negative=5, sample=1e-3, cbow=0, reuse_neg=0, min_count=0, seed=3)
    f.load_graph(g["edges"], V)
    f.init_model()
    f.walk_round(0)
    f.train_round(0)
    sync0, _ = f.embeddings()
    vs = f.vocab()[2]
    buf = torch.zeros(vs * 128, dtype=torch.float32).pin_memory()
    f.embeddings_into_async(ctypes.c_void_p(buf.data_ptr()), vs * 128)
    f.walk_round(1)
    f.train_round(1)  # runs while (or after) the copy of round 0's rows
    f.wait_embeddings()
    np.testing.assert_array_equal(buf.numpy(), sync0)
    sync1, _ = f.embeddings()
    assert not np.array_equal(sync1, sync0)
    f.embeddings_into_async(ctypes.c_void_p(buf.data_ptr()), vs * 128)
    f.wait_embeddings()
    np.testing.assert_array_equal(buf.numpy(), sync1)


def test_streamed_rounds_walk_the_same_corpus():
    """felog_run with stream_walkers walks and trains each round in pieces: the
    walks are the same as in whole rounds (they depend on the graph and the
    stop flags only), each piece is planned and trained on its own, and the
    embedding reaches the same fit quality."""
    import ref_tables as rt

    g = fb.synth_graph(seed=0, v_target=16384, e_target=131072, holdout=0.10)
    V = g["v_num"]
    pairs = rt.fit_pairs(g)
    res = {}
    for piece in (0, 3000):
        f = fb.Felog(v_num=V, size=128, window=10, negative=5, cbow=0, reuse_neg=0, min_count=0, min_rounds=2,
                     max_rounds=2, seed=11, stream_walkers=piece)
        f.load_graph(g["edges"], V)
        rs = f.run()
        res[piece] = (rs, rt.fit_aucs(*rt.tables_by_vertex(f), pairs)["cosine_centered"])
        f.close()
    (a, qa), (b, qb) = res[0], res[3000]
    assert a["rounds"] == b["rounds"] == 2
    assert a["walk_tokens"] == b["walk_tokens"] and a["train_words"] == b["train_words"]
    assert qa > 0.7 and abs(qa - qb) < 0.02, (qa, qb)


def test_convergence_cosines_match_the_reference_kernel():
    """k_converge's per-vertex mean cosine against the reference's own kernel:
    batch_similarity_direct_index_optimized_kernel (word2vec.cu:1448-1506),
    compiled from its source (oracle/_ref/libref_sgns_gpu.so) and launched as
    batch_node_neighbor_direct_index launches it, on the same neighbour choices
    (all neighbours up to 30, else the first 30 of the Philox shuffle), then
    averaged per vertex as its host code does (FP32 sum in neighbour order,
    divided by the count; word2vec.cu:1860-1876).  Bit for bit."""
    import ctypes
    import os

    from conftest import ROOT

    so = os.path.join(ROOT, "oracle", "_ref", "libref_sgns_gpu.so")
    if not os.path.exists(so):
        pytest.skip("reference harness not built (make -C oracle ref)")
    L = ctypes.CDLL(so)
    L.ref_pair_similarity.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong,
                                      ctypes.c_void_p]
    fx = load_golden("walk_rmat4096.npz")
    e, V = fx["edges"], int(fx["V"])
    f = fb.Felog(v_num=V, size=128, window=10, negative=5, cbow=0, reuse_neg=0, min_count=0, seed=31)
    f.load_graph(e, V)
    f.init_model()
    for r in range(2):
        f.walk_round(r)
        f.train_round(r)
    s0, _ = f.embeddings()
    _, id2, vs, _ = f.vocab()
    f.set_stop_flags(np.zeros(V, np.uint8))
    f.budget_check(1)
    sim = f.similarity()
    c = ob.OracleCsr(e, V)
    node, nbr, cnt = [], [], np.zeros(V, np.int64)
    for v in range(V):
        b, d = int(c.row_ptr[v]), int(c.row_ptr[v + 1] - c.row_ptr[v])
        ch = ob.eval_choose(f.opts.seed, 1, v, d)
        node.extend([v] * len(ch))
        nbr.extend(c.nbr[b + ch.astype(np.int64)].tolist())
        cnt[v] = len(ch)
    node = np.array(node, np.uint32)
    nbr = np.array(nbr, np.uint32)
    cos = np.zeros(len(node), np.float32)
    s0c = np.ascontiguousarray(s0, np.float32)
    id2c = np.ascontiguousarray(id2, np.uint32)
    assert L.ref_pair_similarity(s0c.ctypes.data, vs, 128, node.ctypes.data, nbr.ctypes.data, len(node),
                                 id2c.ctypes.data, V, cos.ctypes.data) == 0
    ref = np.zeros(V, np.float32)
    o = 0
    for v in range(V):
        acc = np.float32(0.0)
        for j in range(cnt[v]):
            acc = np.float32(acc + cos[o + j])
        o += cnt[v]
        ref[v] = acc / np.float32(cnt[v]) if cnt[v] else np.float32(0.0)
    np.testing.assert_array_equal(sim, ref)
    np.testing.assert_array_equal(f.stop_flags(), (ref > 0.65).astype(np.uint8))
    f.close()
