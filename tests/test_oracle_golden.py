"""The CPU oracle against the reference's own outputs (golden fixtures).

Pins the oracle before it is trusted as the checker of the CUDA path:
walks (include/walk.hpp under injected draws), the trainer's vocabulary,
unigram table, subsampling thresholds, InitNet rows and batch plan
(src/word2vec.cu).
"""
import hashlib

import numpy as np
import pytest

import oracle_binding as ob
from conftest import walk_draws
from recipes import pack, synth_corpus

WALKS = ["walk_rmat512.npz", "walk_rmat512_stop_w2.npz", "walk_rmat512_minl5.npz", "walk_edgecases.npz",
         "walk_rmat4096.npz"]
PLANS = ["plan_multibatch.npz", "plan_subsample.npz", "plan_nosample_long.npz", "plan_tokens_sub.npz"]


@pytest.mark.parametrize("name", WALKS)
def test_oracle_walk_matches_reference(golden, name):
    fx = golden(name)
    V = int(fx["V"])
    csr = ob.OracleCsr(fx["edges"], V, undirected=True)
    stop = fx.get("stop")
    for r in range(int(fx["rounds"])):
        tok, off, walkers, st = ob.walk_round(csr, int(fx["walker_num"]), int(fx["min_L"]), stop_flags=stop,
                                              draws=walk_draws(fx, r))
        np.testing.assert_array_equal(off, fx[f"r{r}_off"])
        np.testing.assert_array_equal(tok, fx[f"r{r}_tokens"])
        # the start vertex of every walker the reference logged
        np.testing.assert_array_equal(walkers % V, fx[f"r{r}_start"])


def test_oracle_csr_order(golden):
    """Doubling (e, e^T) then bucketing by source in record order (graph.hpp:531-575, :741-772)."""
    fx = golden("walk_edgecases.npz")
    e = fx["edges"]
    V = int(fx["V"])
    csr = ob.OracleCsr(e, V, undirected=True)
    buckets = [[] for _ in range(V)]
    for rec in e:
        buckets[rec["src"]].append((rec["dst"], rec["data"]))
        buckets[rec["dst"]].append((rec["src"], rec["data"]))
    for v in range(V):
        got = list(zip(csr.nbr[csr.row_ptr[v]:csr.row_ptr[v + 1]], csr.data[csr.row_ptr[v]:csr.row_ptr[v + 1]]))
        assert got == buckets[v]


@pytest.mark.parametrize("name", PLANS)
def test_oracle_plan_matches_reference(golden, name):
    fx = golden(name)
    deg = fx["deg"]
    vv, vcn, id2, vs, tw = ob.vocab(deg, int(fx["min_count"]))
    assert vs == int(fx["vocab_size"]) and tw == int(fx["train_words"])
    np.testing.assert_array_equal(vv, fx["vocab_vertex"])
    thr, used = ob.subsample_thresholds(vcn, float(fx["sample"]), tw)
    assert used == (len(fx["thr"]) > 0)
    if used:
        np.testing.assert_array_equal(thr, fx["thr"])
    table = ob.unigram_table(vcn)
    np.testing.assert_array_equal(table[:4096], fx["table_head"])
    assert hashlib.sha256(table.tobytes()).hexdigest() == fx["table_sha256"].item().decode()
    dim = int(fx["dim"])
    syn0, _ = ob.init_net(vs, dim)
    np.testing.assert_array_equal(syn0[: min(vs, 64) * dim], fx["syn0_head"])
    rc = fx["recipe"]
    tok, off = pack(synth_corpus(int(rc[0]), int(rc[1]), int(rc[2]), int(rc[3]), int(rc[4]), int(rc[5])))
    K = int(fx["negative"])
    pl = ob.plan_batches(tok, off, id2, thr, used, table, vs, K)
    bf = pl["batch_first"]
    assert len(bf) - 1 == len(fx["batch_cnt"])
    np.testing.assert_array_equal(np.diff(bf), fx["batch_cnt"])
    # per-batch sentence_length arrays, relative to the batch start
    sl = []
    for b in range(len(bf) - 1):
        ss = pl["sent_start"][bf[b]:bf[b + 1] + 1]
        sl.append((ss - ss[0]).astype(np.int32))
    np.testing.assert_array_equal(np.concatenate(sl), fx["sentence_length"])
    assert hashlib.sha256(pl["sen"].tobytes()).hexdigest() == fx["sen_sha256"].item().decode()
    assert hashlib.sha256(pl["negs"].tobytes()).hexdigest() == fx["negs_sha256"].item().decode()
    np.testing.assert_array_equal(pl["sen"][:20000], fx["sen_head"])


def test_oracle_lr_schedule():
    """alpha_r = 0.025 exp(-0.1 r) in float (lr_scheduler.hpp:23-31)."""
    import ctypes
    libm = ctypes.CDLL("libm.so.6")
    libm.expf.argtypes = [ctypes.c_float]
    libm.expf.restype = ctypes.c_float
    for r in range(8):
        e = np.float32(libm.expf(float(np.float32(-0.1) * np.float32(r))))
        assert ob.lr(0.025, 0.1, r) == np.float32(np.float32(0.025) * e)


def test_oracle_exp_table_shape():
    t = ob.exp_table()
    assert t.shape == (1000,) and np.all(np.diff(t) > 0) and 0 < t[0] < 0.01 and 0.99 < t[-1] < 1


def test_oracle_kl_definition():
    deg = np.array([3, 1, 2, 2], np.uint32)
    freq = np.array([5, 2, 2, 1], np.uint64)
    p = deg / deg.sum()
    q = freq / freq.sum()
    assert abs(ob.round_kl(deg, freq) - float(np.sum(p * (np.log(p) - np.log(q))))) < 1e-15


def test_oracle_eval_choose_is_a_sample_without_replacement():
    for deg in (31, 40, 1000):
        ch = np.zeros(30, np.uint32)
        ob.lib().orc_eval_choose(7, 3, 11, deg, ob.ptr(ch, ob.u32p))
        assert len(set(ch.tolist())) == 30 and ch.max() < deg


def _philox_py(ctr, key):
    """Philox4x32-10 written from the published round function (Salmon et al., SC'11)."""
    c0, c1, c2, c3 = ctr
    k0, k1 = key
    M = 0xFFFFFFFF
    for _ in range(10):
        p0 = 0xD2511F53 * c0
        p1 = 0xCD9E8D57 * c2
        c0, c1, c2, c3 = ((p1 >> 32) ^ c1 ^ k0) & M, p1 & M, ((p0 >> 32) ^ c3 ^ k1) & M, p0 & M
        k0 = (k0 + 0x9E3779B9) & M
        k1 = (k1 + 0xBB67AE85) & M
    return c0, c1, c2, c3


def test_oracle_philox_matches_python_restatement():
    import ctypes
    rng = np.random.default_rng(5)
    out = (ctypes.c_uint32 * 4)()
    for _ in range(200):
        ctr = tuple(int(x) for x in rng.integers(0, 2**32, 4))
        key = tuple(int(x) for x in rng.integers(0, 2**32, 2))
        ob.lib().orc_philox4x32_10((ctypes.c_uint32 * 4)(*ctr), (ctypes.c_uint32 * 2)(*key), out)
        assert tuple(out) == _philox_py(ctr, key)


def test_oracle_walk_draw_uniformity():
    """Native draws: index in [0, deg) and p in [0, 1), roughly uniform."""
    import ctypes
    idx = ctypes.c_uint32()
    p = ctypes.c_double()
    deg = 7
    counts = np.zeros(deg, int)
    ps = []
    for it in range(7000):
        ob.lib().orc_walk_draw(3, 11, 2, it, 0, deg, ctypes.byref(idx), ctypes.byref(p))
        counts[idx.value] += 1
        ps.append(p.value)
    chi2 = float(((counts - 1000) ** 2 / 1000).sum())
    assert chi2 < 25.0  # 6 dof, p ~ 3e-4
    ps = np.array(ps)
    assert ps.min() >= 0 and ps.max() < 1 and abs(ps.mean() - 0.5) < 0.02
