"""ctypes binding of the CPU oracle (oracle/felog_oracle.c).

Test infrastructure: only the tests, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` leg of ``bench.py`` load the oracle, and only as the checker.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "liboracle.so")

u8p = ctypes.POINTER(ctypes.c_uint8)
u16p = ctypes.POINTER(ctypes.c_uint16)
u32p = ctypes.POINTER(ctypes.c_uint32)
u64p = ctypes.POINTER(ctypes.c_uint64)
i32p = ctypes.POINTER(ctypes.c_int32)
i64p = ctypes.POINTER(ctypes.c_longlong)
f32p = ctypes.POINTER(ctypes.c_float)
f64p = ctypes.POINTER(ctypes.c_double)


class Csr(ctypes.Structure):
    _fields_ = [("v_num", ctypes.c_uint32), ("e_num", ctypes.c_uint64), ("row_ptr", u64p),
                ("nbr", u32p), ("data", f32p)]


class Draws(ctypes.Structure):
    _fields_ = [("idx_off", u64p), ("idx", u32p), ("p_off", u64p), ("p", f64p)]


class WalkStats(ctypes.Structure):
    _fields_ = [("n_sentences", ctypes.c_uint64), ("n_tokens", ctypes.c_uint64),
                ("n_traces", ctypes.c_uint64), ("n_iterations", ctypes.c_uint64),
                ("n_long", ctypes.c_uint64)]


class PlanOut(ctypes.Structure):
    _fields_ = [("sen", i32p), ("sen_cap", ctypes.c_uint64), ("sent_start", u64p),
                ("batch_first", u64p), ("negs", i32p), ("n_sentences", ctypes.c_uint64),
                ("n_batches", ctypes.c_uint64), ("n_sen", ctypes.c_uint64),
                ("words_considered", ctypes.c_uint64)]


def ptr(a, t):
    return a.ctypes.data_as(t)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "port"])
        L = ctypes.CDLL(ORACLE_SO)
        L.orc_build_csr.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int,
                                    ctypes.POINTER(Csr)]
        L.orc_free_csr.argtypes = [ctypes.POINTER(Csr)]
        L.orc_walk_round.argtypes = [ctypes.POINTER(Csr), ctypes.c_uint32, u8p, ctypes.c_uint32,
                                     ctypes.c_uint64, ctypes.c_uint32, ctypes.POINTER(Draws), u32p,
                                     ctypes.c_uint64, u64p, u32p, ctypes.POINTER(WalkStats)]
        L.orc_round_kl.argtypes = [u32p, u64p, ctypes.c_uint32]
        L.orc_round_kl.restype = ctypes.c_double
        L.orc_lr.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_int]
        L.orc_lr.restype = ctypes.c_float
        L.orc_vocab.argtypes = [u32p, ctypes.c_uint32, ctypes.c_longlong, u32p, i64p, u32p, i64p, i64p]
        L.orc_unigram_table.argtypes = [i64p, ctypes.c_longlong, i32p, ctypes.c_int64]
        L.orc_subsample_thresholds.argtypes = [i64p, ctypes.c_longlong, ctypes.c_double,
                                               ctypes.c_longlong, u16p]
        L.orc_exp_table.argtypes = [f32p]
        L.orc_plan_batches.argtypes = [u32p, u64p, ctypes.c_uint64, u32p, u16p, ctypes.c_int, i32p,
                                       ctypes.c_int64, ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(PlanOut)]
        L.orc_skipgram_batch.argtypes = [f32p, f32p, f32p, i32p, ctypes.c_int64, ctypes.c_longlong, i32p,
                                         u64p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_float]
        L.orc_negreuse_batch.argtypes = [f32p, f32p, f32p, i32p, u64p, ctypes.c_uint64, ctypes.c_uint64,
                                         i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float]
        L.orc_cbow_batch.argtypes = L.orc_skipgram_batch.argtypes
        L.orc_init_net.argtypes = [f32p, f32p, ctypes.c_longlong, ctypes.c_int]
        L.orc_skipgram_bf16.argtypes = [f32p, u16p, f32p, u16p, ctypes.c_longlong, ctypes.c_uint32, f32p, i32p,
                                        ctypes.c_int64, ctypes.c_longlong, i32p, u64p, ctypes.c_uint64,
                                        ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float]
        L.orc_cbow_bf16.argtypes = L.orc_skipgram_bf16.argtypes
        L.orc_negreuse_tile.argtypes = [f32p, u16p, f32p, u16p, ctypes.c_longlong, ctypes.c_uint32, f32p, i32p, u64p,
                                        ctypes.c_uint64, ctypes.c_uint64, i32p, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_float]
        L.orc_negreuse_tile_tc.argtypes = L.orc_negreuse_tile.argtypes
        L.orc_window_tile.argtypes = L.orc_skipgram_bf16.argtypes
        L.orc_negreuse_bf16.argtypes = [f32p, u16p, f32p, u16p, ctypes.c_longlong, ctypes.c_uint32, f32p, i32p, u64p,
                                        ctypes.c_uint64, ctypes.c_uint64, i32p, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_float]
        L.orc_round_sr_seed.argtypes = [ctypes.c_uint64, ctypes.c_uint32]
        L.orc_budget_features.argtypes = [ctypes.POINTER(Csr), u64p, u32p, f64p]
        L.orc_mlp_loss_grad.argtypes = [f32p, f32p, ctypes.POINTER(ctypes.c_uint8), f32p, ctypes.c_uint64, f64p]
        L.orc_mlp_loss_grad.restype = ctypes.c_double
        L.orc_round_sr_seed.restype = ctypes.c_uint32
        L.orc_convergence.argtypes = [f32p, u32p, ctypes.c_int, ctypes.POINTER(Csr), u8p, ctypes.c_uint64,
                                      ctypes.c_uint32, f32p]
        L.orc_convergence.restype = ctypes.c_uint64
        L.orc_eval_choose.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, u32p]
        L.orc_walk_draw.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                    ctypes.c_uint32, ctypes.c_uint32, u32p, f64p]
        L.orc_common_neighbours.argtypes = [u32p, u32p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int, i32p]
        _lib = L
    return _lib


def common_neighbours(src, dst, v_num, undirected=True):
    """orc_common_neighbours: per input edge, gcn.cpp's common-neighbour count."""
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    cn = np.zeros(len(src), np.int32)
    rc = lib().orc_common_neighbours(ptr(src, u32p), ptr(dst, u32p), len(src), v_num, int(undirected), ptr(cn, i32p))
    assert rc == 0, rc
    return cn


EDGE12 = np.dtype([("src", "<u4"), ("dst", "<u4"), ("data", "<f4")])


class OracleCsr:
    """CSR built by the oracle in the reference's adjacency order."""

    def __init__(self, edges, v_num, undirected=True):
        edges = np.ascontiguousarray(edges, dtype=EDGE12)
        self._edges = edges
        self.c = Csr()
        rc = lib().orc_build_csr(edges.ctypes.data, len(edges), v_num, int(undirected), ctypes.byref(self.c))
        assert rc == 0, rc
        n = self.c.v_num
        self.row_ptr = np.ctypeslib.as_array(self.c.row_ptr, shape=(n + 1,)).copy()
        m = self.c.e_num
        self.nbr = np.ctypeslib.as_array(self.c.nbr, shape=(max(m, 1),))[:m].copy()
        self.data = np.ctypeslib.as_array(self.c.data, shape=(max(m, 1),))[:m].copy()
        self.deg = np.diff(self.row_ptr).astype(np.uint32)

    def __del__(self):
        try:
            lib().orc_free_csr(ctypes.byref(self.c))
        except Exception:
            pass


def walk_round(csr, walker_num, min_len, seed=0, round_=0, stop_flags=None, draws=None, tok_cap=None):
    """Returns (tokens, sent_off, sent_walker, stats)."""
    V = csr.c.v_num
    n_active = walker_num if stop_flags is None else int(sum(
        1 for w in range(walker_num) if not stop_flags[w % V]))
    if tok_cap is None:
        tok_cap = max(1, n_active) * 4096
    tokens = np.zeros(tok_cap, np.uint32)
    sent_off = np.zeros(n_active + 1, np.uint64)
    sent_walker = np.zeros(max(1, n_active), np.uint32)
    st = WalkStats()
    sf = None
    if stop_flags is not None:
        sf_arr = np.ascontiguousarray(stop_flags, dtype=np.uint8)
        sf = ptr(sf_arr, u8p)
    dr = None
    keep = None
    if draws is not None:
        idx_off, idx, p_off, p = draws
        keep = [np.ascontiguousarray(idx_off, np.uint64), np.ascontiguousarray(idx, np.uint32),
                np.ascontiguousarray(p_off, np.uint64), np.ascontiguousarray(p, np.float64)]
        dr = Draws(ptr(keep[0], u64p), ptr(keep[1], u32p), ptr(keep[2], u64p), ptr(keep[3], f64p))
    rc = lib().orc_walk_round(ctypes.byref(csr.c), walker_num, sf, min_len, seed, round_,
                              ctypes.byref(dr) if dr is not None else None, ptr(tokens, u32p), tok_cap,
                              ptr(sent_off, u64p), ptr(sent_walker, u32p), ctypes.byref(st))
    assert rc == 0, rc
    n = int(st.n_tokens)
    return tokens[:n].copy(), sent_off[: st.n_sentences + 1].copy(), sent_walker[: st.n_sentences].copy(), st


def vocab(deg, min_count=0):
    deg = np.ascontiguousarray(deg, np.uint32)
    V = len(deg)
    vv = np.zeros(V, np.uint32)
    vcn = np.zeros(V, np.int64)
    id2 = np.zeros(V, np.uint32)
    vs = ctypes.c_longlong()
    tw = ctypes.c_longlong()
    rc = lib().orc_vocab(ptr(deg, u32p), V, min_count, ptr(vv, u32p), ptr(vcn, i64p), ptr(id2, u32p),
                         ctypes.byref(vs), ctypes.byref(tw))
    assert rc == 0
    n = vs.value
    return vv[:n].copy(), vcn[:n].copy(), id2, n, tw.value


def unigram_table(vocab_cn, table_size=100_000_000):
    vocab_cn = np.ascontiguousarray(vocab_cn, np.int64)
    t = np.zeros(table_size, np.int32)
    lib().orc_unigram_table(ptr(vocab_cn, i64p), len(vocab_cn), ptr(t, i32p), table_size)
    return t


def subsample_thresholds(vocab_cn, sample, train_words):
    vocab_cn = np.ascontiguousarray(vocab_cn, np.int64)
    thr = np.zeros(len(vocab_cn), np.uint16)
    used = lib().orc_subsample_thresholds(ptr(vocab_cn, i64p), len(vocab_cn), sample, train_words,
                                          ptr(thr, u16p))
    return thr, bool(used)


def exp_table():
    t = np.zeros(1000, np.float32)
    lib().orc_exp_table(ptr(t, f32p))
    return t


def plan_batches(tokens, sent_off, id2offset, thr, use_thr, table, vocab_size, negative, rank=0):
    tokens = np.ascontiguousarray(tokens, np.uint32)
    sent_off = np.ascontiguousarray(sent_off, np.uint64)
    n_sent = len(sent_off) - 1
    cap = len(tokens) + 1
    sen = np.zeros(cap, np.int32)
    ss = np.zeros(n_sent + 1, np.uint64)
    bf = np.zeros(n_sent + 2, np.uint64)
    negs = np.zeros(max(1, n_sent * negative), np.int32)
    thr = np.ascontiguousarray(thr if thr is not None else np.zeros(1, np.uint16), np.uint16)
    out = PlanOut(ptr(sen, i32p), cap, ptr(ss, u64p), ptr(bf, u64p), ptr(negs, i32p), 0, 0, 0, 0)
    rc = lib().orc_plan_batches(ptr(tokens, u32p), ptr(sent_off, u64p), n_sent,
                                ptr(np.ascontiguousarray(id2offset, np.uint32), u32p), ptr(thr, u16p),
                                int(use_thr), ptr(table, i32p), len(table), vocab_size, negative, rank,
                                ctypes.byref(out))
    assert rc >= 0, rc
    ns = out.n_sentences
    return dict(sen=sen[: out.n_sen].copy(), sent_start=ss[: ns + 1].copy(),
                batch_first=bf[: out.n_batches + 1].copy(), negs=negs[: ns * negative].copy(),
                words=out.words_considered)


def init_net(vocab_size, dim, with_syn1=True):
    syn0 = np.zeros(vocab_size * dim, np.float32)
    syn1 = np.zeros(vocab_size * dim, np.float32)
    lib().orc_init_net(ptr(syn0, f32p), ptr(syn1, f32p), vocab_size, dim)
    return syn0, syn1


def skipgram_batch(syn0, syn1, exp_tab, table, vocab_size, sen, sent_start, first, n, window, dim,
                   negative, alpha, cbow=False):
    fn = lib().orc_cbow_batch if cbow else lib().orc_skipgram_batch
    fn(ptr(syn0, f32p), ptr(syn1, f32p), ptr(exp_tab, f32p), ptr(table, i32p), len(table), vocab_size,
       ptr(np.ascontiguousarray(sen, np.int32), i32p), ptr(np.ascontiguousarray(sent_start, np.uint64), u64p),
       first, n, window, dim, negative, alpha)


def bf16_rne(x):
    """FP32 -> BF16 bit patterns, round to nearest even (finite values)."""
    b = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    return ((b + 0x7FFF + ((b >> 16) & 1)) >> 16).astype(np.uint16)


def bf16_to_f32(h):
    return (np.asarray(h, np.uint16).astype(np.uint32) << 16).view(np.float32)


class MixedRows:
    """Tables in the BF16 storage form: FP32 rows 0..n_hot-1, BF16 bits after."""

    def __init__(self, full, vocab_size, dim, n_hot):
        full = np.ascontiguousarray(full, np.float32)
        self.dim, self.n_hot = dim, n_hot
        self.f32 = full[: n_hot * dim].copy()
        self.bf = bf16_rne(full[n_hot * dim:])

    def full(self):
        return np.concatenate([self.f32, bf16_to_f32(self.bf)])


def round_sr_seed(seed, round_):
    return lib().orc_round_sr_seed(seed, round_)


def skipgram_bf16(m0, m1, sr_seed, exp_tab, table, vocab_size, sen, sent_start, first, n, window, dim,
                  negative, alpha, cbow=False):
    fn = lib().orc_cbow_bf16 if cbow else lib().orc_skipgram_bf16
    fn(ptr(m0.f32, f32p), ptr(m0.bf, u16p), ptr(m1.f32, f32p), ptr(m1.bf, u16p), m0.n_hot, sr_seed,
       ptr(exp_tab, f32p), ptr(table, i32p), len(table), vocab_size,
       ptr(np.ascontiguousarray(sen, np.int32), i32p), ptr(np.ascontiguousarray(sent_start, np.uint64), u64p),
       first, n, window, dim, negative, alpha)


def budget_features(csr, visits, first_len):
    v = np.ascontiguousarray(visits, np.uint64)
    fl = np.ascontiguousarray(first_len, np.uint32)
    out = np.zeros(csr.c.v_num * 6, np.float64)
    lib().orc_budget_features(ctypes.byref(csr.c), ptr(v, u64p), ptr(fl, u32p), ptr(out, f64p))
    return out.reshape(-1, 6)


def mlp_loss_grad(params, X, count, length):
    p = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(X, np.float32)
    c = np.ascontiguousarray(count, np.uint8)
    l = np.ascontiguousarray(length, np.float32)
    g = np.zeros(5258, np.float64)
    loss = lib().orc_mlp_loss_grad(ptr(p, f32p), ptr(x, f32p), c.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                                   ptr(l, f32p), len(c), ptr(g, f64p))
    return g, loss


def negreuse_bf16(m0, m1, sr_seed, exp_tab, sen, sent_start, first, n, negs, window, dim, negative, alpha):
    lib().orc_negreuse_bf16(ptr(m0.f32, f32p), ptr(m0.bf, u16p), ptr(m1.f32, f32p), ptr(m1.bf, u16p), m0.n_hot,
                            sr_seed, ptr(exp_tab, f32p), ptr(np.ascontiguousarray(sen, np.int32), i32p),
                            ptr(np.ascontiguousarray(sent_start, np.uint64), u64p), first, n,
                            ptr(np.ascontiguousarray(negs, np.int32), i32p), window, dim, negative, alpha)


def negreuse_tile(m0, m1, sr_seed, exp_tab, sen, sent_start, first, n, negs, window, dim, negative, alpha):
    """-reuse-neg 2 center tiles on MixedRows (n_hot = vocab size for the FP32 form)."""
    lib().orc_negreuse_tile(ptr(m0.f32, f32p), ptr(m0.bf, u16p), ptr(m1.f32, f32p), ptr(m1.bf, u16p), m0.n_hot,
                            sr_seed, ptr(exp_tab, f32p), ptr(np.ascontiguousarray(sen, np.int32), i32p),
                            ptr(np.ascontiguousarray(sent_start, np.uint64), u64p), first, n,
                            ptr(np.ascontiguousarray(negs, np.int32), i32p), window, dim, negative, alpha)


def window_tile(m0, m1, sr_seed, exp_tab, table, vocab_size, sen, sent_start, first, n, window, dim, negative,
                alpha):
    """-reuse-neg 4 window tiles (skip-gram windows, the first context's draws as the
    center's shared negatives) on MixedRows."""
    lib().orc_window_tile(ptr(m0.f32, f32p), ptr(m0.bf, u16p), ptr(m1.f32, f32p), ptr(m1.bf, u16p), m0.n_hot,
                          sr_seed, ptr(exp_tab, f32p), ptr(table, i32p), len(table), vocab_size,
                          ptr(np.ascontiguousarray(sen, np.int32), i32p),
                          ptr(np.ascontiguousarray(sent_start, np.uint64), u64p), first, n, window, dim, negative,
                          alpha)


def negreuse_tile_tc(m0, m1, sr_seed, exp_tab, sen, sent_start, first, n, negs, window, dim, negative, alpha):
    """-reuse-neg 3 (tensor-core center tiles) on MixedRows."""
    lib().orc_negreuse_tile_tc(ptr(m0.f32, f32p), ptr(m0.bf, u16p), ptr(m1.f32, f32p), ptr(m1.bf, u16p), m0.n_hot,
                               sr_seed, ptr(exp_tab, f32p), ptr(np.ascontiguousarray(sen, np.int32), i32p),
                               ptr(np.ascontiguousarray(sent_start, np.uint64), u64p), first, n,
                               ptr(np.ascontiguousarray(negs, np.int32), i32p), window, dim, negative, alpha)


def negreuse_batch(syn0, syn1, exp_tab, sen, sent_start, first, n, negs, window, dim, negative, alpha):
    lib().orc_negreuse_batch(ptr(syn0, f32p), ptr(syn1, f32p), ptr(exp_tab, f32p),
                             ptr(np.ascontiguousarray(sen, np.int32), i32p),
                             ptr(np.ascontiguousarray(sent_start, np.uint64), u64p), first, n,
                             ptr(np.ascontiguousarray(negs, np.int32), i32p), window, dim, negative, alpha)


def convergence(syn0, id2offset, dim, csr, stop_flags, seed, round_):
    sf = np.ascontiguousarray(stop_flags, np.uint8).copy()
    sim = np.zeros(csr.c.v_num, np.float32)
    eva = lib().orc_convergence(ptr(syn0, f32p), ptr(np.ascontiguousarray(id2offset, np.uint32), u32p), dim,
                                ctypes.byref(csr.c), ptr(sf, u8p), seed, round_, ptr(sim, f32p))
    return int(eva), sf, sim


def eval_choose(seed, round_, v, deg):
    """The convergence check's neighbour positions of vertex v (degree deg): all of
    them in CSR order when deg <= 30, else the first 30 of the Philox shuffle."""
    if deg <= 30:
        return np.arange(deg, dtype=np.uint32)
    out = np.zeros(30, np.uint32)
    lib().orc_eval_choose(seed, round_, v, deg, ptr(out, u32p))
    return out


def round_kl(deg, freq):
    deg = np.ascontiguousarray(deg, np.uint32)
    freq = np.ascontiguousarray(freq, np.uint64)
    return lib().orc_round_kl(ptr(deg, u32p), ptr(freq, u64p), len(deg))


def lr(initial, decay, r):
    return lib().orc_lr(initial, decay, r)
