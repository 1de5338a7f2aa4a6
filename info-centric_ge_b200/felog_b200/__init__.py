"""Python binding of the B200 FeLoG graph-embedding hot path.

A thin ctypes layer over ``libfelog_gpu.so`` (the C ABI of
``include/felog_gpu.h``) and ``libfelog_tools.so`` (``include/felog_tools.h``).
The binding mirrors the reference's in-process seams: ``Felog.load_graph``
(GraphEngine::load_graph, include/graph.hpp:712-919), ``Felog.walk_round`` (one
round of WalkEngine::random_walk, include/walk.hpp:629-752), ``Felog.train_round``
(TrainModelThreadMemory, src/word2vec.cu:1133-1273), ``Felog.budget_check`` (the
evaluation step of TrainModel, src/word2vec.cu:2016-2080) and ``Felog.run`` (the
whole walk/train loop).  There is no CPU fallback: every call raises
``FelogError`` when the CUDA library or a device is missing.
"""
import ctypes
import os

import numpy as np

__all__ = ["Felog", "FelogError", "FelogOpts", "EDGE12", "synth_graph", "auc", "gpu_lib_path",
           "tools_lib_path", "default_opts"]

_HERE = os.path.dirname(os.path.abspath(__file__))
EDGE12 = np.dtype([("src", "<u4"), ("dst", "<u4"), ("data", "<f4")])

STATUS = {0: "OK", 1: "INVALID_ARG", 2: "OOM", 3: "CUDA_ERROR", 4: "DEVICE_TIMEOUT", 5: "INTERNAL",
          6: "IO_ERROR", 7: "NOT_READY"}


class FelogError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class FelogOpts(ctypes.Structure):
    _fields_ = [
        ("v_num", ctypes.c_uint32), ("walker_num", ctypes.c_uint32), ("min_length", ctypes.c_uint32),
        ("min_rounds", ctypes.c_uint32), ("eval_batch_size", ctypes.c_uint32), ("make_undirected", ctypes.c_int32),
        ("size", ctypes.c_int32), ("window", ctypes.c_int32), ("negative", ctypes.c_int32), ("hs", ctypes.c_int32),
        ("cbow", ctypes.c_int32), ("reuse_neg", ctypes.c_int32), ("iter", ctypes.c_int32),
        ("min_count", ctypes.c_int32), ("classes", ctypes.c_int32), ("binary", ctypes.c_int32),
        ("debug", ctypes.c_int32), ("sample", ctypes.c_float), ("alpha", ctypes.c_float),
        ("use_cli_alpha", ctypes.c_int32), ("precision", ctypes.c_int32), ("deterministic", ctypes.c_int32),
        ("weighted", ctypes.c_int32), ("budget_mode", ctypes.c_int32), ("max_rounds", ctypes.c_int32),
        ("device", ctypes.c_int32), ("slot_len", ctypes.c_int32), ("seed", ctypes.c_uint64),
        ("long_arena_tokens", ctypes.c_uint64), ("wait_limit", ctypes.c_uint64),
        ("hot_rows", ctypes.c_int64), ("budget_confidence", ctypes.c_float), ("budget_audit", ctypes.c_float),
        ("autotune", ctypes.c_int32), ("stream_walkers", ctypes.c_uint32),
        ("bf16_reread", ctypes.c_int32),
    ]


class Draws(ctypes.Structure):
    _fields_ = [("idx_off", ctypes.c_void_p), ("idx", ctypes.c_void_p), ("n_idx", ctypes.c_uint64),
                ("p_off", ctypes.c_void_p), ("p", ctypes.c_void_p), ("n_p", ctypes.c_uint64),
                ("n_walkers", ctypes.c_uint64)]


class WalkStats(ctypes.Structure):
    _fields_ = [("n_sentences", ctypes.c_uint64), ("n_tokens", ctypes.c_uint64), ("n_traces", ctypes.c_uint64),
                ("n_iterations", ctypes.c_uint64), ("n_long", ctypes.c_uint64), ("kl", ctypes.c_double),
                ("ms", ctypes.c_float)]


class TrainStats(ctypes.Structure):
    _fields_ = [("words", ctypes.c_uint64), ("kept_words", ctypes.c_uint64), ("pairs", ctypes.c_uint64),
                ("sentences", ctypes.c_uint64),
                ("batches", ctypes.c_uint64), ("alpha", ctypes.c_float), ("ms_plan", ctypes.c_float),
                ("ms_train", ctypes.c_float)]


class BudgetStats(ctypes.Structure):
    _fields_ = [("evaluated", ctypes.c_uint64), ("unconverged", ctypes.c_uint64),
                ("stopped_total", ctypes.c_uint64), ("predicted", ctypes.c_uint64), ("audited", ctypes.c_uint64),
                ("overruled", ctypes.c_uint64), ("stop_all", ctypes.c_int32), ("ms", ctypes.c_float)]


class MlpOpts(ctypes.Structure):
    _fields_ = [("epochs", ctypes.c_int32), ("batch", ctypes.c_int32), ("lr", ctypes.c_float),
                ("seed", ctypes.c_uint64)]


class MlpStats(ctypes.Structure):
    _fields_ = [("samples", ctypes.c_uint64), ("steps", ctypes.c_uint64), ("loss_first", ctypes.c_double),
                ("loss_last", ctypes.c_double), ("count_accuracy", ctypes.c_double), ("length_mae", ctypes.c_double),
                ("ms", ctypes.c_float)]


MLP_PARAMS = 5258
MLP_STATE = MLP_PARAMS + 12


class RunStats(ctypes.Structure):
    _fields_ = [("rounds", ctypes.c_uint32), ("walk_tokens", ctypes.c_uint64), ("train_words", ctypes.c_uint64),
                ("walk_ms", ctypes.c_double), ("train_ms", ctypes.c_double), ("budget_ms", ctypes.c_double),
                ("total_ms", ctypes.c_double), ("final_unconverged", ctypes.c_uint64),
                ("evaluated", ctypes.c_uint64), ("predicted", ctypes.c_uint64), ("audited", ctypes.c_uint64),
                ("overruled", ctypes.c_uint64), ("pairs", ctypes.c_uint64), ("plan_ms", ctypes.c_double)]


class RmatParams(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint64), ("v_target", ctypes.c_uint64), ("e_target", ctypes.c_uint64),
                ("a", ctypes.c_double), ("b", ctypes.c_double), ("c", ctypes.c_double), ("d", ctypes.c_double),
                ("lognormal", ctypes.c_int32), ("lognormal_mu", ctypes.c_double),
                ("lognormal_sigma", ctypes.c_double), ("permute_ids", ctypes.c_int32)]


class RmatInfo(ctypes.Structure):
    _fields_ = [("v_num", ctypes.c_uint32), ("n_edges", ctypes.c_uint64), ("max_degree", ctypes.c_uint32)]


def _struct_dict(s):
    return {k: getattr(s, k) for k, _ in s._fields_}


def gpu_lib_path():
    return os.path.join(_HERE, "libfelog_gpu.so")


def tools_lib_path():
    return os.path.join(_HERE, "libfelog_tools.so")


_gpu = None
_tools = None

_P = ctypes.c_void_p


def gpu_lib():
    """Loads libfelog_gpu.so; raises if it has not been built."""
    global _gpu
    if _gpu is None:
        path = gpu_lib_path()
        if not os.path.exists(path):
            raise FelogError(3, f"{path} is missing: build it with `make -C info-centric_ge_b200`")
        L = ctypes.CDLL(path)
        L.felog_default_opts.argtypes = [ctypes.POINTER(FelogOpts)]
        L.felog_create.argtypes = [ctypes.POINTER(FelogOpts), ctypes.POINTER(_P)]
        L.felog_destroy.argtypes = [_P]
        L.felog_destroy.restype = None
        L.felog_last_error.argtypes = [_P]
        L.felog_last_error.restype = ctypes.c_char_p
        L.felog_load_graph.argtypes = [_P, _P, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int]
        L.felog_load_graph_file.argtypes = [_P, ctypes.c_char_p, ctypes.c_uint32, ctypes.c_int]
        L.felog_load_rmat.argtypes = [_P, ctypes.POINTER(RmatParams), ctypes.c_int, ctypes.POINTER(RmatInfo)]
        L.felog_graph_info.argtypes = [_P, _P, _P]
        L.felog_get_csr.argtypes = [_P, _P, _P, _P]
        L.felog_get_degrees.argtypes = [_P, _P]
        L.felog_build_alias.argtypes = [_P]
        L.felog_get_alias.argtypes = [_P, _P, _P]
        L.felog_set_stop_flags.argtypes = [_P, _P]
        L.felog_get_stop_flags.argtypes = [_P, _P]
        L.felog_walk_round.argtypes = [_P, ctypes.c_uint32, ctypes.POINTER(Draws), ctypes.POINTER(WalkStats)]
        L.felog_corpus_size.argtypes = [_P, _P, _P]
        L.felog_walk_piece.argtypes = [_P, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, _P,
                                       ctypes.POINTER(WalkStats)]
        L.felog_get_corpus.argtypes = [_P, _P, ctypes.c_uint64, _P, ctypes.c_uint64]
        L.felog_set_corpus.argtypes = [_P, _P, _P, ctypes.c_uint64]
        L.felog_get_visit_freq.argtypes = [_P, _P]
        L.felog_walk_ceiling.argtypes = [_P, _P, _P]
        L.felog_walk_entries.argtypes = [_P, ctypes.c_int, _P]
        L.felog_unigram_starts.argtypes = [_P, ctypes.c_uint64, _P]
        L.felog_pair_row_mix.argtypes = [_P, _P, _P, _P]
        L.felog_format_lf.argtypes = [_P, ctypes.c_uint64, _P, ctypes.c_uint64, _P]
        L.felog_common_neighbours.argtypes = [_P, _P, _P, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int, _P, _P]
        L.felog_init_model.argtypes = [_P]
        L.felog_vocab_info.argtypes = [_P, _P, _P]
        L.felog_get_vocab.argtypes = [_P, _P, _P]
        L.felog_train_round.argtypes = [_P, ctypes.c_uint32, ctypes.c_float, ctypes.POINTER(TrainStats)]
        L.felog_get_embeddings.argtypes = [_P, _P, _P, ctypes.c_uint64]
        L.felog_set_embeddings.argtypes = [_P, _P, _P]
        L.felog_plan_size.argtypes = [_P, _P, _P, _P]
        L.felog_count_lost_updates.argtypes = [_P, ctypes.c_int]
        L.felog_lost_updates.argtypes = [_P, _P, _P]
        L.felog_score_pairs.argtypes = [_P, _P, _P, _P, _P, ctypes.c_uint64, ctypes.c_uint64, _P, _P]
        L.felog_budget_features.argtypes = [_P, _P]
        L.felog_budget_labels.argtypes = [_P, _P, _P]
        L.felog_mlp_train.argtypes = [_P, ctypes.POINTER(MlpOpts), ctypes.POINTER(MlpStats)]
        L.felog_mlp_get_params.argtypes = [_P, _P]
        L.felog_mlp_set_params.argtypes = [_P, _P]
        L.felog_mlp_gradient.argtypes = [_P, _P, _P, _P, _P, ctypes.c_uint64, _P, ctypes.POINTER(ctypes.c_double)]
        L.felog_mlp_predict.argtypes = [_P, _P, _P, _P]
        L.felog_get_plan.argtypes = [_P, _P, _P, _P, _P]
        L.felog_budget_check.argtypes = [_P, ctypes.c_uint32, ctypes.POINTER(BudgetStats)]
        L.felog_get_similarity.argtypes = [_P, _P]
        L.felog_cluster_embeddings.argtypes = [_P, ctypes.c_int32, ctypes.c_int32, _P, _P, _P]
        L.felog_run.argtypes = [_P, ctypes.POINTER(RunStats)]
        L.felog_write_embeddings.argtypes = [_P, ctypes.c_char_p]
        L.felog_kernel_launches.argtypes = [_P]
        L.felog_copy_embeddings_async.argtypes = [_P, _P, ctypes.c_uint64]
        L.felog_wait_embeddings.argtypes = [_P]
        L.felog_tuning_report.argtypes = [_P]
        L.felog_tuning_report.restype = ctypes.c_char_p
        L.felog_kernel_launches.restype = ctypes.c_uint64
        L.felog_timer_mark.argtypes = [_P, ctypes.c_int]
        L.felog_timer_elapsed.argtypes = [_P, ctypes.POINTER(ctypes.c_float)]
        L.felog_build_alias_noalloc.argtypes = [_P, _P, ctypes.c_uint32, ctypes.c_uint64, _P, _P, _P]
        _gpu = L
    return _gpu


def tools_lib():
    global _tools
    if _tools is None:
        path = tools_lib_path()
        if not os.path.exists(path):
            raise FelogError(3, f"{path} is missing: build it with `make -C info-centric_ge_b200`")
        L = ctypes.CDLL(path)
        L.felog_synth_generate.argtypes = [_P, ctypes.POINTER(_P)]
        L.felog_synth_get_info.argtypes = [_P, _P]
        L.felog_synth_copy.argtypes = [_P, _P, _P, _P, _P]
        L.felog_synth_write_graph.argtypes = [_P, ctypes.c_char_p]
        L.felog_synth_free.argtypes = [_P]
        L.felog_synth_free.restype = None
        L.felog_auc.argtypes = [_P, _P, ctypes.c_size_t]
        L.felog_heldout_split.argtypes = [_P, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_double, ctypes.c_uint64, _P,
                                          _P, _P, _P, _P, _P]
        L.felog_auc.restype = ctypes.c_double
        L.felog_read_edge_file.argtypes = [ctypes.c_char_p, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
        L.felog_write_edge_file.argtypes = [ctypes.c_char_p, _P, ctypes.c_size_t]
        _tools = L
    return _tools


def default_opts(**kw):
    o = FelogOpts()
    gpu_lib().felog_default_opts(ctypes.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise AttributeError(k)
        setattr(o, k, v)
    return o


def _addr(a):
    return a.ctypes.data if a is not None and a.size else None


class Felog:
    """One device context (felog_ctx)."""

    def __init__(self, opts=None, **kw):
        L = gpu_lib()
        self.opts = opts if opts is not None else default_opts(**kw)
        h = _P()
        st = L.felog_create(ctypes.byref(self.opts), ctypes.byref(h))
        if st != 0:
            raise FelogError(st, "felog_create failed")
        self.h = h
        self._L = L

    def close(self):
        if getattr(self, "h", None):
            self._L.felog_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _ck(self, st):
        if st != 0:
            raise FelogError(st, self._L.felog_last_error(self.h).decode())

    # ---- graph
    def load_graph(self, edges, v_num, undirected=True):
        e = np.ascontiguousarray(edges, dtype=EDGE12)
        self._ck(self._L.felog_load_graph(self.h, _addr(e), len(e), v_num, int(undirected)))

    def load_rmat(self, seed, v_target, e_target, abcd=(0.57, 0.19, 0.19, 0.05), lognormal=False, permute=True,
                  mu=0.0, sigma=1.0, undirected=True):
        """felog_load_rmat: the seeded R-MAT graph generated and loaded on the device
        (the edges of synth_graph(..., holdout=0)); returns its info."""
        p = RmatParams(seed, v_target, e_target, *abcd, 1 if lognormal else 0, mu, sigma, int(permute))
        info = RmatInfo()
        self._ck(self._L.felog_load_rmat(self.h, ctypes.byref(p), int(undirected), ctypes.byref(info)))
        return _struct_dict(info)

    def load_graph_file(self, path, v_num, undirected=True):
        self._ck(self._L.felog_load_graph_file(self.h, path.encode(), v_num, int(undirected)))

    def graph_info(self):
        v = ctypes.c_uint32()
        m = ctypes.c_uint64()
        self._ck(self._L.felog_graph_info(self.h, ctypes.byref(v), ctypes.byref(m)))
        return v.value, m.value

    def csr(self):
        V, M = self.graph_info()
        rp = np.zeros(V + 1, np.uint64)
        nb = np.zeros(max(M, 1), np.uint32)
        dt = np.zeros(max(M, 1), np.float32)
        self._ck(self._L.felog_get_csr(self.h, _addr(rp), _addr(nb), _addr(dt)))
        return rp, nb[:M], dt[:M]

    def degrees(self):
        V, _ = self.graph_info()
        d = np.zeros(V, np.uint32)
        self._ck(self._L.felog_get_degrees(self.h, _addr(d)))
        return d

    def build_alias(self):
        self._ck(self._L.felog_build_alias(self.h))

    def alias(self):
        _, M = self.graph_info()
        p = np.zeros(max(M, 1), np.float32)
        a = np.zeros(max(M, 1), np.uint32)
        self._ck(self._L.felog_get_alias(self.h, _addr(p), _addr(a)))
        return p[:M], a[:M]

    # ---- walk
    def set_stop_flags(self, flags):
        f = np.ascontiguousarray(flags, np.uint8)
        self._ck(self._L.felog_set_stop_flags(self.h, _addr(f)))

    def stop_flags(self):
        V, _ = self.graph_info()
        f = np.zeros(V, np.uint8)
        self._ck(self._L.felog_get_stop_flags(self.h, _addr(f)))
        return f

    def walk_round(self, round_=0, draws=None):
        st = WalkStats()
        dr = None
        if draws is not None:
            idx_off, idx, p_off, p = draws
            keep = (np.ascontiguousarray(idx_off, np.uint64), np.ascontiguousarray(idx, np.uint32),
                    np.ascontiguousarray(p_off, np.uint64), np.ascontiguousarray(p, np.float64))
            self._keep = keep
            dr = Draws(_addr(keep[0]), _addr(keep[1]), len(keep[1]), _addr(keep[2]), _addr(keep[3]), len(keep[3]),
                       len(keep[0]) - 1)
        self._ck(self._L.felog_walk_round(self.h, round_, ctypes.byref(dr) if dr is not None else None,
                                          ctypes.byref(st)))
        return _struct_dict(st)

    def walk_piece(self, round_, first, count):
        """felog_walk_piece: active walkers first .. first + count - 1 of the round walk; returns
        (stats, number of active walkers of the round)."""
        st = WalkStats()
        na = ctypes.c_uint64()
        self._ck(self._L.felog_walk_piece(self.h, round_, first, count, ctypes.byref(na), ctypes.byref(st)))
        return _struct_dict(st), na.value

    def common_neighbours(self, src, dst, v_num, undirected=True):
        """felog_common_neighbours: per input edge, the common-neighbour count
        of the reference's gcn tool.  Returns (cn int32 array, device ms)."""
        src = np.ascontiguousarray(src, np.uint32)
        dst = np.ascontiguousarray(dst, np.uint32)
        cn = np.zeros(len(src), np.int32)
        ms = ctypes.c_float()
        self._ck(self._L.felog_common_neighbours(self.h, _addr(src), _addr(dst), len(src), v_num, int(undirected),
                                                 _addr(cn), ctypes.byref(ms)))
        return cn, ms.value

    def pair_row_mix(self):
        """felog_pair_row_mix: (pairs, row references, master-row references)
        of the last trained pair-stream chunk."""
        v = [ctypes.c_uint64() for _ in range(3)]
        self._ck(self._L.felog_pair_row_mix(self.h, *[ctypes.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def walk_entries(self, keep=True):
        """Device bytes of the walker entries (felog_walk_entries); 0 when the
        walker reads the plain CSR.  keep=False frees them first."""
        b = ctypes.c_uint64()
        self._ck(self._L.felog_walk_entries(self.h, 1 if keep else 0, ctypes.byref(b)))
        return b.value

    def walk_ceiling(self):
        """Memory skeleton of the last walk round (felog_walk_ceiling):
        returns (ms, tokens), the skeleton's device time and token count."""
        ms = ctypes.c_float()
        tok = ctypes.c_uint64()
        self._ck(self._L.felog_walk_ceiling(self.h, ctypes.byref(ms), ctypes.byref(tok)))
        return ms.value, tok.value

    def corpus(self):
        ns = ctypes.c_uint64()
        nt = ctypes.c_uint64()
        self._ck(self._L.felog_corpus_size(self.h, ctypes.byref(ns), ctypes.byref(nt)))
        tok = np.zeros(max(nt.value, 1), np.uint32)
        off = np.zeros(ns.value + 1, np.uint64)
        self._ck(self._L.felog_get_corpus(self.h, _addr(tok), len(tok), _addr(off), len(off)))
        return tok[: nt.value], off

    def set_corpus(self, tokens, sent_off):
        t = np.ascontiguousarray(tokens, np.uint32)
        o = np.ascontiguousarray(sent_off, np.uint64)
        self._ck(self._L.felog_set_corpus(self.h, _addr(t), _addr(o), len(o) - 1))

    def visit_freq(self):
        V, _ = self.graph_info()
        f = np.zeros(V, np.uint64)
        self._ck(self._L.felog_get_visit_freq(self.h, _addr(f)))
        return f

    # ---- trainer
    def init_model(self):
        self._ck(self._L.felog_init_model(self.h))

    def vocab(self):
        vs = ctypes.c_uint64()
        tw = ctypes.c_uint64()
        self._ck(self._L.felog_vocab_info(self.h, ctypes.byref(vs), ctypes.byref(tw)))
        V, _ = self.graph_info()
        vv = np.zeros(vs.value, np.uint32)
        id2 = np.zeros(V, np.uint32)
        self._ck(self._L.felog_get_vocab(self.h, _addr(vv), _addr(id2)))
        return vv, id2, vs.value, tw.value

    def train_round(self, round_=0, alpha=-1.0):
        st = TrainStats()
        self._ck(self._L.felog_train_round(self.h, round_, alpha, ctypes.byref(st)))
        return _struct_dict(st)

    def embeddings(self):
        vs = ctypes.c_uint64()
        self._ck(self._L.felog_vocab_info(self.h, ctypes.byref(vs), None))
        dim = self.opts.size
        s0 = np.zeros(vs.value * dim, np.float32)
        s1 = np.zeros(vs.value * dim, np.float32)
        self._ck(self._L.felog_get_embeddings(self.h, _addr(s0), _addr(s1), len(s0)))
        return s0, s1

    def set_embeddings(self, syn0, syn1):
        a = np.ascontiguousarray(syn0, np.float32) if syn0 is not None else None
        b = np.ascontiguousarray(syn1, np.float32) if syn1 is not None else None
        self._ck(self._L.felog_set_embeddings(self.h, _addr(a), _addr(b)))

    def score_pairs(self, ctx_rows, tgt_rows, labels, batch_of, n_batches):
        """FP32 dots of syn0[ctx] . syn1[tgt] as the trainer forms them, and the
        FP64 negative-sampling loss summed per batch."""
        c = np.ascontiguousarray(ctx_rows, np.int32)
        t = np.ascontiguousarray(tgt_rows, np.int32)
        lab = np.ascontiguousarray(labels, np.int8)
        b = np.ascontiguousarray(batch_of, np.uint64)
        dots = np.zeros(max(len(c), 1), np.float32)
        loss = np.zeros(max(n_batches, 1), np.float64)
        self._ck(self._L.felog_score_pairs(self.h, _addr(c), _addr(t), _addr(lab), _addr(b), len(c), n_batches,
                                           _addr(dots), _addr(loss)))
        return dots[: len(c)], loss[:n_batches]

    # ---- learned walk budget
    def budget_features(self):
        f = np.zeros(self.opts.v_num * 6, np.float32)
        self._ck(self._L.felog_budget_features(self.h, _addr(f)))
        return f.reshape(-1, 6)

    def budget_labels(self):
        c = np.zeros(self.opts.v_num, np.uint8)
        l = np.zeros(self.opts.v_num, np.float32)
        self._ck(self._L.felog_budget_labels(self.h, _addr(c), _addr(l)))
        return c, l

    def mlp_train(self, epochs=0, batch=0, lr=0.0, seed=1):
        o = MlpOpts(epochs, batch, lr, seed)
        st = MlpStats()
        self._ck(self._L.felog_mlp_train(self.h, ctypes.byref(o), ctypes.byref(st)))
        return _struct_dict(st)

    def mlp_state(self):
        s = np.zeros(MLP_STATE, np.float32)
        self._ck(self._L.felog_mlp_get_params(self.h, _addr(s)))
        return s

    def mlp_set_state(self, state):
        s = np.ascontiguousarray(state, np.float32)
        assert s.size == MLP_STATE
        self._ck(self._L.felog_mlp_set_params(self.h, _addr(s)))

    def mlp_gradient(self, params, X, count, length):
        p = np.ascontiguousarray(params, np.float32)
        x = np.ascontiguousarray(X, np.float32)
        c = np.ascontiguousarray(count, np.uint8)
        l = np.ascontiguousarray(length, np.float32)
        g = np.zeros(MLP_PARAMS, np.float32)
        loss = ctypes.c_double()
        self._ck(self._L.felog_mlp_gradient(self.h, _addr(p), _addr(x), _addr(c), _addr(l), len(c), _addr(g),
                                            ctypes.byref(loss)))
        return g, loss.value

    def mlp_predict(self):
        n = self.opts.v_num
        c = np.zeros(n, np.uint8)
        cf = np.zeros(n, np.float32)
        l = np.zeros(n, np.float32)
        self._ck(self._L.felog_mlp_predict(self.h, _addr(c), _addr(cf), _addr(l)))
        return c, cf, l

    def count_lost_updates(self, on=True):
        self._ck(self._L.felog_count_lost_updates(self.h, int(on)))

    def lost_updates(self):
        """(BF16-row updates, overwritten ones) since counting was turned on."""
        n, lost = ctypes.c_uint64(), ctypes.c_uint64()
        self._ck(self._L.felog_lost_updates(self.h, ctypes.byref(n), ctypes.byref(lost)))
        return n.value, lost.value

    def plan(self):
        ns, nsen, nb = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        self._ck(self._L.felog_plan_size(self.h, ctypes.byref(ns), ctypes.byref(nsen), ctypes.byref(nb)))
        sen = np.zeros(max(nsen.value, 1), np.int32)
        ss = np.zeros(ns.value + 1, np.uint64)
        bf = np.zeros(nb.value + 1, np.uint64)
        negs = np.zeros(max(ns.value * self.opts.negative, 1), np.int32)
        self._ck(self._L.felog_get_plan(self.h, _addr(sen), _addr(ss), _addr(bf), _addr(negs)))
        return dict(sen=sen[: nsen.value], sent_start=ss, batch_first=bf,
                    negs=negs[: ns.value * self.opts.negative])

    # ---- budget
    def budget_check(self, round_):
        st = BudgetStats()
        self._ck(self._L.felog_budget_check(self.h, round_, ctypes.byref(st)))
        return _struct_dict(st)

    def similarity(self):
        V, _ = self.graph_info()
        s = np.zeros(V, np.float32)
        self._ck(self._L.felog_get_similarity(self.h, _addr(s)))
        return s

    def cluster(self, classes, max_iter=10):
        """Spherical K-means over syn0 on the GPU (the -classes output).

        Returns (labels per vocabulary row, objective after each assignment pass)."""
        n = ctypes.c_uint64()
        self._ck(self._L.felog_vocab_info(self.h, ctypes.byref(n), None))
        lab = np.zeros(n.value, np.int32)
        obj = np.zeros(max(max_iter, 1) if max_iter else 10, np.float64)
        it = ctypes.c_int32()
        self._ck(self._L.felog_cluster_embeddings(self.h, classes, max_iter, _addr(lab), _addr(obj),
                                                  ctypes.byref(it)))
        return lab, obj[: it.value]

    # ---- loop
    def run(self):
        st = RunStats()
        self._ck(self._L.felog_run(self.h, ctypes.byref(st)))
        return _struct_dict(st)

    def write_embeddings(self, path):
        self._ck(self._L.felog_write_embeddings(self.h, path.encode()))

    def embeddings_into_async(self, syn0_ptr, n_floats):
        """Starts copying syn0 into caller memory (pinned) behind the next round; finish with wait_embeddings()."""
        self._ck(self._L.felog_copy_embeddings_async(self.h, syn0_ptr, n_floats))

    def wait_embeddings(self):
        self._ck(self._L.felog_wait_embeddings(self.h))

    def tuning_report(self):
        return self._L.felog_tuning_report(self.h).decode()

    def embeddings_into(self, syn0_ptr, n_floats):
        """Copies syn0 (vocabulary order, logical dims) into caller memory at syn0_ptr."""
        self._ck(self._L.felog_get_embeddings(self.h, syn0_ptr, None, n_floats))

    def set_stop_flags_from(self, ptr):
        self._ck(self._L.felog_set_stop_flags(self.h, ptr))

    def kernel_launches(self):
        return int(self._L.felog_kernel_launches(self.h))

    def timer_mark(self, which):
        self._ck(self._L.felog_timer_mark(self.h, which))

    def timer_elapsed(self):
        ms = ctypes.c_float()
        self._ck(self._L.felog_timer_elapsed(self.h, ctypes.byref(ms)))
        return ms.value


class SynthParams(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint64), ("v_target", ctypes.c_uint64), ("e_target", ctypes.c_uint64),
                ("a", ctypes.c_double), ("b", ctypes.c_double), ("c", ctypes.c_double), ("d", ctypes.c_double),
                ("weight_dist", ctypes.c_int), ("lognormal_mu", ctypes.c_double),
                ("lognormal_sigma", ctypes.c_double), ("holdout", ctypes.c_double), ("permute_ids", ctypes.c_int)]


class SynthInfo(ctypes.Structure):
    _fields_ = [("v_num", ctypes.c_uint64), ("n_full_edges", ctypes.c_uint64), ("n_train_edges", ctypes.c_uint64),
                ("n_test", ctypes.c_uint64), ("n_test_pos", ctypes.c_uint64), ("max_degree", ctypes.c_uint64)]


def synth_graph(seed, v_target, e_target, abcd=(0.57, 0.19, 0.19, 0.05), lognormal=False, holdout=0.1,
                permute=True, mu=0.0, sigma=1.0):
    """Seeded R-MAT graph with a held-out link-prediction split.

    Returns dict(v_num, edges (EDGE12 train edges), test_src, test_dst, test_label, info).
    """
    L = tools_lib()
    p = SynthParams(seed, v_target, e_target, *abcd, 1 if lognormal else 0, mu, sigma, holdout, int(permute))
    h = _P()
    rc = L.felog_synth_generate(ctypes.byref(p), ctypes.byref(h))
    if rc != 0:
        raise FelogError(1, f"felog_synth_generate failed ({rc})")
    try:
        info = SynthInfo()
        L.felog_synth_get_info(h, ctypes.byref(info))
        edges = np.zeros(info.n_train_edges, EDGE12)
        ts = np.zeros(info.n_test, np.uint32)
        td = np.zeros(info.n_test, np.uint32)
        tl = np.zeros(info.n_test, np.uint8)
        L.felog_synth_copy(h, _addr(edges), _addr(ts), _addr(td), _addr(tl))
    finally:
        L.felog_synth_free(h)
    return dict(v_num=int(info.v_num), edges=edges, test_src=ts, test_dst=td, test_label=tl,
                info=_struct_dict(info))


NOALLOC_MAX_ENTRIES = 1 << 22  # FELOG_NOALLOC_MAX_ENTRIES


def unigram_starts(counts):
    """First slot of every word in the reference's 1e8-slot unigram table
    (felog_unigram_starts; host only)."""
    c = np.ascontiguousarray(counts, dtype=np.uint64)
    start = np.zeros(len(c), np.uint64)
    st = gpu_lib().felog_unigram_starts(_addr(c), len(c), _addr(start))
    if st != 0:
        raise FelogError(st, "felog_unigram_starts failed (empty or more than 12.5 M words)")
    return start


def build_alias_noalloc(row_ptr_dev, weight_dev, v_num, e_num, prob_dev, alias_dev, stream=None):
    """felog_build_alias_noalloc on caller-owned device buffers (integer device addresses).

    For callers that cannot allocate device memory; raises FelogError on failure."""
    if not 0 < v_num < 2 ** 32:
        raise FelogError(1, f"v_num {v_num} outside [1, 2^32)")
    if not 0 <= e_num <= NOALLOC_MAX_ENTRIES:
        raise FelogError(1, f"e_num {e_num} outside [0, {NOALLOC_MAX_ENTRIES}]")
    L = gpu_lib()
    st = L.felog_build_alias_noalloc(row_ptr_dev, weight_dev, v_num, e_num, prob_dev, alias_dev, stream)
    if st != 0:
        raise FelogError(st, "felog_build_alias_noalloc failed (oversized graph, bad weight or CUDA error)")


def heldout_split(edges, v_num, holdout, seed):
    """felog_heldout_split (the gtrain tool's split): returns (train edges, test_src, test_dst, test_label)."""
    L = tools_lib()
    e = np.ascontiguousarray(edges, dtype=EDGE12)
    n = len(e)
    train = np.zeros(max(n, 1), EDGE12)
    cap = 2 * n + 2
    ts, td, tl = np.zeros(cap, np.uint32), np.zeros(cap, np.uint32), np.zeros(cap, np.uint8)
    nt, nx = ctypes.c_uint64(), ctypes.c_uint64()
    rc = L.felog_heldout_split(_addr(e), n, v_num, holdout, seed, _addr(train), ctypes.byref(nt), _addr(ts),
                               _addr(td), _addr(tl), ctypes.byref(nx))
    if rc != 0:
        raise FelogError(1, f"felog_heldout_split failed ({rc})")
    return train[: nt.value], ts[: nx.value], td[: nx.value], tl[: nx.value]


def auc(scores, labels):
    s = np.ascontiguousarray(scores, np.float32)
    lab = np.ascontiguousarray(labels, np.uint8)
    return tools_lib().felog_auc(_addr(s), _addr(lab), len(s))


def format_lf(values):
    """felog_format_lf: the floats as printf("%lf ") prints them (host only)."""
    x = np.ascontiguousarray(values, np.float32)
    cap = 64 * len(x) + 1
    buf = ctypes.create_string_buffer(cap)
    n = ctypes.c_uint64()
    st = gpu_lib().felog_format_lf(_addr(x) if len(x) else None, len(x), buf, cap, ctypes.byref(n))
    if st != 0:
        raise FelogError(st, "felog_format_lf failed")
    return buf.raw[: n.value].decode()
