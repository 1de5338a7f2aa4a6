"""Trained tables of the reference's own pipeline run, and the link scores the
end-to-end comparison applies to every embedding alike (test and bench
infrastructure).

oracle/_ref/ref_pipeline (the reference's walk engine and CUDA trainer,
compiled from its sources) writes, with its optional last argument, syn0 and
then syn1neg in the reference's -binary 1 layout (word2vec.cu:2119-2126):
"<vocab_size> <dim>\\n", then per vocabulary row "<vertex id> ", dim raw
float32 values and "\\n".
"""
import os
import subprocess
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_PIPELINE = os.path.join(ROOT, "oracle", "_ref", "ref_pipeline")


def _read_table(buf, pos):
    nl = buf.index(b"\n", pos)
    vs, dim = (int(x) for x in buf[pos:nl].split())
    pos = nl + 1
    ids = np.zeros(vs, np.int64)
    rows = np.zeros((vs, dim), np.float32)
    for a in range(vs):
        sp = buf.index(b" ", pos)
        ids[a] = int(buf[pos:sp])
        rows[a] = np.frombuffer(buf, dtype="<f4", count=dim, offset=sp + 1)
        pos = sp + 1 + 4 * dim + 1
    return ids, rows, pos


def read_ref_tables(path, v_num):
    """(syn0, syn1) of a ref_pipeline dump, indexed by vertex id (v_num rows)."""
    buf = open(path, "rb").read()
    ids0, r0, pos = _read_table(buf, 0)
    ids1, r1, pos = _read_table(buf, pos)
    assert pos == len(buf) and np.array_equal(ids0, ids1)
    s0 = np.zeros((v_num, r0.shape[1]), np.float32)
    s1 = np.zeros_like(s0)
    s0[ids0] = r0
    s1[ids1] = r1
    return s0, s1


def run_reference(edges, v_num, rounds, timeout=1800):
    """Runs the reference pipeline for `rounds` rounds (one walker per vertex)
    on the given training edges and returns its (syn0, syn1) by vertex id."""
    with tempfile.TemporaryDirectory() as td:
        gp = os.path.join(td, "g.bin")
        ep = os.path.join(td, "emb.bin")
        edges.tofile(gp)
        r = subprocess.run([REF_PIPELINE, gp, str(v_num), "1", str(rounds - 1), str(v_num), ep],
                           capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"ref_pipeline exited {r.returncode}: {r.stderr[-500:]}")
        return read_ref_tables(ep, v_num)


def link_scores(syn0, syn1, src, dst):
    """FP64 link scores of the pairs (src[i], dst[i]) from tables indexed by
    vertex id: raw cosine of the syn0 rows, the same cosine after removing the
    mean syn0 row, and the skip-gram score (syn0[u] . syn1[v] + syn0[v] .
    syn1[u]) / 2 (the trainer's own logit of a (center, context) pair)."""
    e0 = syn0.astype(np.float64)
    e1 = syn1.astype(np.float64)

    def cos(e):
        n = e / np.maximum(np.linalg.norm(e, axis=1, keepdims=True), 1e-300)
        return np.einsum("ij,ij->i", n[src], n[dst])

    return {
        "cosine": cos(e0),
        "cosine_centered": cos(e0 - e0.mean(axis=0, keepdims=True)),
        "sgns": 0.5 * (np.einsum("ij,ij->i", e0[src], e1[dst]) + np.einsum("ij,ij->i", e0[dst], e1[src])),
    }


def auc(score, label):
    """Exact Mann-Whitney AUC (ties count one half), FP64."""
    from scipy.stats import rankdata

    label = np.asarray(label).astype(bool)
    r = rankdata(np.asarray(score, np.float64), method="average")
    npos = int(label.sum())
    nneg = len(label) - npos
    return float((r[label].sum() - npos * (npos + 1) / 2.0) / (npos * nneg))


def link_aucs(syn0, syn1, g):
    sc = link_scores(syn0, syn1, g["test_src"], g["test_dst"])
    return {k: auc(v, g["test_label"]) for k, v in sc.items()}


def tables_by_vertex(f):
    """(syn0, syn1) of a felog_b200 context, rows indexed by vertex id."""
    s0, s1 = f.embeddings()
    _, id2, vs, _ = f.vocab()
    dim = f.opts.size
    return s0.reshape(vs, dim)[id2], s1.reshape(vs, dim)[id2]


def fit_pairs(g, n=20000, seed=12345):
    """Evaluation pairs of the fit score: n training edges (u, v) as positives
    and, for each, a negative (u, w) with w an endpoint of a uniformly chosen
    training edge (so w is drawn in proportion to its degree, like the
    positives' endpoints) that is neither u nor a neighbour of u.  Returns
    (src, dst, label)."""
    src = g["edges"]["src"].astype(np.int64)
    dst = g["edges"]["dst"].astype(np.int64)
    rng = np.random.default_rng(seed)
    lo, hi = np.minimum(src, dst), np.maximum(src, dst)
    known = set((lo << 32 | hi).tolist())
    ts, td = g["test_src"].astype(np.int64), g["test_dst"].astype(np.int64)
    p = g["test_label"] == 1
    known |= set((np.minimum(ts[p], td[p]) << 32 | np.maximum(ts[p], td[p])).tolist())
    ends = np.concatenate([src, dst])
    m = rng.choice(len(src), min(n, len(src)), replace=False)
    us, vs = src[m], dst[m]
    ws = np.empty_like(us)
    for i, u in enumerate(us.tolist()):
        while True:
            w = int(ends[rng.integers(len(ends))])
            if w != u and (min(u, w) << 32 | max(u, w)) not in known:
                break
        ws[i] = w
    return (np.concatenate([us, us]), np.concatenate([vs, ws]),
            np.concatenate([np.ones(len(us), np.uint8), np.zeros(len(us), np.uint8)]))


def fit_aucs(syn0, syn1, pairs):
    s, d, lab = pairs
    return {k: auc(v, lab) for k, v in link_scores(syn0, syn1, s, d).items()}
