"""Output forms of the -emb_output file on a B200.

-binary 1 (word2vec.cu:2119-2127): "<vocab> <dim>\\n", then per vocabulary row
"<vertex> " followed by dim raw float32 values and "\\n".

-classes k (word2vec.cu:2128-2175 writes one class per vocabulary row): the
library's spherical K-means.  Its stated objective is sum_v x_v . c_label(v)
over unit centroids; the test checks that the objective never decreases, that
a converged run is a fixed point (every centroid is the normalised sum of its
rows and every row's label is its best centroid, ties within FP32 rounding),
and that the objective equals an FP64 recomputation from the rows.
"""
import os
import subprocess

import numpy as np
import pytest

import felog_b200 as fb
from conftest import ROOT

pytestmark = pytest.mark.gpu

CLI = os.path.join(ROOT, "info-centric_ge_b200", "felog_b200", "felog")


def _trained(precision=0, dim=128, seed=5):
    g = fb.synth_graph(seed=seed, v_target=4096, e_target=32768, holdout=0.0)
    V = g["v_num"]
    f = fb.Felog(v_num=V, size=dim, window=10, negative=5, cbow=0, reuse_neg=0, min_count=0, seed=seed,
                 precision=precision)
    f.load_graph(g["edges"], V)
    f.init_model()
    for r in range(2):
        f.walk_round(r)
        f.train_round(r)
    return f, g


def test_binary_output_holds_raw_rows(tmp_path):
    f, g = _trained()
    # binary is a context option: a second context writes the binary form of the same rows
    s0, _ = f.embeddings()
    vv, _, vs, _ = f.vocab()
    V = g["v_num"]
    f2 = fb.Felog(v_num=V, size=128, window=10, negative=5, cbow=0, reuse_neg=0, min_count=0, seed=5, binary=1)
    f2.load_graph(g["edges"], V)
    f2.init_model()
    f2.set_embeddings(s0, f.embeddings()[1])
    p = str(tmp_path / "emb.bin")
    f2.write_embeddings(p)
    data = open(p, "rb").read()
    head, rest = data.split(b"\n", 1)
    assert head == f"{vs} 128".encode()
    pos = 0
    rows = s0.reshape(vs, 128)
    for a in range(vs):
        sp = rest.index(b" ", pos)
        assert int(rest[pos:sp]) == vv[a]
        vals = np.frombuffer(rest[sp + 1: sp + 1 + 4 * 128], dtype="<f4")
        np.testing.assert_array_equal(vals, rows[a])
        assert rest[sp + 1 + 4 * 128: sp + 2 + 4 * 128] == b"\n"
        pos = sp + 2 + 4 * 128
    assert pos == len(rest)
    f.close()
    f2.close()


def _objective_and_fixed_point(rows, lab, k):
    """FP64 objective of the labels with centroids = normalised label sums, and
    the largest amount by which any row prefers another centroid."""
    x = rows.astype(np.float64)
    cent = np.zeros((k, x.shape[1]))
    np.add.at(cent, lab, x)
    nrm = np.linalg.norm(cent, axis=1)
    ok = nrm > 0
    cent[ok] /= nrm[ok, None]
    dots = x @ cent.T
    obj = dots[np.arange(len(lab)), lab].sum()
    regret = (dots.max(axis=1) - dots[np.arange(len(lab)), lab]).max()
    return obj, regret


@pytest.mark.parametrize("precision", [0, 1])
def test_kmeans_objective_rises_to_a_fixed_point(precision):
    f, g = _trained(precision=precision)
    s0, _ = f.embeddings()
    vs = f.vocab()[2]
    rows = s0.reshape(vs, 128)
    k = 16
    lab, obj = f.cluster(k, max_iter=200)
    assert lab.shape == (vs,) and lab.min() >= 0 and lab.max() < k
    assert len(obj) < 200, "did not converge in 200 passes"
    # assignments compare FP32 dots, so a row whose two best centroids tie to
    # FP32 rounding may move and lower the exact objective by a rounding error:
    # the objective never falls by more than FP32 precision (2^-23 relative)
    assert np.all(np.diff(obj) >= -2.0 ** -23 * np.abs(obj[1:])), obj
    # converged: the last pass changed nothing, so labels are a fixed point of both steps
    ref_obj, regret = _objective_and_fixed_point(rows, lab, k)
    assert regret <= 4e-5 * np.abs(rows).sum(axis=1).max()
    assert abs(obj[-1] - ref_obj) <= 1e-5 * abs(ref_obj)
    # deterministic
    lab2, obj2 = f.cluster(k, max_iter=200)
    np.testing.assert_array_equal(lab, lab2)
    np.testing.assert_array_equal(obj, obj2)
    # a capped run reports one objective per pass
    lab3, obj3 = f.cluster(k, max_iter=3)
    assert len(obj3) == 3 and np.array_equal(obj3, obj[:3])
    f.close()


def test_cli_classes_writes_one_class_per_vertex(tmp_path):
    g = fb.synth_graph(seed=0, v_target=4096, e_target=32768, holdout=0.1)
    V = g["v_num"]
    gp = tmp_path / "g.bin"
    g["edges"].tofile(gp)
    out = tmp_path / "cls.txt"
    cmd = [CLI, "-g", str(gp), "-v", str(V), "-w", str(V), "--min_L", "20", "--min_R", "2", "-o", str(tmp_path / "o"),
           "--make-undirected", "-size", "128", "-window", "10", "-negative", "5", "-cbow", "0", "-reuse-neg", "0",
           "-min-count", "0", "-classes", "10", "-emb_output", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = open(out).read().splitlines()
    assert len(lines) == V
    ids = [int(x.split()[0]) for x in lines]
    cls = np.array([int(x.split()[1]) for x in lines])
    assert sorted(ids) == list(range(V))
    assert cls.min() >= 0 and cls.max() < 10 and len(np.unique(cls)) > 1
