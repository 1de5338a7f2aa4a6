"""The drop-in felog CLI end to end on a B200: the reference's flag set runs
the whole loop and writes -emb_output in the reference's text format
(word2vec.cu:2121-2127: "<vocab> <dim>" then "<vertex id> v_1 ... v_dim"); the
B200 forms (--precision bf16, --budget learned with the shipped model) run too."""
import os
import subprocess

import numpy as np
import pytest

import felog_b200 as fb
from conftest import ROOT

pytestmark = pytest.mark.gpu

CLI = os.path.join(ROOT, "info-centric_ge_b200", "felog_b200", "felog")


def read_text_embeddings(path):
    with open(path) as f:
        vs, dim = (int(x) for x in f.readline().split())
        ids, rows = [], []
        for line in f:
            p = line.split()
            ids.append(int(p[0]))
            rows.append([float(x) for x in p[1:]])
    return vs, dim, np.array(ids), np.array(rows, np.float64)


@pytest.mark.parametrize("extra", [[], ["--precision", "bf16", "--budget", "learned"]])
def test_cli_end_to_end(tmp_path, extra):
    g = fb.synth_graph(seed=0, v_target=4096, e_target=32768, holdout=0.1)
    V = g["v_num"]
    gp = tmp_path / "g.bin"
    g["edges"].tofile(gp)
    out = tmp_path / "emb.txt"
    cmd = [CLI, "-g", str(gp), "-v", str(V), "-w", str(V), "--min_L", "20", "--min_R", "2", "-o", str(tmp_path / "o"),
           "--make-undirected", "-size", "128", "-window", "10", "-negative", "5", "-sample", "1e-3", "-cbow", "0",
           "-reuse-neg", "0", "-min-count", "0", "-emb_output", str(out)] + extra
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    vs, dim, ids, rows = read_text_embeddings(out)
    assert dim == 128 and vs == len(ids) == V
    assert sorted(ids.tolist()) == list(range(V))
    assert np.isfinite(rows).all() and np.abs(rows).max() > 0
