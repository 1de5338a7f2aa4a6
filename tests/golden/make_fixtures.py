"""Regenerates the golden fixtures under tests/golden/ from the reference.

Needs the harness
binaries built by ``make -C oracle ref`` (oracle/_ref/) from the reference
checkout that FELOG_REFERENCE names.  Every fixture is the
reference's own output on seeded synthetic inputs:

  walk_*.npz   include/walk.hpp run by oracle/_ref/ref_walk with injected draws:
               the graph, per-walker draw streams and the per-round corpus.
  split_*.npz  src/tools/gtrain.cpp (the held-out split tool) run by
               oracle/_ref/ref_gtrain with its rand() fed from the split's
               seeded stream: the input edges and the tool's train edges,
               test pairs and labels.
  gcn_*.npz    src/tools/gcn.cpp (the offline common-neighbour tool) run by
               oracle/_ref/ref_gcn on text edge lists: per input edge its
               common-neighbour count.
  plan_*.npz   src/word2vec.cu's ReadVocabFromDegree / InitNet /
               InitUnigramTable / TrainModelThreadMemory run by
               oracle/_ref/ref_sgns_plan: vocabulary order, subsampling
               thresholds, unigram table digest, syn0 head and the batch plan
               (sentence_length, sen, negSample per batch).

Usage: python tests/golden/make_fixtures.py [walk] [plan] [gcn] [split]   (default: all)
"""
import hashlib
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REFBIN = os.path.join(ROOT, "oracle", "_ref")
sys.path.insert(0, os.path.join(ROOT, "info-centric_ge_b200"))
sys.path.insert(0, HERE)

import felog_b200 as fb  # noqa: E402  (tools library: synthetic graphs)
from recipes import pack, splitmix64, synth_corpus  # noqa: E402

EDGE12 = fb.EDGE12


def read_walk_output(path, rounds):
    b = np.fromfile(path, dtype=np.uint32)
    i = 0
    corp = []
    for _ in range(rounds):
        n = int(b[i]); i += 1
        sents = []
        for _ in range(n):
            L = int(b[i]); i += 1
            sents.append(b[i:i + L].copy()); i += L
        corp.append(sents)
    nw = int(b[i]); i += 1
    log = []
    for _ in range(nw):
        rnd, st, ni = int(b[i]), int(b[i + 1]), int(b[i + 2]); i += 3
        idx = b[i:i + ni].copy(); i += ni
        npp = int(b[i]); i += 1
        p = b[i:i + npp].view(np.int32).copy(); i += npp
        log.append((rnd, st, idx, p))
    assert i == len(b)
    return corp, log


def run_walk_fixture(name, edges, V, min_L, rounds, seed, stop=None, walker_num=None):
    with tempfile.TemporaryDirectory() as td:
        g = os.path.join(td, "g.bin")
        out = os.path.join(td, "w.bin")
        np.ascontiguousarray(edges, EDGE12).tofile(g)
        cmd = [os.path.join(REFBIN, "ref_walk"), g, str(V), str(min_L), str(rounds), str(seed), out]
        if stop is not None or walker_num is not None:
            sp = os.path.join(td, "stop.u8")
            (stop if stop is not None else np.zeros(V, np.uint8)).astype(np.uint8).tofile(sp)
            cmd += [sp, str(walker_num if walker_num is not None else V)]
        subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
        corp, log = read_walk_output(out, rounds)
    data = dict(edges=np.ascontiguousarray(edges, EDGE12), V=np.uint32(V), min_L=np.uint32(min_L),
                rounds=np.uint32(rounds), walker_num=np.uint32(walker_num if walker_num else V))
    if stop is not None:
        data["stop"] = stop.astype(np.uint8)
    for r in range(rounds):
        tok, off = pack(corp[r])
        ws = [l for l in log if l[0] == r + 1]
        data[f"r{r}_tokens"] = tok
        data[f"r{r}_off"] = off
        data[f"r{r}_start"] = np.array([l[1] for l in ws], np.uint32)
        data[f"r{r}_idx_off"] = pack([l[2] for l in ws])[1]
        data[f"r{r}_idx"] = pack([l[2] for l in ws])[0]
        data[f"r{r}_p_off"] = pack([l[3].view(np.uint32) for l in ws])[1]
        data[f"r{r}_p"] = pack([l[3].view(np.uint32) for l in ws])[0].view(np.int32)
    np.savez_compressed(os.path.join(HERE, name), **data)
    lens = [len(s) for s in corp[0]]
    print(f"{name}: V={V} rounds={rounds} sentences={len(corp[0])} tokens/round={sum(lens)} "
          f"len range {min(lens)}..{max(lens)}")


def edge_case_graph():
    """Hand-made graph exercising self-loops, multi-edges, the degree-2
    self-loop stop (walk.hpp:977-979), step-0 self-loop redraws (:981-983)
    and common-neighbour counts that reach the degree (cn >= deg_s)."""
    rows = []
    V = 40
    s = 11
    for v in range(V):
        # a ring keeps everything connected and visited
        rows.append((v, (v + 1) % V, 0.5))
    for v in range(0, V, 4):
        rows.append((v, (v + 7) % V, 1.0))       # cn = 1
        rows.append((v, (v + 7) % V, 0.25))      # multi-edge
    for v in range(1, V, 5):
        rows.append((v, v, 0.75))                # self-loop on a vertex with other edges
    for v in range(2, V, 6):
        rows.append((v, (v + 13) % V, 3.0))      # cn = 3 (>= small degrees)
    for v in range(3, V, 9):
        rows.append((v, (v + 5) % V, 50.0))      # cn = 50 > deg: negative denominator
    for v in range(5, V, 10):
        rows.append((v, (v + 2) % V, 2.0))       # cn = 2
    # vertex V: its only edge is a self-loop -> degree 2, first neighbour itself
    rows.append((V, V, 0.5))
    V += 1
    rng = []
    for i, (a, b, w) in enumerate(rows):
        s = splitmix64(s + i)
        rng.append(s)
    order = np.argsort(np.array(rng, dtype=np.uint64), kind="stable")
    e = np.zeros(len(rows), EDGE12)
    for k, i in enumerate(order):
        e[k] = rows[i]
    return e, V


def write_corpus(path, sents):
    buf = [np.array([len(sents)], np.uint32)]
    for s in sents:
        buf += [np.array([len(s)], np.uint32), np.asarray(s, np.uint32)]
    np.concatenate(buf).tofile(path)


def run_plan_fixture(name, deg, sents, recipe, dim, window, negative, sample, min_count):
    with tempfile.TemporaryDirectory() as td:
        dp = os.path.join(td, "deg.bin")
        cp = os.path.join(td, "corpus.bin")
        op = os.path.join(td, "plan.bin")
        tp = os.path.join(td, "table.bin")
        np.asarray(deg, np.uint32).tofile(dp)
        write_corpus(cp, sents)
        subprocess.run([os.path.join(REFBIN, "ref_sgns_plan"), dp, cp, op, str(dim), str(window),
                        str(negative), repr(sample), str(min_count), tp], check=True, stdout=subprocess.DEVNULL)
        b = open(op, "rb").read()
        table_sha = hashlib.sha256(open(tp, "rb").read()).hexdigest()
    o = 0

    def take(dt, n):
        nonlocal o
        a = np.frombuffer(b, dtype=dt, count=int(n), offset=o)
        o += a.nbytes
        return a.copy()

    vs, tw = take(np.int64, 2)
    vv = take(np.uint32, vs)
    nthr = take(np.uint32, 1)[0]
    thr = take(np.uint16, nthr)
    take(np.uint64, 1)
    thead = take(np.int32, 4096)
    s0 = take(np.float32, min(vs, 64) * dim)
    nb = take(np.uint32, 1)[0]
    sl, sen, ng = [], [], []
    for _ in range(nb):
        cnt, tot = take(np.uint32, 2)
        sl.append(take(np.int32, cnt + 1))
        sen.append(take(np.int32, tot))
        ng.append(take(np.int32, cnt * negative))
    assert o == len(b)
    sen_all = np.concatenate(sen) if sen else np.zeros(0, np.int32)
    neg_all = np.concatenate(ng) if ng else np.zeros(0, np.int32)
    data = dict(deg=np.asarray(deg, np.uint32), recipe=np.array(recipe, np.int64), dim=np.int32(dim),
                window=np.int32(window), negative=np.int32(negative), sample=np.float64(sample),
                min_count=np.int32(min_count), vocab_size=np.int64(vs), train_words=np.int64(tw),
                vocab_vertex=vv, thr=thr, table_sha256=np.bytes_(table_sha), table_head=thead, syn0_head=s0,
                batch_cnt=np.array([len(x) - 1 for x in sl], np.int64),
                batch_tot=np.array([len(x) for x in sen], np.int64),
                sentence_length=np.concatenate(sl) if sl else np.zeros(0, np.int32),
                sen_sha256=np.bytes_(hashlib.sha256(sen_all.tobytes()).hexdigest()),
                negs_sha256=np.bytes_(hashlib.sha256(neg_all.tobytes()).hexdigest()),
                sen_head=sen_all[:20000], negs_head=neg_all[:20000])
    np.savez_compressed(os.path.join(HERE, name), **data)
    print(f"{name}: vocab={vs} batches={nb} sentences={sum(len(x) - 1 for x in sl)} kept={len(sen_all)} "
          f"subsampled words={int((thr < 65535).sum()) if len(thr) else 0}")


def run_gcn_fixture(name, src, dst, V, undirected):
    with tempfile.TemporaryDirectory() as td:
        ein, eout = os.path.join(td, "e.txt"), os.path.join(td, "o.txt")
        with open(ein, "w") as fh:
            fh.write("".join(f"{a} {b}\n" for a, b in zip(src.tolist(), dst.tolist())))
        subprocess.run([os.path.join(REFBIN, "ref_gcn"), ein, eout, str(V), str(int(undirected))], check=True,
                       stdout=subprocess.DEVNULL)
        out = np.loadtxt(eout, dtype=np.int64, ndmin=2)
    assert out.shape == (len(src), 3) and (out[:, 0] == src).all() and (out[:, 1] == dst).all()
    np.savez_compressed(os.path.join(HERE, name), src=src.astype(np.uint32), dst=dst.astype(np.uint32),
                        v_num=np.uint32(V), undirected=np.uint8(undirected), cn=out[:, 2].astype(np.int32))
    print(name, len(src), "edges", flush=True)


def gcn_fixtures():
    rng = np.random.default_rng(2024)
    # small multigraph: repeated edges, reciprocal pairs and self-loops
    V = 64
    a = rng.integers(0, V, 420)
    b = (a + 1 + rng.zipf(1.6, 420) % (V - 1)) % V
    src = np.concatenate([a, b[:40], a[:30], np.arange(0, V, 9)])
    dst = np.concatenate([b, a[:40], b[:30], np.arange(0, V, 9)])
    run_gcn_fixture("gcn_multi64_undirected.npz", src, dst, V, True)
    # directed: every vertex also gets an out-edge so that no neighbour list is empty
    ring = np.arange(V)
    run_gcn_fixture("gcn_multi64_directed.npz", np.concatenate([src, ring]), np.concatenate([dst, (ring + 1) % V]),
                    V, False)
    # R-MAT graph with hubs (both lists long), plus reciprocal copies of 5% of its edges
    g = fb.synth_graph(seed=4, v_target=4096, e_target=40000, holdout=0.0)
    e = g["edges"]
    k = len(e) // 20
    src = np.concatenate([e["src"], e["dst"][:k]])
    dst = np.concatenate([e["dst"], e["src"][:k]])
    run_gcn_fixture("gcn_rmat4096_undirected.npz", src, dst, g["v_num"], True)


def run_split_fixture(name, edges, V, sample, seed):
    with tempfile.TemporaryDirectory() as td:
        paths = [os.path.join(td, x) for x in ("e.txt", "tr.txt", "te.txt", "tl.txt")]
        with open(paths[0], "w") as fh:
            fh.write("".join(f"{a}\t{b}\t0\n" for a, b in zip(edges["src"].tolist(), edges["dst"].tolist())))
        subprocess.run([os.path.join(REFBIN, "ref_gtrain")] + paths + [repr(sample), str(V), str(seed)], check=True,
                       stdout=subprocess.DEVNULL)
        tr = np.loadtxt(paths[1], dtype=np.uint32, ndmin=2)
        te = np.loadtxt(paths[2], dtype=np.uint32, ndmin=2)
        tl = np.loadtxt(paths[3], dtype=np.uint8, ndmin=1)
    np.savez_compressed(os.path.join(HERE, name), src=edges["src"], dst=edges["dst"], v_num=np.uint32(V),
                        sample=np.float64(sample), seed=np.uint64(seed), train_src=tr[:, 0], train_dst=tr[:, 1],
                        test_src=te[:, 0], test_dst=te[:, 1], test_label=tl)
    print(name, len(edges), "edges ->", len(tr), "train,", len(tl), "test", flush=True)


def split_fixtures():
    g = fb.synth_graph(seed=5, v_target=300, e_target=1200, holdout=0.0)
    run_split_fixture("split_rmat300.npz", g["edges"], g["v_num"], 0.1, 77)
    g = fb.synth_graph(seed=6, v_target=4096, e_target=30000, holdout=0.0)
    run_split_fixture("split_rmat4096.npz", g["edges"], g["v_num"], 0.05, 78)
    # a star and a path: many degree-1 endpoints (redrawn positives), few non-edges per vertex
    star = np.zeros(60, fb.EDGE12)
    star["src"] = 0
    star["dst"] = np.arange(1, 61)
    path = np.zeros(59, fb.EDGE12)
    path["src"] = np.arange(1, 60)
    path["dst"] = np.arange(2, 61)
    run_split_fixture("split_star_path.npz", np.concatenate([star, path]), 61, 0.2, 79)


def main():
    parts = set(sys.argv[1:]) or {"walk", "plan", "gcn", "split"}
    if "split" in parts:
        split_fixtures()
    if "gcn" in parts:
        gcn_fixtures()
    if "walk" not in parts and "plan" not in parts:
        return
    # walks
    g1 = fb.synth_graph(seed=0, v_target=512, e_target=2048, holdout=0.1)
    run_walk_fixture("walk_rmat512.npz", g1["edges"], g1["v_num"], 20, 3, 7)
    V = g1["v_num"]
    stop = np.zeros(V, np.uint8)
    deg = np.bincount(np.concatenate([g1["edges"]["src"], g1["edges"]["dst"]]), minlength=V)
    stop[np.argsort(-deg, kind="stable")[:12]] = 1  # hubs: surely visited by other walkers
    run_walk_fixture("walk_rmat512_stop_w2.npz", g1["edges"], V, 20, 2, 8, stop=stop, walker_num=2 * V)
    run_walk_fixture("walk_rmat512_minl5.npz", g1["edges"], V, 5, 1, 9)
    e, Ve = edge_case_graph()
    run_walk_fixture("walk_edgecases.npz", e, Ve, 20, 2, 10)
    g3 = fb.synth_graph(seed=3, v_target=4096, e_target=32768, holdout=0.1)
    run_walk_fixture("walk_rmat4096.npz", g3["edges"], g3["v_num"], 20, 1, 11)
    # trainer plans: degrees of the 4096 graph, seeded synthetic corpora
    Vd = g3["v_num"]
    deg3 = np.bincount(np.concatenate([g3["edges"]["src"], g3["edges"]["dst"]]), minlength=Vd).astype(np.uint32)
    for name, recipe, sample, mc, win, neg, dim in [
        ("plan_multibatch.npz", (Vd, 40000, 5, 0, 1200, 8), 1e-3, 0, 10, 5, 128),
        ("plan_subsample.npz", (Vd, 3000, 6, 97, 1500, 30), 1e-5, 0, 5, 7, 64),
        ("plan_nosample_long.npz", (Vd, 2000, 7, 2, 1200, 40), 0.0, 0, 10, 5, 128),
        ("plan_tokens_sub.npz", (Vd, 1200, 8, 2, 1100, 40), 1e-4, 0, 8, 5, 128),
    ]:
        sents = synth_corpus(recipe[0], recipe[1], recipe[2], recipe[3], recipe[4], recipe[5])
        run_plan_fixture(name, deg3, sents, recipe, dim, win, neg, sample, mc)


if __name__ == "__main__":
    main()
