#!/usr/bin/env python
"""Benchmark of the FeLoG graph-embedding hot path on B200.

Workload (default): the mid-scale configuration - a seed-1 R-MAT graph
(a, b, c, d = .57, .19, .19, .05) over 2,238,731 vertex ids with 34.7M unique
undirected edges, float32 weights uniform in (0, 1], 5 % of the edges held out
(isolated vertices removed), min_L 20, min_R 2, skip-gram dim 128, window 10,
negative 5, sample 1e-3, reuse-neg 0.  Synthetic data (seeded); the tables and
CSR are larger than L2, so no flush is needed.

Forms (--form): `learned-bf16` (default: BF16 tables with FP32 master rows for
the top 1%, learned walk budget from the committed MLP trained on the
C4-shaped graph) and `plain-fp32` (the reference's arithmetic and criterion).

One step = one round of the hot path: a walk round over every vertex whose
walkers are not stopped (biased walk + information-centric stop), the
trainer's batch plan, pair stream and skip-gram pass over that round's corpus,
and the per-vertex budget check (from round min_R on).  `value` is corpus
tokens per second through the whole round (each token is one walk step and one
trainer word), timed with CUDA events on the library's stream; `e2e` is the
same through the C ABI with the round's stop flags copied in from pinned host
memory and the trained embeddings copied back every round (the reference
copies syn0 back after every round, word2vec.cu:1264).  `forms` runs plain FP32
and learned BF16 end to end (until the stop-all rule) on the same graph and
reports job time, tokens and held-out link-prediction AUC for each.

`--impl reference` times the reference's own implementation of the path
(oracle/_ref/ref_pipeline, compiled from the reference sources) on the box:
its CPU walk engine with all host threads and its CUDA skip-gram kernel.
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "info-centric_ge_b200"))

CONFIGS = {
    "c2": dict(workload="plain FP32, seed-1 R-MAT 2,238,731 vertex ids / 34.7M undirected edges, 5% held out",
               seed=1, v_target=2238731, e_target=34_700_000, abcd=(0.57, 0.19, 0.19, 0.05), lognormal=False,
               holdout=0.05),
    "prof": dict(workload="profiling case, seed-1 R-MAT 524,288 vertex ids / 8M undirected edges, 5% held out",
                 seed=1, v_target=524288, e_target=8_000_000, abcd=(0.57, 0.19, 0.19, 0.05), lognormal=False,
                 holdout=0.05),
    "c4": dict(workload="plain FP32, seed-2 R-MAT (.6/.15/.15/.1) 3,072,441 vertex ids / 117M undirected edges, "
                        "lognormal(0, 1) weights, 5% held out",
               seed=2, v_target=3072441, e_target=117_000_000, abcd=(0.6, 0.15, 0.15, 0.1), lognormal=True,
               holdout=0.05),
    # C4 with the reference's offline step in front: the gcn tool's common-neighbour
    # count of every training edge becomes its edge data (gcn.cpp:304-357), which
    # the walker's trace test reads as cn (walk.hpp:997)
    "c4cn": dict(workload="plain FP32, seed-2 R-MAT (.6/.15/.15/.1) 3,072,441 vertex ids / 117M undirected edges, "
                          "edge data = common-neighbour counts (gcn tool), 5% held out",
                 seed=2, v_target=3072441, e_target=117_000_000, abcd=(0.6, 0.15, 0.15, 0.1), lognormal=True,
                 holdout=0.05, edge_data="cn"),
    "c1": dict(workload="plain FP32, seed-0 R-MAT 16,384 vertex ids / 131,072 undirected edges, 10% held out",
               seed=0, v_target=16384, e_target=131072, abcd=(0.57, 0.19, 0.19, 0.05), lognormal=False,
               holdout=0.10),
}
# Configurations too large for a host edge list: the graph is generated on the
# device (felog_load_rmat, the same edges the host generator would draw, no
# held-out split) and every round is walked and trained in pieces of `piece`
# walkers (a step of the benchmark is one piece).
STREAMED = {
    "c5": dict(workload="learned-bf16, seed-3 R-MAT (.57/.19/.19/.05) 111M vertex ids / 1.6B undirected edges, "
                        "weights uniform in (0, 1], generated on the device",
               seed=3, v_target=111_000_000, e_target=1_600_000_000, abcd=(0.57, 0.19, 0.19, 0.05), piece=8_000_000),
    "c5-small": dict(workload="learned-bf16, seed-3 R-MAT (.57/.19/.19/.05) 4M vertex ids / 60M undirected edges "
                              "(the C5 path at 1/27 scale), generated on the device",
                     seed=3, v_target=4_000_000, e_target=60_000_000, abcd=(0.57, 0.19, 0.19, 0.05), piece=1_000_000),
}
TRAIN = dict(min_length=20, min_rounds=2, size=128, window=10, negative=5, sample=1e-3, cbow=0, reuse_neg=0,
             min_count=0)
FORMS = {
    # the reference's arithmetic, criterion and per-pair negatives
    "plain-fp32": dict(precision=0, budget_mode=0, reuse_neg=0),
    # BF16 tables + learned budget, per-pair negatives
    "learned-bf16": dict(precision=1, budget_mode=1, reuse_neg=0),
    # BF16 tables + learned budget, -reuse-neg 2 center tiles (shared negatives per sentence)
    "learned-bf16-tile": dict(precision=1, budget_mode=1, reuse_neg=2),
    # FP32 tables + learned budget + center tiles
    "learned-fp32-tile": dict(precision=0, budget_mode=1, reuse_neg=2),
    # BF16 tables + learned budget + center tiles scored on the tensor cores
    "learned-bf16-tc": dict(precision=1, budget_mode=1, reuse_neg=3),
    # BF16 tables + learned budget, -reuse-neg 4 window tiles (the skip-gram windows; each center's
    # contexts share the K negatives drawn for its first context)
    "learned-bf16-window": dict(precision=1, budget_mode=1, reuse_neg=4),
}
BUDGET_MODEL = os.path.join(ROOT, "info-centric_ge_b200", "felog_b200", "budget_mlp_c4.npy")
METRIC = "walk+SGNS corpus tokens/s (walk steps/s and SGNS words/s reported alongside)"
# algorithmic bytes of a walk step in the sector model of the reference's CSR:
# the candidate's adjacency sector, its row_ptr sector, the 4-B token; with the
# walker entries a step reads one 32-B sector, which walk_kernel.layout states
WALK_BYTES_PER_STEP = 68
# DRAM bytes per pair of k_sgns_train_pairs<128, 5> (dram__bytes_read.sum + dram__bytes_write.sum of one ncu
# capture of the profiling case's timed round divided by its 66.0 M pairs), scaled to a launch
DRAM_BYTES_PER_PAIR = {"fp32": 1055.6, "bf16": 244.1}  # bf16: 5 blocks per SM; fp32: 4
SGNS_BYTES_PER_PAIR = {"fp32": 7168,   # 14 rows x 128 x 4 B (read + write syn0 row and 6 syn1 rows)
                       "bf16": 3584}   # the same rows at 2 B per value (FP32 master rows: top 1%)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples during the timed region (median SM clock, throttle reasons)."""

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_graph(cfg):
    import felog_b200 as fb
    t = time.time()
    g = fb.synth_graph(seed=cfg["seed"], v_target=cfg["v_target"], e_target=cfg["e_target"], abcd=cfg["abcd"],
                       lognormal=cfg["lognormal"], holdout=cfg["holdout"])
    log(f"graph: {g['info']} in {time.time() - t:.1f}s")
    if cfg.get("edge_data") == "cn":
        f = fb.Felog(v_num=g["v_num"])
        src = np.ascontiguousarray(g["edges"]["src"], np.uint32)
        dst = np.ascontiguousarray(g["edges"]["dst"], np.uint32)
        cn, ms = f.common_neighbours(src, dst, g["v_num"], True)
        f.close()
        g["edges"]["data"] = cn.astype(np.float32)
        log(f"edge data: common neighbours in {ms:.1f} ms (mean {cn.mean():.2f}, max {cn.max()})")
    return g


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(pg, x):
    if pg is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(pg, x):
    if pg is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def cpu_baseline(g, cfg):
    """The reference's own path (oracle/_ref/ref_pipeline: its walk engine on all
    host cores, its CUDA skip_gram_kernel) on a bounded sample of the workload:
    two rounds of the same graph (one warm-up, one timed), reported as corpus
    tokens/s.  Without the harness, the oracle (CPU restatement, one thread) on
    60k walkers and 1500 sentences."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_pipeline")
    if os.path.exists(exe):
        import tempfile
        with tempfile.TemporaryDirectory() as td:
            gp = os.path.join(td, "g.bin")
            g["edges"].tofile(gp)
            res = subprocess.run([exe, gp, str(g["v_num"]), "1", "1", "0"], capture_output=True, text=True)
        lines = re.findall(r'\{"tokens".*?\}', res.stdout)
        if res.returncode == 0 and lines:
            d = json.loads(lines[-1])
            return {"value": d["tokens"] / d["seconds"], "unit": "tokens/s", "cores": d["threads"],
                    "kind": "reference",
                    "sample": f"one timed round after one warm-up round, {d['walkers']} walkers: the reference walk "
                              f"engine on {d['threads']} host threads + the reference skip_gram_kernel",
                    "walk_steps_per_s": d["walk_tokens"] / d["walk_seconds"],
                    "sgns_words_per_s": d["train_words"] / d["train_seconds"]}
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_binding as ob
    V = g["v_num"]
    c = ob.OracleCsr(g["edges"], V)
    nw = min(60000, V)
    t0 = time.perf_counter()
    tok, off, _, st = ob.walk_round(c, nw, TRAIN["min_length"], seed=1, round_=0)
    t_walk = time.perf_counter() - t0
    vv, vcn, id2, vs, tw = ob.vocab(c.deg, 0)
    thr, used = ob.subsample_thresholds(vcn, TRAIN["sample"], tw)
    table = ob.unigram_table(vcn)
    et = ob.exp_table()
    syn0 = np.zeros(vs * 128, np.float32)
    syn0[:] = (np.arange(vs * 128) % 97 - 48).astype(np.float32) / (97 * 128)
    syn1 = np.zeros(vs * 128, np.float32)
    ns = 1500
    t2, o2 = tok[: int(off[ns])], off[: ns + 1]
    pl = ob.plan_batches(t2, o2, id2, thr, used, table, vs, TRAIN["negative"])
    t1 = time.perf_counter()
    ob.skipgram_batch(syn0, syn1, et, table, vs, pl["sen"], pl["sent_start"], 0, len(pl["sent_start"]) - 1,
                      TRAIN["window"], 128, TRAIN["negative"], 0.025)
    t_train = time.perf_counter() - t1
    walk_rate = len(tok) / t_walk
    train_rate = int(o2[-1]) / t_train
    value = 1.0 / (1.0 / walk_rate + 1.0 / train_rate)
    return {"value": value, "unit": "tokens/s", "cores": 1, "kind": "port",
            "sample": f"oracle walk of {nw} walkers ({len(tok)} tokens, {t_walk:.1f}s) + skip-gram over "
                      f"{ns} sentences ({int(o2[-1])} tokens, {t_train:.1f}s), 1 thread",
            "walk_steps_per_s": walk_rate, "sgns_words_per_s": train_rate}


def cpu_baseline_resident(f, V, n_walkers=60000, n_sent=1500):
    """The oracle (CPU restatement, one thread) on a bounded sample of a graph
    that only the device holds (C5, generated in HBM): the CSR copied out of
    the context, the walk of the first n_walkers walkers and the skip-gram pass
    over the first n_sent of their sentences.  syn0 and syn1 span the whole
    vocabulary but only the rows the sample touches are written (syn1 starts at
    zero as in InitNet, syn0 rows of the sample's words get the fixed init), so
    untouched pages are never allocated.  Reported as corpus tokens/s through
    walk + train."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_binding as ob
    rp, nb, dt = f.csr()

    class HostCsr:  # the oracle's CSR view of the copied arrays
        def __init__(self):
            self.c = ob.Csr(V, len(nb), ob.ptr(rp, ob.u64p), ob.ptr(nb, ob.u32p), ob.ptr(dt, ob.f32p))
            self.deg = np.diff(rp).astype(np.uint32)

    c = HostCsr()
    t0 = time.perf_counter()
    tok, off, _, st = ob.walk_round(c, n_walkers, TRAIN["min_length"], seed=1, round_=0)
    t_walk = time.perf_counter() - t0
    vv, vcn, id2, vs, tw = ob.vocab(c.deg, 0)
    thr, used = ob.subsample_thresholds(vcn, TRAIN["sample"], tw)
    table = ob.unigram_table(vcn)
    et = ob.exp_table()
    dim = TRAIN["size"]
    syn0 = np.zeros(vs * dim, np.float32)
    syn1 = np.zeros(vs * dim, np.float32)
    t2, o2 = tok[: int(off[n_sent])], off[: n_sent + 1]
    rows = np.unique(id2[t2]).astype(np.int64)
    s0 = syn0.reshape(vs, dim)
    s0[rows] = ((rows[:, None] * dim + np.arange(dim)[None, :]) % 97 - 48).astype(np.float32) / (97 * dim)
    pl = ob.plan_batches(t2, o2, id2, thr, used, table, vs, TRAIN["negative"])
    t1 = time.perf_counter()
    ob.skipgram_batch(syn0, syn1, et, table, vs, pl["sen"], pl["sent_start"], 0, len(pl["sent_start"]) - 1,
                      TRAIN["window"], dim, TRAIN["negative"], 0.025)
    t_train = time.perf_counter() - t1
    walk_rate = len(tok) / t_walk
    train_rate = int(o2[-1]) / t_train
    return {"value": 1.0 / (1.0 / walk_rate + 1.0 / train_rate), "unit": "tokens/s", "cores": 1, "kind": "port",
            "sample": f"oracle walk of {n_walkers} walkers on the C5 CSR copied out of HBM ({len(tok)} tokens, "
                      f"{t_walk:.1f}s) + skip-gram over {n_sent} sentences ({int(o2[-1])} tokens, {t_train:.1f}s), "
                      f"1 thread",
            "walk_steps_per_s": walk_rate, "sgns_words_per_s": train_rate}


def new_context(fb, g, form, device, seed, model, autotune=1):
    V = g["v_num"]
    f = fb.Felog(v_num=V, device=device, seed=seed, autotune=autotune, **{**TRAIN, **FORMS[form]})
    f.load_graph(g["edges"], V)
    f.init_model()
    if FORMS[form]["budget_mode"] == 1:
        f.mlp_set_state(model)
    return f


def quality(f, g, pairs):
    """Link scores of the context's embedding (tests/ref_tables.py, FP64):
    held-out AUC (held-out edges against the split's uniform non-edges, raw and
    mean-centred cosine) and fit AUC (training edges against degree-matched
    non-edges, mean-centred cosine and the skip-gram score)."""
    import ref_tables as rt
    s0, s1 = rt.tables_by_vertex(f)
    held = rt.link_aucs(s0, s1, g)
    fit = rt.fit_aucs(s0, s1, pairs)
    return {"auc": held["cosine"], "auc_centered": held["cosine_centered"],
            "fit_auc": fit["cosine_centered"], "fit_auc_sgns": fit["sgns"]}


def reference_quality(g, pairs):
    """The same scores of the reference's own run (oracle/_ref/ref_pipeline:
    its walk engine and CUDA skip_gram_kernel) after the same two rounds."""
    import ref_tables as rt
    if not os.path.exists(rt.REF_PIPELINE):
        return {"unavailable": "oracle/_ref/ref_pipeline was not built"}
    t0 = time.perf_counter()
    s0, s1 = rt.run_reference(g["edges"], g["v_num"], TRAIN["min_rounds"])
    held = rt.link_aucs(s0, s1, g)
    fit = rt.fit_aucs(s0, s1, pairs)
    return {"rounds": TRAIN["min_rounds"], "auc": held["cosine"], "auc_centered": held["cosine_centered"],
            "fit_auc": fit["cosine_centered"], "fit_auc_sgns": fit["sgns"],
            "wall_s": time.perf_counter() - t0}


def walk_layout(f):
    wb = f.walk_entries()
    if wb:
        return {"walker_entries_bytes": wb, "dram_sectors_per_step": 1,
                "what": "walker entries (16 B: neighbour, data, its first entry and degree): one dependent random "
                        "read per step; bytes_per_step stays the sector model of the reference's CSR"}
    return {"walker_entries_bytes": 0, "dram_sectors_per_step": 2, "what": "plain CSR: two dependent random reads"}


FORM_SET = ("plain-fp32", "learned-bf16", "learned-bf16-window", "learned-bf16-tile", "learned-fp32-tile")


def compare_forms(fb, g, device, model):
    """Plain FP32 and learned-budget BF16, each run end to end (felog_run: walk,
    train and budget check until the stop-all rule) on the same graph and walk
    seed; job time is the device time of the second of two runs in one context
    (the first one pays for allocations)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import ref_tables as rt
    pairs = rt.fit_pairs(g)
    out = {}
    for form in FORM_SET:
        f = new_context(fb, g, form, device, 77, model)
        f.run()         # untimed first run: device allocations and first-use module loading
        f.init_model()  # the timed run starts over from InitNet with the same walk seed
        t0 = time.perf_counter()
        rs = f.run()
        wall = time.perf_counter() - t0
        out[form] = {"rounds": rs["rounds"], "walk_tokens": rs["walk_tokens"], "train_words": rs["train_words"],
                     "job_ms": rs["total_ms"], "wall_ms": wall * 1e3,
                     "tokens_per_s": rs["walk_tokens"] / (rs["total_ms"] * 1e-3),
                     "budget": {k: rs[k] for k in ("evaluated", "predicted", "audited", "overruled")}}
        out[form].update(quality(f, g, pairs))
        f.close()
    p = out["plain-fp32"]
    for form in FORM_SET[1:]:
        out[form]["end_to_end_speedup_vs_plain_fp32"] = p["job_ms"] / out[form]["job_ms"]
        for k in ("auc", "auc_centered", "fit_auc", "fit_auc_sgns"):
            out[form][k + "_delta_vs_plain_fp32"] = out[form][k] - p[k]
    out["reference"] = reference_quality(g, pairs)
    if "fit_auc" in out["reference"]:
        for k in ("auc", "fit_auc", "fit_auc_sgns"):
            p[k + "_delta_vs_reference"] = p[k] - out["reference"][k]
    out["scores"] = ("auc: held-out edges vs the split's uniform non-edges, raw cosine; fit_auc: training edges vs "
                     "degree-matched non-edges, mean-centred cosine (the score the 0.005 bar applies to); "
                     "fit_auc_sgns: the same pairs by syn0[u].syn1[v] (symmetrised)")
    return out


def bench_mine(args):
    import felog_b200 as fb
    world, rank, local, pg = dist_setup(args)
    cfg = CONFIGS[args.config]
    g = make_graph(cfg)
    V = g["v_num"]
    form = args.form
    prec = "bf16" if FORMS[form]["precision"] else "fp32"
    model = np.load(args.budget_model) if FORMS[form]["budget_mode"] or not args.no_forms else None
    f = new_context(fb, g, form, local, 1000 + rank, model, autotune=0 if args.no_autotune else 1)
    keys = ("tokens", "words", "pairs", "walk_ms", "train_ms", "plan_ms", "budget_ms", "rounds")

    def job(acc, timed=False):
        """One whole job: InitNet, then walk / train / budget-check rounds until
        the stop-all rule (felog_run).  timed: the device time of the rounds
        (InitNet, the vocabulary and the unigram table excluded) is added to
        acc["ms"]."""
        f.init_model()
        if timed:
            f.timer_mark(0)
        rs = f.run()
        if timed:
            f.timer_mark(1)
            acc["ms"] = acc.get("ms", 0.0) + f.timer_elapsed()
        for k, v in (("tokens", rs["walk_tokens"]), ("words", rs["train_words"]), ("pairs", rs["pairs"]),
                     ("walk_ms", rs["walk_ms"]), ("train_ms", rs["train_ms"] - rs["plan_ms"]),
                     ("plan_ms", rs["plan_ms"]), ("budget_ms", rs["budget_ms"]), ("rounds", rs["rounds"])):
            acc[k] = acc.get(k, 0.0) + v

    warm = {}
    for _ in range(args.warmup):
        job(warm)
    log(f"warmup done: {warm}")
    # ---- device-timed region: whole jobs, inputs resident in HBM
    if pg is not None:
        pg.barrier()
    cnt = {}
    launches0 = f.kernel_launches()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            job(cnt, timed=True)
    ms = cnt["ms"]
    launches = f.kernel_launches() - launches0
    lost = None
    if prec == "bf16" and FORMS[form]["reuse_neg"] == 0:
        # one more job with the lost-update count on (outside the timed region)
        f.init_model()
        f.count_lost_updates(True)
        rs_l = f.run()
        nu, nl = f.lost_updates()
        f.count_lost_updates(False)
        lost = {"bf16_row_updates": nu, "overwritten": nl, "share": nl / max(nu, 1), "rounds": rs_l["rounds"],
                "what": "BF16-row stores of one job that overwrote another warp's concurrent update of the row "
                        "(Hogwild plain stores; FP32 master rows add atomically)"}
    # the walker against the attainable rate of its own access pattern: the
    # memory skeleton of the last round (same walkers and lengths, dependent
    # uniform-neighbour gathers, no arithmetic), timed outside the timed region
    ceil_ms, ceil_tok = f.walk_ceiling()
    # walk lengths of the last round and walks per vertex of the last job
    lens = np.diff(f.corpus()[1].astype(np.int64))
    wpv = f.budget_labels()[0].astype(np.int64)

    def summary(x):
        return {"mean": float(x.mean()), "min": int(x.min()), "p10": float(np.percentile(x, 10)),
                "p50": float(np.percentile(x, 50)), "p90": float(np.percentile(x, 90)),
                "p99": float(np.percentile(x, 99)), "max": int(x.max())}

    walks = {"length_last_round": summary(lens), "walks_per_vertex_last_job": summary(wpv),
             "what": "tokens per walk of the last round; walks a vertex made in the last job before a "
                     "convergence check stopped it (budget labels, 2..10)"}
    ms_max = max_over_ranks(pg, ms)
    tokens_all = sum_over_ranks(pg, cnt["tokens"])
    value = tokens_all / (ms_max * 1e-3)
    # ---- end to end through the C ABI with host buffers: per job the edge
    # list goes up from pinned memory (CSR build included) and the trained
    # syn0 comes back to pinned memory
    import torch
    vs = f.vocab()[2]
    edges_h = torch.from_numpy(g["edges"].view(np.uint8)).pin_memory()
    emb_h = torch.empty(vs * 128, dtype=torch.float32).pin_memory()
    edges_pinned = np.frombuffer(edges_h.numpy().data, dtype=g["edges"].dtype)
    e2e = {}

    def e2e_job(acc):
        f.load_graph(edges_pinned, V)
        job(acc)
        f.embeddings_into(emb_h.data_ptr(), vs * 128)

    e2e_job({})
    if pg is not None:
        pg.barrier()
    f.timer_mark(0)
    for _ in range(args.steps):
        e2e_job(e2e)
    f.timer_mark(1)
    e2e_ms = max_over_ranks(pg, f.timer_elapsed())
    e2e_value = sum_over_ranks(pg, e2e["tokens"]) / (e2e_ms * 1e-3)
    last_tok, last_ms = cnt["tokens"], cnt["walk_ms"]
    peak, peak_kind = measured_peaks()
    # dominant kernel: the skip-gram pass
    row_bytes = SGNS_BYTES_PER_PAIR[prec] // 14
    if FORMS[form]["reuse_neg"] in (2, 4):
        # center tiles: per center its contexts and the K + 1 targets, each read and written once
        sg_bytes = 2 * row_bytes * (cnt["pairs"] + (TRAIN["negative"] + 1) * cnt["words"])  # words: centers before subsampling (an upper bound)
        sg_kernel = (f"k_sgns_reuse_tile<128, 5, Rows{prec.upper()}" +
                     (", true>" if FORMS[form]["reuse_neg"] == 4 else ">"))
    elif FORMS[form]["reuse_neg"] == 3:
        sg_bytes = 2 * row_bytes * (cnt["pairs"] + (TRAIN["negative"] + 1) * cnt["words"])  # words: centers before subsampling (an upper bound)
        sg_kernel = "k_sgns_tile_umma<128, 5>"
    else:
        # per pair: each referenced row (context + trained targets) read and
        # written once; in the BF16 form the top-1% rows are FP32 master rows,
        # counted at their FP32 size (shares from the last trained chunk)
        mix_pairs, mix_refs, mix_hot = f.pair_row_mix()
        refs_per_pair = mix_refs / mix_pairs
        hot_share = mix_hot / mix_refs
        per_ref = 2 * (512 * hot_share + 256 * (1 - hot_share)) if prec == "bf16" else 2 * 512
        sg_bytes_per_pair = refs_per_pair * per_ref
        sg_bytes = cnt["pairs"] * sg_bytes_per_pair
        sg_kernel = f"k_sgns_train_pairs<128, 5, Rows{prec.upper()}>"
    sg_achieved = sg_bytes / (cnt["train_ms"] * 1e-3) / 1e9
    walk_achieved = cnt["tokens"] * WALK_BYTES_PER_STEP / (cnt["walk_ms"] * 1e-3) / 1e9
    out = {
        "metric": METRIC,
        "value": value,
        "unit": "tokens/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": ("f32 tables" if prec == "fp32" else "bf16 tables (f32 master rows for the top 1%), f32 arithmetic")
                 + ", f64 walk statistics",
        "data": "synthetic (seeded R-MAT, see config)",
        "config": {"workload": cfg["workload"].replace("plain FP32", form), "form": form,
                   "v_num": V, "train_edges": int(len(g["edges"])),
                   "dim": 128, "window": 10, "negative": 5, "sample": 1e-3, "min_L": 20, "min_R": 2,
                   "skip_gram": True, "reuse_neg": FORMS[form]["reuse_neg"], "precision": prec,
                   "l2": "inputs larger than L2 (CSR + tables > 126 MB)",
                   "step": "one whole job: the rounds (walk, plan, pair stream, train, budget check from min_R "
                           "on) from InitNet until the stop-all rule; the timed region holds the rounds (InitNet, "
                           "vocabulary and unigram table are set up untimed before each job; e2e includes them)",
                   "rounds_per_step": cnt["rounds"] / args.steps,
                   "parallelism": f"replicas x{world}"},
        "walk_steps_per_s": cnt["tokens"] / (cnt["walk_ms"] * 1e-3),
        "sgns_words_per_s": cnt["words"] / ((cnt["train_ms"] + cnt["plan_ms"]) * 1e-3),
        "phase_ms_per_step": {k: cnt[k] / args.steps for k in ("walk_ms", "plan_ms", "train_ms", "budget_ms")},
        "tokens_per_step": cnt["tokens"] / args.steps,
        "pairs_per_step": cnt["pairs"] / args.steps,
        "roofline": {"kernel": sg_kernel, "bound": "hbm",
                     "traffic": (DRAM_BYTES_PER_PAIR[prec] * min(cnt["pairs"] / cnt["rounds"], 2 ** 27)
                                 if FORMS[form]["reuse_neg"] == 0 else None),
                     "traffic_unit": "bytes per launch (ncu per-pair DRAM traffic x pairs per launch: a round's "
                                     "pairs, at most one 2^27-pair chunk)", "achieved": sg_achieved, "peak": peak,
                     "unit": "GB/s", "frac": sg_achieved / peak,
                     "algorithmic_bytes_per_pair": sg_bytes / max(cnt["pairs"], 1),
                     "row_refs_per_pair": refs_per_pair if FORMS[form]["reuse_neg"] in (0, 1) else None,
                     "master_row_share": hot_share if FORMS[form]["reuse_neg"] in (0, 1) else None,
                     "peak_source": peak_kind,
                     "walk_kernel": {"achieved": walk_achieved, "frac": walk_achieved / peak,
                                     "bytes_per_step": WALK_BYTES_PER_STEP,
                                     "layout": walk_layout(f),
                                     "gather_ceiling": {"steps_per_s": ceil_tok / (ceil_ms * 1e-3),
                                                        "walk_steps_per_s": last_tok / (last_ms * 1e-3),
                                                        "frac": (last_tok / last_ms) / (ceil_tok / ceil_ms),
                                                        "what": "felog_walk_ceiling: memory skeleton of the "
                                                                "last round on the same CSR (the walker's rate: "
                                                                "all timed rounds)"}}},
        "e2e": {"value": e2e_value, "unit": "tokens/s", "h2d_bytes_per_step": int(g["edges"].nbytes),
                "d2h_bytes_per_step": int(vs * 128 * 4), "ms_per_step": e2e_ms / args.steps,
                "tokens_per_step": e2e["tokens"] / args.steps,
                "what": "per step one whole job through the C ABI: the edge list from pinned host memory "
                        "(CSR build included), felog_run to the stop-all rule, syn0 back to pinned host memory"},
        "walks": walks,
        "bf16_lost_updates": lost,
        "gpu_launches": int(launches),
        "autotune": f.tuning_report(),
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_forms:
        out["forms"] = compare_forms(fb, g, local, model)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            out["cpu_baseline"] = cpu_baseline(g, cfg)
        except Exception as ex:  # reported, not fatal
            out["cpu_baseline"] = {"error": str(ex)}
    if rank == 0:
        print(json.dumps(out), flush=True)
    f.close()
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


def bench_streamed(args):
    """Streamed configuration (C5): one step = one piece of a round (walk the
    piece's walkers, plan and train on their corpus), inputs resident in HBM.
    e2e = one whole job through the C ABI (device generation from a parameter
    block, felog_run to the stop-all rule, syn0 copied to host memory);
    forms = plain FP32 and learned BF16 jobs on the same graph."""
    import felog_b200 as fb
    cfg = STREAMED[args.config]
    model = np.load(args.budget_model)
    piece = cfg["piece"]

    def context(form):
        f = fb.Felog(v_num=cfg["v_target"], device=0, seed=1000, autotune=0 if args.no_autotune else 1,
                     stream_walkers=piece, **{**TRAIN, **FORMS[form]})
        t0 = time.perf_counter()
        info = f.load_rmat(cfg["seed"], cfg["v_target"], cfg["e_target"], abcd=cfg["abcd"])
        gen_s = time.perf_counter() - t0
        f.init_model()
        if FORMS[form]["budget_mode"] == 1:
            f.mlp_set_state(model)
        return f, info, gen_s

    form = args.form
    prec = "bf16" if FORMS[form]["precision"] else "fp32"
    f, info, gen_s = context(form)
    log(f"graph: {info} generated and loaded in {gen_s:.1f}s")
    V = info["v_num"]
    state = {"round": 0, "first": 0, "na": None}

    def step(acc):
        ws, na = f.walk_piece(state["round"], state["first"], piece)
        ts = f.train_round(state["round"])
        state["first"] += piece
        if state["first"] >= na:
            state["round"] += 1
            state["first"] = 0
        for k, v in (("tokens", ws["n_tokens"]), ("words", ts["words"]), ("pairs", ts["pairs"]),
                     ("kept", ts["kept_words"]), ("walk_ms", ws["ms"]), ("train_ms", ts["ms_train"]),
                     ("plan_ms", ts["ms_plan"])):
            acc[k] = acc.get(k, 0.0) + v

    warm = {}
    for _ in range(args.warmup):
        step(warm)
    log(f"warmup done: {warm}")
    cnt = {}
    launches0 = f.kernel_launches()
    with ClockSampler(0) as clk:
        f.timer_mark(0)
        for _ in range(args.steps):
            step(cnt)
        f.timer_mark(1)
        ms = f.timer_elapsed()
    launches = f.kernel_launches() - launches0
    mix_pairs, mix_refs, mix_hot = f.pair_row_mix()
    refs_per_pair = mix_refs / mix_pairs
    hot_share = mix_hot / mix_refs
    per_ref = 2 * (512 * hot_share + 256 * (1 - hot_share)) if prec == "bf16" else 2 * 512
    peak, peak_kind = measured_peaks()
    sg_achieved = cnt["pairs"] * refs_per_pair * per_ref / (cnt["train_ms"] * 1e-3) / 1e9
    walk_achieved = cnt["tokens"] * WALK_BYTES_PER_STEP / (cnt["walk_ms"] * 1e-3) / 1e9
    # ---- e2e: a whole job through the C ABI, host buffers (syn0 back to host memory)
    vs = f.vocab()[2]
    emb = np.empty(vs * TRAIN["size"], np.float32)
    f.init_model()
    if FORMS[form]["budget_mode"] == 1:
        f.mlp_set_state(model)
    t0 = time.perf_counter()
    job = f.run()
    f.embeddings_into(emb.ctypes.data, emb.size)
    e2e_s = time.perf_counter() - t0
    del emb
    cpu = None
    if not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline_resident(f, V)
        except Exception as ex:  # reported, not fatal
            cpu = {"error": str(ex)}
    layout = walk_layout(f)
    f.close()
    out = {
        "metric": METRIC, "value": cnt["tokens"] / (ms * 1e-3), "unit": "tokens/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": ("f32 tables" if prec == "fp32" else "bf16 tables (f32 master rows for the top 1%), f32 arithmetic")
                 + ", f64 walk statistics",
        "data": "synthetic (seeded R-MAT generated on the device, see config)",
        "config": {"workload": cfg["workload"].replace("learned-bf16", form), "form": form, "v_num": V,
                   "undirected_edges": info["n_edges"], "max_degree": info["max_degree"], "dim": 128, "window": 10,
                   "negative": 5, "sample": 1e-3, "min_L": 20, "min_R": 2, "skip_gram": True, "precision": prec,
                   "step": f"one piece of {piece} walkers of a round: walk, plan, pair stream, train",
                   "unigram_table_slots": f"2^{max(8 * vs - 1, 1).bit_length()} (the power of two >= 8 per word; "
                                          "the reference's 1e8 below 12.5M words)",
                   "l2": "inputs larger than L2", "parallelism": "replicas x1", "graph_gen_s": gen_s},
        "walk_steps_per_s": cnt["tokens"] / (cnt["walk_ms"] * 1e-3),
        "sgns_words_per_s": cnt["words"] / ((cnt["train_ms"] + cnt["plan_ms"]) * 1e-3),
        "phase_ms_per_step": {k: cnt[k] / args.steps for k in ("walk_ms", "plan_ms", "train_ms")},
        "tokens_per_step": cnt["tokens"] / args.steps, "pairs_per_step": cnt["pairs"] / args.steps,
        "roofline": {"kernel": f"k_sgns_train_pairs<128, 5, Rows{prec.upper()}>", "bound": "hbm",
                     "traffic": DRAM_BYTES_PER_PAIR[prec] * min(cnt["pairs"] / args.steps, 2 ** 27),
                     "traffic_unit": "bytes per launch (ncu per-pair DRAM traffic of the profiling case x pairs "
                                     "per launch: one 2^27-pair chunk)",
                     "achieved": sg_achieved, "peak": peak, "unit": "GB/s", "frac": sg_achieved / peak,
                     "algorithmic_bytes_per_pair": refs_per_pair * per_ref, "row_refs_per_pair": refs_per_pair,
                     "master_row_share": hot_share, "peak_source": peak_kind,
                     "walk_kernel": {"achieved": walk_achieved, "frac": walk_achieved / peak,
                                     "bytes_per_step": WALK_BYTES_PER_STEP, "layout": layout}},
        "e2e": {"value": job["walk_tokens"] / e2e_s, "unit": "tokens/s", "h2d_bytes_per_step": 120,
                "d2h_bytes_per_step": int(vs * TRAIN["size"] * 4),
                "what": "one whole job per step: device generation from the parameter block, felog_run to the "
                        "stop-all rule, syn0 copied to host memory", "rounds": job["rounds"], "job_s": e2e_s},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if cpu is not None:
        out["cpu_baseline"] = cpu
    if not args.no_forms:
        forms = {}
        for fm in ("plain-fp32", "learned-bf16"):
            g2, _, gs = context(fm)
            t0 = time.perf_counter()
            rs = g2.run()
            wall = time.perf_counter() - t0
            forms[fm] = {"rounds": rs["rounds"], "walk_tokens": rs["walk_tokens"], "train_words": rs["train_words"],
                         "job_ms": rs["total_ms"], "wall_ms": wall * 1e3,
                         "tokens_per_s": rs["walk_tokens"] / (rs["total_ms"] * 1e-3),
                         "budget": {k: rs[k] for k in ("evaluated", "predicted", "audited", "overruled")}}
            g2.close()
        forms["learned-bf16"]["end_to_end_speedup_vs_plain_fp32"] = (forms["plain-fp32"]["job_ms"]
                                                                     / forms["learned-bf16"]["job_ms"])
        out["forms"] = forms
    print(json.dumps(out), flush=True)


def bench_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_pipeline")
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_pipeline was not built"}))
        return
    cfg = CONFIGS[args.config]
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        gp = os.path.join(td, "g.bin")
        # the graph comes from a child process, so this process maps none of
        # the repository's libraries
        gen = subprocess.run([sys.executable, os.path.abspath(__file__), "--config", args.config,
                              "--write-graph", gp], capture_output=True, text=True)
        if gen.returncode != 0:
            print(json.dumps({"impl": "reference", "unavailable": f"graph generation failed: {gen.stderr[-200:]}"}))
            return
        g = json.loads(gen.stdout.strip().splitlines()[-1])
        cmd = [exe, gp, str(g["v_num"]), str(args.warmup), str(args.steps), str(args.ref_walkers)]
        log("reference:", " ".join(cmd))
        res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        print(json.dumps({"impl": "reference", "unavailable": f"ref_pipeline exited {res.returncode}: "
                                                              f"{res.stderr.strip()[-200:]}"}))
        return
    # the reference's progress output ends in carriage returns, so the result
    # may share a line with it
    lines = re.findall(r'\{"tokens".*?\}', res.stdout)
    if not lines:
        print(json.dumps({"impl": "reference", "unavailable": "ref_pipeline printed no result line: "
                                                              f"{res.stdout.strip()[-200:]}"}))
        return
    d = json.loads(lines[-1])
    value = d["tokens"] / d["seconds"]
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "tokens/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": d["seconds"] * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded R-MAT, see config)",
        "config": {"workload": cfg["workload"], "v_num": g["v_num"], "walkers_per_step": d["walkers"]},
        "walk_steps_per_s": d["walk_tokens"] / d["walk_seconds"],
        "sgns_words_per_s": d["train_words"] / d["train_seconds"],
        "cpu_baseline": {"value": value, "unit": "tokens/s", "cores": d["threads"], "kind": "reference",
                         "sample": f"{d['walkers']} walkers per round, {args.steps} rounds; reference walk "
                                   f"engine on {d['threads']} host threads + reference skip_gram_kernel"},
        "e2e": {"value": value, "unit": "tokens/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def bench_gcn(args):
    """Common neighbours per edge (the reference's offline gcn tool) on the
    configuration's training edges: device time of felog_common_neighbours
    (warm-up calls, then the best of the timed calls), the same call end to end
    with host arrays, and the oracle (the tool restated in C, one thread) on
    the same edges as the CPU baseline.  One JSON line."""
    import felog_b200 as fb
    cfg = CONFIGS[args.config]
    g = make_graph(cfg)
    V = g["v_num"]
    src = np.ascontiguousarray(g["edges"]["src"], np.uint32)
    dst = np.ascontiguousarray(g["edges"]["dst"], np.uint32)
    n = len(src)
    f = fb.Felog(v_num=V, seed=1)
    for _ in range(args.warmup):
        cn, _ = f.common_neighbours(src, dst, V, True)
    dev, wall = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        cn, ms = f.common_neighbours(src, dst, V, True)
        wall.append(time.perf_counter() - t0)
        dev.append(ms)
    launches = f.kernel_launches()
    f.close()
    out = {"metric": "common-neighbour edges/s (gcn tool, undirected)", "value": n / (min(dev) * 1e-3),
           "unit": "edges/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": min(dev), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "u32 ids, i32 counts", "data": "synthetic (seeded R-MAT, see config)",
           "config": {"workload": f"gcn tool on the training edges of the seed-{cfg['seed']} R-MAT "
                                  f"({cfg['v_target']:,} vertex ids / {cfg['e_target']:,} undirected edges)",
                      "v_num": V, "edges": n,
                      "sum_cn": int(cn.astype(np.int64).sum()), "max_degree": g["info"]["max_degree"]},
           "e2e": {"value": n / min(wall), "unit": "edges/s", "h2d_bytes_per_step": 8 * n,
                   "d2h_bytes_per_step": 4 * n}, "gpu_launches_total": int(launches)}
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_binding as ob
        t0 = time.perf_counter()
        ref = ob.common_neighbours(src, dst, V, True)
        t = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": n / t, "unit": "edges/s", "cores": 1, "kind": "port",
                               "sample": f"oracle on all {n} edges, {t:.1f}s, 1 thread"}
        out["parity_vs_oracle"] = bool(np.array_equal(ref, cn))
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--config", default="c2", choices=sorted(CONFIGS) + sorted(STREAMED))
    ap.add_argument("--ref-walkers", type=int, default=0,
                    help="walkers of the reference arm (0: one per vertex; the reference asserts every vertex is visited)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--form", default="learned-bf16", choices=sorted(FORMS))
    ap.add_argument("--budget-model", default=BUDGET_MODEL)
    ap.add_argument("--no-forms", action="store_true", help="skip the end-to-end plain vs learned comparison")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default launch shape (profiling: a tuner timed under ncu is distorted)")
    ap.add_argument("--workload", default="walk-sgns", choices=["walk-sgns", "gcn"],
                    help="gcn: the offline common-neighbour tool instead of the walk + SGNS rounds")
    ap.add_argument("--write-graph", default=None, help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.write_graph:
        # helper of the reference arm: the configuration's training edges as a
        # 12-byte binary edge file, and its vertex count on stdout
        g = make_graph(CONFIGS[args.config])
        g["edges"].tofile(args.write_graph)
        print(json.dumps({"v_num": g["v_num"]}))
        return
    if args.workload == "gcn":
        bench_gcn(args)
    elif args.config in STREAMED:
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference's CPU walk engine needs about 15 min "
                              "per round at 111M vertices (2.6 M steps/s on 16 threads, 2.4 G steps per round) and "
                              "its graph load a host edge list of 19 GB; bench it at c2"}))
        else:
            bench_streamed(args)
    elif args.impl == "reference":
        bench_reference(args)
    else:
        bench_mine(args)


if __name__ == "__main__":
    main()
