#!/usr/bin/env python
"""Benchmark of the one-GPU collapsed-Gibbs LDA iteration.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one full iteration (sample -> log-likelihood -> count rebuild) over
the whole synthetic corpus.  The default workload is the 60M-token one
(V=100k, D=300k, lognormal(5, 0.8) lengths, K=1024, alpha=50/1024, beta=0.01),
generated from a seed; its working set (doc ids, topics, doc-reverse index,
theta) is several times the 126 MB L2, so no flush is needed between steps.

--impl ours (default): W untimed iterations, then K iterations timed with CUDA
events on the sampler's stream, bracketed by a barrier and a synchronize; the
max over ranks is reported.  Under torchrun each rank runs an independent
replica (its own seed): the path has no exchange step on one GPU, so the
scaling is weak and the value is the sum of tokens over ranks / max time.
--impl reference: the reference's own CUDA build (oracle/_ref/culda, compiled
from its sources for sm_100a) on the same corpus files, timed by its own
per-iteration clock; rank 0 only.
Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "tokens/sec on 1 B200 (plain CGS)"
UNIT = "tokens/s"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[tuple[float, str]] = []
        self._t = None
        self.t0 = self.t1 = None

    def start(self):
        """Starts sampling and returns once the first sample has arrived."""
        exe = shutil.which("nvidia-smi")
        if not exe:
            return
        self.proc = subprocess.Popen([exe, f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                      "-lms", "50", "-i", str(self.device)], stdout=subprocess.PIPE,
                                     stderr=subprocess.DEVNULL, text=True)
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()
        deadline = time.time() + 10
        while not self.lines and time.time() < deadline and self.proc.poll() is None:
            time.sleep(0.01)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()
        time.sleep(0.12)  # let the sample that covers the end arrive

    def stop(self) -> dict | None:
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        lines = self.lines
        if self.t0 is not None and self.t1 is not None:
            inside = [x for x in lines if self.t0 <= x[0] <= self.t1 + 0.1]
            if not inside:  # region shorter than the sampling period: nearest samples
                mid = 0.5 * (self.t0 + self.t1)
                inside = sorted(lines, key=lambda x: abs(x[0] - mid))[:2]
            lines = inside
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for _, line in lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------- distributed
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def allreduce_max(pg, x: float) -> float:
    if pg is None:
        return x
    import torch

    dev = "cuda" if torch.cuda.is_available() and pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, tokens_per_rank: int, steps: int, max_seconds: float) -> float:
    """Tokens per second of the whole job: every rank samples its own replica
    of tokens_per_rank tokens for `steps` iterations; the slowest rank's device
    time bounds the job (weak scaling)."""
    return world * tokens_per_rank * steps / max_seconds


def barrier(pg):
    if pg is not None:
        pg.barrier()


def cuda_sync():
    try:
        import torch

        if torch.cuda.is_available():
            torch.cuda.synchronize()
    except Exception:
        pass


def measured_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def ncu_traffic(workload: str):
    """Sampler DRAM bytes per launch from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "sample_kernel_traffic.json"
    if not p.exists():
        return None
    try:
        d = json.loads(p.read_text()).get(workload)
        return int(d["dram_bytes_per_launch"]) if d else None
    except Exception:
        return None


def run_flags(args) -> int:
    import culda_cgs_b200 as cb

    return (cb.CULDA_FLAG_AUTOTUNE if args.autotune else 0) | (cb.CULDA_FLAG_NO_REORDER if args.no_reorder else 0)


def workload(args, seed: int):
    """The named workload with the run's seed; --k replaces K (and alpha = 50/K)."""
    from dataclasses import replace

    from culda_cgs_b200.configs import WORKLOADS

    wl = WORKLOADS[args.workload].with_seed(seed)
    if args.k:
        wl = replace(wl, k=args.k, alpha=50.0 / args.k, name=f"{wl.name.split(' K=')[0]} K={args.k}")
    return wl


# ----------------------------------------------- learned form and fold-in
def measure_learned(args, wl, corpus, device) -> dict:
    """Wall-clock to the plain chain's iteration-100 log-likelihood, plain CGS
    against several schedules of the learned form.  Every state's
    log-likelihood is the per-token value of culda_sample_snapshot (evaluation
    passes are not timed); iterations are timed with CUDA events, the
    host-driven steps (accumulation, training, proposal tables, warm start) by
    the wall clock.

    Schedules (each stops at the target or after its iteration budget):
      mh2        plain 1-40 (states 21-40 accumulated), encoder initialised
                 from the word profiles and trained, then MH iterations mixing
                 the doc and encoder proposals 1:1, 2 steps per token;
      mh8        the same trained state, 8 MH steps per token;
      interleave the same trained state, then a plain sweep and a 2-step MH
                 iteration in turn;
      restart    plain 1-10 (states 6-10 accumulated), the encoder trained 2
                 epochs, every topic redrawn from q_d(k) * phihat_wk (warm
                 start), then plain sweeps.
    The first three share the prefix (plain 1-40 and the training): its time
    is counted in each, and each starts from the prefix's topics."""
    import culda_cgs_b200 as cb

    target_it, first, window, epochs = 100, 20, 20, args.learned_epochs
    with cb.LDA(corpus, wl.k, wl.alpha, wl.beta, seed=args.seed, device=device) as m:
        st = m.iterate(target_it)
        t_plain = sum(x["seconds"] for x in st)
        target = m.sample_snapshot(1 << 30)[1]
        plain_curve = [(i + 1, round(sum(x["seconds"] for x in st[:i + 1]), 4)) for i in (9, 39, 59, 79, 99)]
    out = {"target": "log-likelihood per token of the plain chain's state after iteration 100",
           "target_loglik": round(target, 6), "plain_seconds": round(t_plain, 4), "plain_seconds_at": plain_curve}

    def run(m, t, it, step, max_it, name):
        curve, reached, secs, acc = [], None, [], []
        while it < max_it:
            sts = step(m)
            it += len(sts)
            t += sum(x["seconds"] for x in sts)
            secs += [x["seconds"] for x in sts]
            acc += [x["accept_rate"] for x in sts if x["accept_rate"] > 0]
            ll = m.sample_snapshot(1 << 29)[1]
            curve.append((it, round(t, 4), round(ll, 6)))
            if ll >= target:
                reached = t
                break
        return {"name": name, "reached": reached is not None,
                "seconds_to_target": round(reached, 4) if reached else None,
                "ratio_to_plain": round(reached / t_plain, 4) if reached else None,
                "ms_per_iteration": round(1e3 * statistics.mean(secs), 4) if secs else None,
                "mh_accept_rate": round(statistics.mean(acc), 4) if acc else None,
                "last_loglik": curve[-1][2] if curve else None, "curve": curve[::max(1, len(curve) // 8)]}

    schedules = []
    with cb.LDA(corpus, wl.k, wl.alpha, wl.beta, seed=args.seed, device=device) as m, \
            cb.Encoder(corpus.num_words, wl.k, args.learned_batch, seed=1, device=device) as enc:
        t = sum(x["seconds"] for x in m.iterate(first))
        for _ in range(window):
            t += m.iterate(1)[0]["seconds"]
            t0 = time.perf_counter()
            m.accumulate_theta()
            t += time.perf_counter() - t0
        t0 = time.perf_counter()
        m.init_encoder(enc, seed=3)
        losses = [m.train_encoder(enc, 1, seed=e) for e in range(epochs)]
        m.set_proposal(enc, mix=0.05)
        t_train = time.perf_counter() - t0
        t += t_train
        z_prefix, it_prefix = m.topics(), m.next_iteration
        out.update({"prefix": f"plain 1-{first + window} (states {first + 1}-{first + window} accumulated), "
                              f"encoder trained {epochs} epochs (batch {args.learned_batch})",
                    "prefix_seconds": round(t, 4), "encoder_train_seconds": round(t_train, 4),
                    "encoder_loss": [round(losses[0], 4), round(losses[-1], 4)]})
        budget = first + window + 60
        for name, step in (("mh2", lambda mm: mm.iterate_mh(5, steps=2)),
                           ("mh8", lambda mm: mm.iterate_mh(5, steps=8)),
                           ("interleave", lambda mm: mm.iterate(1) + mm.iterate_mh(1, steps=2))):
            m.set_topics(z_prefix)
            m.set_iteration(it_prefix)
            schedules.append(run(m, t, first + window, step, budget, name))
    with cb.LDA(corpus, wl.k, wl.alpha, wl.beta, seed=args.seed, device=device) as m, \
            cb.Encoder(corpus.num_words, wl.k, args.learned_batch, seed=1, device=device) as enc:
        t = sum(x["seconds"] for x in m.iterate(5))
        for _ in range(5):
            t += m.iterate(1)[0]["seconds"]
            t0 = time.perf_counter()
            m.accumulate_theta()
            t += time.perf_counter() - t0
        t0 = time.perf_counter()
        m.init_encoder(enc, seed=3)
        for e in range(2):
            m.train_encoder(enc, 1, seed=e)
        m.set_proposal(enc, mix=0.05)
        m.warm_start()
        t += time.perf_counter() - t0
        schedules.append(run(m, t, 10, lambda mm: mm.iterate(5), target_it + 20, "restart"))
    best = min((x for x in schedules if x["reached"]), key=lambda x: x["seconds_to_target"], default=None)
    out.update({
        "schedules": schedules,
        "best_schedule": best["name"] if best else None,
        "learned_seconds_to_target": best["seconds_to_target"] if best else None,
        "reached": best is not None,
        "ratio_learned_to_plain": best["ratio_to_plain"] if best else None,
        "mh_ms_per_iteration": schedules[0]["ms_per_iteration"], "mh_accept_rate": schedules[0]["mh_accept_rate"]})
    return out


def measure_foldin(args, device) -> dict:
    """Fold-in of 100k new documents (the SMALL generator, same vocabulary)
    against the frozen counts of a model trained 50 iterations on 10k docs:
    held-out log-likelihood per token per sweep from random initial topics and
    from the encoder's warm start, and held-out docs per second per sweep."""
    import numpy as np

    import culda_cgs_b200 as cb
    from culda_cgs_b200.configs import FOLDIN, FOLDIN_TRAIN_DOCS

    wl = FOLDIN.with_seed(args.seed)
    c = cb.Corpus.generate(wl.gen)
    train = c.split_docs(np.arange(FOLDIN_TRAIN_DOCS))
    held = c.split_docs(np.arange(FOLDIN_TRAIN_DOCS, c.num_docs))
    sweeps = (1, 2, 5, 10, 20, 50)
    out = {"workload": wl.name, "train_docs": train.num_docs, "train_tokens": train.num_tokens,
           "held_docs": held.num_docs, "held_tokens": held.num_tokens}
    with cb.LDA(train, wl.k, wl.alpha, wl.beta, seed=args.seed, device=device) as m, \
            cb.Encoder(c.num_words, wl.k, 512, seed=1, device=device) as enc:
        m.iterate(30)
        for _ in range(20):
            m.iterate(1)
            m.accumulate_theta()
        phi, nk = m.phi()
        t0 = time.perf_counter()
        m.init_encoder(enc, seed=3)
        m.train_encoder(enc, 20, seed=1)
        out["encoder_train_seconds"] = round(time.perf_counter() - t0, 4)
        for mode in ("random", "encoder"):
            with cb.LDA(held, wl.k, wl.alpha, wl.beta, seed=args.seed + 1, device=device) as f:
                f.set_frozen_phi(phi, nk)
                if mode == "encoder":
                    t0 = time.perf_counter()
                    f.set_proposal(enc, mix=0.05)
                    f.warm_start()
                    out["warm_start_seconds"] = round(time.perf_counter() - t0, 4)
                st = f.iterate(max(sweeps))
                out[mode] = {f"sweep_{s}": round(st[s - 1]["loglik"], 6) for s in sweeps}
                out[mode + "_docs_per_sec"] = round(held.num_docs / statistics.mean(x["seconds"] for x in st), 1)
    out["loglik"] = "held-out per-token log-likelihood of the state before each sweep (FP64 sum of FP32 terms)"
    return out


def common_config(wl, num_tokens: int, num_docs: int, num_words: int, seed: int, world: int) -> dict:
    """The `config` object both arms print: the workload and its sizes only,
    so the two lines compare key for key."""
    return {"workload": wl.name, "num_tokens": int(num_tokens), "num_docs": int(num_docs),
            "num_words": int(num_words), "k": wl.k, "alpha": wl.alpha, "beta": wl.beta, "seed": seed,
            "l2": (f"inputs larger than L2 (doc ids, doc-reverse index, topics, uniforms and theta: at least "
                   f"{20 * num_tokens / 1e9:.2f} GB against 126 MB), no flush"
                   if 20 * num_tokens > 126e6 else "inputs smaller than L2 (small workload, not a headline line)"),
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}


def measure_uneven(args, device) -> dict:
    """The batched uneven workload (118M tokens, Pareto document lengths up
    to 50k, V = 1M) with the autotuner on: at K = 1024 the sampler variant and
    the theta rebuild's bin threshold it chose and the iteration times after
    tuning (iterations 4-8, CUDA events); then the rest of the configuration's
    K sweep (256, 2048, 4096, alpha = 50/K) on the same corpus, iterations 4-6
    each, as flat k<K>_* keys."""
    import culda_cgs_b200 as cb
    from culda_cgs_b200.configs import UNEVEN

    wl = UNEVEN.with_seed(args.seed)
    c = cb.Corpus.generate(wl.gen)

    def run(k, steps):
        with cb.LDA(c, k, 50.0 / k, wl.beta, seed=args.seed, device=device, flags=cb.CULDA_FLAG_AUTOTUNE) as m:
            m.iterate(3)  # the autotuner times the variants before iteration 3
            return m.iterate(steps), m.info()

    st, info = run(wl.k, 5)
    sec = [x["seconds"] for x in st]
    out = {"workload": wl.name, "num_tokens": c.num_tokens, "num_docs": c.num_docs, "k": wl.k,
           "autotuned": bool(info["tuned"]), "group_lanes": info["group_lanes"],
           "sample_blocks": info["sample_blocks"], "theta_min_len": info["theta_min_len"],
           "theta_long_docs": info["theta_long_docs"], "sampler_tune_ms": round(info["tune_ms"], 4),
           "rebuild_tune_ms": round(info["theta_tune_ms"], 4),
           "ms_per_iteration": round(1e3 * statistics.mean(sec), 4),
           "sample_ms": round(1e3 * statistics.mean(x["sample_seconds"] for x in st), 4),
           "rebuild_ms": round(1e3 * statistics.mean(x["rebuild_seconds"] for x in st), 4),
           "tokens_per_sec": round(c.num_tokens / statistics.mean(sec), 1)}
    for k in args.uneven_ks:
        st, info = run(k, 3)
        ms = 1e3 * statistics.mean(x["seconds"] for x in st)
        out[f"k{k}_ms_per_iteration"] = round(ms, 4)
        out[f"k{k}_sample_ms"] = round(1e3 * statistics.mean(x["sample_seconds"] for x in st), 4)
        out[f"k{k}_rebuild_ms"] = round(1e3 * statistics.mean(x["rebuild_seconds"] for x in st), 4)
        out[f"k{k}_tokens_per_sec"] = round(c.num_tokens / (ms / 1e3), 1)
        out[f"k{k}_variant"] = f"G={info['group_lanes']} blocks={info['sample_blocks']} " \
                               f"theta_min_len={info['theta_min_len']}"
    return out


# ------------------------------------------------------------------- ours
def run_ours(args, world, rank, local, pg):
    import ctypes as C

    import numpy as np

    import culda_cgs_b200 as cb
    from culda_cgs_b200.configs import WORKLOADS

    wl = workload(args, args.seed + rank)
    t0 = time.perf_counter()
    corpus = cb.Corpus.generate(wl.gen)
    log(f"[rank {rank}] corpus {wl.name}: D={corpus.num_docs} V={corpus.num_words} N={corpus.num_tokens} "
        f"generated in {time.perf_counter() - t0:.1f}s")
    N = corpus.num_tokens

    # ---- device-resident measurement
    m = cb.LDA(corpus, wl.k, wl.alpha, wl.beta, seed=args.seed + rank, device=local, group_lanes=args.group_lanes,
               item_tokens=args.item_tokens, sample_blocks=args.sample_blocks,
               flags=run_flags(args))
    info = m.info()
    log(f"[rank {rank}] info {info}")
    clocks = ClockSampler(local)
    clocks.start()
    warm = m.iterate(args.warmup) if args.warmup > 0 else []
    barrier(pg)
    cuda_sync()
    clocks.mark_start()
    stats = m.iterate(args.steps)
    info = m.info()  # the variant in use (the autotuner may have changed it during warm-up)
    cuda_sync()
    barrier(pg)
    clocks.mark_end()
    clk = clocks.stop()
    dev_seconds = sum(s["seconds"] for s in stats)
    max_seconds = allreduce_max(pg, dev_seconds)
    value = whole_job_rate(world, N, args.steps, max_seconds)
    for s in stats:
        log(f"[rank {rank}] iteration {s['iteration']:4d}: {s['seconds'] * 1e3:8.3f} ms "
            f"(sample {s['sample_seconds'] * 1e3:.3f} ms, rebuild {s['rebuild_seconds'] * 1e3:.3f} ms) "
            f"loglik {s['loglik']:.6f}  {s['tokens_per_sec'] / 1e6:.1f} M tokens/s")

    # ---- roofline of the sampler: algorithmic bytes per launch / event time
    prev = ([warm[-1]] if warm else []) + stats[:-1]
    if len(prev) < len(stats):  # no warm-up: the first sampler walked the initial rows
        prev = [stats[0]] + prev
    sample_bytes = [16 * N + 4 * p["token_nnz"] for p in prev]
    # each array once: doc ids, topics in and out, uniforms, theta entries, row pointers
    compulsory = [12 * N + 8 * p["theta_nnz"] + 8 * corpus.num_docs for p in prev]
    sample_sec = [s["sample_seconds"] for s in stats]
    achieved = sum(sample_bytes) / sum(sample_sec) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = ncu_traffic(args.workload)
    roofline = {"kernel": "sample_kernel", "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                "traffic": traffic, "bytes_per_launch": int(statistics.mean(sample_bytes)),
                "launch_ms": round(1e3 * statistics.mean(sample_sec), 4),
                "rebuild_ms": round(1e3 * statistics.mean(s["rebuild_seconds"] for s in stats), 4),
                "formula": "sum_t (4 doc id + 2 topic in + 2 topic out + 8 row) + 4 * sum_t nnz(row of d(t))",
                "compulsory_bytes_per_launch": int(statistics.mean(compulsory)),
                "compulsory_frac": round(sum(compulsory) / sum(sample_sec) / 1e9 / peak, 4),
                "compulsory_formula": "12 N (doc id, topic in, topic out, uniform) + 8 nnz(theta) + 8 D (rows)",
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch, "
                                  "profiles/sample_kernel_traffic.json" if traffic else None}
    m.close()

    # ---- end to end through the public API from pinned host buffers
    e2e = None
    if not args.no_e2e:
        import torch

        cudart = torch.cuda.cudart()
        c = corpus.c_ptr.contents
        regs = [(C.cast(c.doc_ids, C.c_void_p).value, 4 * N), (C.cast(c.word_ptr, C.c_void_p).value,
                8 * (corpus.num_words + 1)), (C.cast(c.doc_ptr, C.c_void_p).value, 8 * (corpus.num_docs + 1))]
        pinned = all([int(cudart.cudaHostRegister(ptr, nbytes, 0)) == 0 for ptr, nbytes in regs])
        z_host = torch.empty(N, dtype=torch.int16, pin_memory=True)
        # each trial is a whole job (create, K iterations, topic download); the
        # median trial is reported and every trial's seconds are kept beside it
        trials = []
        for _ in range(max(1, args.e2e_trials)):
            barrier(pg)
            cuda_sync()
            t0 = time.perf_counter()
            m2 = cb.LDA(corpus, wl.k, wl.alpha, wl.beta, seed=args.seed + rank, device=local,
                        group_lanes=args.group_lanes, item_tokens=args.item_tokens,
                        sample_blocks=args.sample_blocks, flags=run_flags(args))
            t_created = time.perf_counter()
            lls = [s["loglik"] for s in m2.iterate(args.steps)]
            t_iterated = time.perf_counter()
            st = cb.lib().culda_get_topics(m2._ctx, C.cast(z_host.data_ptr(), C.POINTER(C.c_uint16)))
            cuda_sync()
            t1 = time.perf_counter()
            assert st == 0
            m2.close()
            trials.append({"seconds": allreduce_max(pg, t1 - t0), "create": t_created - t0,
                           "iterations": t_iterated - t_created, "download": t1 - t_iterated, "loglik": lls})
        for ptr, _ in regs:
            cudart.cudaHostUnregister(ptr)
        med = sorted(trials, key=lambda t: t["seconds"])[(len(trials) - 1) // 2]
        e2e_sec = med["seconds"]
        h2d = 4 * N + 8 * (corpus.num_words + 1) + 8 * (corpus.num_docs + 1)
        d2h = 2 * N + 64 * args.steps
        e2e = {"value": world * N * args.steps / e2e_sec, "unit": UNIT,
               "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(d2h / args.steps),
               "seconds": round(e2e_sec, 4), "includes": "culda_create (upload, doc index sort, initial counts, "
               "graph capture) + K iterations each reading its log-likelihood back + final topic download",
               "create_seconds": round(med["create"], 4), "iterations_seconds": round(med["iterations"], 4),
               "download_seconds": round(med["download"], 4),
               "inputs_pinned": pinned, "trials": len(trials), "trial_seconds": ", ".join(f"{t['seconds']:.4f}" for t in trials),
               "trial_create_seconds": ", ".join(f"{t['create']:.4f}" for t in trials),
               "first_trial_value": world * N * args.steps / trials[0]["seconds"],
               "loglik_last": med["loglik"][-1] if med["loglik"] else None}

    # ---- CPU baseline (rank 0, one GPU only): the OpenMP port of the same rule
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O

        t0 = time.perf_counter()
        h = O.CpuCgs(corpus.doc_ptr, corpus.word_ptr, corpus.doc_ids, wl.k, wl.alpha, wl.beta, args.seed)
        setup = time.perf_counter() - t0
        secs = []
        while len(secs) < args.cpu_iterations and sum(secs) < args.cpu_budget:
            s, _ = h.iterate(1)
            secs.append(float(s[0]))
        cpu = {"value": N / statistics.mean(secs), "unit": UNIT, "cores": h.threads, "kind": "port",
               "sample": f"iterations 1-{len(secs)} of a fresh chain on the full {N}-token corpus "
                         f"(set-up {setup:.1f}s untimed); oracle/cgs_cpu.cpp, same sampling rule, FP32, OpenMP"}
        h.close()

    # ---- learned form vs plain, and fold-in (rank 0, one GPU only)
    learned = foldin = None
    if rank == 0 and world == 1 and not args.no_learned:
        try:
            learned = measure_learned(args, wl, corpus, local)
        except Exception as e:  # reported, never hides the main line
            learned = {"error": f"{type(e).__name__}: {e}"}
        try:
            foldin = measure_foldin(args, local)
        except Exception as e:
            foldin = {"error": f"{type(e).__name__}: {e}"}
    uneven = None
    if rank == 0 and world == 1 and not args.no_uneven:
        try:
            uneven = measure_uneven(args, local)
        except Exception as e:
            uneven = {"error": f"{type(e).__name__}: {e}"}

    launches = info["kernels_per_iteration"] * args.steps
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * max_seconds / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32", "data": "synthetic (seeded generator, shapes of the workload)",
        "config": common_config(wl, N, corpus.num_docs, corpus.num_words, args.seed, world),
        "variant": {"group_lanes": info["group_lanes"], "sample_blocks": info["sample_blocks"],
                    "token_order": "input" if args.no_reorder else "by doc length inside each word",
                    "autotuned": bool(info["tuned"]), "items": info["num_items"], "hot_words": info["num_hot"],
                    "theta_min_len": info["theta_min_len"], "theta_long_docs": info["theta_long_docs"],
                    "resident_gb": round(info["device_bytes"] / 1e9, 3)},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk, "gpu_launches": launches,
        "learned": learned, "foldin": foldin, "uneven": uneven,
        "loglik": [round(s["loglik"], 8) for s in stats],
    }
    return line


# ------------------------------------------------------ encoder training
def run_encoder(args, world, rank, local):
    """--mode encoder: the learned proposal's encoder trained on the chain's
    own states (plain iterations 1-40, states 21-40 accumulated), for each
    batch size of --encoder-batches; prints seconds per epoch and the loss.
    Rank 0 only."""
    import torch

    import culda_cgs_b200 as cb

    if rank != 0:
        return None
    wl = workload(args, args.seed)
    c = cb.Corpus.generate(wl.gen)
    out = {"mode": "encoder", "config": common_config(wl, c.num_tokens, c.num_docs, c.num_words, args.seed, 1),
           "epochs": args.learned_epochs, "runs": []}
    with cb.LDA(c, wl.k, wl.alpha, wl.beta, seed=args.seed, device=local) as m:
        m.iterate(20)
        for _ in range(20):
            m.iterate(1)
            m.accumulate_theta()
        for b in (int(x) for x in args.encoder_batches.split(",")):
            with cb.Encoder(c.num_words, wl.k, b, seed=1, device=local) as enc:
                m.init_encoder(enc, seed=3)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                losses = [m.train_encoder(enc, 1, seed=e) for e in range(args.learned_epochs)]
                torch.cuda.synchronize()
                t = time.perf_counter() - t0
            out["runs"].append({"batch": b, "seconds": round(t, 4), "seconds_per_epoch": round(t / len(losses), 4),
                                "docs_per_sec": round(c.num_docs * len(losses) / t, 1),
                                "loss_first_last": [round(losses[0], 4), round(losses[-1], 4)]})
    return out


# ------------------------------------------------- doc-chunk data parallel
def run_dp(args, world, rank, local, pg):
    """--mode dp: one corpus split into `world` token-balanced doc chunks, one
    per rank (the reference's -g N -c N); every iteration each rank samples its
    chunk against the summed counts, then the chunks' counts are summed by an
    NCCL all-reduce.  Total work is fixed (strong scaling); the step time is
    the slowest rank's, on CUDA events around sample + rebuild + exchange."""
    import torch

    import culda_cgs_b200 as cb
    from culda_cgs_b200.chunked import ChunkedLDA

    wl = workload(args, args.seed)
    corpus = cb.Corpus.generate(wl.gen)
    N = corpus.num_tokens
    dp = ChunkedLDA(corpus, wl.k, wl.alpha, wl.beta, seed=args.seed, rank=rank, world=world, device=local)
    log(f"[rank {rank}] chunk docs {dp.doc_range} tokens {dp.chunk.num_tokens} of {N}")
    dp.iterate(args.warmup)
    clocks = ClockSampler(local)
    clocks.start()
    barrier(pg)
    cuda_sync()
    clocks.mark_start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    stats = dp.iterate(args.steps)
    ev1.record()
    cuda_sync()
    barrier(pg)
    clocks.mark_end()
    clk = clocks.stop()
    seconds = allreduce_max(pg, ev0.elapsed_time(ev1) / 1e3)
    dp.close()
    return {
        "metric": METRIC, "value": N * args.steps / seconds, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * seconds / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "fp32",
        "data": "synthetic (seeded generator, shapes of the workload)",
        "config": common_config(wl, N, corpus.num_docs, corpus.num_words, args.seed, world)
        | {"parallelism": f"doc-chunk dp{world} (NCCL all-reduce of V*K+K int32 counts per iteration)"},
        "clocks": clk, "loglik": [round(s["loglik_global"], 8) for s in stats],
        "exchange_bytes_per_step": 4 * (corpus.num_words * wl.k + wl.k),
    }


# -------------------------------------------------------------- reference
ITER_RE = re.compile(r"Iteration\s+(\d+):\s+([\d.]+) sec,\s+([\d.]+) sec, logLikelyhood = ([-\d.naninf]+),\s+([\d.]+) M")


def repo_library_mapped() -> bool:
    """True when this process has mapped the repository's own library."""
    try:
        return "libculda_b200.so" in Path("/proc/self/maps").read_text()
    except OSError:
        return False


def gencorpus_command(gen, prefix: str) -> list[str]:
    """culda_cgs_b200/bin/gencorpus arguments for a GenConfig: the corpus is
    generated and written by that host program, so the reference arm's own
    process never loads the repository's library."""
    law = {0: "poisson", 1: "lognormal", 2: "pareto"}[gen.len_law]
    return [str(ROOT / "culda_cgs_b200" / "bin" / "gencorpus"), "-words", str(gen.num_words),
            "-topics", str(gen.num_topics), "-docs", str(gen.num_docs), "-law", law, "-a", repr(float(gen.len_a)),
            "-b", repr(float(gen.len_b)), "-min", str(gen.len_min), "-max", str(gen.len_max),
            "-zipf", repr(float(gen.zipf_s)), "-wconc", repr(float(gen.word_conc)),
            "-dconc", repr(float(gen.doc_conc)), "-seed", str(gen.seed), "-threads", str(gen.threads), "-o", prefix]


def run_reference(args, world, rank):
    if rank != 0:
        return None
    binary = ROOT / "oracle" / "_ref" / "culda"
    if not binary.exists():
        return {"impl": "reference", "unavailable": "oracle/_ref/culda was not built (reference sources absent)"}
    wl = workload(args, args.seed)
    if wl.k != 1024:
        return {"impl": "reference", "unavailable": "the reference kernel supports only K=1024"}
    tmp = Path(tempfile.mkdtemp(prefix="culda_ref_"))
    try:
        g = subprocess.run(gencorpus_command(wl.gen, str(tmp / "corpus")), capture_output=True, text=True,
                           timeout=600)
        if g.returncode != 0:
            return {"impl": "reference", "unavailable": f"corpus generation failed: {g.stderr.strip()[-200:]}"}
        sizes = json.loads(g.stdout.strip().splitlines()[-1])
        N = int(sizes["num_tokens"])
        iters = args.warmup + args.steps
        cmd = [str(binary), "-g", "1", "-c", "1", "-k", str(wl.k), "-t", str(iters), "-s", "1",
               "-a", repr(float(wl.alpha)), "-b", repr(float(wl.beta)), "-i", str(tmp / "corpus")]
        log("reference:", " ".join(cmd))
        clocks = ClockSampler(0)
        clocks.start()
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=args.ref_timeout)
        clk = clocks.stop()  # the whole run (load included): its iterations are not separable here
        rows = [m.groups() for m in ITER_RE.finditer(r.stdout)]
        if r.returncode != 0 or len(rows) < iters:
            tail = (r.stdout + r.stderr)[-400:].replace("\n", " | ")
            return {"impl": "reference", "unavailable": f"reference run failed (rc={r.returncode}): {tail}"}
        for it, el, st, ll, mt in rows:
            log(f"reference iteration {it}: {float(st) * 1e3:.1f} ms loglik {ll} {mt} M")
        # the printed seconds have two decimals; the M tokens/s column has three
        # significant decimals of a number in the hundreds, so derive each
        # iteration's time from it
        stamps = [N / (float(x[4]) * 1e6) for x in rows[args.warmup:iters]]
        value = N * len(stamps) / sum(stamps)
        return {
            "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sum(stamps) / len(stamps), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp16 phiHead / fp32 sums",
            "data": "synthetic (seeded generator, shapes of the workload)",
            "config": common_config(wl, N, sizes["num_docs"], sizes["num_words"], args.seed, 1),
            "timing": "the reference's own per-iteration host clock (SingleChunkSingleGPU.h:72-127)",
            "binary": "oracle/_ref/culda: the reference's src_culda compiled unmodified for sm_100a "
                      "(oracle/build_oracle.py, compatibility header only)",
            "corpus_writer": "culda_cgs_b200/bin/gencorpus in its own process",
            "repo_library_mapped": repo_library_mapped(),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                             "sample": f"iterations {args.warmup + 1}-{iters} of the reference's CUDA build "
                                       "(oracle/_ref/culda, sm_100a) on one B200, driven by one host thread"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "clocks": clk, "loglik": [float(x[3]) for x in rows[args.warmup:iters]],
        }
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--mode", choices=["replicas", "dp", "encoder"], default="replicas",
                    help="N > 1: independent replicas (default) or doc-chunk data parallelism; "
                         "encoder: time the learned proposal's training only")
    ap.add_argument("--encoder-batches", default="1024,4096", help="--mode encoder: batch sizes")
    ap.add_argument("--workload", default="plain-cgs-scale")
    ap.add_argument("--k", type=int, default=0, help="topics (default: the workload's); alpha = 50/K")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--group-lanes", type=int, default=0)
    ap.add_argument("--item-tokens", type=int, default=0)
    ap.add_argument("--sample-blocks", type=int, default=0, help="sampler register budget (CTAs per SM): 0 (auto), 8, 9 (flat walk), 10 (group samplers)")
    ap.add_argument("--autotune", action="store_true", help="time the sampler variants at create and keep the fastest")
    ap.add_argument("--no-reorder", action="store_true", help="keep tokens in input order inside each word")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-trials", type=int, default=3, help="whole-job end-to-end trials; the median is reported")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-iterations", type=int, default=2)
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of CPU baseline work at most")
    ap.add_argument("--ref-timeout", type=float, default=1200.0)
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-form and fold-in measurements")
    ap.add_argument("--no-uneven", action="store_true", help="skip the autotuned uneven-workload measurement")
    ap.add_argument("--uneven-ks", type=lambda v: [int(x) for x in v.split(",") if x], default=[256, 2048, 4096],
                    help="the rest of the uneven workload's K sweep, measured after K = 1024 (empty: none)")
    ap.add_argument("--learned-epochs", type=int, default=8)
    ap.add_argument("--learned-batch", type=int, default=1024)
    args = ap.parse_args()
    if args.warmup < 0 or args.steps < 1:
        ap.error("--steps >= 1 and --warmup >= 0")

    world, rank, local, pg = dist_setup()
    try:
        if args.impl == "reference":
            line = run_reference(args, world, rank)
        elif args.mode == "dp":
            line = run_dp(args, world, rank, local, pg)
        elif args.mode == "encoder":
            line = run_encoder(args, world, rank, local)
        else:
            line = run_ours(args, world, rank, local, pg)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
