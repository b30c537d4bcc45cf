"""Log-likelihood trajectories on the 60M-token corpus: the reference's own
CUDA build over several runs against this library over several seeds.

TEST INFRASTRUCTURE: run on a B200 host from the repository root, after
`python -c "import __graft_entry__ as g; g.build()"` built oracle/_ref/culda
from the reference's sources:

    python tests/trajectory/make_trajectory.py \
        [--iterations 100] [--runs 5] [--out profiles/trajectory_plain-cgs-scale.json]

Corpus: the plain-cgs-scale generator (V = 100k, D = 300k, lognormal(5, 0.8)
lengths, about 61M tokens), K = 1024, alpha = 50/1024, beta = 0.01, written
once by culda_cgs_b200/bin/gencorpus.

* The reference (`oracle/_ref/culda -g 1 -c 1 -k 1024 -t T ...`) prints, per
  iteration, the log-likelihood of the state before that iteration's sampling
  under its own arithmetic (FP16 phiHead, float sums, every warp's sum
  truncated to int; src_culda/kernel/lda_train_kernel.cu:56-356).  It seeds
  its generators from the clock (doc_chunk.cpp:259-264, lda_train_kernel.cu:14-18),
  so its runs, seconds apart, stand in for seeds.
* This library, seeds 1..R: `loglik` of each iteration, the per-token value
  of the same pre-sampling state in FP64 without truncation, and, at the
  checkpoint iterations, the reference's printed formula evaluated by the
  oracle on the same state (oracle_loglik_reference on this library's topics,
  with the reference's slots restated by oracle_reference_slots).
The record holds every series and, per checkpoint, the means and the gap of
ours to the reference in percent of the reference's magnitude.
"""
from __future__ import annotations

import argparse
import json
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

ITER_RE = re.compile(r"Iteration\s+(\d+):\s+([\d.]+) sec,\s+([\d.]+) sec, logLikelyhood = ([-\d.naninf]+),\s+([\d.]+) M")
CHECKPOINTS = (10, 25, 50, 100)


def reference_runs(prefix: str, iterations: int, runs: int, wl) -> list[dict]:
    binary = ROOT / "oracle" / "_ref" / "culda"
    out = []
    for r in range(runs):
        if r:
            time.sleep(1.5)  # the reference seeds from time(NULL): a new second, a new chain
        cmd = [str(binary), "-g", "1", "-c", "1", "-k", str(wl.k), "-t", str(iterations), "-s", "1",
               "-a", repr(float(wl.alpha)), "-b", repr(float(wl.beta)), "-i", prefix]
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=3600)
        rows = [m.groups() for m in ITER_RE.finditer(p.stdout)]
        if p.returncode != 0 or len(rows) < iterations:
            raise RuntimeError(f"reference run {r} failed (rc={p.returncode}): {(p.stdout + p.stderr)[-400:]}")
        out.append({"run": r, "loglik": [float(x[3]) for x in rows], "seconds": [float(x[2]) for x in rows]})
        print(f"reference run {r}: loglik at 1/{iterations}: {rows[0][3]} / {rows[-1][3]}", flush=True)
    return out


def ours(corpus, iterations: int, seed: int, wl, slots) -> dict:
    import culda_cgs_b200 as cb
    from oracle import oracle as O

    lls, secs, ref_formula = [], [], {}
    with cb.LDA(corpus, wl.k, wl.alpha, wl.beta, seed=seed) as m:
        for it in range(1, iterations + 1):
            if it in CHECKPOINTS:
                z = m.topics()  # the state this iteration samples from
                r = O.RowSnapshot.build(corpus.word_ptr, corpus.doc_ids, corpus.doc_ptr, z, wl.k, wl.alpha,
                                        wl.beta)
                phi, nk = O.phi_counts(corpus.num_words, wl.k, corpus.word_ptr, z)
                head = O.phi_head_f16(corpus.num_words, wl.k, r.beta, phi, nk)
                del phi
                ref_formula[it] = O.loglik_reference(r, corpus.num_tokens, slots[0], slots[1], head)
                del head, r
            st = m.iterate(1)[0]
            assert st["status"] == 0
            lls.append(st["loglik"])
            secs.append(st["seconds"])
    print(f"seed {seed}: loglik at 1/{iterations}: {lls[0]:.6f} / {lls[-1]:.6f}; reference formula "
          f"{ {k: round(v, 6) for k, v in ref_formula.items()} }", flush=True)
    return {"seed": seed, "loglik": lls, "seconds": secs,
            "loglik_reference_formula": {str(k): v for k, v in ref_formula.items()}}


def summarise(ref: list[dict], mine: list[dict], iterations: int) -> list[dict]:
    rows = []
    for it in CHECKPOINTS:
        if it > iterations:
            continue
        r = [x["loglik"][it - 1] for x in ref]
        o = [x["loglik"][it - 1] for x in mine]
        f = [x["loglik_reference_formula"][str(it)] for x in mine]
        rm, om, fm = statistics.mean(r), statistics.mean(o), statistics.mean(f)
        rows.append({"iteration": it, "reference_mean": rm, "reference_min": min(r), "reference_max": max(r),
                     "ours_mean": om, "ours_min": min(o), "ours_max": max(o),
                     "ours_reference_formula_mean": fm,
                     "gap_pct_as_printed": 100.0 * (om - rm) / abs(rm),
                     "gap_pct_reference_formula": 100.0 * (fm - rm) / abs(rm),
                     "within_0_5pct_reference_formula": abs(fm - rm) <= 0.005 * abs(rm)})
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--iterations", type=int, default=100)
    ap.add_argument("--runs", type=int, default=5)
    ap.add_argument("--out", default=str(ROOT / "profiles" / "trajectory_plain-cgs-scale.json"))
    args = ap.parse_args()

    import bench
    import culda_cgs_b200 as cb
    from culda_cgs_b200.configs import SCALE
    from oracle import oracle as O

    wl = SCALE.with_seed(1)
    tmp = Path(tempfile.mkdtemp(prefix="culda_traj_"))
    try:
        g = subprocess.run(bench.gencorpus_command(wl.gen, str(tmp / "corpus")), capture_output=True, text=True,
                           check=True)
        sizes = json.loads(g.stdout.strip().splitlines()[-1])
        ref = reference_runs(str(tmp / "corpus"), args.iterations, args.runs, wl)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    corpus = cb.Corpus.generate(wl.gen)
    assert corpus.num_tokens == sizes["num_tokens"]
    slots = O.reference_slots(corpus.word_ptr)
    mine = [ours(corpus, args.iterations, seed, wl, slots) for seed in range(1, args.runs + 1)]
    rec = {"workload": wl.name, "num_tokens": corpus.num_tokens, "num_docs": corpus.num_docs,
           "num_words": corpus.num_words, "k": wl.k, "alpha": wl.alpha, "beta": wl.beta,
           "iterations": args.iterations, "runs": args.runs, "checkpoints": summarise(ref, mine, args.iterations),
           "reference_ms_per_iteration": 1e3 * statistics.mean(s for x in ref for s in x["seconds"][1:]),
           "ours_ms_per_iteration": 1e3 * statistics.mean(s for x in mine for s in x["seconds"][1:]),
           "reference": ref, "ours": mine,
           "command": "python tests/trajectory/make_trajectory.py --iterations %d --runs %d" % (args.iterations,
                                                                                                 args.runs)}
    Path(args.out).write_text(json.dumps(rec) + "\n")
    for row in rec["checkpoints"]:
        print(json.dumps(row), flush=True)


if __name__ == "__main__":
    main()
