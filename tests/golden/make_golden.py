"""Record golden vectors from the reference's own CUDA code (run on a B200).

For each fixture: generate a seeded corpus, write it in the reference's file
format, pick a topic assignment, and run `oracle/_ref/ref_harness` (the
reference's Document / ModelPhi / ModelTheta classes and its LDAKernelTrain +
LDATrainPerplexity, compiled from its sources by oracle/build_oracle.py).
The fixture keeps the inputs (generator settings, topics) and the reference's
outputs: SHA-256 digests of phi, n_k, the FP16 phiHead table, theta (A, JA,
MaxIA, CurIA) and docRevIdx, the small arrays themselves, the slots, the
log-likelihood the reference prints after one sampling pass, and the topics it
drew in that pass.

    python tests/golden/make_golden.py [out_dir]      (default: tests/golden)
"""
from __future__ import annotations

import hashlib
import json
import subprocess
import sys
import tempfile
from dataclasses import asdict
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import culda_cgs_b200 as cb  # noqa: E402
from culda_cgs_b200._ffi import CULDA_LEN_LOGNORMAL, CULDA_LEN_POISSON  # noqa: E402
from culda_cgs_b200.corpus import GenConfig  # noqa: E402
from oracle import oracle as O  # noqa: E402

K, ALPHA, BETA = 1024, 50.0 / 1024.0, 0.01

FIXTURES = {
    # random initial topics: long theta rows
    "ref_tiny_init": dict(gen=GenConfig(num_words=500, num_topics=8, num_docs=200, len_law=CULDA_LEN_POISSON,
                                        len_a=40.0, len_min=1, len_max=200, seed=11), topics="init", seed=3),
    # topics after a few iterations of this library's sampler: short rows, padding, compaction
    "ref_mini_iter5": dict(gen=GenConfig(num_words=3000, num_topics=40, num_docs=800, len_law=CULDA_LEN_LOGNORMAL,
                                         len_a=4.0, len_b=0.8, len_min=1, len_max=1500, seed=12),
                           topics="chain5", seed=4),
    # docs longer than K (row capacity capped at K) and words split into slots
    "ref_long_docs": dict(gen=GenConfig(num_words=2000, num_topics=20, num_docs=40, len_law=CULDA_LEN_LOGNORMAL,
                                        len_a=7.0, len_b=0.3, len_min=800, len_max=3000, seed=13),
                          topics="init", seed=5),
}

ARRAYS = {  # name: (dtype, digest it)
    "phi": (np.int32, True), "nk": (np.int32, True), "phihead": (np.uint16, True), "theta_a": (np.int16, True),
    "theta_ja": (np.int16, True), "max_ia": (np.int32, True), "cur_ia": (np.int32, True),
    "doc_rev_idx": (np.int32, True), "slot_word": (np.int32, False), "slot_range": (np.int64, False),
    "z_new": (np.int16, False), "loglik": (np.float64, False),
}


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def topics_for(corpus: cb.Corpus, spec: dict) -> np.ndarray:
    if spec["topics"] == "init":
        return O.init_topics(corpus.num_tokens, K, spec["seed"])
    with cb.LDA(corpus, K, ALPHA, BETA, seed=spec["seed"]) as m:
        m.iterate(5)
        return m.topics()


def make(name: str, spec: dict, out_dir: Path) -> None:
    harness = ROOT / "oracle" / "_ref" / "ref_harness"
    corpus = cb.Corpus.generate(spec["gen"])
    z = topics_for(corpus, spec)
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        corpus.write(str(td / "c"))
        z.astype(np.int16).tofile(td / "z.bin")
        r = subprocess.run([str(harness), str(td / "c"), str(K), repr(ALPHA), repr(BETA), str(td / "z.bin"),
                            str(td / "out"), "1"], capture_output=True, text=True, timeout=600)
        if r.returncode != 0:
            raise RuntimeError(f"{name}: harness failed ({r.returncode}): {r.stderr[-2000:]}")
        files = {"corpus": {s: sha(np.fromfile(td / f"c.{s}", dtype=np.uint8))
                            for s in ("vocab", "doc.idx", "chunk", "word.idx", "word.data")}}
        out = {k: np.fromfile(td / f"out.{k}.bin", dtype=dt) for k, (dt, _) in ARRAYS.items()}
    digests = {k: sha(out[k]) for k, (_, d) in ARRAYS.items() if d}
    meta = {"name": name, "gen": asdict(spec["gen"]), "topics": spec["topics"], "seed": spec["seed"], "k": K,
            "alpha": ALPHA, "beta": BETA, "num_tokens": corpus.num_tokens, "digests": digests,
            "files": files["corpus"], "harness_stdout": r.stdout.strip().splitlines()[-2:]}
    np.savez_compressed(out_dir / f"{name}.npz", meta=json.dumps(meta), z=z.astype(np.uint16), nk=out["nk"],
                        max_ia=out["max_ia"], cur_ia=out["cur_ia"], slot_word=out["slot_word"],
                        slot_range=out["slot_range"], z_new=out["z_new"].view(np.uint16), loglik=out["loglik"])
    print(f"{name}: N={corpus.num_tokens} loglik={out['loglik'][0]:.10f} slots={len(out['slot_word'])}")


def main() -> None:
    out_dir = Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent
    out_dir.mkdir(parents=True, exist_ok=True)
    for name, spec in FIXTURES.items():
        make(name, spec, out_dir)


if __name__ == "__main__":
    main()
