"""Synthetic corpora standing in for the reference's unnamed datasets.

Each workload is a seeded generator configuration (same shapes, sizes and
value distributions as the benchmark suite it is quoted on) plus the sampler
settings (K, alpha, beta, iterations).
"""
from __future__ import annotations

from dataclasses import dataclass, replace

from ._ffi import CULDA_LEN_LOGNORMAL, CULDA_LEN_PARETO, CULDA_LEN_POISSON
from .corpus import GenConfig


@dataclass(frozen=True)
class Workload:
    name: str
    gen: GenConfig
    k: int = 1024
    alpha: float = 50.0 / 1024.0
    beta: float = 0.01
    iterations: int = 50

    def with_seed(self, seed: int) -> "Workload":
        return replace(self, gen=replace(self.gen, seed=seed))


# ~1M tokens: V=20k Zipf(1.05) topic-word priors, 100 generating topics,
# 10k docs with Poisson(100) lengths clipped to [10, 1000].
SMALL = Workload("plain-cgs-small V=20k D=10k N~1M K=1024",
                 GenConfig(num_words=20_000, num_topics=100, num_docs=10_000, len_law=CULDA_LEN_POISSON,
                           len_a=100.0, len_min=10, len_max=1000), iterations=50)

# ~60M tokens: V=100k, 500 generating topics, 300k docs, lognormal(5, 0.8)
# lengths clipped to [5, 5000].  The headline workload.
SCALE = Workload("plain-cgs-scale V=100k D=300k N~60M K=1024",
                 GenConfig(num_words=100_000, num_topics=500, num_docs=300_000, len_law=CULDA_LEN_LOGNORMAL,
                           len_a=5.0, len_b=0.8, len_min=5, len_max=5000), iterations=100)

# ~12M tokens, the same generator as SCALE with a fifth of the docs: inputs
# still above the L2 size, small enough for detailed profiler captures.
MEDIUM = Workload("plain-cgs-medium V=100k D=60k N~12M K=1024",
                  GenConfig(num_words=100_000, num_topics=500, num_docs=60_000, len_law=CULDA_LEN_LOGNORMAL,
                            len_a=5.0, len_b=0.8, len_min=5, len_max=5000), iterations=100)

# ~100M tokens of very uneven documents: V=1M Zipf(1.1), 1000 generating
# topics, 2M docs with Pareto(1.5, 20) lengths clipped at 50k.
UNEVEN = Workload("batched-uneven V=1M D=2M N~100M",
                  GenConfig(num_words=1_000_000, num_topics=1000, num_docs=2_000_000, len_law=CULDA_LEN_PARETO,
                            len_a=1.5, len_b=20.0, len_min=20, len_max=50_000, zipf_s=1.1), iterations=50)

# Fold-in: the SMALL generator with 110k docs; the first 10k are the training
# corpus (the SMALL shape), the other 100k are new documents over the same
# vocabulary, sampled against the trained model's frozen counts.
FOLDIN = Workload("foldin V=20k D=10k+100k K=1024",
                  GenConfig(num_words=20_000, num_topics=100, num_docs=110_000, len_law=CULDA_LEN_POISSON,
                            len_a=100.0, len_min=10, len_max=1000), iterations=50)
FOLDIN_TRAIN_DOCS = 10_000

# small corpora for tests
TINY = Workload("tiny V=500 D=200 K=64",
                GenConfig(num_words=500, num_topics=8, num_docs=200, len_law=CULDA_LEN_POISSON, len_a=40.0,
                          len_min=1, len_max=200), k=64, iterations=5)

MINI = Workload("mini V=3k D=2k K=1024",
                GenConfig(num_words=3_000, num_topics=40, num_docs=2_000, len_law=CULDA_LEN_LOGNORMAL, len_a=4.0,
                          len_b=0.8, len_min=1, len_max=1500), k=1024, iterations=5)

WORKLOADS = {w.name.split()[0]: w for w in (SMALL, SCALE, MEDIUM, UNEVEN, FOLDIN, TINY, MINI)}
