"""The sampler autotuner (CULDA_FLAG_AUTOTUNE): it picks one of the timed
variants, leaves the state it timed on untouched (the first iteration still
matches the oracle), and reuses its result from the process cache and from the
file named by CULDA_TUNE_CACHE."""
from __future__ import annotations

import numpy as np
import pytest

import culda_cgs_b200 as cb
from culda_cgs_b200._ffi import CULDA_FLAG_AUTOTUNE
from culda_cgs_b200.configs import MINI, TINY
from oracle import oracle as O

pytestmark = pytest.mark.gpu

VARIANTS = {(-1, 8), (-1, 9), (4, 10), (8, 10), (16, 10), (2, 8), (4, 8), (8, 8)}


def test_autotune_picks_a_variant_and_keeps_parity():
    c = cb.Corpus.generate(MINI.gen)
    seed = 31
    with cb.LDA(c, 1024, 50.0 / 1024, 0.01, seed=seed, flags=CULDA_FLAG_AUTOTUNE) as m:
        assert m.info()["tuned"] == 0  # timed before iteration 3
        m.iterate(2)
        s2 = O.Snapshot.build(c.word_ptr, c.doc_ids, c.doc_ptr, m.topics(), 1024, m.alpha, m.beta)
        z3, margin, ll2 = s2.sample(seed, 3)
        st = m.iterate(1)[0]
        info = m.info()
        assert info["tuned"] == 1 and info["tune_ms"] > 0
        assert (info["group_lanes"], info["sample_blocks"]) in VARIANTS
        # the rebuild's bin threshold was timed too, and its bins are consistent
        assert info["theta_tune_ms"] > 0 and info["theta_min_len"] >= 0
        L = np.diff(c.doc_ptr)
        assert info["theta_long_docs"] == (int((L >= info["theta_min_len"]).sum()) if info["theta_min_len"] else 0)
        # timing the variants left the state alone: iteration 3 samples snapshot 2
        assert st["iteration"] == 3 and st["status"] == 0
        assert abs(st["loglik"] - ll2) <= 1e-6 * max(1.0, abs(ll2))
        far = margin >= 1e-6
        assert np.array_equal(m.topics()[far], z3[far])
    # the same shapes again: the process cache answers
    with cb.LDA(c, 1024, 50.0 / 1024, 0.01, seed=seed + 1, flags=CULDA_FLAG_AUTOTUNE) as m2:
        i2 = m2.info()
        assert i2["tuned"] == 2
        assert (i2["group_lanes"], i2["sample_blocks"]) == (info["group_lanes"], info["sample_blocks"])
        assert i2["theta_min_len"] == info["theta_min_len"]


def test_autotune_reads_the_cache_file(tmp_path, monkeypatch):
    import torch

    c = cb.Corpus.generate(TINY.gen)
    name = torch.cuda.get_device_name(0).replace(" ", "_")
    key = f"{name}:N{c.num_tokens}:D{c.num_docs}:V{c.num_words}:K64"
    f = tmp_path / "tune.txt"
    f.write_text(f"{key} 2 8 0.125\n{key.replace(':K64', ':K96')} 4 8 0.5 48\n")
    monkeypatch.setenv("CULDA_TUNE_CACHE", str(f))
    with cb.LDA(c, 64, 0.1, 0.01, seed=3, flags=CULDA_FLAG_AUTOTUNE) as m:
        info = m.info()
        assert info["tuned"] == 2 and (info["group_lanes"], info["sample_blocks"]) == (2, 8)
        assert info["tune_ms"] == pytest.approx(0.125)
        assert m.iterate(1)[0]["status"] == 0
    # a line with a rebuild threshold applies it
    with cb.LDA(c, 96, 0.1, 0.01, seed=3, flags=CULDA_FLAG_AUTOTUNE) as m:
        info = m.info()
        assert info["tuned"] == 2 and info["theta_min_len"] == 48
        assert info["theta_long_docs"] == int((np.diff(c.doc_ptr) >= 48).sum()) > 0
        assert m.iterate(1)[0]["status"] == 0
    # a new key is timed and appended to the file, with its threshold
    with cb.LDA(c, 32, 0.1, 0.01, seed=3, flags=CULDA_FLAG_AUTOTUNE) as m:
        m.iterate(3)
        assert m.info()["tuned"] == 1
    lines = f.read_text().splitlines()
    assert len(lines) == 3 and lines[2].startswith(f"{name}:N{c.num_tokens}:D{c.num_docs}:V{c.num_words}:K32 ")
    assert len(lines[2].split()) == 5 and int(lines[2].split()[4]) >= 0
