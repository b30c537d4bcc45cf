"""Checkpoint and resume: a chain saved after 3 iterations and restored into a
fresh context continues with exactly the draws of the uninterrupted chain."""
from __future__ import annotations

import numpy as np
import pytest

import culda_cgs_b200 as cb
from culda_cgs_b200.configs import MINI

pytestmark = pytest.mark.gpu


def test_resume_continues_the_same_chain(tmp_path):
    c = cb.Corpus.generate(MINI.gen)
    args = (c, 1024, 50.0 / 1024, 0.01)
    with cb.LDA(*args, seed=77) as a:
        lls = [s["loglik"] for s in a.iterate(6)]
        z_full = a.topics()
    with cb.LDA(*args, seed=77) as b:
        b.iterate(3)
        assert b.next_iteration == 4
        b.save(tmp_path / "chain.npz")
    with cb.LDA(*args, seed=77) as r:
        r.restore(tmp_path / "chain.npz")
        assert r.next_iteration == 4
        st = r.iterate(3)
        assert [s["iteration"] for s in st] == [4, 5, 6]
        assert [s["loglik"] for s in st] == lls[3:]
        assert np.array_equal(r.topics(), z_full)


def test_restore_rejects_other_settings(tmp_path):
    c = cb.Corpus.generate(MINI.gen)
    with cb.LDA(c, 1024, 50.0 / 1024, 0.01, seed=1) as a:
        a.iterate(1)
        a.save(tmp_path / "s.npz")
    with cb.LDA(c, 1024, 50.0 / 1024, 0.01, seed=2) as b:
        with pytest.raises(ValueError):
            b.restore(tmp_path / "s.npz")
        with pytest.raises(cb.CuldaError):
            b.set_iteration(0)
