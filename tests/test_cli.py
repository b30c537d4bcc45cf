"""The `culda` command (culda_cgs_b200/bin/culda): the reference's flags and
its per-iteration output line (src_culda/main.cpp:40-194,
src_culda/train/SingleChunkSingleGPU.h:127).  Argument and file errors are
checked on the CPU; a short run on the GPU prints exactly the reference's line
format, leaves the same topics as the library's own chain and writes the -o
reports in the layouts of the reference's commented-out saveWord / saveDoc
(src_culda/model/model_phi.cpp:283-329, model_theta.cpp:207-242)."""
from __future__ import annotations

import re
import subprocess

import numpy as np
import pytest

import culda_cgs_b200 as cb
from culda_cgs_b200 import build
from culda_cgs_b200.configs import TINY

LINE = re.compile(r"^Iteration +(\d+): +[\d.]+ sec, [\d.]+ sec, logLikelyhood = (-?\d+\.\d{8}), +[\d.]+ M$")


def _run(*args, timeout=300):
    exe = build.build_cli()
    return subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=timeout)


def test_no_arguments_is_an_error():
    r = _run()
    assert r.returncode == 1 and "No argument found" in r.stdout


@pytest.mark.parametrize("args,msg", [
    (["-k", "x"], "should be followed by a positive integer"),
    (["-k", "64", "-t", "2", "-a", "0.1", "-b", "0.01"], "Error"),  # no -i
    (["-k"], "need to specify a value after -k"),
])
def test_bad_arguments(args, msg):
    r = _run(*args)
    assert r.returncode != 0 and msg in r.stdout + r.stderr


def test_missing_corpus_files(tmp_path):
    r = _run("-g", "1", "-c", "1", "-k", "64", "-t", "1", "-a", "0.1", "-b", "0.01", "-i", tmp_path / "nothing")
    assert r.returncode == 2 and "Error" in r.stderr


@pytest.mark.gpu
def test_run_prints_the_reference_line_and_matches_the_library(tmp_path):
    c = cb.Corpus.generate(TINY.gen)
    c.write(str(tmp_path / "c"))
    r = _run("-g", "1", "-c", "1", "-k", "64", "-t", "3", "-a", "0.1", "-b", "0.01", "-i", tmp_path / "c",
             "-z", tmp_path / "z.bin", "-o", tmp_path / "model")
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("Iteration")]
    assert len(lines) == 3 and all(LINE.match(ln) for ln in lines), lines
    z_cli = np.fromfile(tmp_path / "z.bin", dtype=np.int16).view(np.uint16)
    with cb.LDA(c, 64, 0.1, 0.01, seed=1) as m:
        lls = [s["loglik"] for s in m.iterate(3)]
        assert np.array_equal(m.topics(), z_cli)
        phi, nk = m.phi()
    printed = [float(LINE.match(ln).group(2)) for ln in lines]
    assert np.allclose(printed, lls, atol=1e-8)
    vocab = dict(ln.rsplit(" ", 1)[::-1] for ln in (tmp_path / "c.vocab").read_text().splitlines())
    top = (tmp_path / "model.topwords").read_text().splitlines()
    assert top[0] == "topic, total, top words"
    rows = {}
    for ln in top[1:]:
        m = re.match(r"^ *(\d+) (\d+) ((?:\([^,()]+,\d+\) )*)$", ln)
        assert m, ln
        rows[int(m.group(1))] = (int(m.group(2)), re.findall(r"\(([^,()]+),(\d+)\)", m.group(3)))
    assert sorted(rows) == [k for k in range(64) if nk[k] > 0]
    for k, (total, pairs) in rows.items():
        assert total == nk[k]
        want = sorted(((-phi[w, k], w) for w in range(phi.shape[0]) if phi[w, k] > 0))[:20]
        assert pairs == [(vocab[str(w)], str(-c)) for c, w in want]
    doc = (tmp_path / "model.doctopics").read_text().splitlines()
    assert doc[0] == "Doc, total, top topics" and len(doc) == c.num_docs + 1
    doc_of = c.doc_ids  # doc of every token, word-major like the topics
    for d, ln in enumerate(doc[1:]):
        m = re.match(r"^ *(\d+)\| (\d+) ((?:\(\d+,\d+\), )*)$", ln)
        assert m and int(m.group(1)) == d, ln
        pairs = [(int(a), int(b)) for a, b in re.findall(r"\((\d+),(\d+)\)", m.group(3))]
        ks, cs = np.unique(z_cli[doc_of == d], return_counts=True)
        assert int(m.group(2)) == cs.sum()
        assert pairs == sorted(zip(ks.tolist(), cs.tolist()), key=lambda kc: (-kc[1], kc[0]))
