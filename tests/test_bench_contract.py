"""bench.py's reference arm on the host side (no GPU).

The reference arm must not map the repository's library: its corpus files
come from the `gencorpus` command in a child process.  Those files must be the
ones this library's own writer produces for the same workload, so both arms
sample the same corpus, and both arms print the same `config` keys.
"""
from __future__ import annotations

import filecmp
import json
import subprocess

import bench
import culda_cgs_b200 as cb
from culda_cgs_b200 import build
from culda_cgs_b200.configs import MINI, TINY, UNEVEN

SUFFIXES = (".vocab", ".doc.idx", ".chunk", ".word.idx", ".word.data")


def test_gencorpus_writes_the_files_of_the_library_writer(tmp_path):
    build.build_gencorpus_cli()
    for wl in (TINY, MINI):
        r = subprocess.run(bench.gencorpus_command(wl.gen, str(tmp_path / "gen")), capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        sizes = json.loads(r.stdout.strip().splitlines()[-1])
        c = cb.Corpus.generate(wl.gen)
        c.write(str(tmp_path / "lib"))
        assert sizes == {"num_docs": c.num_docs, "num_words": c.num_words, "num_tokens": c.num_tokens}
        for suf in SUFFIXES:
            assert filecmp.cmp(tmp_path / f"gen{suf}", tmp_path / f"lib{suf}", shallow=False), (wl.name, suf)


def test_gencorpus_command_covers_every_length_law():
    for gen in (TINY.gen, MINI.gen, UNEVEN.gen):
        cmd = bench.gencorpus_command(gen, "/tmp/x")
        law = cmd[cmd.index("-law") + 1]
        assert law == {0: "poisson", 1: "lognormal", 2: "pareto"}[gen.len_law]
        assert cmd[cmd.index("-zipf") + 1] == repr(float(gen.zipf_s))


def test_gencorpus_rejects_a_bad_command_line():
    build.build_gencorpus_cli()
    exe = bench.ROOT / "culda_cgs_b200" / "bin" / "gencorpus"
    assert subprocess.run([str(exe), "-words", "10"], capture_output=True).returncode == 1
    assert subprocess.run([str(exe), "-law", "uniform", "-o", "/tmp/x"], capture_output=True).returncode == 1


def test_both_arms_print_the_same_config_keys():
    a = bench.common_config(MINI, 100, 10, 20, 1, 1)
    b = bench.common_config(MINI, 100, 10, 20, 1, 1)
    assert a == b and set(a) == {"workload", "num_tokens", "num_docs", "num_words", "k", "alpha", "beta", "seed",
                                 "l2", "parallelism"}
