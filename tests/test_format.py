"""Text corpus -> word-first files: culda_format_text / Corpus.from_text and
the `format` command against the reference's preprocessing tool
(src_format/format.cpp:19-165, src_format/data_chunk.h:49-67).

The oracle (oracle/format_oracle.py) is pinned to the golden outputs of the
reference's own tool (tests/golden/format_golden.npz, recorded by
tests/golden/make_format_golden.py); the library must write the same bytes as
both, on the golden edge cases and on seeded multi-megabyte texts that the
parser cuts into several ranges.  All of it runs on the CPU."""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import culda_cgs_b200 as cb
from culda_cgs_b200 import CuldaError, build
from culda_cgs_b200._ffi import CULDA_ERR_IO
from oracle import format_oracle

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "tests" / "golden"))
from make_format_golden import CHUNKS, mixed_text  # noqa: E402

GOLDEN = np.load(ROOT / "tests" / "golden" / "format_golden.npz")
CASES = sorted({k.split("/")[0] for k in GOLDEN.files})
REF_FORMAT = ROOT / "oracle" / "_ref" / "format"


def _golden(case: str, chunks: int) -> dict[str, bytes]:
    head = f"{case}/{chunks}/"
    return {k[len(head):]: GOLDEN[k].tobytes() for k in GOLDEN.files if k.startswith(head)}


def _written(prefix: Path, suffixes) -> dict[str, bytes]:
    return {s: Path(str(prefix) + s).read_bytes() for s in suffixes}


@pytest.fixture(scope="module")
def big_text(tmp_path_factory) -> Path:
    """About 3.5 MB: three or more parse ranges of at least 1 MiB each."""
    p = tmp_path_factory.mktemp("fmt") / "big.txt"
    p.write_bytes(mixed_text(seed=17, lines=40000))
    return p


@pytest.mark.parametrize("chunks", CHUNKS)
@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference_tool_golden(case, chunks):
    want = _golden(case, chunks)
    got = format_oracle.format_files(GOLDEN[f"{case}/input"].tobytes(), chunks)
    assert got.keys() == want.keys()
    for suf in want:
        assert got[suf] == want[suf], suf


@pytest.mark.parametrize("threads", [1, 4])
@pytest.mark.parametrize("chunks", CHUNKS)
@pytest.mark.parametrize("case", CASES)
def test_library_matches_reference_tool_golden(tmp_path, case, chunks, threads):
    src = tmp_path / "in.txt"
    src.write_bytes(GOLDEN[f"{case}/input"].tobytes())
    cb.format_text(src, tmp_path / "out", chunks, threads)
    want = _golden(case, chunks)
    assert _written(tmp_path / "out", want) == want


@pytest.mark.parametrize("chunks", [1, 4])
def test_library_matches_oracle_on_multi_range_text(tmp_path, big_text, chunks):
    want = format_oracle.format_files(big_text.read_bytes(), chunks)
    for threads in (0, 2, 7):
        pre = tmp_path / f"t{threads}"
        cb.format_text(big_text, pre, chunks, threads)
        got = _written(pre, want)
        for suf in want:
            assert got[suf] == want[suf], (threads, suf)


@pytest.mark.skipif(not REF_FORMAT.exists(), reason="the reference's tool is built only where its sources are")
def test_command_matches_reference_tool(tmp_path, big_text):
    exe = build.build_format_cli()
    for chunks in (1, 5):
        a = subprocess.run([str(REF_FORMAT), str(big_text), str(tmp_path / "ref"), str(chunks)],
                           capture_output=True, check=True)
        b = subprocess.run([str(exe), str(big_text), str(tmp_path / "our"), str(chunks)], capture_output=True)
        assert b.returncode == 0, b.stdout + b.stderr
        # the progress lines name the output prefix; everything else is the same
        assert b.stdout.replace(b"/our", b"/ref") == a.stdout
        parts = [""] if chunks == 1 else [str(i) for i in range(chunks)]
        sufs = [".vocab", ".doc.idx", ".chunk"] + [s + p for p in parts for s in (".word.idx", ".word.data")]
        assert _written(tmp_path / "our", sufs) == _written(tmp_path / "ref", sufs)


def test_from_text_equals_loading_the_written_files(tmp_path, big_text):
    c = cb.Corpus.from_text(big_text, threads=3)
    c.write(tmp_path / "w")
    d = cb.Corpus.load(tmp_path / "w")
    assert (c.num_docs, c.num_words, c.num_tokens) == (d.num_docs, d.num_words, d.num_tokens)
    assert np.array_equal(c.doc_ptr, d.doc_ptr)
    assert np.array_equal(c.word_ptr, d.word_ptr)
    assert np.array_equal(c.doc_ids, d.doc_ids)
    lines = (tmp_path / "w.vocab").read_bytes().split(b"\n")[:-1]
    tokens = [ln.rsplit(b" ", 1)[0].decode("utf-8", "surrogateescape") for ln in lines]
    assert tokens == c.vocab


def test_missing_input_is_an_io_error(tmp_path):
    with pytest.raises(CuldaError) as e:
        cb.format_text(tmp_path / "absent.txt", tmp_path / "out")
    assert e.value.status == CULDA_ERR_IO and "open failed" in str(e.value)
    assert not (tmp_path / "out.vocab").exists()
    r = subprocess.run([str(build.build_format_cli()), str(tmp_path / "absent.txt"), str(tmp_path / "out")],
                       capture_output=True, text=True)
    assert r.returncode == 2 and "absent.txt open failed" in r.stdout


def test_command_usage(tmp_path):
    r = subprocess.run([str(build.build_format_cli())], capture_output=True, text=True)
    assert r.returncode == 1 and r.stdout.startswith("Usage:./format input output_prefix numChunks")


def test_unwritable_output_is_an_io_error(tmp_path):
    src = tmp_path / "in.txt"
    src.write_bytes(b"d0 a b\n")
    with pytest.raises(CuldaError) as e:
        cb.format_text(src, tmp_path / "no_such_dir" / "out")
    assert e.value.status == CULDA_ERR_IO and ".vocab open failed" in str(e.value)
