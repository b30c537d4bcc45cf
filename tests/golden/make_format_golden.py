"""Record golden outputs of the reference's preprocessing tool.

Runs `oracle/_ref/format` (src_format/format.cpp compiled from the reference's
sources by oracle/build_oracle.py) on small seeded text corpora that hold the
edge cases of its input format, and stores every input with every output file
in tests/golden/format_golden.npz (key "<case>/<chunks>/<suffix>", uint8).

Cases: "mixed" (empty and whitespace-only lines, title-only documents, leading
whitespace, CR LF line ends, \\v \\f \\t separators, repeated tokens, UTF-8 and
non-UTF-8 bytes, a NUL byte inside a token, no final newline), "titles_only"
(documents without tokens: zero tokens in all), "empty" (a 0-byte file) and
"one_word" (a single token).

    python tests/golden/make_format_golden.py [out_dir]      (default: tests/golden)
"""
from __future__ import annotations

import random
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
CHUNKS = (1, 3, 8)
SUFFIXES = (".vocab", ".doc.idx", ".chunk")


def mixed_text(seed: int = 5, lines: int = 400) -> bytes:
    r = random.Random(seed)
    alphabet = [c.encode() for c in "abcdefghijklmnopqrstuvwxyz0123456789_-.,;:!?ÄéßΩ東京"] + [b"\xff", b"\xc3"]
    words = [b"".join(r.choice(alphabet) for _ in range(r.randint(1, 10))) for _ in range(150)]
    words.append(b"nul\x00byte")
    seps = [b" ", b"  ", b"\t", b"\v", b"\f", b" \r ", b"\t \t"]
    out = []
    for i in range(lines):
        u = r.random()
        if u < 0.05:
            out.append(b"")
        elif u < 0.08:
            out.append(r.choice([b" ", b"\t", b"\r", b" \v\f "]))
        elif u < 0.12:
            out.append(b"  title%d" % i + r.choice([b"", b" ", b"\r"]))
        else:
            line = r.choice([b"", b" ", b"\t"]) + b"d%d" % i
            for _ in range(int(r.expovariate(1 / 12))):
                w = words[min(int(r.paretovariate(1.2)) - 1, len(words) - 1)] if r.random() < 0.7 \
                    else r.choice(words)
                line += r.choice(seps) + w
            out.append(line + r.choice([b"", b"", b" ", b"\r"]))
    return b"\n".join(out)  # no final newline


CASES = {
    "mixed": mixed_text(),
    "titles_only": b"a\nb  \n\n  c\r\nd",
    "empty": b"",
    "one_word": b"doc0 w\n",
}


def main(out_dir: Path) -> None:
    exe = ROOT / "oracle" / "_ref" / "format"
    if not exe.exists():
        raise SystemExit(f"{exe} is missing: run oracle/build_oracle.py where the reference sources are")
    arrays = {}
    with tempfile.TemporaryDirectory() as tmp:
        tmp = Path(tmp)
        for name, text in CASES.items():
            src = tmp / f"{name}.txt"
            src.write_bytes(text)
            arrays[f"{name}/input"] = np.frombuffer(text, dtype=np.uint8)
            for ch in CHUNKS:
                pre = tmp / f"{name}_{ch}"
                subprocess.run([str(exe), str(src), str(pre), str(ch)], check=True, stdout=subprocess.DEVNULL)
                parts = [""] if ch == 1 else [str(i) for i in range(ch)]
                names = list(SUFFIXES) + [s + p for p in parts for s in (".word.idx", ".word.data")]
                for suf in names:
                    arrays[f"{name}/{ch}/{suf}"] = np.frombuffer(Path(str(pre) + suf).read_bytes(), dtype=np.uint8)
    np.savez_compressed(out_dir / "format_golden.npz", **arrays)


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent)
