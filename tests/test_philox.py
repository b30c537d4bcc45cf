"""Philox4x32-10: the oracle and the product's header against the published
known-answer vectors (Salmon et al., SC'11; Random123 kat_vectors)."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

ROOT = Path(__file__).resolve().parent.parent

KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,expect", KAT)
def test_oracle_philox_kat(ctr, key, expect):
    assert tuple(int(x) for x in O.philox4x32_10(ctr, key)) == expect


def test_product_philox_header_kat(tmp_path):
    """The device/host header used by the kernels, compiled for the host."""
    src = tmp_path / "kat.cpp"
    src.write_text(
        '#include "philox.h"\n#include <cstdio>\nint main(){\n'
        + "".join(
            f"{{ culda::u32x4 c={{{c[0]}u,{c[1]}u,{c[2]}u,{c[3]}u}}; auto o=culda::philox4x32_10(c,{k[0]}u,{k[1]}u);"
            f' printf("%08x %08x %08x %08x\\n",o.x,o.y,o.z,o.w); }}\n'
            for c, k, _ in KAT)
        + "return 0;}\n")
    exe = tmp_path / "kat"
    subprocess.run(["g++", "-std=c++17", "-I", str(ROOT / "culda_cgs_b200" / "csrc"), "-o", str(exe), str(src)],
                   check=True)
    lines = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    for line, (_, _, expect) in zip(lines, KAT):
        assert line == " ".join(f"{x:08x}" for x in expect)


def test_uniform_is_open_and_exact():
    for x in (0, 1, 511, 512, 0xFFFFFFFF, 0x80000000):
        u = O.uniform(x)
        assert 0.0 < u < 1.0
        assert np.float32(u) == u  # exactly representable in FP32
    assert O.uniform(0) == 2.0 ** -24
    assert O.uniform(0xFFFFFFFF) == 1.0 - 2.0 ** -24


def test_init_topics_range_and_balance():
    z = O.init_topics(200_000, 1024, 7)
    assert z.max() < 1024
    counts = np.bincount(z, minlength=1024)
    expected = 200_000 / 1024
    chi2 = ((counts - expected) ** 2 / expected).sum()
    assert chi2 < 1024 + 6 * np.sqrt(2 * 1024)  # ~6 sigma
    assert not np.array_equal(z, O.init_topics(200_000, 1024, 8))
