"""culda_sample_noalloc: the kernel-level sampler with its scratch in a fixed
device array, for callers that cannot allocate device memory for a workspace
(a serving process whose own pool allocator reserved all device memory up
front and lets no library call cudaMalloc).

Two calls in a row must give the same topics and log-likelihood as
culda_sample with a workspace on the same inputs: the array keeps the last
call's contents, so the second call checks that everything which must start at
zero is cleared again.  This file is collected last, and the test passes
alone in a fresh process as well as after the other tests.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import culda_cgs_b200 as cb
from culda_cgs_b200 import _ffi
from culda_cgs_b200.configs import MINI
from oracle import oracle as O

from kernel_api import doc_term, host, prepare, ptr, sample_args, update_theta

pytestmark = pytest.mark.gpu
LL_RTOL = 1e-6  # the tolerance of the other sampler parity tests


def _run(fn, p, a):
    import torch

    p.d["z_out"].zero_()
    p.d["ll"].zero_()
    p.d["err"].zero_()
    assert fn(a) == _ffi.CULDA_OK, cb.lib().culda_last_error(None)
    torch.cuda.synchronize()
    ll = C.c_double()
    assert cb.lib().culda_loglik(ptr(p.d["ll"]), doc_term(p), p.corpus.num_tokens, C.byref(ll), None) == 0
    assert int(p.d["err"].item()) == 0
    return host(p.d["z_out"], np.uint16).copy(), ll.value


@pytest.mark.parametrize("group_lanes", [_ffi.CULDA_SAMPLER_FLAT, 8], ids=["flat", "g8"])
def test_noalloc_matches_workspace_sampler_twice(group_lanes):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = cb.lib()
    c = cb.Corpus.generate(MINI.gen)
    k = MINI.k
    p = prepare(c, k, MINI.alpha, MINI.beta, O.init_topics(c.num_tokens, k, 8), item_tokens=200)
    assert p.num_hot > 0  # the hot-row part of the scratch is exercised too
    assert update_theta(p) == 0
    a = sample_args(p, seed=77, iteration=5, group_lanes=group_lanes)
    need = lib.culda_sample_workspace(k, p.num_items, p.num_hot)
    assert need <= _ffi.CULDA_NOALLOC_SCRATCH_BYTES
    ws = torch.zeros(need // 4 + 64, dtype=torch.int32, device="cuda")

    z_ref, ll_ref = _run(lambda x: lib.culda_sample(C.byref(x), ptr(ws), ws.numel() * 4, None), p, a)
    for _ in range(2):
        z, ll = _run(lambda x: lib.culda_sample_noalloc(C.byref(x), None), p, a)
        assert np.array_equal(z, z_ref)
        assert abs(ll - ll_ref) <= LL_RTOL * max(1.0, abs(ll_ref))


def test_noalloc_rejects_work_lists_beyond_the_array():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = cb.lib()
    a = _ffi.SampleArgs(k=1024, num_items=2_000_000, num_hot=0)
    assert lib.culda_sample_workspace(1024, 2_000_000, 0) > _ffi.CULDA_NOALLOC_SCRATCH_BYTES
    assert lib.culda_sample_noalloc(C.byref(a), None) == _ffi.CULDA_ERR_UNSUPPORTED
    assert b"fixed device array" in lib.culda_last_error(None)


def test_noalloc_rejects_malformed_sizes():
    """Negative sizes are argument errors, not oversize work lists."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = cb.lib()
    for kw in ({"k": 1024, "num_items": -1, "num_hot": 0}, {"k": 1024, "num_items": 10, "num_hot": -5},
               {"k": -32, "num_items": 10, "num_hot": 0}):
        a = _ffi.SampleArgs(**kw)
        assert lib.culda_sample_noalloc(C.byref(a), None) == _ffi.CULDA_ERR_INVALID_ARG, kw
