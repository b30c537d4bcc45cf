"""The kernel-level C entry points (one per reference kernel API) on device
buffers, against the oracle: culda_update_phi (LDAUpdatePhiAPI),
culda_compute_phi_head (LDAComputePhiHeadAPI), culda_update_theta
(LDAUpdateThetaAPI), culda_sample + culda_loglik (LDAKernelTrain +
LDATrainPerplexity)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import culda_cgs_b200 as cb
from culda_cgs_b200 import _ffi
from culda_cgs_b200.configs import MINI, TINY
from oracle import oracle as O

from kernel_api import dev, doc_term, host, prepare, ptr, sample_args, update_theta

pytestmark = pytest.mark.gpu
BOUNDARY_TOL = 1e-6


@pytest.fixture(scope="module", params=[("tiny", TINY, 64), ("mini", MINI, 1024)], ids=lambda p: p[0])
def problem(request):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    _, wl, k = request.param
    c = cb.Corpus.generate(wl.gen)
    z = O.init_topics(c.num_tokens, k, 4)
    p = prepare(c, k, wl.alpha, wl.beta, z)
    s = O.Snapshot.build(c.word_ptr, c.doc_ids, c.doc_ptr, z, k, wl.alpha, wl.beta)
    return p, s


def test_update_phi_and_phi_head(problem):
    import torch

    p, s = problem
    c = p.corpus
    phi = torch.zeros(c.num_words * p.k, dtype=torch.int32, device="cuda")
    nk = torch.zeros(p.k, dtype=torch.int32, device="cuda")
    lib = cb.lib()
    assert lib.culda_update_phi(p.k, c.num_words, ptr(p.d["word_ptr"]), ptr(p.d["z"]), ptr(phi), ptr(nk), None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(host(phi, np.int32).reshape(c.num_words, p.k), s.phi)
    assert np.array_equal(host(nk, np.int32), s.nk)
    head = torch.zeros(c.num_words * p.k, dtype=torch.float32, device="cuda")
    assert lib.culda_compute_phi_head(p.k, p.beta, c.num_words, ptr(phi), ptr(nk), ptr(head), None) == 0
    torch.cuda.synchronize()
    h = head.cpu().numpy().reshape(c.num_words, p.k)
    # the reference's float quotient (lda_phi_kernel.cu:26) ...
    b = np.float32(p.beta)
    want = (s.phi.astype(np.float32) + b) / (s.nk.astype(np.float32) + b * np.float32(c.num_words))
    assert np.array_equal(h, want)
    # ... and its FP16 rounding is the reference's phiHead table
    assert np.array_equal(h.astype(np.float16).view(np.uint16), O.phi_head_f16(c.num_words, p.k, p.beta, s.phi, s.nk))


def test_update_theta(problem):
    import torch

    p, s = problem
    assert update_theta(p) == 0
    torch.cuda.synchronize()
    t = host(p.d["theta"], np.uint32)
    assert np.array_equal((t & 0xFFFF).astype(np.int16), s.theta_a)
    assert np.array_equal((t >> 18).astype(np.int16), s.theta_ja)
    assert ((t >> 16) & 3 == 0).all()
    rows = host(p.d["rows"], np.int32).reshape(-1, 2)
    assert np.array_equal(rows[:, 0], s.max_ia[:-1]) and np.array_equal(rows[:, 1], s.cur_ia)
    assert np.array_equal(host(p.d["nk"], np.int32), s.nk)
    L = np.diff(s.doc_ptr)
    stats = host(p.d["stats"], np.int64)
    assert stats[0] == int((L * (s.cur_ia - s.max_ia[:-1])).sum())
    assert stats[1] == int((s.theta_a != 0).sum())
    assert int(host(p.d["ws_theta"], np.int32)[0]) == 0


@pytest.mark.parametrize("g", [1, 8, 32, -1])
def test_sample_and_loglik(problem, g):
    import torch

    p, s = problem
    assert update_theta(p) == 0
    lib = cb.lib()
    a = sample_args(p, seed=13, iteration=9, group_lanes=g)
    ws_bytes = lib.culda_sample_workspace(p.k, p.num_items, p.num_hot)
    ws = torch.zeros(ws_bytes // 4 + 64, dtype=torch.int32, device="cuda")
    p.d["err"].zero_()
    assert lib.culda_sample(C.byref(a), ptr(ws), ws.numel() * 4, None) == 0
    ll = C.c_double()
    assert lib.culda_loglik(ptr(p.d["ll"]), doc_term(p), p.corpus.num_tokens, C.byref(ll), None) == 0
    z_gpu = host(p.d["z_out"], np.uint16)
    z_ora, margin, ll_ora = s.sample(13, 9)
    far = margin >= BOUNDARY_TOL
    assert np.array_equal(z_gpu[far], z_ora[far])
    assert abs(ll.value - ll_ora) <= 1e-6 * max(1.0, abs(ll_ora))
    assert int(p.d["err"].item()) == 0


def test_sample_rejects_out_of_range_theta(problem):
    import torch

    p, s = problem
    assert update_theta(p) == 0
    theta = p.d["theta"].clone()
    theta[0] = (p.k << 18) | 1  # topic K: one past the last valid topic
    lib = cb.lib()
    a = sample_args(p, seed=1, iteration=1)
    a.theta = ptr(theta)
    ws = torch.zeros(lib.culda_sample_workspace(p.k, p.num_items, p.num_hot) // 4 + 64, dtype=torch.int32,
                     device="cuda")
    assert lib.culda_sample(C.byref(a), ptr(ws), ws.numel() * 4, None) == _ffi.CULDA_ERR_INVALID_ARG
    assert b"out of range" in lib.culda_last_error(None)
