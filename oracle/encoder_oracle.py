"""TEST INFRASTRUCTURE ONLY: FP64 restatement of the document encoder.

The network (embedding bag over word ids -> GELU(W1 x + b1) -> GELU(W2 h + b2)
-> softmax(W3 h + b3)), its cross-entropy against a target distribution and
the gradients of every weight, in float64 numpy.  With `rounding=True` the
values are rounded to BF16 exactly where the CUDA path stores BF16 (weights,
the bag mean, both activations, and the three back-propagated signals that feed
a GEMM), so the two differ only by FP32 accumulation order and by operands
that land on the other side of a BF16 rounding boundary.  With
`rounding=False` it is a plain FP64 network, whose gradients are checked
against finite differences.  The encoder has no counterpart in CuLDA_CGS.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import erf


def bf16(x) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), through FP32, returned as float64."""
    f = np.ascontiguousarray(np.asarray(x, dtype=np.float64).astype(np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


NAMES = ("E", "W1", "b1", "W2", "b2", "W3", "b3")


class EncoderOracle:
    def __init__(self, tensors: dict):
        self.t = {k: np.asarray(tensors[k], dtype=np.float64) for k in NAMES}

    def bag(self, doc_ptr, words, docs, E):
        rows = []
        for d in docs:
            w = words[doc_ptr[d]:doc_ptr[d + 1]]
            rows.append(E[w].mean(0) if len(w) else np.zeros(E.shape[1]))
        return np.array(rows)

    def run(self, doc_ptr, words, docs, target=None, rounding=True):
        R = bf16 if rounding else (lambda x: np.asarray(x, dtype=np.float64))
        t = self.t
        E, W1, W2, W3 = R(t["E"]), R(t["W1"]), R(t["W2"]), R(t["W3"])
        X0 = R(self.bag(doc_ptr, words, docs, E))
        P1 = X0 @ W1.T + t["b1"]
        H1 = R(gelu(P1))
        P2 = H1 @ W2.T + t["b2"]
        H2 = R(gelu(P2))
        Z = H2 @ W3.T + t["b3"]
        m = Z.max(1, keepdims=True)
        lse = m + np.log(np.exp(Z - m).sum(1, keepdims=True))
        q = np.exp(Z - lse)
        out = {"q": q}
        if target is None:
            return out
        B = len(docs)
        out["loss"] = float((target * (lse - Z)).sum() / B)
        G = (q - target) / B
        dZ = R(G)
        g = {"b3": G.sum(0), "W3": dZ.T @ H2}
        gp2 = (dZ @ W3) * gelu_grad(P2)
        g["b2"] = gp2.sum(0)
        dP2 = R(gp2)
        g["W2"] = dP2.T @ H1
        gp1 = (dP2 @ W2) * gelu_grad(P1)
        g["b1"] = gp1.sum(0)
        dP1 = R(gp1)
        g["W1"] = dP1.T @ X0
        dX0 = dP1 @ W1
        gE = np.zeros_like(t["E"])
        for b, d in enumerate(docs):
            w = words[doc_ptr[d]:doc_ptr[d + 1]]
            if len(w):
                np.add.at(gE, w, dX0[b] / len(w))
        g["E"] = gE
        out["grads"] = g
        return out

    def loss(self, doc_ptr, words, docs, target):
        return self.run(doc_ptr, words, docs, target, rounding=False)["loss"]


def random_batch(rng, num_words, num_docs, max_len):
    """A CSR batch of docs with 1..max_len tokens (word ids in [0, num_words))."""
    lens = rng.integers(1, max_len + 1, size=num_docs)
    doc_ptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    words = rng.integers(0, num_words, size=int(doc_ptr[-1])).astype(np.int32)
    return doc_ptr, words


def random_target(rng, num_docs, k, conc=0.1):
    return rng.dirichlet(np.full(k, conc), size=num_docs)


def random_tensors(rng, num_words, k, embed=256, hidden=512):
    return {"E": rng.uniform(-0.5, 0.5, (num_words, embed)),
            "W1": rng.uniform(-1, 1, (hidden, embed)) * math.sqrt(6.0 / (embed + hidden)),
            "b1": rng.normal(0, 0.1, hidden),
            "W2": rng.uniform(-1, 1, (hidden, hidden)) * math.sqrt(6.0 / (2 * hidden)),
            "b2": rng.normal(0, 0.1, hidden),
            "W3": rng.uniform(-1, 1, (k, hidden)) * math.sqrt(6.0 / (hidden + k)),
            "b3": rng.normal(0, 0.1, k)}
