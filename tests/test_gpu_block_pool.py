"""Context blocks come from a per-device pool that keeps them reserved:
repeated create/destroy cycles reuse the memory and every context still
starts from the same state; culda_trim_memory hands the reserve back."""
import pytest

import culda_cgs_b200 as cb
from culda_cgs_b200 import _ffi
from culda_cgs_b200.configs import MINI

pytestmark = pytest.mark.gpu


def test_recreated_contexts_match_and_trim_releases():
    c = cb.Corpus.generate(MINI.gen)
    runs = []
    for _ in range(3):
        with cb.LDA(c, 256, 50.0 / 256, 0.01, seed=5) as m:
            st = m.iterate(2)
            runs.append((m.topics().copy(), st[-1]["loglik"]))
    for z, ll in runs[1:]:
        assert (z == runs[0][0]).all() and ll == runs[0][1]
    assert cb.lib().culda_trim_memory(0) == _ffi.CULDA_OK
    assert cb.lib().culda_trim_memory(-1) == _ffi.CULDA_ERR_INVALID_ARG
    with cb.LDA(c, 256, 50.0 / 256, 0.01, seed=5) as m:  # a fresh block after the trim
        m.iterate(2)
        assert (m.topics() == runs[0][0]).all()
