"""Host logic of the detector's candidate buffer (no GPU): the timeout mark
that the TMA-staged detector leaves in count[1] raises instead of reading as
an S/N."""

import pytest
import torch

from dsb200 import _lib
from dsb200.search import CandidateBuffer


def test_timeout_mark_raises_on_fetch():
    buf = CandidateBuffer("cpu", capacity=8)
    buf.count[1] = CandidateBuffer.TIMEOUT_BITS
    with pytest.raises(_lib.DsbError, match="timed out"):
        buf.fetch()
    with pytest.raises(_lib.DsbError, match="timed out"):
        buf.fetch_top(4)


def test_no_mark_reads_normally():
    buf = CandidateBuffer("cpu", capacity=8)
    assert buf.fetch().size == 0
    assert buf.fetch_top(4).size == 0
    # the bits of a large finite S/N are below the mark
    assert int(torch.tensor([1e30], dtype=torch.float32).view(torch.int32)) < \
        CandidateBuffer.TIMEOUT_BITS
