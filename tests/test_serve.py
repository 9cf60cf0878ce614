"""Serving several streams on one device: admission by a byte budget,
per-stream order, error reporting (CPU, with stand-in pipelines), and on a
GPU each stream's candidates alone and in the mix."""

import threading
import time

import numpy as np
import pytest
import torch

from dsb200.serve import DeviceBudget, StreamServer


class _FakePipe:
    """Stand-in with the SearchPipeline surface the server uses."""

    def __init__(self, delay=0.002, fail_at=None):
        self.dev = torch.device("cpu")
        self.delay = delay
        self.fail_at = fail_at
        self.seen = 0
        self.state = 0

    def block_packets(self, raw):
        if raw.dtype != torch.uint8 or raw.dim() != 6:
            raise ValueError("bad block")
        return raw.shape[1]

    def process_block(self, raw):
        if self.fail_at is not None and self.seen == self.fail_at:
            raise RuntimeError("stream failed")
        self.seen += 1
        time.sleep(self.delay)
        # depends on this stream's history only, like the real pipeline
        self.state = (self.state * 31 + int(raw.sum())) % 1000003
        return [self.state]


def _blocks(seed, n):
    rng = np.random.default_rng(seed)
    return [torch.from_numpy(rng.integers(0, 255, (2, int(rng.integers(1, 4)) * 4, 3, 2, 2, 2),
                                          dtype=np.uint8)) for _ in range(n)]


def test_budget_admits_within_capacity():
    b = DeviceBudget(100)
    with pytest.raises(ValueError):
        b.acquire(101)
    b.acquire(60)
    with pytest.raises(TimeoutError):
        b.acquire(50, timeout=0.05)
    done = []

    def late():
        b.acquire(50)
        done.append(True)

    th = threading.Thread(target=late)
    th.start()
    time.sleep(0.05)
    assert not done
    b.release(60)
    th.join(2)
    assert done and b.used == 50 and b.peak <= 100
    b.release(50)
    with pytest.raises(RuntimeError):
        b.release(1)


def test_streams_alone_and_mixed_agree():
    streams = [_blocks(s, 6) for s in range(3)]
    alone = []
    for bl in streams:
        p = _FakePipe()
        alone.append([p.process_block(x) for x in bl])
    pipes = [_FakePipe() for _ in streams]
    budget = 2 * max(x.numel() for bl in streams for x in bl)
    srv = StreamServer(pipes, budget).start()
    for k in range(6):                      # interleaved arrivals
        for i, bl in enumerate(streams):
            srv.submit(i, bl[k])
    srv.close()
    srv.join(30)
    for i in range(3):
        assert [r.index for r in srv.results[i]] == list(range(6))
        assert [r.candidates for r in srv.results[i]] == alone[i]
        assert all(r.t_done >= r.t_admit >= r.t_arrival for r in srv.results[i])
    assert srv.budget.peak <= budget and srv.budget.used == 0


def test_prepare_hook_sees_each_block_once_in_order():
    """prepare(stream, block index, device block) runs before the search on
    a private copy: the caller's blocks stay unchanged, and the pipeline sees
    the prepared block."""
    streams = [_blocks(s, 4) for s in range(2)]
    orig = [[x.clone() for x in bl] for bl in streams]
    seen = []

    def prepare(i, k, blk):
        seen.append((i, k))
        blk.view(-1)[0] = 7
    pipes = [_FakePipe(delay=0.0) for _ in streams]
    srv = StreamServer(pipes, 1 << 20, prepare=prepare).start()
    for k in range(4):
        for i, bl in enumerate(streams):
            srv.submit(i, bl[k])
    srv.close()
    srv.join(30)
    assert sorted(seen) == [(i, k) for i in range(2) for k in range(4)]
    for i in range(2):
        assert [k for j, k in seen if j == i] == list(range(4))
        assert all(torch.equal(a, b) for a, b in zip(streams[i], orig[i]))
        want = _FakePipe()
        exp = []
        for x in orig[i]:
            y = x.clone()
            y.view(-1)[0] = 7
            exp.append(want.process_block(y))
        assert [r.candidates for r in srv.results[i]] == exp


def test_stream_error_is_reported():
    pipes = [_FakePipe(), _FakePipe(fail_at=1)]
    srv = StreamServer(pipes, 1 << 20).start()
    for k in range(3):
        for i in range(2):
            srv.submit(i, _blocks(k, 1)[0])
    srv.close()
    with pytest.raises(RuntimeError, match="stream failed"):
        srv.join(30)
    assert len(srv.results[0]) == 3 and len(srv.results[1]) == 1
    with pytest.raises(ValueError):
        srv.submit(0, torch.zeros(5, dtype=torch.uint8))


@pytest.mark.gpu
def test_served_streams_match_alone():
    """Three streams (different seeds, uneven blocks of 1-3 chunks) served
    together under a budget of two blocks give each stream exactly the
    candidates it gives alone: same (time, fine DM, pixel, width) and the
    same S/N bits.  Every stage is order-independent (integer sums, the
    image combine's fixed-point atomics), so serving in a mix changes
    nothing."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dsb200 import synth
    from dsb200.constants import band_from_edges
    from dsb200.pipeline import PipelineConfig, SearchPipeline
    dev = torch.device("cuda", 0)
    band = band_from_edges(2, 32, 1.49875, 1.31125)
    nant, N, C = 16, 64, 32
    e, n = synth.t_layout(nant, seed=5)

    def cfg():
        return PipelineConfig(band=band, nant=nant, npkt_block=4 * C, t_int=8, csf=4,
                              n_grid=N, coarse_dm=np.linspace(0, 30, 4), fine_per_coarse=2,
                              log_max_width=2, threshold=6.0, sky_window=2, sky_warmup=1,
                              chunk_tiles=C, fdm_batch=3)

    import dsb_oracle as O
    ob = O.Band(band.n_chgroup, band.nchan, band.f0_ghz, band.dnu_ghz, band.ch0)
    cell = O.top_of_band_cell_lambda(e, n, ob, N)
    per_chunk = C * 4                         # packets per chunk (t_int 8)
    rng = np.random.default_rng(12)
    streams = []
    for s in range(3):
        # one continuous 16-chunk stream with a burst, cut into blocks of 1-3 chunks
        full = synth.make_block(band=band, nant=nant, npkt=16 * per_chunk, block_index=0,
                                seed=40 + s, antpos_e=e, antpos_n=n, cell_lambda=cell,
                                n_grid=N, bursts=[synth.Burst(dm=20.0, t0_native=1200 + 200 * s,
                                                              width_native=16, amp=1.5,
                                                              dl=2 - s, dm_pix=-4)])
        bl, c0 = [], 0
        while c0 < 16:
            k = min(int(rng.integers(1, 4)), 16 - c0)
            bl.append(torch.from_numpy(np.ascontiguousarray(
                full[:, c0 * per_chunk:(c0 + k) * per_chunk])))
            c0 += k
        streams.append(bl)
    alone = []
    for bl in streams:
        p = SearchPipeline(cfg(), e, n, device=dev)
        got = []
        for x in bl:
            got += p.process_block(x.to(dev))
        torch.cuda.synchronize()
        p.check_status()
        alone.append(got)
    pipes = [SearchPipeline(cfg(), e, n, device=dev) for _ in streams]
    budget = 2 * max(x.numel() for bl in streams for x in bl)
    srv = StreamServer(pipes, budget).start()
    for k in range(max(len(bl) for bl in streams)):
        for i, bl in enumerate(streams):
            if k < len(bl):
                srv.submit(i, bl[k].pin_memory())
    srv.close()
    srv.join(600)
    for p in pipes:
        p.check_status()
    assert srv.budget.peak <= budget
    n_cands = 0
    for i in range(3):
        mixed = [c for r in srv.results[i] for c in r.candidates]
        key = lambda c: (c.t, c.fdm, c.l, c.m, c.width)  # noqa: E731
        a = {key(c): c.snr for c in alone[i]}
        m = {key(c): c.snr for c in mixed}
        assert a == m, (i, sorted(set(a) ^ set(m)))
        n_cands += len(a)
    assert n_cands >= 1
