"""The batched form: several search groups on one GPU -- channel groups of
uneven size, each with its own sub-array of antennas and its own DM plan --
advanced block by block as ONE launch sequence captured in a CUDA graph.

Each group is a ``SearchPipeline`` over its own band (a run of the band's
channels split into chgroups), antennas and DM plan.  For every block the
device work of all groups (correlator, stage 1, the detector cube it
completes: images, Layer-1, detector, Layer-2 samples) is captured on one
stream (``dsb_graph_begin``) and launched as one graph
(``dsb_graph_end_launch``).  The graph of the next block has the same
launches with moved stream times, so the executable graph is updated in
place rather than rebuilt.  After the graph, each group's host work runs:
the Layer-2 update into its divisor buffer (which the next graph reads) and
the candidates' read-back and decode.  The results equal the groups' plain
runs (``SearchPipeline.process_block``) bit for bit: the same kernels on the
same arguments in the same order.

``autotune`` chooses each group's tile shapes (fine DMs per image /
detector launch, coarse DMs per stage-1 block) by timing the candidates on
that group's own geometry, and keeps the fastest.
"""

from __future__ import annotations

import dataclasses
import time
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from .pipeline import PipelineConfig, SearchPipeline, StreamCandidate


class BatchedSearch:
    """Search groups advanced together, one CUDA graph per block."""

    def __init__(self, groups: Sequence[Tuple[PipelineConfig, np.ndarray, np.ndarray]],
                 device="cuda", use_graph: bool = True):
        self.dev = _lib.cuda_device(device)
        self.pipes = [SearchPipeline(cfg, e, n, device=self.dev) for cfg, e, n in groups]
        for p in self.pipes:
            if p.cfg.chunk_tiles != p.cfg.n_fv_block:
                raise ValueError("batched groups run one chunk per block "
                                 "(chunk_tiles = the block's tiles)")
        self.use_graph = bool(use_graph)
        self.stream = torch.cuda.Stream(self.dev)
        self._exec = _lib.ctypes.c_void_p(None)
        self.graph_launches = 0

    def skip_warmup(self) -> None:
        for p in self.pipes:
            p.skip_warmup()

    def process_block(self, raws: Sequence[torch.Tensor], *, collect: bool = True
                      ) -> List[List[StreamCandidate]]:
        """One block of every group (``raws[i]`` the raw pages of group i,
        on the device): the groups' device work as one graph, then their host
        work.  Returns each group's candidates."""
        if len(raws) != len(self.pipes):
            raise ValueError(f"{len(raws)} blocks for {len(self.pipes)} groups")
        L = _lib.lib()
        cur = torch.cuda.current_stream(self.dev)
        self.stream.wait_stream(cur)
        with torch.cuda.stream(self.stream):
            h = _lib.ctypes.c_void_p(self.stream.cuda_stream)
            if self.use_graph:
                _lib.check(L.dsb_graph_begin(h), "dsb_graph_begin")
            cubes = []
            try:
                for p, raw in zip(self.pipes, raws):
                    cubes.append(p.device_block(raw))
            except BaseException:
                if self.use_graph:
                    L.dsb_graph_abort(h)
                raise
            if self.use_graph:
                _lib.check(L.dsb_graph_end_launch(h, _lib.ctypes.byref(self._exec)),
                           "dsb_graph_end_launch")
                self.graph_launches += 1
            out = [p.host_block(c, collect=collect) for p, c in zip(self.pipes, cubes)]
        cur.wait_stream(self.stream)
        return out

    def check_status(self) -> None:
        for p in self.pipes:
            p.check_status()

    def close(self) -> None:
        if self._exec.value:
            _lib.lib().dsb_graph_destroy(self._exec)
            self._exec = _lib.ctypes.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass


def autotune(cfg: PipelineConfig, antpos_e, antpos_n, *, device="cuda",
             fdm_batches: Sequence[int] = (4, 8, 16), dm_groups: Sequence[Optional[int]] = (None, 8),
             blocks: int = 2, seed: int = 0) -> Tuple[PipelineConfig, Dict]:
    """The project's tile-shape autotuner: for one group's geometry, time
    every (fdm_batch, stage1_dm_group) candidate that fits on ``blocks``
    seeded synthetic blocks in steady state (CUDA events, after one
    untimed block) and return the config with the fastest, and the table of
    times (ms per block; None for a candidate that does not fit)."""
    from . import synth
    dev = _lib.cuda_device(device)
    raw = synth.random_block_device(band=cfg.band, nant=cfg.nant, npkt=cfg.npkt_block,
                                    device=dev, seed=seed)
    times: Dict = {}
    best = None
    for fb in fdm_batches:
        for dg in dm_groups:
            c = dataclasses.replace(cfg, fdm_batch=int(fb), stage1_dm_group=dg)
            try:
                p = SearchPipeline(c, antpos_e, antpos_n, device=dev)
            except ValueError:
                times[(fb, dg)] = None              # the stage-1 window does not fit
                continue
            p.skip_warmup()
            p.process_block(raw, collect=False)
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(blocks):
                p.process_block(raw, collect=False)
            e1.record()
            torch.cuda.synchronize(dev)
            ms = e0.elapsed_time(e1) / blocks
            times[(fb, dg)] = ms
            if best is None or ms < best[0]:
                best = (ms, c)
            del p
            torch.cuda.empty_cache()
    if best is None:
        raise ValueError("no tile-shape candidate fits this group")
    return best[1], times


def config3_groups(*, npkt_block: int = 8192, t_int: int = 8, csf: int = 16, n_grid: int = 256,
                   chans=(512, 768, 1024, 1024, 1280, 1536), nants=(96, 96, 64, 64, 48, 48),
                   n_dms=(128, 256, 512, 512, 768, 1024),
                   max_dms=(500.0, 1000.0, 1500.0, 2000.0, 2500.0, 3000.0),
                   chgroup_chans: int = 256, seed: int = 11):
    """The batched configuration: the 1311.25-1498.75 MHz band cut into
    channel groups of uneven size (chgroups of ``chgroup_chans`` channels
    each), each group searched by one sub-array (its first ``nants[i]``
    antennas of a seeded T layout) over its own DM plan (``n_dms[i]`` trials,
    16 fine per coarse, 0..``max_dms[i]``); config 2's block, t_int, channel
    sum and 256^2 grid."""
    from . import synth
    from .constants import Band
    nchan_tot = 6144
    dnu = (1.49875 - 1.31125) / nchan_tot
    e_all, n_all = synth.t_layout(max(nants), seed=seed)
    groups = []
    ch0 = 0
    for nch, na, ndm, mx in zip(chans, nants, n_dms, max_dms):
        if nch % chgroup_chans:
            raise ValueError("group sizes must be whole chgroups")
        band = Band(n_chgroup=nch // chgroup_chans, nchan=chgroup_chans,
                    f0_ghz=1.49875 - ch0 * dnu, dnu_ghz=dnu, ch0=0)
        cfg = PipelineConfig(nant=na, band=band, npkt_block=npkt_block, t_int=t_int, csf=csf,
                             n_grid=n_grid, coarse_dm=np.linspace(0.0, mx, ndm // 16),
                             fine_per_coarse=16, log_max_width=4, threshold=7.0,
                             chunk_tiles=npkt_block * 2 // t_int, fdm_batch=8, ring_dtype="bf16")
        groups.append((cfg, e_all[:na].copy(), n_all[:na].copy()))
        ch0 += nch
    return groups
