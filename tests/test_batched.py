"""The batched form: uneven channel groups with their own sub-arrays and DM
plans, advanced block by block as one captured CUDA graph, give exactly the
per-group plain runs' candidates; the configuration's geometry (CPU)."""

import numpy as np
import pytest
import torch


def test_config3_groups_cover_the_band():
    from dsb200.batched import config3_groups
    g = config3_groups()
    chans = [cfg.band.n_chgroup * cfg.band.nchan for cfg, _, _ in g]
    assert chans == [512, 768, 1024, 1024, 1280, 1536] and sum(chans) == 6144
    assert [cfg.nant for cfg, _, _ in g] == [96, 96, 64, 64, 48, 48]
    assert [cfg.fine_dm.size for cfg, _, _ in g] == [128, 256, 512, 512, 768, 1024]
    assert [cfg.coarse_dm.max() for cfg, _, _ in g] == [500.0, 1000.0, 1500.0, 2000.0,
                                                        2500.0, 3000.0]
    # contiguous channels: each group starts where the previous one ended
    f_next = g[0][0].band.f0_ghz
    for cfg, e, n in g:
        assert cfg.band.f0_ghz == pytest.approx(f_next, abs=1e-12)
        f_next = cfg.band.f0_ghz - cfg.band.n_chgroup * cfg.band.nchan * cfg.band.dnu_ghz
        assert cfg.chunk_tiles == cfg.n_fv_block          # one detector cube per block
        assert e.shape == n.shape == (cfg.nant,)
    assert f_next == pytest.approx(1.31125, abs=1e-9)
    # sub-arrays of one layout: the smaller arrays are its first antennas
    assert np.array_equal(g[4][1], g[0][1][:48]) and np.array_equal(g[2][2], g[0][2][:64])


def _groups():
    from dsb200 import synth
    from dsb200.constants import Band
    from dsb200.pipeline import PipelineConfig
    e, n = synth.t_layout(32, seed=5)
    dnu = (1.49875 - 1.31125) / 192
    plan = [(1, 16, np.linspace(0, 30, 4), 2), (2, 32, np.linspace(0, 45, 3), 4),
            (3, 16, np.linspace(0, 60, 5), 2)]
    out, ch0 = [], 0
    for ng, na, cdm, k in plan:
        band = Band(n_chgroup=ng, nchan=32, f0_ghz=1.49875 - ch0 * dnu, dnu_ghz=dnu, ch0=0)
        cfg = PipelineConfig(band=band, nant=na, npkt_block=128, t_int=8, csf=4, n_grid=64,
                             coarse_dm=cdm, fine_per_coarse=k, log_max_width=2, threshold=6.0,
                             sky_window=2, sky_warmup=1, chunk_tiles=32, fdm_batch=3)
        out.append((cfg, e[:na].copy(), n[:na].copy()))
        ch0 += ng * 32
    return out


@pytest.mark.gpu
def test_batched_graph_equals_plain_runs():
    """Three groups (1, 2, 3 chgroups; 16, 32, 16 antennas; 8, 12, 10 fine
    DMs), each stream carrying a burst, 14 blocks: every block's candidates
    from the graph-batched run equal the group's plain run bit for bit
    (time, fine DM, pixel, width and the S/N's float bits), with the
    Layer-2 state carried across blocks in both."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import dsb_oracle as O
    from dsb200 import synth
    from dsb200.batched import BatchedSearch
    from dsb200.pipeline import SearchPipeline
    dev = torch.device("cuda", 0)
    groups = _groups()
    nblk = 14
    streams = []
    for i, (cfg, e, n) in enumerate(groups):
        b = cfg.band
        ob = O.Band(b.n_chgroup, b.nchan, b.f0_ghz, b.dnu_ghz, b.ch0)
        cell = O.top_of_band_cell_lambda(e, n, ob, 64)
        full = synth.make_block(band=b, nant=cfg.nant, npkt=nblk * cfg.npkt_block, block_index=0,
                                seed=60 + i, antpos_e=e, antpos_n=n, cell_lambda=cell, n_grid=64,
                                bursts=[synth.Burst(dm=20.0, t0_native=1300 + 150 * i,
                                                    width_native=16, amp=1.5, dl=2 - i,
                                                    dm_pix=-3)])
        streams.append([torch.from_numpy(np.ascontiguousarray(
            full[:, k * cfg.npkt_block:(k + 1) * cfg.npkt_block])).to(dev) for k in range(nblk)])
    plain = []
    for (cfg, e, n), bl in zip(groups, streams):
        p = SearchPipeline(cfg, e, n, device=dev)
        plain.append([[tuple(vars(c).values()) for c in p.process_block(x)] for x in bl])
        torch.cuda.synchronize()
        p.check_status()
    bs = BatchedSearch(groups, device=dev)
    got = [[] for _ in groups]
    for k in range(nblk):
        res = bs.process_block([bl[k] for bl in streams])
        for i, r in enumerate(res):
            got[i].append([tuple(vars(c).values()) for c in r])
    torch.cuda.synchronize()
    bs.check_status()
    assert bs.graph_launches == nblk
    for i in range(len(groups)):
        assert got[i] == plain[i], i
    assert sum(len(b) for s in plain for b in s) >= 3
    bs.close()
