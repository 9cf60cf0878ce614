"""Stress/recovery sweep: bursts on an amplitude x width x DM grid, injected
into one continuous stream.

* CPU: the sweep helpers (grid, amplitude rule, matching).
* GPU, reduced sweep (16 antennas, two chgroups of 32 channels, 64^2, ten
  fine DMs 0-40, boxcars 1..8): the pipeline's candidate list equals the
  oracle's on the same seeds (identical keys, S/N within 1e-5 relative,
  the epsilon band of the pipeline tests), the same bursts are recovered by
  both, and every burst of the strongest amplitude is recovered.
"""

import types

import numpy as np
import pytest
import torch

from dsb200 import synth


def test_burst_grid_and_amplitude_rule():
    g = synth.burst_grid(snrs=[6, 50], widths=[32, 1024], dms=[0.0, 3000.0],
                         t_first_native=100, spacing_native=1000, n_grid=512, seed=2)
    assert len(g) == 8
    assert sorted((s, w, d) for s, w, d, *_ in g) == sorted(
        (float(s), w, float(d)) for s in (6, 50) for w in (32, 1024) for d in (0.0, 3000.0))
    assert [t0 for _, _, _, t0, _, _ in g] == [100 + 1000 * k for k in range(8)]
    assert all(abs(dl) <= 248 and abs(dm) <= 248 for *_, dl, dm in g)
    # S/N ~ amp^2 sqrt(width): four times the S/N at the same width = twice the amplitude
    a = synth.amp_for_snr(80, 128, amp_ref=0.1, snr_ref=20, width_ref=128)
    assert a == pytest.approx(0.2)
    # sixteen times the width at the same S/N = half the amplitude
    assert synth.amp_for_snr(20, 2048, amp_ref=0.1, snr_ref=20, width_ref=128) == pytest.approx(0.05)


def test_match_bursts_picks_the_best_nearby_candidate():
    C = types.SimpleNamespace
    fine = np.array([0.0, 10.0, 20.0, 30.0])
    bursts = [(10.0, 32, 20.0, 3200, 3, -5), (10.0, 32, 30.0, 9600, -7, 2)]
    cands = [C(t=100, fdm=2, l=35, m=27, snr=9.0, width=1),
             C(t=101, fdm=2, l=36, m=27, snr=12.0, width=2),     # best of burst 0
             C(t=100, fdm=0, l=35, m=27, snr=30.0, width=1),     # DM too far
             C(t=400, fdm=3, l=25, m=34, snr=8.0, width=1)]      # time too far for burst 1
    from dsb200.constants import band_from_edges
    band = band_from_edges(2, 32, 1.49875, 1.31125)
    nu = band.freq_table()
    k_bot = 4.148808 * (1 / nu.min() ** 2 - 1 / nu[0, 0] ** 2) * 1e3 / 32.768   # samples per DM
    cands[0].t = cands[1].t = round((3200 + k_bot * 20.0) / 32)
    cands[2].t = cands[0].t
    got = synth.match_bursts(bursts, cands, band=band, fine_dm=fine, n_grid=64, t_int=32,
                             r_t=4, dm_abs=5.0)
    assert got[0] is cands[1] and got[1] is None


@pytest.mark.gpu
def test_reduced_stress_sweep_matches_oracle():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import dsb_oracle as O
    from test_pipeline_gpu import compare_candidates
    from dsb200.constants import band_from_edges
    from dsb200.pipeline import PipelineConfig, SearchPipeline
    dev = torch.device("cuda", 0)
    band = band_from_edges(2, 32, 1.49875, 1.31125)
    ob = O.Band(band.n_chgroup, band.nchan, band.f0_ghz, band.dnu_ghz, band.ch0)
    nant, npkt, N, t_int = 16, 256, 64, 8
    e, n = synth.t_layout(nant, seed=5)
    cell = O.top_of_band_cell_lambda(e, n, ob, N)
    coarse = np.linspace(0.0, 40.0, 5)
    off = np.array([-2.5, 2.5])
    fine = np.maximum((coarse[:, None] + off[None]).reshape(-1), 0.0)
    f2c = np.repeat(np.arange(5), 2)
    amps = [0.5, 1.0, 2.0]
    grid = synth.burst_grid(snrs=amps, widths=[8, 32], dms=[10.0, 35.0], t_first_native=1024,
                            spacing_native=600, n_grid=N, seed=3, margin=6)
    bursts = [synth.Burst(dm=d, t0_native=t0, width_native=w, amp=a, dl=dl, dm_pix=dp)
              for a, w, d, t0, dl, dp in grid]
    n_blocks = 20
    blocks = [synth.make_block(band=band, nant=nant, npkt=npkt, block_index=b, seed=17,
                               antpos_e=e, antpos_n=n, bursts=bursts, cell_lambda=cell, n_grid=N)
              for b in range(n_blocks)]
    kw = dict(nant=nant, npkt_block=npkt, t_int=t_int, csf=4, n_grid=N, coarse_dm=coarse,
              fine_dm=fine, fine_to_coarse=f2c, log_max_width=3, threshold=7.0)
    cfg = PipelineConfig(band=band, sky_window=2, sky_warmup=1, chunk_tiles=32, fdm_batch=5,
                         **kw)
    pipe = SearchPipeline(cfg, e, n, device=dev)
    got = []
    for b in blocks:
        got += pipe.process_block(torch.from_numpy(b).to(dev))
    torch.cuda.synchronize()
    pipe.check_status()
    want = O.run_pipeline(blocks, ob, e, n, chunk=32, sky_window=2, sky_warmup=1,
                          keep_images=False, **kw)
    compare_candidates(got, want, threshold=7.0)
    as_obj = [types.SimpleNamespace(t=c[0], fdm=c[1], l=c[2], m=c[3], snr=c[4], width=c[5])
              for c in want]
    m_gpu = synth.match_bursts(grid, got, band=band, fine_dm=fine, n_grid=N, t_int=t_int,
                               dm_abs=6.0)
    m_orc = synth.match_bursts(grid, as_obj, band=band, fine_dm=fine, n_grid=N, t_int=t_int,
                               dm_abs=6.0)
    assert [m is None for m in m_gpu] == [m is None for m in m_orc]
    strongest = [m for m, b in zip(m_gpu, grid) if b[0] == max(amps)]
    assert all(m is not None for m in strongest), grid
    print("recovered:", sum(m is not None for m in m_gpu), "of", len(grid))
