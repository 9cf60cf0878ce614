"""Seeded synthetic inputs: T-layout antenna positions and 4-bit voltage
pages with dispersed point-source bursts.

Voltages: complex Gaussian sigma per component, ``rint``, clipped to
[-8, 7], packed one byte per complex sample (low nibble real, high nibble
imag) in the on-wire order ``(pkt, ant, chan, t, pol)`` of each chgroup
page (src/dsart/common/constants.py:350-361).

Bursts (model after src/dsart/inject/online.py:325-560): a constant complex
amplitude per antenna and channel, on for ``width`` native samples starting
at ``t0 + K*DM*(nu^-2 - nu_top^-2)``, phased so that the source lands at image
offset ``(dl, dm)`` pixels from the image centre under the gridder's
conventions (V_ab = conj(E_b) E_a, u = -(e_a - e_b)/lambda, row = v).
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Sequence

import numpy as np
import torch

from .constants import K_DM_MS_GHZ2_PC, NATIVE_SAMPLE_US, SPEED_OF_LIGHT_M_S, Band


def t_layout(nants: int, seed: int, ew_m: float = 2600.0, ns_m: float = 1600.0):
    """Seeded T layout: 60% of the antennas on the EW arm, the rest south
    along the NS arm (metres, east and north offsets)."""
    rng = np.random.default_rng(seed)
    n_ew = int(round(nants * 0.6))
    e = np.empty(nants)
    n = np.empty(nants)
    e[:n_ew] = np.sort(rng.uniform(-ew_m / 2, ew_m / 2, n_ew))
    n[:n_ew] = rng.normal(0.0, 2.0, n_ew)
    n[n_ew:] = -np.sort(rng.uniform(5.0, ns_m, nants - n_ew))
    e[n_ew:] = rng.normal(0.0, 2.0, nants - n_ew)
    return e, n


@dataclass
class Burst:
    dm: float            # pc cm^-3
    t0_native: int       # arrival sample at the band top (absolute, from stream start)
    width_native: int    # native samples
    amp: float           # complex amplitude added to each voltage sample
    dl: int = 0          # image row offset from the centre (pixels)
    dm_pix: int = 0      # image column offset from the centre (pixels)


def _pack(re: np.ndarray, im: np.ndarray) -> np.ndarray:
    return ((re.astype(np.int16) & 0xF) | ((im.astype(np.int16) & 0xF) << 4)).astype(np.uint8)


def make_block(*, band: Band, nant: int, npkt: int, block_index: int, seed: int,
               antpos_e=None, antpos_n=None, bursts: Sequence[Burst] = (),
               cell_lambda: float = 1.0, n_grid: int = 64, sigma: float = 3.0) -> np.ndarray:
    """One block of raw pages ``(G, npkt, nant, nchan, 2, 2)`` uint8."""
    G, C = band.n_chgroup, band.nchan
    rng = np.random.default_rng([seed, block_index])
    shape = (G, npkt, nant, C, 2, 2)
    re = rng.normal(0.0, sigma, shape)
    im = rng.normal(0.0, sigma, shape)
    if bursts:
        nu = band.freq_table()                                   # (G, C) GHz
        nu_top = float(nu[0, 0])
        s0 = block_index * npkt * 2
        # native sample index of (pkt, t): s0 + 2*pkt + t
        samp = s0 + 2 * np.arange(npkt)[:, None] + np.arange(2)[None, :]      # (npkt, 2)
        for b in bursts:
            delay = K_DM_MS_GHZ2_PC * b.dm * (1.0 / nu ** 2 - 1.0 / nu_top ** 2) * 1e3 \
                / NATIVE_SAMPLE_US                                    # (G, C) native samples
            start = b.t0_native + np.rint(delay).astype(np.int64)
            on = (samp[None, None] >= start[:, :, None, None]) & \
                 (samp[None, None] < start[:, :, None, None] + b.width_native)   # (G, C, npkt, 2)
            if not on.any():
                continue
            wl = SPEED_OF_LIGHT_M_S / (nu * 1e9)                      # (G, C)
            scale = 1.0 / (cell_lambda * n_grid)
            ph = 2 * np.pi * scale * (np.asarray(antpos_n)[:, None, None] * b.dl
                                      + np.asarray(antpos_e)[:, None, None] * b.dm_pix) / wl[None]
            amp = b.amp * np.exp(1j * ph)                             # (nant, G, C)
            gi, ci, pi, ti = np.nonzero(on)
            for pol in range(2):
                a = amp[:, gi, ci]                                    # (nant, n_on)
                re[gi, pi, :, ci, ti, pol] += a.real.T
                im[gi, pi, :, ci, ti, pol] += a.imag.T
    re = np.clip(np.rint(re), -8, 7)
    im = np.clip(np.rint(im), -8, 7)
    return _pack(re, im)


def random_block_device(*, band: Band, nant: int, npkt: int, device, seed: int,
                        sigma: float = 3.0) -> torch.Tensor:
    """Large noise-only block generated on the GPU (same distribution as
    ``make_block`` without bursts; not bit-identical to it)."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    shape = (band.n_chgroup, npkt, nant, band.nchan, 2, 2)
    out = torch.empty(shape, dtype=torch.uint8, device=device)
    flat = out.view(-1)
    step = 1 << 28
    for i in range(0, flat.numel(), step):
        n = min(step, flat.numel() - i)
        re = torch.randn(n, generator=g, device=device).mul_(sigma).round_().clamp_(-8, 7)
        im = torch.randn(n, generator=g, device=device).mul_(sigma).round_().clamp_(-8, 7)
        flat[i:i + n] = ((re.to(torch.int16) & 0xF) | ((im.to(torch.int16) & 0xF) << 4)).to(torch.uint8)
    return out
