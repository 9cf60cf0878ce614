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


def _burst_samples(band: Band, b: Burst, s0: int, n_samp: int):
    """(chgroup, channel, native sample) of every sample burst ``b`` covers in
    [s0, s0 + n_samp), as in ``make_block``."""
    nu = band.freq_table()
    nu_top = float(nu[0, 0])
    delay = K_DM_MS_GHZ2_PC * b.dm * (1.0 / nu ** 2 - 1.0 / nu_top ** 2) * 1e3 / NATIVE_SAMPLE_US
    start = b.t0_native + np.rint(delay).astype(np.int64)              # (G, C)
    lo = np.maximum(start, s0)
    hi = np.minimum(start + b.width_native, s0 + n_samp)
    g, c = np.nonzero(hi > lo)
    cnt = (hi - lo)[g, c]
    if cnt.size == 0:
        z = np.zeros(0, np.int64)
        return z, z, z
    gi = np.repeat(g, cnt)
    ci = np.repeat(c, cnt)
    first = np.repeat(lo[g, c] - np.concatenate([[0], np.cumsum(cnt)[:-1]]), cnt)
    s = first + np.arange(cnt.sum())
    return gi, ci, s


def inject_bursts_device(raw: torch.Tensor, *, band: Band, nant: int, s0: int,
                         bursts: Sequence[Burst], antpos_e, antpos_n, cell_lambda: float,
                         n_grid: int, sigma: float = 3.0, seed: int = 0,
                         max_samples: int = 1 << 20) -> int:
    """Add bursts to a device block of raw pages ``(G, npkt, nant, nchan, 2,
    2)`` uint8 whose first native sample is ``s0``, in place.  Every sample a
    burst covers is drawn afresh (Gaussian ``sigma``, a generator seeded
    with ``(seed, s0, burst)``), the burst added as ``make_block`` adds it
    (same delays, phases and amplitude), then rounded, clipped to [-8, 7] and
    packed.  The noise is independent from sample to sample, so redrawing
    the covered samples leaves the block's distribution that of
    ``make_block``.  Returns the number of samples rewritten."""
    if raw.dtype != torch.uint8 or raw.dim() != 6 or raw.device.type != "cuda":
        raise ValueError("raw must be a device uint8 (G, npkt, nant, nchan, 2, 2) block")
    dev = raw.device
    npkt = raw.shape[1]
    nu = band.freq_table()
    wl = torch.from_numpy(SPEED_OF_LIGHT_M_S / (nu * 1e9)).to(dev)            # (G, C) f64
    an = torch.as_tensor(np.asarray(antpos_n, np.float64), device=dev)
    ae = torch.as_tensor(np.asarray(antpos_e, np.float64), device=dev)
    scale = 1.0 / (cell_lambda * n_grid)
    done = 0
    for bi, b in enumerate(bursts):
        gi, ci, s = _burst_samples(band, b, s0, 2 * npkt)
        if s.size == 0:
            continue
        gen = torch.Generator(device=dev)
        gen.manual_seed(int(np.random.SeedSequence([seed, s0, bi]).generate_state(1)[0]))
        geo = 2 * np.pi * scale * (an * b.dl + ae * b.dm_pix)                # (nant,)
        for k0 in range(0, s.size, max_samples):
            g = torch.from_numpy(gi[k0:k0 + max_samples]).to(dev)
            c = torch.from_numpy(ci[k0:k0 + max_samples]).to(dev)
            rel = torch.from_numpy(s[k0:k0 + max_samples] - s0).to(dev)
            p, t = rel // 2, rel % 2
            n = g.numel()
            ph = geo[None, :] / wl[g, c][:, None]                             # (n, nant)
            re = torch.randn((n, nant, 2), generator=gen, device=dev).mul_(sigma)
            im = torch.randn((n, nant, 2), generator=gen, device=dev).mul_(sigma)
            re += (b.amp * torch.cos(ph)).to(torch.float32)[:, :, None]
            im += (b.amp * torch.sin(ph)).to(torch.float32)[:, :, None]
            qr = re.round_().clamp_(-8, 7).to(torch.int16)
            qi = im.round_().clamp_(-8, 7).to(torch.int16)
            raw[g, p, :, c, t, :] = ((qr & 0xF) | ((qi & 0xF) << 4)).to(torch.uint8)
            done += n
    return done


def burst_grid(*, snrs: Sequence[float], widths: Sequence[int], dms: Sequence[float],
               t_first_native: int, spacing_native: int, n_grid: int, seed: int,
               margin: int = 8):
    """The stress sweep's bursts: every (S/N, width, DM) of the grids once,
    in a seeded random order, arriving ``spacing_native`` native samples
    apart from ``t_first_native`` at seeded random pixels at least
    ``margin`` pixels inside the image.  Returns ``[(snr, width_native, dm,
    t0_native, dl, dm_pix)]``; the amplitude for each S/N is chosen by the
    caller (``amp_for_snr``)."""
    rng = np.random.default_rng(seed)
    cells = [(s, w, d) for s in snrs for w in widths for d in dms]
    order = rng.permutation(len(cells))
    half = n_grid // 2 - margin
    out = []
    for k, j in enumerate(order):
        s, w, d = cells[j]
        dl, dm_pix = (int(v) for v in rng.integers(-half, half + 1, 2))
        out.append((float(s), int(w), float(d), int(t_first_native + k * spacing_native),
                    dl, dm_pix))
    return out


def amp_for_snr(snr: float, width_native: int, *, amp_ref: float, snr_ref: float,
                width_ref: int) -> float:
    """Voltage amplitude giving boxcar S/N ``snr`` for a burst of
    ``width_native`` samples, from one measured reference burst: the
    correlated power is |amp|^2 per sample and the matched boxcar S/N grows
    as the square root of the width, so S/N ~ amp^2 sqrt(width)."""
    return amp_ref * float(np.sqrt((snr / snr_ref) * np.sqrt(width_ref / width_native)))


def match_bursts(bursts, cands, *, band: Band, fine_dm: np.ndarray, n_grid: int, t_int: int,
                 r_pix: int = 2, r_t: int = 8, dm_frac: float = 0.1, dm_abs: float = 30.0):
    """For each burst ``(snr, width_native, dm, t0_native, dl, dm_pix)``, the
    best-S/N candidate within ``r_pix`` pixels of its image position, within
    ``max(dm_abs, dm_frac * dm)`` of its DM and within ``r_t`` search samples
    plus the burst's width of its expected time; None where there is none.
    A candidate's time is that of the dedispersed burst at the bottom of the
    band, so the expected time is ``(t0 + delay(dm, band bottom)) / t_int``.
    Candidates are ``StreamCandidate``-like (t, fdm, l, m, snr, width)."""
    nu = band.freq_table()
    k_bot = K_DM_MS_GHZ2_PC * (1.0 / float(nu.min()) ** 2 - 1.0 / float(nu[0, 0]) ** 2) * 1e3 \
        / NATIVE_SAMPLE_US
    c = n_grid // 2
    out = []
    for (snr, w, dm, t0, dl, dmp) in bursts:
        t_exp = (t0 + k_bot * dm) / t_int
        r = r_t + w / t_int
        best = None
        for q in cands:
            if abs(q.l - (c + dl)) > r_pix or abs(q.m - (c + dmp)) > r_pix:
                continue
            if abs(float(fine_dm[q.fdm]) - dm) > max(dm_abs, dm_frac * dm):
                continue
            if abs(q.t - t_exp) > r:
                continue
            if best is None or q.snr > best.snr:
                best = q
        out.append(best)
    return out
