"""Generate the golden fixtures that pin the oracle to the reference.

Runs the UNMODIFIED dsa110-rt reference (``src/dsart``, imported from a
local checkout given by ``--reference`` / ``$DSART_REFERENCE``) on seeded
inputs at its native geometry (96 antennas, 16 x 384 channels) and writes
small ``.npz`` fixtures next to this script.  Large inputs are not stored:
they are regenerated from the recorded seed with numpy's PCG64 (bit-stable
across platforms) and the fixture stores exact fingerprints (hashes, exact
integer sums, sampled elements).

Usage (in a container where the reference checkout exists):

    python tests/golden/make_golden.py --reference <dsa110-rt>/src

The GPU box never runs this script; tests only read the ``.npz`` files.
"""

from __future__ import annotations

import argparse
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# ---------------------------------------------------------------------------
# Shared seeded-input recipes (the tests import these to regenerate inputs)
# ---------------------------------------------------------------------------

UNPACK_SEED = 20261203
CORR_SEED = 7301
STAGE1_SEED = 4242


def t_layout_antpos(nants: int, seed: int, ew_m: float = 2600.0, ns_m: float = 1600.0):
    """Seeded T layout: ~60% of antennas on the EW arm, the rest on the NS arm."""
    rng = np.random.default_rng(seed)
    n_ew = int(round(nants * 0.6))
    e = np.empty(nants)
    n = np.empty(nants)
    e[:n_ew] = np.sort(rng.uniform(-ew_m / 2, ew_m / 2, n_ew))
    n[:n_ew] = rng.normal(0.0, 2.0, n_ew)
    n[n_ew:] = -np.sort(rng.uniform(5.0, ns_m, nants - n_ew))
    e[n_ew:] = rng.normal(0.0, 2.0, nants - n_ew)
    return e.astype(np.float64), n.astype(np.float64)


def unpack_raw(seed: int = UNPACK_SEED) -> np.ndarray:
    """Full reference fada page: 2048 x 96 x 384 x 2 x 2 bytes."""
    rng = np.random.default_rng(seed)
    return rng.integers(0, 256, size=2048 * 96 * 384 * 4, dtype=np.uint8)


def corr_raw(npkt: int, nant: int, nchan: int, seed: int = CORR_SEED) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.integers(0, 256, size=npkt * nant * nchan * 4, dtype=np.uint8)


def stage1_vis(n_fv: int, nbase: int, nchan_eff: int, seed: int) -> np.ndarray:
    """Integer-valued complex64 visibilities in ``[-50, 50]``."""
    rng = np.random.default_rng(seed)
    re = rng.integers(-50, 51, size=(n_fv, nbase, nchan_eff)).astype(np.float32)
    im = rng.integers(-50, 51, size=(n_fv, nbase, nchan_eff)).astype(np.float32)
    return (re + 1j * im).astype(np.complex64)


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


# ---------------------------------------------------------------------------
# Fixture builders
# ---------------------------------------------------------------------------


def make_unpack():
    import torch
    from dsart.services.slow_corr_kernel import unpack_int4_split
    raw = unpack_raw()
    re, im = unpack_int4_split(raw, device="cpu", scale=1.0, out_dtype=torch.float32)
    re8 = re.numpy().astype(np.int8)
    im8 = im.numpy().astype(np.int8)
    rng = np.random.default_rng(1)
    idx = rng.integers(0, re8.size, 4096)
    np.savez_compressed(
        os.path.join(HERE, "unpack.npz"),
        seed=UNPACK_SEED, shape=np.asarray(re8.shape),
        sha_re=sha(re8), sha_im=sha(im8),
        idx=idx, re_s=re8.reshape(-1)[idx], im_s=im8.reshape(-1)[idx],
    )


def make_corr():
    import torch
    from dsart.services.corr_fast_kernel import FastCorrKernel
    out = {}
    # (a) fused Stokes-I + chan-sum at 96 antennas
    npkt, nant, nchan, t_int, csf = 8, 96, 16, 8, 4
    raw = corr_raw(npkt, nant, nchan).reshape(npkt, nant, nchan, 2, 2)
    r8 = torch.from_numpy(raw.view(np.int8).copy())
    re = ((r8 << 4) >> 4).permute(2, 3, 4, 0, 1).contiguous().to(torch.float32)
    im = (r8 >> 4).permute(2, 3, 4, 0, 1).contiguous().to(torch.float32)
    k = FastCorrKernel(device="cpu", t_int_fast_native=t_int, nants=nant, nchan=nchan)
    vis = k.compute_split(re, im, fuse_stokes_i=True, chan_sum_factor=csf).numpy()
    out.update(si_npkt=npkt, si_nant=nant, si_nchan=nchan, si_t_int=t_int, si_csf=csf,
               si_re=vis.real.astype(np.float32), si_im=vis.imag.astype(np.float32))
    # (b) legacy 2-pol output, small array, n_fv chunking exercised
    npkt, nant, nchan, t_int = 16, 10, 6, 4
    raw = corr_raw(npkt, nant, nchan, seed=CORR_SEED + 1).reshape(npkt, nant, nchan, 2, 2)
    r8 = torch.from_numpy(raw.view(np.int8).copy())
    re = ((r8 << 4) >> 4).permute(2, 3, 4, 0, 1).contiguous().to(torch.float32)
    im = (r8 >> 4).permute(2, 3, 4, 0, 1).contiguous().to(torch.float32)
    k = FastCorrKernel(device="cpu", t_int_fast_native=t_int, nants=nant, nchan=nchan)
    vis = k.compute_split(re, im, n_fv_chunk=3).numpy()
    out.update(p2_npkt=npkt, p2_nant=nant, p2_nchan=nchan, p2_t_int=t_int,
               p2_re=vis.real.astype(np.float32), p2_im=vis.imag.astype(np.float32))
    np.savez_compressed(os.path.join(HERE, "corr.npz"), **out)


def make_grid_and_plan():
    import torch
    from dsart.grid.sparsity_pattern import (build_pattern, compute_top_of_band_cell_lambda)
    from dsart.grid.kernel import FastVisGridder
    from dsart.coarse_dm.synthetic_plan import build_synthetic_summed_plan
    from dsart.coarse_dm.stage2_shifts import compute_stage2_shifts
    from dsart.fine_dm.combiner import compute_time_shift_search
    e, n = t_layout_antpos(96, seed=11)
    n_grid, csf = 256, 8
    cell = compute_top_of_band_cell_lambda(e, n, n_grid=n_grid)
    out = dict(antpos_e=e, antpos_n=n, n_grid=n_grid, csf=csf, cell_lambda=cell)
    for g in (0, 15):
        pat = build_pattern(e, n, chgroup=g, dec_deg=37.0, n_grid=n_grid,
                            chan_sum_factor=csf, cell_lambda=cell)
        grd = FastVisGridder.from_pattern(pat, e, n, device="cpu")
        cim = grd.cell_index_map.numpy().reshape(4656, 384 // csf)
        out[f"ix_row_{g}"] = pat.ix_row
        out[f"ix_col_{g}"] = pat.ix_col
        out[f"cim_{g}"] = cim.astype(np.int32)
        out[f"cellw_{g}"] = grd.cell_weights.numpy()
        if g == 15:
            vis = stage1_vis(2, 4656, 384 // csf, seed=55)
            gv = grd.compute(torch.from_numpy(vis)).numpy()
            out["grid_in_seed"] = 55
            out["grid_out"] = gv
    # DM plan delay bins (all chgroups)
    coarse = np.linspace(0.0, 3000.0, 16)
    plan = build_synthetic_summed_plan(n_coarse=16, dm_max=3000.0, chan_sum_factor=csf,
                                       t_int_fast_us=8 * 32.768)
    out["plan_coarse"] = coarse
    out["plan_bins"] = np.stack([plan.delay_bins_per_chgroup(g) for g in range(16)])
    out["plan_nat"] = np.stack([plan.delay_native_samples_per_chgroup(g) for g in range(16)])
    # stage-2 shifts, all chgroups
    cd = np.asarray([0.0, 50.0, 258.0, 581.5, 1312.0, 2962.0])
    out["s2_coarse"] = cd
    out["s2_shifts"] = np.stack([
        compute_stage2_shifts(chgroup=g, coarse_dm_pc_cm3=cd, t_int_corr_us=262.144).shifts_samples
        for g in range(16)])
    # fine-DM shift table, merged rounding + plain
    coarse8 = np.linspace(100.0, 1500.0, 8)
    fine = np.linspace(60.0, 1540.0, 64)
    f2c = np.clip(np.searchsorted(coarse8, fine) , 0, 7).astype(np.int64)
    t_int = 262.144
    tab_m = compute_time_shift_search(coarse_dm_pc_cm3=coarse8, fine_dm_pc_cm3=fine,
                                      fine_to_coarse=f2c, t_int_search_us=t_int,
                                      merge_coarse_rounding=True, t_int_corr_us=t_int)
    tab_p = compute_time_shift_search(coarse_dm_pc_cm3=coarse8, fine_dm_pc_cm3=fine,
                                      fine_to_coarse=f2c, t_int_search_us=t_int)
    out.update(fs_coarse=coarse8, fs_fine=fine, fs_f2c=f2c, fs_t_int=t_int,
               fs_merged=tab_m.shifts, fs_plain=tab_p.shifts)
    np.savez_compressed(os.path.join(HERE, "grid_plan.npz"), **out)


def make_stage1():
    import torch
    from dsart.grid.sparsity_pattern import build_pattern, compute_top_of_band_cell_lambda
    from dsart.grid.kernel import FastVisGridder
    from dsart.coarse_dm.synthetic_plan import build_synthetic_summed_plan
    from dsart.services.corr_fast_integration import Stage1MultiDMCoarseDM
    e, n = t_layout_antpos(96, seed=11)
    n_grid, csf, g = 256, 8, 15
    cell = compute_top_of_band_cell_lambda(e, n, n_grid=n_grid)
    pat = build_pattern(e, n, chgroup=g, dec_deg=37.0, n_grid=n_grid,
                        chan_sum_factor=csf, cell_lambda=cell)
    grd = FastVisGridder.from_pattern(pat, e, n, device="cpu")
    plan = build_synthetic_summed_plan(n_coarse=6, dm_max=150.0, chan_sum_factor=csf,
                                       t_int_fast_us=8 * 32.768)
    st = Stage1MultiDMCoarseDM(plan=plan, gridder=grd, chgroup=g, sliding_window=True)
    n_fv = 32
    outs = {}
    for blk in range(3):
        vis = stage1_vis(n_fv, 4656, 384 // csf, seed=STAGE1_SEED + blk)
        o = st.dedisperse_from_vis(torch.from_numpy(vis), block_n=blk).numpy()
        re = np.rint(o.real).astype(np.int64)
        im = np.rint(o.imag).astype(np.int64)
        assert np.array_equal(re, o.real) and np.array_equal(im, o.imag)
        outs[f"b{blk}_sum_t_re"] = re.sum(axis=1)
        outs[f"b{blk}_sum_t_im"] = im.sum(axis=1)
        outs[f"b{blk}_sum_c_re"] = re.sum(axis=2)
        outs[f"b{blk}_sum_c_im"] = im.sum(axis=2)
        rng = np.random.default_rng(blk)
        idx = rng.integers(0, o.size, 2048)
        outs[f"b{blk}_idx"] = idx
        outs[f"b{blk}_re_s"] = o.real.reshape(-1)[idx]
        outs[f"b{blk}_im_s"] = o.imag.reshape(-1)[idx]
        outs[f"b{blk}_shape"] = np.asarray(o.shape)
    # non-sliding single window
    st2 = Stage1MultiDMCoarseDM(plan=plan, gridder=grd, chgroup=g, sliding_window=False)
    vis = stage1_vis(n_fv, 4656, 384 // csf, seed=STAGE1_SEED + 9)
    o = st2.dedisperse_from_vis(torch.from_numpy(vis), block_n=0).numpy()
    outs["ns_shape"] = np.asarray(o.shape)
    outs["ns_sum_t_re"] = np.rint(o.real).astype(np.int64).sum(axis=1)
    outs["ns_sum_c_im"] = np.rint(o.imag).astype(np.int64).sum(axis=2)
    outs["bins"] = plan.delay_bins_per_chgroup(g)
    outs.update(seed=STAGE1_SEED, n_fv=n_fv, chgroup=g, csf=csf, n_grid=n_grid,
                dm_max=150.0, n_coarse=6)
    np.savez_compressed(os.path.join(HERE, "stage1.npz"), **outs)


def make_fifos_and_sky():
    import torch
    from dsart.services.corr_fast_integration import StaticSkyMean
    from dsart.coarse_dm.stage2_chgroup_alignment import Stage2InterChgroupShiftFifo
    from dsart.coarse_dm.stage2_per_dm_fifo import PerCoarseDmStage2FIFO
    from dsart.coarse_dm.stage2_shifts import compute_stage2_shifts
    out = {}
    rng = np.random.default_rng(77)
    # static sky
    sky = StaticSkyMean(window_blocks=3, warmup_cubes=2, n_dm=2)
    ins, outs = [], []
    for i in range(9):
        x = (rng.integers(-20, 21, (4, 40)) + 1j * rng.integers(-20, 21, (4, 40))).astype(np.complex64)
        ins.append(x)
        outs.append(sky.apply(torch.from_numpy(x), dm_slot=i % 2).numpy())
    out.update(sky_in=np.stack(ins), sky_out=np.stack(outs))
    # inter-chgroup shift FIFO
    cd = np.asarray([0.0, 300.0, 900.0, 1600.0, 2500.0])
    tab = compute_stage2_shifts(chgroup=2, coarse_dm_pc_cm3=cd, t_int_corr_us=262.144 * 32)
    fifo = Stage2InterChgroupShiftFifo(chgroup=2, coarse_dm_pc_cm3=cd, t_dedisp=16,
                                       t_int_corr_us=262.144 * 32, shift_table=tab)
    ins, outs, emitted = [], [], []
    for i in range(12):
        x = (rng.integers(-9, 10, (5, 16, 3)) + 1j * rng.integers(-9, 10, (5, 16, 3))).astype(np.complex64)
        ins.append(x)
        r = fifo.push(torch.from_numpy(x), block_n=i)
        emitted.append(len(r))
        outs.append(r[0].numpy() if r else np.zeros_like(x))
    out.update(ics_shifts=tab.shifts_samples, ics_in=np.stack(ins), ics_out=np.stack(outs),
               ics_emitted=np.asarray(emitted))
    # per-coarse-DM FIFO
    pf = PerCoarseDmStage2FIFO([0, 1, 3])
    seq = []
    for i in range(6):
        for c in range(3):
            r = pf.push(c, torch.full((2,), float(10 * i + c)))
            seq.append(-1 if r is None else int(r[0].item()))
    out["pdf_seq"] = np.asarray(seq)
    np.savez_compressed(os.path.join(HERE, "fifo_sky.npz"), **out)


def make_image_detector():
    import torch
    from dsart.image.imager import compute_edge_mask, dirty_image_from_uv_grid, apply_edge_mask
    from dsart.fine_dm.combiner import combine_chgroups
    from dsart.detector.forward import precompute_padded_cumsum, boxcar_from_padded_cumsum
    from dsart.detector.decoder import decode_topk_argmax_lowmem
    from dsart.noise_norm.layer1 import sigma_clipped_std_batched
    out = {}
    rng = np.random.default_rng(99)
    # combine_chgroups on dense streams
    N, Ts = 16, 10
    streams = (rng.integers(-5, 6, (16, Ts, N, N)) + 1j * rng.integers(-5, 6, (16, Ts, N, N))).astype(np.complex64)
    shifts = rng.integers(-4, 5, 16).astype(np.int32)
    comb = combine_chgroups(per_chgroup_streams={g: streams[g] for g in range(16)},
                            time_shift_per_chgroup=shifts, t_window=(2, 9))
    out.update(cmb_streams=streams, cmb_shifts=shifts, cmb_out=comb)
    # dirty image + edge mask
    N = 32
    uv = (rng.normal(size=(3, N, N)) + 1j * rng.normal(size=(3, N, N))).astype(np.complex64)
    img = dirty_image_from_uv_grid(uv)
    mask = compute_edge_mask(n_grid=N)
    out.update(img_uv=uv, img_out=img, img_mask=mask, img_masked=apply_edge_mask(img, mask))
    # padded cumsum + boxcars
    cube = rng.normal(size=(40, 2, 5, 6)).astype(np.float32)
    widths = [1, 2, 4, 8, 16]
    cs = precompute_padded_cumsum(torch.from_numpy(cube), axis=0, max_width=16)
    bx = [boxcar_from_padded_cumsum(cs, axis=0, width=w, max_width=16, n_out=24, t_base=8).numpy()
          for w in widths]
    out.update(bc_cube=cube, bc_cs=cs.numpy(), bc_box=np.stack(bx))
    # decode
    score = rng.normal(size=(12, 3, 8, 8)).astype(np.float32)
    score[3, 1, 4, 4] = 9.5
    score[4, 1, 4, 5] = 9.0       # suppressed by merge radius
    score[10, 0, 1, 1] = 8.0
    winner = rng.integers(0, 5, score.shape).astype(np.int16)
    cands = decode_topk_argmax_lowmem(
        torch.from_numpy(score), torch.from_numpy(winner), threshold=3.5,
        kernel_ids=[f"unit_d1_b{w}" for w in widths], kernel_time_widths=widths,
        merge_radius_lm=3, merge_radius_fdm=5, merge_radius_t=128 // 32, n_top=64)
    out.update(dec_score=score, dec_winner=winner,
               dec_out=np.asarray([[c.event_specnum, c.dm_idx, c.l, c.m, c.width_samples, c.snr]
                                   for c in cands], np.float64))
    # Layer-1 clipped std
    s = rng.normal(0, 2.0, (4, 3001)).astype(np.float32)
    s[0, :40] = 50.0
    s[2, 7] = np.nan
    out.update(l1_in=s, l1_out=sigma_clipped_std_batched(torch.from_numpy(s)).numpy())
    np.savez_compressed(os.path.join(HERE, "image_detector.npz"), **out)


RFI_SEED = 515


def rfi_masks(seed: int = RFI_SEED):
    """Seeded flags for a full page (96 ant, 384 ch, 2 pol; 64 accumulations
    of 32 packets): about 2 % of (ant, chan, pol) and 1 % of (acc, chan, pol)."""
    rng = np.random.default_rng(seed)
    return rng.random((96, 384, 2)) < 0.02, rng.random((64, 384, 2)) < 0.01


def make_rfi():
    """apply_rfi_mask_to_voltages (services/corr_fast_integration.py:1249) on
    the unpacked reference page, both masks."""
    import torch
    from dsart.services.corr_fast_integration import apply_rfi_mask_to_voltages
    from dsart.services.slow_corr_kernel import unpack_int4_split
    raw = unpack_raw()
    re, im = unpack_int4_split(raw, device="cpu", scale=1.0, out_dtype=torch.float32)
    m, tm = rfi_masks()
    apply_rfi_mask_to_voltages(re, im, torch.from_numpy(m), time_chan_mask=torch.from_numpy(tm))
    re8, im8 = re.numpy().astype(np.int8), im.numpy().astype(np.int8)
    np.savez_compressed(os.path.join(HERE, "rfi.npz"), sha_re=sha(re8), sha_im=sha(im8),
                        zeros=np.asarray([(re8 == 0).sum(), (im8 == 0).sum()]))


def make_slow_corr():
    """SlowCorrKernel.compute_split (services/slow_corr_kernel.py:576-720) on
    the unpacked reference page in float32 (scale 1: integer codes, exact
    sums), full block, both pols."""
    import torch
    from dsart.services.slow_corr_kernel import SlowCorrKernel, unpack_int4_split
    raw = unpack_raw()
    re, im = unpack_int4_split(raw, device="cpu", scale=1.0, out_dtype=torch.float32)
    vis = SlowCorrKernel(device="cpu").compute_split(re, im).numpy()
    v = np.ascontiguousarray(vis.astype(np.complex64))
    rng = np.random.default_rng(2)
    idx = rng.integers(0, v.size, 4096)
    np.savez_compressed(os.path.join(HERE, "slow_corr.npz"), shape=np.asarray(v.shape),
                        sha=sha(v.view(np.float32)), idx=idx, samples=v.reshape(-1)[idx])


POSTPROC_SEED = 6060


def postproc_fields(seed: int = POSTPROC_SEED, n: int = 500):
    """Seeded candidate fields, clustered so that the mergers suppress: one
    row per candidate (l, m, dm_idx, event_specnum, width, snr, flags,
    kernel index); dm_fine carries the row index."""
    rng = np.random.default_rng(seed)
    centre = rng.integers(0, 12, n)
    l = np.round(rng.normal(centre * 7.0, 2.0), 1)
    m = np.round(rng.normal((centre % 5) * 9.0, 2.0), 1)
    dm_idx = np.maximum(0, centre * 3 + rng.integers(-4, 5, n))
    t = np.maximum(0, centre * 400 + rng.integers(-300, 300, n))
    width = 1 << rng.integers(0, 6, n)
    snr = np.round(rng.uniform(6.0, 30.0, n), 2)
    snr[:20] = snr[20:40]                     # exact SNR ties
    flags = np.where(rng.random(n) < 0.05, 1 << 3, 0)
    kern = rng.integers(0, 4, n)
    return l, m, dm_idx, t, width, snr, flags, kern


def make_postproc():
    """merge_across_kernels_c1 / merge_across_kernels (detector/merger.py)
    and filter_to_canonical (detector/decoder.py:541) on seeded candidates."""
    from dsart.common.contracts import Candidate
    from dsart.detector.decoder import filter_to_canonical
    from dsart.detector.merger import MergerConfig, merge_across_kernels, merge_across_kernels_c1
    l, m, d, t, w, snr, flags, kern = postproc_fields()
    cands = [Candidate(l=float(l[i]), m=float(m[i]), dm_fine=float(i), dm_idx=int(d[i]),
                       event_specnum=int(t[i]), width_samples=int(w[i]),
                       kernel_id=f"unit:d1:b{1 << int(kern[i])}", snr=float(snr[i]),
                       detector_version="v1", flags=int(flags[i]), search_node_id=0, gpu_half=0)
             for i in range(len(l))]
    ids = lambda cs: np.asarray([int(c.dm_fine) for c in cs], np.int64)  # noqa: E731
    out = dict(c1_default=ids(merge_across_kernels_c1(cands, MergerConfig())),
               c1_custom=ids(merge_across_kernels_c1(cands, MergerConfig(
                   lm_max_cells=5, dm_max_trials=1, t_frac=0.5, sample_period_specnum=4))),
               legacy=ids(merge_across_kernels(cands)),
               legacy_custom=ids(merge_across_kernels(cands, merge_radius_lm=2,
                                                      merge_radius_fdm=3, merge_radius_t=50)))
    emit, dropped = filter_to_canonical(cands, dm_idx_canonical_lo=5, dm_idx_canonical_hi=25,
                                        t_det=4000, n_kernel_max_t=128, cube_t_offset=100)
    out.update(emit=ids(emit), dropped=ids(dropped),
               dropped_flags=np.asarray([c.flags for c in dropped], np.int64))
    np.savez_compressed(os.path.join(HERE, "postproc.npz"), **out)


TRANSPORT_SEED = 880


def transport_rows(seed: int = TRANSPORT_SEED) -> np.ndarray:
    """Seeded DM rows (n_fv 24, n_filled 300): Gaussian tiles of spread
    magnitudes, an all-zero tile, and tiles with amax 127 whose values sit
    on half-integers (exact ties of the rounding)."""
    rng = np.random.default_rng(seed)
    n_fv, nf = 24, 300
    mag = 10.0 ** rng.uniform(-3, 6, n_fv)
    row = (rng.standard_normal((n_fv, nf)) + 1j * rng.standard_normal((n_fv, nf))) * mag[:, None]
    row[5] = 0
    for t in (7, 8):
        re = rng.integers(-127, 127, nf) + 0.5
        im = rng.integers(-127, 127, nf) + 0.5
        re[0], im[0] = 127.0, -127.0
        row[t] = re + 1j * im
    return row.astype(np.complex64)


def make_transport():
    """TransportTx._encode_rows (transport/tx.py:825-873) on seeded rows."""
    from dsart.transport.tx import TransportTx
    rows = transport_rows()
    q16, s16 = TransportTx._encode_rows(rows, 16)
    q32, s32 = TransportTx._encode_rows(rows, 32)
    np.savez_compressed(os.path.join(HERE, "transport.npz"), q16=np.asarray(q16),
                        s16=np.asarray(s16), q32=np.asarray(q32), s32=np.asarray(s32))


LAYER2_SEED = 5353

LAYER2_CONFIGS = (
    dict(n_burnin=5),
    dict(n_burnin=3, sigma_floor=0.9, sigma_max_ratio=1.5, clamp_escape_cubes=4),
    dict(n_burnin=2, sigma_floor=(0.5, 0.8, 1.1, 0.2, 0.0), sigma_max_ratio=2.0,
         clamp_escape_cubes=0, tau_s=3.0),
)


def layer2_sequence(seed: int = LAYER2_SEED, n_cubes: int = 60, n_k: int = 5):
    """Seeded per-kernel σ estimates for ``n_cubes`` cubes: noise around 1,
    some zeros (no estimate), a two-cube spike and a lasting level rise on
    kernel 2 (clamp and escape), and invalid cubes."""
    rng = np.random.default_rng(seed)
    sig = (1.0 + 0.05 * rng.standard_normal((n_cubes, n_k))).astype(np.float32)
    sig[rng.random((n_cubes, n_k)) < 0.05] = 0.0
    sig[10:12, 1] *= 3.0
    sig[20:, 2] *= 2.5
    valid = rng.random(n_cubes) > 0.1
    return sig, valid


def make_layer1_state():
    """Layer1State.update_and_query(per_fdm_sigma=) (noise_norm/layer1.py:
    342-600) over the first 12 cubes of the seeded sequence (its 5 columns
    as fine DMs), with and without a floor."""
    import torch

    from dsart.noise_norm.layer1 import Layer1State
    sig, _ = layer2_sequence()
    out = {}
    for ci, kw in enumerate((dict(), dict(n_burnin_cubes=3, sigma_floor=0.97))):
        st = Layer1State(sig.shape[1], **kw)
        out[f"l1_{ci}"] = np.asarray([st.update_and_query(
            per_fdm_sigma=torch.from_numpy(sig[c])).numpy() for c in range(12)], np.float32)
    np.savez_compressed(os.path.join(HERE, "layer1_state.npz"), **out)


def make_layer2():
    """Layer2State.update_and_query(per_kernel_sigma=) (noise_norm/layer2.py:
    113-452) on CPU over a seeded sequence, for three configurations."""
    import torch

    from dsart.noise_norm.layer2 import Layer2State
    sig, valid = layer2_sequence()
    out = {}
    for ci, cfg in enumerate(LAYER2_CONFIGS):
        st = Layer2State(sig.shape[1], **cfg)
        s_k, warm = [], []
        for c in range(sig.shape[0]):
            s, w = st.update_and_query(per_kernel_sigma=torch.from_numpy(sig[c]),
                                       valid=bool(valid[c]))
            s_k.append(s.numpy())
            warm.append(w)
        out[f"s_k_{ci}"] = np.asarray(s_k, np.float32)
        out[f"warm_{ci}"] = np.asarray(warm, bool)
        out[f"counters_{ci}"] = np.asarray([st.n_clamped_high, st.n_clamp_escapes, st.cube_count])
        out[f"per_kernel_{ci}"] = np.stack([st.per_kernel_clamped_high.numpy(),
                                            st.per_kernel_clamp_escapes.numpy(),
                                            st.per_kernel_clamp_streak.numpy()])
    np.savez_compressed(os.path.join(HERE, "layer2.npz"), **out)


CAL_SEED = 4242


def cal_inputs(seed: int = CAL_SEED):
    """Seeded split voltages (nchan 8, 2, 2, npkt 4, nant 96) float16 (the
    fluffed int4 values x 0.05), complex gains (96, 8, 2) of spread
    magnitude and phase, and N-S antenna positions (96,) m."""
    rng = np.random.default_rng(seed)
    shape = (8, 2, 2, 4, 96)
    re = (rng.integers(-8, 8, shape) * 0.05).astype(np.float16)
    im = (rng.integers(-8, 8, shape) * 0.05).astype(np.float16)
    amp = 10.0 ** rng.uniform(-1, 1, (96, 8, 2))
    gains = amp * np.exp(1j * rng.uniform(-np.pi, np.pi, (96, 8, 2)))
    gains[0] = 1.0                                # one antenna at unit gain
    antpos_n = rng.uniform(-800.0, 800.0, 96)
    return re, im, gains, antpos_n


def make_cal():
    """apply_cal_split's eager form (slow_corr_kernel.py:417-423) on CPU
    float16 and float32 tensors, per-channel and broadcast (1-channel) gains,
    make_cal_broadcast_tensors (:531-569), and compute_dec_phase
    (cal/cal_loader.py:209) for chgroup 5 at two declinations."""
    import torch

    from dsart.cal.cal_loader import compute_dec_phase
    from dsart.services.slow_corr_kernel import _apply_cal_split_eager
    re, im, gains, antpos_n = cal_inputs()
    out = {}
    for dt, name in ((torch.float16, "f16"), (torch.float32, "f32")):
        r = torch.from_numpy(re.astype(np.float32)).to(dt)
        i = torch.from_numpy(im.astype(np.float32)).to(dt)
        gr = torch.from_numpy(np.ascontiguousarray(gains.real)).to(dt)
        gi = torch.from_numpy(np.ascontiguousarray(gains.imag)).to(dt)
        gr = gr.permute(1, 2, 0).contiguous().unsqueeze(1).unsqueeze(3)   # (8, 1, 2, 1, 96)
        gi = gi.permute(1, 2, 0).contiguous().unsqueeze(1).unsqueeze(3)
        out[f"g_re_{name}"], out[f"g_im_{name}"] = gr.numpy(), gi.numpy()
        o_re, o_im = _apply_cal_split_eager(r, i, gr, gi)
        out[f"out_re_{name}"], out[f"out_im_{name}"] = o_re.numpy(), o_im.numpy()
        b_re, b_im = _apply_cal_split_eager(r, i, gr[5:6], gi[5:6])      # one channel's gains
        out[f"bout_re_{name}"], out[f"bout_im_{name}"] = b_re.numpy(), b_im.numpy()
    for k, dec in enumerate((0.2, 1.3)):
        ph = compute_dec_phase(chgroup=5, obs_dec_rad=dec, antpos_n=antpos_n)
        out[f"dec_phase_sha_{k}"] = np.asarray(sha(ph.view(np.float64)))
        out[f"dec_phase_cols_{k}"] = ph[:, ::16]
    np.savez_compressed(os.path.join(HERE, "cal.npz"), **out)


CLUSTER_SEED = 7171


def cluster_fields(seed: int = CLUSTER_SEED, n: int = 400):
    """Seeded per-cube candidates: clumps around a few bursts in (l, m,
    fine DM, time, width) plus scattered noise detections.  Rows of (l, m,
    dm_fine, event_specnum, width, snr, search_node_id, gpu_half); the
    geometry is ``cluster_geometry()``."""
    rng = np.random.default_rng(seed)
    grid = cluster_geometry()["fine_dm_pc_cc"]
    n_b = 6
    bl, bm = rng.integers(20, 236, n_b), rng.integers(20, 236, n_b)
    bd, bt = rng.integers(3, 60, n_b), rng.integers(10, 240, n_b)
    which = rng.integers(-1, n_b, n)               # -1: scattered noise
    l = np.where(which >= 0, bl[which] + rng.integers(-3, 4, n), rng.integers(0, 256, n))
    m = np.where(which >= 0, bm[which] + rng.integers(-3, 4, n), rng.integers(0, 256, n))
    d = np.where(which >= 0, np.clip(bd[which] + rng.integers(-3, 4, n), 0, 63),
                 rng.integers(0, 64, n))
    t = np.where(which >= 0, bt[which] + rng.integers(-4, 5, n), rng.integers(0, 256, n))
    # dm_fine near (not on) the grid value, some beyond the grid's ends
    dm = grid[d] + rng.uniform(-4.0, 4.0, n)
    dm[:3] = [grid[0] - 30.0, grid[-1] + 30.0, 0.5 * (grid[10] + grid[11])]
    width = 1 << rng.integers(0, 6, n)
    snr = np.round(rng.uniform(6.0, 40.0, n), 3)
    # sub-pixel positions, exact .5 included (round half to even)
    lf = l + np.where(rng.random(n) < 0.1, 0.5, np.round(rng.uniform(-0.4, 0.4, n), 2))
    mf = m + np.round(rng.uniform(-0.4, 0.4, n), 2)
    return (lf.astype(np.float64), mf.astype(np.float64), dm, 1024 + t, width, snr,
            rng.integers(0, 8, n), rng.integers(0, 2, n))


def cluster_geometry():
    return dict(cube_id=3, specnum_start=1024, sample_period_specnum=16, t_det=256, n_grid=256,
                n_fdm_in_cube=64, sample_period_us=131.072, cell_l_rad=1.5e-4,
                cell_m_rad=1.4e-4, l0_rad=0.001, m0_rad=-0.002,
                fine_dm_pc_cc=np.linspace(50.0, 800.0, 64), mjd_start=60942.5)


RECORD_FIELDS = ("cluster_id", "cube_id", "cntc", "cntb_lm", "cntb_dm", "peak_candidate_idx",
                 "l_rad", "m_rad", "l_pix", "m_pix", "dm_fine_pc_cc", "fine_dm_idx", "t_in_cube",
                 "t_seconds", "width_samples", "snr", "event_specnum", "search_node_id",
                 "gpu_half")


def make_cluster():
    """cluster/features.py and cluster/forward.py (DBSCAN backend) on
    seeded candidates.  The reference's HDBSCAN backend needs the
    ``hdbscan`` package, which this environment lacks: its labels are
    taken from scikit-learn's HDBSCAN on the same weighted features, with
    min_samples + 1 (scikit-learn counts the point itself)."""
    import warnings

    from sklearn.cluster import HDBSCAN

    from dsart.cluster.features import candidates_to_features, candidates_to_real_coords
    from dsart.cluster.forward import ClustererConfig, cluster_candidates
    from dsart.common.contracts import Candidate, CubeGeometry
    l, m, dm, t, w, snr, node, half = cluster_fields()
    geom = CubeGeometry(**cluster_geometry())
    cands = [Candidate(l=float(l[i]), m=float(m[i]), dm_fine=float(dm[i]), dm_idx=0,
                       event_specnum=int(t[i]), width_samples=int(w[i]),
                       kernel_id=f"unit:d1:b{int(w[i])}", snr=float(snr[i]),
                       detector_version="v1", flags=0, search_node_id=int(node[i]),
                       gpu_half=int(half[i])) for i in range(len(l))]
    out = dict(feat_int=candidates_to_features(cands, geom),
               feat_real=candidates_to_features(cands, geom, mode="real",
                                                weights=(1.0, 0.5, 2.0, 3e3, 3e3)),
               coords=np.asarray(candidates_to_real_coords(cands, geom), np.float64))
    for name, cfg in (("db", ClustererConfig(backend="dbscan")),
                      ("dbreal", ClustererConfig(backend="dbscan", feature_mode="real",
                                                 weights=(1.0, 0.02, 20.0, 3e3, 3e3),
                                                 dbscan_eps=2.5, dbscan_min_samples=3))):
        labels, recs = cluster_candidates(cands, geom, config=cfg)
        out[name + "_labels"] = labels
        out[name + "_records"] = np.asarray([[float(getattr(r, f)) for f in RECORD_FIELDS]
                                             for r in recs], np.float64)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        for name, X in (("hdb_int", out["feat_int"]), ("hdb_real", out["feat_real"])):
            out[name] = HDBSCAN(min_cluster_size=2, min_samples=2, cluster_selection_epsilon=10.0,
                                metric="manhattan", allow_single_cluster=True,
                                copy=True).fit_predict(X)
    np.savez_compressed(os.path.join(HERE, "cluster.npz"), **out)


SPARSE_SEED = 808


def sparse_inv_lut(seed: int = SPARSE_SEED, n_sb: int = 5, N: int = 32, n_filled: int = 60):
    """Seeded inverse LUTs [n_sb, N*N]: each stream's n_filled cells (compact
    index 0..n_filled-1 in ascending cell order), -1 elsewhere; some cells
    shared by several streams, some by their mirrors."""
    rng = np.random.default_rng(seed)
    lut = np.full((n_sb, N * N), -1, np.int64)
    for g in range(n_sb):
        cells = np.sort(rng.choice(N * N, n_filled, replace=False))
        lut[g, cells] = np.arange(n_filled)
    return lut


def make_sparse_csr():
    """build_sparse_cell_csr (image/tiled_combine_cuda.py:1092) on torch CPU:
    the combine_sparse_v4 tables, pinned field by field."""
    import torch
    from dsart.image.tiled_combine_cuda import build_sparse_cell_csr
    out = {}
    for name, kw in (("a", dict(n_sb=5, N=32, n_filled=60)),
                     ("b", dict(n_sb=16, N=16, n_filled=100))):
        lut = sparse_inv_lut(**kw)
        csr = build_sparse_cell_csr(torch.from_numpy(lut), n_grid=kw["N"])
        out[f"{name}_lut"] = lut.astype(np.int32)
        out[f"{name}_n_grid"] = kw["N"]
        for f in ("cell_uw", "cell_ptr", "ent_g", "ent_k", "ent_km"):
            out[f"{name}_{f}"] = getattr(csr, f).numpy().astype(np.int32)
        out[f"{name}_buckets"] = np.asarray(csr.buckets, np.int64).reshape(-1, 3)
    np.savez_compressed(os.path.join(HERE, "sparse_csr.npz"), **out)


def make_kernel_bank():
    """build_kernel_bank (detector/kernels.py:191): ids, widths and order of
    the default bank and of the production (unit, d1, b1..b64) bank."""
    from dsart.detector.kernels import build_kernel_bank
    out = {}
    for name, kw in (("full", {}), ("prod", dict(image_tokens=("unit",), dm_tokens=("d1",),
                                                 time_tokens=("b1", "b2", "b4", "b8", "b16",
                                                              "b32", "b64")))):
        bank = build_kernel_bank(**kw)
        out[f"{name}_ids"] = np.asarray([k.kernel_id for k in bank])
        out[f"{name}_w"] = np.asarray([[k.k_dm_width, k.k_time_width, k.image_kernel_size]
                                       for k in bank], np.int64)
    np.savez_compressed(os.path.join(HERE, "kernel_bank.npz"), **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("DSART_REFERENCE", ""))
    ap.add_argument("--only", default="")
    a = ap.parse_args()
    if not a.reference or not os.path.isdir(a.reference):
        sys.exit("need --reference <dsa110-rt>/src")
    sys.path.insert(0, a.reference)
    todo = [make_unpack, make_corr, make_grid_and_plan, make_stage1, make_fifos_and_sky,
            make_image_detector, make_transport, make_rfi, make_slow_corr, make_postproc,
            make_cluster, make_cal, make_layer2, make_layer1_state, make_sparse_csr,
            make_kernel_bank]
    for fn in todo:
        if a.only and a.only not in fn.__name__:
            continue
        print("building", fn.__name__, flush=True)
        fn()


if __name__ == "__main__":
    main()
