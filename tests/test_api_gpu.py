"""GPU parity of the drop-in API kernels against the reference's golden
fixtures (tests/golden) and the CPU oracle.  Integer/index work is
compared bit-exactly; float32 arithmetic with the tolerance stated per test."""

import os
import sys

import numpy as np
import pytest
import torch

import dsb_oracle as O

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden as MG  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def _z(golden_dir, name):
    return np.load(os.path.join(golden_dir, name), allow_pickle=False)


def test_pattern_cellmap_gridder_vs_reference(dev, golden_dir):
    from dsb200.grid import FastVisGridder, build_pattern, compute_top_of_band_cell_lambda
    z = _z(golden_dir, "grid_plan.npz")
    e, n = z["antpos_e"], z["antpos_n"]
    cell = compute_top_of_band_cell_lambda(e, n, n_grid=int(z["n_grid"]))
    assert cell == float(z["cell_lambda"])
    for g in (0, 15):
        pat = build_pattern(e, n, chgroup=g, n_grid=int(z["n_grid"]),
                            chan_sum_factor=int(z["csf"]), cell_lambda=cell, device=dev)
        np.testing.assert_array_equal(pat.ix_row, z[f"ix_row_{g}"])
        np.testing.assert_array_equal(pat.ix_col, z[f"ix_col_{g}"])
        grd = FastVisGridder.from_pattern(pat, e, n, device=dev)
        np.testing.assert_array_equal(grd.cell_index_map.numpy().reshape(4656, -1),
                                      z[f"cim_{g}"].astype(np.int64))
        np.testing.assert_array_equal(grd.cell_weights.cpu().numpy(), z[f"cellw_{g}"])
        if g == 15:
            vis = MG.stage1_vis(2, 4656, 48, seed=int(z["grid_in_seed"]))
            out = grd.compute(torch.from_numpy(vis).to(dev)).cpu().numpy()
            np.testing.assert_array_equal(out, z["grid_out"])


def test_stage1_sliding_window_vs_reference(dev, golden_dir):
    from dsb200.dedisp import DMPlan, Stage1MultiDMCoarseDM
    from dsb200.grid import FastVisGridder, build_pattern, compute_top_of_band_cell_lambda
    z = _z(golden_dir, "stage1.npz")
    e, n = MG.t_layout_antpos(96, seed=11)
    g, csf = int(z["chgroup"]), int(z["csf"])
    cell = compute_top_of_band_cell_lambda(e, n, n_grid=int(z["n_grid"]))
    pat = build_pattern(e, n, chgroup=g, n_grid=int(z["n_grid"]), chan_sum_factor=csf,
                        cell_lambda=cell, device=dev)
    grd = FastVisGridder.from_pattern(pat, e, n, device=dev)
    plan = DMPlan(dm_pc_cc=np.linspace(0.0, float(z["dm_max"]), int(z["n_coarse"])),
                  t_int_fast_us=8 * 32.768, chan_sum_factor=csf)
    np.testing.assert_array_equal(plan.delay_bins_per_chgroup(g), z["bins"])
    st = Stage1MultiDMCoarseDM(plan=plan, gridder=grd, chgroup=g, sliding_window=True)
    for blk in range(3):
        vis = MG.stage1_vis(int(z["n_fv"]), 4656, 48, seed=int(z["seed"]) + blk)
        o = st.dedisperse_from_vis(torch.from_numpy(vis).to(dev), block_n=blk).cpu().numpy()
        assert o.shape == tuple(z[f"b{blk}_shape"])
        re, im = o.real.astype(np.int64), o.imag.astype(np.int64)
        np.testing.assert_array_equal(re.sum(axis=1), z[f"b{blk}_sum_t_re"])
        np.testing.assert_array_equal(im.sum(axis=1), z[f"b{blk}_sum_t_im"])
        np.testing.assert_array_equal(re.sum(axis=2), z[f"b{blk}_sum_c_re"])
        np.testing.assert_array_equal(im.sum(axis=2), z[f"b{blk}_sum_c_im"])
        idx = z[f"b{blk}_idx"]
        np.testing.assert_array_equal(o.real.reshape(-1)[idx], z[f"b{blk}_re_s"])
        np.testing.assert_array_equal(o.imag.reshape(-1)[idx], z[f"b{blk}_im_s"])
    st2 = Stage1MultiDMCoarseDM(plan=plan, gridder=grd, chgroup=g, sliding_window=False)
    vis = MG.stage1_vis(int(z["n_fv"]), 4656, 48, seed=int(z["seed"]) + 9)
    o = st2.dedisperse_from_vis(torch.from_numpy(vis).to(dev), block_n=0).cpu().numpy()
    assert o.shape == tuple(z["ns_shape"])
    np.testing.assert_array_equal(o.real.astype(np.int64).sum(axis=1), z["ns_sum_t_re"])
    np.testing.assert_array_equal(o.imag.astype(np.int64).sum(axis=2), z["ns_sum_c_im"])


def test_static_sky_vs_oracle_and_reference(dev, golden_dir):
    from dsb200.dedisp import StaticSkyMean
    z = _z(golden_dir, "fifo_sky.npz")
    sky = StaticSkyMean(window_blocks=3, warmup_cubes=2, n_dm=2)
    osky = O.StaticSkyMean(window_blocks=3, warmup_cubes=2, n_dm=2)
    for i, (x, ref) in enumerate(zip(z["sky_in"], z["sky_out"])):
        got = sky.apply(torch.from_numpy(x).to(dev), dm_slot=i % 2).cpu().numpy()
        np.testing.assert_array_equal(got, osky.apply(x, dm_slot=i % 2))   # same definition
        np.testing.assert_allclose(got, ref, rtol=0, atol=2e-6 * max(1.0, np.abs(ref).max()))


def test_stage2_fifos_vs_reference(dev, golden_dir):
    from dsb200.dedisp import (PerCoarseDmStage2FIFO, Stage2FIFO, Stage2InterChgroupShiftFifo,
                               compute_stage2_shifts)
    z = _z(golden_dir, "fifo_sky.npz")
    cd = np.asarray([0.0, 300.0, 900.0, 1600.0, 2500.0])
    tab = compute_stage2_shifts(chgroup=2, coarse_dm_pc_cm3=cd, t_int_corr_us=262.144 * 32)
    np.testing.assert_array_equal(tab.shifts_samples, z["ics_shifts"])
    f = Stage2InterChgroupShiftFifo(chgroup=2, coarse_dm_pc_cm3=cd, t_dedisp=16, shift_table=tab)
    for i, (x, ref, n) in enumerate(zip(z["ics_in"], z["ics_out"], z["ics_emitted"])):
        r = f.push(torch.from_numpy(x).to(dev), block_n=i)
        assert len(r) == int(n)
        if r:
            np.testing.assert_array_equal(r[0].cpu().numpy(), ref)
    pf = PerCoarseDmStage2FIFO([0, 1, 3])
    seq = []
    for i in range(6):
        for c in range(3):
            r = pf.push(c, torch.full((2,), float(10 * i + c), device=dev))
            seq.append(-1 if r is None else int(r[0].item()))
    np.testing.assert_array_equal(np.asarray(seq), z["pdf_seq"])
    q = Stage2FIFO(depth=2)
    a, b, c = (torch.zeros(3, device=dev) + k for k in range(3))
    assert q.push(a) is None and q.push(b) is None and q.push(c) is a
    with pytest.raises(ValueError):
        q.push(torch.zeros(4, device=dev))


@pytest.mark.parametrize("half", [False, True])
@pytest.mark.parametrize("calib", [False, True])
def test_dense_combine_vs_oracle(dev, half, calib):
    from dsb200.search import fused_dequant_combine_per_fdm, fused_dequant_combine_per_fdm_half
    rng = np.random.default_rng(4)
    G, T, N, t_det, t_lo = 5, 12, 16, 10, 3
    streams = rng.integers(-100, 100, (G, T, 2, N, N)).astype(np.int8)
    shifts = rng.integers(-3, 4, G).astype(np.int32)
    nw = N // 2 + 1 if half else N
    out = torch.zeros((t_det - t_lo, N, nw), dtype=torch.complex64, device=dev)
    kw = {}
    if calib:
        kw = dict(scales=torch.ones(G, device=dev), offsets_re=torch.zeros(G, device=dev),
                  offsets_im=torch.zeros(G, device=dev))
    fn = fused_dequant_combine_per_fdm_half if half else fused_dequant_combine_per_fdm
    fn(torch.from_numpy(streams).to(dev), torch.from_numpy(shifts).to(dev), out, t_lo=t_lo,
       fftshift=True, **kw)
    cplx = streams[:, :, 0].astype(np.float64) + 1j * streams[:, :, 1].astype(np.float64)
    want = (O.combine_half if half else O.combine_full)(cplx, shifts, t_det, t_lo, fftshift=True)
    np.testing.assert_array_equal(out.cpu().numpy(), want.astype(np.complex64))


def test_edge_mask_and_image_vs_reference(dev, golden_dir):
    from dsb200.search import compute_edge_mask, irfft2_image
    z = _z(golden_dir, "image_detector.npz")
    np.testing.assert_array_equal(compute_edge_mask(n_grid=32), z["img_mask"])
    # half-spectrum identity on the device, vs the reference's dirty image
    uv = z["img_uv"].astype(np.complex128)
    N = uv.shape[-1]
    u = np.arange(N)
    shifted = uv * (1 - 2 * ((u[:, None] + u[None, :]) & 1))   # fftshift folded into the grid
    um = (N - u) % N
    half = 0.5 * (shifted + np.conj(shifted[:, um][:, :, um]))
    half = half[:, :, : N // 2 + 1]
    img = irfft2_image(torch.from_numpy(half.astype(np.complex64)).to(dev), N).cpu().numpy()
    ref = z["img_out"]
    assert np.abs(img - ref).max() <= 1e-5 * np.abs(ref).max()


@pytest.mark.parametrize("N", [32, 64, 128, 256, 512])
def test_dense_irfft2_matches_numpy(dev, N):
    """dsb_irfft2 (the GpuImager's transform) against numpy.fft.irfft2 in
    float64 on random half spectra, Hermitian or not (the imaginary parts of
    columns 0 and N/2 are dropped as numpy drops them): float32 error within
    2e-6 of the image's largest value."""
    from dsb200.search import irfft2_image
    rng = np.random.default_rng(N)
    half = rng.standard_normal((3, N, N // 2 + 1)) + 1j * rng.standard_normal((3, N, N // 2 + 1))
    h = torch.from_numpy(half.astype(np.complex64)).to(dev)
    got = irfft2_image(h, N).cpu().numpy()
    want = np.fft.irfft2(half.astype(np.complex64).astype(np.complex128), s=(N, N))
    assert np.abs(got - want).max() <= 2e-6 * np.abs(want).max()


def test_cumsum_boxcars_argmax_vs_reference(dev, golden_dir):
    from dsb200.search import (boxcar_from_padded_cumsum, multi_boxcar_argmax_triton,
                               precompute_padded_cumsum)
    z = _z(golden_dir, "image_detector.npz")
    cube = torch.from_numpy(z["bc_cube"]).to(dev)
    cs = precompute_padded_cumsum(cube, axis=0, max_width=16)
    np.testing.assert_array_equal(cs.cpu().numpy(), z["bc_cs"])
    widths = [1, 2, 4, 8, 16]
    for k, w in enumerate(widths):
        bx = boxcar_from_padded_cumsum(cs, axis=0, width=w, max_width=16, n_out=24, t_base=8)
        np.testing.assert_array_equal(bx.cpu().numpy(), z["bc_box"][k])
    sinv = np.float32(1.0) / np.sqrt(np.asarray(widths, np.float32))
    offs = O.boxcar_offsets(widths, 16)
    mx, win = multi_boxcar_argmax_triton(
        cs, widths=torch.tensor(widths, dtype=torch.int32, device=dev),
        offsets=torch.tensor(offs, dtype=torch.int32, device=dev),
        sigma_inv=torch.from_numpy(sinv).to(dev), n_out=24, t_base=8)
    omx, owin = O.multi_boxcar_argmax(z["bc_cs"], widths, offs, sinv, 24, 8)
    np.testing.assert_array_equal(mx.cpu().numpy(), omx)
    np.testing.assert_array_equal(win.cpu().numpy(), owin)


@pytest.mark.parametrize("log_w", [2, 4, 6])
@pytest.mark.parametrize("f16", [False, True])
@pytest.mark.parametrize("hw", [(12, 10), (11, 9), (16, 16)])
def test_fused_detector_matches_cumsum_argmax(dev, log_w, f16, hw):
    """Candidates of the streaming detector == every cell above threshold of
    the padded cumsum + boxcar argmax, bit for bit, for even and odd pixel
    counts and float or half cubes (float cubes of 16 x 16 x 3 = 768 cells
    take the TMA-staged kernel, the others the register-prefetch one)."""
    from dsb200.search import CandidateBuffer, detect_cube
    rng = np.random.default_rng(10 + log_w)
    T, F = 70, 3
    H, W = hw
    x = rng.normal(size=(T, F, H, W)).astype(np.float16 if f16 else np.float32)
    x[30:34, 1, 5, 5] += 6.0
    widths = [1 << k for k in range(log_w + 1)]
    maxw = widths[-1]
    t_base, n_out = maxw // 2, T - 2 * (maxw // 2)
    sinv = (np.float32(1.0) / np.sqrt(np.asarray(widths, np.float32))).astype(np.float32)
    buf = CandidateBuffer(dev, 1 << 16)
    detect_cube(torch.from_numpy(x).to(dev), log_max_width=log_w,
                sigma_inv=torch.from_numpy(sinv).to(dev), t_base=t_base, n_out=n_out,
                threshold=2.5, cands=buf)
    got = buf.fetch()
    cs = O.padded_cumsum(x.astype(np.float32), maxw)
    mx, win = O.multi_boxcar_argmax(cs, widths, O.boxcar_offsets(widths, maxw), sinv, n_out, t_base)
    sel = np.nonzero(mx.reshape(-1) > 2.5)[0]
    inner = F * H * W
    want = sorted((int(i // inner), int(i % inner), float(mx.reshape(-1)[i]), int(win.reshape(-1)[i]))
                  for i in sel)
    have = sorted((int(c["t"]), int(c["pix"]), float(c["snr"]), int(c["k"])) for c in got)
    assert have == want


@pytest.mark.parametrize("hw", [(16, 16), (12, 10)])
def test_detector_count_saturates_instead_of_wrapping(dev, hw):
    """When nearly every cell passes the threshold the candidate count stops
    near 2^30 instead of wrapping to negative slots: started just below the
    saturation level, a launch with thousands of hits writes nothing and
    leaves the count between 2^30 and 2^31 (both detector forms)."""
    from dsb200.search import CandidateBuffer, detect_cube
    rng = np.random.default_rng(5)
    T, F = 24, 2
    H, W = hw
    x = (5.0 + rng.random(size=(T, F, H, W))).astype(np.float32)
    sinv = torch.ones(3, dtype=torch.float32, device=dev)
    buf = CandidateBuffer(dev, 64)
    buf.buf.fill_(-7)
    buf.count[0] = (1 << 30) - 3
    detect_cube(torch.from_numpy(x).to(dev), log_max_width=2, sigma_inv=sinv, t_base=2,
                n_out=T - 4, threshold=1.0, cands=buf)
    cnt = buf.count.cpu().numpy()
    assert (1 << 30) <= int(cnt[0]) < (1 << 31) - 1
    assert bool((buf.buf == -7).all())
    assert np.int32(cnt[1]).view(np.float32) > 1.0


@pytest.mark.parametrize("cap", [1 << 16, 600, 300])
def test_candidate_buffer_top_selection_is_exact_or_raises(dev, cap):
    """fetch_top(n) returns every entry whose S/N is at least the n-th
    largest of all cells above threshold (ties included).  With a buffer too
    small for every cell, it returns that same set whenever the cells that
    did not fit rank below it, and raises otherwise -- never a wrong set."""
    from dsb200 import _lib
    from dsb200.search import CandidateBuffer, detect_cube
    rng = np.random.default_rng(21)
    T, F, H, W = 40, 2, 16, 16
    x = rng.normal(size=(T, F, H, W)).astype(np.float32)
    x[10:14, 1, 3, 4] += 9.0
    x[25:27, 0, 8, 8] += 7.0
    sinv = torch.ones(3, dtype=torch.float32, device=dev)
    full = CandidateBuffer(dev, 1 << 16)
    detect_cube(torch.from_numpy(x).to(dev), log_max_width=2, sigma_inv=sinv, t_base=2,
                n_out=T - 4, threshold=1.0, cands=full)
    every = full.fetch()
    assert len(every) > 1000
    n_top = 64
    vk = np.sort(every["snr"])[::-1][n_top - 1]
    want = sorted(tuple(int(v) if k != "snr" else float(v) for k, v in zip(e.dtype.names, e))
                  for e in every[every["snr"] >= vk])
    buf = CandidateBuffer(dev, cap)
    detect_cube(torch.from_numpy(x).to(dev), log_max_width=2, sigma_inv=sinv, t_base=2,
                n_out=T - 4, threshold=1.0, cands=buf)
    try:
        got = buf.fetch_top(n_top)
    except _lib.DsbError:
        assert cap < len(every)
        return
    have = sorted(tuple(int(v) if k != "snr" else float(v) for k, v in zip(e.dtype.names, e))
                  for e in got)
    assert have == want


def test_decode_vs_reference(dev, golden_dir):
    from dsb200.search import decode_topk_argmax_lowmem
    z = _z(golden_dir, "image_detector.npz")
    widths = [1, 2, 4, 8, 16]
    c = decode_topk_argmax_lowmem(torch.from_numpy(z["dec_score"]).to(dev),
                                  torch.from_numpy(z["dec_winner"]).to(dev), threshold=3.5,
                                  kernel_ids=[f"unit_d1_b{w}" for w in widths],
                                  kernel_time_widths=widths, merge_radius_lm=3,
                                  merge_radius_fdm=5, merge_radius_t=4, n_top=64)
    got = np.asarray([[x.event_specnum, x.dm_idx, x.l, x.m, x.width_samples, x.snr] for x in c])
    np.testing.assert_array_equal(got, z["dec_out"])


def test_layer1_vs_reference(dev, golden_dir):
    from dsb200.search import sigma_clipped_std_batched
    z = _z(golden_dir, "image_detector.npz")
    got = sigma_clipped_std_batched(torch.from_numpy(z["l1_in"]).to(dev)).cpu().numpy()
    np.testing.assert_allclose(got, z["l1_out"], rtol=2e-6)
    np.testing.assert_allclose(got, O.sigma_clipped_std_batched(z["l1_in"]), rtol=2e-6)


@pytest.mark.parametrize("m", [4096, 4000, 1000, 37, 2])
def test_layer1_sort_edge_cases(dev, m):
    """The clipped std's in-register / shuffle / shared-memory bitonic sort
    on rows of every fill (power of two or not), with non-finite values,
    signed zeros, heavy ties and outliers, against the oracle."""
    from dsb200.search import sigma_clipped_std_batched
    rng = np.random.default_rng(m)
    rows = rng.standard_normal((6, m)).astype(np.float32)
    rows[1] = np.round(rows[1] * 2) / 2             # many exact ties
    rows[2, ::7] = np.nan
    rows[2, 3::11] = np.inf
    rows[2, 5::13] = -np.inf
    rows[3] = 0.0
    rows[3, ::2] = -0.0
    rows[3, :min(m, 5)] = [1.0, -1.0, 2.0, 0.5, 3.0][:min(m, 5)]
    rows[4, :max(1, m // 50)] = 1e4                 # outliers the clip removes
    rows[5] = np.nan                                # nothing finite
    got = sigma_clipped_std_batched(torch.from_numpy(rows).to(dev)).cpu().numpy()
    np.testing.assert_allclose(got, O.sigma_clipped_std_batched(rows), rtol=2e-6)


def test_uv_cells_fp64_gpu_equals_numpy(dev):
    from dsb200.grid import per_baseline_uv_meters, uv_cells_gpu
    e, n = MG.t_layout_antpos(96, seed=3)
    du, dv, _ = per_baseline_uv_meters(e, n)
    nu = np.linspace(1.31, 1.5, 48)
    cell = 7.3
    r, c = uv_cells_gpu(du, dv, nu, cell, 256, dev)
    wl = 299792458.0 / (nu * 1e9)
    np.testing.assert_array_equal(c, np.rint(-(du[:, None] / wl[None, :]) / cell).astype(np.int64) + 128)
    np.testing.assert_array_equal(r, np.rint(-(dv[:, None] / wl[None, :]) / cell).astype(np.int64) + 128)


def test_layer1_sigma_and_detector_divisor_match_indexed_path(dev):
    """dsb_layer1_sigma (subsample gathered in the kernel) and the detector's
    per-fine-DM sigma divisor give the same bits as indexing the subsample in
    torch, sigma_clipped_std_batched, and a precomputed mask / sigma."""
    from dsb200.search import (CandidateBuffer, detect_images, layer1_sigma,
                               sigma_clipped_std_batched)
    g = torch.Generator(device="cpu").manual_seed(21)
    F, T, H, W = 3, 40, 16, 16
    img = torch.randn((F, T, H, W), generator=g).to(dev)
    img[1] *= 0.0                          # a fine DM whose sigma is 0 -> divisor 1
    img[2, 20:23, 5, 7] += 9.0
    times = torch.tensor([2, 9, 17, 30, 37], dtype=torch.int32, device=dev)
    pix = torch.arange(3, H * W, 7, dtype=torch.int32, device=dev)
    mask = torch.rand((H, W), generator=g).to(dev) + 0.5
    sig = layer1_sigma(img, times, pix)
    samp = img.reshape(F, T, H * W)[:, times.long()][:, :, pix.long()].reshape(F, -1)
    ref = sigma_clipped_std_batched(samp)
    ref = torch.where(ref > 0, ref, torch.ones_like(ref))
    assert torch.equal(sig, ref)
    sinv = (1.0 / torch.sqrt(torch.tensor([1.0, 2.0, 4.0, 8.0]))).to(dev)
    runs = []
    for use_div in (True, False):
        buf = CandidateBuffer(dev, 1 << 16)
        if use_div:
            detect_images(img, mask, log_max_width=3, sigma_inv=sinv, t_base=4, n_out=T - 8,
                          threshold=2.0, cands=buf, sigma_f=sig)
        else:
            mask_f = (mask[None] / ref[:, None, None]).contiguous()
            detect_images(img, mask_f, log_max_width=3, sigma_inv=sinv, t_base=4, n_out=T - 8,
                          threshold=2.0, cands=buf)
        runs.append(sorted((int(c["t"]), int(c["pix"]), float(c["snr"]), int(c["k"]))
                           for c in buf.fetch()))
    assert runs[0] == runs[1] and len(runs[0]) > 0


@pytest.mark.parametrize("cube_dtype", [torch.float32, torch.float16])
def test_gpu_imager_process_cube_vs_oracle(dev, cube_dtype):
    """GpuImager.build / process_cube (image/imager_gpu.py:169-657) on dense
    cint8 streams: per fine DM the half-spectrum combine, irfft2 and the edge
    mask, against the float64 oracle (1e-5 of the peak for float32 cubes,
    the half rounding for float16); the per-fine-DM mask; ping-pong cubes."""
    from dsb200.search import GpuImager, GpuImagerConfig
    rng = np.random.default_rng(31)
    G, Ts, N, t_det, n_fdm = 3, 20, 64, 16, 3
    q = rng.integers(-20, 21, (G, Ts, 2, N, N)).astype(np.int8)
    shifts = rng.integers(-3, 4, (n_fdm, G)).astype(np.int32)
    cfg = GpuImagerConfig(n_grid=N, t_det=t_det, n_fdm=n_fdm, n_chgroup=G, cube_dtype=cube_dtype)
    im = GpuImager.build(cfg)
    streams = torch.from_numpy(q).to(dev)
    cube = im.process_cube(streams_cint8=streams, time_shifts_gpu=torch.from_numpy(shifts).to(dev))
    torch.cuda.synchronize()
    z = q[:, :, 0].astype(np.float64) + 1j * q[:, :, 1].astype(np.float64)
    mask = O.edge_mask(N)
    want = np.stack([np.fft.irfft2(O.combine_half(z, shifts[f], t_det), s=(N, N)) * mask
                     for f in range(n_fdm)], axis=1)            # (t_det, n_fdm, N, N)
    got = cube.float().cpu().numpy()
    tol = (1e-5 if cube_dtype == torch.float32 else 1e-3) * np.abs(want).max()
    assert np.abs(got - want).max() <= tol
    # per-fine-DM mask: edge mask x 1/sigma, and the other output buffer
    sinv = torch.tensor([1.0, 0.5, 2.0], device=dev)
    im.set_edge_mask_per_fdm(sinv)
    cube2 = im.process_cube(streams_cint8=streams, time_shifts_gpu=torch.from_numpy(shifts).to(dev))
    torch.cuda.synchronize()
    assert cube2.data_ptr() != cube.data_ptr()
    want2 = want * np.asarray([1.0, 0.5, 2.0])[None, :, None, None]
    assert np.abs(cube2.float().cpu().numpy() - want2).max() <= 2 * tol
    # the compact path wants the time-minor compact layout, as the reference checks
    with pytest.raises(ValueError):
        im.process_cube(streams_cint8=streams, time_shifts_gpu=torch.from_numpy(shifts).to(dev),
                        compact_inv_lut=torch.zeros(1, device=dev))
