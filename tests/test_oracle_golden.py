"""Pin the CPU oracle against fixtures produced by the reference itself.

Each test regenerates the seeded input (numpy PCG64) that
``tests/golden/make_golden.py`` fed to dsa110-rt, runs the oracle and
compares with the stored reference outputs — bit-exact for integer/index
work, float tolerance only where the reference's own arithmetic is
float32 torch (static-sky mean, dirty image, clipped std).
"""

import hashlib
import os
import sys

import numpy as np

import dsb_oracle as O

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden as MG  # noqa: E402


def _load(golden_dir, name):
    return np.load(os.path.join(golden_dir, name), allow_pickle=False)


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_unpack_full_block_matches_reference(golden_dir):
    z = _load(golden_dir, "unpack.npz")
    raw = MG.unpack_raw(int(z["seed"]))
    re, im = O.unpack_int4_gemm_layout(raw, 2048, 96, 384)
    assert tuple(re.shape) == tuple(z["shape"])
    assert _sha(re) == str(z["sha_re"])
    assert _sha(im) == str(z["sha_im"])
    np.testing.assert_array_equal(re.reshape(-1)[z["idx"]], z["re_s"])
    np.testing.assert_array_equal(im.reshape(-1)[z["idx"]], z["im_s"])


def test_corr_stokes_i_chansum_matches_reference(golden_dir):
    z = _load(golden_dir, "corr.npz")
    npkt, nant, nchan = int(z["si_npkt"]), int(z["si_nant"]), int(z["si_nchan"])
    raw = MG.corr_raw(npkt, nant, nchan)
    vr, vi = O.corr_fast_from_raw(raw, npkt=npkt, nant=nant, nchan=nchan,
                                  t_int=int(z["si_t_int"]), csf=int(z["si_csf"]))
    np.testing.assert_array_equal(vr, z["si_re"].astype(np.int64))
    np.testing.assert_array_equal(vi, z["si_im"].astype(np.int64))


def test_corr_two_pol_matches_reference(golden_dir):
    z = _load(golden_dir, "corr.npz")
    npkt, nant, nchan = int(z["p2_npkt"]), int(z["p2_nant"]), int(z["p2_nchan"])
    raw = MG.corr_raw(npkt, nant, nchan, seed=MG.CORR_SEED + 1)
    re, im = O.unpack_int4_gemm_layout(raw, npkt, nant, nchan)
    vr, vi = O.corr_fast(re, im, t_int=int(z["p2_t_int"]), fuse_stokes_i=False)
    np.testing.assert_array_equal(vr, z["p2_re"].astype(np.int64))
    np.testing.assert_array_equal(vi, z["p2_im"].astype(np.int64))


def test_pattern_cells_and_gridder_match_reference(golden_dir):
    z = _load(golden_dir, "grid_plan.npz")
    e, n = z["antpos_e"], z["antpos_n"]
    n_grid, csf = int(z["n_grid"]), int(z["csf"])
    cell = O.top_of_band_cell_lambda(e, n, O.REFERENCE_BAND, n_grid)
    assert cell == float(z["cell_lambda"])
    for g in (0, 15):
        r, c = O.build_pattern(e, n, O.REFERENCE_BAND, g, n_grid=n_grid, csf=csf,
                               cell_lambda=cell)
        np.testing.assert_array_equal(r, z[f"ix_row_{g}"])
        np.testing.assert_array_equal(c, z[f"ix_col_{g}"])
        cim = O.cell_index_map(e, n, O.REFERENCE_BAND, g, n_grid=n_grid, csf=csf,
                               cell_lambda=cell, ix_row_pat=r, ix_col_pat=c)
        np.testing.assert_array_equal(cim, z[f"cim_{g}"].astype(np.int64))
        w = np.bincount(cim[cim < r.size], minlength=r.size).astype(np.float32)
        np.testing.assert_array_equal(w, z[f"cellw_{g}"])
        if g == 15:
            vis = MG.stage1_vis(2, 4656, 384 // csf, seed=int(z["grid_in_seed"]))
            gv = O.grid_vis(vis.astype(np.complex128), cim, r.size)
            np.testing.assert_array_equal(gv.astype(np.complex64), z["grid_out"])


def test_dm_plan_delays_match_reference(golden_dir):
    z = _load(golden_dir, "grid_plan.npz")
    nat = O.delay_native_table(z["plan_coarse"], O.REFERENCE_BAND.summed_freq_table(8))
    np.testing.assert_array_equal(nat, z["plan_nat"])
    bins = O.delay_bins(nat, 8 * 32.768)
    np.testing.assert_array_equal(bins, z["plan_bins"])
    # Convention A: zero at each chgroup's top channel, monotone down the band
    assert np.all(bins[:, 0, :] == 0)
    assert np.all(np.diff(bins, axis=1) >= 0)


def test_stage2_shifts_match_reference(golden_dir):
    z = _load(golden_dir, "grid_plan.npz")
    got = np.stack([O.stage2_shifts(O.REFERENCE_BAND, g, z["s2_coarse"], 262.144)
                    for g in range(16)])
    np.testing.assert_array_equal(got, z["s2_shifts"])


def test_fine_shift_tables_match_reference(golden_dir):
    z = _load(golden_dir, "grid_plan.npz")
    args = (O.REFERENCE_BAND, z["fs_coarse"], z["fs_fine"], z["fs_f2c"], float(z["fs_t_int"]))
    np.testing.assert_array_equal(O.time_shift_search(*args, merge_coarse_rounding=True),
                                  z["fs_merged"])
    np.testing.assert_array_equal(O.time_shift_search(*args, merge_coarse_rounding=False),
                                  z["fs_plain"])


def _stage1_setup(z):
    gz = None
    e, n = MG.t_layout_antpos(96, seed=11)
    n_grid, csf, g = int(z["n_grid"]), int(z["csf"]), int(z["chgroup"])
    cell = O.top_of_band_cell_lambda(e, n, O.REFERENCE_BAND, n_grid)
    r, c = O.build_pattern(e, n, O.REFERENCE_BAND, g, n_grid=n_grid, csf=csf, cell_lambda=cell)
    cim = O.cell_index_map(e, n, O.REFERENCE_BAND, g, n_grid=n_grid, csf=csf,
                           cell_lambda=cell, ix_row_pat=r, ix_col_pat=c)
    coarse = np.linspace(0.0, float(z["dm_max"]), int(z["n_coarse"]))
    bins = O.stage1_bin_shifts(O.REFERENCE_BAND, coarse, csf, 8 * 32.768)[g]
    return cim, r.size, bins


def test_stage1_sliding_window_matches_reference(golden_dir):
    z = _load(golden_dir, "stage1.npz")
    cim, n_filled, bins = _stage1_setup(z)
    np.testing.assert_array_equal(bins, z["bins"])
    win = O.Stage1Window(bins, cim, n_filled, depth=1)
    n_fv = int(z["n_fv"])
    for blk in range(3):
        vis = MG.stage1_vis(n_fv, 4656, 48, seed=int(z["seed"]) + blk)
        out = _stage1_exact(win, vis)
        assert tuple(out[0].shape) == tuple(z[f"b{blk}_shape"])
        np.testing.assert_array_equal(out[0].sum(axis=1), z[f"b{blk}_sum_t_re"])
        np.testing.assert_array_equal(out[1].sum(axis=1), z[f"b{blk}_sum_t_im"])
        np.testing.assert_array_equal(out[0].sum(axis=2), z[f"b{blk}_sum_c_re"])
        np.testing.assert_array_equal(out[1].sum(axis=2), z[f"b{blk}_sum_c_im"])
        idx = z[f"b{blk}_idx"]
        np.testing.assert_array_equal(out[0].reshape(-1)[idx], z[f"b{blk}_re_s"].astype(np.int64))
        np.testing.assert_array_equal(out[1].reshape(-1)[idx], z[f"b{blk}_im_s"].astype(np.int64))


def _stage1_exact(win, vis):
    """Push integer real and imaginary planes through one window state."""
    if not hasattr(win, "_pair"):
        win._pair = (O.Stage1Window(win.shifts, win.cim, win.n_filled, win.depth),
                     O.Stage1Window(win.shifts, win.cim, win.n_filled, win.depth))
    a = win._pair[0].push(np.rint(vis.real).astype(np.int64))
    b = win._pair[1].push(np.rint(vis.imag).astype(np.int64))
    return a, b


def test_stage1_single_window_matches_reference(golden_dir):
    z = _load(golden_dir, "stage1.npz")
    cim, n_filled, bins = _stage1_setup(z)
    n_fv = int(z["n_fv"])
    vis = MG.stage1_vis(n_fv, 4656, 48, seed=int(z["seed"]) + 9)
    t_d = n_fv - int(bins.max())
    o_re = O.stage1_dedisp(np.rint(vis.real).astype(np.int64), bins, cim, n_filled, t_d)
    o_im = O.stage1_dedisp(np.rint(vis.imag).astype(np.int64), bins, cim, n_filled, t_d)
    assert tuple(o_re.shape) == tuple(z["ns_shape"])
    np.testing.assert_array_equal(o_re.sum(axis=1), z["ns_sum_t_re"])
    np.testing.assert_array_equal(o_im.sum(axis=2), z["ns_sum_c_im"])


def test_static_sky_matches_reference(golden_dir):
    z = _load(golden_dir, "fifo_sky.npz")
    sky = O.StaticSkyMean(window_blocks=3, warmup_cubes=2, n_dm=2)
    for i, (x, ref) in enumerate(zip(z["sky_in"], z["sky_out"])):
        got = sky.apply(x, dm_slot=i % 2)
        np.testing.assert_allclose(got, ref, rtol=0, atol=2e-6 * max(1.0, np.abs(ref).max()))


def test_stage2_interchgroup_fifo_matches_reference(golden_dir):
    z = _load(golden_dir, "fifo_sky.npz")
    f = O.Stage2InterChgroupShiftFifo(z["ics_shifts"], 16)
    for x, ref, n in zip(z["ics_in"], z["ics_out"], z["ics_emitted"]):
        r = f.push(x)
        assert len(r) == int(n)
        if r:
            np.testing.assert_array_equal(r[0], ref)


def test_per_coarse_dm_fifo_matches_reference(golden_dir):
    z = _load(golden_dir, "fifo_sky.npz")
    pf = O.PerCoarseDmStage2FIFO([0, 1, 3])
    seq = []
    for i in range(6):
        for c in range(3):
            r = pf.push(c, 10 * i + c)
            seq.append(-1 if r is None else int(r))
    np.testing.assert_array_equal(np.asarray(seq), z["pdf_seq"])


def test_combine_matches_reference(golden_dir):
    z = _load(golden_dir, "image_detector.npz")
    got = O.combine_full(z["cmb_streams"], z["cmb_shifts"], t_det=9, t_lo=2, fftshift=False)
    np.testing.assert_array_equal(got.astype(np.complex64), z["cmb_out"])


def test_half_spectrum_identity():
    """``irfft2(G_h) == Re(ifft2(G))`` with the folded checkerboard
    (fused_combine_cuda.py:560-620)."""
    rng = np.random.default_rng(5)
    N = 16
    streams = (rng.normal(size=(3, 6, N, N)) + 1j * rng.normal(size=(3, 6, N, N)))
    shifts = np.asarray([0, 2, -1])
    full = O.combine_full(streams, shifts, 6, 0, fftshift=False)
    want = O.dirty_image(full)
    half = O.combine_half(streams, shifts, 6, 0, fftshift=True)
    got = O.image_from_half(half, N)
    np.testing.assert_allclose(got, want, atol=1e-12)


def test_dirty_image_and_mask_match_reference(golden_dir):
    z = _load(golden_dir, "image_detector.npz")
    img = O.dirty_image(z["img_uv"].astype(np.complex128))
    np.testing.assert_allclose(img, z["img_out"], rtol=0, atol=1e-6)
    m = O.edge_mask(32)
    np.testing.assert_array_equal(m, z["img_mask"])


def test_padded_cumsum_and_boxcars_match_reference(golden_dir):
    z = _load(golden_dir, "image_detector.npz")
    cs = O.padded_cumsum(z["bc_cube"], 16)
    np.testing.assert_array_equal(cs, z["bc_cs"])
    offs = O.boxcar_offsets([1, 2, 4, 8, 16], 16)
    for k, w in enumerate([1, 2, 4, 8, 16]):
        t = np.arange(24) + 8
        got = cs[t + offs[k] + w] - cs[t + offs[k]]
        np.testing.assert_array_equal(got, z["bc_box"][k])


def test_decode_matches_reference(golden_dir):
    z = _load(golden_dir, "image_detector.npz")
    c = O.decode_topk(z["dec_score"], z["dec_winner"], threshold=3.5, n_top=64,
                      r_t=4, r_f=5, r_lm=3)
    widths = [1, 2, 4, 8, 16]
    got = np.asarray([[x.t, x.f, x.l, x.m, widths[x.k], x.snr] for x in c], np.float64)
    np.testing.assert_array_equal(got, z["dec_out"].astype(np.float64))


def test_layer1_clipped_std_matches_reference(golden_dir):
    z = _load(golden_dir, "image_detector.npz")
    got = O.sigma_clipped_std_batched(z["l1_in"])
    np.testing.assert_allclose(got, z["l1_out"], rtol=2e-6)
