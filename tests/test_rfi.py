"""RFI excision hook (services/corr_fast_integration.py:1249-1370).

* CPU: the oracle's zero-fill of the raw page, unpacked, equals the
  reference's ``apply_rfi_mask_to_voltages`` on its unpacked voltages (both
  masks, a full 2048-packet page), by content hash.
* GPU: ``dsb_rfi_zero_fill`` equals the oracle byte for byte; the pipeline
  correlates a zero-filled block exactly as the oracle correlates the
  oracle's zero-filled block.
"""

import os
import sys

import numpy as np
import pytest
import torch

import dsb_oracle as O

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden as MG  # noqa: E402


def test_oracle_zero_fill_matches_reference(golden_dir):
    z = np.load(os.path.join(golden_dir, "rfi.npz"))
    m, tm = MG.rfi_masks()
    page = MG.unpack_raw().reshape(2048, 96, 384, 2, 2)
    re, im = O.unpack_int4_gemm_layout(O.rfi_zero_fill_raw(page, m, tm), 2048, 96, 384)
    assert MG.sha(re) == str(z["sha_re"]) and MG.sha(im) == str(z["sha_im"])
    assert [(re == 0).sum(), (im == 0).sum()] == z["zeros"].tolist()


@pytest.mark.gpu
def test_rfi_zero_fill_gpu_matches_oracle():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dsb200.corr import apply_rfi_mask_to_raw
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(8)
    G, npkt, nant, nchan, n_acc = 3, 64, 16, 40, 8
    raw = rng.integers(0, 256, (G, npkt, nant, nchan, 2, 2), dtype=np.uint8)
    m = rng.random((G, nant, nchan, 2)) < 0.05
    tm = rng.random((G, n_acc, nchan, 2)) < 0.05
    for use_m, use_t in ((True, False), (False, True), (True, True)):
        d = torch.from_numpy(raw).to(dev)
        apply_rfi_mask_to_raw(d, torch.from_numpy(m).to(dev) if use_m else None,
                              time_chan_mask=torch.from_numpy(tm).to(dev) if use_t else None)
        want = np.stack([O.rfi_zero_fill_raw(raw[g], m[g] if use_m else None,
                                             tm[g] if use_t else None) for g in range(G)])
        np.testing.assert_array_equal(d.cpu().numpy(), want)
    # one page without a page axis, and the reference's errors
    d = torch.from_numpy(raw[0]).to(dev)
    apply_rfi_mask_to_raw(d, torch.from_numpy(m[0]).to(dev))
    np.testing.assert_array_equal(d.cpu().numpy(), O.rfi_zero_fill_raw(raw[0], m[0]))
    with pytest.raises(TypeError):
        apply_rfi_mask_to_raw(d, torch.zeros((nant, nchan, 2), dtype=torch.uint8, device=dev))
    with pytest.raises(ValueError):
        apply_rfi_mask_to_raw(d, torch.zeros((nant, nchan + 1, 2), dtype=torch.bool, device=dev))
    with pytest.raises(ValueError):
        apply_rfi_mask_to_raw(d, time_chan_mask=torch.zeros((7, nchan, 2), dtype=torch.bool,
                                                            device=dev))


@pytest.mark.gpu
def test_zero_filled_block_correlates_as_oracle():
    """The correlator on a zero-filled block equals the oracle correlator on
    the oracle's zero-filled block, bit for bit: flagged samples add
    nothing to any baseline."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dsb200.corr import FastCorrKernel, apply_rfi_mask_to_raw, unpack_int4_split
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(21)
    npkt, nant, nchan, t_int = 16, 24, 8, 8
    raw = rng.integers(0, 256, (npkt, nant, nchan, 2, 2), dtype=np.uint8)
    m = rng.random((nant, nchan, 2)) < 0.1
    tm = rng.random((2, nchan, 2)) < 0.1
    d = torch.from_numpy(raw).to(dev)
    apply_rfi_mask_to_raw(d, torch.from_numpy(m).to(dev),
                          time_chan_mask=torch.from_numpy(tm).to(dev))
    re, im = unpack_int4_split(d.reshape(-1), device=dev, out_dtype=torch.int8, npkt=npkt,
                               nant=nant, nchan=nchan)
    k = FastCorrKernel(dev, t_int_fast_native=t_int, nants=nant, nchan=nchan)
    vis = k.compute_split(re, im, fuse_stokes_i=True, chan_sum_factor=1).cpu().numpy()
    zf = O.rfi_zero_fill_raw(raw, m, tm)
    ore, oim = O.unpack_int4_gemm_layout(zf, npkt, nant, nchan)
    vr, vi = O.corr_fast(ore, oim, t_int=t_int, csf=1, fuse_stokes_i=True)
    np.testing.assert_array_equal(vis.real.astype(np.int64), vr)
    np.testing.assert_array_equal(vis.imag.astype(np.int64), vi)
    # and the flags changed the visibilities
    ure, uim = O.unpack_int4_gemm_layout(raw, npkt, nant, nchan)
    ur, _ = O.corr_fast(ure, uim, t_int=t_int, csf=1, fuse_stokes_i=True)
    assert not np.array_equal(ur, vr)
